"""B200-native convergent-Born-series ODT solver (drop-in for the CBS path of
BMOLKAIST/Inverse_solver).  The per-illumination work runs in libodt.so
(include/odt.h); this package is the host-side mirror of the reference's
MATLAB classes."""
from .forward import CBSHostSetup, FORWARD_SOLVER_CONVERGENT_BORN  # noqa: F401
from .bpm import FORWARD_SOLVER_BPM  # noqa: F401
from ._lib import OdtError  # noqa: F401
