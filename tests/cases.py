"""Shared small CBS cases for the tests (sizes the oracle finishes in seconds)."""
import numpy as np

from inverse_solver_b200.forward import CBSHostSetup
from inverse_solver_b200.inputs import FIELD_GENERATOR, bead_RI, ring_illumination, sphere_phantom  # noqa: F401

NM = 1.3355
LAM = 0.532


def params(size, bt, res=0.1, NA=1.2, **kw):
    p = CBSHostSetup.get_default_parameters(dict(
        size=list(size), wavelength=LAM, NA=NA, RI_bg=NM, resolution=[res] * 3,
        vector_simulation=False, boundary_thickness=list(bt)))
    p.update(kw)
    return p


def cfg1_params(**kw):
    """64^3 bead, 16-voxel boundary (bt 8.0331 -> 16 px), 0.1 um voxels."""
    return params([64, 64, 64], [8.0331] * 3, **kw)


def cfg1_RI():
    return bead_RI([64, 64, 64], 50, NM, 1.4607)


def normal_field(size, n=1):
    return np.ones((size[0], size[1], 1, n), dtype=np.complex64)


def circle_fields(p, n, seed=0):
    """Normal incidence + plane waves on a circle at 60% of the NA (at 95%,
    the reference default, the rounded k-pixel of a small grid can fall just
    outside the NA circle and the pupil removes the illumination)."""
    fg = FIELD_GENERATOR.get_default_parameters(dict(size=p["size"], wavelength=LAM, NA=p["NA"],
                                                     RI_bg=NM, resolution=p["resolution"],
                                                     vector_simulation=False,
                                                     illumination_style="circle",
                                                     percentage_NA_usage=0.6,
                                                     illumination_number=n, seed=seed))
    f = FIELD_GENERATOR(fg).get_fields()
    return f


# small non-cubic case with odd and prime-factor lengths:
# size [30, 26, 21], bt [2, 3, 1.5] -> bt_px [4, 6, 3] -> padded [38, 38, 27]
SMALL_SIZE = [30, 26, 21]
SMALL_BT = [2, 3, 1.5]


def small_params(**kw):
    return params(SMALL_SIZE, SMALL_BT, **kw)


def small_RI(seed=3):
    return sphere_phantom(SMALL_SIZE, [0.1] * 3, NM, seed=seed, n_spheres=3,
                          radius_um=(0.4, 1.0))


def wrapped_phase(shape, seed, noise=0.6, amp=25.0):
    """Seeded wrapped phase maps [N1, N2, n] (single): a tall Gaussian bump
    (steep enough to wrap many times) at a random centre per slice plus white
    noise of the given standard deviation, wrapped to (-pi, pi]."""
    rng = np.random.default_rng(seed)
    N1, N2, n = shape
    y, x = np.meshgrid(np.linspace(-1, 1, N1), np.linspace(-1, 1, N2), indexing="ij")
    out = np.empty(shape, np.float32)
    for z in range(n):
        c = rng.uniform(-0.5, 0.5, 2)
        phi = amp * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2) / 0.2) + rng.normal(0, noise, (N1, N2))
        out[:, :, z] = np.angle(np.exp(1j * phi)).astype(np.float32)
    return out


def off_axis_holograms(N=128, n=3, seed=0, carrier=(-0.23, -0.27), noise=0.0, phase_amp=2.5):
    """Synthetic off-axis hologram stacks [N, N, n] (single): |R + U|^2 with
    a tilted reference R (carrier in cycles per pixel, placing the sideband
    in the search window of the retrieval) and object waves U: small random
    tilts for the background, the same waves times amp * exp(i phi) (a
    Gaussian phase bump of `phase_amp` rad and a 20 % absorption dip) for the
    sample; scaled to an 8-bit-like range.  Returns (bg, sp, phi)."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    R = np.exp(2j * np.pi * (carrier[0] * y + carrier[1] * x))
    r2 = ((y - N / 2) ** 2 + (x - N / 2) ** 2) / (N / 6) ** 2
    phi = phase_amp * np.exp(-r2)
    amp = 1 - 0.2 * np.exp(-r2)
    bg, sp = [], []
    for _ in range(n):
        t = rng.uniform(-0.02, 0.02, 2)
        U = 0.8 * np.exp(2j * np.pi * (t[0] * y + t[1] * x))
        bg.append(np.abs(R + U) ** 2 * 60 + noise * rng.standard_normal((N, N)))
        sp.append(np.abs(R + U * amp * np.exp(1j * phi)) ** 2 * 60 + noise * rng.standard_normal((N, N)))
    return np.stack(bg, 2).astype(np.float32), np.stack(sp, 2).astype(np.float32), phi
