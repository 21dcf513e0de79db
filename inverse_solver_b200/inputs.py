"""Input generators: phantoms and plane-wave illuminations.

PHANTOM and FIELD_GENERATOR mirror Codes/PHANTOM.m and Codes/FIELD_GENERATOR.m
(bead phantom, 'random' / 'circle' illumination styles).  The reference's
'random' style draws from MATLAB's unseeded ``rand``; here every random draw
comes from a seeded ``numpy.random.Generator``.  ``sphere_phantom`` and
``ring_illumination`` build the seeded multi-sphere phantoms and ring
illumination patterns used for the multi-illumination workloads (they are not
reference styles).
"""
from __future__ import annotations

import math

import numpy as np

from .optics import C64, F32, OpticalTool, basic_optical_parameter, centered_fft2, update_struct

_AA_SHIFTS = [(1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1),
              (1, 1, -1), (-1, 1, -1), (1, -1, -1), (-1, -1, -1)]


class PHANTOM:
    @staticmethod
    def get_default_parameters():
        """PHANTOM.m:3-9."""
        return {"name": "blank", "antialiasing": True, "outer_size": [100, 100, 100],
                "inner_size": [50, 50, 50], "rotation_angles": [0, 0, 0]}

    @staticmethod
    def get(params):
        """PHANTOM.m:10-98 for 'blank' and 'bead' (8-sample antialiasing,
        normalised to [0, 1])."""
        outer = [int(s) for s in params["outer_size"]]
        inner = [float(s) for s in params["inner_size"]]
        if any(abs(a) > 0 for a in params.get("rotation_angles", [0, 0, 0])):
            raise NotImplementedError("rotated phantoms are not supported")
        d = [np.arange(1, n + 1, dtype=F32) - F32(n // 2 + 1) for n in outer]
        ph = np.zeros(outer, dtype=F32)
        shifts = _AA_SHIFTS if params.get("antialiasing", True) else [(0, 0, 0)]
        scale = 0.25 if params.get("antialiasing", True) else 0.0
        for sh in shifts:
            n = [2 * (d[i] + F32(scale * sh[i])) / F32(inner[i]) for i in range(3)]
            r = np.sqrt(n[0][:, None, None] ** 2 + n[1][None, :, None] ** 2 + n[2][None, None, :] ** 2)
            if params["name"] == "bead":
                ph = ph + (r < 1).astype(F32)
            elif params["name"] != "blank":
                raise NotImplementedError("phantom '%s' is not supported" % params["name"])
        ph = ph - ph.min()
        if ph.max() != 0:
            ph = ph / ph.max()
        return ph


def bead_RI(size, diameter_px, n_bg, n_sp):
    """RI map of one antialiased bead (SIMULATION_BEAD.m:25-30, :55-56)."""
    p = PHANTOM.get_default_parameters()
    p.update(name="bead", outer_size=list(size), inner_size=[diameter_px] * 3)
    return (n_bg + PHANTOM.get(p) * (n_sp - n_bg)).astype(F32)


def sphere_phantom(size, resolution, n_bg, seed, n_spheres=None, radius_um=(0.5, 3.0),
                   ri_range=(1.34, 1.46)):
    """Seeded multi-sphere RI map: 1-20 spheres (or ``n_spheres``), radius
    uniform in ``radius_um``, RI uniform in ``ri_range``, centres uniform such
    that each sphere fits inside the grid, painted in order with the 8-sample
    antialiasing of PHANTOM.m (a later sphere overwrites the covered fraction
    of earlier ones)."""
    rng = np.random.default_rng(seed)
    size = [int(s) for s in size]
    res = [float(r) for r in resolution]
    if n_spheres is None:
        n_spheres = int(rng.integers(1, 21))
    RI = np.full(size, n_bg, dtype=np.float64)
    ext = [size[i] * res[i] for i in range(3)]
    coords = [(np.arange(size[i]) + 0.5) * res[i] for i in range(3)]
    for _ in range(n_spheres):
        rmax = min(radius_um[1], 0.5 * min(ext) * 0.999)
        r = float(rng.uniform(radius_um[0], max(radius_um[0], rmax)))
        c = [float(rng.uniform(r, ext[i] - r)) for i in range(3)]
        n_s = float(rng.uniform(*ri_range))
        lo = [max(0, int(math.floor((c[i] - r) / res[i])) - 1) for i in range(3)]
        hi = [min(size[i], int(math.ceil((c[i] + r) / res[i])) + 1) for i in range(3)]
        cov = np.zeros([hi[i] - lo[i] for i in range(3)])
        for sh in _AA_SHIFTS:
            q = [coords[i][lo[i]:hi[i]] + 0.25 * sh[i] * res[i] - c[i] for i in range(3)]
            cov += (q[0][:, None, None] ** 2 + q[1][None, :, None] ** 2 + q[2][None, None, :] ** 2) < r * r
        cov /= len(_AA_SHIFTS)
        sub = RI[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        RI[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = sub * (1 - cov) + n_s * cov
    return RI.astype(F32)


class FIELD_GENERATOR:
    @staticmethod
    def get_default_parameters(init_params=None):
        """FIELD_GENERATOR.m:6-20 (+ ``seed`` for the 'random' style)."""
        p = basic_optical_parameter()
        p.update(percentage_NA_usage=0.95, illumination_style="random", illumination_number=10,
                 illumination_pol=[], start_with_normal=True, seed=0)
        return update_struct(p, init_params) if init_params else p

    def __init__(self, params):
        self.parameters = params

    def get_fields(self):
        """FIELD_GENERATOR.m:25-72: k-space deltas rounded to the grid, then
        fftshift(fft2(ifftshift())).  Output [size(1), size(2), npol, n]."""
        p = self.parameters
        npol = 2 if p["vector_simulation"] else 1
        n = int(p["illumination_number"])
        out = np.zeros((p["size"][0], p["size"][1], npol, n), dtype=C64)
        u = OpticalTool(p)
        rng = np.random.default_rng(p.get("seed", 0))
        for ill in range(1, n + 1):
            d1 = d2 = 1.0
            if p["illumination_style"] == "random":
                while math.sqrt(d1 ** 2 + d2 ** 2) > 1:
                    d1 = 2 * (rng.random() - 0.5)
                    d2 = 2 * (rng.random() - 0.5)
            elif p["illumination_style"] == "circle":
                div = 1 / n if not p["start_with_normal"] else 1 / max(1, n - 1)
                d1 = math.sin((ill - 1) * 2 * math.pi * div)
                d2 = math.cos((ill - 1) * 2 * math.pi * div)
            else:
                raise ValueError("Unknown illumination style name")
            if ill == 1 and p["start_with_normal"]:
                d1 = d2 = 0.0
            i1 = out.shape[0] // 2 + _mround(d1 * p["percentage_NA_usage"] * u.kmax / u.fourier_res[0])
            i2 = out.shape[1] // 2 + _mround(d2 * p["percentage_NA_usage"] * u.kmax / u.fourier_res[1])
            out[i1, i2, 0, ill - 1] = 1
        return centered_fft2(out).astype(C64)


def _mround(x):
    return int(math.copysign(math.floor(abs(x) + 0.5), x))


def ring_illumination(params, rings=((0.3, 8), (0.6, 16), (0.9, 24))):
    """Normal incidence plus plane waves on concentric rings of illumination
    NA (``rings`` = ((NA, count), ...)), each rounded to the k-grid pixel the
    way FIELD_GENERATOR.m:62-65 rounds, returned as spatial fields
    [size(1), size(2), 1, 1 + sum(count)]."""
    u = OpticalTool(params)
    kdirs = [(0.0, 0.0)]
    for na, cnt in rings:
        for j in range(cnt):
            phi = 2 * math.pi * j / cnt
            kdirs.append((na / params["wavelength"] * math.sin(phi),
                          na / params["wavelength"] * math.cos(phi)))
    out = np.zeros((params["size"][0], params["size"][1], 1, len(kdirs)), dtype=C64)
    for i, (k1, k2) in enumerate(kdirs):
        i1 = out.shape[0] // 2 + _mround(k1 / u.fourier_res[0])
        i2 = out.shape[1] // 2 + _mround(k2 / u.fourier_res[1])
        out[i1, i2, 0, i] = 1
    return centered_fft2(out).astype(C64)
