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


def aberrated_fields(N=96, n=7, seed=0, step=4, res=0.1, NA=1.2, wavelength=0.532, RI_bg=1.3355):
    """Synthetic scalar field pairs [N, N, 1, n] (single complex) for the
    aberration and dirty-field tests: tilted plane waves whose spectra sit
    at k0s = (rows, columns) pixels from the centre (columns stepping by
    `step`, rows random with sub-pixel offsets), with and without an
    object (a phase / absorption bump and a broadband phase screen of
    0.5 rad), each passed through the pupil NA .* exp(1i W)
    (W: defocus, astigmatism and coma over the NA circle).  Returns
    (input_field, output_field, k0s [2, n], optical parameters)."""
    rng = np.random.default_rng(seed)
    params = dict(size=[N, N, 1], resolution=[res, res, res], NA=NA, wavelength=wavelength, RI_bg=RI_bg)
    fr = 1.0 / (res * N)
    idx = np.arange(N) - N // 2
    ky, kx = np.meshgrid(idx * fr, idx * fr, indexing="ij")
    kmax = NA / wavelength
    rho_y, rho_x = ky / kmax, kx / kmax
    rho2 = rho_x ** 2 + rho_y ** 2
    W = 0.5 * rho2 + 1.2 * (rho_x ** 2 - rho_y ** 2) + 0.8 * rho_x * rho2
    pupil = np.where(rho2 < 1, np.exp(1j * W), 0)
    y, x = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    g = np.exp(-(((y - N / 2) ** 2 + (x - N / 2) ** 2) / (N / 7) ** 2))
    # broadband phase screen (white noise smoothed over ~1 pixel): the object
    # spectrum fills the pupil, as a cell or a diffuser does
    screen = np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((N, N)))
                                  * np.exp(-0.5 * (2 * np.pi * np.fft.fftfreq(N)[:, None]) ** 2
                                           - 0.5 * (2 * np.pi * np.fft.fftfreq(N)[None, :]) ** 2)))
    screen *= 0.5 / screen.std()
    obj = (1 - 0.1 * g) * np.exp(1j * (0.6 * g + screen))
    cols = (np.arange(n) - (n - 1) / 2) * step
    k0s = np.stack([rng.integers(-3, 4, n) + rng.uniform(-0.3, 0.3, n), cols + rng.uniform(-0.3, 0.3, n)])

    def c2(a, inverse=False):
        a = np.fft.ifftshift(a)
        return np.fft.fftshift(np.fft.ifft2(a) if inverse else np.fft.fft2(a))

    inp, out = [], []
    for k in range(n):
        wave = np.exp(2j * np.pi * (k0s[0, k] * y + k0s[1, k] * x) / N)
        inp.append(c2(c2(wave) * pupil, inverse=True))
        out.append(c2(c2(wave * obj) * pupil, inverse=True))
    inp = np.stack(inp, 2)[:, :, None, :].astype(np.complex64)
    out = np.stack(out, 2)[:, :, None, :].astype(np.complex64)
    return np.asfortranarray(inp), np.asfortranarray(out), k0s.astype(np.float32), params
