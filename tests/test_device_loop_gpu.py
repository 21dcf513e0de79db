"""GPU tests of the device-resident outer loop of BACKWARD_SOLVER_MULTI:

  * a potential built on the GPU from a device RI (set_RI_device,
    odt_potential_eps_device + odt_set_potential_device) against the
    host-built one (set_RI): the same eps_imag to 2 ulp, the same Bornmax,
    and solves / gradients within rel-L2 1e-6 (1e-5 for the reflected
    field, a signal about 100 times weaker than the transmitted one): the
    complex square roots of the RI2potential / potential2RI round trips are
    the device's, so the potentials agree to a few ulp, not bit for bit;
  * the device-resident FISTA loop against the host-array loop: three outer
    iterations, real (kappamax = 0) and complex (kappamax > 0) TV prox,
    rel-L2 <= 1e-5 on RI - RI_bg and the misfits within 1e-5.
"""
import numpy as np
import pytest

import cases
from oracle import cbs

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel(order="F"))).cuda()


@pytest.mark.parametrize("cplx", [False, True])
def test_set_RI_device_matches_host(cplx):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN

    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    if cplx:
        RI = (RI + 1j * 0.004 * (RI - cases.NM) / max(1e-6, float(np.max(RI - cases.NM)))).astype(np.complex64)
    fields = cases.circle_fields(p, 2)
    a = FORWARD_SOLVER_CONVERGENT_BORN(p)
    a.set_RI(RI)
    eps_h, bm_h = float(a.eps_imag), a.Bornmax
    t1, r1, f1 = a.solve(fields)
    b = FORWARD_SOLVER_CONVERGENT_BORN(p)
    b.set_RI_device(_dev(RI))
    eps_d, bm_d = float(b.eps_imag), b.Bornmax
    t2, r2, f2 = b.solve(fields)
    assert abs(eps_d - eps_h) <= 2 * np.spacing(np.float32(eps_h))
    assert bm_d == bm_h
    assert cbs.rel_l2(t1, t2) < 1e-6 and cbs.rel_l2(f1, f2) < 1e-6
    assert cbs.rel_l2(r1, r2) < 1e-5

    # adjoint slot: the gradient from device-built forward + adjoint potentials
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fields)
    RI0 = (np.real(RI) * 0.7 + cases.NM * 0.3).astype(np.float32)
    a.set_RI(RI0)
    a.set_RI_adjoint(RI0)
    g1, e1 = a.gradient(fields, meas)
    b.set_RI_device(_dev(RI0))
    b.set_RI_device(_dev(RI0), adjoint=True)
    g2 = _dev(np.zeros(g1.shape, np.complex64))
    e2 = b.gradient_device(_dev(fields[:, :, 0, :]), _dev(meas[:, :, 0, :]), g2)
    g2 = g2.cpu().numpy().reshape(g1.shape, order="F")
    assert cbs.rel_l2(g1, g2) < 1e-6
    assert abs(e1 - e2) / e1 < 1e-6
    a.delete()
    b.delete()


@pytest.mark.parametrize("kappamax", [0.0, 0.01])
def test_device_loop_matches_host_loop(kappamax):
    from inverse_solver_b200 import FORWARD_SOLVER_CONVERGENT_BORN
    from inverse_solver_b200.backward import BACKWARD_SOLVER_MULTI

    p = cases.small_params(return_transmission=True, return_reflection=True, return_3D=True)
    RI = cases.small_RI()
    fields = cases.circle_fields(p, 3)
    o = cbs.ForwardSolverCBS(p, single=True)
    o.set_RI(RI)
    meas, _, _ = o.solve(fields)

    class Blurred:
        def solve(self, input_field, output_field):
            return (RI * 0.5 + cases.NM * 0.5).astype(np.float32)

    def run(device_loop):
        bp = BACKWARD_SOLVER_MULTI.get_default_parameters(dict(
            RI_bg=cases.NM, wavelength=cases.LAM, NA=p["NA"], resolution=p["resolution"],
            size=p["size"], forward_solver=FORWARD_SOLVER_CONVERGENT_BORN,
            forward_solver_parameters=p, init_solver=Blurred(), step=0.01, tv_param=0.001,
            inner_itt=20, itter_max=3, use_non_negativity=True, nmin=cases.NM, nmax=1.5,
            kappamax=kappamax, device_loop=device_loop))
        b = BACKWARD_SOLVER_MULTI(bp)
        out = b.solve(fields, meas)
        errs = list(b.err_list)
        b.delete()
        return out, errs

    dev, edev = run(True)
    host, ehost = run(False)
    assert dev.shape == host.shape and dev.dtype == np.complex64
    assert cbs.rel_l2(dev - cases.NM, host - cases.NM) < 1e-5
    assert np.allclose(edev, ehost, rtol=1e-5)
    assert edev[-1] < edev[0]
