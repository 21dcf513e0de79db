"""Oracle: CPU restatement of BACKWARD_SOLVER_MULTI and TV_FISTA_inner_v2.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py); parity unpinned -- the
reference is MATLAB and ships no outputs.  Single (MATLAB single) or double
precision through ``cbs.Prec``; the FISTA / TV momentum scalars are double in
both, as in MATLAB (they are double scalars there).
"""
from __future__ import annotations

import math

import numpy as np

from . import cbs


# ------------------------------------------------------------- TV prox
def _tv_L(P):
    """TV_L (sub_code/TV_FISTA_inner_v2.m:99-113): P1+P2+P3 minus the
    periodic backward shifts."""
    out = P[0] + P[1]
    if len(P) == 3:
        out = out + P[2]
        out = out - np.roll(P[0], 1, axis=0)
        out = out - np.roll(P[1], 1, axis=1)
        out = out - np.roll(P[2], 1, axis=2)
    else:
        out = out - np.roll(P[0], 1, axis=0)
        out = out - np.roll(P[1], 1, axis=1)
    return out


def _tv_L_trans(x):
    """TV_L_trans (:114-123): forward differences x - x(+1), periodic."""
    return [x - np.roll(x, -1, axis=k) for k in range(x.ndim)]


def _project_non_neg(x, Vmin, Vmax, Vimag_max, non_neg, dirichlet):
    """project_non_neg (:57-75)."""
    x = x.copy()
    if non_neg:
        if np.iscomplexobj(x):
            m = x.real < Vmin
            x[m] = Vmin + 1j * x.imag[m]
            m = x.real > Vmax
            x[m] = Vmax + 1j * x.imag[m]
        else:
            x[x < Vmin] = Vmin
            x[x > Vmax] = Vmax
    if np.iscomplexobj(x):
        m = x.imag < 0
        x[m] = x.real[m]
        if Vimag_max > 0:
            m = x.imag > Vimag_max
            x[m] = x.real[m] + 1j * Vimag_max
    if dirichlet:
        x[0, :, :] = 0
        x[-1, :, :] = 0
        x[:, 0, :] = 0
        x[:, -1, :] = 0
        x[:, :, 0] = 0
        x[:, :, -1] = 0
    return x


def _project_TV(P):
    """project_TV (:77-88)."""
    if len(P) == 3:
        A = np.sqrt(np.maximum(np.abs(P[0]) ** 2 + np.abs(P[1]) ** 2 + np.abs(P[2]) ** 2, 1))
    else:
        A = np.sqrt(np.maximum(np.abs(P[0]) ** 2 + np.abs(P[1]) ** 2, 1))
    return [p / A for p in P]


def tv_fista_inner_v2(in_mat, lam, Vmin, Vmax, Vimag_max, non_neg, dirichlet, inner_itt, P):
    """TV_FISTA_inner_v2 (sub_code/TV_FISTA_inner_v2.m:1-53): isotropic-TV
    proximal operator by dual FISTA (Beck & Teboulle)."""
    x = P.S(np.asarray(in_mat))
    if Vimag_max == 0:
        x = np.real(x).astype(P.r)
    ndim = x.ndim
    dividend = 12 if ndim >= 3 else 8
    Pnp = [0 * x for _ in range(ndim if ndim in (2, 3) else 2)]
    R = [p.copy() for p in Pnp]
    t_np = 1.0
    for _ in range(inner_itt):
        Pn = Pnp
        t_n = t_np
        Pnp = _tv_L_trans(_project_non_neg(x - lam * _tv_L(R), Vmin, Vmax, Vimag_max, non_neg, dirichlet))
        Pnp = [R[k] + 1 / (dividend * lam) * Pnp[k] for k in range(len(Pnp))]
        Pnp = _project_TV(Pnp)
        t_np = (1 + math.sqrt(1 + 4 * t_n ** 2)) / 2
        R = [Pnp[k] + ((t_n - 1) / t_np) * (Pnp[k] - Pn[k]) for k in range(len(Pnp))]
    return _project_non_neg(x - lam * _tv_L(Pnp), Vmin, Vmax, Vimag_max, non_neg, dirichlet)


# -------------------------------------------------- BACKWARD_SOLVER_MULTI
def multi_default_parameters(init=None):
    """BACKWARD_SOLVER_MULTI.m:9-29 (forward-solver and init-solver objects
    are passed separately)."""
    p = cbs.basic_optical_parameter()
    p.update(step=0.01, tv_param=0.001, use_non_negativity=False, nmin=-math.inf,
             nmax=math.inf, kappamax=0, inner_itt=100, itter_max=100,
             num_scan_per_iteration=0, verbose=False)
    if init is not None:
        p = cbs.update_struct(p, init)
    return p


def get_gradient_static(RI, input_field, output_field, fwd):
    """get_gradiant_static (BACKWARD_SOLVER_MULTI.m:30-54); ``fwd`` is an
    oracle ForwardSolverCBS with return_transmission and return_3D on."""
    P = fwd.P
    fwd.set_RI(RI)
    trans, _, src3d = fwd.solve(input_field)
    diff = trans - P.S(output_field)
    err = float(np.sum(np.abs(diff.astype(np.complex128)) ** 2))
    fwd.set_RI(np.conj(np.flip(RI, axis=2)))
    _, _, d3 = fwd.solve(np.conj(diff))
    d3 = np.flip(np.conj(d3), axis=2)
    grad = -(1j * np.mean(np.conj(src3d) * d3, axis=(3, 4)))
    return P.S(grad), err


def solve_multi(params, init_RI, input_field, output_field, fwd, scan_lists=None):
    """BACKWARD_SOLVER_MULTI.solve (:92-196): FISTA on u = RI^2/n_bg^2 - 1 with
    the TV prox of TV_FISTA_inner_v2.  ``init_RI`` is the init solver's
    output; ``scan_lists[ii]`` (optional) fixes the stochastic subsets."""
    P = fwd.P
    RI = P.S(init_RI).astype(P.c)
    alpha = 1 / params["step"]
    t_np = 1.0
    u_n = RI ** 2 / params["RI_bg"] ** 2 - 1
    x_n = RI ** 2 / params["RI_bg"] ** 2 - 1
    if RI.shape[2] % 2 == 0:
        raise ValueError("need to be odd size")
    nb2 = params["RI_bg"] ** 2
    Vmin = (params["nmin"] ** 2 - params["kappamax"] ** 2) / nb2 - 1
    Vmax = params["nmax"] ** 2 / nb2 - 1
    Vimag_max = 2 * params["kappamax"] * params["nmax"] / nb2
    errs = []
    for ii in range(params["itter_max"]):
        if scan_lists is None:
            sl = np.arange(input_field.shape[3])
        else:
            sl = np.asarray(scan_lists[ii])
        grad, err = get_gradient_static(RI, input_field[:, :, :, sl], output_field[:, :, :, sl], fwd)
        errs.append(err)
        t_n = t_np
        s_n = tv_fista_inner_v2(u_n - (1 / alpha) * grad, params["tv_param"] / alpha, Vmin, Vmax,
                                Vimag_max, params["use_non_negativity"], False,
                                params["inner_itt"], P)
        t_np = (1 + math.sqrt(1 + 4 * t_n ** 2)) / 2
        u_n = s_n + (t_n - 1) / t_np * (s_n - x_n)
        x_n = s_n
        RI = params["RI_bg"] * np.sqrt(P.S(u_n).astype(P.c) + 1)
    return RI, errs
