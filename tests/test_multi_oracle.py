"""CPU checks of the TV-FISTA prox restatement (TV_FISTA_inner_v2.m)."""
import numpy as np

from oracle import cbs, multi


def _tv(x):
    d = [x - np.roll(x, -1, axis=k) for k in range(3)]
    return float(np.sum(np.sqrt(sum(np.abs(q) ** 2 for q in d))))


def test_tv_prox_reduces_tv_and_stays_close():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((12, 10, 9)).astype(np.float32)
    for lam in (1e-3, 1e-1):
        y = multi.tv_fista_inner_v2(x, lam, -np.inf, np.inf, 0, False, False, 60, cbs.Prec(False))
        assert _tv(y) < _tv(x)
        # prox objective 0.5||y-x||^2 + lam TV(y) is below that of x itself
        assert 0.5 * np.sum((y - x) ** 2) + lam * _tv(y) < lam * _tv(x)
    y = multi.tv_fista_inner_v2(x, 1e-6, -np.inf, np.inf, 0, False, False, 20, cbs.Prec(False))
    assert np.abs(y - x).max() < 1e-4


def test_tv_prox_projection_and_precision():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((8, 8, 7)).astype(np.float32)
    y32 = multi.tv_fista_inner_v2(x, 0.05, -0.5, 0.5, 0, True, False, 40, cbs.Prec(True))
    y64 = multi.tv_fista_inner_v2(x, 0.05, -0.5, 0.5, 0, True, False, 40, cbs.Prec(False))
    assert y32.dtype == np.float32 and y32.min() >= -0.5 and y32.max() <= 0.5
    assert cbs.rel_l2(y32, y64) < 1e-5
