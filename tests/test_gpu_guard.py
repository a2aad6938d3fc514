"""The FP32 real-time norm guard: every period (1, 2, 4 steps) and any call
length keep the norm and stay within FP32 round-off of the FP64 form; the
guard factor left by the last step is applied before the call returns."""

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu


def case():
    return dict(cases.DEFAULTS, dim=2, n=128, box=8.0, g=300.0, omega=0.6, gauge=True,
                dt=5e-5, seed=1201, init="phase")


@pytest.mark.parametrize("period", [1, 2, 4])
@pytest.mark.parametrize("steps", [7, 8, 9, 10])
def test_guard_periods_keep_the_norm(period, steps):
    import gpue_b200 as G
    c = case()
    psi0 = cases.initial_psi(c)
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        s.set_wfc(psi0)
        s.evolve(steps, 1)
        ref = s.get_wfc()
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(psi0)
        n0 = s.norm()
        r = s.evolve(steps, 1, norm_guard_period=period)
        psi = s.get_wfc()
        n1 = s.norm()
    assert r["steps_done"] == steps
    assert abs(n1 - n0) <= 1e-6 * n0
    assert float(np.sqrt(np.sum(np.abs(psi - ref) ** 2) * dV(c))) <= 2e-6


def test_sliced_calls_match_one_call_within_round_off():
    """A run sliced at odd step counts (each call starts its own guard) stays
    within FP32 round-off of one call."""
    import gpue_b200 as G
    c = case()
    psi0 = cases.initial_psi(c)
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(psi0)
        s.evolve(60, 1)
        one = s.get_wfc()
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(psi0)
        done = 0
        for n in (7, 13, 21, 19):
            s.evolve(n, 1, step_offset=done)
            done += n
        sliced = s.get_wfc()
    assert float(np.sqrt(np.sum(np.abs(one - sliced) ** 2) * dV(c))) <= 1e-5


def test_invalid_period_is_rejected():
    import gpue_b200 as G
    c = case()
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(cases.initial_psi(c))
        with pytest.raises(G.GpueError):
            s.evolve(2, 1, norm_guard_period=3)
