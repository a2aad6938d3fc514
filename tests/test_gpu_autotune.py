"""The autotuner (gpue_autotune): it may change the radix plan and the lines
per CTA of every axis, never the results beyond round-off."""

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu


def case(**kw):
    c = dict(cases.DEFAULTS, init="gauss")
    c.update(kw)
    return c


def run(c, prec, tune, steps=60, gstate=1):
    import gpue_b200 as G
    with G.Solver(product_params(c, prec)) as s:
        plans = s.autotune(force=True) if tune else [s.plan(a) for a in range(c["dim"])]
        s.set_wfc(cases.initial_psi(c))
        s.evolve(steps, gstate)
        return s.get_wfc(), s.energy(), plans


@pytest.mark.parametrize("c", [
    case(dim=3, n=32, box=6.0, wz=2.0, g=50.0, omega=0.4, gauge=True, dt=1e-4, seed=501,
         init="phase"),
    case(dim=2, n=256, box=10.0, g=200.0, omega=0.6, gauge=True, dt=5e-5, seed=502,
         init="phase"),
    case(dim=3, n=64, box=8.0, wz=3.0, g=100.0, dt=1e-4, seed=503),
], ids=["3d32_gauge", "2d256_gauge", "3d64"])
def test_tuned_plans_give_the_same_results_fp64(c):
    import gpue_b200 as G
    psi_d, E_d, plans_d = run(c, G.PREC_FP64, tune=False)
    psi_t, E_t, plans_t = run(c, G.PREC_FP64, tune=True)
    assert all(p["tuned"] == 1 for p in plans_t)
    assert all(p["us"] <= p["default_us"] for p in plans_t)
    assert float(np.sqrt(np.sum(np.abs(psi_d - psi_t) ** 2) * dV(c))) <= 1e-12
    assert abs(E_d - E_t) <= 1e-12 * abs(E_d)


def test_tuned_plans_fp32_within_fp32_round_off():
    import gpue_b200 as G
    c = case(dim=3, n=64, box=8.0, wz=3.0, g=100.0, omega=0.3, gauge=True, dt=1e-4, seed=504,
             init="phase")
    psi_d, E_d, _ = run(c, G.PREC_FP32, tune=False)
    psi_t, E_t, _ = run(c, G.PREC_FP32, tune=True)
    assert float(np.sqrt(np.sum(np.abs(psi_d - psi_t) ** 2) * dV(c))) <= 1e-5
    assert abs(E_d - E_t) <= 1e-6 * abs(E_d)


def test_choices_are_cached_per_shape():
    import gpue_b200 as G
    c = case(dim=2, n=128, box=8.0, g=10.0, seed=505)
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(cases.initial_psi(c))
        first = s.autotune(force=True)
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(cases.initial_psi(c))
        again = s.autotune()  # cached: no timing, same choice
    for a, b in zip(first, again):
        assert (a["ra"], a["rb"], a["rc"], a["threads_per_line"], a["lines_per_cta"]) == \
            (b["ra"], b["rb"], b["rc"], b["threads_per_line"], b["lines_per_cta"])
        assert b["tuned"] == 1
