"""The serving loop (gpue_server_*): continuous batching of mixed solves.

A solve served in a mix must give the same result as the same solve served
alone, bit for bit (each solve reduces over its own tiles; its step
numbering starts at 0 whenever it is admitted).  Served solves must also
match gpue_evolve run for the same number of steps, and admission must hold
resident memory within the HBM budget.
"""

import time

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu


def case(**kw):
    c = dict(cases.DEFAULTS, init="gauss")
    c.update(kw)
    return c


PROBE = case(dim=2, n=64, box=8.0, g=200.0, omega=0.4, gauge=True, gdt=5e-3, seed=301)
MIX = [
    (case(dim=2, n=96, box=10.0, g=80.0, gdt=5e-3, seed=302), 0, 1000),
    (case(dim=2, n=64, box=8.0, g=50.0, omega=0.6, gauge=True, dt=5e-5, seed=303,
          init="phase"), 1, 300),
    (case(dim=3, n=16, box=6.0, wz=2.0, g=50.0, gdt=5e-3, seed=304), 0, 500),
    (case(dim=2, n=128, box=10.0, g=300.0, wy=1.2, gdt=5e-3, seed=305), 0, 1000),
    (case(dim=3, n=32, box=6.0, wz=2.0, g=30.0, omega=0.3, gauge=True, dt=1e-4, seed=306,
          init="phase"), 1, 200),
    (case(dim=2, n=64, box=8.0, g=120.0, omega=0.2, gauge=True, gdt=5e-3, seed=307), 0, 1000),
]


def serve(reqs, prec, check=50, thr=1e-8, **kw):
    """Submit (case, gstate, max_steps) requests at once; results by tag."""
    import gpue_b200 as G
    out = {}
    with G.Server(precision=prec, check_steps=check, threshold=thr, threshold_abs=True,
                  **kw) as srv:
        for tag, (c, gs, steps) in enumerate(reqs):
            srv.submit(product_params(c, prec), gs, steps, cases.initial_psi(c), tag)
        t_end = time.time() + 300
        while len(out) < len(reqs) and time.time() < t_end:
            for r in srv.poll(timeout=1.0):
                out[r["tag"]] = r
        stats = srv.stats()
    assert len(out) == len(reqs), stats
    return out, stats


@pytest.mark.parametrize("prec", [0, 1])
def test_a_served_solve_is_the_same_alone_and_in_the_mix(prec):
    alone, _ = serve([(PROBE, 0, 1000)], prec)
    mixed, st = serve(MIX[:3] + [(PROBE, 0, 1000)] + MIX[3:], prec)
    a, m = alone[0], mixed[3]
    assert a["status"] == 0 and m["status"] == 0
    assert a["steps_done"] == m["steps_done"] and a["early_stop"] == m["early_stop"]
    assert a["energy"] == m["energy"]
    assert np.array_equal(a["psi"], m["psi"])
    assert all(r["status"] == 0 for r in mixed.values())
    assert st["completed"] == len(MIX) + 1 and st["failed"] == 0


def test_served_solves_match_gpue_evolve_fp64():
    """Same steps through gpue_evolve: FP64 results agree to round-off."""
    import gpue_b200 as G
    res, _ = serve(MIX, G.PREC_FP64)
    for tag, (c, gs, steps) in enumerate(MIX):
        r = res[tag]
        assert r["status"] == 0
        if gs == 1:
            assert r["steps_done"] == steps and r["early_stop"] == 0
        with G.Solver(product_params(c, G.PREC_FP64)) as s:
            s.set_wfc(cases.initial_psi(c))
            s.evolve(r["steps_done"], gs)
            ref = s.get_wfc()
            E = s.energy()
        err = float(np.sqrt(np.sum(np.abs(r["psi"] - ref) ** 2) * dV(c)))
        assert err <= 1e-12, (tag, err)
        # the energy reported is the one of the last check (the final state)
        assert abs(r["energy"] - E) <= 1e-11 * abs(E)


def test_imaginary_time_solves_stop_at_the_threshold():
    import gpue_b200 as G
    reqs = [(c, gs, steps) for c, gs, steps in MIX if gs == 0]
    res, _ = serve(reqs, G.PREC_FP64, check=50, thr=1e-6)
    stopped = [r for r in res.values() if r["early_stop"]]
    assert stopped, res
    for r in stopped:
        assert r["steps_done"] % 50 == 0 and r["steps_done"] >= 100


def test_admission_respects_the_hbm_budget():
    import gpue_b200 as G
    c = MIX[3][0]  # 128^2
    reqs = [(dict(c, seed=400 + k), 1, 100) for k in range(6)]
    # room for two 128^2 FP32 solves (about 0.5 MB each) and not three
    res, st = serve(reqs, G.PREC_FP32, hbm_budget=1_100_000)
    assert all(r["status"] == 0 for r in res.values())
    assert 0 < st["bytes_peak"] <= 1_100_000
    assert st["bytes_resident"] == 0 and st["active"] == 0
    admits = sorted(r["t_admit"] for r in res.values())
    dones = sorted(r["t_done"] for r in res.values())
    # at most two resident at any time: the third admission follows the first finish
    assert admits[2] >= dones[0]


def test_a_request_larger_than_the_budget_fails_alone():
    import gpue_b200 as G
    big = case(dim=2, n=512, box=10.0, g=10.0, seed=410)
    small = case(dim=2, n=32, box=6.0, g=10.0, seed=411)
    res, st = serve([(big, 1, 100), (small, 1, 100)], G.PREC_FP32, hbm_budget=2_000_000)
    assert res[0]["status"] == 4  # GPUE_ERR_OUT_OF_MEMORY
    assert res[1]["status"] == 0
    assert st["failed"] == 1 and st["completed"] == 1
