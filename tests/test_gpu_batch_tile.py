"""Large 3D complex64 solves in a batch run the tile-stream step: three tile
passes per step (forward XY, z, inverse XY), one launch per solve and pass,
instead of the five line passes of a group launch.  A solve whose active flag
the batch check cleared (converged) is left untouched by its later launches.

Checked against each solve run alone through gpue_evolve for the same number
of steps (which runs the same tile passes; complex64 tolerances, since the
norm's partial sums follow the tile tickets), and against the same batch with
the tile path off (GPUE_BATCH_TILE=0: group launches of line passes).
"""
import os

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu


def case(**kw):
    c = dict(cases.DEFAULTS, init="gauss")
    c.update(kw)
    return c


# two 128^3 grids (2^21 points: tile path) and a 96^3 one (below 2^20 points:
# line passes beside them; its small imaginary step keeps it from stopping)
MIX = [
    case(dim=3, n=128, box=8.0, wz=2.0, g=200.0, gdt=5e-3, seed=701),
    case(dim=3, n=128, box=8.0, wz=1.5, g=600.0, gdt=5e-3, seed=702),
    case(dim=3, n=96, box=8.0, wz=2.5, g=100.0, gdt=1e-4, seed=703),
]
TOL_E, TOL_L2 = 1e-6, 1e-5


def run_batch(cs, gstate, steps, kw, tile=True, mega=True):
    import gpue_b200 as G
    env = {"GPUE_BATCH_TILE": "1" if tile else "0", "GPUE_BATCH_MEGA": "1" if mega else "0"}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        ss = []
        for c in cs:
            s = G.Solver(product_params(c, G.PREC_FP32))
            s.set_wfc(cases.initial_psi(c))
            ss.append(s)
        with G.Batch(ss) as b:
            res, stats = b.evolve(gstate, steps, **kw)
        psis = [s.get_wfc() for s in ss]
        for s in ss:
            s.close()
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    return res, stats, psis


def alone(c, gstate, steps, **kw):
    import gpue_b200 as G
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        s.set_wfc(cases.initial_psi(c))
        r = s.evolve(steps, gstate, **kw)
        return s.get_wfc(), r


def l2(a, b, c):
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c)))


def test_imaginary_time_with_early_stop_matches_each_solve_alone():
    """Solves stop at different checks; each ends with the state a lone run
    of its own step count reaches, so a stopped solve stayed frozen."""
    kw = dict(energy_every=100, threshold=1e-6, threshold_abs=True)
    res, _, psis = run_batch(MIX, 0, 1500, kw)
    steps = set()
    for c, r, psi in zip(MIX, res, psis):
        psi_a, ra = alone(c, 0, r["steps_done"], energy_every=100)
        assert abs(r["energy"] - ra["energy"]) <= TOL_E * abs(ra["energy"])
        assert l2(psi, psi_a, c) <= TOL_L2
        steps.add(r["steps_done"])
    assert any(r["early_stop"] for r in res[:2]) and not res[2]["early_stop"]
    assert len(steps) > 1  # the solves stop at different checks


def test_real_time_matches_alone_and_the_line_passes():
    mix = [dict(c, init="phase", dt=1e-4) for c in MIX]
    kw = dict(energy_every=100)
    res, stats, psis = run_batch(mix, 1, 300, kw, mega=False)
    res_l, stats_l, psis_l = run_batch(mix, 1, 300, kw, tile=False, mega=False)
    # three launches per step for each large solve instead of one group
    # launch of five line passes for both
    assert stats["kernel_launches"] > stats_l["kernel_launches"]
    for c, r, psi, rl, psi_l in zip(mix, res, psis, res_l, psis_l):
        psi_a, ra = alone(c, 1, 300, energy_every=100)
        assert r["steps_done"] == 300
        assert abs(r["energy"] - ra["energy"]) <= TOL_E * abs(ra["energy"])
        assert l2(psi, psi_a, c) <= TOL_L2
        assert abs(r["energy"] - rl["energy"]) <= TOL_E * abs(rl["energy"])
        assert l2(psi, psi_l, c) <= TOL_L2
