"""Uneven grid sizes in one persistent launch (k_batch_mega): solves whose
axes all have lengths the persistent kernel covers (64 to 512, 2D and 3D)
take no per-shape launches; one launch per segment walks a queue of
(solve, pass, tile) tickets.

Checked against each solve run alone through gpue_evolve (FP64 to round-off,
FP32 to the complex64 tolerances), against the per-shape group launches
(GPUE_BATCH_MEGA=0), and for bit-identical results alone and in a mix that
also holds solves the persistent kernel does not cover (which keep group
launches beside it).
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


# the batched-sweep sizes and 3D, imaginary time, uneven convergence
UNEVEN = [
    case(dim=2, n=128, box=10.0, g=100.0, gdt=5e-3, seed=601),
    case(dim=2, n=192, box=10.0, g=400.0, wy=1.2, gdt=5e-3, seed=602),
    case(dim=2, n=256, box=10.0, g=50.0, wy=0.85, gdt=5e-3, seed=603),
    case(dim=2, n=384, box=10.0, g=800.0, gdt=5e-3, seed=604),
    case(dim=2, n=512, box=10.0, g=250.0, wy=1.1, gdt=5e-3, seed=605),
    case(dim=2, n=64, box=8.0, g=120.0, omega=0.4, gauge=True, gdt=5e-3, seed=606),
    case(dim=3, n=64, box=6.0, wz=2.0, g=60.0, gdt=5e-3, seed=607),
]
# lengths the persistent kernel does not cover, batched beside it
OTHERS = [
    case(dim=2, n=96, box=8.0, g=90.0, gdt=5e-3, seed=608),
    case(dim=2, n=640, box=12.0, g=300.0, gdt=5e-3, seed=609),
]
KW = dict(energy_every=100, threshold=1e-8, threshold_abs=True)
STEPS = 2000


def solvers(cs, prec):
    import gpue_b200 as G
    out = []
    for c in cs:
        s = G.Solver(product_params(c, prec))
        s.set_wfc(cases.initial_psi(c))
        out.append(s)
    return out


def run_batch(cs, prec, gstate=0, steps=STEPS, kw=KW, mega=True):
    import gpue_b200 as G
    old = os.environ.get("GPUE_BATCH_MEGA")
    os.environ["GPUE_BATCH_MEGA"] = "1" if mega else "0"
    try:
        ss = solvers(cs, prec)
        with G.Batch(ss) as b:
            res, stats = b.evolve(gstate, steps, **kw)
        psis = [s.get_wfc() for s in ss]
        for s in ss:
            s.close()
    finally:
        if old is None:
            del os.environ["GPUE_BATCH_MEGA"]
        else:
            os.environ["GPUE_BATCH_MEGA"] = old
    return res, stats, psis


def alone(c, prec, gstate, steps, **kw):
    import gpue_b200 as G
    with G.Solver(product_params(c, prec)) as s:
        s.set_wfc(cases.initial_psi(c))
        r = s.evolve(steps, gstate, **kw)
        return s.get_wfc(), r


def l2(a, b, c):
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c)))


@pytest.mark.parametrize("prec", [0, 1])
def test_uneven_sizes_in_one_launch_match_each_solve_alone(prec):
    """FP64 with the early stop (solves converge at different checks); FP32
    runs every step, as its energies differ from a lone run's by complex64
    round-off, which moves a stop this close to the threshold by a check."""
    import gpue_b200 as G
    kw = KW if prec == G.PREC_FP64 else dict(energy_every=100)
    res, stats, psis = run_batch(UNEVEN, prec, kw=kw)
    _, stats_g, psis_g = run_batch(UNEVEN, prec, kw=kw, mega=False)
    # one persistent launch per segment instead of a launch per pass and shape
    assert stats["kernel_launches"] < stats_g["kernel_launches"] / 2
    tol_e, tol_l2 = (1e-12, 1e-12) if prec == G.PREC_FP64 else (1e-6, 1e-5)
    steps = set()
    for c, r, psi, psi_g in zip(UNEVEN, res, psis, psis_g):
        psi_a, ra = alone(c, prec, 0, STEPS, **kw)
        assert r["steps_done"] == ra["steps_done"] and r["early_stop"] == ra["early_stop"]
        assert abs(r["energy"] - ra["energy"]) <= tol_e * abs(ra["energy"])
        assert l2(psi, psi_a, c) <= tol_l2
        assert l2(psi, psi_g, c) <= tol_l2
        steps.add(r["steps_done"])
    if prec == G.PREC_FP64:
        assert len(steps) > 1  # the solves converge at different checks


@pytest.mark.parametrize("prec", [0, 1])
def test_real_time_uneven_batch_matches_each_solve_alone(prec):
    import gpue_b200 as G
    mix = [dict(c, init="phase", dt=5e-5) for c in UNEVEN[:3] + UNEVEN[5:]]
    res, _, psis = run_batch(mix, prec, gstate=1, steps=300, kw=dict(energy_every=100))
    tol_e, tol_l2 = (1e-12, 1e-12) if prec == G.PREC_FP64 else (1e-6, 1e-5)
    for c, r, psi in zip(mix, res, psis):
        psi_a, ra = alone(c, prec, 1, 300, energy_every=100)
        assert r["steps_done"] == 300
        assert abs(r["energy"] - ra["energy"]) <= tol_e * abs(ra["energy"])
        assert l2(psi, psi_a, c) <= tol_l2


@pytest.mark.parametrize("prec", [0, 1])
def test_bit_identical_alone_and_beside_group_launched_solves(prec):
    probe = 3
    r1, _, p1 = run_batch([UNEVEN[probe]], prec, steps=600)
    mix = OTHERS[:1] + UNEVEN + OTHERS[1:]
    rm, _, pm = run_batch(mix, prec, steps=600)
    assert r1[0] == rm[probe + 1]
    assert np.array_equal(p1[0], pm[probe + 1])
