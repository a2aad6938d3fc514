"""Batches of independent solves (gpue_batch_*) against the same solves run
one at a time through gpue_evolve, and against themselves in other company.

A batch member must end where gpue_evolve would have left it: same steps,
same early stop, energy and wavefunction within FP64 round-off (the batched
reductions sum in a different order).  A member's result must not depend on
which other solves share the batch: that holds bit for bit, in both
precisions, because each solve reduces over its own tiles in a fixed order.
"""

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu


def case(**kw):
    c = dict(cases.DEFAULTS, init="gauss")
    c.update(kw)
    return c


IMAG_MIX = [
    case(dim=2, n=64, box=8.0, g=100.0, gdt=5e-3, seed=101),
    case(dim=2, n=64, box=8.0, g=300.0, wy=1.2, gdt=5e-3, seed=102),
    case(dim=2, n=96, box=10.0, g=50.0, omega=0.3, gauge=True, gdt=5e-3, seed=103),
    case(dim=2, n=32, box=6.0, gpe=False, gdt=5e-3, seed=104),
    case(dim=3, n=16, box=6.0, wz=2.0, g=50.0, gdt=5e-3, seed=105),
    case(dim=2, n=128, box=10.0, g=500.0, wy=0.9, gdt=5e-3, seed=106),
]

REAL_MIX = [
    case(dim=2, n=64, box=8.0, g=200.0, omega=0.5, gauge=True, dt=5e-5, seed=201, init="phase"),
    case(dim=2, n=64, box=8.0, g=100.0, omega=0.0, gauge=True, dt=5e-5, seed=202, init="phase"),
    case(dim=2, n=32, box=6.0, wy=1.3, gpe=False, dt=1e-4, seed=203, init="phase"),
    case(dim=3, n=16, box=6.0, wz=2.0, g=50.0, omega=0.5, gauge=True, dt=1e-4, seed=204,
         init="phase"),
]


def solvers(cs, prec):
    import gpue_b200 as G
    out = []
    for c in cs:
        s = G.Solver(product_params(c, prec))
        s.set_wfc(cases.initial_psi(c))
        out.append(s)
    return out


def alone(c, prec, gstate, steps, **kw):
    import gpue_b200 as G
    with G.Solver(product_params(c, prec)) as s:
        s.set_wfc(cases.initial_psi(c))
        r = s.evolve(steps, gstate, **kw)
        return s.get_wfc(), r


def l2(a, b, c):
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c)))


def test_imaginary_batch_matches_each_solve_alone_fp64():
    import gpue_b200 as G
    kw = dict(energy_every=50, threshold=1e-8, threshold_abs=True)
    ss = solvers(IMAG_MIX, G.PREC_FP64)
    with G.Batch(ss) as b:
        res, stats = b.evolve(0, 2000, **kw)
    steps = []
    for c, s, r in zip(IMAG_MIX, ss, res):
        psi_a, ra = alone(c, G.PREC_FP64, 0, 2000, **kw)
        assert r["steps_done"] == ra["steps_done"], (c, r, ra)
        assert r["early_stop"] == ra["early_stop"]
        assert abs(r["energy"] - ra["energy"]) <= 1e-12 * abs(ra["energy"])
        assert l2(s.get_wfc(), psi_a, c) <= 1e-12
        assert abs(s.norm() - 1.0) <= 1e-12
        steps.append(r["steps_done"])
        s.close()
    assert any(r["early_stop"] for r in res)
    assert len(set(steps)) > 1  # the solves stop at different checks
    assert stats["point_steps"] == sum(c["n"] ** c["dim"] * k for c, k in zip(IMAG_MIX, steps))
    assert stats["graph_launches"] >= 1 and stats["kernel_launches"] > 0


def test_real_time_batch_matches_each_solve_alone_fp64():
    import gpue_b200 as G
    ss = solvers(REAL_MIX, G.PREC_FP64)
    with G.Batch(ss) as b:
        res, _ = b.evolve(1, 301, energy_every=100)
    for c, s, r in zip(REAL_MIX, ss, res):
        psi_a, ra = alone(c, G.PREC_FP64, 1, 301, energy_every=100)
        assert r["steps_done"] == 301 and r["early_stop"] == 0
        assert abs(r["energy"] - ra["energy"]) <= 1e-12 * abs(ra["energy"])
        assert l2(s.get_wfc(), psi_a, c) <= 1e-12
        s.close()


def test_fp32_batch_matches_each_solve_alone():
    import gpue_b200 as G
    mix = IMAG_MIX[:3] + IMAG_MIX[5:]
    ss = solvers(mix, G.PREC_FP32)
    with G.Batch(ss) as b:
        res, _ = b.evolve(0, 400, energy_every=100)
    for c, s, r in zip(mix, ss, res):
        psi_a, ra = alone(c, G.PREC_FP32, 0, 400, energy_every=100)
        assert r["steps_done"] == 400
        assert abs(r["energy"] - ra["energy"]) <= 1e-6 * abs(ra["energy"])
        assert l2(s.get_wfc(), psi_a, c) <= 1e-5
        s.close()


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("gstate", [0, 1])
def test_a_solve_is_bit_identical_alone_and_in_the_mix(prec, gstate):
    import gpue_b200 as G
    mix = IMAG_MIX if gstate == 0 else REAL_MIX
    kw = dict(energy_every=50, threshold=1e-8, threshold_abs=True) if gstate == 0 else \
        dict(energy_every=100)
    steps = 600 if gstate == 0 else 201
    probe = 1
    (s1,) = solvers([mix[probe]], prec)
    with G.Batch([s1]) as b:
        r1, _ = b.evolve(gstate, steps, **kw)
    ss = solvers(mix, prec)
    with G.Batch(ss) as b:
        rm, _ = b.evolve(gstate, steps, **kw)
    assert r1[0] == rm[probe]
    a, m = s1.get_wfc(), ss[probe].get_wfc()
    assert np.array_equal(a, m)
    for s in ss + [s1]:
        s.close()


def test_batch_runs_again_from_the_state_it_left():
    """A second call continues each solve (graphs are reused)."""
    import gpue_b200 as G
    mix = REAL_MIX[:2]
    ss = solvers(mix, G.PREC_FP64)
    with G.Batch(ss) as b:
        b.evolve(1, 100)
        _, st2 = b.evolve(1, 100)
    for c, s in zip(mix, ss):
        with G.Solver(product_params(c, G.PREC_FP64)) as a:
            a.set_wfc(cases.initial_psi(c))
            a.evolve(100, 1)
            a.evolve(100, 1)
            assert l2(s.get_wfc(), a.get_wfc(), c) <= 1e-12
        s.close()
    assert st2["point_steps"] == sum(c["n"] ** c["dim"] * 100 for c in mix)


def test_batch_rejects_parameter_file_solves():
    import gpue_b200 as G
    c = IMAG_MIX[0]
    ss = solvers([c, IMAG_MIX[1]], G.PREC_FP64)
    ss[1].load_param_text("V = 0.5*(x*x + y*y)")
    with G.Batch(ss) as b:
        with pytest.raises(G.GpueError) as e:
            b.evolve(0, 10)
    assert e.value.status == 2
    for s in ss:
        s.close()
