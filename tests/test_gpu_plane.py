"""The XY passes of the complex64 3D step against the oracle and against the
five-pass line schedule.

A 3D FP32 context with nx = ny of a length that has an XY kernel runs its
steps as XY[scale V/2 Fx Fy] Z[Fz K Iz] XY[Ix Iy V/2 norm], by the
TMA tile-stream XY kernel (tstream.cuh; GPUE_XY=0 turns it off) or the
cluster plane kernel (plane.cuh; GPUE_PLANE=0 turns it off), with the TMA z
pass (tstream.cuh; GPUE_ZTMA=0 turns it off).  Both schedules are the same
arithmetic in another order, so they agree to complex64 round-off; both are
checked against the FP64 oracle with the FP32 tolerances of the other parity
tests (wavefunction L2 <= 1e-5, relative energy <= 1e-5).
"""
import os

import numpy as np
import pytest

import cases
from helpers import dV, oracle_problem, product_params

pytestmark = pytest.mark.gpu

PLANE_LENGTHS = [64, 96, 128, 160, 192, 256]


def run(c, steps, gstate, plane, psi0, ztma=True):
    """plane: "xy" (the cluster-free XY pass where its kernels exist, else
    the cluster plane kernels), "cluster" (the cluster plane kernels), or
    False / "lines" (the five line passes)."""
    import gpue_b200 as G
    if plane is True:
        plane = "xy"
    old = {k: os.environ.get(k) for k in ("GPUE_PLANE", "GPUE_XY", "GPUE_ZTMA")}
    os.environ["GPUE_PLANE"] = "1" if plane in ("cluster", "xy") else "0"
    os.environ["GPUE_XY"] = "1" if plane == "xy" else "0"
    os.environ["GPUE_ZTMA"] = "1" if ztma else "0"
    try:
        with G.Solver(product_params(c, G.PREC_FP32)) as s:
            s.set_wfc(psi0)
            r = s.evolve(steps, gstate, energy_every=c["energy_every"])
            return s.get_wfc(), s.energy(), r
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.mark.parametrize("gstate", [0, 1], ids=["imag", "real"])
@pytest.mark.parametrize("n", PLANE_LENGTHS)
def test_plane_schedule_matches_oracle_and_line_schedule(n, gstate):
    steps = 12 if n <= 128 else 4
    c = dict(cases.DEFAULTS, dim=3, n=n, box=8.0, wz=2.5, g=200.0, gdt=1e-4, dt=1e-4,
             seed=500 + n, init="gauss" if gstate == 0 else "phase",
             energy_every=steps // 2)
    psi0 = cases.initial_psi(c)
    got, E, r = run(c, steps, gstate, "xy", psi0)
    clu, Ec, rc = run(c, steps, gstate, "cluster", psi0)
    lines, El, rl = run(c, steps, gstate, "lines", psi0)
    P = oracle_problem(c)
    ref, res, en = P.evolve(psi0, steps, gstate)
    Eref = P.energy(ref)
    for psi, e in ((got, E), (clu, Ec), (lines, El)):
        assert float(np.sqrt(np.sum(np.abs(psi - ref) ** 2) * dV(c))) <= 1e-5
        assert abs(e - Eref) <= 1e-5 * abs(Eref)
    for psi in (got, clu):
        assert float(np.sqrt(np.sum(np.abs(psi - lines) ** 2) * dV(c))) <= 1e-5
    assert r["n_energies"] == rc["n_energies"] == rl["n_energies"] == res["n_energies"]
    for rr in (r, rc):
        assert abs(rr["energy"] - en[-1]) <= 1e-5 * abs(en[-1])
        # three passes per step instead of five
        assert rr["kernel_launches"] < rl["kernel_launches"]


@pytest.mark.parametrize("n", PLANE_LENGTHS)
def test_tma_z_pass_matches_the_line_z_pass(n):
    """The TMA-fed z pass moves data differently but runs the same operations
    as the line pass along z: the two agree to complex64 round-off (the
    compiler may contract multiply-adds differently in the two kernels)."""
    c = dict(cases.DEFAULTS, dim=3, n=n, box=8.0, wz=2.5, g=200.0, dt=1e-4, seed=520 + n,
             init="phase", energy_every=0)
    psi0 = cases.initial_psi(c)
    a, Ea, ra = run(c, 4, 1, "xy", psi0, ztma=True)
    b, Eb, rb = run(c, 4, 1, "xy", psi0, ztma=False)
    assert float(np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c))) <= 1e-6
    assert abs(Ea - Eb) <= 1e-7 * abs(Eb)


def test_plane_passes_chosen_only_where_they_apply():
    """Gauge fields in the plane keep the line passes (same results as the
    oracle either way); FP64 contexts have no plane kernels."""
    import gpue_b200 as G
    c = dict(cases.DEFAULTS, dim=3, n=64, box=8.0, wz=2.0, g=100.0, omega=0.4, gauge=True,
             dt=1e-4, seed=77, init="phase", energy_every=0)
    psi0 = cases.initial_psi(c)
    got, E, r = run(c, 6, 1, "xy", psi0)
    lines, El, rl = run(c, 6, 1, "lines", psi0)
    assert r["kernel_launches"] == rl["kernel_launches"]
    assert np.array_equal(got, lines)


@pytest.mark.parametrize("gstate", [0, 1], ids=["imag", "real"])
def test_time_passes_reports_the_step_and_leaves_the_state(gstate):
    """gpue_time_passes on a 3D complex64 grid: the three passes of the step
    (forward XY, z, inverse XY), each with a positive device time, and the
    state afterwards exactly as before; a later evolve matches one on a
    context that was never timed (to round-off: the norm's partial sums
    follow the tile tickets, which change from launch to launch)."""
    import gpue_b200 as G
    c = dict(cases.DEFAULTS, dim=3, n=64, box=8.0, wz=2.5, g=200.0, gdt=1e-4, dt=1e-4,
             seed=77, init="gauss" if gstate == 0 else "phase", energy_every=4)
    psi0 = cases.initial_psi(c)
    with G.Solver(product_params(c, G.PREC_FP32)) as s, \
            G.Solver(product_params(c, G.PREC_FP32)) as u:
        s.set_wfc(psi0)
        u.set_wfc(psi0)
        s.evolve(2, gstate)
        u.evolve(2, gstate)
        before = s.get_wfc()
        t = s.time_passes(gstate, nsteps=4)
        assert [k for k, _ in t] == [3, 2, 4]
        assert all(us > 0 for _, us in t)
        assert np.array_equal(s.get_wfc(), before)
        s.evolve(4, gstate, step_offset=2)
        u.evolve(4, gstate, step_offset=2)
        a, b = s.get_wfc(), u.get_wfc()
        assert np.max(np.abs(a - b)) <= 1e-6 * np.max(np.abs(b))

