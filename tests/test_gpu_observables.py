"""Observables (gpue_observables_get): the energy terms julia/calc_energy.jl
prints, the density moments py/en.py integrates and <L_z>, checked against
numpy on the state the library hands back, against gpue_energy / gpue_norm,
and against closed-form values for harmonic-trap ground states."""

import numpy as np
import pytest

import cases
from helpers import dV, oracle_problem, product_params

pytestmark = pytest.mark.gpu

TERMS = ("e_kinetic", "e_potential", "e_interaction", "e_rotation")
MOMENTS = ("x", "y", "z", "r2", "q")


def case(**kw):
    c = dict(cases.DEFAULTS, seed=21, init="phase")
    c.update(kw)
    return c


def derive(f, stride, d):
    """GPUE's derive() over the flat array (src/kernels.cu:58-71): forward
    difference with the given stride; past the end, f/d (no periodic wrap)."""
    out = np.empty_like(f)
    out[:-stride] = (f[stride:] - f[:-stride]) / d
    out[-stride:] = f[-stride:] / d
    return out


def trapz_nd(a, dim):
    """np.trapz over every axis with unit spacing, as py/en.py:44-50 nests it."""
    for _ in range(dim):
        a = np.trapezoid(a, axis=-1)
    return a


def numpy_observables(c, psi):
    """The gpue_observables fields computed with numpy from a complex128
    state [z, y, x], the oracle's V, K and A tables, and the grid."""
    prob = oracle_problem(c)
    dim = c["dim"]
    f = psi.reshape(-1)
    N = f.size
    v = dV(c)
    d = c["box"] / (c["n"] >> 1)
    rho = np.abs(f) ** 2
    out = {"norm": rho.sum() * v}
    psik = np.fft.fftn(psi).reshape(-1)
    out["e_kinetic"] = float(np.sum(prob.K * np.abs(psik) ** 2) / N * v)
    out["e_potential"] = float(np.sum(prob.V * rho) * v)
    out["e_interaction"] = float(np.sum(0.5 * c["g"] * rho * rho) * v) if c["gpe"] else 0.0
    n = c["n"]
    dx_, dy_ = derive(f, 1, d), derive(f, n, d)
    if c["gauge"]:
        l = prob.Ax * dx_ + prob.Ay * dy_
        if dim == 3:
            l = l + prob.Az * derive(f, n * n, d)
        out["e_rotation"] = float(np.sum(np.real(np.conj(f) * 1j * l)) * v)
    else:
        out["e_rotation"] = 0.0
    out["energy"] = sum(out[k] for k in TERMS)
    x = prob.x
    if dim == 2:
        XM, YM = np.meshgrid(x, x)
        ZM = np.zeros_like(XM)
    else:
        ZM, YM, XM = np.meshgrid(x, x, x, indexing="ij")
    dens = np.abs(psi) ** 2
    for key, val in (("x", XM), ("y", YM), ("z", ZM), ("r2", XM ** 2 + YM ** 2),
                     ("q", XM ** 2 - YM ** 2)):
        out[key] = float(trapz_nd(dens * val, dim) * v)
    X, Y = XM.reshape(-1), YM.reshape(-1)
    Lpsi = -1j * (X * dy_ - Y * dx_)
    out["lz"] = float(np.sum(np.real(np.conj(f) * Lpsi)) * v)
    return out


def run(c, steps, gs, precision=None, psi0=None):
    import gpue_b200 as G
    prec = G.PREC_FP64 if precision is None else precision
    with G.Solver(product_params(c, prec)) as s:
        s.set_wfc(cases.initial_psi(c) if psi0 is None else psi0)
        if steps:
            s.evolve(steps, gs)
        obs = s.observables()
        E, nrm = s.energy(), s.norm()
        psi = s.get_wfc()
    return obs, E, nrm, psi


def check_against_numpy(c, obs, psi, rtol):
    ref = numpy_observables(c, psi)
    scale = max(abs(ref["energy"]), 1.0)
    for k in TERMS + ("energy",):
        assert abs(obs[k] - ref[k]) <= rtol * scale, (k, obs[k], ref[k])
    assert obs["norm"] == pytest.approx(ref["norm"], rel=rtol)
    r2 = max(ref["r2"], 1e-3)
    for k in MOMENTS:
        assert abs(obs[k] - ref[k]) <= rtol * r2, (k, obs[k], ref[k])
    lz_scale = max(abs(ref["lz"]), 1.0)
    assert abs(obs["lz"] - ref["lz"]) <= rtol * lz_scale, (obs["lz"], ref["lz"])


@pytest.mark.parametrize("gs", [0, 1])
def test_rotating_2d_fp64_matches_numpy(gs):
    c = case(dim=2, n=128, box=8.0, g=200.0, omega=0.5, gauge=True, dt=5e-5)
    obs, E, nrm, psi = run(c, 200, gs)
    check_against_numpy(c, obs, psi, 1e-11)
    assert obs["energy"] == pytest.approx(E, rel=1e-12)
    assert obs["norm"] == pytest.approx(nrm, rel=1e-12)
    # rotation gauge with omegaX = omegaY: the gauge term is -omega*omegaY*<L_z>
    assert obs["e_rotation"] == pytest.approx(-c["omega"] * c["wy"] * obs["lz"], rel=1e-10,
                                              abs=1e-13)


def test_gauge_3d_fp64_matches_numpy():
    c = case(dim=3, n=32, box=6.0, wz=2.0, g=100.0, omega=0.3, gauge=True)
    obs, E, nrm, psi = run(c, 60, 0)
    check_against_numpy(c, obs, psi, 1e-11)
    assert obs["energy"] == pytest.approx(E, rel=1e-12)
    assert obs["e_rotation"] == pytest.approx(-c["omega"] * c["wy"] * obs["lz"], rel=1e-10,
                                              abs=1e-13)


def test_fp32_state_matches_numpy():
    """The FP32 form reduces in FP64 over the complex64 state it holds; the
    kinetic term goes through the complex64 transform."""
    import gpue_b200 as G
    c = case(dim=2, n=256, box=10.0, g=300.0, omega=0.6, gauge=True, dt=5e-5)
    obs, E, nrm, psi = run(c, 100, 1, precision=G.PREC_FP32)
    ref = numpy_observables(c, psi)
    for k in ("e_potential", "e_interaction", "e_rotation", "norm") + MOMENTS + ("lz",):
        assert obs[k] == pytest.approx(ref[k], rel=1e-6, abs=1e-9), k
    assert obs["e_kinetic"] == pytest.approx(ref["e_kinetic"], rel=1e-5)
    assert obs["energy"] == pytest.approx(E, rel=1e-12)


def test_displaced_trap_ground_state_moments():
    """Linear harmonic oscillator with the trap centre at x = -0.5: the ground
    state has <x> = -0.5, <x^2 + y^2> = 1 + 0.25, <x^2 - y^2> = 0.25 and
    E = 1 (hbar = m = omega = 1)."""
    c = case(dim=2, n=128, box=8.0, gpe=False, gdt=1e-2, init="gauss")
    import gpue_b200 as G
    p = product_params(c, G.PREC_FP64)
    p.x0_shift = 0.5
    with G.Solver(p) as s:
        s.set_wfc(cases.initial_psi(c))
        s.evolve(2500, 0)
        o = s.observables()
    assert o["norm"] == pytest.approx(1.0, rel=1e-12)
    assert o["x"] == pytest.approx(-0.5, abs=1e-3)
    assert abs(o["y"]) < 1e-6
    assert o["r2"] == pytest.approx(1.25, rel=1e-3)
    assert o["q"] == pytest.approx(0.25, abs=1e-3)
    assert o["energy"] == pytest.approx(1.0, rel=1e-3)
    assert abs(o["lz"]) < 1e-6


@pytest.mark.parametrize("charge", [1, -1])
def test_single_vortex_angular_momentum_sign(charge):
    """(x + i q y) exp(-r^2/2) carries L_z = q hbar per particle."""
    c = case(dim=2, n=256, box=8.0, g=0.0, gpe=False)
    x = -c["box"] + (c["box"] / (c["n"] >> 1)) * np.arange(c["n"])
    X, Y = np.meshgrid(x, x)
    psi = (X + 1j * charge * Y) * np.exp(-(X ** 2 + Y ** 2) / 2)
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * dV(c))
    obs, _, _, back = run(c, 0, 0, psi0=psi)
    assert obs["lz"] == pytest.approx(charge, abs=0.05)
    check_against_numpy(c, obs, back, 1e-11)


@pytest.mark.parametrize("gs", [0, 1])
def test_observables_recorded_at_energy_checks(gs):
    """gpue_set_check_observables: every check of an evolve call yields the
    observables of the state it checks (those gpue_observables_get gives for
    that state), without changing the run."""
    import gpue_b200 as G
    c = case(dim=2, n=128, box=8.0, g=200.0, omega=0.5, gauge=True, dt=5e-5)
    psi0 = cases.initial_psi(c)
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        s.set_wfc(psi0)
        plain = s.evolve(400, gs, energy_every=100)
        want_psi = s.get_wfc()
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        s.record_check_observables(8)
        s.set_wfc(psi0)
        r = s.evolve(400, gs, energy_every=100)
        got_psi = s.get_wfc()
        rec = s.check_observables(r["n_energies"])
    assert r["n_energies"] == plain["n_energies"] == 4
    assert np.array_equal(got_psi, want_psi)
    assert r["energy"] == pytest.approx(plain["energy"], rel=1e-13)
    assert rec[-1]["energy"] == pytest.approx(r["energy"], rel=1e-13)
    # the check at step 300 sees the state after 301 steps
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        s.set_wfc(psi0)
        s.evolve(301, gs)
        ref = s.observables()
    for k in ref:
        assert rec[3][k] == pytest.approx(ref[k], rel=1e-12, abs=1e-15), k
    assert rec[0]["norm"] > 0 and len({round(o["lz"], 12) for o in rec}) > 1
