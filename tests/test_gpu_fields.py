"""Tabulated gauge fields (gpue_set_gauge_tables, GPUE's -A file): the
rotation field given as tables must reproduce the preset rotation gauge, and
an arbitrary field must match the oracle run with the same arrays."""

import numpy as np
import pytest

import cases
from cli_helpers import read_wfc, run
from helpers import dV, oracle_problem, product_params

pytestmark = pytest.mark.gpu


def case(**kw):
    c = dict(cases.DEFAULTS, init="phase")
    c.update(kw)
    return c


def l2(a, b, c):
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c)))


def grid_axes(c):
    import oracle
    x, _ = oracle.axis_grid(c["n"], c["box"])
    return x


def rotation_tables(c):
    """A = omega (-wx y, wy x, 0) on the grid, x fastest."""
    x = grid_axes(c)
    if c["dim"] == 2:
        X, Y = x[None, :], x[:, None]
        ones = np.ones((c["n"], c["n"]))
    else:
        X, Y = x[None, None, :], x[None, :, None]
        ones = np.ones((c["n"],) * 3)
    Ax = -c["omega"] * c["wx"] * Y * ones
    Ay = c["omega"] * c["wy"] * X * ones
    return Ax, Ay


def run_product(c, gs, steps, tables=None):
    import gpue_b200 as G
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        if tables is not None:
            s.set_gauge_tables(*tables)
        s.set_wfc(cases.initial_psi(c))
        s.evolve(steps, gs)
        return s.get_wfc(), s.energy()


@pytest.mark.parametrize("c,gs", [
    (case(dim=2, n=64, box=8.0, g=200.0, omega=0.6, gauge=True, dt=5e-5, seed=601), 1),
    (case(dim=2, n=64, box=8.0, g=200.0, omega=0.4, gauge=True, gdt=1e-3, seed=602,
          init="gauss"), 0),
    (case(dim=3, n=16, box=6.0, wz=2.0, g=50.0, omega=0.5, gauge=True, dt=1e-4, seed=603), 1),
], ids=["2d_real", "2d_imag", "3d_real"])
def test_rotation_as_tables_equals_the_preset(c, gs):
    psi_p, E_p = run_product(c, gs, 120)
    psi_t, E_t = run_product(c, gs, 120, rotation_tables(c))
    assert l2(psi_p, psi_t, c) <= 1e-12
    assert abs(E_p - E_t) <= 1e-12 * abs(E_p)


def test_custom_gauge_field_matches_the_oracle():
    c = case(dim=2, n=64, box=8.0, g=150.0, omega=0.0, gauge=True, dt=5e-5, seed=604)
    x = grid_axes(c)
    X, Y = x[None, :], x[:, None]
    Ax = 0.4 * np.sin(0.7 * Y) + 0.05 * X
    Ay = 0.3 * np.cos(0.5 * X) - 0.02 * Y * X
    psi, E = run_product(c, 1, 100, (Ax, Ay, None))
    P = oracle_problem(c)
    P.Ax[:] = Ax.ravel()
    P.Ay[:] = Ay.ravel()
    P.V[:] = P.V + 0.5 * (Ax.ravel() ** 2 + Ay.ravel() ** 2)
    ref, _, _ = P.evolve(cases.initial_psi(c), 100, 1)
    assert l2(psi, ref, c) <= 1e-12
    Eref = P.energy(ref)
    assert abs(E - Eref) <= 1e-12 * abs(Eref)


def test_cli_file_gauge_equals_its_preset(tmp_path):
    """-A file with Axgauge/Aygauge holding the rotation field over omega."""
    n, w = 64, 0.5
    common = ["-x", n, "-y", n, "-s", "-l", "-w", w, "-i", 100, "-g", 60, "-e", 40]
    pre, fil = tmp_path / "preset", tmp_path / "file"
    pre.mkdir()
    fil.mkdir()
    run(common, pre)
    xs = np.loadtxt(pre / "x_0")
    ys = np.loadtxt(pre / "y_0")
    p = {}
    for line in open(pre / "Params.dat"):
        if "=" in line:
            k, v = line.strip().split("=", 1)
            p[k] = float(v)
    X, Y = xs[None, :] * np.ones((n, 1)), ys[:, None] * np.ones((1, n))
    np.savetxt(fil / "Axgauge", (-p["omegaX"] * Y).ravel(), fmt="%.17e")
    np.savetxt(fil / "Aygauge", (p["omegaY"] * X).ravel(), fmt="%.17e")
    run(common + ["-A", "file"], fil)
    a = read_wfc(pre, "wfc_ev_final", 0, (n, n))
    b = read_wfc(fil, "wfc_ev_final", 0, (n, n))
    assert float(np.linalg.norm(a - b) / np.linalg.norm(a)) <= 1e-11
