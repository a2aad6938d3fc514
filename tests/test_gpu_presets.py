"""GPUE's non-separable field presets as tables: the gauge fields of -A
ring_rotation / ring / test and the torus potential and initial state of -v
torus.  The library path (gpue_set_gauge_tables + gpue_set_potential_table)
is checked against the oracle run on the same arrays; the command line,
which tabulates the presets itself, against the library fed with tables
computed here from GPUE's kernel formulas (src/operators.cu:621-720,
1011-1067)."""

import os

import numpy as np
import pytest

import cases
from cli_helpers import params, read_wfc, run
from helpers import dV, oracle_problem, product_params

pytestmark = pytest.mark.gpu


def preset_A(name, X, Y, Z, omega, wx, xmax, ymax, zmax, dim):
    """Ax, Ay, Az of one -A preset on broadcast position arrays."""
    shape = np.broadcast(X, Y, Z).shape
    zero = np.zeros(shape)
    if name == "ring_rotation":
        th = np.arctan2(Y, X)
        Ax = (Z + zmax) * np.cos(th) * omega * wx
        Ay = (Z + zmax) * np.sin(th) * omega * wx
        Az = np.sqrt(X * X + Y * Y) * omega * wx + zero if dim == 3 else zero
        return Ax + zero, Ay + zero, Az
    if name == "ring":
        r = np.sqrt(X * X + Y * Y)
        Az = omega * np.exp(-r * r / (0.0001 * xmax)) * 0.01 + zero if dim == 3 else zero
        return zero, zero, Az
    if name == "test":
        return (np.sin(Y * 100000) + 1) * ymax * omega + zero, zero, zero
    raise ValueError(name)


def torus_V(X, Y, Z, A, p, dim):
    wz = p["omegaZ"] if dim == 3 else 0.0
    z0 = p["z0_shift"] if dim == 3 else 0.0
    rad = np.sqrt((X - p["x0_shift"]) ** 2 + (Y - p["y0_shift"]) ** 2) - 0.5 * p["xMax"]
    wr = p["omegaX"] ** 2 + p["omegaY"] ** 2
    vt = 2 * wz * wz * (Z - z0) ** 2 + wr * (rad * rad + p["fudge"] * rad * Z)
    return 0.5 * p["mass"] * (vt + A[0] ** 2 + A[1] ** 2 + A[2] ** 2)


def grids(c):
    x = cases.grid_x(c["n"], c["box"])
    if c["dim"] == 2:
        return x[None, :], x[:, None], np.zeros((1, 1))
    return x[None, None, :], x[None, :, None], x[:, None, None]


@pytest.mark.parametrize("name", ["ring_rotation", "ring", "test"])
def test_preset_tables_match_the_oracle(name):
    """3D, hbar = m = 1: each gauge preset with the torus potential, real
    then imaginary time, against the oracle given the same arrays."""
    import gpue_b200 as G
    c = dict(cases.DEFAULTS, dim=3, n=16, box=6.0, wz=2.0, g=40.0, omega=0.4, gauge=True,
             dt=1e-4, gdt=1e-3, seed=701, init="phase")
    X, Y, Z = grids(c)
    A = preset_A(name, X, Y, Z, c["omega"], c["wx"], c["box"], c["box"], c["box"], 3)
    p = dict(omegaX=1.0, omegaY=1.0, omegaZ=c["wz"], x0_shift=0.3, y0_shift=-0.2,
             z0_shift=0.1, xMax=c["box"], mass=1.0, fudge=0.5)
    V = torus_V(X, Y, Z, A, p, 3)
    psi0 = cases.initial_psi(c)
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        s.set_gauge_tables(*A)
        s.set_potential_table(V)
        s.set_wfc(psi0)
        s.evolve(60, 1)
        real = s.get_wfc()
        E_real = s.energy()
        s.evolve(60, 0)
        imag = s.get_wfc()
    P = oracle_problem(c)
    for dst, src in ((P.Ax, A[0]), (P.Ay, A[1]), (P.Az, A[2]), (P.V, V)):
        dst[:] = src.ravel()
    ref_real, _, _ = P.evolve(psi0, 60, 1)
    ref_imag, _, _ = P.evolve(ref_real, 60, 0)
    for a, b in ((real, ref_real), (imag, ref_imag)):
        assert np.sqrt(np.sum(np.abs(a - b) ** 2) * dV(c)) <= 1e-12
    assert E_real == pytest.approx(P.energy(ref_real), rel=1e-12)


# In 2D ring_rotation sees zMax = 1 (metres, in GPUE's SI units), so A is
# ~6 omega and the imaginary-time gauge factor exp(-A p gdt) overflows unless
# omega is small; GPUE behaves the same.
@pytest.mark.parametrize("dim,gauge,omega", [(2, "ring_rotation", 1e-4), (3, "ring_rotation", 0.3),
                                             (3, "ring", 0.3), (2, "test", 0.3)])
def test_cli_presets_equal_the_library(tmp_path, dim, gauge, omega):
    import gpue_b200 as G
    from test_gpu_cli import lib_params
    n = 64 if dim == 2 else 16
    args = ["-x", n, "-y", n, "-v", "torus", "-A", gauge, "-l", "-w", omega, "-s", "-i", 50,
            "-F", 0.2, "-U", 1e-6, "-g", 40, "-e", 30]
    if dim == 3:
        args = ["-c", 3, "-z", n] + args
    run(args, tmp_path)
    p = params(args, tmp_path)
    shape = (n,) * dim
    x = np.loadtxt(os.path.join(tmp_path, "x_0"))
    y = np.loadtxt(os.path.join(tmp_path, "y_0"))
    z = np.loadtxt(os.path.join(tmp_path, "z_0")) if dim == 3 else np.zeros(1)
    if dim == 2:
        X, Y, Z = x[None, :], y[:, None], np.zeros((1, 1))
    else:
        X, Y, Z = x[None, None, :], y[None, :, None], z[:, None, None]
    A = preset_A(gauge, X, Y, Z, p["omega"], p["omegaX"], p["xMax"], p["yMax"],
                 p["zMax"] if dim == 3 else 1.0, dim)
    V = torus_V(X, Y, Z, A, p, dim)
    # ktorus_wfc, normalised as init() does (by sqrt(sum |psi| dV))
    rad = np.sqrt((X - p["x0_shift"]) ** 2 + (Y - p["y0_shift"]) ** 2) - 0.5 * p["xMax"]
    az = p["a0z"] if dim == 3 else 1.0
    w0 = np.exp(-((rad / (p["Rxy"] * p["a0x"] * 0.5)) ** 2 + (Z / (p["Rxy"] * az * 0.5)) ** 2))
    w0 = np.broadcast_to(w0, shape).astype(np.complex128)
    dvol = p["dx"] * p["dy"] * (p["dz"] if dim == 3 else 1.0)
    w0 = w0 / np.sqrt(np.sum(np.abs(w0)) * dvol)
    psi0 = read_wfc(tmp_path, "WFC", 0, shape)
    assert np.linalg.norm(psi0 - w0) <= 1e-12 * np.linalg.norm(w0)
    with G.Solver(lib_params(params(args, tmp_path))) as s:
        s.set_gauge_tables(A[0] + np.zeros(shape), A[1] + np.zeros(shape),
                           A[2] + np.zeros(shape))
        s.set_potential_table(V + np.zeros(shape))
        s.set_wfc(psi0)
        s.evolve(40, 0)
        ground = s.get_wfc()
        s.evolve(30, 1)
        final = s.get_wfc()
    for name, ref in (("wfc_0_final", ground), ("wfc_ev_final", final)):
        got = read_wfc(tmp_path, name, 0, shape)
        assert np.isfinite(ref).all(), name
        assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref), name


def test_potential_table_requires_a_full_grid():
    import gpue_b200 as G
    c = dict(cases.DEFAULTS, dim=2, n=32, box=6.0)
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        with pytest.raises(ValueError):
            s.set_potential_table(np.zeros(10))
    assert G.lib().gpue_set_potential_table(None, None) == 1
