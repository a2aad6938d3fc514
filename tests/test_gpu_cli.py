"""The gpue command line on the GPU: GPUE's main() flow (imaginary then real
time, sliced at printSteps writes and energy checks) must leave the same
states as the library stepped in one call each, and write GPUE's files."""

import os

import numpy as np
import pytest

from cli_helpers import params, read_wfc, run

pytestmark = pytest.mark.gpu

FIELDS = ("dimnum", "xDim", "yDim", "zDim", "xMax", "yMax", "zMax", "hbar", "mass", "omegaX",
          "omegaY", "omegaZ", "gammaY", "omega", "interaction", "gDenConst", "gdt", "dt", "gpe",
          "corotating", "gauge", "ramp", "ramp_type", "precision")


def lib_params(p):
    import gpue_b200 as G
    prm = G.default_params()
    for k in FIELDS:
        setattr(prm, k, p[k])
    return prm


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_cli_states_match_the_library(tmp_path, prec, tol):
    import gpue_b200 as G
    n = 64
    args = ["-x", n, "-y", n, "-s", "-l", "-w", 0.5, "-i", 200, "-g", 120, "-e", 60, "-W",
            "-p", 50, "-E", 1e-30, 40, "--precision=" + prec]
    run(args, tmp_path)
    p = params(args, tmp_path)
    psi0 = read_wfc(tmp_path, "WFC", 0, (n, n))
    with G.Solver(lib_params(p)) as s:
        s.set_wfc(psi0)
        s.evolve(50, 0)
        at50 = s.get_wfc()
        s.evolve(70, 0, step_offset=50)
        ground = s.get_wfc()
        s.evolve(60, 1)
        final = s.get_wfc()
    assert rel_l2(read_wfc(tmp_path, "wfc_0_const", 50, (n, n)), at50) <= tol
    assert rel_l2(read_wfc(tmp_path, "wfc_0_final", 0, (n, n)), ground) <= tol
    assert rel_l2(read_wfc(tmp_path, "wfc_ev_final", 0, (n, n)), final) <= tol
    for f in ("wfc_0_const_0", "wfc_0_const_100", "wfc_ev_0", "wfc_ev_50"):
        assert os.path.exists(os.path.join(tmp_path, f)), f
    # checks at steps 0, 40 and 80 of each phase (a 1e-30 threshold never stops early)
    assert len(np.loadtxt(os.path.join(tmp_path, "energyi.dat"))) == 3
    assert len(np.loadtxt(os.path.join(tmp_path, "energy.dat"))) == 2


def test_cli_early_stop_and_autotune(tmp_path):
    """GPUE's relative early-stop rule ends the imaginary-time phase."""
    n = 64
    args = ["-x", n, "-y", n, "-s", "-i", 50, "-g", 20000, "-e", 0, "-T", 1e-3,
            "-E", 1e-6, 100, "--autotune"]
    out = run(args, tmp_path).stdout
    assert "Stopping early at step" in out
    E = np.loadtxt(os.path.join(tmp_path, "energyi.dat"))
    assert 2 <= len(E) < 200
    # GPUE writes energyi.dat with 6 significant digits (the stream default),
    # so the last two printed values agree to that precision
    assert abs(E[-1] - E[-2]) <= 1.5e-5 * abs(E[-2])


def test_cli_finds_vortices_at_print_steps(tmp_path):
    """2D real time: findVortex runs on the device at every print step; the
    marks written (vort_mark_<step>) equal the oracle's findVortex on the
    wfc_ev_<step> state written at the same step."""
    import cases
    import oracle
    from cli_helpers import write_wfc
    n, radius_frac = 128, 0.7
    base = ["-x", n, "-y", n, "-s", "-i", 100, "-l", "-w", 0.4, "-g", 0, "-e", 25, "-W",
            "-p", 10, "-r"]
    probe = tmp_path / "probe"
    probe.mkdir()
    xmax = params(["-x", n, "-y", n], probe)["xMax"]
    x = cases.grid_x(n, xmax)
    X, Y = np.meshgrid(x, x)
    psi = np.exp(-(X ** 2 + Y ** 2) / (0.4 * xmax) ** 2).astype(np.complex128)
    rng = np.random.Generator(np.random.PCG64(77))
    for (xk, yk), q in zip((rng.random((6, 2)) - 0.5) * 0.8 * xmax, (1, -1, 1, 1, -1, 1)):
        psi *= (X - xk) + 1j * q * (Y - yk)
    psi /= np.sqrt(np.sum(np.abs(psi) ** 2) * (x[1] - x[0]) ** 2)
    write_wfc(tmp_path, psi)
    radius = radius_frac * xmax
    out = run(base + ["-m", radius], tmp_path).stdout
    located = [int(l.split()[1]) for l in out.splitlines() if l.startswith("Located")]
    assert len(located) == 3  # steps 0, 10, 20
    for k, step in enumerate((0, 10, 20)):
        state = read_wfc(tmp_path, "wfc_ev", step, (n, n))
        marker, winding, found = oracle.find_vortex(state, x, radius)
        rows = np.loadtxt(tmp_path / ("vort_mark_%d" % step), delimiter=",", comments="#",
                          dtype=np.int64, ndmin=2)
        assert found == located[k] == len(rows) > 0
        ii, jj = np.nonzero(marker)
        assert np.array_equal(rows[:, 0], ii) and np.array_equal(rows[:, 1], jj)
        assert np.array_equal(rows[:, 2], marker[ii, jj])
        assert np.array_equal(rows[:, 3], winding[ii, jj])
