"""The gpue command line: GPUE's flags, init()'s derived values, its initial
state and its text files, checked without a GPU (nothing here creates a
device context: --print-params stops before, and -g 0 -e 0 never steps)."""

import math
import os

import numpy as np
import pytest

from cli_helpers import params, read_wfc, run, write_wfc

HBAR, MASS, AS, PI = 1.05457148e-34, 1.4431607e-25, 4.76e-9, 3.141592653589793


def derived(dim, wx=6.283, wy=6.283, wz=6.283, atoms=1, box=None):
    """init()'s formulas (src/init.cu:98-170)."""
    a0 = [math.sqrt(HBAR / (2 * MASS * w)) for w in (wx, wy, wz)]
    g = atoms * 4 * HBAR * HBAR * PI * (AS / MASS)
    if dim == 2:
        g *= math.sqrt(MASS * wz / (2 * PI * HBAR))
    rxy = 15 ** 0.2 * (atoms * AS * math.sqrt(MASS * wz / HBAR)) ** 0.2
    xmax = [box] * 3 if box else [6 * rxy * a for a in a0]
    return dict(gDenConst=g, xMax=xmax[0], yMax=xmax[1], zMax=xmax[2], Rxy=rxy, a0=a0)


def test_defaults_are_gpues(tmp_path):
    import gpue_b200 as G
    p = params([], tmp_path)
    d = derived(2)
    assert p["dimnum"] == 2 and p["xDim"] == 256 and p["yDim"] == 256 and p["zDim"] == 1
    assert p["gsteps"] == 1 and p["esteps"] == 1
    assert math.isclose(p["xMax"], d["xMax"], rel_tol=1e-15)
    assert math.isclose(p["gDenConst"], d["gDenConst"], rel_tol=1e-15)
    assert p["hbar"] == HBAR and p["mass"] == MASS and p["gdt"] == 1e-4 and p["dt"] == 1e-4
    assert p["gpe"] == 0 and p["corotating"] == 0 and p["precision"] == 0
    ref = G.default_params()  # the ABI's defaults agree with the command line's
    assert math.isclose(ref.xMax, p["xMax"], rel_tol=1e-15)
    assert math.isclose(ref.gDenConst, p["gDenConst"], rel_tol=1e-15)


def test_flags_map_to_parameters(tmp_path):
    p = params(["-x", 128, "-y", 128, "-w", 0.6, "-s", "-l", "-i", 250, "-T", 2e-4,
                "-t", 5e-5, "-X", 10.0, "-Y", 12.0, "-Z", 30.0, "-G", 1.1, "-g", 300, "-e", 40,
                "-A", "constant", "-R", 2, "-E", 1e-7, 25, "--precision=fp32"], tmp_path)
    assert p["xDim"] == 128 and p["omega"] == 0.6 and p["gpe"] == 1 and p["corotating"] == 1
    assert p["interaction"] == 250 and p["gdt"] == 2e-4 and p["dt"] == 5e-5
    assert p["omegaX"] == 10.0 and p["omegaY"] == 12.0 and p["omegaZ"] == 30.0
    assert p["gammaY"] == 1.1 and p["gsteps"] == 300 and p["esteps"] == 40
    assert p["gauge"] == 1 and p["ramp"] == 1 and p["ramp_type"] == 2 and p["precision"] == 1
    assert p["energy_calc_steps"] == 25 and p["energy_calc_threshold"] == 1e-7
    d = derived(2, 10.0, 12.0, 30.0)
    assert math.isclose(p["xMax"], d["xMax"], rel_tol=1e-15)
    assert math.isclose(p["yMax"], d["yMax"], rel_tol=1e-15)
    assert math.isclose(p["gDenConst"], d["gDenConst"], rel_tol=1e-15)


def test_three_dimensions_take_gpues_box_and_coupling(tmp_path):
    p = params(["-c", 3, "-x", 64, "-y", 64, "-z", 64], tmp_path)
    d = derived(3, box=2.5e-5)
    assert p["dimnum"] == 3 and p["zDim"] == 64
    assert p["xMax"] == 2.5e-5 and p["zMax"] == 2.5e-5
    assert math.isclose(p["gDenConst"], d["gDenConst"], rel_tol=1e-15)  # no 2D factor
    p = params(["-c", 3, "-b", 1e-5, "-x", 32, "-y", 32, "-z", 32], tmp_path)
    assert p["xMax"] == 1e-5  # -b after -c wins, as in GPUE


def test_initial_state_and_files(tmp_path):
    """-g 0 -e 0 writes Params.dat, WFC_0 and the axes without stepping."""
    n = 32
    run(["-x", n, "-y", n, "-g", 0, "-e", 0, "-L", 1.0], tmp_path)
    for f in ("Params.dat", "WFC_0", "WFCi_0", "x_0", "y_0", "z_0"):
        assert os.path.exists(os.path.join(tmp_path, f)), f
    text = open(os.path.join(tmp_path, "Params.dat")).read()
    assert text.startswith("[Params]\n") and "xDim=32" in text and "gDenConst=" in text
    psi = read_wfc(tmp_path, "WFC", 0, (n, n))
    # kstd_wfc with winding 1, then init()'s normalisation by sqrt(sum|psi| dV)
    d = derived(2)
    dx = d["xMax"] / (n >> 1)
    x = -d["xMax"] + dx * np.arange(n)
    X, Y = x[None, :], x[:, None]
    phi = -np.fmod(1.0 * np.arctan2(Y, X), 2 * PI)
    e = np.exp(-(X ** 2 / (d["Rxy"] ** 2 * d["a0"][0] ** 2) +
                 Y ** 2 / (d["Rxy"] ** 2 * d["a0"][1] ** 2)))
    ref = e * np.cos(phi) - 1j * e * np.sin(phi)
    ref = ref / np.sqrt(np.sum(np.abs(ref)) * dx * dx)
    assert np.allclose(psi, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    np.testing.assert_allclose(np.loadtxt(os.path.join(tmp_path, "x_0")), x, rtol=0,
                               atol=1e-20)


def test_read_wfc_files(tmp_path):
    n = 16
    psi = (np.arange(n * n) + 1j * np.arange(n * n)[::-1]).reshape(n, n) * 1e-3
    write_wfc(tmp_path, psi)
    run(["-x", n, "-y", n, "-g", 0, "-e", 0, "-r"], tmp_path)
    np.testing.assert_array_equal(read_wfc(tmp_path, "WFC", 0, (n, n)), psi)


@pytest.mark.parametrize("args,msg", [
    (["-r"], "wfc_load"),                       # -r without the input files
    (["-A", "file"], "Axgauge"),                # -A file without the gauge files
    (["-A", "spiral"], "gauge field"),
    (["-v", "box"], "potential"),
    (["-A", "ring", "-I", "params.cfg"], "params.cfg"),
    (["-c", 1], "2D and 3D"),
    (["--no-such-option"], "unknown option"),
])
def test_errors_exit_with_a_message(tmp_path, args, msg):
    p = run(args + ["-g", 0, "-e", 0], tmp_path, check=False)
    assert p.returncode == 1 and msg in p.stderr
