"""The CPU oracle against GPUE's own CUDA build (golden fixtures).

The fixtures were produced by tests/golden/make_golden.py running the
reference's parseArgs/init/set_variables/evolve/energy_calc on a B200.  This
pins the FP64 restatement before it is trusted as the checker.  The vortex
fixtures come from the same build's host-side Tracker::findVortex.
"""
import os

import numpy as np
import pytest

import cases
from helpers import GOLDEN, l2, load_golden, oracle_problem, steps_gstate


@pytest.mark.parametrize("name", cases.FIXTURES)
def test_oracle_matches_reference_build(name):
    ref, meta = load_golden(name)
    c = cases.case(name)
    psi0 = cases.initial_psi(c)
    assert meta["input_sha"] == cases.checksum(psi0), "seeded input changed"
    P = oracle_problem(c)
    steps, gs = steps_gstate(c)
    out, res, en = P.evolve(psi0, steps, gs)
    assert res["steps_done"] == steps
    assert l2(out, ref, c) <= 1e-12
    E = P.energy(out)
    assert abs(E - meta["energy"]) <= 1e-12 * abs(meta["energy"])
    assert abs(en[-1] - meta["last_check_energy"]) <= 1e-12 * abs(meta["last_check_energy"])


def test_oracle_linear_ground_state_energy():
    """evolve_test (src/unit_test.cu:1162-1278): linear harmonic ground state
    energy d/2 hbar omega within 1%, then conserved in real time within 1%."""
    for dim in (2, 3):
        c = dict(cases.DEFAULTS, dim=dim, n=32, box=5.0, seed=3, init="gauss")
        psi0 = cases.initial_psi(c)
        import oracle
        P = oracle.Problem(dim, 32, 5.0, g=0.0, gpe=False, gauge=True, omega=0.0, gdt=1e-3,
                           dt=1e-3, energy_every=500, threshold=1e-4)
        out, res, en = P.evolve(psi0, 30001, 0)
        assert res["early_stop"] == 1
        assert abs(res["energy"] - dim / 2) <= 0.01 * dim / 2
        out2, res2, en2 = P.evolve(out, 2001, 1)
        assert abs(res2["energy"] - res["energy"]) <= 0.01 * dim / 2


def test_oracle_fft_kats():
    """Impulse, single mode and Parseval for the oracle's own DFT."""
    import oracle
    rng = np.random.default_rng(0)
    for n in (16, 32, 96, 128, 160, 192, 384):
        x = np.zeros(n, complex)
        x[0] = 1
        assert np.allclose(oracle.fft1d(x, -1), np.ones(n), atol=1e-15)
        k = 3
        m = np.exp(2j * np.pi * k * np.arange(n) / n)
        X = oracle.fft1d(m, -1)
        e = np.zeros(n, complex)
        e[k] = n
        assert np.allclose(X, e, atol=1e-12)
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        Y = oracle.fft1d(y, -1)
        assert abs(np.sum(abs(Y) ** 2) / n - np.sum(abs(y) ** 2)) <= 1e-12 * np.sum(abs(y) ** 2)
        assert np.allclose(Y, np.fft.fft(y), atol=1e-12 * n)
        assert np.allclose(oracle.fft1d(Y, +1) / n, y, atol=1e-14)


@pytest.mark.parametrize("name", sorted(cases.VORTEX_CASES))
def test_oracle_find_vortex_matches_reference(name):
    """The findVortex restatement against markers written by GPUE's own
    Tracker::findVortex (make_golden.py --vortex)."""
    import json
    import oracle
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(d["meta"]))
    v = cases.VORTEX_CASES[name]
    psi = cases.vortex_psi(v)
    assert cases.checksum(psi) == meta["input_sha"]
    marker, winding, found = oracle.find_vortex(psi, cases.grid_x(v["n"], v["box"]),
                                                v["radius"])
    assert found == meta["found"]
    assert np.array_equal(marker, d["marker"].astype(np.int32))
    assert np.array_equal(np.abs(winding), marker)
