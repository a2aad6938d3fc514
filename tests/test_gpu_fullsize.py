"""The headline configurations at full size against GPUE's own CUDA build.

tests/golden/<case>_digest.npz hold a digest of GPUE's final state on the
1024^2 rotating real-time case (Omega = 0.7 gauge, g = 500, dt = 5e-5, 1000
steps) and the 256^3 anisotropic ground state (g = 1000, gdt = 1e-4, 100
steps), both from the seeded inputs of cases.py (make_golden.py --digest):
its energy, sum |psi|^2 dV, the L2 norm of every row (2D) or z-plane (3D) and
4096 values at seeded indices.  The step being pinned is evolve()'s
(src/evolution.cu:727-870).

Plain FP64 form: energy and norm within 1e-12 relative, every row/plane norm
within 1e-12 of the total, and the sampled values within 1e-12 in L2 (the
sample's squared error scaled up to the whole grid).  Fused FP32 form: energy
within 1e-6 relative.
"""
import json
import os

import numpy as np
import pytest

import cases
from helpers import GOLDEN, dV, run_product

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gpue_b200
    return gpue_b200


def load_digest(name):
    path = os.path.join(GOLDEN, name + "_digest.npz")
    d = np.load(path)
    return d, json.loads(str(d["meta"]))


def full_case(name):
    c = cases.case(name)
    c["gsteps" if c["gsteps"] else "esteps"] = cases.DIGESTS[name]
    c["energy_every"] = 0
    return c


@pytest.mark.parametrize("name", list(cases.DIGESTS))
def test_fp64_full_size_matches_reference_build(G, name):
    d, meta = load_digest(name)
    c = full_case(name)
    psi0 = cases.initial_psi(c)
    assert cases.checksum(psi0) == meta["input_sha"]
    psi, E, r = run_product(c, G.PREC_FP64, psi0=psi0)
    del psi0
    assert r["steps_done"] == cases.DIGESTS[name]
    assert abs(E - meta["energy"]) <= 1e-12 * abs(meta["energy"])
    a2 = np.abs(psi) ** 2
    norm = float(a2.sum() * dV(c))
    assert abs(norm - meta["norm"]) <= 1e-12 * meta["norm"]
    slab = np.sqrt(a2.sum(axis=tuple(range(1, psi.ndim))) * dV(c))
    assert np.max(np.abs(slab - d["slab_norms"])) <= 1e-12 * np.sqrt(meta["norm"])
    got = psi.reshape(-1)[d["sample_idx"]]
    scale = psi.size / got.size
    err = float(np.sqrt(np.sum(np.abs(got - d["sample"]) ** 2) * dV(c) * scale))
    assert err <= 1e-12, err


@pytest.mark.parametrize("name", list(cases.DIGESTS))
def test_fp32_full_size_energy_close_to_reference_build(G, name):
    _, meta = load_digest(name)
    c = full_case(name)
    _, E, r = run_product(c, G.PREC_FP32)
    assert r["steps_done"] == cases.DIGESTS[name]
    assert abs(E - meta["energy"]) <= 1e-6 * abs(meta["energy"])
