"""The device vortex finder (gpue_find_vortices) against GPUE's own
Tracker::findVortex (golden markers) and the oracle's restatement of it, on
imprinted, random-phase and evolved states, in both precisions, with host and
device outputs."""

import json
import os

import numpy as np
import pytest

import cases
from helpers import GOLDEN, product_params

pytestmark = pytest.mark.gpu


def solver_for(n, box, precision=None, dim=2):
    import gpue_b200 as G
    prec = G.PREC_FP64 if precision is None else precision
    return G.Solver(G.make_params(dim, n, box, precision=prec))


def oracle_marks(psi, n, box, radius):
    import oracle
    return oracle.find_vortex(psi, cases.grid_x(n, box), radius)


def check_list(lst, marker, winding, found):
    ii, jj = np.nonzero(marker)  # row-major: findVortex's visiting order
    assert len(lst) == found == len(ii)
    assert np.array_equal(lst["i"], ii) and np.array_equal(lst["j"], jj)
    assert np.array_equal(lst["marker"], marker[ii, jj])
    assert np.array_equal(lst["winding"], winding[ii, jj])


@pytest.mark.parametrize("name", sorted(cases.VORTEX_CASES))
def test_matches_reference_markers(name):
    v = cases.VORTEX_CASES[name]
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(d["meta"]))
    psi = cases.vortex_psi(v)
    with solver_for(v["n"], v["box"]) as s:
        s.set_wfc(psi)
        marker, lst, found = s.find_vortices(v["radius"])
        again = s.find_vortices(v["radius"])
    assert found == meta["found"]
    assert np.array_equal(marker, d["marker"].astype(np.int32))
    _, winding, _ = oracle_marks(psi, v["n"], v["box"], v["radius"])
    check_list(lst, marker, winding, found)
    assert again[2] == found and np.array_equal(again[0], marker)


def test_fp32_state_matches_oracle():
    import gpue_b200 as G
    v = cases.VORTEX_CASES["vtx_imprint_n256"]
    psi = cases.vortex_psi(v).astype(np.complex64)
    with solver_for(v["n"], v["box"], G.PREC_FP32) as s:
        s.set_wfc(psi)
        marker, lst, found = s.find_vortices(v["radius"])
    m_ref, w_ref, f_ref = oracle_marks(psi.astype(np.complex128), v["n"], v["box"], v["radius"])
    assert found == f_ref and np.array_equal(marker, m_ref)
    check_list(lst, marker, w_ref, found)


@pytest.mark.parametrize("gs", [0, 1])
def test_evolved_rotating_state(gs):
    """A state with imprinted vortices evolved in the rotating frame; the
    finder sees the same state get_wfc returns (imaginary time included,
    whose renormalisation is applied first)."""
    import gpue_b200 as G
    v = dict(cases.VORTEX_CASES["vtx_imprint_n128"], seed=41)
    c = dict(cases.DEFAULTS, dim=2, n=v["n"], box=v["box"], g=200.0, omega=0.6, gauge=True,
             dt=5e-5)
    with G.Solver(product_params(c, G.PREC_FP64)) as s:
        s.set_wfc(cases.vortex_psi(v))
        s.evolve(60, gs)
        marker, lst, found = s.find_vortices(v["radius"])
        psi = s.get_wfc()
    m_ref, w_ref, f_ref = oracle_marks(psi, v["n"], v["box"], v["radius"])
    assert found == f_ref > 0
    assert np.array_equal(marker, m_ref)
    check_list(lst, marker, w_ref, found)


def test_large_random_phase_grid():
    """1024^2 random phases: ~1/3 of the plaquettes wind, in long runs of
    neighbours, across every 32-column chunk of a row."""
    n, box, radius = 1024, 10.0, 9.5
    rng = np.random.Generator(np.random.PCG64(42))
    psi = (0.5 + rng.random((n, n))) * np.exp(2j * np.pi * rng.random((n, n)))
    with solver_for(n, box) as s:
        s.set_wfc(psi)
        marker, lst, found = s.find_vortices(radius)
    m_ref, w_ref, f_ref = oracle_marks(psi, n, box, radius)
    assert found == f_ref > 100000
    assert np.array_equal(marker, m_ref)
    check_list(lst, marker, w_ref, found)


def test_device_outputs_and_capacity():
    import ctypes
    import torch
    import gpue_b200 as G
    v = cases.VORTEX_CASES["vtx_noise_n64"]
    psi = cases.vortex_psi(v)
    n = v["n"]
    with solver_for(n, v["box"]) as s:
        s.set_wfc(psi)
        marker, lst, found = s.find_vortices(v["radius"])
        dm = torch.full((n, n), -7, dtype=torch.int32, device="cuda:0")
        dl = torch.zeros((found, 4), dtype=torch.int32, device="cuda:0")
        f = ctypes.c_int32()
        st = G.lib().gpue_find_vortices(s._h, v["radius"], ctypes.c_void_p(dm.data_ptr()),
                                        G.MEM_DEVICE, ctypes.c_void_p(dl.data_ptr()), found,
                                        ctypes.byref(f))
        assert st == 0 and f.value == found
        torch.cuda.synchronize()
        assert np.array_equal(dm.cpu().numpy(), marker)
        got = dl.cpu().numpy()
        assert np.array_equal(got[:, 0], lst["i"]) and np.array_equal(got[:, 3], lst["winding"])
        # a short list keeps the first marks in visiting order; found is the full count
        m3, l3, f3 = s.find_vortices(v["radius"], cap=3)
        assert f3 == found and len(l3) == 3 and np.array_equal(l3, lst[:3])
        _, l0, f0 = s.find_vortices(v["radius"], cap=0)
        assert f0 == found and len(l0) == 0
        # nothing is within a zero radius
        mz, lz, fz = s.find_vortices(0.0)
        assert fz == 0 and not mz.any() and len(lz) == 0


def test_argument_and_dimension_errors():
    import ctypes
    import gpue_b200 as G
    with solver_for(16, 6.0, dim=3) as s:
        s.set_wfc(np.ones((16, 16, 16), np.complex128))
        with pytest.raises(G.GpueError) as e:
            s.find_vortices(1.0)
        assert e.value.status == 2
    with solver_for(64, 6.0) as s:
        s.set_wfc(np.ones((64, 64), np.complex128))
        f = ctypes.c_int32()
        assert G.lib().gpue_find_vortices(s._h, 1.0, None, 5, None, 0, ctypes.byref(f)) == 1
        assert G.lib().gpue_find_vortices(s._h, 1.0, None, 0, None, 4, ctypes.byref(f)) == 1
        assert G.lib().gpue_find_vortices(s._h, 1.0, None, 0, None, 0, ctypes.byref(f)) == 0
        assert f.value == 0
