"""A bounded device wait that runs out, without a fault.

In the XY tile pass of a 3D complex64 step, a y-tile waits (at most 1 s) for
its plane's x-tiles to be stored.  With GPUE_TEST_PLANE_WAIT=1 (a test hook,
read when a context plans its passes) the y-tiles wait for one x-tile more
than a plane has: nothing ever raises the count that far, so every such wait
gives up.  The kernel records it and returns, and gpue_evolve reports
GPUE_ERR_TIMEOUT instead of hanging.  The device stays usable: the same
context answers further calls, and a fresh context in the same process steps
normally and agrees with one that never saw the hook.
"""
import time

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu


def test_plane_wait_runs_out_and_reports_timeout(monkeypatch):
    import gpue_b200 as G
    c = dict(cases.DEFAULTS, dim=3, n=64, box=8.0, wz=2.0, g=100.0, gdt=1e-4, init="gauss",
             seed=801)
    psi0 = cases.initial_psi(c)
    with G.Solver(product_params(c, G.PREC_FP32)) as ref:
        ref.set_wfc(psi0)
        ref.evolve(4, 0)
        psi_ref, E_ref = ref.get_wfc(), ref.energy()

    monkeypatch.setenv("GPUE_TEST_PLANE_WAIT", "1")
    with G.Solver(product_params(c, G.PREC_FP32)) as s:
        monkeypatch.delenv("GPUE_TEST_PLANE_WAIT")
        s.set_wfc(psi0)
        t0 = time.time()
        with pytest.raises(G.GpueError) as e:
            s.evolve(1, 0)
        assert e.value.status == 7  # GPUE_ERR_TIMEOUT
        assert time.time() - t0 < 120  # bounded: about a second per wait
        # the context still answers (its state is not meaningful now)
        assert s.get_wfc().shape == psi0.shape

    with G.Solver(product_params(c, G.PREC_FP32)) as s2:
        s2.set_wfc(psi0)
        s2.evolve(4, 0)
        psi, E = s2.get_wfc(), s2.energy()
    assert abs(E - E_ref) <= 1e-6 * abs(E_ref)
    assert np.sqrt(np.sum(np.abs(psi - psi_ref) ** 2) * dV(c)) <= 1e-5
