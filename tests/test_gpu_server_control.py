"""The serving loop's control paths: admission while a tick runs, request
deadlines and cancellation.

- A request submitted while a tick is running on the device is admitted
  during that tick (server stats count it) and gives the bit-identical result
  of the same request served alone.
- A request whose deadline passes leaves with GPUE_ERR_TIMEOUT: at once when
  still queued, or after the tick in flight when resident, with its state at
  that tick written out (a whole number of ticks run, state normalised as a
  real-time solve keeps it).
- gpue_server_cancel removes a queued request at once and a resident one
  after the tick in flight (GPUE_ERR_CANCELLED); an unknown tag is an error.
"""

import time

import numpy as np
import pytest

import cases
from helpers import dV, product_params

pytestmark = pytest.mark.gpu

TIMEOUT, CANCELLED = 7, 8

LONG = dict(cases.DEFAULTS, dim=2, n=256, box=10.0, g=200.0, omega=0.3, gauge=True, dt=5e-5,
            seed=401, init="phase")
# long ticks (100 steps of 512^2, a few ms), so a submission lands inside one
BIG = dict(cases.DEFAULTS, dim=2, n=512, box=12.0, g=200.0, omega=0.3, gauge=True, dt=5e-5,
           seed=403, init="phase")
PROBE = dict(cases.DEFAULTS, dim=2, n=64, box=8.0, g=150.0, omega=0.5, gauge=True,
             gdt=5e-3, seed=402, init="gauss")


def wait_results(srv, n, limit=120.0):
    out = {}
    t_end = time.time() + limit
    while len(out) < n and time.time() < t_end:
        for r in srv.poll(timeout=0.5):
            out[r["tag"]] = r
    return out


def wait_for(pred, limit=60.0):
    t_end = time.time() + limit
    while time.time() < t_end:
        if pred():
            return True
        time.sleep(0.002)
    return False


@pytest.mark.parametrize("prec", [0, 1])
def test_request_admitted_during_a_tick_matches_it_alone(prec):
    import gpue_b200 as G
    with G.Server(precision=prec, check_steps=100, threshold=1e-8) as srv:
        srv.submit(product_params(PROBE, prec), 0, 1000, cases.initial_psi(PROBE), 0)
        alone = wait_results(srv, 1)[0]
    assert alone["status"] == 0
    with G.Server(precision=prec, check_steps=100, threshold=1e-8) as srv:
        # a long real-time solve keeps ticks running; the probe arrives mid-run
        srv.submit(product_params(BIG, prec), 1, 20000, cases.initial_psi(BIG), 1)
        assert wait_for(lambda: srv.stats()["ticks"] >= 2)
        srv.submit(product_params(PROBE, prec), 0, 1000, cases.initial_psi(PROBE), 0)
        probe = wait_results(srv, 1)
        st = srv.stats()
        srv.cancel(1)
        rest = wait_results(srv, 1)
    assert st["admitted_in_tick"] >= 1
    m = probe[0]
    assert m["status"] == 0
    assert m["steps_done"] == alone["steps_done"] and m["energy"] == alone["energy"]
    assert np.array_equal(m["psi"], alone["psi"])
    assert rest[1]["status"] == CANCELLED


def test_deadline_of_a_resident_solve():
    import gpue_b200 as G
    prec = G.PREC_FP32
    with G.Server(precision=prec, check_steps=50) as srv:
        srv.submit(product_params(LONG, prec), 1, 200000, cases.initial_psi(LONG), 5,
                   deadline=0.5)
        r = wait_results(srv, 1)[5]
        st = srv.stats()
    assert r["status"] == TIMEOUT
    assert 0 < r["steps_done"] < 200000 and r["steps_done"] % 50 == 0
    assert r["t_done"] - r["t_submit"] >= 0.5
    norm = float(np.sum(np.abs(r["psi"]) ** 2) * dV(LONG))
    assert norm == pytest.approx(1.0, rel=1e-5)
    assert st["timed_out"] == 1 and st["active"] == 0


def test_deadline_and_cancel_of_queued_requests():
    import gpue_b200 as G
    prec = G.PREC_FP32
    with G.Server(precision=prec, check_steps=50, max_active=1) as srv:
        srv.submit(product_params(LONG, prec), 1, 200000, cases.initial_psi(LONG), 1)
        assert wait_for(lambda: srv.stats()["active"] == 1)
        # both wait behind the long solve (one slot)
        srv.submit(product_params(PROBE, prec), 0, 1000, cases.initial_psi(PROBE), 2,
                   deadline=0.2)
        srv.submit(product_params(PROBE, prec), 0, 1000, cases.initial_psi(PROBE), 3)
        srv.cancel(3)
        got = wait_results(srv, 2, limit=30.0)
        with pytest.raises(G.GpueError):
            srv.cancel(99)
        srv.cancel(1)
        got.update(wait_results(srv, 1))
        st = srv.stats()
    assert got[3]["status"] == CANCELLED and got[3]["steps_done"] == 0
    assert got[2]["status"] == TIMEOUT and got[2]["steps_done"] == 0
    assert got[1]["status"] == CANCELLED and got[1]["steps_done"] > 0
    assert np.isfinite(got[1]["psi"]).all()
    assert st["cancelled"] == 2 and st["timed_out"] == 1
    assert st["active"] == 0 and st["queued"] == 0
