"""Binary snapshots (gpue_snapshot_save / gpue_snapshot_load): a resumed run
repeats the uninterrupted one bit for bit, including the pending
imaginary-time renormalisation and the early-stop reference energy; damaged
or mismatched snapshots are refused; the command line's --checkpoint-every /
--resume continue GPUE's main() flow where it stopped."""

import os
import shutil

import numpy as np
import pytest

import cases
from cli_helpers import read_wfc, run
from helpers import product_params

pytestmark = pytest.mark.gpu


def case(**kw):
    c = dict(cases.DEFAULTS, dim=2, n=64, box=8.0, g=200.0, omega=0.5, gauge=True, dt=5e-5,
             seed=801, init="phase")
    c.update(kw)
    return c


def solver(c, prec=None):
    import gpue_b200 as G
    return G.Solver(product_params(c, G.PREC_FP64 if prec is None else prec))


@pytest.mark.parametrize("prec_name", ["fp64", "fp32"])
@pytest.mark.parametrize("gs", [0, 1])
def test_resume_repeats_the_uninterrupted_run(tmp_path, prec_name, gs):
    import gpue_b200 as G
    prec = G.PREC_FP64 if prec_name == "fp64" else G.PREC_FP32
    c = case()
    psi0 = cases.initial_psi(c)
    kw = dict(energy_every=20, threshold=1e-14, norm_guard=0)
    with solver(c, prec) as s:
        s.set_wfc(psi0)
        full = s.evolve(80, gs, **kw)
        want = s.get_wfc()
    path = str(tmp_path / "snap.bin")
    with solver(c, prec) as s:
        s.set_wfc(psi0)
        s.evolve(40, gs, **kw)
        s.save_snapshot(path, gs, 40)
    with solver(c, prec) as s:
        assert s.load_snapshot(path) == (gs, 40)
        rest = s.evolve(40, gs, step_offset=40, **kw)
        got = s.get_wfc()
    assert np.array_equal(got, want)
    assert rest["energy"] == full["energy"]


def test_round_trip_and_precision_change(tmp_path):
    import gpue_b200 as G
    c = case()
    path = str(tmp_path / "s.bin")
    with solver(c) as s:
        s.set_wfc(cases.initial_psi(c))
        s.evolve(25, 0)  # leaves a renormalisation pending
        before = s.get_wfc()
        s.save_snapshot(path, 0, 25)
        E = s.energy()
    with solver(c) as s:
        s.load_snapshot(path)
        assert np.array_equal(s.get_wfc(), before)
        assert s.energy() == E
    # an FP64 snapshot loads into an FP32 context (rounded to complex64)
    with solver(c, G.PREC_FP32) as s:
        s.load_snapshot(path)
        got = s.get_wfc()
    assert np.abs(got - before).max() <= 2e-7 * np.abs(before).max()


def test_damaged_or_foreign_snapshots_are_refused(tmp_path):
    import gpue_b200 as G
    c = case()
    path = tmp_path / "s.bin"
    with solver(c) as s:
        s.set_wfc(cases.initial_psi(c))
        s.save_snapshot(str(path), 1, 7)
    raw = path.read_bytes()
    bad = tmp_path / "bad.bin"
    flipped = bytearray(raw)
    flipped[-100] ^= 0x40
    bad.write_bytes(bytes(flipped))
    short = tmp_path / "short.bin"
    short.write_bytes(raw[:-16])
    magic = tmp_path / "magic.bin"
    magic.write_bytes(b"X" + raw[1:])
    for p, msg in ((bad, "checksum"), (short, "truncated"), (magic, "snapshot"),
                   (tmp_path / "missing.bin", "cannot open")):
        with solver(c) as s:
            with pytest.raises(G.GpueError) as e:
                s.load_snapshot(str(p))
            assert e.value.status == 1 and msg in str(e.value)
    for other in (case(n=32), case(omega=0.4), case(box=9.0)):
        with solver(other) as s:
            with pytest.raises(G.GpueError) as e:
                s.load_snapshot(str(path))
            assert "different" in str(e.value)
    # precision and device are not part of the match
    with solver(c, G.PREC_FP32) as s:
        assert s.load_snapshot(str(path)) == (1, 7)


@pytest.mark.parametrize("where", ["imaginary", "real"])
def test_cli_checkpoint_and_resume(tmp_path, where):
    n = 64
    base = ["-x", n, "-y", n, "-s", "-l", "-w", 0.5, "-i", 200, "-g", 60, "-e", 40]
    full, part, resumed = (tmp_path / d for d in ("full", "part", "resumed"))
    for d in (full, part, resumed):
        d.mkdir()
    run(base + ["--checkpoint-every=20"], full)
    # the last snapshot of a run is at real-time step 20; a run without the
    # real-time phase leaves one at imaginary-time step 40
    if where == "real":
        shutil.copy(full / "snapshot.bin", resumed / "snapshot.bin")
    else:
        run(["-x", n, "-y", n, "-s", "-l", "-w", 0.5, "-i", 200, "-g", 60, "-e", 0,
             "--checkpoint-every=20"], part)
        shutil.copy(part / "snapshot.bin", resumed / "snapshot.bin")
    out = run(base + ["--resume"], resumed).stdout
    assert ("Resuming %s-time evolution at step %d" % (where, 20 if where == "real" else 40)) \
        in out
    names = ["wfc_ev_final"] + (["wfc_0_final"] if where == "imaginary" else [])
    for name in names:
        a = read_wfc(full, name, 0, (n, n))
        b = read_wfc(resumed, name, 0, (n, n))
        assert np.array_equal(a, b), name
    assert not os.path.exists(resumed / "snapshot.bin.tmp")
