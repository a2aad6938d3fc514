"""The product library loads and exports the C ABI declared in include/*.h.

No compute calls here: these run without a GPU.
"""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(gpue_[a-z0-9_]+)\s*\(", src):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    import gpue_b200
    L = gpue_b200.lib()
    syms = declared_symbols()
    assert "gpue_evolve" in syms and "gpue_ctx_create" in syms
    missing = [s for s in sorted(syms) if not hasattr(L, s)]
    assert not missing, missing


def test_abi_version_and_defaults():
    import gpue_b200 as G
    assert G.lib().gpue_abi_version() == 2
    p = G.default_params()
    # parseArgs defaults (src/parser.cu:14-67)
    assert (p.xDim, p.yDim, p.dimnum) == (256, 256, 2)
    assert p.omegaX == 6.283 and p.omegaY == 6.283 and p.omegaZ == 6.283
    assert p.gdt == 1e-4 and p.dt == 1e-4 and p.interaction == 1.0
    assert abs(p.hbar - 1.05457148e-34) < 1e-45 and abs(p.mass - 1.4431607e-25) < 1e-35


def test_supported_lengths():
    import gpue_b200 as G
    for n in (16, 32, 64, 96, 128, 160, 192, 256, 320, 384, 512, 640, 768, 1024):
        assert G.supported_length(n, G.PREC_FP64) and G.supported_length(n, G.PREC_FP32)
    for n in (7, 100, 2048):
        assert not G.supported_length(n, G.PREC_FP64)


def test_invalid_arguments_fail_without_touching_the_device():
    import gpue_b200 as G
    L = G.lib()
    h = ctypes.c_void_p()
    bad = G.make_params(2, 64, 8.0)
    bad.yDim = 32  # non-square grids are rejected (GPUE's gauge plans need square)
    assert L.gpue_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    bad = G.make_params(4, 64, 8.0)
    assert L.gpue_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    bad = G.make_params(2, 100, 8.0)  # no FFT plan for 100
    assert L.gpue_ctx_create(ctypes.byref(bad), ctypes.byref(h)) == 2
    assert L.gpue_evolve(None, 1, 0, None, None) == 1
    assert L.gpue_set_operators(None, 0) == 1
    obs = G.Observables()
    assert L.gpue_observables_get(None, ctypes.byref(obs)) == 1
    assert L.gpue_find_vortices(None, 1.0, None, 0, None, 0, None) == 1
    assert L.gpue_snapshot_save(None, b"x", 0, 0) == 1
    assert L.gpue_snapshot_load(None, b"x", None, None) == 1
    # batches: argument checks come before any device call
    out = ctypes.c_void_p()
    assert L.gpue_batch_create(None, 1, ctypes.byref(out)) == 1
    arr = (ctypes.c_void_p * 2)(None, None)
    assert L.gpue_batch_create(arr, 2, ctypes.byref(out)) == 1
    assert L.gpue_batch_create(arr, 0, ctypes.byref(out)) == 1
    assert L.gpue_batch_evolve(None, 0, None, None, None) == 1
    assert L.gpue_batch_destroy(None) == 0
    assert L.gpue_batch_last_error(None) == b""


def test_server_arguments_fail_without_touching_the_device():
    import gpue_b200 as G
    L = G.lib()
    h = ctypes.c_void_p()
    o = G.ServerOpts()
    o.precision, o.check_steps = G.PREC_FP32, 3  # odd tick lengths are rejected
    assert L.gpue_server_create(ctypes.byref(o), ctypes.byref(h)) == 1
    o.check_steps, o.precision = 100, 7
    assert L.gpue_server_create(ctypes.byref(o), ctypes.byref(h)) == 1
    assert L.gpue_server_create(None, ctypes.byref(h)) == 1
    assert L.gpue_server_submit(None, None) == 1
    n = ctypes.c_int32()
    assert L.gpue_server_poll(None, None, 0, ctypes.byref(n), 0.0) == 1
    assert L.gpue_server_destroy(None) == 0
    assert L.gpue_server_last_error(None) == b""
