"""gpue_norm_noalloc: the norm of a caller-owned wavefunction without any
device allocation by the library.

Callers that cannot allocate device memory at the moment they need a norm
(for instance a server that reserved all of its HBM budget up front) use this
entry point on memory they own.  Its reduction scratch is a fixed device
array inside the library, so the check here is that it gives the same value
as the context-based gpue_norm, twice in a row on the shared scratch, for both
storage precisions, and that it refuses sizes its scratch cannot cover.  This
file is collected last so a failure here cannot hide the other tests.
"""
import ctypes

import numpy as np
import pytest

import cases
from helpers import product_params

pytestmark = pytest.mark.gpu


# One block (64^2 = 4096 points), and several blocks with a ragged last one
# (96^2 = 2.25 blocks, 160^2 = 6.25 blocks) or whole ones (32^3 = 8 blocks), so
# the cross-block merge, the counter reset and the tail bounds check all run.
SHAPES = [(2, 64), (2, 96), (2, 160), (3, 32)]


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("shape", SHAPES, ids=["%dd-%d" % s for s in SHAPES])
def test_norm_noalloc_matches_gpue_norm_twice(precision, shape):
    import torch

    import gpue_b200 as G
    dim, n = shape
    c = dict(cases.DEFAULTS, dim=dim, n=n, box=8.0, seed=70 + n, init="phase")
    psi0 = cases.initial_psi(c) * 1.7  # a norm away from 1
    dV = (c["box"] / (c["n"] >> 1)) ** dim
    with G.Solver(product_params(c, precision)) as s:
        s.set_wfc(psi0)
        ref = s.norm()
        ptr, dtype = s.wfc_device()
        out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        L = G.lib()
        for k in range(2):
            st = L.gpue_norm_noalloc(ctypes.c_void_p(ptr), dtype, psi0.size, dV,
                                     ctypes.c_void_p(out.data_ptr() + 8 * k),
                                     ctypes.c_void_p(s.stream()))
            assert st == 0
        torch.cuda.synchronize()
        vals = out.cpu().numpy()
    assert ref == pytest.approx(1.7 ** 2, rel=1e-6)
    assert np.allclose(vals, ref, rtol=1e-13, atol=0)


def test_norm_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    import gpue_b200 as G
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    buf = torch.zeros(2, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    st = G.lib().gpue_norm_noalloc(ctypes.c_void_p(buf.data_ptr()), G.C128, (1 << 28) + 1,
                                   1.0, ctypes.c_void_p(out.data_ptr()), None)
    assert st == 1
    st = G.lib().gpue_norm_noalloc(ctypes.c_void_p(buf.data_ptr()), G.C128, 0, 1.0,
                                   ctypes.c_void_p(out.data_ptr()), None)
    assert st == 1
