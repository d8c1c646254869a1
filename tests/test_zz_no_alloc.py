"""fx_mean_P_noalloc: the mean-polarization reduction for callers that cannot
allocate device memory where they need it (another allocator owns the memory,
or a cudaMalloc would synchronise work they keep in flight).  It must agree
with the context entry point fx_mean_P on two calls in a row, allocating
nothing itself: the device buffers here belong to the test (torch)."""
import ctypes as C

import numpy as np
import pytest

from ferrox_b200 import api, decks

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_mean_P_noalloc_matches_fx_mean_P_twice():
    import torch
    f = api.FerroX(decks.mfim(32, 32, 24, Phi_Bc_hi=0.4))
    f.step(2)
    L = api.lib()
    mask = torch.tensor(f.field("mask").astype(np.uint8).ravel(), device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        Pz = torch.tensor(f.field("Pz").ravel(), device="cuda")
        rc = L.fx_mean_P_noalloc(None, None, _ptr(Pz), _ptr(mask), f.N, _ptr(out), stream)
        assert rc == 0, L.fx_create_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = f.mean_P()
        assert abs(got[2] - ref[2]) <= 1e-12 * max(abs(ref[2]), 1e-30), (got, ref)
        assert got[0] == 0.0 and got[1] == 0.0
        f.step(1)     # the next call sees a different P
    f.close()


def test_mean_P_noalloc_rejects_too_many_cells():
    import torch
    L = api.lib()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    m = torch.zeros(4, dtype=torch.uint8, device="cuda")
    rc = L.fx_mean_P_noalloc(None, None, _ptr(x), _ptr(m), 1 << 25, _ptr(x), None)
    assert rc == -1
    assert b"exceeds" in L.fx_create_error()
