"""fx_mean_P_noalloc: the mean-polarization reduction for callers that cannot
allocate device memory where they need it (another allocator owns the memory,
or a cudaMalloc would synchronise work they keep in flight).  It must agree
with the context entry point fx_mean_P on two calls in a row, for the scalar
form (Px = Py = NULL) and for all three components of a vector-P run, and it
must allocate nothing itself: the device buffers here belong to the test
(torch), and the device's free memory does not move across repeated calls."""
import ctypes as C

import numpy as np
import pytest

from ferrox_b200 import api, decks

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _rand_vector_P(shape, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    return [g.uniform(-0.05, 0.05, shape) for _ in range(3)]


@pytest.mark.parametrize("vector", [False, True], ids=["scalar", "vector"])
def test_mean_P_noalloc_matches_fx_mean_P_twice(vector):
    import torch
    extra = {"is_polarization_scalar": 0} if vector else None
    f = api.FerroX(decks.mfim(32, 32, 24, Phi_Bc_hi=0.4, extra=extra))
    if vector:
        f.set_initial_P(*_rand_vector_P(f.shape, 5))
    f.step(2)
    L = api.lib()
    mask = torch.tensor(f.field("mask").astype(np.uint8).ravel(), device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        P = [torch.tensor(f.field(n).ravel(), device="cuda") for n in ("Px", "Py", "Pz")]
        px, py = (_ptr(P[0]), _ptr(P[1])) if vector else (None, None)
        rc = L.fx_mean_P_noalloc(px, py, _ptr(P[2]), _ptr(mask), f.N, _ptr(out), stream)
        assert rc == 0, L.fx_create_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = f.mean_P()
        for d in range(3) if vector else (2,):
            assert abs(got[d] - ref[d]) <= 1e-12 * max(abs(ref[d]), 1e-30), (d, got, ref)
        if vector:
            assert got[0] != 0.0 and got[1] != 0.0
        else:
            assert got[0] == 0.0 and got[1] == 0.0
        f.step(1)     # the next call sees a different P
    f.close()


def test_mean_P_noalloc_leaves_free_memory_unchanged():
    import torch
    L = api.lib()
    n = 1 << 20
    Pz = torch.ones(n, dtype=torch.float64, device="cuda")
    mask = torch.zeros(n, dtype=torch.uint8, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.fx_mean_P_noalloc(None, None, _ptr(Pz), _ptr(mask), n, _ptr(out), stream) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert L.fx_mean_P_noalloc(None, None, _ptr(Pz), _ptr(mask), n, _ptr(out), stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert out.cpu().numpy()[2] == 1.0


def test_mean_P_noalloc_rejects_too_many_cells():
    import torch
    L = api.lib()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    m = torch.zeros(4, dtype=torch.uint8, device="cuda")
    rc = L.fx_mean_P_noalloc(None, None, _ptr(x), _ptr(m), 1 << 25, _ptr(x), None)
    assert rc == -1
    assert b"exceeds" in L.fx_create_error()
