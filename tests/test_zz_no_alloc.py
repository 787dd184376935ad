"""The search entry point that allocates nothing (emb200_assign_f32_noalloc).

It serves callers that cannot allocate device memory when they search (their
GPU memory belongs to their own pool or budget, or an allocation could stall or
fail on a latency-critical path): they pass every buffer, and the library's
working memory is one static device array shared by all calls. This test runs
it twice in a row through the C ABI and checks both results against the
ordinary entry point (emb200_assign_device), bit for bit, and that sizes beyond
its limits are refused. It lives in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EMB200_ELIMIT = -6
MAX_ROWS = 65536


def noalloc_fn(emb):
    f = emb.lib().emb200_assign_f32_noalloc
    P, S = ctypes.c_void_p, ctypes.c_size_t
    f.argtypes = [P, S, S, P, S, P, P, ctypes.c_int, P]
    f.restype = ctypes.c_int
    return f


def test_noalloc_matches_assign_device_twice(emb):
    import torch

    f = noalloc_fn(emb)
    ref = emb.B200Assigner(0, precision="fp32")
    rng = np.random.default_rng(21)
    for (m, k, d) in [(20_000, 3_000, 96), (777, 1_031, 100)]:  # second call: smaller, other shapes
        x = torch.from_numpy(rng.standard_normal((m, d), dtype=np.float32)).cuda()
        c = torch.from_numpy(rng.standard_normal((k, d), dtype=np.float32)).cuda()
        lab = torch.full((m,), 0xFFFF, dtype=torch.int32, device="cuda")
        dst = torch.full((m,), -1.0, dtype=torch.float32, device="cuda")
        rc = f(x.data_ptr(), m, d, c.data_ptr(), k, lab.data_ptr(), dst.data_ptr(), 0, None)
        assert rc == 0
        torch.cuda.synchronize()
        ref.set_centroids(c.cpu().numpy())
        lab2 = torch.empty((m,), dtype=torch.int32, device="cuda")
        dst2 = torch.empty((m,), dtype=torch.float32, device="cuda")
        ref.assign_device(x.data_ptr(), emb.EMB200_F32, m, lab2.data_ptr(), dst2.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert torch.equal(lab, lab2)
        assert torch.equal(dst.view(torch.int32), dst2.view(torch.int32))
    ref.close()


def test_noalloc_refuses_sizes_beyond_its_limit(emb):
    f = noalloc_fn(emb)
    rc = f(ctypes.c_void_p(16), MAX_ROWS + 1, 8, ctypes.c_void_p(16), 4, ctypes.c_void_p(16), ctypes.c_void_p(16),
           0, None)
    assert rc == EMB200_ELIMIT
