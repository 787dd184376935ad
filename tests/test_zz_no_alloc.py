"""The search entry point that allocates nothing (emb200_assign_f32_noalloc).

It serves callers that cannot allocate device memory when they search (their
GPU memory belongs to their own pool or budget, or an allocation could stall or
fail on a latency-critical path): they pass every buffer, and the library's
working memory is one static device array shared by all calls. These tests call
it through the C ABI, two calls in a row each time, and check its labels and
distances bit for bit against the ordinary entry point (emb200_assign_device)
and against the oracle (the reference CpuAssigner restated), including a full
65,536-row call, rows that the certification cannot settle (duplicated
centroids, exact hits) in all three roundings, and the refusal of sizes beyond
its limits. The file is collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EMB200_ELIMIT = -6
EMB200_EINVAL = -1
MAX_ROWS = 65536
MATCH = {"avx512": 0, "avx2": 1, "portable": 2}


def noalloc_fn(emb):
    f = emb.lib().emb200_assign_f32_noalloc
    P, S = ctypes.c_void_p, ctypes.c_size_t
    f.argtypes = [P, S, S, P, S, P, P, ctypes.c_int, P]
    f.restype = ctypes.c_int
    return f


def run_noalloc(f, x, c, match=0):
    """One call on device copies of x and c; returns host (labels, dist)."""
    import torch

    m, d = x.shape
    k = c.shape[0]
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    cd = torch.from_numpy(np.ascontiguousarray(c)).cuda()
    lab = torch.full((m,), 0x7FFF, dtype=torch.int32, device="cuda")
    dst = torch.full((m,), -1.0, dtype=torch.float32, device="cuda")
    rc = f(xd.data_ptr(), m, d, cd.data_ptr(), k, lab.data_ptr(), dst.data_ptr(), match, None)
    assert rc == 0
    torch.cuda.synchronize()
    return lab.cpu().numpy().view(np.uint32), dst.cpu().numpy()


def same_f32(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


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


def test_noalloc_matches_oracle_full_call_twice(emb, orc):
    # A full call (m = 65536 rows, the limit) of embedding rows against centroids
    # drawn from them, then a smaller call on other shapes: both equal the oracle.
    f = noalloc_fn(emb)
    x = emb.datasets.embeddings(MAX_ROWS, 128, latent=32, seed=5)
    c = x[np.random.default_rng(5).choice(MAX_ROWS, 4096, replace=False)] * np.float32(0.97)
    for (xs, cs) in [(x, c), (x[:5000, :72].copy(), c[:700, :72].copy())]:
        lab, dist = run_noalloc(f, xs, cs)
        rl, rd = orc.cpu_assign(xs, cs, emulate=not orc.has_kernel("avx512"))
        assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("match", ["avx512", "avx2", "portable"])
def test_noalloc_uncertified_rows_match_oracle(emb, orc, match):
    # Every centroid duplicated (so no row's top-2 has a margin: all rows go to
    # the exhaustive re-search), exact hits at distance 0, and d = 37 (not a
    # multiple of 16 or 8: every tail path of the three roundings). Ties go to
    # the lowest index as in the reference's strict-< scan.
    f = noalloc_fn(emb)
    rng = np.random.default_rng(37)
    base = rng.standard_normal((60, 37)).astype(np.float32)
    c = np.concatenate([base, base, base[::-1]])
    x = base[rng.integers(0, 60, 3000)] + rng.standard_normal((3000, 37)).astype(np.float32) * 0.01
    x[:60] = base
    for rows in (x, x[::-1].copy()):  # two calls in a row
        lab, dist = run_noalloc(f, rows, c, MATCH[match])
        rl, rd = orc.cpu_assign(rows, c, kernel=match, emulate=True)
        assert np.array_equal(lab, rl) and same_f32(dist, rd)
        assert np.all(lab < 60)


def test_noalloc_refuses_sizes_beyond_its_limit(emb):
    f = noalloc_fn(emb)
    rc = f(ctypes.c_void_p(16), MAX_ROWS + 1, 8, ctypes.c_void_p(16), 4, ctypes.c_void_p(16), ctypes.c_void_p(16),
           0, None)
    assert rc == EMB200_ELIMIT
    rc = f(ctypes.c_void_p(16), 4, (1 << 31) - 63, ctypes.c_void_p(16), 4, ctypes.c_void_p(16), ctypes.c_void_p(16),
           0, None)
    assert rc == EMB200_EINVAL
