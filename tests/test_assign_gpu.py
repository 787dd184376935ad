"""GPU parity of the fused assign through the C ABI against the oracle.

Every precision mode must return the CpuAssigner's labels and distances bit
for bit (the fast contraction is certified and re-scored in the reference's
own f32 rounding), and the I8 mode CpuI8Assigner(I8)'s bit for bit.
"""
import numpy as np
import pytest

from tests.test_oracle import SHAPES_F32, SHAPES_I8, lcg_f32, lcg_i8

pytestmark = pytest.mark.gpu

PRECISIONS = ["fp32", "bf16", "bf16x1", "fp8"]


def same_f32(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.fixture(scope="module")
def assigners(emb):
    made = {}

    def get(precision="fp32", centroid_bits=0, match="avx512"):
        key = (precision, centroid_bits, match)
        if key not in made:
            made[key] = emb.B200Assigner(0, precision=precision, centroid_bits=centroid_bits, match=match)
        return made[key]

    yield get
    for a in made.values():
        a.close()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("match", ["avx512", "avx2", "portable"])
def test_reference_shapes_bit_exact(orc, assigners, precision, match):
    # The shape list of src/cpu.rs:290 (every tail path), the reference's LCG data.
    a = assigners(precision, 0, match)
    for (n, k, d) in SHAPES_F32:
        x, c = lcg_f32(n * d, 1).reshape(n, d), lcg_f32(k * d, 2).reshape(k, d)
        a.set_centroids(c)
        lab, dist = a.assign(x)
        rl, rd = orc.cpu_assign(x, c, kernel=match, emulate=True)
        assert np.array_equal(lab, rl), (n, k, d)
        assert same_f32(dist, rd), (n, k, d)
        # and the f64 brute-force tolerance of src/cpu.rs:303-305
        _, best = orc.bruteforce_f64(x, c)
        assert np.all(np.abs(dist - best) <= 1e-4 * (1 + best))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_matches_cpu_bar(orc, assigners, precision):
    # src/cuda.rs:221-249: n=3000, k=1031, d=100, >= 99.9% labels; here: all, bit for bit.
    n, k, d = 3000, 1031, 100
    s = lcg_f32((n + k) * d, 1)
    x, c = s[: n * d].reshape(n, d), s[n * d:].reshape(k, d)
    a = assigners(precision)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl)
    assert same_f32(dist, rd)
    st = a.stats()
    assert st["rows"] == n and st["rows_certified"] + st["rows_refined"] == n


@pytest.mark.parametrize("precision", PRECISIONS)
def test_embedding_rows_bit_exact(emb, orc, assigners, precision):
    x = emb.datasets.embeddings(20_000, 128, seed=3)
    c = x[np.random.default_rng(4).choice(len(x), 2048, replace=False)] + np.float32(1e-3)
    a = assigners(precision)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    st = a.stats()
    rl, rd = orc.cpu_assign(x, c, emulate=False if orc.has_kernel("avx512") else True)
    assert np.array_equal(lab, rl)
    assert same_f32(dist, rd)
    # Uncertified rows go through the candidate-collecting refine pass, not the
    # exhaustive search (a handful at most end there).
    assert st["fast_aborted"] == 0
    if precision != "fp8":  # the FP8 bound certifies few rows: many refine sets exceed 32 candidates
        assert st["rows_researched"] <= max(10, st["rows_refined"] // 20), st
    if precision in ("bf16x1", "fp8"):
        assert st["rows_refined"] > 0


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("dtype", [np.int8, np.uint8])
def test_integer_rows_f32_semantics(orc, assigners, precision, dtype):
    # src/cpu.rs:106-127: non-f32 rows widened, identical to f32 input.
    rng = np.random.default_rng(7)
    info = np.iinfo(dtype)
    x = rng.integers(info.min, info.max + 1, (500, 72), dtype=dtype)
    c = rng.standard_normal((300, 72)).astype(np.float32) * 40
    a = assigners(precision)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_bias_is_added_and_reset(orc, assigners, precision):
    # Assigner::set_bias (src/lib.rs:78-81): dist includes the bias; set_centroids resets it.
    rng = np.random.default_rng(9)
    x = rng.standard_normal((777, 33)).astype(np.float32)
    c = rng.standard_normal((250, 33)).astype(np.float32)
    bias = rng.uniform(0, 3, 250).astype(np.float32)
    a = assigners(precision)
    a.set_centroids(c)
    a.set_bias(bias)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, bias=bias, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ties_go_to_lowest_index(orc, assigners, precision):
    rng = np.random.default_rng(11)
    base = rng.standard_normal((40, 16)).astype(np.float32)
    c = np.concatenate([base, base, base[::-1]])  # every centroid duplicated
    x = base[rng.integers(0, 40, 300)] + rng.standard_normal((300, 16)).astype(np.float32) * 0.01
    x[:40] = base  # exact hits: distance 0 with two tied centroids
    a = assigners(precision)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    assert np.all(lab < 40)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_adversarial_bf16_rounding(orc, assigners, precision):
    # Every element of the rows and of centroid 1 is 1 + 2^-8 - 2^-12, which BF16
    # rounds down to 1 with a relative error of almost 2^-8 (its unit roundoff);
    # centroid 0 is all ones, exact in BF16. Centroid 1 is the reference's label
    # (by d e^2, e the excess over 1), yet the single-term BF16 scores put centroid
    # 0 ahead by about 4 d e: a bound that took the unit roundoff for 2^-9 would
    # certify the wrong label. The other centroids have small norms (so the bound's
    # max |c| is the two close ones') and scores far above theirs.
    d = 128
    e = np.float32(2.0 ** -8 - 2.0 ** -12)
    v = np.float32(1.0) + e
    rng = np.random.default_rng(8)
    x = np.full((512, d), v, dtype=np.float32)
    x[256:] += rng.integers(0, 4, (256, d)).astype(np.float32) * np.float32(2.0 ** -20)  # still rounds down
    far = rng.standard_normal((62, d)).astype(np.float32) * np.float32(0.01) - np.float32(0.05)  # small norms
    c = np.concatenate([np.ones((1, d), np.float32), np.full((1, d), v, np.float32), far])
    a = assigners(precision)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    ref_l, ref_d = orc.cpu_assign(x, c, emulate=True)
    assert np.all(ref_l == 1)
    assert np.array_equal(lab, ref_l) and same_f32(dist, ref_d)


def test_edge_cases(orc, assigners):
    a = assigners("fp32")
    # k = 1, d = 1
    a.set_centroids(np.array([[2.0]], np.float32))
    lab, dist = a.assign(np.array([[0.0], [5.0]], np.float32))
    assert lab.tolist() == [0, 0] and dist.tolist() == [4.0, 9.0]
    # m = 0
    a.set_centroids(np.ones((3, 4), np.float32))
    lab, dist = a.assign(np.zeros((0, 4), np.float32))
    assert lab.size == 0
    # NaN row: no score beats +inf, label 0, dist max(NaN, 0) = 0 (src/cpu.rs:149,161)
    c = np.random.default_rng(1).standard_normal((70, 4)).astype(np.float32)
    x = np.random.default_rng(2).standard_normal((5, 4)).astype(np.float32)
    x[2, 1] = np.nan
    a.set_centroids(c)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)


def test_errors_are_reported(emb):
    a = emb.B200Assigner(0)
    with pytest.raises(emb.EngineError, match="set_centroids"):
        a.assign(np.zeros((3, 4), np.float32))
    a.set_centroids(np.ones((3, 4), np.float32))
    with pytest.raises(emb.EngineError, match="bias"):
        a.set_bias(np.ones(5, np.float32))
    with pytest.raises(emb.EngineError):
        emb.B200Assigner(99)
    a.close()


@pytest.mark.parametrize("shape", SHAPES_I8)
def test_i8_mode_integer_exact(orc, assigners, shape):
    # src/cpu_i8.rs:298-324 data; CpuI8Assigner(I8) labels and dists bit for bit.
    n, k, d = shape
    x, ci = lcg_i8(n * d, 1).reshape(n, d), lcg_i8(k * d, 2).reshape(k, d)
    a = assigners("fp32", 8)
    for c in (ci.astype(np.float32), ci.astype(np.float32) * np.float32(0.37) + np.float32(0.5)):
        a.set_centroids(c)
        lab, dist = a.assign(x)
        st = a.stats()
        # tcgen05 kind::i8 for d <= 512, the dp4a kernel beyond
        assert st["fast_kernel"] == (3 if d <= 512 else 2) and st["fast_aborted"] == 0, st
        rl, rd = orc.i8_assign(x, c, bits=8)
        assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("shape", SHAPES_I8 + [(300, 200, 2048), (50, 40, 40000 // 2)])
def test_i16_mode_integer_exact(orc, assigners, shape):
    # CpuI8Assigner(I16) (src/cpu_i8.rs:95-107): centroids in 1/2^s units, s from d
    # (d = 2048 and 20000 take smaller shifts); labels and dists bit for bit.
    n, k, d = shape
    x, ci = lcg_i8(n * d, 1).reshape(n, d), lcg_i8(k * d, 2).reshape(k, d)
    a = assigners("fp32", 16)
    for c in (ci.astype(np.float32), ci.astype(np.float32) * np.float32(0.37) + np.float32(0.5)):
        a.set_centroids(c)
        lab, dist = a.assign(x)
        assert a.stats()["fast_kernel"] == 2
        rl, rd = orc.i8_assign(x, c, bits=16)
        assert np.array_equal(lab, rl) and same_f32(dist, rd), shape


def test_i16_mode_with_bias(orc, assigners):
    rng = np.random.default_rng(6)
    x = rng.integers(-128, 128, (600, 96), dtype=np.int8)
    c = (rng.standard_normal((333, 96)) * 50).astype(np.float32)
    bias = rng.uniform(0, 5000, 333).astype(np.float32)
    a = assigners("fp32", 16)
    a.set_centroids(c)
    a.set_bias(bias)
    lab, dist = a.assign(x)
    rl, rd = orc.i8_assign(x, c, bits=16, bias=bias)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    assert "int16 centroids (1/128 unit)" in a.name()


def test_i8_mode_with_bias(orc, assigners):
    rng = np.random.default_rng(5)
    x = rng.integers(-128, 128, (600, 96), dtype=np.int8)
    c = rng.standard_normal((333, 96)).astype(np.float32) * 50
    bias = rng.uniform(0, 5000, 333).astype(np.float32)
    a = assigners("fp32", 8)
    a.set_centroids(c)
    a.set_bias(bias)
    lab, dist = a.assign(x)
    rl, rd = orc.i8_assign(x, c, bits=8, bias=bias)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_resident_assign_matches_host_path(emb, assigners, precision):
    x = emb.datasets.embeddings(50_000, 64, seed=8)
    c = x[:1500] * np.float32(0.9)
    a = assigners(precision)
    a.set_centroids(c)
    l1, d1 = a.assign(x)
    a.load_rows(x)
    l2, d2 = a.assign_resident()
    assert np.array_equal(l1, l2) and same_f32(d1, d2)


@pytest.mark.parametrize("n,d,k", [(600_000, 128, 512), (70_000, 1024, 64), (131_073, 128, 300)])
def test_host_path_many_chunks(emb, orc, assigners, n, d, k):
    # Host rows go through two staging buffers in 64 MB chunks (600k x 128:
    # five chunks; 70k x 1024: five; 131,073 x 128: a full chunk and one row),
    # so each buffer is reused. Every chunk's results must equal the resident
    # path's, and the first and last rows the oracle's.
    x = emb.datasets.embeddings(n, d, latent=16, seed=n % 97)
    c = x[np.random.default_rng(n).choice(n, k, replace=False)] * np.float32(0.97)
    a = assigners("bf16x1")
    a.set_centroids(c)
    l1, d1 = a.assign(x)
    a.load_rows(x)
    l2, d2 = a.assign_resident()
    assert np.array_equal(l1, l2) and same_f32(d1, d2)
    idx = np.r_[0:3000, n - 20000:n]
    rl, rd = orc.cpu_assign(x[idx], c, emulate=True)
    assert np.array_equal(l1[idx], rl) and same_f32(d1[idx], rd)


@pytest.mark.parametrize("precision", ["bf16x1", "bf16"])
def test_device_rows_not_16_byte_aligned(emb, orc, assigners, precision):
    # Device rows at a 4-byte offset with d % 16 == 0: the fast kernel's row loads
    # and the certify pass take their scalar forms; the results are the oracle's.
    import torch

    n, d = 5000, 128
    x = emb.datasets.embeddings(n, d, latent=16, seed=31)
    c = x[np.random.default_rng(31).choice(n, 300, replace=False)] * np.float32(0.97)
    a = assigners(precision)
    a.set_centroids(c)
    buf = torch.empty(n * d + 1, dtype=torch.float32, device="cuda")
    buf[1:] = torch.from_numpy(x.ravel()).cuda()
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    dst = torch.empty(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    a.assign_device(buf.data_ptr() + 4, emb.EMB200_F32, n, lab.data_ptr(), dst.data_ptr())
    torch.cuda.synchronize()
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab.cpu().numpy().view(np.uint32), rl) and same_f32(dst.cpu().numpy(), rd)


def test_resident_rows_past_one_search_pass(emb, orc, assigners):
    # 2^26 + 4099 resident rows: the search runs in two passes of at most 2^26
    # rows (its kernels index rows in 32 bits). Rows on both sides of the seam,
    # at the ends and at random must match the oracle.
    n = (1 << 26) + 4099
    rng = np.random.default_rng(26)
    x = rng.standard_normal((n, 2), dtype=np.float32)
    c = rng.standard_normal((8, 2), dtype=np.float32)
    a = assigners("bf16x1")
    a.set_centroids(c)
    a.load_rows(x)
    lab, dist = a.assign_resident()
    seam = 1 << 26
    idx = np.unique(np.r_[0:2000, seam - 2000:seam + 2000, n - 2000:n, rng.integers(0, n, 20000)])
    rl, rd = orc.cpu_assign(x[idx], c, emulate=True)
    assert np.array_equal(lab[idx], rl) and same_f32(dist[idx], rd)


@pytest.mark.parametrize("precision", ["bf16", "bf16x1"])
@pytest.mark.parametrize("d", [1, 33, 64, 96, 128])
def test_tcgen05_path_runs_and_certifies(emb, orc, assigners, precision, d):
    # The tensor-core kernel (not the SIMT fallback) must serve d <= 128 and
    # finish without a bounded wait giving up.
    x = emb.datasets.embeddings(4000, d, latent=min(8, d), seed=d)
    c = x[np.random.default_rng(d).choice(len(x), 700, replace=False)] * np.float32(0.98)
    a = assigners(precision)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    st = a.stats()
    assert st["fast_kernel"] == 1 and st["fast_aborted"] == 0, st
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    if precision == "bf16" and d >= 33:  # at d = 1 every centroid ties with others: all rows re-searched
        assert st["rows_researched"] <= 0.02 * len(x), st


def test_i8_mode_c3_like_exact(emb, orc, assigners):
    # The int8 workload's shape at reduced size: unit-norm 64-d-latent rows,
    # faiss calibration to i8, d = 512, k = 512 centroids taken from the codes.
    xf = emb.datasets.embeddings(6_000, 512, latent=64, seed=12)
    codes, _, _ = emb.datasets.faiss_int8(xf)
    c = codes[np.random.default_rng(3).choice(len(codes), 512, replace=False)].astype(np.float32) + np.float32(0.3)
    a = assigners("fp32", 8)
    a.set_centroids(c)
    lab, dist = a.assign(codes)
    assert a.stats()["fast_kernel"] == 3
    rl, rd = orc.i8_assign(codes, c, bits=8)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("n,k", [(94_720, 4096), (76_000, 300)])
def test_certified_in_the_fast_kernel(emb, orc, assigners, n, k):
    # Row tiles in whole waves of 148 SMs, so the search takes one column split
    # (on a 148-SM B200): the single-term search certifies
    # each row tile in its own row-loader warps (no separate certify kernel).
    # Labels and distances must still be the reference's bit for bit, and the
    # certified and refined counts must cover every row.
    x = emb.datasets.embeddings(n, 128, latent=32, seed=17)
    c = x[np.random.default_rng(18).choice(n, k, replace=False)] * np.float32(0.97)
    a = assigners("bf16x1")
    a.set_centroids(c)
    lab, dist = a.assign(x)
    st = a.stats()
    rl, rd = orc.cpu_assign(x, c, emulate=not orc.has_kernel("avx512"))
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    assert st["rows_certified"] + st["rows_refined"] == n and st["rows_refined"] > 0, st
    assert st["fast_aborted"] == 0, st


def test_certified_in_the_fast_kernel_with_bias(emb, orc, assigners):
    # The same one-split search with a per-centroid bias (norms and their bound
    # include it), then reset by set_centroids.
    n, k = 75_776, 2_000
    x = emb.datasets.embeddings(n, 64, latent=16, seed=19)
    c = x[np.random.default_rng(20).choice(n, k, replace=False)] * np.float32(0.97)
    bias = np.random.default_rng(21).uniform(0, 0.05, k).astype(np.float32)
    a = assigners("bf16x1")
    a.set_centroids(c)
    a.set_bias(bias)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, bias=bias, emulate=not orc.has_kernel("avx512"))
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    a.set_centroids(c)
    lab, dist = a.assign(x)
    rl, rd = orc.cpu_assign(x, c, emulate=not orc.has_kernel("avx512"))
    assert np.array_equal(lab, rl) and same_f32(dist, rd)


@pytest.mark.parametrize("precision,bits,n", [("bf16x1", 0, 9_000), ("bf16", 0, 9_000), ("fp32", 8, 9_000),
                                              ("bf16x1", 0, 75_776)])
@pytest.mark.parametrize("stall_tile", [0, 2])
def test_bounded_wait_abort_path(emb, orc, precision, bits, n, stall_tile):
    # One epilogue warp of every CTA of the fast tensor-core kernel waits, at a
    # given centroid tile, on a barrier that nothing completes, with a 2 ms limit.
    # The wait runs out while copies and MMAs are in flight: the kernel drains
    # them, frees TMEM and flags the abort, and the call settles every row with
    # the exact search. Labels and distances must still be the oracle's, and the
    # GPU must serve the next call normally. With 75,776 rows the search runs in
    # one column split and certifies in its row-loader warps, which must list the
    # rows of every unfinished row tile.
    rng = np.random.default_rng(40 + stall_tile)
    k, d = 2_000, 96
    a = emb.B200Assigner(0, precision=precision, centroid_bits=bits)
    if bits:
        x = rng.integers(-128, 128, (n, d), dtype=np.int8)
        c = rng.integers(-128, 128, (k, d)).astype(np.float32)
    else:
        x = emb.datasets.embeddings(n, d, latent=16, seed=stall_tile)
        c = x[rng.choice(n, k, replace=False)] * np.float32(0.97)
    a.set_centroids(c)
    ref = orc.i8_assign(x, c, bits=8) if bits else orc.cpu_assign(x, c, emulate=True)
    a.set_abort_test(stall_tile, 2_000_000)
    lab, dist = a.assign(x)
    st = a.stats()
    assert st["fast_aborted"] == 1, st
    assert np.array_equal(lab, ref[0]) and same_f32(dist, ref[1])
    a.set_abort_test(-1)
    lab, dist = a.assign(x)
    st = a.stats()
    assert st["fast_aborted"] == 0, st
    assert np.array_equal(lab, ref[0]) and same_f32(dist, ref[1])
    a.close()


@pytest.mark.parametrize("d", [8, 100, 128, 200, 256, 300])
@pytest.mark.parametrize("extreme", [False, True])
def test_fp8_search_bit_exact(emb, orc, assigners, d, extreme):
    # tcgen05 kind::f8f6f4 with e4m3 operands and a power-of-two scale per row and
    # per centroid (d <= 256; beyond it the FP32 search serves). With
    # `extreme`, a zero row, rows and centroids whose largest magnitude leaves the
    # FP8 range (tiny and huge) are in the data. Every label and distance must be
    # the oracle's, through the host and the resident paths.
    x = emb.datasets.embeddings(6000, d, latent=min(16, d), seed=d)
    c = x[np.random.default_rng(d).choice(len(x), 900, replace=False)] * np.float32(0.97)
    if extreme:
        x[0] = 0.0
        x[1] *= np.float32(1e-30)
        x[2] *= np.float32(1e15)
        c[5] *= np.float32(1e-25)
        c[6] *= np.float32(1e19)
    a = assigners("fp8")
    a.set_centroids(c)
    lab, dist = a.assign(x)
    st = a.stats()
    # d > 256: neither FP8 operands nor the BF16 split (both need d <= 256): the FP32 search serves
    assert st["fast_kernel"] == (4 if d <= 256 else 0) and st["fast_aborted"] == 0, st
    rl, rd = orc.cpu_assign(x, c, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    a.load_rows(x)
    lab, dist = a.assign_resident()
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
