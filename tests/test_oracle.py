"""Pins the CPU oracle against the reference crate's own known-answer tests.

Each test restates one of the reference's unit tests (cited) against the C++
restatement in oracle/, so the oracle is trusted before it checks the GPU.
"""
import numpy as np
import pytest


def lcg_f32(n, seed):
    """src/cpu.rs:272-280: s = s*1664525 + 1013904223; (s >> 8) / 2^24 - 0.5."""
    out = np.empty(n, np.float32)
    s = np.uint32(seed)
    vals = np.empty(n, np.uint32)
    with np.errstate(over="ignore"):
        for i in range(n):
            s = np.uint32(s * np.uint32(1664525) + np.uint32(1013904223))
            vals[i] = s
    out[:] = (vals >> np.uint32(8)).astype(np.float32) / np.float32(1 << 24) - np.float32(0.5)
    return out


def lcg_i8(n, seed):
    """src/cpu_i8.rs:284-292: (s >> 24) as u8 as i8."""
    s = np.uint32(seed)
    vals = np.empty(n, np.uint32)
    with np.errstate(over="ignore"):
        for i in range(n):
            s = np.uint32(s * np.uint32(1664525) + np.uint32(1013904223))
            vals[i] = s
    return (vals >> np.uint32(24)).astype(np.uint8).view(np.int8)


def test_recipe_matches_reference(orc):
    # src/lib.rs:526-540, values printed by faiss 1.16.0.
    r = orc.resolve_recipe(200_000, 96, 1024)
    assert r["batch_size"] == 16384
    assert abs(r["alpha0"] - 0.728183) < 1e-5
    r = orc.resolve_recipe(1_000_000, 8, 100, orc.make_config(nepochs=2.5))
    assert r["epoch_rows"] == [1_000_000, 500_000, 1_000_000]
    assert r["batch_size"] == 4096
    assert abs(r["alpha0"] - 0.319215) < 1e-5
    r = orc.resolve_recipe(4000, 4, 8)
    assert r["batch_size"] == 32
    assert abs(r["alpha0"] - 0.144604) < 1e-5
    assert orc.resolve_recipe(1000, 2, 10)["unused_threshold"] == 0.0


def test_schedule_endpoints(orc):
    # src/lib.rs:542-546
    assert abs(orc.scheduled_alpha(0.5, 0, 100) - 0.5) < 1e-12
    assert abs(orc.scheduled_alpha(0.5, 100, 100) - 0.05) < 1e-12


def test_full_batch_step_one_is_lloyd(orc):
    # src/lib.rs:548-562
    x = np.array([0.0, 0.0, 0.0, 2.0, 10.0, 0.0, 10.0, 2.0], np.float32).reshape(4, 2)
    cent = np.array([[0.0, 0.0], [10.0, 0.0]], np.float32)
    usage = np.full(2, 1.0 / 65536.0, np.float32)
    sums = np.zeros(4, np.float32)
    for i, row in enumerate(x):
        sums[(i // 2) * 2] += row[0]
        sums[(i // 2) * 2 + 1] += row[1]
    orc.state_apply(cent, usage, [0, 1], [2, 2], sums, 1.0)
    assert cent.ravel().tolist() == [0.0, 1.0, 10.0, 1.0]
    assert usage.tolist() == [2.0, 2.0]


def test_revival_splits_a_donor(orc):
    # src/lib.rs:564-573
    cent = np.array([[1.0, 1.0], [5.0, 5.0], [9.0, 9.0]], np.float32)
    usage = np.array([4.0, 0.0, 4.0], np.float32)
    n = orc.state_revive(cent, usage, 0.1, 1)
    assert n == 1
    assert usage.sum() == 8.0 and usage[1] == 2.0
    src = 0 if usage[0] == 2.0 else 2
    assert abs(cent[1, 0] - cent[src, 0]) < 1e-2
    assert cent[1, 0] != cent[src, 0]


def closing_mean_data(orc):
    """The 20-blob 6-D data of src/lib.rs:577-587, drawn from Rng::new(7)."""
    n, d = 20_000, 6
    u = orc.rng_open01(7, 20 * d + n * d * 4).astype(np.float32)
    centers = np.float32(8.0) * (u[: 20 * d] - np.float32(0.5))
    noise_u = (u[20 * d:] - np.float32(0.5)).reshape(n, d, 4)
    noise = np.full((n, d), -0.0, np.float32)
    for t in range(4):
        noise = noise + noise_u[:, :, t]
    x = centers.reshape(20, d)[np.arange(n) % 20] + noise
    return x.astype(np.float32)


def test_closing_mean_and_loss(orc):
    # src/lib.rs:575-614
    n, d, k = 20_000, 6, 32
    x = closing_mean_data(orc)
    out = orc.train(x, k)
    labels = out["labels"]
    sums = np.zeros((k, d))
    counts = np.bincount(labels, minlength=k)
    np.add.at(sums, labels, x.astype(np.float64))
    assert counts.sum() == n
    for j in np.nonzero(counts)[0]:
        assert np.all(np.abs(out["centroids"][j].astype(np.float64) - sums[j] / counts[j]) < 1e-3)

    def mse(c):
        _, dist = orc.cpu_assign(x, c)
        return dist.astype(np.float64).mean()

    init = x[orc.permutation(1234, n)[:k]]
    trained, start = mse(out["centroids"]), mse(init)
    assert trained < 0.75 * start and trained < 2.0, (trained, start)
    assert np.all(np.diff(out["objective"]) < 0)


SHAPES_F32 = [(1, 1, 1), (5, 3, 7), (13, 9, 16), (37, 70, 33), (130, 257, 100), (64, 1030, 384), (9, 6, 1027)]


@pytest.mark.parametrize("kernel", ["avx512", "avx2", "portable"])
def test_kernels_match_brute_force(orc, kernel):
    # src/cpu.rs:282-309, tolerance 1e-4 * (1 + best) on label and distance.
    for (n, k, d) in SHAPES_F32:
        x, c = lcg_f32(n * d, 1).reshape(n, d), lcg_f32(k * d, 2).reshape(k, d)
        modes = [True] + ([False] if orc.has_kernel(kernel) else [])
        _, best = orc.bruteforce_f64(x, c)
        for emulate in modes:
            labels, dist = orc.cpu_assign(x, c, kernel=kernel, emulate=emulate)
            got = ((x.astype(np.float64) - c[labels].astype(np.float64)) ** 2).sum(1)
            tol = 1e-4 * (1 + best)
            assert np.all(got <= best + tol)
            assert np.all(np.abs(dist - best) <= tol)


@pytest.mark.parametrize("kernel", ["avx512", "avx2"])
def test_simd_and_emulation_are_bit_identical(orc, kernel):
    if not orc.has_kernel(kernel):
        pytest.skip(f"{kernel} not on this CPU")
    rng = np.random.default_rng(3)
    for (n, k, d) in SHAPES_F32 + [(200, 300, 96), (77, 129, 128)]:
        x = rng.standard_normal((n, d), dtype=np.float32)
        c = rng.standard_normal((k, d), dtype=np.float32)
        l1, d1 = orc.cpu_assign(x, c, kernel=kernel)
        l2, d2 = orc.cpu_assign(x, c, kernel=kernel, emulate=True)
        assert np.array_equal(l1, l2)
        assert np.array_equal(d1.view(np.uint32), d2.view(np.uint32))


SHAPES_I8 = [(1, 1, 1), (5, 3, 7), (13, 9, 64), (37, 70, 33), (130, 257, 100), (20, 1030, 512), (9, 6, 1027)]


@pytest.mark.parametrize("bits", [8, 16])
def test_integer_kernels_are_exact(orc, bits):
    # src/cpu_i8.rs:298-324: integer-valued centroids give an exact search.
    for (n, k, d) in SHAPES_I8:
        x, ci = lcg_i8(n * d, 1).reshape(n, d), lcg_i8(k * d, 2).reshape(k, d)
        c = ci.astype(np.float32)
        diff = x.astype(np.int64)[:, None, :] - ci.astype(np.int64)[None, :, :]
        sq = (diff * diff).sum(-1)
        exact_l = sq.argmin(1)
        exact_d = sq[np.arange(n), exact_l]
        labels, dist = orc.i8_assign(x, c, bits=bits)
        assert np.array_equal(labels, exact_l)
        assert np.array_equal(dist, exact_d.astype(np.float32))


def test_i16_resolves_fractional_centroids(orc):
    # src/cpu_i8.rs:326-336
    x = np.array([[1, 0]], np.int8)
    c = np.array([[0.26, 0.0], [-0.26, 0.0]], np.float32)
    labels, dist = orc.i8_assign(x, c, bits=16)
    assert labels[0] == 0
    assert abs(dist[0] - 0.74 * 0.74) < 0.01


def test_faiss_calibration_and_round_trip(orc):
    # src/quantize.rs:102-116
    sample = np.array([15.0, -3.0, 5.0, -3.0, 10.0, -2.0, 10.0, -4.0], np.float32).reshape(4, 2)
    shift, scale = orc.quantizer_fit(sample)
    assert shift.tolist() == [10.0, -3.0]
    assert scale == 16.0
    codes = orc.quantizer_encode(sample, shift, scale)
    assert codes.ravel().tolist() == [80, 0, -80, 0, 0, 16, 0, -16]
    back = codes.astype(np.float32) * np.float32(1.0 / scale) + shift
    assert np.array_equal(back, sample)
    assert orc.quantizer_encode(np.array([[1000.0, -3.0]], np.float32), shift, scale).ravel().tolist() == [127, 0]
    assert np.array_equal(orc.quantizer_decode(codes, shift, scale), sample)
    assert orc.quantizer_clipped(np.array([[1000.0, -3.0]], np.float32), shift, scale) / 2 == 0.5


def test_clipped_calibration(orc):
    # Calibration::clipped(q) (src/quantize.rs:31-33): the peak is the centred
    # magnitude at rank round((n d - 1) q), the scale 127 / peak, not a power of two.
    x = np.array([[0.0], [1.0], [2.0], [3.0], [4.0], [100.0]], np.float32)  # mean 18.333..
    shift, scale = orc.quantizer_fit(x, 127.0, 0.5, False)
    mags = np.sort(np.abs(x[:, 0] - shift[0]))
    assert shift[0] == np.float32(np.float64(110.0) / 6)
    # rank round(5 x 0.5) = 3: f64::round goes half away from zero
    assert scale == np.float32(127.0) / mags[3]


def test_i8_rows_through_cpu_assigner_equal_f32(orc):
    # src/cpu.rs:106-107: non-f32 rows are widened, results identical to f32 input.
    rng = np.random.default_rng(5)
    x8 = rng.integers(-128, 128, (50, 40), dtype=np.int8)
    c = rng.standard_normal((70, 40)).astype(np.float32) * 30
    a = orc.cpu_assign(x8, c)
    b = orc.cpu_assign(x8.astype(np.float32), c)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
