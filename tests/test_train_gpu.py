"""GPU parity of the device-resident training loop (src/lib.rs:348-491) with the
oracle's restatement of the reference's CPU train().

The batch search is bit-exact and the update kernels follow the reference's f32
operation order, so the trained centroids, last-pass labels and revival counts
must equal the oracle's bit for bit; the per-epoch objective (an f64 sum whose
order differs) must agree to 1e-12 relative.
"""
import numpy as np
import pytest

from tests.test_oracle import closing_mean_data

pytestmark = pytest.mark.gpu


def same_f32(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def run_both(emb, orc, x, k, precision="fp32", centroid_bits=0, assigner="cpu", **cfg):
    a = emb.B200Assigner(0, precision=precision, centroid_bits=centroid_bits)
    out = emb.train(x, x.shape[1], k, emb.Config(**cfg), assigner=a)
    st = a.stats()
    a.close()
    ref = orc.train(x, k, orc.make_config(**cfg), assigner=assigner, kernel="avx512", emulate=not orc.has_kernel("avx512"))
    return out, ref, st


def check_same(out, ref):
    assert out.recipe.batch_size == ref["recipe"]["batch_size"]
    assert out.recipe.epoch_rows == ref["recipe"]["epoch_rows"]
    assert out.n_splits == ref["n_splits"]
    assert np.array_equal(out.labels, ref["labels"])
    assert same_f32(out.centroids, ref["centroids"])
    np.testing.assert_allclose(out.objective, ref["objective"], rtol=1e-12)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_closing_mean_data_bit_exact(emb, orc, precision):
    # The 20-blob 6-D data of src/lib.rs:575-614 (quality law, revival every 5 steps).
    x = closing_mean_data(orc)
    out, ref, _ = run_both(emb, orc, x, 32, precision)
    check_same(out, ref)
    # and the reference test's own invariants
    k, d = 32, 6
    sums = np.zeros((k, d))
    counts = np.bincount(out.labels, minlength=k)
    np.add.at(sums, out.labels, x.astype(np.float64))
    for j in np.nonzero(counts)[0]:
        assert np.all(np.abs(out.centroids[j] - sums[j] / counts[j]) < 1e-3)
    assert np.all(np.diff(out.objective) < 0)


@pytest.mark.parametrize("precision", ["fp32", "bf16", "bf16x1"])
def test_blob_mixture_bit_exact(emb, orc, precision):
    x = emb.datasets.blobs(30_000, 96, n_blobs=512, seed=2)
    out, ref, st = run_both(emb, orc, x, 256, precision, nepochs=3.0)
    check_same(out, ref)
    assert st["fast_aborted"] == 0


def test_large_batches_single_term_bit_exact(emb, orc):
    # Batches of 98,304 rows (whole waves of row tiles on 148 SMs, one centroid
    # tile): the single-term search certifies each row tile inside its own kernel,
    # also in the captured epochs. Training must still equal the oracle's.
    x = emb.datasets.blobs(196_608, 32, n_blobs=300, seed=6)
    out, ref, st = run_both(emb, orc, x, 200, "bf16x1", nepochs=2.0, batch_size=98_304)
    check_same(out, ref)
    assert st["fast_aborted"] == 0


@pytest.mark.parametrize("d", [100, 36])
def test_crowded_clusters_bit_exact(emb, orc, d):
    # Most rows in one tight blob: a batch puts hundreds of rows in a few clusters
    # (row lists past 128 entries sorted in scratch, many chunks per warp through
    # the staging ring), with d not a multiple of 32 (a partly filled last warp).
    rng = np.random.default_rng(d)
    big = rng.standard_normal((15_000, d)).astype(np.float32) * np.float32(0.05)
    rest = emb.datasets.blobs(5_000, d, n_blobs=40, seed=d)
    x = np.concatenate([big, rest])[rng.permutation(20_000)]
    out, ref, _ = run_both(emb, orc, x, 24, "fp32", nepochs=2.0, batch_size=8192)
    check_same(out, ref)


def test_embeddings_bit_exact(emb, orc):
    x = emb.datasets.embeddings(40_000, 128, seed=5)
    out, ref, _ = run_both(emb, orc, x, 512, "bf16", nepochs=2.0)
    check_same(out, ref)


def test_fractional_and_short_epochs(emb, orc):
    x = emb.datasets.blobs(6_000, 12, n_blobs=64, seed=3)
    out, ref, _ = run_both(emb, orc, x, 40, "fp32", nepochs=2.5)
    check_same(out, ref)
    assert out.recipe.epoch_rows == [6000, 3000, 6000]
    out, ref, _ = run_both(emb, orc, x, 40, "fp32", nepochs=0.5)
    check_same(out, ref)
    assert (out.labels == 0xFFFFFFFF).sum() == 3000  # rows outside the only (partial) pass


def test_balance_penalty_bit_exact(emb, orc):
    x = emb.datasets.blobs(20_000, 32, n_blobs=300, seed=4)
    out, ref, _ = run_both(emb, orc, x, 128, "bf16", nepochs=3.0, balance=0.3)
    check_same(out, ref)


def test_int8_rows_both_semantics(emb, orc):
    xf = emb.datasets.embeddings(30_000, 64, latent=16, seed=6)
    codes, _, _ = emb.datasets.faiss_int8(xf)
    # CpuI8Assigner(I8): integer search (src/cpu_i8.rs), f32 sums and EMA.
    out, ref, _ = run_both(emb, orc, codes, 200, "fp32", centroid_bits=8, assigner="i8", nepochs=3.0)
    check_same(out, ref)
    # CpuI8Assigner(I16): centroids in 1/128 units, exact integer search.
    out, ref, _ = run_both(emb, orc, codes, 200, "fp32", centroid_bits=16, assigner="i16", nepochs=3.0)
    check_same(out, ref)
    # CpuAssigner on i8 rows: rows widened to f32.
    out, ref, _ = run_both(emb, orc, codes, 200, "bf16", nepochs=3.0)
    check_same(out, ref)


def test_uint8_rows(emb, orc):
    rng = np.random.default_rng(8)
    x = (rng.integers(0, 40, (12_000, 24)) + rng.integers(0, 200, (1, 24))).astype(np.uint8)
    out, ref, _ = run_both(emb, orc, x, 64, "bf16", nepochs=2.0)
    check_same(out, ref)


def test_closing_mean_f64_option(emb):
    x = emb.datasets.blobs(20_000, 16, n_blobs=100, seed=9)
    a = emb.B200Assigner(0, precision="bf16")
    out = emb.train(x, 16, 64, emb.Config(nepochs=2.0, closing_f64=True), assigner=a)
    a.close()
    counts = np.bincount(out.labels, minlength=64)
    sums = np.zeros((64, 16))
    np.add.at(sums, out.labels, x.astype(np.float64))
    for j in np.nonzero(counts)[0]:
        assert np.array_equal(out.centroids[j], (sums[j] / counts[j]).astype(np.float32))


def test_training_argument_errors(emb):
    a = emb.B200Assigner(0)
    a.load_rows(np.zeros((10, 3), np.float32))
    with pytest.raises(emb.EngineError, match="at least k"):
        a.train_resident(11)
    with pytest.raises(emb.EngineError, match="nepochs"):
        a.train_resident(2, emb.Config(nepochs=0.0))
    a.close()


def test_assign_after_training_uses_trained_centroids(emb, orc):
    x = emb.datasets.blobs(10_000, 20, n_blobs=50, seed=10)
    a = emb.B200Assigner(0, precision="bf16")
    out = emb.train(x, 20, 48, emb.Config(nepochs=2.0), assigner=a)
    lab, dist = a.assign_resident()
    rl, rd = orc.cpu_assign(x, out.centroids, emulate=True)
    assert np.array_equal(lab, rl) and same_f32(dist, rd)
    a.close()


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_graph_replay_equals_eager_launches(emb, orc, precision):
    # The training loop replays one captured CUDA graph per epoch length; launching
    # the same kernels one by one must give the same bits (and both the oracle's).
    x = emb.datasets.blobs(12_000, 24, n_blobs=80, seed=14)
    outs = []
    for eager in (False, True):
        a = emb.B200Assigner(0, precision=precision, train_eager=eager)
        outs.append(emb.train(x, 24, 60, emb.Config(nepochs=2.5), assigner=a))
        a.close()
    ref = orc.train(x, 60, orc.make_config(nepochs=2.5), emulate=not orc.has_kernel("avx512"))
    for out in outs:
        check_same(out, ref)


def test_batched_instances_equal_single_runs(emb, orc):
    # Uneven instances over row ranges of one resident matrix (IVF-list-like):
    # each result must equal its own train() call, bit for bit.
    rng = np.random.default_rng(15)
    sizes = [3000, 9000, 1500, 6000, 12000, 2500]
    ks = [16, 40, 16, 30, 60, 20]
    parts = [emb.datasets.blobs(n, 32, n_blobs=50, seed=100 + i) + rng.standard_normal(32).astype(np.float32) * 5
             for i, n in enumerate(sizes)]
    x = np.concatenate(parts).astype(np.float32)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    cfg = emb.Config(nepochs=3.0)
    a = emb.B200Assigner(0, precision="fp32")
    a.load_rows(x)
    outs = a.train_batched([(int(s0), n, k) for s0, n, k in zip(starts, sizes, ks)], cfg, max_concurrency=4)
    a.close()
    for i, (n, k) in enumerate(zip(sizes, ks)):
        b = emb.B200Assigner(0, precision="fp32")
        single = emb.train(parts[i], 32, k, cfg, assigner=b)
        b.close()
        assert np.array_equal(outs[i].labels, single.labels)
        assert same_f32(outs[i].centroids, single.centroids)
        assert outs[i].n_splits == single.n_splits
    ref = orc.train(parts[4], ks[4], orc.make_config(nepochs=3.0), emulate=not orc.has_kernel("avx512"))
    check_same(outs[4], ref)


def test_graph_epoch_with_a_short_last_batch(emb):
    # Full batches of 19,200 rows (150 row tiles: one centroid split) and a last
    # batch of 18,000 (141 tiles: two splits, more partials than a full batch):
    # the captured epoch must not need a buffer the dry run did not size.
    x = emb.datasets.blobs(19_200 * 16 + 18_000, 16, n_blobs=600, seed=16)
    outs = []
    for eager in (False, True):
        a = emb.B200Assigner(0, precision="bf16", train_eager=eager)
        outs.append(emb.train(x, 16, 512, emb.Config(nepochs=1.0, batch_size=19_200), assigner=a))
        a.close()
    assert outs[0].recipe.batch_size == 19_200
    assert np.array_equal(outs[0].labels, outs[1].labels)
    assert same_f32(outs[0].centroids, outs[1].centroids)


def _uneven_instances(emb, d, sizes, ks, seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    parts = [emb.datasets.blobs(n, d, n_blobs=max(8, k // 2), seed=seed + i) + rng.standard_normal(d).astype(np.float32) * 5
             for i, (n, k) in enumerate(zip(sizes, ks))]
    if dtype != np.float32:
        info = np.iinfo(dtype)
        parts = [np.clip(np.rint(p * 6), info.min, info.max).astype(dtype) for p in parts]
    x = np.ascontiguousarray(np.concatenate(parts))
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    return parts, x, [(int(s0), n, k) for s0, n, k in zip(starts, sizes, ks)]


@pytest.mark.parametrize("dtype", [np.float32, np.int8, np.uint8])
@pytest.mark.parametrize("closing_f64", [False, True])
def test_lockstep_instances_equal_single_runs(emb, dtype, closing_f64):
    # The lockstep kernels (every instance advancing one global step at a time,
    # batched search over an (instance, row tile) queue) against each instance's
    # own train(): labels, centroids, revival counts and objective bit for bit.
    # Sizes give instances with a few and with many steps, a batch as large as
    # the rows, and k from 16 to 200.
    sizes = [2500, 14000, 900, 7000, 30000, 4100, 600]
    ks = [16, 60, 30, 200, 120, 25, 40]
    parts, x, inst = _uneven_instances(emb, 24, sizes, ks, 70, dtype)
    cfg = emb.Config(nepochs=3.0, closing_f64=closing_f64)
    a = emb.B200Assigner(0, precision="fp32")
    a.load_rows(x)
    outs = a.train_batched(inst, cfg)
    a.close()
    for i, (n, k) in enumerate(zip(sizes, ks)):
        b = emb.B200Assigner(0, precision="fp32")
        single = emb.train(parts[i], 24, k, cfg, assigner=b)
        b.close()
        assert np.array_equal(outs[i].labels, single.labels), i
        assert same_f32(outs[i].centroids, single.centroids), i
        assert outs[i].n_splits == single.n_splits, i
        assert np.array_equal(outs[i].objective, single.objective), i


@pytest.mark.parametrize("d", [16, 40])
def test_lockstep_every_search_variant(emb, monkeypatch, tmp_path, d):
    # Every search form the autotuner can pick (forced through
    # EMB200_BATCHED_SEARCH_VARIANT; a form that does not apply to d is ignored
    # and the default choice runs) gives the same bits: the certification and
    # the exact re-search settle each row whatever the search's partials were.
    sizes = [9000, 2600, 15000, 700]
    ks = [150, 16, 90, 40]
    _, x, inst = _uneven_instances(emb, d, sizes, ks, 300 + d)
    cfg = emb.Config(nepochs=2.0)
    monkeypatch.setenv("EMB200_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    ref = None
    for v in range(11):
        monkeypatch.setenv("EMB200_BATCHED_SEARCH_VARIANT", str(v))
        a = emb.B200Assigner(0, precision="fp32")
        a.load_rows(x)
        outs = a.train_batched(inst, cfg)
        a.close()
        if ref is None:
            ref = outs
            continue
        for o, q in zip(ref, outs):
            assert np.array_equal(o.labels, q.labels), v
            assert same_f32(o.centroids, q.centroids), v
            assert o.n_splits == q.n_splits, v


def test_lockstep_graph_eager_streams_agree(emb, orc, tmp_path, monkeypatch):
    # The captured global step replayed, the same kernels launched one by one, and
    # the per-instance streams mode give the same bits; k = 5000 takes the
    # revival's global-memory donor sort; the autotuner records its choice.
    monkeypatch.setenv("EMB200_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    sizes = [60000, 3000, 12000]
    ks = [5000, 20, 300]
    parts, x, inst = _uneven_instances(emb, 16, sizes, ks, 90)
    cfg = emb.Config(nepochs=2.0)
    res = []
    for eager, streams in [(False, False), (True, False), (False, True)]:
        a = emb.B200Assigner(0, precision="fp32", train_eager=eager, batched_streams=streams)
        a.load_rows(x)
        res.append(a.train_batched(inst, cfg))
        a.close()
    for r in res[1:]:
        for o, q in zip(res[0], r):
            assert np.array_equal(o.labels, q.labels) and same_f32(o.centroids, q.centroids)
            assert o.n_splits == q.n_splits
    assert res[0][0].n_splits > 0
    ref = orc.train(parts[0], ks[0], orc.make_config(nepochs=2.0), emulate=not orc.has_kernel("avx512"))
    check_same(res[0][0], ref)
    lines = open(tmp_path / "tune.txt").read().split()
    assert lines[0].startswith("b_search:d=16:") and 0 <= int(lines[1]) < 11  # eleven search variants
