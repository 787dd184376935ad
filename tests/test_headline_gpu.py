"""Parity at the headline configuration: 128-d embedding rows (32-d latent,
L2-normalised) against k = 16384 centroids trained by the engine's own e-means.

The labels and distances of every precision mode must equal the reference
CpuAssigner's (src/cpu.rs:108-167, AVX-512 rounding) bit for bit on 65,536 rows
that the training did not see, and agree with an FP64 brute force at least as
well as the reference's own GPU bar asks (>= 99.9 %, src/cuda.rs:243-247).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

K, D = 16384, 128


def same_f32(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.fixture(scope="module")
def headline(emb, orc):
    xt = emb.datasets.embeddings(262_144, D, seed=0)
    a = emb.B200Assigner(0, precision="bf16")
    a.load_rows(xt)
    out = a.train_resident(K, emb.Config(nepochs=2.0))
    a.close()
    x = emb.datasets.embeddings(65_536, D, seed=1)
    ref_l, ref_d = orc.cpu_assign(x, out.centroids, emulate=not orc.has_kernel("avx512"))
    return x, out.centroids, ref_l, ref_d


@pytest.mark.parametrize("precision", ["bf16x1", "bf16", "fp8", "fp32"])
def test_trained_k16384_bit_exact(emb, orc, headline, precision):
    x, c, ref_l, ref_d = headline
    a = emb.B200Assigner(0, precision=precision)
    a.set_centroids(c)
    a.load_rows(x)
    lab, dist = a.assign_resident()
    st = a.stats()
    a.close()
    assert st["fast_aborted"] == 0, st
    assert np.array_equal(lab, ref_l)
    assert same_f32(dist, ref_d)
    # the reference's FP64 tolerance (src/cpu.rs:303-305) and GPU agreement bar
    # (src/cuda.rs:243-247) on a sample
    idx = np.random.default_rng(2).choice(len(x), 4096, replace=False)
    bl, bd = orc.bruteforce_f64(x[idx], c)
    assert np.mean(lab[idx] == bl) >= 0.999
    assert np.all(np.abs(dist[idx] - bd) <= 1e-4 * (1 + bd))


def test_host_path_k16384_equals_resident(emb, headline):
    x, c, ref_l, ref_d = headline
    a = emb.B200Assigner(0, precision="bf16x1")
    a.set_centroids(c)
    lab, dist = a.assign(x)
    a.close()
    assert np.array_equal(lab, ref_l) and same_f32(dist, ref_d)
