"""The learned proposer: its network's gradients against the FP64 oracle
(oracle/mlp_oracle.py, itself pinned by finite differences here on the CPU),
the proposer assign's guarantees against the full exact search, and what the
trained network gains over the nearest-group-centroid proposer.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


# ---- CPU: the oracle itself -------------------------------------------------

def _random_params(rng, d, H, G, scale=0.5):
    L = mo.layout(d, H, G)
    p = np.zeros(L["total"], np.float32)
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        o, n = L[name]
        p[o:o + n] = rng.standard_normal(n).astype(np.float32) * np.float32(scale)
    o, n = L["mean"]
    p[o:o + n] = rng.standard_normal(n).astype(np.float32) * np.float32(0.1)
    o, n = L["istd"]
    p[o:o + n] = (1.0 + rng.random(n)).astype(np.float32)
    return p


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    d, H, G, m = 6, 8, 5, 7
    params = _random_params(rng, d, H, G)
    p, _ = mo.unpack(params, d, H, G, weights_bf16=False)
    x0 = rng.standard_normal((m, d))
    t = rng.integers(0, G, m)
    loss, g = mo.loss_and_grad(x0, t, p)
    assert np.isclose(loss, mo.loss_only(x0, t, p))
    eps = 1e-6
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        num = np.zeros_like(p[name])
        for idx in np.ndindex(p[name].shape):
            q = {k: v.copy() for k, v in p.items()}
            q[name][idx] += eps
            lp = mo.loss_only(x0, t, q)
            q[name][idx] -= 2 * eps
            lm = mo.loss_only(x0, t, q)
            num[idx] = (lp - lm) / (2 * eps)
        np.testing.assert_allclose(g[name], num, rtol=1e-5, atol=1e-8, err_msg=name)


def test_bf16_rounding_ties_to_even():
    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5, 3.0e38], np.float32)
    r = mo.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6 and r[3] == 1.0 and r[4] == -2.5
    assert np.isfinite(r[5])


def test_layout_blocks_aligned():
    L = mo.layout(96, 512, 256)
    assert all(L[n][0] % 8 == 0 for n in ("mean", "istd", "w1", "b1", "w2", "b2", "w3", "b3"))
    assert L["total"] == L["b3"][0] + 256


# ---- GPU ----------------------------------------------------------------------

D, K, G, TOP, HID = 48, 2048, 128, 8, 256  # shapes the fused tcgen05 forward pass covers


@pytest.fixture(scope="module")
def trained(emb):
    """Heavy-tailed rows, k = 2048 centroids from this engine's training, a
    proposer (128 groups, top 8) trained on the training run's labels."""
    xa = emb.datasets.heavy_tailed(140_000, D, latent=16, components=512, seed=21)
    x, xt = xa[:120_000], xa[120_000:]  # held-out rows of the same distribution
    a = emb.B200Assigner(0, precision="bf16x1")
    out = emb.train(x, D, K, emb.Config(nepochs=3.0), assigner=a)
    a.proposer_init(groups=G, hidden=HID, top=TOP, seed=5)
    losses = a.proposer_train(out.labels, 600)
    yield a, x, xt, out, losses
    a.close()


@pytest.mark.gpu
@pytest.mark.parametrize("d,H,Gs,m", [(40, 64, 24, 777), (20, 48, 13, 301)])
def test_gradients_match_fp64_oracle(emb, d, H, Gs, m):
    # The second shape has d, G and m off the 8-element row stride of the GEMM
    # operands (padded strides, zeros past the row).
    rng = np.random.default_rng(3)
    c = rng.standard_normal((200, d)).astype(np.float32)
    a = emb.B200Assigner(0, precision="bf16x1")
    a.set_centroids(c)
    a.proposer_init(groups=Gs, hidden=H, top=4, seed=1)
    params = a.proposer_params()
    L = mo.layout(d, H, Gs)
    assert params.size == L["total"]
    params = _random_params(rng, d, H, Gs, scale=0.3)
    a.set_proposer_params(params)
    assert np.array_equal(a.proposer_params(), params)
    x = (rng.standard_normal((m, d)) * 2 + 0.3).astype(np.float32)
    t = rng.integers(0, Gs, m).astype(np.uint32)
    loss, g = a.proposer_grad(x, t)
    a.close()
    p, _ = mo.unpack(params, d, H, Gs)
    x0 = mo.network_input(x, p["mean"], p["istd"])
    ref_loss, ref = mo.loss_and_grad(x0, t, p)
    # BF16 activations and activation gradients on the GPU, FP64 throughout in the
    # oracle: per-tensor relative L2 error within 2%, and the loss within 0.5%.
    assert abs(loss - ref_loss) <= 5e-3 * abs(ref_loss)
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        o, n = L[name]
        gg = g[o:o + n].astype(np.float64)
        rr = ref[name].reshape(-1)
        err = np.linalg.norm(gg - rr) / np.linalg.norm(rr)
        assert err < 2e-2, (name, err)
    for name in ("mean", "istd"):
        o, n = L[name]
        assert not g[o:o + n].any()


@pytest.mark.gpu
def test_fused_forward_matches_gemm_forward(trained):
    # The fused tcgen05 pass and the GEMM pass of training compute the same network
    # with BF16 activations and FP32 accumulation in different orders: logits agree
    # to BF16 rounding, and the proposals agree wherever the top-8 boundary is not a
    # near-tie.
    a, _, xt, _, _ = trained
    lf = a.proposer_logits(xt[:8192], fused=True)
    lg = a.proposer_logits(xt[:8192], fused=False)
    scale = np.abs(lg).max()
    assert np.abs(lf - lg).max() <= 2e-2 * scale, (np.abs(lf - lg).max(), scale)
    assert np.abs(lf - lg).mean() <= 2e-3 * scale
    groups, conf = a.propose(xt[:8192])
    ref = np.argsort(-lg, axis=1, kind="stable")[:, :TOP]
    same = np.mean([set(g) == set(r) for g, r in zip(groups, ref)])
    assert same > 0.98, same
    # confidence: softmax mass of the proposed groups
    z = lf - lf.max(1, keepdims=True)
    p = np.exp(z) / np.exp(z).sum(1, keepdims=True)
    mass = np.take_along_axis(p, groups.astype(np.int64), 1).sum(1)
    np.testing.assert_allclose(conf, mass, rtol=1e-3, atol=1e-4)
    # most likely first
    assert np.all(np.take_along_axis(lf, groups[:, :1].astype(np.int64), 1)[:, 0] >= lf.max(1) - 1e-6 * scale)


@pytest.mark.gpu
def test_training_reduces_loss(trained):
    _, _, _, _, losses = trained
    first, last = losses[:50].mean(), losses[-50:].mean()
    assert np.all(np.isfinite(losses))
    assert last < 0.5 * first, (first, last)


def _recall(groups_of_label, proposals):
    return float(np.mean([g in row for g, row in zip(groups_of_label, proposals)]))


@pytest.mark.gpu
def test_learned_proposer_beats_group_centroids(trained):
    a, _, xt, _, _ = trained
    lab_full, _ = a.assign(xt)
    gof = a.proposer_groups()
    target = gof[lab_full]
    a.proposer_set("mlp", TOP, 0.0)
    g_mlp, conf = a.propose(xt)
    a.proposer_set("centroids", TOP, 0.0)
    g_cen, _ = a.propose(xt)
    a.proposer_set("mlp", TOP, 0.0)
    r_mlp, r_cen = _recall(target, g_mlp), _recall(target, g_cen)
    assert np.all((conf > 0) & (conf <= 1.0 + 1e-6))
    # Held-out rows: the group of the exact label is among the network's top 8 more
    # often than among the 8 nearest group centroids.
    assert r_mlp > r_cen, (r_mlp, r_cen)
    assert r_mlp > 0.97, r_mlp


@pytest.mark.gpu
@pytest.mark.parametrize("mode,top,mass", [("mlp", TOP, 0.0), ("centroids", TOP, 0.0), ("mlp", 16, 0.99)])
def test_proposer_assign_guarantees(trained, orc, mode, top, mass):
    a, x, _, out, _ = trained
    a.proposer_set(mode, top, 0.0, mass)
    lab_p, dist_p = a.assign_proposed()
    st = a.stats()
    lab_f, dist_f = a.assign_resident()
    n = x.shape[0]
    assert st["rows_proposed"] + st["rows_lowconf"] == n
    assert st["fast_aborted"] == 0
    props, _, cnt = a.propose(x, with_counts=True)
    assert np.all((cnt >= 1) & (cnt <= top))
    if mass == 0.0:
        assert np.all(cnt == top)
    else:
        assert cnt.mean() < top
    # the grouped search scored exactly the proposed (row, group) pairs
    assert st["groups_searched"] == int(cnt.sum())
    gof = a.proposer_groups()
    covered = np.array([gof[l] in row[:c] for l, row, c in zip(lab_f, props, cnt)])
    same = lab_p == lab_f
    # 1. wherever the exact label's group was proposed, the label is the exact one
    assert np.all(same[covered])
    # 2. every distance is the exact distance of the returned label (reference rounding)
    assert np.array_equal(dist_p[same].view(np.uint32), dist_f[same].view(np.uint32))
    for i in np.nonzero(~same)[0][:300]:
        j = int(lab_p[i])
        _, de = orc.cpu_assign(x[i:i + 1], out.centroids[j:j + 1], emulate=True)
        assert de[0].view(np.uint32) == dist_p[i].view(np.uint32)
    # 3. elsewhere the returned label is never nearer than the exact one
    assert np.all(dist_p >= dist_f)
    recall = same.mean()
    assert recall > {"mlp": 0.98, "centroids": 0.9}[mode], recall
    a.proposer_set("mlp", TOP, 0.0)


@pytest.mark.gpu
def test_low_confidence_rows_take_the_full_search(trained):
    a, x, _, _, _ = trained
    a.proposer_set("mlp", TOP, 1.01)  # no row reaches it
    lab_p, dist_p = a.assign_proposed()
    st = a.stats()
    lab_f, dist_f = a.assign_resident()
    assert st["rows_lowconf"] == x.shape[0] and st["rows_proposed"] == 0
    assert np.array_equal(lab_p, lab_f) and np.array_equal(dist_p.view(np.uint32), dist_f.view(np.uint32))
    a.proposer_set("mlp", TOP, 0.9)
    lab_p, dist_p = a.assign_proposed()
    st = a.stats()
    assert 0 < st["rows_lowconf"] < x.shape[0]
    assert np.all(dist_p >= dist_f)
    a.proposer_set("mlp", TOP, 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("d", [96, 32])
def test_grouped_search_with_a_half_k_atom(emb, orc, d):
    # d = 96 and d = 32 leave a 32-wide K remainder: the grouped search covers it with
    # a 64-byte-swizzled half atom; the guarantees must hold exactly as for d = 48.
    x = emb.datasets.heavy_tailed(50_000, d, latent=12, components=256, seed=31)
    a = emb.B200Assigner(0, precision="bf16x1")
    out = emb.train(x, d, 1024, emb.Config(nepochs=2.0), assigner=a)
    a.proposer_init(groups=128, hidden=256, top=8, seed=3)
    a.proposer_train(out.labels, 300)
    lab_p, dist_p = a.assign_proposed()
    lab_f, dist_f = a.assign_resident()
    props, _ = a.propose(x)
    gof = a.proposer_groups()
    covered = np.array([gof[l] in row for l, row in zip(lab_f, props)])
    same = lab_p == lab_f
    assert np.all(same[covered])
    assert np.array_equal(dist_p[same].view(np.uint32), dist_f[same].view(np.uint32))
    assert np.all(dist_p >= dist_f)
    assert same.mean() > 0.9, same.mean()
    a.close()


@pytest.mark.gpu
def test_proposer_in_late_training_epochs(emb):
    # train() with the learned proposer searching the last epoch's batches: the
    # epochs before are the plain training's (bit for bit), the network is fitted
    # on the labels of the epoch before, and the result stays close to the full
    # search's: final MSE within 0.5 %, most last-pass labels equal. With no late
    # epoch the call is train() itself.
    x = emb.datasets.heavy_tailed(120_000, 48, latent=16, components=512, nu=3.0, seed=4)
    k = 2048
    cfg = emb.Config(nepochs=3.0)
    a = emb.B200Assigner(0, precision="bf16")
    a.load_rows(x)
    full = a.train_resident(k, cfg)
    same = a.train_resident_proposed(k, cfg, late_epochs=0, net_steps=10, groups=64, top=8)
    assert np.array_equal(same.labels, full.labels)
    assert np.array_equal(same.centroids.view(np.uint32), full.centroids.view(np.uint32))
    prop = a.train_resident_proposed(k, cfg, late_epochs=1, net_steps=1500, groups=64, top=16, mass=0.999)
    st = prop.stats
    assert st["rows_proposed"] > 0.5 * len(x), st
    assert np.mean(prop.labels == full.labels) > 0.9
    a.set_centroids(full.centroids)
    _, d_full = a.assign_resident()
    a.set_centroids(prop.centroids)
    _, d_prop = a.assign_resident()
    a.close()
    mse_full, mse_prop = d_full.astype(np.float64).mean(), d_prop.astype(np.float64).mean()
    assert abs(mse_prop / mse_full - 1.0) < 0.005, (mse_full, mse_prop)
