"""report() (src/report.rs:121-241): the device version against the oracle's
restatement, field by field and bit for bit, plus the reference's own test."""
import io

import numpy as np
import pytest


def _reference_case():
    # src/report.rs:297-313: 1-D, two big clusters at 0 and 1, a tiny one at 50
    centroids = np.array([[0.0], [1.0], [50.0]], np.float32)
    labels, sq = [], []
    for i in range(200):
        off = np.float32(0.001) * np.float32(i % 100)
        labels.append(i % 2)
        sq.append(off * off)
    labels.append(0)
    sq.append(np.float32(0.45) * np.float32(0.45))  # a fringe point of cluster 0: row 200
    for _ in range(3):
        labels.append(2)
        sq.append(np.float32(1e-4))
    return np.array(labels, np.uint32), np.array(sq, np.float32), centroids


def _check_reference_expectations(r):
    # src/report.rs:314-324
    assert r.clusters["size"].tolist() == [101, 100, 3]
    assert r.top_outliers(1)[0][0] == 200
    assert r.local_z[200] > 10.0
    assert len(r.families) == 2
    assert r.families[0].size == 201
    assert r.clusters[0]["family"] == r.clusters[1]["family"]
    assert r.rare_prototypes(0.25, 2.0) == [(2, 3, np.float32(49.0))]
    buf = io.StringIO()
    r.write_clusters_tsv(buf)
    assert buf.getvalue().count("\n") == 4


def _oracle_report(emb, orc, labels, sq, c, cfg=None):
    cfg = cfg or emb.ReportConfig()
    o = orc.report(labels, sq, c, cfg.family_radius, cfg.min_local_size)
    fams = [emb.Family(l, m, s, sh) for l, m, s, sh in o["families"]]
    return emb.Report(o["clusters"].view(emb.CLUSTER_STATS), fams, o["local_z"], o["global_z"], o["median_dist"],
                      o["median_rms"], o["median_nearest_dist"])


def test_reference_expectations_on_the_oracle(emb, orc):
    labels, sq, c = _reference_case()
    _check_reference_expectations(_oracle_report(emb, orc, labels, sq, c))


def _same_bits(a, b):
    """Bit-identical, except that any NaN equals any NaN: a NaN's payload is the
    hardware's (the GPU's canonical NaN, x86's default NaN for inf / inf)."""
    a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
    if a.dtype.kind != "f":
        return np.array_equal(a, b)
    a32, b32 = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    same = a32.view(np.uint32) == b32.view(np.uint32)
    return bool(np.all(same | (np.isnan(a32) & np.isnan(b32))))


def _assert_same(r, o):
    for f in r.clusters.dtype.names:
        assert _same_bits(r.clusters[f], o.clusters[f]), f
    assert _same_bits(r.local_z, o.local_z)
    assert _same_bits(r.global_z, o.global_z)
    for f in ("median_dist", "median_rms", "median_nearest_dist"):
        assert _same_bits(getattr(r, f), getattr(o, f)), f
    assert len(r.families) == len(o.families)
    for a, b in zip(r.families, o.families):
        assert (a.leader, a.size, a.share) == (b.leader, b.size, b.share)
        assert np.array_equal(a.members, b.members)


@pytest.mark.gpu
def test_reference_case_on_the_gpu(emb, orc):
    labels, sq, c = _reference_case()
    r = emb.report(labels, sq, c, 1)
    _check_reference_expectations(r)
    _assert_same(r, _oracle_report(emb, orc, labels, sq, c))


def _synthetic(n, k, d, seed, empty=0.1, dup=0.0):
    rng = np.random.default_rng(seed)
    c = (rng.standard_normal((k, d)) * rng.uniform(0.5, 3.0, (k, 1))).astype(np.float32)
    live = np.nonzero(rng.random(k) >= empty)[0]
    w = rng.pareto(1.5, live.size) + 0.1
    labels = live[rng.choice(live.size, n, p=w / w.sum())].astype(np.uint32)
    sq = (rng.gamma(2.0, 1.0, n) * rng.uniform(0.2, 2.0, k)[labels]).astype(np.float32)
    if dup:
        sq[rng.random(n) < dup] = np.float32(1.0)  # repeated distances (ties inside clusters)
    return labels, sq, c


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,d", [(0, 5, 3), (1, 1, 1), (7, 3, 16), (500, 40, 15), (3000, 64, 37),
                                   (20000, 200, 128), (50000, 1000, 8), (4000, 33, 200), (60000, 30000, 8)])
def test_report_matches_oracle(emb, orc, n, k, d):
    labels, sq, c = _synthetic(n, k, d, seed=n + k + d, dup=0.05)
    o = _oracle_report(emb, orc, labels, sq, c)
    for family_pass in (1, 2):  # parallel rounds, sequential greedy
        r = emb.report(labels, sq, c, d, emb.ReportConfig(family_pass=family_pass))
        _assert_same(r, o)


@pytest.mark.gpu
def test_report_edge_values(emb, orc):
    # negative, NaN and zero squared distances (max(0) then sqrt), a cluster of
    # equal distances (MAD 0 -> global z), sizes around min_local_size, equal
    # cluster sizes (index order), coincident centroids (nearest distance 0)
    rng = np.random.default_rng(4)
    k, d = 12, 20
    c = rng.standard_normal((k, d)).astype(np.float32)
    c[5] = c[4]
    sizes = [30, 29, 31, 30, 30, 0, 1, 2, 100, 100, 7, 0]
    labels = np.concatenate([np.full(s, j, np.uint32) for j, s in enumerate(sizes)])
    sq = rng.gamma(2.0, 1.0, labels.size).astype(np.float32)
    sq[labels == 0] = 2.0
    sq[:3] = [-1.0, np.nan, 0.0]
    sq[40:43] = [-0.0, np.inf, 1e-30]
    for cfg in (emb.ReportConfig(), emb.ReportConfig(family_radius=3.0, min_local_size=1),
                emb.ReportConfig(family_radius=3.0, min_local_size=1, family_pass=2),
                emb.ReportConfig(family_radius=100.0, family_pass=1),
                emb.ReportConfig(family_radius=0.0, min_local_size=1000)):
        r = emb.report(labels, sq, c, d, cfg)
        _assert_same(r, _oracle_report(emb, orc, labels, sq, c, cfg))


@pytest.mark.gpu
def test_report_rejects_bad_labels(emb):
    with pytest.raises(emb.EngineError):
        emb.report(np.array([0, 3], np.uint32), np.ones(2, np.float32), np.zeros((3, 2), np.float32), 2)


@pytest.mark.gpu
def test_report_after_training_and_resident(emb, orc):
    x = emb.datasets.blobs(200_000, 32, n_blobs=512, seed=3)
    a = emb.B200Assigner(0, precision="bf16x1")
    out = emb.train(x, 32, 1024, emb.Config(nepochs=2.0), assigner=a)
    a.set_centroids(out.centroids)
    labels, sq = a.assign_resident()
    r = emb.report_resident(a)
    o = _oracle_report(emb, orc, labels, sq, out.centroids)
    _assert_same(r, o)
    _assert_same(emb.report(labels, sq, out.centroids, 32, assigner=a), o)
    assert sum(f.size for f in r.families) == 200_000
    assert np.isclose(sum(f.share for f in r.families), 1.0)
    a.close()


@pytest.mark.gpu
def test_report_argument_errors(emb):
    c = np.zeros((3, 2), np.float32)
    ones = np.ones(4, np.float32)
    with pytest.raises(emb.EngineError, match="family_pass"):
        emb.report(np.zeros(4, np.uint32), ones, c, 2, emb.ReportConfig(family_pass=3))
    with pytest.raises(emb.EngineError, match="k <="):
        emb.report(np.zeros(4, np.uint32), ones, np.zeros((131073, 1), np.float32), 1)
    a = emb.B200Assigner(0)
    a.load_rows(np.zeros((4, 2), np.float32))
    a.set_centroids(c)
    with pytest.raises(emb.EngineError, match="assign_resident"):  # nothing assigned yet
        emb.report_resident(a)
    a.assign_resident()
    r = emb.report_resident(a)
    assert r.clusters["size"].sum() == 4
    a.set_centroids(c * 2)  # new centroids: the resident results are stale
    with pytest.raises(emb.EngineError, match="assign_resident"):
        emb.report_resident(a)
    a.close()
