"""The command-line drivers (e-means_b200/cli.py), one per example of the
reference crate (examples/*.rs)."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "e-means_b200", "cli.py")


def _run(*args):
    return subprocess.run([sys.executable, CLI, *args], capture_output=True, text=True, timeout=600)


def test_usage_without_a_gpu():
    r = _run("--help")
    assert r.returncode == 0 and "cluster" in r.stdout and "outliers" in r.stdout
    r = _run("cluster")
    assert r.returncode == 2  # missing arguments, as the example's usage exit


@pytest.mark.gpu
def test_cluster_and_outliers(emb, tmp_path):
    x = emb.datasets.blobs(20_000, 16, n_blobs=128, seed=5)
    path = tmp_path / "v.f32"
    x.astype("<f4").tofile(path)
    out = tmp_path / "c.f32"
    r = _run("cluster", str(path), "16", "64", "--epochs", "2", "--out", str(out), "--precision", "fp32")
    assert r.returncode == 0, r.stderr
    assert "final MSE" in r.stdout and "wrote" in r.stdout
    a = emb.B200Assigner(0, precision="fp32")
    ref = emb.train(x, 16, 64, emb.Config(nepochs=2.0, verbose=True), assigner=a)
    got = np.fromfile(out, dtype="<f4").reshape(64, 16)
    assert np.array_equal(got, ref.centroids)
    prefix = tmp_path / "o"
    r = _run("outliers", str(path), "16", "64", "--epochs", "2", "--top", "50", "--prefix", str(prefix),
             "--precision", "fp32")
    assert r.returncode == 0, r.stderr
    assert "families" in r.stdout and "Top rows" in r.stdout
    a.set_centroids(ref.centroids)
    lab, _ = a.assign(x)
    assert np.array_equal(np.fromfile(f"{prefix}.labels.u32", dtype="<u4"), lab)
    assert open(f"{prefix}.clusters.tsv").read().count("\n") == 65
    assert open(f"{prefix}.outliers.tsv").read().count("\n") == 51
    a.close()


@pytest.mark.gpu
def test_int8_and_balance_sweeps(emb, tmp_path):
    x = emb.datasets.blobs(8_000, 8, n_blobs=64, seed=6)
    path = tmp_path / "v.f32"
    x.astype("<f4").tofile(path)
    r = _run("int8", str(path), "8", "32", "--epochs", "1", "--seeds", "1")
    assert r.returncode == 0, r.stderr
    assert "faiss calibration" in r.stdout and "int8-centroid search" in r.stdout
    r = _run("balance", str(path), "8", "32", "--epochs", "1", "--seeds", "1")
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("|") >= 12  # six lambdas, two columns each


def _oracle_outliers_text(orc, x, k, epochs, top, family_radius=1.25):
    """The stdout and files of examples/outliers.rs (its format strings,
    examples/outliers.rs:39-72), rendered from the oracle's train_cpu, assign and
    report. Equal values keep index order (the engine's documented tie rule)."""
    n, d = x.shape
    tr = orc.train(x, k, orc.make_config(nepochs=epochs), emulate=not orc.has_kernel("avx512"))
    cent = tr["centroids"]
    labels, sq = orc.cpu_assign(x, cent, emulate=not orc.has_kernel("avx512"))
    r = orc.report(labels, sq, cent, family_radius=family_radius)
    c, fams, lz, gz = r["clusters"], r["families"], r["local_z"], r["global_z"]

    def desc(v):  # f32::total_cmp descending, stable
        b = np.ascontiguousarray(v, np.float32).view(np.uint32)
        key = b ^ np.where(b >> 31 != 0, np.uint32(0xFFFFFFFF), np.uint32(0x80000000))
        return np.argsort(np.uint32(0xFFFFFFFF) - key, kind="stable")

    out = [f"{n} rows, {k} clusters, {len(fams)} families (radius {family_radius} x median centroid spacing "
           f"{r['median_nearest_dist']:.3f})",
           f"median distance to centroid {r['median_dist']:.3f}, median cluster rms {r['median_rms']:.3f}",
           "", "Largest families (prevalence):"]
    for (leader, members, _, share) in fams[:5]:
        out.append(f"  {100.0 * share:6.2f}% of rows in {len(members):4d} clusters (leader {leader})")
    singles = sum(1 for f in fams if len(f[1]) == 1)
    rare = sum(1 for f in fams if f[3] < 0.1 / k)
    out.append(f"  {singles} single-cluster families; {rare} families hold under a tenth of an average cluster")
    out += ["", "Loosest clusters (catch-alls):"]
    live = np.nonzero(c["size"])[0]
    for j in live[desc(c["looseness"][live])][:5]:
        out.append(f"  cluster {j:6d}: size {c['size'][j]:6d}, looseness {c['looseness'][j]:.2f}, "
                   f"rms {c['rms'][j]:.3f}, max {c['max'][j]:.3f}")
    out += ["", "Small, isolated clusters (rare prototypes):"]
    mean = np.float32(n) / np.float32(max(len(live), 1))
    sel = (c["size"] > 0) & (c["size"].astype(np.float32) <= np.float32(0.25) * mean) & (c["isolation"] >= np.float32(1.5))
    js = np.nonzero(sel)[0]
    for j in js[desc(c["isolation"][js])][:5]:
        out.append(f"  cluster {j:6d}: size {c['size'][j]:6d}, isolation {c['isolation'][j]:.2f}")
    score = np.fmax(lz, gz)
    z5 = int(np.count_nonzero(score > 5.0))
    out += ["", f"{z5} rows score above 5 ({100.0 * z5 / n:.3f}%). Top rows:"]
    best = desc(score)[:min(top, n)]
    for i in best[:5]:
        out.append(f"  row {i:9d}: score {score[i]:7.2f} (local {lz[i]:.2f}, global {gz[i]:.2f}), cluster {labels[i]}")
    tsv = ["row\tscore\tlocal_z\tglobal_z\tdist\tcluster\tcluster_size\tfamily_share"]
    for i in best:
        cl = c[labels[i]]
        tsv.append(f"{i}\t{score[i]:.3f}\t{lz[i]:.3f}\t{gz[i]:.3f}\t{np.sqrt(sq[i]):.5f}\t{labels[i]}\t{cl['size']}\t"
                   f"{fams[int(cl['family'])][3]:.6f}")
    return tr, labels, sq, out, tsv


@pytest.mark.gpu
def test_cli_matches_oracle(emb, orc, tmp_path):
    # examples/cluster.rs and examples/outliers.rs against the oracle: the written
    # centroids and labels bit for bit, the printed recipe and MSE fields, and
    # the whole outliers summary and outliers table as the example prints them.
    x = emb.datasets.blobs(30_000, 24, n_blobs=300, seed=9)
    n, d, k = 30_000, 24, 96
    path = tmp_path / "v.f32"
    x.astype("<f4").tofile(path)
    tr, labels, sq, text, tsv = _oracle_outliers_text(orc, x, k, 3.0, 40)
    cent = tr["centroids"]
    rec = orc.resolve_recipe(n, d, k, orc.make_config(nepochs=3.0))
    out = tmp_path / "c.f32"
    r = _run("cluster", str(path), str(d), str(k), "--epochs", "3", "--out", str(out))
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(out, dtype="<f4").reshape(k, d).view(np.uint32), cent.view(np.uint32))
    line = r.stdout.strip().splitlines()[-1]
    mse = float(np.sum(sq.astype(np.float64)) / n)
    assert f"| batch {rec['batch_size']} | alpha0 {rec['alpha0']:.4f} | revived {tr['n_splits']} |" in line
    assert line.endswith(f"| final MSE {mse:.4f} | wrote {out}")
    prefix = tmp_path / "o"
    r = _run("outliers", str(path), str(d), str(k), "--epochs", "3", "--top", "40", "--prefix", str(prefix))
    assert r.returncode == 0, r.stderr
    got = r.stdout.splitlines()
    assert got[:len(text)] == text
    assert got[len(text):] == ["", f"wrote {prefix}.clusters.tsv, {prefix}.outliers.tsv and {prefix}.labels.u32"]
    assert np.array_equal(np.fromfile(f"{prefix}.labels.u32", dtype="<u4"), labels)
    assert open(f"{prefix}.outliers.tsv").read().splitlines() == tsv
