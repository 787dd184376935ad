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
