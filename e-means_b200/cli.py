"""Command-line drivers of the B200 engine, one per example of the reference
crate (examples/cluster.rs, outliers.rs, int8.rs, balance.rs), with the same
inputs, options and printed summaries; every computation runs on the B200.

    python e-means_b200/cli.py cluster  vectors.f32 <d> <k> [--epochs 5] [--out centroids.f32]
                                        [--simd avx512|avx2|portable] [--gpu [ordinal]] [--precision fp32|bf16|bf16x1]
    python e-means_b200/cli.py outliers vectors.f32 <d> <k> [--epochs 5] [--balance 0] [--top 1000]
                                        [--family-radius 1.25] [--prefix out]
    python e-means_b200/cli.py int8     vectors.f32 <d> <k> [--epochs 5] [--seeds 3]
    python e-means_b200/cli.py balance  vectors.f32 <d> <k> [--epochs 5] [--seeds 5]

Input: raw little-endian f32, n x d row-major. Output files are written as the
examples write them (little-endian f32 centroids, u32 labels, TSV tables).
"""
import argparse
import importlib.util
import os
import sys
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _package():
    if "emeans_b200" in sys.modules:
        return sys.modules["emeans_b200"]
    spec = importlib.util.spec_from_file_location("emeans_b200", os.path.join(_HERE, "__init__.py"),
                                                  submodule_search_locations=[_HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["emeans_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def read_f32(path, d):
    x = np.fromfile(path, dtype="<f4")
    if x.size % d:
        raise SystemExit(f"{path}: {x.size} values are not whole rows of d = {d}")
    return np.ascontiguousarray(x.reshape(-1, d), np.float32)


def _mse(dist):
    return float(np.sum(dist.astype(np.float64)) / dist.size)


def cmd_cluster(args, emb):
    """examples/cluster.rs: train, exact assign, MSE, centroids written."""
    x = read_f32(args.input, args.d)
    ordinal = args.gpu if args.gpu is not None else 0
    a = emb.B200Assigner(ordinal, precision=args.precision, match=args.simd)
    cfg = emb.Config(nepochs=args.epochs, verbose=True)
    t = time.perf_counter()
    out = emb.train(x, args.d, args.k, cfg, assigner=a)
    train_s = time.perf_counter() - t
    a.set_centroids(out.centroids)
    _, dist = a.assign_resident()
    out.centroids.astype("<f4").tofile(args.out)
    print(f"{a.name()} | train {train_s:.2f} s | batch {out.recipe.batch_size} | alpha0 {out.recipe.alpha0:.4f} | "
          f"revived {out.n_splits} | final MSE {_mse(dist):.4f} | wrote {args.out}")
    a.close()


def cmd_outliers(args, emb):
    """examples/outliers.rs: train, assign, report(); summary, TSVs, labels."""
    x = read_f32(args.input, args.d)
    n, d, k = x.shape[0], args.d, args.k
    a = emb.B200Assigner(0, precision=args.precision)
    out = emb.train(x, d, k, emb.Config(nepochs=args.epochs, balance=args.balance), assigner=a)
    a.set_centroids(out.centroids)
    labels, sq = a.assign_resident()
    r = emb.report_resident(a, emb.ReportConfig(family_radius=args.family_radius))
    print(f"{n} rows, {k} clusters, {len(r.families)} families (radius {args.family_radius} x median centroid "
          f"spacing {r.median_nearest_dist:.3f})")
    print(f"median distance to centroid {r.median_dist:.3f}, median cluster rms {r.median_rms:.3f}")
    print("\nLargest families (prevalence):")
    for f in r.families[:5]:
        print(f"  {100.0 * f.share:6.2f}% of rows in {len(f.members):4d} clusters (leader {f.leader})")
    singles = sum(1 for f in r.families if len(f.members) == 1)
    rare = sum(1 for f in r.families if f.share < 0.1 / k)
    print(f"  {singles} single-cluster families; {rare} families hold under a tenth of an average cluster")
    c = r.clusters
    live = np.nonzero(c["size"])[0]
    key = np.uint32(0xFFFFFFFF) - emb._order_key(c["looseness"][live])
    print("\nLoosest clusters (catch-alls):")
    for j in live[np.argsort(key, kind="stable")][:5]:
        print(f"  cluster {j:6d}: size {c['size'][j]:6d}, looseness {c['looseness'][j]:.2f}, rms {c['rms'][j]:.3f}, "
              f"max {c['max'][j]:.3f}")
    print("\nSmall, isolated clusters (rare prototypes):")
    for j, size, iso in r.rare_prototypes(0.25, 1.5)[:5]:
        print(f"  cluster {j:6d}: size {size:6d}, isolation {iso:.2f}")
    scores = r.scores()
    z5 = int(np.count_nonzero(scores > 5.0))
    print(f"\n{z5} rows score above 5 ({100.0 * z5 / n:.3f}%). Top rows:")
    best = r.top_outliers(args.top)
    for i, s in best[:5]:
        print(f"  row {i:9d}: score {s:7.2f} (local {r.local_z[i]:.2f}, global {r.global_z[i]:.2f}), "
              f"cluster {labels[i]}")
    with open(f"{args.prefix}.clusters.tsv", "w") as w:
        r.write_clusters_tsv(w)
    with open(f"{args.prefix}.outliers.tsv", "w") as w:
        w.write("row\tscore\tlocal_z\tglobal_z\tdist\tcluster\tcluster_size\tfamily_share\n")
        for i, s in best:
            cl = c[labels[i]]
            w.write(f"{i}\t{s:.3f}\t{r.local_z[i]:.3f}\t{r.global_z[i]:.3f}\t{np.sqrt(sq[i]):.5f}\t{labels[i]}\t"
                    f"{cl['size']}\t{r.families[int(cl['family'])].share:.6f}\n")
    labels.astype("<u4").tofile(f"{args.prefix}.labels.u32")
    print(f"\nwrote {args.prefix}.clusters.tsv, {args.prefix}.outliers.tsv and {args.prefix}.labels.u32")
    a.close()


def cmd_int8(args, emb):
    """examples/int8.rs: f32 clustering against int8 codes (faiss and clipped
    calibrations); MSE from an exact f32 assign of the original rows to the
    decoded centroids."""
    x = read_f32(args.input, args.d)
    n, d, k = x.shape[0], args.d, args.k
    exact = emb.B200Assigner(0, precision="bf16")  # CpuAssigner results, tensor-core fast path

    def mse(centroids):
        exact.set_centroids(centroids)
        _, dist = exact.assign(x)
        return _mse(dist)

    print(f"{n} x {d}, k = {k}, {args.epochs} epochs, mean of {args.seeds} seeds")
    print(f"{'configuration':<46} {'train s':>8} {'MSE':>12} {'vs f32':>9}")
    base = [0.0]

    def row(name, run):
        secs = err = 0.0
        for seed in range(args.seeds):
            cfg = emb.Config(nepochs=args.epochs, seed=1234 + seed)
            t = time.perf_counter()
            centroids = run(cfg)
            secs += (time.perf_counter() - t) / args.seeds
            err += mse(centroids) / args.seeds
        if base[0] == 0.0:
            base[0] = err
        print(f"{name:<46} {secs:>8.2f} {err:>12.6f} {100.0 * (err / base[0] - 1.0):>+8.3f}%")

    def train_with(rows, **opts):
        def run(cfg):
            a = emb.B200Assigner(0, **opts)
            out = emb.train(rows, d, k, cfg, assigner=a)
            a.close()
            return out.centroids
        return run

    row("f32 rows, f32 search", train_with(x, precision="fp32"))
    for label, cal in (("faiss calibration", emb.Calibration.faiss()),
                       ("clipped at 99.99%", emb.Calibration.clipped(0.9999))):
        q = emb.Int8Quantizer.fit(x, d, cal, assigner=exact)
        codes = q.encode(x, assigner=exact)
        print(f"-- int8 codes, {label}: scale {q.scale:.4f}, "
              f"{100.0 * q.clipped_fraction(x, assigner=exact):.4f}% of values clipped")
        f32_on_codes = train_with(codes, precision="fp32")
        row("  f32 search (exact on the codes)", lambda cfg: q.decode(f32_on_codes(cfg), assigner=exact))
        i16 = train_with(codes, precision="fp32", centroid_bits=16)
        row("  int16-centroid search (dp2a)", lambda cfg: q.decode(i16(cfg), assigner=exact))
        i8 = train_with(codes, precision="fp32", centroid_bits=8)
        row("  int8-centroid search (kind::i8, as faiss)", lambda cfg: q.decode(i8(cfg), assigner=exact))
    exact.close()


def cmd_balance(args, emb):
    """examples/balance.rs: sweep the balance penalty; MSE and balance of the
    nearest-centroid labels and of training's penalised last-pass labels. The
    penalised MSE is the reference example's own f64 sum over rows."""
    x = read_f32(args.input, args.d)
    n, d, k = x.shape[0], args.d, args.k
    print(f"{n} x {d}, k = {k}, {args.epochs} epochs, mean over {args.seeds} seeds (sd of MSE in brackets)")
    print("lambda | nearest: MSE [sd]    vs 0   imbal  max/mean | penalized: MSE   vs 0   imbal  max/mean  empty")
    base = 0.0
    for lam in (0.0, 0.03, 0.1, 0.3, 1.0, 3.0):
        acc = np.zeros(7)
        sq = 0.0
        for seed in range(args.seeds):
            a = emb.B200Assigner(0, precision="fp32")
            out = emb.train(x, d, k, emb.Config(nepochs=args.epochs, balance=lam, seed=1234 + seed), assigner=a)
            a.set_centroids(out.centroids)
            near, dist = a.assign_resident()
            a.close()
            mse_near = _mse(dist)
            diff = (x - out.centroids[out.labels]).astype(np.float64)
            mse_pen = float(np.sum(diff * diff) / n)
            ni, nm, _ = emb.balance_stats(near, k)
            pi, pm, pe = emb.balance_stats(out.labels, k)
            acc += np.array([mse_near, ni, nm, mse_pen, pi, pm, pe], np.float64) / args.seeds
            sq += mse_near * mse_near / args.seeds
        sd = max(sq - acc[0] * acc[0], 0.0) ** 0.5
        if lam == 0.0:
            base = acc[0]
        print(f"{lam:6.2f} | {acc[0]:10.3f} [{sd:5.2f}] {100.0 * (acc[0] / base - 1.0):+6.2f}%  {acc[1]:5.2f}  "
              f"{acc[2]:8.1f} | {acc[3]:14.3f} {100.0 * (acc[3] / base - 1.0):+6.2f}%  {acc[4]:5.2f}  {acc[5]:8.1f}  "
              f"{acc[6]:5.1f}")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="cli.py", description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("cluster", "outliers", "int8", "balance"):
        p = sub.add_parser(name)
        p.add_argument("input")
        p.add_argument("d", type=int)
        p.add_argument("k", type=int)
        p.add_argument("--epochs", type=float, default=5.0)
        if name == "cluster":
            p.add_argument("--out", default="centroids.f32")
            p.add_argument("--simd", default="avx512", choices=["avx512", "avx2", "portable"],
                           help="which CpuAssigner kernel's rounding the results reproduce")
            p.add_argument("--gpu", type=int, nargs="?", const=0, default=None, help="device ordinal")
        if name in ("cluster", "outliers"):
            p.add_argument("--precision", default="bf16x1", choices=["fp32", "bf16", "bf16x1"])
        if name == "outliers":
            p.add_argument("--balance", type=float, default=0.0)
            p.add_argument("--top", type=int, default=1000)
            p.add_argument("--family-radius", type=float, default=1.25)
            p.add_argument("--prefix", default="out")
        if name in ("int8", "balance"):
            p.add_argument("--seeds", type=int, default=3 if name == "int8" else 5)
    args = ap.parse_args(argv)
    emb = _package()
    {"cluster": cmd_cluster, "outliers": cmd_outliers, "int8": cmd_int8, "balance": cmd_balance}[args.cmd](args, emb)


if __name__ == "__main__":
    main()
