"""Benchmark of the B200 e-means engine on its headline workload.

Metric: rows/s assigned at 1,000,000 x 128-D f32 embedding-like rows against
k = 16384 centroids (the exact nearest-centroid pass of src/lib.rs:512-520).
A step is one full assign pass over the 1M resident rows. The centroids are
the output of the engine's own e-means training on the same rows (untimed).

  value : rows/s with the rows resident in HBM (device-timed, CUDA events)
  e2e   : rows/s through the public C ABI with host buffers (pinned host rows
          copied in, labels and distances copied out, inside the timed region)

`--impl reference` times the reference's CPU implementation (its CpuAssigner
restated in C++, oracle/) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ROWS, DIM, K = 1_000_000, 128, 16384
WORKLOAD = "embeddings 1,000,000 x 128 f32 (32-d latent, L2-normalised), k=16384, exact assign pass"
METRIC = "rows/s assigned (1M x 128-D, k=16384)"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                vals = [v.strip() for v in out.stdout.strip().split(",")]
                if len(vals) == 6:
                    self.samples.append(vals)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return {"hbm_gbs": j["hbm_gbs"], "bf16_tflops": j["bf16_tflops"],
                "bf16_tflops_sustained": j.get("bf16_tflops_sustained"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


def make_workload(seed=0):
    from __graft_entry__ import load_package

    emb = load_package()
    x = emb.datasets.embeddings(N_ROWS, DIM, seed=seed)
    return emb, x


def trained_centroids(emb, x, cache=True):
    """k=16384 centroids from the engine's own e-means (2 epochs) on the rows."""
    path = os.path.join(ROOT, "gpurun_out", "bench_centroids_c2.npy")
    if cache and os.path.exists(path):
        return np.load(path)
    a = emb.B200Assigner(0, precision="bf16")
    try:
        a.load_rows(x)
        out = a.train_resident(K, emb.Config(nepochs=2.0))
        c = out.centroids
    except emb.EngineError:
        # Training not available: seed centroids from a fixed sample of rows.
        c = x[np.random.default_rng(1).choice(len(x), K, replace=False)].copy()
    finally:
        a.close()
    if cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.save(path, c)
    return c


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    emb, x = make_workload(seed=0)
    cent = trained_centroids(emb, x, cache=(world == 1))
    peaks = measured_peaks()
    results = {}
    for prec in args.precisions:
        a = emb.B200Assigner(local, precision=prec)
        a.set_centroids(cent)
        a.load_rows(x)
        results[prec] = time_resident(a, emb, args, prec, world)
        a.close()
    head = args.precisions[0]
    r = results[head]
    value = r["rows_per_s_total"]
    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp32": "f32", "bf16": "bf16x3->f32", "bf16x1": "bf16->f32"}[head],
        "data": "synthetic (seeded numpy generator, shapes and distribution of the workload)",
        "config": {"workload": WORKLOAD, "rows_per_gpu": N_ROWS, "d": DIM, "k": K, "precision": head,
                   "l2": "inputs (512 MB of rows) larger than L2", "parallelism": f"replicas x{world}"},
        "per_precision": {p: {"rows_per_s": results[p]["rows_per_s_total"], "ms_per_step": results[p]["ms_per_step"],
                              "refined_rows": results[p]["refined"], "researched_rows": results[p]["researched"]}
                          for p in results},
        "gpu_launches": r["launches"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def time_resident(a, emb, args, prec, world):
    import torch

    for _ in range(args.warmup):
        a.assign_resident(want_host=False)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(args.steps):
        a.assign_resident(want_host=False)
        ms.append(a.stats()["ms_total"])
    st = a.stats()
    t = float(np.sum(ms))
    if world > 1:
        tt = torch.tensor([t], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t = float(tt.item())
    rows = N_ROWS * args.steps * world
    return {"rows_per_s_total": rows / (t / 1e3), "ms_per_step": t / args.steps, "researched": st["rows_researched"],
            "refined": st["rows_refined"],
            "launches": st["kernel_launches"] * args.steps}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc

    _, x = make_workload(seed=0)
    cent = x[np.random.default_rng(1).choice(len(x), K, replace=False)].copy()
    sample = 16384
    cores = os.cpu_count()
    kern = "avx512" if orc.has_kernel("avx512") else ("avx2" if orc.has_kernel("avx2") else "portable")
    for _ in range(args.warmup and 1):
        orc.cpu_assign(x[:1024], cent, kernel=kern)
    ts = []
    for s in range(args.steps):
        r0 = (s * sample) % (N_ROWS - sample)
        t0 = time.perf_counter()
        orc.cpu_assign(x[r0:r0 + sample], cent, kernel=kern)
        ts.append(time.perf_counter() - t0)
    rps = sample * len(ts) / sum(ts)
    line = {"metric": METRIC, "value": rps, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * N_ROWS / rps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "rows_per_gpu": N_ROWS, "d": DIM, "k": K},
            "cpu_baseline": {"value": rps, "unit": "rows/s", "cores": cores, "kind": "port",
                             "sample": f"{sample} rows per step x {args.steps} steps of the 1M-row pass, CpuAssigner "
                                       f"{kern} kernel restated in C++ (OpenMP, {cores} threads)"},
            "e2e": {"value": rps, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precisions", default="fp32", help="comma list; the first is the headline")
    args = ap.parse_args()
    args.precisions = args.precisions.split(",")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
