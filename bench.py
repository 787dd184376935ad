"""Benchmark of the B200 e-means engine on its headline workload.

Workload: the exact nearest-centroid pass (assign(), src/lib.rs:512-520) over
1,000,000 x 128-D f32 embedding-like rows (32-d N(0,1) latent through a random
Gaussian map, N(0, 0.1^2) noise, L2-normalised; seeded synthetic data) against
k = 16384 centroids trained by the engine's own e-means on the same rows
(2 epochs, untimed). A step is one full pass over the 1M rows.

  value   rows/s with the rows resident in HBM (device-timed with CUDA events on
          the engine's stream; the 512 MB of rows exceed the 126 MB L2)
  e2e     rows/s through the public C ABI call (emb200_assign_f32) with pinned
          host rows: the host->device copy of the rows and the device->host copy
          of labels and distances are inside the timed region
  roofline  the fast contraction kernel (tcgen05): algorithmic flops 2 d k per
          row / its CUDA-event time, against the measured BF16 tensor peak

Every number comes from the bit-exact pipeline: labels and distances equal the
reference CpuAssigner's (AVX-512 rounding) for every row.

`--impl reference` times the reference's CPU search (its CpuAssigner, restated
in C++ in oracle/) on the host cores over a bounded sample of the same rows.
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
WORKLOAD = "assign 1,000,000 x 128 f32 embedding rows (32-d latent, L2-normalised) to k=16384 trained centroids"
METRIC = "rows/s assigned (1M x 128-D, k=16384)"
DTYPES = {"fp32": "f32", "bf16": "bf16x3 (hi/lo split) -> f32 accumulate", "bf16x1": "bf16 -> f32 accumulate",
          "fp8": "e4m3 (power-of-two scale per row and per centroid) -> f32 accumulate"}
CPU_SAMPLE_ROWS = 262_144


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
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

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(s[0]) for s in self.samples if num(s[0]) is not None]
        mx = [num(s[1]) for s in self.samples if num(s[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return {"hbm_gbs": j["hbm_gbs"], "bf16_tflops": j["bf16_tflops"],
                "bf16_tflops_sustained": j.get("bf16_tflops_sustained", j["bf16_tflops"]), "source": "of measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "of fallback"}


def profiled_traffic_per_row():
    """DRAM bytes per row of the fast kernel from the committed ncu summary (or None)."""
    p = os.path.join(ROOT, "profiles", "tc_assign_embeddings_1Mx128_k16384.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_row:"):
            return float(line.split(":")[1])
    return None


def make_rows(seed=0):
    from __graft_entry__ import load_package

    emb = load_package()
    return emb, emb.datasets.embeddings(N_ROWS, DIM, seed=seed)


def set_rows(n):
    """Smaller passes of the same workload (profiling captures); the default is 1M."""
    global N_ROWS
    N_ROWS = n


def centroid_note(kind):
    if kind == "trained":
        return ("k=16384 e-means centroids, 2 epochs of train() on the 1M rows (Config defaults, seed 1234); "
                "the engine's and the oracle's train() give the same bits")
    return "k=16384 rows sampled with seed 1, scaled by 0.97 (profiling captures)"


def trained_centroids(emb, x, ordinal):
    """k = 16384 centroids from the engine's own e-means (2 epochs) on the rows."""
    a = emb.B200Assigner(ordinal, precision="bf16")
    a.load_rows(x)
    out = a.train_resident(K, emb.Config(nepochs=2.0))
    a.close()
    return out.centroids


def init_dist(world, backend="nccl", timeout_s=600):
    """One process per GPU: a process group over NCCL (gloo in the CPU tests of
    this plumbing) with a bounded timeout, so that ranks waiting on a lost peer
    end with an error."""
    if world == 1:
        return
    from datetime import timedelta

    import torch.distributed as dist

    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def shard_seed(rank):
    """Seed of a rank's rows: every rank assigns its own shard (rank 0 holds the
    single-GPU rows), against centroids trained on rank 0's rows."""
    return rank


def job_rows_per_s(rows_per_rank, world, ms_per_step):
    """Whole-job throughput: the rows of all ranks over the slowest rank's time."""
    return rows_per_rank * world / (ms_per_step / 1e3)


def allreduce_max(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch

    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        if torch.cuda.is_available():
            torch.cuda.synchronize()


def time_resident(a, steps, warmup, world):
    for _ in range(warmup):
        a.assign_resident(want_host=False)
    barrier(world)
    ms, fast_ms, launches, fast_launches, refined, researched = [], 0.0, 0, 0, 0, 0
    for _ in range(steps):
        a.assign_resident(want_host=False)
        st = a.stats()
        ms.append(st["ms_total"])
        fast_ms += st["fast_ms"]
        fast_launches += st["fast_launches"]
        launches += st["kernel_launches"]
        refined += st["rows_refined"]
        researched += st["rows_researched"]
    barrier(world)
    t = allreduce_max(float(np.sum(ms)), world)
    return {"ms_total": t, "ms_per_step": t / steps, "fast_ms_per_launch": fast_ms / max(fast_launches, 1),
            "launches": launches, "refined_per_step": refined / steps, "researched_per_step": researched / steps}


def time_e2e(emb, a, x, steps, warmup, world):
    """The C-ABI host call on pinned buffers: copies in, search, copies out."""
    import torch

    xp = torch.from_numpy(x).pin_memory()
    lab = torch.empty(N_ROWS, dtype=torch.int32).pin_memory()
    dst = torch.empty(N_ROWS, dtype=torch.float32).pin_memory()
    for _ in range(warmup):
        a.assign_host_ptr(xp.data_ptr(), emb.EMB200_F32, N_ROWS, lab.data_ptr(), dst.data_ptr())
    barrier(world)
    ms = []
    for _ in range(steps):
        a.assign_host_ptr(xp.data_ptr(), emb.EMB200_F32, N_ROWS, lab.data_ptr(), dst.data_ptr())
        ms.append(a.stats()["ms_total"])
    barrier(world)
    t = allreduce_max(float(np.sum(ms)), world)
    return t / steps


def cpu_baseline(x, cent, rows=None):
    """The oracle's CpuAssigner on the first rows, timed on all host cores.
    Returns the cpu_baseline entry and the oracle's labels and distances."""
    rows = min(rows or CPU_SAMPLE_ROWS, len(x))
    from oracle import oracle as orc

    kern = "avx512" if orc.has_kernel("avx512") else ("avx2" if orc.has_kernel("avx2") else "portable")
    cores = os.cpu_count() or 1
    orc.cpu_assign(x[:256], cent, kernel=kern, nthreads=cores)  # warm the library and threads
    t0 = time.perf_counter()
    lab, dist = orc.cpu_assign(x[:rows], cent, kernel=kern, nthreads=cores)
    dt = time.perf_counter() - t0
    info = {"value": rows / dt, "unit": "rows/s", "cores": cores, "kind": "port",
            "sample": f"first {rows} of the 1M rows, k=16384: the reference CpuAssigner ({kern} kernel, 256 KB "
                      f"blocking, 4x4 micro-kernel) restated in C++, OpenMP over {cores} host threads, {dt:.2f} s"}
    return info, kern, lab, dist


def parity_check(x, cent, lab, dist, ref=None, fp64_rows=16384):
    """Labels and distances of the device pass against the oracle: bit for bit
    against the reference CpuAssigner in AVX-512 rounding (the engine's default
    match kernel) on the rows `ref` covers, and against an FP64 brute force on a
    seeded sample of rows."""
    from oracle import oracle as orc

    out = {}
    if ref is not None:
        rl, rd = ref
        n = len(rl)
        out.update({"reference_rows_checked": n, "labels_equal": bool(np.array_equal(lab[:n], rl)),
                    "dist_bit_exact": bool(np.array_equal(dist[:n].view(np.uint32), rd.view(np.uint32)))})
    idx = np.sort(np.random.default_rng(12345).choice(len(x), min(fp64_rows, len(x)), replace=False))
    bl, bd = orc.bruteforce_f64(x[idx], cent)
    err = np.abs(dist[idx].astype(np.float64) - bd)
    out.update({"fp64_rows_checked": len(idx), "fp64_agreement": float(np.mean(lab[idx] == bl)),
                "sqdist_max_abs_err": float(err.max()),
                "sqdist_max_rel_err": float((err / np.maximum(np.abs(bd), 1e-30)).max()),
                "within_reference_tolerance": bool(np.all(err <= 1e-4 * (1.0 + bd))),
                "tolerance": "labels and distances bit-exact vs the reference CpuAssigner (AVX-512 rounding); "
                             "|d - d_fp64| <= 1e-4 (1 + d_fp64) as src/cpu.rs:303-305; label agreement with FP64 "
                             ">= 0.999 as src/cuda.rs:243-247"})
    return out


def centroid_digest(cent):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(cent, np.float32).tobytes()).hexdigest()[:16]


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    init_dist(world)
    emb, x0 = make_rows(seed=0)
    if args.centroids == "trained":
        cent = trained_centroids(emb, x0, local)
    else:  # profiling captures: no training launches before the measured ones
        cent = x0[np.random.default_rng(1).choice(len(x0), K, replace=False)] * np.float32(0.97)
    x = x0 if shard_seed(rank) == 0 else make_rows(seed=shard_seed(rank))[1]
    del x0
    peaks = measured_peaks()
    results, outputs = {}, {}
    sampler = ClockSampler(local)
    with sampler:
        for prec in args.precisions:
            a = emb.B200Assigner(local, precision=prec)
            a.set_centroids(cent)
            a.load_rows(x)
            steps = args.steps if prec not in ("fp32", "fp8") else max(1, min(args.steps, 3))
            results[prec] = time_resident(a, steps, args.warmup, world)
            results[prec]["steps"] = steps
            if prec == args.precisions[0]:
                e2e_ms = time_e2e(emb, a, x, args.steps, args.warmup, world)
            outputs[prec] = a.assign_resident()  # untimed: the results checked below
            a.close()
    head = args.precisions[0]
    r = results[head]
    value = job_rows_per_s(N_ROWS, world, r["ms_per_step"])
    flops_per_launch = 2.0 * DIM * K * N_ROWS
    achieved = flops_per_launch / (r["fast_ms_per_launch"] / 1e3) / 1e12
    # The kernel is timed in a loop of well under a second: the burst peak.
    peak = peaks["bf16_tflops"]
    tpr = profiled_traffic_per_row()
    workload, metric = WORKLOAD, METRIC
    if N_ROWS != 1_000_000 or args.centroids != "trained":  # profiling passes name their own size
        workload = (f"assign {N_ROWS:,} x 128 f32 embedding rows (32-d latent, L2-normalised) to k=16384 "
                    f"{args.centroids} centroids")
        metric = f"rows/s assigned ({N_ROWS:,} x 128-D, k=16384)"
    line = {
        "metric": metric, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPES[head],
        "data": "synthetic: seeded numpy embedding rows of the workload's shape and distribution",
        "config": {"workload": workload, "rows_per_gpu": N_ROWS, "rows_per_step": N_ROWS, "d": DIM, "k": K,
                   "centroids": centroid_note(args.centroids), "centroid_digest": centroid_digest(cent),
                   "precision": head,
                   "l2": (f"no flush: the {N_ROWS * DIM * 4 / 1e6:.0f} MB of resident rows per pass "
                          + ("exceed the 126 MB L2" if N_ROWS * DIM * 4 > 126e6 else
                             "fit in the 126 MB L2 (a profiling pass, not a bench line)")),
                   "parallelism": f"{world} independent replicas (rows shard, no collective)"},
        "e2e": {"value": job_rows_per_s(N_ROWS, world, e2e_ms), "unit": "rows/s", "h2d_bytes_per_step": N_ROWS * DIM * 4,
                "d2h_bytes_per_step": N_ROWS * 8},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "peak_note": f"bf16 burst {peaks['source']} (kernel timed in a "
                                                           f"loop of {r['ms_total'] / 1e3:.2f} s)",
                     "kernel": "k_assign_tc (fast contraction; with one column split its row-loader warps also certify the rows)",
                     "algorithmic_flops_per_launch": flops_per_launch,
                     "executed_flops_per_launch": flops_per_launch * {"bf16": 3, "bf16x1": 1, "fp8": 1, "fp32": 1}[head],
                     "traffic": None if tpr is None else tpr * N_ROWS},
        "per_precision": {p: {"rows_per_s": N_ROWS * world / (results[p]["ms_per_step"] / 1e3),
                              "ms_per_step": results[p]["ms_per_step"], "steps": results[p]["steps"],
                              "fast_kernel_ms": results[p]["fast_ms_per_launch"],
                              "refined_rows_per_step": results[p]["refined_per_step"],
                              "certified_fraction": 1.0 - results[p]["refined_per_step"] / N_ROWS,
                              "exhaustive_rows_per_step": results[p]["researched_per_step"]} for p in results},
        "gpu_launches": r["launches"],
        "clocks": sampler.summary(),
    }
    if "fp32" in results and head != "fp32":
        line["speedup_vs_fp32_path"] = results["fp32"]["ms_per_step"] / r["ms_per_step"]
    # Rooflines of the other precisions' fast kernels, against peaks measured here.
    for p in results:
        tf = flops_per_launch / (results[p]["fast_ms_per_launch"] / 1e3) / 1e12
        entry = line["per_precision"][p]
        entry["fast_kernel_tflops"] = tf
        if p == "fp32":
            simt, simt2 = emb.measure_simt_peak(local)
            entry["roofline"] = {"bound": "fp32 simt", "achieved": tf, "peak": max(simt, simt2), "unit": "TFLOP/s",
                                 "frac": tf / max(simt, simt2),
                                 "peak_note": f"measured here: FFMA chains {simt:.1f}, paired FFMA2 {simt2:.1f} TFLOP/s "
                                              "(emb200_measure_simt_peak)"}
        elif p == "fp8":
            pk = fp8_gemm_peak_tflops()
            entry["roofline"] = {"bound": "tensor (fp8)", "achieved": tf, "peak": pk, "unit": "TFLOP/s",
                                 "frac": tf / pk,
                                 "peak_note": "measured here: cuBLASLt e4m3 GEMM 8192^3 (torch._scaled_mm)"}
        elif p == "bf16":
            entry["roofline"] = {"bound": "tensor (bf16)", "achieved": tf * 3, "peak": peaks["bf16_tflops"],
                                 "unit": "TFLOP/s", "frac": tf * 3 / peaks["bf16_tflops"],
                                 "peak_note": f"three BF16 terms executed per product; bf16 burst {peaks['source']}"}
    hl, hd = outputs[head]
    line["parity"] = {"all_precisions_identical": bool(all(
        np.array_equal(outputs[p][0], hl) and np.array_equal(outputs[p][1].view(np.uint32), hd.view(np.uint32))
        for p in outputs)), "precisions": list(outputs)}
    if rank == 0 and world == 1 and not args.no_cpu:
        info, kern, rl, rd = cpu_baseline(x, cent)
        line["cpu_baseline"] = info
        if kern != "avx512":  # the engine reproduces the AVX-512 rounding: check against its emulation
            from oracle import oracle as orc

            rl, rd = orc.cpu_assign(x[:32768], cent, kernel="avx512", emulate=True)
        line["parity"].update(parity_check(x, cent, hl, hd, ref=(rl, rd)))
    else:
        line["parity"]["reference"] = "not checked in this run (--no-cpu or N > 1)"
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_c1(args):
    """Plain e-means, the CPU-runnable configuration: 200,000 x 96 f32 rows from a
    4096-blob mixture (centres N(0, 4^2 I), std 1, seed 0), k = 1024, 5 epochs,
    Config::default(); final MSE from an exact assign() pass. The device trains
    with the BF16 search (bit-exact labels), the oracle's train_cpu is timed on the
    host cores and compared centroid for centroid."""
    import torch
    from __graft_entry__ import load_package
    from oracle import oracle as orc

    emb = load_package()
    x = emb.datasets.blobs(200_000, 96, seed=0)
    times = []
    for i in range(args.warmup + args.steps):
        a = emb.B200Assigner(0, precision="bf16")
        t0 = time.perf_counter()
        out = emb.train(x, 96, 1024, emb.Config(), assigner=a)
        lab, dist = a.assign_resident()
        t1 = time.perf_counter()
        a.close()
        if i >= args.warmup:
            times.append(t1 - t0)
    t = float(np.median(times))
    rows = sum(out.recipe.epoch_rows) + len(x)
    # The update kernels' roofline: one run with eager launches, each batch's
    # update chain (label histogram to revival) timed by CUDA events.
    e = emb.B200Assigner(0, precision="bf16", train_eager=True)
    emb.train(x, 96, 1024, emb.Config(), assigner=e)
    ust = e.stats()
    e.close()
    hbm = measured_peaks()
    upd_gbs = ust["update_bytes"] / (ust["update_ms"] / 1e3) / 1e9
    line_update = {"bound": "hbm", "achieved": upd_gbs, "peak": hbm["hbm_gbs"], "unit": "GB/s",
                   "frac": upd_gbs / hbm["hbm_gbs"], "peak_note": f"hbm {hbm['source']}",
                   "kernels": "k_label_hist, k_exclusive_scan, k_label_scatter, k_segment_sums, k_store_labels, "
                              "k_batch_objective, k_apply, k_revive, k_step_incr (per batch)",
                   "algorithmic_bytes": ust["update_bytes"], "device_ms": ust["update_ms"],
                   "training_device_ms_eager": ust["ms_total"],
                   "note": "latency-bound: one warp sums a cluster's rows in row order (the reference's f32 order)"}
    line = {"metric": "e-means train + exact assign, 200k x 96, k=1024, 5 epochs (rows/s)", "value": rows / t,
            "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "dtype": "bf16x3->f32 search, f32 update",
            "config": {"workload": "blobs 200,000 x 96, 4096 blobs, k=1024, Config::default()",
                       "recipe": {"batch": out.recipe.batch_size, "alpha0": out.recipe.alpha0,
                                  "steps": out.recipe.total_steps}},
            "final_mse": float(dist.astype(np.float64).mean()), "n_splits": out.n_splits,
            "update_roofline": line_update,
            "note": "wall clock of the whole host call (upload, training, exact pass, copies)"}
    if not args.no_cpu:
        t0 = time.perf_counter()
        ref = orc.train(x, 1024, orc.make_config(), kernel="avx512" if orc.has_kernel("avx512") else "portable",
                        emulate=not orc.has_kernel("avx512"))
        rl, rd = orc.cpu_assign(x, ref["centroids"], emulate=not orc.has_kernel("avx512"))
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": rows / tc, "unit": "rows/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"the whole workload: train + assign in {tc:.2f} s"}
        line["parity"] = {"centroids_bit_exact": bool(np.array_equal(ref["centroids"].view(np.uint32),
                                                                      out.centroids.view(np.uint32))),
                          "labels_equal": bool(np.array_equal(rl, lab)),
                          "final_mse_reference": float(rd.astype(np.float64).mean())}
    print(json.dumps(line), flush=True)


def fp8_gemm_peak_tflops(reps=20):
    """Dense FP8 (e4m3 x e4m3 -> f32, bf16 out) tensor throughput measured on this
    GPU: cuBLASLt's scaled GEMM (torch._scaled_mm) on 8192^3, CUDA events over
    `reps` launches after warm-up. The denominator of the FP8 search's roofline."""
    import torch

    n = 8192
    a = torch.randn(n, n, device="cuda").to(torch.float8_e4m3fn)
    b = torch.randn(n, n, device="cuda").to(torch.float8_e4m3fn).t()
    one = torch.ones((), device="cuda")
    for _ in range(3):
        torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (ms / 1e3) / 1e12


def int8_gemm_peak_tops(reps=20):
    """Dense int8 tensor throughput measured on this GPU: cuBLASLt's s8 x s8 -> s32
    GEMM (torch._int_mm) on 8192^3, CUDA events over `reps` launches after warm-up.
    The denominator of the int8 roofline, as the cuBLAS BF16 GEMM is for BF16."""
    import torch

    n = 8192
    a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-128, 128, (n, n), dtype=torch.int8, device="cuda").t().contiguous().t()
    for _ in range(3):
        torch._int_mm(a, b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        torch._int_mm(a, b)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (ms / 1e3) / 1e12


def run_c3(args):
    """int8 codes: 2,000,000 x 512 unit-norm f32 rows made resident, then
    quantised on the device (Int8Quantizer fit + encode, faiss calibration); k =
    4096 centroids trained by the engine (int8-centroid search, 2 epochs, untimed);
    one exact assign() pass with CpuI8Assigner(I8) semantics on the tcgen05
    kind::i8 kernel, rows resident."""
    from __graft_entry__ import load_package
    from oracle import oracle as orc

    emb = load_package()
    n = args.rows if args.rows != 1_000_000 else 2_000_000  # --rows: fewer rows for profiling captures
    x = emb.datasets.embeddings(n, 512, latent=64, seed=0)
    a = emb.B200Assigner(0, precision="fp32", centroid_bits=8)
    # f32 rows resident, then Int8Quantizer::fit and encode on the device (faiss calibration)
    a.load_rows(x)
    t0 = time.perf_counter()
    q = emb.Int8Quantizer.fit_resident(a, emb.Calibration.faiss())
    t1 = time.perf_counter()
    st_fit = a.stats()
    clipped = q.quantize_resident(a)
    t2 = time.perf_counter()
    st_enc = a.stats()
    enc_ms = st_enc["ms_total"]
    quant = {"fit_ms": st_fit["ms_total"], "fit_peak_ms": st_fit["fast_ms"], "encode_ms": enc_ms,
             "fit_wall_ms": (t1 - t0) * 1e3, "encode_wall_ms": (t2 - t1) * 1e3,
             "scale": float(q.scale), "clipped_fraction": clipped / x.size,
             "encode_gbs": x.size * 5 / (enc_ms / 1e3) / 1e9,
             "encode_frac_of_measured_hbm": x.size * 5 / (enc_ms / 1e3) / 1e9 / measured_peaks()["hbm_gbs"],
             "note": "CUDA-event times of the kernels on resident f32 rows: fit = f64 column sums in row order "
                     "(a chain of n dependent adds per dimension) + max |x - shift| (fit_peak_ms); encode = one "
                     "pass reading f32 and writing i8 (5 B per value). Wall times include allocation of the "
                     "codes and release of the f32 rows"}
    out = a.train_resident(4096, emb.Config(nepochs=2.0))
    peak_i8 = int8_gemm_peak_tops()
    for _ in range(args.warmup):
        a.assign_resident(want_host=False)
    ms, fast = [], 0.0
    for _ in range(args.steps):
        a.assign_resident(want_host=False)
        st = a.stats()
        ms.append(st["ms_total"])
        fast += st["fast_ms"]
    t = float(np.mean(ms))
    lab_dev, dist_dev = a.assign_resident()  # untimed: the results checked below
    ops = 2.0 * 512 * 4096 * n
    line = {"metric": "rows/s assigned (2M x 512 int8, k=4096, CpuI8Assigner(I8) semantics)",
            "value": n / (t / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t, "higher_is_better": True, "dtype": "s8 x s8 -> s32 (exact)",
            "config": {"workload": f"{n} x 512 int8 codes (faiss calibration of 64-d-latent unit rows), k=4096",
                       "fast_kernel": st["fast_kernel"]},
            "roofline": {"bound": "tensor (int8)", "achieved": ops / (fast / args.steps / 1e3) / 1e12,
                         "peak": peak_i8, "unit": "TOPS", "frac": ops / (fast / args.steps / 1e3) / 1e12 / peak_i8,
                         "kernel": "k_assign_tc_i8 (kind::i8, exact integer keys)",
                         "peak_note": "measured here: cuBLASLt s8 GEMM 8192^3 (torch._int_mm), CUDA events; "
                                      "nominal dense int8 4500 TOPS"},
            "quantizer": quant}
    if not args.no_cpu:
        sample = min(8192, n)
        cores = os.cpu_count() or 1
        codes = q.encode(x[:sample], assigner=a)
        qs = min(262_144, n)
        t0 = time.perf_counter()
        orc.quantizer_encode(x[:qs], *orc.quantizer_fit(x[:qs]))
        quant["cpu_fit_encode_ms_per_1M_rows"] = (time.perf_counter() - t0) * 1e3 * 1e6 / qs
        quant["cpu_sample"] = f"Int8Quantizer fit + encode restated in C++ (one thread) on the first {qs} rows"
        t0 = time.perf_counter()
        rl, rd = orc.i8_assign(codes, out.centroids, bits=8, nthreads=cores)
        tc = time.perf_counter() - t0
        line["parity"] = {"reference_rows_checked": sample, "labels_equal": bool(np.array_equal(lab_dev[:sample], rl)),
                          "dist_bit_exact": bool(np.array_equal(dist_dev[:sample].view(np.uint32), rd.view(np.uint32))),
                          "reference": "CpuI8Assigner(I8) restated (oracle), on the device-encoded codes of the "
                                       "same rows"}
        line["cpu_baseline"] = {"value": sample / tc, "unit": "rows/s", "cores": cores, "kind": "port",
                                "sample": f"first {sample} rows: CpuI8Assigner(I8) restated in C++ (portable "
                                          f"integer kernel), OpenMP {cores} threads, {tc:.2f} s"}
    a.close()
    print(json.dumps(line), flush=True)


def run_report(args):
    """report() (src/report.rs:121-241) on the 1M x 128 embedding rows with k =
    16384 engine-trained centroids, after one exact resident assign: per-cluster
    statistics, medians, nearest other centroid (an exact k^2 d pair pass),
    families and per-row z-scores. value: rows/s of the device report over the
    resident results; e2e: the host-array call (labels, distances and centroids
    uploaded, every output read back); cpu_baseline: the oracle's restatement on
    the same inputs, checked equal to the device report."""
    from __graft_entry__ import load_package
    from oracle import oracle as orc

    emb, x = make_rows(0)
    n, d = x.shape
    cent = trained_centroids(emb, x, 0)
    a = emb.B200Assigner(0, precision="bf16x1")
    a.load_rows(x)
    a.set_centroids(cent)
    labels, sq = a.assign_resident()
    for _ in range(args.warmup):
        emb.report_resident(a)
    ms = []
    clock = ClockSampler(0)
    with clock:
        for _ in range(args.steps):
            r = emb.report_resident(a)
            ms.append(a.stats()["ms_total"])
    t = float(np.mean(ms))
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        emb.report(labels, sq, cent, d, assigner=a)
        e2e.append(time.perf_counter() - t0)
    te = float(np.mean(e2e))
    live = int(np.count_nonzero(r.clusters["size"]))
    pairs = 2.0 * K * K * d  # two exact pair passes (nearest, family radius), each k^2 d
    line = {"metric": "rows/s reported (report() over 1M x 128 rows, k=16384)", "value": n / (t / 1e3),
            "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 / f64 (reference rounding)",
            "data": "synthetic", "gpu_launches": int(a.stats()["kernel_launches"]),
            "config": {"workload": f"report of {n} x {d} embedding rows, k={K} trained centroids",
                       "live_clusters": live, "families": len(r.families)},
            "clocks": clock.summary(),
            "pair_pass": {"element_ops": pairs, "note": "k^2 d (c_i - c_j)^2 terms per pass as the reference "
                                                        "computes them; the device computes each unordered pair once "
                                                        "(the rounding is symmetric), SIMT f32 in the reference's "
                                                        "sqdist rounding (no tensor cores: the order of roundings is "
                                                        "the result)"},
            "e2e": {"value": n / te, "unit": "rows/s", "h2d_bytes_per_step": n * 8 + K * d * 4,
                    "d2h_bytes_per_step": n * 8 + K * 48 + live * 4}}
    if not args.no_cpu:
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        o = orc.report(labels, sq, cent)
        tc = time.perf_counter() - t0
        same = (all(np.array_equal(np.nan_to_num(r.clusters[f]), np.nan_to_num(o["clusters"][f]))
                    for f in r.clusters.dtype.names)
                and np.array_equal(r.local_z, o["local_z"]) and np.array_equal(r.global_z, o["global_z"])
                and len(r.families) == len(o["families"])
                and all(f.leader == g[0] and np.array_equal(f.members, g[1]) for f, g in zip(r.families, o["families"])))
        line["cpu_baseline"] = {"value": n / tc, "unit": "rows/s", "cores": cores, "kind": "port",
                                "sample": f"the whole workload: report() restated in C++ (nearest-centroid pass "
                                          f"OpenMP {cores} threads, the rest one thread), {tc:.2f} s",
                                "identical_to_device": bool(same)}
    a.close()
    print(json.dumps(line), flush=True)


def run_c4(args):
    """Batched uneven instances (configuration 4): (a) PQ training, 4,000,000 x 128
    Gaussian-mixture rows split into 16 sub-spaces of d=8, k=256 each; (b) 48 IVF
    lists, d=64, log-normal sizes (median 20,000, clipped to [2,000, 200,000]),
    k = max(16, n/256). 5 epochs each. All instances of a case train at once
    (emb200_train_batched: one stream and one graph-replayed epoch loop per
    instance); the same instances trained one after the other with per-kernel
    launches are timed beside it."""
    from __graft_entry__ import load_package
    from oracle import oracle as orc

    emb = load_package()
    case = args.workload[-1]
    if case == "a":
        x = emb.datasets.pq_subspaces(4_000_000, 128, 16, seed=0)
        n = 4_000_000
        inst = [(s * n, n, 256) for s in range(16)]
        label = "PQ: 4,000,000 x 128 Gaussian mixture, 16 sub-spaces of d=8, k=256 each"
    else:
        x, sizes, ks = emb.datasets.ivf_lists(48, 64, seed=0)
        starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
        inst = [(int(a), int(b), int(c)) for a, b, c in zip(starts, sizes, ks)]
        label = f"IVF: 48 lists of d=64, {int(sizes.sum())} rows, sizes {int(sizes.min())}..{int(sizes.max())}"
    cfg = emb.Config()
    d = x.shape[1]
    epoch_rows = sum(sum(emb.resolve_recipe(nn, d, kk, cfg).epoch_rows) for (_, nn, kk) in inst)

    def timed_runs(streams):
        a = emb.B200Assigner(0, precision="fp32", batched_streams=streams)
        a.load_rows(x)
        times, dev = [], []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            outs = a.train_batched(inst, cfg, max_concurrency=16)
            t1 = time.perf_counter()
            if i >= args.warmup:
                times.append(t1 - t0)
                dev.append(a.stats()["ms_total"])
        choice = None if streams else a.batched_search_choice()
        a.close()
        return outs, float(np.median(times)), float(np.median(dev)), choice

    outs, t, t_dev, choice = timed_runs(False)
    if args.c4_lockstep_only:  # profiling: the lockstep calls alone
        print(json.dumps({"workload": args.workload, "lockstep_ms": t * 1e3, "device_ms": t_dev,
                          "rows_per_s": epoch_rows / t, "autotuned_search_tile": choice}), flush=True)
        return
    outs_s, t_streams, _, _ = timed_runs(True)
    # Sequential, per-kernel launches, one instance after the other.
    b = emb.B200Assigner(0, precision="fp32", train_eager=True, batched_streams=True)
    b.load_rows(x)
    t0 = time.perf_counter()
    seq = b.train_batched(inst, cfg, max_concurrency=1)
    t_seq = time.perf_counter() - t0
    b.close()
    same = all(np.array_equal(o.centroids.view(np.uint32), q.centroids.view(np.uint32)) for o, q in zip(outs, seq))
    same_s = all(np.array_equal(o.centroids.view(np.uint32), q.centroids.view(np.uint32)) for o, q in zip(outs, outs_s))
    line = {"metric": f"batched e-means training, rows/s over all instances ({label}, 5 epochs)",
            "value": epoch_rows / t, "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "dtype": "f32",
            "config": {"workload": label, "instances": len(inst), "epoch_rows_total": epoch_rows,
                       "recipe_first": vars(emb.resolve_recipe(inst[0][1], d, inst[0][2], cfg)),
                       "mode": "lockstep: one global step of batched kernels over all instances, captured as a "
                               "CUDA graph and replayed; persistent search over an (instance, row tile) queue",
                       "autotuned_search_tile": {"rows": choice[0], "centroids": choice[1],
                                                 "item_covers_one_centroid_tile": choice[2]}},
            "device_ms": t_dev, "streams_mode_ms": t_streams * 1e3, "speedup_vs_streams_mode": t_streams / t,
            "streams_mode_rows_per_s": epoch_rows / t_streams,
            "sequential_eager_ms": t_seq * 1e3, "speedup_vs_sequential_eager": t_seq / t,
            "batched_equals_sequential": bool(same), "lockstep_equals_streams": bool(same_s),
            "note": "wall clock of the whole host call (recipes, row orders drawn on the host, uploads, training, "
                    "copies back), rows resident; device_ms: CUDA events around the call's device work"}
    if not args.no_cpu:
        r0, nn, kk = inst[0]
        t0 = time.perf_counter()
        orc.train(x[r0:r0 + nn], kk, orc.make_config(), kernel="avx512" if orc.has_kernel("avx512") else "portable",
                  emulate=not orc.has_kernel("avx512"))
        tc = time.perf_counter() - t0
        rows0 = sum(emb.resolve_recipe(nn, d, kk, cfg).epoch_rows)
        line["cpu_baseline"] = {"value": rows0 / tc, "unit": "rows/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"instance 0 of {len(inst)} ({nn} rows, k={kk}) trained by the oracle's "
                                          f"train_cpu restatement in {tc:.2f} s"}
    print(json.dumps(line), flush=True)


def run_c5(args):
    """Learned proposer at large k: 10,000,000 x 96 heavy-tailed rows (Student-t
    nu=3 latents in 32 dims through a random 32 x 96 map, 8192-component mixture),
    k = 65536 centroids trained by the engine (5 epochs, BF16 search, untimed).
    The proposer groups the centroids into 256 groups (e-means on the centroids),
    its network 96 -> 512 -> 512 -> 256 is trained on the training run's labels,
    and the final assign scores each row against its top 8 groups only. Timed
    beside it: the full exact search (tcgen05 BF16 and the plain FP32 path) and
    the same grouped search driven by the nearest group centroids."""
    from __graft_entry__ import load_package
    from oracle import oracle as orc

    emb = load_package()
    n = args.c5_rows
    d, k, groups, top_c = 96, 65536, 256, 8
    t0 = time.perf_counter()
    x = emb.datasets.heavy_tailed(n, d, latent=32, components=8192, nu=3.0, seed=0)
    t_data = time.perf_counter() - t0
    a = emb.B200Assigner(0, precision="bf16x1")
    a.load_rows(x)
    # An untimed short run first: the process's one-time costs (kernel loading)
    # do not fall on the timed full-search training, which the proposer-in-
    # training run is compared with.
    a.train_resident(k, emb.Config(nepochs=0.2))
    t0 = time.perf_counter()
    out = a.train_resident(k, emb.Config(nepochs=5.0))
    t_train = time.perf_counter() - t0
    t0 = time.perf_counter()
    a.proposer_init(groups=groups, hidden=512, top=8, seed=7)
    t_group = time.perf_counter() - t0
    t0 = time.perf_counter()
    losses = a.proposer_train(out.labels, args.proposer_steps)
    t_fit = time.perf_counter() - t0

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        ms, st = [], None
        for _ in range(args.steps):
            fn()
            st = a.stats()
            ms.append(st["ms_total"])
        return float(np.mean(ms)), st

    if args.profile_proposer:
        # Profiling captures: one proposer assign (first setting) between
        # cudaProfilerStart/Stop, for ncu --profile-from-start off.
        import torch

        top, conf, mass = (float(v) for v in args.proposer_configs.split(",")[0].split(":"))
        a.proposer_set("mlp", int(top), conf, mass)
        a.assign_proposed(want_host=False)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        a.assign_proposed(want_host=False)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profiled": "one proposer assign", "rows": n, "stats": a.stats()}), flush=True)
        a.close()
        return

    configs = [tuple(float(v) for v in c.split(":")) for c in args.proposer_configs.split(",")]
    sampler = ClockSampler(0)
    runs = []
    with sampler:
        a.set_options(precision="bf16")
        a.set_centroids(out.centroids)
        t_full3, st_full3 = timed(lambda: a.assign_resident(want_host=False))
        a.set_options(precision="bf16x1")
        a.set_centroids(out.centroids)
        t_full, st_full = timed(lambda: a.assign_resident(want_host=False))
        for (top, conf, mass) in configs:
            a.proposer_set("mlp", int(top), conf, mass)
            t, st = timed(lambda: a.assign_proposed(want_host=False))
            lab, dist = a.assign_proposed()
            runs.append(((int(top), conf, mass), t, st, lab, dist))
        a.proposer_set("centroids", top_c, 0.0)
        t_cen, st_cen = timed(lambda: a.assign_proposed(want_host=False))
    lab_f, dist_f = a.assign_resident()
    lab_c, dist_c = a.assign_proposed()
    mse_f = float(dist_f.astype(np.float64).mean())
    # Training with the proposer searching the last epoch's batches, against the
    # full-search training above: rows/s, and the exact assign's MSE with each.
    late = None
    if args.proposer_training:
        p = emb.B200Assigner(0, precision="bf16x1")
        p.load_rows(x)
        # Untimed first, as for the full-search run: the handle's allocations and
        # the first captures of its kernels stay out of the timed training.
        p.train_resident_proposed(k, emb.Config(nepochs=2.0), late_epochs=1, net_steps=args.late_net_steps,
                                  groups=groups, top=32, mass=0.999)
        t0 = time.perf_counter()
        outp = p.train_resident_proposed(k, emb.Config(nepochs=5.0), late_epochs=args.late_epochs,
                                         net_steps=args.late_net_steps, groups=groups, top=32, mass=0.999)
        t_late = time.perf_counter() - t0
        stp = outp.stats
        p.set_centroids(outp.centroids)
        _, dist_p = p.assign_resident()
        p.close()
        rows_trained = sum(out.recipe.epoch_rows)
        late = {"train_rows_per_s": rows_trained / t_late, "train_s": t_late,
                "full_search_train_rows_per_s": rows_trained / t_train, "full_search_train_s": t_train,
                "speedup": t_train / t_late, "late_epochs": args.late_epochs, "net_steps": args.late_net_steps,
                "final_mse_delta": float(dist_p.astype(np.float64).mean()) / mse_f - 1.0,
                "last_pass_label_agreement": float(np.mean(outp.labels == out.labels)),
                "late_epoch_device_ms": stp["late_epochs_ms"], "proposer_fit_ms": stp["late_fit_ms"],
                "full_search_epoch_ms_estimate": t_train * 1e3 / len(out.recipe.epoch_rows),
                "rows_proposed_in_late_epoch": int(stp["rows_proposed"]),
                "rows_lowconf_in_late_epoch": int(stp["rows_lowconf"]),
                "note": "wall clock of each whole train call (the proposed one includes grouping the centroids "
                        "and fitting the network on the previous epoch's labels); MSE from an exact assign of "
                        "all rows to each run's final centroids"}
    # FP64 brute force on a sample of rows: agreement of each path's labels
    sample = np.random.default_rng(3).choice(n, 32768, replace=False)
    bl, _ = orc.bruteforce_f64(x[sample], out.centroids)
    a.close()
    # the plain FP32 path on the first rows (its pass over all rows would take minutes)
    m32 = min(n, 1_000_000)
    b = emb.B200Assigner(0, precision="fp32")
    b.set_centroids(out.centroids)
    b.load_rows(x[:m32])
    b.assign_resident(want_host=False)
    b.assign_resident(want_host=False)
    t_fp32 = b.stats()["ms_total"] * n / m32
    b.close()
    flops_row = 2.0 * (96 * 512 + 512 * 512 + 512 * 256)
    peaks = measured_peaks()

    def entry(t, st, lab, dist):
        return {"rows_per_s": n / (t / 1e3), "ms_per_step": t, "recall_at_1": float(np.mean(lab == lab_f)),
                "mse_delta": float(dist.astype(np.float64).mean()) / mse_f - 1.0,
                "agreement_fp64_sample": float(np.mean(lab[sample] == bl)),
                "propose_ms": st["propose_ms"], "grouped_search_ms": st["fast_ms"],
                "rows_lowconf": st["rows_lowconf"], "rows_refined": st["rows_refined"],
                "rows_researched": st["rows_researched"], "kernel_launches": st["kernel_launches"]}

    (top, conf, mass), t_mlp, st_mlp, lab_m, dist_m = runs[0]
    line = {"metric": "rows/s assigned (10M x 96 heavy-tailed, k=65536): learned proposer vs full search",
            "value": n / (t_mlp / 1e3), "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_mlp, "higher_is_better": True, "dtype": "bf16 -> f32 accumulate",
            "config": {"workload": f"{n} x {d} heavy-tailed rows (Student-t nu=3, 8192 components), k={k}, "
                                   f"{groups} groups, network 96-512-512-256",
                       "top": top, "confidence": conf, "mass": mass, "proposer_steps": args.proposer_steps,
                       "l2": "no flush: the resident rows (3.8 GB) exceed the 126 MB L2"},
            "learned": entry(t_mlp, st_mlp, lab_m, dist_m),
            "learned_settings": [dict(entry(t, st, lab, dist), top=c[0], confidence=c[1], mass=c[2],
                                      groups_per_row=st["groups_searched"] / max(st["rows_proposed"], 1))
                                 for (c, t, st, lab, dist) in runs],
            "group_centroids": dict(entry(t_cen, st_cen, lab_c, dist_c), top=top_c),
            "full_search_bf16x1": {"rows_per_s": n / (t_full / 1e3), "ms_per_step": t_full,
                                   "agreement_fp64_sample": float(np.mean(lab_f[sample] == bl)),
                                   "fast_kernel_ms": st_full["fast_ms"], "rows_refined": st_full["rows_refined"]},
            "full_search_bf16x3": {"rows_per_s": n / (t_full3 / 1e3), "ms_per_step": t_full3,
                                   "fast_kernel_ms": st_full3["fast_ms"], "rows_refined": st_full3["rows_refined"]},
            "full_search_fp32": {"rows_per_s": n / (t_fp32 / 1e3), "ms_per_step": t_fp32,
                                 "note": f"timed on the first {m32} rows, scaled"},
            "speedup_vs_full_search": min(t_full, t_full3) / t_mlp, "speedup_vs_fp32_path": t_fp32 / t_mlp,
            "network_roofline": {"bound": "tensor", "achieved": flops_row * n / (st_mlp["propose_ms"] / 1e3) / 1e12,
                                 "peak": peaks["bf16_tflops_sustained"], "unit": "TFLOP/s",
                                 "kernel": "k_mlp_tc: fused tcgen05 forward pass (standardised input, three "
                                           "layers, top-m group selection in the epilogue)"},
            "times_s": {"data": t_data, "train": t_train, "grouping": t_group, "network_fit": t_fit},
            "proposer_in_training": late,
            "fit_loss_first_last": [float(losses[:20].mean()), float(losses[-20:].mean())],
            "gpu_launches": st_mlp["kernel_launches"], "clocks": sampler.summary()}
    line["network_roofline"]["frac"] = line["network_roofline"]["achieved"] / line["network_roofline"]["peak"]
    if not args.no_cpu:
        cores = os.cpu_count() or 1
        rows = 8192
        kern = "avx512" if orc.has_kernel("avx512") else "portable"
        t0 = time.perf_counter()
        orc.cpu_assign(x[:rows], out.centroids, kernel=kern, nthreads=cores)
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": rows / tc, "unit": "rows/s", "cores": cores, "kind": "port",
                                "sample": f"first {rows} rows, k={k}: CpuAssigner ({kern}) restated in C++, "
                                          f"OpenMP {cores} threads, {tc:.2f} s"}
    print(json.dumps(line), flush=True)


def run_reference(args):
    """The reference arm: the reference's CpuAssigner (restated in C++ in oracle/,
    the reference itself cannot be built here) on the host cores, over the same
    rows and the same centroids as the repo arm. The centroids come from the
    oracle's train() (2 epochs), which gives the same bits as the engine's; each
    timed step is one bounded slice of the 1M-row pass."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc

    _, x = make_rows(seed=0)
    kern = "avx512" if orc.has_kernel("avx512") else ("avx2" if orc.has_kernel("avx2") else "portable")
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    if args.centroids == "trained":
        # AVX-512 rounding, the engine's default: native when the host has it.
        cent = orc.train(x, K, orc.make_config(nepochs=2.0), kernel="avx512", emulate=kern != "avx512",
                         nthreads=cores)["centroids"]
    else:
        cent = x[np.random.default_rng(1).choice(len(x), K, replace=False)] * np.float32(0.97)
    t_train = time.perf_counter() - t0
    sample = min(32768, N_ROWS // 2)  # rows per step: each step a bounded slice of the pass
    for _ in range(min(args.warmup, 1)):
        orc.cpu_assign(x[:1024], cent, kernel=kern, nthreads=cores)
    ts = []
    for s in range(args.steps):
        r0 = (s * sample) % (N_ROWS - sample)
        t0 = time.perf_counter()
        orc.cpu_assign(x[r0:r0 + sample], cent, kernel=kern, nthreads=cores)
        ts.append(time.perf_counter() - t0)
    rps = sample * len(ts) / sum(ts)
    line = {"metric": METRIC, "value": rps, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(ts)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "rows_per_gpu": N_ROWS, "rows_per_step": sample, "d": DIM, "k": K,
                       "centroids": centroid_note(args.centroids), "centroid_digest": centroid_digest(cent)},
            "cpu_baseline": {"value": rps, "unit": "rows/s", "cores": cores, "kind": "port",
                             "sample": f"{sample} rows per step x {args.steps} steps of the 1M-row pass (a step is "
                                       f"one slice, its time is ms_per_step); the reference CpuAssigner ({kern} "
                                       f"kernel) restated in C++, OpenMP, {cores} threads; the centroids' "
                                       f"training by the oracle's train() took {t_train:.1f} s, untimed"},
            "e2e": {"value": rps, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precisions", default="bf16x1,bf16,fp8,fp32", help="comma list; the first is the headline")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--rows", type=int, default=N_ROWS, help="rows per pass (profiling captures use fewer)")
    ap.add_argument("--centroids", default="trained", choices=["trained", "sampled"],
                    help="trained by the engine (default) or a fixed sample of rows (profiling captures)")
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c3", "c4a", "c4b", "c5", "report"],
                    help="c2: the headline assign benchmark; the others: the remaining configurations")
    ap.add_argument("--proposer-steps", type=int, default=8000, help="c5: Adam steps of the network")
    ap.add_argument("--proposer-configs", default="32:0.99:0.9995,32:0:0.999,32:0.999:0.9995,8:0:0",
                    help="c5: top:confidence:mass settings of the proposer assign; the first is the headline")
    ap.add_argument("--c5-rows", type=int, default=10_000_000, help="c5: rows of the workload")
    ap.add_argument("--c4-lockstep-only", action="store_true",
                    help="C4: time the lockstep calls only (no streams-mode or sequential comparison)")
    ap.add_argument("--late-epochs", type=int, default=1,
                    help="C5: last epochs of the proposer-in-training run searched through the proposer")
    ap.add_argument("--late-net-steps", type=int, default=500,
                    help="c5: Adam steps of the network fitted inside the proposed training run")
    ap.add_argument("--proposer-training", type=int, default=1,
                    help="c5: also train with the proposer in the last epoch (1) or not (0)")
    ap.add_argument("--profile-proposer", action="store_true",
                    help="c5: run one proposer assign between cudaProfilerStart/Stop and exit (profiling captures)")
    args = ap.parse_args()
    set_rows(args.rows)
    if args.workload == "c1" and args.impl == "ours":
        return run_c1(args)
    if args.workload == "c3" and args.impl == "ours":
        return run_c3(args)
    if args.workload in ("c4a", "c4b") and args.impl == "ours":
        return run_c4(args)
    if args.workload == "c5" and args.impl == "ours":
        return run_c5(args)
    if args.workload == "report" and args.impl == "ours":
        return run_report(args)
    args.precisions = args.precisions.split(",")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
