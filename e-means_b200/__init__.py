"""B200-native e-means engine: host-side mirror of the crate `emeans` API.

The reference crate (andrewluetgers/e-means) exposes `Config`, `train`,
`assign`, `resolve_recipe` and the `Assigner` / `AssignRows<T>` traits
(src/lib.rs:75-163, 201-225, 348-520). This package offers the same names over
the C ABI of libemb200.so (include/emb200.h), whose CUDA kernels do all of the
work on one B200. There is no CPU fallback: without the built library or a
B200 every call raises.
"""
import ctypes
import enum
import os
import subprocess
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import datasets  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libemb200.so")

EMB200_F32, EMB200_I8, EMB200_U8 = 0, 1, 2
PREC_FP32, PREC_BF16, PREC_BF16X1, PREC_FP8 = 0, 1, 2, 3
CENTROIDS_F32, CENTROIDS_I8, CENTROIDS_I16 = 0, 8, 16
MATCH = {"avx512": 0, "avx2": 1, "portable": 2}
_DTYPES = {np.dtype(np.float32): EMB200_F32, np.dtype(np.int8): EMB200_I8, np.dtype(np.uint8): EMB200_U8}
PRECISIONS = {"fp32": PREC_FP32, "bf16": PREC_BF16, "bf16x1": PREC_BF16X1, "fp8": PREC_FP8}


class EngineError(RuntimeError):
    """A non-zero status from libemb200 (the reference returns Err or panics)."""


class _Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("centroid_bits", ctypes.c_int), ("match_kernel", ctypes.c_int),
                ("train_eager", ctypes.c_int), ("batched_streams", ctypes.c_int), ("reserved", ctypes.c_int * 3)]


class _Config(ctypes.Structure):
    _fields_ = [("nepochs", ctypes.c_double), ("batch_law", ctypes.c_int), ("batch_size", ctypes.c_uint64),
                ("alpha0", ctypes.c_double), ("unused_threshold", ctypes.c_float), ("balance", ctypes.c_float),
                ("seed", ctypes.c_uint64), ("verbose", ctypes.c_int), ("closing_f64", ctypes.c_int)]


class _Recipe(ctypes.Structure):
    _fields_ = [("batch_size", ctypes.c_uint64), ("alpha0", ctypes.c_double), ("n_epochs", ctypes.c_uint64),
                ("total_steps", ctypes.c_uint64), ("unused_threshold", ctypes.c_float)]


class _Stats(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint64), ("rows_certified", ctypes.c_uint64), ("rows_researched", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("ms_total", ctypes.c_double), ("fast_kernel", ctypes.c_int32),
                ("fast_aborted", ctypes.c_int32), ("rows_refined", ctypes.c_uint64), ("fast_ms", ctypes.c_double),
                ("fast_launches", ctypes.c_uint64), ("rows_proposed", ctypes.c_uint64),
                ("rows_lowconf", ctypes.c_uint64), ("propose_ms", ctypes.c_double),
                ("groups_searched", ctypes.c_uint64), ("update_ms", ctypes.c_double),
                ("update_bytes", ctypes.c_uint64), ("late_fit_ms", ctypes.c_double),
                ("late_epochs_ms", ctypes.c_double)]


class _ProposerConfig(ctypes.Structure):
    _fields_ = [("groups", ctypes.c_uint32), ("hidden", ctypes.c_uint32), ("top", ctypes.c_uint32),
                ("mode", ctypes.c_uint32), ("confidence", ctypes.c_float), ("batch", ctypes.c_uint32),
                ("lr", ctypes.c_float), ("group_epochs", ctypes.c_float), ("seed", ctypes.c_uint64),
                ("mass", ctypes.c_float), ("reserved", ctypes.c_uint32 * 3)]


PROPOSER_MODES = {"mlp": 0, "centroids": 1}


class _ReportConfig(ctypes.Structure):
    _fields_ = [("family_radius", ctypes.c_float), ("family_pass", ctypes.c_uint32),
                ("min_local_size", ctypes.c_uint64)]


class _ReportSummary(ctypes.Structure):
    _fields_ = [("median_dist", ctypes.c_float), ("median_rms", ctypes.c_float),
                ("median_nearest_dist", ctypes.c_float), ("n_families", ctypes.c_uint32),
                ("n_live", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


# ClusterStats, src/report.rs:37-56, as emb200_cluster_stats (48 bytes, no padding)
CLUSTER_STATS = np.dtype([("size", "u4"), ("rms", "f4"), ("median", "f4"), ("mad", "f4"), ("p90", "f4"),
                          ("p99", "f4"), ("max", "f4"), ("looseness", "f4"), ("nearest_centroid", "u4"),
                          ("nearest_dist", "f4"), ("isolation", "f4"), ("family", "u4")])


class _Calibration(ctypes.Structure):
    _fields_ = [("target_peak", ctypes.c_float), ("power_of_two", ctypes.c_int32), ("quantile", ctypes.c_double)]


def build(force=False):
    """Compile libemb200.so in-tree with nvcc for sm_100a."""
    args = ["make", "-s", "-C", _HERE] + (["-B"] if force else [])
    subprocess.run(args, check=True)


_lib = None


def lib():
    """Load libemb200.so; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineError(f"{LIB_PATH} is not built: run emeans_b200.build() (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    L.emb200_create.argtypes = [I, ctypes.POINTER(_Opts), ctypes.POINTER(P)]
    L.emb200_destroy.argtypes = [P]
    L.emb200_last_error.restype = ctypes.c_char_p
    L.emb200_last_error.argtypes = [P]
    L.emb200_name.argtypes = [P, ctypes.c_char_p, S]
    L.emb200_set_opts.argtypes = [P, ctypes.POINTER(_Opts)]
    L.emb200_get_stats.argtypes = [P, ctypes.POINTER(_Stats)]
    L.emb200_set_centroids.argtypes = [P, P, S, S]
    L.emb200_set_bias.argtypes = [P, P, S]
    for nm in ("emb200_assign_f32", "emb200_assign_i8", "emb200_assign_u8"):
        getattr(L, nm).argtypes = [P, P, S, P, P]
    L.emb200_assign_device.argtypes = [P, I, P, S, P, P, P]
    L.emb200_load_rows.argtypes = [P, I, P, S, S]
    L.emb200_assign_resident.argtypes = [P, P, P]
    L.emb200_set_abort_test.argtypes = [P, I, ctypes.c_uint64]
    L.emb200_measure_simt_peak.argtypes = [I, P, P]
    L.emb200_measure_mma_peak.argtypes = [I, P, P]
    L.emb200_batched_search_choice.argtypes = [P, P, P, P]
    L.emb200_train_proposed.argtypes = [P, ctypes.POINTER(_Config), S, ctypes.POINTER(_ProposerConfig), ctypes.c_uint32,
                                        ctypes.c_uint32, P, P, P, P, ctypes.POINTER(_Recipe)]
    L.emb200_resolve_recipe.argtypes = [S, S, S, ctypes.POINTER(_Config), ctypes.POINTER(_Recipe), P, S]
    L.emb200_scheduled_alpha.restype = ctypes.c_double
    L.emb200_scheduled_alpha.argtypes = [ctypes.c_double, S, S]
    L.emb200_train.argtypes = [P, ctypes.POINTER(_Config), S, P, P, P, P, ctypes.POINTER(_Recipe)]
    L.emb200_train_batched.argtypes = [P, ctypes.POINTER(_Config), P, S, S, P, P, P, P]
    L.emb200_proposer_init.argtypes = [P, ctypes.POINTER(_ProposerConfig)]
    L.emb200_proposer_train.argtypes = [P, P, S, ctypes.c_uint32, P]
    L.emb200_proposer_set.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float]
    L.emb200_proposer_param_count.restype = S
    L.emb200_proposer_param_count.argtypes = [P]
    L.emb200_proposer_get_params.argtypes = [P, P, S]
    L.emb200_proposer_set_params.argtypes = [P, P, S]
    L.emb200_proposer_grad.argtypes = [P, P, P, S, P, P]
    L.emb200_proposer_groups.argtypes = [P, P]
    L.emb200_proposer_logits.argtypes = [P, P, S, P, I]
    L.emb200_propose.argtypes = [P, P, S, P, P, P]
    L.emb200_assign_proposed_resident.argtypes = [P, P, P]
    L.emb200_assign_proposed_device.argtypes = [P, P, S, P, P, P]
    C = ctypes.POINTER(_Calibration)
    L.emb200_quantizer_fit.argtypes = [P, P, S, S, C, P, P]
    L.emb200_quantizer_fit_device.argtypes = [P, P, S, S, C, P, P]
    L.emb200_quantizer_fit_resident.argtypes = [P, C, P, P]
    L.emb200_quantizer_encode.argtypes = [P, P, S, S, P, ctypes.c_float, P, P]
    L.emb200_quantizer_encode_device.argtypes = [P, P, S, S, P, ctypes.c_float, P, P, P]
    L.emb200_quantize_resident.argtypes = [P, P, ctypes.c_float, P]
    L.emb200_quantizer_decode.argtypes = [P, P, S, S, P, ctypes.c_float, P]
    RC = ctypes.POINTER(_ReportConfig)
    L.emb200_report.argtypes = [P, P, P, S, P, S, S, RC, P, P, P, ctypes.POINTER(_ReportSummary)]
    L.emb200_report_resident.argtypes = [P, RC, P, P, P, ctypes.POINTER(_ReportSummary)]
    L.emb200_report_families.argtypes = [P, P, P, P, P, P]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class BatchLaw(enum.IntEnum):
    """src/lib.rs:93-101."""

    AUTO = 0
    THROUGHPUT = 1
    QUALITY = 2


@dataclass
class Config:
    """src/lib.rs:103-139 (same fields and defaults)."""

    nepochs: float = 5.0
    batch_law: BatchLaw = BatchLaw.AUTO
    batch_size: Optional[int] = None
    alpha0: Optional[float] = None
    unused_threshold: Optional[float] = None
    balance: float = 0.0
    seed: int = 1234
    verbose: bool = False
    closing_f64: bool = False  # FP64 last-pass sums instead of the reference's f32

    def _c(self):
        return _Config(self.nepochs, int(self.batch_law), self.batch_size or 0,
                       self.alpha0 if self.alpha0 is not None else -1.0,
                       self.unused_threshold if self.unused_threshold is not None else -1.0, self.balance, self.seed,
                       int(self.verbose), int(self.closing_f64))


@dataclass
class Recipe:
    """src/lib.rs:141-149."""

    batch_size: int
    alpha0: float
    epoch_rows: List[int]
    total_steps: int
    unused_threshold: float


@dataclass
class Output:
    """src/lib.rs:151-163."""

    centroids: np.ndarray
    labels: np.ndarray
    objective: np.ndarray
    n_splits: int
    recipe: Recipe
    stats: dict = field(default_factory=dict)


def resolve_recipe(n, d, k, cfg: Optional[Config] = None) -> Recipe:
    """resolve_recipe (src/lib.rs:201-225), computed by libemb200's host code."""
    cfg = cfg or Config()
    c = cfg._c()
    r = _Recipe()
    er = np.zeros(int(np.floor(cfg.nepochs)) + 2, np.uint64)
    lib().emb200_resolve_recipe(n, d, k, ctypes.byref(c), ctypes.byref(r), _p(er), er.size)
    return Recipe(int(r.batch_size), float(r.alpha0), [int(v) for v in er[:r.n_epochs]], int(r.total_steps),
                  float(r.unused_threshold))


def scheduled_alpha(alpha0, step, total):
    """src/lib.rs:194-198."""
    return lib().emb200_scheduled_alpha(alpha0, step, total)


def measure_simt_peak(ordinal=0):
    """FP32 SIMT FMA throughput of the GPU in TFLOP/s: (scalar FFMA, paired FFMA2)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = lib().emb200_measure_simt_peak(ordinal, ctypes.byref(a), ctypes.byref(b))
    if rc != 0:
        raise EngineError(f"emb200_measure_simt_peak failed ({rc})")
    return a.value, b.value


def measure_mma_peak(ordinal=0):
    """(cta_group::1 M=128 N=256, cta_group::2 M=256 N=256) tcgen05 BF16 TF/s of
    this device, operands resident in shared memory."""
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = lib().emb200_measure_mma_peak(ordinal, ctypes.byref(a), ctypes.byref(b))
    if rc != 0:
        raise EngineError(f"emb200_measure_mma_peak failed ({rc})")
    return a.value, b.value


def balance_stats(labels, k):
    """balance_stats (src/lib.rs:497-504): (imbalance factor, largest/mean size, empty clusters)."""
    counts = np.bincount(np.asarray(labels, np.int64), minlength=k).astype(np.uint64)
    n = float(len(labels))
    squares = float((counts * counts).astype(np.float64).sum())
    return k * squares / (n * n), float(counts.max()) * k / n, int((counts == 0).sum())


class B200Assigner:
    """Drop-in for the `Assigner` + `AssignRows<T>` traits (src/lib.rs:75-91),
    beside CpuAssigner (src/cpu.rs) and CpuI8Assigner (src/cpu_i8.rs).

    precision: "fp32" (SIMT), "bf16" (tcgen05, three-term split), "bf16x1", "fp8" (tcgen05 e4m3).
    centroid_bits: 0 (CpuAssigner semantics for every row type), 8 or 16
    (CpuI8Assigner(I8) / CpuI8Assigner(I16) semantics for i8 rows). match: which CpuAssigner SIMD
    kernel's rounding the labels and distances reproduce.
    """

    def __init__(self, ordinal=0, precision="fp32", centroid_bits=0, match="avx512", train_eager=False,
                 batched_streams=False):
        self._h = ctypes.c_void_p()
        self._opts = _Opts(PRECISIONS[precision], centroid_bits, MATCH[match], int(train_eager), int(batched_streams))
        rc = lib().emb200_create(ordinal, ctypes.byref(self._opts), ctypes.byref(self._h))
        if rc != 0:
            raise EngineError(f"emb200_create failed ({rc}): no usable B200 (sm_100) device")
        self.k = 0
        self.d = 0

    def _check(self, rc):
        if rc != 0:
            raise EngineError(lib().emb200_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib().emb200_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, precision=None, centroid_bits=None, match=None):
        if precision is not None:
            self._opts.precision = PRECISIONS[precision]
        if centroid_bits is not None:
            self._opts.centroid_bits = centroid_bits
        if match is not None:
            self._opts.match_kernel = MATCH[match]
        self._check(lib().emb200_set_opts(self._h, ctypes.byref(self._opts)))

    def name(self):
        buf = ctypes.create_string_buffer(256)
        self._check(lib().emb200_name(self._h, buf, 256))
        return buf.value.decode()

    def set_centroids(self, centroids, k=None, d=None):
        c = np.ascontiguousarray(centroids, np.float32)
        if k is None:
            k, d = c.shape
        if c.size != k * d:
            raise ValueError("centroids must be k x d")
        self._check(lib().emb200_set_centroids(self._h, _p(c), k, d))
        self.k, self.d = k, d

    def set_bias(self, bias):
        b = np.ascontiguousarray(bias, np.float32)
        self._check(lib().emb200_set_bias(self._h, _p(b), b.size))

    def assign(self, x, labels=None, dist=None):
        """AssignRows::assign: rows (m x d, f32/i8/u8) -> (labels u32, dist f32)."""
        x = np.ascontiguousarray(x)
        if x.dtype not in _DTYPES:
            raise TypeError(f"rows must be float32, int8 or uint8, got {x.dtype}")
        m = x.size // max(self.d, 1)
        labels = np.empty(m, np.uint32) if labels is None else labels
        dist = np.empty(m, np.float32) if dist is None else dist
        fn = {EMB200_F32: lib().emb200_assign_f32, EMB200_I8: lib().emb200_assign_i8,
              EMB200_U8: lib().emb200_assign_u8}[_DTYPES[x.dtype]]
        self._check(fn(self._h, _p(x), m, _p(labels), _p(dist)))
        return labels, dist

    def assign_host_ptr(self, x_ptr, dtype, m, labels_ptr, dist_ptr):
        """Host-memory assign on raw pointers (e.g. pinned torch tensors): the trait
        call with the caller's own buffers."""
        fn = {EMB200_F32: lib().emb200_assign_f32, EMB200_I8: lib().emb200_assign_i8,
              EMB200_U8: lib().emb200_assign_u8}[dtype]
        self._check(fn(self._h, ctypes.c_void_p(x_ptr), m, ctypes.c_void_p(labels_ptr), ctypes.c_void_p(dist_ptr)))

    def assign_device(self, x_ptr, dtype, m, labels_ptr, dist_ptr, stream=None):
        """Device-pointer assign (torch tensors' data_ptr()), enqueued on `stream`."""
        self._check(lib().emb200_assign_device(self._h, dtype, ctypes.c_void_p(x_ptr), m, ctypes.c_void_p(labels_ptr),
                                               ctypes.c_void_p(dist_ptr), ctypes.c_void_p(stream or 0)))

    def load_rows(self, x):
        """Upload rows once; they stay resident in HBM for assign_resident / train."""
        x = np.ascontiguousarray(x)
        n, d = x.shape
        self._check(lib().emb200_load_rows(self._h, _DTYPES[x.dtype], _p(x), n, d))
        self.rows_shape = (n, d)

    def assign_resident(self, want_host=True):
        n = self.rows_shape[0]
        labels = np.empty(n, np.uint32) if want_host else None
        dist = np.empty(n, np.float32) if want_host else None
        self._check(lib().emb200_assign_resident(self._h, _p(labels), _p(dist)))
        return labels, dist

    def set_abort_test(self, stall_tile=-1, stall_ns=0):
        """Test hook of the bounded-wait abort path: the fast tensor-core searches
        stall one epilogue warp at centroid tile `stall_tile` on a barrier nothing
        completes, bounded by `stall_ns`; the call then re-searches its rows
        exactly. stall_tile < 0 turns it off."""
        self._check(lib().emb200_set_abort_test(self._h, int(stall_tile), int(stall_ns)))

    def stats(self):
        s = _Stats()
        self._check(lib().emb200_get_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _Stats._fields_}

    def train_batched(self, instances, cfg: Optional[Config] = None, max_concurrency=0):
        """train() for independent instances over row ranges of the resident rows.

        instances: [(row0, n, k), ...]. Returns one Output per instance (labels in
        the instance's own row order). The instances advance in lockstep, one
        global step at a time through batched kernels (the search a persistent
        kernel over an (instance, row tile) work queue, its tile shape chosen by
        a measured sweep), the step captured once as a CUDA graph; or, with
        batched_streams=True (and for the cases lockstep does not cover), each on
        its own stream with graph-replayed epochs. Either way each instance's
        result equals its own train() call."""
        cfg = cfg or Config()
        n_all, d = self.rows_shape
        inst = np.array([[r0, n, k] for (r0, n, k) in instances], np.uint64).reshape(-1, 3)
        recs = [resolve_recipe(int(n), d, int(k), cfg) for (_, n, k) in instances]
        cent = np.empty(int(sum(int(k) for (_, _, k) in instances)) * d, np.float32)
        labels = np.empty(int(sum(int(n) for (_, n, _) in instances)), np.uint32)
        obj = np.empty(sum(len(r.epoch_rows) for r in recs), np.float64)
        ns = np.zeros(len(instances), np.uint64)
        c = cfg._c()
        self._check(lib().emb200_train_batched(self._h, ctypes.byref(c), _p(inst), len(instances), max_concurrency,
                                               _p(cent), _p(labels), _p(obj), _p(ns)))
        outs, co, lo, oo = [], 0, 0, 0
        for i, (_, n, k) in enumerate(instances):
            n, k = int(n), int(k)
            ne = len(recs[i].epoch_rows)
            outs.append(Output(cent[co:co + k * d].reshape(k, d), labels[lo:lo + n], obj[oo:oo + ne], int(ns[i]),
                               recs[i]))
            co, lo, oo = co + k * d, lo + n, oo + ne
        return outs

    # ---- learned proposer ------------------------------------------------
    def batched_search_choice(self):
        """(rows, centroids, split_all) of the search tile the autotuner chose for
        the last lockstep train_batched call."""
        r, c, sa = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(lib().emb200_batched_search_choice(self._h, ctypes.byref(r), ctypes.byref(c), ctypes.byref(sa)))
        return r.value, c.value, bool(sa.value)

    def proposer_init(self, groups=256, hidden=512, top=8, mode="mlp", confidence=0.0, batch=4096, lr=2e-3,
                      group_epochs=5.0, seed=1234, mass=0.0):
        """Group the current centroids (e-means with k = groups on the centroids),
        build the group-sorted copy and initialise the network d -> hidden ->
        hidden -> groups (input statistics from the resident rows)."""
        c = _ProposerConfig(groups, hidden, top, PROPOSER_MODES[mode], confidence, batch, lr, group_epochs, seed,
                            mass)
        self._check(lib().emb200_proposer_init(self._h, ctypes.byref(c)))
        self.proposer_top = top
        self._proposer_groups_n = groups

    def proposer_train(self, labels, steps):
        """Adam steps on mini-batches of resident rows labelled by `labels` (one
        per resident row, UINT32_MAX = skip). Returns the per-step mean losses."""
        lab = np.ascontiguousarray(labels, np.uint32)
        losses = np.zeros(steps, np.float32)
        self._check(lib().emb200_proposer_train(self._h, _p(lab), lab.size, steps, _p(losses)))
        return losses

    def proposer_set(self, mode="mlp", top=8, confidence=0.0, mass=0.0):
        """mode; at most `top` groups per row; rows whose top-`top` softmax mass is
        below `confidence` take the full search; each row searches the fewest
        groups whose mass reaches `mass` (0: all `top`)."""
        self._check(lib().emb200_proposer_set(self._h, PROPOSER_MODES[mode], top, confidence, mass))
        self.proposer_top = top

    def proposer_params(self):
        n = lib().emb200_proposer_param_count(self._h)
        out = np.empty(n, np.float32)
        self._check(lib().emb200_proposer_get_params(self._h, _p(out), n))
        return out

    def set_proposer_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self._check(lib().emb200_proposer_set_params(self._h, _p(p), p.size))

    def proposer_grad(self, x, targets):
        """(mean cross-entropy, gradient in the parameter layout) on host rows."""
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(targets, np.uint32)
        g = np.empty(lib().emb200_proposer_param_count(self._h), np.float32)
        loss = ctypes.c_float()
        self._check(lib().emb200_proposer_grad(self._h, _p(x), _p(t), t.size, _p(g), ctypes.byref(loss)))
        return float(loss.value), g

    def proposer_logits(self, x, fused=True):
        """Network logits [m][groups] of host rows, by the fused tcgen05 forward
        pass or by the GEMM forward pass of training."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.d)
        g = self._proposer_groups_n
        out = np.empty((x.shape[0], g), np.float32)
        self._check(lib().emb200_proposer_logits(self._h, _p(x), x.shape[0], _p(out), int(fused)))
        return out

    def proposer_groups(self):
        out = np.empty(self.k, np.uint32)
        self._check(lib().emb200_proposer_groups(self._h, _p(out)))
        return out

    def propose(self, x, with_counts=False):
        """(groups[m][top] most likely first, confidence[m][, counts[m] searched])
        for host rows."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.d)
        g = np.empty((x.shape[0], self.proposer_top), np.uint32)
        conf = np.empty(x.shape[0], np.float32)
        cnt = np.empty(x.shape[0], np.uint32)
        self._check(lib().emb200_propose(self._h, _p(x), x.shape[0], _p(g), _p(conf), _p(cnt)))
        return (g, conf, cnt) if with_counts else (g, conf)

    def assign_proposed(self, want_host=True):
        """The proposer assign over the resident rows."""
        n = self.rows_shape[0]
        labels = np.empty(n, np.uint32) if want_host else None
        dist = np.empty(n, np.float32) if want_host else None
        self._check(lib().emb200_assign_proposed_resident(self._h, _p(labels), _p(dist)))
        return labels, dist

    def assign_proposed_device(self, x_ptr, m, labels_ptr, dist_ptr, stream=None):
        self._check(lib().emb200_assign_proposed_device(self._h, ctypes.c_void_p(x_ptr), m,
                                                        ctypes.c_void_p(labels_ptr), ctypes.c_void_p(dist_ptr),
                                                        ctypes.c_void_p(stream or 0)))

    def train_resident(self, k, cfg: Optional[Config] = None) -> Output:
        """train (src/lib.rs:348-491) on the resident rows, entirely on the device."""
        cfg = cfg or Config()
        n, d = self.rows_shape
        c = cfg._c()
        rec = resolve_recipe(n, d, k, cfg)
        cent = np.empty((k, d), np.float32)
        labels = np.empty(n, np.uint32)
        obj = np.empty(len(rec.epoch_rows), np.float64)
        ns = np.zeros(1, np.uint64)
        r = _Recipe()
        self._check(lib().emb200_train(self._h, ctypes.byref(c), k, _p(cent), _p(labels), _p(obj), _p(ns),
                                       ctypes.byref(r)))
        self.k, self.d = k, d
        return Output(cent, labels, obj, int(ns[0]), rec, self.stats())

    def train_resident_proposed(self, k, cfg: Optional[Config] = None, late_epochs=1, net_steps=4000, groups=256,
                                hidden=512, top=32, confidence=0.0, mass=0.999, batch=4096, lr=2e-3,
                                group_epochs=5.0, seed=7) -> Output:
        """train() with the learned proposer searching the last `late_epochs`
        epochs' batches (emb200_train_proposed): the network is fitted on the
        labels the full search gave in the epoch before them."""
        cfg = cfg or Config()
        n, d = self.rows_shape
        c = cfg._c()
        pc = _ProposerConfig(groups, hidden, top, PROPOSER_MODES["mlp"], confidence, batch, lr, group_epochs, seed,
                             mass)
        rec = resolve_recipe(n, d, k, cfg)
        cent = np.empty((k, d), np.float32)
        labels = np.empty(n, np.uint32)
        obj = np.empty(len(rec.epoch_rows), np.float64)
        ns = np.zeros(1, np.uint64)
        r = _Recipe()
        self._check(lib().emb200_train_proposed(self._h, ctypes.byref(c), k, ctypes.byref(pc), late_epochs, net_steps,
                                                _p(cent), _p(labels), _p(obj), _p(ns), ctypes.byref(r)))
        self.k, self.d = k, d
        self.proposer_top = top
        self._proposer_groups_n = groups
        return Output(cent, labels, obj, int(ns[0]), rec, self.stats())


def train(x, d, k, cfg: Optional[Config] = None, assigner: Optional[B200Assigner] = None) -> Output:
    """train (src/lib.rs:348-491): rows uploaded once, the whole loop on the B200."""
    x = np.ascontiguousarray(x)
    x = x.reshape(-1, d)
    a = assigner or B200Assigner()
    a.load_rows(x)
    return a.train_resident(k, cfg)


def assign(x, centroids, d, assigner: B200Assigner):
    """assign (src/lib.rs:512-520): exact labels and squared distances."""
    x = np.ascontiguousarray(x).reshape(-1, d)
    c = np.ascontiguousarray(centroids, np.float32).reshape(-1, d)
    assigner.set_centroids(c)
    return assigner.assign(x)


# ---- int8 quantizer (src/quantize.rs) ---------------------------------------

@dataclass
class Calibration:
    """src/quantize.rs:17-34."""

    target_peak: float
    quantile: float
    power_of_two: bool

    @staticmethod
    def faiss():
        return Calibration(112.0, 1.0, True)

    @staticmethod
    def clipped(quantile):
        return Calibration(127.0, quantile, False)

    def _c(self):
        return _Calibration(self.target_peak, int(bool(self.power_of_two)), self.quantile)


_quant_handle = None


def _default_assigner(assigner):
    """The handle whose GPU runs a quantizer or report call: the given assigner,
    else one module-wide handle on device 0."""
    global _quant_handle
    if assigner is not None:
        return assigner
    if _quant_handle is None:
        _quant_handle = B200Assigner(0)
    return _quant_handle


class Int8Quantizer:
    """Int8Quantizer (src/quantize.rs:36-96): one per-dimension shift and one
    global scale; fit, encode and clipped_fraction run on the B200."""

    def __init__(self, d, shift, scale):
        self.d = int(d)
        self.shift = np.ascontiguousarray(shift, np.float32)
        self.scale = np.float32(scale)

    @classmethod
    def fit(cls, sample, d, cal: Calibration, assigner: Optional[B200Assigner] = None):
        """Int8Quantizer::fit (src/quantize.rs:45-62) on a host sample."""
        x = np.ascontiguousarray(sample, np.float32).reshape(-1)
        n = x.size // d
        if n == 0 or x.size != n * d:
            raise ValueError("the sample must hold n > 0 whole rows of d values")
        a = _default_assigner(assigner)
        shift = np.empty(d, np.float32)
        scale = ctypes.c_float()
        c = cal._c()
        a._check(lib().emb200_quantizer_fit(a._h, _p(x), n, d, ctypes.byref(c), _p(shift), ctypes.byref(scale)))
        return cls(d, shift, scale.value)

    @classmethod
    def fit_resident(cls, assigner: B200Assigner, cal: Calibration):
        """fit on the assigner's resident f32 rows (no host copy)."""
        n, d = assigner.rows_shape
        shift = np.empty(d, np.float32)
        scale = ctypes.c_float()
        c = cal._c()
        assigner._check(lib().emb200_quantizer_fit_resident(assigner._h, ctypes.byref(c), _p(shift),
                                                            ctypes.byref(scale)))
        return cls(d, shift, scale.value)

    def _encode(self, x, codes, assigner):
        x = np.ascontiguousarray(x, np.float32).reshape(-1)
        if x.size % self.d:
            raise ValueError("rows must hold whole rows of d values")
        a = _default_assigner(assigner)
        clipped = ctypes.c_uint64()
        a._check(lib().emb200_quantizer_encode(a._h, _p(x), x.size // self.d, self.d, _p(self.shift),
                                               float(self.scale), _p(codes), ctypes.byref(clipped)))
        return clipped.value, x.size

    def encode(self, x, assigner: Optional[B200Assigner] = None):
        """Int8Quantizer::encode (src/quantize.rs:65-73): codes with x's shape."""
        x = np.asarray(x, np.float32)
        codes = np.empty(x.size, np.int8)
        self._encode(x, codes, assigner)
        return codes.reshape(x.shape)

    def clipped_fraction(self, x, assigner: Optional[B200Assigner] = None):
        """Int8Quantizer::clipped_fraction (src/quantize.rs:87-95)."""
        clipped, size = self._encode(x, None, assigner)
        return clipped / size

    def decode(self, codes, assigner: Optional[B200Assigner] = None):
        """Int8Quantizer::decode (src/quantize.rs:76-79): codes (any numeric array,
        as f32) back to the original units."""
        c = np.ascontiguousarray(codes, np.float32)
        flat = c.reshape(-1)
        if flat.size % self.d:
            raise ValueError("codes must hold whole rows of d values")
        out = np.empty(flat.size, np.float32)
        a = _default_assigner(assigner)
        a._check(lib().emb200_quantizer_decode(a._h, _p(flat), flat.size // self.d, self.d, _p(self.shift),
                                               float(self.scale), _p(out)))
        return out.reshape(c.shape)

    def decode_sqdist(self, sqdist):
        """src/quantize.rs:82-84 (a scalar or array of f32 squared distances)."""
        s = np.float32(self.scale)
        return (np.asarray(sqdist, np.float32) / (s * s)).astype(np.float32)

    def quantize_resident(self, assigner: B200Assigner):
        """Replace the assigner's resident f32 rows by their codes (resident i8
        rows); returns the number of values that clipped."""
        clipped = ctypes.c_uint64()
        assigner._check(lib().emb200_quantize_resident(assigner._h, _p(self.shift), float(self.scale),
                                                       ctypes.byref(clipped)))
        return clipped.value


# ---- report (src/report.rs) --------------------------------------------------

@dataclass
class ReportConfig:
    """src/report.rs:21-34."""

    family_radius: float = 1.25
    min_local_size: int = 30
    family_pass: int = 0  # engine option: 0 auto, 1 parallel rounds, 2 sequential greedy (same result)

    def _c(self):
        return _ReportConfig(self.family_radius, self.family_pass, self.min_local_size)


@dataclass
class Family:
    """src/report.rs:58-66."""

    leader: int
    members: np.ndarray
    size: int
    share: float


def _order_key(v):
    """f32::total_cmp as an unsigned order."""
    b = np.ascontiguousarray(v, np.float32).view(np.uint32)
    return b ^ np.where(b >> 31 != 0, np.uint32(0xFFFFFFFF), np.uint32(0x80000000))


class Report:
    """Report (src/report.rs:68-81): computed by `report()` on the B200; the
    methods below (src/report.rs:243-291) are views over its arrays."""

    def __init__(self, clusters, families, local_z, global_z, median_dist, median_rms, median_nearest_dist):
        self.clusters = clusters  # CLUSTER_STATS array of k
        self.families = families  # list of Family, largest first
        self.local_z = local_z
        self.global_z = global_z
        self.median_dist = np.float32(median_dist)
        self.median_rms = np.float32(median_rms)
        self.median_nearest_dist = np.float32(median_nearest_dist)

    def scores(self):
        """score() of every row: max(local_z, global_z), NaN ignored as f32::max does."""
        return np.fmax(self.local_z, self.global_z)

    def score(self, row):
        """src/report.rs:246-248."""
        return np.float32(np.fmax(self.local_z[row], self.global_z[row]))

    def top_outliers(self, count):
        """The `count` highest-scoring rows as (row, score), best first (total_cmp
        order; equal scores by row index)."""
        s = self.scores()
        count = min(count, s.size)
        key = np.uint32(0xFFFFFFFF) - _order_key(s)
        idx = np.argsort(key, kind="stable")[:count]
        return [(int(i), np.float32(s[i])) for i in idx]

    def rare_prototypes(self, max_size_ratio, min_isolation):
        """(cluster, size, isolation) of small, isolated clusters, most isolated
        first (src/report.rs:264-276; equal isolation by cluster index)."""
        c = self.clusters
        live = max(int(np.count_nonzero(c["size"])), 1)
        mean = np.float32(self.local_z.size) / np.float32(live)
        thr = np.float32(max_size_ratio) * mean
        sel = (c["size"] > 0) & (c["size"].astype(np.float32) <= thr) & (c["isolation"] >= np.float32(min_isolation))
        js = np.nonzero(sel)[0]
        key = np.uint32(0xFFFFFFFF) - _order_key(c["isolation"][js])
        js = js[np.argsort(key, kind="stable")]
        return [(int(j), int(c["size"][j]), np.float32(c["isolation"][j])) for j in js]

    def write_clusters_tsv(self, w):
        """src/report.rs:279-290."""
        w.write("cluster\tsize\trms\tmedian\tmad\tp90\tp99\tmax\tlooseness\tnearest_centroid\tnearest_dist"
                "\tisolation\tfamily\tfamily_share\n")
        for j, c in enumerate(self.clusters):
            share = self.families[int(c["family"])].share if c["size"] > 0 else 0.0
            w.write(f"{j}\t{c['size']}\t{c['rms']:.5f}\t{c['median']:.5f}\t{c['mad']:.5f}\t{c['p90']:.5f}\t"
                    f"{c['p99']:.5f}\t{c['max']:.5f}\t{c['looseness']:.3f}\t{c['nearest_centroid']}\t"
                    f"{c['nearest_dist']:.5f}\t{c['isolation']:.3f}\t{c['family']}\t{share:.6f}\n")


def _report_result(a, n, k, clusters, lz, gz, summ):
    F, live = summ.n_families, summ.n_live
    leader = np.empty(max(F, 1), np.uint32)
    size = np.empty(max(F, 1), np.uint64)
    share = np.empty(max(F, 1), np.float64)
    offs = np.empty(F + 1, np.uint32)
    mem = np.empty(max(live, 1), np.uint32)
    a._check(lib().emb200_report_families(a._h, _p(leader), _p(size), _p(share), _p(offs), _p(mem)))
    fams = [Family(int(leader[f]), mem[offs[f]:offs[f + 1]].copy(), int(size[f]), float(share[f])) for f in range(F)]
    return Report(clusters, fams, lz, gz, summ.median_dist, summ.median_rms, summ.median_nearest_dist)


def report(labels, sqdist_to_centroid, centroids, d, cfg: Optional[ReportConfig] = None,
           assigner: Optional[B200Assigner] = None) -> Report:
    """report() (src/report.rs:121-241) on the B200."""
    cfg = cfg or ReportConfig()
    lab = np.ascontiguousarray(labels, np.uint32)
    sq = np.ascontiguousarray(sqdist_to_centroid, np.float32)
    c = np.ascontiguousarray(centroids, np.float32).reshape(-1)
    if lab.size != sq.size:
        raise ValueError("labels and distances differ in length")
    k = c.size // d
    if c.size != k * d:
        raise ValueError("centroids must be k x d")
    a = _default_assigner(assigner)
    n = lab.size
    clusters = np.zeros(k, CLUSTER_STATS)
    lz = np.empty(n, np.float32)
    gz = np.empty(n, np.float32)
    summ = _ReportSummary()
    cc = cfg._c()
    a._check(lib().emb200_report(a._h, _p(lab), _p(sq), n, _p(c), k, d, ctypes.byref(cc), _p(clusters), _p(lz), _p(gz),
                                 ctypes.byref(summ)))
    return _report_result(a, n, k, clusters, lz, gz, summ)


def report_resident(assigner: B200Assigner, cfg: Optional[ReportConfig] = None) -> Report:
    """report() over the assigner's last assign_resident results and its
    centroids, without leaving HBM."""
    cfg = cfg or ReportConfig()
    n = assigner.rows_shape[0]
    k = assigner.k
    clusters = np.zeros(k, CLUSTER_STATS)
    lz = np.empty(n, np.float32)
    gz = np.empty(n, np.float32)
    summ = _ReportSummary()
    cc = cfg._c()
    assigner._check(lib().emb200_report_resident(assigner._h, ctypes.byref(cc), _p(clusters), _p(lz), _p(gz),
                                                 ctypes.byref(summ)))
    return _report_result(assigner, n, k, clusters, lz, gz, summ)
