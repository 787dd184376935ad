"""ctypes bindings for the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the oracle restates the reference crate's CPU code
(src/lib.rs, src/cpu.rs, src/cpu_i8.rs, src/quantize.rs) so the B200 engine can
be checked against it. Only tests/, the smoke check and the CPU-baseline leg of
bench.py import this module; the engine never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

KERNELS = {"avx512": 0, "avx2": 1, "portable": 2}
DTYPES = {np.dtype(np.float32): 0, np.dtype(np.int8): 1, np.dtype(np.uint8): 2}


class Config(ctypes.Structure):
    """Mirror of src/lib.rs:104-124 (sentinels: batch_size 0, alpha0 <= 0 and
    unused_threshold < 0 mean None)."""

    _fields_ = [
        ("nepochs", ctypes.c_double),
        ("batch_law", ctypes.c_int),
        ("batch_size", ctypes.c_uint64),
        ("alpha0", ctypes.c_double),
        ("unused_threshold", ctypes.c_float),
        ("balance", ctypes.c_float),
        ("seed", ctypes.c_uint64),
    ]


class Recipe(ctypes.Structure):
    _fields_ = [
        ("batch_size", ctypes.c_uint64),
        ("alpha0", ctypes.c_double),
        ("n_epochs", ctypes.c_uint64),
        ("total_steps", ctypes.c_uint64),
        ("unused_threshold", ctypes.c_float),
    ]


def build():
    """Compile liboracle.so from its source with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "emeans_oracle.cpp")):
            build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        S = ctypes.c_size_t
        L.orc_scheduled_alpha.restype = ctypes.c_double
        L.orc_scheduled_alpha.argtypes = [ctypes.c_double, S, S]
        L.orc_resolve_recipe.argtypes = [S, S, S, ctypes.POINTER(Config), ctypes.POINTER(Recipe), P, S]
        L.orc_rng_u64.argtypes = [ctypes.c_uint64, S, P]
        L.orc_rng_open01.argtypes = [ctypes.c_uint64, S, P]
        L.orc_rng_permutation.argtypes = [ctypes.c_uint64, S, P]
        L.orc_cpu_assign.argtypes = [ctypes.c_int, ctypes.c_int, P, S, S, P, S, P, P, P, ctypes.c_int]
        L.orc_i8_assign.argtypes = [ctypes.c_int, P, S, S, P, S, P, P, P, ctypes.c_int]
        L.orc_bruteforce_f64.argtypes = [ctypes.c_int, P, S, S, P, S, P, P, ctypes.c_int]
        L.orc_score.restype = ctypes.c_float
        L.orc_score.argtypes = [ctypes.c_int, P, P, S]
        L.orc_sqnorm.restype = ctypes.c_float
        L.orc_sqnorm.argtypes = [P, S]
        L.orc_state_apply.argtypes = [S, S, P, P, P, S, P, P, ctypes.c_float]
        L.orc_state_revive.restype = S
        L.orc_state_revive.argtypes = [S, S, P, P, ctypes.c_float, ctypes.c_uint64]
        L.orc_train.argtypes = [ctypes.c_int, P, S, S, S, ctypes.POINTER(Config), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, P, P, P, P]
        L.orc_balance_stats.argtypes = [P, S, S, P]
        L.orc_quantizer_fit.argtypes = [P, S, S, ctypes.c_float, ctypes.c_double, ctypes.c_int, P, P]
        L.orc_quantizer_encode.argtypes = [P, S, S, P, ctypes.c_float, P]
        L.orc_quantizer_clipped.restype = ctypes.c_uint64
        L.orc_quantizer_clipped.argtypes = [P, S, S, P, ctypes.c_float]
        L.orc_quantizer_decode.argtypes = [P, S, S, P, ctypes.c_float, P]
        L.orc_cpu_has_kernel.argtypes = [ctypes.c_int]
        L.orc_report.argtypes = [P, P, S, P, S, S, ctypes.c_float, S, P, P, P, P, P, P, P, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def threads():
    return os.cpu_count() or 1


def make_config(nepochs=5.0, batch_law="auto", batch_size=None, alpha0=None, unused_threshold=None, balance=0.0,
                seed=1234):
    law = {"auto": 0, "throughput": 1, "quality": 2}[batch_law]
    return Config(nepochs, law, batch_size or 0, alpha0 if alpha0 is not None else -1.0,
                  unused_threshold if unused_threshold is not None else -1.0, balance, seed)


def resolve_recipe(n, d, k, cfg=None):
    cfg = cfg or make_config()
    r = Recipe()
    er = np.zeros(int(np.floor(cfg.nepochs)) + 2, np.uint64)
    lib().orc_resolve_recipe(n, d, k, ctypes.byref(cfg), ctypes.byref(r), _p(er), er.size)
    return {"batch_size": r.batch_size, "alpha0": r.alpha0, "epoch_rows": [int(v) for v in er[:r.n_epochs]],
            "total_steps": r.total_steps, "unused_threshold": r.unused_threshold}


def scheduled_alpha(alpha0, step, total):
    return lib().orc_scheduled_alpha(alpha0, step, total)


def rng_u64(seed, m):
    out = np.zeros(m, np.uint64)
    lib().orc_rng_u64(seed, m, _p(out))
    return out


def rng_open01(seed, m):
    out = np.zeros(m, np.float64)
    lib().orc_rng_open01(seed, m, _p(out))
    return out


def permutation(seed, n):
    out = np.zeros(n, np.uint32)
    lib().orc_rng_permutation(seed, n, _p(out))
    return out


def has_kernel(kernel):
    return bool(lib().orc_cpu_has_kernel(KERNELS[kernel]))


def cpu_assign(x, c, bias=None, kernel="avx512", emulate=False, nthreads=None):
    """CpuAssigner (src/cpu.rs:83-167): labels (u32) and distances (f32)."""
    x = np.ascontiguousarray(x)
    c = np.ascontiguousarray(c, np.float32)
    m, d = x.shape
    k = c.shape[0]
    labels = np.zeros(m, np.uint32)
    dist = np.zeros(m, np.float32)
    b = None if bias is None else np.ascontiguousarray(bias, np.float32)
    kv = KERNELS[kernel] | (8 if emulate else 0)
    rc = lib().orc_cpu_assign(kv, DTYPES[x.dtype], _p(x), m, d, _p(c), k, None if b is None else _p(b),
                              _p(labels), _p(dist), nthreads or threads())
    if rc != 0:
        raise RuntimeError(f"kernel {kernel} unavailable on this CPU")
    return labels, dist


def i8_assign(x, c, bits=8, bias=None, nthreads=None):
    """CpuI8Assigner (src/cpu_i8.rs:72-191) for i8 rows."""
    x = np.ascontiguousarray(x, np.int8)
    c = np.ascontiguousarray(c, np.float32)
    m, d = x.shape
    k = c.shape[0]
    labels = np.zeros(m, np.uint32)
    dist = np.zeros(m, np.float32)
    b = None if bias is None else np.ascontiguousarray(bias, np.float32)
    rc = lib().orc_i8_assign(bits, _p(x), m, d, _p(c), k, None if b is None else _p(b), _p(labels), _p(dist),
                             nthreads or threads())
    if rc != 0:
        raise RuntimeError("integer assignment supports d <= 32768")
    return labels, dist


def bruteforce_f64(x, c, nthreads=None):
    x = np.ascontiguousarray(x)
    c = np.ascontiguousarray(c, np.float32)
    m, d = x.shape
    labels = np.zeros(m, np.uint32)
    dist = np.zeros(m, np.float64)
    lib().orc_bruteforce_f64(DTYPES[x.dtype], _p(x), m, d, _p(c), c.shape[0], _p(labels), _p(dist),
                             nthreads or threads())
    return labels, dist


def score(x, c, kernel="avx512"):
    x = np.ascontiguousarray(x, np.float32)
    c = np.ascontiguousarray(c, np.float32)
    return lib().orc_score(KERNELS[kernel], _p(x), _p(c), x.size)


def sqnorm(v):
    v = np.ascontiguousarray(v, np.float32)
    return lib().orc_sqnorm(_p(v), v.size)


def state_apply(centroids, usage, touched, counts, sums, alpha):
    k, d = centroids.shape
    t = np.ascontiguousarray(touched, np.uint32)
    lib().orc_state_apply(k, d, _p(centroids), _p(usage), _p(t), t.size, _p(np.ascontiguousarray(counts, np.uint32)),
                          _p(np.ascontiguousarray(sums, np.float32)), alpha)


def state_revive(centroids, usage, tau, rng_seed):
    k, d = centroids.shape
    return lib().orc_state_revive(k, d, _p(centroids), _p(usage), tau, rng_seed)


ASSIGNERS = {"cpu": 0, "i8": 1, "i16": 2}


def train(x, k, cfg=None, assigner="cpu", kernel="avx512", emulate=False, nthreads=None):
    """train (src/lib.rs:348-491). Returns a dict like Output (src/lib.rs:152-163)."""
    cfg = cfg or make_config()
    x = np.ascontiguousarray(x)
    n, d = x.shape
    rec = resolve_recipe(n, d, k, cfg)
    cent = np.zeros((k, d), np.float32)
    labels = np.zeros(n, np.uint32)
    obj = np.zeros(len(rec["epoch_rows"]), np.float64)
    ns = np.zeros(1, np.uint64)
    kv = KERNELS[kernel] | (8 if emulate else 0)
    rc = lib().orc_train(DTYPES[x.dtype], _p(x), n, d, k, ctypes.byref(cfg), ASSIGNERS[assigner], kv,
                         nthreads or threads(), _p(cent), _p(labels), _p(obj), _p(ns))
    if rc != 0:
        raise RuntimeError(f"oracle train failed ({rc})")
    return {"centroids": cent, "labels": labels, "objective": obj, "n_splits": int(ns[0]), "recipe": rec}


def balance_stats(labels, k):
    out = np.zeros(3, np.float64)
    lab = np.ascontiguousarray(labels, np.uint32)
    lib().orc_balance_stats(_p(lab), lab.size, k, _p(out))
    return out[0], out[1], int(out[2])


def quantizer_fit(sample, target_peak=112.0, quantile=1.0, power_of_two=True):
    s = np.ascontiguousarray(sample, np.float32)
    n, d = s.shape
    shift = np.zeros(d, np.float32)
    scale = np.zeros(1, np.float32)
    lib().orc_quantizer_fit(_p(s), n, d, target_peak, quantile, int(power_of_two), _p(shift), _p(scale))
    return shift, float(scale[0])


def quantizer_clipped(x, shift, scale):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    return int(lib().orc_quantizer_clipped(_p(x), n, d, _p(np.ascontiguousarray(shift, np.float32)), scale))


def quantizer_decode(codes, shift, scale):
    c = np.ascontiguousarray(codes, np.float32)
    n, d = c.shape
    out = np.zeros((n, d), np.float32)
    lib().orc_quantizer_decode(_p(c), n, d, _p(np.ascontiguousarray(shift, np.float32)), scale, _p(out))
    return out


def quantizer_encode(x, shift, scale):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    out = np.zeros((n, d), np.int8)
    lib().orc_quantizer_encode(_p(x), n, d, _p(np.ascontiguousarray(shift, np.float32)), scale, _p(out))
    return out


# ClusterStats, src/report.rs:37-56 (field order kept; 48 bytes, no padding)
CLUSTER_STATS = np.dtype([("size", "u4"), ("rms", "f4"), ("median", "f4"), ("mad", "f4"), ("p90", "f4"),
                          ("p99", "f4"), ("max", "f4"), ("looseness", "f4"), ("nearest_centroid", "u4"),
                          ("nearest_dist", "f4"), ("isolation", "f4"), ("family", "u4")])


def report(labels, sqdist, centroids, family_radius=1.25, min_local_size=30):
    """report() (src/report.rs:121-241). Returns a dict: clusters (CLUSTER_STATS
    array), local_z, global_z, median_dist, median_rms, median_nearest_dist,
    families (list of (leader, members, size, share))."""
    labels = np.ascontiguousarray(labels, np.uint32)
    sq = np.ascontiguousarray(sqdist, np.float32)
    c = np.ascontiguousarray(centroids, np.float32)
    k, d = c.shape
    n = labels.size
    clusters = np.zeros(k, CLUSTER_STATS)
    lz = np.zeros(n, np.float32)
    gz = np.zeros(n, np.float32)
    med = np.zeros(3, np.float32)
    nf = np.zeros(1, np.uint32)
    leader = np.zeros(max(k, 1), np.uint32)
    fsize = np.zeros(max(k, 1), np.uint64)
    share = np.zeros(max(k, 1), np.float64)
    offs = np.zeros(k + 1, np.uint32)
    mem = np.zeros(max(k, 1), np.uint32)
    lib().orc_report(_p(labels), _p(sq), n, _p(c), k, d, family_radius, min_local_size, _p(clusters), _p(lz), _p(gz),
                     _p(med), _p(nf), _p(leader), _p(fsize), _p(share), _p(offs), _p(mem))
    F = int(nf[0])
    fams = [(int(leader[f]), mem[offs[f]:offs[f + 1]].copy(), int(fsize[f]), float(share[f])) for f in range(F)]
    return {"clusters": clusters, "local_z": lz, "global_z": gz, "median_dist": med[0], "median_rms": med[1],
            "median_nearest_dist": med[2], "families": fams}
