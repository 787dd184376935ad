"""Seeded synthetic inputs for the five benchmark workloads.

There is no public dataset for this path; these generators stand in for it,
with the shapes, sizes and value distributions each workload names. All use
numpy's default_rng(seed) and return row-major float32 (or int8) arrays.
"""
import numpy as np


def blobs(n=200_000, d=96, n_blobs=4096, centre_std=4.0, blob_std=1.0, seed=0):
    """Equal-weight Gaussian mixture: centres N(0, centre_std^2 I), within-blob N(0, blob_std^2)."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((n_blobs, d), dtype=np.float32) * np.float32(centre_std)
    which = rng.integers(0, n_blobs, n)
    x = centres[which]
    x += rng.standard_normal((n, d), dtype=np.float32) * np.float32(blob_std)
    return x


def embeddings(n=1_000_000, d=128, latent=32, noise=0.1, seed=0, chunk=262_144):
    """Embedding-like rows: N(0,1) latent times a random Gaussian latent x d map, plus
    N(0, noise^2) noise, each row L2-normalised."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((latent, d), dtype=np.float32)
    x = np.empty((n, d), np.float32)
    for r0 in range(0, n, chunk):
        m = min(chunk, n - r0)
        z = rng.standard_normal((m, latent), dtype=np.float32)
        v = z @ w
        v += rng.standard_normal((m, d), dtype=np.float32) * np.float32(noise)
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        x[r0:r0 + m] = v
    return x


def heavy_tailed(n=10_000_000, d=96, latent=32, components=8192, nu=3.0, seed=0, chunk=262_144):
    """Student-t (nu) latents through a random latent x d map, as a mixture of
    `components` such clouds (each with its own latent offset)."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((latent, d), dtype=np.float32)
    offsets = rng.standard_normal((components, latent), dtype=np.float32) * np.float32(3.0)
    x = np.empty((n, d), np.float32)
    for r0 in range(0, n, chunk):
        m = min(chunk, n - r0)
        comp = rng.integers(0, components, m)
        t = rng.standard_t(nu, (m, latent)).astype(np.float32)
        x[r0:r0 + m] = (offsets[comp] + t) @ w
    return x


def gaussian_mixture(n=4_000_000, d=128, components=1024, seed=0, chunk=262_144):
    """Gaussian mixture for product-quantisation training (centres N(0, 4 I), unit spread)."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((components, d), dtype=np.float32) * np.float32(2.0)
    x = np.empty((n, d), np.float32)
    for r0 in range(0, n, chunk):
        m = min(chunk, n - r0)
        x[r0:r0 + m] = centres[rng.integers(0, components, m)] + rng.standard_normal((m, d), dtype=np.float32)
    return x


def ivf_list_sizes(lists=48, median=20_000, sigma=1.0, lo=2_000, hi=200_000, seed=0):
    """Log-normal list sizes (median `median`), clipped to [lo, hi]; k = max(16, n // 256)."""
    rng = np.random.default_rng(seed)
    n = np.clip(np.round(rng.lognormal(np.log(median), sigma, lists)), lo, hi).astype(np.int64)
    k = np.maximum(16, n // 256)
    return n, k


def faiss_int8(x, target_peak=112.0):
    """Per-dimension mean shift and one global power-of-two scale putting the largest
    centred magnitude at or below `target_peak` (the faiss calibration), then round
    half away from zero and clamp to int8. Returns (codes, shift, scale)."""
    shift = x.astype(np.float64).mean(0).astype(np.float32)
    peak = np.float32(0.0)
    for r0 in range(0, x.shape[0], 262_144):
        peak = max(peak, np.abs(x[r0:r0 + 262_144] - shift).max())
    scale = np.float32(target_peak) / peak if peak > 0 else np.float32(1.0)
    scale = np.float32(2.0) ** np.float32(np.floor(np.log2(np.float32(scale))))
    codes = np.empty(x.shape, np.int8)
    for r0 in range(0, x.shape[0], 262_144):
        v = (x[r0:r0 + 262_144] - shift) * scale
        r = np.trunc(v + np.copysign(np.float32(0.5), v))  # half away from zero
        # trunc(v +/- 0.5) can round up values just below .5; fix those with an exact check.
        fix = np.abs(r - v) > np.float32(0.5)
        r[fix] -= np.copysign(np.float32(1.0), v[fix])
        codes[r0:r0 + 262_144] = np.clip(r, -128, 127).astype(np.int8)
    return codes, shift, np.float32(scale)


def embeddings_int8(n=2_000_000, d=512, latent=64, noise=0.1, seed=0, chunk=262_144, target_peak=112.0):
    """The int8 workload: unit-norm embedding rows (as `embeddings`) quantised with
    the faiss calibration (per-dimension mean shift, one power-of-two scale putting
    the largest centred magnitude at or below `target_peak`, round half away from
    zero, clamp). Two passes over regenerated chunks, so only the int8 codes are
    held. Returns (codes, shift, scale)."""
    def chunks():
        rng = np.random.default_rng(seed)
        w = rng.standard_normal((latent, d), dtype=np.float32)
        for r0 in range(0, n, chunk):
            m = min(chunk, n - r0)
            z = rng.standard_normal((m, latent), dtype=np.float32)
            v = z @ w
            v += rng.standard_normal((m, d), dtype=np.float32) * np.float32(noise)
            v /= np.linalg.norm(v, axis=1, keepdims=True)
            yield r0, v
    total = np.zeros(d, np.float64)
    for _, v in chunks():
        total += v.astype(np.float64).sum(0)
    shift = (total / n).astype(np.float32)
    peak = np.float32(0.0)
    for _, v in chunks():
        peak = max(peak, np.abs(v - shift).max())
    scale = np.float32(target_peak) / peak if peak > 0 else np.float32(1.0)
    scale = np.float32(2.0) ** np.float32(np.floor(np.log2(np.float32(scale))))
    codes = np.empty((n, d), np.int8)
    for r0, v in chunks():
        t = (v - shift) * scale
        r = np.trunc(t + np.copysign(np.float32(0.5), t))
        fix = np.abs(r - t) > np.float32(0.5)
        r[fix] -= np.copysign(np.float32(1.0), t[fix])
        codes[r0:r0 + len(v)] = np.clip(r, -128, 127).astype(np.int8)
    return codes, shift, np.float32(scale)


def pq_subspaces(n=4_000_000, d=128, sub=16, seed=0):
    """Product-quantisation training data: `gaussian_mixture` rows split into `sub`
    contiguous sub-spaces of d/sub dimensions, returned sub-space-major as one
    (sub * n) x (d / sub) matrix: sub-space s is rows [s n, (s + 1) n)."""
    x = gaussian_mixture(n, d, seed=seed)
    ds = d // sub
    out = np.empty((sub * n, ds), np.float32)
    for s in range(sub):
        out[s * n:(s + 1) * n] = x[:, s * ds:(s + 1) * ds]
    return out


def ivf_lists(lists=48, d=64, median=20_000, seed=0):
    """IVF-list refinement data: per list a local Gaussian mixture (its own centre,
    64 sub-clusters of spread 0.5 around it), list sizes log-normal with median
    `median` clipped to [2,000, 200,000]. Returns (rows concatenated list by list,
    sizes, k per list = max(16, n // 256))."""
    sizes, ks = ivf_list_sizes(lists, median, seed=seed)
    rng = np.random.default_rng(seed + 1)
    parts = []
    for n in sizes:
        centre = rng.standard_normal(d, dtype=np.float32) * np.float32(4.0)
        subs = centre + rng.standard_normal((64, d), dtype=np.float32)
        rows = subs[rng.integers(0, 64, int(n))] + rng.standard_normal((int(n), d), dtype=np.float32) * np.float32(0.5)
        parts.append(rows.astype(np.float32))
    return np.concatenate(parts), sizes, ks
