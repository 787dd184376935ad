"""Test infrastructure: FP64 CPU oracle of the proposer network.

The reference crate has no learned part, so there is nothing of it to restate
here; this module states the network's mathematics once, in float64 numpy, so
that the GPU forward and backward kernels can be checked against it:

    x0 = bf16((x - mean) * inv_std)            (the network's input, as the GPU rounds it)
    h1 = relu(x0 W1^T + b1), h2 = relu(h1 W2^T + b2), z = h2 W3^T + b3
    loss = mean_i [logsumexp(z_i) - z_i[t_i]]

with the weights taken at their BF16 values (the GEMM operands). The analytic
gradient below is checked against central finite differences in the CPU test
suite, which pins the oracle itself. Only tests/ and the bench's reporting may
import this module.
"""
import numpy as np


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def _round8(v):
    return (v + 7) // 8 * 8


def layout(d, hidden, groups):
    """Offsets of the flat parameter array: mean, inv_std, W1, b1, W2, b2, W3, b3
    (each block starting at a multiple of 8)."""
    off = {}
    o = 0
    for name, n in (("mean", d), ("istd", d), ("w1", hidden * d), ("b1", hidden), ("w2", hidden * hidden),
                    ("b2", hidden), ("w3", groups * hidden), ("b3", groups)):
        off[name] = (o, n)
        o = _round8(o + n)
    off["total"] = o
    return off


def unpack(params, d, hidden, groups, weights_bf16=True):
    L = layout(d, hidden, groups)
    g = {}
    for name in ("mean", "istd", "w1", "b1", "w2", "b2", "w3", "b3"):
        o, n = L[name]
        g[name] = np.asarray(params[o:o + n], np.float32)
    g["w1"] = g["w1"].reshape(hidden, d)
    g["w2"] = g["w2"].reshape(hidden, hidden)
    g["w3"] = g["w3"].reshape(groups, hidden)
    if weights_bf16:
        for name in ("w1", "w2", "w3"):
            g[name] = bf16(g[name])
    return {k: v.astype(np.float64) for k, v in g.items()}, L


def network_input(x, mean, istd):
    """The standardised input exactly as the GPU forms it (f32 arithmetic, then BF16)."""
    x = np.asarray(x, np.float32)
    return bf16((x - mean.astype(np.float32)) * istd.astype(np.float32)).astype(np.float64)


def forward(x0, p):
    z1 = x0 @ p["w1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["w2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    z = h2 @ p["w3"].T + p["b3"]
    return z1, h1, z2, h2, z


def loss_and_grad(x0, targets, p):
    """Mean cross-entropy and its gradient (dict of float64 arrays) in FP64."""
    m = x0.shape[0]
    z1, h1, z2, h2, z = forward(x0, p)
    zmax = z.max(1, keepdims=True)
    e = np.exp(z - zmax)
    s = e.sum(1, keepdims=True)
    loss = float(np.mean(np.log(s[:, 0]) + zmax[:, 0] - z[np.arange(m), targets]))
    dz = e / s
    dz[np.arange(m), targets] -= 1.0
    dz /= m
    g = {"w3": dz.T @ h2, "b3": dz.sum(0)}
    dh2 = (dz @ p["w3"]) * (z2 > 0)
    g["w2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["w2"]) * (z1 > 0)
    g["w1"] = dh1.T @ x0
    g["b1"] = dh1.sum(0)
    return loss, g


def loss_only(x0, targets, p):
    z = forward(x0, p)[-1]
    zmax = z.max(1, keepdims=True)
    return float(np.mean(np.log(np.exp(z - zmax).sum(1)) + zmax[:, 0] - z[np.arange(len(targets)), targets]))


def flat_grad(g, d, hidden, groups):
    """Gradient dict -> flat array in the parameter layout (statistics entries zero)."""
    L = layout(d, hidden, groups)
    out = np.zeros(L["total"], np.float64)
    for name in ("w1", "b1", "w2", "b2", "w3", "b3"):
        o, n = L[name]
        out[o:o + n] = g[name].reshape(-1)
    return out
