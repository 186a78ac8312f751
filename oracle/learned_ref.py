"""CPU reference of the learned per-block preconditioner (test
infrastructure: only tests/ may import it).

The network of batsrus_b200/csrc/bx_learned.cuh restated in numpy: on one
8^3 block, three 3x3x3 convolutions 16 -> 32 -> 32 -> 8 channels with zero
padding at the block faces, ReLU after the first two.  Tensors are
[sample][z][y][x][channel]; the parameter vector is

    W1[27][16][32] b1[32] W2[27][32][32] b2[32] W3[27][32][8] b3[8]

with tap = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1).  With ``bf16=True`` the
operands are rounded to BF16 where the GPU stores them in BF16 (inputs,
weights, activations, output gradients); sums are taken in FP64, so the
GPU's FP32 accumulation differs from this reference by accumulation order
only (plus an occasional one-ulp BF16 rounding difference of an
intermediate value).
"""
import numpy as np

C0, C1, C2, C3 = 16, 32, 32, 8
TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
SHAPES = [("W1", (27, C0, C1)), ("b1", (C1,)), ("W2", (27, C1, C2)), ("b2", (C2,)), ("W3", (27, C2, C3)),
          ("b3", (C3,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(a):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float32).ravel() for name, _ in SHAPES])


def _shift(x, dz, dy, dx):
    """y[.., z, y, x, :] = x[.., z + dz, y + dy, x + dx, :], zero outside."""
    p = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    return p[:, 1 + dz:9 + dz, 1 + dy:9 + dy, 1 + dx:9 + dx, :]


def conv(x, W):
    out = 0.0
    for t, (dz, dy, dx) in enumerate(TAPS):
        out = out + _shift(x, dz, dy, dx) @ W[t]
    return out


def conv_t(g, W):
    """dX[cell][ci] = sum_tap g[cell - tap] . W[tap][ci][:]"""
    out = 0.0
    for t, (dz, dy, dx) in enumerate(TAPS):
        out = out + _shift(g, -dz, -dy, -dx) @ W[t].T
    return out


def weight_grad(x, g):
    """dW[tap][ci][co] = sum over samples, cells of x[cell + tap][ci] g[cell][co]"""
    n = x.shape[0] * 512
    return np.stack([_shift(x, dz, dy, dx).reshape(n, -1).T @ g.reshape(n, -1) for dz, dy, dx in TAPS])


def _round(a, on):
    return bf16(a).astype(np.float64) if on else np.asarray(a, dtype=np.float64)


def forward(p, x0, bf=True, relu=True):
    """x0: [n, 8, 8, 8, 16] network input; returns (out, a1, a2).  relu=False
    is the linear mode (no activation)."""
    P = unpack(p)
    W1, W2, W3 = (_round(P[k], bf) for k in ("W1", "W2", "W3"))
    x0 = _round(x0, bf)
    act = (lambda a: np.maximum(a, 0.0)) if relu else (lambda a: a)
    a1 = _round(act(conv(x0, W1) + P["b1"]), bf)
    a2 = _round(act(conv(a1, W2) + P["b2"]), bf)
    out = conv(a2, W3) + P["b3"]
    return out, a1, a2


def loss_and_grad(p, x0, tgt, bf=True, relu=True):
    """Sum of squares of (out - tgt) and the gradient of its mean over all
    output elements (the GPU's scaling of dL/dY3).  In the linear mode the
    biases and the feature inputs of layer 1 get zero gradients."""
    P = unpack(p)
    W2, W3 = _round(P["W2"], bf), _round(P["W3"], bf)
    x0r = _round(x0, bf)
    out, a1, a2 = forward(p, x0, bf, relu)
    d = out - tgt
    gscale = 2.0 / d.size
    g3 = _round(gscale * d, bf)
    g2 = _round(conv_t(g3, W3) * ((a2 > 0) if relu else 1.0), bf)
    g1 = _round(conv_t(g2, W2) * ((a1 > 0) if relu else 1.0), bf)
    G = {"W3": weight_grad(a2, g3), "b3": g3.sum(axis=(0, 1, 2, 3)),
         "W2": weight_grad(a1, g2), "b2": g2.sum(axis=(0, 1, 2, 3)),
         "W1": weight_grad(x0r, g1), "b1": g1.sum(axis=(0, 1, 2, 3))}
    if not relu:
        G["W1"][:, 8:, :] = 0.0
        for k in ("b1", "b2", "b3"):
            G[k] = 0.0 * G[k]
    return float((d * d).sum()), pack(G)


def apply(p, v, feat, relu=True):
    """The preconditioner on blocks: v [nBlock][8][512] (solver layout, cell
    = x + 8 y + 64 z), feat [nBlock][512][8]; z = s N(v / s, feat) with s the
    RMS of v over the block."""
    nb = v.shape[0]
    s = np.sqrt((v.reshape(nb, -1) ** 2).mean(axis=1))
    inv = np.where(s > 1e-300, 1.0 / np.where(s > 0, s, 1.0), 0.0)
    r = (v * inv[:, None, None]).astype(np.float32)        # [nb][8][512]
    f = feat.astype(np.float32) if relu else np.zeros_like(feat, dtype=np.float32)
    x0 = np.concatenate([r.transpose(0, 2, 1), f], axis=2)  # [nb][512][16]
    out, _, _ = forward(p, x0.reshape(nb, 8, 8, 8, 16), relu=relu)
    return s[:, None, None] * out.reshape(nb, 512, 8).transpose(0, 2, 1)


def init_params(seed=0, out_gain=0.1):
    rng = np.random.default_rng(seed)
    d = {}
    for name, shp in SHAPES:
        if name.startswith("W"):
            gain = out_gain if name == "W3" else 1.0
            d[name] = gain * np.sqrt(2.0 / (27 * shp[1])) * rng.normal(size=shp)
        else:
            d[name] = 0.1 * rng.normal(size=shp)
    return pack(d)
