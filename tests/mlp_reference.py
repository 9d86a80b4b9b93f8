"""CPU FP64 reference of the learned form's network (gradient checks).

Mirrors mapp_b200/csrc/mg_mlp.cu: parameter layout (W1 16x64, b1, W2 64x64, b2,
W3 64x64, b3, W4 64x8, b4; W stored [in][out]), input normalisation over the
training box, standardised MSE over 6 outputs, and the BF16 rounding the
tensor-core kernels apply to GEMM operands (weights, activations, output
gradients); accumulation and everything else in FP64.
"""
import numpy as np

H = 64
SIZES = [("W1", (16, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
         ("W4", (H, 8)), ("b4", (8,))]


def unpack(p):
    out, off = {}, 0
    for name, shp in SIZES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[off:off + n], dtype=np.float64).reshape(shp)
        off += n
    return out


def bf16(a):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = 0x7FFF + ((u >> 16) & 1)
    v = (((u + r) >> 16) << 16).astype(np.uint32)
    return v.view(np.float32).astype(np.float64)


# the network's activation silu_p: z times a degree-15 odd polynomial stand-in
# for the logistic function on z / 8, with u = min(x^2, 1) and the result
# clamped to [0, 1] (mapp_b200/csrc/mg_mlp_common.cuh; the same coefficients)
SIG_Q = np.array([1.981310478e+00, -9.368737072e+00, 3.989676019e+01, -1.137893481e+02,
                  2.023527075e+02, -2.133724498e+02, 1.215064055e+02, -2.870664878e+01])
SIG_Z = 8.0
# MG_MLP_ACT_SPLIT: the first SPLIT_TANH units of each hidden layer use the
# exact SiLU (the GPU's tanh.approx is within about 2^-11 of tanh)
SPLIT_TANH = 48


def sigma_p(z):
    x = np.asarray(z, dtype=np.float64) / SIG_Z
    u = np.minimum(x * x, 1.0)
    return np.clip(0.5 + x * np.polynomial.polynomial.polyval(u, SIG_Q), 0.0, 1.0)


def silu(z):
    return z * sigma_p(z)


def dsilu(z):
    z = np.asarray(z, dtype=np.float64)
    x = z / SIG_Z
    u = np.minimum(x * x, 1.0)
    q = np.polynomial.polynomial.polyval(u, SIG_Q)
    dq = np.polynomial.polynomial.polyval(u, SIG_Q[1:] * np.arange(1, len(SIG_Q)))
    su = 0.5 + x * q
    ds = np.where((np.abs(x) < 1.0) & (su > 0.0) & (su < 1.0), (q + 2.0 * u * dq) / SIG_Z, 0.0)
    return sigma_p(z) + z * ds


def silu_exact(z):
    return z / (1.0 + np.exp(-z))


def dsilu_exact(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def act(z, kind=0):
    """Activation of kind 0 (silu_p), 1 (SiLU) or 2 (split) on z[..., unit]."""
    if kind == 0:
        return silu(z)
    if kind == 1:
        return silu_exact(z)
    out = silu(z)
    out[..., :SPLIT_TANH] = silu_exact(z[..., :SPLIT_TANH])
    return out


def dact(z, kind=0):
    if kind == 0:
        return dsilu(z)
    if kind == 1:
        return dsilu_exact(z)
    out = dsilu(z)
    out[..., :SPLIT_TANH] = dsilu_exact(z[..., :SPLIT_TANH])
    return out


def inputs(x, box):
    r_lo, r_hi, w_lo, w_hi = box
    xin = np.zeros((x.shape[0], 16))
    xin[:, 0] = (x[:, 0] - 0.5 * (r_lo + r_hi)) / (0.5 * (r_hi - r_lo))
    xin[:, 1] = (x[:, 1] - 0.5 * (w_lo + w_hi)) / (0.5 * (w_hi - w_lo))
    xin[:, 2] = (x[:, 2] - 0.5 * (w_lo + w_hi)) / (0.5 * (w_hi - w_lo))
    xin[:, 3] = x[:, 3] - 1.0
    return bf16(np.asarray(xin, dtype=np.float32))


def forward(P, xin, kind=0):
    zs, hs = [], []
    a = xin
    for l, (W, b) in enumerate([("W1", "b1"), ("W2", "b2"), ("W3", "b3")]):
        z = a @ bf16(P[W]) + P[b]
        h = bf16(act(z, kind))
        zs.append(z)
        hs.append(h)
        a = h
    y = a @ bf16(P["W4"]) + P["b4"]
    return zs, hs, y


def loss_and_grad(p, x, y_phys, scaling, box, kind=0):
    P = unpack(p)
    mean, scale = np.asarray(scaling[:6], dtype=np.float64), np.asarray(scaling[6:], dtype=np.float64)
    t = (np.asarray(y_phys, dtype=np.float64) - mean) / scale
    xin = inputs(np.asarray(x, dtype=np.float64), box)
    zs, hs, y = forward(P, xin, kind)
    B = x.shape[0]
    diff = y[:, :6] - t
    loss = np.sum(diff * diff) / (B * 6)
    dy = np.zeros((B, 8))
    dy[:, :6] = 2.0 * diff / (B * 6)
    g = {}
    g["b4"] = dy.sum(0)
    dyb = bf16(dy)
    g["W4"] = hs[2].T @ dyb
    dz = (dyb @ bf16(P["W4"]).T) * dact(zs[2], kind)
    for l in (2, 1, 0):
        g["b%d" % (l + 1)] = dz.sum(0)
        dzb = bf16(dz)
        prev = hs[l - 1] if l > 0 else xin
        g["W%d" % (l + 1)] = prev.T @ dzb
        if l > 0:
            dz = (dzb @ bf16(P["W%d" % (l + 1)]).T) * dact(zs[l - 1], kind)
    flat = np.concatenate([g[name].ravel() for name, _ in SIZES])
    return loss, flat
