"""CPU reference of the learned DME initializer (hw_b200/csrc/mlp.cu).

TEST INFRASTRUCTURE ONLY: used by tests/ to check the CUDA features, targets,
proposals, forward pass and gradients.  It rounds to BF16 at the same points
as the kernels (network input, both hidden activations, and every GEMM
operand including the backward ones) and accumulates in float64, so it
differs from the kernels only by FP32 accumulation order.  With
`bf16_round=False` it is the exact float64 network, which the finite-difference
test checks.
"""
import numpy as np

FEAT, HID, OUT, OUT_USED = 304, 256, 32, 19
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * FEAT
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
N_PARAMS = OFF_B3 + OUT
GELU_K0, GELU_K1 = 0.7978845608028654, 0.044715


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(params):
    p = np.asarray(params)
    p = p if p.dtype == np.float64 else p.astype(np.float32)
    return (p[OFF_W1:OFF_B1].reshape(HID, FEAT), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(OUT, HID), p[OFF_B3:])


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_K0 * (x + GELU_K1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_K0 * (x + GELU_K1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_K0 * (1.0 + 3.0 * GELU_K1 * x * x)


def forward(params, norm, feat, bf16_round=True):
    """Standardised outputs [n][32] and the cached activations."""
    r = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(params)
    in_mean, in_scale = norm[:FEAT], norm[FEAT:2 * FEAT]
    f = np.asarray(feat, np.float32)
    X = r(((f - in_mean) / in_scale).astype(np.float32)).astype(np.float64)
    Z1 = X @ r(W1).astype(np.float64).T + b1
    H1 = r(gelu(Z1).astype(np.float32) if bf16_round else gelu(Z1)).astype(np.float64)
    Z2 = H1 @ r(W2).astype(np.float64).T + b2
    H2 = r(gelu(Z2).astype(np.float32) if bf16_round else gelu(Z2)).astype(np.float64)
    Y = H2 @ r(W3).astype(np.float64).T + b3
    return Y, (X, Z1, H1, Z2, H2)


def loss_and_gradients(params, norm, feat, targets, bf16_round=True):
    """Mean squared error over the 19 used standardised outputs and its
    gradient in the parameter layout of the kernels."""
    r = bf16 if bf16_round else (lambda a: np.asarray(a, np.float64))
    rr = (lambda a: r(np.asarray(a, np.float32)).astype(np.float64)) if bf16_round else (lambda a: a)
    W1, b1, W2, b2, W3, b3 = unpack(params)
    out_mean, out_scale = norm[2 * FEAT:2 * FEAT + OUT], norm[2 * FEAT + OUT:]
    n = feat.shape[0]
    Y, (X, Z1, H1, Z2, H2) = forward(params, norm, feat, bf16_round)
    T = np.zeros((n, OUT))
    T[:, :OUT_USED] = ((np.asarray(targets, np.float32)[:, :OUT_USED] - out_mean[:OUT_USED])
                       / out_scale[:OUT_USED])
    D = np.zeros((n, OUT))
    D[:, :OUT_USED] = Y[:, :OUT_USED] - T[:, :OUT_USED]
    loss = float((D ** 2).sum() / (n * OUT_USED))
    dY = 2.0 * D / (n * OUT_USED)
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = (rr(dY).T @ H2).ravel()
    g[OFF_B3:] = dY.sum(0)
    dZ2 = (rr(dY) @ rr(W3)) * gelu_grad(Z2)
    g[OFF_W2:OFF_B2] = (rr(dZ2).T @ H1).ravel()
    g[OFF_B2:OFF_W3] = dZ2.sum(0)
    dZ1 = (rr(dZ2) @ rr(W2)) * gelu_grad(Z1)
    g[OFF_W1:OFF_B1] = (rr(dZ1).T @ X).ravel()
    g[OFF_B1:OFF_W2] = dZ1.sum(0)
    return loss, g


# ---- features, targets, proposals (FeaturesKernel, TargetsKernel, ProposalKernel)

def features(hist, stats):
    """[lanes * 64][304] float32 from LANE_HIST_DT / BLSTATS_DT records."""
    lanes = hist.shape[0]
    out = np.zeros((lanes, 64, FEAT), np.float32)
    for l in range(lanes):
        c = hist[l]["bin_count"].astype(np.float32)              # [300][64]
        total = np.zeros(64, np.float32)
        for b in range(300):
            total = (total + c[b]).astype(np.float32)
        inv = np.where(total > 0, np.float32(1) / np.maximum(total, np.float32(1)), np.float32(0)).astype(np.float32)
        out[l, :, :300] = np.sqrt((c * inv).astype(np.float32)).T
        lb, bs = hist[l]["low_bound"], hist[l]["bin_size"]
        s = stats[l]["baseline_stats"]
        m0, m1, m2 = s["moment0"], s["moment1"], s["moment2"]
        with np.errstate(all="ignore"):
            mean = np.where(m0 > 0, (m1 / m0 + s["offset"]).astype(np.float32), lb)
            var = np.where(m0 > 1, np.maximum((m2 - m1 * m1 / m0) / (m0 - 1), 0).astype(np.float32), bs * bs)
            fm = ((mean - lb) / bs).astype(np.float32)
            fv = (var / (bs * bs)).astype(np.float32)
        out[l, :, 300] = np.where(np.isfinite(fm), fm, 0)
        out[l, :, 301] = np.where(np.isfinite(fv), fv, 0)
    return out.reshape(lanes * 64, FEAT)


def targets(params, hist, shot_var_coeff):
    """[lanes * 64][32] float32 from fitted parameters [lanes][15][64]."""
    lanes = hist.shape[0]
    out = np.zeros((lanes, 64, OUT), np.float32)
    sv = np.float32(shot_var_coeff)
    for l in range(lanes):
        P = params[l]
        lb, bs = hist[l]["low_bound"], hist[l]["bin_size"]
        bs2 = (bs * bs).astype(np.float32)
        out[l, :, 0] = (P[5] - lb) / bs
        out[l, :, 1] = np.log(np.maximum(P[10], np.float32(1e-6)) / bs2)
        for a in range(4):
            out[l, :, 2 + a] = (P[6 + a] - lb) / bs
            out[l, :, 6 + a] = np.log(np.maximum(P[11 + a], np.float32(1e-6)) / bs2)
            m = P[6 + a]
            out[l, :, 15 + a] = ((P[11 + a] - P[10]) - sv * m) / np.maximum(m * m, np.float32(1e-6))
        out[l, :, 10:15] = P[0:5].T
    return out.reshape(lanes * 64, OUT)


def proposal(y, norm, hist):
    """EM start [lanes][15][64] from standardised outputs [lanes * 64][32]."""
    lanes = hist.shape[0]
    mean, scale = norm[2 * FEAT:2 * FEAT + OUT], norm[2 * FEAT + OUT:]
    o = (np.asarray(y, np.float32) * scale + mean).reshape(lanes, 64, OUT)
    P = np.zeros((lanes, 15, 64), np.float32)
    for l in range(lanes):
        lb, bs = hist[l]["low_bound"], hist[l]["bin_size"]
        r = np.maximum(o[l, :, 10:15], np.float32(0.001))
        P[l, 0:5] = (r / r.sum(1, keepdims=True)).T
        P[l, 5] = lb + o[l, :, 0] * bs
        P[l, 10] = bs * bs * np.maximum(np.exp(np.minimum(o[l, :, 1], 30)), np.float32(1e-3))
        for a in range(4):
            P[l, 6 + a] = lb + o[l, :, 2 + a] * bs
            P[l, 11 + a] = bs * bs * np.maximum(np.exp(np.minimum(o[l, :, 6 + a], 30)), np.float32(1e-3))
    return P
