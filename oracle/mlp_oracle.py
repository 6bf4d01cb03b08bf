"""Float64 forward/backward of the warm-start MLP — TEST INFRASTRUCTURE.

The network is the one of avbd-metal_b200/csrc/learned.cu: 32 -> 128 -> 128
-> 128 -> 16 with ReLU, the first 6 outputs used, mean-squared-error loss on
targets normalised by (ymean, ystd).  With `rounded=True` the oracle rounds
exactly where the kernels store BF16 (normalised inputs, weights, hidden
activations and backward operands) and evaluates everything else in float64,
so the kernels' FP32-accumulated gradients can be compared tightly; with
`rounded=False` it is the plain float64 network (used to check the backward
formulas against finite differences).

Only tests/ may import this module.
"""
import numpy as np

DIN, HID, DOUT, USED = 32, 128, 16, 6
XM, XI, YM, YS = 0, 32, 64, 80          # offsets in the 96-float normalisation block
OW1 = 0
OB1 = OW1 + HID * DIN
OW2 = OB1 + HID
OB2 = OW2 + HID * HID
OW3 = OB2 + HID
OB3 = OW3 + HID * HID
OW4 = OB3 + HID
OB4 = OW4 + DOUT * HID
NPARAM = OB4 + DOUT


def bf16(x):
    """Round to bfloat16 (round to nearest even) through float32."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, np.float64)
    return (p[OW1:OB1].reshape(HID, DIN), p[OB1:OW2], p[OW2:OB2].reshape(HID, HID), p[OB2:OW3],
            p[OW3:OB3].reshape(HID, HID), p[OB3:OW4], p[OW4:OB4].reshape(DOUT, HID), p[OB4:NPARAM])


def forward_backward(params, norm, X, T, rounded=True):
    """Returns (loss, gradient) for features X [B][32] and targets T [B][6]."""
    R = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    F = f32 if rounded else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(params)
    norm = np.asarray(norm, np.float64)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    B = X.shape[0]
    W1b, W2b, W3b, W4b = R(W1), R(W2), R(W3), R(W4)
    Xb = R(F((X - norm[XM:XM + DIN]) * norm[XI:XI + DIN]))
    H1 = R(np.maximum(Xb @ W1b.T + b1, 0.0))
    H2 = R(np.maximum(H1 @ W2b.T + b2, 0.0))
    H3 = R(np.maximum(H2 @ W3b.T + b3, 0.0))
    Y = H3 @ W4b.T + b4
    t = (T - norm[YM:YM + USED]) / norm[YS:YS + USED]
    e = Y[:, :USED] - t
    loss = float(np.sum(e * e)) / B                     # mean over the batch
    dY = np.zeros((B, DOUT))
    dY[:, :USED] = 2.0 * e / B
    dY = F(dY)
    dYb = R(dY)
    g = np.zeros(NPARAM)
    g[OW4:OB4] = (dYb.T @ H3).ravel()
    g[OB4:NPARAM] = dY.sum(axis=0)
    dH3 = F((dYb @ W4b) * (H3 > 0))
    g[OB3:OW4] = dH3.sum(axis=0)
    dH3b = R(dH3)
    g[OW3:OB3] = (dH3b.T @ H2).ravel()
    dH2 = F((dH3b @ W3b) * (H2 > 0))
    g[OB2:OW3] = dH2.sum(axis=0)
    dH2b = R(dH2)
    g[OW2:OB2] = (dH2b.T @ H1).ravel()
    dH1 = F((dH2b @ W2b) * (H1 > 0))
    g[OB1:OW2] = dH1.sum(axis=0)
    dH1b = R(dH1)
    g[OW1:OB1] = (dH1b.T @ Xb).ravel()
    return loss, g


def predict(params, norm, X, rounded=True):
    """Denormalised outputs [B][6] of the network."""
    R = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    F = f32 if rounded else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(params)
    norm = np.asarray(norm, np.float64)
    Xb = R(F((np.asarray(X, np.float64) - norm[XM:XM + DIN]) * norm[XI:XI + DIN]))
    H1 = R(np.maximum(Xb @ R(W1).T + b1, 0.0))
    H2 = R(np.maximum(H1 @ R(W2).T + b2, 0.0))
    H3 = R(np.maximum(H2 @ R(W3).T + b3, 0.0))
    Y = H3 @ R(W4).T + b4
    return Y[:, :USED] * norm[YS:YS + USED] + norm[YM:YM + USED]
