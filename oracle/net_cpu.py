"""CPU restatement of the learned correction's forward and backward (test infrastructure only: the checker of
online-physics-cuda_b200/csrc/corrector.cu, never on a product path).

The network and its operands follow the kernel's definition: per cell the 3 x 3 neighbourhood of (u, v), edge
repeating, as 18 inputs plus a constant 1 (bias) and the time, -> 64 ReLU (+ constant 1) -> 64 ReLU (+ constant 1) -> 2, the output
added to (u, v) at the cell. Every matrix operand is rounded to bfloat16 (round to nearest even) where the kernel stores
it in shared memory — the inputs, the weights, the hidden activations, dY and the dZs — and every product is
accumulated in float64 here (the tensor cores accumulate in FP32, so the two agree to FP32 rounding of the sums).
Loss = 1/2 mean over cells of the squared error; gradients are of that loss. There is no reference counterpart for
this network (the reference's nets are fp16 face-flux MLPs, src/field/nn/Net.cpp:132-243): the restatement is of the
math the kernel implements, checked against finite differences in the tests.
"""
import numpy as np

W1_SHAPE, W2_SHAPE, W3_SHAPE = (32, 64), (80, 64), (80, 16)
SIZES = (32 * 64, 80 * 64, 80 * 16)
# False: no bfloat16 rounding anywhere (the exact math, for checking the backward against finite differences).
ROUND = True


def bf16(x):
    """Rounds float32 values to the nearest bfloat16 (ties to even), returned as float32 (identity when ROUND is off)."""
    if not ROUND:
        return np.asarray(x, np.float64)
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    rounding = ((b >> 16) & 1) + 0x7FFF
    out = ((b + rounding) >> 16) << 16
    nan = np.isnan(a)
    res = out.astype(np.uint32).view(np.float32).reshape(a.shape)
    return np.where(nan, a, res)


def unpack(w):
    w = np.asarray(w, np.float32 if ROUND else np.float64)
    o1, o2 = SIZES[0], SIZES[0] + SIZES[1]
    return w[:o1].reshape(W1_SHAPE), w[o1:o2].reshape(W2_SHAPE), w[o2:].reshape(W3_SHAPE)


def features(u, v, time=0.0):
    """(cells, 32): the 3 x 3 neighbourhood of (u, v) per cell, (dy, dx) row by row as (u, v) pairs, the constant 1 at 18,
    the time at 19."""
    nz, ny, nx = u.shape
    feats = np.zeros((nz, ny, nx, 32), np.float32 if ROUND else np.float64)
    ys, xs = np.arange(ny), np.arange(nx)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            yy = np.clip(ys + dy, 0, ny - 1)
            xx = np.clip(xs + dx, 0, nx - 1)
            k = 2 * (3 * (dy + 1) + (dx + 1))
            feats[..., k] = u[:, yy][:, :, xx]
            feats[..., k + 1] = v[:, yy][:, :, xx]
    feats[..., 18] = 1.0
    feats[..., 19] = time
    return feats.reshape(-1, 32)


def forward(w, u, v, time=0.0):
    """The corrections (cells, 2) and the intermediates the backward needs."""
    W1, W2, W3 = (np.asarray(bf16(m), np.float64) for m in unpack(w))
    X0 = np.asarray(bf16(features(u, v, time)), np.float64)
    f = np.float32 if ROUND else np.float64
    Z1 = (X0 @ W1).astype(f)
    H1 = np.zeros((X0.shape[0], 80), np.float64)
    H1[:, :64] = bf16(np.maximum(Z1, 0.0))
    H1[:, 64] = 1.0
    Z2 = (H1 @ W2).astype(f)
    H2 = np.zeros((X0.shape[0], 80), np.float64)
    H2[:, :64] = bf16(np.maximum(Z2, 0.0))
    H2[:, 64] = 1.0
    Y = (H2 @ W3).astype(f)
    return Y[:, :2], dict(X0=X0, Z1=Z1, H1=H1, Z2=Z2, H2=H2, W1=W1, W2=W2, W3=W3)


def apply(w, u, v, time=0.0):
    y, _ = forward(w, u, v, time)
    shape = u.shape
    return (u.reshape(-1) + y[:, 0]).reshape(shape), (v.reshape(-1) + y[:, 1]).reshape(shape)


def loss_and_grads(w, u, v, tu, tv, time=0.0):
    """(loss, flat gradient of 8448 floats) of 1/2 mean squared error of (u, v) + correction against (tu, tv)."""
    y, c = forward(w, u, v, time)
    n = y.shape[0]
    f = np.float32 if ROUND else np.float64
    pu = u.reshape(-1).astype(f) + y[:, 0]
    pv = v.reshape(-1).astype(f) + y[:, 1]
    eu = (pu - tu.reshape(-1)).astype(f)
    ev = (pv - tv.reshape(-1)).astype(f)
    loss = 0.5 * float(np.sum(eu.astype(np.float64) ** 2 + ev.astype(np.float64) ** 2)) / n
    dY = np.zeros((n, 16), np.float64)
    dY[:, 0] = bf16(eu)
    dY[:, 1] = bf16(ev)
    dH2 = (dY @ c["W3"].T).astype(f)
    dZ2 = np.asarray(bf16(np.where(c["Z2"] > 0, dH2[:, :64], 0.0)), np.float64)
    dH1 = (dZ2 @ c["W2"].T).astype(f)
    dZ1 = np.asarray(bf16(np.where(c["Z1"] > 0, dH1[:, :64], 0.0)), np.float64)
    dW3 = c["H2"].T @ dY
    dW2 = c["H1"].T @ dZ2
    dW1 = c["X0"].T @ dZ1
    g = np.concatenate([dW1.reshape(-1), dW2.reshape(-1), dW3.reshape(-1)]) / n
    mask = pad_mask()
    return loss, np.where(mask, 0.0, g)


def pad_mask():
    """True where a weight is padding that stays zero (W1 inputs past 19; W2, W3 inputs past 64; W3 outputs past 1)."""
    m1 = np.zeros(W1_SHAPE, bool)
    m1[20:] = True
    m2 = np.zeros(W2_SHAPE, bool)
    m2[65:] = True
    m3 = np.zeros(W3_SHAPE, bool)
    m3[65:] = True
    m3[:, 2:] = True
    return np.concatenate([m1.reshape(-1), m2.reshape(-1), m3.reshape(-1)])
