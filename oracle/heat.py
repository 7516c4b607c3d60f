"""The plain heat step d T = diffuse(k, T) (one k everywhere), restated on the CPU. Test infrastructure only.

Two restatements:

* :func:`cpu_step` — the reference's CPU solver (the oracle of record): ``Op::Diffuse`` in double per face with the
  harmonic face conductivity, stored as float (src/field/Law.cpp:986-1018), then the Euler store
  ``delta = float(value * sub_dt)``, ``T += delta`` in float (src/field/Solver.cpp:386-438).
* :func:`gpu_order_step` — the reference's generated CUDA arithmetic for the same term, all fp32, in its order
  (src/field/cuda/CudaCodegen.cpp:193-206 diffuse with a scalar k; :593-601 ping-pong store). numpy float32 operations
  round like IEEE fp32 without FMA, so this matches a correct kernel bit for bit.
"""
import numpy as np


def _faces(T):
    """(neighbour, valid-mask) per face in the order -x, +x, -y, +y, -z, +z; T is (nz, ny, nx)."""
    nz, ny, nx = T.shape
    out = []
    for axis, sign in ((2, -1), (2, 1), (1, -1), (1, 1), (0, -1), (0, 1)):
        nb = np.roll(T, -sign, axis=axis)
        idx = np.arange(T.shape[axis])
        valid_1d = (idx + sign >= 0) & (idx + sign < T.shape[axis])
        shape = [1, 1, 1]
        shape[axis] = T.shape[axis]
        out.append((nb, np.broadcast_to(valid_1d.reshape(shape), T.shape)))
    return out


def cpu_step(T, k, h, dt):
    """One step of the reference CPU solver on float32 T (nz, ny, nx). Law.cpp:986-1018, Solver.cpp:386-438."""
    T = np.asarray(T, dtype=np.float32)
    k = float(k)
    kf = 2.0 * k * k / (k + k) if (k + k) > 0.0 else 0.0  # Law.cpp:996-1000, in double
    v = T.astype(np.float64)
    acc = np.zeros(T.shape, dtype=np.float64)
    for nb, valid in _faces(v):
        acc += np.where(valid, kf * (nb - v), 0.0)
    rate = (acc / (h * h)).astype(np.float32)           # node.buffer[i] = float(acc / (h*h))
    delta = (rate.astype(np.float64) * dt).astype(np.float32)  # Solver.cpp: float(value * sub_dt)
    return (T + delta).astype(np.float32)               # target[i] += delta[i] (float)


def gpu_order_step(T, k, h, dt):
    """The generated kernel's fp32 arithmetic, in its order (CudaCodegen.cpp:193-206, :593-601)."""
    T = np.asarray(T, dtype=np.float32)
    f32 = np.float32
    acc = np.zeros(T.shape, dtype=np.float32)
    for nb, valid in _faces(T):
        acc = np.where(valid, (acc + (nb - T)).astype(f32), acc)
    kk = f32(max(float(f32(k)), 0.0))
    hh = f32(f32(h) * f32(h))
    rate = ((kk * acc).astype(f32) / hh).astype(f32)
    d = (rate * f32(dt)).astype(f32)
    return np.where(d != 0, (T + d).astype(f32), T).astype(f32)


def totals(T):
    """Sum and sum of |T| in double (the conserved-total contract's quantities, Solver.cpp:31-39)."""
    v = np.asarray(T, dtype=np.float64)
    return float(v.sum()), float(np.abs(v).sum())


def gaussian_blobs(n, h, seed, blobs=4, width=0.05):
    """The heat workload's initial state: a sum of `blobs` Gaussians A exp(-|x - c|^2 / (2 width^2)) at cell centres
    (i + 0.5) h, centres U[0.2, 0.8]^3, amplitudes U[0.5, 1], from numpy default_rng(seed). Width is read as sigma."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.2, 0.8, size=(blobs, 3))
    a = rng.uniform(0.5, 1.0, size=blobs)
    x = (np.arange(n) + 0.5) * h
    T = np.zeros((n, n, n), dtype=np.float64)
    for b in range(blobs):
        gx = np.exp(-((x - c[b, 0]) ** 2) / (2 * width * width))
        gy = np.exp(-((x - c[b, 1]) ** 2) / (2 * width * width))
        gz = np.exp(-((x - c[b, 2]) ** 2) / (2 * width * width))
        T += a[b] * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return T.astype(np.float32)
