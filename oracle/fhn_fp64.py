"""FP64 method-of-lines solve of the FitzHugh-Nagumo diffusion-reaction system (test infrastructure only).

The system of tests/laws/fhn_rk4.law and the reference's bench/laws/diff_react.law:18-35 on [-1, 1]^2, cell centred,
zero normal flux (the five-point Laplacian repeating the edge cell):
    u_t = Du lap u + u - u^3 - k - v        v_t = Dv lap v + u - v
discretised in space by that Laplacian and integrated in float64 by the classical fourth-order Runge-Kutta method at
the law's own step rule (max_dt = cfl h^2 / max(Du, Dv), each frame split evenly), as the reference's FP64 twin of the
benchmark does (bench/pdebench.py:46-68 uses a float64 method of lines). This restatement is the judge of the FP32
solves' error, not a thing measured.
"""
import math

import numpy as np

DU, DV, K, CFL = 1e-3, 5e-3, 5e-3, 0.15


def lap(a, h):
    up = np.concatenate([a[:, :1], a[:, :-1]], axis=1)
    dn = np.concatenate([a[:, 1:], a[:, -1:]], axis=1)
    lf = np.concatenate([a[:, :, :1], a[:, :, :-1]], axis=2)
    rt = np.concatenate([a[:, :, 1:], a[:, :, -1:]], axis=2)
    return (up + dn + lf + rt - 4.0 * a) / (h * h)


def rate(u, v, h):
    return DU * lap(u, h) + u - u ** 3 - K - v, DV * lap(v, h) + u - v


def solve(u0, v0, frames, frame=0.05):
    """(frames + 1, 2, nz, n, n) float64 states, frame 0 the start; u0, v0 of shape (nz, n, n)."""
    n = u0.shape[-1]
    h = 2.0 / n
    limit = CFL * h * h / max(DU, DV)
    sub = max(1, math.ceil(frame / limit))
    dt = frame / sub
    u = np.asarray(u0, np.float64).copy()
    v = np.asarray(v0, np.float64).copy()
    out = [np.stack([u, v])]
    for _ in range(frames):
        for _ in range(sub):
            a0, b0 = rate(u, v, h)
            a1, b1 = rate(u + 0.5 * dt * a0, v + 0.5 * dt * b0, h)
            a2, b2 = rate(u + 0.5 * dt * a1, v + 0.5 * dt * b1, h)
            a3, b3 = rate(u + dt * a2, v + dt * b2, h)
            u = u + dt * (a0 + 2 * a1 + 2 * a2 + a3) / 6
            v = v + dt * (b0 + 2 * b1 + 2 * b2 + b3) / 6
        out.append(np.stack([u, v]))
    return np.stack(out)
