"""The learned correction's CPU restatement (oracle/net_cpu.py) and host pieces: the backward against finite
differences of the exact (unrounded) math, bfloat16 rounding against torch's, the weight packing and padding."""
import numpy as np
import pytest


@pytest.fixture
def exact(monkeypatch):
    from oracle import net_cpu
    monkeypatch.setattr(net_cpu, "ROUND", False)
    return net_cpu


def test_bf16_rounding_is_round_to_nearest_even():
    import torch
    from oracle import net_cpu
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=2000).astype(np.float32) * 10.0 ** rng.integers(-20, 20, 2000),
                        np.float32([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38])])
    want = torch.tensor(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(net_cpu.bf16(x).view(np.uint32), want.view(np.uint32))


def test_backward_matches_central_differences(exact):
    from fieldcuda.learned import init_weights
    rng = np.random.default_rng(3)
    shape = (2, 6, 7)
    u, v = rng.normal(size=shape), rng.normal(size=shape)
    tu, tv = u + 0.1 * rng.normal(size=shape), v + 0.1 * rng.normal(size=shape)
    w = init_weights(5, out_scale=0.3).astype(np.float64)
    w += 0.05 * rng.normal(size=w.size) * ~exact.pad_mask()
    loss, g = exact.loss_and_grads(w, u, v, tu, tv)
    idx = rng.choice(np.flatnonzero(~exact.pad_mask()), 40, replace=False)
    for i in idx:
        e = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[i] += e
        wm[i] -= e
        fd = (exact.loss_and_grads(wp, u, v, tu, tv)[0] - exact.loss_and_grads(wm, u, v, tu, tv)[0]) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
    assert np.all(g[exact.pad_mask()] == 0.0)


def test_pack_places_biases_on_the_constant_rows():
    from fieldcuda.learned import pack
    from oracle import net_cpu
    rng = np.random.default_rng(1)
    W1, b1 = rng.normal(size=(18, 64)), rng.normal(size=64)
    W2, b2 = rng.normal(size=(64, 64)), rng.normal(size=64)
    W3, b3 = rng.normal(size=(64, 2)), rng.normal(size=2)
    w = pack(W1, b1, W2, b2, W3, b3)
    m1, m2, m3 = net_cpu.unpack(w)
    assert np.allclose(m1[18], b1) and np.allclose(m2[64], b2) and np.allclose(m3[64, :2], b3)
    assert np.all(w[net_cpu.pad_mask()] == 0.0)
    # A network whose hidden layers pass their inputs through (identity blocks) applies W3's rows to them.
    u = rng.normal(size=(1, 4, 5)).astype(np.float32)
    v = rng.normal(size=(1, 4, 5)).astype(np.float32)
    y, _ = net_cpu.forward(w, u, v)
    assert y.shape == (20, 2) and np.all(np.isfinite(y))
