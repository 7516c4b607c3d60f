"""The learned correction on the tensor cores (fe_corr_*) against its CPU restatement (oracle/net_cpu.py): forward,
loss and gradients; training on the GPU; the on-card guard; and, on FitzHugh-Nagumo, what the trained network gains over
the coarse plain method it corrects."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def law():
    return open(os.path.join(ROOT, "tests", "laws", "fhn_rk4.law")).read()


def tensors(*arrays):
    import torch
    return [torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda") for a in arrays]


def random_case(shape, seed):
    from fieldcuda.learned import init_weights
    rng = np.random.default_rng(seed)
    u = rng.normal(size=shape).astype(np.float32)
    v = rng.normal(size=shape).astype(np.float32)
    w = init_weights(seed, out_scale=0.2)
    w[-1280:] += (0.01 * rng.normal(size=1280)).astype(np.float32)
    from oracle import net_cpu
    w[net_cpu.pad_mask()] = 0.0
    return u, v, w


@pytest.mark.parametrize("shape", [(3, 32, 32), (2, 13, 20), (1, 1, 5)])
def test_forward_matches_the_oracle(cuda, shape):
    from fieldcuda.learned import Corrector
    from oracle import net_cpu
    u, v, w = random_case(shape, 1)
    c = Corrector(w)
    U, V = tensors(u, v)
    assert c.apply(U, V, -1e30, 1e30, time=0.75) is False
    want_u, want_v = net_cpu.apply(w, u, v, time=0.75)
    du_g, du_w = U.cpu().numpy() - u, want_u - u
    dv_g, dv_w = V.cpu().numpy() - v, want_v - v
    scale = max(np.abs(du_w).max(), np.abs(dv_w).max())
    assert scale > 1e-3
    assert np.abs(du_g - du_w).max() <= 2e-3 * scale and np.abs(dv_g - dv_w).max() <= 2e-3 * scale
    assert np.array_equal(c.weights(), w)
    c.close()


def test_loss_and_gradients_match_the_oracle(cuda):
    from fieldcuda.learned import Corrector
    from oracle import net_cpu
    shape = (4, 32, 32)
    u, v, w = random_case(shape, 2)
    rng = np.random.default_rng(9)
    tu = (u + 0.3 * rng.normal(size=shape)).astype(np.float32)
    tv = (v + 0.3 * rng.normal(size=shape)).astype(np.float32)
    c = Corrector(w)
    loss, g = c.grads(*tensors(u, v, tu, tv), time=1.5)
    want_loss, want_g = net_cpu.loss_and_grads(w, u, v, tu, tv, time=1.5)
    assert abs(loss - want_loss) <= 1e-5 * want_loss
    # BF16 operands, FP32 accumulation on both sides: the gradient as a whole to 1 %, its large entries to 3 %.
    assert np.linalg.norm(g - want_g) <= 1e-2 * np.linalg.norm(want_g)
    big = np.abs(want_g) > 0.1 * np.abs(want_g).max()
    assert np.all(np.abs(g[big] - want_g[big]) <= 3e-2 * np.abs(want_g[big]))
    assert np.all(g[net_cpu.pad_mask()] == 0.0)
    # Deterministic: the CTAs' partial sums are added in a fixed order.
    loss2, g2 = c.grads(*tensors(u, v, tu, tv), time=1.5)
    assert loss2 == loss and np.array_equal(g2.view(np.uint32), g.view(np.uint32))
    c.close()


def test_training_on_the_gpu_fits_a_smooth_correction(cuda):
    from fieldcuda.learned import Corrector, init_weights
    rng = np.random.default_rng(4)
    shape = (8, 32, 32)
    u = rng.normal(size=shape).astype(np.float32)
    v = rng.normal(size=shape).astype(np.float32)
    tu = (u + 0.1 * np.tanh(v) - 0.05 * u).astype(np.float32)
    tv = (v + 0.08 * np.tanh(u)).astype(np.float32)
    c = Corrector(init_weights(3))
    U, V, TU, TV = tensors(u, v, tu, tv)
    first = c.train_step(U, V, TU, TV, 3e-3, want_loss=True)
    for _ in range(400):
        c.train_step(U, V, TU, TV, 3e-3)
    last = c.train_step(U, V, TU, TV, 3e-3, want_loss=True)
    assert last < first / 20, (first, last)
    c.close()


def test_the_guard_keeps_the_plain_step_when_a_cell_leaves_the_range(cuda):
    from fieldcuda.learned import Corrector, pack
    rng = np.random.default_rng(5)
    shape = (2, 16, 16)
    u = rng.normal(size=shape).astype(np.float32)
    v = rng.normal(size=shape).astype(np.float32)
    z = np.zeros
    w = pack(z((18, 64)), z(64), z((64, 64)), z(64), z((64, 2)), np.array([50.0, 0.0]))
    c = Corrector(w)
    U, V = tensors(u, v)
    assert c.apply(U, V, -10.0, 10.0) is True
    assert np.array_equal(U.cpu().numpy(), u) and np.array_equal(V.cpu().numpy(), v)
    assert c.apply(U, V, -100.0, 100.0) is False
    assert np.allclose(U.cpu().numpy(), u + 50.0)
    c.close()


def test_trained_correction_beats_the_coarse_plain_method(cuda):
    """FitzHugh-Nagumo, fine 128 x 128 as the judge: the coarse 32 x 32 plain solve with the trained correction ends
    closer to the fine solution (averaged onto 32 x 32) than the coarse plain solve alone, on seeds it did not see."""
    from fieldcuda.learned import Corrector, PlainFHN, fine_frames, init_weights, train_correction
    text = law()
    frames = 20
    train = fine_frames(text, list(range(100, 124)), frames)
    test = fine_frames(text, list(range(900, 906)), frames)
    c = Corrector(init_weights(7))
    best, plain_train = train_correction(c, text, train, iters=600, rounds=1)
    assert best < plain_train

    def rollout(correct):
        s = PlainFHN(text, 32, 6)
        u, v = test[0]
        err = 0.0
        for t in range(frames):
            s.set(u, v)
            s.step()
            u, v = s.get()
            if correct:
                c.apply(u, v, -1000.0, 1000.0, time=(t + 1) * 0.05 * c.time_scale)
            tu, tv = test[t + 1]
            err += float(((u - tu) ** 2 + (v - tv) ** 2).mean())
        s.close()
        return (err / frames) ** 0.5

    plain, learned = rollout(False), rollout(True)
    c.close()
    assert learned < 0.8 * plain, (learned, plain)
