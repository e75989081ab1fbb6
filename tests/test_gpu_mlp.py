"""The learned scorer's CUDA kernels against the torch FP64 restatement:
forward outputs, training-loss gradients, and that Adam steps reduce the loss."""
import numpy as np
import pytest

from mlp_reference import NUM, OFF, forward, loss_and_grad

pytestmark = pytest.mark.gpu

# FP32 accumulation against FP64, on BF16-rounded operands; a hidden activation
# whose FP32 and FP64 values round to different BF16 neighbours moves a few
# gradient entries by one BF16 step, so the check is on relative norms.
OUT_ATOL = 2e-3
GRAD_RTOL = 2e-2


@pytest.fixture(scope="module")
def ctx():
    from remobench_b200 import synth
    from remobench_b200.lod import Context
    cfg = synth.config(1, num_points=65536, batch_size=65536)
    bmin, bmax = synth.scene_box(cfg)
    c = Context(slot_capacity=65536)
    c.allocate(65536, bmin, bmax)
    c.mlp_init(123)
    return c


def data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 2.0, size=(n, 16)).astype(np.float32)
    t = np.stack([rng.uniform(0, 1, n), (rng.uniform(0, 1, n) > 0.5)], 1).astype(np.float32)
    return x, t


def test_forward_matches_reference(ctx):
    import torch
    x, _ = data(3000, 1)
    y = torch.empty((len(x), 2), dtype=torch.float32, device="cuda")
    ctx.mlp_predict(torch.from_numpy(x).cuda(), y)
    ref = forward(ctx.mlp_params(), x).numpy()
    assert np.max(np.abs(y.cpu().numpy() - ref)) <= OUT_ATOL


def test_gradients_match_reference(ctx):
    import torch
    x, t = data(2048, 2)
    g, loss = ctx.mlp_gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    rloss, rg = loss_and_grad(ctx.mlp_params(), x, t)
    assert abs(loss - rloss) <= 1e-3 * max(1.0, abs(rloss))
    for name, lo, hi in [("W1", OFF["W1"], OFF["b1"]), ("b1", OFF["b1"], OFF["W2"]), ("W2", OFF["W2"], OFF["b2"]),
                         ("b2", OFF["b2"], OFF["W3"]), ("W3", OFF["W3"], OFF["b3"]), ("b3", OFF["b3"], NUM)]:
        a, b = g[lo:hi], rg[lo:hi]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel <= GRAD_RTOL, (name, rel)


def test_adam_reduces_loss():
    import torch
    from remobench_b200 import synth
    from remobench_b200.lod import Context
    cfg = synth.config(1, num_points=65536, batch_size=65536)
    bmin, bmax = synth.scene_box(cfg)
    c = Context(slot_capacity=65536)
    c.allocate(65536, bmin, bmax)
    c.mlp_init(7)
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, size=(8192, 16)).astype(np.float32)
    t0 = 3.0 * (0.5 * x[:, 0] * x[:, 1] + 0.3 * np.sin(3 * x[:, 2]) ** 2) / 0.8 * 0.3
    t1 = (x[:, 3] + x[:, 4] > 1.0).astype(np.float32)
    t = np.stack([t0, t1], 1).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = c.mlp_train_step(xd[:1024], td[:1024], 3e-3, want_loss=True)
    for step in range(400):
        k = (step * 1024) % 8192
        c.mlp_train_step(xd[k:k + 1024], td[k:k + 1024], 3e-3)
    _, last = c.mlp_gradients(xd, td)
    assert last < 0.5 * first, (first, last)
