"""The proposal network: the float64 oracle's backward pass against finite
differences (CPU), and the BF16 tensor-core kernels' forward pass and
gradients against the oracle (GPU)."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO

N_PARAMS = 128 * 4 + 128 + 128 * 128 + 128 + 128 * 128 + 128 + 128 + 1


def _params(seed=3):
    rng = np.random.default_rng(seed)
    d = {"W1": rng.uniform(-1.2, 1.2, (128, 4)), "b1": rng.normal(0, 0.1, 128),
         "W2": rng.uniform(-0.2, 0.2, (128, 128)), "b2": rng.normal(0, 0.1, 128),
         "W3": rng.uniform(-0.2, 0.2, (128, 128)), "b3": rng.normal(0, 0.1, 128),
         "w4": rng.uniform(-0.2, 0.2, 128), "b4": np.array([0.3])}
    return MO.flat(d).astype(np.float32).astype(np.float64)


def _data(n, seed=5):
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t = np.sin(3 * q[:, 0]) + q[:, 1] * q[:, 2] - 0.5 * q[:, 3] ** 2
    return q.astype(np.float32), t.astype(np.float32)


def test_oracle_gradient_matches_finite_differences():
    p = _params()
    q, t = _data(37)
    _, g = MO.loss_grad(p, q.astype(np.float64), t.astype(np.float64))
    rng = np.random.default_rng(11)
    idx = np.concatenate([rng.choice(np.arange(0, 512), 4), rng.choice(np.arange(640, 17024), 6),
                          rng.choice(np.arange(17152, 33536), 6), [33600, 33792, 520]])
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = MO.loss_grad(pp, q.astype(np.float64), t.astype(np.float64))
        lm, _ = MO.loss_grad(pm, q.astype(np.float64), t.astype(np.float64))
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), i


def _blocks(v):
    o = 0
    for name, n in (("W1", 512), ("b1", 128), ("W2", 16384), ("b2", 128), ("W3", 16384),
                    ("b3", 128), ("w4", 128), ("b4", 1)):
        yield name, v[o:o + n]
        o += n


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 63, 200, 1000])
def test_gpu_forward_and_gradients_match_oracle(n):
    from mbs_fast_b200.mlp import ProposalNet
    net = ProposalNet(seed=1)
    p = _params()
    net.params = p
    q, t = _data(n)
    y = net.forward(q)
    y_bf, _ = MO.forward(p, q, bf16_round=True)
    y64, _ = MO.forward(p, q, bf16_round=False)
    scale = max(1.0, np.max(np.abs(y64)))
    assert np.max(np.abs(y - y_bf)) <= 2e-3 * scale        # same BF16 rounding points
    assert np.max(np.abs(y - y64)) <= 3e-2 * scale         # BF16 against exact float64
    loss, g = net.loss_grad(q, t)
    loss_bf, g_bf = MO.loss_grad(p, q, t, bf16_round=True)
    _, g64 = MO.loss_grad(p, q, t, bf16_round=False)
    assert abs(loss - loss_bf) <= 2e-3 * max(loss_bf, 1e-3)
    for (name, a), (_, b), (_, c) in zip(_blocks(g), _blocks(g_bf), _blocks(g64)):
        nb = np.linalg.norm(b)
        assert np.linalg.norm(a - b) <= 1e-2 * nb + 1e-7, name
        assert np.linalg.norm(a - c) <= 6e-2 * np.linalg.norm(c) + 1e-7, name
    net.close()


@pytest.mark.gpu
def test_gpu_training_reduces_loss_and_is_repeatable():
    from mbs_fast_b200.mlp import ProposalNet
    q, t = _data(2048)
    losses, outs = [], []
    for _ in range(2):
        net = ProposalNet(seed=2)
        l0, _ = net.loss_grad(q, t)
        l1 = net.train(q, t, epochs=60, batch=256, lr=2e-3, seed=9)
        losses.append((l0, l1))
        outs.append(net.forward(q[:64]))
        net.close()
    assert losses[0][1] < 0.05 * losses[0][0]
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_gemm_barrier_watchdog_reports_and_recovers():
    """The tensor-core GEMMs' bounded barrier wait: with the test hook the
    MMAs and their commit are left out, so the barrier never completes and
    the wait runs out after a short poll limit.  The call must fail with the
    timeout error instead of returning output, and the network must stay
    usable afterwards (its tensor memory freed, the flag cleared): the next
    normal call returns bitwise the result of the call before."""
    from mbs_fast_b200.mlp import ProposalNet
    net = ProposalNet(seed=3)
    q, _ = _data(300)
    y0 = net.forward(q)
    net.set_watchdog(poll_limit=64, skip_mma=True)
    with pytest.raises(RuntimeError, match="timed out"):
        net.forward(q)
    with pytest.raises(RuntimeError, match="timed out"):
        net.loss_grad(q, np.zeros(len(q), np.float32))
    net.set_watchdog(0, False)
    np.testing.assert_array_equal(net.forward(q), y0)
    net.close()
