"""The warm-start MLP: the FP64 oracle against finite differences (CPU), and the
GPU forward/backward kernels (tensor-core GEMMs on split BF16 operands, FP32
accumulation) against the oracle (GPU, called through the C ABI).

Tolerances: the GPU splits GEMM operands into two bfloat16 values exactly as the
oracle's split mode does, so the remaining differences are FP32 accumulation
order and tanh in FP32: relative 1e-4 on gradients and outputs against the
split-mode oracle, 1e-3 against plain FP64 (single bfloat16 operands, the
oracle's bf16 mode, are ~1e-2 from FP64)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M

WIDTHS = [6, 256, 256, 256, 64]


def _data(n=200, seed=0, widths=WIDTHS):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, widths[0]))
    t = np.tanh(x @ rng.standard_normal((widths[0], widths[-1]))) * 0.5
    return x.astype(np.float32), t.astype(np.float32)


def _params(widths, seed=1):
    rng = np.random.default_rng(seed)
    Ws = [rng.uniform(-1, 1, (o, i)) * np.sqrt(6.0 / (i + o)) for i, o in zip(widths[:-1], widths[1:])]
    bs = [rng.standard_normal(o) * 0.05 for o in widths[1:]]
    return M.pack(Ws, bs).astype(np.float32)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, -3.14159, 0.0, 1.0 + 3 * 2 ** -8], dtype=np.float32)
    r = M.to_bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                 # halfway between 1 and 1 + 2^-7: ties to the even mantissa
    assert r[2] == 1.0
    assert r[5] == 1.0 + 2 ** -6       # halfway between 1 + 2^-7 and 1 + 2^-6: ties to even
    assert abs(r[3] + 3.140625) < 1e-12
    assert r[4] == 0.0


def test_split_operands_carry_16_bits():
    """hi + lo reconstructs a float32 value within 2^-16 of it, and split products bring the oracle's
    gradients an order of magnitude or more closer to FP64 than single bfloat16 operands."""
    rng = np.random.default_rng(7)
    v = (rng.standard_normal(10000) * np.exp(rng.uniform(-8, 8, 10000))).astype(np.float32)
    hi, lo = M.split_bf16(v)
    assert np.all(np.abs(hi + lo - v) <= 2.0 ** -16 * np.abs(v))
    assert np.all(M.to_bf16(hi) == hi) and np.all(M.to_bf16(lo) == lo)
    x, t = _data(64)
    p = _params(WIDTHS).astype(np.float64)
    _, g64 = M.loss_and_grads(p, WIDTHS, x, t)
    _, gs = M.loss_and_grads(p, WIDTHS, x, t, arith="split")
    _, gb = M.loss_and_grads(p, WIDTHS, x, t, arith="bf16")
    es, eb = (np.linalg.norm(g - g64) / np.linalg.norm(g64) for g in (gs, gb))
    assert es < 1e-3 and es < eb / 10, (es, eb)


def test_oracle_gradients_match_finite_differences():
    widths = [3, 8, 8, 4]
    x, t = _data(7, seed=3, widths=widths)
    p = _params(widths).astype(np.float64)
    _, g = M.loss_and_grads(p, widths, x, t)
    rng = np.random.default_rng(0)
    for k in rng.choice(p.size, 25, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-6
        num = (M.loss_and_grads(p + e, widths, x, t)[0] - M.loss_and_grads(p - e, widths, x, t)[0]) / 2e-6
        assert num == pytest.approx(g[k], rel=1e-5, abs=1e-9)


@pytest.mark.gpu
def test_gpu_forward_and_gradients_match_oracle():
    from bec_b200.engine import MLP
    x, t = _data(200)
    p = _params(WIDTHS)
    net = MLP(WIDTHS, seed=0)
    net.set_params(p)
    np.testing.assert_array_equal(net.get_params(), p)
    y = net.forward(x)
    y_o = M.forward(p, WIDTHS, x, arith="split")[-1]
    y64 = M.forward(p, WIDTHS, x)[-1]
    loss, g = net.gradients(x, t)
    loss_o, g_o = M.loss_and_grads(p, WIDTHS, x, t, arith="split")
    _, g64 = M.loss_and_grads(p, WIDTHS, x, t)
    from parity_util import record
    record("mlp_grad", out_err_split=np.abs(y - y_o).max() / np.abs(y_o).max(),
           rel_err_split=np.linalg.norm(g - g_o) / np.linalg.norm(g_o),
           out_err_fp64=np.abs(y - y64).max() / np.abs(y64).max(),
           rel_err_fp64=np.linalg.norm(g - g64) / np.linalg.norm(g64))
    assert np.abs(y - y_o).max() < 1e-4 * np.abs(y_o).max()
    assert loss == pytest.approx(loss_o, rel=1e-4)
    assert np.linalg.norm(g - g_o) < 1e-4 * np.linalg.norm(g_o)
    assert np.abs(y - y64).max() < 1e-3 * np.abs(y64).max()
    assert np.linalg.norm(g - g64) < 1e-3 * np.linalg.norm(g64)


@pytest.mark.gpu
@pytest.mark.parametrize("widths,batch", [([5, 70, 130, 3], 100), ([6, 256, 64], 64), ([3, 40, 40, 40, 1], 320)])
def test_gpu_split_gemm_padded_shapes_match_oracle(widths, batch):
    """Widths that are not multiples of 64 (zero-padded on the device) and batches whose last row tile is 64
    rows (the GEMM's zero-filled A rows): outputs and gradients against the split-mode oracle."""
    from bec_b200.engine import MLP
    x, t = _data(batch, seed=11, widths=widths)
    p = _params(widths, seed=4)
    net = MLP(widths, seed=0)
    net.set_params(p)
    y = net.forward(x)
    y_o = M.forward(p, widths, x, arith="split")[-1]
    assert y.shape == y_o.shape
    assert np.abs(y - y_o).max() < 1e-4 * np.abs(y_o).max()
    loss, g = net.gradients(x, t)
    loss_o, g_o = M.loss_and_grads(p, widths, x, t, arith="split")
    assert loss == pytest.approx(loss_o, rel=1e-4)
    assert np.linalg.norm(g - g_o) < 1e-4 * np.linalg.norm(g_o)


@pytest.mark.gpu
def test_gpu_training_reduces_loss():
    from bec_b200.engine import MLP
    x, t = _data(1024, seed=5)
    net = MLP(WIDTHS, seed=3)
    hist = net.train(x, t, steps=400, batch=128, lr=1e-3, seed=1)
    assert np.isfinite(hist).all()
    assert hist[-20:].mean() < 0.1 * hist[:5].mean()
    loss, _ = net.gradients(x, t)
    assert loss < 0.1 * hist[:5].mean()


@pytest.mark.gpu
def test_gemm_wait_that_runs_out_is_reported(monkeypatch):
    """A tensor-core GEMM whose wait runs out (its first K group also waits for a flag that nothing sets, with a
    20 ms limit) ends with BEC_ERR_CUDA after its MMAs have finished and its tensor memory is freed; the device
    stays usable and the next call computes the same bits as a fresh network."""
    from bec_b200._abi import BEC_ERR_CUDA
    from bec_b200.engine import MLP, BecError
    x, _ = _data(100)
    p = _params(WIDTHS)
    monkeypatch.setenv("BEC_STEP_WAIT_LIMIT_MS", "20")
    monkeypatch.setenv("BEC_GEMM_INJECT_STALL", "1")
    net = MLP(WIDTHS, seed=0)
    net.set_params(p)
    with pytest.raises(BecError) as ei:
        net.forward(x)
    assert ei.value.status == BEC_ERR_CUDA
    monkeypatch.delenv("BEC_GEMM_INJECT_STALL")
    monkeypatch.delenv("BEC_STEP_WAIT_LIMIT_MS")
    y = net.forward(x)
    fresh = MLP(WIDTHS, seed=0)
    fresh.set_params(p)
    np.testing.assert_array_equal(y, fresh.forward(x))
