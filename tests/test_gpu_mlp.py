"""The warm-start MLP's tensor-core kernels (gp5cu_gemm_bf16, gp5cu_mlp_*) against the NumPy
FP64 oracle (oracle/mlp_oracle.py)."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _bf16_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to("cuda").to(torch.bfloat16)


@pytest.mark.parametrize("M,N,K,ta,tb", [
    (128, 64, 64, False, False), (128, 256, 128, False, False), (200, 100, 70, False, True),
    (64, 3, 256, True, False), (1, 1, 1, False, False), (130, 300, 65, True, True),
    (512, 256, 256, False, False)])
def test_gemm_bf16_against_numpy(M, N, K, ta, tb):
    import torch
    from gp5_b200 import _abi
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = mo.bf16(rng.standard_normal((M, K)))
    B = mo.bf16(rng.standard_normal((N, K)))
    # storage: A(m, k) either row-major [M][K] or transposed [K][M]; likewise B
    Ad = _bf16_dev(A.T.copy() if ta else A)
    Bd = _bf16_dev(B.T.copy() if tb else B)
    sam, sak = (1, M) if ta else (K, 1)
    sbn, sbk = (1, N) if tb else (K, 1)
    Cd = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    _abi.gemm_bf16(Ad.data_ptr(), sam, sak, Bd.data_ptr(), sbn, sbk, Cd.data_ptr(), N, M, N, K)
    got = Cd.cpu().numpy().astype(np.float64)
    ref = A @ B.T
    bound = 2e-6 * (np.abs(A) @ np.abs(B).T) + 1e-30
    assert np.all(np.abs(got - ref) <= bound), np.max(np.abs(got - ref) / bound)


def _net_with(params):
    from gp5_b200 import _abi
    net = _abi.Mlp(seed=5)
    assert net.nparam == mo.num_params()
    net.set_params(params)
    return net


def test_forward_matches_oracle():
    p = mo.init_params(11)
    rng = np.random.default_rng(2)
    p[-64:] = rng.uniform(-0.1, 0.1, 64)  # non-zero output bias
    net = _net_with(p)
    x = rng.standard_normal((300, 3)).astype(np.float32)
    y = net.forward(x).astype(np.float64)
    yq, _ = mo.forward(p, x, quantize=True)
    y64, _ = mo.forward(p, x)
    assert np.max(np.abs(y - yq)) <= 2e-3 * np.max(np.abs(yq))
    assert np.max(np.abs(y - y64)) <= 3e-2 * np.max(np.abs(y64))
    assert np.array_equal(net.get_params(), p.astype(np.float32))


def test_gradients_match_oracle():
    p = mo.init_params(12)
    rng = np.random.default_rng(3)
    net = _net_with(p)
    x = rng.standard_normal((256, 3)).astype(np.float32)
    t = (0.5 * rng.standard_normal((256, 64))).astype(np.float32)
    g, loss = net.gradients(x, t)
    lq, gq = mo.loss_and_grad(p, x, t, quantize=True)
    l64, g64 = mo.loss_and_grad(p, x, t)
    assert abs(loss - lq) <= 1e-3 * lq
    off = 0
    for o, i in mo.SHAPES:
        for size in (o * i, o):
            a, b, c = g[off:off + size], gq[off:off + size], g64[off:off + size]
            assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b), (o, i, size)
            assert np.linalg.norm(a - c) <= 5e-2 * np.linalg.norm(c), (o, i, size)
            off += size


def test_adam_step_matches_oracle():
    p = mo.init_params(13)
    rng = np.random.default_rng(4)
    net = _net_with(p)
    x = rng.standard_normal((128, 3)).astype(np.float32)
    t = (0.5 * rng.standard_normal((128, 64))).astype(np.float32)
    g, _ = net.gradients(x, t)
    net.train(x, t, epochs=1, batch=128, lr=1e-3, seed=0)  # one step over the whole set
    got = net.get_params().astype(np.float64)
    ref, _, _ = mo.adam_step(p.astype(np.float32).astype(np.float64), g.astype(np.float64),
                             np.zeros_like(p), np.zeros_like(p), 1, 1e-3)
    # components whose gradient is comparable to FP32 summation-order noise may flip sign
    big = np.abs(g) > 1e-4 * np.max(np.abs(g))
    assert np.max(np.abs(got - ref)[big]) <= 2e-6
    assert np.max(np.abs(got - ref)) <= 2e-3 + 1e-6


def test_training_reduces_loss():
    from gp5_b200 import _abi
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (1024, 3)).astype(np.float32)
    w = rng.standard_normal((3, 64))
    t = np.tanh(x @ w).astype(np.float32)
    net = _abi.Mlp(seed=1)
    hist = net.train(x, t, epochs=60, batch=128, lr=1e-3, seed=2)
    assert hist.shape == (60,) and np.all(np.isfinite(hist))
    assert hist[-1] < 0.05 * hist[0]
    y = net.forward(x).astype(np.float64)
    assert np.mean((y - t) ** 2) < 0.05 * np.mean(t ** 2)


def test_gemm_wait_timeout_returns_timeout_status_and_net_stays_usable():
    """A per-chunk MMA wait bound of 0 makes the first wait run out (the MMAs cannot have
    finished at the first, non-blocking probe); the CTA drains its MMAs with the fixed 2 s
    bound, frees its tensor memory and flags the error.  The call returns GP5_ERR_TIMEOUT (not
    GP5_ERR_CUDA), and the next forward on the same handle, with the default bound, matches
    the oracle."""
    from gp5_b200 import _abi
    p = mo.init_params(21)
    net = _net_with(p)
    rng = np.random.default_rng(6)
    x = rng.standard_normal((256, 3)).astype(np.float32)
    net.set_wait_bound(0)
    with pytest.raises(_abi.Gp5Error) as ei:
        net.forward(x)
    assert ei.value.status == _abi.GP5_ERR_TIMEOUT
    assert b"bounded mbarrier wait ran out" in _abi.lib().gp5cu_last_error()
    net.set_wait_bound(_abi.GP5_GEMM_WAIT_DEFAULT_NS)
    for _ in range(2):
        y = net.forward(x).astype(np.float64)
        yq, _ = mo.forward(p, x, quantize=True)
        assert np.max(np.abs(y - yq)) <= 2e-3 * np.max(np.abs(yq))
