"""CPU checks of the warm-start network's oracle (oracle/mlp_oracle.py): its analytic
gradients against central finite differences, its bf16 rounding, GELU and Adam against
PyTorch's CPU implementations, and its parameter layout against the C ABI."""
import numpy as np
import pytest

import mlp_oracle as M


def _problem(rows=6, in_dim=8, out_dim=2, hidden=16, seed=0):
    rng = np.random.default_rng(seed)
    n = hidden * in_dim + hidden + hidden * hidden + hidden + out_dim * hidden + out_dim
    params = rng.normal(0, 0.4, n)
    X = rng.normal(0, 1, (rows, in_dim))
    T = rng.normal(0, 1, (rows, out_dim))
    return params, X, T


@pytest.mark.parametrize("out_dim", [1, 2, 3])
def test_gradients_match_finite_differences(out_dim):
    hidden, in_dim = 16, 8
    params, X, T = _problem(out_dim=out_dim, hidden=hidden, in_dim=in_dim)
    _, g, _ = M.forward_backward(params, X, T, in_dim, out_dim, bf16=False, hidden=hidden)
    rng = np.random.default_rng(1)
    idx = rng.choice(params.size, 60, replace=False)
    # every parameter block is represented
    idx = np.concatenate([idx, [0, hidden * in_dim, hidden * in_dim + hidden, params.size - out_dim - 1,
                                params.size - 1]])
    eps = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        fd = (M.loss_only(p1, X, T, in_dim, out_dim, hidden) - M.loss_only(p2, X, T, in_dim, out_dim, hidden)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-3, 1000), rng.normal(0, 1e4, 1000)]).astype(np.float32)
    x = np.concatenate([x, np.float32([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -1 - 2 ** -8, 0.0, -0.0])])
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(M.bf16_round(x).view(np.uint32), ref.view(np.uint32))
    assert M.bf16_round(np.float32([1 + 2 ** -8]))[0] == 1.0  # tie to even
    assert M.bf16_round(np.float32([1 + 3 * 2 ** -8]))[0] == np.float32(1 + 2 ** -6)


def test_gelu_matches_torch_exact_gelu():
    torch = pytest.importorskip("torch")
    x = np.linspace(-8, 8, 2001)
    ref = torch.nn.functional.gelu(torch.from_numpy(x), approximate="none").numpy()
    assert np.allclose(M.gelu(x), ref, rtol=1e-12, atol=1e-14)
    t = torch.from_numpy(x).requires_grad_(True)
    torch.nn.functional.gelu(t, approximate="none").sum().backward()
    assert np.allclose(M.gelu_grad(x), t.grad.numpy(), rtol=1e-10, atol=1e-12)


def test_adam_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    w0 = rng.normal(0, 1, 500).astype(np.float32)
    grads = [rng.normal(0, s, 500).astype(np.float32) for s in (1.0, 0.1, 3.0)]
    p = torch.nn.Parameter(torch.from_numpy(w0.copy()))
    opt = torch.optim.Adam([p], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    w, m, v = w0.copy(), np.zeros_like(w0), np.zeros_like(w0)
    for t, g in enumerate(grads, start=1):
        p.grad = torch.from_numpy(g.copy())
        opt.step()
        w, m, v = M.adam_step(w, m, v, g, t, 1e-3)
        assert np.allclose(w, p.detach().numpy(), rtol=0, atol=1e-6)


def test_bf16_path_close_to_exact_path():
    params, X, T = _problem(rows=64, in_dim=64, hidden=256, seed=4)
    params = params * 0.1
    l1, g1, y1 = M.forward_backward(params, X, T, 64, 2, bf16=True)
    l2, g2, y2 = M.forward_backward(params, X, T, 64, 2, bf16=False)
    assert abs(l1 - l2) <= 0.02 * l2
    assert np.linalg.norm(g1 - g2) <= 0.05 * np.linalg.norm(g2)


def test_param_layout_matches_abi(ub):
    for i, o in ((64, 2), (128, 3), (64, 1)):
        assert ub.warm_start.param_count(i, o) == M.pack(M.unpack(np.zeros(ub.warm_start.param_count(i, o)), i, o)).size
        assert ub.mlp_init_params(i, o).size == ub.warm_start.param_count(i, o)
    with pytest.raises(ub.UmapError):
        ub.warm_start.param_count(64, 9)
