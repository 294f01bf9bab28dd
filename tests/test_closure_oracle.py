"""Pins the closure oracle (oracle/closure_oracle.c) on the CPU: its forward pass and gradient
against torch autograd in float64 of the same network, with the BF16 roundings placed at the same
points (straight-through: rounded in value, identity in the derivative)."""
import numpy as np
import pytest
import torch

import oracle as O

NP = 8899
OFF = dict(W1=0, b1=320, W2=384, b2=4480, W3=4544, b3=8640, W4=8704, b4=8896)
SHAPES = dict(W1=(64, 5), b1=(64,), W2=(64, 64), b2=(64,), W3=(64, 64), b3=(64,), W4=(3, 64), b4=(3,))


def bf16_np(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_st(t):
    r = torch.from_numpy(bf16_np(t.detach().numpy().astype(np.float32)).astype(np.float64))
    return t + (r - t).detach()


def torch_loss(P, x, t):
    p = {k: P[OFF[k]:OFF[k] + int(np.prod(SHAPES[k]))].reshape(SHAPES[k]) for k in OFF}
    q = {k: (bf16_st(v) if k.startswith("W") else v) for k, v in p.items()}
    gelu = lambda a: 0.5 * a * (1.0 + torch.erf(a / np.sqrt(2.0)))
    h = bf16_st(x)
    for l in (1, 2, 3):
        h = bf16_st(gelu(h @ q[f"W{l}"].T + q[f"b{l}"]))
    y = h @ q["W4"].T + q["b4"]
    return ((y - t) ** 2).sum(1).mean(), y


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(7)
    P = np.zeros(NP, np.float32)
    for k, off in OFF.items():
        n = int(np.prod(SHAPES[k]))
        fan = SHAPES[k][1] if k.startswith("W") else (5 if k == "b1" else 64)
        P[off:off + n] = rng.uniform(-1, 1, n) / np.sqrt(fan)
    x = rng.standard_normal((257, 5)).astype(np.float32)
    t = (0.5 * rng.standard_normal((257, 3))).astype(np.float32)
    return P, x, t


def test_nparam_layout():
    assert O.closure_nparam() == NP


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.01171875, -3.14159, 65504.0, 1e-30], np.float32)
    ref = bf16_np(vals)
    got = np.array([O.lib().orc_bf16(float(v)) for v in vals], np.float32)
    assert np.array_equal(got, ref)
    # ties go to even: 1 + 2^-8 lies halfway between 1 and 1 + 2^-7
    assert O.lib().orc_bf16(1.00390625) == 1.0


def test_forward_matches_torch(case):
    P, x, t = case
    y = O.closure_forward(P, x)
    _, yt = torch_loss(torch.from_numpy(P.astype(np.float64)), torch.from_numpy(x.astype(np.float64)),
                       torch.from_numpy(t.astype(np.float64)))
    yt = yt.detach().numpy()
    assert np.linalg.norm(y - yt) / np.linalg.norm(yt) < 1e-3


def test_gradient_matches_torch_autograd(case):
    P, x, t = case
    g, loss = O.closure_grad(P, x, t)
    Pt = torch.from_numpy(P.astype(np.float64)).requires_grad_(True)
    lt, _ = torch_loss(Pt, torch.from_numpy(x.astype(np.float64)), torch.from_numpy(t.astype(np.float64)))
    lt.backward()
    gt = Pt.grad.numpy()
    assert abs(loss - lt.item()) / lt.item() < 1e-4
    for k, off in OFF.items():
        n = int(np.prod(SHAPES[k]))
        a, b = g[off:off + n], gt[off:off + n]
        # the oracle also rounds dy and dz to BF16 (the tensor cores' operands)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 2e-2, k


def test_adamw_step_matches_formula(case):
    P, x, t = case
    g, _ = O.closure_grad(P, x, t)
    p = P.copy()
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    O.closure_adamw(p, m, v, g.astype(np.float32), 1, 1e-2, 0.9, 0.999, 1e-8, 0.1)
    gf = g.astype(np.float32)
    is_w = np.ones(NP, bool)
    for k in ("b1", "b2", "b3", "b4"):
        is_w[OFF[k]:OFF[k] + SHAPES[k][0]] = False
    mh = (0.1 * gf) / (1 - 0.9)
    vh = (0.001 * gf * gf) / (1 - 0.999)
    ref = np.where(is_w, P - 1e-2 * 0.1 * P, P) - 1e-2 * mh / (np.sqrt(vh) + 1e-8)
    np.testing.assert_allclose(p, ref, rtol=1e-5, atol=1e-7)
