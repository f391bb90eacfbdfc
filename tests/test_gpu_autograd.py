"""The adjoint behind a torch.autograd.Function (test harness only).

``InterfaceLoss.apply(psi0, theta)`` runs ``steps`` loop bodies of the diffusive or advected
model from the initial field psi0 with parameters theta = (eps, alpha, beta, gamma, nu) and
returns the loss the library's adjoint differentiates: the mean sub-grid interface position
(bump tracker along x, in units of lambda0).  The forward calls ``smadft_adjoint`` once, which
computes the loss and all its gradients with checkpointed recomputation; ``backward`` hands
them to autograd scaled by the incoming gradient.  The product library is not written in
terms of torch: this wrapper lives here, in the tests, so that the gradients can be used and
checked inside ordinary autograd graphs.

Checked: backward returns exactly the ABI's gradients, the chain rule through torch ops
before and after the function, and agreement with central differences of the FP64 forward
(difference step 1e-6, as in the adjoint tests: the loss is piecewise smooth, each tracked
column interpolating inside one cell).
"""
import numpy as np
import pytest

import smadft

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

NAMES = ("eps", "alpha", "beta", "gamma", "nu")
TRACK = dict(axis=0, mode=smadft.TRACK_BUMP, hi=0.6, lo=0.1)
H = 1e-6


class InterfaceLoss(torch.autograd.Function):
    """loss(psi0, theta) of `steps` loop bodies; gradients from smadft_adjoint."""

    @staticmethod
    def forward(ctx, psi0, theta, model, shape, steps, checkpoint_every, dt, precision):
        kw = dict(zip(NAMES, (float(v) for v in theta.detach().cpu().tolist())))
        if model == smadft.NOADV:
            kw.pop("nu")
        p = smadft.params(model, shape, precision=precision, dt=dt, **kw)
        with smadft.Solver(p) as s:
            s.set_psi(psi0.detach().cpu().double().numpy())
            g = s.adjoint(steps, checkpoint_every=checkpoint_every, **TRACK)
        dpsi0 = torch.from_numpy(g["psi0"]).to(psi0.device, psi0.dtype)
        dtheta = torch.tensor([g[n] if n in g else 0.0 for n in NAMES], dtype=theta.dtype, device=theta.device)
        ctx.save_for_backward(dpsi0, dtheta)
        ctx.abi = g
        return torch.tensor(g["loss"], dtype=psi0.dtype, device=psi0.device)

    @staticmethod
    def backward(ctx, gout):
        dpsi0, dtheta = ctx.saved_tensors
        return gout * dpsi0, gout * dtheta, None, None, None, None, None, None


def loss_fd(model, shape, steps, dt, psi0, theta):
    kw = dict(zip(NAMES, theta))
    if model == smadft.NOADV:
        kw.pop("nu")
    p = smadft.params(model, shape, dt=dt, **kw)
    with smadft.Solver(p) as s:
        s.set_psi(psi0)
        s.step(steps)
        idx, pos = s.track(**TRACK)
    m = (idx >= 0) & np.isfinite(pos)
    return pos[m].mean() / p.nw


CASES = {
    "noadv": (smadft.NOADV, (32, 16, 24), 30, 8, 0.05),
    "adv": (smadft.ADV, (32, 16, 24), 20, 6, 0.02),
}


@pytest.mark.parametrize("which", list(CASES))
def test_autograd_backward_is_the_adjoint(which):
    model, shape, steps, K, dt = CASES[which]
    theta0 = np.array([-0.7, 1.0, 2.0, 1.0, 1.3])
    psi0_np = smadft.ic_interface(smadft.params(model, shape), A=1.328, bump=0.5 * 2 * np.pi, noise=1e-3,
                                  seed=41)
    psi0 = torch.tensor(psi0_np, dtype=torch.float64, requires_grad=True)
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)

    # chain rule through torch ops on both sides of the function
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    loss = InterfaceLoss.apply(psi0 * scale, theta, model, shape, steps, K, dt, smadft.FP64)
    out = 3.0 * loss + 0.5
    out.backward()

    with smadft.Solver(smadft.params(model, shape, dt=dt, **{k: v for k, v in zip(NAMES, theta0)
                                                                if model == smadft.ADV or k != "nu"})) as s:
        s.set_psi(psi0_np)
        g = s.adjoint(steps, checkpoint_every=K, **TRACK)
    assert abs(loss.item() - g["loss"]) == 0.0
    assert np.array_equal(psi0.grad.numpy(), 3.0 * g["psi0"])
    for i, n in enumerate(NAMES):
        want = 3.0 * (g[n] if model == smadft.ADV or n != "nu" else 0.0)
        assert theta.grad[i].item() == want, n
    # d out / d scale = 3 <dL/dpsi0, psi0>
    assert abs(scale.grad.item() - 3.0 * float(np.sum(g["psi0"] * psi0_np))) <= 1e-12 * abs(scale.grad.item())

    # central differences of the FP64 forward: eps and one direction in psi0
    jp = loss_fd(model, shape, steps, dt, psi0_np, theta0 + H * np.eye(5)[0])
    jm = loss_fd(model, shape, steps, dt, psi0_np, theta0 - H * np.eye(5)[0])
    fd = (jp - jm) / (2 * H)
    assert abs(theta.grad[0].item() / 3.0 - fd) <= 1e-4 * abs(fd) + 1e-8
    x = np.arange(shape[0])[:, None, None]
    z = np.arange(shape[2])[None, None, :]
    d = np.cos(0.3 * x) * np.cos(0.5 * z) * np.ones((1, shape[1], 1))
    jp = loss_fd(model, shape, steps, dt, psi0_np + H * d, theta0)
    jm = loss_fd(model, shape, steps, dt, psi0_np - H * d, theta0)
    fd = (jp - jm) / (2 * H)
    ad = float(torch.sum(psi0.grad * torch.from_numpy(d)).item()) / 3.0
    assert abs(ad - fd) <= 1e-4 * abs(fd) + 1e-8, (ad, fd)


def test_autograd_fp32_matches_fp64_through_the_function():
    """The FP32 adjoint through the function agrees with the FP64 one when both forwards
    track the same set of interface columns (the loss is piecewise smooth)."""
    model, shape, steps, K, dt = CASES["adv"]
    theta0 = torch.tensor([-0.7, 1.0, 2.0, 1.0, 1.3], dtype=torch.float64)
    psi0_np = smadft.ic_interface(smadft.params(model, shape), A=1.328, bump=0.5 * 2 * np.pi, noise=1e-3,
                                  seed=31)
    grads, found = {}, {}
    for prec in (smadft.FP64, smadft.FP32):
        psi0 = torch.tensor(psi0_np, dtype=torch.float64, requires_grad=True)
        theta = theta0.clone().requires_grad_(True)
        out = InterfaceLoss.apply(psi0, theta, model, shape, steps, K, dt, prec)
        out.backward()
        grads[prec] = (psi0.grad.clone(), theta.grad.clone())
        found[prec] = out.grad_fn.abi["found"]
    assert found[smadft.FP32] == found[smadft.FP64]
    (p64, t64), (p32, t32) = grads[smadft.FP64], grads[smadft.FP32]
    print("theta grad fp64", t64.tolist(), "fp32", t32.tolist())
    assert torch.all(torch.abs(t32 - t64) <= 1e-3 * torch.abs(t64) + 1e-7)
    assert (torch.linalg.norm(p32 - p64) / torch.linalg.norm(p64)).item() <= 1e-3
