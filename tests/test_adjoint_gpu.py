"""The hand-written adjoint of the FP64 leapfrog KDK (no counterpart in the reference) against
(1) gradients of an unrolled FP64 forward written in plain torch, (2) FP64 central finite
differences of the library's own forward, (3) itself at other checkpoint intervals.
Loss: mean over bodies of |x_T - x*|^2 (x* = forward final state + Gaussian offsets)."""
import numpy as np
import pytest

from gregpackagescpp_b200.ics import AU, plummer

pytestmark = pytest.mark.gpu
G = 6.674e-11
DT = 3600.0


def torch_kdk(x, v, m, steps):
    import torch

    def acc(x):
        d = x[None, :, :] - x[:, None, :]
        r2 = (d * d).sum(-1)
        eye = torch.eye(len(m), dtype=x.dtype, device=x.device)
        inv3 = (r2 + eye).pow(-1.5) * (1 - eye)
        return G * (d * (m[None, :] * inv3)[..., None]).sum(1)

    a = acc(x)
    for _ in range(steps):
        v = v + 0.5 * DT * a
        x = x + DT * v
        a = acc(x)
        v = v + 0.5 * DT * a
    return x, v


def setup(n, seed):
    import torch
    m, x, v = plummer(n, seed)
    dev = torch.device("cuda:0")
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
    return t(m), t(x), t(v)


# 48 bodies: one 256-body block (the symmetric VJP's diagonal form only); 700: three blocks, the
# last one padded, so the off-diagonal blocks' pairs are taken once for both of their bodies.
@pytest.mark.parametrize("n,steps", [(48, 40), (700, 12)])
def test_adjoint_vs_unrolled_torch_forward(gpu, n, steps):
    import torch

    from gregpackagescpp_b200.adjoint import leapfrog_final_state
    m, x, v = setup(n, 81)
    target = x + 0.01 * AU * torch.randn(x.shape, dtype=torch.float64, device=x.device,
                                         generator=torch.Generator(device="cuda").manual_seed(5))
    xa, va, ma = x.clone().requires_grad_(), v.clone().requires_grad_(), m.clone().requires_grad_()
    xT, vT = leapfrog_final_state(xa, va, ma, G, DT, steps, checkpoint_every=7)
    loss = ((xT - target) ** 2).sum(-1).mean()
    loss.backward()
    xb, vb, mb = x.clone().requires_grad_(), v.clone().requires_grad_(), m.clone().requires_grad_()
    xT2, _ = torch_kdk(xb, vb, mb, steps)
    assert torch.allclose(xT, xT2, rtol=1e-12, atol=0)
    loss2 = ((xT2 - target) ** 2).sum(-1).mean()
    loss2.backward()
    for ga, gb in ((xa.grad, xb.grad), (va.grad, vb.grad), (ma.grad, mb.grad)):
        rel = (ga - gb).abs().max() / gb.abs().max()
        assert rel < 1e-9, float(rel)


def test_adjoint_vs_central_differences(gpu):
    import torch

    from gregpackagescpp_b200.adjoint import leapfrog_final_state
    m, x, v = setup(128, 82)
    steps = 60
    target = x + 0.01 * AU * torch.randn(x.shape, dtype=torch.float64, device=x.device,
                                         generator=torch.Generator(device="cuda").manual_seed(6))

    def loss_of(xx, vv, mm):
        xT, _ = leapfrog_final_state(xx, vv, mm, G, DT, steps)
        return ((xT - target) ** 2).sum(-1).mean()

    xa, va, ma = x.clone().requires_grad_(), v.clone().requires_grad_(), m.clone().requires_grad_()
    loss_of(xa, va, ma).backward()
    rng = np.random.default_rng(7)
    checks = 0
    # h = 1e-6 relative for positions and velocities.  The mass derivatives are small next to the
    # FP64 loss, so their central differences are roundoff-bound: on this problem (checked with an
    # exact-autograd FP64 forward) the error relative to max|grad| is ~1e-7 at h = 1e-4 and ~5e-9 at
    # h = 1e-3, with the truncation error still below that; masses use 1e-3 relative.
    for which, base, grad, hrel in (("x", x, xa.grad, 1e-6), ("v", v, va.grad, 1e-6), ("m", m, ma.grad, 1e-3)):
        flat = base.reshape(-1)
        for idx in rng.choice(flat.numel(), 6, replace=False):
            hstep = hrel * abs(float(flat[idx]))
            args = [x, v, m]
            k = "xvm".index(which)
            plus, minus = [a.clone() for a in args], [a.clone() for a in args]
            plus[k].reshape(-1)[idx] += hstep
            minus[k].reshape(-1)[idx] -= hstep
            with torch.no_grad():
                fd = (float(loss_of(*plus)) - float(loss_of(*minus))) / (2 * hstep)
            g = float(grad.reshape(-1)[idx])
            assert abs(g - fd) <= 1e-5 * abs(fd) + 1e-7 * float(grad.abs().max()), (which, idx, g, fd)
            checks += 1
    assert checks == 18


@pytest.mark.parametrize("n", [64, 600])
def test_checkpoint_interval_invariance(gpu, n):
    import torch

    from gregpackagescpp_b200.adjoint import leapfrog_final_state
    m, x, v = setup(n, 83)
    target = x * 1.0001
    grads = []
    for every in (1, 5, 13, 50):
        xa, va, ma = x.clone().requires_grad_(), v.clone().requires_grad_(), m.clone().requires_grad_()
        xT, _ = leapfrog_final_state(xa, va, ma, G, DT, 50, checkpoint_every=every)
        ((xT - target) ** 2).sum(-1).mean().backward()
        grads.append((xa.grad.clone(), va.grad.clone(), ma.grad.clone()))
    for g in grads[1:]:
        for a, b in zip(g, grads[0]):
            assert torch.equal(a, b)
