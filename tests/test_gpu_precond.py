"""Learned preconditioner: the network's gradients through the tcgen05 conv kernels against
torch autograd, the L-BFGS recursion, and the learned-direction inversion with its plain
L-BFGS fallback.

The network test's reference is float64 torch on the CPU emulating the kernels' BF16
roundings (weights, inter-layer activations, the loss gradient); bound 3e-2 (max-norm
relative) for weight/bias gradients of every layer, 1e-2 for the output.
"""
import numpy as np
import pytest

from conftest import rel_err


def _bf(t):
    import torch
    return t.to(torch.bfloat16).to(t.dtype)


@pytest.mark.gpu
def test_network_gradients_match_torch(cuda):
    import torch
    from elastic_fm_vp_vs_rho_b200 import conv3d
    from elastic_fm_vp_vs_rho_b200.precond import PreconditionerNet, mse_grad
    net = PreconditionerNet(seed=3)
    for L in net.layers:
        L.b.normal_(0.0, 0.05)
    net.prep()
    g = torch.Generator().manual_seed(4)
    shape = (4, 5, 24)
    x = torch.randn(shape + (16,), generator=g).to(torch.bfloat16)
    tgt = torch.randn(shape + (3,), generator=g)
    out = net.forward(x.cuda(), keep=True)
    loss, d = mse_grad(out, tgt.cuda())
    grads = net.backward(d)
    conv3d.status()
    # float64 reference with the kernels' BF16 roundings (straight-through in the backward)
    ws = [conv3d.to_torch_weight(_bf(L.w.cpu())).double().requires_grad_(True) for L in net.layers]
    bs = [L.b.cpu().double().requires_grad_(True) for L in net.layers]
    h = x.permute(3, 0, 1, 2)[None].double()
    for i, L in enumerate(net.layers):
        z = torch.nn.functional.conv3d(h, ws[i], bs[i], padding=1)
        if L.relu:
            z = torch.relu(z)
            z = z + (_bf(z) - z).detach()
        h = z
    ref_out = h[0].permute(1, 2, 3, 0)
    diff = ref_out[..., :3] - tgt.double()
    (diff * diff).mean().backward()
    assert rel_err(out.cpu().numpy(), ref_out.detach().numpy()) < 1e-2
    for i in range(len(net.layers)):
        dw, db = grads[i]
        assert rel_err(dw.cpu().numpy(), conv3d.from_torch_weight(ws[i].grad).numpy()) < 3e-2, i
        assert rel_err(db.cpu().numpy(), bs[i].grad.numpy()) < 3e-2, i


@pytest.mark.gpu
def test_learned_inversion_with_fallback(cuda):
    from elastic_fm_vp_vs_rho_b200.precond import (InversionProblem, PreconditionerNet,
                                                   ProblemSpec, invert, train)
    spec = ProblemSpec(nx=32, ny=32, nz=28, lenpml=6, nt=200, nshots=2, nrec=6, seed=11)
    prob = InversionProblem(spec, illumination=True)
    samples = []
    plain = invert(prob, 3, record=samples)
    assert len(samples) == 3
    Js = [h["misfit"] for h in plain]
    assert all(b < a for a, b in zip(Js, Js[1:]))
    # every iteration: at least one Wolfe trial = one forward + one adjoint solve
    assert all(b["solves"] - a["solves"] >= 2 for a, b in zip(plain, plain[1:]))
    assert all(h["used"] == "lbfgs" for h in plain[1:])
    assert float(samples[0][0][..., 7].float().max()) == 1.0  # illumination channel filled
    net = PreconditionerNet(seed=0)
    losses = train(net, samples, epochs=6)
    assert losses[-1] < losses[0]
    learned = invert(prob, 3, net=net)
    Jl = [h["misfit"] for h in learned]
    assert all(b <= a for a, b in zip(Jl, Jl[1:]))
    assert all(h["used"] in ("learned", "fallback") for h in learned[1:])


@pytest.mark.gpu
def test_gpu_lbfgs_solves_a_quadratic(cuda):
    """The reference's two-loop recursion (GPU, float64 dots) with exact line minimisation
    converges on a convex quadratic."""
    import torch
    from elastic_fm_vp_vs_rho_b200.precond import GpuLBFGS
    rng = np.random.default_rng(0)
    n = 12
    Q = rng.standard_normal((n, n))
    A = torch.as_tensor(Q @ Q.T + n * np.eye(n), dtype=torch.float64)
    b = torch.as_tensor(rng.standard_normal(n), dtype=torch.float64)
    x = torch.zeros(n, dtype=torch.float64)
    lb = GpuLBFGS((n,), layers=n + 2)
    g = A @ x - b
    g0 = float(g.norm())
    for _ in range(2 * n):
        lb.push(x.float().cuda(), g.float().cuda())
        d = lb.direction(g.float().cuda()).double().cpu()
        a = -float(g @ d) / float(d @ A @ d)
        x = x + a * d
        g = A @ x - b
        if float(g.norm()) < 1e-5 * g0:
            break
    assert float(g.norm()) < 1e-4 * g0


def test_network_state_and_adam_on_cpu():
    import torch
    from elastic_fm_vp_vs_rho_b200.precond import PreconditionerNet, features, mse_grad
    net = PreconditionerNet(seed=1, device="cpu")
    assert [(L.cin, L.cout, L.relu) for L in net.layers] == [
        (16, 32, True), (32, 64, True), (64, 32, True), (32, 16, False)]
    sd = net.state_dict()
    other = PreconditionerNet(seed=2, device="cpu")
    other.load_state_dict(sd)
    assert all(torch.equal(a, b) for a, b in zip(net.parameters(), other.parameters()))
    w0 = net.layers[0].w.clone()
    grads = [(torch.ones_like(L.w), torch.ones_like(L.b)) for L in net.layers]
    net.adam_step(grads, lr=1e-3)
    # first Adam step moves every weight by ~lr against the gradient sign
    assert torch.allclose(net.layers[0].w, w0 - 1e-3, atol=1e-6)
    g3 = torch.randn(3, 2, 3, 4)
    p3 = 1.0 + 0.1 * torch.randn(3, 2, 3, 4)
    f = features(g3, p3)
    assert f.shape == (2, 3, 4, 16) and f.dtype == torch.bfloat16
    assert float(f[..., :3].float().abs().max()) <= 1.0
    assert float(f[..., 7].float().abs().max()) == 0.0  # no illumination given
    ill = torch.rand(2, 3, 4) * 1e-12 + 1e-16
    v = features(g3, p3, ill)[..., 7].float()
    assert float(v.min()) >= 0.0 and float(v.max()) == 1.0  # log-compressed, max -> 1
    out = torch.zeros(2, 3, 4, 16)
    loss, d = mse_grad(out, torch.ones(2, 3, 4, 3))
    assert abs(loss - 1.0) < 1e-12 and float(d[..., 3:].abs().max()) == 0.0


@pytest.mark.gpu
def test_learned_preconditioner_needs_fewer_solves(cuda):
    """Train on plain GPU L-BFGS runs of 12 seeded models (targets: the method's own accepted
    updates, summed to each run's last iterate), then, on four unseen seeds, the learned
    direction (first two iterations, Wolfe-tested, L-BFGS afterwards and as fallback) must
    reach plain L-BFGS's final misfit with fewer forward + adjoint solves in total, and on
    no seed with more."""
    from elastic_fm_vp_vs_rho_b200.precond import ProblemSpec, experiment
    spec = ProblemSpec(nx=48, ny=48, nz=40, nt=320, nshots=4, nrec=8)
    r = experiment(train_seeds=tuple(range(100, 112)), test_seeds=(7, 8, 9, 10), iters=10,
                   epochs=40, spec=spec, target="lbfgs", illumination=True,
                   policies={"first2": dict(learned_iters=2)})
    plain = [t["solves_plain"] for t in r["tests"]]
    learned = [t["policies"]["first2"]["solves"] for t in r["tests"]]
    assert all(s is not None for s in learned), learned  # every seed reached the target
    assert all(a <= b for a, b in zip(learned, plain)), (learned, plain)
    assert sum(learned) < sum(plain), (learned, plain)
