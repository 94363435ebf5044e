"""Learned preconditioner for the Vp/Vs/rho inversion (no counterpart in the reference).

The reference preconditions its gradients with a Gaussian filter and margin masks
(mainPropElastic3D_MT.py:2479-2504) and takes L-BFGS steps (lbfgs.py:27-67) after two
fixed-length steps.  Here a small 3-D convolutional network maps the current gradient and
model to a model update:

    features (16 channels, channels-last BF16 volume):
        0-2  gradient of the misfit w.r.t. (Vp, Vs, rho) in normalised units, each scaled
             by its largest magnitude
        3-5  the normalised model (value / mean - 1)
        6    depth z / nz (geometric spreading falls with depth)
        7    with illumination=True: forward illumination of the current model, sum over
             shots and steps of |v|^2 (efm_forward_illumination), as
             log10(I / max I + 1e-4) / 4 + 1 in [0, 1] -- the diagonal a pseudo-Hessian
             preconditioner would divide by; zero otherwise
    network: conv3d 16->32, ReLU, 32->64, ReLU, 64->32, ReLU, 32->16 (3x3x3, zero padding;
             BF16 tcgen05 kernels of efm_conv.cu with FP32 accumulation)
    output:  channels 0-2 = the update direction for (Vp, Vs, rho) in normalised units.

Training pairs come from plain L-BFGS runs on seeded random models: the features of each
iterate (raw gradient, model, depth, forward illumination) and, as target, one of

* "lbfgs" (default): GAIN x (p_N - p_k), the sum of the accepted L-BFGS updates the plain
  run itself takes from iterate k to its last iterate N, in normalised units -- where the
  method ends up, learned from its own accepted steps;
* "update": the single accepted L-BFGS update of iteration k scaled to unit maximum;
* "error": GAIN x (true - current) normalised model (the seeded problems know their true
  model; an upper bound of what a preconditioner could learn, not available in practice);

the loss is the mean squared error over the three used channels; Adam on FP32 master
weights.

:func:`invert` runs an inversion with either plain L-BFGS (the reference's two-loop
recursion and history layout, ``lbfgs.compute_sk_yk`` / ``lbfgs.L_BFGS`` on the GPU with
float64 dot products) or the learned direction.  Every step passes a Wolfe line search
(sufficient decrease and curvature, each trial a misfit + gradient evaluation); a learned
direction that fails it within ``learned_tries`` trials falls back to the plain L-BFGS
direction for that iteration.  Solves are counted as in the reference's loop: a misfit +
gradient evaluation costs one forward and one adjoint solve.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import conv3d

WIDTHS = (16, 32, 64, 32, 16)
NFEAT = 8
GAIN = 10.0  # "error" / "lbfgs" targets: network output = GAIN x (normalised displacement)


# ================================================================================ network
class ConvLayer:
    def __init__(self, cin, cout, relu, gen, device="cuda"):
        import torch
        std = math.sqrt((2.0 if relu else 1.0) / (27 * cin))
        self.cin, self.cout, self.relu = cin, cout, relu
        self.w = (torch.randn((27, cout, cin), generator=gen) * std).to(device)
        self.b = torch.zeros(cout, device=device)
        self.wb = self.wt = None

    def prep(self):
        self.wb, self.wt = conv3d.prep_weights(self.w)


class PreconditionerNet:
    """4 conv layers (16-64 channels) on the tcgen05 conv3d kernels, with Adam."""

    def __init__(self, widths=WIDTHS, seed=0, device="cuda", target="error"):
        import torch
        gen = torch.Generator().manual_seed(seed)
        self.target = target  # what the output predicts: "error" or "update" (see invert)
        n = len(widths) - 1
        self.layers = [ConvLayer(widths[i], widths[i + 1], i < n - 1, gen, device)
                       for i in range(n)]
        self.ws = conv3d.WgradWorkspace()
        self._acts = None
        self._adam = None
        self.steps = 0
        if device == "cuda":
            self.prep()

    def prep(self):
        for L in self.layers:
            L.prep()

    def parameters(self):
        out = []
        for L in self.layers:
            out += [L.w, L.b]
        return out

    def forward(self, x, keep=False):
        """x: (ny, nz, nx, 16) BF16 -> (ny, nz, nx, 16) FP32."""
        acts = [x]
        h = x
        for i, L in enumerate(self.layers):
            last = i == len(self.layers) - 1
            yb, yf = conv3d.forward(h, L.wb, L.b, relu=L.relu, out_bf16=not last, out_f32=last)
            h = yf if last else yb
            acts.append(h)
        if keep:
            self._acts = acts
        return h

    def backward(self, dy):
        """dy: dLoss/dOutput (ny, nz, nx, 16) FP32 -> [(dw, db)] per layer (needs forward(keep=True))."""
        import torch
        acts = self._acts
        g = dy.to(torch.bfloat16).contiguous()
        grads = [None] * len(self.layers)
        for i in reversed(range(len(self.layers))):
            L = self.layers[i]
            grads[i] = conv3d.backward_weights(acts[i], g, self.ws)
            if i > 0:
                # input of layer i = ReLU output of layer i-1: its mask gates the data gradient
                g = conv3d.backward_data(g, L.wt, L.cin, relu_mask=acts[i])
        return grads

    def adam_step(self, grads, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        import torch
        params = self.parameters()
        flat = []
        for dw, db in grads:
            flat += [dw, db]
        if self._adam is None:
            self._adam = [(torch.zeros_like(p), torch.zeros_like(p)) for p in params]
        self.steps += 1
        c1 = 1.0 - beta1 ** self.steps
        c2 = 1.0 - beta2 ** self.steps
        for p, g, (m, v) in zip(params, flat, self._adam):
            m.mul_(beta1).add_(g, alpha=1.0 - beta1)
            v.mul_(beta2).addcmul_(g, g, value=1.0 - beta2)
            p.addcdiv_(m / c1, (v / c2).sqrt_().add_(eps), value=-lr)
        if params[0].is_cuda:
            self.prep()

    def state_dict(self):
        return {f"w{i}": L.w.detach().cpu().numpy() for i, L in enumerate(self.layers)} | \
               {f"b{i}": L.b.detach().cpu().numpy() for i, L in enumerate(self.layers)}

    def load_state_dict(self, sd):
        import torch
        for i, L in enumerate(self.layers):
            L.w = torch.as_tensor(sd[f"w{i}"]).to(L.w.device)
            L.b = torch.as_tensor(sd[f"b{i}"]).to(L.b.device)
        if self.layers[0].w.is_cuda:
            self.prep()


def features(g3, p3, illum=None):
    """(3, ny, nz, nx) gradient and normalised model (and the (ny, nz, nx) forward
    illumination, channel 7 stays zero without it) -> (ny, nz, nx, 16) BF16 features."""
    import torch
    _, ny, nz, nx = g3.shape
    f = torch.zeros((ny, nz, nx, WIDTHS[0]), dtype=torch.float32, device=g3.device)
    for c in range(3):
        s = g3[c].abs().max().clamp_min(1e-30)
        f[..., c] = g3[c] / s
        f[..., 3 + c] = p3[c] - 1.0
    f[..., 6] = (torch.arange(nz, device=g3.device, dtype=torch.float32) / nz)[None, :, None]
    if illum is not None:
        rel = illum.float() / illum.max().clamp_min(1e-30)
        f[..., 7] = torch.log10(rel + 1e-4) / 4.0 + 1.0
    return f.to(torch.bfloat16).contiguous()


def mse_grad(out, target):
    """Loss and dLoss/dout for the mean squared error over channels 0-2."""
    import torch
    d = torch.zeros_like(out)
    diff = out[..., :3] - target
    n = diff.numel()
    d[..., :3] = diff * (2.0 / n)
    return float((diff * diff).sum() / n), d


def train(net, samples, epochs=30, lr=2e-3, seed=0, log=None):
    """samples: list of (features BF16 volume, target (ny, nz, nx, 3) FP32).  Returns the
    mean loss of each epoch."""
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        tot = 0.0
        for k in rng.permutation(len(samples)):
            x, t = samples[k]
            out = net.forward(x, keep=True)
            loss, d = mse_grad(out, t)
            net.adam_step(net.backward(d), lr=lr)
            tot += loss
        hist.append(tot / max(1, len(samples)))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    conv3d.status()
    return hist


# ============================================================================= inversion
@dataclasses.dataclass
class ProblemSpec:
    nx: int = 48
    ny: int = 48
    nz: int = 40
    dx: float = 10.0
    lenpml: int = 8
    fq: float = 12.0
    nt: int = 320
    nshots: int = 4
    nrec: int = 8
    seed: int = 0
    smooth_m: float = 150.0


class InversionProblem:
    """Seeded true / initial model, earthquake-style MT sources at depth and surface
    receivers; misfit and exact gradient evaluations through one ShotBatch."""

    def __init__(self, spec: ProblemSpec, illumination=False):
        import torch
        from . import configs
        from .engine import ShotBatch
        s = self.spec = spec
        self.use_illum = illumination
        self.illum = None  # forward illumination at the model of the last gradient call
        rng = np.random.default_rng(spec.seed)
        vp, vs, rho = configs.layered_anomaly_model(s.ny, s.nz, s.nx, s.dx, spec.seed,
                                                    n_layers=4, n_anomalies=3, sigma_m=60.0,
                                                    vpvs=1.8)
        vp0, vs0, rho0 = configs.smooth_model(vp, vs, rho, s.smooth_m / s.dx)
        self.dt = configs.cfl_dt(s.dx, float(max(vp.max(), vp0.max())))
        self.w = torch.as_tensor(configs.ricker(s.fq, self.dt, s.nt)).cuda()
        self.cp = configs.cpml_profiles(s.fq, self.dt, s.dx, s.lenpml, float(max(vp.max(), vp0.max())),
                                        s.nx, s.ny, s.nz)
        rx, ry, rz = configs.surface_receivers(s.nx, s.ny, s.lenpml, s.nrec, s.nrec)
        self.rec = np.stack([rx, ry, rz], axis=1)
        lo = s.lenpml + 4
        self.srcs = []
        for _ in range(s.nshots):
            self.srcs.append(([int(rng.integers(lo, s.nx - lo)), int(rng.integers(lo, s.ny - lo)),
                               int(rng.integers(s.nz // 2, s.nz - lo))],
                              configs.random_moment_tensor(rng)))
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()  # noqa: E731
        self.true = torch.stack([dev(vp), dev(vs), dev(rho)])
        self.init = torch.stack([dev(vp0), dev(vs0), dev(rho0)])
        self.scale = self.init.mean(dim=(1, 2, 3)).reshape(3, 1, 1, 1)
        self.batch = ShotBatch()
        lam, mu = self._lame(self.true)
        for src, mt in self.srcs:
            self.batch.add(nx=s.nx, ny=s.ny, nz=s.nz, lenpml=s.lenpml, dx=s.dx, dt=self.dt,
                           nt=s.nt, cpml=self.cp, lam=lam, mu=mu, rho=self.true[2], wavelet=self.w,
                           src=[src], mt=[mt], rec=self.rec)
        self.obs = self.batch.forward().clone()
        self.solves = 0

    @staticmethod
    def _lame(m):
        vp, vs, rho = m[0], m[1], m[2]
        mu = (vs * vs * rho).contiguous()
        lam = (vp * vp * rho - 2.0 * mu).contiguous()
        return lam, mu

    def _set(self, m):
        lam, mu = self._lame(m)
        rho = m[2].contiguous()
        for i in range(len(self.srcs)):
            self.batch.set_model(i, lam, mu, rho)

    def misfit(self, p):
        """Misfit of the normalised model p (one forward solve)."""
        self._set(p * self.scale)
        mod = self.batch.forward()
        _, mis = self.batch.residual_misfit(mod, self.obs)
        self.solves += 1
        return float(mis.sum())

    def gradient(self, p):
        """(misfit, dJ/dp) for the normalised model p (forward + adjoint solve); the exact
        gradient, smoothed (sigma 1 cell) and masked at the absorbing frame like the
        reference's post-processing."""
        import torch
        from .engine import chain_rule, smooth_mask
        m = p * self.scale
        self._set(m)
        ill = (torch.zeros(self.batch.illum_size, dtype=torch.float32, device="cuda")
               if self.use_illum else None)
        mod = self.batch.forward(checkpoints=True, illum=ill)
        res, mis = self.batch.residual_misfit(mod, self.obs)
        g, _ = self.batch.gradient(res, exact=True)
        self.solves += 2
        s = self.spec
        if ill is not None:
            self.illum = ill.view(len(self.srcs), s.ny, s.nz, s.nx).sum(dim=0)
        n = s.nx * s.ny * s.nz
        gv = g.reshape(len(self.srcs), 3, s.ny, s.nz, s.nx).sum(dim=0).contiguous()
        gl, gm, gr = gv[0].contiguous(), gv[1].contiguous(), gv[2].contiguous()
        chain_rule(gl, gm, gr, m[0].contiguous(), m[1].contiguous(), m[2].contiguous())
        out = torch.stack([gl, gm, gr])
        tmp = torch.empty_like(out[0])
        for c in range(3):
            smooth_mask(out[c], 1.0, s.lenpml, 2, tmp)
        out *= self.scale  # dJ/dp = dJ/dm * scale
        assert out.numel() == 3 * n
        return float(mis.sum()), out

    def model_error(self, p):
        return float(((p * self.scale - self.true) / self.true).pow(2).mean().sqrt())


def _dot(a, b):
    """float64 dot product on the GPU (efm_dot), as a host float."""
    from .engine import dot
    return float(dot(a.contiguous().reshape(-1), b.contiguous().reshape(-1)))


class GpuLBFGS:
    """Plain L-BFGS: the reference's history layout and two-loop recursion
    (lbfgs.compute_sk_yk / lbfgs.L_BFGS, lbfgs.py:12-67) on the GPU, float64 dot products,
    scalars on the device.  ``layers`` = lbfgsLayers (layers - 2 curvature pairs)."""

    def __init__(self, shape, layers=7, device="cuda"):
        import torch
        self.L = int(layers)
        self.sk = torch.zeros((self.L,) + tuple(shape), dtype=torch.float32, device=device)
        self.yk = torch.zeros_like(self.sk)
        self.work = torch.empty(4 * self.L + 8, dtype=torch.float64, device=device)
        self.k = -1  # pushes - 1: curvature pairs held (capped at layers - 2 by the recursion)

    def reset(self):
        self.sk.zero_()
        self.yk.zero_()
        self.k = -1

    def push(self, p, g):
        """compute_sk_yk with the current model and gradient."""
        from .lbfgs import compute_sk_yk
        self.k += 1
        compute_sk_yk(self.sk, self.yk, p.contiguous(), g.contiguous(), self.L, self.k)

    @property
    def has_pairs(self):
        return self.k >= 1

    def direction(self, g):
        """-H g from the held pairs, or -g without any."""
        from .lbfgs import L_BFGS
        if not self.has_pairs:
            return -g
        return -L_BFGS(self.sk, self.yk, g.contiguous(), self.L, self.k, work=self.work)


def _wolfe(prob, p, J, g, d, a0, tries=6, c1=1e-4, c2=0.9):
    """Wolfe line search along d from p (misfit J, gradient g): sufficient decrease
    J(a) <= J + c1 a g.d and curvature g(a).d >= c2 g.d, bracketing by halving / doubling.
    Every trial is a misfit + gradient evaluation (2 solves).  Returns (a, J(a), g(a)), the
    last trial that passed sufficient decrease when none passed both, or None."""
    gd = _dot(g, d)
    if not gd < 0:
        return None
    lo, hi, a = 0.0, math.inf, a0
    best = None
    for _ in range(tries):
        Jn, gn = prob.gradient(p + a * d)
        if not math.isfinite(Jn) or Jn > J + c1 * a * gd:
            hi = a
            a = 0.5 * (lo + hi)
        elif _dot(gn, d) < c2 * gd:
            best = (a, Jn, gn)
            lo = a
            a = 2.0 * a if math.isinf(hi) else 0.5 * (lo + hi)
        else:
            return a, Jn, gn
    return best


def invert(prob, iters, net=None, first_step=0.02, record=None, target="lbfgs", log=None,
           learned_iters=4, learned_tries=2, layers=7):
    """Plain (net=None) or learned-direction inversion.  Returns a history of dicts
    (iteration, solves so far, misfit, model error, direction used).

    `record`, when a list, receives one training pair per iteration once the run has ended:
    the features of iterate k and its target (see the module docstring: "lbfgs", "update"
    or "error").  A network proposes its output / GAIN with a unit first trial step.

    learned_iters: use the network only in the first that many iterations (None: always;
    the default 4 was the best of 2, 4, 6, 8 and always on the 128 x 128 x 96 problems);
    learned_tries: Wolfe trials a learned direction gets before the iteration falls back to
    L-BFGS."""
    p = (prob.init / prob.scale).contiguous()
    lb = GpuLBFGS(p.shape, layers)
    prob.solves = 0
    J, g = prob.gradient(p)
    hist = [dict(it=0, solves=prob.solves, misfit=J, model_error=prob.model_error(p), used="init")]
    kept = []
    for it in range(1, iters + 1):
        lb.push(p, g)
        use_net = net is not None and (learned_iters is None or it <= learned_iters)
        acc, used, d = None, None, None
        if use_net:
            out = net.forward(features(g, p, prob.illum))
            d = (out[..., :3].permute(3, 0, 1, 2) / GAIN).contiguous()
            if float(d.abs().max()) > 0:
                acc = _wolfe(prob, p, J, g, d, 1.0, tries=learned_tries)
                used = "learned"
        if acc is None:
            d = lb.direction(g)
            a0 = 1.0 if lb.has_pairs else first_step / max(float(d.abs().max()), 1e-30)
            acc = _wolfe(prob, p, J, g, d, a0)
            if acc is None and lb.has_pairs:
                # restart: drop the curvature pairs, retry along the steepest descent
                lb.reset()
                lb.push(p, g)
                d = -g
                acc = _wolfe(prob, p, J, g, d, first_step / max(float(d.abs().max()), 1e-30))
            if acc is None:
                hist.append(dict(it=it, solves=prob.solves, misfit=J,
                                 model_error=prob.model_error(p), used="stalled"))
                break
            used = "fallback" if use_net else "lbfgs"
        a, J_new, g_new = acc
        step = a * d
        if record is not None:
            kept.append((features(g, p, prob.illum), p.clone(), step / step.abs().max()))
        if _dot(step, g_new - g) <= 0:
            lb.reset()  # no curvature along this step (curvature test waived): start afresh
        p, J, g = (p + step).contiguous(), J_new, g_new
        hist.append(dict(it=it, solves=prob.solves, misfit=J, model_error=prob.model_error(p),
                         used=used))
        if log:
            log(f"it {it}: J {J:.4e} solves {prob.solves} ({used})")
    if record is not None:
        for f, pk, unit_step in kept:
            if target == "raw":  # the ingredients of every target (experiment variants)
                record.append((f, pk, unit_step, p, prob.true / prob.scale))
            else:
                record.append((f, make_target(target, prob, pk, p, unit_step)))
    return hist


def make_target(target, prob, pk, p_last, unit_step, true_norm=None):
    """(ny, nz, nx, 3) training target of iterate pk of a plain run ending at p_last."""
    if target == "error":
        t = ((prob.true / prob.scale if true_norm is None else true_norm) - pk) * GAIN
    elif target == "lbfgs":
        t = (p_last - pk) * GAIN
    else:
        t = unit_step
    return t.permute(1, 2, 3, 0).contiguous()


def solves_to_reach(hist, target):
    for h in hist:
        if h["misfit"] <= target:
            return h["solves"]
    return None


POLICIES = {"always": dict(learned_iters=None), "first2": dict(learned_iters=2),
            "first4": dict(learned_iters=4), "first6": dict(learned_iters=6),
            "first8": dict(learned_iters=8)}


def experiment(train_seeds=tuple(range(100, 108)), test_seeds=(7, 8, 9), iters=12, epochs=40,
               spec=None, target="lbfgs", log=None, illumination=True, policies=None):
    """Train on plain-L-BFGS runs of seeded models, then, on unseen seeds, compare plain
    L-BFGS with each learned policy: the solves each needs to reach plain L-BFGS's final
    misfit (None: not reached within `iters` iterations)."""
    import time
    base = spec or ProblemSpec()
    samples = []
    t0 = time.time()
    for s in train_seeds:
        prob = InversionProblem(dataclasses.replace(base, seed=s), illumination)
        invert(prob, iters, record=samples, target=target)
        prob.batch.close()
    t_data = time.time() - t0
    net = PreconditionerNet(seed=0, target=target)
    t0 = time.time()
    losses = train(net, samples, epochs=epochs, log=log)
    t_train = time.time() - t0
    tests = []
    for ts in test_seeds:
        prob = InversionProblem(dataclasses.replace(base, seed=ts), illumination)
        plain = invert(prob, iters, log=log)
        target_j = plain[-1]["misfit"]
        row = dict(seed=ts, target_misfit=target_j, solves_plain=plain[-1]["solves"],
                   plain=plain, policies={})
        for name, kw in (policies or POLICIES).items():
            h = invert(prob, iters, net=net, log=log, **kw)
            row["policies"][name] = dict(solves=solves_to_reach(h, target_j),
                                         final_misfit=h[-1]["misfit"],
                                         fallbacks=sum(x["used"] == "fallback" for x in h),
                                         history=h)
        prob.batch.close()
        tests.append(row)
    summary = {}
    for name in (policies or POLICIES):
        r = [t["solves_plain"] / t["policies"][name]["solves"] if t["policies"][name]["solves"]
             else 0.0 for t in tests]
        summary[name] = dict(solve_ratio_per_seed=r, reached=sum(x > 0 for x in r))
    return dict(spec=dataclasses.asdict(base), target=target, illumination=illumination,
                train_seeds=list(train_seeds),
                test_seeds=list(test_seeds), iters=iters, epochs=epochs, n_samples=len(samples),
                loss_first=losses[0], loss_last=losses[-1], data_s=t_data, train_s=t_train,
                summary=summary, tests=tests)


def variant_experiment(variants, train_seeds=tuple(range(100, 108)), test_seeds=(7, 8, 9),
                       iters=10, spec=None, log=None, illumination=True, policy="first4"):
    """Several networks trained on the SAME plain-L-BFGS runs (one data pass): each variant
    is (target, epochs); on the unseen seeds every variant's learned run is compared with
    plain L-BFGS as in :func:`experiment`, under each policy of ``policy`` (a name or a
    comma list; with several, results are keyed "variant@policy")."""
    import time
    base = spec or ProblemSpec()
    raw = []
    t0 = time.time()
    for s in train_seeds:
        prob = InversionProblem(dataclasses.replace(base, seed=s), illumination)
        invert(prob, iters, record=raw, target="raw")
        prob.batch.close()
    t_data = time.time() - t0
    nets, info = {}, {}
    for target, epochs in variants:
        name = f"{target}_{epochs}"
        samples = [(f, make_target(target, None, pk, pl, us, tn)) for f, pk, us, pl, tn in raw]
        net = PreconditionerNet(seed=0, target=target)
        losses = train(net, samples, epochs=epochs, log=log)
        nets[name] = net
        info[name] = dict(target=target, epochs=epochs, loss_first=losses[0], loss_last=losses[-1])
        del samples
    pols = [p for p in str(policy).split(",") if p]
    runs = {(n if len(pols) == 1 else f"{n}@{p}"): (n, p) for n in nets for p in pols}
    tests = []
    for ts in test_seeds:
        prob = InversionProblem(dataclasses.replace(base, seed=ts), illumination)
        plain = invert(prob, iters, log=log)
        target_j = plain[-1]["misfit"]
        row = dict(seed=ts, target_misfit=target_j, solves_plain=plain[-1]["solves"], variants={})
        for key, (name, pol) in runs.items():
            h = invert(prob, iters, net=nets[name], log=log, **POLICIES[pol])
            row["variants"][key] = dict(solves=solves_to_reach(h, target_j),
                                        final_misfit=h[-1]["misfit"],
                                        fallbacks=sum(x["used"] == "fallback" for x in h))
        prob.batch.close()
        tests.append(row)
    summary = {}
    for key, (name, pol) in runs.items():
        sv = [t["variants"][key]["solves"] for t in tests]
        plain_tot = sum(t["solves_plain"] for t in tests)
        summary[key] = dict(info[name], policy=pol, solves=sv,
                            solves_plain=[t["solves_plain"] for t in tests],
                            total_ratio=(plain_tot / sum(sv)) if all(sv) else None)
    return dict(spec=dataclasses.asdict(base), policy=policy, illumination=illumination,
                train_seeds=list(train_seeds), test_seeds=list(test_seeds), iters=iters,
                n_samples=len(raw), data_s=t_data, summary=summary, tests=tests)


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned-preconditioner experiment")
    ap.add_argument("--iters", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--train", type=int, default=8, help="number of training seeds")
    ap.add_argument("--target", default="lbfgs", choices=["lbfgs", "update", "error"])
    ap.add_argument("--test-seeds", default="7,8,9")
    ap.add_argument("--grid", default="48,48,40", help="nx,ny,nz")
    ap.add_argument("--nt", type=int, default=320)
    ap.add_argument("--shots", type=int, default=4)
    ap.add_argument("--receivers", type=int, default=8, help="per side of the surface grid")
    ap.add_argument("--no-illumination", action="store_true",
                    help="leave feature channel 7 (forward illumination) empty")
    ap.add_argument("--dx", type=float, default=10.0)
    ap.add_argument("--lenpml", type=int, default=8)
    ap.add_argument("--fq", type=float, default=12.0)
    ap.add_argument("--policies", default="first4,first2", help="comma list of " + ",".join(POLICIES))
    ap.add_argument("--out", default=None)
    ap.add_argument("--variants", default=None,
                    help="target:epochs,... -- several networks trained on one data pass")
    a = ap.parse_args()
    gx, gy, gz = (int(v) for v in a.grid.split(","))
    spec = ProblemSpec(nx=gx, ny=gy, nz=gz, nt=a.nt, nshots=a.shots, nrec=a.receivers, dx=a.dx,
                       lenpml=a.lenpml, fq=a.fq)
    if a.variants:
        vs = [(t, int(e)) for t, e in (v.split(":") for v in a.variants.split(","))]
        r = variant_experiment(vs, train_seeds=tuple(range(100, 100 + a.train)),
                               test_seeds=tuple(int(v) for v in a.test_seeds.split(",")),
                               iters=a.iters, spec=ProblemSpec(nx=gx, ny=gy, nz=gz, nt=a.nt,
                                                               nshots=a.shots, nrec=a.receivers,
                                                               dx=a.dx, lenpml=a.lenpml, fq=a.fq),
                               log=print, illumination=not a.no_illumination,
                               policy=a.policies)
        if a.out:
            with open(a.out, "w") as f:
                f.write(json.dumps(r, indent=1))
        print(json.dumps(r["summary"]))
        raise SystemExit(0)
    r = experiment(train_seeds=tuple(range(100, 100 + a.train)),
                   test_seeds=tuple(int(v) for v in a.test_seeds.split(",")),
                   iters=a.iters, epochs=a.epochs, spec=spec, target=a.target, log=print,
                   illumination=not a.no_illumination,
                   policies={k: POLICIES[k] for k in a.policies.split(",")})
    s = json.dumps(r, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s)
    print(json.dumps({k: v for k, v in r.items() if k != "tests"}))
