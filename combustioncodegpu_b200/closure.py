"""Learned transport closure: training data, training and validation.

The closure replaces the Wilke / constant-Schmidt transport evaluation
(Transport.cu:43-96) by an MLP (T, X_1..X_n) -> (log mu, log lambda,
log rhoD_1..rhoD_n) evaluated on the tensor cores (csrc/closure.cuh); points
outside the training hull in T take the exact transport.

Training data: T ~ U[t_min, t_max] and compositions from three equal parts:
X ~ Dirichlet(0.5 * 1_n) (near the edges of the simplex, a few species
dominant), X ~ Dirichlet(4 * 1_n) (mixtures of all species) and
Y ~ Dirichlet(2 * 1_n) (mixtures of all species by mass, whose mole
fractions the light species dominate, as in the synthetic box); targets are the library's own exact FP64 transport of those points
(cc_eval_transport, mode 0).  The network is trained with the arithmetic of
the kernel: inputs as BF16 (hi, lo) pairs, BF16 weights (rounding with a
straight-through gradient), FP32 hidden activations (the kernel keeps them
as BF16 hi/lo pairs), FP32 accumulation and biases; the loss is the mean
squared error of the log properties, i.e. of the relative error.  Training
runs on the GPU with the library's own
forward/backward and Adam kernels (cc_mlp_grad, cc_mlp_adam; an offline
step, not the hot path), checked against the CPU restatement of the same
math in oracle/closure_mlp.py; the result is a dict that Driver.set_closure
takes.  ClosureNet is the plain PyTorch FP32 model of the same network with
the same rounding points (BF16 weights and inputs, FP32 hidden activations,
which the kernel carries as BF16 hi/lo pairs): the reference the inference
kernel is tested against, and the evaluation of the trained weights.

  python -m combustioncodegpu_b200.closure --out closure_weights.npz
"""
import argparse
import ctypes
import json
import os
import time

import numpy as np

HIDDEN = 64
T_MIN, T_MAX = 300.0, 2500.0
T_CENTER, T_SCALE = 0.5 * (T_MIN + T_MAX), 0.5 * (T_MAX - T_MIN)
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "closure_weights.npz")


TRAIN_MIX = (("X", 0.5), ("X", 4.0), ("Y", 2.0))


def sample_states(n, species, seed, mix=TRAIN_MIX, t_range=(T_MIN, T_MAX)):
    """n random states: T [n], Y [ns][n], X [ns][n].  Each state's
    composition comes from one part of `mix` (equal shares), a sequence of
    (space, alpha): X ~ Dirichlet(alpha * 1_n) for space "X", Y ~
    Dirichlet(alpha * 1_n) for "Y"; a single pair is accepted too."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ns = species["n_spec"]
    mw = np.asarray(species["mw"])[:, None]
    if isinstance(mix[0], str):
        mix = (mix,)
    T = rng.uniform(t_range[0], t_range[1], n)
    which = rng.integers(0, len(mix), n)
    X = np.empty((ns, n))
    for i, (space, a) in enumerate(mix):
        m = which == i
        v = rng.dirichlet(np.full(ns, a), int(m.sum())).T
        if space == "Y":
            v = v / mw
            v /= v.sum(axis=0, keepdims=True)
        X[:, m] = v
    Y = X * mw / (X * mw).sum(axis=0, keepdims=True)
    return T, Y, X


def mole_fractions(Y, mw):
    x = Y / np.asarray(mw)[:, None]
    return x / x.sum(axis=0, keepdims=True)


def _bf16(x):
    import torch
    return x.to(torch.bfloat16).to(torch.float32)


def _round_ste(x):
    """BF16 rounding in the forward pass, identity gradient."""
    return x + (_bf16(x) - x).detach()


def features(T, X, torch_device="cpu"):
    """Network inputs as the kernel forms them: [t_hi, t_lo, X_hi, X_lo],
    each BF16, from t = (T - T_CENTER) / T_SCALE and the mole fractions (FP32)."""
    import torch
    t = ((torch.as_tensor(T, dtype=torch.float32, device=torch_device) - np.float32(T_CENTER))
         * np.float32(1.0 / T_SCALE))
    Xt = torch.as_tensor(X, dtype=torch.float32, device=torch_device)  # [ns][n]
    t_hi = _bf16(t)
    x_hi = _bf16(Xt)
    return torch.cat([t_hi[None], _bf16(t - t_hi)[None], x_hi, _bf16(Xt - x_hi)], dim=0).T.contiguous()


class ClosureNet:
    """The closure MLP with the kernel's rounding points (torch, FP32 master)."""

    def __init__(self, n_in, n_out, device, seed=0):
        import torch
        g = torch.Generator(device="cpu").manual_seed(seed)
        dims = [(n_in, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, n_out)]
        self.params = []
        for i, (a, b) in enumerate(dims):
            w = torch.randn(b, a, generator=g) * (1.0 / np.sqrt(a)) * (0.5 if i == 3 else 1.0)
            self.params += [w.to(device).requires_grad_(), torch.zeros(b, device=device).requires_grad_()]

    def forward(self, x, quantized=True):
        import torch
        r = _round_ste if quantized else (lambda v: v)
        h = x  # BF16 (hi, lo) features; the hidden activations stay FP32
        for i in range(4):
            w, b = self.params[2 * i], self.params[2 * i + 1]
            h = h @ r(w).T + b
            if i < 3:
                h = torch.nn.functional.silu(h)
        return h

    def export(self, out_mean, out_scale):
        names = ["w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4"]
        d = {k: p.detach().cpu().numpy().astype(np.float32) for k, p in zip(names, self.params)}
        d.update({"out_mean": np.asarray(out_mean, np.float32), "out_scale": np.asarray(out_scale, np.float32),
                  "t_center": T_CENTER, "t_scale": T_SCALE, "t_min": T_MIN, "t_max": T_MAX})
        return d


def one_cycle(step, total, max_lr, pct_start=0.05, div_factor=25.0, final_div_factor=1e4,
              beta_lo=0.85, beta_hi=0.95):
    """(lr, beta1) of the one-cycle policy (Smith & Topin, 2019) at step
    (0-based) of total: cosine warm-up from max_lr / div_factor to max_lr over
    pct_start of the steps while beta1 falls from beta_hi to beta_lo, then
    cosine decay to max_lr / (div_factor * final_div_factor) while beta1
    returns to beta_hi."""
    lo_lr = max_lr / div_factor
    end1 = pct_start * total - 1.0
    cos = lambda a, b, t: b + (a - b) / 2.0 * (1.0 + np.cos(np.pi * t))
    if step <= end1:
        t = step / end1 if end1 > 0 else 1.0
        return cos(lo_lr, max_lr, t), cos(beta_hi, beta_lo, t)
    t = (step - end1) / max(1.0, (total - 1) - end1)
    return cos(max_lr, lo_lr / final_div_factor, t), cos(beta_lo, beta_hi, t)


def train(driver, species, n_samples=2_000_000, n_val=200_000, epochs=600, batch=4096, lr=4e-3, seed=7,
          device="cuda", log=print):
    """Fit the closure to the exact transport of `driver`'s species tables
    with the library's training kernels (cc_mlp_grad: quantisation-aware
    forward and backward; cc_mlp_adam).  PyTorch only holds the device
    arrays, draws the initial weights and shuffles the batches.
    Returns (weights dict, report dict)."""
    import torch
    from . import load_library

    lib = load_library()
    t0 = time.time()
    T, Y, X = sample_states(n_samples + n_val, species, seed)
    tgt = np.log(driver.eval_transport(T, Y, "exact"))  # [2+ns][n]
    t_data = time.time() - t0
    ns = species["n_spec"]
    n_in, n_out = 2 + 2 * ns, 2 + ns
    mean = tgt[:, :n_samples].mean(axis=1)
    scale = tgt[:, :n_samples].std(axis=1) + 1e-6
    x_all = features(T, X, device)
    y_all = torch.as_tensor(((tgt - mean[:, None]) / scale[:, None]).T, dtype=torch.float32, device=device)
    sc = torch.as_tensor(scale, dtype=torch.float32, device=device)
    xtr, ytr = x_all[:n_samples], y_all[:n_samples]
    net = ClosureNet(n_in, n_out, device, seed)  # initial weights
    params = torch.cat([p.detach().reshape(-1) for p in net.params]).contiguous()
    n_par = lib.cc_mlp_param_count(n_in, HIDDEN, n_out)
    assert n_par == params.numel()
    grad = torch.zeros_like(params)
    m1 = torch.zeros_like(params)
    m2 = torch.zeros_like(params)
    work = torch.empty(lib.cc_mlp_workspace_bytes(n_in, HIDDEN, n_out, batch), dtype=torch.uint8, device=device)
    loss = torch.zeros(1, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream().cuda_stream
    steps = epochs * (n_samples // batch)
    gen = torch.Generator(device=device).manual_seed(seed)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    t1 = time.time()
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(n_samples, device=device, generator=gen)
        tot, cnt = 0.0, 0
        for b in range(n_samples // batch):
            idx = perm[b * batch:(b + 1) * batch]
            xb, yb = xtr[idx].contiguous(), ytr[idx].contiguous()
            rc = lib.cc_mlp_grad(n_in, HIDDEN, n_out, batch, vp(params), vp(xb), vp(yb), vp(sc), vp(grad), vp(loss),
                                 vp(work), ctypes.c_void_p(stream))
            if rc != 0:
                raise RuntimeError(lib.cc_last_error().decode())
            lr_t, beta1 = one_cycle(step, steps, lr)
            step += 1
            rc = lib.cc_mlp_adam(n_par, vp(params), vp(grad), vp(m1), vp(m2), lr_t, beta1, 0.999, 1e-8, step,
                                 ctypes.c_void_p(stream))
            if rc != 0:
                raise RuntimeError(lib.cc_last_error().decode())
            if b % 50 == 0:
                tot, cnt = tot + float(loss), cnt + 1
        if ep % 10 == 0 or ep == epochs - 1:
            log("epoch %d  loss(sampled) %.3e" % (ep, tot / max(1, cnt)))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    off = 0
    for p in net.params:  # the trained weights back into the PyTorch model, for its evaluation below
        with torch.no_grad():
            p.copy_(params[off:off + p.numel()].view_as(p))
        off += p.numel()
    w = net.export(mean, scale)
    with torch.no_grad():
        o = net.forward(x_all[n_samples:]).cpu().numpy() * scale + mean  # the trained model, log space
    rel_torch = np.abs(np.expm1(o.T - tgt[:, n_samples:]))
    report = {"n_samples": n_samples, "n_val": n_val, "epochs": epochs, "batch": batch, "seed": seed,
              "trainer": "cc_mlp_grad + cc_mlp_adam (the library's kernels), one-cycle schedule",
              "seconds_data": t_data, "seconds_train": t_train,
              "torch_model_rel_err": _err_summary(rel_torch)}
    return w, report


def _err_summary(rel):
    """rel: [n_out][n] relative errors."""
    worst = rel.max(axis=0)
    return {"median": float(np.median(rel)), "p99": float(np.percentile(rel, 99)), "max": float(rel.max()),
            "frac_points_above_1e-3": float((worst > 1e-3).mean()),
            "per_output_p99": [float(v) for v in np.percentile(rel, 99, axis=1)]}


def box_states(n, species, seed):
    """About n states of the synthetic multispecies box generator
    (cases.multispecies_fields: T in [300, 1500] K, smooth positive Y_k) on a
    cube of its own seed: T [m], Y [ns][m]."""
    from . import cases
    side = max(4, int(round(n ** (1.0 / 3.0))) - 4)
    bv, yk = cases.multispecies_fields((side, side, side), species, seed=seed)
    return bv[5], yk


def validate(driver, species, n=200_000, seed=99, states="train"):
    """Relative error of the closure kernel (as uploaded to driver) against
    the exact transport on fresh states inside the hull: states "train"
    (the training distribution), "edge" (its X ~ Dirichlet(0.5) part only)
    or "box" (the synthetic box generator's states, box_states)."""
    if states == "box":
        T, Y = box_states(n, species, seed)
    else:
        T, Y, _ = sample_states(n, species, seed, mix=("X", 0.5) if states == "edge" else TRAIN_MIX)
    exact = driver.eval_transport(T, Y, "exact")
    got = driver.eval_transport(T, Y, "closure")
    return _err_summary(np.abs(got / exact - 1.0))


def save(path, weights, report):
    np.savez(path, report=json.dumps(report), **{k: np.asarray(v) for k, v in weights.items()})


def load(path=DEFAULT_WEIGHTS):
    z = np.load(path, allow_pickle=False)
    w = {k: z[k] for k in z.files if k != "report"}
    for k in ("t_center", "t_scale", "t_min", "t_max"):
        w[k] = float(w[k])
    return w, json.loads(str(z["report"]))


def main():
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import cases

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=600)
    ap.add_argument("--lr", type=float, default=4e-3)
    ap.add_argument("--batch", type=int, default=4096)
    args = ap.parse_args()
    sp = cases.synthetic_species()
    d = cc.Driver.from_case(cases.case_box(4, species=sp), "mixed")
    w, report = train(d, sp, n_samples=args.samples, epochs=args.epochs, lr=args.lr, batch=args.batch)
    for states in ("train", "edge", "box"):
        sfx = "" if states == "train" else "_" + states
        d.set_closure(w)
        d.set_closure_bound(0.0)  # the network alone
        report["kernel_rel_err" + sfx] = validate(d, sp, states=states)
        d.set_closure_bound(1e-3)  # with the run-time check: the share of points it sends to the exact transport
        d.set_closure(w)
        report["kernel_rel_err_with_check" + sfx] = validate(d, sp, states=states)
        n_eval, n_hull, n_chk = d.closure_stats()
        report["check_fallback_rate" + sfx] = n_chk / max(1, n_eval)
    d.close()
    save(args.out, w, report)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
