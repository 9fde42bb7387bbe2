"""Learned preconditioner: training pairs from the plain solver, and the
training loop on the device (piro_pcnet_* of include/piro.h).

Problem family (the backward-Euler configuration): alpha a smoothed log-normal
field (sigma 1.5, Gaussian filter over 8 cells), dt = 50 h^2 / (6 max alpha),
A = I - dt diag(alpha) L with the central 7-point L, b the Gaussian bump.

Pairs.  For one alpha field the plain Jacobi-PCG solver (piro_be_solve) gives
the converged x* and the iterate x_k after k inner iterations (one refinement
sweep, inner cap k; x_0 = b).  e_k = x* - x_k is the error and r_k = A e_k the
residual the preconditioner sees at that iterate; both are divided by
rms(r_k) over the interior, as the solver scales the network input.  Random
cubic crops (plus a one-cell zero ghost layer) of r, e and the feature
log(dt alpha / h^2) make the training set.  The loss mask keeps crop cells at
least 4 cells (the network's receptive radius) from every crop face that is
not a face of the domain, where zero padding is the true boundary condition.

Every numerical step -- assembly, the solves, r = A e, the network's forward
and backward passes and Adam -- runs in libpiro_b200.so; torch only holds the
buffers and cuts the crops.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import workloads as W

RADIUS = 4
SNAP_ITERS = (0, 1, 2, 3, 5, 8, 12, 17, 23, 30)


_ALPHA: dict = {}


def _alpha_field(n: int, seed: int) -> np.ndarray:
    return W.smoothed_lognormal(n, 1.5, 8.0, seed)


def prefetch_alpha(n: int, seeds, workers: int | None = None) -> None:
    """Generate the alpha fields of `seeds` in a process pool (started with
    spawn, so it is safe after CUDA initialisation) and keep them for
    be_family."""
    import concurrent.futures as cf
    import multiprocessing as mp
    todo = [s for s in seeds if (n, s) not in _ALPHA]
    if not todo:
        return
    workers = workers or min(len(todo), os.cpu_count() or 1)
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        for s, a in zip(todo, ex.map(_alpha_field, [n] * len(todo), todo)):
            _ALPHA[(n, s)] = a


def be_family(n: int, seed: int):
    """One member of the backward-Euler family on an n^3 grid (ghost-inclusive)."""
    alpha = _ALPHA.get((n, seed))
    if alpha is None:
        alpha = _alpha_field(n, seed)
    dt = np.float32(50.0 / (6.0 * float(alpha.max())))
    s = n / 32.0
    b = W.gaussian_bump(n, 4.0 * s, (n - 1) / 2.0)
    b = W.zero_boundary(b, n, n, n).astype(np.float32)
    return alpha, dt, b


def assemble(ops, n, alpha_t, dt):
    """M = diag(alpha) L (central scheme, h = 1) and A = I - dt M, on the device."""
    N = n ** 3
    M = ops.csr_laplacian(n, n, n, 3, 1.0)
    ops.csr_rowscale(M[0], M[2], alpha_t)
    I = ops.csr_identity(N)
    A = ops.csrgeam2(N, I, -float(dt), M)
    return M, A


def feature(torch, n, alpha_t, dt):
    """log(dt * alpha / h^2) on interior cells, 0 on the boundary (h = 1)."""
    f = torch.log(alpha_t * float(dt)).reshape(n, n, n)
    out = torch.zeros_like(f)
    out[1:-1, 1:-1, 1:-1] = f[1:-1, 1:-1, 1:-1]
    return out.reshape(-1)


def snapshots(torch, ops, n, seed, iters=SNAP_ITERS, net=None):
    """(r_k, e_k) pairs of one alpha field, scaled by 1/rms(r_k), plus the
    feature.  With `net` the iterates x_k come from flexible CG with that
    network (the residuals it meets when it preconditions), else from
    Jacobi-PCG."""
    alpha, dt, b = be_family(n, seed)
    alpha_t = torch.from_numpy(alpha).cuda()
    b_t = torch.from_numpy(b).cuda()
    M, A = assemble(ops, n, alpha_t, dt)
    solver = ops.BESolver(n, n, n, A, alpha_t, stencil=(float(dt), 1.0))
    xs = torch.empty_like(b_t)
    solver.solve(b_t, xs, rtol=1e-10, max_outer=40, strict=False)
    if net is not None:
        solver.set_preconditioner(net)
    n_int = (n - 2) ** 3
    pairs = []
    xk = torch.empty_like(b_t)
    r = torch.empty_like(b_t)
    for k in iters:
        if k == 0:
            xk.copy_(b_t)
        else:
            solver.solve(b_t, xk, rtol=1e-30, max_outer=1, max_inner=k, strict=False)
        e = (xs - xk).reshape(n, n, n)
        e_in = torch.zeros_like(e)
        e_in[1:-1, 1:-1, 1:-1] = e[1:-1, 1:-1, 1:-1]
        e_in = e_in.reshape(-1).contiguous()
        r.zero_()
        ops.csr_i1(n, n, n, M, float(dt), e_in, r)  # r = e - dt M e = A e on interior rows
        rms = float(torch.sqrt((r.double() ** 2).sum() / n_int))
        if not math.isfinite(rms) or rms == 0.0:
            continue
        pairs.append(((r / rms).clone(), (e_in / rms).clone()))
    solver.close()
    return pairs, feature(torch, n, alpha_t, dt)


def crops(torch, n, pairs, feat, c, count, rng, relative=True):
    """`count` random crops of interior size c per pair -> (r, f, e, mask) on (c+2)^3 grids."""
    m = c + 2
    out_r, out_f, out_e, out_m = [], [], [], []
    f3 = feat.reshape(n, n, n)
    for r, e in pairs:
        r3, e3 = r.reshape(n, n, n), e.reshape(n, n, n)
        for _ in range(count):
            o = rng.integers(1, n - 1 - c + 1, size=3)  # crop interior = cells o .. o+c-1 per axis
            sl = tuple(slice(int(o[a]), int(o[a]) + c) for a in (2, 1, 0))  # (z, y, x)
            for src, dst in ((r3, out_r), (f3, out_f), (e3, out_e)):
                t = torch.zeros((m, m, m), device=r.device)
                t[1:-1, 1:-1, 1:-1] = src[sl]
                dst.append(t.reshape(-1))
            mk = torch.zeros((m, m, m), device=r.device)
            lo = [1 if int(o[a]) == 1 else 1 + RADIUS for a in (2, 1, 0)]
            hi = [m - 1 if int(o[a]) + c == n - 1 else m - 1 - RADIUS for a in (2, 1, 0)]
            mk[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = 1.0
            if relative:
                # weight 1 / mean(e^2) over the mask: every crop counts by its
                # relative error, whatever its iteration's error magnitude
                ms = float((mk * out_e[-1].reshape(m, m, m) ** 2).sum() / mk.sum().clamp(min=1.0))
                mk *= 1.0 / ms if ms > 0.0 else 0.0
            out_m.append(mk.reshape(-1))
    st = lambda v: torch.stack(v) if v else None  # noqa: E731
    return st(out_r), st(out_f), st(out_e), st(out_m)


def make_dataset(torch, ops, n, seeds, crop, crops_per_pair, seed=0, log=None, net=None, relative=True):
    rng = np.random.default_rng(seed)
    R, F, E, Mk = [], [], [], []
    for s in seeds:
        pairs, feat = snapshots(torch, ops, n, s, net=net)
        r, f, e, m = crops(torch, n, pairs, feat, crop, crops_per_pair, rng, relative)
        if r is not None:
            R.append(r)
            F.append(f)
            E.append(e)
            Mk.append(m)
        if log:
            log(f"seed {s}: {len(pairs)} pairs")
    return torch.cat(R), torch.cat(F), torch.cat(E), torch.cat(Mk)


def train(torch, ops, net, data, crop, steps, batch=16, lr=2e-3, seed=0, log=None, log_every=100):
    """Adam on the masked MSE, cosine learning-rate decay; returns the loss history."""
    R, F, E, Mk = data
    m = crop + 2
    rng = np.random.default_rng(seed)
    hist = []
    for it in range(steps):
        idx = torch.from_numpy(rng.integers(0, R.shape[0], size=batch)).to(R.device)
        r, f, e, mk = (R[idx].contiguous(), F[idx].contiguous(), E[idx].contiguous(), Mk[idx].contiguous())
        want = (it % log_every == 0) or it == steps - 1
        loss, _ = net.loss_grad(m, m, m, r, f, e, mk, batch=batch, want_loss=want)
        cur = lr * 0.5 * (1.0 + math.cos(math.pi * it / steps))
        net.adam_step(max(cur, lr * 1e-3))
        if want:
            hist.append((it, loss))
            if log:
                log(f"step {it}: loss {loss:.5f}")
    return hist


def compare(torch, ops, net, n, seeds, rtol=1e-8):
    """Plain Jacobi-PCG vs learned FCG on the same problems: iterations, ms, residual."""
    rows = []
    for s in seeds:
        alpha, dt, b = be_family(n, s)
        alpha_t = torch.from_numpy(alpha).cuda()
        b_t = torch.from_numpy(b).cuda()
        _, A = assemble(ops, n, alpha_t, dt)
        row = {"seed": s}
        for name in ("jacobi", "learned"):
            sv = ops.BESolver(n, n, n, A, alpha_t, stencil=(float(dt), 1.0))
            if name == "learned":
                sv.set_preconditioner(net)
            x = torch.empty_like(b_t)
            sv.solve(b_t, x, rtol=rtol, strict=False)  # warm-up
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            info = sv.solve(b_t, x, rtol=rtol, strict=False)
            e1.record()
            torch.cuda.synchronize()
            row[name] = {"status": info.status, "iters": info.inner_iterations, "sweeps": info.outer_iterations,
                         "fallbacks": info.fallbacks, "rel": info.rel_residual, "ms": e0.elapsed_time(e1)}
            sv.close()
        rows.append(row)
    return rows


def summary(rows):
    """Mean iterations and ms of the plain and learned solves over `rows`."""
    out = {}
    for k in ("jacobi", "learned"):
        out[k] = {"iters": float(np.mean([r[k]["iters"] for r in rows])),
                  "ms": float(np.mean([r[k]["ms"] for r in rows])),
                  "worst_rel": float(max(r[k]["rel"] for r in rows)),
                  "fallbacks": int(sum(r[k]["fallbacks"] for r in rows))}
    out["iteration_ratio"] = out["jacobi"]["iters"] / out["learned"]["iters"]
    out["time_ratio"] = out["jacobi"]["ms"] / out["learned"]["ms"]
    return out


def fit(torch, ops, n, seeds, crop, crops_per_pair, steps, batch, lr, rounds, log=None):
    """Train a network: one round on Jacobi-PCG iterates, then `rounds` more
    that add the iterates of flexible CG with the network being trained."""
    data = make_dataset(torch, ops, n, seeds, crop, crops_per_pair, log=log)
    net = ops.PCNet(seed=0)
    hist = [train(torch, ops, net, data, crop, steps, batch, lr, log=log)]
    for rnd in range(1, rounds + 1):
        more = make_dataset(torch, ops, n, seeds, crop, crops_per_pair, seed=rnd, net=net, log=log)
        data = tuple(torch.cat([a, b]) for a, b in zip(data, more))
        del more
        hist.append(train(torch, ops, net, data, crop, steps, batch, lr * 0.5, seed=rnd, log=log))
    return net, int(data[0].shape[0]), hist


def main():
    ap = argparse.ArgumentParser(description="train the learned preconditioner on the device")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--seeds", type=str, default="100:200")
    ap.add_argument("--eval-seeds", type=str, default="200:210")
    ap.add_argument("--crop", type=int, default=32)
    ap.add_argument("--crops-per-pair", type=int, default=10)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--rounds", type=int, default=2, help="on-policy rounds after the first")
    ap.add_argument("--out", type=str, required=True, help="weights file (.npy, float32)")
    ap.add_argument("--report", type=str, default=None, help="JSON report")
    args = ap.parse_args()
    lo, hi = (int(v) for v in args.seeds.split(":"))
    elo, ehi = (int(v) for v in args.eval_seeds.split(":"))
    t0 = time.time()
    prefetch_alpha(args.n, list(range(lo, hi)) + list(range(elo, ehi)))
    import torch

    from . import ops
    t1 = time.time()
    log = lambda s: print(s, flush=True)  # noqa: E731
    net, pairs, hist = fit(torch, ops, args.n, range(lo, hi), args.crop, args.crops_per_pair, args.steps,
                           args.batch, args.lr, args.rounds, log=log)
    torch.cuda.synchronize()
    t2 = time.time()
    np.save(args.out, net.get_params())
    rows = compare(torch, ops, net, args.n, range(elo, ehi))
    rep = {"n": args.n, "train_seeds": [lo, hi], "eval_seeds": [elo, ehi], "pairs": pairs,
           "alpha_s": t1 - t0, "train_s": t2 - t1, "loss": hist, "eval": rows, "summary": summary(rows)}
    print(json.dumps(rep["summary"]), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
