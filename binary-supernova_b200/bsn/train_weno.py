"""Train the default learned-WENO networks on the GPU and write them to
bsn/weno_mlp.npz (or --out).

Training pairs (normalised 5-point stencil, FP64 WENO-Z weights) come from
the method's own FP64 runs on the device, seeded and deterministic:

* Sod shock tube, 64^3 on [0,1]^3 along x, gamma 1.4, CFL 0.4, to t = 0.2
  (test/test_sod3d.jl setup);
* Sedov blast, 128^3 on [-1,1]^3, gamma 5/3, E = 1 in r < 3.5 dx, floors
  1e-6, to t = 0.05 (src/euler3d.jl:275-316 IC);
* n = 1 polytrope (M = 1, R = 0.5, G = 1) in a rho = 1e-8 atmosphere, 128^3 on
  [-1,1]^3, hydro + isolated self-gravity (coupled_step without BHs).

The sample budget (pairs over both networks) is split evenly between the
networks and the sources; Sod and Sedov are sampled after every step, the
polytrope every second step, with a sampling stride chosen so a source's
share spreads over its whole run.
Training runs the library's own forward/backward/Adam kernels; a held-out
1 % reports the mean |reconstruction - WENO-Z| of the network against that
of the linear weights.

    python -m bsn.train_weno [--samples 100000000] [--steps 100000] [--out PATH]
"""
from __future__ import annotations

import argparse
import math
import time

import numpy as np
import torch

from . import api as B
from . import ics
from . import learned as L


def _cand(u, side):
    if side == 0:
        return torch.stack([u[:, 0] / 3 - 7 * u[:, 1] / 6 + 11 * u[:, 2] / 6,
                            -u[:, 1] / 6 + 5 * u[:, 2] / 6 + u[:, 3] / 3,
                            u[:, 2] / 3 + 5 * u[:, 3] / 6 - u[:, 4] / 6], 1)
    return torch.stack([-u[:, 0] / 6 + 5 * u[:, 1] / 6 + u[:, 2] / 3,
                        u[:, 1] / 3 + 5 * u[:, 2] / 6 - u[:, 3] / 6,
                        11 * u[:, 2] / 6 - 7 * u[:, 3] / 6 + u[:, 4] / 3], 1)


def reconstruction_errors(S: torch.Tensor, params: torch.Tensor, side: int):
    """(network, linear weights) mean |sum_k (w_k - omega_k) q_k| over samples S
    (tensor-core inference)."""
    u, t = S[:, :5].contiguous(), S[:, 5:].double()
    q = _cand(u.double(), side)
    w = L.evaluate(u, params, tensor_cores=True).double()
    d = torch.tensor(L.IDEAL[side], device=S.device, dtype=torch.float64)
    return ((w - t) * q).sum(1).abs().mean().item(), ((d[None] - t) * q).sum(1).abs().mean().item()


def _sod(buf, stride, seed):
    n = 64
    U = B.state(n, n, n)
    dx, dy, dz = ics.sod_ic_3d(U, n, n, n, "x", 1.4)
    t, k = 0.0, 0
    while t < 0.2 - 1e-14:
        t, _ = B.run_steps(U, n, n, n, dx, dy, dz, 1.4, 0.4, n_steps=1, t=t, t_end=0.2)
        buf.collect(U, n, n, n, 1.4, stride=stride, seed=seed + k)
        k += 1
    return k


def _sedov(buf, stride, seed):
    n, g = 128, 5 / 3
    dx = 2.0 / n
    U = B.state(n, n, n)
    ics.sedov_ic_3d(U, n, n, n, dx, dx, dx, g, E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5,
                    x_offset=-1.0, y_offset=-1.0, z_offset=-1.0)
    t, k = 0.0, 0
    while t < 0.05 - 1e-14:
        t, _ = B.run_steps(U, n, n, n, dx, dx, dx, g, 0.4, n_steps=1, t=t, t_end=0.05, rho_floor=1e-6,
                           P_floor=1e-6)
        buf.collect(U, n, n, n, g, stride=stride, seed=seed + k)
        k += 1
    return k


def _polytrope(buf, stride, seed, steps=160):
    n, g, Lh = 128, 2.0, 1.0
    dx = 2 * Lh / n
    U = B.state(n, n, n)
    ics.polytrope_ic_3d(U, n, n, n, dx, dx, dx, g, M_star=1.0, R_star=0.5, x0=-Lh, y0=-Lh, z0=-Lh,
                        rho_floor=1e-8, P_floor=1e-10)
    t = 0.0
    for k in range(steps):
        dt = B.cfl_dt_3d(U, n, n, n, dx, dx, dx, g, 0.4)
        B.coupled_step(U, [], dt, t, n, n, n, dx, -Lh, -Lh, -Lh, g, 1.0, 1e-8, 1e-10, True, True, 0.0, 0.0)
        t += dt
        if k % 2 == 1:
            buf.collect(U, n, n, n, g, stride=stride, seed=seed + k)
    return steps // 2


def collect_all(total: int, seed: int = 0, log=print):
    """Device samples (left, right) of about `total` pairs in all (half per
    network, a third of that per source).  A counting pass (1-sample buffer; the library counts every kept
    stencil) measures each source's yield, then the source is re-run with the
    stride that spreads its share over the whole run."""
    per = max(1, total // 6)
    outs = [[], []]
    for name, fn in (("sod", _sod), ("sedov", _sedov), ("polytrope", _polytrope)):
        t0 = time.time()
        probe = L.SampleBuffers(1)
        snaps = fn(probe, 1, seed)
        avail = max(probe.counts)
        stride = max(1, math.ceil(avail / per))
        buf = L.SampleBuffers(min(per, avail) + 1_000_000)
        fn(buf, stride, seed + 1000)
        nl, nr = buf.stored
        outs[0].append(buf.left().clone())
        outs[1].append(buf.right().clone())
        del buf, probe
        torch.cuda.empty_cache()
        log(f"{name}: {snaps} snapshots, {avail} smooth stencils per side, stride {stride}, kept {nl} / {nr} "
            f"({time.time() - t0:.1f} s)")
    return torch.cat(outs[0]), torch.cat(outs[1])


def train_default(samples=100_000_000, steps=100_000, batch=16384, lr=2e-3, seed=0, log=print):
    SL, SR = collect_all(samples, seed, log)
    out, meta = [], {}
    for side, S in ((0, SL), (1, SR)):
        g = torch.Generator(device=S.device).manual_seed(seed + 17 + side)
        perm = torch.randperm(S.shape[0], device=S.device, generator=g)
        S = S[perm]
        nv = max(10_000, S.shape[0] // 100)
        val, tr = S[:nv].contiguous(), S[nv:].contiguous()
        del S
        p = L.init_params(seed=seed + 6 + side, side=side)
        l0 = L.grad(val, p)[1] / nv
        t0 = time.time()
        L.train(tr, p, steps=steps, batch=batch, lr=lr, seed=seed + 7 + side)
        torch.cuda.synchronize()
        l1 = L.grad(val, p)[1] / nv
        en, el = reconstruction_errors(val, p, side)
        log(f"side {side}: {tr.shape[0]} training pairs, {steps} steps x {batch} in {time.time() - t0:.1f} s; "
            f"held-out loss {l0:.3e} -> {l1:.3e}; mean |recon - WENO-Z| network {en:.3e}, linear {el:.3e} "
            f"({el / max(en, 1e-300):.1f}x)")
        meta[f"side{side}_pairs"] = tr.shape[0]
        meta[f"side{side}_val_loss"] = l1
        meta[f"side{side}_err_net"] = en
        meta[f"side{side}_err_lin"] = el
        out.append(p)
        del tr, val
        torch.cuda.empty_cache()
    meta.update(steps=steps, batch=batch, lr=lr, seed=seed)
    return out[0], out[1], meta


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--samples", type=int, default=100_000_000)
    ap.add_argument("--steps", type=int, default=100_000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=L.DEFAULT_PATH)
    a = ap.parse_args()
    pl, pr, meta = train_default(a.samples, a.steps, a.batch, a.lr, a.seed)
    L.save(a.out, pl, pr, **meta)
    print(f"wrote {a.out}")


if __name__ == "__main__":
    main()
