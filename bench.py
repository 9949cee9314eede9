"""Benchmark: cell-updates/s per SSP-RK3 step on the 3D Sedov blast.

Workload (default): Sedov 256^3 on [-1,1]^3, gamma=5/3, ambient rho=1,
p=1e-5, E=1 deposited in r < 3.5 dx (the reference's sedov_ic_3d!), outflow,
floors rho 1e-6 / P 1e-6.  A step is one CFL dt reduction plus one full RK3
step, the loop the reference drivers run (cfl_dt_3d + euler3d_step!).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bsn|reference]
                  [--n 256] [--path learned|f32|f64] [--tile V] [--no-cpu]
                  [--no-accuracy] [--no-fmr]
  python bench.py --workload binary_nested [--paths f64,f32,learned]
                  [--steps K] [--warmup W] [--full]
  python bench.py --workload polytrope_fmr [--omega 0.2] [--steps K]
                  [--warmup W] [--full]

The other forms time only the binary-BH supernova on three nested 128^3
FMR levels (the coupled driver loop on the device) for the listed stencil
paths, or only the self-gravitating polytrope on two 128^3 FMR levels, and
print their JSON object; --full runs the workload's stated length from its
initial state (1000 / 200 steps).  Both report the FP64 mass budget of the
driver loop (gas mass against the ledger of floors, outflow, sink drain and
accretion) where the loop has sinks, and the L1 density and energy
differences of the reduced-precision paths against FP64 at equal time.

`value` is device-resident throughput over K steps (state in HBM).  `e2e`
runs the same step through the public host-buffer path: the state is copied
host->device from pinned memory, stepped, and copied back every step.  With
N>1 (torchrun) every rank runs an independent replica ("replicas only": the
reference path is single-device) and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "binary-supernova_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

NG = 3
GAMMA = 5.0 / 3.0
CFL = 0.4
T_MID = 0.025     # start of the timed steps (Sedov run to t = 0.05)
T_END = 0.05
METRIC = "cell-updates/s per RK3 step (Sedov 3D, WENO5-Z+HLLC+SSP-RK3)"   # both arms


_T0 = time.time()


def log(msg):
    """Progress on stderr (the JSON line is the only stdout output)."""
    print(f"[bench {time.time() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def mass_closure(rec_last, M_start, MBH_start, MBH_end):
    """The mass budget of a driver-loop call from its last diagnostics record
    (bsn.DIAG_FIELDS: the gas mass and the FP64 ledger since the call began):
    the gas-side residual |M_gas - (M_start + floors_in - outflow - drained)|
    and the whole residual with the BHs and the reference's drain / credit
    split, both relative to the mass at the start."""
    import bsn
    f = {k: float(rec_last[i]) for i, k in enumerate(bsn.DIAG_FIELDS)}
    gas = f["M_gas"] - (M_start + f["floors_in"] - f["outflow"] - f["drained"])
    total = (f["M_gas"] + MBH_end - M_start - MBH_start - f["floors_in"] + f["outflow"]
             - (f["accreted"] - f["drained"]))
    return {"M_gas_start": M_start, "M_gas_end": f["M_gas"], "M_bh_start": MBH_start, "M_bh_end": MBH_end,
            "floors_in": f["floors_in"], "outflow": f["outflow"], "drained": f["drained"],
            "accreted": f["accreted"], "gas_residual_rel": abs(gas) / M_start,
            "total_residual_rel": abs(total) / (M_start + MBH_start),
            "accreted_minus_drained": f["accreted"] - f["drained"]}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def sedov_host(n, cpu_leg=False):
    """Sedov initial state (src/euler3d.jl:275-316) on the host, F-ordered:
    from the package's IC generator, or, for the CPU reference leg (which
    must not touch the package), from the oracle's (bit-identical)."""
    import numpy as np
    L = 1.0
    dx = 2 * L / n
    kw = dict(E_blast=1.0, r_inject=3.5 * dx, rho_bg=1.0, P_floor=1e-5, x_offset=-L, y_offset=-L, z_offset=-L)
    if cpu_leg:
        import oracle
        U = oracle.state(n, n, n)
        oracle.sedov_ic_3d(U, dx, dx, dx, GAMMA, **kw)
        return U, dx
    from bsn import ics
    U = np.zeros((5, n + 2 * NG, n + 2 * NG, n + 2 * NG), dtype=np.float64, order="F")
    ics.sedov_ic_3d(U, n, n, n, dx, dx, dx, GAMMA, **kw)
    return U, dx


CPU_SLAB = 32      # z-planes of the CPU sample (both CPU legs)


def cpu_slab(U, n, nz_sample):
    """nz_sample z-planes through the blast centre of a ghosted Sedov state,
    as a grid of its own (ghost planes included, F-ordered)."""
    import numpy as np
    k0 = NG + n // 2 - nz_sample // 2
    return np.asfortranarray(U[:, :, :, k0 - NG:k0 + nz_sample + NG])


def cpu_reference_rate(S, n, dx, threads, steps, min_seconds=0.0, max_steps=64):
    """Oracle (CPU restatement of the reference path) on a z-slab sample S of
    the Sedov n^3 workload, stepped in place: cell-updates/s with `threads`
    OpenMP threads, over `steps` RK3 steps (cfl_dt_3d + euler3d_step!),
    continued until `min_seconds` have elapsed (at most `max_steps`).
    Returns (rate, seconds, steps)."""
    import oracle
    oracle.build()
    oracle.set_threads(threads)
    nz_sample = S.shape[3] - 2 * NG
    t0 = time.perf_counter()
    k = 0
    while k < steps or (time.perf_counter() - t0 < min_seconds and k < max_steps):
        dt = oracle.cfl_dt_3d(S, dx, dx, dx, GAMMA, CFL)
        oracle.euler3d_step(S, dx, dx, dx, dt, GAMMA, rho_floor=1e-6, P_floor=1e-6)
        k += 1
    el = time.perf_counter() - t0
    return n * n * nz_sample * k / el, el, k


def sedov_mid_state(n):
    """The Sedov n^3 state at t = T_MID, the state the GPU arm's timed steps
    start from, on the host.  It is made by the library's FP64 device loop,
    which is bit-identical to the oracle's own loop (FP64 parity tests up to
    the workload's sizes): the oracle would need tens of minutes of host time
    to reach it.  Without a GPU: the initial state (and t = 0)."""
    U0, dx = sedov_host(n, cpu_leg=True)
    try:
        import torch
        if not torch.cuda.is_available():
            return U0, dx, 0.0
        import bsn
        Ud = torch.from_numpy(U0).cuda()
        t, _ = bsn.run_steps(Ud, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=1_000_000, t=0.0, t_end=T_MID,
                             precision="f64", rho_floor=1e-6, P_floor=1e-6)
        return Ud.cpu().numpy(), dx, t
    except ImportError:
        return U0, dx, 0.0


def slab_sedov(args, rank, world, log):
    """Sedov n^3 at t = T_MID split into z-slabs over the ranks (bsn.shard:
    ghost fill, halo exchange over torch.distributed, one fused stage launch
    per RK3 stage, dt as the min over ranks), K steps timed with CUDA events
    (max over ranks); beside it on rank 0 of a one-rank run, the device time
    loop (bsn_run_steps) on the whole grid.  Strong scaling: the grid is the
    same whatever the rank count."""
    import torch
    import bsn
    from bsn import shard
    n = args.n
    # the package's initial condition, run to T_MID by the device loop on every rank
    Uh, dx = sedov_host(n)
    Ud0 = torch.from_numpy(Uh).cuda()
    t0, _ = bsn.run_steps(Ud0, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=1_000_000, t=0.0, t_end=T_MID,
                          precision="f64", rho_floor=1e-6, P_floor=1e-6)
    U0 = Ud0.cpu().numpy()
    del Ud0
    slab = shard.Slab.split(n, n, n, rank, world)
    k0, nzl = slab.k0, slab.nz
    out = {"workload": f"sedov{n}^3 z-slabs", "ranks": world, "planes_per_rank": nzl, "steps": args.steps}
    kw = dict(rho_floor=1e-6, P_floor=1e-6)
    dist = None
    if world > 1:
        import torch.distributed as dist
    ops = shard.DeviceOps()
    for prec in ("f64", "f32"):
        U = bsn.state(n, n, nzl)
        shard._zmajor(U)[...] = torch.from_numpy(U0.T[k0:k0 + nzl + 2 * NG].copy()).cuda()
        t = t0
        for _ in range(max(1, args.warmup)):
            t, _ = shard.run_steps(U, slab, dx, dx, dx, GAMMA, CFL, ops, n_steps=1, t=t, precision=prec, **kw)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t, k = shard.run_steps(U, slab, dx, dx, dx, GAMMA, CFL, ops, n_steps=args.steps, t=t, precision=prec, **kw)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        if dist:
            tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        out[f"{prec}_slab_ms_per_step"] = ms
        out[f"{prec}_slab_value"] = n ** 3 / (ms / 1e3)
        log(f"slab Sedov {n}^3 {prec}, {world} rank(s): {ms:.3f} ms/step")
        if world == 1:
            Ud = torch.from_numpy(U0).cuda()
            tt_, _ = bsn.run_steps(Ud, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=args.warmup, t=t0, precision=prec,
                                   **kw)
            torch.cuda.synchronize()
            e0.record()
            bsn.run_steps(Ud, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=args.steps, t=tt_, precision=prec, **kw)
            e1.record()
            torch.cuda.synchronize()
            out[f"{prec}_device_loop_ms_per_step"] = e0.elapsed_time(e1) / args.steps
        del U
    return out


def slab_fmr(args, rank, world, log):
    """The two-level FMR polytrope (the fmr_polytrope workload: 128^3 base,
    128^3 fine on [-1,1]^3, self-gravity) with the base grid in z-slabs over
    the ranks and the fine level on rank 0 (bsn.shard_fmr: coarse stages per
    slab with the register faces, the owner's window of the coarse grid, the
    fine subcycles, restriction and correction, planes sent back), K FP64
    steps timed with CUDA events (max over ranks); on a one-rank run the
    graph-captured device loop (bsn_fmr3d_run_steps) beside it, from the same
    state with the same dts, and the two results compared bit for bit."""
    import torch
    import bsn
    from bsn import ics, shard, shard_fmr
    nc, ratio, gam = 128, 2, 2.0
    dxc = 4.0 / nc
    lo, hi = 33, 96
    kw = dict(rho_floor=1e-8, P_floor=1e-10)
    U0 = bsn.state(nc, nc, nc)
    ics.polytrope_ic_3d(U0, nc, nc, nc, dxc, dxc, dxc, gam, M_star=1.0, R_star=0.5, x0=-2.0, y0=-2.0, z0=-2.0,
                        **kw)
    bsn.fill_ghost_3d_outflow(U0, nc, nc, nc)
    G = bsn.FMRGrid3D(U0.clone(), nc, nc, nc, dxc, lo, hi, lo, hi, lo, hi, ratio, gam, **kw)
    slab = shard.Slab.split(nc, nc, nc, rank, world)
    Us = bsn.state(nc, nc, slab.nz)
    shard._zmajor(Us)[...] = shard._zmajor(U0)[slab.k0:slab.k0 + slab.nz + 2 * NG]
    S = shard_fmr.SlabFMR(Us, slab, dxc, lo, hi, lo, hi, lo, hi, ratio, gam, shard.DeviceOps(), owner=0,
                          Uf=G.Uf.clone(), **kw)
    nf = (hi - lo + 1) * ratio
    units = nc ** 3 + ratio * nf ** 3
    dist = None
    if world > 1:
        import torch.distributed as dist
    dts = []
    for _ in range(max(1, args.warmup)):
        dt = S.cfl_dt(0.4)
        dts.append(dt)
        S.step(dt, self_gravity=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        dt = S.cfl_dt(0.4)
        dts.append(dt)
        S.step(dt, self_gravity=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    out = {"workload": "polytrope FMR 128^3 + 128^3 (ratio 2), self-gravity, base grid in z-slabs",
           "ranks": world, "planes_per_rank": slab.nz, "steps": args.steps, "unit": "cell-updates/s",
           "units_per_step": units, "f64_slab_ms_per_step": ms, "f64_slab_value": units / (ms / 1e3)}
    log(f"slab FMR polytrope f64, {world} rank(s): {ms:.3f} ms/step")
    if world == 1:   # the fused device step from the same state with the same dts
        for dt in dts[:max(1, args.warmup)]:
            bsn.fmr3d_step(G, dt, self_gravity=True)
        torch.cuda.synchronize()
        e0.record()
        for dt in dts[max(1, args.warmup):]:
            bsn.fmr3d_step(G, dt, self_gravity=True)
        e1.record()
        torch.cuda.synchronize()
        out["f64_fused_step_ms_per_step"] = e0.elapsed_time(e1) / args.steps
        a = (slice(None),) + (slice(NG, -NG),) * 3
        out["bitwise_equal_to_fused_step"] = bool(torch.equal(S.Uc[a], G.Uc[a]) and torch.equal(S.G.Uf[a], G.Uf[a]))
        log(f"fused fmr3d_step: {out['f64_fused_step_ms_per_step']:.3f} ms/step, "
            f"bitwise {out['bitwise_equal_to_fused_step']}")
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    nz = max(4, min(args.n, CPU_SLAB))
    U, dx, t0 = sedov_mid_state(args.n)
    log(f"reference arm: Sedov {args.n}^3 state at t={t0:.4g}; oracle on a {nz}-plane slab, {threads} threads")
    S = cpu_slab(U, args.n, nz)
    del U
    if args.warmup:
        cpu_reference_rate(S.copy(order="F"), args.n, dx, threads, args.warmup)
    rate, el, _ = cpu_reference_rate(S, args.n, dx, threads, args.steps)
    sample = (f"{args.steps} RK3 steps (cfl_dt_3d + euler3d_step!) of a {args.n}x{args.n}x{nz} z-slab through "
              f"the blast centre of Sedov {args.n}^3 at t={t0:.4g}")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate,
        "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (Sedov initial condition, sedov_ic_3d!, run to the timed state)",
        "config": {"workload": f"sedov{args.n}^3", "grid": [args.n, args.n, args.n],
                   "path": "reference CPU restatement (oracle), FP64", "threads": threads,
                   "timed_from": f"Sedov state at t={t0:.4g} (FP64 run from the initial condition)",
                   "sample": sample},
        "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def accuracy(bsn, torch, U0, n, dx, kw, t_end=T_END):
    """Sedov n^3 from the initial state to t_end on each path (device-resident
    CFL loop): L1 density / energy differences against the FP64 path and L1
    density error against the Sedov-Taylor similarity solution for the
    deposited energy (sedov_ic_3d! deposits E_blast (gamma-1))."""
    import numpy as np
    from bsn.analytic import sedov_taylor
    a = (slice(NG, NG + n),) * 3
    E_bg = 1e-5 / (GAMMA - 1)
    E_dep = float((U0[(4,) + a] - E_bg).sum() * dx ** 3)
    xc = (np.arange(1, n + 1) - 0.5) * dx - 1.0
    r = np.sqrt(xc[:, None, None] ** 2 + xc[None, :, None] ** 2 + xc[None, None, :] ** 2)
    rho_ex = sedov_taylor(r, t_end, E=E_dep, rho0=1.0, gamma=GAMMA)[0]
    out = {"t_end": t_end, "E_deposited": E_dep}
    fields = {}
    for p_ in ("f64", "f32", "learned"):
        U = torch.from_numpy(U0).cuda()
        bsn.run_steps(U, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=1, precision=p_, **kw)   # autotune, graph
        U = torch.from_numpy(U0).cuda()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t, k = bsn.run_steps(U, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=1_000_000, t_end=t_end, precision=p_,
                             **kw)
        e1.record()
        torch.cuda.synchronize()
        out[f"{p_}_run_cell_updates_per_s"] = n ** 3 * k / (e0.elapsed_time(e1) / 1e3)
        log(f"accuracy run {p_}: {k} steps to t={t:.4g} in {e0.elapsed_time(e1) / 1e3:.1f} s")
        h = U.cpu().numpy()
        fields[p_] = (h[(0,) + a].copy(), h[(4,) + a].copy())
        out[f"{p_}_steps"] = k
        del U, h
    r64, e64 = fields["f64"]
    for p_, (rh, en) in fields.items():
        out[f"l1_rho_vs_exact_{p_}"] = float(np.abs(rh - rho_ex).sum() / rho_ex.sum())
        if p_ != "f64":
            out[f"l1_rho_vs_f64_{p_}"] = float(np.abs(rh - r64).sum() / np.abs(r64).sum())
            out[f"l1_E_vs_f64_{p_}"] = float(np.abs(en - e64).sum() / np.abs(e64).sum())
    for p_ in ("f32", "learned"):
        out[f"exact_error_ratio_{p_}_over_f64"] = out[f"l1_rho_vs_exact_{p_}"] / out["l1_rho_vs_exact_f64"]
    return out


def fmr_polytrope(bsn, torch, steps, warmup, log, omega_frac=0.0, host_loop=True):
    """Two-level FMR self-gravitating n=1 polytrope (M=1, R=0.5, G=1) in a
    rho=1e-8 atmosphere: 128^3 base on [-2,2]^3, 128^3 fine on [-1,1]^3
    (ratio 2), isolated FFT Poisson every step, optionally in rigid rotation
    at omega_frac of breakup (the driver's overlay,
    scripts/run_sn50_fiducial.jl:421-446).  Times `steps` steps of the
    device loop (one graph per step, coarse step + first subcycle batched)
    for FP32 and FP64 stencils, and the FP64 host-driven loop (cfl_dt_fmr3d +
    fmr3d_step per step, one launch per level and stage) beside them; then
    reruns the FP32 path from the initial state to the FP64 run's end time
    for the L1 density and energy differences on both levels.
    cell-updates/s counts the fine level once per subcycle."""
    import math
    from bsn import ics
    nc, ratio, gam = 128, 2, 2.0
    dxc = 4.0 / nc
    lo, hi = 33, 96          # coarse cells covering [-1, 1]
    kw = dict(rho_floor=1e-8, P_floor=1e-10)
    U0 = bsn.state(nc, nc, nc)
    ics.polytrope_ic_3d(U0, nc, nc, nc, dxc, dxc, dxc, gam, M_star=1.0, R_star=0.5, x0=-2.0, y0=-2.0, z0=-2.0,
                        **kw)
    if omega_frac:
        ics.apply_stellar_rotation(U0, nc, nc, nc, dxc, gam, omega_frac * math.sqrt(1.0 / 0.5 ** 3),
                                   rho_thresh=2.0 * kw["rho_floor"], x0=-2.0, y0=-2.0)
    bsn.fill_ghost_3d_outflow(U0, nc, nc, nc)
    nf = (hi - lo + 1) * ratio
    units = nc ** 3 + ratio * nf ** 3

    def grid():
        return bsn.FMRGrid3D(U0.clone(), nc, nc, nc, dxc, lo, hi, lo, hi, lo, hi, ratio, gam, **kw)

    out = {"workload": "polytrope FMR 128^3 + 128^3 (ratio 2), self-gravity"
                       + (f", rigid rotation {omega_frac} of breakup" if omega_frac else ""),
           "steps": steps, "warmup": warmup, "unit": "cell-updates/s", "units_per_step": units}
    end = {}
    for prec in ("f32", "f64"):
        G = grid()
        t = 0.0
        if warmup:
            t, _ = bsn.fmr3d_run_steps(G, 0.4, n_steps=warmup, precision=prec, self_gravity=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t, _ = bsn.fmr3d_run_steps(G, 0.4, n_steps=steps, t=t, precision=prec, self_gravity=True)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[f"{prec}_batched_ms_per_step"] = ms
        out[f"{prec}_batched_value"] = units / (ms / 1e3)
        out[f"{prec}_end_time"] = t
        log(f"FMR polytrope {prec} batched: {ms:.3f} ms/step")
        if prec == "f64":
            end["f64"] = (G.Uc.clone(), G.Uf.clone())
        del G
    # FP32 against FP64 at the FP64 run's end time
    G = grid()
    t64 = out["f64_end_time"]
    _, k = bsn.fmr3d_run_steps(G, 0.4, n_steps=100 * (steps + warmup), t_end=t64, precision="f32", self_gravity=True)
    a = (slice(3, -3),) * 3
    for lev, A, B in (("coarse", G.Uc, end["f64"][0]), ("fine", G.Uf, end["f64"][1])):
        for q, nm in ((0, "rho"), (4, "E")):
            ref = B[q][a]
            out[f"f32_L1_{nm}_{lev}_vs_f64"] = float((A[q][a] - ref).abs().sum() / ref.abs().sum())
    out["accuracy_t"] = t64
    out["f32_accuracy_steps"] = k
    del G, end
    if not host_loop:
        return out
    G = grid()
    for _ in range(warmup):
        bsn.fmr3d_step(G, bsn.cfl_dt_fmr3d(G, 0.4), self_gravity=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        bsn.fmr3d_step(G, bsn.cfl_dt_fmr3d(G, 0.4), self_gravity=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out["f64_host_loop_ms_per_step"] = ms
    out["f64_host_loop_value"] = units / (ms / 1e3)
    out["speedup_f32_batched_vs_f64_host_loop"] = out["f64_host_loop_ms_per_step"] / out["f32_batched_ms_per_step"]
    log(f"FMR polytrope f64 host loop: {ms:.3f} ms/step")
    return out


def binary_nested(bsn, torch, steps, warmup, log, n=128, paths=("f64", "f32", "learned"), perturbed=False):
    """The binary-BH supernova on three nested FMR levels of n^3 (ratio 2) on
    [-8,8]^3, [-4,4]^3, [-2,2]^3: n=3 polytrope star (M=10, R=1, G=1, gamma
    4/3) with a thermal bomb E=1 in r<0.1 and two m=5 BH sinks at (+-1.5,0,0)
    on their circular orbit (sink radius 4, softening 2 finest cells), every
    level with its own initial state.  Times `steps` level-0 steps of the
    device coupled loop on the nested levels (composite gas force, FP64
    orbit, nested step with BH gravity / self-gravity / sinks on every level
    and the chains of first substeps batched per RK3 stage, accretion,
    diagnostics; one CUDA graph per step) with FP64, FP32 and learned
    stencils.  cell-updates/s counts each level once per substep (7 n^3 per
    level-0 step); the L1 of the finest level's density against FP64 is taken
    at FP64's end time (the other paths rerun from the initial state to it)."""
    import math
    from bsn import ics
    from bsn import learned as Lm
    Lm.install(*Lm.load_params())
    g, L = 4.0 / 3.0, 8.0
    lo, hi = n // 4 + 1, 3 * n // 4
    boxes = ((lo, hi, lo, hi, lo, hi, 2),) * 2
    kw = dict(rho_floor=1e-8, P_floor=1e-10)
    dx0 = 2 * L / n

    def fill(U, dx, x0, bomb=True):
        ics.polytrope_ic_3d(U, n, n, n, dx, dx, dx, g, M_star=10.0, R_star=1.0, x0=x0, y0=x0, z0=x0, **kw)
        if bomb:
            ics.thermal_bomb(U, n, n, n, dx, dx, dx, E_SN=1.0, r_bomb=0.1, x0=x0, y0=x0, z0=x0)

    U0 = bsn.state(n, n, n)
    # no level-0 cell centre lies within r < 0.1 at n = 128 (thermal_bomb! would
    # raise); the covered centre of level 0 takes the finer levels' restriction
    fill(U0, dx0, -L, bomb=2 * L / n < 0.1)
    bsn.fill_ghost_3d_outflow(U0, n, n, n)
    H0 = bsn.FMRHierarchy3D(U0, n, n, n, dx0, boxes, g, **kw)
    x0, dx = -L, dx0
    for k in range(2):
        x0, dx = x0 + (lo - 1) * dx, dx / 2
        fill(H0.levels[k + 1], dx, x0)
        H0.pairs[k].prolong_fine_ghosts()
    # every level holds the restriction of the finer ones (the invariant the
    # step keeps), so level 0's mass is the composite grid's from the start
    H0.pairs[1].restrict()
    H0.pairs[0].restrict()
    dxf = dx
    init = [U.clone() for U in H0.levels]
    del H0
    v = math.sqrt(10.0 / 3.0) / 2.0
    units = 7 * n ** 3
    out = {"workload": f"binary BH supernova, 3 nested FMR levels {n}^3 (ratio 2) on [-8,8]^3/[-4,4]^3/[-2,2]^3, "
                       "sinks + self-gravity", "steps": steps, "unit": "cell-updates/s", "units_per_step": units}
    rho_f = {}

    def fresh(prec, cap):
        U = init[0].clone()
        H = bsn.FMRHierarchy3D(U, n, n, n, dx0, boxes, g, init=False, **kw)
        for Ud, Ui in zip(H.levels[1:], init[1:]):
            Ud.copy_(Ui)
        b = [bsn.BlackHole((1.5, 0.0, 0.0), (0.0, v, 0.0), 5.0, 2 * dxf, 1e6, 4 * dxf),
             bsn.BlackHole((-1.5, 0.0, 0.0), (0.0, -v, 0.0), 5.0, 2 * dxf, 1e6, 4 * dxf)]
        rec = torch.zeros((cap, bsn.DIAG_RECORD), dtype=torch.float64, device="cuda")
        common = dict(f_sink=1.0, torque_free=True, self_gravity=True, rho_sink_min=0.0, evolve_orbit=True,
                      precision=prec, diag=rec)
        return H, b, common

    t64 = None
    E_f = {}
    for prec in paths:
        H, b, common = fresh(prec, steps + warmup)
        t = 0.0
        if warmup:
            t, _ = bsn.coupled_nested_run_steps(H, b, -L, -L, -L, 0.4, n_steps=warmup, **common)
        M_start = float(bsn.diagnostics(H.levels[0], n, n, n, dx0, dx0, dx0, -L, -L, -L, b, g)[9])
        MBH_start = sum(bh.mass for bh in b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t, k = bsn.coupled_nested_run_steps(H, b, -L, -L, -L, 0.4, n_steps=steps, t=t, **common)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[f"{prec}_device_loop_ms_per_step"] = ms
        out[f"{prec}_device_loop_value"] = units / (ms / 1e3)
        out[f"{prec}_end_time"] = t
        out[f"{prec}_mass_closure"] = mass_closure(common["diag"][k - 1].cpu().numpy(), M_start, MBH_start,
                                                   sum(bh.mass for bh in b))
        log(f"binary BH nested {prec}: {ms:.3f} ms/step, mass closure "
            f"{out[f'{prec}_mass_closure']['gas_residual_rel']:.2e}")
        if prec == "f64":
            t64 = t
            rho_f[prec] = H.levels[2][0].clone()
            E_f[prec] = H.levels[2][4].clone()
        del H
    # accuracy at equal time: the reduced-precision paths rerun to FP64's end time
    if t64 is None:
        return out
    out["accuracy_t"] = t64
    others = [p_ for p_ in paths if p_ != "f64"]
    for prec in others:
        H, b, common = fresh(prec, 1)
        common["diag"] = None
        _, k = bsn.coupled_nested_run_steps(H, b, -L, -L, -L, 0.4, n_steps=10 * (steps + warmup), t_end=t64,
                                            **common)
        out[f"{prec}_accuracy_steps"] = k
        rho_f[prec] = H.levels[2][0].clone()
        E_f[prec] = H.levels[2][4].clone()
        del H
    if perturbed:
        # the problem's own conditioning: FP64 again from an initial density
        # perturbed by 1e-15 relative, to the same time
        H, b, common = fresh("f64", 1)
        common["diag"] = None
        gen = torch.Generator(device="cuda").manual_seed(7)
        for U in H.levels:
            U[0].mul_(1.0 + 1e-15 * torch.randn(U[0].shape, device="cuda", dtype=torch.float64, generator=gen))
        _, k = bsn.coupled_nested_run_steps(H, b, -L, -L, -L, 0.4, n_steps=10 * (steps + warmup), t_end=t64,
                                            **common)
        out["f64_perturbed_accuracy_steps"] = k
        rho_f["f64_perturbed"] = H.levels[2][0].clone()
        E_f["f64_perturbed"] = H.levels[2][4].clone()
        others = others + ["f64_perturbed"]
        del H
    a = (slice(3, -3),) * 3
    ref = rho_f["f64"][a]
    refE = E_f["f64"][a]
    for prec in others:
        out[f"{prec}_L1_rho_finest_vs_f64"] = float((rho_f[prec][a] - ref).abs().sum() / ref.abs().sum())
        out[f"{prec}_L1_E_finest_vs_f64"] = float((E_f[prec][a] - refE).abs().sum() / refE.abs().sum())
        if f"{prec}_device_loop_ms_per_step" in out:
            out[f"speedup_{prec}_vs_f64"] = (out["f64_device_loop_ms_per_step"]
                                             / out[f"{prec}_device_loop_ms_per_step"])
    return out


def poisson_solves(bsn, torch, peak_fp, hbm, log, n=128, reps=20):
    """The isolated Poisson solve on an n^3 grid ((2n)^3 zero-padded; the
    self-gravity solve of the FMR and binary-BH workloads), FP64 and FP32
    transforms, against the standard R2C/C2R solve's figures: 3 passes x
    read+write of (2n)^3/2 complex doubles plus the Green's function read,
    and 5 M log2 M flops per complex transform of M = (2n)^3 points (half of
    that for a real one; one forward and one inverse per solve)."""
    M = (2 * n) ** 3
    alg_bytes = 3 * 2 * M / 2 * 16 + (n + 1) ** 3 * 8
    flops = 2 * 0.5 * 5 * M * math.log2(M)
    g = torch.Generator(device="cuda").manual_seed(1)
    rho = bsn.active_grid(n, n, n)   # column-major (nx, ny, nz)
    rho.copy_(torch.rand((n, n, n), device="cuda", dtype=torch.float64, generator=g) + 0.1)
    out = {"workload": f"isolated Poisson solve {n}^3 ({2 * n}^3 padded)", "alg_bytes_per_solve": alg_bytes,
           "flops_per_solve": flops}
    for prec in ("f64", "f32"):
        for _ in range(3):
            bsn.solve_poisson_isolated(rho, n, n, n, 0.01, 0.01, 0.01, precision=prec)
        torch.cuda.synchronize()
        # the reps replayed from one CUDA graph, so the figure is the solves'
        # device time, not the host's call rate (a 0.1 ms solve is shorter
        # than a slow host's Python call); eager calls if capture fails
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        graph = None
        try:
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                for _ in range(reps):
                    bsn.solve_poisson_isolated(rho, n, n, n, 0.01, 0.01, 0.01, precision=prec)
            graph.replay()
            torch.cuda.synchronize()
        except Exception as e:   # noqa: BLE001 -- the eager loop below times it instead
            log(f"Poisson {prec}: graph capture failed ({e}); timing eager calls")
            graph = None
            torch.cuda.synchronize()
        e0.record()
        if graph is not None:
            graph.replay()
        else:
            for _ in range(reps):
                bsn.solve_poisson_isolated(rho, n, n, n, 0.01, 0.01, 0.01, precision=prec)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = alg_bytes / (ms / 1e3) / 1e9
        tf = flops / (ms / 1e3) / 1e12
        pk = peak_fp["f64"] if prec == "f64" else max(peak_fp["f32"], peak_fp["f32x2"])
        out[prec] = {"ms_per_solve": ms, "GB/s": gbs, "hbm_frac": gbs / hbm, "TFLOP/s": tf, "fp_frac": tf / pk,
                     "timing": "one CUDA graph of the reps" if graph is not None else "eager calls"}
        del graph
        log(f"Poisson {n}^3 {prec}: {ms:.3f} ms per solve")
    return out


def coupled_binary(bsn, torch, steps, warmup, log, n=128):
    """Binary-BH supernova physics on a uniform grid: n=3 polytrope star
    (M=10, R=1, G=1, gamma 4/3) at the origin with a thermal bomb E=1 in
    r<0.1, two m=5 BH sinks on the circular orbit of separation 3 in z=0
    (sink radius 4 cells, softening 2 cells), self-gravity, n^3 on [-4,4]^3.
    Times `steps` steps of the device coupled loop (gas force, FP64 N-body
    orbit, stages with BH gravity / self-gravity / sinks, accretion, per-step
    diagnostics; one CUDA graph per step) for FP32 and FP64 stencils, and the
    host-driven FP64 loop (cfl_dt_3d + coupled_step per step) beside them."""
    import math
    from bsn import ics
    L, g = 4.0, 4.0 / 3.0
    dx = 2 * L / n
    kw = dict(rho_floor=1e-8, P_floor=1e-10)
    U0 = bsn.state(n, n, n)
    ics.polytrope_ic_3d(U0, n, n, n, dx, dx, dx, g, M_star=10.0, R_star=1.0, x0=-L, y0=-L, z0=-L, **kw)
    ics.thermal_bomb(U0, n, n, n, dx, dx, dx, E_SN=1.0, r_bomb=0.1, x0=-L, y0=-L, z0=-L)
    v = math.sqrt(10.0 / 3.0) / 2.0

    def bhs():
        return [bsn.BlackHole((1.5, 0.0, 0.0), (0.0, v, 0.0), 5.0, 2 * dx, 1e6, 4 * dx),
                bsn.BlackHole((-1.5, 0.0, 0.0), (0.0, -v, 0.0), 5.0, 2 * dx, 1e6, 4 * dx)]

    out = {"workload": f"binary BH supernova, uniform {n}^3 on [-4,4]^3, sinks + self-gravity", "steps": steps,
           "unit": "cell-updates/s"}
    common = dict(f_sink=1.0, torque_free=True, self_gravity=True, rho_sink_min=0.0, evolve_orbit=True, **kw)
    for prec in ("f32", "f64"):
        U, b = U0.clone(), bhs()
        rec = torch.zeros((steps + warmup, bsn.DIAG_RECORD), dtype=torch.float64, device="cuda")
        t, _ = bsn.coupled_run_steps(U, b, n, n, n, dx, -L, -L, -L, g, 0.4, n_steps=warmup, precision=prec,
                                     diag=rec, **common)
        M_start = float(bsn.diagnostics(U, n, n, n, dx, dx, dx, -L, -L, -L, b, g)[9])
        MBH_start = sum(bh.mass for bh in b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bsn.coupled_run_steps(U, b, n, n, n, dx, -L, -L, -L, g, 0.4, n_steps=steps, t=t, precision=prec, diag=rec,
                              **common)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[f"{prec}_device_loop_ms_per_step"] = ms
        out[f"{prec}_device_loop_value"] = n ** 3 / (ms / 1e3)
        out[f"{prec}_mass_closure"] = mass_closure(rec[steps - 1].cpu().numpy(), M_start, MBH_start,
                                                   sum(bh.mass for bh in b))
        log(f"binary BH {prec} device loop: {ms:.3f} ms/step, mass closure "
            f"{out[f'{prec}_mass_closure']['gas_residual_rel']:.2e}")
    U, b = U0.clone(), bhs()
    t = 0.0
    for k in range(warmup + steps):
        if k == warmup:
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        dt = bsn.cfl_dt_3d(U, n, n, n, dx, dx, dx, g, 0.4)
        bsn.coupled_step(U, b, dt, t, n, n, n, dx, -L, -L, -L, g, 1.0, kw["rho_floor"], kw["P_floor"], True, True,
                         0.0, 0.0)
        t += dt
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out["f64_host_loop_ms_per_step"] = ms
    out["f64_host_loop_value"] = n ** 3 / (ms / 1e3)
    out["speedup_f32_device_vs_f64_host_loop"] = ms / out["f32_device_loop_ms_per_step"]
    log(f"binary BH f64 host loop: {ms:.3f} ms/step")
    return out


# Algorithmic floating-point operations per active cell per RK3 step of the
# reference scheme (every +, -, *, /, sqrt and comparison of euler3d_step!
# counted once; 3647 add, 4426 mul, 768 div, 18 sqrt, 1163 cmp), counted by
# `python oracle/count_flops.py` on the Sedov 128^3 state at t = 0.025, the
# timed workload's state at half the resolution (Sod 64^3: 10111).
FLOPS_PER_CELL_STEP = 10023.4


def fp_pipe(prec, ms, ms_other, cell_steps, peak):
    """FP-pipe fraction of every path's whole step: FLOPS_PER_CELL_STEP per
    cell-step over the measured FMA peak of its arithmetic (FP64; FP32 with
    the better of scalar and packed f32x2 FMA)."""
    out = {"flops_per_cell_step": FLOPS_PER_CELL_STEP, "unit": "TFLOP/s",
           "peaks_measured": {k: round(v, 2) for k, v in peak.items()},
           "note": "operations of the reference scheme (oracle count), not instructions issued: a division "
                   "or square root counts one but costs several pipe operations"}
    for p_, m_ in [(prec, ms)] + list(ms_other.items()):
        a = FLOPS_PER_CELL_STEP * cell_steps / (m_ / 1e3) / 1e12
        pk = peak["f64"] if p_ == "f64" else max(peak["f32"], peak["f32x2"])
        out[p_] = {"achieved": a, "peak": pk, "frac": a / pk}
    return out


def run_bsn(args, rank, world):
    import numpy as np
    import torch
    import bsn

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
    n = args.n
    U0, dx = sedov_host(n)
    log(f"Sedov {n}^3 initial state built")
    ncell = n ** 3
    kw = dict(rho_floor=1e-6, P_floor=1e-6)

    def steps(U, k, prec, t=0.0, t_end=0.0):
        return bsn.run_steps(U, n, n, n, dx, dx, dx, GAMMA, CFL, n_steps=k, t=t, t_end=t_end, precision=prec,
                             **kw)

    # the timed steps start from the blast half-way to t = 0.05 (FP64 run),
    # so every path sees the mix of quiescent, smooth and shocked stencils of
    # the run rather than the nearly empty initial grid
    Ud = torch.from_numpy(U0).cuda()
    t_mid, k_mid = steps(Ud, 1_000_000, "f64", 0.0, T_MID)
    log(f"FP64 run to t={t_mid:.4g}: {k_mid} steps")
    U_mid = Ud.cpu().numpy()

    def timed(prec, k):
        """K device-resident RK3 steps (dt on the device, one graph per step)."""
        U = Ud.clone()
        t, _ = steps(U, args.warmup, prec, t_mid)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = bsn.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        steps(U, k, prec, t)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        return ms, bsn.launch_count() - l0

    prec = args.path
    others = [p_ for p_ in ("learned", "f32", "f64") if p_ != prec]
    if "learned" in (prec,) + tuple(others):
        from bsn import learned as LW
        LW.install(*LW.load_params())
    if args.no_tma:
        bsn.set_tma(False)
    if args.tile >= 0:
        for p_ in ("f32", "f64", "learned"):
            bsn.set_tile(p_, min(args.tile, bsn.tile_variants(p_) - 1))
    with ClockSampler(local) as clk:
        ms, launches = timed(prec, args.steps)
    log(f"{prec}: {ms / args.steps:.3f} ms/step")
    ms_other = {}
    for p_ in others:
        ms_other[p_] = timed(p_, args.steps)[0]
        log(f"{p_}: {ms_other[p_] / args.steps:.3f} ms/step")
    value = world * ncell * args.steps / (ms / 1e3)

    # roofline of the dominant kernel: stage-kernel launches timed with CUDA
    # events around each launch (per-step entry point, same kernels)
    kname = {"f32": "stage_kernel_f32", "f64": "stage_kernel", "learned": "stage_kernel_learned"}[prec]
    step_fn = {"f32": bsn.euler3d_step_f32, "f64": bsn.euler3d_step, "learned": bsn.euler3d_step_learned}[prec]
    Up = Ud.clone()
    dt0 = bsn.cfl_dt_3d(Up, n, n, n, dx, dx, dx, GAMMA, CFL)
    step_fn(Up, n, n, n, dx, dx, dx, dt0, GAMMA, **kw)
    bsn.set_profiling(True)
    for _ in range(3):
        step_fn(Up, n, n, n, dx, dx, dx, dt0, GAMMA, **kw)
    tot, cnt = bsn.kernel_time(kname)
    if prec != "learned":   # the stage kernel with TMA staging, where the grid allows it
        t_, c_ = bsn.kernel_time(kname + "_tma")
        if c_:
            tot, cnt, kname = tot + t_, cnt + c_, kname + "_tma"
    if prec == "learned":   # a learned stage is a screening launch plus the learned launch
        tot += bsn.kernel_time("stage_kernel_learned_screen")[0]
        kname = "stage_kernel_learned_screen + stage_kernel_learned"
    bsn.set_profiling(False)
    t_stage = tot / max(cnt, 1) / 1e3
    alg_bytes = 40 * 8 * ncell / 3.0     # 40 FP64 state words per cell per RK3 step, 3 stage launches
    # DRAM bytes of one stage-1 launch (learned: its screening and learned launches) from an ncu
    # capture at 128^3 (t = 0.025), scaled by the cell count (profiles/stage_kernel_*_sedov128_ncu.md)
    traffic_128 = {"learned": 134.1e6, "f32": 133.7e6, "f64": 133.1e6}.get(prec)
    traffic = traffic_128 * ncell / 128 ** 3 if traffic_128 else None
    hbm, hbm_kind = peaks()
    achieved = alg_bytes / t_stage / 1e9
    tile = bsn.get_tile(n, n, n, prec)
    del Up

    log(f"roofline: {kname} {t_stage * 1e3:.3f} ms per launch")
    # FP-pipe fraction of each path over its whole step: the reference scheme's
    # operations per cell-step against this GPU's measured FMA throughput
    peak_fp = {k_: bsn.fp_peak(k_) for k_ in ("f64", "f32", "f32x2")}
    log("measured FMA peaks (TFLOP/s): " + ", ".join(f"{k_} {v_:.1f}" for k_, v_ in peak_fp.items()))
    acc = accuracy(bsn, torch, U0, n, dx, kw) if not args.no_accuracy else None
    fmr = fmr_polytrope(bsn, torch, max(5, min(args.steps, 20)), args.warmup, log) if not args.no_fmr else None
    coupled = coupled_binary(bsn, torch, max(5, min(args.steps, 20)), args.warmup, log) if not args.no_fmr else None
    nested = binary_nested(bsn, torch, max(5, min(args.steps, 20)), args.warmup, log) if not args.no_fmr else None
    poisson = poisson_solves(bsn, torch, peak_fp, hbm, log) if not args.no_fmr else None

    # e2e: host-buffer path -- pinned host state -> device, one CFL-limited
    # RK3 step through the public entry point, device -> host, every step
    Uh = torch.from_numpy(U_mid.copy(order="F")).pin_memory()
    Ue = torch.empty_like(Ud)
    nbytes = Uh.numel() * 8
    for _ in range(2):
        Ue.copy_(Uh, non_blocking=True)
        steps(Ue, 1, prec, t_mid)
        Uh.copy_(Ue, non_blocking=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    k_e2e = max(2, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(k_e2e):
        Ue.copy_(Uh, non_blocking=True)
        steps(Ue, 1, prec, t_mid)
        Uh.copy_(Ue, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    if dist:
        tt = torch.tensor([ms_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_e2e = float(tt.item())
    e2e = world * ncell * k_e2e / (ms_e2e / 1e3)

    cpu = None
    if rank == 0 and not args.no_cpu:
        # the same sample as the reference arm: the timed state's slab, all threads
        threads = os.cpu_count() or 1
        nz = max(4, min(n, CPU_SLAB))
        rate, el, k = cpu_reference_rate(cpu_slab(U_mid, n, nz), n, dx, threads, 1, min_seconds=12.0)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": threads, "kind": "port",
               "sample": f"{k} RK3 steps (cfl_dt_3d + euler3d_step!, oracle, FP64) of a {n}x{n}x{nz} z-slab "
                         f"through the blast centre of Sedov {n}^3 at t={t_mid:.4g}, {el:.1f} s"}
    if rank == 0:
        desc = {"f32": "FP32 stencils/fluxes, FP64 state and RK3 accumulation",
                "f64": "FP64, bit-identical to the reference CPU path",
                "learned": "FP32 stencils/fluxes with learned WENO weights (BF16 tensor-core MLP, WENO5-Z "
                           "fallback at flagged stencils), FP64 state and RK3 accumulation"}
        compare = {}
        for p_, m_ in ms_other.items():
            v_ = world * ncell * args.steps / (m_ / 1e3)
            compare[f"{p_}_value"] = v_
            compare[f"{p_}_ms_per_step"] = m_ / args.steps
            compare[f"speedup_vs_{p_}"] = value / v_
        line = {
            "metric": METRIC,
            "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == "f64" else ("f32+bf16" if prec == "learned" else "f32"), "data": "synthetic (Sedov initial condition, sedov_ic_3d!)",
            "config": {"workload": f"sedov{n}^3", "grid": [n, n, n], "path": desc[prec],
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "tile": list(tile), "time_loop": "device-resident dt, one CUDA graph per step",
                       "staging": "TMA tensor copies" if bsn.get_tile_tma(n, n, n, prec) else "per-thread loads",
                       "timed_from": f"Sedov state at t={T_MID} (FP64 run from the initial condition)",
                       "l2": f"state {Ud.numel() * 8 / 1e6:.0f} MB per array > 126 MB L2 (no flush needed)"},
            "compare": compare,
            "accuracy": acc,
            "fmr": fmr,
            "coupled": coupled,
            "coupled_nested": nested,
            "poisson": poisson,
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "peak_kind": hbm_kind,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                         "traffic_note": "DRAM read+write of one stage-1 launch, ncu at 128^3 scaled by cells",
                         "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": t_stage * 1e3,
                         "note": "the fused stencil kernel is FP-pipe bound (FP32/FP64), not HBM bound; "
                                 "HBM fraction of the algorithmic 40 words/cell-step"},
            "fp_pipe": fp_pipe(prec, ms, ms_other, ncell * world * args.steps, peak_fp),
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": k_e2e},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bsn", choices=["bsn", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--path", default="learned", choices=["learned", "f32", "f64"],
                    help="stencil path of the headline (the others are timed beside it)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the Sedov-to-t=0.05 accuracy runs of the three paths")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-fmr", action="store_true",
                    help="skip the two-level FMR polytrope and binary-BH coupled-loop timings")
    ap.add_argument("--workload", default="sedov", choices=["sedov", "binary_nested", "polytrope_fmr", "poisson", "slab",
                                                     "slab_fmr"],
                    help="binary_nested: time only the binary-BH supernova on three nested FMR levels; "
                         "polytrope_fmr: only the two-level self-gravitating polytrope; "
                         "poisson: only the isolated Poisson solve at 128^3, --steps solves per precision; "
                         "slab: Sedov --n^3 split into z-slabs over the torchrun ranks (bsn.shard)")
    ap.add_argument("--full", action="store_true",
                    help="with --workload: run the workload's stated length from its initial state (polytrope "
                         "200 steps, binary 1000 steps, no warm-up) instead of --steps")
    ap.add_argument("--omega", type=float, default=0.0,
                    help="--workload polytrope_fmr: rigid rotation as a fraction of breakup (e.g. 0.2)")
    ap.add_argument("--paths", default="f64,f32,learned",
                    help="stencil paths of --workload binary_nested (comma-separated)")
    ap.add_argument("--no-tma", action="store_true",
                    help="stage the stencil tiles with the plain per-thread loader instead of TMA copies")
    ap.add_argument("--tile", type=int, default=-1,
                    help="force this stage-kernel tile variant (index into each precision's table, clamped to "
                         "its last entry) for the Sedov and FMR workloads (default: autotune)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "poisson":
        import torch
        import bsn
        peak_fp = {k_: bsn.fp_peak(k_) for k_ in ("f64", "f32", "f32x2")}
        out = poisson_solves(bsn, torch, peak_fp, peaks()[0], log, reps=max(1, args.steps))
        print(json.dumps(out), flush=True)
        return
    if args.workload in ("binary_nested", "polytrope_fmr"):
        import torch
        import bsn
        if args.tile >= 0:
            for p_ in ("f32", "f64", "learned"):
                bsn.set_tile(p_, min(args.tile, bsn.tile_variants(p_) - 1))
        if args.workload == "binary_nested":
            paths = tuple(p_ for p_ in args.paths.split(",") if p_)
            steps, warmup = (1000, 0) if args.full else (args.steps, args.warmup)
            out = binary_nested(bsn, torch, steps, warmup, log, paths=paths, perturbed=args.full)
        else:
            steps, warmup = (200, 0) if args.full else (args.steps, args.warmup)
            out = fmr_polytrope(bsn, torch, steps, warmup, log, omega_frac=args.omega, host_loop=not args.full)
        out["full_length"] = bool(args.full)
        print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload in ("slab", "slab_fmr"):
            out = (slab_sedov if args.workload == "slab" else slab_fmr)(args, rank, world, log)
            if rank == 0:
                print(json.dumps(out), flush=True)
            return
        run_bsn(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
