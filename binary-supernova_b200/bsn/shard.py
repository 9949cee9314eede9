"""Z-slab domain decomposition of the uniform-grid update across ranks (one
process per GPU; torch.distributed over NCCL between GPUs, gloo on CPU).

Rank r of W holds z-planes [r nz, (r + 1) nz) of an nx x ny x (W nz) grid,
with the usual three ghost planes on every side.  One SSP-RK3 step is the
reference's euler3d_step! (src/euler3d.jl:220-260) with a halo exchange in
front of every right-hand side:

  1. fill the slab's ghosts by the boundary condition (x, then y, then z);
  2. replace the z ghost planes that face a neighbouring rank by that rank's
     three boundary planes (send/recv), floored as the reference floors them
     before its fluxes where they are active cells of the global grid (their
     x/y ghost columns are the copies its ghost fill made; across a periodic
     wrap they are its ghost planes, filled before the floors, and stay raw);
  3. euler3d_rhs! without its own ghost fill (it floors the slab's active
     cells and computes the fluxes with the ghosts as they stand);
  4. the stage combination and floors of euler3d_step!.

The active cells of every slab are then bit-identical to the same cells of
the undivided grid (FP64), and dt = min over ranks of each slab's
cfl_dt_3d equals the undivided grid's (IEEE division is monotone).  The
exchange per stage is 3 planes x 5 variables x (nx+6)(ny+6) words each way.

The operations of steps 1, 3 and 4 come from an `ops` object (`DeviceOps`:
this library's C ABI on CUDA tensors), so the exchange logic is the same
whatever computes the stages.

`poisson_isolated` is the self-gravity solve on the same slabs: local x/y
transforms, an all-to-all transpose to z lines, the z convolution with the
global grid's Green's function, and the transpose back; on the device it is
bit-identical to the undivided bsn_solve_poisson_isolated_f64.

`coupled_step` is the production step (coupled_step!,
scripts/run_sn50_fiducial.jl:756-818) on the slabs: BH gravity and the sink
sources per cell with the global plane index, the gas force on the BHs as an
all-gather of the ranks' compensated partial sums merged in rank order, and
accrete! as an ordered gather of the sink sphere's cell terms; with the orbit
frozen it is the undivided step bit for bit.

Two-level FMR over the same slabs (the refined patch on one rank) is in
`bsn.shard_fmr`.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

NG = 3


@dataclass
class Slab:
    """This rank's part of the global z range and its neighbours (None at an
    outflow boundary; periodic z wraps around)."""
    nx: int
    ny: int
    nz: int           # planes held by this rank
    rank: int
    world: int
    bc: str = "outflow"

    @classmethod
    def split(cls, nx, ny, nz_global, rank, world, bc="outflow"):
        if world < 1 or not 0 <= rank < world:
            raise ValueError(f"rank {rank} of {world}")
        if nz_global % world:
            raise ValueError(f"{nz_global} z-planes do not split evenly over {world} ranks")
        nz = nz_global // world
        if nz < NG:
            raise ValueError(f"{nz} planes per rank: at least {NG} are needed for the 3-plane halo")
        if bc not in ("outflow", "periodic"):
            raise ValueError(f"unknown boundary condition {bc!r}")
        return cls(nx, ny, nz, rank, world, bc)

    @property
    def k0(self) -> int:
        """first global active plane of this slab"""
        return self.rank * self.nz

    @property
    def lo(self):
        if self.rank > 0:
            return self.rank - 1
        return self.world - 1 if (self.bc == "periodic" and self.world > 1) else None

    @property
    def hi(self):
        if self.rank < self.world - 1:
            return self.rank + 1
        return 0 if (self.bc == "periodic" and self.world > 1) else None


def _zmajor(U):
    """(Z, Y, X, 5) C-contiguous view of a state array in the reference layout
    (a torch tensor, or a Fortran-ordered numpy array)."""
    if isinstance(U, torch.Tensor):
        V = U.permute(3, 2, 1, 0)
    else:
        V = torch.from_numpy(U.T)
    assert V.is_contiguous()
    return V


def exchange(U, slab: Slab, ops, group=None, rho_floor=0.0, P_floor=0.0, gamma=1.4):
    """Step 2 above: the z ghost planes facing other ranks from those ranks'
    boundary planes, floored."""
    if slab.world == 1:
        return
    import torch.distributed as dist
    V = _zmajor(U)
    nz = slab.nz
    ops_list, recv = [], []
    # tag 0: my top planes go up (to hi's bottom ghosts); tag 1: my bottom planes go down
    # planes from an interior neighbour are active cells of the global grid and
    # are floored; across the periodic wrap they are the global grid's ghost
    # planes, which the reference fills (unfloored) before it floors
    if slab.hi is not None:
        ops_list.append(dist.P2POp(dist.isend, V[nz:nz + NG].clone(), slab.hi, group, tag=0))
        buf = torch.empty_like(V[NG + nz:])
        ops_list.append(dist.P2POp(dist.irecv, buf, slab.hi, group, tag=1))
        recv.append((slice(NG + nz, 2 * NG + nz), buf, slab.rank < slab.world - 1))
    if slab.lo is not None:
        ops_list.append(dist.P2POp(dist.isend, V[NG:2 * NG].clone(), slab.lo, group, tag=1))
        buf = torch.empty_like(V[:NG])
        ops_list.append(dist.P2POp(dist.irecv, buf, slab.lo, group, tag=0))
        recv.append((slice(0, NG), buf, slab.rank > 0))
    for req in dist.batch_isend_irecv(ops_list):
        req.wait()
    for sl, buf, interior in recv:
        V[sl] = ops.floor_planes(buf, slab.nx, slab.ny, rho_floor, P_floor, gamma) if interior else buf


def _allreduce_min(x: float, ops, group, world):
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=ops.device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())


def cfl_dt(U, slab: Slab, dx, dy, dz, gamma, cfl, ops, group=None) -> float:
    """cfl_dt_3d of the global grid: the min over ranks."""
    return _allreduce_min(ops.cfl(U, slab.nx, slab.ny, slab.nz, dx, dy, dz, gamma, cfl), ops, group, slab.world)


def euler3d_step(U, slab: Slab, dx, dy, dz, dt, gamma, ops, group=None, rho_floor=0.0, P_floor=0.0,
                 self_gravity=False, precision="f64"):
    """euler3d_step! (src/euler3d.jl:220-260) on this rank's slab, with the
    halo exchange before every right-hand side; with self_gravity, the
    self-gravity source of the global grid after each right-hand side, as
    coupled_step! adds it (scripts/run_sn50_fiducial.jl:756-818, no BHs).
    Self-gravity needs outflow boundaries: the isolated solve does not wrap,
    and the reference runs it only with outflow (coupled_step!)."""
    if self_gravity and slab.bc != "outflow":
        raise ValueError("self_gravity needs bc='outflow': the isolated Poisson solve has no periodic form")
    _rk3(U, slab, dx, dy, dz, dt, gamma, ops, group, rho_floor, P_floor, None, self_gravity, precision)


class StageSources:
    """The sources coupled_step! adds after each right-hand side on a slab:
    BH gravity of `bhs`, the sinks of bhs[:nsink], and (filled per stage by
    _rk3) the self-gravity potential with its neighbouring planes."""

    def __init__(self, bhs=(), nsink=0, f_sink=1.0, torque_free=True, rho_sink_min=0.0, x0=0.0, y0=0.0, z0=0.0):
        self.bhs, self.nsink, self.f_sink, self.torque_free = list(bhs), nsink, f_sink, torque_free
        self.rho_sink_min, self.x0, self.y0, self.z0 = rho_sink_min, x0, y0, z0
        self.phi = self.phi_lo = self.phi_hi = None


def _rk3(U, slab: Slab, dx, dy, dz, dt, gamma, ops, group, rho_floor, P_floor, src, self_gravity, precision):
    """The three stages of euler3d_step! on the slab, each one `ops.stage`
    (on the device: one fused launch) after the ghost fill and the halo
    exchange of its input; the stage inputs and outputs alternate (a copy of
    U) -> A -> B -> U, with U^n = U in every combination.  With self-gravity the potential of the stage input's floored
    density (the density euler3d_rhs! leaves before add_self_gravity_source!)
    is solved over the slabs first."""
    nx, ny, nz = slab.nx, slab.ny, slab.nz
    # stage 1 reads a copy of U, whose ghosts the fill and the exchange may
    # change: U^n's own ghost cells enter the final combination unchanged
    C, A, B = ops.copy(U), ops.zeros_like(U), ops.zeros_like(U)
    ins, outs = (C, A, B), (A, B, U)
    if self_gravity and src is None:
        src = StageSources()
    for s in range(3):
        Uin = ins[s]
        ops.fill(Uin, nx, ny, nz, slab.bc)
        exchange(Uin, slab, ops, group, rho_floor, P_floor, gamma)
        if self_gravity:
            rho = ops.active_rho_floored(Uin, nx, ny, nz, rho_floor)
            src.phi = poisson_isolated(rho, slab, dx, dy, dz, ops, group)
            src.phi_lo, src.phi_hi = _phi_neighbours(src.phi, slab, group)
        ops.stage(outs[s], Uin, U, s + 1, slab, dx, dy, dz, dt, gamma, rho_floor, P_floor, src, precision)


# ---------------------------------------------------------------------------
# coupled_step! (scripts/run_sn50_fiducial.jl:756-818) over z-slabs
#
# The per-cell sources (BH gravity, sinks) take the global cell index (k0),
# so they are the undivided grid's bit for bit.  The two grid sums become
# collectives: gas_force_on_bh is each rank's compensated partial sum,
# gathered and merged in rank order (the same force on every rank, within
# the whole-grid sum's rounding of the reference's sequential sum), and
# accrete! gathers the terms of the sink sphere's cells from the ranks whose
# slab meets it, in the reference's (k, j, i) order, and adds them in that
# order on every rank (the undivided accrete! bit for bit).


def _gather_rows(x, world, group, device):
    """all-gather of one float64 vector per rank -> (world, len) numpy, rank order."""
    import numpy as np
    if world == 1:
        return np.asarray(x, dtype=np.float64).reshape(1, -1)
    import torch.distributed as dist
    t = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=device)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    return torch.stack(out).cpu().numpy()


def gas_force(U, slab: Slab, bh, dx, dy, dz, x0, y0, z0, ops, group=None):
    """gas_force_on_bh (src/gravity_bh.jl:91-113) of the global grid on every rank."""
    from . import api
    pairs = ops.gas_force_pairs(U, slab.nx, slab.ny, slab.nz, dx, dy, dz, bh, x0, y0, z0, slab.k0)
    return api.merge_force_pairs(_gather_rows(pairs, slab.world, group, ops.device))


def _slab_box_cells(box, slab: Slab, rank):
    ilo, ihi, jlo, jhi, klo, khi = box
    k0 = rank * slab.nz
    kl, kh = max(klo, k0), min(khi, k0 + slab.nz - 1)
    return max(0, ihi - ilo + 1) * max(0, jhi - jlo + 1) * max(0, kh - kl + 1)


def accrete(bh, U, slab: Slab, dx, dy, dz, x0, y0, z0, dt, ops, group=None, *, f_sink=1.0, rho_sink_min=0.0):
    """accrete! (src/sinks.jl:74-109) of the global grid: the terms of the
    sink box's cells, gathered from the ranks in rank order (each rank's
    count follows from the box, so only the ranks whose slab meets it send
    anything), added in the reference's order on every rank."""
    import numpy as np
    from . import api
    box = api.sink_box(bh, slab.nx, slab.ny, slab.nz * slab.world, dx, dy, dz, x0, y0, z0)
    counts = [_slab_box_cells(box, slab, r) for r in range(slab.world)]
    terms = ops.sink_terms(U, slab.nx, slab.ny, slab.nz, dx, dy, dz, x0, y0, z0, slab.k0, bh, dt, box, f_sink,
                           rho_sink_min)
    assert terms.shape == (counts[slab.rank], 4)
    if slab.world > 1 and max(counts) > 0:
        pad = np.zeros((max(counts), 4))
        pad[:len(terms)] = terms
        rows = _gather_rows(pad.reshape(-1), slab.world, group, ops.device).reshape(slab.world, -1, 4)
        terms = np.concatenate([rows[r, :counts[r]] for r in range(slab.world)])
    api.accrete_from_terms(bh, terms)


def coupled_step(U, bhs, slab: Slab, dt, t, dx, x0, y0, z0, gamma, ops, group=None, *, f_sink=1.0,
                 rho_floor=0.0, P_floor=0.0, torque_free=True, self_gravity=False, t_bh2_sink_on=0.0,
                 rho_sink_min=0.0, evolve_orbit=True, precision="f64"):
    """coupled_step! (scripts/run_sn50_fiducial.jl:756-818) on this rank's slab
    of the global grid (cubic cells dx, outflow boundaries): the gas force on
    every BH with the driver's non-finite / 1e3 guard, nbody_step!, the three
    stages with BH gravity, optional self-gravity and the sinks (only the first
    BH's before t_bh2_sink_on), then accrete! of the active sinks.  `bhs`
    (bsn_bh, the same on every rank) is updated in place; returns F_gas."""
    import math
    import numpy as np
    from . import api
    if slab.bc != "outflow":
        raise ValueError("coupled_step runs with bc='outflow'")
    nbh = len(bhs)
    nsink = min(1, nbh) if t < t_bh2_sink_on else nbh
    F = np.zeros((nbh, 3))
    for i, bh in enumerate(bhs):
        f = gas_force(U, slab, bh, dx, dx, dx, x0, y0, z0, ops, group)
        fin = all(math.isfinite(v) for v in f)
        if fin and not math.sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]) > 1e3:
            F[i] = f
    if evolve_orbit and nbh > 0 and all(math.isfinite(v) for b in bhs for v in (*b.pos, *b.vel)):
        api.nbody_step(bhs, dt, F)
    src = StageSources(bhs, nsink, f_sink, torque_free, rho_sink_min, x0, y0, z0)
    _rk3(U, slab, dx, dx, dx, dt, gamma, ops, group, rho_floor, P_floor, src, self_gravity, precision)
    for i in range(nsink):
        accrete(bhs[i], U, slab, dx, dx, dx, x0, y0, z0, dt, ops, group, f_sink=f_sink, rho_sink_min=rho_sink_min)
    return F


def run_steps(U, slab: Slab, dx, dy, dz, gamma, cfl, ops, *, n_steps, t=0.0, t_end=0.0, group=None,
              rho_floor=0.0, P_floor=0.0, self_gravity=False, precision="f64"):
    """The driver loop `dt = cfl_dt_3d; dt = min(dt, t_end - t); euler3d_step!;
    t += dt` over the slabs (every rank takes the same dts); returns (t, steps)."""
    if self_gravity and slab.bc != "outflow":
        raise ValueError("self_gravity needs bc='outflow': the isolated Poisson solve has no periodic form")
    steps = 0
    while steps < n_steps and (t_end <= 0.0 or t < t_end):
        dt = cfl_dt(U, slab, dx, dy, dz, gamma, cfl, ops, group)
        if t_end > 0.0:
            dt = min(dt, t_end - t)
        if not dt > 0.0:
            raise FloatingPointError(f"time step collapsed to {dt} at t = {t}")
        euler3d_step(U, slab, dx, dy, dz, dt, gamma, ops, group, rho_floor, P_floor, self_gravity, precision)
        t += dt
        steps += 1
    return t, steps


# ---------------------------------------------------------------------------
# solve_poisson_isolated (src/self_gravity.jl:35-76) over z-slabs
#
# The zero-padded convolution transforms x and y within each z-plane, so a
# rank does those for its own planes; the z transform needs whole z lines, so
# the spectrum is transposed (one all-to-all): rank r receives every rank's
# planes for its share [b_r, b_{r+1}) of the 2ny y frequencies, convolves
# those lines with the Green's function of the global grid, and a second
# all-to-all returns each rank's planes.  Per rank and solve the exchange is
# 2 x (nx+1) x 2ny x nzl complex doubles each way (minus the share it keeps).


def ky_shares(ny: int, world: int):
    """[b_r, b_{r+1}) of the 2ny y frequencies that rank r convolves along z."""
    N2 = 2 * ny
    return [(r * N2 // world, (r + 1) * N2 // world) for r in range(world)]


class SlabPoisson:
    """The three local phases of the distributed solve for one rank; the
    caller moves the pieces between them (`poisson_isolated` does it with
    all-to-alls, a one-device emulation by hand)."""

    def __init__(self, slab: Slab, dx, dy, dz, ops):
        self.slab, self.dx, self.dy, self.dz, self.ops = slab, dx, dy, dz, ops
        self.ky = ky_shares(slab.ny, slab.world)
        self.nkx = slab.nx + 1

    def forward(self, rho):
        """x, y transforms of this slab's density; the piece for each rank r
        is its ky share of the slab's planes, (nzl, nky_r, nx+1)."""
        s = self.slab
        W2 = self.ops.poisson_forward(rho, s.nx, s.ny, s.nz)
        return [W2[:, a:b].contiguous() for a, b in self.ky]

    def forward_shapes(self):
        a, b = self.ky[self.slab.rank]
        return [(self.slab.nz, b - a, self.nkx)] * self.slab.world

    def lines(self, recv):
        """z convolution of this rank's ky share over all planes (recv[s]:
        rank s's planes, in z order); the piece for each rank is its planes."""
        s = self.slab
        T = torch.cat(recv, 0).contiguous()
        self.ops.poisson_zconv(T, s.nx, s.ny, s.nz * s.world, self.ky[s.rank][0], self.dx, self.dy, self.dz)
        return [T[r * s.nz:(r + 1) * s.nz] for r in range(s.world)]

    def back_shapes(self):
        return [(self.slab.nz, b - a, self.nkx) for a, b in self.ky]

    def inverse(self, recv):
        """y, x inverse transforms of this slab's planes (recv[r]: rank r's ky
        share): the slab's potential (nx, ny, nzl)."""
        s = self.slab
        return self.ops.poisson_inverse(torch.cat(recv, 1).contiguous(), s.nx, s.ny, s.nz)


def _all_to_all(pieces, shapes, group):
    """pieces[r] goes to rank r; returns what each rank sent here, shaped."""
    import torch.distributed as dist
    send = torch.cat([torch.view_as_real(p).reshape(-1) for p in pieces])
    out = [2 * a * b * c for a, b, c in shapes]
    recv = torch.empty(sum(out), dtype=torch.float64, device=send.device)
    dist.all_to_all_single(recv, send, output_split_sizes=out, input_split_sizes=[2 * p.numel() for p in pieces],
                           group=group)
    return [torch.view_as_complex(c.view(*sh, 2)) for c, sh in zip(recv.split(out), shapes)]


def poisson_isolated(rho, slab: Slab, dx, dy, dz, ops, group=None):
    """solve_poisson_isolated of the global nx x ny x (world nz) grid from this
    rank's density planes rho (nx, ny, nz); returns this rank's planes of phi.
    nx, ny and the global nz are powers of two (the isolated solve's FFTs)."""
    P = SlabPoisson(slab, dx, dy, dz, ops)
    if slab.world == 1:
        return P.inverse(P.lines(P.forward(rho)))
    recv = _all_to_all(P.forward(rho), P.forward_shapes(), group)
    recv = _all_to_all(P.lines(recv), P.back_shapes(), group)
    return P.inverse(recv)


def _phi_neighbours(phi, slab: Slab, group):
    """The plane of Phi next to this slab on each side ((Y, X) tensors; None
    at the global z boundaries: the isolated solve does not wrap)."""
    if slab.world == 1:
        return None, None
    import torch.distributed as dist
    P = phi.permute(2, 1, 0)   # (Z, Y, X) view of the column-major (nx, ny, nzl) array
    lo = slab.rank - 1 if slab.rank > 0 else None
    hi = slab.rank + 1 if slab.rank < slab.world - 1 else None
    ops_list, got = [], {}
    if hi is not None:
        ops_list.append(dist.P2POp(dist.isend, P[-1].contiguous(), hi, group, tag=2))
        got["hi"] = torch.empty_like(P[0].contiguous())
        ops_list.append(dist.P2POp(dist.irecv, got["hi"], hi, group, tag=3))
    if lo is not None:
        ops_list.append(dist.P2POp(dist.isend, P[0].contiguous(), lo, group, tag=3))
        got["lo"] = torch.empty_like(P[0].contiguous())
        ops_list.append(dist.P2POp(dist.irecv, got["lo"], lo, group, tag=2))
    for req in dist.batch_isend_irecv(ops_list):
        req.wait()
    return got.get("lo"), got.get("hi")


def sg_source(dU, U, phi, slab: Slab, dx, dy, dz, ops, lo=None, hi=None):
    """The self-gravity source (src/self_gravity.jl:93-115 after the solve;
    src/gpu_kernels.jl:291-319) on this slab's cells from its planes of Phi and
    the neighbours' planes lo / hi (None at a global boundary, where the
    reference's one-sided difference applies).  Every cell takes the
    undivided grid's arithmetic: interior slab faces the central difference
    with the neighbour's plane, global boundaries the one-sided one."""
    nx, ny, nz = slab.nx, slab.ny, slab.nz
    if lo is None and hi is None:
        ops.sg_gradient(dU, U, phi, nx, ny, nz, dx, dy, dz)
        return
    # the slab's edge planes take the central z difference with the
    # neighbours' planes, in place (no extended copy of the state)
    ops.sg_gradient_slab(dU, U, phi, nx, ny, nz, dx, dy, dz, lo, hi)


def add_self_gravity_source(dU, U, slab: Slab, dx, dy, dz, ops, group=None):
    """add_self_gravity_source! (src/self_gravity.jl:93-115) of the global grid
    on this rank's slab: Phi from the distributed solve of the slabs' active
    densities, one plane of Phi from each neighbour, the source added to dU."""
    phi = poisson_isolated(ops.active_rho(U, slab.nx, slab.ny, slab.nz), slab, dx, dy, dz, ops, group)
    lo, hi = _phi_neighbours(phi, slab, group)
    sg_source(dU, U, phi, slab, dx, dy, dz, ops, lo, hi)


class DeviceOps:
    """The slab operations on CUDA tensors through this library's C ABI."""

    def __init__(self, device="cuda"):
        from . import api
        self.api = api
        self.device = torch.device(device)

    @staticmethod
    def copy(U):
        return U.clone()

    @staticmethod
    def zeros_like(U):
        return torch.zeros_like(U)

    @staticmethod
    def assign(U, V):
        U.copy_(V)

    def zeros(self, shape):
        return torch.zeros(shape, dtype=torch.float64, device=self.device)

    def state(self, nx, ny, nz):
        return self.api.state(nx, ny, nz, device=self.device)

    def active(self, nx, ny, nz):
        return self.api.active_grid(nx, ny, nz, device=self.device)

    def flux_arrays(self, nx, ny, nz):
        return self.api.flux_arrays(nx, ny, nz, device=self.device)

    def rhs_fluxes(self, dU, Fx, Fy, Fz, U, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor):
        """euler3d_rhs! without its ghost fill, keeping the face fluxes."""
        self.api.euler3d_rhs(dU, Fx, Fy, Fz, U, nx, ny, nz, dx, dy, dz, gamma, bc=bc, rho_floor=rho_floor,
                             P_floor=P_floor, fill_ghosts=False)

    def fmr_grid(self, Uc, ncx, ncy, ncz, dxc, dyc, dzc, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio, gamma,
                 rho_floor, P_floor, init):
        return self.api.FMRGrid3D(Uc, ncx, ncy, ncz, dxc, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio, gamma,
                                  rho_floor=rho_floor, P_floor=P_floor, dyc=dyc, dzc=dzc, init=init)

    def fill(self, U, nx, ny, nz, bc):
        (self.api.fill_ghost_3d_outflow if bc == "outflow" else self.api.fill_ghost_3d_periodic)(U, nx, ny, nz)

    def rhs(self, dU, U, nx, ny, nz, dx, dy, dz, gamma, bc, rho_floor, P_floor):
        self.api.euler3d_rhs(dU, None, None, None, U, nx, ny, nz, dx, dy, dz, gamma, bc=bc, rho_floor=rho_floor,
                             P_floor=P_floor, fill_ghosts=False)

    def floors(self, U, nx, ny, nz, rho_floor, P_floor, gamma):
        self.api.apply_floors_3d(U, nx, ny, nz, rho_floor, P_floor, gamma)

    def cfl(self, U, nx, ny, nz, dx, dy, dz, gamma, cfl):
        return self.api.cfl_dt_3d(U, nx, ny, nz, dx, dy, dz, gamma, cfl)

    def poisson_forward(self, rho, nx, ny, nzl):
        return self.api.poisson_slab_forward(rho, nx, ny, nzl)

    def poisson_zconv(self, T, nx, ny, nz, ky0, dx, dy, dz):
        self.api.poisson_slab_zconv(T, nx, ny, nz, ky0, dx, dy, dz)

    def poisson_inverse(self, W2, nx, ny, nzl):
        return self.api.poisson_slab_inverse(W2, nx, ny, nzl)

    def active_rho(self, U, nx, ny, nz):
        rho = self.api.active_grid(nx, ny, nz, device=U.device)
        rho.copy_(U[0, NG:NG + nx, NG:NG + ny, NG:NG + nz])
        return rho

    def sg_gradient(self, dU, U, phi, nx, ny, nz, dx, dy, dz):
        self.api.apply_sg_force_level(dU, U, phi, nx, ny, nz, dx, dy, dz)

    def sg_gradient_slab(self, dU, U, phi, nx, ny, nz, dx, dy, dz, lo, hi):
        self.api.apply_sg_force_slab(dU, U, phi, nx, ny, nz, dx, dy, dz,
                                     None if lo is None else lo.contiguous(),
                                     None if hi is None else hi.contiguous())

    def active_rho_floored(self, U, nx, ny, nz, rho_floor):
        """The active density as euler3d_rhs! leaves it (floored at rho_floor)."""
        rho = self.active_rho(U, nx, ny, nz)
        return rho.clamp_(min=rho_floor)

    def stage(self, Uout, Uin, Un, s, slab, dx, dy, dz, dt, gamma, rho_floor, P_floor, src, precision):
        """One RK3 stage in one fused launch (bsn_euler3d_stage) with Uin's
        ghost cells as filled and exchanged."""
        kw = {}
        if src is not None:
            kw = dict(bhs=src.bhs, nsink=src.nsink, f_sink=src.f_sink, torque_free=src.torque_free,
                      rho_sink_min=src.rho_sink_min, x0=src.x0, y0=src.y0, z0=src.z0, k0=slab.k0, phi=src.phi,
                      phi_lo=None if src.phi_lo is None else src.phi_lo.contiguous(),
                      phi_hi=None if src.phi_hi is None else src.phi_hi.contiguous())
        self.api.euler3d_stage(Uout, Uin, Un, slab.nx, slab.ny, slab.nz, dx, dy, dz, dt, gamma, s,
                               rho_floor=rho_floor, P_floor=P_floor, precision=precision, **kw)

    def bh_gravity(self, dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, k0):
        self.api.add_bh_gravity_source_slab(dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, k0)

    def sink_sources(self, dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, k0, f_sink, torque_free, rho_sink_min):
        self.api.add_sink_sources_slab(dU, U, nx, ny, nz, dx, dy, dz, bhs, x0, y0, z0, k0, f_sink=f_sink,
                                       torque_free=torque_free, rho_sink_min=rho_sink_min)

    def gas_force_pairs(self, U, nx, ny, nz, dx, dy, dz, bh, x0, y0, z0, k0):
        return self.api.gas_force_pairs_slab(U, nx, ny, nz, dx, dy, dz, bh, x0, y0, z0, k0)

    def sink_terms(self, U, nx, ny, nz, dx, dy, dz, x0, y0, z0, k0, bh, dt, box, f_sink, rho_sink_min):
        return self.api.sink_terms_slab(U, nx, ny, nz, dx, dy, dz, x0, y0, z0, k0, bh, dt, box, f_sink=f_sink,
                                        rho_sink_min=rho_sink_min)

    def floor_planes(self, planes, nx, ny, rho_floor, P_floor, gamma):
        """apply_floors_3d! on the active (i, j) cells of NG received z-planes
        ((NG, Y, X, 5) C-contiguous), through a ghosted scratch array."""
        G = self.api.state(nx, ny, NG, device=planes.device)
        _zmajor(G)[NG:2 * NG] = planes
        self.api.apply_floors_3d(G, nx, ny, NG, rho_floor, P_floor, gamma)
        return _zmajor(G)[NG:2 * NG]
