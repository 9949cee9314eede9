"""fmr3d_step! (src/fmr3d.jl:451-604) with the coarse level split into z-slabs
over ranks and the refined patch on one rank (its owner).

Every rank steps its slab of the coarse grid as `shard` steps a uniform grid
(ghost fill, halo exchange, euler3d_rhs!, combination, floors per stage) and
adds the coarse fluxes of the C-F faces its cells own to the flux registers.
The owner holds the fine level and a window of the coarse grid: the planes
[ck_lo - 8, ck_hi + 8] with their full x/y extent, the outer three on each
side serving as the window grid's ghost planes, so that the fine level's
Lagrange-5 ghost prolongation and the trilinear potential read only planes
that some rank owns.  Per coarse step:

  1. the owner gathers the window of U^n (self-gravity: restricts the fine
     density into it, restrict_density_to_coarse!, and sends the patch planes
     back, since the reference overwrites the coarse density there first);
  2. self-gravity: the isolated solve of the coarse density on the slabs
     (`shard.poisson_isolated`), the window's planes of Phi to the owner,
     Phi_f trilinear from them; both scaled by G;
  3. every rank: the three coarse stages on its slab with the register sums
     of its faces (each C-F face is summed by the rank that owns the cell on
     the patch side) and the self-gravity source;
  4. the owner gathers the window of U^{n+1} and the register sums (a sum
     over ranks of arrays that are zero outside each rank's faces), runs the
     `ratio` fine subcycles with ghosts prolonged from the time interpolation
     of the two windows, restricts the fine level into the window and applies
     the Berger-Colella correction from the two registers;
  5. the owner sends the planes [ck_lo - 1, ck_hi + 1] back, and every rank
     floors its slab.

Each operation is the reference's, in the reference's order, on the same
values, so with the same dt the slabs and the fine level are the undivided
fmr3d_step!'s bit for bit (FP64).  The gathers and sends move whole planes
between ranks; the only sums are of a rank's value with zeros, which are
exact.  The patch must keep 8 coarse planes from the global z boundaries.
The operations come from an `ops` object, as in `shard`.
"""
from __future__ import annotations

import torch

from .shard import NG, Slab, _allreduce_min, _phi_neighbours, _zmajor, exchange, poisson_isolated, sg_source

RK_W = (1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0)
MARGIN = 8   # window planes beyond the patch on each side (the outer NG are the window grid's ghosts)


def _combine(s, U, Un, dU, dt):
    """The SSP-RK3 combinations of the reference's stages (in place on U)."""
    if s == 0:
        U[...] = Un + dt * dU
    elif s == 1:
        U[...] = 0.75 * Un + 0.25 * U + 0.25 * dt * dU
    else:
        U[...] = (1.0 / 3.0) * Un + (2.0 / 3.0) * U + (2.0 / 3.0) * dt * dU


def _zyx(a):
    """(Z, Y, X) C-contiguous form of an (nx, ny, nz) grid: a view of a
    column-major one (written through), a copy of any other."""
    V = a.permute(2, 1, 0) if isinstance(a, torch.Tensor) else torch.from_numpy(a.T)
    return V if V.is_contiguous() else V.contiguous()


class Registers:
    """The six flux registers of src/fmr3d.jl:81-96 as [q, a, b] arrays over
    the patch's faces (x faces over (j, k), y over (i, k), z over (i, j))."""

    def __init__(self, ops, nic, njc, nkc):
        self.xlo, self.xhi = ops.zeros((5, njc, nkc)), ops.zeros((5, njc, nkc))
        self.ylo, self.yhi = ops.zeros((5, nic, nkc)), ops.zeros((5, nic, nkc))
        self.zlo, self.zhi = ops.zeros((5, nic, njc)), ops.zeros((5, nic, njc))

    def arrays(self):
        return (self.xlo, self.xhi, self.ylo, self.yhi, self.zlo, self.zhi)


class SlabFMR:
    """A two-level FMR grid whose coarse level is this rank's slab `Uc` of
    the global ncx x ncy x (world nz) grid; the box (1-based global coarse
    indices) and ratio as FMRGrid3D (src/fmr3d.jl:109-122).  On the owner,
    `Uf` is the fine level (prolonged from the coarse window when not given)."""

    def __init__(self, Uc, slab: Slab, dxc, ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi, ratio, gamma, ops,
                 group=None, *, rho_floor=0.0, P_floor=0.0, dyc=None, dzc=None, owner=0, Uf=None):
        nzg = slab.nz * slab.world
        if slab.bc != "outflow":
            raise ValueError("slab FMR runs with bc='outflow'")
        if not (1 <= ci_lo <= ci_hi <= slab.nx and 1 <= cj_lo <= cj_hi <= slab.ny):
            raise ValueError("refined box outside the coarse grid in x or y")
        if ck_lo - MARGIN < 1 or ck_hi + MARGIN > nzg or ck_lo > ck_hi:
            raise ValueError(f"refined planes [{ck_lo}, {ck_hi}] must keep {MARGIN} planes from the z boundaries "
                             f"of the {nzg}-plane grid")
        if not 0 <= owner < slab.world:
            raise ValueError(f"owner {owner} of {slab.world} ranks")
        self.Uc, self.slab, self.ops, self.group, self.owner = Uc, slab, ops, group, owner
        self.dxc, self.dyc = dxc, dxc if dyc is None else dyc
        self.dzc = dxc if dzc is None else dzc
        self.box = (ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi)
        self.ratio, self.gamma, self.rho_floor, self.P_floor = ratio, gamma, rho_floor, P_floor
        self.wlo, self.whi = ck_lo - MARGIN, ck_hi + MARGIN           # global planes held by the window array
        self.nzw = self.whi - self.wlo + 1 - 2 * NG                   # the window grid's active planes
        self.G = None
        W = self._gather(Uc)
        if slab.rank == owner:
            kw = (ck_lo - self.wlo - NG + 1, ck_hi - self.wlo - NG + 1)   # the box in window planes
            self.G = ops.fmr_grid(W, slab.nx, slab.ny, self.nzw, self.dxc, self.dyc, self.dzc, ci_lo, ci_hi, cj_lo,
                                  cj_hi, kw[0], kw[1], ratio, gamma, rho_floor, P_floor, init=Uf is None)
            if Uf is not None:
                ops.assign(self.G.Uf, Uf)
            self.Wn = ops.copy(W)

    # -- plane transfers ----------------------------------------------------
    def _owned(self, r, lo, hi):
        """Global planes [lo, hi] (1-based) that rank r owns, as (a, b) or None."""
        a, b = max(lo, r * self.slab.nz + 1), min(hi, (r + 1) * self.slab.nz)
        return (a, b) if a <= b else None

    def _gather(self, U):
        """The window planes of state U: a new window array on the owner (None elsewhere)."""
        return self._gather_into(U, None, self.wlo, self.whi, state=True)

    def _gather_into(self, A, out, lo, hi, state):
        """Planes [lo, hi] of every rank's array A (state arrays, or column-major
        active grids when state is False), assembled on the owner."""
        slab, ops = self.slab, self.ops
        off = NG if state else 0
        V = _zmajor(A) if state else _zyx(A)
        if out is None and slab.rank == self.owner:
            out = ops.state(slab.nx, slab.ny, hi - lo + 1 - 2 * NG) if state else ops.active(slab.nx, slab.ny,
                                                                                            hi - lo + 1)
        O = None if out is None else (_zmajor(out) if state else _zyx(out))
        mine = self._owned(slab.rank, lo, hi)
        if slab.world == 1:
            O[:] = V[off + lo - 1 - slab.k0:off + hi - slab.k0]
            return out
        import torch.distributed as dist
        spans = [self._owned(r, lo, hi) for r in range(slab.world)]
        npl = max((b - a + 1) for a, b in (s for s in spans if s))
        buf = torch.zeros((npl,) + tuple(V.shape[1:]), dtype=V.dtype, device=ops.device)
        if mine:
            a, b = mine
            buf[:b - a + 1] = V[off + a - 1 - slab.k0:off + b - slab.k0]
        got = [torch.empty_like(buf) for _ in range(slab.world)]
        dist.all_gather(got, buf, group=self.group)
        if O is not None:
            for r, s in enumerate(spans):
                if s:
                    a, b = s
                    O[a - lo:b - lo + 1] = got[r][:b - a + 1]
        return out

    def _send_back(self, U, lo, hi):
        """Planes [lo, hi] of the owner's window to the ranks that own them."""
        slab, ops = self.slab, self.ops
        V = _zmajor(U)
        if slab.rank == self.owner:
            src = _zmajor(self.G.Uc)[lo - self.wlo:hi - self.wlo + 1].contiguous()
        else:
            src = None
        if slab.world > 1:
            import torch.distributed as dist
            shape = (hi - lo + 1,) + tuple(V.shape[1:])
            if src is None:
                src = torch.empty(shape, dtype=V.dtype, device=ops.device)
            dist.broadcast(src, self.owner, group=self.group)
        mine = self._owned(slab.rank, lo, hi)
        if mine:
            a, b = mine
            V[NG + a - 1 - slab.k0:NG + b - slab.k0] = src[a - lo:b - lo + 1]

    def _sum_to_owner(self, R: Registers):
        if self.slab.world == 1:
            return
        import torch.distributed as dist
        for A in R.arrays():
            t = A if isinstance(A, torch.Tensor) else torch.from_numpy(A)
            dist.all_reduce(t, group=self.group)

    # -- the step -----------------------------------------------------------
    def cfl_dt(self, cfl):
        """cfl_dt_fmr3d (src/fmr3d.jl:616-622): min(coarse dt, ratio x fine dt)."""
        slab, ops = self.slab, self.ops
        dtc = _allreduce_min(ops.cfl(self.Uc, slab.nx, slab.ny, slab.nz, self.dxc, self.dyc, self.dzc, self.gamma,
                                     cfl), ops, self.group, slab.world)
        dtf = float("inf")
        if slab.rank == self.owner:
            nf = self.fine_dims
            dtf = ops.cfl(self.G.Uf, *nf, self.dxc / self.ratio, self.dyc / self.ratio, self.dzc / self.ratio,
                          self.gamma, cfl)
        dtf = _allreduce_min(dtf, ops, self.group, slab.world)
        return min(dtc, float(self.ratio) * dtf)

    @property
    def fine_dims(self):
        ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi = self.box
        r = self.ratio
        return (ci_hi - ci_lo + 1) * r, (cj_hi - cj_lo + 1) * r, (ck_hi - ck_lo + 1) * r

    def step(self, dt_c, *, self_gravity=False, G_grav=1.0):
        """fmr3d_step! (src/fmr3d.jl:451-604) over the slabs and the owner's patch."""
        slab, ops, U = self.slab, self.ops, self.Uc
        nx, ny, nz = slab.nx, slab.ny, slab.nz
        g, rfl, Pfl, r = self.gamma, self.rho_floor, self.P_floor, self.ratio
        ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi = self.box
        nic, njc, nkc = ci_hi - ci_lo + 1, cj_hi - cj_lo + 1, ck_hi - ck_lo + 1
        own = slab.rank == self.owner
        # 1. U^n's window (after the fine density's restriction with self-gravity)
        self._gather_into(U, self.G.Uc if own else None, self.wlo, self.whi, state=True)
        phic = phif = lo = hi = None
        if self_gravity:
            if own:
                self.G.restrict_density_to_coarse()
            self._send_back(U, ck_lo, ck_hi)
            # 2. Phi on the slabs, Phi_f from the window's planes of it
            rho = ops.active_rho(U, nx, ny, nz)
            phic = poisson_isolated(rho, slab, self.dxc, self.dyc, self.dzc, ops, self.group)
            pw = self._gather_into(phic, None, self.wlo + NG, self.whi - NG, state=False)
            if own:
                phif = self.G.prolong_scalar_trilinear(pw)
            if G_grav != 1.0:
                phic *= G_grav
                if own:
                    phif *= G_grav
            lo, hi = _phi_neighbours(phic, slab, self.group)
        if own:
            ops.assign(self.Wn, self.G.Uc)
        # 3. the coarse stages on the slab, with this rank's register faces
        frc = Registers(ops, nic, njc, nkc)
        Un, dU = ops.copy(U), ops.zeros_like(U)
        Fx, Fy, Fz = ops.flux_arrays(nx, ny, nz)
        for s in range(3):
            ops.fill(U, nx, ny, nz, slab.bc)
            exchange(U, slab, ops, self.group, rfl, Pfl, g)
            ops.rhs_fluxes(dU, Fx, Fy, Fz, U, nx, ny, nz, self.dxc, self.dyc, self.dzc, g, slab.bc, rfl, Pfl)
            self._coarse_registers(frc, Fx, Fy, Fz, RK_W[s] * dt_c)
            if self_gravity:
                sg_source(dU, U, phic, slab, self.dxc, self.dyc, self.dzc, ops, lo, hi)
            _combine(s, U, Un, dU, dt_c)
            ops.floors(U, nx, ny, nz, rfl, Pfl, g)
        # 4. U^{n+1}'s window and the registers on the owner; the fine subcycles
        self._gather_into(U, self.G.Uc if own else None, self.wlo, self.whi, state=True)
        self._sum_to_owner(frc)
        if own:
            self._fine(dt_c, frc, phif)
        # 5. the corrected planes back, floors
        self._send_back(U, ck_lo - 1, ck_hi + 1)
        ops.floors(U, nx, ny, nz, rfl, Pfl, g)

    def _coarse_registers(self, R: Registers, Fx, Fy, Fz, fac):
        """accumulate_fr_coarse (src/fmr3d.jl:292-326) over the faces this rank
        owns: x and y faces of its planes of the box, the z face below the box
        where it owns plane ck_lo, the one above where it owns ck_hi."""
        slab = self.slab
        ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi = self.box
        span = self._owned(slab.rank, ck_lo, ck_hi)
        if span is None:
            return
        a, b = span
        k = slice(NG + a - 1 - slab.k0, NG + b - slab.k0)            # this rank's planes of the box
        ka, kb = a - ck_lo, b - ck_lo + 1
        j = slice(NG + cj_lo - 1, NG + cj_hi)
        i = slice(NG + ci_lo - 1, NG + ci_hi)
        R.xlo[:, :, ka:kb] += fac * Fx[:, NG + ci_lo - 2, j, k]
        R.xhi[:, :, ka:kb] += fac * Fx[:, NG + ci_hi - 1, j, k]
        R.ylo[:, :, ka:kb] += fac * Fy[:, i, NG + cj_lo - 2, k]
        R.yhi[:, :, ka:kb] += fac * Fy[:, i, NG + cj_hi - 1, k]
        if a == ck_lo:
            R.zlo += fac * Fz[:, i, j, NG + ck_lo - slab.k0 - 2]
        if b == ck_hi:
            R.zhi += fac * Fz[:, i, j, NG + ck_hi - slab.k0 - 1]

    def _fine_registers(self, R: Registers, Fx, Fy, Fz, fac):
        """accumulate_fr_fine (src/fmr3d.jl:331-369): each coarse face sums its
        ratio^2 fine faces in the reference's loop order."""
        r = self.ratio
        nfx, nfy, nfz = self.fine_dims
        for d1 in range(r):          # the outer loop's offset (kf, kf, jf)
            for d2 in range(r):      # the inner loop's offset (jf, ia, ia)
                R.xlo += fac * Fx[:, NG - 1, NG + d2:NG + nfy:r, NG + d1:NG + nfz:r]
                R.xhi += fac * Fx[:, NG + nfx - 1, NG + d2:NG + nfy:r, NG + d1:NG + nfz:r]
        for d1 in range(r):
            for d2 in range(r):
                R.ylo += fac * Fy[:, NG + d2:NG + nfx:r, NG - 1, NG + d1:NG + nfz:r]
                R.yhi += fac * Fy[:, NG + d2:NG + nfx:r, NG + nfy - 1, NG + d1:NG + nfz:r]
        for d1 in range(r):
            for d2 in range(r):
                R.zlo += fac * Fz[:, NG + d2:NG + nfx:r, NG + d1:NG + nfy:r, NG - 1]
                R.zhi += fac * Fz[:, NG + d2:NG + nfx:r, NG + d1:NG + nfy:r, NG + nfz - 1]

    def _fine(self, dt_c, frc: Registers, phif):
        """The fine subcycles, the restriction and bc_correct! (src/fmr3d.jl:
        379-422) on the owner's window."""
        ops, G, r = self.ops, self.G, self.ratio
        g, rfl, Pfl = self.gamma, self.rho_floor, self.P_floor
        ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi = self.box
        nfx, nfy, nfz = self.fine_dims
        dxf, dyf, dzf = self.dxc / r, self.dyc / r, self.dzc / r
        dt_f = dt_c / float(r)
        frf = Registers(ops, ci_hi - ci_lo + 1, cj_hi - cj_lo + 1, ck_hi - ck_lo + 1)
        Uf = G.Uf
        dU = ops.zeros_like(Uf)
        Fx, Fy, Fz = ops.flux_arrays(nfx, nfy, nfz)
        Uci, Un = ops.copy(G.Uc), ops.copy(Uf)
        for s in range(r):
            alpha = s / r
            Uci[...] = (1.0 - alpha) * self.Wn + alpha * G.Uc
            ops.assign(Un, Uf)
            for st in range(3):
                G.prolong_fine_ghosts(Uci)
                ops.rhs_fluxes(dU, Fx, Fy, Fz, Uf, nfx, nfy, nfz, dxf, dyf, dzf, g, "outflow", rfl, Pfl)
                self._fine_registers(frf, Fx, Fy, Fz, RK_W[st] * dt_f / (r * r))
                if phif is not None:
                    ops.sg_gradient(dU, Uf, phif, nfx, nfy, nfz, dxf, dyf, dzf)
                _combine(st, Uf, Un, dU, dt_f)
                ops.floors(Uf, nfx, nfy, nfz, rfl, Pfl, g)
        G.restrict()
        self._bc_correct(G.Uc, frc, frf)

    def _bc_correct(self, W, fc: Registers, ff: Registers):
        """bc_correct! (src/fmr3d.jl:379-422) on the window array: the coarse
        cells beside the box take the fine-minus-coarse register difference."""
        ci_lo, ci_hi, cj_lo, cj_hi, ck_lo, ck_hi = self.box
        kl, kh = ck_lo - self.wlo, ck_hi - self.wlo                   # window array planes of the box
        i = slice(NG + ci_lo - 1, NG + ci_hi)
        j = slice(NG + cj_lo - 1, NG + cj_hi)
        k = slice(kl, kh + 1)
        inv_dx, inv_dy, inv_dz = 1.0 / self.dxc, 1.0 / self.dyc, 1.0 / self.dzc
        W[:, NG + ci_lo - 2, j, k] += (fc.xlo - ff.xlo) * inv_dx
        W[:, NG + ci_hi, j, k] += (ff.xhi - fc.xhi) * inv_dx
        W[:, i, NG + cj_lo - 2, k] += (fc.ylo - ff.ylo) * inv_dy
        W[:, i, NG + cj_hi, k] += (ff.yhi - fc.yhi) * inv_dy
        W[:, i, j, kl - 1] += (fc.zlo - ff.zlo) * inv_dz
        W[:, i, j, kh + 1] += (ff.zhi - fc.zhi) * inv_dz
