"""x-slab domain decomposition of the GMG-preconditioned flexible-CG solve.

The reference solves one grid in one process (src/voxel_mg.py:120-217, experiments/session_i/
run_gpu.py:281-304).  Here the grid is cut into slabs along x, one per GPU (or several on one
device): slab i owns elements ex in [a_i, b_i) and stores node planes a_i..b_i.  In the author
layout x is the slowest index, so a slab's vectors, moduli and masks are contiguous slices of the
global ones.  The planes a_i and b_i are shared with the neighbours and stored by both.

Operator forms (matvec, damped Jacobi sweep, residual, true residual): each slab runs the fused
single-grid kernel on its own slab, which gets every plane right except the shared ones.  For
those it computes its element layer's contribution (vx_layer_partial) on a side stream, the
slabs swap the contributions (SlabComm.swap: NCCL send/recv between processes, device copies
between slabs of one process) while the slab kernel runs, and vx_plane_fix rewrites each shared
plane from lo + hi with the lower slab's contribution first, so both copies are bitwise equal.

Dots and norms run over each slab's owned prefix (planes a_i..b_i - 1; the last slab also owns
b_i) and are summed over slabs (SlabComm.allreduce_) before the FP64 scalar kernels use them.

Transfers: before restriction the shared fine planes of the residual are halved (vx_plane_fix
mode 2 with scale 1/2), each slab restricts locally, and the coarse shared planes are summed
(vx_plane_sum); prolongation is local.  Slab bounds are multiples of 2^(levels-1), so every level
splits at whole elements.  The coarsest level is gathered and solved in every process with the
FP64 inverse Cholesky factor of the global coarsest matrix (replicated, as it is small).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import _lib
from .element import quadrature
from .operators import PREC, STORAGE, VoxelOperator, node_mask_from_dofs, stream_ptr
from .solver import (FIN_BETA_PR, FIN_NB, FIN_PQ, FIN_RZ, FIN_TRUE, S_BREAK, S_CHECK, S_DONE, S_IT, S_MAXIT,
                     S_MV, S_REL, S_TOL, SolveResult, _GraphLoop, hierarchy_shapes)

PLANE_APPLY, PLANE_JACOBI, PLANE_RESIDUAL, PLANE_TRUE_RES = range(4)
_ARITH = {torch.float64: torch.float64, torch.float32: torch.float32, torch.bfloat16: torch.float32}


def slab_bounds(nx: int, nparts: int, levels: int = 1):
    """Element ranges [(a_i, b_i)] of `nparts` slabs along x, as even as the coarsest level allows:
    bounds are multiples of 2^(levels-1) and every slab keeps at least one coarsest element."""
    f = 1 << (levels - 1)
    if nx % f:
        raise ValueError(f"nx={nx} is not divisible by 2^(levels-1)={f}")
    nxc = nx // f
    if not 1 <= nparts <= nxc:
        raise ValueError(f"{nparts} slabs need 1 <= slabs <= {nxc} (coarsest x extent)")
    q, rem = divmod(nxc, nparts)
    out, a = [], 0
    for i in range(nparts):
        s = q + (1 if i < rem else 0)
        out.append((a * f, (a + s) * f))
        a += s
    return out


def _at(t, offset):
    """Device address of element `offset` of a contiguous tensor (None stays None)."""
    return None if t is None else t.data_ptr() + int(offset) * t.element_size()


def _s():
    return stream_ptr()


# ---------------------------------------------------------------------------------------- comm
class SlabComm:
    """Moves shared-plane data between neighbouring slabs and sums per-slab scalars.

    `local` lists the slab indices held by this process.  Slabs held by one process exchange by
    device copies; otherwise slab i lives on rank i of the default process group (one slab per
    process) and neighbours exchange with send/recv: NCCL moves device buffers directly; with a
    gloo group, device buffers are staged through host memory (each exchange then completes on the
    host before the next launch)."""

    def __init__(self, nparts: int, local=None):
        self.nparts = int(nparts)
        distributed = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
        if local is None:
            local = [dist.get_rank()] if distributed else list(range(self.nparts))
        self.local = [int(i) for i in local]
        self.distributed = distributed
        self.staged = distributed and dist.get_backend() != "nccl"
        if distributed:
            if dist.get_world_size() != self.nparts or self.local != [dist.get_rank()]:
                raise ValueError("across processes, slab i must be the only slab of rank i "
                                 f"(world {dist.get_world_size()}, slabs {self.nparts}, local {self.local})")
        elif sorted(self.local) != list(range(self.nparts)):
            raise ValueError(f"one process must hold every slab: {self.local} of {self.nparts}")

    def swap(self, halos):
        """halos: {slab index: _Halo}.  Fills each halo's recv_lo with the lower neighbour's own_hi
        and recv_hi with the upper neighbour's own_lo."""
        ops = []
        for i, h in halos.items():
            if i > 0:
                if i - 1 in halos:
                    h.recv_lo.copy_(halos[i - 1].own_hi)
                else:
                    ops += [dist.P2POp(dist.isend, h.own_lo, i - 1), dist.P2POp(dist.irecv, h.recv_lo, i - 1)]
            if i < self.nparts - 1:
                if i + 1 in halos:
                    h.recv_hi.copy_(halos[i + 1].own_lo)
                else:
                    ops += [dist.P2POp(dist.isend, h.own_hi, i + 1), dist.P2POp(dist.irecv, h.recv_hi, i + 1)]
        if ops:
            back = []
            if self.staged:                     # host copies of device buffers for gloo
                staged = []
                for op in ops:
                    t = op.tensor
                    if t.is_cuda:
                        h = t.cpu() if op.op is dist.isend else torch.empty(t.shape, dtype=t.dtype)
                        if op.op is not dist.isend:
                            back.append((t, h))
                        t = h
                    staged.append(dist.P2POp(op.op, t, op.peer))
                ops = staged
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            for t, h in back:
                t.copy_(h)

    def allreduce_(self, tensors):
        """Sum the per-slab tensors (same shape) over all slabs, in slab order within a process;
        every tensor ends with the total."""
        acc = tensors[0]
        for t in tensors[1:]:
            acc.add_(t)
        if self.distributed:
            if self.staged and acc.is_cuda:
                h = acc.cpu()
                dist.all_reduce(h)
                acc.copy_(h)
            else:
                dist.all_reduce(acc)
        for t in tensors[1:]:
            t.copy_(acc)
        return acc

    def gather(self, pieces, out):
        """Concatenate the slabs' pieces (1-D, slab order) into `out` on every process."""
        if not self.distributed:
            off = 0
            for t in pieces:
                out[off:off + t.numel()].copy_(t)
                off += t.numel()
            return out
        piece = pieces[0]
        if self.staged:
            piece = piece.cpu()
        sizes = torch.tensor([piece.numel()], dtype=torch.int64, device=piece.device)
        all_sizes = [torch.zeros_like(sizes) for _ in range(self.nparts)]
        dist.all_gather(all_sizes, sizes)
        sizes = [int(s) for s in all_sizes]
        width = max(sizes)
        bufs = [torch.zeros(width, dtype=piece.dtype, device=piece.device) for _ in range(self.nparts)]
        mine = torch.zeros(width, dtype=piece.dtype, device=piece.device)
        mine[:piece.numel()].copy_(piece)
        dist.all_gather(bufs, mine)
        off = 0
        for buf, s in zip(bufs, sizes):
            out[off:off + s].copy_(buf[:s])
            off += s
        return out


class _Halo:
    """A slab's shared-plane buffers for one vector type: its own layer contributions (sent) and the
    neighbours' (received), 3 P values each; None at the global ends."""

    def __init__(self, n3, dtype, has_lo, has_hi):
        z = lambda on: torch.zeros(n3, dtype=dtype, device="cuda") if on else None     # noqa: E731
        self.own_lo, self.recv_lo = z(has_lo), z(has_lo)
        self.own_hi, self.recv_hi = z(has_hi), z(has_hi)
        self.has_lo, self.has_hi = has_lo, has_hi


# ---------------------------------------------------------------------------------------- levels
class _SlabLevel:
    """One level of one slab: the slab-local grid and its buffers."""

    def __init__(self, index, nparts, shape, a, ke, dtype, aux):
        self.index, self.shape, self.a = index, tuple(shape), int(a)
        nlx, ny, nz = self.shape
        self.P = (ny + 1) * (nz + 1)
        self.n = 3 * (nlx + 1) * self.P
        self.has_lo, self.has_hi = index > 0, index < nparts - 1
        self.n_own = 3 * (nlx + (0 if self.has_hi else 1)) * self.P
        # node planes that are not shared: the fused reductions' range (shared planes are added
        # by the plane fix, by their owner)
        self.interior = (1 if self.has_lo else 0, nlx if self.has_hi else nlx + 1)
        self.G_fix = int(_lib.load().vx_plane_fix_partials(self.P))
        self.ke = np.ascontiguousarray(ke)
        self.kp = _lib.dptr(self.ke)
        self.op = VoxelOperator(self.shape, self.ke, dtype, aux)
        self.op64 = self.op if dtype == torch.float64 else VoxelOperator(self.shape, self.ke, torch.float64)
        self.halo = _Halo(3 * self.P, _ARITH[dtype], self.has_lo, self.has_hi)
        self.halo64 = self.halo if _ARITH[dtype] == torch.float64 else _Halo(3 * self.P, torch.float64,
                                                                           self.has_lo, self.has_hi)
        self.rhalo = None          # restricted right-hand side planes (auxiliary storage), coarse levels
        self.E64 = self.E = self.mask = self.invd = self.invd64 = None
        self.r = self.x = self.xt = self.res = None
        self._res_buf = None       # the buffer the V-cycle's residual went to (read by the restriction)
        self.omega = 0.0

    # -- the per-slab halves of an operator form
    def partials(self, prec, u, halo, E):
        """This slab's element-layer contributions to its shared planes, for iterate u."""
        nlx, ny, nz = self.shape
        P = self.P
        if self.has_lo:
            _lib.call("vx_layer_partial", prec, ny, nz, self.kp, _at(E, 0), _at(u, 0), _at(self.mask, 0), 0,
                      halo.own_lo.data_ptr(), _s())
        if self.has_hi:
            _lib.call("vx_layer_partial", prec, ny, nz, self.kp, _at(E, (nlx - 1) * ny * nz), _at(u, 3 * (nlx - 1) * P),
                      _at(self.mask, (nlx - 1) * P), 1, halo.own_hi.data_ptr(), _s())

    def fix(self, prec, mode, halo, x, out, r=None, invd=None, omega=0.0, scale=1.0, dot=None, dot_at=0):
        """Rewrite the shared planes of `out` from the two contributions (lower slab first).  With
        `dot` (modes 0 and 3) the rewritten planes' dot terms go to dot[dot_at:] (the lower plane,
        owned by this slab) and dot[dot_at + G:] (the upper plane, owned by the upper neighbour:
        zeros), G = vx_plane_fix_partials(P)."""
        nlx = self.shape[0]
        P = self.P
        G = self.G_fix
        if self.has_lo:
            _lib.call("vx_plane_fix", prec, mode, P, halo.recv_lo.data_ptr(), halo.own_lo.data_ptr(),
                      _at(self.mask, 0), _at(x, 0), _at(r, 0), _at(invd, 0), float(omega), float(scale),
                      _at(out, 0), _at(dot, dot_at), 1, _s())
        if self.has_hi:
            o = 3 * nlx * P
            _lib.call("vx_plane_fix", prec, mode, P, halo.own_hi.data_ptr(), halo.recv_hi.data_ptr(),
                      _at(self.mask, nlx * P), _at(x, o), _at(r, o), _at(invd, o), float(omega), float(scale),
                      _at(out, o), _at(dot, dot_at + G), 0, _s())


class SlabHierarchy:
    """The rediscretised GMG V-cycle (src/voxel_mg.py:120-178, as solver.MGHierarchy) over the slabs
    this process holds, lock-step across slabs: every level step runs for all local slabs, then
    the exchanges they need."""

    def __init__(self, shape, ke, E, node_mask, nparts, comm: SlabComm, dtype=torch.float32, aux_dtype=None,
                 pre=2, post=2, omegas=None, max_coarse_x=16, shapes=None, spectral_seed=20260923):
        aux_dtype = dtype if aux_dtype is None else aux_dtype
        if (dtype, aux_dtype) not in STORAGE:
            raise ValueError(f"unsupported V-cycle storage: iterate {dtype}, auxiliary {aux_dtype}")
        self.shapes = [tuple(s) for s in (shapes or hierarchy_shapes(shape, max_coarse_x))]
        if len(self.shapes) < 2:
            raise ValueError("the slab V-cycle needs at least two levels")
        self.comm, self.nparts = comm, int(nparts)
        self.dtype, self.aux_dtype = dtype, aux_dtype
        self.prec, self.pre, self.post = STORAGE[(dtype, aux_dtype)], int(pre), int(post)
        self.ke = np.asarray(ke, dtype=np.float64).reshape(24, 24)
        nl = len(self.shapes)
        self.bounds = slab_bounds(self.shapes[0][0], self.nparts, nl)
        self.side = torch.cuda.Stream()
        _, ny, nz = self.shapes[0]
        P0 = (ny + 1) * (nz + 1)
        self.parts = {}
        for i in comm.local:
            a, b = self.bounds[i]
            levels = []
            for l, s in enumerate(self.shapes):
                f = 1 << l
                L = _SlabLevel(i, self.nparts, (b // f - a // f, s[1], s[2]), a // f, self.ke * f, dtype, aux_dtype)
                if l == 0:
                    # owned copies: a caller rewriting its global arrays does not change the solver
                    L.E64 = E[a * ny * nz:b * ny * nz].to(torch.float64).clone()
                    L.mask = node_mask[a * P0:(b + 1) * P0].clone()
                else:
                    prev = levels[-1]
                    L.E64 = torch.empty(L.shape[0] * L.shape[1] * L.shape[2], dtype=torch.float64, device="cuda")
                    _lib.call("vx_coarsen_modulus", _lib.VX_F64, *prev.shape, prev.E64.data_ptr(), L.E64.data_ptr(), _s())
                    L.mask = torch.empty((L.shape[0] + 1) * L.P, dtype=torch.uint8, device="cuda")
                    _lib.call("vx_coarsen_mask", *prev.shape, prev.mask.data_ptr(), L.mask.data_ptr(), _s())
                    L.rhalo = _Halo(3 * L.P, aux_dtype, L.has_lo, L.has_hi)
                L.E = L.E64 if aux_dtype == torch.float64 else L.E64.to(aux_dtype)
                L.r = torch.zeros(L.n, dtype=aux_dtype, device="cuda")
                L.x = torch.zeros(L.n, dtype=dtype, device="cuda")
                L.xt = torch.zeros(L.n, dtype=dtype, device="cuda")
                L.res = None if aux_dtype == dtype else torch.zeros(L.n, dtype=aux_dtype, device="cuda")
                levels.append(L)
            self.parts[i] = levels
        self._diagonals()
        self._coarse_setup()
        n_smooth = nl - 1
        if omegas is None:
            om = [0.6] * n_smooth
            self.lambdas = None
        elif isinstance(omegas, str) and omegas == "spectral":
            om, self.lambdas = self.spectral_omegas(seed=spectral_seed)
        elif np.isscalar(omegas):
            om, self.lambdas = [float(omegas)] * n_smooth, None
        else:
            om, self.lambdas = [float(w) for w in omegas], None
        self.set_omegas(om)

    # ------------------------------------------------------------------ set-up
    def set_omegas(self, omegas):
        if len(omegas) != len(self.shapes) - 1:
            raise ValueError(f"need {len(self.shapes) - 1} omegas, got {len(omegas)}")
        self.omegas = [float(w) for w in omegas]
        for levels in self.parts.values():
            for L, w in zip(levels, self.omegas + [0.0]):
                L.omega = w

    def _level(self, l):
        return [(i, lv[l]) for i, lv in self.parts.items()]

    def _diagonals(self):
        """inv_diag per level: the slab diagonals, summed on shared planes, then 1/d on free DOFs."""
        for l in range(len(self.shapes) - 1):
            ds = {}
            for i, L in self._level(l):
                d = L.op64.diagonal(L.E64, None, inverse=False)
                if L.has_lo:
                    L.halo64.own_lo.copy_(d[:3 * L.P])
                if L.has_hi:
                    L.halo64.own_hi.copy_(d[L.n - 3 * L.P:])
                ds[i] = d
            self.comm.swap({i: L.halo64 for i, L in self._level(l)})
            for i, L in self._level(l):
                d = ds[i]
                if L.has_lo:
                    _lib.call("vx_plane_sum", _lib.VX_F64, 3 * L.P, L.halo64.recv_lo.data_ptr(),
                              L.halo64.own_lo.data_ptr(), d.data_ptr(), _s())
                if L.has_hi:
                    o = L.n - 3 * L.P
                    _lib.call("vx_plane_sum", _lib.VX_F64, 3 * L.P, L.halo64.own_hi.data_ptr(),
                              L.halo64.recv_hi.data_ptr(), _at(d, o), _s())
                free = ((L.mask.to(torch.int32)[:, None] >> torch.arange(3, device="cuda")) & 1).reshape(-1).bool()
                inv64 = torch.where(free, 1.0 / d, torch.ones_like(d))
                L.invd = inv64 if self.aux_dtype == torch.float64 else inv64.to(self.aux_dtype)
                L.invd64 = inv64                       # the spectral estimate runs in FP64

    def _coarse_setup(self):
        """The global coarsest grid's moduli and mask (gathered), its dense constrained matrix and the
        packed inverse Cholesky factor, replicated in every process."""
        cs = self.shapes[-1]
        l = len(self.shapes) - 1
        Pc = (cs[1] + 1) * (cs[2] + 1)
        nodes = (cs[0] + 1) * Pc
        Eg = torch.empty(cs[0] * cs[1] * cs[2], dtype=torch.float64, device="cuda")
        self.comm.gather([L.E64 for _, L in self._level(l)], Eg)
        mg = torch.empty(nodes, dtype=torch.uint8, device="cuda")
        self.comm.gather([L.mask[:L.n_own // 3] for _, L in self._level(l)], mg)
        self.coarse_mask, self.coarse_E = mg, Eg
        self.nc = 3 * nodes
        kc = np.ascontiguousarray(self.ke * 2 ** l)
        A = torch.empty(self.nc, self.nc, dtype=torch.float64, device="cuda")
        _lib.call("vx_assemble_dense", *cs, _lib.dptr(kc), Eg.data_ptr(), mg.data_ptr(), A.data_ptr(), _s())
        # banded Cholesky and the packed inverse factor in the library's own kernels (as MGHierarchy)
        bw = min(self.nc - 1, 3 * ((cs[1] + 1) * (cs[2] + 1) + (cs[2] + 1) + 1) + 2)
        work = torch.empty(int(_lib.load().vx_coarse_factor_workspace(self.nc, bw)), dtype=torch.float64, device="cuda")
        info = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.coarse_packed = torch.empty_like(A)
        _lib.call("vx_coarse_factor", self.nc, bw, A.data_ptr(), self.coarse_packed.data_ptr(), work.data_ptr(),
                  info.data_ptr(), _s())
        if int(info) != 0:
            raise ValueError(f"coarsest-level matrix is not positive definite (pivot {int(info)})")
        del A, work
        self._rc = torch.zeros(self.nc, dtype=self.aux_dtype, device="cuda")
        self._zc = torch.zeros(self.nc, dtype=self.dtype, device="cuda")
        self._yc = torch.zeros(self.nc, dtype=torch.float64, device="cuda")

    def spectral_omegas(self, iterations=30, seed=20260923):
        """omega_l = 4 / (3 lambda_l), lambda_l from the seeded FP64 power iteration on D^-1 A over the
        free DOFs (src/voxel_mg.py:228-244), with the same start vector as one grid (sliced)."""
        omegas, lambdas = [], []
        for l in range(len(self.shapes) - 1):
            s = self.shapes[l]
            v0 = np.random.default_rng(seed).standard_normal(3 * (s[0] + 1) * (s[1] + 1) * (s[2] + 1))
            vs, ms, invs, ws = {}, {}, {}, {}
            for i, L in self._level(l):
                lo = 3 * L.a * L.P
                m = ((L.mask.to(torch.int32)[:, None] >> torch.arange(3, device="cuda")) & 1).reshape(-1).double()
                ms[i] = m
                vs[i] = torch.as_tensor(v0[lo:lo + L.n], device="cuda") * m
                invs[i] = L.invd64
                ws[i] = torch.empty(L.n, dtype=torch.float64, device="cuda")
            nrm = self._norm(l, vs)
            for i in vs:
                vs[i] /= nrm
            lam = 0.0
            for _ in range(iterations):
                self.apply64(l, vs, ws)
                for i in ws:
                    ws[i].mul_(invs[i]).mul_(ms[i])
                lam = self._norm(l, ws)
                for i in ws:
                    vs[i].copy_(ws[i] / lam)
            lambdas.append(lam)
            omegas.append(4.0 / (3.0 * lam))
        return omegas, lambdas

    def _norm(self, l, vecs):
        sums = []
        for i, L in self._level(l):
            v = vecs[i][:L.n_own]
            sums.append(torch.dot(v, v).reshape(1))
        return float(self.comm.allreduce_(sums)[0]) ** 0.5

    def apply64(self, l, us, ys):
        """ys = A us on level l in FP64 (the Dirichlet operator M K M + (I - M))."""
        def local(i, L):
            L.op64.matvec(us[i], L.E64, L.mask, out=ys[i])
        self._op(l, lambda i, L: L.partials(_lib.VX_F64, us[i], L.halo64, L.E64), {i: L.halo64 for i, L in self._level(l)},
                 local, lambda i, L: L.fix(_lib.VX_F64, PLANE_APPLY, L.halo64, us[i], ys[i]))

    # ------------------------------------------------------------------ lock-step operator forms
    def _op(self, l, partials, halos, local, fix):
        """Shared-plane contributions and their swap on the side stream, the slab kernels on the
        current stream, then the plane fixes once both are done."""
        main = torch.cuda.current_stream()
        self.side.wait_stream(main)
        with torch.cuda.stream(self.side):
            for i, L in self._level(l):
                partials(i, L)
            self.comm.swap(halos)
        for i, L in self._level(l):
            local(i, L)
        main.wait_stream(self.side)
        for i, L in self._level(l):
            fix(i, L)

    def _jacobi(self, l, src, dst, rs):
        p = self.prec
        self._op(l, lambda i, L: L.partials(p, src[i], L.halo, L.E), {i: L.halo for i, L in self._level(l)},
                 lambda i, L: L.op.jacobi(src[i], rs[i], L.invd, L.E, L.mask, L.omega, out=dst[i]),
                 lambda i, L: L.fix(p, PLANE_JACOBI, L.halo, src[i], dst[i], rs[i], L.invd, L.omega))

    def _residual_split(self, l, src, rs, out):
        """out = (r - A x) M with the shared planes halved (the slab's share for restriction)."""
        p = self.prec
        self._op(l, lambda i, L: L.partials(p, src[i], L.halo, L.E), {i: L.halo for i, L in self._level(l)},
                 lambda i, L: L.op.residual(src[i], rs[i], L.E, L.mask, out=out[i]),
                 lambda i, L: L.fix(p, PLANE_RESIDUAL, L.halo, src[i], out[i], rs[i], None, 0.0, 0.5))

    def _restrict(self, l):
        """levels l+1 r = R res: slab-local restriction, then the shared coarse planes summed."""
        p = self.prec
        for i, L in self._level(l):
            C = self.parts[i][l + 1]
            _lib.call("vx_restrict", p, *L.shape, L._res_buf.data_ptr(), C.mask.data_ptr(), C.r.data_ptr(), _s())
            if C.has_lo:
                C.rhalo.own_lo.copy_(C.r[:3 * C.P])
            if C.has_hi:
                C.rhalo.own_hi.copy_(C.r[C.n - 3 * C.P:])
        self.comm.swap({i: lv[l + 1].rhalo for i, lv in self.parts.items()})
        for i, lv in self.parts.items():
            C = lv[l + 1]
            if C.has_lo:
                _lib.call("vx_plane_sum", p, 3 * C.P, C.rhalo.recv_lo.data_ptr(), C.rhalo.own_lo.data_ptr(),
                          C.r.data_ptr(), _s())
            if C.has_hi:
                _lib.call("vx_plane_sum", p, 3 * C.P, C.rhalo.own_hi.data_ptr(), C.rhalo.recv_hi.data_ptr(),
                          _at(C.r, C.n - 3 * C.P), _s())

    def _coarse(self):
        l = len(self.shapes) - 1
        self.comm.gather([L.r[:L.n_own] for _, L in self._level(l)], self._rc)
        _lib.call("vx_coarse_apply_factor", self.prec, self.nc, self.coarse_packed.data_ptr(), self._rc.data_ptr(),
                  self.coarse_mask.data_ptr(), self._yc.data_ptr(), self._zc.data_ptr(), _s())
        for _, L in self._level(l):
            lo = 3 * L.a * L.P
            L.x.copy_(self._zc[lo:lo + L.n])

    def emit(self, r64s):
        """One V-cycle on the current stream for every local slab: {i: z_i} = M({i: r64_i})."""
        L0s = self._level(0)
        for i, L in L0s:
            r_mg = None if self.dtype == torch.float64 else L.r.data_ptr()
            _lib.call("vx_vcycle_entry", self.prec, L.n, r64s[i].data_ptr(), r_mg, L.invd.data_ptr(), L.omega,
                      L.x.data_ptr(), _s())
        rs = {i: (r64s[i] if self.dtype == torch.float64 else L.r) for i, L in L0s}
        return self._vcycle(0, rs)

    def _vcycle(self, l, rs):
        if l == len(self.shapes) - 1:
            self._coarse()
            return {i: L.x for i, L in self._level(l)}
        bufs = {i: [L.x, L.xt] for i, L in self._level(l)}
        ci = 0
        for _ in range(self.pre - 1):
            self._jacobi(l, {i: b[ci] for i, b in bufs.items()}, {i: b[1 - ci] for i, b in bufs.items()}, rs)
            ci ^= 1
        res = {}
        for i, L in self._level(l):
            L._res_buf = bufs[i][1 - ci] if L.res is None else L.res
            res[i] = L._res_buf
        self._residual_split(l, {i: b[ci] for i, b in bufs.items()}, rs, res)
        self._restrict(l)
        nl = len(self.shapes)
        if l + 1 < nl - 1:
            for i, lv in self.parts.items():
                C = lv[l + 1]
                _lib.call("vx_scaled_product", self.prec, C.n, C.omega, C.invd.data_ptr(), C.r.data_ptr(),
                          C.x.data_ptr(), _s())
        xc = self._vcycle(l + 1, {i: lv[l + 1].r for i, lv in self.parts.items()})
        for i, L in self._level(l):
            _lib.call("vx_prolong_add", self.prec, *L.shape, xc[i].data_ptr(), L.mask.data_ptr(),
                      bufs[i][ci].data_ptr(), _s())
        for _ in range(self.post):
            self._jacobi(l, {i: b[ci] for i, b in bufs.items()}, {i: b[1 - ci] for i, b in bufs.items()}, rs)
            ci ^= 1
        return {i: b[ci] for i, b in bufs.items()}


# ---------------------------------------------------------------------------------------- outer loop
def replay_until_done(replay, read, k, maxiter, it):
    """Host loop of a solve whose body of k iterations (the last one a check) runs as one replay:
    replay, read the device scalars, stop once they say converged or broken down, or before a body
    would pass maxiter.  Every rank reads the same scalars -- they are computed from all-reduced
    sums by the same kernels -- so every rank takes the same decisions and issues the same
    collectives.  Returns (scalars, bodies replayed); the caller finishes the iterations that do not
    fill a whole body one at a time."""
    s = read()
    bodies = 0
    while not s[S_DONE] and not s[S_BREAK] and it + k <= maxiter:
        replay()
        bodies += 1
        s = read()
        it = int(s[S_IT])
    return s, bodies


class _ReplayBody:
    """A body of solver iterations, NCCL exchanges included (neighbour swaps and all-reduces on this
    process's current stream), captured once into a CUDA graph and replayed from the host -- the
    form a slab solve spread over processes can take, since a device-side WHILE loop cannot wait
    for the other ranks' decisions.  The body runs once un-captured first (module loading, NCCL
    communicator set-up); callers re-initialise the solver state afterwards."""

    def __init__(self, stream: torch.cuda.Stream, emit_body):
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            emit_body()
        stream.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        before = _lib.launches
        try:
            with torch.cuda.graph(self.graph, stream=stream):
                emit_body()
        finally:
            self.body_kernels = _lib.launches - before
            _lib.launches = before

    def launch(self):
        self.graph.replay()
        _lib.launches += self.body_kernels

    def close(self):
        if self.graph is not None:
            self.graph.reset()
            self.graph = None


class SlabSolver:
    """K(E) u = f on a global (nx, ny, nz) voxel grid cut into `nparts` x-slabs: the flexible
    (Polak-Ribiere) PCG of src/voxel_mg.py:181-217 in FP64 with the slab V-cycle, the same
    semantics as ElasticitySolver (true residual every `check_every` iterations with residual
    replacement; returns (x, it, converged, rel, matvecs)), driven from the host.

    E (Ne) and mask (3N 0/1 DOF mask or N uint8 node mask) are the GLOBAL arrays; each process
    keeps its slabs' slices.  With torch.distributed initialised and world size > 1 this process
    holds slab `rank` and exchanges with its neighbours over the process group; there
    `dist_graph=True` (NCCL) captures check_every iterations, exchanges included, into a CUDA graph
    that the host replays (replay_until_done) instead of launching every kernel of every iteration.
    Release it with close() before destroy_process_group."""

    def __init__(self, shape, E, mask, nparts, ke=None, precision="mixed", pre=2, post=2, omega=0.6,
                 max_coarse_x=16, levels=None, tol=1e-8, maxiter=200, check_every=1, local=None, graph=True,
                 spectral_seed=20260923, dist_graph=False):
        from .api import _MG_STORAGE, _dev
        if precision not in _MG_STORAGE:
            raise ValueError(f"precision must be one of {tuple(_MG_STORAGE)} for the slab solver")
        self.shape = tuple(int(s) for s in shape)
        self.ke = quadrature([1.0, 1.0, 1.0], 0.3) if ke is None else np.asarray(ke, dtype=np.float64).reshape(24, 24)
        self.comm = SlabComm(nparts, local)
        Eg = _dev(E)
        m = mask.to("cuda") if isinstance(mask, torch.Tensor) else _dev(mask)
        nm = m.contiguous() if m.dtype == torch.uint8 else node_mask_from_dofs(m.to(torch.float64))
        shapes = hierarchy_shapes(self.shape, max_coarse_x)
        if levels is not None:
            if levels > len(shapes):
                raise ValueError(f"{self.shape} supports at most {len(shapes)} levels with max_coarse_x={max_coarse_x}")
            shapes = shapes[:levels]
        dt, aux = _MG_STORAGE[precision]
        self.M = SlabHierarchy(self.shape, self.ke, Eg, nm, nparts, self.comm, dt, aux, pre, post, omega,
                               shapes=shapes, spectral_seed=spectral_seed)
        self.tol, self.maxiter, self.check_every = float(tol), int(maxiter), max(1, int(check_every))
        self.zprec = PREC[dt]
        f64 = dict(dtype=torch.float64, device="cuda")
        self.vec = {}
        for i, L in self.M._level(0):
            n = L.n
            self.vec[i] = dict(b=torch.zeros(n, **f64), x=torch.zeros(n, **f64), r=torch.zeros(n, **f64),
                               p=torch.zeros(n, **f64), q=torch.zeros(n, **f64),
                               z_old=torch.zeros(n, dtype=dt, device="cuda"),
                               part=torch.zeros(2 * int(_lib.load().vx_solver_partials(L.n_own)), **f64),
                               # fused-kernel partials, then the two shared planes' corrections (zero when absent)
                               opp=torch.zeros(L.op64.partials_size + 2 * int(_lib.load().vx_plane_fix_partials(L.P)),
                                               **f64),
                               sums=torch.zeros(2, **f64))
        self.S = torch.zeros(16, **f64)
        self.S_host = torch.zeros(16, dtype=torch.float64, pin_memory=True)
        self.stream = torch.cuda.Stream()
        self.use_graph = bool(graph) and not self.comm.distributed
        self._graph = None
        if dist_graph and not (self.comm.distributed and not self.comm.staged):
            raise ValueError("dist_graph needs a process group with the NCCL backend and one slab per process")
        self.dist_graph = bool(dist_graph)
        self._replay = None

    def close(self):
        """Release the captured replay graph (it holds NCCL work; release it before the process
        group is destroyed)."""
        if self._replay is not None:
            self._replay.close()
            self._replay = None

    # -------------------------------------------------------------- distributed pieces
    def _levels(self):
        return self.M._level(0)

    def _reduce(self, fin, count, fill=None, buf="part"):
        """fill(i, L, partials) writes each slab's dot partials over its owned prefix (or, with
        buf="opp", a fused operator kernel and its plane corrections already did); the slab sums
        are reduced, summed over slabs and handed to vx_solver_finalize(fin)."""
        sums = []
        for i, L in self._levels():
            v = self.vec[i]
            if fill is not None:
                fill(i, L, v[buf].data_ptr())
            G = int(_lib.load().vx_solver_partials(L.n_own)) if buf == "part" else v["opp"].numel()
            _lib.call("vx_reduce_partials", G, count, v[buf].data_ptr(), v["sums"].data_ptr(), _s())
            sums.append(v["sums"][:count])
        acc = self.comm.allreduce_(sums)
        _lib.call("vx_solver_finalize", fin, 1, acc.data_ptr(), self.S.data_ptr(), _s())

    def _dots(self, a, b, zo=None, zprec=_lib.VX_F64, fin=FIN_PQ, count=1):
        self._reduce(fin, count, lambda i, L, pp: _lib.call(
            "vx_dots_pr", _lib.VX_F64, zprec, L.n_own, self.vec[i][a].data_ptr(), b(i).data_ptr(),
            None if zo is None else self.vec[i][zo].data_ptr(), pp, _s()))

    def _apply_dot(self):
        """q = A p and p.q: the fused apply-dot on each slab, its shared planes rewritten with their
        dot terms corrected, the partials summed over slabs (FIN_PQ)."""
        v = self.vec
        self.M._op(0, lambda i, L: L.partials(_lib.VX_F64, v[i]["p"], L.halo64, L.E64),
                   {i: L.halo64 for i, L in self._levels()},
                   lambda i, L: _lib.call("vx_apply_dot_planes", _lib.VX_F64, *L.shape, L.op64._bp, L.E64.data_ptr(),
                                          L.mask.data_ptr(), v[i]["p"].data_ptr(), v[i]["q"].data_ptr(),
                                          v[i]["opp"].data_ptr(), *L.interior, _s()),
                   lambda i, L: L.fix(_lib.VX_F64, PLANE_APPLY, L.halo64, v[i]["p"], v[i]["q"], dot=v[i]["opp"],
                                      dot_at=L.op64.partials_size))
        self._reduce(FIN_PQ, 1, buf="opp")

    def _true_residual(self, out="r"):
        """out = b - A x and |b - A x|^2 (FIN_TRUE), fused the same way."""
        v = self.vec
        self.M._op(0, lambda i, L: L.partials(_lib.VX_F64, v[i]["x"], L.halo64, L.E64),
                   {i: L.halo64 for i, L in self._levels()},
                   lambda i, L: _lib.call("vx_true_residual_planes", _lib.VX_F64, *L.shape, L.op64._bp,
                                          L.E64.data_ptr(), L.mask.data_ptr(), v[i]["x"].data_ptr(),
                                          v[i]["b"].data_ptr(), v[i][out].data_ptr(), v[i]["opp"].data_ptr(),
                                          *L.interior, _s()),
                   lambda i, L: L.fix(_lib.VX_F64, PLANE_TRUE_RES, L.halo64, v[i]["x"], v[i][out], v[i]["b"],
                                      dot=v[i]["opp"], dot_at=L.op64.partials_size))
        self._reduce(FIN_TRUE, 1, buf="opp")

    def _precondition(self):
        return self.M.emit({i: self.vec[i]["r"] for i, _ in self._levels()})

    def _direction(self, z, first):
        S = self.S.data_ptr()
        if first:
            self._dots("r", lambda i: z[i], zprec=self.zprec, fin=FIN_RZ)
        else:
            self._dots("r", lambda i: z[i], zo="z_old", zprec=self.zprec, fin=FIN_BETA_PR, count=2)
        for i, L in self._levels():
            v = self.vec[i]
            if first:
                v["p"].zero_()
            _lib.call("vx_cg_direction", _lib.VX_F64, self.zprec, L.n, S, z[i].data_ptr(), v["p"].data_ptr(),
                      v["z_old"].data_ptr(), _s())

    def _iteration(self, check):
        S = self.S.data_ptr()
        self._apply_dot()
        for i, L in self._levels():
            v = self.vec[i]
            _lib.call("vx_cg_update", _lib.VX_F64, L.n, S, v["x"].data_ptr(), v["p"].data_ptr(), v["r"].data_ptr(),
                      v["q"].data_ptr(), 0 if check else 1, _s())
        if check:
            self._true_residual()
        self._direction(self._precondition(), first=False)

    def _read(self):
        self.S_host.copy_(self.S, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.S_host.numpy().copy()

    def _body(self, k):
        for j in range(k):
            self._iteration(j == k - 1)

    def solve(self, f, x0=None):
        """f (and x0): GLOBAL vectors (3N) or {slab index: local slice}.  Returns SolveResult whose x
        is {slab index: local solution} (gather() assembles the global vector).

        With every slab in this process the loop runs as one CUDA-graph WHILE launch (bodies of
        check_every iterations, as FCGSolver); across processes it is driven from the host, one
        iteration at a time, reading the scalars at every check."""
        k = self.check_every
        full = self.maxiter // k
        use_graph = self.use_graph and full > 0
        caller = torch.cuda.current_stream()
        st = self.stream
        st.wait_stream(caller)
        if use_graph and self._graph is None:
            self._graph = _GraphLoop(st, self.S, lambda: self._body(k))
        if self.dist_graph and full > 0 and self._replay is None:
            self._replay = _ReplayBody(st, lambda: self._body(k))
        with torch.cuda.stream(st):
            s = self._solve(f, x0, k, full, use_graph)
        caller.wait_stream(st)
        return self._result(s)

    def _solve(self, f, x0, k, full, use_graph):
        S = self.S.data_ptr()
        for i, L in self._levels():
            v = self.vec[i]
            lo = 3 * L.a * L.P
            v["b"].copy_(f[i] if isinstance(f, dict) else f[lo:lo + L.n])
            if x0 is None:
                v["x"].zero_()
            else:
                v["x"].copy_(x0[i] if isinstance(x0, dict) else x0[lo:lo + L.n])
        _lib.call("vx_set_scalars", S, 0, 16, 0.0, _s())
        _lib.call("vx_set_scalars", S, S_TOL, 1, self.tol, _s())
        _lib.call("vx_set_scalars", S, S_MAXIT, 1, float(self.maxiter), _s())
        _lib.call("vx_set_scalars", S, S_CHECK, 1, float(k), _s())
        self._dots("b", lambda i: self.vec[i]["b"], fin=FIN_NB)
        if x0 is None:
            for i, _ in self._levels():
                self.vec[i]["r"].copy_(self.vec[i]["b"])
        else:
            self._true_residual()
        self._direction(self._precondition(), first=True)
        s = self._read()
        if x0 is not None and s[S_DONE]:
            return s
        if use_graph:
            self._graph.launch(self.stream)
            s = self._read()
            self._graph.account(max(1, -(-int(s[S_IT]) // k)))
        it = int(s[S_IT])
        if self._replay is not None and not s[S_DONE]:
            s, _ = replay_until_done(self._replay.launch, self._read, k, self.maxiter, it)
            it = int(s[S_IT])
        while not s[S_DONE] and not s[S_BREAK] and it < self.maxiter:
            check = (it + 1) % k == 0
            self._iteration(check)
            it += 1
            if check or it == self.maxiter:
                s = self._read()
        if not s[S_DONE]:
            self._true_residual("q")
            s = self._read()
        return s

    def _result(self, s):
        rel = float(s[S_REL])
        return SolveResult({i: self.vec[i]["x"] for i, _ in self._levels()}, int(s[S_IT]), bool(rel <= self.tol), rel,
                           int(s[S_MV]))

    def gather(self, xs=None):
        """The global solution (3N, FP64) from the slabs' local ones, on every process."""
        xs = xs or {i: self.vec[i]["x"] for i, _ in self._levels()}
        s = self.shape
        out = torch.empty(3 * (s[0] + 1) * (s[1] + 1) * (s[2] + 1), dtype=torch.float64, device="cuda")
        return self.comm.gather([xs[i][:L.n_own] for i, L in self._levels()], out)
