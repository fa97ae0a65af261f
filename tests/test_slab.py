"""The x-slab decomposition on CPU.

1. slab_bounds: bounds are multiples of 2^(levels-1), every slab keeps a coarsest element.
2. The decomposition's algebra, restated with the oracle (src/voxel_mg.py products and transfers
   evaluated on slabs): the global Dirichlet operator equals the slab operators with every shared
   plane rebuilt from the two element-layer contributions, M (lo + hi) + (I - M) u; the global
   restriction of a residual equals the slab restrictions of the residual with its shared planes
   halved, the shared coarse planes summed.  A mask with fixed nodes on the shared planes is
   included.  Bar: 1e-13 relative (FP64 summation order only).
3. SlabComm between two gloo processes: neighbour swap, all-reduce and the gather of uneven pieces
   (the NCCL path of one slab per GPU, run on CPU tensors)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import voxel_oracle as vo

vx = pytest.importorskip("voxel_b200")
from voxel_b200.slab import SlabComm, slab_bounds  # noqa: E402

KE = vo.quadrature([1, 1, 1], 0.3)


def test_slab_bounds():
    assert slab_bounds(128, 4, 4) == [(0, 32), (32, 64), (64, 96), (96, 128)]
    b = slab_bounds(576, 8, 6)                        # coarsest x extent 18 over 8 slabs: 3,3,2,2,2,2,2,2
    assert [(hi - lo) // 32 for lo, hi in b] == [3, 3, 2, 2, 2, 2, 2, 2]
    assert b[0][0] == 0 and b[-1][1] == 576 and all(b[i][1] == b[i + 1][0] for i in range(7))
    assert slab_bounds(10, 3, 1) == [(0, 4), (4, 7), (7, 10)]
    assert len(slab_bounds(64, 8, 4)) == 8             # coarsest extent 8: one coarsest element each
    with pytest.raises(ValueError):
        slab_bounds(32, 5, 4)                          # coarsest extent 4 < 5 slabs
    with pytest.raises(ValueError):
        slab_bounds(30, 2, 3)                          # 30 not divisible by 4


def _mask_with_interior_fixed(shape, seed):
    nx, ny, nz = shape
    m = np.ones((nx + 1, ny + 1, nz + 1, 3))
    m[0] = 0.0
    rng = np.random.default_rng(seed)
    m[rng.random((nx + 1, ny + 1, nz + 1, 3)) < 0.08] = 0.0     # fixed DOFs everywhere, shared planes too
    return m.ravel()


def _layer_part(shape, ke, E, u, m, side):
    """Contribution of the single element layer (ny*nz elements, two node planes) to node plane
    `side`: M K_layer (M u) restricted to that plane."""
    _, ny, nz = shape
    P3 = 3 * (ny + 1) * (nz + 1)
    y = vo.product_raw((1, ny, nz), ke, u * m, E) * m
    return y[side * P3:(side + 1) * P3]


@pytest.mark.parametrize("nparts", [2, 3])
def test_slab_operator_algebra_matches_the_global_operator(nparts):
    shape = (12, 3, 5)
    nx, ny, nz = shape
    rng = np.random.default_rng(nparts)
    E = 1e-3 + rng.random(nx * ny * nz)
    u = rng.standard_normal(3 * vo.n_nodes(shape))
    m = _mask_with_interior_fixed(shape, nparts)
    y = vo.apply_dirichlet(shape, KE, E, m, u)
    P3 = 3 * (ny + 1) * (nz + 1)
    ne = ny * nz
    bounds = slab_bounds(nx, nparts, 1)
    parts = []
    for a, b in bounds:
        s = (b - a, ny, nz)
        sl = slice(a * P3, (b + 1) * P3)
        El, ul, ml = E[a * ne:b * ne], u[sl], m[sl]
        parts.append(dict(a=a, b=b, y=vo.apply_dirichlet(s, KE, El, ml, ul),
                          lo=_layer_part(s, KE, El[:ne], ul[:2 * P3], ml[:2 * P3], 0),
                          hi=_layer_part(s, KE, El[-ne:], ul[-2 * P3:], ml[-2 * P3:], 1), u=ul, m=ml))
    for i, p in enumerate(parts):
        yl = p["y"].copy()
        if i > 0:                          # lower shared plane: lower slab's contribution first
            s = parts[i - 1]["hi"] + p["lo"]
            yl[:P3] = np.where(p["m"][:P3] != 0, s, p["u"][:P3])
        if i < nparts - 1:
            s = p["hi"] + parts[i + 1]["lo"]
            yl[-P3:] = np.where(p["m"][-P3:] != 0, s, p["u"][-P3:])
        ref = y[p["a"] * P3:(p["b"] + 1) * P3]
        assert np.max(np.abs(yl - ref)) <= 1e-13 * np.max(np.abs(y))
        # the slab's own operator is already right away from the shared planes
        assert np.max(np.abs((p["y"] - ref)[P3:-P3])) <= 1e-13 * np.max(np.abs(y))


@pytest.mark.parametrize("nparts", [2, 3])
def test_slab_restriction_algebra_matches_the_global_restriction(nparts):
    shape = (12, 4, 6)
    nx, ny, nz = shape
    coarse = (nx // 2, ny // 2, nz // 2)
    rng = np.random.default_rng(10 + nparts)
    m = _mask_with_interior_fixed(shape, 20 + nparts)
    mc = vo.coarsen_mask(m, shape)
    r = rng.standard_normal(3 * vo.n_nodes(shape)) * m
    rc = vo.restrict(r, shape) * mc
    P3, P3c = 3 * (ny + 1) * (nz + 1), 3 * (coarse[1] + 1) * (coarse[2] + 1)
    bounds = slab_bounds(nx, nparts, 2)
    parts = []
    for i, (a, b) in enumerate(bounds):
        rl = r[a * P3:(b + 1) * P3].copy()
        if i > 0:
            rl[:P3] *= 0.5
        if i < nparts - 1:
            rl[-P3:] *= 0.5
        mcl = mc[(a // 2) * P3c:(b // 2 + 1) * P3c]
        parts.append(dict(a=a // 2, b=b // 2, c=vo.restrict(rl, (b - a, ny, nz)) * mcl))
    for i, p in enumerate(parts):
        c = p["c"].copy()
        if i > 0:
            c[:P3c] = parts[i - 1]["c"][-P3c:] + p["c"][:P3c]
        if i < nparts - 1:
            c[-P3c:] = p["c"][-P3c:] + parts[i + 1]["c"][:P3c]
        ref = rc[p["a"] * P3c:(p["b"] + 1) * P3c]
        assert np.max(np.abs(c - ref)) <= 1e-13 * np.max(np.abs(rc))
    # prolongation needs no exchange: the slab prolongation of the coarse slice is the global one's slice
    xc = rng.standard_normal(3 * vo.n_nodes(coarse)) * mc
    xf = vo.prolong(xc, coarse)
    for (a, b) in bounds:
        loc = vo.prolong(xc[(a // 2) * P3c:(b // 2 + 1) * P3c], (b // 2 - a // 2, coarse[1], coarse[2]))
        assert np.array_equal(loc, xf[a * P3:(b + 1) * P3])


def test_slab_diagonal_algebra():
    """The Jacobi diagonal on a shared plane is the sum of the two slabs' diagonals there."""
    shape = (8, 3, 4)
    nx, ny, nz = shape
    E = 1e-2 + np.random.default_rng(3).random(nx * ny * nz)
    d = vo.product_diagonal(shape, KE, E)
    P3 = 3 * (ny + 1) * (nz + 1)
    ne = ny * nz
    (a0, b0), (a1, b1) = slab_bounds(nx, 2, 1)
    d0 = vo.product_diagonal((b0 - a0, ny, nz), KE, E[a0 * ne:b0 * ne])
    d1 = vo.product_diagonal((b1 - a1, ny, nz), KE, E[a1 * ne:b1 * ne])
    assert np.allclose(d0[-P3:] + d1[:P3], d[b0 * P3:(b0 + 1) * P3], rtol=1e-14, atol=0)


def test_comm_in_one_process():
    """Slabs held by one process swap by copies; validation of the slab-to-rank mapping."""
    from voxel_b200.slab import _Halo

    class CpuHalo(_Halo):
        def __init__(self, n3, has_lo, has_hi, base):
            z = lambda on, v: torch.full((n3,), float(v)) if on else None     # noqa: E731
            self.own_lo, self.recv_lo = z(has_lo, base + 0.25), z(has_lo, -1)
            self.own_hi, self.recv_hi = z(has_hi, base + 0.75), z(has_hi, -1)
            self.has_lo, self.has_hi = has_lo, has_hi

    comm = SlabComm(3)
    assert comm.local == [0, 1, 2] and not comm.distributed
    halos = {i: CpuHalo(6, i > 0, i < 2, i) for i in range(3)}
    comm.swap(halos)
    assert torch.all(halos[1].recv_lo == 0.75) and torch.all(halos[1].recv_hi == 2.25)
    assert torch.all(halos[0].recv_hi == 1.25) and torch.all(halos[2].recv_lo == 1.75)
    sums = [torch.tensor([1.0, 2.0]), torch.tensor([10.0, 20.0]), torch.tensor([100.0, 200.0])]
    comm.allreduce_(sums)
    assert all(torch.equal(s, torch.tensor([111.0, 222.0])) for s in sums)
    out = torch.zeros(6)
    comm.gather([torch.tensor([1.0]), torch.tensor([2.0, 3.0]), torch.tensor([4.0, 5.0, 6.0])], out)
    assert torch.equal(out, torch.arange(1.0, 7.0))
    with pytest.raises(ValueError):
        SlabComm(3, local=[0, 2])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from voxel_b200.slab import SlabComm, _Halo
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        comm = SlabComm(world)
        h = _Halo.__new__(_Halo)
        h.has_lo, h.has_hi = rank > 0, rank < world - 1
        h.own_lo = torch.full((9,), rank + 0.25) if h.has_lo else None
        h.own_hi = torch.full((9,), rank + 0.75) if h.has_hi else None
        h.recv_lo = torch.zeros(9) if h.has_lo else None
        h.recv_hi = torch.zeros(9) if h.has_hi else None
        comm.swap({rank: h})
        s = torch.tensor([float(rank + 1), 10.0 * (rank + 1)], dtype=torch.float64)
        comm.allreduce_([s])
        out = torch.zeros(2 + 3 * (world - 1), dtype=torch.float64)
        piece = torch.full((2 if rank == 0 else 3,), float(rank), dtype=torch.float64)
        comm.gather([piece], out)
        q.put((rank, None if h.recv_lo is None else h.recv_lo.tolist(), None if h.recv_hi is None else h.recv_hi.tolist(),
               s.tolist(), out.tolist(), comm.local, comm.distributed))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_comm_across_gloo_processes(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    got = dict((g[0], g[1:]) for g in (q.get(timeout=10) for _ in range(world)))
    total = [sum(range(1, world + 1)), 10.0 * sum(range(1, world + 1))]
    want = [0.0, 0.0] + sum(([float(r)] * 3 for r in range(1, world)), [])
    for r in range(world):
        recv_lo, recv_hi, s, out, local, distributed = got[r]
        assert local == [r] and distributed
        assert recv_lo == (None if r == 0 else [r - 1 + 0.75] * 9)
        assert recv_hi == (None if r == world - 1 else [r + 1 + 0.25] * 9)
        assert s == total
        assert out == want


def test_slab_solver_rejects_bad_arguments_before_device_work():
    """Unknown precisions and slab-to-process mappings fail with ValueError on the host."""
    from voxel_b200.slab import SlabSolver
    with pytest.raises(ValueError, match="precision"):
        SlabSolver((32, 16, 16), None, None, 2, precision="jacobi")
    with pytest.raises(ValueError):
        SlabComm(2, local=[1])
