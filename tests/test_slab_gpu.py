"""The x-slab decomposition on one B200: several slabs held by one process exchange their shared
planes by device copies, which runs every kernel and every step of the multi-GPU path except the
NCCL transport (covered by the gloo tests of test_slab.py).

Bars: the two slab kernels against the oracle (FP64 1e-13, FP32 1e-5, bf16 inputs exact in the
oracle, FP32 arithmetic 1e-5); the slab FP64 operator and V-cycle against the single-grid ones to
1e-12 (summation order only) with shared planes bitwise equal in both holders; slab solves reach
the FP64 relative residual 1e-8 in the single-grid iteration counts and the single-grid compliance
to 1e-7 relative (the solve tolerance)."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import _lib  # noqa: E402
from voxel_b200 import solver as vs  # noqa: E402
from voxel_b200.api import ElasticitySolver  # noqa: E402
from voxel_b200.slab import SlabComm, SlabHierarchy, SlabSolver  # noqa: E402

KE = vo.quadrature([1, 1, 1], 0.3)
DT = {_lib.VX_F64: (torch.float64, torch.float64), _lib.VX_F32: (torch.float32, torch.float32),
      _lib.VX_BF16_F32: (torch.bfloat16, torch.bfloat16), _lib.VX_F32_BF16AUX: (torch.float32, torch.bfloat16)}


def _s():
    return torch.cuda.current_stream().cuda_stream


def _mask(shape, seed, p=0.06):
    nx, ny, nz = shape
    m = np.ones((nx + 1, ny + 1, nz + 1, 3))
    m[0] = 0.0
    m[np.random.default_rng(seed).random(m.shape) < p] = 0.0
    return m.ravel()


@pytest.mark.parametrize("prec", list(DT))
@pytest.mark.parametrize("ny,nz", [(5, 7), (48, 40)])
def test_layer_partial_matches_oracle(prec, ny, nz):
    it, aux = DT[prec]
    rng = np.random.default_rng(ny + prec)
    P3 = 3 * (ny + 1) * (nz + 1)
    E = torch.as_tensor(1e-3 + rng.random(ny * nz), device="cuda").to(aux)
    u = torch.as_tensor(rng.standard_normal(2 * P3), device="cuda").to(it)
    m = _mask((1, ny, nz), prec, 0.2)
    nm = vx.node_mask_from_dofs(torch.as_tensor(m, device="cuda"))
    ref = vo.product_raw((1, ny, nz), KE, u.double().cpu().numpy() * m, E.double().cpu().numpy()) * m
    arith = torch.float64 if prec == _lib.VX_F64 else torch.float32
    tol = 1e-13 if prec == _lib.VX_F64 else 1e-5
    for side in (0, 1):
        out = torch.empty(P3, dtype=arith, device="cuda")
        _lib.call("vx_layer_partial", prec, ny, nz, _lib.dptr(np.ascontiguousarray(KE)), E.data_ptr(), u.data_ptr(),
                  nm.data_ptr(), side, out.data_ptr(), _s())
        want = ref[side * P3:(side + 1) * P3]
        assert np.max(np.abs(out.double().cpu().numpy() - want)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize("prec", [_lib.VX_F64, _lib.VX_F32])
def test_plane_fix_modes(prec):
    it, aux = DT[prec]
    nodes = 1000
    n3 = 3 * nodes
    rng = np.random.default_rng(5)
    t = lambda a, dt: torch.as_tensor(a, device="cuda").to(dt)          # noqa: E731
    lo, hi, x, r, d = (rng.standard_normal(n3) for _ in range(5))
    bits = rng.integers(0, 8, nodes).astype(np.uint8)
    fr = ((bits[:, None] >> np.arange(3)) & 1).ravel().astype(bool)
    ax = np.where(fr, lo + hi, x)
    want = {0: ax, 1: x + 0.6 * d * (r - ax), 2: 0.5 * np.where(fr, r - ax, 0.0), 3: r - ax}
    tol = 1e-15 if prec == _lib.VX_F64 else 1e-6
    for mode, ref in want.items():
        if mode == 3 and prec != _lib.VX_F64:
            continue
        out = t(rng.standard_normal(n3), it)
        held = [t(lo, it), t(hi, it), t(bits, torch.uint8), t(x, it), t(r, aux), t(d, aux)]   # alive during the call
        with_dot = mode in (0, 3)
        G = int(_lib.load().vx_plane_fix_partials(nodes))
        dot = torch.zeros(G, dtype=torch.float64, device="cuda") if with_dot else None
        _lib.call("vx_plane_fix", prec, mode, nodes, *[h.data_ptr() for h in held[:6]], 0.6, 0.5, out.data_ptr(),
                  None if dot is None else dot.data_ptr(), 1, _s())
        got = out.double().cpu().numpy()
        assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref)) * 4
        if with_dot:                 # owned plane: its rewritten terms x.out or out^2
            w = held[3].double().cpu().numpy() if mode == 0 else got
            assert abs(float(dot.sum()) - float(np.sum(w * got))) <= 1e-12 * np.sum(np.abs(w * got))


def _problem(shape, seed=0, interior_fixed=False):
    rho = vx.problems.gaussian_random_field(shape, 8.0, seed)
    E = vx.problems.simp_modulus(rho, 1e-9)
    mask, force = vx.problems.cantilever_equal_split(shape)
    if interior_fixed:
        mask = mask * torch.as_tensor(_mask(shape, seed, 0.02), device="cuda")
        force = force * mask
    return E, mask, force


def _hier(shape, E, mask, nparts, dtype=torch.float64, aux=None, **kw):
    nm = vx.node_mask_from_dofs(mask)
    return SlabHierarchy(shape, KE, E, nm, nparts, SlabComm(nparts), dtype, aux, **kw), nm


def _split(H, v):
    return {i: v[3 * L.a * L.P:3 * L.a * L.P + L.n].contiguous() for i, L in H._level(0)}


def _join(H, parts):
    return torch.cat([parts[i][:L.n_own] for i, L in H._level(0)])


@pytest.mark.parametrize("nparts", [1, 2, 3])
def test_slab_operator_matches_the_single_grid(nparts):
    shape = (48, 12, 20)
    E, mask, _ = _problem(shape, 1, interior_fixed=True)
    H, nm = _hier(shape, E, mask, nparts, max_coarse_x=12)
    u = torch.randn(3 * vo.n_nodes(shape), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    y = vx.VoxelOperator(shape, KE).matvec(u, E, nm)
    us = _split(H, u)
    ys = {i: torch.empty_like(us[i]) for i in us}
    H.apply64(0, us, ys)
    got = _join(H, ys)
    assert float((got - y).abs().max() / y.abs().max()) <= 1e-12
    for i, L in H._level(0):
        if L.has_hi:                                   # both holders of a shared plane agree exactly
            assert torch.equal(ys[i][L.n - 3 * L.P:], ys[i + 1][:3 * L.P])


@pytest.mark.parametrize("dtype,aux,tol", [(torch.float64, None, 1e-11), (torch.float32, None, 2e-5),
                                           (torch.float32, torch.bfloat16, 3e-2), (torch.bfloat16, None, 3e-2)])
def test_slab_vcycle_matches_the_single_grid(dtype, aux, tol):
    shape = (128, 64, 64)
    E, mask, force = _problem(shape)
    nm = vx.node_mask_from_dofs(mask)
    M = vs.MGHierarchy(shape, KE, E, nm, dtype, pre=2, post=2, omegas=0.6, aux_dtype=aux)
    ref = M(force)
    H = SlabHierarchy(shape, KE, E, nm, 4, SlabComm(4), dtype, aux, pre=2, post=2, omegas=0.6)
    zs = H.emit(_split(H, force))
    got = _join(H, {i: z.double() for i, z in zs.items()})
    d = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
    print(f"slab V-cycle ({dtype}, aux {aux}) vs single grid: {d:.2e}")
    assert d <= tol
    for i, L in H._level(0):
        if L.has_hi:
            assert torch.equal(zs[i][L.n - 3 * L.P:], zs[i + 1][:3 * L.P])


def test_slab_spectral_omegas_match_the_single_grid():
    shape = (128, 64, 64)
    E, mask, _ = _problem(shape)
    nm = vx.node_mask_from_dofs(mask)
    M = vs.MGHierarchy(shape, KE, E, nm, torch.float32, omegas="spectral")
    H = SlabHierarchy(shape, KE, E, nm, 3, SlabComm(3), torch.float32, omegas="spectral")
    assert np.allclose(H.lambdas, M.lambdas, rtol=1e-10, atol=0)


@pytest.mark.parametrize("precision,nparts,extra", [("mixed", 4, 0), ("fp64", 2, 0), ("bf16", 3, 1),
                                                    ("mixed", 1, 0)])
def test_slab_gmg_128x64x64_solve(precision, nparts, extra):
    c = golden("gmg_128x64x64.json")
    shape = (128, 64, 64)
    E, mask, force = _problem(shape)
    s = SlabSolver(shape, E, mask, nparts, precision=precision, pre=2, post=2, omega=0.6, check_every=1)
    res = s.solve(force)
    x = s.gather()
    comp = float(force @ x)
    print(f"slab {precision} x{nparts}: {res.iterations} iterations, rel {res.rel:.3e}, compliance {comp!r}")
    assert res.converged and res.rel <= 1e-8
    assert res.iterations <= c["fp32"]["iterations"] + extra
    assert abs(comp - c["fp64"]["compliance"]) <= 1e-7 * c["fp64"]["compliance"]
    assert torch.all(x[mask == 0] == 0)


def test_slab_solve_with_fixed_nodes_on_shared_planes():
    shape = (64, 32, 32)
    E, mask, force = _problem(shape, 2, interior_fixed=True)
    one = ElasticitySolver(shape, E, mask, precision="mixed", tol=1e-10, maxiter=300)
    r1 = one.solve(force)
    x1 = r1.x.clone()
    s = SlabSolver(shape, E, mask, 3, precision="mixed", tol=1e-10, maxiter=300)
    r3 = s.solve(force)
    x3 = s.gather()
    print(f"fixed interior nodes: single grid {r1.iterations}, 3 slabs {r3.iterations} iterations")
    assert r1.converged and r3.converged and abs(r1.iterations - r3.iterations) <= 1
    assert float((x3 - x1).abs().max() / x1.abs().max()) <= 1e-8
    assert torch.all(x3[mask == 0] == 0)


def test_slab_warm_start_returns_at_once():
    shape = (64, 32, 32)
    E, mask, force = _problem(shape, 4)
    s = SlabSolver(shape, E, mask, 2, precision="mixed")
    r = s.solve(force)
    x = s.gather()
    r2 = s.solve(force, x0=x)
    assert r.converged and r2.converged and r2.iterations == 0


@pytest.mark.parametrize("check_every", [1, 5])
def test_slab_graph_loop_matches_the_host_loop(check_every):
    """The WHILE-graph loop (every slab in one process) and the host-driven loop (the path of one
    slab per process) run the same kernels: identical iterations and bitwise-equal solutions."""
    shape = (128, 64, 64)
    E, mask, force = _problem(shape)
    out = []
    for graph in (True, False):
        s = SlabSolver(shape, E, mask, 3, precision="mixed", check_every=check_every, graph=graph)
        r = s.solve(force)
        out.append((r.iterations, r.rel, s.gather().clone()))
        r2 = s.solve(force)                                # a second solve reuses the captured graph
        assert r2.iterations == r.iterations and torch.equal(s.gather(), out[-1][2])
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1] and torch.equal(out[0][2], out[1][2])


@pytest.mark.parametrize("lo,hi", [(0, 33), (1, 32), (1, 33), (5, 6), (0, 0)])
def test_reductions_over_a_node_plane_range(lo, hi):
    """vx_apply_dot_planes / vx_true_residual_planes: the output as vx_apply_dot / vx_true_residual,
    the partial sums over node planes lo <= ix < hi only."""
    shape = (32, 16, 24)
    E, mask, force = _problem(shape, 3)
    nm = vx.node_mask_from_dofs(mask)
    op = vx.VoxelOperator(shape, KE)
    g = torch.Generator("cuda").manual_seed(4)
    p = torch.randn(op.ndof, dtype=torch.float64, device="cuda", generator=g)
    P3 = 3 * 17 * 25
    G = op.partials_size
    part = torch.zeros(G, dtype=torch.float64, device="cuda")
    q = torch.empty_like(p)
    _lib.call("vx_apply_dot_planes", _lib.VX_F64, *shape, op._bp, E.data_ptr(), nm.data_ptr(), p.data_ptr(),
              q.data_ptr(), part.data_ptr(), lo, hi, _s())
    q_ref = op.matvec(p, E, nm)
    assert torch.equal(q, q_ref)
    want = float(p[lo * P3:hi * P3] @ q_ref[lo * P3:hi * P3])
    assert abs(float(part.sum()) - want) <= 1e-12 * float((p * q_ref).abs().sum())
    res = torch.empty_like(p)
    _lib.call("vx_true_residual_planes", _lib.VX_F64, *shape, op._bp, E.data_ptr(), nm.data_ptr(), p.data_ptr(),
              force.data_ptr(), res.data_ptr(), part.data_ptr(), lo, hi, _s())
    r_ref = force - q_ref
    assert float((res - r_ref).abs().max()) <= 1e-13 * float(r_ref.abs().max())
    want = float(r_ref[lo * P3:hi * P3] @ r_ref[lo * P3:hi * P3])
    assert abs(float(part.sum()) - want) <= 1e-12 * float((r_ref * r_ref).sum()) + 1e-300


def _free_port():
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _slab_rank(rank, world, port, q):
    """One slab per process on the same GPU, exchanging through a gloo group (host-staged): the
    multi-process path of the solver end to end.  Every exchange completes on the host before the
    next launch, so no kernel of one process waits on another's."""
    import datetime
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        E, mask, force = _problem((128, 64, 64))
        s = SlabSolver((128, 64, 64), E, mask, world, precision="mixed", check_every=1)
        res = s.solve(force)
        x = s.gather()
        q.put((rank, s.comm.distributed, s.comm.staged, s.use_graph, res.iterations, res.rel, float(force @ x),
               bool(torch.all(x[mask == 0] == 0)), float(x.abs().sum())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_solve_across_processes(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    c = golden("gmg_128x64x64.json")
    for g in got:
        _, distributed, staged, graph, it, rel, comp, fixed_zero, l1 = g
        print(f"rank {g[0]}/{world}: {it} iterations, rel {rel:.3e}, compliance {comp!r}")
        assert distributed and staged and not graph
        assert it == c["fp32"]["iterations"] and rel <= 1e-8 and fixed_zero
        assert abs(comp - c["fp64"]["compliance"]) <= 1e-7 * c["fp64"]["compliance"]
    assert len({(g[4], g[5], g[6], g[8]) for g in got}) == 1        # every rank holds the same result


def _slab_kat(case, nparts, precision="mixed"):
    """The reference's published known answer (experiments/session_i, V(4,4), spectral omega from
    the FP64 hierarchy) solved on x-slabs."""
    k = golden("kat_inputs.npz")
    kat = golden("kat_session_i.json")
    base = "q64" if case.startswith("q64") else "q96"
    rho_nat, shape = vx.problems.upsample_natural(k[f"{base}_rho"], tuple(int(s) for s in k[f"{base}_shape"]),
                                                  int(case[-1]))
    mask_nat, force_nat = vx.problems.cantilever_line_load(shape)
    floor = kat["_protocol"]["material"]["Emin"]
    cu = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")          # noqa: E731
    E = cu(vx.to_author(floor + (1 - floor) * rho_nat ** 3, shape))
    mask = cu(vx.to_author(mask_nat, shape, True))
    force = cu(vx.to_author(force_nat, shape, True))
    mgp = kat["_protocol"]["multigrid"]
    s = SlabSolver(shape, E, mask, nparts, ke=k[f"{base}_ke"], precision=precision, pre=mgp["pre"], post=mgp["post"],
                   omega="spectral", max_coarse_x=mgp["max_coarse_x"], tol=1e-8, maxiter=200, check_every=1,
                   spectral_seed=kat["_protocol"]["order_seed"])
    assert [list(s_) for s_ in s.M.shapes] == kat[case]["shapes"]
    res = s.solve(force)
    x = s.gather()
    return res, float(force @ x), float(torch.linalg.vector_norm(x)), kat[case]["observations"]


@pytest.mark.parametrize("case,nparts", [("q64x2", 3), ("q96x3", 4)])
def test_slab_reference_published_kat(case, nparts):
    """q64x2 (256x128x128, 14 iterations, 807.19637074) on 3 slabs and the headline q96x3
    (576x288x288, 144.6M DOF, 20 iterations, 543.42238043-543.42238050) on 4 slabs: the published
    iteration counts, compliances and solution norms (1e-9 relative)."""
    res, comp, norm, obs = _slab_kat(case, nparts)
    print(f"slab {case} x{nparts}: {res.iterations} iterations (published {obs[0]['iterations']}), compliance {comp!r}")
    assert res.converged and res.iterations == obs[0]["iterations"]
    ref_c = np.array([o["compliance"] for o in obs])
    assert np.min(np.abs(comp - ref_c)) <= 1e-9 * ref_c.mean()
    ref_n = np.array([o["solution_norm"] for o in obs])
    assert np.min(np.abs(norm - ref_n)) <= 1e-9 * ref_n.mean()
