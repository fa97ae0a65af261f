"""Generate the golden fixtures under tests/golden/ by running the REFERENCE itself.

Run in a container that has the reference checkout (read-only) and g++:

    python tests/golden/make_golden.py [--ref <reference checkout>]    (default: $VOXEL_REF, else /root/reference)

It imports the reference's own Python modules (src/voxel_mg.py, src/voxel_kernels.py,
code/hex_modal/modal.py, experiments/session_a/dependencies/common.py, the donor
experiments/session_a/donor/src/gpu_fem/simp_r2.py with NumPy standing in for CuPy, and
experiments/session_h/run_w1b.py) and the reference's compiled C++ product (built from
experiments/session_a/inputs/reference.cc by ``make -C oracle``), runs them on seeded inputs and
on the reference's own fixtures, and writes small compressed .npz / .json files.  Nothing in the
test suite reads the reference checkout; the fixtures are the only bridge.
"""
from __future__ import annotations

import argparse
import os
import importlib.util
import json
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


DONOR_CASES = (
    ("cant_patch_a", "cantilever", (8, 4, 2), dict(load="patch")),
    ("cant_patch_b", "cantilever", (16, 8, 4), dict(load="patch", patch_frac=0.5)),
    ("cant_patch_c", "cantilever", (12, 6, 6), dict(load="patch", patch_size=0.3, total_load=-2.0)),
    ("cant_point", "cantilever", (16, 8, 4), dict(load="point")),
    ("torsion_a", "torsion", (12, 4, 4), dict()),
    ("torsion_b", "torsion", (9, 6, 6), dict(patch_size=0.4, total_load=2.5)),
)


def donor_problems(ref):
    """The donor's problem builders (simp_r2.py:64-178): supports and loads in author layout."""
    sys.modules["cupy"] = np
    simp = load("ref_simp_r2_problems", ref / "experiments/session_a/donor/src/gpu_fem/simp_r2.py")
    del sys.modules["cupy"]
    out = {}
    for tag, kind, dims, kw in DONOR_CASES:
        fn = simp.build_cantilever if kind == "cantilever" else simp.build_torsion
        d = fn(*dims, **kw)
        out[f"{tag}_fixed"] = np.asarray(d["fixed"])
        out[f"{tag}_F"] = np.asarray(d["F"])
        out[f"{tag}_patch_nodes"] = np.array(d["patch_nodes"])
    np.savez_compressed(HERE / "donor_problems.npz", **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", type=Path, default=Path(os.environ.get("VOXEL_REF", "/root/reference")))
    ap.add_argument("--skip-slow", action="store_true", help="skip the 128x64x64 GMG solves (~1 min)")
    ap.add_argument("--only", choices=("donor_problems",), help="write one fixture file only")
    args = ap.parse_args()
    ref = args.ref.resolve()
    if args.only == "donor_problems":
        donor_problems(ref)
        return

    subprocess.run(["make", "-C", str(REPO / "oracle"), f"REF={ref}"], check=True)
    mg = load("ref_voxel_mg", ref / "src/voxel_mg.py")
    vk = load("ref_voxel_kernels", ref / "src/voxel_kernels.py")
    modal = load("ref_modal", ref / "code/hex_modal/modal.py")
    common = load("ref_common", ref / "experiments/session_a/dependencies/common.py")
    Ref = common.Reference(REPO / "oracle/_ref/libreference.so")

    # ------------------------------------------------------------------ element + lane emulation
    ke_unit = modal.quadrature([1.0, 1.0, 1.0], 0.3)
    m_unit = modal.Modal(ke_unit)
    ke_brick = modal.quadrature([1.0, 0.5, 2.0], 0.25)
    m_brick = modal.Modal(ke_brick)
    ke_c = np.zeros(576)
    Ref.lib.element.argtypes = [__import__("ctypes").c_double, __import__("ctypes").c_double,
                                np.ctypeslib.ndpointer(dtype=np.float64, ndim=1, flags="C_CONTIGUOUS")]
    Ref.lib.element(1.0, 0.3, ke_c)
    smoke = dict(np.load(ref / "experiments/session_a/inputs/smoke-q4.npz"))
    m_fix = modal.Modal(smoke["ke"])
    shape_e = (3, 2, 4)                                     # tests/test_kernels_cpu.py:14-24
    rng = np.random.default_rng(7)
    E_e = 1e-6 + (1 - 1e-6) * rng.random(int(np.prod(shape_e))) ** 3
    u_e = rng.standard_normal(3 * int(np.prod(np.array(shape_e) + 1)))
    np.savez_compressed(
        HERE / "element.npz",
        ke_unit=ke_unit, blocks_unit=m_unit.blocks, discarded_unit=m_unit.discarded_relative,
        ke_c_unit=ke_c.reshape(24, 24), ke_brick=ke_brick, blocks_brick=m_brick.blocks,
        ke_fixture=smoke["ke"], blocks_fixture=m_fix.blocks,
        emu_shape=np.array(shape_e), emu_E=E_e, emu_u=u_e,
        emu_assembled=vk.assembled_reference(shape_e, ke_unit, E_e, u_e),
        emu_modal8_fp64=vk.emulate("modal8", shape_e, ke_unit, E_e, u_e, np.float64),
        emu_modal8_fp32=vk.emulate("modal8", shape_e, ke_unit, E_e, u_e, np.float32),
        emu_dense8_fp64=vk.emulate("dense8", shape_e, ke_unit, E_e, u_e, np.float64),
        element_nodes=vk.element_nodes(shape_e), edof=mg.edof_author(shape_e))

    # ------------------------------------------------------------------ products
    out = {}
    shape_s = tuple(int(s) for s in smoke["shape"])
    u_nat = np.random.default_rng(11).standard_normal(smoke["mask"].size)
    y_c, ce_c, d_c = Ref.product({"shape": smoke["shape"], "rho": smoke["rho"], "ke": smoke["ke"],
                                  "mask": smoke["mask"], "floor": 1e-6}, u_nat)
    out.update(smoke_shape=np.array(shape_s), smoke_rho=smoke["rho"], smoke_mask=smoke["mask"],
               smoke_force=smoke["force"], smoke_ke=smoke["ke"], smoke_u=u_nat,
               smoke_c_y=y_c, smoke_c_ce=ce_c, smoke_c_diag=d_c)
    # heterogeneous density through the C product (natural layout), Emin=1e-9
    rho_h = np.random.default_rng(12).uniform(0.01, 1.0, smoke["rho"].size)
    y_h, ce_h, d_h = Ref.product({"shape": smoke["shape"], "rho": rho_h, "ke": ke_unit,
                                  "mask": smoke["mask"], "floor": 1e-9}, u_nat)
    out.update(het_rho=rho_h, het_c_y=y_h, het_c_ce=ce_h, het_c_diag=d_h)
    for tag, shape in (("s111", (1, 1, 1)), ("s537", (5, 3, 7)), ("s324", (3, 2, 4)), ("s2x", (6, 4, 2))):
        g = np.random.default_rng(sum(map(ord, tag)))
        E = 1e-9 + (1 - 1e-9) * g.random(int(np.prod(shape))) ** 3
        u = g.standard_normal(3 * int(np.prod(np.array(shape) + 1)))
        P = mg.NumpyProduct(shape, ke_unit)
        out.update({f"{tag}_shape": np.array(shape), f"{tag}_E": E, f"{tag}_u": u,
                    f"{tag}_raw": P.raw(u, E), f"{tag}_diag": P.diagonal(E),
                    f"{tag}_raw32": mg.NumpyProduct(shape, ke_unit, np.float32).raw(
                        u.astype(np.float32), E.astype(np.float32))})
    np.savez_compressed(HERE / "products.npz", **out)

    # ------------------------------------------------------------------ transfers / hierarchy
    out = {}
    g = np.random.default_rng(1)
    for tag, coarse in (("a", (2, 1, 1)), ("b", (3, 2, 2)), ("c", (1, 1, 1))):
        fine = tuple(2 * s for s in coarse)
        c = g.standard_normal(3 * int(np.prod(np.array(coarse) + 1)))
        f = g.standard_normal(3 * int(np.prod(np.array(fine) + 1)))
        out.update({f"{tag}_coarse": np.array(coarse), f"{tag}_c": c, f"{tag}_f": f,
                    f"{tag}_prolong": mg.prolong(np, c, coarse), f"{tag}_restrict": mg.restrict(np, f, fine)})
    E_s = common.to_author(1e-6 + (1 - 1e-6) * np.random.default_rng(5).random(128) ** 3, shape_s)
    m_s = common.to_author(smoke["mask"], shape_s, True)
    out.update(cm_E=E_s, cm_mask=m_s, cm_Ec=mg.coarsen_modulus(np, E_s, shape_s),
               cm_maskc=mg.coarsen_mask(np, m_s, shape_s))
    table = {}
    for shape in ((8, 4, 4), (32, 16, 16), (128, 64, 64), (48, 24, 24), (96, 48, 48), (160, 80, 80),
                  (256, 128, 128), (192, 96, 96), (576, 288, 288), (6, 5, 4), (18, 9, 9)):
        for mcx in (2, 16):
            table[f"{shape}|{mcx}"] = mg.hierarchy_shapes(shape, mcx)
    (HERE / "hierarchy.json").write_text(json.dumps(table, indent=0) + "\n")
    # natural <-> author round trip on the smoke fixture
    out.update(layout_nat=smoke["force"], layout_author=common.to_author(smoke["force"], shape_s, True),
               layout_rho_author=common.to_author(smoke["rho"] * np.arange(128), shape_s))
    np.savez_compressed(HERE / "transfers.npz", **out)

    # ------------------------------------------------------------------ multigrid on smoke-q4
    KE = smoke["ke"]
    E = common.to_author(1e-6 + (1 - 1e-6) * smoke["rho"] ** 3, shape_s)
    mask = common.to_author(smoke["mask"], shape_s, True)
    force = common.to_author(smoke["force"], shape_s, True)

    def build(shape, E, mask, dtype=np.float64, max_coarse_x=2, pre=4, post=4, spectral=True):
        shapes = mg.hierarchy_shapes(shape, max_coarse_x)
        prods = [mg.NumpyProduct(s, KE * 2 ** i, dtype) for i, s in enumerate(shapes)]
        Ec, mc = E, mask
        for i in range(1, len(shapes)):
            Ec, mc = mg.coarsen_modulus(np, Ec, shapes[i - 1]), mg.coarsen_mask(np, mc, shapes[i - 1])
        A = mg.assemble_dense(shapes[-1], KE * 2 ** (len(shapes) - 1), Ec, mc)
        factor = np.linalg.cholesky(A)
        M = mg.Multigrid(np, shapes, prods, E, mask, factor, dtype, pre=pre, post=post)
        lambdas = None
        if spectral:
            M.omegas, lambdas = mg.spectral_omegas(np, M.levels)
        return shapes, M, factor, A, lambdas

    def apply_fine(shape, E, mask, ke=KE):
        P = mg.NumpyProduct(shape, ke)
        return lambda u: P.raw(u * mask, E) * mask + u * (1 - mask)

    shapes, M, factor, Acoarse, lambdas = build(shape_s, E, mask)
    r = np.random.default_rng(2).standard_normal(mask.size) * mask
    _, M32, _, _, _ = build(shape_s, E, mask, dtype=np.float32)
    x, it, ok, rel, mv = mg.fcg(np, apply_fine(shape_s, E, mask), force, M, 1e-8, 200)
    x1, it1, ok1, rel1, mv1 = mg.fcg(np, apply_fine(shape_s, E, mask), force, M, 1e-8, 200, check_every=1)
    x7, it7, _, rel7, mv7 = mg.fcg(np, apply_fine(shape_s, E, mask), force, M, 1e-8, 999, fixed_iterations=7)
    _, M06, _, _, _ = build(shape_s, E, mask, pre=2, post=2, spectral=False)
    x06, it06, ok06, rel06, mv06 = mg.fcg(np, apply_fine(shape_s, E, mask), force, M06, 1e-8, 200)
    np.savez_compressed(
        HERE / "mg_smoke.npz", shapes=np.array(shapes), E=E, mask=mask, force=force, ke=KE,
        omegas=np.array(M.omegas), lambdas=np.array(lambdas), factor=factor, A_coarse=Acoarse,
        r=r, vcycle64=M(r), vcycle32=M32(r), inv_diag0=M.levels[0].inv_diag,
        fcg_x=x, fcg_it=it, fcg_ok=ok, fcg_rel=rel, fcg_mv=mv,
        fcg1_x=x1, fcg1_it=it1, fcg1_rel=rel1, fcg1_mv=mv1,
        fcg7_x=x7, fcg7_it=it7, fcg7_rel=rel7, fcg7_mv=mv7,
        fcg06_x=x06, fcg06_it=it06, fcg06_rel=rel06, fcg06_mv=mv06)

    # ------------------------------------------------------------------ 32x16x16, Jacobi
    shape1 = (32, 16, 16)
    Ne1 = int(np.prod(shape1))
    rho1 = np.random.default_rng(0).uniform(0.01, 1.0, Ne1)
    E1 = 1e-9 + (1 - 1e-9) * rho1 ** 3
    nx, ny, nz = shape1
    m1 = np.ones((nx + 1, ny + 1, nz + 1, 3)); m1[0] = 0
    f1 = np.zeros((nx + 1, ny + 1, nz + 1, 3)); f1[nx, :, 0, 2] = -1.0 / (ny + 1)
    m1, f1 = m1.ravel(), f1.ravel()
    P1 = mg.NumpyProduct(shape1, ke_unit)
    A1 = lambda u: P1.raw(u * m1, E1) * m1 + u * (1 - m1)
    d1 = P1.diagonal(E1)
    inv1 = 1 / np.where(m1 != 0, d1, 1.0)
    t = time.perf_counter()
    xj, itj, okj, relj, mvj = mg.fcg(np, A1, f1, lambda v: inv1 * v, 1e-8, 5000, check_every=50)
    tj = time.perf_counter() - t
    # donor Jacobi-PCG, NumPy standing in for CuPy (the donor only uses dot/norm/zeros_like)
    sys.modules["cupy"] = np
    simp = load("ref_simp_r2", ref / "experiments/session_a/donor/src/gpu_fem/simp_r2.py")
    xp_, itp, okp, relp = simp.pcg(A1, f1, inv1, tol=1e-8, maxiter=5000, mask=m1, check_every=50)
    A1_32 = lambda u: (P1.raw(u * m1, E1).astype(np.float32) * m1.astype(np.float32)
                       + u * (1 - m1).astype(np.float32))
    xi, outer_i, inner_i, oki, reli = simp.pcg_ir(A1, f1, A1_32, inv1.astype(np.float32), tol=1e-8,
                                                  mask32=m1.astype(np.float32), inner_tol=1e-1,
                                                  max_outer=40, inner_maxiter=4000, check_every=50)
    del sys.modules["cupy"]
    np.savez_compressed(
        HERE / "jacobi_32x16x16.npz", shape=np.array(shape1), rho=rho1, E=E1, mask=m1, force=f1,
        fcg_x=xj, fcg_it=itj, fcg_ok=okj, fcg_rel=relj, fcg_mv=mvj, fcg_compliance=float(f1 @ xj),
        fcg_seconds=tj, pcg_x=xp_, pcg_it=itp, pcg_ok=okp, pcg_rel=relp,
        ir_x=xi, ir_outer=outer_i, ir_inner=inner_i, ir_ok=oki, ir_rel=reli)

    # ------------------------------------------------------------------ filter + OC (top88)
    rw = load("ref_run_w1b", ref / "experiments/session_h/run_w1b.py")
    out = {}
    for tag, dims, rmin in (("f1", (6, 4, 5), 1.5), ("f2", (5, 7, 3), 2.2), ("f3", (4, 4, 4), 1.0)):
        flt = rw.DensityFilter(dims, rmin)
        g = np.random.default_rng(sum(map(ord, tag)))
        a, b = g.random(int(np.prod(dims))), g.standard_normal(int(np.prod(dims)))
        out.update({f"{tag}_dims": np.array(dims), f"{tag}_rmin": rmin, f"{tag}_a": a, f"{tag}_b": b,
                    f"{tag}_density": flt.density(a), f"{tag}_gradient": flt.gradient(b), f"{tag}_Hs": flt.Hs})
    dims = (12, 6, 6)
    flt = rw.DensityFilter(dims, 1.5)
    g = np.random.default_rng(99)
    x0 = 0.12 + g.uniform(-0.01, 0.01, int(np.prod(dims)))
    dc = -g.random(x0.size) * 10
    dv = flt.gradient(np.ones_like(x0))
    dcx = flt.gradient(dc)
    out.update(oc_dims=np.array(dims), oc_x=x0, oc_dc=dcx, oc_dv=dv,
               oc_new_tol3=rw.oc_top88(x0, dcx, dv, 0.12, 0.2, density=flt.density),
               oc_new_tol6=rw.oc_top88(x0, dcx, dv, 0.12, 0.2, density=flt.density, tol=1e-6))
    np.savez_compressed(HERE / "filter_oc.npz", **out)

    # ------------------------------------------------------------------ reference KAT inputs + numbers
    q64 = dict(np.load(ref / "experiments/session_a/inputs/optimized-q64.npz"))
    q96 = dict(np.load(ref / "experiments/session_a/inputs/optimized-q96.npz"))
    np.savez_compressed(HERE / "kat_inputs.npz",
                        q64_shape=q64["shape"], q64_rho=q64["rho"], q64_ke=q64["ke"],
                        q96_shape=q96["shape"], q96_rho=q96["rho"], q96_ke=q96["ke"])
    numbers = json.loads((ref / "paper/session_i_numbers.json").read_text())
    kat = {}
    for gpu, rec in numbers.items():
        for case, c in rec["cases"].items():
            for o in c["to_tolerance_observations"]:
                kat.setdefault(case, {"shapes": c["shapes"], "observations": []})["observations"].append(
                    {k: o[k] for k in ("arm", "iterations", "compliance", "solution_norm",
                                       "native_true_residual", "solver_seconds")} | {"gpu": rec["gpu"]})
    proto = json.loads((ref / "experiments/session_i/protocol.json").read_text())
    kat["_protocol"] = {"material": proto["material"], "solver": proto["solver"],
                        "multigrid": proto["multigrid"], "order_seed": proto["order_seed"]}
    (HERE / "kat_session_i.json").write_text(json.dumps(kat, indent=1) + "\n")

    # ------------------------------------------------------------------ 128x64x64, GMG
    if not args.skip_slow:
        sys.path.insert(0, str(REPO))
        from oracle.voxel_oracle import gaussian_random_field
        shape2 = (128, 64, 64)
        rho2 = gaussian_random_field(shape2, 8.0, 0)
        E2 = 1e-9 + (1 - 1e-9) * rho2 ** 3
        nx, ny, nz = shape2
        m2 = np.ones((nx + 1, ny + 1, nz + 1, 3)); m2[0] = 0
        f2 = np.zeros((nx + 1, ny + 1, nz + 1, 3)); f2[nx, :, 0, 2] = -1.0 / (ny + 1)
        m2, f2 = m2.ravel(), f2.ravel()
        shapes2 = mg.hierarchy_shapes(shape2, 16)
        Ec, mc = E2, m2
        for i in range(1, len(shapes2)):
            Ec, mc = mg.coarsen_modulus(np, Ec, shapes2[i - 1]), mg.coarsen_mask(np, mc, shapes2[i - 1])
        fac2 = np.linalg.cholesky(mg.assemble_dense(shapes2[-1], ke_unit * 2 ** (len(shapes2) - 1), Ec, mc))
        P2 = mg.NumpyProduct(shape2, ke_unit)
        A2 = lambda u: P2.raw(u * m2, E2) * m2 + u * (1 - m2)
        res2 = {}
        idx = np.random.default_rng(3).choice(m2.size, 4096, replace=False)
        for tag, dt in (("fp64", np.float64), ("fp32", np.float32)):
            prods = [mg.NumpyProduct(s, ke_unit * 2 ** i, dt) for i, s in enumerate(shapes2)]
            M2 = mg.Multigrid(np, shapes2, prods, E2, m2, fac2, dt, pre=2, post=2)
            t = time.perf_counter()
            x2, it2, ok2, rel2, mv2 = mg.fcg(np, A2, f2, M2, 1e-8, 200)
            res2[tag] = {"iterations": it2, "converged": ok2, "rel": rel2, "matvecs": mv2,
                         "compliance": float(f2 @ x2), "norm": float(np.linalg.norm(x2)),
                         "seconds": time.perf_counter() - t}
            res2[tag]["samples"] = x2[idx].tolist()
        res2["sample_index"] = idx.tolist()
        res2["rho_stats"] = [float(rho2.min()), float(rho2.max()), float(rho2.mean())]
        res2["rho_head"] = rho2[:16].tolist()
        res2["shapes"] = shapes2
        (HERE / "gmg_128x64x64.json").write_text(json.dumps(res2) + "\n")
    donor_problems(ref)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
