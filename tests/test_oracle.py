"""Pins the CPU oracle (oracle/voxel_oracle.py) to golden vectors produced by the reference itself
(tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import golden
from oracle import voxel_oracle as vo
from oracle import ref_product


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def maxrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


# ----------------------------------------------------------------------------- element
def test_quadrature_matches_reference():
    g = golden("element.npz")
    assert maxrel(vo.quadrature([1, 1, 1], 0.3), g["ke_unit"]) < 1e-15
    assert maxrel(vo.quadrature([1.0, 0.5, 2.0], 0.25), g["ke_brick"]) < 1e-15
    assert maxrel(g["ke_unit"], g["ke_c_unit"]) < 1e-15          # modal.py quadrature == reference.cc element()


def test_parity_blocks_match_reference_bitwise_structure():
    g = golden("element.npz")
    for ke, blocks in ((g["ke_unit"], g["blocks_unit"]), (g["ke_brick"], g["blocks_brick"]),
                       (g["ke_fixture"], g["blocks_fixture"])):
        b, disc = vo.parity_blocks(ke)
        assert np.abs(b - blocks).max() <= 1e-16 * np.abs(blocks).max() * 8
        assert disc < 2e-14
    nz = int((np.abs(g["blocks_unit"]) > 1e-14 * np.abs(g["blocks_unit"]).max()).sum())
    assert nz == 45                                  # 45 of 72 entries are non-zero for the unit cube


def test_parity_blocks_reject_non_brick_element():
    ke = vo.quadrature([1, 1, 1], 0.3).copy()
    ke[0, 5] += 1e-3
    ke[5, 0] += 1e-3
    with pytest.raises(ValueError):
        vo.parity_blocks(ke)


def test_index_maps_bit_exact():
    g = golden("element.npz")
    shape = tuple(g["emu_shape"])
    assert np.array_equal(vo.element_nodes(shape), g["element_nodes"])
    assert np.array_equal(vo.edof_author(shape), g["edof"])


def test_dense_product_matches_reference_lane_emulation():
    g = golden("element.npz")
    shape = tuple(g["emu_shape"])
    y = vo.product_raw(shape, g["ke_unit"], g["emu_u"], g["emu_E"])
    assert rel(y, g["emu_assembled"]) < 1e-14
    assert rel(y, g["emu_modal8_fp64"]) < 1e-13


# ----------------------------------------------------------------------------- products
@pytest.mark.parametrize("tag", ["s111", "s537", "s324", "s2x"])
def test_product_raw_and_diagonal(tag):
    g = golden("products.npz")
    shape = tuple(g[f"{tag}_shape"])
    assert maxrel(vo.product_raw(shape, vo.quadrature([1, 1, 1], 0.3), g[f"{tag}_u"], g[f"{tag}_E"]),
                  g[f"{tag}_raw"]) < 1e-14
    assert maxrel(vo.product_diagonal(shape, vo.quadrature([1, 1, 1], 0.3), g[f"{tag}_E"]),
                  g[f"{tag}_diag"]) < 1e-15


def test_c_reference_product_restatement():
    g = golden("products.npz")
    shape = tuple(g["smoke_shape"])
    for rho, ke, emin, key in ((g["smoke_rho"], g["smoke_ke"], 1e-6, "smoke"),
                               (g["het_rho"], vo.quadrature([1, 1, 1], 0.3), 1e-9, "het")):
        y, ce, d = vo.c_reference_product(shape, rho, g["smoke_u"], ke, g["smoke_mask"], emin)
        assert maxrel(y, g[f"{key}_c_y"]) < 1e-13
        assert maxrel(ce, g[f"{key}_c_ce"]) < 1e-13
        assert maxrel(d, g[f"{key}_c_diag"]) < 1e-14


@pytest.mark.skipif(not ref_product.available(), reason="oracle/_ref not built (make -C oracle)")
def test_compiled_reference_matches_golden():
    g = golden("products.npz")
    R = ref_product.ReferenceProduct()
    y, ce, d = R.product(g["smoke_shape"], g["smoke_rho"], g["smoke_u"], g["smoke_ke"], g["smoke_mask"], 1e-6)
    assert np.array_equal(y, g["smoke_c_y"]) and np.array_equal(ce, g["smoke_c_ce"])


# ----------------------------------------------------------------------------- transfers / layout
@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_transfers(tag):
    g = golden("transfers.npz")
    coarse = tuple(g[f"{tag}_coarse"])
    fine = tuple(2 * s for s in coarse)
    assert maxrel(vo.prolong(g[f"{tag}_c"], coarse), g[f"{tag}_prolong"]) < 1e-15
    assert maxrel(vo.restrict(g[f"{tag}_f"], fine), g[f"{tag}_restrict"]) < 1e-15


def test_coarsening_and_layout():
    g = golden("transfers.npz")
    shape = (8, 4, 4)
    assert maxrel(vo.coarsen_modulus(g["cm_E"], shape), g["cm_Ec"]) < 1e-15
    assert np.array_equal(vo.coarsen_mask(g["cm_mask"], shape), g["cm_maskc"])
    assert np.array_equal(vo.to_author(g["layout_nat"], shape, True), g["layout_author"])
    assert np.array_equal(vo.to_natural(g["layout_author"], shape, True), g["layout_nat"])


def test_hierarchy_shapes():
    table = golden("hierarchy.json")
    for key, shapes in table.items():
        shape, mcx = key.split("|")
        shape = tuple(int(s) for s in shape.strip("()").split(","))
        assert [list(s) for s in vo.hierarchy_shapes(shape, int(mcx))] == shapes


# ----------------------------------------------------------------------------- multigrid
def _smoke_mg(dtype=np.float64, pre=4, post=4, spectral=True):
    g = golden("mg_smoke.npz")
    shapes = [tuple(s) for s in g["shapes"]]
    M = vo.Multigrid(shapes, g["ke"], g["E"], g["mask"], g["factor"], dtype, pre=pre, post=post)
    lam = None
    if spectral:
        M.omegas, lam = vo.spectral_omegas(M.levels)
    return g, M, lam


def test_coarse_factor_and_spectral_omegas():
    g, M, lam = _smoke_mg()
    shapes = [tuple(s) for s in g["shapes"]]
    assert maxrel(vo.coarse_factor(shapes, g["ke"], g["E"], g["mask"]), g["factor"]) < 1e-13
    assert maxrel(lam, g["lambdas"]) < 1e-12
    assert maxrel(M.levels[0].inv_diag, g["inv_diag0"]) < 1e-15


def test_vcycle_fp64_and_fp32():
    g, M, _ = _smoke_mg()
    assert rel(M(g["r"]), g["vcycle64"]) < 1e-12
    _, M32, _ = _smoke_mg(np.float32)
    assert rel(M32(g["r"]), g["vcycle32"]) < 1e-5


def test_fcg_smoke_iterates():
    g, M, _ = _smoke_mg()
    A = lambda u: vo.apply_dirichlet((8, 4, 4), g["ke"], g["E"], g["mask"], u)
    for key, kw in (("fcg", {}), ("fcg1", {"check_every": 1}), ("fcg7", {"fixed_iterations": 7})):
        x, it, ok, r, mv = vo.fcg(A, g["force"], M, 1e-8, 999 if key == "fcg7" else 200, **kw)
        assert it == int(g[f"{key}_it"]) and mv == int(g[f"{key}_mv"])
        assert rel(x, g[f"{key}_x"]) < 1e-9
    g2, M06, _ = _smoke_mg(pre=2, post=2, spectral=False)
    x, it, ok, r, mv = vo.fcg(A, g["force"], M06, 1e-8, 200)
    assert it == int(g["fcg06_it"]) and rel(x, g["fcg06_x"]) < 1e-9


# ----------------------------------------------------------------------------- 32x16x16 Jacobi case
@pytest.mark.slow
def test_jacobi_32x16x16_fcg_and_donor_pcg():
    g = golden("jacobi_32x16x16.npz")
    shape = tuple(g["shape"])
    ke = vo.quadrature([1, 1, 1], 0.3)
    rho = np.random.default_rng(0).uniform(0.01, 1.0, int(np.prod(shape)))
    assert np.array_equal(rho, g["rho"])
    mask, force = vo.cantilever_equal_split(shape)
    assert np.array_equal(mask, g["mask"]) and np.array_equal(force, g["force"])
    E = vo.simp_modulus(rho, 1e-9)
    assert maxrel(E, g["E"]) < 1e-15
    A = lambda u: vo.apply_dirichlet(shape, ke, E, mask, u)
    inv = 1 / np.where(mask != 0, vo.product_diagonal(shape, ke, E), 1.0)
    x, it, ok, r, mv = vo.fcg(A, force, lambda v: inv * v, 1e-8, 5000, check_every=50)
    assert it == int(g["fcg_it"]) == 650 and ok
    assert abs(force @ x - float(g["fcg_compliance"])) <= 1e-10 * abs(float(g["fcg_compliance"]))
    assert rel(x, g["fcg_x"]) < 1e-8
    xp, itp, okp, relp = vo.pcg(A, force, inv, tol=1e-8, maxiter=5000, mask=mask, check_every=50)
    assert itp == int(g["pcg_it"]) and rel(xp, g["pcg_x"]) < 1e-8


@pytest.mark.slow
def test_jacobi_32x16x16_pcg_ir():
    g = golden("jacobi_32x16x16.npz")
    shape = tuple(g["shape"])
    ke = vo.quadrature([1, 1, 1], 0.3)
    mask, force, E = g["mask"], g["force"], g["E"]
    A = lambda u: vo.apply_dirichlet(shape, ke, E, mask, u)
    A32 = lambda u: (vo.product_raw(shape, ke, u * mask, E).astype(np.float32) * mask.astype(np.float32)
                     + u * (1 - mask).astype(np.float32))
    inv = 1 / np.where(mask != 0, vo.product_diagonal(shape, ke, E), 1.0)
    x, outer, inner, ok, r = vo.pcg_ir(A, force, A32, inv.astype(np.float32), tol=1e-8,
                                       mask32=mask.astype(np.float32))
    assert (outer, inner, ok) == (int(g["ir_outer"]), int(g["ir_inner"]), bool(g["ir_ok"]))
    assert rel(x, g["ir_x"]) < 1e-10


# ----------------------------------------------------------------------------- filter / OC
@pytest.mark.parametrize("tag", ["f1", "f2", "f3"])
def test_cone_filter(tag):
    g = golden("filter_oc.npz")
    f = vo.ConeFilter(tuple(g[f"{tag}_dims"]), float(g[f"{tag}_rmin"]))
    assert maxrel(f.s, g[f"{tag}_Hs"]) < 1e-15
    assert maxrel(f.forward(g[f"{tag}_a"]), g[f"{tag}_density"]) < 1e-14
    assert maxrel(f.transpose(g[f"{tag}_b"]), g[f"{tag}_gradient"]) < 1e-14


def test_oc_top88():
    g = golden("filter_oc.npz")
    f = vo.ConeFilter(tuple(g["oc_dims"]), 1.5)
    for key, tol in (("oc_new_tol3", 1e-3), ("oc_new_tol6", 1e-6)):
        x = vo.oc_top88(g["oc_x"], g["oc_dc"], g["oc_dv"], 0.12, 0.2, density=f.forward, tol=tol)
        assert maxrel(x, g[key]) < 1e-12


# ----------------------------------------------------------------------------- recipes
def test_grf_recipe_matches_the_gmg_128x64x64_record():
    c = golden("gmg_128x64x64.json")
    rho = vo.gaussian_random_field((128, 64, 64), 8.0, 0)
    assert np.allclose([rho.min(), rho.max(), rho.mean()], c["rho_stats"], rtol=1e-14, atol=0)
    assert np.array_equal(rho[:16], np.array(c["rho_head"]))


def test_line_load_recipe_and_upsample():
    g = golden("products.npz")
    mask, force = vo.cantilever_line_load((8, 4, 4))
    assert np.array_equal(mask, g["smoke_mask"]) and np.array_equal(force, g["smoke_force"])
    k = golden("kat_inputs.npz")
    rho2, shape2 = vo.upsample(k["q64_rho"], tuple(k["q64_shape"]), 2)
    assert shape2 == (256, 128, 128) and rho2.size == 256 * 128 * 128


# ----------------------------------------------------------------------------- donor problems
@pytest.mark.parametrize("case", ["cant_patch_a", "cant_patch_b", "cant_patch_c", "cant_point", "torsion_a", "torsion_b"])
def test_donor_problem_builders_match_the_donor(case):
    """voxel_b200.problems.donor_cantilever / donor_torsion against the donor's own builders
    (fixtures from tests/golden/make_golden.py): fixed DOFs and loads bit-exact."""
    from voxel_b200 import problems
    from tests.golden.make_golden import DONOR_CASES
    g = golden("donor_problems.npz")
    _, kind, dims, kw = next(c for c in DONOR_CASES if c[0] == case)
    fn = problems.donor_cantilever if kind == "cantilever" else problems.donor_torsion
    mask, force, count = fn(*dims, **kw)
    assert np.array_equal(np.nonzero(mask == 0)[0], g[f"{case}_fixed"])
    assert np.array_equal(force, g[f"{case}_F"])
    assert count == int(g[f"{case}_patch_nodes"])
