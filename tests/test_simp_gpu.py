"""GPU parity of the SIMP pieces: the hat filter and top88 OC against golden vectors generated from
the reference's own code (experiments/session_h/run_w1b.py DensityFilter / oc_top88), the autograd
compliance sensitivity against the oracle formula and central finite differences, and a short
optimisation against the oracle's restatement of the reference loop.  Tolerances in each test."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle import voxel_oracle as vo

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")


def cu(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda", dtype=torch.float64)


def maxrel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("tag", ["f1", "f2", "f3"])
def test_cone_filter_matches_reference_density_filter(tag):
    g = golden("filter_oc.npz")
    f = vx.ConeFilter(*(int(d) for d in g[f"{tag}_dims"]), float(g[f"{tag}_rmin"]))
    assert maxrel(f.row_sums, g[f"{tag}_Hs"]) < 1e-15
    assert maxrel(f.forward(cu(g[f"{tag}_a"])), g[f"{tag}_density"]) < 1e-14
    assert maxrel(f.transpose(cu(g[f"{tag}_b"])), g[f"{tag}_gradient"]) < 1e-14
    assert f.check_adjoint() < 1e-13


@pytest.mark.parametrize("graph", [True, False])
def test_oc_top88_matches_reference(graph):
    g = golden("filter_oc.npz")
    f = vx.ConeFilter(*(int(d) for d in g["oc_dims"]), 1.5)
    oc = vx.OCUpdater(f, graph=graph)
    for key, tol in (("oc_new_tol3", 1e-3), ("oc_new_tol6", 1e-6)):
        x = oc(cu(g["oc_x"]), cu(g["oc_dc"]), cu(g["oc_dv"]), 0.12, 0.2, tol=tol)
        assert maxrel(x, g[key]) < 1e-12


def _state(shape, rho, tol=1e-12, precision="fp64", levels=None):
    mask, force = vx.problems.cantilever_equal_split(shape)
    s = vx.ElasticitySolver(shape, vx.problems.simp_modulus(rho, 1e-9), mask, precision=precision, tol=tol,
                            maxiter=400, check_every=1, levels=levels, omega="spectral")
    return vx.simp.SimpState(s, force, emin=1e-9, e0=1.0, penal=3.0, warm_start=False)


def test_autograd_sensitivity_equals_reference_formula():
    shape = (32, 16, 16)
    rho = cu(np.random.default_rng(4).uniform(0.05, 1.0, int(np.prod(shape))))
    st = _state(shape, rho, tol=1e-10, precision="mixed")
    r = rho.clone().requires_grad_(True)
    c = vx.compliance(r, st)
    c.backward()
    u = st.u.cpu().numpy()
    ce = vo.element_energy(shape, vo.quadrature([1, 1, 1], 0.3), u)
    ref = -3 * rho.cpu().numpy() ** 2 * (1 - 1e-9) * ce
    assert maxrel(r.grad, ref) < 1e-12
    assert abs(float(c.detach()) - float(st.force @ st.u)) <= 1e-15 * abs(float(c.detach()))


def test_autograd_sensitivity_central_differences():
    """64 seeded elements, step 1e-6, tight direct solves (a single-level hierarchy is the exact
    coarse solve): agreement to 1e-5 relative per element."""
    shape = (12, 6, 6)
    n = int(np.prod(shape))
    rho0 = np.random.default_rng(5).uniform(0.2, 1.0, n)
    st = _state(shape, cu(rho0), tol=1e-13, precision="fp64", levels=1)
    r = cu(rho0).requires_grad_(True)
    vx.compliance(r, st).backward()
    grad = r.grad.cpu().numpy()
    idx = np.random.default_rng(6).choice(n, 64, replace=False)
    h = 1e-6
    fd = []
    for e in idx:
        vals = []
        for sgn in (1, -1):
            rr = rho0.copy()
            rr[e] += sgn * h
            vals.append(float(vx.compliance(cu(rr), st)))
        fd.append((vals[0] - vals[1]) / (2 * h))
    fd = np.array(fd)
    assert np.max(np.abs(fd - grad[idx]) / np.abs(grad[idx])) < 1e-5


def test_short_simp_run_matches_oracle_loop():
    shape = (24, 12, 12)
    steps = 3
    n = int(np.prod(shape))
    x0 = 0.3 + np.random.default_rng(7).uniform(-0.01, 0.01, n)
    ke = vo.quadrature([1, 1, 1], 0.3)
    mask, force = vo.cantilever_equal_split(shape)

    def cpu_solve(E):
        shapes = vo.hierarchy_shapes(shape, 6)
        M = vo.Multigrid(shapes, ke, E, mask, vo.coarse_factor(shapes, ke, E, mask), np.float64, pre=2, post=2)
        A = lambda u: vo.apply_dirichlet(shape, ke, E, mask, u)
        return vo.fcg(A, force, M, 1e-12, 500, check_every=1)[0]

    xo, rho_o, comps_o = vo.simp_top88(shape, x0.copy(), steps, 0.3, 1.5, 0.2, solve=cpu_solve)
    # the same loop on the device (fp64 V-cycle, tight solves)
    filt = vx.ConeFilter(*shape, 1.5)
    oc = vx.OCUpdater(filt)
    x = cu(x0)
    rho = filt.forward(x)
    st = _state(shape, rho, tol=1e-12, precision="fp64")
    dv = filt.transpose(torch.ones(n, dtype=torch.float64, device="cuda"))
    comps = []
    for _ in range(steps):
        r = rho.clone().requires_grad_(True)
        c = vx.compliance(r, st)
        c.backward()
        comps.append(float(c))
        x = oc(x, filt.transpose(r.grad), dv, 0.3, 0.2, tol=1e-6)
        rho = filt.forward(x)
    assert np.allclose(comps, comps_o, rtol=1e-9, atol=0)
    assert maxrel(x, xo) < 1e-8
