"""A reference input case end to end: the session-I q96x1 case (the optimized-q96 design,
192x96x96) written in the reference's npz schema, loaded, solved at the published protocol, and
recorded as the reference's to_tolerance row -- 24 iterations, the published compliance, and
the physical check through the device C product."""
import json

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu
vx = pytest.importorskip("voxel_b200")
from voxel_b200 import records  # noqa: E402


def test_q96x1_case_record(tmp_path):
    k = golden("kat_inputs.npz")
    kat = golden("kat_session_i.json")
    base = tuple(int(s) for s in k["q96_shape"])
    mask, force = records.regenerate(base)
    records.save_case(tmp_path / "optimized-q96.npz",
                      records.Case(base, k["q96_rho"], mask, force, k["q96_ke"]))
    case = records.upsample_case(records.load_case(tmp_path / "optimized-q96.npz"), 1, name="q96x1")
    mgp = kat["_protocol"]["multigrid"]
    E, m, f = case.author_layout()
    s = vx.ElasticitySolver(case.shape, torch.as_tensor(E, device="cuda"), torch.as_tensor(m, device="cuda"),
                            ke=case.ke, precision="mixed", pre=mgp["pre"], post=mgp["post"], omega="spectral",
                            max_coarse_x=mgp["max_coarse_x"], tol=1e-8, maxiter=200, check_every=1,
                            spectral_seed=kat["_protocol"]["order_seed"])
    w = records.ResultWriter(tmp_path / "out")
    row = records.solve_record(case, s, arm="mixed")
    w.append("to_tolerance", row)
    w.finish()
    obs = kat["q96x1"]["observations"]
    assert row["iterations"] == obs[0]["iterations"] == 24 and row["physical_passed"], row
    ref_c = np.array([o["compliance"] for o in obs])
    assert np.min(np.abs(row["compliance"] - ref_c)) <= 1e-9 * ref_c.mean()
    assert np.min(np.abs(row["solution_norm"] - np.array([o["solution_norm"] for o in obs]))) <= 1e-9 * row["solution_norm"]
    disk = json.loads((tmp_path / "out" / "result.json").read_text())
    assert disk["to_tolerance"][0]["solution_sha256"] == row["solution_sha256"]
