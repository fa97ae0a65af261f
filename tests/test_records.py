"""Input cases and result records in the reference's formats (no GPU): the npz schema round trip,
make_inputs' upsampling and regenerated boundary data against the oracle, validation errors, and
the result.json layout."""
import json

import numpy as np
import pytest

from oracle import voxel_oracle as vo

vx = pytest.importorskip("voxel_b200")
from voxel_b200 import records  # noqa: E402


def small_case(shape=(6, 3, 2)):
    rng = np.random.default_rng(0)
    mask, force = vo.cantilever_line_load(shape)
    return records.Case(shape, rng.uniform(0.001, 1, int(np.prod(shape))), mask, force,
                        vo.quadrature([1, 1, 1], 0.3), name="small")


def test_npz_round_trip_and_author_layout(tmp_path):
    c = small_case()
    records.save_case(tmp_path / "small.npz", c)
    d = records.load_case(tmp_path / "small.npz")
    assert d.shape == c.shape and d.name == "small" and len(d.sha256) == 64
    for k in ("rho", "mask", "force", "ke"):
        assert np.array_equal(getattr(d, k), getattr(c, k))
    E, mask, force = d.author_layout()
    assert np.array_equal(E, vo.to_author(1e-6 + (1 - 1e-6) * c.rho ** 3, c.shape))
    assert np.array_equal(mask, vo.to_author(c.mask, c.shape, True))
    assert np.array_equal(force, vo.to_author(c.force, c.shape, True))


def test_upsample_and_regenerate_follow_make_inputs():
    c = small_case()
    up = records.upsample_case(c, 3)
    rho_ref, shape_ref = vo.upsample(c.rho, c.shape, 3)
    assert up.shape == shape_ref and np.array_equal(up.rho, rho_ref)
    m, f = vo.cantilever_line_load(shape_ref)
    assert np.array_equal(up.mask, m) and np.array_equal(up.force, f)
    m1, f1 = records.regenerate(c.shape)                  # factor 1 regenerates the base data exactly
    assert np.array_equal(m1, c.mask) and np.array_equal(f1, c.force)
    assert abs(f1.sum() + 1.0) < 1e-15                    # total load 1 in -z


def test_load_case_rejects_bad_files(tmp_path):
    c = small_case()
    np.savez(tmp_path / "missing.npz", shape=np.array(c.shape), rho=c.rho, mask=c.mask, force=c.force)
    with pytest.raises(ValueError, match="missing"):
        records.load_case(tmp_path / "missing.npz")
    np.savez(tmp_path / "short.npz", shape=np.array(c.shape), rho=c.rho[:-1], mask=c.mask, force=c.force, ke=c.ke)
    with pytest.raises(ValueError, match="rho"):
        records.load_case(tmp_path / "short.npz")


def test_result_writer_layout(tmp_path):
    w = records.ResultWriter(tmp_path / "run", protocol_sha256="ab")
    first = json.loads((tmp_path / "run" / "result.json").read_text())
    assert first["status"] == "running" and first["to_tolerance"] == [] and first["protocol_sha256"] == "ab"
    w.append("to_tolerance", {"case": "q", "iterations": 3})
    w.set(gpu_executed=True)
    out = w.finish()
    disk = json.loads((tmp_path / "run" / "result.json").read_text())
    assert disk == out and disk["status"] == "complete" and disk["gpu_executed"]
    assert disk["to_tolerance"] == [{"case": "q", "iterations": 3}]
    for k in records.ResultWriter.SECTIONS:
        assert k in disk
    with pytest.raises(ValueError):
        w.append("bogus", {})
