"""Stacked-batch geometry (no GPU): every job stays aligned on every level of its hierarchy, with at
least one zero-modulus separator element between neighbours on the coarsest level."""
import pytest

vx = pytest.importorskip("voxel_b200")
from voxel_b200.batch import stack_geometry  # noqa: E402


@pytest.mark.parametrize("shape", [(48, 24, 24), (96, 48, 48), (160, 80, 80), (256, 128, 128), (32, 16, 16)])
@pytest.mark.parametrize("slots", [1, 2, 5, 16])
def test_jobs_stay_aligned_on_every_level(shape, slots):
    g = stack_geometry(shape, slots)
    assert g.levels == len(vx.hierarchy_shapes(shape, 16))
    for l, (gs, js) in enumerate(zip(g.shapes, g.job_shapes)):
        pitch = g.pitch >> l
        assert pitch << l == g.pitch                       # whole element planes on level l
        assert gs[1:] == js[1:]
        assert gs[0] == slots * pitch - (g.separator >> l)
        assert pitch - js[0] >= 1                          # a separator element between neighbours
        assert all(s % 2 == 0 for s in gs) or l == g.levels - 1
    assert g.shapes[-1][0] + 1 == slots * (g.job_shapes[-1][0] + 1)   # coarsest: back-to-back blocks


def test_batch_ladders_and_default_slots():
    """A shape's batch capacities double up to its slot count (the last rung is the slot count), and
    the slot count fills about 32M stacked DOFs, at least one and at most 16 jobs."""
    from voxel_b200.serving import batch_ladder, default_slots
    assert batch_ladder(1) == [1]
    assert batch_ladder(2) == [1, 2]
    assert batch_ladder(10) == [1, 2, 4, 8, 10]
    assert batch_ladder(16) == [1, 2, 4, 8, 16]
    assert default_slots((48, 24, 24)) == 16
    assert default_slots((160, 80, 80)) == 10
    assert default_slots((256, 128, 128)) == 2
    assert default_slots((576, 288, 288)) == 1
