"""Host logic of the donor drop-ins (no GPU): the continuation schedule and the exception type."""
import pytest

vx = pytest.importorskip("voxel_b200")
from voxel_b200 import donor  # noqa: E402


def test_schedule_follows_the_donor_table():
    # experiments/session_a/donor/src/gpu_fem/simp_r2.py:410-431
    assert donor.schedule_at(1) == (1.5, 1.0, 0.20, 1.50, False)
    assert donor.schedule_at(15) == (1.5, 1.0, 0.20, 1.50, False)
    assert donor.schedule_at(16) == (3.5, 4.0, 0.15, 1.35, False)
    assert donor.schedule_at(65) == (4.5, 16.0, 0.08, 1.25, False)
    assert donor.schedule_at(66) == (4.5, 32.0, 0.05, 1.20, True)
    assert donor.schedule_at(500) == (4.5, 32.0, 0.05, 1.20, True)
    assert donor.schedule_at(3, [(5, 2.0, 0.0, 0.1, 2.0)]) == (2.0, 0.0, 0.1, 2.0, True)


def test_fail_closed_exception_is_a_runtime_error():
    assert issubclass(donor.LinearSolveNotConverged, RuntimeError)
