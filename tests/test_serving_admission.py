"""Admission rule of the serving loop (host logic, no GPU)."""
import pytest

pytest.importorskip("torch")

from autoflowcfd_b200.serving import admission  # noqa: E402


def test_admission_decisions():
    GB = 1e9
    assert admission(100 * GB, 10 * GB, 8 * GB, 0, 4) == "admit"
    assert admission(100 * GB, 95 * GB, 8 * GB, 2, 4) == "wait"      # memory frees when a request ends
    assert admission(100 * GB, 95 * GB, 8 * GB, 0, 4) == "reject"    # cannot fit even on an idle device
    assert admission(100 * GB, 1 * GB, 8 * GB, 4, 4) == "wait"       # no slot
