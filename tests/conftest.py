import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN_DIR = os.path.join(REPO, "tests", "golden")
if GOLDEN_DIR not in sys.path:
    sys.path.insert(0, GOLDEN_DIR)  # flows.py: start states shared with the fixture generator

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_path(name):
    return os.path.join(GOLDEN, name + ".npz")


CASES = ["tet_p1_vortex", "prism_p2_sst", "prism_p1_ns", "tet_p3_tgv", "prism_p1_floors", "tet_p1_align"]
# order 0: the finite-volume path of the reference (one point per cell)
P0_CASES = ["prism_p0_ns", "prism_p0_sst", "tet_p0_vortex"]
# steps of the dual-time (BDF1 then BDF2) and IMEX Euler schemes
SCHEME_CASES = ["prism_p1_ns_dual_time", "prism_p1_ns_imex_euler", "prism_p2_sst_dual_time"]
# cases with a wall force integral in their fixture
CD_CASES = ["prism_p2_sst", "prism_p1_ns", "prism_p1_floors", "prism_p0_ns"]


def case_tol(name):
    """Relative max-norm tolerance per case.

    P1/P2: 1e-12, the reference's own bar between two implementations
    (tests/unit/test_fr_residual_inviscid_kernel_crosscheck.py:203-208).
    P3: the reference's tet operators carry entries up to 6e7 and its
    cross-interpolation matrices up to 2e7, so any change of summation order
    moves residuals by ~1e-7 relative; 1e-6 bounds that conditioning noise.
    """
    return 1e-6 if name.endswith("p3_tgv") else 1e-12


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    cache = {}

    def load(name):
        if name not in cache:
            z = np.load(golden_path(name), allow_pickle=False)
            cache[name] = {k: z[k] for k in z.files}
        return cache[name]

    return load
