"""Pin the CPU oracle against the reference's own outputs (golden fixtures).

The fixtures were produced by running the reference implementation
(tests/golden/make_golden.py); the oracle must reproduce them before it may be
used to check the CUDA path."""
import copy

import numpy as np
import pytest

from conftest import CASES, CD_CASES, P0_CASES, SCHEME_CASES, case_tol, golden_path
from oracle import fr_oracle as O


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", CASES + P0_CASES)
def test_residuals_match_reference(name):
    case, m, s = O.load_case(golden_path(name))
    U = case["U0"]
    Q = O.state_primitives(U)
    mu_t = s.mu_t(Q)
    tol = case_tol(name)
    assert rel(O.inviscid_residual(m, U), case["R_inv"][..., :5]) < tol
    assert rel(O.viscous_residual(m, U, s.mu, mu_t), case["R_visc"][..., :5]) < tol
    assert rel(O.local_dt(m, Q, s.mu, mu_t), case["dt_local"]) < 1e-14
    # padded turbulence columns are zero in the reference
    if case["R_inv"].shape[-1] > 5:
        assert np.all(case["R_inv"][..., 5:] == 0) and np.all(case["R_visc"][..., 5:] == 0)


@pytest.mark.parametrize("name", ["prism_p2_sst", "prism_p0_sst"])
def test_sst_source_transport_update_match_reference(name):
    case, m, s = O.load_case(golden_path(name))
    U = case["U0"]
    Q = O.state_primitives(U)
    dt = O.local_dt(m, Q, s.mu, s.mu_t(Q))
    t = copy.deepcopy(s.turb)
    Sk, Sw, tk, tw = O.sst_source_and_update(m, U, Q, t, dt, s.mu, s.wall_distance)
    for a, k in ((Sk, "sst_Sk"), (Sw, "sst_Sw"), (tk, "sst_tk"), (tw, "sst_tw"), (t.k, "sst_k1"),
                 (t.w, "sst_w1"), (t.nut, "sst_nut1")):
        assert rel(a, case[k]) < 1e-12, k


@pytest.mark.parametrize("name", CASES + SCHEME_CASES + P0_CASES)
def test_steps_match_reference(name):
    case, m, s = O.load_case(golden_path(name))
    for i in range(len(case["norms"])):
        n = s.step()
        tol = 1e-12 if not name.endswith("p3_tgv") else 1e-3
        assert rel(s.U, case[f"U_step{i + 1}"]) < tol
        assert abs(n - case["norms"][i]) / case["norms"][i] < max(tol, 1e-12)
        if s.turb is not None:
            assert rel(s.turb.k, case[f"k_step{i + 1}"]) < 1e-12
            assert rel(s.turb.w, case[f"w_step{i + 1}"]) < 1e-12
            assert rel(s.turb.nut, case[f"nut_step{i + 1}"]) < 1e-12


@pytest.mark.parametrize("name", CD_CASES)
def test_force_coefficients_match_reference(name):
    case, m, s = O.load_case(golden_path(name))
    for _ in range(len(case["norms"])):
        s.step()
    cd = O.cd_cl(m, s.U, s.mu, None if s.turb is None else s.turb.nut, case["freestream"])
    assert np.allclose(cd, case["cd_cl"], rtol=1e-10, atol=0)


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle input must break parity (the test has teeth)."""
    case, m, s = O.load_case(golden_path("prism_p1_ns"))
    m.c["g_left"] = m.c["g_left"] * (1 + 1e-9)
    assert rel(O.inviscid_residual(m, case["U0"]), case["R_inv"][..., :5]) > 1e-11


def test_floor_and_clamp_branches_are_exercised(golden):
    """The floors fixture was made from states beyond every clamp of the
    reference's enforce_positivity (core/time_integration/positivity.py:13-45)
    and the AUSM+up floors (core/fr_operators/kernels.py:41-44); the generator
    counted the points each clamp acted on during the two steps."""
    from flows import FLOOR_CELLS

    g = golden("prism_p1_floors")
    assert np.all(g["positivity_trips"] > 0), g["positivity_trips"]  # rho, |u|, p, rho*k, rho*omega
    U0 = g["U0"]
    vac = U0[FLOOR_CELLS["vacuum"]]
    assert np.all(vac[:, 0] < 1e-6) and np.all(0.4 * vac[:, 4] < 10.0)  # below both AUSM floors
    U1 = g["U_step1"]
    assert np.all(U1[FLOOR_CELLS["neg_rho_k"], :, 5] == 0.0)
    assert np.all(U1[FLOOR_CELLS["tiny_rho_w"], :, 6] == 1e-8)


def test_alignment_fallback_is_exercised():
    """In the alignment fixture some true normals point against (or across) the
    adjugate direction, so the reference's alignment < 0.5 fallback
    (core/fr_residual/inviscid_kernel_colored.py:104-108, neighbour side
    :186-190) takes them on both sides of a record; the benign fixtures never
    reach it."""

    def fallback_points(name):
        case, m, _ = O.load_case(golden_path(name))
        adj = m.extras["adj"]
        counts = []
        for owner in (True, False):
            isb = m.c["is_boundary"].astype(bool)
            prim = m.c["owner_is_primary" if owner else "neighbor_is_primary"].astype(bool)
            f = np.flatnonzero(prim if owner else prim & ~isb)
            cell, ax, sd = O._side_geometry(m, f, owner)
            arow = np.matmul(O.extrap_E(m, cell, ax, sd), adj[cell, :, ax, :])
            d = arow / np.linalg.norm(arow, axis=-1, keepdims=True) * sd[:, None, None]
            tn = m.c["true_normal"][f] * (1.0 if owner else -1.0)
            counts.append(int(np.sum(np.sum(d * tn, axis=-1) < 0.5)))
        return counts

    assert min(fallback_points("tet_p1_align")) > 0
    assert fallback_points("tet_p1_vortex") == [0, 0]
