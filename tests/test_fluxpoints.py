"""Flux-point construction, host half (no GPU): the primary records, the
split prism quad halves, the locate jobs and the inverse modal Vandermonde
matrices against the reference's own construction (tests/golden/fp_*.npz,
made by tests/golden/make_golden.py from fr/face_flux_points_merge.py)."""
import numpy as np
import pytest

from autoflowcfd_b200 import facegeom as FG
from conftest import golden_path

FP_CASES = ["fp_prism_p1", "fp_prism_p2", "fp_prism_p3_bump", "fp_tet_p2", "fp_tet_p3"]


def load(name):
    z = np.load(golden_path(name), allow_pickle=False)
    return {k: z[k] for k in z.files}


def face_conn(g):
    return {k[3:]: g[k] for k in g if k.startswith("fc_")}


@pytest.mark.parametrize("name", FP_CASES)
def test_plan_matches_reference(name):
    g = load(name)
    pl = FG.plan_jobs(face_conn(g), g["prism_conn"], g["tet_conn"], int(g["order"]))
    assert np.array_equal(pl["opr"].astype(np.uint8), g["owner_is_primary"])
    assert np.array_equal(pl["npr"].astype(np.uint8), g["neighbor_is_primary"])
    assert np.array_equal(pl["main_nb"], np.flatnonzero(g["nb_src0_cell"] >= 0))
    assert np.array_equal(pl["main_ow"], np.flatnonzero(g["ow_src0_cell"] >= 0))
    assert np.array_equal(pl["ms_nb"], np.flatnonzero(g["nb_src1_idx"] >= 0))
    assert np.array_equal(pl["ms_ow"], np.flatnonzero(g["ow_src1_idx"] >= 0))
    # the half of a split quad a primary record carries: exactly the rows the
    # reference's primary matrix fills (the other half is its second source)
    P = g["true_normal"].shape[1]
    for faces, mask, mat in ((pl["ms_nb"], pl["nb_mask"], g["nb_src0_mat"]),
                             (pl["ms_ow"], pl["ow_mask"], g["ow_src0_mat"])):
        for f in faces:
            rows = np.any(mat[f] != 0, axis=1)
            assert np.array_equal(rows, [(int(mask[f]) >> p) & 1 == 1 for p in range(P)]), f
    if name.startswith("fp_prism"):
        assert len(pl["ms_nb"]) > 0  # split quads present


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("kind", ["prism", "tet"])
def test_vandermonde_rows_sum_and_invert(kind, order):
    """V_inv * V = I at the solution points; the rounding of the reference's
    compiled integer power is reproduced (square-and-multiply)."""
    sps = FG.gauss_legendre(order + 1)[0]
    ga, gb, gc = np.meshgrid(sps, sps, sps, indexing="ij")
    V = FG.modal_vandermonde(kind, order, ga.ravel(), gb.ravel(), gc.ravel())
    Vi = FG.vandermonde_inverse(kind, order)
    assert np.allclose(V @ Vi, np.eye(V.shape[0]), atol=1e-6 if (kind, order) == ("tet", 3) else 1e-9)
    x = np.linspace(0.0, 1.0, 11)
    for n in range(1, 7):
        r = np.ones_like(x)
        for _ in range(n):
            r = r * x
        assert np.allclose(FG.int_power(x, n), r, rtol=1e-15, atol=0)


def test_half_masks_are_complementary_and_cover_the_face():
    g = load("fp_prism_p2")
    pl = FG.plan_jobs(face_conn(g), g["prism_conn"], g["tet_conn"], 2)
    P = g["true_normal"].shape[1]
    m = pl["nb_mask"][pl["ms_nb"]].astype(np.int64)
    counts = np.array([bin(int(v)).count("1") for v in m])
    assert np.all((counts > 0) & (counts < P))


@pytest.mark.parametrize("name", ["prism_p0_ns", "prism_p1_ns", "prism_p2_sst", "tet_p3_tgv"])
def test_distribution_maps_match_reference(golden, name):
    g = golden(name)
    fp, co = FG.distribution_maps(int(g["order"]) + 1)
    assert np.array_equal(fp, g["dist_fp_of_sp"]) and np.array_equal(co, g["dist_axis_coord_of_sp"])
