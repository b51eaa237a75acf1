"""Host logic of the batched ensemble (no GPU): the seeded case draw and the
concatenation of independent cases into one mesh.  The oracle's residuals on
the concatenated tables, restricted to each case, must equal the residuals of
that case alone: the concatenation only offsets indices."""
import numpy as np
import pytest

from autoflowcfd_b200 import ensemble as E
from oracle import fr_oracle as O


def dense(case):
    case = dict(case)
    tab = case.pop("src_mat_table")
    for key in ("nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"):
        case[key] = tab[case.pop(key + "_index")]
    return case


def test_draw_is_seeded_and_in_range():
    a = E.draw_cases(16, seed=3)
    b = E.draw_cases(16, seed=3)
    assert a == b
    for s in a:
        assert s.order in (1, 2)
        assert 0.05 <= s.mach <= 0.3 and 0.0 <= s.bump <= 0.1
        re = E.RHO_INF * s.velocity * s.lengths[0] / E.MU
        assert abs(re - 1e5) < 1e-6 * 1e5
        assert 2000 / 2 <= s.n_cells / 2 <= 64000 * 1.5


@pytest.mark.parametrize("order", [1, 2])
def test_concatenated_residuals_equal_separate(order):
    specs = [E.EnsembleCase((4, 2, 2), order, 0.1, 0.05, 11, (0.2, 0.1, 0.1)),
             E.EnsembleCase((2, 3, 2), order, 0.25, 0.0, 12, (0.1, 0.05, 0.05)),
             E.EnsembleCase((3, 2, 3), order, 0.05, 0.08, 13, (0.4, 0.2, 0.2))]
    cases = [E.build_case(s) for s in specs]
    rng = np.random.default_rng(5)
    states = []
    for s, c in zip(specs, cases):
        U = E.uniform_state(s, int(c["n_cells"]), int(c["n_sps"]))
        U *= 1.0 + 0.01 * rng.standard_normal(U.shape)  # away from free stream (cancellation noise)
        states.append(U)
    merged = E.concatenate(cases)
    assert int(merged["n_cells"]) == sum(int(c["n_cells"]) for c in cases)
    m_all = O.Mesh.from_case(dense(merged))
    R_all = O.inviscid_residual(m_all, np.concatenate(states))
    V_all = O.viscous_residual(m_all, np.concatenate(states), E.MU, None)
    off = 0
    for c, U in zip(cases, states):
        m = O.Mesh.from_case(dense(c))
        n = int(c["n_cells"])
        for got, ref in ((R_all[off:off + n], O.inviscid_residual(m, U)), (V_all[off:off + n], O.viscous_residual(m, U, E.MU, None))):
            assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
        off += n


def test_concatenate_rejects_mixed_orders():
    c1 = E.build_case(E.EnsembleCase((2, 2, 2), 1, 0.1, 0.0, 1, (0.1, 0.05, 0.05)))
    c2 = E.build_case(E.EnsembleCase((2, 2, 2), 2, 0.1, 0.0, 2, (0.1, 0.05, 0.05)))
    with pytest.raises(ValueError):
        E.concatenate([c1, c2])
