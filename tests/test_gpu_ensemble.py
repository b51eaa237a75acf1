"""Batched uneven ensemble on the GPU: every case advanced inside the
ensemble (concatenated per order, CUDA-graph replay, autotuned launch shapes)
gets bitwise the result it gets alone, and per-case norms match."""
import numpy as np
import pytest
import torch

from autoflowcfd_b200 import ensemble as E
from autoflowcfd_b200.solver import B200FRSolver

pytestmark = pytest.mark.gpu

SPECS = [E.EnsembleCase((6, 3, 3), 2, 0.1, 0.05, 21, (0.15, 0.075, 0.075)),
         E.EnsembleCase((4, 2, 2), 1, 0.25, 0.0, 22, (0.06, 0.03, 0.03)),
         E.EnsembleCase((8, 4, 4), 2, 0.05, 0.08, 23, (0.3, 0.15, 0.15)),
         E.EnsembleCase((6, 3, 3), 1, 0.15, 0.02, 24, (0.1, 0.05, 0.05))]


def solo(spec, case, steps, precision):
    s = B200FRSolver(case, turb_model_name="NONE", mu_molecular=E.MU, rho_inf=E.RHO_INF, vel_inf=spec.velocity,
                     p_inf=E.P_INF, precision=precision)
    s.set_state_from_cpu(E.uniform_state(spec, int(case["n_cells"]), int(case["n_sps"])))
    norm = None
    for _ in range(steps):
        norm = s.step()
    out = s.U.cpu().numpy()
    s.cleanup()
    return out, norm


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_ensemble_matches_solo_runs(precision):
    cases = [E.build_case(s) for s in SPECS]
    ens = E.B200Ensemble(SPECS, precision=precision, cases=cases)
    for _ in range(3):
        ens.step()
    norms = ens.norms()
    for i, (spec, case) in enumerate(zip(SPECS, cases)):
        ref, ref_norm = solo(spec, case, 3, precision)
        assert np.array_equal(ens.state(i).cpu().numpy(), ref), i
        assert abs(norms[i] - ref_norm) <= 1e-13 * abs(ref_norm)
    ens.cleanup()


def test_graph_replay_and_autotune_keep_results():
    cases = [E.build_case(s) for s in SPECS]
    eager = E.B200Ensemble(SPECS, cases=cases)
    for _ in range(4):
        eager.step()
    tuned = E.B200Ensemble(SPECS, cases=cases)
    choices = tuned.autotune()
    for pre, face_block, upd in choices:
        assert pre >= 1 and face_block in (64, 128, 256) and upd in (0, 1, 2)
    tuned.capture()          # one eager warm-up step, then the captured step
    tuned.replay(3)
    torch.cuda.synchronize()
    for i in range(len(SPECS)):
        assert np.array_equal(tuned.state(i).cpu().numpy(), eager.state(i).cpu().numpy()), i
    eager.cleanup()
    tuned.cleanup()


def test_nonfinite_case_is_isolated():
    """A NaN injected on the host into one case's start state: that case alone
    is reported non-finite (afr_status per case), every other case gets
    bitwise its clean result, and the healthy cases keep running after the
    status is cleared."""
    cases = [E.build_case(s) for s in SPECS]
    clean = E.B200Ensemble(SPECS, cases=cases)
    bad = E.B200Ensemble(SPECS, cases=cases)
    victim = 2
    st = bad.state(victim)
    st[st.shape[0] // 2, 3, 1] = float("nan")
    for _ in range(2):
        clean.step()
        bad.step()
    status = bad.status(clear=True)
    assert status.tolist() == [4 if i == victim else 0 for i in range(len(SPECS))]  # AFR_ENONFINITE
    assert clean.status().tolist() == [0] * len(SPECS)
    for i in range(len(SPECS)):
        if i != victim:
            assert np.array_equal(bad.state(i).cpu().numpy(), clean.state(i).cpu().numpy()), i
    norms = bad.norms()
    assert not np.isfinite(norms[victim]) and np.all(np.isfinite(np.delete(norms, victim)))
    clean.cleanup()
    bad.cleanup()


def test_step_without_norm_reports_nonfinite_at_the_next_step():
    """afr_step with no norm does not synchronise; the status it leaves in
    pinned host memory makes the next step raise once the device is done."""
    from autoflowcfd_b200._lib import AFR_ENONFINITE, AfrError

    spec = SPECS[1]
    case = E.build_case(spec)
    s = B200FRSolver(case, turb_model_name="NONE", mu_molecular=E.MU, rho_inf=E.RHO_INF, vel_inf=spec.velocity,
                     p_inf=E.P_INF)
    U = E.uniform_state(spec, int(case["n_cells"]), int(case["n_sps"]))
    U[1, 2, 4] = np.inf
    s.set_state_from_cpu(U)
    s.step(want_norm=False)          # returns at once
    torch.cuda.synchronize()
    with pytest.raises(AfrError) as ei:
        s.step(want_norm=False)
    assert ei.value.status == AFR_ENONFINITE
    with pytest.raises(AfrError):
        s.status(clear=True)
    s.set_state_from_cpu(E.uniform_state(spec, int(case["n_cells"]), int(case["n_sps"])))
    assert np.isfinite(s.step())     # cleared status, finite state: healthy again
    s.cleanup()
