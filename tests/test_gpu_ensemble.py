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
