"""Checkpoint layout and round trip (host side, no GPU): the reference's
group / dataset / attribute paths, the cell-averaged solution, the full
state and its primitives (FRState._update_primitives), and an exact reload."""
from types import SimpleNamespace

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from autoflowcfd_b200 import checkpoint as C  # noqa: E402
from conftest import golden_path  # noqa: E402


def stand_in(g):
    U = torch.from_numpy(g["U0"].copy())
    return SimpleNamespace(U=U, k=torch.from_numpy(g["k0"].copy()), omega=torch.from_numpy(g["omega0"].copy()),
                           nu_t=torch.from_numpy(g["nu_t0"].copy()), _U_prev=torch.from_numpy(g["U_step1"].copy()),
                           _has_prev=True, order=int(g["order"]), turb_model_name="SST", precision="fp64",
                           time_scheme="dual_time", freestream={"rho_inf": 1.225, "vel_inf": 34.0, "p_inf": 101325.0},
                           residual_history=[3.0, 2.0, 1.5])


def test_layout_and_round_trip(tmp_path):
    g = np.load(golden_path("prism_p2_sst"))
    s = stand_in(g)
    path = C.save_checkpoint(s, str(tmp_path / "ck"), iteration=7)
    z = np.load(path)
    for key in ("metadata@iteration", "metadata@timestamp", "metadata@config_hash", "metadata@backend",
                "solution/conserved", "solution/U_sps", "solution/Q_sps", "convergence/history/iterations",
                "convergence/history/residuals/total"):
        assert key in z.files, key
    assert np.array_equal(z["solution/conserved"], g["U0"].mean(axis=1))
    sol, hist, it, meta = C.load_checkpoint(path)
    assert it == 7 and meta["order"] == 2 and meta["turbulence_model"] == "SST" and meta["has_prev"]
    assert np.array_equal(meta["fields"]["U_sps"], g["U0"]) and np.array_equal(meta["fields"]["k"], g["k0"])
    assert hist["residuals"]["total"] == [3.0, 2.0, 1.5]
    # primitives as FRState._update_primitives
    Q = meta["fields"]["Q_sps"]
    rho = np.maximum(g["U0"][..., 0], 1e-10)
    assert np.array_equal(Q[..., 1], g["U0"][..., 1] / rho)
    assert np.all(Q[..., 4] >= 1.0) and np.all(Q[..., 5] >= 1e-12)
    # exact reload into a fresh stand-in
    t = stand_in(g)
    for x in (t.U, t.k, t.omega, t.nu_t):
        x.zero_()
    t._U_prev, t._has_prev, t.residual_history = None, False, []
    assert C.resume(t, path) == 7
    assert torch.equal(t.U, s.U) and torch.equal(t.k, s.k) and torch.equal(t._U_prev, s._U_prev) and t._has_prev


def test_resume_refuses_another_shape(tmp_path):
    g = np.load(golden_path("prism_p2_sst"))
    path = C.save_checkpoint(stand_in(g), str(tmp_path / "ck"), iteration=1)
    other = SimpleNamespace(U=torch.zeros(3, 27, 7))
    with pytest.raises(ValueError, match="does not match"):
        C.resume(other, path)
