"""Serving loop on the GPU: requests admitted while others run (continuous
batching on separate streams) finish with bitwise the state they reach alone."""
import numpy as np
import pytest

from autoflowcfd_b200 import ensemble as E
from autoflowcfd_b200 import serving as SV

pytestmark = pytest.mark.gpu


def requests():
    specs = [E.EnsembleCase((6, 3, 3), 2, 0.1, 0.05, 31, (0.15, 0.075, 0.075), bump_x=0.4),
             E.EnsembleCase((4, 2, 2), 1, 0.2, 0.0, 32, (0.07, 0.035, 0.035)),
             E.EnsembleCase((8, 4, 4), 2, 0.08, 0.07, 33, (0.2, 0.1, 0.1), bump_x=0.6)]
    return [SV.SolveRequest(i, 0.0, s) for i, s in enumerate(specs)]


TABLES = {}


def tables():
    if not TABLES:
        TABLES.update({r.rid: E.build_case(r.spec) for r in requests()})
    return TABLES


def loop(**kw):
    # drop 0: every request runs to max_iter, so alone and mixed runs take the same steps
    return SV.ServingLoop(precision="mixed", max_active=2, steps_per_slice=5, drop=0.0, max_iter=20,
                          keep_state=True, **kw)


def test_results_same_alone_and_in_the_mix():
    lp = loop()
    mixed = {r.rid: r for r in lp.run(requests(), tables=tables())}
    assert len(mixed) == 3 and lp.peak_active == 2  # two ran together, the third waited for a slot
    for req in requests():
        alone = loop().run([req], tables=tables())[0]
        got = mixed[req.rid]
        assert got.iterations == alone.iterations == 21  # iteration 1 plus four slices of five
        assert got.status == alone.status == "max_iter"
        assert np.array_equal(got.state, alone.state), req.rid
        assert got.cd == alone.cd
        assert got.latency_s >= 0


def test_latency_summary():
    res = loop().run(requests(), tables=tables())
    s = SV.latency_summary(res, wall_s=10.0)
    assert s["completed"] == 3 and s["p99_s"] >= s["p50_s"] > 0


def test_failures_stay_with_their_request(monkeypatch):
    """One request's state poisoned on the host (NaN), one request whose set-up
    raises (standing in for an out-of-memory handle): each fails alone, with
    its own status, and the healthy request finishes with bitwise its
    result alone."""
    healthy = requests()[1]
    alone = loop().run([healthy], tables=tables())[0]
    real = SV.ServingLoop._prepare

    def prepare(self, req, s, now, stream):
        if req.rid == 0:
            raise RuntimeError("afr status 2 (out of device memory): injected")
        a = real(self, req, s, now, stream)
        if req.rid == 2:
            a.solver.U[0, 0, 0] = float("nan")
        return a

    monkeypatch.setattr(SV.ServingLoop, "_prepare", prepare)
    lp = loop()
    res = {r.rid: r for r in lp.run(requests(), tables=tables())}
    assert res[0].status == "error" and "injected" in lp.errors[0]
    assert res[2].status == "nonfinite"
    assert res[1].status == "max_iter" and np.array_equal(res[1].state, alone.state)


def test_request_too_large_for_the_device_is_rejected():
    """The admission budget faked up (estimated bytes per cell far above the
    device's memory): with nothing running, the request is rejected instead of
    attempted."""
    lp = loop()
    lp.bytes_per_cell = {1: 1e12, 2: 1e12}
    res = lp.run(requests()[:1], tables=tables())
    assert res[0].status == "rejected" and res[0].iterations == 0


def test_residual_drop_stop():
    """The stopping rule: a request finishes as "converged" at the first slice
    boundary where its density residual has dropped to ``drop`` times its
    first step's (the 4x2x2-hex P1 request reaches half at iteration 101 =
    1 + 2 slices of 50), and as "max_iter" when the cap comes first."""
    req = requests()[1]
    lp = SV.ServingLoop(precision="mixed", max_active=1, steps_per_slice=50, drop=0.5, max_iter=500)
    got = lp.run([req], tables=tables())[0]
    assert got.status == "converged"
    assert got.iterations == 101 and got.residual_drop <= 0.5
    slow = requests()[0]  # its residual stays above 0.9 of the first for thousands of steps
    lp = SV.ServingLoop(precision="mixed", max_active=1, steps_per_slice=50, drop=0.5, max_iter=200)
    got = lp.run([slow], tables=tables())[0]
    assert got.status == "max_iter" and got.iterations >= 200 and got.residual_drop > 0.5

