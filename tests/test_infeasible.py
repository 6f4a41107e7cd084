"""Infeasibility detection (isprimalinfeasible / isdualinfeasible, src/IPM/src/ipm/solver/ipm.jl:
494-549, tested in the step! status chain :652-658 and nearstatus :560-570).

The oracle reaches the listed status on each problem, and its final iterate is a certificate: for a
primal-infeasible problem ŷ = y/‖y‖ has gᵀŷ > 0 and −Bᵀŷ in the dual cone; for a dual-infeasible one
p̂ = p/‖p‖ is in the cone with fᵀp̂ > 0 and Bp̂ ≈ 0.  The CUDA solver reaches the same kind of status, its iterate is a
certificate too, and infeasible instances solve bit-identically alone and inside a batch with
feasible ones.  The device and the oracle follow
the same path for the first iterations and then drift apart as the iterates diverge (see the
device test), so the comparison is by status family and certificate, not iteration by iteration."""
import numpy as np
import pytest

from helpers import INFEAS, SMALL, block_problem, cone_violation, oracle_solve
from mumblebee_b200.ipm import Context, IPMProblem, IPMSettings, IPMStatus, batch_solve, init, solve

CERT_TOL = 1e-6


def _check_certificate(pb, p, y, status):
    """p, y in the CSC problem's column and row order (the order results are returned in)."""
    pu, yu, B = p, y, pb["B"]
    tol = CERT_TOL * (100 if status.startswith("NEAR_") else 1)   # near_factor loosens the test
    if "PRIMAL" in status:
        yh = yu / np.linalg.norm(yu)
        assert pb["g"] @ yh > 0
        z = -(B.T @ yh)
        assert cone_violation(z, pb["kinds"], pb["sizes"]) <= tol * max(1.0, np.linalg.norm(z))
    else:
        ph = pu / np.linalg.norm(pu)
        assert pb["f"] @ ph > 0
        assert np.linalg.norm(B @ ph) <= 10 * tol * max(1.0, abs(pb["f"] @ ph))
        assert cone_violation(ph, pb["kinds"], pb["sizes"]) <= tol


@pytest.mark.parametrize("name", list(INFEAS))
def test_oracle_detects_infeasibility(name):
    make, want = INFEAS[name]
    pb = make()
    ref = block_problem(pb)
    _, o = oracle_solve(ref)
    assert o["status"] == want
    _check_certificate(pb, o["p"], o["y"], want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(INFEAS))
def test_device_detects_infeasibility_like_oracle(name):
    """On an infeasible problem the iterates diverge (‖p‖ or ‖y‖ grows like 1/step), so rounding
    differences between the device reductions and the sequential oracle grow with them.  The first
    history rows agree to 1e-5, up to the row of the first step shorter than 0.1.  After that both runs end
    in the same status family (X or NEAR_X) with a valid certificate, within max(4, half the
    oracle's count) iterations of each other."""
    make, want = INFEAS[name]
    pb = make()
    ref = block_problem(pb)
    prob = IPMProblem.from_dict(ref, ctx=Context.default())
    _, o = oracle_solve(ref, vperm=prob.symbolic()["vperm"])
    s = init(prob, IPMSettings())
    s.solve()
    r = s.result()
    h, oh = s.history(), o["history"]
    assert o["status"] == want
    fam = want.replace("NEAR_", "")
    assert r.status in (IPMStatus[fam], IPMStatus["NEAR_" + fam])
    assert abs(r.niter - o["niter"]) <= max(4, o["niter"] // 2)
    for i in range(min(3, len(h), len(oh))):
        for f in ("mu", "pres", "dres", "pobj", "dobj", "step"):
            assert abs(h[i][f] - oh[i][f]) <= 1e-5 * max(1.0, abs(oh[i][f])), (i, f)
        if oh[i]["step"] < 0.1:   # after the first short step the iterates run off towards the certificate
            break
    _check_certificate(pb, r.p, r.y, r.status.name)


@pytest.mark.gpu
def test_device_mixed_precision_detects_infeasibility():
    for name in ("pinf_socp200", "dinf_socp200"):
        make, want = INFEAS[name]
        pb = make()
        ref = block_problem(pb)
        r = solve(IPMProblem.from_dict(ref, ctx=Context.default()), IPMSettings(precision="mixed"))
        assert r.status in (IPMStatus[want], IPMStatus["NEAR_" + want])
        _check_certificate(pb, r.p, r.y, r.status.name)


@pytest.mark.gpu
def test_infeasible_instances_batch_equals_alone():
    ctx = Context.default()
    pbs = [INFEAS[k][0]() for k in ("pinf_socp40", "dinf_socp40", "pinf_pos", "dinf_soc")]
    pbs += [SMALL[k]() for k in ("socp_small", "port_small")]
    probs = [IPMProblem.from_dict(block_problem(pb), ctx=ctx) for pb in pbs]
    many = batch_solve(probs, IPMSettings(), grid=2)
    for p, b in zip(probs, many):
        a = solve(p, IPMSettings())
        assert a.status == b.status and a.niter == b.niter
        np.testing.assert_array_equal(a.p, b.p)
        np.testing.assert_array_equal(a.y, b.y)
