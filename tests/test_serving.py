"""Serving loop: admission by HBM footprint, continuous batching, and the same
result for a request alone and in the mix."""
import numpy as np
import pytest

from mesohops_b200 import serving as sv
from mesohops_b200.workloads import (chain, dimer, ring20, served_request,
                                     served_stream_specs)


def _req(rid, sysp, depth, n_steps, arrival=0.0, adaptive=None, seed=None, dt=4.0):
    n = sysp["HAMILTONIAN"].shape[0]
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[n // 2] = 1.0
    noise = {"SEED": rid if seed is None else seed, "MODEL": "FFT_FILTER",
             "TLEN": (n_steps + 1) * dt, "TAU": dt / 2}
    return sv.TrajectoryRequest(rid, sysp, psi0, n_steps * dt, dt,
                                hierarchy_param={"MAXHIER": depth},
                                eom_param={"EQUATION_OF_MOTION": "NORMALIZED NONLINEAR"},
                                noise_param=noise, adaptive=adaptive, arrival=arrival)


def _chain(n, seed):
    rng = np.random.default_rng(seed)
    return chain(n, 50.0, rng.normal(0, 100, n), 50.0, 50.0)


def test_hierarchy_size_is_exact():
    assert sv.hierarchy_size(20, 4) == 10626
    assert sv.hierarchy_size(20, 6) == 230230
    assert sv.hierarchy_size(200, 8) > 10 ** 13


def test_footprint_kernels_and_scaling():
    small = _req(0, dimer(), 4, 10)
    fp, kern = sv.footprint(small, "mixed")
    assert kern == "resident" and 0 < fp < 1 << 20
    big = _req(1, ring20(), 4, 10)
    fp_m, kern = sv.footprint(big, "mixed")
    assert kern == "streaming"
    # 10626 x 20 elements: complex128 state + 3 complex64 stage vectors + a
    # complex64 shadow of the state at least
    assert fp_m >= 10626 * 20 * (16 + 4 * 8)
    fp_64, _ = sv.footprint(big, "complex64")
    fp_128, _ = sv.footprint(big, "complex128")
    assert fp_64 < fp_m < fp_128
    ad = _req(2, _chain(30, 1), 6, 10, adaptive=(1e-3, 1e-3))
    fp_a, kern = sv.footprint(ad, "mixed")
    assert kern == "adaptive" and fp_a >= sv.ADAPTIVE_ALLOWANCE


def test_admission_first_fit_reject_and_fairness():
    a = _req(0, ring20(), 4, 10)
    b = _req(1, dimer(), 4, 10, arrival=0.001)
    c = _req(2, _chain(200, 2), 8, 10, arrival=0.002)   # can never fit
    fa = sv.footprint(a, "mixed")[0]
    fb = sv.footprint(b, "mixed")[0]
    budget = fa + fb // 2
    arrival = {r.rid: r.arrival for r in (a, b, c)}
    # a does not fit next to what is in use, b does: first fit admits b
    admit, reject = sv.plan_admission([a, b, c], arrival, used=fb, budget=budget, now=0.01,
                                      fairness_s=1.0, precision="mixed")
    assert [r.rid for r, _, _ in admit] == [1]
    assert [r.rid for r, _ in reject] == [2]
    # a has waited past the fairness limit: b may overtake it only while b is
    # small against the budget
    admit, reject = sv.plan_admission([a, b], arrival, used=fb, budget=budget, now=5.0,
                                      fairness_s=1.0, precision="mixed", small_frac=0.0)
    assert admit == [] and reject == []
    admit, _ = sv.plan_admission([a, b], arrival, used=fb, budget=budget, now=5.0,
                                 fairness_s=1.0, precision="mixed", small_frac=0.5)
    assert [r.rid for r, _, _ in admit] == [1]
    admit, _ = sv.plan_admission([a, b], arrival, used=0, budget=budget, now=5.0,
                                 fairness_s=1.0, precision="mixed")
    assert [r.rid for r, _, _ in admit] == [0]


def test_heavy_requests_held_while_light_ones_run():
    """Shortest job first with ageing: a streaming-kernel request waits while
    light requests run, unless it has waited longer than heavy_hold_s."""
    heavy = _req(0, ring20(), 4, 10)
    light = _req(1, dimer(), 4, 10, arrival=0.001)
    assert sv.footprint(heavy, "mixed")[1] == "streaming"
    assert sv.footprint(light, "mixed")[1] == "resident"
    arrival = {0: 0.0, 1: 0.001}
    big = 1 << 40
    admit, _ = sv.plan_admission([heavy, light], arrival, used=0, budget=big, now=1.0,
                                 fairness_s=1.0, precision="mixed", hold_heavy=True,
                                 heavy_hold_s=10.0)
    assert [r.rid for r, _, _ in admit] == [1]
    admit, _ = sv.plan_admission([heavy, light], arrival, used=0, budget=big, now=11.0,
                                 fairness_s=100.0, precision="mixed", hold_heavy=True,
                                 heavy_hold_s=10.0)
    assert [r.rid for r, _, _ in admit] == [0, 1]
    admit, _ = sv.plan_admission([heavy, light], arrival, used=0, budget=big, now=1.0,
                                 fairness_s=1.0, precision="mixed", hold_heavy=False,
                                 heavy_hold_s=10.0)
    assert [r.rid for r, _, _ in admit] == [0, 1]


def test_served_stream_specs_are_seeded():
    s1 = served_stream_specs(64)
    s2 = served_stream_specs(64)
    assert [x["n_site"] for x in s1] == [x["n_site"] for x in s2]
    assert all(2 <= x["n_site"] <= 200 and 3 <= x["depth"] <= 8 for x in s1)
    assert all(200 <= x["t_max"] <= 2000 for x in s1)
    arr = np.array([x["arrival"] for x in served_stream_specs(4096)])
    assert np.all(np.diff(arr) > 0)
    assert 1.5e-3 < arr[-1] / 4096 < 2.5e-3
    r = served_request(s1[0])
    assert r.n_state == s1[0]["n_site"] and r.noise_param["TLEN"] >= r.t_max + r.dt


def _mix():
    return [
        _req(0, dimer(), 4, 40, arrival=0.0),
        _req(1, _chain(6, 1), 3, 25, arrival=0.0),
        _req(2, ring20(), 4, 12, arrival=0.0),
        _req(3, _chain(12, 3), 4, 30, arrival=0.0, adaptive=(1e-3, 1e-3)),
        _req(4, _chain(9, 4), 4, 33, arrival=0.0),
        _req(5, _chain(40, 5), 6, 20, arrival=0.0, adaptive=(1e-3, 1e-3)),
    ]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["complex128", "mixed"])
def test_same_result_alone_and_in_the_mix(precision):
    server = sv.HopsServer(precision=precision, hbm_budget=4 << 30, chunk_steps=16,
                           realtime=False)
    mixed = server.serve(_mix())
    assert all(r.status == "done" for r in mixed), [(r.rid, r.reason) for r in mixed]
    kinds = {r.kernel for r in mixed}
    assert kinds == {"resident", "streaming", "adaptive"}
    for req, res in zip(_mix(), mixed):
        alone = sv.HopsServer(precision=precision, hbm_budget=4 << 30, chunk_steps=16,
                              realtime=False).serve([req])[0]
        assert alone.status == "done"
        assert res.psi_traj.shape == (req.n_steps + 1, req.n_state) or res.kernel == "adaptive"
        # same kernel code and the same step chunks: identical numbers
        assert np.max(np.abs(alone.psi_traj - res.psi_traj)) <= 1e-12
        # another chunking moves only where the lazy renormalisation is applied:
        # identical to rounding in complex128, within float32 storage rounding
        # (1e-6 of max |psi|) with complex64 stage vectors
        other = sv.HopsServer(precision=precision, hbm_budget=4 << 30, chunk_steps=7,
                              realtime=False).serve([req])[0]
        tol = 1e-12 if precision == "complex128" else 1e-6
        assert np.max(np.abs(other.psi_traj - res.psi_traj)) <= tol


@pytest.mark.gpu
def test_served_request_matches_plain_trajectory():
    """A served complex128 request equals HopsTrajectory.propagate of the same inputs."""
    from mesohops_b200 import HopsTrajectory
    req = _mix()[1]
    res = sv.HopsServer(precision="complex128", hbm_budget=1 << 30,
                        realtime=False).serve([req])[0]
    h = HopsTrajectory(req.system_param, eom_param=req.eom_param, noise_param=req.noise_param,
                       hierarchy_param=req.hierarchy_param,
                       device_param={"PRECISION": "complex128"})
    h.initialize(req.psi0)
    h.propagate(req.t_max, req.dt)
    assert np.max(np.abs(np.array(h.storage["psi_traj"]) - res.psi_traj)) <= 1e-12


@pytest.mark.gpu
def test_rejected_requests_get_a_status():
    big = _req(7, _chain(200, 9), 8, 10)
    res = sv.HopsServer(precision="mixed", hbm_budget=1 << 30, realtime=False).serve([big])[0]
    assert res.status == "rejected" and "footprint" in res.reason


@pytest.mark.gpu
def test_adaptive_worker_processes_give_the_same_results():
    """Adaptive requests stepped by worker processes equal the in-process server."""
    mix = _mix()
    local = sv.HopsServer(precision="complex128", hbm_budget=4 << 30, chunk_steps=16,
                          realtime=False).serve(mix)
    srv = sv.HopsServer(precision="complex128", hbm_budget=4 << 30, chunk_steps=16,
                        realtime=False, adaptive_workers=2)
    try:
        pooled = srv.serve(_mix())
    finally:
        srv.close()
    for a, b in zip(local, pooled):
        assert a.status == b.status == "done"
        assert a.kernel == b.kernel
        assert np.max(np.abs(a.psi_traj - b.psi_traj)) <= 1e-12
