"""Failure detection: a trajectory whose state turns NaN/Inf is flagged alone.

Failures are injected on the host -- a NaN written into one trajectory's state,
or into one request's precomputed noise -- never by faulting the GPU.  The
per-trajectory status word (HOPS_ENONFINITE) must flag only the injected
trajectory, TrajectoryError must name it, and every other trajectory must be
bit-identical to a clean run; the serving loop must end only the failing
request as "error" and finish the others unchanged.
"""
import numpy as np
import pytest

from conftest import golden_system, load_golden


# ------------------------------------------------------------------ CPU: host logic
def test_drive_many_isolates_a_failing_coroutine(monkeypatch):
    """Lock-step driving: the request whose step failed gets the error thrown
    into its coroutine; the others finish; collect_errors returns it as that
    coroutine's value, otherwise it is raised after the others finished."""
    from mesohops_b200 import adaptive as ad
    from mesohops_b200.exceptions import TrajectoryError

    class Drv:
        def __init__(self, k):
            self.k = k

    def fake_steps(reqs, device):
        return [TrajectoryError("non-finite state") if r.driver.k == 1 else r.driver.k * 10
                for r in reqs]

    monkeypatch.setattr(ad, "serve_steps", fake_steps)
    finished = []

    def gen(k, n):
        total = 0
        for _ in range(n):
            total += yield ad.StepRequest(Drv(k), None, None, 0.0, 1.0)
        finished.append(k)
        return total

    vals = ad.drive_many([gen(0, 3), gen(1, 3), gen(2, 2)], "cpu", collect_errors=True)
    assert vals[0] == 0 and vals[2] == 40
    assert isinstance(vals[1], TrajectoryError)
    assert sorted(finished) == [0, 2]
    finished.clear()
    with pytest.raises(TrajectoryError):
        ad.drive_many([gen(0, 3), gen(1, 3), gen(2, 2)], "cpu")
    assert sorted(finished) == [0, 2]


# ------------------------------------------------------------------ GPU
def _ensemble(f, B, noise, precision):
    from mesohops_b200 import HopsEnsemble
    ens = HopsEnsemble(golden_system(f), B,
                       noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                    "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision)
    ens.initialize(f["psi0"])
    return ens


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["complex128", "mixed"])
def test_nan_in_one_trajectory_flags_only_it(cuda_device, precision):
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.exceptions import TrajectoryError
    f = load_golden("ring6")
    B, bad, n = 40, 13, 10
    n_l, n_t = f["noise1"].shape
    rng = np.random.default_rng(3)
    noise = ((rng.normal(size=(B, n_l, n_t)) + 1j * rng.normal(size=(B, n_l, n_t))) * 30
             ).astype(np.complex64)
    dt = float(f["dt"])
    runs = {}
    for inject in (False, True):
        ens = _ensemble(f, B, noise, precision)
        ens.propagate(2 * dt, dt)
        ens.batch.settle()   # both runs: the same state with no pending scale
        if inject:   # host-side write into one trajectory's state (aux 0, state 2)
            ens.batch.phi[0, 2, bad] = float("nan")
            if ens.batch.phi_lo is not None:
                ens.batch.phi_lo[0, 2, bad] = float("nan")
        psi = torch.empty((n, B, ens.n_state), dtype=torch.complex128, device="cuda")
        ens.propagate(n * dt, dt, psi_out=psi)
        torch.cuda.synchronize()
        runs[inject] = (psi.cpu().numpy(), ens.batch.status.cpu().numpy(), ens)
    psi_c, st_c, _ = runs[False]
    psi_i, st_i, ens_i = runs[True]
    assert np.count_nonzero(st_c) == 0
    assert st_i[bad] == _lib.HOPS_ENONFINITE
    assert np.count_nonzero(st_i) == 1
    with pytest.raises(TrajectoryError, match=rf"\[{bad}\]"):
        ens_i.check()
    keep = [b for b in range(B) if b != bad]
    assert np.array_equal(psi_i[:, keep], psi_c[:, keep])
    assert not np.all(np.isfinite(psi_i[:, bad]))


def _nan_noise_request(rid, kind):
    """A request of the given kernel kind whose precomputed noise 1 carries a
    NaN at t = 60 fs."""
    from mesohops_b200 import serving as sv
    from mesohops_b200.bath import bcf_exp
    from mesohops_b200.workloads import chain, dimer, ring20
    dt, n_steps = 4.0, 30
    if kind == "resident":
        sysp, depth, adaptive = dimer(), 4, None
    elif kind == "streaming":
        sysp, depth, adaptive = ring20(), 4, None
    else:
        rng = np.random.default_rng(3)
        sysp, depth, adaptive = chain(12, 50.0, rng.normal(0, 100, 12), 50.0, 50.0), 4, (1e-3, 1e-3)
    n = sysp["HAMILTONIAN"].shape[0]
    tlen = (n_steps + 1) * dt
    n_t = int(np.ceil(tlen / (dt / 2))) + 1
    rng = np.random.default_rng(100 + rid)
    z = ((rng.normal(size=(n, n_t)) + 1j * rng.normal(size=(n, n_t))) * 30).astype(np.complex128)
    z[n // 2, 30] = np.nan
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[n // 2] = 1.0
    assert sysp["ALPHA_NOISE1"] is bcf_exp
    return sv.TrajectoryRequest(rid, sysp, psi0, n_steps * dt, dt,
                                hierarchy_param={"MAXHIER": depth},
                                eom_param={"EQUATION_OF_MOTION": "NORMALIZED NONLINEAR"},
                                noise_param={"SEED": z, "MODEL": "PRE_CALCULATED",
                                             "TLEN": tlen, "TAU": dt / 2},
                                adaptive=adaptive, arrival=0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("workers", [0, 2])
def test_server_ends_only_the_failing_requests(cuda_device, workers):
    """One failing request of each kernel kind among the clean mix: those end as
    "error", the clean ones finish with the numbers of a clean run."""
    from mesohops_b200 import serving as sv
    from test_serving import _mix
    kw = dict(precision="complex128", hbm_budget=4 << 30, chunk_steps=16, realtime=False)
    clean = sv.HopsServer(**kw).serve(_mix())
    bad = [_nan_noise_request(10, "resident"), _nan_noise_request(11, "streaming"),
           _nan_noise_request(12, "adaptive")]
    srv = sv.HopsServer(adaptive_workers=workers, **kw)
    try:
        res = srv.serve(_mix() + bad)
    finally:
        srv.close()
    by_id = {r.rid: r for r in res}
    for b in bad:
        r = by_id[b.rid]
        assert r.status == "error", (b.rid, r.status, r.reason)
        assert "non-finite" in r.reason
    for c in clean:
        r = by_id[c.rid]
        assert r.status == "done", (c.rid, r.reason)
        assert np.max(np.abs(r.psi_traj - c.psi_traj)) <= 1e-12


@pytest.mark.gpu
def test_grid_barrier_wait_runs_out_and_reports(cuda_device):
    """The persistent step kernel's grid barrier: with every CTA present it
    passes; with one CTA that never arrives (a flag nothing sets) the others
    give up after the time limit, return, and the error word and their result
    say so -- no hang, no fault, the context stays usable."""
    import time
    import torch
    from mesohops_b200 import _lib
    L = _lib.lib()
    bar = torch.zeros(4, dtype=torch.int32, device="cuda")
    n = 8
    out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(L.hops_grid_barrier_test(bar.data_ptr(), out.data_ptr(), n, 5, -1,
                                        2_000_000_000, s), "barrier test")
    torch.cuda.synchronize()
    assert out.tolist() == [1] * n and int(bar[2]) == 0
    limit_ns = 20_000_000
    t0 = time.perf_counter()
    _lib.check(L.hops_grid_barrier_test(bar.data_ptr(), out.data_ptr(), n, 5, 3, limit_ns, s),
               "barrier test")
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    res = out.tolist()
    assert res[3] == 2 and all(r == 0 for i, r in enumerate(res) if i != 3)
    assert int(bar[2]) == 1
    assert dt < 5.0
    # the context is still usable
    x = torch.ones(1024, device="cuda")
    assert float(x.sum()) == 1024.0
