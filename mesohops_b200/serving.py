"""Serving loop: continuous batching of HOPS trajectory requests on one GPU.

Requests (each one ``HopsTrajectory`` worth of parameters: system, hierarchy,
EOM with or without an adaptive basis, noise, psi_0, t_max, dt) arrive over
time.  The server

* admits a request when its HBM footprint fits what is left of the budget
  (requests that can never fit are rejected with a status; the rest wait),
  holding requests for the streaming kernel back while light ones wait or
  run, up to ``heavy_hold_s`` (shortest job first, with ageing);
* builds its device state (structure tables, correlated noise, phi) on a
  builder thread while the GPU keeps stepping the admitted requests;
* advances every admitted request by up to ``chunk_steps`` RK4 steps per tick:
  all non-adaptive requests whose stage vectors fit one CTA's shared memory in
  ONE persistent launch of the resident kernel (different systems and
  hierarchy sizes side by side), the larger ones with the streaming kernels
  each on its own CUDA stream, and the adaptive ones in lock-step (one launch
  for all their steps, one for all their flux errors) on a third stream, so
  the three kinds overlap on the device while the host runs the adaptive
  basis logic;
* retires finished requests (one device->host copy of the stored psi(t)),
  frees their memory and records their completion time.

The results of a request do not depend on what it shares the GPU with: each
trajectory is computed by the same kernel code whether alone or in the mix.

This is the serving layer the reference does not have (it runs one trajectory
per process, README.md:26-27); each request's numbers are those of
``HopsTrajectory.propagate`` (trajectory/hops_trajectory.py:401-538).
"""
from __future__ import annotations

import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait
from math import comb

import numpy as np
import torch

from . import adaptive as _adaptive
from .constants import hbar
from .engine import ResidentRunner
from .exceptions import TrajectoryError, UnsupportedRequest
from .system import pattern_key

# Device bytes assumed for an adaptive request beyond its noise and psi(t)
# (its basis is rebuilt as it grows; ~1e3 aux x ~30 states at most here).
ADAPTIVE_ALLOWANCE = 64 << 20


class TrajectoryRequest:
    """One trajectory to run: the HopsTrajectory dictionaries plus psi_0, the
    propagation (t_max, dt), an optional adaptive (delta_a, delta_s) and the
    arrival time in seconds from the start of the stream."""

    def __init__(self, rid, system_param, psi0, t_max, dt, hierarchy_param=None,
                 eom_param=None, noise_param=None, adaptive=None, arrival=0.0,
                 update_step=1, f_discard=0.01):
        self.rid = rid
        self.system_param = system_param
        self.psi0 = np.asarray(psi0, dtype=np.complex128)
        self.t_max = float(t_max)
        self.dt = float(dt)
        self.hierarchy_param = dict(hierarchy_param or {})
        self.eom_param = dict(eom_param or {})
        self.noise_param = dict(noise_param or {})
        self.adaptive = adaptive
        self.arrival = float(arrival)
        self.update_step = update_step
        self.f_discard = f_discard

    @property
    def n_steps(self):
        return int(np.ceil(self.t_max / self.dt - 1e-12))

    @property
    def n_state(self):
        H = self.system_param["HAMILTONIAN"]
        return int(H.shape[0])

    @property
    def n_mode(self):
        return len(self.system_param["GW_SYSBATH"])

    @property
    def n_lop(self):
        """Unique L-operators (by nonzero pattern, as HopsSystem counts them)."""
        return len({pattern_key(l) for l in self.system_param["L_HIER"]})


class ServedResult:
    """Outcome of one request: status 'done' | 'rejected' | 'error' | 'cancelled'."""

    def __init__(self, req, status, reason="", t_axis=None, psi_traj=None, admitted=None,
                 completed=None, footprint=0, kernel=None):
        self.rid = req.rid
        self.status = status
        self.reason = reason
        self.t_axis = t_axis
        self.psi_traj = psi_traj
        self.arrival = req.arrival
        self.admitted = admitted
        self.completed = completed
        self.footprint = footprint
        self.kernel = kernel
        self.n_steps = req.n_steps if status == "done" else 0

    @property
    def latency(self):
        return None if self.completed is None else self.completed - self.arrival


def hierarchy_size(n_mode, depth):
    """Aux count of the full triangular hierarchy (an exact Python integer)."""
    return comb(n_mode + depth, depth)


def footprint(req, precision):
    """(device bytes, kernel) one request needs while it is admitted.

    Non-adaptive: the state and stage vectors of the kernel it will run on,
    the structure tables (about 64 B per hierarchy connection and 40 B per aux),
    the correlated noise and the stored psi(t).  Adaptive: a fixed allowance
    for the basis plus noise and psi(t)."""
    S, M = req.n_state, req.n_mode
    n_t = int(np.ceil(req.noise_param.get("TLEN", req.t_max + req.dt)
                      / req.noise_param.get("TAU", req.dt / 2))) + 1
    noise = n_t * req.n_lop * 8
    psi = (req.n_steps + 1) * S * 16
    if req.adaptive is not None:
        return ADAPTIVE_ALLOWANCE + noise + psi, "adaptive"
    d = int(req.hierarchy_param.get("MAXHIER", 3))
    N = hierarchy_size(M, d)
    below = hierarchy_size(M, d - 1) if d > 0 else 0
    table = 64 * below * M + 40 * N
    state_b = 16 if precision in ("complex128", "mixed") else 8
    stage_b = 16 if precision == "complex128" else 8
    n_elem = N * S
    if 4 * n_elem * state_b <= _adaptive.RESIDENT_MAX_BYTES:
        vec = n_elem * (state_b + 3 * stage_b)
        kern = "resident"
    else:
        vec = n_elem * (state_b + 3 * stage_b + (stage_b if precision == "mixed" else 0))
        kern = "streaming"
    return vec + table + noise + psi, kern


def plan_admission(queue, arrival, used, budget, now, fairness_s, precision, small_frac=0.02,
                   hold_heavy=False, heavy_hold_s=0.0):
    """Admission decisions for the waiting requests (in arrival order).

    Returns (admit [(req, bytes, kernel)], reject [(req, bytes)]): a request whose
    footprint exceeds the whole budget is rejected; the others are admitted
    first-fit while the budget lasts.  Once the oldest waiting request has
    waited longer than fairness_s, later requests overtake it only if they are
    small (at most small_frac of the budget), so a large request is not starved
    and small ones do not queue behind it.  hold_heavy (set by the server while
    light requests -- adaptive or resident-kernel ones -- wait or run): heavy
    requests (streaming kernel) younger than heavy_hold_s are held back, so the
    short jobs are not slowed by the long ones sharing the GPU (shortest job
    first, with ageing)."""
    admit, reject = [], []
    blocked = False
    head_seen = False
    for req in queue:
        fp, kern = footprint(req, precision)
        if fp > budget:
            reject.append((req, fp))
            continue
        if hold_heavy and kern == "streaming" and now - arrival[req.rid] <= heavy_hold_s:
            continue
        if blocked and fp > small_frac * budget:
            continue
        if used + fp <= budget:
            admit.append((req, fp, kern))
            used += fp
        elif not head_seen and now - arrival[req.rid] > fairness_s:
            blocked = True
        head_seen = True
    return admit, reject


class _Active:
    """An admitted request and its device state."""

    def __init__(self, req, traj, fp, kernel, admitted):
        self.req = req
        self.traj = traj
        self.fp = fp
        self.kernel = kernel
        self.admitted = admitted
        self.done = 0
        self.psi_dev = None
        self.stream = None
        self.failed = None      # error text once the request's state went non-finite


class HopsServer:
    """Continuous-batching server for HOPS trajectories on one GPU."""

    def __init__(self, device="cuda:0", precision="mixed", hbm_budget=None, chunk_steps=32,
                 builders=2, realtime=True, fairness_s=1.0, adaptive_workers=0,
                 heavy_hold_s=10.0):
        """hbm_budget: device bytes the admitted requests may hold (default: the
        free memory, once the worker processes run, less a reserve).  realtime: honour the arrival times (False: every
        request is present at t = 0).  fairness_s: once the oldest waiting
        request has waited this long, later ones are not admitted ahead of it.
        adaptive_workers: > 0 runs the adaptive requests in that many worker
        processes on the same GPU (adaptive_pool.AdaptiveWorkers), so their
        host-side basis updates run in parallel; 0 steps them in this process.
        heavy_hold_s: while light requests (adaptive, or small enough for the
        resident kernel) wait or run, requests for the streaming kernel are
        admitted only once they have waited this long (0: no holding)."""
        self.device = torch.device(device)
        self.precision = precision
        self.chunk = int(chunk_steps)
        self.builders = int(builders)
        self.realtime = realtime
        self.fairness_s = float(fairness_s)
        self.heavy_hold_s = float(heavy_hold_s)
        self.stats = {}
        self.pool = None
        if adaptive_workers > 0:
            from .adaptive_pool import AdaptiveWorkers
            self.pool = AdaptiveWorkers(adaptive_workers, self.device, precision)
        # the workers' CUDA contexts hold device memory too: the default budget
        # is taken from what is free once they run
        if hbm_budget is None:
            hbm_budget = self.free_budget(self.device)
        self.budget = int(hbm_budget)

    @staticmethod
    def free_budget(device, reserve_frac=0.05, reserve_min=4 << 30):
        """Free device memory less a reserve (5 %, at least 4 GiB) for the
        allocator's slack and the kernels' scratch."""
        free, total = torch.cuda.mem_get_info(torch.device(device))
        return max(0, int(free - max(reserve_min, reserve_frac * total)))

    def close(self):
        """Stop the adaptive worker processes (if any)."""
        if self.pool is not None:
            self.pool.close()
            self.pool = None

    # --------------------------------------------------------------- building
    def _build(self, req, kernel):
        """HopsTrajectory for one request, initialised on the device (builder
        thread; its own stream, synchronised before the request goes live)."""
        from .trajectory import HopsTrajectory
        stream = torch.cuda.Stream(self.device)
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            dp = {"PRECISION": self.precision, "DEVICE": str(self.device)}
            if kernel in ("resident", "streaming"):
                dp["KERNEL"] = kernel
            traj = HopsTrajectory(req.system_param, eom_param=req.eom_param,
                                  noise_param=req.noise_param,
                                  hierarchy_param=req.hierarchy_param,
                                  storage_param={}, device_param=dp)
            if req.adaptive is not None:
                traj.make_adaptive(req.adaptive[0], req.adaptive[1],
                                   update_step=req.update_step, f_discard=req.f_discard)
            traj.initialize(req.psi0)
            if req.adaptive is None:
                S = traj.n_state
                psi_dev = torch.empty((req.n_steps, S), dtype=torch.complex128,
                                      device=self.device)
            else:
                psi_dev = None
            stream.synchronize()
        return traj, psi_dev

    # ------------------------------------------------------------------- loop
    def serve(self, requests, deadline_s=None):
        """Serve the requests (sorted by arrival); returns one ServedResult each,
        in request order.  deadline_s: seconds after which every request not
        finished yet (waiting, building or running) ends as "cancelled"."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        order = {r.rid: i for i, r in enumerate(requests)}
        results = {}
        pending = deque(reqs)
        queue = deque()
        building = []           # (future, req, fp, kernel)
        active = []
        used = 0
        builders = ThreadPoolExecutor(max_workers=max(1, self.builders))
        runner = ResidentRunner(self.device)
        s_res = torch.cuda.Stream(self.device)
        s_ad = torch.cuda.Stream(self.device)
        t0 = time.perf_counter()

        def clock():
            return time.perf_counter() - t0

        arrival = {r.rid: (r.arrival if self.realtime else 0.0) for r in reqs}
        n_ticks = 0
        busy = 0.0
        pool = self.pool
        pooled = {}       # rid -> (request, footprint, admitted time or None)
        try:
            while pending or queue or building or active or pooled:
                now = clock()
                if deadline_s is not None and now > deadline_s:
                    why = f"time cap of {deadline_s:.0f} s reached"
                    for req in list(pending) + list(queue):
                        results[req.rid] = ServedResult(req, "cancelled", why)
                    for _, req, fp, _ in building:
                        results[req.rid] = ServedResult(req, "cancelled", why, footprint=fp)
                    for a in active:
                        results[a.req.rid] = ServedResult(a.req, "cancelled", why, footprint=a.fp)
                    for rid, (req, fp, _) in pooled.items():
                        results[rid] = ServedResult(req, "cancelled", why, footprint=fp)
                    pending, queue, building, active, pooled = deque(), deque(), [], [], {}
                    break
                while pending and arrival[pending[0].rid] <= now:
                    queue.append(pending.popleft())
                light = (bool(pooled) or any(a.kernel != "streaming" for a in active)
                         or any(k != "streaming" for _, _, _, k in building)
                         or any(footprint(r, self.precision)[1] != "streaming" for r in queue))
                admit, reject = plan_admission(list(queue), arrival, used, self.budget, now,
                                               self.fairness_s, self.precision,
                                               hold_heavy=self.heavy_hold_s > 0 and light,
                                               heavy_hold_s=self.heavy_hold_s)
                for req, fp in reject:
                    queue.remove(req)
                    results[req.rid] = ServedResult(
                        req, "rejected", f"footprint {fp} B exceeds the HBM budget "
                                         f"{self.budget} B", footprint=fp)
                for req, fp, kern in admit:
                    queue.remove(req)
                    used += fp
                    if kern == "adaptive" and pool is not None:
                        try:
                            pool.submit(req.rid, req)
                        except (UnsupportedRequest, TrajectoryError, ValueError) as exc:
                            used -= fp
                            results[req.rid] = ServedResult(req, "error", str(exc), footprint=fp)
                            continue
                        pooled[req.rid] = [req, fp, None]
                    else:
                        building.append((builders.submit(self._build, req, kern), req, fp, kern))
                if pool is not None and pooled:
                    pool.step_idle(self.chunk)
                # builds that finished become active
                still = []
                for fut, req, fp, kern in building:
                    if fut.done():
                        try:
                            traj, psi_dev = fut.result()
                        except (UnsupportedRequest, TrajectoryError, ValueError) as exc:
                            used -= fp
                            results[req.rid] = ServedResult(req, "error", str(exc), footprint=fp)
                            continue
                        a = _Active(req, traj, fp, traj.kernel, clock())
                        a.psi_dev = psi_dev
                        if a.kernel == "streaming":
                            a.stream = torch.cuda.Stream(self.device)
                        active.append(a)
                    else:
                        still.append((fut, req, fp, kern))
                building = still
                if pooled:
                    for ev in pool.events(timeout=0.0 if (active or building) else 0.02):
                        self._pool_event(ev, pooled, results, clock(), arrival)
                    used = self._used(active, building, pooled, queue)
                if not active:
                    if building:
                        wait([b[0] for b in building], return_when=FIRST_COMPLETED,
                             timeout=0.02 if pooled else None)
                    elif pending and not queue and not pooled:
                        gap = arrival[pending[0].rid] - clock()
                        if gap > 0:
                            time.sleep(gap)
                    continue
                tb = time.perf_counter()
                self._tick(active, runner, s_res, s_ad)
                busy += time.perf_counter() - tb
                n_ticks += 1
                keep = []
                for a in active:
                    if a.failed is not None:      # this request only; the others go on
                        results[a.req.rid] = ServedResult(a.req, "error", a.failed,
                                                          footprint=a.fp)
                        a.traj = a.psi_dev = None
                        used -= a.fp
                    elif a.done >= a.req.n_steps:
                        results[a.req.rid] = self._retire(a, clock())
                        used -= a.fp
                    else:
                        keep.append(a)
                active = keep
        finally:
            builders.shutdown(wait=True)
        self.stats = {"ticks": n_ticks, "tick_s": busy, "makespan_s": clock()}
        out = [results[r.rid] for r in sorted(requests, key=lambda r: order[r.rid])]
        for r in out:
            r.arrival = arrival[r.rid]
        return out

    @staticmethod
    def _used(active, building, pooled, queue):
        return (sum(a.fp for a in active) + sum(b[2] for b in building)
                + sum(v[1] for v in pooled.values()))

    def _pool_event(self, ev, pooled, results, now, arrival):
        """Book-keeping of one adaptive-worker reply."""
        if ev[0] == "added":
            for rid in ev[1]:
                if rid in pooled:
                    pooled[rid][2] = now
            for rid, text in ev[2]:
                req, fp, _ = pooled.pop(rid)
                results[rid] = ServedResult(req, "error", text, footprint=fp)
        elif ev[0] == "stepped":
            for rid, psi, t_axis, _, _ in ev[1]:
                req, fp, adm = pooled.pop(rid)
                results[rid] = ServedResult(req, "done", t_axis=t_axis, psi_traj=psi,
                                            admitted=adm, completed=now, footprint=fp,
                                            kernel="adaptive")
            for rid, text in ev[2]:
                if rid in pooled:
                    req, fp, _ = pooled.pop(rid)
                    results[rid] = ServedResult(req, "error", text, footprint=fp)

    def _tick(self, active, runner, s_res, s_ad):
        res = [a for a in active if a.kernel == "resident"]
        stm = [a for a in active if a.kernel == "streaming"]
        ada = [a for a in active if a.kernel == "adaptive"]
        handle = None
        plan = {}
        if res:
            trajs, it0s, dis, ns, hs, outs = [], [], [], [], [], []
            for a in res:
                n = min(self.chunk, a.req.n_steps - a.done)
                tr = a.traj
                t = a.done * a.req.dt
                trajs.append(tr._traj)
                it0s.append(tr.noise1.time_index(t))
                dis.append(int(round(a.req.dt * 0.5 / tr.noise1.param["TAU"])))
                ns.append(n)
                hs.append(a.req.dt / hbar)
                outs.append(a.psi_dev[a.done:a.done + n])
                plan[id(a)] = n
            with torch.cuda.stream(s_res):
                s_res.wait_stream(torch.cuda.current_stream(self.device))
                handle = runner.launch(trajs, it0s, dis, ns, hs, psi_out=outs)
        for a in stm:
            n = min(self.chunk, a.req.n_steps - a.done)
            tr = a.traj
            t = a.done * a.req.dt
            with torch.cuda.stream(a.stream):
                tr._traj.propagate(tr.noise1.time_index(t),
                                   int(round(a.req.dt * 0.5 / tr.noise1.param["TAU"])), n,
                                   a.req.dt / hbar,
                                   psi_out=a.psi_dev[a.done:a.done + n].view(n, 1, -1))
            plan[id(a)] = n
        if ada:
            n = min(self.chunk, max(a.req.n_steps - a.done for a in ada))
            with torch.cuda.stream(s_ad):
                for k in range(n):
                    live = [a for a in ada if a.done + k < a.req.n_steps and a.failed is None]
                    gens = [a.traj.adaptive_step_gen((a.done + k + 1) * a.req.dt, a.req.dt,
                                                     a.done + k) for a in live]
                    vals = _adaptive.drive_many(gens, self.device, collect_errors=True)
                    for a, v in zip(live, vals):
                        if isinstance(v, Exception):
                            a.failed = f"{type(v).__name__}: {v}"
            for a in ada:
                plan[id(a)] = min(n, a.req.n_steps - a.done)
        if handle is not None:
            st = runner.collect(handle)
            for i in np.nonzero(st)[0]:
                res[i].failed = "TrajectoryError: non-finite state during propagation"
        for a in stm:
            a.stream.synchronize()
            try:
                a.traj._traj.check_status()
            except TrajectoryError as exc:
                a.failed = f"TrajectoryError: {exc}"
        for a in active:
            a.done += plan.get(id(a), 0)

    def _retire(self, a, now):
        req = a.req
        tr = a.traj
        if a.kernel == "adaptive":
            psi = np.asarray(tr.storage["psi_traj"])
            t_axis = np.asarray(tr.storage["t_axis"])
        else:
            psi0 = req.psi0[tr.state_list]
            rest = a.psi_dev.cpu().numpy()
            psi = np.concatenate([psi0[None, :], rest], axis=0)
            t_axis = np.arange(req.n_steps + 1) * req.dt
        out = ServedResult(req, "done", t_axis=t_axis, psi_traj=psi, admitted=a.admitted,
                           completed=now, footprint=a.fp, kernel=a.kernel)
        a.traj = None
        a.psi_dev = None
        return out


def summarize(results, makespan):
    """Throughput and completion-latency percentiles of a served stream."""
    done = [r for r in results if r.status == "done"]
    lat = np.array([r.latency for r in done]) if done else np.zeros(0)
    steps = sum(r.n_steps for r in done)
    return {
        "completed": len(done),
        "rejected": sum(r.status == "rejected" for r in results),
        "errors": sum(r.status == "error" for r in results),
        "cancelled": sum(r.status == "cancelled" for r in results),
        "traj_steps": int(steps),
        "traj_steps_per_s": steps / makespan if makespan > 0 else None,
        "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
        "makespan_s": makespan,
    }
