"""Adaptive trajectories spread over worker processes that share one GPU.

The adaptive basis update is host work -- thresholds, boundary sets, the
permutation and rebuild of the basis -- of a few milliseconds per trajectory
and step, against microseconds of device time.  ``AdaptiveWorkers`` runs that
host work in parallel: each worker process owns a subset of the adaptive
trajectories and a CUDA context on the same device, and steps its subset in
lock-step (``adaptive.drive_many``: one resident-kernel launch for all its
trajectories' RK4 steps, one launch for all their flux errors).  The kernels of
different workers are independent and short, so the GPU interleaves them; no
kernel waits on another.

Protocol (one duplex pipe per worker): ("add", [(key, request)]) builds and
initialises trajectories; ("step", n) advances every trajectory of the worker
by up to n steps and returns the ones that finished; ("stop",) ends the worker.
A request is a ``serving.TrajectoryRequest`` with ``adaptive`` set.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time
import traceback


def _worker(conn, device, precision):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    import numpy as np
    import torch
    from . import adaptive as ad
    from .trajectory import HopsTrajectory
    torch.set_num_threads(1)
    torch.cuda.set_device(torch.device(device))
    torch.zeros(1, device=device)          # create the CUDA context before reporting ready
    from . import _lib
    _lib.lib()
    conn.send(("ready",))
    live = {}   # key -> [traj, request, steps done]
    while True:
        msg = conn.recv()
        if msg[0] == "stop":
            conn.send(("stopped",))
            return
        if msg[0] == "add":
            errors, added = [], []
            for key, req in msg[1]:
                try:
                    h = HopsTrajectory(req.system_param, eom_param=req.eom_param,
                                       noise_param=req.noise_param,
                                       hierarchy_param=req.hierarchy_param, storage_param={},
                                       device_param={"PRECISION": precision,
                                                     "DEVICE": str(device)})
                    h.make_adaptive(req.adaptive[0], req.adaptive[1],
                                    update_step=req.update_step, f_discard=req.f_discard)
                    h.initialize(req.psi0)
                    live[key] = [h, req, 0]
                    added.append(key)
                except Exception as exc:  # reported to the parent, worker stays up
                    errors.append((key, f"{type(exc).__name__}: {exc}"))
            torch.cuda.synchronize()
            conn.send(("added", added, errors))
        elif msg[0] == "step":
            n = int(msg[1])
            done, errors = [], []
            try:
                for _ in range(n):
                    act = [(k, v) for k, v in live.items() if v[2] < v[1].n_steps]
                    if not act:
                        break
                    gens = [v[0].adaptive_step_gen((v[2] + 1) * v[1].dt, v[1].dt, v[2])
                            for _, v in act]
                    vals = ad.drive_many(gens, device, collect_errors=True)
                    for (k, v), val in zip(act, vals):
                        if isinstance(val, Exception):   # this trajectory only
                            errors.append((k, f"{type(val).__name__}: {val}"))
                            live.pop(k)
                        else:
                            v[2] += 1
            except Exception as exc:
                tb = traceback.format_exc(limit=3)
                errors += [(k, f"{type(exc).__name__}: {exc} {tb}") for k in list(live)]
                live.clear()
            for k in [k for k, v in live.items() if v[2] >= v[1].n_steps]:
                h, req, _ = live.pop(k)
                done.append((k, np.asarray(h.storage["psi_traj"]),
                             np.asarray(h.storage["t_axis"]), int(h.n_hier), int(h.n_state)))
            conn.send(("stepped", done, errors))


class AdaptiveWorkers:
    """A pool of worker processes stepping adaptive trajectories on one GPU.

    Non-blocking: ``submit`` queues a trajectory on the least-loaded worker,
    ``step_idle`` asks every idle worker with trajectories to advance them, and
    ``events`` returns the replies that have arrived ("added" with build
    failures, "stepped" with finished trajectories and failures)."""

    def __init__(self, n_workers, device="cuda:0", precision="mixed"):
        ctx = mp.get_context("spawn")
        self.device = str(device)
        self.conns, self.procs = [], []
        t0 = time.perf_counter()
        for _ in range(int(n_workers)):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_worker, args=(b, self.device, precision), daemon=True)
            p.start()
            self.conns.append(a)
            self.procs.append(p)
        for c in self.conns:                    # every worker has its CUDA context
            if c.recv()[0] != "ready":
                raise RuntimeError("adaptive worker failed to start")
        self.load = [0] * len(self.conns)      # trajectories owned
        self.building = [0] * len(self.conns)  # add messages not yet answered
        self.stepping = [False] * len(self.conns)
        self.owner = {}
        self.start_s = time.perf_counter() - t0

    def submit(self, key, req):
        w = min(range(len(self.conns)), key=lambda i: self.load[i])
        self.conns[w].send(("add", [(key, req)]))
        self.load[w] += 1
        self.building[w] += 1
        self.owner[key] = w

    def step_idle(self, n):
        for w, c in enumerate(self.conns):
            if self.load[w] > self.building[w] and not self.stepping[w]:
                c.send(("step", n))
                self.stepping[w] = True

    def events(self, timeout=0.0):
        """[("added", keys, errors)] and [("stepped", done, errors)] replies
        received within timeout seconds (0: only those already waiting)."""
        from multiprocessing.connection import wait
        out = []
        ready = wait(self.conns, timeout=timeout)
        for c in ready:
            w = self.conns.index(c)
            while c.poll():
                msg = c.recv()
                if msg[0] == "added":
                    self.building[w] -= 1
                    for key, _ in msg[2]:
                        self.load[w] -= 1
                        self.owner.pop(key, None)
                elif msg[0] == "stepped":
                    self.stepping[w] = False
                    for item in msg[1]:
                        self.load[w] -= 1
                        self.owner.pop(item[0], None)
                    for key, _ in msg[2]:
                        self.load[w] -= 1
                        self.owner.pop(key, None)
                out.append(msg)
        return out

    @property
    def active(self):
        return sum(self.load)

    @property
    def busy(self):
        return any(self.stepping) or any(b > 0 for b in self.building)

    def close(self):
        for c in self.conns:
            try:
                c.send(("stop",))
            except (BrokenPipeError, OSError):
                pass
        for p in self.procs:
            p.join(timeout=30)
            if p.is_alive():
                p.terminate()
        self.conns, self.procs = [], []
