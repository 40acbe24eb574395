"""Stage-kernel probe: run or time fixed stage-kernel shapes on a workload.

    python -m mesohops_b200.stage_probe WORKLOAD PRECISION [--steps N] [--warmup N]
                                        [--time] SHAPE [SHAPE ...]

WORKLOAD is a key of mesohops_b200.workloads.WORKLOADS (ring20, chain10, dimer),
PRECISION complex128 | mixed | complex64, SHAPE "nb,chunk_major" (the values the
autotuner chooses between).  Without --time every shape runs --steps RK4 steps
after the warm-up, in argument order, so a profiler can pick out the launches;
with --time each shape is timed with CUDA events and one JSON line is printed:
{shape: [ms per step, ms per stage launch]}.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np
import torch

from . import _lib
from .constants import hbar
from .ensemble import HopsEnsemble
from .workloads import WORKLOADS


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("precision", choices=["complex128", "mixed", "complex64"])
    ap.add_argument("shapes", nargs="+")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--time", action="store_true")
    a = ap.parse_args(argv)
    W = WORKLOADS[a.workload]
    B, dt = W["n_traj"], W["dt"]
    shapes = [tuple(int(x) for x in s.split(",")) for s in a.shapes]
    n_need = a.warmup + (len(shapes) + 1) * (a.steps + 1) + 4
    ens = HopsEnsemble(W["system"](), B,
                       noise_param={"SEED": list(range(B)), "MODEL": "FFT_FILTER",
                                    "TLEN": n_need * dt, "TAU": dt / 2},
                       hierarchy_param={"MAXHIER": W["depth"]}, precision=a.precision,
                       autotune=False)
    psi0 = np.zeros(ens.n_state, complex)
    psi0[0] = 1.0
    ens.initialize(psi0)
    h = dt / hbar
    ens.batch.tuning = shapes[0]
    ens.batch.propagate(0, 1, a.warmup, h)
    L = _lib.lib()
    out = {}
    for sh in shapes:
        ens.batch.tuning = sh
        if not a.time:
            ens.batch.propagate(0, 1, a.steps, h)
            continue
        torch.cuda.synchronize()
        L.hops_kernel_timing(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ens.batch.propagate(0, 1, a.steps, h)
        e1.record()
        torch.cuda.synchronize()
        tot = C.c_double(0)
        nl = C.c_int64(0)
        L.hops_kernel_timing_read(C.byref(tot), C.byref(nl))
        L.hops_kernel_timing(0)
        out[str(sh)] = [round(e0.elapsed_time(e1) / a.steps, 4),
                        round(tot.value / max(nl.value, 1), 4)]
    torch.cuda.synchronize()
    ens.check()
    print(json.dumps(out) if a.time else "ok")


if __name__ == "__main__":
    main()
