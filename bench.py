#!/usr/bin/env python
"""Headline benchmark: RK4 traj.steps/s of the HOPS trajectory hot path on B200.

Default workload (the one the target is quoted on): 20-site ring, depth 4
(10626 aux x 20 states), 128 trajectories per GPU, complex64 state / SpMM with
FP64 <L>, norm and z_mem, dt = 4 fs.  One "step" = one RK4 step of all 128
trajectories (4 stage kernels + 4 FP64 stage-scalar kernels).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload ring20|chain10]
  python bench.py --impl reference ...     # CPU reference arm (the oracle port)
  python bench.py --stage-probe 4,0 [--probe-time] ...   # stage-kernel shapes (profiling)

Multi-GPU: one process per GPU (torchrun); every rank propagates its own 128
trajectories (different seeds), no data-path collective ("scaling": "weak");
the timed region is the max over ranks.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK4 traj·steps/s on 1 B200, served/batched vs plain, ≤1e-5 pop. err; p50/p99"
UNIT = "traj·steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    from mesohops_b200.workloads import WORKLOADS
    ap.add_argument("--workload", default="ring20", choices=sorted(WORKLOADS),
                    help="ring20 (the benchmark), chain10; chain120 and dimer for the stage probe")
    ap.add_argument("--precision", default="complex128",
                    choices=["mixed", "complex64", "complex128"],
                    help="precision of the timed batch (the headline) and of the served and "
                         "adaptive legs: complex128 is the one that meets the 1e-5 population "
                         "bound on every noise realisation measured; mixed = complex128 state "
                         "with complex64 stage vectors; the accuracy leg times and checks the "
                         "reduced precisions on the side")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the plain/accuracy/e2e/CPU/served/adaptive legs (profiling runs)")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream leg")
    ap.add_argument("--no-adaptive", action="store_true", help="skip the adaptive-batch leg")
    ap.add_argument("--served-requests", type=int, default=512)
    ap.add_argument("--served-cap-s", type=float, default=120.0,
                    help="time cap of the served stream; requests unfinished then are "
                         "reported as cancelled")
    ap.add_argument("--served-plain", type=int, default=12,
                    help="completed requests rerun one at a time on the plain path")
    ap.add_argument("--served-plain-cap-s", type=float, default=60.0)
    ap.add_argument("--adaptive-traj", type=int, default=512)
    ap.add_argument("--adaptive-steps", type=int, default=6,
                    help="early phase of the adaptive leg (the inch-worm integrator's 5 steps "
                         "and one more)")
    ap.add_argument("--adaptive-steady-steps", type=int, default=50,
                    help="steady phase of the adaptive leg, timed on its own")
    ap.add_argument("--workers", type=int, default=-1,
                    help="adaptive worker processes (-1: min(12, cores - 4))")
    ap.add_argument("--stage-probe", nargs="+", metavar="NB,CM", default=None,
                    help="profiling mode: run the workload's batched stage kernel in the given "
                         "shapes (trajectories per warp task / 32, chunk-major order) for "
                         "--steps steps each after --warmup steps, in argument order (for a "
                         "profiler to pick out), instead of the benchmark")
    ap.add_argument("--probe-time", action="store_true",
                    help="with --stage-probe: time each shape with CUDA events and print "
                         "{shape: [ms per step, ms per stage launch]}")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples of one GPU during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(parts)
            except Exception:
                pass
        os.remove(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


# ------------------------------------------------------------- GPU pieces --
def algorithmic_bytes_per_step(t, B, precision):
    """Compulsory bytes of one RK4 step: every vector touched once per stage.

    Stage 1 reads phi and writes acc, Y2; stage 2 reads Y, phi, acc and writes
    acc, Y; stage 3 reads Y, phi, acc and writes the partial sum
    P = phi + h/6 (k1 + 2 k2 + 2 k3) and Y; stage 4 reads Y and P and writes
    phi: 16 vector passes, 4 of them on phi.  In the mixed mode phi and P are
    complex128 and the stage vectors complex64; P's halves take the
    accumulator's buffer and that of the complex64 copy of phi, which stage 4
    writes and stage 1 reads for its own element besides phi.  Tables per
    stage: int32 aux + int32 mode per up/down connection, the down
    coefficient and k_decay per aux.
    """
    n = t["n_hier"] * t["n_state"] * B
    sv = 16 if precision == "complex128" else 8          # stage vectors
    sp = 8 if precision == "complex64" else 16            # state
    if precision == "mixed":
        # 12 complex64 passes (the copy of phi's write and read among them),
        # 4 on phi, P (complex128) written and read
        per = 12 * sv + 4 * sp + 2 * 16
    else:
        per = 12 * sv + 4 * sp
    sc = 8 if precision != "complex128" else 16
    t_idx = (len(t["up_aux"]) * 8 + len(t["dn_aux"]) * (8 + sc) + t["n_hier"] * sc)
    return n * per + 4 * t_idx


def workload_config(wl, B, world):
    """The ``config`` object of both arms (GPU and reference) for a workload."""
    from math import comb
    sysp = wl["system"]()
    n_state = sysp["HAMILTONIAN"].shape[0]
    n_mode = len(sysp["GW_SYSBATH"])
    return {"workload": wl["desc"], "n_hier": comb(n_mode + wl["depth"], wl["depth"]),
            "n_state": n_state, "n_traj_per_gpu": B, "dt_fs": wl["dt"],
            "parallelism": f"replicas x{world} (trajectory-sharded, no collectives)"}


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from mesohops_b200 import _lib
    from mesohops_b200.ensemble import HopsEnsemble
    from mesohops_b200.workloads import WORKLOADS

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    wl = WORKLOADS[args.workload]
    B, dt, depth = wl["n_traj"], wl["dt"], wl["depth"]
    K, W = args.steps, max(args.warmup, 3)
    tau_noise = dt / 2.0
    tlen = (W + 2 * K + 120 + wl["n_steps"]) * dt + dt
    noise = {"MODEL": "FFT_FILTER", "TLEN": float(tlen), "TAU": tau_noise,
             "SEED": rank_seeds(rank, B)}
    sysp = wl["system"]()
    ens = HopsEnsemble(sysp, B, noise_param=noise, hierarchy_param={"MAXHIER": depth},
                       precision=args.precision, device=dev)
    psi0 = np.zeros(ens.n_state, dtype=complex)
    psi0[0] = 1.0
    ens.initialize(psi0)
    ens.propagate(W * dt, dt)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.propagate(K * dt, dt)
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    ens.check()
    value = B * K * world / (ms / 1e3)
    # separate launches: per step 4 x (stage scalars + stage kernel); the
    # persistent step kernel: one launch for the call.  After the call
    # k_finalize only (HopsEnsemble defers the renormalisation of its last step)
    persistent = int(getattr(ens.batch, "fusion", 0)) == 2
    launches = (1 if persistent else 8 * K) + 1

    result = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
              "steps": K, "warmup": W, "ms_per_step": round(ms / K, 4),
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
              # mixed: complex128 state and FP64 arithmetic, complex64 stage vectors
              "dtype": {"mixed": "c128/c64", "complex64": "c64",
                        "complex128": "c128"}[args.precision],
              "data": "synthetic (seeded)",
              "gpu_launches": launches}
    t = ens.dstruct.tables
    result["config"] = workload_config(wl, B, world)
    assert result["config"]["n_hier"] == t["n_hier"]
    result["config"].update({
        "precision": {
            "mixed": "complex64 stage vectors and SpMM, complex128 state, FP64 <L>/norm/z_mem",
            "complex64": "complex64 state, stage vectors and SpMM, FP64 <L>/norm/z_mem",
            "complex128": "complex128 throughout"}[args.precision],
        "l2": f"inputs larger than L2: each stage vector is "
              f"{t['n_hier'] * t['n_state'] * B * (16 if args.precision == 'complex128' else 8) / 1e6:.0f}"
              " MB (L2 126 MB)"})

    # ---- roofline of the dominant kernel ----
    L = _lib.lib()
    import ctypes as C
    kr = min(K, 20)
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks and "hbm_gbs" in peaks else 6650.0
    step_bytes = algorithmic_bytes_per_step(t, B, args.precision)
    traffic = None
    if persistent:
        # the persistent step kernel: one launch runs the kr steps of a call
        # (the k_finalize after it is inside the events too, ~0.1 % of them)
        torch.cuda.synchronize()
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        r0.record()
        ens.propagate(kr * dt, dt)
        r1.record()
        torch.cuda.synchronize()
        avg_ms = r0.elapsed_time(r1)
        bytes_launch = step_bytes * kr
        kernel, share = f"k_persist (fused RK4 steps, {kr} steps per launch)", 1.0
        prof = os.path.join(ROOT, "profiles", f"k_persist_{args.workload}_{args.precision}.md")
        key = "dram_bytes_per_step:"
    else:
        L.hops_kernel_timing(1)
        ens.propagate(kr * dt, dt)
        torch.cuda.synchronize()
        tot = C.c_double(0)
        nl = C.c_int64(0)
        L.hops_kernel_timing_read(C.byref(tot), C.byref(nl))
        L.hops_kernel_timing(0)
        avg_ms = tot.value / max(nl.value, 1)
        bytes_launch = step_bytes / 4.0
        kernel = "k_wide (streaming RK4 stage)"
        share = round(tot.value / kr / (ms / K), 3)
        prof = os.path.join(ROOT, "profiles", f"k_wide_{args.workload}_{args.precision}.md")
        key = "dram_bytes_per_launch:"
    achieved = bytes_launch / (avg_ms / 1e3) / 1e9
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith(key):
                traffic = int(line.split(":")[1]) * (kr if persistent else 1)
    result["roofline"] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                          "unit": "GB/s", "frac": round(achieved / peak, 4),
                          "traffic": traffic, "kernel": kernel,
                          "algorithmic_bytes_per_launch": int(bytes_launch),
                          "avg_launch_ms": round(avg_ms, 5),
                          "stage_share_of_step": share,
                          "peak_source": "of measured" if peaks else "of fallback"}
    result["clocks"] = clocks

    if not args.no_extras:
        # every rank: the end-to-end number at N GPUs (max wall clock over ranks)
        sec, ke, h2d, d2h = e2e_leg(ens, B, K, dt, dev)
        result["e2e"] = e2e_record(B, world, max_over_ranks(sec, dev), ke, h2d, d2h)
        # the single-GPU legs take minutes; at N > 1 they would keep the other
        # ranks waiting past the process-group timeout, so they run at N = 1
        if world == 1:
            result.update(extras(args, wl, sysp, ens, dev, value, K))
        else:
            result["single_gpu_legs"] = "reported by the N = 1 run"
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


def e2e_leg(ens, B, K, dt, dev):
    """End to end through the public API with host buffers: every step copies its
    noise window host->device (pinned) and reads psi back device->host.  Returns
    (seconds of this rank's host wall clock, steps, h2d bytes, d2h bytes)."""
    import torch
    ke = min(K, 50)
    noise_host = ens.noise.cpu().pin_memory()
    psi_dev = torch.empty((1, B, ens.n_state), dtype=torch.complex128, device=dev)
    psi_host = torch.empty((1, B, ens.n_state), dtype=torch.complex128).pin_memory()
    di = int(round(dt * 0.5 / ens.noise_param["TAU"]))
    h2d = d2h = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        it0 = int(round(ens.t / ens.noise_param["TAU"]))
        sl = slice(it0, it0 + 2 * di + 1)
        ens.noise[:, :, sl].copy_(noise_host[:, :, sl], non_blocking=True)
        h2d += noise_host[:, :, sl].numel() * 8
        ens.propagate(dt, dt, psi_out=psi_dev)
        psi_host.copy_(psi_dev, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        d2h += psi_host.numel() * 16
    return time.perf_counter() - t0, ke, h2d, d2h


def e2e_record(B, world, seconds, ke, h2d, d2h):
    return {"value": round(B * world * ke / seconds, 2), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / ke), "d2h_bytes_per_step": int(d2h / ke),
            "note": "HopsEnsemble.propagate one step per call, noise window h2d from pinned "
                    "memory and psi d2h each step, host wall clock (max over ranks)"}


def rank_seeds(rank, B):
    """Noise seeds of one rank: disjoint blocks of B per rank (weak scaling)."""
    return list(range(rank * B, rank * B + B))


def max_over_ranks(x, device):
    """Max of a float over the ranks of the process group (x itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def extras(args, wl, sysp, ens, dev, value, K):
    """Single-GPU legs (N = 1 only): plain complex128 path, accuracy of the
    batched reduced-precision path, the CPU baseline, the served stream and the
    adaptive batch."""
    import torch
    from mesohops_b200.ensemble import HopsEnsemble
    out = {}
    B, dt, depth = wl["n_traj"], wl["dt"], wl["depth"]
    tlen = ens.noise_param["TLEN"]
    # plain: one trajectory at a time, complex128 (the reference's call, on GPU)
    kp = min(K, 50)
    plain = HopsEnsemble(sysp, 1, noise_param={"MODEL": "FFT_FILTER", "TLEN": tlen,
                                               "TAU": dt / 2, "SEED": [0]},
                         hierarchy_param={"MAXHIER": depth}, precision="complex128", device=dev)
    psi0 = np.zeros(plain.n_state, dtype=complex)
    psi0[0] = 1.0
    plain.initialize(psi0)
    plain.propagate(3 * dt, dt)
    torch.cuda.synchronize()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record()
    plain.propagate(kp * dt, dt)
    a1.record()
    torch.cuda.synchronize()
    plain_v = kp / (a0.elapsed_time(a1) / 1e3)
    out["plain_c128"] = {"value": round(plain_v, 2), "unit": UNIT,
                         "ms_per_step": round(a0.elapsed_time(a1) / kp, 4),
                         "note": "one trajectory per call, complex128 everywhere"}
    out["batched_over_plain"] = round(value / plain_v, 2)

    # accuracy over independent noise realisations (seed blocks of B): every
    # precision against the CPU oracle; the reduced precisions timed on the
    # first realisation as legs of their own
    acc, ms = accuracy_leg(args, wl, sysp, dev)
    out["accuracy"] = acc
    for prec, m in ms.items():
        if prec == args.precision:
            continue
        key = {"complex128": "batched_c128", "mixed": "batched_mixed",
               "complex64": "batched_complex64"}[prec]
        out[key] = {"value": round(B / (m / 1e3), 2), "unit": UNIT, "ms_per_step": round(m, 4),
                    "max_pop_err_vs_oracle": acc["per_precision"][prec]["max_pop_err_vs_oracle"],
                    "over_plain": round(B / (m / 1e3) / plain_v, 2),
                    "note": f"the same {B}-trajectory batch in {prec}, CUDA events over the "
                            f"{wl['n_steps']} steps of the first accuracy realisation"}

    out["noise_setup"] = noise_setup_leg(ens, dev)
    out["cpu_baseline"] = cpu_baseline(wl, sysp)
    if not args.no_served:
        out["served"] = served_leg(args, dev)
    if not args.no_adaptive:
        out["adaptive_batch"] = adaptive_leg(args, dev)
    return out


def noise_setup_leg(ens, dev, reps=3, host_sample=8):
    """Set-up of the batch's FFT_FILTER noise: the SEEDs hashed into PCG64
    states on the device (wall clock, with their upload), the raw draws on the device
    (hops_noise_draw) and the FP64 filter, CUDA events over `reps` runs each,
    beside numpy's host draws of the same rows (the reference's generator, a
    sample of `host_sample` trajectories scaled to the batch); the sample's
    device rows are checked equal to numpy's bit for bit."""
    import torch
    from mesohops_b200.noise import HopsNoise, draw_from_states, filter_on_device, \
        seed_states_on_device
    from oracle import hops_oracle as O
    B, L, n_t = ens.B, ens.system.n_lop, ens.n_t
    seeds = list(range(B))
    model = ens.noise_param["RAND_MODEL"]
    alpha = HopsNoise({k: v for k, v in ens.noise_param.items() if k != "T_AXIS"},
                      ens.system)._corr()
    seed_states_on_device(seeds, dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = seed_states_on_device(seeds, dev)
    torch.cuda.synchronize()
    hash_ms = (time.perf_counter() - t0) * 1e3
    lp = torch.arange(L, dtype=torch.int32, device=dev)
    draw_from_states(st, lp, n_t, model)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(reps):
        z = draw_from_states(st, lp, n_t, model)
    e[1].record()
    for _ in range(reps):
        filter_on_device(alpha, z, dev)
    e[2].record()
    torch.cuda.synchronize()
    nb = min(host_sample, B)
    t0 = time.perf_counter()
    host = np.concatenate([O.raw_draws(s, range(L), n_t, model) for s in seeds[:nb]], axis=0)
    host_s = (time.perf_counter() - t0) * B / nb
    same = bool(np.array_equal(z[:nb * L].cpu().numpy(), host))
    return {"rows": B * L, "samples_per_row": 2 * (n_t - 1), "rand_model": model,
            "seed_states_ms": round(hash_ms, 3),
            "device_draws_ms": round(e[0].elapsed_time(e[1]) / reps, 4),
            "device_filter_ms": round(e[1].elapsed_time(e[2]) / reps, 3),
            "host_numpy_draws_ms": round(host_s * 1e3, 1),
            "host_sample": f"{nb} of {B} trajectories, scaled to {B}",
            "device_draws_equal_numpy": same}


def _oracle_psi(job):
    """psi(t) of one trajectory by the CPU oracle (process-pool worker)."""
    wl_name, noise, n_steps = job
    os.environ["OMP_NUM_THREADS"] = "1"
    from threadpoolctl import threadpool_limits
    from oracle import hops_oracle as O
    from mesohops_b200.workloads import WORKLOADS
    wl = WORKLOADS[wl_name]
    dt = wl["dt"]
    with threadpool_limits(1):
        b = O.OracleBasis(wl["system"](), wl["depth"])
        psi0 = np.zeros(b.nstate, dtype=complex)
        psi0[0] = 1.0
        _, psi, _, _ = O.propagate(b, psi0, noise, dt / 2, n_steps * dt, dt)
    return psi[1:]


def wl_elems(wl):
    """Aux count of a workload's hierarchy."""
    from math import comb
    n_mode = len(wl["system"]()["GW_SYSBATH"])
    return comb(n_mode + wl["depth"], wl["depth"])


def accuracy_leg(args, wl, sysp, dev, n_real=4, n_oracle=2,
                 precisions=("complex128", "mixed", "complex64")):
    """Population error over n_real independent noise realisations (seeds
    r*B .. r*B + B - 1 of FFT_FILTER noise, r < n_real), each over the
    configuration's full run, for every precision: against the GPU complex128
    path for every trajectory, and against the CPU oracle (the FP64
    restatement of the reference) on the n_oracle trajectories of each
    realisation where the first reduced precision errs most, all on the same
    complex64 noise.  Returns (record, {precision: ms per step of the batch on
    the first realisation})."""
    import multiprocessing as mp
    import torch
    from mesohops_b200.ensemble import HopsEnsemble
    B, dt, depth, na = wl["n_traj"], wl["dt"], wl["depth"], wl["n_steps"]
    name = [k for k, v in __import__("mesohops_b200.workloads", fromlist=["x"]).WORKLOADS.items()
            if v is wl][0]
    tlen = (na + 2) * dt
    psi0 = np.zeros(sysp["HAMILTONIAN"].shape[0], dtype=complex)
    psi0[0] = 1.0
    reduced = [p for p in precisions if p != "complex128"]
    per = {p: {"vs_c128": [], "vs_oracle": 0.0} for p in precisions}
    jobs, picks, ms = [], [], {}
    for r in range(n_real):
        res, noise_host = {}, None
        for prec in precisions:
            e = HopsEnsemble(sysp, B, noise_param={"MODEL": "FFT_FILTER", "TLEN": tlen,
                                                   "TAU": dt / 2,
                                                   "SEED": list(range(r * B, r * B + B))},
                             hierarchy_param={"MAXHIER": depth}, precision=prec, device=dev)
            e.initialize(psi0)
            e.tune(dt)      # the autotuner's candidate runs stay out of the timing
            psi = torch.empty((na, B, e.n_state), dtype=torch.complex128, device=dev)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            e.propagate(na * dt, dt, psi_out=psi)
            e1.record()
            torch.cuda.synchronize()
            if r == 0:
                ms[prec] = e0.elapsed_time(e1) / na
            res[prec] = psi.cpu().numpy()
            if noise_host is None:
                noise_host = e.noise.cpu().numpy()
            del e
        p128 = np.abs(res["complex128"]) ** 2
        worst = None
        for prec in reduced:
            err = np.abs(np.abs(res[prec]) ** 2 - p128).max(axis=(0, 2))
            per[prec]["vs_c128"].append(float(err.max()))
            if worst is None:
                worst = np.argsort(err)[::-1][:n_oracle]
        if worst is None:
            worst = np.arange(n_oracle)
        for b in worst:
            jobs.append((name, noise_host[b], na))
            picks.append({prec: res[prec][:, b] for prec in precisions})
    # the oracle runs after the GPU work, in spawned processes; a full run of a
    # hierarchy of millions of elements would take the oracle hours
    if picks and picks[0]["complex128"].shape[1] * wl_elems(wl) > 5e6:
        jobs, picks = [], []
    oracle = []
    if jobs:
        ctx = mp.get_context("spawn")
        with ctx.Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
            oracle = pool.map(_oracle_psi, jobs)
    c128_rel = 0.0
    for pk, po in zip(picks, oracle):
        for prec in precisions:
            e = float(np.max(np.abs(np.abs(pk[prec]) ** 2 - np.abs(po) ** 2)))
            per[prec]["vs_oracle"] = max(per[prec]["vs_oracle"], e)
        c128_rel = max(c128_rel, float(np.max(np.abs(pk["complex128"] - po)) / np.max(np.abs(po))))
    out = {p: {"max_pop_err_vs_oracle": per[p]["vs_oracle"] if picks else None,
               "max_pop_err_vs_c128_per_realisation": per[p]["vs_c128"] or None}
           for p in precisions}
    rec = {"precision": args.precision,
           "max_pop_err_vs_oracle": out[args.precision]["max_pop_err_vs_oracle"],
           "c128_vs_oracle_max_rel": c128_rel if picks else None,
           "per_precision": out,
           "sample": f"{n_real} noise realisations x {B} trajectories x {na} steps (FFT_FILTER "
                     f"seeds 0..{n_real * B - 1}); every precision against the GPU complex128 "
                     f"path on all trajectories and against the oracle (FP64 CPU restatement of "
                     f"the reference) on the {n_oracle} trajectories of each realisation where "
                     f"{reduced[0] if reduced else 'complex128'} errs most, same complex64 noise"}
    return rec, ms


def served_leg(args, dev):
    """The served request stream (Poisson arrivals, mixed system and hierarchy
    sizes, adaptive or not): its first ``--served-requests`` requests through
    HopsServer (continuous batching, admission by the HBM footprint against
    the device's free memory less a reserve) under a time cap, then the first
    completed ones again one at a time with the plain complex128 path."""
    import torch
    from mesohops_b200 import serving as sv
    from mesohops_b200.trajectory import HopsTrajectory
    from mesohops_b200.workloads import served_request, served_stream_specs
    specs = served_stream_specs()[:args.served_requests]
    reqs = [served_request(s) for s in specs]
    workers = args.workers if args.workers >= 0 else max(0, min(12, (os.cpu_count() or 2) - 4))
    srv = sv.HopsServer(device=dev, precision=args.precision, hbm_budget=None,
                        chunk_steps=32, realtime=True, adaptive_workers=workers)
    budget = srv.budget
    try:
        res = srv.serve(reqs, deadline_s=args.served_cap_s)
    finally:
        srv.close()
    summ = sv.summarize(res, srv.stats["makespan_s"])
    kinds = {}
    for r in res:
        if r.status == "done":
            kinds[r.kernel] = kinds.get(r.kernel, 0) + 1
    # plain: completed requests one at a time, complex128, wall clock
    n_plain, steps_plain, t_plain = 0, 0, 0.0
    for r, q in zip(res, reqs):
        if r.status != "done" or n_plain >= args.served_plain or t_plain > args.served_plain_cap_s:
            continue
        h = HopsTrajectory(q.system_param, eom_param=q.eom_param, noise_param=q.noise_param,
                           hierarchy_param=q.hierarchy_param, storage_param={},
                           device_param={"PRECISION": "complex128", "DEVICE": str(dev)})
        if q.adaptive is not None:
            h.make_adaptive(q.adaptive[0], q.adaptive[1])
        h.initialize(q.psi0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h.propagate(q.t_max, q.dt)
        torch.cuda.synchronize()
        t_plain += time.perf_counter() - t0
        steps_plain += q.n_steps
        n_plain += 1
    return {
        "stream": f"first {len(reqs)} of the 4096-request stream (seed 4): Poisson arrivals "
                  "(mean 2 ms), chains of 2-200 sites, depth 3-8, adaptive by a fair coin",
        "precision": args.precision, "hbm_budget_bytes": budget,
        "hbm_budget": "free device memory after the worker processes started, less a reserve "
                      "of max(4 GiB, 5 %)",
        "time_cap_s": args.served_cap_s,
        "adaptive_worker_processes": workers,
        "completed": summ["completed"], "rejected": summ["rejected"], "errors": summ["errors"],
        "cancelled_at_cap": summ["cancelled"],
        "rejected_why": "device footprint (state, stage vectors, tables, noise, psi(t)) above "
                        "the HBM budget",
        "by_kernel": kinds, "traj_steps": summ["traj_steps"],
        "traj_steps_per_s": round(summ["traj_steps_per_s"], 2),
        "p50_ms": round(summ["p50_ms"], 1) if summ["p50_ms"] is not None else None,
        "p99_ms": round(summ["p99_ms"], 1) if summ["p99_ms"] is not None else None,
        "makespan_s": round(summ["makespan_s"], 2),
        "plain_c128": {"requests": n_plain, "traj_steps": steps_plain,
                       "traj_steps_per_s": round(steps_plain / t_plain, 2) if t_plain > 0 else None,
                       "note": "the first completed requests again (arrival order, up to "
                               f"{args.served_plain} or {args.served_plain_cap_s:.0f} s), one at a "
                               "time, HopsTrajectory complex128, propagate wall clock"},
        "latency": "completion minus arrival, wall clock of the serving loop, completed "
                   "requests"}


def adaptive_leg(args, dev):
    """Adaptive HOPS with uneven bases: the 500-site chain, depth 10,
    delta = 1e-3, many trajectories spread over worker processes on the GPU;
    each worker steps its share in lock-step -- every RK4 step of all of them
    in one persistent resident-kernel launch (each with its own basis), every
    flux-error evaluation in one launch."""
    from mesohops_b200.adaptive_pool import AdaptiveWorkers
    from mesohops_b200.serving import TrajectoryRequest
    from mesohops_b200.workloads import adaptive_chain500
    n, K1, K2 = args.adaptive_traj, args.adaptive_steps, args.adaptive_steady_steps
    K = K1 + K2
    sysp, psi0, seeds = adaptive_chain500(n)
    dt = 4.0
    workers = args.workers if args.workers >= 0 else max(1, min(12, (os.cpu_count() or 2) - 4))
    workers = max(1, workers)
    pool = AdaptiveWorkers(workers, dev, args.precision)
    try:
        t0 = time.perf_counter()
        for sd in seeds:
            pool.submit(sd, TrajectoryRequest(
                sd, sysp, psi0, K * dt, dt, hierarchy_param={"MAXHIER": 10},
                eom_param={"EQUATION_OF_MOTION": "NORMALIZED NONLINEAR"},
                noise_param={"SEED": sd, "MODEL": "FFT_FILTER", "TLEN": (K + 8) * dt,
                             "TAU": dt / 2},
                adaptive=(1e-3, 1e-3)))
        errors = []
        while any(pool.building):
            for ev in pool.events(timeout=1.0):
                errors.extend(ev[2])
        t_init = time.perf_counter() - t0
        done, phases = [], []
        for k in (K1, K2):
            if k <= 0:
                continue
            t0 = time.perf_counter()
            pool.step_idle(k)
            while any(pool.stepping):
                for ev in pool.events(timeout=1.0):
                    done.extend(ev[1])
                    errors.extend(ev[2])
            phases.append((k, time.perf_counter() - t0))
    finally:
        pool.close()
    sizes = np.array([d[3] * d[4] for d in done]) if done else np.zeros(1)
    live = n - len(errors)
    return {"workload": "500-site chain (J=50, eps~N(0,100) seed 3), DL (50,50,295 K) per "
                        "site, depth 10, delta_a = delta_s = 1e-3, dt = 4 fs, psi_0 on a "
                        f"seeded site; {n} trajectories (noise seeds 0..{n - 1})",
            "steps": K, "completed": len(done), "errors": len(errors),
            "traj_steps_per_s_early": round(live * phases[0][0] / phases[0][1], 2),
            "traj_steps_per_s_steady": (round(live * phases[1][0] / phases[1][1], 2)
                                        if len(phases) > 1 else None),
            "traj_steps_per_s": round(live * K / sum(t for _, t in phases), 2),
            "basis_elems_end": {"min": int(sizes.min()), "median": int(np.median(sizes)),
                                "max": int(sizes.max())},
            "worker_processes": workers, "init_s": round(t_init, 2),
            "precision": args.precision,
            "note": f"early phase: the first {K1} steps (inch-worm early integrator); steady "
                    f"phase: the next {K2} steps, timed on its own; wall clock of the stepping; "
                    "each worker process steps its trajectories in lock-step with one resident "
                    "launch per step for all of them"}


def stage_probe(args):
    """Fixed stage-kernel shapes on a workload (profiling aid): no JSON line of
    the benchmark, only "ok" or, with --probe-time, per-shape timings."""
    import ctypes as C
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.constants import hbar
    from mesohops_b200.ensemble import HopsEnsemble
    from mesohops_b200.workloads import WORKLOADS
    W = WORKLOADS[args.workload]
    B, dt = W["n_traj"], W["dt"]
    shapes = [tuple(int(x) for x in sh.split(",")) for sh in args.stage_probe]
    n_need = args.warmup + (len(shapes) + 1) * (args.steps + 1) + 4
    ens = HopsEnsemble(W["system"](), B,
                       noise_param={"SEED": list(range(B)), "MODEL": "FFT_FILTER",
                                    "TLEN": n_need * dt, "TAU": dt / 2},
                       hierarchy_param={"MAXHIER": W["depth"]}, precision=args.precision,
                       autotune=False)
    psi0 = np.zeros(ens.n_state, complex)
    psi0[0] = 1.0
    ens.initialize(psi0)
    h = dt / hbar
    # NB,ORDER[,FUSION]: fusion 1 = separate launches (default), 2 = persistent step kernel
    def use(sh):
        ens.batch.tuning = sh[:2]
        ens.batch.fusion = sh[2] if len(sh) > 2 else 1

    use(shapes[0])
    ens.batch.propagate(0, 1, args.warmup, h)
    L = _lib.lib()
    out = {}
    for sh in shapes:
        use(sh)
        if not args.probe_time:
            ens.batch.propagate(0, 1, args.steps, h)
            continue
        torch.cuda.synchronize()
        L.hops_kernel_timing(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ens.batch.propagate(0, 1, args.steps, h)
        e1.record()
        torch.cuda.synchronize()
        tot = C.c_double(0)
        nl = C.c_int64(0)
        L.hops_kernel_timing_read(C.byref(tot), C.byref(nl))
        L.hops_kernel_timing(0)
        out[str(sh)] = [round(e0.elapsed_time(e1) / args.steps, 4),
                        round(tot.value / max(nl.value, 1), 4)]
    torch.cuda.synchronize()
    ens.check()
    print(json.dumps(out) if args.probe_time else "ok", flush=True)


# ------------------------------------------------------------- CPU legs --
def _oracle_noise(b, seed, n_steps, dt):
    n_l = len(b.sys["L"])
    n_t = int(np.ceil((n_steps + 2) * dt / (dt / 2))) + 1
    rng = np.random.default_rng(seed)
    return ((rng.normal(size=(n_l, n_t)) + 1j * rng.normal(size=(n_l, n_t))) * 40
            ).astype(np.complex64)


def _oracle_worker(args):
    """One trajectory of the oracle: n_warm untimed steps, then n_steps timed
    steps from the same start (single thread)."""
    wl_name, seed, n_steps, n_warm = args
    os.environ["OMP_NUM_THREADS"] = "1"
    from threadpoolctl import threadpool_limits
    from oracle import hops_oracle as O
    from mesohops_b200.workloads import WORKLOADS
    wl = WORKLOADS[wl_name]
    sysp = wl["system"]()
    dt = wl["dt"]
    with threadpool_limits(1):
        b = O.OracleBasis(sysp, wl["depth"])
        noise = _oracle_noise(b, seed, max(n_steps, n_warm), dt)
        psi0 = np.zeros(b.nstate, dtype=complex)
        psi0[0] = 1.0
        if n_warm > 0:
            O.propagate(b, psi0, noise, dt / 2, n_warm * dt, dt)
        t0 = time.perf_counter()
        O.propagate(b, psi0, noise, dt / 2, n_steps * dt, dt)
        return time.perf_counter() - t0


def cpu_baseline(wl, sysp, n_steps=4):
    """The oracle port (numpy, one thread) on one trajectory, n_steps steps."""
    name = [k for k, v in __import__("mesohops_b200.workloads", fromlist=["x"]).WORKLOADS.items()
            if v is wl][0]
    el = _oracle_worker((name, 0, n_steps, 1))
    return {"value": round(n_steps / el, 3), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 trajectory x {n_steps} RK4 steps of the same system with the numpy "
                      "oracle (single thread, after 1 untimed step)"}


def _reference_core(wl_name, seeds, K, W, barrier, out):
    """One host core of the reference arm: its share of the trajectories.

    Every trajectory runs its W warm-up steps first (untimed); after a barrier
    with the other cores, each trajectory advances K steps from its warm state,
    one after the other.  Puts this core's seconds for the timed steps on out."""
    os.environ["OMP_NUM_THREADS"] = "1"
    from threadpoolctl import threadpool_limits
    from oracle import hops_oracle as O
    from mesohops_b200.workloads import WORKLOADS
    wl = WORKLOADS[wl_name]
    dt = wl["dt"]
    with threadpool_limits(1):
        b = O.OracleBasis(wl["system"](), wl["depth"])
        S = b.nstate
        states = []
        for sd in seeds:
            noise = _oracle_noise(b, sd, W + K, dt)
            phi = np.zeros(b.nhier * S, dtype=np.complex128)
            phi[0] = 1.0
            zmem = np.zeros(b.nmode, dtype=np.complex128)
            states.append([noise, phi, zmem])
        t = 0.0

        def advance(st, n0, n):
            noise, phi, zmem = st
            for k in range(n0, n0 + n):
                tt = k * dt
                zr = O.noise_lookup(noise, [tt, tt + dt / 2, tt + dt], dt / 2)
                phi, zmem = O.rk4_step(b, phi, zmem, zr, np.zeros_like(zr), dt)
                phi = O.normalize(phi, S)
            st[1], st[2] = phi, zmem

        for st in states:
            advance(st, 0, W)
        barrier.wait()
        t0 = time.perf_counter()
        for st in states:
            advance(st, W, K)
        t = time.perf_counter() - t0
    out.put(t)


def run_reference(args):
    """CPU arm: the oracle port (the reference algorithm restated in numpy) on
    every host core, on the same workload as the GPU arm: all of its
    trajectories, dealt round-robin to one process per core, W untimed
    warm-up steps and K timed steps each.  The timed region is the slowest
    core's K-step loop; value = trajectories x K / that time."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from mesohops_b200.workloads import WORKLOADS
    wl = WORKLOADS[args.workload]
    B = wl["n_traj"]
    cores = max(1, min(os.cpu_count() or 1, B))
    K = max(1, args.steps)
    W = max(0, args.warmup)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(cores)
    out = ctx.Queue()
    procs = [ctx.Process(target=_reference_core,
                         args=(args.workload, list(range(c, B, cores)), K, W, barrier, out))
             for c in range(cores)]
    for p in procs:
        p.start()
    times = [out.get() for _ in procs]
    for p in procs:
        p.join()
    el = max(times)
    v = B * K / el
    line = {"metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": round(el / K * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic (seeded)", "impl": "reference",
            "config": dict(workload_config(wl, B, world),
                           precision="complex128 throughout (the reference's arithmetic)",
                           l2="host caches; no GPU in this arm"),
            "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"all {B} trajectories of the workload, dealt to {cores} "
                                       f"processes (one per host core, one thread each); {W} "
                                       f"untimed warm-up steps, then {K} timed RK4 steps each "
                                       "(numpy oracle, complex128)"},
            "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.stage_probe:
        stage_probe(a)
    else:
        run_gpu(a)
