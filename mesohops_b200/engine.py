"""Device state and launch wrappers around the C ABI.

StreamBatch    -- B trajectories sharing one DeviceStructure, layout
                  phi[a][s][b] (trajectory fastest); four streaming stage
                  kernels (+ FP64 stage scalars) per RK4 step
                  (hops_rk4_propagate).
ResidentRunner -- any number of trajectories with their own (possibly
                  different) structures; one CTA per trajectory runs every step
                  of a call in one launch (hops_resident_propagate).
Both keep all state on the device between calls; host copies happen only in
set_state / get_state and for the stored psi trajectory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import HopsBatch, HopsTask, PREC_C128, PREC_C64, PREC_MIXED, EOM_CODES
from .exceptions import TrajectoryError


def precision_code(name):
    """complex128 | complex64 | mixed (complex128 state, complex64 stage vectors)."""
    if name in ("complex128", "c128", PREC_C128):
        return PREC_C128
    if name in ("complex64", "c64", PREC_C64):
        return PREC_C64
    if name in ("mixed", PREC_MIXED):
        return PREC_MIXED
    raise ValueError(f"unknown precision {name}")


def dtypes(prec):
    """(state dtype, stage-vector dtype) of a precision code."""
    if prec == PREC_C128:
        return torch.complex128, torch.complex128
    if prec == PREC_MIXED:
        return torch.complex128, torch.complex64
    return torch.complex64, torch.complex64


def _noise_pair(noise1, noise2):
    """Both noises as contiguous tensors of one element type: complex128 when
    either is complex128 (INTERPOLATE noise), else complex64.  Returns
    (noise1, noise2, 1 if complex128)."""
    c128 = any(n is not None and n.dtype == torch.complex128 for n in (noise1, noise2))
    dt = torch.complex128 if c128 else torch.complex64
    out = [n.to(dt).contiguous() if n is not None else None for n in (noise1, noise2)]
    return out[0], out[1], int(c128)


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


# Autotuned stage-kernel shapes per problem class:
# (n_hier, n_state, n_mode, B, precision, site projector) -> ((nb, chunk_major), fusion)
_TUNE_CACHE = {}


class StreamBatch:
    """B trajectories sharing one structure, propagated by the streaming kernels."""

    def __init__(self, dstruct, n_traj, precision="complex128", eom="NORMALIZED NONLINEAR"):
        self.st = dstruct
        self.dev = dstruct.device
        t = dstruct.tables
        self.B = int(n_traj)
        self.S, self.N, self.M, self.L = t["n_state"], t["n_hier"], t["n_mode"], t["n_lop"]
        self.prec = precision_code(precision)
        self.eom = EOM_CODES[eom]
        pdt, cdt = dtypes(self.prec)
        shape = (self.N, self.S, self.B)
        self.phi = torch.zeros(shape, dtype=pdt, device=self.dev)
        self.acc = torch.empty(shape, dtype=cdt, device=self.dev)
        self.y0 = torch.empty(shape, dtype=cdt, device=self.dev)
        self.y1 = torch.empty(shape, dtype=cdt, device=self.dev)
        self.phi_lo = (torch.zeros(shape, dtype=cdt, device=self.dev)
                       if self.prec == PREC_MIXED else None)
        self.zmem = torch.zeros((self.B, max(self.M, 1)), dtype=torch.complex128, device=self.dev)
        nws = int(_lib.lib().hops_scalar_workspace_doubles(self.S, self.M, self.L, self.B))
        self.work = torch.zeros(nws, dtype=torch.float64, device=self.dev)
        self.status = torch.zeros(self.B, dtype=torch.int32, device=self.dev)
        self.noise1 = None
        self.noise2 = None
        b = HopsBatch()
        b.n_traj, b.precision, b.eom = self.B, self.prec, self.eom
        b.phi, b.acc, b.y0, b.y1 = (self.phi.data_ptr(), self.acc.data_ptr(),
                                    self.y0.data_ptr(), self.y1.data_ptr())
        b.zmem, b.work, b.status = self.zmem.data_ptr(), self.work.data_ptr(), self.status.data_ptr()
        b.noise1 = b.noise2 = None
        b.n_t1 = b.n_t2 = 0
        b.phi_lo = self.phi_lo.data_ptr() if self.phi_lo is not None else None
        b.defer_scale = 0
        self.cb = b
        self._pending = False
        self.tuning = None      # (nb, task order) of the stage kernel, None = automatic
        self.fusion = 0         # hops_step_fusion mode: 0 automatic, 1 separate, 2 persistent
        self.reset()

    @property
    def defer_scale(self):
        """Leave the renormalisation after each propagate call pending in the
        workspace (applied on the fly by the next call, or by ``settle``)
        instead of rescaling the whole state in a separate pass."""
        return bool(self.cb.defer_scale)

    @defer_scale.setter
    def defer_scale(self, on):
        if not on:
            self.settle()
        self.cb.defer_scale = 1 if on else 0

    def settle(self):
        """Apply a pending renormalisation to phi (no-op when none is pending)."""
        if self._pending:
            rc = _lib.lib().hops_batch_settle(C.byref(self.st.cstruct), C.byref(self.cb),
                                              _stream(self.dev))
            _lib.check(rc, "hops_batch_settle")
            self._pending = False

    def reset(self):
        rc = _lib.lib().hops_batch_reset(C.byref(self.st.cstruct), C.byref(self.cb), _stream(self.dev))
        _lib.check(rc, "hops_batch_reset")
        self._pending = False

    def set_noise(self, noise1, noise2=None):
        """noise tensors [B, L, n_t] on the device, complex64 or (INTERPOLATE)
        complex128 (noise2 may be None)."""
        self.noise1, self.noise2, self.cb.noise_c128 = _noise_pair(noise1, noise2)
        self.cb.noise1 = self.noise1.data_ptr() if self.noise1 is not None else None
        self.cb.n_t1 = self.noise1.shape[-1] if self.noise1 is not None else 0
        self.cb.noise2 = self.noise2.data_ptr() if self.noise2 is not None else None
        self.cb.n_t2 = self.noise2.shape[-1] if self.noise2 is not None else 0

    def set_state(self, phi, zmem=None):
        """phi: [B, N*S] complex (reference layout per trajectory); zmem: [B, M]."""
        ph = torch.as_tensor(np.asarray(phi), dtype=torch.complex128).reshape(self.B, self.N, self.S)
        self.phi.copy_(ph.permute(1, 2, 0).to(self.dev, dtype=self.phi.dtype))
        if self.phi_lo is not None:
            self.phi_lo.copy_(self.phi)
        if zmem is not None and self.M:
            self.zmem.copy_(torch.as_tensor(np.asarray(zmem), dtype=torch.complex128).reshape(self.B, self.M))
        self.reset()

    def get_state(self):
        self.settle()
        ph = self.phi.permute(2, 0, 1).reshape(self.B, self.N * self.S).to(torch.complex128)
        return ph.cpu().numpy(), self.zmem[:, :self.M].cpu().numpy()

    def tune_key(self):
        return (self.N, self.S, self.M, self.B, self.prec, self.st.tables["site_projector"])

    def autotune(self, it0, di, tau_over_hbar, steps=2):
        """Pick the stage-kernel shape (trajectories per warp task, task order).

        Times every candidate for `steps` RK4 steps on the current state, then
        restores the state; the winner is cached per problem class.  Batches of
        fewer than 32 trajectories use the narrow kernel and need no tuning.
        """
        self.tuning = None
        self.fusion = 0
        if self.B < 32:
            return None
        # timing only: run from noise index 0 and stay inside the noise axis
        it0 = 0
        n_t = min([x for x in (self.cb.n_t1, self.cb.n_t2) if x > 0] or [1 << 30])
        if 2 * (steps + 1) * di >= n_t:
            return None
        key = self.tune_key()
        if key in _TUNE_CACHE:
            self.tuning, self.fusion = _TUNE_CACHE[key]
            return self.tuning
        L = _lib.lib()
        pending = self._pending
        saved = [t.clone() for t in (self.phi, self.zmem, self.work, self.status)]
        if self.phi_lo is not None:
            saved.append(self.phi_lo.clone())
        nbmax = (self.B + 31) // 32
        # task orders 0 and 1 coincide when a warp task covers the whole batch.
        # The persistent step kernel (fusion 2) is not a candidate: on the
        # 20-site ring it ran 1.2-2.1x slower than the separate launches
        cands = [(nb, cm, 1) for nb in (1, 2, 4, 8) if nb == 1 or nb <= 2 * nbmax
                 for cm in (0, 1, 2, 3) if cm != 1 or 32 * nb < self.B]
        best, best_ms = None, float("inf")
        for nb, cm, fu in cands:
            L.hops_stage_tuning(nb, cm)
            L.hops_step_fusion(fu)
            self.propagate(it0, di, 1, tau_over_hbar, tuned=False)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            self.propagate(it0, di, steps, tau_over_hbar, tuned=False)
            e1.record()
            torch.cuda.synchronize(self.dev)
            ms = e0.elapsed_time(e1)
            if ms < best_ms:
                best, best_ms = (nb, cm, fu), ms
            for dst, src in zip((self.phi, self.zmem, self.work, self.status, self.phi_lo), saved):
                dst.copy_(src)
        L.hops_stage_tuning(0, -1)
        L.hops_step_fusion(0)
        self._pending = pending
        self.tuning, self.fusion = best[:2], best[2]
        _TUNE_CACHE[key] = (self.tuning, self.fusion)
        return self.tuning

    def propagate(self, it0, di, n_steps, tau_over_hbar, psi_out=None, tuned=True):
        """n_steps RK4 steps; psi_out: optional device tensor [n_steps, B, S] complex128."""
        L = _lib.lib()
        if tuned:
            nb, cm = getattr(self, "tuning", None) or (0, -1)
            L.hops_stage_tuning(nb, cm)
            L.hops_step_fusion(int(getattr(self, "fusion", 0)))
        ptr = psi_out.data_ptr() if psi_out is not None else None
        rc = L.hops_rk4_propagate(C.byref(self.st.cstruct), C.byref(self.cb), int(it0), int(di),
                                  int(n_steps), float(tau_over_hbar), ptr, _stream(self.dev))
        _lib.check(rc, "hops_rk4_propagate")
        if n_steps > 0 and self.cb.defer_scale:
            self._pending = True

    def check_status(self):
        st = self.status.cpu().numpy()
        if np.any(st == _lib.HOPS_ETIMEOUT):
            raise TrajectoryError("a grid barrier of the step kernel timed out in trajectories "
                                  f"{np.nonzero(st == _lib.HOPS_ETIMEOUT)[0].tolist()}")
        if np.any(st != 0):
            raise TrajectoryError(f"non-finite state in trajectories {np.nonzero(st)[0].tolist()}")

    def dsystem_dt(self, z1, z2=None):
        """One derivative of every trajectory at the current state.

        z1, z2: [B, L] complex64 noise samples.  Returns (dphi [B, N*S] complex128
        in cm^-1, dz [B, M] complex128).
        """
        z1d = torch.as_tensor(np.asarray(z1, dtype=np.complex64)).reshape(self.B, self.L).to(self.dev)
        z2d = (torch.as_tensor(np.asarray(z2, dtype=np.complex64)).reshape(self.B, self.L).to(self.dev)
               if z2 is not None else None)
        dphi = torch.empty(self.phi.shape, dtype=self.acc.dtype, device=self.dev)
        dz = torch.empty((self.B, max(self.M, 1)), dtype=torch.complex128, device=self.dev)
        rc = _lib.lib().hops_dsystem_dt(C.byref(self.st.cstruct), C.byref(self.cb), z1d.data_ptr(),
                                        z2d.data_ptr() if z2d is not None else None,
                                        dphi.data_ptr(), dz.data_ptr(), _stream(self.dev))
        _lib.check(rc, "hops_dsystem_dt")
        out = dphi.permute(2, 0, 1).reshape(self.B, self.N * self.S).to(torch.complex128)
        return out.cpu().numpy(), dz[:, :self.M].cpu().numpy()


class ResidentTrajectory:
    """Device buffers of one trajectory for the resident kernel."""

    def __init__(self, dstruct, precision="complex128", eom="NORMALIZED NONLINEAR"):
        self.st = dstruct
        self.dev = dstruct.device
        t = dstruct.tables
        self.S, self.N, self.M, self.L = t["n_state"], t["n_hier"], t["n_mode"], t["n_lop"]
        self.prec = precision_code(precision)
        self.eom = EOM_CODES[eom]
        pdt, cdt = dtypes(self.prec)
        self.phi = torch.zeros(self.N * self.S, dtype=pdt, device=self.dev)
        self.scratch = torch.empty(3 * self.N * self.S, dtype=cdt, device=self.dev)
        self.zmem = torch.zeros(max(self.M, 1), dtype=torch.complex128, device=self.dev)
        self.noise1 = None
        self.noise2 = None
        self.scale = 1.0
        self.status = 0
        self.sc_doubles = int(_lib.lib().hops_resident_scalar_doubles(self.S, self.M, self.L))

    def set_state(self, phi, zmem=None):
        self.phi.copy_(torch.as_tensor(np.asarray(phi), dtype=torch.complex128).to(self.dev, self.phi.dtype))
        if zmem is not None and self.M:
            self.zmem[:self.M].copy_(torch.as_tensor(np.asarray(zmem), dtype=torch.complex128))
        self.scale = 1.0

    def get_state(self):
        return (self.phi.to(torch.complex128).cpu().numpy() * self.scale,
                self.zmem[:self.M].cpu().numpy())

    def set_noise(self, noise1, noise2=None):
        """[L, n_t] device tensors, complex64 or (INTERPOLATE) complex128."""
        self.noise1, self.noise2, self.noise_c128 = _noise_pair(noise1, noise2)


class ResidentRunner:
    """Launches hops_resident_propagate over a list of ResidentTrajectory."""

    def __init__(self, device):
        self.dev = torch.device(device)

    def run(self, trajs, it0, di, n_steps, tau_over_hbar, psi_out=None):
        """Propagate every trajectory n_steps steps in one launch.

        it0, di, n_steps, tau_over_hbar may be scalars or per-trajectory lists.
        psi_out: optional list of device tensors [n_steps_i, S_i] complex128.
        Returns the per-trajectory status array.
        """
        return self.collect(self.launch(trajs, it0, di, n_steps, tau_over_hbar, psi_out))

    def launch(self, trajs, it0, di, n_steps, tau_over_hbar, psi_out=None, state_ptrs=None):
        """Enqueue the launch of ``run`` on the current stream and return a handle
        for ``collect`` (nothing waits on the device here).  state_ptrs: optional
        per-trajectory (phi, z_mem) device addresses used instead of the
        trajectories' own buffers (which then start unscaled)."""
        n = len(trajs)
        if n == 0:
            return None
        prec = trajs[0].prec
        if any(t.prec != prec for t in trajs):
            raise ValueError("one resident launch needs one precision")

        def per(x, i):
            return x[i] if isinstance(x, (list, tuple, np.ndarray)) else x

        tasks = (HopsTask * n)()
        for i, tr in enumerate(trajs):
            tk = tasks[i]
            tk.st = tr.st.dev_ptr
            if state_ptrs is not None:
                tk.phi, tk.zmem = state_ptrs[i]
            else:
                tk.phi = tr.phi.data_ptr()
                tk.zmem = tr.zmem.data_ptr()
            tk.noise_c128 = getattr(tr, "noise_c128", 0)
            tk.noise1 = tr.noise1.data_ptr() if tr.noise1 is not None else None
            tk.noise2 = tr.noise2.data_ptr() if tr.noise2 is not None else None
            tk.n_t1 = tr.noise1.shape[-1] if tr.noise1 is not None else 0
            tk.n_t2 = tr.noise2.shape[-1] if tr.noise2 is not None else 0
            tk.psi_out = psi_out[i].data_ptr() if psi_out is not None and psi_out[i] is not None else None
            tk.scratch = tr.scratch.data_ptr()
            tk.it0, tk.di, tk.n_steps = int(per(it0, i)), int(per(di, i)), int(per(n_steps, i))
            last = tk.it0 + 2 * tk.n_steps * tk.di
            if tk.n_steps > 0 and ((tr.noise1 is not None and last >= tk.n_t1)
                                   or (tr.noise2 is not None and last >= tk.n_t2)):
                raise TrajectoryError("Trajectory times longer than the noise time axis")
            tk.precision = prec
            tk.eom = tr.eom
            tk.status = 0
            tk.tau_over_hbar = float(per(tau_over_hbar, i))
            tk.scale = tr.scale if state_ptrs is None else 1.0
        raw = np.frombuffer(bytes(tasks), dtype=np.uint8).copy()
        tdev = torch.from_numpy(raw).to(self.dev)
        max_elems = max(t.N * t.S for t in trajs)
        max_sc = max(t.sc_doubles for t in trajs)
        site = int(all(t.st.tables["site_projector"] for t in trajs))
        rc = _lib.lib().hops_resident_propagate(tdev.data_ptr(), n, max_elems, max_sc, prec, site,
                                                _stream(self.dev))
        _lib.check(rc, "hops_resident_propagate")
        return (trajs, tdev, torch.cuda.current_stream(self.dev))

    def run_packed(self, trajs, phis, zmems, it0, di, n_steps, tau_over_hbar):
        """``run`` with the states on the host: every trajectory's phi and z_mem
        travel in one host->device copy each way (packed back to back) instead
        of one per trajectory.  Returns (status, [phi], [z_mem]) with phi
        already renormalised by the kernel."""
        n = len(trajs)
        prec = trajs[0].prec
        pdt = trajs[0].phi.dtype
        npdt = np.complex128 if pdt == torch.complex128 else np.complex64
        sizes = [t.N * t.S for t in trajs]
        zs = [max(t.M, 1) for t in trajs]
        po = np.concatenate([[0], np.cumsum(sizes)])
        zo = np.concatenate([[0], np.cumsum(zs)])
        hphi = np.empty(po[-1], dtype=npdt)
        hz = np.zeros(zo[-1], dtype=np.complex128)
        for i, t in enumerate(trajs):
            hphi[po[i]:po[i + 1]] = phis[i]
            if t.M:
                hz[zo[i]:zo[i] + t.M] = zmems[i]
        dphi = torch.from_numpy(hphi).to(self.dev)
        dz = torch.from_numpy(hz).to(self.dev)
        isz = 16 if pdt == torch.complex128 else 8
        views = []
        for i, t in enumerate(trajs):
            views.append((dphi.data_ptr() + int(po[i]) * isz, dz.data_ptr() + int(zo[i]) * 16))
        handle = self.launch(trajs, it0, di, n_steps, tau_over_hbar, state_ptrs=views)
        status = self.collect(handle)
        ophi = dphi.cpu().numpy().astype(np.complex128)
        oz = dz.cpu().numpy()
        return (status, [ophi[po[i]:po[i + 1]] for i in range(n)],
                [oz[zo[i]:zo[i] + t.M] for i, t in enumerate(trajs)])

    def collect(self, handle):
        """Wait for a launch and return its per-trajectory status array."""
        if handle is None:
            return np.zeros(0, dtype=np.int32)
        trajs, tdev, stream = handle
        n = len(trajs)
        with torch.cuda.stream(stream):
            back = tdev.cpu().numpy().tobytes()
        out = (HopsTask * n).from_buffer_copy(back)
        status = np.array([out[i].status for i in range(n)], dtype=np.int32)
        for i, tr in enumerate(trajs):
            tr.scale = 1.0
            tr.status = int(status[i])
        return status
