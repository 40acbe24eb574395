"""Adaptive HOPS (adHOPS) on the device: flux-error estimates in FP64 on the GPU,
basis decisions on the host, propagation with the resident (or streaming)
kernels.

Restates, for systems whose L-operators have no off-diagonal couplings (every
site-projector system):
  * HopsBasis.define_basis / update_basis        basis/hops_basis.py:117-292
  * _define_state_basis, state_stable_error      hops_basis.py:294-482, 795-912
  * _define_hierarchy_basis, hier_stable_error,
    _determine_boundary_hier                     hops_basis.py:484-793
  * the flux filters                             basis/hops_fluxfilters.py:24-515
  * determine_error_thresh                       basis/basis_functions.py:8-41
  * the error terms                              basis/basis_functions_adaptive.py
  * the adaptive part of the propagate loop, the
    inch-worm early integrator, _prepare_zstep   trajectory/hops_trajectory.py:456-533, 636-714
  * z_mem of modes outside the basis             eom/eom_functions.py:122-154

Every trajectory runs as a coroutine that yields device requests (one RK4
step, one set of flux errors) and receives their results.  ``drive`` serves
one trajectory; ``AdaptiveEnsemble`` advances many in lock-step and serves each
round of requests with ONE resident-kernel launch (trajectories of different
basis sizes in one persistent launch) and ONE flux-error launch.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps
import torch

from . import _lib
from ._lib import HopsFluxTask, EOM_CODES
from .constants import hbar, precision
from .device import DeviceStructure, _state_mode_tables, build_tables
from .engine import ResidentRunner, ResidentTrajectory, StreamBatch
from .exceptions import TrajectoryError, UnsupportedRequest
from .hierarchy import (AuxBasis, AuxKeyer, apply_static_filters, insert_mode, remove_mode,
                        triangular_counts, tuples_of)

# Resident kernel when the four stage vectors fit one CTA's shared memory.
RESIDENT_MAX_BYTES = 200 * 1024


# ------------------------------------------------------------------ helpers
def error_thresh(sorted_error, max_error, offset=0.0):
    """Largest error that may be dropped (basis_functions.py:8-41)."""
    thresh = 0.0
    if len(sorted_error) > 0:
        idx = int(np.argmax(np.cumsum(sorted_error) + offset >= max_error))
        if idx > 0:
            thresh = sorted_error[idx - 1]
        elif sorted_error[0] + offset < max_error:
            thresh = np.inf
    return thresh


def keep_from_list(errors, max_error):
    """Indices of the members to keep (hops_basis.py:1000-1028)."""
    thresh = error_thresh(np.sort(errors), max_error)
    return np.nonzero(errors > thresh)[0]


def gt_precision(z):
    """numpy's ordering of complex values against the real precision (real part
    first, then imaginary), as used by ``z_mem > precision``."""
    return (z.real > precision) | ((z.real == precision) & (z.imag > 0))


# -------------------------------------------------------------------- basis
class Basis:
    """One adaptive basis: states, aux list, mode list and the device structure."""

    def __init__(self, system, keyer, maxhier, counts, states, device, noise_host=(None, None)):
        self.system = system
        self.states = np.array(sorted(int(s) for s in states), dtype=np.int64)
        counts = np.asarray(counts, dtype=np.int16).reshape(-1, system.n_mode)
        hier_modes = set(np.nonzero(counts.sum(axis=0) > 0)[0].tolist())
        state_modes = set(m for s in self.states for m in system.modes_by_state[s])
        # HopsModes.list_absindex_mode: hierarchy modes | modes of the basis states
        self.modes = np.array(sorted(hier_modes | state_modes), dtype=np.int64)
        self.aux = AuxBasis(counts, keyer, maxhier, modes=self.modes)
        self.counts = self.aux.counts
        part = _state_mode_part(system, self.states, self.modes)
        self.tables = build_tables(system, self.aux, self.states, self.modes, small=part["small"])
        # the noise rows of the basis L list travel with the structure tables
        extras = {}
        for name, nh in zip(("noise1", "noise2"), noise_host):
            if nh is not None and self.tables["n_lop"]:
                extras[name] = np.ascontiguousarray(nh[self.tables["l_abs"]])
        self.dstruct = DeviceStructure(self.tables, device, extras)
        self.n_hier = self.aux.n_hier
        self.n_state = len(self.states)
        self.n_mode = len(self.modes)
        self.rel_mode = part["rel_mode"]
        self.depth = self.aux.depth
        # K2_aux_by_mode (hops_basis.py:1140-1151)
        self.k_aux = np.ascontiguousarray(self.counts[:, self.modes].T.astype(np.uint8))
        self.lred, self.m2 = part["lred"], part["m2"]
        self.list_sc, self.h_sc = part["list_sc"], part["h_sc"]

    def same_as(self, states, counts):
        states = np.asarray(states)
        if len(states) != self.n_state or len(counts) != self.n_hier:
            return False
        if not np.array_equal(np.sort(states), self.states):
            return False
        # the aux rows are unique, so equal lengths and equal row sets suffice
        if getattr(self, "_row_set", None) is None:
            self._row_set = {r.tobytes() for r in self.counts}
        rows = np.ascontiguousarray(np.asarray(counts, dtype=self.counts.dtype))
        return {r.tobytes() for r in rows} == self._row_set


# Parts of a basis that depend only on its states and modes, cached on the
# HopsSystem object for every basis with the same two lists: an adaptive basis
# usually changes its aux list while its states stay.
_PART_CACHE_SIZE = 512


def _state_mode_part(system, states, modes):
    cache = system.__dict__.setdefault("_adaptive_part_cache", {})
    key = (states.tobytes(), modes.tobytes())
    part = cache.get(key)
    if part is not None:
        return part
    small = _state_mode_tables(system, states, modes)
    l_abs = small["l_abs"]
    # M2_mode_from_state_diag (hops_basis.py:1031-1050), dense [mode, state]
    lred = [system.lop_block(j, states) for j in l_abs]
    rel_l = {int(j): i for i, j in enumerate(l_abs)}
    m2 = np.zeros((len(modes), len(states)), dtype=np.complex128)
    for i, m in enumerate(modes):
        m2[i] = np.diag(lred[rel_l[int(system.l_by_mode[m])]])
    # HopsSystem.list_sc: states outside the basis coupled to it by H
    sset = set(states.tolist())
    sc = set()
    for s in states:
        sc.update(int(c) for c in system.coupled_states[s])
    list_sc = np.array(sorted(sc - sset), dtype=np.int64)
    h_sc = None
    if len(list_sc):
        H = system.hamiltonian
        blk = (sps.csr_matrix(H)[list_sc][:, states].toarray() if sps.issparse(H)
               else np.asarray(H)[np.ix_(list_sc, states)])
        h_sc = -1j * np.asarray(blk, dtype=np.complex128)
    for a in [m2, list_sc] + lred + ([h_sc] if h_sc is not None else []):
        a.flags.writeable = False
    part = dict(small=small, lred=lred, m2=m2, list_sc=list_sc, h_sc=h_sc,
                rel_mode={int(m): i for i, m in enumerate(modes)})
    if len(cache) >= _PART_CACHE_SIZE:
        cache.pop(next(iter(cache)))
    cache[key] = part
    return part


# ----------------------------------------------------------------- requests
class StepRequest:
    """One RK4 step of ``driver`` in its current basis from (phi, zmem_abs) at t.
    effective: the RK noise slots are EFFECTIVE_NOISE_INTEGRATION window means
    (integrator_rk.py:115-128) instead of the samples at t, t + tau/2, t + tau."""
    __slots__ = ("driver", "phi", "zmem_abs", "t", "tau", "effective")

    def __init__(self, driver, phi, zmem_abs, t, tau, effective=False):
        self.driver, self.phi, self.zmem_abs, self.t, self.tau = driver, phi, zmem_abs, t, tau
        self.effective = effective


class FluxRequest:
    """Flux-error arrays of one normalised phi in the driver's current basis."""
    __slots__ = ("driver", "phi", "z_step", "dt", "mask", "with_flux")

    def __init__(self, driver, phi, z_step, dt, mask=None, with_flux=True):
        self.driver, self.phi, self.z_step, self.dt = driver, phi, z_step, dt
        self.mask, self.with_flux = mask, with_flux


def serve_steps(reqs, device):
    """Run every StepRequest; the resident ones in ONE persistent launch.

    A request whose state turned NaN/Inf gets a TrajectoryError instance in
    place of its result, so the other requests of the launch go on."""
    out = [None] * len(reqs)
    res = [i for i, r in enumerate(reqs) if r.driver.kernel == "resident"]
    if res:
        trajs, phis, zms, it0s, dis, hs = [], [], [], [], [], []
        for i in res:
            r = reqs[i]
            d = r.driver
            b = d.basis
            it0, di = d.bind_noise(r)
            trajs.append(d.engine)
            phis.append(r.phi)
            zms.append(r.zmem_abs[b.modes] if b.n_mode else None)
            it0s.append(it0)
            dis.append(di)
            hs.append(r.tau / hbar)
        st, phis_o, zms_o = ResidentRunner(device).run_packed(trajs, phis, zms, it0s, dis, 1, hs)
        for j, i in enumerate(res):
            out[i] = ((phis_o[j], zms_o[j]) if st[j] == 0 else
                      TrajectoryError("non-finite state during adaptive propagation"))
    for i, r in enumerate(reqs):
        if out[i] is not None:
            continue
        d = r.driver
        b = d.basis
        it0, di = d.bind_noise(r)
        eng = d.engine
        eng.set_state(r.phi.reshape(1, -1),
                      r.zmem_abs[b.modes].reshape(1, -1) if b.n_mode else None)
        eng.propagate(it0, di, 1, r.tau / hbar, tuned=False)
        try:
            eng.check_status()
        except TrajectoryError as exc:
            out[i] = exc
            continue
        phi, z = eng.get_state()
        out[i] = (phi[0], z[0])
    return [o if isinstance(o, TrajectoryError) else r.driver.finish_step(r, o[0], o[1])
            for r, o in zip(reqs, out)]


def _pack(arrays):
    """Byte-pack numpy arrays at 16-byte aligned offsets: (buffer, offsets)."""
    offs, total = [], 0
    for a in arrays:
        offs.append(total)
        total += (a.nbytes + 15) // 16 * 16
    buf = np.zeros(max(total, 16), dtype=np.uint8)
    for a, o in zip(arrays, offs):
        buf[o:o + a.nbytes] = np.ascontiguousarray(a).view(np.uint8).ravel()
    return buf, offs


def serve_flux(reqs, device):
    """Every FluxRequest in ONE hops_flux_errors launch (one CTA per request);
    all inputs go up in one copy and all error arrays come back in one."""
    n = len(reqs)
    if n == 0:
        return []
    dev = torch.device(device)
    L = _lib.lib()
    host = []
    shapes = []
    out_doubles = 0
    for r in reqs:
        b = r.driver.basis
        N, S, M = b.n_hier, b.n_state, b.n_mode
        host.append(np.ascontiguousarray(r.phi, dtype=np.complex128))
        host.append(np.ascontiguousarray(r.z_step[2][b.modes] if M else np.zeros(1),
                                         dtype=np.complex128))
        host.append(np.ascontiguousarray(r.z_step[0], dtype=np.complex64))
        host.append(np.ascontiguousarray(r.z_step[1], dtype=np.complex64))
        host.append(np.ascontiguousarray(r.mask if r.mask is not None else np.zeros(1),
                                         dtype=np.int32))
        host.append(b.k_aux.ravel() if b.k_aux.size else np.zeros(1, np.uint8))
        n_out = N * S + (2 * max(M * N, 1) if r.with_flux else 0)
        shapes.append((N, S, M, out_doubles))
        out_doubles += (n_out + 1) // 2 * 2
    buf, offs = _pack(host)
    dbuf = torch.from_numpy(buf).to(dev)
    dout = torch.empty(max(out_doubles, 2), dtype=torch.float64, device=dev)
    base, obase = dbuf.data_ptr(), dout.data_ptr()
    tasks = (HopsFluxTask * n)()
    max_smem = 0
    for i, r in enumerate(reqs):
        b = r.driver.basis
        N, S, M, o = shapes[i]
        tk = tasks[i]
        tk.st = b.dstruct.dev_ptr
        tk.phi = base + offs[6 * i]
        tk.zmem = base + offs[6 * i + 1]
        tk.z1 = base + offs[6 * i + 2]
        tk.z2 = base + offs[6 * i + 3]
        tk.aux_mask = base + offs[6 * i + 4] if r.mask is not None else None
        tk.k_aux = base + offs[6 * i + 5]
        tk.e_deriv = obase + 8 * o
        tk.e_up = obase + 8 * (o + N * S) if r.with_flux else None
        tk.e_down = obase + 8 * (o + N * S + max(M * N, 1)) if r.with_flux else None
        tk.dt = float(r.dt)
        tk.eom = EOM_CODES[r.driver.eom]
        max_smem = max(max_smem, int(L.hops_flux_errors_smem_doubles(S, M, b.tables["n_lop"])))
    raw = torch.from_numpy(np.frombuffer(bytes(tasks), dtype=np.uint8).copy()).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.hops_flux_errors(raw.data_ptr(), n, max_smem, hbar, stream)
    _lib.check(rc, "hops_flux_errors")
    hout = dout.cpu().numpy()
    res = []
    for r, (N, S, M, o) in zip(reqs, shapes):
        e1 = hout[o:o + N * S].reshape(N, S)
        if not r.with_flux:
            res.append((e1, None, None))
            continue
        q = o + N * S
        mn = max(M * N, 1)
        res.append((e1, hout[q:q + M * N].reshape(M, N), hout[q + mn:q + mn + M * N].reshape(M, N)))
    return res


def drive(gen, device):
    """Run one coroutine to completion, serving its requests one at a time."""
    result = None
    while True:
        try:
            req = gen.send(result)
        except StopIteration as stop:
            return stop.value
        if isinstance(req, StepRequest):
            result = serve_steps([req], device)[0]
            if isinstance(result, TrajectoryError):
                raise result
        else:
            result = serve_flux([req], device)[0]


def drive_many(gens, device, collect_errors=False):
    """Run many coroutines in lock-step: every round serves all pending step
    requests with one launch and all pending flux requests with one launch.
    Returns the coroutines' return values.

    A trajectory whose state turns non-finite has the TrajectoryError thrown
    into its coroutine; the others go on.  collect_errors: the exception (or
    any other exception of that coroutine) becomes its value; otherwise the
    first TrajectoryError is raised once the others have finished."""
    values = [None] * len(gens)
    failed = []
    pending = {}
    for i, g in enumerate(gens):
        try:
            pending[i] = g.send(None)
        except StopIteration as stop:
            values[i] = stop.value
    while pending:
        served = {}
        steps = [i for i, r in pending.items() if isinstance(r, StepRequest)]
        if steps:
            served.update(zip(steps, serve_steps([pending[i] for i in steps], device)))
        flux = [i for i, r in pending.items() if not isinstance(r, StepRequest)]
        if flux:
            served.update(zip(flux, serve_flux([pending[i] for i in flux], device)))
        nxt = {}
        for i, res in served.items():
            try:
                if isinstance(res, TrajectoryError):
                    nxt[i] = gens[i].throw(res)
                else:
                    nxt[i] = gens[i].send(res)
            except StopIteration as stop:
                values[i] = stop.value
            except Exception as exc:
                # collect_errors: any failure of one trajectory's host logic
                # ends that trajectory only
                if not (collect_errors or isinstance(exc, TrajectoryError)):
                    raise
                values[i] = exc
                failed.append(exc)
        pending = nxt
    if failed and not collect_errors:
        raise failed[0]
    return values


# ------------------------------------------------------------------- driver
class AdaptiveHops:
    """Adaptive basis state of one trajectory.

    ``traj`` supplies the parameter dictionaries, the system and the noise
    (a HopsTrajectory after make_adaptive)."""

    def __init__(self, traj):
        self.traj = traj
        self.system = traj.system
        ep = traj.eom_param
        self.adaptive_h = bool(ep["ADAPTIVE_H"])
        self.adaptive_s = bool(ep["ADAPTIVE_S"])
        self.delta_a = float(ep["DELTA_A"])
        self.delta_s = float(ep["DELTA_S"])
        self.update_step = ep["UPDATE_STEP"] or 1
        self.f_discard = float(ep["F_DISCARD"])
        self.maxhier = traj.hierarchy_param["MAXHIER"]
        self.filters = list(traj.hierarchy_param["STATIC_FILTERS"])
        self.only_markovian = all(f[0] == "Markovian" for f in self.filters)
        ip = traj.integration_param
        self.early_steps = ip["EARLY_INTEGRATOR_STEPS"]
        self.inchworm_cap = ip["INCHWORM_CAP"]
        self.early = ip["EARLY_ADAPTIVE_INTEGRATOR"]
        if self.early not in ("INCH_WORM", "STATIC", "STATIC_STATE_INCHWORM_HIERARCHY"):
            raise UnsupportedRequest(self.early, "early time integrator clause of the propagate")
        self.static_states, self.static_counts = self._static_basis(ip["STATIC_BASIS"])
        if self.early == "STATIC_STATE_INCHWORM_HIERARCHY" and self.static_states is None:
            raise UnsupportedRequest("STATIC_STATE_INCHWORM_HIERARCHY without a STATIC_BASIS",
                                     "mesohops_b200 adaptive propagation")
        self.eom = ep["EQUATION_OF_MOTION"]
        if self.eom == "LINEAR":
            raise UnsupportedRequest("LINEAR equation of motion with an adaptive basis",
                                     "HopsTrajectory")
        for j in range(self.system.n_lop):
            if not self.system.lop_is_diagonal(j):
                raise UnsupportedRequest("adaptive basis with off-diagonal L-operator couplings",
                                         "mesohops_b200 adaptive propagation")
        n1, n2 = traj.noise1, traj.noise2
        if n1.interpolate or n2.interpolate:
            raise UnsupportedRequest("INTERPOLATE noise with an adaptive basis",
                                     "mesohops_b200 adaptive propagation")
        if (n2.param["MODEL"] != "ZERO"
                and abs(n2.param["TAU"] - n1.param["TAU"]) >= precision):
            raise UnsupportedRequest("noise 2 on a different time axis with an adaptive basis",
                                     "mesohops_b200 adaptive propagation")
        self.keyer = AuxKeyer(self.system.n_mode, self.maxhier)
        self.device = torch.device(traj.device_param["DEVICE"])
        self.precision = traj.device_param["PRECISION"]
        self.kernel_request = traj.device_param.get("KERNEL", "auto")
        self.prec_bytes = 16 if self.precision in ("complex128", "c128", "mixed") else 8
        Hd = self.system.hamiltonian_dense()
        Hoff = Hd - np.diag(np.diag(Hd))
        # column norms of the off-diagonal H (error_sflux_stable_state); the
        # couplings to states outside a basis come from the basis's own block
        self.h_col_norm2 = np.sum(np.abs(Hoff) ** 2, axis=0)
        del Hd, Hoff
        self.W = self.system.W
        self.G = self.system.G
        self.early_counter = 0
        self.basis = None
        self._engine = None
        self.kernel = None
        self.phi = None
        self.zmem_abs = None
        self.noise1_dev = self.noise2_dev = None
        self.noise1_host = self.noise2_host = None
        self.t = 0.0

    def _static_basis(self, sb):
        """integration_param STATIC_BASIS = [states, aux list] (hops_trajectory.py
        :293-316): absolute states, and aux given as count vectors over all modes,
        as (mode, depth) pairs, or as objects with ``todense()`` (the
        reference's AuxiliaryVector).  Returns (states, count rows) or (None, None)."""
        if sb is None:
            return None, None
        if len(sb) != 2:
            raise UnsupportedRequest("STATIC_BASIS must be [state list, aux list]",
                                     "mesohops_b200 adaptive propagation")
        M = self.system.n_mode
        states = np.array(sorted(set(int(x) for x in sb[0])), dtype=np.int64)
        rows = []
        for a in sb[1]:
            if hasattr(a, "todense"):
                v = np.asarray(a.todense(), dtype=np.int64).ravel()
            else:
                arr = np.asarray(a, dtype=np.int64)
                if arr.ndim == 2 or (arr.ndim == 1 and arr.size == 0):
                    v = np.zeros(M, dtype=np.int64)
                    for m, k in arr.reshape(-1, 2):
                        v[m] = k
                else:
                    v = arr.ravel()
            if v.size != M or np.any(v < 0) or v.sum() > self.maxhier:
                raise UnsupportedRequest("STATIC_BASIS aux outside the hierarchy",
                                         "mesohops_b200 adaptive propagation")
            rows.append(v)
        counts = np.array(rows, dtype=np.int16).reshape(-1, M)
        return states, counts

    def _union_counts(self, a, b):
        """Rows of a followed by the rows of b not in a."""
        allc = np.concatenate([a, b], axis=0)
        keys = self.keyer.sort_keys(allc)
        _, first = np.unique(keys, return_index=True)
        return allc[np.sort(first)]

    # ------------------------------------------------------------ basis setup
    def _set_basis(self, states, counts):
        self.basis = Basis(self.system, self.keyer, self.maxhier, counts, states, self.device,
                           (self.noise1_host, self.noise2_host))
        b = self.basis
        n_elem = b.n_hier * b.n_state
        req = self.kernel_request
        if req in ("resident", "streaming"):
            self.kernel = req
        else:
            self.kernel = ("resident" if 4 * n_elem * self.prec_bytes <= RESIDENT_MAX_BYTES
                           else "streaming")
        self._engine = None

    @property
    def engine(self):
        """Device buffers of the current basis (created on first use)."""
        if self._engine is None:
            b = self.basis
            n1 = b.dstruct.extra.get("noise1")
            n2 = b.dstruct.extra.get("noise2")
            if self.kernel == "resident":
                self._engine = ResidentTrajectory(b.dstruct, self.precision, self.eom)
                self._engine.set_noise(n1, n2)
            else:
                self._engine = StreamBatch(b.dstruct, 1, self.precision, self.eom)
                self._engine.set_noise(n1.unsqueeze(0) if n1 is not None else None,
                                       n2.unsqueeze(0) if n2 is not None else None)
        return self._engine

    def bind_noise(self, req):
        """Bind the noise rows a step request reads to the current engine and
        return its (first noise index, index step): the samples, or for an
        effective-noise request the window means on the half-step grid (the
        slots of the step at t are windows 2t/tau, +1, +2)."""
        eng = self.engine
        b = self.basis
        if not req.effective:
            rows = (b.dstruct.extra.get("noise1"), b.dstruct.extra.get("noise2"))
            it0, di = self.noise_index(req.t), self.noise_di(req.tau)
        else:
            key = ("eff", req.tau)
            if getattr(b, "_eff_key", None) != key:
                e1, e2 = self._effective_host(req.tau)
                l_abs = b.tables["l_abs"]
                dev = self.device
                b._eff_rows = tuple(
                    (torch.from_numpy(np.ascontiguousarray(e[l_abs])).to(dev)
                     if e is not None and b.tables["n_lop"] else None) for e in (e1, e2))
                b._eff_key = key
            rows = b._eff_rows
            half = req.tau * 0.5
            it0 = int(round(req.t / half))
            if abs(it0 * half - req.t) >= precision:
                raise UnsupportedRequest("EFFECTIVE_NOISE_INTEGRATION with a step start off "
                                         "the half-step grid", "mesohops_b200 adaptive")
            di = 1
        if isinstance(eng, StreamBatch):
            eng.set_noise(rows[0].unsqueeze(0) if rows[0] is not None else None,
                          rows[1].unsqueeze(0) if rows[1] is not None else None)
        else:
            eng.set_noise(rows[0], rows[1])
        return it0, di

    def apply_operator(self, op):
        """_operator (hops_trajectory.py:540-577) on the adaptive basis: with state
        adaptivity the states op reaches from the basis join it first (phi
        permuted and rescaled as in update_basis), op acts on the state index of
        every aux, and the early-time integrator restarts so that the next steps
        update the basis by inch-worm again."""
        import scipy.sparse as sps
        b = self.basis
        if self.adaptive_s:
            if sps.issparse(op):
                reach = np.unique(sps.csr_matrix(op)[:, b.states].nonzero()[0])
            else:
                reach = np.nonzero(np.asarray(op)[:, b.states])[0]
            states_u = np.array(sorted(set(b.states.tolist()) | set(int(x) for x in reach)),
                                dtype=np.int64)
            self.phi = self.update_basis(self.phi, states_u, b.counts)
            b = self.basis
        sl = b.states
        if sps.issparse(op):
            sub = sps.csr_matrix(op)[sl, :][:, sl]
        else:
            sub = np.asarray(op)[np.ix_(sl, sl)]
        phi_mat = self.phi.reshape(b.n_hier, b.n_state).T
        self.phi = np.asarray(sub @ phi_mat).T.reshape(-1).astype(np.complex128)
        if self.adaptive_s:
            self.early_counter = 0

    def _effective_host(self, tau):
        """Window means of every noise row for steps of tau (host copies, cached)."""
        if getattr(self, "_eff_tau", None) != tau:
            from .noise import window_means
            k = int(round(tau * 0.5 / self.traj.noise1.param["TAU"]))
            out = []
            for nd in (self.noise1_dev, self.noise2_dev):
                if nd is None:
                    out.append(None)
                    continue
                n_out = nd.shape[-1] // k
                out.append(window_means(nd, 0, k, n_out,
                                        bool(self.traj.noise1.param["FLAG_REAL"])
                                        if nd is self.noise1_dev else
                                        bool(self.traj.noise2.param["FLAG_REAL"])).cpu().numpy())
            self._eff_host_rows = tuple(out)
            self._eff_tau = tau
        return self._eff_host_rows

    def noise_index(self, t):
        return self.traj.noise1.time_index(t)

    def noise_di(self, tau):
        return int(round(tau * 0.5 / self.traj.noise1.param["TAU"]))

    def initialize_gen(self, psi0, noise1_dev, noise2_dev):
        """hops_trajectory.py:282-326 for an adaptive basis (coroutine)."""
        self.noise1_dev, self.noise2_dev = noise1_dev, noise2_dev
        # host copies of the noise rows: each basis packs its rows with its tables
        self.noise1_host = noise1_dev.cpu().numpy() if noise1_dev is not None else None
        self.noise2_host = noise2_dev.cpu().numpy() if noise2_dev is not None else None
        sysm = self.system
        if self.adaptive_h:
            counts = np.zeros((1, sysm.n_mode), dtype=np.int16)
        else:
            counts = triangular_counts(sysm.n_mode, self.maxhier)
            if self.filters:
                counts = apply_static_filters(counts, self.filters, sysm.n_mode)
        states = (np.nonzero(np.abs(psi0) > 0)[0] if self.adaptive_s
                  else np.arange(sysm.n_state))
        self.zmem_abs = np.zeros(sysm.n_mode, dtype=np.complex128)
        self._set_basis(states, counts)
        phi = np.zeros(self.basis.n_hier * self.basis.n_state, dtype=np.complex128)
        phi[:self.basis.n_state] = psi0[self.basis.states]
        self.t = 0.0
        if self.static_states is None:
            z_step = self._z_step(0.0, self.zmem_abs)
            states_u, counts_u = yield from self.define_basis_gen(phi, 1.0, z_step)
        else:
            # the initial basis joined with the static one instead of a first
            # basis update
            states_u = np.array(sorted(set(self.basis.states.tolist())
                                       | set(self.static_states.tolist())), dtype=np.int64)
            counts_u = self._union_counts(self.basis.counts, self.static_counts)
        self.phi = self.update_basis(phi, states_u, counts_u)

    # ------------------------------------------------------------------ noise
    def _z_step(self, t, zmem_abs):
        """[noise1(t), noise2(t), z_mem] over the basis L list (_prepare_zstep)."""
        l_abs = self.basis.tables["l_abs"]
        z1 = self.traj.noise1.get_noise([t], l_abs)[:, 0]
        z2 = self.traj.noise2.get_noise([t], l_abs)[:, 0]
        return z1, z2, zmem_abs.copy()

    # ---------------------------------------------------------------- filters
    def _static_up_filter(self):
        """markov_up * triangular_up * longedge_up (hops_fluxfilters.py:304-505),
        each filter type its own array, combined by logical and."""
        b = self.basis
        M, N = b.n_mode, b.n_hier
        F = np.ones((M, N), dtype=bool)
        if M == 0:
            return F
        cnt = b.counts
        mark = [np.asarray(p, dtype=bool)[b.modes] for (n, p) in self.filters if n == "Markovian"]
        if mark:
            Fm = np.ones((M, N), dtype=bool)
            mask = np.any(mark, axis=0)
            Fm[mask, 1:] = False
            for i in np.nonzero(mask)[0]:
                e = np.zeros((1, self.system.n_mode), dtype=np.int16)
                e[0, b.modes[i]] = 1
                idx = int(b.aux.index_of(e)[0])
                if idx >= 0:
                    Fm[:, idx] = False
            F &= Fm
        tri = [(np.asarray(p[0], dtype=bool)[b.modes], p[1]) for (n, p) in self.filters
               if n == "Triangular"]
        if tri:
            Ft = np.ones((M, N), dtype=bool)
            for mask, kmax2 in tri:
                tot = cnt[:, b.modes[mask]].sum(axis=1)
                Ft[np.ix_(mask, tot >= kmax2)] = False
            F &= Ft
        le = [(np.asarray(p[0], dtype=bool)[b.modes], p[1]) for (n, p) in self.filters
              if n == "LongEdge"]
        if le:
            Fl = np.ones((M, N), dtype=bool)
            for mask, kmax2 in le:
                filt_modes = set(b.modes[mask].tolist())
                for a in np.nonzero(b.depth >= kmax2)[0]:
                    keys = np.nonzero(cnt[a])[0]
                    if any(int(k) in filt_modes for k in keys):
                        Fl[:, a] = False
                        if len(keys) == 1:
                            Fl[b.rel_mode[int(keys[0])], a] = True
                    else:
                        Fl[mask, a] = False
            F &= Fl
        return F

    def _exists_up(self):
        """[M, N]: aux a + e_m is in the basis."""
        b = self.basis
        E = np.zeros((b.n_mode, b.n_hier), dtype=bool)
        E[b.aux.up_m, b.aux.up_a] = True
        return E

    def _exists_down(self):
        """[M, N]: aux a - e_m is in the basis."""
        b = self.basis
        E = np.zeros((b.n_mode, b.n_hier), dtype=bool)
        E[b.aux.dn_m, b.aux.dn_a] = True
        return E

    # -------------------------------------------------------------- hierarchy
    def _sflux_hier(self, phi_sn):
        """error_sflux_hier (basis_functions_adaptive.py:76-163), no LTC."""
        b = self.basis
        if len(b.list_sc) == 0:
            return np.zeros(b.n_hier)
        D = (b.h_sc @ phi_sn) / hbar
        return np.sum(np.abs(D) ** 2, axis=0)

    def _hierarchy_gen(self, phi, dt, z_step):
        """_define_hierarchy_basis + hier_stable_error (hops_basis.py:484-665)."""
        b = self.basis
        N, S, M = b.n_hier, b.n_state, b.n_mode
        phi_sn = phi.reshape(N, S).T
        e_deriv, e_up, e_down = yield FluxRequest(self, phi, z_step, dt)
        E1 = e_deriv.sum(axis=1)
        E1 = E1 + self._sflux_hier(phi_sn)
        F_static = self._static_up_filter()
        stable_up = np.ones((M, N), dtype=bool)
        stable_up[:, b.depth == self.maxhier] = False
        E1 = E1 + np.sum((stable_up & F_static) * e_up, axis=0)
        stable_down = b.k_aux > 0
        E1 = E1 + np.sum(stable_down * e_down, axis=0)
        d2 = self.delta_a ** 2
        idx_stable = keep_from_list(E1, d2 / 2.0)
        unstable = np.setdiff1d(np.arange(N), idx_stable)
        bound_sq = d2 - np.sum(E1[unstable])
        new_aux = self._boundary_hier(e_up, e_down, idx_stable, bound_sq, F_static)
        new_aux = np.array(new_aux, dtype=np.int16).reshape(-1, self.system.n_mode)
        if len(new_aux) and not self.only_markovian:
            new_aux = apply_static_filters(new_aux, self.filters, self.system.n_mode)
        return idx_stable, new_aux

    def _boundary_hier(self, e_up, e_down, idx_stable, bound_sq, F_static):
        """_determine_boundary_hier (hops_basis.py:667-793) with the boundary
        filters of hops_fluxfilters.py:113-216."""
        b = self.basis
        f_up = ~self._exists_up()
        f_up[:, b.depth == self.maxhier] = False
        f_up &= F_static
        f_dn = (b.k_aux > 0) & ~self._exists_down()
        Eu = (e_up * f_up)[:, idx_stable]
        Ed = (e_down * f_dn)[:, idx_stable]
        sorted_err = np.sort(np.append(Eu[Eu != 0], Ed[Ed != 0]))
        thresh = error_thresh(sorted_err, bound_sq * self.f_discard * self.f_discard)
        discarded = np.sum(Eu[Eu <= thresh]) + np.sum(Ed[Ed <= thresh])
        Eu = np.where(Eu <= thresh, 0.0, Eu)
        Ed = np.where(Ed <= thresh, 0.0, Ed)
        # candidate aux with their error terms, in the order of a loop over the
        # stable aux (flux up along each mode, then flux down along each of its
        # modes); the terms of one candidate are summed in that order
        iu, mu = np.nonzero(Eu.T)
        idn, md = np.nonzero(Ed.T)
        # candidate i: the stable aux par[i] with mode mod[i] added (sgn +1) or
        # removed (sgn -1); keyed from its sorted mode tuple
        par = np.concatenate([idx_stable[iu], idx_stable[idn]])
        mod = np.concatenate([b.modes[mu], b.modes[md]]).astype(np.int64)
        sgn = np.concatenate([np.ones(len(iu), np.int64), -np.ones(len(idn), np.int64)])
        vals = np.concatenate([Eu[mu, iu], Ed[md, idn]])
        order = np.argsort(np.concatenate([2 * iu, 2 * idn + 1]), kind="stable")
        par, mod, sgn, vals = par[order], mod[order], sgn[order], vals[order]
        if len(vals) == 0:
            return []
        tup = b.aux.tup[par]
        up = sgn > 0
        tup[up] = insert_mode(tup[up], mod[up])
        tup[~up] = remove_mode(tup[~up], mod[~up])
        keys = self.keyer.keys_from_tuples(tup, b.depth[par] + sgn)
        _, first, inv = np.unique(keys, return_index=True, return_inverse=True)
        sums = np.zeros(len(first))
        np.add.at(sums, inv.ravel(), vals)
        seq = np.argsort(first)                     # first-occurrence order
        sums, pick = sums[seq], first[seq]
        thresh = error_thresh(np.sort(sums), bound_sq, offset=discarded)
        pick = pick[sums > thresh]
        rows = b.counts[par[pick]].copy()
        rows[np.arange(len(pick)), mod[pick]] += sgn[pick].astype(rows.dtype)
        return list(rows)

    # ----------------------------------------------------------------- states
    def _state_gen(self, phi, dt, z_step, idx_stable_aux, bound_aux):
        """_define_state_basis + state_stable_error (hops_basis.py:294-482, 795-912)."""
        b = self.basis
        N, S, M = b.n_hier, b.n_state, b.n_mode
        phi_sn = phi.reshape(N, S).T
        mask = np.zeros(N, dtype=np.int32)
        mask[idx_stable_aux] = 1
        e_deriv, _, _ = yield FluxRequest(self, phi, z_step, dt, mask=mask, with_flux=False)
        E1 = e_deriv[idx_stable_aux].sum(axis=0)
        # error_sflux_stable_state (basis_functions_adaptive.py:893-995)
        C1 = np.sum(np.abs(phi_sn[:, idx_stable_aux]) ** 2, axis=1)
        E1 = E1 + self.h_col_norm2[b.states] * C1 / hbar ** 2
        # construct_filter_state_stable_down / _up (hops_fluxfilters.py:218-302)
        F_down = np.zeros((M, N), dtype=bool)
        F_up = np.zeros((M, N), dtype=bool)
        V = np.asarray(bound_aux, dtype=np.int16).reshape(-1, self.system.n_mode)
        if len(V) and M:
            TV, dV = tuples_of(V, self.maxhier)
            # aux one step up from each boundary aux along every basis mode
            low = np.nonzero(dV < self.maxhier)[0]
            if len(low):
                ups = insert_mode(np.repeat(TV[low], M, axis=0), np.tile(b.modes, len(low)))
                keys = self.keyer.keys_from_tuples(ups, np.repeat(dV[low] + 1, M))
                idx = b.aux.index_of_keys(keys).reshape(len(low), M)
                vi, mi = np.nonzero(idx >= 0)
                F_down[mi, idx[vi, mi]] = True
            # aux one step down from each boundary aux along its own modes
            vi, mabs = np.nonzero(V)
            downs = remove_mode(TV[vi], mabs)
            idx = b.aux.index_of_keys(self.keyer.keys_from_tuples(downs, dV[vi] - 1))
            ok = idx >= 0
            rel = np.array([b.rel_mode[int(m)] for m in mabs[ok]], dtype=np.int64)
            F_up[rel, idx[ok]] = True
        absphi2 = np.abs(phi_sn) ** 2
        if M:
            avg = self._avg_L(phi[:S])
            X2 = np.repeat(avg[b.tables["mode_lop"]][:, None], S, axis=1)
            D2 = np.abs(b.m2 - X2) ** 2
            gw2 = np.abs(self.G[b.modes] / self.W[b.modes]) ** 2
            # error_flux_down_state_stable (:626-758)
            E_down = (D2.T @ (F_down * gw2[:, None])) * absphi2 / hbar ** 2
            KW = np.abs(self.W[b.modes])[:, None] * (1 + b.k_aux.astype(np.float64))
            # error_flux_up_state_stable (:268-384)
            E_up = ((np.abs(b.m2) ** 2).T @ (np.abs(F_up * KW) ** 2)) * absphi2 / hbar ** 2
            E1 = E1 + E_down[:, idx_stable_aux].sum(axis=1) + E_up[:, idx_stable_aux].sum(axis=1)
        d2 = self.delta_s ** 2
        rel_stable = keep_from_list(E1, d2 / 2.0)
        stable_states = b.states[rel_stable]
        unstable = np.setdiff1d(np.arange(S), rel_stable)
        bound_sq = d2 - np.sum(E1[unstable])
        # error_sflux_boundary_state (:997-1132)
        bound_states = []
        if len(rel_stable) < self.system.n_state and len(b.list_sc):
            Hsc = b.h_sc[:, rel_stable]
            Cst = phi_sn[np.ix_(rel_stable, idx_stable_aux)]
            Esc = np.sum(np.abs(Hsc @ (Cst / hbar)) ** 2, axis=1)
            nz = np.nonzero(Esc)[0]
            if len(nz):
                keep = keep_from_list(Esc[nz], bound_sq)
                bound_states = b.list_sc[nz][keep].tolist()
        bound_states = sorted(set(bound_states) - set(b.states.tolist()))
        return stable_states, np.array(bound_states, dtype=np.int64)

    def _avg_L(self, psi):
        """<L_j> over the basis L list (HopsBasis.psi setter, eom_functions.py:11-29)."""
        n2 = np.vdot(psi, psi)
        return np.array([np.vdot(psi, l @ psi) / n2 for l in self.basis.lred])

    # ---------------------------------------------------------- define/update
    def define_basis_gen(self, phi, dt, z_step):
        """New (states, aux counts) for the next step (hops_basis.py:117-182)."""
        b = self.basis
        phin = phi / np.linalg.norm(phi[:b.n_state])
        if self.adaptive_h:
            idx_stable, bound_aux = yield from self._hierarchy_gen(phin, dt, z_step)
            counts_new = (np.concatenate([b.counts[idx_stable], bound_aux], axis=0)
                          if len(bound_aux) else b.counts[idx_stable])
        else:
            idx_stable = np.arange(b.n_hier)
            bound_aux = np.zeros((0, self.system.n_mode), dtype=np.int16)
            counts_new = b.counts
        if self.adaptive_s:
            st, bd = yield from self._state_gen(phin, dt, z_step, idx_stable, bound_aux)
            states_new = np.array(sorted(set(st.tolist()) | set(bd.tolist())), dtype=np.int64)
        else:
            states_new = b.states
        return states_new, counts_new

    def update_basis(self, phi, states_new, counts_new):
        """Permute phi into the new basis keeping ||psi|| (hops_basis.py:184-292)."""
        b = self.basis
        if b.same_as(states_new, counts_new):
            return phi
        old_states, old_keys = b.states, b.aux.keys
        S_old, N_old = b.n_state, b.n_hier
        self._set_basis(states_new, counts_new)
        nb = self.basis
        stable_states = np.intersect1d(old_states, nb.states)
        old_s = np.searchsorted(old_states, stable_states)
        new_s = np.searchsorted(nb.states, stable_states)
        pos = np.minimum(np.searchsorted(old_keys, nb.aux.keys), N_old - 1)
        present = old_keys[pos] == nb.aux.keys
        phi_o = phi.reshape(N_old, S_old)
        phi_n = np.zeros((nb.n_hier, nb.n_state), dtype=np.complex128)
        na = np.nonzero(present)[0]
        phi_n[np.ix_(na, new_s)] = phi_o[np.ix_(pos[na], old_s)]
        norm_old = np.linalg.norm(phi[:S_old])
        phi_n = phi_n.ravel()
        return norm_old * phi_n / np.linalg.norm(phi_n[:nb.n_state])

    # --------------------------------------------------------------- stepping
    def decay_out_of_basis(self, zmem_abs, tau):
        """RK4 of dz = -conj(w) z for modes outside the basis whose z exceeds the
        precision at the stage (eom_functions.py:122-154); in-basis modes are
        overwritten by the device result."""
        z = zmem_abs.copy()
        out = np.ones(self.system.n_mode, dtype=bool)
        out[self.basis.modes] = False
        if not np.any(out):
            return z
        z0 = z[out]
        wc = np.conj(self.W[out])
        kz = []
        for i, c in enumerate((0.0, 0.5, 0.5, 1.0)):
            zi = z0 if i == 0 else z0 + c * kz[-1] * tau / hbar
            kz.append(np.where(gt_precision(zi), -wc * zi, 0.0))
        z[out] = z0 + tau / hbar * (kz[0] + 2.0 * kz[1] + 2.0 * kz[2] + kz[3]) / 6.0
        return z

    def finish_step(self, req, phi, zrel):
        """(phi, z_mem over all modes) after a step: the device result for the
        basis modes, the host decay for the others."""
        z = self.decay_out_of_basis(req.zmem_abs, req.tau)
        if self.basis.n_mode:
            z[self.basis.modes] = zrel
        return phi, z

    def _normalize(self, phi):
        """hops_trajectory.py:616-634"""
        if self.eom == "NORMALIZED NONLINEAR":
            return phi / np.sqrt(np.sum(np.abs(phi[:self.basis.n_state]) ** 2))
        return phi

    def step_gen(self, t, tau, index_t):
        """One pass of the propagate loop (hops_trajectory.py:456-533).

        Returns the z_mem the reference stores with this step (the one from
        before the step: hops_trajectory.py:523-526 stores self.z_mem before
        assigning the new value)."""
        # the propagate loop passes EFFECTIVE_NOISE_INTEGRATION to its steps; the
        # inch-worm re-steps below take the plain samples, as the reference does
        # (hops_trajectory.py:457-460 against :684)
        phi, z = yield StepRequest(self, self.phi, self.zmem_abs, self.t, tau,
                                   effective=self.traj.effective_noise_integration)
        phi = self._normalize(phi)
        if self.early_counter < self.early_steps:
            if self.early in ("INCH_WORM", "STATIC_STATE_INCHWORM_HIERARCHY"):
                # STATIC_STATE_INCHWORM_HIERARCHY: the state basis of the early
                # steps is the static one, the hierarchy inch-worms
                # (hops_trajectory.py:477-491)
                fixed = self.early == "STATIC_STATE_INCHWORM_HIERARCHY"
                z_step = self._z_step(self.t, z)
                states_u, counts_u = yield from self.define_basis_gen(phi, tau, z_step)
                if fixed:
                    states_u = self.static_states
                n_iter = 0
                while not self.basis.same_as(states_u, counts_u):
                    states_u, counts_u, phi, z = yield from self._inchworm_gen(
                        states_u, counts_u, tau)
                    if fixed:
                        states_u = self.static_states
                    n_iter += 1
                    if n_iter >= self.inchworm_cap:
                        break
                phi = self.update_basis(phi, states_u, counts_u)
            self.early_counter += 1
        elif (index_t + 1) % self.update_step == 0:
            z_step = self._z_step(self.t, z)
            states_u, counts_u = yield from self.define_basis_gen(phi, tau, z_step)
            phi = self.update_basis(phi, states_u, counts_u)
        z_store = self.zmem_abs
        self.phi = phi
        self.zmem_abs = z
        self.t = t
        return z_store

    def _inchworm_gen(self, states_new, counts_new, tau):
        """inchworm_integrate (hops_trajectory.py:636-691): grow the basis by the
        proposal, redo the step from the state at the start of the step in the
        grown basis, and propose again."""
        b = self.basis
        states_u = np.array(sorted(set(np.asarray(states_new).tolist())
                                   | set(b.states.tolist())), dtype=np.int64)
        counts_new = np.asarray(counts_new, dtype=np.int16).reshape(-1, self.system.n_mode)
        allc = np.concatenate([b.counts, counts_new], axis=0)
        allk = self.keyer.sort_keys(allc)
        _, first = np.unique(allk, return_index=True)
        counts_u = allc[np.sort(first)]
        self.phi = self.update_basis(self.phi, states_u, counts_u)
        phi, z = yield StepRequest(self, self.phi, self.zmem_abs, self.t, tau)
        phi = self._normalize(phi)
        z_step = self._z_step(self.t, z)
        s2, c2 = yield from self.define_basis_gen(phi, tau, z_step)
        return s2, c2, phi, z

    # -------------------------------------------------------------- read-outs
    def psi_full(self):
        out = np.zeros(self.system.n_state, dtype=np.complex128)
        out[self.basis.states] = self.phi[:self.basis.n_state]
        return out
