"""Drop-in HopsTrajectory running the trajectory hot path on a B200.

Same constructor, parameter dictionaries, ``initialize(psi_0)``,
``propagate(t_advance, tau)`` and read-outs (``phi``, ``psi``, ``z_mem``,
``t``, ``storage``) as trajectory/hops_trajectory.py:84-538 of MesoHOPS.  The
loop body -- noise sampling at t, t+tau/2, t+tau (integrator_rk.py:78-134), the
RK4 step over the nonlinear HOPS equation (integrator_rk.py:10-75,
hops_eom.py:196-441) and the renormalisation (hops_trajectory.py:616-634) --
runs as CUDA kernels; the state stays on the device between calls.

Options of this implementation go in the separate ``device_param`` dictionary
(PRECISION, DEVICE, KERNEL); the reference dictionaries are validated exactly as
MesoHOPS validates them.  ``make_adaptive`` switches to the adaptive basis
(adHOPS): see mesohops_b200/adaptive.py.
"""
from __future__ import annotations

import time as timer

import numpy as np
import scipy.sparse as sps
import torch

from . import adaptive as _adaptive
from .constants import hbar, precision
from .device import hierarchy_structure
from .engine import ResidentRunner, ResidentTrajectory, StreamBatch
from .exceptions import LockedException, TrajectoryError, UnsupportedRequest
from .noise import HopsNoise
from .params import (DEVICE_DICT_DEFAULT, EOM_DICT_DEFAULT, EOM_DICT_TYPES, NOISE_DICT_DEFAULT,
                     HIERARCHY_DICT_DEFAULT, HIERARCHY_DICT_TYPES, INTEGRATION_DICT_DEFAULT,
                     INTEGRATION_DICT_TYPES, initialize_dict)
from .storage import HopsStorage
from .system import HopsSystem

# Resident (one CTA per trajectory) path when the four stage vectors fit the
# per-CTA shared memory budget; larger problems use the streaming kernels.
RESIDENT_MAX_BYTES = 200 * 1024


def choose_kernel(n_elem, prec_bytes, requested="auto"):
    if requested in ("resident", "streaming"):
        return requested
    return "resident" if 4 * n_elem * prec_bytes <= RESIDENT_MAX_BYTES else "streaming"


class HopsTrajectory:
    """One HOPS trajectory (drop-in for mesohops.trajectory.hops_trajectory)."""

    def __init__(self, system_param=None, eom_param=None, noise_param=None,
                 noise2_param=None, hierarchy_param=None, storage_param=None,
                 integration_param=None, device_param=None):
        system_param = {} if system_param is None else system_param
        self.eom_param = initialize_dict(eom_param or {}, EOM_DICT_DEFAULT, EOM_DICT_TYPES,
                                         "HopsEOM")
        eom = self.eom_param["EQUATION_OF_MOTION"]
        if eom not in ("NORMALIZED NONLINEAR", "NONLINEAR", "LINEAR"):
            raise UnsupportedRequest("EQUATION_OF_MOTION =" + eom, "HopsEOM")
        self.eom_param["ADAPTIVE"] = bool(self.eom_param["ADAPTIVE_H"]
                                          or self.eom_param["ADAPTIVE_S"])
        self.system = HopsSystem(system_param)
        self.hierarchy_param = initialize_dict(hierarchy_param or {}, HIERARCHY_DICT_DEFAULT,
                                               HIERARCHY_DICT_TYPES, "HopsHierarchy")
        if self.hierarchy_param["MAXHIER"] > 255:
            self.hierarchy_param["MAXHIER"] = 255
        if self.hierarchy_param["TERMINATOR"]:
            raise UnsupportedRequest("TERMINATOR", "HopsHierarchy")
        noise_param = {} if noise_param is None else noise_param
        if noise2_param is None:
            noise2_param = {"TLEN": noise_param.get("TLEN", 1000.0),
                            "TAU": noise_param.get("TAU", 1.0), "MODEL": "ZERO", "SEED": None}
        self.noise_param = noise_param
        self.noise2_param = noise2_param
        self.noise1 = HopsNoise(noise_param, self.system, noise_type=1)
        self.noise2 = HopsNoise(noise2_param, self.system, noise_type=2)
        if integration_param is None:
            integration_param = INTEGRATION_DICT_DEFAULT
        self.integration_param = initialize_dict(integration_param, INTEGRATION_DICT_DEFAULT,
                                                 INTEGRATION_DICT_TYPES,
                                                 "integration_param in the HopsTrajectory "
                                                 "initialization")
        if self.integration_param["INTEGRATOR"] != "RUNGE_KUTTA":
            raise UnsupportedRequest("Integrator of type " + str(self.integration_param["INTEGRATOR"]),
                                     type(self).__name__)
        self.integrator_step = 0.5
        self.device_param = dict(DEVICE_DICT_DEFAULT)
        self.device_param.update(device_param or {})
        self._storage_param = storage_param
        self.storage = HopsStorage(self.eom_param["ADAPTIVE"], storage_param)
        self.__initialized__ = False
        self._t = 0.0
        self._runner = None
        self._adhops = None

    # ------------------------------------------------------------------ setup
    def initialize(self, psi_0, timer_checkpoint=None):
        """Build the hierarchy, upload the structure, set phi_0 = [psi_0, 0, ...]."""
        t0 = timer.time() if timer_checkpoint is None else timer_checkpoint
        if self.__initialized__:
            raise LockedException("HopsTrajectory.initialize()", "HopsTrajectory")
        psi_0 = np.array(psi_0, dtype=np.complex128)
        dev = torch.device(self.device_param["DEVICE"])
        if self.eom_param["ADAPTIVE"]:
            self._initialize_adaptive(psi_0, dev)
            self.storage.metadata["INITIALIZATION_TIME"] = timer.time() - t0
            self.__initialized__ = True
            return
        self.basis, self.dstruct = hierarchy_structure(self.system, self.hierarchy_param, dev)
        prec = self.device_param["PRECISION"]
        prec_bytes = 16 if prec in ("complex128", "c128", "mixed") else 8
        n_elem = self.dstruct.n_elem
        self.kernel = choose_kernel(n_elem, prec_bytes, self.device_param["KERNEL"])
        eom = self.eom_param["EQUATION_OF_MOTION"]
        if self.kernel == "resident":
            self._traj = ResidentTrajectory(self.dstruct, prec, eom)
            self._runner = ResidentRunner(dev)
        else:
            self._traj = StreamBatch(self.dstruct, 1, prec, eom)
        phi0 = np.zeros(n_elem, dtype=np.complex128)
        phi0[:self.n_state] = psi_0[self.state_list]
        self._set_state(phi0, np.zeros(self.system.n_mode, dtype=np.complex128))
        n1 = self.noise1.prepare(dev)
        n2 = self.noise2.prepare(dev)
        self._bind_noise(n1, n2)
        self._t = 0.0
        self.storage.store(0.0, psi=phi0[:self.n_state].copy(), phi=phi0.copy(),
                           z_mem=np.zeros(self.system.n_mode, dtype=np.complex128))
        self.storage.metadata["INITIALIZATION_TIME"] = timer.time() - t0
        self.__initialized__ = True

    def _bind_noise(self, n1, n2, keep=True):
        """Noise rows the kernels read; keep=False binds a temporary view (the
        effective-noise windows of one propagate call) without replacing the
        trajectory's own noise."""
        if keep:
            self._n1, self._n2 = n1, n2
        if self.kernel == "resident":
            self._traj.set_noise(n1, n2)
        else:
            self._traj.set_noise(n1.unsqueeze(0) if n1 is not None else None,
                                 n2.unsqueeze(0) if n2 is not None else None)

    def _set_state(self, phi, zmem):
        if self.kernel == "resident":
            self._traj.set_state(phi, zmem)
        else:
            self._traj.set_state(phi.reshape(1, -1), zmem.reshape(1, -1))

    def make_adaptive(self, delta_a=1e-4, delta_s=1e-4, update_step=1, f_discard=0.01,
                      adaptive_noise=True):
        """Switch to an adaptive basis before initialize (hops_trajectory.py:338-400).

        adaptive_noise is accepted for interface parity: the correlated noise of
        every L-operator is generated on the device at once, and each row equals
        the row an adaptive (per-L, on demand) generation produces."""
        if float(f_discard) < 0 or float(f_discard) > 1:
            raise UnsupportedRequest("f_discard not in acceptable range of [0,1]",
                                     "make_adaptive")
        if self.__initialized__:
            raise TrajectoryError("Adaptive calculation cannot be turned on after "
                                  "the trajectory is initialized")
        ep = self.eom_param
        if delta_a > 0:
            ep["ADAPTIVE"] = True
            ep["ADAPTIVE_H"] = True
            ep["DELTA_A"] = delta_a
            ep["UPDATE_STEP"] = update_step
            ep["F_DISCARD"] = float(f_discard)
        if delta_s > 0:
            ep["ADAPTIVE"] = True
            ep["ADAPTIVE_S"] = True
            ep["DELTA_S"] = delta_s
            ep["UPDATE_STEP"] = update_step
            ep["F_DISCARD"] = float(f_discard)
        if ep["ADAPTIVE"] and not self.storage.adaptive:
            self.storage = HopsStorage(True, self._storage_param)

    def _initialize_adaptive(self, psi_0, dev):
        """hops_trajectory.py:282-326 with the adaptive basis on the device."""
        self._adhops = _adaptive.AdaptiveHops(self)
        n1 = self.noise1.prepare(dev)
        n2 = self.noise2.prepare(dev)
        self._n1, self._n2 = n1, n2
        _adaptive.drive(self._adhops.initialize_gen(psi_0, n1, n2), dev)
        self.kernel = "adaptive"
        self.storage.n_dim = self.system.n_state
        self._t = 0.0
        self._store_adaptive(0.0, np.zeros(self.system.n_mode, dtype=np.complex128))

    def adaptive_step_gen(self, t, tau, index_t):
        """One adaptive step as a coroutine of device requests (see
        mesohops_b200.adaptive), with the storage of hops_trajectory.py:523-526."""
        z_old = yield from self._adhops.step_gen(t, tau, index_t)
        if self.storage.check_storage_time(t):
            self._store_adaptive(t, z_old)
        self._t = float(t)

    def _store_adaptive(self, t, z_mem):
        ad = self._adhops
        b = ad.basis
        aux_list = [np.array([(int(m), int(c[m])) for m in np.nonzero(c)[0]],
                             dtype=int).reshape(-1, 2) for c in b.counts]
        self.storage.store(float(t), psi=ad.phi[:b.n_state].copy(), phi=ad.phi.copy(),
                           z_mem=z_mem.copy(), aux_list=aux_list,
                           state_list=b.states.copy())

    # -------------------------------------------------------------- propagate
    def _check_tau_step(self, tau):
        """hops_trajectory.py:579-614"""
        ok = True
        for nz in (self.noise1, self.noise2):
            ts = tau * self.integrator_step / nz.param["TAU"]
            ok &= (ts - int(round(ts))) < precision
            ok &= int(round(tau / nz.param["TAU"])) >= 1
        return ok

    def propagate(self, t_advance, tau, timer_checkpoint=None):
        t_start = timer.time() if timer_checkpoint is None else timer_checkpoint
        if not self.__initialized__:
            raise TrajectoryError("propagate called before initialize")
        t0 = self.t
        if not self._check_tau_step(tau):
            raise TrajectoryError(f"Timesteps({tau * self.integrator_step}) that do not match "
                                  f"noise.param['TAU'] ({self.noise1.param['TAU']})")
        if (t0 + t_advance + tau) > self.noise1.param["TLEN"]:
            raise TrajectoryError("Trajectory times longer than noise.param['TLEN'] ="
                                  + str(self.noise1.param["TLEN"]))
        n_steps = int(np.ceil(t_advance / tau))
        t_axis = t0 + np.arange(1, 1 + n_steps) * tau
        if n_steps == 0:
            return
        if self._adhops is not None:
            dev = torch.device(self.device_param["DEVICE"])
            for index_t, t in enumerate(t_axis):
                _adaptive.drive(self.adaptive_step_gen(float(t), tau, index_t), dev)
            self.storage.metadata["LIST_PROPAGATION_TIME"].append(timer.time() - t_start)
            return
        if self.effective_noise_integration:
            # window means of the noise (integrator_rk.py:115-128) on a half-step grid
            # that starts at t0: slots of step n are windows 2n, 2n+1, 2n+2
            self._bind_noise(self.noise1.effective(t0, tau, n_steps),
                             self.noise2.effective(t0, tau, n_steps), keep=False)
            it0, di = 0, 1
        else:
            it0 = self.noise1.time_index(t0)
            di = int(round(tau * 0.5 / self.noise1.param["TAU"]))
            self._align_noise2(it0, di, n_steps)
        h = tau / hbar
        dev = self.dstruct.device
        psi_dev = torch.empty((n_steps, self.n_state), dtype=torch.complex128, device=dev)
        try:
            if self.kernel == "resident":
                st = self._runner.run([self._traj], it0, di, n_steps, h, psi_out=[psi_dev])
                if st[0] != 0:
                    raise TrajectoryError("non-finite state during propagation")
            else:
                self._traj.propagate(it0, di, n_steps, h,
                                     psi_out=psi_dev.view(n_steps, 1, self.n_state))
                self._traj.check_status()
        finally:
            if self.effective_noise_integration:
                self._bind_noise(self._n1, self._n2)
        psi = psi_dev.cpu().numpy()
        need_phi = "phi_traj" in self.storage.data or "z_mem" in self.storage.data
        phi_end = zmem_end = None
        if need_phi:
            phi_end, zmem_end = self._get_state()
        for k, t in enumerate(t_axis):
            if self.storage.check_storage_time(t):
                last = k == n_steps - 1
                self.storage.store(float(t), psi=psi[k].copy(),
                                   phi=phi_end if last else None,
                                   z_mem=zmem_end if last else None)
        self._t = float(t_axis[-1])
        self.storage.metadata["LIST_PROPAGATION_TIME"].append(timer.time() - t_start)

    def _align_noise2(self, it0, di, n_steps):
        """Noise 2 on a different time axis is resampled onto the noise-1 indices."""
        if self._n2 is None:
            return
        if abs(self.noise2.param["TAU"] - self.noise1.param["TAU"]) < precision:
            return
        need = it0 + 2 * n_steps * di + 1
        tau1 = self.noise1.param["TAU"]
        idx = [self.noise2.time_index(i * tau1) for i in range(need)]
        n2 = self._n2[:, idx].contiguous()
        self._bind_noise(self._n1, n2)

    # -------------------------------------------------------------- read-outs
    def _get_state(self):
        if self._adhops is not None:
            return self._adhops.phi.copy(), self._adhops.zmem_abs.copy()
        if self.kernel == "resident":
            return self._traj.get_state()
        phi, z = self._traj.get_state()
        return phi[0], z[0]

    def dsystem_dt(self, phi, z_mem, z_rnd1, z_rnd2):
        """dsystem_dt closure of hops_eom.py:196-441 evaluated on the GPU.

        Returns (dphi, dz_mem) in cm^-1 (not divided by hbar).  z_mem is indexed by
        mode; z_rnd1 / z_rnd2 by unique L.
        """
        zm = z_mem.toarray().ravel() if hasattr(z_mem, "toarray") else np.asarray(z_mem).ravel()
        if not hasattr(self, "_deriv_batch"):
            self._deriv_batch = StreamBatch(self.dstruct, 1, self.device_param["PRECISION"],
                                            self.eom_param["EQUATION_OF_MOTION"])
        b = self._deriv_batch
        b.set_state(np.asarray(phi).reshape(1, -1), zm.reshape(1, -1))
        dphi, dz = b.dsystem_dt(np.asarray(z_rnd1).reshape(1, -1),
                                np.asarray(z_rnd2).reshape(1, -1) if z_rnd2 is not None else None)
        return dphi[0], dz[0]

    @property
    def phi(self):
        return self._get_state()[0]

    @phi.setter
    def phi(self, phi):
        """Replace the hierarchy state in the current basis (z_mem kept)."""
        phi = np.asarray(phi, dtype=np.complex128).reshape(-1)
        if len(phi) != self.n_hier * self.n_state:
            raise UnsupportedRequest(f"phi of length {len(phi)} (expected "
                                     f"{self.n_hier * self.n_state})", "HopsTrajectory.phi")
        if self._adhops is not None:
            self._adhops.phi = phi.copy()
            return
        self._set_state(phi, self._get_state()[1])

    def _operator(self, op):
        """Act an operator on the state index of every aux of the hierarchy
        (hops_trajectory.py:540-577): phi[aux] <- op[state_list, state_list] phi[aux];
        a state-adaptive basis first takes in the states op reaches and restarts
        its early-time integrator."""
        if self._adhops is not None:
            self._adhops.apply_operator(op)
            return
        sl = np.asarray(self.state_list)
        if sps.issparse(op):
            op = sps.csr_matrix(op)[sl, :][:, sl]
        else:
            op = np.asarray(op)[np.ix_(sl, sl)]
        phi = self.phi
        phi_mat = phi.reshape(self.n_hier, self.n_state).T        # [state, aux]
        self.phi = np.asarray(op @ phi_mat).T.reshape(-1)

    @property
    def z_mem(self):
        return self._get_state()[1]

    @property
    def psi(self):
        return self.phi[:self.n_state]

    @property
    def t(self):
        return self._t

    @property
    def effective_noise_integration(self):
        return self.integration_param["EFFECTIVE_NOISE_INTEGRATION"]

    @property
    def n_hier(self):
        if self._adhops is not None:
            return self._adhops.basis.n_hier
        return self.basis.n_hier

    @property
    def n_state(self):
        if self._adhops is not None:
            return self._adhops.basis.n_state
        return self.system.n_state

    @property
    def state_list(self):
        if self._adhops is not None:
            return self._adhops.basis.states.copy()
        return np.arange(self.system.n_state)

    @property
    def auxiliary_list(self):
        """Aux vectors as dense count rows, in the reference order."""
        if self._adhops is not None:
            return self._adhops.basis.counts
        return self.basis.counts

    # ------------------------------------------------------------ checkpoints
    _SYSTEM_KEYS = ("HAMILTONIAN", "GW_SYSBATH", "L_HIER", "L_NOISE1", "ALPHA_NOISE1",
                    "PARAM_NOISE1", "L_NOISE2", "ALPHA_NOISE2", "PARAM_NOISE2", "L_LT_CORR",
                    "PARAM_LT_CORR")

    def save_checkpoint(self, filepath, compress=True, drop_seed=False):
        """Save parameters, state and storage to an .npz file with the keys of
        hops_trajectory.py:853-937 (phi, z_mem, t, state_list, aux_list,
        early_counter, storage_data, storage_meta, params); params also holds
        this implementation's device_param.  drop_seed leaves out the noise
        seeds (to be given again to load_checkpoint)."""
        if not self.__initialized__:
            raise TrajectoryError("save_checkpoint called before initialize")
        eom_param = {k: v for k, v in self.eom_param.items() if k != "ADAPTIVE"}
        for key in ("DELTA_A", "DELTA_S", "F_DISCARD"):
            if key in eom_param:
                eom_param[key] = float(eom_param[key])
        if eom_param.get("UPDATE_STEP") is None:
            eom_param.pop("UPDATE_STEP", None)

        def noise_dict(nz):
            return {k: nz.param[k] for k in NOISE_DICT_DEFAULT
                    if k in nz.param and not (k == "SEED" and drop_seed)}

        storage_param = dict(self.storage.storage_dic)
        storage_param["STORAGE_TIME"] = self.storage.storage_time
        params = {
            "system_param": {k: self.system.param[k] for k in self._SYSTEM_KEYS
                             if k in self.system.param},
            "hierarchy_param": {k: self.hierarchy_param[k] for k in HIERARCHY_DICT_DEFAULT},
            "eom_param": eom_param,
            "noise1_param": noise_dict(self.noise1),
            "noise2_param": noise_dict(self.noise2),
            "integration_param": dict(self.integration_param),
            "storage_param": storage_param,
            "device_param": dict(self.device_param),
        }
        phi, z_mem = self._get_state()
        counts = self.auxiliary_list
        aux_list = np.empty(len(counts), dtype=object)
        for i, c in enumerate(counts):
            nz = np.nonzero(c)[0]
            aux_list[i] = np.array([(int(m), int(c[m])) for m in nz], dtype=int).reshape(-1, 2)
        checkpoint = {
            "phi": phi, "z_mem": z_mem, "t": self.t,
            "state_list": np.array(self.state_list, dtype=int), "aux_list": aux_list,
            "early_counter": self._adhops.early_counter if self._adhops is not None else 0,
            "storage_data": self.storage.data, "storage_meta": self.storage.metadata,
            "params": params,
        }
        (np.savez_compressed if compress else np.savez)(filepath, **checkpoint)

    @classmethod
    def load_checkpoint(cls, filename, add_seed1=None, add_seed2=None, add_system_param=None,
                        device_param=None):
        """A trajectory restored from save_checkpoint (hops_trajectory.py:938-1034):
        same parameters, basis, state, noise memory, time and storage; the
        device_param stored with it unless another is given."""
        data = np.load(filename, allow_pickle=True)
        params = data["params"].item()
        if add_seed1 is not None:
            params["noise1_param"]["SEED"] = add_seed1
        if add_seed2 is not None:
            params["noise2_param"]["SEED"] = add_seed2
        if add_system_param is not None:
            params["system_param"] = add_system_param
        traj = cls(params["system_param"], eom_param=params["eom_param"],
                   noise_param=params["noise1_param"], noise2_param=params["noise2_param"],
                   hierarchy_param=params["hierarchy_param"],
                   storage_param=params["storage_param"],
                   integration_param=params["integration_param"],
                   device_param=device_param or params.get("device_param"))
        states = np.asarray(data["state_list"], dtype=np.int64)
        phi = np.asarray(data["phi"], dtype=np.complex128)
        z_mem = data["z_mem"]
        if z_mem.dtype == object:                      # a sparse matrix
            z_mem = z_mem.item()
            z_mem = np.asarray(z_mem.toarray() if hasattr(z_mem, "toarray") else z_mem)
        z_mem = np.asarray(z_mem, dtype=np.complex128).ravel()
        if len(z_mem) < traj.system.n_mode:
            z_mem = np.concatenate([z_mem, np.zeros(traj.system.n_mode - len(z_mem), complex)])
        psi_0 = np.zeros(traj.system.n_state, dtype=np.complex128)
        psi_0[states] = phi[:len(states)]
        traj.initialize(psi_0)
        if traj._adhops is not None:
            ad = traj._adhops
            counts = np.zeros((len(data["aux_list"]), traj.system.n_mode), dtype=np.int16)
            for i, a in enumerate(data["aux_list"]):
                for (m, k) in np.asarray(a).reshape(-1, 2):
                    counts[i, int(m)] = int(k)
            ad.update_basis(ad.phi, states, counts)
            if len(phi) != ad.basis.n_hier * ad.basis.n_state:
                raise TrajectoryError("checkpoint state does not match its basis")
            ad.phi = phi.copy()
            ad.zmem_abs = z_mem[:traj.system.n_mode].copy()
            ad.t = float(data["t"])
            ad.early_counter = int(data["early_counter"])
        else:
            if len(phi) != traj.n_hier * traj.n_state:
                raise TrajectoryError("checkpoint state does not match the hierarchy")
            traj._set_state(phi, z_mem[:traj.system.n_mode])
        traj._t = float(data["t"])
        traj.storage.data = data["storage_data"].item()
        traj.storage.metadata = data["storage_meta"].item()
        return traj

    def normalize(self, phi):
        """hops_trajectory.py:616-634 (host helper for callers)."""
        if self.eom_param["EQUATION_OF_MOTION"] == "NORMALIZED NONLINEAR":
            return phi / np.sqrt(np.sum(np.abs(phi[:self.n_state]) ** 2))
        return phi
