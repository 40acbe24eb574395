"""Batched ensemble: B trajectories of one system sharing one hierarchy.

Every trajectory has its own noise (seeds SEEDS[b] or precomputed arrays) and
its own state; the structure tables are uploaded once and every stage kernel
streams all B trajectories through each connection list (layout phi[a][s][b]).
This is the batched form of running HopsTrajectory B times (the reference runs
trajectories as independent processes, README.md:26-27).
"""
from __future__ import annotations

import numpy as np
import torch

from .constants import hbar, precision
from .device import hierarchy_structure
from .engine import StreamBatch
from .exceptions import TrajectoryError, UnsupportedRequest
from .noise import HopsNoise, filter_on_device, raw_white_noise
from .params import (EOM_DICT_DEFAULT, EOM_DICT_TYPES, HIERARCHY_DICT_DEFAULT,
                     HIERARCHY_DICT_TYPES, NOISE_DICT_DEFAULT, NOISE_DICT_TYPES,
                     initialize_dict)
from .system import HopsSystem


class HopsEnsemble:
    """B trajectories, one structure, one GPU.

    noise_param is a reference noise dictionary except that SEED may be a list of
    B seeds (FFT_FILTER) or an array [B, N_L2, n_t] (PRE_CALCULATED).
    """

    def __init__(self, system_param, n_traj, eom_param=None, noise_param=None,
                 hierarchy_param=None, precision="mixed", device="cuda:0", autotune=True):
        self.system = HopsSystem(system_param)
        self.eom_param = initialize_dict(eom_param or {}, EOM_DICT_DEFAULT, EOM_DICT_TYPES, "HopsEOM")
        self.hierarchy_param = initialize_dict(hierarchy_param or {}, HIERARCHY_DICT_DEFAULT,
                                               HIERARCHY_DICT_TYPES, "HopsHierarchy")
        self.B = int(n_traj)
        self.precision = precision
        self.device = torch.device(device)
        np_ = dict(noise_param or {})
        seeds = np_.pop("SEED", None)
        self.noise_param = initialize_dict(np_, NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, "HopsNoise")
        self.seeds = seeds
        self.n_t = int(np.ceil(self.noise_param["TLEN"] / self.noise_param["TAU"])) + 1
        self.basis, self.dstruct = hierarchy_structure(self.system, self.hierarchy_param,
                                                       self.device)
        self.batch = StreamBatch(self.dstruct, self.B, precision,
                                 self.eom_param["EQUATION_OF_MOTION"])
        # renormalisation after each call left pending and applied by the next
        # call (or by state()): a call per step costs no extra pass over phi
        self.batch.defer_scale = True
        self.t = 0.0
        self.noise = None
        self.autotune = autotune
        self._tuned = False

    @property
    def n_hier(self):
        return self.basis.n_hier

    @property
    def n_state(self):
        return self.system.n_state

    def prepare_noise(self):
        """Correlated noise [B, N_L2, n_t] complex64 on the device."""
        model = self.noise_param["MODEL"]
        L, n_t = self.system.n_lop, self.n_t
        if model == "ZERO":
            self.noise = None
        elif model == "PRE_CALCULATED":
            arr = np.asarray(self.seeds)
            if arr.shape != (self.B, L, n_t):
                raise UnsupportedRequest("PRE_CALCULATED ensemble noise must be [B, N_L2, n_t]",
                                         "HopsEnsemble", override=True)
            dt = np.complex128 if self.noise_param["INTERPOLATE"] else np.complex64
            self.noise = torch.from_numpy(np.ascontiguousarray(arr.astype(dt))).to(self.device)
        elif model == "FFT_FILTER":
            seeds = self.seeds if self.seeds is not None else [None] * self.B
            if len(seeds) != self.B:
                raise UnsupportedRequest("one SEED per trajectory", "HopsEnsemble", override=True)
            proto = HopsNoise({k: v for k, v in self.noise_param.items() if k != "T_AXIS"},
                              self.system)
            alpha = proto._corr()
            raw = raw_white_noise(seeds, range(L), n_t, self.noise_param["RAND_MODEL"],
                                  self.device)
            out, _ = filter_on_device(alpha, raw, self.device,
                                      complex128=bool(self.noise_param["INTERPOLATE"]))
            self.noise = out.reshape(self.B, L, n_t)
        else:
            raise UnsupportedRequest(f"Noise.param[MODEL] {model}", "HopsEnsemble")
        self.batch.set_noise(self.noise, None)

    def initialize(self, psi_0):
        """psi_0: one initial state for all, or [B, n_state]."""
        psi_0 = np.asarray(psi_0, dtype=np.complex128)
        if psi_0.ndim == 1:
            psi_0 = np.tile(psi_0, (self.B, 1))
        phi = np.zeros((self.B, self.n_hier * self.n_state), dtype=np.complex128)
        phi[:, :self.n_state] = psi_0
        self.batch.set_state(phi, np.zeros((self.B, self.system.n_mode), dtype=np.complex128))
        if self.noise is None and self.noise_param["MODEL"] != "ZERO":
            self.prepare_noise()
        self.t = 0.0

    def steps_for(self, t_advance, tau):
        tau_noise = self.noise_param["TAU"]
        ts = tau * 0.5 / tau_noise
        if ts - int(round(ts)) >= precision or int(round(tau / tau_noise)) < 1:
            raise TrajectoryError(f"Timesteps({tau * 0.5}) that do not match noise.param['TAU'] "
                                  f"({tau_noise})")
        if self.t + t_advance + tau > self.noise_param["TLEN"]:
            raise TrajectoryError("Trajectory times longer than noise.param['TLEN'] ="
                                  + str(self.noise_param["TLEN"]))
        n = int(np.ceil(t_advance / tau))
        it0 = int(round(self.t / tau_noise))
        di = int(round(tau * 0.5 / tau_noise))
        return n, it0, di

    def tune(self, tau):
        """Run the stage-kernel autotuner for steps of tau now (it restores the
        state), so that a later propagate call carries no tuning runs."""
        _, it0, di = self.steps_for(tau, tau)
        if self.autotune and not self._tuned:
            self.batch.autotune(it0, di, tau / hbar)
            self._tuned = True

    def propagate(self, t_advance, tau, psi_out=None):
        """Propagate all trajectories; psi_out: optional device tensor [n, B, S] c128."""
        n, it0, di = self.steps_for(t_advance, tau)
        if self.autotune and not self._tuned:
            self.batch.autotune(it0, di, tau / hbar)
            self._tuned = True
        self.batch.propagate(it0, di, n, tau / hbar, psi_out=psi_out)
        self.t += n * tau
        return n

    def check(self):
        self.batch.check_status()

    def state(self):
        return self.batch.get_state()
