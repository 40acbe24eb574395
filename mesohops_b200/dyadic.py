"""HOPS trajectories in the double (ket, bra) Hilbert space.

Drop-in for mesohops.trajectory.hops_dyadic.DyadicTrajectory
(trajectory/hops_dyadic.py:15-246): the Hamiltonian and every L-operator of
the system dictionary become block-diagonal [[M, 0], [0, M]] operators on the
doubled state space, the initial state is the normalised concatenation of a
ket and a bra wave function, and ket- or bra-side operators act on the running
state between propagation calls while their normalisation factors are
recorded for the response function (util/spectroscopy_analysis.py:67-113).
Propagation is the ordinary trajectory hot path on the doubled system.
"""
from __future__ import annotations

import time as timer

import numpy as np
import scipy.sparse as sps

from .exceptions import UnsupportedRequest
from .trajectory import HopsTrajectory


def dyad_conversion(m2):
    """(N, N) matrix -> (2N, 2N) block-diagonal [[M, 0], [0, M]]; sparse input
    gives a COO matrix (hops_dyadic.py:109-139)."""
    n = np.shape(m2)[0]
    if sps.issparse(m2):
        c = sps.coo_matrix(m2)
        return sps.coo_matrix((np.concatenate((c.data, c.data)),
                               (np.concatenate((c.row, c.row + n)),
                                np.concatenate((c.col, c.col + n)))), shape=(2 * n, 2 * n))
    out = np.zeros((2 * n, 2 * n), dtype=np.complex128)
    out[:n, :n] = m2
    out[n:, n:] = m2
    return out


def response_function_calc(f_op, index_t, traj, list_response_norm_sq):
    """Normalised response-function component prod(norms) <psi|F|psi> / |psi|^2
    at every stored time after index_t (spectroscopy_analysis.py:67-113)."""
    f = sps.csr_matrix(f_op)
    tr = np.asarray(traj).T
    norm = np.prod(list_response_norm_sq)
    return np.array([norm / np.linalg.norm(tr[:, c]) ** 2 * (np.conj(tr[:, c]) @ (f @ tr[:, c]))
                     for c in range(int(index_t) + 1, tr.shape[1])])


class DyadicTrajectory(HopsTrajectory):
    """A HOPS trajectory in the double Hilbert space (hops_dyadic.py:15-246)."""

    def __init__(self, system_param, eom_param=None, noise_param=None, noise2_param=None,
                 hierarchy_param=None, storage_param=None, integration_param=None,
                 device_param=None):
        system_param = {} if system_param is None else system_param
        system_param.update({"HAMILTONIAN": dyad_conversion(system_param["HAMILTONIAN"])})
        for key in ("L_HIER", "L_NOISE1", "L_NOISE2", "L_LT_CORR"):
            if key in system_param:
                system_param.update({key: [dyad_conversion(l) for l in system_param[key]]})
        super().__init__(system_param, eom_param=eom_param, noise_param=noise_param,
                         noise2_param=noise2_param, hierarchy_param=hierarchy_param,
                         storage_param=storage_param, integration_param=integration_param,
                         device_param=device_param)
        self._list_response_norm_sq = []

    def initialize(self, psi_ket, psi_bra, timer_checkpoint=None):
        """phi_0 from psi_0 = [psi_ket, psi_bra] / |[psi_ket, psi_bra]|."""
        if timer_checkpoint is None:
            timer_checkpoint = timer.time()
        psi_0 = np.concatenate((np.asarray(psi_ket), np.asarray(psi_bra)))
        self._list_response_norm_sq = [np.linalg.norm(psi_0) ** 2]
        psi_0 = psi_0 / np.sqrt(self._list_response_norm_sq[0])
        super().initialize(psi_0, timer_checkpoint=timer_checkpoint)

    def _M2_dyad_conversion(self, m2):
        return dyad_conversion(m2)

    def _dyad_operator(self, op_hilbert, side):
        """Act a ket-side operator K as [[K, 0], [0, I]] (bra side: [[I, 0], [0, B]])
        on the state, renormalise (normalised equation of motion) and record the
        factor for the response function (hops_dyadic.py:141-210)."""
        if side not in ("ket", "bra"):
            raise UnsupportedRequest('sides other than "ket" or "bra"', "_dyad_operator")
        n = np.shape(op_hilbert)[0]
        sl = np.asarray(self.state_list)
        deno = np.linalg.norm(self.phi[:len(sl)]) ** 2
        if sps.issparse(op_hilbert):
            c = sps.coo_matrix(op_hilbert)
            if side == "bra":
                keep = sl[sl < n]
                data = np.concatenate((np.ones(len(keep)), c.data))
                row = np.concatenate((keep, c.row + n))
                col = np.concatenate((keep, c.col + n))
            else:
                keep = sl[sl >= n]
                data = np.concatenate((c.data, np.ones(len(keep))))
                row = np.concatenate((c.row, keep))
                col = np.concatenate((c.col, keep))
            op = sps.coo_matrix((data, (row, col)), shape=(2 * n, 2 * n), dtype=np.complex128)
        else:
            op = np.zeros((2 * n, 2 * n), dtype=np.complex128)
            op[sl, sl] = 1
            if side == "bra":
                op[n:, n:] = op_hilbert
            else:
                op[:n, :n] = op_hilbert
        self._operator(op)
        phi = self.phi
        # the state basis may have grown (adaptive): the norm is over the new one
        nrm = np.linalg.norm(phi[:len(self.state_list)]) ** 2
        if self.eom_param["EQUATION_OF_MOTION"] == "NORMALIZED NONLINEAR":
            self._list_response_norm_sq.append(nrm)
            self.phi = phi / np.sqrt(np.sum(np.abs(phi[:self.n_state]) ** 2))
        else:
            self._list_response_norm_sq.append(nrm / deno)

    def _response_function_comp(self, f_op, index_t):
        """Response-function component of a dyadic operator after index_t."""
        return response_function_calc(f_op, index_t, self.storage["psi_traj"],
                                      self._list_response_norm_sq)

    @property
    def list_response_norm_sq(self):
        return self._list_response_norm_sq
