"""System parameter expansion (host side of the drop-in surface).

Restates the parts of basis/system_functions.py:10-172 and
basis/hops_system.py:47-136 that the trajectory hot path consumes: the state
count, the (g, w) mode lists, the unique L-operator list (unique by nonzero
pattern, values of the first mode with that pattern, as in the reference), the
mode -> L map and the noise-mode -> L maps.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps

from .exceptions import UnsupportedRequest


def pattern_key(lop):
    """Nonzero pattern ((rows), (cols)) used to identify unique L-operators.

    Same key as util/helper_functions.py:8-32 (storage order for sparse input,
    row-major for dense input).
    """
    if sps.issparse(lop):
        if lop.getnnz() == 0:
            return tuple()
        nz = lop.nonzero()
    else:
        a = np.asarray(lop)
        if a.size == 0:
            return tuple()
        nz = np.nonzero(a)
    return tuple(tuple(int(x) for x in v) for v in nz)


def _csr(op, n):
    if sps.issparse(op):
        a = sps.csr_matrix(op, dtype=np.complex128)
    else:
        a = sps.csr_matrix(np.asarray(op, dtype=np.complex128))
    if a.shape != (n, n):
        raise UnsupportedRequest(f"operator of shape {a.shape} (expected {(n, n)})",
                                 "HopsSystem", override=True)
    a.eliminate_zeros()
    return a


class HopsSystem:
    """Expanded system parameters (absolute indices)."""

    def __init__(self, system_param):
        if not isinstance(system_param, dict):
            raise TypeError("system_param must be a dictionary.")
        for key in ("HAMILTONIAN", "GW_SYSBATH", "L_HIER", "L_NOISE1", "ALPHA_NOISE1",
                    "PARAM_NOISE1"):
            if key not in system_param:
                raise UnsupportedRequest(f"missing system key {key}", "HopsSystem",
                                         override=True)
        p = dict(system_param)
        H = p["HAMILTONIAN"]
        self.n_state = int(H.shape[0]) if sps.issparse(H) else len(np.asarray(H)[0])
        self.hamiltonian = (sps.csr_matrix(H, dtype=np.complex128) if sps.issparse(H)
                            else np.asarray(H, dtype=np.complex128))
        self.gw = [(complex(g), complex(w)) for (g, w) in p["GW_SYSBATH"]]
        self.n_mode = len(self.gw)
        self.G = np.array([g for g, _ in self.gw], dtype=np.complex128)
        self.W = np.array([w for _, w in self.gw], dtype=np.complex128)
        if len(p["L_HIER"]) != self.n_mode:
            raise UnsupportedRequest("L_HIER and GW_SYSBATH of different lengths",
                                     "HopsSystem", override=True)
        # unique L (system_functions.py:64-107)
        keys = [pattern_key(l) for l in p["L_HIER"]]
        self._key_index = {}
        self.lops_csr = []                  # sparse complex [n_state, n_state]
        self.l_by_mode = np.zeros(self.n_mode, dtype=np.int64)
        for m, k in enumerate(keys):
            if k not in self._key_index:
                self._key_index[k] = len(self.lops_csr)
                self.lops_csr.append(_csr(p["L_HIER"][m], self.n_state))
            self.l_by_mode[m] = self._key_index[k]
        self.n_lop = len(self.lops_csr)
        self._lops_dense = None
        self._coo = None
        self.modes_by_l = [np.nonzero(self.l_by_mode == j)[0] for j in range(self.n_lop)]
        # noise 1 (system_functions.py:135-150)
        self.l_by_nmode1, self.nmodes1_by_l = self._noise_map(p["L_NOISE1"], p["PARAM_NOISE1"])
        self.alpha1 = p["ALPHA_NOISE1"]
        self.param_noise1 = list(p["PARAM_NOISE1"])
        self.has_noise2 = "L_NOISE2" in p
        if self.has_noise2:
            self.l_by_nmode2, self.nmodes2_by_l = self._noise_map(p["L_NOISE2"], p["PARAM_NOISE2"])
            self.alpha2 = p.get("ALPHA_NOISE2")
            self.param_noise2 = list(p.get("PARAM_NOISE2", []))
        # low-temperature corrections: summed per unique L; an operator of no
        # bath is dropped with the reference's warning (system_functions.py:50-56,115-133)
        lt_ops = list(p.get("L_LT_CORR", []))
        lt_par = list(p.get("PARAM_LT_CORR", []))
        if len(lt_ops) != len(lt_par):
            raise UnsupportedRequest("L_LT_CORR and PARAM_LT_CORR of different lengths",
                                     "HopsSystem", override=True)
        self.lt_coef = np.zeros(self.n_lop, dtype=np.complex128)
        for lop, c in zip(lt_ops, lt_par):
            j = self._key_index.get(pattern_key(lop))
            if j is None:
                print("WARNING: the list of low-temperature correction L-operators contains "
                      "an L-operator not associated with any existing thermal environment. "
                      "This low-temperature correction factor will be discarded!")
                continue
            self.lt_coef[j] += complex(c)
        self.has_lt = bool(np.any(self.lt_coef != 0))
        # state <-> mode maps (system_functions.py:33-39) and H couplings
        self.states_by_lop = [np.array(self.states_of_lop(j), dtype=np.int64)
                              for j in range(self.n_lop)]
        self.modes_by_state = [[] for _ in range(self.n_state)]
        for m in range(self.n_mode):
            for st in self.states_by_lop[self.l_by_mode[m]]:
                self.modes_by_state[st].append(m)
        Hd = self.hamiltonian_dense()
        self.coupled_states = [np.nonzero(Hd[i])[0] for i in range(self.n_state)]
        self.param = p
        self.param["NSTATES"] = self.n_state
        self.param["N_HMODES"] = self.n_mode
        self.param["G"] = self.G
        self.param["W"] = self.W
        self.param["N_L2"] = self.n_lop
        self.param["LIST_INDEX_L2_BY_HMODE"] = list(self.l_by_mode)
        self.param["LIST_INDEX_L2_BY_NMODE1"] = list(self.l_by_nmode1)
        self.param["LIST_NMODE1_BY_INDEX_L2"] = [list(x) for x in self.nmodes1_by_l]
        self.param["LIST_LT_PARAM"] = list(self.lt_coef)

    def _noise_map(self, lops, params):
        l_by_nmode = []
        nmodes_by_l = [[] for _ in range(self.n_lop)]
        for i, l in enumerate(lops):
            k = pattern_key(l)
            if k not in self._key_index:
                # the reference discards such noise modes with a warning
                l_by_nmode.append(None)
                continue
            j = self._key_index[k]
            l_by_nmode.append(j)
            nmodes_by_l[j].append(i)
        if len(params) != len(lops):
            raise UnsupportedRequest("noise parameter / L list length mismatch", "HopsSystem",
                                     override=True)
        return l_by_nmode, nmodes_by_l

    def hamiltonian_dense(self):
        H = self.hamiltonian
        return H.toarray() if sps.issparse(H) else np.asarray(H)

    @property
    def lops(self):
        """Unique L-operators as dense arrays (built on first use; small systems)."""
        if self._lops_dense is None:
            self._lops_dense = [l.toarray() for l in self.lops_csr]
        return self._lops_dense

    def lop_block(self, j, states):
        """Dense block L_j[states, states] (O(nnz(L_j)) via a position map)."""
        states = np.asarray(states, dtype=np.int64)
        if self._coo is None:
            self._coo = [(l.tocoo().row, l.tocoo().col, l.tocoo().data) for l in self.lops_csr]
        r, c, v = self._coo[j]
        pos = np.full(self.n_state, -1, dtype=np.int64)
        pos[states] = np.arange(len(states))
        pr, pc = pos[r], pos[c]
        keep = (pr >= 0) & (pc >= 0)
        out = np.zeros((len(states), len(states)), dtype=np.complex128)
        np.add.at(out, (pr[keep], pc[keep]), v[keep])
        return out

    def lop_is_diagonal(self, j):
        r, c = self.lops_csr[j].nonzero()
        return bool(np.all(r == c))

    def states_of_lop(self, j):
        """States touched by L_j (helper_functions.py:50-66)."""
        r, c = self.lops_csr[j].nonzero()
        return sorted(set(r.tolist()) | set(c.tolist()))
