"""Trajectory storage (subset of storage/hops_storage.py:13-209).

Keeps the reference's dictionary interface -- ``storage['psi_traj']``,
``storage['t_axis']``, ``storage.data``, ``storage.metadata`` and the
STORAGE_TIME rule (True/False, a spacing, or a list of times) -- for the keys
psi_traj, t_axis, phi_traj, phi_norm and z_mem, plus the adaptive keys
(aux_list, state_list, list_nhier, list_nstate, list_aux_norm).  For an
adaptive trajectory psi_traj is stored in the basis of each step and
``storage['psi_traj']`` returns the dense [n_t, n_dim] array
(hops_storage.py:71-97); ``storage['psi_traj_sparse']`` the csr form.
"""
from __future__ import annotations

import numpy as np

from .constants import precision
from .exceptions import UnsupportedRequest

SUPPORTED = ("psi_traj", "t_axis", "phi_traj", "phi_norm", "z_mem", "aux_list",
             "state_list", "list_nhier", "list_nstate", "list_aux_norm")


class HopsStorage:
    def __init__(self, adaptive, storage_dic):
        storage_dic = dict(storage_dic or {})
        self.storage_time = storage_dic.pop("STORAGE_TIME", True)
        storage_dic.setdefault("phi_traj", False)
        storage_dic.setdefault("psi_traj", True)
        storage_dic.setdefault("t_axis", True)
        storage_dic.setdefault("z_mem", False)
        if adaptive:
            for k in ("aux_list", "state_list", "list_nhier", "list_nstate", "list_aux_norm"):
                storage_dic.setdefault(k, True)
        for k, v in storage_dic.items():
            if k not in SUPPORTED:
                raise UnsupportedRequest(f"storage key {k}", "HopsStorage")
            if v is not False and not isinstance(v, bool):
                raise UnsupportedRequest("custom storage functions", "HopsStorage")
        self.storage_dic = storage_dic
        self.adaptive = adaptive
        self.data = {k: [] for k, v in storage_dic.items() if v}
        self.metadata = {"INITIALIZATION_TIME": 0, "LIST_PROPAGATION_TIME": []}
        self.n_dim = None

    def __getitem__(self, item):
        if self.adaptive and item == "psi_traj":
            full = np.zeros((len(self.data["t_axis"]), self.n_dim), dtype=np.complex128)
            for i, psi in enumerate(self.data["psi_traj"]):
                full[i, np.asarray(self.data["state_list"][i])] = psi
            return full
        if self.adaptive and item == "psi_traj_sparse":
            import scipy.sparse as sps
            rows, cols, vals = [], [], []
            for i, psi in enumerate(self.data["psi_traj"]):
                vals.extend(list(psi))
                rows.extend([i] * len(psi))
                cols.extend(list(self.data["state_list"][i]))
            return sps.csr_array((vals, (rows, cols)),
                                 shape=(len(self.data["t_axis"]), self.n_dim))
        if item in self.data:
            return self.data[item]
        raise KeyError(f"{item} not a key of storage.data")

    def check_storage_time(self, t):
        st = self.storage_time
        if isinstance(st, (list, np.ndarray)):
            return bool(np.any(np.abs(np.asarray(st) - t) < precision))
        if isinstance(st, bool):
            return st
        if isinstance(st, (int, float)):
            r = t / st
            return abs(r - round(r)) < precision
        raise UnsupportedRequest(f"STORAGE_TIME of type {type(st)}", "HopsStorage")

    def store(self, t, psi=None, phi=None, z_mem=None, aux_list=None, state_list=None):
        d = self.data
        if "t_axis" in d:
            d["t_axis"].append(t)
        if "psi_traj" in d:
            d["psi_traj"].append(psi)
        if "phi_traj" in d:
            d["phi_traj"].append(phi)
        if "phi_norm" in d:
            d["phi_norm"].append(None if phi is None else float(np.linalg.norm(phi)))
        if "z_mem" in d:
            d["z_mem"].append(z_mem)
        if "aux_list" in d:
            d["aux_list"].append(aux_list)
        if "state_list" in d:
            d["state_list"].append(state_list)
        if "list_nhier" in d:
            d["list_nhier"].append(None if aux_list is None else len(aux_list))
        if "list_nstate" in d:
            d["list_nstate"].append(None if state_list is None else len(state_list))
        if "list_aux_norm" in d:
            if phi is None or aux_list is None:
                d["list_aux_norm"].append(None)
            else:
                n_aux = len(aux_list)
                d["list_aux_norm"].append(
                    np.sqrt(np.sum(np.abs(np.asarray(phi)).reshape(n_aux, -1) ** 2, axis=1)))
