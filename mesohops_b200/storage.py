"""Trajectory storage (subset of storage/hops_storage.py:13-209).

Keeps the reference's dictionary interface -- ``storage['psi_traj']``,
``storage['t_axis']``, ``storage.data``, ``storage.metadata`` and the
STORAGE_TIME rule (True/False, a spacing, or a list of times) -- for the keys
psi_traj, t_axis, phi_traj and z_mem.  Adaptive keys (aux_list, state_list,
list_nhier, list_nstate) are stored by the adaptive driver.
"""
from __future__ import annotations

import numpy as np

from .constants import precision
from .exceptions import UnsupportedRequest

SUPPORTED = ("psi_traj", "t_axis", "phi_traj", "z_mem", "aux_list", "state_list",
             "list_nhier", "list_nstate")


class HopsStorage:
    def __init__(self, adaptive, storage_dic):
        storage_dic = dict(storage_dic or {})
        self.storage_time = storage_dic.pop("STORAGE_TIME", True)
        storage_dic.setdefault("phi_traj", False)
        storage_dic.setdefault("psi_traj", True)
        storage_dic.setdefault("t_axis", True)
        storage_dic.setdefault("z_mem", False)
        if adaptive:
            for k in ("aux_list", "state_list", "list_nhier", "list_nstate"):
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

    def __getitem__(self, item):
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
