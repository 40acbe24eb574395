"""Device-resident structure tables of one basis (system x hierarchy).

``build_tables`` turns a state basis, a mode basis and an ``AuxBasis`` into the
flat arrays of ``hops_structure`` (include/hops_b200.h); ``DeviceStructure``
uploads them with torch and exposes the ctypes struct of device pointers.
The arrays encode the super-operators of eom/eom_hops_ksuper.py:36-230:
  K2_k      -> k_decay[a]            = -sum_m k_m(a) w_m
  K2_kp1    -> up list (a, a+e_m, m)   with -(g_m/w_m) L_m applied in-kernel
  K2_km1    -> down list (a, a-e_m, m, k_m(a) w_m) with L_m^H applied in-kernel
  Z2_kp1    -> the same up list with (g_m/w_m) conj(<L>) applied in-kernel
"""
from __future__ import annotations

import ctypes as C
from math import comb

import numpy as np
import torch

from ._lib import HopsStructure


def _csr_of_dense(mats, n):
    """CSR (absolute offsets) of a list of dense n x n complex matrices: block j
    occupies ptr[j*(n+1) : (j+1)*(n+1)], entries in row-major order."""
    if len(mats) == 0:
        return np.zeros(0, dtype=np.int32), np.zeros(0, np.int32), np.zeros(0, np.complex128)
    A = np.asarray(mats, dtype=np.complex128).reshape(len(mats), n, n)
    j, r, c = np.nonzero(A)
    counts = np.zeros(len(mats) * n, dtype=np.int64)
    np.add.at(counts, j * n + r, 1)
    start = np.concatenate([[0], np.cumsum(counts)])
    ptr = np.zeros(len(mats) * (n + 1), dtype=np.int32)
    rows = np.arange(len(mats) * n)
    ptr[(rows // n) * (n + 1) + rows % n] = start[:-1]
    ptr[np.arange(len(mats)) * (n + 1) + n] = start[(np.arange(len(mats)) + 1) * n]
    return ptr, c.astype(np.int32), A[j, r, c]


def _c2d(a):
    """complex -> interleaved float64."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128))
    return a.view(np.float64).copy() if a.size else np.zeros(2, dtype=np.float64)


def _c2f(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.complex64))
    return a.view(np.float32).copy() if a.size else np.zeros(2, dtype=np.float32)


def _c2d_any(a):
    if isinstance(a, torch.Tensor):
        return torch.view_as_real(a.to(torch.complex128).contiguous()).reshape(-1)
    return _c2d(a)


def _c2f_any(a):
    if isinstance(a, torch.Tensor):
        return torch.view_as_real(a.to(torch.complex64).contiguous()).reshape(-1)
    return _c2f(a)


def _i32_any(a):
    if isinstance(a, torch.Tensor):
        return a.to(torch.int32)
    return np.asarray(a).astype(np.int32)


def build_tables(system, basis, state_list=None, mode_list=None, small=None):
    """Host arrays of one basis.

    state_list: sorted absolute states of the state basis (default: all).
    mode_list:  sorted absolute modes of the mode basis (default: basis.modes).
    small:      ``_state_mode_tables`` of these states and modes when the caller
                has them already (copied, not modified).
    Returns a dict of numpy arrays and sizes plus index maps.
    """
    S_abs = system.n_state
    states = np.arange(S_abs) if state_list is None else np.asarray(state_list, dtype=np.int64)
    modes = basis.modes if mode_list is None else np.asarray(mode_list, dtype=np.int64)
    small = _state_mode_tables(system, states, modes) if small is None else dict(small)
    M = small["n_mode"]
    mode_lop, sval = small["mode_lop"], small["lop_sval"]
    W = small["mode_w"]
    counts = basis.counts
    # K2_k diagonal (eom_hops_ksuper.py:78-87): -aux . W over the aux's own modes
    k_decay = -(counts[:, modes].astype(np.float64) @ W) if M else np.zeros(basis.n_hier)
    # connections are along basis.modes (a subset of the sorted mode list);
    # remap to the relative mode list
    bm = np.asarray(basis.modes, dtype=np.int64)
    rel = np.searchsorted(modes, bm).astype(np.int32)
    if len(bm) and (rel.max() >= len(modes) or np.any(modes[rel] != bm)):
        raise ValueError("the basis modes are not in the mode list")
    up_m = rel[np.asarray(basis.up_m, dtype=np.int64)]
    dn_m = rel[np.asarray(basis.dn_m, dtype=np.int64)]
    dn_coef = basis.dn_k.astype(np.float64) * W[dn_m] if len(dn_m) else np.zeros(0, complex)
    first = [(a, int(rel[m])) for (a, m) in basis.first_level()]
    first_aux = np.array([a for a, _ in first], dtype=np.int32)
    first_mode = np.array([m for _, m in first], dtype=np.int32)
    mode_site = small["mode_site"]
    dn_coef_site = dn_coef * np.conj(sval[mode_lop[dn_m]]) if len(dn_m) else np.zeros(0, complex)
    up_site = mode_site[up_m] if len(up_m) else np.zeros(0, dtype=np.int32)
    dn_site = mode_site[dn_m] if len(dn_m) else np.zeros(0, dtype=np.int32)
    up_counts = np.diff(basis.up_ptr)
    dn_counts = np.diff(basis.dn_ptr)
    small.update(
        n_hier=basis.n_hier,
        k_decay=k_decay, up_ptr=basis.up_ptr.astype(np.int32),
        up_aux=basis.up_u.astype(np.int32), up_mode=up_m,
        dn_ptr=basis.dn_ptr.astype(np.int32), dn_aux=basis.dn_d.astype(np.int32),
        dn_mode=dn_m, dn_coef=dn_coef,
        first_aux=first_aux, first_mode=first_mode,
        dn_coef_site=dn_coef_site,
        up_site=np.asarray(up_site, dtype=np.int32), dn_site=np.asarray(dn_site, dtype=np.int32),
        max_up=int(up_counts.max()) if len(up_counts) else 0,
        max_dn=int(dn_counts.max()) if len(dn_counts) else 0,
        n_up_prefix=int(np.flatnonzero(up_counts)[-1]) + 1 if np.any(up_counts) else 0,
    )
    return small


def _state_mode_tables(system, states, modes):
    """Tables that depend only on the state and mode bases: the relative L list
    and its CSR forms, -iH, per-mode coefficients, the site-projector form."""
    S = len(states)
    M = len(modes)
    # relative L list: unique L of the basis modes, sorted (hops_modes.py:123-136)
    l_abs = np.array(sorted(set(int(system.l_by_mode[m]) for m in modes)), dtype=np.int64)
    L = len(l_abs)
    l_rel_of_abs = {int(j): i for i, j in enumerate(l_abs)}
    mode_lop = np.array([l_rel_of_abs[int(system.l_by_mode[m])] for m in modes], dtype=np.int32)
    ix = np.ix_(states, states)
    lops = [system.lop_block(j, states) for j in l_abs]
    lop_active = np.array([1 if np.any(l != 0) else 0 for l in lops], dtype=np.int32)
    # site-projector form: exactly one diagonal nonzero
    site = np.zeros(L, dtype=np.int32)
    sval = np.zeros(L, dtype=np.complex128)
    is_site = True
    for j, l in enumerate(lops):
        r, c = np.nonzero(l)
        if len(r) == 1 and r[0] == c[0]:
            site[j] = r[0]
            sval[j] = l[r[0], c[0]]
        elif len(r) == 0:
            site[j] = -1
        else:
            is_site = False
    l_ptr, l_col, l_val = _csr_of_dense(lops, S)
    lh_ptr, lh_col, lh_val = _csr_of_dense([np.conj(l.T) for l in lops], S)
    H = system.hamiltonian_dense()[ix]
    if is_site:
        # site-projector form: the diagonal of -iH joins the per-state diagonal
        # coefficient; the CSR keeps the couplings only
        h_diag = -1j * np.diag(H).astype(np.complex128)
        h_ptr, h_col, h_val = _csr_of_dense([-1j * (H - np.diag(np.diag(H)))], S)
    else:
        h_diag = None
        h_ptr, h_col, h_val = _csr_of_dense([-1j * H], S)
    G = system.G[modes]
    W = system.W[modes]
    # low-temperature corrections of the relative L list, with the CSR of L_j^2
    # (hops_eom.py:357-403 uses list_L2_sq_csr); none when every c_j is zero
    lt = np.asarray(getattr(system, "lt_coef", np.zeros(system.n_lop)))[l_abs] if L else None
    if lt is not None and np.any(lt != 0):
        l2_ptr, l2_col, l2_val = _csr_of_dense([l @ l for l in lops], S)
    else:
        lt, l2_ptr, l2_col, l2_val = None, None, None, None
    # site-projector coefficients per mode
    mode_site = site[mode_lop] if M else np.zeros(0, dtype=np.int32)
    mode_gwv = (G / W) * sval[mode_lop] if M else np.zeros(0, dtype=complex)
    return dict(
        n_state=S, n_mode=M, n_lop=L, states=states, modes=modes, l_abs=l_abs,
        mode_lop=mode_lop, mode_g=G, mode_w=W, mode_gw=G / W if M else G,
        l_ptr=l_ptr, l_col=l_col, l_val=l_val, lh_ptr=lh_ptr, lh_col=lh_col, lh_val=lh_val,
        lop_active=lop_active, lop_site=site, lop_sval=sval,
        h_ptr=h_ptr, h_col=h_col, h_val=h_val, site_projector=int(is_site),
        mode_site=mode_site.astype(np.int32), mode_gwv=mode_gwv, h_diag=h_diag,
        lt_coef=lt, l2_ptr=l2_ptr, l2_col=l2_col, l2_val=l2_val,
    )


def _binomials(n_max, k_max):
    """int64 table C(n, j), n <= n_max, j <= k_max (row stride k_max + 1)."""
    t = np.zeros((n_max + 1, k_max + 1), dtype=np.int64)
    for n in range(n_max + 1):
        for j in range(min(n, k_max) + 1):
            t[n, j] = comb(n, j)
    return t


def build_tables_triangular(system, depth, device):
    """``build_tables`` for the full triangular hierarchy over every mode and
    state, with the aux-indexed arrays built on the GPU (hops_tri_pass1/2)
    and left there as torch tensors; the state/mode tables stay on the host."""
    from . import _lib
    from .exceptions import UnsupportedRequest
    dev = torch.device(device)
    M, D = system.n_mode, int(depth)
    N = comb(M + D, D)
    n_below = comb(M + D - 1, D - 1) if D > 0 else 0
    if N >= 2 ** 31:
        raise UnsupportedRequest(f"hierarchy of {N} aux (>= 2^31)", "mesohops_b200 build_tables")
    small = _state_mode_tables(system, np.arange(system.n_state), np.arange(M))
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    binom = torch.from_numpy(_binomials(M + D + 1, D + 1)).to(dev)
    w = torch.from_numpy(np.ascontiguousarray(system.W, dtype=np.complex128)).to(dev)
    k_decay = torch.empty(N, dtype=torch.complex128, device=dev)
    dn_count = torch.empty(N, dtype=torch.int32, device=dev)
    _lib.check(L.hops_tri_pass1(M, D, binom.data_ptr(), N, w.data_ptr(), k_decay.data_ptr(),
                                dn_count.data_ptr(), stream), "hops_tri_pass1")
    dn_ptr = torch.zeros(N + 1, dtype=torch.int64, device=dev)
    dn_ptr[1:] = torch.cumsum(dn_count, 0)
    n_dn = int(dn_ptr[-1])
    dn_ptr = dn_ptr.to(torch.int32)
    up_aux = torch.empty(n_below * M, dtype=torch.int32, device=dev)
    up_mode = torch.empty(n_below * M, dtype=torch.int32, device=dev)
    dn_aux = torch.empty(max(n_dn, 1), dtype=torch.int32, device=dev)
    dn_mode = torch.empty(max(n_dn, 1), dtype=torch.int32, device=dev)
    dn_k = torch.empty(max(n_dn, 1), dtype=torch.int32, device=dev)
    _lib.check(L.hops_tri_pass2(M, D, binom.data_ptr(), N, n_below, dn_ptr.data_ptr(),
                                up_aux.data_ptr(), up_mode.data_ptr(), dn_aux.data_ptr(),
                                dn_mode.data_ptr(), dn_k.data_ptr(), stream), "hops_tri_pass2")
    dn_aux, dn_mode, dn_k = dn_aux[:n_dn], dn_mode[:n_dn], dn_k[:n_dn]
    up_ptr = (torch.clamp(torch.arange(N + 1, device=dev), max=n_below) * M).to(torch.int32)
    sval = torch.from_numpy(small["lop_sval"]).to(dev)
    mode_lop = torch.from_numpy(small["mode_lop"].astype(np.int64)).to(dev)
    mode_site = torch.from_numpy(small["mode_site"].astype(np.int64)).to(dev)
    dnm = dn_mode.to(torch.int64)
    dn_coef = dn_k.to(torch.float64) * w[dnm]
    dn_coef_site = dn_coef * torch.conj(sval[mode_lop[dnm]])
    first_aux = np.arange(1, M + 1, dtype=np.int32) if D >= 1 else np.zeros(0, np.int32)
    first_mode = np.arange(M, dtype=np.int32) if D >= 1 else np.zeros(0, np.int32)
    small.update(
        n_hier=int(N), k_decay=k_decay, up_ptr=up_ptr, up_aux=up_aux, up_mode=up_mode,
        dn_ptr=dn_ptr, dn_aux=dn_aux, dn_mode=dn_mode, dn_coef=dn_coef,
        first_aux=first_aux, first_mode=first_mode, dn_coef_site=dn_coef_site,
        up_site=mode_site[up_mode.to(torch.int64)].to(torch.int32),
        dn_site=mode_site[dnm].to(torch.int32),
        max_up=M if n_below > 0 else 0, max_dn=min(D, M) if N > 1 else 0,
        n_up_prefix=int(n_below),
    )
    return small


class DeviceStructure:
    """hops_structure with its arrays resident on one CUDA device.

    Every table and a device copy of the struct itself live in one packed
    buffer uploaded with a single asynchronous host->device copy from pinned
    memory (cheap enough to rebuild at every adaptive basis change, and no
    wait for the work already queued on the stream).  `extras` (name -> numpy
    array) are packed into the same buffer and exposed as device tensors in
    `self.extra` (e.g. the noise rows of an adaptive basis).
    """

    _ALIGN = 256

    def __init__(self, tables, device, extras=None):
        self.tables = tables
        self.device = torch.device(device)
        t = tables
        c2d, c2f = _c2d_any, _c2f_any
        i32 = np.int32
        fields = [
            ("k_decay", c2d(t["k_decay"])), ("k_decay_f", c2f(t["k_decay"])),
            ("up_ptr", _i32_any(t["up_ptr"])), ("up_aux", _i32_any(t["up_aux"])),
            ("up_mode", _i32_any(t["up_mode"])),
            ("dn_ptr", _i32_any(t["dn_ptr"])), ("dn_aux", _i32_any(t["dn_aux"])),
            ("dn_mode", _i32_any(t["dn_mode"])),
            ("dn_coef", c2d(t["dn_coef"])), ("dn_coef_f", c2f(t["dn_coef"])),
            ("mode_lop", t["mode_lop"].astype(i32)), ("mode_g", c2d(t["mode_g"])),
            ("mode_w", c2d(t["mode_w"])), ("mode_gw", c2d(t["mode_gw"])),
            ("mode_gw_f", c2f(t["mode_gw"])),
            ("first_aux", t["first_aux"].astype(i32)), ("first_mode", t["first_mode"].astype(i32)),
            ("l_ptr", t["l_ptr"].astype(i32)), ("l_col", t["l_col"].astype(i32)),
            ("l_val", c2d(t["l_val"])), ("l_val_f", c2f(t["l_val"])),
            ("lh_ptr", t["lh_ptr"].astype(i32)), ("lh_col", t["lh_col"].astype(i32)),
            ("lh_val", c2d(t["lh_val"])), ("lh_val_f", c2f(t["lh_val"])),
            ("lop_active", t["lop_active"].astype(i32)), ("lop_site", t["lop_site"].astype(i32)),
            ("lop_sval", c2d(t["lop_sval"])),
            ("h_ptr", t["h_ptr"].astype(i32)), ("h_col", t["h_col"].astype(i32)),
            ("h_val", c2d(t["h_val"])), ("h_val_f", c2f(t["h_val"])),
            ("mode_site", t["mode_site"].astype(i32)), ("mode_gwv", c2d(t["mode_gwv"])),
            ("mode_gwv_f", c2f(t["mode_gwv"])),
            ("dn_coef_site", c2d(t["dn_coef_site"])), ("dn_coef_site_f", c2f(t["dn_coef_site"])),
            ("up_site", _i32_any(t["up_site"])), ("dn_site", _i32_any(t["dn_site"])),
        ]
        if t["h_diag"] is not None:
            fields.append(("h_diag", c2d(t["h_diag"])))
        if t.get("lt_coef") is not None:
            fields += [("lt_coef", c2d(t["lt_coef"])), ("l2_ptr", t["l2_ptr"].astype(i32)),
                       ("l2_col", t["l2_col"].astype(i32)), ("l2_val", c2d(t["l2_val"]))]
        offs = {}
        off = 0
        extra_names = []
        for name, arr in (extras or {}).items():
            fields.append(("extra:" + name, np.ascontiguousarray(arr)))
            extra_names.append(name)
        for name, arr in fields:
            if isinstance(arr, torch.Tensor):
                a = arr.contiguous()
                if a.numel() == 0:
                    a = torch.zeros(4, dtype=torch.int32, device=self.device)
                nbytes = a.numel() * a.element_size()
            else:
                a = np.ascontiguousarray(arr)
                if a.size == 0:
                    a = np.zeros(4, dtype=np.int32)
                nbytes = a.nbytes
            offs[name] = (off, a, nbytes)
            off += -(-nbytes // self._ALIGN) * self._ALIGN
        struct_off = off
        total = off + C.sizeof(HopsStructure)
        self.buffer = torch.empty(total, dtype=torch.uint8, device=self.device)
        base = self.buffer.data_ptr()
        pinned = torch.empty(total, dtype=torch.uint8,
                             pin_memory=self.device.type == "cuda")
        host = pinned.numpy()
        s = HopsStructure()
        s.n_hier, s.n_state, s.n_mode, s.n_lop = t["n_hier"], t["n_state"], t["n_mode"], t["n_lop"]
        s.n_first = len(t["first_aux"])
        s.n_up = len(t["up_aux"])
        s.n_dn = len(t["dn_aux"])
        s.site_projector = t["site_projector"]
        s.max_up, s.max_dn = t["max_up"], t["max_dn"]
        s.n_up_prefix = t.get("n_up_prefix", 0)
        dev_parts = []
        self.extra = {}
        for name, (o, a, nbytes) in offs.items():
            if isinstance(a, torch.Tensor):
                dev_parts.append((o, a, nbytes))
            else:
                host[o:o + nbytes] = a.view(np.uint8).ravel()
            if name.startswith("extra:"):
                arr = (extras or {})[name[6:]]
                t = torch.from_numpy(np.zeros(0, dtype=arr.dtype)).dtype
                self.extra[name[6:]] = (self.buffer[o:o + arr.nbytes].view(t)
                                        .view(arr.shape) if arr.size else None)
            else:
                setattr(s, name, base + o)
        host[struct_off:] = np.frombuffer(bytes(s), dtype=np.uint8)
        # the pinned staging buffer stays referenced until the copy has run
        self.buffer.copy_(pinned, non_blocking=True)
        self._staging = pinned
        for o, a, nbytes in dev_parts:
            self.buffer[o:o + nbytes].copy_(a.view(torch.uint8).reshape(-1))
        self.cstruct = s
        self.dev_ptr = base + struct_off

    @property
    def n_elem(self):
        return self.tables["n_hier"] * self.tables["n_state"]


# Hierarchies at least this large are built on the GPU when they have no
# static filters (build_tables_triangular); smaller ones on the host.
GPU_BUILD_MIN_AUX = 4096


def hierarchy_structure(system, hierarchy_param, device):
    """(hierarchy, DeviceStructure) of the non-adaptive basis of a trajectory or
    ensemble: all states, all modes, the triangular hierarchy with the static
    filters of hierarchy_param."""
    from .hierarchy import TriangularHierarchy, triangular_basis
    from . import _lib
    dev = torch.device(device)
    depth = int(hierarchy_param["MAXHIER"])
    filters = hierarchy_param.get("STATIC_FILTERS", [])
    if (dev.type == "cuda" and not filters and depth <= int(_lib.lib().hops_tri_max_depth())
            and comb(system.n_mode + depth, depth) >= GPU_BUILD_MIN_AUX):
        h = TriangularHierarchy(system.n_mode, depth)
        return h, DeviceStructure(build_tables_triangular(system, depth, dev), dev)
    basis = triangular_basis(system.n_mode, depth, filters)
    return basis, DeviceStructure(build_tables(system, basis), dev)
