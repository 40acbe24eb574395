"""Binding of the host-array C ABI to MesoHOPS objects.

``desc_arrays`` turns a basis of this package (HopsSystem x AuxBasis) and
``desc_arrays_from_reference`` a reference ``HopsTrajectory`` (its
``basis.system``, ``basis.mode`` and ``basis.hierarchy``) into the arrays of
``hops_structure_desc`` (include/hops_b200.h): the aux connection lists, the
modes, the relative L list and H in the state basis.  ``HostStructure`` and
``HostBatch`` own the library-side objects made from them
(hops_structure_upload / hops_batch_create) and move states, noise and psi(t)
through host buffers only -- what a caller in any language with a C FFI does.

``B200Step`` is the drop-in for the reference's integrator seam: the pair
(step, integration_var) chosen by ``INTEGRATION_DICT["INTEGRATOR"]`` at
trajectory/hops_trajectory.py:235-243.  It has the signature of
``runge_kutta_step`` (integrator/integrator_rk.py:10-75),
``step(dsystem_dt, phi, z_mem, z_rnd, z_rnd2, tau) -> (phi, z_mem)``, and takes
the noise samples ``runge_kutta_variables`` prepared, so noise handling
(including EFFECTIVE_NOISE_INTEGRATION) stays the reference's; ``attach``
installs it on a reference trajectory with a non-adaptive basis.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sps

from . import _lib
from .constants import hbar


def _cplx(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def desc_arrays(system, basis):
    """Description of the full state basis of ``system`` (a HopsSystem) over the
    modes and aux of ``basis`` (an AuxBasis of mesohops_b200.hierarchy)."""
    modes = np.asarray(basis.modes, dtype=np.int64)
    l_abs = np.array(sorted(set(int(system.l_by_mode[m]) for m in modes)), dtype=np.int64)
    rel = {int(j): i for i, j in enumerate(l_abs)}
    states = np.arange(system.n_state)
    lops = np.array([system.lop_block(j, states) for j in l_abs], dtype=np.complex128)
    lt = np.asarray(getattr(system, "lt_coef", np.zeros(system.n_lop)))[l_abs] if len(l_abs) else None
    return dict(
        n_hier=int(basis.n_hier), n_state=int(system.n_state), n_mode=len(modes),
        n_lop=len(l_abs),
        up_ptr=_i32(basis.up_ptr), up_aux=_i32(basis.up_u), up_mode=_i32(basis.up_m),
        dn_ptr=_i32(basis.dn_ptr), dn_aux=_i32(basis.dn_d), dn_mode=_i32(basis.dn_m),
        dn_k=_i32(basis.dn_k),
        mode_lop=_i32([rel[int(system.l_by_mode[m])] for m in modes]),
        mode_g=_cplx(system.G[modes]), mode_w=_cplx(system.W[modes]),
        lops=_cplx(lops).reshape(len(l_abs), system.n_state, system.n_state),
        hamiltonian=_cplx(system.hamiltonian_dense()),
        lt_coef=_cplx(lt) if lt is not None and np.any(lt != 0) else None)


def desc_arrays_from_reference(hops):
    """Description of the current basis of a reference HopsTrajectory (after
    ``initialize``): aux connections from the aux vectors' ``dict_aux_p1`` /
    ``dict_aux_m1`` (basis/hops_aux.py:386-414, 576-582), modes from
    ``basis.mode`` (basis/hops_modes.py:47-171), H in the state basis from
    ``basis.system`` and the low-temperature coefficients LIST_LT_PARAM of the
    relative L list (basis/system_functions.py:115-133)."""
    b = hops.basis
    mode = b.mode
    abs_modes = [int(m) for m in mode.list_absindex_mode]
    rel_mode = {m: i for i, m in enumerate(abs_modes)}
    aux_list = list(b.hierarchy.auxiliary_list)
    N = len(aux_list)
    up_ptr, up_aux, up_mode = [0], [], []
    dn_ptr, dn_aux, dn_mode, dn_k = [0], [], [], []
    for a in sorted(aux_list, key=lambda x: x._index):
        for m, u in sorted(a.dict_aux_p1.items()):
            if m in rel_mode:
                up_aux.append(u._index)
                up_mode.append(rel_mode[m])
        up_ptr.append(len(up_aux))
        for m, d in sorted(a.dict_aux_m1.items()):
            if m in rel_mode:
                dn_aux.append(d._index)
                dn_mode.append(rel_mode[m])
                dn_k.append(int(a[m]))
        dn_ptr.append(len(dn_aux))
    S = len(b.system.state_list)
    lops = np.array([sps.coo_matrix(l).toarray() for l in mode.list_L2_coo],
                    dtype=np.complex128).reshape(-1, S, S)
    H = b.system.hamiltonian
    H = H.toarray() if sps.issparse(H) else np.asarray(H)
    lt_all = b.system.param.get("LIST_LT_PARAM")
    lt = None
    if lt_all is not None:
        lt = np.array([lt_all[int(j)] for j in mode.list_absindex_L2], dtype=np.complex128)
        if not np.any(lt != 0):
            lt = None
    return dict(
        n_hier=N, n_state=S, n_mode=len(abs_modes), n_lop=len(lops),
        up_ptr=_i32(up_ptr), up_aux=_i32(up_aux), up_mode=_i32(up_mode),
        dn_ptr=_i32(dn_ptr), dn_aux=_i32(dn_aux), dn_mode=_i32(dn_mode), dn_k=_i32(dn_k),
        mode_lop=_i32(mode.list_index_L2_by_hmode), mode_g=_cplx(mode.list_g),
        mode_w=_cplx(mode.list_w), lops=_cplx(lops), hamiltonian=_cplx(H),
        lt_coef=_cplx(lt) if lt is not None else None)


def super_operators(d):
    """K2_k, K2_kp1, K2_km1 and Z2_kp1 of a description, in the reference's
    form (eom/eom_hops_ksuper.py:36-230): a check that the description encodes
    the same equation of motion as the super-operators it replaces."""
    N, S, M = d["n_hier"], d["n_state"], d["n_mode"]
    W, G = d["mode_w"], d["mode_g"]
    k2_k = np.zeros(N, dtype=np.complex128)
    for a in range(N):
        for p in range(d["dn_ptr"][a], d["dn_ptr"][a + 1]):
            k2_k[a] -= d["dn_k"][p] * W[d["dn_mode"][p]]
    kp_r, kp_c, kp_v, km_v = [], [], [], []
    z = [([], [], []) for _ in range(d["n_lop"])]
    for a in range(N):
        for p in range(d["up_ptr"][a], d["up_ptr"][a + 1]):
            u, m = int(d["up_aux"][p]), int(d["up_mode"][p])
            j = int(d["mode_lop"][m])
            lm = d["lops"][j]
            # depth of u in mode m: one more than a's, read from u's down list
            ku = [d["dn_k"][q] for q in range(d["dn_ptr"][u], d["dn_ptr"][u + 1])
                  if d["dn_mode"][q] == m][0]
            for r, c in zip(*np.nonzero(lm)):
                kp_r.append(a * S + r)
                kp_c.append(u * S + c)
                kp_v.append(-(G[m] / W[m]) * lm[r, c])
                km_v.append(ku * W[m] * np.conj(lm[r, c]))
            z[j][0].append(a)
            z[j][1].append(u)
            z[j][2].append(G[m] / W[m])
    n = N * S
    kp1 = sps.coo_matrix((kp_v, (kp_r, kp_c)), shape=(n, n)).tocsr()
    km1 = sps.coo_matrix((km_v, (kp_c, kp_r)), shape=(n, n)).tocsr()
    z2 = [sps.coo_matrix((v, (r, c)), shape=(N, N)).tocsr() for r, c, v in z]
    return sps.diags(k2_k).tocsr(), kp1, km1, z2


class HostStructure:
    """hops_structure_upload of a description (library-owned device memory)."""

    def __init__(self, d, stream=None):
        self.d = d
        desc = _lib.HopsStructureDesc()
        desc.n_hier, desc.n_state, desc.n_mode, desc.n_lop = (d["n_hier"], d["n_state"],
                                                              d["n_mode"], d["n_lop"])
        for k in ("up_ptr", "up_aux", "up_mode", "dn_ptr", "dn_aux", "dn_mode", "dn_k",
                  "mode_lop", "mode_g", "mode_w", "lops", "hamiltonian", "lt_coef"):
            a = d[k]
            setattr(desc, k, a.ctypes.data if a is not None and a.size else None)
        h = C.c_void_p()
        rc = _lib.lib().hops_structure_upload(C.byref(desc), stream, C.byref(h))
        _lib.check(rc, "hops_structure_upload")
        self.handle = h
        self.host_view = _lib.lib().hops_structure_host_view(h)
        self.device_view = _lib.lib().hops_structure_device_view(h)

    def close(self):
        if getattr(self, "handle", None):
            _lib.check(_lib.lib().hops_structure_destroy(self.handle), "hops_structure_destroy")
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostBatch:
    """hops_batch_create with host-buffer I/O (hops_batch_*_host)."""

    def __init__(self, structure, n_traj, precision="complex128", eom="NORMALIZED NONLINEAR",
                 stream=None):
        from .engine import precision_code
        self.s = structure
        self.B = int(n_traj)
        self.stream = stream
        d = structure.d
        self.N, self.S, self.M, self.L = d["n_hier"], d["n_state"], d["n_mode"], d["n_lop"]
        p = C.POINTER(_lib.HopsBatch)()
        rc = _lib.lib().hops_batch_create(structure.host_view, self.B, precision_code(precision),
                                          _lib.EOM_CODES[eom], C.byref(p))
        _lib.check(rc, "hops_batch_create")
        self.bt = p

    def set_state(self, phi, zmem=None):
        """phi [B, n_hier*n_state] complex, zmem [B, n_mode] complex or None."""
        ph = np.ascontiguousarray(np.asarray(phi, dtype=np.complex128).reshape(self.B, -1))
        z = (np.ascontiguousarray(np.asarray(zmem, dtype=np.complex128).reshape(self.B, self.M))
             if zmem is not None and self.M else None)
        rc = _lib.lib().hops_batch_set_state_host(self.s.host_view, self.bt, ph.ctypes.data,
                                                  z.ctypes.data if z is not None else None,
                                                  self.stream)
        _lib.check(rc, "hops_batch_set_state_host")

    def set_noise(self, noise1, noise2=None):
        """[B, n_lop, n_t] complex64 arrays (noise2 may be None)."""
        n1 = np.ascontiguousarray(np.asarray(noise1, dtype=np.complex64))
        n2 = np.ascontiguousarray(np.asarray(noise2, dtype=np.complex64)) if noise2 is not None else None
        self._noise = (n1, n2)
        rc = _lib.lib().hops_batch_set_noise_host(self.bt, n1.ctypes.data, n1.shape[-1],
                                                  n2.ctypes.data if n2 is not None else None,
                                                  n2.shape[-1] if n2 is not None else 0,
                                                  self.stream)
        _lib.check(rc, "hops_batch_set_noise_host")

    def propagate(self, it0, di, n_steps, tau_over_hbar):
        """Returns (psi [n_steps, B, n_state] complex128, status [B] int32)."""
        psi = np.empty((n_steps, self.B, self.S), dtype=np.complex128)
        status = np.empty(self.B, dtype=np.int32)
        rc = _lib.lib().hops_batch_propagate_host(self.s.host_view, self.bt, int(it0), int(di),
                                                  int(n_steps), float(tau_over_hbar),
                                                  psi.ctypes.data, status.ctypes.data,
                                                  self.stream)
        _lib.check(rc, "hops_batch_propagate_host")
        return psi, status

    def get_state(self):
        phi = np.empty((self.B, self.N * self.S), dtype=np.complex128)
        z = np.empty((self.B, max(self.M, 1)), dtype=np.complex128)
        rc = _lib.lib().hops_batch_get_state_host(self.s.host_view, self.bt, phi.ctypes.data,
                                                  z.ctypes.data if self.M else None, self.stream)
        _lib.check(rc, "hops_batch_get_state_host")
        return phi, z[:, :self.M]

    def close(self):
        if getattr(self, "bt", None):
            _lib.check(_lib.lib().hops_batch_destroy(self.bt), "hops_batch_destroy")
            self.bt = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class B200Step:
    """``runge_kutta_step`` on the GPU for one reference trajectory.

    Built from the trajectory's (non-adaptive) basis once; every call uploads
    phi, z_mem and the three noise samples of the step, runs one RK4 step in
    complex128 and returns (phi, z_mem) of the same types the reference step
    returns.  With NORMALIZED NONLINEAR the library renormalises the state
    after the step; the reference's own ``normalize`` that follows
    (hops_trajectory.py:466) then divides by a norm of 1 (to rounding)."""

    def __init__(self, hops, precision="complex128"):
        if hops.basis.adaptive:
            from .exceptions import UnsupportedRequest
            raise UnsupportedRequest("the B200 step with an adaptive basis", "B200Step")
        self.desc = desc_arrays_from_reference(hops)
        self.structure = HostStructure(self.desc)
        eom = hops.basis.eom.param["EQUATION_OF_MOTION"]
        self.batch = HostBatch(self.structure, 1, precision, eom)

    def __call__(self, dsystem_dt, phi, z_mem, z_rnd, z_rnd2, tau):
        sparse_z = sps.issparse(z_mem)
        z = np.asarray(z_mem.toarray()).ravel() if sparse_z else np.asarray(z_mem).ravel()
        self.batch.set_state(np.asarray(phi)[None], z[None])
        n1 = np.asarray(z_rnd, dtype=np.complex64)[None]
        n2 = np.asarray(z_rnd2, dtype=np.complex64)[None]
        self.batch.set_noise(n1, n2)
        _, status = self.batch.propagate(0, 1, 1, tau / hbar)
        if status[0] != 0:
            from .exceptions import TrajectoryError
            raise TrajectoryError("non-finite state in the B200 step")
        phi_new, z_new = self.batch.get_state()
        z_new = z_new[0]
        if sparse_z:
            z_new = type(z_mem)(z_new.reshape(-1, 1))
        return phi_new[0], z_new


def attach(hops, precision="complex128"):
    """Replace the integrator step of a reference HopsTrajectory (initialised,
    non-adaptive basis) by ``B200Step``; returns the step object."""
    step = B200Step(hops, precision)
    hops.step = step
    return step
