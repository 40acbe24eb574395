"""The host-array C ABI and its binding to MesoHOPS objects.

CPU (no GPU needed): the description a reference HopsTrajectory is turned into
encodes exactly the reference's own super-operators K2_k, K2_kp1, K2_km1 and
Z2_kp1 (eom/eom_hops_ksuper.py:36-230) and equals the description built from
this package's own system and hierarchy; hops_structure_upload refuses bad
descriptions before it allocates anything.

GPU: structures uploaded from host arrays carry the same tables as the
package's Python builder, batches created and driven through host buffers only
reproduce the reference fixtures, and -- where the reference package is
installed beside the repository (baseline/_ref) -- the reference's own
HopsTrajectory.propagate with the B200 step attached at its integrator seam
reproduces the reference's own RK4 run.
"""
import contextlib
import ctypes as C
import io
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, golden_system, load_golden

FIXTURES = ["ring6", "general_lop", "dod", "chain4_2mode", "ltc_ring6", "c1_dimer"]


def _reference_module():
    """The reference package: the source tree in this container, or an
    installed copy under baseline/_ref; None when neither exists."""
    for path in (os.environ.get("MESOHOPS_SRC", "/root/reference/src"),
                 os.path.join(ROOT, "baseline", "_ref")):
        if os.path.isdir(os.path.join(path, "mesohops")):
            if path not in sys.path:
                sys.path.append(path)
            try:
                from mesohops.trajectory.hops_trajectory import HopsTrajectory
                return HopsTrajectory
            except Exception:
                return None
    return None


def _reference_trajectory(name, noise=None):
    RefTraj = _reference_module()
    if RefTraj is None:
        pytest.skip("reference package not available")
    from mesohops.trajectory.exp_noise import bcf_exp
    f = load_golden(name)
    sysp = golden_system(f)
    sysp["ALPHA_NOISE1"] = bcf_exp
    noise_param = {"SEED": 0, "MODEL": "FFT_FILTER", "TLEN": float(f["tlen"]),
                   "TAU": float(f["tau_noise"])}
    if noise is not None:
        import tempfile
        path = os.path.join(tempfile.mkdtemp(), "noise1.npy")
        np.save(path, noise)
        noise_param = {"SEED": path, "MODEL": "PRE_CALCULATED", "TLEN": float(f["tlen"]),
                       "TAU": float(f["tau_noise"])}
    h = RefTraj(sysp, noise_param=noise_param, hierarchy_param={"MAXHIER": int(f["depth"])},
                eom_param={"EQUATION_OF_MOTION": str(f["eom"])}, storage_param={})
    with contextlib.redirect_stdout(io.StringIO()):
        h.initialize(f["psi0"])
    return f, h


def _own_description(f):
    from mesohops_b200.hierarchy import triangular_basis
    from mesohops_b200.reference_binding import desc_arrays
    from mesohops_b200.system import HopsSystem
    sysm = HopsSystem(golden_system(f))
    return desc_arrays(sysm, triangular_basis(sysm.n_mode, int(f["depth"])))


# --------------------------------------------------------------------- CPU
@pytest.mark.parametrize("name", FIXTURES)
def test_description_encodes_the_reference_super_operators(name):
    from mesohops_b200.reference_binding import desc_arrays_from_reference, super_operators
    f, h = _reference_trajectory(name)
    d = desc_arrays_from_reference(h)
    k2_k, kp1, km1, z2 = super_operators(d)
    eom = h.basis.eom
    assert abs(k2_k - eom.K2_k).max() == 0
    assert abs(kp1 - eom.K2_kp1).max() <= 1e-13 * abs(eom.K2_kp1).max()
    assert abs(km1 - eom.K2_km1).max() <= 1e-13 * abs(eom.K2_km1).max()
    assert len(z2) == len(eom.Z2_kp1)
    for a, b in zip(z2, eom.Z2_kp1):
        assert abs(a - b).max() <= 1e-13 * max(abs(b).max(), 1.0)


@pytest.mark.parametrize("name", FIXTURES)
def test_own_description_equals_the_reference_one(name):
    from mesohops_b200.reference_binding import desc_arrays_from_reference
    f, h = _reference_trajectory(name)
    ref = desc_arrays_from_reference(h)
    own = _own_description(f)
    for k, v in ref.items():
        if v is None or own[k] is None:
            assert v is None and own[k] is None, k
        else:
            assert np.array_equal(np.asarray(v), np.asarray(own[k])), k


def _desc_struct(d):
    from mesohops_b200 import _lib
    desc = _lib.HopsStructureDesc()
    desc.n_hier, desc.n_state, desc.n_mode, desc.n_lop = (d["n_hier"], d["n_state"],
                                                          d["n_mode"], d["n_lop"])
    for k in ("up_ptr", "up_aux", "up_mode", "dn_ptr", "dn_aux", "dn_mode", "dn_k",
              "mode_lop", "mode_g", "mode_w", "lops", "hamiltonian", "lt_coef"):
        a = d[k]
        setattr(desc, k, a.ctypes.data if a is not None and a.size else None)
    return desc


def test_upload_refuses_bad_descriptions_before_allocating():
    """Validation runs on the host before any CUDA call (no GPU needed)."""
    from mesohops_b200 import _lib
    L = _lib.lib()
    d = _own_description(load_golden("ring6"))
    h = C.c_void_p()
    cases = []
    bad = dict(d, n_hier=0)
    cases.append((bad, b"bad sizes"))
    up = d["up_aux"].copy()
    up[3] = d["n_hier"] + 5
    cases.append((dict(d, up_aux=up), b"up connection 3 out of range"))
    w = d["mode_w"].copy()
    w[2] = 0.0
    cases.append((dict(d, mode_w=w), b"w = 0"))
    ml = d["mode_lop"].copy()
    ml[1] = d["n_lop"]
    cases.append((dict(d, mode_lop=ml), b"L index"))
    for dd, text in cases:
        keep = dd   # the arrays stay alive during the call
        rc = L.hops_structure_upload(C.byref(_desc_struct(keep)), None, C.byref(h))
        assert rc == _lib.HOPS_EINVAL
        assert text in L.hops_last_error(), (text, L.hops_last_error())
        assert not h.value


# --------------------------------------------------------------------- GPU
def _read(ptr, n, dtype):
    """n elements of dtype at a device address, copied to the host."""
    import torch
    if n == 0:
        return np.zeros(0, dtype=dtype)

    class Dev:
        __cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str,
                                    "data": (int(ptr), False), "version": 3}
    return torch.as_tensor(Dev(), device="cuda").cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ring6", "general_lop", "ltc_ring6", "dod"])
def test_uploaded_tables_equal_the_python_tables(cuda_device, name):
    """Every table hops_structure_upload derives equals, bit for bit, the one
    the package's Python builder uploads."""
    from mesohops_b200.device import DeviceStructure, build_tables
    from mesohops_b200.hierarchy import triangular_basis
    from mesohops_b200.reference_binding import HostStructure
    from mesohops_b200.system import HopsSystem
    f = load_golden(name)
    sysm = HopsSystem(golden_system(f))
    basis = triangular_basis(sysm.n_mode, int(f["depth"]))
    py = DeviceStructure(build_tables(sysm, basis), "cuda:0")
    hs = HostStructure(_own_description(f))
    a, b = py.cstruct, hs.host_view.contents
    for k in ("n_hier", "n_state", "n_mode", "n_lop", "n_first", "n_up", "n_dn",
              "site_projector", "max_up", "max_dn"):
        assert getattr(a, k) == getattr(b, k), k
    S, N, M, L = a.n_state, a.n_hier, a.n_mode, a.n_lop
    sizes = {  # field -> (element count, dtype)
        "k_decay": (2 * N, np.float64), "k_decay_f": (2 * N, np.float32),
        "up_ptr": (N + 1, np.int32), "up_aux": (a.n_up, np.int32), "up_mode": (a.n_up, np.int32),
        "dn_ptr": (N + 1, np.int32), "dn_aux": (a.n_dn, np.int32), "dn_mode": (a.n_dn, np.int32),
        "dn_coef": (2 * a.n_dn, np.float64), "dn_coef_f": (2 * a.n_dn, np.float32),
        "mode_lop": (M, np.int32), "mode_g": (2 * M, np.float64), "mode_w": (2 * M, np.float64),
        "mode_gw": (2 * M, np.float64), "mode_gw_f": (2 * M, np.float32),
        "first_aux": (a.n_first, np.int32), "first_mode": (a.n_first, np.int32),
        "l_ptr": (L * (S + 1), np.int32), "lh_ptr": (L * (S + 1), np.int32),
        "lop_active": (L, np.int32), "lop_site": (L, np.int32), "lop_sval": (2 * L, np.float64),
        "h_ptr": (S + 1, np.int32), "mode_site": (M, np.int32),
        "mode_gwv": (2 * M, np.float64), "dn_coef_site": (2 * a.n_dn, np.float64),
        "up_site": (a.n_up, np.int32), "dn_site": (a.n_dn, np.int32),
    }
    for k, (n, dt) in sizes.items():
        x, y = _read(getattr(a, k), n, dt), _read(getattr(b, k), n, dt)
        assert np.array_equal(x, y), k
    lptr = _read(a.l_ptr, L * (S + 1), np.int32)
    nl = int(lptr[-1]) if L else 0
    hptr = _read(a.h_ptr, S + 1, np.int32)
    nh = int(hptr[-1])
    for k, n, dt in (("l_col", nl, np.int32), ("l_val", 2 * nl, np.float64),
                     ("lh_col", nl, np.int32), ("lh_val", 2 * nl, np.float64),
                     ("h_col", nh, np.int32), ("h_val", 2 * nh, np.float64)):
        assert np.array_equal(_read(getattr(a, k), n, dt), _read(getattr(b, k), n, dt)), k
    assert bool(a.h_diag) == bool(b.h_diag)
    if a.h_diag:
        assert np.array_equal(_read(a.h_diag, 2 * S, np.float64), _read(b.h_diag, 2 * S, np.float64))
    assert bool(a.lt_coef) == bool(b.lt_coef)
    if a.lt_coef:
        assert np.array_equal(_read(a.lt_coef, 2 * L, np.float64), _read(b.lt_coef, 2 * L, np.float64))
    hs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name,B,precision", [("ring6", 3, "complex128"),
                                              ("ring6", 40, "complex128"),
                                              ("general_lop", 5, "complex128"),
                                              ("ltc_ring6", 2, "complex128"),
                                              ("c1_dimer", 1, "complex128"),
                                              ("ring6", 40, "mixed")])
def test_host_arrays_only_reproduce_the_reference(cuda_device, name, B, precision):
    """Structure, batch, state, noise and psi(t) through host buffers only."""
    from mesohops_b200.constants import hbar
    from mesohops_b200.reference_binding import HostBatch, HostStructure
    f = load_golden(name)
    hs = HostStructure(_own_description(f))
    hb = HostBatch(hs, B, precision, str(f["eom"]))
    N, S = int(f["n_hier"]), int(f["n_state"])
    phi0 = np.zeros((B, N * S), dtype=np.complex128)
    phi0[:, :S] = f["psi0"]
    hb.set_state(phi0)
    n2 = f["noise2"] if np.any(f["noise2"] != 0) else None
    hb.set_noise(np.repeat(f["noise1"][None], B, 0),
                 np.repeat(n2[None], B, 0) if n2 is not None else None)
    dt = float(f["dt"])
    di = int(round(dt * 0.5 / float(f["tau_noise"])))
    n = len(f["psi_traj"]) - 1
    psi, status = hb.propagate(0, di, n, dt / hbar)
    assert not np.any(status)
    ref = f["psi_traj"][1:]
    tol = 1e-10 if precision == "complex128" else 1e-5
    for b in range(B):
        if precision == "complex128":
            assert np.max(np.abs(psi[:, b] - ref)) <= tol * np.max(np.abs(ref))
        else:
            assert np.max(np.abs(np.abs(psi[:, b]) ** 2 - np.abs(ref) ** 2)) <= tol
    phi, z = hb.get_state()
    if precision == "complex128":
        assert np.max(np.abs(phi - f["phi_end"][None])) <= 1e-10 * np.max(np.abs(f["phi_end"]))
        assert np.max(np.abs(z - f["zmem_end"][None])) <= 1e-10 * max(1.0, np.max(np.abs(f["zmem_end"])))
    hb.close()
    hs.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ring6", "general_lop", "c1_dimer"])
def test_reference_trajectory_with_the_b200_step(cuda_device, name):
    """The reference's own HopsTrajectory, its step replaced at the integrator
    seam by the B200 step, equals the same trajectory with the reference's RK4
    step (identical precomputed noise)."""
    from mesohops_b200.reference_binding import attach
    f = load_golden(name)
    runs = []
    for use in (False, True):
        _, h = _reference_trajectory(name, noise=f["noise1"])
        if use:
            attach(h)
        with contextlib.redirect_stdout(io.StringIO()):
            h.propagate(float(f["t_max"]), float(f["dt"]))
        runs.append(np.array(h.storage.data["psi_traj"]))
    ref, b200 = runs
    assert np.max(np.abs(b200 - ref)) <= 1e-10 * np.max(np.abs(ref))
