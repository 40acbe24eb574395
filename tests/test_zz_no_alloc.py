"""The no-allocation RK4 entry point (hops_rk4_propagate_noalloc).

It exists for callers that cannot allocate device memory while they step a
trajectory -- hosts whose own pool owns the GPU's memory, or per-step
callbacks that must not synchronise the device -- and keeps its scratch in a
static device array instead.  These tests call it through the C ABI and check
that two calls in a row give the same states and psi trajectories as the
regular entry point (hops_rk4_propagate with caller-allocated buffers), that
calls of different shapes in a row cannot see each other's left-overs, that
free device memory does not change across a call, that a non-finite flag
survives later calls until the caller clears it, that a rejected call changes
nothing, and that an oversized request is refused.  This file is collected
last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_system, load_golden

pytestmark = pytest.mark.gpu


def _setup(precision, B, name="ring6"):
    import torch
    from mesohops_b200.device import DeviceStructure, build_tables
    from mesohops_b200.engine import StreamBatch
    from mesohops_b200.hierarchy import triangular_basis
    from mesohops_b200.system import HopsSystem
    f = load_golden(name)
    sysm = HopsSystem(golden_system(f))
    basis = triangular_basis(sysm.n_mode, int(f["depth"]))
    ds = DeviceStructure(build_tables(sysm, basis), "cuda:0")
    n_l, n_t = f["noise1"].shape
    rng = np.random.default_rng(21)
    noise = ((rng.normal(size=(B, n_l, n_t)) + 1j * rng.normal(size=(B, n_l, n_t))) * 30
             ).astype(np.complex64)
    phi0 = np.zeros((B, basis.n_hier * sysm.n_state), dtype=np.complex128)
    phi0[:, :sysm.n_state] = f["psi0"]
    ref = StreamBatch(ds, B, precision)
    ref.set_state(phi0, np.zeros((B, sysm.n_mode)))
    nz = torch.from_numpy(noise).to("cuda:0")
    ref.set_noise(nz)
    return f, ds, ref, nz, phi0


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-10), ("mixed", 1e-10)])
def test_noalloc_matches_regular_entry_point_twice(cuda_device, precision, tol):
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.constants import hbar
    from mesohops_b200.engine import precision_code
    B = 40
    f, ds, ref, nz, phi0 = _setup(precision, B)
    L = _lib.lib()
    prec = precision_code(precision)
    S = ds.tables["n_state"]
    dt = float(f["dt"])
    di = int(round(dt * 0.5 / float(f["tau_noise"])))
    n = 6
    # the caller's own buffers: state, memory, outputs
    phi = ref.phi.clone()
    zmem = torch.zeros_like(ref.zmem)
    status = torch.zeros(B, dtype=torch.int32, device="cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    assert L.hops_noalloc_scratch_bytes(C.byref(ds.cstruct), B, prec) <= (64 << 20)
    for call in range(2):
        it0 = 2 * n * di * call
        psi_ref = torch.empty((n, B, S), dtype=torch.complex128, device="cuda:0")
        ref.propagate(it0, di, n, dt / hbar, psi_out=psi_ref)
        psi = torch.empty((n, B, S), dtype=torch.complex128, device="cuda:0")
        rc = L.hops_rk4_propagate_noalloc(C.byref(ds.cstruct), B, prec, 0, phi.data_ptr(),
                                          zmem.data_ptr(), nz.data_ptr(), nz.shape[-1], None, 0,
                                          it0, di, n, dt / hbar, psi.data_ptr(),
                                          status.data_ptr(), stream)
        _lib.check(rc, "hops_rk4_propagate_noalloc")
        torch.cuda.synchronize()
        assert int(status.abs().sum()) == 0
        a, b = psi.cpu().numpy(), psi_ref.cpu().numpy()
        assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b))
        pa = phi.to(torch.complex128).cpu().numpy()
        pb = ref.phi.to(torch.complex128).cpu().numpy()
        assert np.max(np.abs(pa - pb)) <= tol * np.max(np.abs(pb))
        za, zb = zmem.cpu().numpy(), ref.zmem.cpu().numpy()
        assert np.max(np.abs(za - zb)) <= tol * max(1.0, np.max(np.abs(zb)))


def test_noalloc_rejects_oversized_request(cuda_device):
    import torch
    from mesohops_b200 import _lib
    f, ds, ref, nz, phi0 = _setup("complex128", 1, name="chain4_2mode")
    L = _lib.lib()
    B = 1 << 16   # far beyond the static scratch for this structure
    assert L.hops_noalloc_scratch_bytes(C.byref(ds.cstruct), B, 0) > (64 << 20)
    dummy = torch.zeros(4, dtype=torch.complex128, device="cuda:0")
    status = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    rc = L.hops_rk4_propagate_noalloc(C.byref(ds.cstruct), B, 0, 0, dummy.data_ptr(),
                                      dummy.data_ptr(), None, 0, None, 0, 0, 1, 1, 0.001,
                                      None, status.data_ptr(), None)
    assert rc == _lib.HOPS_EINVAL
    assert b"static area" in L.hops_last_error()


def _noalloc(L, ds, B, prec, phi, zmem, nz, it0, di, n, h, psi, status, n_t=None):
    import torch
    return L.hops_rk4_propagate_noalloc(
        C.byref(ds.cstruct), B, prec, 0, phi.data_ptr(), zmem.data_ptr(), nz.data_ptr(),
        nz.shape[-1] if n_t is None else n_t, None, 0, it0, di, n, h,
        psi.data_ptr() if psi is not None else None, status.data_ptr(),
        torch.cuda.current_stream().cuda_stream)


def _one_call_vs_regular(name, B, precision, tol):
    """One no-allocation call against the regular entry point from the same state."""
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.constants import hbar
    from mesohops_b200.engine import precision_code
    f, ds, ref, nz, phi0 = _setup(precision, B, name=name)
    L = _lib.lib()
    prec = precision_code(precision)
    S = ds.tables["n_state"]
    dt = float(f["dt"])
    di = int(round(dt * 0.5 / float(f["tau_noise"])))
    n = 5
    phi = ref.phi.clone()
    zmem = torch.zeros_like(ref.zmem)
    status = torch.zeros(B, dtype=torch.int32, device="cuda:0")
    psi_ref = torch.empty((n, B, S), dtype=torch.complex128, device="cuda:0")
    ref.propagate(0, di, n, dt / hbar, psi_out=psi_ref)
    psi = torch.empty((n, B, S), dtype=torch.complex128, device="cuda:0")
    _lib.check(_noalloc(L, ds, B, prec, phi, zmem, nz, 0, di, n, dt / hbar, psi, status),
               "hops_rk4_propagate_noalloc")
    torch.cuda.synchronize()
    assert int(status.abs().sum()) == 0
    a, b = psi.cpu().numpy(), psi_ref.cpu().numpy()
    assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b)), name
    pa = phi.to(torch.complex128).cpu().numpy()
    pb = ref.phi.to(torch.complex128).cpu().numpy()
    assert np.max(np.abs(pa - pb)) <= tol * np.max(np.abs(pb)), name


@pytest.mark.parametrize("precision", ["complex128", "mixed"])
def test_noalloc_calls_of_different_shapes_in_a_row(cuda_device, precision):
    """A large call, a smaller call on another structure, then the large one
    again: left-overs of one call in the shared array never reach the next."""
    for name, B in (("ring6", 40), ("chain4_2mode", 8), ("ring6", 40)):
        _one_call_vs_regular(name, B, precision, 1e-10)


def test_noalloc_allocates_no_device_memory(cuda_device):
    """Free device memory is the same before and after a call (after a first
    call has loaded the module that holds the static array)."""
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.constants import hbar
    from mesohops_b200.engine import precision_code
    B = 40
    f, ds, ref, nz, phi0 = _setup("mixed", B)
    L = _lib.lib()
    prec = precision_code("mixed")
    dt = float(f["dt"])
    di = int(round(dt * 0.5 / float(f["tau_noise"])))
    phi = ref.phi.clone()
    zmem = torch.zeros_like(ref.zmem)
    status = torch.zeros(B, dtype=torch.int32, device="cuda:0")
    psi = torch.empty((3, B, ds.tables["n_state"]), dtype=torch.complex128, device="cuda:0")
    _lib.check(_noalloc(L, ds, B, prec, phi, zmem, nz, 0, di, 3, dt / hbar, psi, status), "warm")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    _lib.check(_noalloc(L, ds, B, prec, phi, zmem, nz, 6 * di, di, 3, dt / hbar, psi, status),
               "measured")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_status_flag_survives_later_calls(cuda_device):
    """A trajectory whose state turns non-finite in one call keeps its
    HOPS_ENONFINITE word through a later clean call when the caller reads the
    status only at the end; the other trajectories stay clean and equal the
    regular entry point."""
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.constants import hbar
    from mesohops_b200.engine import precision_code
    B, bad = 40, 7
    f, ds, ref, nz, phi0 = _setup("complex128", B)
    L = _lib.lib()
    prec = precision_code("complex128")
    S = ds.tables["n_state"]
    dt = float(f["dt"])
    di = int(round(dt * 0.5 / float(f["tau_noise"])))
    n = 4
    phi = ref.phi.clone()
    clean = phi[:, :, bad].clone()
    phi[0, 0, bad] = float("nan")           # host-side injection into one trajectory
    zmem = torch.zeros_like(ref.zmem)
    status = torch.zeros(B, dtype=torch.int32, device="cuda:0")
    psi = torch.empty((n, B, S), dtype=torch.complex128, device="cuda:0")
    psi_ref = torch.empty((n, B, S), dtype=torch.complex128, device="cuda:0")
    _lib.check(_noalloc(L, ds, B, prec, phi, zmem, nz, 0, di, n, dt / hbar, psi, status), "1")
    ref.propagate(0, di, n, dt / hbar, psi_out=psi_ref)
    # the caller repairs the trajectory without reading the status, then steps on
    phi[:, :, bad] = clean
    zmem[bad].zero_()
    _lib.check(_noalloc(L, ds, B, prec, phi, zmem, nz, 2 * n * di, di, n, dt / hbar, psi,
                        status), "2")
    ref.propagate(2 * n * di, di, n, dt / hbar, psi_out=psi_ref)
    torch.cuda.synchronize()
    st = status.cpu().numpy()
    assert st[bad] == _lib.HOPS_ENONFINITE
    assert np.count_nonzero(st) == 1
    keep = [b for b in range(B) if b != bad]
    a = psi.cpu().numpy()[:, keep]
    b = psi_ref.cpu().numpy()[:, keep]
    assert np.array_equal(a, b)


def test_noalloc_rejected_call_changes_nothing(cuda_device):
    """A call refused by its argument checks (noise axis too short) launches
    nothing: state, memory and status words are as before."""
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.constants import hbar
    from mesohops_b200.engine import precision_code
    B = 40
    f, ds, ref, nz, phi0 = _setup("mixed", B)
    L = _lib.lib()
    prec = precision_code("mixed")
    dt = float(f["dt"])
    di = int(round(dt * 0.5 / float(f["tau_noise"])))
    phi = ref.phi.clone()
    zmem = torch.ones_like(ref.zmem)
    status = torch.zeros(B, dtype=torch.int32, device="cuda:0")
    status[3] = _lib.HOPS_ENONFINITE
    before = (phi.clone(), zmem.clone(), status.clone())
    rc = _noalloc(L, ds, B, prec, phi, zmem, nz, 0, di, 8, dt / hbar, None, status, n_t=4)
    torch.cuda.synchronize()
    assert rc == _lib.HOPS_EINVAL
    assert b"noise 1 too short" in L.hops_last_error()
    for x, y in zip((phi, zmem, status), before):
        assert torch.equal(x, y)
