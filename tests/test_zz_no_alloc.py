"""The no-allocation RK4 entry point (hops_rk4_propagate_noalloc).

It exists for callers that cannot allocate device memory while they step a
trajectory -- hosts whose own pool owns the GPU's memory, or per-step
callbacks that must not synchronise the device -- and keeps its scratch in a
static device array instead.  These tests call it through the C ABI and check
that two calls in a row give the same states and psi trajectories as the
regular entry point (hops_rk4_propagate with caller-allocated buffers), and
that an oversized request is refused.  This file is collected last on purpose.
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
