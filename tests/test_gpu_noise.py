"""GPU FP64 noise filter against the oracle (same FP64 arithmetic, 1e-10) and
against the reference's complex64 output (which carries float32 FFT / angle /
abs artifacts of numpy 2, so 1e-6 relative)."""
import numpy as np
import pytest

from conftest import golden_system, load_golden
from oracle import hops_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model", ["SUM_GAUSSIAN", "BOX_MULLER"])
def test_filter_matches_oracle_fp64(cuda_device, model):
    from mesohops_b200.noise import filter_on_device
    f = load_golden("noise_dimer")
    t = O.noise_t_axis(float(f["tlen"]), float(f["tau"]))
    gw = [[g, w] for g, w in zip(f["G"], f["W"])]
    alpha = O.alpha_by_lop(t, gw, [0, 1], 2)
    raw = f[model + "_raw"]
    out64, nneg = filter_on_device(alpha, raw, cuda_device)
    gpu = out64.cpu().numpy()
    ora = O.correlated_noise(np.complex64(alpha), raw, fp64=True)
    assert np.max(np.abs(gpu - ora)) <= 1e-6 * np.max(np.abs(ora))  # complex64 storage
    ref = f[model + "_eta"]
    assert np.max(np.abs(gpu - ref)) <= 1e-6 * np.max(np.abs(ref))
    assert nneg > 0  # the reference warns about clipped values for this bath too


def test_filter_fp64_output_tight(cuda_device):
    """complex128 output of the C ABI equals the FP64 oracle to 1e-10."""
    import ctypes as C
    import torch
    from mesohops_b200 import _lib
    rng = np.random.default_rng(3)
    n_t = 257
    t = np.arange(n_t) * 1.0
    gw = [[O.dl_to_exp(40.0, 60.0, 300.0)[0], 60.0], [O.dl_to_exp(10.0, 300.0, 300.0)[0], 300.0]]
    alpha = O.alpha_by_lop(t, gw, [0, 1], 2)
    raw = (rng.normal(size=(2, 2 * (n_t - 1))) + 1j * rng.normal(size=(2, 2 * (n_t - 1)))).astype(np.complex64)
    L = _lib.lib()
    a = torch.from_numpy(alpha).to(cuda_device)
    z = torch.from_numpy(raw).to(cuda_device)
    work = torch.empty(int(L.hops_noise_filter_work_doubles(2, n_t)), dtype=torch.float64, device=cuda_device)
    out = torch.empty((2, n_t), dtype=torch.complex128, device=cuda_device)
    nneg = C.c_int64(0)
    rc = L.hops_noise_filter(a.data_ptr(), z.data_ptr(), 2, n_t, work.data_ptr(), out.data_ptr(),
                             None, C.byref(nneg), torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "hops_noise_filter")
    ora = O.correlated_noise(np.complex64(alpha), raw, fp64=True)
    gpu = out.cpu().numpy()
    assert np.max(np.abs(gpu - ora)) <= 1e-10 * np.max(np.abs(ora))


def test_fft_filter_trajectory_noise(cuda_device):
    """HopsTrajectory with FFT_FILTER noise: the device noise equals the oracle."""
    from mesohops_b200 import HopsTrajectory
    f = load_golden("c1_dimer")
    hops = HopsTrajectory(golden_system(f), noise_param={"SEED": 0, "MODEL": "FFT_FILTER",
                                                         "TLEN": 1004.0, "TAU": 2.0},
                          hierarchy_param={"MAXHIER": 2})
    hops.initialize(f["psi0"])
    n = hops.noise1.host()
    t = O.noise_t_axis(1004.0, 2.0)
    gw = [[g, w] for g, w in zip(f["G"], f["W"])]
    ref = O.fft_filter_noise(t, gw, [0, 1], 2, O.raw_draws(0, [0, 1], len(t)), fp64=True)
    assert np.max(np.abs(n - ref)) <= 1e-6 * np.max(np.abs(ref))
    hops.propagate(40.0, 4.0)
    assert np.all(np.isfinite(hops.phi))


def test_shared_alpha_filter_equals_tiled(cuda_device):
    """Rows that share correlation functions (an ensemble's trajectories) give
    bit for bit what the filter gives on alpha tiled to every row, and the same
    clip count."""
    import ctypes as C
    import torch
    from mesohops_b200 import _lib
    from mesohops_b200.noise import filter_on_device
    f = load_golden("noise_dimer")
    t = O.noise_t_axis(float(f["tlen"]), float(f["tau"]))
    gw = [[g, w] for g, w in zip(f["G"], f["W"])]
    alpha = O.alpha_by_lop(t, gw, [0, 1], 2)
    n_t = alpha.shape[1]
    rng = np.random.default_rng(11)
    B = 5
    raw = (rng.normal(size=(2 * B, 2 * (n_t - 1)))
           + 1j * rng.normal(size=(2 * B, 2 * (n_t - 1)))).astype(np.complex64)
    shared, n_shared = filter_on_device(alpha, raw, cuda_device)
    L = _lib.lib()
    dev = torch.device(cuda_device)
    a = torch.from_numpy(np.ascontiguousarray(np.tile(alpha, (B, 1)))).to(dev)
    z = torch.from_numpy(raw).to(dev)
    work = torch.empty(int(L.hops_noise_filter_work_doubles(2 * B, n_t)), dtype=torch.float64,
                       device=dev)
    out = torch.empty((2 * B, n_t), dtype=torch.complex64, device=dev)
    nneg = C.c_int64(0)
    rc = L.hops_noise_filter(a.data_ptr(), z.data_ptr(), 2 * B, n_t, work.data_ptr(), None,
                             out.data_ptr(), C.byref(nneg), torch.cuda.current_stream(dev).cuda_stream)
    assert rc == 0
    assert torch.equal(shared, out)
    assert n_shared == nneg.value
