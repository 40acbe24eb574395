"""The benchmark configurations themselves against reference runs.

c3_ring20 (the configuration the headline number is measured on): 20-site ring,
depth 4, 10626 aux x 20 states, 250 RK4 steps of 4 fs, with the reference's own
FFT-filtered noise of SEED 0..3 (fixture from tests/golden/make_golden.py
--bench-configs).  The GPU runs it as one batch of 128 trajectories -- the
batch shape of the benchmark, so the batched stage kernel in the shape the
autotuner picks for it -- each trajectory with one of the four reference noise
realisations; complex128 must match the reference to 1e-10 relative and the
mixed precision stay within 1e-5 absolute population error.

c2_chain10: 10-site chain, two modes per site, depth 6 (230230 aux x 10
states), 5 steps of 2 fs for two seeded noise arrays: psi(t), a fixed sample of
phi entries and sum |phi|^2 at the end.
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

POP_BOUND = 1e-5      # max | |psi_n(t)|^2 - |psi_n^ref(t)|^2 | of the reduced precisions


def _ring20_batch(precision, B=128):
    import torch
    from mesohops_b200 import HopsEnsemble
    from mesohops_b200.workloads import ring20
    f = load_golden("c3_ring20")
    n_real = f["noise1"].shape[0]
    noise = np.ascontiguousarray(f["noise1"][np.arange(B) % n_real])
    ens = HopsEnsemble(ring20(), B, noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                                 "TLEN": float(f["tlen"]),
                                                 "TAU": float(f["tau_noise"])},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision)
    psi0 = np.zeros(20, dtype=np.complex128)
    psi0[0] = 1.0
    ens.initialize(psi0)
    n = len(f["psi_traj"][0]) - 1
    dt = float(f["dt"])
    psi = torch.empty((n, B, 20), dtype=torch.complex128, device="cuda")
    ens.propagate(n * dt, dt, psi_out=psi)
    ens.check()
    out = psi.cpu().numpy()
    ref = f["psi_traj"][np.arange(B) % n_real][:, 1:]       # [B, n, 20]
    return np.transpose(out, (1, 0, 2)), ref


def test_ring20_complex128_matches_reference(cuda_device):
    psi, ref = _ring20_batch("complex128")
    err = np.max(np.abs(psi - ref)) / np.max(np.abs(ref))
    assert err <= 1e-10, err


# complex64 throughout rounds the state itself every step; over 128 noise
# realisations of this system its worst population error was 1.2e-4, so it is
# held to a looser bound and is not the precision the 1e-5 target is claimed for
C64_POP_BOUND = 5e-4


@pytest.mark.parametrize("precision,bound", [("mixed", POP_BOUND), ("complex64", C64_POP_BOUND)])
def test_ring20_reduced_precision_population_error(cuda_device, precision, bound):
    psi, ref = _ring20_batch(precision)
    err = np.max(np.abs(np.abs(psi) ** 2 - np.abs(ref) ** 2))
    assert err <= bound, (precision, err)


def _chain10(precision, B):
    import torch
    from mesohops_b200 import HopsEnsemble
    from mesohops_b200.workloads import chain10_two_modes
    f = load_golden("c2_chain10")
    k = int(f["n_traj"])
    noise = np.ascontiguousarray(np.array([f[f"noise1_{b % k}"] for b in range(B)]))
    ens = HopsEnsemble(chain10_two_modes(), B,
                       noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                    "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision)
    assert ens.n_hier == int(f["n_hier"])
    psi0 = np.zeros(10, dtype=np.complex128)
    psi0[0] = 1.0
    ens.initialize(psi0)
    dt = float(f["dt"])
    n = len(f["psi_traj_0"]) - 1
    psi = torch.empty((n, B, 10), dtype=torch.complex128, device="cuda")
    ens.propagate(n * dt, dt, psi_out=psi)
    ens.check()
    return f, k, psi.cpu().numpy(), ens


@pytest.mark.parametrize("B", [2, 32])
def test_chain10_complex128_matches_reference(cuda_device, B):
    import torch
    f, k, psi, ens = _chain10("complex128", B)
    phi = ens.batch
    phi.settle()
    for b in range(B):
        ref = f[f"psi_traj_{b % k}"][1:]
        assert np.max(np.abs(psi[:, b] - ref)) <= 1e-10 * np.max(np.abs(ref))
        row = phi.phi[:, :, b].reshape(-1)
        idx = torch.from_numpy(f[f"phi_idx_{b % k}"]).to(row.device)
        samp = row[idx].cpu().numpy()
        ref_s = f[f"phi_sample_{b % k}"]
        assert np.max(np.abs(samp - ref_s)) <= 1e-10 * np.max(np.abs(ref_s))
        n2 = float((row.abs() ** 2).sum())
        assert abs(n2 - float(f[f"phi_norm2_{b % k}"])) <= 1e-10 * n2


def test_chain10_mixed_population_error(cuda_device):
    f, k, psi, _ = _chain10("mixed", 32)
    for b in range(32):
        ref = f[f"psi_traj_{b % k}"][1:]
        assert np.max(np.abs(np.abs(psi[:, b]) ** 2 - np.abs(ref) ** 2)) <= POP_BOUND
