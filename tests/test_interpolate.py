"""Noise with INTERPOLATE = True (hops_noise.py:242-279,379-384).

The reference samples a cubic spline through the correlated noise; its step
check only lets it sample the grid times of the noise axis, where the spline
returns the samples, so the samples stay complex128 instead of being rounded
to complex64.  Fixtures (tests/golden/make_golden.py --interpolate) hold
reference runs with a complex128 PRE_CALCULATED noise array: a 6-site ring
(normalized nonlinear) and a dimer with the LINEAR equation of motion, whose
noise term the reference does not round to complex64 here.
"""
import numpy as np
import pytest

from conftest import golden_system, load_golden
from oracle import hops_oracle as O

CASES = ["interp_ring6", "interp_dimer_linear"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_with_complex128_samples_matches_reference(name):
    f = load_golden(name)
    sysp = golden_system(f)
    b = O.OracleBasis({k: sysp[k] for k in ("HAMILTONIAN", "GW_SYSBATH", "L_HIER")},
                      int(f["depth"]))
    _, psi, _, _ = O.propagate(b, f["psi0"], f["noise1"], float(f["tau_noise"]),
                               float(f["t_max"]), float(f["dt"]), eom=str(f["eom"]),
                               noise_dtype=np.complex128)
    ref = f["psi_traj"]
    assert np.max(np.abs(psi - ref)) <= 1e-10 * np.max(np.abs(ref))
    # with the samples rounded to complex64 the run misses the 1e-10 bound
    _, psi64, _, _ = O.propagate(b, f["psi0"], f["noise1"], float(f["tau_noise"]),
                                 float(f["t_max"]), float(f["dt"]), eom=str(f["eom"]))
    assert np.max(np.abs(psi64 - ref)) > 1e-10 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("kernel", ["resident", "streaming"])
def test_interpolated_noise_trajectory_matches_reference(cuda_device, name, kernel):
    from mesohops_b200 import HopsTrajectory
    f = load_golden(name)
    hops = HopsTrajectory(golden_system(f),
                          noise_param={"SEED": f["noise1"], "MODEL": "PRE_CALCULATED",
                                       "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"]),
                                       "INTERPOLATE": True},
                          hierarchy_param={"MAXHIER": int(f["depth"])},
                          eom_param={"EQUATION_OF_MOTION": str(f["eom"])},
                          device_param={"PRECISION": "complex128", "KERNEL": kernel})
    hops.initialize(f["psi0"])
    hops.propagate(float(f["t_max"]), float(f["dt"]))
    psi = np.array(hops.storage["psi_traj"])
    ref = f["psi_traj"]
    assert np.max(np.abs(psi - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_interpolated_noise_in_an_ensemble(cuda_device):
    import torch
    from mesohops_b200 import HopsEnsemble
    f = load_golden("interp_ring6")
    B = 33
    noise = np.repeat(f["noise1"][None], B, axis=0)
    ens = HopsEnsemble(golden_system(f), B,
                       noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                    "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"]),
                                    "INTERPOLATE": True},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision="complex128")
    ens.initialize(f["psi0"])
    n = len(f["psi_traj"]) - 1
    dt = float(f["dt"])
    psi = torch.empty((n, B, ens.n_state), dtype=torch.complex128, device="cuda")
    ens.propagate(n * dt, dt, psi_out=psi)
    out = psi.cpu().numpy()
    ref = f["psi_traj"][1:]
    for b in (0, B - 1):
        assert np.max(np.abs(out[:, b] - ref)) <= 1e-10 * np.max(np.abs(ref))
