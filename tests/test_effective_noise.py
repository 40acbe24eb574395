"""EFFECTIVE_NOISE_INTEGRATION: the RK4 noise samples replaced by window means
(integrator/integrator_rk.py:115-128).

Fixtures tests/golden/eff_*.npz come from the unmodified reference
(tests/golden/make_golden.py --effective) with PRE_CALCULATED noise on an axis
k = dt / (2 TAU) times finer than dt / 2 (k = 4, 5 and 9).  The oracle is
pinned to them on the CPU; on the GPU the window means
(hops_noise_window_mean) must equal numpy's bit for bit and the trajectories
must match the reference to 1e-10 (complex128)."""
import numpy as np
import pytest

from conftest import golden_system, load_golden
from oracle import hops_oracle as O

FIXTURES = ["eff_dimer_k4", "eff_ring6_k5", "eff_dimer_k9"]


def oracle_basis(f):
    sysp = {"HAMILTONIAN": f["H"], "GW_SYSBATH": [[g, w] for g, w in zip(f["G"], f["W"])],
            "L_HIER": list(f["L"])}
    return O.OracleBasis(sysp, int(f["depth"]))


def oracle_run(f, effective):
    return O.propagate(oracle_basis(f), f["psi0"], f["noise1"], float(f["tau_noise"]),
                       float(f["t_max"]), float(f["dt"]), noise2=f["noise2"],
                       eom=str(f["eom"]), effective=effective)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_effective_noise_pinned(name):
    f = load_golden(name)
    t, psi, _, _ = oracle_run(f, True)
    ref = f["psi_traj"]
    assert np.allclose(t, f["t_axis"])
    assert np.max(np.abs(psi - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the window means matter: the plain samples give a different trajectory
    _, psi_plain, _, _ = oracle_run(f, False)
    assert np.max(np.abs(psi_plain - ref)) > 1e-6


def make_traj(f, kernel, precision="complex128"):
    from mesohops_b200 import HopsTrajectory
    from mesohops_b200.bath import bcf_exp
    sysp = golden_system(f)
    noise2 = None
    if np.any(f["noise2"] != 0):
        sysp["L_NOISE2"] = sysp["L_HIER"]
        sysp["ALPHA_NOISE2"] = bcf_exp
        sysp["PARAM_NOISE2"] = sysp["GW_SYSBATH"]
        noise2 = {"SEED": f["noise2"], "MODEL": "PRE_CALCULATED", "TLEN": float(f["tlen"]),
                  "TAU": float(f["tau_noise"]), "FLAG_REAL": False}
    hops = HopsTrajectory(sysp, noise_param={"SEED": f["noise1"], "MODEL": "PRE_CALCULATED",
                                             "TLEN": float(f["tlen"]),
                                             "TAU": float(f["tau_noise"])},
                          noise2_param=noise2,
                          hierarchy_param={"MAXHIER": int(f["depth"])},
                          eom_param={"EQUATION_OF_MOTION": str(f["eom"])},
                          integration_param={"INTEGRATOR": "RUNGE_KUTTA",
                                             "EFFECTIVE_NOISE_INTEGRATION": True},
                          device_param={"KERNEL": kernel, "PRECISION": precision})
    hops.initialize(f["psi0"])
    return hops


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("real_only", [False, True])
def test_window_means_bit_identical_to_numpy(cuda_device, real_only):
    import torch
    from mesohops_b200.noise import window_means
    rng = np.random.default_rng(7)
    for k in list(range(1, 20)) + [31, 32, 33, 63, 64, 65, 70, 129]:
        n_out, start = 5, 3
        n_t = start + n_out * k + 2
        x = ((rng.normal(size=(3, n_t)) + 1j * rng.normal(size=(3, n_t)))
             * rng.uniform(0.1, 1000)).astype(np.complex64)
        got = window_means(torch.from_numpy(x).to(cuda_device), start, k, n_out,
                           real_only).cpu().numpy()
        src = np.real(x) if real_only else x
        ref = np.stack([np.mean(src[:, start + w * k:start + (w + 1) * k], axis=1)
                        for w in range(n_out)], axis=1)
        assert np.array_equal(got.real, np.real(ref)), k
        assert np.array_equal(got.imag, np.imag(ref) if not real_only else 0 * got.imag), k


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["resident", "streaming"])
@pytest.mark.parametrize("name", FIXTURES)
def test_effective_noise_trajectory_matches_reference(cuda_device, name, kernel):
    f = load_golden(name)
    hops = make_traj(f, kernel)
    hops.propagate(float(f["t_max"]), float(f["dt"]))
    psi = np.array(hops.storage["psi_traj"])
    assert psi.shape == f["psi_traj"].shape
    np.testing.assert_allclose(hops.storage["t_axis"], f["t_axis"])
    assert rel(psi, f["psi_traj"]) <= 1e-10
    assert rel(hops.phi, f["phi_end"]) <= 1e-10


@pytest.mark.gpu
def test_effective_noise_in_pieces_equals_one_call(cuda_device):
    f = load_golden("eff_ring6_k5")
    a = make_traj(f, "streaming")
    a.propagate(float(f["t_max"]), float(f["dt"]))
    b = make_traj(f, "streaming")
    dt = float(f["dt"])
    first = dt * (int(round(float(f["t_max"]) / dt)) // 2)
    b.propagate(first, dt)
    b.propagate(float(f["t_max"]) - first, dt)
    assert rel(np.array(b.storage["psi_traj"]), np.array(a.storage["psi_traj"])) <= 1e-13
