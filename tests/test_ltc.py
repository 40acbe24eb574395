"""Low-temperature correction (LTC) of the equations of motion:
eom/eom_functions.py:215-309 applied as eom/hops_eom.py:357-403 (nonlinear,
normalized or not) and :527-529 (LINEAR).

Fixtures tests/golden/ltc_*.npz come from the unmodified reference
(tests/golden/make_golden.py --ltc): a dimer under the three equations of
motion, a 6-site ring with corrections on three sites plus one operator of no
bath (dropped, as the reference does), and general off-diagonal L-operators
with noise 2.  The oracle is pinned to them on the CPU; the GPU path matches
them to 1e-10 (complex128) and the derivative to 1e-12."""
import numpy as np
import pytest

from conftest import golden_system, load_golden
from oracle import hops_oracle as O

FIXTURES = ["ltc_dimer_norm", "ltc_dimer_nonlinear", "ltc_dimer_linear", "ltc_ring6",
            "ltc_general"]


def oracle_basis(f):
    sysp = golden_system(f)
    return O.OracleBasis(sysp, int(f["depth"]))


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_ltc_derivative(name):
    f = load_golden(name)
    dphi, dz = O.dsystem_dt(oracle_basis(f), f["deriv_phi"], f["deriv_zmem"], f["deriv_z1"],
                            f["deriv_z2"], str(f["eom"]))
    ref = f["deriv_dphi"]
    assert np.max(np.abs(dphi - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_ltc_trajectory(name):
    f = load_golden(name)
    b = oracle_basis(f)
    t, psi, _, _ = O.propagate(b, f["psi0"], f["noise1"], float(f["tau_noise"]),
                               float(f["t_max"]), float(f["dt"]), noise2=f["noise2"],
                               eom=str(f["eom"]))
    ref = f["psi_traj"]
    assert np.max(np.abs(psi - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the correction matters: without it the trajectory differs
    sysp = golden_system(f)
    sysp.pop("L_LT_CORR")
    sysp.pop("PARAM_LT_CORR")
    _, psi0, _, _ = O.propagate(O.OracleBasis(sysp, int(f["depth"])), f["psi0"], f["noise1"],
                                float(f["tau_noise"]), float(f["t_max"]), float(f["dt"]),
                                noise2=f["noise2"], eom=str(f["eom"]))
    assert np.max(np.abs(psi0 - ref)) > 1e-6


def test_ltc_coefficients_by_unique_l():
    """Corrections are summed per unique L and dropped when no bath has that L
    (basis/system_functions.py:115-133)."""
    f = load_golden("ltc_ring6")
    s = O.expand_system(golden_system(f))
    lt = s["LT"]
    assert lt[0] == 0.2 and lt[2] == 0.1 - 0.05j and lt[4] == 0.3j
    assert lt[1] == 0 and lt[3] == 0 and lt[5] == 0


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
                          device_param={"KERNEL": kernel, "PRECISION": precision})
    hops.initialize(f["psi0"])
    return hops


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(np.asarray(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["resident", "streaming"])
@pytest.mark.parametrize("name", FIXTURES)
def test_ltc_trajectory_matches_reference(cuda_device, name, kernel):
    f = load_golden(name)
    hops = make_traj(f, kernel)
    hops.propagate(float(f["t_max"]), float(f["dt"]))
    psi = np.array(hops.storage["psi_traj"])
    assert psi.shape == f["psi_traj"].shape
    assert rel(psi, f["psi_traj"]) <= 1e-10
    assert rel(hops.phi, f["phi_end"]) <= 1e-10
    if str(f["eom"]) != "LINEAR":
        zm = f["zmem_end"]
        assert np.max(np.abs(hops.z_mem - zm)) <= 1e-10 * max(1.0, np.max(np.abs(zm)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_ltc_derivative_matches_reference(cuda_device, name):
    f = load_golden(name)
    hops = make_traj(f, "streaming")
    dphi, dz = hops.dsystem_dt(f["deriv_phi"], f["deriv_zmem"], f["deriv_z1"], f["deriv_z2"])
    ref = f["deriv_dphi"]
    assert np.max(np.abs(np.asarray(dphi) - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["mixed", "complex64"])
def test_ltc_batched_ensemble_matches_oracle(cuda_device, precision):
    """The wide stage kernel (B >= 32) with the correction, against the oracle."""
    import torch
    from mesohops_b200.ensemble import HopsEnsemble
    f = load_golden("ltc_ring6")
    sysp = golden_system(f)
    B, dt, n = 40, float(f["dt"]), 10
    ens = HopsEnsemble(sysp, B, noise_param={"MODEL": "FFT_FILTER", "TLEN": (n + 4) * dt,
                                             "TAU": dt / 2, "SEED": list(range(B))},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision,
                       device=cuda_device, autotune=False)
    ens.initialize(f["psi0"])
    psi = torch.empty((n, B, ens.n_state), dtype=torch.complex128, device=cuda_device)
    ens.propagate(n * dt, dt, psi_out=psi)
    psi = psi.cpu().numpy()
    noise = ens.noise.cpu().numpy()
    b = oracle_basis(f)
    for tr in (0, 17, B - 1):
        _, ref, _, _ = O.propagate(b, f["psi0"], noise[tr], dt / 2, n * dt, dt)
        pop = np.abs(psi[:, tr]) ** 2
        assert np.max(np.abs(pop - np.abs(ref[1:]) ** 2)) <= 1e-5
