"""DyadicTrajectory (trajectory/hops_dyadic.py:15-246) against the reference.

Fixtures tests/golden/dyadic_*.npz come from the unmodified reference
(tests/golden/make_golden.py --dyadic): a 3-site system with a ground state,
ket and bra excitations, propagation, a bra de-excitation and more
propagation, for the normalised equation of motion with dense operators, the
LINEAR one with sparse operators, and the normalised one on an adaptive basis
(which the operators grow).  On the CPU the operator bookkeeping
(states after each operator, normalisation factors, response function) is
checked without propagation, and the adaptive sequence with the device
requests served by the oracle; on the GPU the whole sequence must match the
reference to 1e-10 (complex128)."""
import numpy as np
import pytest
import scipy.sparse as sps

from conftest import load_golden
from mesohops_b200.bath import bcf_exp
from mesohops_b200.dyadic import dyad_conversion, response_function_calc
from mesohops_b200.exceptions import UnsupportedRequest

FIXTURES = ["dyadic_norm_dense", "dyadic_linear_sparse"]
# the same sequence with an adaptive basis (delta_a = delta_s = 1e-3): states the
# operators reach join the basis, which the early-time integrator then updates
ADAPTIVE = ["dyadic_adaptive"]


def system(f):
    sparse = bool(f["sparse_input"])
    conv = (lambda m: sps.coo_matrix(m)) if sparse else (lambda m: np.array(m))
    lops = [conv(l) for l in f["L"]]
    gw = [[g, w] for g, w in zip(f["G"], f["W"])]
    return {"HAMILTONIAN": conv(f["H"]), "GW_SYSBATH": gw, "L_HIER": lops, "L_NOISE1": lops,
            "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw}, conv


def make(f, device):
    from mesohops_b200.dyadic import DyadicTrajectory
    sysp, conv = system(f)
    hops = DyadicTrajectory(sysp, noise_param={"SEED": f["noise1"], "MODEL": "PRE_CALCULATED",
                                               "TLEN": float(f["tlen"]),
                                               "TAU": float(f["tau_noise"])},
                            hierarchy_param={"MAXHIER": int(f["depth"])},
                            eom_param={"EQUATION_OF_MOTION": str(f["eom"])},
                            device_param={"DEVICE": device, "PRECISION": "complex128"})
    if "adaptive" in f and float(f["adaptive"][0]) > 0:
        hops.make_adaptive(float(f["adaptive"][0]), float(f["adaptive"][1]),
                           adaptive_noise=False)
    hops.initialize(f["psi_k"], f["psi_b"])
    return hops, conv


def test_dyad_conversion_dense_and_sparse():
    m = np.array([[1 + 2j, 2 - 1j], [3 + 0j, 4 - 0.5j]])
    ref = np.array([[1 + 2j, 2 - 1j, 0, 0], [3, 4 - 0.5j, 0, 0], [0, 0, 1 + 2j, 2 - 1j],
                    [0, 0, 3, 4 - 0.5j]])
    d = dyad_conversion(m)
    assert d.dtype == np.complex128 and np.array_equal(d, ref)
    s = dyad_conversion(sps.coo_matrix(m))
    assert sps.issparse(s) and np.array_equal(s.toarray(), ref)


@pytest.mark.parametrize("name", FIXTURES)
def test_dyadic_operators_on_host(name):
    f = load_golden(name)
    hops, conv = make(f, "cpu")
    np.testing.assert_allclose(hops.psi, f["psi_init"], rtol=1e-14, atol=1e-15)
    hops._dyad_operator(conv(f["op_ket"]), "ket")
    np.testing.assert_allclose(hops.psi, f["psi_op1"], rtol=1e-13, atol=1e-15)
    hops._dyad_operator(conv(f["op_bra"]), "bra")
    np.testing.assert_allclose(hops.psi, f["psi_op2"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(hops.list_response_norm_sq, f["norm_sq"][:3], rtol=1e-13)
    with pytest.raises(UnsupportedRequest):
        hops._dyad_operator(conv(f["op_bra"]), "braket")


@pytest.mark.parametrize("name", FIXTURES)
def test_response_function_calc_matches_reference(name):
    f = load_golden(name)
    got = response_function_calc(f["f_op"], 5, f["psi_traj"], f["norm_sq"])
    np.testing.assert_allclose(got, f["response"], rtol=1e-13, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES + ADAPTIVE)
def test_dyadic_trajectory_matches_reference(cuda_device, name):
    f = load_golden(name)
    hops, conv = make(f, "cuda:0")
    hops._dyad_operator(conv(f["op_ket"]), "ket")
    np.testing.assert_allclose(hops.psi, f["psi_op1"], rtol=1e-12, atol=1e-14)
    hops._dyad_operator(conv(f["op_bra"]), "bra")
    np.testing.assert_allclose(hops.psi, f["psi_op2"], rtol=1e-12, atol=1e-14)
    dt, t1 = float(f["dt"]), float(f["t1"])
    hops.propagate(t1, dt)
    hops._dyad_operator(conv(f["op_down"]), "bra")
    np.testing.assert_allclose(hops.psi, f["psi_op3"], rtol=1e-10, atol=1e-12)
    hops.propagate(t1, dt)
    psi = np.array(hops.storage["psi_traj"])
    ref = f["psi_traj"]
    assert psi.shape == ref.shape
    assert np.max(np.abs(psi - ref)) <= 1e-10 * np.max(np.abs(ref))
    np.testing.assert_allclose(hops.list_response_norm_sq, f["norm_sq"], rtol=1e-10)
    resp = hops._response_function_comp(f["f_op"], 5)
    scale = max(1e-300, np.max(np.abs(f["response"])))
    assert np.max(np.abs(resp - f["response"])) <= 1e-10 * scale


def test_dyadic_adaptive_sequence_oracle_served(monkeypatch):
    """The adaptive sequence with the device requests served by the oracle: the
    basis grows by the states the operators reach, and states, norms, psi(t)
    and the response function equal the reference's."""
    import mesohops_b200.adaptive as ad
    from test_adaptive import OracleServer
    f = load_golden("dyadic_adaptive")
    from mesohops_b200.dyadic import DyadicTrajectory
    sysp, conv = system(f)
    hops = DyadicTrajectory(sysp, noise_param={"SEED": f["noise1"], "MODEL": "PRE_CALCULATED",
                                               "TLEN": float(f["tlen"]),
                                               "TAU": float(f["tau_noise"])},
                            hierarchy_param={"MAXHIER": int(f["depth"])},
                            eom_param={"EQUATION_OF_MOTION": str(f["eom"])},
                            device_param={"DEVICE": "cpu", "PRECISION": "complex128"})
    server = OracleServer(sysp, f["noise1"], float(f["tau_noise"]))  # sysp is dyadic now
    monkeypatch.setattr(ad, "drive", server.drive)
    hops.make_adaptive(float(f["adaptive"][0]), float(f["adaptive"][1]), adaptive_noise=False)
    hops.initialize(f["psi_k"], f["psi_b"])
    for key, op, side in [("psi_op1", "op_ket", "ket"), ("psi_op2", "op_bra", "bra")]:
        hops._dyad_operator(conv(f[op]), side)
        np.testing.assert_allclose(hops.psi, f[key], rtol=1e-12, atol=1e-14)
    hops.propagate(float(f["t1"]), float(f["dt"]))
    hops._dyad_operator(conv(f["op_down"]), "bra")
    np.testing.assert_allclose(hops.psi, f["psi_op3"], rtol=1e-10, atol=1e-12)
    hops.propagate(float(f["t1"]), float(f["dt"]))
    psi = np.array(hops.storage["psi_traj"])
    assert np.max(np.abs(psi - f["psi_traj"])) <= 1e-10 * np.max(np.abs(f["psi_traj"]))
    np.testing.assert_allclose(hops.list_response_norm_sq, f["norm_sq"], rtol=1e-10)
    np.testing.assert_allclose(hops._response_function_comp(f["f_op"], 5), f["response"],
                               rtol=1e-10, atol=1e-14)
