"""Pins the CPU oracle to the reference: committed fixtures produced by running
unmodified MesoHOPS (tests/golden/make_golden.py) and, when the reference tree is
present, the reference's own golden arrays (tests/dimer_of_dimers/*.npy)."""
import os

import numpy as np
import pytest
import scipy.sparse as sps

from conftest import load_golden
from oracle import hops_oracle as O

FIXTURES = ["c1_dimer", "dod", "general_lop", "ring6", "chain4_2mode", "c1_nonlinear",
            "c1_linear"]
REF_TESTS = os.environ.get("MESOHOPS_TESTS", "/root/reference/tests")


def oracle_basis(f):
    sysp = {"HAMILTONIAN": f["H"], "GW_SYSBATH": [[g, w] for g, w in zip(f["G"], f["W"])],
            "L_HIER": list(f["L"])}
    return O.OracleBasis(sysp, int(f["depth"]))


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_aux_order(name):
    f = load_golden(name)
    assert np.array_equal(oracle_basis(f).aux, f["aux"])


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_derivative(name):
    f = load_golden(name)
    b = oracle_basis(f)
    dphi, dz = O.dsystem_dt(b, f["deriv_phi"], f["deriv_zmem"], f["deriv_z1"], f["deriv_z2"],
                            str(f["eom"]))
    ref = f["deriv_dphi"]
    assert np.max(np.abs(dphi - ref)) <= 1e-13 * np.max(np.abs(ref))
    if str(f["eom"]) != "LINEAR":
        assert np.allclose(dz, f["deriv_dz"], rtol=1e-13, atol=0)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_trajectory(name):
    f = load_golden(name)
    b = oracle_basis(f)
    t, psi, phi, zm = O.propagate(b, f["psi0"], f["noise1"], float(f["tau_noise"]),
                                  float(f["t_max"]), float(f["dt"]), noise2=f["noise2"],
                                  eom=str(f["eom"]))
    assert np.allclose(t, f["t_axis"])
    ref = f["psi_traj"]
    assert np.max(np.abs(psi - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("model", ["SUM_GAUSSIAN", "BOX_MULLER"])
def test_oracle_noise_pinned(model):
    f = load_golden("noise_dimer")
    t = O.noise_t_axis(float(f["tlen"]), float(f["tau"]))
    gw = [[g, w] for g, w in zip(f["G"], f["W"])]
    raw = O.raw_draws(0, [0, 1], len(t), model)
    assert np.array_equal(raw, f[model + "_raw"])
    alpha = np.complex64(O.alpha_by_lop(t, gw, [0, 1], 2))
    assert np.array_equal(alpha, f[model + "_alpha"])
    # reference dtype path: identical to the reference output
    eta_ref = O.fft_filter_noise(t, gw, [0, 1], 2, raw, fp64=False)
    assert np.array_equal(eta_ref, f[model + "_eta"])
    # FP64 path (what the GPU computes): differs only by the reference's float32
    # FFT / angle / abs of complex64 inputs
    eta64 = O.fft_filter_noise(t, gw, [0, 1], 2, raw, fp64=True)
    ref = f[model + "_eta"]
    assert np.max(np.abs(eta64 - ref)) <= 1e-6 * np.max(np.abs(ref))


def test_noise_index_scramble_small():
    # hops_noise.py:617-627 for ntaus = 4: every one of the 12 draws used once
    re, im = O.raw_index(4)
    assert re.tolist() == [0, 2, 6, 10, 8, 4]
    assert im.tolist() == [1, 3, 7, 11, 9, 5]
    assert sorted(np.concatenate([re, im]).tolist()) == list(range(12))


ref_dod = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_TESTS, "dimer_of_dimers")),
                             reason="reference test data not present")


def _dod_basis():
    g0, w0 = O.dl_to_exp(20.0, 50.0, 140.0)
    gw, lops = [], []
    for i in range(4):
        L = np.zeros((4, 4))
        L[i, i] = 1.0
        gw.append([g0, w0])
        lops.append(sps.coo_matrix(L))
        gw.append([-1j * np.imag(g0), 500.0])
        lops.append(L)
    hs = np.zeros((4, 4))
    hs[0, 1] = hs[1, 0] = 40
    hs[1, 2] = hs[2, 1] = 10
    hs[2, 3] = hs[3, 2] = 40
    return O.OracleBasis({"HAMILTONIAN": hs, "GW_SYSBATH": gw, "L_HIER": lops}, 2), gw


@ref_dod
def test_oracle_super_operators_vs_reference_golden():
    b, _ = _dod_basis()
    d = os.path.join(REF_TESTS, "dimer_of_dimers")
    assert np.all(np.load(os.path.join(d, "K2_k.npy")) == np.diag(b.k2_k))
    assert np.all(np.load(os.path.join(d, "K2_kp1.npy")) == b.k2_kp1.toarray())
    assert np.all(np.load(os.path.join(d, "K2_km1.npy")) == b.k2_km1.toarray())
    z = np.load(os.path.join(d, "Z2_kp1.npy"))
    assert all(np.all(z[j] == b.z2_kp1[j].toarray()) for j in range(4))


@ref_dod
def test_oracle_eta_vs_reference_golden():
    _, gw = _dod_basis()
    d = os.path.join(REF_TESTS, "dimer_of_dimers")
    t = O.noise_t_axis(25000.0, 1.0)
    alpha = O.alpha_by_lop(t, gw, [0, 0, 1, 1, 2, 2, 3, 3], 4)
    np.testing.assert_allclose(alpha, np.load(os.path.join(d, "alpha.npy")), rtol=1e-12)
    raw = O.raw_draws(0, [0, 1, 2, 3], len(t), "BOX_MULLER")
    eta = O.correlated_noise(alpha, raw, fp64=False)[0]
    np.testing.assert_allclose(eta, np.load(os.path.join(d, "eta.npy")), rtol=1e-10)
