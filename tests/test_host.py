"""Host-side logic (no GPU): hierarchy order and connections, the device tables
against the oracle's super-operators, parameter validation, raw noise."""
import numpy as np
import pytest

from conftest import golden_system, load_golden
from mesohops_b200 import hierarchy as H
from mesohops_b200.device import build_tables
from mesohops_b200.exceptions import AuxError, UnsupportedRequest
from mesohops_b200.noise import raw_slot_index
from mesohops_b200.params import (NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, initialize_dict)
from mesohops_b200.system import HopsSystem
from oracle import hops_oracle as O

FIXTURES = ["c1_dimer", "dod", "general_lop", "ring6", "chain4_2mode"]


@pytest.mark.parametrize("M,D", [(1, 5), (2, 4), (3, 0), (6, 3), (8, 2), (5, 5)])
def test_triangular_order_matches_oracle(M, D):
    c = H.triangular_counts(M, D)
    assert np.array_equal(c, O.triangular_aux(M, D))
    keys = H.AuxKeyer(M, D).keys_from_counts(c)
    assert np.array_equal(keys, np.arange(len(c)))


def test_keys_sort_arbitrary_subset():
    M, D = 7, 4
    c = O.triangular_aux(M, D)
    rng = np.random.default_rng(0)
    sub = c[np.sort(rng.choice(len(c), 60, replace=False))]
    sub = np.vstack([np.zeros((1, M), dtype=sub.dtype), sub]) if sub[0].sum() else sub
    shuffled = sub[rng.permutation(len(sub))]
    b = H.AuxBasis(shuffled, H.AuxKeyer(M, D), D)
    want = sorted(map(tuple, sub), key=O.aux_sort_key)
    assert [tuple(x) for x in b.counts] == want


def test_big_mode_keys_exact():
    k = H.AuxKeyer(500, 10)
    assert not k.use_int64
    c = np.zeros((4, 500), dtype=np.int16)
    c[1, 499] = 1
    c[2, 0] = 2
    c[3, 0] = 1
    c[3, 1] = 1
    keys = k.keys_from_counts(c)
    assert keys[0] == 0 and keys[1] == 500
    # depth-2 (0,0) comes right after every depth-1 aux, then (0,1)
    assert keys[2] == 501 and keys[3] == 502


@pytest.mark.parametrize("M,D", [(7, 4), (500, 10)])
def test_sort_keys_order_and_equality_are_the_ranks(M, D):
    """sort_keys (int64 ranks, or fixed-width byte keys when the ranks exceed
    int64) orders and identifies aux exactly as the exact global ranks do."""
    k = H.AuxKeyer(M, D)
    rng = np.random.default_rng(1)
    c = np.zeros((400, M), dtype=np.int16)
    for r in range(1, len(c)):
        np.add.at(c[r], rng.integers(0, min(M, 12), rng.integers(1, D + 1)), 1)
    exact = np.array([int(x) for x in k.keys_from_counts(c)], dtype=object)
    sk = k.sort_keys(c)
    o = np.argsort(exact, kind="stable")
    assert np.array_equal(o, np.argsort(sk, kind="stable"))
    assert np.array_equal(exact[o][1:] == exact[o][:-1], sk[o][1:] == sk[o][:-1])
    assert np.array_equal(H.AuxBasis(c[np.unique(sk, return_index=True)[1]], k, D).counts,
                          c[np.unique(sk, return_index=True)[1]][np.argsort(
                              exact[np.unique(sk, return_index=True)[1]], kind="stable")])


@pytest.mark.parametrize("M,D", [(7, 4), (500, 10)])
def test_tuple_keys_equal_count_row_keys(M, D):
    """keys_from_tuples of sorted mode tuples -- and of tuples with one mode
    inserted or removed (how the adaptive basis keys its neighbour candidates)
    -- equal sort_keys of the corresponding count rows, for int64 ranks and
    for byte keys."""
    k = H.AuxKeyer(M, D)
    rng = np.random.default_rng(4)
    c = np.zeros((300, M), dtype=np.int16)
    for r in range(1, len(c)):
        np.add.at(c[r], rng.integers(0, min(M, 15), rng.integers(1, D + 1)), 1)
    tup, depth = H.tuples_of(c, D)
    assert np.array_equal(k.keys_from_tuples(tup, depth), k.sort_keys(c))
    # insert a mode into every row below D
    low = np.nonzero(depth < D)[0]
    m = rng.integers(0, M, len(low))
    up = c[low].copy()
    up[np.arange(len(low)), m] += 1
    assert np.array_equal(k.keys_from_tuples(H.insert_mode(tup[low], m), depth[low] + 1),
                          k.sort_keys(up))
    # remove one of its modes from every row above depth 0
    hi = np.nonzero(depth > 0)[0]
    mm = np.array([rng.choice(np.nonzero(c[r])[0]) for r in hi])
    dn = c[hi].copy()
    dn[np.arange(len(hi)), mm] -= 1
    assert np.array_equal(k.keys_from_tuples(H.remove_mode(tup[hi], mm), depth[hi] - 1),
                          k.sort_keys(dn))


def test_missing_zero_aux_raises():
    c = np.array([[1, 0], [0, 1]])
    with pytest.raises(AuxError):
        H.AuxBasis(c, H.AuxKeyer(2, 2), 2)


@pytest.mark.parametrize("name", FIXTURES)
def test_tables_rebuild_super_operators(name):
    f = load_golden(name)
    sysm = HopsSystem(golden_system(f))
    basis = H.triangular_basis(sysm.n_mode, int(f["depth"]))
    t = build_tables(sysm, basis)
    ob = O.OracleBasis(golden_system(f), int(f["depth"]))
    S, N = t["n_state"], t["n_hier"]
    assert np.array_equal(basis.counts, ob.aux)
    np.testing.assert_allclose(t["k_decay"], ob.k2_k, rtol=1e-15)
    kp = np.zeros((N * S, N * S), dtype=complex)
    km = np.zeros((N * S, N * S), dtype=complex)
    lops = [sysm.lops[j] for j in t["l_abs"]]
    for a in range(N):
        for p in range(t["up_ptr"][a], t["up_ptr"][a + 1]):
            u, m = t["up_aux"][p], t["up_mode"][p]
            Lm = lops[t["mode_lop"][m]]
            for r, c in zip(*np.nonzero(Lm)):
                kp[a * S + r, u * S + c] += -t["mode_gw"][m] * Lm[r, c]
        for p in range(t["dn_ptr"][a], t["dn_ptr"][a + 1]):
            d, m = t["dn_aux"][p], t["dn_mode"][p]
            Lm = lops[t["mode_lop"][m]]
            for r, c in zip(*np.nonzero(Lm)):
                km[a * S + c, d * S + r] += t["dn_coef"][p] * np.conj(Lm[r, c])
    np.testing.assert_allclose(kp, ob.k2_kp1.toarray(), rtol=1e-14, atol=0)
    np.testing.assert_allclose(km, ob.k2_km1.toarray(), rtol=1e-14, atol=0)
    # first-level aux (norm correction) and H
    fl = sorted((int(a), int(m)) for a, m in zip(t["first_aux"], t["first_mode"]))
    assert fl == sorted((a, m) for (a, _, m) in ob.first_level)


def test_unique_l_by_pattern_uses_first_values():
    # two modes share a nonzero pattern with different values: the first wins
    L1 = np.diag([1.0, 0.0])
    L2 = np.diag([np.sqrt(2), 0.0])
    gw = [[10.0, 5.0], [3.0, 2.0]]
    s = HopsSystem({"HAMILTONIAN": np.eye(2), "GW_SYSBATH": gw, "L_HIER": [L1, L2],
                    "L_NOISE1": [L1, L2], "ALPHA_NOISE1": O.bcf_exp, "PARAM_NOISE1": gw})
    assert s.n_lop == 1 and list(s.l_by_mode) == [0, 0]
    assert s.lops[0][0, 0] == 1.0


def test_param_validation_like_reference():
    with pytest.raises(UnsupportedRequest):
        initialize_dict({"BOGUS": 1}, NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, "HopsNoise")
    with pytest.raises(TypeError):
        initialize_dict({"TLEN": 10}, NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, "HopsNoise")
    p = initialize_dict({"TLEN": 10.0}, NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, "HopsNoise")
    assert p["TAU"] == 1.0 and p["MODEL"] == "FFT_FILTER"


@pytest.mark.parametrize("model", ["SUM_GAUSSIAN", "BOX_MULLER"])
def test_raw_noise_matches_reference(model):
    f = load_golden("noise_dimer")
    n_t = int(np.ceil(float(f["tlen"]) / float(f["tau"]))) + 1
    assert np.array_equal(O.raw_draws(0, [0, 1], n_t, model), f[model + "_raw"])


def test_raw_slot_index_matches_oracle():
    for n in (3, 4, 17, 503):
        a, b = raw_slot_index(n)
        c, d = O.raw_index(n)
        assert np.array_equal(a, c) and np.array_equal(b, d)
