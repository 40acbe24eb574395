"""Adaptive basis (adHOPS): host logic and device path against the reference.

Fixtures tests/golden/adaptive_*.npz come from running the unmodified MesoHOPS
adaptive trajectory (tests/golden/make_golden.py --adaptive) with
PRE_CALCULATED noise.  Two ways to run the same driver:

* CPU (not gpu): the device requests of mesohops_b200.adaptive (RK4 step, flux
  errors) are served by the oracle on the same sub-basis, so the basis logic
  (filters, thresholds, boundary sets, inch-worm, permutations) is checked
  without a GPU.
* GPU: the product path (resident kernel + hops_flux_errors) end to end.

Both must reproduce the reference's basis sizes, state lists and aux lists at
every step, and psi(t) to 1e-10.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sps

import mesohops_b200.adaptive as ad
from mesohops_b200 import HopsTrajectory
from mesohops_b200.exceptions import UnsupportedRequest
from oracle import hops_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["adaptive_dod_full", "adaptive_chain8", "adaptive_chain12", "adaptive_chain8_ltc",
         "adaptive_chain8_eff", "adaptive_static_inchworm", "adaptive_static_state"]
# the benchmark's 500-site chain at depth 10 (aux keys beyond int64): the oracle
# would need its 500 dense L-operators, so only the GPU run is compared
GPU_ONLY_CASES = ["adaptive_chain500"]


def load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


def system_param(f):
    gw = [(complex(g), complex(w)) for g, w in zip(f["G"], f["W"])]
    if "L" in f:
        lops = [np.array(l) for l in f["L"]]
    else:   # site projectors stored as each mode's site (systems too large for dense L)
        n = f["H"].shape[0]
        lops = [sps.coo_matrix(([1.0], ([int(i)], [int(i)])), shape=(n, n)) for i in f["L_site"]]
    sysp = {"HAMILTONIAN": np.array(f["H"]), "GW_SYSBATH": gw, "L_HIER": lops,
            "L_NOISE1": lops, "ALPHA_NOISE1": O.bcf_exp, "PARAM_NOISE1": gw}
    if "LT_L" in f:   # low-temperature corrections
        sysp["L_LT_CORR"] = [np.array(l) for l in f["LT_L"]]
        sysp["PARAM_LT_CORR"] = [complex(c) for c in f["LT_P"]]
    return sysp


def make_traj(f, tmp_path, device):
    path = str(tmp_path / "noise1.npy")
    np.save(path, f["noise1"])
    integ = {"INTEGRATOR": "RUNGE_KUTTA",
             # the fixture with noise finer than dt / 2 was made with
             # EFFECTIVE_NOISE_INTEGRATION (make_golden.py --effective-adaptive)
             "EFFECTIVE_NOISE_INTEGRATION": 2 * float(f["tau_noise"]) < float(f["dt"]) - 1e-12}
    if "static_states" in f:   # make_golden.py --static-basis
        integ["STATIC_BASIS"] = [f["static_states"].tolist(), list(f["static_aux"])]
        integ["EARLY_ADAPTIVE_INTEGRATOR"] = str(f["early_integrator"])
    hops = HopsTrajectory(system_param(f),
                          noise_param={"SEED": path, "MODEL": "PRE_CALCULATED",
                                       "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                          hierarchy_param={"MAXHIER": int(f["depth"])},
                          eom_param={"EQUATION_OF_MOTION": "NORMALIZED NONLINEAR"},
                          storage_param={}, device_param={"DEVICE": device,
                                                          "PRECISION": "complex128"},
                          integration_param=integ)
    hops.make_adaptive(float(f["delta_a"]), float(f["delta_s"]),
                       update_step=int(f["update_step"]), f_discard=float(f["f_discard"]),
                       adaptive_noise=False)
    return hops


class OracleServer:
    """Serves the driver's device requests with the oracle (CPU)."""

    def __init__(self, sysp, noise1, tau_noise):
        self.sysp = sysp
        self.full = O.expand_system(sysp)
        self.noise1 = noise1
        self.tau_noise = tau_noise
        self.cache = {}

    def sub(self, basis):
        key = id(basis)
        if key not in self.cache:
            self.cache[key] = (basis, O.OracleSubBasis(self.sysp, basis.states, basis.modes,
                                                       basis.counts, full=self.full))
        return self.cache[key][1]

    def step(self, r):
        d = r.driver
        ob = self.sub(d.basis)
        if r.effective:
            zr = O.effective_noise(self.noise1[ob.l_abs], r.t, r.tau, self.tau_noise)
        else:
            tl = [r.t, r.t + 0.5 * r.tau, r.t + r.tau]
            zr = O.noise_lookup(self.noise1[ob.l_abs], tl, self.tau_noise)
        zm = r.zmem_abs[d.basis.modes]
        phi, z = O.rk4_step(ob, r.phi, zm, zr, np.zeros_like(zr), r.tau)
        return d.finish_step(r, phi, z)

    def flux(self, r):
        ob = self.sub(r.driver.basis)
        return O.flux_errors(ob, r.phi, r.z_step[2][r.driver.basis.modes], r.z_step[0],
                             r.z_step[1], r.dt, mask=r.mask)

    def drive(self, gen, device):
        result = None
        while True:
            try:
                req = gen.send(result)
            except StopIteration as stop:
                return stop.value
            result = self.step(req) if isinstance(req, ad.StepRequest) else self.flux(req)


def aux_sets(f):
    ptr = f["aux_ptr"]
    c = f["aux_counts"]
    return [set(map(tuple, c[ptr[i]:ptr[i + 1]].tolist())) for i in range(len(ptr) - 1)]


def state_lists(f):
    ptr = f["state_ptr"]
    s = f["states"]
    return [sorted(s[ptr[i]:ptr[i + 1]].tolist()) for i in range(len(ptr) - 1)]


def check_against(hops, f):
    d = hops.storage.data
    assert np.array_equal(np.array(d["list_nhier"]), f["list_nhier"])
    assert np.array_equal(np.array(d["list_nstate"]), f["list_nstate"])
    assert [sorted(np.asarray(s).tolist()) for s in d["state_list"]] == state_lists(f)
    mine = []
    n_mode = len(f["G"])
    for aux_list in d["aux_list"]:
        rows = set()
        for a in aux_list:
            v = [0] * n_mode
            for (m, k) in np.asarray(a).reshape(-1, 2):
                v[m] = int(k)
            rows.add(tuple(v))
        mine.append(rows)
    assert mine == aux_sets(f)
    psi = hops.storage["psi_traj"]
    assert np.max(np.abs(psi - f["psi_traj"])) <= 1e-10
    assert np.allclose(d["t_axis"], f["t_axis"])


@pytest.mark.parametrize("name", CASES)
def test_adaptive_host_logic_oracle_served(name, tmp_path, monkeypatch):
    f = load(name)
    server = OracleServer(system_param(f), f["noise1"], float(f["tau_noise"]))
    monkeypatch.setattr(ad, "drive", server.drive)
    hops = make_traj(f, tmp_path, "cpu")
    hops.initialize(f["psi0"])
    hops.propagate(float(f["t_max"]), float(f["dt"]))
    check_against(hops, f)
    assert hops.n_hier == int(f["n_hier_end"])
    assert hops.n_state == int(f["n_state_end"])
    assert np.max(np.abs(hops.phi - f["phi_end"])) <= 1e-10


def test_error_thresh_edges():
    # all below the bound: every member may go (threshold = inf)
    assert ad.error_thresh(np.array([1.0, 2.0]), 10.0) == np.inf
    # first member alone reaches the bound: keep everything
    assert ad.error_thresh(np.array([5.0, 6.0]), 4.0) == 0.0
    # cumulative crossing at index 2: drop the two smallest
    assert ad.error_thresh(np.array([1.0, 2.0, 3.0]), 3.5) == 2.0
    assert ad.error_thresh(np.array([]), 1.0) == 0.0
    assert ad.error_thresh(np.array([1.0, 2.0]), 3.0, offset=1.0) == 1.0
    assert list(ad.keep_from_list(np.array([3.0, 1.0, 2.0]), 3.5)) == [0]


def test_gt_precision_is_lexicographic():
    z = np.array([2e-8 - 1.0j, 1e-8 + 1e-3j, 1e-8 - 1e-3j, 5e-9 + 1.0j])
    assert gt_list(z) == [True, True, False, False]


def gt_list(z):
    return ad.gt_precision(z).tolist()


def test_adaptive_rejects_off_diagonal_lops(tmp_path):
    f = load("adaptive_chain8")
    sysp = system_param(f)
    l = np.array(sysp["L_HIER"][0])
    l[0, 1] = l[1, 0] = 1.0
    sysp["L_HIER"] = [l] + sysp["L_HIER"][1:]
    sysp["L_NOISE1"] = sysp["L_HIER"]
    hops = HopsTrajectory(sysp, noise_param={"MODEL": "ZERO", "TLEN": 100.0, "TAU": 2.0},
                          hierarchy_param={"MAXHIER": 2},
                          device_param={"DEVICE": "cpu"})
    hops.make_adaptive(1e-3, 1e-3)
    with pytest.raises(UnsupportedRequest):
        hops.initialize(f["psi0"])


def test_make_adaptive_validates_f_discard():
    f = load("adaptive_chain8")
    hops = HopsTrajectory(system_param(f), noise_param={"MODEL": "ZERO", "TLEN": 100.0,
                                                        "TAU": 2.0},
                          hierarchy_param={"MAXHIER": 2}, device_param={"DEVICE": "cpu"})
    with pytest.raises(UnsupportedRequest):
        hops.make_adaptive(1e-3, 1e-3, f_discard=2.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES + GPU_ONLY_CASES)
def test_adaptive_gpu_matches_reference(name, tmp_path):
    f = load(name)
    hops = make_traj(f, tmp_path, "cuda:0")
    hops.initialize(f["psi0"])
    hops.propagate(float(f["t_max"]), float(f["dt"]))
    check_against(hops, f)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_flux_errors_kernel_vs_oracle(name, tmp_path):
    """hops_flux_errors against the oracle formulas on the bases the run visits."""
    f = load(name)
    hops = make_traj(f, tmp_path, "cuda:0")
    hops.initialize(f["psi0"])
    hops.propagate(float(f["t_max"]) / 2, float(f["dt"]))
    drv = hops._adhops
    b = drv.basis
    ob = O.OracleSubBasis(system_param(f), b.states, b.modes, b.counts)
    rng = np.random.default_rng(5)
    phi = drv.phi / np.linalg.norm(drv.phi[:b.n_state])
    z_step = drv._z_step(drv.t, drv.zmem_abs + 0.3 * rng.normal(size=drv.zmem_abs.shape))
    for mask in (None, (rng.random(b.n_hier) > 0.3).astype(np.int32)):
        if mask is not None:
            mask[0] = 1
        req = ad.FluxRequest(drv, phi, z_step, float(f["dt"]), mask=mask)
        ed, eu, edn = ad.serve_flux([req], "cuda:0")[0]
        od, ou, odn = O.flux_errors(ob, phi, z_step[2][b.modes], z_step[0], z_step[1],
                                    float(f["dt"]), mask=mask)
        scale = max(np.max(od), 1e-300)
        assert np.max(np.abs(ed - od)) <= 1e-11 * scale
        assert np.allclose(eu, ou, rtol=1e-12, atol=1e-300)
        assert np.allclose(edn, odn, rtol=1e-12, atol=1e-300)


def test_state_mode_part_is_cached_and_read_only():
    """The state/mode-dependent part of an adaptive basis (tables, L blocks,
    M2 diagonal, the H couplings to states outside the basis) is built once per
    (states, modes) pair of a system, is read-only, and its coupling block is
    -i H[outside, basis]."""
    from mesohops_b200.system import HopsSystem
    from mesohops_b200.workloads import chain_sites
    sysp = chain_sites(12)
    system = HopsSystem(sysp)
    states = np.array([3, 4, 5], dtype=np.int64)
    modes = np.array([3, 4, 5], dtype=np.int64)
    p1 = ad._state_mode_part(system, states, modes)
    p2 = ad._state_mode_part(system, states.copy(), modes.copy())
    assert p1 is p2
    assert p1 is not ad._state_mode_part(system, np.array([3, 4], dtype=np.int64),
                                         np.array([3, 4], dtype=np.int64))
    assert p1["list_sc"].tolist() == [2, 6]
    H = np.asarray(sysp["HAMILTONIAN"])
    assert np.array_equal(p1["h_sc"], -1j * H[np.ix_([2, 6], states)])
    for arr in [p1["m2"], p1["list_sc"], p1["h_sc"]] + p1["lred"]:
        with pytest.raises(ValueError):
            arr[(0,) * arr.ndim] = 1


def test_chain500_reference_aux_sets_in_byte_key_order():
    """The reference's aux lists of the 500-site, depth-10 run (ranks beyond
    int64, so byte sort keys) are ordered by the same keys as the exact ranks,
    and every aux's k+1 / k-1 neighbours inside the set are found."""
    from mesohops_b200.hierarchy import AuxBasis, AuxKeyer
    f = load("adaptive_chain500")
    keyer = AuxKeyer(500, int(f["depth"]))
    assert not keyer.use_int64
    ptr, counts = f["aux_ptr"], f["aux_counts"]
    for i in range(len(ptr) - 1):
        c = counts[ptr[i]:ptr[i + 1]]
        b = AuxBasis(c, keyer, int(f["depth"]))
        exact = [int(x) for x in keyer.keys_from_counts(b.counts)]
        assert exact == sorted(exact) and len(set(exact)) == len(exact)
        rows = {r.tobytes(): j for j, r in enumerate(b.counts)}
        for a, u, m in zip(b.up_a, b.up_u, b.up_m):
            v = b.counts[a].copy()
            v[b.modes[m]] += 1
            assert rows[v.tobytes()] == u
        n_up = sum(1 for j, r in enumerate(b.counts) for m in range(len(b.modes))
                   if r.sum() < int(f["depth"])
                   and _plus(r, b.modes[m]).tobytes() in rows)
        assert n_up == len(b.up_a)


def _plus(r, m):
    v = r.copy()
    v[m] += 1
    return v
