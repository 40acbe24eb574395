"""Generate golden fixtures by running the UNMODIFIED MesoHOPS reference on CPU.

Run in a container that has the reference source tree (its ``src`` directory on
``MESOHOPS_SRC`` or at the default path below).  The outputs are small ``.npz``
files committed next to this script; the GPU box never needs the reference.

    python tests/golden/make_golden.py               # plain fixtures
    python tests/golden/make_golden.py --adaptive    # adaptive-basis fixtures
    python tests/golden/make_golden.py --effective   # EFFECTIVE_NOISE_INTEGRATION
    python tests/golden/make_golden.py --ltc         # low-temperature corrections
    python tests/golden/make_golden.py --ltc-adaptive  # the same with an adaptive basis
    python tests/golden/make_golden.py --dyadic      # DyadicTrajectory
    python tests/golden/make_golden.py --effective-adaptive  # effective noise, adaptive basis
    python tests/golden/make_golden.py --bench-configs  # the benchmark's ring20 / chain10
    python tests/golden/make_golden.py --static-basis   # STATIC_BASIS, adaptive
    python tests/golden/make_golden.py --interpolate    # INTERPOLATE noise

Each fixture records the inputs (system, hierarchy depth, noise arrays, psi_0,
time step) together with the reference outputs (psi_traj, derivative values,
correlated noise), so that tests can rebuild the same problem through
``mesohops_b200`` and the oracle.
"""
import os
import sys
import contextlib
import tempfile
import io

import numpy as np
import scipy.sparse as sps

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = os.environ.get("MESOHOPS_SRC", "/root/reference/src")
sys.path.insert(0, REF_SRC)

from mesohops.trajectory.hops_trajectory import HopsTrajectory  # noqa: E402
from mesohops.trajectory.exp_noise import bcf_exp  # noqa: E402
from mesohops.util.bath_corr_functions import bcf_convert_dl_to_exp  # noqa: E402


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def site_system(H, modes_per_site):
    n = H.shape[0]
    gw, lops = [], []
    for i in range(n):
        L = sps.coo_matrix(([1.0], ([i], [i])), shape=(n, n))
        for (lam, gam, T) in modes_per_site:
            g, w = bcf_convert_dl_to_exp(lam, gam, T)
            gw.append([g, w])
            lops.append(L)
    return {"HAMILTONIAN": np.array(H, dtype=np.complex128), "GW_SYSBATH": gw,
            "L_HIER": lops, "L_NOISE1": lops, "ALPHA_NOISE1": bcf_exp,
            "PARAM_NOISE1": gw}


def dense_lops(sysp):
    out = []
    for l in sysp["L_HIER"]:
        out.append(np.array(l.toarray() if sps.issparse(l) else l, dtype=np.complex128))
    return np.array(out)


def n_unique(sysp):
    keys = []
    for l in sysp["L_HIER"]:
        nz = l.nonzero() if sps.issparse(l) else np.nonzero(l)
        k = tuple(tuple(int(x) for x in v) for v in nz)
        if k not in keys:
            keys.append(k)
    return len(keys)


def run_precalc(name, sysp, depth, psi0, t_max, dt, noise_seed, noise2=None,
                eom="NORMALIZED NONLINEAR", extra=None, tau_noise=None, integration=None):
    """Propagate with PRE_CALCULATED noise; record psi_traj, phi, z_mem and derivatives.

    tau_noise: noise time step (default dt / 2); integration: integration_param
    of the reference trajectory (default: the reference's defaults)."""
    tau_noise = dt / 2.0 if tau_noise is None else tau_noise
    tlen = t_max + dt
    n_t = int(np.ceil(tlen / tau_noise)) + 1
    nl = n_unique(sysp)
    rng = np.random.default_rng(noise_seed)
    # Smooth-ish correlated-looking noise; exactly representable in complex64.
    noise = (rng.normal(size=(nl, n_t)) + 1j * rng.normal(size=(nl, n_t))) * 40.0
    noise = noise.astype(np.complex64)
    # The reference compares the two SEEDs with ==, which fails for two arrays:
    # hand both over as .npy file paths instead (hops_noise.py:271-283).
    tmpdir = tempfile.mkdtemp()
    path1 = os.path.join(tmpdir, "noise1.npy")
    np.save(path1, noise)
    noise_param = {"SEED": path1, "MODEL": "PRE_CALCULATED",
                   "TLEN": float(tlen), "TAU": float(tau_noise)}
    noise2_param = None
    if noise2 is not None:
        path2 = os.path.join(tmpdir, "noise2.npy")
        np.save(path2, noise2.astype(np.complex64))
        noise2_param = {"SEED": path2, "MODEL": "PRE_CALCULATED",
                        "TLEN": float(tlen), "TAU": float(tau_noise),
                        "FLAG_REAL": False}
        sysp = dict(sysp)
        sysp["L_NOISE2"] = sysp["L_HIER"]
        sysp["ALPHA_NOISE2"] = bcf_exp
        sysp["PARAM_NOISE2"] = sysp["GW_SYSBATH"]
    kw = {} if integration is None else {"integration_param": integration}
    hops = HopsTrajectory(sysp, noise_param=noise_param, noise2_param=noise2_param,
                          hierarchy_param={"MAXHIER": depth},
                          eom_param={"EQUATION_OF_MOTION": eom}, storage_param={}, **kw)
    quiet(hops.initialize, psi0)
    # one derivative at a random state with non-zero memory and noise
    nh, ns = hops.n_hier, hops.n_state
    phi_r = rng.normal(size=nh * ns) + 1j * rng.normal(size=nh * ns)
    zmem_r = (rng.normal(size=len(sysp["GW_SYSBATH"]))
              + 1j * rng.normal(size=len(sysp["GW_SYSBATH"]))) * 5.0
    z1_r = (rng.normal(size=nl) + 1j * rng.normal(size=nl)).astype(np.complex64) * 30
    z2_r = (rng.normal(size=nl) + 1j * rng.normal(size=nl)).astype(np.complex64) * 10
    zmem_sp = sps.csr_array(zmem_r.reshape(-1, 1))
    dphi_r, dz_r = hops.dsystem_dt(phi_r, zmem_sp, z1_r, z2_r)
    dz_r = np.asarray(dz_r.toarray()).ravel() if sps.issparse(dz_r) else np.asarray(dz_r)
    quiet(hops.propagate, t_max, dt)
    psi_traj = np.array(hops.storage.data["psi_traj"])
    t_axis = np.array(hops.storage.data["t_axis"])
    zmem_end = hops.z_mem.toarray().ravel() if sps.issparse(hops.z_mem) else hops.z_mem
    H = sysp["HAMILTONIAN"]
    H = H.toarray() if sps.issparse(H) else np.asarray(H)
    out = dict(
        H=np.array(H, dtype=np.complex128), G=np.array([g for g, w in sysp["GW_SYSBATH"]]),
        W=np.array([w for g, w in sysp["GW_SYSBATH"]]), L=dense_lops(sysp),
        depth=depth, psi0=np.array(psi0, dtype=np.complex128), t_max=t_max, dt=dt,
        tau_noise=tau_noise, tlen=tlen, noise1=noise,
        noise2=(noise2 if noise2 is not None else np.zeros_like(noise)),
        eom=eom, psi_traj=psi_traj, t_axis=t_axis, phi_end=np.array(hops.phi),
        zmem_end=np.array(zmem_end), n_hier=nh, n_state=ns,
        deriv_phi=phi_r, deriv_zmem=zmem_r, deriv_z1=z1_r, deriv_z2=z2_r,
        deriv_dphi=np.array(dphi_r), deriv_dz=np.array(dz_r),
        aux=np.array([a.todense() for a in hops.auxiliary_list], dtype=np.int64),
    )
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "n_hier", nh, "n_state", ns, "steps", len(psi_traj) - 1)


def make_noise_fixture():
    """Reference FFT_FILTER noise for the dimer (seed 0, SUM_GAUSSIAN and BOX_MULLER)."""
    H = np.array([[0, 50], [50, 0.0]])
    sysp = site_system(H, [(50, 50, 295)])
    out = {}
    for model in ("SUM_GAUSSIAN", "BOX_MULLER"):
        hops = HopsTrajectory(sysp, noise_param={"SEED": 0, "MODEL": "FFT_FILTER",
                                                 "TLEN": 1004.0, "TAU": 2.0,
                                                 "RAND_MODEL": model,
                                                 "STORE_RAW_NOISE": True},
                              hierarchy_param={"MAXHIER": 1}, storage_param={})
        z = quiet(hops.noise1.get_noise, list(np.arange(0, 1004.0 + 1e-9, 2.0)))
        out[model + "_eta"] = np.array(z)
        out[model + "_raw"] = np.array(hops.noise1.param["Z_UNCORRELATED"])
        out[model + "_alpha"] = np.complex64(hops.noise1._corr_func_by_lop_taxis(
            hops.noise1.param["T_AXIS"], [0, 1]))
    out["G"] = np.array([g for g, w in sysp["GW_SYSBATH"]])
    out["W"] = np.array([w for g, w in sysp["GW_SYSBATH"]])
    out["tau"] = 2.0
    out["tlen"] = 1004.0
    np.savez_compressed(os.path.join(HERE, "noise_dimer.npz"), **out)
    print("noise_dimer")


def main():
    # c1: dimer, depth 4 (15 aux x 2 states), dt 4 fs, 1000 fs
    H = np.array([[0, 50], [50, 0.0]])
    run_precalc("c1_dimer", site_system(H, [(50, 50, 295)]), 4,
                np.array([1, 0], dtype=np.complex128), 1000.0, 4.0, noise_seed=11)

    # dimer of dimers: 4 sites, two modes per site (DL + Markovian-like), depth 2
    hs = np.zeros((4, 4))
    hs[0, 1] = hs[1, 0] = 40
    hs[1, 2] = hs[2, 1] = 10
    hs[2, 3] = hs[3, 2] = 40
    g0, w0 = bcf_convert_dl_to_exp(20.0, 50.0, 140.0)
    gw, lops = [], []
    for i in range(4):
        L = np.zeros((4, 4))
        L[i, i] = 1.0
        gw.append([g0, w0])
        lops.append(sps.coo_matrix(L))
        gw.append([-1j * np.imag(g0), 500.0])
        lops.append(L)
    sysp = {"HAMILTONIAN": np.array(hs, dtype=np.complex128), "GW_SYSBATH": gw,
            "L_HIER": lops, "L_NOISE1": lops, "ALPHA_NOISE1": bcf_exp,
            "PARAM_NOISE1": gw}
    psi0 = np.zeros(4, dtype=np.complex128)
    psi0[2] = 1.0
    run_precalc("dod", sysp, 2, psi0, 200.0, 4.0, noise_seed=12)

    # general (off-diagonal, imaginary) L-operators, 3 states, 6 modes, depth 3
    lg = np.zeros((3, 3, 3), dtype=np.complex128)
    lg[0, 0, 1] = 1j
    lg[0, 1, 0] = -1j
    lg[1, 1, 2] = 1
    lg[1, 2, 1] = 1
    lg[2, 0, 0] = 0.5
    lg[2, 1, 1] = 1
    lg[2, 2, 2] = -1
    by_mode = [0, 0, 1, 1, 2, 2]
    gw6 = [[12.0, 18.0], [7.0, 3.0], [11.0, 9.0], [6.0, 4.0], [10.0, 10.0], [5.0, 5.0]]
    base_ham = np.array([[1.0, 14.0, 8.0], [14.0, 0, 10.0], [8.0, 10.0, -1.0]])
    sysg = {"HAMILTONIAN": base_ham, "GW_SYSBATH": gw6,
            "L_HIER": [lg[i] for i in by_mode], "L_NOISE1": [lg[i] for i in by_mode],
            "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw6}
    rngn2 = np.random.default_rng(99)
    n2 = (rngn2.normal(size=(3, int(np.ceil(21.0 / 0.5)) + 1)) * 3.0).astype(np.complex64)
    run_precalc("general_lop", sysg, 3, np.array([1, 0, 0], dtype=np.complex128),
                20.0, 1.0, noise_seed=13, noise2=n2)

    # small ring (c3 shape, reduced): 6 sites, one DL mode per site, depth 3
    n = 6
    rng = np.random.default_rng(2)
    H = np.diag(rng.uniform(-100, 100, n))
    for i in range(n):
        H[i, (i + 1) % n] = H[(i + 1) % n, i] = 80.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    run_precalc("ring6", site_system(H, [(60, 60, 295)]), 3, psi0, 200.0, 4.0,
                noise_seed=14)

    # chain with two modes per site (c2 shape, reduced): 4 sites, depth 3
    n = 4
    rng = np.random.default_rng(1)
    H = np.diag(rng.normal(0, 50, n))
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 100.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    run_precalc("chain4_2mode", site_system(H, [(35, 50, 300), (10, 500, 300)]), 3,
                psi0, 100.0, 2.0, noise_seed=15)

    # non-normalized nonlinear and linear EOM on the dimer
    H = np.array([[0, 50], [50, 0.0]])
    run_precalc("c1_nonlinear", site_system(H, [(50, 50, 295)]), 3,
                np.array([1, 0], dtype=np.complex128), 100.0, 4.0, noise_seed=16,
                eom="NONLINEAR")
    run_precalc("c1_linear", site_system(H, [(50, 50, 295)]), 3,
                np.array([1, 0], dtype=np.complex128), 100.0, 4.0, noise_seed=17,
                eom="LINEAR")

    make_noise_fixture()


def main_effective():
    """EFFECTIVE_NOISE_INTEGRATION: noise on a finer axis than dt / 2, averaged over
    windows of k = dt / (2 TAU) samples (k = 4, 5, 9: the short, 8-partial-sum and
    tail branches of numpy's pairwise sum)."""
    eff = {"INTEGRATOR": "RUNGE_KUTTA", "EFFECTIVE_NOISE_INTEGRATION": True}
    H = np.array([[0, 50], [50, 0.0]])
    run_precalc("eff_dimer_k4", site_system(H, [(50, 50, 295)]), 3,
                np.array([1, 0], dtype=np.complex128), 100.0, 4.0, noise_seed=21,
                tau_noise=0.5, integration=eff)
    n = 6
    rng = np.random.default_rng(2)
    Hr = np.diag(rng.uniform(-100, 100, n))
    for i in range(n):
        Hr[i, (i + 1) % n] = Hr[(i + 1) % n, i] = 80.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    n_t = int(np.ceil(64.0 / 0.4)) + 1
    n2 = (np.random.default_rng(98).normal(size=(n, n_t)) * 3.0).astype(np.complex64)
    run_precalc("eff_ring6_k5", site_system(Hr, [(60, 60, 295)]), 2, psi0, 60.0, 4.0,
                noise_seed=22, noise2=n2, tau_noise=0.4, integration=eff)
    run_precalc("eff_dimer_k9", site_system(H, [(50, 50, 295)]), 2,
                np.array([0, 1], dtype=np.complex128), 40.0, 4.0, noise_seed=23,
                tau_noise=2.0 / 9.0, integration=eff)


def with_ltc(sysp, lt_ops, lt_params):
    """System dictionary with low-temperature corrections (L_LT_CORR, PARAM_LT_CORR)."""
    out = dict(sysp)
    out["L_LT_CORR"] = list(lt_ops)
    out["PARAM_LT_CORR"] = list(lt_params)
    dense = np.array([np.array(l.toarray() if sps.issparse(l) else l, dtype=np.complex128)
                      for l in lt_ops])
    return out, {"LT_L": dense, "LT_P": np.array(lt_params, dtype=np.complex128)}


def main_ltc():
    """Low-temperature correction (eom_functions.py:215-309, hops_eom.py:357-403,
    527-529) on site projectors and on general L, for the three equations of
    motion; one correction names an L-operator of no bath and is dropped."""
    H = np.array([[0, 50], [50, 0.0]])
    base = site_system(H, [(50, 50, 295)])
    l0 = sps.coo_matrix(([1.0], ([0], [0])), shape=(2, 2))
    l1 = sps.coo_matrix(([1.0], ([1], [1])), shape=(2, 2))
    for eom, tag, seed in [("NORMALIZED NONLINEAR", "norm", 41), ("NONLINEAR", "nonlinear", 42),
                           ("LINEAR", "linear", 43)]:
        sysp, extra = with_ltc(base, [l0, l1], [0.25 - 0.1j, 0.125 + 0.05j])
        run_precalc("ltc_dimer_" + tag, sysp, 3, np.array([1, 0], dtype=np.complex128),
                    100.0, 4.0, noise_seed=seed, eom=eom, extra=extra)
    # ring of 6 sites, corrections on three sites plus one operator of no bath
    n = 6
    rng = np.random.default_rng(2)
    Hr = np.diag(rng.uniform(-100, 100, n))
    for i in range(n):
        Hr[i, (i + 1) % n] = Hr[(i + 1) % n, i] = 80.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    ops, pars = [], []
    for i, c in [(0, 0.2), (2, 0.1 - 0.05j), (4, 0.3j)]:
        ops.append(sps.coo_matrix(([1.0], ([i], [i])), shape=(n, n)))
        pars.append(c)
    stray = np.zeros((n, n))
    stray[0, 1] = stray[1, 0] = 1.0
    ops.append(stray)
    pars.append(0.5)
    sysp, extra = with_ltc(site_system(Hr, [(60, 60, 295)]), ops, pars)
    run_precalc("ltc_ring6", sysp, 2, psi0, 60.0, 4.0, noise_seed=44, extra=extra)
    # general (off-diagonal, imaginary) L-operators with noise 2
    lg = np.zeros((3, 3, 3), dtype=np.complex128)
    lg[0, 0, 1] = 1j
    lg[0, 1, 0] = -1j
    lg[1, 1, 2] = 1
    lg[1, 2, 1] = 1
    lg[2, 0, 0] = 0.5
    lg[2, 1, 1] = 1
    lg[2, 2, 2] = -1
    by_mode = [0, 0, 1, 1, 2, 2]
    gw6 = [[12.0, 18.0], [7.0, 3.0], [11.0, 9.0], [6.0, 4.0], [10.0, 10.0], [5.0, 5.0]]
    base_ham = np.array([[1.0, 14.0, 8.0], [14.0, 0, 10.0], [8.0, 10.0, -1.0]])
    sysg = {"HAMILTONIAN": base_ham, "GW_SYSBATH": gw6,
            "L_HIER": [lg[i] for i in by_mode], "L_NOISE1": [lg[i] for i in by_mode],
            "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw6}
    sysg, extra = with_ltc(sysg, [lg[0], lg[2]], [0.4 + 0.1j, 0.15])
    rngn2 = np.random.default_rng(97)
    n2 = (rngn2.normal(size=(3, int(np.ceil(21.0 / 0.5)) + 1)) * 3.0).astype(np.complex64)
    run_precalc("ltc_general", sysg, 3, np.array([1, 0, 0], dtype=np.complex128),
                20.0, 1.0, noise_seed=45, noise2=n2, extra=extra)


def main_ltc_adaptive():
    """Adaptive basis with low-temperature corrections on every site of a chain."""
    n = 8
    rng = np.random.default_rng(3)
    H = np.diag(rng.normal(0, 100, n))
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 50.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[n // 2] = 1.0
    ops = [sps.coo_matrix(([1.0], ([i], [i])), shape=(n, n)) for i in range(n)]
    pars = [0.2 - 0.05j * (i % 3) for i in range(n)]
    sysp, extra = with_ltc(site_system(H, [(50, 50, 295)]), ops, pars)
    run_adaptive("adaptive_chain8_ltc", sysp, 3, psi0, 120.0, 4.0, 3e-4, 3e-4, noise_seed=34,
                 extra=extra)


def run_adaptive(name, sysp, depth, psi0, t_max, dt, delta_a, delta_s, noise_seed,
                 update_step=1, f_discard=0.0, extra=None, tau_noise=None, integration=None,
                 site_map=None):
    """Adaptive propagation with PRE_CALCULATED noise; records the basis per step.
    tau_noise: noise time step (default dt / 2); integration: integration_param;
    site_map: for site-projector systems too large for dense L storage, the
    site of each mode's L = |site><site| is stored instead of L."""
    tau_noise = dt / 2.0 if tau_noise is None else tau_noise
    tlen = t_max + dt
    n_t = int(np.ceil(tlen / tau_noise)) + 1
    nl = n_unique(sysp)
    rng = np.random.default_rng(noise_seed)
    noise = ((rng.normal(size=(nl, n_t)) + 1j * rng.normal(size=(nl, n_t))) * 20.0).astype(np.complex64)
    tmpdir = tempfile.mkdtemp()
    path1 = os.path.join(tmpdir, "noise1.npy")
    np.save(path1, noise)
    hops = HopsTrajectory(sysp, noise_param={"SEED": path1, "MODEL": "PRE_CALCULATED",
                                             "TLEN": float(tlen), "TAU": float(tau_noise)},
                          hierarchy_param={"MAXHIER": depth},
                          eom_param={"EQUATION_OF_MOTION": "NORMALIZED NONLINEAR"},
                          storage_param={},
                          **({} if integration is None else {"integration_param": integration}))
    # adaptive_noise=False: the reference only supports sparse noise storage for
    # FFT_FILTER (hops_noise.py:244-245,320-323); values are the same either way
    hops.make_adaptive(delta_a, delta_s, update_step=update_step, f_discard=f_discard,
                       adaptive_noise=False)
    quiet(hops.initialize, psi0)
    quiet(hops.propagate, t_max, dt)
    d = hops.storage.data
    psi_full = np.array(hops.storage["psi_traj"])
    n_mode = len(sysp["GW_SYSBATH"])
    aux_counts = []
    aux_ptr = [0]
    for aux_list in d["aux_list"]:
        for a in aux_list:
            v = np.zeros(n_mode, dtype=np.int16)
            for (m, k) in np.asarray(a).reshape(-1, 2):
                v[m] = k
            aux_counts.append(v)
        aux_ptr.append(len(aux_counts))
    state_ptr = [0]
    states = []
    for sl in d["state_list"]:
        states.extend(list(sl))
        state_ptr.append(len(states))
    H = sysp["HAMILTONIAN"]
    H = H.toarray() if sps.issparse(H) else np.asarray(H)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        H=np.array(H, dtype=np.complex128), G=np.array([g for g, w in sysp["GW_SYSBATH"]]),
        W=np.array([w for g, w in sysp["GW_SYSBATH"]]), depth=depth,
        **({"L": dense_lops(sysp)} if site_map is None else {"L_site": np.asarray(site_map)}),
        psi0=np.array(psi0, dtype=np.complex128), t_max=t_max, dt=dt, tau_noise=tau_noise,
        tlen=tlen, noise1=noise, delta_a=delta_a, delta_s=delta_s, update_step=update_step,
        f_discard=f_discard, psi_traj=psi_full, t_axis=np.array(d["t_axis"]),
        list_nhier=np.array(d["list_nhier"]), list_nstate=np.array(d["list_nstate"]),
        aux_counts=np.array(aux_counts, dtype=np.int16).reshape(-1, n_mode),
        aux_ptr=np.array(aux_ptr), states=np.array(states), state_ptr=np.array(state_ptr),
        phi_end=np.array(hops.phi), n_hier_end=hops.n_hier, n_state_end=hops.n_state,
        **(extra or {}))
    print(name, "adaptive steps", len(psi_full) - 1, "n_hier", list(d["list_nhier"])[:8],
          "n_state", list(d["list_nstate"])[:8])


def main_adaptive():
    # dimer of dimers, tiny delta_a: the adaptive basis must equal the full one
    hs = np.zeros((4, 4))
    hs[0, 1] = hs[1, 0] = 40
    hs[1, 2] = hs[2, 1] = 10
    hs[2, 3] = hs[3, 2] = 40
    g0, w0 = bcf_convert_dl_to_exp(20.0, 50.0, 140.0)
    gw, lops = [], []
    for i in range(4):
        L = np.zeros((4, 4))
        L[i, i] = 1.0
        gw.append([g0, w0])
        lops.append(sps.coo_matrix(L))
        gw.append([-1j * np.imag(g0), 500.0])
        lops.append(L)
    sysp = {"HAMILTONIAN": np.array(hs, dtype=np.complex128), "GW_SYSBATH": gw,
            "L_HIER": lops, "L_NOISE1": lops, "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw}
    psi0 = np.zeros(4, dtype=np.complex128)
    psi0[2] = 1.0
    run_adaptive("adaptive_dod_full", sysp, 2, psi0, 80.0, 4.0, 1e-15, 1e-100, noise_seed=31)
    # chains with a moderate threshold (the adaptive benchmark shape, reduced)
    for (name, n, depth, delta, seed) in [("adaptive_chain8", 8, 3, 3e-4, 32),
                                          ("adaptive_chain12", 12, 4, 1e-3, 33)]:
        rng = np.random.default_rng(3)
        eps = rng.normal(0, 100, n)
        H = np.diag(eps)
        for i in range(n - 1):
            H[i, i + 1] = H[i + 1, i] = 50.0
        psi0 = np.zeros(n, dtype=np.complex128)
        psi0[n // 2] = 1.0
        run_adaptive(name, site_system(H, [(50, 50, 295)]), depth, psi0, 120.0, 4.0,
                     delta, delta, noise_seed=seed)


def run_interpolate(name, sysp, depth, psi0, t_max, dt, noise_seed, eom):
    """INTERPOLATE noise: a complex128 SEED array through the reference's cubic
    spline (hops_noise.py:255-265), sampled at the step times."""
    tau_noise = dt / 2.0
    tlen = t_max + dt
    n_t = int(np.ceil(tlen / tau_noise)) + 1
    nl = n_unique(sysp)
    rng = np.random.default_rng(noise_seed)
    noise = (rng.normal(size=(nl, n_t)) + 1j * rng.normal(size=(nl, n_t))) * 40.0
    hops = HopsTrajectory(sysp, noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                             "TLEN": float(tlen), "TAU": float(tau_noise),
                                             "INTERPOLATE": True},
                          hierarchy_param={"MAXHIER": depth},
                          eom_param={"EQUATION_OF_MOTION": eom}, storage_param={})
    quiet(hops.initialize, psi0)
    quiet(hops.propagate, t_max, dt)
    H = sysp["HAMILTONIAN"]
    H = H.toarray() if sps.issparse(H) else np.asarray(H)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        H=np.array(H, dtype=np.complex128), G=np.array([g for g, w in sysp["GW_SYSBATH"]]),
        W=np.array([w for g, w in sysp["GW_SYSBATH"]]), L=dense_lops(sysp), depth=depth,
        psi0=np.array(psi0, dtype=np.complex128), t_max=t_max, dt=dt, tau_noise=tau_noise,
        tlen=tlen, noise1=noise, eom=eom, psi_traj=np.array(hops.storage.data["psi_traj"]),
        n_hier=hops.n_hier, n_state=hops.n_state)
    print(name, "steps", len(hops.storage.data["psi_traj"]) - 1)


def main_interpolate():
    n = 6
    rng = np.random.default_rng(2)
    H = np.diag(rng.uniform(-100, 100, n))
    for i in range(n):
        H[i, (i + 1) % n] = H[(i + 1) % n, i] = 80.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    run_interpolate("interp_ring6", site_system(H, [(60, 60, 295)]), 3, psi0, 100.0, 4.0,
                    noise_seed=71, eom="NORMALIZED NONLINEAR")
    H = np.array([[0, 50], [50, 0.0]])
    run_interpolate("interp_dimer_linear", site_system(H, [(50, 50, 295)]), 3,
                    np.array([1, 0], dtype=np.complex128), 100.0, 4.0, noise_seed=72,
                    eom="LINEAR")


def main_static_basis():
    """Adaptive basis with integration_param STATIC_BASIS (states and aux joined
    to the initial basis, hops_trajectory.py:293-316), with the INCH_WORM early
    integrator and with STATIC_STATE_INCHWORM_HIERARCHY (the state basis of the
    early steps fixed to the static states, :477-491)."""
    from mesohops.basis.hops_aux import AuxiliaryVector
    n = 12
    rng = np.random.default_rng(3)
    eps = rng.normal(0, 100, n)
    H = np.diag(eps)
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 50.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[n // 2] = 1.0
    static_states = [4, 5, 6, 7]
    static_aux_pairs = [[(6, 1)], [(5, 1), (6, 1)], [(7, 2)]]
    rows = np.zeros((len(static_aux_pairs), n), dtype=np.int16)
    for i, pairs in enumerate(static_aux_pairs):
        for m, k in pairs:
            rows[i, m] = k
    for name, early in (("adaptive_static_inchworm", "INCH_WORM"),
                        ("adaptive_static_state", "STATIC_STATE_INCHWORM_HIERARCHY")):
        integ = {"INTEGRATOR": "RUNGE_KUTTA", "EARLY_ADAPTIVE_INTEGRATOR": early,
                 "STATIC_BASIS": [list(static_states),
                                  [AuxiliaryVector(p, n) for p in static_aux_pairs]]}
        run_adaptive(name, site_system(H, [(50, 50, 295)]), 4, psi0, 80.0, 4.0, 1e-3, 1e-3,
                     noise_seed=61, integration=integ,
                     extra={"static_states": np.array(static_states),
                            "static_aux": rows, "early_integrator": early})


def run_dyadic(name, eom, sparse_input, noise_seed, adaptive=None):
    """DyadicTrajectory (trajectory/hops_dyadic.py) on a 3-site system with a
    ground state: ket and bra excitations, propagation, a bra de-excitation,
    more propagation; records the states after each operator, psi_traj, the
    response normalisation factors and a response-function component."""
    from mesohops.trajectory.hops_dyadic import DyadicTrajectory
    nsite = 3
    H = np.zeros((nsite + 1, nsite + 1))
    H[1:, 1:] = [[0.0, 50.0, 0.0], [50.0, 30.0, 40.0], [0.0, 40.0, -20.0]]
    lops = []
    for i in range(1, nsite + 1):
        L = np.zeros((nsite + 1, nsite + 1))
        L[i, i] = 1.0
        lops.append(sps.coo_matrix(L) if sparse_input else L)
    gw = [list(bcf_convert_dl_to_exp(50.0, 50.0, 295.0)) for _ in range(nsite)]
    sysp = {"HAMILTONIAN": sps.coo_matrix(H) if sparse_input else H, "GW_SYSBATH": gw,
            "L_HIER": lops, "L_NOISE1": lops, "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw}
    dt, t1 = 2.0, 10.0
    tau_noise, tlen = dt / 2, 2 * t1 + 2 * dt
    n_t = int(np.ceil(tlen / tau_noise)) + 1
    rng = np.random.default_rng(noise_seed)
    noise = ((rng.normal(size=(nsite, n_t)) + 1j * rng.normal(size=(nsite, n_t))) * 20.0
             ).astype(np.complex64)
    path = os.path.join(tempfile.mkdtemp(), "noise1.npy")
    np.save(path, noise)
    hops = DyadicTrajectory(sysp, noise_param={"SEED": path, "MODEL": "PRE_CALCULATED",
                                               "TLEN": float(tlen), "TAU": float(tau_noise)},
                            hierarchy_param={"MAXHIER": 2},
                            eom_param={"EQUATION_OF_MOTION": eom}, storage_param={})
    if adaptive is not None:
        hops.make_adaptive(adaptive[0], adaptive[1], adaptive_noise=False)
    psi_k = np.array([1.0, 0, 0, 0], dtype=np.complex128)
    psi_b = np.array([1.0, 0, 0, 0], dtype=np.complex128)
    op_ket = np.zeros((nsite + 1, nsite + 1))
    op_ket[1:, 0] = [1.0, 0.5, 0.25]
    op_bra = np.zeros((nsite + 1, nsite + 1))
    op_bra[1:, 0] = [0.3, 1.0, 0.6]
    op_down = np.zeros((nsite + 1, nsite + 1))
    op_down[0, 1:] = 1.0
    conv = (lambda m: sps.coo_matrix(m)) if sparse_input else (lambda m: m)
    quiet(hops.initialize, psi_k, psi_b)
    psi_init = np.array(hops.psi)
    quiet(hops._dyad_operator, conv(op_ket), "ket")
    psi_op1 = np.array(hops.psi)
    quiet(hops._dyad_operator, conv(op_bra), "bra")
    psi_op2 = np.array(hops.psi)
    quiet(hops.propagate, t1, dt)
    quiet(hops._dyad_operator, conv(op_down), "bra")
    psi_op3 = np.array(hops.psi)
    quiet(hops.propagate, t1, dt)
    f_op = np.zeros((2 * (nsite + 1), 2 * (nsite + 1)))
    f_op[nsite + 1, 0] = 1.0      # |bra ground><ket ground|
    resp = hops._response_function_comp(f_op, 5)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        H=H, G=np.array([g for g, w in gw]), W=np.array([w for g, w in gw]),
        L=np.array([np.array(l.toarray() if sps.issparse(l) else l) for l in lops]),
        sparse_input=sparse_input, eom=eom, depth=2, dt=dt, t1=t1, tau_noise=tau_noise,
        tlen=tlen, noise1=noise, psi_k=psi_k, psi_b=psi_b, op_ket=op_ket, op_bra=op_bra,
        op_down=op_down, f_op=f_op, psi_init=psi_init, psi_op1=psi_op1, psi_op2=psi_op2,
        psi_op3=psi_op3, psi_traj=np.array(hops.storage["psi_traj"]),
        t_axis=np.array(hops.storage["t_axis"]), phi_end=np.array(hops.phi),
        norm_sq=np.array(hops.list_response_norm_sq), response=np.array(resp),
        adaptive=np.array(adaptive if adaptive is not None else [0.0, 0.0]))
    print(name, "n_hier", hops.n_hier, "n_state", hops.n_state, "norms",
          np.round(hops.list_response_norm_sq, 4))


def main_effective_adaptive():
    """Adaptive basis with EFFECTIVE_NOISE_INTEGRATION (noise axis dt / 8, windows
    of 4 samples); the reference's inch-worm sub-steps take the plain samples."""
    n = 8
    rng = np.random.default_rng(3)
    H = np.diag(rng.normal(0, 100, n))
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 50.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[n // 2] = 1.0
    eff = {"INTEGRATOR": "RUNGE_KUTTA", "EFFECTIVE_NOISE_INTEGRATION": True}
    run_adaptive("adaptive_chain8_eff", site_system(H, [(50, 50, 295)]), 3, psi0, 120.0, 4.0,
                 3e-4, 3e-4, noise_seed=35, tau_noise=0.5, integration=eff)


def main_adaptive_chain500():
    """The adaptive batch workload of the benchmark: 500-site chain (J = 50,
    eps ~ N(0, 100) and psi_0's site from default_rng(3)), one DL mode
    (50, 50, 295 K) per site, depth 10, delta_a = delta_s = 1e-3, 20 steps of
    4 fs, with seeded PRE_CALCULATED noise."""
    n = 500
    rng = np.random.default_rng(3)
    eps = rng.normal(0, 100, n)
    start = int(rng.integers(0, n))
    H = np.diag(eps)
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 50.0
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[start] = 1.0
    run_adaptive("adaptive_chain500", site_system(H, [(50, 50, 295)]), 10, psi0, 80.0, 4.0,
                 1e-3, 1e-3, noise_seed=37, site_map=np.arange(n))


def main_dyadic():
    run_dyadic("dyadic_norm_dense", "NORMALIZED NONLINEAR", False, noise_seed=51)
    run_dyadic("dyadic_linear_sparse", "LINEAR", True, noise_seed=52)
    run_dyadic("dyadic_adaptive", "NORMALIZED NONLINEAR", False, noise_seed=53,
               adaptive=(1e-3, 1e-3))


def _ring20_fft_run(seed):
    """One trajectory of the benchmark's 20-site ring with the reference's own
    FFT_FILTER noise of SEED seed: (psi_traj, complex64 correlated noise)."""
    n = 20
    rng = np.random.default_rng(2)
    H = np.diag(rng.uniform(-100, 100, n))
    for i in range(n):
        H[i, (i + 1) % n] = H[(i + 1) % n, i] = 80.0
    sysp = site_system(H, [(60, 60, 295)])
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    hops = HopsTrajectory(sysp, noise_param={"SEED": seed, "MODEL": "FFT_FILTER",
                                             "TLEN": 1004.0, "TAU": 2.0},
                          hierarchy_param={"MAXHIER": 4}, storage_param={})
    quiet(hops.initialize, psi0)
    quiet(hops.propagate, 1000.0, 4.0)
    eta = quiet(hops.noise1.get_noise, list(np.arange(0, 1004.0 + 1e-9, 2.0)))
    return np.array(hops.storage.data["psi_traj"]), np.array(eta, dtype=np.complex64)


def main_bench_configs():
    """Reference runs of the benchmark configurations themselves.

    c3_ring20: 20-site ring (J = 80, eps ~ U(-100, 100) from default_rng(2)), one DL
    mode (60, 60, 295 K) per site, depth 4 (10626 aux x 20 states), psi_0 = |0>,
    dt = 4 fs, 250 steps, FFT_FILTER noise of SEED 0..3 (TLEN 1004, TAU 2); the
    reference's complex64 correlated noise is stored so that the trajectories can
    be rerun exactly (as PRE_CALCULATED noise).
    c2_chain10: 10-site chain (J = 100, eps ~ N(0, 50) from default_rng(1)), DL
    modes (35, 50, 300 K) + (10, 500, 300 K) per site, depth 6 (230230 aux x 10
    states), dt = 2 fs, 5 steps, seeded PRE_CALCULATED noise for two
    trajectories; psi_traj plus a fixed sample of 4096 phi entries and
    sum |phi|^2 at the end (phi itself is 37 MB)."""
    from concurrent.futures import ProcessPoolExecutor
    seeds = [0, 1, 2, 3]
    with ProcessPoolExecutor(4) as ex:
        runs = list(ex.map(_ring20_fft_run, seeds))
    np.savez_compressed(os.path.join(HERE, "c3_ring20.npz"), seeds=np.array(seeds),
                        psi_traj=np.array([r[0] for r in runs]),
                        noise1=np.array([r[1] for r in runs]), depth=4, dt=4.0,
                        tau_noise=2.0, tlen=1004.0, t_max=1000.0)
    print("c3_ring20", [r[0].shape for r in runs])

    n = 10
    rng = np.random.default_rng(1)
    H = np.diag(rng.normal(0, 50, n))
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 100.0
    sysp = site_system(H, [(35, 50, 300), (10, 500, 300)])
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[0] = 1.0
    out = {}
    for k, seed in enumerate((41, 42)):
        tlen, tau = 12.0, 1.0
        n_t = int(np.ceil(tlen / tau)) + 1
        r = np.random.default_rng(seed)
        noise = ((r.normal(size=(n, n_t)) + 1j * r.normal(size=(n, n_t))) * 40.0
                 ).astype(np.complex64)
        tmp = tempfile.mkdtemp()
        path = os.path.join(tmp, "noise1.npy")
        np.save(path, noise)
        hops = HopsTrajectory(sysp, noise_param={"SEED": path, "MODEL": "PRE_CALCULATED",
                                                 "TLEN": tlen, "TAU": tau},
                              hierarchy_param={"MAXHIER": 6}, storage_param={})
        quiet(hops.initialize, psi0)
        quiet(hops.propagate, 10.0, 2.0)
        phi = np.array(hops.phi)
        idx = np.random.default_rng(7).choice(len(phi), 4096, replace=False)
        out[f"noise1_{k}"] = noise
        out[f"psi_traj_{k}"] = np.array(hops.storage.data["psi_traj"])
        out[f"phi_idx_{k}"] = idx
        out[f"phi_sample_{k}"] = phi[idx]
        out[f"phi_norm2_{k}"] = float(np.sum(np.abs(phi) ** 2))
        out["n_hier"] = hops.n_hier
    np.savez_compressed(os.path.join(HERE, "c2_chain10.npz"), depth=6, dt=2.0, tau_noise=1.0,
                        tlen=12.0, t_max=10.0, n_traj=2, **out)
    print("c2_chain10", out["n_hier"])


if __name__ == "__main__":
    if "--bench-configs" in sys.argv:
        main_bench_configs()
    elif "--static-basis" in sys.argv:
        main_static_basis()
    elif "--interpolate" in sys.argv:
        main_interpolate()
    elif "--dyadic" in sys.argv:
        main_dyadic()
    elif "--effective-adaptive" in sys.argv:
        main_effective_adaptive()
    elif "--adaptive-chain500" in sys.argv:
        main_adaptive_chain500()
    elif "--adaptive" in sys.argv:
        main_adaptive()
    elif "--effective" in sys.argv:
        main_effective()
    elif "--ltc" in sys.argv:
        main_ltc()
    elif "--ltc-adaptive" in sys.argv:
        main_ltc_adaptive()
    else:
        main()
