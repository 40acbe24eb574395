"""CPU oracle for the HOPS trajectory hot path -- TEST INFRASTRUCTURE ONLY.

This module is a plain numpy/scipy restatement of the MesoHOPS (v1.6) algorithms
that the CUDA path in ``mesohops_b200`` replaces.  It exists only so that tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` can check the
GPU results.  Nothing in the product package imports it, and it is never the
thing that is measured as the GPU result.

Every function cites the reference file:line it restates (paths relative to the
MesoHOPS source tree ``src/mesohops``).

Parity status: pinned.  ``tests/test_oracle_pin.py`` checks this module against
(a) the reference's own golden arrays (dimer-of-dimers super-operators, alpha,
eta) when the reference tree is present, and (b) committed fixtures generated
by running the unmodified reference (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import itertools

import numpy as np
import scipy.sparse as sps

# util/physical_constants.py:21,26-28
PRECISION = 1e-8
H_PLANCK = 33357.179          # cm^-1 fs
HBAR = H_PLANCK / (2 * np.pi)  # cm^-1 fs / rad
KB = 0.69503                  # cm^-1 / K


# ---------------------------------------------------------------------------
# Bath correlation functions
# ---------------------------------------------------------------------------
def bcf_exp(t_axis, g, w):
    """alpha(t) = g exp(-w t / hbar).  trajectory/exp_noise.py:5-25"""
    return g * np.exp(-w * np.asarray(t_axis) / HBAR)


def dl_to_exp(lam, gam, temp):
    """High-temperature Drude-Lorentz mode (no Matsubara terms).

    util/bath_corr_functions.py:70-112 with k_matsubara=0:
    g = 2 lambda kB T - i lambda gamma, w = gamma.
    """
    beta = 1.0 / (KB * temp)
    return [2 * lam / beta - 1j * lam * gam, gam]


# ---------------------------------------------------------------------------
# System parameter expansion
# ---------------------------------------------------------------------------
def _pattern_key(lop):
    """Unique-L key = tuple of nonzero (rows, cols).  util/helper_functions.py:8-32"""
    if sps.issparse(lop):
        nz = lop.nonzero()
    else:
        nz = np.nonzero(np.asarray(lop))
    return tuple(tuple(int(x) for x in l) for l in nz)


def expand_system(sys_param):
    """Subset of basis/system_functions.py:10-172 needed by the hot path.

    Returns dict with H (dense complex), G, W, the unique L list (dense, values of
    the first mode with that nonzero pattern), the mode -> unique-L map and LT,
    the low-temperature correction coefficient of each unique L: the sum of the
    PARAM_LT_CORR entries whose L_LT_CORR has that nonzero pattern; entries
    matching no L_HIER operator are dropped (system_functions.py:115-133).
    """
    H = sys_param["HAMILTONIAN"]
    H = H.toarray() if sps.issparse(H) else np.asarray(H)
    H = np.array(H, dtype=np.complex128)
    gw = sys_param["GW_SYSBATH"]
    G = np.array([g for g, _ in gw], dtype=np.complex128)
    W = np.array([w for _, w in gw], dtype=np.complex128)
    lops = sys_param["L_HIER"]
    keys = [_pattern_key(l) for l in lops]
    uniq = {}
    l_unique = []
    l_by_mode = []
    for m, k in enumerate(keys):
        if k not in uniq:
            uniq[k] = len(l_unique)
            lm = lops[m]
            lm = lm.toarray() if sps.issparse(lm) else np.asarray(lm)
            l_unique.append(np.array(lm, dtype=np.complex128))
        l_by_mode.append(uniq[k])
    lt = np.zeros(len(l_unique), dtype=np.complex128)
    for lop, c in zip(sys_param.get("L_LT_CORR", []), sys_param.get("PARAM_LT_CORR", [])):
        j = uniq.get(_pattern_key(lop))
        if j is not None:
            lt[j] += c
    return {"H": H, "G": G, "W": W, "L": l_unique,
            "L_BY_MODE": np.array(l_by_mode, dtype=np.int64),
            "NSTATE": H.shape[0], "NMODE": len(gw), "LT": lt}


# ---------------------------------------------------------------------------
# Hierarchy
# ---------------------------------------------------------------------------
def triangular_aux(n_modes, maxhier):
    """All aux vectors with total depth <= maxhier, in the reference order.

    basis/hops_hierarchy.py:340-368 generates combinations-with-replacement by
    depth; the auxiliary_list setter (hops_hierarchy.py:582) then sorts by the id
    string of hops_aux.py:460-480 (shorter first, then lexicographic), which for
    fixed-width mode digits is exactly depth-then-lexicographic order of the
    sorted mode tuple, i.e. generation order.
    """
    rows = []
    for k in range(maxhier + 1):
        for combo in itertools.combinations_with_replacement(range(n_modes), k):
            v = np.zeros(n_modes, dtype=np.int64)
            for m in combo:
                v[m] += 1
            rows.append(v)
    return np.array(rows, dtype=np.int64).reshape(-1, n_modes)


def aux_sort_key(vec):
    """Sort key equal to the reference id ordering (hops_aux.py:171-177,460-480)."""
    combo = []
    for m, k in enumerate(vec):
        combo.extend([m] * int(k))
    return (len(combo), tuple(combo))


class OracleBasis:
    """Static (non-adaptive) basis: every state, every mode, given aux list."""

    def __init__(self, sys_param, maxhier=None, aux=None):
        self.sys = expand_system(sys_param)
        s = self.sys
        self.nstate = s["NSTATE"]
        self.nmode = s["NMODE"]
        if aux is None:
            aux = triangular_aux(self.nmode, maxhier)
        self.aux = np.asarray(aux, dtype=np.int64)
        self.nhier = len(self.aux)
        self.index = {tuple(v): i for i, v in enumerate(self.aux)}
        self._build_super_operators()

    def _build_super_operators(self):
        """K2_k, K2_kp1, K2_km1, Z2_kp1 -- eom/eom_hops_ksuper.py:36-90,93-230,575-668.

        K2_k[a,a]             = -sum_m k_m w_m
        K2_kp1[a*S+r, u*S+c]  = -(g_m/w_m) L_m[r,c]     for u = a + e_m
        K2_km1[u*S+c, a*S+r]  = k_m(u) w_m conj(L_m[r,c])
        Z2_kp1[l][a, u]       = g_m / w_m               for l = l(m)
        """
        s = self.sys
        S, N = self.nstate, self.nhier
        G, W = s["G"], s["W"]
        self.k2_k = -(self.aux.astype(np.complex128) @ W)
        kp_r, kp_c, kp_v = [], [], []
        km_v = []
        z_rows = [[] for _ in s["L"]]
        z_cols = [[] for _ in s["L"]]
        z_vals = [[] for _ in s["L"]]
        for a, vec in enumerate(self.aux):
            for m in range(self.nmode):
                up = vec.copy()
                up[m] += 1
                u = self.index.get(tuple(up))
                if u is None:
                    continue
                lm = s["L"][s["L_BY_MODE"][m]]
                rr, cc = np.nonzero(lm)
                for r, c in zip(rr, cc):
                    kp_r.append(a * S + r)
                    kp_c.append(u * S + c)
                    kp_v.append(-(G[m] / W[m]) * lm[r, c])
                    km_v.append(up[m] * W[m] * np.conj(lm[r, c]))
                j = s["L_BY_MODE"][m]
                z_rows[j].append(a)
                z_cols[j].append(u)
                z_vals[j].append(G[m] / W[m])
        n_tot = N * S
        self.k2_kp1 = sps.coo_matrix((kp_v, (kp_r, kp_c)), shape=(n_tot, n_tot),
                                     dtype=np.complex128).tocsr()
        self.k2_km1 = sps.coo_matrix((km_v, (kp_c, kp_r)), shape=(n_tot, n_tot),
                                     dtype=np.complex128).tocsr()
        self.z2_kp1 = [sps.coo_matrix((z_vals[j], (z_rows[j], z_cols[j])),
                                      shape=(N, N), dtype=np.complex128).tocsr()
                       for j in range(len(s["L"]))]
        self.k2_stable = (self.k2_kp1 + self.k2_km1).tocsr()
        # first-level aux per mode (hops_eom.py:186-194)
        self.first_level = []
        for m in range(self.nmode):
            e = np.zeros(self.nmode, dtype=np.int64)
            e[m] = 1
            i = self.index.get(tuple(e))
            if i is not None:
                self.first_level.append((i, int(s["L_BY_MODE"][m]), m))
        # active L: every unique L touches at least one state of the full basis
        self.l_active = [j for j, l in enumerate(s["L"]) if np.any(l != 0)]
        # masked sub-blocks of L_j and Z2_kp1[j], as hops_modes.py:158-161 and
        # eom_hops_ksuper.py:663-666 build them for hops_eom.py:410-425
        self.l_mask = []
        for l in s["L"]:
            r, c = np.nonzero(l)
            rows, cols = np.unique(r), np.unique(c)
            self.l_mask.append((rows, cols, np.asarray(l)[np.ix_(rows, cols)]))
        self.z_mask = []
        for z in self.z2_kp1:
            rows = np.unique(z.nonzero()[0])
            self.z_mask.append((rows, z[rows]))


# ---------------------------------------------------------------------------
# Equation of motion (normalized nonlinear / nonlinear / linear)
# ---------------------------------------------------------------------------
def dsystem_dt(basis, phi, zmem, z1, z2, eom="NORMALIZED NONLINEAR"):
    """Derivative of phi (cm^-1 units, caller divides by hbar) and of z_mem.

    Restates eom/hops_eom.py:196-441 (nonlinear, normalized or not) and
    hops_eom.py:445-542 (LINEAR), with eom/eom_functions.py:11-213 for <L>,
    compress_zmem, calc_delta_zmem and calc_norm_corr.  z1, z2 are indexed by the
    unique-L list; zmem by mode.
    """
    s = basis.sys
    S, N = basis.nstate, basis.nhier
    L = s["L"]
    phi = np.asarray(phi, dtype=np.complex128)
    zmem = np.asarray(zmem, dtype=np.complex128)
    z1 = np.asarray(z1)
    z2 = np.asarray(z2)
    pf = phi.reshape(N, S)  # row a = aux, column = state
    lt = s.get("LT", np.zeros(len(L)))
    has_lt = bool(np.any(lt))
    if eom == "LINEAR":
        dphi = basis.k2_stable @ phi
        d = dphi.reshape(N, S)
        d += basis.k2_k[:, None] * pf
        d += pf @ (-1j * s["H"]).T
        if has_lt:
            # calc_LT_corr_linear (eom_functions.py:284-309), physical wavefunction only
            d[0] += -sum(lt[j] * (L[j] @ L[j]) for j in range(len(L))) @ pf[0]
        for j in range(len(L)):
            rows, cols, lsub = basis.l_mask[j]
            d[:, rows] += (np.conj(z1[j]) - 1j * z2[j]) * (pf[:, cols] @ lsub.T)
        return dphi, np.zeros_like(zmem)

    normalized = eom == "NORMALIZED NONLINEAR"
    # compress_zmem: eom_functions.py:32-62
    zhat = np.conj(z1).astype(np.complex128)
    for m in range(basis.nmode):
        zhat[s["L_BY_MODE"][m]] += zmem[m]
    psi0 = pf[0]
    n2 = np.vdot(psi0, psi0)
    avg = np.array([np.vdot(psi0, L[j] @ psi0) / n2 for j in range(len(L))])
    act = basis.l_active
    nc = 0.0
    if normalized:
        # calc_norm_corr: eom_functions.py:163-213
        delta = np.dot(zhat[act], avg[act])
        for (ia, j, m) in basis.first_level:
            phi1 = (s["G"][m] / s["W"][m]) * pf[ia]
            delta -= np.vdot(psi0, L[j] @ phi1)
            delta += np.vdot(psi0, phi1) * avg[j]
        nc = np.real(delta)
    dphi = basis.k2_stable @ phi
    d = dphi.reshape(N, S)
    d += basis.k2_k[:, None] * pf
    d += pf @ (-1j * s["H"]).T
    if has_lt:
        # calc_LT_corr / calc_LT_corr_to_norm_corr (eom_functions.py:215-281),
        # applied as hops_eom.py:357-403
        l2 = [L[j] @ L[j] for j in range(len(L))]
        avg2 = np.array([np.vdot(psi0, l2[j] @ psi0) / n2 for j in range(len(L))])
        c_phys = sum(lt[j] * avg[j] * L[j] - lt[j] * l2[j] for j in act)
        c_hier = sum(np.conj(lt[j]) * avg[j] * L[j] for j in act)
        d += pf @ np.asarray(c_hier).T
        d[0] += np.asarray(c_phys) @ pf[0]
        if normalized:
            nc = nc + np.sum(np.real(lt[act]) * (2 * avg[act] ** 2 - avg2[act]))
    if normalized:
        d -= nc * pf
    for j in act:
        rows, cols, lsub = basis.l_mask[j]
        d[:, rows] += (zhat[j] - 1j * z2[j]) * (pf[:, cols] @ lsub.T)
        zrows, zsub = basis.z_mask[j]
        if len(zrows):
            d[zrows] += np.conj(avg[j]) * (zsub @ pf)
    # calc_delta_zmem: eom_functions.py:65-160 (all modes in basis)
    dz = np.conj(s["G"]) * avg[s["L_BY_MODE"]] - np.conj(s["W"]) * zmem
    return dphi, dz


def rk4_step(basis, phi, zmem, z_rnd, z_rnd2, tau, eom="NORMALIZED NONLINEAR"):
    """Classic RK4.  integrator/integrator_rk.py:10-75.

    z_rnd / z_rnd2 are [n_L, 3] noise samples at t, t+tau/2, t+tau.
    """
    c_rk = (0.0, 0.5, 0.5, 1.0)
    i_z = (0, 1, 1, 2)
    k = [None] * 4
    kz = [None] * 4
    for i in range(4):
        if i == 0:
            p, z = phi, zmem
        else:
            p = phi + c_rk[i] * k[i - 1] * tau / HBAR
            z = zmem + c_rk[i] * kz[i - 1] * tau / HBAR
        k[i], kz[i] = dsystem_dt(basis, p, z, z_rnd[:, i_z[i]], z_rnd2[:, i_z[i]], eom)
    phi = phi + tau / HBAR * (k[0] + 2.0 * k[1] + 2.0 * k[2] + k[3]) / 6.0
    zmem = zmem + tau / HBAR * (kz[0] + 2.0 * kz[1] + 2.0 * kz[2] + kz[3]) / 6.0
    return phi, zmem


def normalize(phi, nstate):
    """phi / ||psi_0||.  trajectory/hops_trajectory.py:616-634"""
    return phi / np.sqrt(np.sum(np.abs(phi[:nstate]) ** 2))


def noise_lookup(noise, t_list, tau_noise, dtype=np.complex64):
    """Exact time lookup + complex64 result.  noise/hops_noise.py:437-451,796-825
    (dtype complex128: INTERPOLATE noise, the cubic spline of hops_noise.py:
    242-265,379-384 at its own sample times)"""
    out = np.zeros((noise.shape[0], len(t_list)), dtype=dtype)
    for i, t in enumerate(t_list):
        it = int(round(t / tau_noise))
        if abs(it * tau_noise - t) >= PRECISION:
            raise ValueError("off-axis noise sample")
        out[:, i] = noise[:, it]
    return out


def effective_noise(noise, t, tau, tau_noise, real=False):
    """EFFECTIVE_NOISE_INTEGRATION samples [n_L, 3]: means of the complex64
    samples in [t, t + tau/2), [t + tau/2, t + tau), [t + tau, t + 3 tau/2)
    taken with np.mean as integrator/integrator_rk.py:115-128 does (real: the
    float32 real parts, FLAG_REAL noise)."""
    r = round(tau / tau_noise)
    raw = noise_lookup(noise, [t + (i / r) * tau for i in range(round(r * 1.5))], tau_noise)
    if real:
        raw = np.real(raw)
    return np.array([np.mean(raw[:, :round(r / 2)], axis=1),
                     np.mean(raw[:, round(r / 2):r], axis=1),
                     np.mean(raw[:, r:], axis=1)]).T


def propagate(basis, psi0, noise1, tau_noise, t_max, dt, noise2=None,
              eom="NORMALIZED NONLINEAR", effective=False, noise_dtype=np.complex64):
    """Run the non-adaptive trajectory loop; returns (t_axis, psi_traj, phi, zmem).

    trajectory/hops_trajectory.py:253-336 (phi_0 = [psi_0, 0 ...], z_mem = 0)
    and :401-538 (runge_kutta_variables -> runge_kutta_step -> normalize);
    effective: EFFECTIVE_NOISE_INTEGRATION window means instead of the samples.
    """
    S, N = basis.nstate, basis.nhier
    phi = np.zeros(N * S, dtype=np.complex128)
    phi[:S] = psi0
    zmem = np.zeros(basis.nmode, dtype=np.complex128)
    n_steps = int(np.ceil(t_max / dt))
    if noise2 is None:
        noise2 = np.zeros_like(noise1)
    psi_traj = [phi[:S].copy()]
    t_axis = [0.0]
    t = 0.0
    for n in range(n_steps):
        if effective:
            zr = effective_noise(noise1, t, dt, tau_noise)
            zr2 = effective_noise(noise2, t, dt, tau_noise)
        else:
            tl = [t, t + dt * 0.5, t + dt]
            zr = noise_lookup(noise1, tl, tau_noise, noise_dtype)
            zr2 = noise_lookup(noise2, tl, tau_noise, noise_dtype)
        phi, zmem = rk4_step(basis, phi, zmem, zr, zr2, dt, eom)
        if eom == "NORMALIZED NONLINEAR":
            phi = normalize(phi, S)
        t = (n + 1) * dt
        psi_traj.append(phi[:S].copy())
        t_axis.append(t)
    return np.array(t_axis), np.array(psi_traj), phi, zmem


# ---------------------------------------------------------------------------
# Adaptive sub-basis and the flux-error terms of the basis update
# ---------------------------------------------------------------------------
class OracleSubBasis(OracleBasis):
    """One adaptive basis: a subset of states, of modes and of aux.

    basis/hops_modes.py:123-171 reduces every unique L of the basis modes to the
    state basis; the relative L list is the sorted absolute unique-L indices of
    the basis modes (list_absindex_L2), so noise rows are noise[l_abs].
    states / modes: sorted absolute indices; aux: count rows over ALL modes.
    """

    def __init__(self, sys_param, states, modes, aux, full=None):
        full = expand_system(sys_param) if full is None else full
        states = np.asarray(states, dtype=np.int64)
        modes = np.asarray(modes, dtype=np.int64)
        self.l_abs = sorted(set(int(full["L_BY_MODE"][m]) for m in modes))
        rel = {j: i for i, j in enumerate(self.l_abs)}
        ix = np.ix_(states, states)
        self.sys = {"H": full["H"][ix], "G": full["G"][modes], "W": full["W"][modes],
                    "L": [full["L"][j][ix] for j in self.l_abs],
                    "L_BY_MODE": np.array([rel[int(full["L_BY_MODE"][m])] for m in modes],
                                          dtype=np.int64),
                    "NSTATE": len(states), "NMODE": len(modes),
                    "LT": np.asarray(full.get("LT", np.zeros(len(full["L"]))))[self.l_abs]}
        self.states, self.modes = states, modes
        self.nstate, self.nmode = len(states), len(modes)
        aux = np.asarray(aux, dtype=np.int64)
        self.aux = aux[:, modes].reshape(len(aux), len(modes))
        self.nhier = len(self.aux)
        self.index = {tuple(v): i for i, v in enumerate(self.aux)}
        self._build_super_operators()


def flux_errors(basis, phi, zmem, z1, z2, dt, mask=None, eom="NORMALIZED NONLINEAR"):
    """Error arrays of the adaptive update for diagonal L-operators.

    e_deriv [N, S]: |dphi/dt / hbar + phi / dt|^2 of the phi restricted to the
        aux with mask != 0 (error_deriv, basis/basis_functions_adaptive.py:10-74);
        rows with mask == 0 are 0.
    e_up [M, N]: |w_m|^2 (1 + k_m(a))^2 sum_s |L_m[s,s]|^2 |phi[a,s]|^2 / hbar^2
        (error_flux_up_hier_stable, :165-266).
    e_down [M, N]: |g_m / w_m|^2 sum_s |L_m[s,s] - <L_m>|^2 |phi[a,s]|^2 / hbar^2
        (error_flux_down_hier_stable, :517-624; <L> of the unmasked psi_0).
    """
    s = basis.sys
    S, N, M = basis.nstate, basis.nhier, basis.nmode
    phi = np.asarray(phi, dtype=np.complex128)
    ph = phi.copy().reshape(N, S)
    if mask is not None:
        ph[np.asarray(mask) == 0] = 0.0
    dphi, _ = dsystem_dt(basis, ph.ravel(), zmem, z1, z2, eom)
    e_deriv = np.abs(dphi / HBAR + ph.ravel() / dt).reshape(N, S) ** 2
    if mask is not None:
        e_deriv[np.asarray(mask) == 0] = 0.0
    pf = phi.reshape(N, S)
    psi0 = pf[0]
    n2 = np.vdot(psi0, psi0)
    avg = np.array([np.vdot(psi0, l @ psi0) / n2 for l in s["L"]])
    m2 = np.array([np.diag(s["L"][s["L_BY_MODE"][m]]) for m in range(M)]).reshape(M, S)
    p2 = np.abs(pf) ** 2                                   # [N, S]
    k = basis.aux.T.astype(np.float64)                     # [M, N]
    w2 = np.abs(s["W"]) ** 2
    e_up = (w2[:, None] * (1.0 + k) ** 2) * ((np.abs(m2) ** 2) @ p2.T) / HBAR ** 2
    d2 = np.abs(m2 - avg[s["L_BY_MODE"]][:, None]) ** 2
    e_down = (np.abs(s["G"] / s["W"]) ** 2)[:, None] * (d2 @ p2.T) / HBAR ** 2
    return e_deriv, e_up, e_down


# ---------------------------------------------------------------------------
# FFT-filtered noise
# ---------------------------------------------------------------------------
def noise_t_axis(tlen, tau):
    """noise/hops_noise.py:154-156"""
    n = int(np.ceil(tlen / tau)) + 1
    return np.arange(n) * tau


def raw_index(ntaus):
    """Slot scrambling of the raw draws (re/g and im/phi).  hops_noise.py:592-628.

    Slot j of the complex white noise takes random number re_idx[j] (real part or
    Box-Muller radius) and im_idx[j] (imaginary part or phase).
    """
    n1 = ntaus - 1
    re = [0] + list(range(2, 4 * (ntaus - 2), 4)) + [4 * n1 - 2] \
        + list(range(4 * (ntaus - 2), 3, -4))
    im = [1] + list(range(3, 4 * (ntaus - 1) - 1, 4)) + [4 * n1 - 1] \
        + list(range(4 * (n1 - 1) + 1, 4, -4))
    return np.array(re, dtype=np.int64), np.array(im, dtype=np.int64)


def raw_draws(seed, lops, ntaus, model="SUM_GAUSSIAN"):
    """Uncorrelated complex64 draws per L.  hops_noise.py:453-590.

    Uses numpy's PCG64(seed).jumped(lop) stream, as the reference does.
    """
    re, im = raw_index(ntaus)
    out = np.zeros((len(lops), 2 * (ntaus - 1)), dtype=np.complex64)
    for i, lop in enumerate(lops):
        rs = np.random.default_rng(np.random.PCG64(seed=seed).jumped(int(lop)))
        if model == "SUM_GAUSSIAN":
            x = rs.normal(loc=0, size=4 * (ntaus - 1))
            out[i] = np.complex64(x[re] + 1j * x[im])
        elif model == "BOX_MULLER":
            x = rs.random(size=4 * (ntaus - 1))
            out[i] = np.complex64(np.sqrt(-2.0 * np.log(x[re]))
                                  * np.exp(2.0j * np.pi * x[im]))
        else:
            raise ValueError(model)
    return out


def alpha_by_lop(t_axis, gw_noise, lop_by_nmode, n_lop):
    """Sum of bcf_exp over the noise modes of each L.  hops_noise.py:167-192"""
    alpha = np.zeros((n_lop, len(t_axis)), dtype=np.complex128)
    for m, (g, w) in enumerate(gw_noise):
        alpha[lop_by_nmode[m]] += bcf_exp(t_axis, g, w)
    return alpha


def correlated_noise(c_t, z_t, fp64=True):
    """Percival circulant-embedding filter.  hops_noise.py:630-716.

    c_t: [n_L, n_t] correlation function (complex64 in the reference, :236);
    z_t: [n_L, 2(n_t-1)] uncorrelated complex64 draws.
    fp64=True evaluates every step in float64 (the arithmetic the GPU filter
    uses).  fp64=False mirrors numpy's dtype propagation in the reference
    (float32 angle/abs of c_t and a float32 FFT of z_t) so that the oracle can be
    pinned against the reference's own golden arrays.
    """
    c_t = np.asarray(c_t)
    z_t = np.asarray(z_t)
    n_t = c_t.shape[1]
    if fp64:
        c = c_t.astype(np.complex128)
        ang = np.angle(c)
        mag = np.abs(c)
    else:
        ang = np.array(np.angle(c_t), dtype=np.float64)
        mag = np.abs(c_t)
    nu = ang[:, -1] / ((n_t - 1.0) * 2.0 * np.pi)
    rot = np.exp(-1.0j * 2.0 * np.pi * np.outer(nu, np.arange(n_t)))
    ct = mag * np.exp(1.0j * ang) * rot
    emb = np.concatenate([ct, np.conj(ct[:, 1:-1][:, ::-1])], axis=1)
    s_w = np.real(np.fft.fft(emb, axis=1))
    s_w[s_w < 0] = 0.0
    zin = z_t.astype(np.complex128) if fp64 else z_t
    z_w = np.array([np.fft.fft(zin[i]) for i in range(zin.shape[0])],
                   dtype=np.complex128)
    y = np.fft.ifft(np.abs(z_w) * np.exp(1.0j * np.angle(z_w)) * np.sqrt(s_w / 2.0),
                    axis=1)[:, :n_t]
    return np.abs(y) * np.exp(1.0j * np.angle(y)) * np.conj(rot)


def fft_filter_noise(t_axis, gw_noise, lop_by_nmode, n_lop, z_t, fp64=True):
    """alpha -> complex64 -> filter -> complex64 storage.  hops_noise.py:232-247"""
    alpha = np.complex64(alpha_by_lop(t_axis, gw_noise, lop_by_nmode, n_lop))
    return np.complex64(correlated_noise(alpha, z_t, fp64=fp64))
