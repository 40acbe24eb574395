"""Synthetic systems of the benchmark configurations (all inputs seeded).

Drude-Lorentz modes use the high-temperature exponential form
g = 2 lambda kB T - i lambda gamma, w = gamma; every L_m is the site projector
|m><m|; noise is FFT-filtered complex Gaussian noise from the given seeds.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps

from .bath import bcf_convert_dl_to_exp, bcf_exp


def site_system(H, modes_per_site):
    """System dictionary with one set of DL modes (lambda, gamma, T) per site."""
    n = H.shape[0]
    gw, lops = [], []
    for i in range(n):
        L = sps.coo_matrix(([1.0], ([i], [i])), shape=(n, n))
        for (lam, gam, temp) in modes_per_site:
            g, w = bcf_convert_dl_to_exp(lam, gam, temp)[:2]
            gw.append([g, w])
            lops.append(L)
    Hd = H.toarray() if sps.issparse(H) else np.asarray(H)
    return {"HAMILTONIAN": np.array(Hd, dtype=np.complex128), "GW_SYSBATH": gw,
            "L_HIER": lops, "L_NOISE1": lops, "ALPHA_NOISE1": bcf_exp, "PARAM_NOISE1": gw}


def dimer():
    """2-site dimer, H=[[0,50],[50,0]], (50, 50, 295 K) per site."""
    H = np.array([[0.0, 50.0], [50.0, 0.0]])
    return site_system(H, [(50.0, 50.0, 295.0)])


def chain10_two_modes():
    """10-site chain, J=100, eps ~ N(0, 50) (seed 1), (35,50,300 K)+(10,500,300 K)."""
    n = 10
    rng = np.random.default_rng(1)
    H = np.diag(rng.normal(0, 50, n))
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = 100.0
    return site_system(H, [(35.0, 50.0, 300.0), (10.0, 500.0, 300.0)])


def ring20():
    """20-site ring, J=80, eps ~ U(-100, 100) (seed 2), (60, 60, 295 K) per site."""
    n = 20
    rng = np.random.default_rng(2)
    H = np.diag(rng.uniform(-100, 100, n))
    for i in range(n):
        H[i, (i + 1) % n] = H[(i + 1) % n, i] = 80.0
    return site_system(H, [(60.0, 60.0, 295.0)])


def chain(n, J, eps, lam, gam, temp=295.0):
    """Linear chain with given site energies and one DL mode per site."""
    H = np.diag(np.asarray(eps, dtype=float))
    for i in range(n - 1):
        H[i, i + 1] = H[i + 1, i] = J
    return site_system(H, [(lam, gam, temp)])


def chain_sites(n):
    """n-site chain, J = 50 cm^-1, eps ~ N(0, 100) from seed 5, one DL mode
    (50, 50, 295 K) per site."""
    return chain(n, 50.0, np.random.default_rng(5).normal(0, 100, n), 50.0, 50.0)


WORKLOADS = {
    "ring20": dict(system=ring20, depth=4, n_traj=128, dt=4.0, n_steps=250,
                   desc="20-site ring (J=80 cm^-1, eps~U(-100,100) seed 2), one Drude-Lorentz "
                        "mode per site (lambda=60, gamma=60 cm^-1, 295 K), depth 4 "
                        "(10626 aux x 20 states), 128 trajectories (noise seeds 0..127), "
                        "dt=4 fs"),
    "chain10": dict(system=chain10_two_modes, depth=6, n_traj=256, dt=2.0, n_steps=250,
                    desc="10-site chain (J=100 cm^-1, eps~N(0,50) seed 1), two DL modes per "
                         "site (35,50)+(10,500) cm^-1 at 300 K, depth 6 (230230 aux x 10 "
                         "states), 256 trajectories (seeds 0..255), dt=2 fs"),
    "chain120": dict(system=lambda: chain_sites(120), depth=3, n_traj=1, dt=4.0, n_steps=250,
                     desc="120-site chain (J=50 cm^-1, eps~N(0,100) seed 5), DL (50,50,295 K) "
                          "per site, depth 3 (302621 aux x 120 states), one trajectory, "
                          "dt=4 fs: a single large trajectory like the served stream's "
                          "streaming requests"),
    "chain128": dict(system=lambda: chain_sites(128), depth=3, n_traj=1, dt=4.0, n_steps=250,
                     desc="128-site chain (J=50 cm^-1, eps~N(0,100) seed 5), DL (50,50,295 K) "
                          "per site, depth 3 (366145 aux x 128 states), one trajectory, dt=4 fs"),
    "chain200": dict(system=lambda: chain_sites(200), depth=3, n_traj=1, dt=4.0, n_steps=250,
                     desc="200-site chain (J=50 cm^-1, eps~N(0,100) seed 5), DL (50,50,295 K) "
                          "per site, depth 3 (1373701 aux x 200 states), one trajectory, dt=4 fs: "
                          "the largest systems of the served stream"),
    "chain200_uncoupled": dict(
        system=lambda: chain(200, 0.0, np.random.default_rng(5).normal(0, 100, 200), 50.0, 50.0),
        depth=3, n_traj=1, dt=4.0, n_steps=250,
        desc="chain200 with J = 0 (diagonal H): the same hierarchy without the -iH couplings"),
    "dimer": dict(system=dimer, depth=4, n_traj=1, dt=4.0, n_steps=250,
                  desc="2-site dimer H=[[0,50],[50,0]], DL (50,50,295 K) per site, depth 4 "
                       "(15 aux x 2 states), one trajectory, dt=4 fs, 1000 fs"),
}


# ----------------------------------------------------------- served stream
def served_stream_specs(n_requests=4096, seed=4, dt=4.0, mean_gap_s=2e-3):
    """Specs of the served request stream: Poisson arrivals (exponential gaps,
    mean 2 ms); each request a linear chain of N_site ~ U{2..200} sites
    (J = 50 cm^-1, eps ~ N(0, 100)), depth ~ U{3..8}, adaptive (delta = 1e-3)
    by a fair coin, one Drude-Lorentz mode per site with lambda ~ U(20, 80),
    gamma ~ U(30, 150) cm^-1 at 295 K, dt = 4 fs, t_max ~ U(200, 2000) fs,
    psi_0 on a uniformly drawn site; all from one generator seeded with 4.
    Returns a list of dicts (cheap; systems are built by ``served_request``)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(mean_gap_s)
        n_site = int(rng.integers(2, 201))
        depth = int(rng.integers(3, 9))
        adaptive = bool(rng.random() < 0.5)
        lam = float(rng.uniform(20, 80))
        gam = float(rng.uniform(30, 150))
        t_max = float(rng.uniform(200, 2000))
        eps = rng.normal(0, 100, n_site)
        start = int(rng.integers(0, n_site))
        out.append(dict(rid=i, arrival=t, n_site=n_site, depth=depth, adaptive=adaptive,
                        lam=lam, gam=gam, t_max=t_max, eps=eps, start=start, dt=dt,
                        noise_seed=i))
    return out


def served_request(spec, delta=1e-3):
    """TrajectoryRequest of one stream spec (FFT-filtered noise, seed = request id)."""
    from .serving import TrajectoryRequest
    n = spec["n_site"]
    sysp = chain(n, 50.0, spec["eps"], spec["lam"], spec["gam"])
    dt = spec["dt"]
    n_steps = int(np.ceil(spec["t_max"] / dt - 1e-12))
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[spec["start"]] = 1.0
    noise = {"SEED": spec["noise_seed"], "MODEL": "FFT_FILTER", "TLEN": (n_steps + 1) * dt,
             "TAU": dt / 2}
    return TrajectoryRequest(spec["rid"], sysp, psi0, n_steps * dt, dt,
                             hierarchy_param={"MAXHIER": spec["depth"]},
                             eom_param={"EQUATION_OF_MOTION": "NORMALIZED NONLINEAR"},
                             noise_param=noise,
                             adaptive=(delta, delta) if spec["adaptive"] else None,
                             arrival=spec["arrival"])


def adaptive_chain500(n_traj=512, seed=3):
    """500-site chain (J = 50 cm^-1, eps ~ N(0, 100) from seed 3), one DL mode
    per site (50, 50, 295 K), depth 10, delta_a = delta_s = 1e-3, dt = 4 fs;
    psi_0 on a site drawn from the same generator.  Returns (system_param,
    psi_0, per-trajectory noise seeds)."""
    n = 500
    rng = np.random.default_rng(seed)
    eps = rng.normal(0, 100, n)
    start = int(rng.integers(0, n))
    sysp = chain(n, 50.0, eps, 50.0, 50.0)
    psi0 = np.zeros(n, dtype=np.complex128)
    psi0[start] = 1.0
    return sysp, psi0, list(range(n_traj))
