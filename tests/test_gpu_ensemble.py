"""Batched ensembles (one structure, B trajectories, layout [aux][state][traj])
against the CPU oracle run trajectory by trajectory.  B = 40, 33 and 129 exercise
the wide kernel with a partial last chunk, B = 32 the smallest wide batch, B = 31
and 7 the narrow kernel, B = 1 the single-trajectory case."""
import numpy as np
import pytest

from conftest import golden_system, load_golden
from oracle import hops_oracle as O

pytestmark = pytest.mark.gpu


def ensemble_noise(f, B, seed):
    n_l, n_t = f["noise1"].shape
    rng = np.random.default_rng(seed)
    return ((rng.normal(size=(B, n_l, n_t)) + 1j * rng.normal(size=(B, n_l, n_t))) * 30
            ).astype(np.complex64)


def run_ensemble(f, B, precision, noise, n_steps):
    import torch
    from mesohops_b200 import HopsEnsemble
    ens = HopsEnsemble(golden_system(f), B,
                       noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                    "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision)
    ens.initialize(f["psi0"])
    dt = float(f["dt"])
    psi = torch.empty((n_steps, B, ens.n_state), dtype=torch.complex128, device="cuda")
    ens.propagate(n_steps * dt, dt, psi_out=psi)
    ens.check()
    return psi.cpu().numpy(), ens


def oracle_psi(f, noise_b, n_steps):
    sysp = golden_system(f)
    b = O.OracleBasis({k: sysp[k] for k in ("HAMILTONIAN", "GW_SYSBATH", "L_HIER")},
                      int(f["depth"]))
    dt = float(f["dt"])
    _, psi, phi, _ = O.propagate(b, f["psi0"], noise_b, float(f["tau_noise"]), n_steps * dt, dt)
    return psi[1:], phi


@pytest.mark.parametrize("name,B", [("ring6", 40), ("ring6", 7), ("general_lop", 33),
                                    ("chain4_2mode", 64), ("ring6", 1), ("ring6", 31),
                                    ("ring6", 32), ("ring6", 129)])
def test_ensemble_c128_matches_oracle(cuda_device, name, B):
    f = load_golden(name)
    n_steps = 12
    noise = ensemble_noise(f, B, 5)
    psi, ens = run_ensemble(f, B, "complex128", noise, n_steps)
    phi, _ = ens.state()
    for b in sorted({0, min(1, B - 1), B // 2, B - 1}):
        ref, phi_ref = oracle_psi(f, noise[b], n_steps)
        assert np.max(np.abs(psi[:, b] - ref)) <= 1e-10 * np.max(np.abs(ref))
        assert np.max(np.abs(phi[b] - phi_ref)) <= 1e-10 * np.max(np.abs(phi_ref))


@pytest.mark.parametrize("precision,bound", [("mixed", 1e-5), ("complex64", 3e-5)])
def test_ensemble_reduced_precision(cuda_device, precision, bound):
    f = load_golden("ring6")
    B, n_steps = 40, int(round(float(f["t_max"]) / float(f["dt"])))
    noise = ensemble_noise(f, B, 6)
    p_lo, _ = run_ensemble(f, B, precision, noise, n_steps)
    p_hi, _ = run_ensemble(f, B, "complex128", noise, n_steps)
    assert np.max(np.abs(np.abs(p_lo) ** 2 - np.abs(p_hi) ** 2)) <= bound


def test_ensemble_derivative_matches_oracle(cuda_device):
    """Stage-4 (single derivative) path of the wide kernel for 40 trajectories."""
    from mesohops_b200 import HopsEnsemble
    f = load_golden("general_lop")
    B = 40
    ens = HopsEnsemble(golden_system(f), B, noise_param={"MODEL": "ZERO", "TLEN": 10.0, "TAU": 0.5},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision="complex128")
    rng = np.random.default_rng(9)
    n = ens.n_hier * ens.n_state
    phi = rng.normal(size=(B, n)) + 1j * rng.normal(size=(B, n))
    zm = rng.normal(size=(B, ens.system.n_mode)) + 1j * rng.normal(size=(B, ens.system.n_mode))
    z1 = (rng.normal(size=(B, 3)) + 1j * rng.normal(size=(B, 3))).astype(np.complex64) * 20
    z2 = (rng.normal(size=(B, 3)) + 1j * rng.normal(size=(B, 3))).astype(np.complex64) * 5
    ens.batch.set_state(phi, zm)
    dphi, dz = ens.batch.dsystem_dt(z1, z2)
    sysp = golden_system(f)
    ob = O.OracleBasis({k: sysp[k] for k in ("HAMILTONIAN", "GW_SYSBATH", "L_HIER")}, int(f["depth"]))
    for b in (0, 17, 39):
        ref, rz = O.dsystem_dt(ob, phi[b], zm[b], z1[b], z2[b])
        assert np.max(np.abs(dphi[b] - ref)) <= 1e-12 * np.max(np.abs(ref))
        assert np.max(np.abs(dz[b] - rz)) <= 1e-12 * np.max(np.abs(rz))



def run_forced(f, B, precision, noise, n_steps, tuning, fusion=1):
    """Ensemble run with a fixed stage-kernel shape (nb, chunk_major) and step
    fusion (1: separate launches, 2: the persistent step kernel)."""
    import torch
    from mesohops_b200 import HopsEnsemble
    ens = HopsEnsemble(golden_system(f), B,
                       noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                    "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                       hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision,
                       autotune=False)
    ens.initialize(f["psi0"])
    ens.batch.tuning = tuning
    ens.batch.fusion = fusion
    dt = float(f["dt"])
    psi = torch.empty((n_steps, B, ens.n_state), dtype=torch.complex128, device="cuda")
    ens.propagate(n_steps * dt, dt, psi_out=psi)
    ens.check()
    return psi.cpu().numpy()



@pytest.mark.parametrize("name", ["ring6", "chain4_2mode"])
@pytest.mark.parametrize("B", [40, 64, 96])
@pytest.mark.parametrize("tuning", [(1, 0), (1, 1), (1, 2), (4, 0), (4, 1), (4, 2), (8, 1),
                                    (8, 2), (1, 3), (4, 3), (8, 3)])
def test_stage_kernel_shapes_agree(cuda_device, name, B, tuning):
    """Every stage-kernel shape the autotuner may pick gives the same numbers."""
    f = load_golden(name)
    n_steps = 8
    noise = ensemble_noise(f, B, 11)
    ref = run_forced(f, B, "complex128", noise, n_steps, (2, 0))
    got = run_forced(f, B, "complex128", noise, n_steps, tuning)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", ["ring6", "chain4_2mode"])
@pytest.mark.parametrize("B", [40, 128, 700])
@pytest.mark.parametrize("precision", ["complex128", "mixed", "complex64"])
@pytest.mark.parametrize("order", [0, 3])
def test_persistent_step_kernel_matches_separate_launches(cuda_device, name, B, precision, order):
    """The persistent step kernel (one cooperative launch per call, grid
    barriers between the scalar and stage phases) gives the numbers of the
    separate scalar and stage launches bit for bit -- including batches with
    more trajectories than CTAs (700 on the 6-site ring: 126 CTAs, each
    computing the scalars of several trajectories) and several chunks."""
    f = load_golden(name)
    n_steps = 6
    noise = ensemble_noise(f, B, 5)
    ref = run_forced(f, B, precision, noise, n_steps, (4, order), fusion=1)
    got = run_forced(f, B, precision, noise, n_steps, (4, order), fusion=2)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("precision", ["complex128", "mixed"])
def test_deferred_renormalisation_one_call_per_step(cuda_device, precision):
    """HopsEnsemble leaves each call's last renormalisation pending (hops_batch
    defer_scale) and the next call applies it on the fly, as the steps within
    a call do: twelve one-step calls give the psi(t), state and z_mem of one
    twelve-step call bit for bit, and the path that rescales the state on
    return agrees to the rounding of its precision."""
    import torch
    from mesohops_b200 import HopsEnsemble
    f = load_golden("ring6")
    B, n = 40, 12
    noise = ensemble_noise(f, B, 9)
    psi_one, ens_one = run_ensemble(f, B, precision, noise, n)
    phi_one, z_one = ens_one.state()
    dt = float(f["dt"])
    out = {}
    for defer in (True, False):
        ens = HopsEnsemble(golden_system(f), B,
                           noise_param={"SEED": noise, "MODEL": "PRE_CALCULATED",
                                        "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                           hierarchy_param={"MAXHIER": int(f["depth"])}, precision=precision)
        ens.batch.defer_scale = defer
        ens.initialize(f["psi0"])
        psi = torch.empty((n, B, ens.n_state), dtype=torch.complex128, device="cuda")
        for k in range(n):
            ens.propagate(dt, dt, psi_out=psi[k:k + 1])
        assert ens.batch._pending == defer
        phi, z = ens.state()
        assert not ens.batch._pending
        ens.check()
        out[defer] = (psi.cpu().numpy(), phi, z)
    psi_d, phi_d, z_d = out[True]
    assert np.array_equal(psi_d, psi_one)
    assert np.array_equal(phi_d, phi_one) and np.array_equal(z_d, z_one)
    # rescaling on return rounds differently: at complex128, or (mixed) where
    # the complex64 copy of the state is taken from the rescaled state
    tol = 1e-12 if precision == "complex128" else 1e-6
    psi_e, phi_e, _ = out[False]
    assert np.max(np.abs(psi_e - psi_one)) <= tol * np.max(np.abs(psi_one))
    assert np.max(np.abs(phi_e - phi_one)) <= tol * np.max(np.abs(phi_one))


def test_c_abi_rejects_bad_propagation_arguments(cuda_device):
    """hops_rk4_propagate refuses a noise window past the noise axis and negative
    step / index arguments with HOPS_EINVAL and an error text, launching nothing:
    the state is unchanged afterwards."""
    import ctypes as C
    from mesohops_b200 import _lib
    from mesohops_b200.engine import _stream
    f = load_golden("ring6")
    B = 40
    noise = ensemble_noise(f, B, 8)
    _, ens = run_ensemble(f, B, "complex128", noise, 1)
    before, _ = ens.state()
    L = _lib.lib()
    b = ens.batch
    n_t = noise.shape[2]
    for it0, di, n in [(0, 1, n_t), (n_t, 1, 1), (-1, 1, 1), (0, -1, 1), (0, 1, -1)]:
        rc = L.hops_rk4_propagate(C.byref(b.st.cstruct), C.byref(b.cb), it0, di, n, 0.01,
                                  None, _stream(cuda_device))
        assert rc == _lib.HOPS_EINVAL, (it0, di, n)
        assert L.hops_last_error()
    after, _ = ens.state()
    assert np.array_equal(before, after)
