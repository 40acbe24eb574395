"""save_checkpoint / load_checkpoint (trajectory/hops_trajectory.py:853-1034):
a run interrupted by a checkpoint and resumed from the file must continue as
if it had not been interrupted."""

import numpy as np
import pytest

import mesohops_b200.adaptive as ad
from conftest import golden_system, load_golden
from mesohops_b200 import HopsTrajectory
from test_adaptive import OracleServer, check_against, load, make_traj, system_param


def _plain_traj(f, tmp_path, device, precision="complex128"):
    path = str(tmp_path / "noise1.npy")
    np.save(path, f["noise1"])
    return HopsTrajectory(golden_system(f),
                          noise_param={"SEED": path, "MODEL": "PRE_CALCULATED",
                                       "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                          hierarchy_param={"MAXHIER": int(f["depth"])},
                          storage_param={"phi_traj": True, "z_mem": True},
                          device_param={"DEVICE": device, "PRECISION": precision})


def test_checkpoint_round_trip_keys_and_state(tmp_path):
    """File layout of the reference and an exact state round trip (no stepping)."""
    f = load_golden("ring6")
    h = _plain_traj(f, tmp_path, "cpu")
    psi0 = np.array(f["psi0"], dtype=complex)
    h.initialize(psi0)
    ck = str(tmp_path / "ck.npz")
    h.save_checkpoint(ck)
    data = np.load(ck, allow_pickle=True)
    assert {"phi", "z_mem", "t", "state_list", "aux_list", "early_counter", "storage_data",
            "storage_meta", "params"} <= set(data.files)
    params = data["params"].item()
    assert {"system_param", "hierarchy_param", "eom_param", "noise1_param", "noise2_param",
            "integration_param", "storage_param"} <= set(params)
    assert len(data["aux_list"]) == h.n_hier
    h2 = HopsTrajectory.load_checkpoint(ck)
    assert np.array_equal(h2.phi, h.phi)
    assert np.array_equal(h2.z_mem, h.z_mem)
    assert h2.t == h.t and h2.n_hier == h.n_hier
    assert h2.noise1.param["MODEL"] == "PRE_CALCULATED"
    np.save(str(tmp_path / "other.npy"), f["noise1"])
    h3 = HopsTrajectory.load_checkpoint(ck, add_seed1=str(tmp_path / "other.npy"))
    assert h3.noise1.param["SEED"].endswith("other.npy")


def test_checkpoint_drop_seed(tmp_path):
    f = load_golden("ring6")
    h = _plain_traj(f, tmp_path, "cpu")
    h.initialize(np.array(f["psi0"], dtype=complex))
    ck = str(tmp_path / "ck.npz")
    h.save_checkpoint(ck, drop_seed=True)
    params = np.load(ck, allow_pickle=True)["params"].item()
    assert "SEED" not in params["noise1_param"]


@pytest.mark.parametrize("name", ["adaptive_chain8", "adaptive_dod_full"])
def test_adaptive_checkpoint_resume_matches_reference(name, tmp_path, monkeypatch):
    """Adaptive run stopped half-way, saved, loaded and finished: the basis per
    step and psi(t) still equal the reference's uninterrupted run (device
    requests served by the oracle, so this runs on the CPU)."""
    f = load(name)
    server = OracleServer(system_param(f), f["noise1"], float(f["tau_noise"]))
    monkeypatch.setattr(ad, "drive", server.drive)
    h = make_traj(f, tmp_path, "cpu")
    h.initialize(f["psi0"])
    dt = float(f["dt"])
    n = len(f["t_axis"]) - 1
    half = n // 2 if name != "adaptive_dod_full" else 3    # inside the early integrator
    h.propagate(half * dt, dt)
    ck = str(tmp_path / "ck.npz")
    h.save_checkpoint(ck)
    h2 = HopsTrajectory.load_checkpoint(ck)
    h2.propagate((n - half) * dt, dt)
    check_against(h2, f)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["complex128", "mixed"])
@pytest.mark.parametrize("name", ["ring6", "c1_dimer"])
def test_checkpoint_resume_equals_uninterrupted(cuda_device, tmp_path, name, precision):
    f = load_golden(name)
    dt = float(f["dt"])
    psi0 = np.array(f["psi0"], dtype=complex)
    ref = _plain_traj(f, tmp_path, "cuda:0", precision)
    ref.initialize(psi0)
    ref.propagate(20 * dt, dt)
    h = _plain_traj(f, tmp_path, "cuda:0", precision)
    h.initialize(psi0)
    h.propagate(8 * dt, dt)
    ck = str(tmp_path / "ck.npz")
    h.save_checkpoint(ck)
    h2 = HopsTrajectory.load_checkpoint(ck)
    h2.propagate(12 * dt, dt)
    a = np.array(ref.storage["psi_traj"])
    b = np.array(h2.storage["psi_traj"])
    assert a.shape == b.shape
    assert np.max(np.abs(a - b)) <= 1e-12
    assert np.max(np.abs(ref.phi - h2.phi)) <= 1e-12
    assert np.max(np.abs(ref.z_mem - h2.z_mem)) <= 1e-12
    assert np.allclose(ref.storage["t_axis"], h2.storage["t_axis"])


@pytest.mark.gpu
def test_adaptive_checkpoint_resume_on_gpu(cuda_device, tmp_path):
    f = load("adaptive_chain12")
    h = make_traj(f, tmp_path, "cuda:0")
    h.initialize(f["psi0"])
    dt = float(f["dt"])
    n = len(f["t_axis"]) - 1
    h.propagate(11 * dt, dt)
    ck = str(tmp_path / "ck.npz")
    h.save_checkpoint(ck)
    h2 = HopsTrajectory.load_checkpoint(ck)
    h2.propagate((n - 11) * dt, dt)
    check_against(h2, f)
