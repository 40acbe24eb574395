"""Triangular hierarchies built on the GPU (hops_tri_pass1/2) against the host
construction: every table identical (indices exact, coefficients to rounding),
and propagation through them equal to the oracle."""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_system, load_golden
from mesohops_b200.workloads import chain, ring20, site_system

pytestmark = pytest.mark.gpu

INT_FIELDS = ["up_ptr", "up_aux", "up_mode", "dn_ptr", "dn_aux", "dn_mode", "up_site", "dn_site",
              "first_aux", "first_mode"]
CPLX_FIELDS = ["k_decay", "dn_coef", "dn_coef_site"]


def _np(x):
    import torch
    return x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def _systems():
    rng = np.random.default_rng(7)
    H = np.diag(rng.normal(0, 50, 5)) + np.diag([30.0] * 4, 1) + np.diag([30.0] * 4, -1)
    two = site_system(H, [(35, 50, 300), (10, 500, 300)])
    return [("ring20_d2", ring20(), 2),
            ("chain9_d4", chain(9, 50.0, rng.normal(0, 100, 9), 50, 50), 4),
            ("two_modes_d5", two, 5),
            ("chain3_d1", chain(3, 40.0, [0, 10, 20], 40, 40), 1)]


@pytest.mark.parametrize("name,sysp,depth", _systems())
def test_gpu_tables_equal_host_tables(cuda_device, name, sysp, depth):
    from mesohops_b200.device import build_tables, build_tables_triangular
    from mesohops_b200.hierarchy import triangular_basis
    from mesohops_b200.system import HopsSystem
    system = HopsSystem(sysp)
    host = build_tables(system, triangular_basis(system.n_mode, depth))
    dev = build_tables_triangular(system, depth, "cuda:0")
    assert dev["n_hier"] == host["n_hier"]
    assert dev["max_up"] == host["max_up"] and dev["max_dn"] == host["max_dn"]
    for k in INT_FIELDS:
        assert np.array_equal(_np(dev[k]).astype(np.int64), _np(host[k]).astype(np.int64)), k
    for k in CPLX_FIELDS:
        a, b = _np(dev[k]), _np(host[k])
        assert a.shape == b.shape, k
        assert np.allclose(a, b, rtol=1e-14, atol=1e-12), k


def test_general_lop_structure_matches(cuda_device):
    """Off-diagonal L-operators: the hierarchy part built on the GPU equals the
    host build as well."""
    from mesohops_b200.device import build_tables, build_tables_triangular
    from mesohops_b200.hierarchy import triangular_basis
    from mesohops_b200.system import HopsSystem
    f = load_golden("general_lop")
    system = HopsSystem(golden_system(f))
    depth = int(f["depth"])
    host = build_tables(system, triangular_basis(system.n_mode, depth))
    dev = build_tables_triangular(system, depth, "cuda:0")
    for k in ["up_aux", "dn_aux", "dn_mode", "up_mode", "dn_ptr"]:
        assert np.array_equal(_np(dev[k]).astype(np.int64), _np(host[k]).astype(np.int64)), k
    assert np.allclose(_np(dev["k_decay"]), host["k_decay"], rtol=1e-14)


@pytest.mark.parametrize("name", ["ring6", "chain4_2mode", "general_lop"])
def test_propagation_through_gpu_built_structure(cuda_device, name, monkeypatch):
    """HopsTrajectory with the GPU-built structure equals the oracle (complex128)."""
    import mesohops_b200.device as dv
    from mesohops_b200 import HopsTrajectory
    from mesohops_b200.hierarchy import TriangularHierarchy
    from oracle import hops_oracle as O
    monkeypatch.setattr(dv, "GPU_BUILD_MIN_AUX", 1)
    f = load_golden(name)
    sysp = golden_system(f)
    noise = f["noise1"]
    path = os.path.join(tempfile.mkdtemp(), "n.npy")
    np.save(path, noise)
    h = HopsTrajectory(sysp, noise_param={"SEED": path, "MODEL": "PRE_CALCULATED",
                                          "TLEN": float(f["tlen"]), "TAU": float(f["tau_noise"])},
                       hierarchy_param={"MAXHIER": int(f["depth"])},
                       device_param={"PRECISION": "complex128"})
    h.initialize(f["psi0"])
    assert isinstance(h.basis, TriangularHierarchy)
    n, dt = 20, float(f["dt"])
    h.propagate(n * dt, dt)
    b = O.OracleBasis({k: sysp[k] for k in ("HAMILTONIAN", "GW_SYSBATH", "L_HIER")},
                      int(f["depth"]))
    _, psi, _, _ = O.propagate(b, f["psi0"], noise, float(f["tau_noise"]), n * dt, dt)
    got = np.array(h.storage["psi_traj"])
    assert np.max(np.abs(got - psi)) <= 1e-10 * np.max(np.abs(psi))
