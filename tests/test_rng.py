"""Raw noise draws: the restated PCG64 jump and normal ziggurat on the CPU
against numpy (the reference's generator, hops_noise.py:583-589), and the
device draws of ``hops_noise_draw`` against the oracle's numpy draws and the
reference's own raw noise (Z_UNCORRELATED of tests/golden/noise_dimer.npz)."""
import os
import sys

import numpy as np
import pytest

from conftest import load_golden
from oracle import hops_oracle as O

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "mesohops_b200", "csrc")
sys.path.insert(0, CSRC)
import make_ziggurat_table as Z  # noqa: E402

M128 = (1 << 128) - 1
MULT = 0x2360ED051FC65DA44385DF649FCCF645
JUMP = 0x9E3779B97F4A7C15F39CC0605CEDC835


def advance(state, inc, delta):
    """PCG state after delta steps (the skip hops_rng.cu pcg_advance takes)."""
    am, ap, cm, cp = 1, 0, MULT, inc
    delta &= M128
    while delta:
        if delta & 1:
            am = (am * cm) & M128
            ap = (ap * cm + cp) & M128
        cp = ((cm + 1) * cp) & M128
        cm = (cm * cm) & M128
        delta >>= 1
    return (am * state + ap) & M128


def xsl_rr(state):
    x = ((state >> 64) ^ state) & ((1 << 64) - 1)
    rot = state >> 122
    return ((x >> rot) | (x << ((64 - rot) & 63))) & ((1 << 64) - 1)


@pytest.mark.parametrize("seed", [0, 7, 123456789, 2**63 + 11])
def test_pcg64_jump_and_output_restated(seed):
    st = np.random.PCG64(seed).state["state"]
    for lop in (0, 1, 2, 19, 499):
        s = advance(st["state"], st["inc"], lop * JUMP)
        assert np.random.PCG64(seed).jumped(lop).state["state"]["state"] == s
        mine = []
        for _ in range(5):
            s = (s * MULT + st["inc"]) & M128
            mine.append(xsl_rr(s))
        assert [int(v) for v in np.random.PCG64(seed).jumped(lop).random_raw(5)] == mine


def test_ziggurat_table_reproduces_numpy_normals():
    """The committed table with the restated sampler gives numpy's normals bit
    for bit, tail draws included."""
    wi, ki, fi = Z.read(os.path.join(CSRC, "hops_ziggurat_table.h"))
    assert len(wi) == len(ki) == len(fi) == 256
    n_tail = 0
    for seed, lop in ((0, 0), (3, 5), (2024, 17)):
        bg = np.random.PCG64(seed).jumped(lop)
        raw = np.random.PCG64(seed).jumped(lop).random_raw(4 * 60000)
        ref = np.random.Generator(bg).normal(loc=0, size=60000)
        got, _ = Z.restated_normals(raw, 60000, wi, ki, fi)
        assert np.array_equal(got, ref)
        n_tail += int(np.count_nonzero(np.abs(ref) > Z.R_DOUBLE))
    assert n_tail > 10


def test_slot_closed_form_matches_indexing():
    """hops_rng.cu places draw pair (d, d+1) in slot 0 (d = 0), (d+2)/4 (d = 2
    mod 4) or 2(n_t-1) - d/4 (d = 0 mod 4, d > 0)."""
    for n in (2, 3, 4, 17, 503):
        re, im = O.raw_index(n)
        n1 = n - 1
        slot_of = {}
        for d in range(0, 4 * n1, 2):
            slot_of[d] = 0 if d == 0 else ((d + 2) // 4 if d % 4 == 2 else 2 * n1 - d // 4)
        assert sorted(slot_of.values()) == list(range(2 * n1))
        for j in range(2 * n1):
            assert slot_of[int(re[j])] == j and int(im[j]) == int(re[j]) + 1


@pytest.mark.gpu
@pytest.mark.parametrize("model", ["SUM_GAUSSIAN", "BOX_MULLER"])
def test_device_draws_match_reference_raw_noise(cuda_device, model):
    from mesohops_b200.noise import raw_white_noise
    f = load_golden("noise_dimer")
    n_t = int(np.ceil(float(f["tlen"]) / float(f["tau"]))) + 1
    z = raw_white_noise([0], [0, 1], n_t, model, cuda_device).cpu().numpy()
    ref = f[model + "_raw"]
    if model == "SUM_GAUSSIAN":
        assert np.array_equal(z, ref)
    else:
        # device log / sincos: at most one complex64 unit in the last place
        for part in (np.real, np.imag):
            a, b = part(z).astype(np.float32), part(ref).astype(np.float32)
            ulps = np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))
            assert ulps.max() <= 1
            assert np.count_nonzero(ulps) <= 4


@pytest.mark.gpu
def test_device_draws_match_numpy_batch(cuda_device):
    """A batch of trajectories with their own SEEDs over several L-operators
    (the ensemble's layout) equals numpy's draws row for row, for time axes
    from the shortest (n_t = 2) to the benchmark ring's."""
    from mesohops_b200.noise import raw_white_noise
    seeds = [0, 1, 99, 12345, 2**40 + 3, 7]
    lops = [0, 3, 1, 19]
    for n_t in (2, 3, 504):
        z = raw_white_noise(seeds, lops, n_t, "SUM_GAUSSIAN", cuda_device).cpu().numpy()
        ref = np.concatenate([O.raw_draws(s, lops, n_t) for s in seeds], axis=0)
        assert z.shape == ref.shape
        assert np.array_equal(z, ref)


@pytest.mark.gpu
def test_device_draws_ring_batch_bitwise(cuda_device):
    """128 trajectories x 20 L-operators x 503 samples (the ring workload's
    raw noise, 5.1 M normals): equal to numpy's draws bit for bit."""
    from mesohops_b200.noise import raw_white_noise
    seeds = list(range(1000, 1128))
    n_t = 503
    z = raw_white_noise(seeds, range(20), n_t, "SUM_GAUSSIAN", cuda_device).cpu().numpy()
    ref = np.concatenate([O.raw_draws(s, range(20), n_t) for s in seeds], axis=0)
    assert np.count_nonzero(z != ref) == 0


@pytest.mark.gpu
def test_device_box_muller_batch_within_one_ulp(cuda_device):
    from mesohops_b200.noise import raw_white_noise
    seeds, lops, n_t = [5, 6, 7], [0, 2, 9], 300
    z = raw_white_noise(seeds, lops, n_t, "BOX_MULLER", cuda_device).cpu().numpy()
    ref = np.concatenate([O.raw_draws(s, lops, n_t, "BOX_MULLER") for s in seeds], axis=0)
    for part in (np.real, np.imag):
        a = part(z).astype(np.float32).view(np.int32).astype(np.int64)
        b = part(ref).astype(np.float32).view(np.int32).astype(np.int64)
        assert np.abs(a - b).max() <= 1
    assert np.count_nonzero(z != ref) <= z.size // 1000


@pytest.mark.gpu
def test_device_draws_unseeded_and_empty(cuda_device):
    """SEED None: fresh entropy per trajectory (the reference seeds PCG64(None)),
    so rows differ and the draws are standard complex Gaussians (variance 1 per
    part); an empty L-operator list gives an empty array without a launch."""
    from mesohops_b200.noise import raw_white_noise
    z = raw_white_noise([None, None], [0, 1], 2001, "SUM_GAUSSIAN", cuda_device).cpu().numpy()
    assert not np.array_equal(z[0], z[2]) and not np.array_equal(z[0], z[1])
    assert abs(np.var(z.real) - 1.0) < 0.05 and abs(np.var(z.imag) - 1.0) < 0.05
    assert abs(np.mean(z)) < 0.05
    e = raw_white_noise([1, 2], [], 50, "SUM_GAUSSIAN", cuda_device)
    assert tuple(e.shape) == (0, 98)


SEEDS = [0, 1, 7, 12345, 2**32 - 1, 2**32 + 5, 2**63 + 11, 2**64 + 9, 2**100 + 3, 2**160 + 17]


def restated_seed_state(seed):
    """numpy's SeedSequence(seed) + PCG64 seeding, the steps k_seed_states takes."""
    m32 = 0xFFFFFFFF
    ent = []
    v = seed
    while True:
        ent.append(v & m32)
        v >>= 32
        if not v:
            break
    hc = [0x43B0D7E5]

    def hashmix(x):
        x = (x ^ hc[0]) & m32
        hc[0] = (hc[0] * 0x931E8875) & m32
        x = (x * hc[0]) & m32
        return x ^ (x >> 16)

    def mix(x, y):
        r = (0xCA01F9DD * x - 0x4973F715 * y) & m32
        return r ^ (r >> 16)

    pool = [hashmix(ent[i] if i < len(ent) else 0) for i in range(4)]
    for s in range(4):
        for d in range(4):
            if s != d:
                pool[d] = mix(pool[d], hashmix(pool[s]))
    for s in range(4, len(ent)):
        for d in range(4):
            pool[d] = mix(pool[d], hashmix(ent[s]))
    hb, out = 0x8B51F9DD, []
    for i in range(8):
        x = (pool[i % 4] ^ hb) & m32
        hb = (hb * 0x58F38DED) & m32
        x = (x * hb) & m32
        out.append(x ^ (x >> 16))
    w = [out[2 * i] | (out[2 * i + 1] << 32) for i in range(4)]
    inc = ((((w[2] << 64) | w[3]) << 1) | 1) & M128
    st = (((inc + ((w[0] << 64) | w[1])) & M128) * MULT + inc) & M128
    return st, inc


def test_seed_hashing_restated():
    for seed in SEEDS:
        st = np.random.PCG64(seed).state["state"]
        assert restated_seed_state(seed) == (st["state"], st["inc"])


@pytest.mark.gpu
def test_device_seed_states_equal_numpy(cuda_device):
    from mesohops_b200.noise import seed_states, seed_states_on_device
    dev = seed_states_on_device(SEEDS, cuda_device).cpu().numpy().view(np.uint64)
    assert np.array_equal(dev, seed_states(SEEDS))
    with pytest.raises(ValueError):
        seed_states_on_device([3, -1], cuda_device)
