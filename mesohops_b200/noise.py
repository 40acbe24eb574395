"""HOPS noise on the device (mirror of noise/hops_noise.py).

Models: FFT_FILTER (correlated complex Gaussian noise), PRE_CALCULATED (a
given correlated trajectory) and ZERO.  The raw white noise is drawn on the
GPU (``hops_noise_draw``) from the reference's PCG64(SEED).jumped(lop) streams
with numpy's normal (or uniform, for BOX_MULLER) sampler restated, so a SEED
gives the reference's raw draws (hops_noise.py:558-628); the SEEDs are hashed
into PCG64 states on the GPU as well (numpy's SeedSequence restated).  The
circulant-embedding filter (hops_noise.py:630-716) runs in FP64 on the GPU
through ``hops_noise_filter``.  The correlated noise is stored as complex64
(hops_noise.py:247), one row per unique L-operator.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from . import _lib
from .constants import precision
from .exceptions import UnsupportedRequest
from .params import NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, initialize_dict


def raw_slot_index(ntaus):
    """Assignment of the 4(n_t-1) draws to the 2(n_t-1) complex samples.

    Keeps the draw used by each time slot independent of the trajectory length
    (hops_noise.py:592-628): slot j takes draw re[j] for its real part (or
    Box-Muller radius) and im[j] for its imaginary part (or phase).
    """
    n1 = ntaus - 1
    re = np.concatenate([[0], np.arange(2, 4 * (ntaus - 2), 4), [4 * n1 - 2],
                         np.arange(4 * (ntaus - 2), 3, -4)]).astype(np.int64)
    im = np.concatenate([[1], np.arange(3, 4 * (ntaus - 1) - 1, 4), [4 * n1 - 1],
                         np.arange(4 * (n1 - 1) + 1, 4, -4)]).astype(np.int64)
    return re, im


RAND_MODELS = {"SUM_GAUSSIAN": 0, "BOX_MULLER": 1}


def seed_states(seeds):
    """uint64 [len(seeds)][4]: each trajectory's un-jumped PCG64 generator as
    numpy seeds it (state high, state low, increment high, increment low),
    computed by numpy on the host.  SEED None takes fresh entropy, as the
    reference's PCG64(seed=None) does.  ``seed_states_on_device`` computes the
    same on the GPU."""
    out = np.empty((len(seeds), 4), dtype=np.uint64)
    m = (1 << 64) - 1
    for i, seed in enumerate(seeds):
        st = np.random.PCG64(seed=seed).state["state"]
        out[i] = (st["state"] >> 64, st["state"] & m, st["inc"] >> 64, st["inc"] & m)
    return out


def seed_states_on_device(seeds, device):
    """int64 device tensor [len(seeds), 4], the ``seed_states`` of the SEEDs
    hashed on the GPU (``hops_noise_seed_states``); the host only splits each
    SEED into 32-bit words.  SEED None draws fresh entropy on the host (numpy's
    SeedSequence()), which is then hashed like an integer SEED."""
    words, ptr = [], [0]
    for seed in seeds:
        v = int(np.random.SeedSequence().entropy) if seed is None else int(seed)
        if v < 0:
            raise ValueError(f"expected non-negative integer SEED, got {seed}")
        w = []
        while True:
            w.append(v & 0xFFFFFFFF)
            v >>= 32
            if not v:
                break
        words.extend(w)
        ptr.append(len(words))
    dev = torch.device(device)
    wd = torch.from_numpy(np.array(words, dtype=np.uint32).view(np.int32)).to(dev)
    pd = torch.from_numpy(np.array(ptr, dtype=np.int32)).to(dev)
    st = torch.empty((len(seeds), 4), dtype=torch.int64, device=dev)
    rc = _lib.lib().hops_noise_seed_states(wd.data_ptr(), pd.data_ptr(), len(seeds), st.data_ptr(),
                                           torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(rc, "hops_noise_seed_states")
    return st


def raw_white_noise(seeds, lops, ntaus, rand_model, device):
    """Uncorrelated complex64 draws on the device, [len(seeds) * len(lops),
    2(ntaus-1)]: row b * len(lops) + j is trajectory b's noise for L-operator
    lops[j] (hops_noise.py:453-628, drawn by ``hops_noise_draw``)."""
    if rand_model not in RAND_MODELS:
        raise UnsupportedRequest(f"Noise.param[RAND_MODEL] {rand_model}", "Noise._prepare_rand")
    lops = [int(x) for x in lops]
    if any(x < 0 for x in lops):
        raise UnsupportedRequest("negative L-operator index", "Noise._prepare_rand")
    dev = torch.device(device)
    if not seeds or not lops:
        return torch.empty((len(seeds) * len(lops), 2 * (ntaus - 1)), dtype=torch.complex64,
                           device=dev)
    st = seed_states_on_device(seeds, dev)
    lp = torch.tensor(lops, dtype=torch.int32, device=dev)
    return draw_from_states(st, lp, ntaus, rand_model)


def draw_from_states(states, lops, ntaus, rand_model):
    """The device draws of ``raw_white_noise`` from seed states already on the
    device (int64 view of ``seed_states``, [n_traj, 4]) and an int32 device
    tensor of L-operator indices."""
    n_traj, n_lop = int(states.shape[0]), int(lops.numel())
    z = torch.empty((n_traj * n_lop, 2 * (ntaus - 1)), dtype=torch.complex64,
                    device=states.device)
    rc = _lib.lib().hops_noise_draw(states.data_ptr(), n_traj, lops.data_ptr(), n_lop,
                                    int(ntaus), RAND_MODELS[rand_model], z.data_ptr(),
                                    torch.cuda.current_stream(states.device).cuda_stream)
    _lib.check(rc, "hops_noise_draw")
    return z


def filter_on_device(alpha, z_raw, device, complex128=False):
    """FP64 circulant-embedding filter on the GPU.

    alpha: complex128 [A, n_t] correlation functions; z_raw: complex64
    [R, 2(n_t-1)], a host array or a device tensor, R a multiple of A; row r
    is filtered with alpha row r % A (the trajectories of an ensemble share
    one system's correlation functions).  Returns (complex64 device tensor
    [R, n_t] -- complex128 if complex128 -- and the number of clipped
    negative spectral values over the R rows).
    """
    L = _lib.lib()
    A, n_t = alpha.shape
    dev = torch.device(device)
    a = torch.from_numpy(np.ascontiguousarray(alpha, dtype=np.complex128)).to(dev)
    if isinstance(z_raw, torch.Tensor):
        z = z_raw.to(device=dev, dtype=torch.complex64).contiguous()
    else:
        z = torch.from_numpy(np.ascontiguousarray(z_raw, dtype=np.complex64)).to(dev)
    R = int(z.shape[0])
    work = torch.empty(int(L.hops_noise_filter_work_doubles(R, n_t)), dtype=torch.float64, device=dev)
    out = torch.empty((R, n_t), dtype=torch.complex128 if complex128 else torch.complex64,
                      device=dev)
    nneg = C.c_int64(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.hops_noise_filter_shared(a.data_ptr(), A, z.data_ptr(), R, n_t, work.data_ptr(),
                                    out.data_ptr() if complex128 else None,
                                    None if complex128 else out.data_ptr(), C.byref(nneg), stream)
    _lib.check(rc, "hops_noise_filter")
    return out, int(nneg.value)


def window_means(noise, start, k, n_out, real_only=False):
    """Means of n_out consecutive windows of k samples from sample `start` of
    each row of a complex64 device tensor [..., n_t], bit-identical to numpy's
    mean of the same complex64 (real_only: float32 real parts) samples
    (hops_noise_window_mean)."""
    noise = noise.contiguous()
    n_t = int(noise.shape[-1])
    rows = noise.numel() // max(n_t, 1)
    out = torch.empty(tuple(noise.shape[:-1]) + (int(n_out),), dtype=torch.complex64,
                      device=noise.device)
    rc = _lib.lib().hops_noise_window_mean(
        noise.data_ptr(), rows, n_t, int(start), int(k), int(n_out), 1 if real_only else 0,
        out.data_ptr(), torch.cuda.current_stream(noise.device).cuda_stream)
    _lib.check(rc, "hops_noise_window_mean")
    return out


class HopsNoise:
    """One noise trajectory (noise 1 or noise 2) of a HOPS trajectory."""

    def __init__(self, noise_param, system, noise_type=1):
        p = dict(noise_param)
        if noise_type == 2 and "FLAG_REAL" not in p and p.get("MODEL") != "ZERO":
            p["FLAG_REAL"] = True   # prepare_functions.py:72-77
        self.param = initialize_dict(p, NOISE_DICT_DEFAULT, NOISE_DICT_TYPES, "HopsNoise")
        # INTERPOLATE (hops_noise.py:242-279,379-384): the reference samples a
        # cubic spline through the correlated noise, and its step check
        # (hops_trajectory.py:434-447, 579-614) only lets it sample at the
        # grid times of the noise axis, where the spline returns the samples
        # themselves; the difference is then only that the samples stay
        # complex128 instead of being rounded to complex64
        self.interpolate = bool(self.param["INTERPOLATE"])
        self.system = system
        self.noise_type = noise_type
        n_t = int(np.ceil(self.param["TLEN"] / self.param["TAU"])) + 1
        self.param["T_AXIS"] = np.arange(n_t) * self.param["TAU"]
        self.n_t = n_t
        self.n_lop = system.n_lop
        self._dev = None
        self._host = None
        self.n_clipped = 0

    # ------------------------------------------------------------------
    def _corr(self):
        """alpha per unique L on the noise time axis (hops_noise.py:167-192)."""
        sysm = self.system
        if self.noise_type == 1:
            fn, params, by_l = sysm.alpha1, sysm.param_noise1, sysm.nmodes1_by_l
        else:
            fn, params, by_l = sysm.alpha2, sysm.param_noise2, sysm.nmodes2_by_l
        t = self.param["T_AXIS"]
        alpha = np.zeros((self.n_lop, len(t)), dtype=np.complex128)
        for j, modes in enumerate(by_l):
            for i in modes:
                alpha[j] += fn(t, *params[i])
        return alpha

    def _uncorrelated(self, device):
        seed = self.param["SEED"]
        shape = (self.n_lop, 2 * (self.n_t - 1))
        if isinstance(seed, str):
            if not os.path.isfile(seed) or seed[-4:] != ".npy":
                raise UnsupportedRequest(f"Noise.param[SEED] {seed} is not a valid .npy file",
                                         "Noise._prepare_rand", True)
            seed = np.load(seed)
        if isinstance(seed, np.ndarray):
            if seed.shape != shape:
                raise UnsupportedRequest("Noise.param[SEED] is an array of the wrong length",
                                         "Noise._prepare_rand", True)
            return seed
        return raw_white_noise([seed], range(self.n_lop), self.n_t, self.param["RAND_MODEL"],
                               device)

    def prepare(self, device):
        """Correlated noise as a device tensor [n_lop, n_t] (None for ZERO):
        complex64, or complex128 with INTERPOLATE."""
        if self._dev is not None or self.param["MODEL"] == "ZERO":
            return self._dev
        model = self.param["MODEL"]
        if model == "FFT_FILTER":
            z = self._uncorrelated(device)
            if self.param["STORE_RAW_NOISE"]:
                self.param["Z_UNCORRELATED"] = (z.cpu().numpy() if isinstance(z, torch.Tensor)
                                                else z)
            noise, self.n_clipped = filter_on_device(self._corr(), z, device,
                                                     complex128=self.interpolate)
        elif model == "PRE_CALCULATED":
            seed = self.param["SEED"]
            if isinstance(seed, str):
                if not os.path.isfile(seed) or seed[-4:] != ".npy":
                    raise UnsupportedRequest(f"Noise.param[SEED] {seed} is not a valid .npy "
                                             "file", "Noise.prepare_noise", True)
                # a file's samples are complex64 (hops_noise.py:287)
                seed = np.complex64(np.load(seed))
            if not isinstance(seed, (list, np.ndarray)):
                raise UnsupportedRequest(f"Noise.param[SEED] of type {type(seed)}",
                                         "Noise.prepare_noise")
            seed = np.asarray(seed)
            if seed.shape != (self.n_lop, self.n_t):
                raise UnsupportedRequest("Noise.param[SEED] is an array of the wrong length",
                                         "Noise.prepare_noise", True)
            dt = np.complex128 if self.interpolate else np.complex64
            noise = torch.from_numpy(np.ascontiguousarray(seed.astype(dt))).to(device)
        else:
            raise UnsupportedRequest(f"Noise.param[MODEL] {model}", "Noise.prepare_noise")
        if self.param["FLAG_REAL"]:
            noise = torch.complex(noise.real, torch.zeros_like(noise.real))
        self._dev = noise.contiguous()
        return self._dev

    def effective(self, t0, tau, n_steps):
        """Effective noise of EFFECTIVE_NOISE_INTEGRATION for n_steps RK4 steps from t0
        (integrator_rk.py:115-128): complex64 device tensor [n_lop, 2 n_steps + 1] of
        the means of consecutive windows of tau / (2 TAU) samples starting at t0, so
        the RK slots of step n are windows 2n, 2n+1, 2n+2.  None for ZERO noise."""
        if self._dev is None:
            return None
        if self.interpolate:
            raise UnsupportedRequest("EFFECTIVE_NOISE_INTEGRATION with INTERPOLATE noise",
                                     "mesohops_b200 HopsNoise")
        k = int(round(tau * 0.5 / self.param["TAU"]))
        start = self.time_index(t0)
        n_out = 2 * int(n_steps) + 1
        if start + n_out * k > self.n_t:
            raise UnsupportedRequest("t-samples outside of the defined t-axis",
                                     "NoiseModel.get_noise()")
        return window_means(self._dev, start, k, n_out, bool(self.param["FLAG_REAL"]))

    def host(self):
        if self._host is None and self._dev is not None:
            self._host = self._dev.cpu().numpy()
        return self._host

    def time_index(self, t):
        """Exact index of time t on the noise axis (hops_noise.py:437-447)."""
        it = int(round(t / self.param["TAU"]))
        if it < 0 or it >= self.n_t or abs(it * self.param["TAU"] - t) >= precision:
            raise UnsupportedRequest("Off axis t-samples when INTERPOLATE = False",
                                     "NoiseModel.get_noise()")
        return it

    def get_noise(self, t_axis, list_lop=None):
        """[len(list_lop), len(t_axis)] samples (hops_noise.py:339-451):
        complex64, or complex128 with INTERPOLATE."""
        if list_lop is None:
            list_lop = np.arange(self.n_lop)
        dt = np.complex128 if self.interpolate else np.complex64
        if self.param["MODEL"] == "ZERO":
            return np.zeros((len(list_lop), len(t_axis)), dtype=dt)
        if self._dev is None:
            self.prepare("cuda")
        h = self.host()
        idx = [self.time_index(t) for t in t_axis]
        return np.ascontiguousarray(h[np.ix_(np.asarray(list_lop, dtype=np.int64), idx)],
                                    dtype=dt)
