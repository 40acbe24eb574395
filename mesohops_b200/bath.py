"""Bath correlation helpers used to build system parameter dictionaries.

bcf_exp restates trajectory/exp_noise.py:5-25; bcf_convert_dl_to_exp restates
util/bath_corr_functions.py:70-112 (Drude-Lorentz -> exponential modes).
"""
import numpy as np

from .constants import hbar, kB


def bcf_exp(t_axis, g, w):
    """alpha(t) = g exp(-w t / hbar)."""
    return g * np.exp(-w * np.asarray(t_axis) / hbar)


def bcf_convert_dl_to_exp(lambda_dl, gamma_dl, temp, k_matsubara=0):
    """High-temperature mode (+ optional Matsubara modes) of a Drude-Lorentz bath.

    Returns [g_0, w_0, g_1, w_1, ...].
    """
    beta = 1.0 / (kB * temp)
    g0 = 2.0 * lambda_dl / beta - 1j * lambda_dl * gamma_dl
    w0 = gamma_dl
    nu = 2.0 * np.pi / beta
    extra = []
    for k in range(1, k_matsubara + 1):
        wk = k * nu
        jk = 2.0 * lambda_dl * gamma_dl * (1j * wk) / ((1j * wk) ** 2 + gamma_dl ** 2)
        extra += [2j * jk / beta, wk]
        g0 += 2.0 * lambda_dl / beta * (2.0 * gamma_dl ** 2) / (gamma_dl ** 2 - wk ** 2)
    return [g0, w0] + extra
