"""Parameter dictionaries of the drop-in surface.

The defaults and accepted types are the reference's (hops_trajectory.py:34-50,
hops_eom.py:20-41, hops_hierarchy.py:16-22, hops_noise.py:20-44) so user
dictionaries written for MesoHOPS are accepted unchanged.  ``initialize_dict``
restates util/dynamic_dict.py:47-79: unknown keys raise UnsupportedRequest,
wrong types raise TypeError, missing keys take their defaults.
"""
import copy

import numpy as np

from .exceptions import UnsupportedRequest

INTEGRATION_DICT_DEFAULT = {
    "INTEGRATOR": "RUNGE_KUTTA",
    "EARLY_ADAPTIVE_INTEGRATOR": "INCH_WORM",
    "EARLY_INTEGRATOR_STEPS": 5,
    "INCHWORM_CAP": 5,
    "STATIC_BASIS": None,
    "EFFECTIVE_NOISE_INTEGRATION": False,
}
INTEGRATION_DICT_TYPES = {
    "INTEGRATOR": [str],
    "EARLY_ADAPTIVE_INTEGRATOR": [str],
    "EARLY_INTEGRATOR_STEPS": [int],
    "INCHWORM_CAP": [int],
    "STATIC_BASIS": [type(None), list, np.ndarray],
    "EFFECTIVE_NOISE_INTEGRATION": [bool],
}

EOM_DICT_DEFAULT = {
    "TIME_DEPENDENCE": False,
    "EQUATION_OF_MOTION": "NORMALIZED NONLINEAR",
    "ADAPTIVE_H": False,
    "ADAPTIVE_S": False,
    "DELTA_A": 0,
    "DELTA_S": 0,
    "UPDATE_STEP": None,
    "F_DISCARD": 0,
}
EOM_DICT_TYPES = {
    "TIME_DEPENDENCE": [bool],
    "EQUATION_OF_MOTION": [str],
    "ADAPTIVE": [bool],
    "ADAPTIVE_H": [bool],
    "ADAPTIVE_S": [bool],
    "DELTA_A": [float, int],
    "DELTA_S": [float, int],
    "UPDATE_STEP": [float, bool, type(None), int],
    "F_DISCARD": [float],
}

HIERARCHY_DICT_DEFAULT = {"MAXHIER": 3, "TERMINATOR": False, "STATIC_FILTERS": []}
HIERARCHY_DICT_TYPES = {
    "MAXHIER": [int],
    "TERMINATOR": [bool, str],
    "STATIC_FILTERS": [list],
}

NOISE_DICT_DEFAULT = {
    "SEED": None,
    "MODEL": "FFT_FILTER",
    "TLEN": 1000.0,
    "TAU": 1.0,
    "INTERPOLATE": False,
    "RAND_MODEL": "SUM_GAUSSIAN",
    "STORE_RAW_NOISE": False,
    "NOISE_WINDOW": None,
    "ADAPTIVE": False,
    "FLAG_REAL": False,
}
NOISE_DICT_TYPES = {
    "SEED": [int, type(None), str, np.ndarray],
    "MODEL": [str],
    "TLEN": [float],
    "TAU": [float],
    "INTERPOLATE": [bool],
    "RAND_MODEL": [str],
    "STORE_RAW_NOISE": [bool],
    "NOISE_WINDOW": [type(None), float, int],
    "ADAPTIVE": [bool],
    "FLAG_REAL": [bool],
}

STORAGE_DICT_DEFAULT = {
    "phi_traj": False,
    "psi_traj": True,
    "t_axis": True,
    "aux_list": False,
    "state_list": False,
    "list_nhier": False,
    "list_nstate": False,
    "z_mem": False,
}

# Options of this implementation; kept in a separate dictionary so that the
# reference dictionaries above stay exactly as MesoHOPS defines them.
DEVICE_DICT_DEFAULT = {
    "PRECISION": "complex128",   # or "mixed" (complex128 state, complex64 stage vectors)
                                 # or "complex64"; FP64 kept for <L>, norm, z_mem
    "DEVICE": "cuda:0",
    "KERNEL": "auto",            # "auto", "resident" or "streaming"
}


def initialize_dict(param, defaults, types, name):
    """Validated copy of a user dictionary with defaults filled in."""
    out = copy.deepcopy(param) if param is not None else {}
    for key in out:
        if key not in defaults:
            raise UnsupportedRequest(key, name)
    for key, default in defaults.items():
        if key in out:
            if type(out[key]) not in types[key]:
                raise TypeError(f"{key}-->{out[key]} is of type {type(out[key])} not the "
                                f"supported types {types[key]}")
        else:
            out[key] = copy.deepcopy(default)
    return out
