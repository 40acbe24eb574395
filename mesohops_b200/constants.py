"""Physical constants in the reference's units (util/physical_constants.py:21-28)."""
import math

precision = 1e-8            # time-point comparison tolerance
h = 33357.179               # cm^-1 fs
hbar = h / (2 * math.pi)    # cm^-1 fs / rad
kB = 0.69503                # cm^-1 / K
