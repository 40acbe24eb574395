"""Writes hops_ziggurat_table.h, the 256-layer normal ziggurat of the device
noise draws (hops_rng.cu).

The reference draws its raw noise with numpy's ``Generator.normal``
(noise/hops_noise.py:583-589), a Marsaglia-Tsang ziggurat ("The Ziggurat
Method for Generating Random Variables", J. Stat. Softw. 5(8), 2000) with 256
layers over a 52-bit mantissa field: the base layer ends at r =
3.6541528853610088 and every layer has the area v = r f(r) + int_r^inf f of
the base strip (f(x) = exp(-x^2/2)).  Layer edges x_255 = r > x_254 > ... >
x_1 follow x_{i-1} = sqrt(-2 log(v / x_i + f(x_i))).  Per layer the sampler
keeps

  wi[i] = x_i / 2^52            (wi[0] = (v / f(r)) / 2^52, the base strip)
  ki[i] = floor(2^52 x_{i-1} / x_i)   (ki[0] = floor(2^52 r f(r) / v), ki[1] = 0)
  fi[i] = f(x_i)                (fi[0] = 1)

Here the edges are computed with 60 significant digits.  numpy's own table
was built in double precision, so its wi differ from the correctly rounded
edges by up to a few tens of units in the last place (a rounding walk that
grows toward the top layers).  A draw is wi[idx] times the 52-bit field, so
bit-identical draws need numpy's wi exactly: for every layer this script
reads wi off seeded numpy draws (the double w with w * field == |draw| for
every fast-path draw of that layer, found among the neighbours of the
correctly rounded edge) and checks that the restated sampler then reproduces
a million numpy draws bit for bit.  ki and fi only decide acceptance; a
difference from numpy's own ki or fi could change a draw only when a
uniform falls within a few units in the last place of a threshold (about
1e-14 per draw), so they are taken from the high-precision edges.

Run: python mesohops_b200/csrc/make_ziggurat_table.py (needs numpy, mpmath).
"""
import math
import os

import mpmath as mp
import numpy as np

R_DOUBLE = 3.6541528853610088
MASK52 = (1 << 52) - 1
U53 = 1.0 / 9007199254740992.0


def layer_edges():
    mp.mp.dps = 60
    r = mp.mpf(R_DOUBLE)
    f = lambda x: mp.e ** (-x * x / 2)  # noqa: E731
    v = r * f(r) + mp.sqrt(mp.pi / 2) * mp.erfc(r / mp.sqrt(2))
    x = [None] * 256
    x[255] = r
    for i in range(254, 0, -1):
        x[i] = mp.sqrt(-2 * mp.log(v / x[i + 1] + f(x[i + 1])))
    two52 = mp.mpf(2) ** 52
    wi = [float(v / f(r) / two52)] + [float(x[i] / two52) for i in range(1, 256)]
    ki = [int(mp.floor(r * f(r) / v * two52)), 0] + \
         [int(mp.floor(x[i - 1] / x[i] * two52)) for i in range(2, 256)]
    fi = [1.0] + [float(f(x[i])) for i in range(1, 256)]
    return wi, ki, fi


def restated_normals(raw, n, wi, ki, fi, record=None):
    """numpy's standard normal from a raw uint64 stream: the low 8 bits pick
    the layer, the next bit the sign, the next 52 bits the field; fast path
    when field < ki; layer 0 falls back to Marsaglia's exponential tail at r;
    the others accept x when a uniform height in the layer lies under f(x).
    record(idx, field, value) sees each draw (idx -1 for a tail draw)."""
    out = np.empty(n)
    pos = 0
    for k in range(n):
        while True:
            r = int(raw[pos])
            pos += 1
            idx = r & 0xFF
            r >>= 8
            field = (r >> 1) & MASK52
            x = field * wi[idx]
            if r & 1:
                x = -x
            if field < ki[idx]:
                break
            if idx == 0:
                while True:
                    u1 = (int(raw[pos]) >> 11) * U53
                    u2 = (int(raw[pos + 1]) >> 11) * U53
                    pos += 2
                    xx = -(1.0 / R_DOUBLE) * math.log1p(-u1)
                    yy = -math.log1p(-u2)
                    if yy + yy > xx * xx:
                        break
                x = -(R_DOUBLE + xx) if (field >> 8) & 1 else R_DOUBLE + xx
                idx = -1
                break
            u = (int(raw[pos]) >> 11) * U53
            pos += 1
            if (fi[idx - 1] - fi[idx]) * u + fi[idx] < math.exp(-0.5 * x * x):
                break
        out[k] = x
        if record is not None:
            record(idx, field, x)
    return out, pos


def fit_wi(wi, ki, fi, seed=20240, n=600000):
    """numpy's wi read off n seeded draws (the decisions use ki/fi, so the
    stream stays in step while wi is still the rounded edge)."""
    raw = np.random.Generator(np.random.PCG64(seed)).bit_generator.random_raw(4 * n)
    ref = np.random.Generator(np.random.PCG64(seed)).normal(size=n)
    seen = {}
    k = [0]

    def rec(idx, field, x):
        if idx >= 0 and field > (1 << 46):
            seen.setdefault(idx, []).append((field, abs(ref[k[0]])))
        k[0] += 1

    restated_normals(raw, n, wi, ki, fi, record=rec)
    fitted = list(wi)
    for idx in range(256):
        pts = seen.get(idx, [])[:400]
        if len(pts) < 20:
            raise RuntimeError(f"layer {idx}: only {len(pts)} draws to fit")
        # the candidates lie within a few units of |draw| / field of any draw
        hits = []
        c0 = pts[0][1] / pts[0][0]
        for d in range(-8, 9):
            c = c0
            for _ in range(abs(d)):
                c = float(np.nextafter(c, np.inf if d > 0 else -np.inf))
            if all(f * c == a for f, a in pts):
                hits.append(c)
        if len(hits) != 1:
            raise RuntimeError(f"layer {idx}: {len(hits)} candidates")
        fitted[idx] = hits[0]
        shift = (hits[0] - wi[idx]) / float(np.spacing(wi[idx]))
        if abs(shift) > 256:
            raise RuntimeError(f"layer {idx}: {shift:.0f} units from its edge")
    return fitted


def check(wi, ki, fi, seed=7, n=1000000):
    raw = np.random.Generator(np.random.PCG64(seed)).bit_generator.random_raw(4 * n)
    ref = np.random.Generator(np.random.PCG64(seed)).normal(size=n)
    got, _ = restated_normals(raw, n, wi, ki, fi)
    bad = int(np.count_nonzero(got != ref))
    if bad:
        raise RuntimeError(f"{bad} of {n} draws differ from numpy")


def write(path, wi, ki, fi):
    def rows(vals, fmt):
        s = [fmt(v) for v in vals]
        return ",\n".join("    " + ", ".join(s[i:i + 4]) for i in range(0, 256, 4))

    with open(path, "w") as fh:
        fh.write("// 256-layer normal ziggurat of the device noise draws; written by\n"
                 "// make_ziggurat_table.py (layer edges, the reading of wi and the check\n"
                 "// against numpy's Generator.normal are described there).  Do not edit.\n"
                 "#pragma once\n\n")
        fh.write("#define HOPS_ZIG_WI {\\\n" + rows(wi, lambda v: float(v).hex())
                 .replace("\n", "\\\n") + "}\n\n")
        fh.write("#define HOPS_ZIG_KI {\\\n" + rows(ki, lambda v: f"0x{v:013x}ull")
                 .replace("\n", "\\\n") + "}\n\n")
        fh.write("#define HOPS_ZIG_FI {\\\n" + rows(fi, lambda v: float(v).hex())
                 .replace("\n", "\\\n") + "}\n")


def read(path):
    """(wi, ki, fi) back from the header (used by the tests)."""
    txt = open(path).read()

    def block(name):
        body = txt.split(f"#define {name} {{")[1].split("}")[0]
        return [t.strip() for t in body.replace("\\", "").split(",") if t.strip()]

    wi = [float.fromhex(t) for t in block("HOPS_ZIG_WI")]
    ki = [int(t.rstrip("ul"), 16) for t in block("HOPS_ZIG_KI")]
    fi = [float.fromhex(t) for t in block("HOPS_ZIG_FI")]
    return wi, ki, fi


if __name__ == "__main__":
    wi, ki, fi = layer_edges()
    wi = fit_wi(wi, ki, fi)
    check(wi, ki, fi)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hops_ziggurat_table.h")
    write(out, wi, ki, fi)
    print("wrote", out)
