#!/usr/bin/env python3
"""Generate ``dd_tables.h``: the double-double constant tables of the array hot path.

Every entry is derived here from its closed form with mpmath at 320-bit working
precision and split into double-double limbs by round-to-nearest
(``hi = RN(v)``, ``lo = RN(v - hi)``).  The tables must be bit-identical to the
ones the reference library compiles in (``src/dd_constants.hh`` of
multifloats 0.10.3), because the device kernels restate the reference's
polynomial and range-reduction steps and are required to reproduce its results
bit for bit.  ``--check REF_HEADER`` parses that header and compares every
value; the comparison ran clean when this file was written.

Closed forms (reference section in ``src/dd_constants.hh``):

* ``log2_e`` = 1/ln 2, ``ln_2`` = ln 2, ``inv_sqrt2`` = 1/sqrt 2, ``pi_quarter`` = pi/4
* ``ln2_cw1..3``: cw1 = RN(ln 2) with the low 20 significand bits cleared (33-bit),
  cw2 = RN(ln2 - cw1), cw3 = RN(ln2 - cw1 - cw2)           (EXP section)
* ``pi_half_cw1..3``: cw1 = RN(pi/2), cw2 = RN(pi/2 - cw1), cw3 = RN(pi/2 - cw1 - cw2)
* ``exp2_coefs[k]`` = (ln 2)^k / k!, k = 0..15                (EXP2 section)
* ``exp2_table[k]`` = 2^((k-128)/256), k = 0..256
* ``exp_max`` = RN(1024 ln 2), ``exp_min`` = -750
* ``exp2_max`` = 1024 - 2^-42, ``exp2_min`` = -1080, ``log10_2`` = log10(2)
* ``log2_narrow[k]`` (k<7), ``log2_wide[k]`` (k<11) = 2 / ((2k+1) ln 2)   (LOG2 section)
* ``log2_centers[i]`` = 1 + (2i+1)/64, ``log2_values[i]`` = log2(centers[i]), i < 32
* ``sin_taylor[k]`` = (-1)^k/(2k+1)!, ``cos_taylor[k]`` = (-1)^k/(2k)!, k < 13

Usage::

    python gen_dd_tables.py                 # (re)write dd_tables.h next to this file
    python gen_dd_tables.py --check HEADER  # compare with a reference dd_constants.hh
"""
from __future__ import annotations

import os
import re
import struct
import sys

from mpmath import mp, mpf, log, pi, sqrt, factorial

mp.prec = 320

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "dd_tables.h")


def rn(v) -> float:
    return float(v)  # mpmath rounds to nearest double


def dd(v):
    hi = rn(v)
    lo = rn(v - mpf(hi))
    return hi, lo


def clear_low_bits(x: float, nbits: int) -> float:
    (u,) = struct.unpack("<Q", struct.pack("<d", x))
    u &= ~((1 << nbits) - 1)
    (r,) = struct.unpack("<d", struct.pack("<Q", u))
    return r


def build() -> dict[str, list[float]]:
    t: dict[str, list[float]] = {}
    ln2 = log(2)

    def put_dd(name, values):
        pairs = [dd(v) for v in values]
        t[name + "_hi"] = [p[0] for p in pairs]
        t[name + "_lo"] = [p[1] for p in pairs]

    put_dd("log2_e", [1 / ln2])
    put_dd("ln_2", [ln2])
    put_dd("inv_sqrt2", [1 / sqrt(2)])
    put_dd("pi_quarter", [pi / 4])

    cw1 = clear_low_bits(rn(ln2), 20)
    cw2 = rn(ln2 - mpf(cw1))
    cw3 = rn(ln2 - mpf(cw1) - mpf(cw2))
    t["ln2_cw"] = [cw1, cw2, cw3]

    ph = pi / 2
    p1 = rn(ph)
    p2 = rn(ph - mpf(p1))
    p3 = rn(ph - mpf(p1) - mpf(p2))
    t["pi_half_cw"] = [p1, p2, p3]

    put_dd("exp2_coefs", [ln2 ** k / factorial(k) for k in range(16)])
    put_dd("exp2_table", [mpf(2) ** (mpf(k - 128) / 256) for k in range(257)])
    t["exp_max"] = [rn(1024 * ln2)]
    t["exp_min"] = [-750.0]
    t["exp2_max"] = [1024.0 - 2.0 ** -42]
    t["exp2_min"] = [-1080.0]
    put_dd("log10_2", [log(2, 10)])

    put_dd("log2_narrow", [2 / ((2 * k + 1) * ln2) for k in range(7)])
    put_dd("log2_wide", [2 / ((2 * k + 1) * ln2) for k in range(11)])
    centers = [1 + mpf(2 * i + 1) / 64 for i in range(32)]
    t["log2_centers"] = [rn(c) for c in centers]
    put_dd("log2_values", [log(c, 2) for c in centers])

    put_dd("sin_taylor", [mpf(-1) ** k / factorial(2 * k + 1) for k in range(13)])
    put_dd("cos_taylor", [mpf(-1) ** k / factorial(2 * k) for k in range(13)])
    return t


# names as the reference header spells them, for --check
REF_NAMES = {
    "log2_e_hi": ["log2_e_hi"], "log2_e_lo": ["log2_e_lo"],
    "ln_2_hi": ["ln_2_hi"], "ln_2_lo": ["ln_2_lo"],
    "inv_sqrt2_hi": ["inv_sqrt2_hi"], "inv_sqrt2_lo": ["inv_sqrt2_lo"],
    "pi_quarter_hi": ["pi_quarter_hi"], "pi_quarter_lo": ["pi_quarter_lo"],
    "ln2_cw": ["ln2_cw1", "ln2_cw2", "ln2_cw3"],
    "pi_half_cw": ["pi_half_cw1", "pi_half_cw2", "pi_half_cw3"],
    "exp_max": ["exp_max"], "exp_min": ["exp_min"],
    "exp2_max": ["exp2_max"], "exp2_min": ["exp2_min"],
    "log10_2_hi": ["log10_2_hi"], "log10_2_lo": ["log10_2_lo"],
}


def hexf(x: float) -> str:
    if x == 0.0:
        return "-0x0.0p+0" if str(x).startswith("-") else "0x0.0p+0"
    return x.hex()


def emit(t: dict[str, list[float]]) -> str:
    lines = [
        "/* Generated by gen_dd_tables.py -- do not edit.",
        " *",
        " * Double-double constant tables of the exp / log / sin / cos kernels, each",
        " * derived from its closed form (see the generator's docstring) and split as",
        " * hi = RN(v), lo = RN(v - hi).  Bit-identical to the tables of multifloats",
        " * 0.10.3 (src/dd_constants.hh), which the kernels must reproduce exactly.",
        " *",
        " * The includer defines MF_TABLE (storage qualifier for tables read with a",
        " * warp-uniform index) and MF_GTABLE (tables read with a per-thread index).",
        " */",
        "#pragma once",
        "#ifndef MF_TABLE",
        "#define MF_TABLE static const",
        "#endif",
        "#ifndef MF_GTABLE",
        "#define MF_GTABLE static const",
        "#endif",
        "",
    ]
    gathered = {"exp2_table_hi", "exp2_table_lo", "log2_values_hi", "log2_values_lo", "log2_centers"}
    for name, vals in t.items():
        qual = "MF_GTABLE" if name in gathered else "MF_TABLE"
        body = ", ".join(hexf(v) for v in vals)
        lines.append(f"{qual} double mf_{name}[{len(vals)}] = {{{body}}};")
    lines.append("")
    return "\n".join(lines)


def parse_ref(path: str) -> dict[str, list[float]]:
    src = open(path).read()
    out: dict[str, list[float]] = {}
    for m in re.finditer(r"inline constexpr double (\w+)(\[\d+\])?\s*=\s*(\{[^}]*\}|[^;]*);", src):
        name, body = m.group(1), m.group(3)
        nums = re.findall(r"-?0x[0-9a-fA-F.]+p[+-]?\d+", body)
        out[name] = [float.fromhex(s) for s in nums]
    return out


def check(t: dict[str, list[float]], ref_header: str) -> int:
    ref = parse_ref(ref_header)
    bad = 0
    checked = 0
    for name, vals in t.items():
        ref_names = REF_NAMES.get(name, [name])
        if len(ref_names) == 1:
            rv = ref[ref_names[0]][: len(vals)]
        else:
            rv = [ref[n][0] for n in ref_names]
        for i, (a, b) in enumerate(zip(vals, rv)):
            checked += 1
            if struct.pack("<d", a) != struct.pack("<d", b):
                bad += 1
                print(f"MISMATCH {name}[{i}]: generated {a.hex()} reference {b.hex()}")
        if len(rv) != len(vals):
            bad += 1
            print(f"LENGTH {name}: generated {len(vals)} reference {len(rv)}")
    print(f"checked {checked} values against {ref_header}: {bad} mismatches")
    return 1 if bad else 0


def main(argv: list[str]) -> int:
    t = build()
    if len(argv) >= 2 and argv[0] == "--check":
        return check(t, argv[1])
    with open(OUT, "w") as f:
        f.write(emit(t))
    print(f"wrote {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
