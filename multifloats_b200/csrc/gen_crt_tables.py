#!/usr/bin/env python3
"""Generate ``crt_tables.h``: the moduli of the CRT (modular) split form.

The moduli are the pairwise-coprime integers m <= 256 taken greedily from 256
down (256, 255, 253, 251, 247, 241, ...): every residue fits a signed byte in
[0, m) as an unsigned byte, so each modulus costs one u8 x u8 -> s32 product
on the tensor cores.  Per modulus the header
holds:

* ``crt_mod[t]``       m_t
* ``crt_lg[t]``        floor(log2(m_0 ... m_{t-1})) (exact: the product's bit
                       length minus one), ``crt_lg[0] = 0``; the plan takes the
                       smallest count N with crt_lg[N] >= the bits it needs
                       (``crt_lg_host``: the same numbers for host code)
* ``crt_digw[t][w]``   the signed bytes c_q = symmetric residue of 256^q mod m_t
                       for q = 4w .. 4w+3 (q < 14; zero above), packed as the
                       four bytes of a word, so that for a balanced base-256
                       representation X = sum_q d_q 256^q (signed byte digits)
                       the dot product sum_q d_q c_q (four dp4a) is congruent
                       to X modulo m_t
* ``crt_mu[t]``        ceil(2^32 / m_t): Barrett reduction of a non-negative
                       u < 2^30 (the quotient umulhi(u, mu) is exact or one
                       too large; one correction)
* ``crt_off18[t]``     a multiple of m_t of at least 2^18, added to a signed
                       value below that bound first

and, per moduli count N (index N - 1), the reconstruction constants of the
set m_0 .. m_{N-1} with M = m_0 ... m_{N-1} (global-memory tables,
``MF_GTABLE``):

* ``crt_M_n[N-1][l]``      M mod 2^256 in 32-bit limbs, least significant first
* ``crt_e_n[N-1][t][l]``   e_t = (M / m_t) ((M / m_t)^-1 mod m_t) mod 2^256
* ``crt_c_n[N-1][t]``      round(((M / m_t)^-1 mod m_t) 2^24 / m_t), the 24-bit
                           fixed point of c_t = e_t / M

Usage::

    python gen_crt_tables.py     # (re)write crt_tables.h next to this file
"""
from __future__ import annotations

import os
import sys
from math import gcd

NMAX = 36   # 266 bits: enough for 2W + log2(k) + 3 with W <= 110, k < 2^31
DIGITS = 14


def moduli(n: int) -> list[int]:
    out: list[int] = []
    m = 256
    while len(out) < n:
        if all(gcd(m, x) == 1 for x in out):
            out.append(m)
        m -= 1
    return out


def sym(v: int, m: int) -> int:
    """Symmetric representative of v mod m in [-floor(m/2), ceil(m/2) - 1]."""
    r = v % m
    return r - m if r >= (m + 1) // 2 else r


def main() -> int:
    ms = moduli(NMAX)
    prod, lg = 1, [0]
    for m in ms:
        prod *= m
        lg.append(prod.bit_length() - 1)
    lines = [
        "// Generated by gen_crt_tables.py -- do not edit.",
        "// Moduli of the CRT split form and their per-modulus constants.",
        "#pragma once",
        "#include <stdint.h>",
        "#ifndef MF_TABLE",
        "#define MF_TABLE static const",
        "#endif",
        f"#define CRT_NMAX {NMAX}",
        f"MF_TABLE uint32_t crt_mod[{NMAX}] = {{" + ", ".join(str(m) for m in ms) + "};",
        f"MF_TABLE int crt_lg[{NMAX + 1}] = {{" + ", ".join(str(v) for v in lg) + "};",
        "#ifdef __cplusplus",
        "// host copy of crt_lg (workspace sizing)",
        f"static constexpr int crt_lg_host[{NMAX + 1}] = {{" + ", ".join(str(v) for v in lg) + "};",
        "#endif",
    ]
    words = []
    for m in ms:
        cs = [sym(pow(256, q, m), m) if q < DIGITS else 0 for q in range(16)]
        w = []
        for k in range(4):
            v = 0
            for b in range(4):
                v |= (cs[4 * k + b] & 0xFF) << (8 * b)
            w.append(f"0x{v:08x}u")
        words.append("{" + ", ".join(w) + "}")
    lines.append(f"MF_TABLE uint32_t crt_digw[{NMAX}][4] = {{" + ",\n    ".join(words) + "};")
    # Barrett reduction of u < 2^30: q = umulhi(u, mu) is floor(u / m) or one more
    lines.append(f"MF_TABLE uint32_t crt_mu[{NMAX}] = {{" + ", ".join(f"{-(-(1 << 32) // m)}u" for m in ms) +
                 "};  // ceil(2^32 / m)")
    # offsets making a signed value non-negative before the reduction
    lines.append(f"MF_TABLE uint32_t crt_off18[{NMAX}] = {{" + ", ".join(f"{m * -(-(1 << 18) // m)}u" for m in ms) +
                 "};  // m ceil(2^18 / m): |v| < 2^18")
    # reconstruction constants per moduli count
    lines += ["#ifndef MF_GTABLE", "#define MF_GTABLE static const", "#endif"]
    mw, ew, cw = [], [], []
    for n in range(1, NMAX + 1):
        sub = ms[:n]
        M = 1
        for m in sub:
            M *= m
        mw.append("{" + ", ".join(f"0x{(M >> (32 * l)) & 0xFFFFFFFF:08x}u" for l in range(8)) + "}")
        rows, cs = [], []
        for t in range(NMAX):
            if t < n:
                q = M // sub[t]
                inv = pow(q % sub[t], -1, sub[t]) if sub[t] > 1 else 0
                e = (q * inv) % (1 << 256)
                c = ((inv << 24) + sub[t] // 2) // sub[t]
            else:
                e, c = 0, 0
            rows.append("{" + ", ".join(f"0x{(e >> (32 * l)) & 0xFFFFFFFF:08x}u" for l in range(8)) + "}")
            cs.append(f"{c}u")
        ew.append("{" + ",\n     ".join(rows) + "}")
        cw.append("{" + ", ".join(cs) + "}")
    lines.append(f"MF_GTABLE uint32_t crt_M_n[{NMAX}][8] = {{" + ",\n    ".join(mw) + "};")
    lines.append(f"MF_GTABLE uint32_t crt_e_n[{NMAX}][{NMAX}][8] = {{" + ",\n    ".join(ew) + "};")
    lines.append(f"MF_GTABLE uint32_t crt_c_n[{NMAX}][{NMAX}] = {{" + ",\n    ".join(cw) + "};")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "crt_tables.h")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
