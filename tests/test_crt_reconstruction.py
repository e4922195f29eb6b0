"""The integer arithmetic of the tensor-core CRT reconstruction
(crt_device.cuh: crt_limbs_nl, used by crt_recon_body and
crt_combine_tc_body), restated in Python and checked against
exact integers on the CPU: for every plan width W and inner size k the kernel
can meet, and for any C' with |C'| < k 2^(2W),

* the column sums S_b = sum_t r_t E[t][b] of the u8 x u8 MMA fit in INT32;
* q = round((S_0 + S_1 2^8 + S_2 2^16) / 2^24) (24-bit fixed-point c_t) is
  the exact CRT quotient;
* the 30-bit partial limbs and the q M subtraction give C' modulo
  2^(8 nbe), and bit 8 nbe - 1 is its sign -- both as a plain int64-carry
  restatement and as the device's NL-limb form (re-cut high halves, q (-M)
  added modulo 2^(32 NL), sign fill);

using the moduli table the device reads (crt_tables.h) and the plan's own
moduli count and byte count."""
import os
import random
import re
from math import prod

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = os.path.join(HERE, "..", "multifloats_b200", "csrc", "crt_tables.h")


def _table(name):
    text = open(TABLES).read()
    body = re.search(name + r"\[\d+\] = \{([^}]*)\}", text).group(1)
    return [int(v.strip().rstrip("u")) for v in body.split(",")]


MODS = _table("crt_mod")
LG = _table("crt_lg")


def ceil_log2(k):
    b = 0
    while b < 63 and (1 << b) < k:
        b += 1
    return b


def plan(W, k):
    """(moduli, nbe, nb) as crt_moduli / crt_tc_bytes / crt_tc_cols."""
    need = 2 * W + ceil_log2(k) + 2
    n = 1
    while n < len(MODS) and LG[n] < need:
        n += 1
    nbe = 4 * ((need + 31) // 32)
    return n, nbe, (nbe + 4 + 15) // 16 * 16


def constants(n, nbe):
    ms = MODS[:n]
    M = prod(ms)
    e, cfix = [], []
    for m in ms:
        inv = pow((M // m) % m, -1, m)
        e.append((M // m) * inv)
        cfix.append(((inv << 24) + m // 2) // m)
    E = [[0] * 48 for _ in range(n)]  # E[t][b]
    for t in range(n):
        for b in range(3):
            E[t][b] = (cfix[t] >> (8 * b)) & 0xFF
        for b in range(4, 4 + nbe):
            E[t][b] = (e[t] >> (8 * (b - 4))) & 0xFF
    Mw = [(M >> (32 * w)) & 0xFFFFFFFF for w in range(8)]
    return ms, E, Mw


def column_sums(r, E, nb):
    S = [sum(rt * Et[b] for rt, Et in zip(r, E)) if b < nb else 0 for b in range(48)]
    assert max(S) < 2 ** 31  # INT32 accumulators of the MMA
    return S


def reconstruct(r, E, Mw, nbe, nb):
    S = column_sums(r, E, nb)
    Q = S[0] + (S[1] << 8) + (S[2] << 16)
    q = (Q + (1 << 23)) >> 24
    limb, carry = [], 0
    for w in range(8):
        lo = S[4 + 4 * w] + (S[5 + 4 * w] << 8)
        hi = S[6 + 4 * w] + (S[7 + 4 * w] << 8)
        assert lo < 2 ** 30 and hi < 2 ** 30  # the kernel's 32-bit partial sums
        v = lo + (hi << 16) - q * Mw[w] + carry
        assert -(2 ** 63) <= v < 2 ** 63  # int64
        limb.append(v & 0xFFFFFFFF)
        carry = v >> 32
    fill = 0xFFFFFFFF if limb[nbe // 4 - 1] >> 31 else 0
    limb = [limb[w] if 4 * w < nbe else fill for w in range(8)]
    val = sum(x << (32 * w) for w, x in enumerate(limb))
    return val - (1 << 256) if val >> 255 else val


def reconstruct_nl(r, E, Mw, nbe, nb):
    """The device's limb arithmetic (crt_limbs_nl): NL = max(5, nbe / 4) 32-bit
    limbs, the quotient in 32-bit steps, the high halves re-cut at limb
    boundaries, r = lo + H + q Mn modulo 2^(32 NL) with Mn = -M mod 2^(32 NL),
    and for NL = 5 with nbe < 20 the limbs above nbe bytes filled with the sign."""
    S = column_sums(r, E, nb)
    m32 = 0xFFFFFFFF
    NL = max(5, nbe // 4)
    assert max(S[:3]) < 2 ** 22
    q = ((((S[0] + (1 << 23)) & m32) >> 8) + S[1] + ((S[2] << 8) & m32)) & m32
    q >>= 16
    lo = [(S[4 + 4 * w] + (S[5 + 4 * w] << 8)) & m32 for w in range(NL)]
    hi = [(S[6 + 4 * w] + (S[7 + 4 * w] << 8)) & m32 for w in range(NL)]
    H = [(hi[0] << 16) & m32] + [((hi[w] << 16) | (hi[w - 1] >> 16)) & m32 for w in range(1, NL)]
    M = sum(x << (32 * w) for w, x in enumerate(Mw))
    mod = 1 << (32 * NL)
    Mn = (-M) % mod
    val = (sum(x << (32 * w) for w, x in enumerate(lo)) + sum(x << (32 * w) for w, x in enumerate(H)) +
           q * Mn) % mod
    limb = [(val >> (32 * w)) & m32 for w in range(NL)]
    if NL == 5 and nbe < 20:
        fill = m32 if limb[nbe // 4 - 1] >> 31 else 0
        limb = [limb[w] if 4 * w < nbe else fill for w in range(NL)]
    val = sum(x << (32 * w) for w, x in enumerate(limb))
    return val - mod if val >> (32 * NL - 1) else val


@pytest.mark.parametrize("W,k", [(8, 1), (40, 3), (77, 200), (92, 4096), (91, 8192), (99, 16), (110, 5),
                                 (110, 300000), (110, 2 ** 31 - 1)])
def test_reconstruction_is_exact(W, k):
    n, nbe, nb = plan(W, k)
    ms, E, Mw = constants(n, nbe)
    assert prod(ms) >= 4 * k * 2 ** (2 * W)  # the moduli bound the plan relies on
    lim = k * (2 ** W - 1) ** 2  # |C'| <= k (2^W - 1)^2
    rng = random.Random(W * 100003 + k)
    cases = [0, 1, -1, lim, -lim, lim - 1, -(lim - 1)] + [rng.randint(-lim, lim) for _ in range(300)]
    for c in cases:
        r = [c % m for m in ms]
        assert reconstruct(r, E, Mw, nbe, nb) == c, (W, k, c)
        assert reconstruct_nl(r, E, Mw, nbe, nb) == c, (W, k, c)
