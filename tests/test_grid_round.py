"""The split forms' rounding to the W-bit grid, on the CPU.

multifloats_b200/csrc/grid_round.cuh is compiled for the host (it is plain
C++ apart from the CUDA qualifiers) and its words Y = X + sum_q 128 * 256^q
are compared with the oracle's restatement (split_round in
oracle/mf_oracle.c, 128-bit integers) over random entries of every exponent
spread, every grid width W, ties, clamps, zeros, subnormal low limbs and
spreads that need ldexp.  The rounding error |X - (hi + lo) 2^(W - sigma)|
is checked against 1 with exact rational arithmetic."""
import ctypes as C
import os
import subprocess
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

HEADER_DIR = os.path.join(ROOT, "multifloats_b200", "csrc")

_HARNESS = r"""
#define __host__
#define __device__
#define __forceinline__ inline
#include "grid_round.cuh"
extern "C" void grid_words(double hi, double lo, int sigma, int W, unsigned *y) {
  using namespace mfcuda::split;
  const GridLimits g = grid_limits(W);
  int64_t T;
  uint64_t R;
  grid_round(hi, lo, sigma, g, W, T, R);
  uint32_t w[4];
  grid_biased_words(T, R, w);
  for (int i = 0; i < 4; ++i) y[i] = w[i];
}
"""


@pytest.fixture(scope="module")
def host_grid(tmp_path_factory):
    d = tmp_path_factory.mktemp("grid")
    src, so = d / "h.cc", d / "h.so"
    src.write_text(_HARNESS)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I", HEADER_DIR,
                    "-o", str(so), str(src)], check=True)
    L = C.CDLL(str(so))
    L.grid_words.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_uint32)]
    return L


def _oracle_x(hi, lo, sigma, W):
    out = (C.c_int64 * 2)()
    O.orc().orc_grid_round(hi, lo, sigma, W, out)
    return (out[1] << 64) | (out[0] & (2 ** 64 - 1))


def _words_x(L, hi, lo, sigma, W):
    y = (C.c_uint32 * 4)()
    L.grid_words(hi, lo, sigma, W, y)
    Y = y[0] | (y[1] << 32) | (y[2] << 64) | (y[3] << 96)
    bias = sum(128 << (8 * q) for q in range(14))
    return Y - bias


def _cases():
    rng = np.random.default_rng(7)
    out = []
    for W in (8, 14, 22, 46, 55, 56, 57, 62, 63, 64, 65, 86, 92, 110):
        for _ in range(300):
            sigma = int(rng.integers(-1070, 1020))
            spread = int(rng.integers(0, 130))
            e = sigma - 1 - spread
            hi = float(np.ldexp(rng.uniform(1.0, 2.0), e)) * (1 if rng.random() < 0.5 else -1)
            if not np.isfinite(hi) or hi == 0.0:
                continue
            ulp = np.spacing(abs(hi))
            lo = float(ulp * rng.uniform(-0.5, 0.5))
            s = hi + lo
            lo = (hi - s) + lo
            out.append((s, lo, sigma, W))
        # ties, values next to the clamp, exact integers, zero and subnormal limbs
        sigma = 3
        t = W - sigma
        for k in (0.5, 1.5, 2.5, -0.5, -2.5, 7.5):
            out.append((float(np.ldexp(k, -t)), 0.0, sigma, W))
            out.append((float(np.ldexp(k, -t)), float(np.ldexp(1.0, -t - 60)), sigma, W))
            out.append((float(np.ldexp(k, -t)), -float(np.ldexp(1.0, -t - 60)), sigma, W))
        top = float(np.ldexp(1.0, sigma)) * (1 - 2.0 ** -53)
        out += [(top, 0.0, sigma, W), (-top, 0.0, sigma, W), (top, np.spacing(top) / 2, sigma, W),
                (0.0, 0.0, sigma, W), (float(np.ldexp(1.0, -1074)), 0.0, 1030 - 1074 + W, W),
                (1.0, 5e-324, 1, W), (-1.0, -5e-324, 1, W)]
    return out


def test_host_compiled_rounding_matches_oracle(host_grid):
    bad = []
    for hi, lo, sigma, W in _cases():
        a = _words_x(host_grid, hi, lo, sigma, W)
        b = _oracle_x(hi, lo, sigma, W)
        if a != b:
            bad.append((hi, lo, sigma, W, a, b))
    assert not bad, bad[:5]


def test_rounding_error_at_most_one_unit():
    for hi, lo, sigma, W in _cases():
        X = _oracle_x(hi, lo, sigma, W)
        exact = (Fraction(hi) + Fraction(lo)) * Fraction(2) ** (W - sigma)
        assert abs(X) <= 2 ** W - 1
        assert abs(Fraction(X) - exact) <= 1, (hi, lo, sigma, W, X, float(exact))
        if abs(exact) < 2 ** W - 1:
            assert abs(Fraction(X) - exact) <= Fraction(1, 2) + Fraction(1, 2 ** 52)
