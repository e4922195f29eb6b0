"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no public dataset is involved).

All generators return float64 numpy arrays with interleaved limbs (hi, lo) and
normalised double-doubles: lo = hi * 2^-53 * U[-1, 1), then (hi, lo) passed
through two_sum so |lo| <= ulp(hi)/2.  Matrices are column-major flat buffers.

  dd_uniform          hi ~ U[-1, 1)                               (GEMM 256^3 / 4096^3, reductions)
  dd_exp_inputs       hi ~ U[-700, 700]                           (exp)
  dd_pow2_inputs      hi = 2^U[-1000, 1000]                       (log, sqrt)
  dd_trig_inputs      hi ~ U[-1e6, 1e6], 10% within 1e-12 of k*pi/2 (sin, cos)
  dd_rowcol_scaled    hi = +-u 2^e, u ~ U[1,2), e ~ U{-R..R} per row of A /
                      column of B                                 (split-INT8 GEMM)
"""
from __future__ import annotations

import numpy as np


def _renorm(hi: np.ndarray, lo: np.ndarray) -> np.ndarray:
    s = hi + lo
    bb = s - hi
    err = (hi - (s - bb)) + (lo - bb)
    out = np.empty(hi.size * 2, dtype=np.float64)
    out[0::2] = s.reshape(-1)
    out[1::2] = err.reshape(-1)
    return out


def with_lo(hi: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    hi = np.asarray(hi, dtype=np.float64).reshape(-1)
    lo = hi * 2.0 ** -53 * rng.uniform(-1.0, 1.0, hi.size)
    return _renorm(hi, lo)


def dd_uniform(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return with_lo(rng.uniform(-1.0, 1.0, n), rng)


def dd_exp_inputs(n: int, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return with_lo(rng.uniform(-700.0, 700.0, n), rng)


def dd_pow2_inputs(n: int, seed: int = 2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return with_lo(np.exp2(rng.uniform(-1000.0, 1000.0, n)), rng)


def dd_trig_inputs(n: int, seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    hi = rng.uniform(-1e6, 1e6, n)
    near = rng.random(n) < 0.10
    kmax = int(1e6 / (np.pi / 2))
    k = rng.integers(-kmax, kmax + 1, n)
    hi = np.where(near, k * (np.pi / 2) + rng.uniform(-1e-12, 1e-12, n), hi)
    return with_lo(hi, rng)


def dd_rowcol_scaled(rows: int, cols: int, R: int, per: str, seed: int) -> np.ndarray:
    """Column-major rows x cols matrix; exponent constant per row ('row') or per column ('col')."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(1.0, 2.0, (cols, rows)) * rng.choice([-1.0, 1.0], (cols, rows))
    if per == "row":
        e = rng.integers(-R, R + 1, rows)[None, :]
    else:
        e = rng.integers(-R, R + 1, cols)[:, None]
    hi = np.ldexp(u, np.broadcast_to(e, u.shape))
    return with_lo(hi, rng)


def complex_from_parts(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    """Interleave two DD arrays into complex64x2 layout (re.hi, re.lo, im.hi, im.lo)."""
    out = np.empty(re.size * 2, dtype=np.float64)
    out.reshape(-1, 4)[:, 0:2] = re.reshape(-1, 2)
    out.reshape(-1, 4)[:, 2:4] = im.reshape(-1, 2)
    return out


ELEMENTWISE_INPUTS = {
    "exp": dd_exp_inputs,
    "log": dd_pow2_inputs,
    "sin": dd_trig_inputs,
    "cos": dd_trig_inputs,
    "sqrt": dd_pow2_inputs,
}


def dd_exp2_inputs(n: int, seed: int = 0) -> np.ndarray:
    """exp2 arguments across its whole range: hi ~ U[-1100, 1030] (past both
    clamps, exp_log.inc:119-128), lo as elsewhere."""
    return with_lo(np.random.default_rng(seed).uniform(-1100.0, 1030.0, n), np.random.default_rng(seed + 1))


# the adjacent elementwise functions (exp2 / log2 / log10), not in the benchmark configs
EXTRA_ELEMENTWISE_INPUTS = {"exp2": dd_exp2_inputs, "log2": dd_pow2_inputs, "log10": dd_pow2_inputs}


# ---- BLAS-style shims (wgemm / wtrsm) ------------------------------------------
def dd_padded(rows: int, cols: int, ld: int, seed: int, zeros: float = 0.0,
              pad: float = np.nan) -> np.ndarray:
    """Column-major rows x cols DD matrix (hi ~ U[-1, 1)) stored with leading
    dimension ld >= rows; the ld - rows padding rows of every column hold `pad`
    (NaN by default, so a kernel that reads or writes padding shows it).  A
    fraction `zeros` of the entries is exactly (0, 0)."""
    rng = np.random.default_rng(seed)
    v = with_lo(rng.uniform(-1.0, 1.0, rows * cols), rng).reshape(cols, rows, 2)
    if zeros > 0:
        v[rng.random((cols, rows)) < zeros] = 0.0
    out = np.full((max(cols, 1), max(ld, 1), 2), pad, dtype=np.float64)
    out[:cols, :rows] = v
    return out[: max(cols, 1)].reshape(-1).copy()


def dd_triangular(n: int, ld: int, seed: int, zeros: float = 0.0) -> np.ndarray:
    """n x n matrix for triangular solves: every entry filled (both triangles,
    so a solve that reads the wrong triangle shows), off-diagonal hi ~ U[-1, 1)/n,
    diagonal hi = +-U[1, 2) (diagonally dominant: no growth), padding NaN.  A
    fraction `zeros` of the off-diagonal entries is exactly (0, 0)."""
    a = dd_padded(n, n, ld, seed, zeros=zeros).reshape(max(n, 1), max(ld, 1), 2)
    if n > 0:
        a[:n, :n] /= float(n)
        rng = np.random.default_rng(seed + 7)
        d = rng.uniform(1.0, 2.0, n) * rng.choice([-1.0, 1.0], n)
        idx = np.arange(n)
        a[idx, idx] = with_lo(d, rng).reshape(n, 2)
    return a.reshape(-1).copy()
