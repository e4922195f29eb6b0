"""Error of EVERY output of a split-INT8 (digit-sliced or CRT) product,
measured on the device.

The split forms promise |C - AB|_ij <= target * k * 2^-104 * (|A||B|)_ij.  An
exact oracle of every output of a 4096^3 or 8192^3 product is out of reach of
the host, but the plain compensated kernel (mfcuda_matmuldd_mm, the
reference's matmul bit for bit) is itself within 1 * k * 2^-104 * (|A||B|)_ij
of the exact product, so

    r_ij = |C_split - C_plain|_ij / (k 2^-104 (|A||B|)_ij)

bounds the split form's true error to within one unit of that scale (true
error <= r_ij + 1) for every output.  (|A||B|) is formed by the plain kernel
on |A| and |B| (limb-wise absolute values) and only its leading limb is used.
Complex products are measured per part: the real part against
|Ar||Br| + |Ai||Bi|, the imaginary part against |Ar||Bi| + |Ai||Br| (the four
real products of the Fortran composition).

These are measurement helpers over CUDA tensors (torch is used only for the
elementwise differences and the max); every product runs through the
library's own kernels.
"""
from __future__ import annotations

from . import api

ULP = 2.0 ** -104


def dd_abs(x):
    """Limb-wise |x| of an interleaved real DD tensor: both limbs flipped where hi < 0."""
    import torch

    v = x.view(-1, 2)
    return (v * torch.where(v[:, :1] < 0, -1.0, 1.0)).reshape(-1)


def _parts(z):
    """Real and imaginary DD parts (contiguous) of an interleaved complex DD tensor."""
    v = z.view(-1, 4)
    return v[:, 0:2].contiguous().reshape(-1), v[:, 2:4].contiguous().reshape(-1)


def _ratio_stats(c, cp, ab_hi, k: int) -> dict:
    """Statistics of |c - cp| / (k 2^-104 ab) over all outputs (DD tensors c, cp
    of the same layout, ab_hi the leading limbs of (|A||B|))."""
    import torch

    cv, pv = c.view(-1, 2), cp.view(-1, 2)
    # the leading limbs agree to a few units in their last place wherever the
    # outputs are accurate, so their difference is exact (Sterbenz)
    diff = ((cv[:, 0] - pv[:, 0]) + (cv[:, 1] - pv[:, 1])).abs()
    denom = ab_hi * (float(k) * ULP)
    pos = denom > 0
    r = torch.where(pos, diff / torch.where(pos, denom, 1.0), torch.zeros_like(diff))
    nonzero_where_ab_zero = int(((~pos) & (diff != 0)).sum().item())
    finite = torch.isfinite(r)
    rf = r[finite]
    return {"max_err_vs_plain_k_ulp_absab": float(rf.max().item()) if rf.numel() else None,
            "mean_err_vs_plain_k_ulp_absab": float(rf.mean().item()) if rf.numel() else None,
            "max_err_vs_plain_ulp_absab": float(rf.max().item()) * k if rf.numel() else None,
            "outputs": int(r.numel()), "nonfinite_outputs": int((~finite).sum().item()),
            "nonzero_where_absab_zero": nonzero_where_ab_zero}


def full_error_real(a, b, c, m: int, k: int, n: int, renorm_interval: int = 8) -> dict:
    """Error of every output of a real split product C ~= A B (CUDA tensors,
    column-major DD) in units of k 2^-104 (|A||B|)_ij, against the plain
    compensated product.  The true error of each output is at most the
    reported value plus 1 in these units."""
    cp = api.matmuldd_mm(a, b, m, k, n, renorm_interval)
    ab = api.matmuldd_mm(dd_abs(a), dd_abs(b), m, k, n, renorm_interval)
    out = _ratio_stats(c, cp, ab.view(-1, 2)[:, 0], k)
    out["reference"] = "plain compensated product (mfcuda_matmuldd_mm, within 1 k-ulp of exact)"
    return out


def full_error_complex(a, b, c, m: int, k: int, n: int, renorm_interval: int = 8) -> dict:
    """As full_error_real for a complex product (complex64x2 tensors), per part."""
    cp = api.cmatmuldd_mm(a, b, m, k, n, renorm_interval)
    ar, ai = (dd_abs(p) for p in _parts(a))
    br, bi = (dd_abs(p) for p in _parts(b))

    def absprod(x, y):
        return api.matmuldd_mm(x, y, m, k, n, renorm_interval).view(-1, 2)[:, 0]

    ab_re = absprod(ar, br) + absprod(ai, bi)
    ab_im = absprod(ar, bi) + absprod(ai, br)
    cre, cim = _parts(c)
    pre, pim = _parts(cp)
    re = _ratio_stats(cre, pre, ab_re, k)
    im = _ratio_stats(cim, pim, ab_im, k)
    keys = ("max_err_vs_plain_k_ulp_absab", "max_err_vs_plain_ulp_absab")
    out = {kk: max(v for v in (re[kk], im[kk]) if v is not None) for kk in keys}
    out.update({"re": re, "im": im,
                "reference": "plain compensated complex product (mfcuda_cmatmuldd_mm), per part"})
    return out
