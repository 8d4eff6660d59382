"""Fit and check the exponential used for resampling weights (pf_expneg in
pf_device.cuh, restated as orc_expneg in the oracle).

The resampling turns max-subtracted FP32 log-weights x <= 0 into linear
weights exp(x).  To make the engine's resampling bit-identical to the oracle's
given identical log-weights, both evaluate exp with the same sequence of
correctly rounded IEEE FP32 operations (no hardware approximation, no
library call):

    n = rint(x * log2(e));  r = x - n ln2 (two fmaf, Cody-Waite split of ln2)
    exp(x) = 2^n * P(r),    P(r) = 1 + r (c1 + r (c2 + ... + r c6))

P is fitted here: a least-squares fit of the relative error on Chebyshev
nodes of [-ln2/2, ln2/2] (slightly widened), refined by Lawson iterations
towards the minimax fit.  The script prints the fitted coefficients beside
the compiled ones and checks the compiled function, emulated with numpy FP32
operations (fmaf as one rounding of the exact FP64 product-sum), against exp
in FP64 on [-87, 0] (below -87 the function returns 0).

Usage: python esthera_b200/csrc/fit_exp.py; exits non-zero when the stated
error bound (2 ulp) is exceeded.
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ULP_BOUND = 2.0
LOG2E = np.float32(1.44269504088896341)
LN2_HI = np.float32(0.693145751953125)        # 0x3f317200: ln 2 with its low 12 bits cleared
LN2_LO = np.float32(0.693147180559945309 - 0.693145751953125)


def fit(nodes=2000, iters=80, degree=6):
    h = 0.5 * np.log(2.0) * 1.02
    k = np.arange(nodes)
    r = h * np.cos(np.pi * (k + 0.5) / nodes)
    y = np.exp(r)
    V = np.stack([r ** j for j in range(1, degree + 1)], axis=1)  # P(r) - 1 = sum c_j r^j
    t = y - 1.0
    w = 1.0 / y  # relative error weights
    c = np.linalg.lstsq(V * w[:, None], t * w, rcond=None)[0]
    lw = np.ones(nodes)
    for _ in range(iters):
        err = np.abs((V @ c - t) / y)
        lw = lw * err
        lw = lw / lw.sum()
        sw = np.sqrt(lw) * w
        c = np.linalg.lstsq(V * sw[:, None], t * sw, rcond=None)[0]
    return c, float(np.max(np.abs((V @ c - t) / y)))


def committed():
    """c1..c6 of pf_expneg, from pf_device.cuh."""
    src = (HERE / "pf_device.cuh").read_text()
    body = src[src.index("float pf_expneg(float x)"):]
    body = body[:body.index("return")]
    first = float(re.search(r"float p = ([-+0-9.eE]+)f;", body).group(1))
    rest = [float(v) for v in re.findall(r"p = fmaf\(p, r, ([-+0-9.eE]+)f\);", body)]
    return np.array([first] + rest[:5], np.float32)  # c6 .. c1 (the last fmaf adds the constant 1)


def fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def expneg32(x, coef_hi_first):
    """The compiled sequence of pf_expneg, operation by operation in FP32."""
    x = np.asarray(x, np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        return _expneg32(x, coef_hi_first)


def _expneg32(x, coef_hi_first):
    n = np.rint((x * LOG2E).astype(np.float32)).astype(np.float32)
    r = fma32(n, -LN2_HI * np.ones_like(n), x)
    r = fma32(n, -LN2_LO * np.ones_like(n), r)
    p = np.full_like(r, coef_hi_first[0])
    for cc in coef_hi_first[1:]:
        p = fma32(p, r, np.full_like(r, cc))
    p = fma32(p, r, np.ones_like(r))
    ni = n.astype(np.int64)
    ok = (x >= np.float32(-87.0)) & (ni >= -126)
    scale = np.where(ok, ((np.where(ok, ni, 0) + 127) << 23), 0).astype(np.uint32).view(np.float32)
    out = np.where(ok, (p * scale).astype(np.float32), np.float32(0))
    return np.where(np.isnan(x), x, out).astype(np.float32)


def main(argv=None):
    c, e = fit()
    cur = committed()
    print("fitted c1..c6 vs committed:")
    for f, g in zip(c, cur[::-1]):
        print("  % .9e   % .9e   diff % .1e" % (f, g, f - g))
    print("fitted polynomial max relative error (FP64 evaluation): %.3e" % e)
    x = np.concatenate([-np.linspace(0, 87, 1 << 22).astype(np.float32), np.float32([0, -1e-30, -0.5, -87])])
    got = expneg32(x, cur).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    ulp = np.spacing(ref.astype(np.float32)).astype(np.float64)
    err = np.abs(got - ref) / ulp
    print("pf_expneg on [-87, 0]: max error %.2f ulp (bound %.1f), mean %.3f ulp" % (err.max(), ULP_BOUND, err.mean()))
    beyond = expneg32(np.float32([-88.0, -100.0, -np.inf]), cur)
    print("below -87 and -inf ->", beyond)
    ok = err.max() <= ULP_BOUND and np.all(beyond == 0) and np.isnan(expneg32(np.float32([np.nan]), cur)[0])
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
