"""Fit and check the atan polynomial of pf_atan2 (pf_device.cuh).

atan(a) on [0, 1] is approximated by a * P(a^2) with P of degree 7 (8
coefficients): a least-squares fit on Chebyshev nodes of a, refined by Lawson
iterations (each pass reweights the nodes by their current absolute error,
which drives the weighted least-squares fit towards the minimax one).  The
script prints the fitted coefficients next to the ones compiled into
pf_device.cuh, then checks the committed coefficients:

  * the polynomial alone, evaluated in FP32 Horner form (fmaf), against atan
    in FP64 on 2^20 points of [0, 1];
  * the whole pf_atan2 (octant reduction as the device code does it, with an
    FP32 division standing in for __fdividef) against numpy's FP64 arctan2 and
    its FP32 arctan2 (the host's atan2f) on 2^20 directions and on the
    octant boundaries.

Usage: python esthera_b200/csrc/fit_atan2.py [--nodes 4000] [--iters 60]
Exits non-zero when an error bound stated in pf_device.cuh is exceeded.
"""
import argparse
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
POLY_BOUND = 1.5e-7   # the polynomial on [0, 1], FP32 Horner
ATAN2_BOUND = 3.5e-7  # the whole pf_atan2, radians


def fit(nodes, iters, degree=7):
    k = np.arange(nodes)
    a = 0.5 + 0.5 * np.cos(np.pi * (k + 0.5) / nodes)  # Chebyshev nodes on [0, 1]
    s = a * a
    V = np.stack([a * s**j for j in range(degree + 1)], axis=1)  # columns a s^j
    y = np.arctan(a)
    w = np.ones(nodes)
    c = np.linalg.lstsq(V, y, rcond=None)[0]
    for _ in range(iters):
        err = np.abs(V @ c - y)
        w = w * err
        w = w / w.sum()
        sw = np.sqrt(w)
        c = np.linalg.lstsq(V * sw[:, None], y * sw, rcond=None)[0]
    return c, np.max(np.abs(V @ c - y))


def committed():
    """The 8 coefficients of pf_atan2, highest power first, from pf_device.cuh."""
    src = (HERE / "pf_device.cuh").read_text()
    body = src[src.index("pf_atan2(float y, float x)"):]
    body = body[:body.index("float r = a * p;")]
    first = float(re.search(r"float p = ([-+0-9.eE]+)f;", body).group(1))
    rest = [float(v) for v in re.findall(r"fmaf\(p, s, ([-+0-9.eE]+)f\)", body)]
    return np.array([first] + rest, np.float32)


def horner32(coef_hi_first, a):
    a = a.astype(np.float32)
    s = (a * a).astype(np.float32)
    p = np.full_like(a, coef_hi_first[0])
    for c in coef_hi_first[1:]:
        # fmaf: one rounding of p*s + c
        p = (p.astype(np.float64) * s.astype(np.float64) + np.float64(c)).astype(np.float32)
    return (a * p).astype(np.float32)


def atan2_device(y, x, coef):
    y = y.astype(np.float32)
    x = x.astype(np.float32)
    ax, ay = np.abs(x), np.abs(y)
    mx, mn = np.maximum(ax, ay), np.minimum(ax, ay)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.where(mx > 0, (mn / mx).astype(np.float32), np.float32(0))
    r = horner32(coef, a)
    r = np.where(ay > ax, (np.float32(1.57079632679489662) - r).astype(np.float32), r)
    r = np.where(x < 0, (np.float32(np.pi) - r).astype(np.float32), r)
    return np.copysign(r, y).astype(np.float32)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nodes", type=int, default=4000)
    ap.add_argument("--iters", type=int, default=60)
    a = ap.parse_args(argv)
    c, e = fit(a.nodes, a.iters)
    cur = committed()
    print("fitted (FP64, highest power first) vs committed:")
    for f, g in zip(c[::-1], cur):
        print("  % .9e   % .9e   diff % .1e" % (f, g, f - g))
    print("fitted polynomial max abs error (FP64 evaluation): %.3e" % e)

    ok = True
    t = np.linspace(0.0, 1.0, 1 << 20)
    pe = np.max(np.abs(horner32(cur, t).astype(np.float64) - np.arctan(t.astype(np.float32).astype(np.float64))))
    print("committed polynomial, FP32 Horner, max abs error on [0, 1]: %.3e (bound %.1e)" % (pe, POLY_BOUND))
    ok &= pe <= POLY_BOUND

    rng = np.random.default_rng(1)
    th = rng.uniform(-np.pi, np.pi, 1 << 20)
    rad = np.exp(rng.uniform(-20, 20, 1 << 20))
    y, x = (rad * np.sin(th)).astype(np.float32), (rad * np.cos(th)).astype(np.float32)
    edge = np.array([0, 1, -1, 1, -1, 0, 0, 1e-30, -1e-30], np.float32)
    edx = np.array([1, 1, 1, -1, -1, -1, 1e-30, 0, -1], np.float32)
    y, x = np.concatenate([y, edge]), np.concatenate([x, edx])
    d = atan2_device(y, x, cur).astype(np.float64)
    ref64 = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    ref32 = np.arctan2(y, x).astype(np.float64)
    err = np.abs(np.angle(np.exp(1j * (d - ref64))))
    print("pf_atan2 vs FP64 atan2: max %.3e rad (bound %.1e); host atan2f vs FP64: max %.3e"
          % (err.max(), ATAN2_BOUND, np.abs(np.angle(np.exp(1j * (ref32 - ref64)))).max()))
    ok &= err.max() <= ATAN2_BOUND
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
