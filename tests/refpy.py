"""Pure-Python restatements of the reference's sub-filter algorithms for SMALL
cases, written straight from the reference loops (independent of the C
oracle), used to cross-check the oracle.  float32 arithmetic is done with
numpy.float32 scalars so every operation rounds like the device code.
"""
import numpy as np

f32 = np.float32


def bitonic_desc(keys, idx=None):
    """bitonic_sort(dir=0) of bitonic-sort.cu:28-61, one comparator per 'thread'."""
    w = [f32(k) for k in keys]
    ix = list(range(len(w))) if idx is None else list(idx)
    n = len(w)
    dirv = 0

    def comparator(a, b, d):
        if int(w[a] > w[b]) == d:
            w[a], w[b] = w[b], w[a]
            ix[a], ix[b] = ix[b], ix[a]

    size = 2
    while size < n:
        stride = size // 2
        while stride > 0:
            for tid in range(n // 2):
                ddd = dirv ^ int((tid & (size // 2)) != 0)
                pos = 2 * tid - (tid & (stride - 1))
                comparator(pos, pos + stride, ddd)
            stride //= 2
        size <<= 1
    stride = n // 2
    while stride > 0:
        for tid in range(n // 2):
            pos = 2 * tid - (tid & (stride - 1))
            comparator(pos, pos + stride, dirv)
        stride //= 2
    return np.array(w, np.float32), np.array(ix, np.int32)


def blelloch(w):
    """prefix_sum of pf_generic_soa.cu:169-216 -> (exclusive scan, total)."""
    e = [f32(x) for x in w]
    n = len(e)
    offset = 1
    d = n // 2
    while d > 0:
        for tid in range(d):
            ai, bi = offset * (2 * tid + 1) - 1, offset * (2 * tid + 2) - 1
            e[bi] = f32(e[bi] + e[ai])
        offset *= 2
        d //= 2
    cum = e[n - 1]
    e[n - 1] = f32(0)
    d = 1
    while d < n:
        offset //= 2
        for tid in range(d):
            ai, bi = offset * (2 * tid + 1) - 1, offset * (2 * tid + 2) - 1
            t = e[ai]
            e[ai] = e[bi]
            e[bi] = f32(e[bi] + t)
        d *= 2
    return np.array(e, np.float32), cum


def binary_search(hay, needle):
    lo, hi = 0, len(hay) - 1
    while True:
        cur = lo + (hi - lo + 1) // 2
        if hay[cur] > needle:
            hi = cur - 1
        else:
            lo = cur
        if not lo < hi:
            return lo


def resample_ref(w, u):
    ex, tot = blelloch(w)
    return np.array([binary_search(ex, f32(f32(ui - f32(1)) * tot)) for ui in u], np.int32)


def scan_f64(w, ept):
    """The canonical FP64 scan: sequential per group of ept, Kogge-Stone over
    32-lane warps, Kogge-Stone over warp totals."""
    m = len(w)
    nt = m // ept
    tt = []
    for j in range(nt):
        s = float(w[j * ept])
        for e in range(1, ept):
            s = s + float(w[j * ept + e])
        tt.append(s)
    inc = list(tt)
    d = 1
    while d < 32:
        inc = [inc[j] + inc[j - d] if (j & 31) >= d else inc[j] for j in range(nt)]
        d *= 2
    ex = [0.0 if (j & 31) == 0 else inc[j - 1] for j in range(nt)]
    nw = (nt + 31) // 32
    wt = [inc[min(w2 * 32 + 31, nt - 1)] for w2 in range(nw)]
    d = 1
    while d < 32:
        wt = [wt[k] + wt[k - d] if k >= d else wt[k] for k in range(nw)]
        d *= 2
    cum = []
    for j in range(nt):
        base = (0.0 if (j >> 5) == 0 else wt[(j >> 5) - 1]) + ex[j]
        c = base + float(w[j * ept])
        cum.append(c)
        for e in range(1, ept):
            c = c + float(w[j * ept + e])
            cum.append(c)
    return cum


def resample_systematic(w, u0, ept):
    cum = scan_f64(w, ept)
    m = len(w)
    step = cum[-1] / m
    out = []
    for i in range(m):
        p = (float(f32(u0)) + i) * step
        c = sum(1 for x in cum if x <= p)
        out.append(min(c, m - 1))
    return np.array(out, np.int32)


def sum_reduce4(arr):
    a = [f32(x) for x in arr]
    off = len(a)
    while off > 2:
        off >>= 2
        for l in range(off):
            x = f32(f32(a[l + off] + a[l + 2 * off]) + a[l + 3 * off])
            a[l] = f32(a[l] + x)
    if off > 1:
        a[0] = f32(a[0] + a[1])
    return a[0]


def vose_build(w):
    """resampling_valias normalisation + vose_alias_init with the atomics
    executed in ascending work-item order."""
    m = len(w)
    s = sum_reduce4(w)
    prob, alias = [], list(range(m))
    for x in w:
        p = f32(x) / s if s > f32(0) else f32(1) / f32(m)
        prob.append(f32(f32(p) * f32(m)))
    sl = [0] * m
    small_end, large_rend = 0, m - 1
    for i in range(m):
        if prob[i] <= f32(1):
            sl[small_end] = i
            small_end += 1
        else:
            sl[large_rend] = i
            large_rend -= 1
    small_begin = 0
    while True:
        se = small_end
        nactive = min(se - small_begin, m - se)
        if nactive <= 0:
            break
        large_rend += nactive
        items = []
        for k in range(nactive):
            si, li = sl[small_begin + k], sl[se + k]
            ps, pl = prob[si], prob[li]
            alias[si] = li
            items.append((li, ps, pl))
        for li, ps, pl in items:
            nl = f32(f32(pl + ps) - f32(1))
            if nl <= f32(1):
                old = small_end
                small_end += 1
            else:
                old = large_rend
                large_rend -= 1
            sl[old] = li
            prob[li] = nl
        small_begin += nactive
    return np.array(prob, np.float32), np.array(alias, np.uint32)


def vose_draw(prob, alias, ux, uy):
    m = len(prob)
    col = min(int(np.floor(f32(ux) * f32(m))), m - 1)
    return col if f32(uy) < prob[col] else int(alias[col])


def torus_dims(N):
    dx = 1
    while (2 * dx) * (2 * dx) <= N:
        dx *= 2
    return dx, N // dx


def exchange_sources(mode, N, m, t, keys=None):
    src = np.arange(N * m, dtype=np.int32)
    if mode == 1:
        for b in range(N):
            for j in range(t):
                src[b * m + m - 1 - j] = ((b - 1) % N) * m + j
    elif mode == 2:
        dx, dy = torus_dims(N)
        for b in range(N):
            x, y = b % dx, b // dx
            fr = [y * dx + (x + 1) % dx, y * dx + (x - 1) % dx, ((y + 1) % dy) * dx + x, ((y - 1) % dy) * dx + x]
            for k in range(4):
                for j in range(t):
                    src[b * m + m - 1 - j - k * t] = fr[k] * m + j
    elif mode == 3:
        cands = [(-float(keys[b * m + j]), b * t + j, b * m + j) for b in range(N) for j in range(t)]
        cands.sort()
        for b in range(N):
            for j in range(t):
                src[b * m + m - 1 - j] = cands[j][2]
    return src
