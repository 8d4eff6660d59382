"""ctypes binding of the CPU oracle (oracle/_build/libpf_oracle.so) and of the
reference's own CPU MTGP32 generator (oracle/_ref/libmtgp_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm -- never by the product.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libpf_oracle.so"
REF_LIB = HERE / "_ref" / "libmtgp_ref.so"

RES_REF, RES_SYSTEMATIC, RES_VOSE = 0, 1, 2
RNG_REFLAYOUT, RNG_SUBFILTER = 0, 1
EXCH_NONE, EXCH_RING, EXCH_TORUS, EXCH_ALL2ALL = 0, 1, 2, 3
MODEL_UNICYCLE, MODEL_DHARM, MODEL_REFARM, MODEL_BEACON, MODEL_CAMARM = 0, 1, 2, 3, 4
MASK_PARAMS, MASK_CUDA_REF = 0, 0xFF800000


class OrcModel(C.Structure):
    _fields_ = [("model", C.c_int), ("num_state", C.c_int), ("num_noise", C.c_int),
                ("dt", C.c_double), ("sq", C.c_double * 3), ("sigma_r", C.c_double), ("sigma_b", C.c_double),
                ("num_landmarks", C.c_int), ("lm", (C.c_double * 2) * 8),
                ("sigma_qd", C.c_double), ("sigma_p", C.c_double), ("sigma_a", C.c_double),
                ("a", C.c_double * 6), ("alpha", C.c_double * 6), ("d", C.c_double * 6),
                ("bnoise", C.c_double * 3), ("num_beacons", C.c_int), ("bc", (C.c_double * 3) * 16),
                ("fc", C.c_double * 2), ("cc", C.c_double * 2), ("kc", C.c_double * 4)]


class OrcFilter(C.Structure):
    _fields_ = [("mdl", OrcModel), ("m", C.c_int), ("N", C.c_int), ("t", C.c_int), ("exchange", C.c_int),
                ("resampler", C.c_int), ("rng", C.c_int), ("G", C.c_int), ("ept", C.c_int),
                ("log_weights", C.c_int), ("freq", C.c_float), ("seed", C.c_uint32), ("mask", C.c_uint32),
                ("T", C.c_int64), ("state", C.POINTER(C.c_float)), ("tmp", C.POINTER(C.c_float)),
                ("tkey", C.POINTER(C.c_float)), ("mtgp", C.POINTER(C.c_uint32)), ("streams", C.c_int),
                ("rbuf", C.POINTER(C.c_float)), ("rtotal", C.c_int64), ("ess_frac", C.c_float),
                ("soff", C.c_int)]


class OrcEstimate(C.Structure):
    _fields_ = [("mean", C.c_double * 16), ("log_norm", C.c_double), ("best_key", C.c_float),
                ("best_sub", C.c_int32), ("best", C.c_float * 16)]


_lib = None
_ref = None


def build(arch="-march=x86-64-v2"):
    """Compile the oracle (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "ARCHFLAGS=%s" % arch], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        _declare(_lib)
    return _lib


def ref_lib():
    """The reference's own mtgp32-fast.c, or None when it was not built here."""
    global _ref
    if _ref is None and REF_LIB.exists():
        _ref = C.CDLL(str(REF_LIB))
        _ref.ref_mtgp_generate.argtypes = [C.c_int, C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_uint32)]
        _ref.ref_mtgp_init_state.argtypes = [C.c_int, C.c_uint32, C.POINTER(C.c_uint32)]
        _ref.ref_mtgp_mask.restype = C.c_uint32
    return _ref


def _declare(L):
    fp, ip, up, dp = (C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_uint32),
                      C.POINTER(C.c_double))
    sig = {
        "orc_mtgp_init_state": (None, [up, C.c_int, C.c_uint32]),
        "orc_mtgp_generate": (None, [up, C.c_int, C.c_uint32, C.c_int, C.c_int64, up]),
        "orc_mtgp_generate_blocks": (None, [up, C.c_int, C.c_uint32, C.c_int, C.c_int64, up]),
        "orc_boxmuller": (None, [fp, C.c_int64]),
        "orc_bitonic_sort_desc": (None, [fp, ip, C.c_int]),
        "orc_blelloch_scan": (C.c_float, [fp, C.c_int]),
        "orc_binary_search": (C.c_int, [fp, C.c_float, C.c_int]),
        "orc_resample_ref": (None, [fp, fp, C.c_int, ip]),
        "orc_scan_f64": (C.c_double, [fp, C.c_int, C.c_int, dp]),
        "orc_resample_systematic": (C.c_double, [fp, C.c_int, C.c_int, C.c_float, ip]),
        "orc_vose_build": (None, [fp, C.c_int, fp, up]),
        "orc_vose_scaled": (None, [fp, C.c_int, fp]),
        "orc_vose_draw": (C.c_uint32, [fp, up, C.c_int, C.c_float, C.c_float]),
        "orc_torus_dims": (None, [C.c_int, ip, ip]),
        "orc_exchange_sources": (None, [C.c_int, C.c_int, C.c_int, C.c_int, fp, ip]),
        "orc_model_step": (C.c_double, [C.POINTER(OrcModel), fp, fp, fp, fp]),
        "orc_filter_init": (C.c_int, [C.POINTER(OrcFilter), C.POINTER(OrcModel), C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                      C.c_uint32, C.c_uint32, fp]),
        "orc_filter_free": (None, [C.POINTER(OrcFilter)]),
        "orc_filter_set_stream_offset": (C.c_int, [C.POINTER(OrcFilter), C.c_int]),
        "orc_filter_step": (C.c_int, [C.POINTER(OrcFilter), fp, fp, C.POINTER(OrcEstimate), ip, C.c_int]),
        "orc_filter_sample": (C.c_int, [C.POINTER(OrcFilter), fp, fp, C.POINTER(OrcEstimate), C.c_int]),
        "orc_filter_resample": (C.c_int, [C.POINTER(OrcFilter), ip, C.c_int]),
        "orc_stream_draws": (C.c_int64, [C.c_int, C.c_int, C.c_int]),
        "orc_expneg": (C.c_float, [C.c_float]),
    }
    for n, (r, a) in sig.items():
        f = getattr(L, n)
        f.restype = r
        f.argtypes = a


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _u(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---- primitives ---------------------------------------------------------------
def mtgp_stream(set_, seed, n, kind=1, mask=MASK_PARAMS):
    st = np.zeros(351, np.uint32)
    lib().orc_mtgp_init_state(_u(st), set_, seed)
    out = np.zeros(n, np.uint32)
    lib().orc_mtgp_generate(_u(st), set_, mask, kind, n, _u(out))
    return out


def mtgp_blocks(G, seed, per_stream, kind=1, mask=MASK_PARAMS, calls=1):
    st = np.zeros(G * 351, np.uint32)
    for g in range(G):
        s = np.zeros(351, np.uint32)
        lib().orc_mtgp_init_state(_u(s), g, (seed + g + 1) & 0xFFFFFFFF)
        st[g * 351:(g + 1) * 351] = s
    outs = []
    for _ in range(calls):
        out = np.zeros(G * per_stream, np.uint32)
        lib().orc_mtgp_generate_blocks(_u(st), G, mask, kind, G * per_stream, _u(out))
        outs.append(out)
    return np.concatenate(outs)


def ref_mtgp_stream(set_, seed, n, kind=1):
    r = ref_lib()
    if r is None:
        return None
    out = np.zeros(n, np.uint32)
    if r.ref_mtgp_generate(set_, seed, kind, n, _u(out)) != 0:
        raise RuntimeError("reference generator failed")
    return out


def boxmuller(data, n=None):
    a = np.array(data, np.float32, copy=True)
    n = len(a) if n is None else n
    lib().orc_boxmuller(_f(a), n)
    return a


def bitonic_sort(keys, m):
    k = np.array(keys, np.float32, copy=True)
    idx = np.tile(np.arange(m, dtype=np.int32), len(k) // m)
    for b in range(len(k) // m):
        kk = k[b * m:(b + 1) * m].copy()
        ii = idx[b * m:(b + 1) * m].copy()
        lib().orc_bitonic_sort_desc(_f(kk), _i(ii), m)
        k[b * m:(b + 1) * m] = kk
        idx[b * m:(b + 1) * m] = ii
    return k, idx


def resample(resampler, w, u, m, ept):
    w = np.ascontiguousarray(w, np.float32)
    u = np.ascontiguousarray(u, np.float32)
    nsub = len(w) // m
    sel = np.zeros(len(w), np.int32)
    for b in range(nsub):
        wb = w[b * m:(b + 1) * m].copy()
        s = np.zeros(m, np.int32)
        if resampler == RES_REF:
            ub = u[b * m:(b + 1) * m].copy()
            lib().orc_resample_ref(_f(wb), _f(ub), m, _i(s))
        elif resampler == RES_SYSTEMATIC:
            lib().orc_resample_systematic(_f(wb), m, ept, C.c_float(float(u[b])), _i(s))
        else:
            prob = np.zeros(m, np.float32)
            al = np.zeros(m, np.uint32)
            lib().orc_vose_build(_f(wb), m, _f(prob), _u(al))
            for i in range(m):
                s[i] = lib().orc_vose_draw(_f(prob), _u(al), m, C.c_float(float(u[2 * (b * m + i)])),
                                           C.c_float(float(u[2 * (b * m + i) + 1])))
        sel[b * m:(b + 1) * m] = s
    return sel


def vose_build(w, m):
    w = np.ascontiguousarray(w, np.float32)
    prob = np.zeros(len(w), np.float32)
    alias = np.zeros(len(w), np.uint32)
    for b in range(len(w) // m):
        wb = w[b * m:(b + 1) * m].copy()
        p = np.zeros(m, np.float32)
        a = np.zeros(m, np.uint32)
        lib().orc_vose_build(_f(wb), m, _f(p), _u(a))
        prob[b * m:(b + 1) * m] = p
        alias[b * m:(b + 1) * m] = a
    return prob, alias


def vose_scaled(w, m):
    """The alias build's starting probabilities (normalised weights x m), per sub-filter."""
    w = np.ascontiguousarray(w, np.float32)
    out = np.zeros(len(w), np.float32)
    for b in range(len(w) // m):
        o = np.zeros(m, np.float32)
        lib().orc_vose_scaled(_f(np.ascontiguousarray(w[b * m:(b + 1) * m])), m, _f(o))
        out[b * m:(b + 1) * m] = o
    return out


def vose_draws(prob, alias, u2, m):
    """orc_vose_draw for every particle on the given tables; u2: 2 uniforms in [0,1) per particle."""
    prob = np.ascontiguousarray(prob, np.float32)
    alias = np.ascontiguousarray(alias, np.uint32)
    u2 = np.ascontiguousarray(u2, np.float32)
    n = len(prob)
    sel = np.zeros(n, np.int32)
    for b in range(n // m):
        pb = np.ascontiguousarray(prob[b * m:(b + 1) * m])
        ab = np.ascontiguousarray(alias[b * m:(b + 1) * m])
        for i in range(m):
            k = b * m + i
            sel[k] = lib().orc_vose_draw(_f(pb), _u(ab), m, C.c_float(float(u2[2 * k])), C.c_float(float(u2[2 * k + 1])))
    return sel


def implied_selection(prob, alias, m):
    """Per slot, the probability that one alias draw selects it: column c uniform,
    c itself with probability clamp(prob[c], 0, 1), alias[c] otherwise (FP64)."""
    prob = np.asarray(prob, np.float64).reshape(-1, m)
    alias = np.asarray(alias, np.int64).reshape(-1, m)
    keep = np.clip(prob, 0.0, 1.0)
    out = keep.copy()
    for b in range(prob.shape[0]):
        np.add.at(out[b], alias[b], 1.0 - keep[b])
    return (out / m).reshape(-1)


def scan_f64(w, m, ept):
    w = np.ascontiguousarray(w, np.float32)
    cum = np.zeros(m, np.float64)
    tot = lib().orc_scan_f64(_f(w), m, ept, _d(cum))
    return cum, tot


def blelloch(w):
    e = np.array(w, np.float32, copy=True)
    tot = lib().orc_blelloch_scan(_f(e), len(e))
    return e, tot


def torus_dims(N):
    dx, dy = C.c_int32(), C.c_int32()
    lib().orc_torus_dims(N, C.byref(dx), C.byref(dy))
    return dx.value, dy.value


def exchange_sources(mode, N, m, t, sorted_keys=None):
    src = np.zeros(N * m, np.int32)
    top = None
    if sorted_keys is not None:
        k = np.ascontiguousarray(sorted_keys, np.float32).reshape(N, m)
        top = np.ascontiguousarray(k[:, :t]).reshape(-1)
    lib().orc_exchange_sources(mode, N, m, t, None if top is None else _f(top), _i(src))
    return src


# ---- models ----------------------------------------------------------------------
def model_from_params(model, p):
    """OrcModel from the engine's ctypes params struct (esthera_b200.*Params)."""
    md = OrcModel()
    md.model = model
    if model == MODEL_UNICYCLE:
        md.num_state, md.num_noise = 3, 3
        md.dt = p.dt
        for i in range(3):
            md.sq[i] = p.sigma_q[i]
        md.sigma_r, md.sigma_b = p.sigma_range, p.sigma_bearing
        md.num_landmarks = p.num_landmarks
        for j in range(8):
            md.lm[j][0], md.lm[j][1] = p.landmarks[j][0], p.landmarks[j][1]
    elif model == MODEL_DHARM:
        md.num_state, md.num_noise = 12, 6
        md.dt, md.sigma_qd, md.sigma_p, md.sigma_a = p.dt, p.sigma_qd, p.sigma_pos, p.sigma_ang
        for i in range(6):
            md.a[i], md.alpha[i], md.d[i] = p.a[i], p.alpha[i], p.d[i]
    elif model == MODEL_BEACON:
        md.num_state, md.num_noise = 3, 3
        md.dt, md.sigma_r = p.dt, p.sigma_range
        for i in range(3):
            md.bnoise[i] = p.noise[i]
        md.num_beacons = p.num_beacons
        for j in range(16):
            for k in range(3):
                md.bc[j][k] = p.beacons[j][k]
    elif model == MODEL_CAMARM:
        md.num_state, md.num_noise = 9, 9
        md.dt = p.dt
        for i in range(2):
            md.fc[i], md.cc[i] = p.fc[i], p.cc[i]
        for i in range(4):
            md.kc[i] = p.kc[i]
    else:
        md.num_state, md.num_noise = 9, 9
        md.dt = p.dt
    return md


def model_step(md, state, noise, control, meas, dt=None):
    """state: S x n, noise: K x n -> (new state, loglik[n]) in double precision math."""
    st = np.array(state, np.float32, copy=True)
    n = st.shape[1]
    ll = np.zeros(n, np.float64)
    c = np.ascontiguousarray(control, np.float32)
    z = np.ascontiguousarray(meas, np.float32)
    md2 = md
    if dt is not None and dt > 0:
        md2 = OrcModel.from_buffer_copy(md)
        md2.dt = dt
    for i in range(n):
        s = np.ascontiguousarray(st[:, i])
        nz = np.ascontiguousarray(np.asarray(noise, np.float32)[:, i])
        ll[i] = lib().orc_model_step(C.byref(md2), _f(s), _f(nz), _f(c), _f(z))
        st[:, i] = s
    return st, ll


class Filter:
    """The oracle's whole filter (orc_filter_*)."""

    def __init__(self, md, m, N, t, exchange, resampler, rng, G, ept, log_weights, freq, seed, mask, init):
        self.f = OrcFilter()
        self.md = md
        self.m, self.N, self.S = m, N, md.num_state
        init = np.ascontiguousarray(init, np.float32)
        lib().orc_filter_init(C.byref(self.f), C.byref(md), m, N, t, exchange, resampler, rng, G, ept,
                              log_weights, freq, seed, mask, _f(init))

    def step(self, control, meas, threads=0, want_sel=False):
        e = OrcEstimate()
        c = np.ascontiguousarray(control, np.float32)
        z = np.ascontiguousarray(meas, np.float32)
        sel = np.zeros(self.m * self.N, np.int32) if want_sel else None
        lib().orc_filter_step(C.byref(self.f), _f(c), _f(z), C.byref(e), None if sel is None else _i(sel), threads)
        return e, sel

    def sample(self, control, meas, threads=0):
        """First half of step(): propagate + weight, sort, estimate."""
        e = OrcEstimate()
        c = np.ascontiguousarray(control, np.float32)
        z = np.ascontiguousarray(meas, np.float32)
        lib().orc_filter_sample(C.byref(self.f), _f(c), _f(z), C.byref(e), threads)
        return e

    def resample(self, threads=0):
        """Second half of step(): exchange + resampling from the sorted copy; the selection."""
        sel = np.zeros(self.m * self.N, np.int32)
        lib().orc_filter_resample(C.byref(self.f), _i(sel), threads)
        return sel

    def set_stream_offset(self, off):
        """Sub-filter b draws the stream of a larger filter's sub-filter off + b."""
        if lib().orc_filter_set_stream_offset(C.byref(self.f), off) != 0:
            raise ValueError("stream offsets need one stream per sub-filter")

    def set_sorted(self, soa, keys):
        """Replace the sorted copy (S x T states, T keys) between sample() and resample()."""
        T = self.m * self.N
        a = np.ascontiguousarray(soa, np.float32).reshape(-1)
        k = np.ascontiguousarray(keys, np.float32).reshape(-1)
        assert a.size == self.S * T and k.size == T
        C.memmove(self.f.tmp, a.ctypes.data, 4 * self.S * T)
        C.memmove(self.f.tkey, k.ctypes.data, 4 * T)

    def set_dt(self, dt):
        self.f.mdl.dt = dt

    def state(self):
        T = self.m * self.N
        return np.ctypeslib.as_array(self.f.state, shape=(self.S * T,)).reshape(self.S, T).copy()

    def sorted(self):
        T = self.m * self.N
        s = np.ctypeslib.as_array(self.f.tmp, shape=(self.S * T,)).reshape(self.S, T).copy()
        k = np.ctypeslib.as_array(self.f.tkey, shape=(T,)).copy()
        return s, k

    def set_state(self, soa):
        T = self.m * self.N
        a = np.ascontiguousarray(soa, np.float32).reshape(-1)
        C.memmove(self.f.state, a.ctypes.data, 4 * self.S * T)

    def close(self):
        if self.f.state:
            lib().orc_filter_free(C.byref(self.f))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def expneg(x):
    """orc_expneg element-wise (FP32 in, FP32 out)."""
    x = np.ascontiguousarray(x, np.float32).reshape(-1)
    return np.array([lib().orc_expneg(C.c_float(float(v))) for v in x], np.float32)


def stream_draws(num_noise, m, resampler):
    return lib().orc_stream_draws(num_noise, m, resampler)
