"""Test infrastructure: ctypes bindings of oracle/_ref/libref_kernels.so, the
reference's own CUDA block_sort / resampling / exchange_ring kernels (built by
oracle/build_ref_kernels.sh from the Esthera tree).  Needs a GPU; used only by
tests and the fixture script tests/golden/make_ref_kernel_golden.py."""
import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libref_kernels.so"
VALIAS_PATH = Path(__file__).resolve().parent / "_ref" / "libref_valias.so"
_lib = None


def available():
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB_PATH))
        fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)
        L.ref_block_sort.argtypes = [fp, C.c_int, C.c_int, ip]
        L.ref_resampling.argtypes = [fp, fp, C.c_int, C.c_int, C.c_float, ip]
        L.ref_exchange_ring.argtypes = [fp, C.c_int, C.c_int, C.c_int, ip]
        L.ref_sampling_importance.argtypes = [fp, fp, fp, fp, C.c_float, C.c_int, fp]
        for f in (L.ref_block_sort, L.ref_resampling, L.ref_exchange_ring, L.ref_sampling_importance):
            f.restype = C.c_int
        _lib = L
    return _lib


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed (%d)" % (what, rc))


def block_sort(keys, m):
    """(sorted keys, permutation within each sub-filter) of nsub = len/m descending sorts."""
    k = np.array(keys, np.float32, copy=True)
    perm = np.zeros(len(k), np.int32)
    _check(lib().ref_block_sort(_f(k), m, len(k) // m, _i(perm)), "ref_block_sort")
    return k, perm


def resampling(weights, u_particles, m, u_decision=None, freq=1.0):
    """Multinomial selections (slot within the sub-filter, -1 where skipped).
    u_particles / u_decision: the MTGP-style uniforms in [1, 2); the reference's
    cuRAND build takes them minus 1 (exact in FP32)."""
    w = np.ascontiguousarray(weights, np.float32)
    nsub = len(w) // m
    ud = np.ones(nsub, np.float32) if u_decision is None else np.asarray(u_decision, np.float32)
    r = np.concatenate([np.asarray(u_particles, np.float32) - np.float32(1.0), ud - np.float32(1.0)]).astype(np.float32)
    sel = np.zeros(len(w), np.int32)
    _check(lib().ref_resampling(_f(w), _f(r), m, nsub, float(freq), _i(sel)), "ref_resampling")
    return sel


def exchange_ring(keys, m, t):
    """(keys after the exchange, source slot of every slot)."""
    k = np.array(keys, np.float32, copy=True)
    src = np.zeros(len(k), np.int32)
    _check(lib().ref_exchange_ring(_f(k), m, len(k) // m, t, _i(src)), "ref_exchange_ring")
    return k, src


def sampling_importance(state, normals, control, meas, dt):
    """The reference's robot-arm propagate + weight: (new state [9][n], linear weights [n])."""
    st = np.array(state, np.float32, copy=True)
    nz = np.ascontiguousarray(normals, np.float32)
    ctl = np.zeros(7, np.float32)
    ctl[:5] = np.asarray(control, np.float32)[:5]
    z = np.ascontiguousarray(meas, np.float32)[:7].copy()
    w = np.zeros(st.shape[1], np.float32)
    _check(lib().ref_sampling_importance(_f(st), _f(nz), _f(ctl), _f(z), float(dt), st.shape[1], _f(w)),
           "ref_sampling_importance")
    return st, w


# ---- the reference unicycle program's kernel (oracle/build_ref_unicycle.sh) ----
UNICYCLE_LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libref_unicycle.so"
_ulib = None


def unicycle_available():
    return UNICYCLE_LIB_PATH.exists()


def unicycle_sampling(state, normals, v, w, dt, ranges):
    """The unicycle program's sampling_importance on n particles (one per block):
    (state out, S x n; linear weight norm * expf(-value), n)."""
    global _ulib
    if _ulib is None:
        L = C.CDLL(str(UNICYCLE_LIB_PATH))
        fp = C.POINTER(C.c_float)
        L.ref_unicycle_sampling.argtypes = [fp, fp, C.c_float, C.c_float, C.c_float, fp, C.c_int, fp, fp]
        L.ref_unicycle_sampling.restype = C.c_int
        _ulib = L
    st = np.ascontiguousarray(state, np.float32)
    nz = np.ascontiguousarray(normals, np.float32)
    z = np.ascontiguousarray(ranges, np.float32)
    n = st.shape[1]
    so = np.zeros_like(st)
    wt = np.zeros(n, np.float32)
    _check(_ulib.ref_unicycle_sampling(_f(st), _f(nz), v, w, dt, _f(z), n, _f(so), _f(wt)), "ref_unicycle_sampling")
    return so, wt


# ---- the reference's pinhole-camera arm model (oracle/build_ref_camarm.sh) ----
CAMARM_LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libref_camarm.so"
_clib = None


def camarm_available():
    return CAMARM_LIB_PATH.exists()


def camarm_sampling(state, normals, controls, meas, dt):
    """The reference's pinhole-camera sampling_iw on n particles (n a multiple of
    256): (state out, 9 x n; linear weight __expf(-value), n)."""
    global _clib
    if _clib is None:
        L = C.CDLL(str(CAMARM_LIB_PATH))
        fp = C.POINTER(C.c_float)
        L.ref_camarm_sampling.argtypes = [fp, fp, fp, fp, C.c_float, C.c_int, fp, fp]
        L.ref_camarm_sampling.restype = C.c_int
        _clib = L
    st = np.ascontiguousarray(state, np.float32)
    nz = np.ascontiguousarray(normals, np.float32)
    c = np.ascontiguousarray(controls[:5], np.float32)
    z = np.ascontiguousarray(meas[:7], np.float32)
    n = st.shape[1]
    so = np.zeros_like(st)
    wt = np.zeros(n, np.float32)
    _check(_clib.ref_camarm_sampling(_f(st), _f(nz), _f(c), _f(z), dt, n, _f(so), _f(wt)), "ref_camarm_sampling")
    return so, wt


_valias = None


def valias_available():
    return VALIAS_PATH.exists()


def valias(weights, u2, m):
    """The reference's own Vose resampler (resampling-valias.cl, compiled as CUDA
    by oracle/build_ref_valias.sh): (scaled starting probabilities, final prob,
    alias, selection) for nsub = len/m sub-filters; u2 holds 2 uniforms in
    [0,1) per particle.  The tables' order follows the GPU's atomics."""
    global _valias
    if _valias is None:
        L = C.CDLL(str(VALIAS_PATH))
        fp, up = C.POINTER(C.c_float), C.POINTER(C.c_uint32)
        L.ref_valias.argtypes = [fp, fp, C.c_int, C.c_int, fp, fp, up, up]
        L.ref_valias.restype = C.c_int
        _valias = L
    w = np.ascontiguousarray(weights, np.float32)
    u = np.ascontiguousarray(u2, np.float32)
    n = len(w)
    scaled, prob = np.zeros(n, np.float32), np.zeros(n, np.float32)
    alias, sel = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    up = C.POINTER(C.c_uint32)
    _check(_valias.ref_valias(_f(w), _f(u), m, n // m, _f(scaled), _f(prob), alias.ctypes.data_as(up),
                              sel.ctypes.data_as(up)), "ref_valias")
    return scaled, prob, alias, sel.astype(np.int32)


DRIVER_PATH = Path(__file__).resolve().parent / "_ref" / "libref_driver.so"
_driver = None


def driver_available():
    return DRIVER_PATH.exists()


def particle_filter(num_particles, num_blocks, num_transfer, resampling_freq, input_file, seed, out_path):
    """The reference's own driver loop (pf_generic_soa.cu particle_filter, MTGP32
    build with DEBUG_ESTIMATE, oracle/build_ref_driver.sh) with its streams
    seeded from `seed`.  Returns (per-step best-particle errors, best-particle
    states [x, y, vX, vY, angles...] and weights per step, final "N m t e"
    mean error) parsed from its output, written to out_path."""
    global _driver
    if _driver is None:
        L = C.CDLL(str(DRIVER_PATH))
        L.ref_particle_filter.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_char_p, C.c_uint, C.c_char_p]
        L.ref_particle_filter.restype = C.c_int
        _driver = L
    rc = _driver.ref_particle_filter(num_particles, num_blocks, num_transfer, resampling_freq,
                                     str(input_file).encode(), seed, str(out_path).encode())
    if rc != 0:
        raise RuntimeError("reference particle_filter returned %d" % rc)
    errs, best, w, mean = [], [], [], None
    for line in Path(out_path).read_text().splitlines():
        if line.startswith("EST "):
            head, wt = line[4:].split(" w: ")
            nums = head.replace("x:", "").replace("y:", "").replace("vX:", "").replace("vY:", "")
            nums = nums.replace("[", " ").replace("]", " ").replace(",", " ").split()
            best.append([float(v) for v in nums])
            w.append(float(wt))
        elif line.startswith("ACT ") and "| err:" in line:
            errs.append(float(line.split("| err:")[1]))
        else:
            tok = line.split()
            if len(tok) == 4 and tok[0].isdigit():
                mean = float(tok[3])
    return np.array(errs), np.array(best, np.float64), np.array(w, np.float64), mean
