"""esthera_b200 -- B200-native particle-filter engine (Python mirror of the C ABI).

The compute path is the CUDA library ``libesthera_b200.so`` built in-tree by
``esthera_b200.build``; this module only binds it with ctypes.  There is no
CPU fallback: importing works without a GPU, but every call that needs one
raises ``PFError`` carrying the library's status and message.

The Python surface mirrors the reference's driver and model hooks
(src/partfilt/cuda/pf_generic_soa.cu:686 ``particle_filter``; model hooks in
src/models/robotarm/cuda/pf_model_soa.cuh) -- see ``ParticleFilter`` and
``particle_filter``.
"""
import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ["ESTHERA_B200_LIB"]) if os.environ.get("ESTHERA_B200_LIB") else _PKG / "libesthera_b200.so"

# enums (include/esthera_b200.h)
PF_OK, PF_ERR_INVALID, PF_ERR_CUDA, PF_ERR_NOMEM, PF_ERR_UNSUPPORTED, PF_ERR_IO = 0, 1, 2, 3, 4, 5
PF_ERR_ADMISSION, PF_ERR_TIMEOUT, PF_ERR_NOT_FOUND, PF_ERR_BUSY = 6, 7, 8, 9
MODEL_UNICYCLE, MODEL_DHARM, MODEL_REFARM, MODEL_BEACON, MODEL_CAMARM = 0, 1, 2, 3, 4
EXCHANGE_NONE, EXCHANGE_RING, EXCHANGE_TORUS, EXCHANGE_ALL2ALL = 0, 1, 2, 3
RESAMPLE_REFERENCE, RESAMPLE_SYSTEMATIC, RESAMPLE_VOSE = 0, 1, 2
RNG_SUBFILTER, RNG_REFLAYOUT = 0, 1
PIPELINE_FUSED, PIPELINE_PHASED, PIPELINE_SPLIT = 0, 1, 2
QUEUE_DEPTH = 64  # PF_QUEUE_DEPTH: steps pf_step_submit may keep pending
MTGP_MASK_PARAMS, MTGP_MASK_CUDA_REF = 0, 0xFF800000
MAX_STATE, MAX_CONTROL, MAX_MEAS = 16, 8, 16


class PFConfig(C.Structure):
    _fields_ = [("particles_per_subfilter", C.c_int32), ("num_subfilters", C.c_int32),
                ("num_transfer", C.c_int32), ("exchange", C.c_int32), ("resampler", C.c_int32),
                ("resampling_freq", C.c_float), ("seed", C.c_uint32), ("rng", C.c_int32),
                ("mtgp_streams", C.c_int32), ("mtgp_mask", C.c_uint32), ("log_weights", C.c_int32),
                ("pipeline", C.c_int32), ("particles_per_thread", C.c_int32), ("device", C.c_int32),
                ("stream_offset", C.c_int32), ("exchange_period", C.c_int32), ("ess_fraction", C.c_float),
                ("threads_per_particle", C.c_int32)]


class StepInput(C.Structure):
    _fields_ = [("dt", C.c_float), ("control", C.c_float * MAX_CONTROL), ("meas", C.c_float * MAX_MEAS),
                ("pad", C.c_float * 7)]


class Estimate(C.Structure):
    _fields_ = [("mean", C.c_double * MAX_STATE), ("log_norm", C.c_double), ("best", C.c_float * MAX_STATE),
                ("best_key", C.c_float), ("best_subfilter", C.c_int32), ("step", C.c_int32),
                ("flags", C.c_int32)]


class UnicycleParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("sigma_q", C.c_float * 3), ("sigma_range", C.c_float),
                ("sigma_bearing", C.c_float), ("num_landmarks", C.c_int32), ("landmarks", (C.c_float * 2) * 8),
                ("init_state", C.c_float * 3)]


class DhArmParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("sigma_qd", C.c_float), ("sigma_pos", C.c_float), ("sigma_ang", C.c_float),
                ("a", C.c_float * 6), ("alpha", C.c_float * 6), ("d", C.c_float * 6), ("init_state", C.c_float * 12)]


class RefArmParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("init_state", C.c_float * 9)]


class CamArmParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("init_state", C.c_float * 9), ("fc", C.c_float * 2), ("cc", C.c_float * 2),
                ("kc", C.c_float * 4)]


class BeaconParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("noise", C.c_float * 3), ("sigma_range", C.c_float),
                ("num_beacons", C.c_int32), ("beacons", (C.c_float * 3) * 16), ("init_state", C.c_float * 3)]


STEP_INPUT_DTYPE = np.dtype([("dt", np.float32), ("control", np.float32, MAX_CONTROL),
                             ("meas", np.float32, MAX_MEAS), ("pad", np.float32, 7)])
ESTIMATE_DTYPE = np.dtype([("mean", np.float64, MAX_STATE), ("log_norm", np.float64),
                           ("best", np.float32, MAX_STATE), ("best_key", np.float32),
                           ("best_subfilter", np.int32), ("step", np.int32), ("flags", np.int32)])
assert STEP_INPUT_DTYPE.itemsize == C.sizeof(StepInput) == 128
assert ESTIMATE_DTYPE.itemsize == C.sizeof(Estimate)

PARAMS_TYPE = {MODEL_UNICYCLE: UnicycleParams, MODEL_DHARM: DhArmParams, MODEL_REFARM: RefArmParams,
               MODEL_BEACON: BeaconParams, MODEL_CAMARM: CamArmParams}


class PFError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (status_string(status), msg))
        self.status = status


_lib = None


def lib():
    """The loaded CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError("libesthera_b200.so not built; run `python -m esthera_b200.build`")
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L):
    P = C.c_void_p
    fp, ip, up = C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_uint32)
    sig = {
        "pf_status_string": (C.c_char_p, [C.c_int]),
        "pf_last_error": (C.c_char_p, []),
        "pf_version": (C.c_int32, []),
        "pf_device_count": (C.c_int32, []),
        "pf_model_info": (C.c_int, [C.c_int, ip, ip, ip, ip]),
        "pf_model_list": (C.c_int32, [P, C.c_int32]),
        "pf_model_name": (C.c_char_p, [C.c_int32]),
        "pf_config_default": (C.c_int, [C.POINTER(PFConfig)]),
        "pf_create": (C.c_int, [C.POINTER(PFConfig), C.c_int, P, C.c_size_t, C.POINTER(P)]),
        "pf_destroy": (C.c_int, [P]),
        "pf_set_initial_state": (C.c_int, [P, fp]),
        "pf_set_particles": (C.c_int, [P, fp]),
        "pf_get_particles": (C.c_int, [P, fp]),
        "pf_get_sorted": (C.c_int, [P, fp, fp]),
        "pf_get_selection": (C.c_int, [P, ip]),
        "pf_record_selection": (C.c_int, [P, C.c_int32]),
        "pf_step": (C.c_int, [P, C.POINTER(StepInput), C.POINTER(Estimate)]),
        "pf_run_device": (C.c_int, [P, P, P, C.c_int32, C.c_int32]),
        "pf_run_device_continue": (C.c_int, [P, C.c_int32]),
        "pf_step_submit": (C.c_int, [P, P]),
        "pfk_bounded_wait_test": (C.c_int, [C.c_int32, P]),
        "pfk_bounded_wait_mixed_test": (C.c_int, [P, C.c_int32, P, P]),
        "pf_step_collect": (C.c_int, [P, P, C.c_int32, C.c_int32, P]),
        "pf_synchronize": (C.c_int, [P]),
        "pf_stream": (P, [P]),
        "pf_set_timing": (C.c_int, [P, C.c_int32]),
        "pf_last_step_timing": (C.c_int, [P, fp, C.c_int32, ip]),
        "pf_phase_name": (C.c_char_p, [P, C.c_int32]),
        "pf_get_info": (C.c_int, [P, ip, ip, ip, ip, C.POINTER(C.c_int64)]),
        "pf_snapshot_size": (C.c_int64, [P]),
        "pf_snapshot": (C.c_int, [P, P]),
        "pf_restore": (C.c_int, [P, P, C.c_size_t]),
        "pf_shard_create": (C.c_int, [C.POINTER(PFConfig), C.c_int, P, C.c_size_t, C.c_int32, C.c_int32,
                                      C.POINTER(P)]),
        "pf_shard_info": (C.c_int, [P, ip, ip, ip, ip, C.POINTER(C.c_int64)]),
        "pf_shard_sample": (C.c_int, [P, C.POINTER(StepInput)]),
        "pf_shard_halo_out": (C.c_int, [P, C.c_int32, P]),
        "pf_shard_halo_in": (C.c_int, [P, C.c_int32, P]),
        "pf_shard_halo_copy": (C.c_int, [P, C.c_int32, P]),
        "pf_shard_resample": (C.c_int, [P]),
        "pf_shard_group_rows": (C.c_int, [P, C.POINTER(C.c_double), fp]),
        "pf_shard_estimate": (C.c_int, [P, C.POINTER(C.c_double), fp, C.c_int32, C.POINTER(Estimate)]),
        "pf_batch_create": (C.c_int, [C.POINTER(PFConfig), C.c_int, C.c_int32, ip, P, C.c_size_t, C.POINTER(P)]),
        "pf_batch_destroy": (C.c_int, [P]),
        "pf_batch_set_initial_states": (C.c_int, [P, fp]),
        "pf_batch_get_particles": (C.c_int, [P, C.c_int32, fp]),
        "pf_batch_step": (C.c_int, [P, P, P]),
        "pf_batch_submit": (C.c_int, [P, P, P, C.c_int32, C.c_int32]),
        "pf_batch_poll": (C.c_int, [P, ip]),
        "pf_batch_synchronize": (C.c_int, [P]),
        "pf_batch_stream": (P, [P]),
        "pf_batch_info": (C.c_int, [P, ip, C.POINTER(C.c_int64), ip, ip, C.POINTER(C.c_int64)]),
        "pf_batch_filter_info": (C.c_int, [P, C.c_int32, ip, ip, C.POINTER(C.c_int64)]),
        "pf_batch_get_sorted": (C.c_int, [P, C.c_int32, fp, fp]),
        "pf_batch_filter_shape": (C.c_int, [P, C.c_int32, ip, ip]),
        "pf_batch_autotune": (C.c_int, [C.POINTER(PFConfig), C.c_int, C.c_int32, ip, P, C.c_size_t, P, fp, C.c_int32,
                                        C.c_int32, ip, C.c_int32, ip, C.c_int32, ip, C.c_int32, ip, C.c_int32,
                                        C.c_float,
                                        C.POINTER(TuneEntry), C.c_int32, ip, C.POINTER(PFConfig)]),
        "pf_server_create": (C.c_int, [C.POINTER(PFConfig), C.c_int64, C.c_int32, C.POINTER(P)]),
        "pf_server_destroy": (C.c_int, [P]),
        "pf_server_footprint": (C.c_int64, [P, C.c_int, C.c_int32]),
        "pf_server_open": (C.c_int, [P, C.c_int, P, C.c_size_t, C.c_int32, C.c_uint32, ip]),
        "pf_server_close": (C.c_int, [P, C.c_int32]),
        "pf_server_update": (C.c_int, [P, C.c_int32, P, C.c_uint64]),
        "pf_server_launch": (C.c_int, [P, ip]),
        "pf_server_poll": (C.c_int, [P, C.c_int32, P, C.c_int32, ip]),
        "pf_server_stats_get": (C.c_int, [P, C.POINTER(ServerStats)]),
        "pf_server_get_particles": (C.c_int, [P, C.c_int32, fp, fp, fp]),
        "pf_server_snapshot_size": (C.c_int64, [P, C.c_int32]),
        "pf_server_snapshot": (C.c_int, [P, C.c_int32, P]),
        "pf_server_restore": (C.c_int, [P, C.c_int32, P, C.c_size_t]),
        "pf_load_default": (C.c_int, [C.POINTER(LoadConfig)]),
        "pf_serve_load": (C.c_int, [C.POINTER(PFConfig), C.POINTER(LoadConfig), C.POINTER(LoadReport)]),
        "pfk_mtgp_generate": (C.c_int, [C.c_int32, C.c_uint32, C.c_uint32, C.c_int32, C.c_int64, C.c_int32, up]),
        "pfk_boxmuller": (C.c_int, [fp, C.c_int64]),
        "pfk_bitonic_sort": (C.c_int, [fp, ip, C.c_int32, C.c_int32, C.c_int32]),
        "pfk_rank_sort": (C.c_int, [fp, ip, C.c_int32, C.c_int32, C.c_int32, ip]),
        "pfk_resample": (C.c_int, [C.c_int32, fp, fp, C.c_int32, C.c_int32, C.c_int32, ip]),
        "pfk_vose_build": (C.c_int, [fp, C.c_int32, C.c_int32, C.c_int32, fp, up]),
        "pfk_exchange_sources": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, fp, ip]),
        "pfk_estimate": (C.c_int, [fp, fp, C.c_int32, C.c_int64, C.c_int32, C.c_uint32, C.c_int32,
                                   C.POINTER(Estimate)]),
        "pfk_estimate_noalloc": (C.c_int, [P, P, C.c_int32, C.c_int64, C.c_int32, C.c_uint32, C.c_int32, P, P]),
        "pfk_model_step": (C.c_int, [C.c_int, P, C.c_size_t, C.POINTER(StepInput), C.c_int32, fp, fp, fp]),
        "pf_unicycle_default_params": (C.c_int, [C.c_uint32, C.c_int32, C.POINTER(UnicycleParams)]),
        "pf_dharm_default_params": (C.c_int, [C.c_uint32, C.POINTER(DhArmParams)]),
        "pf_make_trace": (C.c_int, [C.c_int, P, C.c_uint32, C.c_int32, P, fp]),
        "pf_read_trace_line": (C.c_int, [P, C.c_int, C.POINTER(StepInput), fp]),
        "pf_refarm_estimate_error": (C.c_float, [fp, fp]),
        "pf_particle_filter": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_char_p, fp]),
        "pf_beacon_default_params": (C.c_int, [C.POINTER(BeaconParams)]),
        "pf_camarm_default_params": (C.c_int, [C.POINTER(CamArmParams)]),
        "pf_beacon_estimate_error": (C.c_float, [fp, fp]),
        "pf_beacon_particle_filter": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_char_p, fp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def status_string(s):
    try:
        return lib().pf_status_string(s).decode()
    except Exception:  # library missing: still format the error
        return "status %d" % s


def check(status):
    if status != PF_OK:
        raise PFError(status, lib().pf_last_error().decode())


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _uptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def device_count():
    return int(lib().pf_device_count())


def model_info(model):
    v = [C.c_int32() for _ in range(4)]
    check(lib().pf_model_info(model, *[C.byref(x) for x in v]))
    return tuple(x.value for x in v)  # num_state, num_noise, num_control, num_meas


def default_config(**kw):
    c = PFConfig()
    check(lib().pf_config_default(C.byref(c)))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError("pf_config has no field %r" % k)
        setattr(c, k, v)
    return c


# ---- synthetic traces --------------------------------------------------------
def unicycle_params(seed, num_landmarks=4):
    p = UnicycleParams()
    check(lib().pf_unicycle_default_params(seed, num_landmarks, C.byref(p)))
    return p


def dharm_params(seed):
    p = DhArmParams()
    check(lib().pf_dharm_default_params(seed, C.byref(p)))
    return p


MODEL_USER_BASE = 64  # first id of models added with PF_MODEL (esthera_b200_model.cuh)
MODEL_LINGAUSS = MODEL_USER_BASE  # the linear-Gaussian example model (csrc/pf_model_lingauss.cu)


class LinGaussParams(C.Structure):
    """Parameters of the linear-Gaussian example model (pf_lingauss_params)."""
    _fields_ = [("dt", C.c_float), ("sigma_v", C.c_float), ("sigma_z", C.c_float), ("init_state", C.c_float * 2)]


def model_list():
    """Ids of every model compiled into the library (built-in and registered with PF_MODEL)."""
    n = lib().pf_model_list(None, 0)
    ids = np.zeros(max(n, 1), np.int32)
    lib().pf_model_list(ids.ctypes.data_as(C.c_void_p), n)
    return [int(i) for i in ids[:n]]


def model_name(model):
    r = lib().pf_model_name(model)
    return None if r is None else r.decode()


def refarm_params(dt=1.0):
    p = RefArmParams()
    p.dt = dt
    for i in range(5):
        p.init_state[i] = 0.75 * np.pi
    p.init_state[5] = 7.0
    return p


def beacon_params():
    """The reference unicycle program's constants (pf_beacon_default_params)."""
    p = BeaconParams()
    check(lib().pf_beacon_default_params(C.byref(p)))
    return p


def camarm_params():
    """The reference pinhole camera's calibration and the arm's start state (pf_camarm_default_params)."""
    p = CamArmParams()
    check(lib().pf_camarm_default_params(C.byref(p)))
    return p


def make_trace(model, params, seed, steps):
    """(inputs: structured array of STEP_INPUT_DTYPE, truth: steps x num_state float32)."""
    S = model_info(model)[0]
    inputs = np.zeros(steps, dtype=STEP_INPUT_DTYPE)
    truth = np.zeros((steps, S), dtype=np.float32)
    check(lib().pf_make_trace(model, C.byref(params), seed, steps, inputs.ctypes.data_as(C.c_void_p),
                              _fptr(truth)))
    return inputs, truth


def step_input(rec):
    """A StepInput from one STEP_INPUT_DTYPE record."""
    s = StepInput()
    C.memmove(C.byref(s), np.ascontiguousarray(rec).ctypes.data, 128)
    return s


def estimate_to_numpy(e):
    a = np.zeros(1, dtype=ESTIMATE_DTYPE)
    C.memmove(a.ctypes.data, C.byref(e), ESTIMATE_DTYPE.itemsize)
    return a[0]


# ---- filter ----------------------------------------------------------------------
class ParticleFilter:
    """One distributed particle filter on one GPU (wraps pf_create / pf_step)."""

    def __init__(self, model, params, config=None, **cfg):
        self.model = model
        self.params = params
        self.config = config if config is not None else default_config(**cfg)
        self.num_state, self.num_noise, _, _ = model_info(model)
        h = C.c_void_p()
        check(lib().pf_create(C.byref(self.config), model, C.byref(params), C.sizeof(params), C.byref(h)))
        self._h = h
        self.m = self.config.particles_per_subfilter
        self.N = self.config.num_subfilters
        self.T = self.m * self.N

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().pf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        pp, e, dx, dy, b = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_int64()
        check(lib().pf_get_info(self._h, C.byref(pp), C.byref(e), C.byref(dx), C.byref(dy), C.byref(b)))
        return {"pipeline": pp.value, "particles_per_thread": e.value, "torus": (dx.value, dy.value),
                "device_bytes": b.value}

    def set_initial_state(self, state):
        check(lib().pf_set_initial_state(self._h, _fptr(_f32(state))))

    def set_particles(self, soa):
        a = _f32(soa).reshape(self.num_state, self.T)
        check(lib().pf_set_particles(self._h, _fptr(a)))

    def particles(self):
        a = np.zeros((self.num_state, self.T), np.float32)
        check(lib().pf_get_particles(self._h, _fptr(a)))
        return a

    def sorted(self):
        s = np.zeros((self.num_state, self.T), np.float32)
        k = np.zeros(self.T, np.float32)
        check(lib().pf_get_sorted(self._h, _fptr(s), _fptr(k)))
        return s, k

    def record_selection(self, on=True):
        check(lib().pf_record_selection(self._h, 1 if on else 0))

    def selection(self):
        a = np.zeros(self.T, np.int32)
        check(lib().pf_get_selection(self._h, _iptr(a)))
        return a

    def step(self, inp):
        """One filter step; inp is a STEP_INPUT_DTYPE record or a StepInput."""
        s = inp if isinstance(inp, StepInput) else step_input(inp)
        e = Estimate()
        check(lib().pf_step(self._h, C.byref(s), C.byref(e)))
        return estimate_to_numpy(e)

    def submit(self, inp):
        """Enqueue one step with a host input; returns without waiting (pf_step_submit)."""
        s = inp if isinstance(inp, StepInput) else step_input(inp)
        check(lib().pf_step_submit(self._h, C.byref(s)))

    def collect(self, max_n=None, wait=True):
        """Estimates of submitted steps, oldest first (pf_step_collect): ESTIMATE_DTYPE [n]."""
        max_n = QUEUE_DEPTH if max_n is None else int(max_n)
        out = np.zeros(max(max_n, 1), ESTIMATE_DTYPE)
        n = C.c_int32(0)
        check(lib().pf_step_collect(self._h, out.ctypes.data_as(C.c_void_p), max_n, 1 if wait else 0, C.byref(n)))
        return out[:n.value]

    def run_device(self, d_inputs_ptr, d_estimates_ptr, capacity, steps):
        """Reset the step counter and run `steps` steps over device arrays of `capacity` entries."""
        check(lib().pf_run_device(self._h, C.c_void_p(d_inputs_ptr), C.c_void_p(d_estimates_ptr), capacity, steps))

    def run_continue(self, steps):
        check(lib().pf_run_device_continue(self._h, steps))

    def synchronize(self):
        check(lib().pf_synchronize(self._h))

    def stream(self):
        return lib().pf_stream(self._h)

    def set_timing(self, on=True):
        check(lib().pf_set_timing(self._h, 1 if on else 0))

    def last_step_timing(self):
        """[(phase name, ms)] of the launches of the last step (timing must be on)."""
        ms = np.zeros(8, np.float32)
        n = C.c_int32()
        check(lib().pf_last_step_timing(self._h, _fptr(ms), 8, C.byref(n)))
        return [(lib().pf_phase_name(self._h, i).decode(), float(ms[i])) for i in range(n.value)]

    def snapshot(self):
        n = lib().pf_snapshot_size(self._h)
        buf = np.zeros(n, np.uint8)
        check(lib().pf_snapshot(self._h, buf.ctypes.data_as(C.c_void_p)))
        return buf

    def restore(self, buf):
        b = np.ascontiguousarray(buf, np.uint8)
        check(lib().pf_restore(self._h, b.ctypes.data_as(C.c_void_p), b.nbytes))


SHARD_ROW = 32  # doubles per group row (PF_SHARD_ROW)


class FilterShard(ParticleFilter):
    """Rows [row0, row1) of a torus-exchange filter whose whole size is
    config.num_subfilters sub-filters (pf_shard_*).  A step over all shards:
    sample() on each, send_halos() (or halo_out / halo_in across processes),
    resample() on each, then estimate() from every shard's group_rows() in row
    order.  The shards' particles and estimate equal the whole filter's."""

    def __init__(self, model, params, row0, row1, config=None, **cfg):
        self.model = model
        self.params = params
        self.config = config if config is not None else default_config(**cfg)
        self.num_state, self.num_noise, _, _ = model_info(model)
        h = C.c_void_p()
        check(lib().pf_shard_create(C.byref(self.config), model, C.byref(params), C.sizeof(params), row0, row1,
                                    C.byref(h)))
        self._h = h
        r0, r1, b0, ng = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        hb = C.c_int64()
        check(lib().pf_shard_info(h, C.byref(r0), C.byref(r1), C.byref(b0), C.byref(ng), C.byref(hb)))
        self.rows = (r0.value, r1.value)
        self.first_subfilter = b0.value
        self.num_groups = ng.value
        self.halo_bytes = hb.value
        self.m = self.config.particles_per_subfilter
        self.N_total = self.config.num_subfilters
        dx, rows = self.info()["torus"]
        self.N = dx * rows
        self.T = self.m * self.N

    def sample(self, inp):
        s = inp if isinstance(inp, StepInput) else step_input(inp)
        check(lib().pf_shard_sample(self._h, C.byref(s)))

    def halo_out(self, direction):
        """Block `direction` of this shard's export (0: last row, for the shard below; 1: first row, above)."""
        b = np.zeros(self.halo_bytes, np.uint8)
        check(lib().pf_shard_halo_out(self._h, direction, b.ctypes.data_as(C.c_void_p)))
        return b

    def halo_in(self, direction, buf):
        """Import block `direction` (0: the row above this shard, 1: the row below)."""
        b = np.ascontiguousarray(buf, np.uint8)
        if b.nbytes != self.halo_bytes:
            raise ValueError("halo block of %d bytes, expected %d" % (b.nbytes, self.halo_bytes))
        check(lib().pf_shard_halo_in(self._h, direction, b.ctypes.data_as(C.c_void_p)))

    def send_halo(self, direction, to):
        """Device copy of export block `direction` into shard `to` (its neighbour)."""
        check(lib().pf_shard_halo_copy(self._h, direction, to._h))

    def resample(self):
        check(lib().pf_shard_resample(self._h))

    def group_rows(self):
        rows = np.zeros((self.num_groups, SHARD_ROW), np.float64)
        st = np.zeros((self.num_groups, self.num_state), np.float32)
        check(lib().pf_shard_group_rows(self._h, rows.ctypes.data_as(C.POINTER(C.c_double)), _fptr(st)))
        return rows, st

    def estimate(self, rows, states):
        """The whole filter's estimate from every shard's group rows, in row order."""
        r = np.ascontiguousarray(rows, np.float64)
        st = _f32(states)
        e = Estimate()
        check(lib().pf_shard_estimate(self._h, r.ctypes.data_as(C.POINTER(C.c_double)), _fptr(st), r.shape[0],
                                      C.byref(e)))
        return estimate_to_numpy(e)


def shard_step(shards, inp):
    """One step of a filter spread over `shards` (in row order, one process)."""
    for s in shards:
        s.sample(inp)
    n = len(shards)
    for i, s in enumerate(shards):
        s.send_halo(0, shards[(i + 1) % n])
        s.send_halo(1, shards[(i - 1) % n])
    for s in shards:
        s.resample()
    parts = [s.group_rows() for s in shards]
    rows = np.concatenate([p[0] for p in parts])
    states = np.concatenate([p[1] for p in parts])
    return shards[0].estimate(rows, states)


class FilterBatch:
    """Many independent filters of uneven particle counts stepped together
    (pf_batch_*).  params: a sequence of per-filter model parameter structs."""

    def __init__(self, model, params, num_particles, config=None, **cfg):
        self.model = model
        self.config = config if config is not None else default_config(**cfg)
        self.num_state, self.num_noise, _, _ = model_info(model)
        self.counts = np.ascontiguousarray(num_particles, np.int32)
        self.F = len(self.counts)
        if len(params) != self.F:
            raise ValueError("one parameter struct per filter")
        ptype = type(params[0])
        arr = (ptype * self.F)(*params)
        h = C.c_void_p()
        check(lib().pf_batch_create(C.byref(self.config), model, self.F, _iptr(self.counts), C.cast(arr, C.c_void_p),
                                    C.sizeof(ptype), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().pf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        nf, tp, ns, e, b = C.c_int32(), C.c_int64(), C.c_int32(), C.c_int32(), C.c_int64()
        check(lib().pf_batch_info(self._h, C.byref(nf), C.byref(tp), C.byref(ns), C.byref(e), C.byref(b)))
        return {"num_filters": nf.value, "total_particles": tp.value, "total_subfilters": ns.value,
                "particles_per_thread": e.value, "device_bytes": b.value}

    def filter_info(self, f):
        n, so, po = C.c_int32(), C.c_int32(), C.c_int64()
        check(lib().pf_batch_filter_info(self._h, f, C.byref(n), C.byref(so), C.byref(po)))
        return {"num_subfilters": n.value, "stream_offset": so.value, "particle_offset": po.value}

    def filter_shape(self, f):
        """(sub-filter size m_f, particles per thread) of filter f."""
        m, e = C.c_int32(), C.c_int32()
        check(lib().pf_batch_filter_shape(self._h, f, C.byref(m), C.byref(e)))
        return m.value, e.value

    def set_initial_states(self, states):
        a = _f32(states).reshape(self.F, self.num_state)
        check(lib().pf_batch_set_initial_states(self._h, _fptr(a)))

    def particles(self, f):
        a = np.zeros((self.num_state, int(self.counts[f])), np.float32)
        check(lib().pf_batch_get_particles(self._h, f, _fptr(a)))
        return a

    def step(self, inputs):
        """One step of every filter; inputs: STEP_INPUT_DTYPE array [F]; returns ESTIMATE_DTYPE [F]."""
        a = np.ascontiguousarray(inputs, STEP_INPUT_DTYPE)
        out = np.zeros(self.F, ESTIMATE_DTYPE)
        check(lib().pf_batch_step(self._h, a.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
        return out

    def sorted(self, f):
        n = int(self.counts[f])
        s = np.zeros((self.num_state, n), np.float32)
        k = np.zeros(n, np.float32)
        check(lib().pf_batch_get_sorted(self._h, f, _fptr(s), _fptr(k)))
        return s, k

    def submit(self, d_inputs_ptr, d_estimates_ptr, capacity, steps):
        check(lib().pf_batch_submit(self._h, C.c_void_p(d_inputs_ptr), C.c_void_p(d_estimates_ptr), capacity, steps))

    def poll(self):
        d = C.c_int32()
        check(lib().pf_batch_poll(self._h, C.byref(d)))
        return bool(d.value)

    def synchronize(self):
        check(lib().pf_batch_synchronize(self._h))

    def stream(self):
        return lib().pf_batch_stream(self._h)


class ServerStats(C.Structure):
    _fields_ = [("open_filters", C.c_int32), ("in_flight", C.c_int32), ("resident_particles", C.c_int64),
                ("queued_updates", C.c_int64), ("bytes_in_use", C.c_int64), ("budget", C.c_int64),
                ("launches", C.c_int64), ("updates", C.c_int64), ("particle_steps", C.c_int64)]


SERVER_RESULT_DTYPE = np.dtype([("filter", np.int32), ("step", np.int32), ("tag", np.uint64),
                                ("particles", np.int64), ("estimate", ESTIMATE_DTYPE)])


class Server:
    """Resident filters with continuously batched updates (pf_server_*)."""

    def __init__(self, hbm_budget, max_filters, config=None, **cfg):
        self.config = config if config is not None else default_config(**cfg)
        self.max_filters = max_filters
        h = C.c_void_p()
        check(lib().pf_server_create(C.byref(self.config), int(hbm_budget), max_filters, C.byref(h)))
        self._h = h
        self._out = np.zeros(max_filters, SERVER_RESULT_DTYPE)
        self.models = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().pf_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def footprint(self, model, num_particles):
        return lib().pf_server_footprint(self._h, model, num_particles)

    def open(self, model, params, num_particles, seed):
        i = C.c_int32()
        check(lib().pf_server_open(self._h, model, C.byref(params), C.sizeof(params), num_particles, seed,
                                   C.byref(i)))
        self.models[i.value] = model
        return i.value

    def close_filter(self, fid):
        check(lib().pf_server_close(self._h, fid))
        self.models.pop(fid, None)

    def update(self, fid, inp, tag=0):
        a = np.ascontiguousarray(inp, STEP_INPUT_DTYPE)
        check(lib().pf_server_update(self._h, fid, a.ctypes.data_as(C.c_void_p), tag))

    def launch(self):
        n = C.c_int32()
        check(lib().pf_server_launch(self._h, C.byref(n)))
        return n.value

    def poll(self, wait=True):
        n = C.c_int32()
        check(lib().pf_server_poll(self._h, 1 if wait else 0, self._out.ctypes.data_as(C.c_void_p),
                                   self.max_filters, C.byref(n)))
        return self._out[:n.value].copy()

    def stats(self):
        st = ServerStats()
        check(lib().pf_server_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def particles(self, fid, n):
        S = model_info(self.models[fid])[0]
        a = np.zeros((S, n), np.float32)
        srt = np.zeros((S, n), np.float32)
        k = np.zeros(n, np.float32)
        check(lib().pf_server_get_particles(self._h, fid, _fptr(a), _fptr(srt), _fptr(k)))
        return a, srt, k

    def snapshot(self, fid):
        """Filter fid's particles, streams and update count (pf_server_snapshot), as bytes."""
        n = lib().pf_server_snapshot_size(self._h, fid)
        if n < 0:
            raise PFError(PF_ERR_NOT_FOUND, "no open filter %d" % fid)
        buf = np.zeros(n, np.uint8)
        check(lib().pf_server_snapshot(self._h, fid, buf.ctypes.data_as(C.c_void_p)))
        return buf.tobytes()

    def restore(self, fid, snap):
        buf = np.frombuffer(snap, np.uint8).copy()
        check(lib().pf_server_restore(self._h, fid, buf.ctypes.data_as(C.c_void_p), buf.nbytes))


class LoadConfig(C.Structure):
    _fields_ = [("rate", C.c_double), ("duration_s", C.c_double), ("frac_unicycle", C.c_double),
                ("min_particles", C.c_int32), ("max_particles", C.c_int32), ("min_updates", C.c_int32),
                ("max_updates", C.c_int32), ("min_gap_ms", C.c_double), ("max_gap_ms", C.c_double),
                ("seed", C.c_uint32), ("max_filters", C.c_int32), ("hbm_budget", C.c_int64),
                ("norm_check_every", C.c_int32), ("pad0", C.c_int32), ("drain_limit_s", C.c_double)]


class LoadReport(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("requests", "admitted", "admission_waits", "completed_requests", "updates",
                                         "launches", "max_resident_particles", "max_bytes_in_use")] + \
               [("max_open_filters", C.c_int32), ("incomplete", C.c_int32)] + \
               [(k, C.c_double) for k in ("wall_s", "particle_steps", "particle_steps_per_s",
                                          "demanded_particle_steps_per_s", "mean_batch", "lat_p50_ms", "lat_p99_ms",
                                          "lat_p999_ms", "lat_max_ms")] + \
               [("norm_checked", C.c_int64), ("norm_err_max", C.c_double), ("norm_err_mean", C.c_double)]


def serve_load(filter_config=None, load=None, **load_kw):
    """Run the served tracking load (pf_serve_load); returns the report as a dict."""
    cfg = filter_config if filter_config is not None else default_config(
        particles_per_subfilter=256, particles_per_thread=4, num_transfer=2, exchange=EXCHANGE_RING)
    lc = LoadConfig()
    check(lib().pf_load_default(C.byref(lc)))
    for k, v in dict(load or {}, **load_kw).items():
        if not hasattr(lc, k):
            raise AttributeError("pf_load_config has no field %r" % k)
        setattr(lc, k, v)
    rep = LoadReport()
    check(lib().pf_serve_load(C.byref(cfg), C.byref(lc), C.byref(rep)))
    return {k: getattr(rep, k) for k, _ in LoadReport._fields_}


class TuneEntry(C.Structure):
    _fields_ = [("particles_per_subfilter", C.c_int32), ("particles_per_thread", C.c_int32),
                ("threads_per_particle", C.c_int32), ("exchange_period", C.c_int32), ("status", C.c_int32),
                ("ms_per_step", C.c_float),
                ("accepted", C.c_int32), ("particle_steps_per_s", C.c_double), ("rmse", C.c_double)]


def batch_autotune(model, params, counts, inputs, truth=None, m_list=(128, 256, 512, 1024), ppt_list=(1, 2, 4),
                   period_list=(1, 2, 4), burn_in=0, rmse_tol=0.01, tpp_list=(1,), **cfg):
    """pf_batch_autotune over host inputs [F][steps] (and truth [F][steps][S]):
    returns (best pf_config, [candidate dicts])."""
    base = default_config(**cfg)
    counts = np.ascontiguousarray(counts, np.int32)
    F = len(counts)
    ptype = type(params[0])
    arr = (ptype * F)(*params)
    inp = np.ascontiguousarray(inputs, STEP_INPUT_DTYPE)
    steps = inp.shape[1]
    tr = None if truth is None else _f32(truth)
    ml, pl, tl, ql = (np.ascontiguousarray(x, np.int32) for x in (m_list, ppt_list, tpp_list, period_list))
    cap = len(ml) * len(pl) * len(tl) * len(ql)
    table = (TuneEntry * cap)()
    n = C.c_int32()
    best = PFConfig()
    check(lib().pf_batch_autotune(C.byref(base), model, F, _iptr(counts), C.cast(arr, C.c_void_p), C.sizeof(ptype),
                                  inp.ctypes.data_as(C.c_void_p), None if tr is None else _fptr(tr), steps, burn_in,
                                  _iptr(ml), len(ml), _iptr(pl), len(pl), _iptr(tl), len(tl), _iptr(ql), len(ql),
                                  rmse_tol, table, cap,
                                  C.byref(n), C.byref(best)))
    rows = [{k: getattr(table[i], k) for k, _ in TuneEntry._fields_} for i in range(n.value)]
    return best, rows


def particle_filter(num_particles, num_blocks, num_transfer, resampling_freq, input_file):
    """Drop-in for the reference driver call (pf_generic_soa.cu:686): robot-arm
    model over a reference trace file; returns the mean estimate error."""
    e = C.c_float()
    check(lib().pf_particle_filter(num_particles, num_blocks, num_transfer, resampling_freq,
                                   str(input_file).encode(), C.byref(e)))
    return e.value


def beacon_particle_filter(num_particles, num_blocks, num_transfer, input_file):
    """Drop-in for the reference unicycle program's loop (src/models/unicycle/
    particle_filter.cu:596-1160) over a unicycle trace file; returns the mean
    position error of the best particle."""
    e = C.c_float()
    check(lib().pf_beacon_particle_filter(num_particles, num_blocks, num_transfer, str(input_file).encode(),
                                          C.byref(e)))
    return e.value


# ---- kernel-level entry points (parity tests) --------------------------------------
def mtgp_generate(G, seed, per_stream, kind=1, mask=MTGP_MASK_PARAMS, calls=1):
    out = np.zeros(calls * G * per_stream, np.uint32)
    check(lib().pfk_mtgp_generate(G, seed, mask, kind, per_stream, calls, _uptr(out)))
    return out


def boxmuller(data, n=None):
    n = len(data) if n is None else n
    a = np.array(data, dtype=np.float32, copy=True)
    if len(a) < 2 * ((n + 1) // 2):
        a = np.concatenate([a, np.zeros(2 * ((n + 1) // 2) - len(a), np.float32)])
    check(lib().pfk_boxmuller(_fptr(a), n))
    return a


def bounded_wait_test(limit=2000):
    """Run the bounded mbarrier wait on a phase nothing completes; returns the kernel's status (1: ran out)."""
    st = C.c_int32(-1)
    check(lib().pfk_bounded_wait_test(int(limit), C.byref(st)))
    return st.value


def bounded_wait_mixed_test(limits):
    """CTA-wide bounded wait with a bulk copy in flight and per-thread poll
    limits; returns (outcome per thread, copied flag)."""
    lim = np.ascontiguousarray(limits, np.int32)
    out = np.zeros(len(lim), np.int32)
    copied = C.c_int32(-2)
    check(lib().pfk_bounded_wait_mixed_test(_iptr(lim), len(lim), _iptr(out), C.byref(copied)))
    return out, copied.value


def rank_sort(keys, m, ppt=0):
    """pfk_rank_sort: (sorted keys, permutation, sub-filters that fell back to the full network)."""
    k = np.array(keys, dtype=np.float32, copy=True)
    idx = np.zeros(len(k), np.int32)
    fb = C.c_int32(-1)
    check(lib().pfk_rank_sort(_fptr(k), _iptr(idx), m, len(k) // m, ppt, C.byref(fb)))
    return k, idx, fb.value


def bitonic_sort(keys, m, ppt=0):
    k = np.array(keys, dtype=np.float32, copy=True)
    idx = np.zeros(len(k), np.int32)
    check(lib().pfk_bitonic_sort(_fptr(k), _iptr(idx), m, len(k) // m, ppt))
    return k, idx


def resample(resampler, w, u, m, ppt=0):
    w = _f32(w)
    u = _f32(u)
    sel = np.zeros(len(w), np.int32)
    check(lib().pfk_resample(resampler, _fptr(w), _fptr(u), m, len(w) // m, ppt, _iptr(sel)))
    return sel


def vose_build(w, m, ppt=0):
    w = _f32(w)
    prob = np.zeros(len(w), np.float32)
    alias = np.zeros(len(w), np.uint32)
    check(lib().pfk_vose_build(_fptr(w), m, len(w) // m, ppt, _fptr(prob), _uptr(alias)))
    return prob, alias


def exchange_sources(mode, N, m, t, sorted_keys=None):
    src = np.zeros(N * m, np.int32)
    k = None if sorted_keys is None else _f32(sorted_keys)
    check(lib().pfk_exchange_sources(mode, N, m, t, None if k is None else _fptr(k), _iptr(src)))
    return src


def estimate(keys, state, m, angle_mask=0, log_weights=1):
    """Posterior estimate of SoA particles (pfk_estimate) as an ESTIMATE_DTYPE record."""
    k = _f32(keys)
    st = _f32(state)
    e = Estimate()
    check(lib().pfk_estimate(_fptr(k), _fptr(st), st.shape[0], len(k), m, angle_mask, log_weights, C.byref(e)))
    return estimate_to_numpy(e)


def estimate_noalloc(d_keys, d_state, num_state, num_particles, m, d_out, angle_mask=0, log_weights=1,
                     stream=None):
    """pfk_estimate_noalloc on device pointers (ints); asynchronous on `stream`."""
    check(lib().pfk_estimate_noalloc(C.c_void_p(d_keys), C.c_void_p(d_state), num_state, num_particles, m,
                                     angle_mask, log_weights, C.c_void_p(d_out), C.c_void_p(stream)))


def model_step(model, params, inp, state, noise):
    st = np.array(state, dtype=np.float32, copy=True)
    nz = _f32(noise)
    n = st.shape[1]
    ll = np.zeros(n, np.float32)
    s = inp if isinstance(inp, StepInput) else step_input(inp)
    check(lib().pfk_model_step(model, C.byref(params), C.sizeof(params), C.byref(s), n, _fptr(st), _fptr(nz),
                               _fptr(ll)))
    return st, ll
