"""ctypes binding of libppt.so (the C ABI declared in include/ppt.h).

The library is the only compute path: if it is missing or fails to load,
importing the GPU entry points raises instead of falling back to the CPU.
"""
import ctypes
import os
from ctypes import c_uint32, c_double, c_int, c_int32, c_int64, c_void_p, POINTER
from pathlib import Path

LIB_PATH = Path(os.environ.get("PPT_LIBRARY", Path(__file__).resolve().parent / "lib" / "libppt.so"))

PPT_OK = 0
ERRORS = {-1: "PPT_ERR_ARG", -2: "PPT_ERR_OOM", -3: "PPT_ERR_CUDA", -4: "PPT_ERR_UNSUPPORTED",
          -5: "PPT_ERR_TIMEOUT", -6: "PPT_ERR_DEVICE"}

ALG_IDS = {"leapfrog": 0, "boris": 1, "rk4": 2, "yoshida": 3, "vay_rel": 4, "rk4_rel": 5,
           "yoshida_rel": 6, "boris_rel": 7, "vay": 8}
ABI_VERSION = 4
PREC_F64, PREC_MIXED = 0, 1
DTYPE_F64, DTYPE_F32 = 0, 1
TRACK_INIT, TRACK_FINAL = 1, 2
STATUS_NONFINITE, STATUS_BOUNDS, STATUS_RANGE = 1, 2, 4
MAX_MAPS = 4
COMP_BITS = {"ex": 0x01, "ey": 0x02, "ez": 0x04, "bx": 0x08, "by": 0x10, "bz": 0x20}
FULL_MASK = 0x3F
MOMENTS_LEN = 22


class PptError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class PptUnsupported(PptError, NotImplementedError):
    pass


class GridDesc(ctypes.Structure):
    _fields_ = [("n", c_int64 * 3), ("axis", c_void_p * 3)]


class Fields(ctypes.Structure):
    _fields_ = [("maps", c_void_p * MAX_MAPS), ("n_maps", c_int32),
                ("e_const", c_double * 3), ("b_const", c_double * 3)]


class State(ctypes.Structure):
    _fields_ = [("precision", c_int32), ("algorithm", c_int32), ("n", c_int64),
                ("f64", c_void_p), ("i32", c_void_p), ("f32", c_void_p)]


class TrackArgs(ctypes.Structure):
    _fields_ = [("step0", c_int64), ("nsteps", c_int64), ("nsteps_total", c_int64),
                ("rec_every", c_int64), ("flags", c_int32), ("reserved", c_int32),
                ("dt", c_double), ("q_over_m", c_double), ("t0", c_double),
                ("rf_omega", c_double), ("rf_phase", c_void_p), ("r_hist", c_void_p),
                ("v_hist", c_void_p), ("order", c_void_p), ("status", c_void_p),
                ("counters", c_void_p), ("surface", c_void_p), ("active", c_void_p),
                ("dt_rows", c_void_p)]


class JobDesc(ctypes.Structure):
    _fields_ = [("state", State), ("fields", Fields), ("nsteps_total", c_int64), ("rec_every", c_int64),
                ("dt", c_double), ("q_over_m", c_double), ("t0", c_double), ("rf_omega", c_double),
                ("rf_phase", c_void_p), ("r_hist", c_void_p), ("v_hist", c_void_p), ("status", c_void_p),
                ("steps_done", c_int64), ("tick_steps", c_int64)]


# name -> (restype, argtypes); every symbol include/ppt.h declares
class PolarGrid(ctypes.Structure):
    _fields_ = [("nr", c_int64), ("nt", c_int64), ("r", c_void_p), ("theta", c_void_p)]


class MeshDesc(ctypes.Structure):
    _fields_ = [("extent", c_double * 3), ("cells", c_int64 * 3)]


SIGNATURES = {
    "ppt_fieldmap_create": (c_int, [POINTER(GridDesc), c_int, c_int, c_int, POINTER(c_void_p)]),
    "ppt_fieldmap_layout": (c_int, [c_uint32]),
    "ppt_deposit_cic": (c_int, [c_int64, c_void_p, c_void_p, POINTER(MeshDesc), c_void_p, c_void_p]),
    "ppt_polar_to_cartesian": (c_int, [POINTER(PolarGrid), POINTER(c_void_p * 3), c_int64, c_void_p, c_int64,
                                       c_void_p, c_double, POINTER(c_void_p * 3), c_void_p]),
    "ppt_poisson_scratch_bytes": (c_int64, [POINTER(MeshDesc)]),
    "ppt_poisson_solve": (c_int, [POINTER(MeshDesc), c_void_p, c_void_p, c_void_p, c_double, c_int64,
                                  POINTER(c_int64), POINTER(c_double), c_void_p]),
    "ppt_poisson_coef_scratch_bytes": (c_int64, [POINTER(MeshDesc)]),
    "ppt_poisson_solve_coef": (c_int, [POINTER(MeshDesc), c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                                       c_int64, POINTER(c_int64), POINTER(c_double), c_void_p]),
    "ppt_field_from_potential": (c_int, [POINTER(MeshDesc), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_surface_create": (c_int, [c_int64, c_void_p, c_int64, c_void_p, POINTER(c_void_p)]),
    "ppt_surface_destroy": (c_int, [c_void_p]),
    "ppt_surface_info": (c_int, [c_void_p, POINTER(c_int64), POINTER(c_int32)]),
    "ppt_surface_axis_rays": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_surface_segments_hit": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_fieldmap_create_masked": (c_int, [POINTER(GridDesc), c_uint32, c_int, POINTER(c_void_p)]),
    "ppt_fieldmap_add": (c_int, [c_void_p, POINTER(c_void_p * 6), POINTER(c_double * 6), c_int, c_void_p]),
    "ppt_fieldmap_destroy": (c_int, [c_void_p]),
    "ppt_fieldmap_info": (c_int, [c_void_p, POINTER(c_int64), POINTER(c_int)]),
    "ppt_field_eval": (c_int, [POINTER(Fields), c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_state_load": (c_int, [POINTER(State), POINTER(Fields), c_void_p, c_void_p, c_void_p]),
    "ppt_state_store": (c_int, [POINTER(State), POINTER(Fields), c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_track": (c_int, [POINTER(State), POINTER(Fields), POINTER(TrackArgs), c_void_p]),
    "ppt_cell_sort_scratch_bytes": (c_int64, [c_int64]),
    "ppt_cell_sort": (c_int, [POINTER(State), POINTER(Fields), c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_restore_order": (c_int, [POINTER(State), c_void_p, c_void_p, c_void_p, c_void_p]),
    "ppt_moments_scratch_bytes": (c_int64, [c_int64]),
    "ppt_moments": (c_int, [c_int64, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p]),
    "ppt_moments_noalloc": (c_int, [c_int64, c_void_p, c_void_p, c_double, c_void_p, c_void_p]),
    "ppt_jobs_scratch_bytes": (c_int64, [c_int]),
    "ppt_jobs_create": (c_int, [POINTER(JobDesc), c_int, c_void_p, POINTER(c_void_p), c_void_p]),
    "ppt_jobs_tick": (c_int, [c_void_p, c_int64, c_void_p]),
    "ppt_jobs_progress": (c_int, [c_void_p, POINTER(c_void_p), POINTER(c_void_p)]),
    "ppt_jobs_destroy": (c_int, [c_void_p]),
    "ppt_last_error": (ctypes.c_char_p, []),
    "ppt_abi_version": (c_int, []),
}

_lib = None


def load():
    """Load libppt.so once; raise loudly when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pypatools_b200.build` "
                          "(there is no CPU fallback for the pusher path)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ppt_abi_version() != ABI_VERSION:
        raise ImportError("libppt.so ABI version mismatch; rebuild it")
    _lib = lib
    return lib


def check(rc):
    if rc != PPT_OK:
        msg = load().ppt_last_error().decode("utf-8", "replace")
        if rc == -4:
            raise PptUnsupported(rc, msg)
        raise PptError(rc, msg)
    return rc


def stream_handle(stream=None):
    """cudaStream_t of a torch stream (current stream by default) as int."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
