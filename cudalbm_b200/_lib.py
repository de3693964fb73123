"""ctypes binding of liblbm_b200.so (the C ABI declared in include/lbm_b200.h).

The library is built in-tree by ``cudalbm_b200/build.py`` into
``cudalbm_b200/lib/liblbm_b200.so``.  Importing this module without the built
library raises immediately: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# LBM_B200_LIBRARY selects another build of the same library (A/B timing of
# kernel variants); the default is the in-tree build.
LIB_PATH = os.environ.get("LBM_B200_LIBRARY") or os.path.join(HERE, "lib", "liblbm_b200.so")

LBM_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "device wait timed out",
          5: "I/O error", 6: "parse error", 7: "invalid state", 8: "non-finite value in solution"}

FO_S, FO_SMEAN, FO_K, FO_KMEAN, FO_MOMENTSMEAN = 1, 2, 4, 8, 16
FO_BITS = {"S": FO_S, "SMean": FO_SMEAN, "k": FO_K, "kMean": FO_KMEAN, "momentsMean": FO_MOMENTSMEAN}

FIELDS_MOMENTS, FIELDS_S, FIELDS_SMEAN, FIELDS_K, FIELDS_KMEAN, FIELDS_MOMENTSMEAN = range(6)
FIELD_SET = {"moments": 0, "S": 1, "SMean": 2, "k": 3, "kMean": 4, "momentsMean": 5}
ORDER_GLOBAL, ORDER_TILED = 0, 1
F32, F64 = 0, 1

# every symbol include/lbm_b200.h declares
EXPORTS = ("lbm_config_default", "lbm_create", "lbm_destroy", "lbm_init_regions", "lbm_write_fields",
           "lbm_read_fields", "lbm_step", "lbm_synchronize", "lbm_reduce", "lbm_get_info", "lbm_last_error",
           "lbm_status_string", "lbm_field_set_vars", "lbm_host_alloc", "lbm_host_free", "lbm_case_read",
           "lbm_lbmbin_write", "lbm_reduce_moments_noalloc", "lbm_step_monitored", "lbm_run_streamed",
           "lbm_autotune", "lbm_batch_create", "lbm_batch_destroy", "lbm_batch_cavity", "lbm_batch_step", "lbm_batch_synchronize",
           "lbm_batch_autotune", "lbm_batch_get_info", "lbm_batch_configure", "lbm_cut_plane",
           "lbm_vts_write", "lbm_perturb_velocity", "lbm_filter_2to1", "lbm_trainer_create", "lbm_trainer_destroy",
           "lbm_trainer_add", "lbm_trainer_add_window", "lbm_trainer_samples", "lbm_trainer_fit",
           "lbm_trainer_gradient", "lbm_mlp_infer",
           "lbm_closure_set", "lbm_closure_dtau", "lbm_closure_refresh", "lbm_closure_fused",
           "lbm_selftest_wait_timeout", "lbm_field_statistics")


class Config(ctypes.Structure):
    _fields_ = [("lattice", ctypes.c_int32), ("device", ctypes.c_int32), ("nx", ctypes.c_int64),
                ("ny", ctypes.c_int64), ("nz", ctypes.c_int64), ("Re", ctypes.c_float), ("u_inf", ctypes.c_float),
                ("function_objects", ctypes.c_uint32), ("mean_bits", ctypes.c_int32),
                ("start_step", ctypes.c_int64), ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32),
                ("z_chunk", ctypes.c_int32), ("stages", ctypes.c_int32), ("pop_buffers", ctypes.c_int32),
                ("storage", ctypes.c_int32)]


STORAGE = {"f32": 0, "f16": 1, "bf16": 2}


class Info(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int64), ("nodes", ctypes.c_int64), ("tau", ctypes.c_float),
                ("omega", ctypes.c_float), ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32),
                ("z_chunk", ctypes.c_int32), ("stages", ctypes.c_int32), ("device_bytes", ctypes.c_uint64),
                ("last_step_ms", ctypes.c_double), ("kernel_launches", ctypes.c_uint64)]


class Tuning(ctypes.Structure):
    _fields_ = [("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32), ("z_chunk", ctypes.c_int32),
                ("stages", ctypes.c_int32), ("pop_buffers", ctypes.c_int32), ("ms_per_step", ctypes.c_double),
                ("candidates", ctypes.c_int32), ("from_cache", ctypes.c_int32), ("closure_fused", ctypes.c_int32)]


class StreamOpts(ctypes.Structure):
    _fields_ = [("slab", ctypes.c_int32), ("z_chunk", ctypes.c_int32), ("lead", ctypes.c_int32)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("cavities", ctypes.c_int32), ("items", ctypes.c_int32), ("grid", ctypes.c_int32),
                ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32), ("stages", ctypes.c_int32),
                ("pop_buffers", ctypes.c_int32), ("persistent", ctypes.c_int32), ("nodes", ctypes.c_int64),
                ("step", ctypes.c_int64),
                ("device_bytes", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
                ("graph_launches", ctypes.c_uint64), ("last_step_ms", ctypes.c_double)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32), ("stages", ctypes.c_int32),
                ("pop_buffers", ctypes.c_int32), ("persistent", ctypes.c_int32), ("size_classes", ctypes.c_int32),
                ("candidates", ctypes.c_int32), ("ms_per_step", ctypes.c_double)]


class MLP(ctypes.Structure):
    _fields_ = [("w1", ctypes.c_float * 512), ("b1", ctypes.c_float * 32), ("w2", ctypes.c_float * 1024),
                ("b2", ctypes.c_float * 32), ("w3", ctypes.c_float * 32), ("b3", ctypes.c_float),
                ("in_mean", ctypes.c_float * 16), ("in_scale", ctypes.c_float * 16), ("in_lo", ctypes.c_float * 16),
                ("in_hi", ctypes.c_float * 16), ("out_scale", ctypes.c_float), ("dtau_lo", ctypes.c_float),
                ("dtau_hi", ctypes.c_float)]


class TrainOptions(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("dtau_lo", ctypes.c_float), ("dtau_hi", ctypes.c_float), ("seed", ctypes.c_uint64)]


class TrainReport(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_uint64), ("steps", ctypes.c_uint64), ("loss_first", ctypes.c_double),
                ("loss_last", ctypes.c_double), ("target_rms", ctypes.c_double)]


class Case(ctypes.Structure):
    _fields_ = [("case_name", ctypes.c_char * 256), ("Re", ctypes.c_float), ("u_inf", ctypes.c_float),
                ("n_time_steps", ctypes.c_uint64), ("save_interval", ctypes.c_uint64),
                ("info_interval", ctypes.c_uint64), ("nx", ctypes.c_uint64), ("ny", ctypes.c_uint64),
                ("nz", ctypes.c_uint64), ("Lx", ctypes.c_float), ("Ly", ctypes.c_float), ("Lz", ctypes.c_float),
                ("function_objects", ctypes.c_uint32), ("region", ctypes.c_float * 70),
                ("latest_time", ctypes.c_uint64), ("has_restart", ctypes.c_int32)]


MONITOR_DTYPE = [("mass", "<f8"), ("rho_u2", "<f8"), ("nonfinite", "<u8")]


class LBMError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m cudalbm_b200.build` (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, u64, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint64, ctypes.c_size_t
        L.lbm_config_default.argtypes = [ctypes.POINTER(Config)]
        L.lbm_config_default.restype = None
        L.lbm_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
        L.lbm_destroy.argtypes = [vp]
        L.lbm_init_regions.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
        L.lbm_write_fields.argtypes = [vp, i32, vp, sz, i32, i32]
        L.lbm_read_fields.argtypes = [vp, i32, vp, sz, i32, i32]
        L.lbm_step.argtypes = [vp, u64]
        L.lbm_synchronize.argtypes = [vp]
        L.lbm_reduce.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.lbm_get_info.argtypes = [vp, ctypes.POINTER(Info)]
        L.lbm_last_error.restype = ctypes.c_char_p
        L.lbm_status_string.restype = ctypes.c_char_p
        L.lbm_status_string.argtypes = [i32]
        L.lbm_field_set_vars.argtypes = [i32]
        L.lbm_host_alloc.argtypes = [sz, ctypes.POINTER(vp)]
        L.lbm_host_free.argtypes = [vp]
        L.lbm_case_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(Case)]
        L.lbm_reduce_moments_noalloc.argtypes = [vp, u64, ctypes.POINTER(ctypes.c_double), vp]
        L.lbm_step_monitored.argtypes = [vp, u64, vp]
        L.lbm_run_streamed.argtypes = [vp, vp, u64, ctypes.POINTER(vp), vp, ctypes.POINTER(StreamOpts)]
        L.lbm_autotune.argtypes = [vp, i32, ctypes.POINTER(Tuning)]
        L.lbm_batch_create.argtypes = [ctypes.POINTER(Config), i32, ctypes.POINTER(vp)]
        L.lbm_batch_destroy.argtypes = [vp]
        L.lbm_batch_cavity.argtypes = [vp, i32, ctypes.POINTER(vp)]
        L.lbm_batch_step.argtypes = [vp, u64]
        L.lbm_batch_synchronize.argtypes = [vp]
        L.lbm_batch_autotune.argtypes = [vp, i32, ctypes.POINTER(BatchTuning)]
        L.lbm_batch_get_info.argtypes = [vp, ctypes.POINTER(BatchInfo)]
        L.lbm_batch_configure.argtypes = [vp, ctypes.POINTER(BatchTuning)]
        L.lbm_cut_plane.argtypes = [vp, i32, i32, ctypes.c_float, vp, sz]
        L.lbm_vts_write.argtypes = [ctypes.c_char_p, u64, u64, u64, ctypes.POINTER(ctypes.c_float), i32,
                                    ctypes.POINTER(ctypes.c_char_p), vp]
        L.lbm_perturb_velocity.argtypes = [vp, ctypes.c_float, u64]
        L.lbm_filter_2to1.argtypes = [vp, vp]
        L.lbm_trainer_create.argtypes = [i32, u64, ctypes.POINTER(vp)]
        L.lbm_trainer_destroy.argtypes = [vp]
        L.lbm_trainer_add.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_float, ctypes.POINTER(u64)]
        L.lbm_trainer_add_window.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                             ctypes.POINTER(u64)]
        L.lbm_trainer_samples.argtypes = [vp, u64, u64, vp, vp, ctypes.POINTER(u64)]
        L.lbm_trainer_fit.argtypes = [vp, ctypes.POINTER(TrainOptions), ctypes.POINTER(MLP), ctypes.POINTER(TrainReport)]
        L.lbm_trainer_gradient.argtypes = [vp, ctypes.POINTER(MLP), u64, u64, ctypes.POINTER(MLP),
                                           ctypes.POINTER(ctypes.c_double)]
        L.lbm_mlp_infer.argtypes = [i32, ctypes.POINTER(MLP), vp, u64, vp, i32]
        L.lbm_closure_set.argtypes = [vp, ctypes.POINTER(MLP)]
        L.lbm_closure_dtau.argtypes = [vp, vp, sz]
        L.lbm_closure_refresh.argtypes = [vp, i32]
        L.lbm_closure_fused.argtypes = [vp, i32]
        L.lbm_selftest_wait_timeout.argtypes = [i32, u64]
        L.lbm_field_statistics.argtypes = [i32, vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, i32, i32, vp, vp,
                                           vp]
        L.lbm_lbmbin_write.argtypes = [ctypes.c_char_p, u64, u64, u64, i32, ctypes.POINTER(ctypes.c_char_p), vp, u64,
                                       i32]
        for name in ("lbm_create", "lbm_destroy", "lbm_init_regions", "lbm_write_fields", "lbm_read_fields",
                     "lbm_step", "lbm_synchronize", "lbm_reduce", "lbm_get_info", "lbm_host_alloc", "lbm_host_free",
                     "lbm_case_read", "lbm_lbmbin_write", "lbm_reduce_moments_noalloc", "lbm_step_monitored",
                     "lbm_run_streamed", "lbm_autotune", "lbm_batch_create", "lbm_batch_destroy", "lbm_batch_cavity", "lbm_batch_step",
                     "lbm_batch_synchronize", "lbm_batch_autotune", "lbm_batch_get_info", "lbm_batch_configure",
                     "lbm_cut_plane", "lbm_vts_write", "lbm_perturb_velocity", "lbm_filter_2to1",
                     "lbm_trainer_create", "lbm_trainer_destroy", "lbm_trainer_add", "lbm_trainer_add_window", "lbm_trainer_samples",
                     "lbm_trainer_fit", "lbm_trainer_gradient", "lbm_mlp_infer", "lbm_closure_set",
                     "lbm_closure_dtau", "lbm_closure_refresh", "lbm_closure_fused", "lbm_selftest_wait_timeout",
                     "lbm_field_statistics"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != LBM_OK:
        raise LBMError(status, lib().lbm_last_error().decode(errors="replace"))


class PinnedArray:
    """numpy view of page-locked host memory from lbm_host_alloc."""

    def __init__(self, shape, dtype=None):
        import numpy as np

        dtype = np.dtype(dtype or np.float32)
        n = int(np.prod(shape)) * dtype.itemsize
        p = ctypes.c_void_p()
        check(lib().lbm_host_alloc(max(n, 1), ctypes.byref(p)))
        self._p = p
        buf = (ctypes.c_char * max(n, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self._p:
            self.array = None
            lib().lbm_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def read_case(directory: str) -> dict:
    """Parse a case directory with the library's reader (lbm_case_read)."""
    import numpy as np

    c = Case()
    check(lib().lbm_case_read(directory.encode(), ctypes.byref(c)))
    out = {f: getattr(c, f) for f, _ in Case._fields_ if f not in ("case_name", "region")}
    out["case_name"] = c.case_name.decode()
    out["region"] = np.ctypeslib.as_array(c.region).reshape(10, 7).copy()
    return out
