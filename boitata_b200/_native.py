"""ctypes binding of the engine's C ABI (include/boitata_b200.h).

The shared library is built in-tree (boitata_b200/_lib/libboitata_b200.so)
by boitata_b200/build.py. There is no CPU fallback: a missing library or a
missing CUDA device raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libboitata_b200.so")

OK, EINVAL, EUNSUPPORTED, ECUDA, ENOTFITTED, ENOMEM = 0, -1, -2, -3, -4, -5
ST_OK, ST_SEARCH_FAILED, ST_SINGULAR, ST_UNSUPPORTED, ST_INVALID, ST_FP64_FALLBACK = 0, 1, 2, 3, 4, 0x10
MODELS = {
    "spherical": 0, "exponential": 1, "gaussian": 2, "cubic": 3, "pentaspherical": 4,
    "circular": 5, "sinehole": 6, "matern": 7, "power": 8,
}
ORDINARY, SIMPLE, INDICATOR = 0, 1, 2
FP64, MIXED = 0, 1


class Aniso(ctypes.Structure):
    _fields_ = [("on", ctypes.c_int32), ("azimuth", ctypes.c_double), ("dip", ctypes.c_double),
                ("rake", ctypes.c_double), ("major", ctypes.c_double), ("semi", ctypes.c_double),
                ("minor", ctypes.c_double)]


class StructureC(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int32), ("param", ctypes.c_double), ("sill", ctypes.c_double),
                ("range", ctypes.c_double)]


class VariogramC(ctypes.Structure):
    _fields_ = [("nugget", ctypes.c_double), ("nstruct", ctypes.c_int32), ("s", StructureC * 4), ("aniso", Aniso)]


class SearchC(ctypes.Structure):
    _fields_ = [("min_samples", ctypes.c_int64), ("max_samples", ctypes.c_int64), ("radius", ctypes.c_double),
                ("max_per_hole", ctypes.c_int64), ("octant", ctypes.c_int64), ("sectors", ctypes.c_int64),
                ("max_per_sector", ctypes.c_int64), ("max_per_octant", ctypes.c_int64),
                ("min_sectors", ctypes.c_int64), ("max_empty_sectors", ctypes.c_int64),
                ("min_holes", ctypes.c_int64), ("aniso", Aniso), ("calibration", ctypes.c_int64),
                ("calibration_target", ctypes.c_double)]


class GeometryC(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_double * 3), ("size", ctypes.c_double * 3), ("count", ctypes.c_int64 * 3),
                ("rotation", ctypes.c_double * 3)]


class TuningC(ctypes.Structure):
    _fields_ = [("samples_per_cell", ctypes.c_double), ("tile", ctypes.c_int32 * 3), ("search_warps", ctypes.c_int32),
                ("solve_blocks_per_sm", ctypes.c_int32), ("tile_union", ctypes.c_int32),
                ("host_chunk", ctypes.c_int32), ("tile_tensor", ctypes.c_int32),
                ("mixed_large", ctypes.c_int32)]


class OutputsC(ctypes.Structure):
    _fields_ = [("value", ctypes.c_void_p), ("variance", ctypes.c_void_p), ("lagrange", ctypes.c_void_p),
                ("n_used", ctypes.c_void_p), ("status", ctypes.c_void_p)]


class DiagnosticsC(ctypes.Structure):
    _fields_ = [("negative_weight_sum", ctypes.c_void_p), ("mean_distance", ctypes.c_void_p),
                ("n_holes", ctypes.c_void_p), ("target_met", ctypes.c_void_p)]


P = ctypes.c_void_p
SIGNATURES = {
    "btk_version": (ctypes.c_char_p, []),
    "btk_create": (P, [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    "btk_destroy": (None, [P]),
    "btk_last_error": (ctypes.c_char_p, [P]),
    "btk_fit": (ctypes.c_int, [P, ctypes.c_int64, P, P, P, P, ctypes.POINTER(SearchC), ctypes.POINTER(VariogramC)]),
    "btk_set_search": (ctypes.c_int, [P, ctypes.POINTER(SearchC)]),
    "btk_predict": (ctypes.c_int, [P, ctypes.c_int64, P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                   ctypes.POINTER(OutputsC)]),
    "btk_predict_device": (ctypes.c_int, [P, ctypes.c_int64, P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                          ctypes.POINTER(OutputsC), P]),
    "btk_predict_geometry_device": (ctypes.c_int, [P, ctypes.POINTER(GeometryC), ctypes.c_int32, ctypes.c_double,
                                                   ctypes.c_int32, ctypes.POINTER(OutputsC), P]),
    "btk_predict_kinds": (ctypes.c_int, [P, ctypes.c_int64, P, P, ctypes.c_double, ctypes.c_int32,
                                         ctypes.POINTER(OutputsC)]),
    "btk_sgs_simulate": (ctypes.c_int, [P, ctypes.c_int64, P, ctypes.c_int64, P, P, P]),
    "btk_predict_diagnostics": (ctypes.c_int, [P, ctypes.c_int64, P, ctypes.c_int32, ctypes.c_double,
                                               ctypes.c_int32, ctypes.POINTER(OutputsC),
                                               ctypes.POINTER(DiagnosticsC)]),
    "btk_predict_kinds_device": (ctypes.c_int, [P, ctypes.c_int64, P, P, ctypes.c_double, ctypes.c_int32,
                                                ctypes.POINTER(OutputsC), P]),
    "btk_cross_validate": (ctypes.c_int, [P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                          ctypes.POINTER(OutputsC)]),
    "btk_neighbors": (ctypes.c_int, [P, ctypes.c_int64, P, ctypes.c_int32, P, P, P, P]),
    "btk_set_domains": (ctypes.c_int, [P, P]),
    "btk_predict_ex": (ctypes.c_int, [P, ctypes.c_int64, P, P, P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                      ctypes.POINTER(OutputsC), P]),
    "btk_predict_ex_device": (ctypes.c_int, [P, ctypes.c_int64, P, P, P, ctypes.c_int32, ctypes.c_double,
                                             ctypes.c_int32, ctypes.POINTER(OutputsC), P]),
    "btk_predict_weights": (ctypes.c_int, [P, ctypes.c_int64, P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, P,
                                           ctypes.POINTER(OutputsC), P, P]),
    "btk_centroids": (ctypes.c_int, [P, ctypes.POINTER(GeometryC), ctypes.c_int64, ctypes.c_int64, P]),
    "btk_launch_count": (ctypes.c_int64, [P]),
    "btk_set_support": (ctypes.c_int, [P, P, P, P]),
    "btk_support_variance": (ctypes.c_int, [P, P]),
    "btk_get_tuning": (ctypes.c_int, [P, ctypes.POINTER(TuningC)]),
    "btk_set_tuning": (ctypes.c_int, [P, ctypes.POINTER(TuningC)]),
    "btk_graph_capture_geometry": (ctypes.c_int, [P, ctypes.POINTER(GeometryC), ctypes.c_int32, ctypes.c_double,
                                                  ctypes.c_int32, ctypes.POINTER(OutputsC)]),
    "btk_graph_capture_device": (ctypes.c_int, [P, ctypes.c_int64, P, P, ctypes.c_int32, ctypes.c_double,
                                                ctypes.c_int32, ctypes.POINTER(OutputsC)]),
    "btk_graph_launch": (ctypes.c_int, [P, P]),
    "btk_set_timing": (ctypes.c_int, [P, ctypes.c_int32]),
    "btk_phase_ms": (ctypes.c_int, [P, P]),
    "btk_peak_flops": (ctypes.c_double, [P, ctypes.c_int32]),
    "btk_loo_freeze": (ctypes.c_int, [P]),
    "btk_loo_gradient": (ctypes.c_int, [P, ctypes.POINTER(VariogramC), ctypes.c_int32, ctypes.c_int32, P, P, P, P]),
    "btk_loo_gradient_range": (ctypes.c_int, [P, ctypes.POINTER(VariogramC), ctypes.c_int64, ctypes.c_int64,
                                              ctypes.c_int32, ctypes.c_int32, P]),
    "btk_mean_freeze": (ctypes.c_int, [P, ctypes.POINTER(GeometryC)]),
    "btk_mean_gradient": (ctypes.c_int, [P, ctypes.POINTER(VariogramC), ctypes.c_int32, ctypes.c_int32, P, P, P,
                                         P]),
    "btk_mean_gradient_range": (ctypes.c_int, [P, ctypes.POINTER(VariogramC), ctypes.c_int64, ctypes.c_int64,
                                               ctypes.c_int32, ctypes.c_int32, P]),
    "btk_solve_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(VariogramC), ctypes.c_int32, ctypes.c_double,
                                         P, P, P, P, P, ctypes.c_int64, ctypes.c_int64, P, P, P, P, ctypes.c_int32,
                                         P, P,
                                         ctypes.POINTER(OutputsC), P, ctypes.c_char_p, ctypes.c_size_t]),
}

_lib = None


def library():
    """The loaded engine library; raises ImportError when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"boitata_b200: the CUDA engine {LIB_PATH} is not built; run "
                "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class EngineError(RuntimeError):
    """A failure reported by the CUDA engine."""


class Context:
    """One engine context (device buffers and a CUDA stream) on `device`."""

    def __init__(self, device=0):
        lib = library()
        err = ctypes.create_string_buffer(512)
        self._lib = lib
        self._h = lib.btk_create(int(device), err, len(err))
        if not self._h:
            raise EngineError("boitata_b200 needs a CUDA device: " + err.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.btk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def error(self):
        return self._lib.btk_last_error(self._h).decode()

    def check(self, rc, what):
        if rc == OK:
            return
        from .errors import InvalidInput, Unsupported

        msg = f"{what}: {self.error()}"
        if rc == EINVAL:
            raise InvalidInput(msg)
        if rc == EUNSUPPORTED:
            raise Unsupported(msg)
        raise EngineError(msg)

    def launches(self):
        return int(self._lib.btk_launch_count(self._h))
