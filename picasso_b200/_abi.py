"""ctypes mirror of include/picasso_b200.h and the loader of the CUDA library.

The structures here must match the C header field for field; a CPU test
compiles a small C program that prints sizeof/offsetof of every descriptor
and compares it with these definitions.
"""

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpicasso_b200.so")

# status codes
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_OUT_OF_RANGE = 4
ERR_TIMEOUT = 5
ERR_NO_DEVICE = 6

# dtypes
F64 = 0
F32 = 1
I64_FIXED = 2

# locations
NODE = 0
CELL = 1
FACE_I, FACE_J, FACE_K = 2, 3, 4
EDGE_I, EDGE_J, EDGE_K = 5, 6, 7

SOA_SHIFT = 62


class Mesh(C.Structure):
    _fields_ = [("extent", C.c_int32 * 3), ("own_begin", C.c_int32 * 3),
                ("own_extent", C.c_int32 * 3), ("periodic", C.c_int32 * 3),
                ("low_corner", C.c_double * 3), ("cell_size", C.c_double * 3)]


class Spline(C.Structure):
    _fields_ = [("mesh", Mesh), ("location", C.c_int32), ("order", C.c_int32)]


class ParticleField(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32), ("vector_shift", C.c_int32),
                ("tile_stride", C.c_int64), ("comp_stride", C.c_int64)]


class GridField(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32), ("fixed_bits", C.c_int32),
                ("stride", C.c_int64 * 4)]


class Bins(C.Structure):
    _fields_ = [("tile", C.c_int32 * 3), ("num_tiles", C.c_int32 * 3),
                ("bin_extent", C.c_int32 * 3), ("order", C.c_int32), ("location", C.c_int32),
                ("chunk", C.c_int32), ("p2g_lanes", C.c_int32), ("tile_offset", C.c_void_p),
                ("tile_items", C.c_void_p), ("records", C.c_void_p)]


class Exec(C.Structure):
    _fields_ = [("stream", C.c_void_p), ("error_count", C.c_void_p),
                ("bins", C.POINTER(Bins)), ("overflow_count", C.c_void_p)]


class HaloPeers(C.Structure):
    _fields_ = [("lo_end", C.c_int32), ("hi_begin", C.c_int32), ("lo_shift", C.c_int32),
                ("hi_shift", C.c_int32), ("lo", C.c_void_p * 2), ("hi", C.c_void_p * 2)]


class GridUpdateParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double * 3), ("mass_threshold", C.c_double),
                ("wall", (C.c_int32 * 2) * 3), ("wall_width", C.c_int32)]


WALL_NONE, WALL_NO_SLIP, WALL_FREE_SLIP = 0, 1, 2


class BatchInstance(C.Structure):
    _fields_ = [("spline", Spline), ("num_particles", C.c_int64), ("x_p", ParticleField),
                ("m_p", ParticleField), ("c_p", ParticleField), ("m_i", GridField),
                ("mu_i", GridField), ("u_i", GridField), ("mass_threshold", C.c_double),
                ("bins", Bins), ("error_count", C.c_void_p)]


class BatchInfo(C.Structure):
    _fields_ = [("count", C.c_int32), ("precision_form", C.c_int32),
                ("grid_blocks", C.c_int32), ("smem_bytes", C.c_int32),
                ("items", C.c_int64 * 4), ("particles", C.c_int64)]


BATCH_FUSED, BATCH_PHASED = 0, 1


class TuneResult(C.Structure):
    _fields_ = [("tile", C.c_int32 * 3), ("chunk", C.c_int32), ("p2g_lanes", C.c_int32),
                ("step_ms", C.c_float)]

# (name, restype, argtypes) of every entry point in the header
SIGNATURES = [
    ("picasso_version", C.c_char_p, []),
    ("picasso_status_string", C.c_char_p, [C.c_int]),
    ("picasso_last_cuda_error", C.c_char_p, []),
    ("picasso_apic_p2g", C.c_int,
     [C.POINTER(Spline), C.c_int64, C.c_int32, ParticleField, ParticleField, ParticleField,
      GridField, GridField, C.POINTER(Exec)]),
    ("picasso_apic_g2p", C.c_int,
     [C.POINTER(Spline), C.c_int64, C.c_int32, ParticleField, GridField, ParticleField,
      C.POINTER(Exec)]),
    ("picasso_polypic_p2g", C.c_int,
     [C.POINTER(Spline), C.c_int64, C.c_int32, ParticleField, ParticleField, ParticleField,
      ParticleField, GridField, GridField, C.c_double, C.POINTER(Exec)]),
    ("picasso_polypic_g2p", C.c_int,
     [C.POINTER(Spline), C.c_int64, C.c_int32, ParticleField, GridField, ParticleField,
      C.POINTER(Exec)]),
    ("picasso_grid_fill", C.c_int,
     [C.POINTER(Mesh), C.c_int32, GridField, C.c_double, C.POINTER(Exec)]),
    ("picasso_grid_velocity", C.c_int,
     [C.POINTER(Mesh), C.c_int32, GridField, GridField, C.c_double, GridField, GridField,
      C.POINTER(Exec)]),
    ("picasso_grid_update", C.c_int,
     [C.POINTER(Mesh), GridField, GridField, GridField, C.POINTER(GridUpdateParams), GridField,
      GridField, C.POINTER(Exec)]),
    ("picasso_apic_p2g_halo", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, ParticleField, ParticleField, GridField,
      GridField, C.POINTER(HaloPeers), C.POINTER(Exec)]),
    ("picasso_apic_g2p_halo", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, GridField, ParticleField,
      C.POINTER(HaloPeers), C.POINTER(Exec)]),
    ("picasso_apic_p2g_update_workspace", C.c_int, [C.POINTER(Bins), C.POINTER(C.c_int64)]),
    ("picasso_apic_p2g_update", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, ParticleField, ParticleField, GridField,
      GridField, GridField, C.POINTER(GridUpdateParams), GridField, GridField, C.c_void_p,
      C.c_int64, C.POINTER(Exec)]),
    ("picasso_advect", C.c_int,
     [C.POINTER(Mesh), C.c_int64, C.c_double, ParticleField, ParticleField, C.POINTER(Exec)]),
    ("picasso_apic_g2p_advect", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, GridField, ParticleField, C.c_double,
      C.POINTER(Exec)]),
    ("picasso_apic_g2p_advect_keys", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, GridField, ParticleField, C.c_double,
      C.POINTER(C.c_int32), C.c_void_p, C.POINTER(Exec)]),
    ("picasso_cell_sort_workspace", C.c_int,
     [C.POINTER(Spline), C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    ("picasso_cell_sort", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, C.POINTER(C.c_int32), C.c_int32, C.c_void_p,
      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(Bins),
      C.POINTER(Exec)]),
    ("picasso_cell_sort_keys", C.c_int,
     [C.POINTER(Spline), C.c_int64, C.c_void_p, C.POINTER(C.c_int32), C.c_int32, C.c_void_p,
      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(Bins),
      C.POINTER(Exec)]),
    ("picasso_cell_sort_static", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, C.POINTER(C.c_int32), C.c_int32, C.c_void_p,
      C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Bins), C.POINTER(Exec)]),
    ("picasso_autotune", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, ParticleField, ParticleField, GridField,
      GridField, GridField, C.c_double, C.c_int32, C.POINTER(TuneResult), C.POINTER(Exec)]),
    ("picasso_permute", C.c_int,
     [C.c_int64, C.c_int32, C.c_void_p, ParticleField, ParticleField, C.POINTER(Exec)]),
    ("picasso_mat3_inverse", C.c_int,
     [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
      C.POINTER(Exec)]),
    ("picasso_spline_records", C.c_int,
     [C.POINTER(Spline), C.c_int64, ParticleField, C.POINTER(Bins), C.c_void_p,
      C.POINTER(Exec)]),
    ("picasso_batch_create", C.c_int,
     [C.POINTER(BatchInstance), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    ("picasso_batch_step", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    ("picasso_batch_step_sequential", C.c_int, [C.c_void_p, C.c_void_p]),
    ("picasso_batch_status", C.c_int, [C.c_void_p, C.c_void_p]),
    ("picasso_batch_set_wait_limit", C.c_int, [C.c_void_p, C.c_uint32]),
    ("picasso_batch_cancel", C.c_int, [C.c_void_p, C.c_void_p]),
    ("picasso_batch_get_info", C.c_int, [C.c_void_p, C.POINTER(BatchInfo)]),
    ("picasso_batch_destroy", C.c_int, [C.c_void_p]),
]

_lib = None


class PicassoError(RuntimeError):
    """A C-ABI entry point returned a non-zero status."""

    def __init__(self, status, where):
        lib = _lib
        msg = lib.picasso_status_string(status).decode() if lib else str(status)
        if status == ERR_CUDA and lib:
            msg += ": " + lib.picasso_last_cuda_error().decode()
        super().__init__("%s failed: %s (status %d)" % (where, msg, status))
        self.status = status


def load_library(path=None):
    """Load libpicasso_b200.so (built in-tree by picasso_b200._build).

    Raises ImportError when the library has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError("libpicasso_b200.so not built (%s); run picasso_b200._build.build()" % p)
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status, where):
    if status != OK:
        raise PicassoError(status, where)
