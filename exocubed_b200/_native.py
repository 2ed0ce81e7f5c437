"""ctypes binding of libexo_b200.so (the C ABI declared in include/exo_b200.h).

The shared library is built in-tree by exocubed_b200/csrc/Makefile.  Loading
fails loudly when it is missing: there is no CPU fallback for the product
path.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libexo_b200.so")

EXO_OK = 0
EXO_EQN_SHALLOW_YZ, EXO_EQN_IDEAL = 0, 1
(EXO_OK, EXO_ERR_ARG, EXO_ERR_SHAPE, EXO_ERR_CUDA, EXO_ERR_NONFINITE, EXO_ERR_TIMEOUT,
 EXO_ERR_NOGPU, EXO_ERR_CAPACITY) = range(8)
EXO_RS_ROE_SHALLOW, EXO_RS_LMARS, EXO_RS_HLLC, EXO_RS_LMARS_SHALLOW = 0, 1, 2, 3
EXO_PREC_FP64, EXO_PREC_MIXED, EXO_PREC_MIXED_F32_SOLVE = 0, 1, 2
EXO_CORIOLIS_NONE, EXO_CORIOLIS_W92, EXO_CORIOLIS_3D = 0, 1, 2
EXO_FORCING_NONE, EXO_FORCING_HS94 = 0, 1
NGHOST = 3
EXO_TILE_COUNT = 6
EXO_K_FLUX_X1, EXO_K_FLUX_X23, EXO_K_UPDATE, EXO_K_IMPLICIT, EXO_K_PRIM_GHOST, EXO_K_OTHER = range(6)
NOALLOC_SCRATCH_DOUBLES = 1048576  # EXO_NOALLOC_SCRATCH_DOUBLES

# every symbol include/exo_b200.h declares
EXPORTED = [
    "exo_config_default", "exo_create", "exo_destroy", "exo_cell_geometry", "exo_mesh",
    "exo_shape", "exo_last_error", "exo_set_primitive", "exo_get_conserved",
    "exo_get_primitive", "exo_device_state", "exo_step", "exo_get_dt",
    "exo_get_time", "exo_check_state", "exo_synchronize",
    "exo_calculate_fluxes", "exo_get_flux", "exo_riemann", "exo_weno5",
    "exo_get_stream", "exo_profile", "exo_profile_read", "exo_launch_count",
    "exo_ensemble_create", "exo_ensemble_destroy", "exo_ensemble_footprint",
    "exo_ensemble_add", "exo_ensemble_remove", "exo_ensemble_step",
    "exo_ensemble_synchronize", "exo_ensemble_get_conserved", "exo_ensemble_get_primitive",
    "exo_ensemble_member_time", "exo_ensemble_check_state", "exo_ensemble_stats",
    "exo_set_tiles", "exo_get_tiles", "exo_ensemble_set_tiles", "exo_ensemble_get_tiles",
    "exo_stage", "exo_boundary", "exo_solve_implicit_3d", "exo_change_to_perturbation",
    "exo_restore_from_perturbation",
    "exo_ensemble_get_stream",
    "exo_implicit_columns", "exo_partial_correction_columns", "exo_implicit_columns_noalloc",
    "exo_checkpoint_bytes", "exo_checkpoint_save", "exo_checkpoint_load",
    "exo_ensemble_checkpoint_bytes", "exo_ensemble_checkpoint_save",
    "exo_ensemble_add_checkpoint", "exo_set_max_redo", "exo_redo_count",
    "exo_measure_fma_peak",
    "exo_panel_pack", "exo_save_lr3d", "exo_load_lr3d", "exo_lr3d_arrays",
    "exo_synchronize_faces", "exo_conserved_to_primitive", "exo_primitive_to_conserved",
    "exo_sound_speed", "exo_set_primitive_views", "exo_get_primitive_views",
    "exo_get_conserved_views", "exo_solve_implicit_3d_views", "exo_check_bounded_wait",
    "exo_reciprocal",
]
EXO_DTYPE_F64 = 0
KERNELS = ["flux_x1", "flux_x23", "update", "implicit", "prim_ghost", "other"]


class ExoConfig(ctypes.Structure):
    """exo_config of include/exo_b200.h."""
    _fields_ = [
        ("N", ctypes.c_int), ("L", ctypes.c_int), ("eqn", ctypes.c_int),
        ("rsolver", ctypes.c_int), ("implicit_flag", ctypes.c_int),
        ("precision", ctypes.c_int), ("coriolis", ctypes.c_int),
        ("forcing", ctypes.c_int),
        ("x1min", ctypes.c_double), ("x1max", ctypes.c_double),
        ("gamma", ctypes.c_double), ("Rd", ctypes.c_double),
        ("grav", ctypes.c_double), ("cfl", ctypes.c_double),
        ("omega", ctypes.c_double), ("reserved1", ctypes.c_double),
        ("hs_p0", ctypes.c_double), ("hs_Ts", ctypes.c_double), ("hs_dT", ctypes.c_double),
        ("hs_dtheta", ctypes.c_double), ("hs_Kf", ctypes.c_double), ("hs_Ka", ctypes.c_double),
        ("hs_Ks", ctypes.c_double), ("hs_sigmab", ctypes.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ArrayView(ctypes.Structure):
    """exo_array_view of include/exo_b200.h: a strided (n, k, j, i) view."""
    _fields_ = [
        ("data", ctypes.c_void_p), ("dtype", ctypes.c_int),
        ("nx4", ctypes.c_int), ("nx3", ctypes.c_int), ("nx2", ctypes.c_int), ("nx1", ctypes.c_int),
        ("stride", ctypes.c_int64 * 4), ("device", ctypes.c_int),
    ]


def views_of(panels, device=-1):
    """Six ArrayViews of six 4-D panel arrays: numpy arrays (host, any
    strides) or, with device >= 0, (data_ptr, shape, element strides)
    triples of device arrays.  The result holds a reference to the panels,
    so a temporary list stays alive as long as the views do."""
    out = (ArrayView * 6)()
    out._panels = list(panels)
    for p, a in enumerate(panels):
        if device < 0:
            assert a.dtype.itemsize == 8 and a.ndim == 4
            ptr, shape, strides = a.ctypes.data, a.shape, [st // 8 for st in a.strides]
        else:
            ptr, shape, strides = a
        out[p].data = ptr
        out[p].dtype = EXO_DTYPE_F64
        out[p].nx4, out[p].nx3, out[p].nx2, out[p].nx1 = shape
        for q in range(4):
            out[p].stride[q] = strides[q]
        out[p].device = device
    return out


class CheckpointHeader(ctypes.Structure):
    """exo_checkpoint_header of include/exo_b200.h (512 bytes)."""
    _fields_ = [
        ("magic", ctypes.c_char * 8), ("version", ctypes.c_uint32),
        ("header_bytes", ctypes.c_uint32), ("values", ctypes.c_uint64),
        ("time", ctypes.c_double), ("dt", ctypes.c_double), ("ncycle", ctypes.c_int64),
        ("invalid", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("cfg", ExoConfig), ("pad", ctypes.c_uint8 * (512 - 56 - ctypes.sizeof(ExoConfig))),
    ]


class ExoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"exo error {code}: {msg}")
        self.code = code


_lib = None


def build():
    """Compile the library in-tree (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "csrc")], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`make -C exocubed_b200/csrc` (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    i, d, p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    cfgp = ctypes.POINTER(ExoConfig)
    L.exo_last_error.restype = ctypes.c_char_p
    L.exo_last_error.argtypes = []
    L.exo_config_default.argtypes = [cfgp, i]
    L.exo_create.argtypes = [cfgp, ctypes.POINTER(p)]
    L.exo_destroy.argtypes = [p]
    L.exo_destroy.restype = None
    L.exo_cell_geometry.argtypes = [cfgp, dp, dp, dp, dp]
    L.exo_mesh.argtypes = [cfgp, i, dp, dp, dp]
    L.exo_shape.argtypes = [p] + [ctypes.POINTER(i)] * 4
    L.exo_set_primitive.argtypes = [p, dp]
    L.exo_get_conserved.argtypes = [p, dp]
    L.exo_get_primitive.argtypes = [p, dp]
    L.exo_device_state.argtypes = [p, ctypes.POINTER(p), ctypes.POINTER(p)]
    L.exo_step.argtypes = [p, i, d]
    L.exo_get_dt.argtypes = [p, dp]
    L.exo_get_time.argtypes = [p, dp, ctypes.POINTER(ctypes.c_int64)]
    L.exo_check_state.argtypes = [p, ctypes.POINTER(i)]
    L.exo_synchronize.argtypes = [p]
    L.exo_calculate_fluxes.argtypes = [p]
    L.exo_get_flux.argtypes = [p, i, dp]
    L.exo_riemann.argtypes = [i, i, i, i, d, p, p, p, p, p, p, p, p]
    L.exo_weno5.argtypes = [i, p, p, p, p, p, p, p]
    L.exo_reciprocal.argtypes = [i, i, p, p, p]
    L.exo_implicit_columns.argtypes = [i, i, p, p, p, p, p, p, d, d, d, p, p]
    L.exo_partial_correction_columns.argtypes = [i, i, p, p, p, p, p, p, d, d, d, p, p]
    L.exo_implicit_columns_noalloc.argtypes = [i, i, p, p, p, p, p, p, d, d, d, p]
    sz = ctypes.c_size_t
    L.exo_ensemble_create.argtypes = [i, i, sz, ctypes.POINTER(p)]
    L.exo_ensemble_destroy.argtypes = [p]
    L.exo_ensemble_destroy.restype = None
    L.exo_ensemble_footprint.argtypes = [cfgp, ctypes.POINTER(sz)]
    L.exo_ensemble_add.argtypes = [p, cfgp, dp, ctypes.POINTER(i)]
    L.exo_ensemble_remove.argtypes = [p, i]
    L.exo_ensemble_step.argtypes = [p, i]
    L.exo_ensemble_synchronize.argtypes = [p]
    L.exo_ensemble_get_conserved.argtypes = [p, i, dp]
    L.exo_ensemble_get_primitive.argtypes = [p, i, dp]
    L.exo_ensemble_member_time.argtypes = [p, i, dp, dp, ctypes.POINTER(ctypes.c_int64)]
    L.exo_stage.argtypes = [p, i]
    L.exo_boundary.argtypes = [p]
    L.exo_solve_implicit_3d.argtypes = [p, dp, dp, d]
    L.exo_change_to_perturbation.argtypes = [p, dp]
    L.exo_restore_from_perturbation.argtypes = [p, dp, dp, dp]
    ip = ctypes.POINTER(ctypes.c_int)
    L.exo_set_tiles.argtypes = [p, ip]
    L.exo_get_tiles.argtypes = [p, ip]
    L.exo_ensemble_set_tiles.argtypes = [p, ip]
    L.exo_ensemble_get_tiles.argtypes = [p, ip]
    L.exo_ensemble_check_state.argtypes = [p, i, ctypes.POINTER(i)]
    L.exo_set_max_redo.argtypes = [p, i]
    L.exo_redo_count.argtypes = [p, ctypes.POINTER(ctypes.c_int64)]
    L.exo_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_double)]
    L.exo_panel_pack.argtypes = [p, p, p] + [i] * 8 + [ip, i, i, i, i, p]
    L.exo_save_lr3d.argtypes = [p, p, p, i, i, i, i, i, i, p]
    L.exo_load_lr3d.argtypes = [p, p, p, i, i, i, i, i, i, p]
    L.exo_lr3d_arrays.argtypes = [p] + [ctypes.POINTER(p)] * 4
    L.exo_synchronize_faces.argtypes = [p, p]
    L.exo_conserved_to_primitive.argtypes = [p, p, p, i, i, i, i, i, i, p]
    L.exo_primitive_to_conserved.argtypes = [p, p, p, i, i, i, i, i, i, p]
    L.exo_sound_speed.argtypes = [p, i, p, p, p]
    vp = ctypes.POINTER(ArrayView)
    L.exo_set_primitive_views.argtypes = [p, vp]
    L.exo_get_primitive_views.argtypes = [p, vp]
    L.exo_get_conserved_views.argtypes = [p, vp]
    L.exo_solve_implicit_3d_views.argtypes = [p, vp, vp, d]
    L.exo_check_bounded_wait.argtypes = [ctypes.POINTER(i), dp]
    L.exo_checkpoint_bytes.argtypes = [p, ctypes.POINTER(sz)]
    L.exo_checkpoint_save.argtypes = [p, p, sz]
    L.exo_checkpoint_load.argtypes = [p, p, sz]
    L.exo_ensemble_checkpoint_bytes.argtypes = [p, i, ctypes.POINTER(sz)]
    L.exo_ensemble_checkpoint_save.argtypes = [p, i, p, sz]
    L.exo_ensemble_add_checkpoint.argtypes = [p, p, sz, ctypes.POINTER(i)]
    L.exo_ensemble_stats.argtypes = [p, ctypes.POINTER(i), ctypes.POINTER(sz),
                                     ctypes.POINTER(ctypes.c_int64)]
    L.exo_ensemble_get_stream.argtypes = [p, ctypes.POINTER(p)]
    L.exo_get_stream.argtypes = [p, ctypes.POINTER(p)]
    L.exo_profile.argtypes = [p, i]
    L.exo_profile_read.argtypes = [p, i, ctypes.POINTER(ctypes.c_int64), dp]
    L.exo_launch_count.argtypes = [p, ctypes.POINTER(ctypes.c_int64)]
    _lib = L
    return L


def check(rc):
    if rc != EXO_OK:
        raise ExoError(rc, lib().exo_last_error().decode())
    return rc


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def checkpoint_header(image):
    """The exo_checkpoint_header of a checkpoint image (bytes-like) as a dict:
    magic, version, time, dt, ncycle, invalid and the configuration."""
    mv = memoryview(image).cast("B")
    if len(mv) < ctypes.sizeof(CheckpointHeader):
        raise ValueError("shorter than a checkpoint header")
    h = CheckpointHeader.from_buffer_copy(bytes(mv[:ctypes.sizeof(CheckpointHeader)]))
    return {"magic": bytes(h.magic), "version": h.version, "values": h.values,
            "time": h.time, "dt": h.dt, "ncycle": h.ncycle, "invalid": h.invalid,
            "cfg": h.cfg.as_dict()}


def fma_peak(fp64=True, repeats=3):
    """Best FMA rate (flops/s) of the current device in FP64 or FP32
    (exo_measure_fma_peak)."""
    out = ctypes.c_double()
    check(lib().exo_measure_fma_peak(int(bool(fp64)), int(repeats), ctypes.byref(out)))
    return out.value
