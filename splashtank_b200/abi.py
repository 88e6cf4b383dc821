"""ctypes mirror of include/splashtank_cuda.h (the C ABI of the FLIP step and the PBF solver).

Only plain data crosses the boundary: pointers, sizes and the POD structs below, so the same
declarations bind any library that exports the header's functions (the CUDA library here; a
Node N-API shim binds the same symbols).
"""
import ctypes as C

ST_OK, ST_NOT_READY, ST_POOL_GREW, ST_OVERFLOW, ST_OOM, ST_BAD_ARG, ST_DEVICE_ERROR, ST_TIMEOUT, ST_UNSUPPORTED = range(9)
STATUS_NAMES = ["OK", "NOT_READY", "POOL_GREW", "OVERFLOW", "OOM", "BAD_ARG", "DEVICE_ERROR", "TIMEOUT", "UNSUPPORTED"]
ST_OPT_NO_FOAM, ST_OPT_NO_CULL, ST_OPT_FAST_AIR = 1, 2, 4

f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)


class FlipDesc(C.Structure):
    _fields_ = [("size", C.c_uint32), ("d", C.c_double), ("ratio", C.c_double), ("box", C.c_double * 3),
                ("open", C.c_uint32), ("max_n", C.c_uint32), ("spray_cap", C.c_uint32), ("device", C.c_int32)]


class Sdf(C.Structure):
    _fields_ = [("id", C.c_uint32), ("dims", C.c_uint32 * 3), ("origin", C.c_float * 3), ("cell", C.c_float), ("data", f32p)]


class Collider(C.Structure):
    _fields_ = [("sdf", C.POINTER(Sdf)), ("pos", C.c_float * 3), ("R", C.c_float * 9), ("vel", C.c_float * 3), ("ang", C.c_float * 3)]


class SprayOpts(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("rate", "min", "life", "mist", "drag", "mdrag", "foam_life", "rise", "crest", "impact")]


class StepOpts(C.Structure):
    _fields_ = [("size", C.c_uint32), ("g", C.c_float), ("flip", C.c_float), ("comp", C.c_float), ("omega", C.c_float),
                ("vmax", C.c_float), ("wind", C.c_float * 3), ("drag", C.c_float), ("foam_tau", C.c_float),
                ("foam_sens", C.c_float), ("gust", C.c_float), ("tear", C.c_float), ("vs", C.c_float), ("iters", C.c_int32),
                ("flags", C.c_uint32), ("ncols", C.c_uint32), ("cols", C.POINTER(Collider)), ("spray_on", C.c_int32),
                ("spray", SprayOpts), ("nb_on", C.c_int32), ("nb_band", C.c_float), ("air_on", C.c_int32), ("air_couple", C.c_float), ("air_decay", C.c_float), ("air_blur", C.c_float),
                ("drip_on", C.c_int32), ("drip_rate", C.c_float), ("drip_dry", C.c_float),
                ("ocean_on", C.c_int32), ("ocean_level", C.c_float), ("ocean_layer", C.c_float), ("ocean_length", C.c_float),
                ("ocean_height", C.c_float), ("ocean_dir", C.c_float), ("ocean_spread", C.c_float), ("ocean_seed", C.c_int32),
                ("time", C.c_float), ("pbf_iters", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("sc", C.c_uint32), ("ovf", C.c_uint32), ("fluid", C.c_uint32), ("vmax", C.c_float), ("n", C.c_uint32),
                ("live", C.c_uint32), ("spray_used", C.c_uint32), ("steps", C.c_uint32), ("spray_overflow", C.c_uint32),
                ("launches", C.c_uint64)]


class Grid(C.Structure):
    _fields_ = [("tile_on", u8p), ("cnt", i32p), ("ctype", u32p), ("pres", f32p), ("rhs", f32p), ("vn", f32p), ("vo", f32p), ("velg", f32p)]


class Dims(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("tx", C.c_uint32), ("ty", C.c_uint32), ("tz", C.c_uint32),
                ("h", C.c_float), ("x0", C.c_float), ("y0", C.c_float), ("z0", C.c_float), ("x1", C.c_float), ("y1", C.c_float), ("z1", C.c_float)]


STAGES = ("sort", "blocks", "clear", "p2g", "narrow_band", "classify", "norm_faces", "divergence", "pressure", "project", "g2p",
          "pbf", "spray", "reseed", "total")


class StageTimes(C.Structure):
    _fields_ = [(n, C.c_float) for n in STAGES]


class PbfDesc(C.Structure):
    _fields_ = [("size", C.c_uint32), ("d", C.c_double), ("box", C.c_double * 3), ("open", C.c_uint32), ("max_n", C.c_uint32),
                ("device", C.c_int32), ("eps_k", C.c_double), ("wall_k", C.c_double)]


class PbfOpts(C.Structure):
    _fields_ = [("size", C.c_uint32), ("g", C.c_float), ("visc", C.c_float), ("iters", C.c_int32), ("ncols", C.c_uint32),
                ("cols", C.POINTER(Collider))]


class PoissonDesc(C.Structure):
    _fields_ = [("size", C.c_uint32), ("n", C.c_uint32 * 3), ("open", C.c_uint32), ("device", C.c_int32)]


class PoissonOpts(C.Structure):
    _fields_ = [("size", C.c_uint32), ("mode", C.c_int32), ("tol", C.c_double), ("omega", C.c_float), ("max_sweeps", C.c_int32),
                ("inner_sweeps", C.c_int32), ("check_every", C.c_int32), ("schedule", C.c_int32)]


class PoissonResult(C.Structure):
    _fields_ = [("rel_residual", C.c_double), ("sweeps", C.c_int32), ("refinements", C.c_int32), ("converged", C.c_int32),
                ("ms", C.c_float)]


class PoissonSystem(C.Structure):
    _fields_ = [("size", C.c_uint32), ("n", C.c_uint32 * 3), ("n_tiles", C.c_uint32), ("tiles", C.c_void_p), ("info", C.c_void_p),
                ("b", C.c_void_p)]


NOALLOC_MAX_TILES = 65536

# (name, restype, argtypes) with the prefix left off; "h" stands for the opaque handle
FLIP_FUNCS = [
    ("flip_create", C.c_int, [C.POINTER(FlipDesc), C.POINTER(C.c_void_p)]),
    ("flip_destroy", None, [C.c_void_p]),
    ("flip_clear", C.c_int, [C.c_void_p]),
    ("flip_set_cap", C.c_int, [C.c_void_p, C.c_uint32]),
    ("flip_add", C.c_int, [C.c_void_p, f32p, f32p, C.c_uint32, u32p]),
    ("flip_step", C.c_int, [C.c_void_p, C.c_double, C.POINTER(StepOpts)]),
    ("flip_read_particles", C.c_int, [C.c_void_p, f32p, f32p, C.c_uint32, u32p]),
    ("flip_read_spray", C.c_int, [C.c_void_p, f32p, f32p, C.c_uint32, u32p]),
    ("flip_read_air", C.c_int, [C.c_void_p, f32p, C.c_uint32, u32p]),
    ("flip_read_drips", C.c_int, [C.c_void_p, f32p, C.c_uint32, u32p]),
    ("flip_set_deep_look", C.c_int, [C.c_void_p, C.c_int]),
    ("flip_set_spray_cap", C.c_int, [C.c_void_p, C.c_uint32]),
    ("flip_set_recycle", C.c_int, [C.c_void_p, C.c_int]),
    ("flip_stats", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("flip_read_grid", C.c_int, [C.c_void_p, C.POINTER(Grid)]),
    ("flip_get_dims", C.c_int, [C.c_void_p, C.POINTER(Dims)]),
    ("flip_save_state", C.c_int, [C.c_void_p, f32p, f32p, u32p, C.c_uint32, u32p]),
    ("flip_load_state", C.c_int, [C.c_void_p, f32p, f32p, u32p, C.c_uint32, C.c_double, C.c_uint32]),
    ("flip_nb_fills", C.c_int, [C.c_void_p, f32p, C.c_uint32, f32p, C.c_uint32, C.c_uint32]),
    ("flip_nb_fill_vols", C.c_int, [C.c_void_p, C.POINTER(Collider), C.c_uint32, C.c_uint32]),
]
class BakeDiag(C.Structure):
    _fields_ = [("alive", C.c_uint32), ("gone", C.c_uint32), ("non_finite", C.c_uint32), ("outside_box", C.c_uint32),
                ("at_speed_limit", C.c_uint32), ("foamy", C.c_uint32), ("mean_speed", C.c_double), ("max_speed", C.c_double),
                ("mean_foam", C.c_double), ("center", C.c_double * 3), ("has_bbox", C.c_int32), ("bbox", C.c_double * 6),
                ("height_hist", C.c_uint32 * 16)]


class Mesh(C.Structure):
    _fields_ = [("v", C.POINTER(C.c_double)), ("nv", C.c_uint32), ("idx", u32p), ("len", u32p), ("nf", C.c_uint32)]


class SdfBuild(C.Structure):
    _fields_ = [("size", C.c_uint32), ("dims", C.c_uint32 * 3), ("cell", C.c_double), ("margin", C.c_double), ("origin", C.c_double * 3),
                ("data", f32p), ("cap", C.c_uint64)]


SDF_FUNCS = [("build_sdf", C.c_int, [C.c_int, C.POINTER(Mesh), C.POINTER(SdfBuild)])]
OCEAN_FUNCS = [("ocean_waves", C.c_int, [C.POINTER(StepOpts), C.c_double, f32p])]


class LiveLayout(C.Structure):
    _fields_ = [("size", C.c_uint32), ("n_water", C.c_uint32), ("n_spray", C.c_uint32), ("n_deep", C.c_uint32), ("from_pos", C.c_uint32),
                ("o_wp", C.c_uint32), ("o_ws", C.c_uint32), ("o_wf", C.c_uint32), ("o_sp", C.c_uint32), ("o_sk", C.c_uint32),
                ("o_dp", C.c_uint32), ("o_ds", C.c_uint32), ("words", C.c_uint32)]


CUDA_ONLY_FUNCS = [
    ("flip_pack_live", C.c_int, [C.c_void_p, C.c_float, u32p, C.c_uint64, C.POINTER(LiveLayout)]),
    ("flip_read_deep_points", C.c_int, [C.c_void_p, f32p, C.c_uint32, u32p]),
    ("flip_mem_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("flip_read_deep", C.c_int, [C.c_void_p, C.c_float, C.POINTER(C.c_uint16), u8p, C.c_uint32, u32p]),
    ("flip_read_spray_frame", C.c_int, [C.c_void_p, C.c_uint32, C.c_float, C.POINTER(C.c_uint16), u32p, C.c_uint32, u32p, u32p]),
    ("flip_read_frame", C.c_int, [C.c_void_p, C.c_float, C.POINTER(C.c_uint16), u8p, u8p, C.c_uint32, u32p, C.POINTER(C.c_int32)]),
    ("flip_track", C.c_int, [C.c_void_p, u32p, f32p, f32p]),
    ("flip_stats_async", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("flip_stats_wait", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Stats)]),
    ("flip_read_frame_async", C.c_int, [C.c_void_p, C.c_float, C.POINTER(C.c_uint16), u8p, u8p, C.c_uint32]),
    ("flip_frame_wait", C.c_int, [C.c_void_p, u32p, C.POINTER(C.c_int32)]),
    ("flip_bake_diag", C.c_int, [C.c_void_p, C.c_float, C.POINTER(BakeDiag)]),
    ("flip_save_full", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("flip_load_full", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    ("flip_set_launch", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    ("step_opts_default", None, [C.POINTER(StepOpts)]),
    ("flip_step_timed", C.c_int, [C.c_void_p, C.c_double, C.POINTER(StepOpts), C.POINTER(StageTimes)]),
    ("flip_stream", C.c_void_p, [C.c_void_p]),
    ("flip_set_timing", C.c_int, [C.c_void_p, C.c_int]),
    ("flip_read_timing", C.c_int, [C.c_void_p, C.POINTER(StageTimes), u32p]),
    ("abi_version", C.c_uint32, []),
    ("last_error", C.c_char_p, []),
]
POISSON_FUNCS = [
    ("poisson_create", C.c_int, [C.POINTER(PoissonDesc), C.POINTER(C.c_void_p)]),
    ("poisson_destroy", None, [C.c_void_p]),
    ("poisson_set", C.c_int, [C.c_void_p, u8p, C.POINTER(C.c_double)]),
    ("poisson_solve", C.c_int, [C.c_void_p, C.POINTER(PoissonOpts), C.POINTER(PoissonResult)]),
    ("poisson_sweeps32", C.c_int, [C.c_void_p, C.c_float, C.c_int32, C.POINTER(C.c_float)]),
    ("poisson_read", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
]
class BatchDesc(C.Structure):
    _fields_ = [("size", C.c_uint32), ("mode", C.c_int32)]


ST_BATCH_GRAPH, ST_BATCH_SEQUENTIAL, ST_BATCH_POOLED, ST_BATCH_PERSISTENT = 0, 1, 2, 3
BATCH_FUNCS = [
    ("batch_create", C.c_int, [C.POINTER(BatchDesc), C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(C.c_void_p)]),
    ("batch_destroy", None, [C.c_void_p]),
    ("batch_step", C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.POINTER(StepOpts))]),
    ("batch_set_mode", C.c_int, [C.c_void_p, C.c_int32]),
    ("batch_stream", C.c_void_p, [C.c_void_p]),
    ("batch_launches", C.c_uint64, [C.c_void_p]),
    ("batch_set_sweeps", C.c_int, [C.c_void_p, C.c_int32, C.c_uint32]),
    ("batch_barrier_test", C.c_int, [C.c_int32, C.c_uint32, C.c_uint32, u32p]),
]
class DiffDesc(C.Structure):
    _fields_ = [("size", C.c_uint32), ("n", C.c_uint32), ("steps", C.c_uint32), ("ckpt_every", C.c_uint32), ("fp64", C.c_int32),
                ("device", C.c_int32), ("dt", C.c_float), ("flip", C.c_float), ("g", C.c_float), ("q0", C.c_float), ("margin", C.c_float),
                ("box_half", C.c_float * 3), ("cg_maxit", C.c_uint32), ("cg_tol", C.c_float), ("collider_grid", C.c_int32),
                ("grid_cell", C.c_float)]


DIFF_FUNCS = [
    ("diff_create", C.c_int, [C.POINTER(DiffDesc), f32p, C.c_uint32, f32p, C.POINTER(C.c_void_p)]),
    ("diff_destroy", None, [C.c_void_p]),
    ("diff_forward", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double)]),
    ("diff_backward", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("diff_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]),
    ("diff_read_state", C.c_int, [C.c_void_p, f32p, f32p]),
    ("diff_stream", C.c_void_p, [C.c_void_p]),
]
NOALLOC_FUNCS = [
    ("poisson_residual_noalloc", C.c_int, [C.POINTER(PoissonSystem), C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double), C.POINTER(C.c_double)]),
]
PBF_FUNCS = [
    ("pbf_create", C.c_int, [C.POINTER(PbfDesc), C.POINTER(C.c_void_p)]),
    ("pbf_destroy", None, [C.c_void_p]),
    ("pbf_add", C.c_int, [C.c_void_p, f32p, f32p, C.c_uint32, u32p]),
    ("pbf_step", C.c_int, [C.c_void_p, C.c_double, C.POINTER(PbfOpts)]),
    ("pbf_read", C.c_int, [C.c_void_p, f32p, f32p, C.c_uint32, u32p]),
    ("pbf_set_cap", C.c_int, [C.c_void_p, C.c_uint32]),
    ("pbf_clear", C.c_int, [C.c_void_p]),
    ("pbf_set_recycle", C.c_int, [C.c_void_p, C.c_int32]),
    ("pbf_stream", C.c_void_p, [C.c_void_p]),
]


def bind(lib, prefix, funcs):
    """Set restype/argtypes of prefix+name for every entry; returns {name: function}."""
    out = {}
    for name, res, args in funcs:
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
        out[name] = fn
    return out


def default_opts():
    """st_step_opts_default in Python (src/flip/sim.js:197-230 defaults)."""
    o = StepOpts()
    o.size = C.sizeof(StepOpts)
    o.g = 9.81
    o.flip = 0.95
    o.comp = 6.0
    o.omega = 0.0
    o.vmax = 14.0
    o.foam_tau = 1.2
    o.foam_sens = 1.0
    o.vs = 1.0
    o.iters = 30
    o.spray.foam_life = 3.0
    o.spray.rise = 0.3
    o.spray.crest = 1.0
    o.spray.impact = 0.5
    o.nb_band = 3.0
    return o
