"""ctypes bindings of the C ABI declared in include/velo_b200.h.

Two shared libraries are built in-tree by cuda_hlt_b200/build.py:
  libvelo_host.so  host utilities (SuperPixel tables, generator, MC checker); no CUDA
  libvelo_b200.so  the sm_100a kernels and the chain context (velo_create/run/sync/destroy)
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB_PATH = os.path.join(_HERE, "libvelo_host.so")
GPU_LIB_PATH = os.path.join(_HERE, "libvelo_b200.so")
GEOMETRY_PATH = os.path.join(_HERE, "data", "velo_geometry.bin")


class VeloGenConfig(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("nu_min", C.c_float),
        ("nu_max", C.c_float),
        ("visible_fraction", C.c_float),
        ("tracks_per_pv", C.c_float),
        ("backward_fraction", C.c_float),
        ("pv_sigma_xy", C.c_float),
        ("pv_sigma_z", C.c_float),
        ("hit_efficiency", C.c_float),
        ("p_one_pixel", C.c_float),
        ("p_two_pixels", C.c_float),
        ("noise_per_asic_per_nu", C.c_float),
        ("noisy_event_fraction", C.c_float),
        ("noisy_factor", C.c_float),
    ]


class VeloCheckResult(C.Structure):
    _fields_ = [
        ("events", C.c_uint64),
        ("tracks", C.c_uint64),
        ("ghosts", C.c_uint64),
        ("long_reconstructible", C.c_uint64),
        ("long_found", C.c_uint64),
        ("long_clones", C.c_uint64),
        ("velo_reconstructible", C.c_uint64),
        ("velo_found", C.c_uint64),
        ("velo_clones", C.c_uint64),
        ("long_efficiency", C.c_double),
        ("velo_efficiency", C.c_double),
        ("ghost_rate", C.c_double),
        ("ghost_rate_per_event", C.c_double),
    ]


class VeloConfig(C.Structure):
    _fields_ = [
        ("max_events", C.c_uint32),
        ("max_raw_bytes", C.c_uint64),
        ("max_tracks", C.c_uint32),
        ("max_track_hits", C.c_uint32),
        ("device", C.c_int32),
        ("mode", C.c_uint32),
        ("mapping", C.c_uint32),
        ("use_graphs", C.c_uint32),
    ]


class VeloMlpWeights(C.Structure):
    _fields_ = [
        ("mean", C.c_float * 12),
        ("inv_std", C.c_float * 12),
        ("w1", (C.c_float * 13) * 64),
        ("w2", (C.c_float * 65) * 64),
        ("w3", (C.c_float * 65) * 2),
        ("seed_threshold", C.c_float),
        ("ext_threshold", C.c_float),
        ("max_event_clusters", C.c_uint32),
        ("min_pairs", C.c_uint32),
        ("min_event_clusters", C.c_uint32),
    ]


class VeloOutputs(C.Structure):
    _fields_ = [
        ("n_events", C.c_uint32),
        ("atomics", C.c_void_p),
        ("track_hit_number", C.c_void_p),
        ("track_hits", C.c_void_p),
        ("states", C.c_void_p),
        ("kalman_states", C.c_void_p),
        ("status", C.c_void_p),
        ("module_hit_start", C.c_void_p),
        ("module_hit_num", C.c_void_p),
        ("hit_xyzp", C.c_void_p),
        ("hit_id", C.c_void_p),
        ("hit_capacity", C.c_uint64),
        ("hit_size", C.c_void_p),
        ("hit_keep", C.c_void_p),
        ("pv_vertices", C.c_void_p),
        ("pv_count", C.c_void_p),
        ("pv_zpeaks", C.c_void_p),
        ("pv_npeaks", C.c_void_p),
        ("event_list", C.c_void_p),
        ("n_selected", C.c_void_p),
        ("gec_counts", C.c_void_p),
        ("gec_flags", C.c_void_p),
        ("hit_windows", C.c_void_p),
    ]


class VeloGecInput(C.Structure):
    _fields_ = [
        ("ut_raw", C.c_void_p),
        ("ut_offsets", C.c_void_p),
        ("scifi_raw", C.c_void_p),
        ("scifi_offsets", C.c_void_p),
        ("max_clusters", C.c_uint32),
    ]


# Every symbol include/velo_b200.h declares, per library.
HOST_SYMBOLS = [
    "velo_build_sp_luts",
    "velo_validate_raw_event",
    "velo_gen_default_config",
    "velo_gen_create",
    "velo_gen_raw_bytes",
    "velo_gen_mc_bytes",
    "velo_gen_copy",
    "velo_gen_destroy",
    "velo_check_tracks",
    "velo_mdf_read",
    "velo_mdf_read_banks",
    "velo_mdf_count",
    "velo_mdf_raw_bytes",
    "velo_mdf_copy",
    "velo_mdf_free",
]
GPU_SYMBOLS = [
    "velo_create",
    "velo_run",
    "velo_run_host",
    "velo_run_u32",
    "velo_run_host_u32",
    "velo_run_selected_u32",
    "velo_graph_count",
    "velo_run_gec",
    "velo_run_gec_host",
    "velo_sync",
    "velo_set_mlp",
    "velo_stage_times",
    "velo_set_timing",
    "velo_destroy",
    "velo_download",
    "velo_download_async",
    "velo_set_block_threshold",
    "velo_set_decode_warps",
    "velo_last_launch_count",
    "velo_check_wait_timeout",
    "velo_search_static",
    "velo_version",
    "velo_set_mode",
    "velo_capture_labels",
    "velo_set_pv",
    "velo_mlp_trainer_create",
    "velo_mlp_trainer_destroy",
    "velo_mlp_collect",
    "velo_mlp_samples",
    "velo_mlp_normalize",
    "velo_mlp_train",
    "velo_mlp_get_weights",
    "velo_mlp_set_weights",
    "velo_mlp_gradient",
    "velo_mlp_infer",
]

_host = None
_gpu = None


def host_lib():
    global _host
    if _host is None:
        if not os.path.exists(HOST_LIB_PATH):
            raise RuntimeError(f"{HOST_LIB_PATH} missing: run cuda_hlt_b200/build.py")
        lib = C.CDLL(HOST_LIB_PATH)
        P = C.c_void_p
        lib.velo_build_sp_luts.argtypes = [P, P, P, P]
        lib.velo_build_sp_luts.restype = None
        lib.velo_validate_raw_event.argtypes = [P, C.c_uint64]
        lib.velo_validate_raw_event.restype = C.c_int
        lib.velo_gen_default_config.argtypes = [C.POINTER(VeloGenConfig)]
        lib.velo_gen_default_config.restype = None
        lib.velo_gen_create.argtypes = [C.POINTER(VeloGenConfig), P, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(P)]
        lib.velo_gen_create.restype = C.c_int
        lib.velo_gen_raw_bytes.argtypes = [P]
        lib.velo_gen_raw_bytes.restype = C.c_uint64
        lib.velo_gen_mc_bytes.argtypes = [P]
        lib.velo_gen_mc_bytes.restype = C.c_uint64
        lib.velo_gen_copy.argtypes = [P, P, P, P, P, P]
        lib.velo_gen_copy.restype = C.c_int
        lib.velo_gen_destroy.argtypes = [P]
        lib.velo_gen_destroy.restype = None
        lib.velo_check_tracks.argtypes = [P, P, C.c_uint32, P, P, P, C.POINTER(VeloCheckResult)]
        lib.velo_check_tracks.restype = C.c_int
        lib.velo_mdf_read.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64, C.POINTER(P)]
        lib.velo_mdf_read.restype = C.c_int
        lib.velo_mdf_read_banks.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(P)]
        lib.velo_mdf_read_banks.restype = C.c_int
        lib.velo_mdf_count.argtypes = [P]
        lib.velo_mdf_count.restype = C.c_uint64
        lib.velo_mdf_raw_bytes.argtypes = [P]
        lib.velo_mdf_raw_bytes.restype = C.c_uint64
        lib.velo_mdf_copy.argtypes = [P, P, P, P, P]
        lib.velo_mdf_copy.restype = C.c_int
        lib.velo_mdf_free.argtypes = [P]
        lib.velo_mdf_free.restype = None
        _host = lib
    return _host


def gpu_lib():
    """The CUDA chain library. Raises if it was not built: there is no CPU fallback."""
    global _gpu
    if _gpu is None:
        if not os.path.exists(GPU_LIB_PATH):
            raise RuntimeError(f"{GPU_LIB_PATH} missing: run cuda_hlt_b200/build.py (no CPU fallback exists)")
        lib = C.CDLL(GPU_LIB_PATH)
        P = C.c_void_p
        lib.velo_create.argtypes = [C.POINTER(VeloConfig), P, C.c_size_t, C.POINTER(P)]
        lib.velo_create.restype = C.c_int
        lib.velo_run.argtypes = [P, P, P, C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run.restype = C.c_int
        lib.velo_run_host.argtypes = [P, P, P, C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run_host.restype = C.c_int
        lib.velo_run_u32.argtypes = [P, P, P, C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run_u32.restype = C.c_int
        lib.velo_run_host_u32.argtypes = [P, P, P, C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run_host_u32.restype = C.c_int
        lib.velo_run_selected_u32.argtypes = [P, P, P, C.c_uint32, P, C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run_selected_u32.restype = C.c_int
        lib.velo_graph_count.argtypes = [P, C.POINTER(C.c_uint32)]
        lib.velo_graph_count.restype = C.c_int
        lib.velo_run_gec.argtypes = [P, P, P, C.POINTER(VeloGecInput), C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run_gec.restype = C.c_int
        lib.velo_run_gec_host.argtypes = [P, P, P, C.POINTER(VeloGecInput), C.c_uint32, P, C.POINTER(VeloOutputs)]
        lib.velo_run_gec_host.restype = C.c_int
        lib.velo_sync.argtypes = [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
        lib.velo_sync.restype = C.c_int
        lib.velo_set_mlp.argtypes = [P, P, C.c_size_t]
        lib.velo_set_mlp.restype = C.c_int
        lib.velo_stage_times.argtypes = [P, C.POINTER(C.c_float), C.c_int]
        lib.velo_stage_times.restype = C.c_int
        lib.velo_set_timing.argtypes = [P, C.c_int]
        lib.velo_set_timing.restype = C.c_int
        lib.velo_destroy.argtypes = [P]
        lib.velo_destroy.restype = C.c_int
        lib.velo_download.argtypes = [P, P, P, C.c_size_t]
        lib.velo_download.restype = C.c_int
        lib.velo_download_async.argtypes = [P, P, P, C.c_size_t, P]
        lib.velo_download_async.restype = C.c_int
        lib.velo_set_block_threshold.argtypes = [P, C.c_uint32]
        lib.velo_set_block_threshold.restype = C.c_int
        lib.velo_set_decode_warps.argtypes = [P, C.c_uint32]
        lib.velo_set_decode_warps.restype = C.c_int
        lib.velo_last_launch_count.argtypes = [P, C.POINTER(C.c_uint32)]
        lib.velo_last_launch_count.restype = C.c_int
        lib.velo_check_wait_timeout.argtypes = [P, C.c_uint32, P]
        lib.velo_check_wait_timeout.restype = C.c_int
        lib.velo_search_static.argtypes = [P] * 4 + [C.c_uint32] + [P] * 5
        lib.velo_search_static.restype = C.c_int
        lib.velo_version.argtypes = []
        lib.velo_version.restype = C.c_char_p
        lib.velo_capture_labels.argtypes = [P, C.c_int, C.c_uint32]
        lib.velo_capture_labels.restype = C.c_int
        lib.velo_set_mode.argtypes = [P, C.c_uint32]
        lib.velo_set_mode.restype = C.c_int
        lib.velo_set_pv.argtypes = [P, C.c_int]
        lib.velo_set_pv.restype = C.c_int
        W = C.POINTER(VeloMlpWeights)
        lib.velo_mlp_trainer_create.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(P)]
        lib.velo_mlp_trainer_destroy.argtypes = [P]
        lib.velo_mlp_collect.argtypes = [P, P, C.POINTER(C.c_uint64)]
        lib.velo_mlp_samples.argtypes = [P, C.c_uint64, C.c_uint32, P, P]
        lib.velo_mlp_normalize.argtypes = [P]
        lib.velo_mlp_train.argtypes = [P, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(C.c_float)]
        lib.velo_mlp_get_weights.argtypes = [P, W]
        lib.velo_mlp_set_weights.argtypes = [P, W]
        lib.velo_mlp_gradient.argtypes = [P, P, P, C.c_uint32, W, C.POINTER(C.c_float)]
        lib.velo_mlp_infer.argtypes = [P, P, C.c_uint32, P]
        for name in ("velo_mlp_trainer_create", "velo_mlp_trainer_destroy", "velo_mlp_collect", "velo_mlp_samples",
                     "velo_mlp_normalize", "velo_mlp_train", "velo_mlp_get_weights", "velo_mlp_set_weights",
                     "velo_mlp_gradient", "velo_mlp_infer"):
            getattr(lib, name).restype = C.c_int
        _gpu = lib
    return _gpu
