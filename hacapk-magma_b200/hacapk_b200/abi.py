"""ctypes mirror of include/hacapk_b200.h and include/hacapk_b200_build.h.

The structures below reproduce the C layouts field for field; the leaf
container keeps the HAVE_MAGMA_BATCH prefix of HACApK_MAGMA.h:28-106 so that
`st_lf` sits where a MAGMA build of the Fortran type puts it.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
ENGINE_LIB = os.path.join(_HERE, "libhacapk_b200.so")
BUILD_LIB = os.path.join(_HERE, "libhacapk_build.so")


class LeafMtx(C.Structure):
    """stc_HACApK_leafmtx (HACApK_MAGMA.h:12-20)."""
    _fields_ = [("ltmtx", C.c_int), ("kt", C.c_int), ("nstrtl", C.c_int), ("ndl", C.c_int),
                ("nstrtt", C.c_int), ("ndt", C.c_int), ("a1size", C.c_longlong),
                ("a1", C.POINTER(C.c_double)), ("a2", C.POINTER(C.c_double))]


_VP = C.c_void_p


class LeafMtxP(C.Structure):
    """stc_HACApK_leafmtxp (HACApK_MAGMA.h:28-106, HAVE_MAGMA_BATCH layout)."""
    _fields_ = ([("nd", C.c_int), ("nlf", C.c_int), ("nlfkt", C.c_int), ("ktmax", C.c_int),
                 ("st_lf_stride", C.c_int),
                 ("m", C.c_int), ("n", C.c_int), ("gn", C.c_int), ("max_block", C.c_int),
                 ("gflops", C.c_double)]
                + [(f, _VP) for f in ("mtx1_gpu", "mtx2_gpu", "zu_gpu", "zau_gpu", "zau_pin", "zbu_gpu")]
                + [("num_batch", C.c_int), ("total_size_y", C.c_int), ("transA", C.c_int)]
                + [(f, _VP) for f in ("d_A_array", "d_X_array", "d_Y_array", "d_M", "d_N", "d_lda",
                                      "d_inc", "batch_order", "h_A_array", "h_X_array", "h_Y_array",
                                      "h_type", "h_I", "h_J", "h_M", "h_N", "h_lda", "max_M", "max_N",
                                      "batch_size")]
                + [("num_streamed", C.c_int), ("num_streamed_t", C.c_int)]
                + [(f, _VP) for f in ("h_A_array_streamed", "h_X_array_streamed",
                                      "h_Y_array_streamed", "h_M_streamed", "h_N_streamed",
                                      "h_lda_streamed", "d_A_mgpu", "d_X_mgpu", "d_Y_mgpu",
                                      "d_M_mgpu", "d_N_mgpu", "d_lda_mgpu", "d_inc_mgpu", "zu_mgpu",
                                      "zau_mgpu", "zbu_mgpu", "h_A_mgpu", "h_X_mgpu", "h_Y_mgpu",
                                      "h_type_mgpu", "h_I_mgpu", "h_J_mgpu", "h_M_mgpu", "h_N_mgpu",
                                      "h_lda_mgpu", "max_M_mgpu", "max_N_mgpu", "nlf_mgpu",
                                      "num_batch_mgpu", "total_size_y_mgpu")]
                + [("iwork", C.POINTER(C.c_int)), ("mpi_rank", C.c_int),
                   ("st_lf", C.POINTER(LeafMtx))])


class LControl(C.Structure):
    """stc_HACApK_lcontrol (HACApK_MAGMA.h:108-121)."""
    _fields_ = [("lf_umpi", C.c_int), ("lpmd_offset", C.c_int), ("lod_offset", C.c_int),
                ("lsp_offset", C.c_int), ("lnp_offset", C.c_int), ("lthr_offset", C.c_int),
                ("param", C.POINTER(C.c_double))]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("num_ctas", C.c_int), ("transpose", C.c_int), ("nrhs", C.c_int),
                ("block_cost", C.c_int), ("run_cost", C.c_int), ("merge", C.c_int), ("l2_keep_mb", C.c_int),
                ("reserved", C.c_int * 8)]


class Info(C.Structure):
    _fields_ = [("nd", C.c_int), ("nlf", C.c_int), ("nlfkt", C.c_int), ("ktmax", C.c_int),
                ("num_ctas", C.c_int), ("num_atoms", C.c_int), ("num_runs", C.c_int),
                ("precision", C.c_int), ("stream_bytes", C.c_longlong),
                ("alg_bytes", C.c_longlong), ("alg_flops", C.c_longlong),
                ("zbu_len", C.c_longlong), ("dense_words", C.c_longlong),
                ("lowrank_words", C.c_longlong), ("setup_seconds", C.c_double),
                ("transposed", C.c_int), ("nrhs", C.c_int), ("instances", C.c_int),
                ("block_cost", C.c_int), ("run_cost", C.c_int), ("merge_keep", C.c_int), ("l2_keep_mb", C.c_int),
                ("reserved", C.c_int * 1)]


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int), ("verbose", C.c_int),
                ("batch", C.c_int), ("restart", C.c_int), ("inner_tol", C.c_double),
                ("reserved", C.c_int * 8)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("bnorm", C.c_double),
                ("relres", C.c_double), ("true_relres", C.c_double), ("seconds", C.c_double),
                ("iter_kernel_seconds", C.c_double), ("iter_launches", C.c_int),
                ("launches", C.c_int), ("outer", C.c_int), ("reserved", C.c_int * 5)]


class FillParams(C.Structure):
    _fields_ = [("kernel", C.c_int), ("aca_eps", C.c_double), ("aca_abs_factor", C.c_double), ("kmax", C.c_int),
                ("kmin", C.c_int), ("workspace_mb", C.c_int), ("first_cap", C.c_int), ("reserved", C.c_int * 8)]


class FillStats(C.Structure):
    _fields_ = [("n_lowrank", C.c_int), ("n_dense", C.c_int), ("ktmax", C.c_int), ("words", C.c_longlong),
                ("retried", C.c_longlong), ("seconds", C.c_double), ("reserved", C.c_int * 6)]


class BuildParams(C.Structure):
    _fields_ = [("leaf_size", C.c_int), ("eta", C.c_double), ("aca_eps", C.c_double),
                ("aca_abs_factor", C.c_double), ("kmax", C.c_int), ("kmin", C.c_int),
                ("kernel", C.c_int), ("nthreads", C.c_int), ("fill", C.c_int),
                ("aca_method", C.c_int), ("reserved", C.c_int * 6)]


class BuildStats(C.Structure):
    _fields_ = [("nd", C.c_int), ("nclst", C.c_int), ("n_lowrank", C.c_int), ("n_dense", C.c_int),
                ("n_hnode", C.c_int), ("ktmax", C.c_int), ("mem_words", C.c_longlong),
                ("memh_words", C.c_longlong), ("ncpc7", C.c_longlong),
                ("seconds_tree", C.c_double), ("seconds_fill", C.c_double),
                ("reserved", C.c_int * 8)]


KERNEL_PPOHBEM = 0
KERNEL_LAPLACE = 1

HBX_FP64, HBX_FP32, HBX_BF16 = 0, 1, 2
HBX_NRHS = 64

STATUS = {0: "HBX_OK", 1: "HBX_ERR_INVALID", 2: "HBX_ERR_NOMEM", 3: "HBX_ERR_CUDA",
          4: "HBX_ERR_TIMEOUT", 5: "HBX_ERR_BREAKDOWN", 6: "HBX_ERR_NOT_CONVERGED",
          7: "HBX_ERR_NONFINITE", 8: "HBX_ERR_UNSUPPORTED"}

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)

# (name, restype, argtypes) of every symbol the engine library exports.
ENGINE_SYMBOLS = [
    ("hbx_create", C.c_int, [C.POINTER(LeafMtxP), C.c_int, C.POINTER(Options), C.POINTER(_VP)]),
    ("hbx_create_batch", C.c_int, [C.POINTER(C.POINTER(LeafMtxP)), _IP, C.c_int, C.POINTER(Options),
                                   C.POINTER(_VP)]),
    ("hbx_autotune", C.c_int, [C.POINTER(LeafMtxP), C.c_int, C.POINTER(Options), C.c_int, C.POINTER(Options), _DP,
                               _DP]),
    ("hbx_destroy", C.c_int, [_VP]),
    ("hbx_get_info", C.c_int, [_VP, C.POINTER(Info)]),
    ("hbx_matvec", C.c_int, [_VP, C.c_double, _VP, C.c_double, _VP, _VP, _VP]),
    ("hbx_matvec_noalloc", C.c_int, [_VP, C.c_double, _VP, C.c_double, _VP, _VP, _VP]),
    ("hbx_matmat", C.c_int, [_VP, C.c_double, _VP, C.c_double, _VP, _VP, _VP]),
    ("hbx_bicgstab_batch", C.c_int, [_VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_bicgstab_batch_host", C.c_int, [_VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_bicgstab_multi", C.c_int, [_VP, _VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_bicgstab_multi_host", C.c_int, [_VP, _VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_sync", C.c_int, [_VP, _VP]),
    ("hbx_matvec_host", C.c_int, [_VP, _DP, _DP, C.c_int, _DP, _DP]),
    ("hbx_bicgstab", C.c_int, [_VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_bicgstab_host", C.c_int, [_VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_gcr", C.c_int, [_VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_gcr_host", C.c_int, [_VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_bicgstab_batch_refined", C.c_int, [_VP, _VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_bicgstab_batch_refined_host", C.c_int, [_VP, _VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_bicgstab_pipe", C.c_int, [_VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_bicgstab_pipe_host", C.c_int, [_VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_bicgstab_refined", C.c_int, [_VP, _VP, _VP, _VP, C.POINTER(SolveOpts), C.POINTER(SolveInfo), _VP]),
    ("hbx_bicgstab_refined_host", C.c_int, [_VP, _VP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    ("hbx_gradient_host", C.c_int, [_VP, _VP, _DP, _DP, _DP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveInfo),
                                    C.POINTER(SolveInfo)]),
    ("hbx_debug_phase_stamps", C.c_int, [_VP, C.POINTER(C.c_ulonglong), C.c_int]),
    ("hbx_fill_leaves", C.c_int, [_DP, C.c_int, _IP, C.c_int, _IP, C.POINTER(FillParams), C.POINTER(LeafMtxP),
                                  C.POINTER(_VP), C.POINTER(FillStats)]),
    ("hbx_fill_free", None, [_VP]),
    ("hbx_debug_stall_next_barrier", C.c_int, [_VP]),
    ("hbx_debug_fail_alloc", C.c_int, [C.c_int]),
    ("hbx_status_string", C.c_char_p, [C.c_int]),
    ("hbx_last_error", C.c_char_p, []),
    ("magma_init_", None, []),
    ("magma_finalize_", None, []),
    ("c_hacapk_adot_body_lfcpy_batch_sorted_", None, [_IP, C.POINTER(LeafMtxP)]),
    ("c_hacapk_adot_body_lfmtx_batch_", None, [_DP, C.POINTER(LeafMtxP), _DP, _DP, _DP, _DP, _DP]),
    ("c_hacapk_adot_body_lfdel_batch_", None, [C.POINTER(LeafMtxP)]),
    ("c_hacapk_adot_body_lfcpy_gpu_", None, [_IP, C.POINTER(LeafMtxP)]),
    ("c_hacapk_adot_body_lfmtx_gpu_", None, [_DP, C.POINTER(LeafMtxP), _DP, _DP]),
    ("c_hacapk_adot_body_lfdel_gpu_", None, [C.POINTER(LeafMtxP)]),
    ("c_hacapk_bicgstab_cax_lfmtx_gpu_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_bicgstab_cax_lfmtx_flat_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_bicgstab_cax_lfmtx_pipe_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_bicgstab_cax_lfmtx_pipe2_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_gcrm_lfmtx_gpu_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_bicgstab_cax_lfmtx_mgpu1_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_bicgstab_cax_lfmtx_mgpu2_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
    ("c_hacapk_bicgstab_cax_lfmtx_mgpu3_", None,
     [C.POINTER(LeafMtxP), C.POINTER(LControl), _DP, _DP, _DP, _IP, _IP, _IP]),
]

BUILD_SYMBOLS = [
    ("hbx_build_default_params", None, [C.POINTER(BuildParams)]),
    ("hbx_mesh_icosphere", C.c_int, [C.c_int, _DP, _IP]),
    ("hbx_build", C.c_int, [_DP, C.c_int, _IP, C.c_int, C.POINTER(BuildParams), C.POINTER(_VP)]),
    ("hbx_build_free", None, [_VP]),
    ("hbx_build_leafmtxp", C.POINTER(LeafMtxP), [_VP]),
    ("hbx_build_lod", _IP, [_VP]),
    ("hbx_build_get_stats", C.c_int, [_VP, C.POINTER(BuildStats)]),
    ("hbx_build_centroids", _DP, [_VP]),
    ("hbx_build_entry", C.c_double, [_VP, C.c_int, C.c_int]),
    ("hbx_build_dense_block", C.c_int, [_VP, C.c_int, C.c_int, C.c_int, C.c_int, _DP]),
]

_libs: dict = {}


def _load(path: str, symbols) -> C.CDLL:
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise RuntimeError(
            f"{os.path.basename(path)} is not built ({path}); run __graft_entry__.build() "
            "or `make -C hacapk-magma_b200`")
    lib = C.CDLL(path)
    for name, res, args in symbols:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[path] = lib
    return lib


def engine_lib() -> C.CDLL:
    """The CUDA engine (libhacapk_b200.so).  Raises if it is not built: there
    is no CPU fallback for the hot path."""
    return _load(ENGINE_LIB, ENGINE_SYMBOLS)


def build_lib() -> C.CDLL:
    return _load(BUILD_LIB, BUILD_SYMBOLS)


def dptr(a) -> C.POINTER(C.c_double):
    """ctypes double* of a contiguous float64 numpy array."""
    return a.ctypes.data_as(_DP)


def iptr(a) -> C.POINTER(C.c_int):
    return a.ctypes.data_as(_IP)
