"""ctypes binding of the C-ABI library ``_lib/libebsd_b200.so``.

Every function declared in ``include/ebsd_b200.h`` is bound here with its
exact argument types. ``call(name, *args)`` raises ``ValueError`` for argument
errors (status > 0) and ``RuntimeError`` for CUDA errors (status < 0), with
the library's own message. There is no fallback: if the library is missing,
importing the package's GPU entry points fails loudly.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# EBSD_CHECK_BUILD=1 loads the checking build (`python -m ebsdtorch_b200.build --check`)
LIB_PATH = os.path.join(_HERE, "_lib", "libebsd_b200_check.so" if os.environ.get("EBSD_CHECK_BUILD") == "1"
                        else "libebsd_b200.so")

vp, i32, i64, f32, sz = C.c_void_p, C.c_int, C.c_int64, C.c_float, C.c_size_t

# name -> (restype, argtypes); mirrors include/ebsd_b200.h
SIGNATURES = {
    "ebsd_version": (i32, []),
    "ebsd_debug_check_line": (i32, [C.c_char_p, sz]),
    "ebsd_last_error": (i32, [C.c_char_p, sz]),
    "ebsd_device_check": (i32, [i32]),
    "ebsd_grid_workspace_bytes": (sz, [i32]),
    "ebsd_grid_fz_count": (i32, [i32, i32, vp, sz, vp, vp]),
    "ebsd_grid_fz_write": (i32, [i32, i32, vp, sz, vp, vp, vp, vp]),
    "ebsd_gather_rows": (i32, [vp, i64, i32, vp, i64, vp, vp]),
    "ebsd_project_dictionary": (i32, [vp, i32, i32, vp, i32, vp, i64, i32, vp, i64, vp, i32, i64, vp, vp, vp]),
    "ebsd_prep_patterns": (i32, [vp, i64, i32, i32, i64, i32, vp, i32, i32, vp, i64, vp, i32, i64, vp, vp, vp]),
    "ebsd_prep_patterns_typed": (i32, [vp, i32, i64, i32, i32, i64, i32, vp, i32, i32, vp, i64, vp, i32, i64, vp,
                                       vp, vp]),
    "ebsd_sample_master_pattern": (i32, [vp, i32, i32, vp, i64, i32, vp, vp]),
    "ebsd_avg_pool": (i32, [vp, i64, i32, i32, i32, vp, vp]),
    "ebsd_match_auto_splits": (i32, [i64, i64]),
    "ebsd_match_auto_splits_typed": (i32, [i64, i64, i32]),
    "ebsd_set_wait_limit_ns": (i64, [i64]),
    "ebsd_set_match_pairs": (i32, [i32]),
    "ebsd_set_match_dual": (i32, [i32]),
    "ebsd_match_pair_max_clusters": (i32, []),
    "ebsd_manhattan_topk": (i32, [vp, i64, i64, i64, vp, i64, i64, i32, i32, i32, vp, vp, i32, i32, i32, vp]),
    "ebsd_match_topk": (i32, [vp, i64, vp, i64, i64, i64, i32, vp, i32, i32, vp, vp, i32, i32, i32, vp, vp]),
    "ebsd_match_topk_tiled": (i32, [vp, i64, vp, i64, i64, i64, i32, vp, vp, vp, i32, i32, vp, vp, i32, i32, i32,
                                    i32, i32, vp, vp]),
    "ebsd_merge_rescore": (i32, [vp, vp, i64, i32, i32, vp, i64, vp, i64, i64, i64, i32, vp, vp, vp, i32, i32, i32,
                                 vp, vp, vp, vp, vp]),
    "ebsd_merge_rescore_gated": (i32, [vp, vp, i64, i32, i32, vp, i64, vp, i64, i64, i64, i32, vp, vp, vp, i32, i32, i32,
                                 vp, vp, vp, vp, f32, vp, vp]),
    "ebsd_gemm_nt": (i32, [vp, i64, vp, i64, i64, i32, f32, i32, vp, i64, i64, i64, i32, vp, vp]),
    "ebsd_gemm_f32": (i32, [vp, i64, i64, vp, i64, i64, i64, f32, i32, vp, i64, i32, vp, vp]),
    "ebsd_col_mean": (i32, [vp, i64, i32, i64, vp, vp]),
    "ebsd_split3_bf16": (i32, [vp, i64, i32, i64, vp, i32, i32, vp, i64, i64, vp]),
    "ebsd_disori_angle": (i32, [vp, vp, i64, i32, vp, vp]),
    "ebsd_match_topk_noalloc": (i32, [vp, i64, i64, vp, i64, i64, i64, i32, vp, vp, i32, vp, vp, vp, vp]),
    "ebsd_cell_to_row": (i32, [vp, vp, i64, i64, vp, vp]),
    "ebsd_refine_grid": (i32, [vp, i32, i32, vp, i32, vp, vp, i64, vp, i64, vp, i32, i32, i32, i32, f32, vp, vp,
                               vp]),
    "ebsd_pattern_mean": (i32, [vp, i64, i32, i64, vp, i32, vp, vp]),
    "ebsd_subtract_pattern": (i32, [vp, i64, i32, i64, vp, vp]),
    "ebsd_normalize_patterns": (i32, [vp, i64, i32, i64, i32, vp]),
    "ebsd_clahe": (i32, [vp, i64, i32, i32, i64, vp, i32, f32, i32, i32, i32, i32, vp, i64, vp]),
    "ebsd_nlpar_dists": (i32, [vp, i32, i32, i32, i64, i32, vp, i32, i32, i32, vp, vp]),
    "ebsd_nlpar_average": (i32, [vp, i32, i32, i32, i64, i32, vp, i32, i32, i32, vp, i32, vp, i64, vp]),
    "ebsd_nlpar_workspace_bytes": (sz, [i32, i32]),
    "ebsd_pcfit_prep": (i32, [vp, i32, i32, i32, i32, i32, i32, i32, i32, vp, vp]),
    "ebsd_pcfit_reduce": (i32, [vp, i32, i32, i32, i32, i64, vp, vp, vp]),
    "ebsd_pcfit_xcorr_table_bytes": (i64, [i32, i32]),
    "ebsd_pcfit_xcorr_tables": (i32, [i32, i32, vp, i64, vp]),
    "ebsd_pcfit_spectra": (i32, [vp, i64, i64, i32, i32, vp, vp, vp, vp]),
    "ebsd_pcfit_pattern_terms": (i32, [vp, i64, i32, i32, vp, vp]),
    "ebsd_pcfit_xcorr_max": (i32, [vp, i64, vp, i32, i32, i32, vp, vp, i64, vp, vp]),
    "ebsd_pcfit_fold": (i32, [vp, i64, vp, vp, vp]),
    "ebsd_nlpar_weights": (i32, [vp, i32, i32, i32, vp, i32, f32, f32, f32, vp, sz, vp]),
    "ebsd_local_search": (i32, [vp, i64, i64, vp, i32, i32, vp, vp, vp, i64, vp, i32, i64, vp, vp, i32, i64, i32,
                                i32, f32, i32, vp, vp, vp, vp]),
    "ebsd_zh_to_qu": (i32, [vp, i64, vp, vp, vp]),
    "ebsd_qu_to_zh": (i32, [vp, i64, vp, vp]),
    "ebsd_rot6d_sym_loss": (i32, [vp, vp, i64, i32, f32, vp, vp, vp]),
    "ebsd_cnn_im2col": (i32, [vp, i32, i32, i32, i32, i64, i32, vp, vp]),
    "ebsd_cnn_col2im": (i32, [vp, i64, i32, i32, i32, i32, vp, vp]),
    "ebsd_cnn_bias_act": (i32, [vp, i64, vp, i64, i32, i32, vp, i64, vp, vp]),
    "ebsd_cnn_conv_c1": (i32, [vp, i32, i32, i32, vp, i32, vp, i32, i32, vp, vp, vp]),
    "ebsd_cnn_conv_fwd": (i32, [vp, i64, vp, i64, i64, vp, i32, i64, i32, vp, i64, vp, i32, vp, vp]),
    "ebsd_cnn_relu_grad": (i32, [vp, i64, vp, i64, i64, i32, vp, vp, i64, vp]),
    "ebsd_cnn_col_sum": (i32, [vp, i64, i32, vp, vp]),
    "ebsd_cnn_transpose": (i32, [vp, i32, i64, i64, i64, vp, i64, i64, vp]),
    "ebsd_cnn_scale_cast": (i32, [vp, i64, f32, vp, vp]),
    "ebsd_cnn_dense_fwd": (i32, [vp, i64, vp, vp, i32, i32, i32, i32, vp, vp, vp]),
    "ebsd_cnn_dense_bwd": (i32, [vp, vp, i64, vp, i32, i32, i32, vp, vp, vp, vp]),
    "ebsd_cnn_adam": (i32, [vp, vp, vp, vp, i64, i32, f32, f32, f32, f32, i32, f32, vp, i64, vp, i64, vp]),
}

DT_F32, DT_BF16, DT_E4M3 = 0, 1, 2
SIM_DOT, SIM_COSINE, SIM_EUCLIDEAN, SIM_MANHATTAN = 0, 1, 2, 3
DEVICE_TIMEOUT = 0x7001

# kernels launched by one successful call of each entry point
LAUNCHES_PER_CALL = {
    "ebsd_grid_fz_count": 2, "ebsd_grid_fz_write": 1, "ebsd_gather_rows": 1, "ebsd_project_dictionary": 1,
    "ebsd_prep_patterns": 1, "ebsd_prep_patterns_typed": 1, "ebsd_sample_master_pattern": 1, "ebsd_avg_pool": 1,
    "ebsd_match_topk": 1, "ebsd_match_topk_tiled": 1,
    "ebsd_merge_rescore": 1, "ebsd_merge_rescore_gated": 1, "ebsd_manhattan_topk": 1, "ebsd_gemm_nt": 1, "ebsd_gemm_f32": 1, "ebsd_col_mean": 1, "ebsd_split3_bf16": 1,
    "ebsd_disori_angle": 1, "ebsd_match_topk_noalloc": 2, "ebsd_zh_to_qu": 1, "ebsd_qu_to_zh": 1,
    "ebsd_cell_to_row": 2, "ebsd_local_search": 1, "ebsd_refine_grid": 1,
    "ebsd_pattern_mean": 2, "ebsd_subtract_pattern": 1, "ebsd_normalize_patterns": 1, "ebsd_clahe": 1,
    "ebsd_nlpar_dists": 1, "ebsd_nlpar_average": 1, "ebsd_nlpar_weights": 14,
    "ebsd_pcfit_prep": 1, "ebsd_pcfit_reduce": 1, "ebsd_pcfit_xcorr_tables": 1, "ebsd_pcfit_spectra": 1,
    "ebsd_pcfit_pattern_terms": 1, "ebsd_pcfit_xcorr_max": 1, "ebsd_pcfit_fold": 1,
    "ebsd_rot6d_sym_loss": 1, "ebsd_cnn_im2col": 1, "ebsd_cnn_col2im": 1, "ebsd_cnn_bias_act": 1,
    "ebsd_cnn_conv_fwd": 1, "ebsd_cnn_conv_c1": 1, "ebsd_cnn_relu_grad": 1, "ebsd_cnn_col_sum": 1,
    "ebsd_cnn_transpose": 1, "ebsd_cnn_scale_cast": 1,
    "ebsd_cnn_dense_fwd": 1, "ebsd_cnn_dense_bwd": 2, "ebsd_cnn_adam": 1,
}
launch_count = 0  # running total of kernels launched through call()

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load (once) and return the library; raises ImportError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} not found: build it with `python -m ebsdtorch_b200.build` "
                    "(CUDA toolkit with sm_100a support required)"
                )
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            # EBSD_MATCH_PAIRS=0/1 sets the match kernels' CTA-pair mode
            pairs = os.environ.get("EBSD_MATCH_PAIRS")
            if pairs is not None:
                lib.ebsd_set_match_pairs(0 if pairs.strip() in ("", "0") else 1)
            # EBSD_MATCH_DUAL=0/1/2: two query tiles per match CTA for no, all or
            # e4m3 (the default) launches
            dual = os.environ.get("EBSD_MATCH_DUAL")
            if dual is not None:
                lib.ebsd_set_match_dual({"": 0, "0": 0, "2": 2}.get(dual.strip(), 1))
            _lib = lib
    return _lib


def debug_check() -> tuple:
    """(line, file) of the first failed device check since the last call in
    the checking build, (0, "") when none, (-1, "") in the normal build."""
    buf = C.create_string_buffer(512)
    line = load().ebsd_debug_check_line(buf, len(buf))
    return line, buf.value.decode(errors="replace")


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(2048)
    lib.ebsd_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def call(name: str, *args) -> int:
    """Call an int-status entry point; raise on failure."""
    global launch_count
    fn = getattr(load(), name)
    rc = fn(*args)
    if rc == 0:
        launch_count += LAUNCHES_PER_CALL.get(name, 0)
    if rc > 0:
        raise ValueError(f"{name}: {last_error()}")
    if rc < 0:
        raise RuntimeError(f"{name}: {last_error()} (cudaError {-rc})")
    return rc


def ptr(t) -> int | None:
    """Device pointer of a tensor, or None for a missing optional buffer."""
    if t is None:
        return None
    return t.data_ptr()
