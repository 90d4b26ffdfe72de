"""ctypes binding of librtt_spgemm.so (include/rtt_spgemm.h).

The library is the product: every function here calls one extern "C" entry
point that runs sm_100a kernels.  If the shared library is missing, loading
fails loudly - there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent  # rtt-spgemm_b200/
LIB_PATH = PKG_ROOT / "librtt_spgemm.so"

RTT_OK = 0
RTT_OP_AB = 0
RTT_OP_AAT = 1
# reorder plan stages (rtt_reorder_plan_build_variant)
RTT_REORDER_FULL, RTT_REORDER_COARSE, RTT_REORDER_FINE = 0, 1, 2
RTT_REORDER_COARSE_ROW, RTT_REORDER_COARSE_INNER, RTT_REORDER_UNGUARDED = 3, 4, 5
STATUS = {
    0: "RTT_OK", 1: "RTT_ERR_INVALID_ARGUMENT", 2: "RTT_ERR_INVALID_CSR",
    3: "RTT_ERR_SHAPE_MISMATCH", 4: "RTT_ERR_OUT_OF_MEMORY", 5: "RTT_ERR_CUDA",
    6: "RTT_ERR_UNREPRESENTABLE", 7: "RTT_ERR_NO_DEVICE", 8: "RTT_ERR_DEVICE_CHECK",
    9: "RTT_ERR_INVALID_PERMUTATION", 10: "RTT_ERR_TAIL_NONEMPTY", 11: "RTT_ERR_STATE",
}

# Every symbol include/rtt_spgemm.h declares.
EXPORTS = [
    "rtt_status_string", "rtt_last_error", "rtt_version", "rtt_set_device",
    "rtt_csr2tile_row_major", "rtt_csr2tile_col_major", "rtt_spgemm_tile", "rtt_tile2csr",
    "rtt_tile2csr_restore_rows", "rtt_tile16_to_tile8", "rtt_matrix_destroy",
    "rtt_config_default", "rtt_context_create", "rtt_context_destroy", "rtt_context_set_stream",
    "rtt_context_set_config", "rtt_context_get_stats", "rtt_spgemm_symbolic",
    "rtt_spgemm_numeric", "rtt_spgemm_tiles_view", "rtt_spgemm_csr_host",
    "rtt_spgemm_csr_host_into",
    "rtt_tile2csr_device_noalloc", "rtt_csr_to_hybrid_tiles", "rtt_hybrid_tiles_destroy",
    "rtt_plan_tail_queue", "rtt_spgemm_batched_symbolic", "rtt_spgemm_batched_numeric",
    "rtt_csr_transpose", "rtt_early_split_policy_default", "rtt_plan_early_split",
    "rtt_reorder_plan_build", "rtt_reorder_plan_build_variant", "rtt_reorder_plan_destroy",
    "rtt_csr_permute",
    "rtt_spgemm_numeric_values", "rtt_super16_index_build", "rtt_super16_index_destroy",
    "rtt_spgemm_batched_numeric_values", "rtt_spgemm_symbolic64", "rtt_spgemm_numeric64",
    "rtt_spgemm_update_b", "rtt_mmio_read", "rtt_reorder_plan_dump", "rtt_tile_heatmap",
    "rtt_context_trim",
]

RTT_SUPER16_A8X4 = 1
RTT_SUPER16_B4X8 = 2


class RttError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class SMatrix(C.Structure):
    """The reference SMatrix (src/common.h:50-72), byte for byte."""

    _fields_ = [
        ("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int), ("isSymmetric", C.c_int),
        ("value", C.POINTER(C.c_double)), ("columnindex", C.POINTER(C.c_int)),
        ("rowpointer", C.POINTER(C.c_int)),
        ("tilem", C.c_int), ("tilen", C.c_int),
        ("tile_ptr", C.POINTER(C.c_int)), ("tile_columnidx", C.POINTER(C.c_int)),
        ("tile_rowidx", C.POINTER(C.c_int)), ("tile_nnz", C.POINTER(C.c_int)),
        ("numtile", C.c_int),
        ("tile_csr_Value", C.POINTER(C.c_double)), ("tile_csr_Col", C.POINTER(C.c_ubyte)),
        ("tile_csr_Ptr", C.POINTER(C.c_ubyte)), ("mask", C.POINTER(C.c_ushort)),
        ("csc_tile_ptr", C.POINTER(C.c_int)), ("csc_tile_rowidx", C.POINTER(C.c_int)),
    ]


class CsrView(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_longlong),
                ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("values", C.c_void_p)]


class Config(C.Structure):
    _fields_ = [("dmma_pair_cutoff", C.c_int), ("fused_csr_output", C.c_int),
                ("keep_tiles", C.c_int), ("stage_timing", C.c_int), ("b_staging", C.c_int),
                ("split_target", C.c_int), ("cuda_graphs", C.c_int),
                ("chunk_tiles", C.c_int), ("chunk_nnz", C.c_int),
                ("segment_walk", C.c_int), ("persistent_rows", C.c_int),
                ("sym_window_slots", C.c_int), ("leaf_dmma", C.c_int), ("global_rows", C.c_int)]


class HybridTiles(C.Structure):
    """rtt_hybrid_tiles = the reference's HybridTileMatrix (src/dmma_tiles.h:29-62)."""

    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("tile_rows", C.c_int),
                ("tile_cols", C.c_int), ("tile_row_count", C.c_int), ("tile_col_count", C.c_int),
                ("num_tiles", C.c_int), ("payload_size", C.c_int), ("dense_tiles", C.c_int),
                ("sparse_tiles", C.c_int),
                ("tile_row_ptr", C.POINTER(C.c_int)), ("tile_col_idx", C.POINTER(C.c_int)),
                ("value_offsets", C.POINTER(C.c_int)), ("masks", C.POINTER(C.c_uint)),
                ("values", C.POINTER(C.c_double)), ("tile_col_ptr", C.POINTER(C.c_int)),
                ("tile_row_idx", C.POINTER(C.c_int)), ("csc_tile_ids", C.POINTER(C.c_int))]


class Super16Index(C.Structure):
    """rtt_super16_index = the reference's Super16 DeviceIndexView
    (src/super16_symbolic.cuh:85-106) as host arrays."""

    _fields_ = [("role", C.c_uint), ("rows", C.c_int), ("cols", C.c_int),
                ("parent_row_count", C.c_uint), ("parent_col_count", C.c_uint),
                ("parent_count", C.c_uint),
                ("row_ptr", C.POINTER(C.c_ulonglong)), ("col_idx", C.POINTER(C.c_uint)),
                ("child_ptr", C.POINTER(C.c_ulonglong)), ("child_mask", C.POINTER(C.c_ubyte)),
                ("child_leaf_ids", C.POINTER(C.c_uint)),
                ("boolean_row_masks", C.POINTER(C.c_ushort)),
                ("col_ptr", C.POINTER(C.c_ulonglong)), ("row_idx", C.POINTER(C.c_uint)),
                ("csc_parent_ids", C.POINTER(C.c_uint))]


class TailPolicy(C.Structure):
    _fields_ = [("enabled", C.c_int), ("admission_threshold", C.c_double),
                ("chunk_target", C.c_double), ("max_chunks", C.c_int),
                ("max_heavy_fraction", C.c_double), ("record_capacity", C.c_int),
                ("workspace_limit_bytes", C.c_longlong), ("workspace_reduction", C.c_int)]


class TailCostModel(C.Structure):
    _fields_ = [("intercept", C.c_double), ("scan", C.c_double), ("match", C.c_double),
                ("output", C.c_double)]


class TailPlan(C.Structure):
    _fields_ = [("reason", C.c_int)] + [(k, C.c_longlong) for k in (
        "output_tasks", "ordinary_tasks", "heavy_tasks", "chunks", "descriptor_bytes",
        "heavy_flag_bytes", "partial_workspace_bytes")] + [
        ("heavy_fraction", C.c_double), ("average_chunks", C.c_double)]


class EarlySplitPlan(C.Structure):
    _fields_ = [("reason", C.c_int), ("base_reason", C.c_int)] + [(k, C.c_longlong) for k in (
        "output_tasks", "ordinary_tasks", "heavy_tasks", "chunks")] + [(k, C.c_int) for k in (
        "sm_count", "global_heavy_worker_block_cap", "heavy_worker_blocks",
        "reduction_worker_blocks")] + [(k, C.c_longlong) for k in (
        "descriptor_bytes", "heavy_flag_bytes", "partial_workspace_bytes")] + [
        ("exact_parent_partition", C.c_int)]


class ReorderPlan(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("rows", "cols", "nnz", "active_rows", "active_inner",
                                        "components", "levels", "accepted")] + [
        (k, C.c_longlong) for k in ("tiles_before", "tiles_after", "proposal_tiles",
                                    "moved_rows", "moved_inner")] + [
        (k, C.POINTER(C.c_int)) for k in ("row_old_to_new", "row_new_to_old", "inner_old_to_new",
                                          "inner_new_to_old")] + [
        (k, C.c_int) for k in ("variant", "row_windows", "accepted_row_windows",
                               "inner_windows", "accepted_inner_windows")] + [
        (k, C.c_longlong) for k in ("row_tile_reduction", "inner_tile_reduction",
                                    "row_fanout_before", "row_fanout_after",
                                    "inner_fanout_before", "inner_fanout_after")]


class Stats(C.Structure):
    _fields_ = [("nnz_a", C.c_longlong), ("nnz_b", C.c_longlong), ("nnz_c", C.c_longlong),
                ("nnz_cub", C.c_longlong), ("tiles_a", C.c_longlong),
                ("tiles_b", C.c_longlong), ("tiles_c", C.c_longlong),
                ("dmma_pairs", C.c_longlong), ("sparse_pairs", C.c_longlong),
                ("kernel_launches", C.c_int), ("host_syncs", C.c_int),
                ("csr2tile_ms", C.c_double), ("symbolic_ms", C.c_double),
                ("numeric_kernel_ms", C.c_double), ("split_windows", C.c_longlong),
                ("graph_launched", C.c_int), ("split_multi_window_tasks", C.c_longlong)]


def build(verbose: bool = False) -> Path:
    """Compile librtt_spgemm.so for sm_100a (nvcc cross-compiles without a GPU)."""
    out = subprocess.run(["make", "-s", "-j8", "-C", str(PKG_ROOT / "csrc")],
                         capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("building librtt_spgemm.so failed:\n" + (out.stderr or "")[-4000:])
    return LIB_PATH


_LIB = None


def lib() -> C.CDLL:
    """Load the C-ABI library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing; build it with rtt_spgemm.build()")
    L = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    L.rtt_status_string.restype = C.c_char_p
    L.rtt_status_string.argtypes = [C.c_int]
    L.rtt_last_error.restype = C.c_char_p
    L.rtt_version.restype = C.c_char_p
    L.rtt_set_device.argtypes = [C.c_int]
    for f in ("rtt_csr2tile_row_major", "rtt_csr2tile_col_major"):
        getattr(L, f).argtypes = [P(SMatrix)]
    L.rtt_spgemm_tile.argtypes = [P(SMatrix)] * 3
    L.rtt_tile2csr.argtypes = [P(SMatrix), C.c_int, C.c_int]
    L.rtt_tile2csr_restore_rows.argtypes = [P(SMatrix), P(C.c_int), C.c_int, C.c_int, C.c_int]
    L.rtt_tile16_to_tile8.argtypes = [P(SMatrix), P(SMatrix)]
    L.rtt_csr_to_hybrid_tiles.argtypes = [P(SMatrix), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          P(HybridTiles)]
    L.rtt_plan_tail_queue.argtypes = [C.c_int, P(C.c_int), P(C.c_int), P(C.c_int),
                                      P(TailPolicy), P(TailCostModel), P(C.c_int), P(TailPlan)]
    L.rtt_early_split_policy_default.argtypes = [P(TailPolicy)]
    L.rtt_early_split_policy_default.restype = None
    L.rtt_plan_early_split.argtypes = [C.c_int, P(C.c_int), P(C.c_int), P(C.c_int),
                                       P(TailPolicy), P(TailCostModel), C.c_int, P(C.c_int),
                                       P(EarlySplitPlan)]
    L.rtt_hybrid_tiles_destroy.argtypes = [P(HybridTiles)]
    L.rtt_hybrid_tiles_destroy.restype = None
    L.rtt_super16_index_build.argtypes = [P(HybridTiles), C.c_uint, P(Super16Index)]
    L.rtt_super16_index_destroy.argtypes = [P(Super16Index)]
    L.rtt_super16_index_destroy.restype = None
    L.rtt_tile2csr_device_noalloc.argtypes = [P(SMatrix), C.c_int, C.c_int, C.c_longlong,
                                              P(C.c_longlong), C.c_void_p]
    L.rtt_matrix_destroy.argtypes = [P(SMatrix), C.c_int]
    L.rtt_matrix_destroy.restype = None
    L.rtt_config_default.argtypes = [P(Config)]
    L.rtt_config_default.restype = None
    L.rtt_context_create.argtypes = [P(C.c_void_p), C.c_int]
    L.rtt_context_destroy.argtypes = [C.c_void_p]
    L.rtt_context_destroy.restype = None
    L.rtt_context_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    L.rtt_context_trim.argtypes = [C.c_void_p]
    L.rtt_context_set_config.argtypes = [C.c_void_p, P(Config)]
    L.rtt_context_get_stats.argtypes = [C.c_void_p, P(Stats)]
    L.rtt_spgemm_symbolic.argtypes = [C.c_void_p, P(CsrView), P(CsrView), C.c_int,
                                      P(C.c_longlong), P(C.c_longlong)]
    L.rtt_spgemm_numeric.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.rtt_mmio_read.argtypes = [C.c_char_p, C.c_int, P(SMatrix)]
    L.rtt_reorder_plan_dump.argtypes = [P(ReorderPlan), C.c_char_p, C.c_void_p, C.c_void_p,
                                        C.c_int]
    L.rtt_tile_heatmap.argtypes = [C.c_void_p, C.c_int, C.c_int, P(C.c_ulonglong)]
    L.rtt_spgemm_update_b.argtypes = [C.c_void_p, P(CsrView), C.c_void_p, P(C.c_longlong),
                                      P(C.c_longlong)]
    L.rtt_spgemm_symbolic64.argtypes = [C.c_void_p, P(CsrView), P(CsrView), C.c_int,
                                        P(C.c_longlong)]
    L.rtt_spgemm_numeric64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.rtt_spgemm_tiles_view.argtypes = [C.c_void_p, P(SMatrix)]
    L.rtt_spgemm_csr_host.argtypes = [C.c_void_p, P(SMatrix), P(SMatrix), C.c_int, P(SMatrix)]
    L.rtt_spgemm_csr_host_into.argtypes = [C.c_void_p, P(SMatrix), P(SMatrix), C.c_int,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong,
                                           P(C.c_longlong)]
    L.rtt_spgemm_batched_symbolic.argtypes = [C.c_void_p, C.c_int, P(CsrView), P(CsrView),
                                              P(C.c_longlong), P(C.c_longlong)]
    L.rtt_spgemm_batched_numeric.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.rtt_spgemm_batched_numeric_values.argtypes = [C.c_void_p, P(C.c_void_p), P(C.c_void_p),
                                                    C.c_void_p, C.c_void_p, C.c_void_p]
    L.rtt_csr_transpose.argtypes = [C.c_void_p, P(CsrView), C.c_void_p, C.c_void_p, C.c_void_p]
    L.rtt_spgemm_numeric_values.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p]
    L.rtt_reorder_plan_build.argtypes = [C.c_void_p, P(CsrView), P(ReorderPlan)]
    L.rtt_reorder_plan_build_variant.argtypes = [C.c_void_p, P(CsrView), C.c_int, P(ReorderPlan)]
    L.rtt_reorder_plan_destroy.argtypes = [P(ReorderPlan)]
    L.rtt_reorder_plan_destroy.restype = None
    L.rtt_csr_permute.argtypes = [C.c_void_p, P(CsrView), C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]
    _LIB = L
    return L


def check(status: int) -> None:
    if status != RTT_OK:
        msg = lib().rtt_last_error().decode(errors="replace")
        raise RttError(status, msg)
