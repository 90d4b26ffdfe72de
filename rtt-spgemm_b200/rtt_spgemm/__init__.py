"""B200-native tiled FP64 SpGEMM - Python host mirror of the C ABI.

Function names and argument meanings follow the reference's tiled path
(for-the-juan/RTT-SpGEMM):

==========================  ===========================================
reference                   here (all run on the GPU through the C ABI)
==========================  ===========================================
csr2tile_row_major          csr2tile_row_major(csr) -> tile dict
csr2tile_col_major          csr2tile_col_major(csr) -> tile dict
spgemm_cpu(A, B, C)         spgemm_tile(a_tiles, b_tiles) -> tile dict
tile2csr(C, canonical)      tile2csr(tiles, tile_dim=8, canonical=...)
tile2csr_restore_rows       tile2csr(tiles, ..., new_to_old=perm)
dmma_tilespgemm 8x8 export  tile16_to_tile8(c_tiles)
device CSR -> CSR timed     Context.symbolic / Context.numeric
==========================  ===========================================

Tile matrices are dicts of numpy arrays keyed by SMatrix field name.  Errors
raise :class:`RttError` carrying the rtt_status code.
"""
from __future__ import annotations

import ctypes as C
import weakref
from types import SimpleNamespace

import numpy as np

from . import generators
from ._abi import (EXPORTS, LIB_PATH, RTT_OP_AAT, RTT_OP_AB, RTT_SUPER16_A8X4, RTT_SUPER16_B4X8,
                   RTT_REORDER_FULL, RTT_REORDER_COARSE, RTT_REORDER_FINE, RTT_REORDER_COARSE_ROW,
                   RTT_REORDER_COARSE_INNER, RTT_REORDER_UNGUARDED,
                   Super16Index, Config, CsrView, EarlySplitPlan,
                   HybridTiles, ReorderPlan, RttError, SMatrix, Stats, TailCostModel, TailPlan,
                   TailPolicy, build, check, lib)
from .generators import CSR

__all__ = ["CSR", "Context", "RttError", "build", "csr2tile_col_major", "csr2tile_row_major",
           "mmio_read",
           "generators", "lib", "spgemm_csr_host", "spgemm_tile", "tile16_to_tile8", "tile2csr",
           "tile2csr_device_noalloc", "csr_to_hybrid_tiles", "super16_index", "plan_tail_queue",
           "plan_early_split", "early_split_policy_default",
           "TAIL_POLICY_DEFAULT", "TAIL_MODEL_DEFAULT", "spgemm_batched",
           "EXPORTS", "LIB_PATH", "RTT_OP_AB", "RTT_OP_AAT", "RTT_REORDER_FULL",
           "RTT_REORDER_COARSE", "RTT_REORDER_FINE", "RTT_REORDER_COARSE_ROW",
           "RTT_REORDER_COARSE_INNER", "RTT_REORDER_UNGUARDED"]

TD = 16


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _adopt(p, count: int, dtype) -> np.ndarray:
    """numpy view of an array the library malloc'd; the memory is freed when
    the last view of it goes away (no copy of large outputs)."""
    addr = C.cast(p, C.c_void_p).value if p else None
    if count <= 0 or not addr:
        if addr:
            _libc_free(addr)
        return np.zeros(max(count, 0), dtype=dtype)
    buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(addr)
    weakref.finalize(buf, _libc_free, addr)
    return np.frombuffer(buf, dtype=dtype, count=count)


def _copy(p, count: int, dtype) -> np.ndarray:
    if count <= 0 or not p:
        return np.zeros(max(count, 0), dtype=dtype)
    return np.ctypeslib.as_array(p, shape=(count,)).astype(dtype, copy=True)


def _csr_smatrix(csr):
    rp = np.ascontiguousarray(csr.rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(csr.col, dtype=np.int32)
    v = np.ascontiguousarray(csr.val, dtype=np.float64)
    s = SMatrix()
    s.m, s.n, s.nnz = csr.m, csr.n, int(ci.shape[0])
    s.rowpointer, s.columnindex, s.value = _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v, C.c_double)
    return s, (rp, ci, v)


def _tiles_out(s: SMatrix, ptr_stride: int = TD, csc: bool = False) -> dict:
    nt = s.numtile
    d = {
        "m": s.m, "n": s.n, "nnz": s.nnz, "tilem": s.tilem, "tilen": s.tilen, "numtile": nt,
        "tile_ptr": _copy(s.tile_ptr, s.tilem + 1, np.int32),
        "tile_columnidx": _copy(s.tile_columnidx, nt, np.int32),
        "tile_nnz": _copy(s.tile_nnz, nt + 1, np.int32),
        "tile_csr_Ptr": _copy(s.tile_csr_Ptr, nt * ptr_stride, np.uint8),
        "tile_csr_Col": _copy(s.tile_csr_Col, s.nnz, np.uint8),
        "tile_csr_Value": _copy(s.tile_csr_Value, s.nnz, np.float64),
    }
    if s.tile_rowidx:
        d["tile_rowidx"] = _copy(s.tile_rowidx, nt, np.int32)
    if s.mask:
        d["mask"] = _copy(s.mask, nt * ptr_stride, np.uint16)
    if csc:
        d["csc_tile_ptr"] = _copy(s.csc_tile_ptr, s.tilen + 1, np.int32)
        d["csc_tile_rowidx"] = _copy(s.csc_tile_rowidx, nt, np.int32)
    return d


def _tiles_in(t: dict):
    s = SMatrix()
    keep = []
    s.m, s.n, s.nnz = t["m"], t["n"], t["nnz"]
    s.tilem, s.tilen, s.numtile = t["tilem"], t["tilen"], t["numtile"]
    for name, ct in [("tile_ptr", C.c_int), ("tile_columnidx", C.c_int), ("tile_rowidx", C.c_int),
                     ("tile_nnz", C.c_int), ("tile_csr_Value", C.c_double),
                     ("tile_csr_Col", C.c_ubyte), ("tile_csr_Ptr", C.c_ubyte),
                     ("mask", C.c_ushort), ("csc_tile_ptr", C.c_int), ("csc_tile_rowidx", C.c_int)]:
        if name in t:
            a = np.ascontiguousarray(t[name])
            if a.size == 0:
                a = np.zeros(1, dtype=a.dtype)
            keep.append(a)
            setattr(s, name, _ptr(a, ct))
    return s, keep


def _destroy(s: SMatrix, owned_csr: bool = False) -> None:
    lib().rtt_matrix_destroy(C.byref(s), int(owned_csr))


def mmio_read(path, value_mode: int = 0) -> CSR:
    """Replacement of mmio_allinone (reference src/mmio_highlevel.h:593): a
    Matrix Market coordinate file as CSR, the reference's layout (entries in
    file order, symmetric files expanded); value_mode 1 = the reference
    benchmark's value overwrite i % 10.  Returns CSR with .is_symmetric."""
    s = SMatrix()
    check(lib().rtt_mmio_read(str(path).encode(), int(value_mode), C.byref(s)))
    out = CSR(s.m, s.n, _adopt(s.rowpointer, s.m + 1, np.int32),
              _adopt(s.columnindex, s.nnz, np.int32), _adopt(s.value, s.nnz, np.float64))
    out.is_symmetric = bool(s.isSymmetric)
    return out


def csr2tile_row_major(csr) -> dict:
    """GPU replacement of csr2tile_row_major (reference src/csr2tile.h:196)."""
    s, keep = _csr_smatrix(csr)
    check(lib().rtt_csr2tile_row_major(C.byref(s)))
    d = _tiles_out(s)
    _destroy(s)
    return d


def csr2tile_col_major(csr) -> dict:
    """GPU replacement of csr2tile_col_major (reference src/csr2tile.h:261)."""
    s, keep = _csr_smatrix(csr)
    check(lib().rtt_csr2tile_col_major(C.byref(s)))
    d = _tiles_out(s, csc=True)
    _destroy(s)
    return d


def spgemm_tile(a_tiles: dict, b_tiles: dict) -> dict:
    """GPU replacement of spgemm_cpu(A, B, C) (reference src/spgemm-cpu.h:369):
    A from csr2tile_row_major, B from csr2tile_col_major; returns C's 16x16 tiles."""
    sa, ka = _tiles_in(a_tiles)
    sb, kb = _tiles_in(b_tiles)
    sc = SMatrix()
    check(lib().rtt_spgemm_tile(C.byref(sa), C.byref(sb), C.byref(sc)))
    d = _tiles_out(sc)
    _destroy(sc)
    return d


def tile2csr(tiles: dict, tile_dim: int = 8, canonical: bool = False, new_to_old=None,
             perm_size: int | None = None):
    """GPU replacement of tile2csr / tile2csr_restore_rows (reference
    src/tile2csr.h:232, :337).  Returns a namespace with m, n, rowptr, col, val."""
    s, keep = _tiles_in(tiles)
    if new_to_old is None:
        check(lib().rtt_tile2csr(C.byref(s), tile_dim, int(canonical)))
    else:
        p = np.ascontiguousarray(new_to_old, dtype=np.int32)
        size = p.shape[0] if perm_size is None else perm_size
        check(lib().rtt_tile2csr_restore_rows(C.byref(s), _ptr(p, C.c_int), size, tile_dim,
                                              int(canonical)))
    return SimpleNamespace(m=s.m, n=s.n, rowptr=_adopt(s.rowpointer, s.m + 1, np.int32),
                           col=_adopt(s.columnindex, s.nnz, np.int32),
                           val=_adopt(s.value, s.nnz, np.float64))


_LIBC = C.CDLL(None)
_LIBC.free.argtypes = [C.c_void_p]
_LIBC.free.restype = None


def _libc_free(p) -> None:
    _LIBC.free(p)


def tile16_to_tile8(c_tiles: dict) -> dict:
    """16x16 C tiles -> the reference's native 8x8 output tiles."""
    s, keep = _tiles_in(c_tiles)
    o = SMatrix()
    check(lib().rtt_tile16_to_tile8(C.byref(s), C.byref(o)))
    d = _tiles_out(o, ptr_stride=8)
    _destroy(o)
    return d


HYBRID_FIELDS = ("tile_row_ptr", "tile_col_idx", "value_offsets", "masks", "values",
                 "tile_col_ptr", "tile_row_idx", "csc_tile_ids")


def hybrid_dict(h) -> dict:
    """A HybridTiles structure (either library's) as a dict of numpy arrays."""
    d = {k: getattr(h, k) for k in ("rows", "cols", "tile_rows", "tile_cols", "tile_row_count",
                                    "tile_col_count", "num_tiles", "payload_size", "dense_tiles",
                                    "sparse_tiles")}
    nt = h.num_tiles
    sizes = {"tile_row_ptr": h.tile_row_count + 1, "tile_col_idx": nt, "value_offsets": nt + 1,
             "masks": nt, "values": h.payload_size, "tile_col_ptr": h.tile_col_count + 1,
             "tile_row_idx": nt, "csc_tile_ids": nt}
    types = {"masks": np.uint32, "values": np.float64}
    for k in HYBRID_FIELDS:
        p = getattr(h, k)
        d[k] = _copy(p, sizes[k], types.get(k, np.int32)) if p else None
    return d


def csr_to_hybrid_tiles(csr, tile_rows: int = 8, tile_cols: int = 4, col_major: bool = False,
                        dense_threshold: int = 24, build_csc: bool = False) -> dict:
    """GPU replacement of csr_to_hybrid_tiles (reference src/dmma_tiles.h:243):
    A uses (8, 4, row-major payload), B (4, 8, column-major payload)."""
    s, keep = _csr_smatrix(csr)
    h = HybridTiles()
    check(lib().rtt_csr_to_hybrid_tiles(C.byref(s), tile_rows, tile_cols, int(col_major),
                                        dense_threshold, int(build_csc), C.byref(h)))
    d = hybrid_dict(h)
    lib().rtt_hybrid_tiles_destroy(C.byref(h))
    return d


def _hybrid_struct(d: dict):
    """A HybridTiles structure over the numpy arrays of a hybrid dict (kept
    alive by the returned list)."""
    h = HybridTiles()
    for k in ("rows", "cols", "tile_rows", "tile_cols", "tile_row_count", "tile_col_count",
              "num_tiles", "payload_size", "dense_tiles", "sparse_tiles"):
        setattr(h, k, int(d[k]))
    keep = []
    types = {"masks": (np.uint32, C.c_uint), "values": (np.float64, C.c_double)}
    for k in HYBRID_FIELDS:
        if d.get(k) is None:
            continue
        nt, ct = types.get(k, (np.int32, C.c_int))
        a = np.ascontiguousarray(d[k], dtype=nt)
        if a.size == 0:
            a = np.zeros(1, dtype=nt)
        keep.append(a)
        setattr(h, k, _ptr(a, ct))
    return h, keep


def super16_index(leaf: dict, role: int) -> dict:
    """GPU replacement of build_device_index (reference
    src/super16_symbolic.cuh:2123): the 16x16 parent index of hybrid leaf tiles
    (a dict from csr_to_hybrid_tiles; 8x4 leaves for RTT_SUPER16_A8X4, 4x8 for
    RTT_SUPER16_B4X8)."""
    h, keep = _hybrid_struct(leaf)
    x = Super16Index()
    check(lib().rtt_super16_index_build(C.byref(h), role, C.byref(x)))
    pc, pr, pcol, nt = x.parent_count, x.parent_row_count, x.parent_col_count, int(leaf["num_tiles"])
    d = {k: getattr(x, k) for k in ("role", "rows", "cols", "parent_row_count",
                                    "parent_col_count", "parent_count")}
    d["row_ptr"] = _copy(x.row_ptr, pr + 1, np.uint64)
    d["col_idx"] = _copy(x.col_idx, pc, np.uint32)
    d["child_ptr"] = _copy(x.child_ptr, pc + 1, np.uint64)
    d["child_mask"] = _copy(x.child_mask, pc, np.uint8)
    d["child_leaf_ids"] = _copy(x.child_leaf_ids, nt, np.uint32)
    d["boolean_row_masks"] = _copy(x.boolean_row_masks, pc * 16, np.uint16)
    if role == RTT_SUPER16_B4X8:
        d["col_ptr"] = _copy(x.col_ptr, pcol + 1, np.uint64)
        d["row_idx"] = _copy(x.row_idx, pc, np.uint32)
        d["csc_parent_ids"] = _copy(x.csc_parent_ids, pc, np.uint32)
    else:
        d["col_ptr"] = d["row_idx"] = d["csc_parent_ids"] = None
    lib().rtt_super16_index_destroy(C.byref(x))
    del keep
    return d


# the reference's defaults (src/dmma_tile_tail_queue.h:20-40), enabled
TAIL_POLICY_DEFAULT = dict(enabled=1, admission_threshold=256.0, chunk_target=256.0, max_chunks=8,
                           max_heavy_fraction=0.01, record_capacity=1 << 20,
                           workspace_limit_bytes=1 << 30, workspace_reduction=1)
TAIL_MODEL_DEFAULT = dict(intercept=0.0, scan=1.0, match=8.0, output=0.25)


def plan_tail_queue(scans, matches, output_nnz, policy: dict | None = None,
                    model: dict | None = None):
    """GPU replacement of dmma_plan_tile_tail_queue (reference
    src/dmma_tile_tail_queue.h:190).  Returns (chunks per task, plan dict)."""
    sc = np.ascontiguousarray(scans, dtype=np.int32)
    mt = np.ascontiguousarray(matches, dtype=np.int32)
    on = np.ascontiguousarray(output_nnz, dtype=np.int32)
    n = int(sc.shape[0])
    pol = TailPolicy(**{**TAIL_POLICY_DEFAULT, **(policy or {})})
    mod = TailCostModel(**{**TAIL_MODEL_DEFAULT, **(model or {})})
    chunks = np.zeros(max(n, 1), np.int32)
    plan = TailPlan()
    check(lib().rtt_plan_tail_queue(n, _ptr(sc, C.c_int), _ptr(mt, C.c_int), _ptr(on, C.c_int),
                                    C.byref(pol), C.byref(mod), _ptr(chunks, C.c_int),
                                    C.byref(plan)))
    return chunks[:n], {k: getattr(plan, k) for k, _ in TailPlan._fields_}


def early_split_policy_default() -> dict:
    """The reference's early-split policy defaults (rtt_early_split_policy_default)."""
    pol = TailPolicy()
    lib().rtt_early_split_policy_default(C.byref(pol))
    return {k: getattr(pol, k) for k, _ in TailPolicy._fields_}


def plan_early_split(scans, matches, output_nnz, policy: dict | None = None,
                     model: dict | None = None, sm_count: int = 148):
    """Replacement of dmma_plan_tile_early_split (reference
    src/dmma_tile_early_split.h:152).  Returns (chunks per task, plan dict)."""
    sc = np.ascontiguousarray(scans, dtype=np.int32)
    mt = np.ascontiguousarray(matches, dtype=np.int32)
    on = np.ascontiguousarray(output_nnz, dtype=np.int32)
    n = int(sc.shape[0])
    pol = TailPolicy(**{**early_split_policy_default(), **(policy or {})})
    mod = TailCostModel(**{**TAIL_MODEL_DEFAULT, **(model or {})})
    chunks = np.zeros(max(n, 1), np.int32)
    plan = EarlySplitPlan()
    check(lib().rtt_plan_early_split(n, _ptr(sc, C.c_int), _ptr(mt, C.c_int), _ptr(on, C.c_int),
                                     C.byref(pol), C.byref(mod), int(sm_count),
                                     _ptr(chunks, C.c_int), C.byref(plan)))
    return chunks[:n], {k: getattr(plan, k) for k, _ in EarlySplitPlan._fields_}


def tile2csr_device_noalloc(tiles: dict, rowptr, col=None, val=None, tile_dim: int = 16,
                            canonical: bool = False, stream: int = 0) -> int:
    """tile2csr on device tiles into caller-owned device buffers, allocating
    nothing (rtt_tile2csr_device_noalloc).  ``tiles`` holds m, n, tilem,
    numtile, nnz and torch CUDA tensors tile_ptr, tile_columnidx, tile_nnz,
    tile_csr_Ptr, tile_csr_Col, tile_csr_Value; rowptr (m + 1 int32) is always
    written; col/val None asks for the size only.  Returns nnz of the CSR."""
    s = SMatrix()
    s.m, s.n, s.nnz = tiles["m"], tiles["n"], tiles["nnz"]
    s.tilem, s.numtile = tiles["tilem"], tiles["numtile"]
    for name, ct in [("tile_ptr", C.c_int), ("tile_columnidx", C.c_int), ("tile_nnz", C.c_int),
                     ("tile_csr_Ptr", C.c_ubyte), ("tile_csr_Col", C.c_ubyte),
                     ("tile_csr_Value", C.c_double)]:
        setattr(s, name, C.cast(C.c_void_p(tiles[name].data_ptr()), C.POINTER(ct)))
    s.rowpointer = C.cast(C.c_void_p(rowptr.data_ptr()), C.POINTER(C.c_int))
    cap = 0
    if col is not None:
        s.columnindex = C.cast(C.c_void_p(col.data_ptr()), C.POINTER(C.c_int))
        s.value = C.cast(C.c_void_p(val.data_ptr()), C.POINTER(C.c_double))
        cap = min(int(col.numel()), int(val.numel()))
    nnz = C.c_longlong()
    check(lib().rtt_tile2csr_device_noalloc(C.byref(s), tile_dim, int(canonical), cap,
                                            C.byref(nnz), C.c_void_p(stream)))
    return nnz.value


class Context:
    """Device-resident product: device CSR in -> device CSR out, two phases.

    Operands are torch CUDA tensors (int32 row_ptr / col_idx, float64 values);
    torch only provides device memory and the stream here.
    """

    def __init__(self, device: int = 0, config: dict | None = None, stream=None):
        h = C.c_void_p()
        check(lib().rtt_context_create(C.byref(h), device))
        self.handle = h
        self.device = device
        self.configure(config)
        if stream is not None:
            check(lib().rtt_context_set_stream(self.handle, C.c_void_p(stream)))

    def configure(self, config: dict | None = None):
        """rtt_config from the defaults plus the given fields."""
        cfg = Config()
        lib().rtt_config_default(C.byref(cfg))
        for k, v in (config or {}).items():
            setattr(cfg, k, int(v))
        check(lib().rtt_context_set_config(self.handle, C.byref(cfg)))
        self.config = {k: getattr(cfg, k) for k, _ in Config._fields_}

    def close(self):
        if self.handle:
            lib().rtt_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trim(self):
        """rtt_context_trim: release the context's grown device buffers."""
        check(lib().rtt_context_trim(self.handle))

    def set_stream(self, stream_ptr: int):
        check(lib().rtt_context_set_stream(self.handle, C.c_void_p(stream_ptr)))

    @staticmethod
    def _view(rows, cols, rowptr, col, val) -> CsrView:
        return CsrView(rows, cols, int(col.numel()), rowptr.data_ptr(), col.data_ptr(),
                       val.data_ptr())

    def symbolic(self, a, b=None, op: int = RTT_OP_AB):
        """a, b: (rows, cols, rowptr, col, val) with device tensors.  The
        operands stay borrowed by the library until numeric() returns; the
        context keeps references to them until then."""
        va = self._view(*a)
        vb = self._view(*b) if b is not None else None
        nnz = C.c_longlong()
        tiles = C.c_longlong()
        self._borrowed = (a, b)
        check(lib().rtt_spgemm_symbolic(self.handle, C.byref(va), C.byref(vb) if vb else None,
                                        op, C.byref(nnz), C.byref(tiles)))
        return nnz.value, tiles.value

    def numeric(self, rowptr, col, val):
        try:
            check(lib().rtt_spgemm_numeric(self.handle, C.c_void_p(rowptr.data_ptr()),
                                           C.c_void_p(col.data_ptr()),
                                           C.c_void_p(val.data_ptr())))
        finally:
            self._borrowed = None

    def update_b(self, b, row_new_to_old=None):
        """rtt_spgemm_update_b: the last symbolic's A with a new B (structure
        mode), or B's rows in the order row_new_to_old (a device int32 tensor:
        permutation mode).  Returns (nnz, tiles) of C; numeric() follows."""
        vb = self._view(*b)
        nnz = C.c_longlong()
        tiles = C.c_longlong()
        a = self._borrowed[0] if getattr(self, "_borrowed", None) else None
        self._borrowed = (a, b, row_new_to_old)
        ptr = C.c_void_p(row_new_to_old.data_ptr()) if row_new_to_old is not None else None
        check(lib().rtt_spgemm_update_b(self.handle, C.byref(vb), ptr, C.byref(nnz),
                                        C.byref(tiles)))
        return nnz.value, tiles.value

    def symbolic64(self, a, b=None, op: int = RTT_OP_AB) -> int:
        """rtt_spgemm_symbolic64: phase 1 of a product whose C may exceed
        INT32_MAX entries (chunked over A's tile rows).  Returns nnz(C)."""
        va = self._view(*a)
        vb = self._view(*b) if b is not None else None
        nnz = C.c_longlong()
        self._borrowed = (a, b)
        check(lib().rtt_spgemm_symbolic64(self.handle, C.byref(va), C.byref(vb) if vb else None,
                                          op, C.byref(nnz)))
        return nnz.value

    def numeric64(self, rowptr, col, val):
        """rtt_spgemm_numeric64: C into device tensors rowptr (rows + 1,
        int64), col (int32) and val (float64) of nnz(C) entries."""
        try:
            check(lib().rtt_spgemm_numeric64(self.handle, C.c_void_p(rowptr.data_ptr()),
                                             C.c_void_p(col.data_ptr()),
                                             C.c_void_p(val.data_ptr())))
        finally:
            self._borrowed = None

    def numeric_values(self, a_values, b_values, rowptr, col, val):
        """rtt_spgemm_numeric_values: the last symbolic's product with new values
        of A (device tensor in A's CSR order) and of B (or None).  The caller
        keeps the structure tensors given to symbolic() alive meanwhile."""
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        check(lib().rtt_spgemm_numeric_values(self.handle, ptr(a_values), ptr(b_values),
                                              ptr(rowptr), ptr(col), ptr(val)))

    def batched_symbolic(self, As, Bs=None):
        """Batched form: As (and Bs) are lists of (rows, cols, rowptr, col, val)
        device tuples.  Returns (nnz per instance, total nnz).  The operands
        stay borrowed until batched_numeric() returns."""
        count = len(As)
        va = (CsrView * count)(*[self._view(*a) for a in As])
        vb = (CsrView * count)(*[self._view(*b) for b in Bs]) if Bs is not None else None
        nnz = (C.c_longlong * count)()
        tot = C.c_longlong()
        self._borrowed = (As, Bs)
        check(lib().rtt_spgemm_batched_symbolic(self.handle, count, va, vb, nnz, C.byref(tot)))
        return list(nnz), tot.value

    def batched_numeric(self, rowptr, col, val):
        try:
            check(lib().rtt_spgemm_batched_numeric(self.handle, C.c_void_p(rowptr.data_ptr()),
                                                   C.c_void_p(col.data_ptr()),
                                                   C.c_void_p(val.data_ptr())))
        finally:
            self._borrowed = None

    def batched_numeric_values(self, a_values, b_values, rowptr, col, val):
        """rtt_spgemm_batched_numeric_values: the last batch again with new
        values of every A_i (device tensors, each in its CSR order) and of
        every B_i (or None), into the same kind of outputs as
        batched_numeric()."""
        n = len(a_values)
        pa = (C.c_void_p * n)(*[t.data_ptr() for t in a_values])
        pb = (C.c_void_p * n)(*[t.data_ptr() for t in b_values]) if b_values is not None else None
        check(lib().rtt_spgemm_batched_numeric_values(self.handle, pa, pb,
                                                      C.c_void_p(rowptr.data_ptr()),
                                                      C.c_void_p(col.data_ptr()),
                                                      C.c_void_p(val.data_ptr())))

    def tile_heatmap(self, which: str = "C", bins: int = 64) -> np.ndarray:
        """rtt_tile_heatmap: tile counts of A, B or C of the last symbolic
        phase on a bins x bins grid."""
        h = np.zeros(bins * bins, dtype=np.uint64)
        check(lib().rtt_tile_heatmap(self.handle, {"A": 0, "B": 1, "C": 2}[which], int(bins),
                                     h.ctypes.data_as(C.POINTER(C.c_ulonglong))))
        return h.reshape(bins, bins)

    def reorder_plan_dump(self, a, stem: str, dump_matrix: bool = True) -> dict:
        """Build A's reorder plan and write it as the reference's dump does
        (rtt_reorder_plan_dump: <stem>_permutations.csv, _unified_stats.csv,
        _A_reordered.mtx).  Returns the plan."""
        v = self._view(*a)
        p = ReorderPlan()
        check(lib().rtt_reorder_plan_build(self.handle, C.byref(v), C.byref(p)))
        try:
            check(lib().rtt_reorder_plan_dump(C.byref(p), str(stem).encode(),
                                              C.c_void_p(a[2].data_ptr()),
                                              C.c_void_p(a[3].data_ptr()), int(dump_matrix)))
            out = {k: getattr(p, k) for k, t in ReorderPlan._fields_
                   if t is not C.POINTER(C.c_int)}
            for k, n in (("row_old_to_new", p.rows), ("inner_old_to_new", p.cols)):
                out[k] = np.ctypeslib.as_array(getattr(p, k), shape=(n,)).copy() if n else \
                    np.zeros(0, np.int32)
        finally:
            lib().rtt_reorder_plan_destroy(C.byref(p))
        return out

    def reorder_plan(self, a, variant: int = 0) -> dict:
        """Row / inner reorder plan of a device CSR tuple (rtt_reorder_plan_build,
        the reference's build_dmma_reorder_plan), with the stages of variant
        (RTT_REORDER_*; 0 = all): counters and numpy maps."""
        v = self._view(*a)
        p = ReorderPlan()
        check(lib().rtt_reorder_plan_build_variant(self.handle, C.byref(v), int(variant),
                                                   C.byref(p)))
        out = {k: getattr(p, k) for k, t in ReorderPlan._fields_ if t is not C.POINTER(C.c_int)}
        for k, n in (("row_old_to_new", p.rows), ("row_new_to_old", p.rows),
                     ("inner_old_to_new", p.cols), ("inner_new_to_old", p.cols)):
            out[k] = np.ctypeslib.as_array(getattr(p, k), shape=(n,)).copy() if n else \
                np.zeros(0, np.int32)
        lib().rtt_reorder_plan_destroy(C.byref(p))
        return out

    def permute(self, a, row_new_to_old=None, col_old_to_new=None):
        """rtt_csr_permute: rows taken in row_new_to_old order, columns mapped by
        col_old_to_new (device int32 tensors or None), rows re-sorted."""
        import torch

        rows, cols, rp, ci, va = a
        nnz = int(ci.numel())
        orp = torch.empty(rows + 1, dtype=torch.int32, device=rp.device)
        oci = torch.empty(max(nnz, 1), dtype=torch.int32, device=rp.device)
        ova = torch.empty(max(nnz, 1), dtype=torch.float64, device=rp.device)
        v = self._view(*a)
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        check(lib().rtt_csr_permute(self.handle, C.byref(v), ptr(row_new_to_old),
                                    ptr(col_old_to_new), ptr(orp), ptr(oci), ptr(ova)))
        return (rows, cols, orp, oci[:nnz], ova[:nnz])

    def transpose(self, a):
        """A^T of a device CSR tuple, as a device CSR tuple (new tensors)."""
        import torch

        rows, cols, rp, ci, va = a
        trp = torch.empty(cols + 1, dtype=torch.int32, device=rp.device)
        tci = torch.empty(max(int(ci.numel()), 1), dtype=torch.int32, device=rp.device)
        tva = torch.empty(max(int(ci.numel()), 1), dtype=torch.float64, device=rp.device)
        v = self._view(*a)
        check(lib().rtt_csr_transpose(self.handle, C.byref(v), C.c_void_p(trp.data_ptr()),
                                      C.c_void_p(tci.data_ptr()), C.c_void_p(tva.data_ptr())))
        n = int(ci.numel())
        return (cols, rows, trp, tci[:n], tva[:n])

    def stats(self) -> dict:
        st = Stats()
        check(lib().rtt_context_get_stats(self.handle, C.byref(st)))
        return {k: getattr(st, k) for k, _ in Stats._fields_}

    def spgemm_csr_host(self, a, b=None, op: int = RTT_OP_AB):
        """Host CSR in -> host CSR out through the device path (copies inside)."""
        sa, ka = _csr_smatrix(a)
        sb, kb = _csr_smatrix(b) if b is not None else (None, None)
        sc = SMatrix()
        check(lib().rtt_spgemm_csr_host(self.handle, C.byref(sa),
                                        C.byref(sb) if sb is not None else None, op,
                                        C.byref(sc)))
        # C's arrays were malloc'd by the library: hand them to numpy as they are
        return CSR(sc.m, sc.n, _adopt(sc.rowpointer, sc.m + 1, np.int32),
                   _adopt(sc.columnindex, sc.nnz, np.int32), _adopt(sc.value, sc.nnz, np.float64))

    def spgemm_csr_host_into(self, a, out, b=None, op: int = RTT_OP_AB) -> int:
        """Host CSR in -> C into the caller's host arrays out = (rowptr, col,
        val) (numpy; page-locked ones take the DMA directly), reused from call
        to call (rtt_spgemm_csr_host_into).  Returns nnz(C); raises RttError
        when col / val are shorter than nnz(C) (the error says the size)."""
        sa, ka = _csr_smatrix(a)
        sb, kb = _csr_smatrix(b) if b is not None else (None, None)
        rp, col, val = out
        if rp.dtype != np.int32 or col.dtype != np.int32 or val.dtype != np.float64:
            raise TypeError("out arrays must be int32, int32, float64")
        if rp.size < a.m + 1:
            raise ValueError("out rowptr must hold m + 1 entries")
        cap = min(col.size, val.size)
        nnz = C.c_longlong(0)
        check(lib().rtt_spgemm_csr_host_into(
            self.handle, C.byref(sa), C.byref(sb) if sb is not None else None, op,
            C.c_void_p(rp.ctypes.data), C.c_void_p(col.ctypes.data) if cap else None,
            C.c_void_p(val.ctypes.data) if cap else None, cap, C.byref(nnz)))
        return int(nnz.value)


def spgemm_batched(ctx: "Context", As, Bs=None, tuner=None):
    """C_i = A_i * B_i (or A_i^2) for a list of device CSR tuples, through one
    pipeline run.  Returns per-instance (rowptr, col, val) device tensor views
    of three concatenated output buffers.  With a tuner (autotune.Tuner) the
    context takes the tuned configuration of the batch's shape class first."""
    import torch

    if tuner is not None:
        tuner.configure_batch(ctx, As, Bs)
    nnz, total = ctx.batched_symbolic(As, Bs)
    dev = As[0][2].device
    rows = [int(a[0]) for a in As]
    rp = torch.empty(sum(r + 1 for r in rows), dtype=torch.int32, device=dev)
    col = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
    val = torch.empty(max(total, 1), dtype=torch.float64, device=dev)
    ctx.batched_numeric(rp, col, val)
    out, r0, e0 = [], 0, 0
    for r, z in zip(rows, nnz):
        out.append((rp[r0:r0 + r + 1], col[e0:e0 + z], val[e0:e0 + z]))
        r0 += r + 1
        e0 += z
    return out


def spgemm_csr_host(a, b=None, op: int = RTT_OP_AB, device: int = 0) -> CSR:
    ctx = Context(device)
    try:
        return ctx.spgemm_csr_host(a, b, op)
    finally:
        ctx.close()
