"""ctypes front end of the CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and bench.py's
CPU-baseline leg as the checker.  The product (rtt-spgemm_b200/) never
imports it.

Two back ends share one numpy-level interface:

* ``Oracle``     liboracle.so, the C restatement (oracle.c) - always built.
* ``Reference``  oracle/_ref/libref_*.so, the reference's own CPU code
                 compiled unmodified from its sources (built only where the
                 reference checkout exists; the built files travel with the
                 repository snapshot).

Tile matrices are plain dicts of numpy arrays keyed by SMatrix field name.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
TD = 16


class SMatrix(C.Structure):
    """Same layout as SMatrix in include/rtt_spgemm.h (reference src/common.h:50-72)."""

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


_CT = {np.int32: C.c_int, np.float64: C.c_double, np.uint8: C.c_ubyte, np.uint16: C.c_ushort}


def _ptr(arr: np.ndarray, ctype):
    return arr.ctypes.data_as(C.POINTER(ctype))


def _copy(ptr, count: int, dtype) -> np.ndarray:
    if count <= 0 or not ptr:
        return np.zeros(max(count, 0), dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)


def csr_smatrix(csr):
    """SMatrix over the CSR arrays of ``csr`` (kept alive by the returned tuple)."""
    rp = np.ascontiguousarray(csr.rowptr, dtype=np.int32)
    ci = np.ascontiguousarray(csr.col, dtype=np.int32)
    v = np.ascontiguousarray(csr.val, dtype=np.float64)
    s = SMatrix()
    s.m, s.n, s.nnz = csr.m, csr.n, int(ci.shape[0])
    s.rowpointer, s.columnindex, s.value = _ptr(rp, C.c_int), _ptr(ci, C.c_int), _ptr(v, C.c_double)
    return s, (rp, ci, v)


def tiles_from_smatrix(s: SMatrix, ptr_stride: int = TD, csc: bool = False) -> dict:
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


def smatrix_from_tiles(t: dict):
    """SMatrix pointing at the arrays of a tile dict (plus keep-alive list)."""
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


class _Base:
    lib: C.CDLL

    def _free_tiles(self, s: SMatrix):
        for name in ("tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Value",
                     "tile_csr_Col", "tile_csr_Ptr", "mask", "csc_tile_ptr", "csc_tile_rowidx"):
            p = getattr(s, name)
            if p:
                self._free(C.cast(p, C.c_void_p))
                setattr(s, name, None)

    def _free_csr(self, s: SMatrix):
        for name in ("rowpointer", "columnindex", "value"):
            p = getattr(s, name)
            if p:
                self._free(C.cast(p, C.c_void_p))
                setattr(s, name, None)


class HybridTiles(C.Structure):
    """HybridTileMatrix flattened (oracle/ref_tiles.cpp ref_hybrid; the
    reference's src/dmma_tiles.h:29-62 with MAT_PTR_TYPE = int)."""

    _fields_ = [(k, C.c_int) for k in ("rows", "cols", "tile_rows", "tile_cols",
                                       "tile_row_count", "tile_col_count", "num_tiles",
                                       "payload_size", "dense_tiles", "sparse_tiles")] + [
        ("tile_row_ptr", C.POINTER(C.c_int)), ("tile_col_idx", C.POINTER(C.c_int)),
        ("value_offsets", C.POINTER(C.c_int)), ("masks", C.POINTER(C.c_uint)),
        ("values", C.POINTER(C.c_double)), ("tile_col_ptr", C.POINTER(C.c_int)),
        ("tile_row_idx", C.POINTER(C.c_int)), ("csc_tile_ids", C.POINTER(C.c_int))]


HYBRID_FIELDS = ("tile_row_ptr", "tile_col_idx", "value_offsets", "masks", "values",
                 "tile_col_ptr", "tile_row_idx", "csc_tile_ids")


def hybrid_to_dict(h) -> dict:
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


def csr_to_hybrid_tiles(csr, tile_rows: int, tile_cols: int, col_major: bool,
                        dense_threshold: int, build_csc: bool) -> dict:
    """Restatement of csr_to_hybrid_tiles (src/dmma_tiles.h:243-438) in numpy:
    per tile row, entries keyed by (tile column, physical index) where the
    physical index is r * tile_cols + c (row-major payload) or c * tile_rows + r
    (column-major payload) (:163-224); repeated coordinates summed in CSR
    order; a tile with >= dense_threshold distinct entries stores 32 values in
    physical order, otherwise its values packed in mask-bit order (:334-351);
    optional tile CSC in tile-row order (:372-409)."""
    m, n = csr.m, csr.n
    trc = -(-m // tile_rows) if m else 0
    tcc = -(-n // tile_cols) if n else 0
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(csr.rowptr))
    cols = csr.col.astype(np.int64)
    lr, lc = rows % tile_rows, cols % tile_cols
    phys = lc * tile_rows + lr if col_major else lr * tile_cols + lc
    trow, tcol = rows // tile_rows, cols // tile_cols
    key = (trow << 40) | (tcol << 5) | phys
    order = np.argsort(key, kind="stable")
    ks, vs = key[order], csr.val[order]
    head = np.ones(ks.size, bool)
    head[1:] = ks[1:] != ks[:-1]
    starts = np.flatnonzero(head)
    ukey = ks[starts]
    uval = np.add.reduceat(vs, starts) if ks.size else np.zeros(0)
    tkey = ukey >> 5
    thead = np.ones(ukey.size, bool)
    thead[1:] = tkey[1:] != tkey[:-1]
    tstart = np.flatnonzero(thead)
    ntiles = tstart.size
    tend = np.append(tstart[1:], ukey.size)
    counts = tend - tstart
    uph = (ukey & 31).astype(np.int64)
    masks = np.array([np.bitwise_or.reduce(np.left_shift(np.uint32(1), uph[a:b].astype(np.uint32)))
                      for a, b in zip(tstart, tend)], dtype=np.uint32) if ntiles else np.zeros(0, np.uint32)
    dense = counts >= dense_threshold
    sizes = np.where(dense, 32, counts)
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    values = np.zeros(int(offs[-1]))
    for t in range(ntiles):
        a, b = tstart[t], tend[t]
        if dense[t]:
            values[offs[t] + uph[a:b]] = uval[a:b]
        else:
            values[offs[t]:offs[t] + (b - a)] = uval[a:b]
    t_row = (ukey[tstart] >> 40).astype(np.int64)
    t_col = ((ukey[tstart] >> 5) & ((1 << 35) - 1)).astype(np.int32)
    tile_row_ptr = np.concatenate([[0], np.cumsum(np.bincount(t_row, minlength=trc))]).astype(np.int32)
    d = {"rows": m, "cols": n, "tile_rows": tile_rows, "tile_cols": tile_cols,
         "tile_row_count": trc, "tile_col_count": tcc, "num_tiles": ntiles,
         "payload_size": int(offs[-1]), "dense_tiles": int(dense.sum()),
         "sparse_tiles": int(ntiles - dense.sum()), "tile_row_ptr": tile_row_ptr,
         "tile_col_idx": t_col, "value_offsets": offs, "masks": masks, "values": values,
         "tile_col_ptr": None, "tile_row_idx": None, "csc_tile_ids": None}
    if build_csc:
        corder = np.argsort(t_col, kind="stable")
        d["tile_col_ptr"] = np.concatenate([[0], np.cumsum(np.bincount(t_col, minlength=tcc))]).astype(np.int32)
        d["csc_tile_ids"] = corder.astype(np.int32)
        d["tile_row_idx"] = t_row[corder].astype(np.int32)
    return d


def super16_index(leaf: dict, role: int) -> dict:
    """Restatement of build_device_index (src/super16_symbolic.cuh:2123-2323)
    over hybrid leaf tiles.  A parent groups RG x CG leaves: 2 x 4 of the 8x4
    A leaves (role 1), 4 x 2 of the 4x8 B leaves (role 2) (:2145-2160).  Per
    parent row the parent columns are the distinct leaf_col // CG of its leaf
    rows (:674-718); a parent's leaves are listed leaf row by leaf row in leaf
    order, and child_mask bit child_row * CG + leaf_col % CG marks each
    (:720-789); the 16 Boolean rows have bit c for column c of the parent
    (:797-864); B also gets its parent CSC ordered by (column, row)
    (:866-907, :2262-2311)."""
    a_role = role == 1
    RG, CG = (2, 4) if a_role else (4, 2)
    def arr(k, dt):  # absent arrays of an empty leaf matrix
        return np.zeros(0, dt) if leaf[k] is None else np.asarray(leaf[k], dt)

    trp, tci, masks = arr("tile_row_ptr", np.int64), arr("tile_col_idx", np.int64), arr("masks", np.uint64)
    lrows, nt = int(leaf["tile_row_count"]), int(leaf["num_tiles"])
    prows = 0 if lrows == 0 else 1 + (lrows - 1) // RG
    pcols = 0 if leaf["tile_col_count"] == 0 else 1 + (int(leaf["tile_col_count"]) - 1) // CG
    lrow = np.repeat(np.arange(lrows, dtype=np.int64), np.diff(trp))
    prow, pcol, child = lrow // RG, tci // CG, lrow % RG
    W = max(pcols, 1)
    ukey, parent = np.unique(prow * W + pcol, return_inverse=True)
    pc = ukey.size
    row_ptr = np.concatenate([[0], np.cumsum(np.bincount(ukey // W, minlength=prows))])
    order = np.lexsort((np.arange(nt), child, parent))
    child_ptr = np.concatenate([[0], np.cumsum(np.bincount(parent, minlength=pc))])
    child_mask = np.zeros(pc, np.uint8)
    np.bitwise_or.at(child_mask, parent, (1 << (child * CG + tci % CG)).astype(np.uint8))
    rows = np.zeros(pc * 16, np.uint16)
    if a_role:
        for lr in range(8):  # leaf row lr of the leaf is parent row 8 child + lr
            bits = ((masks >> np.uint64(4 * lr)) & np.uint64(0xF)) << (4 * (tci % 4)).astype(np.uint64)
            np.bitwise_or.at(rows, parent * 16 + child * 8 + lr, bits.astype(np.uint16))
    else:
        for k in range(4):  # leaf row k is parent row 4 child + k
            bits = np.zeros(nt, np.uint64)
            for c in range(8):
                bits |= ((masks >> np.uint64(4 * c + k)) & np.uint64(1)) << np.uint64(c)
            bits <<= (8 * (tci % 2)).astype(np.uint64)
            np.bitwise_or.at(rows, parent * 16 + child * 4 + k, bits.astype(np.uint16))
    d = {"role": role, "rows": int(leaf["rows"]), "cols": int(leaf["cols"]),
         "parent_row_count": prows, "parent_col_count": pcols, "parent_count": pc,
         "row_ptr": row_ptr.astype(np.uint64), "col_idx": (ukey % W).astype(np.uint32),
         "child_ptr": child_ptr.astype(np.uint64), "child_mask": child_mask,
         "child_leaf_ids": order.astype(np.uint32), "boolean_row_masks": rows,
         "col_ptr": None, "row_idx": None, "csc_parent_ids": None}
    if not a_role:
        p_row = np.repeat(np.arange(prows, dtype=np.int64), np.diff(row_ptr))
        ckey = (ukey % W) * max(prows, 1) + p_row
        corder = np.argsort(ckey, kind="stable")
        d["col_ptr"] = np.concatenate([[0], np.cumsum(np.bincount(ukey % W, minlength=pcols))]
                                      ).astype(np.uint64)
        d["row_idx"] = p_row[corder].astype(np.uint32)
        d["csc_parent_ids"] = corder.astype(np.uint32)
    return d


def tiles_8x4(a, row_old_to_new=None, col_old_to_new=None) -> int:
    """Distinct 8x4 tiles of A under row / column maps: the quantity of the
    reference's exact reorder commit rule (src/dmma_reorder.h:1671-1727)."""
    rows = np.repeat(np.arange(a.m), np.diff(a.rowptr))
    cols = np.asarray(a.col, np.int64)
    if row_old_to_new is not None:
        rows = np.asarray(row_old_to_new)[rows]
    if col_old_to_new is not None:
        cols = np.asarray(col_old_to_new)[cols]
    keys = (rows.astype(np.int64) // 8) * ((a.n + 3) // 4) + cols // 4
    return int(np.unique(keys).size)


def reorder_cm(a, max_components: int = 256):
    """Restatement of the reorder proposal of this build (rtt_reorder_plan_build):
    a breadth-first traversal alternating rows and columns, each level ordered
    by (position of the earliest-placed neighbour, degree, index); components
    start at the unplaced row of least (degree, index); unreached rows and
    columns follow in index order.  Returns (row_old_to_new, col_old_to_new,
    components, levels).  Pure Python: small inputs only."""
    m, n = a.m, a.n
    rp = np.asarray(a.rowptr, np.int64)
    col = np.asarray(a.col, np.int64)
    deg_r = np.diff(rp)
    rows_of = np.repeat(np.arange(m), deg_r)
    o = np.lexsort((rows_of, col))
    tcol_rows = rows_of[o]
    tp = np.zeros(n + 1, np.int64)
    tp[1:] = np.cumsum(np.bincount(col, minlength=n))
    deg_c = np.diff(tp)
    adj_r = [col[rp[i]:rp[i + 1]] for i in range(m)]
    adj_c = [tcol_rows[tp[j]:tp[j + 1]] for j in range(n)]
    pos = [np.full(m, -1, np.int64), np.full(n, -1, np.int64)]
    deg = [deg_r, deg_c]
    adj = [adj_r, adj_c]
    placed = [0, 0]
    comps = levels = 0
    for _ in range(max_components):
        cand = np.nonzero((pos[0] == -1) & (deg_r > 0))[0]
        if cand.size == 0:
            break
        r0 = int(cand[np.lexsort((cand, deg_r[cand]))[0]])
        comps += 1
        pos[0][r0] = placed[0]
        placed[0] += 1
        front, side = [r0], 0
        while front:
            other = 1 - side
            claim = {}
            for v in front:
                pv = pos[side][v]
                for u in adj[side][v]:
                    u = int(u)
                    if pos[other][u] == -1:
                        claim[u] = min(claim.get(u, 1 << 62), pv)
            new = sorted(claim, key=lambda u: (claim[u], deg[other][u], u))
            for i, u in enumerate(new):
                pos[other][u] = placed[other] + i
            placed[other] += len(new)
            if new:
                levels += 1
            front, side = new, other
    for s in (0, 1):
        rest = np.nonzero(pos[s] == -1)[0]
        pos[s][rest] = placed[s] + np.arange(rest.size)
    return pos[0], pos[1], comps, levels


M64 = (1 << 64) - 1


def _ro_mix(k: int) -> int:
    """MurmurHash3's 64-bit finaliser (the fine passes' fingerprint mixer)."""
    k ^= k >> 33
    k = (k * 0xFF51AFD7ED558CCD) & M64
    k ^= k >> 33
    k = (k * 0xC4CEB9FE1A85EC53) & M64
    k ^= k >> 33
    return k


def _axis_profile(idx, other_positions, panel):
    """Profile of one index of an axis: entry count, soft bucket (log2 / 2),
    panel range and span, the two fingerprint words, their occupancy."""
    deg = len(other_positions)
    if deg == 0:
        return dict(id=idx, degree=0, bucket=-1, occ=0, pmin=-1, pmax=-1, span=0, f0=0, f1=0)
    f0 = f1 = 0
    ps = [int(p) // panel for p in other_positions]
    for p in ps:
        f0 |= 1 << (_ro_mix(2 * p + 1) & 63)
        f1 |= 1 << (_ro_mix(2 * p + 2) & 63)
    lo, hi = min(ps), max(ps)
    return dict(id=idx, degree=deg, bucket=(deg.bit_length() - 1) // 2,
                occ=bin(f0).count("1") + bin(f1).count("1"), pmin=lo, pmax=hi,
                span=hi - lo + 1, f0=f0, f1=f1)


def _coarse_key(q):
    """The coarse profile order (src/dmma_reorder.h:1287-1311), least first."""
    return (q["degree"] == 0, -q["bucket"], -q["occ"], q["pmin"], q["span"], -q["degree"],
            q["f0"], q["f1"], q["id"])


def _pack_window(profs, group):
    """Greedy packing of one window (src/dmma_reorder.h:1511-1608): an anchor,
    the least unused profile in the coarse order, then the unused profile of
    best score against the group (:1386-1416) until the group is full.
    Returns the window's old ids in their new order."""
    from fractions import Fraction

    unused = list(range(len(profs)))
    out = []
    while unused:
        a = min(unused, key=lambda i: _coarse_key(profs[i]))
        unused.remove(a)
        A = profs[a]
        out.append(A["id"])
        g0, g1, gmin, gmax = A["f0"], A["f1"], A["pmin"], A["pmax"]
        for _ in range(1, group):
            if not unused:
                break

            def score(i):
                q = profs[i]
                overlap = bin(g0 & q["f0"]).count("1") + bin(g1 & q["f1"]).count("1")
                adds = (bin(~g0 & M64 & q["f0"]).count("1") +
                        bin(~g1 & M64 & q["f1"]).count("1"))
                uni = max(bin(g0 | q["f0"]).count("1") + bin(g1 | q["f1"]).count("1"), 1)
                nmin, nmax = gmin, gmax
                if q["pmin"] >= 0:
                    nmin = q["pmin"] if gmin < 0 else min(gmin, q["pmin"])
                    nmax = max(gmax, q["pmax"])
                cur = 0 if gmin < 0 else gmax - gmin + 1
                nxt = 0 if nmin < 0 else nmax - nmin + 1
                return (abs(A["bucket"] - q["bucket"]), adds, -Fraction(overlap, uni), -overlap,
                        nxt - cur, abs(A["degree"] - q["degree"]), q["id"])
            b = min(unused, key=score)
            unused.remove(b)
            B = profs[b]
            out.append(B["id"])
            if B["pmin"] >= 0:
                gmin = B["pmin"] if gmin < 0 else min(gmin, B["pmin"])
                gmax = max(gmax, B["pmax"])
            g0 |= B["f0"]
            g1 |= B["f1"]
    return out


def reorder_fine_pass(a, row_o2n, col_o2n, rows: bool, guarded: bool = True):
    """One fine pass of the reorder (src/dmma_reorder.h:2865-2990) on top of
    the maps: rows in windows of 32 and groups of 8 against 4-column panels,
    or (rows=False) columns in windows of 16 and groups of 4 against 8-row
    panels.  A window's packing replaces its order only if it has fewer 8x4
    tiles, or as many and a smaller fan-out (the sum over its groups of the
    span of the opposite tiles), :1841-1887.  Returns (row_o2n, col_o2n,
    stats: windows, accepted, tile reduction, fan-out before / after)."""
    W, G, panel = (32, 8, 4) if rows else (16, 4, 8)
    row_o2n = np.asarray(row_o2n, np.int64).copy()
    col_o2n = np.asarray(col_o2n, np.int64).copy()
    rp = np.asarray(a.rowptr, np.int64)
    col = np.asarray(a.col, np.int64)
    ent_r = np.repeat(np.arange(a.m), np.diff(rp))
    if rows:
        count, mine, other = a.m, row_o2n, col_o2n
        adj = [col[rp[i]:rp[i + 1]] for i in range(a.m)]
    else:
        count, mine, other = a.n, col_o2n, row_o2n
        order = np.lexsort((ent_r, col))
        tp = np.zeros(a.n + 1, np.int64)
        tp[1:] = np.cumsum(np.bincount(col, minlength=a.n))
        adj = [ent_r[order][tp[j]:tp[j + 1]] for j in range(a.n)]
    n2o = np.empty(count, np.int64)
    n2o[mine] = np.arange(count)
    prop = n2o.copy()
    windows = (count + W - 1) // W
    for w in range(windows):
        ids = n2o[w * W:(w + 1) * W]
        profs = [_axis_profile(int(i), other[adj[i]], panel) for i in ids]
        prop[w * W:w * W + len(ids)] = _pack_window(profs, G)
    prop_o2n = np.empty(count, np.int64)
    prop_o2n[prop] = np.arange(count)
    # tiles and fan-out per window under the current order and the proposal
    opp_tiles = (a.n + 3) // 4 if rows else (a.m + 7) // 8

    def per_window(pos_of):
        tiles = [set() for _ in range(windows)]
        spans = [[None] * (W // G) for _ in range(windows)]
        for r, c in zip(ent_r, col):
            R, Cc = int(row_o2n[r]), int(col_o2n[c])
            pos = int(pos_of[r]) if rows else int(pos_of[c])
            opp = Cc // 4 if rows else R // 8
            w, g = pos // W, (pos % W) // G
            tiles[w].add((g, opp))
            s = spans[w][g]
            spans[w][g] = (opp, opp) if s is None else (min(s[0], opp), max(s[1], opp))
        fan = [sum(s[1] - s[0] + 1 for s in sp if s is not None) for sp in spans]
        return [len(t) for t in tiles], fan

    cur_t, cur_f = per_window(mine)
    prop_t, prop_f = per_window(prop_o2n)
    new_n2o = n2o.copy()
    acc = red = fb = fa = 0
    for w in range(windows):
        ok = (not guarded) or prop_t[w] < cur_t[w] or (prop_t[w] == cur_t[w] and
                                                       prop_f[w] < cur_f[w])
        fb += cur_f[w]
        fa += prop_f[w] if ok else cur_f[w]
        if ok:
            new_n2o[w * W:(w + 1) * W] = prop[w * W:(w + 1) * W]
            acc += 1
            red += max(cur_t[w] - prop_t[w], 0)
    new_o2n = np.empty(count, np.int64)
    new_o2n[new_n2o] = np.arange(count)
    if rows:
        row_o2n = new_o2n
    else:
        col_o2n = new_o2n
    return row_o2n, col_o2n, dict(windows=windows, accepted=acc, reduction=red,
                                  fanout_before=fb, fanout_after=fa)


def reorder_plan(a, variant: int = 0):
    """Restatement of rtt_reorder_plan_build_variant: the coarse traversal of
    reorder_cm under the exact commit rule, then the row and inner fine
    passes, as the variant selects (0 full, 1 coarse, 2 fine, 3 coarse+row,
    4 coarse+inner, 5 unguarded).  Returns (row_o2n, col_o2n, info)."""
    coarse = variant != 2
    row_fine = variant not in (1, 4)
    inner_fine = variant not in (1, 3)
    guarded = variant != 5
    r, c = np.arange(a.m), np.arange(a.n)
    info = {"tiles_before": tiles_8x4(a), "accepted": 0}
    info["proposal_tiles"] = info["tiles_before"]
    if coarse:
        pr, pc, comps, levels = reorder_cm(a)
        info.update(components=comps, levels=levels, proposal_tiles=tiles_8x4(a, pr, pc))
        if (not guarded) or info["proposal_tiles"] < info["tiles_before"]:
            r, c = pr, pc
            info["accepted"] = 1
    if row_fine:
        r, c, info["row"] = reorder_fine_pass(a, r, c, True, guarded)
    if inner_fine:
        r, c, info["inner"] = reorder_fine_pass(a, r, c, False, guarded)
    info["tiles_after"] = tiles_8x4(a, r, c)
    return r, c, info


def plan_tail_queue(scans, matches, output_nnz, policy: dict, model: dict):
    """Restatement of dmma_plan_tile_tail_queue (src/dmma_tile_tail_queue.h:190-291)
    with the chunk rule of :148-176 in numpy float32 (round-to-nearest, no
    contraction).  Returns (chunks per task, summary dict)."""
    sc = np.asarray(scans, np.int64)
    mt = np.asarray(matches, np.int64)
    on = np.asarray(output_nnz, np.int64)
    n = sc.size
    plan = dict(reason=0, output_tasks=n, ordinary_tasks=n, heavy_tasks=0, chunks=0,
                descriptor_bytes=0, heavy_flag_bytes=0, partial_workspace_bytes=0,
                heavy_fraction=0.0, average_chunks=0.0)
    zero = np.zeros(n, np.int32)
    if not policy["enabled"]:
        return zero, plan
    fin = np.isfinite
    ok = (fin(policy["admission_threshold"]) and policy["admission_threshold"] > 0 and
          fin(policy["chunk_target"]) and policy["chunk_target"] > 0 and
          2 <= policy["max_chunks"] <= 32 and fin(policy["max_heavy_fraction"]) and
          0 <= policy["max_heavy_fraction"] <= 1 and policy["record_capacity"] > 0 and
          all(fin(model[k]) and model[k] >= 0 for k in ("intercept", "scan", "match", "output")))
    if not ok:
        plan["reason"] = 2
        return zero, plan
    f32 = np.float32
    work = f32(model["scan"]) * sc.astype(f32) + f32(model["match"]) * mt.astype(f32)
    admit = (work > f32(policy["admission_threshold"])) & (sc > 1)
    req = np.ceil(work / f32(policy["chunk_target"]))
    ch = np.where(req >= f32(policy["max_chunks"]), policy["max_chunks"],
                  np.clip(req, -2**31, 2**31 - 1).astype(np.int64))
    ch = np.minimum(np.maximum(ch, 2), sc)
    ch = np.where(admit & (ch >= 2), ch, 0).astype(np.int64)
    invalid = (sc < 0) | (mt < 0) | (mt > sc) | (on < 0) | (on > 64)
    ch[invalid] = 0
    heavy = ch > 0
    first_invalid = int(np.argmax(invalid)) if invalid.any() else n
    over = np.cumsum(heavy) > policy["record_capacity"]
    first_over = int(np.argmax(over)) if over.any() else n
    if first_invalid < n or first_over < n:
        plan["reason"] = 3 if first_invalid <= first_over else 5
        return zero, plan
    h, c = int(heavy.sum()), int(ch.sum())
    plan.update(heavy_tasks=h, ordinary_tasks=n - h, chunks=c,
                heavy_fraction=0.0 if n == 0 else h / n, average_chunks=0.0 if h == 0 else c / h,
                heavy_flag_bytes=((n + 31) // 32) * 4, descriptor_bytes=c * 16,
                partial_workspace_bytes=c * 512)
    if h == 0:
        plan["reason"] = 4
    elif plan["heavy_fraction"] > policy["max_heavy_fraction"]:
        plan["reason"] = 6
    elif policy["workspace_reduction"] and plan["partial_workspace_bytes"] > policy["workspace_limit_bytes"]:
        plan["reason"] = 7
    else:
        plan["reason"] = 1
    return ch.astype(np.int32), plan


EARLY_SPLIT_POLICY = dict(enabled=0, admission_threshold=684947.875, chunk_target=342473.938,
                          max_chunks=8, max_heavy_fraction=0.001, record_capacity=131072,
                          workspace_limit_bytes=512 * 1024 * 1024, workspace_reduction=1)


def plan_early_split(scans, matches, output_nnz, policy: dict, model: dict, sm_count: int):
    """Restatement of dmma_plan_tile_early_split (src/dmma_tile_early_split.h:152-229):
    the tail-queue partition (plan_tail_queue with the policy switched on), a
    global cap of ceil(sm_count / 2) persistent heavy CTAs (:98-110) and the
    exact-parent-partition check (:127-150).  Returns (chunks per task, plan)."""
    n = len(scans)
    plan = dict(reason=0, base_reason=0, output_tasks=n, ordinary_tasks=n, heavy_tasks=0,
                chunks=0, sm_count=sm_count, global_heavy_worker_block_cap=0,
                heavy_worker_blocks=0, reduction_worker_blocks=0, descriptor_bytes=0,
                heavy_flag_bytes=0, partial_workspace_bytes=0, exact_parent_partition=1)
    zero = np.zeros(n, np.int32)
    if not policy["enabled"]:
        return zero, plan
    if sm_count <= 0:
        plan["reason"] = 2
        return zero, plan
    ch, base = plan_tail_queue(scans, matches, output_nnz, {**policy, "enabled": 1}, model)
    plan["base_reason"] = base["reason"]
    if base["reason"] != 1:
        plan["reason"] = 3
        return zero, plan
    cap = (sm_count + 1) // 2
    plan.update(reason=1, ordinary_tasks=base["ordinary_tasks"], heavy_tasks=base["heavy_tasks"],
                chunks=base["chunks"], global_heavy_worker_block_cap=cap,
                heavy_worker_blocks=min(base["chunks"], cap),
                reduction_worker_blocks=min(base["heavy_tasks"], cap) if policy["workspace_reduction"] else 0,
                descriptor_bytes=base["descriptor_bytes"], heavy_flag_bytes=base["heavy_flag_bytes"],
                partial_workspace_bytes=base["partial_workspace_bytes"])
    exact = (plan["ordinary_tasks"] + plan["heavy_tasks"] == n and not np.any(ch == 1)
             and int((ch > 0).sum()) == plan["heavy_tasks"])
    plan["exact_parent_partition"] = int(exact)
    if not exact or plan["heavy_worker_blocks"] <= 0:
        plan.update(reason=3, ordinary_tasks=n, heavy_tasks=0, chunks=0, heavy_worker_blocks=0,
                    reduction_worker_blocks=0, descriptor_bytes=0, heavy_flag_bytes=0,
                    partial_workspace_bytes=0)
        return zero, plan
    return ch, plan


def build(reference_dir: str | None = None) -> None:
    """Compile liboracle.so, and the reference's own CPU code into _ref/ when
    reference_dir (or the environment's RTT_REFERENCE_DIR) names a reference
    checkout that exists."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    ref = reference_dir or os.environ.get("RTT_REFERENCE_DIR")
    if ref and Path(ref, "src").is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "REF=" + str(ref)], check=True)


class Oracle(_Base):
    """The C restatement (oracle.c)."""

    def __init__(self, path: Path | None = None):
        path = path or HERE / "liboracle.so"
        if not path.exists():
            build(reference=False)
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.orc_free.argtypes = [C.c_void_p]
        self._free = L.orc_free
        for f in ("orc_csr2tile_row_major", "orc_csr2tile_col_major"):
            getattr(L, f).argtypes = [C.POINTER(SMatrix)]
            getattr(L, f).restype = C.c_int
        L.orc_spgemm_tile.argtypes = [C.POINTER(SMatrix)] * 3 + [C.c_int]
        L.orc_spgemm_tile.restype = C.c_int
        L.orc_tile2csr.argtypes = [C.POINTER(SMatrix), C.c_int, C.c_int]
        L.orc_tile2csr.restype = C.c_int
        L.orc_tile2csr_restore_rows.argtypes = [C.POINTER(SMatrix), C.POINTER(C.c_int), C.c_int,
                                                C.c_int, C.c_int]
        L.orc_tile2csr_restore_rows.restype = C.c_int
        L.orc_tile16_to_tile8.argtypes = [C.POINTER(SMatrix), C.POINTER(SMatrix)]
        L.orc_tile16_to_tile8.restype = C.c_int
        L.orc_spgemm_csr.argtypes = [C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_spgemm_csr.restype = C.c_longlong
        L.orc_nnzcub.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_nnzcub.restype = C.c_longlong
        L.orc_num_threads.restype = C.c_int

    def threads(self) -> int:
        return int(self.lib.orc_num_threads())

    def csr2tile_row_major(self, csr) -> dict:
        s, keep = csr_smatrix(csr)
        st = self.lib.orc_csr2tile_row_major(C.byref(s))
        if st:
            raise ValueError(f"orc_csr2tile_row_major status {st}")
        d = tiles_from_smatrix(s)
        self._free_tiles(s)
        return d

    def csr2tile_col_major(self, csr) -> dict:
        s, keep = csr_smatrix(csr)
        st = self.lib.orc_csr2tile_col_major(C.byref(s))
        if st:
            raise ValueError(f"orc_csr2tile_col_major status {st}")
        d = tiles_from_smatrix(s, csc=True)
        self._free_tiles(s)
        return d

    def spgemm_tile(self, a: dict, b: dict, quirk: bool = False) -> dict:
        sa, ka = smatrix_from_tiles(a)
        sb, kb = smatrix_from_tiles(b)
        sc = SMatrix()
        st = self.lib.orc_spgemm_tile(C.byref(sa), C.byref(sb), C.byref(sc), int(quirk))
        if st:
            raise ValueError(f"orc_spgemm_tile status {st}")
        d = tiles_from_smatrix(sc)
        self._free_tiles(sc)
        return d

    def tile2csr(self, t: dict, tile_dim: int = TD, canonical: bool = True, new_to_old=None,
                 perm_size: int | None = None):
        from types import SimpleNamespace
        s, keep = smatrix_from_tiles(t)
        if new_to_old is None:
            st = self.lib.orc_tile2csr(C.byref(s), tile_dim, int(canonical))
        else:
            p = np.ascontiguousarray(new_to_old, dtype=np.int32)
            size = p.shape[0] if perm_size is None else perm_size
            st = self.lib.orc_tile2csr_restore_rows(C.byref(s), _ptr(p, C.c_int), size, tile_dim,
                                                    int(canonical))
        if st:
            return st
        out = SimpleNamespace(m=s.m, n=s.n, rowptr=_copy(s.rowpointer, s.m + 1, np.int32),
                              col=_copy(s.columnindex, s.nnz, np.int32),
                              val=_copy(s.value, s.nnz, np.float64))
        self._free_csr(s)
        return out

    def tile16_to_tile8(self, t: dict) -> dict:
        s, keep = smatrix_from_tiles(t)
        o = SMatrix()
        st = self.lib.orc_tile16_to_tile8(C.byref(s), C.byref(o))
        if st:
            raise ValueError(f"orc_tile16_to_tile8 status {st}")
        d = tiles_from_smatrix(o, ptr_stride=8)
        self._free_tiles(o)
        return d

    def spgemm_csr(self, a, b, with_abs: bool = True):
        """FP64 row SPA: returns (rowptr int64, col int32, val f64, abs f64|None)."""
        rp = np.zeros(a.m + 1, dtype=np.int64)
        args = (a.m, a.n, b.n, a.rowptr.ctypes.data, a.col.ctypes.data, a.val.ctypes.data,
                b.rowptr.ctypes.data, b.col.ctypes.data, b.val.ctypes.data)
        nnz = self.lib.orc_spgemm_csr(*args, rp.ctypes.data, None, None, None)
        col = np.zeros(max(nnz, 1), dtype=np.int32)
        val = np.zeros(max(nnz, 1), dtype=np.float64)
        ab = np.zeros(max(nnz, 1), dtype=np.float64) if with_abs else None
        self.lib.orc_spgemm_csr(*args, rp.ctypes.data, col.ctypes.data, val.ctypes.data,
                                ab.ctypes.data if with_abs else None)
        return rp, col[:nnz], val[:nnz], (ab[:nnz] if with_abs else None)

    def csr_to_hybrid_tiles(self, csr, tile_rows=8, tile_cols=4, col_major=False,
                            dense_threshold=24, build_csc=False) -> dict:
        return csr_to_hybrid_tiles(csr, tile_rows, tile_cols, col_major, dense_threshold,
                                   build_csc)

    def super16_index(self, leaf: dict, role: int) -> dict:
        return super16_index(leaf, role)

    def nnzcub(self, a, b) -> int:
        return int(self.lib.orc_nnzcub(a.m, a.rowptr.ctypes.data, a.col.ctypes.data,
                                       b.rowptr.ctypes.data))


def reference_available() -> bool:
    return (HERE / "_ref" / "libref_tiles.so").exists() and (HERE / "_ref" / "libref_spa.so").exists()


class Reference(_Base):
    """The reference's own CPU functions (compiled from its sources)."""

    def __init__(self):
        self.lib = C.CDLL(str(HERE / "_ref" / "libref_tiles.so"))
        self.spa = C.CDLL(str(HERE / "_ref" / "libref_spa.so"))
        L = self.lib
        L.ref_free.argtypes = [C.c_void_p]
        self._free = L.ref_free
        for f in ("ref_csr2tile_row_major", "ref_csr2tile_col_major"):
            getattr(L, f).argtypes = [C.POINTER(SMatrix)]
        L.ref_spgemm_cpu_fixed.argtypes = [C.POINTER(SMatrix)] * 3
        L.ref_tile2csr.argtypes = [C.POINTER(SMatrix), C.c_int]
        L.ref_tile2csr.restype = C.c_int
        L.ref_tile2csr_restore_rows.argtypes = [C.POINTER(SMatrix), C.POINTER(C.c_int), C.c_int,
                                                C.c_int]
        L.ref_tile2csr_restore_rows.restype = C.c_int
        L.ref_output_tile_rows.restype = C.c_int
        self.spa.ref_spgemm_serialref.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                  C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_int, C.c_int, C.c_int,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_int]

    def csr2tile_row_major(self, csr) -> dict:
        s, keep = csr_smatrix(csr)
        self.lib.ref_csr2tile_row_major(C.byref(s))
        d = tiles_from_smatrix(s)
        self._free_tiles(s)
        return d

    def csr2tile_col_major(self, csr) -> dict:
        s, keep = csr_smatrix(csr)
        self.lib.ref_csr2tile_col_major(C.byref(s))
        d = tiles_from_smatrix(s, csc=True)
        self._free_tiles(s)
        return d

    def spgemm_cpu(self, a: dict, b: dict) -> dict:
        """spgemm_cpu with the in-tile column fix applied at the call site."""
        sa, ka = smatrix_from_tiles(a)
        sb, kb = smatrix_from_tiles(b)
        sc = SMatrix()
        self.lib.ref_spgemm_cpu_fixed(C.byref(sa), C.byref(sb), C.byref(sc))
        sc.m, sc.n, sc.tilem, sc.tilen = a["m"], b["n"], a["tilem"], b["tilen"]
        d = tiles_from_smatrix(sc)
        self._free_tiles(sc)
        return d

    def tile2csr(self, t: dict, canonical: bool = True, new_to_old=None, perm_size=None):
        """The reference tile2csr (8x8 tiles)."""
        from types import SimpleNamespace
        s, keep = smatrix_from_tiles(t)
        if new_to_old is None:
            ok = self.lib.ref_tile2csr(C.byref(s), int(canonical))
        else:
            p = np.ascontiguousarray(new_to_old, dtype=np.int32)
            size = p.shape[0] if perm_size is None else perm_size
            ok = self.lib.ref_tile2csr_restore_rows(C.byref(s), _ptr(p, C.c_int), size,
                                                    int(canonical))
        if not ok:
            return None
        out = SimpleNamespace(m=s.m, n=s.n, rowptr=_copy(s.rowpointer, s.m + 1, np.int32),
                              col=_copy(s.columnindex, s.nnz, np.int32),
                              val=_copy(s.value, s.nnz, np.float64))
        self._free_csr(s)
        return out

    def csr_to_hybrid_tiles(self, csr, tile_rows=8, tile_cols=4, col_major=False,
                            dense_threshold=24, build_csc=False):
        """The reference's csr_to_hybrid_tiles; None when it returns false."""
        s, keep = csr_smatrix(csr)
        h = HybridTiles()
        L = self.lib
        L.ref_csr_to_hybrid_tiles.argtypes = [C.POINTER(SMatrix), C.c_int, C.c_int, C.c_int,
                                              C.c_int, C.c_int, C.POINTER(HybridTiles)]
        if not L.ref_csr_to_hybrid_tiles(C.byref(s), tile_rows, tile_cols, int(col_major),
                                         dense_threshold, int(build_csc), C.byref(h)):
            return None
        d = hybrid_to_dict(h)
        for k in HYBRID_FIELDS:
            p = getattr(h, k)
            if p:
                self._free(C.cast(p, C.c_void_p))
        return d

    def plan_tail_queue(self, scans, matches, output_nnz, policy: dict, model: dict):
        """The reference's dmma_plan_tile_tail_queue (via ref_plan_tile_tail_queue)."""
        L = self.lib
        L.ref_plan_tile_tail_queue.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_double, C.c_double, C.c_int, C.c_double,
                                               C.c_int, C.c_longlong, C.c_int, C.c_double,
                                               C.c_double, C.c_double, C.c_double, C.c_void_p,
                                               C.c_void_p]
        sc = np.ascontiguousarray(scans, np.int32)
        mt = np.ascontiguousarray(matches, np.int32)
        on = np.ascontiguousarray(output_nnz, np.int32)
        n = sc.size
        ch = np.zeros(max(n, 1), np.int32)
        summ = np.zeros(5, np.int64)
        if not policy["enabled"]:
            return ch[:n], 0
        reason = L.ref_plan_tile_tail_queue(
            n, sc.ctypes.data, mt.ctypes.data, on.ctypes.data, policy["admission_threshold"],
            policy["chunk_target"], policy["max_chunks"], policy["max_heavy_fraction"],
            policy["record_capacity"], policy["workspace_limit_bytes"],
            policy["workspace_reduction"], model["intercept"], model["scan"], model["match"],
            model["output"], ch.ctypes.data, summ.ctypes.data)
        return ch[:n], (reason, summ)

    def plan_early_split(self, scans, matches, output_nnz, policy: dict, model: dict,
                         sm_count: int):
        """The reference's dmma_plan_tile_early_split (via ref_plan_tile_early_split)."""
        L = self.lib
        L.ref_plan_tile_early_split.argtypes = [
            C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double,
            C.c_int, C.c_double, C.c_int, C.c_longlong, C.c_int, C.c_double, C.c_double,
            C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        sc = np.ascontiguousarray(scans, np.int32)
        mt = np.ascontiguousarray(matches, np.int32)
        on = np.ascontiguousarray(output_nnz, np.int32)
        n = sc.size
        ch = np.zeros(max(n, 1), np.int32)
        summ = np.zeros(11, np.int64)
        reason = L.ref_plan_tile_early_split(
            n, sc.ctypes.data, mt.ctypes.data, on.ctypes.data, int(policy["enabled"]),
            policy["admission_threshold"], policy["chunk_target"], policy["max_chunks"],
            policy["max_heavy_fraction"], policy["record_capacity"],
            policy["workspace_limit_bytes"], policy["workspace_reduction"], model["intercept"],
            model["scan"], model["match"], model["output"], sm_count, ch.ctypes.data,
            summ.ctypes.data)
        keys = ("base_reason", "ordinary_tasks", "heavy_tasks", "chunks",
                "global_heavy_worker_block_cap", "heavy_worker_blocks", "reduction_worker_blocks",
                "descriptor_bytes", "heavy_flag_bytes", "partial_workspace_bytes",
                "exact_parent_partition")
        return ch[:n], dict(reason=reason, **{k: int(v) for k, v in zip(keys, summ)})

    def mmio_allinone(self, path):
        """The reference's Matrix Market reader: (m, n, is_symmetric, rowptr,
        col, val) as numpy arrays."""
        L = self.lib
        L.ref_mmio_allinone.argtypes = [C.c_char_p] + [C.c_void_p] * 7
        m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        rp, col, val = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
        st = L.ref_mmio_allinone(str(path).encode(), C.addressof(m), C.addressof(n),
                                 C.addressof(nnz), C.addressof(sym), C.addressof(rp),
                                 C.addressof(col), C.addressof(val))
        if st != 0:
            raise ValueError(f"mmio_allinone status {st}")
        out = (m.value, n.value, sym.value, _copy(rp, m.value + 1, np.int32),
               _copy(col, nnz.value, np.int32), _copy(val, nnz.value, np.float64))
        for p in (rp, col, val):
            self._free(C.cast(p, C.c_void_p))
        return out

    def spgemm_serialref(self, a, b):
        rp = np.zeros(a.m + 1, dtype=np.int32)
        nnz = C.c_int(0)
        args = [a.rowptr.ctypes.data, a.col.ctypes.data, a.val.ctypes.data, a.m, a.n, a.nnz,
                b.rowptr.ctypes.data, b.col.ctypes.data, b.val.ctypes.data, b.m, b.n, b.nnz]
        self.spa.ref_spgemm_serialref(*args, rp.ctypes.data, None, None, C.addressof(nnz), 1)
        col = np.zeros(max(nnz.value, 1), dtype=np.int32)
        val = np.zeros(max(nnz.value, 1), dtype=np.float64)
        self.spa.ref_spgemm_serialref(*args, rp.ctypes.data, col.ctypes.data, val.ctypes.data,
                                      C.addressof(nnz), 0)
        return rp, col[:nnz.value], val[:nnz.value]
