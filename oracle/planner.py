"""Restatement of the reference pack-once planner and exporter (oracle).

TEST INFRASTRUCTURE: see oracle/__init__.py.

The steps, tie-breaks and random-number consumption are those of the
reference (they have to be, for byte-for-byte pack parity); the code is an
independent restatement.  Each function cites what it follows:

* row grouping              src/nufft_layout_oracle.py:243-309 (+ morton2d :110-121)
* column -> K-tile split    src/nufft_layout_oracle.py:323-372 ("search")
                            src/export_torchkbnufft_gpu_case.py:102-162 ("optimized")
* quartet arrangement       src/nufft_layout_oracle.py:375-442 ("search")
                            src/export_torchkbnufft_gpu_case.py:165-214 ("optimized")
* whole-view packers        pack_view :445-497, fast_split24_pack :46-99,
                            optimized_split24_pack :270-299
* split24 / CSR residual    src/export_gpu_case.py:77-155
* FP16 2:4 compression      src/export_gpu_case.py:41-74 (+ vectorized twin
                            src/export_torchkbnufft_gpu_case.py:302-324)
* packed_header_v2          src/export_gpu_case.py:242-256

Sparse views are plain tuples ``(row_ids, cols_per_row, vals_per_row,
coords, output_size, n_cols)`` built by ``view_from_csr`` / ``transpose``.
"""

from __future__ import annotations

import math
import random
import struct
from dataclasses import dataclass

import numpy as np

M_TILE = 16
K_TILE = 32
MAGIC = 0x4E55464654323431
VERSION = 2
N_CHANNELS = 16


@dataclass
class View:
    row_ids: np.ndarray          # logical output row of each active row
    cols: list                   # list[list[int]]
    vals: list                   # list[list[float]]
    coords: np.ndarray           # [active, 2] float64 (morton ordering input)
    output_size: int
    n_cols: int

    @property
    def nnz(self) -> int:
        return sum(len(c) for c in self.cols)


@dataclass
class Tile:
    row_ids: np.ndarray   # [16] int32, -1 pads
    col_ids: list         # [k] int, -1 pads
    values: np.ndarray    # [16, k] float64
    legal: bool
    violation: int = 0


def view_from_csr(row_ptr, cols, vals, coords, n_cols, row_ids=None) -> View:
    m = len(row_ptr) - 1
    cl = [list(map(int, cols[row_ptr[r]:row_ptr[r + 1]])) for r in range(m)]
    vl = [list(map(float, vals[row_ptr[r]:row_ptr[r + 1]])) for r in range(m)]
    ids = np.arange(m, dtype=np.int64) if row_ids is None else np.asarray(row_ids, dtype=np.int64)
    return View(ids, cl, vl, np.asarray(coords, dtype=np.float64), m, int(n_cols))


def transpose(view: View, grid_size: int) -> View:
    """Exact active-row transpose (src/nufft_layout_oracle.py:209-231)."""
    rows: dict[int, list[int]] = {}
    vals: dict[int, list[float]] = {}
    for local, (cols, vs) in enumerate(zip(view.cols, view.vals)):
        logical = int(view.row_ids[local])
        for c, v in zip(cols, vs):
            rows.setdefault(c, []).append(logical)
            vals.setdefault(c, []).append(v)
    active = sorted(rows)
    coords = np.asarray([(a % grid_size, a // grid_size) for a in active], dtype=np.float64).reshape(-1, 2)
    return View(np.asarray(active, dtype=np.int64), [rows[a] for a in active], [vals[a] for a in active],
                coords, view.n_cols, view.output_size)


def morton2d(x: int, y: int) -> int:
    def spread(v: int) -> int:
        v &= 0xFFFF
        v = (v | (v << 8)) & 0x00FF00FF
        v = (v | (v << 4)) & 0x0F0F0F0F
        v = (v | (v << 2)) & 0x33333333
        v = (v | (v << 1)) & 0x55555555
        return v
    return spread(x) | (spread(y) << 1)


def row_order(view: View, policy: str, k_tile: int = K_TILE) -> list[int]:
    n = len(view.cols)
    if policy == "trajectory":
        return list(range(n))
    keys = [morton2d(max(0, int(round(view.coords[r, 0]))), max(0, int(round(view.coords[r, 1]))))
            for r in range(n)]
    order = sorted(range(n), key=keys.__getitem__)
    if policy == "morton":
        return order
    if policy not in ("overlap", "packing256"):
        raise ValueError(policy)
    sup = [set(c) for c in view.cols]
    window = 4 * M_TILE if policy == "overlap" else 16 * M_TILE
    out: list[int] = []
    for start in range(0, n, window):
        rem = order[start:start + window]
        while rem:
            group = [rem.pop(0)]
            union = set(sup[group[0]])
            while rem and len(group) < M_TILE:
                best, best_key = 0, None
                if policy == "overlap":
                    for pos, cand in enumerate(rem):
                        s = sup[cand]
                        key = (len(s & union), -len(s - union))
                        if best_key is None or key > best_key:
                            best, best_key = pos, key
                else:
                    nnz_now = sum(len(sup[r]) for r in group)
                    deg_now = max(len(sup[r]) for r in group)
                    for pos, cand in enumerate(rem):
                        s = sup[cand]
                        comb = len(union | s)
                        tiles = max(math.ceil(comb / k_tile), math.ceil(max(deg_now, len(s)) / (k_tile // 2)), 1)
                        util = (nnz_now + len(s)) / (tiles * M_TILE * k_tile // 2)
                        key = (util, len(s & union), -comb)
                        if best_key is None or key > best_key:
                            best, best_key = pos, key
                chosen = rem.pop(best)
                group.append(chosen)
                union |= sup[chosen]
            out.extend(group)
    return out


def column_masks(view: View, local_rows) -> dict[int, int]:
    masks: dict[int, int] = {}
    for slot, r in enumerate(local_rows):
        if r < 0:
            continue
        for c in view.cols[r]:
            masks[c] = masks.get(c, 0) | (1 << slot)
    return masks


def _bits(mask: int) -> list[int]:
    return [(mask >> i) & 1 for i in range(M_TILE)]


def _popcount_order(columns, masks, rng):
    tie = {c: rng.random() for c in columns}
    return sorted(columns, key=lambda c: (-bin(masks[c]).count("1"), tie[c]))


def assign_search(masks: dict[int, int], k_tile: int, seed: int) -> list[list[int]]:
    columns = list(masks)
    if not columns:
        return [[]]
    max_deg = max(sum(1 for m in masks.values() if m & (1 << r)) for r in range(M_TILE))
    min_tiles = max(math.ceil(len(columns) / k_tile), math.ceil(max_deg / (k_tile // 2)), 1)
    rng = random.Random(seed)
    for tile_count in range(min_tiles, min_tiles + 9):
        for _restart in range(24):
            ordered = _popcount_order(columns, masks, rng)
            tiles = [[] for _ in range(tile_count)]
            counts = [[0] * M_TILE for _ in range(tile_count)]
            ok = True
            for c in ordered:
                b = _bits(masks[c])
                best = None
                for t in range(tile_count):
                    if len(tiles[t]) >= k_tile:
                        continue
                    upd = [x + y for x, y in zip(counts[t], b)]
                    if max(upd) > k_tile // 2:
                        continue
                    ds = float(sum(u * u - x * x for u, x in zip(upd, counts[t])))
                    score = ds + len(tiles[t]) / k_tile + rng.random() * 1e-6
                    if best is None or (score, t) < best:
                        best = (score, t)
                if best is None:
                    ok = False
                    break
                t = best[1]
                tiles[t].append(c)
                counts[t] = [x + y for x, y in zip(counts[t], b)]
            if ok:
                return [t for t in tiles if t]
    raise RuntimeError("failed to partition columns into half-density tiles")


def assign_optimized(masks: dict[int, int], seed: int) -> list[list[int]]:
    columns = list(masks)
    if not columns:
        return [[]]
    max_deg = max(sum(1 for m in masks.values() if m & (1 << r)) for r in range(M_TILE))
    min_tiles = max(math.ceil(len(columns) / K_TILE), math.ceil(max_deg / (K_TILE // 2)), 1)
    rng = random.Random(seed)
    for tile_count in range(min_tiles, min_tiles + 9):
        for _restart in range(8):
            ordered = _popcount_order(columns, masks, rng)
            tiles = [[] for _ in range(tile_count)]
            counts = [[0] * M_TILE for _ in range(tile_count)]
            ok = True
            for c in ordered:
                b = _bits(masks[c])
                upds = [[x + y for x, y in zip(counts[t], b)] for t in range(tile_count)]
                valid = [len(tiles[t]) < K_TILE and max(upds[t]) <= K_TILE // 2 for t in range(tile_count)]
                if not any(valid):          # fails before drawing this column's tie-break noise
                    ok = False
                    break
                best, best_score = -1, math.inf
                for t in range(tile_count):
                    ds = float(sum(u * u - x * x for u, x in zip(upds[t], counts[t])))
                    score = (ds + len(tiles[t]) / K_TILE) + rng.random() * 1e-6
                    if valid[t] and score < best_score:
                        best, best_score = t, score
                tiles[best].append(c)
                counts[best] = [x + y for x, y in zip(counts[best], b)]
            if ok:
                return [t for t in tiles if t]
    raise RuntimeError("optimized column assignment failed")


def _quartets_flat(groups: list[list[int]]) -> list[int]:
    return [c for g in groups for c in (g + [-1] * (4 - len(g)))]


def arrange_search(columns, masks, k_tile: int, seed: int):
    if len(columns) > k_tile:
        raise ValueError("too many columns for tile")
    n_groups = k_tile // 4
    rng = random.Random(seed)
    for _restart in range(64):
        ordered = _popcount_order(columns, masks, rng)
        groups = [[] for _ in range(n_groups)]
        counts = [[0] * M_TILE for _ in range(n_groups)]
        ok = True
        for c in ordered:
            b = _bits(masks[c])
            best = None
            for g in range(n_groups):
                if len(groups[g]) >= 4:
                    continue
                upd = [x + y for x, y in zip(counts[g], b)]
                if max(upd) > 2:
                    continue
                overlap = sum(x * y for x, y in zip(counts[g], b))
                score = overlap * 100.0 + len(groups[g]) + rng.random() * 1e-6
                if best is None or (score, g) < best:
                    best = (score, g)
            if best is None:
                ok = False
                break
            g = best[1]
            groups[g].append(c)
            counts[g] = [x + y for x, y in zip(counts[g], b)]
        if ok:
            return _quartets_flat(groups), True, 0
    padded = list(columns) + [-1] * (k_tile - len(columns))
    worst = None
    for off in range(0, k_tile, 4):
        v = 0
        for r in range(M_TILE):
            cnt = sum(1 for c in padded[off:off + 4] if c >= 0 and masks[c] & (1 << r))
            v += max(0, cnt - 2)
        worst = v if worst is None else min(worst, v)
    return padded, False, int(worst)


def arrange_optimized(columns, masks, seed: int):
    n_groups = K_TILE // 4
    rng = random.Random(seed)
    for _restart in range(16):
        ordered = _popcount_order(columns, masks, rng)
        groups = [[] for _ in range(n_groups)]
        counts = [[0] * M_TILE for _ in range(n_groups)]
        ok = True
        for c in ordered:
            b = _bits(masks[c])
            valid = [len(groups[g]) < 4 and max(x + y for x, y in zip(counts[g], b)) <= 2
                     for g in range(n_groups)]
            if not any(valid):              # fails before drawing this column's tie-break noise
                ok = False
                break
            best, best_score = -1, math.inf
            for g in range(n_groups):
                overlap = sum(x * y for x, y in zip(counts[g], b))
                score = (overlap * 100.0 + len(groups[g])) + rng.random() * 1e-6
                if valid[g] and score < best_score:
                    best, best_score = g, score
            groups[best].append(c)
            counts[best] = [x + y for x, y in zip(counts[best], b)]
        if ok:
            return _quartets_flat(groups), True
    return list(columns) + [-1] * (K_TILE - len(columns)), False


def legal_24(values: np.ndarray) -> tuple[bool, int]:
    viol = 0
    for off in range(0, values.shape[1], 4):
        cnt = np.count_nonzero(values[:, off:off + 4], axis=1)
        viol += int(np.maximum(cnt - 2, 0).sum())
    return viol == 0, viol


def _materialize(view: View, local_rows, arranged, k_tile) -> tuple[np.ndarray, np.ndarray]:
    row_ids = np.asarray([int(view.row_ids[r]) if r >= 0 else -1 for r in local_rows], dtype=np.int32)
    values = np.zeros((M_TILE, k_tile), dtype=np.float64)
    for slot, r in enumerate(local_rows):
        if r < 0:
            continue
        row_map = dict(zip(view.cols[r], view.vals[r]))
        for j, c in enumerate(arranged):
            if c >= 0:
                values[slot, j] = row_map.get(c, 0.0)
    return row_ids, values


def split_illegal(tile: Tile) -> tuple[Tile, Tile]:
    """split24: first two nonzeros of every row-quartet to layer 0, the rest to layer 1."""
    l0 = np.zeros_like(tile.values)
    l1 = np.zeros_like(tile.values)
    k = tile.values.shape[1]
    for r in range(M_TILE):
        for off in range(0, k, 4):
            nz = [p for p in range(4) if tile.values[r, off + p] != 0.0]
            for p in nz[:2]:
                l0[r, off + p] = tile.values[r, off + p]
            for p in nz[2:]:
                l1[r, off + p] = tile.values[r, off + p]
    return (Tile(tile.row_ids.copy(), list(tile.col_ids), l0, True),
            Tile(tile.row_ids.copy(), list(tile.col_ids), l1, True))


def _groups(view: View, policy: str, k_tile: int):
    order = row_order(view, policy, k_tile)
    for gi, off in enumerate(range(0, len(order), M_TILE)):
        rows = order[off:off + M_TILE]
        yield gi, rows + [-1] * (M_TILE - len(rows))


def pack_search(view: View, policy: str, k_tile: int, seed: int) -> list[Tile]:
    """pack_view (src/nufft_layout_oracle.py:445-497)."""
    tiles: list[Tile] = []
    for gi, rows in _groups(view, policy, k_tile):
        masks = column_masks(view, rows)
        for ti, cols in enumerate(assign_search(masks, k_tile, seed + gi * 1009)):
            arranged, legal, viol = arrange_search(cols, masks, k_tile, seed + gi * 1009 + ti * 9176)
            row_ids, values = _materialize(view, rows, arranged, k_tile)
            tiles.append(Tile(row_ids, arranged, values, legal, viol))
    return tiles


def pack_fast(view: View, policy: str, seed: int) -> list[Tile]:
    """fast_split24_pack (src/export_torchkbnufft_gpu_case.py:46-99)."""
    del seed
    tiles: list[Tile] = []
    for _gi, rows in _groups(view, policy, K_TILE):
        union = sorted({c for r in rows if r >= 0 for c in view.cols[r]})
        for off in range(0, len(union), K_TILE):
            cols = union[off:off + K_TILE]
            cols = cols + [-1] * (K_TILE - len(cols))
            row_ids, values = _materialize(view, rows, cols, K_TILE)
            tile = Tile(row_ids, cols, values, legal_24(values)[0])
            tiles.extend([tile] if tile.legal else split_illegal(tile))
    return tiles


def pack_optimized(view: View, policy: str, seed: int) -> list[Tile]:
    """optimized_split24_pack (src/export_torchkbnufft_gpu_case.py:220-299)."""
    tiles: list[Tile] = []
    for gi, rows in _groups(view, policy, K_TILE):
        masks = column_masks(view, rows)
        for ti, cols in enumerate(assign_optimized(masks, seed + gi * 1009)):
            arranged, legal = arrange_optimized(cols, masks, seed + gi * 1009 + ti * 9176)
            row_ids, values = _materialize(view, rows, arranged, K_TILE)
            tile = Tile(row_ids, arranged, values, legal)
            tiles.extend([tile] if legal else split_illegal(tile))
    return tiles


def split_legal_and_residual(view: View, tiles: list[Tile], mode: str):
    """group offsets / row ids and split24 or CSR residual (src/export_gpu_case.py:110-155)."""
    offsets = [0]
    rows = []
    legal_tiles: list[Tile] = []
    res_cols = [[] for _ in range(view.output_size)]
    res_vals = [[] for _ in range(view.output_size)]
    prev = None
    for t in tiles:
        cur = tuple(int(v) for v in t.row_ids)
        if cur != prev:
            if prev is not None:
                offsets.append(len(legal_tiles))
            rows.append(t.row_ids.astype(np.int32))
            prev = cur
        if legal_24(t.values)[0]:
            legal_tiles.append(t)
        elif mode == "split24":
            legal_tiles.extend(split_illegal(t))
        else:
            for slot, lr in enumerate(t.row_ids):
                if lr < 0:
                    continue
                for j, lc in enumerate(t.col_ids):
                    v = float(t.values[slot, j])
                    if lc >= 0 and v != 0.0:
                        res_cols[int(lr)].append(int(lc))
                        res_vals[int(lr)].append(v)
    offsets.append(len(legal_tiles))
    ptr = np.zeros(view.output_size + 1, dtype=np.uint32)
    ptr[1:] = np.cumsum([len(c) for c in res_cols], dtype=np.uint64)
    return (np.asarray(offsets, dtype=np.uint32), np.stack(rows).astype(np.int32), legal_tiles, ptr,
            np.asarray([c for r in res_cols for c in r], dtype=np.int32),
            np.asarray([v for r in res_vals for v in r], dtype=np.float16))


def pair_metadata(row_meta: np.ndarray) -> np.ndarray:
    """mma.sp register pairing of per-row 4-bit codes (src/export_gpu_case.py:41-48)."""
    rm = np.asarray(row_meta, dtype=np.uint32).reshape(-1, M_TILE)
    out = np.zeros_like(rm)
    for g in range(8):
        a, b = rm[:, g], rm[:, g + 8]
        out[:, 2 * g] = (a & 0xFFFF) | ((b & 0xFFFF) << 16)
        out[:, 2 * g + 1] = (a >> 16) | (b & 0xFFFF0000)
    return out


def unpair_metadata(pair: np.ndarray) -> np.ndarray:
    """Inverse of pair_metadata (experiments/packing/prepare_dense_control.py:27-36)."""
    pm = np.asarray(pair, dtype=np.uint32).reshape(-1, M_TILE)
    out = np.zeros_like(pm)
    for g in range(8):
        a, b = pm[:, 2 * g], pm[:, 2 * g + 1]
        out[:, g] = (a & 0xFFFF) | ((b & 0xFFFF) << 16)
        out[:, g + 8] = (a >> 16) | (b & 0xFFFF0000)
    return out


def compress(tiles: list[Tile]) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """FP16 2:4 compression -> (values [T,16,16] f16, row codes [T,16] u32, pair meta [T,16] u32)."""
    n = len(tiles)
    comp = np.zeros((n, M_TILE, K_TILE // 2), dtype=np.float16)
    codes = np.zeros((n, M_TILE), dtype=np.uint32)
    for i, t in enumerate(tiles):
        half = t.values.astype(np.float16)
        for r in range(M_TILE):
            word = 0
            for q in range(K_TILE // 4):
                four = half[r, 4 * q:4 * q + 4]
                nz = [p for p in range(4) if four[p] != 0]
                if len(nz) > 2:
                    raise ValueError("tile is not legal 2:4 after FP16 rounding")
                sel = nz + [p for p in range(4) if p not in nz][: 2 - len(nz)]
                p0, p1 = sorted(sel)
                comp[i, r, 2 * q] = four[p0]
                comp[i, r, 2 * q + 1] = four[p1]
                word |= (p0 | (p1 << 2)) << (4 * q)
            codes[i, r] = word
    return comp, codes, pair_metadata(codes)


def header_bytes(output_size, n_cols, active_rows, nnz, groups, tiles, residual_nnz) -> bytes:
    return struct.pack("<Q11I", MAGIC, VERSION, N_CHANNELS, output_size, n_cols, active_rows, nnz,
                       groups, tiles, residual_nnz, M_TILE, K_TILE)


def component_tiles(structure_tiles: list[Tile], component: View) -> list[Tile]:
    """Real/imag values on the shared structure (src/export_torchkbnufft_gpu_case.py:356-384)."""
    lookup = {int(r): i for i, r in enumerate(component.row_ids)}
    maps = [dict(zip(c, v)) for c, v in zip(component.cols, component.vals)]
    out = []
    for st in structure_tiles:
        vals = np.zeros_like(st.values)
        for slot, lr in enumerate(st.row_ids):
            if lr < 0:
                continue
            rm = maps[lookup[int(lr)]]
            for j, lc in enumerate(st.col_ids):
                if lc >= 0 and st.values[slot, j] != 0.0:
                    vals[slot, j] = rm.get(int(lc), 0.0)
        out.append(Tile(st.row_ids.copy(), list(st.col_ids), vals, True))
    return out


def export_component_arrays(component: View, offsets, row_ids, structure_tiles) -> dict[str, bytes]:
    """The six production pack arrays + header of one component directory."""
    tiles = component_tiles(structure_tiles, component)
    col_ids = np.asarray([t.col_ids for t in tiles], dtype=np.int32)
    col_ids[col_ids < 0] = 0
    comp, _codes, pair = compress(tiles)
    header = header_bytes(component.output_size, component.n_cols, len(component.cols), component.nnz,
                          len(offsets) - 1, len(tiles), 0)
    return {
        "header.bin": header,
        "group_offsets.bin": np.ascontiguousarray(offsets, dtype=np.uint32).tobytes(),
        "group_row_ids.bin": np.ascontiguousarray(row_ids, dtype=np.int32).tobytes(),
        "tile_col_ids.bin": col_ids.tobytes(),
        "tile_a_comp.bin": comp.tobytes(),
        "tile_pair_meta.bin": pair.astype(np.uint32).tobytes(),
    }
