"""Pack once: KB coefficients, the 2:4 planner and the reference pack-directory format.

Python mirror of the reference's pack-once entry points, each served by the C++
planner through the C ABI:

* ``kb_interpolation_csr``  the complex KB matrix (replaces
  ``tkbn.calc_tensor_spmatrix``, src/export_torchkbnufft_gpu_case.py:537-567)
* ``pack_view``             src/nufft_layout_oracle.py:445-497 (planner="search"),
  ``fast_split24_pack`` / ``optimized_split24_pack``
  (src/export_torchkbnufft_gpu_case.py:46-99, :270-299)
* ``export_view_dir``       export_case arrays (src/export_gpu_case.py:171-321)
* ``export_production``     the production G / G_T real+imag directories
  (src/export_torchkbnufft_gpu_case.py:513-646 with --optimized-pack --production-only)
* ``decode_row_metadata``   the pair-metadata inverse
  (experiments/packing/prepare_dense_control.py:27-36)
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check, lib, ptr

M_TILE = 16
K_TILE = 32
MAGIC = 0x4E55464654323431
HEADER_FIELDS = ("magic", "version", "n_channels", "output_size", "n_cols", "active_rows", "nnz", "groups",
                 "tiles", "residual_nnz", "m_tile", "k_tile")


@dataclass
class PackedTile:
    row_ids: np.ndarray
    col_ids: np.ndarray
    values: np.ndarray
    legal_24: bool


def _f32_traj(trajectory) -> np.ndarray:
    t = np.ascontiguousarray(np.asarray(trajectory, dtype=np.float32).reshape(-1, 2))
    return t


def kb_interpolation_csr(trajectory, im_size: int, grid_size: int, width: int):
    """(row_ptr, cols, re, im) of the complex KB interpolation matrix (FP64)."""
    t = _f32_traj(trajectory)
    m = t.shape[0]
    nnz = C.c_int64(0)
    check(lib().tsn_kb_interpolation_csr(ptr(t, C.c_float), m, im_size, grid_size, width, None, None, None, None,
                                         C.byref(nnz)))
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    cols = np.zeros(nnz.value, dtype=np.int64)
    re = np.zeros(nnz.value, dtype=np.float64)
    im = np.zeros(nnz.value, dtype=np.float64)
    check(lib().tsn_kb_interpolation_csr(ptr(t, C.c_float), m, im_size, grid_size, width, ptr(row_ptr, C.c_int64),
                                         ptr(cols, C.c_int64), ptr(re, C.c_double), ptr(im, C.c_double),
                                         C.byref(nnz)))
    return row_ptr, cols, re, im


def kb_deapodization(im_size: int, grid_size: int, width: int) -> np.ndarray:
    out = np.zeros((im_size, im_size), dtype=np.float64)
    check(lib().tsn_kb_deapodization(im_size, grid_size, width, ptr(out, C.c_double)))
    return out


def kb_weights_csr3(trajectory, im_size: int, grid_size: int, width: int):
    """(row_ptr, cols, w) of the real KB weights of a [M, 3] trajectory (volume layout)."""
    t = np.ascontiguousarray(np.asarray(trajectory, dtype=np.float32).reshape(-1, 3))
    m = t.shape[0]
    nnz = C.c_int64(0)
    check(lib().tsn_kb_weights_csr3(ptr(t, C.c_float), m, im_size, grid_size, width, None, None, None, C.byref(nnz)))
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    cols = np.zeros(nnz.value, dtype=np.int64)
    w = np.zeros(nnz.value, dtype=np.float64)
    check(lib().tsn_kb_weights_csr3(ptr(t, C.c_float), m, im_size, grid_size, width, ptr(row_ptr, C.c_int64),
                                    ptr(cols, C.c_int64), ptr(w, C.c_double), C.byref(nnz)))
    return row_ptr, cols, w


def kb_deapodization3(im_size: int, grid_size: int, width: int) -> np.ndarray:
    out = np.zeros((im_size,) * 3, dtype=np.float64)
    check(lib().tsn_kb_deapodization3(im_size, grid_size, width, ptr(out, C.c_double)))
    return out


def _csr_args(row_ptr, cols, vals, row_ids, coords):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    vals = None if vals is None else np.ascontiguousarray(vals, dtype=np.float64)
    row_ids = None if row_ids is None else np.ascontiguousarray(row_ids, dtype=np.int64)
    coords = None if coords is None else np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 2)
    return row_ptr, cols, vals, row_ids, coords


def pack_view(row_ptr, cols, vals, *, row_ids=None, coords=None, output_size: int, n_cols: int,
              policy: str = "overlap", k_tile: int = 32, seed: int = 20260823, planner: str = "search",
              threads: int = 0) -> list[PackedTile]:
    """Pack one real sparse view into M16 x K tiles (legal 2:4 unless the search gave up)."""
    row_ptr, cols, vals, row_ids, coords = _csr_args(row_ptr, cols, vals, row_ids, coords)
    rows = len(row_ptr) - 1
    n = C.c_int64(0)
    args = (ptr(row_ptr, C.c_int64), ptr(cols, C.c_int64), ptr(vals, C.c_double), ptr(row_ids, C.c_int64),
            ptr(coords, C.c_double), rows, output_size, n_cols, _lib.PLANNER[planner], _lib.POLICY[policy],
            k_tile, seed, threads)
    check(lib().tsn_pack_view_tiles(*args, C.byref(n), None, None, None, None))
    t = n.value
    rid = np.zeros((t, M_TILE), dtype=np.int32)
    cid = np.zeros((t, k_tile), dtype=np.int32)
    val = np.zeros((t, M_TILE, k_tile), dtype=np.float64)
    legal = np.zeros(t, dtype=np.uint8)
    check(lib().tsn_pack_view_tiles(*args, C.byref(n), ptr(rid, C.c_int32), ptr(cid, C.c_int32),
                                    ptr(val, C.c_double), ptr(legal, C.c_uint8)))
    return [PackedTile(rid[i], cid[i], val[i], bool(legal[i])) for i in range(t)]


def export_view_dir(row_ptr, cols, vals, out_dir, *, row_ids=None, coords=None, output_size: int, n_cols: int,
                    policy: str = "overlap", seed: int = 20260823, illegal_mode: str = "csr_residual",
                    planner: str = "search", threads: int = 0) -> Path:
    row_ptr, cols, vals, row_ids, coords = _csr_args(row_ptr, cols, vals, row_ids, coords)
    out = Path(out_dir)
    check(lib().tsn_export_view_dir(ptr(row_ptr, C.c_int64), ptr(cols, C.c_int64), ptr(vals, C.c_double),
                                    ptr(row_ids, C.c_int64), ptr(coords, C.c_double), len(row_ptr) - 1, output_size,
                                    n_cols, _lib.PLANNER[planner], _lib.POLICY[policy], seed,
                                    _lib.ILLEGAL[illegal_mode], threads, str(out).encode()))
    return out


def export_csr_dirs(row_ptr, cols, re, im, trajectory, grid_size: int, out_dir, *, view: str = "G",
                    planner: str = "optimized", policy: str = "morton", seed: int = 20260823,
                    threads: int = 0) -> Path:
    """Production real/imag directories of one view from a complex CSR over samples."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    re = np.ascontiguousarray(re, dtype=np.float64)
    im = np.ascontiguousarray(im, dtype=np.float64)
    t = _f32_traj(trajectory)
    out = Path(out_dir)
    check(lib().tsn_pack_csr_to_dirs(ptr(row_ptr, C.c_int64), ptr(cols, C.c_int64), ptr(re, C.c_double),
                                     ptr(im, C.c_double), len(row_ptr) - 1, grid_size, ptr(t, C.c_float),
                                     _lib.VIEW[view], _lib.PLANNER[planner], _lib.POLICY[policy], seed, threads,
                                     str(out).encode()))
    return out


def export_production(trajectory, out_root, *, im_size: int = 256, grid_size: int = 512, width: int = 6,
                      planner: str = "optimized", policy: str = "morton", seed: int = 20260823,
                      threads: int = 0) -> dict[str, Path]:
    """Write out_root/{G,G_T}/{real,imag} for a trajectory in cycles/pixel."""
    row_ptr, cols, re, im = kb_interpolation_csr(trajectory, im_size, grid_size, width)
    root = Path(out_root)
    dirs = {}
    for view in ("G", "G_T"):
        dirs[view] = export_csr_dirs(row_ptr, cols, re, im, trajectory, grid_size, root / view, view=view,
                                     planner=planner, policy=policy, seed=seed, threads=threads)
    return dirs


def read_header(directory) -> dict:
    raw = (Path(directory) / "header.bin").read_bytes()
    vals = np.frombuffer(raw[:8], dtype="<u8").tolist() + np.frombuffer(raw[8:52], dtype="<u4").tolist()
    return dict(zip(HEADER_FIELDS, vals))


def decode_row_metadata(pair_meta: np.ndarray) -> np.ndarray:
    """Per-row 4-bit-code words from mma.sp pair metadata ([tiles, 16] u32)."""
    pm = np.asarray(pair_meta, dtype=np.uint32).reshape(-1, M_TILE)
    out = np.zeros_like(pm)
    for g in range(8):
        a, b = pm[:, 2 * g], pm[:, 2 * g + 1]
        out[:, g] = (a & 0xFFFF) | ((b & 0xFFFF) << 16)
        out[:, g + 8] = (a >> 16) | (b & 0xFFFF0000)
    return out


def expand_tiles(directory) -> np.ndarray:
    """Dense [tiles, 16, 32] FP16 tiles of one component directory."""
    d = Path(directory)
    h = read_header(d)
    t = h["tiles"]
    comp = np.fromfile(d / "tile_a_comp.bin", dtype=np.float16).reshape(t, M_TILE, K_TILE // 2)
    meta = decode_row_metadata(np.fromfile(d / "tile_pair_meta.bin", dtype=np.uint32).reshape(t, M_TILE))
    dense = np.zeros((t, M_TILE, K_TILE), dtype=np.float16)
    rows = np.arange(M_TILE)[None, :]
    tiles = np.arange(t)[:, None]
    for q in range(K_TILE // 4):
        code = (meta >> np.uint32(4 * q)) & np.uint32(0xF)
        p0 = (code & 3).astype(np.int64)
        p1 = ((code >> 2) & 3).astype(np.int64)
        dense[tiles, rows, 4 * q + p0] = comp[:, :, 2 * q]
        dense[tiles, rows, 4 * q + p1] = comp[:, :, 2 * q + 1]
    return dense
