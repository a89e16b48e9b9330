"""Readers for the committed golden fixtures (tests only)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
PACK_FILES = ("header.bin", "group_offsets.bin", "group_row_ids.bin", "tile_col_ids.bin",
              "tile_a_comp.bin", "tile_pair_meta.bin")


def layout_packs():
    z = np.load(GOLDEN / "layout_packs.npz")
    index = json.loads(bytes(z["index"]).decode())
    return z, index


def csr_view(z, name):
    return {k: z[f"{name}/csr/{k}"] for k in ("row_ptr", "cols", "vals", "row_ids", "coords",
                                                "output_size", "n_cols")}


def read_dir(path: Path, names=PACK_FILES) -> dict[str, bytes]:
    return {n: (path / n).read_bytes() for n in names}


def prod_input(name: str):
    return dict(np.load(GOLDEN / name / "input_csr.npz"))
