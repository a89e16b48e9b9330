#!/usr/bin/env python3
"""Generate the committed golden pack fixtures by running the reference itself.

Run in a container where the reference repository is checked out, naming its root:

    python tests/golden/make_golden.py --reference-root <path of the reference checkout>

(or set TSN_REFERENCE_ROOT).  The GPU box never runs this script; tests read only the
files it writes next to it.

Fixtures
--------
layout_packs.npz
    ``pack_view`` outputs (src/nufft_layout_oracle.py:445-497) for the
    reference unit-test trajectory (tests/test_oracle.py:20-22) and a small
    spiral over every row-grouping policy and both K tiles; per tile:
    row_ids, col_ids, FP64 values, legality flag.  The input CSR is stored too.
export_*/
    ``export_case`` directories (src/export_gpu_case.py:171-321) including
    the tests/test_export_gpu_case.py:18-33 case, in both illegal-tile modes.
prod_*/
    production directories (G and G_T, real + imag) made by the reference's
    ``optimized_split24_pack`` / ``fast_split24_pack`` / ``pack_view`` +
    ``split_legal_tiles_and_residual(..., "split24")`` + ``export_component``
    (src/export_torchkbnufft_gpu_case.py:270-299, :387-489) on a complex KB
    matrix from oracle/kb.py (torchkbnufft is not available); the CSR it was
    given is stored as prod_*/input_csr.npz so the C++ planner can be fed the
    identical coefficients.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import shutil
import sys
import types
from argparse import Namespace
from contextlib import redirect_stdout
from io import StringIO
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from oracle import kb  # noqa: E402
from trajsparsenufft_b200 import synth  # noqa: E402

# the reference's modules, bound by load_reference()
ref_oracle = ref_export = ref_prod = None


def load_reference(root: Path) -> None:
    """Import the reference's src/ modules from the checkout at `root`."""
    global ref_oracle, ref_export, ref_prod
    sys.path.insert(0, str(root))
    # export_torchkbnufft_gpu_case imports torchkbnufft at module load but its
    # planner functions never call it.
    sys.modules.setdefault("torchkbnufft", types.ModuleType("torchkbnufft"))
    ref_oracle = importlib.import_module("src.nufft_layout_oracle")
    ref_export = importlib.import_module("src.export_gpu_case")
    ref_prod = importlib.import_module("src.export_torchkbnufft_gpu_case")


def csr_of(view) -> dict:
    counts = np.asarray([len(c) for c in view.cols], dtype=np.int64)
    ptr = np.zeros(len(counts) + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(counts)
    return {
        "row_ptr": ptr,
        "cols": np.concatenate(view.cols).astype(np.int64) if len(view.cols) else np.zeros(0, np.int64),
        "vals": np.concatenate(view.vals).astype(np.float64) if len(view.vals) else np.zeros(0),
        "row_ids": np.asarray(view.row_ids, dtype=np.int64),
        "coords": np.asarray(view.coords, dtype=np.float64),
        "output_size": np.int64(view.output_size),
        "n_cols": np.int64(view.n_cols),
    }


def pack_arrays(packed) -> dict:
    return {
        "row_ids": np.stack([t.row_ids for t in packed.tiles]).astype(np.int32),
        "col_ids": np.stack([t.col_ids for t in packed.tiles]).astype(np.int32),
        "values": np.stack([t.values for t in packed.tiles]).astype(np.float64),
        "legal": np.asarray([t.legal_24 for t in packed.tiles], dtype=np.bool_),
        "violation": np.asarray([t.violation_count for t in packed.tiles], dtype=np.int64),
    }


def make_layout_packs() -> None:
    out: dict[str, np.ndarray] = {}
    cases = []
    traj = ref_oracle.generate_trajectory("radial", 24, 96)
    fwd = ref_oracle.build_interpolation(traj, 24, 4)
    adj = ref_oracle.transpose_sparse(fwd, 24)
    cases.append(("radial24_G", fwd, [("overlap", 32, 7), ("overlap", 32, 11)]))
    cases.append(("radial24_GT", adj, [("overlap", 32, 13)]))
    traj = ref_oracle.generate_trajectory("spiral", 32, 256)
    fwd = ref_oracle.build_interpolation(traj, 32, 6)
    adj = ref_oracle.transpose_sparse(fwd, 32)
    plans = [(p, k, 20260823 + k) for p in ref_oracle.ROW_GROUPING_POLICIES for k in (32, 64)]
    cases.append(("spiral32_G", fwd, plans))
    cases.append(("spiral32_GT", adj, plans))
    index = []
    for name, view, specs in cases:
        for key, value in csr_of(view).items():
            out[f"{name}/csr/{key}"] = value
        for policy, k_tile, seed in specs:
            packed = ref_oracle.pack_view(view, policy, k_tile, seed)
            tag = f"{name}/{policy}/k{k_tile}/s{seed}"
            for key, value in pack_arrays(packed).items():
                out[f"{tag}/{key}"] = value
            index.append({"view": name, "policy": policy, "k_tile": k_tile, "seed": seed, "tag": tag})
    out["index"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "layout_packs.npz", **out)


def make_exports() -> None:
    specs = [
        ("export_spiral24_gt_csr", dict(trajectory="spiral", view="G_T", grid=24, width=4, samples=192,
                                          policy="overlap", illegal_mode="csr_residual", seed=23)),
        ("export_spiral24_gt_split", dict(trajectory="spiral", view="G_T", grid=24, width=4, samples=192,
                                            policy="overlap", illegal_mode="split24", seed=23)),
        ("export_radial32_g_split", dict(trajectory="radial", view="G", grid=32, width=6, samples=256,
                                           policy="morton", illegal_mode="split24", seed=20260823)),
    ]
    for name, spec in specs:
        target = HERE / name
        if target.exists():
            shutil.rmtree(target)
        args = Namespace(trajectory_file=None, periodic=False, output_dir=target, **spec)
        with redirect_stdout(StringIO()):
            ref_export.export_case(args)
        (target / "spec.json").write_text(json.dumps(spec, sort_keys=True) + "\n")


def sparse_rows(name, row_ptr, cols, vals, output_size, n_cols, coords):
    return ref_oracle.SparseRows(
        name=name,
        output_size=int(output_size),
        n_cols=int(n_cols),
        row_ids=np.arange(int(output_size), dtype=np.int32),
        coords=np.asarray(coords, dtype=np.float64),
        cols=tuple(np.asarray(cols[row_ptr[r]:row_ptr[r + 1]], dtype=np.int32) for r in range(int(output_size))),
        vals=tuple(np.asarray(vals[row_ptr[r]:row_ptr[r + 1]], dtype=np.float64) for r in range(int(output_size))),
    )


def make_production(name: str, trajectory: np.ndarray, im_size: int, grid: int, width: int,
                    planner: str, policy: str, seed: int) -> None:
    target = HERE / name
    if target.exists():
        shutil.rmtree(target)
    target.mkdir(parents=True)
    row_ptr, cols, re, im = kb.interpolation_csr(trajectory, im_size, grid, width)
    m = len(row_ptr) - 1
    coords = np.mod(trajectory.astype(np.float64) * grid + grid / 2.0, grid)
    np.savez_compressed(target / "input_csr.npz", row_ptr=row_ptr, cols=cols, re=re, im=im,
                        trajectory=trajectory, im_size=im_size, grid=grid, width=width, seed=seed)
    real_f = sparse_rows("KB_REAL_G", row_ptr, cols, re, m, grid * grid, coords)
    imag_f = sparse_rows("KB_IMAG_G", row_ptr, cols, im, m, grid * grid, coords)
    struct_f = sparse_rows("KB_STRUCTURE_G", row_ptr, cols, np.ones_like(re), m, grid * grid, coords)
    for view_name in ("G", "G_T"):
        if view_name == "G_T":
            real_v = ref_oracle.transpose_sparse(real_f, grid)
            imag_v = ref_oracle.transpose_sparse(imag_f, grid)
            struct_v = ref_oracle.transpose_sparse(struct_f, grid)
        else:
            real_v, imag_v, struct_v = real_f, imag_f, struct_f
        if planner == "optimized":
            packed = ref_prod.optimized_split24_pack(struct_v, policy, seed, 1)
        elif planner == "fast":
            packed = ref_prod.fast_split24_pack(struct_v, policy, seed)
        else:
            packed = ref_oracle.pack_view(struct_v, policy, ref_export.K_TILE, seed)
        offsets, row_ids, tiles, _, residual_cols, _ = ref_export.split_legal_tiles_and_residual(
            struct_v, packed, "split24")
        assert len(residual_cols) == 0
        rng = np.random.default_rng(seed)
        dense_input = np.clip(rng.standard_normal((struct_v.n_cols, ref_export.N_CHANNELS)), -3.0, 3.0).astype(np.float16)
        common = {"experiment_id": "golden", "view": view_name, "im_size": im_size, "grid_size": grid,
                  "numpoints": width, "samples": m, "policy": policy, "illegal_mode": "split24",
                  "seed": seed, "n_channels": ref_export.N_CHANNELS, "m_tile": ref_oracle.M_TILE,
                  "k_tile": ref_export.K_TILE, "planner": planner}
        for comp_name, comp in (("real", real_v), ("imag", imag_v)):
            ref_prod.export_component(target / view_name / comp_name, comp_name, comp, offsets, row_ids,
                                      tiles, dense_input, common, False)


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference-root", default=os.environ.get("TSN_REFERENCE_ROOT"),
                    help="root of the reference checkout (or TSN_REFERENCE_ROOT)")
    args = ap.parse_args()
    if not args.reference_root:
        ap.error("name the reference checkout with --reference-root or TSN_REFERENCE_ROOT")
    root = Path(args.reference_root)
    if not (root / "src" / "nufft_layout_oracle.py").is_file():
        print(f"reference not found at {root}", file=sys.stderr)
        return 2
    load_reference(root)
    make_layout_packs()
    make_exports()
    small = synth.golden_radial(16, 32)
    make_production("prod_radial16_opt", small, 16, 32, 6, "optimized", "morton", 20260823)
    make_production("prod_radial16_fast", small, 16, 32, 6, "fast", "morton", 20260823)
    make_production("prod_radial16_oracle", small, 16, 32, 6, "oracle", "overlap", 20260823)
    spiral = synth.vd_spiral(4, 256)
    make_production("prod_spiral32_opt", spiral, 32, 64, 6, "optimized", "morton", 20260823)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
