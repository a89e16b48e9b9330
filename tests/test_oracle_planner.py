"""The oracle planner restatement reproduces the reference's own packs byte-for-byte.

Goldens come from tests/golden/make_golden.py, which runs the reference
(src/nufft_layout_oracle.py, src/export_gpu_case.py,
src/export_torchkbnufft_gpu_case.py) on the same inputs.
"""
import json

import numpy as np
import pytest

from golden_io import GOLDEN, PACK_FILES, csr_view, layout_packs, prod_input, read_dir
from oracle import planner as P


def _view(c):
    v = P.view_from_csr(c["row_ptr"], c["cols"], c["vals"], c["coords"], int(c["n_cols"]), c["row_ids"])
    v.output_size = int(c["output_size"])
    return v


def _cases():
    z, index = layout_packs()
    return [(e["tag"], e) for e in index]


@pytest.mark.parametrize("tag,entry", _cases(), ids=[t for t, _ in _cases()])
def test_pack_search_matches_reference(tag, entry):
    z, _ = layout_packs()
    view = _view(csr_view(z, entry["view"]))
    tiles = P.pack_search(view, entry["policy"], entry["k_tile"], entry["seed"])
    assert len(tiles) == len(z[f"{tag}/legal"])
    np.testing.assert_array_equal(np.stack([t.row_ids for t in tiles]), z[f"{tag}/row_ids"])
    np.testing.assert_array_equal(np.asarray([t.col_ids for t in tiles]), z[f"{tag}/col_ids"])
    np.testing.assert_array_equal(np.stack([t.values for t in tiles]), z[f"{tag}/values"])
    np.testing.assert_array_equal(np.asarray([t.legal for t in tiles]), z[f"{tag}/legal"])


def _prod_arrays(name, view_name, planner):
    inp = prod_input(name)
    g = int(inp["grid"])
    traj = inp["trajectory"]
    coords = np.mod(traj.astype(np.float64) * g + g / 2.0, g)
    n_cols = g * g
    re = P.view_from_csr(inp["row_ptr"], inp["cols"], inp["re"], coords, n_cols)
    im = P.view_from_csr(inp["row_ptr"], inp["cols"], inp["im"], coords, n_cols)
    st = P.view_from_csr(inp["row_ptr"], inp["cols"], np.ones_like(inp["re"]), coords, n_cols)
    if view_name == "G_T":
        re, im, st = P.transpose(re, g), P.transpose(im, g), P.transpose(st, g)
    seed = int(inp["seed"])
    if planner == "optimized":
        tiles = P.pack_optimized(st, "morton", seed)
    elif planner == "fast":
        tiles = P.pack_fast(st, "morton", seed)
    else:
        tiles = P.pack_search(st, "overlap", P.K_TILE, seed)
    offsets, row_ids, legal, _, res_cols, _ = P.split_legal_and_residual(st, tiles, "split24")
    assert len(res_cols) == 0
    return {"real": P.export_component_arrays(re, offsets, row_ids, legal),
            "imag": P.export_component_arrays(im, offsets, row_ids, legal)}


@pytest.mark.parametrize("name,planner", [("prod_radial16_opt", "optimized"),
                                          ("prod_radial16_fast", "fast"),
                                          ("prod_radial16_oracle", "search")])
@pytest.mark.parametrize("view_name", ["G", "G_T"])
def test_production_component_dirs_match_reference(name, planner, view_name):
    arrays = _prod_arrays(name, view_name, planner)
    for comp in ("real", "imag"):
        want = read_dir(GOLDEN / name / view_name / comp)
        for f in PACK_FILES:
            assert arrays[comp][f] == want[f], f"{name}/{view_name}/{comp}/{f}"


def test_pair_metadata_roundtrip():
    rng = np.random.default_rng(5)
    codes = rng.integers(0, 2**32, size=(7, 16), dtype=np.uint64).astype(np.uint32)
    np.testing.assert_array_equal(P.unpair_metadata(P.pair_metadata(codes)), codes)


@pytest.mark.parametrize("name", ["export_spiral24_gt_csr", "export_spiral24_gt_split", "export_radial32_g_split"])
def test_export_case_dirs_match_reference(name):
    """export_case (src/export_gpu_case.py:171-321) pack arrays + residual CSR."""
    from oracle import layout
    spec = json.loads((GOLDEN / name / "spec.json").read_text())
    view = layout.build_view(spec)
    tiles = P.pack_search(view, spec["policy"], P.K_TILE, spec["seed"])
    offsets, row_ids, legal, rptr, rcols, rvals = P.split_legal_and_residual(view, tiles, spec["illegal_mode"])
    col_ids = np.asarray([t.col_ids for t in legal], dtype=np.int32)
    col_ids[col_ids < 0] = 0
    comp, _, pair = P.compress(legal)
    got = {
        "header.bin": P.header_bytes(view.output_size, view.n_cols, len(view.cols), view.nnz,
                                     len(offsets) - 1, len(legal), len(rcols)),
        "group_offsets.bin": offsets.tobytes(), "group_row_ids.bin": row_ids.tobytes(),
        "tile_col_ids.bin": col_ids.tobytes(), "tile_a_comp.bin": comp.tobytes(),
        "tile_pair_meta.bin": pair.tobytes(), "residual_row_ptr.bin": rptr.tobytes(),
        "residual_cols.bin": rcols.tobytes(), "residual_vals.bin": rvals.tobytes(),
    }
    want = read_dir(GOLDEN / name, tuple(got))
    for f in got:
        assert got[f] == want[f], f
