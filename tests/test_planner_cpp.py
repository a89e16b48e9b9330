"""The C++ pack-once planner (through the C ABI) matches the reference byte-for-byte.

Golden packs were produced by the reference itself (tests/golden/make_golden.py);
additional seeds/policies are checked against the oracle restatement, which is
itself pinned to those goldens (tests/test_oracle_planner.py).
"""
import json
import re
from pathlib import Path

import numpy as np
import pytest

from golden_io import GOLDEN, PACK_FILES, csr_view, layout_packs, prod_input, read_dir
from oracle import kb as okb
from oracle import layout as olayout
from oracle import planner as P
from trajsparsenufft_b200 import _lib, packing

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "trajsparsenufft.h").read_text()
    declared = set(re.findall(r"\b(tsn_[a-z0-9_]+)\s*\(", header))
    L = _lib.lib()
    for name in sorted(declared):
        assert hasattr(L, name), name
    assert declared == set(_lib.EXPORTED)
    assert b"sm_100a" in L.tsn_version()


def _golden_cases():
    _, index = layout_packs()
    return [(e["tag"], e) for e in index]


@pytest.mark.parametrize("tag,entry", _golden_cases(), ids=[t for t, _ in _golden_cases()])
def test_cpp_pack_view_matches_reference(tag, entry):
    z, _ = layout_packs()
    c = csr_view(z, entry["view"])
    tiles = packing.pack_view(c["row_ptr"], c["cols"], c["vals"], row_ids=c["row_ids"], coords=c["coords"],
                              output_size=int(c["output_size"]), n_cols=int(c["n_cols"]), policy=entry["policy"],
                              k_tile=entry["k_tile"], seed=entry["seed"], planner="search")
    assert len(tiles) == len(z[f"{tag}/legal"])
    np.testing.assert_array_equal(np.stack([t.row_ids for t in tiles]), z[f"{tag}/row_ids"])
    np.testing.assert_array_equal(np.stack([t.col_ids for t in tiles]), z[f"{tag}/col_ids"])
    np.testing.assert_array_equal(np.stack([t.values for t in tiles]), z[f"{tag}/values"])
    np.testing.assert_array_equal(np.asarray([t.legal_24 for t in tiles]), z[f"{tag}/legal"])


@pytest.mark.parametrize("name,planner,policy", [("prod_radial16_opt", "optimized", "morton"),
                                                 ("prod_radial16_fast", "fast", "morton"),
                                                 ("prod_radial16_oracle", "search", "overlap"),
                                                 ("prod_spiral32_opt", "optimized", "morton")])
@pytest.mark.parametrize("view", ["G", "G_T"])
def test_cpp_production_dirs_match_reference(tmp_path, name, planner, policy, view):
    inp = prod_input(name)
    out = packing.export_csr_dirs(inp["row_ptr"], inp["cols"], inp["re"], inp["im"], inp["trajectory"],
                                  int(inp["grid"]), tmp_path / view, view=view, planner=planner, policy=policy,
                                  seed=int(inp["seed"]))
    for comp in ("real", "imag"):
        got = read_dir(out / comp)
        want = read_dir(GOLDEN / name / view / comp)
        for f in PACK_FILES:
            assert got[f] == want[f], f"{name}/{view}/{comp}/{f}"
        manifest = json.loads((out / comp / "manifest.json").read_text())
        assert {e["file"] for e in manifest["files"]} == set(PACK_FILES)
        assert manifest["tiles"] == packing.read_header(out / comp)["tiles"]


@pytest.mark.parametrize("name", ["export_spiral24_gt_csr", "export_spiral24_gt_split", "export_radial32_g_split"])
def test_cpp_export_case_matches_reference(tmp_path, name):
    spec = json.loads((GOLDEN / name / "spec.json").read_text())
    view = olayout.build_view(spec)
    counts = [len(c) for c in view.cols]
    row_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    out = packing.export_view_dir(row_ptr, np.concatenate(view.cols), np.concatenate(view.vals), tmp_path,
                                  row_ids=view.row_ids, coords=view.coords, output_size=view.output_size,
                                  n_cols=view.n_cols, policy=spec["policy"], seed=spec["seed"],
                                  illegal_mode=spec["illegal_mode"])
    names = PACK_FILES + ("residual_row_ptr.bin", "residual_cols.bin", "residual_vals.bin")
    got, want = read_dir(out, names), read_dir(GOLDEN / name, names)
    for f in names:
        assert got[f] == want[f], f


def _random_view(seed: int, kind: str):
    rng = np.random.default_rng(seed)
    grid = int(rng.choice([16, 24, 32]))
    samples = int(rng.integers(40, 160))
    traj = olayout.generate_trajectory(kind, grid, samples)
    traj = traj + rng.uniform(-0.3, 0.3, traj.shape)
    traj = np.clip(traj, 0.0, grid - 1.0)
    fwd = olayout.build_interpolation(traj, grid, int(rng.choice([4, 6])))
    return (P.transpose(fwd, grid) if rng.random() < 0.5 else fwd), grid


@pytest.mark.parametrize("seed", range(12))
def test_cpp_planner_matches_oracle_on_random_views(seed):
    view, _ = _random_view(1000 + seed, "radial" if seed % 2 else "spiral")
    counts = [len(c) for c in view.cols]
    row_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    cols, vals = np.concatenate(view.cols), np.concatenate(view.vals)
    policy = ["trajectory", "morton", "overlap", "packing256"][seed % 4]
    planner = ["search", "fast", "optimized"][seed % 3]
    pseed = 7 + 31 * seed
    got = packing.pack_view(row_ptr, cols, vals, row_ids=view.row_ids, coords=view.coords,
                            output_size=view.output_size, n_cols=view.n_cols, policy=policy, k_tile=32,
                            seed=pseed, planner=planner, threads=3)
    if planner == "search":
        want = P.pack_search(view, policy, 32, pseed)
    elif planner == "fast":
        want = P.pack_fast(view, policy, pseed)
    else:
        want = P.pack_optimized(view, policy, pseed)
    assert len(got) == len(want)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g.row_ids, w.row_ids)
        np.testing.assert_array_equal(g.col_ids, np.asarray(w.col_ids))
        np.testing.assert_array_equal(g.values, w.values)
        assert g.legal_24 == w.legal


def test_cpp_fp16_compression_matches_numpy(tmp_path):
    """Round-to-nearest-even FP64->FP16 incl. ties, subnormals and overflow (compress_tile)."""
    rng = np.random.default_rng(3)
    special = np.array([2.0 ** -25, 2.0 ** -24 * 1.5, 2.0 ** -24 * 2.5, 65504.0, 65519.9, 6.1e-5,
                        1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, -0.0, 3.0e-8, 1e-30, 0.33325195])
    vals = np.concatenate([special, rng.standard_normal(200) * 10.0 ** rng.uniform(-7, 4, 200)])
    rows = len(vals)
    cols = np.zeros(rows, dtype=np.int64)   # one column per row -> one nonzero per row-quartet
    row_ptr = np.arange(rows + 1, dtype=np.int64)
    vals = np.where(vals == 0, 1.0, vals)   # structural zeros are not stored
    out = packing.export_view_dir(row_ptr, cols, vals, tmp_path, output_size=rows, n_cols=1,
                                  policy="trajectory", seed=1, illegal_mode="split24")
    bits = np.fromfile(out / "tile_a_comp.bin", dtype=np.uint16).reshape(-1, 16)[:rows]
    nonzero = (bits & 0x7FFF) != 0
    assert np.all(nonzero.sum(axis=1) <= 1)          # one stored coefficient per row
    got = np.where(nonzero.any(axis=1), bits[np.arange(rows), nonzero.argmax(axis=1)], 0)
    want = vals.astype(np.float16).view(np.uint16)
    want = np.where((want & 0x7FFF) != 0, want, 0)  # a value rounding to +-0 is stored as a zero slot
    np.testing.assert_array_equal(got, want)


def test_cpp_kb_coefficients_match_oracle():
    from trajsparsenufft_b200 import synth
    traj = synth.golden_radial(12, 64)
    got = packing.kb_interpolation_csr(traj, 32, 64, 6)
    want = okb.interpolation_csr(traj, 32, 64, 6)
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])
    np.testing.assert_allclose(got[2], want[2], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(got[3], want[3], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(packing.kb_deapodization(32, 64, 6), okb.deapodization(32, 64, 6), rtol=1e-13)


def test_pair_metadata_decode_is_inverse():
    codes = np.random.default_rng(2).integers(0, 2 ** 32, size=(9, 16), dtype=np.uint64).astype(np.uint32)
    np.testing.assert_array_equal(packing.decode_row_metadata(P.pair_metadata(codes)), codes)


def test_plan_from_pack_rejects_bad_header(tmp_path):
    """Host-side failure injection: bad magic / short file -> FORMAT / IO, no GPU touched."""
    import shutil
    src = GOLDEN / "prod_radial16_opt" / "G" / "real"
    bad = tmp_path / "bad"
    shutil.copytree(src, bad)
    raw = bytearray((bad / "header.bin").read_bytes())
    raw[0] ^= 0xFF
    (bad / "header.bin").write_bytes(bytes(raw))
    from trajsparsenufft_b200.operator import Plan
    with pytest.raises(_lib.TsnError) as e:
        Plan.from_pack(str(bad), None, None, None, im_size=16, grid_size=32, coils=4, width=6)
    assert e.value.kind == "FORMAT"
    short = tmp_path / "short"
    shutil.copytree(src, short)
    data = (short / "tile_a_comp.bin").read_bytes()
    (short / "tile_a_comp.bin").write_bytes(data[:-2])
    with pytest.raises(_lib.TsnError) as e:
        Plan.from_pack(str(short), None, None, None, im_size=16, grid_size=32, coils=4, width=6)
    assert e.value.kind == "IO"
    # mismatched real/imag structure (load_direction, nufft_integrated_bench.cu:187-194)
    other = tmp_path / "other"
    shutil.copytree(GOLDEN / "prod_radial16_fast" / "G" / "imag", other)
    with pytest.raises(_lib.TsnError) as e:
        Plan.from_pack(str(src), str(other), None, None, im_size=16, grid_size=32, coils=4, width=6)
    assert e.value.kind == "FORMAT"
