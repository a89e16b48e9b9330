// Pack-once planner: sparse views, row grouping, 2:4 tile packing, split24/CSR residual,
// FP16 compression and the packed_header_v2 component arrays.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "common.hpp"

namespace tsn {

constexpr int kMTile = 16;
constexpr int kKTile = 32;
constexpr uint64_t kPackMagic = 0x4E55464654323431ull;  // "NUFFT241"
constexpr uint32_t kPackVersion = 2;
constexpr uint32_t kPackChannels = 16;

// CSR over active rows with the logical output row of each (SparseRows,
// src/nufft_layout_oracle.py:34-52).
struct SparseView {
  std::vector<int64_t> row_ids;
  std::vector<int64_t> row_ptr;  // rows + 1
  std::vector<int64_t> cols;
  std::vector<double> vals;
  std::vector<double> coords;  // [rows][dims] (morton keys)
  int dims = 2;
  int64_t output_size = 0;
  int64_t n_cols = 0;
  int64_t rows() const { return static_cast<int64_t>(row_ptr.size()) - 1; }
  int64_t nnz() const { return row_ptr.empty() ? 0 : row_ptr.back(); }
};

// Active-row transpose with grid-cell coordinates (transpose_sparse, :209-231). A 3D view
// (dims 3, cells (q0 G + q1) G + q2) gets coordinates (q2, q1, q0).
SparseView transpose_view(const SparseView& v, int64_t grid_size);

struct PackTile {
  int32_t row_ids[kMTile];
  std::vector<int32_t> col_ids;  // k_tile entries, -1 pads
  std::vector<double> values;    // [16][k_tile]
  bool legal = true;
  int32_t violation = 0;
};

std::vector<int64_t> row_order(const SparseView& v, int policy, int k_tile);

// pack_view / fast_split24_pack / optimized_split24_pack. Fast and optimized split illegal
// tiles themselves (as the reference does); search keeps illegal tiles.
std::vector<PackTile> pack_view(const SparseView& v, int planner, int policy, int k_tile,
                                uint64_t seed, int threads);
// The tiles of row groups [g0, g1) of a row order, in group order (pack_view is row_order
// followed by this over every group); lets large views be packed and compressed in batches.
// With the optimized planner and fast_above > 0, a group whose column union is larger than
// fast_above is packed the fast way (sorted union in K32 runs, split24): the optimized
// search grows faster than linearly in the union, and the grid cells next to the centre of
// a 3D radial trajectory have unions of tens of thousands of samples.
std::vector<PackTile> pack_groups(const SparseView& v, const std::vector<int64_t>& order, int64_t g0,
                                  int64_t g1, int planner, int k_tile, uint64_t seed, int threads,
                                  int64_t fast_above);

struct GroupedTiles {
  std::vector<uint32_t> group_offsets;
  std::vector<int32_t> group_row_ids;  // [groups][16]
  std::vector<PackTile> tiles;         // all legal
  std::vector<uint32_t> residual_row_ptr;
  std::vector<int32_t> residual_cols;
  std::vector<uint16_t> residual_vals;  // f16 bits
};
// split_legal_tiles_and_residual (src/export_gpu_case.py:110-155).
GroupedTiles split_legal_and_residual(const SparseView& v, const std::vector<PackTile>& tiles,
                                      int illegal_mode);
bool legal_24(const PackTile& t, int* violations = nullptr);

// Component values on the shared structure (materialize_component_tiles,
// src/export_torchkbnufft_gpu_case.py:356-384).
std::vector<PackTile> component_tiles(const std::vector<PackTile>& structure,
                                      const SparseView& component);

struct CompressedTiles {
  std::vector<uint16_t> values;    // [tiles][16][16] f16 bits
  std::vector<uint32_t> row_meta;  // [tiles][16] 4-bit codes, 8 quartets
  std::vector<uint32_t> pair_meta; // [tiles][16] mma.sp register pairing
  std::vector<int32_t> col_ids;    // [tiles][32], -1 -> 0
};
// compress_tile / compress_tiles_vectorized + pair_metadata (src/export_gpu_case.py:41-74).
CompressedTiles compress_tiles(const std::vector<PackTile>& tiles);
uint32_t pair_word(const uint32_t* row_meta16, int word);

struct PackHeader {
  uint64_t magic;
  uint32_t version, n_channels, output_size, n_cols, active_rows, nnz, groups, tiles,
      residual_nnz, m_tile, k_tile;
};
static_assert(sizeof(PackHeader) == 56 || sizeof(PackHeader) == 52, "header layout");
std::string header_bytes(uint32_t output_size, uint32_t n_cols, uint32_t active_rows,
                         uint32_t nnz, uint32_t groups, uint32_t tiles, uint32_t residual_nnz);
PackHeader parse_header(const std::string& bytes);

int resolve_threads(int threads);

}  // namespace tsn
