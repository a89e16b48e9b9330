// packed_header_v2 directory format (src/export_gpu_case.py:242-321,
// src/export_torchkbnufft_gpu_case.py:407-488) and its reader
// (read_header/read_array/load_direction, nufft_spmma_bench.cu:61-98,
// nufft_integrated_bench.cu:135-226).
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "planner.hpp"

namespace tsn {

std::string sha256_hex(const void* data, size_t n);

struct PackArrays {
  PackHeader h{};
  std::vector<uint32_t> group_offsets;  // groups+1
  std::vector<int32_t> group_row_ids;   // groups*16
  std::vector<int32_t> tile_col_ids;    // tiles*32
  std::vector<uint16_t> tile_a_comp;    // tiles*16*16 f16 bits
  std::vector<uint32_t> tile_pair_meta; // tiles*16
};

// One file entry of manifest.json.
struct FileEntry {
  std::string file, dtype;
  std::vector<int64_t> shape;
  int64_t bytes = 0;
  std::string sha256;
};

void make_dirs(const std::string& path);
FileEntry write_file(const std::string& dir, const std::string& name, const void* data, size_t bytes,
                     const std::string& dtype, std::vector<int64_t> shape);
void write_manifest(const std::string& dir, const std::vector<std::pair<std::string, std::string>>& fields,
                    const std::vector<FileEntry>& files);
std::string read_file(const std::string& path);
PackArrays read_pack_dir(const std::string& dir);

}  // namespace tsn
