// Host-side C ABI: error strings, KB coefficients, pack-once export entry points.
#include <chrono>
#include <cmath>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "kb.hpp"
#include "pack_io.hpp"
#include "planner.hpp"

namespace tsn {

static thread_local std::string g_last_error;

void set_last_error(const std::string& text) { g_last_error = text; }

tsn_status guard_status(const std::exception& e) {
  set_last_error(e.what());
  if (const auto* te = dynamic_cast<const Error*>(&e)) return te->status;
  if (dynamic_cast<const std::bad_alloc*>(&e)) return TSN_ERR_NOMEM;
  return TSN_ERR_ARG;
}

SparseView sample_view(const std::vector<int64_t>& row_ptr, const std::vector<int64_t>& cols,
                       const std::vector<double>& vals, const float* traj, int64_t m, int64_t g);

static SparseView csr_view(const int64_t* row_ptr, const int64_t* cols, const double* vals,
                           const int64_t* row_ids, const double* coords, int64_t rows, int64_t output_size,
                           int64_t n_cols) {
  if (!row_ptr || (!cols && row_ptr[rows] > 0) || rows < 0) fail(TSN_ERR_ARG, "invalid CSR arguments");
  SparseView v;
  v.output_size = output_size;
  v.n_cols = n_cols;
  v.row_ptr.assign(row_ptr, row_ptr + rows + 1);
  const int64_t nnz = v.row_ptr.back();
  if (v.row_ptr.front() != 0) fail(TSN_ERR_ARG, "row_ptr[0] must be 0");
  for (int64_t r = 0; r < rows; ++r)
    if (v.row_ptr[r] > v.row_ptr[r + 1]) fail(TSN_ERR_ARG, "row_ptr is not monotone");
  v.cols.assign(cols, cols + nnz);
  for (int64_t c : v.cols)
    if (c < 0 || c >= n_cols) fail(TSN_ERR_SHAPE, "column id out of range");
  if (vals) v.vals.assign(vals, vals + nnz);
  else v.vals.assign(nnz, 1.0);
  v.row_ids.resize(rows);
  for (int64_t r = 0; r < rows; ++r) {
    v.row_ids[r] = row_ids ? row_ids[r] : r;
    if (v.row_ids[r] < 0 || v.row_ids[r] >= output_size) fail(TSN_ERR_SHAPE, "row id out of range");
  }
  v.coords.assign(2 * rows, 0.0);
  if (coords) std::memcpy(v.coords.data(), coords, sizeof(double) * 2 * rows);
  return v;
}

static std::string jnum(double v) {
  std::ostringstream o;
  o.precision(17);
  o << v;
  return o.str();
}
static std::string jstr(const std::string& s) { return "\"" + s + "\""; }

static const char* planner_name(int p) {
  return p == TSN_PLANNER_OPTIMIZED ? "optimized" : p == TSN_PLANNER_FAST ? "fast" : "search";
}
static const char* policy_name(int p) {
  return p == TSN_POLICY_TRAJECTORY ? "trajectory" : p == TSN_POLICY_MORTON ? "morton"
         : p == TSN_POLICY_OVERLAP ? "overlap" : "packing256";
}

// One production component directory (export_component, src/export_torchkbnufft_gpu_case.py:387-489,
// production_only arrays).
static void write_component_dir(const std::string& dir, const std::string& comp_name, const SparseView& comp,
                                const GroupedTiles& gt, const std::vector<std::pair<std::string, std::string>>& common,
                                double seconds) {
  const auto t0 = std::chrono::steady_clock::now();
  const CompressedTiles ct = compress_tiles(component_tiles(gt.tiles, comp));
  make_dirs(dir);
  const uint32_t groups = static_cast<uint32_t>(gt.group_offsets.size() - 1);
  const uint32_t tiles = static_cast<uint32_t>(gt.tiles.size());
  const std::string header = header_bytes(static_cast<uint32_t>(comp.output_size), static_cast<uint32_t>(comp.n_cols),
                                          static_cast<uint32_t>(comp.rows()), static_cast<uint32_t>(comp.nnz()), groups,
                                          tiles, 0);
  std::vector<FileEntry> files;
  files.push_back(write_file(dir, "header.bin", header.data(), header.size(), "packed_header_v2", {1}));
  files.push_back(write_file(dir, "group_offsets.bin", gt.group_offsets.data(), gt.group_offsets.size() * 4, "uint32",
                             {static_cast<int64_t>(gt.group_offsets.size())}));
  files.push_back(write_file(dir, "group_row_ids.bin", gt.group_row_ids.data(), gt.group_row_ids.size() * 4, "int32",
                             {static_cast<int64_t>(groups), kMTile}));
  files.push_back(write_file(dir, "tile_col_ids.bin", ct.col_ids.data(), ct.col_ids.size() * 4, "int32",
                             {static_cast<int64_t>(tiles), kKTile}));
  files.push_back(write_file(dir, "tile_a_comp.bin", ct.values.data(), ct.values.size() * 2, "float16",
                             {static_cast<int64_t>(tiles), kMTile, kKTile / 2}));
  files.push_back(write_file(dir, "tile_pair_meta.bin", ct.pair_meta.data(), ct.pair_meta.size() * 4, "uint32",
                             {static_cast<int64_t>(tiles), kMTile}));
  int64_t nonzero = 0;
  for (double v : comp.vals) nonzero += f16_bits_nonzero(f64_to_f16_bits(v));
  const double slots = static_cast<double>(tiles) * kMTile * kKTile / 2;
  auto fields = common;
  fields.emplace_back("component", jstr(comp_name));
  fields.emplace_back("output_size", std::to_string(comp.output_size));
  fields.emplace_back("logical_k", std::to_string(comp.n_cols));
  fields.emplace_back("active_rows", std::to_string(comp.rows()));
  fields.emplace_back("nnz_structural", std::to_string(comp.nnz()));
  fields.emplace_back("nnz_nonzero_fp16", std::to_string(nonzero));
  fields.emplace_back("groups", std::to_string(groups));
  fields.emplace_back("tiles", std::to_string(tiles));
  fields.emplace_back("sparse_value_slots", std::to_string(static_cast<int64_t>(slots)));
  fields.emplace_back("fp16_useful_slot_utilization", jnum(slots > 0 ? nonzero / slots : 0.0));
  fields.emplace_back("shared_structure_pack_seconds", jnum(seconds));
  fields.emplace_back("component_export_seconds",
                      jnum(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()));
  fields.emplace_back("production_only", "true");
  write_manifest(dir, fields, files);
}

}  // namespace tsn

using namespace tsn;

extern "C" {

const char* tsn_version(void) { return "trajsparsenufft-b200 0.1.0 (sm_100a)"; }

const char* tsn_get_last_error_string(void) { return g_last_error.c_str(); }

tsn_status tsn_plan_desc_default(tsn_plan_desc* d) {
  if (!d) return TSN_ERR_ARG;
  std::memset(d, 0, sizeof *d);
  d->im_size = 256;
  d->grid_size = 512;
  d->coils = 8;
  d->kernel_width = 6;
  d->planner = TSN_PLANNER_OPTIMIZED;
  d->policy = TSN_POLICY_MORTON;
  d->seed = 20260823u;
  d->threads = 0;
  d->flags = 0;
  d->interp = TSN_INTERP_AUTO;
  return TSN_OK;
}

tsn_status tsn_kb_interpolation_csr(const float* traj, int64_t m, int32_t im_size, int32_t grid_size, int32_t width,
                                    int64_t* row_ptr, int64_t* cols, double* re, double* im, int64_t* nnz) {
  try {
    if (!traj || !nnz) fail(TSN_ERR_ARG, "NULL argument");
    const KbCsr kb = kb_interpolation_csr(traj, m, im_size, grid_size, width);
    const int64_t n = static_cast<int64_t>(kb.cols.size());
    if (cols) {
      if (*nnz < n) fail(TSN_ERR_ARG, "output arrays too small");
      if (!row_ptr || !re || !im) fail(TSN_ERR_ARG, "NULL output array");
      std::memcpy(row_ptr, kb.row_ptr.data(), sizeof(int64_t) * kb.row_ptr.size());
      std::memcpy(cols, kb.cols.data(), sizeof(int64_t) * n);
      std::memcpy(re, kb.re.data(), sizeof(double) * n);
      std::memcpy(im, kb.im.data(), sizeof(double) * n);
    }
    *nnz = n;
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_kb_weights_csr3(const float* traj, int64_t m, int32_t im_size, int32_t grid_size, int32_t width,
                               int64_t* row_ptr, int64_t* cols, double* w, int64_t* nnz) {
  try {
    if (!traj || !nnz) fail(TSN_ERR_ARG, "NULL argument");
    const KbCsr kb = kb_weights_csr3(traj, m, im_size, grid_size, width, 0);
    const int64_t n = static_cast<int64_t>(kb.cols.size());
    if (cols) {
      if (*nnz < n) fail(TSN_ERR_ARG, "output arrays too small");
      if (!row_ptr || !w) fail(TSN_ERR_ARG, "NULL output array");
      std::memcpy(row_ptr, kb.row_ptr.data(), sizeof(int64_t) * kb.row_ptr.size());
      std::memcpy(cols, kb.cols.data(), sizeof(int64_t) * n);
      std::memcpy(w, kb.re.data(), sizeof(double) * n);
    }
    *nnz = n;
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_kb_deapodization3(int32_t im_size, int32_t grid_size, int32_t width, double* out) {
  try {
    if (!out || im_size <= 0 || grid_size < im_size || width <= 0) fail(TSN_ERR_ARG, "invalid argument");
    const auto d = deapodization3(im_size, grid_size, width);
    std::memcpy(out, d.data(), sizeof(double) * d.size());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_kb_deapodization(int32_t im_size, int32_t grid_size, int32_t width, double* out) {
  try {
    if (!out || im_size <= 0 || grid_size < im_size || width <= 0) fail(TSN_ERR_ARG, "invalid argument");
    const auto d = deapodization(im_size, grid_size, width);
    std::memcpy(out, d.data(), sizeof(double) * d.size());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_pack_csr_to_dirs(const int64_t* row_ptr, const int64_t* cols, const double* re, const double* im,
                                int64_t rows, int32_t grid_size, const float* traj, int32_t view, int32_t planner,
                                int32_t policy, uint64_t seed, int32_t threads, const char* out_dir) {
  try {
    if (!row_ptr || !cols || !re || !im || !traj || !out_dir) fail(TSN_ERR_ARG, "NULL argument");
    if (view != TSN_VIEW_G && view != TSN_VIEW_GT) fail(TSN_ERR_ARG, "unknown view");
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t g = grid_size;
    std::vector<int64_t> rp(row_ptr, row_ptr + rows + 1), cl(cols, cols + row_ptr[rows]);
    std::vector<double> ones(cl.size(), 1.0), vr(re, re + cl.size()), vi(im, im + cl.size());
    for (int64_t c : cl)
      if (c < 0 || c >= g * g) fail(TSN_ERR_SHAPE, "column id out of range");
    SparseView st = sample_view(rp, cl, ones, traj, rows, g);
    SparseView cr = sample_view(rp, cl, vr, traj, rows, g);
    SparseView ci = sample_view(rp, cl, vi, traj, rows, g);
    if (view == TSN_VIEW_GT) {
      st = transpose_view(st, g);
      cr = transpose_view(cr, g);
      ci = transpose_view(ci, g);
    }
    const auto packed = pack_view(st, planner, policy, kKTile, seed, threads);
    const GroupedTiles gt = split_legal_and_residual(st, packed, TSN_ILLEGAL_SPLIT24);
    if (!gt.residual_cols.empty()) fail(TSN_ERR_FORMAT, "split24 structure export left residual entries");
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::vector<std::pair<std::string, std::string>> common = {
        {"experiment_id", jstr("trajsparsenufft_b200_export")},
        {"source", jstr("trajsparsenufft_b200 KB planner")},
        {"view", jstr(view == TSN_VIEW_G ? "G" : "G_T")},
        {"grid_size", std::to_string(grid_size)},
        {"samples", std::to_string(rows)},
        {"planner", jstr(planner_name(planner))},
        {"policy", jstr(policy_name(policy))},
        {"illegal_mode", jstr("split24")},
        {"seed", std::to_string(seed)},
        {"n_channels", std::to_string(kPackChannels)},
        {"m_tile", std::to_string(kMTile)},
        {"k_tile", std::to_string(kKTile)},
    };
    write_component_dir(std::string(out_dir) + "/real", "real", cr, gt, common, secs);
    write_component_dir(std::string(out_dir) + "/imag", "imag", ci, gt, common, secs);
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_pack_view_tiles(const int64_t* row_ptr, const int64_t* cols, const double* vals,
                               const int64_t* logical_row_ids, const double* coords, int64_t rows, int64_t output_size,
                               int64_t n_cols, int32_t planner, int32_t policy, int32_t k_tile, uint64_t seed,
                               int32_t threads, int64_t* tile_count, int32_t* row_ids, int32_t* col_ids, double* values,
                               uint8_t* legal) {
  try {
    if (!tile_count) fail(TSN_ERR_ARG, "NULL tile_count");
    const SparseView v = csr_view(row_ptr, cols, vals, logical_row_ids, coords, rows, output_size, n_cols);
    const auto tiles = pack_view(v, planner, policy, k_tile, seed, threads);
    const int64_t n = static_cast<int64_t>(tiles.size());
    if (row_ids) {
      if (*tile_count < n) fail(TSN_ERR_ARG, "output arrays too small");
      for (int64_t t = 0; t < n; ++t) {
        std::memcpy(row_ids + t * kMTile, tiles[t].row_ids, sizeof(int32_t) * kMTile);
        if (col_ids) std::memcpy(col_ids + t * k_tile, tiles[t].col_ids.data(), sizeof(int32_t) * k_tile);
        if (values)
          std::memcpy(values + t * kMTile * k_tile, tiles[t].values.data(), sizeof(double) * kMTile * k_tile);
        if (legal) legal[t] = tiles[t].legal ? 1 : 0;
      }
    }
    *tile_count = n;
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_export_view_dir(const int64_t* row_ptr, const int64_t* cols, const double* vals,
                               const int64_t* logical_row_ids, const double* coords, int64_t rows, int64_t output_size,
                               int64_t n_cols, int32_t planner, int32_t policy, uint64_t seed, int32_t illegal_mode,
                               int32_t threads, const char* out_dir) {
  try {
    if (!out_dir) fail(TSN_ERR_ARG, "NULL output directory");
    const SparseView v = csr_view(row_ptr, cols, vals, logical_row_ids, coords, rows, output_size, n_cols);
    const auto tiles = pack_view(v, planner, policy, kKTile, seed, threads);
    const GroupedTiles gt = split_legal_and_residual(v, tiles, illegal_mode);
    if (gt.tiles.empty()) fail(TSN_ERR_FORMAT, "export produced no legal Sparse-MMA tiles");
    const CompressedTiles ct = compress_tiles(gt.tiles);
    const std::string dir(out_dir);
    make_dirs(dir);
    const uint32_t groups = static_cast<uint32_t>(gt.group_offsets.size() - 1);
    const std::string header =
        header_bytes(static_cast<uint32_t>(v.output_size), static_cast<uint32_t>(v.n_cols), static_cast<uint32_t>(v.rows()),
                     static_cast<uint32_t>(v.nnz()), groups, static_cast<uint32_t>(gt.tiles.size()),
                     static_cast<uint32_t>(gt.residual_cols.size()));
    std::vector<FileEntry> files;
    files.push_back(write_file(dir, "header.bin", header.data(), header.size(), "packed_header_v2", {1}));
    files.push_back(write_file(dir, "group_offsets.bin", gt.group_offsets.data(), gt.group_offsets.size() * 4, "uint32",
                               {static_cast<int64_t>(gt.group_offsets.size())}));
    files.push_back(write_file(dir, "group_row_ids.bin", gt.group_row_ids.data(), gt.group_row_ids.size() * 4, "int32",
                               {static_cast<int64_t>(groups), kMTile}));
    files.push_back(write_file(dir, "tile_col_ids.bin", ct.col_ids.data(), ct.col_ids.size() * 4, "int32",
                               {static_cast<int64_t>(gt.tiles.size()), kKTile}));
    files.push_back(write_file(dir, "tile_a_comp.bin", ct.values.data(), ct.values.size() * 2, "float16",
                               {static_cast<int64_t>(gt.tiles.size()), kMTile, kKTile / 2}));
    files.push_back(write_file(dir, "tile_pair_meta.bin", ct.pair_meta.data(), ct.pair_meta.size() * 4, "uint32",
                               {static_cast<int64_t>(gt.tiles.size()), kMTile}));
    files.push_back(write_file(dir, "residual_row_ptr.bin", gt.residual_row_ptr.data(), gt.residual_row_ptr.size() * 4,
                               "uint32", {static_cast<int64_t>(gt.residual_row_ptr.size())}));
    files.push_back(write_file(dir, "residual_cols.bin", gt.residual_cols.data(), gt.residual_cols.size() * 4, "int32",
                               {static_cast<int64_t>(gt.residual_cols.size())}));
    files.push_back(write_file(dir, "residual_vals.bin", gt.residual_vals.data(), gt.residual_vals.size() * 2,
                               "float16", {static_cast<int64_t>(gt.residual_vals.size())}));
    write_manifest(dir,
                   {{"experiment_id", jstr("trajsparsenufft_b200_export")},
                    {"illegal_mode", jstr(illegal_mode == TSN_ILLEGAL_SPLIT24 ? "split24" : "csr_residual")},
                    {"output_size", std::to_string(v.output_size)},
                    {"logical_k", std::to_string(v.n_cols)},
                    {"active_rows", std::to_string(v.rows())},
                    {"groups", std::to_string(groups)},
                    {"tiles_legal", std::to_string(gt.tiles.size())},
                    {"residual_nnz_fp64", std::to_string(gt.residual_cols.size())}},
                   files);
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

}  // extern "C"
