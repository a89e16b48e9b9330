// Plans (device-resident packs + workspaces) and the device-side C ABI:
// tsn_plan_create_from_pack / _from_trajectory, tsn_forward, tsn_adjoint, tsn_cg_sense,
// tsn_interp_component. Replaces load_direction + launch_integrated_once + launch_cg of
// experiments/production/src/nufft_integrated_bench.cu:135-226, :604-674 and
// nufft_fp16x2_cg_bench.cu:203-268 with one plan object and one CUDA graph per solve.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <iterator>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "kb.hpp"
#include "kernels.cuh"
#include "pack_io.hpp"
#include "planner.hpp"

using namespace tsn;

#define CUDA_OK(expr)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) fail(TSN_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace tsn {
tsn_status guard_status(const std::exception& e);
}

namespace {

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() {
    if (ptr) cudaFree(ptr);
  }
  void alloc(size_t n) {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = n;
    if (n) CUDA_OK(cudaMalloc(&ptr, n));
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
  template <class T>
  void upload(const std::vector<T>& v) {
    alloc(v.size() * sizeof(T));
    if (!v.empty()) CUDA_OK(cudaMemcpy(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  }
};

// Host image of one view before upload (reference index space).
struct HostView {
  int64_t output_size = 0, n_cols = 0, active_rows = 0, nnz = 0;
  std::vector<uint32_t> group_offsets;
  std::vector<int32_t> group_row_ids;  // reference row ids
  std::vector<int32_t> tile_col_ids;   // reference col ids
  std::vector<std::vector<uint16_t>> a;     // per component [tiles][16][16]
  std::vector<std::vector<uint32_t>> meta;  // per component [tiles][16] pair layout
  int64_t tiles() const { return static_cast<int64_t>(tile_col_ids.size() / kKTile); }
  int64_t groups() const { return static_cast<int64_t>(group_offsets.size()) - 1; }
};

struct DevView {
  DeviceBuffer records, counters, partials, ranges;
  InterpView v;
  // tcgen05 step stream (when the plan runs this view on the tensor-memory kernel)
  DeviceBuffer tc_steps, tc_ranges, tc_counters, tc_partials;
  InterpTcView tc;
  bool use_tc = false;
  // warp runs cut for a 1/share slice of the GPU (batched cases run side by side)
  std::vector<int64_t> item_ends;  // record position after each work item, stream order
  DeviceBuffer ranges_shared;
  InterpView v_shared;
  int share = 0;
  int64_t tiles = 0, groups = 0, active_rows = 0, nnz = 0, output_size = 0, n_cols = 0;
  bool present = false;
};

struct GraphKey {
  const void *y, *smaps, *density, *x;
  int iters;
  uint32_t lam_bits, scale_bits;
  cudaStream_t stream;
  int reliable;       // reliable-update period * 2 + direction
  int ref_period;     // scheduled reference-step period
  uint64_t ref_steps; // explicit reference steps
  bool operator<(const GraphKey& o) const {
    return std::tie(y, smaps, density, x, iters, lam_bits, scale_bits, stream, reliable, ref_period, ref_steps) <
           std::tie(o.y, o.smaps, o.density, o.x, o.iters, o.lam_bits, o.scale_bits, o.stream, o.reliable, o.ref_period,
                    o.ref_steps);
  }
};

// __constant__ twiddle tables are per device: filled once for each device a plan lives on
std::mutex g_const_mutex;
std::vector<int> g_const_devices;

}  // namespace

struct tsn_plan {
  tsn_plan_desc desc{};
  int N = 0, G = 0, C = 0, J = 0, ncomp = 0, shift = 0, rowh = 0;
  bool use_tc = false;    // interpolation on tcgen05.mma.sp (TSN_INTERP_TCGEN05)
  DevView view_ref[2];    // FP32-class views (TSN_FLAG_REFERENCE_STEPS): coefficient high + low parts
  DeviceBuffer tc_error;  // int32, set by a tensor-core launch whose bounded wait gave up
  int dims = 2;  // 2: [N][N] images on a G^2 grid; 3: [N][N][N] volumes on a G^3 grid
  int64_t M = 0;
  DevView view[2];
  DeviceBuffer scaling, tw, z1, z2, panel, spanel, grid, r, p, ap, rhs, parts_pap, parts_rr, norm_parts, state;
  DeviceBuffer adj_parts;  // 5 x 296 FP64 partials of the reverse-mode CG step
  tsn_plan_info info{};
  std::map<GraphKey, cudaGraphExec_t> graphs;
  ~tsn_plan() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  }
};

struct tsn_batch {
  std::vector<tsn_plan*> plans;
  std::vector<int> lane;             // stream of each case
  int streams = 1;
  int device = 0;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  std::map<std::vector<uint64_t>, cudaGraphExec_t> graphs;
  ~tsn_batch() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    for (cudaEvent_t e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    for (cudaStream_t st : side) cudaStreamDestroy(st);
  }
};

namespace {

// reference cell index q0*G + q1 -> internal q1*G + q0
inline int64_t cell_to_internal(int64_t q, int64_t g) { return (q % g) * g + q / g; }
// volume cell (q0*G + q1)*G + q2 -> internal (q2*G + q1)*G + q0 (the row the column FFT
// stage writes: its item q2*G + q1 runs over q0)
inline int64_t cell_to_internal3(int64_t q, int64_t g) {
  const int64_t q0 = q / (g * g), q1 = (q / g) % g, q2 = q % g;
  return (q2 * g + q1) * g + q0;
}
inline int64_t to_internal(const tsn_plan* P, int64_t q) {
  return P->dims == 3 ? cell_to_internal3(q, P->G) : cell_to_internal(q, P->G);
}
// pixels (voxels) of one image and grid cells
inline int64_t image_pixels(const tsn_plan* P) {
  return static_cast<int64_t>(P->N) * P->N * (P->dims == 3 ? P->N : 1);
}
inline int64_t grid_cells(const tsn_plan* P) {
  return static_cast<int64_t>(P->G) * P->G * (P->dims == 3 ? P->G : 1);
}

// Bit j set when column j of tile t has a nonzero coefficient in some row of some
// component.  The others are the planner's padding (stored as column 0 in the pack files)
// or columns whose entries all rounded to zero; the kernel zero-fills them instead of
// gathering, which gives the same products for finite panels and keeps thousands of
// gathers per launch off one panel row.
uint32_t live_columns(const HostView& h, int64_t t) {
  uint32_t m = 0;
  for (size_t c = 0; c < h.a.size(); ++c) {
    const uint32_t* pm = &h.meta[c][t * kMTile];
    const uint16_t* a = &h.a[c][t * kMTile * (kKTile / 2)];
    for (int r = 0; r < kMTile; ++r) {
      // per-row 4-bit codes back from the mma.sp pair layout (rows g and g+8 share words)
      const uint32_t lo = pm[2 * (r & 7)], hi = pm[2 * (r & 7) + 1];
      const uint32_t word = r < 8 ? ((lo & 0xFFFFu) | ((hi & 0xFFFFu) << 16)) : ((lo >> 16) | (hi & 0xFFFF0000u));
      for (int q = 0; q < kKTile / 4; ++q) {
        const uint32_t code = (word >> (4 * q)) & 0xFu;
        if (f16_bits_nonzero(a[r * (kKTile / 2) + 2 * q])) m |= 1u << (4 * q + (code & 3u));
        if (f16_bits_nonzero(a[r * (kKTile / 2) + 2 * q + 1])) m |= 1u << (4 * q + ((code >> 2) & 3u));
      }
    }
  }
  return m;
}

// Persistent-warp runs: contiguous item runs with the smallest possible longest run. A binary
// search finds the least T for which a greedy fill (each run takes items while it stays at or
// under T tiles) needs at most `warps` runs; the runs are that fill. Items are never split, so
// T >= the longest item.
std::vector<int2> cut_ranges(const std::vector<int64_t>& item_ends, int64_t tiles, int warps) {
  warps = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(warps, static_cast<int64_t>(item_ends.size()))));
  auto fill = [&](int64_t cap, std::vector<int2>* out) {
    int64_t runs = 0, start = 0, prev = 0;
    for (size_t i = 0; i < item_ends.size(); ++i) {
      if (item_ends[i] - start > cap) {  // item i starts a new run
        if (out) out->push_back(make_int2(static_cast<int>(start), static_cast<int>(prev)));
        ++runs;
        start = prev;
      }
      prev = item_ends[i];
    }
    if (prev > start) {
      if (out) out->push_back(make_int2(static_cast<int>(start), static_cast<int>(prev)));
      ++runs;
    }
    return runs;
  };
  int64_t longest = 0, prev = 0;
  for (int64_t e : item_ends) {
    longest = std::max(longest, e - prev);
    prev = e;
  }
  int64_t lo = std::max<int64_t>(longest, (tiles + warps - 1) / warps), hi = std::max<int64_t>(lo, tiles);
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (fill(mid, nullptr) <= warps) hi = mid;
    else lo = mid + 1;
  }
  std::vector<int2> ranges;
  fill(lo, &ranges);
  return ranges;
}

constexpr int64_t kLocalityPanelBytes = 64ll << 20;  // about half of the 126 MB L2

int device_sm_count() {
  int dev = 0, sms = 0;
  CUDA_OK(cudaGetDevice(&dev));
  CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return std::max(1, sms);
}

// tcgen05 step stream of one real-pack view (layout in kernels.cuh).  Work items are the
// view's row groups, cut into chunks of at most kTcChunkTiles tiles (longer than the warp
// kernel's: every split chunk publishes its partial sums through a fence and an atomic, which
// here stalls a whole CTA pipeline rather than one warp).  The items, in row-group order, are
// cut into one contiguous run per CTA (one CTA per SM) with balanced tile counts; inside a CTA
// the items go longest first to the slot that frees first (lowest slot on ties), each item's
// tiles on consecutive steps.  Column ids keep the warp records' dead-column marking (-1); A
// is re-laid into the canonical K-major layout and the pair metadata into tensor-memory lane
// order (lane l of a tile holds pair word 2 (l % 8) + l / 8: the lower or upper 16 metadata
// bits of rows l % 8 and l % 8 + 8).
constexpr uint32_t kTcChunkTiles = 32;

void build_tc_steps(tsn_plan* P, DevView& d, const HostView& h, bool rows_are_cells, bool cols_are_cells) {
  const int64_t tiles = h.tiles(), groups = h.groups();
  struct Item {
    int32_t group;
    uint32_t t0, t1;
    int32_t split, first_slot, chunk, nchunks;
  };
  std::vector<Item> items;
  std::vector<int64_t> ends;
  int32_t slots = 0, nsplit = 0;
  int64_t pos = 0;
  for (int64_t g = 0; g < groups; ++g) {
    const uint32_t a = h.group_offsets[g], b = h.group_offsets[g + 1];
    if (a == b) continue;
    const int32_t nch = static_cast<int32_t>((b - a + kTcChunkTiles - 1) / kTcChunkTiles);
    const uint32_t len = (b - a + nch - 1) / nch;  // balanced chunk lengths
    for (int32_t k = 0; k < nch; ++k) {
      const uint32_t t0 = a + k * len, t1 = std::min<uint32_t>(b, a + (k + 1) * len);
      items.push_back(Item{static_cast<int32_t>(g), t0, t1, nch > 1 ? nsplit : -1, slots, k, nch});
      pos += t1 - t0;
      ends.push_back(pos);
    }
    if (nch > 1) {
      slots += nch;
      ++nsplit;
    }
  }
  if (pos != tiles) fail(TSN_ERR_FORMAT, "group offsets do not cover the tiles");
  const int ctas = device_sm_count();
  const std::vector<int2> runs = cut_ranges(ends, tiles, ctas);
  struct Place { size_t item; int32_t slot, step; };
  std::vector<std::vector<Place>> per_cta(runs.size());
  std::vector<int2> cta_steps(runs.size());
  size_t it = 0;
  int64_t total_steps = 0;
  for (size_t c = 0; c < runs.size(); ++c) {
    std::vector<size_t> mine;
    while (it < ends.size() && ends[it] <= runs[c].y) mine.push_back(it++);
    std::stable_sort(mine.begin(), mine.end(), [&](size_t x, size_t y) {
      return items[x].t1 - items[x].t0 > items[y].t1 - items[y].t0;
    });
    int32_t free_at[kTcSlots] = {0};
    for (size_t m : mine) {
      const int slot = static_cast<int>(std::min_element(free_at, free_at + kTcSlots) - free_at);
      per_cta[c].push_back(Place{m, slot, free_at[slot]});
      free_at[slot] += static_cast<int32_t>(items[m].t1 - items[m].t0);
    }
    const int32_t steps = *std::max_element(free_at, free_at + kTcSlots);
    cta_steps[c] = make_int2(static_cast<int>(total_steps), static_cast<int>(total_steps + steps));
    total_steps += steps;
  }
  if (it != ends.size()) fail(TSN_ERR_FORMAT, "tensor-core step schedule lost work items");
  std::vector<uint8_t> steps(static_cast<size_t>(std::max<int64_t>(total_steps, 1)) * kTcStepBytes, 0);
  // idle slots: every column dead (the gathers read nothing), flags 0 (nothing accumulates)
  for (int64_t st = 0; st < total_steps; ++st)
    for (int j = 0; j < kTcSlots; ++j)
      std::memset(steps.data() + st * kTcStepBytes + kTcStepABytes + j * kTcSlotInfoBytes, 0xFF, 128);
  for (size_t c = 0; c < runs.size(); ++c)
    for (const Place& pl : per_cta[c]) {
      const Item& itm = items[pl.item];
      int32_t live_rows = 0;
      uint8_t rows24[48];
      for (int s = 0; s < kMTile; ++s) {
        const int32_t v = h.group_row_ids[static_cast<size_t>(itm.group) * kMTile + s];
        if (v >= 0) live_rows |= static_cast<int32_t>(1u << (kRecLiveShift + s));
        const int64_t row = v < 0 ? kRecRowPad : (rows_are_cells ? to_internal(P, v) : v);
        for (int k = 0; k < 3; ++k) rows24[3 * s + k] = static_cast<uint8_t>((row >> (8 * k)) & 0xFF);
      }
      for (uint32_t t = itm.t0; t < itm.t1; ++t) {
        const int64_t step = cta_steps[c].x + pl.step + (t - itm.t0);
        uint8_t* blk = steps.data() + step * static_cast<int64_t>(kTcStepBytes);
        uint8_t* a = blk + pl.slot * kTcSlotABytes;
        for (int row = 0; row < 16; ++row)
          for (int kc = 0; kc < 16; ++kc)
            std::memcpy(a + (row % 8) * 16 + (row / 8) * 256 + (kc / 8) * 128 + (kc % 8) * 2,
                        &h.a[0][static_cast<size_t>(t) * 256 + row * 16 + kc], 2);
        uint8_t* info = blk + kTcStepABytes + pl.slot * kTcSlotInfoBytes;
        const uint32_t live = live_columns(h, t);
        int32_t cols[kKTile];
        for (int q = 0; q < kKTile; ++q) {
          int64_t col = h.tile_col_ids[static_cast<size_t>(t) * kKTile + q];
          if (cols_are_cells) col = to_internal(P, col);
          cols[q] = ((live >> q) & 1u) ? static_cast<int32_t>(col) : -1;
        }
        std::memcpy(info, cols, sizeof cols);
        uint32_t lanes[16];
        for (int l = 0; l < 16; ++l) lanes[l] = h.meta[0][static_cast<size_t>(t) * 16 + 2 * (l % 8) + l / 8];
        std::memcpy(info + 128, lanes, 64);
        RecordInfo ri;
        ri.flags = live_rows | (t == itm.t0 ? kRecFirst : 0) | (t + 1 == itm.t1 ? kRecLast : 0);
        ri.split = itm.split;
        ri.first_slot = itm.first_slot;
        ri.chunk = itm.chunk | (itm.nchunks << 16);
        std::memcpy(info + 192, &ri, sizeof ri);
        std::memcpy(info + 208, rows24, 48);
      }
    }
  d.tc_counters.upload(std::vector<int32_t>(std::max(nsplit, 1), 0));
  d.tc_partials.alloc(sizeof(float) * static_cast<size_t>(std::max(slots, 1)) * kTcPartialFloats);
  d.tc.counters = d.tc_counters.as<int32_t>();
  d.tc.partials = d.tc_partials.as<float>();
  d.tc_steps.upload(steps);
  d.tc_ranges.upload(cta_steps);
  d.tc.steps = d.tc_steps.as<uint8_t>();
  d.tc.cta_steps = d.tc_ranges.as<int2>();
  d.tc.n_ctas = static_cast<int32_t>(cta_steps.size());
  d.use_tc = true;
}

// Uploads one view into P->view[which], or into `target` (the reference-step views, which
// leave the plan's info and the tensor-core stream alone).
void upload_view(tsn_plan* P, int which, const HostView& h, bool rows_are_cells, bool cols_are_cells,
                 DevView* target = nullptr) {
  DevView& d = target ? *target : P->view[which];
  const int64_t tiles = h.tiles(), groups = h.groups();
  const int ncomp = static_cast<int>(h.a.size());
  const int rec = record_bytes(ncomp);
  if (h.output_size > kMaxInterpRows) fail(TSN_ERR_UNSUPPORTED, "too many output rows for 24-bit record rows");
  // work items: groups of at most kChunkTiles tiles run whole; longer groups are split into
  // at most kMaxChunks chunks (scheduled first, they are the long poles) reduced in chunk
  // order
  struct Item {
    int32_t group;
    uint32_t t0, t1;
    int32_t split, first_slot, chunk, nchunks;
  };
  std::vector<Item> items, small;
  int32_t slots = 0, nsplit = 0;
  for (int64_t g = 0; g < groups; ++g) {
    const uint32_t a = h.group_offsets[g], b = h.group_offsets[g + 1];
    if (a == b) continue;  // no tiles: nothing to stream (grid rows stay zero)
    if (b - a <= static_cast<uint32_t>(kChunkTiles)) {
      small.push_back(Item{static_cast<int32_t>(g), a, b, -1, 0, 0, 1});
      continue;
    }
    const uint32_t len = std::max<uint32_t>(kChunkTiles, (b - a + kMaxChunks - 1) / kMaxChunks);
    const int32_t nch = static_cast<int32_t>((b - a + len - 1) / len);
    for (int32_t k = 0; k < nch; ++k)
      items.push_back(Item{static_cast<int32_t>(g), a + k * len, std::min<uint32_t>(b, a + (k + 1) * len), nsplit,
                           slots, k, nch});
    slots += nch;
    ++nsplit;
  }
  // stream order. When the gathered panel is much larger than L2 (volume grids, large sample
  // sets), the chunks of split groups come first and the whole small groups after them, each
  // list in row-group (Morton) order: consecutive groups share panel rows, and a warp's
  // contiguous run then finds them in L2. Otherwise each chunk of a split group (the long
  // poles, first in their run) is followed by whole small groups up to the average run length,
  // so runs can be cut close to the average instead of at multiples of the chunk length.
  const bool large_panel = h.n_cols * 8 * static_cast<int64_t>(P->C) > kLocalityPanelBytes;
  const int stages = large_panel ? 4 : 3;
  if (large_panel) {
    items.insert(items.end(), small.begin(), small.end());
  } else {
    int64_t total = 0;
    for (const Item& it : items) total += it.t1 - it.t0;
    for (const Item& it : small) total += it.t1 - it.t0;
    const int warps_full = interp_resident_warps(4 * P->C, ncomp, stages);
    const double avg = static_cast<double>(total) / std::max(1, warps_full);
    std::vector<Item> order;
    order.reserve(items.size() + small.size());
    size_t si = 0;
    for (const Item& chunk : items) {
      order.push_back(chunk);
      double run = chunk.t1 - chunk.t0;
      while (si < small.size() && run + 0.5 * (small[si].t1 - small[si].t0) <= avg) {
        run += small[si].t1 - small[si].t0;
        order.push_back(small[si++]);
      }
    }
    order.insert(order.end(), small.begin() + static_cast<std::ptrdiff_t>(si), small.end());
    items.swap(order);
  }
  // persistent warps: contiguous runs of items with about the same number of tiles each;
  // records are stored in that stream order so each warp reads one contiguous range
  std::vector<uint8_t> records(static_cast<size_t>(tiles) * rec, 0);
  d.item_ends.clear();
  int64_t pos = 0;
  for (const Item& it : items) {
    for (uint32_t t = it.t0; t < it.t1; ++t, ++pos) {
      uint8_t* r = records.data() + pos * rec;
      const uint32_t live = live_columns(h, t);
      int32_t cols[kKTile];
      for (int j = 0; j < kKTile; ++j) {
        int64_t c = h.tile_col_ids[t * kKTile + j];
        if (cols_are_cells) c = to_internal(P, c);
        cols[j] = ((live >> j) & 1u) ? static_cast<int32_t>(c) : -1;
      }
      std::memcpy(r, cols, sizeof cols);
      for (int c = 0; c < ncomp; ++c) {
        // A: 16 rows of 32 B; the two 16-B halves of row r are swapped when (r >> 2) & 1 so
        // ldmatrix reads 8 rows of one half without shared-memory bank conflicts
        for (int row = 0; row < 16; ++row)
          for (int half = 0; half < 2; ++half)
            std::memcpy(r + 128 + 576 * c + row * 32 + ((half ^ ((row >> 2) & 1)) * 16),
                        &h.a[c][t * 256 + row * 16 + half * 8], 16);
        std::memcpy(r + 640 + 576 * c, &h.meta[c][t * 16], 64);
      }
      RecordInfo info;
      info.flags = (t == it.t0 ? kRecFirst : 0) | (t + 1 == it.t1 ? kRecLast : 0);
      for (int s = 0; s < kMTile; ++s)
        if (h.group_row_ids[static_cast<size_t>(it.group) * kMTile + s] >= 0)
          info.flags |= static_cast<int32_t>(1u << (kRecLiveShift + s));
      info.split = it.split;
      info.first_slot = it.first_slot;
      info.chunk = it.chunk | (it.nchunks << 16);
      std::memcpy(r + 128 + 576 * ncomp, &info, sizeof info);
      uint8_t* orow = r + 128 + 576 * ncomp + sizeof info;  // 24-bit little-endian rows
      for (int s = 0; s < kMTile; ++s) {
        const int32_t v = h.group_row_ids[static_cast<size_t>(it.group) * kMTile + s];
        const int64_t row = v < 0 ? kRecRowPad : (rows_are_cells ? to_internal(P, v) : v);
        for (int k = 0; k < 3; ++k) orow[3 * s + k] = static_cast<uint8_t>((row >> (8 * k)) & 0xFF);
      }
    }
    d.item_ends.push_back(pos);
  }
  if (pos != tiles) fail(TSN_ERR_FORMAT, "group offsets do not cover the tiles");
  const std::vector<int2> ranges = cut_ranges(d.item_ends, tiles, interp_resident_warps(4 * P->C, ncomp, stages));
  if (P->use_tc && !target) build_tc_steps(P, d, h, rows_are_cells, cols_are_cells);
  d.records.upload(records);
  d.counters.upload(std::vector<int32_t>(std::max(nsplit, 1), 0));
  d.partials.alloc(sizeof(float) * static_cast<size_t>(std::max(slots, 1)) * kPartialFloats * 32);
  d.ranges.upload(ranges);
  d.v.records = d.records.as<uint8_t>();
  d.v.counters = d.counters.as<int32_t>();
  d.v.partials = d.partials.as<float>();
  d.v.warp_ranges = d.ranges.as<int2>();
  d.v.n_warps = static_cast<int32_t>(ranges.size());
  d.v.groups = static_cast<int32_t>(groups);
  d.v.ncomp = ncomp;
  d.v.rec_bytes = rec;
  d.v.stages = stages;
  d.tiles = tiles;
  d.groups = groups;
  d.active_rows = h.active_rows;
  d.nnz = h.nnz;
  d.output_size = h.output_size;
  d.n_cols = h.n_cols;
  d.present = true;
  d.share = 0;
  if (target) return;
  P->info.groups[which] = groups;
  P->info.tiles[which] = tiles;
  P->info.active_rows[which] = h.active_rows;
  P->info.nnz[which] = h.nnz;
  P->info.pack_bytes[which] = static_cast<int64_t>(records.size());
}

void check_desc(const tsn_plan_desc* d) {
  if (!d) fail(TSN_ERR_ARG, "plan descriptor is NULL");
  if (d->dims != 0 && d->dims != 2 && d->dims != 3) fail(TSN_ERR_ARG, "dims must be 2 or 3 (0 = 2)");
  if (d->dims == 3 && static_cast<int64_t>(d->grid_size) * d->grid_size * d->grid_size > kMaxInterpRows)
    fail(TSN_ERR_UNSUPPORTED, "volume grids are limited to 2^24 cells (G <= 256)");
  if (d->im_size <= 0 || d->im_size % 2 || d->grid_size < d->im_size) fail(TSN_ERR_SHAPE, "need an even image size <= grid size");
  if (d->coils < 4 || d->coils > 16 || d->coils % 4) fail(TSN_ERR_UNSUPPORTED, "coil count must be 4, 8, 12 or 16");
  if (d->kernel_width < 1 || d->kernel_width > 16) fail(TSN_ERR_ARG, "kernel width out of range");
  if (d->interp != TSN_INTERP_AUTO && d->interp != TSN_INTERP_MMA_SP && d->interp != TSN_INTERP_TCGEN05)
    fail(TSN_ERR_ARG, "unknown interpolation kernel");
}

// Interpolation kernel of a plan: tcgen05.mma.sp when asked for (real-coefficient pack with 8
// coils only), the warp mma.sp kernel otherwise.
bool choose_tc(const tsn_plan_desc* d, int ncomp, int coils) {
  const bool ok = interp_tc_supported(4 * coils, ncomp);
  if (d->interp == TSN_INTERP_TCGEN05 && !ok)
    fail(TSN_ERR_UNSUPPORTED,
         "the tcgen05 interpolation is built for the real-coefficient pack (centred layout) with 8 coils");
  return d->interp == TSN_INTERP_TCGEN05 && ok;
}

// Error word of the tensor-core views (after allocate_workspaces).
void setup_tc(tsn_plan* P) {
  if (!P->use_tc) return;
  P->tc_error.upload(std::vector<int32_t>(1, 0));
  for (DevView& d : P->view)
    if (d.present && d.use_tc) d.tc.error = P->tc_error.as<int32_t>();
}

// FFT endpoints are built for power-of-two grids of 128..1024 points.
void need_fft(const tsn_plan* P) {
  const int G = P->G;
  if (!fft_grid_supported(G))
    fail(TSN_ERR_UNSUPPORTED, "FFT endpoints need a grid size of 128, 256, 384, 512, 640 or 1024");
  // image rows (and FP32 deapodization rows) are streamed as whole 16-byte chunks
  if (P->N % 4) fail(TSN_ERR_UNSUPPORTED, "FFT endpoints need an image size that is a multiple of 4");
}

// Device arrays the kernels stream with 16-byte copies (images, maps, samples, grids, panels)
// must start on a 16-byte boundary; cudaMalloc and torch allocations always do.
void need_aligned(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs)
    if (p && (reinterpret_cast<uintptr_t>(p) & 15u)) fail(TSN_ERR_ARG, "device arrays must be 16-byte aligned");
}

void allocate_workspaces(tsn_plan* P) {
  const int64_t N = P->N, G = P->G, C = P->C, M = P->M;
  P->rowh = static_cast<int>(4 * C);
  std::vector<float2> tw(G);
  for (int64_t e = 0; e < G; ++e) {
    const double a = -2.0 * M_PI * static_cast<double>(e) / static_cast<double>(G);
    tw[e] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  P->tw.upload(tw);
  const int64_t pix = image_pixels(P), cells = grid_cells(P);
  const int64_t lines = pix / N;  // image lines along the last axis: partials of the row stages
  if (P->dims == 3) {
    P->z1.alloc(sizeof(float2) * N * G * N * C);  // [i0][q2][i1][c] and [q2][i0][i1][c]
    P->z2.alloc(sizeof(float2) * G * G * N * C);  // [q2][q1][i0][c]
  } else {
    P->z1.alloc(sizeof(float2) * G * N * C);
  }
  P->panel.alloc(sizeof(__half) * cells * 4 * C);
  P->spanel.alloc(sizeof(__half) * std::max<int64_t>(M, 1) * 4 * C);
  P->grid.alloc(sizeof(float2) * cells * C);
  CUDA_OK(cudaMemset(P->grid.ptr, 0, P->grid.bytes));  // inactive grid rows stay zero
  P->r.alloc(sizeof(float2) * pix);
  P->p.alloc(sizeof(float2) * pix);
  P->ap.alloc(sizeof(float2) * pix);
  P->rhs.alloc(sizeof(float2) * pix);
  // four sections of one partial per line (pAp, Re r.Ap, Ap.Ap, r.r), plus one slot: stage
  // profiling of volumes writes partials at +1 so the solve's totals in slot 0 stay readable
  P->parts_pap.alloc(sizeof(double) * std::max<int64_t>(4 * lines + 1, kNormParts));
  P->parts_rr.alloc(sizeof(double) * std::max<int64_t>(4 * lines + 1, kNormParts));
  P->norm_parts.alloc(sizeof(double) * kNormParts);
  P->state.alloc(sizeof(CgState));
  CUDA_OK(cudaMemset(P->state.ptr, 0, sizeof(CgState)));
  P->adj_parts.alloc(sizeof(double) * 5 * 296);
  P->info.dims = P->dims;
  P->info.workspace_bytes = static_cast<int64_t>(P->z1.bytes + P->z2.bytes + P->panel.bytes + P->spanel.bytes +
                                                 P->grid.bytes + 4 * P->r.bytes + P->state.bytes);
  {
    std::lock_guard<std::mutex> lock(g_const_mutex);
    int dev = 0;
    CUDA_OK(cudaGetDevice(&dev));
    if (std::find(g_const_devices.begin(), g_const_devices.end(), dev) == g_const_devices.end()) {
      set_twiddle_constants(nullptr);
      g_const_devices.push_back(dev);
    }
  }
  CUDA_OK(cudaGetLastError());
}

FftArgs fft_args(const tsn_plan* P, const void* smaps, int share = 1) {
  FftArgs f;
  f.share = share;
  f.N = P->N;
  f.G = P->G;
  f.C = P->C;
  f.shift = P->shift;
  f.tw = P->tw.as<float2>();
  f.scaling = P->scaling.as<float>();
  f.smaps = static_cast<const float2*>(smaps);
  f.dims = P->dims;
  return f;
}

// Forward FFT chain, image (or coil images) -> grid panel: rows, then (volumes) the middle
// axis, then the first axis into the panel.
void fwd_chain(tsn_plan* P, const FftArgs& f, const float2* x, int mode, float2* p, float2* r,
               const double* parts, int nparts, CgState* st, int iter, __half* panel, cudaStream_t s,
               float2* xs = nullptr, const float2* ap = nullptr) {
  launch_fwd_rows(f, x, P->z1.as<float2>(), mode, p, r, parts, nparts, st, iter, s, xs, ap);
  if (P->dims == 3) {
    launch_fwd_mid(f, P->z1.as<float2>(), P->z2.as<float2>(), s);
    launch_fwd_cols(f, P->z2.as<float2>(), panel, s);
  } else {
    launch_fwd_cols(f, P->z1.as<float2>(), panel, s);
  }
}

// Inverse FFT chain up to the row stage's input (z1): first axis, then (volumes) the middle.
void inv_to_lines(tsn_plan* P, const FftArgs& f, const float2* grid, cudaStream_t s) {
  if (P->dims == 3) {
    launch_inv_cols(f, grid, P->z2.as<float2>(), s);
    launch_inv_mid(f, P->z2.as<float2>(), P->z1.as<float2>(), s);
  } else {
    launch_inv_cols(f, grid, P->z1.as<float2>(), s);
  }
}

// Partials written per image line are summed once for volumes (N^2 of them would be re-read
// by every CTA of the next stage); returns how many partials the consumer reads. `sections`
// runs of partials, one line count apart, are summed in one launch.
int settle_partials(const tsn_plan* P, double* parts, cudaStream_t s, int sections = 1) {
  if (P->dims != 3) return P->N;
  const int64_t lines = image_pixels(P) / P->N;
  launch_reduce_partials(parts, static_cast<int>(lines), s, sections, lines);
  return 1;
}

HostView host_view_from_dirs(const char* real_dir, const char* imag_dir) {
  const PackArrays re = read_pack_dir(real_dir);
  HostView h;
  h.output_size = re.h.output_size;
  h.n_cols = re.h.n_cols;
  h.active_rows = re.h.active_rows;
  h.nnz = re.h.nnz;
  if (re.h.residual_nnz != 0) fail(TSN_ERR_FORMAT, "incompatible packed direction: residual_nnz != 0");
  h.group_offsets = re.group_offsets;
  h.group_row_ids = re.group_row_ids;
  h.tile_col_ids = re.tile_col_ids;
  h.a.push_back(re.tile_a_comp);
  h.meta.push_back(re.tile_pair_meta);
  if (imag_dir) {
    const PackArrays im = read_pack_dir(imag_dir);
    // same checks as load_direction (nufft_integrated_bench.cu:141-194)
    if (std::memcmp(&re.h, &im.h, sizeof(PackHeader)) != 0)
      fail(TSN_ERR_FORMAT, "incompatible real/imag packed direction (headers differ)");
    if (re.group_offsets != im.group_offsets || re.group_row_ids != im.group_row_ids ||
        re.tile_col_ids != im.tile_col_ids)
      fail(TSN_ERR_FORMAT, "real/imag structures differ");
    h.a.push_back(im.tile_a_comp);
    h.meta.push_back(im.tile_pair_meta);
  }
  return h;
}

HostView host_view_from_tiles(const SparseView& structure, const std::vector<const SparseView*>& comps,
                              const tsn_plan_desc* d) {
  const auto packed = pack_view(structure, d->planner, d->policy, kKTile, d->seed, d->threads);
  const GroupedTiles gt = split_legal_and_residual(structure, packed, TSN_ILLEGAL_SPLIT24);
  HostView h;
  h.output_size = structure.output_size;
  h.n_cols = structure.n_cols;
  h.active_rows = structure.rows();
  h.nnz = structure.nnz();
  h.group_offsets = gt.group_offsets;
  h.group_row_ids = gt.group_row_ids;
  for (const SparseView* comp : comps) {
    const CompressedTiles ct = compress_tiles(component_tiles(gt.tiles, *comp));
    if (h.tile_col_ids.empty()) h.tile_col_ids = ct.col_ids;
    h.a.push_back(ct.values);
    h.meta.push_back(ct.pair_meta);
  }
  return h;
}

// One component view packed and compressed in batches of row groups: the unpacked tiles of
// one batch at a time (a few hundred MB) instead of the whole view, which for a 256^3 grid
// would need tens of GB of host memory. The tiles are those of pack_view (same row order,
// same per-group seeds); the fast and optimized planners emit legal tiles only.
constexpr int64_t kVolumeFastUnion = 2048;  // column union above which a group is packed the fast way
HostView host_view_batched(const SparseView& v, const tsn_plan_desc* d) {
  if (d->planner != TSN_PLANNER_FAST && d->planner != TSN_PLANNER_OPTIMIZED)
    fail(TSN_ERR_UNSUPPORTED, "volume plans use the fast or optimized planner");
  const std::vector<int64_t> order = row_order(v, d->policy, kKTile);
  const int64_t n_groups = (static_cast<int64_t>(order.size()) + kMTile - 1) / kMTile;
  HostView h;
  h.output_size = v.output_size;
  h.n_cols = v.n_cols;
  h.active_rows = v.rows();
  h.nnz = v.nnz();
  h.a.resize(1);
  h.meta.resize(1);
  constexpr int64_t kBatchGroups = 8192;
  int32_t prev[kMTile];
  bool have_prev = false;
  for (int64_t g0 = 0; g0 < n_groups; g0 += kBatchGroups) {
    const int64_t g1 = std::min(n_groups, g0 + kBatchGroups);
    const std::vector<PackTile> tiles =
        pack_groups(v, order, g0, g1, d->planner, kKTile, d->seed, d->threads, kVolumeFastUnion);
    const size_t base = h.tile_col_ids.size() / kKTile;
    for (size_t i = 0; i < tiles.size(); ++i) {
      const PackTile& tl = tiles[i];
      if (!legal_24(tl)) fail(TSN_ERR_FORMAT, "planner emitted an illegal 2:4 tile");
      if (!have_prev || std::memcmp(prev, tl.row_ids, sizeof prev) != 0) {  // a group starts here
        h.group_offsets.push_back(static_cast<uint32_t>(base + i));
        h.group_row_ids.insert(h.group_row_ids.end(), tl.row_ids, tl.row_ids + kMTile);
        std::memcpy(prev, tl.row_ids, sizeof prev);
        have_prev = true;
      }
    }
    const CompressedTiles ct = compress_tiles(tiles);
    if (g0 == 0 && g1 < n_groups) {
      // reserve once from the first batch's tiles per group (+25%): growing by doubling would
      // touch fresh memory again at every step, which dominates planning time on hosts where
      // first touch is slow
      const double per_group = static_cast<double>(tiles.size()) / static_cast<double>(g1 - g0);
      const size_t est = static_cast<size_t>(per_group * static_cast<double>(n_groups) * 1.25) + 1;
      h.tile_col_ids.reserve(est * kKTile);
      h.a[0].reserve(est * kMTile * (kKTile / 2));
      h.meta[0].reserve(est * kMTile);
    }
    h.tile_col_ids.insert(h.tile_col_ids.end(), ct.col_ids.begin(), ct.col_ids.end());
    h.a[0].insert(h.a[0].end(), ct.values.begin(), ct.values.end());
    h.meta[0].insert(h.meta[0].end(), ct.pair_meta.begin(), ct.pair_meta.end());
  }
  h.group_offsets.push_back(static_cast<uint32_t>(h.tile_col_ids.size() / kKTile));
  return h;
}

}  // namespace

namespace tsn {

// numpy.mod(x, g) for float64 (fmod with the sign of the divisor)
double np_mod(double x, double g) {
  double m = std::fmod(x, g);
  if (m != 0.0) {
    if ((g < 0) != (m < 0)) m += g;
  } else {
    m = std::copysign(0.0, g);
  }
  return m;
}

// G-view sparse structure over samples from a KB CSR, with the reference's morton coords
// (np.mod(traj*G + G/2, G), src/export_torchkbnufft_gpu_case.py:550-553).
SparseView sample_view(const std::vector<int64_t>& row_ptr, const std::vector<int64_t>& cols,
                       const std::vector<double>& vals, const float* traj, int64_t m, int64_t g) {
  SparseView v;
  v.output_size = m;
  v.n_cols = g * g;
  v.row_ptr = row_ptr;
  v.cols = cols;
  v.vals = vals;
  v.row_ids.resize(m);
  v.coords.resize(2 * m);
  for (int64_t i = 0; i < m; ++i) {
    v.row_ids[i] = i;
    v.coords[2 * i] = np_mod(static_cast<double>(traj[2 * i]) * g + g / 2.0, static_cast<double>(g));
    v.coords[2 * i + 1] = np_mod(static_cast<double>(traj[2 * i + 1]) * g + g / 2.0, static_cast<double>(g));
  }
  return v;
}

}  // namespace tsn

// ---- C ABI: plans -------------------------------------------------------------------------
extern "C" {

tsn_status tsn_plan_create_from_pack(const char* fwd_real, const char* fwd_imag, const char* adj_real,
                                     const char* adj_imag, const float* scaling, const tsn_plan_desc* desc,
                                     tsn_plan** out) {
  try {
    if (!out) fail(TSN_ERR_ARG, "plan output pointer is NULL");
    *out = nullptr;
    check_desc(desc);
    if (desc->flags & TSN_FLAG_REFERENCE_STEPS)
      fail(TSN_ERR_UNSUPPORTED, "reference steps are built for trajectory plans (centred real-coefficient pack)");
    if (desc->dims == 3) fail(TSN_ERR_UNSUPPORTED, "pack directories hold image (2D) views");
    if (!fwd_real && !adj_real) fail(TSN_ERR_ARG, "at least one view directory is required");
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<tsn_plan> P(new tsn_plan);
    P->desc = *desc;
    P->N = desc->im_size;
    P->G = desc->grid_size;
    P->C = desc->coils;
    P->J = desc->kernel_width;
    P->shift = 0;  // reference layout: image at [0, N)
    const int64_t cells = static_cast<int64_t>(P->G) * P->G;
    HostView hv[2];
    if (fwd_real) {
      hv[0] = host_view_from_dirs(fwd_real, fwd_imag);
      if (hv[0].n_cols != cells) fail(TSN_ERR_SHAPE, "forward pack columns != grid_size^2");
      P->M = hv[0].output_size;
    }
    if (adj_real) {
      hv[1] = host_view_from_dirs(adj_real, adj_imag);
      if (hv[1].output_size != cells) fail(TSN_ERR_SHAPE, "adjoint pack rows != grid_size^2");
      if (fwd_real && hv[1].n_cols != P->M) fail(TSN_ERR_SHAPE, "forward output_size != adjoint n_cols");
      P->M = hv[1].n_cols;
    }
    if (fwd_real && adj_real && hv[0].a.size() != hv[1].a.size())
      fail(TSN_ERR_FORMAT, "forward and adjoint packs have different component counts");
    P->ncomp = static_cast<int>((fwd_real ? hv[0] : hv[1]).a.size());
    CUDA_OK(cudaSetDevice(desc->device));  // all host-side checks are done: touch the device now
    std::vector<float> sc(static_cast<size_t>(P->N) * P->N);
    if (scaling) {
      std::memcpy(sc.data(), scaling, sc.size() * sizeof(float));
    } else {
      const auto d = deapodization(P->N, P->G, P->J);
      for (size_t i = 0; i < sc.size(); ++i) sc[i] = static_cast<float>(d[i]);
    }
    P->scaling.upload(sc);
    P->use_tc = choose_tc(desc, P->ncomp, P->C);
    if (fwd_real) upload_view(P.get(), TSN_VIEW_G, hv[0], false, true);
    if (adj_real) upload_view(P.get(), TSN_VIEW_GT, hv[1], true, false);
    allocate_workspaces(P.get());
    setup_tc(P.get());
    P->info.samples = P->M;
    P->info.im_size = P->N;
    P->info.grid_size = P->G;
    P->info.coils = P->C;
    P->info.kernel_width = P->J;
    P->info.components = P->ncomp;
    P->info.interp = P->use_tc ? TSN_INTERP_TCGEN05 : TSN_INTERP_MMA_SP;
    P->info.plan_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = P.release();
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_plan_create_from_trajectory(const float* traj, int64_t m, const tsn_plan_desc* desc, tsn_plan** out) {
  try {
    if (!out || !traj) fail(TSN_ERR_ARG, "NULL argument");
    *out = nullptr;
    check_desc(desc);
    if (m <= 0) fail(TSN_ERR_SHAPE, "trajectory is empty");
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<tsn_plan> P(new tsn_plan);
    P->desc = *desc;
    P->N = desc->im_size;
    P->G = desc->grid_size;
    P->C = desc->coils;
    P->J = desc->kernel_width;
    P->M = m;
    P->dims = desc->dims == 3 ? 3 : 2;
    const bool reference_layout = (desc->flags & TSN_FLAG_REFERENCE_LAYOUT) != 0;
    const bool reference_steps = (desc->flags & TSN_FLAG_REFERENCE_STEPS) != 0;
    if (reference_steps && (reference_layout || P->dims == 3))
      fail(TSN_ERR_UNSUPPORTED, "reference steps are built for 2D plans with the centred real-coefficient pack");
    P->shift = reference_layout ? 0 : P->N / 2;
    for (int64_t i = 0; i < P->dims * m; ++i)
      if (!std::isfinite(traj[i]) || std::fabs(traj[i]) > 0.500001f)
        fail(TSN_ERR_ARG, "trajectory must use normalized [-0.5, 0.5] coordinates");
    if (P->dims == 3) {
      // volume: real KB weights on the centred layout, views packed in batches
      if (reference_layout) fail(TSN_ERR_UNSUPPORTED, "volume plans use the centred layout (real KB weights)");
      if (m > kMaxInterpRows) fail(TSN_ERR_UNSUPPORTED, "a volume plan holds at most 2^24 samples");
      KbCsr kb = kb_weights_csr3(traj, m, P->N, P->G, P->J, desc->threads);
      HostView hv[2];
      {
        SparseView w_g;
        w_g.dims = 3;
        w_g.output_size = m;
        w_g.n_cols = static_cast<int64_t>(P->G) * P->G * P->G;
        w_g.row_ptr = std::move(kb.row_ptr);
        w_g.cols = std::move(kb.cols);
        w_g.vals = std::move(kb.re);
        w_g.row_ids.resize(m);
        w_g.coords.resize(3 * m);
        const double g = P->G;
        for (int64_t i = 0; i < m; ++i) {
          w_g.row_ids[i] = i;
          for (int d = 0; d < 3; ++d) w_g.coords[3 * i + d] = np_mod(static_cast<double>(traj[3 * i + d]) * g + g / 2.0, g);
        }
        hv[0] = host_view_batched(w_g, desc);
        const SparseView w_gt = transpose_view(w_g, P->G);
        w_g = SparseView();
        hv[1] = host_view_batched(w_gt, desc);
      }
      P->ncomp = 1;
      const auto d3 = deapodization3(P->N, P->G, P->J);
      std::vector<float> sc(d3.size());
      for (size_t i = 0; i < sc.size(); ++i) sc[i] = static_cast<float>(d3[i]);
      CUDA_OK(cudaSetDevice(desc->device));
      P->scaling.upload(sc);
      P->info.plan_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      P->use_tc = choose_tc(desc, P->ncomp, P->C);
      upload_view(P.get(), TSN_VIEW_G, hv[0], false, true);
      hv[0] = HostView();
      upload_view(P.get(), TSN_VIEW_GT, hv[1], true, false);
      hv[1] = HostView();
      allocate_workspaces(P.get());
      setup_tc(P.get());
      P->info.samples = P->M;
      P->info.im_size = P->N;
      P->info.grid_size = P->G;
      P->info.coils = P->C;
      P->info.kernel_width = P->J;
      P->info.components = P->ncomp;
      P->info.interp = P->use_tc ? TSN_INTERP_TCGEN05 : TSN_INTERP_MMA_SP;
      P->info.dims = 3;
      *out = P.release();
      return TSN_OK;
    }
    const KbCsr kb = kb_interpolation_csr(traj, m, P->N, P->G, P->J);
    std::vector<double> ones(kb.cols.size(), 1.0), weights(kb.cols.size());
    for (size_t i = 0; i < weights.size(); ++i) weights[i] = std::hypot(kb.re[i], kb.im[i]);
    const SparseView st_g = sample_view(kb.row_ptr, kb.cols, ones, traj, m, P->G);
    const SparseView st_gt = transpose_view(st_g, P->G);
    HostView hv[2], hv_ref[2];
    if (reference_layout) {
      const SparseView re_g = sample_view(kb.row_ptr, kb.cols, kb.re, traj, m, P->G);
      const SparseView im_g = sample_view(kb.row_ptr, kb.cols, kb.im, traj, m, P->G);
      const SparseView re_gt = transpose_view(re_g, P->G), im_gt = transpose_view(im_g, P->G);
      hv[0] = host_view_from_tiles(st_g, {&re_g, &im_g}, desc);
      hv[1] = host_view_from_tiles(st_gt, {&re_gt, &im_gt}, desc);
      P->ncomp = 2;
    } else if (reference_steps) {
      // centred real pack plus its FP32-class twin: every weight as FP16 high part + FP16
      // residual on the same tiles (one planner pass serves both)
      const SparseView w_g = sample_view(kb.row_ptr, kb.cols, weights, traj, m, P->G);
      std::vector<double> lows(weights.size());
      for (size_t i = 0; i < lows.size(); ++i) lows[i] = weights[i] - f16_bits_to_f64(f64_to_f16_bits(weights[i]));
      const SparseView l_g = sample_view(kb.row_ptr, kb.cols, lows, traj, m, P->G);
      const SparseView w_gt = transpose_view(w_g, P->G), l_gt = transpose_view(l_g, P->G);
      hv_ref[0] = host_view_from_tiles(st_g, {&w_g, &l_g}, desc);
      hv_ref[1] = host_view_from_tiles(st_gt, {&w_gt, &l_gt}, desc);
      for (int v = 0; v < 2; ++v) {
        hv[v] = hv_ref[v];
        hv[v].a.resize(1);
        hv[v].meta.resize(1);
      }
      P->ncomp = 1;
    } else {
      // centred image: the phase exp(2 pi i q c/G) moves into the FFT shift, coefficients are
      // the real KB weights
      const SparseView w_g = sample_view(kb.row_ptr, kb.cols, weights, traj, m, P->G);
      const SparseView w_gt = transpose_view(w_g, P->G);
      hv[0] = host_view_from_tiles(st_g, {&w_g}, desc);
      hv[1] = host_view_from_tiles(st_gt, {&w_gt}, desc);
      P->ncomp = 1;
    }
    const auto d = deapodization(P->N, P->G, P->J);
    std::vector<float> sc(d.size());
    for (size_t i = 0; i < sc.size(); ++i) sc[i] = static_cast<float>(d[i]);
    CUDA_OK(cudaSetDevice(desc->device));
    P->scaling.upload(sc);
    P->info.plan_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    P->use_tc = choose_tc(desc, P->ncomp, P->C);
    upload_view(P.get(), TSN_VIEW_G, hv[0], false, true);
    upload_view(P.get(), TSN_VIEW_GT, hv[1], true, false);
    if (reference_steps) {
      upload_view(P.get(), TSN_VIEW_G, hv_ref[0], false, true, &P->view_ref[TSN_VIEW_G]);
      upload_view(P.get(), TSN_VIEW_GT, hv_ref[1], true, false, &P->view_ref[TSN_VIEW_GT]);
      for (DevView& d : P->view_ref) d.v.sum_components = 1;
    }
    allocate_workspaces(P.get());
    setup_tc(P.get());
    P->info.samples = P->M;
    P->info.im_size = P->N;
    P->info.grid_size = P->G;
    P->info.coils = P->C;
    P->info.kernel_width = P->J;
    P->info.components = P->ncomp;
    P->info.interp = P->use_tc ? TSN_INTERP_TCGEN05 : TSN_INTERP_MMA_SP;
    P->info.dims = 2;
    *out = P.release();
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_plan_destroy(tsn_plan* plan) {
  if (plan) cudaSetDevice(plan->desc.device);
  delete plan;
  return TSN_OK;
}

tsn_status tsn_plan_get_info(const tsn_plan* plan, tsn_plan_info* info) {
  if (!plan || !info) {
    set_last_error("NULL argument");
    return TSN_ERR_ARG;
  }
  *info = plan->info;
  info->device_error = 0;
  if (plan->use_tc && plan->tc_error.ptr) {
    cudaSetDevice(plan->desc.device);
    int32_t err = 0;
    if (cudaMemcpy(&err, plan->tc_error.ptr, sizeof err, cudaMemcpyDeviceToHost) == cudaSuccess) info->device_error = err;
  }
  return TSN_OK;
}

}  // extern "C"

// ---- operators ----------------------------------------------------------------------------
namespace {

void need_views(const tsn_plan* P, bool fwd, bool adj) {
  need_fft(P);
  CUDA_OK(cudaSetDevice(P->desc.device));
  if ((fwd && !P->view[TSN_VIEW_G].present) || (adj && !P->view[TSN_VIEW_GT].present))
    fail(TSN_ERR_ARG, "plan lacks the pack view this operator needs");
}

// One interpolation launch of a view: the tensor-core kernel when the plan uses it, else the
// warp mma.sp kernel (on a 1/share slice of the GPU for batched cases); `reference` selects the
// FP32-class views of the CG's reference steps.  The tensor-core
// kernel always runs its one-CTA-per-SM schedule; batched cases then share SMs as they free.
void run_interp(const tsn_plan* P, int which, int share, int epi, const InterpOut& o, cudaStream_t s,
                bool reference = false) {
  const __half* panel = which == TSN_VIEW_G ? P->panel.as<__half>() : P->spanel.as<__half>();
  if (reference) {  // FP32-class views: warp kernel summing the coefficients' high and low parts
    launch_interp(P->view_ref[which].v, panel, P->rowh, true, epi, false, o, s);
    return;
  }
  const DevView& d = P->view[which];
  if (d.use_tc) {
    launch_interp_tc(d.tc, panel, epi, o, s);
    return;
  }
  const InterpView& v = share > 1 ? d.v_shared : d.v;
  launch_interp(v, panel, P->rowh, true, epi, which == TSN_VIEW_GT, o, s);
}

void enqueue_forward(tsn_plan* P, const void* x, const void* smaps, void* y, cudaStream_t s, bool reference = false) {
  const FftArgs f = fft_args(P, smaps);
  CgState* st = P->state.as<CgState>();
  const int64_t n = image_pixels(P) * (smaps ? 1 : P->C);
  launch_norm_partials(static_cast<const float2*>(x), n, P->norm_parts.as<double>(), s);
  fwd_chain(P, f, static_cast<const float2*>(x), 0, nullptr, nullptr, P->norm_parts.as<double>(), kNormParts, st, 0,
            P->panel.as<__half>(), s);
  InterpOut o;
  o.c64 = static_cast<float2*>(y);
  o.rows = P->M;
  o.coils = P->C;
  o.scale_ptr = &st->sigma_x;
  o.scale_inv = 1;
  o.scale_mul = f.gs();
  run_interp(P, TSN_VIEW_G, 1, EPI_SAMPLES, o, s, reference);
}

// q = A^H W A p + lambda p through the plan's operator (the CG's normal operator at operator
// scale 1), with the optional coil images A_c^H W A p before the coil combine and the optional
// FP64 Re <p, q>: the plain forward's panel scale, both interpolations, the inverse FFTs and
// the combine epilogue (inv_rows mode 5).
static_assert(kCgStepParts == TSN_CG_STEP_PARTS, "CG-step partial count of the kernels and the header");

void enqueue_normal(tsn_plan* P, const void* p, const void* smaps, const float* density, float lambda, void* q,
                    void* coils, double* pq, const double* p_parts, int n_p_parts, cudaStream_t s) {
  const FftArgs f = fft_args(P, smaps);
  CgState* st = P->state.as<CgState>();
  const float2* pv = static_cast<const float2*>(p);
  if (!p_parts) {  // the panel scale of p from |p|^2 partials, unless the caller has them
    launch_norm_partials(pv, image_pixels(P), P->norm_parts.as<double>(), s);
    p_parts = P->norm_parts.as<double>();
    n_p_parts = kNormParts;
  }
  fwd_chain(P, f, pv, 0, nullptr, nullptr, p_parts, n_p_parts, st, 0, P->panel.as<__half>(), s);
  InterpOut of;
  of.panel = P->spanel.as<__half>();
  of.density = density;
  of.rows = P->M;
  of.coils = P->C;
  run_interp(P, TSN_VIEW_G, 1, EPI_PANEL, of, s);
  InterpOut oa;
  oa.c64 = P->grid.as<float2>();
  oa.rows = grid_cells(P);
  oa.coils = P->C;
  run_interp(P, TSN_VIEW_GT, 1, EPI_GRID, oa, s);
  inv_to_lines(P, f, P->grid.as<float2>(), s);
  double* parts = P->parts_rr.as<double>();
  launch_inv_rows(f, P->z1.as<float2>(), static_cast<float2*>(q), 5, static_cast<float2*>(coils), nullptr, pv, parts, st,
                  0, 1.0f, lambda, s);
  if (pq) launch_sum_partials_to(parts, settle_partials(P, parts, s), pq, s);
}

// Cuts (once per share value, outside any stream capture) the interpolation warp runs for a
// 1/share slice of the GPU, so cases of a batch run their launches side by side.
void prepare_share(tsn_plan* P, int share) {
  if (share <= 1) return;
  for (DevView& d : P->view) {
    if (!d.present || d.share == share) continue;
    const int warps = std::max(kInterpWarpsPerCta, interp_resident_warps(4 * P->C, d.v.ncomp, d.v.stages) / share);
    const std::vector<int2> ranges = cut_ranges(d.item_ends, d.tiles, warps);
    d.ranges_shared.upload(ranges);
    d.v_shared = d.v;
    d.v_shared.programmatic = 0;  // slices of the GPU shared with other cases' kernels
    d.v_shared.warp_ranges = d.ranges_shared.as<int2>();
    d.v_shared.n_warps = static_cast<int32_t>(ranges.size());
    d.share = share;
  }
}

void enqueue_adjoint_grid(tsn_plan* P, const void* y, const float* density, cudaStream_t s, int share = 1,
                          bool reference = false) {
  CgState* st = P->state.as<CgState>();
  launch_norm_partials(static_cast<const float2*>(y), P->M * P->C, P->norm_parts.as<double>(), s);
  launch_split_samples(static_cast<const float2*>(y), density, P->M, P->C, P->spanel.as<__half>(),
                       P->norm_parts.as<double>(), kNormParts, st, s);
  InterpOut o;
  o.c64 = P->grid.as<float2>();
  o.rows = grid_cells(P);
  o.coils = P->C;
  run_interp(P, TSN_VIEW_GT, share, EPI_GRID, o, s, reference);
}

// The CG-SENSE solve (launch_cg, nufft_fp16x2_cg_bench.cu:241-268). With reliable_period > 0,
// after every reliable_period-th iteration except the last the recursive residual is replaced
// by r = b - M x and p restarts as r (direction 0) or continues as r + beta p (direction 1), as
// in reference_sparse_solver.py:297-323.  Reference steps (completed iteration s a multiple of
// ref_period, or bit s-1 of ref_steps) take A^H W A p through the plan's FP32-class views; when
// the plan has them and any reference step or reliable update is asked for, the right-hand side
// and the reliable residuals use them too (rhs_adjoint / reliable_forward of :200-332).
void enqueue_cg(tsn_plan* P, const void* y, const void* smaps, const float* density, float lambda, float scale,
                int iters, void* x, cudaStream_t s, int share = 1, int reliable_period = 0,
                int reliable_direction = 0, int ref_period = 0, uint64_t ref_steps = 0) {
  const bool have_ref = P->view_ref[TSN_VIEW_G].present && P->view_ref[TSN_VIEW_GT].present;
  const bool ref_needed = have_ref && (reliable_period > 0 || ref_period > 0 || ref_steps != 0);
  auto ref_step = [&](int k) {  // iteration k (0-based) completes iteration k + 1
    return have_ref && ((k < 64 && ((ref_steps >> k) & 1ull)) || (ref_period > 0 && (k + 1) % ref_period == 0));
  };
  const FftArgs f = fft_args(P, smaps, share);
  CgState* st = P->state.as<CgState>();
  const float inv_s2 = 1.0f / (scale * scale);
  const float lam = lambda * inv_s2;
  float2* X = static_cast<float2*>(x);
  float2 *R = P->r.as<float2>(), *Pv = P->p.as<float2>(), *AP = P->ap.as<float2>();
  double *pap = P->parts_pap.as<double>(), *rr = P->parts_rr.as<double>();
  const int lines = f.lines();
  enqueue_adjoint_grid(P, y, density, s, share, ref_needed);
  inv_to_lines(P, f, P->grid.as<float2>(), s);
  launch_inv_rows(f, P->z1.as<float2>(), nullptr, 1, X, R, nullptr, rr, st, 0, inv_s2, 0.f, s);
  int n_rr = settle_partials(P, rr, s);
  if (reliable_period > 0)  // keep b for the reliable residuals
    CUDA_OK(cudaMemcpyAsync(P->rhs.ptr, R, P->rhs.bytes, cudaMemcpyDeviceToDevice, s));
  // An iteration followed by a plain one leaves its x / r update to the next forward rows
  // (mode 4), which read alpha and rho from four partial sections of the inverse rows; the
  // last iteration and those before a reliable residual run cg_update.
  bool restart = false, fused = false;
  int n_pap = 0;
  for (int k = 0; k < iters; ++k) {
    if (fused)
      fwd_chain(P, f, nullptr, 4, Pv, R, pap, n_pap, st, k, P->panel.as<__half>(), s, X, AP);
    else
      fwd_chain(P, f, nullptr, restart ? 2 : 1, Pv, R, rr, n_rr, st, k, P->panel.as<__half>(), s);
    restart = false;
    InterpOut of;
    of.panel = P->spanel.as<__half>();
    of.density = density;
    of.rows = P->M;
    of.coils = P->C;
    const bool ref = ref_step(k);
    run_interp(P, TSN_VIEW_G, share, EPI_PANEL, of, s, ref);
    InterpOut oa;
    oa.c64 = P->grid.as<float2>();
    oa.rows = grid_cells(P);
    oa.coils = P->C;
    run_interp(P, TSN_VIEW_GT, share, EPI_GRID, oa, s, ref);
    inv_to_lines(P, f, P->grid.as<float2>(), s);
    const bool reliable = reliable_period > 0 && (k + 1) % reliable_period == 0 && k + 1 < iters;
    fused = k + 1 < iters && !reliable;
    launch_inv_rows(f, P->z1.as<float2>(), AP, 2, nullptr, R, Pv, pap, st, k, inv_s2, lam, s);
    n_pap = settle_partials(P, pap, s, 4);
    if (fused) continue;
    launch_cg_update(P->N, lines, n_pap, X, R, Pv, AP, pap, rr, st, k, s);
    n_rr = settle_partials(P, rr, s);
    if (reliable) {
      // r = b - (A^H W A + lambda) x: plain forward of x, then the adjoint into residual mode
      launch_norm_partials(X, image_pixels(P), P->norm_parts.as<double>(), s);
      fwd_chain(P, f, X, 0, nullptr, nullptr, P->norm_parts.as<double>(), kNormParts, st, 0, P->panel.as<__half>(), s);
      run_interp(P, TSN_VIEW_G, share, EPI_PANEL, of, s, ref_needed);
      run_interp(P, TSN_VIEW_GT, share, EPI_GRID, oa, s, ref_needed);
      inv_to_lines(P, f, P->grid.as<float2>(), s);
      launch_inv_rows(f, P->z1.as<float2>(), R, 3, P->rhs.as<float2>(), nullptr, X, rr, st, k, inv_s2, lam, s);
      n_rr = settle_partials(P, rr, s);
      restart = reliable_direction == 0;
    }
  }
  launch_cg_finish(n_rr, rr, st, iters, s);
}

// Reads a finished solve's scalar state (synchronizes s) into the optional host outputs and
// returns the failure status of the solve (TSN_OK when finite with positive curvature).
tsn_status read_cg_state(const tsn_plan* P, int iters, double* residual_history, tsn_cg_status* status,
                         cudaStream_t s) {
  CgState host;
  int32_t tc_err = 0;
  CUDA_OK(cudaMemcpyAsync(&host, P->state.ptr, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  if (P->use_tc) CUDA_OK(cudaMemcpyAsync(&tc_err, P->tc_error.ptr, sizeof tc_err, cudaMemcpyDeviceToHost, s));
  CUDA_OK(cudaStreamSynchronize(s));
  if (residual_history)
    for (int k = 0; k <= iters; ++k) residual_history[k] = std::sqrt(std::max(host.rho[k], 0.0));
  if (status) {
    status->completed_iterations = host.completed;
    status->positive_curvature = host.curvature_ok;
    status->finite = host.finite_ok && std::isfinite(host.rho[iters]);
    status->timeout = tc_err != 0;
    status->residual0 = std::sqrt(std::max(host.rho[0], 0.0));
    status->residual_final = std::sqrt(std::max(host.rho[iters], 0.0));
  }
  if (tc_err) {
    set_last_error("a tensor-core interpolation launch gave up a bounded wait");
    return TSN_ERR_TIMEOUT;
  }
  if (!host.finite_ok || !std::isfinite(host.rho[iters])) return TSN_ERR_NONFINITE;
  if (!host.curvature_ok) return TSN_ERR_CURVATURE;
  return TSN_OK;
}

// Rough cost of one CG iteration of a plan in tile units (sparse tiles plus FFT points).
double case_cost(const tsn_plan* P) {
  return static_cast<double>(P->view[TSN_VIEW_G].tiles + P->view[TSN_VIEW_GT].tiles) +
         static_cast<double>(P->C) * static_cast<double>(grid_cells(P)) / 25.0;
}

}  // namespace

extern "C" {

static tsn_status forward_entry(tsn_plan* plan, const void* x, const void* smaps, void* y, tsn_stream_t stream,
                                bool reference) {
  try {
    if (!plan || !x || !y) fail(TSN_ERR_ARG, "NULL argument");
    need_aligned({x, smaps, y});
    need_views(plan, true, false);
    if (reference && !plan->view_ref[TSN_VIEW_G].present)
      fail(TSN_ERR_ARG, "the reference operator needs a plan built with TSN_FLAG_REFERENCE_STEPS");
    enqueue_forward(plan, x, smaps, y, reinterpret_cast<cudaStream_t>(stream), reference);
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

static tsn_status adjoint_entry(tsn_plan* plan, const void* y, const void* smaps, void* x, tsn_stream_t stream,
                                bool reference) {
  try {
    if (!plan || !x || !y) fail(TSN_ERR_ARG, "NULL argument");
    need_aligned({x, smaps, y});
    need_views(plan, false, true);
    if (reference && !plan->view_ref[TSN_VIEW_GT].present)
      fail(TSN_ERR_ARG, "the reference operator needs a plan built with TSN_FLAG_REFERENCE_STEPS");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    enqueue_adjoint_grid(plan, y, nullptr, s, 1, reference);
    const FftArgs f = fft_args(plan, smaps);
    inv_to_lines(plan, f, plan->grid.as<float2>(), s);
    launch_inv_rows(f, plan->z1.as<float2>(), static_cast<float2*>(x), 0, nullptr, nullptr, nullptr, nullptr,
                    plan->state.as<CgState>(), 0, 1.0f, 0.f, s);
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_forward(tsn_plan* plan, const void* x, const void* smaps, void* y, tsn_stream_t stream) {
  return forward_entry(plan, x, smaps, y, stream, false);
}

tsn_status tsn_adjoint(tsn_plan* plan, const void* y, const void* smaps, void* x, tsn_stream_t stream) {
  return adjoint_entry(plan, y, smaps, x, stream, false);
}

tsn_status tsn_normal(tsn_plan* plan, const void* p, const void* smaps, const float* density, float lambda, void* q,
                      void* coil_images, double* pq, const double* p_norm_parts, int32_t n_p_norm_parts,
                      tsn_stream_t stream) {
  try {
    if (!plan || !p || !smaps || !q) fail(TSN_ERR_ARG, "NULL argument (p, smaps and q are required)");
    if (!std::isfinite(lambda)) fail(TSN_ERR_ARG, "lambda must be finite");
    if (p_norm_parts && n_p_norm_parts <= 0) fail(TSN_ERR_ARG, "n_p_norm_parts must be positive");
    need_aligned({p, smaps, q, coil_images, density});
    need_views(plan, true, true);
    enqueue_normal(plan, p, smaps, density, lambda, q, coil_images, pq, p_norm_parts, n_p_norm_parts,
                   reinterpret_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_rdot(tsn_plan* plan, const void* a, const void* b, int64_t n, double* out, tsn_stream_t stream) {
  try {
    if (!plan || !a || !b || !out) fail(TSN_ERR_ARG, "NULL argument");
    if (n < 0) fail(TSN_ERR_ARG, "n must be >= 0");
    CUDA_OK(cudaSetDevice(plan->desc.device));
    launch_rdot(static_cast<const float2*>(a), static_cast<const float2*>(b), n, plan->norm_parts.as<double>(), out,
                reinterpret_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_cg_step(tsn_plan* plan, int64_t n, const double* rho, const double* gamma, const void* x, const void* p,
                       const void* r, const void* q, void* x_out, void* r_out, void* p_out, double* rho_out,
                       double* p_norm_parts, tsn_stream_t stream) {
  try {
    if (!plan || !rho || !gamma || !p || !r || !q || !r_out || !p_out || !rho_out) fail(TSN_ERR_ARG, "NULL argument");
    if ((x == nullptr) != (x_out == nullptr)) fail(TSN_ERR_ARG, "x and x_out go together");
    if (n < 0) fail(TSN_ERR_ARG, "n must be >= 0");
    CUDA_OK(cudaSetDevice(plan->desc.device));
    launch_cg_step(n, plan->adj_parts.as<double>(), rho, gamma, static_cast<const float2*>(x),
                   static_cast<const float2*>(p), static_cast<const float2*>(r), static_cast<const float2*>(q),
                   static_cast<float2*>(x_out), static_cast<float2*>(r_out), static_cast<float2*>(p_out), rho_out,
                   p_norm_parts, reinterpret_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_cg_adjoint_step(tsn_plan* plan, int64_t n, const double* rho, const double* rho_next,
                               const double* gamma, const double* rhob, double* rhob_out, void* rb, void* pb,
                               const void* p, const void* q, const void* r_next, const void* xb, void* qb,
                               double* qb_norm_parts, tsn_stream_t stream) {
  try {
    if (!plan || !rho || !rho_next || !gamma || !rhob || !rhob_out || !rb || !pb || !p || !q || !r_next || !xb || !qb)
      fail(TSN_ERR_ARG, "NULL argument");
    if (n < 0) fail(TSN_ERR_ARG, "n must be >= 0");
    CUDA_OK(cudaSetDevice(plan->desc.device));
    launch_cg_adjoint_step(n, plan->adj_parts.as<double>(), rho, rho_next, gamma, rhob, rhob_out,
                           static_cast<float2*>(rb), static_cast<float2*>(pb), static_cast<const float2*>(p),
                           static_cast<const float2*>(q), static_cast<const float2*>(r_next),
                           static_cast<const float2*>(xb), static_cast<float2*>(qb), qb_norm_parts,
                           reinterpret_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_cg_adjoint_finish(tsn_plan* plan, int64_t n, int32_t coils, void* pb, const void* mqb, const void* qb,
                                 const void* coil_images, const void* coil_images_bar, const void* p, void* sb,
                                 tsn_stream_t stream) {
  try {
    if (!plan || !pb || !mqb) fail(TSN_ERR_ARG, "NULL argument");
    if (n < 0 || coils < 0) fail(TSN_ERR_ARG, "n and coils must be >= 0");
    if (sb && (!qb || !coil_images || !coil_images_bar || !p)) fail(TSN_ERR_ARG, "the map cotangent needs qb, t, tb and p");
    CUDA_OK(cudaSetDevice(plan->desc.device));
    launch_cg_adjoint_finish(n, coils, static_cast<float2*>(pb), static_cast<const float2*>(mqb),
                             static_cast<const float2*>(qb), static_cast<const float2*>(coil_images),
                             static_cast<const float2*>(coil_images_bar), static_cast<const float2*>(p),
                             static_cast<float2*>(sb), reinterpret_cast<cudaStream_t>(stream));
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_forward_reference(tsn_plan* plan, const void* x, const void* smaps, void* y, tsn_stream_t stream) {
  return forward_entry(plan, x, smaps, y, stream, true);
}

tsn_status tsn_adjoint_reference(tsn_plan* plan, const void* y, const void* smaps, void* x, tsn_stream_t stream) {
  return adjoint_entry(plan, y, smaps, x, stream, true);
}

tsn_status tsn_cg_sense_ex(tsn_plan* plan, const void* y, const void* smaps, const float* density, float lambda,
                           float operator_scale, int32_t iters, const tsn_cg_options* options, void* x,
                           double* residual_history, tsn_cg_status* status, tsn_stream_t stream) {
  try {
    const int period = options ? options->reliable_update_period : 0;
    const int direction = options ? options->reliable_update_direction : 0;
    const int ref_period = options ? options->scheduled_reference_period : 0;
    const uint64_t ref_steps = options ? options->reference_steps : 0;
    if (period < 0 || direction < 0 || direction > 1) fail(TSN_ERR_ARG, "invalid reliable-update options");
    if (ref_period < 0) fail(TSN_ERR_ARG, "scheduled_reference_period must be >= 0");
    if ((ref_period > 0 || ref_steps) && plan && !plan->view_ref[TSN_VIEW_G].present)
      fail(TSN_ERR_ARG, "reference steps need a plan built with TSN_FLAG_REFERENCE_STEPS");
    if (!plan || !y || !smaps || !x) fail(TSN_ERR_ARG, "NULL argument (y, smaps and x are required)");
    if (iters < 0 || iters > kMaxCgIter) fail(TSN_ERR_ARG, "iteration count out of range");
    if (!(operator_scale > 0.0f) || !std::isfinite(lambda)) fail(TSN_ERR_ARG, "invalid operator scale or lambda");
    need_aligned({y, smaps, x});
    if (reinterpret_cast<uintptr_t>(density) & 3u) fail(TSN_ERR_ARG, "density must be 4-byte aligned");
    need_views(plan, true, true);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    GraphKey key{y, smaps, density, x, iters, 0, 0, s, period * 2 + direction, ref_period, ref_steps};
    std::memcpy(&key.lam_bits, &lambda, 4);
    std::memcpy(&key.scale_bits, &operator_scale, 4);
    auto it = plan->graphs.find(key);
    if (it == plan->graphs.end()) {
      cudaStream_t cap = s;
      bool own = false;
      if (cap == nullptr) {  // the legacy stream cannot be captured: capture on a private stream
        CUDA_OK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        own = true;
      }
      cudaGraph_t g = nullptr;
      CUDA_OK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed));
      enqueue_cg(plan, y, smaps, density, lambda, operator_scale, iters, x, cap, 1, period, direction, ref_period,
                 ref_steps);
      const cudaError_t launch_err = cudaGetLastError();
      const cudaError_t end_err = cudaStreamEndCapture(cap, &g);
      if (own) cudaStreamDestroy(cap);
      if (launch_err != cudaSuccess) fail(TSN_ERR_CUDA, cudaGetErrorString(launch_err));
      if (end_err != cudaSuccess) fail(TSN_ERR_CUDA, cudaGetErrorString(end_err));
      cudaGraphExec_t exec = nullptr;
      const cudaError_t inst = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      if (inst != cudaSuccess) fail(TSN_ERR_CUDA, cudaGetErrorString(inst));
      if (plan->graphs.size() >= 8) {
        cudaGraphExecDestroy(plan->graphs.begin()->second);
        plan->graphs.erase(plan->graphs.begin());
      }
      it = plan->graphs.emplace(key, exec).first;
    }
    CUDA_OK(cudaGraphLaunch(it->second, s));
    if (residual_history || status) {
      const tsn_status rc = read_cg_state(plan, iters, residual_history, status, s);
      if (rc == TSN_ERR_TIMEOUT) fail(TSN_ERR_TIMEOUT, "a bounded device wait gave up during the solve");
      if (rc == TSN_ERR_NONFINITE) fail(TSN_ERR_NONFINITE, "CG produced non-finite values");
      if (rc == TSN_ERR_CURVATURE) fail(TSN_ERR_CURVATURE, "CG denominator <= 0 (positive_curvature = 0)");
    }
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_cg_sense(tsn_plan* plan, const void* y, const void* smaps, const float* density, float lambda,
                        float operator_scale, int32_t iters, void* x, double* residual_history,
                        tsn_cg_status* status, tsn_stream_t stream) {
  return tsn_cg_sense_ex(plan, y, smaps, density, lambda, operator_scale, iters, nullptr, x, residual_history, status,
                         stream);
}

tsn_status tsn_batch_create(tsn_plan* const* plans, int32_t count, int32_t streams, tsn_batch** out) {
  try {
    if (!plans || !out || count <= 0) fail(TSN_ERR_ARG, "invalid argument");
    *out = nullptr;
    auto b = std::make_unique<tsn_batch>();
    b->plans.assign(plans, plans + count);
    for (tsn_plan* P : b->plans) {
      if (!P) fail(TSN_ERR_ARG, "NULL plan in batch");
      need_views(P, true, true);
      if (P->desc.device != b->plans[0]->desc.device) fail(TSN_ERR_ARG, "batch plans must share one device");
    }
    b->device = b->plans[0]->desc.device;
    CUDA_OK(cudaSetDevice(b->device));
    b->streams = std::max(1, std::min<int>(count, streams > 0 ? streams : 8));
    // longest-first onto the least-loaded stream
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return case_cost(b->plans[a]) > case_cost(b->plans[c]); });
    std::vector<double> load(b->streams, 0.0);
    b->lane.assign(count, 0);
    for (int i : order) {
      const int k = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
      b->lane[i] = k;
      load[k] += case_cost(b->plans[i]);
    }
    for (tsn_plan* P : b->plans) prepare_share(P, b->streams);
    b->side.resize(b->streams);
    b->join.resize(b->streams);
    CUDA_OK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (int k = 0; k < b->streams; ++k) {
      CUDA_OK(cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking));
      CUDA_OK(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming));
    }
    CUDA_OK(cudaGetLastError());
    *out = b.release();
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_batch_destroy(tsn_batch* batch) {
  if (batch) {
    cudaSetDevice(batch->device);
    delete batch;
  }
  return TSN_OK;
}

tsn_status tsn_batch_cg_sense(tsn_batch* batch, const void* const* y, const void* const* smaps,
                              const float* const* density, float lambda, float operator_scale, int32_t iters,
                              void* const* x, tsn_cg_status* statuses, tsn_stream_t stream) {
  try {
    if (!batch || !y || !smaps || !x) fail(TSN_ERR_ARG, "NULL argument (y, smaps and x are required)");
    if (iters < 0 || iters > kMaxCgIter) fail(TSN_ERR_ARG, "iteration count out of range");
    if (!(operator_scale > 0.0f) || !std::isfinite(lambda)) fail(TSN_ERR_ARG, "invalid operator scale or lambda");
    const int count = static_cast<int>(batch->plans.size());
    std::vector<uint64_t> key;
    key.reserve(4 * count + 4);
    for (int i = 0; i < count; ++i) {
      const float* w = density ? density[i] : nullptr;
      if (!y[i] || !smaps[i] || !x[i]) fail(TSN_ERR_ARG, "NULL per-case pointer (y, smaps and x are required)");
      need_aligned({y[i], smaps[i], x[i]});
      if (reinterpret_cast<uintptr_t>(w) & 3u) fail(TSN_ERR_ARG, "density must be 4-byte aligned");
      for (const void* q : {y[i], smaps[i], static_cast<const void*>(w), static_cast<const void*>(x[i])})
        key.push_back(static_cast<uint64_t>(reinterpret_cast<uintptr_t>(q)));
    }
    uint32_t lam_bits = 0, scale_bits = 0;
    std::memcpy(&lam_bits, &lambda, 4);
    std::memcpy(&scale_bits, &operator_scale, 4);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    key.push_back(static_cast<uint64_t>(iters));
    key.push_back((static_cast<uint64_t>(lam_bits) << 32) | scale_bits);
    key.push_back(static_cast<uint64_t>(reinterpret_cast<uintptr_t>(s)));
    CUDA_OK(cudaSetDevice(batch->device));
    auto it = batch->graphs.find(key);
    if (it == batch->graphs.end()) {
      cudaStream_t cap = s;
      bool own = false;
      if (cap == nullptr) {  // the legacy stream cannot be captured: capture on a private stream
        CUDA_OK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        own = true;
      }
      cudaGraph_t g = nullptr;
      CUDA_OK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed));
      // fork every side stream off the capture, run each case on its stream, join back
      cudaEventRecord(batch->fork, cap);
      for (int k = 0; k < batch->streams; ++k) cudaStreamWaitEvent(batch->side[k], batch->fork, 0);
      for (int i = 0; i < count; ++i)
        enqueue_cg(batch->plans[i], y[i], smaps[i], density ? density[i] : nullptr, lambda, operator_scale, iters,
                   x[i], batch->side[batch->lane[i]], batch->streams);
      for (int k = 0; k < batch->streams; ++k) {
        cudaEventRecord(batch->join[k], batch->side[k]);
        cudaStreamWaitEvent(cap, batch->join[k], 0);
      }
      const cudaError_t launch_err = cudaGetLastError();
      const cudaError_t end_err = cudaStreamEndCapture(cap, &g);
      if (own) cudaStreamDestroy(cap);
      if (launch_err != cudaSuccess) fail(TSN_ERR_CUDA, cudaGetErrorString(launch_err));
      if (end_err != cudaSuccess) fail(TSN_ERR_CUDA, cudaGetErrorString(end_err));
      cudaGraphExec_t exec = nullptr;
      const cudaError_t inst = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      if (inst != cudaSuccess) fail(TSN_ERR_CUDA, cudaGetErrorString(inst));
      if (batch->graphs.size() >= 4) {
        cudaGraphExecDestroy(batch->graphs.begin()->second);
        batch->graphs.erase(batch->graphs.begin());
      }
      it = batch->graphs.emplace(key, exec).first;
    }
    CUDA_OK(cudaGraphLaunch(it->second, s));
    if (statuses) {
      tsn_status first = TSN_OK;
      int bad = -1;
      for (int i = 0; i < count; ++i) {
        const tsn_status rc = read_cg_state(batch->plans[i], iters, nullptr, &statuses[i], s);
        if (rc != TSN_OK && first == TSN_OK) {
          first = rc;
          bad = i;
        }
      }
      if (first != TSN_OK)
        fail(first, "batch case " + std::to_string(bad) +
                        (first == TSN_ERR_NONFINITE ? ": CG produced non-finite values"
                                                    : ": CG denominator <= 0 (positive_curvature = 0)"));
    }
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_profile_stages(tsn_plan* plan, const void* y, const void* smaps, int32_t reps, double* stage_ms,
                              tsn_stream_t stream) {
  try {
    if (!plan || !y || !smaps || !stage_ms || reps <= 0) fail(TSN_ERR_ARG, "invalid argument");
    need_aligned({y, smaps});
    need_views(plan, true, true);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    DeviceBuffer xbuf;
    xbuf.alloc(sizeof(float2) * image_pixels(plan));
    enqueue_cg(plan, y, smaps, nullptr, 1e-4f, 1.0f, 2, xbuf.ptr, s);
    const bool vol = plan->dims == 3;
    const int nparts = vol ? 1 : plan->N;  // the solve left single totals for volumes
    float2* z_cols = vol ? plan->z2.as<float2>() : plan->z1.as<float2>();  // first-axis stage data
    const FftArgs f = fft_args(plan, smaps);
    CgState* st = plan->state.as<CgState>();
    float2 *X = xbuf.as<float2>(), *R = plan->r.as<float2>(), *Pv = plan->p.as<float2>(), *AP = plan->ap.as<float2>();
    double *pap = plan->parts_pap.as<double>(), *rr = plan->parts_rr.as<double>();
    // iteration index 1 keeps p = r + beta p live; the stages read state written by the solve.
    // The row stages run as in the solve's inner iterations: forward rows finishing the
    // previous update (mode 4), inverse rows writing the four partial sections; x, r and p
    // drift over the repetitions, and only the times are kept.
    auto stage = [&](int which) {
      switch (which) {
        case TSN_STAGE_FWD_ROWS:
          launch_fwd_rows(f, nullptr, plan->z1.as<float2>(), 4, Pv, R, pap, nparts, st, 1, s, X, AP);
          break;
        case TSN_STAGE_FWD_COLS: launch_fwd_cols(f, z_cols, plan->panel.as<__half>(), s); break;
        case TSN_STAGE_FWD_MID:
          if (vol) launch_fwd_mid(f, plan->z1.as<float2>(), plan->z2.as<float2>(), s);
          break;
        case TSN_STAGE_INV_MID:
          if (vol) launch_inv_mid(f, plan->z2.as<float2>(), plan->z1.as<float2>(), s);
          break;
        case TSN_STAGE_INTERP_FWD: {
          InterpOut o;
          o.panel = plan->spanel.as<__half>();
          o.rows = plan->M;
          o.coils = plan->C;
          run_interp(plan, TSN_VIEW_G, 1, EPI_PANEL, o, s);
        } break;
        case TSN_STAGE_INTERP_ADJ: {
          InterpOut o;
          o.c64 = plan->grid.as<float2>();
          o.rows = grid_cells(plan);
          o.coils = plan->C;
          run_interp(plan, TSN_VIEW_GT, 1, EPI_GRID, o, s);
        } break;
        case TSN_STAGE_INV_COLS: launch_inv_cols(f, plan->grid.as<float2>(), z_cols, s); break;
        case TSN_STAGE_INV_ROWS:
          // volumes: partials stay per line here; cg_update below reads the solve's total
          launch_inv_rows(f, plan->z1.as<float2>(), AP, 2, nullptr, R, Pv, vol ? rr + 1 : pap, st, 1, 1.0f,
                          1e-4f, s);
          break;
        default: launch_cg_update(plan->N, f.lines(), nparts, X, R, Pv, AP, pap, vol ? rr + 1 : rr, st, 1, s); break;
      }
    };
    cudaEvent_t e0, e1;
    CUDA_OK(cudaEventCreate(&e0));
    CUDA_OK(cudaEventCreate(&e1));
    for (int which = 0; which < TSN_STAGE_COUNT; ++which) {
      if (!vol && (which == TSN_STAGE_FWD_MID || which == TSN_STAGE_INV_MID)) {
        stage_ms[which] = 0.0;  // images have no middle axis
        continue;
      }
      stage(which);  // warm
      CUDA_OK(cudaEventRecord(e0, s));
      for (int r = 0; r < reps; ++r) stage(which);
      CUDA_OK(cudaEventRecord(e1, s));
      CUDA_OK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
      stage_ms[which] = static_cast<double>(ms) / reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CUDA_OK(cudaGetLastError());
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_fft_forward_panel(tsn_plan* plan, const void* x, const void* smaps, void* panel_f16,
                                 float* panel_scale, tsn_stream_t stream) {
  try {
    if (!plan || !x || !panel_f16) fail(TSN_ERR_ARG, "NULL argument");
    need_aligned({x, smaps, panel_f16});
    need_views(plan, false, false);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const FftArgs f = fft_args(plan, smaps);
    CgState* st = plan->state.as<CgState>();
    const int64_t n = image_pixels(plan) * (smaps ? 1 : plan->C);
    launch_norm_partials(static_cast<const float2*>(x), n, plan->norm_parts.as<double>(), s);
    fwd_chain(plan, f, static_cast<const float2*>(x), 0, nullptr, nullptr, plan->norm_parts.as<double>(), kNormParts,
              st, 0, static_cast<__half*>(panel_f16), s);
    CUDA_OK(cudaGetLastError());
    if (panel_scale) {
      float sigma = 0.f;
      CUDA_OK(cudaMemcpyAsync(&sigma, &st->sigma_x, sizeof(float), cudaMemcpyDeviceToHost, s));
      CUDA_OK(cudaStreamSynchronize(s));
      *panel_scale = sigma / f.gs();
    }
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_fft_adjoint_image(tsn_plan* plan, const void* grid_c64, const void* smaps, void* x,
                                 tsn_stream_t stream) {
  try {
    if (!plan || !grid_c64 || !x) fail(TSN_ERR_ARG, "NULL argument");
    need_aligned({grid_c64, smaps, x});
    need_views(plan, false, false);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const FftArgs f = fft_args(plan, smaps);
    CgState* st = plan->state.as<CgState>();
    // unit sample scale for the plain adjoint epilogue (factor = 1 / sigma_y)
    const float one = 1.0f;
    CUDA_OK(cudaMemcpyAsync(&st->sigma_y, &one, sizeof(float), cudaMemcpyHostToDevice, s));
    inv_to_lines(plan, f, static_cast<const float2*>(grid_c64), s);
    launch_inv_rows(f, plan->z1.as<float2>(), static_cast<float2*>(x), 0, nullptr, nullptr, nullptr, nullptr, st, 0,
                    1.0f, 0.f, s);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(s));
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

tsn_status tsn_interp_component(tsn_plan* plan, int32_t view, int32_t component, const void* dense_f16, float* out,
                                tsn_stream_t stream) {
  try {
    if (!plan || !dense_f16 || !out) fail(TSN_ERR_ARG, "NULL argument");
    need_aligned({dense_f16, out});
    if (view != TSN_VIEW_G && view != TSN_VIEW_GT) fail(TSN_ERR_ARG, "unknown view");
    const DevView& d = plan->view[view];
    if (!d.present) fail(TSN_ERR_ARG, "plan lacks this view");
    CUDA_OK(cudaSetDevice(plan->desc.device));
    if (component < 0 || component >= d.v.ncomp) fail(TSN_ERR_ARG, "component out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t G = plan->G;
    // internal <-> reference index maps of this view
    std::vector<int32_t> col_map(d.n_cols), row_map(d.output_size);
    for (int64_t j = 0; j < d.n_cols; ++j)
      col_map[j] = static_cast<int32_t>(view == TSN_VIEW_G ? cell_to_internal(j, G) : j);  // internal j <- ref
    for (int64_t j = 0; j < d.output_size; ++j)
      row_map[j] = static_cast<int32_t>(view == TSN_VIEW_GT ? cell_to_internal(j, G) : j);
    DeviceBuffer cm, rm, din, dout;
    cm.upload(col_map);
    rm.upload(row_map);
    din.alloc(sizeof(__half) * d.n_cols * 16);
    dout.alloc(sizeof(float) * d.output_size * 16);
    CUDA_OK(cudaMemsetAsync(dout.ptr, 0, dout.bytes, s));
    // cell_to_internal is an involution on square grids: internal row j holds reference row map[j]
    launch_gather_rows_f16(static_cast<const __half*>(dense_f16), cm.as<int32_t>(), d.n_cols, 16, din.as<__half>(), s);
    InterpView v = d.v;
    std::vector<uint8_t> dummy;
    InterpOut o;
    o.raw = dout.as<float>();
    o.rows = d.output_size;
    // component selection: a two-component view gets a single-component record copy
    // (columns | A and metadata of the component | record info and rows)
    DeviceBuffer shifted;
    if (d.v.ncomp == 2) {
      const int one_rec = record_bytes(1);
      std::vector<uint8_t> host(static_cast<size_t>(d.tiles) * d.v.rec_bytes);
      CUDA_OK(cudaMemcpy(host.data(), d.v.records, host.size(), cudaMemcpyDeviceToHost));
      std::vector<uint8_t> one(static_cast<size_t>(d.tiles) * one_rec);
      for (int64_t t = 0; t < d.tiles; ++t) {
        const uint8_t* src = &host[t * d.v.rec_bytes];
        uint8_t* dst = &one[t * one_rec];
        std::memcpy(dst, src, 128);
        std::memcpy(dst + 128, src + 128 + 576 * component, 576);
        std::memcpy(dst + 128 + 576, src + 128 + 576 * 2, kRecInfoBytes);
      }
      shifted.upload(one);
      v.records = shifted.as<uint8_t>();
      v.rec_bytes = one_rec;
    }
    v.ncomp = 1;
    launch_interp(v, din.as<__half>(), 16, false, EPI_RAW, false, o, s);
    launch_gather_rows_f32(dout.as<float>(), rm.as<int32_t>(), d.output_size, 16, out, s);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaStreamSynchronize(s));
    return TSN_OK;
  } catch (const std::exception& e) {
    return guard_status(e);
  }
}

}  // extern "C"
