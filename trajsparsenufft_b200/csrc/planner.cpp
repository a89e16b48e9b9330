// Pack-once planner (C++). The steps, tie-breaks and random-number consumption follow
// the reference planner exactly so that packs are byte-identical:
//   row grouping             src/nufft_layout_oracle.py:243-309, morton2d :110-121
//   column -> K-tile split   src/nufft_layout_oracle.py:323-372 (search),
//                            src/export_torchkbnufft_gpu_case.py:102-162 (optimized)
//   quartet arrangement      src/nufft_layout_oracle.py:375-442 (search),
//                            src/export_torchkbnufft_gpu_case.py:165-214 (optimized)
//   whole-view packers       pack_view :445-497, fast_split24_pack :46-99,
//                            optimized_split24_pack :270-299
//   split24 / CSR residual   src/export_gpu_case.py:77-155
//   FP16 2:4 compression     src/export_gpu_case.py:41-74
// Groups are independent (their seeds depend only on the group index), so they are
// planned on a thread pool and concatenated in group order.
#include "planner.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <memory>
#include <thread>
#include <unordered_map>

namespace tsn {

int resolve_threads(int threads) {
  if (threads > 0) return threads;
  const unsigned hc = std::thread::hardware_concurrency();
  return hc ? static_cast<int>(hc) : 1;
}

template <class F>
static void parallel_for(int64_t n, int threads, F&& body) {
  threads = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(threads, n)));
  if (threads <= 1) {
    for (int64_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  std::exception_ptr err;
  std::atomic<bool> failed{false};
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&]() {
      try {
        for (;;) {
          const int64_t i = next.fetch_add(1);
          if (i >= n || failed.load()) break;
          body(i);
        }
      } catch (...) {
        if (!failed.exchange(true)) err = std::current_exception();
      }
    });
  }
  for (auto& th : pool) th.join();
  if (err) std::rethrow_exception(err);
}

// Volume transpose on all host cores without a random scatter over the whole matrix: entries
// are streamed into buckets of 2^14 consecutive cells (each thread owns a contiguous run of
// source rows, so a bucket holds every cell's entries in ascending source-row order), then
// each bucket is counting-sorted by cell into its contiguous output range. The layout is
// exactly the serial transpose's.
static SparseView transpose_view_parallel(const SparseView& v, int64_t grid_size) {
  const int threads = resolve_threads(0);
  const int64_t n_rows = v.rows(), nnz = v.nnz(), n_cols = v.n_cols;
  constexpr int kBucketShift = 14;
  const int64_t buckets = (n_cols + (int64_t(1) << kBucketShift) - 1) >> kBucketShift;
  if (n_cols > (int64_t(1) << 31) || n_rows > (int64_t(1) << 31)) fail(TSN_ERR_UNSUPPORTED, "view too large");
  for (int64_t k = 0; k < nnz; k += std::max<int64_t>(1, nnz / 4096))
    if (v.cols[k] < 0 || v.cols[k] >= n_cols) fail(TSN_ERR_SHAPE, "column id out of range");
  // pass 1: per-thread bucket histograms over contiguous source-row runs
  const int T = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(threads, n_rows)));
  std::vector<int64_t> hist(static_cast<size_t>(T) * buckets, 0);
  std::atomic<bool> bad{false};
  auto row_run = [&](int th, int64_t& r0, int64_t& r1) {
    r0 = n_rows * th / T;
    r1 = n_rows * (th + 1) / T;
  };
  parallel_for(T, T, [&](int64_t th) {
    int64_t r0, r1;
    row_run(static_cast<int>(th), r0, r1);
    int64_t* h = &hist[static_cast<size_t>(th) * buckets];
    for (int64_t k = v.row_ptr[r0]; k < v.row_ptr[r1]; ++k) {
      const int64_t c = v.cols[k];
      if (c < 0 || c >= n_cols) {
        bad.store(true);
        return;
      }
      ++h[c >> kBucketShift];
    }
  });
  if (bad.load()) fail(TSN_ERR_SHAPE, "column id out of range");
  // write offsets: bucket-major, thread order within a bucket
  std::vector<int64_t> bucket_start(buckets + 1, 0);
  std::vector<int64_t> off(static_cast<size_t>(T) * buckets);
  int64_t pos = 0;
  for (int64_t b = 0; b < buckets; ++b) {
    bucket_start[b] = pos;
    for (int th = 0; th < T; ++th) {
      off[static_cast<size_t>(th) * buckets + b] = pos;
      pos += hist[static_cast<size_t>(th) * buckets + b];
    }
  }
  bucket_start[buckets] = pos;
  hist.clear();
  hist.shrink_to_fit();
  struct Entry {
    int32_t cell, row;
    double val;
  };
  std::vector<Entry> staged;
  resize_huge(staged, static_cast<size_t>(nnz));
  parallel_for(T, T, [&](int64_t th) {
    int64_t r0, r1;
    row_run(static_cast<int>(th), r0, r1);
    int64_t* o = &off[static_cast<size_t>(th) * buckets];
    for (int64_t r = r0; r < r1; ++r) {
      const int32_t logical = static_cast<int32_t>(v.row_ids[r]);
      for (int64_t k = v.row_ptr[r]; k < v.row_ptr[r + 1]; ++k) {
        const int64_t c = v.cols[k];
        staged[o[c >> kBucketShift]++] = Entry{static_cast<int32_t>(c), logical, v.vals[k]};
      }
    }
  });
  off.clear();
  off.shrink_to_fit();
  // pass 2: per-bucket cell counts, then the global row structure
  std::vector<int32_t> count;
  resize_huge(count, static_cast<size_t>(n_cols));
  parallel_for(buckets, threads, [&](int64_t b) {
    for (int64_t k = bucket_start[b]; k < bucket_start[b + 1]; ++k) ++count[staged[k].cell];
  });
  SparseView t;
  t.output_size = n_cols;
  t.n_cols = v.output_size;
  t.dims = v.dims;
  t.row_ptr.push_back(0);
  std::vector<int64_t> row_start;
  resize_huge(row_start, static_cast<size_t>(n_cols));
  for (int64_t c = 0; c < n_cols; ++c) {
    row_start[c] = t.row_ptr.back();
    if (!count[c]) continue;
    t.row_ids.push_back(c);
    t.coords.push_back(static_cast<double>(c % grid_size));
    t.coords.push_back(static_cast<double>((c / grid_size) % grid_size));
    t.coords.push_back(static_cast<double>(c / (grid_size * grid_size)));
    t.row_ptr.push_back(t.row_ptr.back() + count[c]);
  }
  count.clear();
  count.shrink_to_fit();
  resize_huge(t.cols, static_cast<size_t>(nnz));
  resize_huge(t.vals, static_cast<size_t>(nnz));
  // pass 3: stable scatter of each bucket into its contiguous output range
  parallel_for(buckets, threads, [&](int64_t b) {
    for (int64_t k = bucket_start[b]; k < bucket_start[b + 1]; ++k) {
      const Entry& e = staged[k];
      const int64_t at = row_start[e.cell]++;
      t.cols[at] = e.row;
      t.vals[at] = e.val;
    }
  });
  return t;
}

SparseView transpose_view(const SparseView& v, int64_t grid_size) {
  if (v.dims == 3) return transpose_view_parallel(v, grid_size);
  std::vector<int64_t> count(v.n_cols, 0);
  for (int64_t c : v.cols) {
    if (c < 0 || c >= v.n_cols) fail(TSN_ERR_SHAPE, "column id out of range");
    ++count[c];
  }
  SparseView t;
  t.output_size = v.n_cols;
  t.n_cols = v.output_size;
  t.dims = v.dims;
  std::vector<int64_t> slot(v.n_cols, -1);
  t.row_ptr.push_back(0);
  for (int64_t c = 0; c < v.n_cols; ++c) {
    if (!count[c]) continue;
    slot[c] = static_cast<int64_t>(t.row_ids.size());
    t.row_ids.push_back(c);
    t.coords.push_back(static_cast<double>(c % grid_size));
    t.coords.push_back(static_cast<double>((c / grid_size) % (v.dims == 3 ? grid_size : INT64_MAX)));
    if (v.dims == 3) t.coords.push_back(static_cast<double>(c / (grid_size * grid_size)));
    t.row_ptr.push_back(t.row_ptr.back() + count[c]);
  }
  std::vector<int64_t> fill(t.row_ids.size(), 0);
  t.cols.resize(v.nnz());
  t.vals.resize(v.nnz());
  for (int64_t r = 0; r < v.rows(); ++r) {
    const int64_t logical = v.row_ids[r];
    for (int64_t k = v.row_ptr[r]; k < v.row_ptr[r + 1]; ++k) {
      const int64_t s = slot[v.cols[k]];
      const int64_t at = t.row_ptr[s] + fill[s]++;
      t.cols[at] = logical;
      t.vals[at] = v.vals[k];
    }
  }
  return t;
}

static uint32_t spread16(uint32_t v) {
  v &= 0xFFFFu;
  v = (v | (v << 8)) & 0x00FF00FFu;
  v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

// 3D morton: bit b of v goes to bit 3b.
static uint64_t spread21(uint32_t v) {
  uint64_t out = 0;
  for (int b = 0; b < 21; ++b) out |= static_cast<uint64_t>((v >> b) & 1u) << (3 * b);
  return out;
}

// Python int(round(x)): round half to even.
static int64_t py_round(double x) { return static_cast<int64_t>(std::nearbyint(x)); }

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

std::vector<int64_t> row_order(const SparseView& v, int policy, int k_tile) {
  const int64_t n = v.rows();
  std::vector<int64_t> order(n);
  for (int64_t i = 0; i < n; ++i) order[i] = i;
  if (policy == TSN_POLICY_TRAJECTORY) return order;
  std::vector<uint64_t> key(n);
  if (v.dims == 3) {
    for (int64_t r = 0; r < n; ++r) {
      uint64_t k = 0;
      for (int d = 0; d < 3; ++d) {
        const int64_t c = std::max<int64_t>(0, py_round(v.coords[3 * r + d]));
        k |= spread21(static_cast<uint32_t>(c & 0x1FFFFF)) << d;
      }
      key[r] = k;
    }
  } else {
    for (int64_t r = 0; r < n; ++r) {
      const int64_t x = std::max<int64_t>(0, py_round(v.coords[2 * r]));
      const int64_t y = std::max<int64_t>(0, py_round(v.coords[2 * r + 1]));
      key[r] = static_cast<uint64_t>(spread16(static_cast<uint32_t>(x & 0xFFFF))) |
               (static_cast<uint64_t>(spread16(static_cast<uint32_t>(y & 0xFFFF))) << 1);
    }
  }
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
  if (policy == TSN_POLICY_MORTON) return order;
  if (policy != TSN_POLICY_OVERLAP && policy != TSN_POLICY_PACKING256)
    fail(TSN_ERR_ARG, "unknown row grouping policy");
  const int64_t window = policy == TSN_POLICY_OVERLAP ? 4 * kMTile : 16 * kMTile;
  std::vector<int64_t> out(n);
  const int64_t n_windows = ceil_div(n, window);
  parallel_for(n_windows, resolve_threads(0), [&](int64_t w) {
    const int64_t start = w * window;
    const int64_t stop = std::min(n, start + window);
    std::vector<int64_t> rem(order.begin() + start, order.begin() + stop);
    // local column ids within the window -> bitset unions
    std::unordered_map<int64_t, int32_t> local;
    std::vector<std::vector<int32_t>> sup(rem.size());
    for (size_t i = 0; i < rem.size(); ++i) {
      const int64_t r = rem[i];
      for (int64_t k = v.row_ptr[r]; k < v.row_ptr[r + 1]; ++k) {
        auto it = local.emplace(v.cols[k], static_cast<int32_t>(local.size())).first;
        sup[i].push_back(it->second);
      }
      std::sort(sup[i].begin(), sup[i].end());
      sup[i].erase(std::unique(sup[i].begin(), sup[i].end()), sup[i].end());
    }
    std::vector<int32_t> remi(rem.size());
    for (size_t i = 0; i < rem.size(); ++i) remi[i] = static_cast<int32_t>(i);
    std::vector<uint8_t> in_union(local.size(), 0);
    int64_t pos_out = start;
    while (!remi.empty()) {
      std::fill(in_union.begin(), in_union.end(), 0);
      std::vector<int32_t> group{remi.front()};
      remi.erase(remi.begin());
      int64_t union_size = 0;
      for (int32_t c : sup[group[0]]) {
        in_union[c] = 1;
        ++union_size;
      }
      int64_t nnz_now = static_cast<int64_t>(sup[group[0]].size());
      int64_t deg_now = nnz_now;
      while (!remi.empty() && static_cast<int>(group.size()) < kMTile) {
        size_t best = 0;
        bool have = false;
        double b_util = 0.0;
        int64_t b_inter = 0, b_second = 0;
        for (size_t p = 0; p < remi.size(); ++p) {
          const auto& s = sup[remi[p]];
          int64_t inter = 0;
          for (int32_t c : s) inter += in_union[c];
          const int64_t sz = static_cast<int64_t>(s.size());
          if (policy == TSN_POLICY_OVERLAP) {
            const int64_t second = -(sz - inter);
            if (!have || inter > b_inter || (inter == b_inter && second > b_second)) {
              have = true;
              best = p;
              b_inter = inter;
              b_second = second;
            }
          } else {
            const int64_t comb = union_size + sz - inter;
            const int64_t tiles = std::max<int64_t>(
                std::max<int64_t>(ceil_div(comb, k_tile), ceil_div(std::max(deg_now, sz), k_tile / 2)), 1);
            const double util = static_cast<double>(nnz_now + sz) /
                                static_cast<double>(tiles * kMTile * k_tile / 2);
            const int64_t second = -comb;
            bool better;
            if (!have) better = true;
            else if (util != b_util) better = util > b_util;
            else if (inter != b_inter) better = inter > b_inter;
            else better = second > b_second;
            if (better) {
              have = true;
              best = p;
              b_util = util;
              b_inter = inter;
              b_second = second;
            }
          }
        }
        const int32_t chosen = remi[best];
        remi.erase(remi.begin() + static_cast<std::ptrdiff_t>(best));
        group.push_back(chosen);
        for (int32_t c : sup[chosen]) {
          if (!in_union[c]) {
            in_union[c] = 1;
            ++union_size;
          }
        }
        nnz_now += static_cast<int64_t>(sup[chosen].size());
        deg_now = std::max<int64_t>(deg_now, static_cast<int64_t>(sup[chosen].size()));
      }
      for (int32_t g : group) out[pos_out++] = rem[g];
    }
  });
  return out;
}

namespace {

struct Masks {
  std::vector<int64_t> cols;   // first-appearance order (dict insertion order)
  std::vector<uint32_t> mask;  // 16-bit row masks
};

Masks column_masks(const SparseView& v, const int64_t* local_rows) {
  Masks m;
  std::unordered_map<int64_t, int32_t> index;
  index.reserve(1024);
  for (int slot = 0; slot < kMTile; ++slot) {
    const int64_t r = local_rows[slot];
    if (r < 0) continue;
    for (int64_t k = v.row_ptr[r]; k < v.row_ptr[r + 1]; ++k) {
      auto it = index.find(v.cols[k]);
      if (it == index.end()) {
        index.emplace(v.cols[k], static_cast<int32_t>(m.cols.size()));
        m.cols.push_back(v.cols[k]);
        m.mask.push_back(1u << slot);
      } else {
        m.mask[it->second] |= 1u << slot;
      }
    }
  }
  return m;
}

inline int popcount16(uint32_t x) { return __builtin_popcount(x & 0xFFFFu); }

// sorted(columns, key=(-popcount, tie_break)) with the tie_break dict drawn in column order.
std::vector<int32_t> popcount_order(const std::vector<int32_t>& items, const Masks& m, PyRandom& rng) {
  std::vector<double> tie(items.size());
  for (size_t i = 0; i < items.size(); ++i) tie[i] = rng.random();
  std::vector<int32_t> idx(items.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = static_cast<int32_t>(i);
  std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) {
    const int pa = popcount16(m.mask[items[a]]), pb = popcount16(m.mask[items[b]]);
    if (pa != pb) return pa > pb;
    return tie[a] < tie[b];
  });
  std::vector<int32_t> out(items.size());
  for (size_t i = 0; i < idx.size(); ++i) out[i] = items[idx[i]];
  return out;
}

// returns lists of indices into m.cols
std::vector<std::vector<int32_t>> assign_columns(const Masks& m, int k_tile, uint64_t seed, bool optimized) {
  const int64_t n = static_cast<int64_t>(m.cols.size());
  if (n == 0) return {std::vector<int32_t>{}};
  int max_deg = 0;
  for (int r = 0; r < kMTile; ++r) {
    int d = 0;
    for (uint32_t x : m.mask) d += (x >> r) & 1u;
    max_deg = std::max(max_deg, d);
  }
  const int64_t min_tiles =
      std::max<int64_t>(std::max<int64_t>(ceil_div(n, k_tile), ceil_div(max_deg, k_tile / 2)), 1);
  std::vector<int32_t> items(n);
  for (int64_t i = 0; i < n; ++i) items[i] = static_cast<int32_t>(i);
  PyRandom rng(seed);
  const int restarts = optimized ? 8 : 24;
  const int half = k_tile / 2;
  for (int64_t tc = min_tiles; tc < min_tiles + 9; ++tc) {
    for (int restart = 0; restart < restarts; ++restart) {
      const std::vector<int32_t> ordered = popcount_order(items, m, rng);
      std::vector<std::vector<int32_t>> tiles(tc);
      std::vector<int32_t> counts(tc * kMTile, 0);
      std::vector<uint8_t> valid(tc);
      std::vector<int64_t> dsq(tc);
      bool ok = true;
      for (int32_t c : ordered) {
        const uint32_t mk = m.mask[c];
        bool any = false;
        for (int64_t t = 0; t < tc; ++t) {
          int32_t* cnt = &counts[t * kMTile];
          int mx = 0;
          int64_t ds = 0;
          for (int r = 0; r < kMTile; ++r) {
            const int b = (mk >> r) & 1u;
            const int u = cnt[r] + b;
            mx = std::max(mx, u);
            ds += static_cast<int64_t>(u) * u - static_cast<int64_t>(cnt[r]) * cnt[r];
          }
          dsq[t] = ds;
          valid[t] = static_cast<int64_t>(tiles[t].size()) < k_tile && mx <= half;
          any = any || valid[t];
        }
        int64_t best = -1;
        double best_score = std::numeric_limits<double>::infinity();
        if (optimized) {
          if (!any) {
            ok = false;
            break;
          }
          for (int64_t t = 0; t < tc; ++t) {
            double s = static_cast<double>(dsq[t]) +
                       static_cast<double>(tiles[t].size()) / static_cast<double>(k_tile);
            s = s + rng.random() * 1e-6;
            if (valid[t] && s < best_score) {
              best = t;
              best_score = s;
            }
          }
        } else {
          for (int64_t t = 0; t < tc; ++t) {
            if (!valid[t]) continue;
            double s = static_cast<double>(dsq[t]) +
                       static_cast<double>(tiles[t].size()) / static_cast<double>(k_tile);
            s = s + rng.random() * 1e-6;
            if (best < 0 || s < best_score) {
              best = t;
              best_score = s;
            }
          }
          if (best < 0) {
            ok = false;
            break;
          }
        }
        tiles[best].push_back(c);
        int32_t* cnt = &counts[best * kMTile];
        for (int r = 0; r < kMTile; ++r) cnt[r] += (mk >> r) & 1u;
      }
      if (ok) {
        std::vector<std::vector<int32_t>> out;
        for (auto& t : tiles)
          if (!t.empty()) out.push_back(std::move(t));
        return out;
      }
    }
  }
  fail(TSN_ERR_FORMAT, "failed to partition columns into half-density tiles");
}

// returns (arranged column ids (global, -1 pads), legal, violation)
std::vector<int64_t> arrange_24(const std::vector<int32_t>& cols, const Masks& m, int k_tile,
                                uint64_t seed, bool optimized, bool* legal, int32_t* violation) {
  if (static_cast<int>(cols.size()) > k_tile) fail(TSN_ERR_FORMAT, "too many columns for tile");
  const int ng = k_tile / 4;
  PyRandom rng(seed);
  const int restarts = optimized ? 16 : 64;
  for (int restart = 0; restart < restarts; ++restart) {
    const std::vector<int32_t> ordered = popcount_order(cols, m, rng);
    std::vector<std::vector<int32_t>> groups(ng);
    std::vector<int32_t> counts(ng * kMTile, 0);
    std::vector<uint8_t> valid(ng);
    std::vector<int32_t> overlap(ng);
    bool ok = true;
    for (int32_t c : ordered) {
      const uint32_t mk = m.mask[c];
      bool any = false;
      for (int g = 0; g < ng; ++g) {
        const int32_t* cnt = &counts[g * kMTile];
        int mx = 0, ov = 0;
        for (int r = 0; r < kMTile; ++r) {
          const int b = (mk >> r) & 1u;
          mx = std::max(mx, cnt[r] + b);
          ov += cnt[r] * b;
        }
        overlap[g] = ov;
        valid[g] = groups[g].size() < 4 && mx <= 2;
        any = any || valid[g];
      }
      int best = -1;
      double best_score = std::numeric_limits<double>::infinity();
      if (optimized) {
        if (!any) {
          ok = false;
          break;
        }
        for (int g = 0; g < ng; ++g) {
          double s = overlap[g] * 100.0 + static_cast<double>(groups[g].size());
          s = s + rng.random() * 1e-6;
          if (valid[g] && s < best_score) {
            best = g;
            best_score = s;
          }
        }
      } else {
        for (int g = 0; g < ng; ++g) {
          if (!valid[g]) continue;
          double s = overlap[g] * 100.0 + static_cast<double>(groups[g].size());
          s = s + rng.random() * 1e-6;
          if (best < 0 || s < best_score) {
            best = g;
            best_score = s;
          }
        }
        if (best < 0) {
          ok = false;
          break;
        }
      }
      groups[best].push_back(c);
      int32_t* cnt = &counts[best * kMTile];
      for (int r = 0; r < kMTile; ++r) cnt[r] += (mk >> r) & 1u;
    }
    if (!ok) continue;
    std::vector<int64_t> flat;
    flat.reserve(k_tile);
    for (auto& g : groups) {
      for (int32_t c : g) flat.push_back(m.cols[c]);
      for (size_t p = g.size(); p < 4; ++p) flat.push_back(-1);
    }
    *legal = true;
    *violation = 0;
    return flat;
  }
  std::vector<int64_t> padded;
  for (int32_t c : cols) padded.push_back(m.cols[c]);
  while (static_cast<int>(padded.size()) < k_tile) padded.push_back(-1);
  *legal = false;
  *violation = 0;
  if (!optimized) {
    std::unordered_map<int64_t, uint32_t> mk;
    for (size_t i = 0; i < m.cols.size(); ++i) mk[m.cols[i]] = m.mask[i];
    int32_t best = std::numeric_limits<int32_t>::max();
    for (int off = 0; off < k_tile; off += 4) {
      int32_t v = 0;
      for (int r = 0; r < kMTile; ++r) {
        int cnt = 0;
        for (int p = 0; p < 4; ++p) {
          const int64_t c = padded[off + p];
          if (c >= 0 && (mk[c] >> r) & 1u) ++cnt;
        }
        v += std::max(0, cnt - 2);
      }
      best = std::min(best, v);
    }
    *violation = best;
  }
  return padded;
}

void materialize(const SparseView& v, const int64_t* local_rows, const std::vector<int64_t>& arranged,
                 int k_tile, PackTile& t) {
  t.col_ids.assign(k_tile, -1);
  for (int j = 0; j < k_tile; ++j) t.col_ids[j] = static_cast<int32_t>(arranged[j]);
  t.values.assign(static_cast<size_t>(kMTile) * k_tile, 0.0);
  std::unordered_map<int64_t, int> where;
  for (int j = 0; j < k_tile; ++j)
    if (arranged[j] >= 0) where[arranged[j]] = j;
  for (int slot = 0; slot < kMTile; ++slot) {
    const int64_t r = local_rows[slot];
    t.row_ids[slot] = r >= 0 ? static_cast<int32_t>(v.row_ids[r]) : -1;
    if (r < 0) continue;
    // dict(zip(cols, vals)): a repeated column keeps its last value
    for (int64_t k = v.row_ptr[r]; k < v.row_ptr[r + 1]; ++k) {
      auto it = where.find(v.cols[k]);
      if (it != where.end()) t.values[static_cast<size_t>(slot) * k_tile + it->second] = v.vals[k];
    }
  }
}

// materialize for a tile whose column ids are an ascending run (then -1 pads), over rows whose
// CSR columns ascend without repeats: one binary search per row instead of a scan of the
// whole row (rows next to the centre of a 3D radial trajectory hold tens of thousands).
void materialize_run(const SparseView& v, const int64_t* local_rows, const std::vector<int64_t>& cols, int k_tile,
                     PackTile& t) {
  t.col_ids.assign(k_tile, -1);
  int nlive = 0;
  for (int j = 0; j < k_tile; ++j) {
    t.col_ids[j] = static_cast<int32_t>(cols[j]);
    if (cols[j] >= 0) nlive = j + 1;
  }
  t.values.assign(static_cast<size_t>(kMTile) * k_tile, 0.0);
  for (int slot = 0; slot < kMTile; ++slot) {
    const int64_t r = local_rows[slot];
    t.row_ids[slot] = r >= 0 ? static_cast<int32_t>(v.row_ids[r]) : -1;
    if (r < 0 || nlive == 0) continue;
    const int64_t* base = v.cols.data();
    const int64_t* it = std::lower_bound(base + v.row_ptr[r], base + v.row_ptr[r + 1], cols[0]);
    const int64_t* end = base + v.row_ptr[r + 1];
    int j = 0;
    while (it != end && j < nlive) {
      if (*it < cols[j]) {
        ++it;
      } else if (*it > cols[j]) {
        ++j;
      } else {
        t.values[static_cast<size_t>(slot) * k_tile + j] = v.vals[it - base];
        ++it;
        ++j;
      }
    }
  }
}

void split_illegal(const PackTile& t, PackTile& l0, PackTile& l1) {
  const int k = static_cast<int>(t.col_ids.size());
  l0 = t;
  l1 = t;
  std::fill(l0.values.begin(), l0.values.end(), 0.0);
  std::fill(l1.values.begin(), l1.values.end(), 0.0);
  for (int r = 0; r < kMTile; ++r) {
    for (int off = 0; off < k; off += 4) {
      int seen = 0;
      for (int p = 0; p < 4; ++p) {
        const double val = t.values[static_cast<size_t>(r) * k + off + p];
        if (val == 0.0) continue;
        (seen < 2 ? l0 : l1).values[static_cast<size_t>(r) * k + off + p] = val;
        ++seen;
      }
    }
  }
  l0.legal = l1.legal = true;
  l0.violation = l1.violation = 0;
  if (!legal_24(l0) || !legal_24(l1)) fail(TSN_ERR_FORMAT, "split24 failed to legalize a tile");
}

}  // namespace

bool legal_24(const PackTile& t, int* violations) {
  const int k = static_cast<int>(t.col_ids.size());
  int viol = 0;
  for (int r = 0; r < kMTile; ++r)
    for (int off = 0; off < k; off += 4) {
      int cnt = 0;
      for (int p = 0; p < 4; ++p) cnt += t.values[static_cast<size_t>(r) * k + off + p] != 0.0;
      viol += std::max(0, cnt - 2);
    }
  if (violations) *violations = viol;
  return viol == 0;
}

std::vector<PackTile> pack_view(const SparseView& v, int planner, int policy, int k_tile, uint64_t seed,
                                int threads) {
  if (k_tile <= 0 || k_tile % 4) fail(TSN_ERR_ARG, "k_tile must be a positive multiple of 4");
  if ((planner == TSN_PLANNER_FAST || planner == TSN_PLANNER_OPTIMIZED) && k_tile != kKTile)
    fail(TSN_ERR_ARG, "fast/optimized planners use K32 tiles");
  const std::vector<int64_t> order = row_order(v, policy, k_tile);
  const int64_t n_groups = ceil_div(static_cast<int64_t>(order.size()), kMTile);
  return pack_groups(v, order, 0, n_groups, planner, k_tile, seed, threads, 0);
}

std::vector<PackTile> pack_groups(const SparseView& v, const std::vector<int64_t>& order, int64_t g0,
                                  int64_t g1, int planner, int k_tile, uint64_t seed, int threads,
                                  int64_t fast_above) {
  std::vector<std::vector<PackTile>> per_group(std::max<int64_t>(g1 - g0, 0));
  parallel_for(g1 - g0, resolve_threads(threads), [&](int64_t li) {
    const int64_t gi = g0 + li;
    int64_t rows[kMTile];
    for (int s = 0; s < kMTile; ++s) {
      const int64_t at = gi * kMTile + s;
      rows[s] = at < static_cast<int64_t>(order.size()) ? order[at] : -1;
    }
    auto& out = per_group[li];
    const uint64_t gseed = seed + static_cast<uint64_t>(gi) * 1009u;
    const bool optimized = planner == TSN_PLANNER_OPTIMIZED;
    const Masks m = (planner == TSN_PLANNER_FAST) ? Masks{} : column_masks(v, rows);
    if (planner == TSN_PLANNER_FAST ||
        (optimized && fast_above > 0 && static_cast<int64_t>(m.cols.size()) > fast_above)) {
      std::vector<int64_t> uni;
      for (int s = 0; s < kMTile; ++s)
        if (rows[s] >= 0)
          for (int64_t k = v.row_ptr[rows[s]]; k < v.row_ptr[rows[s] + 1]; ++k) uni.push_back(v.cols[k]);
      std::sort(uni.begin(), uni.end());
      uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
      for (size_t off = 0; off < uni.size(); off += kKTile) {
        std::vector<int64_t> cols(kKTile, -1);
        for (size_t j = 0; j < kKTile && off + j < uni.size(); ++j) cols[j] = uni[off + j];
        PackTile t;
        if (fast_above > 0) materialize_run(v, rows, cols, kKTile, t);
        else materialize(v, rows, cols, kKTile, t);
        t.legal = legal_24(t);
        if (t.legal) {
          out.push_back(std::move(t));
        } else {
          PackTile a, b;
          split_illegal(t, a, b);
          out.push_back(std::move(a));
          out.push_back(std::move(b));
        }
      }
      return;
    }
    const auto tiles = assign_columns(m, k_tile, gseed, optimized);
    for (size_t ti = 0; ti < tiles.size(); ++ti) {
      bool legal = true;
      int32_t viol = 0;
      const auto arranged = arrange_24(tiles[ti], m, k_tile, gseed + static_cast<uint64_t>(ti) * 9176u,
                                       optimized, &legal, &viol);
      PackTile t;
      materialize(v, rows, arranged, k_tile, t);
      t.legal = legal;
      t.violation = viol;
      if (optimized && !legal) {
        PackTile a, b;
        split_illegal(t, a, b);
        out.push_back(std::move(a));
        out.push_back(std::move(b));
      } else {
        out.push_back(std::move(t));
      }
    }
  });
  std::vector<PackTile> all;
  size_t total = 0;
  for (auto& g : per_group) total += g.size();
  all.reserve(total);
  for (auto& g : per_group)
    for (auto& t : g) all.push_back(std::move(t));
  return all;
}

GroupedTiles split_legal_and_residual(const SparseView& v, const std::vector<PackTile>& tiles, int illegal_mode) {
  GroupedTiles g;
  g.group_offsets.push_back(0);
  std::vector<std::vector<std::pair<int32_t, double>>> residual(static_cast<size_t>(v.output_size));
  bool have_prev = false;
  int32_t prev[kMTile];
  for (const auto& t : tiles) {
    if (!have_prev || std::memcmp(prev, t.row_ids, sizeof prev) != 0) {
      if (have_prev) g.group_offsets.push_back(static_cast<uint32_t>(g.tiles.size()));
      g.group_row_ids.insert(g.group_row_ids.end(), t.row_ids, t.row_ids + kMTile);
      std::memcpy(prev, t.row_ids, sizeof prev);
      have_prev = true;
    }
    if (legal_24(t)) {
      g.tiles.push_back(t);
    } else if (illegal_mode == TSN_ILLEGAL_SPLIT24) {
      PackTile a, b;
      split_illegal(t, a, b);
      g.tiles.push_back(std::move(a));
      g.tiles.push_back(std::move(b));
    } else {
      const int k = static_cast<int>(t.col_ids.size());
      for (int s = 0; s < kMTile; ++s) {
        if (t.row_ids[s] < 0) continue;
        for (int j = 0; j < k; ++j) {
          const double val = t.values[static_cast<size_t>(s) * k + j];
          if (t.col_ids[j] >= 0 && val != 0.0) residual[t.row_ids[s]].emplace_back(t.col_ids[j], val);
        }
      }
    }
  }
  g.group_offsets.push_back(static_cast<uint32_t>(g.tiles.size()));
  g.residual_row_ptr.assign(static_cast<size_t>(v.output_size) + 1, 0);
  for (int64_t r = 0; r < v.output_size; ++r) {
    g.residual_row_ptr[r + 1] = g.residual_row_ptr[r] + static_cast<uint32_t>(residual[r].size());
    for (auto& e : residual[r]) {
      g.residual_cols.push_back(e.first);
      g.residual_vals.push_back(f64_to_f16_bits(e.second));
    }
  }
  return g;
}

std::vector<PackTile> component_tiles(const std::vector<PackTile>& structure, const SparseView& comp) {
  std::unordered_map<int64_t, int64_t> lookup;
  lookup.reserve(comp.row_ids.size() * 2);
  for (int64_t i = 0; i < comp.rows(); ++i) lookup[comp.row_ids[i]] = i;
  std::vector<PackTile> out(structure.size());
  for (size_t ti = 0; ti < structure.size(); ++ti) {
    const PackTile& st = structure[ti];
    PackTile& t = out[ti];
    std::memcpy(t.row_ids, st.row_ids, sizeof t.row_ids);
    t.col_ids = st.col_ids;
    const int k = static_cast<int>(st.col_ids.size());
    t.values.assign(st.values.size(), 0.0);
    for (int s = 0; s < kMTile; ++s) {
      if (st.row_ids[s] < 0) continue;
      auto it = lookup.find(st.row_ids[s]);
      if (it == lookup.end()) fail(TSN_ERR_FORMAT, "structure row missing from component");
      const int64_t r = it->second;
      for (int j = 0; j < k; ++j) {
        if (st.col_ids[j] < 0 || st.values[static_cast<size_t>(s) * k + j] == 0.0) continue;
        double val = 0.0;  // row_map.get(col, 0.0), last duplicate wins
        for (int64_t q = comp.row_ptr[r]; q < comp.row_ptr[r + 1]; ++q)
          if (comp.cols[q] == st.col_ids[j]) val = comp.vals[q];
        t.values[static_cast<size_t>(s) * k + j] = val;
      }
    }
    t.legal = true;
    if (!legal_24(t)) fail(TSN_ERR_FORMAT, "materialized component is not legal 2:4");
  }
  return out;
}

uint32_t pair_word(const uint32_t* rm, int word) {
  const int g = word / 2;
  const uint32_t a = rm[g], b = rm[g + 8];
  return (word & 1) ? ((a >> 16) | (b & 0xFFFF0000u)) : ((a & 0xFFFFu) | ((b & 0xFFFFu) << 16));
}

CompressedTiles compress_tiles(const std::vector<PackTile>& tiles) {
  CompressedTiles c;
  const size_t n = tiles.size();
  c.values.assign(n * kMTile * (kKTile / 2), 0);
  c.row_meta.assign(n * kMTile, 0);
  c.pair_meta.assign(n * kMTile, 0);
  c.col_ids.assign(n * kKTile, 0);
  for (size_t ti = 0; ti < n; ++ti) {
    const PackTile& t = tiles[ti];
    if (t.col_ids.size() != static_cast<size_t>(kKTile)) fail(TSN_ERR_FORMAT, "compression needs K32 tiles");
    for (int j = 0; j < kKTile; ++j) c.col_ids[ti * kKTile + j] = t.col_ids[j] < 0 ? 0 : t.col_ids[j];
    for (int r = 0; r < kMTile; ++r) {
      uint32_t word = 0;
      for (int q = 0; q < kKTile / 4; ++q) {
        uint16_t h[4];
        int nz[4], nnz = 0;
        for (int p = 0; p < 4; ++p) {
          h[p] = f64_to_f16_bits(t.values[static_cast<size_t>(r) * kKTile + 4 * q + p]);
          if (f16_bits_nonzero(h[p])) nz[nnz++] = p;
        }
        if (nnz > 2) fail(TSN_ERR_FORMAT, "tile is not legal 2:4 after FP16 rounding");
        int sel[2], ns = 0;
        for (int i = 0; i < nnz; ++i) sel[ns++] = nz[i];
        for (int p = 0; p < 4 && ns < 2; ++p) {
          bool used = false;
          for (int i = 0; i < ns; ++i) used = used || sel[i] == p;
          if (!used) sel[ns++] = p;
        }
        if (sel[0] > sel[1]) std::swap(sel[0], sel[1]);
        c.values[(ti * kMTile + r) * (kKTile / 2) + 2 * q] = h[sel[0]];
        c.values[(ti * kMTile + r) * (kKTile / 2) + 2 * q + 1] = h[sel[1]];
        word |= static_cast<uint32_t>(sel[0] | (sel[1] << 2)) << (4 * q);
      }
      c.row_meta[ti * kMTile + r] = word;
    }
    for (int w = 0; w < kMTile; ++w) c.pair_meta[ti * kMTile + w] = pair_word(&c.row_meta[ti * kMTile], w);
  }
  return c;
}

std::string header_bytes(uint32_t output_size, uint32_t n_cols, uint32_t active_rows, uint32_t nnz,
                         uint32_t groups, uint32_t tiles, uint32_t residual_nnz) {
  std::string s(52, '\0');
  const uint32_t f[11] = {kPackVersion, kPackChannels, output_size, n_cols, active_rows, nnz,
                          groups,       tiles,         residual_nnz, kMTile, kKTile};
  std::memcpy(&s[0], &kPackMagic, 8);
  std::memcpy(&s[8], f, sizeof f);
  return s;
}

PackHeader parse_header(const std::string& bytes) {
  if (bytes.size() != 52) fail(TSN_ERR_FORMAT, "packed header must be 52 bytes");
  PackHeader h{};
  std::memcpy(&h.magic, bytes.data(), 8);
  uint32_t f[11];
  std::memcpy(f, bytes.data() + 8, sizeof f);
  h.version = f[0];
  h.n_channels = f[1];
  h.output_size = f[2];
  h.n_cols = f[3];
  h.active_rows = f[4];
  h.nnz = f[5];
  h.groups = f[6];
  h.tiles = f[7];
  h.residual_nnz = f[8];
  h.m_tile = f[9];
  h.k_tile = f[10];
  if (h.magic != kPackMagic || h.version != kPackVersion || h.n_channels != kPackChannels ||
      h.m_tile != kMTile || h.k_tile != kKTile)
    fail(TSN_ERR_FORMAT, "unsupported input header");
  return h;
}

}  // namespace tsn
