// sm_100a kernels of the NUFFT CG-SENSE operator pipeline.
//
// Data layouts in HBM (internal; the C ABI converts at its edges):
//   grid panel    [G*G][4C] f16, row q1*G + q0 (q1-major), per row hi(2C) | res(2C),
//                 complex interleaved per coil (re, im)
//   sample panel  [M][4C] f16, same row format
//   grid          [G*G][C] c64, row q1*G + q0
//   z1 / w1       [G][N][C] c64 (one FFT axis done)
//   CG vectors    [N][N] c64 FP32, scalars FP64 (CgState)
// The reference's equivalents are the N16 panels of nufft_integrated_bench.cu:339-359 and
// the coil-major grids of nufft_custom_fft_forward_bench.cu:538-747; here every stage
// reads and writes contiguous slabs and the panel row carries hi and res together so one
// gather feeds both sparse MMAs.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cmath>

#include "fft.cuh"
#include "kernels.cuh"

namespace tsn {

using namespace dev;

// The warp interpolation is launched with programmatic stream serialization: its CTAs start
// (launch, shared-memory carve-up, the first plan-record copies) while the kernel ahead of it
// in the stream drains, and wait in pdl_wait before touching its results. Every kernel of the
// CG iteration calls pdl_trigger once it has passed its own wait, so the interpolation behind
// it may launch then. On the 256^2 / 8-coil headline solve this took a CG iteration from 71.8
// to 69.5 us. Batched cases, whose kernels run side by side on slices of the GPU, launch it
// plainly: early CTAs would wait beside the other cases' kernels (the 48-case batch measured
// 1191 recons/s with it, 1325-1390 without it on other boxes; 1329 plain vs 1325 with every
// launch plain on one box). The FFT stages are launched plainly: their CTAs, started early beside a kernel
// that leaves room on the SMs (the row stages hold ~1.7 of 3 CTAs per SM; the interpolation
// leaves room for one more), made the solve 3-9% slower although each stage timed alone
// back to back got faster. They keep the same prologue split (plan rows before pdl_wait) for
// when they are. TSN_PDL=0 in the environment launches everything plainly (same results,
// bit for bit).
static bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("TSN_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename... KArgs, typename... Args>
static void launch_k(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, bool programmatic,
                     Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(static_cast<unsigned>(grid));
  cfg.blockDim = dim3(static_cast<unsigned>(block));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = programmatic && pdl_enabled() ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

void set_twiddle_constants(cudaStream_t s) {
  std::vector<float2> w(1024);
  for (int e = 0; e < 1024; ++e) {
    const double a = -2.0 * M_PI * e / 1024.0;
    w[e] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  cudaMemcpyToSymbolAsync(dev::c_w1024, w.data(), sizeof(float2) * 1024, 0, cudaMemcpyHostToDevice, s);
  // W_R^j with the plan tables' expression (-2 pi e) / G at e = B j, G = R B: for a power-of-two
  // B that is exactly (-2 pi j) / R, so these equal the plans' tw[B j]
  float2 w3[3], w5[5];
  for (int j = 0; j < 3; ++j) {
    const double a = -2.0 * M_PI * j / 3.0;
    w3[j] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  for (int j = 0; j < 5; ++j) {
    const double a = -2.0 * M_PI * j / 5.0;
    w5[j] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  cudaMemcpyToSymbolAsync(dev::c_wr3, w3, sizeof w3, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(dev::c_wr5, w5, sizeof w5, 0, cudaMemcpyHostToDevice, s);
  cudaStreamSynchronize(s);
}

// ------------------------------------------------------------------------------------------
// Sparse interpolation: one warp per 16-row group, 2:4 tiles through mma.sp m16n8k32.
// Per tile the 32 gathered panel rows (hi and res together) are brought to shared memory
// with 16-byte cp.async through a per-warp ring, swizzled so ldmatrix.trans is
// conflict-free; dead (padding) columns are zero-stored and never read.
// Reference: nufft_gt_spmma_complex_fused_f16_f32 (nufft_spmma_bench.cu:402-663), which
// gathers B with 2-byte loads and reduces 4 warps through shared memory.
// ------------------------------------------------------------------------------------------
template <int CH>
__device__ __forceinline__ int chunk_swizzle(int ch, int row) {
  if constexpr (CH == 2 || CH == 6) return ch ^ ((row >> 2) & 1);
  else if constexpr (CH == 4) return ch ^ ((row >> 1) & 3);
  else if constexpr (CH == 8) return ch ^ (row & 7);
  else return ch;
}

constexpr int kInterpWarps = 4;

// Output row s (0..15) of a record: 24-bit little-endian fields; -1 for a pad row (live bit
// 16 + s of the record flags clear), so every one of the 2^24 row indices is addressable.
__device__ __forceinline__ int32_t record_row(const uint8_t* rows24, int32_t flags, int s) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(rows24);
  const int bit = 24 * s, off = bit & 31;
  const uint32_t lo = w[bit >> 5];
  const uint32_t hi = off > 8 ? w[(bit >> 5) + 1] : 0u;  // stays inside the 48-byte field
  const uint32_t v = __funnelshift_r(lo, hi, off) & 0xFFFFFFu;
  return ((static_cast<uint32_t>(flags) >> (kRecLiveShift + s)) & 1u) ? static_cast<int32_t>(v) : -1;
}

// Per-warp shared-memory ring: stage = tile record (cols, A, meta) + 32 gathered panel rows.
// Records are fetched kRecAhead tiles ahead, gathers kGatherAhead tiles ahead (the gather
// needs the record's column ids), so a warp waits only on cp.async groups, never on a
// register load.  Warps are persistent: each streams a contiguous, tile-balanced run of
// work items and the pipeline runs across item boundaries.  The ring depth STAGES is per
// view (InterpView::stages): three stages (34 KB per 4-warp CTA, 24 warps per SM) when the
// gathered panel sits in L2, which measured faster than deeper rings with fewer warps;
// four stages (45 KB, 20 warps per SM, records one tile further ahead) when it does not and
// gathers wait on DRAM (3D grids: 1.33 vs 1.79 ms per forward launch).  Records run
// STAGES - 1 tiles ahead, gathers kGatherAhead.
constexpr int kGatherAhead = 1;

// Writes one finished item: split chunks publish their accumulators and the last chunk of
// the group reduces all chunks in chunk order; whole groups and finishing chunks apply the
// epilogue.
template <int ROWH, int NCOMP, int NA, int EPI, bool CONJ, bool SUMC>
__device__ __forceinline__ void interp_finish_item(float (&acc)[NCOMP][NA][4], const InterpView& v,
                                                   const InterpOut& o, const RecordInfo& info, int lane,
                                                   const int32_t (&rows)[2], const float (&wrow)[2], float scale) {
  const int t = lane & 3;
  if (info.split >= 0) {
    const int split = info.split;
    const int chunk = info.chunk & 0xFFFF, nchunks = info.chunk >> 16;
    float* mine = v.partials + static_cast<size_t>(info.first_slot + chunk) * kPartialFloats * 32;
#pragma unroll
    for (int c = 0; c < NCOMP; ++c)
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
        for (int i = 0; i < 4; ++i) mine[((c * NA + a2) * 4 + i) * 32 + lane] = acc[c][a2][i];
    __threadfence();
    __syncwarp();
    int prior = 0;
    if (lane == 0) prior = atomicAdd(&v.counters[split], 1);
    prior = __shfl_sync(0xFFFFFFFFu, prior, 0);
    if (prior != nchunks - 1) return;
    __threadfence();
#pragma unroll
    for (int c = 0; c < NCOMP; ++c)
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[c][a2][i] = 0.f;
    for (int k = 0; k < nchunks; ++k) {
      const float* src = v.partials + static_cast<size_t>(info.first_slot + k) * kPartialFloats * 32;
#pragma unroll
      for (int c = 0; c < NCOMP; ++c)
#pragma unroll
        for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[c][a2][i] += __ldcg(src + ((c * NA + a2) * 4 + i) * 32 + lane);
    }
    if (lane == 0) v.counters[split] = 0;  // ready for the next launch
  }
  if constexpr (EPI == EPI_RAW) {
#pragma unroll
    for (int hr = 0; hr < 2; ++hr) {
      if (rows[hr] < 0) continue;
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2) {
        float2 val = make_float2(acc[0][a2][2 * hr] * scale, acc[0][a2][2 * hr + 1] * scale);
        *reinterpret_cast<float2*>(o.raw + static_cast<size_t>(rows[hr]) * ROWH + 8 * a2 + 2 * t) = val;
      }
    }
  } else {
    const int C = o.coils;
#pragma unroll
    for (int hr = 0; hr < 2; ++hr) {
      const int32_t row = rows[hr];
      if (row < 0) continue;
      const float w = scale * wrow[hr];
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2) {
        const int coil = 4 * a2 + t;
        float re = acc[0][a2][2 * hr], im = acc[0][a2][2 * hr + 1];
        if constexpr (NCOMP == 2 && SUMC) {  // real coefficients split into FP16 high + low parts
          re += acc[1][a2][2 * hr];
          im += acc[1][a2][2 * hr + 1];
        } else if constexpr (NCOMP == 2) {
          const float qre = acc[1][a2][2 * hr], qim = acc[1][a2][2 * hr + 1];
          if (CONJ) {
            re = re + qim;
            im = im - qre;
          } else {
            re = re - qim;
            im = im + qre;
          }
        }
        re *= w;
        im *= w;
        if constexpr (EPI == EPI_SAMPLES) {
          o.c64[static_cast<size_t>(coil) * o.rows + row] = make_float2(re, im);
        } else if constexpr (EPI == EPI_GRID) {
          o.c64[static_cast<size_t>(row) * C + coil] = make_float2(re, im);
        } else {
          uint32_t hw, rw;
          split_hi_res2(re, im, hw, rw);
          uint32_t* rowp = reinterpret_cast<uint32_t*>(o.panel + static_cast<size_t>(row) * ROWH);
          rowp[coil] = hw;
          rowp[C + coil] = rw;
        }
      }
    }
  }
}

template <int ROWH, bool SPLIT, int NCOMP, int EPI, bool CONJ, int STAGES, bool SUMC = false>
__global__ void __launch_bounds__(kInterpWarps * 32) interp_mmasp_kernel(InterpView v, const __half* __restrict__ panel,
                                                                         InterpOut o) {
  constexpr int kStages = STAGES;
  constexpr int kRecAhead = STAGES - 1;
  constexpr int BYTES = ROWH * 2;
  constexpr int CH = BYTES / 16;
  constexpr int NB = ROWH / 8;
  constexpr int NA = SPLIT ? NB / 2 : NB;
  constexpr int NACC = NCOMP * NA * 4;
  constexpr int INFO = 128 + 576 * NCOMP;         // RecordInfo offset in the record
  constexpr int REC = record_bytes(NCOMP);        // record bytes (all staged)
  constexpr int STAGE = REC + 32 * BYTES;
  constexpr unsigned FULL = 0xFFFFFFFFu;
  static_assert(NACC <= kPartialFloats, "partials slot too small");
  static_assert(REC % 16 == 0 && STAGE % 16 == 0, "16-byte stages");
  static_assert(kGatherAhead >= 1 && kRecAhead > kGatherAhead && kStages == kRecAhead + 1, "ring arithmetic");
  extern __shared__ __align__(128) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wid = blockIdx.x * kInterpWarps + warp;
  if (wid >= v.n_warps) return;
  const int2 range = v.warp_ranges[wid];
  const int n = range.y - range.x;
  const uint8_t* recs = v.records + static_cast<size_t>(range.x) * REC;
  uint8_t* ring = smem + warp * kStages * STAGE;
  const uint8_t* pb = reinterpret_cast<const uint8_t*>(panel);
  const int g = lane >> 2;
  float scale = o.scale_mul;
  // records are plan data: their first copies stream in while the preceding kernel drains;
  // the panel, the scale and every output wait for it
  bool dep_ready = false;
  auto wait_dep = [&]() {
    if (dep_ready) return;
    pdl_wait();
    pdl_trigger();
    dep_ready = true;
    if (o.scale_ptr) {
      const float sp = *o.scale_ptr;
      scale *= o.scale_inv ? 1.0f / sp : sp;
    }
  };
  float wrow[2] = {1.f, 1.f};  // density of the open item's rows (EPI_PANEL)

  float acc[NCOMP][NA][4];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c)
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[c][a][i] = 0.f;

  // Per-lane gather constants: chunk i of this lane is 16-byte chunk (lane + 32 i) % CH of
  // gathered row (lane + 32 i) / CH; its swizzled shared offset and source byte offset.
  int g_row[CH];
  uint32_t g_dst[CH], g_src[CH];
#pragma unroll
  for (int i = 0; i < CH; ++i) {
    const int ci = lane + 32 * i;
    const int row = ci / CH, ch = ci % CH;
    g_row[i] = row;
    g_dst[i] = static_cast<uint32_t>(REC + row * BYTES + chunk_swizzle<CH>(ch, row) * 16);
    g_src[i] = static_cast<uint32_t>(ch * 16);
  }
  // k-th record of this warp -> ring stage st
  auto issue_record = [&](int k, uint8_t* st) {
    if (k < n) {
      const uint8_t* src = recs + static_cast<size_t>(k) * REC;
#pragma unroll
      for (int c0 = 0; c0 < REC / 16; c0 += 32)
        if (c0 + 32 <= REC / 16 || lane < REC / 16 - c0) cp_async16(st + 16 * (c0 + lane), src + 16 * (c0 + lane));
    }
    cp_async_commit();  // empty groups keep the group arithmetic uniform
  };
  auto issue_gather = [&](int k, uint8_t* st) {
    if (k >= 0 && k < n) {
      wait_dep();
      const int32_t col = reinterpret_cast<const int32_t*>(st)[lane];
#pragma unroll
      for (int i = 0; i < CH; ++i) {
        const int src = __shfl_sync(FULL, col, g_row[i]);
        cp_async16_or_zero(st + g_dst[i], pb + static_cast<size_t>(static_cast<uint32_t>(max(src, 0)) * BYTES) + g_src[i],
                           src >= 0);
      }
    }
    cp_async_commit();
  };
  auto compute = [&](uint8_t* st) {
    wait_dep();
    const RecordInfo info = *reinterpret_cast<const RecordInfo*>(st + INFO);
    const uint8_t* trow = st + INFO + 16;
    if constexpr (EPI == EPI_PANEL) {  // density weights at the item's first tile
      if (o.density && (info.flags & kRecFirst)) {
        const int32_t r0 = record_row(trow, info.flags, g), r1 = record_row(trow, info.flags, g + 8);
        wrow[0] = r0 >= 0 ? __ldg(o.density + r0) : 1.f;
        wrow[1] = r1 >= 0 ? __ldg(o.density + r1) : 1.f;
      }
    }
    uint32_t a[NCOMP][4], meta[NCOMP];
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
      // A rows of 32 B; the 16-B halves of row r are stored swapped when (r >> 2) & 1
      const int r = (lane & 7) + ((lane >> 3) & 1) * 8;
      const int half = lane >> 4;
      ldmatrix_x4(a[c], st + 128 + 576 * c + r * 32 + ((half ^ ((r >> 2) & 1)) * 16));
      meta[c] = reinterpret_cast<const uint32_t*>(st + 640 + 576 * c)[g * 2 + (lane & 1)];
    }
    const uint8_t* B = st + REC;
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
      uint32_t b[4];
      ldmatrix_x4_trans(b, B + lane * BYTES + chunk_swizzle<CH>(nb, lane) * 16);
      const int ai = SPLIT ? (nb % NA) : nb;
#pragma unroll
      for (int c = 0; c < NCOMP; ++c) mma_sp_16832(acc[c][ai], a[c], b, meta[c]);
    }
    int32_t rows[2] = {-1, -1};
    if (info.flags & kRecLast) {
      rows[0] = record_row(trow, info.flags, g);
      rows[1] = record_row(trow, info.flags, g + 8);
    }
    __syncwarp();  // this stage is refilled by the next iteration's record copy
    if (info.flags & kRecLast) {  // last tile of its item
      interp_finish_item<ROWH, NCOMP, NA, EPI, CONJ, SUMC>(acc, v, o, info, lane, rows, wrow, scale);
#pragma unroll
      for (int c = 0; c < NCOMP; ++c)
#pragma unroll
        for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[c][a2][i] = 0.f;
    }
  };
  // Iterations k = -kRecAhead .. n-1, two commit groups each (empty when out of range):
  // rec(k + R) then gat(k + Ga), with R = kRecAhead, Ga = kGatherAhead.  Tile k lives in
  // stage (k + R) % kStages; unrolling by kStages makes every stage address a constant.
  // After committing rec(k + R), the groups newer than rec(k + Ga) are gat(k + 2Ga - R)
  // and the 2(R - Ga) - 1 groups of the later iterations, so wait<2(R - Ga)> lands the
  // record the next gather reads; after committing gat(k + Ga), wait<2 Ga> lands gat(k).
  for (int k0 = -kRecAhead; k0 < n; k0 += kStages) {
#pragma unroll
    for (int u = 0; u < kStages; ++u) {
      const int k = k0 + u;
      if (k >= n) break;
      issue_record(k + kRecAhead, ring + ((u + kRecAhead) % kStages) * STAGE);
      cp_async_wait<2 * (kRecAhead - kGatherAhead)>();
      __syncwarp();
      issue_gather(k + kGatherAhead, ring + ((u + kGatherAhead) % kStages) * STAGE);
      cp_async_wait<2 * kGatherAhead>();
      __syncwarp();
      if (k >= 0) compute(ring + u * STAGE);
    }
  }
  cp_async_wait<0>();
}

template <int ROWH, bool SPLIT, int NCOMP, int EPI, bool CONJ, int STAGES, bool SUMC = false>
static void launch_interp_s(const InterpView& v, const __half* panel, const InterpOut& o, cudaStream_t s) {
  const int blocks = (v.n_warps + kInterpWarps - 1) / kInterpWarps;
  const size_t smem = static_cast<size_t>(kInterpWarps) * STAGES * (record_bytes(NCOMP) + 32 * ROWH * 2);
  auto k = interp_mmasp_kernel<ROWH, SPLIT, NCOMP, EPI, CONJ, STAGES, SUMC>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (blocks > 0) launch_k(k, blocks, kInterpWarps * 32, smem, s, v.programmatic != 0, v, panel, o);
}

template <int ROWH, bool SPLIT, int NCOMP, int EPI, bool CONJ, bool SUMC = false>
static void launch_interp_t(const InterpView& v, const __half* panel, const InterpOut& o, cudaStream_t s) {
  if (v.stages == 4) launch_interp_s<ROWH, SPLIT, NCOMP, EPI, CONJ, 4, SUMC>(v, panel, o, s);
  else launch_interp_s<ROWH, SPLIT, NCOMP, EPI, CONJ, 3, SUMC>(v, panel, o, s);
}

template <int ROWH>
static void dispatch_epi(const InterpView& v, const __half* panel, int epi, bool conj, const InterpOut& o, cudaStream_t s) {
  if (v.sum_components) {  // FP16 high + low coefficient parts of a real pack
    if (epi == EPI_PANEL) launch_interp_t<ROWH, true, 2, EPI_PANEL, false, true>(v, panel, o, s);
    else if (epi == EPI_GRID) launch_interp_t<ROWH, true, 2, EPI_GRID, false, true>(v, panel, o, s);
    else launch_interp_t<ROWH, true, 2, EPI_SAMPLES, false, true>(v, panel, o, s);
    return;
  }
  if (v.ncomp == 2) {
    if (epi == EPI_SAMPLES) conj ? launch_interp_t<ROWH, true, 2, EPI_SAMPLES, true>(v, panel, o, s)
                                 : launch_interp_t<ROWH, true, 2, EPI_SAMPLES, false>(v, panel, o, s);
    else if (epi == EPI_PANEL) launch_interp_t<ROWH, true, 2, EPI_PANEL, false>(v, panel, o, s);
    else launch_interp_t<ROWH, true, 2, EPI_GRID, true>(v, panel, o, s);
  } else {
    if (epi == EPI_SAMPLES) launch_interp_t<ROWH, true, 1, EPI_SAMPLES, false>(v, panel, o, s);
    else if (epi == EPI_PANEL) launch_interp_t<ROWH, true, 1, EPI_PANEL, false>(v, panel, o, s);
    else launch_interp_t<ROWH, true, 1, EPI_GRID, false>(v, panel, o, s);
  }
}

static int sm_count();

template <int ROWH, int NCOMP, int STAGES>
static int resident_warps_s() {
  const size_t smem = static_cast<size_t>(kInterpWarps) * STAGES * (record_bytes(NCOMP) + 32 * ROWH * 2);
  auto k = interp_mmasp_kernel<ROWH, true, NCOMP, EPI_GRID, NCOMP == 2, STAGES>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kInterpWarps * 32, smem);
  return std::max(1, per_sm) * kInterpWarps * sm_count();
}

template <int ROWH, int NCOMP>
static int resident_warps_t(int stages) {
  return stages == 4 ? resident_warps_s<ROWH, NCOMP, 4>() : resident_warps_s<ROWH, NCOMP, 3>();
}

int interp_resident_warps(int rowh, int ncomp, int stages) {
  switch (rowh * 4 + ncomp) {
    case 16 * 4 + 1: return resident_warps_t<16, 1>(stages);
    case 16 * 4 + 2: return resident_warps_t<16, 2>(stages);
    case 32 * 4 + 1: return resident_warps_t<32, 1>(stages);
    case 32 * 4 + 2: return resident_warps_t<32, 2>(stages);
    case 48 * 4 + 1: return resident_warps_t<48, 1>(stages);
    case 48 * 4 + 2: return resident_warps_t<48, 2>(stages);
    case 64 * 4 + 1: return resident_warps_t<64, 1>(stages);
    default: return resident_warps_t<64, 2>(stages);
  }
}

void launch_interp(const InterpView& v, const __half* panel, int rowh, bool split, int epi, bool conj,
                   const InterpOut& o, cudaStream_t s) {
  if (!split) {  // raw single-component product for the reference.bin gate (16 channels)
    launch_interp_t<16, false, 1, EPI_RAW, false>(v, panel, o, s);
    return;
  }
  switch (rowh) {
    case 16: dispatch_epi<16>(v, panel, epi, conj, o, s); break;
    case 32: dispatch_epi<32>(v, panel, epi, conj, o, s); break;
    case 48: dispatch_epi<48>(v, panel, epi, conj, o, s); break;
    case 64: dispatch_epi<64>(v, panel, epi, conj, o, s); break;
    default: break;
  }
}

// ------------------------------------------------------------------------------------------
// Reductions
// ------------------------------------------------------------------------------------------
__global__ void norm_partials_kernel(const float2* __restrict__ v, int64_t n, double* __restrict__ part) {
  __shared__ double scratch[33];
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 x = v[i];
    acc += static_cast<double>(x.x) * x.x + static_cast<double>(x.y) * x.y;
  }
  const double t = block_sum(acc, scratch);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

void launch_norm_partials(const float2* v, int64_t n, double* part, cudaStream_t s) {
  norm_partials_kernel<<<kNormParts, 256, 0, s>>>(v, n, part);
}

// Sum of nparts partials, identical (fixed tree) in every block. Call with all threads.
__device__ __forceinline__ double sum_partials(const double* part, int nparts, double* scratch) {
  double a = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) a += part[i];
  return block_sum(a, scratch);
}

// Sums of four partial sections [nparts] spaced `stride` apart, as sum_partials does each.
__device__ __forceinline__ double4 sum_partials4(const double* part, int nparts, int64_t stride, double* scratch) {
  double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    a += part[i];
    b += part[stride + i];
    c += part[2 * stride + i];
    d += part[3 * stride + i];
  }
  return block_sum4(a, b, c, d, scratch);
}

// ------------------------------------------------------------------------------------------
// FFT endpoints. One warp per coil (blockDim = 32*C), one CTA per image row / grid column.
// ------------------------------------------------------------------------------------------
template <int G>
struct FftSmem {
  static constexpr int SCR = FftPlan<G>::SCRATCH;
};

// Copy `bytes` (multiple of 16) from global to shared with 16-byte cp.async, all threads.
__device__ __forceinline__ void cp_async_bytes(void* dst, const void* src, int bytes) {
  uint8_t* d = static_cast<uint8_t*>(dst);
  const uint8_t* q = static_cast<const uint8_t*>(src);
  for (int i = threadIdx.x * 16; i < bytes; i += blockDim.x * 16) cp_async16(d + i, q + i);
}

// [rows][C] complex slabs in shared memory hold each row's C/2 16-byte chunks XOR-swizzled
// by the row index, so a warp reading one coil down 32 consecutive rows touches distinct
// banks (unswizzled, 64-byte rows make that a 16-way conflict).
__device__ __forceinline__ int slab_swz(int n, int chn) {
  return chn == 2 ? (n >> 2) & 1 : chn == 4 ? (n >> 1) & 3 : chn == 8 ? (n & 7) : 0;
}
__device__ __forceinline__ int slab_idx(int n, int c, int C) {
  return n * C + 2 * ((c >> 1) ^ slab_swz(n, C >> 1)) + (c & 1);
}
// copy `rows` contiguous rows of C complex values into a swizzled slab (all threads; the
// block has 32*C threads, so every thread keeps one 16-byte chunk column, 64 rows apart)
__device__ __forceinline__ void cp_async_slab(float2* dst, const float2* src, int rows, int C) {
  const int chn = C >> 1;
  const int k = threadIdx.x % chn;
  for (int n = threadIdx.x / chn; n < rows; n += 64) cp_async16(dst + n * C + 2 * (k ^ slab_swz(n, chn)), src + n * C + 2 * k);
}

// The four FFT stages run one warp per coil in CTAs of 32*C threads (instantiated per coil
// count). With C <= 8 and G <= 512 the 80-register cap keeps three CTAs resident per SM (two
// at 128 registers for larger grids). The per-warp FFT scratch and the output staging reuse
// the input slab's shared memory once it is consumed, which keeps a CTA near 72 KB. The
// column stages double-buffer the slab when two regions fit, so the next item streams in
// while the current one is transformed.
#define TSN_FFT_BOUNDS(G, MAXW) __launch_bounds__((MAXW) * 32, (MAXW) > 8 ? 1 : ((G) <= 512 ? 3 : 2))

// Forward rows (x-stage). Image row i0 -> z1[q1][i0][c] for all q1. Fuses the SENSE
// multiply, deapodization, power-of-two panel scaling, zero-padding and (CG) p = r + beta p.
// Shared memory: twiddles [G] | one region that holds, in turn,
//   the input slab  [row0 N][row1 N][maps C*N] float2 + [scaling N] float
//     mode 0 with smaps:  row0 = x row, maps = S_c rows      (row1 unused)
//     mode 0 without:     maps = coil-image rows
//     mode 1 (CG):        row0 = r row, row1 = p row, maps = S_c rows
//     mode 4 (CG, fused update): row0 = r, row1 = p, row2 = A p, row3 = x rows, maps = S_c rows
//   the per-warp FFT scratch [C][SCR], and the output rows [G][C+1] float2.
// Mode 4 also finishes CG iteration iter-1, which then needs no cg_update launch: parts holds
// four sections [lines] of <p, Ap>, Re <r, Ap>, <Ap, Ap> and <r, r> from the inverse rows, so
// rho = <r, r> (a direct sum over the stored r, as the reference's rs_old), alpha = rho / pAp,
// and rho' = |r - alpha Ap|^2 = rho - 2 alpha Re <r, Ap> + alpha^2 <Ap, Ap> (FP64, a negative
// rounding residue clamped to 0).  The expansion restarts from the direct sum every
// iteration, so its rounding does not accumulate while rho falls.  Each row updates
// x += alpha p and r -= alpha Ap before p = r + beta p.
// Reference: fft512_rows4_shared16_pad_scale<true> (nufft_custom_fft_forward_bench.cu:1600-1844);
// the CG update of reference_sparse_solver.py:297-323.
template <int G, int CC>
__global__ void TSN_FFT_BOUNDS(G, (CC <= 8 ? 8 : 16)) fwd_rows_kernel(FftArgs f, const float2* __restrict__ x, float2* __restrict__ z1,
                                                     int mode, float2* __restrict__ p, float2* __restrict__ r,
                                                     const double* __restrict__ parts, int nparts,
                                                     CgState* __restrict__ st, int iter, float2* __restrict__ xs,
                                                     const float2* __restrict__ ap) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  const int N = f.N;
  const int lines = f.lines();
  const int64_t pix = f.pix();
  constexpr int C = CC;  // coils (one warp each), a compile-time stride
  const int nrow = mode == 4 ? 4 : 2;
  const int in_f2 = (nrow + C) * N;  // float2 of the slab before the scaling row
  float2* tw_s = reinterpret_cast<float2*>(sm);
  uint8_t* reg = reinterpret_cast<uint8_t*>(tw_s + G);
  float2* row0 = reinterpret_cast<float2*>(reg);
  float2* row1 = row0 + N;
  float2* row2 = row1 + N;
  float2* row3 = row2 + N;
  float2* maps = row0 + nrow * N;
  const float* srow = reinterpret_cast<const float*>(reg + in_f2 * 8);
  float2* scr = reinterpret_cast<float2*>(reg);
  float2* out_s = reinterpret_cast<float2*>(reg);  // [G][C+1]
  __shared__ double red[132];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // part 1: rows no kernel of a solve writes (coil maps, deapodization); part 2: the rest
  auto issue = [&](int i0, int part) {
    const size_t off = static_cast<size_t>(i0) * N;
    if (part & 2) {
      if (mode >= 1) {
        cp_async_bytes(row0, r + off, N * 8);
        if ((mode == 1 && iter > 0) || mode == 4) cp_async_bytes(row1, p + off, N * 8);
        if (mode == 4) {
          cp_async_bytes(row2, ap + off, N * 8);
          cp_async_bytes(row3, xs + off, N * 8);
        }
      } else if (f.smaps) {
        cp_async_bytes(row0, x + off, N * 8);
      }
    }
    if (part & (f.smaps ? 1 : 2)) {
      const float2* msrc = f.smaps ? f.smaps : x;
      for (int c = 0; c < C; ++c) cp_async_bytes(maps + c * N, msrc + static_cast<size_t>(c) * pix + off, N * 8);
    }
    if (part & 1) cp_async_bytes(reg + in_f2 * 8, f.scaling + off, N * 4);
    cp_async_commit();
  };
  // the twiddles and the first item's map rows stream in while the preceding kernel drains,
  // its other rows while the panel scale is reduced
  cp_async_bytes(tw_s, f.tw, G * 8);
  if (blockIdx.x < lines) issue(blockIdx.x, 1);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < lines) issue(blockIdx.x, 2);
  double total, alpha = 0.0, rho_prev = 0.0;
  if (mode == 4) {  // finish iteration iter-1 (the cg_update scalars)
    const double4 s3 = sum_partials4(parts, nparts, lines, red);
    const double rho = s3.w;  // |r_{iter-1}|^2 summed directly
    rho_prev = rho;
    const bool ok = isfinite(s3.x) && s3.x > 0.0;
    alpha = ok ? rho / s3.x : 0.0;
    const double rn = rho - 2.0 * alpha * s3.y + alpha * alpha * s3.z;
    total = rn < 0.0 ? 0.0 : rn;  // a negative rounding residue clamps to 0; NaN stays NaN
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->rho[iter - 1] = rho;  // the history keeps the direct sum
      st->pap[iter - 1] = s3.x;
      st->alpha[iter - 1] = alpha;
      // the iteration count stops at the first failing iteration, as the reference solver
      // stops there (reference_sparse_solver.py:281-293); the solve itself runs on with alpha 0
      const bool fin = isfinite(s3.x) && isfinite(rho) && isfinite(total);
      const bool prior_ok = st->curvature_ok && st->finite_ok;
      if (!ok) st->curvature_ok = 0;
      if (!fin) st->finite_ok = 0;
      if (prior_ok && ok && fin) st->completed = iter;
    }
  } else {
    total = sum_partials(parts, nparts, red);
  }
  const float af = static_cast<float>(alpha);
  float sigma;
  double beta = 0.0;
  if (mode == 0) {
    sigma = pow2_scale(total, static_cast<double>(pix) * (f.smaps ? 1 : C), kPanelTarget);
    if (blockIdx.x == 0 && threadIdx.x == 0) st->sigma_x = sigma;
  } else {
    sigma = pow2_scale(total, static_cast<double>(pix), kPanelTarget);
    // mode 4 divides by its own direct rho (block 0 rewrites st->rho[iter - 1] concurrently)
    const double rho_old = mode == 4 ? rho_prev : (iter > 0 ? st->rho[iter - 1] : 1.0);
    beta = (iter == 0 || mode == 2) ? 0.0 : total / fmax(rho_old, 1e-30);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->rho[iter] = total;
      st->beta[iter] = beta;
      st->sigma[iter] = sigma;
    }
  }
  const float bf = static_cast<float>(beta);
  const float scl = sigma / f.gs();
  // output copy: C/2 16-byte chunks per grid row, 64 rows per pass of the 32*C threads
  const int ch2 = C >> 1;
  const int ck = threadIdx.x % ch2, crow = threadIdx.x / ch2;
  for (int i0 = blockIdx.x; i0 < lines; i0 += gridDim.x) {
    if (i0 != blockIdx.x) {
      __syncthreads();  // the previous item's output rows are copied out
      issue(i0, 3);
    }
    cp_async_wait<0>();
    __syncthreads();
    if (mode >= 1) {  // p = r + beta p (p = r at iteration 0 and after a restart); row0 becomes p
      for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const size_t px = static_cast<size_t>(i0) * N + i;
        float2 pv = row0[i];
        if (mode == 4) {  // x += alpha p, r -= alpha Ap (the previous iteration's update)
          const float2 po = row1[i], av = row2[i], xv = row3[i];
          pv.x -= af * av.x;
          pv.y -= af * av.y;
          r[px] = pv;
          xs[px] = make_float2(xv.x + af * po.x, xv.y + af * po.y);
        }
        if ((mode == 1 && iter > 0) || mode == 4) {
          const float2 po = row1[i];
          pv = make_float2(pv.x + bf * po.x, pv.y + bf * po.y);
        }
        row0[i] = pv;
        p[px] = pv;
      }
      __syncthreads();
    }
    float2 v[P];
    const int c = warp;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = warp_fft_in_index<G>(j);
      int i1 = n + f.shift;
      if (i1 >= G) i1 -= G;
      float2 val = make_float2(0.f, 0.f);
      if (i1 < N) {
        const float d = srow[i1] * scl;
        val = (f.smaps || mode >= 1) ? cscale(cmul(row0[i1], maps[c * N + i1]), d) : cscale(maps[c * N + i1], d);
      }
      v[j] = val;
    }
    __syncthreads();  // slab consumed: the region becomes FFT scratch
    warp_fft<G, false>(v, scr + c * FftSmem<G>::SCR, tw_s);
    __syncthreads();  // scratch free: the region becomes the output rows
#pragma unroll
    for (int m = 0; m < P; ++m) out_s[warp_fft_out_index<G>(m) * (C + 1) + c] = v[m];
    __syncthreads();
    // line i0 = (slab, row): z1 [slab][q][row][c] (one slab for images)
    const size_t obase = static_cast<size_t>(i0 / N) * G * N + i0 % N;
    for (int q1 = crow; q1 < G; q1 += 64) {
      const float2 a = out_s[q1 * (C + 1) + 2 * ck], b = out_s[q1 * (C + 1) + 2 * ck + 1];
      *reinterpret_cast<float4*>(z1 + (obase + static_cast<size_t>(q1) * N) * C + 2 * ck) = make_float4(a.x, a.y, b.x, b.y);
    }
  }
}

// Forward columns (y-stage): z1[q1][*][c] -> panel rows q1*G + q0, FP16 hi | res.
// Shared memory: twiddles [G] | nbuf regions of `region` bytes, each holding in turn the
// swizzled input slab [N][C], the per-warp FFT scratch and the output rows [G][2C+1] words.
// Reference: fft512_allcoils1_shared16_to_n16 (nufft_custom_fft_forward_bench.cu:538-747).
template <int G, int CC>
__global__ void TSN_FFT_BOUNDS(G, (CC <= 8 ? 8 : 16)) fwd_cols_kernel(FftArgs f, const float2* __restrict__ z1,
                                                     __half* __restrict__ panel, int region, int nbuf) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  const int N = f.N;
  constexpr int C = CC;  // coils (one warp each), a compile-time stride
  float2* tw_s = reinterpret_cast<float2*>(sm);
  uint8_t* regs = reinterpret_cast<uint8_t*>(tw_s + G);
  const int OP = 2 * C + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto issue = [&](int q1, int b) {
    cp_async_slab(reinterpret_cast<float2*>(regs + b * region), z1 + static_cast<size_t>(q1) * N * C, N, C);
    cp_async_commit();
  };
  const int items = f.gcols();
  cp_async_bytes(tw_s, f.tw, G * 8);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < items) issue(blockIdx.x, 0);
  const int ch2 = C >> 1;  // 16-byte chunks per panel row
  const int ck = threadIdx.x % ch2, crow = threadIdx.x / ch2;
  const int c = warp;
  const int lane_off = 2 * ((c >> 1) ^ slab_swz(lane + f.shift, C >> 1)) + (c & 1);
  int it = 0;
  for (int q1 = blockIdx.x; q1 < items; q1 += gridDim.x, ++it) {
    const int b = nbuf == 2 ? (it & 1) : 0;
    if (nbuf == 1 && it > 0) {
      __syncthreads();  // the previous item's output rows are copied out
      issue(q1, 0);
    }
    cp_async_wait<0>();
    __syncthreads();
    if (nbuf == 2 && q1 + gridDim.x < items) issue(q1 + gridDim.x, b ^ 1);
    uint8_t* reg = regs + b * region;
    const float2* in_s = reinterpret_cast<const float2*>(reg);
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = warp_fft_in_index<G>(j);
      int i0 = n + f.shift;
      if (i0 >= G) i0 -= G;
      // power-of-two grids: the lane's low five index bits (and so its swizzle) are fixed
      const int idx = FftPlan<G>::R == 1 ? i0 * C + lane_off : slab_idx(i0, c, C);
      v[j] = i0 < N ? in_s[idx] : make_float2(0.f, 0.f);
    }
    __syncthreads();  // slab consumed
    warp_fft<G, false>(v, reinterpret_cast<float2*>(reg) + c * FftSmem<G>::SCR, tw_s);
    __syncthreads();  // scratch free
    uint32_t* out_s = reinterpret_cast<uint32_t*>(reg);
#pragma unroll
    for (int m = 0; m < P; ++m) {
      const int q0 = warp_fft_out_index<G>(m);
      uint32_t hw, rw;
      split_hi_res2(v[m].x, v[m].y, hw, rw);
      out_s[q0 * OP + c] = hw;
      out_s[q0 * OP + C + c] = rw;
    }
    __syncthreads();
    uint32_t* dst = reinterpret_cast<uint32_t*>(panel + static_cast<size_t>(q1) * G * 4 * C);
    for (int q0 = crow; q0 < G; q0 += 64) {
      const uint32_t* s = out_s + q0 * OP + 4 * ck;
      *reinterpret_cast<uint4*>(dst + q0 * 2 * C + 4 * ck) = make_uint4(s[0], s[1], s[2], s[3]);
    }
  }
}

// Forward middle axis of a volume: z1[i0][q2][i1][c] -> z2[q2][q1][i0][c]. One item per
// (i0, q2) line: its [N][C] run of z1 is contiguous; FFT over i1 with the zero padding and
// centring shift of the other axes; each q1 writes one 8C-byte run of z2.
// Shared memory: twiddles [G] | nbuf regions, each holding in turn the swizzled slab [N][C],
// the per-warp FFT scratch and the output rows [G][C+1] float2.
template <int G, int CC>
__global__ void TSN_FFT_BOUNDS(G, (CC <= 8 ? 8 : 16)) fwd_mid_kernel(FftArgs f, const float2* __restrict__ z1,
                                                    float2* __restrict__ z2, int region, int nbuf) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  const int N = f.N;
  constexpr int C = CC;
  const int items = N * G;
  float2* tw_s = reinterpret_cast<float2*>(sm);
  uint8_t* regs = reinterpret_cast<uint8_t*>(tw_s + G);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto issue = [&](int t, int b) {
    cp_async_slab(reinterpret_cast<float2*>(regs + b * region), z1 + static_cast<size_t>(t) * N * C, N, C);
    cp_async_commit();
  };
  cp_async_bytes(tw_s, f.tw, G * 8);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < items) issue(blockIdx.x, 0);
  const int ch2 = C >> 1;
  const int ck = threadIdx.x % ch2, crow = threadIdx.x / ch2;
  const int c = warp;
  const int lane_off = 2 * ((c >> 1) ^ slab_swz(lane + f.shift, C >> 1)) + (c & 1);
  int it = 0;
  for (int t = blockIdx.x; t < items; t += gridDim.x, ++it) {
    const int b = nbuf == 2 ? (it & 1) : 0;
    if (nbuf == 1 && it > 0) {
      __syncthreads();  // the previous item's output rows are copied out
      issue(t, 0);
    }
    cp_async_wait<0>();
    __syncthreads();
    if (nbuf == 2 && t + gridDim.x < items) issue(t + gridDim.x, b ^ 1);
    uint8_t* reg = regs + b * region;
    const float2* in_s = reinterpret_cast<const float2*>(reg);
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = warp_fft_in_index<G>(j);
      int i1 = n + f.shift;
      if (i1 >= G) i1 -= G;
      const int idx = FftPlan<G>::R == 1 ? i1 * C + lane_off : slab_idx(i1, c, C);
      v[j] = i1 < N ? in_s[idx] : make_float2(0.f, 0.f);
    }
    __syncthreads();  // slab consumed
    warp_fft<G, false>(v, reinterpret_cast<float2*>(reg) + c * FftSmem<G>::SCR, tw_s);
    __syncthreads();  // scratch free
    float2* out_s = reinterpret_cast<float2*>(reg);  // [G][C+1]
#pragma unroll
    for (int m = 0; m < P; ++m) out_s[warp_fft_out_index<G>(m) * (C + 1) + c] = v[m];
    __syncthreads();
    const int i0 = t / G, q2 = t - (t / G) * G;
    float2* dst = z2 + (static_cast<size_t>(q2) * G * N + i0) * C;
    for (int q1 = crow; q1 < G; q1 += 64) {
      const float2 a = out_s[q1 * (C + 1) + 2 * ck], bb = out_s[q1 * (C + 1) + 2 * ck + 1];
      *reinterpret_cast<float4*>(dst + static_cast<size_t>(q1) * N * C + 2 * ck) = make_float4(a.x, a.y, bb.x, bb.y);
    }
  }
}

// Measurement / adjoint input [C][M] -> sample panel [M][4C] with sigma_y and density.
// Reference: integrated_complex_to_split2_half_rows (nufft_integrated_bench.cu:339-359).
__global__ void split_samples_kernel(const float2* __restrict__ y, const float* __restrict__ density, int64_t m,
                                     int C, __half* __restrict__ panel, const double* __restrict__ parts, int nparts,
                                     CgState* __restrict__ st) {
  __shared__ double red[33];
  const double total = sum_partials(parts, nparts, red);
  const float sigma = pow2_scale(total, static_cast<double>(m) * C, kPanelTarget);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->sigma_y = sigma;
    st->curvature_ok = 1;  // a solve starts here: reset the status words
    st->finite_ok = 1;
    st->completed = 0;
  }
  const int chunks = C / 4;
  uint32_t* pu = reinterpret_cast<uint32_t*>(panel);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m * chunks;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / chunks;
    const int q = static_cast<int>(i - row * chunks);
    const float w = sigma * (density ? density[row] : 1.0f);
    uint32_t hi[4], res[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 val = y[static_cast<size_t>(4 * q + k) * m + row];
      split_hi_res2(val.x * w, val.y * w, hi[k], res[k]);
    }
    *reinterpret_cast<uint4*>(pu + row * 2 * C + 4 * q) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(pu + row * 2 * C + C + 4 * q) = make_uint4(res[0], res[1], res[2], res[3]);
  }
}

// Inverse columns: grid rows q1*G + [0,G) (all coils) -> w1[q1][i0][c], i0 < N (crop).
// Shared memory: twiddles [G] | nbuf regions, each holding in turn the swizzled slab [G][C],
// the per-warp FFT scratch and the cropped output rows [N][C+1] float2.
// Reference: ifft512_rows8_regular_transposed (nufft_custom_fft_forward_bench.cu:1463-1515).
template <int G, int CC>
__global__ void TSN_FFT_BOUNDS(G, (CC <= 8 ? 8 : 16)) inv_cols_kernel(FftArgs f, const float2* __restrict__ grid,
                                                     float2* __restrict__ w1, int region, int nbuf) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  const int N = f.N;
  constexpr int C = CC;  // coils (one warp each), a compile-time stride
  float2* tw_s = reinterpret_cast<float2*>(sm);
  uint8_t* regs = reinterpret_cast<uint8_t*>(tw_s + G);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto issue = [&](int q1, int b) {
    cp_async_slab(reinterpret_cast<float2*>(regs + b * region), grid + static_cast<size_t>(q1) * G * C, G, C);
    cp_async_commit();
  };
  const int items = f.gcols();
  cp_async_bytes(tw_s, f.tw, G * 8);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < items) issue(blockIdx.x, 0);
  const int ch2 = C >> 1;  // 16-byte chunks per output row
  const int ck = threadIdx.x % ch2, crow = threadIdx.x / ch2;
  const int c = warp;
  const int lane_off = 2 * ((c >> 1) ^ slab_swz(lane, C >> 1)) + (c & 1);
  int it = 0;
  for (int q1 = blockIdx.x; q1 < items; q1 += gridDim.x, ++it) {
    const int b = nbuf == 2 ? (it & 1) : 0;
    if (nbuf == 1 && it > 0) {
      __syncthreads();
      issue(q1, 0);
    }
    cp_async_wait<0>();
    __syncthreads();
    if (nbuf == 2 && q1 + gridDim.x < items) issue(q1 + gridDim.x, b ^ 1);
    uint8_t* reg = regs + b * region;
    const float2* in_s = reinterpret_cast<const float2*>(reg);
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = warp_fft_in_index<G>(j);
      v[j] = in_s[FftPlan<G>::R == 1 ? n * C + lane_off : slab_idx(n, c, C)];
    }
    __syncthreads();
    warp_fft<G, true>(v, reinterpret_cast<float2*>(reg) + c * FftSmem<G>::SCR, tw_s);
    __syncthreads();
    float2* out_s = reinterpret_cast<float2*>(reg);  // [N][C+1]
#pragma unroll
    for (int m = 0; m < P; ++m) {
      int i0 = warp_fft_out_index<G>(m) + f.shift;
      if (i0 >= G) i0 -= G;
      if (i0 < N) out_s[i0 * (C + 1) + c] = v[m];
    }
    __syncthreads();
    float2* dst = w1 + static_cast<size_t>(q1) * N * C;
    for (int i0 = crow; i0 < N; i0 += 64) {
      const float2 a = out_s[i0 * (C + 1) + 2 * ck], bb = out_s[i0 * (C + 1) + 2 * ck + 1];
      *reinterpret_cast<float4*>(dst + i0 * C + 2 * ck) = make_float4(a.x, a.y, bb.x, bb.y);
    }
  }
}

// Inverse middle axis of a volume: z2[q2][q1][i0][c] -> z1[q2][i0][i1][c], i1 < N (crop).
// One item per (q2, i0): G runs of C values, N*C apart, gathered into a swizzled slab; the
// cropped output of the item is one contiguous [N][C] run.
// Shared memory: twiddles [G] | nbuf regions, each holding in turn the slab [G][C], the
// per-warp FFT scratch and the output rows [N][C+1] float2.
template <int G, int CC>
__global__ void TSN_FFT_BOUNDS(G, (CC <= 8 ? 8 : 16)) inv_mid_kernel(FftArgs f, const float2* __restrict__ z2,
                                                    float2* __restrict__ z1, int region, int nbuf) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  const int N = f.N;
  constexpr int C = CC;
  const int items = G * N;
  float2* tw_s = reinterpret_cast<float2*>(sm);
  uint8_t* regs = reinterpret_cast<uint8_t*>(tw_s + G);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto issue = [&](int t, int b) {
    float2* dst = reinterpret_cast<float2*>(regs + b * region);
    const int q2 = t / N, i0 = t - (t / N) * N;
    const float2* src = z2 + (static_cast<size_t>(q2) * G * N + i0) * C;
    const int chn = C / 2;
    const int k = threadIdx.x % chn;  // 32*C threads: 64 rows per pass
    for (int q1 = threadIdx.x / chn; q1 < G; q1 += 64)
      cp_async16(dst + q1 * C + 2 * (k ^ slab_swz(q1, chn)), src + static_cast<size_t>(q1) * N * C + 2 * k);
    cp_async_commit();
  };
  cp_async_bytes(tw_s, f.tw, G * 8);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < items) issue(blockIdx.x, 0);
  const int ch2 = C >> 1;
  const int ck = threadIdx.x % ch2, crow = threadIdx.x / ch2;
  const int c = warp;
  const int lane_off = 2 * ((c >> 1) ^ slab_swz(lane, C >> 1)) + (c & 1);
  int it = 0;
  for (int t = blockIdx.x; t < items; t += gridDim.x, ++it) {
    const int b = nbuf == 2 ? (it & 1) : 0;
    if (nbuf == 1 && it > 0) {
      __syncthreads();
      issue(t, 0);
    }
    cp_async_wait<0>();
    __syncthreads();
    if (nbuf == 2 && t + gridDim.x < items) issue(t + gridDim.x, b ^ 1);
    uint8_t* reg = regs + b * region;
    const float2* in_s = reinterpret_cast<const float2*>(reg);
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = warp_fft_in_index<G>(j);
      v[j] = in_s[FftPlan<G>::R == 1 ? n * C + lane_off : slab_idx(n, c, C)];
    }
    __syncthreads();
    warp_fft<G, true>(v, reinterpret_cast<float2*>(reg) + c * FftSmem<G>::SCR, tw_s);
    __syncthreads();
    float2* out_s = reinterpret_cast<float2*>(reg);  // [N][C+1]
#pragma unroll
    for (int m = 0; m < P; ++m) {
      int i1 = warp_fft_out_index<G>(m) + f.shift;
      if (i1 >= G) i1 -= G;
      if (i1 < N) out_s[i1 * (C + 1) + c] = v[m];
    }
    __syncthreads();
    float2* dst = z1 + static_cast<size_t>(t) * N * C;
    for (int i1 = crow; i1 < N; i1 += 64) {
      const float2 a = out_s[i1 * (C + 1) + 2 * ck], bb = out_s[i1 * (C + 1) + 2 * ck + 1];
      *reinterpret_cast<float4*>(dst + i1 * C + 2 * ck) = make_float4(a.x, a.y, bb.x, bb.y);
    }
  }
}

// Inverse rows + crop + deapodization + SENSE coil combine (+ CG epilogues).
// Shared memory: twiddles [G] | a region holding in turn the swizzled slab [G][C], the
// per-warp FFT scratch and the coil images [C][N] | (epi_smem) the epilogue inputs of the
// row, fetched in the slab's copy group: maps [C][N] (with smaps), p row [N] (mode 2),
// scaling row [N] float. Without epi_smem the epilogue reads them from global memory.
// Mode 2 with r given also writes Re <r, Ap>, <Ap, Ap> and <r, r> per line into
// parts[lines + i0], parts[2 lines + i0] and parts[3 lines + i0], for the next forward rows to
// finish the CG update (mode 4 there).
// Reference: ifft512_rows8_regular_crop_scale (nufft_custom_fft_forward_bench.cu:1517-1552)
// followed by sense_combine_scaled (nufft_fp16x2_cg_bench.cu:27-54).
template <int G, int CC>
__global__ void TSN_FFT_BOUNDS(G, (CC <= 8 ? 8 : 16)) inv_rows_kernel(FftArgs f, const float2* __restrict__ w1, float2* __restrict__ out,
                                                     int mode, float2* __restrict__ x, float2* __restrict__ r,
                                                     const float2* __restrict__ p, double* __restrict__ parts,
                                                     CgState* __restrict__ st, int iter, float inv_scale2,
                                                     float lambda_scaled, int region, int epi_smem) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  const int N = f.N;
  constexpr int C = CC;  // coils (one warp each), a compile-time stride
  const int lines = f.lines();
  const int64_t pix_n = f.pix();
  float2* tw_s = reinterpret_cast<float2*>(sm);
  uint8_t* reg = reinterpret_cast<uint8_t*>(tw_s + G);
  float2* emaps = reinterpret_cast<float2*>(reg + region);
  float2* eprow = emaps + (f.smaps ? C * N : 0);
  float* escale = reinterpret_cast<float*>(eprow + (mode >= 2 ? N : 0));
  __shared__ double red[132];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // part 1: rows no kernel of a solve writes (coil maps, deapodization); part 2: the rest
  auto issue = [&](int i0, int part) {
    const size_t off = static_cast<size_t>(i0) * N;
    if (part & 2) {
      float2* dst = reinterpret_cast<float2*>(reg);
      // G runs of C complex values (8C bytes each, 16-byte aligned for even C), swizzled
      const int chn = C / 2;
      const int k = threadIdx.x % chn;  // 32*C threads: 64 rows per pass
      for (int q1 = threadIdx.x / chn; q1 < G; q1 += 64)
        cp_async16(dst + q1 * C + 2 * (k ^ slab_swz(q1, chn)), w1 + (static_cast<size_t>(q1) * lines + i0) * C + 2 * k);
      if (epi_smem && mode >= 2) cp_async_bytes(eprow, p + off, N * 8);
    }
    if (epi_smem && (part & 1)) {
      if (f.smaps)
        for (int c = 0; c < C; ++c) cp_async_bytes(emaps + c * N, f.smaps + static_cast<size_t>(c) * pix_n + off, N * 8);
      cp_async_bytes(escale, f.scaling + off, N * 4);
    }
    cp_async_commit();
  };
  cp_async_bytes(tw_s, f.tw, G * 8);
  if (blockIdx.x < lines) issue(blockIdx.x, 1);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < lines) issue(blockIdx.x, 2);
  float factor;
  if (mode == 2) factor = f.gs() / st->sigma[iter] * inv_scale2;
  else if (mode == 3 || mode == 5) factor = f.gs() / st->sigma_x * inv_scale2;
  else factor = inv_scale2 / st->sigma_y;
  const int c = warp;
  const int lane_off = 2 * ((c >> 1) ^ slab_swz(lane, C >> 1)) + (c & 1);
  for (int i0 = blockIdx.x; i0 < lines; i0 += gridDim.x) {
    if (i0 != blockIdx.x) {
      __syncthreads();
      issue(i0, 3);
    }
    cp_async_wait<0>();
    __syncthreads();
    const float2* in_s = reinterpret_cast<const float2*>(reg);
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = warp_fft_in_index<G>(j);
      v[j] = in_s[FftPlan<G>::R == 1 ? n * C + lane_off : slab_idx(n, c, C)];
    }
    __syncthreads();
    warp_fft<G, true>(v, reinterpret_cast<float2*>(reg) + c * FftSmem<G>::SCR, tw_s);
    __syncthreads();
    float2* img_s = reinterpret_cast<float2*>(reg);  // [C][N]
#pragma unroll
    for (int m = 0; m < P; ++m) {
      int i1 = warp_fft_out_index<G>(m) + f.shift;
      if (i1 >= G) i1 -= G;
      if (i1 < N) img_s[c * N + i1] = v[m];
    }
    __syncthreads();
    double dot = 0.0, dot_r = 0.0, dot_a = 0.0, dot_rr = 0.0;
    for (int i1 = threadIdx.x; i1 < N; i1 += blockDim.x) {
      const size_t pix = static_cast<size_t>(i0) * N + i1;
      const float d = (epi_smem ? escale[i1] : f.scaling[pix]) * factor;
      if (!f.smaps) {  // coil images out [C][N][N]
        for (int cc = 0; cc < C; ++cc) out[static_cast<size_t>(cc) * pix_n + pix] = cscale(img_s[cc * N + i1], d);
        continue;
      }
      if (mode == 5 && x)  // the coil images before the combine, [C][N][N]
        for (int cc = 0; cc < C; ++cc) x[static_cast<size_t>(cc) * pix_n + pix] = cscale(img_s[cc * N + i1], d);
      float2 acc = make_float2(0.f, 0.f);
      for (int cc = 0; cc < C; ++cc) {
        const float2 s = epi_smem ? emaps[cc * N + i1] : f.smaps[static_cast<size_t>(cc) * pix_n + pix];
        acc = cadd(acc, cmulc(img_s[cc * N + i1], s));
      }
      acc = cscale(acc, d);
      if (mode == 0) {
        out[pix] = acc;
      } else if (mode == 1) {
        r[pix] = acc;
        x[pix] = make_float2(0.f, 0.f);
        dot += static_cast<double>(acc.x) * acc.x + static_cast<double>(acc.y) * acc.y;
      } else {
        const float2 pv = epi_smem ? eprow[i1] : p[pix];
        acc.x += lambda_scaled * pv.x;
        acc.y += lambda_scaled * pv.y;
        if (mode == 2 || mode == 5) {
          out[pix] = acc;
          dot += static_cast<double>(pv.x) * acc.x + static_cast<double>(pv.y) * acc.y;
          if (mode == 2 && r) {
            const float2 rv = r[pix];
            dot_r += static_cast<double>(rv.x) * acc.x + static_cast<double>(rv.y) * acc.y;
            dot_a += static_cast<double>(acc.x) * acc.x + static_cast<double>(acc.y) * acc.y;
            dot_rr += static_cast<double>(rv.x) * rv.x + static_cast<double>(rv.y) * rv.y;
          }
        } else {  // reliable residual r = b - M v (b read through x)
          const float2 bv = x[pix];
          const float2 rv = make_float2(bv.x - acc.x, bv.y - acc.y);
          out[pix] = rv;
          dot += static_cast<double>(rv.x) * rv.x + static_cast<double>(rv.y) * rv.y;
        }
      }
    }
    if (mode == 2 && r) {
      const double4 t = block_sum4(dot, dot_r, dot_a, dot_rr, red);
      if (threadIdx.x == 0) {
        parts[i0] = t.x;
        parts[lines + i0] = t.y;
        parts[2 * static_cast<int64_t>(lines) + i0] = t.z;
        parts[3 * static_cast<int64_t>(lines) + i0] = t.w;
      }
    } else if (mode != 0) {
      const double t = block_sum(dot, red);
      if (threadIdx.x == 0) parts[i0] = t;
    }
  }
}

constexpr int kCgRowPix = 4;  // pixels per thread of cg_update: rows up to 1024 pixels at 256 threads

__global__ void cg_update_kernel(int N, int nparts, int lines, float2* __restrict__ x, float2* __restrict__ r,
                                 const float2* __restrict__ p, const float2* __restrict__ ap,
                                 const double* __restrict__ pap_parts, double* __restrict__ rr_parts,
                                 CgState* __restrict__ st, int iter) {
  __shared__ double red[33];
  // the row's vectors stream in while the pAp partials are reduced (N <= kCgRowPix * blockDim)
  const int i0 = blockIdx.x;
  float2 pv[kCgRowPix], av[kCgRowPix], xv[kCgRowPix], rv[kCgRowPix];
#pragma unroll
  for (int j = 0; j < kCgRowPix; ++j) {
    const int i1 = threadIdx.x + j * blockDim.x;
    if (i1 < N) {
      const size_t pix = static_cast<size_t>(i0) * N + i1;
      pv[j] = p[pix];
      av[j] = ap[pix];
      xv[j] = x[pix];
      rv[j] = r[pix];
    }
  }
  // <p, Ap> and the direct <r, r> of the r this iteration started from (sections 0 and 3 of
  // the inverse rows' partials)
  const double pap = sum_partials(pap_parts, nparts, red);
  const double rho = sum_partials(pap_parts + 3 * static_cast<int64_t>(lines), nparts, red);
  const bool ok = isfinite(pap) && pap > 0.0;
  const double alpha = ok ? rho / pap : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rho[iter] = rho;
    st->pap[iter] = pap;
    st->alpha[iter] = alpha;
    const bool prior_ok = st->curvature_ok && st->finite_ok;  // completed stops at a failure
    if (!ok) st->curvature_ok = 0;
    if (!isfinite(pap)) st->finite_ok = 0;
    if (prior_ok && ok) st->completed = iter + 1;
  }
  const float af = static_cast<float>(alpha);
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < kCgRowPix; ++j) {
    const int i1 = threadIdx.x + j * blockDim.x;
    if (i1 >= N) continue;
    const size_t pix = static_cast<size_t>(i0) * N + i1;
    xv[j].x += af * pv[j].x;
    xv[j].y += af * pv[j].y;
    rv[j].x -= af * av[j].x;
    rv[j].y -= af * av[j].y;
    x[pix] = xv[j];
    r[pix] = rv[j];
    acc += static_cast<double>(rv[j].x) * rv[j].x + static_cast<double>(rv[j].y) * rv[j].y;
  }
  const double t = block_sum(acc, red);
  if (threadIdx.x == 0) rr_parts[i0] = t;
}

__global__ void cg_finish_kernel(int nparts, const double* __restrict__ rr_parts, CgState* __restrict__ st,
                                 int iters) {
  __shared__ double red[33];
  const double rho = sum_partials(rr_parts, nparts, red);
  if (threadIdx.x == 0) {
    st->rho[iters] = rho;
    if (!isfinite(rho)) {  // a non-finite last update: the last iteration did not complete
      if (st->curvature_ok && st->finite_ok && st->completed == iters) st->completed = iters - 1;
      st->finite_ok = 0;
    }
  }
}

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------
constexpr size_t kFftTwoCtaSmem = 114 * 1024;  // at most this per CTA keeps two CTAs per SM

static size_t align16(size_t b) { return (b + 15) & ~static_cast<size_t>(15); }

template <int G>
static size_t fft_scratch_bytes(int C) {
  return sizeof(float2) * static_cast<size_t>(C) * FftSmem<G>::SCR;
}
template <int G>
static size_t fwd_rows_region(const FftArgs& f, int mode) {
  const size_t in = static_cast<size_t>((mode == 4 ? 4 : 2) + f.C) * f.N * 8 + static_cast<size_t>(f.N) * 4;
  const size_t out = sizeof(float2) * static_cast<size_t>(G) * (f.C + 1);
  return align16(std::max({in, out, fft_scratch_bytes<G>(f.C)}));
}
template <int G>
static size_t fwd_cols_region(const FftArgs& f) {
  const size_t in = sizeof(float2) * static_cast<size_t>(f.N) * f.C;
  const size_t out = sizeof(uint32_t) * static_cast<size_t>(G) * (2 * f.C + 1);
  return align16(std::max({in, out, fft_scratch_bytes<G>(f.C)}));
}
template <int G>
static size_t inv_cols_region(const FftArgs& f) {
  const size_t in = sizeof(float2) * static_cast<size_t>(G) * f.C;
  const size_t out = sizeof(float2) * static_cast<size_t>(f.N) * (f.C + 1);
  return align16(std::max({in, out, fft_scratch_bytes<G>(f.C)}));
}
// middle stages: [G][C+1] float2 covers the [N][C] / [G][C] slabs and the [N][C+1] output
template <int G>
static size_t mid_region(const FftArgs& f) {
  const size_t rows = sizeof(float2) * static_cast<size_t>(G) * (f.C + 1);
  return align16(std::max(rows, fft_scratch_bytes<G>(f.C)));
}
template <int G>
static size_t inv_rows_region(const FftArgs& f) {
  const size_t in = sizeof(float2) * static_cast<size_t>(G) * f.C;
  const size_t img = sizeof(float2) * static_cast<size_t>(f.C) * f.N;
  return align16(std::max({in, img, fft_scratch_bytes<G>(f.C)}));
}
static size_t inv_rows_epi(const FftArgs& f, int mode) {
  const size_t maps = f.smaps ? sizeof(float2) * static_cast<size_t>(f.C) * f.N : 0;
  const size_t prow = mode >= 2 ? sizeof(float2) * static_cast<size_t>(f.N) : 0;
  return align16(maps + prow + sizeof(float) * static_cast<size_t>(f.N));
}

template <class K>
static void ensure_smem(K k, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// persistent grid: resident CTAs per SM x SMs (a 1/share slice of them when batched cases
// run side by side), capped by the item count
template <class K>
static int persistent_grid(K k, int threads, size_t smem, int items, int share = 1) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
  const int grid = std::max(1, std::max(1, per_sm) * sm_count() / std::max(1, share));
  return std::max(1, std::min(grid, items));
}

#define TSN_G_SWITCH(G_, ...)                                  \
  switch (G_) {                                                \
    case 128: { constexpr int GG = 128; __VA_ARGS__; } break;  \
    case 256: { constexpr int GG = 256; __VA_ARGS__; } break;  \
    case 384: { constexpr int GG = 384; __VA_ARGS__; } break;  \
    case 512: { constexpr int GG = 512; __VA_ARGS__; } break;  \
    case 640: { constexpr int GG = 640; __VA_ARGS__; } break;  \
    case 1024: { constexpr int GG = 1024; __VA_ARGS__; } break; \
    default: break;                                            \
  }
// FFT stage instantiation per coil count (4, 8, 12, 16): the index arithmetic folds to
// constants, and CTAs of up to 8 warps keep three per SM
#define TSN_FFT_C(C_, ...)                                  \
  switch (C_) {                                             \
    case 4: { constexpr int CC = 4; __VA_ARGS__; } break;   \
    case 8: { constexpr int CC = 8; __VA_ARGS__; } break;   \
    case 12: { constexpr int CC = 12; __VA_ARGS__; } break; \
    case 16: { constexpr int CC = 16; __VA_ARGS__; } break; \
    default: break;                                         \
  }

void launch_fwd_rows(const FftArgs& f, const float2* x, float2* z1, int mode, float2* p, float2* r,
                     const double* partials, int nparts, CgState* st, int iter, cudaStream_t s, float2* xs,
                     const float2* ap) {
  TSN_G_SWITCH(f.G, {
    const size_t sm = sizeof(float2) * GG + fwd_rows_region<GG>(f, mode);
    TSN_FFT_C(f.C, {
      auto k = fwd_rows_kernel<GG, CC>;
      ensure_smem(k, sm);
      const int grid = persistent_grid(k, 32 * f.C, sm, f.lines(), f.share);
      launch_k(k, grid, 32 * f.C, sm, s, false, f, x, z1, mode, p, r, partials, nparts, st, iter, xs, ap);
    });
  });
}

void launch_fwd_cols(const FftArgs& f, const float2* z1, __half* panel, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t region = fwd_cols_region<GG>(f);
    const size_t base = sizeof(float2) * GG;
    const int nbuf = base + 2 * region <= kFftTwoCtaSmem ? 2 : 1;
    const size_t sm = base + nbuf * region;
    TSN_FFT_C(f.C, {
      auto k = fwd_cols_kernel<GG, CC>;
      ensure_smem(k, sm);
      const int grid = persistent_grid(k, 32 * f.C, sm, f.gcols(), f.share);
      launch_k(k, grid, 32 * f.C, sm, s, false, f, z1, panel, static_cast<int>(region), nbuf);
    });
  });
}

void launch_fwd_mid(const FftArgs& f, const float2* z1, float2* z2, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t region = mid_region<GG>(f);
    const size_t base = sizeof(float2) * GG;
    const int nbuf = base + 2 * region <= kFftTwoCtaSmem ? 2 : 1;
    const size_t sm = base + nbuf * region;
    TSN_FFT_C(f.C, {
      auto k = fwd_mid_kernel<GG, CC>;
      ensure_smem(k, sm);
      const int grid = persistent_grid(k, 32 * f.C, sm, f.N * f.G, f.share);
      launch_k(k, grid, 32 * f.C, sm, s, false, f, z1, z2, static_cast<int>(region), nbuf);
    });
  });
}

void launch_inv_mid(const FftArgs& f, const float2* z2, float2* z1, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t region = mid_region<GG>(f);
    const size_t base = sizeof(float2) * GG;
    const int nbuf = base + 2 * region <= kFftTwoCtaSmem ? 2 : 1;
    const size_t sm = base + nbuf * region;
    TSN_FFT_C(f.C, {
      auto k = inv_mid_kernel<GG, CC>;
      ensure_smem(k, sm);
      const int grid = persistent_grid(k, 32 * f.C, sm, f.N * f.G, f.share);
      launch_k(k, grid, 32 * f.C, sm, s, false, f, z2, z1, static_cast<int>(region), nbuf);
    });
  });
}

void launch_split_samples(const float2* y, const float* density, int64_t m, int c, __half* panel,
                          const double* partials, int nparts, CgState* st, cudaStream_t s) {
  const int64_t blocks = std::min<int64_t>((m * (c / 4) + 255) / 256, 8 * 148);
  split_samples_kernel<<<static_cast<int>(std::max<int64_t>(blocks, 1)), 256, 0, s>>>(y, density, m, c, panel, partials,
                                                                                        nparts, st);
}

void launch_inv_cols(const FftArgs& f, const float2* grid, float2* w1, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t region = inv_cols_region<GG>(f);
    const size_t base = sizeof(float2) * GG;
    const int nbuf = base + 2 * region <= kFftTwoCtaSmem ? 2 : 1;
    const size_t sm = base + nbuf * region;
    TSN_FFT_C(f.C, {
      auto k = inv_cols_kernel<GG, CC>;
      ensure_smem(k, sm);
      const int g = persistent_grid(k, 32 * f.C, sm, f.gcols(), f.share);
      launch_k(k, g, 32 * f.C, sm, s, false, f, grid, w1, static_cast<int>(region), nbuf);
    });
  });
}

void launch_inv_rows(const FftArgs& f, const float2* w1, float2* out, int mode, float2* x, float2* r, const float2* p,
                     double* partials, CgState* st, int iter, float inv_scale2, float lambda_scaled, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t region = inv_rows_region<GG>(f);
    const size_t base = sizeof(float2) * GG + region;
    const size_t epi = inv_rows_epi(f, mode);
    const int epi_smem = base + epi <= kFftTwoCtaSmem ? 1 : 0;
    const size_t sm = base + (epi_smem ? epi : 0);
    TSN_FFT_C(f.C, {
      auto k = inv_rows_kernel<GG, CC>;
      ensure_smem(k, sm);
      const int g = persistent_grid(k, 32 * f.C, sm, f.lines(), f.share);
      launch_k(k, g, 32 * f.C, sm, s, false, f, w1, out, mode, x, r, p, partials, st, iter, inv_scale2, lambda_scaled,
                 static_cast<int>(region), epi_smem);
    });
  });
}

void launch_cg_update(int N, int lines, int nparts, float2* x, float2* r, const float2* p, const float2* ap,
                      const double* pap_parts, double* rr_parts, CgState* st, int iter, cudaStream_t s) {
  cg_update_kernel<<<lines, 256, 0, s>>>(N, nparts, lines, x, r, p, ap, pap_parts, rr_parts, st, iter);
}

void launch_cg_finish(int nparts, const double* rr_parts, CgState* st, int iters, cudaStream_t s) {
  cg_finish_kernel<<<1, 256, 0, s>>>(nparts, rr_parts, st, iters);
}

// Block b sums section b (part + b * stride, n values) into its first value.
__global__ void reduce_partials_kernel(double* part, int n, int64_t stride) {
  __shared__ double red[33];
  double* sec = part + blockIdx.x * stride;
  const double t = sum_partials(sec, n, red);  // every read lands before block_sum's first barrier
  if (threadIdx.x == 0) sec[0] = t;
}

void launch_reduce_partials(double* part, int n, cudaStream_t s, int sections, int64_t stride) {
  reduce_partials_kernel<<<sections, 1024, 0, s>>>(part, n, stride);
}

// FP64 partials of Re <a, b> over n complex values (grid-stride, one per block).
__global__ void rdot_partials_kernel(const float2* __restrict__ a, const float2* __restrict__ b, int64_t n,
                                     double* __restrict__ part) {
  __shared__ double scratch[33];
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 u = a[i], v = b[i];
    acc += static_cast<double>(u.x) * v.x + static_cast<double>(u.y) * v.y;
  }
  const double t = block_sum(acc, scratch);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// out[0] = the sum of n partials, in a fixed order (one block).
__global__ void sum_partials_to_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
  __shared__ double red[33];
  const double t = sum_partials(part, n, red);
  if (threadIdx.x == 0) out[0] = t;
}

void launch_rdot(const float2* a, const float2* b, int64_t n, double* parts, double* out, cudaStream_t s) {
  rdot_partials_kernel<<<kNormParts, 256, 0, s>>>(a, b, n, parts);
  sum_partials_to_kernel<<<1, 256, 0, s>>>(parts, kNormParts, out);
}

void launch_sum_partials_to(const double* parts, int n, double* out, cudaStream_t s) {
  sum_partials_to_kernel<<<1, 256, 0, s>>>(parts, n, out);
}

// ---- reverse-mode CG step (the adjoint recurrences of one CG iteration) -------------------
// Forward step k: alpha = rho / gamma (gamma = Re <p, q>, q = M p), x' = x + alpha p,
// r' = r - alpha q, rho' = |r'|^2, beta = rho' / rho, p' = r' + beta p. Given the cotangents
// xb (of x', constant over the solve), rb (of r'), pb (of p'), rhob (of rho'), the step makes
//   rb2   = rb + pb + 2 rhob_n r'                 rhob_n = rhob + <pb, p> / rho
//   alphab = <xb, p> - <rb2, q>                   gammab = -alphab rho / gamma^2
//   qb    = -alpha rb2 + gammab p
//   pbk   = beta pb + alpha xb + gammab q         (pb of step k = pbk + M qb, added later)
//   rhobk = -<pb, p> rho' / rho^2 + alphab / gamma
// with <rb2, q> = <rb, q> + <pb, q> + 2 rhob_n <r', q>, so the five FP64 inner products come
// from one pass over the vectors before any of them changes.
constexpr int kCgbBlocks = kCgStepParts;  // 2 x 148 SMs

__global__ void cgb_dots_kernel(int64_t n, const float2* __restrict__ rb, const float2* __restrict__ pb,
                                const float2* __restrict__ p, const float2* __restrict__ q,
                                const float2* __restrict__ rn, const float2* __restrict__ xb,
                                double* __restrict__ parts) {
  __shared__ double red[165];
  double d[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 vpb = pb[i], vp = p[i], vq = q[i], vrb = rb[i], vrn = rn[i], vxb = xb[i];
    d[0] += static_cast<double>(vpb.x) * vp.x + static_cast<double>(vpb.y) * vp.y;
    d[1] += static_cast<double>(vrb.x) * vq.x + static_cast<double>(vrb.y) * vq.y;
    d[2] += static_cast<double>(vpb.x) * vq.x + static_cast<double>(vpb.y) * vq.y;
    d[3] += static_cast<double>(vrn.x) * vq.x + static_cast<double>(vrn.y) * vq.y;
    d[4] += static_cast<double>(vxb.x) * vp.x + static_cast<double>(vxb.y) * vp.y;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double v = warp_sum(d[k]);
    if (lane == 0) red[33 * k + warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    const int nw = (blockDim.x + 31) >> 5;
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[33 * threadIdx.x + w];
    parts[static_cast<int64_t>(threadIdx.x) * gridDim.x + blockIdx.x] = t;
  }
}

// sc (device FP64): [0] rho, [1] rho', [2] gamma, [3] rhob in; [4] rhob of step k out.
__global__ void cgb_update_kernel(int64_t n, int nparts, const double* __restrict__ parts,
                                  const double* __restrict__ rho_p, const double* __restrict__ rhon_p,
                                  const double* __restrict__ gamma_p, const double* __restrict__ rhob_p,
                                  double* __restrict__ rhob_out, float2* __restrict__ rb, float2* __restrict__ pb,
                                  const float2* __restrict__ p, const float2* __restrict__ q,
                                  const float2* __restrict__ rn, const float2* __restrict__ xb,
                                  float2* __restrict__ qb, double* __restrict__ qnorm_parts) {
  __shared__ double red[132];
  __shared__ double dl[5];
  const double4 s4 = sum_partials4(parts, nparts, nparts, red);
  if (threadIdx.x == 0) {
    dl[0] = s4.x;
    dl[1] = s4.y;
    dl[2] = s4.z;
    dl[3] = s4.w;
  }
  const double d5 = sum_partials(parts + 4 * static_cast<int64_t>(nparts), nparts, red);
  __syncthreads();
  const double rho = *rho_p, rho_n = *rhon_p, gamma = *gamma_p, rhob = *rhob_p;
  const double alpha = rho / gamma, beta = rho_n / rho;
  const double betab = dl[0];
  const double rhob_n = rhob + betab / rho;
  const double rb2q = dl[1] + dl[2] + 2.0 * rhob_n * dl[3];
  const double alphab = d5 - rb2q;
  const double gammab = -alphab * rho / (gamma * gamma);
  if (blockIdx.x == 0 && threadIdx.x == 0) *rhob_out = -betab * rho_n / (rho * rho) + alphab / gamma;
  const float a = static_cast<float>(alpha), b = static_cast<float>(beta), g = static_cast<float>(gammab),
              h = static_cast<float>(2.0 * rhob_n);
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 vrb = rb[i], vpb = pb[i], vp = p[i], vq = q[i], vrn = rn[i], vxb = xb[i];
    const float2 r2 = make_float2(vrb.x + vpb.x + h * vrn.x, vrb.y + vpb.y + h * vrn.y);
    rb[i] = r2;
    const float2 qv = make_float2(-a * r2.x + g * vp.x, -a * r2.y + g * vp.y);
    qb[i] = qv;
    acc += static_cast<double>(qv.x) * qv.x + static_cast<double>(qv.y) * qv.y;
    pb[i] = make_float2(b * vpb.x + a * vxb.x + g * vq.x, b * vpb.y + a * vxb.y + g * vq.y);
  }
  if (qnorm_parts) {  // |qb|^2 partials: the panel scale of the M qb that follows
    const double t = block_sum(acc, red);
    if (threadIdx.x == 0) qnorm_parts[blockIdx.x] = t;
  }
}

// pb += M qb; with sb given, sb[c] += conj(qb) t[c] + tb[c] conj(p) over `coils` planes of n.
__global__ void cgb_finish_kernel(int64_t n, int coils, float2* __restrict__ pb, const float2* __restrict__ mqb,
                                  const float2* __restrict__ qb, const float2* __restrict__ t,
                                  const float2* __restrict__ tb, const float2* __restrict__ p,
                                  float2* __restrict__ sb) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 vm = mqb[i];
    float2 vpb = pb[i];
    vpb.x += vm.x;
    vpb.y += vm.y;
    pb[i] = vpb;
    if (!sb) continue;
    const float2 vq = qb[i], vp = p[i];
    for (int c = 0; c < coils; ++c) {
      const size_t j = static_cast<size_t>(c) * n + i;
      const float2 vt = t[j], vtb = tb[j];
      float2 acc = sb[j];
      // conj(qb) t + tb conj(p)
      acc.x += vq.x * vt.x + vq.y * vt.y + vtb.x * vp.x + vtb.y * vp.y;
      acc.y += vq.x * vt.y - vq.y * vt.x + vtb.y * vp.x - vtb.x * vp.y;
      sb[j] = acc;
    }
  }
}

// ---- one forward CG step on caller-owned vectors (differentiable solves) ------------------
// alpha = rho / gamma; x' = x + alpha p (when x is given); r' = r - alpha q; rho' = |r'|^2
// (FP64, fixed order); p' = r' + (rho' / rho) p. Outputs are separate arrays.
__global__ void cgf_update_kernel(int64_t n, const double* __restrict__ rho_p, const double* __restrict__ gamma_p,
                                  const float2* __restrict__ x, const float2* __restrict__ p,
                                  const float2* __restrict__ r, const float2* __restrict__ q,
                                  float2* __restrict__ x_out, float2* __restrict__ r_out, double* __restrict__ parts) {
  __shared__ double red[33];
  const float a = static_cast<float>(*rho_p / *gamma_p);
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 vp = p[i], vr = r[i], vq = q[i];
    if (x) {
      const float2 vx = x[i];
      x_out[i] = make_float2(vx.x + a * vp.x, vx.y + a * vp.y);
    }
    const float2 rn = make_float2(vr.x - a * vq.x, vr.y - a * vq.y);
    r_out[i] = rn;
    acc += static_cast<double>(rn.x) * rn.x + static_cast<double>(rn.y) * rn.y;
  }
  const double t = block_sum(acc, red);
  if (threadIdx.x == 0) parts[blockIdx.x] = t;
}

// With pnorm_parts given, also one FP64 partial of |p'|^2 per block (the panel scale of the
// next normal-operator application, which then needs no norm pass of its own).
__global__ void cgf_direction_kernel(int64_t n, int nparts, const double* __restrict__ parts,
                                     const double* __restrict__ rho_p, double* __restrict__ rho_out,
                                     const float2* __restrict__ p, const float2* __restrict__ r_new,
                                     float2* __restrict__ p_out, double* __restrict__ pnorm_parts) {
  __shared__ double red[33];
  const double rho_n = sum_partials(parts, nparts, red);
  if (blockIdx.x == 0 && threadIdx.x == 0) *rho_out = rho_n;
  const float b = static_cast<float>(rho_n / *rho_p);
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 vp = p[i], vr = r_new[i];
    const float2 pn = make_float2(vr.x + b * vp.x, vr.y + b * vp.y);
    p_out[i] = pn;
    acc += static_cast<double>(pn.x) * pn.x + static_cast<double>(pn.y) * pn.y;
  }
  if (pnorm_parts) {
    const double t = block_sum(acc, red);
    if (threadIdx.x == 0) pnorm_parts[blockIdx.x] = t;
  }
}

void launch_cg_step(int64_t n, double* parts, const double* rho, const double* gamma, const float2* x, const float2* p,
                    const float2* r, const float2* q, float2* x_out, float2* r_out, float2* p_out, double* rho_out,
                    double* p_norm_parts, cudaStream_t s) {
  cgf_update_kernel<<<kCgbBlocks, 256, 0, s>>>(n, rho, gamma, x, p, r, q, x_out, r_out, parts);
  cgf_direction_kernel<<<kCgbBlocks, 256, 0, s>>>(n, kCgbBlocks, parts, rho, rho_out, p, r_out, p_out, p_norm_parts);
}

void launch_cg_adjoint_step(int64_t n, double* parts, const double* rho, const double* rho_n, const double* gamma,
                            const double* rhob, double* rhob_out, float2* rb, float2* pb, const float2* p,
                            const float2* q, const float2* rn, const float2* xb, float2* qb, double* qb_norm_parts,
                            cudaStream_t s) {
  cgb_dots_kernel<<<kCgbBlocks, 256, 0, s>>>(n, rb, pb, p, q, rn, xb, parts);
  cgb_update_kernel<<<kCgbBlocks, 256, 0, s>>>(n, kCgbBlocks, parts, rho, rho_n, gamma, rhob, rhob_out, rb, pb, p, q,
                                                rn, xb, qb, qb_norm_parts);
}

void launch_cg_adjoint_finish(int64_t n, int coils, float2* pb, const float2* mqb, const float2* qb, const float2* t,
                              const float2* tb, const float2* p, float2* sb, cudaStream_t s) {
  cgb_finish_kernel<<<kCgbBlocks, 256, 0, s>>>(n, coils, pb, mqb, qb, t, tb, p, sb);
}

template <class T>
__global__ void gather_rows_kernel(const T* __restrict__ src, const int32_t* __restrict__ map, int64_t rows, int width,
                                   T* __restrict__ dst) {
  const int64_t n = rows * width;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t row = i / width, col = i - row * width;
    dst[i] = src[static_cast<int64_t>(map[row]) * width + col];
  }
}

void launch_gather_rows_f16(const __half* src, const int32_t* map, int64_t rows, int width, __half* dst, cudaStream_t s) {
  gather_rows_kernel<__half><<<592, 256, 0, s>>>(src, map, rows, width, dst);
}
void launch_gather_rows_f32(const float* src, const int32_t* map, int64_t rows, int width, float* dst, cudaStream_t s) {
  gather_rows_kernel<float><<<592, 256, 0, s>>>(src, map, rows, width, dst);
}

}  // namespace tsn
