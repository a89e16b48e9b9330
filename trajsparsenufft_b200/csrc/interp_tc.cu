// Sparse Kaiser-Bessel interpolation on the 5th-generation tensor cores: tcgen05.mma.sp
// (kind::f16, 2:4 sparse A from shared memory, FP32 accumulators in tensor memory), one
// persistent CTA per SM with warp-specialized roles.
//
// The reference runs warp-level mma.sp m16n8k32 per 16-row tile and gathers B with 2-byte
// loads (nufft_gt_spmma_complex_fused_f16_f32, experiments/production/src/nufft_spmma_bench.cu:
// 402-663).  Its pack gives every 16-row group its own K32 column set, so tiles cannot share a
// B operand.  Here seven tiles are stacked into one M = 128 A operand and their gathered rows
// side by side into one N = 224 B operand: one MMA per seven tiles, of which each tile keeps
// its diagonal 16 x 32 block of the accumulator (the off-diagonal products are not read).
// The pack's mma.sp pair metadata maps onto the tensor-memory metadata column as it is
// (lane 16 j + l holds pair word 2 (l % 8) + l / 8 of tile j; reordered at upload).
//
// Roles (416 threads):
//   warps 0-3   write each step's metadata into tensor memory (lane = warp's quarter), then
//               read the previous step's accumulators (tcgen05.ld), keep a running sum per
//               tile row in registers and write finished rows (the three epilogues of the
//               warp kernel, including the deterministic split-group reduction);
//   warp 4      record producer: TMA bulk copies of the step records (A + slot info) into a
//               12-slot record ring, refilled once the epilogue has finished a step;
//   warp 5      one lane issues tcgen05.mma.sp into one of two accumulator buffers and
//               commits it to an mbarrier;
//   warps 6-12  gather producers, one per slot: the slot's 32 panel rows (64 B each) with
//               16-byte cp.async, four lanes per row so every instruction moves eight whole
//               rows, into a 10-slot B ring freed by the MMA's completion; up to ten steps of
//               row gathers (224 rows each) are in flight per SM.
// The B rows are gathered with cp.async rather than TMA tile::gather4: the tensor map variant
// was correct but spent ~75 cycles of TMA time per four 64-byte rows (82-92 us per headline
// launch against 17 us for the warp kernel).
// Every mbarrier wait is bounded in wall time; a wait that gives up sets the view's error
// word, every role leaves its loop, waits (bounded) for its copies or MMAs in flight, and the
// tensor memory is freed before the CTA exits.
#include <algorithm>
#include <cstdio>

#include "device.cuh"
#include "kernels.cuh"
#include "tc05.cuh"

namespace tsn {

using namespace dev;
using namespace tc;

namespace {

// Two shared-memory rings.  Record slots (A of the seven tiles + zero rows, slot info) are
// refilled once the epilogue has finished their step; B slots (the gathered rows) are freed by
// the MMA's completion itself, so gathers run up to kBSlots steps ahead of the MMA and record
// copies up to kRecSlots steps ahead of the epilogue.
constexpr int kRecSlots = 12;
constexpr int kRecA = 0;                          // 4096 B: slots 0..6 + zero rows 112..127
constexpr int kRecInfo = 4096;                    // 1792 B of slot info
constexpr int kRecBytes = 6144;
constexpr int kBSlots = 10;
constexpr int kBBytes = kTcSlots * 2048;          // 14336 B, 64-byte-swizzled MN-major
constexpr int kBOffset = 0;                       // B ring first: 1024-aligned slots
constexpr int kRecOffset = kBSlots * kBBytes;
constexpr uint32_t kRecTx = kTcStepBytes;         // A + slot info bytes per step
constexpr int kGatherWarp0 = 6;                   // warps 6..12 gather slots 0..6
constexpr int kThreads = 32 * (kGatherWarp0 + kTcSlots);
constexpr uint32_t kTmemCols = 512;
// Tensor memory: accumulator buffer b = columns [256 b, 256 b + 224); metadata of step k in
// column 480 + 4 (k % kMetaBufs), written kMetaAhead steps before the step is read out.
__device__ __forceinline__ uint32_t d_col(int b) { return 256u * static_cast<uint32_t>(b); }
constexpr int kMetaBufs = 4;
constexpr int kMetaAhead = 2;
__device__ __forceinline__ uint32_t meta_col(int k) { return 480u + 4u * static_cast<uint32_t>(k % kMetaBufs); }
constexpr uint64_t kWaitNs = 50ull * 1000 * 1000;  // 50 ms: a healthy wait is microseconds
constexpr uint32_t kIdesc = idesc_f16_sparse(128, kTcSlots * 32, true);
static_assert(kRecInfo + kTcSlots * kTcSlotInfoBytes <= kRecBytes, "record slot layout");
static_assert(kTcStepABytes + kTcSlotABytes == kRecInfo, "A region holds seven tiles plus the zero tile");
static_assert(kBBytes % 1024 == 0 && kRecBytes % 1024 == 0, "ring slot alignment");

struct Bars {
  uint64_t rec_full[kRecSlots];   // A + slot info landed (bulk-copy tx)
  uint64_t rec_empty[kRecSlots];  // step finished by the epilogue (4 epilogue warps)
  uint64_t b_full[kBSlots];       // gathered rows landed (one cp.async arrival per row)
  uint64_t b_empty[kBSlots];      // the MMA reading the slot completed (MMA commit)
  uint64_t dfull[2];              // accumulator buffer written (MMA commit)
  uint64_t dempty[2];             // accumulator buffer read out (4 epilogue warps)
  uint64_t mfull[kMetaBufs];      // metadata column written (4 epilogue warps)
  uint32_t tmem;
  int32_t abort;
};
constexpr int kBarOffset = kRecOffset + kRecSlots * kRecBytes;
constexpr size_t kSmemBytes = kBarOffset + sizeof(Bars) + 1024;  // + alignment slack
static_assert(kSmemBytes <= 232448, "fits the 227 KB shared-memory opt-in of a block");

__device__ __forceinline__ int32_t tc_record_row(const uint8_t* rows24, int32_t flags, int s) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(rows24);
  const int bit = 24 * s, off = bit & 31;
  const uint32_t lo = w[bit >> 5];
  const uint32_t hi = off > 8 ? w[(bit >> 5) + 1] : 0u;
  const uint32_t v = __funnelshift_r(lo, hi, off) & 0xFFFFFFu;
  return ((static_cast<uint32_t>(flags) >> (kRecLiveShift + s)) & 1u) ? static_cast<int32_t>(v) : -1;
}

__device__ __forceinline__ void set_abort(Bars* b, int32_t* err, int code) {
  *reinterpret_cast<volatile int32_t*>(&b->abort) = 1;
  if (err) atomicOr(err, code);
}
__device__ __forceinline__ bool aborted(Bars* b) { return *reinterpret_cast<volatile int32_t*>(&b->abort) != 0; }

struct TcArgs {
  InterpTcView v;
  InterpOut o;
  const __half* panel;  // [rows][32] f16 panel the view gathers from
};

// Finished tile row of an item: the row's 32 accumulator columns (16 FP16-high products, then
// 16 residual products, interleaved (re, im) per coil) are summed pairwise, scaled and stored.
template <int EPI>
__device__ __forceinline__ void tc_store_row(const float (&acc)[32], int32_t row, float scale, const InterpOut& o) {
  if (row < 0) return;
  constexpr int C = 8;
  float w = scale;
  if constexpr (EPI == EPI_PANEL)
    if (o.density) w *= __ldg(o.density + row);
  float v[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) v[c] = (acc[c] + acc[16 + c]) * w;
  if constexpr (EPI == EPI_GRID) {
    float4* dst = reinterpret_cast<float4*>(o.c64 + static_cast<size_t>(row) * C);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else if constexpr (EPI == EPI_PANEL) {
    uint32_t hw[8], rw[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) split_hi_res2(v[2 * c], v[2 * c + 1], hw[c], rw[c]);
    uint4* dst = reinterpret_cast<uint4*>(o.panel + static_cast<size_t>(row) * 4 * C);
    dst[0] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    dst[1] = make_uint4(hw[4], hw[5], hw[6], hw[7]);
    dst[2] = make_uint4(rw[0], rw[1], rw[2], rw[3]);
    dst[3] = make_uint4(rw[4], rw[5], rw[6], rw[7]);
  } else {  // EPI_SAMPLES: [C][rows]
#pragma unroll
    for (int c = 0; c < 8; ++c) o.c64[static_cast<size_t>(c) * o.rows + row] = make_float2(v[2 * c], v[2 * c + 1]);
  }
}

template <int EPI>
__global__ void __launch_bounds__(kThreads, 1) interp_tc_kernel(const __grid_constant__ TcArgs args) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
  Bars* bars = reinterpret_cast<Bars*>(smem + kBarOffset);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const InterpTcView& v = args.v;
  const int2 range = v.cta_steps[blockIdx.x];
  const int n = range.y - range.x;
  const uint8_t* steps = v.steps + static_cast<size_t>(range.x) * kTcStepBytes;
  auto rec_slot = [&](int k) { return smem + kRecOffset + (k % kRecSlots) * kRecBytes; };
  auto b_slot = [&](int k) { return smem + kBOffset + (k % kBSlots) * kBBytes; };

  if (threadIdx.x == 0) {
    for (int i = 0; i < kRecSlots; ++i) {
      mbar_init(&bars->rec_full[i], 1);
      mbar_init(&bars->rec_empty[i], 4);
    }
    for (int i = 0; i < kBSlots; ++i) {
      mbar_init(&bars->b_full[i], kTcSlots * 32);  // one cp.async arrival per gathered row
      mbar_init(&bars->b_empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&bars->dfull[b], 1);
      mbar_init(&bars->dempty[b], 4);
    }
    for (int b = 0; b < kMetaBufs; ++b) mbar_init(&bars->mfull[b], 4);
    bars->abort = 0;
    mbar_fence_init();
  }
  // rows 112..127 of every record slot's A operand stay zero (no copy writes them)
  for (int i = threadIdx.x; i < kRecSlots * (kTcSlotABytes / 16); i += blockDim.x) {
    const int st = i / (kTcSlotABytes / 16), c = i % (kTcSlotABytes / 16);
    *reinterpret_cast<uint4*>(smem + kRecOffset + st * kRecBytes + kRecA + kTcStepABytes + 16 * c) =
        make_uint4(0, 0, 0, 0);
  }
  if (warp == 0) {
    tmem_alloc(&bars->tmem, kTmemCols);
    tmem_relinquish();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = bars->tmem;

  if (warp == 4) {
    // ---------------------------------------------------------------- record producer
    // A and slot info of step k as soon as step k - kRecSlots is finished
    int issued = 0;
    if (lane == 0) {
      for (int k = 0; k < n && !aborted(bars); ++k) {
        const int rs = k % kRecSlots, use = k / kRecSlots;
        if (use > 0 && !mbar_wait(&bars->rec_empty[rs], (use - 1) & 1, kWaitNs)) {
          set_abort(bars, v.error, 1);
          break;
        }
        mbar_arrive_expect_tx(&bars->rec_full[rs], kRecTx);
        const uint8_t* src = steps + static_cast<size_t>(k) * kTcStepBytes;
        uint8_t* slot = rec_slot(k);
        bulk_g2s(slot + kRecA, src, kTcStepABytes, &bars->rec_full[rs]);
        bulk_g2s(slot + kRecInfo, src + kTcStepABytes, kTcSlots * kTcSlotInfoBytes, &bars->rec_full[rs]);
        ++issued;
      }
      if (aborted(bars))  // the copies in flight land before the CTA can exit
        for (int k = max(0, issued - kRecSlots); k < issued; ++k)
          mbar_wait(&bars->rec_full[k % kRecSlots], (k / kRecSlots) & 1, kWaitNs);
    }
  } else if (warp >= kGatherWarp0) {
    // ---------------------------------------------------------------- gather producers
    // warp 6 + j gathers slot j: 32 panel rows of 64 B, 128 16-byte chunks; copy i of lane l
    // is chunk l % 4 of row l / 4 + 8 i, so each warp instruction moves eight whole rows
    // (coalesced 64-byte segments).  Rows land 64-byte swizzled (chunk c of row k at chunk
    // c ^ ((k % 8) >> 1) of its 64-byte line); a dead column is zero-filled without a global
    // read.  The barrier counts each lane's arrival once its copies have landed.
    const int j = warp - kGatherWarp0;
    const uint8_t* panel = reinterpret_cast<const uint8_t*>(args.panel);
    const int c = lane & 3, r0 = lane >> 2;  // chunk, first row (r0 + 8 i)
    const uint32_t dst_off = static_cast<uint32_t>(j * 2048 + r0 * 64) + 16u * static_cast<uint32_t>(c ^ (r0 >> 1));
    for (int k = 0; k < n; ++k) {
      if (__any_sync(0xFFFFFFFFu, aborted(bars))) break;
      const int rs = k % kRecSlots, bs = k % kBSlots, ub = k / kBSlots;
      const bool ok = mbar_wait(&bars->rec_full[rs], (k / kRecSlots) & 1, kWaitNs) &&
                      (ub == 0 || mbar_wait(&bars->b_empty[bs], (ub - 1) & 1, kWaitNs));
      if (!__all_sync(0xFFFFFFFFu, ok)) {
        set_abort(bars, v.error, 1);
        break;
      }
      const int32_t* cols = reinterpret_cast<const int32_t*>(rec_slot(k) + kRecInfo + j * kTcSlotInfoBytes);
      uint8_t* dst = b_slot(k) + dst_off;  // rows r0 + 8 i share r0 % 8 and so the swizzle
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int32_t col = cols[r0 + 8 * i];
        const uint8_t* src = panel + static_cast<size_t>(col < 0 ? 0 : col) * 64 + 16 * c;
        cp_async16_zfill(dst + i * 512, src, col < 0 ? 0u : 16u);
      }
      cp_async_arrive_noinc(&bars->b_full[bs]);
    }
    // copies in flight land before the CTA can exit
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  } else if (warp == 5) {
    // ---------------------------------------------------------------- MMA issue
    if (lane == 0) {
      int issued = 0;
      for (int k = 0; k < n && !aborted(bars); ++k) {
        const int rs = k % kRecSlots, bs = k % kBSlots, b = k & 1, bu = k >> 1;
        const bool ok = mbar_wait(&bars->rec_full[rs], (k / kRecSlots) & 1, kWaitNs) &&
                        mbar_wait(&bars->b_full[bs], (k / kBSlots) & 1, kWaitNs) &&
                        mbar_wait(&bars->mfull[k % kMetaBufs], (k / kMetaBufs) & 1, kWaitNs) &&
                        (k < 2 || mbar_wait(&bars->dempty[b], (bu - 1) & 1, kWaitNs));
        if (!ok) {
          set_abort(bars, v.error, 2);
          break;
        }
        fence_proxy_async_smem();  // the gathered rows (generic-proxy cp.async writes) reach the MMA
        tc_fence_after();
        const uint64_t ad = smem_desc(smem_addr(rec_slot(k) + kRecA), 128, 256, kLayoutNone);
        const uint64_t bd = smem_desc(smem_addr(b_slot(k)), 2048, 512, kLayoutSw64);
        mma_sp_f16(tbase + d_col(b), ad, bd, kIdesc, tbase + meta_col(k), 0u);
        mma_commit(&bars->dfull[b]);     // accumulators ready
        mma_commit(&bars->b_empty[bs]);  // B slot free for the gathers
        ++issued;
      }
      if (aborted(bars) && issued > 0) {  // the last MMAs finish before the memory is freed
        const int k = issued - 1;
        mbar_wait(&bars->dfull[k & 1], (k >> 1) & 1, kWaitNs);
        if (k >= 1) mbar_wait(&bars->dfull[(k - 1) & 1], ((k - 1) >> 1) & 1, kWaitNs);
      }
    }
  } else {
    // ---------------------------------------------------------------- metadata + epilogue
    const int slot = threadIdx.x >> 4, r = threadIdx.x & 15, half = slot & 1;
    const bool live_slot = slot < kTcSlots;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;
    const unsigned hmask = 0xFFFFu << (16 * half);
    float scale = args.o.scale_mul;
    if (args.o.scale_ptr) {
      const float sp = *args.o.scale_ptr;
      scale *= args.o.scale_inv ? 1.0f / sp : sp;
    }
    float acc[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = 0.f;
    constexpr unsigned kFull = 0xFFFFFFFFu;
    // Control flow stays warp-uniform around the .sync.aligned tensor-memory instructions:
    // every exit is decided with __any_sync / __all_sync and the warp reconverges at the top
    // of each step (the per-slot work below diverges by half-warp).
    // Metadata of step k goes into column buffer k % 4, two steps ahead of the accumulators
    // being read, so the MMAs of the next steps run while a step is read out.
    auto write_meta = [&](int k) -> bool {
      if (!__all_sync(kFull, mbar_wait(&bars->rec_full[k % kRecSlots], (k / kRecSlots) & 1, kWaitNs))) return false;
      const uint8_t* info = rec_slot(k) + kRecInfo;
      const uint32_t meta =
          live_slot ? *reinterpret_cast<const uint32_t*>(info + slot * kTcSlotInfoBytes + 128 + 4 * r) : 0u;
      tmem_st1(tbase + lane_base + meta_col(k), meta);
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars->mfull[k % kMetaBufs]);
      return true;
    };
    bool meta_ok = true;
    for (int k = 0; k < min(kMetaAhead, n) && meta_ok; ++k) meta_ok = write_meta(k);
    if (!meta_ok) set_abort(bars, v.error, 4);
    for (int p = 0; p < n && meta_ok; ++p) {
      __syncwarp();
      if (__any_sync(kFull, aborted(bars))) break;
      // buffer (p + 2) % 4 was last read by the MMA of step p - 2, complete since step p - 1
      // was read out
      if (p + kMetaAhead < n && !write_meta(p + kMetaAhead)) {
        set_abort(bars, v.error, 4);
        break;
      }
      // accumulators of step p: each half-warp reads its own slot's diagonal 16 x 32 block
      const int pb = p & 1, pbu = p >> 1;
      if (!__all_sync(kFull, mbar_wait(&bars->dfull[pb], pbu & 1, kWaitNs))) {
        set_abort(bars, v.error, 8);
        break;
      }
      tc_fence_after();
      // a 32-lane load gives every lane the same columns: both slots' blocks are read and each
      // half-warp keeps its own (the 16-lane shapes repeat one half's lanes, so they cannot help)
      float d0[32], d1[32];
      tmem_ld32(tbase + lane_base + d_col(pb) + 64 * warp, d0);
      tmem_ld32(tbase + lane_base + d_col(pb) + 64 * warp + 32, d1);
      const uint8_t* sinfo = rec_slot(p) + kRecInfo + (live_slot ? slot : 0) * kTcSlotInfoBytes;
      const RecordInfo info = *reinterpret_cast<const RecordInfo*>(sinfo + 192);
      const int32_t row = (live_slot && (info.flags & kRecLast)) ? tc_record_row(sinfo + 208, info.flags, r) : -1;
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&bars->dempty[pb]);
        mbar_arrive(&bars->rec_empty[p % kRecSlots]);  // record slot fully read
      }
      if (!live_slot || info.flags == 0) continue;      // slot 7 or an idle slot
#pragma unroll
      for (int i = 0; i < 32; ++i) acc[i] += half ? d1[i] : d0[i];
      if (!(info.flags & kRecLast)) continue;
      if (info.split >= 0) {  // chunk of a split group: publish, the last chunk reduces in order
        const int chunk = info.chunk & 0xFFFF, nchunks = info.chunk >> 16;
        float* mine = v.partials + static_cast<size_t>(info.first_slot + chunk) * kTcPartialFloats;
#pragma unroll
        for (int i = 0; i < 32; ++i) mine[i * 16 + r] = acc[i];
        __threadfence();
        __syncwarp(hmask);
        int prior = 0;
        if (r == 0) prior = atomicAdd(&v.counters[info.split], 1);
        prior = __shfl_sync(hmask, prior, 16 * half);
        if (prior != nchunks - 1) {
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[i] = 0.f;
          continue;
        }
        __threadfence();
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[i] = 0.f;
        for (int cc = 0; cc < nchunks; ++cc) {
          const float* src = v.partials + static_cast<size_t>(info.first_slot + cc) * kTcPartialFloats;
#pragma unroll
          for (int i = 0; i < 32; ++i) acc[i] += __ldcg(src + i * 16 + r);
        }
        if (r == 0) v.counters[info.split] = 0;  // ready for the next launch
      }
      tc_store_row<EPI>(acc, row, scale, args.o);
#pragma unroll
      for (int i = 0; i < 32; ++i) acc[i] = 0.f;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, kTmemCols);
  }
}

}  // namespace

size_t interp_tc_smem_bytes() { return kSmemBytes; }

template <int EPI>
static void launch_tc_t(const TcArgs& a, int ctas, cudaStream_t s) {
  auto k = interp_tc_kernel<EPI>;
  static thread_local int configured = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (configured != dev) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSmemBytes));
    configured = dev;
  }
  k<<<ctas, kThreads, kSmemBytes, s>>>(a);
}

void launch_interp_tc(const InterpTcView& v, const __half* panel, int epi, const InterpOut& o, cudaStream_t s) {
  if (v.n_ctas <= 0) return;
  TcArgs a;
  a.v = v;
  a.o = o;
  a.panel = panel;
  switch (epi) {
    case EPI_SAMPLES: launch_tc_t<EPI_SAMPLES>(a, v.n_ctas, s); break;
    case EPI_GRID: launch_tc_t<EPI_GRID>(a, v.n_ctas, s); break;
    default: launch_tc_t<EPI_PANEL>(a, v.n_ctas, s); break;
  }
}

}  // namespace tsn
