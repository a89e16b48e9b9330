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
#include <cstdio>
#include <vector>
#include <cmath>

#include "fft.cuh"
#include "kernels.cuh"

namespace tsn {

using namespace dev;

void set_twiddle_constants(cudaStream_t s) {
  std::vector<float2> w(1024);
  for (int e = 0; e < 1024; ++e) {
    const double a = -2.0 * M_PI * e / 1024.0;
    w[e] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
  }
  cudaMemcpyToSymbolAsync(dev::c_w1024, w.data(), sizeof(float2) * 1024, 0, cudaMemcpyHostToDevice, s);
  cudaStreamSynchronize(s);
}

// ------------------------------------------------------------------------------------------
// Sparse interpolation: one warp per 16-row group, 2:4 tiles through mma.sp m16n8k32.
// Per tile the 32 gathered panel rows (hi and res together) are brought to shared memory
// with 16-byte cp.async (double-buffered), swizzled so ldmatrix.trans is conflict-free.
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

template <int ROWH, bool SPLIT, int NCOMP, int EPI, bool CONJ>
__global__ void __launch_bounds__(kInterpWarps * 32) interp_mmasp_kernel(InterpView v, const __half* __restrict__ panel,
                                                                         InterpOut o) {
  constexpr int BYTES = ROWH * 2;
  constexpr int CH = BYTES / 16;
  constexpr int NB = ROWH / 8;
  constexpr int NA = SPLIT ? NB / 2 : NB;
  constexpr int NACC = NCOMP * NA * 4;
  static_assert(NACC <= kPartialFloats, "partials slot too small");
  extern __shared__ __align__(128) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item_idx = blockIdx.x * kInterpWarps + warp;
  if (item_idx >= v.n_items) return;
  const WorkItem item = v.items[item_idx];
  const int gidx = item.group;
  uint8_t* sb = smem + warp * 2 * 32 * BYTES;
  const uint8_t* pb = reinterpret_cast<const uint8_t*>(panel);
  const uint32_t t0 = item.t0, t1 = item.t1;
  const int g = lane >> 2, t = lane & 3;

  float acc[NCOMP][NA][4];
#pragma unroll
  for (int c = 0; c < NCOMP; ++c)
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[c][a][i] = 0.f;

  auto load_col = [&](uint32_t tile) {
    return __ldg(reinterpret_cast<const int32_t*>(v.records + static_cast<size_t>(tile) * v.rec_bytes) + lane);
  };
  auto issue = [&](int32_t col, int buf) {
    uint8_t* dst = sb + buf * 32 * BYTES;
#pragma unroll
    for (int i = 0; i < CH; ++i) {
      const int ci = lane + 32 * i;
      const int row = ci / CH, ch = ci % CH;
      const int src = __shfl_sync(0xFFFFFFFFu, col, row);
      cp_async16(dst + row * BYTES + chunk_swizzle<CH>(ch, row) * 16, pb + static_cast<size_t>(src) * BYTES + ch * 16);
    }
    cp_async_commit();
  };

  // column ids run two tiles ahead of the MMAs, the gather one tile ahead
  int32_t col_next = 0;
  if (t0 < t1) issue(load_col(t0), 0);
  if (t0 + 1 < t1) col_next = load_col(t0 + 1);
  for (uint32_t tile = t0; tile < t1; ++tile) {
    const int buf = (tile - t0) & 1;
    const bool more = tile + 1 < t1;
    if (more) {
      issue(col_next, buf ^ 1);
      if (tile + 2 < t1) col_next = load_col(tile + 2);
    }
    const uint8_t* rec = v.records + static_cast<size_t>(tile) * v.rec_bytes;
    uint32_t a[NCOMP][4], meta[NCOMP];
#pragma unroll
    for (int c = 0; c < NCOMP; ++c) {
      const uint32_t* A = reinterpret_cast<const uint32_t*>(rec + 128 + 576 * c);
      a[c][0] = __ldg(A + g * 8 + t);
      a[c][1] = __ldg(A + (g + 8) * 8 + t);
      a[c][2] = __ldg(A + g * 8 + 4 + t);
      a[c][3] = __ldg(A + (g + 8) * 8 + 4 + t);
      meta[c] = __ldg(reinterpret_cast<const uint32_t*>(rec + 640 + 576 * c) + g * 2 + (t & 1));
    }
    if (more) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncwarp();
    const uint8_t* B = sb + buf * 32 * BYTES;
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
      uint32_t b[4];
      ldmatrix_x4_trans(b, B + lane * BYTES + chunk_swizzle<CH>(nb, lane) * 16);
      const int ai = SPLIT ? (nb % NA) : nb;
#pragma unroll
      for (int c = 0; c < NCOMP; ++c) mma_sp_16832(acc[c][ai], a[c], b, meta[c]);
    }
    __syncwarp();
  }

  if (item.split >= 0) {
    // split group: publish this chunk, the last chunk to arrive reduces all in order
    const SplitGroup sg = v.splits[item.split];
    const int chunk = static_cast<int>((t0 - v.group_offsets[gidx]) / kChunkTiles);
    float* mine = v.partials + static_cast<size_t>(sg.first_slot + chunk) * kPartialFloats * 32;
#pragma unroll
    for (int c = 0; c < NCOMP; ++c)
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
        for (int i = 0; i < 4; ++i) mine[((c * NA + a2) * 4 + i) * 32 + lane] = acc[c][a2][i];
    __threadfence();
    __syncwarp();
    int prior = 0;
    if (lane == 0) prior = atomicAdd(&v.counters[item.split], 1);
    prior = __shfl_sync(0xFFFFFFFFu, prior, 0);
    if (prior != sg.nchunks - 1) return;
    __threadfence();
#pragma unroll
    for (int c = 0; c < NCOMP; ++c)
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[c][a2][i] = 0.f;
    for (int k = 0; k < sg.nchunks; ++k) {
      const float* src = v.partials + static_cast<size_t>(sg.first_slot + k) * kPartialFloats * 32;
#pragma unroll
      for (int c = 0; c < NCOMP; ++c)
#pragma unroll
        for (int a2 = 0; a2 < NA; ++a2)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[c][a2][i] += __ldcg(src + ((c * NA + a2) * 4 + i) * 32 + lane);
    }
    if (lane == 0) v.counters[item.split] = 0;  // ready for the next launch
  }

  const int32_t rows[2] = {v.group_rows[gidx * 16 + g], v.group_rows[gidx * 16 + g + 8]};
  float scale = o.scale_mul;
  if (o.scale_ptr) {
    const float sp = *o.scale_ptr;
    scale *= o.scale_inv ? 1.0f / sp : sp;
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
      float w = scale;
      if constexpr (EPI == EPI_PANEL) {
        if (o.density) w *= o.density[row];
      }
#pragma unroll
      for (int a2 = 0; a2 < NA; ++a2) {
        const int coil = 4 * a2 + t;
        float re = acc[0][a2][2 * hr], im = acc[0][a2][2 * hr + 1];
        if constexpr (NCOMP == 2) {
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
          __half hr_, rr_, hi_, ri_;
          split_hi_res(re, hr_, rr_);
          split_hi_res(im, hi_, ri_);
          uint32_t* rowp = reinterpret_cast<uint32_t*>(o.panel + static_cast<size_t>(row) * ROWH);
          rowp[coil] = pack_half2(hr_, hi_);
          rowp[C + coil] = pack_half2(rr_, ri_);
        }
      }
    }
  }
}

template <int ROWH, bool SPLIT, int NCOMP, int EPI, bool CONJ>
static void launch_interp_t(const InterpView& v, const __half* panel, const InterpOut& o, cudaStream_t s) {
  const int blocks = (v.n_items + kInterpWarps - 1) / kInterpWarps;
  const size_t smem = static_cast<size_t>(kInterpWarps) * 2 * 32 * ROWH * 2;
  auto k = interp_mmasp_kernel<ROWH, SPLIT, NCOMP, EPI, CONJ>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (blocks > 0) k<<<blocks, kInterpWarps * 32, smem, s>>>(v, panel, o);
}

template <int ROWH>
static void dispatch_epi(const InterpView& v, const __half* panel, int epi, bool conj, const InterpOut& o, cudaStream_t s) {
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

// ------------------------------------------------------------------------------------------
// FFT endpoints. One warp per coil (blockDim = 32*C), one CTA per image row / grid column.
// ------------------------------------------------------------------------------------------
template <int G>
struct FftSmem {
  static constexpr int SCR = WarpFftShape<G>::SCRATCH;
};

__device__ __forceinline__ void load_twiddles(float2* tw_s, const float2* tw, int G) {
  for (int i = threadIdx.x; i < G; i += blockDim.x) tw_s[i] = tw[i];
}

// Forward rows (x-stage). Image row i0 -> z1[q1][i0][c] for all q1. Fuses the SENSE
// multiply, deapodization, power-of-two panel scaling, zero-padding and (CG) p = r + beta p.
// Reference: fft512_rows4_shared16_pad_scale<true> (nufft_custom_fft_forward_bench.cu:1600-1844).
template <int G>
__global__ void fwd_rows_kernel(FftArgs f, const float2* __restrict__ x, float2* __restrict__ z1, int mode,
                                float2* __restrict__ p, const float2* __restrict__ r, const double* __restrict__ parts,
                                int nparts, CgState* __restrict__ st, int iter) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  float2* tw_s = reinterpret_cast<float2*>(sm);
  float2* row_s = tw_s + G;                        // [N]
  float2* out_s = row_s + f.N;                     // [G][C]
  float2* scr = out_s + G * f.C;                   // [C][SCR]
  __shared__ double red[33];
  const int i0 = blockIdx.x, N = f.N, C = f.C;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(tw_s, f.tw, G);
  const double total = sum_partials(parts, nparts, red);
  float sigma;
  if (mode == 0) {
    const double count = static_cast<double>(N) * N * (f.smaps ? 1 : C);
    sigma = pow2_scale(total, count, kPanelTarget);
    if (i0 == 0 && threadIdx.x == 0) st->sigma_x = sigma;
    if (f.smaps) {
      for (int i = threadIdx.x; i < N; i += blockDim.x) row_s[i] = x[static_cast<size_t>(i0) * N + i];
    }
  } else {
    const double rho = total;
    sigma = pow2_scale(rho, static_cast<double>(N) * N, kPanelTarget);
    const double beta = iter == 0 ? 0.0 : rho / fmax(st->rho[iter - 1], 1e-30);
    if (i0 == 0 && threadIdx.x == 0) {
      st->rho[iter] = rho;
      st->beta[iter] = beta;
      st->sigma[iter] = sigma;
    }
    const float bf = static_cast<float>(beta);
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const size_t idx = static_cast<size_t>(i0) * N + i;
      const float2 rv = r[idx];
      float2 pv = rv;
      if (iter > 0) {
        const float2 po = p[idx];
        pv = make_float2(rv.x + bf * po.x, rv.y + bf * po.y);
      }
      p[idx] = pv;
      row_s[i] = pv;
    }
  }
  __syncthreads();
  const float scl = sigma / static_cast<float>(G);
  if (warp < C) {
    const int c = warp;
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = lane + 32 * j;
      int i1 = n + f.shift;
      if (i1 >= G) i1 -= G;
      float2 val = make_float2(0.f, 0.f);
      if (i1 < N) {
        const size_t pix = static_cast<size_t>(i0) * N + i1;
        const float d = f.scaling[pix] * scl;
        if (f.smaps) {
          val = cscale(cmul(row_s[i1], f.smaps[static_cast<size_t>(c) * N * N + pix]), d);
        } else {
          val = cscale(x[static_cast<size_t>(c) * N * N + pix], d);
        }
      }
      v[j] = val;
    }
    warp_fft<G, false>(v, scr + c * FftSmem<G>::SCR, tw_s);
#pragma unroll
    for (int m = 0; m < P; ++m) out_s[warp_fft_out_index<G>(m) * C + c] = v[m];
  }
  __syncthreads();
  // z1[q1][i0][c]: C contiguous values per q1
  for (int e = threadIdx.x; e < G * C; e += blockDim.x) {
    const int q1 = e / C, c = e - q1 * C;
    z1[(static_cast<size_t>(q1) * N + i0) * C + c] = out_s[e];
  }
}

// Forward columns (y-stage): z1[q1][*][c] -> panel rows q1*G + q0, FP16 hi | res.
// Reference: fft512_allcoils1_shared16_to_n16 (nufft_custom_fft_forward_bench.cu:538-747).
template <int G>
__global__ void fwd_cols_kernel(FftArgs f, const float2* __restrict__ z1, __half* __restrict__ panel) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  float2* tw_s = reinterpret_cast<float2*>(sm);
  float2* in_s = tw_s + G;               // [N][C]
  float2* scr = in_s + f.N * f.C;        // [C][SCR]
  uint32_t* out_s = reinterpret_cast<uint32_t*>(scr + f.C * FftSmem<G>::SCR);  // [G][2C] half2
  const int q1 = blockIdx.x, N = f.N, C = f.C;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(tw_s, f.tw, G);
  {
    const float4* src = reinterpret_cast<const float4*>(z1 + static_cast<size_t>(q1) * N * C);
    float4* dst = reinterpret_cast<float4*>(in_s);
    for (int i = threadIdx.x; i < N * C / 2; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  if (warp < C) {
    const int c = warp;
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
      const int n = lane + 32 * j;
      int i0 = n + f.shift;
      if (i0 >= G) i0 -= G;
      v[j] = i0 < N ? in_s[i0 * C + c] : make_float2(0.f, 0.f);
    }
    warp_fft<G, false>(v, scr + c * FftSmem<G>::SCR, tw_s);
#pragma unroll
    for (int m = 0; m < P; ++m) {
      const int q0 = warp_fft_out_index<G>(m);
      __half hr, rr, hi, ri;
      split_hi_res(v[m].x, hr, rr);
      split_hi_res(v[m].y, hi, ri);
      out_s[q0 * 2 * C + c] = pack_half2(hr, hi);
      out_s[q0 * 2 * C + C + c] = pack_half2(rr, ri);
    }
  }
  __syncthreads();
  const int4* src = reinterpret_cast<const int4*>(out_s);
  int4* dst = reinterpret_cast<int4*>(panel + static_cast<size_t>(q1) * G * 4 * C);
  for (int i = threadIdx.x; i < G * C / 2; i += blockDim.x) dst[i] = src[i];
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
      __half hr, rr, hi_, ri;
      split_hi_res(val.x * w, hr, rr);
      split_hi_res(val.y * w, hi_, ri);
      hi[k] = pack_half2(hr, hi_);
      res[k] = pack_half2(rr, ri);
    }
    *reinterpret_cast<uint4*>(pu + row * 2 * C + 4 * q) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4*>(pu + row * 2 * C + C + 4 * q) = make_uint4(res[0], res[1], res[2], res[3]);
  }
}

// Inverse columns: grid rows q1*G + [0,G) (all coils) -> w1[q1][i0][c], i0 < N (crop).
// Reference: ifft512_rows8_regular_transposed (nufft_custom_fft_forward_bench.cu:1463-1515).
template <int G>
__global__ void inv_cols_kernel(FftArgs f, const float2* __restrict__ grid, float2* __restrict__ w1) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  float2* tw_s = reinterpret_cast<float2*>(sm);
  float2* in_s = tw_s + G;               // [G][C]
  float2* out_s = in_s + G * f.C;        // [N][C]
  float2* scr = out_s + f.N * f.C;       // [C][SCR]
  const int q1 = blockIdx.x, N = f.N, C = f.C;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(tw_s, f.tw, G);
  {
    const float4* src = reinterpret_cast<const float4*>(grid + static_cast<size_t>(q1) * G * C);
    float4* dst = reinterpret_cast<float4*>(in_s);
    for (int i = threadIdx.x; i < G * C / 2; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  if (warp < C) {
    const int c = warp;
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) v[j] = in_s[(lane + 32 * j) * C + c];
    warp_fft<G, true>(v, scr + c * FftSmem<G>::SCR, tw_s);
#pragma unroll
    for (int m = 0; m < P; ++m) {
      int i0 = warp_fft_out_index<G>(m) + f.shift;
      if (i0 >= G) i0 -= G;
      if (i0 < N) out_s[i0 * C + c] = v[m];
    }
  }
  __syncthreads();
  const float4* src = reinterpret_cast<const float4*>(out_s);
  float4* dst = reinterpret_cast<float4*>(w1 + static_cast<size_t>(q1) * N * C);
  for (int i = threadIdx.x; i < N * C / 2; i += blockDim.x) dst[i] = src[i];
}

// Inverse rows + crop + deapodization + SENSE coil combine (+ CG epilogues).
// Reference: ifft512_rows8_regular_crop_scale (nufft_custom_fft_forward_bench.cu:1517-1552)
// followed by sense_combine_scaled (nufft_fp16x2_cg_bench.cu:27-54).
template <int G>
__global__ void inv_rows_kernel(FftArgs f, const float2* __restrict__ w1, float2* __restrict__ out, int mode,
                                float2* __restrict__ x, float2* __restrict__ r, const float2* __restrict__ p,
                                double* __restrict__ parts, CgState* __restrict__ st, int iter, float inv_scale2,
                                float lambda_scaled) {
  constexpr int P = G / 32;
  extern __shared__ __align__(16) uint8_t sm[];
  float2* tw_s = reinterpret_cast<float2*>(sm);
  float2* in_s = tw_s + G;               // [G][C]
  float2* img_s = in_s + G * f.C;        // [C][N]
  float2* scr = img_s + f.N * f.C;       // [C][SCR]
  __shared__ double red[33];
  const int i0 = blockIdx.x, N = f.N, C = f.C;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  load_twiddles(tw_s, f.tw, G);
  for (int e = threadIdx.x; e < G * C; e += blockDim.x) {
    const int q1 = e / C, c = e - q1 * C;
    in_s[e] = w1[(static_cast<size_t>(q1) * N + i0) * C + c];
  }
  __syncthreads();
  if (warp < C) {
    const int c = warp;
    float2 v[P];
#pragma unroll
    for (int j = 0; j < P; ++j) v[j] = in_s[(lane + 32 * j) * C + c];
    warp_fft<G, true>(v, scr + c * FftSmem<G>::SCR, tw_s);
#pragma unroll
    for (int m = 0; m < P; ++m) {
      int i1 = warp_fft_out_index<G>(m) + f.shift;
      if (i1 >= G) i1 -= G;
      if (i1 < N) img_s[c * N + i1] = v[m];
    }
  }
  __syncthreads();
  float factor;
  if (mode == 2) factor = static_cast<float>(G) / st->sigma[iter] * inv_scale2;
  else factor = inv_scale2 / st->sigma_y;
  double dot = 0.0;
  for (int i1 = threadIdx.x; i1 < N; i1 += blockDim.x) {
    const size_t pix = static_cast<size_t>(i0) * N + i1;
    const float d = f.scaling[pix] * factor;
    if (!f.smaps) {  // coil images out [C][N][N]
      for (int c = 0; c < C; ++c) out[static_cast<size_t>(c) * N * N + pix] = cscale(img_s[c * N + i1], d);
      continue;
    }
    float2 acc = make_float2(0.f, 0.f);
    for (int c = 0; c < C; ++c) acc = cadd(acc, cmulc(img_s[c * N + i1], f.smaps[static_cast<size_t>(c) * N * N + pix]));
    acc = cscale(acc, d);
    if (mode == 0) {
      out[pix] = acc;
    } else if (mode == 1) {
      r[pix] = acc;
      x[pix] = make_float2(0.f, 0.f);
      dot += static_cast<double>(acc.x) * acc.x + static_cast<double>(acc.y) * acc.y;
    } else {
      const float2 pv = p[pix];
      acc.x += lambda_scaled * pv.x;
      acc.y += lambda_scaled * pv.y;
      out[pix] = acc;
      dot += static_cast<double>(pv.x) * acc.x + static_cast<double>(pv.y) * acc.y;
    }
  }
  if (mode != 0) {
    const double t = block_sum(dot, red);
    if (threadIdx.x == 0) parts[i0] = t;
  }
}

__global__ void cg_update_kernel(int N, float2* __restrict__ x, float2* __restrict__ r, const float2* __restrict__ p,
                                 const float2* __restrict__ ap, const double* __restrict__ pap_parts,
                                 double* __restrict__ rr_parts, CgState* __restrict__ st, int iter) {
  __shared__ double red[33];
  const double pap = sum_partials(pap_parts, N, red);
  const double rho = st->rho[iter];
  const bool ok = isfinite(pap) && pap > 0.0;
  const double alpha = ok ? rho / pap : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->pap[iter] = pap;
    st->alpha[iter] = alpha;
    if (!ok) st->curvature_ok = 0;
    if (!isfinite(pap)) st->finite_ok = 0;
    st->completed = iter + 1;
  }
  const float af = static_cast<float>(alpha);
  double acc = 0.0;
  const int i0 = blockIdx.x;
  for (int i1 = threadIdx.x; i1 < N; i1 += blockDim.x) {
    const size_t pix = static_cast<size_t>(i0) * N + i1;
    const float2 pv = p[pix], av = ap[pix];
    float2 xv = x[pix], rv = r[pix];
    xv.x += af * pv.x;
    xv.y += af * pv.y;
    rv.x -= af * av.x;
    rv.y -= af * av.y;
    x[pix] = xv;
    r[pix] = rv;
    acc += static_cast<double>(rv.x) * rv.x + static_cast<double>(rv.y) * rv.y;
  }
  const double t = block_sum(acc, red);
  if (threadIdx.x == 0) rr_parts[i0] = t;
}

__global__ void cg_finish_kernel(int N, const double* __restrict__ rr_parts, CgState* __restrict__ st, int iters) {
  __shared__ double red[33];
  const double rho = sum_partials(rr_parts, N, red);
  if (threadIdx.x == 0) {
    st->rho[iters] = rho;
    if (!isfinite(rho)) st->finite_ok = 0;
  }
}

// ------------------------------------------------------------------------------------------
// Launchers
// ------------------------------------------------------------------------------------------
template <int G>
static size_t fwd_rows_smem(const FftArgs& f) {
  return sizeof(float2) * (G + f.N + static_cast<size_t>(G) * f.C + static_cast<size_t>(f.C) * FftSmem<G>::SCR);
}
template <int G>
static size_t fwd_cols_smem(const FftArgs& f) {
  return sizeof(float2) * (G + static_cast<size_t>(f.N) * f.C + static_cast<size_t>(f.C) * FftSmem<G>::SCR) +
         sizeof(uint32_t) * static_cast<size_t>(G) * 2 * f.C;
}
template <int G>
static size_t inv_cols_smem(const FftArgs& f) {
  return sizeof(float2) * (G + static_cast<size_t>(G) * f.C + static_cast<size_t>(f.N) * f.C +
                           static_cast<size_t>(f.C) * FftSmem<G>::SCR);
}
template <int G>
static size_t inv_rows_smem(const FftArgs& f) {
  return inv_cols_smem<G>(f);
}

template <class K>
static void ensure_smem(K k, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

#define TSN_G_SWITCH(G_, ...)                                  \
  switch (G_) {                                                \
    case 128: { constexpr int GG = 128; __VA_ARGS__; } break;  \
    case 256: { constexpr int GG = 256; __VA_ARGS__; } break;  \
    case 512: { constexpr int GG = 512; __VA_ARGS__; } break;  \
    case 1024: { constexpr int GG = 1024; __VA_ARGS__; } break; \
    default: break;                                            \
  }

void launch_fwd_rows(const FftArgs& f, const float2* x, float2* z1, int mode, float2* p, const float2* r,
                     const double* partials, int nparts, CgState* st, int iter, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t sm = fwd_rows_smem<GG>(f);
    ensure_smem(fwd_rows_kernel<GG>, sm);
    fwd_rows_kernel<GG><<<f.N, 32 * f.C, sm, s>>>(f, x, z1, mode, p, r, partials, nparts, st, iter);
  });
}

void launch_fwd_cols(const FftArgs& f, const float2* z1, __half* panel, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t sm = fwd_cols_smem<GG>(f);
    ensure_smem(fwd_cols_kernel<GG>, sm);
    fwd_cols_kernel<GG><<<f.G, 32 * f.C, sm, s>>>(f, z1, panel);
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
    const size_t sm = inv_cols_smem<GG>(f);
    ensure_smem(inv_cols_kernel<GG>, sm);
    inv_cols_kernel<GG><<<f.G, 32 * f.C, sm, s>>>(f, grid, w1);
  });
}

void launch_inv_rows(const FftArgs& f, const float2* w1, float2* out, int mode, float2* x, float2* r, const float2* p,
                     double* partials, CgState* st, int iter, float inv_scale2, float lambda_scaled, cudaStream_t s) {
  TSN_G_SWITCH(f.G, {
    const size_t sm = inv_rows_smem<GG>(f);
    ensure_smem(inv_rows_kernel<GG>, sm);
    inv_rows_kernel<GG><<<f.N, 32 * f.C, sm, s>>>(f, w1, out, mode, x, r, p, partials, st, iter, inv_scale2,
                                                   lambda_scaled);
  });
}

void launch_cg_update(int N, float2* x, float2* r, const float2* p, const float2* ap, const double* pap_parts,
                      double* rr_parts, CgState* st, int iter, cudaStream_t s) {
  cg_update_kernel<<<N, 256, 0, s>>>(N, x, r, p, ap, pap_parts, rr_parts, st, iter);
}

void launch_cg_finish(int N, const double* rr_parts, CgState* st, int iters, cudaStream_t s) {
  cg_finish_kernel<<<1, 256, 0, s>>>(N, rr_parts, st, iters);
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
