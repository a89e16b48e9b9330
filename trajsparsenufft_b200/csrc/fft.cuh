// Warp-level FFT of length G = 32*P (P in {4, 8, 16, 32}, or R times such a length for
// R in {3, 5}; see FftPlan) in FP32 registers.
//
// One warp transforms one G-point sequence held as P values per lane
// (lane l, register j <-> element l + 32 j). Four-step decomposition G = P x 32:
//   1. P-point DFT over j in registers (radix-2 DIT, compile-time twiddles),
//   2. twiddle W_G^(l k),
//   3. transpose through a padded per-warp shared buffer,
//   4. 32-point DFTs over l, each split across T = 32/P lanes: a P-point register DFT
//      per lane, twiddle W_32^(h m), then a T-point DFT across the T lanes by shuffles.
// Output: lane (k = lane / T, h = lane % T) holds X[k + P q + P^2 k3] in register m, with
// (q, k3) from the cross-lane step (warp_fft_pow2_out_index).
// Forward = exp(-2 pi i nk/G), inverse = exp(+2 pi i nk/G), both unnormalized.
// Twiddles are FP64-computed, FP32-stored tables (host fills them once per plan).
// The reference's FFT endpoints are SIMT FP32 shared-memory radix-8/16/32 kernels
// (nufft_custom_fft_forward_bench.cu:918-999, :1463-1552); this is an independent design.
#pragma once

#include "device.cuh"

namespace tsn {
namespace dev {

// exp(-2 pi i e / 1024), e in [0, 1024); defined here, filled once per process by the host.
// (included by exactly one translation unit)
__constant__ float2 c_w1024[1024];

// exp(-2 pi i j / R) for R = 3 and 5, filled with the plan twiddle tables' FP64 expression
// (so equal to tw[B j] of a G = R B plan): uniform across lanes, read as constant operands
__constant__ float2 c_wr3[3];
__constant__ float2 c_wr5[5];

template <int R, bool INV>
__device__ __forceinline__ float2 radix_twiddle(int j) {
  const float2 w = R == 3 ? c_wr3[j] : c_wr5[j];
  return INV ? make_float2(w.x, -w.y) : w;
}

template <bool INV>
__device__ __forceinline__ float2 const_twiddle(int e1024) {
  const float2 w = c_w1024[e1024 & 1023];
  return INV ? make_float2(w.x, -w.y) : w;
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
__host__ __device__ constexpr int bitrev(int x, int bits) {
  return bits == 0 ? 0 : (((x & 1) << (bits - 1)) | bitrev(x >> 1, bits - 1));
}

// One radix-2 DIT stage of butterfly span LEN, then the next stage (compile-time
// recursion keeps every register index a constant, so the array never spills to
// local memory).
template <int P, bool INV, int LEN>
struct DitStage {
  static __device__ __forceinline__ void run(float2 (&a)[P]) {
    constexpr int HALF = LEN / 2;
#pragma unroll
    for (int i = 0; i < P; i += LEN) {
#pragma unroll
      for (int j = 0; j < HALF; ++j) {
        const float2 u = a[i + j];
        float2 t = a[i + j + HALF];
        if (j != 0) {
          if (4 * j == LEN) {  // W_LEN^(LEN/4) = -i (forward) / +i (inverse)
            t = INV ? make_float2(-t.y, t.x) : make_float2(t.y, -t.x);
          } else {
            t = cmul(const_twiddle<INV>(j * (1024 / LEN)), t);
          }
        }
        a[i + j] = cadd(u, t);
        a[i + j + HALF] = csub(u, t);
      }
    }
    DitStage<P, INV, LEN * 2>::run(a);
  }
};
template <int P, bool INV>
struct DitStage<P, INV, 2 * P> {
  static __device__ __forceinline__ void run(float2 (&)[P]) {}
};

template <int P, int I>
struct BitReverse {
  static __device__ __forceinline__ void run(float2 (&a)[P]) {
    constexpr int J = bitrev(I, ilog2(P));
    if constexpr (J > I) {
      const float2 t = a[I];
      a[I] = a[J];
      a[J] = t;
    }
    BitReverse<P, I + 1>::run(a);
  }
};
template <int P>
struct BitReverse<P, P> {
  static __device__ __forceinline__ void run(float2 (&)[P]) {}
};

// In-register DFT of length P (power of two), natural order in and out.
template <int P, bool INV>
__device__ __forceinline__ void dft_reg(float2 (&a)[P]) {
  BitReverse<P, 0>::run(a);
  DitStage<P, INV, 2>::run(a);
}

template <int G>
struct WarpFftShape {
  static constexpr int P = G / 32;
  static constexpr int T = 32 / P;
  static constexpr int PITCH = 32 + T;        // padded row pitch (float2) of the transpose buffer
  static constexpr int SCRATCH = P * PITCH;   // float2 per warp
  static_assert(P * 32 == G && (P & (P - 1)) == 0 && P >= 4 && P <= 32, "G must be 32*P, P in {4..32}");
};

// Power-of-two warp FFT. tw: shared table exp(-2 pi i e / (G * TS)), e in [0, G * TS); the
// transform reads every TS-th entry (TS > 1 when it is the base of a mixed-radix length).
template <int G, bool INV, int TS = 1>
__device__ __forceinline__ void warp_fft_pow2(float2 (&v)[G / 32], float2* scratch, const float2* tw) {
  using S = WarpFftShape<G>;
  constexpr int P = S::P, T = S::T;
  const int lane = threadIdx.x & 31;
  dft_reg<P, INV>(v);
  // twiddles W_G^(lane k): the power-of-two exponents come from the table, the others are
  // products of at most three of them (W^k = W^(high bit of k) W^(rest)), which trades shared
  // memory loads for FP32 multiplies at an error of a few ulp
  {
    float2 wk[P];
    wk[0] = make_float2(1.f, 0.f);
#pragma unroll
    for (int k = 1; k < P; ++k) {
      if ((k & (k - 1)) == 0) {
        wk[k] = tw[TS * ((lane * k) & (G - 1))];
        if (INV) wk[k].y = -wk[k].y;
      } else {
        const int hb = 1 << (31 - __clz(k));
        wk[k] = cmul(wk[hb], wk[k - hb]);
      }
      v[k] = cmul(v[k], wk[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < P; ++k) scratch[k * S::PITCH + lane] = v[k];
  __syncwarp();
  const int kk = lane / T, h = lane % T;
#pragma unroll
  for (int i = 0; i < P; ++i) v[i] = scratch[kk * S::PITCH + T * i + h];
  __syncwarp();
  dft_reg<P, INV>(v);
  if (T > 1) {
#pragma unroll
    for (int m = 1; m < P; ++m) {
      float2 w = tw[TS * ((h * m * P) & (G - 1))];
      if (INV) w.y = -w.y;
      v[m] = cmul(v[m], w);
    }
    if (T == 2) {
#pragma unroll
      for (int m = 0; m < P; ++m) {
        float2 o;
        o.x = __shfl_xor_sync(0xFFFFFFFFu, v[m].x, 1);
        o.y = __shfl_xor_sync(0xFFFFFFFFu, v[m].y, 1);
        v[m] = h == 0 ? cadd(v[m], o) : csub(o, v[m]);
      }
    } else if (T == 4) {
      // The 4-point DFTs across lanes go through the warp scratch instead of shuffles: lane
      // (kk, h) takes the Q = P/4 columns m = h Q + i and, for each, the values of the four
      // lanes kk*4 + h2. Rows are XOR-swizzled by the column group m / Q, which makes both the
      // row writes and these reads conflict-free. Then a register DFT-4 per column.
      constexpr int Q = P / 4;
      __syncwarp();
#pragma unroll
      for (int m = 0; m < P; ++m) scratch[m * 32 + (lane ^ (m / Q))] = v[m];
      __syncwarp();
      float2 u[Q][4];
#pragma unroll
      for (int i = 0; i < Q; ++i)
#pragma unroll
        for (int h2 = 0; h2 < 4; ++h2) u[i][h2] = scratch[(h * Q + i) * 32 + ((kk * 4 + h2) ^ h)];
      __syncwarp();
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        dft_reg<4, INV>(u[i]);
#pragma unroll
        for (int k3 = 0; k3 < 4; ++k3) v[i * 4 + k3] = u[i][k3];
      }
    } else {
      // T == 8 (P == 4): each 8-point DFT across lanes is split over a lane pair. Lane (kk, h)
      // takes column m = h / 2 and the four values of lanes kk*8 + 2 j + e (e = h % 2) from the
      // scratch (XOR swizzle 2m: conflict-free), a register DFT-4 gives the even (e = 0) or odd
      // (e = 1) half, the odd half is multiplied by W_8^k, and one shuffle exchange across the
      // pair forms X[k] = E[k] + W_8^k O[k] (e = 0) and X[k + 4] = E[k] - W_8^k O[k] (e = 1).
      __syncwarp();
#pragma unroll
      for (int m = 0; m < P; ++m) scratch[m * 32 + (lane ^ (2 * m))] = v[m];
      __syncwarp();
      const int mm = h >> 1, e = h & 1;
      float2 u[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) u[j] = scratch[mm * 32 + ((kk * 8 + 2 * j + e) ^ (2 * mm))];
      __syncwarp();
      dft_reg<4, INV>(u);
#pragma unroll
      for (int k = 1; k < 4; ++k)
        if (e) u[k] = cmul(u[k], const_twiddle<INV>(k * 128));  // W_8^k = exp(-2 pi i k / 8)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float2 o;
        o.x = __shfl_xor_sync(0xFFFFFFFFu, u[k].x, 1);
        o.y = __shfl_xor_sync(0xFFFFFFFFu, u[k].y, 1);
        v[k] = e ? csub(o, u[k]) : cadd(u[k], o);
      }
    }
  }
}

// Output element index held in register m after warp_fft_pow2<G>: lane (kk = lane / T,
// h = lane % T) holds X[kk + P q + P^2 k3] with, by the cross-lane step,
//   T <= 2: q = m, k3 = h;
//   T == 4: q = h (P/4) + m / 4, k3 = m % 4;
//   T == 8: q = h / 2, k3 = m + 4 (h % 2).
template <int G>
__device__ __forceinline__ int warp_fft_pow2_out_index(int m) {
  using S = WarpFftShape<G>;
  constexpr int P = S::P, T = S::T;
  const int lane = threadIdx.x & 31;
  const int kk = lane / T, h = lane % T;
  if constexpr (T == 4) return kk + P * (h * (P / 4) + m / 4) + P * P * (m % 4);
  else if constexpr (T == 8) return kk + P * (h >> 1) + P * P * (m + 4 * (h & 1));
  else return kk + P * m + P * P * h;
}

// Lengths G = R * B with R in {1, 3, 5} and a power-of-two base B = 32 * 2^k >= 128; the
// radix-3 and radix-5 factors give the grids 2N of image sizes N = 192 and 320.
template <int G>
struct FftPlan {
  static constexpr int R = (G % 5 == 0) ? 5 : (G % 3 == 0) ? 3 : 1;
  static constexpr int B = G / R;                           // power-of-two base length
  static constexpr int P = G / 32;                          // registers per lane
  static constexpr int PB = B / 32;                         // registers per lane of one base FFT
  static constexpr int SCRATCH = WarpFftShape<B>::SCRATCH;  // float2 per warp
};

// Input element held in register j before warp_fft: lane + 32 j for power-of-two lengths;
// for G = R B, register r * PB + j' holds x[R (lane + 32 j') + r] (decimation by R).
template <int G>
__device__ __forceinline__ int warp_fft_in_index(int j) {
  using F = FftPlan<G>;
  const int lane = threadIdx.x & 31;
  if constexpr (F::R == 1) return lane + 32 * j;
  else return F::R * (lane + 32 * (j % F::PB)) + j / F::PB;
}

// Output element index held in register m after warp_fft.
template <int G>
__device__ __forceinline__ int warp_fft_out_index(int m) {
  using F = FftPlan<G>;
  if constexpr (F::R == 1) return warp_fft_pow2_out_index<G>(m);
  else return warp_fft_pow2_out_index<F::B>(m % F::PB) + F::B * (m / F::PB);
}

// Warp FFT of length G (see FftPlan). tw: shared table exp(-2 pi i e / G), e in [0, G).
// For G = R B: R base FFTs of the decimated sequences Y_r, then for each base output k a
// radix-R step in registers, X[k + B q] = sum_r W_G^{r k} Y_r[k] W_R^{r q}.
template <int G, bool INV>
__device__ __forceinline__ void warp_fft(float2 (&v)[G / 32], float2* scratch, const float2* tw) {
  using F = FftPlan<G>;
  if constexpr (F::R == 1) {
    warp_fft_pow2<G, INV>(v, scratch, tw);
  } else {
    constexpr int R = F::R, B = F::B, PB = F::PB;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 sub[PB];
#pragma unroll
      for (int j = 0; j < PB; ++j) sub[j] = v[r * PB + j];
      warp_fft_pow2<B, INV, R>(sub, scratch, tw);  // W_B^e = tw[R e]
#pragma unroll
      for (int j = 0; j < PB; ++j) v[r * PB + j] = sub[j];
    }
#pragma unroll
    for (int m = 0; m < PB; ++m) {
      const int k = warp_fft_pow2_out_index<B>(m);
      float2 t[R];
      t[0] = v[m];
      // W_G^(r k), r < R: W^k and (R == 5) W^2k from the table, the rest as products
      float2 wr[R];
      wr[1] = tw[k];
      if (INV) wr[1].y = -wr[1].y;
      if constexpr (R == 3) {
        wr[2] = cmul(wr[1], wr[1]);
      } else {
        wr[2] = tw[2 * k];  // 2 k < G
        if (INV) wr[2].y = -wr[2].y;
        wr[3] = cmul(wr[2], wr[1]);
        wr[4] = cmul(wr[2], wr[2]);
      }
#pragma unroll
      for (int r = 1; r < R; ++r) t[r] = cmul(v[r * PB + m], wr[r]);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        float2 acc = t[0];
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const float2 w = radix_twiddle<R, INV>((r * q) % R);  // W_R^{r q}, a constant operand
          acc = cadd(acc, cmul(t[r], w));
        }
        v[q * PB + m] = acc;
      }
    }
  }
}

}  // namespace dev
}  // namespace tsn
