// Device helpers shared by the sm_100a kernels: complex arithmetic, asynchronous copies,
// ldmatrix / warp sparse MMA wrappers, FP16 hi+residual split.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tsn {
namespace dev {

// Complex add / subtract as one paired FP32 instruction (sm_100 FADD2; each lane rounds
// exactly like the scalar add).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Programmatic dependent launch. pdl_wait blocks until the kernel this one was launched
// behind (with cudaLaunchAttributeProgrammaticStreamSerialization) has completed and its
// writes are visible; pdl_trigger lets the next such kernel of the stream start its prologue.
// Both return at once in a kernel launched without the attribute.  A kernel reads nothing
// that an earlier kernel may write, and writes nothing, before pdl_wait.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src));
}
// 16-byte copy when `live`, else a 16-byte zero store to the same shared address (no global
// read); predicated, so a warp with mixed lanes does not branch.
__device__ __forceinline__ void cp_async16_or_zero(void* smem_dst, const void* gmem_src, bool live) {
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  setp.ne.b32 p, %2, 0;\n"
      "  @p cp.async.cg.shared.global [%0], [%1], 16;\n"
      "  @!p st.shared.v4.u32 [%0], {%3, %3, %3, %3};\n"
      "}\n" ::"r"(smem_u32(smem_dst)),
      "l"(gmem_src), "r"(static_cast<int>(live)), "r"(0)
      : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Four 8x8 b16 matrices (rows addressed by lanes 0-7, 8-15, 16-23, 24-31).
__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void* smem_row) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(smem_row)));
}

// Four transposed 8x8 b16 matrices (rows addressed by lanes 0-7, 8-15, 16-23, 24-31).
__device__ __forceinline__ void ldmatrix_x4_trans(uint32_t (&r)[4], const void* smem_row) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(smem_row)));
}

// Warp-level 2:4 sparse MMA m16n8k32, FP16 inputs, FP32 accumulate, metadata selector 0.
__device__ __forceinline__ void mma_sp_16832(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[4],
                                             uint32_t meta) {
  asm volatile(
      "mma.sp::ordered_metadata.sync.aligned.m16n8k32.row.col.f32.f16.f16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9,%10,%11}, {%0,%1,%2,%3}, %12, 0x0;\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(meta));
}

// FP32 value -> FP16 high part + FP16 residual (value - float(high)), the reference's
// split2 panel (reference_sparse_solver.py:66-76, integrated_complex_to_split2_half_rows).
__device__ __forceinline__ void split_hi_res(float v, __half& hi, __half& res) {
  hi = __float2half_rn(v);
  res = __float2half_rn(v - __half2float(hi));
}

__device__ __forceinline__ uint32_t pack_half2(__half lo, __half hi) {
  return static_cast<uint32_t>(__half_as_ushort(lo)) | (static_cast<uint32_t>(__half_as_ushort(hi)) << 16);
}

// Complex (re, im) -> packed FP16 high parts (re low, im high) and packed FP16 residuals:
// split_hi_res on each component, with the paired conversions (same rounding, same bits).
__device__ __forceinline__ void split_hi_res2(float re, float im, uint32_t& hi, uint32_t& res) {
  const __half2 h = __floats2half2_rn(re, im);
  const float2 back = __half22float2(h);
  const __half2 r = __floats2half2_rn(re - back.x, im - back.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  res = *reinterpret_cast<const uint32_t*>(&r);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

// Deterministic block sum of one double per thread (fixed reduction tree), returned to
// every thread. `scratch` holds 33 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  v = warp_sum(v);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += scratch[w];
    scratch[32] = t;
  }
  __syncthreads();
  const double t = scratch[32];
  __syncthreads();  // scratch may be reused by the caller's next block_sum
  return t;
}

// Three deterministic block sums at once (one pass of barriers); `scratch` holds 99 doubles.
__device__ __forceinline__ double3 block_sum3(double a, double b, double c, double* scratch) {
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    scratch[warp] = a;
    scratch[33 + warp] = b;
    scratch[66 + warp] = c;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int nw = (blockDim.x + 31) >> 5;
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += scratch[33 * threadIdx.x + w];
    scratch[33 * threadIdx.x + 32] = t;
  }
  __syncthreads();
  const double3 t = make_double3(scratch[32], scratch[65], scratch[98]);
  __syncthreads();
  return t;
}

// Four deterministic block sums at once; `scratch` holds 132 doubles.
__device__ __forceinline__ double4 block_sum4(double a, double b, double c, double d, double* scratch) {
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  d = warp_sum(d);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    scratch[warp] = a;
    scratch[33 + warp] = b;
    scratch[66 + warp] = c;
    scratch[99 + warp] = d;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int nw = (blockDim.x + 31) >> 5;
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += scratch[33 * threadIdx.x + w];
    scratch[33 * threadIdx.x + 32] = t;
  }
  __syncthreads();
  const double4 t = make_double4(scratch[32], scratch[65], scratch[98], scratch[131]);
  __syncthreads();
  return t;
}

// Power-of-two scale bringing rms to ~target (FP16 rounding commutes with it).
__device__ __forceinline__ float pow2_scale(double sum_sq, double count, float target) {
  const double rms = sqrt(sum_sq / count);
  if (!(rms > 0.0) || !isfinite(rms)) return 1.0f;
  const double e = rint(log2(static_cast<double>(target) / rms));
  return static_cast<float>(exp2(fmin(fmax(e, -100.0), 100.0)));
}

}  // namespace dev
}  // namespace tsn
