// Kernel argument structs and launchers of the sm_100a operator pipeline.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tsn {

constexpr int kMaxCgIter = 256;
constexpr int kNormParts = 296;      // 2 x 148 SMs
constexpr float kPanelTarget = 8.0f; // rms target of the FP16 panels (power-of-two scaling)

// Device scalar state of one solve (FP64 CG scalars, per-iteration panel scales).
struct CgState {
  double rho[kMaxCgIter + 2];    // <r_k, r_k>
  double pap[kMaxCgIter + 1];    // Re <p_k, A p_k>
  double alpha[kMaxCgIter + 1];
  double beta[kMaxCgIter + 1];
  float sigma[kMaxCgIter + 2];   // forward panel scale of p_k
  float sigma_y;                 // sample panel scale of the measurement / adjoint input
  float sigma_x;                 // forward panel scale of a plain forward call
  int curvature_ok;
  int finite_ok;
  int completed;
  int pad_;
};

// Interpolation view on the device: AoS tile records, in the order the persistent warps
// stream them (warp w owns records [warp_ranges[w].x, warp_ranges[w].y))
//   [0,128)                  int32 gather row per column (internal panel row), -1 = dead
//                            column (all coefficients zero: zero-filled, never read)
//   [128+576c, +512)         f16 compressed A of component c, [16][16]
//   [640+576c, +64)          u32 mma.sp pair metadata of component c, [16]
//   [128+576n, +16)          RecordInfo (n = component count)
//   [128+576n+16, +48)       24-bit output row of each of the 16 tile rows (little endian;
//                            pad rows are the ones whose live bit in RecordInfo.flags is clear)
// A one-component record is 768 bytes: records and the gathered rows after them stay on
// 128-byte boundaries.
// Work item: a run of at most kChunkTiles tiles of one 16-row group. Groups with more
// tiles are split; their chunks write raw accumulators to `partials` and the warp that
// arrives last (counter) sums all chunks in chunk order, so results stay deterministic.
constexpr int kChunkTiles = 8;
// A group is cut into at most this many chunks (longer chunks for longer groups), so the
// warp that reduces a split group reads a bounded number of partials.
constexpr int kMaxChunks = 64;
constexpr int kRecInfoBytes = 64;
constexpr int32_t kRecRowPad = 0xFFFFFF;                      // row field of a pad row
constexpr int64_t kMaxInterpRows = static_cast<int64_t>(1) << 24;  // output rows addressable by a record
constexpr int kRecFirst = 1;       // first tile of a work item
constexpr int kRecLast = 2;        // last tile of a work item: apply the epilogue
constexpr int kRecLiveShift = 16;  // flags bit 16 + s: tile row s is a real output row
struct RecordInfo {
  int32_t flags;
  int32_t split;       // -1: whole group; else split-group id (counter index)
  int32_t first_slot;  // partials slot of chunk 0 of the split group
  int32_t chunk;       // chunk index | nchunks << 16
};
static_assert(sizeof(RecordInfo) == 16, "record info is 16 bytes");
__host__ __device__ constexpr int record_bytes(int ncomp) { return 128 + 576 * ncomp + kRecInfoBytes; }

struct InterpView {
  const uint8_t* records = nullptr;
  int32_t* counters = nullptr;          // one per split group, zero between launches
  float* partials = nullptr;            // [slots][kPartialFloats][32]
  const int2* warp_ranges = nullptr;    // per persistent warp: [first record, end record)
  int32_t n_warps = 0;
  int32_t groups = 0;
  int32_t ncomp = 0;
  int32_t rec_bytes = 0;
  int32_t stages = 3;                   // per-warp ring depth: 3, or 4 when the gathered panel exceeds L2
  int32_t programmatic = 1;             // 1: launched with programmatic dependent launch (0 for the
                                        //    1/share slices of batched cases, which share the SMs)
  int32_t sum_components = 0;           // 1: the two components are a real coefficient's FP16 high and
                                        //    low parts, summed (else real / imaginary parts)
};
constexpr int kPartialFloats = 32;  // >= NCOMP * NA * 4 for every instantiation

enum InterpEpilogue { EPI_SAMPLES = 0, EPI_GRID = 1, EPI_PANEL = 2, EPI_RAW = 3 };

struct InterpOut {
  float2* c64 = nullptr;          // EPI_SAMPLES: [C][rows]; EPI_GRID: [rows][C]
  __half* panel = nullptr;        // EPI_PANEL: [rows][4C] (hi | res, interleaved complex)
  float* raw = nullptr;           // EPI_RAW: [rows][16]
  const float* density = nullptr; // EPI_PANEL weight per row
  const float* scale_ptr = nullptr;  // device scalar (nullable)
  int scale_inv = 0;              // use 1/(*scale_ptr)
  float scale_mul = 1.0f;
  int64_t rows = 0;               // row count (coil stride for EPI_SAMPLES)
  int32_t coils = 0;
};

struct FftArgs {
  int N = 0, G = 0, C = 0, shift = 0;   // grid position n holds image index (n + shift) mod G
  const float2* tw = nullptr;           // exp(-2 pi i e/G), e in [0,G)
  const float* scaling = nullptr;       // [N]^dims deapodization
  const float2* smaps = nullptr;        // [C][N]^dims or null
  int share = 1;                        // persistent grids use 1/share of the resident CTAs
  int dims = 2;                         // 2: image [N][N]; 3: volume [N][N][N]
  // image lines along the last axis (items of the row stages)
  __host__ __device__ int lines() const { return dims == 3 ? N * N : N; }
  // pixels (voxels) of one image
  __host__ __device__ int64_t pix() const { return static_cast<int64_t>(lines()) * N; }
  // grid lines of the first-axis stages (fwd_cols / inv_cols items)
  __host__ __device__ int gcols() const { return dims == 3 ? G * G : G; }
  // divisor applied with the panel scale before the forward FFTs (the transform's gain per
  // axis is up to G): G for images, G * 2^floor(floor(log2 G) / 2) for volumes; the
  // interpolation multiplies it back
  __host__ __device__ float gs() const {
    if (dims != 3) return static_cast<float>(G);
    int l = 0;
    while ((2 << l) <= G) ++l;
    return static_cast<float>(G) * static_cast<float>(1 << (l / 2));
  }
};

void set_twiddle_constants(cudaStream_t s);

// Grid sizes the warp FFT stages are built for: 32 * 2^k (128..1024) and 3 * 128, 5 * 128.
inline bool fft_grid_supported(int g) {
  return g == 128 || g == 256 || g == 384 || g == 512 || g == 640 || g == 1024;
}

void launch_interp(const InterpView& v, const __half* panel, int rowh, bool split, int epi, bool conj,
                   const InterpOut& o, cudaStream_t s);

// ---- interpolation on tcgen05.mma.sp (real pack, 8 coils) ------------------------------------
// Seven 16-row tiles are stacked into one M = 128 sparse A operand (rows 112..127 zero) and
// their 32 gathered panel rows side by side into one N = 7 x 32 = 224 B operand; one
// tcgen05.mma.sp (K = 32) per step, of which each tile keeps its diagonal 16 x 32 block.  The
// record stream is cut into steps of seven slot records:
//   [0, 3584)        A of slots 0..6: 512 B each, the canonical K-major layout without swizzle
//                    (rows 0-7 k-chunk 0 | rows 0-7 chunk 1 | rows 8-15 chunk 0 | chunk 1,
//                    8 rows x 16 B each)
//   [3584 + 256 j)   slot j: int32 gather row per column (-1: dead column or idle slot),
//                    [+128) u32 sparse metadata in tensor-memory lane order,
//                    [+192) RecordInfo (flags 0: idle slot), [+208) 24-bit output rows
constexpr int kTcSlots = 7;
constexpr int kTcSlotABytes = 512;
constexpr int kTcSlotInfoBytes = 256;
constexpr int kTcStepABytes = kTcSlots * kTcSlotABytes;                          // 3584
constexpr int kTcStepBytes = kTcStepABytes + kTcSlots * kTcSlotInfoBytes;        // 5376
constexpr int kTcPartialFloats = 32 * 16;  // one split-group chunk: 32 columns x 16 rows

struct InterpTcView {
  const uint8_t* steps = nullptr;      // step blocks, grouped by CTA
  const int2* cta_steps = nullptr;     // per CTA: [first step, end step)
  int32_t* counters = nullptr;         // one per split group, zero between launches
  float* partials = nullptr;           // [chunk slots][kTcPartialFloats]
  int32_t* error = nullptr;            // nonzero after a bounded wait gave up
  int32_t n_ctas = 0;
};
// whether the tensor-core interpolation is built for this view shape
inline bool interp_tc_supported(int rowh, int ncomp) { return rowh == 32 && ncomp == 1; }
// epi: EPI_SAMPLES, EPI_GRID or EPI_PANEL; panel: the [rows][32] f16 panel the view gathers
void launch_interp_tc(const InterpTcView& v, const __half* panel, int epi, const InterpOut& o, cudaStream_t s);
// shared memory of one CTA of the tensor-core interpolation
size_t interp_tc_smem_bytes();
// warps the persistent interpolation kernel keeps resident on this device for a panel row
// width / component count (used to cut the item list into per-warp runs)
int interp_resident_warps(int rowh, int ncomp, int stages);
constexpr int kInterpWarpsPerCta = 4;

void launch_norm_partials(const float2* v, int64_t n, double* part, cudaStream_t s);

// Stage layouts (images: i0 slow, i1 fast; volumes: i0, i1, i2; grids in internal rows
// q1*G + q0 for images, (q2*G + q1)*G + q0 for volumes):
//   image:  x -rows-> z1 [q1][i0][c] -cols-> panel
//   volume: x -rows-> z1 [i0][q2][i1][c] -mid-> z2 [q2][q1][i0][c] -cols-> panel
//   inverse image:  grid -cols-> z1 [q1][i0][c] -rows-> image
//   inverse volume: grid -cols-> z2 [q2][q1][i0][c] -mid-> z1 [q2][i0][i1][c] -rows-> volume
// forward rows: x (image with smaps, coil images [C][...] without) -> z1
// mode 0: plain, sigma from norm partials -> state->sigma_x
// mode 1: CG iteration k: p = r + beta p (p = r at k == 0), rho_k from rr partials
// mode 2: CG iteration k after a reliable restart: p = r (beta = 0)
// mode 4: CG iteration k that first finishes iteration k-1 (x += alpha p, r -= alpha Ap, with
//         alpha, rho_{k-1} and rho_k from the four partial sections [lines] that inv_rows
//         wrote with r)
void launch_fwd_rows(const FftArgs& f, const float2* x, float2* z1, int mode, float2* p, float2* r,
                     const double* partials, int nparts, CgState* st, int iter, cudaStream_t s,
                     float2* xs = nullptr, const float2* ap = nullptr);
// forward columns: z1 (z2 for volumes) -> panel [G^dims][4C] in internal rows, FP16 hi | res
void launch_fwd_cols(const FftArgs& f, const float2* z1, __half* panel, cudaStream_t s);
// forward middle axis of a volume: z1 [i0][q2][i1][c] -> z2 [q2][q1][i0][c]
void launch_fwd_mid(const FftArgs& f, const float2* z1, float2* z2, cudaStream_t s);
// inverse middle axis of a volume: z2 [q2][q1][i0][c] -> z1 [q2][i0][i1][c] (crop)
void launch_inv_mid(const FftArgs& f, const float2* z2, float2* z1, cudaStream_t s);
// totals of `sections` runs of n partials (stride apart) into each run's first value, one CTA
// per run in a fixed order
void launch_reduce_partials(double* part, int n, cudaStream_t s, int sections = 1, int64_t stride = 0);
// samples [C][M] (scaled by sigma_y, density) -> sample panel [M][4C]
void launch_split_samples(const float2* y, const float* density, int64_t m, int c, __half* panel,
                          const double* partials, int nparts, CgState* st, cudaStream_t s);
// inverse columns: grid [G^dims][C] -> w1 [G][N][C] (images) or z2 (volumes)
void launch_inv_cols(const FftArgs& f, const float2* grid, float2* w1, cudaStream_t s);
// inverse rows + crop + deapod + coil combine
// mode 0: plain adjoint (factor 1/sigma_y): out = [N][N] (smaps) or [C][N][N]
// mode 1: CG RHS: r = b, x = 0, rr partials
// mode 2: CG iteration k: ap = factor*AHAp + lambda p, pap partials (with r given, also
//         Re <r, ap>, <ap, ap> and <r, r> partials at partials + lines, + 2 lines, + 3 lines)
// mode 3: reliable residual: out = x - (factor*AHAp + lambda p) with x = the right-hand
//         side b, p = the iterate and factor from the plain forward's sigma_x; rr partials
// mode 5: normal operator of a plain forward: out = factor*AHAp + lambda p, factor from
//         sigma_x, <p, out> partials; with x given, also the coil images [C][N][N] of
//         factor*AHAp before the coil combine
void launch_inv_rows(const FftArgs& f, const float2* w1, float2* out, int mode, float2* x, float2* r,
                     const float2* p, double* partials, CgState* st, int iter, float inv_scale2,
                     float lambda_scaled, cudaStream_t s);
// CG update over `lines` lines of N pixels: x += alpha p, r -= alpha ap, one rr partial per
// line; alpha = <r, r> / <p, Ap> from the first `nparts` partials of sections 3 and 0 of the
// inverse rows' four partial sections (`lines` apart)
void launch_cg_update(int N, int lines, int nparts, float2* x, float2* r, const float2* p, const float2* ap,
                      const double* pap_parts, double* rr_parts, CgState* st, int iter, cudaStream_t s);
void launch_cg_finish(int nparts, const double* rr_parts, CgState* st, int iters, cudaStream_t s);
// out[0] = Re <a, b> over n complex values in FP64 (kNormParts partials in parts, fixed order)
void launch_rdot(const float2* a, const float2* b, int64_t n, double* parts, double* out, cudaStream_t s);
// out[0] = the sum of n partials in a fixed order
void launch_sum_partials_to(const double* parts, int n, double* out, cudaStream_t s);
// Forward CG step on caller-owned vectors: alpha = rho / gamma, x_out = x + alpha p (x may be
// null), r_out = r - alpha q, rho_out = |r_out|^2 (FP64, 296 partials in parts, fixed order),
// p_out = r_out + (rho_out / rho) p.
void launch_cg_step(int64_t n, double* parts, const double* rho, const double* gamma, const float2* x, const float2* p,
                    const float2* r, const float2* q, float2* x_out, float2* r_out, float2* p_out, double* rho_out,
                    double* p_norm_parts, cudaStream_t s);
constexpr int kCgStepParts = 296;  // FP64 partials of the CG-step kernels (one per block)
// Reverse-mode CG step (kernels.cu): five FP64 inner products in one pass (parts: 5 x 296
// doubles), then rb, pb updated in place, qb written and rhob of the step to *rhob_out.
void launch_cg_adjoint_step(int64_t n, double* parts, const double* rho, const double* rho_n, const double* gamma,
                            const double* rhob, double* rhob_out, float2* rb, float2* pb, const float2* p,
                            const float2* q, const float2* rn, const float2* xb, float2* qb, double* qb_norm_parts,
                            cudaStream_t s);
// pb += mqb and, with sb given, the coil-map cotangent sb[c] += conj(qb) t[c] + tb[c] conj(p).
void launch_cg_adjoint_finish(int64_t n, int coils, float2* pb, const float2* mqb, const float2* qb, const float2* t,
                              const float2* tb, const float2* p, float2* sb, cudaStream_t s);

void launch_gather_rows_f16(const __half* src, const int32_t* map, int64_t rows, int width, __half* dst,
                            cudaStream_t s);
void launch_gather_rows_f32(const float* src, const int32_t* map, int64_t rows, int width, float* dst,
                            cudaStream_t s);

}  // namespace tsn
