/*
 * trajsparsenufft.h — C ABI of the B200 (sm_100a) fixed-trajectory NUFFT CG-SENSE library.
 *
 * The reference exposes this path as files + argv + a 7-function FFT C ABI:
 *   - pack directories written by src/export_gpu_case.py:171-321 and
 *     src/export_torchkbnufft_gpu_case.py:387-489 (packed_header_v2),
 *   - loaded by load_direction()     experiments/production/src/nufft_integrated_bench.cu:135-226,
 *   - runtime inputs (measurement.c64.bin [C][M], sensitivity_maps.c64.bin [C][N][N],
 *     scaling.f32.bin [N][N], density.f32.bin [M])
 *                                      experiments/data_prep/export_real_runtime_inputs.py:92-113,
 *   - FFT endpoints                    experiments/production/src/nufft_custom_fft_f30_api.h:6-34,
 *   - the CG driver main()             experiments/production/src/nufft_fp16x2_cg_bench.cu:279-518.
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions (kept from the reference):
 *   - complex data are interleaved float pairs (float2 / complex64);
 *   - coil-major layouts: samples [C][M], coil images / maps [C][N][N], image [N][N];
 *   - grid cell index = q0*G + q1 in pack files (nufft_custom_fft_forward_bench.cu:699-701);
 *   - the image sits at [0,N) of the G x G grid and the phase is carried by the
 *     complex coefficients;
 *   - trajectories are cycles/pixel in [-0.5, 0.5), axis 0 pairs with image axis 0.
 * Every call returns a tsn_status; nothing calls exit().  Device pointers are
 * caller-owned; the plan owns packs and workspaces.  A plan is not thread-safe,
 * separate plans may be used concurrently from separate threads/streams.
 */
#ifndef TRAJSPARSENUFFT_H_
#define TRAJSPARSENUFFT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same underlying type as cudaStream_t; NULL is the legacy default stream. */
typedef struct CUstream_st* tsn_stream_t;

typedef enum tsn_status {
  TSN_OK = 0,
  TSN_ERR_IO = 1,          /* file missing, short or unwritable     (reference: exit(1)) */
  TSN_ERR_FORMAT = 2,      /* bad magic/version/header, real/imag mismatch (exit(2))  */
  TSN_ERR_SHAPE = 3,       /* sizes inconsistent with the plan                         */
  TSN_ERR_NONFINITE = 4,   /* non-finite input or CG state (reference exit(3))        */
  TSN_ERR_CURVATURE = 5,   /* CG denominator <= 0 (positive_curvature flag = 0)        */
  TSN_ERR_TIMEOUT = 6,     /* a bounded device wait gave up                            */
  TSN_ERR_CUDA = 7,        /* CUDA runtime error                                       */
  TSN_ERR_ARG = 8,         /* invalid argument / NULL where required                   */
  TSN_ERR_UNSUPPORTED = 9, /* shape or option not built for sm_100a here               */
  TSN_ERR_NOMEM = 10
} tsn_status;

/* Planner variants of the reference (pack once, CPU). */
enum {
  TSN_PLANNER_OPTIMIZED = 0, /* optimized_split24_pack  src/export_torchkbnufft_gpu_case.py:270-299 */
  TSN_PLANNER_FAST = 1,      /* fast_split24_pack       src/export_torchkbnufft_gpu_case.py:46-99   */
  TSN_PLANNER_SEARCH = 2     /* pack_view               src/nufft_layout_oracle.py:445-497          */
};
/* Row-grouping policies, src/nufft_layout_oracle.py:243-309. */
enum { TSN_POLICY_TRAJECTORY = 0, TSN_POLICY_MORTON = 1, TSN_POLICY_OVERLAP = 2, TSN_POLICY_PACKING256 = 3 };
/* Illegal-tile handling, src/export_gpu_case.py:110-155. */
enum { TSN_ILLEGAL_SPLIT24 = 0, TSN_ILLEGAL_CSR_RESIDUAL = 1 };
/* Views. */
enum { TSN_VIEW_G = 0, TSN_VIEW_GT = 1 };
/* Interpolation kernel choice (the reference runs warp mma.sp m16n8k32 per 16-row tile,
 * nufft_spmma_bench.cu:402-663).  TSN_INTERP_MMA_SP: the same instruction family, one warp per
 * tile stream.  TSN_INTERP_TCGEN05: tcgen05.mma.sp with seven 16-row tiles stacked into one
 * M = 128 operand, B rows gathered by TMA, accumulators in tensor memory; built for the
 * real-coefficient pack (trajectory plans without TSN_FLAG_REFERENCE_LAYOUT) with 8 coils,
 * refused with TSN_ERR_UNSUPPORTED otherwise.  TSN_INTERP_AUTO picks the faster one measured
 * for the shape. */
enum { TSN_INTERP_AUTO = 0, TSN_INTERP_MMA_SP = 1, TSN_INTERP_TCGEN05 = 2 };
/* Plan flags. */
enum {
  TSN_FLAG_REFERENCE_LAYOUT = 1 << 0, /* complex real/imag packs, image at [0,N) (reference pack format);
                                         default for trajectory plans is the real-coefficient pack
                                         with the image centred on the grid (same operator, half the
                                         coefficient bytes) */
  TSN_FLAG_REFERENCE_STEPS = 1 << 1   /* also keep an FP32-class operator for the CG's reference
                                         steps (tsn_cg_options): the same packs with every
                                         coefficient split into an FP16 high part and an FP16
                                         residual (the reference's "split2" matrix mode,
                                         reference_sparse_solver.py:80-110), both against the FP16
                                         high + residual panels.  2D trajectory plans with the
                                         centred real-coefficient pack only. */
};

typedef struct tsn_plan_desc {
  int32_t im_size;      /* N  (reference: kImage = 256, nufft_integrated_bench.cu:111)   */
  int32_t grid_size;    /* G  (kGrid = 512)                                              */
  int32_t coils;        /* C  (kCoils = 8), multiple of 4, <= 16                         */
  int32_t kernel_width; /* J  (numpoints = 6)                                            */
  int32_t planner;      /* TSN_PLANNER_*                                                 */
  int32_t policy;       /* TSN_POLICY_*  (production: morton, run_fast_planner_matrix.py) */
  uint64_t seed;        /* planner seed (20260823)                                       */
  int32_t threads;      /* planner threads, 0 = all host cores                           */
  int32_t flags;        /* TSN_FLAG_*                                                    */
  int32_t interp;       /* TSN_INTERP_*                                                  */
  int32_t device;       /* CUDA device ordinal the plan lives on (made current at every call) */
  int32_t dims;         /* 2 (0 also means 2): [N][N] images; 3: [N][N][N] volumes on a G^3
                           grid (trajectory [M][3], centred layout, fast/optimized planner,
                           G^3 <= 2^24 cells, M <= 2^24 samples)                          */
  int32_t reserved[5];
} tsn_plan_desc;

typedef struct tsn_plan_info {
  int64_t samples;            /* M                                           */
  int32_t im_size, grid_size, coils, kernel_width, components;
  int64_t groups[2], tiles[2], active_rows[2], nnz[2]; /* [TSN_VIEW_G], [TSN_VIEW_GT] */
  int64_t pack_bytes[2];      /* device bytes of each view's pack              */
  int64_t workspace_bytes;    /* device workspace owned by the plan            */
  double plan_seconds;        /* host planner wall time                        */
  int32_t interp;             /* kernel actually used (TSN_INTERP_MMA_SP or _TCGEN05)   */
  int32_t dims;               /* 2 or 3                                                 */
  int32_t device_error;       /* nonzero once a tcgen05 launch of this plan gave up a bounded
                                 wait (read at call time: synchronize the plan's streams first) */
  int32_t reserved[5];
} tsn_plan_info;

typedef struct tsn_cg_status {
  int32_t completed_iterations;
  int32_t positive_curvature;  /* 1 unless a denominator was <= 0 or non-finite   */
  int32_t finite;              /* 1 unless the solution / residual went non-finite */
  int32_t timeout;             /* 1 when a bounded device wait of the solve gave up */
  double residual0, residual_final;
} tsn_cg_status;

typedef struct tsn_plan tsn_plan;

/* ---- library ------------------------------------------------------------------------ */
const char* tsn_version(void);
/* Thread-local text of the last error (never NULL). */
const char* tsn_get_last_error_string(void);
tsn_status tsn_plan_desc_default(tsn_plan_desc* desc);

/* ---- pack once (CPU) ------------------------------------------------------------------ */
/* Complex KB interpolation matrix of a trajectory as CSR (rows = samples, columns sorted,
 * exact zeros dropped).  Replaces tkbn.calc_tensor_spmatrix at
 * src/export_torchkbnufft_gpu_case.py:537-567.  Two-call pattern: pass cols == NULL to get
 * *nnz, then call again with arrays of that size.  row_ptr has m+1 entries. */
tsn_status tsn_kb_interpolation_csr(const float* traj_cycles, int64_t m, int32_t im_size,
                                    int32_t grid_size, int32_t width, int64_t* row_ptr,
                                    int64_t* cols, double* re, double* im, int64_t* nnz);
/* [N][N] deapodization table (the scaling.f32.bin role, export_real_runtime_inputs.py:97-101). */
tsn_status tsn_kb_deapodization(int32_t im_size, int32_t grid_size, int32_t width, double* out);

/* Volumes: real KB weights of a [M][3] trajectory for the centred-image layout, CSR over
 * samples, cells (q0 G + q1) G + q2, weight (phi0 phi1) phi2, columns sorted, zeros dropped
 * (the 3D extension of tsn_kb_interpolation_csr; the reference is 2D only).  Same two-call
 * pattern on *nnz. */
tsn_status tsn_kb_weights_csr3(const float* traj_cycles, int64_t m, int32_t im_size, int32_t grid_size,
                               int32_t width, int64_t* row_ptr, int64_t* cols, double* w, int64_t* nnz);
/* [N][N][N] deapodization of the volume layout. */
tsn_status tsn_kb_deapodization3(int32_t im_size, int32_t grid_size, int32_t width, double* out);

/* Pack one view of a complex sparse matrix given as CSR over samples (G) and write the
 * production directories out_dir/real and out_dir/imag (packed_header_v2 + six arrays +
 * manifest.json).  The structure (ones) is packed once and both components are placed on
 * it — src/export_torchkbnufft_gpu_case.py:513-646 with --production-only. */
tsn_status tsn_pack_csr_to_dirs(const int64_t* row_ptr, const int64_t* cols, const double* re,
                                const double* im, int64_t rows, int32_t grid_size,
                                const float* traj_cycles, int32_t view, int32_t planner,
                                int32_t policy, uint64_t seed, int32_t threads,
                                const char* out_dir);

/* One real view packed like pack_view / fast / optimized, returned as raw tiles for parity
 * checks against src/nufft_layout_oracle.py:445-497.  coords [rows][2] drive morton order.
 * Two-call pattern on *tile_count (pass row_ids == NULL first).  row_ids [T][16],
 * col_ids [T][k_tile], values [T][16][k_tile], legal [T]. */
tsn_status tsn_pack_view_tiles(const int64_t* row_ptr, const int64_t* cols, const double* vals,
                               const int64_t* logical_row_ids, const double* coords,
                               int64_t rows, int64_t output_size, int64_t n_cols, int32_t planner,
                               int32_t policy, int32_t k_tile, uint64_t seed, int32_t threads,
                               int64_t* tile_count, int32_t* row_ids, int32_t* col_ids,
                               double* values, uint8_t* legal);

/* export_case (src/export_gpu_case.py:171-321) arrays for one real view, either illegal
 * mode: writes header.bin, group_offsets.bin, group_row_ids.bin, tile_col_ids.bin,
 * tile_a_comp.bin, tile_pair_meta.bin, residual_{row_ptr,cols,vals}.bin into out_dir. */
tsn_status tsn_export_view_dir(const int64_t* row_ptr, const int64_t* cols, const double* vals,
                               const int64_t* logical_row_ids, const double* coords, int64_t rows,
                               int64_t output_size, int64_t n_cols, int32_t planner, int32_t policy,
                               uint64_t seed, int32_t illegal_mode, int32_t threads,
                               const char* out_dir);

/* ---- plans (device residency) --------------------------------------------------------- */
/* Load the four reference pack directories (load_direction x2, nufft_integrated_bench.cu:
 * 135-226, same header/structure checks) plus an [N][N] deapodization table (host, may be
 * NULL to use the KB table of desc).  Replaces the FWD_REAL FWD_IMAG ADJ_REAL ADJ_IMAG argv
 * of nufft_fp16x2_cg_bench.cu:279-297. */
tsn_status tsn_plan_create_from_pack(const char* fwd_real_dir, const char* fwd_imag_dir,
                                     const char* adj_real_dir, const char* adj_imag_dir,
                                     const float* scaling, const tsn_plan_desc* desc,
                                     tsn_plan** plan);
/* Build both packs from a trajectory with the C++ planner (pack once) and upload them.
 * traj_cycles is [M][desc->dims] in cycles/pixel, [-0.5, 0.5].  Volumes (dims 3): x, smaps
 * and coil images are [N][N][N] / [C][N][N][N], the grid has G^3 cells, and the operators,
 * CG-SENSE, batches and stage profiling take the same calls as images. */
tsn_status tsn_plan_create_from_trajectory(const float* traj_cycles, int64_t m,
                                           const tsn_plan_desc* desc, tsn_plan** plan);
tsn_status tsn_plan_destroy(tsn_plan* plan);
tsn_status tsn_plan_get_info(const tsn_plan* plan, tsn_plan_info* info);

/* ---- operators (device pointers, asynchronous on stream) ------------------------------ */
/* y[C][M] = A x.  With smaps != NULL, x is the image [N][N] and the coil images are x*S_c
 * (jkf_launch_custom_fft_f30_forward_sense_split2 + forward fused interpolation,
 * nufft_integrated_bench.cu:527-585,604-627); with smaps == NULL, x is coil images [C][N][N]
 * (jkf_launch_custom_fft_f30_forward_split2).  Unnormalized NUFFT units. */
tsn_status tsn_forward(tsn_plan* plan, const void* x, const void* smaps, void* y,
                       tsn_stream_t stream);
/* x = A^H y: [N][N] coil-combined when smaps != NULL (launch_adjoint_image,
 * nufft_fp16x2_cg_bench.cu:203-222, without the Tikhonov term), else coil images [C][N][N]. */
tsn_status tsn_adjoint(tsn_plan* plan, const void* y, const void* smaps, void* x,
                       tsn_stream_t stream);
/* Pieces of the CG for callers that run their own (differentiable) recursion: the reference
 * solver's normal operator `adjoint(forward(p)) + lam p` with its W weighting
 * (reference_sparse_solver.py:200-332 cg_sense, forward/adjoint of :590-630) and its inner
 * products.  tsn_normal: q[N][N] = sum_c conj(S_c) F^H W F(S_c p) + lambda p (device arrays;
 * density W [M] may be NULL), with, when coil_images != NULL, the coil images
 * F^H W F(S_c p) [C][N][N] before the combine, and, when pq != NULL, Re <p, q> summed in FP64
 * in a fixed order into the device double *pq.  Same units as tsn_forward / tsn_adjoint.
 * p_norm_parts (optional): n_p_norm_parts device doubles whose sum is |p|^2, such as the
 * TSN_CG_STEP_PARTS partials tsn_cg_step writes for its p' (they set the FP16 panel scale;
 * NULL: computed here by one more pass over p).
 * tsn_rdot: *out (device) = Re <a, b> = sum a.re b.re + a.im b.im over n complex values, FP64,
 * fixed order.  Both use the plan's workspaces: calls on one plan are ordered by their stream. */
tsn_status tsn_normal(tsn_plan* plan, const void* p, const void* smaps, const float* density, float lambda,
                      void* q, void* coil_images, double* pq, const double* p_norm_parts,
                      int32_t n_p_norm_parts, tsn_stream_t stream);
/* Number of FP64 partials tsn_cg_step / tsn_cg_adjoint_step write to their optional
 * p_norm_parts / qb_norm_parts outputs. */
#define TSN_CG_STEP_PARTS 296
tsn_status tsn_rdot(tsn_plan* plan, const void* a, const void* b, int64_t n, double* out,
                    tsn_stream_t stream);
/* One CG step on caller-owned vectors (the update of reference_sparse_solver.py:288-332
 * cg_sense for callers that keep their own states): alpha = *rho / *gamma; x_out = x + alpha p
 * (x and x_out may both be NULL); r_out = r - alpha q; *rho_out = |r_out|^2 in FP64 (fixed
 * order); p_out = r_out + (*rho_out / *rho) p.  Scalars are device doubles, vectors n complex64
 * on the device; outputs must not alias inputs.  p_norm_parts (optional, TSN_CG_STEP_PARTS
 * device doubles) receives partial sums of |p_out|^2 for the next tsn_normal. */
tsn_status tsn_cg_step(tsn_plan* plan, int64_t n, const double* rho, const double* gamma, const void* x,
                       const void* p, const void* r, const void* q, void* x_out, void* r_out,
                       void* p_out, double* rho_out, double* p_norm_parts, tsn_stream_t stream);
/* One reverse-mode CG step (the adjoint of alpha = rho / gamma, x' = x + alpha p, r' = r -
 * alpha q, rho' = |r'|^2, p' = r' + (rho'/rho) p with q = M p, gamma = Re <p, q>) for
 * differentiable unrolled solves; no counterpart in the reference, which has no gradients.
 * Device scalars (FP64): rho, rho_next = rho', gamma, rhob (cotangent of rho'); rhob_out
 * receives the cotangent of rho.  Vectors of n complex64: rb, pb (cotangents of r', p') are
 * updated in place to r-bar of this step and to p-bar minus M qb; qb receives the cotangent
 * of q; p, q, r_next = r', xb (cotangent of x') are read.  Five FP64 inner products come
 * from one pass before any vector changes.  tsn_cg_adjoint_finish then adds M qb (mqb) to
 * pb and, with sb != NULL, adds conj(qb) t_c + tb_c conj(p) to the coil-map cotangent sb
 * [coils][n] (t = coil images of M p, tb = those of M qb, as tsn_normal returns them).
 * qb_norm_parts (optional, TSN_CG_STEP_PARTS device doubles) receives partial sums of |qb|^2
 * for the tsn_normal of qb. */
tsn_status tsn_cg_adjoint_step(tsn_plan* plan, int64_t n, const double* rho, const double* rho_next,
                               const double* gamma, const double* rhob, double* rhob_out, void* rb,
                               void* pb, const void* p, const void* q, const void* r_next,
                               const void* xb, void* qb, double* qb_norm_parts,
                               tsn_stream_t stream);
tsn_status tsn_cg_adjoint_finish(tsn_plan* plan, int64_t n, int32_t coils, void* pb, const void* mqb,
                                 const void* qb, const void* coil_images, const void* coil_images_bar,
                                 const void* p, void* sb, tsn_stream_t stream);
/* The FP32-class operators of a plan built with TSN_FLAG_REFERENCE_STEPS (the reference's
 * forward_reference / adjoint_reference, reference_sparse_solver.py:590-630, which its CG uses
 * for scheduled reference steps): same arguments and units as tsn_forward / tsn_adjoint, every
 * KB weight applied as its FP16 high part plus its FP16 residual.  TSN_ERR_ARG on other plans. */
tsn_status tsn_forward_reference(tsn_plan* plan, const void* x, const void* smaps, void* y,
                                 tsn_stream_t stream);
tsn_status tsn_adjoint_reference(tsn_plan* plan, const void* y, const void* smaps, void* x,
                                 tsn_stream_t stream);
/* CG-SENSE on (A^H W A + lambda) x = A^H W y from x0 = 0, operator divided by operator_scale
 * (launch_cg, nufft_fp16x2_cg_bench.cu:241-268; reference_sparse_solver.py cg_sense).
 * density (W, [M]) may be NULL.  The whole solve runs as one CUDA graph (captured on first
 * use per argument set).  residual_history (host, iters+1 entries) and status may be NULL;
 * when either is given the call synchronizes the stream to fill them. */
tsn_status tsn_cg_sense(tsn_plan* plan, const void* y, const void* smaps, const float* density,
                        float lambda, float operator_scale, int32_t iters, void* x,
                        double* residual_history, tsn_cg_status* status, tsn_stream_t stream);
/* Reliable-update CG (reference_sparse_solver.py:200-332 cg_sense, reliable_update_period and
 * reliable_update_direction): after every `reliable_update_period`-th iteration except the
 * last, the recursive residual is replaced by r = b - (A^H W A + lambda) x through the same
 * operator; p then restarts as r (direction 0, "restart") or continues as r + beta p
 * (direction 1, "beta").  The residual history records the replaced residual.  A zero period
 * is tsn_cg_sense. */
typedef struct tsn_cg_options {
  int32_t reliable_update_period;
  int32_t reliable_update_direction;
  /* Scheduled reference steps (reference_sparse_solver.py:200-332, scheduled_reference_period and
   * explicit_reference_steps): completed iteration s (1-based) computes A^H W A p through the
   * FP32-class operator of a plan built with TSN_FLAG_REFERENCE_STEPS when s is a multiple of
   * scheduled_reference_period (0: none) or bit s-1 of reference_steps is set (s <= 64).  When
   * any reference step or reliable update is asked for on such a plan, the right-hand side and
   * the reliable residuals use that operator too, as in the reference. */
  int32_t scheduled_reference_period;
  int32_t reserved0;
  uint64_t reference_steps;
  int32_t reserved[2];
} tsn_cg_options;
tsn_status tsn_cg_sense_ex(tsn_plan* plan, const void* y, const void* smaps, const float* density,
                           float lambda, float operator_scale, int32_t iters,
                           const tsn_cg_options* options, void* x, double* residual_history,
                           tsn_cg_status* status, tsn_stream_t stream);

/* ---- batches of independent reconstructions ------------------------------------------- */
/* The reference runs one case per CG process (nufft_fp16x2_cg_bench.cu:279-297 argv).  A
 * batch holds `count` plans of one device (any image size, coil count and trajectory) and
 * solves them together: one CUDA graph forks the cases over `streams` streams (0: up to 8)
 * and every persistent launch of a case uses a 1/streams slice of the GPU, so small cases run
 * side by side instead of one after another.  Cases go to streams longest-first by estimated
 * cost.  The plans stay owned by the caller and must outlive the batch; a plan may belong to
 * one batch and must not run elsewhere while a batch solve is in flight. */
typedef struct tsn_batch tsn_batch;
tsn_status tsn_batch_create(tsn_plan* const* plans, int32_t count, int32_t streams, tsn_batch** out);
tsn_status tsn_batch_destroy(tsn_batch* batch);
/* CG-SENSE of every case (arrays of `count` device pointers; density may be NULL or hold NULL
 * entries) with one lambda, operator scale and iteration count.  statuses (host, `count`
 * entries) may be NULL; when given, the call synchronizes and returns the first failing
 * case's status (NONFINITE / CURVATURE) after filling every entry. */
tsn_status tsn_batch_cg_sense(tsn_batch* batch, const void* const* y, const void* const* smaps,
                              const float* const* density, float lambda, float operator_scale,
                              int32_t iters, void* const* x, tsn_cg_status* statuses,
                              tsn_stream_t stream);

/* ---- FFT endpoints (the role of nufft_custom_fft_f30_api.h:6-34) ---------------------- */
/* Forward endpoint: panel[G*G][4C] f16 = s * FFT_G(pad(x * S_c * scaling)), rows q1*G + q0
 * (q1-major), each row = FP16 high parts then FP16 residuals, (re, im) interleaved per coil;
 * s is a power of two chosen from the input norm and written to *panel_scale (host; the
 * call synchronizes when panel_scale != NULL).  Replaces
 * jkf_launch_custom_fft_f30_forward_sense_split2 (x-stage + y-stage). */
tsn_status tsn_fft_forward_panel(tsn_plan* plan, const void* x, const void* smaps, void* panel_f16,
                                 float* panel_scale, tsn_stream_t stream);
/* Adjoint endpoint: x = sum_c conj(S_c) * scaling * crop(IFFT_G(grid_c)) (unnormalized inverse)
 * from grid[G*G][C] c64 with rows q1*G + q0; coil images [C][N][N] when smaps == NULL.
 * Replaces jkf_launch_custom_ifft_f31_adjoint + sense_combine_scaled. */
tsn_status tsn_fft_adjoint_image(tsn_plan* plan, const void* grid_c64, const void* smaps, void* x,
                                 tsn_stream_t stream);

/* No counterpart in the reference.  The adjoint FFT endpoint for callers that cannot call
 * cudaMalloc (hosts whose device allocator is frozen after start-up, services that reserve
 * all device memory up front, plug-ins inside an application that owns the device memory):
 * no plan, every input and output from the caller, the one intermediate in a fixed device
 * array of grid_size * im_size * coils <= 1 Mi complex values (8 MiB, enough for
 * 512 x 256 x 8); larger shapes return TSN_ERR_SHAPE.  Computes the same as
 * tsn_fft_adjoint_image (grid[G*G][C] c64 with rows q1*G + q0; centered != 0 when the image
 * is centred on the grid, as in trajectory plans without TSN_FLAG_REFERENCE_LAYOUT).  The
 * first call on a device sets up the device that is current at that call: it looks up the
 * arrays' device addresses and fills the twiddle tables of every supported grid size, so
 * make it before any stream capture.  Later calls write only the scratch array and the
 * output; every call in the process shares the scratch array, so calls that overlap on the
 * GPU race and must be ordered by the caller.  Allocates nothing. */
tsn_status tsn_fft_adjoint_image_static(int32_t im_size, int32_t grid_size, int32_t coils,
                                        int32_t centered, const void* grid_c64, const void* smaps,
                                        const float* scaling, void* x, tsn_stream_t stream);

/* ---- stage timing (autotuner and roofline reporting) ---------------------------------- */
enum {
  TSN_STAGE_FWD_ROWS = 0,   /* forward FFT x-stage (SENSE, deapodization, padding; in CG    *
                             * iterations after the first, the previous x, r update)       */
  TSN_STAGE_FWD_COLS = 1,   /* forward FFT y-stage -> FP16 hi|res grid panel                 */
  TSN_STAGE_INTERP_FWD = 2, /* sparse G interpolation -> FP16 hi|res sample panel            */
  TSN_STAGE_INTERP_ADJ = 3, /* sparse G^H gather -> grid                                     */
  TSN_STAGE_INV_COLS = 4,   /* inverse FFT first stage                                       */
  TSN_STAGE_INV_ROWS = 5,   /* inverse FFT second stage + crop + deapod + coil combine      */
  TSN_STAGE_CG_UPDATE = 6,  /* x, r update + FP64 partial dots (after the last iteration)    */
  TSN_STAGE_FWD_MID = 7,    /* volumes: forward FFT over the middle axis (0 ms for images)   */
  TSN_STAGE_INV_MID = 8,    /* volumes: inverse FFT over the middle axis (0 ms for images)   */
  TSN_STAGE_COUNT = 9
};
/* Runs one CG-SENSE solve of `iters` iterations to populate the workspaces, then times each
 * stage of a CG iteration `reps` times in isolation with CUDA events on `stream` and writes
 * the mean milliseconds per launch to stage_ms[TSN_STAGE_COUNT] (synchronizes). The row
 * stages are timed in the form the inner iterations run (forward rows with the previous
 * update, inverse rows with its partials); the plan's solve state is left overwritten. */
tsn_status tsn_profile_stages(tsn_plan* plan, const void* y, const void* smaps, int32_t reps,
                              double* stage_ms, tsn_stream_t stream);

/* ---- raw interpolation (parity with the reference GPU gate) --------------------------- */
/* out[rows][16] f32 = component(view) x dense[n_cols][16] f16 for one real/imag component of
 * a plan built from packs: the nufft_gt_spmma_*_f16_f32 contract checked against
 * reference.bin (nufft_spmma_bench.cu:1090-1109).  component 0 = real, 1 = imag. */
tsn_status tsn_interp_component(tsn_plan* plan, int32_t view, int32_t component,
                                const void* dense_f16, float* out, tsn_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* TRAJSPARSENUFFT_H_ */
