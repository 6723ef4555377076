/* ftdx.h -- C ABI of the B200 (sm_100a) X-engine correlator.
 *
 * One call computes, for every channel (batch entry) b,
 *     C_b = alpha * A_b * A_b^H + beta * C_b
 * where A_b is an N x K complex voltage matrix (N inputs = antennas x pols,
 * K time samples) and C_b is stored as the packed lower triangle, row-major:
 * element (i, j <= i) at i(i+1)/2 + j, interleaved (re, im), with Im(C_ii)
 * forced to 0 before beta is applied (as the reference's direct HERK kernel
 * does; its CUTLASS baseline path instead zeroes Im(C_ii) after beta, which
 * differs only when the old C has a non-zero imaginary diagonal).
 *
 * All data pointers are DEVICE pointers owned by the caller.  Work is queued
 * on the caller's stream (`stream` is a cudaStream_t; NULL = legacy default
 * stream).  Calls return immediately; a device-side wait that timed out is
 * reported by ftdx_device_status().  No function throws, aborts or exits.
 * A handle is not thread-safe: use one handle per host thread.
 *
 * Reference interfaces replaced (paths within cpviolator/ftd):
 *   cutlass_interface/cutlass_gemm_api.h:157-789   class CutlassComplexGemm
 *   lib/cutlass_interface.cu:150-307               ggp::initCutlassApi,
 *                                                  ggp::herkBatchedCutlassQC{,_FP16},
 *                                                  ggp::herkBatchedCutlassFP16
 */
#ifndef FTDX_H_
#define FTDX_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FTDX_API __attribute__((visibility("default")))
#else
#define FTDX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FTDX_VERSION_MAJOR 0
#define FTDX_VERSION_MINOR 1

typedef enum ftdx_status {
  FTDX_OK = 0,
  FTDX_ERR_INVALID_ARG = 1,   /* bad size, null or misaligned pointer, bad enum */
  FTDX_ERR_UNSUPPORTED = 2,   /* valid request this build does not implement */
  FTDX_ERR_CUDA = 3,          /* a CUDA runtime/driver call failed */
  FTDX_ERR_NO_DEVICE = 4,     /* no CUDA device, or not an sm_100 device */
  FTDX_ERR_ALLOC = 5,         /* workspace allocation failed */
  FTDX_ERR_CAPACITY = 6,      /* workspace too small while a graph is being captured */
  FTDX_ERR_TIMEOUT = 7,       /* a bounded device-side wait gave up */
  FTDX_ERR_CACHE = 8          /* tune cache file unreadable / malformed */
} ftdx_status;

/* Values equal the reference's enum class ordinals
 * (cutlass_interface/cutlass_gemm_api.h:37-59). */
typedef enum ftdx_input {
  FTDX_IN_FP16 = 0,
  FTDX_IN_INT4 = 1,
  FTDX_IN_FP32 = 2   /* interleaved complex64 [batch][N][K][2] float (this library only) */
} ftdx_input;
typedef enum ftdx_compute {
  FTDX_COMPUTE_FP8 = 0,        /* INT4: exact; FP16: unscaled E4M3 (as the reference);
                                  FP32: E4M3 with a per-channel scale */
  FTDX_COMPUTE_FP6 = 1,        /* INT4 input only: E3M2 operands (every QC value exact), so
                                  the result equals FP8's; other inputs: UNSUPPORTED */
  FTDX_COMPUTE_FP4 = 2,        /* NVFP4: E2M1 with one E4M3 scale per 16 values (FP32 input) */
  FTDX_COMPUTE_FP8_SPLIT = 3,  /* FP32 input: hi + lo E4M3, hi.hi^H + hi.lo^H + lo.hi^H */
  FTDX_COMPUTE_FP4_SPLIT = 4   /* FP32 input: hi + lo NVFP4 (lo = NVFP4 of the residual, own
                                  block scales), hi.hi^H + hi.lo^H + lo.hi^H; FP32 output */
} ftdx_compute;
typedef enum ftdx_output { FTDX_OUT_FP16 = 0, FTDX_OUT_FP32 = 1 } ftdx_output;
typedef enum ftdx_format { FTDX_FORMAT_PACKED_TRIANGLE = 0 } ftdx_format;

typedef struct ftdx_context* ftdx_handle;

/* Handle configuration; zero-initialise and set what you need. */
typedef struct ftdx_config {
  int device;               /* CUDA device ordinal; <0 = current device */
  int verbosity;            /* 0 silent, 1 summary, 2+ detailed (stderr) */
  const char* tune_cache;   /* autotune cache file; NULL = $FTDX_TUNE_CACHE or none */
  int reserved[8];
} ftdx_config;

/* Library version as (major << 16) | minor. */
FTDX_API int ftdx_version(void);

/* Human-readable text for a status code (static storage). */
FTDX_API const char* ftdx_status_string(ftdx_status s);

/* Create / destroy a handle.  Replaces CutlassComplexGemm::CutlassComplexGemm
 * and ~CutlassComplexGemm (cutlass_gemm_api.h:159-164). cfg may be NULL. */
FTDX_API ftdx_status ftdx_create(ftdx_handle* h, const ftdx_config* cfg);
FTDX_API ftdx_status ftdx_destroy(ftdx_handle h);

/* Text of the last error raised on this handle (static until the next call).
 * With h = NULL: the text of the last failure of a handle-less entry point
 * (ftdx_herk_static) on the calling thread, or "null handle" if none. */
FTDX_API const char* ftdx_last_error(ftdx_handle h);

/* Batched HERK.  Replaces CutlassComplexGemm::herk (cutlass_gemm_api.h:750-760,
 * cutlass_gemm_api.cu:1707-1878).
 *   A: INT4 -> [batch][N][K] QC bytes (high nibble Re, low nibble Im,
 *             sign-magnitude); FP16 -> [batch][N][K][2] __half.
 *   C: FP32 -> [batch][N(N+1)/2][2] float; FP16 -> [batch][N(N+1)/2][2] __half.
 *   compute must be FTDX_COMPUTE_FP8 (FP6/FP4 -> FTDX_ERR_UNSUPPORTED).
 *   Any K >= 1 is accepted (tails are zero-padded internally).
 *   tune != 0 consults/updates the autotune cache for this shape. */
FTDX_API ftdx_status ftdx_herk(ftdx_handle h, const void* A, void* C, int N, int K, int batch,
                      ftdx_input input, ftdx_compute compute, ftdx_output output,
                      ftdx_format format, float alpha, float beta, void* stream, int tune);

/* ---- uneven, flagged channels in one launch --------------------------------
 * No single counterpart in the reference, which batches only uniform
 * (N, K, batch) problems and loops over channel groups in its callers
 * (lib/visibility_pipeline.cu:268-277).  One call correlates n_chans
 * channels, each with its own QC rows, integration length and output:
 * channel c's output (packed lower triangle over its n_inputs active inputs,
 * in the order of `active`) is
 *   C_c = alpha * A_c A_c^H + beta * C_c,  A_c = rows active[0..n_inputs) of
 *   the [rows][lda] QC block at A (rows 0..n_inputs-1 when active == NULL).
 * All channels run in one persistent correlator launch (longest K first),
 * on the single-CTA or the CTA-pair kernel (ftdx_set_strategy / tune).
 * A plan is built on the first call with a given descriptor set (pointers
 * and sizes; the contents of `active` are read on every call) and cached. */
typedef struct ftdx_channel_desc {
  const void* A;           /* QC int4 bytes of this channel (device) */
  void* C;                 /* its packed triangle, n_inputs*(n_inputs+1)/2 complex (device) */
  int n_inputs;            /* inputs correlated (active inputs after flagging) */
  int K;                   /* time samples, >= 1 */
  int64_t lda;             /* row pitch of A in bytes (0: K) */
  const int32_t* active;   /* device array of n_inputs row indices, or NULL */
} ftdx_channel_desc;

FTDX_API ftdx_status ftdx_herk_batched_v(ftdx_handle h, const ftdx_channel_desc* chans,
                                         int n_chans, ftdx_output output, float alpha,
                                         float beta, void* stream, int tune);

/* Correlation straight from raw packet-ordered QC voltages: the corner turn
 * into per-(channel, pol, time_inner) antenna rows is fused into the operand
 * promotion pass, so the raw buffer is read once and no batch-first copy is
 * made.  Two source layouts of the reference are accepted:
 *   FTDX_LAYOUT_TIME_ANT_CHAN_POL: byte [t][ant][chan][pol], t = k*n_time_inner
 *     + ti (the FTD packet order of tests/visibility_pipeline_test.cpp:55-96,
 *     cpu_herk_ftd);
 *   FTDX_LAYOUT_CHAN_POL_ANT_TIME: byte [chan][pol][ant][t], t = ti*K + k (the
 *     order qc_pol_gather_transpose_kernel reads, lib/bench_pipeline.cu:306-331).
 * K = n_time / n_time_inner (n_time must be a multiple of n_time_inner).
 * Output: one packed lower triangle (N = n_ant) per batch b = (chan*n_pol +
 * pol)*n_time_inner + ti, the batch order of cpu_herk_ftd.  With pol_sum = 1
 * the polarisations are summed, R = sum_pol V_pol V_pol^H, one triangle per
 * b = chan*n_time_inner + ti (what the reference's two HERKs with beta = 1 on
 * pol-separated buffers produce, lib/bench_pipeline.cu:1366-1378); it runs as
 * one HERK over n_pol*K samples.  QC int4 input, FP8 compute. */
typedef enum {
  FTDX_LAYOUT_TIME_ANT_CHAN_POL = 0,
  FTDX_LAYOUT_CHAN_POL_ANT_TIME = 1
} ftdx_layout;

typedef struct ftdx_ftd_desc {
  int n_ant, n_chan, n_pol, n_time, n_time_inner;
  ftdx_layout layout;
  int pol_sum;
  int reserved[4];
} ftdx_ftd_desc;

FTDX_API ftdx_status ftdx_herk_ftd(ftdx_handle h, const void* raw, void* C,
                                   const ftdx_ftd_desc* desc, ftdx_output output, float alpha,
                                   float beta, void* stream);

/* Host-to-host correlation pipeline: replaces the CUTLASS branch of
 * ggp::VisibilityPipeline::correlate and ::correlate_pipelined
 * (lib/visibility_pipeline.cu:253-308, 483-549).  For every payload: H2D of
 * the raw QC bytes, correlation, D2H of the packed triangles (split over two
 * streams, i.e. two copy engines) with two device buffer sets, so that
 * payload p's D2H overlaps payload p+1's H2D and correlation.  Host buffers may be pinned (DMA
 * directly) or pageable (staged through pinned buffers, copied by
 * host_threads threads).  A payload is batch-first QC [batch][N][K] bytes, or,
 * when ftd is set, raw packet-ordered bytes described by *ftd (see
 * ftdx_herk_ftd).  ftdx_pipeline_correlate returns when every output is in
 * host memory.  The pipeline uses the handle's correlator (its workspace,
 * tuning cache and strategy); one pipeline per handle at a time. */
typedef struct ftdx_pipeline* ftdx_pipeline_t;

typedef struct ftdx_pipeline_config {
  int N, K, batch;          /* batch-first payload geometry (ignored when ftd is set) */
  ftdx_output output;
  const ftdx_ftd_desc* ftd; /* raw packet-ordered payloads instead (copied at create) */
  int host_threads;         /* threads for pageable staging copies (0: up to 8) */
  int reserved[7];
} ftdx_pipeline_config;

FTDX_API ftdx_status ftdx_pipeline_create(ftdx_handle h, const ftdx_pipeline_config* cfg,
                                          ftdx_pipeline_t* out);
FTDX_API ftdx_status ftdx_pipeline_correlate(ftdx_pipeline_t p, void* const* vis_outputs,
                                             const void* const* raw_inputs, int n_payloads);
FTDX_API ftdx_status ftdx_pipeline_destroy(ftdx_pipeline_t p);
/* Bytes of one payload's input and output. */
FTDX_API ftdx_status ftdx_pipeline_sizes(ftdx_pipeline_t p, size_t* in_bytes, size_t* out_bytes);

/* ---- imaging from the packed triangles -----------------------------------
 * Replaces imaging_pipeline::ImagingPipeline::grid_and_image
 * (include/imaging_pipeline.h, lib/imaging_pipeline.cu) and stages 2-5 of
 * VisibilityBeamformer::compute (lib/visibility_bf.cpp:305-380) for FP32
 * visibilities and an FP32 FFT.  Per channel f: every baseline k of the packed
 * lower triangle (n_bl = n_ant(n_ant+1)/2, row i, column j <= i) is summed over
 * the n_pol polarisation triangles (fused pol reduction), pillbox-gridded at
 *   (iu, iv) = round((u_k, v_k) / lambda_f / cell + Ng/2)
 * and, when i != j, its conjugate at round((-u, -v) / lambda_f / cell + Ng/2)
 * (cells outside [0, Ng) dropped), each contribution multiplied by the taper
 * weight of its cell (the taper fused into the scatter); then an unnormalised
 * inverse 2-D FFT (cuFFT C2C), and beam b of channel f = |image(row_b, col_b)|^2
 * * norm, norm = 1/Ng^2 (0 for pixels outside the image).
 * vis: device FP32 [n_chan][n_pol][n_bl][2]; beams: device FP32 [n_chan][n_beam].
 * output_stage: 0 = beams; 1 = the tapered UV grid and 2 = the image, both
 * [n_chan][Ng][Ng] complex64 written to grid_out (for checking; beams then
 * untouched).  The grid workspace holds chan_tile channels (at most 64; 0: as many as
 * fit in 64 MiB, so that the atomics stay in L2). */
typedef struct ftdx_imaging_config {
  int n_ant, n_chan, n_pol, n_grid, n_beam;
  int chan_tile;
  float cell_size_rad;
  const float* baseline_uv_m;  /* device [n_bl][2] (u, v) in metres */
  const double* freq_hz;       /* device [n_chan] */
  const float* taper;          /* device [n_grid * n_grid], or NULL */
  const int* beam_pixels;      /* device [n_beam][2] (row, col), or NULL if n_beam == 0 */
  int output_stage;
  int reserved[7];
} ftdx_imaging_config;

FTDX_API ftdx_status ftdx_image_beams(ftdx_handle h, const ftdx_imaging_config* cfg,
                                      const void* vis, float* beams, void* grid_out,
                                      void* stream);

/* Failure-path self-test of the bounded device waits (no counterpart in the
 * reference): one kernel waits, for timeout_ms (1..2000) each, on an mbarrier
 * that nothing arrives on and on a global flag that nothing sets (the waits
 * inside the correlators and between the blocks of the FP8 promotion), gives
 * up on both and records the timeout in the status word; ftdx_device_status
 * then returns FTDX_ERR_TIMEOUT and the handle stays usable.  Nothing traps
 * or faults. */
FTDX_API ftdx_status ftdx_wait_selftest(ftdx_handle h, int timeout_ms, void* stream);

/* The XEngine's correlation (ggp::XEngine::compute, lib/xengine.cpp:108-178:
 * promoteData, the strided-batch GEMM C = M^H M, triangulateFromHerm), with the
 * conventions its test checks (tests/xengine_test.cpp:213-321): each of the
 * batch payload blocks is M [K][n_ant] of (4,4)b two's-complement bytes (low
 * nibble Re, high nibble Im, each in [-8, 7]; promote_data.cuh:66-67), and
 * C(r, c) = sum_t conj(M(t, r)) M(t, c) is written per block as
 *   mat_format 1 (QUDA_XENGINE_MAT_TRI): the packed upper triangle, row-major
 *     (element (r, c >= r) at r*n - r(r-1)/2 + c - r);
 *   mat_format 0 (QUDA_XENGINE_MAT_HERM): the full n_ant x n_ant matrix.
 * Exact (integer sums) like the rest; FP32 or FP16 output. */
FTDX_API ftdx_status ftdx_xengine(ftdx_handle h, const void* payload, void* out, int n_ant, int K,
                                  int batch, int mat_format, ftdx_output output, void* stream);

/* The HERK branch of quda::stridedBatchGEMMCutlass (lib/cutlass_interface.cu:316-381),
 * the XEngine's BLAS entry: when A == B, trans_a is the conjugate transpose
 * (QUDA_BLAS_OP_C = 2), trans_b none (QUDA_BLAS_OP_N = 0), m == n and data_type
 * is single complex (QUDA_BLAS_DATATYPE_C = 2), C = A A^H is computed for the
 * [batch][n][k] interleaved complex64 A into the packed lower triangle
 * (complex64) at C, and the reference's flop count 8*m*n*k*batch is returned
 * after the stream is synchronised.  Any other pattern returns -1 with the last
 * error set (the reference reports it through errorQuda).
 * Arithmetic (ftdx_set_strided_mode): by default the reference's own
 * (FTDX_STRIDED_REFERENCE_FP16, lib/cutlass_interface.cu:333-367): each FP32
 * component narrowed to FP16 (round to nearest), FP16 -> E4M3 unscaled
 * (round to nearest, saturating at 448), FP32 accumulation, every result
 * rounded to FP16 and widened to FP32 -- so results agree with the reference
 * and share its range limits (FP16 output overflows past 65504).  Uses a
 * library staging buffer of 4*(batch*n*k + batch*n(n+1)/2) bytes. */
FTDX_API long long ftdx_strided_batch_gemm(ftdx_handle h, const void* A, const void* B, void* C,
                                           int m, int n, int k, int trans_a, int trans_b,
                                           int batch, int data_type, void* stream);
/* Arithmetic of ftdx_strided_batch_gemm on this handle (no counterpart in the
 * reference, which has only the first): FTDX_STRIDED_SCALED_FP8 runs the
 * FP32-input FP8 mode with a per-channel scale (448 / max |component|) and
 * FP32 output, for inputs outside FP16 / E4M3 range. */
enum { FTDX_STRIDED_REFERENCE_FP16 = 0, FTDX_STRIDED_SCALED_FP8 = 1 };
FTDX_API ftdx_status ftdx_set_strided_mode(ftdx_handle h, int mode);

/* Kahan-compensated accumulation across integration dumps (no counterpart
 * in the reference): sum += A A^H with the FP32 rounding error of every
 * addition carried in `comp` (same packed layout and size as `sum`, complex64,
 * zero it before the first dump).  After n dumps, sum + comp holds the total
 * to about FP32 precision independently of n.  Both buffers are read and
 * written by every call; FP32 output only. */
FTDX_API ftdx_status ftdx_herk_kahan(ftdx_handle h, const void* A, void* sum, void* comp, int N,
                                     int K, int batch, ftdx_input input, ftdx_compute compute,
                                     void* stream);

/* Pre-size the workspace for problems up to (N, K, batch) so that later
 * ftdx_herk calls allocate nothing (required before graph capture).
 * Replaces CutlassComplexGemm::init_herk / end_herk (cutlass_gemm_api.h:617-624). */
FTDX_API ftdx_status ftdx_init_herk(ftdx_handle h, int N, int K, int batch, void* stream);
FTDX_API ftdx_status ftdx_end_herk(ftdx_handle h);

/* Synchronise `stream`, then read and clear the device status word written by
 * bounded waits inside the kernels.  *bits = 0 means no wait timed out.
 * Returns FTDX_ERR_TIMEOUT if any bit was set. */
FTDX_API ftdx_status ftdx_device_status(ftdx_handle h, void* stream, uint32_t* bits);

/* ---- autotuning and graph replay ------------------------------------------
 * Replace tune_herk / strategy_cache::run_autotune and the direct-HERK graph
 * cache of the reference (cutlass_gemm_api.cu:1389-1409, 200-315, 1738-1807;
 * strategy_cache.hpp:504-721).
 *
 * The autotuner times every launch strategy (epilogue store mode x number
 * of persistent CTAs) for a problem shape on the caller's buffers and keeps
 * the fastest, in memory and appended to a text cache file (one line per
 * entry: "ftdx-tune 1 <device> <N> <Kp> <batch> <input> <output> <store>
 * <grid> <ms>").  ftdx_herk(..., tune=1) looks the shape up and tunes on a
 * miss (only when beta == 0 and the stream is not capturing). */

/* Set the cache file and load its entries.  Malformed lines are skipped and
 * reported as FTDX_ERR_CACHE (the valid entries are still loaded). */
FTDX_API ftdx_status ftdx_set_tune_cache(ftdx_handle h, const char* path);

/* Run the strategy sweep now for this shape (C is overwritten; beta = 0). */
FTDX_API ftdx_status ftdx_tune(ftdx_handle h, const void* A, void* C, int N, int K, int batch,
                               ftdx_input input, ftdx_output output, void* stream,
                               int* store_mode, int* grid, float* ms);

/* Query the tuned strategy of a shape (FTDX_ERR_CACHE when there is none),
 * for calls with FP8 compute. */
FTDX_API ftdx_status ftdx_lookup_tuned(ftdx_handle h, int N, int K, int batch, ftdx_input input,
                                       ftdx_output output, int* store_mode, int* grid, float* ms);
/* The same for calls with the given compute mode (the tuner keeps separate
 * entries per compute mode, e.g. FP8 and NVFP4 on the same FP32 input). */
FTDX_API ftdx_status ftdx_lookup_tuned_compute(ftdx_handle h, int N, int K, int batch,
                                               ftdx_input input, ftdx_compute compute,
                                               ftdx_output output, int* store_mode, int* grid,
                                               float* ms);

/* Graph mode: each distinct call (pointers, sizes, precisions, alpha, beta,
 * strategy) is captured once into a CUDA graph and replayed afterwards
 * (4-entry LRU).  Disabling releases the graphs. */
FTDX_API ftdx_status ftdx_set_graph_mode(ftdx_handle h, int enable);
FTDX_API int ftdx_graph_count(ftdx_handle h);

/* Strategy for calls that are not tuned (tune = 0, or no cache entry):
 * store_mode 0 = direct stores, 1 = shared-memory staging + bulk copies,
 * 2 = CTA-pair kernel (one tcgen05 cta_group::2 MMA over two SMs per
 * 256 x 128 tile; uniform ftdx_herk calls, ftdx_herk_batched_v and
 * ftdx_xengine (which takes 3 as 2 and 1 as 0: direct stores), others use 0);
 * 3 = CTA-pair kernel with bulk-copy stores for interior tiles (FP32 output,
 * alpha = 1, beta = 0; other tiles and calls as 2);
 * + 4 = operands as packed FP6 E3M2 planes (INT4 input; exact);
 * 2 + 8, 3 + 8 = CTA-pair kernel on signed 8-bit operands (kind::i8, S32
 * accumulation; uniform INT4 input; exact; ftdx_herk_batched_v runs these
 * as 2 and 3 on E4M3 operands);
 * 16 = the single-CTA kernel with the INT4 -> E4M3 promotion fused into it:
 * raw QC bytes are loaded by the correlator and converted in shared memory,
 * so no operand planes are written to or read from HBM and no workspace is
 * allocated for them (uniform INT4 calls with FP8 compute, K a multiple of 16
 * and A 16-byte aligned; other calls run as 0; not combinable with 4 or 8).
 * For NVFP4 compute, store_mode 2 selects the NVFP4 CTA-pair kernel and 0 / 1
 * the single-CTA one.
 * grid > 0 = that many persistent CTAs (capped at one per SM; even and capped
 * at the co-resident pairs for store_mode 2), 0 = one per SM, -1 = one CTA
 * (pair) per tile (a plain, non-persistent launch).  The tuner also times
 * store_mode 2, 3, 2 + 8, 3 + 8 and 16 for uniform INT4 calls, 2 and 3 for
 * ftdx_herk_batched_v, and both NVFP4 kernels. */
FTDX_API ftdx_status ftdx_set_strategy(ftdx_handle h, int store_mode, int grid);

/* Split-K for untuned calls: K is cut into `splits` (1..32) ranges of
 * k-blocks, each correlated into its own partial triangle, and a reduction
 * pass adds them (C = alpha * sum + beta * C).  Fills the GPU when a call has
 * fewer tiles than SMs (few inputs, long integrations); integer inputs stay
 * exact.  Not used with Kahan accumulation, the XEngine formats or NVFP4.
 * The autotuner also times split-K candidates for such calls and records the
 * choice in the cache (version 2 lines); ftdx_tuned_split_k returns it (-1: no
 * tuned entry). */
FTDX_API ftdx_status ftdx_set_split_k(ftdx_handle h, int splits);
FTDX_API int ftdx_tuned_split_k(ftdx_handle h, int N, int K, int batch, ftdx_input input,
                                ftdx_output output);

/* ---- correlation without any allocation -----------------------------------
 * No counterpart in the reference.  For callers that must not have the
 * library allocate GPU memory once they run: real-time pipelines that size
 * every buffer up front and cannot afford a cudaMalloc stalling or failing
 * mid-observation, and host frameworks whose device memory all comes from
 * their own pool.  Same result as
 *   ftdx_herk(h, A, C, N, K, batch, FTDX_IN_INT4, FTDX_COMPUTE_FP8,
 *             FTDX_OUT_FP32, FTDX_FORMAT_PACKED_TRIANGLE, 1, 0, stream, 0)
 * (QC int4 in, complex64 packed lower triangles out), but no handle and no
 * workspace: all scratch lives in one static device array of
 * FTDX_STATIC_SCRATCH_BYTES that every GPU loading this library holds until
 * the process exits.  Bytes needed, exactly:
 *   round_up(256 + 40*batch + 8*tiles, 1024) + 2*N*batch*Kp
 * with Kp = K rounded up to 128 and tiles = batch*nb*(nb+1)/2, nb = ceil(N/128)
 * (a 40-byte table entry per channel, 8 bytes per lower-triangle tile of
 * 128 x 128 inputs); scratch_used (may be NULL) receives it, also on refusal.
 * Larger problems return FTDX_ERR_CAPACITY before any GPU work, with the
 * sizes in ftdx_last_error(NULL); e.g. N = 1024 inputs, K = 1024 samples fits
 * 15 channels per call.  The first call on a device looks up the array's
 * device address (a one-time set-up); make that first call before any stream
 * capture.  All calls share the one array: calls that overlap on the GPU
 * (other streams, other threads) race and corrupt each other's results;
 * serialise them.  If status_out is not NULL the call synchronises `stream`
 * (an ordered copy on that stream, no device-wide wait) and stores the
 * device status bits there (FTDX_ERR_TIMEOUT if any is set); status_out must
 * be NULL while `stream` is being captured (FTDX_ERR_INVALID_ARG otherwise). */
#define FTDX_STATIC_SCRATCH_BYTES (32u << 20)
FTDX_API ftdx_status ftdx_herk_static(const void* A, void* C, int N, int K, int batch,
                                      void* stream, uint32_t* status_out, size_t* scratch_used);

/* ---- differentiation -------------------------------------------------------
 * No counterpart in the reference.
 *
 * Adjoint of the correlator: for visibilities R = V V^H and an upstream
 * gradient G = dL/dR (N x N complex64 per channel, row-major, batch back to
 * back; any matrix, not only Hermitian), dV = (G + G^H) V (N x K complex64
 * per channel, row-major).  V is QC int4 [batch][N][K] (FTDX_IN_INT4).
 * G + G^H is carried as bf16 hi + lo on the tensor cores with FP32
 * accumulation (relative error ~1e-5 of max|dV|).  N must be a multiple of 8.
 * Uses the handle's workspace (2 bytes x (4 N^2 + 2 N K) per channel). */
FTDX_API ftdx_status ftdx_herk_adjoint(ftdx_handle h, const void* G, const void* V, void* dV,
                                       int N, int K, int batch, ftdx_input input, void* stream);

/*
 * Gain calibration: for per-input complex gains g[N] shared by all channels,
 * observed and model visibilities R_obs, R_mod (packed lower triangles of
 * complex64, n_chans back to back, as ftdx_herk writes them) and real
 * weights W (packed, float, same layout),
 *   L = sum_f sum_{i,j} W_ij |R_obs,ij - g_i R_mod,ij conj(g_j)|^2
 * over the full Hermitian matrices (off-diagonal entries of the triangle
 * count twice), and grad[k] = dL/dRe(g_k) + i dL/dIm(g_k).  grad is
 * complex128 [N] (two doubles per input), loss one double; both are device
 * pointers, overwritten (not accumulated) by the call. */
FTDX_API ftdx_status ftdx_gain_gradient(ftdx_handle h, const void* R_obs, const void* R_mod,
                                        const float* W, const void* g, int N, int n_chans,
                                        double* grad, double* loss, void* stream);

/* Dense tensor-core throughput of this GPU (no counterpart in the reference),
 * for roofline denominators: back-to-back tcgen05 MMAs from shared-memory
 * tiles, FP32 accumulation, no loads or stores.
 *   kind 0: every SM pair issues `iters` cta_group::2 M = N = 256 FP8 E4M3
 *           (K = 32) MMAs on zero tiles;
 *   kind 1: the same with NVFP4 E2M1 and UE4M3 block-16 scales (K = 64);
 *   kind 2: as kind 0 on QC-valued operands (E4M3 codes of integers -7..7),
 *           in the CTA-pair correlator's order (two MMAs per 32 samples);
 *   kind 3: every SM issues `iters` cta_group::1 M = N = 128 FP8 MMAs on
 *           QC-valued operands in the single-CTA correlator's order (four
 *           per 32 samples into two accumulators).
 * Kinds 2 and 3 round `iters` up to whole 32-sample steps.  The fastest of
 * `reps` timed launches (after one warm-up) gives
 * *tflops = 2 M N K x MMAs x issuers / time.  Synchronises the device. */
FTDX_API ftdx_status ftdx_peak_probe(ftdx_handle h, int kind, int iters, int reps, double* tflops);

/* Kernel timing (no counterpart in the reference; its benches time whole
 * calls).  While enabled, CUDA events are recorded on the caller's stream
 * around every kernel this handle launches.  ftdx_profile_read synchronises,
 * returns the summed device time (ms) and launch count of the correlator
 * kernel (`herk_*`) and of the operand-promotion kernel (`prep_*`), and resets
 * the counters.  Any pointer may be NULL. */
FTDX_API ftdx_status ftdx_set_profiling(ftdx_handle h, int enable);
FTDX_API ftdx_status ftdx_profile_read(ftdx_handle h, double* herk_ms, int* herk_launches,
                                       double* prep_ms, int* prep_launches);

#ifdef __cplusplus
}
#endif
#endif /* FTDX_H_ */
