/*
 * b200d2.h -- C ABI of the B200 coarse-pass diff2 library (libb200d2.so).
 *
 * RELION's coarse expectation step scores every particle image against every
 * projected reference orientation at every trial translation:
 *
 *   diff2[p][o][t] = sum_px  corr_p(px)/2 * | proj_o(px) - shift_t(img_p)(px) |^2
 *
 * This header is the drop-in boundary that replaces the reference harness's
 * C++ entry points (Edgarrrrrr/T2-RELION-kernel; file:line given per entry).
 * All pointers named d_* are device pointers; h_* are host pointers.  Every
 * call returns a b200d2_status (0 = success) instead of raising SIGSEGV as the
 * reference's HANDLE_ERROR does (src/common.h:20-36).  Calls taking a stream
 * are asynchronous on that stream and do no host synchronisation.
 */
#ifndef B200D2_H_
#define B200D2_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum b200d2_status {
  B200D2_OK = 0,
  B200D2_ERR_INVALID = 1,     /* bad argument / shape */
  B200D2_ERR_UNSUPPORTED = 2, /* configuration outside the supported path */
  B200D2_ERR_CUDA = 3,        /* CUDA runtime error */
  B200D2_ERR_OOM = 4,         /* device allocation failed */
  B200D2_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  B200D2_ERR_NO_DEVICE = 6,   /* no usable sm_100 device */
  B200D2_ERR_TOO_LARGE = 7,   /* request exceeds a fixed capacity */
  B200D2_ERR_CANCELLED = 8    /* a served request was cancelled before it ran */
} b200d2_status;

/* How the projector volume is interpolated. */
enum {
  /* cudaArray + cudaFilterModeLinear texture, clamp, unnormalised
   * coordinates: the reference's default (src/acc_projector_impl.h:40-107). */
  B200D2_INTERP_TEXTURE = 0,
  /* linear device arrays + software trilinear with exact FP32 weights: the
   * reference's PROJECTOR_NO_TEXTURES path (src/acc_projector_impl.h:109-116,
   * src/cuda_device_utils.cuh:73-108). */
  B200D2_INTERP_LINEAR = 1
};

/* Precision of the cross term in the tensor-core path. */
enum {
  B200D2_PREC_FP32 = 0,    /* plain FP32 CUDA-core kernel (the drop-in) */
  B200D2_PREC_TF32 = 1,    /* one TF32 product, FP32 accumulation in TMEM */
  B200D2_PREC_TF32X3 = 2,  /* hi*hi + hi*lo + lo*hi TF32 split */
  B200D2_PREC_BF16X3 = 3,  /* hi*hi + hi*lo + lo*hi BF16 split */
  B200D2_PREC_FP64 = 4,    /* FP64 CUDA-core kernel (GPU oracle) */
  /* FP16 operands with power-of-two scales: every particle's weighted image
   * and every orientation's projection are scaled so that their largest
   * component lies in [2^13, 2^14); the scales are undone exactly in the
   * final combination. */
  B200D2_PREC_FP16 = 5,    /* one scaled FP16 product */
  B200D2_PREC_FP16X3 = 6   /* hi*hi + hi*lo + lo*hi scaled FP16 split */
};

/*
 * Kernel-side projector view, passed by value to kernels.  Mirrors
 * AccProjectorKernel (src/acc_projectorkernel_impl.h:15-60): same field names
 * and meaning, plus the texture handles and the linear arrays.
 */
typedef struct b200d2_view {
  int mdlX, mdlXY, mdlZ;
  int imgX, imgY, imgZ;
  int mdlInitY, mdlInitZ;
  int maxR, maxR2, maxR2_padded;
  float padding_factor;
  unsigned long long tex_re; /* cudaTextureObject_t, 0 if absent */
  unsigned long long tex_im;
  const float* lin_re; /* device [mdlZ][mdlY][mdlX], NULL if absent */
  const float* lin_im;
  int interp; /* B200D2_INTERP_* used by kernels taking this view */
  /* the same volume as one float2 (re, im) texture, 0 if absent: kernels
   * fetch both channels at once from it (identical values: the filtering
   * weights are per fetch, not per channel) */
  unsigned long long tex_c;
} b200d2_view;

typedef struct b200d2_projector b200d2_projector; /* opaque, owns device memory */

/* ------------------------------------------------------------------------
 * Projector (replaces AccProjector::setMdlDim + initMdl,
 * src/acc_projector_impl.h:10-216, and constructFromFile :300-356)
 * ---------------------------------------------------------------------- */

/* Upload a padded Hermitian-half Fourier volume [mdlZ][mdlY][mdlX] (x fastest)
 * from host memory.  use_texture: 1 = texture objects only, 0 = linear arrays
 * only, 2 = both.  Only 3D references (mdlZ > 1) are supported. */
int b200d2_projector_create(int mdlX, int mdlY, int mdlZ, int mdlInitY,
                            int mdlInitZ, int mdlMaxR, float padding_factor,
                            const float* h_real, const float* h_imag,
                            int use_texture, b200d2_projector** out);

/* Load the reference harness's projector_proc_*.dat format
 * (src/acc_projector_impl.h:300-356). */
int b200d2_projector_load_dat(const char* path, int use_texture,
                              b200d2_projector** out);

/* Free all device memory of the projector (AccProjector::clear). */
int b200d2_projector_destroy(b200d2_projector* p);

/* Model geometry: dims[0..5] = mdlX, mdlY, mdlZ, mdlInitY, mdlInitZ, mdlMaxR. */
int b200d2_projector_dims(const b200d2_projector* p, int* dims, float* pf);

/* AccProjectorKernel::makeKernel (src/acc_projectorkernel_impl.h:410-433):
 * maxR = min(mdlMaxR, imgMaxR), maxR2 = maxR^2,
 * maxR2_padded = int(maxR^2 * pf * pf).  interp selects the projection path
 * (the projector must hold the matching representation). */
int b200d2_projector_view(const b200d2_projector* p, int imgX, int imgY,
                          int imgZ, int imgMaxR, int interp, b200d2_view* out);

/* Central-slice projections of O orientations at K pixels (project3Dmodel,
 * src/acc_projectorkernel_impl.h:178-252): d_out_re/d_out_im[o*K + k] for
 * pixel (d_px[k], d_py[k]), 0 outside the projector radius. */
int b200d2_project_pixels(const b200d2_view* view, const float* d_eulers,
                          int O, const int* d_px, const int* d_py, int K,
                          float* d_out_re, float* d_out_im, void* stream);

/* ------------------------------------------------------------------------
 * Single-particle drop-in (replaces runDiff2KernelCoarse,
 * src/acc_helper_functions_impl.h:15-499, non-CC 3D-reference 2D-image branch)
 *
 * d_diff2s[o*T + t] += diff2(o, t), accumulating onto the caller's buffer
 * exactly as the reference does (src/diff2.cuh:533-536).  d_eulers holds 9
 * floats per orientation (row-major 3x3); image arrays hold N_img half-plane
 * pixels in pixel_index2coor order.  corr must be >= 0.
 * precision: B200D2_PREC_FP32 (FP32 CUDA cores, within 1e-5 of the
 * reference's own kernel), or a tensor-core precision: the particle then runs
 * through the batch pipeline (projection, FP64 norms, tcgen05 contraction)
 * on a workspace the library owns, one per (device, stream), allocated with
 * cudaMallocAsync on `stream` when first needed and grown the same way (the
 * first call per stream, and a larger problem, allocate).  At C2 sizes (4608
 * orientations x 113 translations, image 64) BF16x3 takes 0.18 ms per
 * particle against 0.45 ms for the FP32 kernel.
 * ---------------------------------------------------------------------- */
int b200d2_diff2_coarse(const b200d2_view* view, const float* d_trans_x,
                        const float* d_trans_y, const float* d_corr,
                        const float* d_real, const float* d_imag,
                        const float* d_eulers, float* d_diff2s, size_t O,
                        size_t T, size_t N_img, void* stream, int precision);

/* FP64 variant (replaces runDiff2KernelCoarseDouble,
 * src/acc_helper_functions_impl.h:503-854): double arithmetic for the phase
 * shift, the differences and the sum; projections are the same FP32
 * interpolated samples.  filter_img zeroes image pixels outside the radius as
 * the reference's filter_img flag does (src/diff2.cuh:339-345). */
int b200d2_diff2_coarse_f64(const b200d2_view* view, const float* d_trans_x,
                            const float* d_trans_y, const float* d_corr,
                            const float* d_real, const float* d_imag,
                            const float* d_eulers, double* d_diff2s, size_t O,
                            size_t T, size_t N_img, int filter_img,
                            void* stream);

/* Cross-correlation coarse score (replaces the do_CC branch of
 * runDiff2KernelCoarse, src/acc_helper_functions_impl.h:441-498, 3D reference
 * and 2D images: cuda_kernel_diff2_CC_coarse, src/diff2.cuh:691-809):
 *   d_diff2s[o*T + t] = -(sum_px corr Re(conj(A_o) S_t)) / sqrt(sum_px corr |A_o|^2)
 * written, not accumulated (as the reference does).  Pixels outside the
 * projector radius have A = 0 and take no part.  FP32 sums
 * (precision B200D2_PREC_FP32); the _f64 form sums in FP64.  The reference's
 * local_sqrtXi2 argument is not used by its kernel and is not taken here. */
int b200d2_diff2_coarse_cc(const b200d2_view* view, const float* d_trans_x,
                           const float* d_trans_y, const float* d_corr,
                           const float* d_real, const float* d_imag,
                           const float* d_eulers, float* d_diff2s, size_t O,
                           size_t T, size_t N_img, void* stream, int precision);
int b200d2_diff2_coarse_cc_f64(const b200d2_view* view, const float* d_trans_x,
                               const float* d_trans_y, const float* d_corr,
                               const float* d_real, const float* d_imag,
                               const float* d_eulers, double* d_diff2s, size_t O,
                               size_t T, size_t N_img, void* stream);

/* Fine-pass diff2 over a job list (replaces cuda_kernel_diff2_fine,
 * src/diff2.cuh:540-682, 2D image against a 3D reference; the reference has
 * no host wrapper for it).  Job j (j < todo_blocks) scores orientation
 * d_rot_idx[d_job_idx[j]] of d_eulers[][9] against the d_job_num[j]
 * consecutive translations starting at d_trans_idx[d_job_idx[j]] and writes
 *   d_diff2s[d_job_idx[j] + i] = sum_init + sum_px corr/2 |proj - shift_i(img)|^2
 * over all image_size pixels (the fine kernel's pixel mapping).  FP32, like
 * the reference.  Any number of translations per job.  Index arrays are
 * device uint64 (the reference's unsigned long). */
int b200d2_diff2_fine(const b200d2_view* view, const float* d_eulers,
                      const float* d_real, const float* d_imag,
                      const float* d_trans_x, const float* d_trans_y,
                      const float* d_corr, float* d_diff2s, size_t image_size,
                      float sum_init, size_t todo_blocks,
                      const uint64_t* d_rot_idx, const uint64_t* d_trans_idx,
                      const uint64_t* d_job_idx, const uint64_t* d_job_num,
                      void* stream);

/* CC form of the fine pass (replaces cuda_kernel_diff2_CC_fine,
 * src/diff2.cuh:811-960): same job list, writes
 *   d_diff2s[d_job_idx[j] + i] = -sum_px corr Re(conj(proj) shift_i(img))
 *                                / sqrt(sum_px corr |proj|^2)
 * (full corr, no sum_init; the reference passes sum_init and
 * exp_local_sqrtXi2 but does not read them).  FP32 cross sums, FP64 norm and
 * quotient. */
int b200d2_diff2_fine_cc(const b200d2_view* view, const float* d_eulers,
                         const float* d_real, const float* d_imag,
                         const float* d_trans_x, const float* d_trans_y,
                         const float* d_corr, float* d_diff2s, size_t image_size,
                         size_t todo_blocks, const uint64_t* d_rot_idx,
                         const uint64_t* d_trans_idx, const uint64_t* d_job_idx,
                         const uint64_t* d_job_num, void* stream);

/* ------------------------------------------------------------------------
 * Batched coarse pass (layout diff2[p][o][t]).  The reference
 * launches one runDiff2KernelCoarse per particle (src/main.cu:483-503); this
 * call scores P particles that share the orientation and translation sets in
 * one pass.  Image p lives at d_real/d_imag/d_corr + p * img_stride.
 * ---------------------------------------------------------------------- */
typedef struct b200d2_batch {
  const float* d_eulers; /* [O][9] */
  int O;
  const float* d_trans_x; /* [T] phase slopes (RELION: -2*pi*shift/ori_size) */
  const float* d_trans_y;
  int T;
  int P;
  int N_img;
  const float* d_real; /* [P][img_stride] CTF-folded image (RELION Fimg) */
  const float* d_imag;
  const float* d_corr; /* [P][img_stride] Minvsigma2 * CTF^2 (>= 0) */
  long long img_stride;
  float* d_diff2;      /* [P][O][T] */
  int accumulate;      /* 1: d_diff2 += diff2 (drop-in), 0: d_diff2 = diff2 */
  double* d_min;       /* optional [P]: per-particle minimum diff2 */
  long long* d_argmin; /* optional [P]: o*T + t of that minimum (lowest index on ties) */
  /* Optional listed pixels (the reference's filtered layout, src/main.cu:88-151
   * and the coor_xy argument of its optimised functors): when d_coor_xy is not
   * NULL the first n_listed image entries are the pixels at integer-valued
   * coordinates (d_coor_xy[2i], d_coor_xy[2i+1]), |x|,|y| <= 512, shared by
   * all particles, and entries n_listed .. N_img-1 lie outside the projector
   * radius (they add only corr/2 |X|^2).  Tensor-core precisions only.  The
   * coordinates are device data, checked on the device: x outside [0, 512],
   * y outside [-512, 512] or a value that is not an integer sets the
   * workspace status word to B200D2_ERR_INVALID (b200d2_workspace_status),
   * and the scores of that call are not to be used. */
  const float* d_coor_xy;
  int n_listed;
  /* B200D2_SCORE_DIFF2 (0): diff2 as above.  B200D2_SCORE_CC (1): the
   * cross-correlation score of cuda_kernel_diff2_CC_coarse
   * (src/diff2.cuh:691-809), d_diff2[p][o][t] = -sum corr Re(conj(A_o) S_t)
   * / sqrt(sum corr |A_o|^2), with d_min / d_argmin the most negative score.
   * FP32 CUDA cores and the tensor-core forms (norms in FP64). */
  int score;
} b200d2_batch;

enum { B200D2_SCORE_DIFF2 = 0, B200D2_SCORE_CC = 1 };

/* Bytes of device scratch the batch needs for `precision` (0 for the
 * CUDA-core paths). */
size_t b200d2_diff2_coarse_batch_workspace(const b200d2_view* view,
                                           const b200d2_batch* batch,
                                           int precision);

/* Run the batch.  precision: B200D2_PREC_FP32 (CUDA cores) or one of the
 * tensor-core forms.  d_workspace must hold the bytes reported above. */
int b200d2_diff2_coarse_batch(const b200d2_view* view, const b200d2_batch* batch,
                              int precision, void* d_workspace,
                              size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------
 * Plans: uneven batches in one persistent contraction launch, autotuned and
 * captured in a CUDA graph.  Each particle has its own orientation subset
 * (indices into the plan's orientation set) and its own translation set; its
 * output is diff2[o_local][t] in its own buffer.  The reference scores such
 * particles one runDiff2KernelCoarse call at a time (src/main.cu:483-503).
 * A plan owns its workspace and tables; b200d2_plan_run replays the captured
 * pipeline on the same device buffers, so callers refill the images in place.
 * ---------------------------------------------------------------------- */
typedef struct b200d2_particle_desc {
  const float* d_real;  /* [N_img] device, CTF-folded image */
  const float* d_imag;
  const float* d_corr;  /* [N_img] device, Minvsigma2 * CTF^2 */
  float* d_diff2;       /* [O][T] device output of this particle */
  const int* h_orient;  /* host [O]: indices into the plan's orientations, NULL = 0..O-1 */
  int O;
  const float* h_trans_x; /* host [T] phase slopes */
  const float* h_trans_y;
  int T;
} b200d2_particle_desc;

enum {
  B200D2_PLAN_AUTOTUNE = 1,   /* time the contraction variants, keep the fastest */
  B200D2_PLAN_GRAPH = 2,      /* capture the whole pipeline in a CUDA graph */
  B200D2_PLAN_ACCUMULATE = 4, /* add onto d_diff2 instead of overwriting */
  /* order orientations by viewing direction (Hilbert curve over the
   * projection normal's z and azimuth) and particles by the column blocks
   * their subsets touch, so that local orientation subsets touch few output
   * tiles; outputs are unchanged */
  B200D2_PLAN_REORDER = 8
};

#define B200D2_PLAN_MAX_VARIANTS 16
typedef struct b200d2_plan_info {
  int P, O_all, rows, tiles, tiles_dense, row_bytes, graph, stages;
  long long evals;        /* sum over particles of O * T */
  size_t workspace_bytes; /* plan-owned device bytes (workspace and tables) */
  /* chosen contraction variant: tile width (orientations per tile) and
   * k-splits per tile (row_bytes above is its k-block row width) */
  int tile_n, split;
  int pair;               /* 1: CTA-pair 256 x 256 tiles */
  int tiles_n128;         /* work-list length with 128-wide tiles */
  int tiles_pair;         /* work-list length with 256 x 256 tiles */
  /* autotuner: variants timed, each (row_bytes, tile_n, split, pair) and its
   * contraction time in ms (n_tuned = 0 without B200D2_PLAN_AUTOTUNE) */
  int n_tuned;
  int tuned_variant[B200D2_PLAN_MAX_VARIANTS][4];
  double tuned_ms[B200D2_PLAN_MAX_VARIANTS];
  /* FP64 norm stage: blocks of (particle tile x 64 orientations) that some
   * particle needs, for particle tiles of 64, 32 and 16 (plan order); the
   * tile height in use; with B200D2_PLAN_AUTOTUNE each height's time in ms */
  int norm_tiles[3];
  int norm_tile_p;
  double norm_tuned_ms[3];
} b200d2_plan_info;

typedef struct b200d2_plan b200d2_plan;

/* Build a plan for P particles against O_all orientations d_eulers[O_all][9].
 * Host metadata is copied; device pointers must stay valid while the plan
 * is used.  precision: a tensor-core precision.  d_min/d_argmin (optional,
 * device [P]) receive each particle's minimum diff2 and o_local*T + t. */
int b200d2_plan_create(const b200d2_view* view, const float* d_eulers, int O_all,
                       int N_img, const b200d2_particle_desc* particles, int P,
                       int precision, int flags, double* d_min,
                       long long* d_argmin, b200d2_plan** out);
int b200d2_plan_run(b200d2_plan* plan, void* stream);
int b200d2_plan_get_info(const b200d2_plan* plan, b200d2_plan_info* info);
int b200d2_plan_destroy(b200d2_plan* plan);

/* ------------------------------------------------------------------------
 * Serving: a request loop over resident references with continuous
 * batching.  No counterpart in the reference (it has no serving path).
 * Requests (a set of particles scored against an orientation subset of one
 * reference at one translation set) are queued by b200d2_server_submit and
 * admitted by a scheduler thread as soon as a stream slot is free and their
 * device footprint fits the HBM budget, so requests that arrive while others
 * run start at once and overlap on the GPU.  Each admitted request copies its
 * host inputs in, runs the tensor-core pipeline and copies its outputs out on
 * its own stream; its device memory is released stream-ordered.
 * ---------------------------------------------------------------------- */
typedef struct b200d2_server b200d2_server;

typedef struct b200d2_request {
  int ref;              /* reference id from b200d2_server_add_reference */
  int P;                /* particles */
  const float* h_real;  /* host [P][N_img]; pageable host buffers (inputs and
                           outputs) go through the server's page-locked staging
                           buffers, page-locked ones are copied directly */
  const float* h_imag;
  const float* h_corr;
  const int* h_orient;  /* host [O]: indices into the reference's orientations */
  int O;
  const float* h_trans_x; /* host [T] phase slopes */
  const float* h_trans_y;
  int T;
  float* h_diff2;       /* optional host [P][O][T] output */
  double* h_min;        /* optional host [P]: minimum diff2 per particle */
  long long* h_argmin;  /* optional host [P]: o_local*T + t of that minimum */
} b200d2_request;

typedef struct b200d2_server_stats {
  long long submitted, completed, rejected, evals;
  int in_flight, queued, max_in_flight;
  size_t bytes_in_use, peak_bytes;
  double admit_host_s; /* scheduler-thread time spent issuing admitted requests' work */
  long long cancelled;
  /* merged admissions (b200d2_server_set_merging) and the requests they ran */
  long long merged_admissions, merged_requests;
  double stream_s; /* slot-stream time of the completed admissions (first copy in to
                      last copy out; a merged admission counted once) */
  /* longest scheduler-thread time of one admission, and of two of its
   * phases: the slot's device buffer (growth maps memory) and the launch of
   * the request's work; each covers the time since the previous
   * b200d2_server_get_stats, which resets them */
  double admit_host_max_s, admit_grow_max_s, admit_launch_max_s;
  /* since the previous read as well: the longest wait of a request from
   * submission to admission, and the longest time from an admission to its
   * completion callback beyond its stream time */
  double queue_wait_max_s, done_lag_max_s;
} b200d2_server_stats;

/* slots: concurrent streams; hbm_budget_bytes: device bytes the in-flight
 * requests may hold; precision: tensor-core precision or B200D2_PREC_FP32.
 * Each slot keeps a device buffer between requests (powers of two from
 * 32 MiB, released for idle slots when a growth would pass the budget), from
 * a memory pool of the server's own; creation maps min(budget, 8 GiB) of it.
 * The default memory pool of the process is not touched. */
int b200d2_server_create(int slots, size_t hbm_budget_bytes, int precision,
                         b200d2_server** out);
/* Register a resident reference: a projector view and its host orientation
 * grid h_eulers[O_all][9] (copied); image geometry from the view, N_img
 * pixels per image. */
int b200d2_server_add_reference(b200d2_server* s, const b200d2_view* view,
                                const float* h_eulers, int O_all, int N_img,
                                int* ref_id);
/* Queue a request (host buffers must stay valid until it completes).
 * Returns B200D2_ERR_TOO_LARGE if it can never fit the budget. */
int b200d2_server_submit(b200d2_server* s, const b200d2_request* req,
                         long long* ticket);
/* Wait for a request: status of the request, its latency (submit to
 * completion, seconds) and its device time (seconds: the stream time of the
 * run that carried it, shared by the requests of a merged admission). */
int b200d2_server_wait(b200d2_server* s, long long ticket, double timeout_s,
                       double* latency_s, double* device_s);
int b200d2_server_get_stats(b200d2_server* s, b200d2_server_stats* st);
/* Merged admissions.  When a slot frees up while more requests are queued
 * than slots are idle, the scheduler runs the first queued request that fits
 * together with later queued requests on the same reference (arrival order),
 * each of at most max_request_particles particles (a larger request fills
 * the GPU on its own), up to max_requests requests and max_particles
 * particles in all, as one batch: one copy-in, one pipeline run and one
 * copy-out on one slot, instead of a pipeline per request, when the merged
 * run fits the buffer an idle slot already holds (a merge never grows a
 * slot's buffer, which maps memory while the queue waits).  The batch is
 * block-diagonal: each request's particles are scored against its own
 * orientations at its own translations only, so no request pays for
 * another's, and each result equals the request's result alone (same
 * kernels, same sums).  The merged requests complete together.  Tensor-core
 * servers only; max_requests = 1 turns merging off.  Default: 8 requests,
 * 512 particles, 128 particles per request. */
int b200d2_server_set_merging(b200d2_server* s, int max_requests, int max_particles,
                              int max_request_particles);
/* Cancel a queued request: it will not run, and b200d2_server_wait returns
 * B200D2_ERR_CANCELLED for it.  B200D2_ERR_UNSUPPORTED when the request has
 * been admitted already (work on the GPU is not interrupted; wait for it),
 * B200D2_ERR_INVALID for an unknown ticket. */
int b200d2_server_cancel(b200d2_server* s, long long ticket);
/* Drain all requests and free the server. */
int b200d2_server_destroy(b200d2_server* s);

/* Tensor-core batch that allocates nothing.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: a host whose device memory is
 * owned by another allocator (RELION's caching allocator reserves most of the
 * card), a request path that must not pay cudaMalloc's device
 * synchronisation, or a plug-in that receives only its input and output
 * buffers.  Same semantics and outputs as b200d2_diff2_coarse_batch with a
 * tensor-core precision, but the workspace is a fixed scratch area of
 * B200D2_STATIC_SCRATCH_BYTES inside the library's device image, held by
 * every GPU that loads the library until the process exits.  This entry
 * point never splits the contraction over k, so it needs the batch's
 * workspace without the split-K partial-sum buffer, which can be less than
 * b200d2_diff2_coarse_batch_workspace reports; a batch whose need exceeds
 * the scratch is rejected with B200D2_ERR_TOO_LARGE before anything runs
 * (64 MiB holds, for example, 8 particles x 576 orientations x 21
 * translations at image 32, or 16 particles x 1024 orientations x 113
 * translations at image 64).  The scratch address is looked up on the first
 * call on each device, and again after the device's context is recreated
 * (cudaDeviceReset): make those calls before any stream capture.  Calls share the scratch, so calls that
 * overlap on the GPU race; serialise them.  Runs all stages on `stream`. */
#define B200D2_STATIC_SCRATCH_BYTES (64ull << 20)
int b200d2_diff2_coarse_batch_static(const b200d2_view* view,
                                     const b200d2_batch* batch, int precision,
                                     void* stream);

/* Per-particle minimum and its index over d_diff2[p][0 .. n) (FP64 min,
 * lowest index on ties).  Used by the CUDA-core path; fused into the
 * tensor-core epilogue. */
int b200d2_minloc(const float* d_diff2, long long n, int P, double* d_min,
                  long long* d_argmin, void* stream);

/* Batched multi-particle CTF folding (no counterpart in the reference, which
 * receives folded inputs from RELION): for P raw particle transforms X
 * (d_real/d_imag + p * img_stride, N_img half-plane pixels in
 * pixel_index2coor order) and each particle's CTF d_ctf[p] (device array),
 *   Fimg = X / CTF  (X where |CTF| <= 1e-8),   corr = Minvsigma2 * CTF^2
 * into d_fimg_real/d_fimg_imag/d_corr (same layout), the inputs of the coarse
 * pass.  CTF = -(sqrt(1-Q^2) sin(chi) + Q cos(chi)) * scale * exp(-B k^2/4),
 * chi = pi lambda dz k^2 - pi/2 Cs lambda^3 k^4 + phase_shift, dz the
 * astigmatic defocus at the pixel's azimuth, k = (x, y) / (ori_size *
 * pixel_A), all in FP64.  d_minvsigma2 is one row per particle
 * (minvsigma2_stride = N_img or more) or one row shared by all (stride 0).
 * maxR is the image radius used by pixel_index2coor. */
typedef struct b200d2_ctf {
  float defocus_u_A, defocus_v_A, defocus_angle_deg; /* astigmatic defocus (A) */
  float voltage_kV, cs_mm, amp_contrast, phase_shift_deg;
  float bfactor; /* envelope exp(-B k^2 / 4); 0 = none */
  float scale;   /* 0 is taken as 1 */
} b200d2_ctf;
int b200d2_ctf_fold(const float* d_real, const float* d_imag, long long img_stride,
                    int P, int N_img, int imgX, int imgY, int maxR, int ori_size,
                    float pixel_A, const b200d2_ctf* d_ctf,
                    const float* d_minvsigma2, long long minvsigma2_stride,
                    float* d_fimg_real, float* d_fimg_imag, float* d_corr,
                    void* stream);

/* Coarse weights of a scored batch, the step after the coarse pass (its
 * RELION driver kernel_weights_exponent_coarse is a commented stub at
 * src/utilities.h:405-443 of the reference harness):
 *   w[p][o][t] = pdf_orient[o] * pdf_offset[t] * exp(-(diff2[p][o][t] - min_p))
 * computed in FP64 from the FP32 diff2 block diff2[P][O][T].  min_p is
 * d_min[p] (e.g. the batch's per-particle minimum) or, with d_min NULL, the
 * minimum of the particle's block.  d_pdf_orient [O] / d_pdf_offset [T] may be
 * NULL (all ones); a zero prior gives a zero weight.  d_sum[p] receives the
 * sum of the particle's weights, added in a fixed order (bit-reproducible).
 * With normalize != 0 the stored weights are w / d_sum[p].  d_weights may be
 * NULL when normalize == 0 (sums only).  The workspace is
 * b200d2_coarse_weights_workspace(P, O*T) bytes of device memory, contents
 * ignored; one call at a time per workspace.  Asynchronous on `stream`. */
size_t b200d2_coarse_weights_workspace(int P, long long n);
int b200d2_coarse_weights(const float* d_diff2, int P, int O, int T,
                          const double* d_min, const double* d_pdf_orient,
                          const double* d_pdf_offset, int normalize,
                          double* d_weights, double* d_sum, void* d_workspace,
                          size_t workspace_bytes, void* stream);

/* Significant samples of a weighted batch, the step after the coarse weights
 * (RELION's pass-0 significance; its device kernels in the reference harness
 * are cuda_kernel_find_threshold_idx_in_cumulative and
 * cuda_kernel_array_over_threshold, src/cuda_device_utils.cuh:238-266).  For
 * particle p, over its weights d_weights[p][0..n) that are > 0 and finite,
 * sorted ascending with inclusive cumulative sums c_k:
 *   thr  = (1 - adaptive_fraction) * d_sum[p]
 *   idx  = i + 1 for the i with c_i <= thr < c_{i+1}, else 0
 *   nsig = count - idx; if max_significants > 0 and nsig > max_significants:
 *          nsig = max_significants, idx = count - nsig
 *   d_sig_weight[p] = sorted[idx],  d_nsig[p] = nsig,
 *   d_passed[p][i]  = d_weights[p][i] >= d_sig_weight[p]   (0 or 1; optional)
 * The cumulative sums are taken exactly (no sort: radix selection with exact
 * integer bucket sums, double-double across buckets), so the result is that
 * of exact arithmetic; a particle with no positive weight gets nsig = 0 and
 * d_sig_weight = +inf (nothing passes).  n < 2^27 per particle.  The
 * workspace is b200d2_significance_workspace(P, n) bytes of device memory
 * (about 8 bytes per weight), contents ignored; one call at a time per
 * workspace.  Asynchronous on `stream`. */
size_t b200d2_significance_workspace(int P, long long n);
int b200d2_significance(const double* d_weights, int P, long long n,
                        const double* d_sum, double adaptive_fraction,
                        long long max_significants, double* d_sig_weight,
                        long long* d_nsig, uint8_t* d_passed,
                        void* d_workspace, size_t workspace_bytes,
                        void* stream);

/* A significance mask (or any byte mask) d_mask[P][n] packed to bits for a
 * copy to the host, eight times smaller: d_bits[P][(n + 31) / 32] words, word
 * j of particle p holding samples 32 j .. 32 j + 31, sample 32 j + i in bit i
 * (set when the byte is non-zero; bits past n zero).  No counterpart in the
 * reference, whose mask stays one byte per sample.  Asynchronous on
 * `stream`. */
int b200d2_pack_mask(const unsigned char* d_mask, int P, long long n,
                     unsigned int* d_bits, void* stream);

/* Final combination diff2 = nA - 2 cross of the tensor-core forms, where nA =
 * sum w|X|^2 + sum w|A|^2 is accumulated in FP64 and cross comes from the
 * FP32 tensor-core accumulator.  B200D2_COMBINE_DF32 (default): nA is kept as
 * an unevaluated sum of two floats (48-bit significand) and the combine is
 * one FMA and one add, within 2 ulp of the FP64 combine rounded to FP32;
 * B200D2_COMBINE_FP64: FP64 arithmetic, rounded once.  Process-wide; read
 * when a contraction is launched (plans capture it in their graph). */
enum { B200D2_COMBINE_DF32 = 0, B200D2_COMBINE_FP64 = 1 };
int b200d2_set_combine(int mode);

/* Contraction variant used by the tensor-core batch entry points
 * (b200d2_diff2_coarse_batch, _stage, _static and the server), process-wide:
 * row_bytes 64 or 128 (k-block row width), tile_n 256 or 128 (orientations
 * per tile), split = k-splits per tile (partial sums added in split order in
 * FP64), pair = 1 for CTA-pair tiles (a cluster of two CTAs computes a
 * 256 x 256 tile with cta_group::2 MMAs; 256-wide, no k-splits), 2 for
 * single-CTA tiles.  0 in any field restores the default (64-byte rows,
 * 256-wide tiles, k-splits chosen from the tile count, at most the
 * workspace's capacity, CTA pairs when the pair tiles fill the GPU).  Plans
 * created with B200D2_PLAN_AUTOTUNE choose their own variant; other plans take
 * this setting at creation (single-CTA 256-wide tiles when it is 0). */
int b200d2_set_gemm_variant(int row_bytes, int tile_n, int split, int pair);

/* CUDA graphs of the batch entry point (b200d2_diff2_coarse_batch with a
 * tensor-core precision), process-wide, on by default: a call's launches are
 * fixed by its arguments (view, batch fields and device pointers, precision,
 * workspace, stream, device) and the process-wide settings above, so the
 * second call with the same arguments captures the pipeline into a graph and
 * later calls launch that graph, which takes about a tenth of the host time
 * of the dozen launches and stream waits it replaces.  Input contents may
 * change between calls; the pointers may not, without making a new
 * signature.  Up to 32 signatures are kept (least recently used evicted).
 * Calls made while the caller captures `stream` into its own graph launch
 * directly.  enable: 1 on, 0 off (every call launches directly). */
int b200d2_set_batch_graphs(int enable);

/* Run a single stage of the batch pipeline, so that a caller can time one
 * kernel with events on its stream.  Stages are numbered in pipeline order
 * from 0; b200d2_stage_name returns NULL past the last stage of `precision`.
 * Running every stage in order is equivalent to b200d2_diff2_coarse_batch,
 * except that the CUDA-core path then always accumulates. */
int b200d2_diff2_coarse_batch_stage(const b200d2_view* view,
                                    const b200d2_batch* batch, int precision,
                                    int stage, void* d_workspace,
                                    size_t workspace_bytes, void* stream);
const char* b200d2_stage_name(int precision, int stage);

/* Status word of the last tensor-core batch run in this workspace: 0,
 * B200D2_ERR_INVALID when caller-listed pixel coordinates were out of range
 * or not integers, or B200D2_ERR_TIMEOUT when a bounded device-side wait gave
 * up (the outputs of that run are then incomplete).  Synchronises `stream`. */
int b200d2_workspace_status(const void* d_workspace, void* stream,
                            int* status);

/* How the tensor-core contraction gets its A operand (the weighted,
 * phase-shifted images; the reference builds it per output tile in shared
 * memory, src/translation_matrix_handler.cuh:279-369,432-511).  0 (default):
 * A is written to the workspace by its own kernel and read back by TMA.  1:
 * generator warps of the contraction write each k-block of A into shared
 * memory from the weighted image and the translation's separable phase rows,
 * so A never goes through device memory (no operand-generation stage, no A
 * planes in the workspace: 385 MB less at 256 x 4608 x 113 at image 64), at
 * the cost of shared-memory bandwidth (that contraction is 1.3x slower).
 * Both give bit-identical scores.  Process-wide; read when a workspace size
 * is queried, a batch runs or a plan is created, so query, run and plan
 * creation must see the same mode. */
int b200d2_set_operand_gen(int mode);

/* Projection cache of b200d2_diff2_coarse with a tensor-core precision (on by
 * default).  The library-owned workspace keeps the last call's projections;
 * a call skips its projection stage when its Euler matrices equal, bit for
 * bit, those that were projected (compared on the device) and nothing else
 * they depend on has changed: the view, the precision, the workspace layout,
 * and no projector created or destroyed since.  Scores are bit-identical
 * either way.  The FP16 forms, and projections of fewer than 2^20 samples
 * (orientations x pixels, quicker than the check), always project.  0 turns
 * it off. */
int b200d2_set_projection_cache(int enable);

/* Test hook for the give-up path of the bounded device-side waits (no
 * counterpart in the reference, whose waits cannot hang: it recomputes instead
 * of spinning, src/translation_matrix_handler.cuh:145-206).  Sets, process
 * wide, the limit in nanoseconds of the single-CTA contraction's pipeline
 * waits (its shared-memory stage ring and accumulator hand-over); 0 restores
 * the default of 4 s.  When a wait runs out the kernel raises an abort flag
 * that its other roles see, lets its copies and MMAs in flight finish (those
 * drain waits keep the 4 s limit), frees its tensor memory and returns, and
 * b200d2_workspace_status reports B200D2_ERR_TIMEOUT.  The CTA-pair
 * contraction keeps the default limit.  Read when a contraction is launched
 * (plans capture it in their graph).  For tests only: a short limit makes
 * correct runs fail. */
int b200d2_set_wait_limit_ns(unsigned long long ns);

/* Number of kernels this library has launched in the process so far (all
 * entry points, all devices).  Lets a caller count launches in a region. */
unsigned long long b200d2_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* B200D2_H_ */
