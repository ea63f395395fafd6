/* libmvs_b200 -- C ABI of the B200 (sm_100a) multiview-stereo kernels.
 *
 * Plain C: POD structs, raw pointers, sizes and an opaque stream handle
 * (a cudaStream_t passed as void*; NULL is the legacy default stream).  Every
 * call returns an int status (MVS_OK == 0, negative on failure); the message
 * of the last failure on the calling thread is mvs_last_error().  No call
 * resets the device.
 *
 * Pointer naming: d_* are device pointers, h_* host pointers.  Images are
 * dense row-major float32, stride == width, as the reference forces for every
 * image it allocates (memory.h:113-122).
 *
 * Each entry point names the reference interface it replaces.  The reference
 * exposes no C or FFI surface of its own: its callers are the C++ class
 * PlaneSweep (planesweep.h:27-510) and the free kernel wrappers of
 * kernels.cu.h and fusion.cu.h.  The class-level API is mirrored by the
 * mvs_ps_* and mvs_fusion_* handle functions below and by the C++ classes in
 * include/mvs_b200.hpp.
 */
#ifndef MVS_B200_H
#define MVS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------ */
#define MVS_OK 0
#define MVS_ERR_ARG -1      /* bad argument (null pointer, size, even window ...) */
#define MVS_ERR_NOMEM -2    /* device or host allocation failed */
#define MVS_ERR_CUDA -3     /* a CUDA runtime call or launch failed */
#define MVS_ERR_TIMEOUT -4  /* a bounded device-side wait gave up */
#define MVS_ERR_STATE -5    /* call out of order (e.g. denoise before a sweep) */
#define MVS_ERR_NOTBUILT -6 /* library built without the requested variant */

/* Message of the last failing call on this thread ("" after success). */
const char *mvs_last_error(void);
/* 10000 * major + 100 * minor + patch. */
int mvs_version(void);
/* Page-locked host memory (falls back to ordinary memory if page-locking
 * fails); free it with mvs_host_free.  The C++ layer keeps host images in it. */
void *mvs_host_alloc(size_t bytes);
void mvs_host_free(void *p);
/* Select the device for the calling thread (replaces PlaneSweep::cudaDevInit,
 * planesweep.cpp:30-58, without the device reset of cudaReset()). */
int mvs_set_device(int device);

/* ---- plane sweep ----------------------------------------------------------
 * Replaces the per-plane launch chain of PlaneSweep::PlaneSweepThread
 * (planesweep.cpp:163-259: transform_indexes, bilinear_interpolation,
 * windowed_mean_row/column, calculate_STD, element_multiply, calcNCC,
 * update_arrays, kernels.cu:4-235) and the epilogue of
 * PlaneSweep::RunAlgorithm (sum_depthmap_NCC, element_rdivide,
 * set_QNAN_value, kernels.cu:84-101,145-157,331-340; planesweep.cpp:105-131)
 * with fused kernels. */

#define MVS_MOMENTS_REFERENCE 0   /* the reference's naive box means, its order
                                     of operations and roundings */
#define MVS_MOMENTS_COMPENSATED 1 /* shifted FP32 window sums: E[x^2]-E[x]^2
                                     without catastrophic cancellation */

#define MVS_SWEEP_PER_VIEW 0   /* the reference: per-view NCC argmax, then the
                                  average of per-view depths above the NCC
                                  threshold (NaN -> zfar) */
#define MVS_SWEEP_AGGREGATED 1 /* extension: cost = 1 - mean NCC over views,
                                  stored as a BF16 cost volume [P][H][W],
                                  winner-take-all argmin per pixel */

typedef struct mvs_sweep_desc {
    int32_t width, height;  /* all views share the reference's size */
    int32_t n_views;        /* source views */
    int32_t n_planes;
    int32_t window;         /* odd, 3..15 (PlaneSweep::setWindowSize, planesweep.h:234) */
    int32_t moments;        /* MVS_MOMENTS_* */
    int32_t mode;           /* MVS_SWEEP_* */
    float std_threshold;    /* NCC := 0 where either window std is below (kernels.cu:59) */
    float ncc_threshold;    /* per-view depths with best NCC <= this are not averaged (kernels.cu:96) */
    float zfar;             /* depth written where no view passes (planesweep.cpp:131) */
} mvs_sweep_desc;

/* Bytes of device workspace mvs_sweep needs for `desc` when the optional
 * per-view outputs are not supplied. */
size_t mvs_sweep_workspace_bytes(const mvs_sweep_desc *desc);

/* Per-plane homographies built in FP64 on the device and stored as float:
 * H[v][p] = K (Rrel_v + trel_v e3^T / depth_p) K^-1, normalised so H22 = 1
 * (the matrix PlaneSweepThread builds in float on the host,
 * planesweep.cpp:195-203).  K is the reference's 1-based calibration matrix
 * (pixel (l,k) is (l+1,k+1)); Rrel/trel are reference->source
 * (PlaneSweep::RelativeMatrices).  h_K9: 9 doubles, h_Rrel: n_views*9,
 * h_trel: n_views*3 (host); d_depths: n_planes floats; d_H: n_views*n_planes*9
 * floats (device). */
int mvs_sweep_homographies(const mvs_sweep_desc *desc, const double *h_K9, const double *h_Rrel,
                           const double *h_trel, const float *d_depths, float *d_H, void *stream);

/* The fused sweep.  d_ref: H*W; d_srcs: n_views*H*W (0..255 grey);
 * d_H: n_views*n_planes*9 (as above); d_depths: n_planes.
 * Outputs (device):
 *   d_depth   H*W, required.  PER_VIEW: the averaged depthmap RunAlgorithm
 *             copies back.  AGGREGATED: depth of the winning plane.
 *   d_labels  PER_VIEW: n_views*H*W best plane index per view (-1: no plane
 *             with NCC > 0); AGGREGATED: H*W winning plane.  May be NULL.
 *   d_best    PER_VIEW: n_views*H*W best NCC per view (devbestNCC);
 *             AGGREGATED: H*W winning cost.  May be NULL.
 *   d_cost    AGGREGATED only: n_planes*H*W BF16 cost volume.  May be NULL.
 * d_workspace/workspace_bytes: at least mvs_sweep_workspace_bytes(desc) when
 * d_labels or d_best is NULL (PER_VIEW), else may be NULL. */
int mvs_sweep(const mvs_sweep_desc *desc, const float *d_ref, const float *d_srcs, const float *d_H,
              const float *d_depths, float *d_depth, int32_t *d_labels, float *d_best, uint16_t *d_cost,
              void *d_workspace, size_t workspace_bytes, void *stream);

/* mvs_sweep without caller workspace (no counterpart in the reference).
 * For callers that cannot allocate device memory while they run -- host
 * frameworks or plugin hosts that fix a library's device memory at start-up,
 * real-time loops that cannot take cudaMalloc's latency and implicit
 * synchronisation.  The sweep's scratch (one 64-bit word per pixel and view,
 * or per pixel in the aggregated mode) lives in a fixed device array of
 * mvs_sweep_noalloc_scratch_bytes() = 32 MiB inside the library, which a GPU
 * holds from the first call on it until the process exits; a larger sweep
 * is rejected with MVS_ERR_ARG.  The call itself allocates nothing (no
 * cudaMalloc, no cudaFree).  The array is reserved when CUDA loads the module
 * that holds it, which under CUDA's default lazy module loading happens at the
 * first call on each device: that call looks up the array's device address
 * (cudaGetSymbolAddress), which loads the module and reserves the 32 MiB then.
 * So make that first call at start-up (a small frame will do) and outside any
 * stream capture.  Every call looks the address up again for the current
 * device and context.  All calls share the one array,
 * which keeps the last call's contents: calls that can overlap on the GPU
 * (other streams, other host threads) race and must be serialised by the
 * caller.  Arguments and outputs as mvs_sweep. */
int mvs_sweep_noalloc(const mvs_sweep_desc *desc, const float *d_ref, const float *d_srcs, const float *d_H,
                      const float *d_depths, float *d_depth, int32_t *d_labels, float *d_best, uint16_t *d_cost,
                      void *stream);
size_t mvs_sweep_noalloc_scratch_bytes(void);

/* Winner-take-all argmin over a stored BF16 cost volume (d_cost:
 * n_planes * n_pixels, as mvs_sweep writes it: costs >= 0; n_pixels divisible
 * by 8; n_planes <= 65535).
 * Writes the winning plane's depth (zfar if none), optional label and cost. */
int mvs_sweep_wta_volume(const uint16_t *d_cost, const float *d_depths, int32_t n_pixels, int32_t n_planes,
                         float zfar, float *d_depth, int32_t *d_labels, float *d_best, void *stream);

/* ---- TGV2 multiview refinement ------------------------------------------
 * Replaces the launch chain of PlaneSweep::TGV (planesweep.cpp:381-536):
 * Anisotropic_diffusion_tensor, the per-view linearisation
 * (TGV2_transform_coordinates, TGV2_calculate_coordinate_derivatives,
 * TGV2_calculate_derivativeF, bilinear_interpolation, TGV2_calculate_Iu,
 * subtract) and the iteration (TGV2_updateP_tensor_weighed, TGV2_updateQ,
 * TGV2_updateR, TGV2_updateU_tensor_weighed), TGV2_kernels.cu:54-365. */
typedef struct mvs_tgv2_params {
    int32_t niters;       /* iterations per linearisation (reference: niters) */
    int32_t warps;        /* linearisations (reference: warps) */
    double lambda, alpha0, alpha1, tau, sigma, beta, gamma; /* as PlaneSweep::TGV */
    double tol;           /* extension: energy tolerance, 0 = fixed count.  The
                             energy E (FP64, on the device) is evaluated every
                             check_every iterations of a linearisation; the run
                             stops at the first check j >= stop_window with
                             |E_j - E_{j-W}| <= tol * W * |E_{j-W}|, W =
                             stop_window: the mean relative change per check
                             over the last W checks is at most tol.  (The
                             primal-dual energy is not monotone: a single
                             check's change dips below tol on the way down.) */
    int32_t check_every;  /* iterations between energy evaluations (tol > 0) */
    int32_t max_iters;    /* extension: total cap (0 = warps * niters) */
    int32_t iteration_kernel; /* MVS_TGV2_ITER_*: how the iterations run (same results) */
    int32_t stop_window;  /* checks W of the stopping test, 1..MVS_TGV2_STOP_WINDOW_MAX;
                             0 = MVS_TGV2_STOP_WINDOW_DEFAULT.  W = 1 compares
                             consecutive checks only. */
} mvs_tgv2_params;

#define MVS_TGV2_STOP_WINDOW_DEFAULT 5
#define MVS_TGV2_STOP_WINDOW_MAX 16

#define MVS_TGV2_ITER_AUTO 0     /* the fastest measured form: as MVS_TGV2_ITER_LAUNCH */
#define MVS_TGV2_ITER_LAUNCH 1   /* one fused launch per iteration (dependent launches, state in
                                    L2), energy checks and the stopping test on the device */
#define MVS_TGV2_ITER_PERSISTENT 2 /* one cooperative launch per linearisation with the state on
                                    chip, when the image fits one tile per SM (else as LAUNCH) */

size_t mvs_tgv2_workspace_bytes(int32_t width, int32_t height, int32_t n_views);

/* d_ref255: H*W, d_srcs255: n_views*H*W (0..255).  h_K9/h_invK9: the
 * reference's float K (1-based) and K^-1; h_Rrel: n_views*9, h_trel:
 * n_views*3 (float, as PlaneSweep::RelativeMatrices computes them).
 * d_u: H*W, in: start depth (NULL-equivalent: pass u_init_const = 1 and the
 * reference's constant start is used when `u_from_input` is 0); out: result.
 * iters_out / energy_out (host, may be NULL): iterations run and last
 * energy (FP64, evaluated on the device). */
int mvs_tgv2_run(int32_t width, int32_t height, int32_t n_views, const float *d_ref255, const float *d_srcs255,
                 const float *h_K9, const float *h_invK9, const float *h_Rrel, const float *h_trel,
                 const mvs_tgv2_params *params, int32_t u_from_input, float u_init_const, float *d_u,
                 int32_t *iters_out, double *energy_out, void *d_workspace, size_t workspace_bytes,
                 void *stream);

/* Extension, no counterpart in the reference: TGV2 from a warm start.  The
 * data term is linearised at d_u_lin (H*W; the plain run's start, e.g. the
 * sweep's winner-take-all depth), so the energy is the plain run's; the
 * primal starts at d_u (H*W, in/out) and d_v (2*H*W, vx then vy, in/out; NULL
 * starts v at 0 and discards it).  dual_sigma > 0 starts the regulariser's
 * duals p, q, and dual_sigma_r > 0 the data duals r, one dual step of that
 * size from zero (0: at zero, as the plain run; a large dual_sigma_r starts r
 * at the sign of each view's residual).  d_pq (5*H*W: px, py, qx, qy, qz)
 * and d_r (n_views*H*W), when not NULL, are instead the start of those duals
 * and receive their final values, so a run can continue another exactly.
 * With d_u equal to d_u_lin, v = 0 and both steps 0 this is mvs_tgv2_run
 * with u_from_input = 1.  Later linearisations (warps > 1) restart as the
 * plain run does. */
int mvs_tgv2_run_warm(int32_t width, int32_t height, int32_t n_views, const float *d_ref255, const float *d_srcs255,
                      const float *h_K9, const float *h_invK9, const float *h_Rrel, const float *h_trel,
                      const mvs_tgv2_params *params, const float *d_u_lin, float *d_u, float *d_v, double dual_sigma,
                      double dual_sigma_r, float *d_pq, float *d_r, int32_t *iters_out, double *energy_out, void *d_workspace, size_t workspace_bytes,
                      void *stream);

/* ---- TGV2 towards a sparse depthmap -----------------------------------------
 * Replaces PlaneSweep::TGVdenoiseFromSparse's chain (planesweep.cpp:596-674):
 * Anisotropic_diffusion_tensor, then niters x (TGV2_updateP_tensor_weighed on
 * u, TGV2_updateQ, TGV2_updateU_sparseDepthTensor with v passed as its own
 * over-relaxation; TGV2_kernels.cu:54-85,340-445), data weight 1 where
 * d_sparse > 0.  d_depthmap: the start depth (the sweep result), d_sparse: the
 * sparse depth (0 = none), both in depth units, H*W; d_out = u * zfar.  theta
 * is accepted for the reference's signature; it only reaches the over-relaxed
 * u, which the iteration never reads, so it does not change the result. */
size_t mvs_tgv2_sparse_workspace_bytes(int32_t width, int32_t height);

int mvs_tgv2_sparse(int32_t width, int32_t height, const float *d_ref255, const float *d_depthmap,
                    const float *d_sparse, float zfar, int32_t niters, double alpha0, double alpha1, double tau,
                    double sigma, double theta, double beta, double gamma, float *d_out, void *d_workspace,
                    size_t workspace_bytes, void *stream);

/* ---- TV-L1 depth denoise --------------------------------------------------
 * Replaces PlaneSweep::CudaDenoise's chain (planesweep.cpp:297-379):
 * Anisotropic_diffusion_tensor + denoising_TVL1_calculateP_tensor_weighed +
 * denoising_TVL1_update (kernels.cu:283-370). d_depth: in/out, H*W. */
typedef struct mvs_tvl1_params {
    int32_t niters;
    double lambda, tau, sigma, theta, beta, gamma; /* as PlaneSweep::CudaDenoise */
} mvs_tvl1_params;

size_t mvs_tvl1_workspace_bytes(int32_t width, int32_t height);

int mvs_tvl1_denoise(int32_t width, int32_t height, const float *d_ref255, float *d_depth, float znear, float zfar,
                     const mvs_tvl1_params *params, void *d_workspace, size_t workspace_bytes, void *stream);

/* ---- back-projection --------------------------------------------------------
 * Replaces compute3D (kernels.cu:405-429) as PlaneSweep::get3Dcoordinates
 * drives it (planesweep.cpp:551-586): for z < 5.5, X = Rr (z K^-1 (x+1,y+1,1)) + t;
 * else Z = -9 and X, Y are left untouched.  h_* are float 3x3 / 3-vectors. */
int mvs_compute3d(int32_t width, int32_t height, const float *d_depth, const float *h_invK9, const float *h_Rr9,
                  const float *h_t3, float *d_X, float *d_Y, float *d_Z, void *stream);

/* ---- TV-L1 histogram fusion -------------------------------------------------
 * Replaces fusionData<N, Device> (fusion.h:105-1055) and the launch wrappers
 * FusionUpdateHistogram / FusionUpdateU / FusionUpdateP /
 * FusionUpdateIteration (fusion.cu:72-99, fusion.cu.h:40-173).
 *
 * Layout (SoA, x fastest, n = width*height*depth voxels):
 *   u[n], v[n] float; p[3][n] float; hist[n][hist_stride] uint16 (bins counts
 *   per voxel, padded to hist_stride = 8 or 16 for 128-bit access). */
typedef struct mvs_fusion mvs_fusion;

int mvs_fusion_create(int32_t width, int32_t height, int32_t depth, int32_t bins, const float *corner_a,
                      const float *corner_b, mvs_fusion **out);
int mvs_fusion_destroy(mvs_fusion *f);
int mvs_fusion_set_volume(mvs_fusion *f, const float *corner_a, const float *corner_b);
/* Zero u, v, p and the histograms. */
int mvs_fusion_reset(mvs_fusion *f, void *stream);
/* Histogram votes of n_maps depthmaps (d_depths: n_maps*h*w device floats,
 * h_K/h_R: n_maps*9 floats, h_t: n_maps*3: world->camera, 0-based K), in map
 * order, in one voxel pass (fusion.cu:5-43 + fusionData::updateHist). */
int mvs_fusion_histogram(mvs_fusion *f, const float *d_depths, int32_t n_maps, int32_t w, int32_t h,
                         const float *h_K, const float *h_R, const float *h_t, float threshold, void *stream);
/* n_iters TV-L1 primal-dual iterations, each FusionUpdateU then
 * FusionUpdateP (fusion.cu:45-70), fused into one voxel pass per iteration. */
int mvs_fusion_tvl1(mvs_fusion *f, int32_t n_iters, double tau, double lambda, double sigma, void *stream);
/* Single steps at the reference's granularity. */
int mvs_fusion_update_u(mvs_fusion *f, double tau, double lambda, void *stream);
int mvs_fusion_update_p(mvs_fusion *f, double sigma, void *stream);
/* FusionUpdateIteration: one depthmap's histogram votes, then U, then P. */
int mvs_fusion_iteration(mvs_fusion *f, const float *d_depth, int32_t w, int32_t h, const float *h_K9,
                         const float *h_R9, const float *h_t3, float threshold, double tau, double lambda,
                         double sigma, void *stream);
/* Host copies of the state (NULL skips a field).  h_p: 3*n, h_hist: bins*n
 * (plane per bin). */
int mvs_fusion_download(mvs_fusion *f, float *h_u, float *h_v, float *h_p, uint16_t *h_hist);
int mvs_fusion_upload(mvs_fusion *f, const float *h_u, const float *h_v, const float *h_p, const uint16_t *h_hist);
/* Device pointers of the current state (valid until the next call on f). */
int mvs_fusion_device_state(mvs_fusion *f, float **d_u, float **d_v, float **d_p, uint16_t **d_hist,
                            int32_t *hist_stride);
/* World coordinates of the voxels with lo < u < hi (the GUI keeps
 * -1 < u < 0, pclviewer.cpp:1058-1074), x fastest; h_xyz: 3*capacity floats.
 * *count receives the number of such voxels (may exceed capacity). */
int mvs_fusion_extract(mvs_fusion *f, float lo, float hi, float *h_xyz, int64_t capacity, int64_t *count);

/* ---- PlaneSweep drop-in handle ------------------------------------------------
 * Mirrors class PlaneSweep (planesweep.h:27-510) for callers that bind C:
 * host images in, host depthmaps out; device buffers are owned by the handle
 * and reused across calls.  Bool results of the reference map to MVS_OK /
 * negative codes.  Getters copy into caller memory (the reference returns
 * pointers to its internal CamImage objects). */
typedef struct mvs_planesweep mvs_planesweep;

int mvs_ps_create(mvs_planesweep **out);
int mvs_ps_destroy(mvs_planesweep *ps);
/* HostRef / HostSrc with their R, t (planesweep.h:31-34, cam_image.h:10-11).
 * The images are copied into the handle's page-locked host images and
 * uploaded to the device in the same pass (on the default stream, MB by MB as
 * they are copied); RunAlgorithm then uploads neither.  Images in page-locked
 * memory (mvs_host_alloc, cudaHostAlloc, registered) are uploaded in one copy
 * from the caller's buffer while they are copied, which the link runs faster.
 * Either way the caller's buffers are free again when the call returns.
 * Without a device the images stay on the host. */
int mvs_ps_set_reference(mvs_planesweep *ps, const float *h_img, int32_t width, int32_t height, const float *R9,
                         const float *t3);
int mvs_ps_set_sources(mvs_planesweep *ps, const float *h_imgs, int32_t n, const float *R9s, const float *t3s);
int mvs_ps_set_K(mvs_planesweep *ps, const float *K9);            /* setK */
int mvs_ps_set_z(mvs_planesweep *ps, float znear, float zfar);     /* setZ */
int mvs_ps_set_number_of_planes(mvs_planesweep *ps, int32_t n);    /* setNumberofPlanes */
int mvs_ps_set_number_of_images(mvs_planesweep *ps, int32_t n);    /* setNumberofImages */
int mvs_ps_set_window_size(mvs_planesweep *ps, int32_t n);         /* setWindowSize (odd only) */
int mvs_ps_set_std_threshold(mvs_planesweep *ps, float th);        /* setSTDthreshold */
int mvs_ps_set_ncc_threshold(mvs_planesweep *ps, float th);        /* setNCCthreshold */
int mvs_ps_set_alternative_relative_matrix_method(mvs_planesweep *ps, int32_t alt);
/* Extensions: explicit plane list (NULL/0 restores the reference's znear..zfar
 * float loop), moments/mode/homography precision. */
int mvs_ps_set_plane_depths(mvs_planesweep *ps, const float *depths, int32_t n);
int mvs_ps_set_sweep_options(mvs_planesweep *ps, int32_t moments, int32_t mode, int32_t fp64_homographies);
int mvs_ps_run_algorithm(mvs_planesweep *ps);                      /* RunAlgorithm */
int mvs_ps_cuda_denoise(mvs_planesweep *ps, int32_t niters, double lambda, double tau, double sigma,
                        double theta, double beta, double gamma);  /* CudaDenoise */
int mvs_ps_tgv(mvs_planesweep *ps, int32_t niters, int32_t warps, double lambda, double alpha0, double alpha1,
               double tau, double sigma, double beta, double gamma); /* TGV (u = 1 start) */
/* TGVdenoiseFromSparse: TGV2 from the last sweep depthmap towards h_sparse
 * (width*height, 0 = no sample); the result replaces the TGV depthmap. */
int mvs_ps_tgv_denoise_from_sparse(mvs_planesweep *ps, const float *h_sparse, int32_t niters, double alpha0,
                                   double alpha1, double tau, double sigma, double theta, double beta, double gamma);
/* Extension: TGV2 started from the last sweep depthmap (start = 1), from
 * h_u_init (start = 2) or from 1 (start = 0), with an energy tolerance. */
int mvs_ps_tgv_ext(mvs_planesweep *ps, const mvs_tgv2_params *params, int32_t start, const float *h_u_init,
                   int32_t *iters_out, double *energy_out);
/* Getters (planesweep.h:287-437).  Image getters copy width*height values of
 * the current reference frame (mvs_ps_get_size); a result of a frame of
 * another size (the reference was set again since) is refused with
 * MVS_ERR_STATE. */
int mvs_ps_get_size(mvs_planesweep *ps, int32_t *width, int32_t *height);
int mvs_ps_get_depthmap(mvs_planesweep *ps, float *out);
int mvs_ps_get_depthmap8u(mvs_planesweep *ps, uint8_t *out);
int mvs_ps_get_depthmap_denoised(mvs_planesweep *ps, float *out);
int mvs_ps_get_depthmap8u_denoised(mvs_planesweep *ps, uint8_t *out);
int mvs_ps_get_depthmap_tgv(mvs_planesweep *ps, float *out);
int mvs_ps_get_depthmap8u_tgv(mvs_planesweep *ps, uint8_t *out);
/* getDepthmapDenoisedPtr: device pointer, overwritten by each CudaDenoise. */
int mvs_ps_get_depthmap_denoised_ptr(mvs_planesweep *ps, float **d_ptr);
/* Per-view labels / best NCC of the last sweep (n_views*H*W, n_views the
 * views that sweep used: at most the number of sources), extension. */
int mvs_ps_get_view_labels(mvs_planesweep *ps, int32_t *out);
int mvs_ps_get_view_best(mvs_planesweep *ps, float *out);
int mvs_ps_get_3d_coordinates(mvs_planesweep *ps, float *X, float *Y, float *Z); /* get3Dcoordinates */
int mvs_ps_get_plane_count(mvs_planesweep *ps, int32_t *n);
/* ---- data formats either side of the path ---------------------------------
 * ICL-NUIM camera file (Reader::getcamParameters / getcamK / computeRT,
 * reader.cpp:181-296): the cam_pos, cam_dir, cam_up and cam_right lines give
 * the 1-based K of a width x height image (negative fy), the camera->world
 * rotation R (columns: right, down, forward) and t = cam_pos, in the reader's
 * float arithmetic; the pose is for PlaneSweep's alternative relative-matrix
 * method (setAlternativeRelativeMatrixMethod(true)).  The reference fixes the
 * image at 640 x 480. */
int mvs_read_icl_camera(const char *path, int32_t width, int32_t height, float *h_K9, float *h_R9, float *h_t3);
/* PLY point cloud (x y z float, optional red green blue uchar), ASCII or
 * binary little-endian; replaces the PCL cloud of pclviewer.cpp:1058-1083. */
int mvs_write_ply(const char *path, const float *h_xyz, const uint8_t *h_rgb, int64_t n, int32_t binary);
/* The depth colour map of the reference's viewer (PCLViewer::RGBdepthmapColor,
 * pclviewer.cpp:1084-1115): n gray values -> n RGB triples. */
void mvs_depth_color(const uint8_t *h_gray, int64_t n, uint8_t *h_rgb);

/* ---- synthetic scenes (no counterpart in the reference) -------------------
 * Ray casts the seeded box scenes that stand in for the reference's datasets
 * (ICL-NUIM, KITTI; reader.cpp, kitti_reader.cpp): an optional room seen
 * from inside plus axis-aligned boxes, textured by value noise (a periodic
 * lattice^3 table, `octaves` octaves from base_freq, each octave shifted by
 * offsets[o]).  All FP64.  d_gray255 (may be NULL: depth only) receives
 * 255 * intensity (0.5 where nothing is hit), d_depth the camera z (50 where
 * nothing is hit).  h_invK9: inverse of the 0-based K; h_R9: world->camera
 * rotation; h_center3: camera centre in the world. */
typedef struct mvs_box_scene {
    int32_t inside_room, n_boxes;      /* n_boxes <= 32 */
    double room_min[3], room_max[3];
    const double *h_boxes;             /* n_boxes x (min xyz, max xyz) */
    const double *d_noise;             /* lattice^3 doubles, x slowest */
    int32_t lattice, octaves;          /* octaves <= 8 */
    double base_freq;
    double offsets[8][3];
} mvs_box_scene;

int mvs_render_scene(const mvs_box_scene *scene, const double *h_invK9, const double *h_R9, const double *h_center3,
                     int32_t width, int32_t height, float *d_gray255, float *d_depth, void *stream);

/* ---- batched frames (extension: the reference sweeps one frame per call) --
 * Many reference frames of any size, view count (<= 16), plane count and
 * window go through one CUDA-graph launch: FP64 homographies of every
 * (frame, view, plane), then one persistent sweep kernel over a work list of
 * (frame, tile, plane chunk) items, in the aggregated mode (cost = 1 - mean
 * NCC over views, winner-take-all; outputs as mvs_sweep's aggregated mode).
 * Per-frame completion times are recorded on the device.
 *
 * The work list's plane chunk, persistent CTAs per SM and item order come from
 * `tuning`, or, when it is NULL, from an autotuner that times every candidate
 * on the batch itself (once per batch shape in a process; the choice is
 * cached).  Device pointers and K stay the caller's and must outlive the
 * batch; h_K9 (1-based K), h_Rrel and h_trel (n_views x 9 / x 3, as
 * mvs_sweep_homographies takes them) are read at creation. */
#define MVS_BATCH_ORDER_FRAME 0          /* frame by frame, in the given order */
#define MVS_BATCH_ORDER_LARGEST_FIRST 1  /* frame by frame, most work first */
#define MVS_BATCH_ORDER_INTERLEAVED 2    /* round robin over frames */

typedef struct mvs_batch_frame {
    int32_t width, height, n_views, n_planes, window;
    float std_threshold, zfar;
    const float *d_ref, *d_srcs, *d_depths;   /* H*W, n_views*H*W (0..255), n_planes */
    const double *h_K9, *h_Rrel, *h_trel;
    float *d_depth;                           /* outputs, H*W; labels and best may be NULL */
    int32_t *d_labels;
    float *d_best;
} mvs_batch_frame;

typedef struct mvs_batch_tuning {
    int32_t planes_per_chunk;   /* 0: whole plane range per item */
    int32_t ctas_per_sm;        /* persistent CTAs per SM (1..3) */
    int32_t order;              /* MVS_BATCH_ORDER_* */
    int32_t tile_step;          /* tile shape: 32 rows x (64 - 8 tile_step) columns for windows up to
                                   9x9, x (56 - 8 tile_step) above; 0 or 1.  The compensated
                                   moments shift each tile's sums by the tile's reference mean, so
                                   two tile shapes agree to rounding, not bit for bit: pass an
                                   explicit tuning for bit-reproducible batches. */
} mvs_batch_tuning;

typedef struct mvs_batch mvs_batch;

int mvs_batch_create(mvs_batch **out, const mvs_batch_frame *frames, int32_t n, int32_t moments,
                     const mvs_batch_tuning *tuning);
int mvs_batch_destroy(mvs_batch *batch);
int mvs_batch_get_tuning(const mvs_batch *batch, mvs_batch_tuning *tuning);
/* new relative poses for every frame (views of frame 0 first) */
int mvs_batch_set_poses(mvs_batch *batch, const double *h_Rrel, const double *h_trel, void *stream);
/* one graph launch: homographies + sweep + winner-take-all of every frame */
int mvs_batch_run(mvs_batch *batch, void *stream);
/* per-frame latency of the last run (ms from the launch's start to the
 * frame's last tile), after synchronising `stream` */
int mvs_batch_frame_latency_ms(mvs_batch *batch, float *h_ms, void *stream);
int64_t mvs_batch_work_items(const mvs_batch *batch);

/* ---- TGV2 warm-start network (no counterpart in the reference) -----------
 * A 4-level U-Net (16/32/64/128 channels, 3x3 convolutions with ReLU, 2x2
 * average pooling, nearest upsampling with skip concatenation, a 1x1 head)
 * mapping the sweep's winner-take-all depth, its matching cost and the
 * reference image to a prediction of the converged TGV2 primal (u, v) for
 * mvs_tgv2_run_warm.  BF16 activations and weights on the tensor cores with
 * FP32 accumulation; FP32 master weights and Adam.
 *
 * norm7 (may be NULL for the defaults {0.25, -1, 2, 1, 0.01, 1, 1}):
 *   depth_scale, depth_shift  input channel 0 = depth * scale + shift
 *   cost_clip                 input channel 1 = 1 - min(cost, clip)
 *   u_scale, v_scale          u = wta + u_scale * head0, v = v_scale * head{1,2}
 *   w_u, w_v                  loss = mean(w_u (u - u*)^2 + w_v |v - v*|^2)
 * height and width must be multiples of 8.  Tensors are batch-major:
 * d_wta, d_cost, d_ref255, d_u: batch*H*W; d_v: batch*2*H*W (vx then vy).
 * Parameters are one FP32 array: per 3x3 layer W[cout][cin][3][3] then
 * bias[cout] (mvs_unet_layer_info gives the offsets; layer 14 is the head,
 * W[3][16] then bias[3]). */
typedef struct mvs_unet mvs_unet;

int mvs_unet_create(mvs_unet **out, int32_t batch, int32_t height, int32_t width, const float *norm7);
int mvs_unet_destroy(mvs_unet *net);
int64_t mvs_unet_param_count(const mvs_unet *net);
int mvs_unet_layer_info(const mvs_unet *net, int32_t layer, int32_t *cin, int32_t *cout, int64_t *w_off,
                        int64_t *b_off);
int mvs_unet_set_params(mvs_unet *net, const float *h_params);            /* also resets Adam */
int mvs_unet_get_params(mvs_unet *net, float *h_params, float *h_grads);  /* either may be NULL */
int mvs_unet_forward(mvs_unet *net, const float *d_wta, const float *d_cost, const float *d_ref255, float *d_u,
                     float *d_v, void *stream);
/* gradients of the loss of the last forward against (d_u_target, d_v_target) */
int mvs_unet_backward(mvs_unet *net, const float *d_u_target, const float *d_v_target, double *loss_out,
                      void *stream);
int mvs_unet_adam_step(mvs_unet *net, float lr, float beta1, float beta2, float eps, void *stream);
int mvs_unet_train_step(mvs_unet *net, const float *d_wta, const float *d_cost, const float *d_ref255,
                        const float *d_u_target, const float *d_v_target, float lr, double *loss_out, void *stream);
/* MVS_ERR_TIMEOUT if a bounded tensor-core wait gave up since the net was made */
int mvs_unet_check(mvs_unet *net, void *stream);

/* Single 3x3 layers (zero padding, NHWC bf16 bits, channels multiples of 16),
 * for checks against a CPU restatement.  d_w: FP32 W[cout][cin][3][3];
 * d_wpack: scratch of 2*9*cin*cout bf16; d_err: device int set on a timeout.
 * backward: d_dw (9*cin*cout) and d_db (cout, may be NULL) are accumulated
 * into; d_dx (may be NULL) = input gradient, times (x > 0) when mask_x;
 * tensor_cores = 0 computes the weight gradient on the CUDA cores instead. */
int mvs_conv3x3_forward(const uint16_t *d_in, int32_t cin, const float *d_w, const float *d_bias, int32_t cout,
                        int32_t batch, int32_t height, int32_t width, int32_t relu, uint16_t *d_out,
                        uint16_t *d_wpack, int32_t *d_err, void *stream);
int mvs_conv3x3_backward(const uint16_t *d_x, int32_t cin, const float *d_w, const uint16_t *d_dz, int32_t cout,
                         int32_t batch, int32_t height, int32_t width, int32_t mask_x, uint16_t *d_dx, float *d_dw,
                         float *d_db, uint16_t *d_wpack, int32_t *d_err, int32_t tensor_cores, void *stream);

/* Device time (ms) of the last run_algorithm / tgv / cuda_denoise call,
 * measured with CUDA events around the kernels only. */
int mvs_ps_get_last_kernel_ms(mvs_planesweep *ps, float *ms);

#ifdef __cplusplus
}
#endif
#endif
