/* CPU oracle for the multiview-stereo hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's plane sweep, TGV2 refinement,
 * TV-L1 depth denoise and TV-L1 histogram fusion.  Only the tests, the
 * fixture generator, the smoke check and the CPU-baseline legs of bench.py
 * call it, and only as the checker; the product path never does.
 *
 * Every routine exists twice, generated from oracle/mvs_oracle_impl.h:
 *   *_f32  mirrors the reference's own arithmetic (float storage, the same
 *          double intermediates, the same operation order) and is checked
 *          bit for bit against the reference compiled for the CPU;
 *   *_f64  is the same algorithm with every float replaced by double -- the
 *          FP64 oracle that error bounds are stated against.
 *
 * Images are dense row-major (stride = width).  Homographies are row-major
 * 3x3 and already normalised (H[8] == 1).
 */
#ifndef MVS_ORACLE_H
#define MVS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_DECL(R, S)                                                                          \
    void orc_inv3_##S(const R *M9, R *out9);                                                    \
    void orc_relative_##S(const R *Rref9, const R *tref3, const R *Rsrc9, const R *tsrc3,        \
                          int alternative, R *Rrel9, R *trel3);                                 \
    void orc_homography_##S(const R *K9, const R *invK9, const R *Rrel9, const R *trel3, R d,    \
                            R *H9);                                                             \
    void orc_sweep_view_##S(int w, int h, const float *ref, const float *src, const R *H,       \
                            const float *depths, int nplanes, int winsize, double stdthresh,    \
                            R *best, R *depth, int32_t *label);                                 \
    void orc_sweep_ncc_##S(int w, int h, const float *ref, const float *src, const R *H9,       \
                           int winsize, double stdthresh, R *ncc);                              \
    void orc_sweep_ncc_band_##S(int w, int h, int nview, const float *ref, const float *srcs,       \
                                const R *H, int nplanes, int winsize, double stdthresh, int y0,  \
                                int y1, R *out);                                                 \
    void orc_sweep_combine_##S(int w, int h, int nview, const R *best, const R *depth,          \
                               double nccthresh, double zfar, R *out);                          \
    void orc_tensor_##S(int w, int h, const R *img, double beta, double gamma, R *T11, R *T12,  \
                        R *T21, R *T22);                                                        \
    void orc_tgv2_linearize_##S(int w, int h, const R *src01, const R *ref01, const R *u0,      \
                                const R *K9, const R *invK9, const R *Rrel9, const R *trel3,    \
                                R *It, R *Iu);                                                  \
    void orc_tgv2_iteration_##S(int w, int h, int nview, const R *T11, const R *T12,            \
                                const R *T21, const R *T22, const R *It, const R *Iu,           \
                                const R *u0, R *u, R *u1x, R *u1y, R *ubar, R *u1xbar,          \
                                R *u1ybar, R *Px, R *Py, R *Qx, R *Qy, R *Qz, R *Qw, R *r,       \
                                R *prodsum, double lambda, double alpha0, double alpha1,        \
                                double tau, double sigma);                                      \
    double orc_tgv2_energy_##S(int w, int h, int nview, const R *T11, const R *T12,             \
                               const R *T21, const R *T22, const R *It, const R *Iu,            \
                               const R *u0, const R *u, const R *u1x, const R *u1y,             \
                               double lambda, double alpha0, double alpha1);                    \
    void orc_tgv_sparse_iteration_##S(int w, int h, const R *T11, const R *T12, const R *T21,    \
                                      const R *T22, const R *wgt, const R *Ds, R *u, R *vx,     \
                                      R *vy, R *Px, R *Py, R *Qx, R *Qy, R *Qz, R *Qw,          \
                                      double alpha0, double alpha1, double tau, double sigma);  \
    void orc_tvl1_denoise_##S(int w, int h, const R *ref255, const R *depth, double znear,      \
                              double zfar, int niters, double lambda, double tau, double sigma, \
                              double theta, double beta, double gamma, R *out);                 \
    void orc_fusion_histogram_##S(int bins, int vw, int vh, int vd, const float *a,              \
                                  const float *b, uint16_t *hist, const float *depth, int w,    \
                                  int h, const R *K9, const R *R9, const R *t3, double thr);     \
    void orc_fusion_u_##S(int bins, int vw, int vh, int vd, const uint16_t *hist, R *u, R *v,   \
                          const R *p, double tau, double lambda);                               \
    void orc_fusion_p_##S(int vw, int vh, int vd, const R *v, R *p, double sigma);              \
    void orc_compute3d_##S(int w, int h, const R *depth, const R *invK9, const R *Rr9,           \
                           const R *t3, R *X, R *Y, R *Z);

ORC_DECL(float, f32)
ORC_DECL(double, f64)
#undef ORC_DECL

/* Bin centres of an N-bin fusion histogram (fusion.h:1041-1054). */
void orc_bin_centers(int bins, float *out);

/* Median of {bin centres, u, u + tau*lambda*W_j (j = 1..N)} exactly as the
 * reference's sortedHist insertion (structs.h:212-284) leaves it, including
 * its handling of values below the smallest element. */
float orc_prox_hist_f32(int bins, const uint16_t *h, float u, float tau, float lambda);

/* Depths of the reference's float plane loop (planesweep.cpp:169,200). */
int orc_plane_list(float znear, float zfar, int nplanes, float *out, int cap);

#ifdef __cplusplus
}
#endif
#endif
