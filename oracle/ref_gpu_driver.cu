/* Driver for the reference's own CUDA kernels on the GPU (oracle/_ref/libmvs_ref_gpu.so).
 *
 * REFERENCE-GPU TIMING AND TEST INFRASTRUCTURE ONLY.  Linked with the reference's
 * kernels.cu and TGV2_kernels.cu, compiled unchanged for sm_100a where they
 * lie in the reference tree (oracle/Makefile, target ref_gpu).  The functions
 * replay the call sequences of PlaneSweep::RunAlgorithm / PlaneSweepThread
 * (planesweep.cpp:74-259), PlaneSweep::TGV (planesweep.cpp:381-536) and
 * PlaneSweep::TGVdenoiseFromSparse (planesweep.cpp:596-674) on device images,
 * exactly as ref_driver.cpp replays them on host images for the CPU build:
 * the reference's wrappers, kernels and Matrix3D arithmetic,
 * one launch per wrapper call.  Buffers are allocated before the timed
 * region; buffers the reference leaves uninitialised are zero-filled.
 */
#include <kernels.cu.h>
#include <helper_structs.h>

#include <cuda_runtime.h>

#include <cstring>
#include <vector>

namespace {

struct Dev {
    float *p = nullptr;
    size_t n = 0;
    explicit Dev(size_t count, bool zero = true) : n(count)
    {
        cudaMalloc(&p, count * sizeof(float));
        if (zero) cudaMemset(p, 0, count * sizeof(float));
    }
    ~Dev() { cudaFree(p); }
    Dev(const Dev &) = delete;
    Dev &operator=(const Dev &) = delete;
};

Matrix3D mat(const float *m) { return Matrix3D(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]); }
Vector3D vec(const float *v) { return Vector3D(v[0], v[1], v[2]); }

/* PlaneSweep::RelativeMatrices, planesweep.cpp:538-549 */
void relative(Matrix3D &Rrel, Vector3D &trel, const Matrix3D &Rref, const Vector3D &tref, const Matrix3D &Rsrc,
              const Vector3D &tsrc, bool alternative)
{
    if (!alternative) {
        Rrel = Rsrc * Rref.inv();
        trel = tsrc - Rrel * tref;
    } else {
        Rrel = Rsrc.trans() * Rref;
        trel = Rsrc.trans() * (tref - tsrc);
    }
}

/* launch geometry of the reference (planesweep.cpp:70,100-101) */
struct Grid {
    dim3 blocks, threads;
    Grid(int w, int h) : threads(32, 32) { blocks = dim3((w + 31) / 32, (h + 31) / 32); }
};

}  // namespace

extern "C" {

/* RunAlgorithm + PlaneSweepThread on the GPU.  Returns the device time (ms)
 * of the compute (after the uploads, before the download), or a negative
 * value on a CUDA error; out_depth receives the depthmap. */
double ref_gpu_sweep(int w, int h, const float *ref, const float *srcs, int nsrc, const float *K9, const float *Rref9,
                     const float *tref3, const float *Rsrc9, const float *tsrc3, int alternative, const float *planes,
                     int nplanes, float znear, float zfar, int winsize, float stdthresh, float nccthresh,
                     float *out_depth)
{
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    Matrix3D K = mat(K9), invK = K.inv();
    Matrix3D Rref = mat(Rref9);
    Vector3D tref = vec(tref3);
    Dev dref(n, false), dsrcs(n * nsrc, false), refmean(n), refstd(n), inter(n), depthsum(n), count(n);
    Dev ncc(n), best(n), depth(n), i1(n), x(n), y(n), warped(n);
    cudaMemcpy(dref.p, ref, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dsrcs.p, srcs, n * nsrc * sizeof(float), cudaMemcpyHostToDevice);
    std::vector<float> dlist;
    if (planes) {
        dlist.assign(planes, planes + nplanes);
    } else {
        float dstep = (zfar - znear) / (nplanes - 1);
        for (float d = znear; d <= zfar; d += dstep) dlist.push_back(d);
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    windowed_mean_column(inter.p, dref.p, winsize, false, w, h, g.blocks, g.threads);
    windowed_mean_row(refmean.p, inter.p, winsize, false, w, h, g.blocks, g.threads);
    windowed_mean_column(inter.p, dref.p, winsize, true, w, h, g.blocks, g.threads);
    windowed_mean_row(refstd.p, inter.p, winsize, false, w, h, g.blocks, g.threads);
    calculate_STD(refstd.p, refmean.p, refstd.p, w, h, g.blocks, g.threads);
    for (int v = 0; v < nsrc; ++v) {
        const float *src = dsrcs.p + (size_t)v * n;
        cudaMemset(best.p, 0, n * sizeof(float));
        cudaMemset(depth.p, 0, n * sizeof(float));
        Matrix3D Rrel, tr;
        Vector3D trel;
        relative(Rrel, trel, Rref, tref, mat(Rsrc9 + 9 * v), vec(tsrc3 + 3 * v), alternative != 0);
        tr.row(2) = trel;
        tr = tr.trans();
        for (float d : dlist) {
            Matrix3D H = K * (Rrel + tr / d) * invK;
            H = H / H(2, 2);
            transform_indexes(x.p, y.p, H, w, h, g.blocks, g.threads);
            bilinear_interpolation(warped.p, src, x.p, y.p, w, h, w, h, g.blocks, g.threads);
            windowed_mean_column(i1.p, warped.p, winsize, false, w, h, g.blocks, g.threads);
            windowed_mean_row(x.p, i1.p, winsize, false, w, h, g.blocks, g.threads);
            windowed_mean_column(y.p, warped.p, winsize, true, w, h, g.blocks, g.threads);
            windowed_mean_row(i1.p, y.p, winsize, false, w, h, g.blocks, g.threads);
            calculate_STD(y.p, x.p, i1.p, w, h, g.blocks, g.threads);
            element_multiply(i1.p, dref.p, warped.p, w, h, g.blocks, g.threads);
            windowed_mean_column(warped.p, i1.p, winsize, false, w, h, g.blocks, g.threads);
            windowed_mean_row(i1.p, warped.p, winsize, false, w, h, g.blocks, g.threads);
            calcNCC(ncc.p, i1.p, refmean.p, x.p, refstd.p, y.p, stdthresh, stdthresh, w, h, g.blocks, g.threads);
            update_arrays(depth.p, best.p, ncc.p, d, w, h, g.blocks, g.threads);
        }
        sum_depthmap_NCC(depthsum.p, count.p, depth.p, best.p, nccthresh, w, h, g.blocks, g.threads);
    }
    element_rdivide(depthsum.p, depthsum.p, count.p, w, h, g.blocks, g.threads);
    set_QNAN_value(depthsum.p, zfar, w, h, g.blocks, g.threads);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaMemcpy(out_depth, depthsum.p, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    return ms;
}

/* PlaneSweep::TGV on the GPU (planesweep.cpp:381-536); u_init NULL starts
 * from u = 1 as the reference, else from the given depthmap.  Returns the
 * device time (ms) of the iterations, negative on a CUDA error. */
double ref_gpu_tgv(int w, int h, const float *refimg, const float *srcs, int nsrc, const float *K9,
                   const float *Rref9, const float *tref3, const float *Rsrc9, const float *tsrc3, int alternative,
                   int niters, int warps, double lambda, double alpha0, double alpha1, double tau, double sigma,
                   double beta, double gamma, const float *u_init, float *out_u)
{
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    const dim3 &B = g.blocks, &T = g.threads;
    Matrix3D K = mat(K9), invK = K.inv();
    Dev Ref(n, false), Px(n), Py(n), u(n), u0(n), u1x(n), u1y(n), ubar(n), u1xbar(n), u1ybar(n), qx(n), qy(n),
        qz(n), qw(n), prodsum(n), x(n), y(n), X(n), Y(n), Z(n), dX(n), dY(n), dZ(n), dfx(n), dfy(n), T1(n), T2(n),
        T3(n), T4(n);
    std::vector<Dev *> Src, It, Iu, r;
    for (int i = 0; i < nsrc; ++i) {
        Src.push_back(new Dev(n, false));
        It.push_back(new Dev(n));
        Iu.push_back(new Dev(n));
        r.push_back(new Dev(n));
    }
    cudaMemcpy(Ref.p, refimg, n * sizeof(float), cudaMemcpyHostToDevice);
    for (int i = 0; i < nsrc; ++i)
        cudaMemcpy(Src[i]->p, srcs + (size_t)i * n, n * sizeof(float), cudaMemcpyHostToDevice);
    if (u_init) cudaMemcpy(u.p, u_init, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaEvent_t ea, eb;
    cudaEventCreate(&ea);
    cudaEventCreate(&eb);
    cudaDeviceSynchronize();
    cudaEventRecord(ea);
    if (!u_init) set_value(u.p, 1.f, w, h, B, T);
    cudaMemcpy(ubar.p, u.p, n * sizeof(float), cudaMemcpyDeviceToDevice);
    element_scale(Ref.p, 1 / 255.f, w, h, B, T);
    Anisotropic_diffusion_tensor(T1.p, T2.p, T3.p, T4.p, Ref.p, beta, gamma, w, h, B, T);
    std::vector<Matrix3D> Rrel(nsrc);
    std::vector<Vector3D> Trel(nsrc);
    double fx = K(0, 0), fy = K(1, 1);
    for (int i = 0; i < nsrc; ++i) {
        element_scale(Src[i]->p, 1 / 255.f, w, h, B, T);
        relative(Rrel[i], Trel[i], mat(Rref9), vec(tref3), mat(Rsrc9 + 9 * i), vec(tsrc3 + 3 * i), alternative != 0);
    }
    for (int l = 0; l < warps; ++l) {
        cudaMemcpy(u0.p, u.p, n * sizeof(float), cudaMemcpyDeviceToDevice);
        cudaMemcpy(ubar.p, u.p, n * sizeof(float), cudaMemcpyDeviceToDevice);
        for (Dev *q : {&Px, &Py, &qx, &qy, &qz, &qw, &u1x, &u1y, &u1xbar, &u1ybar}) set_value(q->p, 0.f, w, h, B, T);
        for (int i = 0; i < nsrc; ++i) {
            TGV2_transform_coordinates(x.p, y.p, X.p, Y.p, Z.p, u0.p, K, Rrel[i], Trel[i], invK, w, h, B, T);
            TGV2_calculate_coordinate_derivatives(dX.p, dY.p, dZ.p, invK, Rrel[i], w, h, B, T);
            TGV2_calculate_derivativeF(dfx.p, dfy.p, X.p, dX.p, Y.p, dY.p, Z.p, dZ.p, fx, fy, w, h, B, T);
            bilinear_interpolation(X.p, Src[i]->p, x.p, y.p, w, h, w, h, B, T);
            TGV2_calculate_Iu(Iu[i]->p, X.p, dfx.p, dfy.p, w, h, B, T);
            subtract(It[i]->p, X.p, Ref.p, w, h, B, T);
            set_value(r[i]->p, 0.f, w, h, B, T);
        }
        for (int it = 0; it < niters; ++it) {
            TGV2_updateP_tensor_weighed(Px.p, Py.p, T1.p, T2.p, T3.p, T4.p, ubar.p, u1xbar.p, u1ybar.p, alpha1, sigma,
                                        w, h, B, T);
            TGV2_updateQ(qx.p, qy.p, qz.p, qw.p, u1xbar.p, u1ybar.p, alpha0, sigma, w, h, B, T);
            set_value(prodsum.p, 0.f, w, h, B, T);
            for (int j = 0; j < nsrc; ++j)
                TGV2_updateR(r[j]->p, prodsum.p, u.p, u0.p, It[j]->p, Iu[j]->p, sigma, lambda, w, h, B, T);
            TGV2_updateU_tensor_weighed(u.p, u1x.p, u1y.p, T1.p, T2.p, T3.p, T4.p, ubar.p, u1xbar.p, u1ybar.p, Px.p,
                                        Py.p, qx.p, qy.p, qz.p, qw.p, prodsum.p, alpha0, alpha1, tau, lambda, w, h, B,
                                        T);
        }
    }
    cudaEventRecord(eb);
    cudaEventSynchronize(eb);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ea, eb);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    cudaMemcpy(out_u, u.p, n * sizeof(float), cudaMemcpyDeviceToHost);
    for (int i = 0; i < nsrc; ++i) {
        delete Src[i];
        delete It[i];
        delete Iu[i];
        delete r[i];
    }
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    return ms;
}

/* PlaneSweep::TGVdenoiseFromSparse (planesweep.cpp:596-674) on the GPU:
 * weights, scaled sparse and start depth, the tensor, then niters x (P on u,
 * Q, the sparse tensor U step with vxbar / vybar passed as both v and its
 * over-relaxation), u * zfar.  Returns the device time (ms) from the first
 * kernel to the last, or a negative value on a CUDA error. */
double ref_gpu_tgv_sparse(int w, int h, const float *refimg, const float *depthmap, const float *sparse, float zfar,
                          int niters, double alpha0, double alpha1, double tau, double sigma, double theta,
                          double beta, double gamma, float *out)
{
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    const dim3 &B = g.blocks, &T = g.threads;
    Dev px(n), py(n), qx(n), qy(n), qz(n), qw(n), ubar(n), vxbar(n), vybar(n), weights(n), Ds(n), ref(n), T1(n),
        T2(n), T3(n), T4(n), u(n);
    cudaMemcpy(Ds.p, sparse, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(ubar.p, depthmap, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(ref.p, refimg, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaEvent_t ea, eb;
    cudaEventCreate(&ea);
    cudaEventCreate(&eb);
    cudaDeviceSynchronize();
    cudaEventRecord(ea);
    calculateWeights_sparseDepth(weights.p, Ds.p, w, h, B, T);
    element_scale(Ds.p, 1.f / zfar, w, h, B, T);
    element_scale(ubar.p, 1.f / zfar, w, h, B, T);
    cudaMemcpy(u.p, ubar.p, n * sizeof(float), cudaMemcpyDeviceToDevice);
    element_scale(ref.p, 1.f / 255.f, w, h, B, T);
    Anisotropic_diffusion_tensor(T1.p, T2.p, T3.p, T4.p, ref.p, beta, gamma, w, h, B, T);
    for (int i = 0; i < niters; ++i) {
        TGV2_updateP_tensor_weighed(px.p, py.p, T1.p, T2.p, T3.p, T4.p, u.p, vxbar.p, vybar.p, alpha1, sigma, w, h, B,
                                    T);
        TGV2_updateQ(qx.p, qy.p, qz.p, qw.p, vxbar.p, vybar.p, alpha0, sigma, w, h, B, T);
        TGV2_updateU_sparseDepthTensor(u.p, vxbar.p, vybar.p, ubar.p, vxbar.p, vybar.p, T1.p, T2.p, T3.p, T4.p, px.p,
                                       py.p, qx.p, qy.p, qz.p, qw.p, weights.p, Ds.p, alpha0, alpha1, tau, theta, w, h,
                                       B, T);
    }
    element_scale(u.p, zfar, w, h, B, T);
    cudaEventRecord(eb);
    cudaEventSynchronize(eb);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ea, eb);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    cudaMemcpy(out, u.p, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    return ms;
}

}  // extern "C"
