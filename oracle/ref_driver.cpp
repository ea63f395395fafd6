/* Driver for the reference's own kernels compiled for the CPU (oracle/_ref).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is linked with the reference's
 * kernels.cu, TGV2_kernels.cu and fusion.cu, compiled in place from the
 * reference tree by oracle/Makefile under oracle/ref_shim.h, into
 * oracle/_ref/libmvs_ref.so.  Only the tests, the fixture generator and the
 * CPU-baseline legs of bench.py load that library; the product never does.
 *
 * Each function below replays, call for call, the sequence of reference
 * wrapper calls that the reference's host code makes (planesweep.cpp and
 * pclviewer.cpp), on host buffers instead of device images.  The arithmetic
 * is the reference's own: the wrappers, kernels, Matrix3D/Vector3D operators
 * and fusionData members are the reference's code.  Device buffers that the
 * reference leaves uninitialised are zero-filled here (they are zero in
 * practice on a fresh allocation).
 */
#include <kernels.cu.h>
#include <helper_structs.h>
#include <fusion.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

/* fusion.h:192 (the fusionData destructor) calls CleanUp unqualified from a
 * dependent base, which g++ resolves only if some CleanUp is visible when the
 * destructor is instantiated.  Nothing in this driver ever owns voxel memory
 * (the `own` flag is always false), so this overload is never called. */
template <typename T>
static void CleanUp(T *) {}

thread_local uint3 shim_threadIdx;
thread_local uint3 shim_blockIdx;
dim3 shim_blockDim;
dim3 shim_gridDim;

/* Explicitly instantiated in the reference's fusion.cu (fusion.cu.h:235-272). */
template <unsigned char B>
void FusionUpdateHistogram(fusionData<B> f, const float *depthmap, const Matrix3D K, const Matrix3D R,
                           const Vector3D t, const float threshold, const int width, const int height,
                           dim3 blocks, dim3 threads);
template <unsigned char B>
void FusionUpdateU(fusionData<B> f, const double tau, const double lambda, dim3 blocks, dim3 threads);
template <unsigned char B>
void FusionUpdateP(fusionData<B> f, const double sigma, dim3 blocks, dim3 threads);

namespace {

using img = std::vector<float>;

Matrix3D mat(const float *m) { return Matrix3D(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8]); }
Vector3D vec(const float *v) { return Vector3D(v[0], v[1], v[2]); }

/* PlaneSweep::RelativeMatrices, planesweep.cpp:538-549 */
void relative(Matrix3D &Rrel, Vector3D &trel, const Matrix3D &Rref, const Vector3D &tref,
              const Matrix3D &Rsrc, const Vector3D &tsrc, bool alternative)
{
    if (!alternative) {
        Rrel = Rsrc * Rref.inv();
        trel = tsrc - Rrel * tref;
    } else {
        Rrel = Rsrc.trans() * Rref;
        trel = Rsrc.trans() * (tref - tsrc);
    }
}

/* Launch geometry of the reference: 32 x (maxThreadsPerBlock/32) threads,
 * blocks = ceil(w/tx) x ceil(h/ty) (planesweep.cpp:70,100-101).  The result
 * does not depend on the block shape (one thread per pixel, no sharing). */
struct Grid {
    dim3 blocks, threads;
    Grid(int w, int h) : threads(32, 32)
    {
        blocks = dim3((w + 31) / 32, (h + 31) / 32);
    }
};

double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

} // namespace

extern "C" {

/* PlaneSweep::RunAlgorithm + PlaneSweepThread (planesweep.cpp:74-161,163-259).
 *
 * K is the reference's 1-based calibration matrix; poses world->camera unless
 * `alternative`.  When `planes` is NULL the depth list is the reference's own
 * float loop `for (d = znear; d <= zfar; d += dstep)`; otherwise the given
 * list is swept in order.  Optional per-view outputs capture the per-view best
 * NCC and depth buffers (devbestNCC / devDepth) that the reference keeps
 * internally.  Returns the compute time in seconds. */
double ref_sweep(int w, int h, const float *ref, const float *srcs, int nsrc,
                 const float *K9, const float *Rref9, const float *tref3,
                 const float *Rsrc9, const float *tsrc3, int alternative,
                 const float *planes, int nplanes, float znear, float zfar,
                 int winsize, float stdthresh, float nccthresh,
                 float *out_depth, float *out_view_best, float *out_view_depth)
{
    const double t0 = now();
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    Matrix3D K = mat(K9), invK = K.inv();   /* setK, planesweep.h:179 */
    Matrix3D Rref = mat(Rref9);
    Vector3D tref = vec(tref3);

    img refmean(n, 0.f), refstd(n, 0.f), inter(n, 0.f);
    windowed_mean_column(inter.data(), ref, winsize, false, w, h, g.blocks, g.threads);
    windowed_mean_row(refmean.data(), inter.data(), winsize, false, w, h, g.blocks, g.threads);
    windowed_mean_column(inter.data(), ref, winsize, true, w, h, g.blocks, g.threads);
    windowed_mean_row(refstd.data(), inter.data(), winsize, false, w, h, g.blocks, g.threads);
    calculate_STD(refstd.data(), refmean.data(), refstd.data(), w, h, g.blocks, g.threads);

    img depthsum(n, 0.f), count(n, 0.f);
    std::vector<float> dlist;
    if (planes) {
        dlist.assign(planes, planes + nplanes);
    } else {
        float dstep = (zfar - znear) / (nplanes - 1);
        for (float d = znear; d <= zfar; d += dstep) dlist.push_back(d);
    }

    for (int v = 0; v < nsrc; ++v) {
        const float *src = srcs + (size_t)v * n;
        img ncc(n, 0.f), best(n, 0.f), depth(n, 0.f), i1(n, 0.f), x(n, 0.f), y(n, 0.f), warped(n, 0.f);
        Matrix3D Rrel, tr;
        Vector3D trel;
        relative(Rrel, trel, Rref, tref, mat(Rsrc9 + 9 * v), vec(tsrc3 + 3 * v), alternative != 0);
        tr.row(2) = trel;
        tr = tr.trans();
        for (float d : dlist) {
            Matrix3D H = K * (Rrel + tr / d) * invK;
            H = H / H(2, 2);
            transform_indexes(x.data(), y.data(), H, w, h, g.blocks, g.threads);
            bilinear_interpolation(warped.data(), src, x.data(), y.data(), w, h, w, h, g.blocks, g.threads);
            windowed_mean_column(i1.data(), warped.data(), winsize, false, w, h, g.blocks, g.threads);
            windowed_mean_row(x.data(), i1.data(), winsize, false, w, h, g.blocks, g.threads);
            windowed_mean_column(y.data(), warped.data(), winsize, true, w, h, g.blocks, g.threads);
            windowed_mean_row(i1.data(), y.data(), winsize, false, w, h, g.blocks, g.threads);
            calculate_STD(y.data(), x.data(), i1.data(), w, h, g.blocks, g.threads);
            element_multiply(i1.data(), ref, warped.data(), w, h, g.blocks, g.threads);
            windowed_mean_column(warped.data(), i1.data(), winsize, false, w, h, g.blocks, g.threads);
            windowed_mean_row(i1.data(), warped.data(), winsize, false, w, h, g.blocks, g.threads);
            calcNCC(ncc.data(), i1.data(), refmean.data(), x.data(), refstd.data(), y.data(),
                    stdthresh, stdthresh, w, h, g.blocks, g.threads);
            update_arrays(depth.data(), best.data(), ncc.data(), d, w, h, g.blocks, g.threads);
        }
        sum_depthmap_NCC(depthsum.data(), count.data(), depth.data(), best.data(), nccthresh, w, h,
                         g.blocks, g.threads);
        if (out_view_best) std::memcpy(out_view_best + (size_t)v * n, best.data(), n * sizeof(float));
        if (out_view_depth) std::memcpy(out_view_depth + (size_t)v * n, depth.data(), n * sizeof(float));
    }
    element_rdivide(depthsum.data(), depthsum.data(), count.data(), w, h, g.blocks, g.threads);
    set_QNAN_value(depthsum.data(), zfar, w, h, g.blocks, g.threads);
    std::memcpy(out_depth, depthsum.data(), n * sizeof(float));
    return now() - t0;
}

/* The reference's plane list for (znear, zfar, nplanes); returns its length. */
int ref_plane_list(float znear, float zfar, int nplanes, float *out, int cap)
{
    float dstep = (zfar - znear) / (nplanes - 1);
    int k = 0;
    for (float d = znear; d <= zfar; d += dstep) {
        if (k < cap) out[k] = d;
        ++k;
    }
    return k;
}

/* Homography of one plane exactly as PlaneSweepThread builds it
 * (planesweep.cpp:195-203), for checking the product's homographies. */
void ref_homography(const float *K9, const float *Rref9, const float *tref3, const float *Rsrc9,
                    const float *tsrc3, int alternative, float d, float *H9)
{
    Matrix3D K = mat(K9), invK = K.inv(), Rrel, tr;
    Vector3D trel;
    relative(Rrel, trel, mat(Rref9), vec(tref3), mat(Rsrc9), vec(tsrc3), alternative != 0);
    tr.row(2) = trel;
    tr = tr.trans();
    Matrix3D H = K * (Rrel + tr / d) * invK;
    H = H / H(2, 2);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) H9[3 * r + c] = H(r, c);
}

/* PlaneSweep::TGV (planesweep.cpp:381-536).  `u_init` NULL gives the
 * reference's constant u = 1 start (planesweep.cpp:414); otherwise the given
 * depthmap is the start (the same kernels, started from a sweep result). */
double ref_tgv(int w, int h, const float *refimg, const float *srcs, int nsrc,
               const float *K9, const float *Rref9, const float *tref3,
               const float *Rsrc9, const float *tsrc3, int alternative,
               int niters, int warps, double lambda, double alpha0, double alpha1,
               double tau, double sigma, double beta, double gamma,
               const float *u_init, float *out_u)
{
    const double t0 = now();
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    const dim3 &B = g.blocks, &T = g.threads;
    Matrix3D K = mat(K9), invK = K.inv();
    img Ref(n), Px(n, 0.f), Py(n, 0.f), u(n, 0.f), u0(n, 0.f), u1x(n, 0.f), u1y(n, 0.f), ubar(n, 0.f),
        u1xbar(n, 0.f), u1ybar(n, 0.f), qx(n, 0.f), qy(n, 0.f), qz(n, 0.f), qw(n, 0.f), prodsum(n, 0.f),
        x(n, 0.f), y(n, 0.f), X(n, 0.f), Y(n, 0.f), Z(n, 0.f), dX(n, 0.f), dY(n, 0.f), dZ(n, 0.f),
        dfx(n, 0.f), dfy(n, 0.f), T1(n, 0.f), T2(n, 0.f), T3(n, 0.f), T4(n, 0.f);
    std::vector<img> Src(nsrc, img(n)), It(nsrc, img(n, 0.f)), Iu(nsrc, img(n, 0.f)), r(nsrc, img(n, 0.f));

    if (u_init) std::memcpy(u.data(), u_init, n * sizeof(float));
    else set_value(u.data(), 1.f, w, h, B, T);
    ubar = u;
    std::memcpy(Ref.data(), refimg, n * sizeof(float));
    element_scale(Ref.data(), 1 / 255.f, w, h, B, T);
    Anisotropic_diffusion_tensor(T1.data(), T2.data(), T3.data(), T4.data(), Ref.data(), beta, gamma, w, h, B, T);

    std::vector<Matrix3D> Rrel(nsrc);
    std::vector<Vector3D> Trel(nsrc);
    double fx = K(0, 0), fy = K(1, 1);
    for (int i = 0; i < nsrc; ++i) {
        std::memcpy(Src[i].data(), srcs + (size_t)i * n, n * sizeof(float));
        element_scale(Src[i].data(), 1 / 255.f, w, h, B, T);
        relative(Rrel[i], Trel[i], mat(Rref9), vec(tref3), mat(Rsrc9 + 9 * i), vec(tsrc3 + 3 * i),
                 alternative != 0);
    }
    for (int l = 0; l < warps; ++l) {
        u0 = u;
        ubar = u;
        set_value(Px.data(), 0.f, w, h, B, T);
        set_value(Py.data(), 0.f, w, h, B, T);
        set_value(qx.data(), 0.f, w, h, B, T);
        set_value(qy.data(), 0.f, w, h, B, T);
        set_value(qz.data(), 0.f, w, h, B, T);
        set_value(qw.data(), 0.f, w, h, B, T);
        set_value(u1x.data(), 0.f, w, h, B, T);
        set_value(u1y.data(), 0.f, w, h, B, T);
        set_value(u1xbar.data(), 0.f, w, h, B, T);
        set_value(u1ybar.data(), 0.f, w, h, B, T);
        for (int i = 0; i < nsrc; ++i) {
            TGV2_transform_coordinates(x.data(), y.data(), X.data(), Y.data(), Z.data(), u0.data(), K, Rrel[i],
                                       Trel[i], invK, w, h, B, T);
            TGV2_calculate_coordinate_derivatives(dX.data(), dY.data(), dZ.data(), invK, Rrel[i], w, h, B, T);
            TGV2_calculate_derivativeF(dfx.data(), dfy.data(), X.data(), dX.data(), Y.data(), dY.data(), Z.data(),
                                       dZ.data(), fx, fy, w, h, B, T);
            bilinear_interpolation(X.data(), Src[i].data(), x.data(), y.data(), w, h, w, h, B, T);
            TGV2_calculate_Iu(Iu[i].data(), X.data(), dfx.data(), dfy.data(), w, h, B, T);
            subtract(It[i].data(), X.data(), Ref.data(), w, h, B, T);
            set_value(r[i].data(), 0.f, w, h, B, T);
        }
        for (int it = 0; it < niters; ++it) {
            TGV2_updateP_tensor_weighed(Px.data(), Py.data(), T1.data(), T2.data(), T3.data(), T4.data(),
                                        ubar.data(), u1xbar.data(), u1ybar.data(), alpha1, sigma, w, h, B, T);
            TGV2_updateQ(qx.data(), qy.data(), qz.data(), qw.data(), u1xbar.data(), u1ybar.data(), alpha0, sigma,
                         w, h, B, T);
            set_value(prodsum.data(), 0.f, w, h, B, T);
            for (int j = 0; j < nsrc; ++j)
                TGV2_updateR(r[j].data(), prodsum.data(), u.data(), u0.data(), It[j].data(), Iu[j].data(), sigma,
                             lambda, w, h, B, T);
            TGV2_updateU_tensor_weighed(u.data(), u1x.data(), u1y.data(), T1.data(), T2.data(), T3.data(),
                                        T4.data(), ubar.data(), u1xbar.data(), u1ybar.data(), Px.data(), Py.data(),
                                        qx.data(), qy.data(), qz.data(), qw.data(), prodsum.data(), alpha0,
                                        alpha1, tau, lambda, w, h, B, T);
        }
    }
    std::memcpy(out_u, u.data(), n * sizeof(float));
    return now() - t0;
}

/* PlaneSweep::TGVdenoiseFromSparse (planesweep.cpp:596-674): TGV2 of the
 * sweep's depthmap towards a sparse depth (weight 1 where the sparse depth is
 * positive), both divided by zfar.  The call at planesweep.cpp:645 hands the
 * update kernel vxbar / vybar as both v and its over-relaxation, and the P
 * step reads u itself (d_depthmap) rather than ubar: replayed as written. */
double ref_tgv_sparse(int w, int h, const float *refimg, const float *depthmap, const float *sparse, float zfar,
                      int niters, double alpha0, double alpha1, double tau, double sigma, double theta, double beta,
                      double gamma, float *out)
{
    const double t0 = now();
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    const dim3 &B = g.blocks, &T = g.threads;
    img px(n, 0.f), py(n, 0.f), qx(n, 0.f), qy(n, 0.f), qz(n, 0.f), qw(n, 0.f), ubar(depthmap, depthmap + n),
        vxbar(n, 0.f), vybar(n, 0.f), weights(n, 0.f), Ds(sparse, sparse + n), ref(refimg, refimg + n), T1(n, 0.f),
        T2(n, 0.f), T3(n, 0.f), T4(n, 0.f);
    calculateWeights_sparseDepth(weights.data(), Ds.data(), w, h, B, T);
    element_scale(Ds.data(), 1.f / zfar, w, h, B, T);
    element_scale(ubar.data(), 1.f / zfar, w, h, B, T);
    img u(ubar);   /* d_depthmap = ubar */
    element_scale(ref.data(), 1.f / 255.f, w, h, B, T);
    Anisotropic_diffusion_tensor(T1.data(), T2.data(), T3.data(), T4.data(), ref.data(), beta, gamma, w, h, B, T);
    for (int i = 0; i < niters; i++) {
        TGV2_updateP_tensor_weighed(px.data(), py.data(), T1.data(), T2.data(), T3.data(), T4.data(), u.data(),
                                    vxbar.data(), vybar.data(), alpha1, sigma, w, h, B, T);
        TGV2_updateQ(qx.data(), qy.data(), qz.data(), qw.data(), vxbar.data(), vybar.data(), alpha0, sigma, w, h, B,
                     T);
        TGV2_updateU_sparseDepthTensor(u.data(), vxbar.data(), vybar.data(), ubar.data(), vxbar.data(), vybar.data(),
                                       T1.data(), T2.data(), T3.data(), T4.data(), px.data(), py.data(), qx.data(),
                                       qy.data(), qz.data(), qw.data(), weights.data(), Ds.data(), alpha0, alpha1, tau,
                                       theta, w, h, B, T);
    }
    element_scale(u.data(), zfar, w, h, B, T);
    std::memcpy(out, u.data(), n * sizeof(float));
    return now() - t0;
}

/* PlaneSweep::CudaDenoise (planesweep.cpp:297-379): TV-L1 with the tensor
 * weighted dual step, on a depthmap normalised to [0,1] over [znear, zfar]. */
double ref_tvl1_denoise(int w, int h, const float *refimg, const float *depth, float znear, float zfar,
                        int niters, double lambda, double tau, double sigma, double theta, double beta,
                        double gamma, float *out)
{
    const double t0 = now();
    const size_t n = (size_t)w * h;
    Grid g(w, h);
    const dim3 &B = g.blocks, &T = g.threads;
    img d(depth, depth + n), R(n, 0.f), Px(n, 0.f), Py(n, 0.f), raw(depth, depth + n), T11(n, 0.f),
        T12(n, 0.f), T21(n, 0.f), T22(n, 0.f), ref(refimg, refimg + n);
    element_scale(ref.data(), 1 / 255.f, w, h, B, T);
    Anisotropic_diffusion_tensor(T11.data(), T12.data(), T21.data(), T22.data(), ref.data(), beta, gamma, w, h, B,
                                 T);
    element_add(d.data(), -znear, w, h, B, T);
    element_add(raw.data(), -znear, w, h, B, T);
    double xscale = 1.f / (zfar - znear);
    double inputscale = -sigma / (zfar - znear);
    element_scale(d.data(), xscale, w, h, B, T);
    element_scale(raw.data(), inputscale, w, h, B, T);
    for (int i = 0; i < niters; ++i) {
        double currsigma = i == 0 ? 1 + sigma : sigma;
        denoising_TVL1_calculateP_tensor_weighed(Px.data(), Py.data(), T11.data(), T12.data(), T21.data(),
                                                 T22.data(), d.data(), currsigma, w, h, B, T);
        denoising_TVL1_update(d.data(), R.data(), Px.data(), Py.data(), raw.data(), tau, theta, lambda, sigma, w,
                              h, B, T);
    }
    element_scale(d.data(), (zfar - znear), w, h, B, T);
    element_add(d.data(), znear, w, h, B, T);
    std::memcpy(out, d.data(), n * sizeof(float));
    return now() - t0;
}

/* compute3D (kernels.cu:405-429) as get3Dcoordinates drives it
 * (planesweep.cpp:551-586): reference camera -> world coordinates. */
void ref_compute3d(int w, int h, const float *depth, const float *K9, const float *Rref9, const float *tref3,
                   int alternative, float *X, float *Y, float *Z)
{
    Grid g(w, h);
    Matrix3D K = mat(K9), invK = K.inv(), Rr, I;
    Vector3D t, T0(0, 0, 0);
    I.makeIdentity();
    relative(Rr, t, mat(Rref9), vec(tref3), I, T0, alternative != 0);
    const size_t n = (size_t)w * h;
    std::memcpy(Z, depth, n * sizeof(float));
    compute3D(X, Y, Z, Rr, t, invK, w, h, g.blocks, g.threads);
}

} // extern "C"

/* ---- fusion (fusion.cu, fusion.h) ------------------------------------- */

struct RefFusion {
    int bins, w, h, d;
    float a[3], b[3];
    std::vector<unsigned char> store;   /* fusionvoxel<bins> array, dense */
    size_t voxel_bytes;
};

/* A fusionData whose settings point at RefFusion's dense voxel store.  The
 * settings are written through a derived class because fusionData keeps them
 * protected; the object never owns the store. */
template <unsigned char B>
struct FusionView : public fusionData<B> {
    explicit FusionView(const fusionDataSettings<B> &s) { this->stg = s; }
};

template <unsigned char B>
static fusionData<B> view(RefFusion *f)
{
    fusionData<B> base;
    base.setManageData(false);
    fusionDataSettings<B> s = base.exportSettings();
    s.width = f->w;
    s.height = f->h;
    s.depth = f->d;
    s.pitch = f->w * sizeof(fusionvoxel<B>);
    s.spitch = s.pitch * f->h;
    s.own = false;
    s.ptr = reinterpret_cast<fusionvoxel<B> *>(f->store.data());
    s.volume = Rectangle3D(make_float3(f->a[0], f->a[1], f->a[2]), make_float3(f->b[0], f->b[1], f->b[2]));
    FusionView<B> v(s);
    return fusionData<B>(v);
}

static void fusion_grid(RefFusion *f, dim3 &blocks, dim3 &threads)
{
    /* pclviewer.cpp:1000-1007 with the default 16 x 16 x 1 threads */
    threads = dim3(16, 16, 1);
    blocks = dim3((f->w + 15) / 16, (f->h + 15) / 16, f->d);
}

#define REF_BINS(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

extern "C" void *ref_fusion_create(int bins, int w, int h, int d, const float *a, const float *b)
{
    if (bins < 2 || bins > 10) return nullptr;
    RefFusion *f = new RefFusion{bins, w, h, d, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {}, 0};
    switch (bins) {
#define SZ(N) case N: f->voxel_bytes = sizeof(fusionvoxel<N>); break;
        REF_BINS(SZ)
#undef SZ
    }
    f->store.assign((size_t)w * h * d * f->voxel_bytes, 0);
    return f;
}

extern "C" void ref_fusion_destroy(void *p) { delete static_cast<RefFusion *>(p); }

extern "C" size_t ref_fusion_voxel_bytes(void *p) { return static_cast<RefFusion *>(p)->voxel_bytes; }

extern "C" double ref_fusion_histogram(void *p, const float *depth, int w, int h, const float *K9, const float *R9,
                            const float *t3, float threshold)
{
    const double t0 = now();
    RefFusion *f = static_cast<RefFusion *>(p);
    dim3 blocks, threads;
    fusion_grid(f, blocks, threads);
    switch (f->bins) {
#define H(N) case N: FusionUpdateHistogram<N>(view<N>(f), depth, mat(K9), mat(R9), vec(t3), threshold, w, h, \
                                              blocks, threads); break;
        REF_BINS(H)
#undef H
    }
    return now() - t0;
}

extern "C" double ref_fusion_u(void *p, double tau, double lambda)
{
    const double t0 = now();
    RefFusion *f = static_cast<RefFusion *>(p);
    dim3 blocks, threads;
    fusion_grid(f, blocks, threads);
    switch (f->bins) {
#define U(N) case N: FusionUpdateU<N>(view<N>(f), tau, lambda, blocks, threads); break;
        REF_BINS(U)
#undef U
    }
    return now() - t0;
}

extern "C" double ref_fusion_p(void *p, double sigma)
{
    const double t0 = now();
    RefFusion *f = static_cast<RefFusion *>(p);
    dim3 blocks, threads;
    fusion_grid(f, blocks, threads);
    switch (f->bins) {
#define P(N) case N: FusionUpdateP<N>(view<N>(f), sigma, blocks, threads); break;
        REF_BINS(P)
#undef P
    }
    return now() - t0;
}

/* Copy the AoS voxels out as SoA: u, v, p (3 planes), hist (bins planes). */
template <unsigned char B>
static void get_soa(RefFusion *f, float *u, float *v, float *p, uint16_t *hist)
{
    const size_t n = (size_t)f->w * f->h * f->d;
    const fusionvoxel<B> *vx = reinterpret_cast<const fusionvoxel<B> *>(f->store.data());
    for (size_t i = 0; i < n; ++i) {
        if (u) u[i] = vx[i].u;
        if (v) v[i] = vx[i].v;
        if (p) { p[i] = vx[i].p.x; p[n + i] = vx[i].p.y; p[2 * n + i] = vx[i].p.z; }
        if (hist) for (int k = 0; k < B; ++k) hist[k * n + i] = vx[i].h.bin[k];
    }
}

template <unsigned char B>
static void set_soa(RefFusion *f, const float *u, const float *v, const float *p, const uint16_t *hist)
{
    const size_t n = (size_t)f->w * f->h * f->d;
    fusionvoxel<B> *vx = reinterpret_cast<fusionvoxel<B> *>(f->store.data());
    for (size_t i = 0; i < n; ++i) {
        if (u) vx[i].u = u[i];
        if (v) vx[i].v = v[i];
        if (p) vx[i].p = make_float3(p[i], p[n + i], p[2 * n + i]);
        if (hist) for (int k = 0; k < B; ++k) vx[i].h.bin[k] = (unsigned char)hist[k * n + i];
    }
}

extern "C" void ref_fusion_get(void *p, float *u, float *v, float *pp, uint16_t *hist)
{
    RefFusion *f = static_cast<RefFusion *>(p);
    switch (f->bins) {
#define G(N) case N: get_soa<N>(f, u, v, pp, hist); break;
        REF_BINS(G)
#undef G
    }
}

extern "C" void ref_fusion_set(void *p, const float *u, const float *v, const float *pp, const uint16_t *hist)
{
    RefFusion *f = static_cast<RefFusion *>(p);
    switch (f->bins) {
#define S(N) case N: set_soa<N>(f, u, v, pp, hist); break;
        REF_BINS(S)
#undef S
    }
}

/* The reference's bin centres (fusion.h:1041-1054). */
extern "C" void ref_fusion_bin_centers(int bins, float *out)
{
    switch (bins) {
#define C(N) case N: { fusionData<N> fd; fd.setManageData(false); \
                        for (int i = 0; i < N; ++i) out[i] = fd.binCenter(i); } break;
        REF_BINS(C)
#undef C
    }
}


