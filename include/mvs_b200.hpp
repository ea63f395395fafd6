/* libmvs_b200 -- C++ drop-in for the reference's plane-sweep API.
 *
 * The classes below keep the names, members and call signatures of the
 * reference's host API so that its callers (the GUI, pclviewer.cpp) compile
 * against them unchanged:
 *   Matrix3D, Vector3D        float 3x3 / 3-vector (structs.h:410-895,
 *                             helper_structs.h:159-291) with the same float
 *                             arithmetic (row-major rows, dot-product order,
 *                             cofactor inverse);
 *   CamImage<T>               host image with a world->camera pose R, t
 *                             (cam_image.h:8-57);
 *   PlaneSweep                planesweep.h:27-510;
 *   fusionData<N>, fusionvoxel<N>, histogram<N>, FusionUpdate*
 *                             fusion.h:105-1055, structs.h:44-189,
 *                             fusion.cu.h:40-173.
 * Behind them is the C ABI of include/mvs_b200.h.  Failures are reported as
 * the reference does: `false` from the bool methods, with the reason in
 * mvs_last_error(); the device is never reset.
 */
#ifndef MVS_B200_HPP
#define MVS_B200_HPP

#include <vector_types.h>   /* float3, int3, dim3 (plain C header of the CUDA toolkit) */

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <new>
#include <vector>

#include "mvs_b200.h"

typedef unsigned char uchar;

/* ---- small float vector / matrix types ------------------------------------ */

struct Vector3D {
    float x, y, z;
    Vector3D(float x_ = 0, float y_ = 0, float z_ = 0) : x(x_), y(y_), z(z_) {}
    Vector3D(const float v[3]) : x(v[0]), y(v[1]), z(v[2]) {}
    Vector3D(const double v[3]) : x((float)v[0]), y((float)v[1]), z((float)v[2]) {}
    Vector3D(float3 f) : x(f.x), y(f.y), z(f.z) {}
    operator float3() const { float3 f; f.x = x; f.y = y; f.z = z; return f; }
    float &operator()(unsigned char e) { return e == 2 ? z : (e == 1 ? y : x); }
    const float &operator()(unsigned char e) const { return e == 2 ? z : (e == 1 ? y : x); }
    float &at(unsigned char e) { return (*this)(e); }
    const float &at(unsigned char e) const { return (*this)(e); }
};

struct Matrix3D {
    float m[3][3]; /* m[row][col] */
    Matrix3D() { for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) m[r][c] = 0.f; }
    Matrix3D(float r11, float r12, float r13, float r21, float r22, float r23, float r31, float r32, float r33)
    {
        m[0][0] = r11; m[0][1] = r12; m[0][2] = r13;
        m[1][0] = r21; m[1][1] = r22; m[1][2] = r23;
        m[2][0] = r31; m[2][1] = r32; m[2][2] = r33;
    }
    Matrix3D(const float v[9]) { for (int k = 0; k < 9; ++k) m[k / 3][k % 3] = v[k]; }
    Matrix3D(const double v[9]) { for (int k = 0; k < 9; ++k) m[k / 3][k % 3] = (float)v[k]; }
    float &operator()(unsigned char r, unsigned char c) { return m[r][c]; }
    const float &operator()(unsigned char r, unsigned char c) const { return m[r][c]; }
    float &at(unsigned char r, unsigned char c) { return m[r][c]; }
    const float &at(unsigned char r, unsigned char c) const { return m[r][c]; }
    Vector3D row(unsigned char r) const { return Vector3D(m[r][0], m[r][1], m[r][2]); }
    void setRow(unsigned char r, const Vector3D &v) { m[r][0] = v.x; m[r][1] = v.y; m[r][2] = v.z; }
    Matrix3D trans() const
    {
        Matrix3D t;
        for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) t.m[r][c] = m[c][r];
        return t;
    }
    float det() const
    {
        return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    }
    /* cofactors divided by the determinant, as Matrix3D::inv (structs.h:584-593) */
    Matrix3D inv() const
    {
        const float d = det();
        return Matrix3D((m[1][1] * m[2][2] - m[1][2] * m[2][1]) / d, (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / d,
                        (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / d, (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / d,
                        (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / d, (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / d,
                        (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / d, (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / d,
                        (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / d);
    }
    void makeIdentity() { *this = Matrix3D(1, 0, 0, 0, 1, 0, 0, 0, 1); }
    static Matrix3D identityMatrix() { return Matrix3D(1, 0, 0, 0, 1, 0, 0, 0, 1); }
    void toArray(float out[9]) const { for (int k = 0; k < 9; ++k) out[k] = m[k / 3][k % 3]; }
};

inline float mvs_dot3(float a0, float a1, float a2, float b0, float b1, float b2) { return a0 * b0 + a1 * b1 + a2 * b2; }

inline Vector3D operator*(const Matrix3D &R, const Vector3D &v)
{
    return Vector3D(mvs_dot3(R.m[0][0], R.m[0][1], R.m[0][2], v.x, v.y, v.z),
                    mvs_dot3(R.m[1][0], R.m[1][1], R.m[1][2], v.x, v.y, v.z),
                    mvs_dot3(R.m[2][0], R.m[2][1], R.m[2][2], v.x, v.y, v.z));
}
inline Matrix3D operator*(const Matrix3D &A, const Matrix3D &B)
{
    Matrix3D C;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) C.m[r][c] = mvs_dot3(A.m[r][0], A.m[r][1], A.m[r][2], B.m[0][c], B.m[1][c], B.m[2][c]);
    return C;
}
inline Matrix3D operator*(const Matrix3D &A, float b)
{
    Matrix3D C;
    for (int k = 0; k < 9; ++k) C.m[k / 3][k % 3] = A.m[k / 3][k % 3] * b;
    return C;
}
inline Matrix3D operator*(float b, const Matrix3D &A) { return A * b; }
inline Matrix3D operator/(const Matrix3D &A, float b)
{
    Matrix3D C;
    for (int k = 0; k < 9; ++k) C.m[k / 3][k % 3] = A.m[k / 3][k % 3] / b;
    return C;
}
inline Matrix3D operator+(const Matrix3D &A, const Matrix3D &B)
{
    Matrix3D C;
    for (int k = 0; k < 9; ++k) C.m[k / 3][k % 3] = A.m[k / 3][k % 3] + B.m[k / 3][k % 3];
    return C;
}
inline Matrix3D operator-(const Matrix3D &A, const Matrix3D &B)
{
    Matrix3D C;
    for (int k = 0; k < 9; ++k) C.m[k / 3][k % 3] = A.m[k / 3][k % 3] - B.m[k / 3][k % 3];
    return C;
}
inline Vector3D operator+(const Vector3D &a, const Vector3D &b) { return Vector3D(a.x + b.x, a.y + b.y, a.z + b.z); }
inline Vector3D operator-(const Vector3D &a, const Vector3D &b) { return Vector3D(a.x - b.x, a.y - b.y, a.z - b.z); }

/* ---- images ------------------------------------------------------------------ */

/* Allocator of page-locked host memory (mvs_host_alloc): host images that the
 * library uploads or downloads then move at full PCIe / C2C speed. */
template <typename T>
struct PinnedAllocator {
    typedef T value_type;
    PinnedAllocator() {}
    template <typename U>
    PinnedAllocator(const PinnedAllocator<U> &) {}
    T *allocate(size_t n)
    {
        void *p = mvs_host_alloc(n * sizeof(T));
        if (!p) throw std::bad_alloc();
        return static_cast<T *>(p);
    }
    void deallocate(T *p, size_t) { mvs_host_free(p); }
    template <typename U>
    bool operator==(const PinnedAllocator<U> &) const { return true; }
    template <typename U>
    bool operator!=(const PinnedAllocator<U> &) const { return false; }
};

/* Host image, dense (pitch == width * sizeof(T)), with its world->camera pose.
 * reset() keeps the storage when the size does not change (the contents are
 * then the previous image's, as the reference's re-allocated images hold
 * whatever the allocator returns). */
template <typename T>
class CamImage {
public:
    Matrix3D R;
    Vector3D t;
    CamImage() : w_(0), h_(0) {}
    CamImage(size_t w, size_t h) : w_(w), h_(h), px_(w * h) {}
    void reset(size_t w, size_t h) { w_ = w; h_ = h; px_.resize(w * h); }
    T *data() { return px_.data(); }
    const T *data() const { return px_.data(); }
    size_t width() const { return w_; }
    size_t height() const { return h_; }
    size_t pitch() const { return w_ * sizeof(T); }
    size_t elements() const { return w_ * h_; }
    bool empty() const { return px_.empty(); }

private:
    size_t w_, h_;
    std::vector<T, PinnedAllocator<T>> px_;
};

/* ---- PlaneSweep ----------------------------------------------------------------- */

namespace mvs { struct PlaneSweepImpl; }

class PlaneSweep {
public:
    CamImage<float> HostRef;
    std::vector<CamImage<float>> HostSrc;
    CamImage<uchar> HostRef8u;
    std::vector<CamImage<uchar>> HostSrc8u;

    PlaneSweep();
    PlaneSweep(int argc, char **argv);
    ~PlaneSweep();
    PlaneSweep(const PlaneSweep &) = delete;
    PlaneSweep &operator=(const PlaneSweep &) = delete;

    bool RunAlgorithm(int argc, char **argv);
    /* OpenCV CPU denoise of the reference: not part of the GPU path; returns false. */
    bool Denoise(unsigned int niter, double lambda);
    bool CudaDenoise(int argc, char **argv, const unsigned int niters = 100, const double lambda = .3,
                     const double tau = 0.02, const double sigma = 6.f, const double theta = 1.f,
                     const double beta = 0.f, const double gamma = 1.f);
    bool TGV(int argc, char **argv, const unsigned int niters = 30, const unsigned int warps = 15,
             const double lambda = 0.5, const double alpha0 = 2.0, const double alpha1 = 1.5, const double tau = 0.02,
             const double sigma = 1.f, const double beta = 0.f, const double gamma = 1.f);
    /* TGV2 from the last sweep depthmap towards a sparse depthmap (0 = no
     * sample); the result is the TGV depthmap (planesweep.cpp:596-674). */
    bool TGVdenoiseFromSparse(int argc, char **argv, const CamImage<float> &depth, const unsigned int niters,
                              const double alpha0, const double alpha1, const double tau, const double sigma,
                              const double theta, const double beta, const double gamma);
    /* Extension: TGV2 from the last sweep depthmap (start = 1), a given
     * depthmap (start = 2) or 1 (start = 0), with an energy tolerance. */
    bool TGVext(const mvs_tgv2_params &p, int start, const CamImage<float> *init = 0, int *iters = 0,
                double *energy = 0);
    void RelativeMatrices(Matrix3D &Rrel, Vector3D &trel, const Matrix3D &Rref, const Vector3D &tref,
                          const Matrix3D &Rsrc, const Vector3D &tsrc) const;

    void setAlternativeRelativeMatrixMethod(bool method) { alternativemethod = method; }
    void setK(const Matrix3D &Km) { K = Km; invK = Km.inv(); }
    void setZ(float n, float f) { znear = n; zfar = f; }
    void setZnear(float n) { znear = n; }
    void setZfar(float f) { zfar = f; }
    void setNumberofPlanes(unsigned int n) { numberplanes = n; }
    void setNumberofImages(unsigned int n) { numberimages = n; }
    void setWindowSize(unsigned int sz);
    void setSTDthreshold(float th) { stdthresh = th; }
    void setNCCthreshold(float th) { nccthresh = th; }
    void setThreadsPerBlock(dim3 tpb) { threads = tpb; }
    void setBlockXdim(int &threadsx) { threads.x = threadsx; }
    void setBlockYdim(int &threadsy) { threads.y = threadsy; }
    /* extensions */
    void setPlaneDepths(const std::vector<float> &d) { planelist = d; }
    void setSweepOptions(int moments, int mode, bool fp64_homographies)
    {
        sweepmoments = moments;
        sweepmode = mode;
        fp64homography = fp64_homographies;
    }

    bool getAlternativeRelativeMatrixMethod() const { return alternativemethod; }
    Matrix3D getK() const { return K; }
    Matrix3D getInverseK() const { return invK; }
    CamImage<float> *getDepthmap() { return &depthmap; }
    CamImage<float> *getDepthmapDenoised() { return &depthmapdenoised; }
    float *getDepthmapDenoisedPtr();
    CamImage<uchar> *getDepthmap8u() { return &depthmap8u; }
    CamImage<uchar> *getDepthmap8uDenoised() { return &depthmap8udenoised; }
    CamImage<float> *getDepthmapTGV() { return &depthmapTGV; }
    CamImage<uchar> *getDepthmap8uTGV() { return &depthmap8uTGV; }
    void get3Dcoordinates(CamImage<float> *&x, CamImage<float> *&y, CamImage<float> *&z);
    float getZnear() const { return znear; }
    float getZfar() const { return zfar; }
    unsigned int getNumberofPlanes() const { return numberplanes; }
    unsigned int getNumberofImages() const { return numberimages; }
    unsigned int getWindowSize() const { return winsize; }
    float getSTDthreshold() const { return stdthresh; }
    float getNCCthreshold() const { return nccthresh; }
    unsigned int getMaxThreadsPerBlock() const { return 1024; }
    dim3 getThreadsPerBlock() const { return threads; }
    /* extensions */
    const std::vector<int32_t> &getViewLabels();
    const std::vector<float> &getViewBest();
    const std::vector<float> &getPlaneDepths() const { return lastplanes; }
    float getLastKernelMs() const { return lastms; }

protected:
    Matrix3D K, invK;
    CamImage<float> depthmap, depthmapdenoised, depthmapTGV;
    CamImage<uchar> depthmap8u, depthmap8udenoised, depthmap8uTGV;
    CamImage<float> coord_x, coord_y, coord_z;
    float znear = 0.1f, zfar = 1.0f;
    unsigned int numberplanes = 200, numberimages = 4, winsize = 5;
    float stdthresh = 0.0001f, nccthresh = 0.5f;
    dim3 threads;
    bool depthavailable = false, alternativemethod = false;
    std::vector<float> planelist, lastplanes;
    int sweepmoments = MVS_MOMENTS_REFERENCE, sweepmode = MVS_SWEEP_PER_VIEW;
    bool fp64homography = false;   /* reference-float homographies: bit-exact with the reference */
    std::vector<int32_t> viewlabels;
    std::vector<float> viewbest;
    float lastms = 0.f;
    mvs::PlaneSweepImpl *impl;
    /* the C-ABI image setters stage and upload the images in one pass */
    friend int ::mvs_ps_set_reference(mvs_planesweep *, const float *, int32_t, int32_t, const float *, const float *);
    friend int ::mvs_ps_set_sources(mvs_planesweep *, const float *, int32_t, const float *, const float *);

    void ConvertDepthtoUChar(const CamImage<float> &input, CamImage<uchar> &output);
    std::vector<float> planeDepths() const;
};

/* ---- fusion ------------------------------------------------------------------------ */

template <unsigned char N>
struct histogram {
    unsigned char bin[N];
    histogram() { for (unsigned char i = 0; i < N; ++i) bin[i] = 0; }
    unsigned char &first() { return bin[0]; }
    unsigned char &last() { return bin[N - 1]; }
    unsigned char &operator()(unsigned char i) { return bin[i]; }
};

/* Host-side voxel in the reference's AoS form (structs.h:131-189). */
template <unsigned char N>
struct fusionvoxel {
    float u;
    float v;
    float3 p;
    histogram<N> h;
};

struct Rectangle3D {
    float3 a, b;
    Rectangle3D() { a.x = a.y = a.z = b.x = b.y = b.z = 0.f; }
    Rectangle3D(float3 x, float3 y) : a(x), b(y) {}
    float3 size() const { float3 s; s.x = b.x - a.x; s.y = b.y - a.y; s.z = b.z - a.z; return s; }
};

enum MemoryKind { Standard, Host, Device };

/* Fusion volume on the device (structure of arrays behind an mvs_fusion
 * handle).  Copies share the handle without owning it, as the reference's
 * shallow copies (fusion.h:176-182). */
template <unsigned char N, MemoryKind memT = Device>
class fusionData {
public:
    fusionData() : f_(0), own_(false), w_(0), h_(0), d_(0) {}
    fusionData(size_t w, size_t h, size_t d) : fusionData(w, h, d, float3{0, 0, 0}, float3{0, 0, 0}) {}
    fusionData(size_t w, size_t h, size_t d, float3 a, float3 b) : f_(0), own_(true), w_(w), h_(h), d_(d), vol_(a, b)
    {
        const float fa[3] = {a.x, a.y, a.z}, fb[3] = {b.x, b.y, b.z};
        if (mvs_fusion_create((int)w, (int)h, (int)d, N, fa, fb, &f_) != MVS_OK) f_ = 0;
    }
    fusionData(size_t w, size_t h, size_t d, Rectangle3D &vol) : fusionData(w, h, d, vol.a, vol.b) {}
    fusionData(const fusionData &o) : f_(o.f_), own_(false), w_(o.w_), h_(o.h_), d_(o.d_), vol_(o.vol_) {}
    fusionData &operator=(const fusionData &o)
    {
        if (this == &o) return *this;
        if (own_) mvs_fusion_destroy(f_);
        f_ = o.f_;
        own_ = false;
        w_ = o.w_; h_ = o.h_; d_ = o.d_;
        vol_ = o.vol_;
        return *this;
    }
    ~fusionData() { if (own_) mvs_fusion_destroy(f_); }

    size_t width() const { return w_; }
    size_t height() const { return h_; }
    size_t depth() const { return d_; }
    size_t elements() const { return w_ * h_ * d_; }
    unsigned char bins() const { return N; }
    Rectangle3D volume() const { return vol_; }
    bool valid() const { return f_ != 0; }
    mvs_fusion *handle() const { return f_; }
    /* Resize (fusion.h:298-306): new storage of w x h x d voxels, managed by
     * this object from now on; the bounding volume is kept. */
    void Resize(size_t w, size_t h, size_t d)
    {
        if (own_) mvs_fusion_destroy(f_);
        f_ = 0;
        const float fa[3] = {vol_.a.x, vol_.a.y, vol_.a.z}, fb[3] = {vol_.b.x, vol_.b.y, vol_.b.z};
        if (mvs_fusion_create((int)w, (int)h, (int)d, N, fa, fb, &f_) != MVS_OK) f_ = 0;
        own_ = true;
        w_ = w; h_ = h; d_ = d;
    }
    void setVolume(Rectangle3D &vol)
    {
        vol_ = vol;
        const float fa[3] = {vol.a.x, vol.a.y, vol.a.z}, fb[3] = {vol.b.x, vol.b.y, vol.b.z};
        if (f_) mvs_fusion_set_volume(f_, fa, fb);
    }
    void setVolume(float3 x, float3 y) { Rectangle3D r(x, y); setVolume(r); }
    /* fusionData::worldCoords (fusion.h:360-364) */
    float3 worldCoords(int x, int y, int z) const
    {
        const float3 s = vol_.size();
        float3 c;
        c.x = vol_.a.x + s.x * (float)((x + .5) / w_);
        c.y = vol_.a.y + s.y * (float)((y + .5) / h_);
        c.z = vol_.a.z + s.z * (float)((z + .5) / d_);
        return c;
    }
    /* copyTo (fusion.h:933-947): the volume as AoS voxels in host memory,
     * npitch bytes per row (>= width * sizeof(fusionvoxel<N>)). */
    void copyTo(fusionvoxel<N> *data, size_t npitch)
    {
        const size_t n = elements();
        std::vector<float> u(n), v(n), p(3 * n);
        std::vector<uint16_t> hist((size_t)N * n);
        if (mvs_fusion_download(f_, u.data(), v.data(), p.data(), hist.data()) != MVS_OK) return;
        for (size_t z = 0; z < d_; ++z)
            for (size_t y = 0; y < h_; ++y) {
                fusionvoxel<N> *row = (fusionvoxel<N> *)((char *)data + (z * h_ + y) * npitch);
                for (size_t x = 0; x < w_; ++x) {
                    const size_t i = x + w_ * (y + h_ * z);
                    row[x].u = u[i];
                    row[x].v = v[i];
                    row[x].p.x = p[i];
                    row[x].p.y = p[n + i];
                    row[x].p.z = p[2 * n + i];
                    for (int k = 0; k < N; ++k) row[x].h.bin[k] = (unsigned char)hist[(size_t)k * n + i];
                }
            }
    }

private:
    mvs_fusion *f_;
    bool own_;
    size_t w_, h_, d_;
    Rectangle3D vol_;
};

/* FusionUpdate* (fusion.cu.h:40-173).  `blocks`/`threads` are accepted for
 * signature compatibility; the library chooses its own launch shape. */
template <unsigned char N>
inline void FusionUpdateHistogram(fusionData<N> f, const float *depthmap, const Matrix3D K, const Matrix3D R,
                                  const Vector3D t, const float threshold, const int width, const int height,
                                  dim3 = dim3(), dim3 = dim3())
{
    float k9[9], r9[9], t3[3] = {t.x, t.y, t.z};
    K.toArray(k9);
    R.toArray(r9);
    mvs_fusion_histogram(f.handle(), depthmap, 1, width, height, k9, r9, t3, threshold, 0);
}
template <unsigned char N>
inline void FusionUpdateU(fusionData<N> f, const double tau, const double lambda, dim3 = dim3(), dim3 = dim3())
{
    mvs_fusion_update_u(f.handle(), tau, lambda, 0);
}
template <unsigned char N>
inline void FusionUpdateP(fusionData<N> f, const double sigma, dim3 = dim3(), dim3 = dim3())
{
    mvs_fusion_update_p(f.handle(), sigma, 0);
}
template <unsigned char N>
inline void FusionUpdateIteration(fusionData<N> f, const float *depthmap, const Matrix3D K, const Matrix3D R,
                                  const Vector3D t, const float threshold, const double tau, const double lambda,
                                  const double sigma, const int width, const int height, dim3 = dim3(), dim3 = dim3())
{
    float k9[9], r9[9], t3[3] = {t.x, t.y, t.z};
    K.toArray(k9);
    R.toArray(r9);
    mvs_fusion_iteration(f.handle(), depthmap, width, height, k9, r9, t3, threshold, tau, lambda, sigma, 0);
}

#endif
