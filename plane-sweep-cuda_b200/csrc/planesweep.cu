// PlaneSweep (planesweep.h:27-510 of the reference) on top of the C ABI, and
// the mvs_ps_* handle functions that expose it to C callers.
//
// Host-side arithmetic that feeds the kernels (K^-1, RelativeMatrices, the
// float homographies of the reference path, the plane list, the 8-bit
// conversion) is done in float exactly as the reference does it on the
// host; device buffers are kept across calls and only grow.
#include <math.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/mvs_b200.hpp"
#include "common.cuh"

#if defined(__x86_64__) && !defined(__CUDA_ARCH__)
#include <emmintrin.h>
#define MVS_STREAM_STORES 1
#endif

namespace mvs {

// Device buffer that only grows.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int ensure(size_t need)
    {
        if (need <= bytes) return MVS_OK;
        cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (need == 0) return MVS_OK;
        cudaError_t e = cudaMalloc(&p, need);
        if (e != cudaSuccess) return set_error(MVS_ERR_NOMEM, "cudaMalloc(%zu): %s", need, cudaGetErrorString(e));
        bytes = need;
        return MVS_OK;
    }
    template <typename T>
    T *as() const { return (T *)p; }
    ~DevBuf() { cudaFree(p); }
};

// Host copies of whole images into the page-locked buffers of the handle.
// The stores are non-temporal (straight to memory, not into the CPU caches):
// the copy engine that uploads the images next then reads them from DRAM,
// whereas lines left dirty in the cores' caches made that upload about
// 0.8 ms slower for the 11 MB of a 640x480, 8-view frame.  Copies of a few
// MB are split over up to 8 threads (each piece at least 1 MiB).
void stream_copy(void *dst, const void *src, size_t bytes)
{
#ifdef MVS_STREAM_STORES
    char *d = (char *)dst;
    const char *s = (const char *)src;
    size_t head = (16 - ((uintptr_t)d & 15)) & 15;
    if (head > bytes) head = bytes;
    memcpy(d, s, head);
    d += head;
    s += head;
    bytes -= head;
    const size_t blocks = bytes / 64;
    for (size_t i = 0; i < blocks; ++i, d += 64, s += 64) {
        const __m128i a = _mm_loadu_si128((const __m128i *)s), b = _mm_loadu_si128((const __m128i *)(s + 16)),
                      c = _mm_loadu_si128((const __m128i *)(s + 32)), e = _mm_loadu_si128((const __m128i *)(s + 48));
        _mm_stream_si128((__m128i *)d, a);
        _mm_stream_si128((__m128i *)(d + 16), b);
        _mm_stream_si128((__m128i *)(d + 32), c);
        _mm_stream_si128((__m128i *)(d + 48), e);
    }
    memcpy(d, s, bytes - blocks * 64);
    _mm_sfence();
#else
    memcpy(dst, src, bytes);
#endif
}

struct CopyPiece {
    void *dst;
    const void *src;
    size_t bytes;
    void *dev = nullptr;   // if set: dst is page-locked and is uploaded here as it fills
};

// Upload granule: a thread stages this many bytes, then queues their
// upload on the stream, so the copy engine starts after the first MB
// instead of after the whole frame (256 KB granules made the 8 staging
// threads wait on each other in the driver: 44 calls for an 11 MB frame).
constexpr size_t kUploadChunk = (size_t)1 << 20;

// Worker threads for parallel_copy, made on first use and kept for the
// process (spawning seven threads for every frame cost more than the copies
// they shared).  A job is fn(0 .. parts-1): the caller and the workers claim
// parts from one counter, and the caller returns once every worker has
// checked in for that job, so none still holds it.  The pool is never
// destroyed (its workers wait on it until the process ends).  A process
// forked after the pool was made has none of its threads, so it does not use
// it.
class CopyPool {
public:
    static CopyPool *get()
    {
        static CopyPool *pool = new CopyPool(std::min(7u, std::max(1u, std::thread::hardware_concurrency()) - 1));
        return pool;
    }
    int workers() const { return nworkers_; }
    // false if another caller holds the pool (that caller's job is not
    // shared), or in a process forked after the pool was made
    bool try_run(int parts, const std::function<void(int)> &fn)
    {
        if (getpid() != owner_) return false;
        std::unique_lock<std::mutex> busy(busy_, std::try_to_lock);
        if (!busy.owns_lock()) return false;
        {
            std::lock_guard<std::mutex> lk(mu_);
            fn_ = &fn;
            parts_ = parts;
            next_.store(0);
            pending_ = nworkers_;
            ++gen_;
        }
        work_.notify_all();
        for (int k; (k = next_.fetch_add(1)) < parts;) fn(k);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return pending_ == 0; });
        fn_ = nullptr;
        return true;
    }

private:
    explicit CopyPool(int n) : nworkers_(n), owner_(getpid())
    {
        for (int k = 0; k < n; ++k) std::thread([this] { loop(); }).detach();
    }
    void loop()
    {
        unsigned long long seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            work_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            const std::function<void(int)> *fn = fn_;
            const int parts = parts_;
            lk.unlock();
            for (int k; (k = next_.fetch_add(1)) < parts;) (*fn)(k);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    const int nworkers_;
    const pid_t owner_;
    std::mutex busy_, mu_;
    std::condition_variable work_, done_;
    const std::function<void(int)> *fn_ = nullptr;
    int parts_ = 0, pending_ = 0;
    unsigned long long gen_ = 0;
    std::atomic<int> next_{0};
};

// Returns 0, or the first CUDA error of a queued upload.
int parallel_copy(const std::vector<CopyPiece> &pieces, cudaStream_t st = 0)
{
    size_t total = 0;
    for (const CopyPiece &c : pieces) total += c.bytes;
    // a part of at least 256 KB: a 640x480 float image is shared by four threads
    const size_t min_part = (size_t)1 << 18;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int parts = (int)std::min<size_t>(std::min(8u, hw), std::max<size_t>(1, total / min_part));
    std::atomic<int> err{0};
    // uploads queued from other threads go to the caller's device (a thread
    // starts on device 0), so stream 0 there is the caller's stream 0
    int dev = 0;
    cudaGetDevice(&dev);
    const std::thread::id caller = std::this_thread::get_id();
    auto run = [&](int k) {
        if (std::this_thread::get_id() != caller) cudaSetDevice(dev);
        // part k copies bytes [k * total / parts, (k + 1) * total / parts) of the concatenation
        const size_t lo = total * k / parts, hi = total * (k + 1) / parts;
        size_t base = 0;
        for (const CopyPiece &c : pieces) {
            const size_t a = std::max(lo, base), b = std::min(hi, base + c.bytes);
            for (size_t x = a; x < b;) {
                const size_t e = c.dev ? std::min(b, x + kUploadChunk) : b;
                stream_copy((char *)c.dst + (x - base), (const char *)c.src + (x - base), e - x);
                // the non-temporal stores are fenced inside stream_copy, so the
                // bytes are in memory before the copy engine reads them
                if (c.dev) {
                    const cudaError_t ce = cudaMemcpyAsync((char *)c.dev + (x - base), (const char *)c.dst + (x - base),
                                                           e - x, cudaMemcpyHostToDevice, st);
                    if (ce != cudaSuccess) err.store((int)ce);
                }
                x = e;
            }
            base += c.bytes;
        }
    };
    if (parts <= 1) {
        run(0);
        return err.load();
    }
    const std::function<void(int)> job = run;
    if (CopyPool *pool = CopyPool::get(); pool->workers() >= parts - 1 && pool->try_run(parts, job)) return err.load();
    std::vector<std::thread> th;
    th.reserve(parts - 1);
    for (int k = 1; k < parts; ++k) th.emplace_back(run, k);
    run(0);
    for (std::thread &t : th) t.join();
    return err.load();
}

// True when the host range [p, p + bytes) starts and ends in page-locked
// memory (cudaHostAlloc'd or registered), which the copy engine reads
// directly: then one copy of the whole range beats staging it.
bool page_locked(const void *p, size_t bytes)
{
    for (const void *q : {p, (const void *)((const char *)p + bytes - 1)}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();   // not a pointer the runtime knows: pageable
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

// A caller's page-locked images: one upload of the whole range from the
// caller's memory on stream 0, while the pool threads copy the same bytes
// into the handle's host images (`pieces`, concatenated in order, nothing
// uploaded from them).  Returns once both are done, so the caller may reuse
// its memory; true if the upload was made (else the images stay on the host
// for RunAlgorithm).
bool direct_upload(void *dev, const void *src, size_t bytes, const std::vector<CopyPiece> &pieces, cudaEvent_t done)
{
    const bool up = cudaMemcpyAsync(dev, src, bytes, cudaMemcpyHostToDevice, 0) == cudaSuccess;
    parallel_copy(pieces, 0);
    const bool ok = up && cudaEventRecord(done, 0) == cudaSuccess && cudaEventSynchronize(done) == cudaSuccess;
    if (!ok) cudaGetLastError();
    return ok;
}

// ConvertDepthtoUChar (planesweep.cpp:279-290) per pixel, for the sweep
// result while it is still on the device: the same float division, clamp
// and truncation, so the bytes equal the host conversion's.
__global__ void depth_to_u8_kernel(const float *__restrict__ d, size_t n, float znear, float zfar,
                                   uint8_t *__restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = d[i];
        const float x = (v - znear) / (zfar - znear);
        float c = x < 0.f ? 0.f : x;   // std::max(x, 0.f), then std::min(c, 1.f)
        c = 1.f < c ? 1.f : c;
        out[i] = v == v ? (uint8_t)(UCHAR_MAX * c) : UCHAR_MAX;
    }
}

struct PlaneSweepImpl {
    DevBuf ref, srcs, H, depths, depth, depth8, labels, best, ws, denoised, tvws, tvu, cx, cy, cz, tvsrc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int n_views = 0, n_planes = 0, w = 0, h = 0;
    // Images that the C-ABI setters (the only writers of the host images of a
    // handle) uploaded while staging them: RunAlgorithm then uploads neither.
    // `uploaded[0]` marks the end of the reference image's copies and
    // `uploaded[1]` that of the sources': each host image is not rewritten or
    // freed before its own event (so the sources are staged while the
    // reference is still on its way).
    bool ref_dev = false;
    int srcs_dev = 0, dev_w = 0, dev_h = 0;
    cudaEvent_t uploaded[2] = {nullptr, nullptr};
    // the plane depths on the device (RunAlgorithm uploads them when they change)
    std::vector<float> dev_planes;
    PlaneSweepImpl()
    {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (cudaEvent_t &e : uploaded)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) e = nullptr;
    }
    bool can_upload() const { return uploaded[0] && uploaded[1]; }
    ~PlaneSweepImpl()
    {
        for (cudaEvent_t e : uploaded)
            if (e) {
                cudaEventSynchronize(e);
                cudaEventDestroy(e);
            }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

}  // namespace mvs

using mvs::PlaneSweepImpl;

PlaneSweep::PlaneSweep() : threads(32, 32), impl(new PlaneSweepImpl) {}
PlaneSweep::PlaneSweep(int, char **) : threads(32, 32), impl(new PlaneSweepImpl) {}
PlaneSweep::~PlaneSweep() { delete impl; }

void PlaneSweep::setWindowSize(unsigned int sz)
{
    // odd sizes only (planesweep.h:234); even sizes are ignored
    if (sz % 2 == 0) mvs::set_error(MVS_ERR_ARG, "Window size must be an odd number");
    else winsize = sz;
}

bool PlaneSweep::Denoise(unsigned int, double)
{
    mvs::set_error(MVS_ERR_NOTBUILT, "Denoise is the reference's OpenCV CPU path; use CudaDenoise");
    return false;
}

void PlaneSweep::RelativeMatrices(Matrix3D &Rrel, Vector3D &trel, const Matrix3D &Rref, const Vector3D &tref,
                                  const Matrix3D &Rsrc, const Vector3D &tsrc) const
{
    // planesweep.cpp:538-549
    if (!alternativemethod) {
        Rrel = Rsrc * Rref.inv();
        trel = tsrc - Rrel * tref;
    } else {
        Rrel = Rsrc.trans() * Rref;
        trel = Rsrc.trans() * (tref - tsrc);
    }
}

std::vector<float> PlaneSweep::planeDepths() const
{
    if (!planelist.empty()) return planelist;
    // PlaneSweepThread's float loop (planesweep.cpp:169,200)
    std::vector<float> out;
    if (numberplanes < 2) {
        out.push_back(znear);
        return out;
    }
    const float dstep = (zfar - znear) / (numberplanes - 1);
    for (float d = znear; d <= zfar; d += dstep) {
        out.push_back(d);
        if (out.size() > 1u << 20) break;
    }
    return out;
}

void PlaneSweep::ConvertDepthtoUChar(const CamImage<float> &input, CamImage<uchar> &output)
{
    // planesweep.cpp:279-290
    output.reset(input.width(), input.height());
    for (size_t i = 0; i < input.elements(); ++i) {
        const float v = input.data()[i];
        if (v == v)
            output.data()[i] = uchar(UCHAR_MAX * std::min(std::max((v - znear) / (zfar - znear), 0.f), 1.f));
        else
            output.data()[i] = UCHAR_MAX;
    }
}

bool PlaneSweep::RunAlgorithm(int, char **)
{
    PlaneSweepImpl &I = *impl;
    const int w = (int)HostRef.width(), h = (int)HostRef.height();
    depthmap.reset(w, h);
    depthavailable = false;
    if (w == 0 || h == 0 || HostSrc.empty()) {
        mvs::set_error(MVS_ERR_STATE, "reference or source images missing");
        return false;
    }
    const int nimgs = std::min(std::max((int)numberimages, 1), (int)HostSrc.size());
    for (int v = 0; v < nimgs; ++v)
        if ((int)HostSrc[v].width() != w || (int)HostSrc[v].height() != h) {
            mvs::set_error(MVS_ERR_ARG, "source %d is %zux%zu, reference %dx%d", v, HostSrc[v].width(),
                           HostSrc[v].height(), w, h);
            return false;
        }
    const std::vector<float> planes = planeDepths();
    const int P = (int)planes.size();
    const size_t n = (size_t)w * h;
    mvs_sweep_desc d;
    d.width = w;
    d.height = h;
    d.n_views = nimgs;
    d.n_planes = P;
    d.window = (int)winsize;
    d.moments = sweepmoments;
    d.mode = sweepmode;
    d.std_threshold = stdthresh;
    d.ncc_threshold = nccthresh;
    d.zfar = zfar;
    const size_t wsb = mvs_sweep_workspace_bytes(&d);
    if (wsb == 0) return false;
    const size_t lab_n = sweepmode == MVS_SWEEP_PER_VIEW ? n * nimgs : n;
    // images the C-ABI setters uploaded already (buffers that do not grow keep them)
    const bool ref_up = I.ref_dev && I.dev_w == w && I.dev_h == h && I.ref.bytes >= n * 4;
    const bool srcs_up = I.srcs_dev >= nimgs && I.dev_w == w && I.dev_h == h && I.srcs.bytes >= n * 4 * nimgs;
    if (I.ref.ensure(n * 4) || I.srcs.ensure(n * 4 * nimgs) || I.H.ensure((size_t)nimgs * P * 9 * 4) ||
        I.depths.ensure((size_t)P * 4) || I.depth.ensure(n * 4) || I.labels.ensure(lab_n * 4) ||
        I.best.ensure(lab_n * 4) || I.ws.ensure(wsb) || I.depth8.ensure(n))
        return false;
    depthmap8u.reset(w, h);
    cudaStream_t st = 0;
    if (!ref_up && cudaMemcpyAsync(I.ref.p, HostRef.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        goto cuda_fail;
    for (int v = 0; v < nimgs && !srcs_up; ++v)
        if (cudaMemcpyAsync(I.srcs.as<float>() + v * n, HostSrc[v].data(), n * 4, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
            goto cuda_fail;
    // a pageable copy may wait for the uploads queued before it: only when the
    // planes change (the buffer grows only for more planes, which differ)
    if (planes != I.dev_planes) {
        I.dev_planes.clear();
        if (cudaMemcpyAsync(I.depths.p, planes.data(), (size_t)P * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
            goto cuda_fail;
        I.dev_planes = planes;
    }
    {
        cudaEventRecord(I.e0, st);
        if (fp64homography) {
            std::vector<double> Rrel(9 * (size_t)nimgs), trel(3 * (size_t)nimgs);
            double K9[9];
            for (int k = 0; k < 9; ++k) K9[k] = K(k / 3, k % 3);
            for (int v = 0; v < nimgs; ++v) {
                // RelativeMatrices in double from the float poses
                double Rr[9], tr[3], Rs[9], ts[3];
                for (int k = 0; k < 9; ++k) {
                    Rr[k] = HostRef.R(k / 3, k % 3);
                    Rs[k] = HostSrc[v].R(k / 3, k % 3);
                }
                for (int k = 0; k < 3; ++k) {
                    tr[k] = HostRef.t(k);
                    ts[k] = HostSrc[v].t(k);
                }
                double *Ro = &Rrel[9 * v], *to = &trel[3 * v];
                if (!alternativemethod) {
                    // Rsrc * Rref^-1 with the exact inverse (adjugate / det)
                    const double *m = Rr;
                    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                                       m[2] * (m[3] * m[7] - m[4] * m[6]);
                    const double inv[9] = {(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det,
                                           (m[1] * m[5] - m[2] * m[4]) / det, (m[5] * m[6] - m[3] * m[8]) / det,
                                           (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                                           (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det,
                                           (m[0] * m[4] - m[1] * m[3]) / det};
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c)
                            Ro[3 * r + c] = Rs[3 * r] * inv[c] + Rs[3 * r + 1] * inv[3 + c] + Rs[3 * r + 2] * inv[6 + c];
                    for (int r = 0; r < 3; ++r)
                        to[r] = ts[r] - (Ro[3 * r] * tr[0] + Ro[3 * r + 1] * tr[1] + Ro[3 * r + 2] * tr[2]);
                } else {
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c)
                            Ro[3 * r + c] = Rs[r] * Rr[c] + Rs[3 + r] * Rr[3 + c] + Rs[6 + r] * Rr[6 + c];
                    const double dt[3] = {tr[0] - ts[0], tr[1] - ts[1], tr[2] - ts[2]};
                    for (int r = 0; r < 3; ++r) to[r] = Rs[r] * dt[0] + Rs[3 + r] * dt[1] + Rs[6 + r] * dt[2];
                }
            }
            if (mvs_sweep_homographies(&d, K9, Rrel.data(), trel.data(), I.depths.as<float>(), I.H.as<float>(), st))
                return false;
        } else {
            // the reference's float homographies (planesweep.cpp:195-203)
            std::vector<float> Hh(9 * (size_t)nimgs * P);
            for (int v = 0; v < nimgs; ++v) {
                Matrix3D Rrel, tr;
                Vector3D trel;
                RelativeMatrices(Rrel, trel, HostRef.R, HostRef.t, HostSrc[v].R, HostSrc[v].t);
                tr.setRow(2, trel);
                tr = tr.trans();
                for (int p = 0; p < P; ++p) {
                    Matrix3D Hm = K * (Rrel + tr / planes[p]) * invK;
                    Hm = Hm / Hm(2, 2);
                    Hm.toArray(&Hh[9 * ((size_t)v * P + p)]);
                }
            }
            if (cudaMemcpyAsync(I.H.p, Hh.data(), Hh.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
                goto cuda_fail;
        }
        if (mvs_sweep(&d, I.ref.as<float>(), I.srcs.as<float>(), I.H.as<float>(), I.depths.as<float>(),
                      I.depth.as<float>(), I.labels.as<int32_t>(), I.best.as<float>(), nullptr, I.ws.p, I.ws.bytes, st))
            return false;
        cudaEventRecord(I.e1, st);
        mvs::depth_to_u8_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 4 * 148), 256, 0, st>>>(
            I.depth.as<float>(), n, znear, zfar, I.depth8.as<uint8_t>());
    }
    if (cudaMemcpyAsync(depthmap.data(), I.depth.p, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) goto cuda_fail;
    if (cudaMemcpyAsync(depthmap8u.data(), I.depth8.p, n, cudaMemcpyDeviceToHost, st) != cudaSuccess) goto cuda_fail;
    if (cudaStreamSynchronize(st) != cudaSuccess) goto cuda_fail;
    cudaEventElapsedTime(&lastms, I.e0, I.e1);
    I.n_views = nimgs;
    I.n_planes = P;
    I.w = w;
    I.h = h;
    lastplanes = planes;
    viewlabels.clear();
    viewbest.clear();
    depthavailable = true;
    return true;
cuda_fail:
    mvs::set_error(MVS_ERR_CUDA, "RunAlgorithm: %s", cudaGetErrorString(cudaGetLastError()));
    return false;
}

// The per-view results are copied back on the first request after a sweep.  A
// failed copy leaves the vector empty (nothing stale is cached) with the CUDA
// error as the last error message.
const std::vector<int32_t> &PlaneSweep::getViewLabels()
{
    PlaneSweepImpl &I = *impl;
    if (viewlabels.empty() && depthavailable) {
        const size_t m = (size_t)I.w * I.h * (sweepmode == MVS_SWEEP_PER_VIEW ? I.n_views : 1);
        viewlabels.resize(m);
        const cudaError_t e = cudaMemcpy(viewlabels.data(), I.labels.p, m * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            viewlabels.clear();
            mvs::set_error(MVS_ERR_CUDA, "getViewLabels: %s", cudaGetErrorString(e));
        }
    }
    return viewlabels;
}

const std::vector<float> &PlaneSweep::getViewBest()
{
    PlaneSweepImpl &I = *impl;
    if (viewbest.empty() && depthavailable) {
        const size_t m = (size_t)I.w * I.h * (sweepmode == MVS_SWEEP_PER_VIEW ? I.n_views : 1);
        viewbest.resize(m);
        const cudaError_t e = cudaMemcpy(viewbest.data(), I.best.p, m * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            viewbest.clear();
            mvs::set_error(MVS_ERR_CUDA, "getViewBest: %s", cudaGetErrorString(e));
        }
    }
    return viewbest;
}

float *PlaneSweep::getDepthmapDenoisedPtr() { return impl->denoised.as<float>(); }

bool PlaneSweep::CudaDenoise(int, char **, const unsigned int niters, const double lambda, const double tau,
                             const double sigma, const double theta, const double beta, const double gamma)
{
    PlaneSweepImpl &I = *impl;
    if (!depthavailable) {
        mvs::set_error(MVS_ERR_STATE, "CudaDenoise needs a depthmap from RunAlgorithm");
        return false;
    }
    const int w = (int)depthmap.width(), h = (int)depthmap.height();
    const size_t n = (size_t)w * h;
    if (I.denoised.ensure(n * 4) || I.tvws.ensure(mvs_tvl1_workspace_bytes(w, h)) || I.ref.ensure(n * 4)) return false;
    depthmapdenoised.reset(w, h);
    depthmap8udenoised.reset(w, h);
    cudaStream_t st = 0;
    mvs_tvl1_params p;
    p.niters = (int)niters;
    p.lambda = lambda;
    p.tau = tau;
    p.sigma = sigma;
    p.theta = theta;
    p.beta = beta;
    p.gamma = gamma;
    if (cudaMemcpyAsync(I.ref.p, HostRef.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(I.denoised.p, depthmap.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        mvs::set_error(MVS_ERR_CUDA, "CudaDenoise copy: %s", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    cudaEventRecord(I.e0, st);
    if (mvs_tvl1_denoise(w, h, I.ref.as<float>(), I.denoised.as<float>(), znear, zfar, &p, I.tvws.p, I.tvws.bytes, st))
        return false;
    cudaEventRecord(I.e1, st);
    if (cudaMemcpyAsync(depthmapdenoised.data(), I.denoised.p, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        mvs::set_error(MVS_ERR_CUDA, "CudaDenoise: %s", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    cudaEventElapsedTime(&lastms, I.e0, I.e1);
    ConvertDepthtoUChar(depthmapdenoised, depthmap8udenoised);
    return true;
}

bool PlaneSweep::TGVext(const mvs_tgv2_params &prm, int start, const CamImage<float> *init, int *iters, double *energy)
{
    PlaneSweepImpl &I = *impl;
    const int w = (int)HostRef.width(), h = (int)HostRef.height();
    const size_t n = (size_t)w * h;
    if (w == 0 || HostSrc.empty()) {
        mvs::set_error(MVS_ERR_STATE, "reference or source images missing");
        return false;
    }
    if (start == 1 && !depthavailable) {
        mvs::set_error(MVS_ERR_STATE, "TGV from the sweep needs a depthmap from RunAlgorithm");
        return false;
    }
    if (start == 2 && (!init || (int)init->width() != w || (int)init->height() != h)) {
        mvs::set_error(MVS_ERR_ARG, "TGV start depthmap missing or of the wrong size");
        return false;
    }
    const int nimgs = std::min(std::max((int)numberimages, 1), (int)HostSrc.size());
    depthmapTGV.reset(w, h);
    depthmap8uTGV.reset(w, h);
    if (I.ref.ensure(n * 4) || I.tvsrc.ensure(n * 4 * nimgs) || I.tvu.ensure(n * 4) ||
        I.tvws.ensure(std::max(mvs_tgv2_workspace_bytes(w, h, nimgs), mvs_tvl1_workspace_bytes(w, h))))
        return false;
    cudaStream_t st = 0;
    bool ok = cudaMemcpyAsync(I.ref.p, HostRef.data(), n * 4, cudaMemcpyHostToDevice, st) == cudaSuccess;
    for (int v = 0; ok && v < nimgs; ++v)
        ok = cudaMemcpyAsync(I.tvsrc.as<float>() + v * n, HostSrc[v].data(), n * 4, cudaMemcpyHostToDevice, st) ==
             cudaSuccess;
    if (ok && start == 1) ok = cudaMemcpyAsync(I.tvu.p, I.depth.p, n * 4, cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    if (ok && start == 2) ok = cudaMemcpyAsync(I.tvu.p, init->data(), n * 4, cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (!ok) {
        mvs::set_error(MVS_ERR_CUDA, "TGV copy: %s", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    std::vector<float> Rrel(9 * (size_t)nimgs), trel(3 * (size_t)nimgs);
    for (int v = 0; v < nimgs; ++v) {
        Matrix3D R;
        Vector3D t;
        RelativeMatrices(R, t, HostRef.R, HostRef.t, HostSrc[v].R, HostSrc[v].t);
        R.toArray(&Rrel[9 * v]);
        trel[3 * v] = t.x;
        trel[3 * v + 1] = t.y;
        trel[3 * v + 2] = t.z;
    }
    float K9[9], iK9[9];
    K.toArray(K9);
    invK.toArray(iK9);
    int it = 0;
    double e = 0;
    cudaEventRecord(I.e0, st);
    if (mvs_tgv2_run(w, h, nimgs, I.ref.as<float>(), I.tvsrc.as<float>(), K9, iK9, Rrel.data(), trel.data(), &prm,
                     start != 0, 1.f, I.tvu.as<float>(), &it, &e, I.tvws.p, I.tvws.bytes, st))
        return false;
    cudaEventRecord(I.e1, st);
    if (cudaMemcpyAsync(depthmapTGV.data(), I.tvu.p, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        mvs::set_error(MVS_ERR_CUDA, "TGV: %s", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    cudaEventElapsedTime(&lastms, I.e0, I.e1);
    if (iters) *iters = it;
    if (energy) *energy = e;
    ConvertDepthtoUChar(depthmapTGV, depthmap8uTGV);
    return true;
}

bool PlaneSweep::TGVdenoiseFromSparse(int, char **, const CamImage<float> &depth, const unsigned int niters,
                                      const double alpha0, const double alpha1, const double tau, const double sigma,
                                      const double theta, const double beta, const double gamma)
{
    PlaneSweepImpl &I = *impl;
    const int w = (int)HostRef.width(), h = (int)HostRef.height();
    const size_t n = (size_t)w * h;
    if (!depthavailable || (int)depthmap.width() != w || (int)depthmap.height() != h) {
        mvs::set_error(MVS_ERR_STATE, "TGVdenoiseFromSparse needs a depthmap from RunAlgorithm");
        return false;
    }
    if ((int)depth.width() != w || (int)depth.height() != h) {
        mvs::set_error(MVS_ERR_ARG, "sparse depthmap of the wrong size");
        return false;
    }
    depthmapTGV.reset(w, h);
    depthmap8uTGV.reset(w, h);
    if (I.ref.ensure(n * 4) || I.tvu.ensure(n * 4) || I.tvsrc.ensure(n * 4) ||
        I.tvws.ensure(std::max(mvs_tgv2_sparse_workspace_bytes(w, h), mvs_tvl1_workspace_bytes(w, h))))
        return false;
    cudaStream_t st = 0;
    if (cudaMemcpyAsync(I.ref.p, HostRef.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(I.tvsrc.p, depth.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        mvs::set_error(MVS_ERR_CUDA, "TGVdenoiseFromSparse copy: %s", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    cudaEventRecord(I.e0, st);
    if (mvs_tgv2_sparse(w, h, I.ref.as<float>(), I.depth.as<float>(), I.tvsrc.as<float>(), zfar, (int)niters, alpha0,
                        alpha1, tau, sigma, theta, beta, gamma, I.tvu.as<float>(), I.tvws.p, I.tvws.bytes, st))
        return false;
    cudaEventRecord(I.e1, st);
    if (cudaMemcpyAsync(depthmapTGV.data(), I.tvu.p, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        mvs::set_error(MVS_ERR_CUDA, "TGVdenoiseFromSparse: %s", cudaGetErrorString(cudaGetLastError()));
        return false;
    }
    cudaEventElapsedTime(&lastms, I.e0, I.e1);
    ConvertDepthtoUChar(depthmapTGV, depthmap8uTGV);
    return true;
}

bool PlaneSweep::TGV(int, char **, const unsigned int niters, const unsigned int warps, const double lambda,
                     const double alpha0, const double alpha1, const double tau, const double sigma, const double beta,
                     const double gamma)
{
    mvs_tgv2_params p;
    memset(&p, 0, sizeof(p));
    p.niters = (int)niters;
    p.warps = (int)warps;
    p.lambda = lambda;
    p.alpha0 = alpha0;
    p.alpha1 = alpha1;
    p.tau = tau;
    p.sigma = sigma;
    p.beta = beta;
    p.gamma = gamma;
    return TGVext(p, 0);
}

void PlaneSweep::get3Dcoordinates(CamImage<float> *&x, CamImage<float> *&y, CamImage<float> *&z)
{
    // planesweep.cpp:551-586: reference camera -> world, on the denoised depthmap
    PlaneSweepImpl &I = *impl;
    const int w = (int)HostRef.width(), h = (int)HostRef.height();
    const size_t n = (size_t)w * h;
    x = y = z = nullptr;
    if ((int)depthmapdenoised.width() != w || (int)depthmapdenoised.height() != h || n == 0) {
        mvs::set_error(MVS_ERR_STATE, "get3Dcoordinates needs a CudaDenoise result");
        return;
    }
    Matrix3D Rr, Id;
    Vector3D t, T0(0, 0, 0);
    Id.makeIdentity();
    RelativeMatrices(Rr, t, HostRef.R, HostRef.t, Id, T0);
    if (I.cx.ensure(n * 4) || I.cy.ensure(n * 4) || I.cz.ensure(n * 4)) return;
    cudaMemset(I.cx.p, 0, n * 4);
    cudaMemset(I.cy.p, 0, n * 4);
    if (cudaMemcpy(I.cz.p, depthmapdenoised.data(), n * 4, cudaMemcpyHostToDevice) != cudaSuccess) return;
    float ik[9], R9[9], t3[3] = {t.x, t.y, t.z};
    invK.toArray(ik);
    Rr.toArray(R9);
    if (mvs_compute3d(w, h, I.cz.as<float>(), ik, R9, t3, I.cx.as<float>(), I.cy.as<float>(), I.cz.as<float>(), 0))
        return;
    coord_x.reset(w, h);
    coord_y.reset(w, h);
    coord_z.reset(w, h);
    cudaMemcpy(coord_x.data(), I.cx.p, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(coord_y.data(), I.cy.p, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(coord_z.data(), I.cz.p, n * 4, cudaMemcpyDeviceToHost);
    x = &coord_x;
    y = &coord_y;
    z = &coord_z;
}

// ---- C handle ------------------------------------------------------------------------

struct mvs_planesweep {
    PlaneSweep ps;
};

#define PS_CHECK(ps)                                                      \
    do {                                                                  \
        if (!(ps)) return mvs::set_error(MVS_ERR_ARG, "null PlaneSweep"); \
    } while (0)

extern "C" {

int mvs_ps_create(mvs_planesweep **out)
{
    if (!out) return mvs::set_error(MVS_ERR_ARG, "null output");
    *out = new (std::nothrow) mvs_planesweep;
    return *out ? MVS_OK : mvs::set_error(MVS_ERR_NOMEM, "host allocation failed");
}

int mvs_ps_destroy(mvs_planesweep *ps)
{
    delete ps;
    return MVS_OK;
}

int mvs_ps_set_reference(mvs_planesweep *ps, const float *img, int32_t w, int32_t h, const float *R9, const float *t3)
{
    PS_CHECK(ps);
    if (!img || w <= 0 || h <= 0 || !R9 || !t3) return mvs::set_error(MVS_ERR_ARG, "bad reference image");
    PlaneSweepImpl &I = *ps->ps.impl;
    // the previous uploads still read the host images (no event: no device,
    // the images stay on the host for RunAlgorithm)
    if (I.uploaded[0]) cudaEventSynchronize(I.uploaded[0]);
    const size_t bytes = sizeof(float) * (size_t)w * h;
    ps->ps.HostRef.reset(w, h);
    ps->ps.HostRef.R = Matrix3D(R9);
    ps->ps.HostRef.t = Vector3D(t3);
    I.ref_dev = false;
    if (w != I.dev_w || h != I.dev_h) I.srcs_dev = 0;
    // staged and uploaded together (RunAlgorithm's stream), or uploaded from
    // the caller's page-locked image while it is copied; a failed upload
    // leaves the image to RunAlgorithm
    const bool up = I.can_upload() && I.ref.ensure(bytes) == MVS_OK;
    if (up && mvs::page_locked(img, bytes)) {
        if (mvs::direct_upload(I.ref.p, img, bytes, {{ps->ps.HostRef.data(), img, bytes}}, I.uploaded[0])) {
            I.ref_dev = true;
            I.dev_w = w;
            I.dev_h = h;
        }
        return MVS_OK;
    }
    const int rc = mvs::parallel_copy({{ps->ps.HostRef.data(), img, bytes, up ? I.ref.p : nullptr}}, 0);
    if (up && rc == 0 && cudaEventRecord(I.uploaded[0], 0) == cudaSuccess) {
        I.ref_dev = true;
        I.dev_w = w;
        I.dev_h = h;
    }
    return MVS_OK;
}

int mvs_ps_set_sources(mvs_planesweep *ps, const float *imgs, int32_t n, const float *R9s, const float *t3s)
{
    PS_CHECK(ps);
    const int w = (int)ps->ps.HostRef.width(), h = (int)ps->ps.HostRef.height();
    if (w == 0) return mvs::set_error(MVS_ERR_STATE, "set the reference image first");
    if (n < 0 || (n > 0 && (!imgs || !R9s || !t3s))) return mvs::set_error(MVS_ERR_ARG, "bad source images");
    PlaneSweepImpl &I = *ps->ps.impl;
    if (I.uploaded[1]) cudaEventSynchronize(I.uploaded[1]);
    const size_t bytes = sizeof(float) * (size_t)w * h;
    I.srcs_dev = 0;
    const bool up = I.can_upload() && n > 0 && I.srcs.ensure(bytes * n) == MVS_OK;
    ps->ps.HostSrc.resize(n);
    const bool direct = up && mvs::page_locked(imgs, bytes * n);
    std::vector<mvs::CopyPiece> pieces;
    for (int v = 0; v < n; ++v) {
        ps->ps.HostSrc[v].reset(w, h);
        pieces.push_back({ps->ps.HostSrc[v].data(), imgs + (size_t)v * w * h, bytes,
                          up && !direct ? (void *)(I.srcs.as<char>() + bytes * v) : nullptr});
        ps->ps.HostSrc[v].R = Matrix3D(R9s + 9 * v);
        ps->ps.HostSrc[v].t = Vector3D(t3s + 3 * v);
    }
    if (direct) {
        if (mvs::direct_upload(I.srcs.p, imgs, bytes * n, pieces, I.uploaded[1])) {
            I.srcs_dev = n;
            I.dev_w = w;
            I.dev_h = h;
        }
        return MVS_OK;
    }
    const int rc = mvs::parallel_copy(pieces, 0);
    if (up && rc == 0 && cudaEventRecord(I.uploaded[1], 0) == cudaSuccess) {
        I.srcs_dev = n;
        I.dev_w = w;
        I.dev_h = h;
    }
    return MVS_OK;
}

int mvs_ps_set_K(mvs_planesweep *ps, const float *K9)
{
    PS_CHECK(ps);
    if (!K9) return mvs::set_error(MVS_ERR_ARG, "null K");
    ps->ps.setK(Matrix3D(K9));
    return MVS_OK;
}

int mvs_ps_set_z(mvs_planesweep *ps, float n, float f)
{
    PS_CHECK(ps);
    ps->ps.setZ(n, f);
    return MVS_OK;
}

int mvs_ps_set_number_of_planes(mvs_planesweep *ps, int32_t n)
{
    PS_CHECK(ps);
    if (n <= 0) return mvs::set_error(MVS_ERR_ARG, "plane count must be positive");
    ps->ps.setNumberofPlanes(n);
    return MVS_OK;
}

int mvs_ps_set_number_of_images(mvs_planesweep *ps, int32_t n)
{
    PS_CHECK(ps);
    if (n <= 0) return mvs::set_error(MVS_ERR_ARG, "image count must be positive");
    ps->ps.setNumberofImages(n);
    return MVS_OK;
}

int mvs_ps_set_window_size(mvs_planesweep *ps, int32_t n)
{
    PS_CHECK(ps);
    if (n <= 0 || n % 2 == 0) return mvs::set_error(MVS_ERR_ARG, "Window size must be an odd number");
    ps->ps.setWindowSize(n);
    return MVS_OK;
}

int mvs_ps_set_std_threshold(mvs_planesweep *ps, float th)
{
    PS_CHECK(ps);
    ps->ps.setSTDthreshold(th);
    return MVS_OK;
}

int mvs_ps_set_ncc_threshold(mvs_planesweep *ps, float th)
{
    PS_CHECK(ps);
    ps->ps.setNCCthreshold(th);
    return MVS_OK;
}

int mvs_ps_set_alternative_relative_matrix_method(mvs_planesweep *ps, int32_t alt)
{
    PS_CHECK(ps);
    ps->ps.setAlternativeRelativeMatrixMethod(alt != 0);
    return MVS_OK;
}

int mvs_ps_set_plane_depths(mvs_planesweep *ps, const float *depths, int32_t n)
{
    PS_CHECK(ps);
    if (n < 0 || (n > 0 && !depths)) return mvs::set_error(MVS_ERR_ARG, "bad plane list");
    ps->ps.setPlaneDepths(std::vector<float>(depths, depths + n));
    return MVS_OK;
}

int mvs_ps_set_sweep_options(mvs_planesweep *ps, int32_t moments, int32_t mode, int32_t fp64)
{
    PS_CHECK(ps);
    if (moments != MVS_MOMENTS_REFERENCE && moments != MVS_MOMENTS_COMPENSATED)
        return mvs::set_error(MVS_ERR_ARG, "unknown moments mode %d", moments);
    if (mode != MVS_SWEEP_PER_VIEW && mode != MVS_SWEEP_AGGREGATED)
        return mvs::set_error(MVS_ERR_ARG, "unknown sweep mode %d", mode);
    ps->ps.setSweepOptions(moments, mode, fp64 != 0);
    return MVS_OK;
}

int mvs_ps_run_algorithm(mvs_planesweep *ps)
{
    PS_CHECK(ps);
    mvs::set_error(MVS_OK, "");
    if (ps->ps.RunAlgorithm(0, nullptr)) return MVS_OK;
    return mvs_last_error()[0] ? MVS_ERR_CUDA : MVS_ERR_STATE;
}

int mvs_ps_cuda_denoise(mvs_planesweep *ps, int32_t niters, double lambda, double tau, double sigma, double theta,
                        double beta, double gamma)
{
    PS_CHECK(ps);
    if (niters < 0) return mvs::set_error(MVS_ERR_ARG, "negative iteration count");
    return ps->ps.CudaDenoise(0, nullptr, niters, lambda, tau, sigma, theta, beta, gamma) ? MVS_OK : MVS_ERR_STATE;
}

int mvs_ps_tgv(mvs_planesweep *ps, int32_t niters, int32_t warps, double lambda, double alpha0, double alpha1,
               double tau, double sigma, double beta, double gamma)
{
    PS_CHECK(ps);
    if (niters < 0 || warps < 0) return mvs::set_error(MVS_ERR_ARG, "negative iteration count");
    return ps->ps.TGV(0, nullptr, niters, warps, lambda, alpha0, alpha1, tau, sigma, beta, gamma) ? MVS_OK
                                                                                                  : MVS_ERR_STATE;
}

int mvs_ps_tgv_denoise_from_sparse(mvs_planesweep *ps, const float *h_sparse, int32_t niters, double alpha0,
                                   double alpha1, double tau, double sigma, double theta, double beta, double gamma)
{
    PS_CHECK(ps);
    if (!h_sparse) return mvs::set_error(MVS_ERR_ARG, "null sparse depthmap");
    if (niters < 0) return mvs::set_error(MVS_ERR_ARG, "negative iteration count");
    CamImage<float> sp;
    sp.reset(ps->ps.HostRef.width(), ps->ps.HostRef.height());
    memcpy(sp.data(), h_sparse, sizeof(float) * sp.elements());
    return ps->ps.TGVdenoiseFromSparse(0, nullptr, sp, niters, alpha0, alpha1, tau, sigma, theta, beta, gamma)
               ? MVS_OK
               : MVS_ERR_STATE;
}

int mvs_ps_tgv_ext(mvs_planesweep *ps, const mvs_tgv2_params *p, int32_t start, const float *u_init, int32_t *iters,
                   double *energy)
{
    PS_CHECK(ps);
    if (!p || start < 0 || start > 2) return mvs::set_error(MVS_ERR_ARG, "bad TGV arguments");
    CamImage<float> init;
    if (start == 2) {
        if (!u_init) return mvs::set_error(MVS_ERR_ARG, "null start depthmap");
        init.reset(ps->ps.HostRef.width(), ps->ps.HostRef.height());
        memcpy(init.data(), u_init, sizeof(float) * init.elements());
    }
    int it = 0;
    const bool ok = ps->ps.TGVext(*p, start, start == 2 ? &init : nullptr, &it, energy);
    if (iters) *iters = it;
    return ok ? MVS_OK : MVS_ERR_STATE;
}

int mvs_ps_get_size(mvs_planesweep *ps, int32_t *w, int32_t *h)
{
    PS_CHECK(ps);
    if (w) *w = (int32_t)ps->ps.HostRef.width();
    if (h) *h = (int32_t)ps->ps.HostRef.height();
    return MVS_OK;
}

// The image getters copy width * height values of the current reference
// frame (mvs_ps_get_size): a result of a frame of another size (the reference
// was set again since) is refused rather than copied past the caller's buffer.
static int frame_check(const mvs_planesweep *ps, size_t w, size_t h, const char *what)
{
    const size_t W = ps->ps.HostRef.width(), H = ps->ps.HostRef.height();
    if (w != W || h != H)
        return mvs::set_error(MVS_ERR_STATE, "the %s is of a %zux%zu frame, the reference is now %zux%zu: run again",
                              what, w, h, W, H);
    return MVS_OK;
}

extern "C++" {
template <typename T>
static int copy_image(const mvs_planesweep *ps, const CamImage<T> *img, T *out)
{
    if (!out) return mvs::set_error(MVS_ERR_ARG, "null output");
    if (!img || img->empty()) return mvs::set_error(MVS_ERR_STATE, "no such depthmap yet");
    if (int rc = frame_check(ps, img->width(), img->height(), "depthmap")) return rc;
    // the pool's threads share a large copy; nothing is uploaded
    mvs::parallel_copy({{out, img->data(), sizeof(T) * img->elements(), nullptr}}, 0);
    return MVS_OK;
}
}

int mvs_ps_get_depthmap(mvs_planesweep *ps, float *out) { PS_CHECK(ps); return copy_image(ps, ps->ps.getDepthmap(), out); }
int mvs_ps_get_depthmap8u(mvs_planesweep *ps, uint8_t *out)
{
    PS_CHECK(ps);
    return copy_image(ps, ps->ps.getDepthmap8u(), out);
}
int mvs_ps_get_depthmap_denoised(mvs_planesweep *ps, float *out)
{
    PS_CHECK(ps);
    return copy_image(ps, ps->ps.getDepthmapDenoised(), out);
}
int mvs_ps_get_depthmap8u_denoised(mvs_planesweep *ps, uint8_t *out)
{
    PS_CHECK(ps);
    return copy_image(ps, ps->ps.getDepthmap8uDenoised(), out);
}
int mvs_ps_get_depthmap_tgv(mvs_planesweep *ps, float *out)
{
    PS_CHECK(ps);
    return copy_image(ps, ps->ps.getDepthmapTGV(), out);
}
int mvs_ps_get_depthmap8u_tgv(mvs_planesweep *ps, uint8_t *out)
{
    PS_CHECK(ps);
    return copy_image(ps, ps->ps.getDepthmap8uTGV(), out);
}

int mvs_ps_get_depthmap_denoised_ptr(mvs_planesweep *ps, float **d_ptr)
{
    PS_CHECK(ps);
    if (!d_ptr) return mvs::set_error(MVS_ERR_ARG, "null output");
    *d_ptr = ps->ps.getDepthmapDenoisedPtr();
    return MVS_OK;
}

int mvs_ps_get_view_labels(mvs_planesweep *ps, int32_t *out)
{
    PS_CHECK(ps);
    mvs::clear_error();
    const std::vector<int32_t> &v = ps->ps.getViewLabels();
    if (v.empty())   // no sweep yet, or the copy back failed (its CUDA error is set)
        return mvs_last_error()[0] ? MVS_ERR_CUDA : mvs::set_error(MVS_ERR_STATE, "no sweep result");
    if (!out) return mvs::set_error(MVS_ERR_ARG, "null output");
    const CamImage<float> *d = ps->ps.getDepthmap();   // of the same sweep
    if (int rc = frame_check(ps, d->width(), d->height(), "sweep result")) return rc;
    memcpy(out, v.data(), v.size() * 4);
    return MVS_OK;
}

int mvs_ps_get_view_best(mvs_planesweep *ps, float *out)
{
    PS_CHECK(ps);
    mvs::clear_error();
    const std::vector<float> &v = ps->ps.getViewBest();
    if (v.empty())   // no sweep yet, or the copy back failed (its CUDA error is set)
        return mvs_last_error()[0] ? MVS_ERR_CUDA : mvs::set_error(MVS_ERR_STATE, "no sweep result");
    if (!out) return mvs::set_error(MVS_ERR_ARG, "null output");
    const CamImage<float> *d = ps->ps.getDepthmap();
    if (int rc = frame_check(ps, d->width(), d->height(), "sweep result")) return rc;
    memcpy(out, v.data(), v.size() * 4);
    return MVS_OK;
}

int mvs_ps_get_3d_coordinates(mvs_planesweep *ps, float *X, float *Y, float *Z)
{
    PS_CHECK(ps);
    CamImage<float> *x, *y, *z;
    ps->ps.get3Dcoordinates(x, y, z);
    if (!x) return MVS_ERR_STATE;
    if (int rc = frame_check(ps, x->width(), x->height(), "point map")) return rc;
    if (X) memcpy(X, x->data(), x->elements() * 4);
    if (Y) memcpy(Y, y->data(), y->elements() * 4);
    if (Z) memcpy(Z, z->data(), z->elements() * 4);
    return MVS_OK;
}

int mvs_ps_get_plane_count(mvs_planesweep *ps, int32_t *n)
{
    PS_CHECK(ps);
    if (!n) return mvs::set_error(MVS_ERR_ARG, "null output");
    *n = (int32_t)ps->ps.getPlaneDepths().size();
    return MVS_OK;
}

int mvs_ps_get_last_kernel_ms(mvs_planesweep *ps, float *ms)
{
    PS_CHECK(ps);
    if (!ms) return mvs::set_error(MVS_ERR_ARG, "null output");
    *ms = ps->ps.getLastKernelMs();
    return MVS_OK;
}

}  // extern "C"
