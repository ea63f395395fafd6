// Batched sweeps of uneven frames (no counterpart in the reference, whose
// PlaneSweep handles one reference frame per call): many reference frames of
// any size, view count, plane count and window go through one CUDA-graph
// launch -- a timestamp kernel, one launch of FP64 homographies for every
// (frame, view, plane), one launch building every frame's 2x2 source
// neighbourhoods and one persistent sweep kernel over a work list of
// (frame, tile, plane chunk) items (sweep.cu).  The aggregated mode (cost =
// 1 - mean NCC over views, winner-take-all) is computed, with the moments the
// caller picks.
//
// The work list's plane chunk size, the number of persistent CTAs per SM, the
// item order and the tile shape are chosen by an autotuner that times each
// candidate on the batch itself; its choice is cached per batch shape (the
// only global mutable state of the library).
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace mvs {
int sweep_tile_width(int win, int tws);
int sweep_tile_height();
int sweep_batch_launch(const BatchFrameDev *frames, const uint4 *items, int n_items, unsigned int *next,
                       unsigned long long *t_start, const BatchCamDev *cams, const int *hom_offsets, int n_frames,
                       int n_hom, int moments, int ctas, int tws, void *stream);
}  // namespace mvs

using namespace mvs;

struct mvs_batch {
    int n = 0, moments = 0;
    std::vector<mvs_batch_frame> frames;
    std::vector<BatchFrameDev> fdev;   // host copy of the device descriptors
    std::vector<BatchCamDev> cams;
    std::vector<int> hom_off;
    mvs_batch_tuning tuning{};
    int n_items = 0, n_hom = 0;
    // device memory
    char *mem = nullptr;
    BatchFrameDev *d_frames = nullptr;
    BatchCamDev *d_cams = nullptr;
    int *d_hom_off = nullptr;
    uint4 *d_items = nullptr;
    unsigned int *d_next = nullptr;
    unsigned long long *d_t0 = nullptr;
    unsigned long long *d_done = nullptr;   // [n]
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    float last_ms = 0.f;
};

namespace {

constexpr int kBatchTileSteps = 2;   // tile shapes the batched sweep is compiled for
std::mutex g_tune_lock;
std::map<std::string, mvs_batch_tuning> g_tune_cache;

std::string signature(const mvs_batch *b)
{
    std::string s = std::to_string(b->moments);
    for (const auto &f : b->frames)
        s += "|" + std::to_string(f.width) + "x" + std::to_string(f.height) + "v" + std::to_string(f.n_views) + "p" +
             std::to_string(f.n_planes) + "w" + std::to_string(f.window);
    return s;
}

int validate(const mvs_batch_frame &f, int i)
{
    if (f.width < 16 || f.height < 16) return set_error(MVS_ERR_ARG, "frame %d: size %dx%d", i, f.width, f.height);
    if (f.n_views < 1 || f.n_views > kBatchMaxViews)
        return set_error(MVS_ERR_ARG, "frame %d: 1..%d views", i, kBatchMaxViews);
    if (f.n_planes < 1 || f.n_planes > 65535) return set_error(MVS_ERR_ARG, "frame %d: 1..65535 planes", i);
    if (f.window < 3 || f.window > 15 || f.window % 2 == 0)
        return set_error(MVS_ERR_ARG, "frame %d: window %d (odd, 3..15)", i, f.window);
    if (f.width < f.window || f.height < f.window) return set_error(MVS_ERR_ARG, "frame %d: narrower than its window", i);
    if (!f.d_ref || !f.d_srcs || !f.d_depths || !f.d_depth || !f.h_K9 || !f.h_Rrel || !f.h_trel)
        return set_error(MVS_ERR_ARG, "frame %d: null pointer", i);
    return MVS_OK;
}

// K^-1 as mvs_sweep_homographies forms it (adjugate / determinant), so a
// batched frame gets the single-frame path's homographies bit for bit
void inv3(const double *m, double *o)
{
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    const double inv[9] = {(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det,
                           (m[1] * m[5] - m[2] * m[4]) / det, (m[5] * m[6] - m[3] * m[8]) / det,
                           (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                           (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det,
                           (m[0] * m[4] - m[1] * m[3]) / det};
    for (int k = 0; k < 9; ++k) o[k] = inv[k];
}

void fill_cams(mvs_batch *b)
{
    for (int i = 0; i < b->n; ++i) {
        const mvs_batch_frame &f = b->frames[i];
        BatchCamDev &c = b->cams[i];
        for (int k = 0; k < 9; ++k) c.K[k] = f.h_K9[k];
        inv3(c.K, c.invK);
        for (int v = 0; v < f.n_views; ++v) {
            for (int k = 0; k < 9; ++k) c.Rrel[v][k] = f.h_Rrel[9 * v + k];
            for (int k = 0; k < 3; ++k) c.trel[v][k] = f.h_trel[3 * v + k];
        }
    }
}

// Work list and per-frame chunking for one tuning; uploads descriptors,
// items and re-armed counters (synchronously, outside any capture).
int build_items(mvs_batch *b, const mvs_batch_tuning &t)
{
    std::vector<uint4> items;
    std::vector<std::vector<uint4>> per(b->n);
    std::vector<std::vector<unsigned>> tile_init(b->n);
    for (int i = 0; i < b->n; ++i) {
        BatchFrameDev &d = b->fdev[i];
        const mvs_batch_frame &f = b->frames[i];
        d.tile_w = sweep_tile_width(f.window, t.tile_step);
        d.tiles_x = ceil_div(f.width, d.tile_w);
        d.n_tiles = d.tiles_x * ceil_div(f.height, sweep_tile_height());
        const int ppc = t.planes_per_chunk > 0 ? std::min(t.planes_per_chunk, f.n_planes) : f.n_planes;
        d.planes_per_chunk = ppc;
        d.n_chunks = ceil_div(f.n_planes, ppc);
        for (int tile = 0; tile < d.n_tiles; ++tile)
            for (int c = 0; c < d.n_chunks; ++c) per[i].push_back(make_uint4(i, tile, c, 0));
        tile_init[i].assign(d.n_tiles, (unsigned)d.n_chunks);
    }
    std::vector<int> order(b->n);
    for (int i = 0; i < b->n; ++i) order[i] = i;
    if (t.order == MVS_BATCH_ORDER_LARGEST_FIRST)
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            const auto &a = b->frames[x], &c = b->frames[y];
            return (double)a.width * a.height * a.n_planes * a.n_views > (double)c.width * c.height * c.n_planes * c.n_views;
        });
    if (t.order == MVS_BATCH_ORDER_INTERLEAVED) {
        size_t k = 0;
        bool any = true;
        while (any) {
            any = false;
            for (int i : order)
                if (k < per[i].size()) {
                    items.push_back(per[i][k]);
                    any = true;
                }
            ++k;
        }
    } else {
        for (int i : order) items.insert(items.end(), per[i].begin(), per[i].end());
    }
    b->n_items = (int)items.size();
    // device buffers that depend on the tuning
    cudaFree(b->d_items);
    b->d_items = nullptr;
    MVS_TRY_CUDA(cudaMalloc(&b->d_items, items.size() * sizeof(uint4)));
    MVS_TRY_CUDA(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    for (int i = 0; i < b->n; ++i) {
        const BatchFrameDev &d = b->fdev[i];
        MVS_TRY_CUDA(cudaMemcpy(d.tile_left, tile_init[i].data(), tile_init[i].size() * sizeof(unsigned),
                                cudaMemcpyHostToDevice));
        const unsigned tl = (unsigned)d.n_tiles;
        MVS_TRY_CUDA(cudaMemcpy(d.frame_left, &tl, sizeof(unsigned), cudaMemcpyHostToDevice));
    }
    MVS_TRY_CUDA(cudaMemcpy(b->d_frames, b->fdev.data(), b->n * sizeof(BatchFrameDev), cudaMemcpyHostToDevice));
    return MVS_OK;
}

int capture(mvs_batch *b, const mvs_batch_tuning &t)
{
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    int sms = 0, dev = 0;
    MVS_TRY_CUDA(cudaGetDevice(&dev));
    MVS_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int ctas = std::max(1, t.ctas_per_sm) * sms;
    cudaGraph_t g = nullptr;
    MVS_TRY_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    int rc = sweep_batch_launch(b->d_frames, b->d_items, b->n_items, b->d_next, b->d_t0, b->d_cams, b->d_hom_off, b->n,
                                b->n_hom, b->moments, ctas, t.tile_step, b->cap);
    cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return set_error(MVS_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return set_error(MVS_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e));
    return MVS_OK;
}

int apply(mvs_batch *b, const mvs_batch_tuning &t)
{
    if (t.tile_step < 0 || t.tile_step > kBatchTileSteps - 1)
        return set_error(MVS_ERR_ARG, "tile_step %d (0..%d)", t.tile_step, kBatchTileSteps - 1);
    if (t.ctas_per_sm < 1 || t.ctas_per_sm > 3) return set_error(MVS_ERR_ARG, "ctas_per_sm %d (1..3)", t.ctas_per_sm);
    int rc = build_items(b, t);
    if (rc) return rc;
    rc = capture(b, t);
    if (rc) return rc;
    b->tuning = t;
    return MVS_OK;
}

int run_timed(mvs_batch *b, cudaStream_t st, float *ms)
{
    cudaEvent_t a, c;
    MVS_TRY_CUDA(cudaEventCreate(&a));
    MVS_TRY_CUDA(cudaEventCreate(&c));
    cudaEventRecord(a, st);
    cudaError_t e = cudaGraphLaunch(b->exec, st);
    cudaEventRecord(c, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(c);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, a, c);
    cudaEventDestroy(a);
    cudaEventDestroy(c);
    if (e != cudaSuccess) return set_error(MVS_ERR_CUDA, "batch launch: %s", cudaGetErrorString(e));
    return MVS_OK;
}

// Search: plane chunk x CTAs per SM x item order on the widest tile, then the
// best of those on the narrower tile (72 candidates would double the tuning
// time; the tile shape interacts mostly with the chunk size and CTA count).
int autotune(mvs_batch *b, mvs_batch_tuning *best)
{
    const int chunks[] = {16, 32, 64, 0};
    const int ctas[] = {1, 2, 3};
    const int orders[] = {MVS_BATCH_ORDER_FRAME, MVS_BATCH_ORDER_LARGEST_FIRST, MVS_BATCH_ORDER_INTERLEAVED};
    float best_ms = 1e30f;
    auto trial = [&](const mvs_batch_tuning &t) -> int {
        int rc = apply(b, t);
        if (rc) return rc;
        float ms = 0.f, m2 = 0.f;
        if ((rc = run_timed(b, b->cap, &ms))) return rc;   // warm-up
        if ((rc = run_timed(b, b->cap, &ms))) return rc;
        if ((rc = run_timed(b, b->cap, &m2))) return rc;
        ms = std::min(ms, m2);
        if (ms < best_ms) {
            best_ms = ms;
            *best = t;
        }
        return MVS_OK;
    };
    for (int c : chunks)
        for (int k : ctas)
            for (int o : orders) {
                mvs_batch_tuning t{c, k, o, 0};
                if (int rc = trial(t)) return rc;
            }
    // the narrower tile with the chunk sizes and CTA counts around the best so far
    const mvs_batch_tuning w = *best;
    for (int c : chunks)
        for (int k : ctas)
            if (int rc = trial(mvs_batch_tuning{c, k, w.order, 1})) return rc;
    return MVS_OK;
}

}  // namespace

extern "C" {

int mvs_batch_create(mvs_batch **out, const mvs_batch_frame *frames, int32_t n, int32_t moments,
                     const mvs_batch_tuning *tuning)
{
    if (!out || !frames || n <= 0) return set_error(MVS_ERR_ARG, "null argument or empty batch");
    *out = nullptr;
    if (moments != MVS_MOMENTS_REFERENCE && moments != MVS_MOMENTS_COMPENSATED)
        return set_error(MVS_ERR_ARG, "moments %d", moments);
    for (int i = 0; i < n; ++i)
        if (int rc = validate(frames[i], i)) return rc;
    mvs_batch *b = new mvs_batch();
    b->n = n;
    b->moments = moments;
    b->frames.assign(frames, frames + n);
    b->fdev.resize(n);
    b->cams.resize(n);
    b->hom_off.assign(n + 1, 0);
    // one allocation for descriptors, homographies, winner words, counters
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_frames = take(n * sizeof(BatchFrameDev)), o_cams = take(n * sizeof(BatchCamDev));
    const size_t o_hom = take((n + 1) * sizeof(int)), o_next = take(sizeof(unsigned)), o_t0 = take(8);
    const size_t o_done = take(n * 8);
    std::vector<size_t> o_H(n), o_wta(n), o_tiles(n), o_fl(n), o_quad(n);
    for (int i = 0; i < n; ++i) {
        const mvs_batch_frame &f = frames[i];
        // tile counts of the widest tile here; build_items sets those of the tuning
        const int tw = sweep_tile_width(f.window, 0), th = sweep_tile_height();
        const int tiles_max = ceil_div(f.width, sweep_tile_width(f.window, kBatchTileSteps - 1)) * ceil_div(f.height, th);
        BatchFrameDev &d = b->fdev[i];
        d.w = f.width;
        d.h = f.height;
        d.V = f.n_views;
        d.P = f.n_planes;
        d.win = f.window;
        d.tile_w = tw;
        d.tiles_x = ceil_div(f.width, tw);
        d.n_tiles = d.tiles_x * ceil_div(f.height, th);
        d.stdthresh = f.std_threshold;
        d.zfar = f.zfar;
        b->hom_off[i + 1] = b->hom_off[i] + f.n_views * f.n_planes;
        o_H[i] = take((size_t)f.n_views * f.n_planes * 9 * sizeof(float));
        o_wta[i] = take((size_t)f.width * f.height * 8);
        o_tiles[i] = take((size_t)tiles_max * sizeof(unsigned));
        o_fl[i] = take(sizeof(unsigned));
        // 2x2 source neighbourhoods, rebuilt from the sources at every launch
        o_quad[i] = take((size_t)f.width * f.height * f.n_views * sizeof(float4));
    }
    b->n_hom = b->hom_off[n];
    cudaError_t e = cudaMalloc(&b->mem, off);
    if (e != cudaSuccess) {
        delete b;
        return set_error(MVS_ERR_NOMEM, "batch: %zu bytes: %s", off, cudaGetErrorString(e));
    }
    b->d_frames = (BatchFrameDev *)(b->mem + o_frames);
    b->d_cams = (BatchCamDev *)(b->mem + o_cams);
    b->d_hom_off = (int *)(b->mem + o_hom);
    b->d_next = (unsigned *)(b->mem + o_next);
    b->d_t0 = (unsigned long long *)(b->mem + o_t0);
    b->d_done = (unsigned long long *)(b->mem + o_done);
    for (int i = 0; i < n; ++i) {
        const mvs_batch_frame &f = frames[i];
        BatchFrameDev &d = b->fdev[i];
        d.ref = f.d_ref;
        d.srcs = f.d_srcs;
        d.depths = f.d_depths;
        float *Hf = (float *)(b->mem + o_H[i]);
        d.H = Hf;
        d.depth = f.d_depth;
        d.labels = f.d_labels;
        d.best = f.d_best;
        d.wta = (unsigned long long *)(b->mem + o_wta[i]);
        d.tile_left = (unsigned *)(b->mem + o_tiles[i]);
        d.frame_left = (unsigned *)(b->mem + o_fl[i]);
        d.done_ns = b->d_done + i;
        d.quad = (const float4 *)(b->mem + o_quad[i]);
        BatchCamDev &c = b->cams[i];
        c.depths = f.d_depths;
        c.H = Hf;
        c.V = f.n_views;
        c.P = f.n_planes;
        e = cudaMemset(d.wta, 0xff, (size_t)f.width * f.height * 8);
        if (e != cudaSuccess) break;
    }
    int rc = e == cudaSuccess ? MVS_OK : set_error(MVS_ERR_CUDA, "batch init: %s", cudaGetErrorString(e));
    if (!rc) {
        fill_cams(b);
        e = cudaMemcpy(b->d_cams, b->cams.data(), n * sizeof(BatchCamDev), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->d_hom_off, b->hom_off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = set_error(MVS_ERR_CUDA, "batch init: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        mvs_batch_tuning t{};
        if (tuning) {
            t = *tuning;
        } else {
            const std::string key = signature(b);
            bool cached = false;
            {
                std::lock_guard<std::mutex> g(g_tune_lock);
                auto it = g_tune_cache.find(key);
                if (it != g_tune_cache.end()) {
                    t = it->second;
                    cached = true;
                }
            }
            if (!cached) {
                rc = autotune(b, &t);
                if (!rc) {
                    std::lock_guard<std::mutex> g(g_tune_lock);
                    g_tune_cache[key] = t;
                }
            }
        }
        if (!rc) rc = apply(b, t);
    }
    if (rc) {
        mvs_batch_destroy(b);
        return rc;
    }
    *out = b;
    return MVS_OK;
}

int mvs_batch_destroy(mvs_batch *b)
{
    if (!b) return MVS_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->cap) cudaStreamDestroy(b->cap);
    cudaFree(b->d_items);
    cudaFree(b->mem);
    delete b;
    return MVS_OK;
}

int mvs_batch_get_tuning(const mvs_batch *b, mvs_batch_tuning *t)
{
    if (!b || !t) return set_error(MVS_ERR_ARG, "null argument");
    *t = b->tuning;
    return MVS_OK;
}

int mvs_batch_set_poses(mvs_batch *b, const double *h_Rrel, const double *h_trel, void *stream)
{
    if (!b || !h_Rrel || !h_trel) return set_error(MVS_ERR_ARG, "null argument");
    size_t v0 = 0;
    for (int i = 0; i < b->n; ++i) {
        BatchCamDev &c = b->cams[i];
        for (int v = 0; v < c.V; ++v) {
            for (int k = 0; k < 9; ++k) c.Rrel[v][k] = h_Rrel[9 * (v0 + v) + k];
            for (int k = 0; k < 3; ++k) c.trel[v][k] = h_trel[3 * (v0 + v) + k];
        }
        v0 += c.V;
    }
    // synchronous: the host array is reused by the caller
    MVS_TRY_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    MVS_TRY_CUDA(cudaMemcpy(b->d_cams, b->cams.data(), b->n * sizeof(BatchCamDev), cudaMemcpyHostToDevice));
    return MVS_OK;
}

int mvs_batch_run(mvs_batch *b, void *stream)
{
    if (!b || !b->exec) return set_error(MVS_ERR_STATE, "batch not ready");
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(MVS_ERR_CUDA, "batch launch: %s", cudaGetErrorString(e));
    return MVS_OK;
}

int mvs_batch_frame_latency_ms(mvs_batch *b, float *h_ms, void *stream)
{
    if (!b || !h_ms) return set_error(MVS_ERR_ARG, "null argument");
    std::vector<unsigned long long> t(b->n + 1);
    cudaStream_t st = (cudaStream_t)stream;
    MVS_TRY_CUDA(cudaStreamSynchronize(st));
    MVS_TRY_CUDA(cudaMemcpy(t.data(), b->d_t0, 8, cudaMemcpyDeviceToHost));
    MVS_TRY_CUDA(cudaMemcpy(t.data() + 1, b->d_done, b->n * 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < b->n; ++i) h_ms[i] = (float)((double)(t[i + 1] - t[0]) * 1e-6);
    return MVS_OK;
}

int64_t mvs_batch_work_items(const mvs_batch *b) { return b ? b->n_items : 0; }

}  // extern "C"
