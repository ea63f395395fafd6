// Warm-start network for TGV2 (no counterpart in the reference): a 4-level
// U-Net (16/32/64/128 channels) that maps the sweep's winner-take-all depth,
// its matching confidence and the reference image to a prediction of the
// converged TGV2 primal (u, v).  Training and inference run on the kernels of
// this file.
//
// Activations are NHWC bf16 with channel counts that are multiples of 16.  A
// 3x3 convolution is an implicit GEMM on the 5th-generation tensor cores:
//   D[128 pixels][Cout] += A_tap[128 pixels][16 ch] * B_tap[Cout][16 ch]
// for every tap and 16-channel slice, one tcgen05.mma (kind::f16, BF16 in,
// FP32 accumulator in tensor memory) each.  A CTA owns an 8 x 16 pixel tile;
// its (8+2) x (16+2) input halo sits in shared memory as two planes of 8
// channels, 16 bytes per pixel, which is exactly the "no swizzle, K-major"
// operand layout (8 rows x 16 bytes per core matrix), so every tap's A operand
// is the same halo addressed from a different start: no im2col copy.  The
// weights of a slice are staged as [tap][8-ch plane][Cout][8].  Two stages
// alternate: the copy of slice c+1 overlaps the MMAs of slice c, and an
// mbarrier signalled by tcgen05.commit says when a stage may be refilled.
// The epilogue reads the accumulator with tcgen05.ld (one pixel per thread),
// adds the bias, applies ReLU or the ReLU mask of the backward pass and
// stores bf16.
//
// The backward pass w.r.t. the input is the same kernel with the weights
// flipped and transposed; the weight gradient is a per-tap reduction over
// pixels on the CUDA cores (FP32), with the bias gradient.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace mvs {
namespace unet {

typedef uint16_t bf16;   // raw bits

constexpr int TW = 8, TH = 16;               // output tile (M = 128 pixels)
constexpr int HW_ = TW + 2, HH_ = TH + 2;     // halo
constexpr int HALO_PIX = HW_ * HH_;           // 180
constexpr int HALO_BYTES = 2 * HALO_PIX * 16; // two 8-channel planes
constexpr int CONV_THREADS = 128;
// output tiles per CTA of the convolution at 16 and 32 output channels
constexpr int CONV_MT16 = 2, CONV_MT32 = 2;

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier helpers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------


// shared-memory matrix descriptor: no swizzle, K-major core matrices of 8 rows
// x 16 bytes; lbo = byte distance between the two 8-element K halves, sbo =
// byte distance between consecutive 8-row groups; version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D f32, A and B bf16, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}


__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid)
{
    // src-size 0 zero-fills the 16 bytes (padding outside the image)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) { return (uint32_t)f2bf(a) | ((uint32_t)f2bf(b) << 16); }

// ---------------------------------------------------------------------------
// 3x3 convolution, zero padding, on tensor cores
// ---------------------------------------------------------------------------

struct ConvArgs {
    const bf16 *in;     // [B][H][W][cin]
    const bf16 *wpack;  // [9][cin/8][COUT][8]
    const float *bias;  // [COUT] or null
    const bf16 *mask;   // [B][H][W][COUT] or null: out *= (mask > 0)
    bf16 *out;          // [B][H][W][COUT]
    int *err;           // set to 1 when a bounded wait gives up
    int H, W, cin, relu, tiles_x;
};

constexpr uint64_t kWaitNs = 1000000000ull;   // 1 s

#define MVS_RC_(x)                \
    do {                          \
        int rc__ = (x);           \
        if (rc__) return rc__;    \
    } while (0)

// MT output tiles of 8 x 16 pixels stacked vertically per CTA: they share
// one (MT * 16 + 2)-row halo and one copy of the weights, and accumulate in
// MT column blocks of COUT in tensor memory.
template <int COUT, int MT = 1>
struct ConvSmem {
    static constexpr int HALO_ROWS = MT * TH + 2;
    static constexpr int HPIX = HW_ * HALO_ROWS;          // halo pixels
    static constexpr int HBYTES = 2 * HPIX * 16;          // two 8-channel planes
    static constexpr int W_BYTES = 9 * 2 * COUT * 16;
    static constexpr int STAGE = (HBYTES + W_BYTES + 127) / 128 * 128;
    static constexpr int BYTES = 2 * STAGE + 64;
    static constexpr int TMEM_COLS = MT * COUT <= 32 ? 32 : MT * COUT <= 64 ? 64 : MT * COUT <= 128 ? 128 : 256;
};

template <int COUT, int MT = 1>
__global__ void __launch_bounds__(CONV_THREADS) conv3x3_tc_kernel(ConvArgs a)
{
    using S = ConvSmem<COUT, MT>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int H = a.H, W = a.W, cin = a.cin;
    const int nslices = cin >> 4;
    // one 16-channel slice needs one stage (launch_conv_t gives the CTA that much)
    const int nstages = nslices > 1 ? 2 : 1;
    uint64_t *bars = (uint64_t *)(smem + nstages * S::STAGE);
    uint32_t *tmem_slot = (uint32_t *)(smem + nstages * S::STAGE + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int b = blockIdx.y;
    const int tx = blockIdx.x % a.tiles_x, ty = blockIdx.x / a.tiles_x;
    const int x0 = tx * TW, y0 = ty * (MT * TH);
    const size_t img = (size_t)H * W;

    if (warp == 0) tmem_alloc(tmem_slot, S::TMEM_COLS);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t sbase = smem_u32(smem);

    // stage slice c into buffer s: halo pixels (2 x 16 B) and 9 taps of weights
    auto load = [&](int c, int s) {
        const uint32_t hb = sbase + s * S::STAGE, wb = hb + S::HBYTES;
        for (int k = tid; k < 2 * S::HPIX; k += CONV_THREADS) {
            const int pix = k >> 1, half = k & 1;
            const int hy = pix / HW_, hx = pix - hy * HW_;
            const int gy = y0 - 1 + hy, gx = x0 - 1 + hx;
            const bool ok = gy >= 0 && gy < H && gx >= 0 && gx < W;
            const bf16 *src = a.in + ((size_t)b * img + (ok ? (size_t)gy * W + gx : 0)) * cin + 16 * c + 8 * half;
            cp_async16(hb + (half * S::HPIX + pix) * 16, src, ok);
        }
        constexpr int WV = 2 * COUT;   // 16-byte vectors per tap
        for (int k = tid; k < 9 * WV; k += CONV_THREADS) {
            const int t = k / WV, r = k - t * WV;   // r = plane * COUT + co
            const bf16 *src = a.wpack + ((size_t)(t * (cin >> 3) + 2 * c) * COUT) * 8 + (size_t)r * 8;
            cp_async16(wb + (t * WV + r) * 16, src, true);
        }
        cp_async_wait_all();
        fence_async_smem();
    };

    constexpr uint32_t idesc = idesc_bf16(128, COUT);
    bool failed = false;
    load(0, 0);
    __syncthreads();
    for (int c = 0; c < nslices; ++c) {
        const int s = c & 1;
        if (tid == 0) {
            tc_fence_after();
            const uint32_t hb = sbase + s * S::STAGE, wb = hb + S::HBYTES;
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int ky = t / 3, kx = t - 3 * ky;
                const uint64_t bd = smem_desc(wb + t * 2 * COUT * 16, COUT * 16, 128);
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    const uint64_t ad = smem_desc(hb + ((mt * TH + ky) * HW_ + kx) * 16, S::HPIX * 16, HW_ * 16);
                    mma_bf16(tmem + (uint32_t)(mt * COUT), ad, bd, idesc, (c > 0 || t > 0) ? 1u : 0u);
                }
            }
            mma_commit(&bars[s]);
        }
        if (c + 1 < nslices) {
            if (c >= 1) {
                // stage s^1 was last read by the MMAs of slice c-1
                const bool ok = mbar_wait_bounded(&bars[s ^ 1], ((c - 1) >> 1) & 1, kWaitNs);
                failed = __syncthreads_or(!ok) != 0;
                if (failed) break;
            }
            load(c + 1, s ^ 1);
            __syncthreads();
        }
    }
    if (!failed) {
        const int last = nslices - 1;
        const bool ok = mbar_wait_bounded(&bars[last & 1], (last >> 1) & 1, kWaitNs);
        failed = __syncthreads_or(!ok) != 0;
    }
    if (failed) {
        if (tid == 0) atomicExch(a.err, 1);
        // give the tensor core a second bounded chance to finish before the
        // accumulator columns are released
        const int last = nslices - 1;
        mbar_wait_bounded(&bars[last & 1], (last >> 1) & 1, kWaitNs);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) {
            tc_fence_after();
            tmem_dealloc(tmem, S::TMEM_COLS);
        }
        return;
    }
    tc_fence_after();

    // epilogue: thread = accumulator row = pixel (of each of the MT tiles)
    const int m = warp * 32 + lane;
#pragma unroll 1
    for (int mt = 0; mt < MT; ++mt) {
    const int py = y0 + mt * TH + (m >> 3), px = x0 + (m & 7);
    const bool inside = py < H && px < W;
    const size_t pidx = (size_t)b * img + (size_t)min(py, H - 1) * W + min(px, W - 1);
#pragma unroll 1
    for (int c0 = 0; c0 < COUT; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * COUT + c0), v);
        if (a.bias) {
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] += a.bias[c0 + k];
        }
        if (a.relu) {
#pragma unroll
            for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k], 0.f);
        }
        if (a.mask && inside) {
            const uint4 *mp = (const uint4 *)(a.mask + pidx * COUT + c0);
            const uint4 m0 = mp[0], m1 = mp[1];
            const uint32_t mw[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (!(bf2f((uint16_t)(mw[k] & 0xffffu)) > 0.f)) v[2 * k] = 0.f;
                if (!(bf2f((uint16_t)(mw[k] >> 16)) > 0.f)) v[2 * k + 1] = 0.f;
            }
        }
        if (inside) {
            uint4 *op = (uint4 *)(a.out + pidx * COUT + c0);
            op[0] = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                               pack_bf16x2(v[6], v[7]));
            op[1] = make_uint4(pack_bf16x2(v[8], v[9]), pack_bf16x2(v[10], v[11]), pack_bf16x2(v[12], v[13]),
                               pack_bf16x2(v[14], v[15]));
        }
    }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

template <int COUT, int MT = 1>
int launch_conv_t(const ConvArgs &a, int B, cudaStream_t st)
{
    using S = ConvSmem<COUT, MT>;
    MVS_TRY_CUDA(cudaFuncSetAttribute(conv3x3_tc_kernel<COUT, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      S::BYTES));
    const int tiles = a.tiles_x * ceil_div(a.H, MT * TH);
    // a 16-channel input is one slice: one stage, so more CTAs share an SM
    const int bytes = a.cin > 16 ? S::BYTES : S::STAGE + 64;
    conv3x3_tc_kernel<COUT, MT><<<dim3(tiles, B), CONV_THREADS, bytes, st>>>(a);
    return MVS_OK;
}

int launch_conv(const bf16 *in, int cin, const bf16 *wpack, const float *bias, const bf16 *mask, bf16 *out, int cout,
                int B, int H, int W, int relu, int *err, cudaStream_t st)
{
    if (cin <= 0 || cin % 16 || cin > 512) return set_error(MVS_ERR_ARG, "conv input channels %d (multiple of 16)", cin);
    ConvArgs a{in, wpack, bias, mask, out, err, H, W, cin, relu, ceil_div(W, TW)};
    switch (cout) {
    case 16: return launch_conv_t<16, CONV_MT16>(a, B, st);
    case 32: return launch_conv_t<32, CONV_MT32>(a, B, st);
    case 48: return launch_conv_t<48>(a, B, st);
    case 64: return launch_conv_t<64>(a, B, st);
    case 96: return launch_conv_t<96>(a, B, st);
    case 128: return launch_conv_t<128>(a, B, st);
    case 192: return launch_conv_t<192>(a, B, st);
    default: return set_error(MVS_ERR_ARG, "conv output channels %d not built (16/32/48/64/96/128/192)", cout);
    }
}

// ---------------------------------------------------------------------------
// weight gradient on tensor cores: for every tap t = (ky, kx),
//   D[co][t][ci] += sum_p dz[p][co] * x[p + off_t][ci]
// with K = pixels, for 16-channel chunks of the input.  A = dz^T (M = co, up
// to 128 rows) and B = the nine tap-shifted copies of the input tile (N = 9
// taps x 16 channels = 144) are both MN-major with the same layout,
// [8-group][pixel][8]: A as [co/8][pixel][8], B as [tap][ci/8][pixel][8] where
// plane (t, g) holds x at the tile's pixels shifted by tap t's offset.  One K
// step of 16 pixels (two tile rows) is then a single MMA for all nine taps (8
// per tile, with N = 144), instead of one MMA per tap (72 with N = 16).  A CTA
// takes NCH = 1 or 2 chunks (16 or 32 input channels) against one staged dz
// tile: NCH MMAs per K step into NCH accumulators.  The tap planes are built
// in shared memory from the tile's input halo (wgrad_tc_kernel below); each
// CTA sums a run of pixel tiles in TMEM (144 NCH columns) and adds them to the
// FP32 gradient with one atomic per weight.
// ---------------------------------------------------------------------------

struct WgArgs {
    const bf16 *x;    // [B][H][W][cin]
    const bf16 *dz;   // [B][H][W][cout]
    float *dW;        // [cout][cin][9]
    int *err;
    int B, H, W, cin, cout, tiles_x, tiles_y, tiles_per_cta, n_tiles;
    int ci_base;      // first input channel of blockIdx.y == 0
};

constexpr int WG_TC_THREADS = 256;
constexpr int WG_NC = 16;                           // input channels per chunk
constexpr int WG_PLANES = 9 * WG_NC / 8;            // 18 B planes per chunk: (tap, channel group)

// Shared memory of wgrad_tc_kernel<NCH, R> for `cg` groups of 8 output
// channels (cg <= 16):
//   two MMA buffers, each A = dz [cg][128 pixels][16 B] followed by, per
//     16-channel chunk, B = the nine tap-shifted input planes
//     [tap][channel group][128 pixels][16 B] (18 planes);
//   R raw stages, each the dz tile [cg][128][16 B] and, per chunk, the input
//     halo [channel group][18 rows][10 columns][16 B], filled by cp.async.
// The A descriptor of an M = 128 MMA spans 16 groups (32 KB) from A's start;
// groups past cg read the B planes that follow and only fill accumulator rows
// co >= cout, which are never stored, so A needs no zero padding.
constexpr int WG_HALO_W = TW + 2, WG_HALO_H = TH + 2;          // 10 x 18 input pixels around an 8 x 16 tile
constexpr int WG_HALO_BYTES = 2 * WG_HALO_H * WG_HALO_W * 16;  // per chunk: 5760
constexpr int WG_PLANES_BYTES = WG_PLANES * 128 * 16;          // per chunk: 36864
constexpr int WG_SMEM_MAX = 227 * 1024;
constexpr int WG_SMEM_SM = 228 * 1024;   // shared memory of an SM, 1 KB of it reserved per CTA

struct WgLayout {
    int a_bytes, buf_bytes, raw_bytes, bytes;
};

__host__ __device__ inline WgLayout wg_layout(int nch, int stages, int cg)
{
    WgLayout L;
    L.a_bytes = cg * 128 * 16;
    L.buf_bytes = L.a_bytes + nch * WG_PLANES_BYTES;
    L.raw_bytes = L.a_bytes + nch * WG_HALO_BYTES;
    L.bytes = 2 * L.buf_bytes + stages * L.raw_bytes + 64;
    return L;
}

// MN-major descriptors have the instruction descriptor's transpose bits set
__host__ __device__ constexpr uint32_t idesc_bf16_mn(int M, int N) { return idesc_bf16(M, N) | (1u << 15) | (1u << 16); }

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The weight gradient of a 3x3 convolution on the tensor cores:
// dW[co][ci][tap] = sum over pixels of dz[co][p] x[ci][p + tap], K = pixels.
// Per 8 x 16 tile: the raw stage lands (cp.async, R - 1 tiles ahead), the CTA
// copies its dz tile and expands its input halo into the nine tap-shifted
// planes of an MMA buffer (shared-memory loads and stores: the input crosses
// L2 once instead of nine times), and one thread issues 8 K-steps of one
// MMA of 128 x (9 taps x 16 channels) x 16 pixels per chunk.  The two MMA
// buffers alternate; a buffer is rebuilt once the MMAs that read it have
// signalled its mbarrier (tcgen05.commit).  Every wait is bounded.
template <int NCH, int R>
__global__ void __launch_bounds__(WG_TC_THREADS) wgrad_tc_kernel(WgArgs a)
{
    static_assert(R >= 2, "at least two raw stages");
    constexpr int NBUF = 2;   // MMA buffers
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ci0 = a.ci_base + blockIdx.y * NCH * WG_NC, co0 = blockIdx.z * 128;
    const int cg = min(a.cout - co0, 128) >> 3;
    const WgLayout L = wg_layout(NCH, R, cg);
    uint64_t *bars = (uint64_t *)(smem + NBUF * L.buf_bytes + R * L.raw_bytes);
    uint32_t *tmem_slot = (uint32_t *)(smem + NBUF * L.buf_bytes + R * L.raw_bytes + 32);
    const int t_begin = blockIdx.x * a.tiles_per_cta;
    const int t_end = min(t_begin + a.tiles_per_cta, a.n_tiles);
    const int H = a.H, W = a.W, cin = a.cin, cout = a.cout;
    const size_t img = (size_t)H * W;
    constexpr int TMEM_COLS = NCH == 1 ? 256 : 512;   // 144 NCH used

    if (warp == 0) tmem_alloc(tmem_slot, TMEM_COLS);
    if (tid == 0) {
        for (int k = 0; k < NBUF; ++k) mbar_init(&bars[k], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t sbase = smem_u32(smem);
    const uint32_t rbase = sbase + NBUF * L.buf_bytes;

    // Each thread's copies are the same for every tile: dz pixel (tid & 127) of
    // the groups tid >> 7, + 2, ...; halo items tid, tid + 256, ... (chunk and
    // channel group, halo row, halo column), worked out once here.
    constexpr int HP = WG_HALO_H * WG_HALO_W;
    constexpr int HALO_ITEMS = NCH * 2 * HP;
    constexpr int HI = (HALO_ITEMS + WG_TC_THREADS - 1) / WG_TC_THREADS;
    const int dz_m = tid & 127, dz_y = dz_m >> 3, dz_x = dz_m & 7, dz_g0 = tid >> 7;
    int h_jg[HI], h_y[HI], h_x[HI];
#pragma unroll
    for (int i = 0; i < HI; ++i) {
        const int k = tid + i * WG_TC_THREADS;
        const int jg = k / HP, pix = k - jg * HP;
        h_jg[i] = k < HALO_ITEMS ? jg : -1;
        h_y[i] = pix / WG_HALO_W - 1;
        h_x[i] = pix - (pix / WG_HALO_W) * WG_HALO_W - 1;
    }
    // cp.async of tile `tile`'s dz and input halo into raw stage s (one commit group)
    auto load = [&](int tile, int s) {
        const int b = tile / (a.tiles_x * a.tiles_y), r = tile - b * a.tiles_x * a.tiles_y;
        const int y0 = (r / a.tiles_x) * TH, x0 = (r % a.tiles_x) * TW;
        const uint32_t ab = rbase + s * L.raw_bytes, hb = ab + L.a_bytes;
        const bf16 *xb = a.x + (size_t)b * img * cin + ci0;
        {
            const int gy = y0 + dz_y, gx = x0 + dz_x;
            const bool ok = gy < H && gx < W;
            const bf16 *src = a.dz + ((size_t)b * img + (ok ? (size_t)gy * W + gx : 0)) * cout + co0 + 8 * dz_g0;
            for (int g = dz_g0, i = 0; g < cg; g += 2, ++i) cp_async16(ab + (g * 128 + dz_m) * 16, src + 16 * i, ok);
        }
#pragma unroll
        for (int i = 0; i < HI; ++i) {
            if (h_jg[i] < 0) continue;
            const int gy = y0 + h_y[i], gx = x0 + h_x[i];
            const bool ok = gy >= 0 && gy < H && gx >= 0 && gx < W;
            const bf16 *src = xb + (ok ? (size_t)gy * W + gx : 0) * cin + 8 * h_jg[i];
            cp_async16(hb + (tid + i * WG_TC_THREADS) * 16, src, ok);
        }
        cp_async_commit();
    };
    // raw stage s -> MMA buffer q: the dz tile as is, the halo as nine
    // tap-shifted planes (thread = tile pixel m and one of the two channel
    // groups of each chunk, 16 B per plane)
    auto build = [&](int s, int q) {
        const uint4 *ra = (const uint4 *)(smem + NBUF * L.buf_bytes + s * L.raw_bytes);
        const uint4 *rh = ra + L.a_bytes / 16;
        uint4 *ba = (uint4 *)(smem + q * L.buf_bytes);
        uint4 *bp = ba + L.a_bytes / 16;
        for (int k = tid; k < cg * 128; k += WG_TC_THREADS) ba[k] = ra[k];
        const int m = tid & 127, my = m >> 3, mx = m & 7, g = tid >> 7;
#pragma unroll
        for (int j = 0; j < NCH; ++j) {
            const int jg = 2 * j + g;
            const uint4 *h = rh + jg * WG_HALO_H * WG_HALO_W;
            uint4 *dst = bp + j * (WG_PLANES_BYTES / 16) + g * 128 + m;
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int ky = t / 3, kx = t - 3 * ky;
                dst[t * 2 * 128] = h[(my + ky) * WG_HALO_W + mx + kx];
            }
        }
    };

    constexpr uint32_t idesc = idesc_bf16_mn(128, 9 * WG_NC);
    const int n = t_end - t_begin;
    bool failed = false;
    int last = -1;   // the last tile whose MMAs were issued (the same in every thread)
    for (int k = 0; k < R - 1; ++k) {
        if (k < n) load(t_begin + k, k);
        else cp_async_commit();   // empty groups keep the group count per tile fixed
    }
    // tile c's MMAs read buffer c % NBUF and signal bars[c % NBUF]; that is the
    // barrier's (c / NBUF)-th completion, of parity (c / NBUF) & 1
    for (int c = 0; c < n; ++c) {
        const int q = c % NBUF;
        cp_async_wait_group<R - 2>();   // tile c's group landed (R - 2 newer ones may be in flight)
        // the MMAs of tile c - NBUF read buffer q
        const bool ok = c < NBUF || mbar_wait_bounded(&bars[q], (uint32_t)(((c - NBUF) / NBUF) & 1), kWaitNs);
        // every thread's copies of tile c landed, buffer q is free, raw stage (c - 1) % R is free
        failed = __syncthreads_or(!ok) != 0;
        if (failed) break;
        if (c + R - 1 < n) load(t_begin + c + R - 1, (c + R - 1) % R);
        else cp_async_commit();
        build(c % R, q);
        fence_async_smem();   // the generic-proxy stores, visible to the MMAs
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t ab = sbase + q * L.buf_bytes, bb = ab + L.a_bytes;
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const uint64_t ad = smem_desc(ab + ks * 256, 128, 128 * 16);
#pragma unroll
                for (int j = 0; j < NCH; ++j) {
                    const uint64_t bd = smem_desc(bb + j * WG_PLANES_BYTES + ks * 256, 128, 128 * 16);
                    mma_bf16(tmem + j * 9 * WG_NC, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
                }
            }
            mma_commit(&bars[q]);
        }
        last = c;
    }
    if (!failed && last >= 0) {
        const bool ok = mbar_wait_bounded(&bars[last % NBUF], (uint32_t)((last / NBUF) & 1), kWaitNs);
        failed = __syncthreads_or(!ok) != 0;
    }
    if (failed) {
        if (tid == 0) atomicExch(a.err, 1);
        cp_async_wait_group<0>();   // copies in flight
        if (last >= 0)              // the MMAs in flight (they complete in order)
            mbar_wait_bounded(&bars[last % NBUF], (uint32_t)((last / NBUF) & 1), kWaitNs);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) {
            tc_fence_after();
            tmem_dealloc(tmem, TMEM_COLS);
        }
        return;
    }
    cp_async_wait_group<0>();   // the trailing empty groups
    tc_fence_after();
    if (n > 0) {
        // D[co][n], n = tap * 16 + channel: TMEM lane = co; warps w and w + 4
        // read lanes 32 (w % 4) .. + 31, the even and the odd (chunk, tap) columns
        const int quarter = warp & 3;
        const int co = co0 + quarter * 32 + lane;
#pragma unroll 1
        for (int qq = warp >> 2; qq < 9 * NCH; qq += 2) {   // (chunk, tap)
            const int j = qq / 9, t = qq - 9 * j;
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + qq * WG_NC, v);
            if (co < cout) {
                float *dst = a.dW + ((size_t)co * cin + ci0 + WG_NC * j) * 9 + t;
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(dst + 9 * i, v[i]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// One launch over `groups` channel groups of NCH chunks from input channel
// a.ci_base on, in one wave of `per_sm` CTAs per SM (the buffers fill an SM's
// shared memory): the CTAs of every (group, output block) split the tiles
// evenly, at most per_sm * kSMs CTAs in all (a last wave of a few CTAs would
// cost a whole run of tiles).
template <int NCH, int R>
int launch_wgrad_tc_t(WgArgs a, int groups, int coblocks, int per_sm, cudaStream_t st)
{
    const WgLayout L = wg_layout(NCH, R, std::min(a.cout, 128) >> 3);
    const int xctas = std::max(1, per_sm * kSMs / (groups * coblocks));
    a.tiles_per_cta = ceil_div(a.n_tiles, xctas);
    auto kernel = wgrad_tc_kernel<NCH, R>;
    MVS_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, L.bytes));
    MVS_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
    const int ctas = ceil_div(a.n_tiles, a.tiles_per_cta);
    kernel<<<dim3(ctas, groups, coblocks), WG_TC_THREADS, L.bytes, st>>>(a);
    return MVS_OK;
}

// Shared memory one CTA may use at `per_sm` CTAs per SM.
inline int wg_limit(int per_sm) { return per_sm == 1 ? WG_SMEM_MAX : WG_SMEM_SM / per_sm - 1024; }

// The deepest raw ring that fits (at most 8 stages), or 0.
inline int wg_stages(int nch, int cg, int per_sm)
{
    for (int r = 8; r >= 2; --r)
        if (wg_layout(nch, r, cg).bytes <= wg_limit(per_sm)) return r;
    return 0;
}

template <int NCH>
int launch_wgrad_tc_n(WgArgs a, int groups, int coblocks, int per_sm, cudaStream_t st)
{
    switch (wg_stages(NCH, std::min(a.cout, 128) >> 3, per_sm)) {
    case 8: return launch_wgrad_tc_t<NCH, 8>(a, groups, coblocks, per_sm, st);
    case 7: return launch_wgrad_tc_t<NCH, 7>(a, groups, coblocks, per_sm, st);
    case 6: return launch_wgrad_tc_t<NCH, 6>(a, groups, coblocks, per_sm, st);
    case 5: return launch_wgrad_tc_t<NCH, 5>(a, groups, coblocks, per_sm, st);
    case 4: return launch_wgrad_tc_t<NCH, 4>(a, groups, coblocks, per_sm, st);
    case 3: return launch_wgrad_tc_t<NCH, 3>(a, groups, coblocks, per_sm, st);
    case 2: return launch_wgrad_tc_t<NCH, 2>(a, groups, coblocks, per_sm, st);
    default: return set_error(MVS_ERR_ARG, "wgrad: %d chunks do not fit", NCH);
    }
}

int launch_wgrad_tc(const bf16 *x, int cin, const bf16 *dz, int cout, int B, int H, int W, float *dW, int *err,
                    cudaStream_t st)
{
    if (cout % 8 || cin % WG_NC) return set_error(MVS_ERR_ARG, "wgrad: cin %d, cout %d", cin, cout);
    WgArgs a{x, dz, dW, err, B, H, W, cin, cout, ceil_div(W, TW), ceil_div(H, TH), 1, 0, 0};
    a.n_tiles = B * a.tiles_x * a.tiles_y;
    const int chunks = cin / WG_NC, coblocks = ceil_div(cout, 128);
    const int cg = std::min(cout, 128) >> 3;
    // Two CTAs per SM, one chunk each, where one chunk's buffers and at least
    // three raw stages fit in half an SM (16 output channels): the two CTAs'
    // barrier-separated phases overlap.  Otherwise one CTA per SM: pairs of
    // 16-channel chunks share a staged dz tile where two chunks' buffers and
    // two raw stages fit, and an odd chunk runs alone.  (A single MMA buffer
    // to fit two CTAs per SM at 32 and 64 output channels measured no faster.)
    if (wg_stages(1, cg, 2) >= 3) return launch_wgrad_tc_n<1>(a, chunks, coblocks, 2, st);
    const bool pairs = chunks >= 2 && wg_stages(2, cg, 1) >= 2;
    if (pairs)
        if (int rc = launch_wgrad_tc_n<2>(a, chunks / 2, coblocks, 1, st)) return rc;
    const int first = pairs ? chunks & ~1 : 0;
    if (first < chunks) {
        a.ci_base = first * WG_NC;
        if (int rc = launch_wgrad_tc_n<1>(a, chunks - first, coblocks, 1, st)) return rc;
    }
    return MVS_OK;
}

// ---------------------------------------------------------------------------
// weight gradient (CUDA cores, FP32): dW[co][ci][t] += sum_p x[p + off_t][ci] dz[p][co]
// (the reference formulation the tensor-core kernel is tested against)
// ---------------------------------------------------------------------------

constexpr int WG_THREADS = 256;

// Each thread owns a 4 (ci) x 4 (co) block of one tap; a CTA covers a
// TCI x TCO tile of one tap, G = 256 / ((TCI/4)(TCO/4)) thread groups split
// the CTA's pixels, and the groups' sums meet in shared memory before one
// atomic add per weight.
template <int TCI, int TCO>
__global__ void __launch_bounds__(WG_THREADS) wgrad_kernel(const bf16 *__restrict__ x, const bf16 *__restrict__ dz,
                                                           int B, int H, int W, int cin, int cout, int px_per_cta,
                                                           float *__restrict__ dW)
{
    constexpr int TPG = (TCI / 4) * (TCO / 4);   // threads per group
    constexpr int G = WG_THREADS / TPG;
    __shared__ float red[WG_THREADS][17];
    const int tid = threadIdx.x, g = tid / TPG, r = tid - g * TPG;
    const int ci4 = (r % (TCI / 4)) * 4, co4 = (r / (TCI / 4)) * 4;
    const int t = blockIdx.y, ky = t / 3, kx = t - 3 * ky;
    const int ntile_ci = cin / TCI;
    const int ci0 = (blockIdx.z % ntile_ci) * TCI + ci4, co0 = (blockIdx.z / ntile_ci) * TCO + co4;
    const long long npix = (long long)B * H * W;
    const long long p0 = (long long)blockIdx.x * px_per_cta;
    const long long p1 = min(p0 + px_per_cta, npix);
    float acc[4][4] = {};
    for (long long p = p0 + g; p < p1; p += G) {
        const int bb = (int)(p / ((long long)H * W));
        const int rem = (int)(p - (long long)bb * H * W);
        const int y = rem / W, xx = rem - y * W;
        const int sy = y + ky - 1, sx = xx + kx - 1;
        if (sy < 0 || sy >= H || sx < 0 || sx >= W) continue;
        const uint2 xv = *(const uint2 *)(x + (((size_t)bb * H + sy) * W + sx) * cin + ci0);
        const uint2 dv = *(const uint2 *)(dz + (size_t)p * cout + co0);
        const float xf[4] = {bf2f((uint16_t)(xv.x & 0xffffu)), bf2f((uint16_t)(xv.x >> 16)),
                             bf2f((uint16_t)(xv.y & 0xffffu)), bf2f((uint16_t)(xv.y >> 16))};
        const float df[4] = {bf2f((uint16_t)(dv.x & 0xffffu)), bf2f((uint16_t)(dv.x >> 16)),
                             bf2f((uint16_t)(dv.y & 0xffffu)), bf2f((uint16_t)(dv.y >> 16))};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(xf[i], df[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) red[tid][4 * i + j] = acc[i][j];
    __syncthreads();
    if (g == 0) {
        for (int q = 1; q < G; ++q)
#pragma unroll
            for (int k = 0; k < 16; ++k) red[tid][k] += red[q * TPG + r][k];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) atomicAdd(&dW[((size_t)(co0 + j) * cin + ci0 + i) * 9 + t], red[tid][4 * i + j]);
    }
}

// bias gradient: db[co] += sum_p dz[p][co]
__global__ void bgrad_kernel(const bf16 *__restrict__ dz, long long npix, int cout, int px_per_cta,
                             float *__restrict__ db)
{
    __shared__ float red[256];
    const int tid = threadIdx.x;
    const int lanes = 256 / cout * cout;   // threads used: a multiple of cout
    float s = 0.f;
    if (tid < lanes) {
        const int co = tid % cout, row = tid / cout, rows = lanes / cout;
        const long long p0 = (long long)blockIdx.x * px_per_cta;
        const long long p1 = min(p0 + px_per_cta, npix);
        for (long long p = p0 + row; p < p1; p += rows) s += bf2f(dz[(size_t)p * cout + co]);
    }
    red[tid] = s;
    __syncthreads();
    if (tid < cout) {
        float t = 0.f;
        for (int k = tid; k < lanes; k += cout) t += red[k];
        atomicAdd(&db[tid], t);
    }
}

int launch_wgrad_cuda_cores(const bf16 *x, int cin, const bf16 *dz, int cout, int B, int H, int W, float *dW,
                            cudaStream_t st);

int launch_wgrad(const bf16 *x, int cin, const bf16 *dz, int cout, int B, int H, int W, float *dW, float *db, int *err,
                 cudaStream_t st, bool tensor_cores = true)
{
    const long long npix = (long long)B * H * W;
    if (tensor_cores) {
        MVS_RC_(launch_wgrad_tc(x, cin, dz, cout, B, H, W, dW, err, st));
    } else {
        MVS_RC_(launch_wgrad_cuda_cores(x, cin, dz, cout, B, H, W, dW, st));
    }
    if (db) bgrad_kernel<<<(int)((npix + 2047) / 2048), 256, 0, st>>>(dz, npix, cout, 2048, db);
    return MVS_OK;
}

int launch_wgrad_cuda_cores(const bf16 *x, int cin, const bf16 *dz, int cout, int B, int H, int W, float *dW,
                            cudaStream_t st)
{
    const long long npix = (long long)B * H * W;
    const int px = 4096;
    const int chunks = (int)((npix + px - 1) / px);
    const int tci = cin % 64 == 0 ? 64 : cin % 32 == 0 ? 32 : 16;
    const int tco = cout % 64 == 0 ? 64 : cout % 32 == 0 ? 32 : 16;
    const dim3 g(chunks, 9, (cin / tci) * (cout / tco));
#define MVS_WG(A, B_)                                                                              \
    if (tci == A && tco == B_) wgrad_kernel<A, B_><<<g, WG_THREADS, 0, st>>>(x, dz, B, H, W, cin, cout, px, dW); \
    else
    MVS_WG(16, 16) MVS_WG(16, 32) MVS_WG(16, 64) MVS_WG(32, 16) MVS_WG(32, 32) MVS_WG(32, 64) MVS_WG(64, 16)
    MVS_WG(64, 32) MVS_WG(64, 64) return set_error(MVS_ERR_ARG, "wgrad tile %dx%d", tci, tco);
#undef MVS_WG
    return MVS_OK;
}

// ---------------------------------------------------------------------------
// elementwise layers (8 channels = 16 bytes per thread)
// ---------------------------------------------------------------------------

__device__ __forceinline__ void unpack8(const uint4 &q, float (&f)[8])
{
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        f[2 * k] = bf2f((uint16_t)(w[k] & 0xffffu));
        f[2 * k + 1] = bf2f((uint16_t)(w[k] >> 16));
    }
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8])
{
    return make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                      pack_bf16x2(f[6], f[7]));
}

// 2x2 average pool: out [B][H/2][W/2][C]
__global__ void pool_kernel(const bf16 *__restrict__ in, int B, int H, int W, int C, bf16 *__restrict__ out)
{
    const int C8 = C >> 3, Ho = H >> 1, Wo = W >> 1;
    const long long n = (long long)B * Ho * Wo * C8;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(k % C8);
        const long long q = k / C8;
        const int x = (int)(q % Wo), y = (int)((q / Wo) % Ho), b = (int)(q / ((long long)Wo * Ho));
        float s[8] = {}, f[8];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int yy = 2 * y + (d >> 1), xx = 2 * x + (d & 1);
            unpack8(*(const uint4 *)(in + (((size_t)b * H + yy) * W + xx) * C + 8 * c8), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) s[j] += f[j];
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] *= 0.25f;
        *(uint4 *)(out + (size_t)k * 8) = pack8(s);
    }
}

// gradient into an encoder output e (C channels, H x W) from the pool that read
// it (dp, H/2 x W/2) and from the skip half of a concat gradient (dc with
// ctot channels, the skip starting at coff), masked by e > 0
__global__ void pool_back_kernel(const bf16 *__restrict__ dp, const bf16 *__restrict__ dc, int ctot, int coff,
                                 const bf16 *__restrict__ e, int B, int H, int W, int C, bf16 *__restrict__ de)
{
    const int C8 = C >> 3;
    const long long n = (long long)B * H * W * C8;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(k % C8);
        const long long p = k / C8;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
        float g[8], f[8], m[8];
        unpack8(*(const uint4 *)(dp + (((size_t)b * (H >> 1) + (y >> 1)) * (W >> 1) + (x >> 1)) * C + 8 * c8), g);
#pragma unroll
        for (int j = 0; j < 8; ++j) g[j] *= 0.25f;
        if (dc) {
            unpack8(*(const uint4 *)(dc + (size_t)p * ctot + coff + 8 * c8), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) g[j] += f[j];
        }
        unpack8(*(const uint4 *)(e + (size_t)p * C + 8 * c8), m);
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (!(m[j] > 0.f)) g[j] = 0.f;
        *(uint4 *)(de + (size_t)p * C + 8 * c8) = pack8(g);
    }
}

// concat(nearest-upsampled prev (cp channels, H/2 x W/2), skip (cs channels))
__global__ void upcat_kernel(const bf16 *__restrict__ prev, int cp, const bf16 *__restrict__ skip, int cs, int B,
                             int H, int W, bf16 *__restrict__ out)
{
    const int ct8 = (cp + cs) >> 3;
    const long long n = (long long)B * H * W * ct8;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(k % ct8);
        const long long p = k / ct8;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
        const int c = 8 * c8;
        uint4 v;
        if (c < cp)
            v = *(const uint4 *)(prev + (((size_t)b * (H >> 1) + (y >> 1)) * (W >> 1) + (x >> 1)) * cp + c);
        else
            v = *(const uint4 *)(skip + (size_t)p * cs + (c - cp));
        *(uint4 *)(out + (size_t)k * 8) = v;
    }
}

// gradient of the upsampled half: dprev[y][x] = sum of the 2x2 block of dc
// (already masked by the concat's ReLU mask, which is prev's)
__global__ void upcat_back_kernel(const bf16 *__restrict__ dc, int ctot, int B, int H, int W, int cp,
                                  bf16 *__restrict__ dprev)
{
    const int C8 = cp >> 3, Hp = H >> 1, Wp = W >> 1;
    const long long n = (long long)B * Hp * Wp * C8;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int c8 = (int)(k % C8);
        const long long q = k / C8;
        const int x = (int)(q % Wp), y = (int)((q / Wp) % Hp), b = (int)(q / ((long long)Wp * Hp));
        float s[8] = {}, f[8];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const int yy = 2 * y + (d >> 1), xx = 2 * x + (d & 1);
            unpack8(*(const uint4 *)(dc + (((size_t)b * H + yy) * W + xx) * ctot + 8 * c8), f);
#pragma unroll
            for (int j = 0; j < 8; ++j) s[j] += f[j];
        }
        *(uint4 *)(dprev + (size_t)k * 8) = pack8(s);
    }
}

// ---------------------------------------------------------------------------
// input features, prediction head and loss
// ---------------------------------------------------------------------------

struct Norm {
    float depth_scale, depth_shift;   // channel 0 = depth * scale + shift
    float cost_clip;                  // channel 1 = 1 - min(cost, clip)
    float u_scale, v_scale;           // u = wta + u_scale * out0, v = v_scale * out{1,2}
    float w_u, w_v;                   // loss weights of (u - u*)^2 and |v - v*|^2
};

__global__ void features_kernel(const float *__restrict__ wta, const float *__restrict__ cost,
                                const float *__restrict__ ref255, long long npix, Norm nm, bf16 *__restrict__ x0)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        float d = wta[p];
        if (!(d == d)) d = 0.f;
        float c = cost ? cost[p] : 0.f;
        if (!(c == c)) c = nm.cost_clip;
        float f[8] = {d * nm.depth_scale + nm.depth_shift, 1.f - fminf(fmaxf(c, 0.f), nm.cost_clip),
                      ref255[p] * (1.f / 255.f) - 0.5f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const float z[8] = {};
        uint4 *o = (uint4 *)(x0 + (size_t)p * 16);
        o[0] = pack8(f);
        o[1] = pack8(z);
    }
}

// u, v from the last decoder activation d (16 channels) by the 1x1 head
__global__ void head_kernel(const bf16 *__restrict__ d, const float *__restrict__ Wh, const float *__restrict__ bh,
                            const float *__restrict__ wta, long long npix, long long img, Norm nm,
                            float *__restrict__ u, float *__restrict__ v)
{
    __shared__ float w[51];
    if (threadIdx.x < 48) w[threadIdx.x] = Wh[threadIdx.x];
    if (threadIdx.x < 3) w[48 + threadIdx.x] = bh[threadIdx.x];
    __syncthreads();
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        float a[16], t[8];
        unpack8(*(const uint4 *)(d + (size_t)p * 16), t);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = t[j];
        unpack8(*(const uint4 *)(d + (size_t)p * 16 + 8), t);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[8 + j] = t[j];
        float o[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float s = w[48 + k];
#pragma unroll
            for (int c = 0; c < 16; ++c) s = fmaf(w[16 * k + c], a[c], s);
            o[k] = s;
        }
        const long long b = p / img, q = p - b * img;
        float dw = wta[p];
        if (!(dw == dw)) dw = 0.f;
        u[p] = dw + nm.u_scale * o[0];
        v[(size_t)b * 2 * img + q] = nm.v_scale * o[1];
        v[(size_t)b * 2 * img + img + q] = nm.v_scale * o[2];
    }
}

// loss = mean_p [w_u (u - u*)^2 + w_v |v - v*|^2] and its gradient down to
// the last decoder activation (masked by its ReLU), the head's weight and bias
// gradients; partial sums per block, one atomic add per quantity.
__global__ void __launch_bounds__(256) head_back_kernel(const bf16 *__restrict__ d, const float *__restrict__ Wh,
                                                        const float *__restrict__ u, const float *__restrict__ v,
                                                        const float *__restrict__ ut, const float *__restrict__ vt,
                                                        long long npix, long long img, Norm nm,
                                                        bf16 *__restrict__ dz, float *__restrict__ dWh,
                                                        float *__restrict__ dbh, double *__restrict__ loss)
{
    __shared__ float w[48];
    __shared__ float red[8][52];
    if (threadIdx.x < 48) w[threadIdx.x] = Wh[threadIdx.x];
    __syncthreads();
    float gw[48] = {}, gb[3] = {};
    double ls = 0.0;
    const float inv_n = 1.f / (float)npix;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        const long long b = p / img, q = p - b * img;
        const size_t iv0 = (size_t)b * 2 * img + q, iv1 = iv0 + img;
        const float eu = u[p] - ut[p], ex = v[iv0] - vt[iv0], ey = v[iv1] - vt[iv1];
        ls += (double)nm.w_u * eu * eu + (double)nm.w_v * (ex * ex + ey * ey);
        const float go[3] = {2.f * nm.w_u * eu * nm.u_scale * inv_n, 2.f * nm.w_v * ex * nm.v_scale * inv_n,
                             2.f * nm.w_v * ey * nm.v_scale * inv_n};
        float a[16], t[8];
        unpack8(*(const uint4 *)(d + (size_t)p * 16), t);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = t[j];
        unpack8(*(const uint4 *)(d + (size_t)p * 16 + 8), t);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[8 + j] = t[j];
        float g[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const float s = go[0] * w[c] + go[1] * w[16 + c] + go[2] * w[32 + c];
            g[c] = a[c] > 0.f ? s : 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) gw[16 * k + c] = fmaf(go[k], a[c], gw[16 * k + c]);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) gb[k] += go[k];
        float g0[8], g1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            g0[j] = g[j];
            g1[j] = g[8 + j];
        }
        uint4 *o = (uint4 *)(dz + (size_t)p * 16);
        o[0] = pack8(g0);
        o[1] = pack8(g1);
    }
    // block reduction of 48 + 3 floats and the loss
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 51; ++k) {
        float s = k < 48 ? gw[k] : gb[k - 48];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][k] = s;
    }
    for (int o = 16; o > 0; o >>= 1) ls += __shfl_down_sync(0xffffffffu, ls, o);
    __shared__ double lred[8];
    if (lane == 0) lred[warp] = ls;
    __syncthreads();
    if (threadIdx.x < 51) {
        float s = 0.f;
        for (int q = 0; q < 8; ++q) s += red[q][threadIdx.x];
        atomicAdd(threadIdx.x < 48 ? &dWh[threadIdx.x] : &dbh[threadIdx.x - 48], s);
    }
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < 8; ++q) s += lred[q];
        atomicAdd(loss, s / (double)npix);
    }
}

// ---------------------------------------------------------------------------
// parameters: FP32 master copy, Adam, bf16 packs for the tensor cores
// ---------------------------------------------------------------------------

__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    }
}

// W [cout][cin][9] (FP32) -> forward pack [9][cin/8][cout][8] and the
// backward-data pack [9][cout/8][cin][8] of the flipped, transposed kernel
__global__ void pack_kernel(const float *__restrict__ Wt, int cin, int cout, bf16 *__restrict__ fwd,
                            bf16 *__restrict__ bwd)
{
    const int n = 9 * cin * cout;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int t = k % 9, ci = (k / 9) % cin, co = k / (9 * cin);
        const uint16_t b = f2bf(Wt[k]);
        fwd[(((size_t)t * (cin >> 3) + (ci >> 3)) * cout + co) * 8 + (ci & 7)] = b;
        if (bwd) bwd[(((size_t)(8 - t) * (cout >> 3) + (co >> 3)) * cin + ci) * 8 + (co & 7)] = b;
    }
}

}  // namespace unet
}  // namespace mvs

// ===========================================================================
// network driver
// ===========================================================================

namespace {

using namespace mvs;
using namespace mvs::unet;

struct ConvLayer {
    int cin, cout;
    size_t w_off, b_off;   // offsets into the FP32 parameter array
    bf16 *wf, *wb;         // packs
};

// layer indices
enum {
    E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, D0A, D0B, NCONV
};

}  // namespace

struct mvs_unet {
    int B, H, W;
    Norm nm;
    ConvLayer L[NCONV];
    size_t n_params, head_w, head_b;
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    bf16 *packs = nullptr;
    // activations (and their gradients, prefixed g)
    bf16 *x0, *e0a, *e0, *p0, *e1a, *e1, *p1, *e2a, *e2, *p2, *e3a, *e3, *c2, *d2a, *d2, *c1, *d1a, *d1, *c0, *d0a, *d0;
    bf16 *gd0, *gd0a, *gc0, *gd1, *gd1a, *gc1, *gd2, *gd2a, *gc2, *ge3, *ge3a, *gp2, *ge2, *ge2a, *gp1, *ge1, *ge1a,
        *gp0, *ge0, *ge0a;
    float *u = nullptr, *v = nullptr;   // predictions
    double *loss = nullptr;
    int *err = nullptr;
    void *act_mem = nullptr;
    long long step = 0;
};

namespace {

int alloc_net(mvs_unet *n)
{
    static const int spec[NCONV][2] = {{16, 16},  {16, 16}, {16, 32}, {32, 32}, {32, 64},  {64, 64}, {64, 128},
                                       {128, 128}, {192, 64}, {64, 64}, {96, 32}, {32, 32}, {48, 16}, {16, 16}};
    size_t off = 0, pack = 0;
    for (int l = 0; l < NCONV; ++l) {
        n->L[l].cin = spec[l][0];
        n->L[l].cout = spec[l][1];
        n->L[l].w_off = off;
        off += (size_t)9 * spec[l][0] * spec[l][1];
        n->L[l].b_off = off;
        off += spec[l][1];
        pack += (size_t)2 * 9 * spec[l][0] * spec[l][1];
    }
    n->head_w = off;
    off += 48;
    n->head_b = off;
    off += 3;
    n->n_params = off;
    MVS_TRY_CUDA(cudaMalloc(&n->params, off * sizeof(float)));
    MVS_TRY_CUDA(cudaMalloc(&n->grads, off * sizeof(float)));
    MVS_TRY_CUDA(cudaMalloc(&n->adam_m, off * sizeof(float)));
    MVS_TRY_CUDA(cudaMalloc(&n->adam_v, off * sizeof(float)));
    MVS_TRY_CUDA(cudaMemset(n->adam_m, 0, off * sizeof(float)));
    MVS_TRY_CUDA(cudaMemset(n->adam_v, 0, off * sizeof(float)));
    MVS_TRY_CUDA(cudaMalloc(&n->packs, pack * sizeof(bf16)));
    bf16 *pp = n->packs;
    for (int l = 0; l < NCONV; ++l) {
        const size_t s = (size_t)9 * n->L[l].cin * n->L[l].cout;
        n->L[l].wf = pp;
        n->L[l].wb = pp + s;
        pp += 2 * s;
    }
    // activations
    const size_t B = n->B, H = n->H, W = n->W;
    auto px = [&](int lvl) { return B * (H >> lvl) * (W >> lvl); };
    struct Item {
        bf16 **p;
        size_t elems;
    };
    std::vector<Item> items = {
        {&n->x0, px(0) * 16},   {&n->e0a, px(0) * 16},  {&n->e0, px(0) * 16},   {&n->p0, px(1) * 16},
        {&n->e1a, px(1) * 32},  {&n->e1, px(1) * 32},   {&n->p1, px(2) * 32},   {&n->e2a, px(2) * 64},
        {&n->e2, px(2) * 64},   {&n->p2, px(3) * 64},   {&n->e3a, px(3) * 128}, {&n->e3, px(3) * 128},
        {&n->c2, px(2) * 192},  {&n->d2a, px(2) * 64},  {&n->d2, px(2) * 64},   {&n->c1, px(1) * 96},
        {&n->d1a, px(1) * 32},  {&n->d1, px(1) * 32},   {&n->c0, px(0) * 48},   {&n->d0a, px(0) * 16},
        {&n->d0, px(0) * 16},   {&n->gd0, px(0) * 16},  {&n->gd0a, px(0) * 16}, {&n->gc0, px(0) * 48},
        {&n->gd1, px(1) * 32},  {&n->gd1a, px(1) * 32}, {&n->gc1, px(1) * 96},  {&n->gd2, px(2) * 64},
        {&n->gd2a, px(2) * 64}, {&n->gc2, px(2) * 192}, {&n->ge3, px(3) * 128}, {&n->ge3a, px(3) * 128},
        {&n->gp2, px(3) * 64},  {&n->ge2, px(2) * 64},  {&n->ge2a, px(2) * 64}, {&n->gp1, px(2) * 32},
        {&n->ge1, px(1) * 32},  {&n->ge1a, px(1) * 32}, {&n->gp0, px(1) * 16},  {&n->ge0, px(0) * 16},
        {&n->ge0a, px(0) * 16}};
    size_t bytes = 0;
    for (auto &it : items) bytes += (it.elems * sizeof(bf16) + 255) / 256 * 256;
    const size_t fbytes = (B * H * W * 3 * sizeof(float) + 255) / 256 * 256;
    MVS_TRY_CUDA(cudaMalloc(&n->act_mem, bytes + fbytes + 256));
    char *q = (char *)n->act_mem;
    for (auto &it : items) {
        *it.p = (bf16 *)q;
        q += (it.elems * sizeof(bf16) + 255) / 256 * 256;
    }
    n->u = (float *)q;
    n->v = n->u + B * H * W;
    q += fbytes;
    n->loss = (double *)q;
    n->err = (int *)(q + 8);
    MVS_TRY_CUDA(cudaMemset(q, 0, 256));
    return MVS_OK;
}

int repack(mvs_unet *n, cudaStream_t st)
{
    for (int l = 0; l < NCONV; ++l) {
        const ConvLayer &c = n->L[l];
        const int cnt = 9 * c.cin * c.cout;
        pack_kernel<<<ceil_div(cnt, 256), 256, 0, st>>>(n->params + c.w_off, c.cin, c.cout, c.wf, l == E0A ? nullptr : c.wb);
    }
    return check_launch("unet weight pack");
}

#define MVS_RC(x)                 \
    do {                          \
        int rc__ = (x);           \
        if (rc__) return rc__;    \
    } while (0)

inline int grid_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 16LL * kSMs); }

int conv_fwd(mvs_unet *n, int l, const bf16 *in, bf16 *out, int lvl, cudaStream_t st)
{
    const ConvLayer &c = n->L[l];
    return launch_conv(in, c.cin, c.wf, n->params + c.b_off, nullptr, out, c.cout, n->B, n->H >> lvl, n->W >> lvl, 1,
                       n->err, st);
}

int forward(mvs_unet *n, const float *wta, const float *cost, const float *ref255, cudaStream_t st)
{
    const long long npix = (long long)n->B * n->H * n->W;
    features_kernel<<<grid_for(npix), 256, 0, st>>>(wta, cost, ref255, npix, n->nm, n->x0);
    const int B = n->B, H = n->H, W = n->W;
    auto pool = [&](const bf16 *in, int lvl, int C, bf16 *out) {
        const long long m = (long long)B * (H >> (lvl + 1)) * (W >> (lvl + 1)) * (C / 8);
        pool_kernel<<<grid_for(m), 256, 0, st>>>(in, B, H >> lvl, W >> lvl, C, out);
    };
    auto upcat = [&](const bf16 *prev, int cp, const bf16 *skip, int cs, int lvl, bf16 *out) {
        const long long m = (long long)B * (H >> lvl) * (W >> lvl) * ((cp + cs) / 8);
        upcat_kernel<<<grid_for(m), 256, 0, st>>>(prev, cp, skip, cs, B, H >> lvl, W >> lvl, out);
    };
    MVS_RC(conv_fwd(n, E0A, n->x0, n->e0a, 0, st));
    MVS_RC(conv_fwd(n, E0B, n->e0a, n->e0, 0, st));
    pool(n->e0, 0, 16, n->p0);
    MVS_RC(conv_fwd(n, E1A, n->p0, n->e1a, 1, st));
    MVS_RC(conv_fwd(n, E1B, n->e1a, n->e1, 1, st));
    pool(n->e1, 1, 32, n->p1);
    MVS_RC(conv_fwd(n, E2A, n->p1, n->e2a, 2, st));
    MVS_RC(conv_fwd(n, E2B, n->e2a, n->e2, 2, st));
    pool(n->e2, 2, 64, n->p2);
    MVS_RC(conv_fwd(n, E3A, n->p2, n->e3a, 3, st));
    MVS_RC(conv_fwd(n, E3B, n->e3a, n->e3, 3, st));
    upcat(n->e3, 128, n->e2, 64, 2, n->c2);
    MVS_RC(conv_fwd(n, D2A, n->c2, n->d2a, 2, st));
    MVS_RC(conv_fwd(n, D2B, n->d2a, n->d2, 2, st));
    upcat(n->d2, 64, n->e1, 32, 1, n->c1);
    MVS_RC(conv_fwd(n, D1A, n->c1, n->d1a, 1, st));
    MVS_RC(conv_fwd(n, D1B, n->d1a, n->d1, 1, st));
    upcat(n->d1, 32, n->e0, 16, 0, n->c0);
    MVS_RC(conv_fwd(n, D0A, n->c0, n->d0a, 0, st));
    MVS_RC(conv_fwd(n, D0B, n->d0a, n->d0, 0, st));
    head_kernel<<<grid_for(npix), 256, 0, st>>>(n->d0, n->params + n->head_w, n->params + n->head_b, wta, npix,
                                                (long long)H * W, n->nm, n->u, n->v);
    return check_launch("unet forward");
}

// backward of conv layer l: dz = gradient at its (pre-ReLU-masked) output;
// weight/bias gradients from its input x; dx (optional) masked by x > 0 when
// mask_x
int conv_bwd(mvs_unet *n, int l, const bf16 *x, const bf16 *dz, bf16 *dx, bool mask_x, int lvl, cudaStream_t st)
{
    const ConvLayer &c = n->L[l];
    const int H = n->H >> lvl, W = n->W >> lvl;
    MVS_RC(launch_wgrad(x, c.cin, dz, c.cout, n->B, H, W, n->grads + c.w_off, n->grads + c.b_off, n->err, st));
    if (dx)
        MVS_RC(launch_conv(dz, c.cout, c.wb, nullptr, mask_x ? x : nullptr, dx, c.cin, n->B, H, W, 0, n->err, st));
    return MVS_OK;
}

int backward(mvs_unet *n, const float *ut, const float *vt, cudaStream_t st)
{
    const int B = n->B, H = n->H, W = n->W;
    const long long npix = (long long)B * H * W;
    MVS_TRY_CUDA(cudaMemsetAsync(n->grads, 0, n->n_params * sizeof(float), st));
    MVS_TRY_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(double), st));
    head_back_kernel<<<std::min<long long>((npix + 255) / 256, 4LL * kSMs), 256, 0, st>>>(
        n->d0, n->params + n->head_w, n->u, n->v, ut, vt, npix, (long long)H * W, n->nm, n->gd0,
        n->grads + n->head_w, n->grads + n->head_b, n->loss);
    auto upback = [&](const bf16 *dc, int ctot, int lvl, int cp, bf16 *dprev) {
        const long long m = (long long)B * (H >> (lvl + 1)) * (W >> (lvl + 1)) * (cp / 8);
        upcat_back_kernel<<<grid_for(m), 256, 0, st>>>(dc, ctot, B, H >> lvl, W >> lvl, cp, dprev);
    };
    auto poolback = [&](const bf16 *dp, const bf16 *dc, int ctot, int coff, const bf16 *e, int lvl, int C, bf16 *de) {
        const long long m = (long long)B * (H >> lvl) * (W >> lvl) * (C / 8);
        pool_back_kernel<<<grid_for(m), 256, 0, st>>>(dp, dc, ctot, coff, e, B, H >> lvl, W >> lvl, C, de);
    };
    // decoder level 0
    MVS_RC(conv_bwd(n, D0B, n->d0a, n->gd0, n->gd0a, true, 0, st));
    MVS_RC(conv_bwd(n, D0A, n->c0, n->gd0a, n->gc0, true, 0, st));
    upback(n->gc0, 48, 0, 32, n->gd1);
    // decoder level 1
    MVS_RC(conv_bwd(n, D1B, n->d1a, n->gd1, n->gd1a, true, 1, st));
    MVS_RC(conv_bwd(n, D1A, n->c1, n->gd1a, n->gc1, true, 1, st));
    upback(n->gc1, 96, 1, 64, n->gd2);
    // decoder level 2
    MVS_RC(conv_bwd(n, D2B, n->d2a, n->gd2, n->gd2a, true, 2, st));
    MVS_RC(conv_bwd(n, D2A, n->c2, n->gd2a, n->gc2, true, 2, st));
    upback(n->gc2, 192, 2, 128, n->ge3);
    // bottleneck
    MVS_RC(conv_bwd(n, E3B, n->e3a, n->ge3, n->ge3a, true, 3, st));
    MVS_RC(conv_bwd(n, E3A, n->p2, n->ge3a, n->gp2, false, 3, st));
    // encoder level 2
    poolback(n->gp2, n->gc2, 192, 128, n->e2, 2, 64, n->ge2);
    MVS_RC(conv_bwd(n, E2B, n->e2a, n->ge2, n->ge2a, true, 2, st));
    MVS_RC(conv_bwd(n, E2A, n->p1, n->ge2a, n->gp1, false, 2, st));
    // encoder level 1
    poolback(n->gp1, n->gc1, 96, 64, n->e1, 1, 32, n->ge1);
    MVS_RC(conv_bwd(n, E1B, n->e1a, n->ge1, n->ge1a, true, 1, st));
    MVS_RC(conv_bwd(n, E1A, n->p0, n->ge1a, n->gp0, false, 1, st));
    // encoder level 0
    poolback(n->gp0, n->gc0, 48, 32, n->e0, 0, 16, n->ge0);
    MVS_RC(conv_bwd(n, E0B, n->e0a, n->ge0, n->ge0a, true, 0, st));
    MVS_RC(conv_bwd(n, E0A, n->x0, n->ge0a, nullptr, false, 0, st));
    return check_launch("unet backward");
}

int read_err(mvs_unet *n, cudaStream_t st)
{
    int e = 0;
    MVS_TRY_CUDA(cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MVS_TRY_CUDA(cudaStreamSynchronize(st));
    if (e) return set_error(MVS_ERR_TIMEOUT, "unet: a tensor-core wait gave up");
    return MVS_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int mvs_unet_create(mvs_unet **out, int32_t batch, int32_t height, int32_t width, const float *norm7)
{
    if (!out) return set_error(MVS_ERR_ARG, "null output");
    *out = nullptr;
    if (batch <= 0 || height <= 0 || width <= 0 || height % 8 || width % 8)
        return set_error(MVS_ERR_ARG, "unet needs batch > 0 and height, width multiples of 8 (got %d, %dx%d)", batch,
                         width, height);
    mvs_unet *n = new mvs_unet();
    n->B = batch;
    n->H = height;
    n->W = width;
    const float def[7] = {0.25f, -1.f, 2.f, 1.f, 0.01f, 1.f, 1.f};
    const float *s = norm7 ? norm7 : def;
    n->nm = Norm{s[0], s[1], s[2], s[3], s[4], s[5], s[6]};
    int rc = alloc_net(n);
    if (rc) {
        mvs_unet_destroy(n);
        return rc;
    }
    *out = n;
    return MVS_OK;
}

int mvs_unet_destroy(mvs_unet *n)
{
    if (!n) return MVS_OK;
    cudaFree(n->params);
    cudaFree(n->grads);
    cudaFree(n->adam_m);
    cudaFree(n->adam_v);
    cudaFree(n->packs);
    cudaFree(n->act_mem);
    delete n;
    return MVS_OK;
}

int64_t mvs_unet_param_count(const mvs_unet *n) { return n ? (int64_t)n->n_params : 0; }

int mvs_unet_layer_info(const mvs_unet *n, int32_t layer, int32_t *cin, int32_t *cout, int64_t *w_off, int64_t *b_off)
{
    if (!n || layer < 0 || layer > NCONV) return set_error(MVS_ERR_ARG, "layer %d", layer);
    if (layer == NCONV) {   // the 1x1 head
        if (cin) *cin = 16;
        if (cout) *cout = 3;
        if (w_off) *w_off = (int64_t)n->head_w;
        if (b_off) *b_off = (int64_t)n->head_b;
        return MVS_OK;
    }
    if (cin) *cin = n->L[layer].cin;
    if (cout) *cout = n->L[layer].cout;
    if (w_off) *w_off = (int64_t)n->L[layer].w_off;
    if (b_off) *b_off = (int64_t)n->L[layer].b_off;
    return MVS_OK;
}

int mvs_unet_set_params(mvs_unet *n, const float *h_params)
{
    if (!n || !h_params) return set_error(MVS_ERR_ARG, "null argument");
    MVS_TRY_CUDA(cudaMemcpy(n->params, h_params, n->n_params * sizeof(float), cudaMemcpyHostToDevice));
    MVS_TRY_CUDA(cudaMemset(n->adam_m, 0, n->n_params * sizeof(float)));
    MVS_TRY_CUDA(cudaMemset(n->adam_v, 0, n->n_params * sizeof(float)));
    n->step = 0;
    MVS_RC(repack(n, 0));
    MVS_TRY_CUDA(cudaDeviceSynchronize());
    return MVS_OK;
}

int mvs_unet_get_params(mvs_unet *n, float *h_params, float *h_grads)
{
    if (!n) return set_error(MVS_ERR_ARG, "null net");
    MVS_TRY_CUDA(cudaDeviceSynchronize());
    if (h_params) MVS_TRY_CUDA(cudaMemcpy(h_params, n->params, n->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    if (h_grads) MVS_TRY_CUDA(cudaMemcpy(h_grads, n->grads, n->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    return MVS_OK;
}

int mvs_unet_forward(mvs_unet *n, const float *d_wta, const float *d_cost, const float *d_ref255, float *d_u,
                     float *d_v, void *stream)
{
    if (!n || !d_wta || !d_ref255) return set_error(MVS_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    MVS_RC(forward(n, d_wta, d_cost, d_ref255, st));
    const size_t img = (size_t)n->B * n->H * n->W;
    if (d_u) MVS_TRY_CUDA(cudaMemcpyAsync(d_u, n->u, img * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (d_v) MVS_TRY_CUDA(cudaMemcpyAsync(d_v, n->v, 2 * img * sizeof(float), cudaMemcpyDeviceToDevice, st));
    return MVS_OK;
}

int mvs_unet_backward(mvs_unet *n, const float *d_u_target, const float *d_v_target, double *loss_out, void *stream)
{
    if (!n || !d_u_target || !d_v_target) return set_error(MVS_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    MVS_RC(backward(n, d_u_target, d_v_target, st));
    if (loss_out) {
        MVS_TRY_CUDA(cudaMemcpyAsync(loss_out, n->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        MVS_RC(read_err(n, st));
    }
    return MVS_OK;
}

int mvs_unet_adam_step(mvs_unet *n, float lr, float beta1, float beta2, float eps, void *stream)
{
    if (!n) return set_error(MVS_ERR_ARG, "null net");
    cudaStream_t st = (cudaStream_t)stream;
    n->step += 1;
    const float c1 = 1.f - powf(beta1, (float)n->step), c2 = 1.f - powf(beta2, (float)n->step);
    adam_kernel<<<grid_for((long long)n->n_params), 256, 0, st>>>(n->params, n->grads, n->adam_m, n->adam_v,
                                                                  (long long)n->n_params, lr, beta1, beta2, eps, c1,
                                                                  c2);
    MVS_RC(repack(n, st));
    return MVS_OK;
}

int mvs_unet_train_step(mvs_unet *n, const float *d_wta, const float *d_cost, const float *d_ref255,
                        const float *d_u_target, const float *d_v_target, float lr, double *loss_out, void *stream)
{
    MVS_RC(mvs_unet_forward(n, d_wta, d_cost, d_ref255, nullptr, nullptr, stream));
    MVS_RC(mvs_unet_backward(n, d_u_target, d_v_target, nullptr, stream));
    MVS_RC(mvs_unet_adam_step(n, lr, 0.9f, 0.999f, 1e-8f, stream));
    if (loss_out) {
        cudaStream_t st = (cudaStream_t)stream;
        MVS_TRY_CUDA(cudaMemcpyAsync(loss_out, n->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
        MVS_RC(read_err(n, st));
    }
    return MVS_OK;
}

int mvs_unet_check(mvs_unet *n, void *stream)
{
    if (!n) return set_error(MVS_ERR_ARG, "null net");
    return read_err(n, (cudaStream_t)stream);
}

// single layers, for gradient checks against the CPU restatement
int mvs_conv3x3_forward(const uint16_t *d_in, int32_t cin, const float *d_w, const float *d_bias, int32_t cout,
                        int32_t batch, int32_t height, int32_t width, int32_t relu, uint16_t *d_out,
                        uint16_t *d_wpack, int32_t *d_err, void *stream)
{
    if (!d_in || !d_w || !d_out || !d_wpack || !d_err) return set_error(MVS_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    pack_kernel<<<ceil_div(9 * cin * cout, 256), 256, 0, st>>>(d_w, cin, cout, d_wpack, nullptr);
    MVS_RC(launch_conv(d_in, cin, d_wpack, d_bias, nullptr, d_out, cout, batch, height, width, relu, d_err, st));
    return check_launch("conv3x3 forward");
}

int mvs_conv3x3_backward(const uint16_t *d_x, int32_t cin, const float *d_w, const uint16_t *d_dz, int32_t cout,
                         int32_t batch, int32_t height, int32_t width, int32_t mask_x, uint16_t *d_dx, float *d_dw,
                         float *d_db, uint16_t *d_wpack, int32_t *d_err, int32_t tensor_cores, void *stream)
{
    if (!d_x || !d_w || !d_dz || !d_dw || !d_wpack || !d_err) return set_error(MVS_ERR_ARG, "null argument");
    if (cout % 16 || cin % 16) return set_error(MVS_ERR_ARG, "channels must be multiples of 16");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t s = (size_t)9 * cin * cout;
    pack_kernel<<<ceil_div((int)s, 256), 256, 0, st>>>(d_w, cin, cout, d_wpack, d_wpack + s);
    MVS_RC(launch_wgrad(d_x, cin, d_dz, cout, batch, height, width, d_dw, d_db, d_err, st, tensor_cores != 0));
    if (d_dx)
        MVS_RC(launch_conv(d_dz, cout, d_wpack + s, nullptr, mask_x ? d_x : nullptr, d_dx, cin, batch, height, width,
                           0, d_err, st));
    return check_launch("conv3x3 backward");
}

}  // extern "C"
