// Ray caster for the seeded synthetic box scenes (walls, floor, boxes,
// textured with 3-D value noise) that stand in for the reference's datasets
// (ICL-NUIM living room, KITTI; reader.cpp, kitti_reader.cpp), which are not
// shipped with it.  It produces training frames for the depth warm-start
// network and the batched-frame workloads at device speed; the CPU ray caster
// in mvs_b200/scenes.py defines the scenes and is the parity reference.
//
// Everything is FP64, in the CPU caster's order of operations, so both agree
// to the last few bits (the test tolerates rounding-order differences of the
// 3x3 products and lattice cells picked differently at exact cell borders).
#include <math.h>

#include "common.cuh"

namespace mvs {
namespace {

constexpr int kMaxBoxes = 32;
constexpr int kMaxOctaves = 8;

struct SceneArgs {
    double invK[9], R[9], c[3];
    double room_min[3], room_max[3];
    double boxes[kMaxBoxes][6];
    double offsets[kMaxOctaves][3];
    double base_freq;
    int n_boxes, inside_room, lattice, octaves;
};

__device__ __forceinline__ double safe_inv(double d) { return 1.0 / (fabs(d) < 1e-12 ? 1e-12 : d); }

// one octave of the value noise: smoothstep-weighted trilinear blend of the
// 8 lattice corners (periodic lattice)
__device__ double octave(const double *__restrict__ T, int n, double qx, double qy, double qz)
{
    const double fx0 = floor(qx), fy0 = floor(qy), fz0 = floor(qz);
    double fx = qx - fx0, fy = qy - fy0, fz = qz - fz0;
    fx = fx * fx * (3.0 - 2.0 * fx);
    fy = fy * fy * (3.0 - 2.0 * fy);
    fz = fz * fz * (3.0 - 2.0 * fz);
    long long ix = (long long)fx0 % n, iy = (long long)fy0 % n, iz = (long long)fz0 % n;
    if (ix < 0) ix += n;
    if (iy < 0) iy += n;
    if (iz < 0) iz += n;
    const long long jx = (ix + 1) % n, jy = (iy + 1) % n, jz = (iz + 1) % n;
    const long long nn = (long long)n * n;
    const double c000 = T[ix * nn + iy * n + iz], c100 = T[jx * nn + iy * n + iz];
    const double c010 = T[ix * nn + jy * n + iz], c110 = T[jx * nn + jy * n + iz];
    const double c001 = T[ix * nn + iy * n + jz], c101 = T[jx * nn + iy * n + jz];
    const double c011 = T[ix * nn + jy * n + jz], c111 = T[jx * nn + jy * n + jz];
    const double c00 = c000 + fx * (c100 - c000);
    const double c10 = c010 + fx * (c110 - c010);
    const double c01 = c001 + fx * (c101 - c001);
    const double c11 = c011 + fx * (c111 - c011);
    const double c0 = c00 + fy * (c10 - c00);
    const double c1 = c01 + fy * (c11 - c01);
    return c0 + fz * (c1 - c0);
}

__global__ void render_kernel(SceneArgs s, const double *__restrict__ table, int w, int h,
                              float *__restrict__ gray255, float *__restrict__ depth)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    // camera ray through the pixel (z == 1 in the camera frame), rotated to
    // the world frame: dir = R^T (K^-1 (x, y, 1))
    const double px = x, py = y;
    double rc[3];
    for (int j = 0; j < 3; ++j) rc[j] = px * s.invK[3 * j] + py * s.invK[3 * j + 1] + 1.0 * s.invK[3 * j + 2];
    double d[3];
    for (int j = 0; j < 3; ++j) d[j] = rc[0] * s.R[j] + rc[1] * s.R[3 + j] + rc[2] * s.R[6 + j];
    const double inv[3] = {safe_inv(d[0]), safe_inv(d[1]), safe_inv(d[2])};
    double best = INFINITY;
    if (s.inside_room) {
        double tfar = INFINITY;
        for (int j = 0; j < 3; ++j) {
            const double t1 = (s.room_min[j] - s.c[j]) * inv[j], t2 = (s.room_max[j] - s.c[j]) * inv[j];
            tfar = fmin(tfar, fmax(t1, t2));
        }
        if (tfar > 1e-6) best = tfar;
    }
    for (int b = 0; b < s.n_boxes; ++b) {
        double tnear = -INFINITY, tfar = INFINITY;
        for (int j = 0; j < 3; ++j) {
            const double t1 = (s.boxes[b][j] - s.c[j]) * inv[j], t2 = (s.boxes[b][3 + j] - s.c[j]) * inv[j];
            tnear = fmax(tnear, fmin(t1, t2));
            tfar = fmin(tfar, fmax(t1, t2));
        }
        if (tnear <= tfar && tnear > 1e-6 && tnear < best) best = tnear;
    }
    const bool miss = !(best < INFINITY);
    const double sd = miss ? 50.0 : best;
    const int i = y * w + x;
    depth[i] = (float)sd;
    if (!gray255) return;
    double inten = 0.5;
    if (!miss) {
        const double p[3] = {s.c[0] + d[0] * sd, s.c[1] + d[1] * sd, s.c[2] + d[2] * sd};
        double acc = 0.0, amp = 1.0, freq = s.base_freq, norm = 0.0;
        for (int o = 0; o < s.octaves; ++o) {
            acc += amp * octave(table, s.lattice, p[0] * freq + s.offsets[o][0], p[1] * freq + s.offsets[o][1],
                                p[2] * freq + s.offsets[o][2]);
            norm += amp;
            amp *= 0.5;
            freq *= 2.0;
        }
        inten = acc / norm;
    }
    gray255[i] = (float)(inten * 255.0);
}

}  // namespace
}  // namespace mvs

extern "C" int mvs_render_scene(const mvs_box_scene *sc, const double *h_invK9, const double *h_R9,
                                const double *h_center3, int32_t w, int32_t h, float *d_gray255, float *d_depth,
                                void *stream)
{
    using namespace mvs;
    if (!sc || !h_invK9 || !h_R9 || !h_center3 || !d_depth) return set_error(MVS_ERR_ARG, "null argument");
    if (w <= 0 || h <= 0) return set_error(MVS_ERR_ARG, "bad image size %dx%d", w, h);
    if (sc->n_boxes < 0 || sc->n_boxes > kMaxBoxes) return set_error(MVS_ERR_ARG, "at most %d boxes", kMaxBoxes);
    if (sc->n_boxes > 0 && !sc->h_boxes) return set_error(MVS_ERR_ARG, "null box list");
    if (d_gray255 && (!sc->d_noise || sc->lattice <= 0 || sc->octaves < 1 || sc->octaves > kMaxOctaves))
        return set_error(MVS_ERR_ARG, "noise table needs a lattice > 0 and 1..%d octaves", kMaxOctaves);
    SceneArgs a{};
    for (int k = 0; k < 9; ++k) {
        a.invK[k] = h_invK9[k];
        a.R[k] = h_R9[k];
    }
    // the camera centre is where the rays start
    for (int k = 0; k < 3; ++k) {
        a.c[k] = h_center3[k];
        a.room_min[k] = sc->room_min[k];
        a.room_max[k] = sc->room_max[k];
    }
    for (int b = 0; b < sc->n_boxes; ++b)
        for (int k = 0; k < 6; ++k) a.boxes[b][k] = sc->h_boxes[6 * b + k];
    for (int o = 0; o < kMaxOctaves; ++o)
        for (int k = 0; k < 3; ++k) a.offsets[o][k] = sc->offsets[o][k];
    a.base_freq = sc->base_freq;
    a.n_boxes = sc->n_boxes;
    a.inside_room = sc->inside_room;
    a.lattice = sc->lattice;
    a.octaves = sc->octaves;
    const dim3 b(32, 8), g(ceil_div(w, 32), ceil_div(h, 8));
    render_kernel<<<g, b, 0, (cudaStream_t)stream>>>(a, sc->d_noise, w, h, d_gray255, d_depth);
    return check_launch("render scene");
}
