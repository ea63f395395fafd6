// Data formats either side of the hot path (host code): the ICL-NUIM camera
// files the reference reads (reader.cpp:181-296) and a PLY writer for the
// fused surface, which the reference shows through PCL (pclviewer.cpp:1058-1083).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "common.cuh"

namespace {

struct V3 {
    float x, y, z;
};

// the float3 helpers the reference's reader uses (length, cross, normalize
// with a host reciprocal square root of 1 / sqrtf)
float length3(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
V3 cross3(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 normalize3(V3 a)
{
    const float inv = 1.0f / sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    return V3{a.x * inv, a.y * inv, a.z * inv};
}

// The text between the last '[' and the last ']' of a line, split at commas
// (Reader::getcamParameters, reader.cpp:252-258); 3 numbers expected.
bool bracket_vector(const char *line, V3 *out)
{
    const char *a = strrchr(line, '['), *b = strrchr(line, ']');
    if (!a || !b || b <= a) return false;
    char buf[512];
    const size_t len = (size_t)(b - a - 1);
    if (len >= sizeof(buf)) return false;
    memcpy(buf, a + 1, len);
    buf[len] = 0;
    double v[3];
    int k = 0;
    for (char *tok = strtok(buf, ","); tok && k < 3; tok = strtok(nullptr, ",")) {
        char *end = nullptr;
        v[k] = strtod(tok, &end);
        if (end == tok) return false;
        ++k;
    }
    if (k != 3) return false;
    *out = V3{(float)v[0], (float)v[1], (float)v[2]};   // Vector3D holds floats
    return true;
}

}  // namespace

extern "C" {

int mvs_read_icl_camera(const char *path, int32_t width, int32_t height, float *K9, float *R9, float *t3)
{
    using namespace mvs;
    if (!path || !K9 || !R9 || !t3) return set_error(MVS_ERR_ARG, "null argument");
    FILE *f = fopen(path, "r");
    if (!f) return set_error(MVS_ERR_ARG, "cannot open %s", path);
    V3 pos{}, dir{}, up{}, right{};
    int have = 0;
    char line[1024];
    while (fgets(line, sizeof(line), f)) {
        // keys as the reader matches them: the line starts with the key (reader.cpp:261-288)
        V3 v;
        if (!strncmp(line, "cam_pos", 7) && bracket_vector(line, &v)) {
            pos = v;
            have |= 1;
        } else if (!strncmp(line, "cam_dir", 7) && bracket_vector(line, &v)) {
            dir = v;
            have |= 2;
        } else if (!strncmp(line, "cam_up", 6) && bracket_vector(line, &v)) {
            up = v;
            have |= 4;
        } else if (!strncmp(line, "cam_right", 9) && bracket_vector(line, &v)) {
            right = v;
            have |= 8;
        }
    }
    fclose(f);
    if (have != 15) return set_error(MVS_ERR_ARG, "%s: cam_pos, cam_dir, cam_up and cam_right are required", path);
    // Reader::getcamK (reader.cpp:181-207): focal and aspect from the camera
    // vectors, pixel sizes for width x height, 1-based principal point, negative fy
    const double focal = length3(dir);
    double aspect = length3(right);
    const double angle = 2 * atan(aspect / 2 / focal);
    aspect = aspect / length3(up);
    double psx = 2 * focal * tan(0.5 * angle) / width;
    double psy = 2 * focal * tan(0.5 * angle) / aspect / height;
    psx = psx / focal;
    psy = psy / focal;
    const double Ox = (width + 1) * 0.5, Oy = (height + 1) * 0.5;
    const float K[9] = {(float)(1.f / psx), 0.f, (float)Ox, 0.f, (float)(-1.f / psy), (float)Oy, 0.f, 0.f, 1.f};
    memcpy(K9, K, sizeof(K));
    // Reader::computeRT (reader.cpp:209-225): rows x, y, z of the camera, transposed
    const float flen = length3(dir);   // z = cam_dir / length(cam_dir), in float
    const V3 z = V3{dir.x / flen, dir.y / flen, dir.z / flen};
    const V3 x = normalize3(cross3(up, z));
    const V3 y = cross3(z, x);
    const float R[9] = {x.x, y.x, z.x, x.y, y.y, z.y, x.z, y.z, z.z};
    memcpy(R9, R, sizeof(R));
    t3[0] = pos.x;
    t3[1] = pos.y;
    t3[2] = pos.z;
    return MVS_OK;
}

int mvs_write_ply(const char *path, const float *xyz, const uint8_t *rgb, int64_t n, int32_t binary)
{
    using namespace mvs;
    if (!path || (n > 0 && !xyz) || n < 0) return set_error(MVS_ERR_ARG, "bad point cloud");
    FILE *f = fopen(path, binary ? "wb" : "w");
    if (!f) return set_error(MVS_ERR_ARG, "cannot write %s", path);
    fprintf(f, "ply\nformat %s 1.0\nelement vertex %lld\nproperty float x\nproperty float y\nproperty float z\n",
            binary ? "binary_little_endian" : "ascii", (long long)n);
    if (rgb) fprintf(f, "property uchar red\nproperty uchar green\nproperty uchar blue\n");
    fprintf(f, "end_header\n");
    bool ok = true;
    for (int64_t i = 0; i < n && ok; ++i) {
        if (binary) {
            ok = fwrite(xyz + 3 * i, sizeof(float), 3, f) == 3;
            if (ok && rgb) ok = fwrite(rgb + 3 * i, 1, 3, f) == 3;
        } else if (rgb) {
            ok = fprintf(f, "%.9g %.9g %.9g %u %u %u\n", xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], rgb[3 * i],
                         rgb[3 * i + 1], rgb[3 * i + 2]) > 0;
        } else {
            ok = fprintf(f, "%.9g %.9g %.9g\n", xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]) > 0;
        }
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? MVS_OK : set_error(MVS_ERR_ARG, "writing %s failed", path);
}

// PCLViewer::RGBdepthmapColor (pclviewer.cpp:1084-1115): blue, light blue,
// yellow, red, dark red bands over 0..255, in unsigned-char arithmetic.
void mvs_depth_color(const uint8_t *gray, int64_t n, uint8_t *rgb)
{
    for (int64_t i = 0; i < n; ++i) {
        const unsigned d = gray[i];
        unsigned char r = 0, g = 0, b = 0;
        if (d < 32) {
            b = (unsigned char)(128 + d * 4);
        } else if (d < 96) {
            g = (unsigned char)((d - 32) * 4);
            b = 255;
        } else if (d < 160) {
            r = (unsigned char)((d - 96) * 4);
            g = 255;
            b = (unsigned char)(255 - r);
        } else if (d < 224) {
            r = 255;
            g = (unsigned char)(255 - (d - 160) * 4);
        } else {
            r = (unsigned char)(255 - (d - 224) * 4);
        }
        rgb[3 * i] = r;
        rgb[3 * i + 1] = g;
        rgb[3 * i + 2] = b;
    }
}

}  // extern "C"
