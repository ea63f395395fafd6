// The C++ fusion drop-in (include/mvs_b200.hpp) driven as the reference's GUI
// drives fusionData (pclviewer.cpp:972-1083): construct fusionData<8> over a
// bounding volume, FusionUpdateIteration<8> per depthmap, then copyTo into
// AoS fusionvoxel<8> rows at a caller pitch (fusion.h:933-947).  Also checks
// the ownership rules of fusion.h:176-182 (a copy shares the storage and does
// not free it) and Resize (fusion.h:298-306: new storage, same volume).
//
//   fusion_dropin <in.bin> <out.bin>
// in.bin : int32 w, h, d, n_maps, map_w, map_h; float a[3], b[3], thr; double tau, lambda, sigma;
//          float depth[n_maps][map_h][map_w], K[n_maps][9], R[n_maps][9], t[n_maps][3]
// out.bin: int32 pitch, then two snapshots of the AoS rows (`pitch` bytes each,
//          h * d rows): after the per-map iterations, and after one more U and
//          P step made once the shallow copies are gone.
// Exit status 0 when every in-program check held.
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "mvs_b200.hpp"

static int fail(const char *what)
{
    std::fprintf(stderr, "fusion_dropin: %s\n", what);
    return 1;
}

int main(int argc, char **argv)
{
    if (argc != 3) return fail("usage: fusion_dropin in.bin out.bin");
    FILE *fi = std::fopen(argv[1], "rb");
    if (!fi) return fail("cannot open input");
    int32_t hdr[6];
    float box[6], thr;
    double prm[3];   // tau, lambda, sigma: doubles, as the FusionUpdate* wrappers take them
    if (std::fread(hdr, 4, 6, fi) != 6 || std::fread(box, 4, 6, fi) != 6 || std::fread(&thr, 4, 1, fi) != 1 ||
        std::fread(prm, 8, 3, fi) != 3)
        return fail("short header");
    const int w = hdr[0], h = hdr[1], d = hdr[2], nm = hdr[3], mw = hdr[4], mh = hdr[5];
    std::vector<float> depth((size_t)nm * mw * mh), K((size_t)nm * 9), R((size_t)nm * 9), t((size_t)nm * 3);
    if (std::fread(depth.data(), 4, depth.size(), fi) != depth.size() || std::fread(K.data(), 4, K.size(), fi) != K.size() ||
        std::fread(R.data(), 4, R.size(), fi) != R.size() || std::fread(t.data(), 4, t.size(), fi) != t.size())
        return fail("short data");
    std::fclose(fi);

    const float3 a = {box[0], box[1], box[2]}, b = {box[3], box[4], box[5]};
    fusionData<8> f(w, h, d, a, b);
    if (!f.valid()) return fail("fusionData construction failed");
    float *d_depth = nullptr;
    if (cudaMalloc(&d_depth, (size_t)mw * mh * 4) != cudaSuccess) return fail("cudaMalloc");
    for (int m = 0; m < nm; ++m) {
        if (cudaMemcpy(d_depth, depth.data() + (size_t)m * mw * mh, (size_t)mw * mh * 4, cudaMemcpyHostToDevice) !=
            cudaSuccess)
            return fail("upload");
        // fusionData is passed by value, as the reference's wrappers take it:
        // the callee's copy shares the storage and must not free it
        FusionUpdateIteration<8>(f, d_depth, Matrix3D(&K[9 * m]), Matrix3D(&R[9 * m]), Vector3D(&t[3 * m]), thr,
                                 prm[0], prm[1], prm[2], mw, mh);
    }
    const size_t pitch = (size_t)w * sizeof(fusionvoxel<8>) + 36;   // not a multiple of the voxel size
    const size_t rows = (size_t)h * d;
    std::vector<unsigned char> buf(2 * rows * pitch, 0xAB);
    f.copyTo(reinterpret_cast<fusionvoxel<8> *>(buf.data()), pitch);
    {
        fusionData<8> g(f);   // shallow copy
        if (g.handle() != f.handle() || g.elements() != f.elements()) return fail("copy does not share the volume");
        fusionData<8> k;
        k = f;                // shallow assignment
        if (k.handle() != f.handle()) return fail("assignment does not share the volume");
    }                          // g, k go out of scope: the storage must survive
    FusionUpdateU<8>(f, prm[0], prm[1]);
    FusionUpdateP<8>(f, prm[2]);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail("CUDA error after the updates");

    f.copyTo(reinterpret_cast<fusionvoxel<8> *>(buf.data() + rows * pitch), pitch);
    for (size_t r = 0; r < 2 * rows; ++r)
        for (size_t k = (size_t)w * sizeof(fusionvoxel<8>); k < pitch; ++k)
            if (buf[r * pitch + k] != 0xAB) return fail("copyTo wrote into the row padding");

    // worldCoords (fusion.h:360-364) and Resize (fusion.h:298-306)
    const float3 c = f.worldCoords(1, 2, 3);
    if (c.x != a.x + (b.x - a.x) * (float)((1 + .5) / w) || c.z != a.z + (b.z - a.z) * (float)((3 + .5) / d))
        return fail("worldCoords");
    fusionData<8> r(4, 3, 2, a, b);
    r.Resize(5, 4, 3);
    if (!r.valid() || r.elements() != 60 || r.volume().b.x != b.x || r.volume().a.z != a.z)
        return fail("Resize");

    FILE *fo = std::fopen(argv[2], "wb");
    if (!fo) return fail("cannot open output");
    const int32_t p32 = (int32_t)pitch;
    std::fwrite(&p32, 4, 1, fo);
    std::fwrite(buf.data(), 1, buf.size(), fo);
    std::fclose(fo);
    cudaFree(d_depth);
    return 0;
}
