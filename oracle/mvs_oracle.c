/* CPU oracle for the multiview-stereo hot path -- TEST INFRASTRUCTURE ONLY.
 * See mvs_oracle.h.  Built by oracle/Makefile with -ffp-contract=off so that
 * the float variant performs exactly the reference's roundings. */
#include "mvs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Loops whose iterations touch disjoint outputs run over OpenMP threads; the
 * arithmetic of each element is unchanged, so results do not depend on the
 * thread count. */
#ifdef _OPENMP
#define ORC_PAR _Pragma("omp parallel for schedule(static)")
#else
#define ORC_PAR
#endif

/* Bin centres (fusion.h:1041-1054): -1, linspace over bins 1..N-2, +1. */
void orc_bin_centers(int bins, float *out)
{
    out[0] = -1.f;
    out[bins - 1] = 1.f;
    if (bins > 3)
        for (int i = 1; i < bins - 1; ++i) out[i] = 2.f * (float)(i - 1) / (float)(bins - 3) - 1.f;
    else if (bins == 3)
        out[1] = 0.f;
}

/* sortedHist<N>::insert (structs.h:241-262), statement for statement: the
 * element is shifted up while smaller than its left neighbour; a value
 * smaller than element[0] ends the loop without being stored, which leaves
 * element[0] duplicated. */
static void sorted_insert(float *el, int *count, int size, float val)
{
    int elements = *count;
    if (elements != 0) {
        for (int i = elements - 1; i >= 0; i--) {
            int next = i + 1 < size - 1 ? i + 1 : size - 1;
            if (val < el[i]) el[next] = el[i];
            else {
                el[next] = val;
                break;
            }
        }
    } else {
        el[0] = val;
    }
    elements = elements + 1 < size ? elements + 1 : size;
    *count = elements;
}

/* fusionData::proxHist (fusion.h:851-858) with Wi (:813-820) and pi (:834-838). */
float orc_prox_hist_f32(int bins, const uint16_t *h, float u, float tau, float lambda)
{
    float el[33];
    float centers[16];
    orc_bin_centers(bins, centers);
    memcpy(el, centers, sizeof(float) * bins);
    int count = bins;
    const int size = 2 * bins + 1;
    sorted_insert(el, &count, size, u);
    for (int j = 1; j <= bins; ++j) {
        int W = 0;
        for (int k = 1; k <= j; ++k) W -= h[k - 1];
        for (int k = j + 1; k <= bins; ++k) W += h[k - 1];
        float pj = u + tau * lambda * (float)W;
        sorted_insert(el, &count, size, pj);
    }
    return el[bins];
}

/* planesweep.cpp:169,200: dstep = (zfar - znear)/(n - 1); for (d = znear; d <= zfar; d += dstep) */
int orc_plane_list(float znear, float zfar, int nplanes, float *out, int cap)
{
    float dstep = (zfar - znear) / (float)(nplanes - 1);
    int k = 0;
    for (float d = znear; d <= zfar; d += dstep) {
        if (k < cap) out[k] = d;
        ++k;
    }
    return k;
}

/* ---- float variant: the reference's arithmetic ---- */
#define R float
#define FN(name) name##_f32
#define ORC_IS_F32 1
#define SQRTR sqrtf
#define FABSR fabsf
#define FLOORR floorf
#define ROUNDR roundf
#define EXPR expf
#define POWR powf
#define FMAXR(a, b) fmaxf((float)(a), (float)(b))
#define FMINR(a, b) fminf((float)(a), (float)(b))
#include "mvs_oracle_impl.h"
#undef R
#undef FN
#undef ORC_IS_F32
#undef SQRTR
#undef FABSR
#undef FLOORR
#undef ROUNDR
#undef EXPR
#undef POWR
#undef FMAXR
#undef FMINR

/* ---- double variant: the FP64 oracle ---- */
#define R double
#define FN(name) name##_f64
#define ORC_IS_F32 0
#define SQRTR sqrt
#define FABSR fabs
#define FLOORR floor
#define ROUNDR round
#define EXPR exp
#define POWR pow
#define FMAXR(a, b) fmax((double)(a), (double)(b))
#define FMINR(a, b) fmin((double)(a), (double)(b))
#include "mvs_oracle_impl.h"
