// tlfr_common.cuh — arithmetic shared by the hierarchy build and the query
// kernels.  Every expression keeps the reference's single-precision operation
// order; the whole library is compiled with -fmad=false (no FMA contraction) and
// IEEE division and square root, so results are bit-identical to the reference's
// CPU code built with -ffp-contract=off.
#pragma once
#include <cstdint>
#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define TLFR_HD __host__ __device__ __forceinline__
#else
#define TLFR_HD inline
#endif

namespace tlfr
{

constexpr float kF32Max = 3.402823466e+38f;     // FW_F32_MAX (framework/base/Defs.hpp:118)

// rcp: 1/a, and 0 for a == 0 (framework/base/Math.hpp:112)
TLFR_HD float rcp(float a) { return a ? 1.0f / a : 0.0f; }
// scalar min/max as the framework defines them: (a<b)?a:b, (a>b)?a:b (Defs.hpp:196-197)
TLFR_HD float minr(float a, float b) { return (a < b) ? a : b; }
TLFR_HD float maxr(float a, float b) { return (a > b) ? a : b; }
TLFR_HD int   mini(int a, int b) { return (a < b) ? a : b; }
TLFR_HD int   maxi(int a, int b) { return (a > b) ? a : b; }
TLFR_HD float absf(float a) { return fabsf(a); }
// double -> float, round to nearest even
TLFR_HD float d2f_rn(double x)
{
#ifdef __CUDA_ARCH__
    return __double2float_rn(x);
#else
    return (float)x;
#endif
}

// getCocRadius(C, w) = C0/w + C1 (reconstruction_lib/common/CameraParams.hpp:72)
TLFR_HD float coc_radius(float c0, float c1, float w) { return c0 / w + c1; }

// ---------------------------------------------------------------------------
// Time/lens bounds: four hyperplanes x = A*t + B*u + C (xmin, xmax, ymin, ymax)
// plus the valid time span (reconstruction/Reconstruction.hpp:149-167).
// ---------------------------------------------------------------------------
struct Bounds
{
    float p[4][3];
    float tspan[2];
};

TLFR_HD bool bounds_valid(const Bounds& b) { return b.tspan[0] < b.tspan[1]; }

TLFR_HD void bounds_zero(Bounds& b)
{
    for (int i = 0; i < 4; i++) { b.p[i][0] = 0.0f; b.p[i][1] = 0.0f; b.p[i][2] = 0.0f; }
    b.tspan[0] = 0.0f; b.tspan[1] = 0.0f;
}

// TimeLensBounds::evaluate (Reconstruction.hpp:162)
TLFR_HD float plane_eval(const float* p, float t, float uv) { return (t * p[0] + p[1] * uv) + p[2]; }

// computePerspectivePlanes1D (reconstruction_lib/common/TimeBounds.cpp:228-332):
// bounding lines (t slope, constant) of a homogeneous 1D point x0/w0 moving by
// (dx, dw) over t in [0,1], clipped to [xmin, xmax] and to w > 0.
TLFR_HD bool perspective_planes_1d(float x0, float w0, float dx, float dw, float xmin, float xmax,
                                   float (*dest)[2], float* span)
{
    if (dx == 0.0f && dw == 0.0f)
    {
        float xow0 = x0 / w0;
        dest[0][0] = 0.0f; dest[0][1] = xow0;
        dest[1][0] = 0.0f; dest[1][1] = xow0;
        span[0] = 0.0f; span[1] = 1.0f;
        return w0 > 0.0f;
    }
    float tb0 = 0.0f, tb1 = 1.0f;
    if (dw != 0.0f)
    {
        float tw0 = -w0 / dw;
        if (tw0 >= 0 && tw0 <= 1)
        {
            if (w0 < 0) tb0 = tw0;
            else        tb1 = tw0;
        }
    }
    bool movesright = dx * w0 > dw * x0;
    bool movesforward = dw > 0;
    float tmin = (xmin * w0 - x0) / (dx - xmin * dw);
    if (w0 + tmin * dw >= 0)
    {
        if (movesright) tb0 = maxr(tb0, tmin);
        else            tb1 = minr(tb1, tmin);
    }
    float tmax = (xmax * w0 - x0) / (dx - xmax * dw);
    if (w0 + tmax * dw >= 0)
    {
        if (!movesright) tb0 = maxr(tb0, tmax);
        else             tb1 = minr(tb1, tmax);
    }
    if (tb0 > tb1)
        return false;
    float thalf = 0.5f * (tb0 + tb1);
    float px = (x0 + thalf * dx) / (w0 + thalf * dw);
    float dxdt = dx / (w0 + thalf * dw) - (dw * (x0 + thalf * dx)) / ((w0 + thalf * dw) * (w0 + thalf * dw));
    float xa = (x0 + tb0 * dx) / (w0 + tb0 * dw);
    float xb = (x0 + tb1 * dx) / (w0 + tb1 * dw);
    float p10 = dxdt, p11 = (px - dxdt * thalf);
    float p20 = -(xb - xa) / (tb0 - tb1), p21 = xa + ((xb - xa) * tb0) / (tb0 - tb1);
    if (movesright == movesforward)
    {
        dest[1][0] = p10; dest[1][1] = p11;
        dest[0][0] = p20; dest[0][1] = p21;
    }
    else
    {
        dest[0][0] = p10; dest[0][1] = p11;
        dest[1][0] = p20; dest[1][1] = p21;
    }
    span[0] = tb0; span[1] = tb1;
    return true;
}

// computeTUXPlanes (TimeBounds.cpp:73-147) for the sample's t=0 homogeneous
// position pos and motion mot, screen [0,W]x[0,H], CoC coefficients (c0, c1).
// On failure the planes stay zero and tspan keeps whatever
// computePerspectivePlanes (TimeBounds.cpp:44-62) wrote.
TLFR_HD void tux_planes(const float* pos, const float* mot, float W, float H, float c0, float c1, Bounds& out)
{
    bounds_zero(out);
    float planes[4][2];
    float sx[2], sy[2];
    bool bx = perspective_planes_1d(pos[0], pos[2], mot[0], mot[2], 0.0f, W, &planes[0], sx);
    bool by = perspective_planes_1d(pos[1], pos[2], mot[1], mot[2], 0.0f, H, &planes[2], sy);
    if (!bx || !by)
        return;
    out.tspan[0] = maxr(sx[0], sy[0]);
    out.tspan[1] = minr(sx[1], sy[1]);
    if (!(out.tspan[0] < out.tspan[1]))
        return;
    float fT[3] = { out.tspan[0], out.tspan[1], 0.5f * (out.tspan[0] + out.tspan[1]) };
    float ep[3][2], fc[3];
    for (int i = 0; i < 3; i++)
    {
        float xw = pos[0] + mot[0] * fT[i];
        float yw = pos[1] + mot[1] * fT[i];
        float w = pos[2] + mot[2] * fT[i];
        float c = rcp(w);
        ep[i][0] = xw * c;
        ep[i][1] = yw * c;
        fc[i] = c0 / w + c1;
    }
    float avg = (1.f / 3.f) * ((fc[0] + fc[1]) + fc[2]);
    out.p[0][0] = planes[0][0]; out.p[0][1] = avg; out.p[0][2] = FLT_MAX;
    out.p[1][0] = planes[1][0]; out.p[1][1] = avg; out.p[1][2] = -FLT_MAX;
    out.p[2][0] = planes[2][0]; out.p[2][1] = avg; out.p[2][2] = FLT_MAX;
    out.p[3][0] = planes[3][0]; out.p[3][1] = avg; out.p[3][2] = -FLT_MAX;
    for (int i = 0; i < 3; i++)
    {
        float x11 = ((1.0f * (ep[i][0] - fc[i])) - planes[0][0] * fT[i]) - avg * (-1.0f);
        float x21 = ((1.0f * (ep[i][0] + fc[i])) - planes[0][0] * fT[i]) - avg * (1.0f);
        float x12 = ((1.0f * (ep[i][0] - fc[i])) - planes[1][0] * fT[i]) - avg * (-1.0f);
        float x22 = ((1.0f * (ep[i][0] + fc[i])) - planes[1][0] * fT[i]) - avg * (1.0f);
        float y11 = ((1.0f * (ep[i][1] - fc[i])) - planes[2][0] * fT[i]) - avg * (-1.0f);
        float y21 = ((1.0f * (ep[i][1] + fc[i])) - planes[2][0] * fT[i]) - avg * (1.0f);
        float y12 = ((1.0f * (ep[i][1] - fc[i])) - planes[3][0] * fT[i]) - avg * (-1.0f);
        float y22 = ((1.0f * (ep[i][1] + fc[i])) - planes[3][0] * fT[i]) - avg * (1.0f);
        out.p[0][2] = minr(minr(out.p[0][2], x11), x21);
        out.p[1][2] = maxr(maxr(out.p[1][2], x12), x22);
        out.p[2][2] = minr(minr(out.p[2][2], y11), y21);
        out.p[3][2] = maxr(maxr(out.p[3][2], y12), y22);
    }
}

// mergeTUXPlanes for one plane pair (TimeBounds.cpp:154-212): least-squares
// plane through the per-corner maxima over the (t,u) rectangle, lifted by the
// largest residual.
TLFR_HD void merge_plane(const float* p1, const float* p2, float* out)
{
    float x1[4], x2[4], m[4];
    x1[0] = -p1[1] + p1[2]; x1[1] = (p1[0] - p1[1]) + p1[2];
    x1[2] = (p1[0] + p1[1]) + p1[2]; x1[3] = p1[1] + p1[2];
    x2[0] = -p2[1] + p2[2]; x2[1] = (p2[0] - p2[1]) + p2[2];
    x2[2] = (p2[0] + p2[1]) + p2[2]; x2[3] = p2[1] + p2[2];
    for (int k = 0; k < 4; k++)
        m[k] = maxr(x1[k], x2[k]);
    float c0 = m[1] + m[2];
    float c1 = ((m[2] + m[3]) - m[0]) - m[1];
    float c2 = ((m[0] + m[1]) + m[2]) + m[3];
    float a = c0 - 0.5f * c2;
    float b = 0.25f * c1;
    float d = m[0] - (-b);
    d = maxr(d, m[1] - (a - b));
    d = maxr(d, m[2] - (a + b));
    d = maxr(d, m[3] - b);
    out[0] = a; out[1] = b; out[2] = d;
}

// mergeTUXPlanes for a plane set (TimeBounds.cpp:216-224); xmin/ymin through
// negation.
TLFR_HD void merge_bounds(const Bounds& a, const Bounds& b, Bounds& r)
{
    for (int p = 0; p < 4; p++)
    {
        if (p == 0 || p == 2)
        {
            float na[3] = { -a.p[p][0], -a.p[p][1], -a.p[p][2] };
            float nb[3] = { -b.p[p][0], -b.p[p][1], -b.p[p][2] };
            float m[3];
            merge_plane(na, nb, m);
            r.p[p][0] = -m[0]; r.p[p][1] = -m[1]; r.p[p][2] = -m[2];
        }
        else
            merge_plane(a.p[p], b.p[p], r.p[p]);
    }
    r.tspan[0] = minr(a.tspan[0], b.tspan[0]);
    r.tspan[1] = maxr(a.tspan[1], b.tspan[1]);
}

// TimeLensBounds(tb0, tb1) (Reconstruction.hpp:153-160)
TLFR_HD void combine_bounds(const Bounds& tb0, const Bounds& tb1, Bounds& out)
{
    bool v0 = bounds_valid(tb0), v1 = bounds_valid(tb1);
    if (v0 && v1)   { Bounds r; merge_bounds(tb0, tb1, r); out = r; }
    else if (v0)    out = tb0;
    else if (v1)    out = tb1;
    else            bounds_zero(out);
}

// Node::getExpectedCost (Reconstruction.hpp:184-202), including its use of the
// X planes' t slopes in the y extent.
TLFR_HD float bounds_cost(const Bounds& b, int ns)
{
    float dx = ((b.p[1][2] - b.p[0][2]) + absf(b.p[1][1] - b.p[0][1])) + absf(b.p[1][0] - b.p[0][0]);
    float dy = ((b.p[3][2] - b.p[2][2]) + absf(b.p[3][1] - b.p[2][1])) + absf(b.p[1][0] - b.p[0][0]);
    return (dx * dy) * (float)ns;
}

// ternaryCompare / ternaryEqual (Reconstruction.hpp:428-449).
// Written as selects and an integer product rather than the reference's
// if/else chain and ||-chain: with nvcc 12.9 for sm_100a at -O3 the inlined
// nesting ternaryEqual(ternaryCompare(..), ternaryCompare(..)) in that form
// evaluated wrongly on the device (checked against the host on 20k random node
// pairs); these forms give the reference's results on both.
TLFR_HD int ternary_compare(float a, float b, float eps)
{
    const int sgn = (a < b) ? -1 : 1;
    return (absf(a - b) < eps) ? 0 : sgn;
}
// a == 0 || b == 0 || a == b, for a, b in {-1, 0, 1}
TLFR_HD bool ternary_equal2(int a, int b) { return a * b != -1; }
TLFR_HD bool ternary_equal4(int a, int b, int c, int d)
{
    int mn = mini(mini(mini(a, b), c), d);
    int mx = maxi(maxi(maxi(a, b), c), d);
    return mx - mn < 2;
}

// ---------------------------------------------------------------------------
// FW::sort (framework/base/Sort.cpp:36-165, 203-211): quicksort with a
// median-of-3 pivot and insertion sort below 16 elements.  Unstable; the exact
// permutation it produces for equal keys is part of the reference's results, so
// the same algorithm runs here.  A is an accessor with cmp(i, j) -> -1/0/1 and
// swap(i, j).
// ---------------------------------------------------------------------------
template <class A>
TLFR_HD void fw_insertion_sort(A& a, int start, int size)
{
    for (int i = 1; i < size; i++)
    {
        int j = start + i - 1;
        while (j >= start && a.cmp(j, j + 1) > 0)
        {
            a.swap(j, j + 1);
            j--;
        }
    }
}

template <class A>
TLFR_HD int fw_median3(A& a, int low, int high)
{
    int l = low;
    int c = (low + high) >> 1;
    int h = high - 2;
    if (a.cmp(l, h) > 0) { int t = l; l = h; h = t; }
    if (a.cmp(l, c) > 0) c = l;
    return (a.cmp(c, h) > 0) ? h : c;
}

template <class A>
TLFR_HD int fw_partition(A& a, int low, int high)
{
    a.swap(fw_median3(a, low, high), high - 1);
    int i = low - 1;
    int j = high - 1;
    for (;;)
    {
        // Both scans stop inside [low, high-1]: the pivot at high-1 stops i, and
        // the median-of-3 leaves an element <= pivot at or above low for j.
        do i++; while (a.cmp(i, high - 1) < 0);
        do j--; while (j > low && a.cmp(j, high - 1) > 0);
        if (i >= j)
            break;
        a.swap(i, j);
    }
    a.swap(i, high - 1);
    return i;
}

template <class A>
TLFR_HD void fw_sort(A& a, int start, int end)
{
    if (end - start < 2)
        return;
    int low = start, high = end;
    int stack[32];
    int sp = 0;
    stack[sp++] = high;
    while (sp)
    {
        high = stack[--sp];
        if (high - low < 16 || sp + 2 > 32)
        {
            fw_insertion_sort(a, low, high - low);
            low = high + 1;
            continue;
        }
        int i = fw_partition(a, low, high);
        if (high - i > 2)
            stack[sp++] = high;
        if (i - low > 1)
            stack[sp++] = i;
        else
            low = i + 1;
    }
}

// Jenkins hash hashBits(a, b) (framework/base/Hash.hpp:169-183)
TLFR_HD uint32_t hash_bits(uint32_t a, uint32_t b)
{
    uint32_t c = 0x9e3779b9u;
    a -= b; a -= c; a ^= (c >> 13);
    b -= c; b -= a; b ^= (a << 8);
    c -= a; c -= b; c ^= (b >> 13);
    a -= b; a -= c; a ^= (c >> 12);
    b -= c; b -= a; b ^= (a << 16);
    c -= a; c -= b; c ^= (b >> 5);
    a -= b; a -= c; a ^= (c >> 3);
    b -= c; b -= a; b ^= (a << 10);
    c -= a; c -= b; c ^= (b >> 15);
    return c;
}

// Dispersion (radius of the largest empty circle) by samples per pixel
// (reconstruction/ReconstructionOur.cpp:63-76).
TLFR_HD float dispersion_for_spp(int spp)
{
    switch (spp)
    {
    case 256: return 0.14f;
    case 128: return 0.18f;
    case 64:  return 0.27f;
    case 32:  return 0.37f;
    case 16:  return 0.50f;
    case 8:   return 0.80f;
    case 4:   return 1.10f;
    case 2:   return 1.34f;
    default:  return 2.00f;
    }
}

} // namespace tlfr
