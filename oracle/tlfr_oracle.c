/*
 * tlfr_oracle.c — CPU restatement (plain C99) of the reference's temporal light
 * field reconstruction path: sample reprojection and bucketing, the 5D hierarchy
 * build, the output sampling pattern, and the per-output-sample filter.
 *
 * TEST INFRASTRUCTURE ONLY — the checker for the CUDA path, never the product.
 * Pinned against the reference itself (oracle/build_ref.sh builds the reference
 * sources; tests/test_oracle_vs_reference.py compares trees, queries and pixels).
 *
 * Every function cites the reference file:line it restates.  Paths are relative
 * to the reference's src/ directory:
 *   R.hpp/R.cpp  = reconstruction_lib/reconstruction/Reconstruction.hpp/.cpp
 *   RTB.cpp      = reconstruction_lib/reconstruction/ReconstructionTreeBuilder.cpp
 *   RO.cpp       = reconstruction_lib/reconstruction/ReconstructionOur.cpp
 *   TB.cpp       = reconstruction_lib/common/TimeBounds.cpp
 *   EF.cpp/.hpp  = reconstruction_lib/common/EdgeFunction.cpp/.hpp
 *   Util.cpp/.hpp= reconstruction_lib/common/Util.cpp/.hpp
 *   Sort.cpp, Hash.hpp, Random.cpp, Math.hpp, Defs.hpp, Array.hpp = framework/base/
 *
 * Floating point: IEEE single precision, no FMA contraction (build with
 * -O2 -ffp-contract=off -fno-fast-math); every vector expression of the reference
 * is written out in its evaluation order.
 */
#include "tlfr_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define F32_MAX 3.402823466e+38f          /* FW_F32_MAX, Defs.hpp:118 */

static char g_err[512];
const char* orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------- */
/* Scalar helpers (Math.hpp, Defs.hpp).                                       */
/* ------------------------------------------------------------------------- */

/* rcp: Math.hpp:112 — 1/a, and 0 for a == 0 */
static inline float rcpf_(float a) { return a ? 1.0f / a : 0.0f; }
/* min/max for scalars: Defs.hpp:196-197 ((a<b)?a:b, (a>b)?a:b) */
static inline float fminr(float a, float b) { return (a < b) ? a : b; }
static inline float fmaxr(float a, float b) { return (a > b) ? a : b; }
static inline int   iminr(int a, int b) { return (a < b) ? a : b; }
static inline int   imaxr(int a, int b) { return (a > b) ? a : b; }

/* getCocRadius: CameraParams.hpp:72 */
static inline float coc_radius(const float cc[2], float w) { return cc[0] / w + cc[1]; }

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------------- */
/* FW::sort — Sort.cpp:36-165, 203-211.  Quicksort with median-of-3 pivot,    */
/* insertion sort below 16 elements; unstable.  The compare/swap callbacks    */
/* act on indices of an opaque array.                                         */
/* ------------------------------------------------------------------------- */

typedef int  (*cmp_fn)(void* data, int a, int b);
typedef void (*swp_fn)(void* data, int a, int b);

static void fw_insertion_sort(int start, int size, void* data, cmp_fn cmp, swp_fn swp)   /* Sort.cpp:63-77 */
{
    for (int i = 1; i < size; i++)
    {
        int j = start + i - 1;
        while (j >= start && cmp(data, j, j + 1) > 0)
        {
            swp(data, j, j + 1);
            j--;
        }
    }
}

static int fw_median3(int low, int high, void* data, cmp_fn cmp)                         /* Sort.cpp:81-93 */
{
    int l = low;
    int c = (low + high) >> 1;
    int h = high - 2;
    if (cmp(data, l, h) > 0) { int t = l; l = h; h = t; }
    if (cmp(data, l, c) > 0) c = l;
    return (cmp(data, c, h) > 0) ? h : c;
}

static int fw_partition(int low, int high, void* data, cmp_fn cmp, swp_fn swp)          /* Sort.cpp:97-127 */
{
    swp(data, fw_median3(low, high, data, cmp), high - 1);
    int i = low - 1;
    int j = high - 1;
    for (;;)
    {
        do i++; while (cmp(data, i, high - 1) < 0);
        do j--; while (cmp(data, j, high - 1) > 0);
        if (i >= j)
            break;
        swp(data, i, j);
    }
    swp(data, i, high - 1);
    return i;
}

static void fw_qsort(int low, int high, void* data, cmp_fn cmp, swp_fn swp)             /* Sort.cpp:131-165 */
{
    int stack[32];
    int sp = 0;
    stack[sp++] = high;
    while (sp)
    {
        high = stack[--sp];
        if (high - low < 16 || sp + 2 > 32)
        {
            fw_insertion_sort(low, high - low, data, cmp, swp);
            low = high + 1;
            continue;
        }
        int i = fw_partition(low, high, data, cmp, swp);
        if (high - i > 2)
            stack[sp++] = high;
        if (i - low > 1)
            stack[sp++] = i;
        else
            low = i + 1;
    }
}

static void fw_sort(int start, int end, void* data, cmp_fn cmp, swp_fn swp)             /* Sort.cpp:203-211 */
{
    if (end - start < 2)
        return;
    fw_qsort(start, end, data, cmp, swp);
}

/* ------------------------------------------------------------------------- */
/* hashBits (Hash.hpp:169-183) and RANROT-A (Random.cpp:52-92).               */
/* ------------------------------------------------------------------------- */

static uint32_t hash_bits(uint32_t a, uint32_t b, uint32_t c)
{
    c += 0x9e3779b9u;
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

typedef struct { int32_t p1, p2; uint32_t buf[11]; } ranrot;

static uint32_t ranrot_get(ranrot* r)
{
    uint32_t x = r->buf[r->p1] + r->buf[r->p2];
    x = (x << 13) | (x >> 19);
    r->buf[r->p1] = x;
    r->p1--; r->p1 += (r->p1 >> 31) & 11;
    r->p2--; r->p2 += (r->p2 >> 31) & 11;
    return x;
}

static void ranrot_reset(ranrot* r, uint32_t seed)
{
    if (seed == 0)
        seed--;
    for (int i = 0; i < 11; i++)
    {
        seed ^= seed << 13;
        seed ^= seed >> 17;
        seed ^= seed << 5;
        r->buf[i] = seed;
    }
    r->p1 = 0;
    r->p2 = 7;
    for (int i = 0; i < 11; i++)
        ranrot_get(r);
}

/* Random::getF32, Random.hpp:57 */
static float ranrot_f32(ranrot* r) { return (float)ranrot_get(r) * (1.0f / 4294967296.0f); }

/* ------------------------------------------------------------------------- */
/* Low-discrepancy sequences (Util.cpp:229-300).                              */
/* ------------------------------------------------------------------------- */

static float hammersley(int i, int num) { return ((float)i + 0.5f) / (float)num; }   /* Util.cpp:229-233 */

static float halton(int base, int i)                                                   /* Util.cpp:235-250 */
{
    float h = 0.0f;
    float half = rcpf_((float)base);
    while (i)
    {
        int digit = i % base;
        h = h + (float)digit * half;
        i = (i - digit) / base;
        half = half / (float)base;
    }
    return h;
}

/* sobol(3, i) (Util.cpp:256-264).  The dimension-3 generating matrix is the
 * standard Sobol construction for the primitive polynomial x^3 + x + 1 with
 * initial direction numbers m = (1, 3, 1): v_k = m_k / 2^k for k <= 3 and
 * v_k = v_{k-2} ^ v_{k-3} ^ (v_{k-3} >> 3) beyond. */
static uint32_t g_sobol3[32];
static void sobol3_init(void)
{
    uint32_t v[32];
    v[0] = 1u << 31; v[1] = 3u << 30; v[2] = 1u << 29;
    for (int k = 3; k < 32; k++)
        v[k] = v[k - 2] ^ v[k - 3] ^ (v[k - 3] >> 3);
    memcpy(g_sobol3, v, sizeof(v));
}

static float sobol3(int i)
{
    uint32_t result = 0;
    for (unsigned c = 0; i; i >>= 1, ++c)
        if (i & 1)
            result ^= g_sobol3[c];
    return (float)result * (1.0f / 4294967296.0f);
}

static void sobol2d(int i, float* out)                                                 /* Util.cpp:266-289 */
{
    uint32_t r1 = 0, r2 = 0;
    for (uint32_t v1 = 1u << 31, v2 = 3u << 30; i; i >>= 1)
    {
        if (i & 1)
        {
            r1 ^= v1;
            r2 ^= v2 << 1;
        }
        v1 |= v1 >> 1;
        v2 ^= v2 >> 1;
    }
    out[0] = (float)r1 * (1.0f / 4294967296.0f);
    out[1] = (float)r2 * (1.0f / 4294967296.0f);
}

static float larcher_pillichshammer(int i)                                             /* Util.cpp:291-299 */
{
    uint32_t r = 0;
    for (uint32_t v = 1u << 31; i; i >>= 1, v |= v >> 1)
        if (i & 1)
            r ^= v;
    return (float)((double)r / (double)0x100000000LL);
}

static void to_unit_disk(float sx, float sy, float* ou, float* ov)                     /* Util.cpp:37-74 */
{
    const float PI = 3.1415926535897932384626433832795f;
    float phi, r;
    float a = 2.0f * sx - 1.0f;
    float b = 2.0f * sy - 1.0f;
    if (a > -b)
    {
        if (a > b) { r = a; phi = (PI / 4) * (b / a); }
        else       { r = b; phi = (PI / 4) * (2.0f - (a / b)); }
    }
    else
    {
        if (a < b) { r = -a; phi = (PI / 4) * (4.0f + (b / a)); }
        else
        {
            r = -b;
            if (b != 0) phi = (PI / 4) * (6.0f - (a / b));
            else        phi = 0;
        }
    }
    *ou = r * cosf(phi);
    *ov = r * sinf(phi);
}

/* ------------------------------------------------------------------------- */
/* Data types (R.hpp:73-231).                                                 */
/* ------------------------------------------------------------------------- */

typedef struct
{
    float x, y;          /* xy */
    float u, v;          /* uv */
    float t;
    float col[4];
    float mv[3];
    float w;
    float wg[2];
    float density;
    float key;
    int   id;            /* input record index (instrumentation) */
} osample;

typedef struct
{
    float planes[4][3];  /* xmin, xmax, ymin, ymax: (t, uv, const) */
    float tspan[2];
} tlb_t;

typedef struct
{
    tlb_t tlb;
    int   child0, child1;
    int   s0, s1;
    int   ns;
} onode;

typedef struct { int x0, y0, x1, y1, child0, child1, numSamples; } inode;

/* growable arrays */
#define DEFINE_VEC(name, T)                                                        \
    typedef struct { T* p; int n, cap; } name;                                     \
    static T* name##_add(name* v)                                                  \
    {                                                                              \
        if (v->n == v->cap)                                                        \
        {                                                                          \
            v->cap = v->cap ? 2 * v->cap : 16;                                     \
            v->p = (T*)realloc(v->p, sizeof(T) * (size_t)v->cap);                  \
        }                                                                          \
        return &v->p[v->n++];                                                      \
    }                                                                              \
    static void name##_reserve(name* v, int cap)                                   \
    {                                                                              \
        if (cap > v->cap) { v->cap = cap; v->p = (T*)realloc(v->p, sizeof(T) * (size_t)cap); } \
    }

DEFINE_VEC(vec_node, onode)
DEFINE_VEC(vec_int, int)
DEFINE_VEC(vec_samp, osample)

/* ------------------------------------------------------------------------- */
/* TUX hyperplanes (TB.cpp).                                                  */
/* ------------------------------------------------------------------------- */

/* computePerspectivePlanes1D, TB.cpp:228-332; pDest: 2 lines (t slope, const) */
static int perspective_planes_1d(float x0, float w0, float dx, float dw, float xmin, float xmax,
                                 float dest[2][2], float span[2])
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
    int movesright = dx * w0 > dw * x0;
    int movesforward = dw > 0;

    float tmin = (xmin * w0 - x0) / (dx - xmin * dw);
    if (w0 + tmin * dw >= 0)
    {
        if (movesright) tb0 = fmaxr(tb0, tmin);
        else            tb1 = fminr(tb1, tmin);
    }
    float tmax = (xmax * w0 - x0) / (dx - xmax * dw);
    if (w0 + tmax * dw >= 0)
    {
        if (!movesright) tb0 = fmaxr(tb0, tmax);
        else             tb1 = fminr(tb1, tmax);
    }
    if (tb0 > tb1)
        return 0;

    float thalf = 0.5f * (tb0 + tb1);
    float px = (x0 + thalf * dx) / (w0 + thalf * dw);
    float dxdt = dx / (w0 + thalf * dw) - (dw * (x0 + thalf * dx)) / ((w0 + thalf * dw) * (w0 + thalf * dw));
    float xa = (x0 + tb0 * dx) / (w0 + tb0 * dw);
    float xb = (x0 + tb1 * dx) / (w0 + tb1 * dw);
    float p1[2] = { dxdt, (px - dxdt * thalf) };
    float p2[2] = { -(xb - xa) / (tb0 - tb1), xa + ((xb - xa) * tb0) / (tb0 - tb1) };
    if (movesright == movesforward)
    {
        dest[1][0] = p1[0]; dest[1][1] = p1[1];
        dest[0][0] = p2[0]; dest[0][1] = p2[1];
    }
    else
    {
        dest[0][0] = p1[0]; dest[0][1] = p1[1];
        dest[1][0] = p2[0]; dest[1][1] = p2[1];
    }
    span[0] = tb0; span[1] = tb1;
    return 1;
}

/* computePerspectivePlanes, TB.cpp:44-62 */
static int perspective_planes(const float pos[3], const float mot[3], const float bbmin[2], const float bbmax[2],
                              float planes[4][2], float tspan[2])
{
    float sx[2], sy[2];
    int bx = perspective_planes_1d(pos[0], pos[2], mot[0], mot[2], bbmin[0], bbmax[0], (float (*)[2])planes[0], sx);
    int by = perspective_planes_1d(pos[1], pos[2], mot[1], mot[2], bbmin[1], bbmax[1], (float (*)[2])planes[2], sy);
    if (!bx || !by)
        return 0;
    tspan[0] = fmaxr(sx[0], sy[0]);
    tspan[1] = fminr(sx[1], sy[1]);
    return tspan[0] < tspan[1];
}

/* computeTUXPlanes, TB.cpp:73-147.  On failure the planes are left zero (the
 * TimeLensBounds members are value-initialised, R.hpp:152) and tspan holds what
 * computePerspectivePlanes wrote. */
static void tux_planes(const float pos[3], const float mot[3], const float bbmin[2], const float bbmax[2],
                       const float cc[2], tlb_t* out)
{
    memset(out, 0, sizeof(*out));
    float planes[4][2];
    float* tspan = out->tspan;
    tspan[0] = 0.0f; tspan[1] = 0.0f;
    if (!perspective_planes(pos, mot, bbmin, bbmax, planes, tspan))
        return;
    float fT[3];
    fT[0] = tspan[0];
    fT[1] = tspan[1];
    fT[2] = 0.5f * (tspan[0] + tspan[1]);
    float xyw[3][3], ep[3][2], fc[3];
    for (int i = 0; i < 3; i++)
    {
        xyw[i][0] = pos[0] + mot[0] * fT[i];
        xyw[i][1] = pos[1] + mot[1] * fT[i];
        xyw[i][2] = pos[2] + mot[2] * fT[i];
    }
    for (int i = 0; i < 3; i++)
    {
        float c = rcpf_(xyw[i][2]);
        ep[i][0] = xyw[i][0] * c;
        ep[i][1] = xyw[i][1] * c;
    }
    for (int i = 0; i < 3; i++)
        fc[i] = cc[0] / xyw[i][2] + cc[1];
    float avg = (1.f / 3.f) * ((fc[0] + fc[1]) + fc[2]);
    float (*P)[3] = out->planes;
    P[0][0] = planes[0][0]; P[0][1] = avg; P[0][2] = FLT_MAX;
    P[1][0] = planes[1][0]; P[1][1] = avg; P[1][2] = -FLT_MAX;
    P[2][0] = planes[2][0]; P[2][1] = avg; P[2][2] = FLT_MAX;
    P[3][0] = planes[3][0]; P[3][1] = avg; P[3][2] = -FLT_MAX;
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
        P[0][2] = fminr(fminr(P[0][2], x11), x21);
        P[1][2] = fmaxr(fmaxr(P[1][2], x12), x22);
        P[2][2] = fminr(fminr(P[2][2], y11), y21);
        P[3][2] = fmaxr(fmaxr(P[3][2], y12), y22);
    }
}

/* mergeTUXPlanes (single plane pair), TB.cpp:154-212 */
static void merge_plane(const float p1[3], const float p2[3], float out[3])
{
    float x1[4], x2[4], m[4];
    x1[0] = -p1[1] + p1[2]; x1[1] = (p1[0] - p1[1]) + p1[2];
    x1[2] = (p1[0] + p1[1]) + p1[2]; x1[3] = p1[1] + p1[2];
    x2[0] = -p2[1] + p2[2]; x2[1] = (p2[0] - p2[1]) + p2[2];
    x2[2] = (p2[0] + p2[1]) + p2[2]; x2[3] = p2[1] + p2[2];
    for (int k = 0; k < 4; k++)
        m[k] = fmaxr(x1[k], x2[k]);
    float c0 = m[1] + m[2];
    float c1 = ((m[2] + m[3]) - m[0]) - m[1];
    float c2 = ((m[0] + m[1]) + m[2]) + m[3];
    float a = c0 - 0.5f * c2;
    float b = 0.25f * c1;
    float k0 = -b, k1 = a - b, k2 = a + b, k3 = b;
    float d = m[0] - k0;
    d = fmaxr(d, m[1] - k1);
    d = fmaxr(d, m[2] - k2);
    d = fmaxr(d, m[3] - k3);
    out[0] = a; out[1] = b; out[2] = d;
}

/* mergeTUXPlanes (4 planes + tspan), TB.cpp:216-224 */
static void merge_tux(const tlb_t* a, const tlb_t* b, tlb_t* out)
{
    tlb_t r;
    for (int p = 0; p < 4; p++)
    {
        if (p == 0 || p == 2)
        {
            float na[3] = { -a->planes[p][0], -a->planes[p][1], -a->planes[p][2] };
            float nb[3] = { -b->planes[p][0], -b->planes[p][1], -b->planes[p][2] };
            float m[3];
            merge_plane(na, nb, m);
            r.planes[p][0] = -m[0]; r.planes[p][1] = -m[1]; r.planes[p][2] = -m[2];
        }
        else
            merge_plane(a->planes[p], b->planes[p], r.planes[p]);
    }
    r.tspan[0] = fminr(a->tspan[0], b->tspan[0]);
    r.tspan[1] = fmaxr(a->tspan[1], b->tspan[1]);
    *out = r;
}

static inline int tlb_valid(const tlb_t* t) { return t->tspan[0] < t->tspan[1]; }   /* R.hpp:163 */

/* TimeLensBounds(tb0, tb1), R.hpp:153-160 */
static void tlb_combine(const tlb_t* tb0, const tlb_t* tb1, tlb_t* out)
{
    if (tlb_valid(tb0) && tlb_valid(tb1)) merge_tux(tb0, tb1, out);
    else if (tlb_valid(tb0))              *out = *tb0;
    else if (tlb_valid(tb1))              *out = *tb1;
    else                                  memset(out, 0, sizeof(*out));
}

/* TimeLensBounds::evaluate, R.hpp:162 */
static inline float tlb_eval(const tlb_t* t, int idx, float tt, float uv)
{
    return (tt * t->planes[idx][0] + t->planes[idx][1] * uv) + t->planes[idx][2];
}

/* Node::getExpectedCost, R.hpp:184-202 (dy's last term uses the X planes, as written) */
static float node_cost(const onode* n)
{
    const float (*P)[3] = n->tlb.planes;
    float dx = ((P[1][2] - P[0][2]) + fabsf(P[1][1] - P[0][1])) + fabsf(P[1][0] - P[0][0]);
    float dy = ((P[3][2] - P[2][2]) + fabsf(P[3][1] - P[2][1])) + fabsf(P[1][0] - P[0][0]);
    return (dx * dy) * (float)n->ns;
}

/* Node(n0, n1), R.hpp:218-224 */
static void node_merge(const onode* n0, const onode* n1, onode* out)
{
    tlb_t t;
    tlb_combine(&n0->tlb, &n1->tlb, &t);
    out->tlb = t;
    out->ns = n0->ns + n1->ns;
    out->child0 = -1;
    out->child1 = -1;
    out->s0 = -1;
    out->s1 = -1;
}

/* ------------------------------------------------------------------------- */
/* The oracle state (TreeGather members, R.hpp:287-308).                      */
/* ------------------------------------------------------------------------- */

typedef struct
{
    int       W, H, spp_in;
    float     cc0[2];            /* header C0, C1 (drive the reprojection, R.cpp:519) */
    float     cc[2];             /* refocused C0', C1' (R.cpp:77-87) */
    int       spp;               /* m_spp: power of two */
    int       lens_filter, time_filter;
    int       override_uvt;
    float     uvt[3];
    int       out_spp;
    int       nthreads;

    /* reprojection grid */
    int       gw, gh;
    float     scale;
    int*      cell_start;        /* gw*gh+1 */
    osample*  cell_samples;      /* bucketed, input order within each cell */

    inode*    init_nodes;
    int       num_init;

    osample*  samples;           /* m_samples */
    int       num_samples;
    vec_node  hier;              /* m_hierarchy */
    int       root;
    int       num_invalid;

    osample*  outs;              /* m_outputSamples: 64 * out_spp */
} oracle;

/* ---- generateOutputSamples, R.cpp:452-512 ---- */

static int cmp_osample_key(void* d, int a, int b)
{
    osample* e = (osample*)d;
    return (e[a].key < e[b].key) ? -1 : (e[a].key > e[b].key) ? 1 : 0;
}
static void swp_osample(void* d, int a, int b)
{
    osample* e = (osample*)d;
    osample t = e[a]; e[a] = e[b]; e[b] = t;
}

static void generate_output_samples(oracle* o)
{
    const int M = o->out_spp;
    ranrot rnd;
    ranrot_reset(&rnd, 242);
    o->outs = (osample*)calloc((size_t)64 * M, sizeof(osample));
    for (int j = 0; j < 64; j++)
    {
        float xyoff[2] = { hammersley(j, 64), larcher_pillichshammer(j) };
        float uvoff[2] = { halton(2, j), halton(3, j) };
        float tJitter = ranrot_f32(&rnd);
        for (int i = 0; i < M; i++)
        {
            float s2d[2];
            sobol2d(i + 1, s2d);
            float x = sobol3(i + 1);
            float y = larcher_pillichshammer(i + 1);
            float u = s2d[0], v = s2d[1];
            float t = ((float)i + tJitter) / (float)M;
            float xy[2] = { x + xyoff[0], y + xyoff[1] };
            float uv[2] = { u + uvoff[0], v + uvoff[1] };
            if (xy[0] >= 1.f) xy[0] -= 1.f;
            if (xy[1] >= 1.f) xy[1] -= 1.f;
            if (uv[0] >= 1.f) uv[0] -= 1.f;
            if (uv[1] >= 1.f) uv[1] -= 1.f;
            int ub = (int)floorf(256.0f * uv[0]);
            int vb = (int)floorf(256.0f * uv[1]);
            int tb = (int)floorf(256.0f * t);
            int key = 0;
            for (int k = 0; k < 8; k++)
                key |= ((ub >> k) & 1) << (3 * k + 2) | ((vb >> k) & 1) << (3 * k + 1) | ((tb >> k) & 1) << (3 * k + 0);
            to_unit_disk(uv[0], uv[1], &uv[0], &uv[1]);
            if (o->override_uvt)
            {
                uv[0] = o->uvt[0]; uv[1] = o->uvt[1];
                t = o->uvt[2];
            }
            if (M == 1)
                xy[0] = xy[1] = 0.5f;
            osample* s = &o->outs[j * M + i];
            memset(s, 0, sizeof(*s));
            s->x = xy[0]; s->y = xy[1];
            s->u = uv[0]; s->v = uv[1];
            s->t = t;
            s->key = (float)key;
        }
        fw_sort(j * M, (j + 1) * M, o->outs, cmp_osample_key, swp_osample);
    }
}

/* ---- Sample::reprojectToUVTCenter, R.hpp:93-121 ---- */
static int reproject_uvt_center(osample* s, const float cc[2])
{
    float coc = coc_radius(cc, s->w);
    float px = s->x - s->u * coc;
    float py = s->y - s->v * coc;
    float P[3] = { px * s->w, py * s->w, 1.0f * s->w };
    float newt = 0.5f;
    float P0[3];
    for (int k = 0; k < 3; k++)
        P0[k] = (P[k] - s->mv[k] * s->t) + s->mv[k] * newt;
    if (P0[2] <= 0.f)
    {
        newt = 0.0f;
        for (int k = 0; k < 3; k++)
            P0[k] = (P[k] - s->mv[k] * s->t) + s->mv[k] * newt;
    }
    if (P0[2] <= 0.f)
    {
        newt = 1.0f;
        for (int k = 0; k < 3; k++)
            P0[k] = (P[k] - s->mv[k] * s->t) + s->mv[k] * newt;
    }
    if (P0[2] <= 0.f)
        return 0;
    s->w = P0[2];
    float c = rcpf_(P0[2]);
    s->x = P0[0] * c;
    s->y = P0[1] * c;
    s->u = 0.0f; s->v = 0.0f;
    s->t = newt;
    s->key = s->w;
    return 1;
}

/* ---- TreeGather::reprojectToUVTCenter, R.cpp:514-640 ---- */
static int reproject_and_bucket(oracle* o, const float* rec)
{
    const int W = o->W, H = o->H, spp = o->spp_in;
    const int n = W * H * spp;
    osample* s = (osample*)malloc(sizeof(osample) * (size_t)(n ? n : 1));
    int sidx = 0;
    for (int k = 0; k < n; k++)
    {
        const float* e = rec + (size_t)k * 16;
        osample* d = &s[sidx];
        memset(d, 0, sizeof(*d));
        d->x = e[0]; d->y = e[1]; d->w = e[3]; d->u = e[4]; d->v = e[5]; d->t = e[6];
        d->col[0] = e[7]; d->col[1] = e[8]; d->col[2] = e[9]; d->col[3] = 1.0f;
        d->mv[0] = e[11]; d->mv[1] = e[12]; d->mv[2] = e[13];
        d->wg[0] = e[14]; d->wg[1] = e[15];
        d->density = 1.0f;
        d->id = k;
        if (reproject_uvt_center(d, o->cc0))
            sidx++;
    }
    /* The reference then walks all n entries (R.cpp:561-575, 610-626) and so reads
     * uninitialised tail entries when a sample was discarded.  Only the kept
     * samples are used here; buffers whose samples all stay in front of the
     * camera (w > 0 at some time) are unaffected. */
    const int nk = sidx;
    float bbmin[2] = { F32_MAX, F32_MAX }, bbmax[2] = { -F32_MAX, -F32_MAX };
    int* hits = (int*)calloc((size_t)W * H, sizeof(int));
    for (int k = 0; k < nk; k++)
    {
        bbmin[0] = fminr(bbmin[0], s[k].x); bbmin[1] = fminr(bbmin[1], s[k].y);
        bbmax[0] = fmaxr(bbmax[0], s[k].x); bbmax[1] = fmaxr(bbmax[1], s[k].y);
        int sx = (int)floorf(s[k].x), sy = (int)floorf(s[k].y);
        if (sx >= 0 && sy >= 0 && sx < W && sy < H)
            hits[sy * W + sx]++;
    }
    int maxHits = 0;
    for (int k = 0; k < W * H; k++)
        maxHits = imaxr(maxHits, hits[k]);
    free(hits);
    if (maxHits == 0)
    {
        free(s);
        snprintf(g_err, sizeof(g_err), "All samples were discarded in reprojection to (u,v,t)=0");
        return 0;
    }
    float scale = sqrtf(1.f * (float)maxHits / 48.0f);
    float ext = fmaxr(bbmax[0] - bbmin[0], bbmax[1] - bbmin[1]);
    if (scale * ext > 4096)
        scale = 4096 / ext;
    bbmin[0] *= scale; bbmin[1] *= scale;
    bbmax[0] *= scale; bbmax[1] *= scale;
    int bminx = (int)floorf(bbmin[0]), bminy = (int)floorf(bbmin[1]);
    int bmaxx = (int)floorf(bbmax[0]) + 1, bmaxy = (int)floorf(bbmax[1]) + 1;
    o->gw = bmaxx - bminx;
    o->gh = bmaxy - bminy;
    o->scale = scale;
    const size_t ncell = (size_t)o->gw * o->gh;
    int* cellOf = (int*)malloc(sizeof(int) * (size_t)(nk ? nk : 1));
    o->cell_start = (int*)calloc(ncell + 1, sizeof(int));
    int accepted = 0;
    for (int k = 0; k < nk; k++)
    {
        int sx = (int)floorf(scale * s[k].x) - bminx;
        int sy = (int)floorf(scale * s[k].y) - bminy;
        if (sx < 0 || sy < 0 || sx >= o->gw || sy >= o->gh) { cellOf[k] = -1; continue; }
        cellOf[k] = sy * o->gw + sx;
        o->cell_start[cellOf[k] + 1]++;
        accepted++;
    }
    for (size_t c = 0; c < ncell; c++)
        o->cell_start[c + 1] += o->cell_start[c];
    o->cell_samples = (osample*)malloc(sizeof(osample) * (size_t)(accepted ? accepted : 1));
    int* cursor = (int*)malloc(sizeof(int) * ncell);
    memcpy(cursor, o->cell_start, sizeof(int) * ncell);
    for (int k = 0; k < nk; k++)
        if (cellOf[k] >= 0)
            o->cell_samples[cursor[cellOf[k]]++] = s[k];
    free(cursor);
    free(cellOf);
    free(s);
    if (accepted == 0)
    {
        snprintf(g_err, sizeof(g_err), "All samples were discarded in reprojection to (u,v,t)=0");
        return 0;
    }
    return 1;
}

static inline int cell_count(const oracle* o, int x, int y)
{
    int c = y * o->gw + x;
    return o->cell_start[c + 1] - o->cell_start[c];
}

/* ---- buildInitialRecursive, RTB.cpp:34-96 ---- */
static int build_initial(oracle* o, int* cap, int x0, int x1, int y0, int y1)
{
    const int dx = x1 - x0, dy = y1 - y0;
    const int idx = o->num_init;
    if (o->num_init == *cap)
    {
        *cap *= 2;
        o->init_nodes = (inode*)realloc(o->init_nodes, sizeof(inode) * (size_t)*cap);
    }
    o->num_init++;
    o->init_nodes[idx].x0 = x0; o->init_nodes[idx].x1 = x1;
    o->init_nodes[idx].y0 = y0; o->init_nodes[idx].y1 = y1;
    int leaf = imaxr(dx, dy) == 1;
    if (!leaf && dx * dy <= 64)
    {
        int ns = 0;
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++)
                ns += cell_count(o, x, y);
        leaf = (ns <= 48);
    }
    int c0, c1, ns = 0;
    if (leaf)
    {
        c0 = -1; c1 = -1;
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++)
                ns += cell_count(o, x, y);
    }
    else
    {
        if (dx > dy)
        {
            int xmid = (x1 + x0) / 2;
            c0 = build_initial(o, cap, x0, xmid, y0, y1);
            c1 = build_initial(o, cap, xmid, x1, y0, y1);
        }
        else
        {
            int ymid = (y1 + y0) / 2;
            c0 = build_initial(o, cap, x0, x1, y0, ymid);
            c1 = build_initial(o, cap, x0, x1, ymid, y1);
        }
        ns = o->init_nodes[c0].numSamples + o->init_nodes[c1].numSamples;
    }
    o->init_nodes[idx].child0 = c0;
    o->init_nodes[idx].child1 = c1;
    o->init_nodes[idx].numSamples = ns;
    return idx;
}

/* ---- per-task build state (BuildTask, R.hpp:250-280) ---- */

/* The four box arrays (RTB.cpp:159-169) are reused across all leaves of a task
 * and resized with Array::resize (Array.hpp:365-371, 668-692): contents are kept
 * up to the previous size; a reallocation (to 32 * 2^k elements of Vec2f:
 * MinBytes = 256) zero-fills everything beyond the previous size.  A candidate
 * whose bounds are invalid does not write its boxes (RTB.cpp:184-212), so it
 * reads whatever this state holds at its index. */
typedef struct
{
    oracle*   o;
    int       node;            /* entry point */
    int       sampleIndex;     /* currentSampleIndex */
    vec_node  hier;            /* private hierarchy, slot 0 reserved */
    vec_node  frontier;
    /* box arrays: [k][i] k = boxa, boxb, boxaT1, boxbT1 ; each Vec2f */
    float*    box[4];
    int       box_size, box_alloc;
    /* scratch */
    int*      perm;
    osample*  cand;
    int       cand_cap;
    tlb_t*    bounds;
    int*      surface;
    int       scratch_cap;
    int       num_invalid;
} btask;

static void box_resize(btask* bt, int n)
{
    if (n > bt->box_alloc)
    {
        int rounded = 32;
        while (n > rounded)
            rounded <<= 1;
        for (int k = 0; k < 4; k++)
        {
            float* np = (float*)calloc((size_t)rounded * 2, sizeof(float));
            int keep = iminr(rounded, bt->box_size);
            if (bt->box[k] && keep > 0)
                memcpy(np, bt->box[k], sizeof(float) * 2 * (size_t)keep);
            free(bt->box[k]);
            bt->box[k] = np;
        }
        bt->box_alloc = rounded;
    }
    bt->box_size = n;
}

/* sampleCompareFuncInc, RTB.cpp:99-117 */
static int cmp_tw(void* d, int a, int b)
{
    osample* s = (osample*)d;
    if (s[a].t < s[b].t) return -1;
    else if (s[a].t > s[b].t) return 1;
    else
    {
        if (s[a].w < s[b].w) return -1;
        else if (s[a].w > s[b].w) return 1;
        else return 0;
    }
}

static inline int ternary_compare(float a, float b, float eps)        /* R.hpp:428-436 */
{
    if (fabsf(a - b) < eps) return 0;
    else if (a < b) return -1;
    else return 1;
}
static inline int ternary_equal4(int a, int b, int c, int d)            /* R.hpp:444-449 */
{
    int mn = iminr(iminr(iminr(a, b), c), d);
    int mx = imaxr(imaxr(imaxr(a, b), c), d);
    return mx - mn < 2;
}
static inline int ternary_equal2(int a, int b) { return a == 0 || b == 0 || a == b; }   /* R.hpp:438-441 */

/* emitNodes, RTB.cpp:409-451 */
static void emit_nodes(int isRoot, int maxFrontier, vec_node* frontier, vec_node* hier)
{
    const int lim = isRoot ? 1 : maxFrontier;
    while (frontier->n > lim)
    {
        float minCost = F32_MAX;
        int mi = -1, mj = -1;
        for (int i = 0; i < frontier->n; i++)
            for (int j = i + 1; j < frontier->n; j++)
            {
                const onode* n0 = &frontier->p[i];
                const onode* n1 = &frontier->p[j];
                onode n01;
                node_merge(n0, n1, &n01);
                float cost = node_cost(&n01) - (node_cost(n0) + node_cost(n1));
                if (cost < minCost)
                {
                    minCost = cost;
                    mi = i; mj = j;
                }
            }
        if (mi < 0)
        {
            /* every pair cost was NaN or >= FLT_MAX; the reference would index
             * frontier[-1] here.  Not reached with finite bounds. */
            mi = 0; mj = 1;
        }
        onode n0 = frontier->p[mi], n1 = frontier->p[mj];
        onode n;
        node_merge(&n0, &n1, &n);
        n.child0 = hier->n; *vec_node_add(hier) = n0;
        n.child1 = hier->n; *vec_node_add(hier) = n1;
        frontier->p[mi] = n;
        frontier->p[mj] = frontier->p[frontier->n - 1];   /* removeSwap */
        frontier->n--;
    }
    if (isRoot)
    {
        hier->p[0] = frontier->p[frontier->n - 1];
        frontier->n--;
    }
}

/* buildRecursive, RTB.cpp:119-403 */
static void build_recursive(btask* bt, int nodeIndex, vec_node* frontier)
{
    if (nodeIndex == -1)
        return;
    oracle* o = bt->o;
    const inode* in = &o->init_nodes[nodeIndex];
    if (in->child0 == -1)
    {
        /* candidates in row-major cell order, bucket order within a cell */
        int n = 0;
        for (int y = in->y0; y < in->y1; y++)
            for (int x = in->x0; x < in->x1; x++)
                n += cell_count(o, x, y);
        if (n == 0)
            return;
        if (n > bt->cand_cap)
        {
            bt->cand_cap = n * 2;
            bt->cand = (osample*)realloc(bt->cand, sizeof(osample) * (size_t)bt->cand_cap);
        }
        if (n > bt->scratch_cap)
        {
            bt->scratch_cap = n * 2;
            bt->bounds = (tlb_t*)realloc(bt->bounds, sizeof(tlb_t) * (size_t)bt->scratch_cap);
            bt->surface = (int*)realloc(bt->surface, sizeof(int) * (size_t)bt->scratch_cap);
        }
        osample* cand = bt->cand;
        int k = 0;
        for (int y = in->y0; y < in->y1; y++)
            for (int x = in->x0; x < in->x1; x++)
            {
                int c = y * o->gw + x;
                for (int q = o->cell_start[c]; q < o->cell_start[c + 1]; q++)
                    cand[k++] = o->cell_samples[q];
            }
        const float bbmin[2] = { 0.0f, 0.0f };
        const float bbmax[2] = { (float)o->W, (float)o->H };
        fw_sort(0, n, cand, cmp_tw, swp_osample);

        box_resize(bt, n);
        float* boxa = bt->box[0]; float* boxb = bt->box[1];
        float* boxaT1 = bt->box[2]; float* boxbT1 = bt->box[3];
        tlb_t* bounds = bt->bounds;
        int* surface = bt->surface;
        const float* cc = o->cc;
        for (int i = 0; i < n; i++)
        {
            const osample* s = &cand[i];
            float xywt0[3] = { s->x * s->w - s->mv[0] * s->t, s->y * s->w - s->mv[1] * s->t, s->w - s->mv[2] * s->t };
            tux_planes(xywt0, s->mv, bbmin, bbmax, cc, &bounds[i]);
            if (tlb_valid(&bounds[i]))
            {
                float ta = bounds[i].tspan[0];
                float tb = bounds[i].tspan[1];
                float xywta[3], xywtb[3];
                float base[3] = { s->x * s->w, s->y * s->w, s->w };
                for (int q = 0; q < 3; q++)
                {
                    xywta[q] = base[q] + s->mv[q] * (ta - s->t);
                    xywtb[q] = base[q] + s->mv[q] * (tb - s->t);
                }
                float ca = rcpf_(xywta[2]), cb = rcpf_(xywtb[2]);
                float xyta[2] = { xywta[0] * ca, xywta[1] * ca };
                float xytb[2] = { xywtb[0] * cb, xywtb[1] * cb };
                float oodt = 1.0f / (tb - ta);
                float dxdt = (xytb[0] - xyta[0]) * oodt;
                float dydt = (xytb[1] - xyta[1]) * oodt;
                float xyt0[2] = { xyta[0] - dxdt * ta, xyta[1] - dydt * ta };
                float xyt1[2] = { xytb[0] + dxdt * (1.0f - tb), xytb[1] + dydt * (1.0f - tb) };
                float cocta = cc[0] / xywta[2] + cc[1];
                float coctb = cc[0] / xywtb[2] + cc[1];
                boxa[2 * i] = xyt0[0] + cocta;   boxa[2 * i + 1] = xyt0[1] + cocta;
                boxb[2 * i] = xyt0[0] - cocta;   boxb[2 * i + 1] = xyt0[1] - cocta;
                boxaT1[2 * i] = xyt1[0] + coctb; boxaT1[2 * i + 1] = xyt1[1] + coctb;
                boxbT1[2 * i] = xyt1[0] - coctb; boxbT1[2 * i + 1] = xyt1[1] - coctb;
            }
            else
                bt->num_invalid++;
        }

        /* surface scan, RTB.cpp:222-340 */
        frontier->n = 0;
        int surfacebegin = 0, currsurface = 0;
        surface[0] = 0;
        int reset = 1;
        float cb0[2] = { 0, 0 }, cb1[2] = { 0, 0 }, mvmin[2] = { 0, 0 }, mvmax[2] = { 0, 0 };
        float surfacet = 0.0f;
        const float TH = 1 * 2.0f;
        for (int cur = 1; cur < n; ++cur)
        {
            if (reset)
            {
                const int b = surfacebegin;
                cb0[0] = cb0[1] = 0.5f * (boxa[2 * b] - boxb[2 * b]);
                cb1[0] = cb1[1] = 0.5f * (boxaT1[2 * b] - boxbT1[2 * b]);
                for (int q = 0; q < 2; q++)
                    mvmin[q] = 0.5f * (boxaT1[2 * b + q] + boxbT1[2 * b + q]) - 0.5f * (boxa[2 * b + q] + boxb[2 * b + q]);
                mvmax[0] = mvmin[0]; mvmax[1] = mvmin[1];
                surfacet = cand[surfacebegin].t;
                reset = 0;
            }
            int conflict = 0, early = 0;
            if (surfacet != cand[cur].t)
            {
                surfacebegin = cur;
                surface[cur] = ++currsurface;
                reset = 1;
                continue;
            }
            float coct0 = 0.5f * (boxa[2 * cur] - boxb[2 * cur]);
            float coct1 = 0.5f * (boxaT1[2 * cur] - boxbT1[2 * cur]);
            float mv[2];
            for (int q = 0; q < 2; q++)
                mv[q] = 0.5f * (boxaT1[2 * cur + q] + boxbT1[2 * cur + q]) - 0.5f * (boxa[2 * cur + q] + boxb[2 * cur + q]);
            float e0 = fmaxr(fabsf(coct0 - cb0[0]), fabsf(coct0 - cb0[1]));
            float e1 = fmaxr(fabsf(coct1 - cb1[0]), fabsf(coct1 - cb1[1]));
            float a0 = fmaxr(fabsf(mvmin[0] - mv[0]), fabsf(mvmin[1] - mv[1]));
            float a1 = fmaxr(fabsf(mvmax[0] - mv[0]), fabsf(mvmax[1] - mv[1]));
            if (e0 < 0.5f * TH && e1 < 0.5f * TH && fmaxr(a0, a1) < TH)
                early = 1;
            if (!early)
            {
                for (int test = surfacebegin; test < cur; ++test)
                {
                    int bX = ternary_equal4(
                        ternary_compare(boxa[2 * test], boxa[2 * cur], TH),
                        ternary_compare(boxb[2 * test], boxb[2 * cur], TH),
                        ternary_compare(boxaT1[2 * test], boxaT1[2 * cur], TH),
                        ternary_compare(boxbT1[2 * test], boxbT1[2 * cur], TH));
                    int bY = ternary_equal4(
                        ternary_compare(boxa[2 * test + 1], boxa[2 * cur + 1], TH),
                        ternary_compare(boxb[2 * test + 1], boxb[2 * cur + 1], TH),
                        ternary_compare(boxaT1[2 * test + 1], boxaT1[2 * cur + 1], TH),
                        ternary_compare(boxbT1[2 * test + 1], boxbT1[2 * cur + 1], TH));
                    if (!(bX && bY))
                    {
                        surfacebegin = cur;
                        surface[cur] = ++currsurface;
                        conflict = 1;
                        reset = 1;
                        break;
                    }
                }
            }
            if (!conflict)
            {
                surface[cur] = currsurface;
                cb0[0] = fminr(coct0, cb0[0]);
                cb0[1] = fmaxr(coct0, cb0[0]);
                cb1[0] = fminr(coct1, cb1[0]);
                cb1[1] = fmaxr(coct1, cb1[0]);
                mvmin[0] = fminr(mvmin[0], mv[0]); mvmin[1] = fminr(mvmin[1], mv[1]);
                mvmax[0] = fmaxr(mvmax[0], mv[0]); mvmax[1] = fmaxr(mvmax[1], mv[1]);
            }
        }

        /* create nodes, RTB.cpp:345-378 */
        for (int i = 0; i < n;)
        {
            int j;
            for (j = i + 1; j < n && surface[i] == surface[j]; ++j) {}
            onode node;
            memset(&node, 0, sizeof(node));     /* default TimeLensBounds: planes 0, tspan 0 */
            node.s0 = bt->sampleIndex;
            node.child0 = -1;
            node.child1 = -1;
            for (int q = i; q < j; ++q)
            {
                o->samples[bt->sampleIndex++] = cand[q];
                tlb_t t;
                tlb_combine(&bounds[q], &node.tlb, &t);
                node.tlb = t;
            }
            node.s1 = bt->sampleIndex;
            node.ns = node.s1 - node.s0;
            *vec_node_add(frontier) = node;
            i = j;
        }
    }
    else
    {
        vec_node f1 = { 0 }, f2 = { 0 };
        build_recursive(bt, in->child0, &f1);
        build_recursive(bt, in->child1, &f2);
        frontier->n = 0;
        for (int k = 0; k < f1.n; k++) *vec_node_add(frontier) = f1.p[k];
        for (int k = 0; k < f2.n; k++) *vec_node_add(frontier) = f2.p[k];
        free(f1.p); free(f2.p);
        emit_nodes(nodeIndex == 0, 4, frontier, &bt->hier);
    }
}

static void* build_task_thread(void* arg)
{
    btask* bt = (btask*)arg;
    build_recursive(bt, bt->node, &bt->frontier);
    return NULL;
}

/* ---- TreeGather::init, R.cpp:52-215 ---- */
static int build(oracle* o, const float* rec)
{
    /* spp (R.cpp:63-73), roundUpToNearestPowerOfTwo Util.hpp:64-73 */
    uint32_t v = (uint32_t)o->spp_in;
    v--; v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    o->spp = imaxr(1, (int)(v + 1));

    if (!reproject_and_bucket(o, rec))
        return 0;

    /* initial hierarchy, R.cpp:103-107 */
    int cap = 1024;
    o->init_nodes = (inode*)malloc(sizeof(inode) * (size_t)cap);
    o->num_init = 0;
    build_initial(o, &cap, 0, o->gw, 0, o->gh);

    /* entry points, R.cpp:110-126 */
    int entry[32];
    for (int i = 0; i < 32; i++)
    {
        int node = 0;
        for (int j = 0; j < 5; j++)
        {
            if (node == -1)
                continue;
            int isLeaf = o->init_nodes[node].child0 == -1;
            if (i & (1 << j)) node = (!isLeaf) ? o->init_nodes[node].child1 : -1;
            else              node = (!isLeaf) ? o->init_nodes[node].child0 : node;
        }
        entry[i] = node;
    }

    o->num_samples = o->init_nodes[0].numSamples;
    o->samples = (osample*)calloc((size_t)(o->num_samples ? o->num_samples : 1), sizeof(osample));

    btask* bt = (btask*)calloc(32, sizeof(btask));
    int sampleIndex = 0;
    for (int i = 0; i < 32; i++)
    {
        bt[i].o = o;
        bt[i].node = entry[i];
        bt[i].sampleIndex = sampleIndex;
        vec_node_add(&bt[i].hier);              /* slot 0 reserved (R.hpp:261) */
        memset(&bt[i].hier.p[0], 0, sizeof(onode));
        bt[i].hier.p[0].child0 = -1;
        bt[i].hier.p[0].child1 = -1;
        bt[i].hier.p[0].s0 = -1;
        bt[i].hier.p[0].s1 = -1;
        if (entry[i] != -1)
            sampleIndex += o->init_nodes[entry[i]].numSamples;
    }

    /* 32 tasks (R.cpp:152-155) */
    int nth = o->nthreads > 0 ? o->nthreads : 1;
    if (nth > 1)
    {
        pthread_t th[32];
        for (int base = 0; base < 32; base += nth)
        {
            int cnt = iminr(nth, 32 - base);
            for (int k = 0; k < cnt; k++)
                pthread_create(&th[k], NULL, build_task_thread, &bt[base + k]);
            for (int k = 0; k < cnt; k++)
                pthread_join(th[k], NULL);
        }
    }
    else
        for (int i = 0; i < 32; i++)
            build_task_thread(&bt[i]);

    /* merge sub-hierarchies, R.cpp:159-188 */
    int numNodes = 0;
    for (int i = 0; i < 32; i++)
        numNodes += bt[i].hier.n;
    vec_node_reserve(&o->hier, numNodes + 64);
    o->hier.n = numNodes;
    int nodeBase = 0;
    for (int i = 0; i < 32; i++)
    {
        memcpy(&o->hier.p[nodeBase], bt[i].hier.p, sizeof(onode) * (size_t)bt[i].hier.n);
        for (int j = 0; j < bt[i].hier.n; j++)
        {
            onode* nd = &o->hier.p[nodeBase + j];
            if (nd->child0 != -1) nd->child0 += nodeBase;
            if (nd->child1 != -1) nd->child1 += nodeBase;
        }
        for (int j = 0; j < bt[i].frontier.n; j++)
        {
            if (bt[i].frontier.p[j].child0 != -1) bt[i].frontier.p[j].child0 += nodeBase;
            if (bt[i].frontier.p[j].child1 != -1) bt[i].frontier.p[j].child1 += nodeBase;
        }
        nodeBase += bt[i].hier.n;
    }

    /* serial top of tree, R.cpp:192-203 */
    for (int j = 0; j < 5; j++)
    {
        int offset = 1 << j;
        for (int i = 0; i < 32; i += 2 * offset)
        {
            for (int k = 0; k < bt[i + offset].frontier.n; k++)
                *vec_node_add(&bt[i].frontier) = bt[i + offset].frontier.p[k];
            emit_nodes(j == 4, 4, &bt[i].frontier, &o->hier);
        }
    }
    o->root = 0;
    o->num_invalid = 0;
    for (int i = 0; i < 32; i++)
    {
        o->num_invalid += bt[i].num_invalid;
        free(bt[i].hier.p); free(bt[i].frontier.p);
        for (int k = 0; k < 4; k++) free(bt[i].box[k]);
        free(bt[i].cand); free(bt[i].bounds); free(bt[i].surface); free(bt[i].perm);
    }
    free(bt);
    return 1;
}

/* ------------------------------------------------------------------------- */
/* Query (Filterer, RO.cpp:50-511).                                           */
/* ------------------------------------------------------------------------- */

typedef struct { float x, y; int index; int rpos; float key; } rsample;   /* ReconSample, R.hpp:124-132 */
typedef struct { int nodeIndex; float key; } leaf_t;                     /* R.hpp:353-357 */

typedef struct
{
    rsample* s;
    int      n, cap;
    float    minDist;
    int      minIndex;
    int      quadrantMask;
} surface_t;

typedef struct
{
    leaf_t*    leaves; int nleaves, capleaves;
    int*       stack;  int nstack, capstack;
    surface_t* surf;   int nsurf, capsurf;
} filterer;

typedef struct { double v[8][2]; } ostats;   /* Stats, R.hpp:134-147 (value, count) */

static int cmp_leaf(void* d, int a, int b)
{
    leaf_t* e = (leaf_t*)d;
    return (e[a].key < e[b].key) ? -1 : (e[a].key > e[b].key) ? 1 : 0;
}
static void swp_leaf(void* d, int a, int b)
{
    leaf_t* e = (leaf_t*)d;
    leaf_t t = e[a]; e[a] = e[b]; e[b] = t;
}

static void surf_add_sample(surface_t* s, const rsample* r)
{
    if (s->n == s->cap)
    {
        s->cap = s->cap ? 2 * s->cap : 64;
        s->s = (rsample*)realloc(s->s, sizeof(rsample) * (size_t)s->cap);
    }
    s->s[s->n++] = *r;
}

/* sameSurface, R.hpp:457-525 */
static int same_surface(const onode* n0, const onode* n1, const float uvtmin[3], const float uvtmax[3])
{
    const float TH = 1 * 0.1f;
    float tmid = 0.5f * (uvtmin[2] + uvtmax[2]);
    const tlb_t* a = &n0->tlb;
    const tlb_t* b = &n1->tlb;
    float Xmin00 = tlb_eval(a, 0, tmid, uvtmin[0]), Xmin10 = tlb_eval(a, 0, tmid, uvtmax[0]);
    float Xmax00 = tlb_eval(a, 1, tmid, uvtmin[0]), Xmax10 = tlb_eval(a, 1, tmid, uvtmax[0]);
    float Ymin00 = tlb_eval(a, 2, tmid, uvtmin[1]), Ymin10 = tlb_eval(a, 2, tmid, uvtmax[1]);
    float Ymax00 = tlb_eval(a, 3, tmid, uvtmin[1]), Ymax10 = tlb_eval(a, 3, tmid, uvtmax[1]);
    float Xmin01 = tlb_eval(b, 0, tmid, uvtmin[0]), Xmin11 = tlb_eval(b, 0, tmid, uvtmax[0]);
    float Xmax01 = tlb_eval(b, 1, tmid, uvtmin[0]), Xmax11 = tlb_eval(b, 1, tmid, uvtmax[0]);
    float Ymin01 = tlb_eval(b, 2, tmid, uvtmin[1]), Ymin11 = tlb_eval(b, 2, tmid, uvtmax[1]);
    float Ymax01 = tlb_eval(b, 3, tmid, uvtmin[1]), Ymax11 = tlb_eval(b, 3, tmid, uvtmax[1]);
    int bCoC =
        ternary_equal2(ternary_compare(Xmin00, Xmin01, TH), ternary_compare(Xmin10, Xmin11, TH)) &&
        ternary_equal2(ternary_compare(Ymin00, Ymin01, TH), ternary_compare(Ymin10, Ymin11, TH)) &&
        ternary_equal2(ternary_compare(Xmax00, Xmax01, TH), ternary_compare(Xmax10, Xmax11, TH)) &&
        ternary_equal2(ternary_compare(Ymax00, Ymax01, TH), ternary_compare(Ymax10, Ymax11, TH));
    if (!bCoC)
        return 0;
    float xa0 = tlb_eval(a, 0, uvtmin[2], 0.0f), xb0 = tlb_eval(a, 0, uvtmax[2], 0.0f);
    float ya0 = tlb_eval(a, 2, uvtmin[2], 0.0f), yb0 = tlb_eval(a, 2, uvtmax[2], 0.0f);
    float Xa0 = tlb_eval(a, 1, uvtmin[2], 0.0f), Xb0 = tlb_eval(a, 1, uvtmax[2], 0.0f);
    float Ya0 = tlb_eval(a, 3, uvtmin[2], 0.0f), Yb0 = tlb_eval(a, 3, uvtmax[2], 0.0f);
    float xa1 = tlb_eval(b, 0, uvtmin[2], 0.0f), xb1 = tlb_eval(b, 0, uvtmax[2], 0.0f);
    float ya1 = tlb_eval(b, 2, uvtmin[2], 0.0f), yb1 = tlb_eval(b, 2, uvtmax[2], 0.0f);
    float Xa1 = tlb_eval(b, 1, uvtmin[2], 0.0f), Xb1 = tlb_eval(b, 1, uvtmax[2], 0.0f);
    float Ya1 = tlb_eval(b, 3, uvtmin[2], 0.0f), Yb1 = tlb_eval(b, 3, uvtmax[2], 0.0f);
    return ternary_equal2(ternary_compare(xa0, xa1, TH), ternary_compare(xb0, xb1, TH)) &&
           ternary_equal2(ternary_compare(Xa0, Xa1, TH), ternary_compare(Xb0, Xb1, TH)) &&
           ternary_equal2(ternary_compare(ya0, ya1, TH), ternary_compare(yb0, yb1, TH)) &&
           ternary_equal2(ternary_compare(Ya0, Ya1, TH), ternary_compare(Yb0, Yb1, TH));
}

/* Node::intersect, R.hpp:204-216 */
static int node_intersect(const onode* n, const osample* s, float R)
{
    float mnx = tlb_eval(&n->tlb, 0, s->t, s->u) - R;
    float mny = tlb_eval(&n->tlb, 2, s->t, s->v) - R;
    float mxx = tlb_eval(&n->tlb, 1, s->t, s->u) + R;
    float mxy = tlb_eval(&n->tlb, 3, s->t, s->v) + R;
    return (s->x >= mnx && s->y >= mny && s->x <= mxx && s->y <= mxy);
}

/* collectInputSamples2, RO.cpp:361-511 */
static int collect(const oracle* o, filterer* f, const osample* q, float R, ostats* st)
{
    f->nleaves = 0;
    f->nstack = 0;
    f->stack[f->nstack++] = o->root;
    while (f->nstack > 0)
    {
        const int ni = f->stack[--f->nstack];
        const onode* node = &o->hier.p[ni];
        if (node_intersect(node, q, R))
        {
            if (node->child0 == -1)
            {
                if (f->nleaves == f->capleaves)
                {
                    f->capleaves *= 2;
                    f->leaves = (leaf_t*)realloc(f->leaves, sizeof(leaf_t) * (size_t)f->capleaves);
                }
                const osample* s = &o->samples[node->s0];
                f->leaves[f->nleaves].nodeIndex = ni;
                f->leaves[f->nleaves].key = s->w + (q->t - s->t) * s->mv[2];
                f->nleaves++;
            }
            else
            {
                if (f->nstack + 2 > f->capstack)
                {
                    f->capstack *= 2;
                    f->stack = (int*)realloc(f->stack, sizeof(int) * (size_t)f->capstack);
                }
                f->stack[f->nstack++] = node->child0;
                f->stack[f->nstack++] = node->child1;
            }
        }
    }
    st->v[0][0] += f->nleaves;
    fw_sort(0, f->nleaves, f->leaves, cmp_leaf, swp_leaf);

    f->nsurf = 0;
    int total = 0, surfaceStart = 0;
    const float RANGE = 1.0f / sqrtf(128.0f);
    float uvtmin[3] = { q->u - RANGE, q->v - RANGE, q->t - 0.5f * RANGE };
    float uvtmax[3] = { q->u + RANGE, q->v + RANGE, q->t + 0.5f * RANGE };
    for (int lidx = 0; lidx < f->nleaves; lidx++)
    {
        int first = 1;
        const onode* node = &o->hier.p[f->leaves[lidx].nodeIndex];
        st->v[1][0] += node->ns;
        for (int i = node->s0; i < node->s1; i++)
        {
            const osample* s = &o->samples[i];
            float x, y, w;
            if (s->mv[0] != 0.0f || s->mv[1] != 0.0f || s->mv[2] != 0.0f)
            {
                float P0[3] = { s->x * s->w, s->y * s->w, 1.0f * s->w };
                float dt = q->t - s->t;
                float P[3] = { P0[0] + s->mv[0] * dt, P0[1] + s->mv[1] * dt, P0[2] + s->mv[2] * dt };
                w = P[2];
                float c = rcpf_(P[2]);
                float coc = coc_radius(o->cc, w);
                x = P[0] * c + q->u * coc;
                y = P[1] * c + q->v * coc;
            }
            else
            {
                w = s->w;
                float coc = coc_radius(o->cc, s->w);
                x = s->x + q->u * coc;
                y = s->y + q->v * coc;
            }
            float dx = x - q->x, dy = y - q->y;
            float dist2 = dx * dx + dy * dy;
            if (dist2 <= R * R)
            {
                rsample r;
                r.x = x; r.y = y;
                r.rpos = (dx >= 0 ? 1 : 4) | (dy >= 0 ? 2 : 8);
                r.key = w;
                r.index = i;
                if (first)
                {
                    first = 0;
                    int same = 1;
                    for (int j = surfaceStart; j < lidx && same; ++j)
                        same = same_surface(node, &o->hier.p[f->leaves[j].nodeIndex], uvtmin, uvtmax);
                    if (!same || f->nsurf == 0)
                    {
                        surfaceStart = lidx;
                        if (f->nsurf == f->capsurf)
                        {
                            int nc = f->capsurf * 2;
                            f->surf = (surface_t*)realloc(f->surf, sizeof(surface_t) * (size_t)nc);
                            memset(f->surf + f->capsurf, 0, sizeof(surface_t) * (size_t)(nc - f->capsurf));
                            f->capsurf = nc;
                        }
                        surface_t* sf = &f->surf[f->nsurf++];
                        sf->n = 0;
                        sf->minDist = F32_MAX;
                        sf->minIndex = -1;
                        sf->quadrantMask = 0;
                    }
                }
                surface_t* sf = &f->surf[f->nsurf - 1];
                surf_add_sample(sf, &r);
                sf->quadrantMask |= (1 << (r.rpos & 3));
                float dist = sqrtf(dist2);
                if (dist < sf->minDist)
                {
                    sf->minDist = dist;
                    sf->minIndex = sf->n - 1;
                }
                total++;
            }
        }
    }
    st->v[3][0] += total;
    return total;
}

/* EdgeFunction, EF.cpp:39-45, EF.hpp:45-47 */
typedef struct { double A, B, C; int acceptEqual; } edgefn;
static void edge_init(edgefn* e, double x0, double y0, double x1, double y1)
{
    e->A = y0 - y1;
    e->B = x1 - x0;
    e->C = (-x0) * e->A - y0 * e->B;
    e->acceptEqual = (e->A == 0.) ? (e->B > 0.) : (e->A > 0.);
}
static inline float edge_eval(const edgefn* e, double x, double y) { return (float)((x * e->A + y * e->B) + e->C); }
static inline int edge_test(const edgefn* e, float d) { return d > 0.f ? 1 : (d == 0.f && e->acceptEqual); }

static inline float len2f(float dx, float dy) { return sqrtf(dx * dx + dy * dy); }

/* Gaussian, R.hpp:378 */
static float gaussian(float x, float stddev, float mean)
{
    float e = 2.718281828f;
    return powf(e, -((x - mean) * (x - mean)) / (2.0f * (stddev * stddev)));
}

/* Filterer::reconstruct, RO.cpp:50-359.  trace: see ref_query. */
static void reconstruct_one(const oracle* o, filterer* f, const osample* q, ostats* st, float rgba[4],
                            int* trace, int trace_cap, int* trace_len)
{
    float dispersion;
    switch (o->spp)
    {
    case 256: dispersion = 0.14f; break;
    case 128: dispersion = 0.18f; break;
    case 64:  dispersion = 0.27f; break;
    case 32:  dispersion = 0.37f; break;
    case 16:  dispersion = 0.50f; break;
    case 8:   dispersion = 0.80f; break;
    case 4:   dispersion = 1.10f; break;
    case 2:   dispersion = 1.34f; break;
    default:  dispersion = 2.00f; break;   /* case 1 (other values fail at create) */
    }
    int flags = 0;
    int n1 = collect(o, f, q, dispersion, st);
    int n2 = 0, nN = 0;
    const int fetch2R = f->nsurf == 0 || (f->surf[0].quadrantMask != 0xF && f->nsurf > 1);
    if (fetch2R)
    {
        flags |= 1;
        n2 = collect(o, f, q, dispersion * 2, st);
        if (n2 == 0)
        {
            flags |= 2;
            st->v[7][0] += 1;
            nN = n2;
            for (int k = 0; k < 3 && !nN; k++)
            {
                dispersion *= 2.f;
                nN = collect(o, f, q, dispersion * 2, st);
            }
        }
    }
    st->v[5][0] += fetch2R ? 1 : 0;
    st->v[2][0] += n1;
    (void)nN;

    int numSurfaces = f->nsurf;
    if (fetch2R)
        for (int sidx = 0; sidx < f->nsurf - 1; sidx++)
        {
            surface_t* src = &f->surf[sidx];
            if (src->n < 4)
            {
                surface_t* dst = &f->surf[sidx + 1];
                for (int k = 0; k < src->n; k++)
                    surf_add_sample(dst, &src->s[k]);
                src->n = 0;
                if (src->minDist < dst->minDist)
                {
                    dst->minDist = src->minDist;
                    dst->minIndex = src->minIndex;
                }
                numSurfaces--;
            }
        }
    st->v[4][0] += numSurfaces;
    if (numSurfaces != f->nsurf)
    {
        st->v[6][0] += 1;
        flags |= 4;
    }

    int found = 0;
    float res[4] = { 0, 0, 0, 0 };
    float nearestDist = F32_MAX;
    int nearS = -1, nearI = 1;
    for (int sidx = 0; sidx < f->nsurf && !found; sidx++)
    {
        const surface_t* sf = &f->surf[sidx];
        const rsample* in = sf->s;
        const int n = sf->n;
        if (n == 0)
            continue;
        if (sf->minDist < nearestDist)
        {
            nearestDist = sf->minDist;
            nearS = sidx; nearI = sf->minIndex;
        }
        if (!fetch2R || sf->minDist < 0.f || sidx == f->nsurf - 1)
            found = 1;
        if (n >= 200)
            found = 1;
        for (int m = 0; m < n - 2 && !found; m++)
            for (int k = m + 1; k < n - 1 && !found; k++)
                for (int l = k + 1; l < n && !found; l++)
                {
                    const rsample* r0 = &in[m];
                    const rsample* r1 = &in[k];
                    const rsample* r2 = &in[l];
                    if ((r0->rpos | r1->rpos | r2->rpos) != 15)
                        continue;
                    if (len2f(r0->x - r1->x, r0->y - r1->y) > 2 * dispersion ||
                        len2f(r0->x - r2->x, r0->y - r2->y) > 2 * dispersion ||
                        len2f(r1->x - r2->x, r1->y - r2->y) > 2 * dispersion)
                        continue;
                    if (len2f(r0->x - q->x, r0->y - q->y) > dispersion &&
                        len2f(r1->x - q->x, r1->y - q->y) > dispersion &&
                        len2f(r2->x - q->x, r2->y - q->y) > dispersion)
                        continue;
                    edgefn e0, e1, e2;
                    edge_init(&e0, r1->x, r1->y, r2->x, r2->y);
                    edge_init(&e1, r2->x, r2->y, r0->x, r0->y);
                    edge_init(&e2, r0->x, r0->y, r1->x, r1->y);
                    float d0 = edge_eval(&e0, q->x, q->y);
                    float d1 = edge_eval(&e1, q->x, q->y);
                    float d2 = edge_eval(&e2, q->x, q->y);
                    int p0 = edge_test(&e0, d0), p1 = edge_test(&e1, d1), p2 = edge_test(&e2, d2);
                    found = (p0 && p1 && p2) || (!p0 && !p1 && !p2);
                }
        if (found)
        {
            res[0] = res[1] = res[2] = res[3] = 0.0f;
            for (int k = 0; k < n; k++)
            {
                const rsample* r = &in[k];
                const osample* s = &o->samples[r->index];
                float dx = q->x - r->x, dy = q->y - r->y;
                float weight = 1 - len2f(dx, dy) / dispersion;
                if (weight <= 0)
                    continue;
                for (int c = 0; c < 4; c++)
                    res[c] += s->col[c] * weight;
            }
            float oow = rcpf_(res[3]);
            for (int c = 0; c < 4; c++)
                res[c] *= oow;
            nearS = sidx; nearI = sf->minIndex;
        }
    }

    if (trace)
    {
        int tn = 0;
#define PUT(v) do { if (tn < trace_cap) trace[tn] = (v); tn++; } while (0)
        PUT(flags);
        PUT(f->nsurf);
        for (int s = 0; s < f->nsurf; s++)
        {
            PUT(f->surf[s].n);
            PUT(f->surf[s].minIndex);
            for (int k = 0; k < f->surf[s].n; k++)
                PUT(f->surf[s].s[k].index);
        }
#undef PUT
        *trace_len = (tn <= trace_cap) ? tn : -1;
    }

    if (nearS == -1)
    {
        rgba[0] = rgba[1] = rgba[2] = rgba[3] = 0.0f;
        return;
    }
    const rsample* na = &f->surf[nearS].s[nearI];
    const osample* nearest = &o->samples[na->index];
    if (res[3] == 0)
        for (int c = 0; c < 4; c++)
            res[c] = nearest->col[c];
    if (o->lens_filter == 1)
    {
        float g = gaussian(q->u, 0.5f, 0) * gaussian(q->v, 0.5f, 0);
        for (int c = 0; c < 4; c++) res[c] *= g;
    }
    if (o->time_filter == 1)
    {
        float g = gaussian(q->t, 0.25f, 0.5f);
        for (int c = 0; c < 4; c++) res[c] *= g;
    }
    for (int c = 0; c < 4; c++)
        rgba[c] = res[c];
}

static void filterer_init(filterer* f)
{
    memset(f, 0, sizeof(*f));
    f->capleaves = 128; f->leaves = (leaf_t*)malloc(sizeof(leaf_t) * 128);
    f->capstack = 128;  f->stack = (int*)malloc(sizeof(int) * 128);
    f->capsurf = 32;    f->surf = (surface_t*)calloc(32, sizeof(surface_t));
}

static void filterer_free(filterer* f)
{
    for (int k = 0; k < f->capsurf; k++)
        free(f->surf[k].s);
    free(f->surf); free(f->leaves); free(f->stack);
}

/* output sample i of pixel (x, y): FilterTask::process, R.cpp:653, 692-693 */
static void make_query(const oracle* o, int x, int y, int i, osample* q)
{
    int pattern = (int)(hash_bits((uint32_t)x, (uint32_t)y, 0) % 64u);
    *q = o->outs[pattern * o->out_spp + i];
    q->x += (float)x;
    q->y += (float)y;
}

/* FilterTask::process(pixel), R.cpp:649-720 */
static void process_pixel(const oracle* o, filterer* f, int x, int y, ostats* st, float out[4])
{
    float pc[4] = { 0, 0, 0, 0 };
    for (int i = 0; i < o->out_spp; i++)
    {
        osample q;
        make_query(o, x, y, i, &q);
        float c[4];
        reconstruct_one(o, f, &q, st, c, NULL, 0, NULL);
        for (int k = 0; k < 4; k++)
            pc[k] += c[k];
    }
    if (pc[3] == 0)
    {
        pc[0] = 1; pc[1] = 0; pc[2] = 0; pc[3] = 1;
    }
    float r = rcpf_(pc[3]);
    for (int k = 0; k < 4; k++)
        out[k] = pc[k] * r;
}

typedef struct
{
    const oracle* o;
    float*  rgba;
    int     y0, y1, row_base;
    int*    next_row;
    pthread_mutex_t* lock;
    ostats  st;
} rowjob;

static void* row_thread(void* arg)
{
    rowjob* j = (rowjob*)arg;
    filterer f;
    filterer_init(&f);
    for (;;)
    {
        pthread_mutex_lock(j->lock);
        int y = (*j->next_row)++;
        pthread_mutex_unlock(j->lock);
        if (y >= j->y1)
            break;
        for (int x = 0; x < j->o->W; x++)
            process_pixel(j->o, &f, x, y, &j->st, j->rgba + ((size_t)(y - j->row_base) * j->o->W + x) * 4);
    }
    filterer_free(&f);
    return NULL;
}

static void run_rows(const oracle* o, int y0, int y1, float* rgba, int row_base, double* stats)
{
    int nth = o->nthreads > 0 ? o->nthreads : 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nth);
    rowjob* jobs = (rowjob*)calloc((size_t)nth, sizeof(rowjob));
    pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
    int next = y0;
    for (int k = 0; k < nth; k++)
    {
        jobs[k].o = o; jobs[k].rgba = rgba; jobs[k].y0 = y0; jobs[k].y1 = y1;
        jobs[k].row_base = row_base; jobs[k].next_row = &next; jobs[k].lock = &lock;
        pthread_create(&th[k], NULL, row_thread, &jobs[k]);
    }
    for (int k = 0; k < nth; k++)
        pthread_join(th[k], NULL);
    if (stats)
    {
        memset(stats, 0, sizeof(double) * 16);
        double nq = (double)(y1 - y0) * o->W * o->out_spp;
        for (int k = 0; k < nth; k++)
            for (int s = 0; s < 8; s++)
                stats[2 * s] += jobs[k].st.v[s][0];
        for (int s = 0; s < 8; s++)
            stats[2 * s + 1] = nq;
    }
    free(th);
    free(jobs);
}

/* ------------------------------------------------------------------------- */
/* API                                                                        */
/* ------------------------------------------------------------------------- */

int orc_create(const float* records, int W, int H, int spp, float C0, float C1,
               float aperture, float focus, const float* uvt, int lens_filter, int time_filter,
               int output_spp, int nthreads, void** out, double* build_seconds)
{
    if (!records || W <= 0 || H <= 0 || spp <= 0 || !out)
    {
        snprintf(g_err, sizeof(g_err), "bad argument");
        return 1;
    }
    sobol3_init();
    oracle* o = (oracle*)calloc(1, sizeof(oracle));
    o->W = W; o->H = H; o->spp_in = spp;
    o->cc0[0] = C0; o->cc0[1] = C1;
    /* refocus round trip, R.cpp:77-87 */
    {
        float ccx = C0, ccy = C1;
        float a = -ccx;
        float f = (-ccx) * rcpf_(ccy);
        a *= aperture;
        f *= focus;
        o->cc[0] = -a;
        o->cc[1] = a * rcpf_(f);
    }
    o->lens_filter = lens_filter;
    o->time_filter = time_filter;
    o->override_uvt = uvt != NULL;
    if (uvt) { o->uvt[0] = uvt[0]; o->uvt[1] = uvt[1]; o->uvt[2] = uvt[2]; }
    o->out_spp = output_spp > 0 ? output_spp : (uvt ? 1 : 128);
    o->nthreads = nthreads > 0 ? nthreads : 1;
    double t0 = now_s();
    if (!build(o, records))
    {
        orc_destroy(o);
        return 1;
    }
    if (build_seconds)
        *build_seconds = now_s() - t0;
    if (o->spp > 256)
    {
        snprintf(g_err, sizeof(g_err), "TreeGather::Filterer::reconstruct -- unknown SPP");
        orc_destroy(o);
        return 1;
    }
    generate_output_samples(o);
    *out = o;
    return 0;
}

int orc_reconstruct(void* h, float* rgba, double* seconds, double* stats)
{
    oracle* o = (oracle*)h;
    double t0 = now_s();
    run_rows(o, 0, o->H, rgba, 0, stats);
    if (seconds)
        *seconds = now_s() - t0;
    return 0;
}

int orc_reconstruct_rows(void* h, int y0, int y1, float* rgba_rows, double* seconds)
{
    oracle* o = (oracle*)h;
    if (y0 < 0 || y1 > o->H || y0 >= y1)
        return 1;
    double t0 = now_s();
    run_rows(o, y0, y1, rgba_rows, y0, NULL);
    if (seconds)
        *seconds = now_s() - t0;
    return 0;
}

static int node_height(const oracle* o, int ni)
{
    /* iterative max depth */
    int best = 0;
    int cap = 256, n = 0;
    int* st = (int*)malloc(sizeof(int) * 2 * (size_t)cap);
    st[n * 2] = ni; st[n * 2 + 1] = 1; n++;
    while (n)
    {
        n--;
        int id = st[n * 2], d = st[n * 2 + 1];
        if (d > best) best = d;
        const onode* nd = &o->hier.p[id];
        if (nd->child0 != -1)
        {
            if (n + 2 > cap) { cap *= 2; st = (int*)realloc(st, sizeof(int) * 2 * (size_t)cap); }
            st[n * 2] = nd->child0; st[n * 2 + 1] = d + 1; n++;
            st[n * 2] = nd->child1; st[n * 2 + 1] = d + 1; n++;
        }
    }
    free(st);
    return best;
}

int orc_tree_info(void* h, int* num_nodes, int* num_samples, int* root, int* spp_pow2,
                  float* coc_adjusted, int* output_spp, int* height)
{
    oracle* o = (oracle*)h;
    if (num_nodes) *num_nodes = o->hier.n;
    if (num_samples) *num_samples = o->num_samples;
    if (root) *root = o->root;
    if (spp_pow2) *spp_pow2 = o->spp;
    if (coc_adjusted) { coc_adjusted[0] = o->cc[0]; coc_adjusted[1] = o->cc[1]; }
    if (output_spp) *output_spp = o->out_spp;
    if (height) *height = node_height(o, o->root);
    return 0;
}

int orc_grid_info(void* h, int* grid_w, int* grid_h, float* scale, int* num_initial_nodes, int* num_invalid_bounds)
{
    oracle* o = (oracle*)h;
    if (grid_w) *grid_w = o->gw;
    if (grid_h) *grid_h = o->gh;
    if (scale) *scale = o->scale;
    if (num_initial_nodes) *num_initial_nodes = o->num_init;
    if (num_invalid_bounds) *num_invalid_bounds = o->num_invalid;
    return 0;
}

int orc_tree_export(void* h, float* nodef, int* nodei, float* samplef, int* sample_ids)
{
    oracle* o = (oracle*)h;
    for (int i = 0; i < o->hier.n; i++)
    {
        const onode* n = &o->hier.p[i];
        if (nodef)
        {
            for (int p = 0; p < 4; p++)
                for (int k = 0; k < 3; k++)
                    nodef[i * 14 + p * 3 + k] = n->tlb.planes[p][k];
            nodef[i * 14 + 12] = n->tlb.tspan[0];
            nodef[i * 14 + 13] = n->tlb.tspan[1];
        }
        if (nodei)
        {
            int leaf = n->child0 == -1;
            nodei[i * 5 + 0] = n->child0;
            nodei[i * 5 + 1] = n->child1;
            nodei[i * 5 + 2] = leaf ? n->s0 : -1;
            nodei[i * 5 + 3] = leaf ? n->s1 : -1;
            nodei[i * 5 + 4] = n->ns;
        }
    }
    for (int j = 0; j < o->num_samples; j++)
    {
        const osample* s = &o->samples[j];
        if (samplef)
        {
            float* d = samplef + (size_t)j * 12;
            d[0] = s->x; d[1] = s->y; d[2] = s->w; d[3] = s->t;
            d[4] = s->mv[0]; d[5] = s->mv[1]; d[6] = s->mv[2];
            d[7] = s->col[0]; d[8] = s->col[1]; d[9] = s->col[2]; d[10] = s->col[3];
            d[11] = s->key;
        }
        if (sample_ids)
            sample_ids[j] = s->id;
    }
    return 0;
}

int orc_output_samples(void* h, float* out5)
{
    oracle* o = (oracle*)h;
    const int n = 64 * o->out_spp;
    for (int i = 0; i < n; i++)
    {
        out5[i * 5 + 0] = o->outs[i].x; out5[i * 5 + 1] = o->outs[i].y;
        out5[i * 5 + 2] = o->outs[i].u; out5[i * 5 + 3] = o->outs[i].v;
        out5[i * 5 + 4] = o->outs[i].t;
    }
    return n;
}

int orc_query(void* h, int x, int y, int i, float* rgba, int* trace, int trace_cap)
{
    oracle* o = (oracle*)h;
    static __thread filterer* f = NULL;
    if (!f)
    {
        f = (filterer*)malloc(sizeof(filterer));
        filterer_init(f);
    }
    osample q;
    make_query(o, x, y, i, &q);
    ostats st;
    memset(&st, 0, sizeof(st));
    int tl = 0;
    reconstruct_one(o, f, &q, &st, rgba, trace, trace_cap, &tl);
    return trace ? tl : 0;
}

void orc_destroy(void* h)
{
    oracle* o = (oracle*)h;
    if (!o)
        return;
    free(o->cell_start);
    free(o->cell_samples);
    free(o->init_nodes);
    free(o->samples);
    free(o->hier.p);
    free(o->outs);
    free(o);
}
