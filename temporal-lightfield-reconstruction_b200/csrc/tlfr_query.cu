// tlfr_query.cu — per-output-sample reconstruction on the GPU.
//
// Every output sample (x, y, u, v, t) is answered with the reference's Filterer
// (reconstruction/ReconstructionOur.cpp:50-511):
//   collect(R)   traversal (DFS, child1 popped first), leaf sort by w at the
//                output time (FW::sort), per-sample reprojection and R test, and
//                surface separation with sameSurface (Reconstruction.hpp:457-525)
//   fetch2R      2R refetch and up to three widenings (RO.cpp:94-121)
//   merge        tiny-surface merging (RO.cpp:137-156)
//   resolve      per surface front to back: nearest tracking, coverage by
//                triangles with double-precision edge functions, tent filter
//                (RO.cpp:165-304), nearest-sample fallback (RO.cpp:318-348)
// Pixels are the sum of their output samples normalised by alpha, red when
// nothing was found (Reconstruction.cpp:649-720).
//
// The work runs in passes:
//   k_query_light     every output sample: each lane collects its own leaves at
//                     1R into shared memory, then the warp scans each lane's
//                     sample in turn; settles the samples the 1R fetch settles
//                     (fetch2R false) and queues the rest
//   k_query_coop      the queue, warp-cooperatively: the full path from the 2R
//                     fetch (or from 1R for samples that outgrew the light pass)
//   k_query_overflow  the few samples that outgrow the cooperative pass's lists,
//                     with large capacities from a global arena; a sample that
//                     outgrows those too is reported as TLFR_OVERFLOW
//   k_resolve         pixels from their output samples in sample order
// plus the statistics, trace and allocation-free variants of the full path, the
// router's probe pass, and the capture-safe frame pipeline used by batches.
#include "tlfr_common.cuh"
#include "tlfr_internal.h"

#include <array>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace tlfr
{

namespace
{

struct Leaf { int node; float key; };
struct RSample { float x, y; int index; int rpos; };        // ReconSample (Reconstruction.hpp:124-132)
struct Surf { int start, n; float minDist; int minIndex; int quad; };

struct Store
{
    int*     stack;   int stack_cap;
    Leaf*    leaves;  int leaf_cap;
    RSample* rs;      int rs_cap;
    Surf*    surf;    int surf_cap;
};

struct QParams
{
    const QNode*  nodes;
    const float4* s_rec;        // 2 per sample: (x, y, w, t), (mv, coc radius at w)
    const float4* s_col;
    const float*  pattern;      // 64 * M * 5
    int   M, W, H, root;
    float c0, c1;               // refocused CoC coefficients
    float disp0;
    int   lens_filter, time_filter;
    const unsigned char* route_fast;   // per pixel, nonzero: first-surface fast path (or null)
};

struct QStats
{
    unsigned leaves, in_leaves, within1r, fetched, surfaces, two_r, merged, at_least_one, empty;
    int overflow_reason;        // 0, or the capacity that was exceeded (1..4)
};

struct Query { float x, y, u, v, t; };

// Sample record i (32 bytes, 32-byte aligned) in one 256-bit load.
TLFR_HD void load_sample(const float4* rec, int i, float4& pos, float4& mot)
{
#ifdef __CUDA_ARCH__
    asm("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(pos.x), "=f"(pos.y), "=f"(pos.z), "=f"(pos.w), "=f"(mot.x), "=f"(mot.y), "=f"(mot.z), "=f"(mot.w)
        : "l"(rec + 2 * (size_t)i));
#else
    pos = rec[2 * (size_t)i];
    mot = rec[2 * (size_t)i + 1];
#endif
}



enum { kQOk = 0, kQOverflow = 1 };

// Node i (64 bytes, 64-byte aligned) in two 256-bit loads.
TLFR_HD QNode load_node(const QNode* nodes, int i)
{
#ifdef __CUDA_ARCH__
    unsigned u[16];
    const QNode* p = nodes + i;
    asm("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(u[0]), "=r"(u[1]), "=r"(u[2]), "=r"(u[3]), "=r"(u[4]), "=r"(u[5]), "=r"(u[6]), "=r"(u[7])
        : "l"(p));
    asm("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=r"(u[8]), "=r"(u[9]), "=r"(u[10]), "=r"(u[11]), "=r"(u[12]), "=r"(u[13]), "=r"(u[14]), "=r"(u[15])
        : "l"(reinterpret_cast<const char*>(p) + 32));
    QNode n;
    n.a = make_float4(__uint_as_float(u[0]), __uint_as_float(u[1]), __uint_as_float(u[2]), __uint_as_float(u[3]));
    n.b = make_float4(__uint_as_float(u[4]), __uint_as_float(u[5]), __uint_as_float(u[6]), __uint_as_float(u[7]));
    n.c = make_float4(__uint_as_float(u[8]), __uint_as_float(u[9]), __uint_as_float(u[10]), __uint_as_float(u[11]));
    n.d = make_int4((int)u[12], (int)u[13], (int)u[14], (int)u[15]);
    return n;
#else
    return nodes[i];
#endif
}

struct LeafSort
{
    Leaf* l;
    TLFR_HD int cmp(int a, int b) const { return (l[a].key < l[b].key) ? -1 : (l[a].key > l[b].key) ? 1 : 0; }
    TLFR_HD void swap(int a, int b) { Leaf t = l[a]; l[a] = l[b]; l[b] = t; }
};

TLFR_HD void node_planes(const QNode& n, float (&p)[4][3])
{
    p[0][0] = n.a.x; p[0][1] = n.a.y; p[0][2] = n.a.z;
    p[1][0] = n.a.w; p[1][1] = n.b.x; p[1][2] = n.b.y;
    p[2][0] = n.b.z; p[2][1] = n.b.w; p[2][2] = n.c.x;
    p[3][0] = n.c.y; p[3][1] = n.c.z; p[3][2] = n.c.w;
}

// sameSurface (Reconstruction.hpp:457-525)
TLFR_HD bool same_surface(const QNode& n0, const QNode& n1, const float* uvtmin, const float* uvtmax)
{
    const float TH = 1 * 0.1f;
    float a[4][3], b[4][3];
    node_planes(n0, a);
    node_planes(n1, b);
    float tmid = 0.5f * (uvtmin[2] + uvtmax[2]);
    bool bCoC =
        ternary_equal2(ternary_compare(plane_eval(a[0], tmid, uvtmin[0]), plane_eval(b[0], tmid, uvtmin[0]), TH),
                       ternary_compare(plane_eval(a[0], tmid, uvtmax[0]), plane_eval(b[0], tmid, uvtmax[0]), TH)) &&
        ternary_equal2(ternary_compare(plane_eval(a[2], tmid, uvtmin[1]), plane_eval(b[2], tmid, uvtmin[1]), TH),
                       ternary_compare(plane_eval(a[2], tmid, uvtmax[1]), plane_eval(b[2], tmid, uvtmax[1]), TH)) &&
        ternary_equal2(ternary_compare(plane_eval(a[1], tmid, uvtmin[0]), plane_eval(b[1], tmid, uvtmin[0]), TH),
                       ternary_compare(plane_eval(a[1], tmid, uvtmax[0]), plane_eval(b[1], tmid, uvtmax[0]), TH)) &&
        ternary_equal2(ternary_compare(plane_eval(a[3], tmid, uvtmin[1]), plane_eval(b[3], tmid, uvtmin[1]), TH),
                       ternary_compare(plane_eval(a[3], tmid, uvtmax[1]), plane_eval(b[3], tmid, uvtmax[1]), TH));
    if (!bCoC)
        return false;
    const float ta = uvtmin[2], tb = uvtmax[2];
    return ternary_equal2(ternary_compare(plane_eval(a[0], ta, 0.0f), plane_eval(b[0], ta, 0.0f), TH),
                          ternary_compare(plane_eval(a[0], tb, 0.0f), plane_eval(b[0], tb, 0.0f), TH)) &&
           ternary_equal2(ternary_compare(plane_eval(a[1], ta, 0.0f), plane_eval(b[1], ta, 0.0f), TH),
                          ternary_compare(plane_eval(a[1], tb, 0.0f), plane_eval(b[1], tb, 0.0f), TH)) &&
           ternary_equal2(ternary_compare(plane_eval(a[2], ta, 0.0f), plane_eval(b[2], ta, 0.0f), TH),
                          ternary_compare(plane_eval(a[2], tb, 0.0f), plane_eval(b[2], tb, 0.0f), TH)) &&
           ternary_equal2(ternary_compare(plane_eval(a[3], ta, 0.0f), plane_eval(b[3], ta, 0.0f), TH),
                          ternary_compare(plane_eval(a[3], tb, 0.0f), plane_eval(b[3], tb, 0.0f), TH));
}

// Node::intersect (Reconstruction.hpp:204-216)
TLFR_HD bool node_intersect(const QNode& n, const Query& o, float R)
{
    float mnx = ((o.t * n.a.x + n.a.y * o.u) + n.a.z) - R;
    float mny = ((o.t * n.b.z + n.b.w * o.v) + n.c.x) - R;
    float mxx = ((o.t * n.a.w + n.b.x * o.u) + n.b.y) + R;
    float mxy = ((o.t * n.c.y + n.c.z * o.v) + n.c.w) + R;
    return (o.x >= mnx && o.y >= mny && o.x <= mxx && o.y <= mxy);
}

// collectInputSamples2 (RO.cpp:361-511).  Returns the number of samples within
// R, or a negative code when a capacity was exceeded (-1 leaves, -2 stack,
// -3 surfaces, -4 accepted samples).
TLFR_HD int collect(const QParams& P, Store& S, const Query& o, float R, int& nsurf, QStats& st)
{
    int nleaves = 0, sp = 0;
    S.stack[sp++] = P.root;
    while (sp > 0)
    {
        const int ni = S.stack[--sp];
        const QNode node = load_node(P.nodes, ni);
        if (node_intersect(node, o, R))
        {
            if (node.d.x < 0)
            {
                if (nleaves == S.leaf_cap)
                    return -1;   // leaf list full
                const int s0 = node.d.z;
                const float4 sp0 = P.s_rec[2 * (s0)];
                const float mvw = P.s_rec[2 * (s0) + 1].z;
                S.leaves[nleaves].node = ni;
                S.leaves[nleaves].key = sp0.z + (o.t - sp0.w) * mvw;
                nleaves++;
            }
            else
            {
                if (sp + 2 > S.stack_cap)
                    return -2;   // traversal stack full
                S.stack[sp++] = node.d.x;
                S.stack[sp++] = node.d.y;
            }
        }
    }
    st.leaves += nleaves;
    LeafSort ls{ S.leaves };
    fw_sort(ls, 0, nleaves);

    nsurf = 0;
    int nrs = 0, total = 0, surfaceStart = 0;
    const float RANGE = 1.0f / sqrtf(128.0f);
    const float uvtmin[3] = { o.u - RANGE, o.v - RANGE, o.t - 0.5f * RANGE };
    const float uvtmax[3] = { o.u + RANGE, o.v + RANGE, o.t + 0.5f * RANGE };
    const float R2 = R * R;
    for (int lidx = 0; lidx < nleaves; lidx++)
    {
        bool first = true;
        const QNode node = load_node(P.nodes, S.leaves[lidx].node);
        const int s0 = node.d.z, s1 = node.d.w;
        st.in_leaves += (unsigned)(s1 - s0);
        for (int i = s0; i < s1; i++)
        {
            float4 sp4, sm;     // (x, y, w, t), (mv, coc(w))
            load_sample(P.s_rec, i, sp4, sm);
            float x, y, w;
            if (sm.x != 0.0f || sm.y != 0.0f || sm.z != 0.0f)
            {
                const float dt = o.t - sp4.w;
                const float Px = sp4.x * sp4.z + sm.x * dt;
                const float Py = sp4.y * sp4.z + sm.y * dt;
                const float Pw = (1.0f * sp4.z) + sm.z * dt;
                w = Pw;
                const float cr = rcp(Pw);
                const float coc = P.c0 / w + P.c1;
                x = Px * cr + o.u * coc;
                y = Py * cr + o.v * coc;
            }
            else
            {
                w = sp4.z;
                x = sp4.x + o.u * sm.w;
                y = sp4.y + o.v * sm.w;
            }
            const float dx = x - o.x, dy = y - o.y;
            const float dist2 = dx * dx + dy * dy;
            if (dist2 <= R2)
            {
                if (first)
                {
                    first = false;
                    bool same = true;
                    for (int j = surfaceStart; j < lidx && same; ++j)
                        same = same_surface(node, load_node(P.nodes, S.leaves[j].node), uvtmin, uvtmax);
                    if (!same || nsurf == 0)
                    {
                        surfaceStart = lidx;
                        if (nsurf == S.surf_cap)
                            return -3;   // surface list full
                        Surf& sf = S.surf[nsurf++];
                        sf.start = nrs; sf.n = 0; sf.minDist = kF32Max; sf.minIndex = -1; sf.quad = 0;
                    }
                }
                if (nrs == S.rs_cap)
                    return -4;   // accepted-sample list full
                Surf& sf = S.surf[nsurf - 1];
                RSample r;
                r.x = x; r.y = y; r.index = i;
                r.rpos = (dx >= 0 ? 1 : 4) | (dy >= 0 ? 2 : 8);
                S.rs[nrs++] = r;
                sf.n++;
                sf.quad |= (1 << (r.rpos & 3));
                const float dist = sqrtf(dist2);
                if (dist < sf.minDist)
                {
                    sf.minDist = dist;
                    sf.minIndex = sf.n - 1;
                }
                total++;
            }
        }
    }
    st.fetched += total;
    return total;
}

TLFR_HD void reverse(RSample* a, int lo, int hi)    // [lo, hi)
{
    for (hi--; lo < hi; lo++, hi--) { RSample t = a[lo]; a[lo] = a[hi]; a[hi] = t; }
}

TLFR_HD float len2(float dx, float dy) { return sqrtf(dx * dx + dy * dy); }

struct EdgeFn { double A, B, C; bool acceptEqual; };

// EdgeFunction (reconstruction_lib/common/EdgeFunction.cpp:39-45, .hpp:45-47)
TLFR_HD EdgeFn edge_make(double x0, double y0, double x1, double y1)
{
    EdgeFn e;
    e.A = y0 - y1;
    e.B = x1 - x0;
    e.C = (-x0) * e.A - y0 * e.B;
    e.acceptEqual = (e.A == 0.) ? (e.B > 0.) : (e.A > 0.);
    return e;
}
TLFR_HD bool edge_test(const EdgeFn& e, double x, double y)
{
    float d = d2f_rn((x * e.A + y * e.B) + e.C);
    return d > 0.f ? true : (d == 0.f && e.acceptEqual);
}

TLFR_HD float gaussian(float x, float stddev, float mean)
{
    float e = 2.718281828f;
    return powf(e, -((x - mean) * (x - mean)) / (2.0f * (stddev * stddev)));
}

// A shadow query (TreeGather::reconstructShadows, R.cpp:302-344): the light-space
// depth of the query and the input samples' depth gradients (dw/dx, dw/dy per
// tree-ordered sample), against which each filtered sample's visibility is
// tested (RO.cpp:283-291, 337-347).
struct ShadowQ
{
    float w;                    // query's w
    float dispersion;           // dispersion * sqrt(light-space density) (RO.cpp:78-80)
    const float2* wg;           // per tree-ordered sample
};

constexpr float kShadowBias = 0.01f;     // SHADOW_BIAS (RO.cpp:46)

// The nearest sample of a reconstruction (Filterer::Result, RO.cpp:325-332):
// its position reprojected to the output (u,v,t), its w at the output t and
// its tree-ordered index (for its dw/dx, dw/dy and light-space density).
struct QNear
{
    float x, y, w;
    int index;
};

// w of sample i at time t (the ReconSample key of collectInputSamples2)
TLFR_HD float sample_w_at(const QParams& P, int i, float t)
{
    const float4 sp4 = P.s_rec[2 * i];
    const float4 sm = P.s_rec[2 * i + 1];
    if (sm.x != 0.0f || sm.y != 0.0f || sm.z != 0.0f)
        return (1.0f * sp4.z) + sm.z * (t - sp4.w);
    return sp4.z;
}

// Filterer::reconstruct (RO.cpp:50-359).  trace, when given, receives the
// flags and the final surfaces (layout documented in tlfr.h).  sh, when given,
// makes it the shadow reconstruction: the dispersion scaled by the light-space
// density, each filtered sample's colour kept where the query is lit by it and
// (0, 0, 0, alpha) where it is shadowed, no lens or time weights.
template <bool TRACE>
TLFR_HD int reconstruct_query(const QParams& P, Store& S, const Query& o, QStats& st, float4& out,
                                 int* trace, int trace_cap, const ShadowQ* sh = nullptr, QNear* nearp = nullptr)
{
    float dispersion = sh ? sh->dispersion : P.disp0;
    int nsurf = 0;
    int flags = 0;
    int n1 = collect(P, S, o, dispersion, nsurf, st);
    if (n1 < 0) { st.overflow_reason = -n1; return kQOverflow; }
    const bool fetch2R = nsurf == 0 || (S.surf[0].quad != 0xF && nsurf > 1);
    if (fetch2R)
    {
        flags |= 1;
        int n2 = collect(P, S, o, dispersion * 2, nsurf, st);
        if (n2 < 0) { st.overflow_reason = -n2; return kQOverflow; }
        if (n2 == 0)
        {
            flags |= 2;
            st.at_least_one++;
            int nN = n2;
            for (int k = 0; k < 3 && !nN; k++)
            {
                dispersion *= 2.f;
                nN = collect(P, S, o, dispersion * 2, nsurf, st);
                if (nN < 0) { st.overflow_reason = -nN; return kQOverflow; }
            }
        }
    }
    st.two_r += fetch2R ? 1 : 0;
    st.within1r += n1;

    // tiny-surface merging: dst.samples += src.samples (src appended after dst)
    int numSurfaces = nsurf;
    if (fetch2R)
        for (int sidx = 0; sidx < nsurf - 1; sidx++)
        {
            Surf& src = S.surf[sidx];
            if (src.n < 4)
            {
                Surf& dst = S.surf[sidx + 1];
                // src occupies [src.start, src.start+src.n), dst follows it; rotate to dst ++ src
                const int lo = src.start, mid = src.start + src.n, hi = dst.start + dst.n;
                if (src.n > 0 && mid == dst.start)
                {
                    reverse(S.rs, lo, mid);
                    reverse(S.rs, mid, hi);
                    reverse(S.rs, lo, hi);
                }
                dst.start = lo;
                dst.n = hi - lo;
                src.n = 0;
                if (src.minDist < dst.minDist)
                {
                    dst.minDist = src.minDist;
                    dst.minIndex = src.minIndex;
                }
                numSurfaces--;
            }
        }
    st.surfaces += numSurfaces;
    if (numSurfaces != nsurf)
    {
        st.merged++;
        flags |= 4;
    }

    bool found = false;
    float4 res = make_float4(0, 0, 0, 0);
    float nearestDist = kF32Max;
    int nearS = -1, nearI = 1;
    for (int sidx = 0; sidx < nsurf && !found; sidx++)
    {
        const Surf sf = S.surf[sidx];
        const int n = sf.n;
        if (n == 0)
            continue;
        const RSample* in = S.rs + sf.start;
        if (sf.minDist < nearestDist)
        {
            nearestDist = sf.minDist;
            nearS = sidx; nearI = sf.minIndex;
        }
        if (!fetch2R || sf.minDist < 0.f || sidx == nsurf - 1)
            found = true;
        if (n >= 200)
            found = true;
        for (int m = 0; m < n - 2 && !found; m++)
            for (int k = m + 1; k < n - 1 && !found; k++)
            {
                const RSample r0 = in[m], r1 = in[k];
                const int rp01 = r0.rpos | r1.rpos;
                for (int l = k + 1; l < n && !found; l++)
                {
                    const RSample r2 = in[l];
                    if ((rp01 | r2.rpos) != 15)
                        continue;
                    if (len2(r0.x - r1.x, r0.y - r1.y) > 2 * dispersion ||
                        len2(r0.x - r2.x, r0.y - r2.y) > 2 * dispersion ||
                        len2(r1.x - r2.x, r1.y - r2.y) > 2 * dispersion)
                        continue;
                    if (len2(r0.x - o.x, r0.y - o.y) > dispersion &&
                        len2(r1.x - o.x, r1.y - o.y) > dispersion &&
                        len2(r2.x - o.x, r2.y - o.y) > dispersion)
                        continue;
                    EdgeFn e0 = edge_make(r1.x, r1.y, r2.x, r2.y);
                    EdgeFn e1 = edge_make(r2.x, r2.y, r0.x, r0.y);
                    EdgeFn e2 = edge_make(r0.x, r0.y, r1.x, r1.y);
                    bool p0 = edge_test(e0, o.x, o.y);
                    bool p1 = edge_test(e1, o.x, o.y);
                    bool p2 = edge_test(e2, o.x, o.y);
                    found = (p0 && p1 && p2) || (!p0 && !p1 && !p2);
                }
            }
        if (found)
        {
            res = make_float4(0, 0, 0, 0);
            for (int k = 0; k < n; k++)
            {
                const RSample r = in[k];
                const float dx = o.x - r.x, dy = o.y - r.y;
                const float weight = 1 - len2(dx, dy) / dispersion;
                if (weight <= 0)
                    continue;
                float4 c = P.s_col[r.index];
                if (sh)
                {
                    const float2 g = sh->wg[r.index];
                    const float key = sample_w_at(P, r.index, o.t);
                    const bool lit = sh->w - kShadowBias <= key + (dx * g.x + dy * g.y);
                    if (!lit)
                        c = make_float4(0, 0, 0, c.w);
                }
                res.x += c.x * weight;
                res.y += c.y * weight;
                res.z += c.z * weight;
                res.w += c.w * weight;
            }
            const float oow = rcp(res.w);
            res.x *= oow; res.y *= oow; res.z *= oow; res.w *= oow;
            nearS = sidx; nearI = sf.minIndex;
        }
    }

    if (TRACE && trace)
    {
        int tn = 0;
        auto put = [&](int v) { if (tn < trace_cap) trace[tn] = v; tn++; };
        put(flags);
        put(nsurf);
        for (int s = 0; s < nsurf; s++)
        {
            put(S.surf[s].n);
            put(S.surf[s].minIndex);
            for (int k = 0; k < S.surf[s].n; k++)
                put(S.rs[S.surf[s].start + k].index);
        }
        if (tn > trace_cap && trace_cap > 1)
            trace[1] = -1;
    }

    if (nearS == -1)
    {
        st.empty++;
        out = make_float4(0, 0, 0, 0);
        return kQOk;
    }
    if (nearp)
    {
        const RSample na = S.rs[S.surf[nearS].start + nearI];
        nearp->x = na.x;
        nearp->y = na.y;
        nearp->w = sample_w_at(P, na.index, o.t);
        nearp->index = na.index;
    }
    if (res.w == 0)
    {
        const RSample na = S.rs[S.surf[nearS].start + nearI];
        res = P.s_col[na.index];
        if (sh)
        {
            const float2 g = sh->wg[na.index];
            const float dx = o.x - na.x, dy = o.y - na.y;
            const bool lit = sh->w - kShadowBias <= sample_w_at(P, na.index, o.t) + (dx * g.x + dy * g.y);
            if (!lit)
                res = make_float4(0, 0, 0, res.w);
        }
    }
    if (sh)
    {
        out = res;
        return kQOk;
    }
    if (P.lens_filter == 1)
    {
        float g = gaussian(o.u, 0.5f, 0) * gaussian(o.v, 0.5f, 0);
        res.x *= g; res.y *= g; res.z *= g; res.w *= g;
    }
    if (P.time_filter == 1)
    {
        float g = gaussian(o.t, 0.25f, 0.5f);
        res.x *= g; res.y *= g; res.z *= g; res.w *= g;
    }
    out = res;
    return kQOk;
}

// output sample i of pixel (x, y) (Reconstruction.cpp:653, 692-693)
TLFR_HD Query make_query(const QParams& P, int x, int y, int i)
{
    const int pattern = (int)(hash_bits((uint32_t)x, (uint32_t)y) % 64u);
    const float* s = P.pattern + ((size_t)pattern * P.M + i) * 5;
    Query q;
    q.x = s[0] + (float)x;
    q.y = s[1] + (float)y;
    q.u = s[2];
    q.v = s[3];
    q.t = s[4];
    return q;
}

__device__ __forceinline__ void add_stats(QStats& a, const QStats& b)
{
    a.leaves += b.leaves; a.in_leaves += b.in_leaves; a.within1r += b.within1r; a.fetched += b.fetched;
    a.surfaces += b.surfaces; a.two_r += b.two_r; a.merged += b.merged; a.at_least_one += b.at_least_one;
    a.empty += b.empty;
}

__device__ void flush_stats(const QStats& st, DevStats* ds)
{
    // block-level reduction then one atomic per counter
    __shared__ unsigned long long red[9];
    if (threadIdx.x < 9) red[threadIdx.x] = 0;
    __syncthreads();
    unsigned v[9] = { st.leaves, st.in_leaves, st.within1r, st.fetched, st.surfaces, st.two_r, st.merged,
                      st.at_least_one, st.empty };
    for (int k = 0; k < 9; k++)
    {
        unsigned long long x = v[k];
        for (int o = 16; o > 0; o >>= 1)
            x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0)
            atomicAdd(&red[k], x);
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        atomicAdd(&ds->leaf_nodes, red[0]);
        atomicAdd(&ds->samples_in_leaves, red[1]);
        atomicAdd(&ds->within_1r, red[2]);
        atomicAdd(&ds->fetched, red[3]);
        atomicAdd(&ds->surfaces, red[4]);
        atomicAdd(&ds->num_2r, red[5]);
        atomicAdd(&ds->merged, red[6]);
        atomicAdd(&ds->at_least_one, red[7]);
        atomicAdd(&ds->empty, red[8]);
    }
}

constexpr int kBlock = 128;
// capacities of the full per-query path (statistics pass and heavy pass)
constexpr int kStackCap = 96, kLeafCap = 256, kRsCap = 512, kSurfCap = 64;
// capacities of the light pass: traversal stack and leaf list per output
// sample, both in shared memory.  kLLeaf is also the most leaves the warp's
// scan holds (one per lane).  The single-frame path runs a first light pass
// with fewer leaves (kL1Leaf), which fits seven blocks per SM, and retries the
// output samples that outgrow it with the full kLLeaf and a deeper stack.
constexpr int kLStack = 16, kLLeaf = 32;
constexpr int kL1Stack = 12, kL1Leaf = 24;
constexpr int kL2Stack = 30, kL2Leaf = 32;

// Per-thread column of a shared-memory array laid out [slot][thread]: a warp
// whose lanes touch different slots still hits distinct banks.  The host build
// (stride 1) runs the same code on a plain array.
template <class T>
struct Column
{
    T* base;
    int stride;
    TLFR_HD T& operator[](int k) const { return base[k * stride]; }
};

TLFR_HD float int_as_float_bits(int v)
{
#ifdef __CUDA_ARCH__
    return __int_as_float(v);
#else
    float f;
    memcpy(&f, &v, 4);
    return f;
#endif
}
TLFR_HD int float_as_int_bits(float v)
{
#ifdef __CUDA_ARCH__
    return __float_as_int(v);
#else
    int i;
    memcpy(&i, &v, 4);
    return i;
#endif
}

// A leaf found by the light pass's traversal: (sort key = w at the output
// sample's time (RO.cpp:390-392), node index as bits).
struct LLeafSort
{
    Column<float2> l;
    TLFR_HD int cmp(int a, int b) const { const float ka = l[a].x, kb = l[b].x; return (ka < kb) ? -1 : (ka > kb) ? 1 : 0; }
    TLFR_HD void swap(int a, int b) { const float2 t = l[a]; l[a] = l[b]; l[b] = t; }
};
TLFR_HD int leaf_node(const Column<float2>& leaves, int k) { return float_as_int_bits(leaves[k].y); }

// Appends leaf node ni (first sample s0) with its key; false when full.
TLFR_HD bool leaf_append(const QParams& P, const Query& o, const Column<float2>& leaves, int cap, int& nleaves, int ni,
                         int s0)
{
    if (nleaves == cap)
        return false;
    const float4 sp0 = P.s_rec[2 * (s0)];
    const float mvw = P.s_rec[2 * (s0) + 1].z;
    leaves[nleaves++] = make_float2(sp0.z + (o.t - sp0.w) * mvw, int_as_float_bits(ni));
    return true;
}

// collectInputSamples2's traversal and leaf sort (RO.cpp:368-407) for one output
// sample at radius R: DFS in the reference's order (push child0, child1, pop the
// last) into the leaf column, then FW::sort of the leaves by key.  Children are
// stored as pairs, so a node that intersects has both children loaded and
// tested together and only those that intersect are pushed (a leaf child waits
// on the stack only behind an internal child1).  The loop has no early exit (an
// overflow sets a flag), so a warp reconverges at the end of every step.
// Returns the leaf count, or -1 when the stack or the leaf column is full.
TLFR_HD int collect_pairs(const QParams& P, const Column<int>& stack, int stack_cap, const Column<float2>& leaves,
                          int leaf_cap, const Query& o, float R)
{
    int nleaves = 0, sp = 0;
    bool ok = true;
    {
        const QNode rn = load_node(P.nodes, P.root);
        if (node_intersect(rn, o, R))
        {
            if (rn.d.x < 0)
                ok = leaf_append(P, o, leaves, leaf_cap, nleaves, P.root, rn.d.z);
            else
                stack[sp++] = rn.d.x;
        }
    }
    // stack entries: >= 0 the first child of an intersecting internal node;
    // < 0 (~node) an intersecting leaf
    while (sp > 0 && ok)
    {
        const int e = stack[--sp];
        if (e < 0)
            ok = leaf_append(P, o, leaves, leaf_cap, nleaves, ~e, P.nodes[~e].d.z);
        else
        {
            const QNode n0 = load_node(P.nodes, e);
            const QNode n1 = load_node(P.nodes, e + 1);
            const bool h0 = node_intersect(n0, o, R);
            const bool h1 = node_intersect(n1, o, R);
            if (h1 && n1.d.x >= 0)
            {
                // child1's subtree comes first; child0 waits below it
                if (sp + 2 > stack_cap)
                    ok = false;
                else
                {
                    if (h0)
                        stack[sp++] = n0.d.x >= 0 ? n0.d.x : ~e;
                    stack[sp++] = n1.d.x;
                }
            }
            else
            {
                if (h1)
                    ok = leaf_append(P, o, leaves, leaf_cap, nleaves, e + 1, n1.d.z);
                if (h0 && ok)
                {
                    if (n0.d.x < 0)
                        ok = leaf_append(P, o, leaves, leaf_cap, nleaves, e, n0.d.z);
                    else if (sp + 1 > stack_cap)
                        ok = false;
                    else
                        stack[sp++] = n0.d.x;
                }
            }
        }
    }
    if (!ok)
        return -1;
    LLeafSort ls{ leaves };
    fw_sort(ls, 0, nleaves);
    return nleaves;
}

// Light pass, part 1: each lane collects its own output sample's leaves at 1R.
template <int LEAF, int STACK>
TLFR_HD int light_collect(const QParams& P, const Column<int>& stack, const Column<float2>& leaves, const Query& o)
{
    static_assert(LEAF <= 32, "the warp's scan holds one leaf per lane");
    return collect_pairs(P, stack, STACK, leaves, LEAF, o, P.disp0);
}

// sameSurface's sixteen plane values of one node for one output sample: each
// bounding plane (xmin, ymin, xmax, ymax) at the lens extremes of the output
// sample's (u, v) +- RANGE window at the window's middle time, and at the
// window's two time extremes at the lens centre (Reconstruction.hpp:457-525).
// Pairs are (low, high) ends in the order the reference tests them.
struct SurfVals { float v[8][2]; };

TLFR_HD void surf_vals(const QNode& n, const float* uvtmin, const float* uvtmax, SurfVals& s)
{
    float a[4][3];
    node_planes(n, a);
    const float tmid = 0.5f * (uvtmin[2] + uvtmax[2]);
    const float ta = uvtmin[2], tb = uvtmax[2];
    s.v[0][0] = plane_eval(a[0], tmid, uvtmin[0]); s.v[0][1] = plane_eval(a[0], tmid, uvtmax[0]);
    s.v[1][0] = plane_eval(a[2], tmid, uvtmin[1]); s.v[1][1] = plane_eval(a[2], tmid, uvtmax[1]);
    s.v[2][0] = plane_eval(a[1], tmid, uvtmin[0]); s.v[2][1] = plane_eval(a[1], tmid, uvtmax[0]);
    s.v[3][0] = plane_eval(a[3], tmid, uvtmin[1]); s.v[3][1] = plane_eval(a[3], tmid, uvtmax[1]);
    s.v[4][0] = plane_eval(a[0], ta, 0.0f);        s.v[4][1] = plane_eval(a[0], tb, 0.0f);
    s.v[5][0] = plane_eval(a[1], ta, 0.0f);        s.v[5][1] = plane_eval(a[1], tb, 0.0f);
    s.v[6][0] = plane_eval(a[2], ta, 0.0f);        s.v[6][1] = plane_eval(a[2], tb, 0.0f);
    s.v[7][0] = plane_eval(a[3], ta, 0.0f);        s.v[7][1] = plane_eval(a[3], tb, 0.0f);
}

// same_surface() from precomputed values: the two nodes differ where, for some
// plane, one is more than the threshold below the other at one end and more
// than the threshold above it at the other (ternaryEqual of two opposite
// ternaryCompare results, Reconstruction.hpp:428-449, 457-525).  The test is
// symmetric in its arguments.
TLFR_HD bool same_surface_vals(const SurfVals& a, const SurfVals& b)
{
    const float TH = 1 * 0.1f;
    bool same = true;
#pragma unroll
    for (int k = 0; k < 8; k++)
        same = same && ternary_equal2(ternary_compare(a.v[k][0], b.v[k][0], TH), ternary_compare(a.v[k][1], b.v[k][1], TH));
    return same;
}

// Light pass, part 2 (RO.cpp:94-99, 165-304 for the common case): the 1R scan
// of one output sample's sorted leaves by the whole warp, lanes over
// consecutive samples of a leaf (coalesced 32-byte records).  It settles the
// output sample when the 1R fetch ends with exactly one surface, or when the
// first surface holds samples in all four quadrants by the time a second one
// opens (fetch2R is false in both cases and the first surface is resolved).
// Accepted samples update the surface state in sample order: quadrant mask,
// first strict minimum distance, and the tent filter, summed in acceptance
// order (the reference's filter order, RO.cpp:274-294).  At the first accepted
// sample of a later leaf, sameSurface (Reconstruction.hpp:457-525) is tested
// against every leaf since the surface opened (RO.cpp:465-470), lanes over
// those leaves; when one fails the scan stops there.  All lanes call it with
// the same arguments and get the same result: 0 with the colour in out, 1
// when the output sample needs the 2R fetch.
// first_surface (the learned router's fast path for pixels it marks as holding
// a single apparent surface; no reference counterpart): when a second surface
// opens, the first one is taken even if its samples do not cover all four
// quadrants, where the reference would refetch at 2R.  Output samples with
// nothing within 1R still take the full path.
__device__ int light_scan_warp(const QParams& P, const Column<float2>& leaves, int nleaves, const Query& o,
                               float4& out, bool first_surface = false)
{
    const int lane = threadIdx.x & 31;
    const float R = P.disp0;
    const float R2 = R * R;
    const float RANGE = 1.0f / sqrtf(128.0f);
    const float uvtmin[3] = { o.u - RANGE, o.v - RANGE, o.t - 0.5f * RANGE };
    const float uvtmax[3] = { o.u + RANGE, o.v + RANGE, o.t + 0.5f * RANGE };
    // sample range of leaf k, held by lane k (the leaf column holds at most 32),
    // and F_k, its offset in the output sample's flat sequence of samples (the
    // leaves' samples one after another in leaf order).  Lane k also holds leaf
    // k's sameSurface values for this output sample.
    int my_s0 = 0, my_n = 0;
    SurfVals my_sv;
    if (lane < nleaves)
    {
        const QNode nd = load_node(P.nodes, leaf_node(leaves, lane));
        my_s0 = nd.d.z;
        my_n = nd.d.w - nd.d.z;
        surf_vals(nd, uvtmin, uvtmax, my_sv);
    }
    int my_f = my_n;
    for (int off = 1; off < 32; off <<= 1)
    {
        const int v = __shfl_up_sync(0xffffffffu, my_f, off);
        if (lane >= off)
            my_f += v;
    }
    const int total = __shfl_sync(0xffffffffu, my_f, 31);
    my_f -= my_n;
    // Leaf and sample of flat index base + lane: the last leaf k with F_k <= f.
    // Every leaf holds at least one sample (one leaf node per surface run of the
    // build), so leaf starts are distinct: the leaves starting inside
    // (base, base + lane] are counted from a mask of the chunk's leaf starts.
    // All lanes call it; lanes with f >= total get an unused answer.
    auto locate = [&](int base, int& k, int& i) {
        const bool starts_in = lane < nleaves && my_f > base && my_f < base + 32;
        const unsigned starts = __reduce_or_sync(0xffffffffu, starts_in ? 1u << (my_f - base) : 0u);
        const int kfirst = __popc(__ballot_sync(0xffffffffu, lane < nleaves && my_f <= base)) - 1;
        k = kfirst + __popc(starts & ((2u << lane) - 1u));
        i = __shfl_sync(0xffffffffu, my_s0, k & 31) + (base + lane - __shfl_sync(0xffffffffu, my_f, k & 31));
    };
    // chunks of 32 consecutive flat samples, which may span several leaves; the
    // next chunk's records are loaded while the current one is processed
    int ck, ci;
    locate(0, ck, ci);
    bool cvalid = lane < total;
    float4 cpos = make_float4(0, 0, 0, 0), cmot = cpos, ccol = cpos;
    if (cvalid)
    {
        load_sample(P.s_rec, ci, cpos, cmot);
        ccol = P.s_col[ci];
    }
    int nsurf = 0, lidx0 = 0, quad = 0, nearest = -1, result = -1, first_leaf = -1;
    float minDist = kF32Max;
    float4 acc = make_float4(0, 0, 0, 0);
    for (int base = 0; base < total && result < 0; base += 32)
    {
        int nk, ni;
        locate(base + 32, nk, ni);
        const bool nvalid = base + 32 + lane < total;
        float4 npos = make_float4(0, 0, 0, 0), nmot = npos, ncol = npos;
        if (nvalid)
        {
            load_sample(P.s_rec, ni, npos, nmot);
            ncol = P.s_col[ni];
        }
        // the current chunk
        float dx = 0, dy = 0, dist2 = 0;
        bool ok = false;
        if (cvalid)
        {
            float x, y;
            if (cmot.x != 0.0f || cmot.y != 0.0f || cmot.z != 0.0f)
            {
                const float dt = o.t - cpos.w;
                const float Px = cpos.x * cpos.z + cmot.x * dt;
                const float Py = cpos.y * cpos.z + cmot.y * dt;
                const float Pw = (1.0f * cpos.z) + cmot.z * dt;
                const float cr = rcp(Pw);
                const float coc = P.c0 / Pw + P.c1;
                x = Px * cr + o.u * coc;
                y = Py * cr + o.v * coc;
            }
            else
            {
                x = cpos.x + o.u * cmot.w;
                y = cpos.y + o.v * cmot.w;
            }
            dx = x - o.x;
            dy = y - o.y;
            dist2 = dx * dx + dy * dy;
            ok = dist2 <= R2;
        }
        unsigned accm = __ballot_sync(0xffffffffu, ok);
        if (accm)
        {
            const float dist = ok ? sqrtf(dist2) : __int_as_float(0x7f800000);
            const float weight = 1 - dist / R;
            const bool inc = ok && weight > 0;
            const float4 pr = inc ? make_float4(ccol.x * weight, ccol.y * weight, ccol.z * weight, ccol.w * weight)
                                  : make_float4(0, 0, 0, 0);
            const int qbit = ok ? 1 << (((dx >= 0 ? 1 : 4) | (dy >= 0 ? 2 : 8)) & 3) : 0;
            const unsigned incm = __ballot_sync(0xffffffffu, inc);
            // the chunk's leaves in order, those with accepted samples
            while (accm)
            {
                const int kseg = __shfl_sync(0xffffffffu, ck, __ffs(accm) - 1);
                const bool inseg = ck == kseg;
                const unsigned segm = __ballot_sync(0xffffffffu, inseg);
                accm &= ~segm;
                if (first_leaf != kseg)
                {
                    // first accepted sample of this leaf
                    first_leaf = kseg;
                    if (nsurf == 0)
                    {
                        nsurf = 1;
                        lidx0 = kseg;
                    }
                    else
                    {
                        // lanes j in [lidx0, kseg) test leaf j against this leaf
                        // (leaf indices are lanes: the column holds at most 32)
                        SurfVals cur;
#pragma unroll
                        for (int a = 0; a < 8; a++)
                        {
                            cur.v[a][0] = __shfl_sync(0xffffffffu, my_sv.v[a][0], kseg);
                            cur.v[a][1] = __shfl_sync(0xffffffffu, my_sv.v[a][1], kseg);
                        }
                        const bool sj = (lane >= lidx0 && lane < kseg) ? same_surface_vals(cur, my_sv) : true;
                        if (!__all_sync(0xffffffffu, sj))   // a second surface opens: the first one is final
                        {
                            result = (quad == 0xF || first_surface) ? 0 : 1;
                            break;
                        }
                    }
                }
                const bool sok = ok && inseg;
                quad |= __reduce_or_sync(0xffffffffu, sok ? qbit : 0);
                // first strict minimum in sample order (RO.cpp:494-499); distances
                // are non-negative, so their bit patterns order as unsigned integers
                const unsigned dbits = sok ? __float_as_uint(dist) : 0x7f800000u;
                const unsigned mbits = __reduce_min_sync(0xffffffffu, dbits);
                const float cmin = __uint_as_float(mbits);
                if (cmin < minDist)
                {
                    const unsigned at = __ballot_sync(0xffffffffu, sok && dbits == mbits);
                    minDist = cmin;
                    nearest = __shfl_sync(0xffffffffu, ci, __ffs(at) - 1);
                }
                // tent filter products summed in sample order
                for (unsigned mi = incm & segm; mi; mi &= mi - 1)
                {
                    const int src = __ffs(mi) - 1;
                    acc.x += __shfl_sync(0xffffffffu, pr.x, src);
                    acc.y += __shfl_sync(0xffffffffu, pr.y, src);
                    acc.z += __shfl_sync(0xffffffffu, pr.z, src);
                    acc.w += __shfl_sync(0xffffffffu, pr.w, src);
                }
            }
        }
        ck = nk; ci = ni; cvalid = nvalid;
        cpos = npos; cmot = nmot; ccol = ncol;
    }
    if (result < 0)
        result = (nsurf == 0) ? 1 : 0;
    if (result != 0)
        return result;
    const float oow = rcp(acc.w);
    acc.x *= oow; acc.y *= oow; acc.z *= oow; acc.w *= oow;
    if (acc.w == 0)
        acc = P.s_col[nearest];
    if (P.lens_filter == 1)
    {
        float g = gaussian(o.u, 0.5f, 0) * gaussian(o.v, 0.5f, 0);
        acc.x *= g; acc.y *= g; acc.z *= g; acc.w *= g;
    }
    if (P.time_filter == 1)
    {
        float g = gaussian(o.t, 0.25f, 0.5f);
        acc.x *= g; acc.y *= g; acc.z *= g; acc.w *= g;
    }
    out = acc;
    return 0;
}

__device__ __forceinline__ Query query_of(const QParams& P, long long q)
{
    const long long pix = q / P.M;
    const int i = (int)(q - pix * P.M);
    return make_query(P, (int)(pix % P.W), (int)(pix / P.W), i);
}

// Append value to a queue when pred holds, one atomic per warp.  All 32 lanes
// of the warp must call it.
__device__ __forceinline__ void warp_append(int* queue, int* count, bool pred, int value)
{
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m)
        return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader)
        base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred)
        queue[base + __popc(m & ((1u << lane) - 1))] = value;
}

// Pass 1: every output sample through the light path; the rest are queued.
// Query id q = pixel * M + i.  The queue holds up to num_queries entries; an
// entry with kQueueRestart set outgrew the light pass's capacities, so it is
// not known to need the 2R fetch and the full path starts it over.
constexpr int kQueueRestart = 1 << 30;

constexpr int kProbe = 4;
// resident light-pass blocks per SM: shared memory (40 KB per block) allows 5,
// and a 5-block register budget (<= 102 per thread) measured 9% faster than 4.
// The first tier (24 leaves, 12 stack entries: 30 KB) fits 7 at <= 72
// registers (a few spilled): 1340 ms per 1920x1080x8 frame against 1378 at
// 6 blocks with 28 leaves and 1492 with one tier; the retry tier (47 KB) 4.
constexpr int kLightBlocksPerSM = 5;
constexpr int kL1BlocksPerSM = 7;
constexpr int kL2BlocksPerSM = 4;
// Light-pass kinds: every output sample of a map, overflow to the full path
// (kLightPlain); the same with overflow to a retry list (kLightFirst); the
// output samples of a retry list (kLightRetry), overflow to the full path.
enum { kLightPlain = 0, kLightFirst = 1, kLightRetry = 2 };

// PROBE: the router's coarse pass.  Query k of pixel p is output sample
// (k % kProbe) * M / kProbe (four per pixel); nothing is written but the count of
// the pixel's probed output samples that the plain 1R pass sends to the full path.
// Lane -> output sample maps of the light pass.  The 32 lanes of a warp scan
// each other's leaves one output sample after another, so a warp's output
// samples should reach nearly the same hierarchy nodes.  The output samples of
// a pixel are spread over the whole lens and shutter (the reference sorts each
// pattern's samples by a (u,v,t) Morton key, Reconstruction.cpp:484-510, so
// sample i of every pattern sits near the same place on that curve):
//   kMapTiles: a warp takes a tile of tw x th pixels (px = tw*th lanes per
//     sample) and sw = 32/px consecutive output samples of each; a block
//     iteration covers the tile and 4*sw consecutive samples (its four warps).
//     The default tile is 4x2 pixels x 4 samples: the union of the hierarchy
//     nodes a warp reaches is then 3.8x one output sample's at 1920x1080x8
//     (5.3x for a pixel's 32 consecutive samples); batches choose the shape
//     per frame by timing (autotuner).
//   kMapLinear: q = block iteration * 128 + thread (the pinhole image's one
//     sample per pixel, and M not a multiple of 4*sw).
// Output sample ids q = pixel * M + i are unchanged (qcol, queues).
enum { kMapLinear = 0, kMapTiles = 1 };

struct LightMap
{
    int mode;
    long long units;        // block iterations
    int tw, th, sw;         // kMapTiles: tile width and height (pixels), output samples per lane column
    int tiles_x;            // kMapTiles: tiles per row
    int groups;             // kMapTiles: groups of 4*sw output samples per pixel (M / (4*sw))
};

// tile shapes the autotuner tries: (tw, th), sw = 32 / (tw*th)
constexpr int kTileShapes[5][2] = { { 4, 2 }, { 8, 4 }, { 4, 4 }, { 2, 2 }, { 2, 1 } };
constexpr int kDefaultShape = 0;

// Output sample of thread t in block iteration u; false past the frame's end.
__device__ __forceinline__ bool light_query_id(const QParams& P, const LightMap& L, long long u, int t,
                                               long long num_queries, long long& q)
{
    if (L.mode == kMapLinear)
    {
        q = u * kBlock + t;
        return q < num_queries;
    }
    const long long tile = u / L.groups;
    const int g = (int)(u - tile * L.groups);
    const int px = L.tw * L.th;
    const int l = t & 31, p = l % px;
    const int x = (int)(tile % L.tiles_x) * L.tw + p % L.tw;
    const int y = (int)(tile / L.tiles_x) * L.th + p / L.tw;
    const int i = (g * 4 + (t >> 5)) * L.sw + l / px;
    q = ((long long)y * P.W + x) * P.M + i;
    return x < P.W && y < P.H;
}

// Shared-memory columns of a light-pass block.
template <int LEAF, int STACK>
struct LightShared
{
    float2 leaves[LEAF][kBlock];
    int stack[STACK][kBlock];
};

// One block iteration u of the light pass.  kLightRetry: the output samples
// are retry[u * kBlock + thread] for indices below num_queries; kLightFirst:
// those that outgrow the capacities are appended to retry.
template <bool PROBE, int LEAF, int STACK, int MODE>
__device__ __forceinline__ void light_unit(const QParams& P, const LightMap& L, long long u, long long num_queries,
                                           float4* __restrict__ qcol, int* __restrict__ heavy,
                                           int* __restrict__ heavy_count, LightShared<LEAF, STACK>& sh,
                                           int* __restrict__ retry = nullptr, int* __restrict__ retry_count = nullptr)
{
    float2 (&sh_leaves)[LEAF][kBlock] = sh.leaves;
    const int lane = threadIdx.x & 31;
    const int wbase = threadIdx.x & ~31;
    const Column<int> stack{ &sh.stack[0][threadIdx.x], kBlock };
    {
        // each lane: traversal and leaf sort of its own output sample
        long long q = 0;
        bool valid;
        if (MODE == kLightRetry)
        {
            const long long k = u * kBlock + threadIdx.x;
            valid = k < num_queries;
            q = valid ? retry[k] : 0;
        }
        else
            valid = light_query_id(P, L, u, threadIdx.x, num_queries, q);
        Query o{};
        int nl = -2;
        const long long pix = valid ? (PROBE ? q / kProbe : q / P.M) : 0;
        const bool fast = !PROBE && valid && P.route_fast && P.route_fast[pix];
        if (valid)
        {
            o = PROBE ? make_query(P, (int)(pix % P.W), (int)(pix / P.W), (int)((q % kProbe) * P.M / kProbe))
                      : query_of(P, q);
            nl = light_collect<LEAF, STACK>(P, stack, Column<float2>{ &sh_leaves[0][threadIdx.x], kBlock }, o);
        }
        const unsigned fast_lanes = __ballot_sync(0xffffffffu, fast);
        __syncwarp();
        // the warp: the 1R scan of each lane's output sample in turn
        int code = 2;
        float4 col = make_float4(0, 0, 0, 0);
        for (int j = 0; j < 32; j++)
        {
            const int nlj = __shfl_sync(0xffffffffu, nl, j);
            if (nlj < 0)
                continue;
            Query oj;
            oj.x = __shfl_sync(0xffffffffu, o.x, j);
            oj.y = __shfl_sync(0xffffffffu, o.y, j);
            oj.u = __shfl_sync(0xffffffffu, o.u, j);
            oj.v = __shfl_sync(0xffffffffu, o.v, j);
            oj.t = __shfl_sync(0xffffffffu, o.t, j);
            float4 c;
            const Column<float2> lj{ &sh_leaves[0][wbase + j], kBlock };
            const int r = light_scan_warp(P, lj, nlj, oj, c, (fast_lanes >> j) & 1u);
            if (lane == j)
            {
                code = r;
                col = c;
            }
        }
        __syncwarp();
        if (PROBE)
        {
            // heavy_count is the per-pixel count here
            if (valid && code != 0)
                atomicAdd(&heavy_count[pix], 1);
            return;
        }
        bool hv = false, rt = false;
        int entry = 0;
        if (valid)
        {
            if (code == 0)
                qcol[q] = col;
            else if (MODE == kLightFirst && code == 2)
                rt = true;
            else
            {
                hv = true;
                entry = (int)q | (code == 2 ? kQueueRestart : 0);
            }
        }
        warp_append(heavy, heavy_count, hv, entry);
        if (MODE == kLightFirst)
            warp_append(retry, retry_count, rt, (int)q);
    }
}

// The light pass over a map (kLightPlain, kLightFirst) or over a retry list
// of *retry_count output samples (kLightRetry).
template <bool PROBE, int LEAF, int STACK, int BLOCKS_PER_SM, int MODE>
__global__ void __launch_bounds__(kBlock, BLOCKS_PER_SM)
k_query_light(QParams P, LightMap L, long long num_queries, float4* __restrict__ qcol, int* __restrict__ heavy,
              int* __restrict__ heavy_count, int* __restrict__ retry, int* __restrict__ retry_count)
{
    __shared__ LightShared<LEAF, STACK> sh;
    if (MODE == kLightRetry)
    {
        const long long n = *retry_count;
        for (long long u = blockIdx.x; u * kBlock < n; u += gridDim.x)
            light_unit<PROBE, LEAF, STACK, MODE>(P, L, u, n, qcol, heavy, heavy_count, sh, retry);
    }
    else
        for (long long u = blockIdx.x; u < L.units; u += gridDim.x)
            light_unit<PROBE, LEAF, STACK, MODE>(P, L, u, num_queries, qcol, heavy, heavy_count, sh, retry,
                                                 retry_count);
}

// the light-pass instances
#define K_LIGHT_PLAIN(PROBE) k_query_light<PROBE, kLLeaf, kLStack, kLightBlocksPerSM, kLightPlain>
#define K_LIGHT_FIRST k_query_light<false, kL1Leaf, kL1Stack, kL1BlocksPerSM, kLightFirst>
#define K_LIGHT_RETRY k_query_light<false, kL2Leaf, kL2Stack, kL2BlocksPerSM, kLightRetry>

// ---------------------------------------------------------------------------
// Pass 2, warp-cooperative: output samples known to need the 2R fetch (the
// light pass found fetch2R true, RO.cpp:99), and those that outgrew the light
// pass's capacities, which start over from the 1R fetch and its fetch2R
// decision.  A warp takes 32 queued samples:
//   1. each lane traverses the hierarchy at 2R for its own sample and sorts its
//      leaves (32 independent traversals hide each other's latency);
//   2. then, one sample at a time, the 32 lanes scan that sample's leaves
//      together: 32 samples tested per step, accepted ones appended in order with
//      a ballot, surface separation tested against up to 32 earlier leaves per
//      step (RO.cpp:427-503); a sample whose 2R fetch found nothing is set aside
//      and traversed again, wider, in a later round (RO.cpp:110-120);
//      tiny-surface merging; per surface front to back the triangle search
//      spread over the lanes (any covering triangle settles it, the search
//      order does not change the answer); the tent filter's products in
//      parallel, summed in sample order from shuffles (RO.cpp:137-304).
// Working lists live in a per-warp region of a global arena.  A sample that
// outgrows them goes to the large-capacity pass, which starts it over.
// ---------------------------------------------------------------------------
constexpr int kCWarps = 4;
// blocks of the cooperative full-path pass (its working lists are per warp):
// 5 per SM leave it its 95 registers without spills; at 1920x1080x8 it measured
// 404 ms against 512 ms at 6 (80 registers, spills; earlier 563 against 651
// and 699 at 8 blocks)
#ifndef TLFR_COOP_BLOCKS_PER_SM
#define TLFR_COOP_BLOCKS_PER_SM 5
#endif
constexpr int kCoopBlocksPerSM = TLFR_COOP_BLOCKS_PER_SM;
constexpr int kCLeaf = 256;         // leaves per lane's traversal
constexpr int kCRs = 4096;          // accepted samples per sample
constexpr int kCSurf = 512;         // surfaces per sample
constexpr int kCStack = 96;

struct CoopScratch
{
    Leaf    leaves[32][kCLeaf];
    RSample rs[kCRs];
    Surf    surf[kCSurf];
};

__device__ __forceinline__ unsigned lanes_below(int lane) { return (1u << lane) - 1u; }

// Reprojection of sample i to the query's (u,v,t) and its squared distance
// (RO.cpp:436-454); the same operations as collect().
__device__ __forceinline__ float reproject(const QParams& P, int i, const Query& o, float& x, float& y)
{
    float4 sp4, sm;
    load_sample(P.s_rec, i, sp4, sm);
    if (sm.x != 0.0f || sm.y != 0.0f || sm.z != 0.0f)
    {
        const float dt = o.t - sp4.w;
        const float Px = sp4.x * sp4.z + sm.x * dt;
        const float Py = sp4.y * sp4.z + sm.y * dt;
        const float Pw = (1.0f * sp4.z) + sm.z * dt;
        const float cr = rcp(Pw);
        const float coc = P.c0 / Pw + P.c1;
        x = Px * cr + o.u * coc;
        y = Py * cr + o.v * coc;
    }
    else
    {
        x = sp4.x + o.u * sm.w;
        y = sp4.y + o.v * sm.w;
    }
    const float dx = x - o.x, dy = y - o.y;
    return dx * dx + dy * dy;
}

// DFS traversal into leaves[] with leaf keys (RO.cpp:368-395) and FW::sort of
// the leaves (RO.cpp:407).  Returns the leaf count or -1 on overflow.
__device__ int traverse_sorted(const QParams& P, const Query& o, float R, Leaf* leaves, int cap)
{
    int stack[kCStack];
    int nleaves = 0, sp = 0;
    stack[sp++] = P.root;
    while (sp > 0)
    {
        const int ni = stack[--sp];
        const QNode node = load_node(P.nodes, ni);
        if (node_intersect(node, o, R))
        {
            if (node.d.x < 0)
            {
                if (nleaves == cap)
                    return -1;
                const int s0 = node.d.z;
                const float4 sp0 = P.s_rec[2 * (s0)];
                const float mvw = P.s_rec[2 * (s0) + 1].z;
                leaves[nleaves].node = ni;
                leaves[nleaves].key = sp0.z + (o.t - sp0.w) * mvw;
                nleaves++;
            }
            else
            {
                if (sp + 2 > kCStack)
                    return -1;
                stack[sp++] = node.d.x;
                stack[sp++] = node.d.y;
            }
        }
    }
    LeafSort ls{ leaves };
    fw_sort(ls, 0, nleaves);
    return nleaves;
}

// Cooperative collectInputSamples2 scan (RO.cpp:412-503) over sorted leaves.
// The leaves are taken 32 at a time: lane k holds leaf g+k's sample range, and
// the group's samples are scanned as one flat sequence in chunks of 32 that
// span leaf boundaries (as in the light pass).  A chunk's accepted samples are
// handled leaf by leaf in order: sameSurface at the leaf's first accepted
// sample against every leaf since the open surface began (lanes over those
// leaves), then the samples appended to rs in sample order with the surface's
// quadrant mask and first strict minimum.  All lanes call it with the same
// arguments; returns the accepted count (same on all lanes) or -1 when rs /
// surf outgrow the scratch.
constexpr int kTriMax = 200;                    // n >= 200 is accepted without the search (RO.cpp:215)
constexpr int kTriWords = (kTriMax + 31) / 32;

// Per-warp shared memory of the full path: the coverage search's bit rows, and
// the sameSurface values of the current group of 32 leaves ([value][leaf]).
struct CoopShared
{
    unsigned row[kTriWords];                    // samples l > m within 2*dispersion of m
    unsigned mask[5 * kTriWords];               // quadrant patterns 3, 6, 9, 12; within dispersion
    float sv[16][32];
};

__device__ int coop_scan(const QParams& P, const Query& o, float R, const Leaf* leaves, int nleaves,
                         CoopScratch& S, CoopShared& T, int& nsurf_out)
{
    const int lane = threadIdx.x & 31;
    const float RANGE = 1.0f / sqrtf(128.0f);
    const float uvtmin[3] = { o.u - RANGE, o.v - RANGE, o.t - 0.5f * RANGE };
    const float uvtmax[3] = { o.u + RANGE, o.v + RANGE, o.t + 0.5f * RANGE };
    const float R2 = R * R;
    int nsurf = 0, nrs = 0, surfaceStart = 0, last_leaf = -1;
    // the open surface's running state, identical on all lanes
    float minDist = kF32Max;
    int minIndex = -1, quad = 0, sstart = 0;
    for (int g = 0; g < nleaves; g += 32)
    {
        const int ng = mini(32, nleaves - g);
        int my_s0 = 0, my_n = 0;
        __syncwarp();   // the previous group's values have been read
        if (lane < ng)
        {
            const QNode nd = load_node(P.nodes, leaves[g + lane].node);
            my_s0 = nd.d.z;
            my_n = nd.d.w - nd.d.z;
            SurfVals v;
            surf_vals(nd, uvtmin, uvtmax, v);
#pragma unroll
            for (int a = 0; a < 8; a++)
            {
                T.sv[2 * a][lane] = v.v[a][0];
                T.sv[2 * a + 1][lane] = v.v[a][1];
            }
        }
        __syncwarp();
        int my_f = my_n;
        for (int off = 1; off < 32; off <<= 1)
        {
            const int v = __shfl_up_sync(0xffffffffu, my_f, off);
            if (lane >= off)
                my_f += v;
        }
        const int total = __shfl_sync(0xffffffffu, my_f, 31);
        my_f -= my_n;
        for (int base = 0; base < total; base += 32)
        {
            // leaf (within the group) and sample of flat index base + lane; every
            // leaf holds at least one sample, so leaf starts are distinct
            const bool starts_in = lane < ng && my_f > base && my_f < base + 32;
            const unsigned starts = __reduce_or_sync(0xffffffffu, starts_in ? 1u << (my_f - base) : 0u);
            const int k = __popc(__ballot_sync(0xffffffffu, lane < ng && my_f <= base)) - 1 +
                          __popc(starts & ((2u << lane) - 1u));
            const int i = __shfl_sync(0xffffffffu, my_s0, k & 31) + (base + lane - __shfl_sync(0xffffffffu, my_f, k & 31));
            float x = 0, y = 0, d2 = 0;
            bool acc = false;
            if (base + lane < total)
            {
                d2 = reproject(P, i, o, x, y);
                acc = d2 <= R2;
            }
            unsigned accm = __ballot_sync(0xffffffffu, acc);
            if (!accm)
                continue;
            const float dx = x - o.x, dy = y - o.y;
            const int rpos = (dx >= 0 ? 1 : 4) | (dy >= 0 ? 2 : 8);
            const float dist = acc ? sqrtf(d2) : kF32Max;
            while (accm)
            {
                const int kseg = __shfl_sync(0xffffffffu, k, __ffs(accm) - 1);
                const unsigned m = accm & __ballot_sync(0xffffffffu, k == kseg);
                accm &= ~m;
                const int lidx = g + kseg;
                if (lidx != last_leaf)
                {
                    // first accepted sample of this leaf
                    last_leaf = lidx;
                    bool same = true;
                    if (nsurf > 0)
                    {
                        // leaves of earlier groups since the surface opened (rare)
                        if (surfaceStart < g)
                        {
                            const QNode node = load_node(P.nodes, leaves[lidx].node);
                            for (int jb = surfaceStart; jb < g && same; jb += 32)
                            {
                                const int j = jb + lane;
                                const bool ok = (j < g) ? same_surface(node, load_node(P.nodes, leaves[j].node), uvtmin, uvtmax) : true;
                                same = __all_sync(0xffffffffu, ok);
                            }
                        }
                        // this group's leaves: lane j - g tests leaf j from the precomputed values
                        if (same)
                        {
                            const int j = g + lane;
                            bool ok = true;
                            if (j >= surfaceStart && j < lidx)
                            {
                                SurfVals cur, mine;
#pragma unroll
                                for (int a = 0; a < 8; a++)
                                {
                                    cur.v[a][0] = T.sv[2 * a][kseg];
                                    cur.v[a][1] = T.sv[2 * a + 1][kseg];
                                    mine.v[a][0] = T.sv[2 * a][lane];
                                    mine.v[a][1] = T.sv[2 * a + 1][lane];
                                }
                                ok = same_surface_vals(cur, mine);
                            }
                            same = __all_sync(0xffffffffu, ok);
                        }
                    }
                    if (!same || nsurf == 0)
                    {
                        if (nsurf > 0 && lane == 0)
                        {
                            Surf& p = S.surf[nsurf - 1];
                            p.n = nrs - sstart; p.minDist = minDist; p.minIndex = minIndex; p.quad = quad;
                        }
                        if (nsurf == kCSurf)
                            return -1;
                        surfaceStart = lidx;
                        nsurf++;
                        sstart = nrs;
                        minDist = kF32Max; minIndex = -1; quad = 0;
                        if (lane == 0) S.surf[nsurf - 1].start = nrs;
                    }
                }
                const int cnt = __popc(m);
                if (nrs + cnt > kCRs)
                    return -1;
                const bool mine = (m >> lane) & 1u;
                if (mine)
                {
                    RSample r;
                    r.x = x; r.y = y; r.index = i; r.rpos = rpos;
                    S.rs[nrs + __popc(m & lanes_below(lane))] = r;
                }
                quad |= __reduce_or_sync(0xffffffffu, mine ? (1 << (rpos & 3)) : 0);
                // first strict minimum in acceptance order (RO.cpp:494-499);
                // distances are non-negative, so their bits order as integers
                const unsigned dbits = mine ? __float_as_uint(dist) : 0x7f800000u;
                const unsigned mbits = __reduce_min_sync(0xffffffffu, dbits);
                if (__uint_as_float(mbits) < minDist)
                {
                    const int fl = __ffs(__ballot_sync(0xffffffffu, mine && dbits == mbits)) - 1;
                    minDist = __uint_as_float(mbits);
                    minIndex = nrs + __popc(m & lanes_below(fl)) - sstart;
                }
                nrs += cnt;
            }
        }
    }
    if (nsurf > 0 && lane == 0)
    {
        Surf& p = S.surf[nsurf - 1];
        p.n = nrs - sstart; p.minDist = minDist; p.minIndex = minIndex; p.quad = quad;
    }
    __syncwarp();
    nsurf_out = nsurf;
    return nrs;
}

__device__ __forceinline__ void coop_reverse(RSample* a, int lo, int hi)     // [lo, hi)
{
    const int lane = threadIdx.x & 31;
    const int n = hi - lo;
    for (int k = lane; k < n / 2; k += 32)
    {
        RSample t = a[lo + k];
        a[lo + k] = a[hi - 1 - k];
        a[hi - 1 - k] = t;
    }
    __syncwarp();
}

// Coverage test of one surface (RO.cpp:221-259): is there a triangle of three
// of its samples m < k < l that together hold all four quadrant bits, whose
// sides are at most 2*dispersion long, with a vertex within dispersion of the
// output sample, and that contains the output sample (double-precision edge
// functions)?  Any such triangle settles it, so the search order does not
// change the answer.  For each first vertex m the warp builds one bit row: the
// samples l > m within 2*dispersion of m; lanes then take the second vertices
// k of that row, and the third vertices of (m, k) are the set bits of the row
// beyond k that complete the quadrants (bit masks per quadrant pattern) and the
// within-dispersion condition (a bit mask), each checked against k's side
// length before the edge functions.


__device__ bool coop_triangle(const RSample* in, int n, const Query& o, float dispersion, CoopShared& T)
{
    const int lane = threadIdx.x & 31;
    const int W = (n + 31) >> 5;
    const float side = 2 * dispersion;
    for (int w = 0; w < W; w++)
    {
        const int i = (w << 5) + lane;
        const bool v = i < n;
        RSample r{};
        if (v)
            r = in[i];
        const bool near = v && !(len2(r.x - o.x, r.y - o.y) > dispersion);
        const unsigned q3 = __ballot_sync(0xffffffffu, v && r.rpos == 3);
        const unsigned q6 = __ballot_sync(0xffffffffu, v && r.rpos == 6);
        const unsigned q9 = __ballot_sync(0xffffffffu, v && r.rpos == 9);
        const unsigned q12 = __ballot_sync(0xffffffffu, v && r.rpos == 12);
        const unsigned nr = __ballot_sync(0xffffffffu, near);
        if (lane == 0)
        {
            T.mask[0 * kTriWords + w] = q3; T.mask[1 * kTriWords + w] = q6;
            T.mask[2 * kTriWords + w] = q9; T.mask[3 * kTriWords + w] = q12;
            T.mask[4 * kTriWords + w] = nr;
        }
    }
    for (int m = 0; m < n - 2; m++)
    {
        const RSample r0 = in[m];
        for (int w = (m + 1) >> 5; w < W; w++)
        {
            const int k = (w << 5) + lane;
            bool b = false;
            if (k > m && k < n)
            {
                const RSample rk = in[k];
                b = !(len2(r0.x - rk.x, r0.y - rk.y) > side);
            }
            const unsigned bits = __ballot_sync(0xffffffffu, b);
            if (lane == 0)
                T.row[w] = bits;
        }
        __syncwarp();
        const bool near0 = (T.mask[4 * kTriWords + (m >> 5)] >> (m & 31)) & 1u;
        for (int kb = m + 1; kb < n - 1; kb += 32)
        {
            const int k = kb + lane;
            bool found = false;
            if (k < n - 1 && ((T.row[k >> 5] >> (k & 31)) & 1u))
            {
                const RSample r1 = in[k];
                const int missing = 15 & ~(r0.rpos | r1.rpos);
                const bool nearpair = near0 || ((T.mask[4 * kTriWords + (k >> 5)] >> (k & 31)) & 1u);
                for (int w = k >> 5; w < W && !found; w++)
                {
                    unsigned c = T.row[w];
                    if (w == (k >> 5))
                        c &= ~((2u << (k & 31)) - 1u);          // third vertices l > k
                    if (missing)
                    {
                        unsigned q = 0;
                        if ((3 & missing) == missing) q |= T.mask[0 * kTriWords + w];
                        if ((6 & missing) == missing) q |= T.mask[1 * kTriWords + w];
                        if ((9 & missing) == missing) q |= T.mask[2 * kTriWords + w];
                        if ((12 & missing) == missing) q |= T.mask[3 * kTriWords + w];
                        c &= q;
                    }
                    if (!nearpair)
                        c &= T.mask[4 * kTriWords + w];
                    while (c && !found)
                    {
                        const int l = (w << 5) + __ffs(c) - 1;
                        c &= c - 1;
                        const RSample r2 = in[l];
                        if (len2(r1.x - r2.x, r1.y - r2.y) > side)
                            continue;
                        EdgeFn e0 = edge_make(r1.x, r1.y, r2.x, r2.y);
                        EdgeFn e1 = edge_make(r2.x, r2.y, r0.x, r0.y);
                        EdgeFn e2 = edge_make(r0.x, r0.y, r1.x, r1.y);
                        bool p0 = edge_test(e0, o.x, o.y);
                        bool p1 = edge_test(e1, o.x, o.y);
                        bool p2 = edge_test(e2, o.x, o.y);
                        found = (p0 && p1 && p2) || (!p0 && !p1 && !p2);
                    }
                }
            }
            if (__any_sync(0xffffffffu, found))
                return true;
        }
        __syncwarp();       // the next row overwrites T.row
    }
    return false;
}

// One warp: the queued output samples queue[b .. b+32) (of n) through the full
// path, with the warp's working lists S and shared triangle-search bits T.
__device__ __forceinline__ void coop_group(const QParams& P, const int* __restrict__ queue, int n, int b,
                                           float4* __restrict__ qcol, int* __restrict__ ovf_queue,
                                           int* __restrict__ ovf_count, int ovf_cap, CoopScratch& S, CoopShared& T)
{
    const int lane = threadIdx.x & 31;
    {
        // 1. per-lane traversal and leaf sort: at 2R for output samples the light
        // pass found to need it, at 1R for those that outgrew the light pass's
        // capacities (they start over from the 1R fetch)
        const int entry = (b + lane < n) ? queue[b + lane] : -1;
        bool restart = entry >= 0 && (entry & kQueueRestart);
        const bool valid = entry >= 0;
        const int myq = valid ? (entry & ~kQueueRestart) : 0;
        Query myo = query_of(P, myq);
        int mycount = 0;
        float mydisp = P.disp0;     // this lane's dispersion (doubled by each widening)
        int mywiden = 0;
        // 2. each sample of the batch by the whole warp, in rounds.  A sample is
        // set aside for the next round (its lane traverses again, all such lanes
        // in parallel) when a restarted sample's 1R fetch ends with fetch2R true
        // (RO.cpp:94-99; the next round fetches at 2R), and when a 2R fetch found
        // nothing (the widening, RO.cpp:110-120: at most three times, each
        // doubling the dispersion).  Every traversal and every fetch goes through
        // one call site (the kernel's instruction footprint is what limits it).
        unsigned todo = __ballot_sync(0xffffffffu, valid);
        for (int round = 0; round < 5 && todo; round++)
        {
        if ((todo >> lane) & 1u)
            mycount = traverse_sorted(P, myo, restart ? mydisp : mydisp * 2, S.leaves[lane], kCLeaf);
        __syncwarp();
        unsigned redo = 0;
        for (unsigned jm = todo; jm; jm &= jm - 1)
        {
            const int j = __ffs(jm) - 1;
            const int qj = __shfl_sync(0xffffffffu, myq, j);
            const int nl = __shfl_sync(0xffffffffu, mycount, j);
            bool ovf = nl < 0;
            Query o;
            o.x = __shfl_sync(0xffffffffu, myo.x, j);
            o.y = __shfl_sync(0xffffffffu, myo.y, j);
            o.u = __shfl_sync(0xffffffffu, myo.u, j);
            o.v = __shfl_sync(0xffffffffu, myo.v, j);
            o.t = __shfl_sync(0xffffffffu, myo.t, j);
            const float dispersion = __shfl_sync(0xffffffffu, mydisp, j);
            const bool rs = __shfl_sync(0xffffffffu, restart, j);
            const int widened = __shfl_sync(0xffffffffu, mywiden, j);
            int nsurf = 0, total = 0;
            bool fetch2R = true;
            if (!ovf)
            {
                total = coop_scan(P, o, rs ? dispersion : dispersion * 2, S.leaves[j], nl, S, T, nsurf);
                ovf = total < 0;
            }
            bool set_aside = false;
            if (!ovf && rs)
            {
                fetch2R = nsurf == 0 || (S.surf[0].quad != 0xF && nsurf > 1);
                set_aside = fetch2R;
            }
            else if (!ovf && total == 0 && widened < 3)
                set_aside = true;
            if (set_aside)
            {
                redo |= 1u << j;
                if (lane == j)
                {
                    if (restart)
                        restart = false;
                    else
                    {
                        mydisp *= 2.f;
                        mywiden++;
                    }
                }
                continue;
            }
            if (ovf)
            {
                if (lane == 0)
                {
                    int slot = atomicAdd(ovf_count, 1);
                    if (slot < ovf_cap)
                        ovf_queue[slot] = qj;
                }
                __syncwarp();
                continue;
            }
            // tiny-surface merging (RO.cpp:137-156): dst.samples += src.samples
            for (int sidx = 0; fetch2R && sidx < nsurf - 1; sidx++)
            {
                Surf src = S.surf[sidx], dst = S.surf[sidx + 1];
                __syncwarp();
                if (src.n < 4)
                {
                    const int lo = src.start, mid = src.start + src.n, hi = dst.start + dst.n;
                    if (src.n > 0 && mid == dst.start)
                    {
                        coop_reverse(S.rs, lo, mid);
                        coop_reverse(S.rs, mid, hi);
                        coop_reverse(S.rs, lo, hi);
                    }
                    if (lane == 0)
                    {
                        Surf& d = S.surf[sidx + 1];
                        d.start = lo;
                        d.n = hi - lo;
                        if (src.minDist < dst.minDist)
                        {
                            d.minDist = src.minDist;
                            d.minIndex = src.minIndex;
                        }
                        S.surf[sidx].n = 0;
                    }
                    __syncwarp();
                }
            }
            // resolve (RO.cpp:165-304)
            bool found = false;
            float4 res = make_float4(0, 0, 0, 0);
            float nearestDist = kF32Max;
            int nearS = -1, nearI = 1;
            for (int sidx = 0; sidx < nsurf && !found; sidx++)
            {
                const Surf sf = S.surf[sidx];
                const int cnt = sf.n;
                if (cnt == 0)
                    continue;
                const RSample* in = S.rs + sf.start;
                if (sf.minDist < nearestDist)
                {
                    nearestDist = sf.minDist;
                    nearS = sidx; nearI = sf.minIndex;
                }
                if (!fetch2R || sf.minDist < 0.f || sidx == nsurf - 1)
                    found = true;
                if (cnt >= kTriMax)
                    found = true;
                if (!found && cnt >= 3)
                    found = coop_triangle(in, cnt, o, dispersion, T);
                if (found)
                {
                    // tent filter (RO.cpp:274-294): products in parallel, summed
                    // in sample order by every lane from shuffles
                    res = make_float4(0, 0, 0, 0);
                    for (int kb = 0; kb < cnt; kb += 32)
                    {
                        const int k = kb + lane;
                        float4 pr = make_float4(0, 0, 0, 0);
                        bool inc = false;
                        if (k < cnt)
                        {
                            const RSample r = in[k];
                            const float dx = o.x - r.x, dy = o.y - r.y;
                            const float weight = 1 - len2(dx, dy) / dispersion;
                            if (weight > 0)
                            {
                                const float4 c = P.s_col[r.index];
                                pr = make_float4(c.x * weight, c.y * weight, c.z * weight, c.w * weight);
                                inc = true;
                            }
                        }
                        for (unsigned mi = __ballot_sync(0xffffffffu, inc); mi; mi &= mi - 1)
                        {
                            const int src = __ffs(mi) - 1;
                            res.x += __shfl_sync(0xffffffffu, pr.x, src);
                            res.y += __shfl_sync(0xffffffffu, pr.y, src);
                            res.z += __shfl_sync(0xffffffffu, pr.z, src);
                            res.w += __shfl_sync(0xffffffffu, pr.w, src);
                        }
                    }
                    const float oow = rcp(res.w);
                    res.x *= oow; res.y *= oow; res.z *= oow; res.w *= oow;
                    nearS = sidx; nearI = sf.minIndex;
                }
            }
            if (lane == 0)
            {
                float4 out = make_float4(0, 0, 0, 0);
                if (nearS != -1)
                {
                    if (res.w == 0)
                        res = P.s_col[S.rs[S.surf[nearS].start + nearI].index];
                    if (P.lens_filter == 1)
                    {
                        float g = gaussian(o.u, 0.5f, 0) * gaussian(o.v, 0.5f, 0);
                        res.x *= g; res.y *= g; res.z *= g; res.w *= g;
                    }
                    if (P.time_filter == 1)
                    {
                        float g = gaussian(o.t, 0.25f, 0.5f);
                        res.x *= g; res.y *= g; res.z *= g; res.w *= g;
                    }
                    out = res;
                }
                qcol[qj] = out;
            }
            __syncwarp();
        }
        todo = redo;
        }
    }
}

__global__ void __launch_bounds__(kCWarps * 32, TLFR_COOP_BLOCKS_PER_SM)
k_query_coop(QParams P, const int* __restrict__ queue, const int* __restrict__ queue_count,
             float4* __restrict__ qcol, int* __restrict__ ovf_queue, int* __restrict__ ovf_count, int ovf_cap,
             CoopScratch* __restrict__ scratch)
{
    __shared__ CoopShared sh_tri[kCWarps];
    const int warp = blockIdx.x * kCWarps + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * kCWarps;
    const int n = *queue_count;
    for (int b = warp * 32; b < n; b += nwarps * 32)
        coop_group(P, queue, n, b, qcol, ovf_queue, ovf_count, ovf_cap, scratch[warp], sh_tri[threadIdx.x >> 5]);
}

// Statistics pass: every output sample through the full path with the
// reference's counters (TreeGather::Stats).
__global__ void __launch_bounds__(kBlock)
k_query_stats(QParams P, long long num_queries, float4* __restrict__ qcol, int* __restrict__ ovf_queue,
              int* __restrict__ ovf_count, int ovf_cap, DevStats* ds)
{
    int stack[kStackCap];
    Leaf leaves[kLeafCap];
    RSample rs[kRsCap];
    Surf surf[kSurfCap];
    Store S{ stack, kStackCap, leaves, kLeafCap, rs, kRsCap, surf, kSurfCap };
    QStats st{};
    for (long long base = (long long)blockIdx.x * kBlock; base < num_queries; base += (long long)gridDim.x * kBlock)
    {
        const long long q = base + threadIdx.x;
        if (q < num_queries)
        {
            QStats qs{};
            float4 c;
            if (reconstruct_query<false>(P, S, query_of(P, q), qs, c, nullptr, 0) == kQOk)
            {
                qcol[q] = c;
                add_stats(st, qs);
            }
            else
            {
                atomicAdd(&ds->overflow_by_reason[qs.overflow_reason & 3], 1ull);
                int slot = atomicAdd(ovf_count, 1);
                if (slot < ovf_cap)
                    ovf_queue[slot] = (int)q;
            }
        }
    }
    flush_stats(st, ds);
}

// Pass 3: large capacities for queries that overflowed pass 2 (or the
// statistics pass).  Each thread slot owns a fixed region of the arena.
__global__ void __launch_bounds__(64)
k_query_overflow(QParams P, const int* __restrict__ queue, const int* __restrict__ count_ptr, int cap,
                 float4* __restrict__ qcol, char* arena, size_t slot_bytes, int num_slots, int stack_cap, int leaf_cap,
                 int rs_cap, int surf_cap, int* hard_fail, DevStats* ds, int stats)
{
    const int count = min(*count_ptr, cap);
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    QStats st{};
    if (slot < num_slots)
    {
        char* base = arena + (size_t)slot * slot_bytes;
        Store S;
        S.stack = (int*)base;                      S.stack_cap = stack_cap;
        S.leaves = (Leaf*)(S.stack + stack_cap);   S.leaf_cap = leaf_cap;
        S.rs = (RSample*)(S.leaves + leaf_cap);    S.rs_cap = rs_cap;
        S.surf = (Surf*)(S.rs + rs_cap);           S.surf_cap = surf_cap;
        for (int k = slot; k < count; k += num_slots)
        {
            const int q = queue[k];
            float4 c;
            QStats qs{};
            if (reconstruct_query<false>(P, S, query_of(P, q), qs, c, nullptr, 0) != kQOk)
            {
                atomicAdd(hard_fail, 1);
                qcol[q] = make_float4(0, 0, 0, 0);
                continue;
            }
            add_stats(st, qs);
            qcol[q] = c;
        }
    }
    if (stats)
        flush_stats(st, ds);
}

// ---------------------------------------------------------------------------
// The reference's GPU-toggle algorithm (CameraParams::enableCuda): its CUDA
// kernels recKernel / failKernel / nearestKernel (ReconstructionCudaKernels.cu:
// 242-868) and their CPU restatement CudaReconstruction::reconstructCPUSingle /
// reconstructCPUFailed / reconstructCPUNearest (ReconstructionCuda.cpp:261-872),
// whose semantics are followed here operation for operation, with IEEE
// arithmetic (the reference compiles its kernels with -use_fast_math) and no
// capacity limits: output samples that outgrow the per-thread lists run again
// with large lists from a global arena instead of going back to the CPU.
//   first surface at 1R: leaves with a sample within R, in order of depth at
//     the output time; stop at the first leaf that fails sameSurface against an
//     earlier one; coverage by the "wedge box" of the accepted samples' dx/dy
//     slopes above and below the output sample; tent-filtered colour
//   2R surfaces: surfaces of at least 4 samples split at sameSurface failures,
//     each tested by the wedge boxes and a triangle fan test over every sample
//     collected so far (the reference never clears that list)
//   nearest: the nearest sample within R, 2R, ..., 16R (last one on ties)
// The hierarchy's node pairs are the reference's (child0 < child1 there, so its
// traversal, which pushes the larger index first, visits child0 first).
// ---------------------------------------------------------------------------
struct TStore
{
    int*    stack;  int stack_cap;
    int*    leaves; int leaf_cap;
    float2* xy;     int xy_cap;
};

// collectNodes (ReconstructionCuda.cpp:545-590): DFS, child0's subtree first;
// leaves ordered by depth at the output time with the reference's selection
// sort (first minimum).  Returns the leaf count or -1 when a list is full.
TLFR_HD int toggle_collect(const QParams& P, TStore& S, const Query& o, float radius)
{
    int n = 0, sp = 0;
    S.stack[sp++] = P.root;
    while (sp > 0)
    {
        const int idx = S.stack[--sp];
        const QNode node = load_node(P.nodes, idx);
        if (!node_intersect(node, o, radius))
            continue;
        if (node.d.x < 0)
        {
            if (n == S.leaf_cap)
                return -1;
            S.leaves[n++] = idx;
        }
        else
        {
            if (sp + 2 > S.stack_cap)
                return -1;
            S.stack[sp++] = node.d.x + 1;      // child1 (the reference's idx1 after its swap: pushed first)
            S.stack[sp++] = node.d.x;          // child0
        }
    }
    for (int i = 0; i < n - 1; i++)
    {
        const int s0 = P.nodes[S.leaves[i]].d.z;
        const float4 p0 = P.s_rec[2 * s0];
        float w = p0.z + (o.t - p0.w) * P.s_rec[2 * s0 + 1].z;
        int mn = i;
        for (int j = i + 1; j < n; j++)
        {
            const int s1 = P.nodes[S.leaves[j]].d.z;
            const float4 p1 = P.s_rec[2 * s1];
            const float w1 = p1.z + (o.t - p1.w) * P.s_rec[2 * s1 + 1].z;
            if (w1 < w)
            {
                w = w1;
                mn = j;
            }
        }
        if (mn != i)
        {
            const int t = S.leaves[i];
            S.leaves[i] = S.leaves[mn];
            S.leaves[mn] = t;
        }
    }
    return n;
}

// Reprojection of sample j to the output sample (ReconstructionCuda.cpp:594-604):
// division forms, no zero-motion shortcut.
TLFR_HD float toggle_reproject(const QParams& P, int j, const Query& o, float& dx, float& dy)
{
    const float4 p = P.s_rec[2 * j];
    const float4 m = P.s_rec[2 * j + 1];
    const float p0x = p.x * p.z;
    const float p0y = p.y * p.z;
    const float p0w = p.z;
    const float px = p0x + (o.t - p.w) * m.x;
    const float py = p0y + (o.t - p.w) * m.y;
    const float pw = p0w + (o.t - p.w) * m.z;
    const float cocr = P.c0 / pw + P.c1;
    const float x = px / pw + cocr * o.u;
    const float y = py / pw + cocr * o.v;
    dx = x - o.x;
    dy = y - o.y;
    return dx * dx + dy * dy;
}

// sameSurface of the GPU toggle (ReconstructionCuda.cpp:127-190): the same
// sixteen plane comparisons as the Filterer's.
TLFR_HD bool toggle_same(const QParams& P, int a, int b, const Query& o)
{
    const float RANGE = 1.0f / sqrtf(128.0f);
    const float uvtmin[3] = { o.u - RANGE, o.v - RANGE, o.t - 0.5f * RANGE };
    const float uvtmax[3] = { o.u + RANGE, o.v + RANGE, o.t + 0.5f * RANGE };
    return same_surface(load_node(P.nodes, a), load_node(P.nodes, b), uvtmin, uvtmax);
}

TLFR_HD void wbox_add(float* box, float dx, float dy)
{
    const float k = dx / dy;
    if (dy >= 0.f)
    {
        box[0] = minr(box[0], k);
        box[1] = maxr(box[1], k);
    }
    else
    {
        box[2] = minr(box[2], k);
        box[3] = maxr(box[3], k);
    }
}

// checkTriangles (ReconstructionCuda.cpp:193-219) over offsets from the output sample.
TLFR_HD bool toggle_triangles(const float2* xy, int n, float dispersion)
{
    for (int m = 0; m < n - 2; m++)
        for (int k = m + 1; k < n - 1; k++)
            for (int l = k + 1; l < n; l++)
            {
                const float2 p0 = xy[m], p1 = xy[k], p2 = xy[l];
                if (len2(p0.x - p1.x, p0.y - p1.y) > 2 * dispersion || len2(p1.x - p2.x, p1.y - p2.y) > 2 * dispersion ||
                    len2(p2.x - p0.x, p2.y - p0.y) > 2 * dispersion)
                    continue;
                const float c0 = p0.x * p1.y - p1.x * p0.y;
                const float c1 = p1.x * p2.y - p2.x * p1.y;
                const float c2 = p2.x * p0.y - p0.x * p2.y;
                if (c0 <= 0.f && c1 <= 0.f && c2 <= 0.f)
                    return true;
                if (c0 >= 0.f && c1 >= 0.f && c2 >= 0.f)
                    return true;
            }
    return false;
}

// reconstructCPUNearest (ReconstructionCuda.cpp:700-744).  false when a list is full.
TLFR_HD bool toggle_nearest(const QParams& P, TStore& S, const Query& o, float4& out)
{
    for (float rmul = 1.f; rmul <= 16.f; rmul *= 2.f)
    {
        const float radius = rmul * P.disp0;
        const int n = toggle_collect(P, S, o, radius);
        if (n < 0)
            return false;
        int minIdx = -1;
        float minDist = kF32Max;
        for (int i = 0; i < n; i++)
        {
            const int4 d = P.nodes[S.leaves[i]].d;
            for (int j = d.z; j < d.w; j++)
            {
                float dx, dy;
                const float dist2 = toggle_reproject(P, j, o, dx, dy);
                if (dist2 <= minDist)
                {
                    minDist = dist2;
                    minIdx = j;
                }
            }
        }
        if (minIdx >= 0)
        {
            out = P.s_col[minIdx];
            return true;
        }
    }
    out = make_float4(0, 0, 0, 0);
    return true;
}

// reconstructCPUFailed (ReconstructionCuda.cpp:748-872).  false when a list is full.
TLFR_HD bool toggle_failed(const QParams& P, TStore& S, const Query& o, float4& out)
{
    const float dispersion = P.disp0;
    const float radius = 2.f * dispersion;
    const int nleaves = toggle_collect(P, S, o, radius);
    if (nleaves < 0)
        return false;
    if (nleaves == 0)
        return toggle_nearest(P, S, o, out);
    int nxy = 0, numPoints = 0, sfirst = 0, lidx = 0;
    float4 color = make_float4(0, 0, 0, 0);
    const int MIN_SAMPLES_PER_SURFACE = 4;
    do
    {
        sfirst = lidx;
        numPoints = 0;
        color = make_float4(0, 0, 0, 0);
        float abox[4] = { kF32Max, -kF32Max, kF32Max, -kF32Max };
        float wbox[4] = { kF32Max, -kF32Max, kF32Max, -kF32Max };
        do
        {
            const int leaf = S.leaves[lidx];
            bool endSurface = false;
            if (numPoints >= MIN_SAMPLES_PER_SURFACE)
                for (int j = sfirst; j < lidx; ++j)
                    if (!toggle_same(P, leaf, S.leaves[j], o))
                    {
                        endSurface = true;
                        break;
                    }
            if (endSurface)
                break;
            const int4 d = P.nodes[leaf].d;
            for (int i = d.z; i < d.w; i++)
            {
                float dx, dy;
                const float dist2 = toggle_reproject(P, i, o, dx, dy);
                if (dist2 <= radius * radius)
                {
                    if (nxy == S.xy_cap)
                        return false;
                    S.xy[nxy++] = make_float2(dx, dy);
                    numPoints++;
                    const float w = 1.f - sqrtf(dist2) / dispersion;
                    if (w <= 0.f)
                        wbox_add(abox, dx, dy);
                    else
                    {
                        wbox_add(wbox, dx, dy);
                        const float4 c = P.s_col[i];
                        color.x += w * c.x; color.y += w * c.y; color.z += w * c.z; color.w += w * c.w;
                    }
                }
            }
            lidx++;
        } while (lidx < nleaves);
        if (lidx < nleaves)
        {
            abox[0] = minr(abox[0], wbox[0]);
            abox[1] = maxr(abox[1], wbox[1]);
            abox[2] = minr(abox[2], wbox[2]);
            abox[3] = maxr(abox[3], wbox[3]);
            if (abox[1] > abox[2] && abox[0] < abox[3])
                if ((wbox[1] > wbox[2] && wbox[0] < wbox[3]) || toggle_triangles(S.xy, nxy, dispersion))
                    break;
        }
    } while (lidx < nleaves);
    if (color.w > 0.f)
    {
        const float r = 1.f / color.w;
        out = make_float4(color.x * r, color.y * r, color.z * r, color.w * r);
        return true;
    }
    return toggle_nearest(P, S, o, out);
}

// reconstructCPUSingle (ReconstructionCuda.cpp:592-698).  false when a list is full.
TLFR_HD bool toggle_single(const QParams& P, TStore& S, const Query& o, float4& out)
{
    const float radius = P.disp0;
    int n = toggle_collect(P, S, o, radius);
    if (n < 0)
        return false;
    // leaves without a sample within R are dropped
    int lcount = 0;
    for (int i = 0; i < n; i++)
    {
        const int4 d = P.nodes[S.leaves[i]].d;
        bool empty = true;
        for (int j = d.z; j < d.w && empty; j++)
        {
            float dx, dy;
            if (toggle_reproject(P, j, o, dx, dy) <= radius * radius)
                empty = false;
        }
        if (!empty)
            S.leaves[lcount++] = S.leaves[i];
    }
    n = lcount;
    if (n == 0)
        return toggle_failed(P, S, o, out);
    float wbox[4] = { kF32Max, -kF32Max, kF32Max, -kF32Max };
    bool multi = false;
    float4 color = make_float4(0, 0, 0, 0);
    for (int i = 0; i < n; i++)
    {
        for (int j = 0; j < i; j++)
            if (!toggle_same(P, S.leaves[i], S.leaves[j], o))
            {
                multi = true;
                break;
            }
        if (multi)
            break;
        const int4 d = P.nodes[S.leaves[i]].d;
        for (int j = d.z; j < d.w; j++)
        {
            float dx, dy;
            const float dist2 = toggle_reproject(P, j, o, dx, dy);
            if (dist2 <= radius * radius)
            {
                wbox_add(wbox, dx, dy);
                const float w = maxr(0.f, 1.f - sqrtf(dist2) / radius);
                const float4 c = P.s_col[j];
                color.x += w * c.x; color.y += w * c.y; color.z += w * c.z; color.w += w * c.w;
            }
        }
    }
    if (color.w > 0.f && wbox[1] > wbox[2] && wbox[0] < wbox[3])
    {
        const float r = 1.f / color.w;
        out = make_float4(color.x * r, color.y * r, color.z * r, color.w * r);
        return true;
    }
    if (multi)
        return toggle_failed(P, S, o, out);
    return toggle_nearest(P, S, o, out);
}

constexpr int kTgStack = 128, kTgLeaf = 256, kTgXy = 512;

// Every output sample of the frame, one thread each, lists in local memory;
// output samples that outgrow them are queued for k_toggle_large.
__global__ void __launch_bounds__(kBlock)
k_toggle(QParams P, long long num_queries, float4* __restrict__ qcol, int* __restrict__ ovf_queue,
         int* __restrict__ ovf_count, int ovf_cap)
{
    int stack[kTgStack];
    int leaves[kTgLeaf];
    float2 xy[kTgXy];
    TStore S{ stack, kTgStack, leaves, kTgLeaf, xy, kTgXy };
    for (long long q = blockIdx.x * (long long)kBlock + threadIdx.x; q < num_queries; q += (long long)gridDim.x * kBlock)
    {
        float4 c;
        if (toggle_single(P, S, query_of(P, q), c))
            qcol[q] = c;
        else
        {
            const int slot = atomicAdd(ovf_count, 1);
            if (slot < ovf_cap)
                ovf_queue[slot] = (int)q;
        }
    }
}

// The queued output samples with large lists from a global arena (one slot
// per thread); a sample that outgrows those too is counted as a hard failure.
__global__ void __launch_bounds__(64)
k_toggle_large(QParams P, const int* __restrict__ queue, const int* __restrict__ count_ptr, int cap,
               float4* __restrict__ qcol, char* arena, size_t slot_bytes, int num_slots, int stack_cap, int leaf_cap,
               int xy_cap, int* hard_fail)
{
    const int count = min(*count_ptr, cap);
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= num_slots)
        return;
    char* base = arena + (size_t)slot * slot_bytes;
    TStore S;
    S.stack = (int*)base;                       S.stack_cap = stack_cap;
    S.leaves = S.stack + stack_cap;             S.leaf_cap = leaf_cap;
    S.xy = (float2*)(S.leaves + leaf_cap);      S.xy_cap = xy_cap;
    for (int k = slot; k < count; k += num_slots)
    {
        const int q = queue[k];
        float4 c;
        if (!toggle_single(P, S, query_of(P, q), c))
        {
            atomicAdd(hard_fail, 1);
            c = make_float4(0, 0, 0, 0);
        }
        qcol[q] = c;
    }
}

// overflow pass capacities
constexpr int kOvStack = 512, kOvLeaf = 16384, kOvRs = 65536, kOvSurf = 4096;
constexpr int kOvSlots = 4096;

// ---------------------------------------------------------------------------
// Shadow reconstruction (TreeGather::reconstructShadows, R.cpp:302-344): the
// hierarchy holds light-space samples; each query is a light-space sample of
// the view (x, y, u, v, t, w and its light-space density) and receives, from
// the Filterer in shadow mode, the colour of the samples that light it
// (RO.cpp:78-80, 283-291, 337-347).  Queries are 8 floats: x, y, u, v, t, w,
// density, unused.
// ---------------------------------------------------------------------------
__device__ __forceinline__ Query shadow_query(const float* q8, float& w, float& density)
{
    Query o;
    o.x = q8[0]; o.y = q8[1]; o.u = q8[2]; o.v = q8[3]; o.t = q8[4];
    w = q8[5];
    density = q8[6];
    return o;
}

// dw/dx, dw/dy of every tree-ordered sample from its input record
__global__ void k_gather_wg(const float* __restrict__ records, const int* __restrict__ s_id, int n,
                            float2* __restrict__ wg)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    {
        const float* r = records + (size_t)s_id[k] * 16;
        wg[k] = make_float2(r[14], r[15]);
    }
}

__global__ void __launch_bounds__(kBlock)
k_query_shadow(QParams P, const float* __restrict__ queries, int n, const float2* __restrict__ wg,
               float4* __restrict__ out, int* __restrict__ ovf_queue, int* __restrict__ ovf_count, int ovf_cap)
{
    int stack[kStackCap];
    Leaf leaves[kLeafCap];
    RSample rs[kRsCap];
    Surf surf[kSurfCap];
    Store S{ stack, kStackCap, leaves, kLeafCap, rs, kRsCap, surf, kSurfCap };
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < n; k += gridDim.x * kBlock)
    {
        float w, density;
        const Query o = shadow_query(queries + 8 * (size_t)k, w, density);
        const ShadowQ sh{ w, P.disp0 * sqrtf(density), wg };
        QStats qs{};
        float4 c;
        if (reconstruct_query<false>(P, S, o, qs, c, nullptr, 0, &sh) == kQOk)
            out[k] = c;
        else
        {
            const int slot = atomicAdd(ovf_count, 1);
            if (slot < ovf_cap)
                ovf_queue[slot] = k;
        }
    }
}

__global__ void __launch_bounds__(64)
k_query_shadow_large(QParams P, const float* __restrict__ queries, const int* __restrict__ queue,
                     const int* __restrict__ count_ptr, int cap, const float2* __restrict__ wg, float4* __restrict__ out,
                     char* arena, size_t slot_bytes, int num_slots, int* hard_fail)
{
    const int count = min(*count_ptr, cap);
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= num_slots)
        return;
    char* base = arena + (size_t)slot * slot_bytes;
    Store S;
    S.stack = (int*)base;                      S.stack_cap = kOvStack;
    S.leaves = (Leaf*)(S.stack + kOvStack);    S.leaf_cap = kOvLeaf;
    S.rs = (RSample*)(S.leaves + kOvLeaf);     S.rs_cap = kOvRs;
    S.surf = (Surf*)(S.rs + kOvRs);            S.surf_cap = kOvSurf;
    for (int j = slot; j < count; j += num_slots)
    {
        const int k = queue[j];
        float w, density;
        const Query o = shadow_query(queries + 8 * (size_t)k, w, density);
        const ShadowQ sh{ w, P.disp0 * sqrtf(density), wg };
        QStats qs{};
        float4 c;
        if (reconstruct_query<false>(P, S, o, qs, c, nullptr, 0, &sh) != kQOk)
        {
            atomicAdd(hard_fail, 1);
            c = make_float4(0, 0, 0, 0);
        }
        out[k] = c;
    }
}

// ---------------------------------------------------------------------------
// Motion and defocus with soft shadows from a square area light
// (TreeGather::reconstructDofMotionShadows, R.cpp:355-433; FilterTask::process2,
// R.cpp:723-829).  Every output sample is reconstructed from the camera's
// hierarchy; the nearest sample's position and w place it in the light's
// image through the camera-to-light matrix; a point on the light source
// (Sobol dimensions 3 and 4 of the sample, rotated per pixel) moves it across
// the light's lens; the light's hierarchy reconstructs it in shadow mode, and
// the result is shaded with the normal rebuilt from the nearest sample's w
// gradients (lightSpaceDot, viewSpaceNormalFromWGradients, Util.cpp:174-224).
// The matrix and vector arithmetic keeps the framework's operation order
// (framework/base/Math.hpp: sums accumulate from 0 in index order, rcp(0) = 0,
// normalized = v * (1 * rcp(length))), so the results are bit-identical.
// ---------------------------------------------------------------------------
struct DmsParams
{
    float c2l[16];          // ws * cameraToShadow * invws * cameraProjectedZfromW (row-major)
    float clip_xyw[16];     // invws * cameraProjectedZfromW
    float ip[16];           // invCameraProjection, rows 2 and 3 = (0,0,-1,0), (0,0,0,1)
    float light_pos[16];    // cameraToShadow2 * invCameraProjection
    float c2s_inv_t[16];    // cameraToShadow2 inverted, transposed
    float c2w_inv_t[16];    // cameraToWorld inverted, transposed
    float cam_far_w;        // camera far - 1e-2
    float ccoc0, ccoc1;     // CameraParams::getCocCoeffs of the camera
    float lcoc0, lcoc1;     // and of the light
    int   cw, ch;           // image size (the camera's and the light's)
    const float2* light_uv; // (sobol(3, i+1), sobol(4, i+1)) per output sample i
    const float2* cam_wg;   // dw/dx, dw/dy per camera tree-ordered sample
    const float*  cam_density;   // light-space density per camera tree-ordered sample (null: 1)
    const float2* light_wg; // dw/dx, dw/dy per light tree-ordered sample
};

// Mat4f * Vec4f (Math.hpp:1000-1011)
TLFR_HD float4 m4_apply(const float* m, float4 v)
{
    float r[4];
    for (int i = 0; i < 4; i++)
    {
        float a = 0.0f;
        a += m[4 * i + 0] * v.x;
        a += m[4 * i + 1] * v.y;
        a += m[4 * i + 2] * v.z;
        a += m[4 * i + 3] * v.w;
        r[i] = a;
    }
    return make_float4(r[0], r[1], r[2], r[3]);
}

TLFR_HD float3 v3_normalized(float3 v)
{
    float l2 = 0.0f;
    l2 += v.x * v.x;
    l2 += v.y * v.y;
    l2 += v.z * v.z;
    const float k = 1.0f * rcp(sqrtf(l2));
    return make_float3(v.x * k, v.y * k, v.z * k);
}

TLFR_HD float v3_dot(float3 a, float3 b)
{
    float r = 0.0f;
    r += a.x * b.x;
    r += a.y * b.y;
    r += a.z * b.z;
    return r;
}

// The light-source offset of pixel (x, y): the framework's Random seeded with
// hashBits(x, y) (Ranrot-A, framework/base/Random.cpp), two draws.  The
// reference builds the offset as Vec2f(random.getF32(), random.getF32()), whose
// arguments its compilers evaluate right to left: x takes the second draw.
TLFR_HD void light_uv_offset(int x, int y, float& ou, float& ov)
{
    uint32_t seed = hash_bits((uint32_t)x, (uint32_t)y);
    uint32_t buf[11];
    if (seed == 0)
        seed--;
    for (int k = 0; k < 11; k++)
    {
        seed ^= seed << 13;
        seed ^= seed >> 17;
        seed ^= seed << 5;
        buf[k] = seed;
    }
    int p1 = 0, p2 = 7;
    uint32_t draw = 0;
    for (int k = 0; k < 13; k++)
    {
        uint32_t v = buf[p1] + buf[p2];
        v = (v << 13) | (v >> 19);
        buf[p1] = v;
        p1--; p1 += (p1 >> 31) & 11;
        p2--; p2 += (p2 >> 31) & 11;
        if (k == 11)
            draw = v;
        if (k == 12)
        {
            ou = (float)v * (1.0f / 4294967296.0f);
            ov = (float)draw * (1.0f / 4294967296.0f);
        }
    }
}

// Output sample i of pixel (x, y).  red: the camera reconstruction found
// nothing, which turns the whole pixel red (R.cpp:764-768).
TLFR_HD int dms_sample(const QParams& Pc, const QParams& Pl, const DmsParams& D, Store& S, int x, int y, int i,
                       float4& col, bool& red, QStats& st)
{
    const Query o = make_query(Pc, x, y, i);
    QNear nr{ 0.0f, 0.0f, 0.0f, 0 };
    float4 cc;
    if (reconstruct_query<false>(Pc, S, o, st, cc, nullptr, 0, nullptr, &nr) != kQOk)
        return kQOverflow;
    red = cc.x == 0.0f && cc.y == 0.0f && cc.z == 0.0f && cc.w == 0.0f;
    col = cc;
    if (red || !(nr.w <= D.cam_far_w))
        return kQOk;

    // Sample::reprojectToUVCenter (Reconstruction.hpp:93-97) with the camera's CoC
    const float cr = D.ccoc0 / nr.w + D.ccoc1;
    const float sx = nr.x - o.u * cr, sy = nr.y - o.v * cr;
    const float4 xyw = make_float4(sx * nr.w, sy * nr.w, 1.0f, nr.w);
    float4 lp = m4_apply(D.c2l, xyw);
    const float lc = rcp(lp.w);
    lp.x *= lc; lp.y *= lc; lp.z *= lc;
    if (!(lp.x >= 0.0f && lp.y >= 0.0f && lp.x <= (float)D.cw && lp.y <= (float)D.ch && lp.w > 0.0f))
        return kQOk;

    // the light-space query: a point on the square light source [-1,1]^2
    float ou = 0.0f, ov = 0.0f;
    light_uv_offset(x, y, ou, ov);
    const float2 s34 = D.light_uv[i];
    float u = s34.x + ou, v = s34.y + ov;
    if (u >= 1.0f) u -= 1.0f;
    if (v >= 1.0f) v -= 1.0f;
    Query ls;
    ls.u = 2.0f * u - 1.0f;
    ls.v = 2.0f * v - 1.0f;
    ls.t = o.t;
    const float lr = D.lcoc0 / lp.w + D.lcoc1;
    ls.x = lp.x + ls.u * lr;
    ls.y = lp.y + ls.v * lr;
    const float density = D.cam_density ? D.cam_density[nr.index] : 1.0f;
    const ShadowQ sh{ lp.w, Pl.disp0 * sqrtf(density), D.light_wg };
    float4 sc;
    if (reconstruct_query<false>(Pl, S, ls, st, sc, nullptr, 0, &sh) != kQOk)
        return kQOverflow;

    // lightSpaceDot: the view-space normal from the w gradients, against the
    // direction to the light
    const float4 p = m4_apply(D.clip_xyw, xyw);
    const float pu = p.x / p.w, pv = p.y / p.w;
    const float2 g = D.cam_wg[nr.index];
    const float dwdu = g.x * ((float)D.cw / 2.0f);
    const float dwdv = g.y * ((float)D.ch / 2.0f);
    const float4 b1 = m4_apply(D.ip, make_float4(p.w + pu * dwdu, pv * dwdu, dwdu, 0.0f));
    const float4 b2 = m4_apply(D.ip, make_float4(pu * dwdv, p.w + pv * dwdv, dwdv, 0.0f));
    const float3 n = v3_normalized(make_float3(b1.y * b2.z - b1.z * b2.y, b1.z * b2.x - b1.x * b2.z,
                                               b1.x * b2.y - b1.y * b2.x));
    const float4 nl = m4_apply(D.c2s_inv_t, make_float4(n.x, n.y, n.z, 0.0f));
    const float4 pl = m4_apply(D.light_pos, p);
    const float plc = rcp(pl.w);
    const float ldotn = -v3_dot(v3_normalized(make_float3(pl.x * plc, pl.y * plc, pl.z * plc)),
                                v3_normalized(make_float3(nl.x, nl.y, nl.z)));
    const float4 wn = m4_apply(D.c2w_inv_t, make_float4(n.x, n.y, n.z, 0.0f));
    const float ambient = wn.y * 0.5f + 0.5f;
    const float k = maxr(ldotn, 0.0f) * 1.5f;     // LIGHTING_SCALE (R.cpp:34)
    const float a = ambient * 0.5f;               // AMBIENT_SCALE (R.cpp:35)
    col = make_float4(sc.x * k + cc.x * a, sc.y * k + cc.y * a, sc.z * k + cc.z * a, 1.0f);
    return kQOk;
}

// dw/dx, dw/dy and the light-space density of every tree-ordered sample (density null: skipped)
__global__ void k_gather_wg_density(const float* __restrict__ records, const int* __restrict__ s_id, int n,
                                    const float* __restrict__ density_in, float2* __restrict__ wg,
                                    float* __restrict__ density)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    {
        const int id = s_id[k];
        const float* r = records + (size_t)id * 16;
        wg[k] = make_float2(r[14], r[15]);
        if (density_in)
            density[k] = density_in[id];
    }
}

__global__ void __launch_bounds__(kBlock)
k_query_dms(QParams Pc, QParams Pl, DmsParams D, float4* __restrict__ qcol, int* __restrict__ red,
            int* __restrict__ ovf_queue, int* __restrict__ ovf_count, int ovf_cap)
{
    int stack[kStackCap];
    Leaf leaves[kLeafCap];
    RSample rs[kRsCap];
    Surf surf[kSurfCap];
    Store S{ stack, kStackCap, leaves, kLeafCap, rs, kRsCap, surf, kSurfCap };
    const long long n = (long long)Pc.W * Pc.H * Pc.M;
    for (long long q = blockIdx.x * (long long)kBlock + threadIdx.x; q < n; q += (long long)gridDim.x * kBlock)
    {
        const int pix = (int)(q / Pc.M), i = (int)(q % Pc.M);
        QStats qs{};
        float4 c;
        bool r = false;
        if (dms_sample(Pc, Pl, D, S, pix % Pc.W, pix / Pc.W, i, c, r, qs) == kQOk)
        {
            qcol[q] = c;
            if (r)
                red[pix] = 1;
        }
        else
        {
            const int slot = atomicAdd(ovf_count, 1);
            if (slot < ovf_cap)
                ovf_queue[slot] = (int)q;
        }
    }
}

__global__ void __launch_bounds__(64)
k_query_dms_large(QParams Pc, QParams Pl, DmsParams D, const int* __restrict__ queue, const int* __restrict__ count_ptr,
                  int cap, float4* __restrict__ qcol, int* __restrict__ red, char* arena, size_t slot_bytes,
                  int num_slots, int* hard_fail)
{
    const int count = min(*count_ptr, cap);
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= num_slots)
        return;
    char* base = arena + (size_t)slot * slot_bytes;
    Store S;
    S.stack = (int*)base;                      S.stack_cap = kOvStack;
    S.leaves = (Leaf*)(S.stack + kOvStack);    S.leaf_cap = kOvLeaf;
    S.rs = (RSample*)(S.leaves + kOvLeaf);     S.rs_cap = kOvRs;
    S.surf = (Surf*)(S.rs + kOvRs);            S.surf_cap = kOvSurf;
    for (int j = slot; j < count; j += num_slots)
    {
        const int q = queue[j];
        const int pix = q / Pc.M, i = q % Pc.M;
        QStats qs{};
        float4 c;
        bool r = false;
        if (dms_sample(Pc, Pl, D, S, pix % Pc.W, pix / Pc.W, i, c, r, qs) != kQOk)
        {
            atomicAdd(hard_fail, 1);
            c = make_float4(0, 0, 0, 0);
        }
        qcol[q] = c;
        if (r)
            red[pix] = 1;
    }
}

// Pixel of the shadowed reconstruction: red when one of its output samples
// found nothing in the camera's hierarchy, else the sum of its samples in
// order times rcp(alpha), red when alpha is 0 (R.cpp:764-768, 823-828).
__global__ void k_resolve_dms(const float4* __restrict__ qcol, const int* __restrict__ red, int M,
                              float4* __restrict__ out, long long npix)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x)
    {
        float4 s = make_float4(0, 0, 0, 0);
        if (red[p])
            s = make_float4(1, 0, 0, 1);
        else
        {
            const float4* c = qcol + p * M;
            for (int i = 0; i < M; i++)
            {
                const float4 v = c[i];
                s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
            }
            if (s.w == 0)
                s = make_float4(1, 0, 0, 1);
        }
        const float r = rcp(s.w);
        out[p] = make_float4(s.x * r, s.y * r, s.z * r, s.w * r);
    }
}

// Pixel = sum of its output samples in sample order, times rcp(alpha); red
// when empty (Reconstruction.cpp:665-719).
__global__ void k_resolve(const float4* __restrict__ qcol, int M, float4* __restrict__ out, long long npix)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x)
    {
        const float4* c = qcol + p * M;
        float4 s = make_float4(0, 0, 0, 0);
        for (int i = 0; i < M; i++)
        {
            const float4 v = c[i];
            s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
        }
        if (s.w == 0)
            s = make_float4(1, 0, 0, 1);
        const float r = rcp(s.w);
        out[p] = make_float4(s.x * r, s.y * r, s.z * r, s.w * r);
    }
}

// Traced queries (parity tests): one thread per listed query, large capacities.
__global__ void k_query_trace(QParams P, const int* __restrict__ xyi, int n, float4* __restrict__ rgba,
                              int* __restrict__ trace, int stride, char* arena, size_t slot_bytes, int stack_cap,
                              int leaf_cap, int rs_cap, int surf_cap)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    char* base = arena + (size_t)k * slot_bytes;
    Store S;
    S.stack = (int*)base;                      S.stack_cap = stack_cap;
    S.leaves = (Leaf*)(S.stack + stack_cap);   S.leaf_cap = leaf_cap;
    S.rs = (RSample*)(S.leaves + leaf_cap);    S.rs_cap = rs_cap;
    S.surf = (Surf*)(S.rs + rs_cap);           S.surf_cap = surf_cap;
    QStats st{};
    const Query o = make_query(P, xyi[3 * k], xyi[3 * k + 1], xyi[3 * k + 2]);
    float4 c = make_float4(0, 0, 0, 0);
    int* tr = trace + (size_t)k * stride;
    int r = reconstruct_query<true>(P, S, o, st, c, tr, stride);
    if (r != kQOk && stride > 1)
        tr[1] = -1;
    rgba[k] = c;
}

size_t slot_bytes_for(int stack_cap, int leaf_cap, int rs_cap, int surf_cap)
{
    size_t b = sizeof(int) * stack_cap + sizeof(Leaf) * leaf_cap + sizeof(RSample) * rs_cap + sizeof(Surf) * surf_cap;
    return (b + 255) & ~(size_t)255;
}

QParams make_params(const Ctx& c)
{
    QParams P;
    P.nodes = c.nodes;
    P.s_rec = c.s_rec;
    P.s_col = c.s_col;
    P.pattern = c.d_pattern;
    P.M = c.out_spp;
    P.W = c.W;
    P.H = c.H;
    P.root = c.root;
    P.c0 = c.coc[0];
    P.c1 = c.coc[1];
    P.disp0 = dispersion_for_spp(c.spp);
    P.lens_filter = c.params.lens_filter;
    P.time_filter = c.params.time_filter;
    P.route_fast = nullptr;
    return P;
}

int coop_blocks(const Ctx& c) { return c.num_sms * kCoopBlocksPerSM; }


} // namespace

#define CKQ(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { c.error = std::string(#x) + ": " + cudaGetErrorString(_e); return (_e == cudaErrorMemoryAllocation) ? TLFR_OOM : TLFR_CUDA; } } while (0)

size_t coop_scratch_bytes(int num_sms) { return sizeof(CoopScratch) * (size_t)num_sms * kCoopBlocksPerSM * kCWarps; }

// light pass iterations and lane map of a frame (nq_probe > 0: the router's
// probe pass over nq_probe output samples, linear)
static LightMap light_map(const Ctx& c, long long nq_probe = 0, int shape = kDefaultShape)
{
    LightMap L{};
    const int tw = kTileShapes[shape][0], th = kTileShapes[shape][1], sw = 32 / (tw * th);
    if (nq_probe > 0 || c.out_spp % (4 * sw) != 0)
    {
        const long long nq = nq_probe > 0 ? nq_probe : (long long)c.W * c.H * c.out_spp;
        L.mode = kMapLinear;
        L.units = (nq + kBlock - 1) / kBlock;
        return L;
    }
    L.mode = kMapTiles;
    L.tw = tw; L.th = th; L.sw = sw;
    L.tiles_x = (c.W + tw - 1) / tw;
    L.groups = c.out_spp / (4 * sw);
    L.units = (long long)L.tiles_x * ((c.H + th - 1) / th) * L.groups;
    return L;
}
size_t overflow_scratch_bytes() { return slot_bytes_for(kOvStack, kOvLeaf, kOvRs, kOvSurf) * kOvSlots; }

tlfr_status route_probe(Ctx& c, int* d_counts)
{
    cudaStream_t s = c.stream;
    const long long npix = (long long)c.W * c.H;
    const long long nq = npix * kProbe;
    if (nq >= kQueueRestart)
    {
        c.error = "route probe: frame too large";
        return TLFR_BAD_ARG;
    }
    QParams P = make_params(c);
    CKQ(cudaMemsetAsync(d_counts, 0, sizeof(int) * npix, s));
    const LightMap L = light_map(c, nq);
    const int blocks = (int)std::min<long long>(L.units, (long long)c.num_sms * 64);
    TLFR_LAUNCH(c, K_LIGHT_PLAIN(true), blocks, kBlock, s, P, L, nq, nullptr, nullptr, d_counts, nullptr, nullptr);
    CKQ(cudaGetLastError());
    return TLFR_OK;
}

int light_default_blocks(const Ctx& c)
{
    const LightMap L = light_map(c);
    return (int)std::min<long long>(L.units, (long long)c.num_sms * 64);
}

// ---------------------------------------------------------------------------
// Batches: many frames (contexts of any size and spp, or one context under
// several output settings, each with its own output pattern) in one CUDA graph.
// Each pass runs as ONE persistent launch over all frames of a chunk: blocks
// (warps for the full path) take work items from a device counter, find their
// frame by a binary search over the items' frame offsets and run that frame's
// unit with its parameters from a device table of frame descriptors.  The
// working storage (per-output-sample colours and queues) belongs to the batch;
// frames are grouped into chunks whose storage fits the budget, and the chunks
// run one after another in the graph, reusing it.  The light pass's tile shape
// is chosen per frame by timing each shape (autotune).
// ---------------------------------------------------------------------------
struct FrameDesc
{
    QParams P;
    LightMap L;
    long long nq;
    long long npix;
    float4* qcol;
    int* heavy;
    int* ovf;
    int* counters;          // [0] overflow queue, [1] capacity failures, [2] heavy queue, [3] retry list
    float4* out;
};

namespace
{

// frame of global index x: the last f with begin[f] <= x
__device__ __forceinline__ int frame_of(const long long* __restrict__ begin, int n, long long x)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (begin[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Light pass over every frame of a chunk: a block takes one unit at a time.
// FIRST: every output sample of every frame (LightMap units), those that
// outgrow the first tier's capacities appended to the frame's retry list (its
// overflow queue, counters[3]); otherwise the retry lists (units of kBlock
// entries, offsets from k_batch_retry_units), overflow to the full path.
template <bool FIRST>
__global__ void __launch_bounds__(kBlock, FIRST ? kL1BlocksPerSM : kL2BlocksPerSM)
k_batch_light(const FrameDesc* __restrict__ fd, const long long* __restrict__ unit_begin, int nframes,
              unsigned long long* __restrict__ next_unit)
{
    __shared__ LightShared<FIRST ? kL1Leaf : kL2Leaf, FIRST ? kL1Stack : kL2Stack> sh;
    __shared__ QParams sP;
    __shared__ LightMap sL;
    __shared__ long long sU;
    __shared__ int sF;
    const long long total = unit_begin[nframes];
    int cur = -1;
    for (;;)
    {
        if (threadIdx.x == 0)
        {
            const long long u = (long long)atomicAdd(next_unit, 1ull);
            sU = u;
            sF = u < total ? frame_of(unit_begin, nframes, u) : -1;
            if (sF >= 0 && sF != cur)
            {
                sP = fd[sF].P;
                sL = fd[sF].L;
            }
        }
        __syncthreads();
        const long long u = sU;
        const int f = sF;
        if (u >= total)
            break;
        cur = f;
        const FrameDesc& D = fd[f];
        if constexpr (FIRST)
            light_unit<false, kL1Leaf, kL1Stack, kLightFirst>(sP, sL, u - unit_begin[f], D.nq, D.qcol, D.heavy,
                                                              D.counters + 2, sh, D.ovf, D.counters + 3);
        else
            light_unit<false, kL2Leaf, kL2Stack, kLightRetry>(sP, sL, u - unit_begin[f], D.counters[3], D.qcol,
                                                              D.heavy, D.counters + 2, sh, D.ovf);
        __syncthreads();
    }
}

// Units of the retry pass: kBlock retried output samples each.
__global__ void k_batch_retry_units(const FrameDesc* __restrict__ fd, int nframes, long long* __restrict__ unit_begin)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    long long acc = 0;
    for (int f = 0; f < nframes; f++)
    {
        unit_begin[f] = acc;
        acc += (fd[f].counters[3] + kBlock - 1) / kBlock;
    }
    unit_begin[nframes] = acc;
}

// Work items of the full-path pass: 32 queued output samples each.
__global__ void k_batch_items(const FrameDesc* __restrict__ fd, int nframes, long long* __restrict__ item_begin)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    long long acc = 0;
    for (int f = 0; f < nframes; f++)
    {
        item_begin[f] = acc;
        acc += (fd[f].counters[2] + 31) / 32;
    }
    item_begin[nframes] = acc;
}

// Full-path pass over every frame of a chunk: a warp takes one item at a time.
__global__ void __launch_bounds__(kCWarps * 32, TLFR_COOP_BLOCKS_PER_SM)
k_batch_coop(const FrameDesc* __restrict__ fd, const long long* __restrict__ item_begin, int nframes,
             unsigned long long* __restrict__ next_item, CoopScratch* __restrict__ scratch)
{
    __shared__ CoopShared sh_tri[kCWarps];
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * kCWarps + (threadIdx.x >> 5);
    const long long total = item_begin[nframes];
    for (;;)
    {
        long long it = 0;
        if (lane == 0)
            it = (long long)atomicAdd(next_item, 1ull);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= total)
            break;
        const int f = frame_of(item_begin, nframes, it);
        const FrameDesc& D = fd[f];
        coop_group(D.P, D.heavy, D.counters[2], (int)(it - item_begin[f]) * 32, D.qcol, D.ovf, D.counters + 0,
                   (int)D.nq, scratch[warp], sh_tri[threadIdx.x >> 5]);
    }
}

// Pixels of every frame of a chunk (k_resolve per frame).
__global__ void k_batch_resolve(const FrameDesc* __restrict__ fd, const long long* __restrict__ pix_begin, int nframes)
{
    const long long total = pix_begin[nframes];
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x)
    {
        const int f = frame_of(pix_begin, nframes, g);
        const FrameDesc& D = fd[f];
        const long long p = g - pix_begin[f];
        const int M = D.P.M;
        const float4* c = D.qcol + p * M;
        float4 s = make_float4(0, 0, 0, 0);
        for (int i = 0; i < M; i++)
        {
            const float4 v = c[i];
            s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
        }
        if (s.w == 0)
            s = make_float4(1, 0, 0, 1);
        const float r = rcp(s.w);
        D.out[p] = make_float4(s.x * r, s.y * r, s.z * r, s.w * r);
    }
}

} // namespace

struct BatchChunk
{
    int first = 0, count = 0;           // frames [first, first + count)
    FrameDesc* d_desc = nullptr;        // into BatchPlan::d_desc
    long long* d_unit_begin = nullptr;  // count + 1
    long long* d_item_begin = nullptr;  // count + 1
    long long* d_pix_begin = nullptr;   // count + 1
    long long* d_retry_begin = nullptr; // count + 1
    unsigned long long* d_work = nullptr;   // [0] next light unit, [1] next full-path item, [2] next retry unit
};

struct BatchPlan
{
    std::vector<BatchEntry> entries;
    std::vector<FrameDesc> desc;        // host copy
    std::vector<BatchChunk> chunks;
    std::vector<int> shape;             // tile shape per frame
    std::vector<float*> patterns;       // per frame: its own output pattern (or null)
    FrameDesc* d_desc = nullptr;
    long long* d_offsets = nullptr;
    unsigned long long* d_work = nullptr;
    int* d_counters = nullptr;          // 4 per frame
    float4* qcol = nullptr;
    int* heavy = nullptr;
    int* ovf = nullptr;
    void* coop_scratch = nullptr;
    void* ovf_scratch = nullptr;
    int num_sms = 0;
};

size_t batch_storage_bytes(long long nq) { return (size_t)nq * (sizeof(float4) + 2 * sizeof(int)); }

void batch_release(BatchPlan& bp)
{
    for (float* p : bp.patterns)
        if (p) cudaFree(p);
    void* ptrs[] = { bp.d_desc, bp.d_offsets, bp.d_work, bp.d_counters, bp.qcol, bp.heavy, bp.ovf, bp.coop_scratch,
                     bp.ovf_scratch };
    for (void* p : ptrs)
        if (p) cudaFree(p);
    bp = BatchPlan{};
}

#define CKB(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { err = std::string(#x) + ": " + cudaGetErrorString(_e); return (_e == cudaErrorMemoryAllocation) ? TLFR_OOM : TLFR_CUDA; } } while (0)

// The light pass of one frame alone with a given tile shape (autotune), over
// its first eighth of block iterations (the top rows of the frame's tiles).
static tlfr_status light_trial(const FrameDesc& D, const Ctx& c, int shape, cudaStream_t s, float* ms,
                               std::string& err)
{
    cudaEvent_t e0, e1;
    CKB(cudaEventCreate(&e0));
    CKB(cudaEventCreate(&e1));
    LightMap L = D.L;
    {
        // the shape's map for this frame's output samples
        Ctx tmp;
        tmp.W = c.W; tmp.H = c.H; tmp.out_spp = D.P.M;
        L = light_map(tmp, 0, shape);
        L.units = std::max<long long>(std::min<long long>(L.units, 4096), L.units / 8);
    }
    const int blocks = (int)std::min<long long>(L.units, (long long)c.num_sms * 64);
    CKB(cudaMemsetAsync(D.counters, 0, 4 * sizeof(int), s));
    CKB(cudaEventRecord(e0, s));
    K_LIGHT_PLAIN(false)<<<blocks, kBlock, 0, s>>>(D.P, L, D.nq, D.qcol, D.heavy, D.counters + 2, nullptr, nullptr);
    CKB(cudaEventRecord(e1, s));
    CKB(cudaEventSynchronize(e1));
    CKB(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CKB(cudaGetLastError());
    return TLFR_OK;
}

tlfr_status batch_build(BatchPlan& bp, const std::vector<BatchEntry>& entries, cudaStream_t s, bool autotune,
                        size_t budget, std::string& err)
{
    const int n = (int)entries.size();
    bp.entries = entries;
    bp.num_sms = entries[0].ctx->num_sms;
    bp.desc.resize(n);
    bp.shape.assign(n, kDefaultShape);
    bp.patterns.assign(n, nullptr);
    // per frame: output pattern, parameters, sizes
    std::vector<long long> nq(n), npix(n);
    for (int f = 0; f < n; f++)
    {
        Ctx& c = *entries[f].ctx;
        FrameDesc& D = bp.desc[f];
        D.P = make_params(c);
        if (entries[f].output)
        {
            const tlfr_params& o = *entries[f].output;
            const bool ov = o.override_uvt != 0;
            const int M = o.output_spp > 0 ? o.output_spp : (ov ? 1 : 128);
            if (M > 1024)
            {
                err = "frame " + std::to_string(f) + ": output_spp out of range";
                return TLFR_BAD_ARG;
            }
            std::vector<float> pat;
            generate_output_pattern(M, ov, o.uvt, pat);
            CKB(cudaMalloc(&bp.patterns[f], sizeof(float) * pat.size()));
            CKB(cudaMemcpy(bp.patterns[f], pat.data(), sizeof(float) * pat.size(), cudaMemcpyHostToDevice));
            D.P.pattern = bp.patterns[f];
            D.P.M = M;
            D.P.lens_filter = o.lens_filter;
            D.P.time_filter = o.time_filter;
        }
        npix[f] = (long long)c.W * c.H;
        nq[f] = npix[f] * D.P.M;
        if (nq[f] >= kQueueRestart)
        {
            err = "frame " + std::to_string(f) + ": more than 2^30 output samples";
            return TLFR_BAD_ARG;
        }
        D.nq = nq[f];
        D.npix = npix[f];
        D.out = entries[f].out;
        Ctx tmp;
        tmp.W = c.W; tmp.H = c.H; tmp.out_spp = D.P.M;
        D.L = light_map(tmp, 0, kDefaultShape);
    }
    // chunks: consecutive frames whose storage fits the budget (a frame larger
    // than the budget is a chunk of its own)
    size_t largest = 0;
    for (int f = 0; f < n;)
    {
        BatchChunk ch;
        ch.first = f;
        size_t bytes = 0;
        while (f < n && (ch.count == 0 || bytes + batch_storage_bytes(nq[f]) <= budget))
        {
            bytes += batch_storage_bytes(nq[f]);
            f++;
            ch.count++;
        }
        largest = std::max(largest, bytes);
        bp.chunks.push_back(ch);
    }
    long long cap = 0;
    for (const BatchChunk& ch : bp.chunks)
    {
        long long t = 0;
        for (int f = ch.first; f < ch.first + ch.count; f++)
            t += nq[f];
        cap = std::max(cap, t);
    }
    CKB(cudaMalloc(&bp.qcol, sizeof(float4) * cap));
    CKB(cudaMalloc(&bp.heavy, sizeof(int) * cap));
    CKB(cudaMalloc(&bp.ovf, sizeof(int) * cap));
    CKB(cudaMalloc(&bp.d_counters, sizeof(int) * 4 * n));
    CKB(cudaMalloc(&bp.coop_scratch, coop_scratch_bytes(bp.num_sms)));
    CKB(cudaMalloc(&bp.ovf_scratch, overflow_scratch_bytes()));
    for (const BatchChunk& ch : bp.chunks)
    {
        long long off = 0;
        for (int f = ch.first; f < ch.first + ch.count; f++)
        {
            FrameDesc& D = bp.desc[f];
            D.qcol = bp.qcol + off;
            D.heavy = bp.heavy + off;
            D.ovf = bp.ovf + off;
            D.counters = bp.d_counters + 4 * f;
            off += nq[f];
        }
    }
    // router flags of frames with a router (and their context's own pattern)
    for (int f = 0; f < n; f++)
    {
        Ctx& c = *entries[f].ctx;
        if (c.router && !entries[f].output && !c.route_prob)
        {
            CKB(cudaMalloc(&c.route_feats, sizeof(float) * kRouteFeatures * npix[f]));
            CKB(cudaMalloc(&c.route_prob, sizeof(float) * npix[f]));
            CKB(cudaMalloc(&c.route_fast, npix[f]));
        }
        if (c.router && !entries[f].output)
            bp.desc[f].P.route_fast = c.route_fast;
    }
    // autotune: each frame's light pass alone with every tile shape, once per
    // frame class (size, input spp, output samples per pixel)
    if (autotune)
    {
        std::vector<std::array<int, 5>> seen;    // (W, H, spp, M, shape)
        for (int f = 0; f < n; f++)
        {
            const Ctx& cf = *entries[f].ctx;
            bool known = false;
            for (const auto& k : seen)
                if (k[0] == cf.W && k[1] == cf.H && k[2] == cf.spp_in && k[3] == bp.desc[f].P.M)
                {
                    bp.shape[f] = k[4];
                    known = true;
                }
            float best = known ? -1.0f : 1e30f;
            for (int sh = 0; sh < (int)(sizeof(kTileShapes) / sizeof(kTileShapes[0])); sh++)
            {
                if (known)
                    break;
                float ms = 0;
                const tlfr_status st = light_trial(bp.desc[f], *entries[f].ctx, sh, s, &ms, err);
                if (st != TLFR_OK)
                    return st;
                if (ms < best)
                {
                    best = ms;
                    bp.shape[f] = sh;
                }
            }
            if (!known)
                seen.push_back({ cf.W, cf.H, cf.spp_in, bp.desc[f].P.M, bp.shape[f] });
            Ctx tmp;
            tmp.W = entries[f].ctx->W; tmp.H = entries[f].ctx->H; tmp.out_spp = bp.desc[f].P.M;
            bp.desc[f].L = light_map(tmp, 0, bp.shape[f]);
        }
    }
    // device tables
    CKB(cudaMalloc(&bp.d_desc, sizeof(FrameDesc) * n));
    CKB(cudaMalloc(&bp.d_offsets, sizeof(long long) * 4 * (n + bp.chunks.size())));
    CKB(cudaMalloc(&bp.d_work, sizeof(unsigned long long) * 3 * bp.chunks.size()));
    std::vector<long long> offs;
    offs.reserve(4 * (n + bp.chunks.size()));
    for (size_t k = 0; k < bp.chunks.size(); k++)
    {
        BatchChunk& ch = bp.chunks[k];
        ch.d_desc = bp.d_desc + ch.first;
        ch.d_work = bp.d_work + 3 * k;
        const size_t base = offs.size();
        long long u = 0, pxl = 0;
        std::vector<long long> ub, pb;
        for (int f = ch.first; f < ch.first + ch.count; f++)
        {
            ub.push_back(u);
            pb.push_back(pxl);
            u += bp.desc[f].L.units;
            pxl += npix[f];
        }
        ub.push_back(u);
        pb.push_back(pxl);
        offs.insert(offs.end(), ub.begin(), ub.end());
        offs.insert(offs.end(), pb.begin(), pb.end());
        offs.insert(offs.end(), 2 * (ch.count + 1), 0LL);    // item and retry offsets, filled on the device
        ch.d_unit_begin = bp.d_offsets + base;
        ch.d_pix_begin = bp.d_offsets + base + ch.count + 1;
        ch.d_item_begin = bp.d_offsets + base + 2 * (ch.count + 1);
        ch.d_retry_begin = bp.d_offsets + base + 3 * (ch.count + 1);
    }
    CKB(cudaMemcpy(bp.d_offsets, offs.data(), sizeof(long long) * offs.size(), cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(bp.d_desc, bp.desc.data(), sizeof(FrameDesc) * n, cudaMemcpyHostToDevice));
    return TLFR_OK;
}

// Every pass of every chunk, on stream s, with no host synchronisation (the
// counts the full-path and large-capacity passes need are read on the device).
tlfr_status batch_enqueue(BatchPlan& bp, cudaStream_t s, std::string& err, long long* launches)
{
    const int n = (int)bp.entries.size();
    long long L = 0;
    CKB(cudaMemsetAsync(bp.d_counters, 0, sizeof(int) * 4 * n, s));
    CKB(cudaMemsetAsync(bp.d_work, 0, sizeof(unsigned long long) * 3 * bp.chunks.size(), s));
    for (const BatchChunk& ch : bp.chunks)
    {
        // the router's flags for this chunk's routed frames (their descriptors
        // point at the context's flags)
        for (int f = ch.first; f < ch.first + ch.count; f++)
        {
            Ctx& c = *bp.entries[f].ctx;
            if (!c.router || bp.entries[f].output)
                continue;
            cudaStream_t saved = c.stream;
            c.stream = s;
            const long long np = (long long)c.W * c.H;
            tlfr_status rs = route_features(c, c.route_feats, err);
            if (rs == TLFR_OK)
                rs = route_predict(*c.router, c.route_feats, np, c.route_prob, s, err);
            if (rs == TLFR_OK)
                rs = route_flags(c, c.route_prob, c.route_hi, c.route_fast, err);
            c.stream = saved;
            if (rs != TLFR_OK)
                return rs;
            L += 7;
        }
        // first light pass, then the retry lists (in the frames' overflow
        // queues, which the full-path pass fills only after they are read)
        k_batch_light<true><<<bp.num_sms * kL1BlocksPerSM, kBlock, 0, s>>>(ch.d_desc, ch.d_unit_begin, ch.count,
                                                                         ch.d_work + 0);
        k_batch_retry_units<<<1, 32, 0, s>>>(ch.d_desc, ch.count, ch.d_retry_begin);
        k_batch_light<false><<<bp.num_sms * kL2BlocksPerSM, kBlock, 0, s>>>(ch.d_desc, ch.d_retry_begin, ch.count,
                                                                          ch.d_work + 2);
        k_batch_items<<<1, 32, 0, s>>>(ch.d_desc, ch.count, ch.d_item_begin);
        k_batch_coop<<<bp.num_sms * kCoopBlocksPerSM, kCWarps * 32, 0, s>>>(ch.d_desc, ch.d_item_begin, ch.count,
                                                                           ch.d_work + 1,
                                                                           reinterpret_cast<CoopScratch*>(bp.coop_scratch));
        L += 5;
        for (int f = ch.first; f < ch.first + ch.count; f++)
        {
            const FrameDesc& D = bp.desc[f];
            k_query_overflow<<<kOvSlots / 64, 64, 0, s>>>(D.P, D.ovf, D.counters + 0, (int)D.nq, D.qcol,
                                                         (char*)bp.ovf_scratch,
                                                         slot_bytes_for(kOvStack, kOvLeaf, kOvRs, kOvSurf), kOvSlots,
                                                         kOvStack, kOvLeaf, kOvRs, kOvSurf, D.counters + 1, nullptr, 0);
            L++;
        }
        k_batch_resolve<<<bp.num_sms * 32, 128, 0, s>>>(ch.d_desc, ch.d_pix_begin, ch.count);
        L++;
    }
    CKB(cudaGetLastError());
    if (launches)
        *launches = L;
    return TLFR_OK;
}

BatchPlan* batch_plan_new() { return new (std::nothrow) BatchPlan(); }

void batch_plan_delete(BatchPlan* bp)
{
    if (bp)
    {
        batch_release(*bp);
        delete bp;
    }
}

// tile shape (index into kTileShapes) per frame, chunk per frame
void batch_info(const BatchPlan& bp, int* shapes, int* chunks)
{
    for (size_t f = 0; f < bp.entries.size(); f++)
        if (shapes)
            shapes[f] = bp.shape[f];
    for (size_t k = 0; k < bp.chunks.size(); k++)
        for (int f = bp.chunks[k].first; f < bp.chunks[k].first + bp.chunks[k].count; f++)
            if (chunks)
                chunks[f] = (int)k;
}

// Output samples that exceeded every capacity, over all frames of the last run.
tlfr_status batch_failures(BatchPlan& bp, cudaStream_t s, std::vector<int>& hard, std::string& err)
{
    const int n = (int)bp.entries.size();
    std::vector<int> cnt(4 * n);
    CKB(cudaMemcpyAsync(cnt.data(), bp.d_counters, sizeof(int) * 4 * n, cudaMemcpyDeviceToHost, s));
    CKB(cudaStreamSynchronize(s));
    hard.resize(n);
    for (int f = 0; f < n; f++)
        hard[f] = cnt[4 * f + 1] + (cnt[4 * f + 0] > (int)bp.desc[f].nq ? 1 : 0);
    return TLFR_OK;
}

// capacities of the GPU-toggle algorithm's large pass (one arena slot per thread)
constexpr int kTgLargeStack = 512, kTgLargeLeaf = 8192, kTgLargeXy = 32768, kTgLargeSlots = 512;

static size_t toggle_slot_bytes()
{
    const size_t b = sizeof(int) * (kTgLargeStack + kTgLargeLeaf) + sizeof(float2) * kTgLargeXy;
    return (b + 255) & ~(size_t)255;
}

// A frame with the reference's GPU-toggle algorithm (enable_cuda): every output
// sample with per-thread lists, the ones that outgrew them with large lists,
// then the pixel resolve.
static tlfr_status reconstruct_toggle(Ctx& c, float4* d_rgba)
{
    cudaStream_t s = c.stream;
    const long long npix = (long long)c.W * c.H;
    const long long nq = npix * c.out_spp;
    int* counters = reinterpret_cast<int*>(c.d_stats + 1);
    QParams P = make_params(c);
    CKQ(cudaMemsetAsync(c.d_stats, 0, sizeof(DevStats) + 8 * sizeof(int), s));
    if (!c.evq0)
    {
        CKQ(cudaEventCreate(&c.evq0));
        CKQ(cudaEventCreate(&c.evq1));
        CKQ(cudaEventCreate(&c.evq2));
    }
    CKQ(cudaEventRecord(c.evq0, s));
    const int blocks = (int)std::min<long long>((nq + kBlock - 1) / kBlock, (long long)c.num_sms * 16);
    TLFR_LAUNCH(c, k_toggle, blocks, kBlock, s, P, nq, c.qcol, c.ovf_queue, counters + 0, (int)c.ovf_cap);
    CKQ(cudaEventRecord(c.evq1, s));
    int novf = 0;
    CKQ(cudaMemcpyAsync(&novf, counters + 0, sizeof(int), cudaMemcpyDeviceToHost, s));
    CKQ(cudaStreamSynchronize(s));
    int hard = 0;
    if (novf > 0)
    {
        if (!c.toggle_arena)
            CKQ(cudaMalloc(&c.toggle_arena, toggle_slot_bytes() * kTgLargeSlots));
        const int slots = std::min(kTgLargeSlots, novf);
        TLFR_LAUNCH(c, k_toggle_large, (slots + 63) / 64, 64, s, P, c.ovf_queue, counters + 0, (int)c.ovf_cap, c.qcol,
                    (char*)c.toggle_arena, toggle_slot_bytes(), slots, kTgLargeStack, kTgLargeLeaf, kTgLargeXy,
                    counters + 1);
        CKQ(cudaMemcpyAsync(&hard, counters + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    CKQ(cudaEventRecord(c.evq2, s));
    TLFR_LAUNCH(c, k_resolve, (int)std::min<long long>((npix + 127) / 128, (long long)c.num_sms * 32), 128, s, c.qcol,
                c.out_spp, d_rgba, npix);
    CKQ(cudaGetLastError());
    CKQ(cudaStreamSynchronize(s));
    float ms = 0, ms2 = 0;
    CKQ(cudaEventElapsedTime(&ms, c.evq0, c.evq1));
    CKQ(cudaEventElapsedTime(&ms2, c.evq1, c.evq2));
    c.last.light_ms = ms;
    c.last.heavy_ms = ms2;
    c.last.query_kernel_ms = ms + ms2;
    c.last.num_overflow_queries = novf;
    c.last.num_heavy_queries = novf;
    if (hard > 0)
    {
        c.error = "a query exceeded the largest supported capacity";
        return TLFR_OVERFLOW;
    }
    return TLFR_OK;
}

// Output-sample colours, the full-path and overflow queues of a frame of nq
// output samples, and the statistics block.  The overflow queue holds every
// output sample in the worst case, so no scene can exceed it.
tlfr_status frame_buffers(Ctx& c, long long nq)
{
    if ((size_t)nq > c.qcol_cap)
    {
        cudaFree(c.qcol); cudaFree(c.heavy_queue); cudaFree(c.ovf_queue);
        c.qcol = nullptr; c.heavy_queue = nullptr; c.ovf_queue = nullptr; c.qcol_cap = 0; c.ovf_cap = 0;
        CKQ(cudaMalloc(&c.qcol, sizeof(float4) * nq));
        CKQ(cudaMalloc(&c.heavy_queue, sizeof(int) * nq));
        CKQ(cudaMalloc(&c.ovf_queue, sizeof(int) * nq));
        c.qcol_cap = (size_t)nq;
        c.ovf_cap = (size_t)nq;
    }
    if (!c.d_stats)
        CKQ(cudaMalloc(&c.d_stats, sizeof(DevStats) + 8 * sizeof(int)));
    return TLFR_OK;
}

tlfr_status reconstruct_frame(Ctx& c, float4* d_rgba, bool collect_stats)
{
    cudaStream_t s = c.stream;
    const long long npix = (long long)c.W * c.H;
    const long long nq = npix * c.out_spp;
    if (nq >= kQueueRestart)
    {
        c.error = "more than 2^30 output samples in one frame";
        return TLFR_BAD_ARG;
    }
    tlfr_status fb = frame_buffers(c, nq);
    if (fb != TLFR_OK)
        return fb;
    if (c.params.enable_cuda)
        return reconstruct_toggle(c, d_rgba);
    int* counters = reinterpret_cast<int*>(c.d_stats + 1);   // [0] overflow, [1] hard, [2] heavy, [3] retry
    QParams P = make_params(c);
    CKQ(cudaMemsetAsync(c.d_stats, 0, sizeof(DevStats) + 8 * sizeof(int), s));
    if ((c.router || c.route_all_fast) && !c.route_prob)
    {
        CKQ(cudaMalloc(&c.route_feats, sizeof(float) * kRouteFeatures * npix));
        CKQ(cudaMalloc(&c.route_prob, sizeof(float) * npix));
        CKQ(cudaMalloc(&c.route_fast, npix));
    }
    if (c.route_all_fast)
    {
        // every pixel on the single-surface fast path (router labels)
        CKQ(cudaMemsetAsync(c.route_fast, 1, npix, s));
        P.route_fast = c.route_fast;
    }
    const int blocks = (int)std::min<long long>((nq + kBlock - 1) / kBlock, (long long)c.num_sms * 64);
    if (!c.evq0)
    {
        CKQ(cudaEventCreate(&c.evq0));
        CKQ(cudaEventCreate(&c.evq1));
        CKQ(cudaEventCreate(&c.evq2));
    }
    CKQ(cudaEventRecord(c.evq0, s));
    if (c.router && !c.route_all_fast && !collect_stats)
    {
        // learned routing: features, network, fast-path flags
        std::string err;
        tlfr_status rs = route_features(c, c.route_feats, err);
        if (rs == TLFR_OK)
            rs = route_predict(*c.router, c.route_feats, npix, c.route_prob, s, err);
        if (rs == TLFR_OK)
            rs = route_flags(c, c.route_prob, c.route_hi, c.route_fast, err);
        if (rs != TLFR_OK)
        {
            c.error = err;
            return rs;
        }
        c.launches++;
        P.route_fast = c.route_fast;
    }
    if (collect_stats)
    {
        TLFR_LAUNCH(c, k_query_stats, blocks, kBlock, s, P, nq, c.qcol, c.ovf_queue, counters + 0, (int)c.ovf_cap,
                    c.d_stats);
        CKQ(cudaEventRecord(c.evq1, s));
    }
    else
    {
        if (!c.coop_scratch)
        {
            c.coop_scratch_bytes = coop_scratch_bytes(c.num_sms);
            CKQ(cudaMalloc(&c.coop_scratch, c.coop_scratch_bytes));
        }
        // first light pass; the output samples that outgrow it are retried with
        // larger capacities (the retry list lives in the overflow queue, which
        // the full-path pass only fills after the retry pass has read it)
        TLFR_LAUNCH(c, K_LIGHT_FIRST, light_default_blocks(c), kBlock, s, P, light_map(c), nq, c.qcol,
                    c.heavy_queue, counters + 2, c.ovf_queue, counters + 3);
        TLFR_LAUNCH(c, K_LIGHT_RETRY, c.num_sms * kL2BlocksPerSM, kBlock, s, P, light_map(c), nq, c.qcol,
                    c.heavy_queue, counters + 2, c.ovf_queue, counters + 3);
        CKQ(cudaEventRecord(c.evq1, s));
        TLFR_LAUNCH(c, k_query_coop, coop_blocks(c), kCWarps * 32, s, P, c.heavy_queue, counters + 2, c.qcol,
                    c.ovf_queue, counters + 0, (int)c.ovf_cap, reinterpret_cast<CoopScratch*>(c.coop_scratch));
    }
    CKQ(cudaEventRecord(c.evq2, s));
    CKQ(cudaGetLastError());
    int host_counts[4] = { 0, 0, 0, 0 };
    CKQ(cudaMemcpyAsync(host_counts, counters, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
    CKQ(cudaStreamSynchronize(s));
    const int novf = host_counts[0];
    c.last.num_heavy_queries = host_counts[2];
    c.last.num_retried_queries = collect_stats ? 0 : host_counts[3];
    if (novf > (int)c.ovf_cap)
    {
        c.error = "overflow queue capacity exceeded";
        return TLFR_OVERFLOW;
    }
    int hard = 0;
    if (novf > 0)
    {
        const size_t sb = slot_bytes_for(kOvStack, kOvLeaf, kOvRs, kOvSurf);
        if (!c.ovf_scratch)
        {
            c.ovf_scratch_bytes = overflow_scratch_bytes();
            CKQ(cudaMalloc(&c.ovf_scratch, c.ovf_scratch_bytes));
        }
        const int slots = std::min(kOvSlots, novf);
        TLFR_LAUNCH(c, k_query_overflow, (slots + 63) / 64, 64, s, P, c.ovf_queue, counters + 0, (int)c.ovf_cap,
                    c.qcol, (char*)c.ovf_scratch,
                    sb, slots, kOvStack, kOvLeaf, kOvRs, kOvSurf, counters + 1, c.d_stats, collect_stats ? 1 : 0);
        CKQ(cudaGetLastError());
        CKQ(cudaMemcpyAsync(&hard, counters + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    TLFR_LAUNCH(c, k_resolve, (int)std::min<long long>((npix + 127) / 128, (long long)c.num_sms * 32), 128, s, c.qcol,
                c.out_spp, d_rgba, npix);
    CKQ(cudaGetLastError());
    {
        float ms = 0, ms2 = 0;
        CKQ(cudaEventElapsedTime(&ms, c.evq0, c.evq1));
        CKQ(cudaEventElapsedTime(&ms2, c.evq1, c.evq2));
        c.last.light_ms = ms;
        c.last.heavy_ms = ms2;
        c.last.query_kernel_ms = ms + ms2;
    }
    if (collect_stats || novf > 0)
    {
        DevStats ds;
        CKQ(cudaMemcpyAsync(&ds, c.d_stats, sizeof(ds), cudaMemcpyDeviceToHost, s));
        CKQ(cudaStreamSynchronize(s));
        if (collect_stats)
        {
            c.last.num_output_samples = (double)nq;
            c.last.num_leaf_nodes = (double)ds.leaf_nodes;
            c.last.num_samples_in_leaf_nodes = (double)ds.samples_in_leaves;
            c.last.num_samples_within_1r = (double)ds.within_1r;
            c.last.num_samples_fetched = (double)ds.fetched;
            c.last.num_surfaces = (double)ds.surfaces;
            c.last.num_2r = (double)ds.num_2r;
            c.last.num_surfaces_merged = (double)ds.merged;
            c.last.num_at_least_one = (double)ds.at_least_one;
            c.last.num_empty = (double)ds.empty;
            c.last.overflow_leaves = (double)ds.overflow_by_reason[1];
            c.last.overflow_stack = (double)ds.overflow_by_reason[2];
            c.last.overflow_surfaces = (double)ds.overflow_by_reason[3];
            c.last.overflow_samples = (double)ds.overflow_by_reason[0];
        }
    }
    c.last.num_overflow_queries = novf;
    if (hard > 0)
    {
        c.error = "a query exceeded the largest supported capacity";
        return TLFR_OVERFLOW;
    }
    return TLFR_OK;
}


// Shadow reconstruction of n queries (device, 8 floats each) into out (device).
tlfr_status reconstruct_shadows(Ctx& c, const float* d_queries, int n, float4* d_out)
{
    cudaStream_t s = c.stream;
    if (n <= 0)
        return TLFR_OK;
    if (!c.cur_records)
    {
        c.error = "no input records on the device";
        return TLFR_BAD_ARG;
    }
    QParams P = make_params(c);
    float2* wg = nullptr;
    int* queue = nullptr;
    CKQ(cudaMalloc(&wg, sizeof(float2) * (size_t)c.num_samples));
    tlfr_status st = TLFR_OK;
    if (cudaMalloc(&queue, sizeof(int) * (size_t)n) != cudaSuccess)
    {
        cudaFree(wg);
        c.error = "shadow queue allocation failed";
        return TLFR_OOM;
    }
    do
    {
        if (!c.d_stats && cudaMalloc(&c.d_stats, sizeof(DevStats) + 8 * sizeof(int)) != cudaSuccess)
        {
            st = TLFR_OOM;
            break;
        }
        int* counters = reinterpret_cast<int*>(c.d_stats + 1);
        cudaMemsetAsync(counters, 0, 8 * sizeof(int), s);
        const int gb = (int)std::min<long long>(((long long)c.num_samples + 255) / 256, (long long)c.num_sms * 16);
        TLFR_LAUNCH(c, k_gather_wg, gb > 0 ? gb : 1, 256, s, c.cur_records, c.s_id, c.num_samples, wg);
        const int blocks = (int)std::min<long long>(((long long)n + kBlock - 1) / kBlock, (long long)c.num_sms * 16);
        TLFR_LAUNCH(c, k_query_shadow, blocks, kBlock, s, P, d_queries, n, wg, d_out, queue, counters + 0, n);
        int novf = 0, hard = 0;
        cudaMemcpyAsync(&novf, counters + 0, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess)
        {
            st = TLFR_CUDA;
            break;
        }
        if (novf > 0)
        {
            if (!c.ovf_scratch)
            {
                c.ovf_scratch_bytes = overflow_scratch_bytes();
                if (cudaMalloc(&c.ovf_scratch, c.ovf_scratch_bytes) != cudaSuccess)
                {
                    st = TLFR_OOM;
                    break;
                }
            }
            const int slots = std::min(kOvSlots, novf);
            TLFR_LAUNCH(c, k_query_shadow_large, (slots + 63) / 64, 64, s, P, d_queries, queue, counters + 0, n, wg,
                        d_out, (char*)c.ovf_scratch, slot_bytes_for(kOvStack, kOvLeaf, kOvRs, kOvSurf), slots,
                        counters + 1);
            cudaMemcpyAsync(&hard, counters + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (cudaStreamSynchronize(s) != cudaSuccess)
            {
                st = TLFR_CUDA;
                break;
            }
        }
        if (hard > 0)
        {
            c.error = "a query exceeded the largest supported capacity";
            st = TLFR_OVERFLOW;
        }
    } while (0);
    if (st == TLFR_CUDA)
        c.error = std::string("reconstruct_shadows: ") + cudaGetErrorString(cudaGetLastError());
    cudaFree(wg);
    cudaFree(queue);
    return st;
}

// Motion and defocus with soft shadows (TreeGather::reconstructDofMotionShadows,
// Reconstruction.cpp:355-433): camera context c, light context l (same image
// size), derived views v, the camera buffer's light-space density per input
// record (device, or null), the image into d_img (device).
tlfr_status reconstruct_dof_motion_shadows(Ctx& c, Ctx& l, const DmsView& v, const float* d_density,
                                           float4* d_img)
{
    cudaStream_t s = c.stream;
    if (!c.cur_records || !l.cur_records)
    {
        c.error = "no input records on the device";
        return TLFR_BAD_ARG;
    }
    const long long npix = (long long)c.W * c.H;
    const long long nq = npix * c.out_spp;
    if (nq >= kQueueRestart)
    {
        c.error = "more than 2^30 output samples in one frame";
        return TLFR_BAD_ARG;
    }
    if ((int)v.light_uv.size() != 2 * c.out_spp)
    {
        c.error = "light-source pattern size mismatch";
        return TLFR_BAD_ARG;
    }
    tlfr_status st = frame_buffers(c, nq);
    if (st != TLFR_OK)
        return st;
    // the light's hierarchy was built on the light context's own stream
    if (cudaStreamSynchronize(l.stream) != cudaSuccess)
    {
        c.error = std::string("light context: ") + cudaGetErrorString(cudaGetLastError());
        return TLFR_CUDA;
    }
    float2* cam_wg = nullptr;
    float2* light_wg = nullptr;
    float* cam_density = nullptr;
    float2* light_uv = nullptr;
    int* red = nullptr;
    auto release = [&]() { cudaFree(cam_wg); cudaFree(light_wg); cudaFree(cam_density); cudaFree(light_uv); cudaFree(red); };
    if (cudaMalloc(&cam_wg, sizeof(float2) * (size_t)std::max(1, c.num_samples)) != cudaSuccess ||
        cudaMalloc(&light_wg, sizeof(float2) * (size_t)std::max(1, l.num_samples)) != cudaSuccess ||
        (d_density && cudaMalloc(&cam_density, sizeof(float) * (size_t)std::max(1, c.num_samples)) != cudaSuccess) ||
        cudaMalloc(&light_uv, sizeof(float2) * (size_t)c.out_spp) != cudaSuccess ||
        cudaMalloc(&red, sizeof(int) * (size_t)npix) != cudaSuccess)
    {
        release();
        c.error = "shadow reconstruction: allocation failed";
        return TLFR_OOM;
    }
    DmsParams D;
    memcpy(D.c2l, v.c2l, sizeof(D.c2l));
    memcpy(D.clip_xyw, v.clip_xyw, sizeof(D.clip_xyw));
    memcpy(D.ip, v.ip, sizeof(D.ip));
    memcpy(D.light_pos, v.light_pos, sizeof(D.light_pos));
    memcpy(D.c2s_inv_t, v.c2s_inv_t, sizeof(D.c2s_inv_t));
    memcpy(D.c2w_inv_t, v.c2w_inv_t, sizeof(D.c2w_inv_t));
    D.cam_far_w = v.cam_far_w;
    D.ccoc0 = v.ccoc[0]; D.ccoc1 = v.ccoc[1];
    D.lcoc0 = v.lcoc[0]; D.lcoc1 = v.lcoc[1];
    D.cw = c.W; D.ch = c.H;
    D.light_uv = light_uv;
    D.cam_wg = cam_wg;
    D.cam_density = cam_density;
    D.light_wg = light_wg;
    const QParams Pc = make_params(c);
    const QParams Pl = make_params(l);
    int* counters = reinterpret_cast<int*>(c.d_stats + 1);
    do
    {
        cudaMemcpyAsync(light_uv, v.light_uv.data(), sizeof(float2) * (size_t)c.out_spp, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(red, 0, sizeof(int) * (size_t)npix, s);
        cudaMemsetAsync(counters, 0, 8 * sizeof(int), s);
        const int gc = (int)std::min<long long>(((long long)c.num_samples + 255) / 256, (long long)c.num_sms * 16);
        TLFR_LAUNCH(c, k_gather_wg_density, gc > 0 ? gc : 1, 256, s, c.cur_records, c.s_id, c.num_samples, d_density,
                    cam_wg, cam_density);
        const int gl = (int)std::min<long long>(((long long)l.num_samples + 255) / 256, (long long)c.num_sms * 16);
        TLFR_LAUNCH(c, k_gather_wg_density, gl > 0 ? gl : 1, 256, s, l.cur_records, l.s_id, l.num_samples, nullptr,
                    light_wg, nullptr);
        const int blocks = (int)std::min<long long>((nq + kBlock - 1) / kBlock, (long long)c.num_sms * 16);
        TLFR_LAUNCH(c, k_query_dms, blocks, kBlock, s, Pc, Pl, D, c.qcol, red, c.ovf_queue, counters + 0,
                    (int)c.ovf_cap);
        int novf = 0, hard = 0;
        cudaMemcpyAsync(&novf, counters + 0, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess)
        {
            st = TLFR_CUDA;
            break;
        }
        if (novf > 0)
        {
            if (!c.ovf_scratch)
            {
                c.ovf_scratch_bytes = overflow_scratch_bytes();
                if (cudaMalloc(&c.ovf_scratch, c.ovf_scratch_bytes) != cudaSuccess)
                {
                    c.error = "shadow reconstruction: allocation failed";
                    st = TLFR_OOM;
                    break;
                }
            }
            const int slots = std::min(kOvSlots, novf);
            TLFR_LAUNCH(c, k_query_dms_large, (slots + 63) / 64, 64, s, Pc, Pl, D, c.ovf_queue, counters + 0,
                        (int)c.ovf_cap, c.qcol, red, (char*)c.ovf_scratch,
                        slot_bytes_for(kOvStack, kOvLeaf, kOvRs, kOvSurf), slots, counters + 1);
            cudaMemcpyAsync(&hard, counters + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (cudaStreamSynchronize(s) != cudaSuccess)
            {
                st = TLFR_CUDA;
                break;
            }
        }
        if (hard > 0)
        {
            c.error = "an output sample exceeded the largest supported capacity";
            st = TLFR_OVERFLOW;
            break;
        }
        const int rb = (int)std::min<long long>((npix + 255) / 256, (long long)c.num_sms * 16);
        TLFR_LAUNCH(c, k_resolve_dms, rb > 0 ? rb : 1, 256, s, c.qcol, red, c.out_spp, d_img, npix);
        if (cudaStreamSynchronize(s) != cudaSuccess)
            st = TLFR_CUDA;
    } while (0);
    if (st == TLFR_CUDA)
        c.error = std::string("reconstruct_dof_motion_shadows: ") + cudaGetErrorString(cudaGetLastError());
    release();
    return st;
}

tlfr_status trace_queries(Ctx& c, const int* h_xyi, int n, float* h_rgba, int* h_trace, int stride)
{
    if (n <= 0)
        return TLFR_OK;
    cudaStream_t s = c.stream;
    const int stack_cap = 1024, leaf_cap = 16384, rs_cap = 65536, surf_cap = 4096;
    const size_t sb = slot_bytes_for(stack_cap, leaf_cap, rs_cap, surf_cap);
    int* d_xyi = nullptr; float4* d_rgba = nullptr; int* d_trace = nullptr; char* arena = nullptr;
    tlfr_status st = TLFR_OK;
    const int chunk = 1024;
    QParams P = make_params(c);
    do
    {
        if (cudaMalloc(&d_xyi, sizeof(int) * 3 * chunk) != cudaSuccess ||
            cudaMalloc(&d_rgba, sizeof(float4) * chunk) != cudaSuccess ||
            cudaMalloc(&d_trace, sizeof(int) * (size_t)stride * chunk) != cudaSuccess ||
            cudaMalloc(&arena, sb * chunk) != cudaSuccess)
        {
            c.error = "trace_queries: allocation failed";
            st = TLFR_OOM;
            break;
        }
        for (int b = 0; b < n; b += chunk)
        {
            int m = std::min(chunk, n - b);
            cudaMemcpyAsync(d_xyi, h_xyi + 3 * b, sizeof(int) * 3 * m, cudaMemcpyHostToDevice, s);
            TLFR_LAUNCH(c, k_query_trace, (m + 63) / 64, 64, s, P, d_xyi, m, d_rgba, d_trace, stride, arena, sb, stack_cap,
                                                       leaf_cap, rs_cap, surf_cap);
            cudaMemcpyAsync(h_rgba + 4 * (size_t)b, d_rgba, sizeof(float4) * m, cudaMemcpyDeviceToHost, s);
            cudaMemcpyAsync(h_trace + (size_t)stride * b, d_trace, sizeof(int) * (size_t)stride * m,
                            cudaMemcpyDeviceToHost, s);
        }
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
        {
            c.error = std::string("trace_queries: ") + cudaGetErrorString(e);
            st = TLFR_CUDA;
        }
    } while (0);
    cudaFree(d_xyi); cudaFree(d_rgba); cudaFree(d_trace); cudaFree(arena);
    return st;
}

// ---------------------------------------------------------------------------
// Allocation-free output-sample queries.
//
// Callers that must not allocate device memory while they run (a renderer that
// reserves all its memory up front, a host thread that must not block on the
// allocator, code that owns the device heap through its own allocator) can still
// reconstruct individual output samples.  The per-query working storage that
// tlfr_trace_queries allocates per call lives here in one fixed device array
// instead: kNaSlots working slots of kNaSlotBytes each (9.75 MiB in all), which
// every device that loads this library keeps until the process exits.  Each
// slot runs the full per-sample path with capacities kNaStack / kNaLeaf /
// kNaRs / kNaSurf; a query that needs more is reported as (0, 0, 0, -1) and
// counted, not retried.
//
// All calls share the array: two calls whose kernels overlap on the GPU (on
// different streams, or from different contexts on the same device) race on it.
// The kernel needs nothing in the array to start at zero.
// ---------------------------------------------------------------------------
namespace
{
constexpr int kNaSlots = 256;
constexpr int kNaStack = 96, kNaLeaf = 512, kNaRs = 2048, kNaSurf = 128;
constexpr size_t kNaSlotBytes =
    (sizeof(int) * kNaStack + sizeof(Leaf) * kNaLeaf + sizeof(RSample) * kNaRs + sizeof(Surf) * kNaSurf + 255) &
    ~(size_t)255;
constexpr size_t kNaArenaBytes = kNaSlots * kNaSlotBytes;
static_assert(kNaArenaBytes == 10223616, "the documented size of the fixed array (9.75 MiB) follows the constants");
constexpr int kNaMaxQueries = 1 << 18;
constexpr int kNaMaxDevices = 64;
}

static __device__ __align__(256) unsigned char g_noalloc_arena[kNaArenaBytes];

namespace
{

__global__ void __launch_bounds__(32)
k_query_noalloc(QParams P, const int* __restrict__ xyi, int n, float4* __restrict__ rgba, unsigned char* arena,
                int* overflow)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= kNaSlots)
        return;
    unsigned char* base = arena + (size_t)slot * kNaSlotBytes;
    Store S;
    S.stack = (int*)base;                      S.stack_cap = kNaStack;
    S.leaves = (Leaf*)(S.stack + kNaStack);    S.leaf_cap = kNaLeaf;
    S.rs = (RSample*)(S.leaves + kNaLeaf);     S.rs_cap = kNaRs;
    S.surf = (Surf*)(S.rs + kNaRs);            S.surf_cap = kNaSurf;
    for (int k = slot; k < n; k += kNaSlots)
    {
        const int x = xyi[3 * k], y = xyi[3 * k + 1], i = xyi[3 * k + 2];
        float4 c = make_float4(0, 0, 0, -1);
        bool ok = x >= 0 && x < P.W && y >= 0 && y < P.H && i >= 0 && i < P.M;
        if (ok)
        {
            QStats qs{};
            ok = reconstruct_query<false>(P, S, make_query(P, x, y, i), qs, c, nullptr, 0) == kQOk;
        }
        if (!ok)
        {
            c = make_float4(0, 0, 0, -1);
            if (overflow)
                atomicAdd(overflow, 1);
        }
        rgba[k] = c;
    }
}

// Device address of g_noalloc_arena for each device, looked up on the first
// call made with that device current.  A later call checks that the address
// still belongs to the device (cudaPointerGetAttributes allocates nothing) and
// looks it up again when it does not (after a cudaDeviceReset the module and
// its array are loaded anew).
std::mutex g_na_lock;
void* g_na_ptr[kNaMaxDevices] = {};

} // namespace

tlfr_status query_samples_noalloc(Ctx& c, const int* d_xyi, int n, float* d_rgba, int* d_overflow)
{
    if (n < 0 || n > kNaMaxQueries)
    {
        c.error = "tlfr_query_samples_noalloc: num_queries " + std::to_string(n) + " outside [0, " +
                  std::to_string(kNaMaxQueries) + "]";
        return TLFR_BAD_ARG;
    }
    // colours are written as float4 and queries read as int: a misaligned
    // pointer would fault the kernel
    if (n > 0 && (!d_xyi || !d_rgba || (reinterpret_cast<uintptr_t>(d_rgba) & 15) != 0 ||
                  (reinterpret_cast<uintptr_t>(d_xyi) & 3) != 0))
    {
        c.error = "tlfr_query_samples_noalloc: d_rgba must be 16-byte aligned and d_xyi 4-byte aligned (non-null)";
        return TLFR_BAD_ARG;
    }
    if (d_overflow && (reinterpret_cast<uintptr_t>(d_overflow) & 3) != 0)
    {
        c.error = "tlfr_query_samples_noalloc: d_overflow must be 4-byte aligned";
        return TLFR_BAD_ARG;
    }
    if (c.device < 0 || c.device >= kNaMaxDevices)
    {
        c.error = "tlfr_query_samples_noalloc: device ordinal beyond the supported " + std::to_string(kNaMaxDevices);
        return TLFR_BAD_ARG;
    }
    void* arena = nullptr;
    {
        std::lock_guard<std::mutex> g(g_na_lock);
        void*& cached = g_na_ptr[c.device];
        if (cached)
        {
            cudaPointerAttributes a{};
            if (cudaPointerGetAttributes(&a, cached) != cudaSuccess || a.type != cudaMemoryTypeDevice ||
                a.device != c.device)
            {
                cudaGetLastError();
                cached = nullptr;
            }
        }
        if (!cached)
        {
            // the context's device is current (set by the caller of this function)
            cudaError_t e = cudaGetSymbolAddress(&cached, g_noalloc_arena);
            if (e != cudaSuccess)
            {
                cached = nullptr;
                c.error = std::string("tlfr_query_samples_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return TLFR_CUDA;
            }
        }
        arena = cached;
    }
    if (d_overflow)
    {
        cudaError_t e = cudaMemsetAsync(d_overflow, 0, sizeof(int), c.stream);
        if (e != cudaSuccess)
        {
            c.error = std::string("tlfr_query_samples_noalloc: ") + cudaGetErrorString(e);
            return TLFR_CUDA;
        }
    }
    if (n == 0)
        return TLFR_OK;
    QParams P = make_params(c);
    // 32-thread blocks spread the slots over kNaSlots / 32 multiprocessors
    TLFR_LAUNCH(c, k_query_noalloc, kNaSlots / 32, 32, c.stream, P, d_xyi, n, reinterpret_cast<float4*>(d_rgba),
                static_cast<unsigned char*>(arena), d_overflow);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        c.error = std::string("tlfr_query_samples_noalloc: ") + cudaGetErrorString(e);
        return TLFR_CUDA;
    }
    return TLFR_OK;
}

} // namespace tlfr
