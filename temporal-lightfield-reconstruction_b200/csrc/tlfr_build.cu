// tlfr_build.cu — GPU construction of the 5D sample hierarchy.
//
// Reproduces the reference builder (reconstruction/Reconstruction.cpp:52-215,
// ReconstructionTreeBuilder.cpp:34-451) node for node:
//
//   k_reproject       Sample::reprojectToUVTCenter (Reconstruction.hpp:93-121),
//                     bounding box and per-pixel hit histogram (Reconstruction.cpp:553-575)
//   k_grid_setup      grid scale and extent (Reconstruction.cpp:579-603)
//   k_bucket_*        bucketing in input order (Reconstruction.cpp:605-626): counting
//                     sort by cell, then each cell's list sorted by input index
//   k_kd_level        buildInitialRecursive (ReconstructionTreeBuilder.cpp:34-96), one
//                     launch per tree level
//   k_entry_points    the 32 build tasks (Reconstruction.cpp:110-126, 132-143)
//   k_leaf_prepare    per kd leaf: candidates in row-major cell order, FW::sort by (t,w),
//                     computeTUXPlanes and the t=0/t=1 boxes (RTB.cpp:131-213)
//   k_stale_boxes     a candidate with invalid bounds leaves its boxes unwritten and so
//                     reads what earlier leaves of its task left in the reused arrays
//                     (RTB.cpp:159-169, 184-212; Array::resize, Array.hpp:365-371, 668-692)
//   k_leaf_scan       surface scan and leaf nodes (RTB.cpp:222-378)
//   k_emit_level      emitNodes at every kd node inside a task, deepest level first
//                     (RTB.cpp:384-451)
//   k_top             serial top of the tree (Reconstruction.cpp:192-203)
//
// Node indices differ from the reference's (nodes are emitted in parallel), the
// tree structure, the child order, every bound and the sample order do not.
#include "tlfr_common.cuh"
#include "tlfr_internal.h"

#include <cstdio>
#include <cstring>

namespace tlfr
{

namespace
{

constexpr int kMaxKdLevels = 40;
constexpr int kTopCap = 1 << 16;

// error codes written to GridInfo::error
enum { kErrNone = 0, kErrKdDepth = 1, kErrTopCap = 2, kErrEmpty = 3 };

__device__ __forceinline__ unsigned float_to_ordered(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(unsigned u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

struct GridAccum
{
    unsigned bbmin[2], bbmax[2];
    int max_hits;
    int num_valid;
};

// ---------------------------------------------------------------------------
// Reprojection to (u,v,t) = centre, input order.
// ---------------------------------------------------------------------------
__global__ void k_reproject(const float4* __restrict__ rec, size_t n, int W, int H, float c0, float c1,
                            float4* __restrict__ rp_pos, float4* __restrict__ rp_mot,
                            int* __restrict__ hits, GridAccum* acc)
{
    float mnx = kF32Max, mny = kF32Max, mxx = -kF32Max, mxy = -kF32Max;
    int valid_count = 0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    {
        // record: x y z/w w | u v t r | g b a mv_x | mv_y mv_w dwdx dwdy
        float4 r0 = __ldg(&rec[k * 4 + 0]);
        float4 r1 = __ldg(&rec[k * 4 + 1]);
        float4 r2 = __ldg(&rec[k * 4 + 2]);
        float4 r3 = __ldg(&rec[k * 4 + 3]);
        float x = r0.x, y = r0.y, w = r0.w, u = r1.x, v = r1.y, t = r1.z;
        float mv[3] = { r2.w, r3.x, r3.y };
        // Sample::reprojectToUVTCenter (Reconstruction.hpp:93-121) with the header C0, C1
        float coc = c0 / w + c1;
        float px = x - u * coc;
        float py = y - v * coc;
        float P[3] = { px * w, py * w, 1.0f * w };
        float newt = 0.5f;
        float P0[3];
        for (int q = 0; q < 3; q++) P0[q] = (P[q] - mv[q] * t) + mv[q] * newt;
        if (P0[2] <= 0.f)
        {
            newt = 0.0f;
            for (int q = 0; q < 3; q++) P0[q] = (P[q] - mv[q] * t) + mv[q] * newt;
        }
        if (P0[2] <= 0.f)
        {
            newt = 1.0f;
            for (int q = 0; q < 3; q++) P0[q] = (P[q] - mv[q] * t) + mv[q] * newt;
        }
        bool valid = P0[2] > 0.f;
        float sw = P0[2];
        float cr = rcp(P0[2]);
        float sx = P0[0] * cr, sy = P0[1] * cr;
        rp_pos[k] = make_float4(sx, sy, sw, newt);
        rp_mot[k] = make_float4(mv[0], mv[1], mv[2], valid ? 1.0f : 0.0f);
        if (valid)
        {
            valid_count++;
            mnx = minr(mnx, sx); mny = minr(mny, sy);
            mxx = maxr(mxx, sx); mxy = maxr(mxy, sy);
            int ix = (int)floorf(sx), iy = (int)floorf(sy);
            if (ix >= 0 && iy >= 0 && ix < W && iy < H)
                atomicAdd(&hits[(size_t)iy * W + ix], 1);
        }
    }
    // block reduction of the bounding box and the valid count
    __shared__ float s[4][32];
    __shared__ int sc[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1)
    {
        mnx = minr(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = minr(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxx = maxr(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = maxr(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        valid_count += __shfl_xor_sync(0xffffffffu, valid_count, o);
    }
    if (lane == 0) { s[0][wid] = mnx; s[1][wid] = mny; s[2][wid] = mxx; s[3][wid] = mxy; sc[wid] = valid_count; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int q = 1; q < (int)(blockDim.x >> 5); q++)
        {
            mnx = minr(mnx, s[0][q]); mny = minr(mny, s[1][q]);
            mxx = maxr(mxx, s[2][q]); mxy = maxr(mxy, s[3][q]);
            valid_count += sc[q];
        }
        atomicMin(&acc->bbmin[0], float_to_ordered(mnx));
        atomicMin(&acc->bbmin[1], float_to_ordered(mny));
        atomicMax(&acc->bbmax[0], float_to_ordered(mxx));
        atomicMax(&acc->bbmax[1], float_to_ordered(mxy));
        atomicAdd(&acc->num_valid, valid_count);
    }
}

__global__ void k_max_hits(const int* __restrict__ hits, size_t n, GridAccum* acc)
{
    int m = 0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        m = maxi(m, hits[k]);
    for (int o = 16; o > 0; o >>= 1)
        m = maxi(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(&acc->max_hits, m);
}

// Reconstruction.cpp:579-603
__global__ void k_grid_setup(const GridAccum* acc, GridInfo* g)
{
    float bbmin[2] = { ordered_to_float(acc->bbmin[0]), ordered_to_float(acc->bbmin[1]) };
    float bbmax[2] = { ordered_to_float(acc->bbmax[0]), ordered_to_float(acc->bbmax[1]) };
    g->bbmin[0] = bbmin[0]; g->bbmin[1] = bbmin[1];
    g->bbmax[0] = bbmax[0]; g->bbmax[1] = bbmax[1];
    g->max_hits = acc->max_hits;
    g->num_valid = acc->num_valid;
    g->error = kErrNone;
    if (acc->max_hits == 0)
    {
        g->error = kErrEmpty;
        g->gw = g->gh = 0;
        return;
    }
    float scale = sqrtf(1.f * (float)acc->max_hits / 48.0f);
    float ext = maxr(bbmax[0] - bbmin[0], bbmax[1] - bbmin[1]);
    if (scale * ext > 4096)
        scale = 4096 / ext;
    bbmin[0] *= scale; bbmin[1] *= scale;
    bbmax[0] *= scale; bbmax[1] *= scale;
    g->scale = scale;
    g->bmin_x = (int)floorf(bbmin[0]);
    g->bmin_y = (int)floorf(bbmin[1]);
    g->gw = ((int)floorf(bbmax[0]) + 1) - g->bmin_x;
    g->gh = ((int)floorf(bbmax[1]) + 1) - g->bmin_y;
}

// ---------------------------------------------------------------------------
// Bucketing (Reconstruction.cpp:605-626).
// ---------------------------------------------------------------------------
__global__ void k_bucket_count(const float4* __restrict__ rp_pos, const float4* __restrict__ rp_mot, size_t n,
                               const GridInfo* g, int* __restrict__ cell_of, int* __restrict__ count)
{
    const float scale = g->scale;
    const int bx = g->bmin_x, by = g->bmin_y, gw = g->gw, gh = g->gh;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    {
        int cell = -1;
        if (rp_mot[k].w != 0.0f)
        {
            float4 p = rp_pos[k];
            int sx = (int)floorf(scale * p.x) - bx;
            int sy = (int)floorf(scale * p.y) - by;
            if (!(sx < 0 || sy < 0 || sx >= gw || sy >= gh))
            {
                cell = sy * gw + sx;
                atomicAdd(&count[cell], 1);
            }
        }
        cell_of[k] = cell;
    }
}

__global__ void k_bucket_scatter(const int* __restrict__ cell_of, size_t n, int* __restrict__ cursor,
                                 int* __restrict__ items)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    {
        int c = cell_of[k];
        if (c >= 0)
            items[atomicAdd(&cursor[c], 1)] = (int)k;
    }
}

// restore input order inside each cell
__global__ void k_cell_sort(const int* __restrict__ start, int ncell, int* __restrict__ items)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x)
    {
        int b = start[c], e = start[c + 1];
        for (int i = b + 1; i < e; i++)
        {
            int v = items[i];
            int j = i - 1;
            while (j >= b && items[j] > v) { items[j + 1] = items[j]; j--; }
            items[j + 1] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Exclusive scan of int counts (n+1 outputs; out[n] = total).
// ---------------------------------------------------------------------------
constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ int block_exclusive_scan(int v, int* smem, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem[wid] = x;
    __syncthreads();
    if (wid == 0)
    {
        int s = (lane < (int)(blockDim.x >> 5)) ? smem[lane] : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        smem[lane] = s;
    }
    __syncthreads();
    int warp_off = wid ? smem[wid - 1] : 0;
    *total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_off + x - v;
}

__global__ void k_scan_tiles(const int* __restrict__ in, size_t n, int* __restrict__ out, int* __restrict__ tile_sums)
{
    __shared__ int smem[32];
    size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
    for (int i = 0; i < kScanItems; i++)
    {
        v[i] = (base + i < n) ? in[base + i] : 0;
        sum += v[i];
    }
    int total;
    int off = block_exclusive_scan(sum, smem, &total);
    for (int i = 0; i < kScanItems; i++)
    {
        if (base + i < n) out[base + i] = off;
        off += v[i];
    }
    if (threadIdx.x == 0)
        tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(int* sums, int ntiles, int* total_out)
{
    __shared__ int smem[32];
    int carry = 0;
    for (int b = 0; b < ntiles; b += blockDim.x)
    {
        int i = b + threadIdx.x;
        int v = (i < ntiles) ? sums[i] : 0;
        int total;
        int off = block_exclusive_scan(v, smem, &total);
        if (i < ntiles) sums[i] = carry + off;
        carry += total;
    }
    if (threadIdx.x == 0)
        *total_out = carry;
}

__global__ void k_scan_add(int* __restrict__ out, size_t n, const int* __restrict__ tile_off)
{
    size_t base = (size_t)blockIdx.x * kScanTile;
    int add = tile_off[blockIdx.x];
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x)
        if (base + i < n) out[base + i] += add;
}

// ---------------------------------------------------------------------------
// kd split of the grid (ReconstructionTreeBuilder.cpp:34-96), level by level.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int rect_count(const int* start, int gw, int x0, int x1, int y0, int y1)
{
    int s = 0;
    for (int y = y0; y < y1; y++)
        s += start[y * gw + x1] - start[y * gw + x0];
    return s;
}

__global__ void k_kd_init(KdNode* kd, int* levels, GridInfo* g, int* counter)
{
    KdNode r;
    r.x0 = 0; r.y0 = 0; r.x1 = g->gw; r.y1 = g->gh;
    r.child0 = r.child1 = -1;
    r.num_samples = 0; r.depth = 0; r.path = 0; r.parent = -1;
    r.leaf_count = 0; r.preorder_leaf = 0; r.preorder_sample = 0; r.sample_offset = 0; r.frontier = 0; r.pad = 0;
    kd[0] = r;
    levels[0] = 0; levels[1] = 1;
    *counter = 1;
    g->kd_levels = 1;
}

// Nodes of level L occupy [levels[2L], levels[2L+1]); their children are
// allocated in pairs at the end of the node array, which becomes level L+1.
__global__ void k_kd_level(KdNode* kd, const int* levels_in, int L, const int* __restrict__ cell_start,
                           const GridInfo* g, int* counter)
{
    const int lo = levels_in[2 * L], hi = levels_in[2 * L + 1];
    const int gw = g->gw;
    for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    {
        KdNode nd = kd[i];
        const int dx = nd.x1 - nd.x0, dy = nd.y1 - nd.y0;
        bool leaf = maxi(dx, dy) == 1;
        if (!leaf && dx * dy <= 64)
            leaf = rect_count(cell_start, gw, nd.x0, nd.x1, nd.y0, nd.y1) <= 48;
        if (leaf)
        {
            kd[i].child0 = -1;
            kd[i].child1 = -1;
            kd[i].num_samples = rect_count(cell_start, gw, nd.x0, nd.x1, nd.y0, nd.y1);
            kd[i].leaf_count = 1;
            continue;
        }
        int c = atomicAdd(counter, 2);
        KdNode a = nd, b = nd;
        if (dx > dy)
        {
            int xmid = (nd.x1 + nd.x0) / 2;
            a.x1 = xmid; b.x0 = xmid;
        }
        else
        {
            int ymid = (nd.y1 + nd.y0) / 2;
            a.y1 = ymid; b.y0 = ymid;
        }
        a.depth = b.depth = nd.depth + 1;
        a.parent = b.parent = i;
        a.child0 = a.child1 = b.child0 = b.child1 = -1;
        a.path = nd.path;
        b.path = nd.path | ((nd.depth < 5) ? (1 << nd.depth) : 0);
        kd[c] = a;
        kd[c + 1] = b;
        kd[i].child0 = c;
        kd[i].child1 = c + 1;
    }
}

__global__ void k_kd_next(int* levels, int L, const int* counter, GridInfo* g)
{
    levels[2 * (L + 1)] = levels[2 * L + 1];
    levels[2 * (L + 1) + 1] = *counter;
    if (levels[2 * L + 1] != *counter)
        g->kd_levels = L + 2;
}

__global__ void k_kd_up(KdNode* kd, const int* levels, int L)
{
    const int lo = levels[2 * L], hi = levels[2 * L + 1];
    for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    {
        if (kd[i].child0 < 0)
            continue;
        const KdNode& a = kd[kd[i].child0];
        const KdNode& b = kd[kd[i].child1];
        kd[i].num_samples = a.num_samples + b.num_samples;
        kd[i].leaf_count = a.leaf_count + b.leaf_count;
    }
}

__global__ void k_kd_down(KdNode* kd, const int* levels, int L)
{
    const int lo = levels[2 * L], hi = levels[2 * L + 1];
    for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    {
        if (kd[i].child0 < 0)
            continue;
        KdNode& a = kd[kd[i].child0];
        KdNode& b = kd[kd[i].child1];
        a.preorder_leaf = kd[i].preorder_leaf;
        a.preorder_sample = kd[i].preorder_sample;
        b.preorder_leaf = kd[i].preorder_leaf + a.leaf_count;
        b.preorder_sample = kd[i].preorder_sample + a.num_samples;
    }
}

// Entry points of the 32 build tasks and their sample / leaf bases
// (Reconstruction.cpp:110-126, 132-143).
__global__ void k_entry_points(const KdNode* kd, GridInfo* g, int num_kd)
{
    int sb = 0, lb = 0;
    for (int i = 0; i < 32; i++)
    {
        int node = 0;
        for (int j = 0; j < 5; j++)
        {
            if (node == -1)
                continue;
            bool isLeaf = kd[node].child0 < 0;
            if (i & (1 << j)) node = (!isLeaf) ? kd[node].child1 : -1;
            else              node = (!isLeaf) ? kd[node].child0 : node;
        }
        g->entry[i] = node;
        g->task_sample_base[i] = sb;
        g->task_leaf_base[i] = lb;
        if (node != -1)
        {
            sb += kd[node].num_samples;
            lb += kd[node].leaf_count;
        }
    }
    g->task_leaf_base[32] = lb;
    g->num_kd = num_kd;
    g->num_kd_leaves = lb;
    g->num_accepted = sb;
}

// Final sample offsets and build-task order of the kd leaves.  A node at depth
// >= 5, or a leaf at depth < 5, belongs to the task given by its first five
// child choices (its path bits).
__global__ void k_kd_assign(KdNode* kd, int num_kd, const GridInfo* g, int* leaves_ordered)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < num_kd; i += gridDim.x * blockDim.x)
    {
        KdNode& nd = kd[i];
        bool in_task = nd.depth >= 5 || nd.child0 < 0;
        if (!in_task)
        {
            nd.sample_offset = -1;
            continue;
        }
        int t = nd.path;
        int e = g->entry[t];
        if (e < 0)
        {   // cannot happen: a node under the depth-5 frontier always has an entry
            nd.sample_offset = -1;
            continue;
        }
        const KdNode& en = kd[e];
        nd.sample_offset = g->task_sample_base[t] + (nd.preorder_sample - en.preorder_sample);
        if (nd.child0 < 0)
        {
            int rank = g->task_leaf_base[t] + (nd.preorder_leaf - en.preorder_leaf);
            leaves_ordered[rank] = i;
        }
    }
}

// ---------------------------------------------------------------------------
// Leaf construction, part 1: candidates, sort, bounds and boxes
// (ReconstructionTreeBuilder.cpp:131-213).
// ---------------------------------------------------------------------------
struct TWSortAccessor
{
    int* perm;
    const float4* pos;
    __device__ int cmp(int a, int b) const
    {
        float4 sa = pos[perm[a]], sb = pos[perm[b]];
        if (sa.w < sb.w) return -1;             // t
        else if (sa.w > sb.w) return 1;
        else
        {
            if (sa.z < sb.z) return -1;         // w
            else if (sa.z > sb.z) return 1;
            else return 0;
        }
    }
    __device__ void swap(int a, int b) { int t = perm[a]; perm[a] = perm[b]; perm[b] = t; }
};

__global__ void k_leaf_prepare(const int* __restrict__ leaves_ordered, int num_leaves, const KdNode* __restrict__ kd,
                               const int* __restrict__ cell_start, const int* __restrict__ cell_items, const GridInfo* g,
                               const float4* __restrict__ rp_pos, const float4* __restrict__ rp_mot,
                               const float4* __restrict__ rec, float W, float H, float c0, float c1,
                               int* __restrict__ perm, float* __restrict__ box, Bounds* __restrict__ sbounds,
                               float4* __restrict__ s_rec, float4* __restrict__ s_col,
                               int* __restrict__ s_id, int* __restrict__ ordered_n, int* invalid_count)
{
    const int gw = g->gw;
    int invalid = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < num_leaves; r += gridDim.x * blockDim.x)
    {
        const KdNode nd = kd[leaves_ordered[r]];
        const int n = nd.num_samples;
        ordered_n[r] = n;
        if (n == 0)
            continue;
        const int off = nd.sample_offset;
        int k = 0;
        for (int y = nd.y0; y < nd.y1; y++)
            for (int x = nd.x0; x < nd.x1; x++)
            {
                int c = y * gw + x;
                for (int q = cell_start[c]; q < cell_start[c + 1]; q++)
                    perm[off + k++] = cell_items[q];
            }
        TWSortAccessor acc{ perm + off, rp_pos };
        fw_sort(acc, 0, n);
        for (int j = 0; j < n; j++)
        {
            const int id = perm[off + j];
            const float4 p = rp_pos[id];
            const float4 m = rp_mot[id];
            const float sx = p.x, sy = p.y, sw = p.z, st = p.w;
            const float mv[3] = { m.x, m.y, m.z };
            float xywt0[3] = { sx * sw - mv[0] * st, sy * sw - mv[1] * st, sw - mv[2] * st };
            Bounds b;
            tux_planes(xywt0, mv, W, H, c0, c1, b);
            sbounds[off + j] = b;
            float* bx = box + (size_t)(off + j) * 8;
            if (bounds_valid(b))
            {
                float ta = b.tspan[0], tb = b.tspan[1];
                float base[3] = { sx * sw, sy * sw, sw };
                float xa[3], xb[3];
                for (int q = 0; q < 3; q++)
                {
                    xa[q] = base[q] + mv[q] * (ta - st);
                    xb[q] = base[q] + mv[q] * (tb - st);
                }
                float ca = rcp(xa[2]), cb = rcp(xb[2]);
                float xyta[2] = { xa[0] * ca, xa[1] * ca };
                float xytb[2] = { xb[0] * cb, xb[1] * cb };
                float oodt = 1.0f / (tb - ta);
                float dxdt = (xytb[0] - xyta[0]) * oodt;
                float dydt = (xytb[1] - xyta[1]) * oodt;
                float xyt0[2] = { xyta[0] - dxdt * ta, xyta[1] - dydt * ta };
                float xyt1[2] = { xytb[0] + dxdt * (1.0f - tb), xytb[1] + dydt * (1.0f - tb) };
                float cocta = c0 / xa[2] + c1;
                float coctb = c0 / xb[2] + c1;
                bx[0] = xyt0[0] + cocta; bx[1] = xyt0[1] + cocta;
                bx[2] = xyt0[0] - cocta; bx[3] = xyt0[1] - cocta;
                bx[4] = xyt1[0] + coctb; bx[5] = xyt1[1] + coctb;
                bx[6] = xyt1[0] - coctb; bx[7] = xyt1[1] - coctb;
            }
            else
                invalid++;
            // tree-ordered sample record (Reconstruction.hpp:73-86 Sample, color alpha 1)
            float4 r1 = __ldg(&rec[(size_t)id * 4 + 1]);
            float4 r2 = __ldg(&rec[(size_t)id * 4 + 2]);
            s_rec[2 * (off + j)] = p;
            s_rec[2 * (off + j) + 1] = make_float4(mv[0], mv[1], mv[2], c0 / sw + c1);
            s_col[off + j] = make_float4(r1.w, r2.x, r2.y, 1.0f);
            s_id[off + j] = id;
        }
    }
    if (invalid)
        atomicAdd(invalid_count, invalid);
}

// Per build task: exclusive running maximum of the candidate counts and the
// count of the previous non-empty leaf, over the task's leaves in build order.
__global__ void k_task_prefix(const GridInfo* g, const int* __restrict__ ordered_n, int* __restrict__ prefmax,
                              int* __restrict__ prevn)
{
    const int t = blockIdx.x;
    const int b = g->task_leaf_base[t], e = g->task_leaf_base[t + 1];
    __shared__ int s_max[1024], s_last[1024];
    const int tid = threadIdx.x, B = blockDim.x;
    int carry_max = 0, carry_last = 0;
    for (int base = b; base < e; base += B)
    {
        const int i = base + tid;
        const int v = (i < e) ? ordered_n[i] : 0;
        s_max[tid] = v;
        s_last[tid] = v;
        __syncthreads();
        for (int o = 1; o < B; o <<= 1)
        {
            int m = s_max[tid], l = s_last[tid];
            if (tid >= o)
            {
                m = maxi(m, s_max[tid - o]);
                if (l == 0) l = s_last[tid - o];
            }
            __syncthreads();
            s_max[tid] = m;
            s_last[tid] = l;
            __syncthreads();
        }
        int ex_max = maxi(carry_max, (tid > 0) ? s_max[tid - 1] : 0);
        int ex_last = (tid > 0) ? s_last[tid - 1] : 0;
        if (ex_last == 0) ex_last = carry_last;
        if (i < e)
        {
            prefmax[i] = ex_max;
            prevn[i] = ex_last;
        }
        carry_max = maxi(carry_max, s_max[B - 1]);
        if (s_last[B - 1] != 0) carry_last = s_last[B - 1];
        __syncthreads();
    }
}

// Array::reallocRound for Vec2f (Array.hpp:686-692): MinBytes 256 -> 32 elements, doubling.
__device__ __forceinline__ int alloc_round(int m)
{
    if (m == 0) return 0;
    int r = 32;
    while (m > r) r <<= 1;
    return r;
}

// Candidates with invalid bounds take the boxes the reused per-task arrays hold
// at their index: the value written there by the most recent earlier leaf of the
// task, unless a reallocation in between cleared it (elements at or beyond the
// previous size are zero after Array::realloc).
__global__ void k_stale_boxes(const int* __restrict__ leaves_ordered, const GridInfo* g, const KdNode* __restrict__ kd,
                              const int* __restrict__ ordered_n, const int* __restrict__ prefmax,
                              const int* __restrict__ prevn, const Bounds* __restrict__ sbounds,
                              float* __restrict__ box, int num_leaves, int task_of_first)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < num_leaves; r += gridDim.x * blockDim.x)
    {
        const int n = ordered_n[r];
        if (n == 0)
            continue;
        const KdNode nd = kd[leaves_ordered[r]];
        const int off = nd.sample_offset;
        // task of this ordered rank
        int t = 0;
        while (t < 31 && g->task_leaf_base[t + 1] <= r) t++;
        const int tb = g->task_leaf_base[t];
        for (int i = 0; i < n; i++)
        {
            if (bounds_valid(sbounds[off + i]))
                continue;
            float v[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
            // state after this leaf's resize
            bool realloc_here = n > alloc_round(prefmax[r]);
            if (!(realloc_here && i >= prevn[r]))
            {
                for (int k = r - 1; k >= tb; k--)
                {
                    const int nk = ordered_n[k];
                    if (nk == 0)
                        continue;
                    const int offk = kd[leaves_ordered[k]].sample_offset;
                    if (nk > i && bounds_valid(sbounds[offk + i]))
                    {
                        for (int q = 0; q < 8; q++) v[q] = box[(size_t)(offk + i) * 8 + q];
                        break;
                    }
                    if (nk > alloc_round(prefmax[k]) && i >= prevn[k])
                        break;      // cleared by the reallocation at leaf k
                }
            }
            for (int q = 0; q < 8; q++) box[(size_t)(off + i) * 8 + q] = v[q];
        }
    }
    (void)task_of_first;
}

__device__ __forceinline__ void bnode_from_bounds(BNode& n, const Bounds& b)
{
    for (int p = 0; p < 4; p++)
        for (int k = 0; k < 3; k++)
            n.p[p * 3 + k] = b.p[p][k];
    n.tspan[0] = b.tspan[0];
    n.tspan[1] = b.tspan[1];
}
__device__ __forceinline__ void bounds_from_bnode(Bounds& b, const BNode& n)
{
    for (int p = 0; p < 4; p++)
        for (int k = 0; k < 3; k++)
            b.p[p][k] = n.p[p * 3 + k];
    b.tspan[0] = n.tspan[0];
    b.tspan[1] = n.tspan[1];
}

// Leaf construction, part 2: surface scan and leaf nodes (RTB.cpp:222-378).
__global__ void k_leaf_scan(const int* __restrict__ leaves_ordered, int num_leaves, KdNode* __restrict__ kd,
                            const float4* __restrict__ s_rec, const float* __restrict__ box,
                            const Bounds* __restrict__ sbounds, int* __restrict__ surface, BNode* __restrict__ pending)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < num_leaves; r += gridDim.x * blockDim.x)
    {
        const int kid = leaves_ordered[r];
        const KdNode nd = kd[kid];
        const int n = nd.num_samples;
        if (n == 0)
        {
            kd[kid].frontier = 0;
            continue;
        }
        const int off = nd.sample_offset;
        const float* B = box + (size_t)off * 8;
        int* surf = surface + off;
        int surfacebegin = 0, currsurface = 0;
        surf[0] = 0;
        bool reset = true;
        float cb0[2] = { 0, 0 }, cb1[2] = { 0, 0 }, mvmin[2] = { 0, 0 }, mvmax[2] = { 0, 0 };
        float surfacet = 0.0f;
        const float TH = 1 * 2.0f;
        for (int cur = 1; cur < n; ++cur)
        {
            if (reset)
            {
                const float* bb = B + surfacebegin * 8;
                cb0[0] = cb0[1] = 0.5f * (bb[0] - bb[2]);
                cb1[0] = cb1[1] = 0.5f * (bb[4] - bb[6]);
                for (int q = 0; q < 2; q++)
                    mvmin[q] = 0.5f * (bb[4 + q] + bb[6 + q]) - 0.5f * (bb[q] + bb[2 + q]);
                mvmax[0] = mvmin[0]; mvmax[1] = mvmin[1];
                surfacet = s_rec[2 * (off + surfacebegin)].w;
                reset = false;
            }
            bool conflict = false, early = false;
            if (surfacet != s_rec[2 * (off + cur)].w)
            {
                surfacebegin = cur;
                surf[cur] = ++currsurface;
                reset = true;
                continue;
            }
            const float* bc = B + cur * 8;
            float coct0 = 0.5f * (bc[0] - bc[2]);
            float coct1 = 0.5f * (bc[4] - bc[6]);
            float mv[2];
            for (int q = 0; q < 2; q++)
                mv[q] = 0.5f * (bc[4 + q] + bc[6 + q]) - 0.5f * (bc[q] + bc[2 + q]);
            float e0 = maxr(absf(coct0 - cb0[0]), absf(coct0 - cb0[1]));
            float e1 = maxr(absf(coct1 - cb1[0]), absf(coct1 - cb1[1]));
            float a0 = maxr(absf(mvmin[0] - mv[0]), absf(mvmin[1] - mv[1]));
            float a1 = maxr(absf(mvmax[0] - mv[0]), absf(mvmax[1] - mv[1]));
            if (e0 < 0.5f * TH && e1 < 0.5f * TH && maxr(a0, a1) < TH)
                early = true;
            if (!early)
            {
                for (int test = surfacebegin; test < cur; ++test)
                {
                    const float* bt = B + test * 8;
                    bool bX = ternary_equal4(ternary_compare(bt[0], bc[0], TH), ternary_compare(bt[2], bc[2], TH),
                                             ternary_compare(bt[4], bc[4], TH), ternary_compare(bt[6], bc[6], TH));
                    bool bY = ternary_equal4(ternary_compare(bt[1], bc[1], TH), ternary_compare(bt[3], bc[3], TH),
                                             ternary_compare(bt[5], bc[5], TH), ternary_compare(bt[7], bc[7], TH));
                    if (!(bX && bY))
                    {
                        surfacebegin = cur;
                        surf[cur] = ++currsurface;
                        conflict = true;
                        reset = true;
                        break;
                    }
                }
            }
            if (!conflict)
            {
                surf[cur] = currsurface;
                cb0[0] = minr(coct0, cb0[0]);
                cb0[1] = maxr(coct0, cb0[0]);
                cb1[0] = minr(coct1, cb1[0]);
                cb1[1] = maxr(coct1, cb1[0]);
                mvmin[0] = minr(mvmin[0], mv[0]); mvmin[1] = minr(mvmin[1], mv[1]);
                mvmax[0] = maxr(mvmax[0], mv[0]); mvmax[1] = maxr(mvmax[1], mv[1]);
            }
        }
        // leaf nodes, one per surface run (RTB.cpp:345-378)
        int nf = 0;
        for (int i = 0; i < n;)
        {
            int j;
            for (j = i + 1; j < n && surf[i] == surf[j]; ++j) {}
            Bounds tl;
            bounds_zero(tl);
            for (int q = i; q < j; ++q)
            {
                Bounds t;
                combine_bounds(sbounds[off + q], tl, t);
                tl = t;
            }
            BNode bn;
            bnode_from_bounds(bn, tl);
            bn.ref = ~(off + i);
            bn.ns = j - i;
            bn.height = 1;
            bn.pad = 0;
            pending[off + nf] = bn;
            nf++;
            i = j;
        }
        kd[kid].frontier = nf;
    }
}

// ---------------------------------------------------------------------------
// emitNodes (ReconstructionTreeBuilder.cpp:409-451) on a frontier stored in
// global memory.  Merged-away nodes are written to the final node array in
// pairs (child0, child1 = child0 + 1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void node_merge(const BNode& n0, const BNode& n1, BNode& out)
{
    Bounds a, b, r;
    bounds_from_bnode(a, n0);
    bounds_from_bnode(b, n1);
    combine_bounds(a, b, r);
    bnode_from_bounds(out, r);
    out.ns = n0.ns + n1.ns;
    out.ref = 0;
    out.height = 1 + maxi(n0.height, n1.height);
    out.pad = 0;
}

__device__ __forceinline__ float bnode_cost(const BNode& n)
{
    Bounds b;
    bounds_from_bnode(b, n);
    return bounds_cost(b, n.ns);
}

__device__ __forceinline__ QNode to_qnode(const BNode& n)
{
    QNode q;
    q.a = make_float4(n.p[0], n.p[1], n.p[2], n.p[3]);
    q.b = make_float4(n.p[4], n.p[5], n.p[6], n.p[7]);
    q.c = make_float4(n.p[8], n.p[9], n.p[10], n.p[11]);
    if (n.ref < 0)
    {
        int s0 = ~n.ref;
        q.d = make_int4(-1, -1, s0, s0 + n.ns);
    }
    else
        q.d = make_int4(n.ref, n.ref + 1, -1, -1);
    return q;
}

__device__ __forceinline__ void store_node(QNode* nodes, float2* tspans, int slot, const BNode& n)
{
    nodes[slot] = to_qnode(n);
    tspans[slot] = make_float2(n.tspan[0], n.tspan[1]);
}

__device__ int emit_nodes(bool is_root, BNode* f, int size, QNode* nodes, float2* tspans, int* node_counter)
{
    const int lim = is_root ? 1 : 4;
    // node costs of the frontier entries (recomputed per step as the reference does)
    while (size > lim)
    {
        float minCost = kF32Max;
        int mi = -1, mj = -1;
        for (int i = 0; i < size; i++)
        {
            const BNode n0 = f[i];
            const float c0 = bnode_cost(n0);
            for (int j = i + 1; j < size; j++)
            {
                const BNode n1 = f[j];
                BNode m;
                node_merge(n0, n1, m);
                float cost = bnode_cost(m) - (c0 + bnode_cost(n1));
                if (cost < minCost)
                {
                    minCost = cost;
                    mi = i; mj = j;
                }
            }
        }
        if (mi < 0) { mi = 0; mj = 1; }
        const BNode n0 = f[mi], n1 = f[mj];
        BNode m;
        node_merge(n0, n1, m);
        int slot = atomicAdd(node_counter, 2);
        store_node(nodes, tspans, slot, n0);
        store_node(nodes, tspans, slot + 1, n1);
        m.ref = slot;
        f[mi] = m;
        f[mj] = f[size - 1];
        size--;
    }
    return size;
}

__global__ void k_emit_level(KdNode* kd, const int* levels, int L, BNode* pending, QNode* nodes, float2* tspans,
                             int* node_counter)
{
    const int lo = levels[2 * L], hi = levels[2 * L + 1];
    for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x)
    {
        const KdNode nd = kd[i];
        if (nd.child0 < 0 || nd.depth < 5)
            continue;
        const KdNode a = kd[nd.child0], b = kd[nd.child1];
        const int off = nd.sample_offset;
        const int fa = a.frontier, fb = b.frontier;
        // child0's frontier is at [off, off+fa); bring child1's next to it
        BNode* f = pending + off;
        const BNode* src = pending + b.sample_offset;
        for (int q = 0; q < fb; q++)
            f[fa + q] = src[q];
        int size = emit_nodes(false, f, fa + fb, nodes, tspans, node_counter);
        kd[i].frontier = size;
    }
}

// Serial top of the tree (Reconstruction.cpp:192-203) and the root.
__global__ void k_top(KdNode* kd, GridInfo* g, BNode* pending, BNode* top, QNode* nodes, float2* tspans,
                      int* node_counter)
{
    int start[32], count[32];
    int used = 0;
    for (int i = 0; i < 32; i++)
    {
        start[i] = used;
        count[i] = 0;
        int e = g->entry[i];
        if (e < 0)
            continue;
        const KdNode nd = kd[e];
        int fs = nd.frontier;
        if (used + fs > kTopCap) { g->error = kErrTopCap; return; }
        for (int q = 0; q < fs; q++)
            top[used + q] = pending[nd.sample_offset + q];
        count[i] = fs;
        used += fs;
    }
    for (int j = 0; j < 5; j++)
    {
        int offset = 1 << j;
        for (int i = 0; i < 32; i += 2 * offset)
        {
            int na = count[i], nb = count[i + offset];
            if (used + na + nb > kTopCap) { g->error = kErrTopCap; return; }
            int s = used;
            for (int q = 0; q < na; q++) top[s + q] = top[start[i] + q];
            for (int q = 0; q < nb; q++) top[s + na + q] = top[start[i + offset] + q];
            used += na + nb;
            int size = emit_nodes(j == 4, top + s, na + nb, nodes, tspans, node_counter);
            start[i] = s;
            count[i] = size;
        }
    }
    if (count[0] == 1)
    {
        int slot = atomicAdd(node_counter, 1);
        store_node(nodes, tspans, slot, top[start[0]]);
        g->root = slot;
        g->height = top[start[0]].height;
    }
    else
    {
        g->root = -1;
        g->height = 0;
    }
    g->num_nodes = *node_counter;
}

int grid_for(const Ctx& c, size_t n, int block)
{
    size_t b = (n + block - 1) / block;
    const size_t cap = (size_t)c.num_sms * 16;
    if (b > cap) b = cap;
    return (int)(b ? b : 1);
}

} // namespace

const char* cuda_error_string(cudaError_t e) { return cudaGetErrorString(e); }

#define CK(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { c.error = std::string(#x) + ": " + cudaGetErrorString(_e); return (_e == cudaErrorMemoryAllocation) ? TLFR_OOM : TLFR_CUDA; } } while (0)

// Frees the hierarchy build's working storage of a built context (reprojected
// samples, grid buckets, kd split, per-sample scratch) and trims the node
// arrays, allocated for the worst case of two nodes per sample, to the nodes
// the build emitted.  The hierarchy and its samples stay; a later rebuild
// allocates the working storage again.
tlfr_status release_build_scratch(Ctx& c)
{
    void** scratch[] = { (void**)&c.rp_pos, (void**)&c.rp_mot, (void**)&c.rp_cell, (void**)&c.cell_count,
                         (void**)&c.cell_start, (void**)&c.cell_items, (void**)&c.kd, (void**)&c.kd_leaves_ordered,
                         (void**)&c.perm, (void**)&c.box, (void**)&c.sbounds, (void**)&c.surface, (void**)&c.pending,
                         (void**)&c.top, (void**)&c.ordered_n, (void**)&c.ordered_prefmax, (void**)&c.leaf_task_rank };
    CK(cudaStreamSynchronize(c.stream));
    for (void** p : scratch)
    {
        if (*p)
            cudaFree(*p);
        *p = nullptr;
    }
    c.cell_cap = 0;
    c.kd_cap = 0;
    c.leaf_cap = 0;
    if (c.nodes && c.num_nodes > 0 && (size_t)c.num_nodes < c.node_cap)
    {
        QNode* nodes = nullptr;
        float2* tspan = nullptr;
        CK(cudaMalloc(&nodes, sizeof(QNode) * c.num_nodes));
        CK(cudaMalloc(&tspan, sizeof(float2) * c.num_nodes));
        CK(cudaMemcpy(nodes, c.nodes, sizeof(QNode) * c.num_nodes, cudaMemcpyDeviceToDevice));
        CK(cudaMemcpy(tspan, c.node_tspan, sizeof(float2) * c.num_nodes, cudaMemcpyDeviceToDevice));
        cudaFree(c.nodes);
        cudaFree(c.node_tspan);
        c.nodes = nodes;
        c.node_tspan = tspan;
        c.node_cap = c.num_nodes;
    }
    // the per-sample arrays are reallocated with the node arrays at the next build
    c.samp_cap = 0;
    return TLFR_OK;
}

tlfr_status build_hierarchy(Ctx& c, const float* d_records)
{
    cudaStream_t s = c.stream;
    const size_t n = c.n_in;
    const float4* rec = reinterpret_cast<const float4*>(d_records);

    // --- per-input buffers (sized once per context) ---
    if (!c.rp_pos)
    {
        CK(cudaMalloc(&c.rp_pos, sizeof(float4) * n));
        CK(cudaMalloc(&c.rp_mot, sizeof(float4) * n));
        CK(cudaMalloc(&c.rp_cell, sizeof(int) * n));
    }
    if (!c.hits)
        CK(cudaMalloc(&c.hits, sizeof(int) * (size_t)c.W * c.H));
    if (!c.d_grid)
        CK(cudaMalloc(&c.d_grid, sizeof(GridInfo) + sizeof(GridAccum) + 64 * sizeof(int)));
    if (!c.kd_level)
        CK(cudaMalloc(&c.kd_level, sizeof(int) * 2 * (kMaxKdLevels + 2)));
    GridAccum* acc = reinterpret_cast<GridAccum*>(reinterpret_cast<char*>(c.d_grid) + sizeof(GridInfo));
    int* counters = reinterpret_cast<int*>(acc + 1);    // [0] kd counter, [1] node counter, [2] invalid, [3] scan total

    // --- reprojection, bounding box, hit histogram ---
    CK(cudaMemsetAsync(c.hits, 0, sizeof(int) * (size_t)c.W * c.H, s));
    GridAccum init{};
    init.bbmin[0] = init.bbmin[1] = 0xffffffffu;
    init.bbmax[0] = init.bbmax[1] = 0u;
    CK(cudaMemcpyAsync(acc, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(counters, 0, 64 * sizeof(int), s));
    TLFR_LAUNCH(c, k_reproject, grid_for(c, n, 256), 256, s, rec, n, c.W, c.H, c.coc0_raw[0], c.coc0_raw[1],
                                                 c.rp_pos, c.rp_mot, c.hits, acc);
    TLFR_LAUNCH(c, k_max_hits, grid_for(c, (size_t)c.W * c.H, 256), 256, s, c.hits, (size_t)c.W * c.H, acc);
    TLFR_LAUNCH(c, k_grid_setup, 1, 1, s, acc, c.d_grid);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&c.grid, c.d_grid, sizeof(GridInfo), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (c.grid.error == kErrEmpty)
    {
        c.error = "All samples were discarded in reprojection to (u,v,t)=0";
        return TLFR_EMPTY;
    }

    // --- bucketing ---
    const size_t ncell = (size_t)c.grid.gw * c.grid.gh;
    if (ncell + 1 > c.cell_cap)
    {
        if (c.cell_count) { cudaFree(c.cell_count); cudaFree(c.cell_start); }
        c.cell_count = c.cell_start = nullptr;
        c.cell_cap = 0;
        CK(cudaMalloc(&c.cell_count, sizeof(int) * (ncell + 1)));
        CK(cudaMalloc(&c.cell_start, sizeof(int) * (ncell + 1 + (ncell + kScanTile) / kScanTile + 1)));
        c.cell_cap = ncell + 1;
    }
    if (!c.cell_items)
        CK(cudaMalloc(&c.cell_items, sizeof(int) * n));
    CK(cudaMemsetAsync(c.cell_count, 0, sizeof(int) * (ncell + 1), s));
    TLFR_LAUNCH(c, k_bucket_count, grid_for(c, n, 256), 256, s, c.rp_pos, c.rp_mot, n, c.d_grid, c.rp_cell, c.cell_count);
    {
        const size_t m = ncell + 1;
        const int tiles = (int)((m + kScanTile - 1) / kScanTile);
        int* tile_sums = c.cell_start + m;
        TLFR_LAUNCH(c, k_scan_tiles, tiles, kScanBlock, s, c.cell_count, m, c.cell_start, tile_sums);
        TLFR_LAUNCH(c, k_scan_sums, 1, 1024, s, tile_sums, tiles, counters + 3);
        TLFR_LAUNCH(c, k_scan_add, tiles, kScanBlock, s, c.cell_start, m, tile_sums);
    }
    // scatter with a cursor copy of the starts (reuse cell_count as the cursor)
    CK(cudaMemcpyAsync(c.cell_count, c.cell_start, sizeof(int) * ncell, cudaMemcpyDeviceToDevice, s));
    TLFR_LAUNCH(c, k_bucket_scatter, grid_for(c, n, 256), 256, s, c.rp_cell, n, c.cell_count, c.cell_items);
    TLFR_LAUNCH(c, k_cell_sort, grid_for(c, ncell, 256), 256, s, c.cell_start, (int)ncell, c.cell_items);
    CK(cudaGetLastError());

    // --- kd split, level by level ---
    const size_t kd_max = 2 * ncell + 2;
    if (kd_max > c.kd_cap)
    {
        if (c.kd) { cudaFree(c.kd); cudaFree(c.kd_leaves_ordered); }
        c.kd = nullptr; c.kd_leaves_ordered = nullptr; c.kd_cap = 0;
        CK(cudaMalloc(&c.kd, sizeof(KdNode) * kd_max));
        CK(cudaMalloc(&c.kd_leaves_ordered, sizeof(int) * kd_max));
        c.kd_cap = kd_max;
    }
    TLFR_LAUNCH(c, k_kd_init, 1, 1, s, c.kd, c.kd_level, c.d_grid, counters + 0);
    for (int L = 0; L < kMaxKdLevels; L++)
    {
        TLFR_LAUNCH(c, k_kd_level, c.num_sms * 4, 256, s, c.kd, c.kd_level, L, c.cell_start, c.d_grid, counters + 0);
        TLFR_LAUNCH(c, k_kd_next, 1, 1, s, c.kd_level, L, counters + 0, c.d_grid);
    }
    for (int L = kMaxKdLevels - 1; L >= 0; L--)
        TLFR_LAUNCH(c, k_kd_up, c.num_sms * 4, 256, s, c.kd, c.kd_level, L);
    for (int L = 0; L < kMaxKdLevels; L++)
        TLFR_LAUNCH(c, k_kd_down, c.num_sms * 4, 256, s, c.kd, c.kd_level, L);
    CK(cudaGetLastError());
    int num_kd = 0;
    CK(cudaMemcpyAsync(&num_kd, counters + 0, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    {
        int last[2];
        CK(cudaMemcpy(last, c.kd_level + 2 * kMaxKdLevels, sizeof(int) * 2, cudaMemcpyDeviceToHost));
        if (last[1] != last[0])
        {
            c.error = "kd split deeper than supported";
            return TLFR_OVERFLOW;
        }
    }
    TLFR_LAUNCH(c, k_entry_points, 1, 1, s, c.kd, c.d_grid, num_kd);
    TLFR_LAUNCH(c, k_kd_assign, grid_for(c, num_kd, 256), 256, s, c.kd, num_kd, c.d_grid, c.kd_leaves_ordered);
    CK(cudaMemcpyAsync(&c.grid, c.d_grid, sizeof(GridInfo), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int num_leaves = c.grid.num_kd_leaves;
    const size_t nacc = (size_t)c.grid.num_accepted;
    if (nacc == 0)
    {
        c.error = "All samples were discarded in reprojection to (u,v,t)=0";
        return TLFR_EMPTY;
    }

    // --- per-sample scratch and final sample arrays ---
    if (nacc > c.samp_cap)
    {
        cudaFree(c.perm); cudaFree(c.box); cudaFree(c.sbounds); cudaFree(c.surface); cudaFree(c.pending);
        cudaFree(c.s_rec); cudaFree(c.s_col); cudaFree(c.s_id);
        cudaFree(c.top);
        cudaFree(c.nodes); cudaFree(c.node_tspan);
        c.samp_cap = 0;
        CK(cudaMalloc(&c.perm, sizeof(int) * nacc));
        CK(cudaMalloc(&c.box, sizeof(float) * 8 * nacc));
        CK(cudaMalloc(&c.sbounds, sizeof(Bounds) * nacc));
        CK(cudaMalloc(&c.surface, sizeof(int) * nacc));
        CK(cudaMalloc(&c.pending, sizeof(BNode) * nacc));
        CK(cudaMalloc(&c.s_rec, sizeof(float4) * 2 * nacc));
        CK(cudaMalloc(&c.s_col, sizeof(float4) * nacc));
        CK(cudaMalloc(&c.s_id, sizeof(int) * nacc));
        CK(cudaMalloc(&c.top, sizeof(BNode) * kTopCap));
        CK(cudaMalloc(&c.nodes, sizeof(QNode) * (2 * nacc + 2)));
        CK(cudaMalloc(&c.node_tspan, sizeof(float2) * (2 * nacc + 2)));
        c.node_cap = 2 * nacc + 2;
        c.samp_cap = nacc;
    }
    if ((size_t)num_leaves + 1 > c.leaf_cap)
    {
        cudaFree(c.ordered_n); cudaFree(c.ordered_prefmax); cudaFree(c.leaf_task_rank);
        c.leaf_cap = 0;
        CK(cudaMalloc(&c.ordered_n, sizeof(int) * (num_leaves + 1)));
        CK(cudaMalloc(&c.ordered_prefmax, sizeof(int) * (num_leaves + 1)));
        CK(cudaMalloc(&c.leaf_task_rank, sizeof(int) * (num_leaves + 1)));
        c.leaf_cap = num_leaves + 1;
    }

    // --- leaves ---
    TLFR_LAUNCH(c, k_leaf_prepare, grid_for(c, num_leaves, 128), 128, s, 
        c.kd_leaves_ordered, num_leaves, c.kd, c.cell_start, c.cell_items, c.d_grid, c.rp_pos, c.rp_mot, rec,
        (float)c.W, (float)c.H, c.coc[0], c.coc[1], c.perm, c.box, c.sbounds, c.s_rec, c.s_col, c.s_id,
        c.ordered_n, counters + 2);
    TLFR_LAUNCH(c, k_task_prefix, 32, 1024, s, c.d_grid, c.ordered_n, c.ordered_prefmax, c.leaf_task_rank);
    TLFR_LAUNCH(c, k_stale_boxes, grid_for(c, num_leaves, 128), 128, s, c.kd_leaves_ordered, c.d_grid, c.kd, c.ordered_n,
                                                            c.ordered_prefmax, c.leaf_task_rank, c.sbounds, c.box,
                                                            num_leaves, 0);
    TLFR_LAUNCH(c, k_leaf_scan, grid_for(c, num_leaves, 128), 128, s, c.kd_leaves_ordered, num_leaves, c.kd, c.s_rec, c.box,
                                                          c.sbounds, c.surface, c.pending);
    CK(cudaGetLastError());

    // --- emitNodes bottom-up, then the serial top ---
    for (int L = c.grid.kd_levels; L >= 5; L--)
        TLFR_LAUNCH(c, k_emit_level, c.num_sms * 4, 128, s, c.kd, c.kd_level, L, c.pending, c.nodes, c.node_tspan, counters + 1);
    TLFR_LAUNCH(c, k_top, 1, 1, s, c.kd, c.d_grid, c.pending, c.top, c.nodes, c.node_tspan, counters + 1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&c.grid, c.d_grid, sizeof(GridInfo), cudaMemcpyDeviceToHost, s));
    int inv = 0;
    CK(cudaMemcpyAsync(&inv, counters + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c.grid.num_invalid = inv;
    if (c.grid.error == kErrTopCap)
    {
        c.error = "top-of-tree frontier exceeds capacity";
        return TLFR_OVERFLOW;
    }
    if (c.grid.root < 0)
    {
        c.error = "hierarchy build did not produce a single root";
        return TLFR_CUDA;
    }
    c.num_samples = (int)nacc;
    c.num_nodes = c.grid.num_nodes;
    c.root = c.grid.root;
    c.height = c.grid.height;
    return TLFR_OK;
}

} // namespace tlfr
