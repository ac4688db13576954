// tlfr_route.cu — learned routing (no counterpart in the reference: it is the
// addition that sends easy pixels to a fast path).  The fast path is the plain
// 1R pass that keeps the first surface when a second one opens instead of
// refetching at 2R (light_scan_warp in tlfr_query.cu), so the expensive full
// path runs only where the network is not confident.
//
//   features   eight cheap per-pixel features: depth, depth range and CoC
//              radius in the pixel, depth ranges within 3x3 and 5x5 tiles of
//              8x8 pixels (about the defocus radius), how much nearer the
//              nearest surface in that window is, motion magnitude, and a
//              coarse pass: the plain 1R pass on four of the pixel's output
//              samples, of which the fraction that needs the full path.
//   labels     1 when the fast path is as good as the plain method at the
//              pixel: within a tolerance of the plain pixel on every channel,
//              or, given the scene's ground truth, with a squared error against
//              it at most a tolerance above the plain pixel's (the plain method
//              and the fast path are both run on the frame).
//   network    8-64-64-1 MLP, ReLU, sigmoid output, binary cross-entropy.
//              Forward, backward and inference run on the tensor cores
//              (mma.sync m16n8k16, BF16 operands, FP32 accumulation); the
//              activations stay in registers between layers (the accumulator
//              tiles of one layer are the A operand tiles of the next).  Adam
//              updates FP32 master weights, which are then packed to BF16.
#include "tlfr_internal.h"

#include <cuda_bf16.h>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace tlfr
{

namespace
{

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------

// Per pixel over its input records ((y*W+x)*spp + k, 16 floats each:
// x, y, z/w, w, u, v, t, rgba, mv (3), dw/dx, dw/dy):
//   a = (log w min, log w max, CoC min, CoC max), b = (mean log w, max |motion|, hits, 0)
__global__ void k_feat_pixel(const float* __restrict__ rec, const int* __restrict__ hits, long long npix, int spp,
                             float c0, float c1, float4* __restrict__ fa, float4* __restrict__ fb)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x)
    {
        float lmin = 1e30f, lmax = -1e30f, cmin = 1e30f, cmax = -1e30f, lsum = 0, mmax = 0;
        for (int k = 0; k < spp; k++)
        {
            const float* r = rec + ((size_t)p * spp + k) * 16;
            const float w = fmaxf(r[3], 1e-6f);
            const float lw = logf(w);
            const float coc = c0 / w + c1;
            const float mx = r[11] / w, my = r[12] / w;
            lmin = fminf(lmin, lw);
            lmax = fmaxf(lmax, lw);
            cmin = fminf(cmin, coc);
            cmax = fmaxf(cmax, coc);
            lsum += lw;
            mmax = fmaxf(mmax, sqrtf(mx * mx + my * my));
        }
        fa[p] = make_float4(lmin, lmax, cmin, cmax);
        fb[p] = make_float4(lsum / (float)spp, mmax, (float)hits[p], 0.0f);
    }
}

// Coarse pass: 8x8-pixel tiles of (log w min, log w max, max |CoC|).
constexpr int kTile = 8;
__global__ void k_feat_tile(const float4* __restrict__ fa, int W, int H, int TW, int TH, float4* __restrict__ tiles)
{
    const int ntile = TW * TH;
    for (int ti = blockIdx.x * blockDim.x + threadIdx.x; ti < ntile; ti += gridDim.x * blockDim.x)
    {
        const int tx = ti % TW, ty = ti / TW;
        float lmin = 1e30f, lmax = -1e30f, cmax = 0;
        for (int y = ty * kTile; y < min(H, ty * kTile + kTile); y++)
            for (int x = tx * kTile; x < min(W, tx * kTile + kTile); x++)
            {
                const float4 a = fa[(long long)y * W + x];
                lmin = fminf(lmin, a.x);
                lmax = fmaxf(lmax, a.y);
                cmax = fmaxf(cmax, fmaxf(fabsf(a.z), fabsf(a.w)));
            }
        tiles[ti] = make_float4(lmin, lmax, cmax, 0.0f);
    }
}

// The eight features of each pixel (row-major [npix][8]):
//   0 mean log w            1 log w range in the pixel     2 max |CoC| in the pixel
//   3 mean log w minus the smallest log w within 5x5 tiles (a nearer surface that may blur over)
//   4 log w range within 3x3 tiles   5 log w range within 5x5 tiles
//   6 fraction of the pixel's probed output samples that the plain 1R pass sends to the full path
//   7 largest screen motion in the pixel
__global__ void k_feat_final(const float4* __restrict__ fa, const float4* __restrict__ fb,
                             const float4* __restrict__ tiles, const int* __restrict__ probe, int W, int H, int TW,
                             int TH, float* __restrict__ feats)
{
    const long long npix = (long long)W * H;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x)
    {
        const int x = (int)(p % W), y = (int)(p / W);
        const int tx = x / kTile, ty = y / kTile;
        const float4 a = fa[p], b = fb[p];
        float l3min = 1e30f, l3max = -1e30f, l5min = 1e30f, l5max = -1e30f, c5 = 0;
        for (int dy = -2; dy <= 2; dy++)
            for (int dx = -2; dx <= 2; dx++)
            {
                const int xx = tx + dx, yy = ty + dy;
                if (xx < 0 || yy < 0 || xx >= TW || yy >= TH)
                    continue;
                const float4 t = tiles[yy * TW + xx];
                l5min = fminf(l5min, t.x);
                l5max = fmaxf(l5max, t.y);
                c5 = fmaxf(c5, t.z);
                if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1)
                {
                    l3min = fminf(l3min, t.x);
                    l3max = fmaxf(l3max, t.y);
                }
            }
        float* f = feats + p * kRouteFeatures;
        f[0] = b.x;
        f[1] = a.y - a.x;
        f[2] = fmaxf(fabsf(a.z), fabsf(a.w));
        f[3] = b.x - l5min;
        f[4] = l3max - l3min;
        f[5] = l5max - l5min;
        f[6] = (float)probe[p] * (1.0f / kRouteProbes);
        f[7] = b.y;
    }
}

// Label 1 where the fast path is as good as the plain method: without a
// reference image, where it reproduces the plain pixel within tol on every
// channel; with one (the scene's ground truth), where its squared RGB error
// against the reference exceeds the plain pixel's by at most tol.
__global__ void k_labels(const float4* __restrict__ plain, const float4* __restrict__ fast,
                         const float4* __restrict__ ref, long long npix, float tol, float* __restrict__ labels)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x)
    {
        const float4 a = plain[p], b = fast[p];
        bool ok;
        if (ref)
        {
            const float4 r = ref[p];
            const float ea = (a.x - r.x) * (a.x - r.x) + (a.y - r.y) * (a.y - r.y) + (a.z - r.z) * (a.z - r.z);
            const float eb = (b.x - r.x) * (b.x - r.x) + (b.y - r.y) * (b.y - r.y) + (b.z - r.z) * (b.z - r.z);
            ok = eb <= ea + tol;
        }
        else
        {
            const float d = fmaxf(fmaxf(fabsf(a.x - b.x), fabsf(a.y - b.y)), fmaxf(fabsf(a.z - b.z), fabsf(a.w - b.w)));
            ok = d <= tol;
        }
        labels[p] = ok ? 1.0f : 0.0f;
    }
}

__global__ void k_route_flags(const float* __restrict__ prob, long long npix, float hi, unsigned char* __restrict__ fast)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x)
        fast[p] = prob[p] > hi ? 1 : 0;
}

// ---------------------------------------------------------------------------
// network
// ---------------------------------------------------------------------------

constexpr int kF = kRouteFeatures;   // 8 inputs, padded to K = 16 for the first layer
constexpr int kK1 = 16;
constexpr int kH = 64;

// FP32 parameter block (row-major [out][in]); the trainable part is a prefix.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * kK1;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH;
constexpr int kNumTrain = kOffB3 + 1;
constexpr int kOffMean = kNumTrain;               // input standardisation (fixed)
constexpr int kOffInvStd = kOffMean + kF;
constexpr int kNumParams = kOffInvStd + kF;

// BF16 operand block: w1 [64][16], w2 [64][64], w2 transposed [64][64], w3 padded to [8][64]
constexpr int kHW1 = 0;
constexpr int kHW2 = kHW1 + kH * kK1;
constexpr int kHW2T = kHW2 + kH * kH;
constexpr int kHW3 = kHW2T + kH * kH;
constexpr int kNumHalf = kHW3 + 8 * kH;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    uint32_t u;
    memcpy(&u, &v, 4);
    return u;
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D += A * B, m16n8k16, BF16 operands, FP32 accumulators.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B operand (16 x 8, "col": element (k, n) at n * ld + k) from a row-major
// [n][k] BF16 matrix: rows n0 + g, columns k0 + 2t (+1) and k0 + 2t + 8 (+1).
__device__ __forceinline__ void load_b(const __nv_bfloat16* w, int ld, int n0, int k0, int g, int t, uint32_t& b0,
                                       uint32_t& b1)
{
    const __nv_bfloat16* r = w + (size_t)(n0 + g) * ld + k0 + 2 * t;
    b0 = *reinterpret_cast<const uint32_t*>(r);
    b1 = *reinterpret_cast<const uint32_t*>(r + 8);
}

// Accumulator tiles c[2kk], c[2kk+1] (16 x 8 each) as the A operand of k-tile kk.
__device__ __forceinline__ void acc_to_a(const float (&c0)[4], const float (&c1)[4], uint32_t (&a)[4])
{
    a[0] = pack_bf16(c0[0], c0[1]);
    a[1] = pack_bf16(c0[2], c0[3]);
    a[2] = pack_bf16(c1[0], c1[1]);
    a[3] = pack_bf16(c1[2], c1[3]);
}

// Forward pass of one 16-row tile.  Lane (g = lane/4, t = lane%4) holds rows
// g and g + 8.  Outputs: h1, h2 after ReLU, rounded to BF16 (the values the
// next layer multiplies), columns 8j + 2t (+1); logits y for rows g and g+8
// (valid on lanes with t == 0).
struct Tile
{
    float h1[8][4], h2[8][4];
    uint32_t x[4];
    float y0, y8;
};

__device__ __forceinline__ void tile_forward(const float* __restrict__ P, const __nv_bfloat16* __restrict__ Wh,
                                             const float* __restrict__ feats, const int* rows, int nrows, Tile& T)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float xv[2][2];
    for (int h = 0; h < 2; h++)
    {
        const int r = g + 8 * h;
        for (int q = 0; q < 2; q++)
        {
            const int col = 2 * t + q;
            float v = 0.0f;
            if (r < nrows)
                v = (feats[(size_t)rows[r] * kF + col] - P[kOffMean + col]) * P[kOffInvStd + col];
            xv[h][q] = v;
        }
    }
    T.x[0] = pack_bf16(xv[0][0], xv[0][1]);
    T.x[1] = pack_bf16(xv[1][0], xv[1][1]);
    T.x[2] = 0;
    T.x[3] = 0;
    // layer 1
    for (int j = 0; j < 8; j++)
    {
        float c[4] = { 0, 0, 0, 0 };
        uint32_t b0, b1;
        load_b(Wh + kHW1, kK1, 8 * j, 0, g, t, b0, b1);
        mma16816(c, T.x, b0, b1);
        for (int q = 0; q < 4; q++)
            T.h1[j][q] = bf16_round(fmaxf(c[q] + P[kOffB1 + 8 * j + 2 * t + (q & 1)], 0.0f));
    }
    // layer 2
    uint32_t a[4][4];
    for (int kk = 0; kk < 4; kk++)
        acc_to_a(T.h1[2 * kk], T.h1[2 * kk + 1], a[kk]);
    for (int j = 0; j < 8; j++)
    {
        float c[4] = { 0, 0, 0, 0 };
        for (int kk = 0; kk < 4; kk++)
        {
            uint32_t b0, b1;
            load_b(Wh + kHW2, kH, 8 * j, 16 * kk, g, t, b0, b1);
            mma16816(c, a[kk], b0, b1);
        }
        for (int q = 0; q < 4; q++)
            T.h2[j][q] = bf16_round(fmaxf(c[q] + P[kOffB2 + 8 * j + 2 * t + (q & 1)], 0.0f));
    }
    // layer 3 (one output column of an 8-wide tile)
    for (int kk = 0; kk < 4; kk++)
        acc_to_a(T.h2[2 * kk], T.h2[2 * kk + 1], a[kk]);
    float c[4] = { 0, 0, 0, 0 };
    for (int kk = 0; kk < 4; kk++)
    {
        uint32_t b0, b1;
        load_b(Wh + kHW3, kH, 0, 16 * kk, g, t, b0, b1);
        mma16816(c, a[kk], b0, b1);
    }
    T.y0 = c[0] + P[kOffB3];
    T.y8 = c[2] + P[kOffB3];
}

__device__ __forceinline__ float sigmoid(float y) { return 1.0f / (1.0f + expf(-y)); }

// Inference: probability that each pixel is a single surface.
__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ P, const __nv_bfloat16* __restrict__ Wh,
                                                    const float* __restrict__ feats, long long n, float* __restrict__ prob)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    int rows[16];
    for (long long tile = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile * 16 < n; tile += warps)
    {
        const long long r0 = tile * 16;
        const int nrows = (int)min(16LL, n - r0);
        for (int r = 0; r < 16; r++)
            rows[r] = (int)(r0 + (r < nrows ? r : 0));
        Tile T;
        tile_forward(P, Wh, feats, rows, nrows, T);
        if (t == 0)
        {
            if (g < nrows)
                prob[r0 + g] = sigmoid(T.y0);
            if (g + 8 < nrows)
                prob[r0 + g + 8] = sigmoid(T.y8);
        }
    }
}

// Row index of the k-th example of a training step's minibatch.
__device__ __forceinline__ int batch_row(unsigned seed, unsigned step, unsigned k, unsigned n)
{
    unsigned h = k * 0x9e3779b1u ^ (step * 0x85ebca6bu + seed);
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    return (int)(h % n);
}

// Sum over the 8 row groups (lanes with the same t) of a per-lane value.
__device__ __forceinline__ float sum_groups(float v)
{
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

constexpr int kTrainWarps = 4;

// Forward + backward of binary cross-entropy (mean over the batch) for a
// minibatch; gradients are added into grad (FP32, kNumTrain).  Rows are the
// minibatch rows: row k = batch_row(seed, step, k, n), or k itself when
// all_rows is set (the gradient over exactly rows 0..batch-1).
__global__ void __launch_bounds__(kTrainWarps * 32)
k_mlp_train(const float* __restrict__ P, const __nv_bfloat16* __restrict__ Wh, const float* __restrict__ feats,
            const float* __restrict__ labels, int n, int batch, unsigned seed, unsigned step, int all_rows,
            float* __restrict__ grad, float* __restrict__ loss_out)
{
    __shared__ float s_grad[kNumTrain];
    __shared__ __nv_bfloat16 s_h1[kTrainWarps][16][kH];
    __shared__ __nv_bfloat16 s_dh2[kTrainWarps][16][kH];
    __shared__ __nv_bfloat16 s_dh1[kTrainWarps][16][kH];
    __shared__ __nv_bfloat16 s_x[kTrainWarps][16][kK1];
    __shared__ float s_loss;
    for (int i = threadIdx.x; i < kNumTrain; i += blockDim.x)
        s_grad[i] = 0.0f;
    if (threadIdx.x == 0)
        s_loss = 0.0f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const float inv_batch = 1.0f / (float)batch;
    float loss = 0.0f;
    int rows[16];
    for (int tile = blockIdx.x * kTrainWarps + warp; tile * 16 < batch; tile += gridDim.x * kTrainWarps)
    {
        const int k0 = tile * 16;
        const int nrows = min(16, batch - k0);
        for (int r = 0; r < 16; r++)
        {
            const int k = k0 + (r < nrows ? r : 0);
            rows[r] = all_rows ? k : batch_row(seed, step, (unsigned)k, (unsigned)n);
        }
        Tile T;
        tile_forward(P, Wh, feats, rows, nrows, T);
        // dL/dy = (p - label) / batch for rows g and g + 8, broadcast to the lane group
        float dy0 = 0.0f, dy8 = 0.0f;
        if (t == 0)
        {
            if (g < nrows)
            {
                const float p = sigmoid(T.y0), lab = labels[rows[g]];
                dy0 = (p - lab) * inv_batch;
                loss -= (lab * logf(fmaxf(p, 1e-7f)) + (1 - lab) * logf(fmaxf(1 - p, 1e-7f))) * inv_batch;
            }
            if (g + 8 < nrows)
            {
                const float p = sigmoid(T.y8), lab = labels[rows[g + 8]];
                dy8 = (p - lab) * inv_batch;
                loss -= (lab * logf(fmaxf(p, 1e-7f)) + (1 - lab) * logf(fmaxf(1 - p, 1e-7f))) * inv_batch;
            }
        }
        dy0 = __shfl_sync(0xffffffffu, dy0, lane & ~3);
        dy8 = __shfl_sync(0xffffffffu, dy8, lane & ~3);
        // layer 3: grad w3, b3; dh2 = dy * w3 * relu'(h2)
        float dh2[8][4];
        for (int j = 0; j < 8; j++)
            for (int q = 0; q < 2; q++)
            {
                const int col = 8 * j + 2 * t + q;
                const float w3 = bf16_round(P[kOffW3 + col]);
                const float gw = sum_groups(dy0 * T.h2[j][q] + dy8 * T.h2[j][q + 2]);
                if (g == 0)
                    atomicAdd(&s_grad[kOffW3 + col], gw);
                dh2[j][q] = T.h2[j][q] > 0.0f ? bf16_round(dy0 * w3) : 0.0f;
                dh2[j][q + 2] = T.h2[j][q + 2] > 0.0f ? bf16_round(dy8 * w3) : 0.0f;
                const float gb = sum_groups(dh2[j][q] + dh2[j][q + 2]);
                if (g == 0)
                    atomicAdd(&s_grad[kOffB2 + col], gb);
            }
        {
            const float gb3 = sum_groups(t == 0 ? dy0 + dy8 : 0.0f);
            if (lane == 0)
                atomicAdd(&s_grad[kOffB3], gb3);
        }
        // dh1 = dh2 * W2 (row-major [n][k]; the B operand is W2 transposed) * relu'(h1)
        uint32_t a[4][4];
        for (int kk = 0; kk < 4; kk++)
            acc_to_a(dh2[2 * kk], dh2[2 * kk + 1], a[kk]);
        float dh1[8][4];
        for (int j = 0; j < 8; j++)
        {
            float c[4] = { 0, 0, 0, 0 };
            for (int kk = 0; kk < 4; kk++)
            {
                uint32_t b0, b1;
                load_b(Wh + kHW2T, kH, 8 * j, 16 * kk, g, t, b0, b1);
                mma16816(c, a[kk], b0, b1);
            }
            for (int q = 0; q < 4; q++)
                dh1[j][q] = T.h1[j][q] > 0.0f ? bf16_round(c[q]) : 0.0f;
            for (int q = 0; q < 2; q++)
            {
                const float gb = sum_groups(dh1[j][q] + dh1[j][q + 2]);
                if (g == 0)
                    atomicAdd(&s_grad[kOffB1 + 8 * j + 2 * t + q], gb);
            }
        }
        // stage h1, dh2, dh1, x (row-major [row][col]) for the weight gradients,
        // which contract over the rows
        for (int j = 0; j < 8; j++)
            for (int q = 0; q < 4; q++)
            {
                const int r = g + 8 * (q >> 1), col = 8 * j + 2 * t + (q & 1);
                s_h1[warp][r][col] = __float2bfloat16_rn(T.h1[j][q]);
                s_dh2[warp][r][col] = __float2bfloat16_rn(dh2[j][q]);
                s_dh1[warp][r][col] = __float2bfloat16_rn(dh1[j][q]);
            }
        {
            const __nv_bfloat162* xs = reinterpret_cast<const __nv_bfloat162*>(T.x);
            for (int q = 0; q < 2; q++)
            {
                s_x[warp][g + 8 * q][2 * t] = xs[q].x;
                s_x[warp][g + 8 * q][2 * t + 1] = xs[q].y;
                s_x[warp][g + 8 * q][2 * t + 8] = __float2bfloat16_rn(0.0f);
                s_x[warp][g + 8 * q][2 * t + 9] = __float2bfloat16_rn(0.0f);
            }
        }
        __syncwarp();
        // grad W2[n][k] = sum_rows dh2[row][n] * h1[row][k]; grad W1[n][k] = sum_rows dh1[row][n] * x[row][k].
        // A = (dh)^T tile [n][row] (16 x 16), B = (h1 or x) as (k = row, n = col).
        auto at = [&](__nv_bfloat16 (*m)[kH], int r, int c) {
            uint32_t lo = reinterpret_cast<const uint16_t&>(m[r][c]);
            return lo;
        };
        for (int mt = 0; mt < 4; mt++)
        {
            uint32_t A2[4], A1[4];
            for (int q = 0; q < 4; q++)
            {
                const int nn = 16 * mt + g + 8 * (q & 1);
                const int rr = 2 * t + 8 * (q >> 1);
                A2[q] = at(s_dh2[warp], rr, nn) | (at(s_dh2[warp], rr + 1, nn) << 16);
                A1[q] = at(s_dh1[warp], rr, nn) | (at(s_dh1[warp], rr + 1, nn) << 16);
            }
            for (int j = 0; j < 8; j++)
            {
                const int kc = 8 * j + g;
                const uint32_t b0 = at(s_h1[warp], 2 * t, kc) | (at(s_h1[warp], 2 * t + 1, kc) << 16);
                const uint32_t b1 = at(s_h1[warp], 2 * t + 8, kc) | (at(s_h1[warp], 2 * t + 9, kc) << 16);
                float c[4] = { 0, 0, 0, 0 };
                mma16816(c, A2, b0, b1);
                for (int q = 0; q < 4; q++)
                {
                    const int nn = 16 * mt + g + 8 * (q >> 1), kcol = 8 * j + 2 * t + (q & 1);
                    atomicAdd(&s_grad[kOffW2 + nn * kH + kcol], c[q]);
                }
            }
            {
                const int kc = g;   // x columns 0..7
                const uint32_t b0 = reinterpret_cast<const uint16_t&>(s_x[warp][2 * t][kc]) |
                                    ((uint32_t)reinterpret_cast<const uint16_t&>(s_x[warp][2 * t + 1][kc]) << 16);
                const uint32_t b1 = reinterpret_cast<const uint16_t&>(s_x[warp][2 * t + 8][kc]) |
                                    ((uint32_t)reinterpret_cast<const uint16_t&>(s_x[warp][2 * t + 9][kc]) << 16);
                float c[4] = { 0, 0, 0, 0 };
                mma16816(c, A1, b0, b1);
                for (int q = 0; q < 4; q++)
                {
                    const int nn = 16 * mt + g + 8 * (q >> 1), kcol = 2 * t + (q & 1);
                    atomicAdd(&s_grad[kOffW1 + nn * kK1 + kcol], c[q]);
                }
            }
        }
        __syncwarp();
    }
    loss = sum_groups(loss);
    loss += __shfl_xor_sync(0xffffffffu, loss, 1);
    loss += __shfl_xor_sync(0xffffffffu, loss, 2);
    if (lane == 0)
        atomicAdd(&s_loss, loss);
    __syncthreads();
    for (int i = threadIdx.x; i < kNumTrain; i += blockDim.x)
        if (s_grad[i] != 0.0f)
            atomicAdd(&grad[i], s_grad[i]);
    if (threadIdx.x == 0 && loss_out)
        atomicAdd(loss_out, s_loss);
}

// Adam on the FP32 master weights; clears the gradient for the next step.
__global__ void k_adam(float* __restrict__ P, float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                       float lr, float b1, float b2, float eps, float bc1, float bc2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNumTrain; i += gridDim.x * blockDim.x)
    {
        const float gi = grad[i];
        const float mi = b1 * m[i] + (1 - b1) * gi;
        const float vi = b2 * v[i] + (1 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        grad[i] = 0.0f;
    }
}

// BF16 operand block from the FP32 master weights.
__global__ void k_pack(const float* __restrict__ P, __nv_bfloat16* __restrict__ Wh)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNumHalf; i += gridDim.x * blockDim.x)
    {
        float v;
        if (i < kHW2)
            v = P[kOffW1 + i];
        else if (i < kHW2T)
            v = P[kOffW2 + (i - kHW2)];
        else if (i < kHW3)
        {
            const int e = i - kHW2T, r = e / kH, c = e % kH;   // W2T[r][c] = W2[c][r]
            v = P[kOffW2 + c * kH + r];
        }
        else
        {
            const int e = i - kHW3, r = e / kH, c = e % kH;
            v = r == 0 ? P[kOffW3 + c] : 0.0f;
        }
        Wh[i] = __float2bfloat16_rn(v);
    }
}

} // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

#define CKR(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { err = std::string(#x) + ": " + cudaGetErrorString(_e); return (_e == cudaErrorMemoryAllocation) ? TLFR_OOM : TLFR_CUDA; } } while (0)

int route_num_params() { return kNumParams; }
int route_num_trainable() { return kNumTrain; }

tlfr_status route_alloc(Route& r, std::string& err)
{
    CKR(cudaDeviceGetAttribute(&r.num_sms, cudaDevAttrMultiProcessorCount, r.device));
    CKR(cudaMalloc(&r.params, sizeof(float) * kNumParams));
    CKR(cudaMalloc(&r.grad, sizeof(float) * kNumTrain));
    CKR(cudaMalloc(&r.m, sizeof(float) * kNumTrain));
    CKR(cudaMalloc(&r.v, sizeof(float) * kNumTrain));
    CKR(cudaMalloc(&r.half, sizeof(__nv_bfloat16) * kNumHalf));
    CKR(cudaMalloc(&r.loss, sizeof(float)));
    CKR(cudaMemset(r.grad, 0, sizeof(float) * kNumTrain));
    CKR(cudaMemset(r.m, 0, sizeof(float) * kNumTrain));
    CKR(cudaMemset(r.v, 0, sizeof(float) * kNumTrain));
    return TLFR_OK;
}

void route_free(Route& r)
{
    void* p[] = { r.params, r.grad, r.m, r.v, r.half, r.loss };
    for (void* q : p)
        if (q) cudaFree(q);
    r = Route{};
}

// He-style initialisation from a fixed seed; standardisation from the caller.
tlfr_status route_init(Route& r, unsigned seed, const float* mean, const float* inv_std, cudaStream_t s, std::string& err)
{
    std::vector<float> h(kNumParams, 0.0f);
    uint32_t st = seed * 747796405u + 2891336453u;
    auto rnd = [&]() {   // uniform in [-1, 1)
        st = st * 747796405u + 2891336453u;
        uint32_t w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
        w = (w >> 22u) ^ w;
        return (float)w / 2147483648.0f - 1.0f;
    };
    const float s1 = sqrtf(6.0f / kF), s2 = sqrtf(6.0f / kH), s3 = sqrtf(3.0f / kH);
    for (int n = 0; n < kH; n++)
        for (int k = 0; k < kF; k++)
            h[kOffW1 + n * kK1 + k] = s1 * rnd();
    for (int i = 0; i < kH * kH; i++)
        h[kOffW2 + i] = s2 * rnd();
    for (int i = 0; i < kH; i++)
        h[kOffW3 + i] = s3 * rnd();
    for (int k = 0; k < kF; k++)
    {
        h[kOffMean + k] = mean ? mean[k] : 0.0f;
        h[kOffInvStd + k] = inv_std ? inv_std[k] : 1.0f;
    }
    r.step = 0;
    CKR(cudaMemcpyAsync(r.params, h.data(), sizeof(float) * kNumParams, cudaMemcpyHostToDevice, s));
    CKR(cudaMemsetAsync(r.m, 0, sizeof(float) * kNumTrain, s));
    CKR(cudaMemsetAsync(r.v, 0, sizeof(float) * kNumTrain, s));
    CKR(cudaMemsetAsync(r.grad, 0, sizeof(float) * kNumTrain, s));
    k_pack<<<(kNumHalf + 255) / 256, 256, 0, s>>>(r.params, r.half);
    CKR(cudaStreamSynchronize(s));
    return TLFR_OK;
}

tlfr_status route_set_params(Route& r, const float* host_params, cudaStream_t s, std::string& err)
{
    CKR(cudaMemcpyAsync(r.params, host_params, sizeof(float) * kNumParams, cudaMemcpyHostToDevice, s));
    k_pack<<<(kNumHalf + 255) / 256, 256, 0, s>>>(r.params, r.half);
    CKR(cudaStreamSynchronize(s));
    return TLFR_OK;
}

tlfr_status route_get_params(Route& r, float* host_params, cudaStream_t s, std::string& err)
{
    CKR(cudaMemcpyAsync(host_params, r.params, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost, s));
    CKR(cudaStreamSynchronize(s));
    return TLFR_OK;
}

static int train_blocks(const Route& r, int batch)
{
    return std::max(1, std::min(r.num_sms * 4, (batch + 16 * kTrainWarps - 1) / (16 * kTrainWarps)));
}

tlfr_status route_gradient(Route& r, const float* d_feats, const float* d_labels, int n, float* host_grad,
                           float* host_loss, cudaStream_t s, std::string& err)
{
    CKR(cudaMemsetAsync(r.grad, 0, sizeof(float) * kNumTrain, s));
    CKR(cudaMemsetAsync(r.loss, 0, sizeof(float), s));
    k_mlp_train<<<train_blocks(r, n), kTrainWarps * 32, 0, s>>>(r.params, r.half, d_feats, d_labels, n, n, 0, 0, 1,
                                                             r.grad, r.loss);
    CKR(cudaGetLastError());
    CKR(cudaMemcpyAsync(host_grad, r.grad, sizeof(float) * kNumTrain, cudaMemcpyDeviceToHost, s));
    if (host_loss)
        CKR(cudaMemcpyAsync(host_loss, r.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    CKR(cudaStreamSynchronize(s));
    CKR(cudaMemsetAsync(r.grad, 0, sizeof(float) * kNumTrain, s));
    return TLFR_OK;
}

tlfr_status route_train(Route& r, const float* d_feats, const float* d_labels, int n, int steps, int batch, float lr,
                        unsigned seed, float* host_loss, cudaStream_t s, std::string& err)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    CKR(cudaMemsetAsync(r.loss, 0, sizeof(float), s));
    for (int k = 0; k < steps; k++)
    {
        r.step++;
        const bool last = k == steps - 1;
        if (last)
            CKR(cudaMemsetAsync(r.loss, 0, sizeof(float), s));
        k_mlp_train<<<train_blocks(r, batch), kTrainWarps * 32, 0, s>>>(r.params, r.half, d_feats, d_labels, n, batch,
                                                                     seed, (unsigned)r.step, 0, r.grad, r.loss);
        k_adam<<<(kNumTrain + 255) / 256, 256, 0, s>>>(r.params, r.grad, r.m, r.v, lr, b1, b2, eps,
                                                       1.0f - powf(b1, (float)r.step), 1.0f - powf(b2, (float)r.step));
        k_pack<<<(kNumHalf + 255) / 256, 256, 0, s>>>(r.params, r.half);
    }
    CKR(cudaGetLastError());
    if (host_loss)
        CKR(cudaMemcpyAsync(host_loss, r.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    CKR(cudaStreamSynchronize(s));
    return TLFR_OK;
}

tlfr_status route_predict(Route& r, const float* d_feats, long long n, float* d_prob, cudaStream_t s, std::string& err)
{
    const long long tiles = (n + 15) / 16;
    const int blocks = (int)std::max(1LL, std::min((long long)r.num_sms * 8, (tiles + 3) / 4));
    k_mlp_infer<<<blocks, 128, 0, s>>>(r.params, r.half, d_feats, n, d_prob);
    CKR(cudaGetLastError());
    return TLFR_OK;
}

tlfr_status route_features(Ctx& c, float* d_feats, std::string& err)
{
    const long long npix = (long long)c.W * c.H;
    const int TW = (c.W + kTile - 1) / kTile, TH = (c.H + kTile - 1) / kTile;
    if (!c.route_fa)
    {
        CKR(cudaMalloc(&c.route_fa, sizeof(float4) * (2 * npix + (size_t)TW * TH) + sizeof(int) * npix));
    }
    float4* fa = c.route_fa;
    float4* fb = c.route_fa + npix;
    float4* tiles = c.route_fa + 2 * npix;
    int* probe = reinterpret_cast<int*>(c.route_fa + 2 * npix + (size_t)TW * TH);
    const int blocks = (int)std::max(1LL, std::min((long long)c.num_sms * 16, (npix + 255) / 256));
    k_feat_pixel<<<blocks, 256, 0, c.stream>>>(c.cur_records, c.hits, npix, c.spp_in, c.coc[0], c.coc[1], fa, fb);
    k_feat_tile<<<(TW * TH + 127) / 128, 128, 0, c.stream>>>(fa, c.W, c.H, TW, TH, tiles);
    const tlfr_status ps = route_probe(c, probe);
    if (ps != TLFR_OK)
    {
        err = c.error;
        return ps;
    }
    k_feat_final<<<blocks, 256, 0, c.stream>>>(fa, fb, tiles, probe, c.W, c.H, TW, TH, d_feats);
    c.launches += 3;
    CKR(cudaGetLastError());
    return TLFR_OK;
}

tlfr_status route_labels_from(Ctx& c, const float4* d_plain, const float4* d_fast, const float4* d_ref, float tol,
                              float* d_labels, std::string& err)
{
    const long long npix = (long long)c.W * c.H;
    const int blocks = (int)std::max(1LL, std::min((long long)c.num_sms * 16, (npix + 255) / 256));
    k_labels<<<blocks, 256, 0, c.stream>>>(d_plain, d_fast, d_ref, npix, tol, d_labels);
    c.launches++;
    CKR(cudaGetLastError());
    return TLFR_OK;
}

tlfr_status route_flags(Ctx& c, const float* d_prob, float hi, unsigned char* d_fast, std::string& err)
{
    const long long npix = (long long)c.W * c.H;
    const int blocks = (int)std::max(1LL, std::min((long long)c.num_sms * 16, (npix + 255) / 256));
    k_route_flags<<<blocks, 256, 0, c.stream>>>(d_prob, npix, hi, d_fast);
    c.launches++;
    CKR(cudaGetLastError());
    return TLFR_OK;
}

} // namespace tlfr
