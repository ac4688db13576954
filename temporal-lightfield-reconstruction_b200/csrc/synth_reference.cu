// synth_reference.cu — reference images of the synthetic scenes: the exact
// lens/time/pixel integral of the analytic scene that the seeded sample
// buffers are drawn from, estimated per pixel by dense sampling on the GPU.
// It is the ground truth against which a reconstruction's error (PSNR) is
// measured; it plays no part in a reconstruction.
#include "synth_model.h"
#include "tlfr.h"

#include <cuda_runtime.h>

namespace tlfr_synth
{

namespace
{

// Per pixel: `samples` points, (u, v) stratified on the unit lens disk
// (stratified square mapped by radius sqrt(s) and angle 2*pi*s'), pixel
// position and time uniform, each from a counter-based hash.
__global__ void k_integrate(const Card* __restrict__ cards, const int* __restrict__ tile_start,
                            const int* __restrict__ tile_items, int tiles_x, int tile_size, float C0, float C1,
                            int W, int H, int samples, int gx, int gy, unsigned long long seed,
                            float4* __restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)W * H)
        return;
    const int x = (int)(p % W), y = (int)(p / W);
    const int tile = (y / tile_size) * tiles_x + (x / tile_size);
    const int* cand = tile_items + tile_start[tile];
    const int ncand = tile_start[tile + 1] - tile_start[tile];
    const uint64_t ph = hash3(seed, 20, (uint64_t)p);
    float r = 0, g = 0, b = 0;
    for (int k = 0; k < samples; k++)
    {
        const uint64_t sh = hash3(ph, 21, (uint64_t)k);
        const float s0 = ((float)(k % gx) + u01(hash3(sh, 22, 0))) / gx;
        const float s1 = ((float)((k / gx) % gy) + u01(hash3(sh, 22, 1))) / gy;
        const float rad = sqrtf(s0), ang = 6.2831853f * s1;
        const float u = rad * cosf(ang), v = rad * sinf(ang);
        const float xs = (float)x + u01(hash3(sh, 22, 2));
        const float ys = (float)y + u01(hash3(sh, 22, 3));
        const float t = u01(hash3(sh, 22, 4));
        float Wv, a, bb;
        int ci = shade(cards, cand, ncand, C0, C1, xs, ys, u, v, t, &Wv, &a, &bb);
        if (ci < 0)
        {
            ci = 0; a = 0; bb = 0;
        }
        const Card& c = cards[ci];
        r += value_noise(c, a, bb, 0);
        g += value_noise(c, a, bb, 1);
        b += value_noise(c, a, bb, 2);
    }
    const float inv = 1.0f / samples;
    out[p] = make_float4(r * inv, g * inv, b * inv, 1.0f);
}

} // namespace

int integrate_image(const Card* cards, int num_cards, const int* tile_start, const int* tile_items, int num_items,
                    int tiles_x, int tile_size, float C0, float C1, int width, int height, int samples,
                    unsigned long long seed, float* rgba)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return TLFR_NO_DEVICE;
    const long long npix = (long long)width * height;
    const int ntiles = tiles_x * ((height + tile_size - 1) / tile_size);
    Card* d_cards = nullptr;
    int *d_start = nullptr, *d_items = nullptr;
    float4* d_out = nullptr;
    int st = TLFR_OK;
    if (cudaMalloc(&d_cards, sizeof(Card) * num_cards) != cudaSuccess ||
        cudaMalloc(&d_start, sizeof(int) * (ntiles + 1)) != cudaSuccess ||
        cudaMalloc(&d_items, sizeof(int) * (num_items > 0 ? num_items : 1)) != cudaSuccess ||
        cudaMalloc(&d_out, sizeof(float4) * npix) != cudaSuccess)
        st = TLFR_OOM;
    if (st == TLFR_OK)
    {
        cudaMemcpy(d_cards, cards, sizeof(Card) * num_cards, cudaMemcpyHostToDevice);
        cudaMemcpy(d_start, tile_start, sizeof(int) * (ntiles + 1), cudaMemcpyHostToDevice);
        if (num_items > 0)
            cudaMemcpy(d_items, tile_items, sizeof(int) * num_items, cudaMemcpyHostToDevice);
        int gx = 1, gy = 1;
        while (gx * gy * 4 <= samples) { gx *= 2; gy *= 2; }
        k_integrate<<<(unsigned)((npix + 127) / 128), 128>>>(d_cards, d_start, d_items, tiles_x, tile_size, C0, C1,
                                                             width, height, samples, gx, gy, seed, d_out);
        if (cudaMemcpy(rgba, d_out, sizeof(float4) * npix, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = TLFR_CUDA;
    }
    cudaFree(d_cards); cudaFree(d_start); cudaFree(d_items); cudaFree(d_out);
    return st;
}

} // namespace tlfr_synth
