// synth_model.h — the analytic scene of the seeded sample-buffer generator
// (synth_scene.cpp): counter-based hashing, textured cards, and the visible
// card of one (x, y, u, v, t) sample.  Shared by the host generator and the
// device kernel that integrates the scene into a reference image
// (synth_reference.cu).
#pragma once
#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define SYN_HD __host__ __device__ __forceinline__
#else
#define SYN_HD inline
#endif

namespace tlfr_synth
{

SYN_HD uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

SYN_HD uint64_t hash3(uint64_t a, uint64_t b, uint64_t c)
{
    return mix64(a ^ mix64(b ^ mix64(c)));
}

// uniform float in [0,1) from a hash
SYN_HD float u01(uint64_t h) { return (float)((h >> 40) * (1.0 / 16777216.0)); }

struct Card
{
    float w0, dw;
    float cx, cy;       // pinhole centre at t=0, pixels
    float hx, hy;       // half-size at depth w0, pixels
    float dx, dy;       // screen motion over the shutter, pixels
    int   disk;
    float cell;         // value-noise lattice spacing, pixels at w0
    uint64_t tex;       // texture seed
    float bx0, by0, bx1, by1;   // sample-space bounding box (all t, all lens positions)
};

SYN_HD float value_noise(const Card& c, float a, float b, int ch)
{
    // lattice in card-local pixel units
    float fx = (a * c.hx + c.hx) / c.cell;
    float fy = (b * c.hy + c.hy) / c.cell;
    float ix = floorf(fx), iy = floorf(fy);
    float tx = fx - ix, ty = fy - iy;
    tx = tx * tx * (3.0f - 2.0f * tx);
    ty = ty * ty * (3.0f - 2.0f * ty);
    auto v = [&](float i, float j) {
        return u01(hash3(c.tex, (uint64_t)(int64_t)i * 2654435761ull + (uint64_t)ch, (uint64_t)(int64_t)j));
    };
    float v00 = v(ix, iy), v10 = v(ix + 1, iy), v01 = v(ix, iy + 1), v11 = v(ix + 1, iy + 1);
    float r = (v00 * (1 - tx) + v10 * tx) * (1 - ty) + (v01 * (1 - tx) + v11 * tx) * ty;
    r = (r < 0.0f) ? 0.0f : r;
    return (1.0f < r) ? 1.0f : r;
}

SYN_HD float coc(float C0, float C1, float w) { return C0 / w + C1; }

// Visible card and its local coordinates for one sample: the nearest of the
// candidate cards whose footprint holds the inverse-lens position; returns the
// card index or -1.
SYN_HD int shade(const Card* cards, const int* cand, int ncand, float C0, float C1, float x, float y, float u,
                 float v, float t, float* W_out, float* a_out, float* b_out)
{
    int best = -1;
    float bestW = 3.0e38f, ba = 0, bb = 0;
    for (int k = 0; k < ncand; k++)
    {
        const int idx = cand[k];
        const Card& c = cards[idx];
        float W = c.w0 + t * c.dw;
        if (!(W < bestW))
            continue;
        float r = coc(C0, C1, W);
        float px = x - r * u, py = y - r * v;
        float s = W / c.w0;
        float lx = px * s - c.cx - t * c.dx;
        float ly = py * s - c.cy - t * c.dy;
        float a = lx / c.hx, b = ly / c.hy;
        bool inside = c.disk ? (a * a + b * b <= 1.0f) : (fabsf(a) <= 1.0f && fabsf(b) <= 1.0f);
        if (!inside)
            continue;
        best = idx; bestW = W; ba = a; bb = b;
    }
    *W_out = bestW; *a_out = ba; *b_out = bb;
    return best;
}

// Reference image of the scene (synth_reference.cu): per pixel the mean colour
// over `samples` points (x, y) in the pixel, (u, v) on the unit lens disk and t
// in [0, 1]; rgba receives width*height*4 floats (host memory).  Returns a
// tlfr_status value.
int integrate_image(const Card* cards, int num_cards, const int* tile_start, const int* tile_items, int num_items,
                    int tiles_x, int tile_size, float C0, float C1, int width, int height, int samples,
                    unsigned long long seed, float* rgba);

} // namespace tlfr_synth
