// Seeded synthetic sample-buffer generator.
//
// The reference reconstructs sample buffers exported by a modified renderer
// (reference README.txt:113-124, 160-164); none ship with it (its only buffer,
// data/butterflies-1spp.bin, is missing).  This generator produces buffers with
// the same record layout (16 floats: x,y,z/w,w,u,v,t,r,g,b,a,mv_x,mv_y,mv_w,dwdx,dwdy,
// SampleBuffer.cpp:283-286) from an analytic scene of textured, moving,
// fronto-parallel cards, so that every record is exactly consistent with the
// reference's thin-lens / affine-motion model:
//
//   screen position at lens (u,v), time t:   xy = p(t) + coc(w(t)) * (u,v)
//   coc(w) = C0/w + C1                        (CameraParams.hpp:72)
//   homogeneous pinhole position (p*w, w) moves linearly in t by mv
//                                             (Reconstruction.hpp:93-121)
//
// A card o has depth w_o(t) = w0 + t*dw, a footprint of half-size (hx,hy) pixels
// at depth w0 (rectangle or disk), pinhole centre c at t=0 and screen motion d
// (pixels over the shutter, at constant depth).  A material point with local
// coordinates (a,b) in [-1,1]^2 sits at homogeneous position
//     X(t) = w0*(c + (a*hx, b*hy)) + t*w0*d,   W(t) = w0 + t*dw,
// so its homogeneous motion vector is mv = (w0*d.x, w0*d.y, dw) for the whole card.
// For each sample (x,y,u,v,t) the visible card is the nearest one whose footprint
// contains the inverse-lens position p = (x,y) - coc(W(t))*(u,v); a background
// card at the largest depth covers the screen and its lens margin, so every
// sample hits something.  Colour = per-card value noise in [0,1], alpha 1.
//
// Sample placement: (x,y) jittered-stratified inside the pixel, (u,v) stratified
// on [-1,1]^2 and t stratified on [0,1], each with an independent per-pixel
// permutation.  All randomness comes from a counter-based hash of (seed, stream,
// index), so the output does not depend on the thread count.
#include "tlfr.h"
#include "synth_model.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace
{

using namespace tlfr_synth;

void card_bounds(Card& c, float C0, float C1)
{
    float mx0 = 1e30f, my0 = 1e30f, mx1 = -1e30f, my1 = -1e30f;
    const int NT = 9;
    for (int k = 0; k < NT; k++)
    {
        float t = (float)k / (NT - 1);
        float W = c.w0 + t * c.dw;
        float s = c.w0 / W;
        float px0 = (c.cx - c.hx + t * c.dx) * s, px1 = (c.cx + c.hx + t * c.dx) * s;
        float py0 = (c.cy - c.hy + t * c.dy) * s, py1 = (c.cy + c.hy + t * c.dy) * s;
        float r = std::fabs(coc(C0, C1, W));
        mx0 = std::min(mx0, px0 - r); mx1 = std::max(mx1, px1 + r);
        my0 = std::min(my0, py0 - r); my1 = std::max(my1, py1 + r);
    }
    // depth is affine in t, so 1/W is monotone and the 9 samples bracket the
    // extremes of the scaled footprint only approximately: pad by 2 pixels
    c.bx0 = mx0 - 2; c.by0 = my0 - 2; c.bx1 = mx1 + 2; c.by1 = my1 + 2;
}

// Per-configuration scene description.
struct SceneDesc
{
    int   W, H, spp;
    float C0, C1;
    int   mode;         // 0 = three fronto-parallel planes; 1 = random cards
    int   num_rects, num_disks;
    float w_min, w_max; // log-uniform card depth
    float side_min, side_max;
    float motion_max;   // radius of the screen-motion disk, pixels
    float dw_frac;      // mv_w uniform in +-dw_frac*w
    float bg_w;         // background depth
    uint64_t seed;
};

std::vector<Card> make_cards(const SceneDesc& d)
{
    std::vector<Card> cards;
    const float margin = std::fabs(d.C0) / std::min(d.w_min, d.bg_w) + std::fabs(d.C1) + 4.0f * d.motion_max + 64.0f;

    // background card: static, covers the screen plus lens/motion margin
    Card bg{};
    bg.w0 = d.bg_w; bg.dw = 0;
    bg.cx = 0.5f * d.W; bg.cy = 0.5f * d.H;
    bg.hx = 0.5f * d.W + margin; bg.hy = 0.5f * d.H + margin;
    bg.disk = 0; bg.cell = 24.0f; bg.tex = hash3(d.seed, 1, 0);
    cards.push_back(bg);

    if (d.mode == 0)
    {
        // two partial planes in front of the background plane (w=5 and w=2)
        Card p5{};
        p5.w0 = 5.0f; p5.cx = 0.42f * d.W; p5.cy = 0.40f * d.H; p5.hx = 0.26f * d.W; p5.hy = 0.24f * d.H;
        p5.cell = 16.0f; p5.tex = hash3(d.seed, 1, 1);
        Card p2{};
        p2.w0 = 2.0f; p2.cx = 0.66f * d.W; p2.cy = 0.64f * d.H; p2.hx = 0.20f * d.W; p2.hy = 0.22f * d.H;
        p2.cell = 12.0f; p2.tex = hash3(d.seed, 1, 2);
        cards.push_back(p5);
        cards.push_back(p2);
    }
    else
    {
        const int n = d.num_rects + d.num_disks;
        for (int k = 0; k < n; k++)
        {
            uint64_t s = hash3(d.seed, 2, (uint64_t)k);
            auto r = [&](int j) { return u01(hash3(s, 3, (uint64_t)j)); };
            Card c{};
            c.w0 = d.w_min * std::pow(d.w_max / d.w_min, r(0));
            c.dw = (2.0f * r(1) - 1.0f) * d.dw_frac * c.w0;
            c.hx = 0.5f * (d.side_min + (d.side_max - d.side_min) * r(2));
            c.hy = 0.5f * (d.side_min + (d.side_max - d.side_min) * r(3));
            c.cx = -0.1f * d.W + 1.2f * d.W * r(4);
            c.cy = -0.1f * d.H + 1.2f * d.H * r(5);
            float ang = 6.2831853f * r(6), rad = d.motion_max * std::sqrt(r(7));
            c.dx = rad * std::cos(ang);
            c.dy = rad * std::sin(ang);
            c.disk = (k >= d.num_rects);
            if (c.disk)
                c.hy = c.hx;
            c.cell = 6.0f + 18.0f * r(8);
            c.tex = hash3(s, 4, 0);
            cards.push_back(c);
        }
    }
    for (auto& c : cards)
        card_bounds(c, d.C0, d.C1);
    return cards;
}

// spp samples on an nx*ny stratification grid, nx >= ny (exact for powers of two)
int grid_nx(int n) { int nx = 1, ny = 1; while (nx * ny < n) { if (nx <= ny) nx *= 2; else ny *= 2; } return nx; }
int grid_ny(int n) { int nx = 1, ny = 1; while (nx * ny < n) { if (nx <= ny) nx *= 2; else ny *= 2; } return ny; }

void generate(const SceneDesc& d, float* out, int num_threads)
{
    std::vector<Card> cards = make_cards(d);

    // bin cards into 32x32-pixel tiles by their sample-space bounding boxes
    const int TS = 32;
    const int tx = (d.W + TS - 1) / TS, ty = (d.H + TS - 1) / TS;
    std::vector<std::vector<int>> bins((size_t)tx * ty);
    for (int k = 0; k < (int)cards.size(); k++)
    {
        const Card& c = cards[k];
        int x0 = std::max(0, (int)std::floor(c.bx0 / TS)), x1 = std::min(tx - 1, (int)std::floor(c.bx1 / TS));
        int y0 = std::max(0, (int)std::floor(c.by0 / TS)), y1 = std::min(ty - 1, (int)std::floor(c.by1 / TS));
        for (int j = y0; j <= y1; j++)
            for (int i = x0; i <= x1; i++)
                bins[(size_t)j * tx + i].push_back(k);
    }

    const int spp = d.spp;
    const int gx = grid_nx(spp), gy = grid_ny(spp);
    auto work = [&](int row0, int row1) {
        std::vector<int> perm_uv(spp), perm_t(spp);
        for (int y = row0; y < row1; y++)
        for (int x = 0; x < d.W; x++)
        {
            const std::vector<int>& cand = bins[(size_t)(y / TS) * tx + (x / TS)];
            uint64_t ph = hash3(d.seed, 10, (uint64_t)y * d.W + x);
            for (int i = 0; i < spp; i++) { perm_uv[i] = i; perm_t[i] = i; }
            for (int i = spp - 1; i > 0; i--)
            {
                int j = (int)(hash3(ph, 11, (uint64_t)i) % (uint64_t)(i + 1));
                std::swap(perm_uv[i], perm_uv[j]);
                j = (int)(hash3(ph, 12, (uint64_t)i) % (uint64_t)(i + 1));
                std::swap(perm_t[i], perm_t[j]);
            }
            for (int i = 0; i < spp; i++)
            {
                uint64_t sh = hash3(ph, 13, (uint64_t)i);
                auto r = [&](int j) { return u01(hash3(sh, 14, (uint64_t)j)); };
                int sx = i % gx, sy = (i / gx) % gy;
                float fx = ((float)sx + r(0)) / gx, fy = ((float)sy + r(1)) / gy;
                if (fx >= 1.0f) fx = 0.99999994f;
                if (fy >= 1.0f) fy = 0.99999994f;
                float x_s = (float)x + fx, y_s = (float)y + fy;
                int k = perm_uv[i];
                int ux = k % gx, vy = (k / gx) % gy;
                float u = -1.0f + 2.0f * (((float)ux + r(2)) / gx);
                float v = -1.0f + 2.0f * (((float)vy + r(3)) / gy);
                u = std::min(std::max(u, -1.0f), 1.0f);
                v = std::min(std::max(v, -1.0f), 1.0f);
                float t = ((float)perm_t[i] + r(4)) / spp;
                if (t > 1.0f) t = 1.0f;
                float Wv, a, b;
                int ci = shade(cards.data(), cand.data(), (int)cand.size(), d.C0, d.C1, x_s, y_s, u, v, t, &Wv, &a, &b);
                if (ci < 0)
                {   // cannot happen with the background card; keep the record valid
                    ci = 0; Wv = cards[0].w0; a = 0; b = 0;
                }
                const Card& c = cards[ci];
                float* e = out + ((size_t)((size_t)y * d.W + x) * spp + i) * 16;
                e[0] = x_s; e[1] = y_s; e[2] = 1.0f / Wv; e[3] = Wv;
                e[4] = u; e[5] = v; e[6] = t;
                e[7] = value_noise(c, a, b, 0);
                e[8] = value_noise(c, a, b, 1);
                e[9] = value_noise(c, a, b, 2);
                e[10] = 1.0f;
                e[11] = c.w0 * c.dx; e[12] = c.w0 * c.dy; e[13] = c.dw;
                e[14] = 0.0f; e[15] = 0.0f;
            }
        }
    };

    int nt = std::max(1, num_threads);
    nt = std::min(nt, d.H);
    std::vector<std::thread> th;
    for (int k = 0; k < nt; k++)
    {
        int r0 = (int)((int64_t)d.H * k / nt), r1 = (int)((int64_t)d.H * (k + 1) / nt);
        th.emplace_back(work, r0, r1);
    }
    for (auto& t : th)
        t.join();
}

} // namespace

namespace
{

// Scene description of a preset (TLFR_SCENE_*); false for an unknown preset.
bool preset_desc(int preset, int width, int height, int spp, unsigned long long seed, SceneDesc& d)
{
    d = SceneDesc{};
    d.W = width; d.H = height; d.spp = spp; d.seed = seed;
    switch (preset)
    {
    case TLFR_SCENE_PLANES:         // three fronto-parallel planes, defocus only
        d.mode = 0; d.C0 = -15.24f; d.C1 = 19.05f; d.bg_w = 12.0f; d.w_min = 2.0f; d.w_max = 12.0f;
        return true;
    case TLFR_SCENE_CARDS:          // 64 moving rectangles, defocus + motion
        d.mode = 1; d.C0 = -15.24f; d.C1 = 19.05f; d.num_rects = 64; d.num_disks = 0;
        d.w_min = 1.0f; d.w_max = 50.0f; d.side_min = 20.0f; d.side_max = 300.0f;
        d.motion_max = 40.0f; d.dw_frac = 0.1f; d.bg_w = 60.0f;
        return true;
    case TLFR_SCENE_CARDS_LARGE:    // 256 rectangles + 64 disks, strong blur, fast motion
        d.mode = 1; d.C0 = -30.0f; d.C1 = 40.0f; d.num_rects = 256; d.num_disks = 64;
        d.w_min = 0.5f; d.w_max = 100.0f; d.side_min = 20.0f; d.side_max = 300.0f;
        d.motion_max = 60.0f; d.dw_frac = 0.1f; d.bg_w = 120.0f;
        return true;
    default:
        return false;
    }
}

} // namespace

extern "C" tlfr_status tlfr_synth_scene(int preset, int width, int height, int spp, unsigned long long seed,
                                        float* records, float* coc_out)
{
    if (!records || width <= 0 || height <= 0 || spp <= 0 || spp > 256)
        return TLFR_BAD_ARG;
    SceneDesc d;
    if (!preset_desc(preset, width, height, spp, seed, d))
        return TLFR_BAD_ARG;
    unsigned hc = std::thread::hardware_concurrency();
    generate(d, records, hc ? (int)hc : 1);
    if (coc_out)
    {
        coc_out[0] = d.C0;
        coc_out[1] = d.C1;
    }
    return TLFR_OK;
}

#ifndef TLFR_SYNTH_HOST_ONLY
extern "C" tlfr_status tlfr_synth_reference_image(int preset, int width, int height, int samples,
                                                  unsigned long long seed, float* rgba)
{
    if (!rgba || width <= 0 || height <= 0 || samples <= 0 || samples > (1 << 16))
        return TLFR_BAD_ARG;
    SceneDesc d;
    if (!preset_desc(preset, width, height, 1, seed, d))
        return TLFR_BAD_ARG;
    std::vector<Card> cards = make_cards(d);
    // cards binned into 32x32-pixel tiles by their sample-space bounding boxes
    // (as the generator does), as one list per tile
    const int TS = 32;
    const int tx = (d.W + TS - 1) / TS, ty = (d.H + TS - 1) / TS;
    std::vector<std::vector<int>> bins((size_t)tx * ty);
    for (int k = 0; k < (int)cards.size(); k++)
    {
        const Card& c = cards[k];
        int x0 = std::max(0, (int)std::floor(c.bx0 / TS)), x1 = std::min(tx - 1, (int)std::floor(c.bx1 / TS));
        int y0 = std::max(0, (int)std::floor(c.by0 / TS)), y1 = std::min(ty - 1, (int)std::floor(c.by1 / TS));
        for (int j = y0; j <= y1; j++)
            for (int i = x0; i <= x1; i++)
                bins[(size_t)j * tx + i].push_back(k);
    }
    std::vector<int> start(1, 0), items;
    for (auto& b : bins)
    {
        items.insert(items.end(), b.begin(), b.end());
        start.push_back((int)items.size());
    }
    return (tlfr_status)tlfr_synth::integrate_image(cards.data(), (int)cards.size(), start.data(), items.data(), (int)items.size(),
                                       tx, TS, d.C0, d.C1, d.W, d.H, samples, seed, rgba);
}
#endif
