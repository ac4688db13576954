// tlfr_api.cpp — the C ABI (include/tlfr.h): sample-buffer IO, the output
// sampling pattern, context lifetime, and the calls into the CUDA build and
// query code.  Host code; compiled with -ffp-contract=off so that the pattern
// arithmetic matches the reference's IEEE single-precision host code.
#include "tlfr.h"
#include "tlfr_common.cuh"
#include "tlfr_internal.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

// Records live in page-locked memory when a CUDA device is present (full-rate
// host-to-device copies), in ordinary memory otherwise.
struct tlfr_buffer
{
    int W = 0, H = 0, spp = 0;
    float coc[2] = { 0, 0 };
    float* rec = nullptr;       // W*H*spp*16
    size_t n = 0;               // records
    bool pinned = false;

    bool alloc(size_t records)
    {
        n = records;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0 &&
            cudaMallocHost((void**)&rec, sizeof(float) * 16 * (n ? n : 1)) == cudaSuccess)
            pinned = true;
        else
        {
            cudaGetLastError();
            rec = (float*)malloc(sizeof(float) * 16 * (n ? n : 1));
            pinned = false;
        }
        return rec != nullptr;
    }
    ~tlfr_buffer()
    {
        if (!rec) return;
        if (pinned) cudaFreeHost(rec);
        else        free(rec);
    }
};

struct tlfr_ctx
{
    tlfr::Ctx c;
    bool own_stream = false;
};

namespace
{

thread_local std::string g_create_error;

tlfr_status fail(tlfr_ctx* ctx, tlfr_status s, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->c.error = buf;
    else     g_create_error = buf;
    return s;
}

// ---------------------------------------------------------------------------
// Text record parsing: the framework's float parser (framework/base/String.cpp:
// 428-480) accumulates digits in single precision and scales the exponent with
// powf; text buffers load bit-identically only through the same steps.
// ---------------------------------------------------------------------------
bool parse_float(const char*& ptr, float& value)
{
    const char* tmp = ptr;
    bool neg = false;
    if (*tmp == '+') tmp++;
    else if (*tmp == '-') { neg = true; tmp++; }
    float v = 0.0f;
    int digits = 0;
    while (*tmp >= '0' && *tmp <= '9')
    {
        v = v * 10.0f + (float)(*tmp++ - '0');
        digits++;
    }
    if (*tmp == '.')
    {
        tmp++;
        float scale = 1.0f;
        while (*tmp >= '0' && *tmp <= '9')
        {
            scale *= 0.1f;
            v += scale * (float)(*tmp++ - '0');
            digits++;
        }
    }
    if (!digits)
        return false;
    ptr = tmp;
    if (*ptr == '#')
    {
        struct { const char* lit; uint32_t pos, neg; } specials[] = {
            { "#INF", 0x7F800000u, 0xFF800000u }, { "#SNAN", 0x7F800001u, 0xFF800001u },
            { "#QNAN", 0x7FC00001u, 0xFFC00001u }, { "#IND", 0x7FC00000u, 0xFFC00000u } };
        for (auto& sp : specials)
        {
            size_t L = strlen(sp.lit);
            if (strncmp(ptr, sp.lit, L) == 0)
            {
                ptr += L;
                uint32_t bits = neg ? sp.neg : sp.pos;
                memcpy(&value, &bits, 4);
                return true;
            }
        }
    }
    if (*tmp == 'e' || *tmp == 'E')
    {
        const char* t2 = tmp + 1;
        bool eneg = false;
        if (*t2 == '+') t2++;
        else if (*t2 == '-') { eneg = true; t2++; }
        if (*t2 >= '0' && *t2 <= '9')
        {
            int e = 0;
            while (*t2 >= '0' && *t2 <= '9')
                e = e * 10 + (*t2++ - '0');
            if (eneg) e = -e;
            ptr = t2;
            if (e)
                v *= powf(10.0f, (float)e);
        }
    }
    value = neg ? -v : v;
    return true;
}

// ---------------------------------------------------------------------------
// Output sampling pattern (Reconstruction.cpp:452-512) and the sequences it
// uses (reconstruction_lib/common/Util.cpp:37-74, 229-300;
// framework/base/Random.cpp:52-92).
// ---------------------------------------------------------------------------
struct Ranrot
{
    int32_t p1, p2;
    uint32_t buf[11];
    explicit Ranrot(uint32_t seed)
    {
        if (seed == 0) seed--;
        for (int i = 0; i < 11; i++)
        {
            seed ^= seed << 13;
            seed ^= seed >> 17;
            seed ^= seed << 5;
            buf[i] = seed;
        }
        p1 = 0; p2 = 7;
        for (int i = 0; i < 11; i++) next();
    }
    uint32_t next()
    {
        uint32_t x = buf[p1] + buf[p2];
        x = (x << 13) | (x >> 19);
        buf[p1] = x;
        p1--; p1 += (p1 >> 31) & 11;
        p2--; p2 += (p2 >> 31) & 11;
        return x;
    }
    float f32() { return (float)next() * (1.0f / 4294967296.0f); }
};

float hammersley(int i, int num) { return ((float)i + 0.5f) / (float)num; }

float halton(int base, int i)
{
    float h = 0.0f;
    float half = tlfr::rcp((float)base);
    while (i)
    {
        int digit = i % base;
        h = h + (float)digit * half;
        i = (i - digit) / base;
        half = half / (float)base;
    }
    return h;
}

// Sobol dimension 3: primitive polynomial x^3 + x + 1, initial direction
// numbers m = (1, 3, 1).
float sobol_dim3(int i)
{
    static uint32_t v[32];
    static bool init = false;
    if (!init)
    {
        v[0] = 1u << 31; v[1] = 3u << 30; v[2] = 1u << 29;
        for (int k = 3; k < 32; k++)
            v[k] = v[k - 2] ^ v[k - 3] ^ (v[k - 3] >> 3);
        init = true;
    }
    uint32_t r = 0;
    for (unsigned c = 0; i; i >>= 1, ++c)
        if (i & 1) r ^= v[c];
    return (float)r * (1.0f / 4294967296.0f);
}

// Sobol dimension 4: primitive polynomial x^3 + x^2 + 1, initial direction
// numbers m = (1, 1, 1).
float sobol_dim4(int i)
{
    static uint32_t v[32];
    static bool init = false;
    if (!init)
    {
        v[0] = 1u << 31; v[1] = 1u << 30; v[2] = 1u << 29;
        for (int k = 3; k < 32; k++)
            v[k] = v[k - 1] ^ v[k - 3] ^ (v[k - 3] >> 3);
        init = true;
    }
    uint32_t r = 0;
    for (unsigned c = 0; i; i >>= 1, ++c)
        if (i & 1) r ^= v[c];
    return (float)r * (1.0f / 4294967296.0f);
}

void sobol_2d(int i, float* out)
{
    uint32_t r1 = 0, r2 = 0;
    for (uint32_t v1 = 1u << 31, v2 = 3u << 30; i; i >>= 1)
    {
        if (i & 1) { r1 ^= v1; r2 ^= v2 << 1; }
        v1 |= v1 >> 1;
        v2 ^= v2 >> 1;
    }
    out[0] = (float)r1 * (1.0f / 4294967296.0f);
    out[1] = (float)r2 * (1.0f / 4294967296.0f);
}

float larcher_pillichshammer(int i)
{
    uint32_t r = 0;
    for (uint32_t v = 1u << 31; i; i >>= 1, v |= v >> 1)
        if (i & 1) r ^= v;
    return (float)((double)r / (double)0x100000000LL);
}

// Shirley-Chiu concentric square-to-disk map
void to_unit_disk(float sx, float sy, float& ou, float& ov)
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
            phi = (b != 0) ? (PI / 4) * (6.0f - (a / b)) : 0.0f;
        }
    }
    ou = r * cosf(phi);
    ov = r * sinf(phi);
}

struct PatSample { float x, y, u, v, t, key; };

struct KeySort
{
    PatSample* e;
    int cmp(int a, int b) const { return (e[a].key < e[b].key) ? -1 : (e[a].key > e[b].key) ? 1 : 0; }
    void swap(int a, int b) { PatSample t = e[a]; e[a] = e[b]; e[b] = t; }
};

} // namespace

namespace tlfr
{

void generate_output_pattern(int M, bool override_uvt, const float* uvt, std::vector<float>& out5)
{
    Ranrot rnd(242);
    std::vector<PatSample> all((size_t)64 * M);
    for (int j = 0; j < 64; j++)
    {
        const float xo[2] = { hammersley(j, 64), larcher_pillichshammer(j) };
        const float uo[2] = { halton(2, j), halton(3, j) };
        const float tj = rnd.f32();
        PatSample* p = &all[(size_t)j * M];
        for (int i = 0; i < M; i++)
        {
            float s2[2];
            sobol_2d(i + 1, s2);
            float x = sobol_dim3(i + 1);
            float y = larcher_pillichshammer(i + 1);
            float t = ((float)i + tj) / (float)M;
            float xy[2] = { x + xo[0], y + xo[1] };
            float uv[2] = { s2[0] + uo[0], s2[1] + uo[1] };
            if (xy[0] >= 1.f) xy[0] -= 1.f;
            if (xy[1] >= 1.f) xy[1] -= 1.f;
            if (uv[0] >= 1.f) uv[0] -= 1.f;
            if (uv[1] >= 1.f) uv[1] -= 1.f;
            // (u,v,t) Morton key for coherence (Reconstruction.cpp:482-489)
            int ub = (int)floorf(256.0f * uv[0]);
            int vb = (int)floorf(256.0f * uv[1]);
            int tb = (int)floorf(256.0f * t);
            int key = 0;
            for (int k = 0; k < 8; k++)
                key |= ((ub >> k) & 1) << (3 * k + 2) | ((vb >> k) & 1) << (3 * k + 1) | ((tb >> k) & 1) << (3 * k + 0);
            to_unit_disk(uv[0], uv[1], uv[0], uv[1]);
            if (override_uvt)
            {
                uv[0] = uvt[0]; uv[1] = uvt[1];
                t = uvt[2];
            }
            if (M == 1)
                xy[0] = xy[1] = 0.5f;
            p[i] = PatSample{ xy[0], xy[1], uv[0], uv[1], t, (float)key };
        }
        KeySort ks{ p };
        fw_sort(ks, 0, M);
    }
    out5.resize((size_t)64 * M * 5);
    for (size_t k = 0; k < all.size(); k++)
    {
        out5[k * 5 + 0] = all[k].x; out5[k * 5 + 1] = all[k].y;
        out5[k * 5 + 2] = all[k].u; out5[k * 5 + 3] = all[k].v;
        out5[k * 5 + 4] = all[k].t;
    }
}

} // namespace tlfr

namespace
{

tlfr_status upload_pattern(tlfr_ctx* ctx)
{
    tlfr::Ctx& c = ctx->c;
    const bool ov = c.params.override_uvt != 0;
    c.out_spp = c.params.output_spp > 0 ? c.params.output_spp : (ov ? 1 : 128);
    if (c.out_spp > 1024)
        return fail(ctx, TLFR_BAD_ARG, "output_spp %d out of range [1,1024]", c.out_spp);
    tlfr::generate_output_pattern(c.out_spp, ov, c.params.uvt, c.h_pattern);
    if (c.d_pattern) cudaFree(c.d_pattern);
    c.d_pattern = nullptr;
    cudaError_t e = cudaMalloc(&c.d_pattern, sizeof(float) * c.h_pattern.size());
    if (e != cudaSuccess)
        return fail(ctx, TLFR_OOM, "pattern allocation: %s", cudaGetErrorString(e));
    e = cudaMemcpyAsync(c.d_pattern, c.h_pattern.data(), sizeof(float) * c.h_pattern.size(), cudaMemcpyHostToDevice,
                        c.stream);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "pattern upload: %s", cudaGetErrorString(e));
    return TLFR_OK;
}

void free_ctx_buffers(tlfr::Ctx& c)
{
    void* ptrs[] = { c.own_records ? c.d_records : nullptr, c.rp_pos, c.rp_mot, c.rp_cell, c.hits, c.d_grid,
                     c.cell_count, c.cell_start, c.cell_items, c.kd, c.kd_level, c.kd_leaves_ordered, c.perm, c.box,
                     c.sbounds, c.surface, c.pending, c.leaf_task_rank, c.ordered_n, c.ordered_prefmax, c.top,
                     c.nodes, c.node_tspan, c.s_rec, c.s_col, c.s_id, c.d_pattern, c.qcol, c.heavy_queue, c.ovf_queue,
                     c.ovf_scratch, c.coop_scratch, c.toggle_arena, c.d_stats, c.d_out, c.route_fa, c.route_feats, c.route_prob,
                     c.route_fast, c.route_img };
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c.ev0) cudaEventDestroy(c.ev0);
    if (c.ev1) cudaEventDestroy(c.ev1);
    if (c.ev2) cudaEventDestroy(c.ev2);
    if (c.evq0) cudaEventDestroy(c.evq0);
    if (c.evq1) cudaEventDestroy(c.evq1);
    if (c.evq2) cudaEventDestroy(c.evq2);
}

tlfr_status begin_ctx(const tlfr_params* params, void* stream, int W, int H, int spp, float c0, float c1,
                      tlfr_ctx** out, tlfr_ctx*& ctx)
{
    if (!out || W <= 0 || H <= 0 || spp <= 0)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_create: bad argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    {
        cudaGetLastError();
        return fail(nullptr, TLFR_NO_DEVICE, "no CUDA device");
    }
    ctx = new (std::nothrow) tlfr_ctx();
    if (!ctx)
        return fail(nullptr, TLFR_OOM, "host allocation failed");
    tlfr::Ctx& c = ctx->c;
    if (params) c.params = *params;
    else        tlfr_params_default(&c.params);
    if (c.params.device < 0 || c.params.device >= ndev)
        return fail(ctx, TLFR_BAD_ARG, "device %d out of range", c.params.device);
    c.device = c.params.device;
    cudaError_t e = cudaSetDevice(c.device);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    e = cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device);
    if (e != cudaSuccess || c.num_sms <= 0)
        return fail(ctx, TLFR_CUDA, "cudaDeviceGetAttribute(multiprocessor count): %s", cudaGetErrorString(e));
    c.stream = (cudaStream_t)stream;
    c.W = W; c.H = H; c.spp_in = spp;
    c.n_in = (size_t)W * H * spp;
    c.coc0_raw[0] = c0; c.coc0_raw[1] = c1;
    // refocus round trip (Reconstruction.cpp:77-87)
    {
        float a = -c0;
        float f = (-c0) * tlfr::rcp(c1);
        a *= c.params.aperture_adjust;
        f *= c.params.focus_adjust;
        c.coc[0] = -a;
        c.coc[1] = a * tlfr::rcp(f);
    }
    // m_spp: next power of two (Reconstruction.cpp:63-73, Util.hpp:64-73)
    uint32_t v = (uint32_t)spp;
    v--; v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    c.spp = tlfr::maxi(1, (int)(v + 1));
    if (c.spp > 256)
        return fail(ctx, TLFR_BAD_ARG, "TreeGather::Filterer::reconstruct -- unknown SPP (%d)", spp);
    if (cudaEventCreate(&c.ev0) != cudaSuccess || cudaEventCreate(&c.ev1) != cudaSuccess ||
        cudaEventCreate(&c.ev2) != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "cudaEventCreate failed");
    tlfr_status st = upload_pattern(ctx);
    if (st != TLFR_OK)
        return st;
    *out = nullptr;
    return TLFR_OK;
}

tlfr_status run_build(tlfr_ctx* ctx, const float* d_rec)
{
    tlfr::Ctx& c = ctx->c;
    cudaEventRecord(c.ev0, c.stream);
    const long long l0 = c.launches;
    c.cur_records = d_rec;
    tlfr_status st = tlfr::build_hierarchy(c, d_rec);
    c.last.build_launches = (double)(c.launches - l0);
    if (st != TLFR_OK)
        return st;
    cudaEventRecord(c.ev1, c.stream);
    cudaError_t e = cudaEventSynchronize(c.ev1);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "build: %s", cudaGetErrorString(e));
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    c.last.build_ms = ms;
    return TLFR_OK;
}

} // namespace

namespace
{

// 4x4 float matrices with the framework's arithmetic (framework/base/Math.hpp):
// products accumulate from 0 in index order; the inverse is the adjugate by
// cofactors times rcp of the determinant summed along all four columns, times 4
// (MatrixBase::inverted); 3x3 determinants by the rule of Sarrus in the
// framework's term order (detImpl).
struct Mat4
{
    float m[4][4];
    Mat4()
    {
        for (int r = 0; r < 4; r++)
            for (int c = 0; c < 4; c++)
                m[r][c] = r == c ? 1.0f : 0.0f;
    }
    static Mat4 rows(const float* a)
    {
        Mat4 r;
        for (int i = 0; i < 16; i++)
            r.m[i / 4][i % 4] = a[i];
        return r;
    }
    void store(float* a) const
    {
        for (int i = 0; i < 16; i++)
            a[i] = m[i / 4][i % 4];
    }
};

Mat4 operator*(const Mat4& a, const Mat4& b)
{
    Mat4 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
        {
            float s = 0.0f;
            for (int k = 0; k < 4; k++)
                s += a.m[i][k] * b.m[k][j];
            r.m[i][j] = s;
        }
    return r;
}

Mat4 operator-(const Mat4& a, const Mat4& b)
{
    Mat4 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            r.m[i][j] = a.m[i][j] - b.m[i][j];
    return r;
}

Mat4 transposed(const Mat4& a)
{
    Mat4 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            r.m[i][j] = a.m[j][i];
    return r;
}

float det3(const float s[3][3])
{
    return s[0][0] * s[1][1] * s[2][2] - s[0][0] * s[1][2] * s[2][1] +
           s[1][0] * s[2][1] * s[0][2] - s[1][0] * s[2][2] * s[0][1] +
           s[2][0] * s[0][1] * s[1][2] - s[2][0] * s[0][2] * s[1][1];
}

Mat4 inverted(const Mat4& a)
{
    Mat4 r;
    float d = 0.0f;
    float si = 1.0f;
    for (int i = 0; i < 4; i++)
    {
        float sj = si;
        for (int j = 0; j < 4; j++)
        {
            float sub[3][3];
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++)
                    sub[k][l] = a.m[k < j ? k : k + 1][l < i ? l : l + 1];
            const float dd = det3(sub) * sj;
            r.m[i][j] = dd;
            d += dd * a.m[j][i];
            sj = -sj;
        }
        si = -si;
    }
    const float rd = tlfr::rcp(d);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            r.m[i][j] = (r.m[i][j] * rd) * 4.0f;
    return r;
}

Mat4 scale3(float x, float y, float z)
{
    Mat4 r;
    r.m[0][0] = x; r.m[1][1] = y; r.m[2][2] = z;
    return r;
}

Mat4 translate3(float x, float y, float z)
{
    Mat4 r;
    r.m[0][3] = x; r.m[1][3] = y; r.m[2][3] = z;
    return r;
}

// CameraParams::getCocCoeffs (CameraParams.hpp:112-132): the projection of the
// lens's half extent, scaled to the window width
void view_coc(const tlfr_view& v, float coc[2])
{
    const Mat4 P = Mat4::rows(v.projection);
    Mat4 dof;
    const float ux = 0.5f, uy = 0.0f;
    dof.m[0][2] = (ux * v.aperture_radius) / v.focus_distance;
    dof.m[1][2] = (uy * v.aperture_radius) / v.focus_distance;
    dof.m[2][2] = 1.0f;
    dof.m[3][2] = 0.0f;
    dof.m[0][3] = ux * v.aperture_radius;
    dof.m[1][3] = uy * v.aperture_radius;
    dof.m[2][3] = 0.0f;
    dof.m[3][3] = 1.0f;
    const Mat4 m = P * dof - P;
    coc[0] = -m.m[0][3] * (float)v.window_size[0];
    coc[1] = m.m[0][2] * (float)v.window_size[0];
}

// The matrices of TreeGather::reconstructDofMotionShadows (Reconstruction.cpp:365-392)
// for an image of w x h pixels, and the light-source pattern of M output samples.
void derive_dms_view(const tlfr_view& cam, const tlfr_view& light, int w, int h, int M, tlfr::DmsView& out)
{
    const Mat4 Pl = Mat4::rows(light.projection);
    const Mat4 Pc = Mat4::rows(cam.projection);
    const Mat4 invPc = inverted(Pc);
    const Mat4 c2w = Mat4::rows(cam.camera_to_world);
    const Mat4 lw2c = Mat4::rows(light.world_to_camera);
    const Mat4 c2s = Pl * lw2c * c2w * invPc;
    const Mat4 c2s2 = lw2c * c2w;
    const Mat4 c2s2_inv_t = transposed(inverted(c2s2));
    const Mat4 c2w_inv_t = transposed(inverted(c2w));
    const Mat4 ws = scale3(0.5f * (float)w, 0.5f * (float)h, 0.5f) * translate3(1.0f, 1.0f, 1.0f);
    const Mat4 invws = translate3(-1.0f, -1.0f, -1.0f) * scale3(2.f / (float)w, 2.f / (float)h, 2.f);
    const Mat4 wsPc = ws * Pc;
    Mat4 zfromw;
    zfromw.m[2][2] = wsPc.m[2][3];
    zfromw.m[2][3] = -wsPc.m[2][2];
    const Mat4 c2l = ws * c2s * invws * zfromw;
    (c2l).store(out.c2l);
    (invws * zfromw).store(out.clip_xyw);
    Mat4 ip = invPc;
    for (int c = 0; c < 4; c++)
    {
        ip.m[2][c] = c == 2 ? -1.0f : 0.0f;
        ip.m[3][c] = c == 3 ? 1.0f : 0.0f;
    }
    ip.store(out.ip);
    (c2s2 * invPc).store(out.light_pos);
    c2s2_inv_t.store(out.c2s_inv_t);
    c2w_inv_t.store(out.c2w_inv_t);
    out.cam_far_w = cam.far_plane - 1e-2f;
    view_coc(cam, out.ccoc);
    view_coc(light, out.lcoc);
    out.light_uv.resize(2 * (size_t)M);
    for (int i = 0; i < M; i++)
    {
        out.light_uv[2 * i + 0] = sobol_dim3(i + 1);
        out.light_uv[2 * i + 1] = sobol_dim4(i + 1);
    }
}

} // namespace

extern "C" {

void tlfr_params_default(tlfr_params* p)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->aperture_adjust = 1.0f;
    p->focus_adjust = 1.0f;
    p->lens_filter = TLFR_FILTER_BOX;
    p->time_filter = TLFR_FILTER_BOX;
    p->override_uvt = 0;
    p->output_spp = 0;
    p->device = 0;
}

tlfr_status tlfr_buffer_from_host(const float* rec, int W, int H, int spp, float c0, float c1, tlfr_buffer** out)
{
    if (!rec || !out || W <= 0 || H <= 0 || spp <= 0)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_buffer_from_host: bad argument");
    tlfr_buffer* b = new (std::nothrow) tlfr_buffer();
    if (!b)
        return fail(nullptr, TLFR_OOM, "host allocation failed");
    b->W = W; b->H = H; b->spp = spp;
    b->coc[0] = c0; b->coc[1] = c1;
    const size_t n = (size_t)W * H * spp;
    if (!b->alloc(n)) { delete b; return fail(nullptr, TLFR_OOM, "host allocation failed"); }
    memcpy(b->rec, rec, sizeof(float) * 16 * n);
    for (size_t k = 0; k < n; k++)
        b->rec[k * 16 + 10] = 1.0f;     // alpha forced to 1 (SampleBuffer.cpp:343, 372)
    *out = b;
    return TLFR_OK;
}

// UVTSampleBuffer(const char*) (SampleBuffer.cpp:230-387)
tlfr_status tlfr_buffer_load(const char* path, tlfr_buffer** out)
{
    if (!path || !out)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_buffer_load: bad argument");
    FILE* fp = fopen(path, "rb");
    if (!fp)
        return fail(nullptr, TLFR_IO, "File not found: %s", path);
    std::string hp = std::string(path) + ".header";
    FILE* fph = fopen(hp.c_str(), "rt");
    const bool separate = fph != nullptr;
    if (!separate)
        fph = fp;
    tlfr_buffer* b = new (std::nothrow) tlfr_buffer();
    auto cleanup = [&]() { fclose(fp); if (separate) fclose(fph); };
    float version = 0;
    int W = 0, H = 0, spp = 0;
    if (fscanf(fph, "Version %f\n", &version) != 1 || fscanf(fph, "Width %d\n", &W) != 1 ||
        fscanf(fph, "Height %d\n", &H) != 1 || fscanf(fph, "Samples per pixel %d\n", &spp) != 1)
    {
        cleanup(); delete b;
        return fail(nullptr, TLFR_FORMAT, "malformed sample buffer header: %s", path);
    }
    if (version != 1.3f)
    {
        cleanup(); delete b;
        return fail(nullptr, TLFR_FORMAT, "Unsupported sample stream version (%.1f)", version);
    }
    if (W <= 0 || H <= 0 || spp <= 0 || (double)W * H * spp > 2.0e9)
    {
        cleanup(); delete b;
        return fail(nullptr, TLFR_FORMAT, "bad buffer size %dx%dx%d", W, H, spp);
    }
    char motion[1024], enc[1024], desc[1024];
    if (fscanf(fph, "Motion model: %1023s\n", motion) != 1) { /* optional line, as in the reference */ }
    float c0 = 0, c1 = 0;
    if (fscanf(fph, "CoC coefficients (coc radius = C0/w+C1): %f,%f\n", &c0, &c1) != 2)
    {
        cleanup(); delete b;
        return fail(nullptr, TLFR_FORMAT, "missing CoC coefficients in header");
    }
    bool binary = false;
    if (fscanf(fph, "Encoding = %1023s\n", enc) == 1)
        binary = strcmp(enc, "binary") == 0;
    if (fscanf(fph, "\n") < 0) {}
    if (fscanf(fph, "%1023s\n", desc) != 1) {}
    b->W = W; b->H = H; b->spp = spp; b->coc[0] = c0; b->coc[1] = c1;
    const size_t n = (size_t)W * H * spp;
    if (!b->alloc(n)) { cleanup(); delete b; return fail(nullptr, TLFR_OOM, "host allocation failed"); }
    memset(b->rec, 0, sizeof(float) * 16 * n);
    if (binary)
    {
        size_t got = fread(b->rec, 64, n, fp);
        if (got != n)
        {
            cleanup(); delete b;
            return fail(nullptr, TLFR_FORMAT, "truncated binary records (%zu of %zu)", got, n);
        }
    }
    else
    {
        std::vector<char> line(4096);
        for (size_t k = 0; k < n; k++)
        {
            if (!fgets(line.data(), 4096, fp))
            {
                cleanup(); delete b;
                return fail(nullptr, TLFR_FORMAT, "truncated text records (%zu of %zu)", k, n);
            }
            const char* p = line.data();
            float* e = &b->rec[k * 16];
            for (int v = 0; v < 16; v++)
            {
                if (v > 0)
                {
                    while (*p != ',' && *p != '\n' && *p != '\0') p++;
                    if (*p) p++;
                }
                float val = 0.0f;
                if (!parse_float(p, val))
                    val = 0.0f;     // the reference leaves the value unset here
                e[v] = val;
            }
        }
    }
    for (size_t k = 0; k < n; k++)
        b->rec[k * 16 + 10] = 1.0f;
    cleanup();
    *out = b;
    return TLFR_OK;
}

// UVTSampleBuffer::serialize (SampleBuffer.cpp:404-564), version 1.3.  As in the
// reference the alpha field is written with the blue channel, and binary
// output needs a separate header.
tlfr_status tlfr_buffer_save(const tlfr_buffer* b, const char* path, int separate_header, int binary)
{
    if (!b || !path)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_buffer_save: bad argument");
    if (binary && !separate_header)
        return fail(nullptr, TLFR_BAD_ARG, "binary serialization supported only with a separate header");
    FILE* fp = fopen(path, binary ? "wb" : "wt");
    if (!fp)
        return fail(nullptr, TLFR_IO, "cannot open %s", path);
    FILE* fph = fp;
    if (separate_header)
    {
        fph = fopen((std::string(path) + ".header").c_str(), "wt");
        if (!fph) { fclose(fp); return fail(nullptr, TLFR_IO, "cannot open %s.header", path); }
    }
    fprintf(fph, "Version 1.3\n");
    fprintf(fph, "Width %d\n", b->W);
    fprintf(fph, "Height %d\n", b->H);
    fprintf(fph, "Samples per pixel %d\n", b->spp);
    fprintf(fph, "CoC coefficients (coc radius = C0/w+C1): %f,%f\n", b->coc[0], b->coc[1]);
    fprintf(fph, "Encoding = %s\n", binary ? "binary" : "text");
    fprintf(fph, "x,y,z/w,w,u,v,t,r,g,b,a,mv_x,mv_y,mv_w,dwdx,dwdy\n");
    const size_t n = (size_t)b->W * b->H * b->spp;
    bool ok = true;
    if (binary)
    {
        std::vector<float> tmp(b->rec, b->rec + 16 * n);
        for (size_t k = 0; k < n; k++)
            tmp[k * 16 + 10] = tmp[k * 16 + 9];
        ok = fwrite(tmp.data(), 64, n, fp) == n;
    }
    else
    {
        for (size_t k = 0; k < n && ok; k++)
        {
            const float* e = &b->rec[k * 16];
            for (int v = 0; v < 16; v++)
                fprintf(fp, "%f,", (v == 10) ? e[9] : e[v]);
            fprintf(fp, "\n");
        }
        ok = !ferror(fp);
    }
    fflush(fp);
    fclose(fp);
    if (separate_header) { fflush(fph); fclose(fph); }
    return ok ? TLFR_OK : fail(nullptr, TLFR_IO, "write failed: %s", path);
}

tlfr_status tlfr_buffer_info(const tlfr_buffer* b, int* W, int* H, int* spp, float* c0, float* c1)
{
    if (!b)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_buffer_info: null buffer");
    if (W) *W = b->W;
    if (H) *H = b->H;
    if (spp) *spp = b->spp;
    if (c0) *c0 = b->coc[0];
    if (c1) *c1 = b->coc[1];
    return TLFR_OK;
}

const float* tlfr_buffer_records(const tlfr_buffer* b) { return b ? b->rec : nullptr; }
void tlfr_buffer_free(tlfr_buffer* b) { delete b; }

tlfr_status tlfr_create(const tlfr_buffer* buf, const tlfr_params* params, void* stream, tlfr_ctx** out)
{
    if (!buf || !out)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_create: bad argument");
    tlfr_ctx* ctx = nullptr;
    tlfr_status st = begin_ctx(params, stream, buf->W, buf->H, buf->spp, buf->coc[0], buf->coc[1], out, ctx);
    if (st != TLFR_OK)
    {
        if (ctx) { g_create_error = ctx->c.error; free_ctx_buffers(ctx->c); delete ctx; }
        return st;
    }
    tlfr::Ctx& c = ctx->c;
    cudaError_t e = cudaMalloc(&c.d_records, sizeof(float) * 16 * c.n_in);
    if (e == cudaSuccess)
    {
        c.own_records = true;
        e = cudaMemcpyAsync(c.d_records, buf->rec, sizeof(float) * 16 * c.n_in, cudaMemcpyHostToDevice, c.stream);
    }
    if (e != cudaSuccess)
    {
        g_create_error = std::string("record upload: ") + cudaGetErrorString(e);
        free_ctx_buffers(c); delete ctx;
        return e == cudaErrorMemoryAllocation ? TLFR_OOM : TLFR_CUDA;
    }
    st = run_build(ctx, c.d_records);
    if (st != TLFR_OK)
    {
        g_create_error = c.error;
        free_ctx_buffers(c); delete ctx;
        return st;
    }
    *out = ctx;
    return TLFR_OK;
}

tlfr_status tlfr_create_device(const float* d_rec, int W, int H, int spp, float c0, float c1,
                               const tlfr_params* params, void* stream, tlfr_ctx** out)
{
    if (!d_rec || !out)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_create_device: bad argument");
    tlfr_ctx* ctx = nullptr;
    tlfr_status st = begin_ctx(params, stream, W, H, spp, c0, c1, out, ctx);
    if (st != TLFR_OK)
    {
        if (ctx) { g_create_error = ctx->c.error; free_ctx_buffers(ctx->c); delete ctx; }
        return st;
    }
    st = run_build(ctx, d_rec);
    if (st != TLFR_OK)
    {
        g_create_error = ctx->c.error;
        free_ctx_buffers(ctx->c); delete ctx;
        return st;
    }
    *out = ctx;
    return TLFR_OK;
}

tlfr_status tlfr_rebuild_device(tlfr_ctx* ctx, const float* d_rec)
{
    if (!ctx || !d_rec)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_rebuild_device: bad argument");
    cudaSetDevice(ctx->c.device);
    return run_build(ctx, d_rec);
}

tlfr_status tlfr_rebuild(tlfr_ctx* ctx, const tlfr_buffer* buf)
{
    if (!ctx || !buf)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_rebuild: bad argument");
    tlfr::Ctx& c = ctx->c;
    if (buf->W != c.W || buf->H != c.H || buf->spp != c.spp_in || buf->coc[0] != c.coc0_raw[0] ||
        buf->coc[1] != c.coc0_raw[1])
        return fail(ctx, TLFR_BAD_ARG, "tlfr_rebuild: buffer size or CoC coefficients differ from the context's");
    cudaSetDevice(c.device);
    cudaError_t e = cudaSuccess;
    if (!c.d_records || !c.own_records)
    {
        e = cudaMalloc(&c.d_records, sizeof(float) * 16 * c.n_in);
        if (e != cudaSuccess)
            return fail(ctx, TLFR_OOM, "record allocation: %s", cudaGetErrorString(e));
        c.own_records = true;
    }
    e = cudaMemcpyAsync(c.d_records, buf->rec, sizeof(float) * 16 * c.n_in, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "record upload: %s", cudaGetErrorString(e));
    return run_build(ctx, c.d_records);
}

tlfr_status tlfr_reconstruct(tlfr_ctx* ctx, float* rgba, int rgba_on_device, tlfr_stats* stats)
{
    if (!ctx || !rgba)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_reconstruct: bad argument");
    tlfr::Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    const size_t npix = (size_t)c.W * c.H;
    float4* dst = reinterpret_cast<float4*>(rgba);
    if (!rgba_on_device)
    {
        if (!c.d_out)
        {
            cudaError_t e = cudaMalloc(&c.d_out, sizeof(float4) * npix);
            if (e != cudaSuccess)
                return fail(ctx, TLFR_OOM, "output allocation: %s", cudaGetErrorString(e));
        }
        dst = c.d_out;
    }
    cudaEventRecord(c.ev1, c.stream);
    const long long l0 = c.launches;
    tlfr_status st = tlfr::reconstruct_frame(c, dst, stats != nullptr);
    c.last.query_launches = (double)(c.launches - l0);
    cudaEventRecord(c.ev2, c.stream);
    if (st != TLFR_OK)
        return st;
    if (!rgba_on_device)
    {
        cudaError_t e = cudaMemcpyAsync(rgba, dst, sizeof(float4) * npix, cudaMemcpyDeviceToHost, c.stream);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess)
            return fail(ctx, TLFR_CUDA, "reconstruct: %s", cudaGetErrorString(e));
    }
    if (stats)
    {
        cudaError_t e = cudaEventSynchronize(c.ev2);
        if (e != cudaSuccess)
            return fail(ctx, TLFR_CUDA, "reconstruct: %s", cudaGetErrorString(e));
        float ms = 0;
        cudaEventElapsedTime(&ms, c.ev1, c.ev2);
        c.last.query_ms = ms;
        *stats = c.last;
    }
    return TLFR_OK;
}

tlfr_status tlfr_set_output(tlfr_ctx* ctx, const tlfr_params* params)
{
    if (!ctx || !params)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_set_output: bad argument");
    cudaSetDevice(ctx->c.device);
    ctx->c.params.override_uvt = params->override_uvt;
    memcpy(ctx->c.params.uvt, params->uvt, sizeof(params->uvt));
    ctx->c.params.output_spp = params->output_spp;
    ctx->c.params.lens_filter = params->lens_filter;
    ctx->c.params.time_filter = params->time_filter;
    return upload_pattern(ctx);
}

tlfr_status tlfr_trim(tlfr_ctx* ctx)
{
    if (!ctx)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_trim: null context");
    cudaSetDevice(ctx->c.device);
    const tlfr_status st = tlfr::release_build_scratch(ctx->c);
    return st == TLFR_OK ? TLFR_OK : fail(ctx, st, "tlfr_trim: %s", ctx->c.error.c_str());
}

tlfr_status tlfr_sync(tlfr_ctx* ctx)
{
    if (!ctx)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_sync: null context");
    cudaError_t e = cudaStreamSynchronize(ctx->c.stream);
    return e == cudaSuccess ? TLFR_OK : fail(ctx, TLFR_CUDA, "%s", cudaGetErrorString(e));
}

tlfr_status tlfr_get_stats(tlfr_ctx* ctx, tlfr_stats* stats)
{
    if (!ctx || !stats)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_get_stats: bad argument");
    *stats = ctx->c.last;
    return TLFR_OK;
}

void tlfr_destroy(tlfr_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    free_ctx_buffers(ctx->c);
    delete ctx;
}

const char* tlfr_last_error(const tlfr_ctx* ctx)
{
    return ctx ? ctx->c.error.c_str() : g_create_error.c_str();
}

tlfr_status tlfr_tree_info(tlfr_ctx* ctx, int* num_nodes, int* num_samples, int* root, int* height)
{
    if (!ctx)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_tree_info: null context");
    if (num_nodes) *num_nodes = ctx->c.num_nodes;
    if (num_samples) *num_samples = ctx->c.num_samples;
    if (root) *root = ctx->c.root;
    if (height) *height = ctx->c.height;
    return TLFR_OK;
}

tlfr_status tlfr_tree_export(tlfr_ctx* ctx, float* nodef, int* nodei, float* samplef, int* sample_ids)
{
    if (!ctx)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_tree_export: null context");
    tlfr::Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    const int nn = c.num_nodes, ns = c.num_samples;
    std::vector<tlfr::QNode> q(nn);
    std::vector<float2> ts(nn);
    std::vector<float4> rec2(2 * (size_t)ns), col(ns);
    std::vector<int> id(ns);
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemcpy(q.data(), c.nodes, sizeof(tlfr::QNode) * nn, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(ts.data(), c.node_tspan, sizeof(float2) * nn, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(rec2.data(), c.s_rec, sizeof(float4) * 2 * ns, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(col.data(), c.s_col, sizeof(float4) * ns, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(id.data(), c.s_id, sizeof(int) * ns, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "tree export: %s", cudaGetErrorString(e));
    for (int i = 0; i < nn; i++)
    {
        const tlfr::QNode& n = q[i];
        if (nodef)
        {
            float* f = nodef + (size_t)i * 14;
            f[0] = n.a.x; f[1] = n.a.y; f[2] = n.a.z; f[3] = n.a.w;
            f[4] = n.b.x; f[5] = n.b.y; f[6] = n.b.z; f[7] = n.b.w;
            f[8] = n.c.x; f[9] = n.c.y; f[10] = n.c.z; f[11] = n.c.w;
            f[12] = ts[i].x; f[13] = ts[i].y;
        }
        if (nodei)
        {
            int* d = nodei + (size_t)i * 5;
            const bool leaf = n.d.x < 0;
            d[0] = leaf ? -1 : n.d.x;
            d[1] = leaf ? -1 : n.d.y;
            d[2] = leaf ? n.d.z : -1;
            d[3] = leaf ? n.d.w : -1;
            d[4] = 0;
        }
    }
    if (nodei)
    {
        // sample counts: leaves directly, internal nodes by a post-order pass from the root
        std::vector<int> order;
        order.reserve(nn);
        std::vector<int> stack{ c.root };
        while (!stack.empty())
        {
            int i = stack.back(); stack.pop_back();
            order.push_back(i);
            if (q[i].d.x >= 0) { stack.push_back(q[i].d.x); stack.push_back(q[i].d.y); }
        }
        for (auto it = order.rbegin(); it != order.rend(); ++it)
        {
            int i = *it;
            int* d = nodei + (size_t)i * 5;
            d[4] = (q[i].d.x < 0) ? (q[i].d.w - q[i].d.z) : (nodei[(size_t)q[i].d.x * 5 + 4] + nodei[(size_t)q[i].d.y * 5 + 4]);
        }
    }
    for (int j = 0; j < ns; j++)
    {
        if (samplef)
        {
            float* f = samplef + (size_t)j * 12;
            const float4& p = rec2[2 * (size_t)j];
            const float4& m = rec2[2 * (size_t)j + 1];
            f[0] = p.x; f[1] = p.y; f[2] = p.z; f[3] = p.w;
            f[4] = m.x; f[5] = m.y; f[6] = m.z;
            f[7] = col[j].x; f[8] = col[j].y; f[9] = col[j].z; f[10] = col[j].w;
            f[11] = p.z;     // key = w after reprojection (Reconstruction.hpp:119)
        }
        if (sample_ids) sample_ids[j] = id[j];
    }
    return TLFR_OK;
}

int tlfr_output_samples(tlfr_ctx* ctx, float* out5)
{
    if (!ctx)
        return -1;
    if (out5)
        memcpy(out5, ctx->c.h_pattern.data(), sizeof(float) * ctx->c.h_pattern.size());
    return (int)(ctx->c.h_pattern.size() / 5);
}

// TreeGather::reconstructShadows (Reconstruction.cpp:302-344) for a flat list of
// light-space query samples.
// Motion and defocus with soft shadows (TreeGather::reconstructDofMotionShadows,
// Reconstruction.cpp:355-433).
tlfr_status tlfr_reconstruct_dof_motion_shadows(tlfr_ctx* camera, const tlfr_view* camera_view,
                                                const float* camera_density, tlfr_ctx* light,
                                                const tlfr_view* light_view, float* rgba, int rgba_on_device)
{
    if (!camera || !light || !camera_view || !light_view || !rgba || camera == light)
        return fail(camera, TLFR_BAD_ARG, "tlfr_reconstruct_dof_motion_shadows: bad argument");
    tlfr::Ctx& c = camera->c;
    tlfr::Ctx& l = light->c;
    if (c.params.enable_cuda || l.params.enable_cuda)
        return fail(camera, TLFR_BAD_ARG, "tlfr_reconstruct_dof_motion_shadows: the Filterer only (enable_cuda = 0)");
    if (c.W != l.W || c.H != l.H)
        return fail(camera, TLFR_BAD_ARG, "TreeGather::FilterTask::process2 -- cw!=lw || ch!=lh");
    if (c.device != l.device)
        return fail(camera, TLFR_BAD_ARG, "tlfr_reconstruct_dof_motion_shadows: contexts on different devices");
    cudaSetDevice(c.device);
    tlfr::DmsView v;
    derive_dms_view(*camera_view, *light_view, c.W, c.H, c.out_spp, v);
    const size_t npix = (size_t)c.W * c.H;
    const size_t nrec = npix * (size_t)c.spp_in;
    float* d_density = nullptr;
    float4* d_img = rgba_on_device ? reinterpret_cast<float4*>(rgba) : nullptr;
    tlfr_status st = TLFR_OK;
    if (camera_density && cudaMalloc(&d_density, sizeof(float) * nrec) != cudaSuccess)
        st = fail(camera, TLFR_OOM, "tlfr_reconstruct_dof_motion_shadows: allocation failed");
    if (st == TLFR_OK && !d_img && cudaMalloc(&d_img, sizeof(float4) * npix) != cudaSuccess)
        st = fail(camera, TLFR_OOM, "tlfr_reconstruct_dof_motion_shadows: allocation failed");
    if (st == TLFR_OK && camera_density &&
        cudaMemcpyAsync(d_density, camera_density, sizeof(float) * nrec, cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
        st = fail(camera, TLFR_CUDA, "tlfr_reconstruct_dof_motion_shadows: upload failed");
    if (st == TLFR_OK)
    {
        st = tlfr::reconstruct_dof_motion_shadows(c, l, v, d_density, d_img);
        if (st != TLFR_OK)
            st = fail(camera, st, "tlfr_reconstruct_dof_motion_shadows: %s", c.error.c_str());
    }
    if (st == TLFR_OK && !rgba_on_device)
    {
        if (cudaMemcpyAsync(rgba, d_img, sizeof(float4) * npix, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
            cudaStreamSynchronize(c.stream) != cudaSuccess)
            st = fail(camera, TLFR_CUDA, "tlfr_reconstruct_dof_motion_shadows: download failed");
    }
    cudaFree(d_density);
    if (!rgba_on_device)
        cudaFree(d_img);
    return st;
}

tlfr_status tlfr_reconstruct_shadows(tlfr_ctx* ctx, const float* queries16, int n, const float* density, float* rgba)
{
    if (!ctx || n < 0 || (n > 0 && (!queries16 || !rgba)))
        return fail(ctx, TLFR_BAD_ARG, "tlfr_reconstruct_shadows: bad argument");
    tlfr::Ctx& c = ctx->c;
    if (c.params.enable_cuda)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_reconstruct_shadows: the Filterer only (enable_cuda = 0)");
    if (n == 0)
        return TLFR_OK;
    cudaSetDevice(c.device);
    std::vector<float> q8((size_t)n * 8);
    for (int k = 0; k < n; k++)
    {
        const float* e = queries16 + (size_t)k * 16;
        float* d = &q8[(size_t)k * 8];
        d[0] = e[0]; d[1] = e[1]; d[2] = e[4]; d[3] = e[5]; d[4] = e[6]; d[5] = e[3];
        d[6] = density ? density[k] : 1.0f;
        d[7] = 0.0f;
    }
    float* d_q = nullptr;
    float4* d_out = nullptr;
    if (cudaMalloc(&d_q, sizeof(float) * q8.size()) != cudaSuccess ||
        cudaMalloc(&d_out, sizeof(float4) * (size_t)n) != cudaSuccess)
    {
        cudaFree(d_q);
        return fail(ctx, TLFR_OOM, "tlfr_reconstruct_shadows: allocation failed");
    }
    tlfr_status st = TLFR_OK;
    if (cudaMemcpyAsync(d_q, q8.data(), sizeof(float) * q8.size(), cudaMemcpyHostToDevice, c.stream) != cudaSuccess)
        st = fail(ctx, TLFR_CUDA, "tlfr_reconstruct_shadows: upload failed");
    if (st == TLFR_OK)
    {
        st = tlfr::reconstruct_shadows(c, d_q, n, d_out);
        if (st != TLFR_OK)
            st = fail(ctx, st, "tlfr_reconstruct_shadows: %s", c.error.c_str());
    }
    if (st == TLFR_OK)
    {
        if (cudaMemcpyAsync(rgba, d_out, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
            cudaStreamSynchronize(c.stream) != cudaSuccess)
            st = fail(ctx, TLFR_CUDA, "tlfr_reconstruct_shadows: download failed");
    }
    cudaFree(d_q);
    cudaFree(d_out);
    return st;
}

// The reconstruction's output-sample buffer (the m_obuf debug dump,
// Reconstruction.cpp:290-294, 696-712): one record per output sample (x, y, i)
// with the sample's position, lens and time coordinates and its reconstructed
// colour, the rest of the record as a fresh buffer holds it (w = 1, no motion).
tlfr_status tlfr_output_sample_buffer(tlfr_ctx* ctx, tlfr_buffer** out)
{
    if (!ctx || !out)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_output_sample_buffer: bad argument");
    tlfr::Ctx& c = ctx->c;
    const int M = c.out_spp;
    const size_t n = (size_t)c.W * c.H * M;
    if (!c.qcol || c.qcol_cap < n)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_output_sample_buffer: no reconstruction yet");
    cudaSetDevice(c.device);
    std::vector<float> col(4 * n);
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e == cudaSuccess)
        e = cudaMemcpy(col.data(), c.qcol, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "tlfr_output_sample_buffer: %s", cudaGetErrorString(e));
    tlfr_buffer* b = new (std::nothrow) tlfr_buffer();
    if (!b)
        return fail(ctx, TLFR_OOM, "host allocation failed");
    b->W = c.W; b->H = c.H; b->spp = M;
    b->coc[0] = c.coc[0]; b->coc[1] = c.coc[1];
    if (!b->alloc(n))
    {
        delete b;
        return fail(ctx, TLFR_OOM, "host allocation failed");
    }
    for (int y = 0; y < c.H; y++)
        for (int x = 0; x < c.W; x++)
        {
            const int pattern = (int)(tlfr::hash_bits((uint32_t)x, (uint32_t)y) % 64u);
            for (int i = 0; i < M; i++)
            {
                const size_t k = ((size_t)y * c.W + x) * M + i;
                const float* o = &c.h_pattern[((size_t)pattern * M + i) * 5];
                float* r = b->rec + 16 * k;
                r[0] = o[0] + (float)x; r[1] = o[1] + (float)y;
                r[2] = 1.0f; r[3] = 1.0f;
                r[4] = o[2]; r[5] = o[3]; r[6] = o[4];
                r[7] = col[4 * k]; r[8] = col[4 * k + 1]; r[9] = col[4 * k + 2]; r[10] = col[4 * k + 3];
                r[11] = r[12] = r[13] = r[14] = r[15] = 0.0f;
            }
        }
    *out = b;
    return TLFR_OK;
}

tlfr_status tlfr_query_samples_noalloc(tlfr_ctx* ctx, const int* d_xyi, int n, float* d_rgba, int* d_overflow)
{
    if (!ctx || (n > 0 && (!d_xyi || !d_rgba)))
        return fail(ctx, TLFR_BAD_ARG, "tlfr_query_samples_noalloc: bad argument");
    if (ctx->c.params.enable_cuda)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_query_samples_noalloc: the Filterer only (enable_cuda = 0)");
    tlfr::Ctx& c = ctx->c;
    cudaError_t e = cudaSetDevice(c.device);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "tlfr_query_samples_noalloc: %s", cudaGetErrorString(e));
    return tlfr::query_samples_noalloc(c, d_xyi, n, d_rgba, d_overflow);
}

tlfr_status tlfr_trace_queries(tlfr_ctx* ctx, const int* xyi, int n, float* rgba, int* trace, int stride)
{
    if (!ctx || (n > 0 && (!xyi || !rgba || !trace || stride < 2)))
        return fail(ctx, TLFR_BAD_ARG, "tlfr_trace_queries: bad argument");
    if (ctx->c.params.enable_cuda)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_trace_queries: traces follow the Filterer (enable_cuda = 0)");
    tlfr::Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    for (int k = 0; k < n; k++)
        if (xyi[3 * k] < 0 || xyi[3 * k] >= c.W || xyi[3 * k + 1] < 0 || xyi[3 * k + 1] >= c.H ||
            xyi[3 * k + 2] < 0 || xyi[3 * k + 2] >= c.out_spp)
            return fail(ctx, TLFR_BAD_ARG, "tlfr_trace_queries: query %d out of range", k);
    return tlfr::trace_queries(c, xyi, n, rgba, trace, stride);
}

/* ---- learned routing ------------------------------------------------------ */

struct tlfr_router
{
    tlfr::Route r;
};

tlfr_status tlfr_route_features(tlfr_ctx* ctx, float* d_feats)
{
    if (!ctx || !d_feats)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_route_features: bad argument");
    tlfr::Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    std::string err;
    tlfr_status st = tlfr::route_features(c, d_feats, err);
    if (st != TLFR_OK)
        return fail(ctx, st, "tlfr_route_features: %s", err.c_str());
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "tlfr_route_features: %s", cudaGetErrorString(e));
    return TLFR_OK;
}

tlfr_status tlfr_route_labels(tlfr_ctx* ctx, float tol, float* d_labels, float* d_rgba)
{
    return tlfr_route_labels_ref(ctx, nullptr, tol, d_labels, d_rgba);
}

tlfr_status tlfr_route_labels_ref(tlfr_ctx* ctx, const float* d_ref, float tol, float* d_labels, float* d_rgba)
{
    if (!ctx || !d_labels || !d_rgba || !(tol >= 0.0f))
        return fail(ctx, TLFR_BAD_ARG, "tlfr_route_labels: bad argument");
    tlfr::Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    const size_t npix = (size_t)c.W * c.H;
    if (!c.route_img)
    {
        cudaError_t e = cudaMalloc(&c.route_img, sizeof(float4) * npix);
        if (e != cudaSuccess)
            return fail(ctx, TLFR_OOM, "tlfr_route_labels: %s", cudaGetErrorString(e));
    }
    tlfr::Route* saved = c.router;
    c.router = nullptr;
    tlfr_status st = tlfr::reconstruct_frame(c, reinterpret_cast<float4*>(d_rgba), false);
    if (st == TLFR_OK)
    {
        c.route_all_fast = true;
        st = tlfr::reconstruct_frame(c, c.route_img, false);
        c.route_all_fast = false;
    }
    c.router = saved;
    if (st != TLFR_OK)
        return fail(ctx, st, "tlfr_route_labels: %s", c.error.c_str());
    std::string err;
    st = tlfr::route_labels_from(c, reinterpret_cast<const float4*>(d_rgba), c.route_img,
                                 reinterpret_cast<const float4*>(d_ref), tol, d_labels, err);
    if (st != TLFR_OK)
        return fail(ctx, st, "tlfr_route_labels: %s", err.c_str());
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess)
        return fail(ctx, TLFR_CUDA, "tlfr_route_labels: %s", cudaGetErrorString(e));
    return TLFR_OK;
}

tlfr_status tlfr_router_create(int device, void* stream, unsigned seed, const float* mean8, const float* inv_std8,
                               tlfr_router** out)
{
    if (!out)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_router_create: bad argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, TLFR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev)
        return fail(nullptr, TLFR_BAD_ARG, "tlfr_router_create: device %d out of range", device);
    cudaSetDevice(device);
    tlfr_router* r = new (std::nothrow) tlfr_router;
    if (!r)
        return fail(nullptr, TLFR_OOM, "host allocation failed");
    r->r.device = device;
    r->r.stream = static_cast<cudaStream_t>(stream);
    std::string err;
    tlfr_status st = tlfr::route_alloc(r->r, err);
    if (st == TLFR_OK)
        st = tlfr::route_init(r->r, seed, mean8, inv_std8, r->r.stream, err);
    if (st != TLFR_OK)
    {
        g_create_error = err;
        tlfr::route_free(r->r);
        delete r;
        return st;
    }
    *out = r;
    return TLFR_OK;
}

void tlfr_router_destroy(tlfr_router* r)
{
    if (!r)
        return;
    cudaSetDevice(r->r.device);
    tlfr::route_free(r->r);
    delete r;
}

const char* tlfr_router_last_error(const tlfr_router* r) { return r ? r->r.error.c_str() : g_create_error.c_str(); }

int tlfr_router_num_params(void) { return tlfr::route_num_params(); }

#define ROUTER_CALL(name, expr)                                                       \
    do {                                                                              \
        cudaSetDevice(r->r.device);                                                   \
        std::string err;                                                              \
        tlfr_status st = (expr);                                                      \
        if (st != TLFR_OK)                                                            \
            r->r.error = std::string(name) + ": " + err;                              \
        return st;                                                                    \
    } while (0)

tlfr_status tlfr_router_train(tlfr_router* r, const float* d_feats, const float* d_labels, int n, int steps, int batch,
                              float lr, unsigned seed, float* final_loss)
{
    if (!r || !d_feats || !d_labels || n <= 0 || steps < 0 || batch <= 0)
        return r ? (r->r.error = "tlfr_router_train: bad argument", TLFR_BAD_ARG) : TLFR_BAD_ARG;
    ROUTER_CALL("tlfr_router_train",
                tlfr::route_train(r->r, d_feats, d_labels, n, steps, batch, lr, seed, final_loss, r->r.stream, err));
}

tlfr_status tlfr_router_gradient(tlfr_router* r, const float* d_feats, const float* d_labels, int n, float* grad,
                                 float* loss)
{
    if (!r || !d_feats || !d_labels || n <= 0 || !grad)
        return r ? (r->r.error = "tlfr_router_gradient: bad argument", TLFR_BAD_ARG) : TLFR_BAD_ARG;
    ROUTER_CALL("tlfr_router_gradient",
                tlfr::route_gradient(r->r, d_feats, d_labels, n, grad, loss, r->r.stream, err));
}

tlfr_status tlfr_router_predict(tlfr_router* r, const float* d_feats, long long n, float* d_prob)
{
    if (!r || !d_feats || n <= 0 || !d_prob)
        return r ? (r->r.error = "tlfr_router_predict: bad argument", TLFR_BAD_ARG) : TLFR_BAD_ARG;
    cudaSetDevice(r->r.device);
    std::string err;
    tlfr_status st = tlfr::route_predict(r->r, d_feats, n, d_prob, r->r.stream, err);
    if (st == TLFR_OK && cudaStreamSynchronize(r->r.stream) != cudaSuccess)
    {
        err = cudaGetErrorString(cudaGetLastError());
        st = TLFR_CUDA;
    }
    if (st != TLFR_OK)
        r->r.error = "tlfr_router_predict: " + err;
    return st;
}

tlfr_status tlfr_router_get_params(tlfr_router* r, float* params)
{
    if (!r || !params)
        return r ? (r->r.error = "tlfr_router_get_params: bad argument", TLFR_BAD_ARG) : TLFR_BAD_ARG;
    ROUTER_CALL("tlfr_router_get_params", tlfr::route_get_params(r->r, params, r->r.stream, err));
}

tlfr_status tlfr_router_set_params(tlfr_router* r, const float* params)
{
    if (!r || !params)
        return r ? (r->r.error = "tlfr_router_set_params: bad argument", TLFR_BAD_ARG) : TLFR_BAD_ARG;
    ROUTER_CALL("tlfr_router_set_params", tlfr::route_set_params(r->r, params, r->r.stream, err));
}

tlfr_status tlfr_set_routing(tlfr_ctx* ctx, tlfr_router* r, float threshold)
{
    if (!ctx || (r && !(threshold >= 0.0f && threshold < 1.0f)))
        return fail(ctx, TLFR_BAD_ARG, "tlfr_set_routing: bad argument");
    if (r && r->r.device != ctx->c.device)
        return fail(ctx, TLFR_BAD_ARG, "tlfr_set_routing: router and context are on different devices");
    ctx->c.router = r ? &r->r : nullptr;
    ctx->c.route_hi = threshold;
    return TLFR_OK;
}

/* ---- batches of frames (one CUDA graph) ------------------------------------ */

struct tlfr_batch
{
    std::vector<tlfr_ctx*> ctx;
    tlfr::BatchPlan* plan = nullptr;
    std::vector<tlfr_params> outputs;   // per-frame output settings (kept alive for the plan)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long launches = 0;             // kernel launches of one run
    std::string error;
};

static tlfr_status batch_fail(tlfr_batch* b, tlfr_status st, const std::string& msg)
{
    if (b)
        b->error = msg;
    else
        g_create_error = msg;
    return st;
}

static void batch_free(tlfr_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    tlfr::batch_plan_delete(b->plan);
    delete b;
}

tlfr_status tlfr_batch_create_frames(const tlfr_batch_frame* frames, int n, void* stream, int autotune,
                                     size_t budget_bytes, tlfr_batch** out)
{
    if (!frames || n <= 0 || !out)
        return batch_fail(nullptr, TLFR_BAD_ARG, "tlfr_batch_create: bad argument");
    for (int i = 0; i < n; i++)
        if (!frames[i].ctx || !frames[i].d_rgba)
            return batch_fail(nullptr, TLFR_BAD_ARG, "tlfr_batch_create: null context or output " + std::to_string(i));
    for (int i = 0; i < n; i++)
        if (frames[i].ctx->c.params.enable_cuda)
            return batch_fail(nullptr, TLFR_BAD_ARG, "tlfr_batch_create: frame " + std::to_string(i) +
                                                         " uses the GPU-toggle algorithm (enable_cuda), which batches "
                                                         "do not run");
    const int dev = frames[0].ctx->c.device;
    for (int i = 1; i < n; i++)
        if (frames[i].ctx->c.device != dev)
            return batch_fail(nullptr, TLFR_BAD_ARG, "tlfr_batch_create: contexts on different devices");
    cudaSetDevice(dev);
    tlfr_batch* b = new (std::nothrow) tlfr_batch;
    if (!b)
        return batch_fail(nullptr, TLFR_OOM, "host allocation failed");
    b->device = dev;
    b->plan = tlfr::batch_plan_new();
    if (!b->plan)
    {
        delete b;
        return batch_fail(nullptr, TLFR_OOM, "host allocation failed");
    }
    b->outputs.resize(n);
    std::vector<tlfr::BatchEntry> entries(n);
    for (int i = 0; i < n; i++)
    {
        b->ctx.push_back(frames[i].ctx);
        if (frames[i].output)
            b->outputs[i] = *frames[i].output;
        entries[i].ctx = &frames[i].ctx->c;
        entries[i].output = frames[i].output ? &b->outputs[i] : nullptr;
        entries[i].out = reinterpret_cast<float4*>(frames[i].d_rgba);
    }
    b->stream = static_cast<cudaStream_t>(stream);
    if (!b->stream)
    {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        {
            batch_free(b);
            return batch_fail(nullptr, TLFR_CUDA, "tlfr_batch_create: stream creation failed");
        }
        b->own_stream = true;
    }
    auto cuda_fail = [&](const char* what, cudaError_t e) {
        const std::string m = std::string("tlfr_batch_create: ") + what + ": " + cudaGetErrorString(e);
        batch_free(b);
        return batch_fail(nullptr, TLFR_CUDA, m);
    };
    std::string err;
    tlfr_status st = TLFR_OK;
    // the batch only queries its contexts: their build working storage goes
    for (int i = 0; i < n && st == TLFR_OK; i++)
    {
        bool seen = false;
        for (int j = 0; j < i; j++)
            seen = seen || frames[j].ctx == frames[i].ctx;
        if (!seen)
            st = tlfr::release_build_scratch(frames[i].ctx->c);
    }
    if (st != TLFR_OK)
    {
        const std::string m = frames[0].ctx->c.error;
        batch_free(b);
        return batch_fail(nullptr, st, "tlfr_batch_create: " + m);
    }
    if (budget_bytes == 0)
    {
        // default: half of the free device memory, at most 32 GiB
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        budget_bytes = std::min<size_t>(fr / 2, (size_t)32 << 30);
    }
    st = tlfr::batch_build(*b->plan, entries, b->stream, autotune != 0, budget_bytes, err);
    if (st != TLFR_OK)
    {
        batch_free(b);
        return batch_fail(nullptr, st, "tlfr_batch_create: " + err);
    }
    // one eager run (lazy scratch of the router), then the capture
    for (int pass = 0; pass < 2; pass++)
    {
        cudaError_t e = cudaSuccess;
        if (pass == 1 && (e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail("cudaStreamBeginCapture", e);
        st = tlfr::batch_enqueue(*b->plan, b->stream, err, &b->launches);
        if (st != TLFR_OK)
        {
            if (pass == 1)
            {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(b->stream, &g);
                if (g) cudaGraphDestroy(g);
            }
            batch_free(b);
            return batch_fail(nullptr, st, "tlfr_batch_create: " + err);
        }
        if (pass == 0 && (e = cudaStreamSynchronize(b->stream)) != cudaSuccess)
            return cuda_fail("warm-up run", e);
        if (pass == 1)
        {
            if ((e = cudaStreamEndCapture(b->stream, &b->graph)) != cudaSuccess)
                return cuda_fail("cudaStreamEndCapture", e);
            if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
                return cuda_fail("cudaGraphInstantiate", e);
        }
    }
    if (cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess)
        return cuda_fail("cudaEventCreate", cudaGetLastError());
    *out = b;
    return TLFR_OK;
}

tlfr_status tlfr_batch_create(tlfr_ctx* const* ctxs, int n, float* const* d_rgba, void* stream, int autotune,
                              tlfr_batch** out)
{
    if (!ctxs || !d_rgba || n <= 0 || !out)
        return batch_fail(nullptr, TLFR_BAD_ARG, "tlfr_batch_create: bad argument");
    std::vector<tlfr_batch_frame> fr(n);
    for (int i = 0; i < n; i++)
        fr[i] = tlfr_batch_frame{ ctxs[i], nullptr, d_rgba[i] };
    return tlfr_batch_create_frames(fr.data(), n, stream, autotune, 0, out);
}

tlfr_status tlfr_batch_run(tlfr_batch* b)
{
    if (!b)
        return TLFR_BAD_ARG;
    cudaSetDevice(b->device);
    cudaError_t e = cudaEventRecord(b->ev0, b->stream);
    if (e == cudaSuccess)
        e = cudaGraphLaunch(b->exec, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->ev1, b->stream);
    if (e != cudaSuccess)
        return batch_fail(b, TLFR_CUDA, std::string("tlfr_batch_run: ") + cudaGetErrorString(e));
    return TLFR_OK;
}

tlfr_status tlfr_batch_sync(tlfr_batch* b, double* ms)
{
    if (!b)
        return TLFR_BAD_ARG;
    cudaSetDevice(b->device);
    cudaError_t e = cudaEventSynchronize(b->ev1);
    if (e != cudaSuccess)
        return batch_fail(b, TLFR_CUDA, std::string("tlfr_batch_sync: ") + cudaGetErrorString(e));
    if (ms)
    {
        float f = 0;
        cudaEventElapsedTime(&f, b->ev0, b->ev1);
        *ms = f;
    }
    std::vector<int> hard;
    std::string err;
    if (tlfr::batch_failures(*b->plan, b->stream, hard, err) != TLFR_OK)
        return batch_fail(b, TLFR_CUDA, "tlfr_batch_sync: " + err);
    for (size_t i = 0; i < hard.size(); i++)
        if (hard[i] > 0)
            return batch_fail(b, TLFR_OVERFLOW, "tlfr_batch_sync: frame " + std::to_string(i) +
                                                    ": a query exceeded the largest supported capacity");
    return TLFR_OK;
}

tlfr_status tlfr_batch_info(const tlfr_batch* b, int* tile_shapes)
{
    if (!b || !tile_shapes)
        return TLFR_BAD_ARG;
    tlfr::batch_info(*b->plan, tile_shapes, nullptr);
    return TLFR_OK;
}

tlfr_status tlfr_batch_layout(const tlfr_batch* b, int* chunks, long long* launches)
{
    if (!b)
        return TLFR_BAD_ARG;
    if (chunks)
        tlfr::batch_info(*b->plan, nullptr, chunks);
    if (launches)
        *launches = b->launches;
    return TLFR_OK;
}

const char* tlfr_batch_last_error(const tlfr_batch* b) { return b ? b->error.c_str() : g_create_error.c_str(); }

void tlfr_batch_destroy(tlfr_batch* b)
{
    if (!b)
        return;
    cudaSetDevice(b->device);
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    batch_free(b);
}

} // extern "C"
