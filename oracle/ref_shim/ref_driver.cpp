// C entry points over the reference's own CPU reconstruction (TreeGather,
// reference src/reconstruction_lib/reconstruction/Reconstruction.hpp:42-48),
// built by oracle/build_ref.sh into oracle/_ref/libtlfr_ref*.so.
//
// Test infrastructure only: the tests and bench.py's CPU-baseline leg load this
// library through ctypes to (1) pin the CPU restatement in oracle/tlfr_oracle.c
// and (2) check the CUDA path, query by query and pixel by pixel.
//
// Instrumentation: private members of TreeGather are made visible to this one
// translation unit (the '#define private public' below) so that the built tree,
// the output sampling pattern and per-query surfaces can be read back.  No
// algorithm code is changed; every computation runs in the reference's own
// functions.
#include <cstring>
#include <cstdio>
#include <chrono>
#include <stdexcept>
#include <string>
#include <vector>

#define private public
#define protected public
#include "Reconstruction.hpp"
#include "ref_handle.h"
#undef private
#undef protected

using namespace FW;

namespace
{
std::string g_error;


double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Builds a UVTSampleBuffer from 16-float records laid out pixel-major,
// (y*W+x)*spp+i, with the field order of the reference file format
// (SampleBuffer.cpp:283-286).  Field assignment mirrors the binary loader
// (SampleBuffer.cpp:360-373), alpha forced to 1.
UVTSampleBuffer* buffer_from_records(const float* rec, int W, int H, int spp, float C0, float C1)
{
    UVTSampleBuffer* b = new UVTSampleBuffer();
    b->m_width = W;
    b->m_height = H;
    b->m_numSamplesPerPixel = spp;
    b->m_cocCoeff = Vec2f(C0, C1);
    const int n = W * H * spp;
    b->m_xy.reset(n); b->m_uv.reset(n); b->m_t.reset(n); b->m_color.reset(n);
    b->m_depth.reset(n); b->m_w.reset(n); b->m_mv.reset(n); b->m_wg.reset(n);
    b->m_weight.reset(n);
    for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++)
    for (int i = 0; i < spp; i++)
    {
        const float* e = rec + (size_t)((y * W + x) * spp + i) * 16;
        b->setSampleXY(x, y, i, Vec2f(e[0], e[1]));
        b->setSampleDepth(x, y, i, e[2]);
        b->setSampleW(x, y, i, e[3]);
        b->setSampleUV(x, y, i, Vec2f(e[4], e[5]));
        b->setSampleT(x, y, i, e[6]);
        b->setSampleColor(x, y, i, Vec4f(e[7], e[8], e[9], 1.0f));
        b->setSampleMV(x, y, i, Vec3f(e[11], e[12], e[13]));
        b->setSampleWG(x, y, i, Vec2f(e[14], e[15]));
    }
    return b;
}

int finish_create(RefHandle* h, float aperture, float focus, const float* uvt, int lensFilter, int timeFilter,
                  void** out, double* build_seconds)
{
    h->params = new CameraParams();
    if (uvt)
        h->params->overrideUVT = Vec3f(uvt[0], uvt[1], uvt[2]);
    h->params->lensFilter = (LensFilter)lensFilter;
    h->params->timeFilter = (TimeFilter)timeFilter;
    h->params->enableCuda = false;
    auto t0 = std::chrono::steady_clock::now();
    h->tg = new TreeGather(*h->sbuf, *h->params, aperture, focus);
    if (build_seconds)
        *build_seconds = seconds_since(t0);
    h->tg->generateOutputSamples(*h->params);
    *out = h;
    return 0;
}
} // namespace

#ifdef TLFR_REF_NO_GPU_TOGGLE
// The 64-output-sample variant does not carry the GPU-toggle translation unit
// (ref_gpu_toggle.cpp); CameraParams::enableCuda is always false there.
void TreeGather::cudaReconstruction(Image& resultImage, const CameraParams& params)
{
    (void)resultImage; (void)params;
    fail("TreeGather::cudaReconstruction is not part of this build");
}
#endif

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_num_output_samples_default(void) { return TreeGather::NUM_OUTPUT_SAMPLES; }

// Build the hierarchy from in-memory records (TreeGather ctor, Reconstruction.cpp:43-215).
// uvt: NULL, or the overrideUVT triple (pinhole t=1 is {0,0,1}, App.cpp:450).
int ref_create(const float* records, int W, int H, int spp, float C0, float C1,
               float aperture, float focus, const float* uvt, int lensFilter, int timeFilter,
               void** out, double* build_seconds)
{
    RefHandle* h = new RefHandle();
    try
    {
        h->sbuf = buffer_from_records(records, W, H, spp, C0, C1);
        return finish_create(h, aperture, focus, uvt, lensFilter, timeFilter, out, build_seconds);
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        delete h->tg; delete h->params; delete h->sbuf; delete h;
        return 1;
    }
}

// ref_create with the buffer's LIGHTSPACE_DENSITY channel (one float per record,
// record order), which TreeGather reads into each sample's density
// (Reconstruction.cpp:522, 547).
int ref_create_density(const float* records, int W, int H, int spp, float C0, float C1, const float* density,
                       float aperture, float focus, const float* uvt, int lensFilter, int timeFilter,
                       void** out, double* build_seconds)
{
    RefHandle* h = new RefHandle();
    try
    {
        h->sbuf = buffer_from_records(records, W, H, spp, C0, C1);
        const int cid = h->sbuf->reserveChannel<float>("LIGHTSPACE_DENSITY");
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                for (int i = 0; i < spp; i++)
                    (*(Array<float>*)(h->sbuf->m_channels[cid]))[h->sbuf->getIndex(x, y, i)] =
                        density[((size_t)y * W + x) * spp + i];
        return finish_create(h, aperture, focus, uvt, lensFilter, timeFilter, out, build_seconds);
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        delete h->tg; delete h->params; delete h->sbuf; delete h;
        return 1;
    }
}

// The CameraParams fields the shadowed reconstruction reads (CameraParams.hpp:
// 96-104): projection, the camera's matrices and far plane (row-major 4x4),
// window size, aperture radius, focus distance.
int ref_set_view(void* handle, const float* projection, const float* camera_to_world, const float* world_to_camera,
                 float far_plane, int window_w, int window_h, float aperture_radius, float focus_distance)
{
    RefHandle* h = (RefHandle*)handle;
    Mat4f P, C2W, W2C;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++)
        {
            P(r, c) = projection[4 * r + c];
            C2W(r, c) = camera_to_world[4 * r + c];
            W2C(r, c) = world_to_camera[4 * r + c];
        }
    h->params->projection = P;
    h->params->camera.setMatrices(C2W, W2C);
    h->params->camera.setFar(far_plane);
    h->params->windowSize = Vec2i(window_w, window_h);
    h->params->apertureRadius = aperture_radius;
    h->params->focusDistance = focus_distance;
    return 0;
}

// TreeGather::reconstructDofMotionShadows (Reconstruction.cpp:355-433): camera
// handle, light handle; rgba receives the W*H image.
int ref_reconstruct_dof_motion_shadows(void* camera, void* light, float* rgba)
{
    RefHandle* c = (RefHandle*)camera;
    RefHandle* l = (RefHandle*)light;
    try
    {
        const int W = c->sbuf->getWidth(), H = c->sbuf->getHeight();
        Image img(Vec2i(W, H));
        c->tg->reconstructDofMotionShadows(img, *l->tg);
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
            {
                const Vec4f v = img.getVec4f(Vec2i(x, y));
                float* o = rgba + ((size_t)y * W + x) * 4;
                o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
            }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return 1;
    }
}

// Same, loading the buffer with the reference loader UVTSampleBuffer(const char*)
// (SampleBuffer.cpp:230-387), which reads <path> and <path>.header.
int ref_create_from_file(const char* path, float aperture, float focus, const float* uvt,
                         int lensFilter, int timeFilter, void** out, double* build_seconds)
{
    RefHandle* h = new RefHandle();
    try
    {
        h->sbuf = new UVTSampleBuffer(path);
        return finish_create(h, aperture, focus, uvt, lensFilter, timeFilter, out, build_seconds);
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        delete h->tg; delete h->params; delete h->sbuf; delete h;
        return 1;
    }
}

// Buffer contents as loaded (for loader parity): W,H,spp,C0,C1 and 16-float records.
int ref_buffer_info(void* handle, int* W, int* H, int* spp, float* C0, float* C1)
{
    RefHandle* h = (RefHandle*)handle;
    *W = h->sbuf->getWidth(); *H = h->sbuf->getHeight(); *spp = h->sbuf->getNumSamples();
    *C0 = h->sbuf->getCocCoeffs().x; *C1 = h->sbuf->getCocCoeffs().y;
    return 0;
}

int ref_buffer_records(void* handle, float* out)
{
    RefHandle* h = (RefHandle*)handle;
    const UVTSampleBuffer& b = *h->sbuf;
    for (int y = 0; y < b.getHeight(); y++)
    for (int x = 0; x < b.getWidth(); x++)
    for (int i = 0; i < b.getNumSamples(); i++)
    {
        float* e = out + (size_t)((y * b.getWidth() + x) * b.getNumSamples() + i) * 16;
        e[0] = b.getSampleXY(x, y, i).x; e[1] = b.getSampleXY(x, y, i).y;
        e[2] = b.getSampleDepth(x, y, i); e[3] = b.getSampleW(x, y, i);
        e[4] = b.getSampleUV(x, y, i).x; e[5] = b.getSampleUV(x, y, i).y;
        e[6] = b.getSampleT(x, y, i);
        Vec4f c = b.getSampleColor(x, y, i);
        e[7] = c.x; e[8] = c.y; e[9] = c.z; e[10] = c.w;
        Vec3f mv = b.getSampleMV(x, y, i);
        e[11] = mv.x; e[12] = mv.y; e[13] = mv.z;
        e[14] = b.getSampleWG(x, y, i).x; e[15] = b.getSampleWG(x, y, i).y;
    }
    return 0;
}

// reconstructDofMotion (Reconstruction.cpp:221-295) into an RGBA float image.
// stats: 16 doubles = the Stats struct (Reconstruction.hpp:134-147), may be NULL.
int ref_reconstruct(void* handle, float* rgba, double* seconds, double* stats)
{
    RefHandle* h = (RefHandle*)handle;
    try
    {
        const int W = h->sbuf->getWidth(), H = h->sbuf->getHeight();
        Image img(Vec2i(W, H));
        auto t0 = std::chrono::steady_clock::now();
        h->tg->reconstructDofMotion(img);
        if (seconds)
            *seconds = seconds_since(t0);
        memcpy(rgba, img.getPtr(), sizeof(float) * 4 * (size_t)W * H);
        (void)stats;
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return 1;
    }
}

// Reconstruct only the scanlines [y0, y1) with the reference's per-scanline task
// (FilterTask::process, Reconstruction.cpp:642-720), on the launcher's threads.
// Used for a bounded CPU-baseline sample of a large frame.
int ref_reconstruct_rows(void* handle, int y0, int y1, float* rgba_rows, double* seconds)
{
    RefHandle* h = (RefHandle*)handle;
    try
    {
        const int W = h->sbuf->getWidth();
        TreeGather* tg = h->tg;
        tg->generateOutputSamples(*h->params);
        MulticoreLauncher launcher;
        Array<TreeGather::FilterTask> ftasks;
        ftasks.reset(y1 - y0);
        tg->m_multicore = true;
        auto t0 = std::chrono::steady_clock::now();
        for (int y = y0; y < y1; y++)
        {
            ftasks[y - y0].init(tg);
            launcher.push(TreeGather::FilterTask::dispatcher, &ftasks[y - y0], y, 1);
        }
        // dispatcher calls process(task.idx); tasks index ftasks by data pointer
        launcher.popAll();
        if (seconds)
            *seconds = seconds_since(t0);
        for (int y = y0; y < y1; y++)
            for (int x = 0; x < W; x++)
            {
                Vec4f c = ftasks[y - y0].m_outputColors[x];
                float* o = rgba_rows + ((size_t)(y - y0) * W + x) * 4;
                o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
            }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return 1;
    }
}

// Reconstruct the listed scanlines rows[0..n) with the reference's per-scanline
// task, all of them pushed to the launcher at once (so they run in parallel on
// its threads); rgba_rows receives n*W*4 floats in list order.  Used for a CPU
// sample of a frame's rows spread over its whole height.
int ref_reconstruct_rowlist(void* handle, const int* rows, int n, float* rgba_rows, double* seconds)
{
    RefHandle* h = (RefHandle*)handle;
    try
    {
        const int W = h->sbuf->getWidth();
        TreeGather* tg = h->tg;
        tg->generateOutputSamples(*h->params);
        MulticoreLauncher launcher;
        Array<TreeGather::FilterTask> ftasks;
        ftasks.reset(n);
        tg->m_multicore = true;
        auto t0 = std::chrono::steady_clock::now();
        for (int k = 0; k < n; k++)
        {
            ftasks[k].init(tg);
            launcher.push(TreeGather::FilterTask::dispatcher, &ftasks[k], rows[k], 1);
        }
        launcher.popAll();
        if (seconds)
            *seconds = seconds_since(t0);
        for (int k = 0; k < n; k++)
            for (int x = 0; x < W; x++)
            {
                Vec4f c = ftasks[k].m_outputColors[x];
                float* o = rgba_rows + ((size_t)k * W + x) * 4;
                o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
            }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return 1;
    }
}

// TreeGather::reconstructShadows (Reconstruction.cpp:302-344) with a query buffer of
// the light buffer's size and qspp samples per pixel (16-float records, pixel-major)
// and its LIGHTSPACE_DENSITY channel; rgba receives the query buffer's sample
// colours afterwards (W*H*qspp*4).
int ref_reconstruct_shadows(void* handle, const float* queries, int qspp, const float* density, float* rgba)
{
    RefHandle* h = (RefHandle*)handle;
    try
    {
        const int W = h->sbuf->getWidth(), H = h->sbuf->getHeight();
        UVTSampleBuffer* q = buffer_from_records(queries, W, H, qspp, 0.0f, 0.0f);
        const int cid = q->reserveChannel<float>("LIGHTSPACE_DENSITY");
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                for (int i = 0; i < qspp; i++)
                    (*(Array<float>*)(q->m_channels[cid]))[q->getIndex(x, y, i)] =
                        density[((size_t)y * W + x) * qspp + i];
        h->tg->reconstructShadows(q, NULL);
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
                for (int i = 0; i < qspp; i++)
                {
                    const Vec4f c = q->getSampleColor(x, y, i);
                    float* o = rgba + (((size_t)y * W + x) * qspp + i) * 4;
                    o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
                }
        h->tg->m_qbuf = NULL;
        delete q;
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return 1;
    }
}

int ref_tree_info(void* handle, int* num_nodes, int* num_samples, int* root, int* spp_pow2,
                  float* coc_adjusted, int* output_spp)
{
    RefHandle* h = (RefHandle*)handle;
    *num_nodes = h->tg->m_hierarchy.getSize();
    *num_samples = h->tg->m_samples.getSize();
    *root = h->tg->m_rootIndex;
    *spp_pow2 = h->tg->m_spp;
    coc_adjusted[0] = h->tg->m_cocCoeffs.x;
    coc_adjusted[1] = h->tg->m_cocCoeffs.y;
    *output_spp = h->tg->m_outputSpp;
    return 0;
}

// Node i: planes (12 floats: xmin,xmax,ymin,ymax as (t,uv,const)), tspan (2) ->
// nodef[i*14..]; child0, child1, s0, s1, ns -> nodei[i*5..].  Leaf iff child0==-1.
// Sample j: xy, w, t, mv(3), color(4), key -> samplef[j*12..].
int ref_tree_export(void* handle, float* nodef, int* nodei, float* samplef)
{
    RefHandle* h = (RefHandle*)handle;
    const Array<TreeGather::Node>& nodes = h->tg->m_hierarchy;
    for (int i = 0; i < nodes.getSize(); i++)
    {
        const TreeGather::Node& n = nodes[i];
        for (int p = 0; p < 4; p++)
            for (int k = 0; k < 3; k++)
                nodef[i * 14 + p * 3 + k] = n.tlb.planes[p][k];
        nodef[i * 14 + 12] = n.tlb.tspan.x;
        nodef[i * 14 + 13] = n.tlb.tspan.y;
        nodei[i * 5 + 0] = n.child0;
        nodei[i * 5 + 1] = n.child1;
        nodei[i * 5 + 2] = n.isLeaf() ? n.s0 : -1;
        nodei[i * 5 + 3] = n.isLeaf() ? n.s1 : -1;
        nodei[i * 5 + 4] = n.ns;
    }
    const Array<TreeGather::Sample>& s = h->tg->m_samples;
    for (int j = 0; j < s.getSize(); j++)
    {
        float* o = samplef + (size_t)j * 12;
        o[0] = s[j].xy.x; o[1] = s[j].xy.y; o[2] = s[j].w; o[3] = s[j].t;
        o[4] = s[j].mv.x; o[5] = s[j].mv.y; o[6] = s[j].mv.z;
        o[7] = s[j].color.x; o[8] = s[j].color.y; o[9] = s[j].color.z; o[10] = s[j].color.w;
        o[11] = s[j].key;
    }
    return 0;
}

// Output sampling pattern (generateOutputSamples, Reconstruction.cpp:452-512):
// 64*M entries of (x, y, u, v, t).
int ref_output_samples(void* handle, float* out)
{
    RefHandle* h = (RefHandle*)handle;
    const Array<TreeGather::Sample>& os = h->tg->m_outputSamples;
    for (int i = 0; i < os.getSize(); i++)
    {
        out[i * 5 + 0] = os[i].xy.x; out[i * 5 + 1] = os[i].xy.y;
        out[i * 5 + 2] = os[i].uv.x; out[i * 5 + 3] = os[i].uv.y;
        out[i * 5 + 4] = os[i].t;
    }
    return os.getSize();
}

// One output sample (x, y, i) through Filterer::reconstruct (ReconstructionOur.cpp:50-359),
// constructed as FilterTask::process does (Reconstruction.cpp:653, 692-693).
// rgba: the query's result colour.  trace (int32, optional):
//   [0] flags: bit0 = 2R fetch, bit1 = "at least one" widening, bit2 = surfaces merged
//   [1] number of surfaces S (after the final fetch, after tiny-surface merging)
//   then per surface: count n, minIndex, then n sample indices (into the tree's sample array)
// Returns the number of ints written, or -1 if trace_cap is too small.
int ref_query(void* handle, int x, int y, int i, float* rgba, int* trace, int trace_cap)
{
    RefHandle* h = (RefHandle*)handle;
    TreeGather* tg = h->tg;
    const int pattern = hashBits(x, y) % TreeGather::NUM_PATTERNS;
    TreeGather::Sample o = tg->m_outputSamples[pattern * tg->m_outputSpp + i];
    o.xy += Vec2f(Vec2i(x, y));
    static thread_local TreeGather::Filterer* f = nullptr;
    static thread_local TreeGather* f_tg = nullptr;
    if (!f || f_tg != tg)
    {
        delete f;
        f = new TreeGather::Filterer();
        f->setTreeGather(tg);
        f_tg = tg;
    }
    tg->m_multicore = true;
    TreeGather::Stats stats;
    Vec4f debugColor;
    TreeGather::Filterer::Result r = f->reconstruct(o, 1.f, false, stats, debugColor);
    rgba[0] = r.color.x; rgba[1] = r.color.y; rgba[2] = r.color.z; rgba[3] = r.color.w;
    if (!trace)
        return 0;
    int n = 0;
    auto put = [&](int v) { if (n < trace_cap) trace[n] = v; n++; };
    int flags = (stats.num2R[0] > 0 ? 1 : 0) | (stats.numAtLeastOne[0] > 0 ? 2 : 0) | (stats.numSurfacesMerged[0] > 0 ? 4 : 0);
    put(flags);
    const Array<TreeGather::Filterer::Surface>& S = f->m_surfaces;
    put(S.getSize());
    for (int s = 0; s < S.getSize(); s++)
    {
        put(S[s].samples.getSize());
        put(S[s].minIndex);
        for (int k = 0; k < S[s].samples.getSize(); k++)
            put(S[s].samples[k].index);
    }
    return (n <= trace_cap) ? n : -1;
}

void ref_destroy(void* handle)
{
    RefHandle* h = (RefHandle*)handle;
    if (!h)
        return;
    delete h->tg;
    delete h->params;
    delete h->sbuf;
    delete h;
}

} // extern "C"
