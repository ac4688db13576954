// C entry points over the reference's CPU restatement of its GPU-toggle
// algorithm (CameraParams::enableCuda): CudaReconstruction::reconstructCPU and
// reconstructCPUSingle (reference src/reconstruction_lib/reconstruction/
// ReconstructionCuda.cpp:261-872), the checker of the library's enable_cuda
// mode.  Test infrastructure only (oracle/_ref/libtlfr_ref.so).
//
// The reference's own translation unit is compiled here with its private
// members visible.  Its TreeGather::cudaReconstruction fills the GPU layout and
// then launches the CUDA kernels, which this CPU build cannot; the same inputs
// (output sample templates, nodes with internal children ordered larger index
// first, points) are filled here from the TreeGather and handed to
// CudaReconstruction::init, and the reference's CPU functions do the rest.
#include <chrono>
#include <string>

#define private public
#define protected public
#include "ReconstructionCuda.cpp"
#include "ref_handle.h"
#undef private
#undef protected

// Timer is used only by the GPU launch path (ReconstructionCuda.cpp:389-459).
F64 Timer::s_ticksToSecsCoef = -1.0;
S64 Timer::s_prevTicks = 0;
F32 Timer::end(void) { return 0.0f; }
S64 Timer::queryTicks(void) { return 0; }
F32 Timer::ticksToSecs(S64 ticks) { (void)ticks; return 0.0f; }
S64 Timer::getElapsedTicks(void) { return 0; }

namespace
{

std::string g_toggle_error;

struct ToggleInput
{
    Array<CudaSample>        osmp;
    Array<CudaNode>          nodes;
    Array<CudaTraversalNode> tnodes;
    Array<CudaPoint>         points;
    Array<Vec4f>             results;
};

// the GPU layout of the built hierarchy (what cudaReconstruction uploads)
void fill_input(TreeGather* tg, ToggleInput& in)
{
    const int npat = TreeGather::NUM_PATTERNS * tg->m_outputSpp;
    in.osmp.reset(npat);
    for (int i = 0; i < npat; i++)
    {
        const TreeGather::Sample& o = tg->m_outputSamples[i];
        in.osmp[i].x = o.xy.x; in.osmp[i].y = o.xy.y;
        in.osmp[i].u = o.uv.x; in.osmp[i].v = o.uv.y;
        in.osmp[i].t = o.t;
    }
    const int nn = tg->m_hierarchy.getSize();
    in.nodes.reset(nn);
    in.tnodes.reset(nn);
    for (int i = 0; i < nn; i++)
    {
        const TreeGather::Node& src = tg->m_hierarchy[i];
        CudaNode& dst = in.nodes[i];
        if (src.isLeaf())
        {
            dst.idx0 = src.s0;
            dst.idx1 = src.s1;
        }
        else
        {
            dst.idx0 = max(src.child0, src.child1);
            dst.idx1 = min(src.child0, src.child1);
        }
        for (int p = 0; p < 4; p++)
            dst.planes[p] = src.tlb.planes[p];
        dst.tspan = src.tlb.tspan;
    }
    const int np = tg->m_samples.getSize();
    in.points.reset(np);
    for (int i = 0; i < np; i++)
    {
        const TreeGather::Sample& s = tg->m_samples[i];
        CudaPoint& p = in.points[i];
        p.x = s.xy.x; p.y = s.xy.y; p.w = s.w; p.t = s.t;
        p.mvx = s.mv.x; p.mvy = s.mv.y; p.mvw = s.mv.z;
        p.c = s.color;
    }
}

} // namespace

extern "C" {

const char* ref_gpu_toggle_last_error(void) { return g_toggle_error.c_str(); }

// Output samples (x, y, i) of xyi[3k..] through reconstructCPUSingle: rgba[4k..].
int ref_gpu_toggle_queries(void* handle, const int* xyi, int n, float* rgba)
{
    RefHandle* h = (RefHandle*)handle;
    try
    {
        TreeGather* tg = h->tg;
        tg->generateOutputSamples(*h->params);
        const int W = h->sbuf->getWidth(), H = h->sbuf->getHeight(), M = tg->m_outputSpp;
        ToggleInput in;
        fill_input(tg, in);
        Image img(Vec2i(W, H));
        CudaReconstruction cr;
        cr.init(tg->m_spp, M, TreeGather::NUM_PATTERNS, Vec2i(W, H), img, in.osmp, in.results, in.nodes,
                tg->m_rootIndex, in.tnodes, in.points, tg->m_cocCoeffs);
        for (int k = 0; k < n; k++)
        {
            const int id = (xyi[3 * k + 1] * W + xyi[3 * k]) * M + xyi[3 * k + 2];
            const Vec4f c = cr.reconstructCPUSingle(id);
            rgba[4 * k] = c.x; rgba[4 * k + 1] = c.y; rgba[4 * k + 2] = c.z; rgba[4 * k + 3] = c.w;
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_toggle_error = e.what();
        return 1;
    }
}

// The whole image through reconstructCPU (every output sample in order, then
// the normalisation), into rgba (W*H*4).
int ref_gpu_toggle_image(void* handle, float* rgba, double* seconds)
{
    RefHandle* h = (RefHandle*)handle;
    try
    {
        TreeGather* tg = h->tg;
        tg->generateOutputSamples(*h->params);
        const int W = h->sbuf->getWidth(), H = h->sbuf->getHeight(), M = tg->m_outputSpp;
        ToggleInput in;
        fill_input(tg, in);
        Image img(Vec2i(W, H));
        CudaReconstruction cr;
        cr.init(tg->m_spp, M, TreeGather::NUM_PATTERNS, Vec2i(W, H), img, in.osmp, in.results, in.nodes,
                tg->m_rootIndex, in.tnodes, in.points, tg->m_cocCoeffs);
        auto t0 = std::chrono::steady_clock::now();
        cr.reconstructCPU();
        if (seconds)
            *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++)
            {
                const Vec4f c = img.getVec4f(Vec2i(x, y));
                float* o = rgba + ((size_t)y * W + x) * 4;
                o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
            }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_toggle_error = e.what();
        return 1;
    }
}

} // extern "C"
