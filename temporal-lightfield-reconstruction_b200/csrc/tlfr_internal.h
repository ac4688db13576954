// tlfr_internal.h — device data layout and the context shared by the build,
// query and API translation units.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <string>
#include <vector>
#include "tlfr.h"
#include "tlfr_common.cuh"

// Kernel launch on the context's stream, counted in Ctx::launches.
#define TLFR_LAUNCH(ctx, kern, grid, block, stream, ...) \
    do { kern<<<(grid), (block), 0, (stream)>>>(__VA_ARGS__); (ctx).launches++; } while (0)

namespace tlfr
{

// Hierarchy node as the query reads it: 64 bytes, one aligned 64-byte load.
//   a = (xmin.t, xmin.uv, xmin.c, xmax.t)
//   b = (xmax.uv, xmax.c, ymin.t, ymin.uv)
//   c = (ymin.c, ymax.t, ymax.uv, ymax.c)
//   d = (child0 or -1 for a leaf, child1, s0, s1)
// Internal nodes' children are emitted as a pair, so child1 == child0 + 1.
struct __align__(16) QNode
{
    float4 a, b, c;
    int4   d;
};

// Node while the hierarchy is being built (Reconstruction.hpp:179-231 Node):
// bounds, sample count, and either the sample range (leaf) or the emitted
// children (internal).  80 bytes.
struct __align__(16) BNode
{
    float p[12];        // planes xmin, xmax, ymin, ymax as (t, uv, const)
    float tspan[2];
    int   ref;          // >= 0: child0 slot of an internal node; < 0: leaf with s0 = ~ref
    int   ns;
    int   height;       // longest path to a leaf below, 1 for a leaf
    int   pad;
};

// kd split of the reprojection grid (Reconstruction.hpp:169-177 InitialNode)
struct __align__(16) KdNode
{
    int x0, y0, x1, y1;
    int child0, child1;     // -1 for a leaf
    int num_samples;        // samples in the subtree
    int depth;
    int path;               // child choices at depths 0..4 (bit j = depth j), i.e. the build task
    int parent;
    int leaf_count;         // kd leaves in the subtree
    int preorder_leaf;      // preorder rank of the first kd leaf of the subtree
    int preorder_sample;    // sample offset of the subtree in preorder
    int sample_offset;      // final sample offset (task order, as the reference lays samples out)
    int frontier;           // size of the subtree's frontier after emitNodes
    int pad;
};

// Scalars computed on the device during the build.
struct GridInfo
{
    float bbmin[2], bbmax[2];   // reprojected bounding box (before scaling)
    int   max_hits;
    int   num_valid;            // samples kept by the reprojection (w > 0)
    float scale;
    int   bmin_x, bmin_y;       // integer grid origin
    int   gw, gh;               // grid size
    int   num_kd;               // kd nodes
    int   num_kd_leaves;
    int   num_accepted;         // samples bucketed into the grid
    int   num_nodes;            // emitted hierarchy nodes
    int   root;
    int   height;
    int   entry[32];            // build task entry points (kd node or -1)
    int   task_sample_base[32];
    int   task_leaf_base[33];
    int   num_invalid;          // samples with invalid bounds
    int   error;                // nonzero: build capacity error code
    int   kd_levels;
};

// Per-reconstruction device counters (TreeGather::Stats, Reconstruction.hpp:134-147).
struct DevStats
{
    unsigned long long leaf_nodes, samples_in_leaves, within_1r, fetched, surfaces,
                       num_2r, merged, at_least_one, overflow, empty;
    unsigned long long overflow_by_reason[4];   // [reason & 3]: 1 leaves, 2 stack, 3 surfaces, 0 samples
};

struct Ctx
{
    // configuration
    int W = 0, H = 0, spp_in = 0, spp = 1;
    float coc0_raw[2] = { 0, 0 };   // header coefficients: drive the reprojection (Reconstruction.cpp:519)
    float coc[2] = { 0, 0 };        // refocused coefficients (Reconstruction.cpp:77-87)
    tlfr_params params{};
    int out_spp = 128;
    int device = 0;
    int num_sms = 148;              // multiprocessors of the device (read at creation)
    cudaStream_t stream = nullptr;
    std::string error;

    size_t n_in = 0;                // input records

    // device buffers owned by the context
    float* d_records = nullptr;     // 16-float records (owned copy when created from host)
    const float* cur_records = nullptr;   // records of the current hierarchy (read by the router)
    bool   own_records = false;

    // reprojected samples in input order
    float4* rp_pos = nullptr;       // x, y, w, t
    float4* rp_mot = nullptr;       // mv (3), valid flag
    int*    rp_cell = nullptr;
    int*    hits = nullptr;         // W*H
    GridInfo* d_grid = nullptr;
    GridInfo  grid{};               // host copy

    // grid buckets
    int* cell_count = nullptr;      // gw*gh (+1)
    int* cell_start = nullptr;
    int* cell_items = nullptr;      // input indices, bucketed
    size_t cell_cap = 0;

    // kd tree
    KdNode* kd = nullptr;
    int*    kd_level = nullptr;     // level ranges: [2*L], [2*L+1]
    int*    kd_leaves_ordered = nullptr;   // kd leaf ids in build-task order
    size_t  kd_cap = 0;

    // per-sample build scratch (indexed by final sample slot)
    int*    perm = nullptr;         // input index per slot (sorted candidates)
    float*  box = nullptr;          // 8 floats per slot: boxa, boxb, boxaT1, boxbT1
    Bounds* sbounds = nullptr;      // per-sample bounds
    int*    surface = nullptr;      // surface id per slot
    BNode*  pending = nullptr;      // frontier storage (indexed by slot)
    int*    leaf_task_rank = nullptr;
    int*    ordered_n = nullptr;    // candidate count per ordered leaf
    int*    ordered_prefmax = nullptr;
    BNode*  top = nullptr;          // serial-top scratch
    size_t  samp_cap = 0;
    size_t  leaf_cap = 0;

    // final hierarchy
    QNode*  nodes = nullptr;
    float2* node_tspan = nullptr;   // time span per node (tree export only)
    size_t  node_cap = 0;
    // samples in tree order, one 32-byte record each (a single 256-bit load):
    // s_rec[2i] = (x, y, w, t), s_rec[2i+1] = (mv (3), coc radius at w)
    float4* s_rec = nullptr;
    float4* s_col = nullptr;        // rgba
    int*    s_id = nullptr;         // input record index
    int     num_samples = 0;
    int     num_nodes = 0;
    int     root = 0;
    int     height = 0;

    // output sampling pattern (64 * out_spp entries of x, y, u, v, t)
    float*  d_pattern = nullptr;
    std::vector<float> h_pattern;

    // reconstruction
    float4* qcol = nullptr;         // colour of every output sample of the frame
    int*    heavy_queue = nullptr;  // output samples for the full path
    size_t  qcol_cap = 0;
    int*    ovf_queue = nullptr;    // overflowing query ids
    int*    ovf_count = nullptr;
    size_t  ovf_cap = 0;
    float*  ovf_scratch = nullptr;  // large-capacity per-query storage
    size_t  ovf_scratch_bytes = 0;
    void*   coop_scratch = nullptr; // per-warp working lists of the cooperative full-path pass
    void*   toggle_arena = nullptr; // large lists of the GPU-toggle algorithm's second pass
    size_t  coop_scratch_bytes = 0;
    DevStats* d_stats = nullptr;
    float4* d_out = nullptr;        // device output when the caller passes host memory

    // learned routing (tlfr_route.cu)
    float4* route_fa = nullptr;             // per-pixel feature scratch (2 * W*H)
    float*  route_feats = nullptr;          // W*H*8 features of the routed reconstruction
    float*  route_prob = nullptr;           // W*H single-surface probabilities
    unsigned char* route_fast = nullptr;    // W*H fast-path flags (first-surface 1R pass)
    float4* route_img = nullptr;            // W*H fast-path image (router labels)
    struct Route* router = nullptr;         // null: plain reconstruction
    float   route_hi = 0.8f;                // probability above which a pixel takes the fast path
    bool    route_all_fast = false;         // every pixel on the fast path (router labels)

    tlfr_stats last{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    cudaEvent_t evq0 = nullptr, evq1 = nullptr, evq2 = nullptr;   // around the query passes
    long long launches = 0;                         // kernels launched by this context
};

// Learned router: FP32 master parameters, Adam moments, gradient, BF16 operands.
constexpr int kRouteFeatures = 8;
struct Route
{
    float* params = nullptr;
    float* grad = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    float* loss = nullptr;
    __nv_bfloat16* half = nullptr;
    int step = 0;
    int device = 0;
    int num_sms = 148;          // multiprocessors of the device (read at allocation)
    cudaStream_t stream = nullptr;
    std::string error;
};
int route_num_params();
int route_num_trainable();
tlfr_status route_alloc(Route& r, std::string& err);
void route_free(Route& r);
tlfr_status route_init(Route& r, unsigned seed, const float* mean, const float* inv_std, cudaStream_t s, std::string& err);
tlfr_status route_set_params(Route& r, const float* host_params, cudaStream_t s, std::string& err);
tlfr_status route_get_params(Route& r, float* host_params, cudaStream_t s, std::string& err);
tlfr_status route_gradient(Route& r, const float* d_feats, const float* d_labels, int n, float* host_grad,
                           float* host_loss, cudaStream_t s, std::string& err);
tlfr_status route_train(Route& r, const float* d_feats, const float* d_labels, int n, int steps, int batch, float lr,
                        unsigned seed, float* host_loss, cudaStream_t s, std::string& err);
tlfr_status route_predict(Route& r, const float* d_feats, long long n, float* d_prob, cudaStream_t s, std::string& err);
// router coarse pass: per pixel, how many of four probed output samples the
// plain 1R pass sends to the full path (tlfr_query.cu)
tlfr_status route_probe(Ctx& c, int* d_counts);
constexpr int kRouteProbes = 4;
tlfr_status route_features(Ctx& c, float* d_feats, std::string& err);
tlfr_status route_labels_from(Ctx& c, const float4* d_plain, const float4* d_fast, const float4* d_ref, float tol,
                              float* d_labels, std::string& err);
tlfr_status route_flags(Ctx& c, const float* d_prob, float hi, unsigned char* d_fast, std::string& err);

// build: reprojection, bucketing, kd split, leaf construction, emitNodes, top.
tlfr_status build_hierarchy(Ctx& c, const float* d_records);
// frees the build's working storage and trims the node arrays of a built context
tlfr_status release_build_scratch(Ctx& c);
// query: all output samples of the frame into rgba (device pointer).
tlfr_status reconstruct_frame(Ctx& c, float4* d_rgba, bool collect_stats);
// Batches (tlfr_query.cu): frames reconstructed together in one CUDA graph with
// one persistent launch per pass per chunk of frames.
struct BatchEntry
{
    Ctx* ctx;
    const tlfr_params* output;      // the frame's own output settings (null: the context's)
    float4* out;                    // device pixels
};
struct BatchPlan;
BatchPlan* batch_plan_new();
void batch_plan_delete(BatchPlan* bp);
tlfr_status batch_build(BatchPlan& bp, const std::vector<BatchEntry>& entries, cudaStream_t s, bool autotune,
                        size_t budget, std::string& err);
tlfr_status batch_enqueue(BatchPlan& bp, cudaStream_t s, std::string& err, long long* launches);
tlfr_status batch_failures(BatchPlan& bp, cudaStream_t s, std::vector<int>& hard, std::string& err);
void batch_info(const BatchPlan& bp, int* shapes, int* chunks);
int light_default_blocks(const Ctx& c);
size_t overflow_scratch_bytes();
size_t coop_scratch_bytes(int num_sms);
tlfr_status trace_queries(Ctx& c, const int* h_xyi, int n, float* h_rgba, int* h_trace, int stride);
// shadow reconstruction of n light-space queries (8 floats each, device) into d_out (device)
tlfr_status reconstruct_shadows(Ctx& c, const float* d_queries, int n, float4* d_out);
// Views of the shadowed reconstruction, derived on the host from the camera's
// and the light's CameraParams (Reconstruction.cpp:365-392); matrices row-major.
struct DmsView
{
    float c2l[16];          // ws * cameraToShadow * invws * cameraProjectedZfromW
    float clip_xyw[16];     // invws * cameraProjectedZfromW
    float ip[16];           // invCameraProjection with rows 2 and 3 replaced (Util.cpp:190-192)
    float light_pos[16];    // cameraToShadow2 * invCameraProjection
    float c2s_inv_t[16];    // cameraToShadow2 inverted, transposed
    float c2w_inv_t[16];    // cameraToWorld inverted, transposed
    float cam_far_w;        // camera far - 1e-2
    float ccoc[2], lcoc[2]; // CameraParams::getCocCoeffs of the camera and the light
    std::vector<float> light_uv;   // (sobol(3, i+1), sobol(4, i+1)) per output sample
};
tlfr_status reconstruct_dof_motion_shadows(Ctx& c, Ctx& l, const DmsView& v, const float* d_density, float4* d_img);
// output samples through the full path with working storage in a fixed device array
tlfr_status query_samples_noalloc(Ctx& c, const int* d_xyi, int n, float* d_rgba, int* d_overflow);
// host-side output pattern (Reconstruction.cpp:452-512)
void generate_output_pattern(int out_spp, bool override_uvt, const float* uvt, std::vector<float>& out5);

const char* cuda_error_string(cudaError_t e);

} // namespace tlfr
