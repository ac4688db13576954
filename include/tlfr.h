/*
 * tlfr.h — C ABI of the B200 temporal light field reconstruction library
 * (libtlfr.so).  Plain C types only: pointers, sizes, status codes.
 *
 * The entry points replace the reference reconstruction library's API
 * (jiawen/temporal-lightfield-reconstruction, src/reconstruction_lib):
 *
 *   tlfr_buffer_load        UVTSampleBuffer::UVTSampleBuffer(const char*)      common/SampleBuffer.cpp:230-387
 *   tlfr_buffer_from_host   UVTSampleBuffer filled in memory (App import path) reconstruction_app/App.cpp:334-433
 *   tlfr_buffer_save        UVTSampleBuffer::serialize(...)                    common/SampleBuffer.cpp:404-564
 *   tlfr_create             TreeGather::TreeGather(sbuf, params, aperture, focus)
 *                                                                              reconstruction/Reconstruction.hpp:45,
 *                                                                              reconstruction/Reconstruction.cpp:43-215
 *   tlfr_reconstruct        TreeGather::reconstructDofMotion(Image&)           reconstruction/Reconstruction.cpp:221-295
 *                           with CameraParams::enableCuda (the CPU/GPU toggle, Reconstruction.cpp:233) always "GPU"
 *   tlfr_params             the CameraParams fields the path reads              common/CameraParams.hpp:74-107
 *
 * Error behaviour: the reference aborts through fail() (framework/base/Defs.hpp:142);
 * every entry point here returns a tlfr_status instead and records a message
 * retrievable with tlfr_last_error().  There is no CPU fallback: when the CUDA
 * device or kernels are unavailable the calls fail with TLFR_CUDA / TLFR_NO_DEVICE.
 *
 * Threading: a context is externally synchronised (one host thread at a time).
 * All device work of a context is issued on the stream given at creation; calls
 * that return host data synchronise that stream.
 */
#ifndef TLFR_H
#define TLFR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tlfr_status
{
    TLFR_OK        = 0,
    TLFR_BAD_ARG   = 1,   /* invalid argument (null pointer, bad size, unknown mode)     */
    TLFR_IO        = 2,   /* file could not be opened / read / written                   */
    TLFR_FORMAT    = 3,   /* unsupported header version or malformed records             */
    TLFR_OOM       = 4,   /* device or host allocation failed                            */
    TLFR_CUDA      = 5,   /* a CUDA call or kernel failed                                */
    TLFR_OVERFLOW  = 6,   /* a query or build exceeded the largest supported capacity    */
    TLFR_TIMEOUT   = 7,   /* a bounded device wait gave up                               */
    TLFR_NO_DEVICE = 8,   /* no CUDA device                                              */
    TLFR_EMPTY     = 9    /* every sample was discarded (Reconstruction.cpp:587-588)     */
} tlfr_status;

typedef struct tlfr_buffer tlfr_buffer;   /* host sample buffer (UVTSampleBuffer)      */
typedef struct tlfr_ctx    tlfr_ctx;      /* device hierarchy + query state (TreeGather) */

/* Lens/time output-sample weighting, CameraParams.hpp:48-58. */
enum { TLFR_FILTER_BOX = 0, TLFR_FILTER_GAUSSIAN = 1 };

/* Reconstruction parameters (the CameraParams fields the path reads). */
typedef struct tlfr_params
{
    float aperture_adjust;   /* TreeGather ctor apertureAdjust, default 1 (Reconstruction.hpp:45) */
    float focus_adjust;      /* TreeGather ctor focalDistanceAdjust, default 1                  */
    int   lens_filter;       /* TLFR_FILTER_*, CameraParams::lensFilter                          */
    int   time_filter;       /* TLFR_FILTER_*, CameraParams::timeFilter                          */
    int   override_uvt;      /* nonzero: CameraParams::overrideUVT = uvt (one output sample per
                                pixel at the pixel centre, Reconstruction.cpp:454-500);
                                the t=1 pinhole image is uvt = {0,0,1} (App.cpp:450)           */
    float uvt[3];
    int   output_spp;        /* output samples per pixel; 0 = reference default (128, or 1 with
                                override_uvt; Reconstruction.hpp:67-68).  Any value in [1,1024]. */
    int   device;            /* CUDA device ordinal                                              */
    int   enable_cuda;       /* CameraParams::enableCuda, the reference's CPU/GPU toggle
                                (CameraParams.hpp:88, Reconstruction.cpp:233): 0 (default) = the
                                algorithm of its CPU reconstruction (TreeGather::Filterer,
                                ReconstructionOur.cpp:50-511); 1 = the algorithm of its GPU
                                reconstruction (first surface, wedge-box coverage, 2R surfaces
                                with fan triangles, nearest sample; ReconstructionCuda.cpp:
                                261-872, ReconstructionCudaKernels.cu:242-868), here with no
                                capacity limit and no CPU overflow.  Both run on the GPU.       */
} tlfr_params;

/* Fills p with the reference defaults (CameraParams ctor, CameraParams.hpp:77-90). */
void tlfr_params_default(tlfr_params* p);

/* Per-reconstruction counters.  The first eight follow TreeGather::Stats
 * (Reconstruction.hpp:134-147), summed over all output samples; the rest are
 * device-side query classes.                                                   */
typedef struct tlfr_stats
{
    double num_output_samples;
    double num_leaf_nodes;            /* leaves intersected, summed over fetch passes      */
    double num_samples_in_leaf_nodes; /* samples tested, summed over fetch passes          */
    double num_samples_within_1r;
    double num_samples_fetched;       /* samples accepted, summed over fetch passes        */
    double num_surfaces;
    double num_2r;                    /* output samples that did a 2R fetch                */
    double num_surfaces_merged;
    double num_at_least_one;          /* output samples that widened beyond 2R             */
    double num_overflow_queries;      /* queries re-run by the large-capacity pass          */
    double num_empty;                 /* output samples that found no sample at all        */
    double build_ms;                  /* device time of the last hierarchy build           */
    double query_ms;                  /* device time of the last reconstruction            */
    double query_kernel_ms;           /* device time of the main query kernel alone        */
    double build_launches;            /* kernels launched by the last hierarchy build      */
    double query_launches;            /* kernels launched by the last reconstruction       */
    double overflow_leaves;           /* queries that outgrew the main pass, by capacity:  */
    double overflow_stack;            /*   leaf list, traversal stack, surface list,       */
    double overflow_surfaces;         /*   accepted-sample list (counted when stats are    */
    double overflow_samples;          /*   requested)                                      */
    double num_heavy_queries;         /* output samples that needed the full (2R) path      */
    double light_ms;                  /* device time of the light (1R) pass                 */
    double heavy_ms;                  /* device time of the full-path pass                  */
    double num_retried_queries;       /* output samples that outgrew the first light tier   */
                                      /*   and were run again with larger capacities        */
} tlfr_stats;

/* ---- sample buffers ------------------------------------------------------- */

/* Load <path> (+ <path>.header when present), header version 1.3, text or binary
 * 16-float records; alpha forced to 1 (SampleBuffer.cpp:343, 372).              */
tlfr_status tlfr_buffer_load(const char* path, tlfr_buffer** out);

/* Wrap host records (16 floats each, pixel-major, index (y*W+x)*spp+i, field order
 * x,y,z/w,w,u,v,t,r,g,b,a,mv_x,mv_y,mv_w,dwdx,dwdy).  The records are copied;
 * alpha is forced to 1 as the loader does.                                     */
tlfr_status tlfr_buffer_from_host(const float* records16, int width, int height, int spp,
                                  float coc0, float coc1, tlfr_buffer** out);

/* Write a buffer in the reference format (SampleBuffer.cpp:404-564): header v1.3,
 * separate "<path>.header" when separate_header, binary or text records.        */
tlfr_status tlfr_buffer_save(const tlfr_buffer* buf, const char* path, int separate_header, int binary);

tlfr_status  tlfr_buffer_info(const tlfr_buffer* buf, int* width, int* height, int* spp,
                              float* coc0, float* coc1);
const float* tlfr_buffer_records(const tlfr_buffer* buf);
void         tlfr_buffer_free(tlfr_buffer* buf);

/* ---- hierarchy build and reconstruction ------------------------------------ */

/* TreeGather ctor: upload the buffer and build the 5D sample hierarchy on the GPU.
 * stream: a cudaStream_t (NULL = the legacy default stream).                     */
tlfr_status tlfr_create(const tlfr_buffer* buf, const tlfr_params* params, void* stream, tlfr_ctx** out);

/* Same, from records already in device memory (16 floats each, layout as above). */
tlfr_status tlfr_create_device(const float* d_records16, int width, int height, int spp,
                               float coc0, float coc1, const tlfr_params* params, void* stream,
                               tlfr_ctx** out);

/* Rebuild the hierarchy of an existing context from new device records of the same
 * size, reusing its device memory (no allocation when the sizes still fit).       */
tlfr_status tlfr_rebuild_device(tlfr_ctx* ctx, const float* d_records16);

/* Same from a host buffer of the same size: the records are copied to the
 * context's device memory on its stream, then the hierarchy is rebuilt.  Buffers
 * made by tlfr_buffer_from_host / tlfr_buffer_load live in page-locked memory when
 * a CUDA device is present, so the copy runs at full PCIe rate.                   */
tlfr_status tlfr_rebuild(tlfr_ctx* ctx, const tlfr_buffer* buf);

/* reconstructDofMotion: one RGBA float pixel per buffer pixel, row-major, alpha 1,
 * (1,0,0,1) where no sample was found (Reconstruction.cpp:716-719).
 * rgba_on_device: 0 = rgba is host memory (the call synchronises), 1 = device memory
 * (the call returns once the work is queued on the context's stream).
 * stats may be NULL.                                                              */
tlfr_status tlfr_reconstruct(tlfr_ctx* ctx, float* rgba, int rgba_on_device, tlfr_stats* stats);

/* Change the output-sample parameters (override_uvt/uvt, output_spp, filters) of an
 * existing context; the hierarchy is kept (App.cpp:616-694 refocus/animation loop). */
tlfr_status tlfr_set_output(tlfr_ctx* ctx, const tlfr_params* params);

/* Frees the hierarchy build's working storage of a built context (about 190
 * bytes per input sample) and trims its node arrays to the nodes emitted; the
 * hierarchy stays and reconstructions go on as before, a later rebuild
 * allocates the storage again.  For many contexts held at once (batches).     */
tlfr_status tlfr_trim(tlfr_ctx* ctx);
tlfr_status tlfr_sync(tlfr_ctx* ctx);
tlfr_status tlfr_get_stats(tlfr_ctx* ctx, tlfr_stats* stats);
void        tlfr_destroy(tlfr_ctx* ctx);

/* Message of the last failed call on ctx (ctx may be NULL for creation errors). */
const char* tlfr_last_error(const tlfr_ctx* ctx);

/* ---- introspection (parity tests, profiling) -------------------------------- */

/* Sizes of the built hierarchy.  nodes: hierarchy nodes; samples: samples stored in
 * leaves (TreeGather::m_samples); height: longest root-to-leaf path.              */
tlfr_status tlfr_tree_info(tlfr_ctx* ctx, int* num_nodes, int* num_samples, int* root, int* height);

/* Copy the hierarchy to host memory.  Node i: nodef[i*14 .. +14) = 4 planes
 * (xmin,xmax,ymin,ymax) as (t, uv, const) then tspan (2); nodei[i*5 .. +5) =
 * child0, child1, s0, s1, ns (child0 == -1 for leaves; s0/s1 == -1 for internal
 * nodes).  Sample j: samplef[j*12 .. +12) = x, y, w, t, mv(3), rgba(4), key;
 * sample_ids[j] = index of the input record it came from.  Any pointer may be NULL. */
tlfr_status tlfr_tree_export(tlfr_ctx* ctx, float* nodef, int* nodei, float* samplef, int* sample_ids);

/* Output sampling pattern: 64 patterns x output_spp entries of (x, y, u, v, t)
 * (generateOutputSamples, Reconstruction.cpp:452-512).  Returns the entry count.  */
int tlfr_output_samples(tlfr_ctx* ctx, float* out5);

/* The output samples of the last reconstruction as a sample buffer
 * (Reconstruction.cpp:290-294, 696-712: the m_obuf debug dump, which the
 * reference writes with UVTSampleBuffer::serialize): W*H*M records, record
 * (x, y, i) holding the output sample's x, y, u, v, t and its reconstructed
 * RGBA; z/w = w = 1 and no motion.  Save it with tlfr_buffer_save; free it
 * with tlfr_buffer_free.                                                     */
tlfr_status tlfr_output_sample_buffer(tlfr_ctx* ctx, tlfr_buffer** out);

/* Shadow reconstruction, TreeGather::reconstructShadows (Reconstruction.cpp:
 * 302-344; the reference notes it is not callable from its application): the
 * context's hierarchy holds light-space samples (their dw/dx, dw/dy in record
 * fields 14-15); each of the n query samples (16-float records of the view in
 * light space: x, y, w, u, v, t are read, fields 0,1,3,4,5,6) runs the Filterer
 * in shadow mode (ReconstructionOur.cpp:78-80, 283-291, 337-347): dispersion
 * scaled by sqrt(density[k]) (the query buffer's LIGHTSPACE_DENSITY channel;
 * NULL reads 1), each filtered sample's colour kept where it lights the query
 * (w - 0.01 <= sample w at t + (query - sample) . (dw/dx, dw/dy)) and black
 * with its alpha where it shadows it, no lens or time weights.  rgba receives
 * 4 floats per query (host memory); the reference writes them into the query
 * buffer's sample colours.  Host buffers; synchronous.                       */
tlfr_status tlfr_reconstruct_shadows(tlfr_ctx* ctx, const float* queries16, int num_queries, const float* density,
                                     float* rgba);

/* A camera as the shadowed reconstruction reads it from CameraParams
 * (CameraParams.hpp:74-141) and its CameraControls.  Matrices row-major,
 * element (r, c) at [4*r + c], as the framework's Mat4f::get(r, c).         */
typedef struct tlfr_view
{
    float projection[16];       /* CameraParams::projection                    */
    float camera_to_world[16];  /* CameraParams::camera.getCameraToWorld()     */
    float world_to_camera[16];  /* CameraParams::camera.getWorldToCamera()     */
    float far_plane;            /* CameraParams::camera.getFar()               */
    int   window_size[2];       /* CameraParams::windowSize                    */
    float aperture_radius;      /* CameraParams::apertureRadius                */
    float focus_distance;       /* CameraParams::focusDistance                 */
} tlfr_view;

/* Motion and defocus with soft shadows from a square area light,
 * TreeGather::reconstructDofMotionShadows (Reconstruction.cpp:355-433, with
 * FilterTask::process2, 723-829; the reference notes it is not callable from
 * its application).  camera: the camera's context; light: a context over the
 * light-space buffer of the same image size (its dw/dx, dw/dy in record fields
 * 14-15); both with enable_cuda = 0.  Every output sample of the camera is
 * reconstructed; its nearest sample, reprojected to the lens centre with the
 * camera view's CoC, is mapped into the light's image; the light's hierarchy
 * reconstructs it in shadow mode from a point on the light source (Sobol
 * dimensions 3 and 4, rotated per pixel) with the dispersion scaled by
 * sqrt(camera_density) of the nearest sample (the camera buffer's
 * LIGHTSPACE_DENSITY channel, one float per input record in record order;
 * NULL reads 1); the colour is lit by 1.5 * max(0, -L.N) with N rebuilt from
 * the nearest sample's w gradients (lightSpaceDot, Util.cpp:202-224), plus
 * 0.5 * ambient * the camera colour.  Samples beyond camera far - 0.01 or
 * outside the light's image keep the camera colour; a pixel with an output
 * sample the camera cannot reconstruct is red.  rgba: W*H*4 floats (device
 * memory when rgba_on_device).  Synchronous.                                 */
tlfr_status tlfr_reconstruct_dof_motion_shadows(tlfr_ctx* camera, const tlfr_view* camera_view,
                                                const float* camera_density, tlfr_ctx* light,
                                                const tlfr_view* light_view, float* rgba, int rgba_on_device);

/* Run the output samples (x, y, i) listed in xyi[3*k ..] through the device query
 * path with tracing on.  rgba[4*k ..] = the query colour.  trace[k*trace_stride ..]:
 *   [0] flags: bit0 = 2R fetch, bit1 = widened beyond 2R, bit2 = surfaces merged,
 *       bit3 = ran in the large-capacity pass
 *   [1] S = number of surfaces after the final fetch and tiny-surface merging,
 *   then per surface: n, minIndex, n sample indices (into the hierarchy's samples).
 * A trace that does not fit its stride is cut and its [1] set to -1.             */
tlfr_status tlfr_trace_queries(tlfr_ctx* ctx, const int* xyi, int num_queries,
                               float* rgba, int* trace, int trace_stride);

/* Allocation-free output-sample queries.  No counterpart in the reference: an
 * addition for callers that cannot allocate device memory while they run (all
 * memory reserved up front, an external allocator that owns the device heap, a
 * thread that must not block on the allocator).  Same results as the colours of
 * tlfr_trace_queries, for the output samples (x, y, i) in d_xyi[3*k ..] (device
 * memory, 4-byte aligned), written to d_rgba[4*k ..] (device memory, 16-byte
 * aligned: the colours are stored as float4; a misaligned pointer is refused
 * with TLFR_BAD_ARG).  The per-query working storage is a fixed 9.75 MiB device
 * array inside the library (256 working slots), which every device that loads
 * the library keeps until the process exits; nothing is allocated by the call.
 * A query that needs more than a slot holds (or an (x, y, i) out of range)
 * yields (0, 0, 0, -1) and is counted in *d_overflow (device memory, may be
 * NULL; set to zero by the call, also when num_queries is 0).
 * num_queries <= 262144 per call, else TLFR_BAD_ARG: the 256 slots each run one
 * query at a time, so a call is meant for a few thousand to a few hundred
 * thousand output samples.  Asynchronous on the context's stream.  The first
 * call on a device looks up the array's device address with that device
 * current: make it before any stream capture.  All calls share the array, so
 * calls whose work overlaps on the GPU race.                                   */
tlfr_status tlfr_query_samples_noalloc(tlfr_ctx* ctx, const int* d_xyi, int num_queries, float* d_rgba,
                                       int* d_overflow);

/* ---- synthetic scenes (tests, benchmarks) ---------------------------------- */

enum
{
    TLFR_SCENE_PLANES      = 0,   /* three fronto-parallel planes at w=2,5,12; defocus only       */
    TLFR_SCENE_CARDS       = 1,   /* 64 moving textured rectangles, w in [1,50]; defocus + motion */
    TLFR_SCENE_CARDS_LARGE = 2    /* 256 rectangles + 64 disks, w in [0.5,100]; strong blur       */
};

/* Fill records (width*height*spp*16 floats) with a seeded analytic scene; coc_out
 * receives (C0, C1).  Host-side, multithreaded, deterministic for a given seed.   */
tlfr_status tlfr_synth_scene(int preset, int width, int height, int spp, unsigned long long seed,
                             float* records, float* coc_out);

/* Reference image of a synthetic scene (the ground truth against which a
 * reconstruction's PSNR is measured): per pixel the mean colour of the
 * analytic scene over `samples` points spread over the pixel, the unit lens
 * disk and the shutter [0, 1], computed on the current CUDA device; rgba
 * receives width*height*4 floats (host memory).  No counterpart in the
 * reference, whose ground-truth images came from its renderer.              */
tlfr_status tlfr_synth_reference_image(int preset, int width, int height, int samples, unsigned long long seed,
                                       float* rgba);

/* ---- learned routing (no counterpart in the reference) --------------------
 * The router has no counterpart in the reference: a small network predicts, per pixel,
 * whether the fast path reproduces the plain method there; pixels above the
 * threshold take the fast path (the plain 1R pass, which keeps the first
 * surface when a second one opens instead of refetching at 2R; only output
 * samples with nothing within 1R still take the full path), the rest take the
 * plain method.  Features, labels and the
 * network are described in temporal-lightfield-reconstruction_b200/csrc/tlfr_route.cu. */
#define TLFR_ROUTE_FEATURES 8
typedef struct tlfr_router tlfr_router;

/* Eight features per pixel of the context's current hierarchy and records,
 * written to d_feats (device, width*height*8 floats, row-major). */
tlfr_status tlfr_route_features(tlfr_ctx* ctx, float* d_feats);
/* Plain reconstruction of the current frame into d_rgba (device, RGBA float)
 * and the per-pixel labels (device, width*height floats): 1 where the fast
 * path reproduces the plain pixel within tol on every channel, 0 elsewhere. */
tlfr_status tlfr_route_labels(tlfr_ctx* ctx, float tol, float* d_labels, float* d_rgba);
/* The same with the scene's ground truth d_ref (device RGBA, W*H*4 floats): a
 * pixel's label is 1 where the fast path's squared RGB error against d_ref is
 * at most tol above the plain method's.                                      */
tlfr_status tlfr_route_labels_ref(tlfr_ctx* ctx, const float* d_ref, float tol, float* d_labels, float* d_rgba);
/* New 8-64-64-1 network on a device, He-initialised from seed; mean8/inv_std8
 * (host, 8 floats each, may be null) standardise the features. */
tlfr_status tlfr_router_create(int device, void* stream, unsigned seed, const float* mean8, const float* inv_std8,
                               tlfr_router** out);
void        tlfr_router_destroy(tlfr_router* router);
const char* tlfr_router_last_error(const tlfr_router* router);
/* Number of floats of the parameter block of tlfr_router_get/set_params. */
int         tlfr_router_num_params(void);
/* steps Adam steps (lr; betas 0.9, 0.999) of binary cross-entropy over minibatches
 * of batch rows drawn from the n (feature, label) rows (device pointers). */
tlfr_status tlfr_router_train(tlfr_router* router, const float* d_feats, const float* d_labels, int n, int steps,
                              int batch, float lr, unsigned seed, float* final_loss);
/* Gradient of the mean cross-entropy over exactly rows 0..n-1, copied to grad
 * (host, the trainable prefix of the parameter block), and the loss. */
tlfr_status tlfr_router_gradient(tlfr_router* router, const float* d_feats, const float* d_labels, int n, float* grad,
                                 float* loss);
/* Single-surface probability of n pixels (device in, device out). */
tlfr_status tlfr_router_predict(tlfr_router* router, const float* d_feats, long long n, float* d_prob);
tlfr_status tlfr_router_get_params(tlfr_router* router, float* params);
tlfr_status tlfr_router_set_params(tlfr_router* router, const float* params);
/* Routed reconstruction: tlfr_reconstruct then computes the features, runs the
 * network and sends pixels with probability above threshold to the fast path.
 * router = null restores the plain method.  The router must outlive the
 * setting, and records passed by device pointer must stay valid. */
tlfr_status tlfr_set_routing(tlfr_ctx* ctx, tlfr_router* router, float threshold);

/* ---- batches -----------------------------------------------------------------
 * Many frames reconstructed as one CUDA graph replayed on one stream, with no
 * host synchronisation inside.  A frame is a built context (a sample buffer of
 * any resolution and spp) with either its own output settings or, for sweeps
 * over one hierarchy, output settings of the frame's own (override_uvt / uvt,
 * output_spp, lens and time filters; aperture and focus adjustments change the
 * hierarchy and need a context of their own).  Each pass runs as ONE persistent
 * launch over all frames of a chunk: blocks take work items (frame, unit) from
 * a device counter and read the frame's parameters from a device table.
 * Frames are grouped into chunks whose per-output-sample storage (24 bytes per
 * output sample) fits budget_bytes (0: half the free device memory, at most
 * 32 GiB); chunks run one after another and share the storage.  With autotune,
 * each frame's light-pass tile shape is chosen by timing every shape at
 * creation.  A frame's router (set on its context, own output settings only)
 * runs before its chunk.  Replaces the reference's per-frame reconstruct loops
 * of the animation and export paths (reconstruction_app/App.cpp:616-694,
 * a new TreeGather per (u,v) frame).  Creating a batch frees its contexts'
 * hierarchy-build working storage (a later rebuild allocates it again), and
 * the graph holds the contexts' buffers as they are at creation: after
 * rebuilding a context, create the batch again.  The contexts (and routers) must outlive the
 * batch.  Outputs are device RGBA float images. */
typedef struct tlfr_batch tlfr_batch;
typedef struct tlfr_batch_frame
{
    tlfr_ctx*          ctx;
    const tlfr_params* output;     /* NULL: the context's own output settings */
    float*             d_rgba;     /* device RGBA image, width*height*4 floats */
} tlfr_batch_frame;
tlfr_status tlfr_batch_create_frames(const tlfr_batch_frame* frames, int n, void* stream, int autotune,
                                     size_t budget_bytes, tlfr_batch** out);
/* The same for n contexts with their own output settings and the default budget. */
tlfr_status tlfr_batch_create(tlfr_ctx* const* ctxs, int n, float* const* d_rgba, void* stream, int autotune,
                              tlfr_batch** out);
/* Replays the batch on its stream (asynchronous). */
tlfr_status tlfr_batch_run(tlfr_batch* batch);
/* Waits for the last run; device time in ms (optional); TLFR_OVERFLOW when an
 * output sample exceeded every capacity. */
tlfr_status tlfr_batch_sync(tlfr_batch* batch, double* ms);
/* The light-pass tile shape chosen for each frame (n entries): 0 = 4x2 pixels
 * x 4 output samples per warp, 1 = 8x4 x 1, 2 = 4x4 x 2, 3 = 2x2 x 8, 4 = 2x1 x 16. */
tlfr_status tlfr_batch_info(const tlfr_batch* batch, int* tile_shapes);
/* The chunk of each frame (n entries, optional) and the kernel launches of one run. */
tlfr_status tlfr_batch_layout(const tlfr_batch* batch, int* chunks, long long* launches);
const char* tlfr_batch_last_error(const tlfr_batch* batch);
void        tlfr_batch_destroy(tlfr_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* TLFR_H */
