/*
 * rtpg.h -- C ABI of rtlib_b200, a B200-native (sm_100a) implementation of RTLib's
 * path-guiding hot path.
 *
 * Conventions (the reference has no C ABI; these replace its C++ template API):
 *   - every function returns int: 0 (RTPG_OK) on success, a negative RTPG_E* code on error;
 *     rtpg_last_error() returns a message for the calling thread's last error;
 *   - handles are opaque; all array arguments are DEVICE pointers unless the parameter name
 *     starts with "host_"; sizes are element counts;
 *   - "stream" is a cudaStream_t passed as void* (NULL = legacy default stream); calls are
 *     asynchronous on that stream unless documented otherwise;
 *   - a handle is not thread-safe: one host thread (or external synchronisation) per handle;
 *   - device-side failures (capacity exhausted, fixed-point saturation) never trap: they set
 *     bits in the handle's device status word, which rtpg_*_status() reads (synchronising).
 */
#ifndef RTPG_H
#define RTPG_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif
#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */
#define RTPG_OK 0
#define RTPG_EINVAL -1   /* bad argument */
#define RTPG_ENOMEM -2   /* device allocation failed */
#define RTPG_ECUDA -3    /* CUDA runtime error */
#define RTPG_ECAPACITY -4 /* a fixed capacity would be exceeded */
#define RTPG_ESTATE -5   /* call not valid in the current state */

/* device status bits (rtpg_sdtree_status / rtpg_mqt_status / ...) */
#define RTPG_STATUS_FX_SATURATED 0x1u      /* a fixed-point value or sum saturated */
#define RTPG_STATUS_DTREE_NODE_CAP 0x2u    /* a quadtree reset hit the per-tree node cap */
#define RTPG_STATUS_STREE_CAPACITY 0x4u    /* spatial refine skipped: STree/DTree capacity */
#define RTPG_STATUS_DNODE_CAPACITY 0x8u    /* quadtree pool capacity exhausted */
#define RTPG_STATUS_HASH_FULL 0x10u        /* a hash bucket was full (slot = UINT32_MAX) */
#define RTPG_STATUS_QUEUE_OVERFLOW 0x20u   /* a wavefront queue overflowed */
#define RTPG_STATUS_TIMEOUT 0x40u          /* a bounded wait on the tensor cores gave up */

const char* rtpg_last_error(void);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int rtpg_version(void);
/* Fixed limits compiled into the library: per-quadtree node cap, maximum quadtree depth,
 * hash bucket size. */
int rtpg_query_limits(uint32_t* host_dtree_node_cap, uint32_t* host_max_dtree_depth, uint32_t* host_hash_block);

/* ================================================================ SD-tree
 * Replaces RTSTreeWrapperT / STreeT / DTreeWrapperT of RTLib
 * (RTLib/Src/Ext/OPX7/Include/RTLib/Ext/OPX7/Utils/OPX7UtilsPathGuiding.h, "PG.h" below).
 * The whole tree lives on the GPU: there is no Upload/Download round trip
 * (PG.h:1353-1615); build, refine and reset run as kernels. */
typedef struct rtpg_sdtree rtpg_sdtree;

typedef struct rtpg_sdtree_caps {
    uint32_t max_stree_nodes;       /* default 1<<20 */
    uint32_t max_dtrees;            /* default 1<<19 */
    uint32_t max_dtree_nodes_total; /* quadtree node pool (building and sampling), default 1<<23 */
    int32_t fixed_point_bits;       /* sums are int64(value * 2^bits); default 24 */
} rtpg_sdtree_caps;

/* RTSTreeWrapperT(ctx, aabbMin, aabbMax, maxDTreeDepth = 20, fraction = 0.3), PG.h:1352.
 * The AABB is cubified to its largest extent (RTSTreeT ctor, PG.h:1211-1217).  caps may be
 * NULL for the defaults.  The new tree is one leaf with a one-node quadtree (PG.h:880-887). */
int rtpg_sdtree_create(const float host_aabb_min[3], const float host_aabb_max[3], uint32_t max_dtree_depth,
                       float fraction, const rtpg_sdtree_caps* caps, rtpg_sdtree** out);
/* RTSTreeWrapperT::Destroy, PG.h:1616-1633 (also frees the handle). */
int rtpg_sdtree_destroy(rtpg_sdtree* h);
/* RTSTreeWrapperT::Clear, PG.h:1634-1636: back to a single leaf with an empty quadtree. */
int rtpg_sdtree_clear(rtpg_sdtree* h, void* stream);

/* Batch of radiance records: STreeT::GetDTreeWrapper (PG.h:639-648) + DTreeWrapperT::Record
 * (PG.h:514-520) + DTreeT::Impl<DirectionalFilterNearest>::RecordIrradiance (PG.h:417-428) +
 * DTreeNodeT::Record (PG.h:113-125), i.e. what TraceVertexT::Commit<Nearest,Nearest> records
 * (PG.h:830-866).  pos: n x float3; dir: n x float2 canonical (dir_is_canonical = 1) or
 * n x float3 unit vectors; radiance: n floats (the channel-averaged local radiance); wo_pdf,
 * stat_weight, is_delta: optional (NULL = 1, 1, 0).  Sums accumulate as int64 fixed point
 * with 64-bit integer atomics, so the result does not depend on record order. */
int rtpg_sdtree_record(rtpg_sdtree* h, int64_t n, const float* pos, const float* dir, int dir_is_canonical,
                       const float* radiance, const float* wo_pdf, const float* stat_weight,
                       const uint8_t* is_delta, void* stream);
/* RTSTreeWrapperT::Build, PG.h:1657-1663 -> RTDTreeWrapperT::Build, PG.h:1086-1090:
 * bottom-up sums, area and root sum of every building quadtree, then sampling = building. */
int rtpg_sdtree_build(rtpg_sdtree* h, void* stream);
/* RTSTreeT::Refine(spatial_threshold, max_mb) (PG.h:1275-1311) followed by
 * RTDTreeWrapperT::Reset(max_dtree_depth, dtree_subdiv_th) on every leaf (PG.h:1091-1094,
 * 888-947).  max_mb < 0 disables the memory-footprint guard. */
int rtpg_sdtree_refine(rtpg_sdtree* h, uint64_t spatial_threshold, int32_t max_mb, float dtree_subdiv_th,
                       void* stream);
/* RTSTreeWrapperT::Reset(iter, samplesPerPass), PG.h:1645-1656: no-op for iter <= 0, else
 * threshold = size_t(sqrt(2^iter * spp / 4) * 4000), refine with 2000 MB, subdiv 0.01. */
int rtpg_sdtree_reset(rtpg_sdtree* h, int32_t iteration, int32_t samples_per_pass, void* stream);
/* Guided sample + pdf for a batch of points, as the closest-hit program uses the guide
 * (SimpleGuide.cu:322-369): leaf = STreeT::GetDTreeWrapper(pos); uv = DTreeT::Sample(rng)
 * (PG.h:478-484, 229-277); pdf_uv = DTreeT::Pdf(uv) (PG.h:485-490).  One Xorshift32 per
 * query seeded with seeds[i] (or, seeds == NULL, with pcg1d(seed_base + i) | 1).
 * Optional outputs (NULL = not written): out_uv n x float2, out_pdf_uv n, out_dir n x float3
 * = normalize(canonical_to_dir(uv)), out_pdf_dir n = DTreeWrapperT::Pdf(out_dir). */
int rtpg_sdtree_sample_pdf(rtpg_sdtree* h, int64_t n, const float* pos, const uint32_t* seeds, uint32_t seed_base,
                           float* out_uv, float* out_pdf_uv, float* out_dir, float* out_pdf_dir, void* stream);
/* DTreeT::Pdf (PG.h:485-490) at given canonical points (dir_is_canonical = 1) or
 * directions (DTreeWrapperT::Pdf, PG.h:529-531). */
int rtpg_sdtree_pdf(rtpg_sdtree* h, int64_t n, const float* pos, const float* dir, int dir_is_canonical,
                    float* out_pdf, void* stream);
/* Sizes of the current tree (synchronises the stream). */
int rtpg_sdtree_stats(rtpg_sdtree* h, uint32_t* host_stree_nodes, uint32_t* host_dtrees,
                      uint32_t* host_dtree_nodes, void* stream);
/* RTSTreeWrapperT::GetMemoryFootPrint (PG.h:1729-1748) analogue: bytes in use on the device. */
int rtpg_sdtree_memory_footprint(rtpg_sdtree* h, uint64_t* host_bytes);
/* Device status word (RTPG_STATUS_* bits), synchronising; clear = 1 resets it. */
int rtpg_sdtree_status(rtpg_sdtree* h, uint32_t* host_status, int clear, void* stream);
/* Canonical export (download for inspection, like RTSTreeWrapperT::Dump, PG.h:1749-1756).
 * Pre-order streams: stree_mask (1 interior / 0 leaf, child 0 first); per leaf 4 floats
 * {building stat-weight, sampling sum, sampling area, sampling stat-weight} and the node
 * count of its quadtree; per quadtree node (pre-order, quadrant 0..3) a child mask byte and
 * 4 float sums.  sampling = 1 exports the sampling trees, 0 the building trees.
 * Call with NULL buffers to get the sizes (host_sizes[3] = {stree nodes, leaves,
 * quadtree nodes}), then with buffers of those sizes.  Synchronises the stream. */
int rtpg_sdtree_export(rtpg_sdtree* h, int sampling, int64_t* host_sizes, uint8_t* host_stree_mask,
                       float* host_leaf_scalars, int64_t* host_leaf_counts, uint8_t* host_dnode_mask,
                       float* host_dnode_sums, void* stream);
/* Inverse of rtpg_sdtree_export, for checkpoints and for trees built elsewhere (e.g. on the
 * host): replaces the whole tree with the one described by the streams of two exports of it,
 * one with sampling = 0 (building quadtrees) and one with sampling = 1 (sampling quadtrees).
 * The STree mask (stree_nodes bytes) and the leaf scalars (4 floats per leaf) are those of
 * either export; each quadtree stream gives per leaf its node count and, per node in pre-order,
 * the child mask and 4 sums (building_nodes / sampling_nodes nodes in all).  Building sums and
 * stat-weights become fixed point (round to nearest), sampling sums stay float, and every
 * sampling tree's guided flag (DTreeT::GetMean() > 0, PG.h:447-451) is recomputed from its
 * scalars, so an exported tree imported again exports identically and samples identically.
 * RTLib's counterpart is RTSTreeWrapperT::Upload (PG.h:1353-1564) of the host trees that
 * RTSTreeWrapperT::Dump (PG.h:1749-1756) writes out.  Synchronises the stream. */
int rtpg_sdtree_import(rtpg_sdtree* h, int64_t stree_nodes, int64_t leaves, const uint8_t* host_stree_mask,
                       const float* host_leaf_scalars, int64_t building_nodes, const int64_t* host_building_counts,
                       const uint8_t* host_building_mask, const float* host_building_sums, int64_t sampling_nodes,
                       const int64_t* host_sampling_counts, const uint8_t* host_sampling_mask,
                       const float* host_sampling_sums, void* stream);

/* ---------------------------------------------------------------- pass controller
 * RTSTreeControllerT (PG.h:1769-1920): the doubling pass schedule.  Host-side state only;
 * begin/end call rtpg_sdtree_reset / rtpg_sdtree_build on the tree at the right moments. */
typedef struct rtpg_controller rtpg_controller;
#define RTPG_TRACE_RECORD 0
#define RTPG_TRACE_RECORD_AND_SAMPLE 1
#define RTPG_TRACE_SAMPLE 2
int rtpg_controller_create(rtpg_sdtree* tree, uint32_t sample_for_budget, uint32_t iteration_for_built,
                           float ratio_for_budget, uint32_t samples_per_launch, rtpg_controller** out);
int rtpg_controller_destroy(rtpg_controller* c);
int rtpg_controller_start(rtpg_controller* c);
int rtpg_controller_begin(rtpg_controller* c, void* stream);
int rtpg_controller_end(rtpg_controller* c, void* stream);
/* state (RTPG_TRACE_*), current iteration, samples done in this pass, whether tracing is
 * still executing. */
int rtpg_controller_get(rtpg_controller* c, int32_t* host_state, uint32_t* host_iteration,
                        uint32_t* host_samples_in_pass, int32_t* host_executing);

/* ================================================================ hash grid
 * Replaces DoubleBufferedHashGrid3T (RTLib/Src/Ext/OPX7/Include/RTLib/Ext/OPX7/Utils/
 * OPX7UtilsGrid.h:157-353, "GR.h") and its host buffer DoubleBufferedHashGrid3Buffer
 * (RTLib/Src/Ext/OPX7/Test/Include/RTLibExtOPX7Test.h:1472-1570, "T.h"). */
typedef struct rtpg_hashgrid rtpg_hashgrid;
#define RTPG_HASH_KEY_REFERENCE 0 /* RTLib's bucket hash (pcg1d chain) and uint32 checksum */
#define RTPG_HASH_KEY_MORTON 1    /* 63-bit Morton code of the cell (21 bits per axis) */
/* DoubleBufferedHashGrid3Buffer::Alloc(gridSize, cellSize) + GetHandle (T.h:1503-1507,
 * 1561-1568): grid `bounds` over [aabb_min, aabb_max], num_slots slots (a multiple of 32,
 * buckets of 32).  max_batch bounds the scratch of one insert chunk (0 = 1<<22). */
int rtpg_hashgrid_create(const float host_aabb_min[3], const float host_aabb_max[3], const uint32_t host_bounds[3],
                         uint32_t num_slots, int32_t keying, uint32_t max_batch, rtpg_hashgrid** out);
int rtpg_hashgrid_destroy(rtpg_hashgrid* h);
/* DoubleBufferedHashGrid3Buffer::Clear (T.h:1529-1543): empty both tables. */
int rtpg_hashgrid_clear(rtpg_hashgrid* h, void* stream);
/* DoubleBufferedHashGrid3Buffer::Update (T.h:1544-1559): previous := current. */
int rtpg_hashgrid_swap(rtpg_hashgrid* h, void* stream);
/* DoubleBufferedHashGrid3T::FindFromCur (GR.h:189-216, 246-277) for a batch of points:
 * out_slot[i] = slot of the point's cell in the current table (inserted if absent), or
 * UINT32_MAX when the bucket is full.  Slots are those of inserting the points one by one
 * in index order.  out_key (optional) receives each point's key. */
int rtpg_hashgrid_insert(rtpg_hashgrid* h, int64_t n, const float* pos, uint32_t* out_slot, uint64_t* out_key,
                         void* stream);
/* DoubleBufferedHashGrid3T::FindFromPrv (GR.h:217-237, 278-300): slot in the previous table
 * or UINT32_MAX. */
int rtpg_hashgrid_lookup(rtpg_hashgrid* h, int64_t n, const float* pos, uint32_t* out_slot, void* stream);
/* Cell coordinates (n x uint3) and keys of points (either output optional). */
int rtpg_hashgrid_cells(rtpg_hashgrid* h, int64_t n, const float* pos, uint32_t* out_cell_xyz, uint64_t* out_key,
                        void* stream);
/* Copy the current (previous = 0) or previous (1) table (num_slots keys, 0 = empty). */
int rtpg_hashgrid_export(rtpg_hashgrid* h, int previous, uint64_t* host_table, void* stream);
int rtpg_hashgrid_status(rtpg_hashgrid* h, uint32_t* host_status, int clear, void* stream);
/* Device pointers of the two tables (uint64 keys), for kernels that probe them directly. */
int rtpg_hashgrid_device_view(rtpg_hashgrid* h, void** dev_current, void** dev_previous);
/* Allocation-free batch insert.  No counterpart in the reference: RTLib only inserts from
 * inside its OptiX programs.  It is for callers that cannot allocate device memory -- a host
 * application that owns every allocation under a fixed budget, code that enqueues work while
 * another component captures the stream into a CUDA graph (where cudaMalloc is not allowed),
 * or a real-time loop that must not block in the allocator.  Same slots and table contents as
 * rtpg_hashgrid_insert on a handle with the same grid: the caller passes the grid parameters,
 * the current table (num_slots uint64 keys, device, in/out, zero = empty), an optional device
 * status word (RTPG_STATUS_HASH_FULL; NULL = not reported), and the points and out_slot.
 * At most 65536 points per call (RTPG_ECAPACITY beyond).  The sort scratch is one
 * file-scope device array of about 7.8 MB that every GPU loading the library reserves until
 * the process exits; the first call on a device looks up its address (make that first call
 * before any stream capture).  All calls share that array, so calls that overlap on the GPU
 * (different streams, or different host threads on one device) race and must be ordered by
 * the caller; each call overwrites the scratch it reads, so nothing carries over. */
int rtpg_hashgrid_insert_noalloc(const float host_aabb_min[3], const float host_aabb_max[3],
                                 const uint32_t host_bounds[3], uint32_t num_slots, int32_t keying, uint64_t* table,
                                 uint32_t* status, int64_t n, const float* pos, uint32_t* out_slot, void* stream);

/* ================================================================ Morton quadtrees
 * Replaces MortonQuadTreeT / MortonQuadTreeWrapperT / RTMortonQuadTreeWrapperT
 * (RTLib/Src/Ext/OPX7/Include/RTLib/Ext/OPX7/Utils/OPX7UtilsMorton.h, "MO.h") and
 * mortonBuildKernel (OPX7UtilsMortonBuild.cu:2-16): one complete quadtree of `level`
 * levels per hash-grid cell. */
typedef struct rtpg_mqt rtpg_mqt;
/* RTMortonQuadTreeWrapperT(ctx, maxHashSize, maxTreeLevel, fraction) + Allocate
 * (MO.h:597-638); leaves accumulate as int64(value * 2^fixed_point_bits) (0 = 24). */
int rtpg_mqt_create(uint32_t num_cells, uint32_t level, float fraction, int32_t fixed_point_bits, rtpg_mqt** out);
int rtpg_mqt_destroy(rtpg_mqt* h);
/* zero the building leaves and the sampling pyramid (Allocate on a live wrapper, MO.h:618-637) */
int rtpg_mqt_clear(rtpg_mqt* h, void* stream);
/* MortonQuadTreeWrapperT::Record (MO.h:477-484) -> MortonQuadTreeT::Record (MO.h:262-285):
 * leaf-only accumulation; cell UINT32_MAX, non-finite and non-positive values are skipped. */
int rtpg_mqt_record(rtpg_mqt* h, int64_t n, const uint32_t* cell, const float* dir, int dir_is_canonical,
                    const float* value, void* stream);
/* RTMortonQuadTreeWrapperT::Update + mortonBuildKernel (MO.h:640-651, 916-941): the sampling
 * pyramid is rebuilt from the building leaves, which are then zeroed. */
int rtpg_mqt_update(rtpg_mqt* h, void* stream);
/* MortonQuadTreeWrapperT::SampleAndPdf (MO.h:486-500): out_pdf includes 1/(4 pi);
 * out_pdf_tree is the tree-level pdf of MortonQuadTreeT::SampleAndPdf (MO.h:286-344). */
int rtpg_mqt_sample_pdf(rtpg_mqt* h, int64_t n, const uint32_t* cell, const uint32_t* seeds, uint32_t seed_base,
                        float* out_uv, float* out_pdf, float* out_dir, float* out_pdf_tree, void* stream);
/* MortonQuadTreeWrapperT::Pdf (MO.h:515-524), or MortonQuadTreeT::Pdf (MO.h:401-414) when
 * tree_level = 1. */
int rtpg_mqt_pdf(rtpg_mqt* h, int64_t n, const uint32_t* cell, const float* dir, int dir_is_canonical, float* out,
                 int tree_level, void* stream);
/* Copy the building leaves (int64) and / or the sampling pyramid (float); NULL skips. */
int rtpg_mqt_export(rtpg_mqt* h, int64_t* host_leaves, float* host_pyramid, void* stream);
int rtpg_mqt_status(rtpg_mqt* h, uint32_t* host_status, int clear, void* stream);

/* RTMortonQuadTreeControllerT (MO.h:766-993): the doubling pass schedule of the hash-grid
 * guide.  States as its TraceState enum; begin at a start clears the quadtrees (Allocate),
 * end after a finished pass beyond iteration_for_built calls rtpg_mqt_update. */
typedef struct rtpg_mqt_controller rtpg_mqt_controller;
#define RTPG_MQT_TRACE_RECORD 0
#define RTPG_MQT_TRACE_RECORD_AND_SAMPLE 1
#define RTPG_MQT_TRACE_SAMPLE 2
#define RTPG_MQT_TRACE_LOCATE 3
int rtpg_mqt_controller_create(rtpg_mqt* tree, uint32_t sample_for_budget, uint32_t iteration_for_built,
                               uint32_t iteration_for_locate, float ratio_for_budget, uint32_t samples_per_launch,
                               rtpg_mqt_controller** out);
int rtpg_mqt_controller_destroy(rtpg_mqt_controller* c);
int rtpg_mqt_controller_start(rtpg_mqt_controller* c);
int rtpg_mqt_controller_begin(rtpg_mqt_controller* c, void* stream);
int rtpg_mqt_controller_end(rtpg_mqt_controller* c, void* stream);
int rtpg_mqt_controller_get(rtpg_mqt_controller* c, int32_t* host_state, uint32_t* host_iteration,
                            uint32_t* host_samples_in_pass, int32_t* host_executing);

/* ================================================================ learned guide
 * No counterpart in RTLib: a 3 x 64 ReLU MLP (inputs: position with 12 sin/cos frequencies per
 * axis, shading normal, outgoing direction) emitting an 8-lobe von Mises-Fisher mixture, with
 * BF16 weights and FP32 accumulation on the tensor cores, trained online by Adam on the
 * radiance records the tracer writes (the SD-tree's record: luminance of incident radiance x
 * |cos| / pdf in the sampled direction), minimising -sum w log q(wi) / sum w. */
typedef struct rtpg_mlp rtpg_mlp;
#define RTPG_MLP_PARAMS 16384 /* fp32 parameters: W0 80x64, W1 64x64, W2 64x64, W3 64x48, [in][out] */
/* aabb: the positions' box (features use the normalised position); seed: initialisation;
 * learning_rate <= 0: 1e-3; record_capacity: records the tracer may write per pass. */
int rtpg_mlp_create(const float* aabb_min, const float* aabb_max, uint32_t seed, float learning_rate,
                    uint32_t record_capacity, rtpg_mlp** out);
int rtpg_mlp_destroy(rtpg_mlp* h);
/* copy the fp32 parameters out (host_get) and / or in (host_set, which also resets Adam) */
int rtpg_mlp_params(rtpg_mlp* h, float* host_get, const float* host_set, void* stream);
/* n samples (device, 3 floats each): raw outputs (48 per sample) and / or the mixture
 * (8 lobes x mu xyz, kappa, weight = 40 per sample); either output may be NULL */
int rtpg_mlp_eval(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, float* out_raw,
                  float* out_lobes, void* stream);
/* gradient of the loss over n records ADDED to grads (device, RTPG_MLP_PARAMS floats, [in][out]);
 * host_loss: the loss (NULL: not read) */
int rtpg_mlp_loss_grad(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, const float* wi,
                       const float* w, float* grads, float* host_loss, void* stream);
/* epochs x (n / batch) Adam steps on the given records, or on the record buffer when pos is
 * NULL; host_last_loss: the last minibatch's loss (NULL: not read) */
int rtpg_mlp_train(rtpg_mlp* h, int64_t n, const float* pos, const float* nrm, const float* wo, const float* wi,
                   const float* w, uint32_t batch, uint32_t epochs, float* host_last_loss, void* stream);
/* records written so far (may exceed the capacity: the excess was dropped); clear = 1 empties */
int rtpg_mlp_records(rtpg_mlp* h, uint32_t* host_count, int clear, void* stream);
int rtpg_mlp_record_arrays(rtpg_mlp* h, float** pos, float** nrm, float** wo, float** wi, float** w);
/* device pointer of the records' sampling densities (1 float per record): the woPdf the tracer
 * sampled the record's direction with, so that the integrand value of a record is w * pdf */
int rtpg_mlp_record_pdfs(rtpg_mlp* h, float** wo_pdf);
int rtpg_mlp_status(rtpg_mlp* h, uint32_t* host_status, int clear, void* stream);
/* Test mode of the bounded waits on the tensor cores (no counterpart in RTLib): skip_mma = 1
 * makes this guide's kernels issue no MMA and no commit, so every completion wait runs out after
 * poll_limit polls; the kernel then sets RTPG_STATUS_TIMEOUT, issues nothing more, frees its
 * tensor memory and returns, leaving the context usable.  skip_mma = 0, poll_limit = 0 restore
 * normal operation (poll limit 2^22). */
int rtpg_mlp_set_wait_test(rtpg_mlp* h, int skip_mma, uint32_t poll_limit);

/* ================================================================ scene / hit queries
 * The integrator's closest-hit and any-hit queries (RTLib: optixTrace inside TraceRadiance /
 * TraceOccluded, RTLib/Src/Ext/OPX7/Test/cuda/SimpleKernel.h:347-366, "SK.h") answered by a
 * linear BVH built on the GPU.  vertices: num_vertices x float3; indices: num_triangles x
 * uint3 (device).  Creation synchronises the stream. */
typedef struct rtpg_scene rtpg_scene;
int rtpg_scene_create(const float* vertices, uint32_t num_vertices, const uint32_t* indices, uint32_t num_triangles,
                      void* stream, rtpg_scene** out);
int rtpg_scene_destroy(rtpg_scene* s);
/* Batched queries: ray n has origin org[3n..], direction dir[3n..], interval (tmin, tmax)
 * (NULL = 0 / 1e20).  any_hit = 0: closest hit (TraceRadiance), 1: any hit (TraceOccluded).
 * out_t = -1 and out_prim = UINT32_MAX on a miss; out_uv: barycentrics (u, v) of vertices
 * 1 and 2 (float2).  Outputs optional. */
int rtpg_scene_intersect(rtpg_scene* s, int64_t n, const float* org, const float* dir, const float* tmin,
                         const float* tmax, int any_hit, float* out_t, uint32_t* out_prim, float* out_uv, void* stream);

/* ================================================================ path tracer
 * The guided integrator of RTLib's OptiX programs (SimpleGuide.cu / SimpleTrace.cu, "SG.cu" /
 * "ST.cu", with SK.h) as a wavefront of CUDA kernels. */
typedef struct rtpg_tracer rtpg_tracer;
/* HitgroupType (SK.h:232-239) */
#define RTPG_MAT_PHONG 0
#define RTPG_MAT_GLASS 1
#define RTPG_MAT_NEE_LIGHT 2 /* emitter that NEE samples (emission counted only after delta bounces / camera rays) */
#define RTPG_MAT_DEF_LIGHT 3 /* emitter outside the NEE list (emission always counted) */
typedef struct rtpg_material {
    float diffuse[3];
    float specular[3];
    float emission[3];
    float shininess;
    float ref_index;
    int32_t type;            /* RTPG_MAT_* */
    int32_t diffuse_texture; /* -1 = none, else index given to rtpg_tracer_set_texture */
} rtpg_material;
/* RayGenData (SK.h:191-199): direction = normalize(x * u + y * v + w), x, y in [-1, 1] */
typedef struct rtpg_camera {
    float eye[3], u[3], v[3], w[3];
} rtpg_camera;
typedef struct rtpg_tracer_desc {
    uint32_t width, height;
    uint32_t max_depth;          /* Params::maxDepth */
    uint32_t num_candidates;     /* RIS candidates (Ris.NumCandidates, default 32) */
    float background[3];         /* MissData::bgColor */
    uint32_t seed;               /* per-pixel Xorshift32 streams are derived from it */
    const float* light_emission; /* host, 3 floats per light mesh (MeshLight::emission) */
} rtpg_tracer_desc;
/* Params::flags (SK.h:145-154) */
#define RTPG_TRACE_FLAG_NEE 1u
#define RTPG_TRACE_FLAG_RIS 2u
#define RTPG_TRACE_FLAG_USE_GRID 4u /* hash-grid + Morton quadtree guide (SimpleGuide2.cu) */
#define RTPG_TRACE_FLAG_USE_TREE 8u /* SD-tree guide (SimpleGuide.cu) */
#define RTPG_TRACE_FLAG_BUILD 16u
#define RTPG_TRACE_FLAG_FINAL 32u
#define RTPG_TRACE_FLAG_LOCATE 64u /* insert unseen cells into the current hash table */
#define RTPG_TRACE_FLAG_USE_MLP 128u /* learned vMF-mixture guide (rtpg_tracer_render_mlp) */
/* tri_vertices: num_triangles x 9 floats (v0, v1, v2 of triangle i, the scene's order);
 * tri_material: uint32 per triangle; tri_uv: 6 floats per triangle or NULL; light_tris:
 * triangle ids of the emitters, light mesh i = light_tris[first[i] .. first[i] + count[i])
 * (MeshLightList, SK.h:107-122).  Device arrays are referenced, not copied. */
int rtpg_tracer_create(rtpg_scene* scene, const float* tri_vertices, const uint32_t* tri_material, const float* tri_uv,
                       const rtpg_material* host_materials, uint32_t num_materials, const uint32_t* light_tris,
                       const uint32_t* host_light_mesh_first, const uint32_t* host_light_mesh_count,
                       uint32_t num_light_meshes, const rtpg_camera* host_camera, const rtpg_tracer_desc* host_desc,
                       rtpg_tracer** out);
int rtpg_tracer_destroy(rtpg_tracer* h);
/* diffuse texture `index`: width x height RGB floats (device, referenced), nearest texel, wrap */
int rtpg_tracer_set_texture(rtpg_tracer* h, uint32_t index, uint32_t width, uint32_t height, const float* rgb);
int rtpg_tracer_set_seed(rtpg_tracer* h, uint32_t seed);
/* zero the FP64 accumulation and reseed the per-pixel streams */
int rtpg_tracer_clear(rtpg_tracer* h, void* stream);
/* `spp` samples per pixel with RTPG_TRACE_FLAG_* (tree required with USE_TREE) */
int rtpg_tracer_render(rtpg_tracer* h, uint32_t spp, uint32_t flags, rtpg_sdtree* tree, void* stream);
/* TracePipeline's loop for the guided tracers: controller begin / render / end, at most
 * max_launches launches of samples_per_launch samples, flags from the controller state. */
int rtpg_tracer_render_guided(rtpg_tracer* h, rtpg_sdtree* tree, rtpg_controller* ctrl, uint32_t base_flags,
                              uint32_t samples_per_launch, uint32_t max_launches, void* stream);
/* `spp` samples per pixel guided by the hash grid and its Morton quadtrees
 * (SimpleGuide2.cu:48-520): flags must hold RTPG_TRACE_FLAG_USE_GRID and not USE_TREE.
 * Every Phong hit looks its cell up in the grid's previous table; with BUILD a found cell's
 * quadtree is mixed into the direction pdf; with LOCATE an unseen cell is inserted into the
 * current table; trace vertices are committed into the quadtrees' building leaves unless
 * FINAL.  mqt must have at least as many cells as the grid has slots. */
int rtpg_tracer_render_grid(rtpg_tracer* h, uint32_t spp, uint32_t flags, rtpg_hashgrid* grid, rtpg_mqt* mqt,
                            void* stream);
/* TracePipeline's loop for the hash-grid tracers (RTLibExtOPX7TestApplication.cpp:2174-2222):
 * controller begin, flags by state (LOCATE: USE_GRID|LOCATE, RECORD: USE_GRID,
 * RECORD_AND_SAMPLE: +BUILD, SAMPLE: +BUILD|FINAL, plus NEE / RIS of base_flags), render,
 * controller end, and the grid's current -> previous copy (rtpg_hashgrid_swap) after every
 * finished pass. */
int rtpg_tracer_render_grid_guided(rtpg_tracer* h, rtpg_hashgrid* grid, rtpg_mqt* mqt, rtpg_mqt_controller* ctrl,
                                   uint32_t base_flags, uint32_t samples_per_launch, uint32_t max_launches,
                                   void* stream);
/* `spp` samples per pixel with the learned guide (no counterpart in RTLib): flags = USE_MLP
 * [| NEE | RIS] [| BUILD: sample the mixture with probability `fraction`, woPdf = (1 - fraction)
 * bsdfPdf + fraction q] [| FINAL: no training records].  Unless FINAL, every committed trace
 * vertex (the SD-tree's record) is appended to the guide's record buffer with probability
 * record_keep, up to its capacity.  fallback (may be NULL): an SD-tree mixed into the guide
 * density, q = mlp_share * network + (1 - mlp_share) * SD-tree, which then also receives the
 * vertices' records (its build / refine stay with the caller or its controller).  The tracer
 * and the guide must be on the same device. */
int rtpg_tracer_render_mlp(rtpg_tracer* h, uint32_t spp, uint32_t flags, rtpg_mlp* mlp, rtpg_sdtree* fallback,
                           float fraction, float mlp_share, float record_keep, void* stream);
/* Emitter radiances (no counterpart in RTLib, which fixes them at load): light mesh i gets
 * host_rgb[3i..3i+2], both as MeshLight::emission for NEE and as the emission of its material.
 * Every light mesh must have its own emissive material. */
int rtpg_tracer_set_light_emission(rtpg_tracer* h, const float* host_rgb, uint32_t num_lights);
/* Path-replay backpropagation (no counterpart in RTLib).  Replays the spp samples that
 * rtpg_tracer_render(h, spp, flags, NULL) would draw from the current per-pixel streams
 * (call rtpg_tracer_clear first to restart them) and ADDS to the gradient buffers the
 * derivatives of a loss whose gradient with respect to the mean image of those samples is
 * d_image (RGB float per pixel, device):
 *   grad_texture        3 floats per texel of diffuse texture texture_index (-1: none);
 *   grad_light_emission 3 floats per light mesh (NULL: none).
 * flags: 0 or RTPG_TRACE_FLAG_NEE (RIS resampling depends on the radiances, guiding on
 * recorded radiance; neither is differentiated).  Per sample, one primal wave recomputes every
 * path's radiance and one adjoint wave replays the path, subtracting each term as it passes
 * it: nothing per vertex is stored.  The accumulation is not touched; the streams advance
 * as the render would advance them. */
int rtpg_tracer_render_adjoint(rtpg_tracer* h, uint32_t spp, uint32_t flags, const float* d_image,
                               int32_t texture_index, float* grad_texture, float* grad_light_emission, void* stream);
/* mean radiance per pixel, width x height x RGB float (device) */
int rtpg_tracer_image(rtpg_tracer* h, float* out_rgb, void* stream);
/* the same in FP64 (double per channel) */
int rtpg_tracer_image_f64(rtpg_tracer* h, double* out_rgb, void* stream);
int rtpg_tracer_accumulation(rtpg_tracer* h, const double** dev_accum, uint64_t* host_samples);
int rtpg_tracer_stats(rtpg_tracer* h, uint64_t* host_samples, uint64_t* host_paths);
/* Device counters since the last clear: path-bounces shaded (bounce visits) and shadow rays
 * traced.  Synchronises the stream. */
int rtpg_tracer_counters(rtpg_tracer* h, uint64_t* host_path_bounces, uint64_t* host_shadow_rays, void* stream);
/* Measurement mode: enable = 1 makes rtpg_tracer_render launch waves without the CUDA graph,
 * bracket every kernel with CUDA events on the stream and synchronise per wave; the summed
 * device milliseconds of raygen / bounce / finish (and their launch counts) are read into
 * three-element arrays with rtpg_tracer_timings.  Enabling or disabling resets the sums. */
int rtpg_tracer_set_timing(rtpg_tracer* h, int enable);
/* Debug view: the final bounce index of every path of the last wave (uint32 per pixel,
 * device); with recording on, a path commits min(depth, 10) trace vertices. */
int rtpg_tracer_path_depths(rtpg_tracer* h, uint32_t* out_depth, void* stream);
int rtpg_tracer_timings(rtpg_tracer* h, double* host_ms3, uint64_t* host_launches3);

#ifdef __cplusplus
}
#endif
#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#endif /* RTPG_H */
