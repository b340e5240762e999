/*
 * warpsolve.h -- C ABI of the B200 (sm_100a) warp-field solver.
 *
 * Drop-in boundary for StarHub's per-frame non-rigid warp-field solve
 * (changhaonan/StarHub).  Every entry point takes plain pointers and sizes
 * (device pointers where noted), returns an int status (WS_OK = 0) and never
 * aborts the process.  The reference interfaces each entry point replaces are
 * cited beside it; paths are relative to the reference repository root.
 *
 * Threading: a ws_solver is used by one host thread at a time.  All device
 * work of a solver is issued on the stream passed to ws_solve; nothing in a
 * solve synchronises the host, so a solve can be captured in a CUDA graph.
 */
#ifndef STARHUB_B200_WARPSOLVE_H
#define STARHUB_B200_WARPSOLVE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define WS_OK 0
#define WS_ERR_INVALID_ARGUMENT (-1)
#define WS_ERR_CAPACITY (-2)        /* input exceeds the capacity given at creation */
#define WS_ERR_CUDA (-3)            /* a CUDA runtime call failed */
#define WS_ERR_NAN (-4)             /* NaN in the right-hand side (WarpSolverPCG.cu:21-31 exits instead) */
#define WS_ERR_TIMEOUT (-5)         /* a bounded device-side wait gave up */
#define WS_ERR_NOT_READY (-6)       /* no inputs set / no solution yet */
#define WS_ERR_NO_DEVICE (-7)

/* Precision modes. */
#define WS_PREC_MIXED 0             /* FP32 bulk, FP64 PCG reductions and FP64 6x6 Cholesky inverse */
#define WS_PREC_FP32 1              /* FP32 everywhere, Gauss-Jordan inverse as the reference */

typedef struct ws_solver ws_solver;

/* Capacities of one solver object (cf. the reference's kMaxNumNodes,
 * image-sized buffers and kMaxNumNodePairs, examples/mono_star/common/Constants.cpp:14-18). */
typedef struct ws_config {
    int max_scenes;             /* scenes per batched solve (1 for the plain path) */
    int max_total_nodes;        /* sum of node counts over a batch */
    int max_total_pixels;       /* sum of width*height over a batch */
    int max_total_edges;        /* sum of node-graph edges over a batch */
    int max_total_features;     /* sum of feature (keypoint) terms over a batch */
    int precision;              /* WS_PREC_MIXED or WS_PREC_FP32 */
    int device;                 /* CUDA device ordinal */
} ws_config;

/*
 * One scene's solver inputs.  Replaces SetSolverInputs' seven structs
 * (examples/mono_star/opt/WarpSolver.h:34-42): Measure4Solver, Render4Solver,
 * OpticalFlow4Solver, KeyPoint4Solver (libs/star/opt/solver_types.h:21-89),
 * Geometry4Solver (libs/star/geometry/surfel/SurfelGeometry.h:76-82),
 * NodeGraph4Solver (libs/star/geometry/node_graph/NodeGraph.h:89-99),
 * NodeFlow4Solver, the camera extrinsic, and the PenaltyConstants
 * (examples/mono_star/opt/PenaltyConstants.cu:8-33).  Image maps are
 * pitch-linear device arrays instead of texture objects; the C++ facade in
 * include/starhub_b200/warp_solver.hpp converts texture objects.
 * Every pointer is a device pointer and must stay valid until the solve ends.
 */
typedef struct ws_inputs {
    int width, height;          /* image size */
    int pitch;                  /* row pitch in texels (0 = width) */
    float fx, fy, cx, cy;       /* pinhole intrinsics of the (downsampled) image */
    float cam2world[16];        /* row-major 4x4 rigid transform */
    const void *measure_vertex_confid;   /* float4 per texel, camera frame */
    const void *measure_normal_radius;   /* float4 per texel, camera frame */
    const void *reference_vertex;        /* float4 per texel, world frame */
    const void *reference_normal;        /* float4 per texel, world frame */
    const uint32_t *index_map;           /* surfel id per texel, 0xFFFFFFFF = none */
    const void *opticalflow;             /* float2 per texel in pixels, NULL = zero flow */
    int num_surfels;
    const uint16_t *surfel_knn;          /* 4 node ids per surfel */
    const float *surfel_knn_spatial_weight;  /* 4 per surfel */
    const float *surfel_knn_connect_weight;  /* 4 per surfel */
    int num_nodes;                       /* <= 65535, includes the two anchor nodes */
    const float *reference_node_coords;  /* float4 per node */
    int num_edges;
    const uint16_t *node_graph;          /* (i, j, k) per edge, j = k-th neighbour of i */
    int graph_k;                         /* neighbours per node (stride of the connect weights) */
    const float *node_knn_connect_weight;/* graph_k per node */
    float node_radius_square;
    const float *node_motion_pred;       /* float4 per node, NULL = none */
    int num_features;
    const uint16_t *feature_knn;         /* 4 node ids per feature term, NULL if none */
    float lambda_depth, lambda_optical_flow, lambda_reg, lambda_node_translation, lambda_feature;
    const float *init_node_se3;          /* 8 floats per node (q0.xyzw, q1.xyzw), NULL = identity */
} ws_inputs;

/* Reference defaults for the penalty weights (PenaltyConstants.cu:8-33). */
void ws_default_penalties(ws_inputs *in);

/* WarpSolver::WarpSolver / AllocateBuffer (examples/mono_star/opt/WarpSolver.cu:50-103). */
int ws_create(const ws_config *config, ws_solver **out);
/* WarpSolver::~WarpSolver (WarpSolver.cu:75-80). */
int ws_destroy(ws_solver *solver);

/* WarpSolver::SetSolverInputs (WarpSolver.cu:125-155): one scene. */
int ws_set_inputs(ws_solver *solver, const ws_inputs *inputs);
/* Batched form: num_scenes independent scenes solved together (no reference counterpart;
 * each scene's result equals the single-scene result bit for bit). */
int ws_set_batch(ws_solver *solver, const ws_inputs *scenes, int num_scenes);

/* WarpSolver::SolveStreamed (WarpSolver.cu:260-279) with the Gauss-Newton and PCG
 * iteration counts as parameters (reference: 6 and 10, Constants.cpp:33, WarpSolver.cu:303).
 * Asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream). */
int ws_solve(ws_solver *solver, int gn_iters, int pcg_iters, void *stream);
/* Same solve launched through a CUDA graph that is captured on first use and replayed. */
int ws_solve_graph(ws_solver *solver, int gn_iters, int pcg_iters, void *stream);

/* Synchronises the solver's last stream and reports device-side errors
 * (timeouts, NaN right-hand side, capacity overflow found on the device). */
int ws_sync_status(ws_solver *solver);

/* WarpSolver::SolvedNodeSE3 / OptimizationProcessorWarpSolver::SolvedSE3
 * (WarpSolver.h:45, OptimizationProcessorWarpSolver.h:28-30): device pointer to
 * 8 floats per node of `scene`, valid until the next ws_set_* on this solver. */
int ws_get_solution(ws_solver *solver, int scene, const float **dev_node_se3, int *num_nodes);

/* ApplySpMVBinBlockCSR::ApplySpMV / BinBlockCSR<6>::SparseMV
 * (libs/star/pcg_solver/ApplySpMVBinBlockCSR.cuh:12-27,92-111, BinBlockCSR.cuh:6-34):
 * y = A x with the block matrix assembled in the last Gauss-Newton iteration of the last
 * solve, for every scene of the batch at once.  x and y are device arrays of 8 floats per
 * node (6 used) in batch order: scene i's nodes follow those of scenes 0..i-1.  In
 * WS_PREC_MIXED the unknowns are node-centred twists (t' = t - c x w), as in the solve.
 * The products meet in y through atomic adds, so y may differ in the last bits between calls.
 * Asynchronous on `stream`; WS_ERR_NOT_READY before the first solve. */
int ws_spmv(ws_solver *solver, const float *x, float *y, void *stream);
/* Failure-detection self-test, no reference counterpart (the reference has no bounded waits):
 * one warp runs the PCG's scene wait on a generation counter that nothing advances.  Returns
 * WS_ERR_TIMEOUT after about two seconds of requested sleep when the bound works (the device
 * stays usable), WS_ERR_CUDA if a CUDA call fails.  Synchronises `stream`. */
int ws_selftest_wait_timeout(void *stream);
/* Failure-detection self-test of the grid barrier that node construction and growth use
 * between the rounds of their overlap check (ws_init_nodes, ws_expand_nodes on more than 16k
 * candidates); no reference counterpart (the reference runs that check on the host).  Two
 * blocks are launched and only one arrives at the barrier, which nothing completes.  Returns
 * WS_ERR_TIMEOUT after about two seconds of requested sleep when the bound works (the device
 * stays usable), WS_OK if the wait ended otherwise, WS_ERR_CUDA if a CUDA call fails.
 * Synchronises `stream`. */
int ws_selftest_grid_barrier_timeout(void *stream);
/* The same operator applied matrix-free from the term records of the last Gauss-Newton
 * iteration (J x per term, then J^T (J x) gathered per node over the node->term lists, plus
 * the diagonal regulariser), without the assembled blocks.  No reference counterpart (the
 * reference materialises A, ApplySpMVBinBlockCSR); it is the ApplySpMVBase plugin point
 * (libs/star/pcg_solver/ApplySpMVBase.h:8-45) filled without a matrix, for callers that
 * cannot hold one.  Allocates 16 bytes per pixel and edge of capacity on first use. */
int ws_spmv_matrix_free(ws_solver *solver, const float *x, float *y, void *stream);

/* Counts of the last index build (host copies; synchronises). */
int ws_get_counts(ws_solver *solver, int scene, int *num_dense_terms, int *num_half_pairs, int *num_n2t_kv);

/* Copies of the index structures of one scene to host memory (synchronise), for parity tests.
 * ImageTermKNNFetcher::GetImageTermPixelAndKNN (ImageTermKNNFetcher.h:55-83). */
int ws_get_dense_terms(ws_solver *solver, int scene, uint16_t *pixels, uint16_t *knn,
                       float *spatial_w, float *connect_w, int capacity, int *count);
/* Node2TermsIndex::GetNode2TermMap (examples/mono_star/opt/Node2TermsIndex.h:79-94). */
int ws_get_node2term(ws_solver *solver, int scene, uint32_t *offsets, uint32_t *term_index,
                     int capacity, int *count);
/* NodePair2TermsIndex::GetNodePair2TermMap (NodePair2TermsIndex.h:44-55): unique (i<j) pairs,
 * their term ranges into term_index, and the sorted pair->term list. */
int ws_get_node_pairs(ws_solver *solver, int scene, uint32_t *rows, uint32_t *cols,
                      uint32_t *begin, uint32_t *end, int capacity, int *count,
                      uint32_t *term_index, int term_capacity, int *term_count);
/* The assembled block system of the last Gauss-Newton iteration: block-CSR with the
 * diagonal block first in every row; A[6*row+r][6*col+c] = blocks[36*k + 6*r + c].
 * JtJMaterializer::AssembleBinBlockCSR (JtJMaterializerBinBlockCSR.cu:44-75). */
int ws_get_system(ws_solver *solver, int scene, uint32_t *rowptr, uint32_t *cols, float *blocks,
                  int block_capacity, int *num_blocks, float *inv_diag, float *jtr, float *step);
/* Dense term residuals (3 per term) and gradients (18 per term) of the last iteration
 * (DenseImageHandler::Term2JacobianMap, DenseImageHandler.cu:384-398). */
int ws_get_dense_jacobian(ws_solver *solver, int scene, float *residual, float *gradient,
                          int capacity, int *count);

/* ---- Node graph, skinning and warp (bit-exact to the reference's integer outputs) ---- */

/* NodeGraph::InitializeNodeGraphFromVertex (libs/star/geometry/node_graph/NodeGraph.cu:460-498):
 * voxel subsample (VoxelSubsamplerSorting.cu:8-96) and the greedy overlap check of
 * AppendNodeFromVertexHost (NodeGraph.cu:652-704), both on the GPU, two anchor nodes prepended.
 * `surfels` is a device float4 array; `nodes_host` receives float4 nodes.  *num_nodes is set
 * also when the count exceeds `capacity` (WS_ERR_CAPACITY); a NaN candidate gives
 * WS_ERR_INVALID_ARGUMENT.  Synchronises `stream`. */
int ws_init_nodes(const float *surfels, int num_surfels, float node_radius, float *nodes_host,
                  int capacity, int *num_nodes, void *stream);
/* NodeGraph::NaiveExpandNodeGraphFromVertexUnsupported (NodeGraph.cu:500-532) with
 * AppendNodeFromVertexHost (NodeGraph.cu:652-704) and updateAppendNodeInitialTime
 * (NodeGraph.cu:316-337), on the GPU: the unsupported vertices (device float4, w ignored) are
 * subsampled on a 0.7 R voxel grid, the candidates that no earlier kept candidate overlaps
 * (0.85 R) are kept, and they are appended (w = 1) after the first *num_nodes nodes of
 * `reference_nodes` and of `live_nodes` (device float4; `live_nodes` may be NULL).  `node_time`
 * (device, may be NULL) gets `current_time` for the appended nodes.  On WS_OK *num_nodes is the
 * new count.  WS_ERR_CAPACITY when it would exceed `capacity`: the arrays are unchanged and
 * *num_nodes holds the count needed.  No vertices: WS_OK, nothing changes.  Synchronises `stream`. */
int ws_expand_nodes(const float *vertices, int num_vertices, float node_radius, float *reference_nodes,
                    float *live_nodes, unsigned *node_time, unsigned current_time, int capacity, int *num_nodes,
                    void *stream);
/* UpdateNodeDistanceKernel + BuildNodeGraphKernel + BuildNodeGraphPairKernel
 * (NodeGraph.cu:10-118): device in/out; k = 4 or 8; edges gets (i, knn[i][k], k).  The
 * n x n half-distance table is not built: each node scans runs of 32 nodes and skips the runs
 * whose bounding box cannot enter its heap (same results).  Asynchronous on `stream`. */
int ws_build_node_graph(const float *nodes, int num_nodes, int k, float node_radius,
                        uint16_t *knn, float *spatial_w, uint16_t *edges, void *stream);
/* SkinnerKernel (libs/star/geometry/node_graph/Skinner.cu:10-94): device in/out, weights divided
 * by their sum (the mono_star configuration's USE_INTERPOLATE_WEIGHT_NORMALIZATION). */
int ws_skinning(const float *nodes, int num_nodes, const float *verts, int num_verts,
                float node_radius, uint16_t *knn, float *spatial_w, float *connect_w, void *stream);

/* Node status: two uint32 per node, (compression, frozen time) as NodeGraph::m_node_status
 * (libs/star/geometry/node_graph/NodeGraph.h:157); a node whose second word is
 * WS_DELETED_NODE_STATUS (NodeGraph.h:18) is left out of the node graph and of skinning. */
#define WS_DELETED_NODE_STATUS 0xFFFFFFFFu
/* ws_build_node_graph with a node status (NULL = no node deleted; a pair with a deleted node has
 * an infinite half distance, NodeGraph.cu:20-35) and a choice of weights: normalize_weights = 1
 * divides each node's K weights by their sum (NodeGraph.cu:87-99 with
 * USE_INTERPOLATE_WEIGHT_NORMALIZATION, examples/mono_star/common/global_configs.h:31-32), 0 keeps
 * the raw __expf weights, which is what the reference's geometry library computes: it is compiled
 * without that header. */
int ws_build_node_graph_ex(const float *nodes, const uint32_t *node_status, int num_nodes, int k, float node_radius,
                           int normalize_weights, uint16_t *knn, float *spatial_w, uint16_t *edges, void *stream);
/* Skinner::PerformSkinningFromRef / PerformSkinningFromLive (Skinner.cu:336-372, kernel :10-94) with
 * a node status (deleted nodes are skipped, Skinner.cu:39-48; NULL = none) and the choice of
 * weights of ws_build_node_graph_ex.  Device in/out. */
int ws_skinning_ex(const float *nodes, const uint32_t *node_status, int num_nodes, const float *verts, int num_verts,
                   float node_radius, int normalize_weights, uint16_t *knn, float *spatial_w, float *connect_w,
                   void *stream);
/* Skinner::PerformIncSkinnningFromLive with IncSkinnerKernel (Skinner.cu:211-302, 395-415): after
 * nodes num_prev_nodes .. num_nodes - 1 were appended, surfels num_remaining_surfels .. num_verts - 1
 * are re-skinned from their current neighbours (`knn` on input, their distances recomputed) and the
 * appended nodes only; earlier surfels are left as they are.  Device in/out. */
int ws_skinning_incremental(const float *nodes, const uint32_t *node_status, int num_nodes, int num_prev_nodes,
                            const float *verts, int num_verts, int num_remaining_surfels, float node_radius,
                            int normalize_weights, uint16_t *knn, float *spatial_w, float *connect_w, void *stream);
/* ForwardWarpVertexAndNodeKernel (libs/star/geometry/surfel/SurfelNodeDeformer.cu:13-79):
 * warps float4 vertices (and optional normals) by the normalized-DQ blend of `num_nodes` node DQs. */
int ws_forward_warp(const float *node_se3, int num_nodes, const float *verts, const float *normals, int num_verts,
                    const uint16_t *knn, const float *spatial_w, const float *connect_w,
                    float *out_verts, float *out_normals, void *stream);
/* Solver-map producer: z-buffered point splat of surfels into index / vertex / normal maps
 * (replaces the OpenGL solver maps, RendererDraw.cu:167-230 with shaders/solver_map.vert:21-53;
 * index = surfel id, vertex/normal copied from `attr_verts`/`attr_normals`).  `verts` are
 * positions in the camera frame used for projection.  `footprint` is the splat half-width in
 * pixels.  Writes width*height texels of every output; empty texels get index 0xFFFFFFFF and
 * zero vectors. */
int ws_splat_maps(const float *verts, const float *attr_verts, const float *attr_normals,
                  int num_verts, int width, int height, float fx, float fy, float cx, float cy,
                  int footprint, uint32_t *index_map, float *vertex_map, float *normal_map,
                  void *stream);
/* Solver maps as the reference's solver-map pass draws them (Render4Solver): Renderer::DrawSolverMaps
 * and DrawSolverMapsWithRecentObservation (libs/star/geometry/render/RendererDraw.cu:105-175) with
 * shaders/solver_map.vert:21-53 and solver_map.frag:10-17, on the GPU without a graphics stack.
 * Surfels (device float4 arrays): vertex_confid (world xyz, confidence), normal_radius (world
 * normal, radius) and color_time (x: colour bytes as float bits, z: last observed time; NULL = every
 * surfel observed at current_time).  A surfel is drawn unless its camera-frame z is > max_depth or
 * <= 0, or its confidence is below confidence_threshold while |time - current_time| >=
 * time_threshold (-1: every unstable surfel is culled); it lands in pixel floor(f x / z + c + 0.5)
 * and the `footprint` pixels around it (0 = the single pixel of a unit point), the nearest z wins and
 * equal depths keep the lower surfel id.  Writes width*height texels of each non-NULL output:
 * index (surfel id, 0xFFFFFFFF = none), vertex (xyz, 1), normal (xyz, 0), rgbd (colour / 127.5 - 1,
 * 1 / z); empty texels are zero.  The depth compare is on the float camera z (the GL depth buffer
 * quantises it). */
typedef struct ws_render_params {
    int width, height;
    float fx, fy, cx, cy;
    float world2camera[16];     /* row-major 4x4 */
    float max_depth;            /* width_height_maxdepth_currtime.z */
    float current_time;         /* width_height_maxdepth_currtime.w */
    float confidence_threshold; /* confid_time_threshold.x (d_stable_surfel_confidence_threshold = 1) */
    float time_threshold;       /* confid_time_threshold.y (d_rendering_recent_time_threshold = 3, or -1) */
    int footprint;
} ws_render_params;
int ws_render_solver_maps(const float *vertex_confid, const float *normal_radius, const float *color_time,
                          int num_surfels, const ws_render_params *params, uint32_t *index_map, float *vertex_map,
                          float *normal_map, float *rgbd_map, void *stream);
/* Observation maps as Renderer::DrawObservationMaps (libs/star/geometry/render/RendererDraw.cu:353-394)
 * draws them with shaders/geometry.vert:40-86 and observation_map.frag:13-17, with
 * GL_PROGRAM_POINT_SIZE on (Renderer.cu:87-90).  Same inputs, transform, culls and depth rule as
 * ws_render_solver_maps (drawn iff 0 < z < max_depth and not an unstable surfel outside the time
 * threshold; nearest z, equal depths to the lower id), but normal_radius is required and each
 * surfel is a point as wide as its disk's image: the smaller image extent of the four points
 * v_cam +- x1, v_cam +- y1 (x1 = normalize(n.y - n.z, -n.x, n.x) * radius * 1.41421356 mm in the
 * camera frame, y1 = n x x1), clamped to [1, 2047]; it covers the pixels i with
 * u - S/2 < i <= u + S/2 around u = f x / z + c (rows likewise).  params->footprint is unused.
 * Writes width*height texels: index (surfel id, 0xFFFFFFFF = none) and, when rgbd_map is not
 * NULL, rgbd = ((colour byte / 255) * 2 - 1 for r, g, b; 1 / z); empty texels are zero. */
int ws_render_observation_maps(const float *vertex_confid, const float *normal_radius, const float *color_time,
                               int num_surfels, const ws_render_params *params, uint32_t *index_map, float *rgbd_map,
                               void *stream);
/* Measurement maps from a depth image in millimetres (device, `pitch` elements per row):
 * createVertexConfidMapKernel (libs/star/img_proc/vertex_map.cu:13-33), the depth clip of
 * filterAndScaleVertexKernel (libs/star/geometry/geometry_map/SurfelMapInitializer.cu:107-137,
 * here on the depth in metres at full resolution) and createNormalRadiusMapKernel with eigen33
 * (libs/star/img_proc/normal_map.cu:32-118, libs/star/math/eigen33.hpp).  Writes width*height
 * float4 texels of each output: vertex_confid = (x, y, z, 1), or zeros outside the clip;
 * normal_radius = (normal facing the camera, radius in mm), or zeros where fewer than half of
 * the 7x7 window holds vertices. */
int ws_measure_maps(const uint16_t *depth_mm, int width, int height, int pitch, float fx, float fy,
                    float cx, float cy, float clip_near, float clip_far, float radius_scale,
                    float *vertex_confid, float *normal_radius, void *stream);

/* ---- Measurement hooks ---- */

/* Enables (1) or disables (0) per-phase CUDA-event timing of ws_solve on the solve stream
 * (disabled inside graph capture).  Phases: 0 index build, 1 term evaluation, 2 diagonal
 * blocks + right-hand side, 3 off-diagonal blocks, 4 persistent PCG + warp update. */
int ws_set_profiling(ws_solver *solver, int enable);
/* Milliseconds per phase of the last profiled solve, summed over its Gauss-Newton
 * iterations (synchronises).  `launches` (optional) gets the launches of each phase. */
int ws_get_phase_times(ws_solver *solver, float *ms, int *launches, int capacity, int *count);
/* Kernel launches in one replay of the graph captured by ws_solve_graph. */
int ws_graph_kernel_count(ws_solver *solver, int *count);

/* ws_splat_maps without any device allocation.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc or cudaMallocAsync once they are running: a
 * frame loop or serving process that reserves its whole device budget at start-up and
 * admits work by footprint, or a host whose own pool owns all device memory.  Such a
 * caller must not have an allocation fail, or block, in the middle of a frame.
 * The z-buffer scratch is a file-scope __device__ array of WS_NOALLOC_MAX_PIXELS 64-bit
 * keys (7.4 MB), which every GPU that loads this library holds until the process exits.
 * The first call on a device looks up that array's device address (cudaGetSymbolAddress)
 * with that device current, so make the first call before any stream capture.  Every call
 * shares the one array and clears it on `stream` before use, so calls that overlap on the
 * GPU race.  width * height above WS_NOALLOC_MAX_PIXELS returns WS_ERR_CAPACITY. */
#define WS_NOALLOC_MAX_PIXELS (1280 * 720)
int ws_splat_maps_noalloc(const float *verts, const float *attr_verts, const float *attr_normals,
                          int num_verts, int width, int height, float fx, float fy, float cx, float cy,
                          int footprint, uint32_t *index_map, float *vertex_map, float *normal_map,
                          void *stream);

/* ---- Serving: a persistent request loop with continuous batching -----------------------
 * No reference counterpart: the reference solves one frame of one stream per call
 * (OptimizationProcessorWarpSolver::ProcessFrame).  A server keeps the node graph, surfel
 * skinning and warp of every registered stream resident on its device, takes one frame
 * per request, and solves the requests that are waiting as batches on `executors` streams,
 * so that batches overlap on the device.  A new batch starts as soon as an executor is free,
 * from the oldest waiting frames that fit its capacities, at most one frame per stream
 * (a stream's frames are solved in submission order, each starting from the warp its
 * previous frame produced).  A request's result is bit-identical whatever it was batched with.
 * Memory admission: executors are sized at creation and scenes are admitted by the bytes they
 * keep resident; the sum never exceeds memory_budget. */
typedef struct ws_server ws_server;

typedef struct ws_server_config {
    int device;
    unsigned long long memory_budget; /* bytes of device memory for executors + resident scenes */
    int executors;              /* batches in flight at once (one stream and solver each) */
    int max_batch_scenes;       /* capacities of one batch (one executor) */
    int max_batch_nodes;
    int max_batch_pixels;
    int max_batch_edges;
    int gn_iters, pcg_iters;    /* per solve */
    int precision;              /* WS_PREC_MIXED or WS_PREC_FP32 */
} ws_server_config;

/* One frame of a stream: non-owning device views, valid until the request is done. */
typedef struct ws_frame {
    const void *measure_vertex_confid;
    const void *measure_normal_radius;
    const void *reference_vertex;
    const void *reference_normal;
    const uint32_t *index_map;
    const void *opticalflow;          /* NULL = zero flow */
    int pitch;                        /* texels, 0 = width */
    float cam2world[16];
    const float *node_motion_pred;    /* NULL = none */
    float *solution_out;              /* optional device buffer (8 floats per node) that receives
                                         this frame's solution; NULL = only the resident warp */
} ws_frame;

typedef struct ws_request_info {
    int status;                 /* WS_OK when solved, WS_ERR_NOT_READY while waiting or running */
    int scene;                  /* stream (scene) id */
    int num_nodes;
    int batch_scenes;           /* frames in the batch that solved it */
    double queue_ms;            /* submit -> batch launch (host clock) */
    double solve_ms;            /* batch launch -> batch done */
    double latency_ms;          /* submit -> done */
} ws_request_info;

typedef struct ws_server_stats {
    unsigned long long submitted, completed, failed, batches;
    double mean_batch_scenes;
    double p50_latency_ms, p99_latency_ms, mean_latency_ms;   /* over completed requests */
    unsigned long long executor_bytes, resident_bytes, memory_budget;
    int scenes;
} ws_server_stats;

/* Creates the executors (WS_ERR_CAPACITY if they alone exceed memory_budget) and starts the
 * scheduler and completion threads. */
int ws_server_create(const ws_server_config *cfg, ws_server **out);
/* Finishes the batches in flight, drops waiting requests, frees everything. */
int ws_server_destroy(ws_server *s);
/* Copies a stream's static state (surfel knn and weights, node coordinates, graph, connect
 * weights, camera, penalties) and its initial warp into resident device memory.  Map fields
 * of `scene` are ignored.  WS_ERR_CAPACITY if the resident bytes would exceed the budget. */
int ws_server_add_scene(ws_server *s, const ws_inputs *scene, int *scene_id);
/* WS_ERR_NOT_READY while the scene has frames waiting or in flight. */
int ws_server_remove_scene(ws_server *s, int scene_id);
/* Queues one frame of a stream.  WS_ERR_CAPACITY if the scene alone exceeds a batch. */
int ws_submit(ws_server *s, int scene_id, const ws_frame *frame, unsigned long long *request_id);
/* Non-blocking status; a finished request stays queryable until ws_server_forget. */
int ws_poll(ws_server *s, unsigned long long request_id, ws_request_info *info);
/* Blocks until the request is done (or the server stops). */
int ws_wait(ws_server *s, unsigned long long request_id, ws_request_info *info);
int ws_server_forget(ws_server *s, unsigned long long request_id);
/* The stream's resident warp (its latest solution), device pointer to 8 floats per node. */
int ws_server_get_warp(ws_server *s, int scene_id, const float **dev_dq, int *num_nodes);
/* Copies the stream's resident warp into `dev_out` (device, 8 floats per node) and waits for
 * the copy; WS_ERR_NOT_READY while the stream has frames waiting or in flight. */
int ws_server_copy_warp(ws_server *s, int scene_id, float *dev_out);
/* Overwrites the stream's resident warp from device memory (8 floats per node);
 * WS_ERR_NOT_READY while the stream has frames waiting or in flight. */
int ws_server_set_warp(ws_server *s, int scene_id, const float *dev_dq);
int ws_server_get_stats(ws_server *s, ws_server_stats *stats);

/* ---- Autotuning of launch shapes ------------------------------------------------------
 * No reference counterpart.  ws_autotune runs one Gauss-Newton iteration of the inputs set on
 * the solver, then times, on that data, the node and pair assembly kernels at 64, 128 and
 * 256 threads per block (the FP64 node kernel offers 64 and 128) and the persistent PCG at
 * 1..k blocks per SM (k = what fits on an SM), which sets how many rows each warp owns; it keeps
 * the fastest of each for the solver's later solves and reports the timings.  No choice changes
 * a result: every sum runs in the same order at every shape.  Synchronises `stream`. */
typedef struct ws_tuning {
    int node_threads;           /* chosen threads per block, node assembly */
    int pair_threads;           /* chosen threads per block, pair assembly */
    int pcg_blocks_per_sm;      /* chosen PCG blocks per SM */
    float node_ms[3];           /* per candidate 64 / 128 / 256 threads; < 0 = not offered */
    float pair_ms[3];
    float pcg_ms[8];            /* per candidate 1..8 blocks per SM; < 0 = not offered */
} ws_tuning;
int ws_autotune(ws_solver *solver, int pcg_iters, void *stream, ws_tuning *result);
/* Applies a tuning (e.g. one stored from an earlier ws_autotune on the same workload). */
int ws_set_tuning(ws_solver *solver, const ws_tuning *tuning);

/* Library version / build identification. */
int ws_version(void);
const char *ws_error_string(int status);

#ifdef __cplusplus
}
#endif
#endif
