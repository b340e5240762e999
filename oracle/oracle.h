/*
 * CPU oracle for StarHub's per-frame warp-field solve -- TEST INFRASTRUCTURE ONLY.
 *
 * This header and warp_oracle.cpp restate, in plain C++ on the host, the
 * algorithm that StarHub (changhaonan/StarHub) runs on the GPU for one frame:
 * node construction, node graph, skinning, pixel-term compaction, the
 * node->term and node-pair->term indices, Gauss-Newton with a point-to-plane
 * depth term, an optical-flow term and node-graph ARAP smoothness, and a
 * block-Jacobi PCG on 6x6 node blocks.  It is the checker for the CUDA
 * library in starhub_b200/ and the timed CPU baseline of bench.py; nothing in
 * the product links or calls it.
 *
 * Parity status: parity unpinned.  The reference ships no tests, golden
 * vectors or fixtures for this path, and its sources cannot be compiled here
 * (every header on the path includes Eigen, OpenCV, PCL, Boost and
 * nlohmann-json, none of which is present).  The restatement follows the
 * reference sources line by line (file:line cited at each function) and is
 * pinned by first-principles known-answer tests under tests/.
 */
#ifndef STARHUB_ORACLE_H
#define STARHUB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One camera, one frame.  All image maps are row-major, width*height texels. */
typedef struct orc_problem {
    int width, height;
    float fx, fy, cx, cy;
    float world2cam[12];            /* row-major [R | t] */
    const float *measure_vertex;    /* float4 per pixel, camera frame, w = confidence */
    const float *measure_normal;    /* float4 per pixel, camera frame, w = radius */
    const float *ref_vertex;        /* float4 per pixel, world frame */
    const float *ref_normal;        /* float4 per pixel, world frame */
    const uint32_t *index_map;      /* surfel id per pixel, 0xFFFFFFFF = empty */
    const float *flow;              /* float2 per pixel (pixels), NULL = zero flow */
    int num_surfels;
    const uint16_t *surfel_knn;     /* 4 node ids per surfel */
    const float *surfel_sw;         /* 4 spatial weights per surfel */
    const float *surfel_cw;         /* 4 connect weights per surfel */
    int num_nodes;
    const float *node_coords;       /* float4 per node (reference frame) */
    int graph_k;                    /* neighbours per node in the node graph (self included) */
    int num_edges;
    const uint16_t *edges;          /* (i, j, k) per edge */
    const float *node_cw;           /* graph_k connect weights per node */
    float node_radius_square;
    const float *node_motion_pred;  /* float4 per node or NULL */
    int num_features;
    const uint16_t *feature_knn;    /* 4 node ids per feature term or NULL */
    const float *init_dq;           /* 8 floats per node (q0.xyzw, q1.xyzw) or NULL = identity */
} orc_problem;

enum {
    ORC_PREC_FP64 = 0,              /* everything in double: the accuracy oracle */
    ORC_PREC_FP32_REFERENCE = 1,    /* float everywhere, Gauss-Jordan inverse, float dots */
    ORC_PREC_MIXED = 2,             /* float bulk with double dots, double block accumulation and
                                       Cholesky, cancellation-free residuals: the device's design */
};

typedef struct orc_settings {
    int gn_iters;
    int pcg_iters;
    float lambda_depth, lambda_of, lambda_reg, lambda_node, lambda_feature;
    int precision;
    int threads;                    /* OpenMP threads, <= 0 = all */
} orc_settings;

/* First-iteration intermediates for stage-level parity (all optional, NULL = skip). */
typedef struct orc_debug {
    int capacity_terms;             /* capacity of the per-dense-term arrays */
    int capacity_pairs;             /* capacity of the symmetric off-diagonal arrays */
    int num_dense_terms;            /* out */
    int num_sym_pairs;              /* out */
    float *dense_residual;          /* 3 per dense term */
    float *dense_gradient;          /* 18 per dense term */
    float *diag_blocks;             /* 36 per node, before inversion (includes +1e-3) */
    float *inv_diag_blocks;         /* 36 per node */
    float *jtr;                     /* 6 per node */
    uint32_t *sym_rows, *sym_cols;  /* symmetric off-diagonal entries, sorted by (row, col) */
    float *offdiag_blocks;          /* 36 per symmetric entry: A[6*row+r][6*col+c] at r*6+c */
    float *pcg_x;                   /* 6 per node: the first Gauss-Newton step */
} orc_debug;

int orc_version(void);

/* Node construction (NodeGraph::InitializeNodeGraphFromVertex). */
int orc_voxel_subsample(const float *pts4, int n, float voxel, float *out4, int cap, int *n_out);
int orc_init_nodes(const float *pts4, int n, float node_radius, float *out4, int cap, int *n_nodes);
int orc_node_graph(const float *nodes4, int n, int k, float node_radius,
                   uint16_t *knn, float *spatial_w);
int orc_skinning(const float *nodes4, int n_nodes, const float *verts4, int n_verts,
                 float node_radius, uint16_t *knn, float *spatial_w, float *connect_w, int threads);
/* The same with node status (2 words per node, NULL = none deleted; .y == 0xFFFFFFFF is a deleted
 * node, NodeGraph.h:18), weights divided by their sum or not, and for skinning the incremental form
 * of IncSkinnerKernel (Skinner.cu:211-302: surfels first_vert.. keep their knn and take the nodes
 * prev_nodes..). */
int orc_node_graph_ex(const float *nodes4, const uint32_t *status, int n, int k, float node_radius, int normalize,
                      uint16_t *knn, float *spatial_w);
int orc_skinning_ex(const float *nodes4, const uint32_t *status, int n_nodes, int prev_nodes, const float *verts4,
                    int first_vert, int n_verts, float node_radius, int normalize, uint16_t *knn, float *spatial_w,
                    float *connect_w, int threads);

/* Index build. */
int orc_compact_pixels(int width, int height, const uint32_t *index_map, const float *flow,
                       const uint16_t *surfel_knn, const float *surfel_sw, const float *surfel_cw,
                       uint16_t *pixels, uint16_t *knn, float *sw, float *cw, int cap, int *n_terms);
int orc_node2term(int n_dense, const uint16_t *dense_knn, int n_edges, const uint16_t *edges,
                  int n_nodes, int n_feat, const uint16_t *feat_knn,
                  uint32_t *offsets, uint32_t *term_index, int cap_kv, int *n_kv);
int orc_nodepair2term(int n_dense, const uint16_t *dense_knn, int n_edges, const uint16_t *edges,
                      int n_nodes, int n_feat, const uint16_t *feat_knn,
                      uint32_t *half_rows, uint32_t *half_cols, uint32_t *half_begin,
                      uint32_t *half_end, int cap_half, int *n_half,
                      uint32_t *term_index, int cap_kv, int *n_kv,
                      uint32_t *sym_rows, uint32_t *sym_cols, uint32_t *sym_begin,
                      uint32_t *sym_end, uint32_t *blkrow_offset);
int orc_binblock_csr(int n_nodes, int n_sym, const uint32_t *sym_rows, const uint32_t *sym_cols,
                     int *rowptr, int cap_rowptr, int *n_rowptr, int *colptr, int cap_colptr);

/* The solve. */
int orc_solve(const orc_problem *p, const orc_settings *s, float *out_dq, orc_debug *dbg);

/* SurfelNodeDeformer::ForwardWarpVertexAndNode for the warped-position metric. */
int orc_forward_warp(const float *node_dq, int n_nodes, const float *verts4, int n_verts,
                     const uint16_t *knn, const float *sw, const float *cw, float *out4, int threads);

/* Measurement maps from a depth image in millimetres: createVertexConfidMapKernel
 * (img_proc/vertex_map.cu:13-33), the clip of filterAndScaleVertexKernel
 * (geometry_map/SurfelMapInitializer.cu:107-137, on the depth in metres) and
 * createNormalRadiusMapKernel with eigen33 (img_proc/normal_map.cu:32-118, math/eigen33.hpp),
 * in FP32 with the reference's host arithmetic (1 / sqrt for the inverse square roots).
 * Outputs width*height float4 each. */
int orc_measure_maps(const uint16_t *depth_mm, int width, int height, float fx, float fy, float cx, float cy,
                     float clip_near, float clip_far, float radius_scale, float *vertex4, float *normal4);

/* The solver-map pass (Renderer::DrawSolverMaps, RendererDraw.cu:105-175, with
 * shaders/solver_map.vert:21-53 and solver_map.frag:10-17): per surfel the camera transform
 * ((m0 x + m1 y) + m2 z) + m3, the culls (z > max depth or z <= 0 or the depth buffer's far plane;
 * confidence < conf_threshold with |time - current| >= time_threshold), the pixel
 * floor(f x / z + c + 0.5) and `footprint` pixels around it, nearest z first, equal z to the lower
 * id.  world2camera is row-major 4x4; color_time may be NULL.  Outputs width*height texels each:
 * index (0xFFFFFFFF = none), vertex (xyz, 1), normal (xyz, 0), rgbd (colour / 127.5 - 1, 1 / z). */
int orc_render_solver_maps(const float *vertex_confid4, const float *normal_radius4, const float *color_time4,
                           int n, int width, int height, float fx, float fy, float cx, float cy,
                           const float *world2camera, float max_depth, float current_time,
                           float conf_threshold, float time_threshold, int footprint, uint32_t *index_map,
                           float *vertex4, float *normal4, float *rgbd4);
/* The observation-map pass (Renderer::DrawObservationMaps, libs/star/geometry/render/
 * RendererDraw.cu:353-394, shaders/geometry.vert:40-86 and observation_map.frag:13-17): the same
 * camera transform, confidence/time cull and depth rule as the solver-map pass (drawn iff
 * 0 < z < max depth), but each surfel is a GL point whose size is the smaller image extent of its
 * disk (four points v_cam +- x1, +- y1 of radius * 1.41421356 mm), clamped to [1, 2047]; it covers
 * the pixels i with u - S/2 < i <= u + S/2 around u = f x / z + c (rows likewise).  Outputs
 * width*height texels: index (0xFFFFFFFF = none) and rgbd ((colour / 255) * 2 - 1, 1 / z). */
int orc_render_observation_maps(const float *vertex_confid4, const float *normal_radius4, const float *color_time4,
                                int n, int width, int height, float fx, float fy, float cx, float cy,
                                const float *world2camera, float max_depth, float current_time,
                                float conf_threshold, float time_threshold, uint32_t *index_map, float *rgbd4);

#ifdef __cplusplus
}
#endif
#endif
