// warp_solver.hpp -- header-only C++ facade over include/warpsolve.h.
//
// Re-creates the call surface of StarHub's solver so the per-frame pipeline
// keeps its call sites:
//   * star::b200::WarpSolver mirrors star::WarpSolver
//     (examples/mono_star/opt/WarpSolver.h:34-52): SetSolverInputs,
//     SolveStreamed, SolvedNodeSE3;
//   * star::b200::OptimizationProcessorWarpSolver mirrors the processor entry
//     (examples/mono_star/opt/OptimizationProcessorWarpSolver.h:18-30):
//     ProcessFrame with the reference's seven input structs, the frame index and the
//     stream (frame 0 is a no-op, OptimizationProcessorWarpSolver.cu:35-36), and
//     SolvedSE3, which converts to GArrayView<DualQuaternion>;
//   * the input structs (Measure4Solver ... KeyPoint4Solver, GArrayView, floatX,
//     DualQuaternion, Extrinsic) with the reference's members, for callers without
//     the reference's headers (the calls are templates and take the reference's own);
//   * star::b200::NodeGraph mirrors the node construction and growth of
//     star::NodeGraph (libs/star/geometry/node_graph/NodeGraph.h:23-60):
//     InitializeNodeGraphFromVertex, NaiveExpandNodeGraphFromVertexUnsupported,
//     BuildNodeGraphFromScratch and the accessors of the node arrays.
// Maps arrive as cudaTextureObject_t like in Measure4Solver / Render4Solver
// (libs/star/opt/solver_types.h:21-37); TextureMap resolves a texture object to
// the pitch-linear device array the C ABI reads (pitch-2D resources are used in
// place, CUDA arrays are copied into an owned pitched buffer on the solve stream).
// Errors are reported as exceptions carrying the C status (the reference aborts).
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../warpsolve.h"

namespace star {
namespace b200 {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string &what) : std::runtime_error(what + ": " + ws_error_string(s)), status(s) {}
};

inline void check(int s, const char *what) {
    if (s != WS_OK) throw Error(s, what);
}

// Pitch-linear view of a texture object's texels.
class TextureMap {
public:
    TextureMap() = default;
    TextureMap(const TextureMap &) = delete;
    TextureMap &operator=(const TextureMap &) = delete;
    ~TextureMap() { if (owned_) cudaFree(owned_); }

    // Resolves `tex` (width x height texels of `texel_bytes`) and returns a device pointer
    // with a row pitch of `width` texels.
    const void *resolve(cudaTextureObject_t tex, int width, int height, size_t texel_bytes, cudaStream_t st) {
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        check(cudaGetTextureObjectResourceDesc(&rd, tex) == cudaSuccess ? WS_OK : WS_ERR_CUDA, "texture resource");
        const size_t row = (size_t)width * texel_bytes;
        if (rd.resType == cudaResourceTypePitch2D && rd.res.pitch2D.pitchInBytes == row)
            return rd.res.pitch2D.devPtr;
        if (!owned_ || owned_bytes_ < row * height) {
            if (owned_) cudaFree(owned_);
            check(cudaMalloc(&owned_, row * height) == cudaSuccess ? WS_OK : WS_ERR_CUDA, "texture copy buffer");
            owned_bytes_ = row * height;
        }
        cudaError_t e;
        if (rd.resType == cudaResourceTypePitch2D)
            e = cudaMemcpy2DAsync(owned_, row, rd.res.pitch2D.devPtr, rd.res.pitch2D.pitchInBytes, row, height,
                                  cudaMemcpyDeviceToDevice, st);
        else if (rd.resType == cudaResourceTypeArray)
            e = cudaMemcpy2DFromArrayAsync(owned_, row, rd.res.array.array, 0, 0, row, height,
                                           cudaMemcpyDeviceToDevice, st);
        else
            e = cudaErrorInvalidValue;
        check(e == cudaSuccess ? WS_OK : WS_ERR_CUDA, "texture copy");
        return owned_;
    }

private:
    void *owned_ = nullptr;
    size_t owned_bytes_ = 0;
};

// ---- Types with the reference's member names and layouts ------------------------------
// The facade's solver calls are templates over the seven input structs, so a pipeline that
// includes the reference's own headers passes star::Measure4Solver ... star::KeyPoint4Solver
// unchanged.  A caller without those headers uses these: same names, same members, same
// layouts (libs/star/opt/solver_types.h:21-89, NodeGraph.h:89-99, SurfelGeometry.h:76-82,
// libs/star/common/ArrayView.h:13-47, libs/star/common/types/floatX.h, ushortX.h,
// libs/star/math/DualQuaternion.hpp:206, common_types.h:55-94).
constexpr unsigned d_max_cam = 3;            // libs/star/common/constants.h:6
constexpr unsigned d_node_knn_size = 4;      // libs/star/geometry/constants.h:6
constexpr unsigned d_surfel_knn_size = 4;    // libs/star/geometry/constants.h:7

template <typename T>
class GArrayView {
public:
    GArrayView() = default;
    GArrayView(const T *arr, size_t size) : m_array(arr), m_array_size(size) {}
    size_t Size() const { return m_array_size; }
    size_t ByteSize() const { return m_array_size * sizeof(T); }
    const T *Ptr() const { return m_array; }
    operator const T *() const { return m_array; }

private:
    const T *m_array = nullptr;
    size_t m_array_size = 0;
};

template <unsigned dim>
struct floatX {
    float data[dim];
};
template <unsigned dim>
struct ushortX {
    unsigned short data[dim];
};

struct Quaternion {
    float4 q0;                               // (x, y, z, w)
};
struct DualQuaternion {
    Quaternion q0, q1;                       // real and dual part, 32 bytes
};
static_assert(sizeof(DualQuaternion) == 32, "DualQuaternion is 8 floats");

struct Intrinsic {
    float principal_x = 0.f, principal_y = 0.f, focal_x = 0.f, focal_y = 0.f;
};

// A 4x4 float matrix stored column-major with Eigen::Matrix4f's element access, so that
// `const Extrinsic *camera2world` reads the same either way.
struct Extrinsic {
    float m[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    float &operator()(int r, int c) { return m[c * 4 + r]; }
    float operator()(int r, int c) const { return m[c * 4 + r]; }
    static Extrinsic Identity() { return Extrinsic(); }
};

struct Measure4Solver {
    cudaTextureObject_t vertex_confid_map[d_max_cam];
    cudaTextureObject_t normal_radius_map[d_max_cam];
    cudaTextureObject_t index_map[d_max_cam];
    unsigned num_cam;
};
struct Render4Solver {
    cudaTextureObject_t reference_vertex_map[d_max_cam];
    cudaTextureObject_t reference_normal_map[d_max_cam];
    cudaTextureObject_t index_map[d_max_cam];
    unsigned num_cam;
};
struct OpticalFlow4Solver {
    cudaTextureObject_t opticalflow_map[d_max_cam];
    unsigned num_cam;
};
struct NodeFlow4Solver {
    GArrayView<float4> node_motion_pred;
    unsigned num_node;
};
struct KeyPoint4Solver {
    GArrayView<int2> kp_match;
    GArrayView<float4> d_kp_vertex_confid;
    GArrayView<float4> d_kp_normal_radius;
    GArrayView<float4> kp_vertex_confid;
    GArrayView<float4> kp_normal_radius;
    GArrayView<ushortX<d_surfel_knn_size>> kp_knn;
    GArrayView<floatX<d_surfel_knn_size>> kp_knn_spatial_weight;
    GArrayView<floatX<d_surfel_knn_size>> kp_knn_connect_weight;
};
struct Geometry4Solver {
    GArrayView<ushortX<d_surfel_knn_size>> surfel_knn;
    GArrayView<floatX<d_surfel_knn_size>> surfel_knn_spatial_weight;
    GArrayView<floatX<d_surfel_knn_size>> surfel_knn_connect_weight;
    unsigned num_vertex;
};
// NodeGraph::NodeGraph4Solver with the graph's K as a parameter (the reference fixes it at
// d_node_knn_size = 4; the 8-NN graph uses BasicNodeGraph4Solver<8>).
template <unsigned K = d_node_knn_size>
struct BasicNodeGraph4Solver {
    GArrayView<float4> reference_node_coords;
    GArrayView<ushort3> node_graph;
    GArrayView<floatX<K>> node_knn_connect_weight;
    GArrayView<ushortX<d_surfel_knn_size>> nodel_knn;
    GArrayView<floatX<d_surfel_knn_size>> node_knn_spatial_weight;
    unsigned num_node;
    float node_radius_square;
};
using NodeGraph4Solver = BasicNodeGraph4Solver<>;

// What the reference's WarpSolver and OptimizationProcessorWarpSolver read from
// ConfigParser::Instance() at construction (WarpSolver.cu:50-73, DenseImageHandler.cu:11,
// OptimizationProcessorWarpSolver.cu:4-15), plus the capacities the reference fixes at
// compile time (Constants.cpp:14-18) and the iteration counts (Constants.cpp:33,
// WarpSolver.cu:303).
struct SolverConfig {
    unsigned num_cam = 1;                        // this solver takes one camera
    unsigned downsample_img_cols = 640;          // config.downsample_img_cols(0)
    unsigned downsample_img_rows = 480;          // config.downsample_img_rows(0)
    Intrinsic rgb_intrinsic_downsample;          // config.rgb_intrinsic_downsample(0)
    Extrinsic extrinsic;                         // config.extrinsic()[0], camera to world
    unsigned max_num_nodes = 2048;               // d_max_num_nodes
    unsigned max_node_knn = 8;                   // largest node-graph K the solver takes
    unsigned max_num_features = 2000;            // d_max_num_keypoints
    int gauss_newton_iterations = 6;             // kNumGaussNewtonIterations
    int pcg_iterations = 10;
    int precision = WS_PREC_MIXED;
    int device = 0;

    // The process-wide configuration the default constructors read, as the reference's read
    // ConfigParser::Instance(): a pipeline fills it once at start-up.
    static SolverConfig &Instance() {
        static SolverConfig instance;
        return instance;
    }
};

// A {pointer, size} view of the solved node warps.  It converts to any view type constructible
// from (const T *, size_t) with a 32-byte T, such as the reference's GArrayView<DualQuaternion>.
class SE3View {
public:
    SE3View() = default;
    SE3View(const DualQuaternion *p, size_t n) : ptr_(p), size_(n) {}
    size_t Size() const { return size_; }
    const DualQuaternion *Ptr() const { return ptr_; }
    template <template <class> class View, class T>
    operator View<T>() const {
        static_assert(sizeof(T) == sizeof(DualQuaternion), "a dual quaternion is 8 floats");
        return View<T>(reinterpret_cast<const T *>(ptr_), size_);
    }

private:
    const DualQuaternion *ptr_ = nullptr;
    size_t size_ = 0;
};

// One frame's maps as texture objects (the pitch-linear maps the C ABI reads are resolved from
// these), for callers that fill ws_inputs themselves.
struct FrameMaps {
    cudaTextureObject_t vertex_confid_map = 0;     // Measure4Solver::vertex_confid_map (float4)
    cudaTextureObject_t normal_radius_map = 0;     // Measure4Solver::normal_radius_map (float4)
    cudaTextureObject_t reference_vertex_map = 0;  // Render4Solver::reference_vertex_map (float4)
    cudaTextureObject_t reference_normal_map = 0;  // Render4Solver::reference_normal_map (float4)
    cudaTextureObject_t index_map = 0;             // Render4Solver::index_map (uint32)
    cudaTextureObject_t opticalflow_map = 0;       // OpticalFlow4Solver::opticalflow_map (float2), 0 = none
};

namespace detail {
template <class View>
using view_elem = typename std::remove_cv<typename std::remove_pointer<decltype(std::declval<View>().Ptr())>::type>::type;
}

// star::WarpSolver (examples/mono_star/opt/WarpSolver.h:25-60) over the C ABI.
class WarpSolver {
public:
    using Ptr = std::shared_ptr<WarpSolver>;
    explicit WarpSolver(const SolverConfig &config = SolverConfig::Instance()) : config_(config) {
        ws_config c;
        c.max_scenes = 1;
        c.max_total_nodes = (int)config.max_num_nodes;
        c.max_total_pixels = (int)(config.downsample_img_cols * config.downsample_img_rows);
        c.max_total_edges = (int)(config.max_num_nodes * config.max_node_knn);
        c.max_total_features = (int)config.max_num_features;
        c.precision = config.precision;
        c.device = config.device;
        check(ws_create(&c, &h_), "ws_create");
    }
    // Capacity form (kept for callers that size the solver themselves).
    WarpSolver(int max_nodes, int max_pixels, int max_edges, int precision = WS_PREC_MIXED, int device = 0) {
        ws_config c;
        c.max_scenes = 1;
        c.max_total_nodes = max_nodes;
        c.max_total_pixels = max_pixels;
        c.max_total_edges = max_edges;
        c.max_total_features = 4096;
        c.precision = precision;
        c.device = device;
        check(ws_create(&c, &h_), "ws_create");
    }
    ~WarpSolver() { if (h_) ws_destroy(h_); }
    WarpSolver(const WarpSolver &) = delete;
    WarpSolver &operator=(const WarpSolver &) = delete;

    // WarpSolver::SetSolverInputs (WarpSolver.cu:125-155) with the reference's parameter list.
    // The types are any structs with the reference's member names (the reference's own, or the
    // ones above); the node graph's K is taken from its connect-weight element type.  Image size
    // and intrinsics come from the SolverConfig, as the reference reads them from ConfigParser.
    template <class M, class R, class G, class NG, class NF, class OF, class KP, class E>
    void SetSolverInputs(M measure4solver, R render4solver, G geometry4solver, NG node_graph4solver,
                         NF nodeflow4solver, OF opticalflow4solver, KP keypoint4solver, const E *camera2world,
                         cudaStream_t stream = 0) {
        if (measure4solver.num_cam != 1) throw Error(WS_ERR_INVALID_ARGUMENT, "SetSolverInputs: one camera");
        ws_inputs in;
        std::memset(&in, 0, sizeof(in));
        ws_default_penalties(&in);
        in.width = (int)config_.downsample_img_cols;
        in.height = (int)config_.downsample_img_rows;
        in.fx = config_.rgb_intrinsic_downsample.focal_x;
        in.fy = config_.rgb_intrinsic_downsample.focal_y;
        in.cx = config_.rgb_intrinsic_downsample.principal_x;
        in.cy = config_.rgb_intrinsic_downsample.principal_y;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) in.cam2world[4 * r + c] = camera2world[0](r, c);
        FrameMaps maps;
        maps.vertex_confid_map = measure4solver.vertex_confid_map[0];
        maps.normal_radius_map = measure4solver.normal_radius_map[0];
        maps.reference_vertex_map = render4solver.reference_vertex_map[0];
        maps.reference_normal_map = render4solver.reference_normal_map[0];
        maps.index_map = render4solver.index_map[0];
        maps.opticalflow_map = opticalflow4solver.num_cam > 0 ? opticalflow4solver.opticalflow_map[0] : 0;
        using SurfelKnn = detail::view_elem<decltype(geometry4solver.surfel_knn)>;
        using ConnectW = detail::view_elem<decltype(node_graph4solver.node_knn_connect_weight)>;
        static_assert(sizeof(SurfelKnn) == 4 * sizeof(uint16_t), "4 skinning neighbours per surfel");
        in.num_surfels = (int)geometry4solver.surfel_knn.Size();
        in.surfel_knn = reinterpret_cast<const uint16_t *>(geometry4solver.surfel_knn.Ptr());
        in.surfel_knn_spatial_weight = reinterpret_cast<const float *>(geometry4solver.surfel_knn_spatial_weight.Ptr());
        in.surfel_knn_connect_weight = reinterpret_cast<const float *>(geometry4solver.surfel_knn_connect_weight.Ptr());
        in.num_nodes = (int)node_graph4solver.num_node;
        in.reference_node_coords = reinterpret_cast<const float *>(node_graph4solver.reference_node_coords.Ptr());
        in.num_edges = (int)node_graph4solver.node_graph.Size();
        in.node_graph = reinterpret_cast<const uint16_t *>(node_graph4solver.node_graph.Ptr());
        in.graph_k = (int)(sizeof(ConnectW) / sizeof(float));
        in.node_knn_connect_weight = reinterpret_cast<const float *>(node_graph4solver.node_knn_connect_weight.Ptr());
        in.node_radius_square = node_graph4solver.node_radius_square;
        in.node_motion_pred = nodeflow4solver.node_motion_pred.Size() > 0
                                  ? reinterpret_cast<const float *>(nodeflow4solver.node_motion_pred.Ptr())
                                  : nullptr;
        in.num_features = (int)keypoint4solver.kp_knn.Size();
        in.feature_knn = in.num_features > 0 ? reinterpret_cast<const uint16_t *>(keypoint4solver.kp_knn.Ptr())
                                             : nullptr;
        SetSolverInputs(maps, in, stream);
    }

    // Texture-object maps plus a ws_inputs holding the node graph, geometry and camera; the map
    // pointers of `in` are filled from `maps`.
    void SetSolverInputs(const FrameMaps &maps, ws_inputs in, cudaStream_t st = 0) {
        in.pitch = 0;
        in.measure_vertex_confid = tex_[0].resolve(maps.vertex_confid_map, in.width, in.height, 16, st);
        in.measure_normal_radius = tex_[1].resolve(maps.normal_radius_map, in.width, in.height, 16, st);
        in.reference_vertex = tex_[2].resolve(maps.reference_vertex_map, in.width, in.height, 16, st);
        in.reference_normal = tex_[3].resolve(maps.reference_normal_map, in.width, in.height, 16, st);
        in.index_map = static_cast<const uint32_t *>(tex_[4].resolve(maps.index_map, in.width, in.height, 4, st));
        in.opticalflow = maps.opticalflow_map ? tex_[5].resolve(maps.opticalflow_map, in.width, in.height, 8, st)
                                              : nullptr;
        inputs_ = in;
        check(ws_set_inputs(h_, &inputs_), "ws_set_inputs");
    }
    // Device-pointer form (maps already pitch-linear).
    void SetSolverInputs(const ws_inputs &in) {
        inputs_ = in;
        check(ws_set_inputs(h_, &inputs_), "ws_set_inputs");
    }
    // WarpSolver::SolveStreamed (WarpSolver.cu:260-279) with the configured iteration counts.
    void SolveStreamed(cudaStream_t st = 0) {
        check(ws_solve(h_, config_.gauss_newton_iterations, config_.pcg_iterations, st), "ws_solve");
    }
    void SolveStreamed(cudaStream_t st, int gn_iters, int pcg_iters) {
        check(ws_solve(h_, gn_iters, pcg_iters, st), "ws_solve");
    }
    // WarpSolver::SolvedNodeSE3 (WarpSolver.h:45): the solved warp of every node, valid until the
    // next SetSolverInputs.
    SE3View SolvedNodeSE3() const {
        const float *p = nullptr;
        int n = 0;
        check(ws_get_solution(h_, 0, &p, &n), "ws_get_solution");
        return SE3View(reinterpret_cast<const DualQuaternion *>(p), (size_t)n);
    }
    // Pointer form: device pointer to num_nodes dual quaternions (8 floats each).
    const float *SolvedNodeSE3(int *num_nodes) const {
        const float *p = nullptr;
        int n = 0;
        check(ws_get_solution(h_, 0, &p, &n), "ws_get_solution");
        if (num_nodes) *num_nodes = n;
        return p;
    }
    int Status() { return ws_sync_status(h_); }
    ws_solver *handle() { return h_; }
    const SolverConfig &config() const { return config_; }

private:
    SolverConfig config_;
    ws_solver *h_ = nullptr;
    ws_inputs inputs_;
    TextureMap tex_[6];
};

// star::OptimizationProcessorWarpSolver (examples/mono_star/opt/OptimizationProcessorWarpSolver.h:10-37):
// ProcessFrame with the reference's parameter list and SolvedSE3 as a view of dual quaternions.
class OptimizationProcessorWarpSolver {
public:
    using Ptr = std::shared_ptr<OptimizationProcessorWarpSolver>;
    explicit OptimizationProcessorWarpSolver(const SolverConfig &config = SolverConfig::Instance())
        : solver_(config), cam2world_(config.extrinsic) {}
    // Capacity form (kept for callers that fill ws_inputs themselves).
    OptimizationProcessorWarpSolver(int max_nodes, int max_pixels, int max_edges, int gn_iters = 6,
                                    int pcg_iters = 10)
        : solver_(max_nodes, max_pixels, max_edges), gn_(gn_iters), pcg_(pcg_iters) {}
    OptimizationProcessorWarpSolver(const OptimizationProcessorWarpSolver &) = delete;
    OptimizationProcessorWarpSolver &operator=(const OptimizationProcessorWarpSolver &) = delete;

    // OptimizationProcessorWarpSolver::ProcessFrame (OptimizationProcessorWarpSolver.cu:22-52):
    // frame 0 only initialises the model; later frames set the inputs, solve on `stream` and wait
    // for it, and a device-side error (NaN right-hand side, capacity, timeout) throws.
    template <class M, class R, class G, class NG, class NF, class OF, class KP>
    void ProcessFrame(M &measure4solver, R &render4solver, G &geometry4solver, NG &node_graph4solver,
                      NF &nodeflow4solver, OF &opticalflow4solver, KP &keypoint4solver, const unsigned frame_idx,
                      cudaStream_t stream) {
        if (frame_idx == 0) return;
        solver_.SetSolverInputs(measure4solver, render4solver, geometry4solver, node_graph4solver, nodeflow4solver,
                                opticalflow4solver, keypoint4solver, &cam2world_, stream);
        solver_.SolveStreamed(stream);
        check(solver_.Status(), "ProcessFrame");
        solved_ = true;
    }
    // Form with texture-object maps and a filled ws_inputs.
    void ProcessFrame(const FrameMaps &maps, const ws_inputs &in, unsigned frame_idx, cudaStream_t st) {
        if (frame_idx == 0) return;
        solver_.SetSolverInputs(maps, in, st);
        solver_.SolveStreamed(st, gn_, pcg_);
        solved_ = true;
    }
    // OptimizationProcessorWarpSolver::SolvedSE3: converts to GArrayView<DualQuaternion>; empty
    // before the first solved frame.
    SE3View SolvedSE3() const { return solved_ ? solver_.SolvedNodeSE3() : SE3View(); }
    const float *SolvedSE3(int *num_nodes) const {
        if (!solved_) {
            if (num_nodes) *num_nodes = 0;
            return nullptr;
        }
        return solver_.SolvedNodeSE3(num_nodes);
    }

private:
    WarpSolver solver_;
    Extrinsic cam2world_;
    int gn_ = 6, pcg_ = 10;
    bool solved_ = false;
};

// Skinner::PerformSkinning* inputs (libs/star/geometry/node_graph/skinner_types.h:10-33): the
// surfel side writes its knn and weights, the node side is read.
struct Geometry4Skinner {
    GArrayView<float4> reference_vertex_confid;
    GArrayView<float4> reference_normal_radius;
    GArrayView<float4> live_vertex_confid;
    GArrayView<float4> live_normal_radius;
    ushortX<d_surfel_knn_size> *surfel_knn = nullptr;
    floatX<d_surfel_knn_size> *surfel_knn_spatial_weight = nullptr;
    floatX<d_surfel_knn_size> *surfel_knn_connect_weight = nullptr;
};
struct NodeGraph4Skinner {
    GArrayView<float4> reference_node_coords;
    GArrayView<float4> live_node_coords;
    GArrayView<uint2> node_status;
    float node_radius_square = 0.f;
};

// star::NodeGraph's node construction and growth over ws_init_nodes, ws_expand_nodes and
// ws_build_node_graph_ex, with the node status and NodeGraph::ReAnchor.  The node arrays are device
// memory owned here and sized for max_nodes, like the reference's preallocation; GetNodeKnn returns
// k ids per node, edges are (i, knn, k).  `normalize_weights` chooses the node-graph weights: the
// reference's geometry library is compiled without USE_INTERPOLATE_WEIGHT_NORMALIZATION, so its
// weights are the raw exponentials (false, the default); true divides them by their sum.
class NodeGraph {
public:
    using Ptr = std::shared_ptr<NodeGraph>;
    using ConstPtr = std::shared_ptr<NodeGraph const>;

    NodeGraph(float node_radius, int max_nodes, int knn = 4, bool normalize_weights = false)
        : radius_(node_radius), cap_(max_nodes), k_(knn), normalize_(normalize_weights) {
        if (!(node_radius > 0.f) || max_nodes < 2 || max_nodes > 65535 || (knn != 4 && knn != 8))
            throw Error(WS_ERR_INVALID_ARGUMENT, "NodeGraph");
        try {
            alloc(&ref_, 16ull * cap_);
            alloc(&live_, 16ull * cap_);
            alloc(&time_, 4ull * cap_);
            alloc(&status_, 8ull * cap_);
            alloc(&knn_, 2ull * k_ * cap_);
            alloc(&weight_, 4ull * k_ * cap_);
            alloc(&connect_, 4ull * k_ * cap_);
            alloc(&edges_, 6ull * k_ * cap_);
            check(cudaMemset(status_, 0, 8ull * cap_) == cudaSuccess ? WS_OK : WS_ERR_CUDA, "NodeGraph");
        } catch (...) {
            release();
            throw;
        }
    }
    ~NodeGraph() { release(); }
    NodeGraph(const NodeGraph &) = delete;
    NodeGraph &operator=(const NodeGraph &) = delete;

    // InitializeNodeGraphFromVertex (NodeGraph.cu:460-498): nodes from `vertex` (device float4),
    // two anchors first, reference = live coordinates, initial time `current_time`, status cleared,
    // then the graph.
    void InitializeNodeGraphFromVertex(const float4 *vertex, unsigned num_vertex, unsigned current_time, bool use_ref,
                                       cudaStream_t stream = 0) {
        std::vector<float4> host((size_t)cap_);
        int n = 0;
        check(ws_init_nodes(reinterpret_cast<const float *>(vertex), (int)num_vertex, radius_,
                            reinterpret_cast<float *>(host.data()), cap_, &n, stream),
              "InitializeNodeGraphFromVertex");
        const std::vector<unsigned> times((size_t)n, current_time);
        check(cudaMemcpyAsync(ref_, host.data(), 16ull * n, cudaMemcpyHostToDevice, stream) == cudaSuccess &&
                      cudaMemcpyAsync(live_, host.data(), 16ull * n, cudaMemcpyHostToDevice, stream) == cudaSuccess &&
                      cudaMemcpyAsync(time_, times.data(), 4ull * n, cudaMemcpyHostToDevice, stream) == cudaSuccess &&
                      cudaMemsetAsync(status_, 0, 8ull * n, stream) == cudaSuccess &&
                      cudaStreamSynchronize(stream) == cudaSuccess
                  ? WS_OK
                  : WS_ERR_CUDA,
              "InitializeNodeGraphFromVertex");
        prev_size_ = 0;
        size_ = (unsigned)n;
        BuildNodeGraphFromScratch(use_ref, stream);
    }

    // NaiveExpandNodeGraphFromVertexUnsupported (NodeGraph.cu:500-532): appends the greedy
    // nodes of `vertex_unsupported` (device float4) to both coordinate arrays with initial time
    // `current_time` and a cleared status.  The graph is rebuilt by a later BuildNodeGraphFromScratch.
    void NaiveExpandNodeGraphFromVertexUnsupported(const float4 *vertex_unsupported, unsigned num_vertex,
                                                   unsigned current_time, cudaStream_t stream) {
        int n = (int)size_;
        check(ws_expand_nodes(reinterpret_cast<const float *>(vertex_unsupported), (int)num_vertex, radius_,
                              reinterpret_cast<float *>(ref_), reinterpret_cast<float *>(live_), time_, current_time,
                              cap_, &n, stream),
              "NaiveExpandNodeGraphFromVertexUnsupported");
        if ((unsigned)n > size_)
            check(cudaMemsetAsync(status_ + size_, 0, 8ull * ((unsigned)n - size_), stream) == cudaSuccess
                      ? WS_OK
                      : WS_ERR_CUDA,
                  "NaiveExpandNodeGraphFromVertexUnsupported");
        prev_size_ = size_;
        size_ = (unsigned)n;
    }

    // BuildNodeGraphFromScratch (NodeGraph.cu:357-365): k-NN graph of the reference (use_ref)
    // or live coordinates; deleted nodes (status .y == WS_DELETED_NODE_STATUS) are left out.
    void BuildNodeGraphFromScratch(bool use_ref, cudaStream_t stream) {
        if (size_ == 0) return;
        check(ws_build_node_graph_ex(reinterpret_cast<const float *>(use_ref ? ref_ : live_),
                                     reinterpret_cast<const uint32_t *>(status_), (int)size_, k_, radius_,
                                     normalize_ ? 1 : 0, knn_, weight_, edges_, stream),
              "BuildNodeGraphFromScratch");
    }

    // ResetNodeGraphConnection (NodeGraph.cu:296-303): every connect weight to 1.
    void ResetNodeGraphConnection(cudaStream_t stream) {
        std::vector<float> ones((size_t)k_ * size_, 1.f);
        if (!ones.empty())
            check(cudaMemcpyAsync(connect_, ones.data(), 4ull * ones.size(), cudaMemcpyHostToDevice, stream) ==
                              cudaSuccess &&
                          cudaStreamSynchronize(stream) == cudaSuccess
                      ? WS_OK
                      : WS_ERR_CUDA,
                  "ResetNodeGraphConnection");
    }

    // NodeGraph::ReAnchor (NodeGraph.cu:574-650): `tar` takes `src`'s graph (knn, weights, connect
    // weights, edges), node status and initial times, its reference coordinates become `src`'s
    // live coordinates, and it takes `src`'s node counts.  The reference also copies its n x n
    // half-distance table, which this node graph does not keep (the graph is built without it).
    static void ReAnchor(ConstPtr src_node_graph, Ptr tar_node_graph, cudaStream_t stream) {
        const NodeGraph &s = *src_node_graph;
        NodeGraph &t = *tar_node_graph;
        if (s.k_ != t.k_ || t.cap_ < (int)s.size_) throw Error(WS_ERR_CAPACITY, "ReAnchor");
        const size_t n = s.size_, k = (size_t)s.k_;
        const bool ok =
            cudaMemcpyAsync(t.knn_, s.knn_, 2 * k * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaMemcpyAsync(t.weight_, s.weight_, 4 * k * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaMemcpyAsync(t.connect_, s.connect_, 4 * k * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaMemcpyAsync(t.edges_, s.edges_, 6 * k * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaMemcpyAsync(t.status_, s.status_, 8 * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaMemcpyAsync(t.time_, s.time_, 4 * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaMemcpyAsync(t.ref_, s.live_, 16 * n, cudaMemcpyDeviceToDevice, stream) == cudaSuccess &&
            cudaStreamSynchronize(stream) == cudaSuccess;
        check(ok ? WS_OK : WS_ERR_CUDA, "ReAnchor");
        t.size_ = s.size_;
        t.prev_size_ = s.prev_size_;
    }

    // NodeGraph::GenerateNodeGraph4Skinner (NodeGraph.cu:534-545).
    NodeGraph4Skinner GenerateNodeGraph4Skinner() const {
        NodeGraph4Skinner out;
        out.reference_node_coords = GArrayView<float4>(ref_, size_);
        out.live_node_coords = GArrayView<float4>(live_, size_);
        out.node_status = GArrayView<uint2>(status_, size_);
        out.node_radius_square = radius_ * radius_;
        return out;
    }

    const float4 *GetReferenceNodeCoordinate() const { return ref_; }
    const float4 *GetLiveNodeCoordinate() const { return live_; }
    float4 *LiveNodeCoordinate() { return live_; }
    const uint16_t *GetNodeKnn() const { return knn_; }
    const float *GetNodeKnnSpatialWeight() const { return weight_; }
    const float *GetNodeKnnConnectWeight() const { return connect_; }
    const uint16_t *GetNodeGraph() const { return edges_; }
    const unsigned *GetNodeInitialTime() const { return time_; }
    uint2 *GetNodeStatus() { return status_; }
    const uint2 *GetNodeStatusReadOnly() const { return status_; }
    unsigned GetNodeSize() const { return size_; }
    unsigned GetPrevNodeSize() const { return prev_size_; }
    float GetNodeRadiusSquare() const { return radius_ * radius_; }

private:
    template <class T>
    static void alloc(T **p, size_t bytes) {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes) != cudaSuccess) throw Error(WS_ERR_CUDA, "NodeGraph allocation");
        *p = static_cast<T *>(q);
    }
    void release() {
        void *ptrs[] = {ref_, live_, time_, status_, knn_, weight_, connect_, edges_};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        ref_ = live_ = nullptr;
        time_ = nullptr;
        status_ = nullptr;
        knn_ = edges_ = nullptr;
        weight_ = connect_ = nullptr;
    }

    float radius_;
    int cap_, k_;
    bool normalize_;
    unsigned size_ = 0, prev_size_ = 0;
    float4 *ref_ = nullptr, *live_ = nullptr;
    unsigned *time_ = nullptr;
    uint2 *status_ = nullptr;
    uint16_t *knn_ = nullptr, *edges_ = nullptr;
    float *weight_ = nullptr, *connect_ = nullptr;
};

// star::Skinner (libs/star/geometry/node_graph/Skinner.h:6-28) over ws_skinning_ex and
// ws_skinning_incremental.  Templates over any structs with the members of Geometry4Skinner and
// NodeGraph4Skinner (the reference's or the ones above).  `normalize_weights` as in NodeGraph.
struct Skinner {
    // PerformSkinningFromRef (Skinner.cu:336-352): reference surfels against reference nodes.
    template <class G, class N>
    static void PerformSkinningFromRef(G &geometry, N &node_graph, cudaStream_t stream = 0,
                                       bool normalize_weights = false) {
        skin(geometry.reference_vertex_confid, node_graph.reference_node_coords, geometry, node_graph, 0, 0,
             normalize_weights, stream, "PerformSkinningFromRef");
    }
    // PerformSkinningFromLive (Skinner.cu:354-372): live surfels against live nodes.
    template <class G, class N>
    static void PerformSkinningFromLive(G &geometry, N &node_graph, cudaStream_t stream = 0,
                                        bool normalize_weights = false) {
        skin(geometry.live_vertex_confid, node_graph.live_node_coords, geometry, node_graph, 0, 0, normalize_weights,
             stream, "PerformSkinningFromLive");
    }
    // PerformIncSkinnningFromLive (Skinner.cu:395-415): surfels from num_remaining_surfel on take
    // the nodes from num_prev_node_size on into their current neighbours.
    template <class G, class N>
    static void PerformIncSkinnningFromLive(G &geometry, N &node_graph, const unsigned num_prev_node_size,
                                            const unsigned num_remaining_surfel, cudaStream_t stream = 0,
                                            bool normalize_weights = false) {
        skin(geometry.live_vertex_confid, node_graph.live_node_coords, geometry, node_graph, num_prev_node_size,
             num_remaining_surfel, normalize_weights, stream, "PerformIncSkinnningFromLive");
    }

private:
    template <class V, class NV, class G, class N>
    static void skin(const V &verts, const NV &nodes, G &geometry, N &node_graph, unsigned prev_nodes,
                     unsigned remaining, bool normalize, cudaStream_t stream, const char *what) {
        const int status = ws_skinning_incremental(
            reinterpret_cast<const float *>(nodes.Ptr()), reinterpret_cast<const uint32_t *>(node_graph.node_status.Ptr()),
            (int)node_graph.node_status.Size(), (int)prev_nodes, reinterpret_cast<const float *>(verts.Ptr()),
            (int)verts.Size(), (int)remaining, std::sqrt(node_graph.node_radius_square), normalize ? 1 : 0,
            reinterpret_cast<uint16_t *>(&geometry.surfel_knn[0]),
            reinterpret_cast<float *>(&geometry.surfel_knn_spatial_weight[0]),
            reinterpret_cast<float *>(&geometry.surfel_knn_connect_weight[0]), stream);
        check(status, what);
    }
};

}  // namespace b200
}  // namespace star
