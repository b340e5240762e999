// warp_solver.hpp -- header-only C++ facade over include/warpsolve.h.
//
// Re-creates the call surface of StarHub's solver so the per-frame pipeline
// keeps its call sites:
//   * star::b200::WarpSolver mirrors star::WarpSolver
//     (examples/mono_star/opt/WarpSolver.h:34-52): SetSolverInputs,
//     SolveStreamed, SolvedNodeSE3;
//   * star::b200::OptimizationProcessorWarpSolver mirrors the processor entry
//     (examples/mono_star/opt/OptimizationProcessorWarpSolver.h:18-30):
//     ProcessFrame (frame 0 is a no-op, OptimizationProcessorWarpSolver.cu:35-36)
//     and SolvedSE3;
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

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
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

// One frame's maps as texture objects, as the reference's *4Solver structs carry them.
struct FrameMaps {
    cudaTextureObject_t vertex_confid_map = 0;     // Measure4Solver::vertex_confid_map (float4)
    cudaTextureObject_t normal_radius_map = 0;     // Measure4Solver::normal_radius_map (float4)
    cudaTextureObject_t reference_vertex_map = 0;  // Render4Solver::reference_vertex_map (float4)
    cudaTextureObject_t reference_normal_map = 0;  // Render4Solver::reference_normal_map (float4)
    cudaTextureObject_t index_map = 0;             // Render4Solver::index_map (uint32)
    cudaTextureObject_t opticalflow_map = 0;       // OpticalFlow4Solver::opticalflow_map (float2), 0 = none
};

class WarpSolver {
public:
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

    // WarpSolver::SetSolverInputs: `in` holds the node graph, geometry and camera;
    // its map pointers are filled from `maps`.
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
    // WarpSolver::SolveStreamed with the reference's default counts (6 GN x 10 PCG).
    void SolveStreamed(cudaStream_t st = 0, int gn_iters = 6, int pcg_iters = 10) {
        check(ws_solve(h_, gn_iters, pcg_iters, st), "ws_solve");
    }
    // Device pointer to num_nodes DualQuaternions (8 floats each), valid until the next SetSolverInputs.
    const float *SolvedNodeSE3(int *num_nodes = nullptr) const {
        const float *p = nullptr;
        int n = 0;
        check(ws_get_solution(h_, 0, &p, &n), "ws_get_solution");
        if (num_nodes) *num_nodes = n;
        return p;
    }
    int Status() { return ws_sync_status(h_); }
    ws_solver *handle() { return h_; }

private:
    ws_solver *h_ = nullptr;
    ws_inputs inputs_;
    TextureMap tex_[6];
};

// OptimizationProcessorWarpSolver::ProcessFrame / SolvedSE3.
class OptimizationProcessorWarpSolver {
public:
    OptimizationProcessorWarpSolver(int max_nodes, int max_pixels, int max_edges, int gn_iters = 6,
                                    int pcg_iters = 10)
        : solver_(max_nodes, max_pixels, max_edges), gn_(gn_iters), pcg_(pcg_iters) {}

    void ProcessFrame(const FrameMaps &maps, const ws_inputs &in, unsigned frame_idx, cudaStream_t st) {
        if (frame_idx == 0) return;   // the first frame only initialises the model
        solver_.SetSolverInputs(maps, in, st);
        solver_.SolveStreamed(st, gn_, pcg_);
        solved_ = true;
    }
    const float *SolvedSE3(int *num_nodes = nullptr) const {
        return solved_ ? solver_.SolvedNodeSE3(num_nodes) : nullptr;
    }

private:
    WarpSolver solver_;
    int gn_, pcg_;
    bool solved_ = false;
};

// star::NodeGraph's node construction and growth over ws_init_nodes, ws_expand_nodes and
// ws_build_node_graph.  The node arrays are device memory owned here and sized for max_nodes,
// like the reference's preallocation; GetNodeKnn returns k ids per node, edges are (i, knn, k).
class NodeGraph {
public:
    NodeGraph(float node_radius, int max_nodes, int knn = 4) : radius_(node_radius), cap_(max_nodes), k_(knn) {
        if (!(node_radius > 0.f) || max_nodes < 2 || max_nodes > 65535 || (knn != 4 && knn != 8))
            throw Error(WS_ERR_INVALID_ARGUMENT, "NodeGraph");
        try {
            alloc(&ref_, 16ull * cap_);
            alloc(&live_, 16ull * cap_);
            alloc(&time_, 4ull * cap_);
            alloc(&knn_, 2ull * k_ * cap_);
            alloc(&weight_, 4ull * k_ * cap_);
            alloc(&edges_, 6ull * k_ * cap_);
        } catch (...) {
            release();
            throw;
        }
    }
    ~NodeGraph() { release(); }
    NodeGraph(const NodeGraph &) = delete;
    NodeGraph &operator=(const NodeGraph &) = delete;

    // InitializeNodeGraphFromVertex (NodeGraph.cu:460-498): nodes from `vertex` (device float4),
    // two anchors first, reference = live coordinates, initial time `current_time`, then the graph.
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
    // `current_time`.  The graph is rebuilt by a later BuildNodeGraphFromScratch, as there.
    void NaiveExpandNodeGraphFromVertexUnsupported(const float4 *vertex_unsupported, unsigned num_vertex,
                                                   unsigned current_time, cudaStream_t stream) {
        int n = (int)size_;
        check(ws_expand_nodes(reinterpret_cast<const float *>(vertex_unsupported), (int)num_vertex, radius_,
                              reinterpret_cast<float *>(ref_), reinterpret_cast<float *>(live_), time_, current_time,
                              cap_, &n, stream),
              "NaiveExpandNodeGraphFromVertexUnsupported");
        prev_size_ = size_;
        size_ = (unsigned)n;
    }

    // BuildNodeGraphFromScratch (NodeGraph.cu:357-365): k-NN graph of the reference (use_ref)
    // or live coordinates.
    void BuildNodeGraphFromScratch(bool use_ref, cudaStream_t stream) {
        if (size_ == 0) return;
        check(ws_build_node_graph(reinterpret_cast<const float *>(use_ref ? ref_ : live_), (int)size_, k_, radius_,
                                  knn_, weight_, edges_, stream),
              "BuildNodeGraphFromScratch");
    }

    const float4 *GetReferenceNodeCoordinate() const { return ref_; }
    const float4 *GetLiveNodeCoordinate() const { return live_; }
    const uint16_t *GetNodeKnn() const { return knn_; }
    const float *GetNodeKnnSpatialWeight() const { return weight_; }
    const uint16_t *GetNodeGraph() const { return edges_; }
    const unsigned *GetNodeInitialTime() const { return time_; }
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
        void *ptrs[] = {ref_, live_, time_, knn_, weight_, edges_};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        ref_ = live_ = nullptr;
        time_ = nullptr;
        knn_ = edges_ = nullptr;
        weight_ = nullptr;
    }

    float radius_;
    int cap_, k_;
    unsigned size_ = 0, prev_size_ = 0;
    float4 *ref_ = nullptr, *live_ = nullptr;
    unsigned *time_ = nullptr;
    uint16_t *knn_ = nullptr, *edges_ = nullptr;
    float *weight_ = nullptr;
};

}  // namespace b200
}  // namespace star
