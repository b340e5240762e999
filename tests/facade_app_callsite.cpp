// The pipeline's solver call site, written as examples/mono_star/app.cu:45-150 writes it, against
// the C++ facade include/starhub_b200/warp_solver.hpp.  The geometry and measurement processors
// of the pipeline are stood in for by arrays read from files (written by the test that builds
// this program); everything from the construction of the processor to SolvedSE3() is the
// reference's own sequence of calls, with `star::b200` for `star`.
//
// usage: facade_app_callsite <dir>   reads <dir>/params.txt and <dir>/*.bin, writes <dir>/se3.bin
#include <cstdio>
#include <string>
#include <vector>

#include "starhub_b200/warp_solver.hpp"

namespace {

std::vector<char> read_file(const std::string &path) {
    std::vector<char> out;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return out;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) out.insert(out.end(), buf, buf + n);
    std::fclose(f);
    return out;
}

template <class T>
const T *upload(const std::string &dir, const char *name, size_t *count) {
    const std::vector<char> host = read_file(dir + "/" + name);
    void *dev = nullptr;
    if (cudaMalloc(&dev, host.size() ? host.size() : 16) != cudaSuccess) return nullptr;
    cudaMemcpy(dev, host.data(), host.size(), cudaMemcpyHostToDevice);
    *count = host.size() / sizeof(T);
    return static_cast<const T *>(dev);
}

// A pitch-linear texture over `ptr` (what the reference's surfel maps hand the solver).
cudaTextureObject_t texture(const void *ptr, int width, int height, cudaChannelFormatDesc fmt, size_t texel) {
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = const_cast<void *>(ptr);
    rd.res.pitch2D.desc = fmt;
    rd.res.pitch2D.width = width;
    rd.res.pitch2D.height = height;
    rd.res.pitch2D.pitchInBytes = width * texel;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    cudaCreateTextureObject(&t, &rd, &td, nullptr);
    return t;
}

struct Params {
    int width, height, graph_k, frame_idx;
    float fx, fy, cx, cy, node_radius_square;
};

template <unsigned K>
int run(const std::string &dir, const Params &prm) {
    using namespace star::b200;   // app.cu:19 `using namespace star;`

    // What ConfigParser::Instance() holds in the pipeline (read by the processor's constructor).
    auto &solver_config = SolverConfig::Instance();
    solver_config.downsample_img_cols = prm.width;
    solver_config.downsample_img_rows = prm.height;
    solver_config.rgb_intrinsic_downsample.focal_x = prm.fx;
    solver_config.rgb_intrinsic_downsample.focal_y = prm.fy;
    solver_config.rgb_intrinsic_downsample.principal_x = prm.cx;
    solver_config.rgb_intrinsic_downsample.principal_y = prm.cy;
    solver_config.extrinsic = Extrinsic::Identity();
    solver_config.max_num_nodes = 65535;
    solver_config.max_node_knn = K;

    // app.cu:49
    auto opt_processor = std::make_shared<OptimizationProcessorWarpSolver>();

    // stand-ins for the processors' outputs
    size_t n_pix, n_sknn, n_ssw, n_scw, n_nodes, n_edges, n_ncw;
    const float4 *meas_vertex = upload<float4>(dir, "meas_vertex.bin", &n_pix);
    const float4 *meas_normal = upload<float4>(dir, "meas_normal.bin", &n_pix);
    const float4 *ref_vertex = upload<float4>(dir, "ref_vertex.bin", &n_pix);
    const float4 *ref_normal = upload<float4>(dir, "ref_normal.bin", &n_pix);
    const unsigned *index = upload<unsigned>(dir, "index.bin", &n_pix);
    const ushortX<d_surfel_knn_size> *sknn = upload<ushortX<d_surfel_knn_size>>(dir, "surfel_knn.bin", &n_sknn);
    const floatX<d_surfel_knn_size> *ssw = upload<floatX<d_surfel_knn_size>>(dir, "surfel_sw.bin", &n_ssw);
    const floatX<d_surfel_knn_size> *scw = upload<floatX<d_surfel_knn_size>>(dir, "surfel_cw.bin", &n_scw);
    const float4 *nodes = upload<float4>(dir, "nodes.bin", &n_nodes);
    const ushort3 *edges = upload<ushort3>(dir, "edges.bin", &n_edges);
    const floatX<K> *ncw = upload<floatX<K>>(dir, "node_cw.bin", &n_ncw);
    const cudaChannelFormatDesc f4 = cudaCreateChannelDesc<float4>(), u1 = cudaCreateChannelDesc<unsigned>();
    struct {
        cudaTextureObject_t vertex_confid, normal_radius, index;
    } surfel_map_this{texture(meas_vertex, prm.width, prm.height, f4, 16),
                      texture(meas_normal, prm.width, prm.height, f4, 16), 0},
        surfel_map_prev{texture(ref_vertex, prm.width, prm.height, f4, 16),
                        texture(ref_normal, prm.width, prm.height, f4, 16),
                        texture(index, prm.width, prm.height, u1, 4)};
    Geometry4Solver geometry4solver_of_processor{GArrayView<ushortX<d_surfel_knn_size>>(sknn, n_sknn),
                                                 GArrayView<floatX<d_surfel_knn_size>>(ssw, n_ssw),
                                                 GArrayView<floatX<d_surfel_knn_size>>(scw, n_scw),
                                                 (unsigned)n_sknn};
    BasicNodeGraph4Solver<K> node_graph4solver_of_processor{};
    node_graph4solver_of_processor.reference_node_coords = GArrayView<float4>(nodes, n_nodes);
    node_graph4solver_of_processor.node_graph = GArrayView<ushort3>(edges, n_edges);
    node_graph4solver_of_processor.node_knn_connect_weight = GArrayView<floatX<K>>(ncw, n_ncw);
    node_graph4solver_of_processor.num_node = (unsigned)n_nodes;
    node_graph4solver_of_processor.node_radius_square = prm.node_radius_square;
    const unsigned frame_idx = (unsigned)prm.frame_idx;

    // ---- app.cu:97-140, as written there ----
    auto geometry4solver = geometry4solver_of_processor;
    auto node_graph4solver = node_graph4solver_of_processor;

    Measure4Solver measure4solver;
    measure4solver.num_cam = 1;
    measure4solver.vertex_confid_map[0] = surfel_map_this.vertex_confid;
    measure4solver.normal_radius_map[0] = surfel_map_this.normal_radius;
    measure4solver.index_map[0] = surfel_map_this.index;

    Render4Solver render4solver;
    render4solver.num_cam = 1;
    render4solver.reference_vertex_map[0] = surfel_map_prev.vertex_confid;
    render4solver.reference_normal_map[0] = surfel_map_prev.normal_radius;
    render4solver.index_map[0] = surfel_map_prev.index;

    OpticalFlow4Solver opticalflow4solver;
    opticalflow4solver.num_cam = 1;
    opticalflow4solver.opticalflow_map[0] = 0;   // GetOpticalFlow(): no flow in this frame

    NodeFlow4Solver nodeflow4solver;
    nodeflow4solver.num_node = 0;                 // GetNodeMotionPred().Size()
    nodeflow4solver.node_motion_pred = GArrayView<float4>();

    KeyPoint4Solver keypoint4solver;              // no matched key points

    // Solve
    opt_processor->ProcessFrame(
        measure4solver,
        render4solver,
        geometry4solver,
        node_graph4solver,
        nodeflow4solver,
        opticalflow4solver,
        keypoint4solver,
        frame_idx,
        0);

    // Apply the warp: geometry_processor->ProcessFrame(..., opt_processor->SolvedSE3(), ...)
    GArrayView<DualQuaternion> solved_se3 = opt_processor->SolvedSE3();
    // ---- end of the call site ----

    std::vector<DualQuaternion> host(solved_se3.Size());
    if (!host.empty())
        cudaMemcpy(host.data(), solved_se3.Ptr(), host.size() * sizeof(DualQuaternion), cudaMemcpyDeviceToHost);
    FILE *f = std::fopen((dir + "/se3.bin").c_str(), "wb");
    if (!f) return 4;
    if (!host.empty()) std::fwrite(host.data(), sizeof(DualQuaternion), host.size(), f);
    std::fclose(f);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 2) return 2;
    const std::string dir = argv[1];
    Params prm;
    FILE *f = std::fopen((dir + "/params.txt").c_str(), "r");
    if (!f) return 3;
    const int got = std::fscanf(f, "%d %d %d %d %f %f %f %f %f", &prm.width, &prm.height, &prm.graph_k,
                                &prm.frame_idx, &prm.fx, &prm.fy, &prm.cx, &prm.cy, &prm.node_radius_square);
    std::fclose(f);
    if (got != 9) return 3;
    try {
        return prm.graph_k == 8 ? run<8>(dir, prm) : run<4>(dir, prm);
    } catch (const star::b200::Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 5;
    }
}
