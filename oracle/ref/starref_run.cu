// Test infrastructure: runs the reference's own CUDA warp solver (examples/mono_star/opt, compiled
// in place from the reference tree by oracle/ref/Makefile) on one scene and writes what it built
// and solved, so that the tests can compare the B200 solver with the reference itself.
//
// usage: starref_run <dir>
//   reads  <dir>/params.txt and the input arrays <dir>/*.bin (written by oracle/ref_oracle.py),
//   writes <dir>/out_*.bin: the compacted dense terms (ImageTermKNNFetcher), the node->term map
//   (Node2TermsIndex), the node-pair->term map (NodePair2TermsIndex), the first Gauss-Newton
//   iteration's diagonal blocks, J^T r, inverse blocks and PCG step, and the solved node warps.
//
// The solve follows WarpSolver::SolveStreamed (WarpSolver.cu:260-337) call for call, with the
// Gauss-Newton and PCG iteration counts as parameters (the reference fixes them at
// Constants::kNumGaussNewtonIterations = 6 and SolvePCGMaterialized(10)); with 6 and 10 it calls
// SolveStreamed itself.  The steps it needs are private members of WarpSolver, reached through
// explicit template instantiation (which the language exempts from access checks), so the
// reference's sources and headers are used unmodified.
//
// ConfigParser::Instance() is the only reference symbol not compiled: its definition
// (ConfigParser.cu) parses JSON files.  It is defined below over a small struct instead, through
// the reference's own declaration of loadCameraConfigFromJson.
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <mono_star/common/ConfigParser.h>
#include <mono_star/opt/WarpSolver.h>

namespace {

struct RefCamera {
    unsigned width, height;
    float fx, fy, cx, cy;
};

}  // namespace

// ---- ConfigParser: the values the solver reads, set by the harness ----
star::ConfigParser::ConfigParser() { m_num_cam = 1; }

star::ConfigParser &star::ConfigParser::Instance() {
    static ConfigParser instance;
    return instance;
}

void star::ConfigParser::loadCameraConfigFromJson(const void *camera) {
    const RefCamera &c = *static_cast<const RefCamera *>(camera);
    m_num_cam = 1;
    m_downsample_image_cols[0] = c.width;
    m_downsample_image_rows[0] = c.height;
    m_raw_img_cols[0] = c.width;
    m_raw_img_rows[0] = c.height;
    downsample_rgb_intrinsic[0].focal_x = c.fx;
    downsample_rgb_intrinsic[0].focal_y = c.fy;
    downsample_rgb_intrinsic[0].principal_x = c.cx;
    downsample_rgb_intrinsic[0].principal_y = c.cy;
    raw_rgb_intrinsic[0] = downsample_rgb_intrinsic[0];
    raw_depth_intrinsic[0] = downsample_rgb_intrinsic[0];
    m_cam2world[0] = Eigen::Matrix4f::Identity();
}

// ---- access to WarpSolver's private steps (explicit instantiation ignores access) ----
namespace {
template <typename Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type get(Tag) { return M; }
};
#define STARREF_EXPOSE(NAME, TYPE, MEMBER)               \
    struct NAME {                                        \
        using type = TYPE;                               \
        friend type get(NAME);                           \
    };                                                   \
    template struct Expose<NAME, &star::WarpSolver::MEMBER>;

STARREF_EXPOSE(FetcherTag, star::ImageTermKNNFetcher::Ptr star::WarpSolver::*, m_image_term_knn_fetcher)
STARREF_EXPOSE(Node2TermTag, star::Node2TermsIndex::Ptr star::WarpSolver::*, m_node2term_index)
STARREF_EXPOSE(PairTag, star::NodePair2TermsIndex::Ptr star::WarpSolver::*, m_nodepair2term_index)
STARREF_EXPOSE(RhsTag, star::PreconditionerRhsBuilder::Ptr star::WarpSolver::*, m_preconditioner_rhs_builder)
STARREF_EXPOSE(JtJTag, star::JtJMaterializer::Ptr star::WarpSolver::*, m_jtj_materializer)
STARREF_EXPOSE(IterTag, star::SolverIterationData star::WarpSolver::*, m_iteration_data)
STARREF_EXPOSE(StreamTag, cudaStream_t (star::WarpSolver::*)[4], m_solver_stream)
STARREF_EXPOSE(ComputeJTag, void (star::WarpSolver::*)(), computeNode2JacobianSync)

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

bool write_file(const std::string &path, const void *data, size_t bytes) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes;
    std::fclose(f);
    return ok;
}

// Uploads <dir>/<name>.bin (at least `min_bytes`, zero-filled beyond the file) to the device.
template <typename T>
T *upload(const std::string &dir, const char *name, size_t min_bytes, size_t *count) {
    std::vector<char> host = read_file(dir + "/" + name + ".bin");
    if (host.size() < min_bytes) host.resize(min_bytes, 0);
    void *dev = nullptr;
    if (cudaMalloc(&dev, host.size() ? host.size() : 16) != cudaSuccess) return nullptr;
    if (!host.empty() && cudaMemcpy(dev, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    if (count) *count = host.size() / sizeof(T);
    return static_cast<T *>(dev);
}

template <typename T>
bool download(const std::string &path, const T *dev, size_t count) {
    std::vector<T> host(count);
    if (count && cudaMemcpy(host.data(), dev, count * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    return write_file(path, host.data(), count * sizeof(T));
}

cudaTextureObject_t texture(void *ptr, unsigned width, unsigned height, cudaChannelFormatDesc fmt, size_t texel) {
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = ptr;
    rd.res.pitch2D.desc = fmt;
    rd.res.pitch2D.width = width;
    rd.res.pitch2D.height = height;
    rd.res.pitch2D.pitchInBytes = width * texel;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) return 0;
    return t;
}

struct Params {
    unsigned width, height, num_nodes, num_surfels, num_edges, num_kp;
    float fx, fy, cx, cy, node_radius_square;
    int gn_iters, pcg_iters;
};

}  // namespace

static int run(const std::string &dir);

// The reference reports a failed check by throwing a heap-allocated std::runtime_error
// (LogMessageFatal, libs/star/common/logging.h:107-131); its message is printed here.
int main(int argc, char **argv) {
    if (argc != 2) return 2;
    try {
        return run(argv[1]);
    } catch (std::runtime_error *e) {
        std::fprintf(stderr, "starref_run: the reference stopped: %s\n", e->what());
        return 7;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "starref_run: %s\n", e.what());
        return 7;
    }
}

static int run(const std::string &dir) {
    Params p;
    {
        FILE *f = std::fopen((dir + "/params.txt").c_str(), "r");
        if (!f) return 3;
        const int got = std::fscanf(f, "%u %u %f %f %f %f %u %u %u %f %u %d %d", &p.width, &p.height, &p.fx, &p.fy,
                                    &p.cx, &p.cy, &p.num_nodes, &p.num_surfels, &p.num_edges, &p.node_radius_square,
                                    &p.num_kp, &p.gn_iters, &p.pcg_iters);
        std::fclose(f);
        if (got != 13) return 3;
    }
    // The reference's fixed capacities (Constants.cpp:7-18, geometry/constants.h:11-14): the harness
    // refuses inputs beyond them instead of letting the reference overrun its buffers.
    if (p.num_nodes < 3 || p.num_nodes > star::Constants::kMaxNumNodes || p.num_surfels == 0 ||
        p.num_surfels > star::Constants::kMaxNumSurfels || p.num_edges > p.num_nodes * star::d_node_knn_size ||
        p.num_kp == 0 || p.num_kp > star::Constants::kMaxMatchedSparseFeature || p.width == 0 || p.height == 0 ||
        p.gn_iters < 1 || p.pcg_iters < 1) {
        std::fprintf(stderr, "starref_run: input outside the reference's capacities\n");
        return 4;
    }

    const RefCamera cam{p.width, p.height, p.fx, p.fy, p.cx, p.cy};
    star::ConfigParser::Instance().loadCameraConfigFromJson(&cam);

    const size_t npix = (size_t)p.width * p.height;
    float4 *meas_vertex = upload<float4>(dir, "meas_vertex", 16 * npix, nullptr);
    float4 *meas_normal = upload<float4>(dir, "meas_normal", 16 * npix, nullptr);
    float4 *ref_vertex = upload<float4>(dir, "ref_vertex", 16 * npix, nullptr);
    float4 *ref_normal = upload<float4>(dir, "ref_normal", 16 * npix, nullptr);
    unsigned *index = upload<unsigned>(dir, "index", 4 * npix, nullptr);
    float2 *flow = upload<float2>(dir, "flow", 8 * npix, nullptr);   // zeros when no file
    auto *sknn = upload<ushortX<star::d_surfel_knn_size>>(dir, "surfel_knn", 8 * p.num_surfels, nullptr);
    auto *ssw = upload<floatX<star::d_surfel_knn_size>>(dir, "surfel_sw", 16 * p.num_surfels, nullptr);
    auto *scw = upload<floatX<star::d_surfel_knn_size>>(dir, "surfel_cw", 16 * p.num_surfels, nullptr);
    float4 *nodes = upload<float4>(dir, "nodes", 16 * p.num_nodes, nullptr);
    ushort3 *edges = upload<ushort3>(dir, "edges", 6 * p.num_edges, nullptr);
    auto *ncw = upload<floatX<star::d_node_knn_size>>(dir, "node_cw", 16 * p.num_nodes, nullptr);
    auto *nknn = upload<ushortX<star::d_surfel_knn_size>>(dir, "node_knn", 8 * p.num_nodes, nullptr);
    auto *nsw = upload<floatX<star::d_surfel_knn_size>>(dir, "node_sw", 16 * p.num_nodes, nullptr);
    float4 *motion = upload<float4>(dir, "node_motion", 16 * p.num_nodes, nullptr);   // zeros: no prediction
    auto *kp_knn = upload<ushortX<star::d_surfel_knn_size>>(dir, "kp_knn", 8 * p.num_kp, nullptr);
    auto *kp_sw = upload<floatX<star::d_surfel_knn_size>>(dir, "kp_sw", 16 * p.num_kp, nullptr);
    auto *kp_cw = upload<floatX<star::d_surfel_knn_size>>(dir, "kp_cw", 16 * p.num_kp, nullptr);
    float4 *kp_vertex = upload<float4>(dir, "kp_vertex", 16 * p.num_kp, nullptr);
    float4 *kp_normal = upload<float4>(dir, "kp_normal", 16 * p.num_kp, nullptr);
    int2 *kp_match = upload<int2>(dir, "kp_match", 8 * p.num_kp, nullptr);
    if (!meas_vertex || !meas_normal || !ref_vertex || !ref_normal || !index || !flow || !sknn || !ssw || !scw ||
        !nodes || !edges || !ncw || !nknn || !nsw || !motion || !kp_knn || !kp_sw || !kp_cw || !kp_vertex ||
        !kp_normal || !kp_match) {
        std::fprintf(stderr, "starref_run: upload failed\n");
        return 5;
    }
    const cudaChannelFormatDesc f4 = cudaCreateChannelDesc<float4>();
    const cudaTextureObject_t t_mv = texture(meas_vertex, p.width, p.height, f4, 16);
    const cudaTextureObject_t t_mn = texture(meas_normal, p.width, p.height, f4, 16);
    const cudaTextureObject_t t_rv = texture(ref_vertex, p.width, p.height, f4, 16);
    const cudaTextureObject_t t_rn = texture(ref_normal, p.width, p.height, f4, 16);
    const cudaTextureObject_t t_idx = texture(index, p.width, p.height, cudaCreateChannelDesc<unsigned>(), 4);
    const cudaTextureObject_t t_flow = texture(flow, p.width, p.height, cudaCreateChannelDesc<float2>(), 8);
    if (!t_mv || !t_mn || !t_rv || !t_rn || !t_idx || !t_flow) {
        std::fprintf(stderr, "starref_run: texture creation failed\n");
        return 5;
    }

    // the seven input structs, filled as examples/mono_star/app.cu:97-130 fills them
    star::Measure4Solver measure4solver;
    measure4solver.num_cam = 1;
    measure4solver.vertex_confid_map[0] = t_mv;
    measure4solver.normal_radius_map[0] = t_mn;
    measure4solver.index_map[0] = t_idx;
    star::Render4Solver render4solver;
    render4solver.num_cam = 1;
    render4solver.reference_vertex_map[0] = t_rv;
    render4solver.reference_normal_map[0] = t_rn;
    render4solver.index_map[0] = t_idx;
    star::OpticalFlow4Solver opticalflow4solver;
    opticalflow4solver.num_cam = 1;
    opticalflow4solver.opticalflow_map[0] = t_flow;
    star::NodeFlow4Solver nodeflow4solver;
    nodeflow4solver.num_node = p.num_nodes;
    nodeflow4solver.node_motion_pred = star::GArrayView<float4>(motion, p.num_nodes);
    star::KeyPoint4Solver keypoint4solver;
    keypoint4solver.kp_match = star::GArrayView<int2>(kp_match, p.num_kp);
    keypoint4solver.d_kp_vertex_confid = star::GArrayView<float4>(kp_vertex, p.num_kp);
    keypoint4solver.d_kp_normal_radius = star::GArrayView<float4>(kp_normal, p.num_kp);
    keypoint4solver.kp_vertex_confid = star::GArrayView<float4>(kp_vertex, p.num_kp);
    keypoint4solver.kp_normal_radius = star::GArrayView<float4>(kp_normal, p.num_kp);
    keypoint4solver.kp_knn = star::GArrayView<ushortX<star::d_surfel_knn_size>>(kp_knn, p.num_kp);
    keypoint4solver.kp_knn_spatial_weight = star::GArrayView<floatX<star::d_surfel_knn_size>>(kp_sw, p.num_kp);
    keypoint4solver.kp_knn_connect_weight = star::GArrayView<floatX<star::d_surfel_knn_size>>(kp_cw, p.num_kp);
    star::Geometry4Solver geometry4solver;
    geometry4solver.surfel_knn = star::GArrayView<ushortX<star::d_surfel_knn_size>>(sknn, p.num_surfels);
    geometry4solver.surfel_knn_spatial_weight = star::GArrayView<floatX<star::d_surfel_knn_size>>(ssw, p.num_surfels);
    geometry4solver.surfel_knn_connect_weight = star::GArrayView<floatX<star::d_surfel_knn_size>>(scw, p.num_surfels);
    geometry4solver.num_vertex = p.num_surfels;
    star::NodeGraph4Solver node_graph4solver;
    node_graph4solver.reference_node_coords = star::GArrayView<float4>(nodes, p.num_nodes);
    node_graph4solver.node_graph = star::GArrayView<ushort3>(edges, p.num_edges);
    node_graph4solver.node_knn_connect_weight = star::GArrayView<floatX<star::d_node_knn_size>>(ncw, p.num_nodes);
    node_graph4solver.nodel_knn = star::GArrayView<ushortX<star::d_surfel_knn_size>>(nknn, p.num_nodes);
    node_graph4solver.node_knn_spatial_weight = star::GArrayView<floatX<star::d_surfel_knn_size>>(nsw, p.num_nodes);
    node_graph4solver.num_node = p.num_nodes;
    node_graph4solver.node_radius_square = p.node_radius_square;
    const star::Extrinsic cam2world[star::d_max_cam] = {Eigen::Matrix4f::Identity(), Eigen::Matrix4f::Identity(),
                                                        Eigen::Matrix4f::Identity()};

    star::WarpSolver solver;
    solver.SetSolverInputs(measure4solver, render4solver, geometry4solver, node_graph4solver, nodeflow4solver,
                           opticalflow4solver, keypoint4solver, cam2world);

    auto &streams = solver.*get(StreamTag());
    auto &iteration = solver.*get(IterTag());
    const bool reference_counts = p.gn_iters == star::Constants::kNumGaussNewtonIterations && p.pcg_iters == 10;
    std::vector<float> diag, jtr, inv, step;
    if (reference_counts) {
        // WarpSolver::SolveStreamed itself; its index and last-iteration structures are read below
        solver.SolveStreamed();
    } else {
        solver.syncAllSolverStream();
        solver.buildSolverIndexStreamed();
        for (int it = 0; it < p.gn_iters; ++it) {
            (solver.*get(ComputeJTag()))();
            solver.SetPreconditionerBuilderAndJtJApplierInput();
            solver.SetJtJMaterializerInput();
            solver.BuildPreconditioner(streams[0]);
            solver.ComputeJtResidualIndexed(streams[1]);
            solver.MaterializeJtJNondiagonalBlocks(streams[2]);
            cudaSafeCall(cudaStreamSynchronize(streams[0]));
            cudaSafeCall(cudaStreamSynchronize(streams[1]));
            cudaSafeCall(cudaStreamSynchronize(streams[2]));
            const auto &rhs_builder = solver.*get(RhsTag());
            (solver.*get(JtJTag()))->AssembleBinBlockCSR(rhs_builder->JtJDiagonalBlocks(), streams[0]);
            solver.SolvePCGMaterialized(p.pcg_iters);
            if (it == 0) {
                cudaSafeCall(cudaDeviceSynchronize());
                rhs_builder->JtJDiagonalBlocks().Download(diag);
                rhs_builder->JtDotResidualValue().Download(jtr);
                rhs_builder->InversedPreconditioner().Download(inv);
                star::GArrayView<float>(iteration.CurrentWarpFieldUpdateBuffer().Ptr(),
                                        iteration.CurrentWarpFieldUpdateBuffer().Size())
                    .Download(step);
            }
            iteration.ApplyWarpFieldUpdate(streams[0]);
            cudaSafeCall(cudaStreamSynchronize(streams[0]));
        }
        solver.syncAllSolverStream();
    }
    cudaSafeCall(cudaDeviceSynchronize());

    // index structures (they depend on the inputs only)
    const auto terms = (solver.*get(FetcherTag()))->GetImageTermPixelAndKNN();
    bool ok = download(dir + "/out_pixels.bin", terms.pixels[0].Ptr(), terms.pixels[0].Size()) &&
              download(dir + "/out_term_knn.bin", terms.surfel_knn_patch_all.Ptr(), terms.surfel_knn_patch_all.Size()) &&
              download(dir + "/out_term_sw.bin", terms.knn_patch_spatial_weight_all.Ptr(),
                       terms.knn_patch_spatial_weight_all.Size()) &&
              download(dir + "/out_term_cw.bin", terms.knn_patch_connect_weight_all.Ptr(),
                       terms.knn_patch_connect_weight_all.Size());
    const auto n2t = (solver.*get(Node2TermTag()))->GetNode2TermMap();
    ok = ok && download(dir + "/out_n2t_offset.bin", n2t.offset.Ptr(), n2t.offset.Size()) &&
         download(dir + "/out_n2t_terms.bin", n2t.term_index.Ptr(), n2t.term_index.Size());
    const auto p2t = (solver.*get(PairTag()))->GetNodePair2TermMap();
    ok = ok && download(dir + "/out_pair_keys.bin", p2t.encoded_nodepair.Ptr(), p2t.encoded_nodepair.Size()) &&
         download(dir + "/out_pair_range.bin", p2t.nodepair_term_range.Ptr(), p2t.nodepair_term_range.Size()) &&
         download(dir + "/out_pair_terms.bin", p2t.nodepair_term_index.Ptr(), p2t.nodepair_term_index.Size()) &&
         download(dir + "/out_blkrow_offset.bin", p2t.blkrow_offset.Ptr(), p2t.blkrow_offset.Size());
    if (!reference_counts)
        ok = ok && write_file(dir + "/out_diag.bin", diag.data(), 4 * diag.size()) &&
             write_file(dir + "/out_jtr.bin", jtr.data(), 4 * jtr.size()) &&
             write_file(dir + "/out_inv_diag.bin", inv.data(), 4 * inv.size()) &&
             write_file(dir + "/out_step.bin", step.data(), 4 * step.size());
    const auto se3 = solver.SolvedNodeSE3();
    ok = ok && download(dir + "/out_se3.bin", se3.Ptr(), se3.Size());
    if (!ok) {
        std::fprintf(stderr, "starref_run: writing the outputs failed\n");
        return 6;
    }
    return 0;
}
