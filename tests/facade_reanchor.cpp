// star::b200::NodeGraph::ReAnchor and star::b200::Skinner through the C++ facade
// (include/starhub_b200/warp_solver.hpp), called as the reference's geometry processor calls
// star::NodeGraph::ReAnchor and star::Skinner (libs/star/geometry/node_graph/NodeGraph.cu:574-650,
// Skinner.cu:336-415).
//
// usage: facade_reanchor <surfels.bin> <out.bin>
//   builds graph A from the surfels (node radius 2 cm, K = 4), moves A's live nodes by +1 cm in x,
//   marks node 7 deleted and rebuilds A's graph from the live coordinates; re-anchors B from A;
//   skins the surfels against B's reference nodes.  Writes, in order: A's node count, A's live
//   nodes, B's node count, B's reference nodes, A's and B's knn, B's status, and the surfels' knn
//   and spatial weights.
#include <cstdio>
#include <vector>

#include "starhub_b200/warp_solver.hpp"

using namespace star::b200;

int main(int argc, char **argv) {
    if (argc != 3) return 2;
    std::vector<float4> surfels;
    {
        FILE *f = std::fopen(argv[1], "rb");
        if (!f) return 3;
        float4 p;
        while (std::fread(&p, sizeof(p), 1, f) == 1) surfels.push_back(p);
        std::fclose(f);
    }
    const unsigned ns = (unsigned)surfels.size();
    float4 *d_surfels = nullptr;
    ushortX<4> *d_knn = nullptr;
    floatX<4> *d_sw = nullptr, *d_cw = nullptr;
    cudaMalloc(&d_surfels, 16ull * ns);
    cudaMalloc(&d_knn, 8ull * ns);
    cudaMalloc(&d_sw, 16ull * ns);
    cudaMalloc(&d_cw, 16ull * ns);
    cudaMemcpy(d_surfels, surfels.data(), 16ull * ns, cudaMemcpyHostToDevice);
    try {
        auto a = std::make_shared<NodeGraph>(0.02f, 8192, 4);
        auto b = std::make_shared<NodeGraph>(0.02f, 8192, 4);
        a->InitializeNodeGraphFromVertex(d_surfels, ns, 1, true, 0);
        const unsigned n = a->GetNodeSize();
        std::vector<float4> live(n);
        cudaMemcpy(live.data(), a->GetLiveNodeCoordinate(), 16ull * n, cudaMemcpyDeviceToHost);
        for (auto &v : live) v.x += 0.01f;
        cudaMemcpy(a->LiveNodeCoordinate(), live.data(), 16ull * n, cudaMemcpyHostToDevice);
        const uint2 deleted = make_uint2(0u, WS_DELETED_NODE_STATUS);
        cudaMemcpy(a->GetNodeStatus() + 7, &deleted, 8, cudaMemcpyHostToDevice);
        a->BuildNodeGraphFromScratch(false, 0);
        a->ResetNodeGraphConnection(0);
        NodeGraph::ReAnchor(a, b, 0);

        Geometry4Skinner geometry;
        geometry.reference_vertex_confid = GArrayView<float4>(d_surfels, ns);
        geometry.live_vertex_confid = GArrayView<float4>(d_surfels, ns);
        geometry.surfel_knn = d_knn;
        geometry.surfel_knn_spatial_weight = d_sw;
        geometry.surfel_knn_connect_weight = d_cw;
        NodeGraph4Skinner skinner_graph = b->GenerateNodeGraph4Skinner();
        Skinner::PerformSkinningFromRef(geometry, skinner_graph, 0);
        cudaDeviceSynchronize();

        const unsigned nb = b->GetNodeSize();
        std::vector<float4> bref(nb);
        std::vector<uint16_t> aknn(4ull * n), bknn(4ull * nb), sknn(4ull * ns);
        std::vector<uint2> bst(nb);
        std::vector<float> ssw(4ull * ns);
        cudaMemcpy(bref.data(), b->GetReferenceNodeCoordinate(), 16ull * nb, cudaMemcpyDeviceToHost);
        cudaMemcpy(aknn.data(), a->GetNodeKnn(), 8ull * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(bknn.data(), b->GetNodeKnn(), 8ull * nb, cudaMemcpyDeviceToHost);
        cudaMemcpy(bst.data(), b->GetNodeStatusReadOnly(), 8ull * nb, cudaMemcpyDeviceToHost);
        cudaMemcpy(sknn.data(), d_knn, 8ull * ns, cudaMemcpyDeviceToHost);
        cudaMemcpy(ssw.data(), d_sw, 16ull * ns, cudaMemcpyDeviceToHost);
        FILE *f = std::fopen(argv[2], "wb");
        if (!f) return 4;
        std::fwrite(&n, 4, 1, f);
        std::fwrite(live.data(), 16, n, f);
        std::fwrite(&nb, 4, 1, f);
        std::fwrite(bref.data(), 16, nb, f);
        std::fwrite(aknn.data(), 2, 4ull * n, f);
        std::fwrite(bknn.data(), 2, 4ull * nb, f);
        std::fwrite(bst.data(), 8, nb, f);
        std::fwrite(sknn.data(), 2, 4ull * ns, f);
        std::fwrite(ssw.data(), 4, 4ull * ns, f);
        std::fclose(f);
    } catch (const Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 5;
    }
    return 0;
}
