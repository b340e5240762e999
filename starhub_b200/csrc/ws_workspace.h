// Device workspace of one solver object: every buffer the solve touches is
// allocated once at creation, sized by the ws_config capacities, and reused by
// every solve (the reference preallocates at kMaxNumNodes and image size the
// same way, examples/mono_star/opt/WarpSolver.cu:82-103).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "ws_common.cuh"

namespace ws {

struct Workspace {
    // capacities
    int cap_scenes = 0;
    uint32_t cap_nodes = 0, cap_pixels = 0, cap_edges = 0, cap_features = 0;
    uint32_t cap_tiles = 0, cap_chunks = 0;
    uint32_t cap_n2t = 0, cap_pair_kv = 0, cap_half = 0, cap_blocks = 0;
    int precision = WS_PREC_MIXED;
    int device = 0;
    int num_sms = 0;
    int pcg_grid = 0;           // co-resident blocks for the persistent PCG kernel
    // launch shapes picked by ws_autotune (defaults until then); none of them changes a result
    struct Tuning {
        int node_threads = 128;     // threads per block of the node assembly (64, 128, 256)
        int pair_threads = 128;     // threads per block of the pair assembly
        int pcg_blocks_per_sm = 64; // upper bound on PCG blocks per SM (capped by co-residency)
        bool tuned = false;
    } tune;

    // current batch (host mirror)
    int num_scenes = 0;
    uint32_t total_nodes = 0, total_edges = 0, total_tiles = 0, total_chunks = 0, total_features = 0;
    int node_bits = 1;
    std::vector<Scene> h_scenes;
    bool have_inputs = false;
    bool have_solution = false;

    // scene tables
    Scene *scenes = nullptr;            // [cap_scenes]
    Plan *plan = nullptr;               // [cap_scenes]
    uint32_t *counts = nullptr;         // [8]: dense total, n2t kv total, pair kv total, half total, ...
    uint32_t *tile_scene = nullptr;     // [cap_tiles]
    uint32_t *tile_count = nullptr;     // [cap_tiles + 1] (exclusive offsets after the scan)
    uint32_t *node_scene = nullptr;     // [cap_nodes]
    uint32_t *edge_scene = nullptr;     // [cap_edges]
    uint32_t *chunk_scene = nullptr;    // [cap_chunks]
    uint32_t *chunk_row = nullptr;      // [cap_chunks] first global row of the chunk
    uint32_t *scan_tmp = nullptr;       // scan tile sums
    uint32_t *sort_hist = nullptr;      // radix histograms
    uint32_t *sort_digit = nullptr;     // [256]

    // dense terms (compacted pixels)
    ushort4 *d_pixels = nullptr;        // [cap_pixels]
    ushort4 *d_knn = nullptr;           // [cap_pixels]
    float4 *d_sw = nullptr, *d_cw = nullptr;
    uint32_t *d_scene = nullptr;        // [cap_pixels]
    float *d_record = nullptr;          // [cap_pixels * kDenseRecord]
    int dense_channels = 3;             // 3 when a scene of the batch has the flow term, else 1 (64-byte records)
    float *r_record = nullptr;          // [cap_edges * kRegRecord]

    // node->term
    uint32_t *n2t_key = nullptr, *n2t_val = nullptr;         // [cap_n2t]
    uint32_t *n2t_key_alt = nullptr, *n2t_val_alt = nullptr;
    uint32_t *n2t_offset = nullptr;                          // [cap_nodes + 1]
    const uint32_t *n2t_sorted_val = nullptr;                // points into val or val_alt
    const uint32_t *n2t_sorted_key = nullptr;

    // pair->term, built row by row: per row its upper pairs' columns and entry counts (at most
    // kRowPairsMax a row), its first pair and first entry; pair_val holds every pair's term list
    uint32_t *row_pair_cols = nullptr, *row_pair_cnts = nullptr;   // [cap_nodes * kRowPairsMax]
    uint32_t *row_pair_first = nullptr, *row_entry_first = nullptr;   // [cap_nodes + 1]
    uint32_t *pair_val = nullptr;                            // [cap_pair_kv]
    const uint32_t *pair_sorted_val = nullptr;
    uint32_t *half_row = nullptr, *half_col = nullptr;       // [cap_half]
    uint32_t *half_begin = nullptr, *half_end = nullptr;
    uint32_t *half_scene = nullptr;                          // [cap_half] scene of the pair's nodes
    uint32_t *half_slot_up = nullptr, *half_slot_lo = nullptr;

    // block CSR
    uint32_t *row_cnt_up = nullptr, *row_cnt_lo = nullptr;   // [cap_nodes]
    uint32_t *row_first = nullptr;                           // [cap_nodes]
    uint32_t *rowptr = nullptr;                              // [cap_nodes + 1]
    uint32_t *col_key = nullptr, *col_val = nullptr, *col_key_alt = nullptr, *col_val_alt = nullptr; // [cap_half]
    uint32_t *colidx = nullptr;                              // [cap_blocks]
    // Symmetric block store: row by row, the diagonal block and then one block per upper pair
    // (row < col, column order).  These are the row's items, item_ptr[row] .. item_ptr[row + 1);
    // pair h is item h + row + 1.  item_info holds per item the column, with kItemRowStart set
    // on a row's first (diagonal) item, and then the lower entry of the transposed use (an upper
    // item) or the row's scene (a diagonal item); lower entries are numbered by row, then
    // column, and contrib holds one 6-float vector per lower entry for the PCG.
    uint32_t cap_items = 0;                                  // cap_nodes + cap_half
    uint32_t *item_ptr = nullptr;                            // [cap_nodes + 1]
    uint2 *item_info = nullptr;                              // [cap_items]
    // Per item, 4 bytes for the standalone SpMV: the column, with kItemRowStart set on a row's
    // first (diagonal) item; rows follow from counting those marks.
    uint32_t *item_col = nullptr;                            // [cap_items]
    float *sym_blocks = nullptr;                             // [cap_items * 36]
    float *contrib = nullptr;                                // [cap_half * 6]
    uint32_t *pcg_warp_groups = nullptr;                     // [kPcgUnitsPerWarp * pcg_grid * warps per block + 2]:
                                                             // first row group of every PCG work unit, the
                                                             // group count, the first half's unit count
    uint4 *pcg_unit_info = nullptr;                          // [2 * PCG work units]: groups, rows, items, scenes
    uint32_t *pcg_tickets = nullptr;                         // [4]: [0] PCG work-unit tickets, zeroed per launch
    float *mf_ux = nullptr;             // matrix-free SpMV scratch: J x per dense term and edge (float4),
                                        // allocated on first use

    // per-node system and PCG state (stride kVecStride)
    float *inv_diag = nullptr;          // [cap_nodes * 36]
    double *diag64 = nullptr;           // [cap_nodes * 21] FP64 diagonal blocks (upper triangle)
    float *jtr = nullptr, *x = nullptr, *r = nullptr, *q = nullptr;
    // PCG search vectors: per node s (6) then d (6), kSdStride floats, two copies that swap
    // roles every iteration (the SpMV reads one while the other is written)
    float *sd0 = nullptr, *sd1 = nullptr;
    float *se3 = nullptr;               // [cap_nodes * 8] current warp
    float4 *centers = nullptr;          // [cap_nodes] twist centre per node (current GN iteration)
    double *chunk_partial = nullptr;    // [cap_chunks]
    double *scene_scalars = nullptr;    // [cap_scenes * 8]: delta, alpha, beta, dq ...
    uint32_t *scene_counter = nullptr;  // [cap_scenes * 64]: PCG tickets and generations per scene
    int *error_flag = nullptr;          // [4]

    // pinned host staging of the scene tables (uploaded at the start of every solve)
    void *h_tables = nullptr;
    size_t h_tables_bytes = 0;
    std::vector<const float *> init_ptrs;     // per-scene initial warp (device) or null
    cudaEvent_t tables_free = nullptr;        // recorded once a solve has consumed the tables
    bool tables_in_flight = false;

    // per-phase event timing (ws_set_profiling)
    bool profiling = false;
    static constexpr int kPhases = 5;
    std::vector<cudaEvent_t> prof_events;       // recorded in order
    std::vector<int> prof_phase;                // phase id of the interval ending at each event
    std::vector<int> prof_launches;             // launches in that interval
    int launches = 0;                           // launch counter of the current interval
    int prof_count = 0;                         // events recorded by the last profiled solve
    int graph_kernels = 0;                      // kernel nodes of the captured graph

    // graph capture cache
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<uint64_t> graph_key;
    std::vector<const float *> graph_init;
    cudaStream_t last_stream = nullptr;
};

// Index build (ws_index.cu): compaction, node->term, pair->term, block CSR.
void index_build(Workspace &w, cudaStream_t st);
// One Gauss-Newton iteration (ws_solve.cu): term evaluation, assembly, PCG, update,
// and its four phases.
cudaError_t gn_iteration(Workspace &w, int pcg_iters, cudaStream_t st);
void gn_eval(Workspace &w, cudaStream_t st);
void gn_assemble_node(Workspace &w, cudaStream_t st);
void gn_assemble_pair(Workspace &w, cudaStream_t st);
cudaError_t gn_pcg(Workspace &w, int pcg_iters, cudaStream_t st);
// Initialise the warp field of every scene (identity or the given initial warp).
void init_warp(Workspace &w, cudaStream_t st);
// Occupancy of the persistent PCG kernel.
int pcg_max_blocks(int device);
int pcg_launch_blocks(const Workspace &w);
void pcg_ranges(Workspace &w, cudaStream_t st);
// First row group of the second half of the scenes in the PCG's schedule (a scene boundary).
uint32_t pcg_split_group(const Workspace &w);
cudaError_t gn_spmv(Workspace &w, const float *x, float *y, cudaStream_t st);
// Runs the PCG's bounded scene wait on a generation nothing advances; *status gets the flag it left.
cudaError_t pcg_wait_selftest(int *status, cudaStream_t st);
cudaError_t grid_barrier_selftest(int *flags, cudaStream_t st);
cudaError_t gn_spmv_matrix_free(Workspace &w, const float *x, float *y, float *ux_dense, float *ux_reg,
                                cudaStream_t st);
int pcg_warps_per_block();

// Launch accounting for the measurement hooks.
inline void count_launch(Workspace &w, int n = 1) { w.launches += n; }

// Counters slot indices.
enum { kCntDense = 0, kCntN2T = 1, kCntPairKV = 2, kCntHalf = 3, kCntPairValid = 4 };

}  // namespace ws
