// ws_server.cu -- persistent request loop with continuous batching (host code).
//
// A server owns `executors` solvers, each with its own stream and completion event and a
// host thread.  A free executor's thread takes, under the server lock, waiting frames whose
// streams have no frame in flight and that fit the executor's capacities (longest waits
// relative to their solve's size first, see form_batch), launches them as one batched solve
// (ws_set_batch + ws_solve), copies every solution back
// into its stream's resident warp on the same stream, waits for the batch (blocking event,
// no spinning), and marks its requests done.  So a batch starts as soon as an executor is
// free, requests that arrive while others are on the GPU join the next batch, and batches
// on different executors overlap on the device.  The per-scene results do not depend on the
// batch (the batched solver is scene-local), so a request's result is the same alone and
// in any mix.
//
// Memory admission: executors are sized at creation (bytes measured around their
// allocation); a scene is admitted by the bytes of its resident copy; executor bytes +
// resident bytes never exceed the budget.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/warpsolve.h"
#include "ws_workspace.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t rounded(size_t bytes) { return (bytes + 511) & ~size_t(511); }

struct Resident {
    ws_inputs in{};               // static fields point at `buffers`; map fields unused
    std::vector<void *> buffers;
    size_t bytes = 0;
    float *warp = nullptr;        // 8 floats per node: the stream's latest solution
    int pending = 0;              // frames waiting or in flight
    bool in_flight = false;
};

struct Request {
    int scene = -1;
    ws_frame frame{};
    Clock::time_point t_submit, t_launch, t_done;
    int status = WS_ERR_NOT_READY;
    int batch_scenes = 0;
    int num_nodes = 0;
    bool done = false;
};

struct Executor {
    ws_solver *solver = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::thread thread;
};

}  // namespace

struct ws_server {
    ws_server_config cfg{};
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    std::deque<unsigned long long> waiting;
    std::unordered_map<unsigned long long, Request> requests;
    std::map<int, Resident> scenes;
    std::vector<Executor> execs;
    cudaStream_t control = nullptr;
    bool stop = false;
    unsigned long long next_id = 1;
    int next_scene = 0;
    size_t exec_bytes = 0, resident_bytes = 0;
    unsigned long long submitted = 0, completed = 0, failed = 0, batches = 0, batch_scene_sum = 0;
    std::vector<double> latencies;
};

namespace {

// A waiting frame whose stream has nothing in flight (the server lock is held).
bool has_ready(const ws_server *s) {
    for (unsigned long long id : s->waiting) {
        const Request &r = s->requests.at(id);
        if (!s->scenes.at(r.scene).in_flight) return true;
    }
    return false;
}

// Batch for one executor (the server lock is held).  Ready frames are taken in the order of
// their wait relative to the size of their own solve, wait / (1 + nodes / kSolveNodes): a lone
// solve costs about a fixed latency plus a part that grows with the nodes, so a small scene's
// frame, whose solve is short, comes before a larger one that has waited as long.  The first
// frame sets the batch's scale: later ones join only up to kBatchSizeRatio times its nodes,
// so a small frame does not wait for a much larger scene's solve.  The first frame always fits
// an empty batch (checked at submit), and every frame's priority grows while it waits.
constexpr double kSolveNodes = 12000.0;
constexpr double kBatchSizeRatio = 2.0;
std::vector<unsigned long long> form_batch(ws_server *s) {
    std::vector<unsigned long long> batch;
    const ws_server_config &c = s->cfg;
    const Clock::time_point now = Clock::now();
    std::vector<std::pair<double, unsigned long long>> order;
    for (unsigned long long id : s->waiting) {
        const Request &r = s->requests.at(id);
        const Resident &sc = s->scenes.at(r.scene);
        if (sc.in_flight) continue;
        const double waited = ms_between(r.t_submit, now);
        order.push_back({waited / (1.0 + sc.in.num_nodes / kSolveNodes), id});
    }
    // highest priority first; equal priorities keep the arrival order
    std::stable_sort(order.begin(), order.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    long long nodes = 0, pixels = 0, edges = 0;
    int head_nodes = 0;
    for (const auto &o : order) {
        Request &r = s->requests.at(o.second);
        Resident &sc = s->scenes.at(r.scene);
        if (sc.in_flight) continue;   // the stream's earlier frame is already in this batch
        if (!batch.empty() && sc.in.num_nodes > kBatchSizeRatio * head_nodes) continue;
        const long long px = (long long)sc.in.width * sc.in.height;
        const bool fits = (int)batch.size() < c.max_batch_scenes && nodes + sc.in.num_nodes <= c.max_batch_nodes &&
                          pixels + px <= c.max_batch_pixels && edges + sc.in.num_edges <= c.max_batch_edges;
        if (!fits) continue;
        if (batch.empty()) head_nodes = sc.in.num_nodes;
        sc.in_flight = true;
        nodes += sc.in.num_nodes;
        pixels += px;
        edges += sc.in.num_edges;
        batch.push_back(o.second);
    }
    for (unsigned long long id : batch) s->waiting.erase(std::find(s->waiting.begin(), s->waiting.end(), id));
    return batch;
}

void executor_loop(ws_server *s, int index) {
    cudaSetDevice(s->cfg.device);
    Executor &x = s->execs[index];
    std::vector<ws_inputs> ins;
    std::vector<float *> outs;
    for (;;) {
        std::vector<unsigned long long> batch;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [&] { return s->stop || has_ready(s); });
            if (s->stop) return;
            batch = form_batch(s);
            if (batch.empty()) continue;
            const Clock::time_point now = Clock::now();
            ins.clear();
            outs.clear();
            for (unsigned long long id : batch) {
                Request &r = s->requests.at(id);
                const Resident &sc = s->scenes.at(r.scene);
                ws_inputs in = sc.in;
                in.measure_vertex_confid = r.frame.measure_vertex_confid;
                in.measure_normal_radius = r.frame.measure_normal_radius;
                in.reference_vertex = r.frame.reference_vertex;
                in.reference_normal = r.frame.reference_normal;
                in.index_map = r.frame.index_map;
                in.opticalflow = r.frame.opticalflow;
                in.pitch = r.frame.pitch;
                std::memcpy(in.cam2world, r.frame.cam2world, sizeof(in.cam2world));
                in.node_motion_pred = r.frame.node_motion_pred;
                in.init_node_se3 = sc.warp;
                ins.push_back(in);
                outs.push_back(r.frame.solution_out);
                r.t_launch = now;
                r.batch_scenes = (int)batch.size();
                r.num_nodes = sc.in.num_nodes;
            }
            ++s->batches;
            s->batch_scene_sum += batch.size();
            if (has_ready(s)) s->cv_work.notify_one();   // frames left over for another free executor
        }
        // launch outside the lock; resident warps are only written by the executor whose
        // batch holds their stream, and their buffers live until the stream is removed,
        // which waits for its frames
        int st = ws_set_batch(x.solver, ins.data(), (int)ins.size());
        if (st == WS_OK) st = ws_solve(x.solver, s->cfg.gn_iters, s->cfg.pcg_iters, x.stream);
        if (st == WS_OK) {
            for (int i = 0; i < (int)ins.size(); ++i) {
                const float *sol = nullptr;
                int n = 0;
                st = ws_get_solution(x.solver, i, &sol, &n);
                if (st != WS_OK) break;
                if (cudaMemcpyAsync(const_cast<float *>(ins[i].init_node_se3), sol, 32ull * n,
                                    cudaMemcpyDeviceToDevice, x.stream) != cudaSuccess) {
                    st = WS_ERR_CUDA;
                    break;
                }
                if (outs[i] && cudaMemcpyAsync(outs[i], sol, 32ull * n, cudaMemcpyDeviceToDevice, x.stream) !=
                                   cudaSuccess) {
                    st = WS_ERR_CUDA;
                    break;
                }
            }
        }
        if (cudaEventRecord(x.done, x.stream) != cudaSuccess && st == WS_OK) st = WS_ERR_CUDA;
        if (cudaEventSynchronize(x.done) != cudaSuccess && st == WS_OK) st = WS_ERR_CUDA;
        if (st == WS_OK) st = ws_sync_status(x.solver);
        const Clock::time_point t = Clock::now();
        {
            std::lock_guard<std::mutex> lk(s->m);
            for (unsigned long long id : batch) {
                Request &r = s->requests.at(id);
                r.status = st;
                r.t_done = t;
                r.done = true;
                Resident &sc = s->scenes.at(r.scene);
                sc.in_flight = false;
                --sc.pending;
                if (st == WS_OK) {
                    ++s->completed;
                    s->latencies.push_back(ms_between(r.t_submit, t));
                } else {
                    ++s->failed;
                }
            }
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

void free_resident(Resident &r) {
    for (void *p : r.buffers) cudaFree(p);
    r.buffers.clear();
}

// Device copy of `n` bytes from the caller's pointer into a new resident buffer.
int copy_in(ws_server *s, Resident &r, const void *src, size_t n, void **dst) {
    *dst = nullptr;
    if (!src || n == 0) return WS_OK;
    if (cudaMalloc(dst, n) != cudaSuccess) {
        cudaGetLastError();
        return WS_ERR_CAPACITY;
    }
    r.buffers.push_back(*dst);
    return cudaMemcpyAsync(*dst, src, n, cudaMemcpyDeviceToDevice, s->control) == cudaSuccess ? WS_OK : WS_ERR_CUDA;
}

void fill_info(const Request &r, ws_request_info *info) {
    info->status = r.done ? r.status : WS_ERR_NOT_READY;
    info->scene = r.scene;
    info->num_nodes = r.num_nodes;
    info->batch_scenes = r.batch_scenes;
    info->queue_ms = r.batch_scenes ? ms_between(r.t_submit, r.t_launch) : 0.0;
    info->solve_ms = r.done ? ms_between(r.t_launch, r.t_done) : 0.0;
    info->latency_ms = r.done ? ms_between(r.t_submit, r.t_done) : 0.0;
}

void destroy_all(ws_server *s) {
    for (Executor &x : s->execs) {
        if (x.solver) ws_destroy(x.solver);
        if (x.done) cudaEventDestroy(x.done);
        if (x.stream) cudaStreamDestroy(x.stream);
    }
    s->execs.clear();
    for (auto &kv : s->scenes) free_resident(kv.second);
    s->scenes.clear();
    if (s->control) cudaStreamDestroy(s->control);
    s->control = nullptr;
}

}  // namespace

extern "C" {

int ws_server_create(const ws_server_config *cfg, ws_server **out) {
    if (!cfg || !out) return WS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cfg->executors < 1 || cfg->max_batch_scenes < 1 || cfg->max_batch_nodes < 1 || cfg->max_batch_pixels < 1 ||
        cfg->max_batch_edges < 1 || cfg->gn_iters < 0 || cfg->pcg_iters < 0 ||
        (cfg->precision != WS_PREC_MIXED && cfg->precision != WS_PREC_FP32))
        return WS_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return WS_ERR_NO_DEVICE;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return WS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(cfg->device);
    ws_server *s = new (std::nothrow) ws_server;
    if (!s) return WS_ERR_CAPACITY;
    s->cfg = *cfg;
    int st = WS_OK;
    if (cudaStreamCreateWithFlags(&s->control, cudaStreamNonBlocking) != cudaSuccess) st = WS_ERR_CUDA;
    ws_config wc;
    wc.max_scenes = cfg->max_batch_scenes;
    wc.max_total_nodes = cfg->max_batch_nodes;
    wc.max_total_pixels = cfg->max_batch_pixels;
    wc.max_total_edges = cfg->max_batch_edges;
    wc.max_total_features = 1024 * cfg->max_batch_scenes;
    wc.precision = cfg->precision;
    wc.device = cfg->device;
    s->execs.resize(cfg->executors);
    // The persistent PCG is a cooperative launch that needs all of its blocks resident, so two
    // batches' PCGs overlap only when their grids fit on the SMs together: every executor's PCG
    // gets an equal share of the blocks an SM holds (at least one per SM).
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device);
    const int pcg_per_sm = std::max(1, ws::pcg_max_blocks(cfg->device) / std::max(1, sms) / cfg->executors);
    for (int i = 0; i < cfg->executors && st == WS_OK; ++i) {
        size_t free0 = 0, free1 = 0, total = 0;
        cudaMemGetInfo(&free0, &total);
        Executor &x = s->execs[i];
        st = ws_create(&wc, &x.solver);
        if (st == WS_OK) {
            ws_tuning t{};
            t.node_threads = 128;
            t.pair_threads = 128;
            t.pcg_blocks_per_sm = pcg_per_sm;
            st = ws_set_tuning(x.solver, &t);
        }
        if (st == WS_OK && cudaStreamCreateWithFlags(&x.stream, cudaStreamNonBlocking) != cudaSuccess) st = WS_ERR_CUDA;
        if (st == WS_OK && cudaEventCreateWithFlags(&x.done, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess)
            st = WS_ERR_CUDA;
        cudaMemGetInfo(&free1, &total);
        s->exec_bytes += free0 > free1 ? free0 - free1 : 0;
        if (st == WS_OK && s->exec_bytes > cfg->memory_budget) st = WS_ERR_CAPACITY;
    }
    if (st != WS_OK) {
        destroy_all(s);
        delete s;
        return st;
    }
    for (int i = 0; i < cfg->executors; ++i) s->execs[i].thread = std::thread(executor_loop, s, i);
    *out = s;
    return WS_OK;
}

int ws_server_destroy(ws_server *s) {
    if (!s) return WS_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (Executor &x : s->execs)
        if (x.thread.joinable()) x.thread.join();   // a launched batch always runs to completion first
    s->cv_done.notify_all();
    cudaSetDevice(s->cfg.device);
    destroy_all(s);
    delete s;
    return WS_OK;
}

int ws_server_add_scene(ws_server *s, const ws_inputs *in, int *scene_id) {
    if (!s || !in || !scene_id) return WS_ERR_INVALID_ARGUMENT;
    if (in->width <= 0 || in->height <= 0 || in->num_nodes <= 0 || in->num_nodes > 65535 || in->num_surfels < 0 ||
        in->num_edges < 0 || in->graph_k <= 0 || !in->reference_node_coords || !in->node_knn_connect_weight ||
        (in->num_surfels > 0 && (!in->surfel_knn || !in->surfel_knn_spatial_weight || !in->surfel_knn_connect_weight)) ||
        (in->num_edges > 0 && !in->node_graph) || in->num_features < 0 || (in->num_features > 0 && !in->feature_knn))
        return WS_ERR_INVALID_ARGUMENT;
    const ws_server_config &c = s->cfg;
    if (in->num_nodes > c.max_batch_nodes || (long long)in->width * in->height > c.max_batch_pixels ||
        in->num_edges > c.max_batch_edges)
        return WS_ERR_CAPACITY;
    const size_t S = (size_t)in->num_surfels, N = (size_t)in->num_nodes, E = (size_t)in->num_edges;
    const size_t F = (size_t)in->num_features, K = (size_t)in->graph_k;
    const size_t bytes = rounded(8 * S) + 2 * rounded(16 * S) + rounded(16 * N) + rounded(6 * E) + rounded(4 * K * N) +
                         rounded(8 * F) + rounded(32 * N);
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->exec_bytes + s->resident_bytes + bytes > c.memory_budget) return WS_ERR_CAPACITY;
        s->resident_bytes += bytes;   // reserved now, released below on failure
    }
    cudaSetDevice(c.device);
    Resident r;
    r.in = *in;
    r.bytes = bytes;
    void *p = nullptr;
    int st = WS_OK;
    if (st == WS_OK) st = copy_in(s, r, in->surfel_knn, 8 * S, &p), r.in.surfel_knn = (const uint16_t *)p;
    if (st == WS_OK) st = copy_in(s, r, in->surfel_knn_spatial_weight, 16 * S, &p), r.in.surfel_knn_spatial_weight = (const float *)p;
    if (st == WS_OK) st = copy_in(s, r, in->surfel_knn_connect_weight, 16 * S, &p), r.in.surfel_knn_connect_weight = (const float *)p;
    if (st == WS_OK) st = copy_in(s, r, in->reference_node_coords, 16 * N, &p), r.in.reference_node_coords = (const float *)p;
    if (st == WS_OK) st = copy_in(s, r, in->node_graph, 6 * E, &p), r.in.node_graph = (const uint16_t *)p;
    if (st == WS_OK) st = copy_in(s, r, in->node_knn_connect_weight, 4 * K * N, &p), r.in.node_knn_connect_weight = (const float *)p;
    if (st == WS_OK) st = copy_in(s, r, in->feature_knn, 8 * F, &p), r.in.feature_knn = (const uint16_t *)p;
    if (st == WS_OK) {
        void *w = nullptr;
        if (cudaMalloc(&w, 32 * N) != cudaSuccess) {
            cudaGetLastError();
            st = WS_ERR_CAPACITY;
        } else {
            r.buffers.push_back(w);
            r.warp = (float *)w;
            if (in->init_node_se3) {
                if (cudaMemcpyAsync(w, in->init_node_se3, 32 * N, cudaMemcpyDeviceToDevice, s->control) != cudaSuccess)
                    st = WS_ERR_CUDA;
            } else {
                std::vector<float> ident(8 * N, 0.f);
                for (size_t i = 0; i < N; ++i) ident[8 * i + 3] = 1.f;   // q0 = (0, 0, 0, 1) (xyzw), q1 = 0
                if (cudaMemcpyAsync(w, ident.data(), 32 * N, cudaMemcpyHostToDevice, s->control) != cudaSuccess)
                    st = WS_ERR_CUDA;
                if (st == WS_OK && cudaStreamSynchronize(s->control) != cudaSuccess) st = WS_ERR_CUDA;
            }
        }
    }
    if (st == WS_OK && cudaStreamSynchronize(s->control) != cudaSuccess) st = WS_ERR_CUDA;
    // frame fields belong to ws_submit
    r.in.measure_vertex_confid = r.in.measure_normal_radius = r.in.reference_vertex = r.in.reference_normal = nullptr;
    r.in.index_map = nullptr;
    r.in.opticalflow = nullptr;
    r.in.node_motion_pred = nullptr;
    r.in.init_node_se3 = nullptr;
    std::lock_guard<std::mutex> lk(s->m);
    if (st != WS_OK) {
        free_resident(r);
        s->resident_bytes -= bytes;
        return st;
    }
    const int id = s->next_scene++;
    s->scenes.emplace(id, std::move(r));
    *scene_id = id;
    return WS_OK;
}

int ws_server_remove_scene(ws_server *s, int scene_id) {
    if (!s) return WS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->scenes.find(scene_id);
    if (it == s->scenes.end()) return WS_ERR_INVALID_ARGUMENT;
    if (it->second.pending > 0) return WS_ERR_NOT_READY;
    cudaSetDevice(s->cfg.device);
    free_resident(it->second);
    s->resident_bytes -= it->second.bytes;
    s->scenes.erase(it);
    return WS_OK;
}

int ws_submit(ws_server *s, int scene_id, const ws_frame *frame, unsigned long long *request_id) {
    if (!s || !frame || !request_id) return WS_ERR_INVALID_ARGUMENT;
    if (!frame->measure_vertex_confid || !frame->measure_normal_radius || !frame->reference_vertex ||
        !frame->reference_normal || !frame->index_map || frame->pitch < 0)
        return WS_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(s->m);
        if (s->stop) return WS_ERR_NOT_READY;
        auto it = s->scenes.find(scene_id);
        if (it == s->scenes.end()) return WS_ERR_INVALID_ARGUMENT;
        const unsigned long long id = s->next_id++;
        Request &r = s->requests[id];
        r.scene = scene_id;
        r.frame = *frame;
        r.t_submit = Clock::now();
        r.num_nodes = it->second.in.num_nodes;
        ++it->second.pending;
        ++s->submitted;
        s->waiting.push_back(id);
        *request_id = id;
    }
    s->cv_work.notify_one();
    return WS_OK;
}

int ws_poll(ws_server *s, unsigned long long request_id, ws_request_info *info) {
    if (!s || !info) return WS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return WS_ERR_INVALID_ARGUMENT;
    fill_info(it->second, info);
    return info->status;
}

int ws_wait(ws_server *s, unsigned long long request_id, ws_request_info *info) {
    if (!s || !info) return WS_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return WS_ERR_INVALID_ARGUMENT;
    s->cv_done.wait(lk, [&] { return it->second.done || s->stop; });
    fill_info(it->second, info);
    return info->status;
}

int ws_server_forget(ws_server *s, unsigned long long request_id) {
    if (!s) return WS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return WS_ERR_INVALID_ARGUMENT;
    if (!it->second.done) return WS_ERR_NOT_READY;
    s->requests.erase(it);
    return WS_OK;
}

int ws_server_get_warp(ws_server *s, int scene_id, const float **dev_dq, int *num_nodes) {
    if (!s || !dev_dq || !num_nodes) return WS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->scenes.find(scene_id);
    if (it == s->scenes.end()) return WS_ERR_INVALID_ARGUMENT;
    *dev_dq = it->second.warp;
    *num_nodes = it->second.in.num_nodes;
    return WS_OK;
}

int ws_server_copy_warp(ws_server *s, int scene_id, float *dev_out) {
    if (!s || !dev_out) return WS_ERR_INVALID_ARGUMENT;
    const float *src = nullptr;
    size_t n = 0;
    {
        std::lock_guard<std::mutex> lk(s->m);
        auto it = s->scenes.find(scene_id);
        if (it == s->scenes.end()) return WS_ERR_INVALID_ARGUMENT;
        if (it->second.pending > 0) return WS_ERR_NOT_READY;
        src = it->second.warp;
        n = (size_t)it->second.in.num_nodes;
    }
    cudaSetDevice(s->cfg.device);
    if (cudaMemcpyAsync(dev_out, src, 32 * n, cudaMemcpyDeviceToDevice, s->control) != cudaSuccess ||
        cudaStreamSynchronize(s->control) != cudaSuccess)
        return WS_ERR_CUDA;
    return WS_OK;
}

int ws_server_set_warp(ws_server *s, int scene_id, const float *dev_dq) {
    if (!s || !dev_dq) return WS_ERR_INVALID_ARGUMENT;
    float *dst = nullptr;
    size_t n = 0;
    {
        std::lock_guard<std::mutex> lk(s->m);
        auto it = s->scenes.find(scene_id);
        if (it == s->scenes.end()) return WS_ERR_INVALID_ARGUMENT;
        if (it->second.pending > 0) return WS_ERR_NOT_READY;
        dst = it->second.warp;
        n = (size_t)it->second.in.num_nodes;
    }
    cudaSetDevice(s->cfg.device);
    if (cudaMemcpyAsync(dst, dev_dq, 32 * n, cudaMemcpyDeviceToDevice, s->control) != cudaSuccess ||
        cudaStreamSynchronize(s->control) != cudaSuccess)
        return WS_ERR_CUDA;
    return WS_OK;
}

int ws_server_get_stats(ws_server *s, ws_server_stats *st) {
    if (!s || !st) return WS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->m);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->batches = s->batches;
    st->mean_batch_scenes = s->batches ? (double)s->batch_scene_sum / (double)s->batches : 0.0;
    st->p50_latency_ms = st->p99_latency_ms = st->mean_latency_ms = 0.0;
    if (!s->latencies.empty()) {
        std::vector<double> v = s->latencies;
        auto pct = [&](double q) {
            const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return v[k];
        };
        st->p50_latency_ms = pct(0.50);
        st->p99_latency_ms = pct(0.99);
        double sum = 0.0;
        for (double x : s->latencies) sum += x;
        st->mean_latency_ms = sum / (double)s->latencies.size();
    }
    st->executor_bytes = s->exec_bytes;
    st->resident_bytes = s->resident_bytes;
    st->memory_budget = s->cfg.memory_budget;
    st->scenes = (int)s->scenes.size();
    return WS_OK;
}

}  // extern "C"
