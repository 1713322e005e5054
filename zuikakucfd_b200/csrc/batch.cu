// Batched runner (zk_batch_*): many independent WENO / DG problems of uneven
// sizes advanced together on one GPU.
//
// Per group (problems sharing method, precision, order) and per RK step the
// device runs, with no host round trip:
//   max wave speed of every running problem (one persistent launch)
//   -> per-problem dt from its CFL rule (control kernel)
//   -> stage 1, 2, 3 (one persistent launch each; two for FP64 DG)
//   -> step count, completion time, failure check (control kernel).
// Each group is an independent chain; graph_steps steps of all chains are
// captured once into a CUDA graph whose branches run concurrently, and the
// graph is replayed until every problem has its step count.  The kernels find
// their tiles through device-side directories that the host rewrites between
// replays, so admission changes never re-capture the graph.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "batch.cuh"
#include "dg_common.cuh"
#include "zk_internal.h"
#include "zuikaku.h"

namespace zk {
cudaError_t launch_weno_stage_fp64_batch(int variant, const WenoItem* items, const int* dir, int cap, int stage,
                                         int grid, cudaStream_t s);
int weno_fp64_batch_occupancy(int variant);
cudaError_t launch_weno_stage_mixed_batch(int variant, const WenoItem* items, const int* dir, int cap, int stage,
                                          int grid, cudaStream_t s);
int weno_mixed_batch_occupancy(int variant);
bool encode_weno_state_map(CUtensorMap* m, const double* base, const Grid& g, const char** err, int rows);
cudaError_t launch_dg_stage_fp64_batch(int P, const DgItem* items, const int* dir_face, const int* dir_cell, int cap,
                                       int stage, int grid_face, int grid_cell, cudaStream_t s);
int dg_fp64_batch_occupancy(int P, int pass);
int dg_fp64_batch_tiles(int pass, int ny, int nx);
cudaError_t launch_dg_stage_mixed_batch(int P, int variant, int stage, const DgItem* items, const int* dir, int cap,
                                        int grid, cudaStream_t s);
int dg_mixed_batch_occupancy(int P, int variant, int stage);
int dg_mixed_batch_tiles(int variant, int ny, int nx);
int dg_upload_tables_f32(int P);
int batch_red_tiles(int ny, int nx);
cudaError_t launch_batch_max_speed(int method, const void* items, const int* dir, int cap, int grid, cudaStream_t s);
cudaError_t launch_batch_ctl(int post, BatchCtl* ctl, const int* members, int n, const int* admitted,
                             cudaStream_t s);
cudaError_t launch_batch_clock(unsigned long long* t, cudaStream_t s);
}  // namespace zk

using namespace zk;

namespace {

int bfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return zk_internal_fail(code, buf);
}

#define BK_CUDA(call)                                                                                 \
    do {                                                                                              \
        cudaError_t _e = (call);                                                                      \
        if (_e != cudaSuccess)                                                                        \
            return bfail(ZK_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

constexpr int kRedCtasPerSm = 4;

struct BProblem {
    zk_options opt{};
    int ny = 0, nx = 0, nm = 1, nsteps = 0;
    double da = 0.0, gamma = 0.0, cfl = 0.0;
    Grid g{};
    double* U[3] = {nullptr, nullptr, nullptr};
    float* F[2] = {nullptr, nullptr};
    double* fx = nullptr;
    double* fy = nullptr;
    int xpitch = 0;
    int8_t* kind = nullptr;
    int32_t* gsrc = nullptr;
    double* phic = nullptr;
    double s0 = 0.0;
    size_t updated = 0;  // updated (bctype 0, interior) cells
    int group = -1, slot = -1;
    double cost = 0.0;   // algorithmic flops of the whole run (scheduling order)
};

// Directory tilings of a group.
enum { DIR_STAGE = 0, DIR_RED = 1, DIR_CELL = 2, NDIR = 3 };

struct BGroup {
    int method = 0, precision = 0, order = 0;
    std::vector<int> members;  // problem ids, slot order
    void* d_items = nullptr;
    int* d_members = nullptr;
    int* d_dir[NDIR] = {nullptr, nullptr, nullptr};
    int cap = 0;
    int variant = 1;    // tile variant of the stage kernel (batch.cuh)
    int ctas = 0;       // CTAs per SM of the stage kernel
    int ctas_cell = 0;  // FP64 DG cell pass
    double tune_ms = 0.0;
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;
    bool dg() const { return method == ZK_METHOD_DG; }
    bool mixed() const { return precision == ZK_PREC_MIXED; }
};

// Autotuning results per process: (device, method, precision, order) ->
// (variant, CTAs per SM).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, std::pair<int, int>> g_tune;

}  // namespace

struct zk_batch {
    zk_batch_options opt{};
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr;
    std::vector<BProblem> probs;
    std::vector<BGroup> groups;
    BatchCtl* d_ctl = nullptr;
    int* d_admitted = nullptr;
    double* d_dtlog = nullptr;
    unsigned long long* d_t0 = nullptr;
    std::vector<BatchCtl> ctl0;  // initial control blocks
    std::vector<BatchCtl> ctl;   // last copy read back
    std::vector<int> admitted;
    unsigned long long t0 = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long launches_per_graph = 0;
    bool finalized = false, ran = false;
    char* arena = nullptr;
    size_t arena_used = 0;
    std::vector<void*> allocs;
};

namespace {

int balloc(zk_batch* b, void** p, size_t bytes) {
    bytes = (bytes + 255) / 256 * 256;
    if (b->arena && b->arena_used + bytes <= b->opt.arena_bytes) {
        *p = b->arena + b->arena_used;
        b->arena_used += bytes;
        return ZK_OK;
    }
    BK_CUDA(cudaMalloc(p, bytes));
    b->allocs.push_back(*p);
    return ZK_OK;
}

template <typename T>
int balloc_t(zk_batch* b, T** p, size_t count) {
    void* v = nullptr;
    int rc = balloc(b, &v, sizeof(T) * count);
    *p = static_cast<T*>(v);
    return rc;
}

// Tiles of problem p in tiling d of its group (tile variant v).
int tiles_of(const BGroup& g, const BProblem& p, int d, int v) {
    if (d == DIR_RED) return batch_red_tiles(p.ny, p.nx);
    if (!g.dg()) return ((p.nx + 31) / 32) * ((p.ny + weno_variant_rows(v) - 1) / weno_variant_rows(v));
    if (g.mixed()) return dg_mixed_batch_tiles(v, p.ny, p.nx);
    return dg_fp64_batch_tiles(d == DIR_STAGE ? 0 : 1, p.ny, p.nx);
}

// Write group g's directories for the listed slots.
int upload_dirs(zk_batch* b, BGroup& g, const std::vector<int>& slots) {
    const int cap = g.cap;
    std::vector<int> h(2 + 2 * (size_t)cap, 0);
    for (int d = 0; d < NDIR; ++d) {
        if (!g.d_dir[d]) continue;
        std::fill(h.begin(), h.end(), 0);
        long long total = 0;
        for (size_t s = 0; s < slots.size(); ++s) {
            total += tiles_of(g, b->probs[g.members[slots[s]]], d, g.variant);
            if (total > INT32_MAX) return bfail(ZK_ERR_ARG, "batch group too large for 32-bit tile indices");
            h[2 + s] = slots[s];
            h[2 + cap + s] = (int)total;
        }
        h[0] = (int)slots.size();
        h[1] = (int)total;
        BK_CUDA(cudaMemcpyAsync(g.d_dir[d], h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, b->stream));
    }
    return ZK_OK;
}

int occupancy(const BGroup& g, int v) {
    if (!g.dg()) return g.mixed() ? weno_mixed_batch_occupancy(v) : weno_fp64_batch_occupancy(v);
    if (g.mixed()) {
        int n = 1 << 30;
        for (int s = 1; s <= 3; ++s) n = std::min(n, dg_mixed_batch_occupancy(g.order, v, s));
        return n;
    }
    return dg_fp64_batch_occupancy(g.order, 0);
}

// Enqueue stage `stage` of group g with ctas CTAs per SM.
cudaError_t launch_stage(zk_batch* b, BGroup& g, int stage, int variant, int ctas, cudaStream_t s) {
    const int grid = std::max(1, ctas) * b->sms;
    if (!g.dg()) {
        const WenoItem* it = static_cast<const WenoItem*>(g.d_items);
        return g.mixed() ? launch_weno_stage_mixed_batch(variant, it, g.d_dir[DIR_STAGE], g.cap, stage, grid, s)
                         : launch_weno_stage_fp64_batch(variant, it, g.d_dir[DIR_STAGE], g.cap, stage, grid, s);
    }
    const DgItem* it = static_cast<const DgItem*>(g.d_items);
    if (g.mixed()) return launch_dg_stage_mixed_batch(g.order, variant, stage, it, g.d_dir[DIR_STAGE], g.cap, grid, s);
    const int grid_cell = std::max(1, g.ctas_cell) * b->sms;
    return launch_dg_stage_fp64_batch(g.order, it, g.d_dir[DIR_STAGE], g.d_dir[DIR_CELL], g.cap, stage, grid, grid_cell,
                                      s);
}

// One RK step of group g on stream s; returns kernels launched, or -1.
int enqueue_group_step(zk_batch* b, BGroup& g, cudaStream_t s) {
    int n = 0;
    if (launch_batch_max_speed(g.method, g.d_items, g.d_dir[DIR_RED], g.cap, kRedCtasPerSm * b->sms, s) != cudaSuccess)
        return -1;
    if (launch_batch_ctl(0, b->d_ctl, g.d_members, (int)g.members.size(), b->d_admitted, s) != cudaSuccess) return -1;
    n += 2;
    for (int st = 1; st <= 3; ++st) {
        if (launch_stage(b, g, st, g.variant, g.ctas, s) != cudaSuccess) return -1;
        n += (g.dg() && !g.mixed()) ? 2 : 1;
    }
    if (launch_batch_ctl(1, b->d_ctl, g.d_members, (int)g.members.size(), nullptr, s) != cudaSuccess) return -1;
    return n + 1;
}

// Algorithmic flops per updated cell and RK stage (scheduling weights).
double stage_flops(const zk_options& o) {
    if (o.method != ZK_METHOD_DG) return 1330.0;
    return o.order == 1 ? 1700.0 : o.order == 2 ? 5300.0 : 13200.0;
}

// Time the tile variants x persistent grid sizes of group g's stage-1 kernel
// on a sample of its problems (up to 8M updated cells); keep the fastest.  A
// pinned variant is timed alone and its result is not cached.
int autotune(zk_batch* b, BGroup& g) {
    int dev = 0;
    BK_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, g.method, g.precision, g.order);
    const bool pinned = g.dg() ? (g.mixed() && b->opt.dg_variant >= 0) : b->opt.weno_variant >= 0;
    if (b->opt.autotune == 1 && !pinned) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            g.variant = it->second.first;
            g.ctas = it->second.second;
            if (g.dg() && !g.mixed()) g.ctas_cell = std::min(g.ctas, dg_fp64_batch_occupancy(g.order, 1));
            return ZK_OK;
        }
    }
    std::vector<int> sample;
    double cells = 0.0;
    for (size_t s = 0; s < g.members.size() && (sample.empty() || cells < 8e6); ++s) {
        sample.push_back((int)s);
        cells += (double)b->probs[g.members[s]].updated;
    }
    std::vector<int> adm(b->probs.size(), 0);
    for (int s : sample) adm[g.members[s]] = 1;
    BK_CUDA(cudaMemcpyAsync(b->d_admitted, adm.data(), sizeof(int) * adm.size(), cudaMemcpyHostToDevice, b->stream));
    const bool fp64dg = g.dg() && !g.mixed();
    const int nvar = (fp64dg || pinned) ? 1 : g.dg() ? kDgVariants : kWenoVariants;
    float best = 3.0e38f;
    int best_v = g.variant, best_c = g.ctas;
    for (int v = 0; v < nvar; ++v) {
        const int var = (fp64dg || pinned) ? g.variant : v;
        const int keep = g.variant;
        g.variant = var;
        const int rc = upload_dirs(b, g, sample);
        g.variant = keep;
        if (rc) return rc;
        BK_CUDA(launch_batch_max_speed(g.method, g.d_items, g.d_dir[DIR_RED], g.cap, kRedCtasPerSm * b->sms, b->stream));
        BK_CUDA(launch_batch_ctl(0, b->d_ctl, g.d_members, (int)g.members.size(), b->d_admitted, b->stream));
        int occ = occupancy(g, var);
        if (fp64dg) occ = std::min(occ, dg_fp64_batch_occupancy(g.order, 1));
        for (int c = 1; c <= occ; ++c) {
            if (fp64dg) g.ctas_cell = c;
            BK_CUDA(launch_stage(b, g, 1, var, c, b->stream));  // warm-up
            BK_CUDA(cudaEventRecord(b->ev0, b->stream));
            for (int r = 0; r < 3; ++r) BK_CUDA(launch_stage(b, g, 1, var, c, b->stream));
            BK_CUDA(cudaEventRecord(b->ev1, b->stream));
            BK_CUDA(cudaEventSynchronize(b->ev1));
            float ms = 0.0f;
            BK_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
            if (ms < best) {
                best = ms;
                best_v = var;
                best_c = c;
            }
        }
    }
    g.variant = best_v;
    g.ctas = best_c;
    if (fp64dg) g.ctas_cell = best_c;
    g.tune_ms = best / 3.0;
    // undo the sample's control-block changes
    BK_CUDA(cudaMemcpyAsync(b->d_ctl, b->ctl0.data(), sizeof(BatchCtl) * b->ctl0.size(), cudaMemcpyHostToDevice,
                            b->stream));
    BK_CUDA(cudaMemsetAsync(b->d_admitted, 0, sizeof(int) * b->probs.size(), b->stream));
    BK_CUDA(cudaStreamSynchronize(b->stream));
    if (pinned) return ZK_OK;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = {g.variant, g.ctas};
    return ZK_OK;
}

// Capture graph_steps steps of every group (one branch per group).
int capture(zk_batch* b) {
    BK_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    long long n = 0;
    bool ok = cudaEventRecord(b->fork, b->stream) == cudaSuccess;
    for (BGroup& g : b->groups) {
        ok = ok && cudaStreamWaitEvent(g.stream, b->fork, 0) == cudaSuccess;
        for (int s = 0; ok && s < b->opt.graph_steps; ++s) {
            const int k = enqueue_group_step(b, g, g.stream);
            ok = k >= 0;
            n += k;
        }
        ok = ok && cudaEventRecord(g.join, g.stream) == cudaSuccess;
        ok = ok && cudaStreamWaitEvent(b->stream, g.join, 0) == cudaSuccess;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (!ok || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        const cudaError_t last = cudaGetLastError();
        return bfail(ZK_ERR_CUDA, "batch graph capture failed: %s",
                     cudaGetErrorString(e != cudaSuccess ? e : last));
    }
    b->graph = graph;
    BK_CUDA(cudaGraphInstantiate(&b->exec, graph, 0));
    b->launches_per_graph = n;
    return ZK_OK;
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return -1.0;
    std::sort(v.begin(), v.end());
    size_t r = (size_t)std::ceil(q / 100.0 * (double)v.size());
    r = std::min(std::max<size_t>(r, 1), v.size());
    return v[r - 1];
}

// Group the problems, build items, control blocks and directories, tune and
// capture.  Runs once, at the first zk_batch_run.
int finalize(zk_batch* b) {
    if (b->probs.empty()) return bfail(ZK_ERR_STATE, "batch has no problems");
    std::map<std::tuple<int, int, int>, int> index;
    for (size_t i = 0; i < b->probs.size(); ++i) {
        BProblem& p = b->probs[i];
        const auto key = std::make_tuple(p.opt.method, p.opt.precision, p.opt.method == ZK_METHOD_DG ? p.opt.order : 0);
        auto it = index.find(key);
        if (it == index.end()) {
            it = index.emplace(key, (int)b->groups.size()).first;
            BGroup g;
            g.method = p.opt.method;
            g.precision = p.opt.precision;
            g.order = std::get<2>(key);
            b->groups.push_back(g);
        }
        BGroup& g = b->groups[it->second];
        p.group = it->second;
        p.slot = (int)g.members.size();
        g.members.push_back((int)i);
    }
    // control blocks and dt logs
    size_t total_steps = 0;
    for (const BProblem& p : b->probs) total_steps += (size_t)p.nsteps;
    if (int rc = balloc_t(b, &b->d_dtlog, total_steps)) return rc;
    if (int rc = balloc_t(b, &b->d_ctl, b->probs.size())) return rc;
    if (int rc = balloc_t(b, &b->d_admitted, b->probs.size())) return rc;
    if (int rc = balloc_t(b, &b->d_t0, 1)) return rc;
    b->ctl0.assign(b->probs.size(), BatchCtl{});
    size_t off = 0;
    for (size_t i = 0; i < b->probs.size(); ++i) {
        const BProblem& p = b->probs[i];
        BatchCtl& c = b->ctl0[i];
        std::memset(&c, 0, sizeof c);
        c.cfl = p.cfl;
        c.da = p.da;
        c.dtlog = b->d_dtlog + off;
        off += (size_t)p.nsteps;
        c.steps_target = p.nsteps;
        c.state = BATCH_WAITING;
        c.method = p.opt.method;
        c.order = p.opt.order;
    }
    b->ctl = b->ctl0;
    BK_CUDA(cudaMemcpyAsync(b->d_ctl, b->ctl0.data(), sizeof(BatchCtl) * b->ctl0.size(), cudaMemcpyHostToDevice,
                            b->stream));
    BK_CUDA(cudaMemsetAsync(b->d_admitted, 0, sizeof(int) * b->probs.size(), b->stream));
    // per-group items, members, directories
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        BGroup& g = b->groups[gi];
        BK_CUDA(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        BK_CUDA(cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming));
        g.cap = (int)g.members.size();
        if (int rc = balloc_t(b, &g.d_members, g.members.size())) return rc;
        BK_CUDA(cudaMemcpyAsync(g.d_members, g.members.data(), sizeof(int) * g.members.size(), cudaMemcpyHostToDevice,
                                b->stream));
        for (int d = 0; d < NDIR; ++d) {
            if (d == DIR_CELL && !(g.dg() && !g.mixed())) continue;
            if (int rc = balloc_t(b, &g.d_dir[d], 2 + 2 * (size_t)g.cap)) return rc;
            BK_CUDA(cudaMemsetAsync(g.d_dir[d], 0, sizeof(int) * (2 + 2 * (size_t)g.cap), b->stream));
        }
        if (!g.dg()) {
            std::vector<WenoItem> items(g.members.size());
            for (size_t s = 0; s < g.members.size(); ++s) {
                const int id = g.members[s];
                BProblem& p = b->probs[id];
                WenoItem& it = items[s];
                std::memset(&it, 0, sizeof it);
                for (int k = 0; k < 3; ++k) it.U[k] = p.U[k];
                it.kind = p.kind;
                it.gsrc = p.gsrc;
                it.ctl = b->d_ctl + id;
                it.g = p.g;
                it.gamma = p.gamma;
                if (g.mixed())
                    for (int v = 0; v < 2; ++v)
                        for (int k = 0; k < 3; ++k) {
                            const char* err = nullptr;
                            if (!encode_weno_state_map(&it.tmap[v][k], p.U[k], p.g, &err, kWenoTileRows[v]))
                                return bfail(ZK_ERR_CUDA, "tensor map of problem %d: %s", id, err);
                        }
            }
            if (int rc = balloc(b, &g.d_items, sizeof(WenoItem) * items.size())) return rc;
            BK_CUDA(cudaMemcpyAsync(g.d_items, items.data(), sizeof(WenoItem) * items.size(), cudaMemcpyHostToDevice,
                                    b->stream));
            BK_CUDA(cudaStreamSynchronize(b->stream));  // items is a pageable local
        } else {
            std::vector<DgItem> items(g.members.size());
            for (size_t s = 0; s < g.members.size(); ++s) {
                const int id = g.members[s];
                BProblem& p = b->probs[id];
                DgItem& it = items[s];
                std::memset(&it, 0, sizeof it);
                for (int k = 0; k < 3; ++k) it.U[k] = p.U[k];
                it.F[0] = p.F[0];
                it.F[1] = p.F[1];
                it.fx = p.fx;
                it.fy = p.fy;
                it.kind = p.kind;
                it.gsrc = p.gsrc;
                it.phic = p.phic;
                it.ctl = b->d_ctl + id;
                it.g = p.g;
                it.xpitch = p.xpitch;
                it.nm = p.nm;
                it.inv2h = 0.5 / p.da;
                it.gamma = p.gamma;
                it.s0 = p.s0;
                it.limiter = p.opt.limiter;
                it.hll = p.opt.flux == ZK_FLUX_HLL;
            }
            if (int rc = balloc(b, &g.d_items, sizeof(DgItem) * items.size())) return rc;
            BK_CUDA(cudaMemcpyAsync(g.d_items, items.data(), sizeof(DgItem) * items.size(), cudaMemcpyHostToDevice,
                                    b->stream));
            BK_CUDA(cudaStreamSynchronize(b->stream));
        }
        if (!g.dg()) g.variant = b->opt.weno_variant >= 0 ? b->opt.weno_variant : kWenoDefaultVariant;
        else g.variant = (g.mixed() && b->opt.dg_variant >= 0) ? b->opt.dg_variant : kDgDefaultVariant;
        g.ctas = occupancy(g, g.variant);
        if (g.dg() && !g.mixed()) g.ctas_cell = dg_fp64_batch_occupancy(g.order, 1);
        if (g.ctas <= 0) return bfail(ZK_ERR_CUDA, "stage kernel of group %d cannot be resident", (int)gi);
    }
    BK_CUDA(cudaStreamSynchronize(b->stream));
    if (b->opt.autotune)
        for (BGroup& g : b->groups)
            if (int rc = autotune(b, g)) return rc;
    if (int rc = capture(b)) return rc;
    b->finalized = true;
    return ZK_OK;
}

}  // namespace

extern "C" {

void zk_batch_default_options(zk_batch_options* o) {
    if (!o) return;
    o->device = 0;
    o->policy = ZK_BATCH_ALL;
    o->active_cells = 8e6;
    o->graph_steps = 10;
    o->autotune = 1;
    o->arena_bytes = 0;
    o->weno_variant = -1;
    o->dg_variant = -1;
}

int zk_batch_create(const zk_batch_options* o, zk_batch** out) {
    if (!o || !out) return bfail(ZK_ERR_ARG, "null argument");
    *out = nullptr;
    if (o->policy != ZK_BATCH_ALL && o->policy != ZK_BATCH_SJF) return bfail(ZK_ERR_ARG, "unknown policy %d", o->policy);
    if (o->graph_steps < 1 || o->graph_steps > 1000) return bfail(ZK_ERR_ARG, "graph_steps must be 1..1000");
    if (o->autotune < 0 || o->autotune > 2) return bfail(ZK_ERR_ARG, "autotune must be 0, 1 or 2");
    if (o->weno_variant < -1 || o->weno_variant >= kWenoVariants)
        return bfail(ZK_ERR_ARG, "weno_variant must be -1 or 0..%d", kWenoVariants - 1);
    if (o->dg_variant < -1 || o->dg_variant >= kDgVariants)
        return bfail(ZK_ERR_ARG, "dg_variant must be -1 or 0..%d", kDgVariants - 1);
    BK_CUDA(cudaSetDevice(o->device));
    zk_batch* b = new zk_batch();
    b->opt = *o;
    if (!(b->opt.active_cells > 0.0)) b->opt.active_cells = 8e6;
    int rc = ZK_OK;
    auto cu = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == ZK_OK) rc = bfail(ZK_ERR_CUDA, "batch setup: %s", cudaGetErrorString(e));
    };
    cu(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, o->device));
    cu(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    cu(cudaEventCreate(&b->ev0));
    cu(cudaEventCreate(&b->ev1));
    cu(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    if (rc == ZK_OK && o->arena_bytes > 0) cu(cudaMalloc(reinterpret_cast<void**>(&b->arena), o->arena_bytes));
    if (rc != ZK_OK) {
        zk_batch_destroy(b);
        return rc;
    }
    *out = b;
    return ZK_OK;
}

int zk_batch_add(zk_batch* b, const zk_options* o, int ny, int nx, double da, double gamma, const int32_t* bct,
                 const double* state, int nsteps, double cfl, int* id) {
    if (!b || !o || !bct || !state || !id) return bfail(ZK_ERR_ARG, "null argument");
    if (b->finalized || b->ran) return bfail(ZK_ERR_STATE, "zk_batch_add after zk_batch_run");
    if (o->method != ZK_METHOD_WENO && o->method != ZK_METHOD_DG) return bfail(ZK_ERR_ARG, "unknown method %d", o->method);
    if (o->method == ZK_METHOD_DG && (o->order < 1 || o->order > 3))
        return bfail(ZK_ERR_ARG, "DG order must be 1..3, got %d", o->order);
    if (o->precision != ZK_PREC_FP64 && o->precision != ZK_PREC_MIXED)
        return bfail(ZK_ERR_ARG, "unknown precision %d", o->precision);
    if (o->recon != ZK_RECON_WENO5) return bfail(ZK_ERR_UNSUPPORTED, "the batched runner reconstructs with WENO5 only");
    if (o->limiter < ZK_LIMITER_REFERENCE || o->limiter > ZK_LIMITER_TVB_MLP)
        return bfail(ZK_ERR_ARG, "unknown limiter %d", o->limiter);
    if (o->method == ZK_METHOD_DG && o->limiter >= ZK_LIMITER_TVB)
        return bfail(ZK_ERR_UNSUPPORTED, "batched DG problems take the REFERENCE or NONE limiter");
    if (o->flux != ZK_FLUX_HLLC && o->flux != ZK_FLUX_HLL) return bfail(ZK_ERR_ARG, "unknown flux %d", o->flux);
    if (o->boundary != ZK_BOUNDARY_EXCHANGE && o->boundary != ZK_BOUNDARY_PERIODIC)
        return bfail(ZK_ERR_ARG, "unknown boundary %d", o->boundary);
    if (o->device != b->opt.device) return bfail(ZK_ERR_ARG, "problem device differs from the batch device");
    if (ny < 7 || nx < 7) return bfail(ZK_ERR_ARG, "grid %dx%d too small (needs >= 7x7)", ny, nx);
    if ((size_t)ny * (size_t)round_pitch(nx) >= (size_t)INT32_MAX)
        return bfail(ZK_ERR_ARG, "grid %dx%d too large for 32-bit cell indices", ny, nx);
    if (!(da > 0.0) || !(gamma > 1.0)) return bfail(ZK_ERR_ARG, "need da > 0 and gamma > 1");
    if (nsteps < 1) return bfail(ZK_ERR_ARG, "nsteps must be >= 1");
    if (!(cfl > 0.0) || !std::isfinite(cfl)) return bfail(ZK_ERR_ARG, "cfl must be finite and > 0");
    const bool periodic = o->boundary == ZK_BOUNDARY_PERIODIC;
    if (periodic)
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                const bool ring = i < 3 || i >= ny - 3 || j < 3 || j >= nx - 3;
                if (ring && bct[(size_t)i * nx + j] != -3)
                    return bfail(ZK_ERR_ARG, "periodic boundary needs the 3-wide ring marked -3");
            }
    BK_CUDA(cudaSetDevice(b->opt.device));
    BProblem p;
    p.opt = *o;
    p.ny = ny;
    p.nx = nx;
    p.da = da;
    p.gamma = gamma;
    p.nsteps = nsteps;
    p.cfl = cfl;
    p.g.ny = ny;
    p.g.nx = nx;
    p.g.pitch = round_pitch(nx);
    p.g.plane = (size_t)ny * p.g.pitch;
    const bool dg = o->method == ZK_METHOD_DG, mixed = o->precision == ZK_PREC_MIXED;
    const int P = o->order, NQ = P + 1;
    p.nm = dg ? NQ * NQ : 1;
    std::vector<int8_t> kind;
    std::vector<int32_t> src;
    build_ghost_map(ny, nx, p.g.pitch, bct, dg, periodic, kind, src);
    for (int8_t k : kind) p.updated += (k & KIND_MASK) == KIND_UPDATED;
    p.cost = (double)p.updated * stage_flops(*o) * nsteps;
    const size_t nvar = 4 * (size_t)p.nm, bytes = sizeof(double) * nvar * p.g.plane;
    cudaStream_t s = b->stream;
    if (int rc = balloc_t(b, &p.kind, kind.size())) return rc;
    if (int rc = balloc_t(b, &p.gsrc, src.size())) return rc;
    BK_CUDA(cudaMemcpyAsync(p.kind, kind.data(), kind.size(), cudaMemcpyHostToDevice, s));
    BK_CUDA(cudaMemcpyAsync(p.gsrc, src.data(), src.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    if (int rc = balloc(b, reinterpret_cast<void**>(&p.U[0]), bytes)) return rc;
    BK_CUDA(cudaMemsetAsync(p.U[0], 0, bytes, s));
    BK_CUDA(cudaMemcpy2DAsync(p.U[0], sizeof(double) * p.g.pitch, state, sizeof(double) * nx, sizeof(double) * nx,
                              nvar * ny, cudaMemcpyHostToDevice, s));
    if (!(dg && mixed))
        for (int k = 1; k < 3; ++k) {
            if (int rc = balloc(b, reinterpret_cast<void**>(&p.U[k]), bytes)) return rc;
            BK_CUDA(cudaMemsetAsync(p.U[k], 0, bytes, s));
        }
    if (dg) {
        DGTab tab;
        double phic[DG_MAXNM * 4];
        dg_make_tables(P, &tab, phic);
        if (dg_upload_tables(P, tab) != ZK_OK) return bfail(ZK_ERR_CUDA, "DG table upload failed");
        if (mixed && dg_upload_tables_f32(P) != ZK_OK) return bfail(ZK_ERR_CUDA, "DG FP32 table upload failed");
        p.s0 = (P >= 3) ? -3.0 * std::log10((double)P) : -4.0 * std::log10((double)P);
        if (int rc = balloc_t(b, &p.phic, (size_t)p.nm * 4)) return rc;
        BK_CUDA(cudaMemcpyAsync(p.phic, phic, sizeof(double) * p.nm * 4, cudaMemcpyHostToDevice, s));
        if (mixed) {
            for (int k = 0; k < 2; ++k) {
                if (int rc = balloc_t(b, &p.F[k], nvar * p.g.plane)) return rc;
                BK_CUDA(cudaMemsetAsync(p.F[k], 0, sizeof(float) * nvar * p.g.plane, s));
            }
        } else {
            p.xpitch = p.g.pitch + 32;
            if (int rc = balloc_t(b, &p.fx, (size_t)NQ * 4 * ny * p.xpitch)) return rc;
            if (int rc = balloc_t(b, &p.fy, (size_t)NQ * 4 * (ny + 1) * p.g.pitch)) return rc;
        }
        BK_CUDA(cudaStreamSynchronize(s));  // phic is a stack array
    }
    BK_CUDA(cudaStreamSynchronize(s));
    *id = (int)b->probs.size();
    b->probs.push_back(p);
    return ZK_OK;
}

int zk_batch_run(zk_batch* b, zk_batch_report* r) {
    if (!b) return bfail(ZK_ERR_ARG, "null batch");
    if (b->ran) return bfail(ZK_ERR_STATE, "zk_batch_run already ran on this batch");
    BK_CUDA(cudaSetDevice(b->opt.device));
    if (!b->finalized)
        if (int rc = finalize(b)) return rc;
    b->ran = true;
    const int n = (int)b->probs.size(), G = b->opt.graph_steps;
    const bool sjf = b->opt.policy == ZK_BATCH_SJF;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    if (sjf)
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int c) { return b->probs[a].cost < b->probs[c].cost; });
    std::vector<std::vector<int>> slots(b->groups.size());
    std::vector<char> retired(n, 0);
    b->admitted.assign(n, 0);
    size_t next = 0;
    double active = 0.0;
    int running = 0;
    auto admit = [&]() {
        bool changed = false;
        while (next < order.size() && (!sjf || running == 0 || active < b->opt.active_cells)) {
            const int id = order[next++];
            const BProblem& p = b->probs[id];
            b->admitted[id] = 1;
            active += (double)p.updated;
            ++running;
            slots[p.group].push_back(p.slot);
            changed = true;
        }
        return changed;
    };
    auto upload = [&]() -> int {
        BK_CUDA(cudaMemcpyAsync(b->d_admitted, b->admitted.data(), sizeof(int) * n, cudaMemcpyHostToDevice, b->stream));
        for (size_t gi = 0; gi < b->groups.size(); ++gi)
            if (int rc = upload_dirs(b, b->groups[gi], slots[gi])) return rc;
        return ZK_OK;
    };
    admit();
    if (int rc = upload()) return rc;
    BK_CUDA(launch_batch_clock(b->d_t0, b->stream));
    BK_CUDA(cudaEventRecord(b->ev0, b->stream));
    int max_steps = 0;
    long long sum_steps = 0;
    for (const BProblem& p : b->probs) {
        max_steps = std::max(max_steps, p.nsteps);
        sum_steps += p.nsteps;
    }
    int launches = 0;
    if (!sjf) {
        const int ng = (max_steps + G - 1) / G;
        for (; launches < ng; ++launches) BK_CUDA(cudaGraphLaunch(b->exec, b->stream));
    } else {
        // every replay advances each running problem by G steps, so this bounds the loop
        const long long bound = sum_steps / G + 2LL * n + 2;
        int finished = 0;
        while (finished < n) {
            if (launches >= bound) return bfail(ZK_ERR_STATE, "batch scheduler did not converge");
            BK_CUDA(cudaGraphLaunch(b->exec, b->stream));
            ++launches;
            BK_CUDA(cudaMemcpyAsync(b->ctl.data(), b->d_ctl, sizeof(BatchCtl) * n, cudaMemcpyDeviceToHost, b->stream));
            BK_CUDA(cudaStreamSynchronize(b->stream));
            bool removed = false;
            for (int id = 0; id < n; ++id) {
                if (!b->admitted[id] || retired[id] || b->ctl[id].state < BATCH_DONE) continue;
                retired[id] = 1;
                ++finished;
                --running;
                active -= (double)b->probs[id].updated;
                auto& sl = slots[b->probs[id].group];
                sl.erase(std::find(sl.begin(), sl.end(), b->probs[id].slot));
                removed = true;
            }
            if (finished >= n) break;
            if (admit() || removed)
                if (int rc = upload()) return rc;
        }
    }
    BK_CUDA(cudaEventRecord(b->ev1, b->stream));
    BK_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0.0f;
    BK_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    BK_CUDA(cudaMemcpyAsync(b->ctl.data(), b->d_ctl, sizeof(BatchCtl) * n, cudaMemcpyDeviceToHost, b->stream));
    BK_CUDA(cudaMemcpyAsync(&b->t0, b->d_t0, sizeof b->t0, cudaMemcpyDeviceToHost, b->stream));
    BK_CUDA(cudaStreamSynchronize(b->stream));
    if (r) {
        std::memset(r, 0, sizeof *r);
        std::vector<double> lat;
        for (int id = 0; id < n; ++id) {
            const BatchCtl& c = b->ctl[id];
            const BProblem& p = b->probs[id];
            r->cell_updates += (double)p.updated * c.steps_done;
            r->dof_updates += (double)p.updated * 4.0 * p.nm * c.steps_done;
            if (c.state == BATCH_DONE) ++r->done;
            if (c.state == BATCH_FAILED) ++r->failed;
            if (c.state >= BATCH_DONE && c.t_done >= b->t0) lat.push_back((double)(c.t_done - b->t0) * 1e-6);
        }
        r->ms = ms;
        r->problems = n;
        r->latency_p50_ms = percentile(lat, 50.0);
        r->latency_p99_ms = percentile(lat, 99.0);
        r->latency_max_ms = percentile(lat, 100.0);
        r->graph_launches = launches;
        r->graph_steps = G;
        r->kernel_launches = (long long)launches * b->launches_per_graph + 1;
    }
    return ZK_OK;
}

int zk_batch_get_state(zk_batch* b, int id, double* host) {
    if (!b || !host) return bfail(ZK_ERR_ARG, "null argument");
    if (id < 0 || id >= (int)b->probs.size()) return bfail(ZK_ERR_ARG, "no problem %d", id);
    const BProblem& p = b->probs[id];
    BK_CUDA(cudaSetDevice(b->opt.device));
    BK_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * p.nx, p.U[0], sizeof(double) * p.g.pitch, sizeof(double) * p.nx,
                              (size_t)4 * p.nm * p.ny, cudaMemcpyDeviceToHost, b->stream));
    BK_CUDA(cudaStreamSynchronize(b->stream));
    return ZK_OK;
}

int zk_batch_problem_info(zk_batch* b, int id, zk_batch_problem* out) {
    if (!b || !out) return bfail(ZK_ERR_ARG, "null argument");
    if (id < 0 || id >= (int)b->probs.size()) return bfail(ZK_ERR_ARG, "no problem %d", id);
    std::memset(out, 0, sizeof *out);
    out->group = b->probs[id].group;
    out->latency_ms = -1.0;
    if (!b->ran || b->ctl.size() != b->probs.size()) return ZK_OK;
    const BatchCtl& c = b->ctl[id];
    out->state = c.state;
    out->steps_done = c.steps_done;
    out->t = c.t;
    out->status = c.status;
    if (c.state >= BATCH_DONE && c.t_done >= b->t0) out->latency_ms = (double)(c.t_done - b->t0) * 1e-6;
    return ZK_OK;
}

int zk_batch_dt_history(zk_batch* b, int id, double* dts, int n) {
    if (!b || !dts) return bfail(ZK_ERR_ARG, "null argument");
    if (id < 0 || id >= (int)b->probs.size()) return bfail(ZK_ERR_ARG, "no problem %d", id);
    if (n < 0 || n > b->probs[id].nsteps) return bfail(ZK_ERR_ARG, "n must be 0..%d", b->probs[id].nsteps);
    if (!b->finalized) return bfail(ZK_ERR_STATE, "batch has not run");
    BK_CUDA(cudaSetDevice(b->opt.device));
    BK_CUDA(cudaMemcpyAsync(dts, b->ctl0[id].dtlog, sizeof(double) * n, cudaMemcpyDeviceToHost, b->stream));
    BK_CUDA(cudaStreamSynchronize(b->stream));
    return ZK_OK;
}

int zk_batch_group_config(zk_batch* b, int g, int* method, int* precision, int* order, int* variant,
                          int* ctas_per_sm, int* ngroups) {
    if (!b) return bfail(ZK_ERR_ARG, "null batch");
    if (ngroups) *ngroups = (int)b->groups.size();
    if (g == -1) return ZK_OK;  // count only
    if (g < 0 || g >= (int)b->groups.size()) return bfail(ZK_ERR_ARG, "no group %d (groups form at zk_batch_run)", g);
    const BGroup& G = b->groups[g];
    if (method) *method = G.method;
    if (precision) *precision = G.precision;
    if (order) *order = G.order;
    if (variant) *variant = G.variant;
    if (ctas_per_sm) *ctas_per_sm = G.ctas;
    return ZK_OK;
}

int zk_batch_group_tile(zk_batch* b, int g, int* tile_rows, int* tile_cols, int* threads_per_tile) {
    if (!b) return bfail(ZK_ERR_ARG, "null batch");
    if (g < 0 || g >= (int)b->groups.size()) return bfail(ZK_ERR_ARG, "no group %d (groups form at zk_batch_run)", g);
    const BGroup& G = b->groups[g];
    int rows = 1, cols = 32, threads = 32;
    if (!G.dg()) {
        rows = weno_variant_rows(G.variant);
        threads = 32 * weno_variant_warps(G.variant);
    } else if (G.mixed()) {
        rows = dg_variant_rows(G.variant);
        threads = rows * cols * dg_variant_tpc(G.variant);
    } else {
        cols = kDgCellBlock;  // the FP64 DG cell pass
        threads = cols;
    }
    if (tile_rows) *tile_rows = rows;
    if (tile_cols) *tile_cols = cols;
    if (threads_per_tile) *threads_per_tile = threads;
    return ZK_OK;
}

void zk_batch_destroy(zk_batch* b) {
    if (!b) return;
    cudaSetDevice(b->opt.device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (BGroup& g : b->groups) {
        if (g.stream) cudaStreamDestroy(g.stream);
        if (g.join) cudaEventDestroy(g.join);
    }
    for (void* p : b->allocs) cudaFree(p);
    if (b->arena) cudaFree(b->arena);
    for (cudaEvent_t e : {b->ev0, b->ev1, b->fork})
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"
