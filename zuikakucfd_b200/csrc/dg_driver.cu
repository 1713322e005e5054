// DG driver: buffers, tables and the SSP-RK3 stage sequence of updateMesh
// (src_DG/fluid.cpp:1005-1054) on the device state.
#include <cmath>
#include <cstring>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include <cuda_bf16.h>

#include "dg_common.cuh"
#include "mlp_infer.cuh"
#include "zk_internal.h"
#include "zk_mlp.h"

namespace zk {
cudaError_t launch_dg_stage_fp64(int P, const DGArgs& a, cudaStream_t s);
cudaError_t launch_dg_limit_fp64(int P, const DGArgs& a, cudaStream_t s);
int dg_upload_tables_f32(int P);
cudaError_t launch_dg_tvb(int P, void* state, bool fp64, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                          double da, double gamma, double M, uint8_t* flags, const MlpPacked* mlp,
                          float* features, uint32_t* nflag, float* logits, const void* means, bool means_fp64,
                          float screen, cudaStream_t s);
cudaError_t launch_dg_tvb_list(int P, void* state, bool fp64, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                               double da, double gamma, double M, uint8_t* flags, uint32_t* nflag,
                               const int32_t* list, const uint32_t* count, int grid, cudaStream_t s);
cudaError_t launch_dg_stage_mixed(int P, const void* cur, int in_fp64, const double* un, void* out, int out_fp64,
                                  const int8_t* kind, const int32_t* gsrc, const Grid& g, double dt, double da,
                                  double gamma, int stage, int limiter, int hll, double s0, uint32_t* status,
                                  const FusedIndicator* ind, int tpc, cudaStream_t s);
bool dg_mixed_fuses_indicator(int P);
int dg_mixed_default_tpc(int P);
int dg_upload_sep_f64(int P);
cudaError_t launch_dg_stage_fused_fp64(int P, const double* cur, const double* un, double* out, const int8_t* kind,
                                       const int32_t* gsrc, const Grid& g, double dt, double da, double gamma,
                                       int stage, int limiter, int hll, double s0, uint32_t* status, cudaStream_t s);
}  // namespace zk

namespace zk_fma {  // dg_fp64.cu compiled with fused multiply-adds (ZK_PREC_FP64_FMA)
cudaError_t launch_dg_stage_fp64(int P, const zk::DGArgs& a, cudaStream_t s);
cudaError_t launch_dg_limit_fp64(int P, const zk::DGArgs& a, cudaStream_t s);
int dg_upload_tables(int P, const zk::DGTab& T);
}  // namespace zk_fma

namespace {

// The FP64 stage / reference limiter of a context's precision: the
// reference-arithmetic launches, or with FMA contraction the fused FP64 stage
// kernel (dg_fused_fp64.cu; stages 1-3) and the contracted build of the
// reference-arithmetic kernels (the RHS alone, stage 0).
cudaError_t stage_f64(zk_ctx* c, const zk::DGArgs& a) {
    if (c->fma() && a.stage >= 1)
        return zk::launch_dg_stage_fused_fp64(c->opt.order, a.cur, a.un, a.out, a.kind, a.gsrc, a.g, a.dt, c->da,
                                              a.gamma, a.stage, a.limiter, a.hll, a.s0, a.status, c->stream);
    return c->fma() ? zk_fma::launch_dg_stage_fp64(c->opt.order, a, c->stream)
                    : zk::launch_dg_stage_fp64(c->opt.order, a, c->stream);
}
cudaError_t limit_f64(zk_ctx* c, const zk::DGArgs& a) {
    return c->fma() ? zk_fma::launch_dg_limit_fp64(c->opt.order, a, c->stream)
                    : zk::launch_dg_limit_fp64(c->opt.order, a, c->stream);
}

struct DGState {
    double* fx = nullptr;  // x-face fluxes [NQ][4][ny][xpitch]
    double* fy = nullptr;  // y-face fluxes [NQ][4][ny+1][pitch]
    int xpitch = 0;
    double s0 = 0.0;
};

DGState* st(zk_ctx* c) { return static_cast<DGState*>(c->dg); }

zk::DGArgs args(zk_ctx* c, const double* cur, const double* un, double* out, double dt, int stage) {
    zk::DGArgs a{};
    a.cur = cur;
    a.un = un;
    a.out = out;
    a.kind = c->kind;
    a.gsrc = c->gsrc;
    a.fx = st(c)->fx;
    a.fy = st(c)->fy;
    a.g = c->g;
    a.xpitch = st(c)->xpitch;
    a.dt = dt;
    a.inv2h = 0.5 / c->da;
    a.gamma = c->gamma;
    a.stage = stage;
    a.limiter = c->opt.limiter;
    a.hll = c->opt.flux == ZK_FLUX_HLL;
    a.s0 = st(c)->s0;
    a.status = c->d_status;
    return a;
}

int cuda_fail(cudaError_t e) { return zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e)); }

// The learned indicator runs fused in the stage kernel (mixed precision, an
// order whose single-problem stage has two threads per cell); otherwise a
// TVB_MLP context runs the indicator-gated pass after each stage.
bool fused_indicator(const zk_ctx* c) {
    return c->opt.limiter == ZK_LIMITER_TVB_MLP && c->opt.precision == ZK_PREC_MIXED &&
           zk::dg_mixed_fuses_indicator(c->opt.order);
}

// Output and input buffers of stage `stage` (1..3) of a step: FP64 U^n -> S1
// -> S2 -> U^n; mixed U^n -> F1 -> F2 -> U^n (stage states FP32).
struct StageIO {
    void* out;
    bool out64;
    const void* in;
    bool in64;
};
StageIO stage_io(zk_ctx* c, int stage) {
    if (c->opt.precision == ZK_PREC_MIXED) {
        void* outs[3] = {c->F1, c->F2, c->Un};
        const void* ins[3] = {c->Un, c->F1, c->F2};
        return {outs[stage - 1], stage == 3, ins[stage - 1], stage == 1};
    }
    void* outs[3] = {c->S1, c->S2, c->Un};
    const void* ins[3] = {c->Un, c->S1, c->S2};
    return {outs[stage - 1], true, ins[stage - 1], true};
}

// Mixed stage `stage` (1..3), with the fused indicator when the context runs it.
cudaError_t mixed_stage(zk_ctx* c, double dt, int stage, float* dbg = nullptr) {
    const StageIO io = stage_io(c, stage);
    zk::FusedIndicator ind{c->mlp_frag, c->d_list, c->d_lcount ? c->d_lcount + (stage - 1) : nullptr,
                           (uint32_t)c->g.plane, dbg, c->mlp_screen};
    return zk::launch_dg_stage_mixed(c->opt.order, io.in, io.in64, c->Un, io.out, io.out64, c->kind, c->gsrc, c->g,
                                     dt, c->da, c->gamma, stage, c->opt.limiter, c->opt.flux == ZK_FLUX_HLL,
                                     st(c)->s0, c->d_status, fused_indicator(c) ? &ind : nullptr, c->dg_tpc,
                                     c->stream);
}

// Threads per cell of the mixed stage kernel: pinned (opt.tile_tpc), two with
// the fused indicator, else tuned once per (device, order, grid) by timing
// stage 1 of each choice on this context's state (both give the same bits;
// the timing launches write only the stage-1 buffer, which the step then
// rewrites).  Skipped, with the default, while the stream is being captured.
int choose_tpc(zk_ctx* c, double dt) {
    using Key = std::tuple<int, int, int, int>;
    static std::mutex mu;
    static std::map<Key, int> cache;
    if (c->opt.tile_tpc == 1 || c->opt.tile_tpc == 2) {
        c->dg_tpc = c->opt.tile_tpc;
        return ZK_OK;
    }
    if (fused_indicator(c)) {
        c->dg_tpc = 2;
        return ZK_OK;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        c->dg_tpc = zk::dg_mixed_default_tpc(c->opt.order);
        return ZK_OK;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    const Key key{dev, c->opt.order, c->g.ny, c->g.nx};
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            c->dg_tpc = it->second;
            return ZK_OK;
        }
    }
    float best = 0.0f;
    int best_tpc = zk::dg_mixed_default_tpc(c->opt.order);
    for (int tpc : {1, 2}) {
        c->dg_tpc = tpc;
        cudaError_t e = mixed_stage(c, dt, 1);  // first use (and warm-up)
        if (e == cudaSuccess) e = cudaEventRecord(c->ev0, c->stream);
        for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = mixed_stage(c, dt, 1);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(c->ev1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        if (e != cudaSuccess) return cuda_fail(e);
        if (tpc == 1 || ms < best) {
            best = ms;
            best_tpc = tpc;
        }
    }
    c->dg_tpc = best_tpc;
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = best_tpc;
    return ZK_OK;
}

}  // namespace

int zk_dg_setup(zk_ctx* c) {
    const int P = c->opt.order;
    if (c->opt.limiter >= ZK_LIMITER_TVB && !(c->opt.tvb_M >= 0.0))
        return zk_internal_fail(ZK_ERR_ARG, "TVB constant M must be >= 0");
    DGState* s = new DGState();
    c->dg = s;
    zk::DGTab tab;
    double phic[zk::DG_MAXNM * 4];
    zk::dg_make_tables(P, &tab, phic);
    if (zk::dg_upload_tables(P, tab) != ZK_OK) return zk_internal_fail(ZK_ERR_CUDA, "DG table upload failed");
    if (c->fma() && (zk_fma::dg_upload_tables(P, tab) != ZK_OK || zk::dg_upload_sep_f64(P) != ZK_OK))
        return zk_internal_fail(ZK_ERR_CUDA, "DG table upload failed");
    s->s0 = (P >= 3) ? -3.0 * std::log10((double)P) : -4.0 * std::log10((double)P);
    s->xpitch = c->g.pitch + 32;
    const int NQ = P + 1, NM = NQ * NQ;
    cudaError_t e = cudaMalloc(&c->d_phic, sizeof(double) * NM * 4);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d_phic, phic, sizeof(double) * NM * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMalloc(&s->fx, sizeof(double) * NQ * 4 * (size_t)c->g.ny * s->xpitch);
    if (e == cudaSuccess) e = cudaMalloc(&s->fy, sizeof(double) * NQ * 4 * (size_t)(c->g.ny + 1) * c->g.pitch);
    if (e == cudaSuccess && c->opt.precision == ZK_PREC_MIXED) {
        if (zk::dg_upload_tables_f32(P) != ZK_OK) return zk_internal_fail(ZK_ERR_CUDA, "DG FP32 table upload failed");
        const size_t n = (size_t)4 * NM * c->g.plane;
        e = cudaMalloc(&c->F1, sizeof(float) * n);
        if (e == cudaSuccess) e = cudaMalloc(&c->F2, sizeof(float) * n);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->F1, 0, sizeof(float) * n, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->F2, 0, sizeof(float) * n, c->stream);
    }
    if (e == cudaSuccess && !c->d_flags) e = cudaMalloc(&c->d_flags, c->g.plane);
    if (e == cudaSuccess && !c->d_nflag) e = cudaMalloc(&c->d_nflag, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_nflag, 0, sizeof(uint32_t), c->stream);
    if (e == cudaSuccess && c->opt.limiter == ZK_LIMITER_TVB_MLP && !c->mlp)
        e = cudaMalloc(&c->mlp, sizeof(zk::MlpPacked));
    if (e == cudaSuccess && fused_indicator(c)) {
        if (!c->mlp_frag) e = cudaMalloc(&c->mlp_frag, sizeof(zk::MlpFrag));
        if (e == cudaSuccess && !c->d_list) e = cudaMalloc(&c->d_list, sizeof(int32_t) * c->g.plane);
        if (e == cudaSuccess && !c->d_lcount) e = cudaMalloc(&c->d_lcount, 3 * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMemsetAsync(c->d_lcount, 0, 3 * sizeof(uint32_t), c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// TVB work after stage `stage` (1..3) wrote its output, when configured: the
// plain TVB pass over every cell; with the fused indicator, the TVB pass over
// the cells the stage listed; otherwise the indicator-gated pass over every
// cell (features: the output's modes, the stage input's means).
int zk_dg_after_stage(zk_ctx* c, int stage) {
    if (c->opt.limiter < ZK_LIMITER_TVB) return ZK_OK;
    const StageIO io = stage_io(c, stage);
    cudaError_t e;
    if (fused_indicator(c)) {
        e = zk::launch_dg_tvb_list(c->opt.order, io.out, io.out64, c->kind, c->gsrc, c->g, c->da, c->gamma,
                                   c->opt.tvb_M, nullptr, c->d_nflag, c->d_list, c->d_lcount + (stage - 1),
                                   c->sms * 4, c->stream);
    } else {
        const zk::MlpPacked* w = nullptr;
        if (c->opt.limiter == ZK_LIMITER_TVB_MLP) {
            if (!c->mlp_set) return zk_internal_fail(ZK_ERR_STATE, "indicator weights not set (zk_set_indicator)");
            w = static_cast<const zk::MlpPacked*>(c->mlp);
        }
        e = zk::launch_dg_tvb(c->opt.order, io.out, io.out64, c->kind, c->gsrc, c->g, c->da, c->gamma, c->opt.tvb_M,
                              c->d_flags, w, nullptr, c->d_nflag, nullptr, w ? io.in : nullptr, io.in64,
                              c->mlp_screen, c->stream);
    }
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// The TVB_MLP limiter of a step or stage 1 needs its weights; the fused
// indicator's list counters restart at stage 1.
static int begin_step(zk_ctx* c) {
    if (c->opt.limiter == ZK_LIMITER_TVB_MLP && !c->mlp_set)
        return zk_internal_fail(ZK_ERR_STATE, "indicator weights not set (zk_set_indicator)");
    if (fused_indicator(c)) {
        const cudaError_t e = cudaMemsetAsync(c->d_lcount, 0, 3 * sizeof(uint32_t), c->stream);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    return ZK_OK;
}

void zk_dg_release(zk_ctx* c) {
    DGState* s = st(c);
    if (!s) return;
    if (s->fx) cudaFree(s->fx);
    if (s->fy) cudaFree(s->fy);
    delete s;
    c->dg = nullptr;
    for (void* p : {(void*)c->mlp, (void*)c->mlp_frag, (void*)c->d_flags, (void*)c->d_nflag, (void*)c->d_list,
                    (void*)c->d_lcount})
        if (p) cudaFree(p);
    c->mlp = nullptr;
    c->mlp_frag = nullptr;
    c->d_flags = nullptr;
    c->d_nflag = nullptr;
    c->d_list = nullptr;
    c->d_lcount = nullptr;
    c->mlp_set = false;
}

static int dg_step_mixed(zk_ctx* c, double dt) {
    if (!c->dg_tpc)
        if (int rc = choose_tpc(c, dt)) return rc;
    if (int rc = begin_step(c)) return rc;
    for (int k = 1; k <= 3; ++k) {
        const cudaError_t e = mixed_stage(c, dt, k);
        if (e != cudaSuccess) return cuda_fail(e);
        if (int rc = zk_dg_after_stage(c, k)) return rc;
    }
    return ZK_OK;
}

int zk_dg_step(zk_ctx* c, double dt) {
    if (c->opt.precision == ZK_PREC_MIXED) return dg_step_mixed(c, dt);
    if (int rc = begin_step(c)) return rc;
    for (int k = 1; k <= 3; ++k) {
        const StageIO io = stage_io(c, k);
        const cudaError_t e = stage_f64(c, args(c, static_cast<const double*>(io.in), c->Un,
                                                static_cast<double*>(io.out), dt, k));
        if (e != cudaSuccess) return cuda_fail(e);
        if (int rc = zk_dg_after_stage(c, k)) return rc;
    }
    return ZK_OK;
}

// Stage `stage` (1..3) of zk_dg_step alone, without the TVB pass after it:
// the same launch with the same buffers (FP64: U^n -> S1 -> S2 -> U^n;
// mixed: U^n -> F1 -> F2 -> U^n).
int zk_dg_stage(zk_ctx* c, double dt, int stage) {
    if (c->opt.precision == ZK_PREC_MIXED && !c->dg_tpc)
        if (int rc = choose_tpc(c, dt)) return rc;
    if (stage == 1)
        if (int rc = begin_step(c)) return rc;
    cudaError_t e;
    if (c->opt.precision == ZK_PREC_MIXED) {
        e = mixed_stage(c, dt, stage);
    } else {
        const StageIO io = stage_io(c, stage);
        e = stage_f64(c, args(c, static_cast<const double*>(io.in), c->Un, static_cast<double*>(io.out), dt, stage));
    }
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// The TVB pass zk_dg_step runs after stage `stage` (nothing for the other
// limiters), on that stage's output.
int zk_dg_stage_limit(zk_ctx* c, int stage) { return zk_dg_after_stage(c, stage); }

int zk_dg_rhs(zk_ctx* c, double* dU_dev) {
    cudaError_t e = stage_f64(c, args(c, c->Un, c->Un, dU_dev, 0.0, 0));
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

int zk_dg_limit(zk_ctx* c) {
    if (c->opt.limiter >= ZK_LIMITER_TVB) {
        // applyLimiter on the current state: the TVB pass over every cell (the
        // gated one with the state's own means as the indicator's inputs)
        const zk::MlpPacked* w = nullptr;
        if (c->opt.limiter == ZK_LIMITER_TVB_MLP) {
            if (!c->mlp_set) return zk_internal_fail(ZK_ERR_STATE, "indicator weights not set (zk_set_indicator)");
            w = static_cast<const zk::MlpPacked*>(c->mlp);
        }
        cudaError_t e = zk::launch_dg_tvb(c->opt.order, c->Un, true, c->kind, c->gsrc, c->g, c->da, c->gamma,
                                          c->opt.tvb_M, c->d_flags, w, nullptr, c->d_nflag, nullptr, nullptr, true,
                                          c->mlp_screen, c->stream);
        return e == cudaSuccess ? ZK_OK : cuda_fail(e);
    }
    zk::DGArgs a = args(c, c->Un, c->Un, c->Un, 0.0, 1);
    cudaError_t e = limit_f64(c, a);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// ---- learned indicator: weights, features, counters ------------------------------
extern "C" int zk_set_indicator(zk_ctx* c, const float* params, int nparams) {
    if (!c || !params) return zk_internal_fail(ZK_ERR_ARG, "null argument");
    if (nparams != zk::MLP_NPARAM) return zk_internal_fail(ZK_ERR_ARG, "indicator needs exactly MLP_NPARAM parameters");
    if (c->opt.limiter != ZK_LIMITER_TVB_MLP || !c->mlp)
        return zk_internal_fail(ZK_ERR_STATE, "context is not a DG TVB_MLP context with a mesh");
    // BF16 inference weights, packed in the shared-memory layout of the
    // tensor-core inference (zk_mlp.h: MlpPacked)
    zk::MlpWeights W;
    std::memcpy(&W, params, sizeof W);
    zk::MlpPacked K;
    std::memset(&K, 0, sizeof K);
    auto bits = [](float x) {
        __nv_bfloat16 b = __float2bfloat16(x);
        uint16_t u;
        std::memcpy(&u, &b, 2);
        return u;
    };
    for (int o = 0; o < zk::MLP_H; ++o) {
        for (int i = 0; i < zk::MLP_IN; ++i) K.w1[o][i] = bits(W.w1[o][i]);
        for (int i = 0; i < zk::MLP_H; ++i) {
            K.w2[o][i] = bits(W.w2[o][i]);
            K.w3[o][i] = bits(W.w3[o][i]);
        }
        K.b1[o] = zk::bf16_round_host(W.b1[o]);
        K.b2[o] = zk::bf16_round_host(W.b2[o]);
        K.b3[o] = zk::bf16_round_host(W.b3[o]);
        K.w4[o] = zk::bf16_round_host(W.w4[o]);
    }
    K.b4 = zk::bf16_round_host(W.b4);
    cudaError_t e = cudaMemcpyAsync(c->mlp, &K, sizeof K, cudaMemcpyHostToDevice, c->stream);
    zk::MlpFrag Fr;
    if (c->mlp_frag) {
        zk::pack_mlp_frag(W, &Fr);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->mlp_frag, &Fr, sizeof Fr, cudaMemcpyHostToDevice, c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    c->mlp_set = true;
    return ZK_OK;
}

extern "C" int zk_set_indicator_screen(zk_ctx* c, float screen) {
    if (!c) return zk_internal_fail(ZK_ERR_ARG, "null argument");
    if (!(screen == screen)) return zk_internal_fail(ZK_ERR_ARG, "screen must not be NaN");
    c->mlp_screen = screen;
    // captured steps hold the old value: drop them
    if (c->step_graph) {
        cudaGraphExecDestroy(c->step_graph);
        c->step_graph = nullptr;
    }
    return ZK_OK;
}

extern "C" int zk_indicator_features(zk_ctx* c, float* features, uint8_t* labels) {
    if (!c || !c->Un || c->opt.method != ZK_METHOD_DG) return zk_internal_fail(ZK_ERR_STATE, "needs a DG context with a mesh");
    const size_t ncell = (size_t)c->g.ny * c->g.nx;
    float* df = nullptr;
    cudaError_t e = cudaMalloc(&df, sizeof(float) * zk::MLP_IN * ncell);
    if (e == cudaSuccess) e = cudaMemsetAsync(df, 0, sizeof(float) * zk::MLP_IN * ncell, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_dg_tvb(c->opt.order, c->Un, true, c->kind, c->gsrc, c->g, c->da, c->gamma, c->opt.tvb_M,
                              c->d_flags, nullptr, df, nullptr, nullptr, nullptr, true, -1.0f, c->stream);
    if (e == cudaSuccess && features)
        e = cudaMemcpyAsync(features, df, sizeof(float) * zk::MLP_IN * ncell, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && labels)
        e = cudaMemcpy2DAsync(labels, c->g.nx, c->d_flags, c->g.pitch, c->g.nx, c->g.ny, cudaMemcpyDeviceToHost,
                              c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (df) cudaFree(df);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

extern "C" int zk_limited_cells(zk_ctx* c, uint32_t* count) {
    if (!c || !count) return zk_internal_fail(ZK_ERR_ARG, "null argument");
    if (!c->d_nflag) { *count = 0; return ZK_OK; }
    cudaError_t e = cudaMemcpyAsync(count, c->d_nflag, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

extern "C" int zk_indicator_logits(zk_ctx* c, float* logits) {
    if (!c || !logits) return zk_internal_fail(ZK_ERR_ARG, "null argument");
    if (!c->Un || c->opt.limiter != ZK_LIMITER_TVB_MLP || !c->mlp_set)
        return zk_internal_fail(ZK_ERR_STATE, "needs a DG TVB_MLP context with a mesh and indicator weights");
    const size_t ncell = (size_t)c->g.ny * c->g.nx;
    float* dl = nullptr;
    cudaError_t e = cudaMalloc(&dl, sizeof(float) * ncell);
    if (e == cudaSuccess) e = cudaMemsetAsync(dl, 0, sizeof(float) * ncell, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_dg_tvb(c->opt.order, c->Un, true, c->kind, c->gsrc, c->g, c->da, c->gamma, c->opt.tvb_M,
                              nullptr, static_cast<const zk::MlpPacked*>(c->mlp), nullptr, nullptr, dl, nullptr, true,
                              -1.0f, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(logits, dl, sizeof(float) * ncell, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (dl) cudaFree(dl);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// Per cell of stage `stage`'s output (run just before by zk_stage): the
// indicator's 40 features (the output's modes, the stage input's means) and
// the plain TVB indicator's label of the output.
extern "C" int zk_indicator_stage_features(zk_ctx* c, int stage, float* features, uint8_t* labels) {
    if (!c || !c->Un || c->opt.method != ZK_METHOD_DG) return zk_internal_fail(ZK_ERR_STATE, "needs a DG context with a mesh");
    if (stage < 1 || stage > 3) return zk_internal_fail(ZK_ERR_ARG, "stage must be 1, 2 or 3");
    const size_t ncell = (size_t)c->g.ny * c->g.nx;
    const StageIO io = stage_io(c, stage);
    float* df = nullptr;
    cudaError_t e = cudaSetDevice(c->opt.device);
    if (e == cudaSuccess) e = cudaMalloc(&df, sizeof(float) * zk::MLP_IN * ncell);
    if (e == cudaSuccess) e = cudaMemsetAsync(df, 0, sizeof(float) * zk::MLP_IN * ncell, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_dg_tvb(c->opt.order, io.out, io.out64, c->kind, c->gsrc, c->g, c->da, c->gamma, c->opt.tvb_M,
                              c->d_flags, nullptr, df, nullptr, nullptr, io.in, io.in64, -1.0f, c->stream);
    if (e == cudaSuccess && features)
        e = cudaMemcpyAsync(features, df, sizeof(float) * zk::MLP_IN * ncell, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && labels)
        e = cudaMemcpy2DAsync(labels, c->g.nx, c->d_flags, c->g.pitch, c->g.nx, c->g.ny, cudaMemcpyDeviceToHost,
                              c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (df) cudaFree(df);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// zk_stage(stage) of a context running the fused indicator, returning per
// cell the features and logit the stage kernel computed (updated cells; 0
// elsewhere) and the number of cells it listed.
extern "C" int zk_indicator_stage_logits(zk_ctx* c, double dt, int stage, float* features, float* logits,
                                         uint32_t* listed) {
    if (!c || !c->Un || c->opt.method != ZK_METHOD_DG) return zk_internal_fail(ZK_ERR_STATE, "needs a DG context with a mesh");
    if (!fused_indicator(c))
        return zk_internal_fail(ZK_ERR_UNSUPPORTED, "needs a mixed-precision DG P=2/3 TVB_MLP context");
    if (stage < 1 || stage > 3) return zk_internal_fail(ZK_ERR_ARG, "stage must be 1, 2 or 3");
    if (!(dt > 0.0)) return zk_internal_fail(ZK_ERR_ARG, "dt must be > 0");
    cudaError_t e = cudaSetDevice(c->opt.device);
    if (e != cudaSuccess) return cuda_fail(e);
    if (stage == 1)
        if (int rc = begin_step(c)) return rc;
    const size_t n = (size_t)41 * c->g.plane;
    float* dbg = nullptr;
    e = cudaMalloc(&dbg, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemsetAsync(dbg, 0, sizeof(float) * n, c->stream);
    if (e == cudaSuccess) e = mixed_stage(c, dt, stage, dbg);
    std::vector<float> h;
    if (e == cudaSuccess) {
        h.resize(n);
        e = cudaMemcpyAsync(h.data(), dbg, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess && listed)
        e = cudaMemcpyAsync(listed, c->d_lcount + (stage - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (dbg) cudaFree(dbg);
    if (e != cudaSuccess) return cuda_fail(e);
    for (int i = 0; i < c->g.ny; ++i)
        for (int j = 0; j < c->g.nx; ++j) {
            const float* src = h.data() + ((size_t)i * c->g.pitch + j) * 41;
            const size_t cell = (size_t)i * c->g.nx + j;
            if (features) std::memcpy(features + cell * zk::MLP_IN, src, sizeof(float) * zk::MLP_IN);
            if (logits) logits[cell] = src[40];
        }
    return ZK_OK;
}

extern "C" int zk_tile_tpc(zk_ctx* c, int* tpc) {
    if (!c || !tpc) return zk_internal_fail(ZK_ERR_ARG, "null argument");
    *tpc = c->dg_tpc;
    return ZK_OK;
}
