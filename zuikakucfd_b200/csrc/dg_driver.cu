// DG driver: buffers, tables and the SSP-RK3 stage sequence of updateMesh
// (src_DG/fluid.cpp:1005-1054) on the device state.
#include <cmath>
#include <cstring>

#include <vector>

#include <cuda_bf16.h>

#include "dg_common.cuh"
#include "zk_internal.h"
#include "zk_mlp.h"

namespace zk {
cudaError_t launch_dg_stage_fp64(int P, const DGArgs& a, cudaStream_t s);
cudaError_t launch_dg_limit_fp64(int P, const DGArgs& a, cudaStream_t s);
int dg_upload_tables_f32(int P);
cudaError_t launch_dg_tvb(int P, void* state, bool fp64, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                          double da, double gamma, double M, uint8_t* flags, const MlpPacked* mlp,
                          float* features, uint32_t* nflag, float* logits, cudaStream_t s);
cudaError_t launch_dg_stage_mixed(int P, const void* cur, int in_fp64, const double* un, void* out, int out_fp64,
                                  const int8_t* kind, const int32_t* gsrc, const Grid& g, double dt, double da,
                                  double gamma, int stage, int limiter, int hll, double s0, uint32_t* status,
                                  cudaStream_t s);
}  // namespace zk

namespace {

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
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// TVB pass (plain or indicator-gated) on a stage output, when configured.
int zk_dg_after_stage(zk_ctx* c, void* state, bool fp64) {
    if (c->opt.limiter < ZK_LIMITER_TVB) return ZK_OK;
    const zk::MlpPacked* w = nullptr;
    if (c->opt.limiter == ZK_LIMITER_TVB_MLP) {
        if (!c->mlp_set) return zk_internal_fail(ZK_ERR_STATE, "indicator weights not set (zk_set_indicator)");
        w = static_cast<const zk::MlpPacked*>(c->mlp);
    }
    cudaError_t e = zk::launch_dg_tvb(c->opt.order, state, fp64, c->kind, c->gsrc, c->g, c->da, c->gamma,
                                      c->opt.tvb_M, c->d_flags, w, nullptr, c->d_nflag, nullptr, c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

void zk_dg_release(zk_ctx* c) {
    DGState* s = st(c);
    if (!s) return;
    if (s->fx) cudaFree(s->fx);
    if (s->fy) cudaFree(s->fy);
    delete s;
    c->dg = nullptr;
    for (void* p : {(void*)c->mlp, (void*)c->d_flags, (void*)c->d_nflag})
        if (p) cudaFree(p);
    c->mlp = nullptr;
    c->d_flags = nullptr;
    c->d_nflag = nullptr;
    c->mlp_set = false;
}

static int dg_step_mixed(zk_ctx* c, double dt) {
    const int P = c->opt.order, lim = c->opt.limiter, hll = c->opt.flux == ZK_FLUX_HLL;
    const double s0 = st(c)->s0;
    cudaError_t e = zk::launch_dg_stage_mixed(P, c->Un, 1, c->Un, c->F1, 0, c->kind, c->gsrc, c->g, dt, c->da,
                                              c->gamma, 1, lim, hll, s0, c->d_status, c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    if (int rc = zk_dg_after_stage(c, c->F1, false)) return rc;
    e = zk::launch_dg_stage_mixed(P, c->F1, 0, c->Un, c->F2, 0, c->kind, c->gsrc, c->g, dt, c->da, c->gamma, 2,
                                  lim, hll, s0, c->d_status, c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    if (int rc = zk_dg_after_stage(c, c->F2, false)) return rc;
    e = zk::launch_dg_stage_mixed(P, c->F2, 0, c->Un, c->Un, 1, c->kind, c->gsrc, c->g, dt, c->da, c->gamma, 3,
                                  lim, hll, s0, c->d_status, c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    return zk_dg_after_stage(c, c->Un, true);
}

int zk_dg_step(zk_ctx* c, double dt) {
    if (c->opt.precision == ZK_PREC_MIXED) return dg_step_mixed(c, dt);
    const int P = c->opt.order;
    cudaError_t e = zk::launch_dg_stage_fp64(P, args(c, c->Un, c->Un, c->S1, dt, 1), c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    if (int rc = zk_dg_after_stage(c, c->S1, true)) return rc;
    e = zk::launch_dg_stage_fp64(P, args(c, c->S1, c->Un, c->S2, dt, 2), c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    if (int rc = zk_dg_after_stage(c, c->S2, true)) return rc;
    e = zk::launch_dg_stage_fp64(P, args(c, c->S2, c->Un, c->Un, dt, 3), c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    return zk_dg_after_stage(c, c->Un, true);
}

// Stage `stage` (1..3) of zk_dg_step alone, without the TVB pass after it:
// the same launch with the same buffers (FP64: U^n -> S1 -> S2 -> U^n;
// mixed: U^n -> F1 -> F2 -> U^n).
int zk_dg_stage(zk_ctx* c, double dt, int stage) {
    const int P = c->opt.order;
    cudaError_t e;
    if (c->opt.precision == ZK_PREC_MIXED) {
        const void* in = stage == 1 ? (const void*)c->Un : (const void*)(stage == 2 ? c->F1 : c->F2);
        void* out = stage == 3 ? (void*)c->Un : (void*)(stage == 1 ? c->F1 : c->F2);
        e = zk::launch_dg_stage_mixed(P, in, stage == 1, c->Un, out, stage == 3, c->kind, c->gsrc, c->g, dt, c->da,
                                      c->gamma, stage, c->opt.limiter, c->opt.flux == ZK_FLUX_HLL, st(c)->s0,
                                      c->d_status, c->stream);
    } else {
        double* in[3] = {c->Un, c->S1, c->S2};
        double* out[3] = {c->S1, c->S2, c->Un};
        e = zk::launch_dg_stage_fp64(P, args(c, in[stage - 1], c->Un, out[stage - 1], dt, stage), c->stream);
    }
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

// The TVB pass zk_dg_step runs after stage `stage` (nothing for the other
// limiters), on that stage's output.
int zk_dg_stage_limit(zk_ctx* c, int stage) {
    if (c->opt.precision == ZK_PREC_MIXED)
        return stage == 3 ? zk_dg_after_stage(c, c->Un, true) : zk_dg_after_stage(c, stage == 1 ? c->F1 : c->F2, false);
    double* out[3] = {c->S1, c->S2, c->Un};
    return zk_dg_after_stage(c, out[stage - 1], true);
}

int zk_dg_rhs(zk_ctx* c, double* dU_dev) {
    cudaError_t e = zk::launch_dg_stage_fp64(c->opt.order, args(c, c->Un, c->Un, dU_dev, 0.0, 0), c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

int zk_dg_limit(zk_ctx* c) {
    if (c->opt.limiter >= ZK_LIMITER_TVB) return zk_dg_after_stage(c, c->Un, true);
    zk::DGArgs a = args(c, c->Un, c->Un, c->Un, 0.0, 1);
    cudaError_t e = zk::launch_dg_limit_fp64(c->opt.order, a, c->stream);
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
        K.b1[o] = W.b1[o]; K.b2[o] = W.b2[o]; K.b3[o] = W.b3[o]; K.w4[o] = W.w4[o];
    }
    K.b4 = W.b4;
    cudaError_t e = cudaMemcpyAsync(c->mlp, &K, sizeof K, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    c->mlp_set = true;
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
                              c->d_flags, nullptr, df, nullptr, nullptr, c->stream);
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
                              nullptr, static_cast<const zk::MlpPacked*>(c->mlp), nullptr, nullptr, dl, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(logits, dl, sizeof(float) * ncell, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (dl) cudaFree(dl);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}
