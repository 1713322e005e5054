// DG driver: buffers, tables and the SSP-RK3 stage sequence of updateMesh
// (src_DG/fluid.cpp:1005-1054) on the device state.
#include <cmath>

#include "dg_common.cuh"
#include "zk_internal.h"

namespace zk {
cudaError_t launch_dg_stage_fp64(int P, const DGArgs& a, cudaStream_t s);
cudaError_t launch_dg_limit_fp64(int P, const DGArgs& a, cudaStream_t s);
int dg_upload_tables_f32(int P);
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
    if (c->opt.limiter != ZK_LIMITER_REFERENCE && c->opt.limiter != ZK_LIMITER_NONE)
        return zk_internal_fail(ZK_ERR_UNSUPPORTED, "DG TVB limiters are not available in this build");
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
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

void zk_dg_release(zk_ctx* c) {
    DGState* s = st(c);
    if (!s) return;
    if (s->fx) cudaFree(s->fx);
    if (s->fy) cudaFree(s->fy);
    delete s;
    c->dg = nullptr;
}

static int dg_step_mixed(zk_ctx* c, double dt) {
    const int P = c->opt.order, lim = c->opt.limiter, hll = c->opt.flux == ZK_FLUX_HLL;
    const double s0 = st(c)->s0;
    cudaError_t e = zk::launch_dg_stage_mixed(P, c->Un, 1, c->Un, c->F1, 0, c->kind, c->gsrc, c->g, dt, c->da,
                                              c->gamma, 1, lim, hll, s0, c->d_status, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_dg_stage_mixed(P, c->F1, 0, c->Un, c->F2, 0, c->kind, c->gsrc, c->g, dt, c->da, c->gamma, 2,
                                      lim, hll, s0, c->d_status, c->stream);
    if (e == cudaSuccess)
        e = zk::launch_dg_stage_mixed(P, c->F2, 0, c->Un, c->Un, 1, c->kind, c->gsrc, c->g, dt, c->da, c->gamma, 3,
                                      lim, hll, s0, c->d_status, c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

int zk_dg_step(zk_ctx* c, double dt) {
    if (c->opt.precision == ZK_PREC_MIXED) return dg_step_mixed(c, dt);
    const int P = c->opt.order;
    cudaError_t e = zk::launch_dg_stage_fp64(P, args(c, c->Un, c->Un, c->S1, dt, 1), c->stream);
    if (e == cudaSuccess) e = zk::launch_dg_stage_fp64(P, args(c, c->S1, c->Un, c->S2, dt, 2), c->stream);
    if (e == cudaSuccess) e = zk::launch_dg_stage_fp64(P, args(c, c->S2, c->Un, c->Un, dt, 3), c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

int zk_dg_rhs(zk_ctx* c, double* dU_dev) {
    cudaError_t e = zk::launch_dg_stage_fp64(c->opt.order, args(c, c->Un, c->Un, dU_dev, 0.0, 0), c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

int zk_dg_limit(zk_ctx* c) {
    zk::DGArgs a = args(c, c->Un, c->Un, c->Un, 0.0, 1);
    cudaError_t e = zk::launch_dg_limit_fp64(c->opt.order, a, c->stream);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}
