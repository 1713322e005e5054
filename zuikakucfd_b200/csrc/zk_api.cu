// C ABI of the ZuikakuCFD B200 library (include/zuikaku.h): context, device
// state, the ghost source map, the SSP-RK3 step loop and the host-facing
// copies.  Kernel launches live in the per-kernel .cu files.
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "zk_common.cuh"
#include "zk_kernels.h"
#include "zk_internal.h"
#include "zuikaku.h"

using namespace zk;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define ZK_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess)                                                           \
            return fail(ZK_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(_e),    \
                        __FILE__, __LINE__);                                             \
    } while (0)

void free_device(zk_ctx* c) {
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);  // it captured the buffers freed below
    c->step_graph = nullptr;
    for (void* p : {(void*)c->Un, (void*)c->S1, (void*)c->S2, (void*)c->kind, (void*)c->gsrc,
                    (void*)c->d_max, (void*)c->d_status, (void*)c->d_phic, (void*)c->d_tmp,
                    (void*)c->F1, (void*)c->F2})
        if (p) cudaFree(p);
    c->Un = c->S1 = c->S2 = c->d_tmp = nullptr;
    c->F1 = c->F2 = nullptr;
    c->kind = nullptr;
    c->gsrc = nullptr;
    c->d_max = nullptr;
    c->d_status = nullptr;
    c->d_phic = nullptr;
}

}  // namespace

// Ghost source map on the host, pitched indices.  The reference fills ghosts
// with a row sweep then a column sweep over the fluid cells
// (src_WENO/fluid.cpp:338-370, src_DG/fluid.cpp:581-635); a ghost ends up with
// the value of the LAST source that wrote it: the largest source column of the
// column sweep, else the largest source row of the row sweep.
void build_ghost_map(int ny, int nx, int pitch, const int32_t* bct, bool slip, bool periodic,
                     std::vector<int8_t>& kind, std::vector<int32_t>& src) {
    kind.assign((size_t)ny * pitch, KIND_PASSIVE);
    src.assign((size_t)ny * pitch, -1);
    auto B = [&](int i, int j) { return bct[(size_t)i * nx + j]; };
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            const size_t k = (size_t)i * pitch + j;
            const int b = B(i, j);
            int8_t kd = (b == 0 && i >= 3 && i < ny - 3 && j >= 3 && j < nx - 3) ? KIND_UPDATED : KIND_PASSIVE;
            int32_t s = -1;
            if (periodic && b == -3) {
                const int iy = ny - 6, ix = nx - 6;
                const int si = 3 + (((i - 3) % iy) + iy) % iy;
                const int sj = 3 + (((j - 3) % ix) + ix) % ix;
                s = si * pitch + sj;
                kd = KIND_COPY;
            } else if (b == -1 || (slip && b == 1)) {
                int best = -1;
                if (i >= 3 && i < ny - 3)
                    for (int jj = j - 3; jj <= j + 3; ++jj)
                        if (jj != j && jj >= 3 && jj < nx - 3 && B(i, jj) == 0) best = jj;
                if (best >= 0) {
                    s = i * pitch + best;
                    kd = (b == 1) ? KIND_SLIP_X : KIND_COPY;
                } else {
                    if (j >= 3 && j < nx - 3)
                        for (int ii = i - 3; ii <= i + 3; ++ii)
                            if (ii != i && ii >= 3 && ii < ny - 3 && B(ii, j) == 0) best = ii;
                    if (best >= 0) {
                        s = best * pitch + j;
                        kd = (b == 1) ? KIND_SLIP_Y : KIND_COPY;
                    }
                }
            }
            kind[k] = (int8_t)(kd | (b == 0 ? KIND_FLUID : 0));
            src[k] = s;
        }
}

namespace {

int check_ctx(zk_ctx* c, bool need_state) {
    if (!c) return fail(ZK_ERR_ARG, "null context");
    if (need_state && !c->Un) return fail(ZK_ERR_STATE, "zk_set_mesh has not been called");
    return ZK_OK;
}

}  // namespace

int zk_internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }

extern "C" {

void zk_default_options(zk_options* o) {
    if (!o) return;
    o->method = ZK_METHOD_WENO;
    o->order = 2;
    o->precision = ZK_PREC_FP64;
    o->limiter = ZK_LIMITER_REFERENCE;
    o->flux = ZK_FLUX_HLLC;
    o->boundary = ZK_BOUNDARY_EXCHANGE;
    o->device = 0;
    o->tvb_M = 50.0;
    o->recon = ZK_RECON_WENO5;
    o->tile_tpc = 0;
}

int zk_version(void) { return 100; }

const char* zk_last_error(void) { return g_err.c_str(); }

int zk_create(const zk_options* opt, zk_ctx** out) {
    if (!opt || !out) return fail(ZK_ERR_ARG, "null argument");
    *out = nullptr;
    if (opt->method != ZK_METHOD_WENO && opt->method != ZK_METHOD_DG)
        return fail(ZK_ERR_ARG, "unknown method %d", opt->method);
    if (opt->method == ZK_METHOD_DG && (opt->order < 1 || opt->order > 3))
        return fail(ZK_ERR_ARG, "DG order must be 1..3, got %d", opt->order);
    if (opt->precision != ZK_PREC_FP64 && opt->precision != ZK_PREC_MIXED && opt->precision != ZK_PREC_FP64_FMA)
        return fail(ZK_ERR_ARG, "unknown precision %d", opt->precision);
    if (opt->limiter < ZK_LIMITER_REFERENCE || opt->limiter > ZK_LIMITER_TVB_MLP)
        return fail(ZK_ERR_ARG, "unknown limiter %d", opt->limiter);
    if (opt->flux != ZK_FLUX_HLLC && opt->flux != ZK_FLUX_HLL)
        return fail(ZK_ERR_ARG, "unknown flux %d", opt->flux);
    if (opt->boundary != ZK_BOUNDARY_EXCHANGE && opt->boundary != ZK_BOUNDARY_PERIODIC)
        return fail(ZK_ERR_ARG, "unknown boundary %d", opt->boundary);
    if (opt->recon < ZK_RECON_WENO5 || opt->recon > ZK_RECON_MUSCL_SUPERBEE)
        return fail(ZK_ERR_ARG, "unknown reconstruction %d", opt->recon);
    if (opt->tile_tpc < 0 || opt->tile_tpc > 2) return fail(ZK_ERR_ARG, "tile_tpc must be 0, 1 or 2");
    if (opt->tile_tpc == 1 && opt->limiter == ZK_LIMITER_TVB_MLP && opt->method == ZK_METHOD_DG && opt->order >= 2 &&
        opt->precision == ZK_PREC_MIXED)
        return fail(ZK_ERR_UNSUPPORTED, "the fused learned indicator runs two threads per cell");
    if (opt->recon != ZK_RECON_WENO5 && (opt->method != ZK_METHOD_WENO || opt->precision == ZK_PREC_MIXED))
        return fail(ZK_ERR_UNSUPPORTED, "MUSCL reconstruction runs on WENO contexts at FP64 / FP64_FMA precision");
    int ndev = 0;
    ZK_CUDA(cudaGetDeviceCount(&ndev));
    if (opt->device < 0 || opt->device >= ndev)
        return fail(ZK_ERR_ARG, "device %d out of range (%d devices)", opt->device, ndev);
    ZK_CUDA(cudaSetDevice(opt->device));
    zk_ctx* c = new zk_ctx();
    c->opt = *opt;
    c->nm = (opt->method == ZK_METHOD_DG) ? (opt->order + 1) * (opt->order + 1) : 1;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, opt->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e != cudaSuccess) {
        delete c;
        return fail(ZK_ERR_CUDA, "context setup: %s", cudaGetErrorString(e));
    }
    c->sms = prop.multiProcessorCount;
    c->stream = c->own_stream;
    *out = c;
    return ZK_OK;
}

int zk_destroy(zk_ctx* c) {
    if (!c) return ZK_OK;
    cudaSetDevice(c->opt.device);
    cudaStreamSynchronize(c->stream);
    free_device(c);
    zk_dg_release(c);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return ZK_OK;
}

int zk_set_mesh(zk_ctx* c, int ny, int nx, double da, double gamma, const int32_t* bctype) {
    if (!c || !bctype) return fail(ZK_ERR_ARG, "null argument");
    if (ny < 7 || nx < 7) return fail(ZK_ERR_ARG, "grid %dx%d too small (needs >= 7x7)", ny, nx);
    if ((size_t)ny * (size_t)round_pitch(nx) >= (size_t)INT32_MAX)
        return fail(ZK_ERR_ARG, "grid %dx%d too large for 32-bit cell indices", ny, nx);
    if (!(da > 0.0) || !(gamma > 1.0)) return fail(ZK_ERR_ARG, "need da > 0 and gamma > 1");
    const bool periodic = c->opt.boundary == ZK_BOUNDARY_PERIODIC;
    if (periodic) {
        for (int i = 0; i < ny; ++i)
            for (int j = 0; j < nx; ++j) {
                const bool ring = i < 3 || i >= ny - 3 || j < 3 || j >= nx - 3;
                if (ring && bctype[(size_t)i * nx + j] != -3)
                    return fail(ZK_ERR_ARG, "periodic boundary needs the 3-wide ring marked -3");
            }
    }
    ZK_CUDA(cudaSetDevice(c->opt.device));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    free_device(c);
    zk_dg_release(c);
    c->g.ny = ny;
    c->g.nx = nx;
    c->g.pitch = round_pitch(nx);
    c->g.plane = (size_t)ny * c->g.pitch;
    c->da = da;
    c->gamma = gamma;
    c->nvar = 4 * c->nm;
    c->bct.assign(bctype, bctype + (size_t)ny * nx);
    const size_t bytes = sizeof(double) * c->nvar * c->g.plane;
    std::vector<int8_t> kind;
    std::vector<int32_t> src;
    build_ghost_map(ny, nx, c->g.pitch, bctype, c->opt.method == ZK_METHOD_DG, periodic, kind, src);
    ZK_CUDA(cudaMalloc(&c->Un, bytes));
    ZK_CUDA(cudaMalloc(&c->S1, bytes));
    ZK_CUDA(cudaMalloc(&c->S2, bytes));
    ZK_CUDA(cudaMalloc(&c->kind, kind.size()));
    ZK_CUDA(cudaMalloc(&c->gsrc, src.size() * sizeof(int32_t)));
    ZK_CUDA(cudaMalloc(&c->d_max, sizeof(unsigned long long)));
    ZK_CUDA(cudaMalloc(&c->d_status, sizeof(uint32_t)));
    ZK_CUDA(cudaMemsetAsync(c->Un, 0, bytes, c->stream));
    ZK_CUDA(cudaMemsetAsync(c->S1, 0, bytes, c->stream));
    ZK_CUDA(cudaMemsetAsync(c->S2, 0, bytes, c->stream));
    ZK_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream));
    ZK_CUDA(cudaMemcpyAsync(c->kind, kind.data(), kind.size(), cudaMemcpyHostToDevice, c->stream));
    ZK_CUDA(cudaMemcpyAsync(c->gsrc, src.data(), src.size() * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    if (c->opt.method == ZK_METHOD_DG) {
        int rc = zk_dg_setup(c);
        if (rc) return rc;
    } else if (c->opt.precision == ZK_PREC_MIXED) {
        int rc = zk_weno_mixed_setup(c);
        if (rc) return rc;
    }
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

size_t zk_state_size(const zk_ctx* c) {
    if (!c) return 0;
    return (size_t)c->nvar * c->g.ny * c->g.nx;
}

int zk_set_state(zk_ctx* c, const double* host) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!host) return fail(ZK_ERR_ARG, "null state");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    ZK_CUDA(cudaMemcpy2DAsync(c->Un, sizeof(double) * c->g.pitch, host, sizeof(double) * c->g.nx,
                              sizeof(double) * c->g.nx, (size_t)c->nvar * c->g.ny,
                              cudaMemcpyHostToDevice, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_get_state(zk_ctx* c, double* host) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!host) return fail(ZK_ERR_ARG, "null state");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    ZK_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * c->g.nx, c->Un, sizeof(double) * c->g.pitch,
                              sizeof(double) * c->g.nx, (size_t)c->nvar * c->g.ny,
                              cudaMemcpyDeviceToHost, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_state_device(zk_ctx* c, double** dptr, int* pitch) {
    if (int rc = check_ctx(c, true)) return rc;
    if (dptr) *dptr = c->Un;
    if (pitch) *pitch = c->g.pitch;
    return ZK_OK;
}

// Mesh(folder): params.txt = "nx ny da gamma", then row-major text matrices
// (src_WENO/fluid.cpp:33-94; src_DG/fluid.cpp:148-244 + initDGModes).
int zk_load_case(zk_ctx* c, const char* dir) {
    if (!c || !dir) return fail(ZK_ERR_ARG, "null argument");
    const std::string d(dir);
    std::ifstream pf(d + "/params.txt");
    if (!pf) return fail(ZK_ERR_IO, "Cannot open params.txt in %s", dir);
    int nx = 0, ny = 0;
    double da = 0, gamma = 0;
    pf >> nx >> ny >> da >> gamma;
    if (!pf || nx <= 0 || ny <= 0) return fail(ZK_ERR_IO, "malformed params.txt in %s", dir);
    const size_t n = (size_t)ny * nx;
    std::vector<double> prim(4 * n);
    std::vector<int32_t> bct(n);
    const char* names[4] = {"rho.dat", "u.dat", "v.dat", "p.dat"};
    for (int f = 0; f < 4; ++f) {
        std::ifstream in(d + "/" + names[f]);
        if (!in) return fail(ZK_ERR_IO, "Cannot open file: %s/%s", dir, names[f]);
        for (size_t k = 0; k < n; ++k)
            if (!(in >> prim[f * n + k])) return fail(ZK_ERR_IO, "short file %s/%s", dir, names[f]);
    }
    {
        std::ifstream in(d + "/bctype.dat");
        if (!in) return fail(ZK_ERR_IO, "Cannot open file: %s/bctype.dat", dir);
        for (size_t k = 0; k < n; ++k)
            if (!(in >> bct[k])) return fail(ZK_ERR_IO, "short file %s/bctype.dat", dir);
    }
    if (int rc = zk_set_mesh(c, ny, nx, da, gamma, bct.data())) return rc;
    std::vector<double> state(zk_state_size(c), 0.0);
    const size_t vs = (size_t)c->nm * n;  // variable stride (mode 0 of each variable)
    for (size_t k = 0; k < n; ++k) {
        const double r = prim[k], ux = prim[n + k], vy = prim[2 * n + k], pr = prim[3 * n + k];
        state[k] = r;
        state[vs + k] = r * ux;
        state[2 * vs + k] = r * vy;
        state[3 * vs + k] = pr / (gamma - 1.0) + 0.5 * r * (ux * ux + vy * vy);
    }
    return zk_set_state(c, state.data());
}

int zk_set_stream(zk_ctx* c, void* s) {
    if (int rc = check_ctx(c, false)) return rc;
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    return ZK_OK;
}

int zk_synchronize(zk_ctx* c) {
    if (int rc = check_ctx(c, false)) return rc;
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_status_word(zk_ctx* c, uint32_t* out) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!out) return fail(ZK_ERR_ARG, "null argument");
    ZK_CUDA(cudaMemcpyAsync(out, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

// One SSP-RK3 step of the WENO path on the device state (enqueue only).
static int weno_step_fp64(zk_ctx* c, double dt) {
    const double dtdx = dt / c->da, dtdy = dt / c->da;
    ZK_CUDA(launch_weno_stage_f64(c->fma(), c->Un, c->Un, c->S1, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma, 1, c->d_status, c->stream, c->opt.recon));
    ZK_CUDA(launch_weno_stage_f64(c->fma(), c->S1, c->Un, c->S2, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma, 2, c->d_status, c->stream, c->opt.recon));
    ZK_CUDA(launch_weno_stage_f64(c->fma(), c->S2, c->Un, c->Un, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma, 3, c->d_status, c->stream, c->opt.recon));
    return ZK_OK;
}

static int step_once(zk_ctx* c, double dt) {
    if (c->opt.method == ZK_METHOD_DG) return zk_dg_step(c, dt);
    if (c->opt.precision == ZK_PREC_MIXED) return zk_weno_mixed_step(c, dt);
    return weno_step_fp64(c, dt);
}

// Steps per captured graph.  A step's launches are the same every step for a
// given dt (the stage buffers rotate within the step), so kGraphSteps steps
// are captured once and replayed; small grids, where a stage kernel lasts a
// few microseconds, then run without host launch gaps.
constexpr int kGraphSteps = 16;

// c->step_graph for dt: kept while dt and the buffers (freed with the graph
// by free_device) stay the same.  Leaves it null when capture is not possible
// (the stream is already being captured by the caller, or the legacy default
// stream); the caller then launches eagerly.
static int ensure_step_graph(zk_ctx* c, double dt) {
    if (c->step_graph && c->step_graph_dt == dt) return ZK_OK;
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return ZK_OK;
    }
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return ZK_OK;
    }
    int rc = ZK_OK;
    for (int i = 0; i < kGraphSteps && rc == ZK_OK; ++i) rc = step_once(c, dt);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);  // always ends the capture
    cudaGraphExec_t x = nullptr;
    cudaError_t ei = cudaSuccess;
    if (rc == ZK_OK && e == cudaSuccess && g) ei = cudaGraphInstantiate(&x, g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc != ZK_OK) return rc;
    if (e != cudaSuccess) return fail(ZK_ERR_CUDA, "step graph capture: %s", cudaGetErrorString(e));
    if (ei != cudaSuccess) return fail(ZK_ERR_CUDA, "step graph instantiate: %s", cudaGetErrorString(ei));
    c->step_graph = x;
    c->step_graph_dt = dt;
    return ZK_OK;
}

// nsteps steps: the first eagerly (any first-use set-up of the kernels runs
// outside a capture), then whole blocks of kGraphSteps as graph replays, then
// the rest eagerly.  The same kernels in the same order either way.
static int enqueue_steps(zk_ctx* c, double dt, int nsteps) {
    int s = 0;
    if (nsteps > 0) {
        if (int rc = step_once(c, dt)) return rc;
        s = 1;
    }
    const int blocks = (nsteps - s) / kGraphSteps;
    if (blocks > 0) {
        if (int rc = ensure_step_graph(c, dt)) return rc;
        if (c->step_graph) {
            for (int b = 0; b < blocks; ++b) ZK_CUDA(cudaGraphLaunch(c->step_graph, c->stream));
            s += blocks * kGraphSteps;
        }
    }
    for (; s < nsteps; ++s)
        if (int rc = step_once(c, dt)) return rc;
    return ZK_OK;
}

int zk_step(zk_ctx* c, double dt, int nsteps) {
    if (int rc = check_ctx(c, true)) return rc;
    if (nsteps < 0) return fail(ZK_ERR_ARG, "nsteps < 0");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(ZK_ERR_ARG, "dt must be finite and > 0");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    ZK_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream));
    if (c->d_nflag) ZK_CUDA(cudaMemsetAsync(c->d_nflag, 0, sizeof(uint32_t), c->stream));
    if (int rc = enqueue_steps(c, dt, nsteps)) return rc;
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_step_timed(zk_ctx* c, double dt, int nsteps, float* ms) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!ms || nsteps < 0) return fail(ZK_ERR_ARG, "bad argument");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(ZK_ERR_ARG, "dt must be finite and > 0");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    ZK_CUDA(cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream));
    ZK_CUDA(cudaEventRecord(c->ev0, c->stream));
    if (int rc = enqueue_steps(c, dt, nsteps)) return rc;
    ZK_CUDA(cudaEventRecord(c->ev1, c->stream));
    ZK_CUDA(cudaEventSynchronize(c->ev1));
    ZK_CUDA(cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return ZK_OK;
}

int zk_rhs(zk_ctx* c, double dt, double* host_dU) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!host_dU) return fail(ZK_ERR_ARG, "null dU");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    // The reference fills the ghosts of the state it is given, in place.
    ZK_CUDA(launch_fill_ghosts(c->Un, c->kind, c->gsrc, c->g, c->nvar, c->nm, c->sms, c->stream));
    if (c->opt.method == ZK_METHOD_DG) {
        if (int rc = zk_dg_rhs(c, c->S1)) return rc;
    } else {
        const double dtdx = dt / c->da, dtdy = dt / c->da;
        ZK_CUDA(launch_weno_stage_f64(c->fma(), c->Un, c->Un, c->S1, c->kind, c->gsrc, c->g, dtdx, dtdy, c->gamma, 0, c->d_status, c->stream, c->opt.recon));
    }
    ZK_CUDA(cudaMemcpy2DAsync(host_dU, sizeof(double) * c->g.nx, c->S1, sizeof(double) * c->g.pitch,
                              sizeof(double) * c->g.nx, (size_t)c->nvar * c->g.ny,
                              cudaMemcpyDeviceToHost, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_limit(zk_ctx* c) {
    if (int rc = check_ctx(c, true)) return rc;
    if (c->opt.method != ZK_METHOD_DG) return fail(ZK_ERR_UNSUPPORTED, "zk_limit is a DG operation");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    if (int rc = zk_dg_limit(c)) return rc;
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_max_speed(zk_ctx* c, double* out) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!out) return fail(ZK_ERR_ARG, "null argument");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    if (c->opt.method == ZK_METHOD_DG) {
        ZK_CUDA(launch_max_speed_dg(c->Un, c->kind, c->g, c->nm, c->gamma, c->d_phic, c->d_max, c->sms, c->stream));
    } else {
        ZK_CUDA(launch_max_speed_weno(c->Un, c->g, c->gamma, c->d_max, c->sms, c->stream));
    }
    unsigned long long bits = 0;
    ZK_CUDA(cudaMemcpyAsync(&bits, c->d_max, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    double v;
    std::memcpy(&v, &bits, sizeof v);
    *out = v;
    return ZK_OK;
}

int zk_recover_primitives(zk_ctx* c, double* host_prim) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!host_prim) return fail(ZK_ERR_ARG, "null argument");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    ZK_CUDA(launch_recover(c->Un, c->g, c->nm, c->gamma, c->S2, c->sms, c->stream));
    ZK_CUDA(cudaMemcpy2DAsync(host_prim, sizeof(double) * c->g.nx, c->S2, sizeof(double) * c->g.pitch,
                              sizeof(double) * c->g.nx, (size_t)4 * c->g.ny,
                              cudaMemcpyDeviceToHost, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

int zk_mach_number(zk_ctx* c, double* host_mach, double* host_speed) {
    if (int rc = check_ctx(c, true)) return rc;
    if (!host_mach) return fail(ZK_ERR_ARG, "null argument");
    ZK_CUDA(cudaSetDevice(c->opt.device));
    double* mach = c->S2;
    double* speed = c->S2 + c->g.plane;
    ZK_CUDA(launch_mach(c->Un, c->g, c->nm, c->gamma, mach, speed, c->sms, c->stream));
    ZK_CUDA(cudaMemcpy2DAsync(host_mach, sizeof(double) * c->g.nx, mach, sizeof(double) * c->g.pitch,
                              sizeof(double) * c->g.nx, c->g.ny, cudaMemcpyDeviceToHost, c->stream));
    if (host_speed)
        ZK_CUDA(cudaMemcpy2DAsync(host_speed, sizeof(double) * c->g.nx, speed, sizeof(double) * c->g.pitch,
                                  sizeof(double) * c->g.nx, c->g.ny, cudaMemcpyDeviceToHost, c->stream));
    ZK_CUDA(cudaStreamSynchronize(c->stream));
    return ZK_OK;
}

}  // extern "C"
