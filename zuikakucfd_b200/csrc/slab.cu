// x-slab decomposition of one grid over several contexts (one per GPU): the
// SSP-RK3 step one stage at a time, and the 3-column halos of a slab's state
// packed into / unpacked from a contiguous device buffer, so that a caller can
// move them with NCCL, CUDA-aware MPI or a peer copy between the stages.
//
// The reference splits the grid into x-slabs with 3 exchange columns
// (bctype -3) on each inner side (splitMeshVertically, src_WENO/fluid.cpp:99-152)
// and swaps 3 columns per field with each neighbour after every stage
// (exchangeColumns, src_WENO/fluid.cpp:160-198; the DG version packs all
// 4*NM fields into one message, src_DG/fluid.cpp:342-400).  Here a stage is
// the same kernel launch zk_step makes; bctype -3 cells of a non-periodic
// context are passive (read as stored, never written by a stage's update), so
// the values the exchange stores there are what the stencils of the slab's
// edge cells read.
#include <algorithm>
#include <cmath>

#include "zk_common.cuh"
#include "zk_internal.h"
#include "zk_kernels.h"
#include "zuikaku.h"

namespace {

// One thread per halo element; buffer layout [plane][row][3], the state's
// [plane][row][pitch].  pack: buffer <- columns col0..col0+2; else the reverse.
template <typename T>
__global__ void __launch_bounds__(256) halo_copy_kernel(T* __restrict__ buf, T* __restrict__ state, int nplane,
                                                        int ny, int pitch, size_t plane, int col0, int pack) {
    const size_t n = (size_t)nplane * ny * 3;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(t % 3);
        const size_t pr = t / 3;
        const int i = (int)(pr % (size_t)ny);
        const size_t p = pr / (size_t)ny;
        const size_t k = p * plane + (size_t)i * pitch + col0 + c;
        if (pack) buf[t] = state[k];
        else state[k] = buf[t];
    }
}

int check(zk_ctx* c, int stage, int lo) {
    if (!c) return zk_internal_fail(ZK_ERR_ARG, "null context");
    if (!c->Un) return zk_internal_fail(ZK_ERR_STATE, "zk_set_mesh has not been called");
    if (stage < lo || stage > 3) return zk_internal_fail(ZK_ERR_ARG, "stage out of range");
    return ZK_OK;
}

int cuda_fail(cudaError_t e) { return zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e)); }

// The state written by `stage` (0 and 3: U^n) and its element size: FP32 for
// the stage states of a mixed-precision DG context, else FP64.
void* stage_state(zk_ctx* c, int stage, size_t* elem) {
    const bool f32 = c->opt.method == ZK_METHOD_DG && c->opt.precision == ZK_PREC_MIXED && (stage == 1 || stage == 2);
    *elem = f32 ? sizeof(float) : sizeof(double);
    if (f32) return stage == 1 ? (void*)c->F1 : (void*)c->F2;
    return stage == 1 ? (void*)c->S1 : stage == 2 ? (void*)c->S2 : (void*)c->Un;
}

int halo_copy(zk_ctx* c, int stage, int side, void* dev_buf, int pack) {
    if (int rc = check(c, stage, 0)) return rc;
    if (side != 0 && side != 1) return zk_internal_fail(ZK_ERR_ARG, "side must be 0 (left) or 1 (right)");
    if (!dev_buf) return zk_internal_fail(ZK_ERR_ARG, "null halo buffer");
    const int nx = c->g.nx;
    if (nx < 6) return zk_internal_fail(ZK_ERR_ARG, "a slab needs at least 6 columns");
    size_t elem = 0;
    void* state = stage_state(c, stage, &elem);
    // sent: the 3 owned columns next to the exchange columns; received: the exchange columns
    const int col0 = pack ? (side == 0 ? 3 : nx - 6) : (side == 0 ? 0 : nx - 3);
    const size_t n = (size_t)c->nvar * c->g.ny * 3;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)c->sms * 8);
    cudaError_t e = cudaSetDevice(c->opt.device);
    if (e != cudaSuccess) return cuda_fail(e);
    if (elem == sizeof(float))
        halo_copy_kernel<float><<<blocks, 256, 0, c->stream>>>((float*)dev_buf, (float*)state, c->nvar, c->g.ny,
                                                               c->g.pitch, c->g.plane, col0, pack);
    else
        halo_copy_kernel<double><<<blocks, 256, 0, c->stream>>>((double*)dev_buf, (double*)state, c->nvar, c->g.ny,
                                                                c->g.pitch, c->g.plane, col0, pack);
    e = cudaGetLastError();
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

}  // namespace

extern "C" {

int zk_stage(zk_ctx* c, double dt, int stage) {
    if (int rc = check(c, stage, 1)) return rc;
    if (!(dt > 0.0) || !std::isfinite(dt)) return zk_internal_fail(ZK_ERR_ARG, "dt must be finite and > 0");
    cudaError_t e = cudaSetDevice(c->opt.device);
    if (e == cudaSuccess && stage == 1) e = cudaMemsetAsync(c->d_status, 0, sizeof(uint32_t), c->stream);
    if (e == cudaSuccess && stage == 1 && c->d_nflag) e = cudaMemsetAsync(c->d_nflag, 0, sizeof(uint32_t), c->stream);
    if (e != cudaSuccess) return cuda_fail(e);
    if (c->opt.method == ZK_METHOD_DG) return zk_dg_stage(c, dt, stage);
    if (c->opt.precision == ZK_PREC_MIXED) return zk_weno_mixed_stage(c, dt, stage);
    double* in[3] = {c->Un, c->S1, c->S2};
    double* out[3] = {c->S1, c->S2, c->Un};
    e = zk::launch_weno_stage_f64(c->fma(), in[stage - 1], c->Un, out[stage - 1], c->kind, c->gsrc, c->g, dt / c->da,
                                   dt / c->da, c->gamma, stage, c->d_status, c->stream, c->opt.recon);
    return e == cudaSuccess ? ZK_OK : cuda_fail(e);
}

int zk_stage_limit(zk_ctx* c, int stage) {
    if (int rc = check(c, stage, 1)) return rc;
    if (c->opt.method != ZK_METHOD_DG) return ZK_OK;
    const cudaError_t e = cudaSetDevice(c->opt.device);
    if (e != cudaSuccess) return cuda_fail(e);
    return zk_dg_stage_limit(c, stage);
}

int zk_halo_bytes(zk_ctx* c, int stage, size_t* bytes) {
    if (int rc = check(c, stage, 0)) return rc;
    if (!bytes) return zk_internal_fail(ZK_ERR_ARG, "null argument");
    size_t elem = 0;
    stage_state(c, stage, &elem);
    *bytes = (size_t)c->nvar * c->g.ny * 3 * elem;
    return ZK_OK;
}

int zk_halo_pack(zk_ctx* c, int stage, int side, void* dev_buf) { return halo_copy(c, stage, side, dev_buf, 1); }

int zk_halo_unpack(zk_ctx* c, int stage, int side, const void* dev_buf) {
    return halo_copy(c, stage, side, const_cast<void*>(dev_buf), 0);
}

}  // extern "C"
