// zk_weno_step_noalloc: the FP64 WENO5 SSP-RK3 step (the same stage kernel as
// zk_step) for callers that cannot allocate device memory.
//
// Who needs it: an application whose GPU memory belongs to another allocator
// -- a framework's caching allocator or a memory pool reserved at start-up
// that forbids further cudaMalloc -- and loops that must not pay the implicit
// device-wide synchronisation of cudaMalloc/cudaFree.  Such a caller owns the
// state and bctype arrays and hands them in; every other buffer the step
// needs (two stage states, the ghost source map, the status word) lives in
// the file-scope array below, which each GPU that loads this library holds
// from load until process exit (about 17.3 MiB).
//
// Limits and rules:
//   * grid: ny * pitch <= ZK_NOALLOC_MAX_CELLS (262,144 cells, e.g. 512 x 512);
//     larger grids are rejected with ZK_ERR_ARG before any work is queued;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture.  The address is cached with the id of the
//     device's CUDA context; after a context reset (cudaDeviceReset anywhere in
//     the process) the next call looks it up again, so it too must come before
//     any stream capture;
//   * all calls share the one array: calls whose GPU work overlaps (two
//     streams, two host threads) race.  The status word is cleared by each
//     call; the stage states and the ghost map are rewritten in full before
//     they are read, so a previous call's contents never leak into a result.
#include <cstdio>
#include <mutex>

#include "zk_common.cuh"
#include "zk_internal.h"
#include "zk_kernels.h"

namespace {

constexpr size_t kMaxCells = 262144;  // ny * pitch
constexpr size_t kStageBytes = 4 * kMaxCells * sizeof(double);
constexpr size_t kOffStage0 = 0;
constexpr size_t kOffStage1 = kStageBytes;
constexpr size_t kOffSrc = 2 * kStageBytes;
constexpr size_t kOffKind = kOffSrc + kMaxCells * sizeof(int32_t);
constexpr size_t kOffStatus = kOffKind + kMaxCells;
constexpr size_t kScratchBytes = kOffStatus + 256;

// The scratch.  In host code this name is only a stand-in: its device
// address comes from cudaGetSymbolAddress, per device, below.
static __device__ __align__(256) unsigned char zk_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// Per device: the scratch address and the unique id of the CUDA context it
// was looked up in.  A context reset (cudaDeviceReset by any code in the
// process) gives the device a new context, possibly with the array at another
// address; the id tells the cached address apart from a stale one.
struct ScratchSlot {
    unsigned char* addr = nullptr;
    unsigned long long ctx_id = 0;
};
ScratchSlot g_slot[kMaxDevices];

// Ghost source map on the device, same rule as the host builder in
// zk_api.cu (row sweep then column sweep of src_WENO/fluid.cpp:338-370, last
// writer wins), for bctype -1 ghosts; exchange (-3) cells stay passive.
__global__ void ghost_map_kernel(const int32_t* bct, zk::Grid g, int8_t* kind, int32_t* src) {
    const size_t total = (size_t)g.ny * g.pitch;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / g.pitch), j = (int)(k - (size_t)i * g.pitch);
        int8_t kd = zk::KIND_PASSIVE;
        int32_t s = -1;
        if (j < g.nx) {
            const int b = bct[(size_t)i * g.nx + j];
            if (b == 0 && i >= 3 && i < g.ny - 3 && j >= 3 && j < g.nx - 3) kd = zk::KIND_UPDATED;
            if (b == -1) {
                int best = -1;
                if (i >= 3 && i < g.ny - 3)
                    for (int jj = j - 3; jj <= j + 3; ++jj)
                        if (jj != j && jj >= 3 && jj < g.nx - 3 && bct[(size_t)i * g.nx + jj] == 0) best = jj;
                if (best >= 0) {
                    s = i * g.pitch + best;
                    kd = zk::KIND_COPY;
                } else if (j >= 3 && j < g.nx - 3) {
                    for (int ii = i - 3; ii <= i + 3; ++ii)
                        if (ii != i && ii >= 3 && ii < g.ny - 3 && bct[(size_t)ii * g.nx + j] == 0) best = ii;
                    if (best >= 0) {
                        s = best * g.pitch + j;
                        kd = zk::KIND_COPY;
                    }
                }
            }
            if (b == 0) kd |= zk::KIND_FLUID;
        }
        kind[k] = kd;
        src[k] = s;
    }
}

// Unique id of the calling thread's current CUDA context (driver entry
// points cuCtxGetCurrent / cuCtxGetId, looked up through the runtime so the
// library needs no link-time libcuda); false when there is none yet or the
// driver lacks them.
bool current_context_id(unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
    });
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of the scratch on the current device.  Set-up: the first
// call on a device (and the first after that device's context was reset)
// looks the address up with cudaGetSymbolAddress, with the device current;
// later calls reuse it while the context id is unchanged.
int scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return zk_internal_fail(ZK_ERR_UNSUPPORTED, "device ordinal >= 64");
    std::lock_guard<std::mutex> lock(g_mu);
    ScratchSlot& slot = g_slot[dev];
    unsigned long long id = 0;
    if (slot.addr && current_context_id(&id) && id == slot.ctx_id) {
        *out = slot.addr;
        return ZK_OK;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, zk_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        char msg[256];
        snprintf(msg, sizeof msg, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
        return zk_internal_fail(ZK_ERR_CUDA, msg);
    }
    // the lookup made the device's context current; without an id (old
    // driver) nothing is cached and every call looks the address up again
    if (current_context_id(&id)) {
        slot.addr = static_cast<unsigned char*>(p);
        slot.ctx_id = id;
    } else {
        slot.addr = nullptr;
    }
    *out = static_cast<unsigned char*>(p);
    return ZK_OK;
}

}  // namespace

extern "C" int zk_weno_step_noalloc(double* state, int ny, int nx, int pitch, double da, double gamma,
                                    const int32_t* bctype, double dt, int nsteps, void* stream,
                                    uint32_t* status_out) {
    if (!state || !bctype) return zk_internal_fail(ZK_ERR_ARG, "null state or bctype");
    if (ny < 7 || nx < 7 || pitch < nx || nsteps < 0)
        return zk_internal_fail(ZK_ERR_ARG, "need ny, nx >= 7, pitch >= nx, nsteps >= 0");
    if ((size_t)ny * (size_t)pitch > kMaxCells) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "grid %d x %d (pitch %d) needs %zu cells of scratch; zk_weno_step_noalloc holds %zu "
                 "(use zk_step for larger grids)", ny, nx, pitch, (size_t)ny * pitch, kMaxCells);
        return zk_internal_fail(ZK_ERR_ARG, msg);
    }
    if (!(da > 0.0) || !(gamma > 1.0) || !(dt > 0.0)) return zk_internal_fail(ZK_ERR_ARG, "need da, dt > 0, gamma > 1");
    unsigned char* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    double* S1 = reinterpret_cast<double*>(base + kOffStage0);
    double* S2 = reinterpret_cast<double*>(base + kOffStage1);
    int32_t* src = reinterpret_cast<int32_t*>(base + kOffSrc);
    int8_t* kind = reinterpret_cast<int8_t*>(base + kOffKind);
    uint32_t* status = reinterpret_cast<uint32_t*>(base + kOffStatus);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    zk::Grid g{ny, nx, pitch, (size_t)ny * pitch};
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        const size_t total = g.plane;
        int blocks = (int)((total + 255) / 256);
        if (blocks > 4096) blocks = 4096;
        ghost_map_kernel<<<blocks, 256, 0, s>>>(bctype, g, kind, src);
        e = cudaGetLastError();
    }
    const double dtdx = dt / da, dtdy = dt / da;
    for (int n = 0; n < nsteps && e == cudaSuccess; ++n) {
        e = zk::launch_weno_stage_fp64(state, state, S1, kind, src, g, dtdx, dtdy, gamma, 1, status, s);
        if (e == cudaSuccess) e = zk::launch_weno_stage_fp64(S1, state, S2, kind, src, g, dtdx, dtdy, gamma, 2, status, s);
        if (e == cudaSuccess) e = zk::launch_weno_stage_fp64(S2, state, state, kind, src, g, dtdx, dtdy, gamma, 3, status, s);
    }
    if (e == cudaSuccess && status_out) {
        e = cudaMemcpyAsync(status_out, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e != cudaSuccess) return zk_internal_fail(ZK_ERR_CUDA, cudaGetErrorString(e));
    return ZK_OK;
}
