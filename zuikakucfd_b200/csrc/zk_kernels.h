// Host-side launchers of the sm_100a kernels (one per .cu file group).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include "zk_common.cuh"

namespace zk {

// ---- FP64 reference-arithmetic kernels (built with --fmad=false) ----------
// recon: ZK_RECON_* face reconstruction (0 = WENO5, the reference's scheme)
cudaError_t launch_weno_stage_fp64(const double* Ucur, const double* Un, double* Uout,
                                   const int8_t* kind, const int32_t* gsrc, const Grid& g,
                                   double dtdx, double dtdy, double gamma, int stage,
                                   uint32_t* status, cudaStream_t s, int recon = 0);

}  // namespace zk

namespace zk_fma {
// The FP64 WENO stage compiled with fused multiply-add contraction
// (ZK_PREC_FP64_FMA); same arguments as zk::launch_weno_stage_fp64.
cudaError_t launch_weno_stage_fp64(const double* Ucur, const double* Un, double* Uout,
                                   const int8_t* kind, const int32_t* gsrc, const zk::Grid& g,
                                   double dtdx, double dtdy, double gamma, int stage,
                                   uint32_t* status, cudaStream_t s, int recon = 0);
}  // namespace zk_fma

namespace zk {

// The FP64 WENO stage of a context's precision: the reference-arithmetic
// kernel, or (fma) the contracted one.
inline cudaError_t launch_weno_stage_f64(bool fma, const double* Ucur, const double* Un, double* Uout,
                                         const int8_t* kind, const int32_t* gsrc, const Grid& g, double dtdx,
                                         double dtdy, double gamma, int stage, uint32_t* status, cudaStream_t s,
                                         int recon) {
    return fma ? zk_fma::launch_weno_stage_fp64(Ucur, Un, Uout, kind, gsrc, g, dtdx, dtdy, gamma, stage, status, s,
                                                recon)
               : launch_weno_stage_fp64(Ucur, Un, Uout, kind, gsrc, g, dtdx, dtdy, gamma, stage, status, s, recon);
}

cudaError_t launch_fill_ghosts(double* U, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                               int nvar, int nm, int sms, cudaStream_t s);
cudaError_t launch_max_speed_weno(const double* U, const Grid& g, double gamma,
                                  unsigned long long* out, int sms, cudaStream_t s);
cudaError_t launch_max_speed_dg(const double* dof, const int8_t* kind, const Grid& g, int nm,
                                double gamma, const double* phic, unsigned long long* out, int sms,
                                cudaStream_t s);
cudaError_t launch_recover(const double* U, const Grid& g, int nm, double gamma, double* prim,
                           int sms, cudaStream_t s);
cudaError_t launch_mach(const double* U, const Grid& g, int nm, double gamma, double* mach, double* speed, int sms,
                        cudaStream_t s);

}  // namespace zk
