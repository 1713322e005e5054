// Internal definition of the opaque zk_ctx and the hooks between the API
// layer (zk_api.cu) and the method-specific drivers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "zk_common.cuh"
#include "zuikaku.h"

struct zk_ctx {
    zk_options opt{};
    bool fma() const { return opt.precision == ZK_PREC_FP64_FMA; }
    zk::Grid g{};
    double da = 0.0, gamma = 0.0;
    int nm = 1;    // modes per variable (1 for WENO)
    int nvar = 4;  // planes of the state (4 * nm)
    int sms = 148;
    std::vector<int32_t> bct;  // host copy of bctype, row-major ny x nx

    double* Un = nullptr;  // FP64 state (the step's U^n, updated in place by the last stage)
    double* S1 = nullptr;  // stage scratch
    double* S2 = nullptr;  // stage scratch
    double* d_tmp = nullptr;
    float* F1 = nullptr;  // FP32 stage states of the mixed-precision path
    float* F2 = nullptr;
    int8_t* kind = nullptr;   // per-cell kind byte (zk::KIND_*), pitched
    int32_t* gsrc = nullptr;  // fill source (pitched linear index) of ghost cells
    unsigned long long* d_max = nullptr;
    uint32_t* d_status = nullptr;
    double* d_phic = nullptr;  // DG basis at the 4 cell corners, [NM][4]

    CUtensorMap tmap[3];  // TMA maps over Un, S1, S2 (mixed WENO path)

    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void* dg = nullptr;  // DG driver state
    void* mlp = nullptr;          // device MlpPacked (learned indicator, separate gated pass), BF16-rounded
    void* mlp_frag = nullptr;     // device MlpFrag (the same weights for the indicator fused in the stage)
    bool mlp_set = false;
    float mlp_screen = -1.0f;     // indicator screen (zk_set_indicator_screen); < 0: every cell evaluated
    int dg_tpc = 0;               // threads per cell of the mixed DG stage kernel (0: not chosen yet)
    int32_t* d_list = nullptr;    // cells the fused indicator flagged in the current stage (pitched indices)
    uint32_t* d_lcount = nullptr; // their counts, one per RK stage, cleared at each step's stage 1
    uint8_t* d_flags = nullptr;   // TVB troubled-cell flags of the last pass, pitched
    uint32_t* d_nflag = nullptr;  // cells the TVB passes limited during the last zk_step

    cudaGraphExec_t step_graph = nullptr;  // kGraphSteps steps at step_graph_dt (zk_step)
    double step_graph_dt = 0.0;
};

int zk_internal_fail(int code, const char* msg);

// Ghost source map (kind byte and fill source per pitched cell) of a bctype
// field; slip: DG slip walls (bctype 1); periodic: the -3 ring wraps.
void build_ghost_map(int ny, int nx, int pitch, const int32_t* bct, bool slip, bool periodic,
                     std::vector<int8_t>& kind, std::vector<int32_t>& src);

// DG driver (dg_driver.cu)
int zk_dg_setup(zk_ctx* c);
void zk_dg_release(zk_ctx* c);
int zk_dg_step(zk_ctx* c, double dt);
int zk_dg_rhs(zk_ctx* c, double* dU_dev);
int zk_dg_limit(zk_ctx* c);
int zk_dg_after_stage(zk_ctx* c, int stage);
int zk_dg_stage(zk_ctx* c, double dt, int stage);
int zk_dg_stage_limit(zk_ctx* c, int stage);

// WENO mixed-precision driver (weno_mixed.cu)
int zk_weno_mixed_setup(zk_ctx* c);
int zk_weno_mixed_step(zk_ctx* c, double dt);
int zk_weno_mixed_stage(zk_ctx* c, double dt, int stage);
