// TVB limiter pass of the DG path (Cockburn-Shu TVB minmod with characteristic
// decomposition; no reference implementation -- the reference documents this
// design for its DG limiter at src_DG/fluid.h:140-147 but ships a Persson +
// Zhang-Shu limiter instead), the troubled-cell features of the learned
// indicator, and the indicator-gated variant.
//
// One thread per cell, in place on the stage output: a cell reads its own
// linear modes and the MEANS of its four neighbours (through the ghost map);
// means are never modified, so the sweep is race-free in place.  Compiled with
// --fmad=false: the FP64 instantiation is bit-identical to the oracle's C
// restatement (oracle/dg_oracle.c: limit_tvb_all).
#include "dg_common.cuh"
#include "zk_internal.h"
#include "zk_mlp.h"

namespace zk {
namespace {

template <typename T>
__device__ __forceinline__ T tmin_(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T tmax_(T a, T b) { return (a < b) ? b : a; }

template <typename T>
__device__ __forceinline__ T tvb_minmod(T a, T b, T c, T mh2) {
    if (fabs(a) <= mh2) return a;
    if (a > T(0) && b > T(0) && c > T(0)) return tmin_(a, tmin_(b, c));
    if (a < T(0) && b < T(0) && c < T(0)) return tmax_(a, tmax_(b, c));
    return T(0);
}

// Euler eigenvectors in direction dir at conserved state u (oracle:
// od_euler_eigen); false for a non-physical state.
template <typename T>
__device__ __forceinline__ bool euler_eigen(const T u[4], T gamma, int dir, T L[4][4], T R[4][4]) {
    const T rho = u[0];
    if (!(rho > T(0))) return false;
    const T vx = u[1] / rho, vy = u[2] / rho;
    const T q2 = vx * vx + vy * vy;
    const T p = (gamma - T(1)) * (u[3] - T(0.5) * rho * q2);
    if (!(p > T(0))) return false;
    const T c = sqrt(gamma * p / rho);
    const T H = (u[3] + p) / rho;
    const T b1 = (gamma - T(1)) / (c * c), b2 = T(0.5) * q2 * b1;
    const T un = dir == 0 ? vx : vy, ut = dir == 0 ? vy : vx;
    const int in = dir == 0 ? 1 : 2, it = dir == 0 ? 2 : 1;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int k = 0; k < 4; ++k) L[r][k] = R[r][k] = T(0);
    R[0][0] = T(1); R[in][0] = un - c; R[it][0] = ut; R[3][0] = H - un * c;
    R[0][1] = T(1); R[in][1] = un;     R[it][1] = ut; R[3][1] = T(0.5) * q2;
    R[0][2] = T(0); R[in][2] = T(0);   R[it][2] = T(1); R[3][2] = ut;
    R[0][3] = T(1); R[in][3] = un + c; R[it][3] = ut; R[3][3] = H + un * c;
    L[0][0] = T(0.5) * (b2 + un / c); L[0][in] = -T(0.5) * (b1 * un + T(1) / c); L[0][it] = -T(0.5) * b1 * ut; L[0][3] = T(0.5) * b1;
    L[1][0] = T(1) - b2;              L[1][in] = b1 * un;                        L[1][it] = b1 * ut;             L[1][3] = -b1;
    L[2][0] = -ut;                    L[2][in] = T(0);                           L[2][it] = T(1);                L[2][3] = T(0);
    L[3][0] = T(0.5) * (b2 - un / c); L[3][in] = -T(0.5) * (b1 * un - T(1) / c); L[3][it] = -T(0.5) * b1 * ut; L[3][3] = T(0.5) * b1;
    return true;
}

template <typename T>
__device__ __forceinline__ bool tvb_dir(const T ub[4], T gamma, int dir, T mh2, const T a[4], const T dp[4],
                                        const T dm[4], T out[4]) {
    T L[4][4], R[4][4];
    const bool phys = euler_eigen<T>(ub, gamma, dir, L, R);
    T w[4], wl[4];
    bool changed = false;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        T wp, wm;
        if (phys) {
            w[r] = L[r][0] * a[0] + L[r][1] * a[1] + L[r][2] * a[2] + L[r][3] * a[3];
            wp = L[r][0] * dp[0] + L[r][1] * dp[1] + L[r][2] * dp[2] + L[r][3] * dp[3];
            wm = L[r][0] * dm[0] + L[r][1] * dm[1] + L[r][2] * dm[2] + L[r][3] * dm[3];
        } else {
            w[r] = a[r]; wp = dp[r]; wm = dm[r];
        }
        wl[r] = tvb_minmod<T>(w[r], wp, wm, mh2);
        if (wl[r] != w[r]) changed = true;
    }
    if (!changed) return false;
#pragma unroll
    for (int r = 0; r < 4; ++r)
        out[r] = phys ? R[r][0] * wl[0] + R[r][1] * wl[1] + R[r][2] * wl[2] + R[r][3] * wl[3] : wl[r];
    return true;
}

// Mean of the cell at k, gathered through the fill map.
template <typename T>
__device__ __forceinline__ void nb_mean(const T* d, const int8_t* kind, const int32_t* gsrc, size_t k, size_t vs,
                                        T out[4]) {
    const int8_t kd = kind[k] & KIND_MASK;
    size_t s = k;
    int neg = -1;
    if (kd >= KIND_COPY) {
        s = (size_t)gsrc[k];
        neg = kd == KIND_SLIP_X ? 1 : (kd == KIND_SLIP_Y ? 2 : -1);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const T v = d[(size_t)c * vs + s];
        out[c] = (neg == c) ? -v : v;
    }
}

struct TvbArgs {
    void* state;       // T planes [4][NM][ny][pitch]
    const int8_t* kind;
    const int32_t* gsrc;
    Grid g;
    double da, gamma, M;
    uint8_t* flags;    // per cell (pitched), may be null
    const MlpWeights* mlp;  // non-null: only cells the indicator flags are limited
    float* features;   // features mode: [ncell][40] output, no limiting
    uint32_t* nflag;   // count of limited cells, may be null
};

template <typename T, int P>
__global__ void __launch_bounds__(128) tvb_kernel(TvbArgs a) {
    constexpr int NM = (P + 1) * (P + 1);
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= a.g.nx || i >= a.g.ny) return;
    const size_t k = (size_t)i * a.g.pitch + j, plane = a.g.plane, vs = (size_t)NM * plane;
    T* d = static_cast<T*>(a.state);
    if (a.flags) a.flags[k] = 0;
    if ((a.kind[k] & KIND_MASK) != KIND_UPDATED) return;
    const int nx = a.g.nx;
    T ub[4], uL[4], uR[4], uU[4], uD[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) ub[c] = d[(size_t)c * vs + k];
    nb_mean<T>(d, a.kind, a.gsrc, k - 1, vs, uL);
    nb_mean<T>(d, a.kind, a.gsrc, k + 1, vs, uR);
    nb_mean<T>(d, a.kind, a.gsrc, k - (size_t)a.g.pitch, vs, uU);
    nb_mean<T>(d, a.kind, a.gsrc, k + (size_t)a.g.pitch, vs, uD);
    (void)nx;
    if (a.features || a.mlp) {
        float f[MLP_IN];
        // rho and E modes, slot px*4+py, scaled by the largest |mean| around
        const float sr = (float)tmax_(tmax_(tmax_(fabs(ub[0]), fabs(uL[0])), tmax_(fabs(uR[0]), fabs(uU[0]))),
                                      fabs(uD[0])) + 1e-12f;
        const float se = (float)tmax_(tmax_(tmax_(fabs(ub[3]), fabs(uL[3])), tmax_(fabs(uR[3]), fabs(uU[3]))),
                                      fabs(uD[3])) + 1e-12f;
#pragma unroll
        for (int s = 0; s < 16; ++s) { f[s] = 0.0f; f[16 + s] = 0.0f; }
#pragma unroll
        for (int m = 0; m < NM; ++m) {
            const int slot = (m / (P + 1)) * 4 + m % (P + 1);
            f[slot] = (float)d[(size_t)m * plane + k] / sr;
            f[16 + slot] = (float)d[3 * vs + (size_t)m * plane + k] / se;
        }
        const T* nb[4] = {uL, uR, uU, uD};
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            f[32 + n] = (float)(nb[n][0] - ub[0]) / sr;
            f[36 + n] = (float)(nb[n][3] - ub[3]) / se;
        }
        if (a.features) {
            const size_t cell = (size_t)i * a.g.nx + j;
#pragma unroll
            for (int s = 0; s < MLP_IN; ++s) a.features[cell * MLP_IN + s] = f[s];
        } else if (mlp_logit(*a.mlp, f) <= 0.0f) {
            return;  // indicator says smooth: skip the characteristic branch
        }
    }
    const T mh2 = T(a.M) * T(a.da) * T(a.da);
    T ax[4], ay[4], dxp[4], dxm[4], dyp[4], dym[4], lx[4], ly[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        ax[c] = d[(size_t)c * vs + (size_t)(P + 1) * plane + k];
        ay[c] = d[(size_t)c * vs + plane + k];
        dxp[c] = uR[c] - ub[c];
        dxm[c] = ub[c] - uL[c];
        dyp[c] = uD[c] - ub[c];  // eta grows with the row index
        dym[c] = ub[c] - uU[c];
    }
    const bool tx = tvb_dir<T>(ub, T(a.gamma), 0, mh2, ax, dxp, dxm, lx);
    const bool ty = tvb_dir<T>(ub, T(a.gamma), 1, mh2, ay, dyp, dym, ly);
    if (!(tx || ty)) return;
    if (a.flags) a.flags[k] = 1;
    if (a.features) return;  // features mode labels only
    if (a.nflag) atomicAdd(a.nflag, 1u);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (tx) d[(size_t)c * vs + (size_t)(P + 1) * plane + k] = lx[c];
        if (ty) d[(size_t)c * vs + plane + k] = ly[c];
#pragma unroll
        for (int m = 0; m < NM; ++m)
            if (m / (P + 1) + m % (P + 1) > 1) d[(size_t)c * vs + (size_t)m * plane + k] = T(0);
    }
}

template <typename T>
cudaError_t launch_t(int P, const TvbArgs& a, cudaStream_t s) {
    dim3 grid((a.g.nx + 127) / 128, a.g.ny);
    switch (P) {
        case 1: tvb_kernel<T, 1><<<grid, 128, 0, s>>>(a); break;
        case 2: tvb_kernel<T, 2><<<grid, 128, 0, s>>>(a); break;
        case 3: tvb_kernel<T, 3><<<grid, 128, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dg_tvb(int P, void* state, bool fp64, const int8_t* kind, const int32_t* gsrc, const Grid& g,
                          double da, double gamma, double M, uint8_t* flags, const MlpWeights* mlp,
                          float* features, uint32_t* nflag, cudaStream_t s) {
    TvbArgs a{state, kind, gsrc, g, da, gamma, M, flags, mlp, features, nflag};
    return fp64 ? launch_t<double>(P, a, s) : launch_t<float>(P, a, s);
}

}  // namespace zk
