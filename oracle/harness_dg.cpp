// C entry points over the UNMODIFIED reference DG sources (src_DG/fluid.cpp and
// src_DG/solver.cpp, compiled once per DG_P_VAL in {1,2,3} with the Eigen/MPI
// shims in oracle/shim).  Test infrastructure: the checker for the GPU path.
//
// Array convention at this boundary (the same as the GPU library's C ABI):
//   dof    double[4][NM][ny][nx]  modal coefficients, variable c, mode
//                                 m = px*(P+1)+py (src_DG/fluid.cpp:63-65)
//   bct    int32[ny][nx]          bctype codes (0 fluid, -1 copy, 1 slip, -3 MPI ghost)
// Rows are y (row 0 = top), columns x; the Mesh itself is column-major.

#define main zk_reference_dg_main
#include "solver.cpp"
#undef main

#include <cstdint>
#include <thread>

// Defined in src_DG/fluid.cpp:525 without a declaration in fluid.h (the header
// declares the never-defined name hll3Flux instead, src_DG/fluid.h:179).
void hlleFlux(double UL0, double UL1, double UL2, double UL3, double UR0, double UR1, double UR2,
              double UR3, double gamma, double& F0, double& F1, double& F2, double& F3);

namespace {

Mesh make_mesh(int ny, int nx, double da, double gamma, const double* dof, const int* bct) {
    Mesh m(ny, nx, da, gamma);
    const size_t plane = static_cast<size_t>(ny) * nx;
    for (int c = 0; c < 4; ++c)
        for (int md = 0; md < DG_NM; ++md) {
            const double* src = dof + (static_cast<size_t>(c) * DG_NM + md) * plane;
            for (int i = 0; i < ny; ++i)
                for (int j = 0; j < nx; ++j) m.dof[c][md](i, j) = src[static_cast<size_t>(i) * nx + j];
        }
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) m.bctype(i, j) = bct[static_cast<size_t>(i) * nx + j];
    m.syncCellAverages();
    return m;
}

void store_dof(const Mesh& m, double* dof) {
    const int ny = m.ny, nx = m.nx;
    const size_t plane = static_cast<size_t>(ny) * nx;
    for (int c = 0; c < 4; ++c)
        for (int md = 0; md < DG_NM; ++md) {
            double* dst = dof + (static_cast<size_t>(c) * DG_NM + md) * plane;
            for (int i = 0; i < ny; ++i)
                for (int j = 0; j < nx; ++j) dst[static_cast<size_t>(i) * nx + j] = m.dof[c][md](i, j);
        }
}

// Periodic image of the 3-wide ring marked -3 (all modes), refilled before
// every computeRHS: the reference itself has no periodic boundary.
void fill_periodic(Mesh& m) {
    const int ny = m.ny, nx = m.nx, iy = ny - 6, ix = nx - 6;
    auto wrap = [](int k, int n) { return 3 + (((k - 3) % n) + n) % n; };
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            if (m.bctype(i, j) != -3) continue;
            const int si = wrap(i, iy), sj = wrap(j, ix);
            for (int c = 0; c < 4; ++c)
                for (int md = 0; md < DG_NM; ++md) m.dof[c][md](i, j) = m.dof[c][md](si, sj);
        }
}

// updateMesh (src_DG/fluid.cpp:1005-1054) with a periodic refill before each
// computeRHS.  At one rank exchangeConservativeColumns only syncs mode 0.
void update_mesh_periodic(Mesh& mesh, double dt) {
    const int ny = mesh.ny, nx = mesh.nx;
    vector<MatrixXd> dof_n[4];
    for (int c = 0; c < 4; ++c) {
        dof_n[c].resize(DG_NM);
        for (int md = 0; md < DG_NM; ++md) dof_n[c][md] = mesh.dof[c][md];
    }
    vector<MatrixXd> dU[4];
    for (int c = 0; c < 4; ++c) dU[c].resize(DG_NM, MatrixXd::Zero(ny, nx));

    fill_periodic(mesh);
    computeRHS(mesh, dt, dU);
    exchangeConservativeColumns(mesh, 0, 1);
    for (int c = 0; c < 4; ++c)
        for (int md = 0; md < DG_NM; ++md) mesh.dof[c][md] = dof_n[c][md] + dt * dU[c][md];
    applyLimiter(mesh);
    exchangeConservativeColumns(mesh, 0, 1);
    mesh.syncCellAverages();
    exchangeConservativeColumns(mesh, 0, 1);

    fill_periodic(mesh);
    computeRHS(mesh, dt, dU);
    exchangeConservativeColumns(mesh, 0, 1);
    for (int c = 0; c < 4; ++c)
        for (int md = 0; md < DG_NM; ++md)
            mesh.dof[c][md] = 0.75 * dof_n[c][md] + 0.25 * (mesh.dof[c][md] + dt * dU[c][md]);
    applyLimiter(mesh);
    exchangeConservativeColumns(mesh, 0, 1);
    mesh.syncCellAverages();
    exchangeConservativeColumns(mesh, 0, 1);

    fill_periodic(mesh);
    computeRHS(mesh, dt, dU);
    for (int c = 0; c < 4; ++c)
        for (int md = 0; md < DG_NM; ++md)
            mesh.dof[c][md] = (1.0 / 3.0) * dof_n[c][md] + (2.0 / 3.0) * (mesh.dof[c][md] + dt * dU[c][md]);
    exchangeConservativeColumns(mesh, 0, 1);
    applyLimiter(mesh);
    exchangeConservativeColumns(mesh, 0, 1);
    mesh.syncCellAverages();
    exchangeConservativeColumns(mesh, 0, 1);
}

}  // namespace

extern "C" {

// Timing emulation of the reference's MPI run with `nthreads` ranks: the grid
// is split into x-slabs by the reference's own splitMeshVertically
// (fluid.cpp), and each slab runs nsteps x updateMesh on its own thread.  With
// the single-rank MPI stub the 3-column halo exchange between slabs is a no-op
// (a memcpy of 3 columns in the real build), so the numbers are a throughput
// sample only.  Returns the wall time in ms of the slowest slab; *cells gets
// the number of cells the slabs update.
double refd_step_slabs_timed(int ny, int nx, double da, double gamma, const double* state,
                               const int* bct, double dt, int nsteps, int nthreads, long* cells) {
    Mesh full = make_mesh(ny, nx, da, gamma, state, bct);
    vector<Mesh> subs = splitMeshVertically(full, nthreads);
    long n = 0;
    for (auto& m : subs)
        for (int i = 3; i < m.ny - 3; ++i)
            for (int j = 3; j < m.nx - 3; ++j) n += (m.bctype(i, j) == 0);
    *cells = n;
    std::vector<double> ms(subs.size(), 0.0);
    std::vector<std::thread> th;
    for (size_t r = 0; r < subs.size(); ++r)
        th.emplace_back([&, r] {
            auto t0 = now();
            for (int s = 0; s < nsteps; ++s) updateMesh(subs[r], dt, 0, 1);
            ms[r] = elapsed_ms(t0, now());
        });
    for (auto& t : th) t.join();
    return *std::max_element(ms.begin(), ms.end());
}

int refd_order(void) { return DG_P; }

int refd_case_info(const char* dir, int* ny, int* nx, double* da, double* gamma) {
    try {
        Mesh m{std::string(dir)};
        *ny = m.ny; *nx = m.nx; *da = m.da; *gamma = m.gamma;
        return 0;
    } catch (...) { return 1; }
}

// Mesh(folder) + initDGModes (src_DG/fluid.cpp:216-244, :173-182).
int refd_load_case(const char* dir, double* dof, int* bct) {
    try {
        Mesh m{std::string(dir)};
        store_dof(m, dof);
        for (int i = 0; i < m.ny; ++i)
            for (int j = 0; j < m.nx; ++j) bct[static_cast<size_t>(i) * m.nx + j] = m.bctype(i, j);
        return 0;
    } catch (...) { return 1; }
}

// computeRHS (src_DG/fluid.cpp:656-807): ghost fill in place, dU = d(dof)/dt (no dt).
int refd_rhs(int ny, int nx, double da, double gamma, double* dof, const int* bct, double dt,
             double* dU) {
    Mesh m = make_mesh(ny, nx, da, gamma, dof, bct);
    vector<MatrixXd> d[4];
    for (int c = 0; c < 4; ++c) d[c].resize(DG_NM, MatrixXd::Zero(ny, nx));
    computeRHS(m, dt, d);
    store_dof(m, dof);
    const size_t plane = static_cast<size_t>(ny) * nx;
    for (int c = 0; c < 4; ++c)
        for (int md = 0; md < DG_NM; ++md) {
            double* dst = dU + (static_cast<size_t>(c) * DG_NM + md) * plane;
            for (int i = 0; i < ny; ++i)
                for (int j = 0; j < nx; ++j) dst[static_cast<size_t>(i) * nx + j] = d[c][md](i, j);
        }
    return 0;
}

// applyLimiter (src_DG/fluid.cpp:824-992), in place.
int refd_limit(int ny, int nx, double da, double gamma, double* dof, const int* bct) {
    Mesh m = make_mesh(ny, nx, da, gamma, dof, bct);
    applyLimiter(m);
    store_dof(m, dof);
    return 0;
}

// nsteps x updateMesh (src_DG/fluid.cpp:1005-1054) at one rank, fixed dt.
int refd_step(int ny, int nx, double da, double gamma, double* dof, const int* bct, double dt,
              int nsteps, int periodic) {
    Mesh m = make_mesh(ny, nx, da, gamma, dof, bct);
    for (int s = 0; s < nsteps; ++s) {
        if (periodic) update_mesh_periodic(m, dt);
        else updateMesh(m, dt, 0, 1);
    }
    store_dof(m, dof);
    return 0;
}

double refd_step_timed(int ny, int nx, double da, double gamma, double* dof, const int* bct,
                       double dt, int nsteps) {
    Mesh m = make_mesh(ny, nx, da, gamma, dof, bct);
    double ms = 0.0;
    for (int s = 0; s < nsteps; ++s) {
        auto t0 = now();
        updateMesh(m, dt, 0, 1);
        ms += elapsed_ms(t0, now());
    }
    store_dof(m, dof);
    return ms;
}

// computeMaxSpeedDG_omp (src_DG/solver.cpp:26-64).
double refd_max_speed(int ny, int nx, double da, double gamma, const double* dof, const int* bct) {
    Mesh m = make_mesh(ny, nx, da, gamma, dof, bct);
    return computeMaxSpeedDG_omp(m);
}

// dgSafeDt (src_DG/solver.cpp:19-23) and dgCFLLimit (:15-17).
double refd_safe_dt(double lambda_max, double h) { return dgSafeDt(lambda_max, h); }
double refd_cfl_limit(void) { return dgCFLLimit(); }

void refd_hllc(const double* UL, const double* UR, double gamma, double* F) {
    hllcFlux(UL[0], UL[1], UL[2], UL[3], UR[0], UR[1], UR[2], UR[3], gamma, F[0], F[1], F[2], F[3]);
}

void refd_hlle(const double* UL, const double* UR, double gamma, double* F) {
    hlleFlux(UL[0], UL[1], UL[2], UL[3], UR[0], UR[1], UR[2], UR[3], gamma, F[0], F[1], F[2], F[3]);
}

double refd_phi2(int m, double xi, double eta) { return phi2(m, xi, eta); }

}  // extern "C"
