// GPU backend for the reference DG solver (src_DG, DG_P_VAL = 1..3): the
// fluid.h hot-path functions defined on top of the C ABI (include/zuikaku.h),
// so the reference's own solver.cpp runs its loop on a B200 unchanged.
//
// Replaced (src_DG/fluid.h): computeRHS (:137-138), applyLimiter (:147),
// updateMesh (:160).  Build: compile the reference fluid.cpp with those names
// renamed to zk_ref_<name>, then link solver.cpp unchanged, this file and
// libzuikaku.so (oracle/Makefile target `dropin`).
//
// The reference driver's CFL check (computeMaxSpeedDG_omp, file-static in
// src_DG/solver.cpp:26) reads mesh.dof on the host, so after every step the
// modes are copied back and the cell averages synced (Mesh::syncCellAverages,
// as the reference's updateMesh ends).  One rank owns the whole grid.
// ZK_PRECISION=mixed selects the mixed-precision path (default FP64);
// ZK_DEVICE picks the GPU.
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "fluid.h"
#include "zuikaku.h"

namespace {

struct Backend {
    zk_ctx* ctx = nullptr;
    const Mesh* bound = nullptr;
    std::vector<double> buf;
    ~Backend() {
        if (ctx) zk_destroy(ctx);
    }
} g;

void check(int rc) {
    if (rc != ZK_OK) throw std::runtime_error(std::string("zuikaku: ") + zk_last_error());
}

// dof[c][m] (Eigen, column-major) <-> ABI [c][m][ny][nx]
void pack(const Mesh& m) {
    const size_t plane = (size_t)m.ny * m.nx;
    g.buf.resize((size_t)4 * DG_NM * plane);
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < DG_NM; ++k)
            for (int i = 0; i < m.ny; ++i)
                for (int j = 0; j < m.nx; ++j)
                    g.buf[((size_t)c * DG_NM + k) * plane + (size_t)i * m.nx + j] = m.dof[c][k](i, j);
}

void unpack(Mesh& m) {
    const size_t plane = (size_t)m.ny * m.nx;
    for (int c = 0; c < 4; ++c)
        for (int k = 0; k < DG_NM; ++k)
            for (int i = 0; i < m.ny; ++i)
                for (int j = 0; j < m.nx; ++j)
                    m.dof[c][k](i, j) = g.buf[((size_t)c * DG_NM + k) * plane + (size_t)i * m.nx + j];
}

void bind(const Mesh& m) {
    if (g.bound == &m) return;
    if (!g.ctx) {
        zk_options o;
        zk_default_options(&o);
        o.method = ZK_METHOD_DG;
        o.order = DG_P;
        const char* p = std::getenv("ZK_PRECISION");
        if (p && std::string(p) == "mixed") o.precision = ZK_PREC_MIXED;
        if (const char* d = std::getenv("ZK_DEVICE")) o.device = std::atoi(d);
        check(zk_create(&o, &g.ctx));
    }
    std::vector<int32_t> bct((size_t)m.ny * m.nx);
    for (int i = 0; i < m.ny; ++i)
        for (int j = 0; j < m.nx; ++j) bct[(size_t)i * m.nx + j] = m.bctype(i, j);
    check(zk_set_mesh(g.ctx, m.ny, m.nx, m.da, m.gamma, bct.data()));
    g.bound = &m;
}

// Upload the host modes, run `op` on the device state, bring the modes back.
template <typename Op>
void on_device(Mesh& m, Op op) {
    bind(m);
    pack(m);
    check(zk_set_state(g.ctx, g.buf.data()));
    op();
    check(zk_get_state(g.ctx, g.buf.data()));
    unpack(m);
}

}  // namespace

void updateMesh(Mesh& mesh, double dt, int rank, int num_procs) {
    (void)rank;
    if (num_procs != 1) throw std::runtime_error("zuikaku: one GPU rank owns the whole grid (num_procs must be 1)");
    on_device(mesh, [&] { check(zk_step(g.ctx, dt, 1)); });
    mesh.syncCellAverages();
}

void computeRHS(Mesh& mesh, double dt, vector<MatrixXd> dU[4]) {
    const size_t plane = (size_t)mesh.ny * mesh.nx;
    std::vector<double> d((size_t)4 * DG_NM * plane);
    on_device(mesh, [&] { check(zk_rhs(g.ctx, dt, d.data())); });  // ghosts filled in place, as the reference
    for (int c = 0; c < 4; ++c) {
        dU[c].assign(DG_NM, MatrixXd::Zero(mesh.ny, mesh.nx));
        for (int k = 0; k < DG_NM; ++k)
            for (int i = 0; i < mesh.ny; ++i)
                for (int j = 0; j < mesh.nx; ++j)
                    dU[c][k](i, j) = d[((size_t)c * DG_NM + k) * plane + (size_t)i * mesh.nx + j];
    }
}

void applyLimiter(Mesh& mesh) {
    on_device(mesh, [&] { check(zk_limit(g.ctx)); });
}
