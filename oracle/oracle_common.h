/* Shared helpers of the CPU oracle (a C restatement of ZuikakuCFD's hot path).
 * TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the CPU-baseline
 * legs of bench.py load it, as the checker.  The product never does.
 *
 * Array convention: row-major planes, row i = y index (row 0 = top), column j = x.
 *   WENO state  U[4][ny][nx];  DG state dof[4][NM][ny][nx];  bct int32[ny][nx]. */
#ifndef ZK_ORACLE_COMMON_H
#define ZK_ORACLE_COMMON_H

#include <stddef.h>
#include <math.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* std::max / std::min as the reference calls them: std::max(a,b) returns
 * (a<b)?b:a and std::min(a,b) returns (b<a)?b:a, so a NaN first argument is
 * passed through unchanged (unlike fmax). */
static inline double zk_max(double a, double b) { return (a < b) ? b : a; }
static inline double zk_min(double a, double b) { return (b < a) ? b : a; }

/* Cell kinds of the ghost source map (shared meaning with the GPU library). */
enum {
    ZK_CELL_UPDATED = 0,  /* bctype 0 inside [3,ny-3)x[3,nx-3): receives dU      */
    ZK_CELL_PASSIVE = 1,  /* never written by the fill, dU = 0                   */
    ZK_CELL_COPY = 2,     /* filled with a copy of src before every RHS          */
    ZK_CELL_SLIP_X = 3,   /* DG slip wall, x normal: copy with rho*u negated     */
    ZK_CELL_SLIP_Y = 4    /* DG slip wall, y normal: copy with rho*v negated     */
};

/* Ghost source map.  The reference fills ghosts with two serial sweeps over the
 * fluid cells (src_WENO/fluid.cpp:338-370, src_DG/fluid.cpp:581-635): a row
 * sweep writing (i+dk, j), then a column sweep writing (i, j+dk), dk in
 * {-3..3}\{0}.  Sources are fluid cells, which are never written, so the fill is
 * a gather; the LAST writer in loop order wins: the largest source column of
 * the column sweep if there is one, else the largest source row of the row
 * sweep.  Ghosts no sweep reaches (the corners) keep their value.
 *
 * with_slip: bctype 1 cells are slip walls (DG only); periodic: bctype -3 cells
 * take their periodic image inside the 3-wide ring (a harness-side boundary:
 * the reference leaves -3 cells to MPI).
 * Writes kind[ny*nx] (ZK_CELL_*) and src[ny*nx] (-1 where no fill). */
static inline void zk_ghost_map(int ny, int nx, const int* bct, int with_slip, int periodic,
                                signed char* kind, int* src) {
    for (int i = 0; i < ny; ++i)
        for (int j = 0; j < nx; ++j) {
            const size_t k = (size_t)i * nx + j;
            const int b = bct[k];
            src[k] = -1;
            kind[k] = (b == 0 && i >= 3 && i < ny - 3 && j >= 3 && j < nx - 3) ? ZK_CELL_UPDATED
                                                                                 : ZK_CELL_PASSIVE;
            if (periodic && b == -3) {
                const int iy = ny - 6, ix = nx - 6;
                const int si = 3 + (((i - 3) % iy) + iy) % iy;
                const int sj = 3 + (((j - 3) % ix) + ix) % ix;
                src[k] = si * nx + sj;
                kind[k] = ZK_CELL_COPY;
                continue;
            }
            if (!(b == -1 || (with_slip && b == 1))) continue;
            /* column sweep (runs second, so it wins): sources (i, jj), i in range */
            int best = -1;
            if (i >= 3 && i < ny - 3)
                for (int jj = j - 3; jj <= j + 3; ++jj) {
                    if (jj == j || jj < 3 || jj >= nx - 3) continue;
                    if (bct[(size_t)i * nx + jj] == 0) best = jj;
                }
            if (best >= 0) {
                src[k] = i * nx + best;
                kind[k] = (b == 1) ? ZK_CELL_SLIP_X : ZK_CELL_COPY;
                continue;
            }
            /* row sweep: sources (ii, j), j in range */
            if (j >= 3 && j < nx - 3)
                for (int ii = i - 3; ii <= i + 3; ++ii) {
                    if (ii == i || ii < 3 || ii >= ny - 3) continue;
                    if (bct[(size_t)ii * nx + j] == 0) best = ii;
                }
            if (best >= 0) {
                src[k] = best * nx + j;
                kind[k] = (b == 1) ? ZK_CELL_SLIP_Y : ZK_CELL_COPY;
            }
        }
}

#endif
