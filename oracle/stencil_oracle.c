/*
 * CPU oracle for the fused DFT-tile stencil path.  TEST INFRASTRUCTURE ONLY:
 * tests/, the smoke check and the bench's cpu_baseline leg call this library
 * as the checker; the product path (libffs.so) never links or calls it.
 *
 * It restates the reference's CPU stencils as a direct FP64 time-stepping loop:
 *   - src/1D/check_correct.hpp:15-38   stencil1D  (periodic, single step, serial)
 *   - src/2D/check_correct.hpp:53-61   getElement (periodic wrap)
 *   - src/2D/check_correct.hpp:64-100  stencil2D  (periodic, single step, OpenMP,
 *                                       output written shifted by +K/2)
 * and extends them in the ways the stencil solver needs:
 *   - centred correlation out[i] = sum_k w[k] * in[i + k - r] (the +K/2 output
 *     shift of stencil2D is removed; the reference feeds stencil2D a kernel it
 *     first rotates by 180 degrees, src/2D/check_correct.hpp:17-33, so its GPU
 *     path is a convolution with the unrotated weights - the same thing),
 *   - a third dimension (the reference has no 3D CPU stencil),
 *   - a "fixed" boundary: every cell within r of a face (the ring/shell of
 *     width r) keeps its initial value; all other cells are updated,
 *   - a T-step driver that feeds the output of step t into step t+1.
 *
 * Parity is pinned by tests/golden (fixtures produced by the unmodified
 * reference functions compiled from the reference sources by oracle/Makefile)
 * and by the known-answer cases the reference's own code produces.
 *
 * Layout: row-major with x fastest: idx = (z * ny + y) * nx + x.
 * Weights: dense (2r+1)^dim array, dx fastest: w[((dz+r)*K + (dy+r))*K + (dx+r)].
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FFS_ORACLE_PERIODIC 0
#define FFS_ORACLE_FIXED 1

static inline int64_t wrap_index(int64_t i, int64_t n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

/* One time step.  Returns 0 on success, non-zero on a bad argument. */
int ffs_oracle_step(int dim, int64_t nx, int64_t ny, int64_t nz, int r,
                    const double *w, int boundary, const double *in, double *out)
{
    if (dim < 1 || dim > 3 || r < 0 || nx < 1 || ny < 1 || nz < 1 || !w || !in || !out)
        return 1;
    if (in == out)
        return 1;
    const int K = 2 * r + 1;
    const int ry = dim >= 2 ? r : 0;
    const int rz = dim >= 3 ? r : 0;
    const int Ky = 2 * ry + 1;
    /* indices of non-zero taps, so star shapes skip their zero corners */
    int ntap = 0;
    int *tdx = (int *)malloc(sizeof(int) * K * K * K);
    int *tdy = (int *)malloc(sizeof(int) * K * K * K);
    int *tdz = (int *)malloc(sizeof(int) * K * K * K);
    double *tw = (double *)malloc(sizeof(double) * K * K * K);
    for (int dz = -rz; dz <= rz; ++dz)
        for (int dy = -ry; dy <= ry; ++dy)
            for (int dx = -r; dx <= r; ++dx) {
                double v = w[((dz + rz) * Ky + (dy + ry)) * K + (dx + r)];
                if (v != 0.0) {
                    tdx[ntap] = dx; tdy[ntap] = dy; tdz[ntap] = dz; tw[ntap] = v; ++ntap;
                }
            }
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y) {
            const int64_t row = (z * ny + y) * nx;
            const int zfix = rz > 0 && (z < rz || z >= nz - rz);
            const int yfix = ry > 0 && (y < ry || y >= ny - ry);
            for (int64_t x = 0; x < nx; ++x) {
                if (boundary == FFS_ORACLE_FIXED) {
                    if (zfix || yfix || (r > 0 && (x < r || x >= nx - r))) {
                        out[row + x] = in[row + x];
                        continue;
                    }
                    double s = 0.0;
                    for (int t = 0; t < ntap; ++t)
                        s += tw[t] * in[((z + tdz[t]) * ny + (y + tdy[t])) * nx + (x + tdx[t])];
                    out[row + x] = s;
                } else {
                    double s = 0.0;
                    for (int t = 0; t < ntap; ++t) {
                        int64_t zz = wrap_index(z + tdz[t], nz);
                        int64_t yy = wrap_index(y + tdy[t], ny);
                        int64_t xx = wrap_index(x + tdx[t], nx);
                        s += tw[t] * in[(zz * ny + yy) * nx + xx];
                    }
                    out[row + x] = s;
                }
            }
        }
    free(tdx); free(tdy); free(tdz); free(tw);
    return 0;
}

/* T time steps, out = S^T(in).  in and out must not alias. */
int ffs_oracle_run(int dim, int64_t nx, int64_t ny, int64_t nz, int r,
                   const double *w, int boundary, int T, const double *in, double *out)
{
    if (T < 0 || in == out)
        return 1;
    const int64_t n = nx * ny * nz;
    if (T == 0) {
        memcpy(out, in, sizeof(double) * n);
        return 0;
    }
    double *tmp = T > 1 ? (double *)malloc(sizeof(double) * n) : NULL;
    if (T > 1 && !tmp)
        return 2;
    /* ping-pong so that the final step lands in out */
    const double *src = in;
    for (int t = 0; t < T; ++t) {
        int remaining = T - t; /* steps left including this one */
        double *dst = (remaining % 2 == 1) ? out : tmp;
        int rc = ffs_oracle_step(dim, nx, ny, nz, r, w, boundary, src, dst);
        if (rc) {
            free(tmp);
            return rc;
        }
        src = dst;
    }
    free(tmp);
    return 0;
}

int ffs_oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ffs_oracle_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#else
    (void)n;
#endif
}
