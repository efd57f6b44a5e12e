/* CPU oracle for the Jacobi chares. TEST INFRASTRUCTURE ONLY: imported by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker or the timed CPU baseline; never part of the product path.
 *
 * Restates the arithmetic of the reference's Jacobi examples:
 *   2-D: examples/jacobi2d/jacobi2d.cu:327-334
 *        new[i][j] = (t[i][j] + t[i][j-1] + t[i][j+1] + t[i-1][j] + t[i+1][j]) * 0.2
 *        evaluated left to right in the grid's type, then one multiply by the
 *        double literal 0.2. Float grids (the reference has none): float
 *        sum s, then fmaf(s, C_HI, s * C_LO) with C_HI = 0.2f and C_LO the
 *        float nearest 0.2 - C_HI (the GPU's FP32 sweep does the same).
 *   1-D: examples/jacobi1d/jacobi1d.cu:160-170
 *        sum = 0; for j in -2..2: sum += t[i+j]; new[i] = sum / 5
 *   Residual (project-defined, the reference has none): r = S(u) - u with S
 *   evaluated in FP64 from the grid values; returns sum of r^2 in FP64.
 * Grids are row-major (ny+2) x (nx+2) with a fixed boundary ring.
 * Build with -O2 -ffp-contract=off (no fused multiply-add, no fast-math) so
 * the serial and OpenMP versions are bit-identical to each other and to the
 * GPU. Parity of the 2-D FP64 sweep is pinned against the reference's own
 * jacobi_2d_kernel (examples/jacobi-kernel/jacobi_kernel.cu:26-34) by the
 * fixtures in tests/golden/.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* One sweep in FP64 of rows [r0, r1) (1-based interior rows). */
static void sweep_rows_f64(const double* t, double* n, int nx, int r0, int r1) {
  const size_t w = (size_t)nx + 2;
  for (int i = r0; i < r1; i++) {
    const double* up = t + (size_t)(i - 1) * w;
    const double* c = t + (size_t)i * w;
    const double* dn = t + (size_t)(i + 1) * w;
    double* o = n + (size_t)i * w;
    for (int j = 1; j <= nx; j++) {
      o[j] = (c[j] + c[j - 1] + c[j + 1] + up[j] + dn[j]) * 0.2;
    }
  }
}

#define STENCIL_C_HI 0.2f                     /* 0x3e4ccccd */
#define STENCIL_C_LO (-2.9802322831784522e-09f)  /* 0xb14ccccd */

static void sweep_rows_f32(const float* t, float* n, int nx, int r0, int r1) {
  const size_t w = (size_t)nx + 2;
  for (int i = r0; i < r1; i++) {
    const float* up = t + (size_t)(i - 1) * w;
    const float* c = t + (size_t)i * w;
    const float* dn = t + (size_t)(i + 1) * w;
    float* o = n + (size_t)i * w;
    for (int j = 1; j <= nx; j++) {
      float s = c[j] + c[j - 1];
      s = s + c[j + 1];
      s = s + up[j];
      s = s + dn[j];
      const float lo = s * STENCIL_C_LO;
      o[j] = fmaf(s, STENCIL_C_HI, lo);
    }
  }
}

static void copy_ring_f64(const double* a, double* b, int nx, int ny) {
  const size_t w = (size_t)nx + 2;
  memcpy(b, a, w * sizeof(double));
  memcpy(b + (size_t)(ny + 1) * w, a + (size_t)(ny + 1) * w, w * sizeof(double));
  for (int i = 1; i <= ny; i++) {
    b[(size_t)i * w] = a[(size_t)i * w];
    b[(size_t)i * w + nx + 1] = a[(size_t)i * w + nx + 1];
  }
}

static void copy_ring_f32(const float* a, float* b, int nx, int ny) {
  const size_t w = (size_t)nx + 2;
  memcpy(b, a, w * sizeof(float));
  memcpy(b + (size_t)(ny + 1) * w, a + (size_t)(ny + 1) * w, w * sizeof(float));
  for (int i = 1; i <= ny; i++) {
    b[(size_t)i * w] = a[(size_t)i * w];
    b[(size_t)i * w + nx + 1] = a[(size_t)i * w + nx + 1];
  }
}

/* Serial FP64: `sweeps` Jacobi sweeps in place on grid (result in grid). */
int oracle_jacobi2d_f64(double* grid, int nx, int ny, int sweeps) {
  size_t n = ((size_t)nx + 2) * ((size_t)ny + 2);
  double* tmp = (double*)malloc(n * sizeof(double));
  if (!tmp) return -1;
  copy_ring_f64(grid, tmp, nx, ny);
  double* a = grid;
  double* b = tmp;
  for (int s = 0; s < sweeps; s++) {
    sweep_rows_f64(a, b, nx, 1, ny + 1);
    double* x = a; a = b; b = x;
  }
  if (a != grid) memcpy(grid, a, n * sizeof(double));
  free(tmp);
  return 0;
}

/* OpenMP FP64 (same arithmetic; rows split over threads). */
int oracle_jacobi2d_f64_omp(double* grid, int nx, int ny, int sweeps, int threads) {
  size_t n = ((size_t)nx + 2) * ((size_t)ny + 2);
  double* tmp = (double*)malloc(n * sizeof(double));
  if (!tmp) return -1;
  copy_ring_f64(grid, tmp, nx, ny);
  double* a = grid;
  double* b = tmp;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  for (int s = 0; s < sweeps; s++) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ny; i++) sweep_rows_f64(a, b, nx, i, i + 1);
    double* x = a; a = b; b = x;
  }
  if (a != grid) memcpy(grid, a, n * sizeof(double));
  free(tmp);
  return 0;
}

int oracle_jacobi2d_f32(float* grid, int nx, int ny, int sweeps, int threads) {
  size_t n = ((size_t)nx + 2) * ((size_t)ny + 2);
  float* tmp = (float*)malloc(n * sizeof(float));
  if (!tmp) return -1;
  copy_ring_f32(grid, tmp, nx, ny);
  float* a = grid;
  float* b = tmp;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  for (int s = 0; s < sweeps; s++) {
#pragma omp parallel for schedule(static) if (threads != 1)
    for (int i = 1; i <= ny; i++) sweep_rows_f32(a, b, nx, i, i + 1);
    float* x = a; a = b; b = x;
  }
  if (a != grid) memcpy(grid, a, n * sizeof(float));
  free(tmp);
  return 0;
}

/* Sum of (S(u) - u)^2 over the interior, S evaluated in FP64. */
double oracle_residual2_f64(const double* g, int nx, int ny) {
  const size_t w = (size_t)nx + 2;
  double acc = 0.0;
  for (int i = 1; i <= ny; i++) {
    for (int j = 1; j <= nx; j++) {
      size_t k = (size_t)i * w + j;
      double s = (g[k] + g[k - 1] + g[k + 1] + g[k - w] + g[k + w]) * 0.2;
      double r = s - g[k];
      acc += r * r;
    }
  }
  return acc;
}

double oracle_residual2_f32(const float* g, int nx, int ny) {
  const size_t w = (size_t)nx + 2;
  double acc = 0.0;
  for (int i = 1; i <= ny; i++) {
    for (int j = 1; j <= nx; j++) {
      size_t k = (size_t)i * w + j;
      double s = ((double)g[k] + (double)g[k - 1] + (double)g[k + 1] + (double)g[k - w] +
                  (double)g[k + w]) * 0.2;
      double r = s - (double)g[k];
      acc += r * r;
    }
  }
  return acc;
}

/* 1-D: array of width + 4 points (2 ghost points each side, fixed). */
int oracle_jacobi1d_f64(double* a0, int width, int sweeps) {
  size_t n = (size_t)width + 4;
  double* b = (double*)malloc(n * sizeof(double));
  if (!b) return -1;
  memcpy(b, a0, n * sizeof(double));
  double* a = a0;
  for (int s = 0; s < sweeps; s++) {
    for (size_t i = 2; i < (size_t)width + 2; i++) {
      double sum = 0;
      for (int j = -2; j <= 2; j++) sum += a[i + j];
      b[i] = sum / 5;
    }
    double* x = a; a = b; b = x;
  }
  if (a != a0) {
    memcpy(a0, a, n * sizeof(double));
    free(a);
  } else {
    free(b);
  }
  return 0;
}

/* ---- jacobi2d-decomp1d (examples/jacobi2d-decomp1d/jacobi2d.cu) ----------
 * Row decomposition of an ny x nx FP32 grid over n chares, restating
 * Block::init (:128-198): chunk_low = (ny-2)/n, chunk_high = chunk_low+1,
 * num_ranks_low = n*chunk_low + n - (ny-2); chare i has chunk rows (low for
 * i < num_ranks_low), iy_start_global as computed there, iy_end_global
 * clamped to ny-4, local rows 1..iy_end-1 computed, and periodic neighbours
 * top = i-1 (n-1 for chare 0), bottom = (i+1) % n. Each chare holds two
 * buffers of (chunk_high+2) x nx floats, zero except columns 0 and nx-1 of
 * its rows 1..chunk, which hold bc_rows[g] for the row's global index g
 * (the reference computes sin(2*PI*(g-1)/(ny-3)) on the device, :424-433;
 * the caller supplies the values). One iteration (jacobi_kernel, :374-383):
 *   new[iy][ix] = 0.25 * (a[iy][ix+1] + a[iy][ix-1] + a[iy+1][ix] + a[iy-1][ix])
 * in float, left to right, for ix in 1..nx-2; then the first computed row
 * goes to the top neighbour's bottom ghost row (its chunk+1) and the last
 * computed row to the bottom neighbour's row 0, columns 1..nx-2 (:386-401),
 * into the buffer the neighbour reads next (the reference always writes its
 * first buffer). out receives the chares' rows 1..chunk in order ((ny-2) x nx
 * floats) from the buffer of the last iteration. Returns 0, or -1 for sizes
 * the decomposition does not cover (chunk_low < 2, nx < 3). */
int oracle_decomp1d_f32(int n, int nx, int ny, int iters, const float* bc_rows, float* out) {
  if (n < 1 || nx < 3 || ny < 4 || iters < 0) return -1;
  const int low = (ny - 2) / n, high = low + 1;
  if (low < 2) return -1;
  const int n_low = n * low + n - (ny - 2);
  const size_t cnt = (size_t)nx * (high + 2);
  float* buf = (float*)calloc((size_t)n * 2 * cnt, sizeof(float));
  int* chunk = (int*)malloc(sizeof(int) * n);
  int* g0 = (int*)malloc(sizeof(int) * n);
  int* iend = (int*)malloc(sizeof(int) * n);
  if (!buf || !chunk || !g0 || !iend) {
    free(buf); free(chunk); free(g0); free(iend);
    return -1;
  }
  for (int i = 0; i < n; i++) {
    chunk[i] = i < n_low ? low : high;
    g0[i] = i < n_low ? i * low + 1 : n_low * low + (i - n_low) * high + 1;
    int gend = g0[i] + chunk[i] - 1;
    if (gend > ny - 4) gend = ny - 4;
    iend[i] = (gend - g0[i] + 1) + 1;
    for (int b = 0; b < 2; b++) {
      float* a = buf + ((size_t)i * 2 + b) * cnt;
      for (int r = 1; r <= chunk[i]; r++) {
        const float v = bc_rows[g0[i] + r - 1];
        a[(size_t)r * nx] = v;
        a[(size_t)r * nx + nx - 1] = v;
      }
    }
  }
  for (int k = 0; k < iters; k++) {
    for (int i = 0; i < n; i++) {
      const float* a = buf + ((size_t)i * 2 + (k & 1)) * cnt;
      float* o = buf + ((size_t)i * 2 + ((k + 1) & 1)) * cnt;
      for (int iy = 1; iy < iend[i]; iy++)
        for (int ix = 1; ix < nx - 1; ix++) {
          float s = a[(size_t)iy * nx + ix + 1] + a[(size_t)iy * nx + ix - 1];
          s = s + a[(size_t)(iy + 1) * nx + ix];
          s = s + a[(size_t)(iy - 1) * nx + ix];
          o[(size_t)iy * nx + ix] = (float)(0.25 * (double)s);
        }
    }
    for (int i = 0; i < n; i++) {
      const int top = i > 0 ? i - 1 : n - 1, bot = (i + 1) % n;
      const float* o = buf + ((size_t)i * 2 + ((k + 1) & 1)) * cnt;
      float* t = buf + ((size_t)top * 2 + ((k + 1) & 1)) * cnt;
      float* b = buf + ((size_t)bot * 2 + ((k + 1) & 1)) * cnt;
      memcpy(t + (size_t)(chunk[top] + 1) * nx + 1, o + (size_t)1 * nx + 1, sizeof(float) * (nx - 2));
      memcpy(b + 1, o + (size_t)(iend[i] - 1) * nx + 1, sizeof(float) * (nx - 2));
    }
  }
  size_t row = 0;
  for (int i = 0; i < n; i++) {
    const float* a = buf + ((size_t)i * 2 + (iters & 1)) * cnt;
    for (int r = 1; r <= chunk[i]; r++, row++) memcpy(out + row * nx, a + (size_t)r * nx, sizeof(float) * nx);
  }
  free(buf); free(chunk); free(g0); free(iend);
  return 0;
}

/* ---- 3-D (examples/jacobi-kernel/jacobi_kernel.cu:36-48) -----------------
 * One sweep of the 7-point stencil over the interior of an (nz+2) x (ny+2) x
 * (nx+2) FP64 grid, x fastest (IDX_3D, jacobi_kernel.h:7):
 *   new = (c + x-1 + x+1 + y-1 + y+1 + z-1 + z+1) * 0.142857
 * added left to right, one multiply by the double literal (DIVIDEBY7, :16).
 * `sweeps` sweeps alternate between two buffers; threads > 1 splits the z
 * planes over OpenMP threads (bit-identical to the serial order). */
static void sweep3d_planes(const double* t, double* o, int nx, int ny, int z0, int z1) {
  const size_t sy = (size_t)nx + 2, sz = sy * ((size_t)ny + 2);
  for (int k = z0; k < z1; k++)
    for (int j = 1; j <= ny; j++) {
      const double* c = t + (size_t)k * sz + (size_t)j * sy;
      double* w = o + (size_t)k * sz + (size_t)j * sy;
      for (int i = 1; i <= nx; i++)
        w[i] = (c[i] + c[i - 1] + c[i + 1] + c[i - sy] + c[i + sy] + c[i - sz] + c[i + sz]) * 0.142857;
    }
}

int oracle_jacobi3d_f64(double* grid, int nx, int ny, int nz, int sweeps, int threads) {
  const size_t n = ((size_t)nx + 2) * ((size_t)ny + 2) * ((size_t)nz + 2);
  double* b = (double*)malloc(n * sizeof(double));
  if (!b) return -1;
  memcpy(b, grid, n * sizeof(double));
  double *a = grid, *o = b;
  for (int s = 0; s < sweeps; s++) {
#ifdef _OPENMP
    if (threads > 1) {
#pragma omp parallel for num_threads(threads) schedule(static)
      for (int k = 1; k <= nz; k++) sweep3d_planes(a, o, nx, ny, k, k + 1);
    } else
#endif
      sweep3d_planes(a, o, nx, ny, 1, nz + 1);
    double* t = a; a = o; o = t;
  }
  if (a != grid) memcpy(grid, a, n * sizeof(double));
  free(b);
  return 0;
}
