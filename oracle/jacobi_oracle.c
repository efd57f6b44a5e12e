/* CPU oracle for the Jacobi chares. TEST INFRASTRUCTURE ONLY: imported by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker or the timed CPU baseline; never part of the product path.
 *
 * Restates the arithmetic of the reference's Jacobi examples:
 *   2-D: examples/jacobi2d/jacobi2d.cu:327-334
 *        new[i][j] = (t[i][j] + t[i][j-1] + t[i][j+1] + t[i-1][j] + t[i+1][j]) * 0.2
 *        evaluated left to right in the grid's type, then one multiply by the
 *        double literal 0.2 (for float grids: float sum, double multiply,
 *        rounded to float on store, as C/C++ promotion gives).
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
      o[j] = (float)((double)s * 0.2);
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
