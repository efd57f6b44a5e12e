// 3-D Jacobi sweeps (7-point, FP64): the stencil of the reference's
// standalone kernel, examples/jacobi-kernel/jacobi_kernel.cu:36-48,
//   new[i][j][k] = (t + t[i-1] + t[i+1] + t[j-1] + t[j+1] + t[k-1] + t[k+1])
//                  * 0.142857
// added left to right in FP64, then one multiply by the double literal
// 0.142857 (DIVIDEBY7 there, :16). Grid layout as its IDX_3D: x fastest,
// (nx+2) x (ny+2) x (nz+2) doubles with a fixed boundary shell. Unlike the
// reference's benchmark loop (which launches temp -> new_temp every time),
// sweeps alternate between two buffers, so the result is `sweeps` Jacobi
// iterations.
//
// Two kernels, the same arithmetic. Each block owns a 32 x 16 tile of (x, y)
// columns and a run of z planes and marches up z.
//   jacobi3d_async_kernel (grids of at least one 34 x 18 box in x and y):
//     the tile's planes, rim included, stream through a ring of J3_S
//     shared-memory slots by per-thread asynchronous copies (cp.async, one
//     commit group per plane), J3_S - 2 planes ahead of the one computed
//     (J3_S = 10 by default; 256 threads, two tile rows each).
//     Each input value is read from DRAM once per sweep (16 B per lattice
//     update with the store); the rim cells come from L2.
//   jacobi3d_kernel (any shape): per-thread loads, the planes below and
//     above a thread's cell and one more in registers, the current plane
//     with its rim in shared memory.
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION
#include "jacobi_sweep.cuh"
#include "../host.cuh"
#include <cmath>
#include <cstdlib>

namespace {

constexpr int J3_TX = 32, J3_TY = 16;
constexpr int J3_BW = J3_TX + 2, J3_BH = J3_TY + 2;          // tensor box: tile + rim
// 10 slots and 2 tile rows per thread: 293 GLUP/s at 640^3, against 265
// with 8 slots and one row, 282 with 12 slots and two rows
constexpr int J3_S_DEFAULT = 10;                             // plane slots
constexpr int J3_RPT_DEFAULT = 2;                            // tile rows per thread

__device__ __forceinline__ double j3_stencil(double c, double xm, double xp, double ym, double yp, double zm,
    double zp) {
  return __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(c, xm), xp), ym), yp), zm), zp),
                   0.142857);
}

// Planes z0-1 .. z1 of the tile stream through J3_S shared-memory slots:
// plane p lives in slot (p - z0 + 1) % J3_S, one cp.async group per plane
// (8-byte copies of the 34 x 18 box: the tile and its rim; cells outside the
// grid are zero-filled and never used). Before output plane z is computed,
// planes up to z + J3_S - 2 are issued and wait_group leaves J3_S - 3 of
// them in flight, so planes z-1, z, z+1 have landed. The block has
// 32 x (16 / RPT) threads; each computes RPT rows of the tile.
template <int J3_S, int RPT>
__global__ void __launch_bounds__(J3_TX * J3_TY / RPT, 3 * RPT) jacobi3d_async_kernel(
    const double* __restrict__ in, double* __restrict__ out, int nx, int ny, int nz, int zrun) {
  extern __shared__ __align__(16) double j3_slots[];  // [J3_S][J3_BH][J3_BW]
  constexpr int TY = J3_TY / RPT, NT = J3_TX * TY;
  constexpr int BOX = J3_BW * J3_BH, SLOT = BOX;  // doubles per slot
  constexpr int NC = (BOX + NT - 1) / NT;         // box cells per thread
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * J3_TX + tx;
  const int bx0 = blockIdx.x * J3_TX, by0 = blockIdx.y * J3_TY;
  const int x = bx0 + tx + 1;
  const int z0 = 1 + blockIdx.z * zrun, z1 = min(nz + 1, z0 + zrun);
  const long long sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
  int cell[NC], goff[NC];
  bool inside[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) {
    const int e = tid + k * NT;
    cell[k] = e < BOX ? e : -1;
    const int gx = bx0 + e % J3_BW, gy = by0 + e / J3_BW;
    inside[k] = e < BOX && gx <= nx + 1 && gy <= ny + 1;
    goff[k] = inside[k] ? (int)(gy * sy + gx) : 0;
  }
  auto issue = [&](int p) {
    if (p <= z1) {
      double* slot = j3_slots + ((p - z0 + 1) % J3_S) * SLOT;
      const double* src = in + (long long)p * sz;
#pragma unroll
      for (int k = 0; k < NC; k++) {
        if (cell[k] < 0) continue;
        // zero-fill (source size 0) outside the grid, from a valid address
        const unsigned n = inside[k] ? 8u : 0u;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(jac::smem_u32(slot + cell[k])),
                     "l"(inside[k] ? src + goff[k] : in), "r"(n) : "memory");
      }
    }
    jac::cp_async_commit();  // one group per plane, empty past z1
  };
  for (int p = z0 - 1; p <= z0 + J3_S - 3; p++) issue(p);
  for (int z = z0; z < z1; z++) {
    issue(z + J3_S - 2);              // into the slot plane z-2 used
    jac::cp_async_wait<J3_S - 3>();  // planes up to z+1 have landed (this thread's copies)
    __syncthreads();                 // ... and every other thread's
    const double* m = j3_slots + ((z - z0 + 1) % J3_S) * SLOT;
    const double* lo = j3_slots + ((z - z0) % J3_S) * SLOT;
    const double* hi = j3_slots + ((z - z0 + 2) % J3_S) * SLOT;
#pragma unroll
    for (int r = 0; r < RPT; r++) {
      const int yy = ty + r * TY, y = by0 + yy + 1;
      if (x <= nx && y <= ny) {
        const int c = (yy + 1) * J3_BW + tx + 1;
        out[(long long)y * sy + x + (long long)z * sz] =
            j3_stencil(m[c], m[c - 1], m[c + 1], m[c - J3_BW], m[c + J3_BW], lo[c], hi[c]);
      }
    }
    __syncthreads();  // plane z-1's slot takes plane z+J3_S-1 next
  }
  jac::cp_async_wait<0>();
}

__global__ void __launch_bounds__(J3_TX * J3_TY) jacobi3d_kernel(const double* __restrict__ in,
    double* __restrict__ out, int nx, int ny, int nz, int zrun) {
  __shared__ double plane[J3_TY + 2][J3_TX + 2];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x = blockIdx.x * J3_TX + tx + 1, y = blockIdx.y * J3_TY + ty + 1;
  const int z0 = 1 + blockIdx.z * zrun, z1 = min(nz + 1, z0 + zrun);
  const long long sx = 1, sy = nx + 2, sz = (long long)(nx + 2) * (ny + 2);
  const bool inx = x <= nx + 1, iny = y <= ny + 1;       // a cell of the grid (rim included)
  const bool own = x <= nx && y <= ny;                   // an interior column
  const long long col = (long long)(inx ? x : nx + 1) * sx + (long long)(iny ? y : ny + 1) * sy;
  auto at = [&](int z) { return in[col + (long long)z * sz]; };
  double prev = at(z0 - 1), cur = at(z0), next = at(z0 + 1);
  for (int z = z0; z < z1; z++) {
    const double nn = z + 2 <= nz + 1 ? at(z + 2) : 0.0;  // one plane ahead
    plane[ty + 1][tx + 1] = cur;
    const long long zo = (long long)z * sz;
    if (tx == 0) plane[ty + 1][0] = in[col - sx + zo];
    if (tx == J3_TX - 1 && inx && x + 1 <= nx + 1) plane[ty + 1][J3_TX + 1] = in[col + sx + zo];
    if (ty == 0) plane[0][tx + 1] = in[col - sy + zo];
    if (ty == J3_TY - 1 && iny && y + 1 <= ny + 1) plane[J3_TY + 1][tx + 1] = in[col + sy + zo];
    __syncthreads();
    if (own) {
      out[col + zo] = j3_stencil(cur, plane[ty + 1][tx], plane[ty + 1][tx + 2], plane[ty][tx + 1],
                                 plane[ty + 2][tx + 1], prev, next);
    }
    __syncthreads();
    prev = cur;
    cur = next;
    next = nn;
  }
}

// The shared-memory pipeline needs no alignment beyond 8 bytes: any shape
// with at least one full box in x and y takes it.
bool async_shape_ok(int nx, int ny) { return nx + 2 >= J3_BW && ny + 2 >= J3_BH; }

constexpr size_t j3_async_smem(int stages) { return (size_t)stages * J3_BW * J3_BH * 8; }

// z planes per block for the register kernel: enough blocks to fill the GPU
// several times over
int jacobi3d_zrun(int nx, int ny, int nz, int n_sms) {
  const long long cols = (long long)((nx + J3_TX - 1) / J3_TX) * ((ny + J3_TY - 1) / J3_TY);
  long long want = 8LL * n_sms;  // blocks
  long long runs = (want + cols - 1) / cols;
  if (runs < 1) runs = 1;
  int zrun = (int)((nz + runs - 1) / runs);
  if (zrun < 16) zrun = 16;
  return zrun;
}

// z planes per block for the pipelined kernel. Blocks = tiles x runs; the
// GPU holds `slots` of them at once, so the launch takes ceil(blocks /
// slots) waves and the last one may run part-empty, while every run reads
// two planes more than it writes. Picks the run count (1..32) with the best
// product of wave fill and plane efficiency.
int jacobi3d_async_zrun(int nx, int ny, int nz, int n_sms, int per_sm) {
  const long long tiles = (long long)((nx + J3_TX - 1) / J3_TX) * ((ny + J3_TY - 1) / J3_TY);
  const double slots = (double)n_sms * (per_sm > 0 ? per_sm : 1);
  int best_zrun = nz;
  double best = -1.0;
  for (int runs = 1; runs <= 32; runs++) {
    const int zrun = (nz + runs - 1) / runs;
    if (zrun < 8 && runs > 1) break;
    const long long blocks = tiles * ((nz + zrun - 1) / zrun);
    const double waves = (double)blocks / slots;
    const double fill = waves / std::ceil(waves);
    const double eff = fill * zrun / (zrun + 2.0);
    if (eff > best + 1e-9) {
      best = eff;
      best_zrun = zrun;
    }
  }
  return best_zrun;
}

// Rows per thread of the pipelined kernel: CHARMING_J3_RPT (1 or 2) with
// CHARMING_J3_STAGES (8 with 1 row, 10 or 12 with 2), else the defaults.
int jacobi3d_rpt() {
  static int rpt = 0;
  if (!rpt) {
    rpt = J3_RPT_DEFAULT;
    if (const char* ev = getenv("CHARMING_J3_RPT")) {
      const int v = atoi(ev);
      if (v == 1 || v == 2) rpt = v;
    }
  }
  return rpt;
}

// Stage count of the pipelined kernel (see jacobi3d_rpt).
int jacobi3d_stages() {
  static int stages = 0;
  if (!stages) {
    stages = J3_S_DEFAULT;
    if (const char* ev = getenv("CHARMING_J3_STAGES")) {
      const int v = atoi(ev);
      if (v == 8 || v == 10 || v == 12) stages = v;
    }
  }
  return stages;
}

template <int S, int RPT>
cudaError_t jacobi3d_async_sweeps(double*& a, double*& b, int nx, int ny, int nz, int sweeps, int n_sms,
    cudaStream_t s) {
  int per_sm = 0;
  cudaError_t e = cudaSuccess;
  const void* fn = (const void*)jacobi3d_async_kernel<S, RPT>;
  if (j3_async_smem(S) > 48 * 1024)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)j3_async_smem(S));
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi3d_async_kernel<S, RPT>,
                                                      J3_TX * J3_TY / RPT, j3_async_smem(S));
  if (e != cudaSuccess) return e;
  const int zrun = jacobi3d_async_zrun(nx, ny, nz, n_sms, per_sm);
  const dim3 block(J3_TX, J3_TY / RPT), grid((nx + J3_TX - 1) / J3_TX, (ny + J3_TY - 1) / J3_TY, (nz + zrun - 1) / zrun);
  for (int k = 0; k < sweeps && e == cudaSuccess; k++) {
    jacobi3d_async_kernel<S, RPT><<<grid, block, j3_async_smem(S), s>>>(a, b, nx, ny, nz, zrun);
    e = cudaGetLastError();
    double* t = a;
    a = b;
    b = t;
  }
  return e;
}

// `sweeps` sweeps alternating between a and b (both hold the input,
// boundary shell included); returns the buffer holding the result.
double* jacobi3d_run(double* a, double* b, int nx, int ny, int nz, int sweeps, cudaStream_t s, cudaError_t* err) {
  const int n_sms = charm_host::info().n_sms;
  *err = cudaSuccess;
  const dim3 block(J3_TX, J3_TY);
  if (async_shape_ok(nx, ny)) {
    const int st = jacobi3d_stages(), rpt = jacobi3d_rpt();
    if (st == 8 && rpt == 1) *err = jacobi3d_async_sweeps<8, 1>(a, b, nx, ny, nz, sweeps, n_sms, s);
    else if (st == 12 && rpt == 2) *err = jacobi3d_async_sweeps<12, 2>(a, b, nx, ny, nz, sweeps, n_sms, s);
    else *err = jacobi3d_async_sweeps<10, 2>(a, b, nx, ny, nz, sweeps, n_sms, s);
    return a;
  }
  const int zrun = jacobi3d_zrun(nx, ny, nz, n_sms);
  const dim3 grid((nx + J3_TX - 1) / J3_TX, (ny + J3_TY - 1) / J3_TY, (nz + zrun - 1) / zrun);
  for (int k = 0; k < sweeps && *err == cudaSuccess; k++) {
    jacobi3d_kernel<<<grid, block, 0, s>>>(a, b, nx, ny, nz, zrun);
    *err = cudaGetLastError();
    double* t = a;
    a = b;
    b = t;
  }
  return a;
}

}  // namespace

extern "C" int charming_jacobi3d(int nx, int ny, int nz, int sweeps, double* grid, double* out_ms) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (nx < 1 || ny < 1 || nz < 1 || sweeps < 0 || !grid) return CHARMING_ERR_CONFIG;
  const size_t n = ((size_t)nx + 2) * ((size_t)ny + 2) * ((size_t)nz + 2);
  double *a = nullptr, *b = nullptr;
  cudaError_t e = cudaMalloc(&a, n * 8);
  if (e == cudaSuccess) e = cudaMalloc(&b, n * 8);
  cudaStream_t s = charm_host::stream();
  if (e == cudaSuccess) e = cudaMemcpyAsync(a, grid, n * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b, a, n * 8, cudaMemcpyDeviceToDevice, s);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double* res = a;
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) res = jacobi3d_run(a, b, nx, ny, nz, sweeps, s, &e);
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(grid, res, n * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (out_ms) *out_ms = ms;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  return charm_host::cuda_fail(e, "jacobi3d");
}
#endif
