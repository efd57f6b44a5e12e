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
// Kernel: each block owns a 32 x 16 tile of (x, y) columns and a run of z
// planes, and marches up z: the planes below and above a thread's cell (and
// the next three, already loading) stay in its registers, the current plane
// (with a one-cell x/y rim) sits in shared memory for the x and y
// neighbours. Each input value is read from
// DRAM once per sweep (16 B per lattice update with the store); the rim
// cells are read by two blocks and mostly come from L2.
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION
#include "../host.cuh"

namespace {

constexpr int J3_TX = 32, J3_TY = 16;

__device__ __forceinline__ double j3_stencil(double c, double xm, double xp, double ym, double yp, double zm,
    double zp) {
  return __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(c, xm), xp), ym), yp), zm), zp),
                   0.142857);
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
  auto at = [&](int z) { return z <= nz + 1 ? in[col + (long long)z * sz] : 0.0; };
  // planes z-1 .. z+3 of this column in registers: three loads in flight
  // per thread keep enough bytes moving to cover the memory latency
  double prev = at(z0 - 1), cur = at(z0), next = at(z0 + 1), n2 = at(z0 + 2), n3 = at(z0 + 3);
  for (int z = z0; z < z1; z++) {
    const double n4 = at(z + 4);
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
    next = n2;
    n2 = n3;
    n3 = n4;
  }
}

// Host: `sweeps` sweeps alternating between a and b (both hold the input,
// boundary shell included); returns the buffer holding the result.
double* jacobi3d_run(double* a, double* b, int nx, int ny, int nz, int sweeps, int zrun, cudaStream_t s,
    cudaError_t* err) {
  const dim3 block(J3_TX, J3_TY), grid((nx + J3_TX - 1) / J3_TX, (ny + J3_TY - 1) / J3_TY, (nz + zrun - 1) / zrun);
  *err = cudaSuccess;
  for (int k = 0; k < sweeps && *err == cudaSuccess; k++) {
    jacobi3d_kernel<<<grid, block, 0, s>>>(a, b, nx, ny, nz, zrun);
    *err = cudaGetLastError();
    double* t = a;
    a = b;
    b = t;
  }
  return a;
}

// z planes per block: enough blocks to fill the GPU several times over
int jacobi3d_zrun(int nx, int ny, int nz, int n_sms) {
  const long long cols = (long long)((nx + J3_TX - 1) / J3_TX) * ((ny + J3_TY - 1) / J3_TY);
  long long want = 8LL * n_sms;  // blocks
  long long runs = (want + cols - 1) / cols;
  if (runs < 1) runs = 1;
  int zrun = (int)((nz + runs - 1) / runs);
  if (zrun < 16) zrun = 16;
  return zrun;
}

}  // namespace

extern "C" int charming_jacobi3d(int nx, int ny, int nz, int sweeps, double* grid, double* out_ms) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (nx < 1 || ny < 1 || nz < 1 || sweeps < 0 || !grid) return CHARMING_ERR_CONFIG;
  const size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
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
  if (e == cudaSuccess) {
    res = jacobi3d_run(a, b, nx, ny, nz, sweeps, jacobi3d_zrun(nx, ny, nz, charm_host::info().n_sms), s, &e);
  }
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
