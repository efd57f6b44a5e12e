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
//   jacobi3d_tma_kernel (rows of a multiple of 16 bytes, grid at least one
//     tile with its rim): one thread streams the tile's planes, rim
//     included (a 34 x 18 box whose first column is 16-byte aligned), into a
//     ring of J3_S shared-memory slots with 3-D tensor copies (TMA, no
//     multicast), each slot completing on its own mbarrier; J3_S - 2 planes
//     are in flight while the block computes from the three it holds. Each
//     input value is read from DRAM once per sweep (16 B per lattice update
//     with the store); the rim cells come from L2.
//   jacobi3d_kernel (any shape): per-thread loads, the planes below and
//     above a thread's cell and one more in registers, the current plane
//     with its rim in shared memory.
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION
#include <cuda.h>  // CUtensorMap and its enums; the encoder comes from the runtime's entry-point lookup
#include "jacobi_sweep.cuh"
#include "../host.cuh"

namespace {

constexpr int J3_TX = 32, J3_TY = 16;
constexpr int J3_BW = J3_TX + 2, J3_BH = J3_TY + 2;          // tensor box: tile + rim
constexpr unsigned J3_BOX_BYTES = J3_BW * J3_BH * 8;         // 4896
constexpr int J3_SLOT_BYTES = (J3_BOX_BYTES + 127) / 128 * 128;
constexpr int J3_S = 8;                                      // plane slots
constexpr unsigned J3_SPIN_MAX = 1u << 22;                   // bounded mbarrier waits

__device__ __forceinline__ double j3_stencil(double c, double xm, double xp, double ym, double yp, double zm,
    double zp) {
  return __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(c, xm), xp), ym), yp), zm), zp),
                   0.142857);
}

// 3-D tiled tensor copy global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
    unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];"
      :: "r"(jac::smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(jac::smem_u32(bar)) : "memory");
}

// Planes z0-1 .. z1 of the tile stream through the slots: plane p lives in
// slot (p - z0 + 1) % J3_S, its use number of that slot gives the mbarrier
// parity. Plane z-1+J3_S is issued once every thread is past plane z-1.
// A wait that runs out ends the block after the copies in flight have
// landed and sets *err.
__global__ void __launch_bounds__(J3_TX * J3_TY, 3) jacobi3d_tma_kernel(const __grid_constant__ CUtensorMap map,
    double* __restrict__ out, int nx, int ny, int nz, int zrun, int* err) {
  extern __shared__ __align__(128) unsigned char j3_smem[];
  __shared__ __align__(8) unsigned long long full[J3_S];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * J3_TX + tx;
  const int bx0 = blockIdx.x * J3_TX, by0 = blockIdx.y * J3_TY;
  const int x = bx0 + tx + 1, y = by0 + ty + 1;
  const int z0 = 1 + blockIdx.z * zrun, z1 = min(nz + 1, z0 + zrun);
  const bool own = x <= nx && y <= ny;
  const long long col = (long long)y * (nx + 2) + x, sz = (long long)(nx + 2) * (ny + 2);
  const double* slots = reinterpret_cast<const double*>(j3_smem);
  const int c = (ty + 1) * J3_BW + tx + 1;  // this thread's cell in a slot
  auto slot_of = [&](int p) { return (p - z0 + 1) % J3_S; };
  auto parity_of = [&](int p) { return (unsigned)(((p - z0 + 1) / J3_S) & 1); };
  auto issue = [&](int p) {
    const int s = slot_of(p);
    jac::mbar_expect_tx(&full[s], J3_BOX_BYTES);
    tma_load_3d(j3_smem + s * J3_SLOT_BYTES, &map, bx0, by0, p, &full[s]);
  };
  auto wait = [&](int p) {
    unsigned spins = 0;
    while (!jac::mbar_try_wait(&full[slot_of(p)], parity_of(p)))
      if (++spins > J3_SPIN_MAX) return false;
    return true;
  };
  if (tid == 0) {
    for (int s = 0; s < J3_S; s++) jac::mbar_init(&full[s], 1);
    jac::fence_mbar_init();
  }
  __syncthreads();
  int issued = z0 - 2;  // last plane issued (thread 0)
  if (tid == 0) {
    for (int p = z0 - 1; p <= z1 && p <= z0 - 2 + J3_S; p++) issue(p);
    issued = min(z1, z0 - 2 + J3_S);
  }
  bool ok = wait(z0 - 1) && wait(z0);
  int z = z0;
  for (; z < z1; z++) {
    ok = ok && wait(z + 1);
    if (ok && own) {
      const double* m = slots + slot_of(z) * (J3_SLOT_BYTES / 8);
      const double* lo = slots + slot_of(z - 1) * (J3_SLOT_BYTES / 8);
      const double* hi = slots + slot_of(z + 1) * (J3_SLOT_BYTES / 8);
      out[col + (long long)z * sz] = j3_stencil(m[c], m[c - 1], m[c + 1], m[c - J3_BW], m[c + J3_BW], lo[c], hi[c]);
    }
    if (__syncthreads_or(!ok)) break;
    // every thread is done with plane z-1: its slot takes plane z-1+J3_S
    if (tid == 0 && z - 1 + J3_S <= z1) {
      jac::fence_proxy_async_smem();
      issue(z - 1 + J3_S);
      issued = z - 1 + J3_S;
    }
  }
  if (tid == 0) {
    if (z < z1) {
      // a wait ran out: let the copies still in flight land, then report
      for (int p = z + 1; p <= issued; p++) wait(p);
      atomicExch(err, 1);
    }
    for (int s = 0; s < J3_S; s++) jac::mbar_inval(&full[s]);
  }
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

using encode_tiled_fn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
    const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once; null when unavailable.
encode_tiled_fn tensor_map_encoder() {
  static encode_tiled_fn fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<encode_tiled_fn>(p);
    cudaGetLastError();
  }
  return fn;
}

// The TMA kernel needs rows of a multiple of 16 bytes (tensor-map strides)
// and a grid no smaller than one box in x and y.
bool tma_shape_ok(int nx, int ny) { return (nx + 2) % 2 == 0 && nx + 2 >= J3_BW && ny + 2 >= J3_BH; }

// Tensor map over one (nx+2) x (ny+2) x (nz+2) grid of doubles, box 34 x 18 x 1.
bool make_grid_map(CUtensorMap* m, double* base, int nx, int ny, int nz) {
  encode_tiled_fn enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx + 2, (cuuint64_t)ny + 2, (cuuint64_t)nz + 2};
  const cuuint64_t strides[2] = {((cuuint64_t)nx + 2) * 8, ((cuuint64_t)nx + 2) * ((cuuint64_t)ny + 2) * 8};
  const cuuint32_t box[3] = {J3_BW, J3_BH, 1}, estr[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr size_t J3_TMA_SMEM = (size_t)J3_S * J3_SLOT_BYTES;

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

// z planes per block for the TMA kernel: one wave of resident blocks when
// the tiles leave room for it (each run adds two planes of reads).
int jacobi3d_tma_zrun(int nx, int ny, int nz, int n_sms, int per_sm) {
  const long long tiles = (long long)((nx + J3_TX - 1) / J3_TX) * ((ny + J3_TY - 1) / J3_TY);
  long long runs = (long long)n_sms * per_sm / tiles;
  if (runs < 1) runs = 1;
  if (runs > nz / 8) runs = nz / 8 > 0 ? nz / 8 : 1;
  return (int)((nz + runs - 1) / runs);
}

// `sweeps` sweeps alternating between a and b (both hold the input,
// boundary shell included); returns the buffer holding the result.
double* jacobi3d_run(double* a, double* b, int nx, int ny, int nz, int sweeps, cudaStream_t s, int* d_err,
    cudaError_t* err, bool* used_tma) {
  const int n_sms = charm_host::info().n_sms;
  *err = cudaSuccess;
  *used_tma = false;
  CUtensorMap ma, mb;
  if (tma_shape_ok(nx, ny) && make_grid_map(&ma, a, nx, ny, nz) && make_grid_map(&mb, b, nx, ny, nz)) {
    int per_sm = 0;
    *err = cudaFuncSetAttribute((const void*)jacobi3d_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)J3_TMA_SMEM);
    if (*err == cudaSuccess)
      *err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi3d_tma_kernel, J3_TX * J3_TY, J3_TMA_SMEM);
    if (*err != cudaSuccess) return a;
    const int zrun = jacobi3d_tma_zrun(nx, ny, nz, n_sms, per_sm > 0 ? per_sm : 1);
    const dim3 block(J3_TX, J3_TY), grid((nx + J3_TX - 1) / J3_TX, (ny + J3_TY - 1) / J3_TY, (nz + zrun - 1) / zrun);
    *used_tma = true;
    for (int k = 0; k < sweeps && *err == cudaSuccess; k++) {
      jacobi3d_tma_kernel<<<grid, block, J3_TMA_SMEM, s>>>((k & 1) ? mb : ma, (k & 1) ? a : b, nx, ny, nz, zrun,
                                                           d_err);
      *err = cudaGetLastError();
    }
    return (sweeps & 1) ? b : a;
  }
  const int zrun = jacobi3d_zrun(nx, ny, nz, n_sms);
  const dim3 block(J3_TX, J3_TY), grid((nx + J3_TX - 1) / J3_TX, (ny + J3_TY - 1) / J3_TY, (nz + zrun - 1) / zrun);
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
  int* d_err = nullptr;
  cudaError_t e = cudaMalloc(&a, n * 8);
  if (e == cudaSuccess) e = cudaMalloc(&b, n * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_err, sizeof(int));
  cudaStream_t s = charm_host::stream();
  if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(a, grid, n * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b, a, n * 8, cudaMemcpyDeviceToDevice, s);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double* res = a;
  bool used_tma = false;
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess) res = jacobi3d_run(a, b, nx, ny, nz, sweeps, s, d_err, &e, &used_tma);
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(grid, res, n * 8, cudaMemcpyDeviceToHost, s);
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  if (out_ms) *out_ms = ms;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  cudaFree(d_err);
  if (e == cudaSuccess && herr) {
    charm_host::set_error_text("jacobi3d: a plane copy did not arrive in time");
    return CHARMING_ERR_PIPELINE;
  }
  return charm_host::cuda_fail(e, "jacobi3d");
}
#endif
