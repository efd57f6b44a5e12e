// Jacobi2d over a 1-D row decomposition: the scenario of the reference's
// examples/jacobi2d-decomp1d/jacobi2d.cu (an FP32 4-point stencil, each
// chare a band of rows, periodic top/bottom neighbours, left/right columns
// fixed), with three ways to meet the neighbours every iteration:
//   mode 0 (WAIT):  write the boundary rows straight into the neighbours'
//                   next-input buffers, signal them (release store of the
//                   iteration number, as nvshmemx_signal_op does there,
//                   :405-414), and wait for their signals inside the entry
//                   method (nvshmem_uint64_wait_until_all, :419); one chare
//                   per PE, as the reference needs
//   mode 1 (ASYNC): the same writes and signals, then async_wait on the two
//                   signal words; the scheduler resumes the chare when both
//                   have arrived (the reference's ASYNC_WAIT build, :251-290)
//   mode 2 (MSG):   the boundary rows go as runtime messages tagged with
//                   the iteration as refnum (the reference's commented-out
//                   send_halo / recv_halo, :335-370)
// The chunking, clamps and neighbours follow Block::init (:128-198); the
// boundary columns are the host's (sin(2*PI*(g-1)/(ny-3)) per global row g,
// computed there on the device, :424-433). The rows go into the buffer the
// neighbour reads next (the reference always writes its first buffer).
#include "suite.cuh"
#include "decomp1d.h"
#ifndef CHARMING_HOST_EMULATION
#include "../host.cuh"
#endif
#include <cmath>

// Block::init's decomposition (examples/jacobi2d-decomp1d/jacobi2d.cu:144-198)
// and the boundary columns; false when a chare would get fewer than 2 rows.
bool decomp1d_plan(int n, int ny, std::vector<d1_desc>& descs, std::vector<int>& g0, std::vector<float>& bc) {
  const int low = (ny - 2) / n, high = low + 1;
  if (n < 1 || ny < 4 || low < 2) return false;
  const int n_low = n * low + n - (ny - 2);
  descs.assign(n, d1_desc{});
  g0.assign(n, 0);
  for (int i = 0; i < n; i++) {
    d1_desc& d = descs[i];
    d.chunk = i < n_low ? low : high;
    g0[i] = i < n_low ? i * low + 1 : n_low * low + (i - n_low) * high + 1;
    int gend = g0[i] + d.chunk - 1;
    if (gend > ny - 4) gend = ny - 4;
    d.iy_end = (gend - g0[i] + 1) + 1;
    d.top = i > 0 ? i - 1 : n - 1;
    d.bottom = (i + 1) % n;
    d.top_ghost = (d.top < n_low ? low : high) + 1;
  }
  bc.assign(ny, 0.f);
  const double pi = (double)(float)3.141592;
  for (int g = 0; g < ny; g++) bc[g] = (float)std::sin(2.0 * pi * (double)(g - 1) / (double)(ny - 3));
  return true;
}

namespace {

using namespace charm::rt;

enum : int { EP_D_ITER = 0, EP_D_RESUME = 1, EP_D_HALO = 2 };
enum : int { D_WAIT = 0, D_ASYNC = 1, D_MSG = 2 };

// g_app: a[0] n chares, a[1] nx, a[2] iterations, a[3] mode, a[4] floats per
// buffer; p[0] buffers (float, [n][2][cnt]), p[1] d1_desc[n], p[2] signal
// words (u64[n][2]: [0] from the top neighbour, [1] from the bottom one),
// p[3] counters (u64: chares done).
struct d1 {
  __device__ static int n() { return (int)g_app.a[0]; }
  __device__ static int nx() { return (int)g_app.a[1]; }
  __device__ static int iters() { return (int)g_app.a[2]; }
  __device__ static int mode() { return (int)g_app.a[3]; }
  __device__ static float* buf(int c, int b) {
    return reinterpret_cast<float*>(g_app.p[0]) + ((size_t)c * 2 + b) * (size_t)g_app.a[4];
  }
  __device__ static const d1_desc& desc(int c) { return reinterpret_cast<const d1_desc*>(g_app.p[1])[c]; }
  __device__ static unsigned long long* sig(int c) {
    return reinterpret_cast<unsigned long long*>(g_app.p[2]) + 2 * (size_t)c;
  }
  __device__ static unsigned long long* done() { return reinterpret_cast<unsigned long long*>(g_app.p[3]); }
};

struct D1Chare : charm::chare {
  int k;     // iterations done
  int got;   // halos of the next iteration received (message mode)
  int next;  // the halo just received completed the iteration (message mode)
  int ok;    // mode 0: both neighbours' signals arrived
  __device__ D1Chare() : k(0), got(0), next(0), ok(0) {}
};
// SM-level mode: each PE block creates its own proxy; GPU-level mode: one
// proxy for the single PE, seen by every block.
__shared__ charm::chare_proxy<D1Chare>* d1_proxy_block;
__device__ charm::chare_proxy<D1Chare>* d1_proxy_gpu;
__device__ __forceinline__ charm::chare_proxy<D1Chare>* d1_proxy() {
  return charm::is_gpu_level() ? d1_proxy_gpu : d1_proxy_block;
}

struct d1_halo {  // message payload header; nx-2 floats follow
  int to_top_ghost;  // 1: the receiver's row 0, 0: its bottom ghost row
  int iter;
  int pad[2];
};

constexpr int D1_STEP = 4;  // rows loaded together per warp step (8 measured slower)

__device__ __forceinline__ float d1_stencil(float r, float l, float d, float u) {
  return __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(r, l), d), u), 0.25f);
}

// The PE's threads (all of them, pe_thread() / pe_threads()): rows
// [1, iy_end) of o from a (row pitch nx, nx % 4 == 0). Work items are
// (column strip of 32 float4, run of rows); each warp walks its items'
// rows downwards, the three rows around the output in registers,
// neighbours across lanes by shuffle, D1_STEP rows loaded at once. Row runs
// split the strips when there are more warps than strips (a GPU-level PE
// has thousands).
__device__ void d1_sweep(const float* __restrict__ a, float* __restrict__ o, int nx, int iy_end) {
  constexpr unsigned FULL = 0xffffffffu;
  const int tid = charm::pe_thread(), nthreads = charm::pe_threads();
  if (iy_end < 2) return;
  if (blockDim.x < 32) {  // blocks under a warp (host checks): element by element
    for (long long x = tid; x < (long long)(iy_end - 1) * (nx - 2); x += nthreads) {
      const int iy = 1 + (int)(x / (nx - 2)), ix = 1 + (int)(x % (nx - 2));
      const float* m = a + (size_t)iy * nx + ix;
      o[(size_t)iy * nx + ix] = d1_stencil(m[1], m[-1], m[nx], m[-nx]);
    }
    return;
  }
  const int nv = nx / 4, warp = tid >> 5, lane = tid & 31, nw = nthreads >> 5;
  const int strips = (nv + 31) / 32, rows = iy_end - 1;
  int runs = nw / strips;
  if (runs > rows / 8) runs = rows / 8;  // at least 8 rows per run
  if (runs < 1) runs = 1;
  const int run_rows = (rows + runs - 1) / runs;
  runs = (rows + run_rows - 1) / run_rows;  // every run starts inside the band
  for (int item = warp; item < strips * runs; item += nw) {
    const int s = item % strips, r0 = 1 + (item / strips) * run_rows;
    const int r1 = min(iy_end, r0 + run_rows);
    if (r0 >= iy_end) continue;  // (none by construction; the loads below need it)
    const int v = s * 32 + lane;
    const bool act = v < nv;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    // rows past the ghost row iy_end are never read (zeros stand in)
    auto ld = [&](int iy) {
      return act && iy <= iy_end ? *reinterpret_cast<const float4*>(a + (size_t)iy * nx + 4 * v) : z;
    };
    // output row iy from the rows above (U), at (M) and below (D)
    auto row = [&](int iy, const float4& U, const float4& M, const float4& D) {
      float left = __shfl_up_sync(FULL, M.w, 1);
      float right = __shfl_down_sync(FULL, M.x, 1);
      const bool out_row = act && iy < r1;  // the last step may run past the run
      if (out_row && lane == 0 && v > 0) left = a[(size_t)iy * nx + 4 * v - 1];
      if (out_row && lane == 31 && v + 1 < nv) right = a[(size_t)iy * nx + 4 * v + 4];
      if (out_row) {
        float4 out;
        out.x = d1_stencil(M.y, left, D.x, U.x);
        out.y = d1_stencil(M.z, M.x, D.y, U.y);
        out.z = d1_stencil(M.w, M.y, D.z, U.z);
        out.w = d1_stencil(right, M.z, D.w, U.w);
        float* op = o + (size_t)iy * nx + 4 * v;
        if (v > 0 && v + 1 < nv) {
          *reinterpret_cast<float4*>(op) = out;
        } else {  // the vectors holding columns 0 and nx-1 keep those
          if (4 * v + 0 >= 1 && 4 * v + 0 <= nx - 2) op[0] = out.x;
          if (4 * v + 1 >= 1 && 4 * v + 1 <= nx - 2) op[1] = out.y;
          if (4 * v + 2 >= 1 && 4 * v + 2 <= nx - 2) op[2] = out.z;
          if (4 * v + 3 >= 1 && 4 * v + 3 <= nx - 2) op[3] = out.w;
        }
      }
    };
    // D1_STEP rows per step: their loads are in flight together
    float4 U = ld(r0 - 1), M = ld(r0);
    for (int iy = r0; iy < r1; iy += D1_STEP) {
      float4 b[D1_STEP];
#pragma unroll
      for (int k = 0; k < D1_STEP; k++) b[k] = ld(iy + 1 + k);
      row(iy, U, M, b[0]);
      row(iy + 1, M, b[0], b[1]);
#pragma unroll
      for (int k = 2; k < D1_STEP; k++) row(iy + k, b[k - 2], b[k - 1], b[k]);
      U = b[D1_STEP - 2];
      M = b[D1_STEP - 1];
    }
  }
}

__device__ void d1_count_done() {
  if (charm::pe_thread() == 0) {
    if (atomicAdd(d1::done(), 1ULL) + 1 == (unsigned long long)d1::n()) charm::end();
  }
  charm::pe_sync();
}

__device__ void d1_iterate(D1Chare& c);

// All threads: the end of iteration c.k in the signal modes: the boundary
// rows into the neighbours' next buffers, then the signals.
__device__ void d1_put_and_signal(D1Chare& c) {
  const d1_desc& d = d1::desc(c.i);
  const int nx = d1::nx(), nb = (c.k + 1) & 1;
  const float* o = d1::buf(c.i, nb);
  const size_t tid = (size_t)charm::pe_thread(), nt = (size_t)charm::pe_threads();
  charm::copy_cooperative(d1::buf(d.top, nb) + (size_t)d.top_ghost * nx + 1, o + nx + 1,
                          sizeof(float) * (nx - 2), tid, nt);
  charm::copy_cooperative(d1::buf(d.bottom, nb) + 1, o + (size_t)(d.iy_end - 1) * nx + 1,
                          sizeof(float) * (nx - 2), tid, nt);
  charm::pe_sync();  // the rows are written before the signals (release is cumulative)
  if (tid == 0) {
    st_release_u64(&d1::sig(d.top)[1], (unsigned long long)c.k + 1);
    st_release_u64(&d1::sig(d.bottom)[0], (unsigned long long)c.k + 1);
  }
}

// All threads: sends the boundary rows of iteration c.k as messages tagged
// k + 1.
__device__ void d1_send_halos(D1Chare& c) {
  const d1_desc& d = d1::desc(c.i);
  const int nx = d1::nx(), nb = (c.k + 1) & 1;
  const float* o = d1::buf(c.i, nb);
  const size_t bytes = sizeof(d1_halo) + sizeof(float) * (nx - 2);
  const int tid = charm::pe_thread();
  for (int side = 0; side < 2; side++) {
    const int to = side == 0 ? d.top : d.bottom;
    charm::message msg;
    if (!d1_proxy()->alloc_msg(msg, to, bytes)) return;
    d1_halo* h = reinterpret_cast<d1_halo*>(msg.payload());
    if (tid == 0) {
      h->to_top_ghost = side == 1;  // my last row is the bottom neighbour's row 0
      h->iter = c.k + 1;
    }
    const float* row = side == 0 ? o + nx + 1 : o + (size_t)(d.iy_end - 1) * nx + 1;
    charm::copy_cooperative(reinterpret_cast<char*>(h) + sizeof(d1_halo), row, sizeof(float) * (nx - 2),
                            (size_t)tid, (size_t)charm::pe_threads());
    d1_proxy()->invoke(to, EP_D_HALO, msg, bytes, c.k + 1);
  }
}

// All threads: iteration c.k (and, in mode 0, the following ones).
__device__ void d1_iterate(D1Chare& c) {
  const d1_desc& d = d1::desc(c.i);
  const int mode = d1::mode(), nx = d1::nx();
  const int tid = charm::pe_thread();
  while (true) {
    if (c.k >= d1::iters()) {
      d1_count_done();
      return;
    }
    if (mode == D_MSG && tid == 0) d1_proxy()->set_refnum(c.i, c.k + 1);
    d1_sweep(d1::buf(c.i, c.k & 1), d1::buf(c.i, (c.k + 1) & 1), nx, d.iy_end);
    charm::pe_sync();
    if (mode == D_MSG) {
      d1_send_halos(c);
      return;  // the halos' entry method continues
    }
    d1_put_and_signal(c);
    if (mode == D_ASYNC) {
      if (tid == 0)
        d1_proxy()->async_wait(reinterpret_cast<uint64_t*>(d1::sig(c.i)), 2, charm::CMP_GE,
                               (unsigned long long)c.k + 1, c.i, EP_D_RESUME);
      charm::pe_sync();
      return;
    }
    // mode 0: wait here for both neighbours (bounded by the run deadline)
    if (tid == 0) {
      const unsigned long long want = (unsigned long long)c.k + 1;
      unsigned long long* w = d1::sig(c.i);
      unsigned spins = 0;
      int ok = 1;
      while (ld_acquire_u64(&w[0]) < want || ld_acquire_u64(&w[1]) < want) {
        if ((++spins & 255) == 0 && (terminated() || past_deadline())) {
          if (!terminated()) set_error(CHARMING_ERR_DEADLINE, 3, c.i);
          ok = 0;
          break;
        }
      }
      c.ok = ok;
      if (ok) c.k++;
    }
    charm::pe_sync();
    if (!c.ok) return;
  }
}

__device__ void em_iter(D1Chare& c, void* arg) { d1_iterate(c); }

__device__ void em_resume(D1Chare& c, void* arg) {
  if (charm::pe_thread() == 0) c.k++;
  charm::pe_sync();
  d1_iterate(c);
}

__device__ void em_halo(D1Chare& c, void* arg) {
  const d1_halo* h = reinterpret_cast<const d1_halo*>(arg);
  const d1_desc& d = d1::desc(c.i);
  const int nx = d1::nx(), nb = h->iter & 1;
  float* dst = d1::buf(c.i, nb) + (h->to_top_ghost ? 0 : (size_t)(d.chunk + 1) * nx) + 1;
  charm::copy_cooperative(dst, reinterpret_cast<const char*>(arg) + sizeof(d1_halo), sizeof(float) * (nx - 2),
                          (size_t)charm::pe_thread(), (size_t)charm::pe_threads());
  if (charm::pe_thread() == 0) {
    c.next = ++c.got == 2;
    if (c.next) {
      c.got = 0;
      c.k++;
    }
  }
  charm::pe_sync();
  if (c.next) d1_iterate(c);
}

}  // namespace

__device__ void suite::decomp1d_main(int pe) {
  if (charm::pe_thread() == 0) {
    charm::chare_proxy<D1Chare>* p = new charm::chare_proxy<D1Chare>();
    p->add_entry_method<&em_iter>();
    p->add_entry_method<&em_resume>();
    p->add_entry_method<&em_halo>();
    p->create(d1::n());
    if (charm::is_gpu_level()) d1_proxy_gpu = p;
    else d1_proxy_block = p;
  }
  charm::pe_sync();
  charm::barrier();
  charm::chare_proxy<D1Chare>* p = d1_proxy();
  for (int i = p->start_idx; i <= p->end_idx && p->n_local > 0; i++) p->invoke(i, EP_D_ITER);
}

#ifndef CHARMING_HOST_EMULATION
namespace {
__global__ void d1_init_kernel(float* base, size_t cnt, const d1_desc* descs, const int* g0, const float* bc,
    int n, int nx) {
  // columns 0 and nx-1 of rows 1..chunk of both buffers of every chare
  for (int c = blockIdx.x; c < n; c += gridDim.x) {
    for (int r = 1 + threadIdx.x; r <= descs[c].chunk; r += blockDim.x) {
      const float v = bc[g0[c] + r - 1];
      for (int b = 0; b < 2; b++) {
        float* a = base + ((size_t)c * 2 + b) * cnt;
        a[(size_t)r * nx] = v;
        a[(size_t)r * nx + nx - 1] = v;
      }
    }
  }
}
}  // namespace

extern "C" int charming_jacobi2d_decomp1d(int n_chares, int nx, int ny, int iters, int mode, float* host_out,
    double* out_ms) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  const charming_info& inf = charm_host::info();
  if (n_chares < 1 || nx < 8 || (nx % 4) || ny < 4 || iters < 0 || mode < 0 || mode > 2 || !host_out) {
    charm_host::set_error_text("decomp1d: bad arguments (nx a multiple of 4 and >= 8)");
    return CHARMING_ERR_CONFIG;
  }
  std::vector<d1_desc> descs;
  std::vector<int> g0;
  std::vector<float> bc;
  if (!decomp1d_plan(n_chares, ny, descs, g0, bc)) {
    charm_host::set_error_text("decomp1d: fewer than 2 rows per chare");
    return CHARMING_ERR_CONFIG;
  }
  if (mode == D_WAIT && n_chares > inf.n_pes) {
    charm_host::set_error_text("decomp1d: waiting inside the entry method needs one chare per PE");
    return CHARMING_ERR_CONFIG;
  }
  if (mode == D_MSG && (size_t)(32 + 16 + 4 * (size_t)nx) > inf.max_msg_bytes) return CHARMING_ERR_MSG_TOO_LARGE;
  const int high = (ny - 2) / n_chares + 1;
  const size_t cnt = (size_t)nx * (high + 2);
  float* d_buf = nullptr;
  d1_desc* d_desc = nullptr;
  int* d_g0 = nullptr;
  float* d_bc = nullptr;
  unsigned long long* d_sig = nullptr;
  cudaError_t e = cudaMalloc(&d_buf, sizeof(float) * cnt * 2 * n_chares);
  if (e == cudaSuccess) e = cudaMalloc(&d_desc, sizeof(d1_desc) * n_chares);
  if (e == cudaSuccess) e = cudaMalloc(&d_g0, sizeof(int) * n_chares);
  if (e == cudaSuccess) e = cudaMalloc(&d_bc, sizeof(float) * ny);
  if (e == cudaSuccess) e = cudaMalloc(&d_sig, sizeof(unsigned long long) * (2 * (size_t)n_chares + 8));
  if (e == cudaSuccess) e = cudaMemset(d_buf, 0, sizeof(float) * cnt * 2 * n_chares);
  if (e == cudaSuccess) e = cudaMemset(d_sig, 0, sizeof(unsigned long long) * (2 * (size_t)n_chares + 8));
  if (e == cudaSuccess) e = cudaMemcpy(d_desc, descs.data(), sizeof(d1_desc) * n_chares, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_g0, g0.data(), sizeof(int) * n_chares, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_bc, bc.data(), sizeof(float) * ny, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    d1_init_kernel<<<148, 256>>>(d_buf, cnt, d_desc, d_g0, d_bc, n_chares, nx);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) {
    suite::app_params p{};
    p.id = suite::APP_DECOMP1D;
    p.a[0] = n_chares;
    p.a[1] = nx;
    p.a[2] = iters;
    p.a[3] = mode;
    p.a[4] = (long long)cnt;
    p.p[0] = d_buf;
    p.p[1] = d_desc;
    p.p[2] = d_sig;
    p.p[3] = d_sig + 2 * (size_t)n_chares;
    rc = suite_run(p);
    size_t row = 0;
    for (int i = 0; i < n_chares && e == cudaSuccess; i++) {
      const float* a = d_buf + ((size_t)i * 2 + (iters & 1)) * cnt + nx;
      e = cudaMemcpy(host_out + row * nx, a, sizeof(float) * nx * descs[i].chunk, cudaMemcpyDeviceToHost);
      row += descs[i].chunk;
    }
    charming_stats st;
    charming_last_stats(&st);
    if (out_ms) *out_ms = st.loop_ms;
  }
  cudaFree(d_buf);
  cudaFree(d_desc);
  cudaFree(d_g0);
  cudaFree(d_bc);
  cudaFree(d_sig);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "decomp1d");
  return rc;
}
#endif
