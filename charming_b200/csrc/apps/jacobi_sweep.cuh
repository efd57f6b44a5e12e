// Jacobi sweep of one chare block, executed inside an entry method by all
// threads of the PE block.
//
// Arithmetic (reference examples/jacobi2d/jacobi2d.cu:327-334):
//   new = (c + l + r + u + d) * 0.2, added left to right in T, one multiply
//   by the double 0.2 for double grids. Float grids (the reference has none)
//   add in float and multiply by 0.2 as the float pair C_HI + C_LO
//   (C_HI = 0.2f, C_LO = the float nearest 0.2 - C_HI) with one FMA:
//   fma(s, C_HI, s * C_LO), within an ulp of the product with the double
//   0.2 and without its two conversions. Written with _rn intrinsics so no
//   contraction can change it.
//
// Block layout in HBM (per chare, two buffers): rows 0..h+1 (0 and h+1 are
// ghost rows), row pitch `pitch` elements (a multiple of 128 bytes); column
// c in 0..w+1 sits at element OFF-1+c, so the first interior column starts
// on a 128-byte boundary (OFF = 128 / sizeof(T)).
//
// Two implementations with identical results:
//   sweep_direct: warps walk column strips down the rows, keeping three
//                 rows in registers (each input row loaded once per strip).
//   sweep_tma:    rows stream through a ring of shared-memory slots filled
//                 by cp.async.bulk (TMA 1-D bulk copies, no multicast), one
//                 mbarrier per slot; each input row is read from HBM once
//                 per column tile, so the compulsory traffic is one read and
//                 one write per point (16 B/LUP FP64, 8 B/LUP FP32).
#pragma once

#include <climits>
#include "suite.cuh"
#include "jacobi_types.cuh"

namespace jac {

template <typename T> struct traits;
template <> struct traits<double> {
  static constexpr int VEC = 2;   // elements per 16-byte vector
  static constexpr int OFF = 16;  // element offset of interior column 1
  static constexpr int TW_MAX = 1024;
};
template <> struct traits<float> {
  static constexpr int VEC = 4;
  static constexpr int OFF = 32;
  static constexpr int TW_MAX = 2048;
};

__device__ __forceinline__ double stencil(double c, double l, double r, double u, double d) {
  return __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(c, l), r), u), d), 0.2);
}
constexpr float STENCIL_C_HI = 0.2f;                     // 0x3e4ccccd
constexpr float STENCIL_C_LO = -2.9802322831784522e-09f;  // 0xb14ccccd: 0.2 - C_HI, rounded
__device__ __forceinline__ float stencil(float c, float l, float r, float u, float d) {
  float s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(c, l), r), u), d);
  return __fmaf_rn(s, STENCIL_C_HI, __fmul_rn(s, STENCIL_C_LO));
}
// Residual term (S(u) - u)^2 with S in FP64.
template <typename T>
__device__ __forceinline__ double resid2(T c, T l, T r, T u, T d) {
  double s = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn((double)c, (double)l), (double)r),
                                           (double)u), (double)d), 0.2);
  double e = __dsub_rn(s, (double)c);
  return __dmul_rn(e, e);
}

template <typename T>
struct block_view {
  T* base;      // element (row 0, column 0 of the pitched layout)
  int pitch;    // elements
  __device__ __forceinline__ T* row(int r) const { return base + (size_t)r * pitch; }
  // pointer to column c (0..w+1) of row r
  __device__ __forceinline__ T* at(int r, int c) const {
    return base + (size_t)r * pitch + traits<T>::OFF - 1 + c;
  }
};

// Computes VEC outputs of one row from the 5 input vectors and stores the
// valid ones. mid points at interior column j0 of the row (vector aligned),
// left/right are the scalars at j0-1 and j0+VEC. Returns the residual sum.
template <typename T, bool RESID>
__device__ __forceinline__ double compute_vec(const T* up, const T* mid, const T* dn, T left,
    T right, T* out, int nvalid) {
  constexpr int V = traits<T>::VEC;
  T u[V], m[V], d[V], o[V];
  if (V == 2) {
    double2 a = *reinterpret_cast<const double2*>(up);
    double2 b = *reinterpret_cast<const double2*>(mid);
    double2 c = *reinterpret_cast<const double2*>(dn);
    u[0] = (T)a.x; u[1] = (T)a.y; m[0] = (T)b.x; m[1] = (T)b.y; d[0] = (T)c.x; d[1] = (T)c.y;
  } else {
    float4 a = *reinterpret_cast<const float4*>(up);
    float4 b = *reinterpret_cast<const float4*>(mid);
    float4 c = *reinterpret_cast<const float4*>(dn);
    u[0] = (T)a.x; u[1] = (T)a.y; u[2] = (T)a.z; u[3] = (T)a.w;
    m[0] = (T)b.x; m[1] = (T)b.y; m[2] = (T)b.z; m[3] = (T)b.w;
    d[0] = (T)c.x; d[1] = (T)c.y; d[2] = (T)c.z; d[3] = (T)c.w;
  }
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < V; k++) {
    T l = (k == 0) ? left : m[k - 1];
    T r = (k == V - 1) ? right : m[k + 1];
    o[k] = stencil(m[k], l, r, u[k], d[k]);
    if (RESID && k < nvalid) acc += resid2<T>(m[k], l, r, u[k], d[k]);
  }
  if (nvalid == V) {
    if (V == 2) {
      *reinterpret_cast<double2*>(out) = make_double2((double)o[0], (double)o[1]);
    } else {
      *reinterpret_cast<float4*>(out) = make_float4((float)o[0], (float)o[1], (float)o[2], (float)o[3]);
    }
  } else {
    #pragma unroll
    for (int k = 0; k < V; k++)  // static indices keep o[] in registers
      if (k < nvalid) out[k] = o[k];
  }
  return acc;
}

// ---------------------------------------------------------------------------
// PTX helpers: mbarriers, bulk copies, per-thread async copies.
// ---------------------------------------------------------------------------
#ifndef CHARMING_HOST_EMULATION
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long* b) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" :: "r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(b)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done) : "r"(smem_u32(b)), "r"(parity) : "memory");
  return done != 0;
}
// 1-D bulk copy global -> shared, completion counted on the mbarrier.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
    unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(b)) : "memory");
}
// 16-byte asynchronous global -> shared copy (zero fill when src_bytes is 0),
// committed per row; wait_group<N> waits until at most N groups are pending.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* b, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done) : "r"(smem_u32(b)), "r"(parity) : "memory");
  return done != 0;
}
#else
// The CPU check of the chare code models these (tests/emu).
void mbar_init(unsigned long long* b, unsigned count);
void mbar_inval(unsigned long long* b);
void mbar_expect_tx(unsigned long long* b, unsigned bytes);
bool mbar_try_wait(unsigned long long* b, unsigned parity);
bool mbar_test_wait(unsigned long long* b, unsigned parity);
void mbar_arrive(unsigned long long* b);
void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar);
inline void fence_proxy_async_global() {}
inline void fence_proxy_async_smem() {}
inline void fence_mbar_init() {}
// per-thread copies: done at once on the host
inline void cp_async16(void* dst, const void* src, unsigned src_bytes) {
  memset(dst, 0, 16);
  if (src_bytes) memcpy(dst, src, src_bytes);
}
inline void cp_async_commit() {}
template <int N> inline void cp_async_wait() {}
#endif

// ---------------------------------------------------------------------------
// Direct-load sweep, simple form: thread i of the block handles vectors
// i, i+n, ... of the (h rows x ceil(w/VEC) vectors) output. Used for blocks
// of fewer than 32 threads.
// ---------------------------------------------------------------------------
template <typename T, bool RESID>
__device__ double sweep_simple(block_view<T> in, block_view<T> out, int w, int h) {
  constexpr int V = traits<T>::VEC;
  const int nv = (w + V - 1) / V;
  const long long total = (long long)nv * h;
  double acc = 0.0;
  for (long long x = threadIdx.x; x < total; x += blockDim.x) {
    int r = (int)(x / nv) + 1;
    int v = (int)(x % nv);
    int j0 = 1 + v * V;
    const T* mid = in.at(r, j0);
    int nvalid = min(V, w - v * V);
    acc += compute_vec<T, RESID>(in.at(r - 1, j0), mid, in.at(r + 1, j0), mid[-1], mid[V],
                                 out.at(r, j0), nvalid);
  }
  return acc;
}

// ---------------------------------------------------------------------------
// Direct-load sweep, strip walker. The block's work is split into items: a
// column strip of 32*J vectors (lane l of a warp owns vectors l, l+32, ...)
// times a run of rows. A warp walks its rows top to bottom keeping the
// rows above, at and below the output row in registers, so each input row
// is loaded once per strip; it loads G rows ahead at a time, which keeps
// G*J 16-byte loads per thread in flight. Left/right neighbours come from
// the neighbouring lanes by shuffle; only the strip's two edge columns are
// loaded as scalars. No block barrier inside the sweep.
// ---------------------------------------------------------------------------
template <typename T> struct vec_of;
template <> struct vec_of<double> { using type = double2; };
template <> struct vec_of<float> { using type = float4; };

template <typename T, int J>
struct walk_row {
  typename vec_of<T>::type v[J];
  T left, right;  // columns just outside the strip (same for all lanes)
};

template <typename T>
__device__ __forceinline__ T vec_elem(const double2& x, int k) { return (T)(k == 0 ? x.x : x.y); }
template <typename T>
__device__ __forceinline__ T vec_elem(const float4& x, int k) {
  return (T)(k == 0 ? x.x : k == 1 ? x.y : k == 2 ? x.z : x.w);
}

// Loads row r of a strip: vector v_j = vbase + lane + 32 j when v_j <= nv
// (vector nv holds the right ghost column and padding, inside the pitched
// row), plus the two edge scalars.
template <typename T, int J>
__device__ __forceinline__ void walk_load(walk_row<T, J>& R, const block_view<T>& in, int r,
    int vbase, int nv, int lane, bool has_right) {
  constexpr int V = traits<T>::VEC;
  using VT = typename vec_of<T>::type;
  const T* row = in.at(r, 1);
#pragma unroll
  for (int j = 0; j < J; j++) {
    int v = vbase + lane + 32 * j;
    if (v <= nv) R.v[j] = *reinterpret_cast<const VT*>(row + (size_t)v * V);
    else R.v[j] = VT{};
  }
  R.left = row[(size_t)vbase * V - 1];
  R.right = has_right ? row[(size_t)(vbase + 32 * J) * V] : (T)0;
}

template <typename T, bool RESID, int J>
__device__ __forceinline__ double walk_compute(const walk_row<T, J>& U, const walk_row<T, J>& M,
    const walk_row<T, J>& D, T* orow, int vbase, int w, int lane) {
  constexpr int V = traits<T>::VEC;
  constexpr unsigned FULL = 0xffffffffu;
  using VT = typename vec_of<T>::type;
  double acc = 0.0;
  T first[J], last[J];
#pragma unroll
  for (int j = 0; j < J; j++) {
    first[j] = vec_elem<T>(M.v[j], 0);
    last[j] = vec_elem<T>(M.v[j], V - 1);
  }
#pragma unroll
  for (int j = 0; j < J; j++) {
    T up_last = __shfl_up_sync(FULL, last[j], 1);
    T dn_first = __shfl_down_sync(FULL, first[j], 1);
    T wrap_l = __shfl_sync(FULL, last[j > 0 ? j - 1 : 0], 31);
    T wrap_r = __shfl_sync(FULL, first[j < J - 1 ? j + 1 : 0], 0);
    T left = lane > 0 ? up_last : (j > 0 ? wrap_l : M.left);
    T right = lane < 31 ? dn_first : (j < J - 1 ? wrap_r : M.right);
    int v = vbase + lane + 32 * j;
    int nvalid = w - v * V;
    if (nvalid > 0) {
      if (nvalid > V) nvalid = V;
      T m[V], u[V], d[V], o[V];
#pragma unroll
      for (int k = 0; k < V; k++) {
        m[k] = vec_elem<T>(M.v[j], k);
        u[k] = vec_elem<T>(U.v[j], k);
        d[k] = vec_elem<T>(D.v[j], k);
      }
#pragma unroll
      for (int k = 0; k < V; k++) {
        T l = (k == 0) ? left : m[k - 1];
        T r = (k == V - 1) ? right : m[k + 1];
        o[k] = stencil(m[k], l, r, u[k], d[k]);
        if (RESID && k < nvalid) acc += resid2<T>(m[k], l, r, u[k], d[k]);
      }
      T* op = orow + (size_t)v * V;
      if (nvalid == V) {
        VT ov;
        if constexpr (V == 2) ov = make_double2((double)o[0], (double)o[1]);
        else ov = make_float4((float)o[0], (float)o[1], (float)o[2], (float)o[3]);
        *reinterpret_cast<VT*>(op) = ov;
      } else {
        #pragma unroll
        for (int k = 0; k < V; k++)  // static indices keep o[] in registers
          if (k < nvalid) op[k] = o[k];
      }
    }
  }
  return acc;
}

// Rows r0..r1-1 of the strip starting at vector vbase (one warp).
template <typename T, bool RESID, int J, int G>
__device__ double walk_item(const block_view<T>& in, const block_view<T>& out, int w, int nv,
    int vbase, int r0, int r1, int lane) {
  const bool has_right = vbase + 32 * J <= nv;
  walk_row<T, J> U, M, D[G];
  walk_load<T, J>(U, in, r0 - 1, vbase, nv, lane, has_right);
  walk_load<T, J>(M, in, r0, vbase, nv, lane, has_right);
  double acc = 0.0;
  for (int r = r0; r < r1; r += G) {
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (r + 1 + g <= r1) walk_load<T, J>(D[g], in, r + 1 + g, vbase, nv, lane, has_right);
    }
#pragma unroll
    for (int g = 0; g < G; g++) {
      if (r + g < r1) {
        acc += walk_compute<T, RESID, J>(U, M, D[g], out.at(r + g, 1), vbase, w, lane);
        U = M;
        M = D[g];
      }
    }
  }
  return acc;
}

template <typename T> struct walk_shape;
template <> struct walk_shape<double> { static constexpr int J = 2, G = 4; };
template <> struct walk_shape<float> { static constexpr int J = 2, G = 4; };

// Not inlined: the walker gets the whole register budget, whatever the
// caller keeps live.
template <typename T, bool RESID>
__device__ __noinline__ double sweep_direct(block_view<T> in, block_view<T> out, int w, int h) {
  if (blockDim.x < 32) return sweep_simple<T, RESID>(in, out, w, h);
  constexpr int V = traits<T>::VEC, J = walk_shape<T>::J, G = walk_shape<T>::G;
  const int nv = (w + V - 1) / V;
  const int n_strips = (nv + 32 * J - 1) / (32 * J);
  const int nw = (int)(blockDim.x / 32), warp = (int)(threadIdx.x / 32), lane = (int)(threadIdx.x & 31);
  if (warp >= nw) return 0.0;  // threads of a partial warp (host emulation only)
  // Enough row runs that every warp gets an item; runs of at least 8 rows.
  int segs = (nw + n_strips - 1) / n_strips;
  if (segs > (h + 7) / 8) segs = (h + 7) / 8;
  if (segs < 1) segs = 1;
  const int items = n_strips * segs;
  double acc = 0.0;
  for (int it = warp; it < items; it += nw) {
    int s = it % n_strips, g = it / n_strips;
    int r0 = 1 + (int)((long long)h * g / segs), r1 = 1 + (int)((long long)h * (g + 1) / segs);
    acc += walk_item<T, RESID, J, G>(in, out, w, nv, s * 32 * J, r0, r1, lane);
  }
  return acc;
}

// ---------------------------------------------------------------------------
// Multi-sweep pass (temporal blocking): L sweeps (2 <= L <= LMAX) from a
// grid whose ghost zone is at least L deep, without writing the
// intermediate sweeps. A warp owns a strip of 32 vectors (one per lane) and
// streams level-0 rows down it; level l row r is computed when level l-1
// row r+1 arrives, from a three-row register window per level, so the pass
// is a wavefront L rows deep. Every level loses one valid column at each
// strip edge (the neighbour value is in another warp), so strips overlap by
// 2*ceil(L/VEC) vectors and each owns the 32 - 2*ceil(L/VEC) in the middle;
// row runs overlap by 2L rows. Cells on the domain boundary (row 0 / h+1,
// column 0 / w+1 of a chare without a neighbour there) keep their value at
// every level; cells beyond it are never used by a stored result. Each
// stored value is computed from the same five operands in the same order as
// a single sweep, so L passes of one sweep give the same bits.
// `fixed`: bit 0 top, 1 bottom, 2 left, 3 right side is the domain boundary.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void vec_to(const typename vec_of<T>::type& x, T (&a)[traits<T>::VEC]) {
#pragma unroll
  for (int k = 0; k < traits<T>::VEC; k++) a[k] = vec_elem<T>(x, k);
}
__device__ __forceinline__ double2 vec_from(const double (&a)[2]) { return make_double2(a[0], a[1]); }
__device__ __forceinline__ float4 vec_from(const float (&a)[4]) {
  return make_float4(a[0], a[1], a[2], a[3]);
}

// Per-lane constants of one strip item.
template <typename T>
struct deep_lane {
  bool own;                        // this lane stores its vector / counts the residual
  int v, col0;                     // vector index, its first column
  bool fixc[traits<T>::VEC];       // column on the domain boundary (kept at every level)
  bool inw[traits<T>::VEC];        // column inside the chare (1..w)
  bool anyfix;                     // some fixc[k]
  int fix_r0, fix_r1;              // rows kept at every level (0 / h+1), or INT_MIN
};

// The lane constants of the strip whose owned vectors are own0..own0+nown-1
// (the lane's vector starts E = ceil(L/VEC) vectors before them).
template <typename T, int L>
__device__ __forceinline__ deep_lane<T> make_lane(int w, int h, int fixed, int own0, int nown, int lane) {
  constexpr int V = traits<T>::VEC, E = (L + V - 1) / V;
  deep_lane<T> ln;
  ln.v = own0 - E + lane;
  ln.col0 = 1 + ln.v * V;
  ln.own = ln.v >= own0 && ln.v < own0 + nown;
  ln.anyfix = false;
#pragma unroll
  for (int k = 0; k < V; k++) {
    const int c = ln.col0 + k;
    ln.fixc[k] = (c == 0 && (fixed & 4)) || (c == w + 1 && (fixed & 8));
    ln.inw[k] = c >= 1 && c <= w;
    ln.anyfix = ln.anyfix || ln.fixc[k];
  }
  ln.fix_r0 = (fixed & 1) ? 0 : INT_MIN;
  ln.fix_r1 = (fixed & 2) ? h + 1 : INT_MIN;
  return ln;
}

// All L levels of the wavefront at sub-step K of a three-step cycle (level-l
// row r lives in W[l][(r - qs) mod 3], so every window index is static).
// CHECK: a level runs only once its three input rows exist (the first 2L
// steps of an item). Domain-boundary cells keep their value at every level:
// a whole row by a warp-uniform branch, a column by a per-lane fix-up.
// ROWFIX / COLFIX false: the step cannot meet a domain-boundary row / the
// strip holds no domain-boundary column, so those tests are left out.
template <typename T, bool RESID, int L, int K, bool CHECK, bool ROWFIX = true, bool COLFIX = true>
__device__ __forceinline__ void deep_step(typename vec_of<T>::type (&W)[L][3], int q, int qs, int w,
    const deep_lane<T>& ln, int r0, int r1, const block_view<T>& out, double& acc) {
  constexpr int V = traits<T>::VEC;
  constexpr unsigned FULL = 0xffffffffu;
  using VT = typename vec_of<T>::type;
#pragma unroll
  for (int l = 1; l <= L; l++) {
    if (CHECK && q < qs + 2 * l) continue;
    const int r = q - l;  // row of level l computed now
    const int su = ((K - l - 1) % 3 + 6) % 3, sm = ((K - l) % 3 + 6) % 3, sd = ((K - l + 1) % 3 + 6) % 3;
    T m[V], u[V], d[V], o[V];
    vec_to<T>(W[l - 1][sm], m);
    vec_to<T>(W[l - 1][su], u);
    vec_to<T>(W[l - 1][sd], d);
    T left = __shfl_up_sync(FULL, m[V - 1], 1);
    T right = __shfl_down_sync(FULL, m[0], 1);
    if (ROWFIX && (r == ln.fix_r0 || r == ln.fix_r1)) {  // domain-boundary row: kept (warp-uniform)
#pragma unroll
      for (int k = 0; k < V; k++) o[k] = m[k];
    } else {
#pragma unroll
      for (int k = 0; k < V; k++) {
        T lk = (k == 0) ? left : m[k - 1];
        T rk = (k == V - 1) ? right : m[k + 1];
        o[k] = stencil(m[k], lk, rk, u[k], d[k]);
        if (RESID && l == 1 && ln.own && ln.inw[k] && r >= r0 && r < r1)
          acc += resid2<T>(m[k], lk, rk, u[k], d[k]);
      }
      if (COLFIX && ln.anyfix) {  // the lane holding column 0 or w+1 of the domain
#pragma unroll
        for (int k = 0; k < V; k++)
          if (ln.fixc[k]) o[k] = m[k];
      }
    }
    if (l == L) {
      if (ln.own) {
        T* op = out.at(r, ln.col0);
        int nvalid = w - ln.v * V;
        if (nvalid >= V) {
          *reinterpret_cast<VT*>(op) = vec_from(o);
        } else {
          #pragma unroll
        for (int k = 0; k < V; k++)  // static indices keep o[] in registers
          if (k < nvalid) op[k] = o[k];
        }
      }
    } else {
      W[l][sm] = vec_from(o);
    }
  }
}

// One strip item: level-0 rows stream through this lane's private ring of P
// 16-byte slots in shared memory (cp.async, P-1 rows ahead), the levels
// through registers.
template <typename T, int P>
__device__ __forceinline__ void deep_fetch(typename vec_of<T>::type* ring, int lane, int& slot, int q,
    int qe, const block_view<T>& in, long long eo, unsigned nb, typename vec_of<T>::type& x) {
  cp_async_wait<P - 2>();
  x = ring[slot * 32 + lane];
  const int nslot = slot == 0 ? P - 1 : slot - 1;  // slot of row q-1, read last step
  if (q + P - 1 <= qe) cp_async16(&ring[nslot * 32 + lane], in.row(q + P - 1) + eo, nb);
  cp_async_commit();
  slot = slot + 1 == P ? 0 : slot + 1;
}

template <typename T, bool RESID, int L, int P>
__device__ __forceinline__ double deep_item(const block_view<T>& in, const block_view<T>& out, int w,
    const deep_lane<T>& ln, int r0, int r1, int lane, typename vec_of<T>::type* ring) {
  constexpr int V = traits<T>::VEC;
  using VT = typename vec_of<T>::type;
  const long long e0 = (long long)traits<T>::OFF - 1 + ln.col0;  // element index in a row
  const bool can_load = e0 >= 0 && e0 + V <= in.pitch;
  const long long eo = can_load ? e0 : 0;
  const unsigned nb = can_load ? 16u : 0u;
  const int qs = r0 - L, qe = r1 - 1 + L;             // level-0 rows streamed
#pragma unroll
  for (int k = 0; k < P - 1; k++) {
    if (qs + k <= qe) cp_async16(&ring[k * 32 + lane], in.row(qs + k) + eo, nb);
    cp_async_commit();
  }
  VT W[L][3];
  double acc = 0.0;
  int slot = 0;                                       // ring slot of row q
  // fill: until every level has its three rows (checked steps)
  constexpr int F = (2 * L + 2) / 3 * 3;
  int q0 = qs;
  for (; q0 < qs + F && q0 <= qe; q0 += 3) {
#pragma unroll
    for (int K = 0; K < 3; K++) {
      const int q = q0 + K;
      if (q > qe) break;
      deep_fetch<T, P>(ring, lane, slot, q, qe, in, eo, nb, W[0][K]);
      if (K == 0) deep_step<T, RESID, L, 0, true>(W, q, qs, w, ln, r0, r1, out, acc);
      else if (K == 1) deep_step<T, RESID, L, 1, true>(W, q, qs, w, ln, r0, r1, out, acc);
      else deep_step<T, RESID, L, 2, true>(W, q, qs, w, ln, r0, r1, out, acc);
    }
  }
  // steady state: all levels every step
  for (; q0 <= qe; q0 += 3) {
#pragma unroll
    for (int K = 0; K < 3; K++) {
      const int q = q0 + K;
      if (q > qe) break;
      deep_fetch<T, P>(ring, lane, slot, q, qe, in, eo, nb, W[0][K]);
      if (K == 0) deep_step<T, RESID, L, 0, false>(W, q, qs, w, ln, r0, r1, out, acc);
      else if (K == 1) deep_step<T, RESID, L, 1, false>(W, q, qs, w, ln, r0, r1, out, acc);
      else deep_step<T, RESID, L, 2, false>(W, q, qs, w, ln, r0, r1, out, acc);
    }
  }
  cp_async_wait<0>();
  return acc;
}

// ---------------------------------------------------------------------------
// The same item, with the tests taken out of the steady state: a group of
// three steps that cannot need them (past the fill, before the steps that
// can meet the bottom boundary row, in a strip without a domain-boundary
// column) runs a step without the fill check, the boundary-row test and the
// column fix-up; the other groups run the general step. One loop and two
// step versions keep the code (and so the instruction cache footprint) as
// small as deep_item's. Same arithmetic and results as deep_item.
// ---------------------------------------------------------------------------
template <typename T, bool RESID, int L, int P>
__device__ __forceinline__ double lean_item(const block_view<T>& in, const block_view<T>& out, int w,
    const deep_lane<T>& ln, int r0, int r1, int lane, typename vec_of<T>::type* ring) {
  constexpr int V = traits<T>::VEC;
  using VT = typename vec_of<T>::type;
  const long long e0 = (long long)traits<T>::OFF - 1 + ln.col0;  // element index in a row
  const bool can_load = e0 >= 0 && e0 + V <= in.pitch;
  const long long eo = can_load ? e0 : 0;
  const unsigned nb = can_load ? 16u : 0u;
  const int qs = r0 - L, qe = r1 - 1 + L;  // level-0 rows streamed
  constexpr int F = (2 * L + 2) / 3 * 3;   // steps of the fill (every level has its rows after)
  // steady groups: from the end of the fill to before the first step at
  // which a level can compute the bottom boundary row R (level l computes
  // row q - l, so levels 1..L-1 reach R at steps R+1..R+L-1); none in a
  // strip holding a domain-boundary column
  int q_lean_end = (ln.fix_r1 != INT_MIN && ln.fix_r1 + 1 <= qe) ? ln.fix_r1 + 1 : qe + 1;
  if (__any_sync(0xffffffffu, ln.anyfix)) q_lean_end = INT_MIN;
#pragma unroll
  for (int k = 0; k < P - 1; k++) {
    if (qs + k <= qe) cp_async16(&ring[k * 32 + lane], in.row(qs + k) + eo, nb);
    cp_async_commit();
  }
  VT W[L][3];
  double acc = 0.0;
  int slot = 0;
  for (int q0 = qs; q0 <= qe; q0 += 3) {
    if (q0 >= qs + F && q0 + 2 < q_lean_end) {
      deep_fetch<T, P>(ring, lane, slot, q0, qe, in, eo, nb, W[0][0]);
      deep_step<T, RESID, L, 0, false, false, false>(W, q0, qs, w, ln, r0, r1, out, acc);
      deep_fetch<T, P>(ring, lane, slot, q0 + 1, qe, in, eo, nb, W[0][1]);
      deep_step<T, RESID, L, 1, false, false, false>(W, q0 + 1, qs, w, ln, r0, r1, out, acc);
      deep_fetch<T, P>(ring, lane, slot, q0 + 2, qe, in, eo, nb, W[0][2]);
      deep_step<T, RESID, L, 2, false, false, false>(W, q0 + 2, qs, w, ln, r0, r1, out, acc);
    } else {
#pragma unroll
      for (int K = 0; K < 3; K++) {
        const int q = q0 + K;
        if (q > qe) break;
        deep_fetch<T, P>(ring, lane, slot, q, qe, in, eo, nb, W[0][K]);
        if (K == 0) deep_step<T, RESID, L, 0, true>(W, q, qs, w, ln, r0, r1, out, acc);
        else if (K == 1) deep_step<T, RESID, L, 1, true>(W, q, qs, w, ln, r0, r1, out, acc);
        else deep_step<T, RESID, L, 2, true>(W, q, qs, w, ln, r0, r1, out, acc);
      }
    }
  }
  cp_async_wait<0>();
  return acc;
}

// The same pass, computed by thread 0 alone for blocks under one warp, with
// levels 1..L-1 kept as three-row rings in the block's scratch.
template <typename T, bool RESID>
__device__ double sweep_deep_simple(block_view<T> in, block_view<T> out, int w, int h, int L,
    int fixed) {
  if (threadIdx.x != 0) return 0.0;
  size_t cap = 0;
  T* ring = reinterpret_cast<T*>(charm::smem_scratch(&cap));
  const int W = w + 2 * L;  // columns 1-L .. w+L
  if ((size_t)(L - 1) * 3 * W * sizeof(T) > cap) {
    charm::detail::report_error(CHARMING_ERR_CONFIG, w, L);
    return 0.0;
  }
  auto slot = [&](int l, int r) -> T* { return ring + ((size_t)(l - 1) * 3 + ((r % 3) + 3) % 3) * W; };
  auto lv = [&](int l, int r, int c) -> T { return l == 0 ? *in.at(r, c) : slot(l, r)[c + L - 1]; };
  double acc = 0.0;
  for (int q = 1 - L; q <= h + L; q++) {
    for (int l = 1; l <= L; l++) {
      const int r = q - l, ext = L - l;
      if (r < 1 - ext || r > h + ext) continue;
      const bool fixr = (r == 0 && (fixed & 1)) || (r == h + 1 && (fixed & 2));
      for (int c = 1 - ext; c <= w + ext; c++) {
        const bool fixc = (c == 0 && (fixed & 4)) || (c == w + 1 && (fixed & 8));
        T m = lv(l - 1, r, c), v = m;
        if (!fixr && !fixc) {
          T lc = lv(l - 1, r, c - 1), rc = lv(l - 1, r, c + 1);
          T up = lv(l - 1, r - 1, c), dn = lv(l - 1, r + 1, c);
          v = stencil(m, lc, rc, up, dn);
          if (RESID && l == 1 && r >= 1 && r <= h && c >= 1 && c <= w)
            acc += resid2<T>(m, lc, rc, up, dn);
        }
        if (l == L) {
          if (r >= 1 && r <= h && c >= 1 && c <= w) *out.at(r, c) = v;
        } else {
          slot(l, r)[c + L - 1] = v;
        }
      }
    }
  }
  return acc;
}

// The items of one pass of L sweeps (one warp); one register allocation per L.
template <typename T, bool RESID, int L, bool LEAN>
__device__ __noinline__ double sweep_deep_items(block_view<T> in, block_view<T> out, int w, int h,
    int fixed, typename vec_of<T>::type* ring, int nw, int warp, int lane) {
  constexpr int V = traits<T>::VEC, P = 8;
  constexpr int E = (L + V - 1) / V;    // vectors lost at each strip edge over L levels
  constexpr int SS = 32 - 2 * E;        // vectors a strip owns
  const int nv = (w + V - 1) / V;
  const int n_strips = (nv + SS - 1) / SS;
  // row runs: balance items over warps; each run at least 4L rows
  int segs = 1, best = 0x7fffffff;
  for (int sg = 1; sg <= 8; sg++) {
    if (sg > 1 && h / sg < 4 * L) break;
    int rounds = (n_strips * sg + nw - 1) / nw;
    int cost = rounds * ((h + sg - 1) / sg + 2 * L);
    if (cost < best) {
      best = cost;
      segs = sg;
    }
  }
  const int items = n_strips * segs;
  double acc = 0.0;
  for (int it = warp; it < items; it += nw) {
    int s = it % n_strips, g = it / n_strips;
    int r0 = 1 + (int)((long long)h * g / segs), r1 = 1 + (int)((long long)h * (g + 1) / segs);
    int own0 = s * SS;
    int nown = min(SS, nv - own0);
    const deep_lane<T> ln = make_lane<T, L>(w, h, fixed, own0, nown, lane);
    if (LEAN) acc += lean_item<T, RESID, L, P>(in, out, w, ln, r0, r1, lane, ring);
    else acc += deep_item<T, RESID, L, P>(in, out, w, ln, r0, r1, lane, ring);
  }
  return acc;
}

// lean: the phase-split items (lean_item) instead of deep_item; same
// results bit for bit.
template <typename T, bool RESID>
__device__ __noinline__ double sweep_deep(block_view<T> in, block_view<T> out, int w, int h, int L,
    int fixed, bool lean = true) {
  if (blockDim.x < 32) return sweep_deep_simple<T, RESID>(in, out, w, h, L, fixed);
  using VT = typename vec_of<T>::type;
  const int P = 8;
  const int nw = (int)(blockDim.x / 32), warp = (int)(threadIdx.x / 32), lane = (int)(threadIdx.x & 31);
  if (warp >= nw) return 0.0;
  size_t sbytes = 0;
  VT* rings = reinterpret_cast<VT*>(charm::smem_scratch(&sbytes));
  if ((size_t)nw * P * 32 * sizeof(VT) > sbytes) {
    if (threadIdx.x == 0) charm::detail::report_error(CHARMING_ERR_CONFIG, (int)sbytes, nw);
    return 0.0;
  }
  VT* ring = rings + (size_t)warp * P * 32;
#define CHARMING_DEEP_CASE(LL)                                                                 \
  if (L == LL)                                                                                 \
    return lean ? sweep_deep_items<T, RESID, LL, true>(in, out, w, h, fixed, ring, nw, warp, lane) \
                : sweep_deep_items<T, RESID, LL, false>(in, out, w, h, fixed, ring, nw, warp, lane);
  CHARMING_DEEP_CASE(2)
  CHARMING_DEEP_CASE(3)
  CHARMING_DEEP_CASE(5)
  CHARMING_DEEP_CASE(6)
  CHARMING_DEEP_CASE(7)
  CHARMING_DEEP_CASE(8)
#undef CHARMING_DEEP_CASE
  return lean ? sweep_deep_items<T, RESID, 4, true>(in, out, w, h, fixed, ring, nw, warp, lane)
              : sweep_deep_items<T, RESID, 4, false>(in, out, w, h, fixed, ring, nw, warp, lane);
}

// ---------------------------------------------------------------------------
// TMA row pipeline.
// ---------------------------------------------------------------------------

constexpr int MAX_SLOTS = 64;        // mbarrier pairs in the first 1 KiB
constexpr int BAR_BYTES = 2 * MAX_SLOTS * 8;

// Column tiling and ring size of one sweep. Each warp owns a strip of
// 32 * VEC columns of the tile and walks all rows of it.
struct tma_plan {
  int ntiles;     // column tiles
  int tws;        // tile stride (columns), multiple of VEC
  int NS;         // ring slots (rows in flight)
  int slot_elems; // elements per slot
};

template <typename T>
__host__ __device__ inline size_t tma_slot_bytes(int tws) {
  size_t e = (size_t)tws + 2 * traits<T>::VEC;
  return (e * sizeof(T) + 127) / 128 * 128;
}

template <typename T>
__device__ bool make_plan(int w, int nthreads, size_t smem_bytes, int tile_w_opt, tma_plan* p) {
  constexpr int V = traits<T>::VEC;
  int twmax = (nthreads / 32) * 32 * V;  // one vector per lane
  if (tile_w_opt > 0 && tile_w_opt < twmax) twmax = tile_w_opt;
  twmax = (twmax + V - 1) / V * V;
  p->ntiles = (w + twmax - 1) / twmax;
  int tw = (w + p->ntiles - 1) / p->ntiles;
  p->tws = (tw + V - 1) / V * V;
  size_t sb = tma_slot_bytes<T>(p->tws);
  p->slot_elems = (int)(sb / sizeof(T));
  size_t avail = smem_bytes > (size_t)BAR_BYTES ? smem_bytes - BAR_BYTES : 0;
  long ns = (long)(avail / sb);
  if (ns > MAX_SLOTS) ns = MAX_SLOTS;
  p->NS = (int)ns;
  return p->NS >= 4;
}

// One sweep in -> out. Row segments (tile columns + 16-byte halo each side)
// stream through NS shared-memory slots. full[s] completes when the bulk
// copy into slot s landed; empty[s] when every warp is done with it. Lane 0
// of warp 0 issues copies whenever a slot is empty (it also polls while
// waiting, so it never blocks the pipeline it feeds). Returns false (error
// recorded) if a wait ran out.
template <typename T, bool RESID>
__device__ bool sweep_tma(block_view<T> in, block_view<T> out, int w, int h, void* smem,
    size_t smem_bytes, const tma_plan& P, double* acc_out) {
  constexpr int V = traits<T>::VEC;
  constexpr int H = V;  // halo elements each side of a slot row (16 bytes)
  constexpr unsigned FULL = 0xffffffffu;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem);
  unsigned long long* empty = full + MAX_SLOTS;
  T* slots = reinterpret_cast<T*>(reinterpret_cast<char*>(smem) + BAR_BYTES);
  const int rows = h + 2;
  const long long total = (long long)P.ntiles * rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  __shared__ int s_fail;
  __shared__ long long s_issued;

  fence_proxy_async_global();  // earlier generic writes to `in` -> bulk copies
  if (threadIdx.x == 0) {
    for (int s = 0; s < P.NS; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (unsigned)nw);
    }
    fence_mbar_init();
    s_fail = 0;
  }
  __syncthreads();

  long long issued = 0;  // producer state (lane 0 of warp 0)
  auto try_issue = [&]() {
    while (issued < total) {
      long long j = issued;
      int s = (int)(j % P.NS);
      long long u = j / P.NS;
      if (u > 0 && !mbar_test_wait(&empty[s], (unsigned)((u - 1) & 1))) break;
      int t = (int)(j / rows), r = (int)(j % rows);
      int c0 = t * P.tws;
      int tw = min(P.tws, w - c0);
      unsigned bytes = (unsigned)(((size_t)(tw + 2 * H) * sizeof(T) + 15) / 16 * 16);
      // checked build: 16-byte aligned source, copy fits its slot
      if (!CHARM_VERIFY(((reinterpret_cast<uintptr_t>(in.row(r) + traits<T>::OFF + c0 - H) & 15) == 0) &&
                        bytes <= (unsigned)(P.slot_elems * sizeof(T)),
                        CHARMING_ERR_PIPELINE, (int)j, (int)bytes))
        break;
      mbar_expect_tx(&full[s], bytes);
      bulk_g2s(slots + (size_t)s * P.slot_elems, in.row(r) + traits<T>::OFF + c0 - H, bytes,
               &full[s]);
      issued = j + 1;
    }
  };
  const bool producer = (warp == 0 && lane == 0);
  if (producer) {
    fence_proxy_async_smem();
    try_issue();
  }
  __syncwarp();

  double acc = 0.0;
  bool fail = false;
  for (int t = 0; t < P.ntiles && !fail; t++) {
    const int c0 = t * P.tws;
    const int tw = min(P.tws, w - c0);
    const long long ibase = (long long)t * rows;
    const int v = warp * 32 + lane;      // vector of the tile row this lane owns
    const bool active = v * V < tw;
    const bool next_active = (v + 1) * V < tw;
    const int nvalid = active ? min(V, tw - v * V) : 0;
    const int s_off = H + v * V;         // slot element of interior column c0 + v*V
    for (int r = 0; r < rows; r++) {
      const long long j = ibase + r;
      const unsigned parity = (unsigned)((j / P.NS) & 1);
      unsigned long long* fb = &full[j % P.NS];
      unsigned spins = 0;
      while (true) {
        // The producer's warp must not be suspended inside try_wait while
        // copies wait to be issued: it polls with the non-blocking test.
        bool ok = (warp == 0) ? mbar_test_wait(fb, parity) : mbar_try_wait(fb, parity);
        if (__all_sync(FULL, ok)) break;
        if (producer) try_issue();
        __syncwarp();
        if (++spins > (1u << 22) || *reinterpret_cast<volatile int*>(&s_fail)) {
          fail = true;
          break;
        }
      }
      if (fail) break;
      if (r >= 2) {
        const T* up = slots + (size_t)((j - 2) % P.NS) * P.slot_elems;
        const T* mid = slots + (size_t)((j - 1) % P.NS) * P.slot_elems;
        const T* dn = slots + (size_t)(j % P.NS) * P.slot_elems;
        T m[V];
        if (active) {
          if (V == 2) {
            double2 b = *reinterpret_cast<const double2*>(mid + s_off);
            m[0] = (T)b.x;
            m[1] = (T)b.y;
          } else {
            float4 b = *reinterpret_cast<const float4*>(mid + s_off);
            m[0] = (T)b.x; m[1] = (T)b.y; m[2] = (T)b.z; m[3] = (T)b.w;
          }
        } else {
#pragma unroll
          for (int k = 0; k < V; k++) m[k] = (T)0;
        }
        T left = __shfl_up_sync(FULL, m[V - 1], 1);
        T right = __shfl_down_sync(FULL, m[0], 1);
        if (active) {
          if (lane == 0) left = mid[s_off - 1];
          if (lane == 31 || !next_active) right = mid[s_off + V];
          acc += compute_vec<T, RESID>(up + s_off, mid + s_off, dn + s_off, left, right,
                                       out.at(r - 1, 1 + c0 + v * V), nvalid);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[(j - 2) % P.NS]);
        if (producer) try_issue();
      }
    }
    if (!fail) {
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&empty[(ibase + h) % P.NS]);
        mbar_arrive(&empty[(ibase + h + 1) % P.NS]);
      }
    }
  }
  if (fail) atomicExch(&s_fail, 1);
  if (producer) s_issued = issued;
  __syncthreads();
  fail = s_fail != 0;
  if (threadIdx.x == 0) {
    if (fail) {
      // Let copies still in flight land before the slots are reused.
      for (long long j = (s_issued > P.NS ? s_issued - P.NS : 0); j < s_issued; j++) {
        unsigned spins = 0;
        while (!mbar_try_wait(&full[j % P.NS], (unsigned)((j / P.NS) & 1)) && ++spins < (1u << 20)) {
        }
      }
      charm::detail::report_error(CHARMING_ERR_PIPELINE, (int)s_issued, h);
    }
    for (int s = 0; s < P.NS; s++) {
      mbar_inval(&full[s]);
      mbar_inval(&empty[s]);
    }
  }
  fence_proxy_async_global();  // outputs (generic stores) -> next sweep's copies
  __syncthreads();
  *acc_out = acc;
  return !fail;
}

}  // namespace jac
