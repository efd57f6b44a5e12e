// Host-side layout of a set of Jacobi2d problems: decomposition into
// chares, residual tree, neighbours, placement on PEs, and where each
// chare's two grids sit in one device allocation. Plain C++ (no CUDA
// calls), shared by charming_jacobi2d_create and the CPU check of the chare
// code, so both run the same decomposition.
//
// Decomposition (reference: examples/jacobi2d/jacobi2d.cu:37-65): problem p
// is split into px x py chares (px, py from the problem, or from the target
// chare side), chare (cx, cy) gets rows/columns by an even split. Ghost
// depth D: every chare keeps D ghost rows/columns on each side; with D > 1
// the chare runs D sweeps per halo exchange and also needs its diagonal
// neighbours' corners.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <cstdint>
#include <functional>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "charming_c.h"
#include "jacobi_types.cuh"

namespace jac {

struct layout {
  std::vector<chare_desc> chares;       // placed order; buf[] are byte offsets until placed
  std::vector<prob_desc> probs;
  std::vector<int> block_map;           // chares per PE
  std::vector<int> chare_of;            // [prob offset + cy*px + cx] -> placed chare index
  std::vector<size_t> chare_of_off;
  std::vector<int> px, py;
  std::vector<size_t> buf_off;          // 2 per chare: byte offset of the grid (its row 1-D)
  size_t total_bytes = 0;               // one allocation for all grids
  int max_per_pe = 0;
  uint64_t points = 0;
  uint64_t halo_msgs = 0;               // halo messages per exchange
};

// Sweeps per exchange chosen when none is requested: deeper passes mean
// fewer messages, but the wavefront's registers spill beyond this.
constexpr int DEPTH_AUTO = 6;

// Halos at ghost depth > 1 go in two phases without corner messages unless
// CHARMING_HALO_CORNERS=1 asks for the one-phase exchange with them.
inline bool halo_corner_messages() {
  const char* ev = getenv("CHARMING_HALO_CORNERS");
  return ev && ev[0] == '1';
}

// Ghost depth of a problem whose smallest chare is wmin x hmin. Automatic
// choice: DEPTH_AUTO, or with a residual period K the balanced split of K
// into passes of at most DEPTH_AUTO (passes end at every check, so K = 10
// runs passes of 5 + 5 instead of 6 + 4).
inline int choose_depth(int requested, int pipeline, int wmin, int hmin, int off, int check_every = 0) {
  int auto_d = DEPTH_AUTO;
  if (check_every > 0) {
    const int n = (check_every + DEPTH_AUTO - 1) / DEPTH_AUTO;
    auto_d = (check_every + n - 1) / n;
  }
  int d = requested > 0 ? requested : (pipeline ? 1 : auto_d);
  if (pipeline) d = 1;  // the bulk-copy sweep runs one sweep per exchange
  d = std::min(d, DEPTH_MAX);
  d = std::min(d, std::min(wmin, hmin));
  d = std::min(d, off);
  return std::max(d, 1);
}

// Builds the layout. esz: element bytes; off: element offset of interior
// column 1 in a row (a 128-byte boundary); vec: elements per 16-byte vector.
// Returns false with a message on bad input.
inline bool build_layout(const charming_jacobi_problem* probs, int n, int side, int balance,
    int depth_req, int pipeline, int n_pes, int esz, int off, int vec, layout* L,
    std::string* err) {
  const int align_el = 128 / esz;
  side = side > 0 ? side : 256;
  std::vector<chare_desc> raw;
  std::vector<int> root_raw(n);
  L->probs.assign(n, prob_desc{});
  L->px.clear();
  L->py.clear();
  L->points = 0;
  L->halo_msgs = 0;
  for (int p = 0; p < n; p++) {
    const charming_jacobi_problem& q = probs[p];
    if (q.nx < 1 || q.ny < 1 || q.max_sweeps < 0 || q.check_every < 0) {
      *err = "jacobi2d: problem size";
      return false;
    }
    int px = q.px > 0 ? q.px : (q.nx + side - 1) / side;
    int py = q.py > 0 ? q.py : (q.ny + side - 1) / side;
    if (px > q.nx || py > q.ny) {
      *err = "jacobi2d: more chares than rows/columns";
      return false;
    }
    L->px.push_back(px);
    L->py.push_back(py);
    const int wmin = q.nx / px, hmin = q.ny / py;
    const int D = choose_depth(depth_req, pipeline, wmin, hmin, off, q.check_every);
    int base = (int)raw.size();
    root_raw[p] = base;
    int nc = px * py;
    auto id = [&](int cx, int cy) {
      return (cx >= 0 && cx < px && cy >= 0 && cy < py) ? base + cy * px + cx : -1;
    };
    for (int cy = 0; cy < py; cy++) {
      for (int cx = 0; cx < px; cx++) {
        chare_desc d{};
        d.prob = p;
        d.slot = p;
        d.cx = cx;
        d.cy = cy;
        d.x0 = split_start(q.nx, px, cx);
        d.y0 = split_start(q.ny, py, cy);
        d.w = split_start(q.nx, px, cx + 1) - d.x0;
        d.h = split_start(q.ny, py, cy + 1) - d.y0;
        d.depth = D;
        // row: D ghost columns before column 1 (inside the OFF-element lead),
        // the interior, D ghost columns, one spare vector for whole-vector loads
        d.pitch = (off + d.w + D + 2 * vec + align_el - 1) / align_el * align_el;
        d.nbr[TOP] = id(cx, cy - 1);
        d.nbr[BOTTOM] = id(cx, cy + 1);
        d.nbr[LEFT] = id(cx - 1, cy);
        d.nbr[RIGHT] = id(cx + 1, cy);
        // depth > 1: the two-phase exchange carries the corners in the
        // top/bottom halos (CHARMING_HALO_CORNERS=1: corner messages instead)
        const bool corners = D > 1 && halo_corner_messages();
        d.ext = (D > 1 && !corners) ? (D + vec - 1) / vec * vec : 0;
        d.pad_ = 0;
        d.nbr[TOP_LEFT] = corners ? id(cx - 1, cy - 1) : -1;
        d.nbr[TOP_RIGHT] = corners ? id(cx + 1, cy - 1) : -1;
        d.nbr[BOTTOM_LEFT] = corners ? id(cx - 1, cy + 1) : -1;
        d.nbr[BOTTOM_RIGHT] = corners ? id(cx + 1, cy + 1) : -1;
        int r = cy * px + cx;
        d.rank = r;
        d.parent = r > 0 ? base + (r - 1) / 2 : -1;
        d.child[0] = 2 * r + 1 < nc ? base + 2 * r + 1 : -1;
        d.child[1] = 2 * r + 2 < nc ? base + 2 * r + 2 : -1;
        raw.push_back(d);
        for (int k = 0; k < N_DIRS; k++) L->halo_msgs += d.nbr[k] >= 0;
      }
    }
    prob_desc& pd = L->probs[p];
    pd.nx = q.nx;
    pd.ny = q.ny;
    pd.px = px;
    pd.py = py;
    pd.max_sweeps = q.max_sweeps;
    pd.check_every = q.check_every;
    pd.tol = q.tol;
    pd.n_chares = nc;
    pd.depth = D;
    for (int k = 0; k < 4; k++) pd.bc[k] = q.bc[k];
    L->points += (uint64_t)q.nx * q.ny;
  }
  const int nch = (int)raw.size();

  // placement: chares -> PEs (work-balanced greedy, or the reference's
  // default block map over problem order, include/chare.h:136-176)
  std::vector<int> pe_of(nch);
  L->block_map.assign(n_pes, 0);
  if (balance) {
    std::vector<int> order(nch);
    std::iota(order.begin(), order.end(), 0);
    auto work = [&](int i) { return (double)raw[i].w * raw[i].h + 4096.0; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
    using item = std::pair<double, int>;
    std::priority_queue<item, std::vector<item>, std::greater<item>> pq;
    for (int pe = 0; pe < n_pes; pe++) pq.push({0.0, pe});
    for (int i : order) {
      item t = pq.top();
      pq.pop();
      pe_of[i] = t.second;
      pq.push({t.first + work(i), t.second});
    }
  } else {
    int per = nch / n_pes, rem = nch % n_pes, k = 0;
    for (int pe = 0; pe < n_pes; pe++) {
      int cnt = per + (pe < rem ? 1 : 0);
      for (int j = 0; j < cnt; j++) pe_of[k++] = pe;
    }
  }
  std::vector<int> perm(nch);  // placed index -> raw index
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return pe_of[a] < pe_of[b]; });
  std::vector<int> inv(nch);
  for (int k = 0; k < nch; k++) inv[perm[k]] = k;
  auto remap = [&](int x) { return x < 0 ? -1 : inv[x]; };
  L->chares.resize(nch);
  for (int k = 0; k < nch; k++) {
    chare_desc d = raw[perm[k]];
    for (int q = 0; q < N_DIRS; q++) d.nbr[q] = remap(d.nbr[q]);
    d.parent = remap(d.parent);
    d.child[0] = remap(d.child[0]);
    d.child[1] = remap(d.child[1]);
    L->chares[k] = d;
    L->block_map[pe_of[perm[k]]]++;
  }
  for (int p = 0; p < n; p++) L->probs[p].root = inv[root_raw[p]];
  L->max_per_pe = nch ? *std::max_element(L->block_map.begin(), L->block_map.end()) : 0;
  L->chare_of.clear();
  L->chare_of_off.clear();
  for (int p = 0, o = 0; p < n; p++) {
    L->chare_of_off.push_back(o);
    for (int r = 0; r < L->px[p] * L->py[p]; r++) L->chare_of.push_back(inv[root_raw[p] + r]);
    o += L->px[p] * L->py[p];
  }

  // grids: two per chare, rows 1-D .. h+D, each 256-byte aligned
  L->total_bytes = 0;
  L->buf_off.assign(2 * (size_t)nch, 0);
  for (int k = 0; k < nch; k++) {
    const chare_desc& d = L->chares[k];
    size_t b = ((size_t)d.pitch * (d.h + 2 * d.depth) * esz + 255) / 256 * 256;
    L->buf_off[2 * k] = L->total_bytes;
    L->buf_off[2 * k + 1] = L->total_bytes + b;
    L->total_bytes += 2 * b;
  }
  return true;
}

// Points the chares' buf[] at row 0 of their grids inside `base`.
inline void place_buffers(layout* L, char* base, int esz) {
  for (size_t k = 0; k < L->chares.size(); k++) {
    chare_desc& d = L->chares[k];
    for (int b = 0; b < 2; b++)
      d.buf[b] = base + L->buf_off[2 * k + b] + (size_t)(d.depth - 1) * d.pitch * esz;
  }
}

}  // namespace jac
