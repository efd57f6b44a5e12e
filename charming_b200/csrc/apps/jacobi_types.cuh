// Descriptors shared by the Jacobi2d host code and its chares.
#pragma once

namespace jac {

// Neighbour directions; opposite directions differ in bit 0. The corners are
// used with ghost depth > 1 only.
enum dir : int {
  TOP = 0, BOTTOM = 1, LEFT = 2, RIGHT = 3,
  TOP_LEFT = 4, BOTTOM_RIGHT = 5, TOP_RIGHT = 6, BOTTOM_LEFT = 7
};
constexpr int N_DIRS = 8;
constexpr int DEPTH_MAX = 8;  // sweeps per halo exchange, at most
__host__ __device__ inline int opposite(int d) { return d ^ 1; }
__host__ __device__ inline bool dir_top(int d) { return d == TOP || d == TOP_LEFT || d == TOP_RIGHT; }
__host__ __device__ inline bool dir_bottom(int d) {
  return d == BOTTOM || d == BOTTOM_LEFT || d == BOTTOM_RIGHT;
}
__host__ __device__ inline bool dir_left(int d) { return d == LEFT || d == TOP_LEFT || d == BOTTOM_LEFT; }
__host__ __device__ inline bool dir_right(int d) {
  return d == RIGHT || d == TOP_RIGHT || d == BOTTOM_RIGHT;
}

// Rectangle of a chare's grid in its own coordinates (interior rows and
// columns 1..h, 1..w).
struct region {
  int r0, c0, nr, nc;
};
// The ghost cells a halo from direction `d` fills (depth D).
__host__ __device__ inline region ghost_region(int d, int D, int w, int h) {
  region g;
  g.r0 = dir_top(d) ? 1 - D : dir_bottom(d) ? h + 1 : 1;
  g.nr = (dir_top(d) || dir_bottom(d)) ? D : h;
  g.c0 = dir_left(d) ? 1 - D : dir_right(d) ? w + 1 : 1;
  g.nc = (dir_left(d) || dir_right(d)) ? D : w;
  return g;
}
// The boundary cells a chare sends to its neighbour in direction `d`.
__host__ __device__ inline region edge_region(int d, int D, int w, int h) {
  region e;
  e.r0 = dir_top(d) ? 1 : dir_bottom(d) ? h - D + 1 : 1;
  e.nr = (dir_top(d) || dir_bottom(d)) ? D : h;
  e.c0 = dir_left(d) ? 1 : dir_right(d) ? w - D + 1 : 1;
  e.nc = (dir_left(d) || dir_right(d)) ? D : w;
  return e;
}

// One chare block of one problem (host-built, read-only on the device).
struct chare_desc {
  int prob;            // problem index (serving: the worker's own prob_desc copy)
  int slot;            // problem index (serving: the request's device slot)
  int cx, cy;          // chare column / row within the problem
  int x0, y0;          // first interior column / row of the block (0-based)
  int w, h;            // interior columns / rows of the block
  int pitch;           // row pitch, elements
  int depth;           // ghost depth D: rows/columns 1-D..h+D / 1-D..w+D exist
  int nbr[N_DIRS];     // global chare index per direction, -1 at the boundary
  int parent;          // residual tree: parent chare (-1 at the root)
  int child[2];        // residual tree: children (-1 if none)
  int rank;            // index within the problem (tree position; 0 = root)
  int ext;             // 0: one exchange phase, corner halos from the diagonal
                       // neighbours. > 0 (depth > 1): two phases, left/right
                       // halos first, then top/bottom halos that also carry
                       // ext ghost columns each side (ext >= D, whole 16-byte
                       // vectors), so the corners arrive through the
                       // top/bottom neighbours and no corner messages exist
  int pad_;
  void* buf[2];        // the two pitched grids, pointing at row 0 (ghost rows
                       // 1-D..0 lie before it)
};

// The cells a halo from / to direction d covers, with the two-phase
// exchange's wider top/bottom halos.
__host__ __device__ inline region halo_ghost(int d, const chare_desc& c) {
  region g = ghost_region(d, c.depth, c.w, c.h);
  if (c.ext > 0 && (d == TOP || d == BOTTOM)) {
    g.c0 = 1 - c.ext;
    g.nc = c.w + 2 * c.ext;
  }
  return g;
}
__host__ __device__ inline region halo_edge(int d, const chare_desc& c) {
  region e = edge_region(d, c.depth, c.w, c.h);
  if (c.ext > 0 && (d == TOP || d == BOTTOM)) {
    e.c0 = 1 - c.ext;
    e.nc = c.w + 2 * c.ext;
  }
  return e;
}

struct prob_desc {
  int nx, ny, px, py;
  int max_sweeps;
  int check_every;     // 0: no residual
  double tol;          // 0: never stop early
  int root;            // global chare index of the problem's tree root
  int n_chares;
  int depth;           // ghost depth of the problem's chares
  double bc[4];        // boundary values: top, bottom, left, right
};

struct prob_result {
  int sweeps;
  int checks;
  double res0;
  double res_last;
};

// Payload header of a halo message; the values follow (16-byte aligned).
struct halo_hdr {
  int dir;             // ghost side at the receiver
  int len;             // values (the ghost region, row-major)
  int pass;            // exchange the values belong to (the sender's pass count)
  unsigned gen;        // request generation (serving; 0 otherwise)
};

struct partial_msg {
  int check;
  int slot;            // 0 or 1: which child of the receiver sent it
  unsigned gen;
  int pad;
  double value;
};

struct decision_msg {
  int check;
  int stop;
  unsigned gen;
  int pad;
  double res0;
  double res;
};

struct start_msg {
  unsigned gen;        // request generation (serving; 0 otherwise)
  int slot;
};

// Serving: one admitted request, posted by the host into a ring in mapped
// host memory that the server chare polls. seq = ticket + 1, written last.
struct serve_req {
  unsigned long long seq;
  int slot;            // device problem slot (prob_desc table index)
  int root;            // worker that holds the request's chare 0
  unsigned gen;
  int pad[3];
};

// Serving: completion record written by the request's last chare into a
// ring in mapped host memory. seq = ticket + 1, written last.
struct serve_comp {
  unsigned long long seq;
  int slot;
  unsigned gen;
  int sweeps;
  int checks;
  int final_buf;       // buffer (0/1) of every chare holding the result
  int status;
  double res0, res_last;
  unsigned long long t_ns;   // %globaltimer at completion
};

// Even split of n cells into k parts: part i starts at split_start(n, k, i).
__host__ __device__ inline int split_start(int n, int k, int i) {
  int base = n / k, rem = n % k;
  return i * base + (i < rem ? i : rem);
}
__host__ __device__ inline int split_owner(int n, int k, int x) {
  int base = n / k, rem = n % k;
  int big = rem * (base + 1);
  return x < big ? x / (base + 1) : rem + (x - big) / base;
}

}  // namespace jac
