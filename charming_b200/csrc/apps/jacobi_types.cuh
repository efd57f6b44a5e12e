// Descriptors shared by the Jacobi2d host code and its chares.
#pragma once

namespace jac {

enum dir : int { TOP = 0, BOTTOM = 1, LEFT = 2, RIGHT = 3 };
__host__ __device__ inline int opposite(int d) { return d ^ 1; }

// One chare block of one problem (host-built, read-only on the device).
struct chare_desc {
  int prob;            // problem index
  int cx, cy;          // chare column / row within the problem
  int x0, y0;          // first interior column / row of the block (0-based)
  int w, h;            // interior columns / rows of the block
  int pitch;           // row pitch, elements
  int nbr[4];          // global chare index per direction, -1 at the boundary
  int parent;          // residual tree: parent chare (-1 at the root)
  int child[2];        // residual tree: children (-1 if none)
  int rank;            // index within the problem (tree position; 0 = root)
  void* buf[2];        // the two pitched grids (ghost ring included)
};

struct prob_desc {
  int nx, ny, px, py;
  int max_sweeps;
  int check_every;     // 0: no residual
  double tol;          // 0: never stop early
  int root;            // global chare index of the problem's tree root
  int n_chares;
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
  int len;             // values
  int iter;            // sweep the values belong to
  int pad;
};

struct partial_msg {
  int check;
  int slot;            // 0 or 1: which child of the receiver sent it
  double value;
};

struct decision_msg {
  int check;
  int stop;
  double res0;
  double res;
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
