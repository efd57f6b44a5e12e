// Jacobi2d over a 1-D row decomposition (apps/decomp1d.cu): per-chare plan
// shared by the program, its C ABI entry point and the CPU check.
#pragma once
#include <vector>

struct d1_desc {
  int chunk;      // rows of the band
  int iy_end;     // rows 1..iy_end-1 are computed
  int top, bottom;
  int top_ghost;  // the top neighbour's bottom ghost row (its chunk + 1)
  int pad[3];
};

// The reference's decomposition of ny rows over n chares (examples/
// jacobi2d-decomp1d/jacobi2d.cu:144-198): per chare its band, computed rows
// and neighbours, g0[i] = global index of its row 1, bc[g] = the fixed value
// of columns 0 and nx-1 in global row g. False when a chare would get fewer
// than 2 rows.
bool decomp1d_plan(int n, int ny, std::vector<d1_desc>& descs, std::vector<int>& g0, std::vector<float>& bc);
