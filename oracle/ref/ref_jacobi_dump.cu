// Runs the reference's own 2-D Jacobi kernel (jacobi_2d_kernel from
// examples/jacobi-kernel/jacobi_kernel.cu:26-34, compiled from where it lies
// by oracle/ref/Makefile) on a seeded grid and writes the result, so that
// the CPU oracle can be checked against the reference bit for bit.
// TEST INFRASTRUCTURE ONLY.
//
// usage: ref_jacobi_dump nx ny sweeps seed out.bin
// Grid: (ny+2) x (nx+2) doubles, row-major; every cell (boundary ring
// included) starts at u[k] = (mix64(seed * 2^32 + k) >> 11) * 2^-53.
// Output file: the grid after `sweeps` sweeps, raw little-endian doubles.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>

__global__ void jacobi_2d_kernel(double* temp, double* new_temp, int width, int height);

static unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s nx ny sweeps seed out.bin\n", argv[0]);
    return 2;
  }
  int nx = atoi(argv[1]), ny = atoi(argv[2]), sweeps = atoi(argv[3]);
  unsigned long long seed = strtoull(argv[4], nullptr, 0);
  size_t n = (size_t)(nx + 2) * (ny + 2);
  std::vector<double> h(n);
  for (size_t k = 0; k < n; k++) h[k] = (double)(mix64((seed << 32) + k) >> 11) * (1.0 / 9007199254740992.0);
  double *a = nullptr, *b = nullptr;
  if (cudaMalloc(&a, n * 8) != cudaSuccess || cudaMalloc(&b, n * 8) != cudaSuccess) return 1;
  cudaMemcpy(a, h.data(), n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(b, h.data(), n * 8, cudaMemcpyHostToDevice);
  dim3 block(32, 32);
  dim3 grid((nx + block.x - 1) / block.x, (ny + block.y - 1) / block.y);
  for (int s = 0; s < sweeps; s++) {
    jacobi_2d_kernel<<<grid, block>>>(a, b, nx, ny);
    double* t = a; a = b; b = t;
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
    return 1;
  }
  cudaMemcpy(h.data(), a, n * 8, cudaMemcpyDeviceToHost);
  FILE* f = fopen(argv[5], "wb");
  if (!f) return 1;
  fwrite(h.data(), 8, n, f);
  fclose(f);
  cudaFree(a);
  cudaFree(b);
  printf("wrote %s (%d x %d, %d sweeps)\n", argv[5], nx, ny, sweeps);
  return 0;
}
