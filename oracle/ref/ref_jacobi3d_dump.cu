// Runs the reference's own 3-D Jacobi kernel (jacobi_3d_kernel from
// examples/jacobi-kernel/jacobi_kernel.cu:36-48, compiled from where it lies
// by oracle/ref/Makefile, launched with its (8, 8, 8) blocks, :163-170) on a
// seeded grid and writes the result, so that the CPU oracle can be checked
// against the reference bit for bit. Sweeps alternate between two buffers.
// TEST INFRASTRUCTURE ONLY.
//
// usage: ref_jacobi3d_dump nx ny nz sweeps seed out.bin
// Grid: (nz+2) x (ny+2) x (nx+2) doubles, x fastest; every cell (shell
// included) starts at u[k] = (mix64(seed * 2^32 + k) >> 11) * 2^-53.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>

__global__ void jacobi_3d_kernel(double* temp, double* new_temp, int width, int height, int depth);

static unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

int main(int argc, char** argv) {
  if (argc != 7) {
    fprintf(stderr, "usage: %s nx ny nz sweeps seed out.bin\n", argv[0]);
    return 2;
  }
  int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]), sweeps = atoi(argv[4]);
  unsigned long long seed = strtoull(argv[5], nullptr, 0);
  size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
  std::vector<double> h(n);
  for (size_t k = 0; k < n; k++) h[k] = (double)(mix64((seed << 32) + k) >> 11) * (1.0 / 9007199254740992.0);
  double *a = nullptr, *b = nullptr;
  if (cudaMalloc(&a, n * 8) != cudaSuccess || cudaMalloc(&b, n * 8) != cudaSuccess) return 1;
  cudaMemcpy(a, h.data(), n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(b, h.data(), n * 8, cudaMemcpyHostToDevice);
  dim3 block(8, 8, 8);
  dim3 grid((nx + 7) / 8, (ny + 7) / 8, (nz + 7) / 8);
  for (int s = 0; s < sweeps; s++) {
    jacobi_3d_kernel<<<grid, block>>>(a, b, nx, ny, nz);
    double* t = a; a = b; b = t;
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
    return 1;
  }
  cudaMemcpy(h.data(), a, n * 8, cudaMemcpyDeviceToHost);
  FILE* f = fopen(argv[6], "wb");
  if (!f) return 1;
  fwrite(h.data(), 8, n, f);
  fclose(f);
  cudaFree(a);
  cudaFree(b);
  printf("wrote %s (%d x %d x %d, %d sweeps)\n", argv[6], nx, ny, nz, sweeps);
  return 0;
}
