// Compares the device reciprocal of the flux formulas (vt::recip_nr) with the
// IEEE division 1.0 / x on the GPU over pseudo-random x in [2^-10, 2^10) and
// prints the largest difference in units in the last place and how many
// results differ. Built and run by tests/test_gpu_reciprocal.py.
#include <cstdio>
#include <cstring>

#include "vt_device.cuh"

__global__ void compare(int per_thread, unsigned long long* out) {
  const unsigned long long tid = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
  for (int k = 0; k < per_thread; ++k) {
    unsigned long long h = (tid * per_thread + k + 1) * 0x9E3779B97F4A7C15ull;  // splitmix64
    h ^= h >> 30;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27;
    h *= 0x94D049BB133111EBull;
    h ^= h >> 31;
    const double u = static_cast<double>(h >> 11) * (1.0 / 9007199254740992.0);
    const double x = exp2(-10.0 + 20.0 * u);
    const double got = vt::recip_nr(x), want = 1.0 / x;
    long long a, b;
    memcpy(&a, &got, 8);
    memcpy(&b, &want, 8);
    const unsigned long long ulp = a > b ? a - b : b - a;
    atomicMax(&out[0], ulp);
    if (ulp) atomicAdd(&out[1], 1ull);
  }
}

int main() {
  const int blocks = 148, threads = 256, per_thread = 64;
  unsigned long long* d = nullptr;
  if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  cudaMemset(d, 0, 2 * sizeof(unsigned long long));
  compare<<<blocks, threads>>>(per_thread, d);
  unsigned long long h[2] = {0, 0};
  if (cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
  cudaFree(d);
  printf("samples %d max_ulp %llu differing %llu\n", blocks * threads * per_thread, h[0], h[1]);
  return 0;
}
