// On-device planning: monitor gather plans packed per point (nonzero weights
// first, offsets remapped to the device layout) and the voxel-id histogram
// behind the codebook's compact material indices.  beamz does both on the
// host (beamz/simulation/cuda/runtime.py:530-618, compile.py:146-187).

#include "kernels.cuh"

namespace fdtd {

namespace {

constexpr int kPackThreads = 256;
constexpr int kMaxSlots = 32;

__device__ __forceinline__ int remap_offset(int flat, const GatherPackDev& g) {
  const int64_t n = static_cast<int64_t>(g.dz) * g.dy * g.dx;
  if (flat < 0 || flat >= n) return -1;
  const int i = flat % g.dx;
  const int r = flat / g.dx;
  const int j = r % g.dy, k = r / g.dy;
  return static_cast<int>(k * g.plane + j * g.row + i);
}

__global__ void __launch_bounds__(kPackThreads) gather_pack_kernel(GatherPackDev g) {
  const int p = blockIdx.x * kPackThreads + threadIdx.x;
  if (p >= g.points) return;
  const int* idx = g.idx_in + static_cast<int64_t>(p) * g.slots_in;
  const float* w = g.w_in + static_cast<int64_t>(p) * g.slots_in;
  int n = 0;
  for (int pass = 0; pass < 2; ++pass) {  // nonzero weights, then zero weights
    for (int s = 0; s < g.slots_in; ++s) {
      const float ws = w[s];
      if ((ws != 0.0f) != (pass == 0)) continue;
      if (n < g.rows) {  // rows past the output's K hold only zero weights (the caller sizes K)
        g.idx_out[static_cast<int64_t>(n) * g.pmax + p] = remap_offset(idx[s], g);
        g.w_out[static_cast<int64_t>(n) * g.pmax + p] = ws;
      }
      ++n;
    }
  }
}

__global__ void __launch_bounds__(kPackThreads) voxel_histogram_kernel(const uint8_t* v, int64_t n, int* counts) {
  __shared__ int h[256];
  for (int b = threadIdx.x; b < 256; b += kPackThreads) h[b] = 0;
  __syncthreads();
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * kPackThreads + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * kPackThreads)
    atomicAdd(&h[v[e]], 1);
  __syncthreads();
  for (int b = threadIdx.x; b < 256; b += kPackThreads)
    if (h[b]) atomicAdd(&counts[b], h[b]);
}

}  // namespace

cudaError_t launch_gather_pack(cudaStream_t s, const GatherPackDev& g) {
  if (g.points <= 0) return cudaSuccess;
  if (g.slots_in > kMaxSlots) return cudaErrorInvalidValue;
  gather_pack_kernel<<<(g.points + kPackThreads - 1) / kPackThreads, kPackThreads, 0, s>>>(g);
  return cudaPeekAtLastError();
}

cudaError_t launch_voxel_histogram(cudaStream_t s, const uint8_t* v, int64_t n, int* counts) {
  cudaError_t err = cudaMemsetAsync(counts, 0, 256 * sizeof(int), s);
  if (err != cudaSuccess || n <= 0) return err;
  int blocks = static_cast<int>((n + kPackThreads - 1) / kPackThreads);
  if (blocks > 4 * 148) blocks = 4 * 148;
  voxel_histogram_kernel<<<blocks, kPackThreads, 0, s>>>(v, n, counts);
  return cudaPeekAtLastError();
}

}  // namespace fdtd
