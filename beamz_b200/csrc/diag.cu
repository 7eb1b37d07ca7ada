// Device reductions behind automatic termination: field diagnostics
// (integrated energy, largest |field|, non-finite count) and the change of
// each DFT monitor vector between checks.
//
// beamz evaluates both between run chunks with jnp reductions
// (beamz/simulation/execute.py:184-222 _field_diagnostics, 294-316
// _relative_monitor_change, driven by run_until_terminated 1312-1484).  Here
// each is a bandwidth-bound read of the fields or the arena: coalesced row
// sweeps, float products with double accumulation across rows, warp-shuffle
// and shared-memory block reductions, and a fixed partition and summation
// order, so a result is identical from run to run.

#include "kernels.cuh"

namespace fdtd {

namespace {

constexpr int kDiagThreads = 256;
constexpr int kDiagWarps = kDiagThreads / 32;

__device__ __forceinline__ void warp_reduce(double& s, float& m, unsigned& n) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    n += __shfl_down_sync(0xffffffffu, n, o);
  }
}

// Block reduction of (sum, max, count); the result is valid in thread 0.
__device__ __forceinline__ void block_reduce(double& s, float& m, unsigned& n) {
  __shared__ double ss[kDiagWarps];
  __shared__ float sm[kDiagWarps];
  __shared__ unsigned sn[kDiagWarps];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  warp_reduce(s, m, n);
  if (l == 0) {
    ss[w] = s;
    sm[w] = m;
    sn[w] = n;
  }
  __syncthreads();
  if (w == 0) {
    s = l < kDiagWarps ? ss[l] : 0.0;
    m = l < kDiagWarps ? sm[l] : 0.0f;
    n = l < kDiagWarps ? sn[l] : 0u;
    warp_reduce(s, m, n);
  }
}

// Rows (k, j) of one component, one warp per row: warp w of block b sweeps
// rows b * warps_per_block + w, then + all warps of the grid; its lanes stride
// along x, eight loads in flight each.  A lane forms each product eps * v^2 in
// float and sums its products of a row in float; each row then enters the
// double accumulator once, weighted by its y/z factor, with the two end sites
// of an edge-aligned x axis taken at half weight.  MAT: 0 eps_r = 1, 1
// codebook ids and table, 2 per-site array.
template <int MAT>
__device__ __forceinline__ void diag_rows(const DiagComp& q, double& s, float& mx, unsigned& bad) {
  const int rows = q.d.z * q.d.y;  // < 2^31: component arrays are validated below 2^31 elements
  const int lane = threadIdx.x & 31;
  const int step = gridDim.x * kDiagWarps;
  for (int r = blockIdx.x * kDiagWarps + (threadIdx.x >> 5); r < rows; r += step) {
    const int k = r / q.d.y, j = r - k * q.d.y;
    const int64_t base = k * q.plane + j * q.row;
    const float* f = q.field + base;
    float acc = 0.0f, ends = 0.0f;
#pragma unroll 8
    for (int i = lane; i < q.d.x; i += 32) {
      const float x = f[i];
      float e = 1.0f;
      if constexpr (MAT == 1) e = q.table[(q.ids[base + i] >> q.shift) & 0xffu];
      if constexpr (MAT == 2) e = q.eps[static_cast<int64_t>(r) * q.d.x + i];
      if (!isfinite(x)) {
        ++bad;
        continue;
      }
      mx = fmaxf(mx, fabsf(x));
      const float prod = e * x * x;
      acc += prod;
      if (i == 0 || i == q.d.x - 1) ends += prod;
    }
    double h = 1.0;
    if (q.integrate_z && q.edge_z && (k == 0 || k == q.d.z - 1)) h *= 0.5;
    if (q.edge_y && (j == 0 || j == q.d.y - 1)) h *= 0.5;
    s += h * (static_cast<double>(acc) - (q.edge_x ? 0.5 * static_cast<double>(ends) : 0.0));
  }
}

__global__ void __launch_bounds__(kDiagThreads) diag_partial_kernel(DiagArgs a) {
  const int c = blockIdx.y;
  double s = 0.0;
  float mx = 0.0f;
  unsigned bad = 0;
  if ((a.active >> c) & 1) {
    const DiagComp& q = a.comp[c];
    if (q.ids) diag_rows<1>(q, s, mx, bad);
    else if (q.eps) diag_rows<2>(q, s, mx, bad);
    else diag_rows<0>(q, s, mx, bad);
  }
  block_reduce(s, mx, bad);
  if (threadIdx.x == 0) {
    double* o = a.partials + (static_cast<int64_t>(c) * gridDim.x + blockIdx.x) * 3;
    o[0] = s;
    o[1] = mx;
    o[2] = bad;
  }
}

// One block per component: the partials in block order.
__global__ void __launch_bounds__(kDiagThreads) diag_final_kernel(const double* partials, int blocks, double* out) {
  const int c = blockIdx.x;
  double s = 0.0;
  float mx = 0.0f;
  unsigned bad = 0;
  for (int b = threadIdx.x; b < blocks; b += kDiagThreads) {
    const double* o = partials + (static_cast<int64_t>(c) * blocks + b) * 3;
    s += o[0];
    mx = fmaxf(mx, static_cast<float>(o[1]));
    bad += static_cast<unsigned>(o[2]);
  }
  block_reduce(s, mx, bad);
  if (threadIdx.x == 0) {
    out[c * 3 + 0] = s;
    out[c * 3 + 1] = mx;
    out[c * 3 + 2] = bad;
  }
}

// One block per (monitor, component, frequency): squared norms of the change,
// the current and the previous vector, then prev <- current.
__global__ void __launch_bounds__(kDiagThreads) dft_change_kernel(DftDev d, float* prev_re, float* prev_im,
                                                                  double* out) {
  const int key = blockIdx.x;
  const int f = key % d.max_freqs, mc = key / d.max_freqs;
  const int m = mc / 6, c = mc % 6;
  const int* cnt = d.counts + 5 * m;
  const int nf = min(max(cnt[0], 0), d.max_freqs);
  const int np = min(max(cnt[1], 0), d.max_points);
  const int voff = cnt[3];
  double dd = 0.0, cc = 0.0, pp = 0.0;
  const bool on = d.masks[m * 6 + c] != 0.0f && f < nf && voff >= 0 &&
                  voff + static_cast<int64_t>(6) * nf * np <= d.arena_len;
  if (on) {
    const int64_t base = voff + (static_cast<int64_t>(c) * nf + f) * np;
    for (int p = threadIdx.x; p < np; p += kDiagThreads) {
      const float re = d.re[base + p], im = d.im[base + p];
      const double dr = static_cast<double>(re) - prev_re[base + p], di = static_cast<double>(im) - prev_im[base + p];
      const double pr = prev_re[base + p], pi = prev_im[base + p];
      dd += dr * dr + di * di;
      cc += static_cast<double>(re) * re + static_cast<double>(im) * im;
      pp += pr * pr + pi * pi;
      prev_re[base + p] = re;
      prev_im[base + p] = im;
    }
  }
  // Three block sums in sequence; each total lands in thread 0's variable and
  // stays there through the later reductions.
  float unused = 0.0f;
  unsigned none = 0;
  block_reduce(dd, unused, none);
  __syncthreads();
  block_reduce(cc, unused, none);
  __syncthreads();
  block_reduce(pp, unused, none);
  if (threadIdx.x == 0) {
    out[key * 3 + 0] = dd;
    out[key * 3 + 1] = cc;
    out[key * 3 + 2] = pp;
  }
}

}  // namespace

cudaError_t launch_field_diagnostics(cudaStream_t s, const DiagArgs& a, double* out) {
  diag_partial_kernel<<<dim3(FDTD_DIAG_BLOCKS, 6, 1), kDiagThreads, 0, s>>>(a);
  cudaError_t err = cudaPeekAtLastError();
  if (err != cudaSuccess) return err;
  diag_final_kernel<<<6, kDiagThreads, 0, s>>>(a.partials, FDTD_DIAG_BLOCKS, out);
  return cudaPeekAtLastError();
}

cudaError_t launch_dft_change(cudaStream_t s, const DftDev& d, float* prev_re, float* prev_im, double* out) {
  const int keys = d.monitor_count * 6 * d.max_freqs;
  if (keys <= 0) return cudaSuccess;
  dft_change_kernel<<<keys, kDiagThreads, 0, s>>>(d, prev_re, prev_im, out);
  return cudaPeekAtLastError();
}

}  // namespace fdtd
