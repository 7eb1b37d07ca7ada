// Monitor-plane reductions over the DFT arena: the sums behind beamz's DFT
// flux through a monitor (beamz/simulation/observe.py:166-234
// monitor_dft_component, _flux_component, monitor_dft_flux) and its modal
// overlaps with mode profiles (beamz/devices/modes/fields.py:76-129
// _modal_overlap, used by beamz/analysis/mode_projection.py and
// sparameters.py).
//
// One block per (profile row, frequency) sweeps the monitor's points with a
// fixed stride, forms each point's term in double in the reference's operand
// order, and sums in a fixed order (per-thread partial sums, then warp
// shuffles, then the block's warps in order), so a result is identical from
// run to run.  The arena is read once per row; the work is a few MB against
// the hundreds of MB an arena copy to the host would move.

#include "kernels.cuh"

namespace fdtd {

namespace {

constexpr int kReduceThreads = 256;
constexpr int kReduceWarps = kReduceThreads / 32;

struct Cplx {
  double re, im;
};

// (a)(b) as numpy's complex128 multiply: (ar br - ai bi) + (ar bi + ai br) i.
__device__ __forceinline__ Cplx cmul(Cplx a, Cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ Cplx conj(Cplx a) { return {a.re, -a.im}; }
__device__ __forceinline__ Cplx cadd(Cplx a, Cplx b) { return {a.re + b.re, a.im + b.im}; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum of v over the block, valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  v = warp_sum(v);
  __syncthreads();  // scratch reuse between calls
  if (l == 0) scratch[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = l < kReduceWarps ? scratch[l] : 0.0;
    s = warp_sum(s);
  }
  return s;
}

__global__ void __launch_bounds__(kReduceThreads) monitor_reduce_kernel(MonitorReduceDev r) {
  __shared__ double scratch[kReduceWarps];
  const int f = blockIdx.x % r.freqs;
  const int row = blockIdx.x / r.freqs;
  const int64_t P = r.points;
  // Per-frequency scales of the stored sums: E = alpha v, H = (alpha v) phase.
  const double alpha = r.scale[3 * f];
  const Cplx phase = {r.scale[3 * f + 1], r.scale[3 * f + 2]};
  double acc[4] = {0.0, 0.0, 0.0, 0.0};  // pair 0 re, im, pair 1 re, im
  for (int64_t p = threadIdx.x; p < P; p += kReduceThreads) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int64_t oe = r.value_offset + (static_cast<int64_t>(r.e[q]) * r.freqs + f) * P + p;
      const int64_t oh = r.value_offset + (static_cast<int64_t>(r.h[q]) * r.freqs + f) * P + p;
      const Cplx ef = {alpha * static_cast<double>(r.re[oe]), alpha * static_cast<double>(r.im[oe])};
      const Cplx hf = cmul({alpha * static_cast<double>(r.re[oh]), alpha * static_cast<double>(r.im[oh])}, phase);
      Cplx u;
      if (r.rows == 0) {
        u = cmul(ef, conj(hf));  // flux: E conj(H)
      } else {
        const int64_t base = ((static_cast<int64_t>(row) * r.freqs + f) * 4) * P + p;
        const Cplx em = {r.prof_re[base + q * P], r.prof_im[base + q * P]};
        const Cplx hm = {r.prof_re[base + (2 + q) * P], r.prof_im[base + (2 + q) * P]};
        u = cadd(cmul(ef, conj(hm)), cmul(conj(em), hf));  // E conj(Hm) + conj(Em) H
      }
      const double w = r.weights[q * P + p];
      acc[2 * q] += w * u.re;
      acc[2 * q + 1] += w * u.im;
    }
  }
  double* out = r.out + (static_cast<int64_t>(row) * r.freqs + f) * 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double s = block_sum(acc[k], scratch);
    if (threadIdx.x == 0) out[k] = s;
  }
}

}  // namespace

cudaError_t launch_monitor_reduce(cudaStream_t s, const MonitorReduceDev& r) {
  const int64_t blocks = static_cast<int64_t>(r.rows > 0 ? r.rows : 1) * r.freqs;
  if (blocks <= 0) return cudaSuccess;
  if (blocks > (int64_t{1} << 31) - 1) return cudaErrorInvalidValue;
  monitor_reduce_kernel<<<static_cast<unsigned>(blocks), kReduceThreads, 0, s>>>(r);
  return cudaPeekAtLastError();
}

}  // namespace fdtd
