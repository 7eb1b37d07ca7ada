// Slab sources, DFT monitors and the device step counter.

#include "kernels.cuh"

namespace fdtd {

namespace {

// field[start + idx] += coeff[idx] * waveform[clamp(step)]
// (beamz/simulation/execute.py:374-433; cuda/src/io.cu:65-168).  H/E-timing
// additions on PEC-constrained cells are skipped: the step zeroes those cells
// after the update, and beamz re-applies its masks after the injection
// (execute.py:506-522), so the two orders agree.
__global__ void source_kernel(SourceDev s, float* target, Dims td, int64_t row, int64_t plane, int timing,
                              int metallic, const int* counter, int step_offset) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= s.ex || y >= s.ey || z >= s.ez) return;
  const int k = s.z0 + z, j = s.y0 + y, i = s.x0 + x;
  if (k < 0 || j < 0 || i < 0 || k >= td.z || j >= td.y || i >= td.x) return;
  if (timing == FDTD_TIMING_H && h_constrained(metallic, s.component, td, k, j, i)) return;
  if (timing == FDTD_TIMING_E && e_constrained(metallic, s.component, td, k, j, i)) return;
  const float amp = source_amplitude(s, counter[0] + step_offset);
  const int64_t co = (static_cast<int64_t>(z) * s.ey + y) * s.ex + x;
  const int64_t to = k * plane + j * row + i;
  target[to] = target[to] + s.coeff[co] * amp;
}

__global__ void copy3d_kernel(const float* src, int64_t sr, int64_t sp, float* dst, int64_t dr, int64_t dp,
                              int64_t ny, int64_t nx) {
  const int64_t k = blockIdx.z;
  for (int64_t j = blockIdx.y * blockDim.y + threadIdx.y; j < ny; j += gridDim.y * blockDim.y)
    for (int64_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x)
      dst[k * dp + j * dr + i] = src[k * sp + j * sr + i];
}

// One block per (monitor, component, point tile).  The per-frequency phase and
// window are evaluated once per block into shared memory.
// beamz/simulation/observe.py:327-357 (gate, window, scale) and 529-585.
constexpr int kDftThreads = 256;
constexpr int kDftMaxFreqs = 64;

// Interpolated sample of one (monitor, component, point).  Neighbour-major
// plan: consecutive points of one neighbour slot are contiguous, and per point
// the nonzero weights come first, so the sum runs over the slots before the
// first zero weight, in slot order (the same sum as skipping zeros).  The
// first kGatherSlots slots' weights and indices are loaded together, then
// their field values together: two dependent memory round trips per point
// instead of one per slot (plane monitors interpolate over at most four).
constexpr int kGatherSlots = 4;

__device__ __forceinline__ float dft_gather(const DftDev& d, int m, int c, int p) {
  const int K = d.neighbors;
  const int64_t stride = d.max_points;
  const int64_t base = ((static_cast<int64_t>(m) * 6 + c) * K) * stride + p;
  const float* field = d.fields[c];
  const int64_t len = d.field_len[c];
  float w[kGatherSlots], f[kGatherSlots];
  int idx[kGatherSlots];
#pragma unroll
  for (int n = 0; n < kGatherSlots; ++n) {
    w[n] = n < K ? d.weights[base + n * stride] : 0.0f;
    idx[n] = n < K ? d.indices[base + n * stride] : -1;
  }
#pragma unroll
  for (int n = 0; n < kGatherSlots; ++n) f[n] = (w[n] != 0.0f && idx[n] >= 0 && idx[n] < len) ? field[idx[n]] : 0.0f;
  float v = 0.0f;
#pragma unroll
  for (int n = 0; n < kGatherSlots; ++n) {
    if (w[n] == 0.0f) return v;
    if (idx[n] >= 0 && idx[n] < len) v = v + f[n] * w[n];
  }
  for (int n = kGatherSlots; n < K; ++n) {
    const float wn = d.weights[base + n * stride];
    if (wn == 0.0f) break;
    const int i = d.indices[base + n * stride];
    if (i >= 0 && i < len) v = v + field[i] * wn;
  }
  return v;
}

__global__ void __launch_bounds__(kDftThreads) dft_kernel(DftDev d, const int* counter, int step_offset) {
  const int mc = blockIdx.y;
  const int m = mc / 6;
  const int c = mc % 6;
  const int* cnt = d.counts + 5 * m;
  // Counts live on the device; clamp them to the arena extents so that a
  // malformed plan can never address outside the buffers it names.
  const int nf = min(max(cnt[0], 0), d.max_freqs);
  const int np = min(max(cnt[1], 0), d.max_points);
  const int interval = cnt[2] > 0 ? cnt[2] : 1;
  const int voff = cnt[3], woff = cnt[4];
  const int step = counter[0] + step_offset;
  if (step % interval != 0) return;
  int ti = step < 0 ? 0 : step;
  ti = ti >= d.step_time_len ? d.step_time_len - 1 : ti;
  const float t = d.step_time[ti];
  const float t0 = d.windows[3 * m], t1 = d.windows[3 * m + 1], unit = d.windows[3 * m + 2];
  if (!(t >= t0 && t <= t1)) return;

  __shared__ float s_cos[kDftMaxFreqs];
  __shared__ float s_sin[kDftMaxFreqs];
  __shared__ float s_scale;
  __shared__ float s_window;
  if (threadIdx.x == 0) {
    float window = 1.0f;
    if (d.codes[2 * m] == 1 && isfinite(t1) && t1 > t0) {
      const float span = fmaxf(t1 - t0, 1e-30f);
      const float tau = fminf(fmaxf((t - t0) / span, 0.0f), 1.0f);
      window = 0.5f * (1.0f - cosf(6.2831855f * tau));
    }
    float scale = fmaxf(window, 0.0f);
    if (d.codes[2 * m + 1] == 1) {
      // ((dt * interval) * c / L) / sqrt(2 pi), each step in float32 (observe.py:352-356).
      const float phys = ((d.dt * static_cast<float>(interval)) * 299792458.0f) / unit;
      scale = scale * (phys / sqrtf(6.2831855f));
    }
    s_scale = scale;
    s_window = window;
  }
  for (int f = threadIdx.x; f < nf; f += blockDim.x) {
    // theta = (fl32(2 pi) * f) * t, all float32 (observe.py:533-538).
    const float theta = (6.2831855f * d.freqs[m * d.max_freqs + f]) * t;
    float sn, cs;
    sincosf(theta, &sn, &cs);
    s_cos[f] = cs;
    s_sin[f] = sn;
  }
  __syncthreads();
  if (c == 0 && blockIdx.x == 0) {
    for (int f = threadIdx.x; f < nf; f += blockDim.x)
      if (woff >= 0 && woff + f < d.weight_len) d.weight_sum[woff + f] += s_window;
  }
  const float mask = d.masks[m * 6 + c];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np || mask == 0.0f) return;
  if (voff < 0 || voff + static_cast<int64_t>(6) * nf * np > d.arena_len) return;
  const float v = dft_gather(d, m, c, p);
  const float sm = s_scale * mask;
  const int64_t out = voff + (static_cast<int64_t>(c) * nf) * np + p;
  for (int f = 0; f < nf; ++f) {
    d.re[out + static_cast<int64_t>(f) * np] += sm * (s_cos[f] * v);
    d.im[out + static_cast<int64_t>(f) * np] += sm * (s_sin[f] * v);
  }
}

// Step batching: dft_sample_kernel stores one step's gathered sample of every
// (monitor, component, point) into slot `slot` of a [batch, M, 6, P] buffer;
// dft_flush_kernel then adds `count` buffered steps to the arena in step
// order, with the same gate, window, scale and phase per step as dft_kernel,
// so the arena is bit-identical to per-step accumulation while it is read
// and written once per batch.
constexpr int kDftMaxBatch = 16;

// 128-thread blocks at 32 registers: one fits on an SM beside five resident
// step CTAs, so sampling on a side stream overlaps the next step.
constexpr int kDftSampleThreads = 128;

// A (monitor, component) whose plan has the affine form (FdtdDft::affine) is
// sampled without reading the plan: the block's 128 threads take tiles of
// 32 points along b by 4 along a, so the rows that neighbouring points share
// (the other slot of a two-plane interpolation) are read once through L1.
__global__ void __launch_bounds__(kDftSampleThreads, 16) dft_sample_kernel(DftDev d, float* samples, int slot) {
  const int mc = blockIdx.y;
  const int m = mc / 6, c = mc % 6;
  const int np = min(max(d.counts[5 * m + 1], 0), d.max_points);
  if (d.masks[m * 6 + c] == 0.0f) return;
  float* out = samples + ((static_cast<int64_t>(slot) * d.monitor_count + m) * 6 + c) * d.max_points;
  const int* af = d.affine != nullptr ? d.affine + mc * 24 : nullptr;
  if (af != nullptr && af[0] == 1) {
    const int na = af[1], nb = af[2], base = af[3], sa = af[4], sb = af[5], k = min(af[6], kGatherSlots);
    if (static_cast<int64_t>(na) * nb > np) return;  // not this plan's form: nothing is sampled
    int delta[kGatherSlots];
    float w[kGatherSlots];
#pragma unroll
    for (int s = 0; s < kGatherSlots; ++s) {
      delta[s] = af[8 + s];
      w[s] = __int_as_float(af[16 + s]);
    }
    const float* field = d.fields[c];
    const int64_t len = d.field_len[c];
    const int tb = (nb + 31) / 32, tiles = tb * ((na + 3) / 4);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
      const int a = (t / tb) * 4 + ty, b = (t % tb) * 32 + tx;
      if (a >= na || b >= nb) continue;
      const int64_t i0 = base + static_cast<int64_t>(a) * sa + static_cast<int64_t>(b) * sb;
      float f[kGatherSlots];
#pragma unroll
      for (int s = 0; s < kGatherSlots; ++s) {
        const int64_t i = i0 + delta[s];
        f[s] = (s < k && i >= 0 && i < len) ? field[i] : 0.0f;
      }
      float v = 0.0f;
#pragma unroll
      for (int s = 0; s < kGatherSlots; ++s) {
        const int64_t i = i0 + delta[s];
        if (s < k && i >= 0 && i < len) v = v + f[s] * w[s];
      }
      out[static_cast<int64_t>(a) * nb + b] = v;
    }
    return;
  }
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  out[p] = dft_gather(d, m, c, p);
}

__global__ void __launch_bounds__(kDftThreads) dft_flush_kernel(DftDev d, const float* samples, const int* counter,
                                                                int first, int count) {
  const int mc = blockIdx.y;
  const int m = mc / 6, c = mc % 6;
  const int* cnt = d.counts + 5 * m;
  const int nf = min(max(cnt[0], 0), d.max_freqs);
  const int np = min(max(cnt[1], 0), d.max_points);
  const int interval = cnt[2] > 0 ? cnt[2] : 1;
  const int voff = cnt[3], woff = cnt[4];
  const float t0 = d.windows[3 * m], t1 = d.windows[3 * m + 1], unit = d.windows[3 * m + 2];
  __shared__ float s_cos[kDftMaxBatch][kDftMaxFreqs];
  __shared__ float s_sin[kDftMaxBatch][kDftMaxFreqs];
  __shared__ float s_scale[kDftMaxBatch];
  __shared__ float s_window[kDftMaxBatch];
  __shared__ float s_time[kDftMaxBatch];
  __shared__ int s_on[kDftMaxBatch];
  for (int s = threadIdx.x; s < count; s += blockDim.x) {
    const int step = counter[0] + first + s;
    int ti = step < 0 ? 0 : step;
    ti = ti >= d.step_time_len ? d.step_time_len - 1 : ti;
    const float t = d.step_time[ti];
    const bool on = step % interval == 0 && t >= t0 && t <= t1;
    float window = 1.0f;
    if (on && d.codes[2 * m] == 1 && isfinite(t1) && t1 > t0) {
      const float span = fmaxf(t1 - t0, 1e-30f);
      const float tau = fminf(fmaxf((t - t0) / span, 0.0f), 1.0f);
      window = 0.5f * (1.0f - cosf(6.2831855f * tau));
    }
    float scale = fmaxf(window, 0.0f);
    if (d.codes[2 * m + 1] == 1) {
      const float phys = ((d.dt * static_cast<float>(interval)) * 299792458.0f) / unit;
      scale = scale * (phys / sqrtf(6.2831855f));
    }
    s_on[s] = on ? 1 : 0;
    s_scale[s] = scale;
    s_window[s] = window;
    s_time[s] = t;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < count * nf; e += blockDim.x) {
    const int s = e / nf, f = e % nf;
    const float theta = (6.2831855f * d.freqs[m * d.max_freqs + f]) * s_time[s];
    float sn, cs;
    sincosf(theta, &sn, &cs);
    s_cos[s][f] = cs;
    s_sin[s][f] = sn;
  }
  __syncthreads();
  if (c == 0 && blockIdx.x == 0) {
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
      if (woff < 0 || woff + f >= d.weight_len) continue;
      float ws = d.weight_sum[woff + f];
      for (int s = 0; s < count; ++s)
        if (s_on[s]) ws += s_window[s];
      d.weight_sum[woff + f] = ws;
    }
  }
  const float mask = d.masks[m * 6 + c];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np || mask == 0.0f) return;
  if (voff < 0 || voff + static_cast<int64_t>(6) * nf * np > d.arena_len) return;
  const int64_t out = voff + (static_cast<int64_t>(c) * nf) * np + p;
  const int64_t stride = static_cast<int64_t>(d.monitor_count) * 6 * d.max_points;
  const float* v = samples + (static_cast<int64_t>(m) * 6 + c) * d.max_points + p;
  // The point's buffered samples are loaded once, and the arena words of
  // kFlushFreqs frequencies together, so a flush costs a few memory round
  // trips per point; each arena word still adds the steps in step order.
  constexpr int kFlushFreqs = 4;
  float vs[kDftMaxBatch];
#pragma unroll
  for (int s = 0; s < kDftMaxBatch; ++s) vs[s] = s < count && s_on[s] ? v[s * stride] : 0.0f;
  for (int f0 = 0; f0 < nf; f0 += kFlushFreqs) {
    float re[kFlushFreqs], im[kFlushFreqs];
#pragma unroll
    for (int q = 0; q < kFlushFreqs; ++q) {
      const int64_t o = out + static_cast<int64_t>(f0 + q) * np;
      re[q] = f0 + q < nf ? d.re[o] : 0.0f;
      im[q] = f0 + q < nf ? d.im[o] : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < kFlushFreqs; ++q) {
      const int f = f0 + q;
      if (f >= nf) break;
#pragma unroll
      for (int s = 0; s < kDftMaxBatch; ++s) {
        if (s >= count) break;
        if (!s_on[s]) continue;
        const float sm = s_scale[s] * mask;
        re[q] += sm * (s_cos[s][f] * vs[s]);
        im[q] += sm * (s_sin[s][f] * vs[s]);
      }
      const int64_t o = out + static_cast<int64_t>(f) * np;
      d.re[o] = re[q];
      d.im[o] = im[q];
    }
  }
}

__global__ void counter_kernel(int* counter, int nsteps) { counter[0] += nsteps; }

}  // namespace

cudaError_t launch_copy3d(cudaStream_t s, const float* src, int64_t src_row, int64_t src_plane, float* dst,
                          int64_t dst_row, int64_t dst_plane, int64_t nz, int64_t ny, int64_t nx) {
  if (nz <= 0 || ny <= 0 || nx <= 0) return cudaSuccess;
  const dim3 block(128, 2, 1);
  const dim3 grid(static_cast<unsigned>((nx + 127) / 128 > 64 ? 64 : (nx + 127) / 128),
                  static_cast<unsigned>((ny + 1) / 2 > 512 ? 512 : (ny + 1) / 2), static_cast<unsigned>(nz));
  copy3d_kernel<<<grid, block, 0, s>>>(src, src_row, src_plane, dst, dst_row, dst_plane, ny, nx);
  return cudaPeekAtLastError();
}

cudaError_t launch_source(cudaStream_t s, const SourceDev& src, float* target, Dims td, int64_t row, int64_t plane,
                          int timing, int metallic, const int* counter, int step_offset) {
  if (src.ex <= 0 || src.ey <= 0 || src.ez <= 0) return cudaSuccess;
  const int bx = src.ex >= 32 ? 32 : (src.ex >= 8 ? 8 : 1);
  const int by = 256 / bx > 32 ? 32 : 256 / bx;
  const dim3 block(bx, by, 1);
  const dim3 grid((src.ex + bx - 1) / bx, (src.ey + by - 1) / by, src.ez);
  source_kernel<<<grid, block, 0, s>>>(src, target, td, row, plane, timing, metallic, counter, step_offset);
  return cudaPeekAtLastError();
}

cudaError_t launch_dft(cudaStream_t s, const DftDev& dft, const int* counter, int step_offset) {
  if (dft.monitor_count <= 0 || dft.max_points <= 0) return cudaSuccess;
  if (dft.max_freqs > kDftMaxFreqs) return cudaErrorInvalidValue;
  const dim3 grid((dft.max_points + kDftThreads - 1) / kDftThreads, dft.monitor_count * 6, 1);
  dft_kernel<<<grid, kDftThreads, 0, s>>>(dft, counter, step_offset);
  return cudaPeekAtLastError();
}

cudaError_t launch_dft_sample(cudaStream_t s, const DftDev& dft, float* samples, int slot) {
  if (dft.monitor_count <= 0 || dft.max_points <= 0) return cudaSuccess;
  const dim3 grid((dft.max_points + kDftSampleThreads - 1) / kDftSampleThreads, dft.monitor_count * 6, 1);
  dft_sample_kernel<<<grid, kDftSampleThreads, 0, s>>>(dft, samples, slot);
  return cudaPeekAtLastError();
}

cudaError_t launch_dft_flush(cudaStream_t s, const DftDev& dft, const float* samples, const int* counter, int first,
                             int count) {
  if (dft.monitor_count <= 0 || dft.max_points <= 0 || count <= 0) return cudaSuccess;
  if (dft.max_freqs > kDftMaxFreqs || count > kDftMaxBatch) return cudaErrorInvalidValue;
  const dim3 grid((dft.max_points + kDftThreads - 1) / kDftThreads, dft.monitor_count * 6, 1);
  dft_flush_kernel<<<grid, kDftThreads, 0, s>>>(dft, samples, counter, first, count);
  return cudaPeekAtLastError();
}

cudaError_t launch_counter_advance(cudaStream_t s, int* counter, int nsteps) {
  counter_kernel<<<1, 1, 0, s>>>(counter, nsteps);
  return cudaPeekAtLastError();
}

}  // namespace fdtd
