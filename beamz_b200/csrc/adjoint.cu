// Discrete adjoint of the leapfrog step (dense layout, per-site E material).
//
// The step without its sources is linear in the state u = (E, H, psi_H,
// psi_E); the adjoint applies the exact transpose of each of its linear maps
// in reverse order (beamz/simulation/execute.py:467-541 gives the forward
// order):
//
//   forward step n                      adjoint step n (on lambda)
//   1. H <- mask_H (dec H - src curl'E)  5. DFT source: lambda += dJ/du_{n+1}
//   2. E <- mask_E (E + c curl'H)        4. E transpose (per E site, then
//   3. DFT of u_{n+1}                       Bx^T gather per H site)
//                                        3. H transpose (per H site, then
//                                           D^T gather per E site)
//
// where curl' sums the CPML-corrected derivatives d' of each term
// (psi' = b psi + a d, d' = d / kappa + psi'; beamz/simulation/kernels.py:
// 257-264), D is the forward difference E -> H and B the ghost-padded
// backward difference H -> E (zero ghost on a metallic face, edge copy
// elsewhere; beamz/lattice.py:523-551).  Transposes:
//   CPML:  acc = lam_psi' + lam_d';  lam_psi = b acc;  lam_d = lam_d' / kappa + a acc
//   D^T:   (D^T u)[m] = (u[m-1] - u[m]) / res   (u outside [0, N) is zero)
//   B^T:   (B^T t)[h] = (r(h) t[h] - r(h+1) t[h+1]) / res, r(m) = 1 for the
//          rows of B that difference two samples or a metallic ghost, 0 for
//          the rows whose edge-copy ghost makes them zero.
//   With derivative metrics (axis-uniform / rectilinear grids) each
//   difference carries its coordinate's inverse distance instead of 1/res:
//   (D^T u)[m] = mh[m-1] u[m-1] - mh[m] u[m] and
//   (B^T t)[h] = r(h) me[h] t[h] - r(h+1) me[h+1] t[h+1].
// Each transpose is split into a per-target pass that writes lam_d into a
// scratch array (one per derivative term) and a per-source gather, so no
// two threads write one element.  The permittivity gradient accumulates
// mu * curl'_n per E site over a design box, mu = the masked E adjoint and
// curl'_n the forward curl recomputed from a checkpoint.


#include "kernels.cuh"

namespace fdtd {

namespace {

// Term tables (3D order: H 0 Hx-y, 1 Hx-z, 2 Hy-z, 3 Hy-x, 4 Hz-x, 5 Hz-y;
// E likewise for Ex, Ey, Ez; even terms enter with +, odd with -).
// The kernels take their component as a template argument, so that these
// lookups (and the term loops of the gathers) resolve at compile time.
__host__ __device__ constexpr int adj_h_src(int t) { return 2 - t % 3; }  // E component an H term differentiates
__host__ __device__ constexpr int adj_e_src(int t) { return 5 - t % 3; }  // H component an E term differentiates
// Axis of term t's derivative, for H and E terms alike: 1, 0, 0, 2, 2, 1.
__host__ __device__ constexpr int adj_axis(int t) { return (t == 0 || t == 5) ? 1 : ((t == 1 || t == 2) ? 0 : 2); }

constexpr int kAdjThreads = 256;

// Element offsets of a component fit 32 bits (every entry point validates
// arrays below 2^31 elements), so the split is two 32-bit divisions rather
// than 64-bit ones, which the GPU emulates in dozens of instructions.
__device__ __forceinline__ void unflat(int64_t idx, const Dims& d, int& k, int& j, int& i) {
  const unsigned id = static_cast<unsigned>(idx), dx = static_cast<unsigned>(d.x), dy = static_cast<unsigned>(d.y);
  const unsigned r = id / dx;
  i = static_cast<int>(id - r * dx);
  k = static_cast<int>(r / dy);
  j = static_cast<int>(r - static_cast<unsigned>(k) * dy);
}

__device__ __forceinline__ int coord_of(int axis, int k, int j, int i) { return axis == 0 ? k : (axis == 1 ? j : i); }

__device__ __forceinline__ int64_t psi_index(const CpmlTermDev& t, int axis, int slot, int k, int j, int i) {
  const int pk = axis == 0 ? slot : k, pj = axis == 1 ? slot : j, pi = axis == 2 ? slot : i;
  return (static_cast<int64_t>(pk) * t.pdy + pj) * static_cast<int64_t>(t.pdx) + pi;
}

// Transpose of one CPML-corrected derivative at a site: lam_d' -> lam_d,
// updating the adjoint memory (held in psi_out) in place.
__device__ __forceinline__ float cpml_transpose(const CpmlTermDev& t, int axis, int k, int j, int i, float ld) {
  const int slot = cpml_slot(t, coord_of(axis, k, j, i));
  if (slot < 0) return ld;
  const int64_t off = psi_index(t, axis, slot, k, j, i);
  const float acc = t.psi_out[off] + ld;
  t.psi_out[off] = t.b[slot] * acc;
  return t.k[slot] * ld + t.a[slot] * acc;
}

__device__ __forceinline__ float coef_at(const float* p, int full, int64_t idx) { return p[full ? idx : 0]; }

// 4a. E transpose, per E site of component c: mask, identity part, the two
// terms' lam_d into scratch, and the design-box gradient.
template <int c>
__global__ void __launch_bounds__(kAdjThreads) adj_e_kernel(Step3D p, AdjDev a) {
  const Dims d = component_dims(c, p.Z, p.Y, p.X);
  const int64_t n = static_cast<int64_t>(d.z) * d.y * d.x;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int k, j, i;
    unflat(idx, d, k, j, i);
    float mu = a.lam[c][idx];
    if (e_constrained(p.metallic, c, d, k, j, i)) mu = 0.0f;
    a.lam[c][idx] = coef_at(p.em.decay[c], p.em.decay_full[c], idx) * mu;
    const float src = coef_at(p.em.source[c], p.em.source_full[c], idx);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int t = 2 * c + s;
      if (a.scratch_e[t] == nullptr) continue;
      float ld = (s == 0 ? src : -src) * mu;
      if (p.cpml) ld = cpml_transpose(p.et[t], adj_axis(t), k, j, i, ld);
      a.scratch_e[t][idx] = ld;
    }
    if (a.grad[c] != nullptr && k >= a.box_lo[0] && k < a.box_hi[0] && j >= a.box_lo[1] && j < a.box_hi[1] &&
        i >= a.box_lo[2] && i < a.box_hi[2]) {
      const int64_t b = (static_cast<int64_t>(k - a.box_lo[0]) * (a.box_hi[1] - a.box_lo[1]) + (j - a.box_lo[1])) *
                            (a.box_hi[2] - a.box_lo[2]) +
                        (i - a.box_lo[2]);
      a.grad[c][b] += mu * a.curl[c][b];
    }
  }
}

// 4b. B^T gather, per H site of component h.
template <int h>
__global__ void __launch_bounds__(kAdjThreads) adj_hgather_kernel(Step3D p, AdjDev a) {
  const Dims d = component_dims(h, p.Z, p.Y, p.X);
  const int64_t n = static_cast<int64_t>(d.z) * d.y * d.x;
  const float inv_res = 1.0f / p.res;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int k, j, i;
    unflat(idx, d, k, j, i);
    float acc = 0.0f;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      if (adj_e_src(t) != h || a.scratch_e[t] == nullptr) continue;
      const int e = t / 2, axis = adj_axis(t);
      const Dims de = component_dims(e, p.Z, p.Y, p.X);
      const int N = axis == 0 ? d.z : (axis == 1 ? d.y : d.x);  // H samples; E has N + 1
      const int m = coord_of(axis, k, j, i);
      const bool lw = wall(p.metallic, axis, false), hw = wall(p.metallic, axis, true);
      auto row = [&](int r) { return (r >= 1 && r <= N - 1) || (r == 0 && lw) || (r == N && hw); };
      const int k1 = axis == 0 ? k + 1 : k, j1 = axis == 1 ? j + 1 : j, i1 = axis == 2 ? i + 1 : i;
      const float t0 = row(m) ? a.scratch_e[t][lin(de, k, j, i)] : 0.0f;
      const float t1 = row(m + 1) ? a.scratch_e[t][lin(de, k1, j1, i1)] : 0.0f;
      // Derivative metrics: the backward difference at E coordinate m was
      // scaled by metric_e[m] (and the ghost rows by metric_e[0] / [N]).
      const float* me = p.metric_e[axis];
      if (me != nullptr)
        acc += t0 * me[m] - t1 * me[m + 1];
      else
        acc += (t0 - t1) * inv_res;
    }
    a.lam[h][idx] += acc;
  }
}

// 3a. H transpose, per H site of component h.
template <int h>
__global__ void __launch_bounds__(kAdjThreads) adj_h_kernel(Step3D p, AdjDev a) {
  const Dims d = component_dims(h, p.Z, p.Y, p.X);
  const int64_t n = static_cast<int64_t>(d.z) * d.y * d.x;
  const int hc = h - 3;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int k, j, i;
    unflat(idx, d, k, j, i);
    float mu = a.lam[h][idx];
    if (h_constrained(p.metallic, h, d, k, j, i)) mu = 0.0f;
    a.lam[h][idx] = coef_at(p.hm.decay[hc], p.hm.decay_full[hc], idx) * mu;
    const float src = coef_at(p.hm.source[hc], p.hm.source_full[hc], idx);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int t = 2 * hc + s;
      if (a.scratch_h[t] == nullptr) continue;
      float ld = (s == 0 ? -src : src) * mu;
      if (p.cpml) ld = cpml_transpose(p.ht[t], adj_axis(t), k, j, i, ld);
      a.scratch_h[t][idx] = ld;
    }
  }
}

// 3b. D^T gather, per E site of component e.
template <int e>
__global__ void __launch_bounds__(kAdjThreads) adj_egather_kernel(Step3D p, AdjDev a) {
  const Dims d = component_dims(e, p.Z, p.Y, p.X);
  const int64_t n = static_cast<int64_t>(d.z) * d.y * d.x;
  const float inv_res = 1.0f / p.res;
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < n;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int k, j, i;
    unflat(idx, d, k, j, i);
    float acc = 0.0f;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      if (adj_h_src(t) != e || a.scratch_h[t] == nullptr) continue;
      const int hcomp = 3 + t / 2, axis = adj_axis(t);
      const Dims dh = component_dims(hcomp, p.Z, p.Y, p.X);
      const int N = axis == 0 ? dh.z : (axis == 1 ? dh.y : dh.x);
      const int m = coord_of(axis, k, j, i);
      const int k0 = axis == 0 ? k - 1 : k, j0 = axis == 1 ? j - 1 : j, i0 = axis == 2 ? i - 1 : i;
      const float u_prev = m >= 1 ? a.scratch_h[t][lin(dh, k0, j0, i0)] : 0.0f;
      const float u_here = m <= N - 1 ? a.scratch_h[t][lin(dh, k, j, i)] : 0.0f;
      // Derivative metrics: the forward difference at H coordinate m was
      // scaled by metric_h[m].
      const float* mh = p.metric_h[axis];
      if (mh != nullptr)
        acc += (m >= 1 ? u_prev * mh[m - 1] : 0.0f) - (m <= N - 1 ? u_here * mh[m] : 0.0f);
      else
        acc += (u_prev - u_here) * inv_res;
    }
    a.lam[e][idx] += acc;
  }
}

// 5. DFT adjoint source for the sample at absolute step `step`:
// lambda[c][idx_k] += w_k * sum_f s (g_re cos(theta_f) + g_im sin(theta_f)),
// the transpose of the accumulation in io.cu (observe.py:529-585).
constexpr int kAdjMaxFreqs = 64;

__global__ void __launch_bounds__(kAdjThreads) adj_dft_kernel(DftDev d, AdjDev a, int step) {
  const int mc = blockIdx.y;
  const int m = mc / 6, c = mc % 6;
  const int* cnt = d.counts + 5 * m;
  const int nf = min(max(cnt[0], 0), d.max_freqs);
  const int np = min(max(cnt[1], 0), d.max_points);
  const int interval = cnt[2] > 0 ? cnt[2] : 1;
  const int voff = cnt[3];
  if (step % interval != 0 || a.lam[c] == nullptr) return;
  int ti = step < 0 ? 0 : step;
  ti = ti >= d.step_time_len ? d.step_time_len - 1 : ti;
  const float t = d.step_time[ti];
  const float t0 = d.windows[3 * m], t1 = d.windows[3 * m + 1], unit = d.windows[3 * m + 2];
  if (!(t >= t0 && t <= t1)) return;
  __shared__ float s_cos[kAdjMaxFreqs], s_sin[kAdjMaxFreqs];
  __shared__ float s_scale;
  if (threadIdx.x == 0) {
    float window = 1.0f;
    if (d.codes[2 * m] == 1 && isfinite(t1) && t1 > t0) {
      const float span = fmaxf(t1 - t0, 1e-30f);
      const float tau = fminf(fmaxf((t - t0) / span, 0.0f), 1.0f);
      window = 0.5f * (1.0f - cosf(6.2831855f * tau));
    }
    float scale = fmaxf(window, 0.0f);
    if (d.codes[2 * m + 1] == 1) {
      const float phys = ((d.dt * static_cast<float>(interval)) * 299792458.0f) / unit;
      scale = scale * (phys / sqrtf(6.2831855f));
    }
    s_scale = scale;
  }
  for (int f = threadIdx.x; f < nf; f += blockDim.x) {
    const float theta = (6.2831855f * d.freqs[m * d.max_freqs + f]) * t;
    float sn, cs;
    sincosf(theta, &sn, &cs);
    s_cos[f] = cs;
    s_sin[f] = sn;
  }
  __syncthreads();
  const float mask = d.masks[m * 6 + c];
  const int pidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (pidx >= np || mask == 0.0f) return;
  if (voff < 0 || voff + static_cast<int64_t>(6) * nf * np > d.arena_len) return;
  const int64_t out = voff + (static_cast<int64_t>(c) * nf) * np + pidx;
  float g = 0.0f;
  for (int f = 0; f < nf; ++f) {
    const int64_t o = out + static_cast<int64_t>(f) * np;
    g += a.dft_grad_re[o] * s_cos[f] + a.dft_grad_im[o] * s_sin[f];
  }
  g *= s_scale * mask;
  if (g == 0.0f) return;
  const int64_t base = ((static_cast<int64_t>(m) * 6 + c) * d.neighbors) * d.max_points + pidx;
  for (int nb = 0; nb < d.neighbors; ++nb) {
    const float w = d.weights[base + static_cast<int64_t>(nb) * d.max_points];
    if (w == 0.0f) break;
    const int idx = d.indices[base + static_cast<int64_t>(nb) * d.max_points];
    if (idx >= 0 && idx < d.field_len[c]) atomicAdd(a.lam[c] + idx, w * g);
  }
}

// Forward curl of E component c over the design box from the current H
// (interior sites: plain differences, no ghost and no CPML; validated).
__global__ void __launch_bounds__(kAdjThreads) adj_curl_kernel(Step3D p, AdjDev a, int c) {
  const int bz = a.box_hi[0] - a.box_lo[0], by = a.box_hi[1] - a.box_lo[1], bx = a.box_hi[2] - a.box_lo[2];
  const int64_t n = static_cast<int64_t>(bz) * by * bx;
  const float res = p.res;
  const Dims dx = component_dims(3, p.Z, p.Y, p.X), dy = component_dims(4, p.Z, p.Y, p.X),
             dz = component_dims(5, p.Z, p.Y, p.X);
  for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b < n;
       b += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = a.box_lo[2] + static_cast<int>(b % bx);
    const int j = a.box_lo[1] + static_cast<int>((b / bx) % by);
    const int k = a.box_lo[0] + static_cast<int>(b / (static_cast<int64_t>(bx) * by));
    const float* Hx = p.hin[0];
    const float* Hy = p.hin[1];
    const float* Hz = p.hin[2];
    // A backward difference along `axis` at E coordinate `at`: divided by the
    // cell size, or times the derivative metric there.
    auto sc = [&](float diff, int axis, int at) {
      const float* me = p.metric_e[axis];
      return me != nullptr ? diff * me[at] : diff / res;
    };
    float curl;
    if (c == 0) {
      curl = sc(Hz[lin(dz, k, j, i)] - Hz[lin(dz, k, j - 1, i)], 1, j);
      if (Hy) curl -= sc(Hy[lin(dy, k, j, i)] - Hy[lin(dy, k - 1, j, i)], 0, k);
    } else if (c == 1) {
      curl = -sc(Hz[lin(dz, k, j, i)] - Hz[lin(dz, k, j, i - 1)], 2, i);
      if (Hx) curl += sc(Hx[lin(dx, k, j, i)] - Hx[lin(dx, k - 1, j, i)], 0, k);
    } else {
      curl = sc(Hy[lin(dy, k, j, i)] - Hy[lin(dy, k, j, i - 1)], 2, i) -
             sc(Hx[lin(dx, k, j, i)] - Hx[lin(dx, k, j - 1, i)], 1, j);
    }
    a.curl[c][b] = curl;
  }
}

// Grid-stride launches of 16 blocks per SM: each thread then takes a few
// dozen elements of a large component rather than one, so block scheduling
// does not dominate these short per-element passes.
unsigned blocks_for(int64_t n) {
  int dev = 0, sms = 0;  // the current device's SM count (a cheap attribute query)
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      sms <= 0)
    sms = 148;
  const int64_t b = (n + kAdjThreads - 1) / kAdjThreads;
  const int64_t cap = static_cast<int64_t>(sms) * 16;
  return static_cast<unsigned>(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

cudaError_t launch_adjoint_step(cudaStream_t s, const Step3D& p, const DftDev* dft, const AdjDev& a, int active,
                                int step) {
  if (dft != nullptr && dft->monitor_count > 0 && dft->max_points > 0 && a.dft_grad_re != nullptr) {
    if (dft->max_freqs > kAdjMaxFreqs) return cudaErrorInvalidValue;
    const dim3 grid((dft->max_points + kAdjThreads - 1) / kAdjThreads, dft->monitor_count * 6, 1);
    adj_dft_kernel<<<grid, kAdjThreads, 0, s>>>(*dft, a, step);
  }
  // One launch per active component and pass, in the component order of the
  // transpose (E sites, B^T gathers, H sites, D^T gathers).
  auto grid = [&](int c) {
    const Dims d = component_dims(c, p.Z, p.Y, p.X);
    return blocks_for(static_cast<int64_t>(d.z) * d.y * d.x);
  };
  if (active & 1) adj_e_kernel<0><<<grid(0), kAdjThreads, 0, s>>>(p, a);
  if (active & 2) adj_e_kernel<1><<<grid(1), kAdjThreads, 0, s>>>(p, a);
  if (active & 4) adj_e_kernel<2><<<grid(2), kAdjThreads, 0, s>>>(p, a);
  if (active & 8) adj_hgather_kernel<3><<<grid(3), kAdjThreads, 0, s>>>(p, a);
  if (active & 16) adj_hgather_kernel<4><<<grid(4), kAdjThreads, 0, s>>>(p, a);
  if (active & 32) adj_hgather_kernel<5><<<grid(5), kAdjThreads, 0, s>>>(p, a);
  if (active & 8) adj_h_kernel<3><<<grid(3), kAdjThreads, 0, s>>>(p, a);
  if (active & 16) adj_h_kernel<4><<<grid(4), kAdjThreads, 0, s>>>(p, a);
  if (active & 32) adj_h_kernel<5><<<grid(5), kAdjThreads, 0, s>>>(p, a);
  if (active & 1) adj_egather_kernel<0><<<grid(0), kAdjThreads, 0, s>>>(p, a);
  if (active & 2) adj_egather_kernel<1><<<grid(1), kAdjThreads, 0, s>>>(p, a);
  if (active & 4) adj_egather_kernel<2><<<grid(2), kAdjThreads, 0, s>>>(p, a);
  return cudaPeekAtLastError();
}

// ---- adjoint step without caller scratch -----------------------------------
// The per-term scratch of fdtd_adjoint_step_noalloc lives in this one
// file-scope device array (FDTD_ADJOINT_NOALLOC_MAX_FLOATS floats, 16 MiB),
// so that entry point allocates no device memory.  Every call shares it:
// calls that overlap on the GPU race.  Nothing in it needs clearing: each
// call writes every scratch element it reads before reading it.
static __device__ __align__(256) float g_adjoint_scratch[FDTD_ADJOINT_NOALLOC_MAX_FLOATS];

namespace {

// Device address of g_adjoint_scratch on the current device.  Looked up on
// every call (a cheap runtime query) rather than cached, so that the address
// stays right after the device's context is torn down and re-created (the
// module, and with it the array, may then sit elsewhere).
cudaError_t adjoint_scratch_address(float** out) {
  void* p = nullptr;
  const cudaError_t err = cudaGetSymbolAddress(&p, g_adjoint_scratch);
  if (err != cudaSuccess) return err;
  *out = static_cast<float*>(p);
  return cudaSuccess;
}

}  // namespace

int64_t adjoint_noalloc_span(int64_t floats) { return (floats + 63) / 64 * 64; }

cudaError_t launch_adjoint_step_noalloc(cudaStream_t s, const Step3D& p, const DftDev* dft, AdjDev a, int active,
                                        int step, const int64_t e_len[6], const int64_t h_len[6]) {
  int64_t need = 0;
  for (int t = 0; t < 6; ++t) {
    need += e_len[t] > 0 ? adjoint_noalloc_span(e_len[t]) : 0;
    need += h_len[t] > 0 ? adjoint_noalloc_span(h_len[t]) : 0;
  }
  if (need > FDTD_ADJOINT_NOALLOC_MAX_FLOATS) return cudaErrorInvalidValue;  // before any work
  float* base = nullptr;
  const cudaError_t err = adjoint_scratch_address(&base);
  if (err != cudaSuccess) return err;
  int64_t off = 0;
  for (int t = 0; t < 6; ++t) {
    a.scratch_e[t] = e_len[t] > 0 ? base + off : nullptr;
    off += e_len[t] > 0 ? adjoint_noalloc_span(e_len[t]) : 0;
  }
  for (int t = 0; t < 6; ++t) {
    a.scratch_h[t] = h_len[t] > 0 ? base + off : nullptr;
    off += h_len[t] > 0 ? adjoint_noalloc_span(h_len[t]) : 0;
  }
  return launch_adjoint_step(s, p, dft, a, active, step);
}

cudaError_t launch_adjoint_curl(cudaStream_t s, const Step3D& p, const AdjDev& a, int active) {
  const int64_t n = static_cast<int64_t>(a.box_hi[0] - a.box_lo[0]) * (a.box_hi[1] - a.box_lo[1]) *
                    (a.box_hi[2] - a.box_lo[2]);
  if (n <= 0) return cudaSuccess;
  for (int c = 0; c < 3; ++c) {
    if (!((active >> c) & 1) || a.curl[c] == nullptr) continue;
    adj_curl_kernel<<<blocks_for(n), kAdjThreads, 0, s>>>(p, a, c);
  }
  return cudaPeekAtLastError();
}

}  // namespace fdtd
