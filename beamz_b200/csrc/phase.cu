// In-place half-step kernels: H from E, then E from H.
//
// These are the phase-level entry (beamz: UpdateFusedComponents,
// cuda/src/update.cu:309-427, which serves beamz/simulation/cuda/runtime.py
// update_h/update_e) and the one-bank step schedule.  Every thread owns one
// (z, y, x) lattice point and updates each active component defined there.
// H phase reads only E and its own H/psi cell, E phase only H and its own E/psi
// cell, so updating in place is race-free.
//
// 2D programs run through the same kernels: TM (Ez, Hx, Hy) as a z extent of
// one cell, TE (Ex, Ey, Hz) as a zero-cell z axis whose E/Hz supports still
// hold one plane; inactive components read as zero and are never written.

#include "kernels.cuh"

namespace fdtd {

namespace {

template <int Active>
__device__ __forceinline__ bool active(int c) {
  return (Active >> c) & 1;
}

template <int Active>
__device__ __forceinline__ float ld(const Step3D& p, const float* const* base, int c, int k, int j, int i) {
  if (!active<Active>(c)) return 0.0f;
  const Dims d = component_dims(c, p.Z, p.Y, p.X);
  return base[c < 3 ? c : c - 3][lin(d, k, j, i)];
}

// Forward difference of E component `c` along `axis` at (k, j, i), divided by
// the cell size (beamz/simulation/kernels.py:477-488: jnp.diff(...) / resolution)
// or scaled by the grid's metric (kernels.py:506-551).
template <int Active, bool Metric>
__device__ __forceinline__ float fdiff(const Step3D& p, int c, int axis, int k, int j, int i) {
  if (!active<Active>(c)) return 0.0f;
  const float lo = ld<Active>(p, p.ein, c, k, j, i);
  const float hi = ld<Active>(p, p.ein, c, k + (axis == 0), j + (axis == 1), i + (axis == 2));
  return dh<Metric>(p, axis, axis == 0 ? k : (axis == 1 ? j : i), hi - lo);
}

// Backward difference of H component `c` along `axis` with beamz's ghost
// planes: zero beyond a metallic wall, else a copy of the edge plane
// (beamz/lattice.py:523-551, beamz/simulation/kernels.py:574-586).
template <int Active, bool Metric>
__device__ __forceinline__ float bdiff(const Step3D& p, int c, int axis, int k, int j, int i) {
  if (!active<Active>(c)) return 0.0f;
  const Dims d = component_dims(c, p.Z, p.Y, p.X);
  const int n = axis == 0 ? d.z : (axis == 1 ? d.y : d.x);
  const int coord = axis == 0 ? k : (axis == 1 ? j : i);
  if (n == 0) return 0.0f;
  if (coord == 0) {
    if (!wall(p.metallic, axis, false)) return 0.0f;
    return de<Metric>(p, axis, coord, ld<Active>(p, p.hin, c, k, j, i) - 0.0f);
  }
  if (coord == n) {
    if (!wall(p.metallic, axis, true)) return 0.0f;
    return de<Metric>(p, axis, coord, 0.0f - ld<Active>(p, p.hin, c, k - (axis == 0), j - (axis == 1), i - (axis == 2)));
  }
  const float hi = ld<Active>(p, p.hin, c, k, j, i);
  const float lo = ld<Active>(p, p.hin, c, k - (axis == 0), j - (axis == 1), i - (axis == 2));
  return de<Metric>(p, axis, coord, hi - lo);
}

template <int Active, bool Cpml, int Mat, bool Metric>
__global__ void __launch_bounds__(256) phase_h_kernel(Step3D p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  // Hx: curl_x = dEz/dy - dEy/dz (terms Hxy +, Hxz -).
  if (active<Active>(3)) {
    const Dims d = component_dims(3, p.Z, p.Y, p.X);
    if (k < d.z && j < d.y && i < d.x) {
      float d0 = fdiff<Active, Metric>(p, 2, 1, k, j, i);
      float d1 = fdiff<Active, Metric>(p, 1, 0, k, j, i);
      if (Cpml) {
        d0 = cpml_correct<1>(p.ht[0], d0, k, j, i, true);
        d1 = cpml_correct<0>(p.ht[1], d1, k, j, i, true);
      }
      const int64_t o = lin(d, k, j, i);
      float h = h_update(p.hm, 0, o, p.hin[0][o], d0 - d1);
      if ((i == 0 && wall(p.metallic, 2, false)) || (i == d.x - 1 && wall(p.metallic, 2, true))) h = 0.0f;
      p.hout[0][o] = h;
    }
  }
  // Hy: curl_y = dEx/dz - dEz/dx (terms Hyz +, Hyx -).
  if (active<Active>(4)) {
    const Dims d = component_dims(4, p.Z, p.Y, p.X);
    if (k < d.z && j < d.y && i < d.x) {
      float d0 = fdiff<Active, Metric>(p, 0, 0, k, j, i);
      float d1 = fdiff<Active, Metric>(p, 2, 2, k, j, i);
      if (Cpml) {
        d0 = cpml_correct<0>(p.ht[2], d0, k, j, i, true);
        d1 = cpml_correct<2>(p.ht[3], d1, k, j, i, true);
      }
      const int64_t o = lin(d, k, j, i);
      float h = h_update(p.hm, 1, o, p.hin[1][o], d0 - d1);
      if ((j == 0 && wall(p.metallic, 1, false)) || (j == d.y - 1 && wall(p.metallic, 1, true))) h = 0.0f;
      p.hout[1][o] = h;
    }
  }
  // Hz: curl_z = dEy/dx - dEx/dy (terms Hzx +, Hzy -).
  if (active<Active>(5)) {
    const Dims d = component_dims(5, p.Z, p.Y, p.X);
    if (k < d.z && j < d.y && i < d.x) {
      float d0 = fdiff<Active, Metric>(p, 1, 2, k, j, i);
      float d1 = fdiff<Active, Metric>(p, 0, 1, k, j, i);
      if (Cpml) {
        d0 = cpml_correct<2>(p.ht[4], d0, k, j, i, true);
        d1 = cpml_correct<1>(p.ht[5], d1, k, j, i, true);
      }
      const int64_t o = lin(d, k, j, i);
      float h = h_update(p.hm, 2, o, p.hin[2][o], d0 - d1);
      if ((k == 0 && wall(p.metallic, 0, false)) || (k == d.z - 1 && wall(p.metallic, 0, true))) h = 0.0f;
      p.hout[2][o] = h;
    }
  }
}

template <int Active, bool Cpml, int Mat, bool Metric>
__global__ void __launch_bounds__(256) phase_e_kernel(Step3D p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  // Ex: dHz/dy - dHy/dz (terms Exy +, Exz -).
  if (active<Active>(0)) {
    const Dims d = component_dims(0, p.Z, p.Y, p.X);
    if (k < d.z && j < d.y && i < d.x) {
      float d0 = bdiff<Active, Metric>(p, 5, 1, k, j, i);
      float d1 = bdiff<Active, Metric>(p, 4, 0, k, j, i);
      if (Cpml) {
        d0 = cpml_correct<1>(p.et[0], d0, k, j, i, true);
        d1 = cpml_correct<0>(p.et[1], d1, k, j, i, true);
      }
      const int64_t o = lin(d, k, j, i);
      float e = e_update<Mat>(p, 0, o, k, j, i, p.ein[0][o], d0 - d1);
      if (e_constrained(p.metallic, 0, d, k, j, i)) e = 0.0f;
      p.eout[0][o] = e;
    }
  }
  // Ey: dHx/dz - dHz/dx (terms Eyz +, Eyx -).
  if (active<Active>(1)) {
    const Dims d = component_dims(1, p.Z, p.Y, p.X);
    if (k < d.z && j < d.y && i < d.x) {
      float d0 = bdiff<Active, Metric>(p, 3, 0, k, j, i);
      float d1 = bdiff<Active, Metric>(p, 5, 2, k, j, i);
      if (Cpml) {
        d0 = cpml_correct<0>(p.et[2], d0, k, j, i, true);
        d1 = cpml_correct<2>(p.et[3], d1, k, j, i, true);
      }
      const int64_t o = lin(d, k, j, i);
      float e = e_update<Mat>(p, 1, o, k, j, i, p.ein[1][o], d0 - d1);
      if (e_constrained(p.metallic, 1, d, k, j, i)) e = 0.0f;
      p.eout[1][o] = e;
    }
  }
  // Ez: dHy/dx - dHx/dy (terms Ezx +, Ezy -).
  if (active<Active>(2)) {
    const Dims d = component_dims(2, p.Z, p.Y, p.X);
    if (k < d.z && j < d.y && i < d.x) {
      float d0 = bdiff<Active, Metric>(p, 4, 2, k, j, i);
      float d1 = bdiff<Active, Metric>(p, 3, 1, k, j, i);
      if (Cpml) {
        d0 = cpml_correct<2>(p.et[4], d0, k, j, i, true);
        d1 = cpml_correct<1>(p.et[5], d1, k, j, i, true);
      }
      const int64_t o = lin(d, k, j, i);
      float e = e_update<Mat>(p, 2, o, k, j, i, p.ein[2][o], d0 - d1);
      if (e_constrained(p.metallic, 2, d, k, j, i)) e = 0.0f;
      p.eout[2][o] = e;
    }
  }
}

template <int Active, bool Cpml, int Mat>
cudaError_t launch_phase_t(cudaStream_t s, const Step3D& p, int phase) {
  int zmax = 0, ymax = 0, xmax = 0;
  for (int c = 0; c < 6; ++c) {
    if (!((Active >> c) & 1)) continue;
    const Dims d = component_dims(c, p.Z, p.Y, p.X);
    zmax = d.z > zmax ? d.z : zmax;
    ymax = d.y > ymax ? d.y : ymax;
    xmax = d.x > xmax ? d.x : xmax;
  }
  if (zmax == 0 || ymax == 0 || xmax == 0) return cudaSuccess;
  const dim3 block(32, 8, 1);
  const dim3 grid((xmax + 31) / 32, (ymax + 7) / 8, zmax);
  const bool metric = has_metric(p);
  if (phase == 0) {
    if (metric) phase_h_kernel<Active, Cpml, Mat, true><<<grid, block, 0, s>>>(p);
    else phase_h_kernel<Active, Cpml, Mat, false><<<grid, block, 0, s>>>(p);
  } else {
    if (metric) phase_e_kernel<Active, Cpml, Mat, true><<<grid, block, 0, s>>>(p);
    else phase_e_kernel<Active, Cpml, Mat, false><<<grid, block, 0, s>>>(p);
  }
  return cudaPeekAtLastError();
}

template <int Active>
cudaError_t launch_phase_a(cudaStream_t s, const Step3D& p, int phase, int mat) {
  if (p.cpml) {
    return mat ? launch_phase_t<Active, true, 1>(s, p, phase) : launch_phase_t<Active, true, 0>(s, p, phase);
  }
  return mat ? launch_phase_t<Active, false, 1>(s, p, phase) : launch_phase_t<Active, false, 0>(s, p, phase);
}

}  // namespace

cudaError_t launch_phase(cudaStream_t s, const Step3D& p, int phase, int mat, int active_mask) {
  switch (active_mask) {
    case kActive3D: return launch_phase_a<kActive3D>(s, p, phase, mat);
    case kActiveTM: return launch_phase_a<kActiveTM>(s, p, phase, mat);
    case kActiveTE: return launch_phase_a<kActiveTE>(s, p, phase, mat);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fdtd
