// Shared device-side definitions for the B200 FDTD kernels.
//
// Arithmetic contract: this translation unit family is compiled with
// -fmad=false so that every product and sum rounds separately, in the order
// written, exactly as beamz's JAX CPU path evaluates
// (beamz/simulation/kernels.py:257-264, 458-626).  Where a fused multiply-add
// is wanted it is written explicitly with fmaf().
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/fdtd_b200.h"

namespace fdtd {

// Maximum number of h-timing sources fused into the z-marching step kernel.
constexpr int kMaxFusedSources = FDTD_MAX_SOURCES;

// A component's storage extents (z, y, x).  2D programs use z = 1.
struct Dims {
  int z, y, x;
};

__host__ __device__ inline Dims component_dims(int c, int Z, int Y, int X) {
  // beamz/lattice.py:14-45: +1 on every axis where the Yee offset is 0.
  switch (c) {
    case 0: return {Z + 1, Y + 1, X};  // Ex
    case 1: return {Z + 1, Y, X + 1};  // Ey
    case 2: return {Z, Y + 1, X + 1};  // Ez
    case 3: return {Z, Y, X + 1};      // Hx
    case 4: return {Z, Y + 1, X};      // Hy
    default: return {Z + 1, Y, X};     // Hz
  }
}

__host__ __device__ inline Dims component_dims_2d(int c, int pol, int Y, int X) {
  // beamz/lattice.py:789-813, canonical xy plane, z extent 1.
  if (pol == 0) {
    if (c == 2) return {1, Y + 1, X + 1};  // Ez
    if (c == 3) return {1, Y, X + 1};      // Hx
    if (c == 4) return {1, Y + 1, X};      // Hy
  } else {
    if (c == 0) return {1, Y + 1, X};  // Ex
    if (c == 1) return {1, Y, X + 1};  // Ey
    if (c == 5) return {1, Y, X};      // Hz
  }
  return {1, 1, 1};
}

__device__ __forceinline__ int64_t lin(const Dims& d, int k, int j, int i) {
  return (static_cast<int64_t>(k) * d.y + j) * static_cast<int64_t>(d.x) + i;
}

// Power-of-two scale of div_rn's residual (exact in both directions).
constexpr float kDivScale = 0x1p50f;
constexpr float kDivUnscale = 0x1p-50f;

// Correctly rounded a / b from bs = b 2^50 and rs = RN(1 / b) 2^-50: one
// residual FMA and one corrective FMA (Markstein, "IA-64 and Elementary
// Functions", 2000, thm 8.10), evaluated on a 2^50 a.  The theorem needs the
// residual a - q b exactly representable, which fails once it falls into the
// subnormal range (|a| below about 2^-103: the leading edge of a wavefront
// grown from zero fields); scaled by 2^50 it never does for |a| >= 2^-149.
// q = (2^50 a) rs is the same product as a RN(1/b), so for every other a the
// result equals the unscaled form.  Valid while a RN(1/b) is normal and
// |a| < 2^78 (fields in SI units on cells below 0.1 mm).
__device__ __forceinline__ float div_rn(float a, float bs, float rs) {
  const float as = a * kDivScale;
  const float q = as * rs;
  const float e = fmaf(-q, bs, as);
  return fmaf(e, rs, q);
}

// One packed CPML recurrence term as seen by a kernel.
struct CpmlTermDev {
  const float* a;
  const float* b;
  const float* k;
  const float* psi_in;
  float* psi_out;
  int low, high;
  int n_axis;   // target component extent along the derivative axis
  int pdy, pdx; // psi extents along y and x (psi z extent implied)
};

// Packed slab coordinate of `coord` along the term axis, or -1 outside.
__device__ __forceinline__ int cpml_slot(const CpmlTermDev& t, int coord) {
  if (coord < t.low) return coord;
  if (t.high > 0 && coord >= t.n_axis - t.high) return t.low + coord - (t.n_axis - t.high);
  return -1;
}

// Apply one recurrence in place (psi_out may alias psi_in) and return the
// corrected derivative d' = d / kappa + psi (beamz/simulation/kernels.py:257-264).
// `write` false evaluates without storing (halo recomputation).
template <int Axis>
__device__ __forceinline__ float cpml_correct(const CpmlTermDev& t, float d, int k, int j, int i,
                                              bool write) {
  const int coord = Axis == 0 ? k : (Axis == 1 ? j : i);
  const int slot = cpml_slot(t, coord);
  if (slot < 0) return d;
  const int pk = Axis == 0 ? slot : k;
  const int pj = Axis == 1 ? slot : j;
  const int pi = Axis == 2 ? slot : i;
  const int64_t off = (static_cast<int64_t>(pk) * t.pdy + pj) * static_cast<int64_t>(t.pdx) + pi;
  const float psi = t.b[slot] * t.psi_in[off] + t.a[slot] * d;
  if (write) t.psi_out[off] = psi;
  return d * t.k[slot] + psi;
}

// Device view of one slab source.
struct SourceDev {
  const float* coeff;
  const float* waveform;
  int wave_len;
  int component;
  int z0, y0, x0;
  int ez, ey, ex;
};

__device__ __forceinline__ float source_amplitude(const SourceDev& s, int step) {
  int w = step < 0 ? 0 : step;
  w = w >= s.wave_len ? s.wave_len - 1 : w;
  return s.waveform[w];
}

// PEC bit helpers: bit 2*axis = low wall, 2*axis+1 = high wall (axis 0=z,1=y,2=x).
__device__ __forceinline__ bool wall(int metallic, int axis, bool high) {
  return (metallic >> (2 * axis + (high ? 1 : 0))) & 1;
}

}  // namespace fdtd
