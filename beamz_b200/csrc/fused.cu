// One-kernel leapfrog step: H(t+1/2) and E(t+1) from bank A into bank B.
//
// Each CTA owns a TX x TY column of (y, x) lattice points and a chunk of z
// planes, and marches along z.  For plane k it computes H(k) on the tile plus
// its low y/x halo (recomputing the neighbour's values, so E never waits for
// another CTA), then E(k) from H(k) in shared memory and H(k-1) from the
// previous plane's buffer.  Fields and the H-term CPML memories are
// double-banked (read A, write B), so halo recomputation never reads a value
// another CTA has already advanced; E-term CPML memories are only touched by
// their owning thread and stay in place.  A chunk recomputes H of the plane
// below it (no writes) before its first E plane.
//
// Staging: E planes and H(old) planes arrive through a DEPTH-plane ring of
// cp.async copies (LDGSTS, 4 B: the component arrays keep beamz's unpadded
// rows, whose pitches X or X+1 floats are not 16 B multiples, which rules out
// TMA tensor copies); voxel ids come one plane ahead through registers.  Two
// CTA barriers per plane.  Each field element is read once from DRAM and
// written once per step (halo re-reads hit L2): 48 B + 1 B per cell.
//
// Arithmetic follows beamz/simulation/kernels.py:458-626 operation for
// operation (see fdtd_common.cuh for the rounding contract); PEC, CPML and
// H-timing sources follow beamz/simulation/execute.py:467-522.

#include "kernels.cuh"

namespace fdtd {

namespace {

constexpr int kDepth = 2;  // planes of E/H prefetched ahead of the plane being computed

template <int TX, int TY>
struct FusedSmem {
  static constexpr int EW = TX + 2, EH = TY + 2;  // E plane region [j0-1, j0+TY] x [i0-1, i0+TX]
  static constexpr int HW = TX + 1, HH = TY + 1;  // H region [j0-1, j0+TY) x [i0-1, i0+TX)
  static constexpr int ES = kDepth + 2;           // E ring slots
  static constexpr int HS = kDepth + 1;           // H(old) ring slots
  float e[ES][3][EH][EW];
  float ho[HS][3][HH][HW];
  float hn[2][3][HH][HW];
  float eps[3][HH][HW];
  float table[256];
  float amp[kMaxFusedSources];
  float eamp[kMaxFusedSources];
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? 4 : 0;  // src-size 0 zero-fills the destination
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Planes that hold any active component of the given range (E: 0-2, H:
// 3-5): the 2D TM embedding (Z = 1) keeps Ez, Hx and Hy on plane 0 only, so
// its plane 1 holds nothing to stage or update.
template <int Active>
__device__ __forceinline__ int active_planes(const Step3D& p, int first, int last) {
  int n = 0;
#pragma unroll
  for (int c = first; c <= last; ++c)
    if ((Active >> c) & 1) n = max(n, component_dims(c, p.Z, p.Y, p.X).z);
  return n;
}

// Issue the copies of E plane q (all three components) into its ring slot.
template <int TX, int TY, int Active>
__device__ __forceinline__ void issue_e_plane(FusedSmem<TX, TY>& sm, const Step3D& p, int q, int j0, int i0,
                                              int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  if (q >= active_planes<Active>(p, 0, 2)) return;  // beyond the last E plane: slot is never read
  const int slot = q % S::ES;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((Active >> c) & 1)) continue;
    const Dims d = component_dims(c, p.Z, p.Y, p.X);
    const float* base = p.ein[c];
    for (int e = tid; e < S::EH * S::EW; e += NT) {
      const int ly = e / S::EW, lx = e - ly * S::EW;
      const int j = j0 - 1 + ly, i = i0 - 1 + lx;
      const bool ok = q < d.z && j >= 0 && j < d.y && i >= 0 && i < d.x;
      cp_async4(&sm.e[slot][c][ly][lx], ok ? base + lin(d, q, j, i) : base, ok);
    }
  }
}

template <int TX, int TY, int Active>
__device__ __forceinline__ void issue_h_plane(FusedSmem<TX, TY>& sm, const Step3D& p, int q, int j0, int i0,
                                              int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  if (q >= active_planes<Active>(p, 3, 5)) return;
  const int slot = q % S::HS;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((Active >> (c + 3)) & 1)) continue;
    const Dims d = component_dims(c + 3, p.Z, p.Y, p.X);
    const float* base = p.hin[c];
    for (int e = tid; e < S::HH * S::HW; e += NT) {
      const int ly = e / S::HW, lx = e - ly * S::HW;
      const int j = j0 - 1 + ly, i = i0 - 1 + lx;
      const bool ok = q < d.z && j >= 0 && j < d.y && i >= 0 && i < d.x;
      cp_async4(&sm.ho[slot][c][ly][lx], ok ? base + lin(d, q, j, i) : base, ok);
    }
  }
}

// Voxel ids of plane clip(q) for this thread's (up to two) H-region cells.
template <int TX, int TY>
struct VoxelPrefetch {
  uint8_t v[2];
};

template <int TX, int TY>
__device__ __forceinline__ VoxelPrefetch<TX, TY> load_voxels(const Step3D& p, int q, int j0, int i0, int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  VoxelPrefetch<TX, TY> r{};
  const int kq = clampi(q, p.Z - 1);
#pragma unroll
  for (int n = 0; n < 2; ++n) {
    const int e = tid + n * NT;
    if (e < S::HH * S::HW) {
      const int ly = e / S::HW, lx = e - ly * S::HW;
      const int j = clampi(j0 - 1 + ly, p.Y - 1), i = clampi(i0 - 1 + lx, p.X - 1);
      r.v[n] = __ldg(p.em.voxels + (static_cast<int64_t>(kq) * p.Y + j) * p.X + i);
    }
  }
  return r;
}

template <int TX, int TY>
__device__ __forceinline__ void store_voxels(FusedSmem<TX, TY>& sm, const VoxelPrefetch<TX, TY>& r, int q, int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  const int slot = (q + 3) % 3;
#pragma unroll
  for (int n = 0; n < 2; ++n) {
    const int e = tid + n * NT;
    if (e < S::HH * S::HW) {
      const int ly = e / S::HW, lx = e - ly * S::HW;
      sm.eps[slot][ly][lx] = sm.table[r.v[n]];
    }
  }
}

// The pre-E source phase (beamz/simulation/execute.py:467-480) on the staged
// copy of E plane q: every pre-E source adds coeff * amplitude to the cells of
// its box, in source order, the halo included, so each CTA sees what the
// separate source kernel would have written into the bank (same rounding).
template <int TX, int TY, int Active>
__device__ __forceinline__ void add_pre_e_sources(FusedSmem<TX, TY>& sm, const Step3D& p, int q, int j0, int i0,
                                                  int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  const int slot = q % S::ES;
  for (int s = 0; s < p.n_esrc; ++s) {
    const SourceDev& src = p.esrc[s];
    const int c = src.component;
    if (c > 2 || !((Active >> c) & 1)) continue;
    const Dims d = component_dims(c, p.Z, p.Y, p.X);
    const int z = q - src.z0;
    if (z < 0 || z >= src.ez || q >= d.z) continue;
    for (int e = tid; e < S::EH * S::EW; e += NT) {  // a cell stays with one thread for every source
      const int ly = e / S::EW, lx = e - ly * S::EW;
      const int j = j0 - 1 + ly, i = i0 - 1 + lx;
      const int y = j - src.y0, x = i - src.x0;
      if (j < 0 || i < 0 || j >= d.y || i >= d.x || y < 0 || x < 0 || y >= src.ey || x >= src.ex) continue;
      float& v = sm.e[slot][c][ly][lx];
      v = v + src.coeff[(static_cast<int64_t>(z) * src.ey + y) * src.ex + x] * sm.eamp[s];
    }
  }
}

// Adds every h-timing source covering (k, j, i) of H component c (3..5).
__device__ __forceinline__ float add_h_sources(const Step3D& p, const float* amp, int c, int k, int j, int i,
                                               float h) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    if (src.component != c) continue;
    const int z = k - src.z0, y = j - src.y0, x = i - src.x0;
    if (z < 0 || y < 0 || x < 0 || z >= src.ez || y >= src.ey || x >= src.ex) continue;
    h = h + src.coeff[(static_cast<int64_t>(z) * src.ey + y) * src.ex + x] * amp[s];
  }
  return h;
}

// Backward difference at `coord` of an axis with n samples, with beamz's ghost
// planes (beamz/lattice.py:523-551): zero beyond a metallic wall, otherwise a
// copy of the edge sample, so the edge derivative vanishes.
template <bool Metric>
__device__ __forceinline__ float ghost_diff(const Step3D& p, int axis, float center, float below, int coord, int n,
                                            bool low_wall, bool high_wall) {
  if (n == 0) return 0.0f;
  if (coord == 0) return low_wall ? de<Metric>(p, axis, coord, center - 0.0f) : 0.0f;
  if (coord == n) return high_wall ? de<Metric>(p, axis, coord, 0.0f - below) : 0.0f;
  return de<Metric>(p, axis, coord, center - below);
}

// Staged E value; components outside the active set read as zero (2D).
template <int Active, typename S>
__device__ __forceinline__ float ev(const S& sm, int slot, int c, int ly, int lx) {
  return ((Active >> c) & 1) ? sm.e[slot][c][ly][lx] : 0.0f;
}

template <int TX, int TY, int Active, bool Cpml, int Mat, bool Metric>
__global__ void __launch_bounds__(TX* TY) fused_step_kernel(Step3D p) {
  using S = FusedSmem<TX, TY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);
  constexpr int NT = TX * TY;
  const int tid = threadIdx.y * TX + threadIdx.x;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int kmax = max(active_planes<Active>(p, 0, 2), active_planes<Active>(p, 3, 5));  // planes with an active component
  const int k0 = blockIdx.z * p.z_chunk;
  const int k1 = min(k0 + p.z_chunk, kmax);
  const int kstart = k0 > 0 ? k0 - 1 : 0;

  if (Mat == FDTD_MATERIAL_VOXEL) {
    for (int e = tid; e < 256; e += NT) sm.table[e] = p.em.eps_table[e];
  }
  if (tid < p.n_hsrc) sm.amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);
  if (tid < p.n_esrc) sm.eamp[tid] = source_amplitude(p.esrc[tid], p.step_counter[0] + p.step_offset);

  // Prologue: E(kstart) joins the first group; groups m = 0..kDepth-1 carry
  // E(kstart + 1 + m) and H(kstart + m).
  issue_e_plane<TX, TY, Active>(sm, p, kstart, j0, i0, tid);
#pragma unroll
  for (int m = 0; m < kDepth; ++m) {
    issue_e_plane<TX, TY, Active>(sm, p, kstart + 1 + m, j0, i0, tid);
    issue_h_plane<TX, TY, Active>(sm, p, kstart + m, j0, i0, tid);
    cp_async_commit();
  }
  // Voxel planes clip(k0 - 1) and clip(k0) for the first E plane; plane
  // clip(k + 1) is fetched into registers at plane k and stored after its E.
  VoxelPrefetch<TX, TY> vox{};
  if (Mat == FDTD_MATERIAL_VOXEL) {
    __syncthreads();  // eps table visible
    store_voxels<TX, TY>(sm, load_voxels<TX, TY>(p, k0 - 1, j0, i0, tid), k0 - 1, tid);
    store_voxels<TX, TY>(sm, load_voxels<TX, TY>(p, k0, j0, i0, tid), k0, tid);
  }

  const int oly = threadIdx.y + 1, olx = threadIdx.x + 1;
  const int oj = j0 + threadIdx.y, oi = i0 + threadIdx.x;
  const Dims dEx = component_dims(0, Z, Y, X), dEy = component_dims(1, Z, Y, X), dEz = component_dims(2, Z, Y, X);
  const Dims dHx = component_dims(3, Z, Y, X), dHy = component_dims(4, Z, Y, X), dHz = component_dims(5, Z, Y, X);
  const bool wz0 = wall(p.metallic, 0, false), wz1 = wall(p.metallic, 0, true);
  const bool wy0 = wall(p.metallic, 1, false), wy1 = wall(p.metallic, 1, true);
  const bool wx0 = wall(p.metallic, 2, false), wx1 = wall(p.metallic, 2, true);

  for (int k = kstart; k < k1; ++k) {
    const bool emit = k >= k0;
    cp_async_wait<kDepth - 1>();
    __syncthreads();
    // Refill the ring kDepth planes ahead (into slots last read at k - 1).
    issue_e_plane<TX, TY, Active>(sm, p, k + 1 + kDepth, j0, i0, tid);
    issue_h_plane<TX, TY, Active>(sm, p, k + kDepth, j0, i0, tid);
    cp_async_commit();
    if (p.n_esrc) {  // pre-E sources on the newly staged E plane(s), before any H reads them
      if (k == kstart) add_pre_e_sources<TX, TY, Active>(sm, p, k, j0, i0, tid);
      add_pre_e_sources<TX, TY, Active>(sm, p, k + 1, j0, i0, tid);
      __syncthreads();
    }
    if (Mat == FDTD_MATERIAL_VOXEL && emit) vox = load_voxels<TX, TY>(p, k + 1, j0, i0, tid);

    const int e0 = k % S::ES, e1 = (k + 1) % S::ES, hs = k % S::HS, hb = k & 1;
    // ---- H(k) on the tile and its low halo -------------------------------
    for (int e = tid; e < S::HH * S::HW; e += NT) {
      const int ly = e / S::HW, lx = e - ly * S::HW;
      if (ly == 0 && lx == 0) continue;  // corner is never read
      const int j = j0 - 1 + ly, i = i0 - 1 + lx;
      const bool own = ly > 0 && lx > 0 && emit;
      float hx = 0.0f, hy = 0.0f, hz = 0.0f;
      if (((Active >> 3) & 1) && k < dHx.z && j >= 0 && j < dHx.y && i >= 0 && i < dHx.x) {
        float d0 = dh<Metric>(p, 1, j, ev<Active>(sm, e0, 2, ly + 1, lx) - ev<Active>(sm, e0, 2, ly, lx));
        float d1 = dh<Metric>(p, 0, k, ev<Active>(sm, e1, 1, ly, lx) - ev<Active>(sm, e0, 1, ly, lx));
        if (Cpml) {
          d0 = cpml_correct<1>(p.ht[0], d0, k, j, i, own);
          d1 = cpml_correct<0>(p.ht[1], d1, k, j, i, own);
        }
        const int64_t o = lin(dHx, k, j, i);
        hx = h_update(p.hm, 0, o, sm.ho[hs][0][ly][lx], d0 - d1);
        if (p.n_hsrc) hx = add_h_sources(p, sm.amp, 3, k, j, i, hx);
        if ((i == 0 && wx0) || (i == dHx.x - 1 && wx1)) hx = 0.0f;
        if (own) p.hout[0][o] = hx;
      }
      if (((Active >> 4) & 1) && k < dHy.z && j >= 0 && j < dHy.y && i >= 0 && i < dHy.x) {
        float d0 = dh<Metric>(p, 0, k, ev<Active>(sm, e1, 0, ly, lx) - ev<Active>(sm, e0, 0, ly, lx));
        float d1 = dh<Metric>(p, 2, i, ev<Active>(sm, e0, 2, ly, lx + 1) - ev<Active>(sm, e0, 2, ly, lx));
        if (Cpml) {
          d0 = cpml_correct<0>(p.ht[2], d0, k, j, i, own);
          d1 = cpml_correct<2>(p.ht[3], d1, k, j, i, own);
        }
        const int64_t o = lin(dHy, k, j, i);
        hy = h_update(p.hm, 1, o, sm.ho[hs][1][ly][lx], d0 - d1);
        if (p.n_hsrc) hy = add_h_sources(p, sm.amp, 4, k, j, i, hy);
        if ((j == 0 && wy0) || (j == dHy.y - 1 && wy1)) hy = 0.0f;
        if (own) p.hout[1][o] = hy;
      }
      if (((Active >> 5) & 1) && k < dHz.z && j >= 0 && j < dHz.y && i >= 0 && i < dHz.x) {
        float d0 = dh<Metric>(p, 2, i, ev<Active>(sm, e0, 1, ly, lx + 1) - ev<Active>(sm, e0, 1, ly, lx));
        float d1 = dh<Metric>(p, 1, j, ev<Active>(sm, e0, 0, ly + 1, lx) - ev<Active>(sm, e0, 0, ly, lx));
        if (Cpml) {
          d0 = cpml_correct<2>(p.ht[4], d0, k, j, i, own);
          d1 = cpml_correct<1>(p.ht[5], d1, k, j, i, own);
        }
        const int64_t o = lin(dHz, k, j, i);
        hz = h_update(p.hm, 2, o, sm.ho[hs][2][ly][lx], d0 - d1);
        if (p.n_hsrc) hz = add_h_sources(p, sm.amp, 5, k, j, i, hz);
        if ((k == 0 && wz0) || (k == dHz.z - 1 && wz1)) hz = 0.0f;
        if (own) p.hout[2][o] = hz;
      }
      sm.hn[hb][0][ly][lx] = hx;
      sm.hn[hb][1][ly][lx] = hy;
      sm.hn[hb][2][ly][lx] = hz;
    }
    __syncthreads();

    // ---- E(k) on the tile ---------------------------------------------------
    if (emit) {
      const int ly = oly, lx = olx, j = oj, i = oi;
      const int pb = hb ^ 1;  // H(k-1), never read at k == 0 (ghost branch)
      const int v0 = (k + 2) % 3, v1 = k % 3;  // voxel planes clip(k-1), clip(k)
      if (((Active >> 0) & 1) && k < dEx.z && j < dEx.y && i < dEx.x) {
        float d0 = ghost_diff<Metric>(p, 1, sm.hn[hb][2][ly][lx], sm.hn[hb][2][ly - 1][lx], j, dHz.y, wy0, wy1);
        float d1 = ghost_diff<Metric>(p, 0, sm.hn[hb][1][ly][lx], sm.hn[pb][1][ly][lx], k, dHy.z, wz0, wz1);
        if (Cpml) {
          d0 = cpml_correct<1>(p.et[0], d0, k, j, i, true);
          d1 = cpml_correct<0>(p.et[1], d1, k, j, i, true);
        }
        const int64_t o = lin(dEx, k, j, i);
        float e;
        if (Mat == FDTD_MATERIAL_VOXEL) {
          const float eps = 0.5f * (0.5f * (sm.eps[v0][ly - 1][lx] + sm.eps[v1][ly - 1][lx]) +
                                    0.5f * (sm.eps[v0][ly][lx] + sm.eps[v1][ly][lx]));
          e = ev<Active>(sm, e0, 0, ly, lx) + (p.dt_over_eps * __frcp_rn(eps)) * (d0 - d1);
        } else {
          e = e_update<Mat>(p, 0, o, k, j, i, ev<Active>(sm, e0, 0, ly, lx), d0 - d1);
        }
        if (e_constrained(p.metallic, 0, dEx, k, j, i)) e = 0.0f;
        p.eout[0][o] = e;
      }
      if (((Active >> 1) & 1) && k < dEy.z && j < dEy.y && i < dEy.x) {
        float d0 = ghost_diff<Metric>(p, 0, sm.hn[hb][0][ly][lx], sm.hn[pb][0][ly][lx], k, dHx.z, wz0, wz1);
        float d1 = ghost_diff<Metric>(p, 2, sm.hn[hb][2][ly][lx], sm.hn[hb][2][ly][lx - 1], i, dHz.x, wx0, wx1);
        if (Cpml) {
          d0 = cpml_correct<0>(p.et[2], d0, k, j, i, true);
          d1 = cpml_correct<2>(p.et[3], d1, k, j, i, true);
        }
        const int64_t o = lin(dEy, k, j, i);
        float e;
        if (Mat == FDTD_MATERIAL_VOXEL) {
          const float eps = 0.5f * (0.5f * (sm.eps[v0][ly][lx - 1] + sm.eps[v1][ly][lx - 1]) +
                                    0.5f * (sm.eps[v0][ly][lx] + sm.eps[v1][ly][lx]));
          e = ev<Active>(sm, e0, 1, ly, lx) + (p.dt_over_eps * __frcp_rn(eps)) * (d0 - d1);
        } else {
          e = e_update<Mat>(p, 1, o, k, j, i, ev<Active>(sm, e0, 1, ly, lx), d0 - d1);
        }
        if (e_constrained(p.metallic, 1, dEy, k, j, i)) e = 0.0f;
        p.eout[1][o] = e;
      }
      if (((Active >> 2) & 1) && k < dEz.z && j < dEz.y && i < dEz.x) {
        float d0 = ghost_diff<Metric>(p, 2, sm.hn[hb][1][ly][lx], sm.hn[hb][1][ly][lx - 1], i, dHy.x, wx0, wx1);
        float d1 = ghost_diff<Metric>(p, 1, sm.hn[hb][0][ly][lx], sm.hn[hb][0][ly - 1][lx], j, dHx.y, wy0, wy1);
        if (Cpml) {
          d0 = cpml_correct<2>(p.et[4], d0, k, j, i, true);
          d1 = cpml_correct<1>(p.et[5], d1, k, j, i, true);
        }
        const int64_t o = lin(dEz, k, j, i);
        float e;
        if (Mat == FDTD_MATERIAL_VOXEL) {
          const float eps = 0.5f * (0.5f * (sm.eps[v1][ly - 1][lx - 1] + sm.eps[v1][ly][lx - 1]) +
                                    0.5f * (sm.eps[v1][ly - 1][lx] + sm.eps[v1][ly][lx]));
          e = ev<Active>(sm, e0, 2, ly, lx) + (p.dt_over_eps * __frcp_rn(eps)) * (d0 - d1);
        } else {
          e = e_update<Mat>(p, 2, o, k, j, i, ev<Active>(sm, e0, 2, ly, lx), d0 - d1);
        }
        if (e_constrained(p.metallic, 2, dEz, k, j, i)) e = 0.0f;
        p.eout[2][o] = e;
      }
      // Voxel plane clip(k + 1) for the next E plane; its slot was last read at k - 1.
      if (Mat == FDTD_MATERIAL_VOXEL) store_voxels<TX, TY>(sm, vox, k + 1, tid);
    }
  }
  cp_async_wait<0>();
}

template <int TX, int TY, int Active, bool Cpml, int Mat, bool Metric>
cudaError_t launch_fused_t(cudaStream_t s, const Step3D& p) {
  using S = FusedSmem<TX, TY>;
  const size_t smem = sizeof(S);
  auto kern = fused_step_kernel<TX, TY, Active, Cpml, Mat, Metric>;
  // The dynamic shared-memory limit is a per-device function attribute: set it
  // on every launch (cheap) rather than once per process.
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  const int kmax = p.Z + 1;
  const int zc = p.z_chunk > 0 ? p.z_chunk : kmax;
  const dim3 grid((p.X + 1 + TX - 1) / TX, (p.Y + 1 + TY - 1) / TY, (kmax + zc - 1) / zc);
  Step3D q = p;
  q.z_chunk = zc;
  kern<<<grid, dim3(TX, TY, 1), smem, s>>>(q);
  return cudaPeekAtLastError();
}

template <int Active, bool Cpml, int Mat>
cudaError_t launch_fused_tile(cudaStream_t s, const Step3D& p, int tx, int ty) {
  (void)tx;
  (void)ty;
  if (has_metric(p)) return launch_fused_t<32, 8, Active, Cpml, Mat, true>(s, p);
  return launch_fused_t<32, 8, Active, Cpml, Mat, false>(s, p);
}

template <int Active>
cudaError_t launch_fused_a(cudaStream_t s, const Step3D& p, int mat, int tx, int ty) {
  if (p.cpml) {
    return mat ? launch_fused_tile<Active, true, 1>(s, p, tx, ty) : launch_fused_tile<Active, true, 0>(s, p, tx, ty);
  }
  return mat ? launch_fused_tile<Active, false, 1>(s, p, tx, ty) : launch_fused_tile<Active, false, 0>(s, p, tx, ty);
}

}  // namespace

cudaError_t launch_fused(cudaStream_t s, const Step3D& p, int mat, int active_mask, int tile_x, int tile_y) {
  // 3D programs use the lean z-marching kernel (fused3d.cu); this one serves
  // the 2D polarizations.
  switch (active_mask) {
    case kActiveTM: return launch_fused_a<kActiveTM>(s, p, mat, tile_x, tile_y);
    case kActiveTE: return launch_fused_a<kActiveTE>(s, p, mat, tile_x, tile_y);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fdtd
