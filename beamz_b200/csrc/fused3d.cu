// One-kernel 3D leapfrog step, lean z-marching form: H(t+1/2) and E(t+1)
// from bank A into bank B.
//
// A CTA is NW warps; warp w owns R consecutive y rows of a 32-wide x strip,
// so the tile is 32 x (NW * R) lattice points, and the CTA marches along a
// chunk of z planes.  Per plane k:
//   1. wait for the cp.async group holding E(k+1) and H(k) (the ring runs D
//      planes ahead), then one CTA barrier;
//   2. issue the copies of E(k+1+D) and H(k+D) into the ring slots freed at k-1;
//   3. H(k): every thread its R own cells, warp 0 the y-halo row (Hx, Hz) and
//      warp 1 the x-halo column (Hy, Hz), recomputed so no CTA waits on
//      another; second CTA barrier;
//   4. E(k) on the own cells from H(k) and H(k-1) (double-buffered in shared
//      memory).
// Fields and the H-term CPML memories are double-banked (read A, write B);
// E-term memories are touched only by their owning thread and stay in place.
// A z chunk recomputes H of the plane below it (no writes) before its first E.
//
// Everything that does not change along z -- validity of each component at
// the thread's cells, wall flags, global offsets -- is computed once per CTA;
// CPML slot tests run only on tiles/planes that can touch an absorber slab and
// source tests only on planes a source box crosses.  Component arrays keep
// beamz's unpadded rows (pitches of X or X+1 floats are not 16 B multiples,
// which rules out TMA tensor copies), so planes are staged with 4-byte
// LDGSTS; element offsets are 32-bit (the host rejects larger arrays).
//
// Arithmetic follows beamz/simulation/kernels.py:458-626 operation for
// operation (rounding contract in fdtd_common.cuh); PEC, CPML and H-timing
// sources follow beamz/simulation/execute.py:467-522.

#include "kernels.cuh"

namespace fdtd {

namespace {

template <int NW, int R, int D>
struct Lean {
  static constexpr int TX = 32, TY = NW * R, NT = 32 * NW;
  static constexpr int EW = TX + 2, EH = TY + 2;  // E region [j0-1, j0+TY] x [i0-1, i0+TX]
  static constexpr int HW = TX + 1, HH = TY + 1;  // H region [j0-1, j0+TY) x [i0-1, i0+TX)
  static constexpr int ES = D + 2, HS = D + 1;
  struct Smem {
    float e[ES][3][EH][EW];
    float ho[HS][3][HH][HW];
    float hn[2][3][HH][HW];
    float eps[3][HH][HW];
    float table[256];
    float amp[kMaxFusedSources];
  };
};

__device__ __forceinline__ void ldgsts4(float* dst, const float* src, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void commit_group() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Per-component geometry as 32-bit element counts.
struct Geo {
  int dz, dy, dx, plane;
};
__device__ __forceinline__ Geo geo(int c, int Z, int Y, int X) {
  const Dims d = component_dims(c, Z, Y, X);
  return {d.z, d.y, d.x, d.y * d.x};
}

// Stage E plane q (rows j0-1 .. j0+TY, columns i0-1 .. i0+TX) into ring slot q % ES.
template <class L>
__device__ __forceinline__ void stage_e(typename L::Smem& sm, const Step3D& p, int q, int j0, int i0, int warp,
                                        int lane) {
  if (q > p.Z) return;
  const int slot = q % L::ES;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Geo g = geo(c, p.Z, p.Y, p.X);
    const float* base = p.ein[c];
    const bool zok = q < g.dz;
    const int i_a = i0 - 1 + lane, i_b = i0 + 31 + lane;
    const bool xa = i_a >= 0 && i_a < g.dx, xb = lane < 2 && i_b < g.dx;
    for (int ly = warp; ly < L::EH; ly += L::NT / 32) {
      const int j = j0 - 1 + ly;
      const bool ok = zok && j >= 0 && j < g.dy;
      const int row = q * g.plane + j * g.dx;
      ldgsts4(&sm.e[slot][c][ly][lane], base + (ok && xa ? row + i_a : 0), ok && xa);
      if (lane < 2) ldgsts4(&sm.e[slot][c][ly][lane + 32], base + (ok && xb ? row + i_b : 0), ok && xb);
    }
  }
}

// Stage H(old) plane q (rows j0-1 .. j0+TY-1, columns i0-1 .. i0+TX-1).
template <class L>
__device__ __forceinline__ void stage_h(typename L::Smem& sm, const Step3D& p, int q, int j0, int i0, int warp,
                                        int lane) {
  if (q > p.Z) return;
  const int slot = q % L::HS;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const Geo g = geo(c + 3, p.Z, p.Y, p.X);
    const float* base = p.hin[c];
    const bool zok = q < g.dz;
    const int i_a = i0 - 1 + lane, i_b = i0 + 31;
    const bool xa = i_a >= 0 && i_a < g.dx, xb = lane == 0 && i_b < g.dx;
    for (int ly = warp; ly < L::HH; ly += L::NT / 32) {
      const int j = j0 - 1 + ly;
      const bool ok = zok && j >= 0 && j < g.dy;
      const int row = q * g.plane + j * g.dx;
      ldgsts4(&sm.ho[slot][c][ly][lane], base + (ok && xa ? row + i_a : 0), ok && xa);
      if (lane == 0) ldgsts4(&sm.ho[slot][c][ly][32], base + (ok && xb ? row + i_b : 0), ok && xb);
    }
  }
}

// Voxel ids a thread stages per plane: its R own cells, plus the y-halo row
// (warp 0, with the corner on lane 0) or the x-halo column (warp 1).
template <int R>
struct VoxRegs {
  uint8_t own[R];
  uint8_t halo;
  uint8_t corner;
};

template <class L, int R>
__device__ __forceinline__ VoxRegs<R> fetch_vox(const Step3D& p, int q, int j0, int i0, int warp, int lane) {
  VoxRegs<R> v{};
  const int kq = clampi(q, p.Z - 1);
  const uint8_t* plane = p.em.voxels + static_cast<int64_t>(kq) * p.Y * p.X;
  const int i = clampi(i0 + lane, p.X - 1);
#pragma unroll
  for (int r = 0; r < R; ++r) v.own[r] = __ldg(plane + clampi(j0 + warp * R + r, p.Y - 1) * p.X + i);
  if (warp == 0) {
    v.halo = __ldg(plane + clampi(j0 - 1, p.Y - 1) * p.X + i);
    if (lane == 0) v.corner = __ldg(plane + clampi(j0 - 1, p.Y - 1) * p.X + clampi(i0 - 1, p.X - 1));
  } else if (warp == 1 && lane < L::TY) {
    v.halo = __ldg(plane + clampi(j0 + lane, p.Y - 1) * p.X + clampi(i0 - 1, p.X - 1));
  }
  return v;
}

template <class L, int R>
__device__ __forceinline__ void store_vox(typename L::Smem& sm, const VoxRegs<R>& v, int q, int warp, int lane) {
  const int s = (q + 3) % 3;
#pragma unroll
  for (int r = 0; r < R; ++r) sm.eps[s][1 + warp * R + r][1 + lane] = sm.table[v.own[r]];
  if (warp == 0) {
    sm.eps[s][0][1 + lane] = sm.table[v.halo];
    if (lane == 0) sm.eps[s][0][0] = sm.table[v.corner];
  } else if (warp == 1 && lane < L::TY) {
    sm.eps[s][1 + lane][0] = sm.table[v.halo];
  }
}

template <bool Metric>
__device__ __forceinline__ float ghost(const Step3D& p, float m, float center, float below, bool at_low,
                                       bool at_high, bool low_wall, bool high_wall) {
  // beamz/lattice.py:523-551: zero beyond a metallic wall, else a copy of the
  // edge sample so that the edge derivative vanishes.  `m`: the coordinate's
  // inverse distance (Metric).
  if (at_low) return low_wall ? dm<Metric>(p, center - 0.0f, m) : 0.0f;
  if (at_high) return high_wall ? dm<Metric>(p, 0.0f - below, m) : 0.0f;
  return dm<Metric>(p, center - below, m);
}

__device__ __forceinline__ float h_sources(const Step3D& p, const float* amp, int c, int k, int j, int i, float h) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    const int z = k - src.z0, y = j - src.y0, x = i - src.x0;
    if (src.component != c || z < 0 || y < 0 || x < 0 || z >= src.ez || y >= src.ey || x >= src.ex) continue;
    h = h + src.coeff[(static_cast<int64_t>(z) * src.ey + y) * src.ex + x] * amp[s];
  }
  return h;
}

// Does any h-timing source box cross plane k and columns/rows of this tile?
__device__ __forceinline__ bool sources_hit(const Step3D& p, int k, int jlo, int jhi, int ilo, int ihi) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    if (k >= src.z0 && k < src.z0 + src.ez && jhi >= src.y0 && jlo < src.y0 + src.ey && ihi >= src.x0 &&
        ilo < src.x0 + src.ex)
      return true;
  }
  return false;
}

template <int NW, int R, int D, bool Cpml, int Mat, bool Metric>
__global__ void __launch_bounds__(32 * NW) lean_step_kernel(Step3D p) {
  using L = Lean<NW, R, D>;
  using S = typename L::Smem;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);
  const int lane = threadIdx.x, warp = threadIdx.y;
  const int tid = warp * 32 + lane;
  const int i0 = blockIdx.x * L::TX, j0 = blockIdx.y * L::TY;
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int k0 = blockIdx.z * p.z_chunk;
  const int k1 = min(k0 + p.z_chunk, Z + 1);
  const int kstart = k0 > 0 ? k0 - 1 : 0;
  if (Mat == FDTD_MATERIAL_VOXEL)
    for (int e = tid; e < 256; e += L::NT) sm.table[e] = p.em.eps_table[e];
  if (tid < p.n_hsrc) sm.amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);

  stage_e<L>(sm, p, kstart, j0, i0, warp, lane);
#pragma unroll
  for (int m = 0; m < D; ++m) {
    stage_e<L>(sm, p, kstart + 1 + m, j0, i0, warp, lane);
    stage_h<L>(sm, p, kstart + m, j0, i0, warp, lane);
    commit_group();
  }
  VoxRegs<R> vox{};
  if (Mat == FDTD_MATERIAL_VOXEL) {
    __syncthreads();  // table
    store_vox<L, R>(sm, fetch_vox<L, R>(p, k0 - 1, j0, i0, warp, lane), k0 - 1, warp, lane);
    store_vox<L, R>(sm, fetch_vox<L, R>(p, k0, j0, i0, warp, lane), k0, warp, lane);
  }

  // ---- per-thread constants (independent of z) ------------------------------
  const Geo gEx = geo(0, Z, Y, X), gEy = geo(1, Z, Y, X), gEz = geo(2, Z, Y, X);
  const Geo gHx = geo(3, Z, Y, X), gHy = geo(4, Z, Y, X), gHz = geo(5, Z, Y, X);
  const bool wz0 = wall(p.metallic, 0, false), wz1 = wall(p.metallic, 0, true);
  const bool wy0 = wall(p.metallic, 1, false), wy1 = wall(p.metallic, 1, true);
  const bool wx0 = wall(p.metallic, 2, false), wx1 = wall(p.metallic, 2, true);
  const float dto = p.dt_over_eps;
  // Uniform H coefficients (VOXEL programs carry scalars).
  const bool h_uniform = !(p.hm.decay_full[0] | p.hm.decay_full[1] | p.hm.decay_full[2] | p.hm.source_full[0] |
                           p.hm.source_full[1] | p.hm.source_full[2]);
  const float hdec0 = p.hm.decay[0][0], hdec1 = p.hm.decay[1][0], hdec2 = p.hm.decay[2][0];
  const float hsrc0 = p.hm.source[0][0], hsrc1 = p.hm.source[1][0], hsrc2 = p.hm.source[2][0];
  const int i = i0 + lane;                       // own x
  const bool xX = i < X, xX1 = i <= X;           // x-extent X (Ex Hy Hz) / X+1 (Ey Ez Hx)
  const bool xlo = i == 0, xhi = i == X;         // ghost planes in x
  // CPML reach of this tile (x/y) -- planes test z separately.
  const bool cpml_xy = Cpml && !(i0 - 1 >= p.cpml_inner[2][0] && i0 + L::TX < p.cpml_inner[2][1] &&
                                 j0 - 1 >= p.cpml_inner[1][0] && j0 + L::TY < p.cpml_inner[1][1]);
  // Metric grids: the inverse distances of this thread's columns and rows,
  // loaded once (the plane's z values once per plane).
  float mhx = 0.0f, mhx_halo = 0.0f, mhy_halo = 0.0f, mhy_col = 0.0f, mex = 0.0f;
  float mhy[R], mey[R];
#pragma unroll
  for (int r = 0; r < R; ++r) mhy[r] = mey[r] = 0.0f;
  if constexpr (Metric) {
    mhx = p.metric_h[2][clampi(i, X - 1)];
    mhx_halo = p.metric_h[2][clampi(i0 - 1, X - 1)];
    mhy_halo = p.metric_h[1][clampi(j0 - 1, Y - 1)];
    mhy_col = p.metric_h[1][clampi(j0 + lane, Y - 1)];
    mex = p.metric_e[2][clampi(i, X)];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      mhy[r] = p.metric_h[1][clampi(j0 + warp * R + r, Y - 1)];
      mey[r] = p.metric_e[1][clampi(j0 + warp * R + r, Y)];
    }
  }

  for (int k = kstart; k < k1; ++k) {
    const bool emit = k >= k0;
    wait_group<D - 1>();
    __syncthreads();
    stage_e<L>(sm, p, k + 1 + D, j0, i0, warp, lane);
    stage_h<L>(sm, p, k + D, j0, i0, warp, lane);
    commit_group();
    if (Mat == FDTD_MATERIAL_VOXEL && emit) vox = fetch_vox<L, R>(p, k + 1, j0, i0, warp, lane);

    const int e0 = k % L::ES, e1 = (k + 1) % L::ES, hs = k % L::HS, hb = k & 1;
    const bool zZ = k < Z;  // Ez Hx Hy exist on this plane (Ex Ey Hz always do: k <= Z)
    const bool cpml = Cpml && (cpml_xy || !(k >= p.cpml_inner[0][0] && k < p.cpml_inner[0][1]));
    const bool src = p.n_hsrc > 0 && sources_hit(p, k, j0 - 1, j0 + L::TY, i0 - 1, i0 + L::TX);
    const float mhz = Metric ? p.metric_h[0][clampi(k, Z - 1)] : 0.0f;
    const float mez = Metric ? p.metric_e[0][clampi(k, Z)] : 0.0f;

    // ---- H(k) ----------------------------------------------------------------
    // One H cell at region position (ly, lx) = lattice (k, j, ii); `own` cells
    // are written back, halo cells only feed E.  Which components: bit 0 Hx,
    // 1 Hy, 2 Hz.
    auto h_cell = [&](int ly, int lx, int j, int ii, bool own, int which, float mx, float my) {
      const bool yY = j >= 0 && j < Y, yY1 = j >= 0 && j <= Y;
      const bool iX = ii >= 0 && ii < X, iX1 = ii >= 0 && ii <= X;
      const float ez = sm.e[e0][2][ly][lx], ey = sm.e[e0][1][ly][lx], ex = sm.e[e0][0][ly][lx];
      if (which & 1) {  // Hx: dEz/dy - dEy/dz
        const bool ok = zZ && yY && iX1;
        float d0 = dm<Metric>(p, sm.e[e0][2][ly + 1][lx] - ez, my);
        float d1 = dm<Metric>(p, sm.e[e1][1][ly][lx] - ey, mhz);
        if (cpml && ok) {
          d0 = cpml_correct<1>(p.ht[0], d0, k, j, ii, own);
          d1 = cpml_correct<0>(p.ht[1], d1, k, j, ii, own);
        }
        const int o = k * gHx.plane + j * gHx.dx + ii;
        float h = h_uniform ? hdec0 * sm.ho[hs][0][ly][lx] - hsrc0 * (d0 - d1)
                            : h_update(p.hm, 0, ok ? o : 0, sm.ho[hs][0][ly][lx], d0 - d1);
        if (src) h = h_sources(p, sm.amp, 3, k, j, ii, h);
        if ((ii == 0 && wx0) || (ii == X && wx1)) h = 0.0f;
        sm.hn[hb][0][ly][lx] = h;
        if (own && ok) p.hout[0][o] = h;
      }
      if (which & 2) {  // Hy: dEx/dz - dEz/dx
        const bool ok = zZ && yY1 && iX;
        float d0 = dm<Metric>(p, sm.e[e1][0][ly][lx] - ex, mhz);
        float d1 = dm<Metric>(p, sm.e[e0][2][ly][lx + 1] - ez, mx);
        if (cpml && ok) {
          d0 = cpml_correct<0>(p.ht[2], d0, k, j, ii, own);
          d1 = cpml_correct<2>(p.ht[3], d1, k, j, ii, own);
        }
        const int o = k * gHy.plane + j * gHy.dx + ii;
        float h = h_uniform ? hdec1 * sm.ho[hs][1][ly][lx] - hsrc1 * (d0 - d1)
                            : h_update(p.hm, 1, ok ? o : 0, sm.ho[hs][1][ly][lx], d0 - d1);
        if (src) h = h_sources(p, sm.amp, 4, k, j, ii, h);
        if ((j == 0 && wy0) || (j == Y && wy1)) h = 0.0f;
        sm.hn[hb][1][ly][lx] = h;
        if (own && ok) p.hout[1][o] = h;
      }
      if (which & 4) {  // Hz: dEy/dx - dEx/dy
        const bool ok = yY && iX;
        float d0 = dm<Metric>(p, sm.e[e0][1][ly][lx + 1] - ey, mx);
        float d1 = dm<Metric>(p, sm.e[e0][0][ly + 1][lx] - ex, my);
        if (cpml && ok) {
          d0 = cpml_correct<2>(p.ht[4], d0, k, j, ii, own);
          d1 = cpml_correct<1>(p.ht[5], d1, k, j, ii, own);
        }
        const int o = k * gHz.plane + j * gHz.dx + ii;
        float h = h_uniform ? hdec2 * sm.ho[hs][2][ly][lx] - hsrc2 * (d0 - d1)
                            : h_update(p.hm, 2, ok ? o : 0, sm.ho[hs][2][ly][lx], d0 - d1);
        if (src) h = h_sources(p, sm.amp, 5, k, j, ii, h);
        if ((k == 0 && wz0) || (k == Z && wz1)) h = 0.0f;
        sm.hn[hb][2][ly][lx] = h;
        if (own && ok) p.hout[2][o] = h;
      }
    };
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int ly = 1 + warp * R + r;
      h_cell(ly, 1 + lane, j0 + ly - 1, i, emit, 7, mhx, mhy[r]);
    }
    if (warp == 0) h_cell(0, 1 + lane, j0 - 1, i, false, 1 | 4, mhx, mhy_halo);  // y halo row: Hx, Hz
    if (warp == 1 && lane < L::TY)
      h_cell(1 + lane, 0, j0 + lane, i0 - 1, false, 2 | 4, mhx_halo, mhy_col);  // x halo column: Hy, Hz
    __syncthreads();

    // ---- E(k) ----------------------------------------------------------------
    if (emit) {
      const int pb = hb ^ 1;
      const int v0 = (k + 2) % 3, v1 = k % 3;  // voxel planes clip(k-1), clip(k)
      const bool zlo = k == 0, zhiZ = k == Z;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int ly = 1 + warp * R + r, lx = 1 + lane;
        const int j = j0 + ly - 1;
        const bool yY = j < Y, yY1 = j <= Y, ylo = j == 0, yhi = j == Y;
        const float hx = sm.hn[hb][0][ly][lx], hy = sm.hn[hb][1][ly][lx], hz = sm.hn[hb][2][ly][lx];
        // Ex: dHz/dy - dHy/dz
        if (yY1 && xX) {
          float d0 = ghost<Metric>(p, mey[r], hz, sm.hn[hb][2][ly - 1][lx], ylo, yhi, wy0, wy1);
          float d1 = ghost<Metric>(p, mez, hy, sm.hn[pb][1][ly][lx], zlo, zhiZ, wz0, wz1);
          if (cpml) {
            d0 = cpml_correct<1>(p.et[0], d0, k, j, i, true);
            d1 = cpml_correct<0>(p.et[1], d1, k, j, i, true);
          }
          const int o = k * gEx.plane + j * gEx.dx + i;
          float e;
          if (Mat == FDTD_MATERIAL_VOXEL) {
            const float eps = 0.5f * (0.5f * (sm.eps[v0][ly - 1][lx] + sm.eps[v1][ly - 1][lx]) +
                                      0.5f * (sm.eps[v0][ly][lx] + sm.eps[v1][ly][lx]));
            e = sm.e[e0][0][ly][lx] + (dto * __frcp_rn(eps)) * (d0 - d1);
          } else {
            e = e_update<Mat>(p, 0, o, k, j, i, sm.e[e0][0][ly][lx], d0 - d1);
          }
          if ((zlo && wz0) || (zhiZ && wz1) || (ylo && wy0) || (yhi && wy1)) e = 0.0f;
          p.eout[0][o] = e;
        }
        // Ey: dHx/dz - dHz/dx
        if (yY && xX1) {
          float d0 = ghost<Metric>(p, mez, hx, sm.hn[pb][0][ly][lx], zlo, zhiZ, wz0, wz1);
          float d1 = ghost<Metric>(p, mex, hz, sm.hn[hb][2][ly][lx - 1], xlo, xhi, wx0, wx1);
          if (cpml) {
            d0 = cpml_correct<0>(p.et[2], d0, k, j, i, true);
            d1 = cpml_correct<2>(p.et[3], d1, k, j, i, true);
          }
          const int o = k * gEy.plane + j * gEy.dx + i;
          float e;
          if (Mat == FDTD_MATERIAL_VOXEL) {
            const float eps = 0.5f * (0.5f * (sm.eps[v0][ly][lx - 1] + sm.eps[v1][ly][lx - 1]) +
                                      0.5f * (sm.eps[v0][ly][lx] + sm.eps[v1][ly][lx]));
            e = sm.e[e0][1][ly][lx] + (dto * __frcp_rn(eps)) * (d0 - d1);
          } else {
            e = e_update<Mat>(p, 1, o, k, j, i, sm.e[e0][1][ly][lx], d0 - d1);
          }
          if ((zlo && wz0) || (zhiZ && wz1) || (xlo && wx0) || (xhi && wx1)) e = 0.0f;
          p.eout[1][o] = e;
        }
        // Ez: dHy/dx - dHx/dy
        if (zZ && yY1 && xX1) {
          float d0 = ghost<Metric>(p, mex, hy, sm.hn[hb][1][ly][lx - 1], xlo, xhi, wx0, wx1);
          float d1 = ghost<Metric>(p, mey[r], hx, sm.hn[hb][0][ly - 1][lx], ylo, yhi, wy0, wy1);
          if (cpml) {
            d0 = cpml_correct<2>(p.et[4], d0, k, j, i, true);
            d1 = cpml_correct<1>(p.et[5], d1, k, j, i, true);
          }
          const int o = k * gEz.plane + j * gEz.dx + i;
          float e;
          if (Mat == FDTD_MATERIAL_VOXEL) {
            const float eps = 0.5f * (0.5f * (sm.eps[v1][ly - 1][lx - 1] + sm.eps[v1][ly][lx - 1]) +
                                      0.5f * (sm.eps[v1][ly - 1][lx] + sm.eps[v1][ly][lx]));
            e = sm.e[e0][2][ly][lx] + (dto * __frcp_rn(eps)) * (d0 - d1);
          } else {
            e = e_update<Mat>(p, 2, o, k, j, i, sm.e[e0][2][ly][lx], d0 - d1);
          }
          if ((ylo && wy0) || (yhi && wy1) || (xlo && wx0) || (xhi && wx1)) e = 0.0f;
          p.eout[2][o] = e;
        }
      }
      if (Mat == FDTD_MATERIAL_VOXEL) store_vox<L, R>(sm, vox, k + 1, warp, lane);
    }
  }
  wait_group<0>();
}

template <int NW, int R, int D, bool Cpml, int Mat, bool Metric = false>
cudaError_t launch_lean_t(cudaStream_t s, const Step3D& p) {
  using L = Lean<NW, R, D>;
  const size_t smem = sizeof(typename L::Smem);
  auto kern = lean_step_kernel<NW, R, D, Cpml, Mat, Metric>;
  // The dynamic shared-memory limit is a per-device function attribute: set it
  // on every launch (cheap) rather than once per process.
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  const int kmax = p.Z + 1;
  const int zc = p.z_chunk > 0 ? p.z_chunk : kmax;
  const dim3 grid((p.X + 1 + L::TX - 1) / L::TX, (p.Y + 1 + L::TY - 1) / L::TY, (kmax + zc - 1) / zc);
  Step3D q = p;
  q.z_chunk = zc;
  kern<<<grid, dim3(32, NW, 1), smem, s>>>(q);
  return cudaPeekAtLastError();
}

template <bool Cpml, int Mat>
cudaError_t launch_lean_shape(cudaStream_t s, const Step3D& p, int ty) {
  if (has_metric(p)) return launch_lean_t<8, 1, 1, Cpml, Mat, true>(s, p);  // metric grids: 32 x 8 tiles
  switch (ty) {
    case 8: return launch_lean_t<8, 1, 1, Cpml, Mat>(s, p);
    case 32: return launch_lean_t<8, 4, 1, Cpml, Mat>(s, p);
    case 4: return launch_lean_t<4, 1, 1, Cpml, Mat>(s, p);
    default: return launch_lean_t<8, 2, 1, Cpml, Mat>(s, p);  // 32 x 16
  }
}

}  // namespace

cudaError_t launch_fused_lean(cudaStream_t s, const Step3D& p, int mat, int tile_y) {
  if (p.cpml) return mat ? launch_lean_shape<true, 1>(s, p, tile_y) : launch_lean_shape<true, 0>(s, p, tile_y);
  return mat ? launch_lean_shape<false, 1>(s, p, tile_y) : launch_lean_shape<false, 0>(s, p, tile_y);
}

}  // namespace fdtd
