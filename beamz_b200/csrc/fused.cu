// One-kernel leapfrog step: H(t+1/2) and E(t+1) from bank A into bank B.
//
// Each CTA owns a TX x TY column of (y, x) lattice points and marches along z.
// For every plane k it stages E(k), E(k+1), H(k) and the voxel permittivities
// in shared memory, computes H(k+1/2) on the tile plus its low y/x halo
// (recomputing the neighbour's values so that E never waits for another
// CTA), then E(k) from H(k) in shared memory and H(k-1) kept in registers.
// Fields and the H-term CPML memories are double-banked (read A, write B), so
// halo recomputation never reads a value another CTA has already advanced;
// E-term CPML memories are only touched by their owning thread and stay in
// place.  Each field element is read once from DRAM and written once per step
// (halo re-reads are L2 hits), the 48 B + 1 B per cell of an FP32 Yee step.
//
// Arithmetic follows beamz/simulation/kernels.py:458-626 operation for
// operation (see fdtd_common.cuh for the rounding contract); PEC, CPML and
// H-timing sources follow beamz/simulation/execute.py:467-522.

#include "kernels.cuh"

namespace fdtd {

namespace {

template <int TX, int TY>
struct FusedSmem {
  static constexpr int EW = TX + 2, EH = TY + 2;  // E plane region [j0-1, j0+TY] x [i0-1, i0+TX]
  static constexpr int HW = TX + 1, HH = TY + 1;  // H region [j0-1, j0+TY) x [i0-1, i0+TX)
  float e[2][3][EH][EW];
  float ho[3][HH][HW];
  float hn[3][HH][HW];
  float eps[2][HH][HW];
  float table[256];
  float amp[kMaxFusedSources];
};

template <int TX, int TY, int Active>
__device__ __forceinline__ void load_e_plane(FusedSmem<TX, TY>& sm, const Step3D& p, int q, int j0, int i0,
                                             int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  const int slot = q & 1;
  for (int e = tid; e < S::EH * S::EW; e += NT) {
    const int ly = e / S::EW, lx = e - ly * S::EW;
    const int j = j0 - 1 + ly, i = i0 - 1 + lx;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float v = 0.0f;
      if ((Active >> c) & 1) {
        const Dims d = component_dims(c, p.Z, p.Y, p.X);
        if (q >= 0 && q < d.z && j >= 0 && j < d.y && i >= 0 && i < d.x) v = __ldg(p.ein[c] + lin(d, q, j, i));
      }
      sm.e[slot][c][ly][lx] = v;
    }
  }
}

template <int TX, int TY, int Active>
__device__ __forceinline__ void load_h_plane(FusedSmem<TX, TY>& sm, const Step3D& p, int q, int j0, int i0,
                                             int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  for (int e = tid; e < S::HH * S::HW; e += NT) {
    const int ly = e / S::HW, lx = e - ly * S::HW;
    const int j = j0 - 1 + ly, i = i0 - 1 + lx;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float v = 0.0f;
      if ((Active >> (c + 3)) & 1) {
        const Dims d = component_dims(c + 3, p.Z, p.Y, p.X);
        if (q < d.z && j >= 0 && j < d.y && i >= 0 && i < d.x) v = __ldg(p.hin[c] + lin(d, q, j, i));
      }
      sm.ho[c][ly][lx] = v;
    }
  }
}

template <int TX, int TY>
__device__ __forceinline__ void load_eps_plane(FusedSmem<TX, TY>& sm, const Step3D& p, int q, int j0, int i0,
                                               int tid) {
  using S = FusedSmem<TX, TY>;
  constexpr int NT = TX * TY;
  const int slot = q & 1;
  const int kq = clampi(q, p.Z - 1);
  for (int e = tid; e < S::HH * S::HW; e += NT) {
    const int ly = e / S::HW, lx = e - ly * S::HW;
    const int j = clampi(j0 - 1 + ly, p.Y - 1), i = clampi(i0 - 1 + lx, p.X - 1);
    sm.eps[slot][ly][lx] = sm.table[__ldg(p.em.voxels + (static_cast<int64_t>(kq) * p.Y + j) * p.X + i)];
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

template <int TX, int TY, int Active, bool Cpml, int Mat>
__global__ void __launch_bounds__(TX* TY) fused_step_kernel(Step3D p) {
  using S = FusedSmem<TX, TY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);
  constexpr int NT = TX * TY;
  const int tid = threadIdx.y * TX + threadIdx.x;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int kmax = Z + 1;  // planes holding any component
  const int k0 = blockIdx.z * p.z_chunk;
  const int k1 = min(k0 + p.z_chunk, kmax);
  const int kstart = k0 > 0 ? k0 - 1 : 0;

  if (Mat == FDTD_MATERIAL_VOXEL) {
    for (int e = tid; e < 256; e += NT) sm.table[e] = p.em.eps_table[e];
  }
  if (tid < p.n_hsrc) sm.amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);
  __syncthreads();

  load_e_plane<TX, TY, Active>(sm, p, kstart, j0, i0, tid);
  // Voxel plane clip(k0 - 1); plane clip(k) is staged at iteration k >= k0.
  if (Mat == FDTD_MATERIAL_VOXEL) load_eps_plane<TX, TY>(sm, p, k0 - 1, j0, i0, tid);

  // Own cell in H-region coordinates.
  const int oly = threadIdx.y + 1, olx = threadIdx.x + 1;
  const int oj = j0 + threadIdx.y, oi = i0 + threadIdx.x;
  float prev_hx = 0.0f, prev_hy = 0.0f;

  const Dims dEx = component_dims(0, Z, Y, X), dEy = component_dims(1, Z, Y, X), dEz = component_dims(2, Z, Y, X);
  const Dims dHx = component_dims(3, Z, Y, X), dHy = component_dims(4, Z, Y, X), dHz = component_dims(5, Z, Y, X);

  for (int k = kstart; k < k1; ++k) {
    const bool emit = k >= k0;
    load_e_plane<TX, TY, Active>(sm, p, k + 1, j0, i0, tid);
    load_h_plane<TX, TY, Active>(sm, p, k, j0, i0, tid);
    if (Mat == FDTD_MATERIAL_VOXEL && emit) load_eps_plane<TX, TY>(sm, p, k, j0, i0, tid);
    __syncthreads();

    const int s0 = k & 1, s1 = (k + 1) & 1;
    // ---- H(k) on the tile and its low halo -------------------------------
    for (int e = tid; e < S::HH * S::HW; e += NT) {
      const int ly = e / S::HW, lx = e - ly * S::HW;
      if (ly == 0 && lx == 0) continue;  // corner is never read
      const int j = j0 - 1 + ly, i = i0 - 1 + lx;
      const bool own = ly > 0 && lx > 0 && emit;
      float hx = 0.0f, hy = 0.0f, hz = 0.0f;
      if (((Active >> 3) & 1) && k < dHx.z && j >= 0 && j < dHx.y && i >= 0 && i < dHx.x) {
        float d0 = div_rn(sm.e[s0][2][ly + 1][lx] - sm.e[s0][2][ly][lx], p.res, p.inv_res);
        float d1 = div_rn(sm.e[s1][1][ly][lx] - sm.e[s0][1][ly][lx], p.res, p.inv_res);
        if (Cpml) {
          d0 = cpml_correct<1>(p.ht[0], d0, k, j, i, own);
          d1 = cpml_correct<0>(p.ht[1], d1, k, j, i, own);
        }
        const int64_t o = lin(dHx, k, j, i);
        hx = h_update(p.hm, 0, o, sm.ho[0][ly][lx], d0 - d1);
        hx = add_h_sources(p, sm.amp, 3, k, j, i, hx);
        if ((i == 0 && wall(p.metallic, 2, false)) || (i == dHx.x - 1 && wall(p.metallic, 2, true))) hx = 0.0f;
        if (own) p.hout[0][o] = hx;
      }
      if (((Active >> 4) & 1) && k < dHy.z && j >= 0 && j < dHy.y && i >= 0 && i < dHy.x) {
        float d0 = div_rn(sm.e[s1][0][ly][lx] - sm.e[s0][0][ly][lx], p.res, p.inv_res);
        float d1 = div_rn(sm.e[s0][2][ly][lx + 1] - sm.e[s0][2][ly][lx], p.res, p.inv_res);
        if (Cpml) {
          d0 = cpml_correct<0>(p.ht[2], d0, k, j, i, own);
          d1 = cpml_correct<2>(p.ht[3], d1, k, j, i, own);
        }
        const int64_t o = lin(dHy, k, j, i);
        hy = h_update(p.hm, 1, o, sm.ho[1][ly][lx], d0 - d1);
        hy = add_h_sources(p, sm.amp, 4, k, j, i, hy);
        if ((j == 0 && wall(p.metallic, 1, false)) || (j == dHy.y - 1 && wall(p.metallic, 1, true))) hy = 0.0f;
        if (own) p.hout[1][o] = hy;
      }
      if (((Active >> 5) & 1) && k < dHz.z && j >= 0 && j < dHz.y && i >= 0 && i < dHz.x) {
        float d0 = div_rn(sm.e[s0][1][ly][lx + 1] - sm.e[s0][1][ly][lx], p.res, p.inv_res);
        float d1 = div_rn(sm.e[s0][0][ly + 1][lx] - sm.e[s0][0][ly][lx], p.res, p.inv_res);
        if (Cpml) {
          d0 = cpml_correct<2>(p.ht[4], d0, k, j, i, own);
          d1 = cpml_correct<1>(p.ht[5], d1, k, j, i, own);
        }
        const int64_t o = lin(dHz, k, j, i);
        hz = h_update(p.hm, 2, o, sm.ho[2][ly][lx], d0 - d1);
        hz = add_h_sources(p, sm.amp, 5, k, j, i, hz);
        if ((k == 0 && wall(p.metallic, 0, false)) || (k == dHz.z - 1 && wall(p.metallic, 0, true))) hz = 0.0f;
        if (own) p.hout[2][o] = hz;
      }
      sm.hn[0][ly][lx] = hx;
      sm.hn[1][ly][lx] = hy;
      sm.hn[2][ly][lx] = hz;
    }
    __syncthreads();

    // ---- E(k) on the tile ---------------------------------------------------
    if (emit) {
      const int ly = oly, lx = olx, j = oj, i = oi;
      const float inv_res = p.inv_res, res = p.res;
      if (((Active >> 0) & 1) && k < dEx.z && j < dEx.y && i < dEx.x) {
        // dHz/dy with y ghosts, dHy/dz with z ghosts (register H(k-1)).
        float d0, d1;
        if (j == 0) d0 = wall(p.metallic, 1, false) ? div_rn(sm.hn[2][ly][lx] - 0.0f, res, inv_res) : 0.0f;
        else if (j == dHz.y) d0 = wall(p.metallic, 1, true) ? div_rn(0.0f - sm.hn[2][ly - 1][lx], res, inv_res) : 0.0f;
        else d0 = div_rn(sm.hn[2][ly][lx] - sm.hn[2][ly - 1][lx], res, inv_res);
        if (k == 0) d1 = wall(p.metallic, 0, false) ? div_rn(sm.hn[1][ly][lx] - 0.0f, res, inv_res) : 0.0f;
        else if (k == dHy.z) d1 = wall(p.metallic, 0, true) ? div_rn(0.0f - prev_hy, res, inv_res) : 0.0f;
        else d1 = div_rn(sm.hn[1][ly][lx] - prev_hy, res, inv_res);
        if (dHy.z == 0) d1 = 0.0f;
        if (Cpml) {
          d0 = cpml_correct<1>(p.et[0], d0, k, j, i, true);
          d1 = cpml_correct<0>(p.et[1], d1, k, j, i, true);
        }
        const int64_t o = lin(dEx, k, j, i);
        float e;
        if (Mat == FDTD_MATERIAL_VOXEL) {
          const float eps = 0.5f * (0.5f * (sm.eps[(k - 1) & 1][ly - 1][lx] + sm.eps[s0][ly - 1][lx]) +
                                    0.5f * (sm.eps[(k - 1) & 1][ly][lx] + sm.eps[s0][ly][lx]));
          e = sm.e[s0][0][ly][lx] + (p.dt_over_eps * __frcp_rn(eps)) * (d0 - d1);
        } else {
          e = e_update<Mat>(p, 0, o, k, j, i, sm.e[s0][0][ly][lx], d0 - d1);
        }
        if (e_constrained(p.metallic, 0, dEx, k, j, i)) e = 0.0f;
        p.eout[0][o] = e;
      }
      if (((Active >> 1) & 1) && k < dEy.z && j < dEy.y && i < dEy.x) {
        // dHx/dz with z ghosts, dHz/dx with x ghosts.
        float d0, d1;
        if (k == 0) d0 = wall(p.metallic, 0, false) ? div_rn(sm.hn[0][ly][lx] - 0.0f, res, inv_res) : 0.0f;
        else if (k == dHx.z) d0 = wall(p.metallic, 0, true) ? div_rn(0.0f - prev_hx, res, inv_res) : 0.0f;
        else d0 = div_rn(sm.hn[0][ly][lx] - prev_hx, res, inv_res);
        if (dHx.z == 0) d0 = 0.0f;
        if (i == 0) d1 = wall(p.metallic, 2, false) ? div_rn(sm.hn[2][ly][lx] - 0.0f, res, inv_res) : 0.0f;
        else if (i == dHz.x) d1 = wall(p.metallic, 2, true) ? div_rn(0.0f - sm.hn[2][ly][lx - 1], res, inv_res) : 0.0f;
        else d1 = div_rn(sm.hn[2][ly][lx] - sm.hn[2][ly][lx - 1], res, inv_res);
        if (Cpml) {
          d0 = cpml_correct<0>(p.et[2], d0, k, j, i, true);
          d1 = cpml_correct<2>(p.et[3], d1, k, j, i, true);
        }
        const int64_t o = lin(dEy, k, j, i);
        float e;
        if (Mat == FDTD_MATERIAL_VOXEL) {
          const float eps = 0.5f * (0.5f * (sm.eps[(k - 1) & 1][ly][lx - 1] + sm.eps[s0][ly][lx - 1]) +
                                    0.5f * (sm.eps[(k - 1) & 1][ly][lx] + sm.eps[s0][ly][lx]));
          e = sm.e[s0][1][ly][lx] + (p.dt_over_eps * __frcp_rn(eps)) * (d0 - d1);
        } else {
          e = e_update<Mat>(p, 1, o, k, j, i, sm.e[s0][1][ly][lx], d0 - d1);
        }
        if (e_constrained(p.metallic, 1, dEy, k, j, i)) e = 0.0f;
        p.eout[1][o] = e;
      }
      if (((Active >> 2) & 1) && k < dEz.z && j < dEz.y && i < dEz.x) {
        // dHy/dx with x ghosts, dHx/dy with y ghosts.
        float d0, d1;
        if (i == 0) d0 = wall(p.metallic, 2, false) ? div_rn(sm.hn[1][ly][lx] - 0.0f, res, inv_res) : 0.0f;
        else if (i == dHy.x) d0 = wall(p.metallic, 2, true) ? div_rn(0.0f - sm.hn[1][ly][lx - 1], res, inv_res) : 0.0f;
        else d0 = div_rn(sm.hn[1][ly][lx] - sm.hn[1][ly][lx - 1], res, inv_res);
        if (j == 0) d1 = wall(p.metallic, 1, false) ? div_rn(sm.hn[0][ly][lx] - 0.0f, res, inv_res) : 0.0f;
        else if (j == dHx.y) d1 = wall(p.metallic, 1, true) ? div_rn(0.0f - sm.hn[0][ly - 1][lx], res, inv_res) : 0.0f;
        else d1 = div_rn(sm.hn[0][ly][lx] - sm.hn[0][ly - 1][lx], res, inv_res);
        if (Cpml) {
          d0 = cpml_correct<2>(p.et[4], d0, k, j, i, true);
          d1 = cpml_correct<1>(p.et[5], d1, k, j, i, true);
        }
        const int64_t o = lin(dEz, k, j, i);
        float e;
        if (Mat == FDTD_MATERIAL_VOXEL) {
          const float eps = 0.5f * (0.5f * (sm.eps[s0][ly - 1][lx - 1] + sm.eps[s0][ly][lx - 1]) +
                                    0.5f * (sm.eps[s0][ly - 1][lx] + sm.eps[s0][ly][lx]));
          e = sm.e[s0][2][ly][lx] + (p.dt_over_eps * __frcp_rn(eps)) * (d0 - d1);
        } else {
          e = e_update<Mat>(p, 2, o, k, j, i, sm.e[s0][2][ly][lx], d0 - d1);
        }
        if (e_constrained(p.metallic, 2, dEz, k, j, i)) e = 0.0f;
        p.eout[2][o] = e;
      }
    }
    prev_hx = sm.hn[0][oly][olx];
    prev_hy = sm.hn[1][oly][olx];
    __syncthreads();
  }
}

template <int TX, int TY, int Active, bool Cpml, int Mat>
cudaError_t launch_fused_t(cudaStream_t s, const Step3D& p) {
  using S = FusedSmem<TX, TY>;
  const size_t smem = sizeof(S);
  auto kern = fused_step_kernel<TX, TY, Active, Cpml, Mat>;
  static bool configured = false;
  if (!configured) {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    configured = true;
  }
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
  if (tx == 32 && ty == 4) return launch_fused_t<32, 4, Active, Cpml, Mat>(s, p);
  if (tx == 32 && ty == 16) return launch_fused_t<32, 16, Active, Cpml, Mat>(s, p);
  if (tx == 64 && ty == 4) return launch_fused_t<64, 4, Active, Cpml, Mat>(s, p);
  if (tx == 64 && ty == 8) return launch_fused_t<64, 8, Active, Cpml, Mat>(s, p);
  return launch_fused_t<32, 8, Active, Cpml, Mat>(s, p);
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
  switch (active_mask) {
    case kActive3D: return launch_fused_a<kActive3D>(s, p, mat, tile_x, tile_y);
    case kActiveTM: return launch_fused_a<kActiveTM>(s, p, mat, tile_x, tile_y);
    case kActiveTE: return launch_fused_a<kActiveTE>(s, p, mat, tile_x, tile_y);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fdtd
