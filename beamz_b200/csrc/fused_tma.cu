// One-kernel 3D leapfrog step on the pitched field layout, staged by TMA.
//
// Pitched layout: every field component is a (Z+1, Y+1, P) float array with
// the same 16-byte-multiple row pitch P >= X+1 (the component's own extent is
// its corner (dz, dy, dx) block), and the voxel ids are a (Z, Y, Pv) byte
// array with Pv a multiple of 16.  One element offset (k*(Y+1) + j)*P + i
// then addresses a lattice point in all six components, and each plane of
// each component is a legal TMA box.
//
// A CTA of NW warps owns a 32 x (NW*R) tile of (y, x) lattice points and a
// chunk of z planes.  Per plane k:
//   1. wait on the mbarrier of bundle k = {E(k+1), H(k), voxels(k)} (one TMA
//      box per component), then one CTA barrier;
//   2. thread 0 issues bundle k+1 into the buffers plane k-1 released;
//   3. voxel ids of plane k become permittivities; H(k) on the own cells
//      (R per thread), the y-halo row (warp 0: Hx, Hz) and the x-halo column
//      (warp 1: Hy, Hz) -- recomputed, so no CTA waits on another; barrier;
//   4. E(k) on the own cells from H(k) and H(k-1) (double-buffered in shared
//      memory).  Cells on a domain face take the general branch (ghost
//      planes, clamped voxel sampling, PEC); all others the straight one.
// TMA zero-fills outside each component's extent, so halo and face reads
// need no predicates.  Fields and the H-term CPML memories are
// double-banked (read A, write B); E-term memories stay in place.  Every
// mbarrier wait is bounded: on expiry the kernel records an error word and
// returns.
//
// Arithmetic follows beamz/simulation/kernels.py:458-626 operation for
// operation (rounding contract in fdtd_common.cuh); PEC, CPML and H-timing
// sources follow beamz/simulation/execute.py:467-522.

#include <cuda.h>

#include "kernels.cuh"

namespace fdtd {

namespace {

// CPML coefficient slots staged in shared memory per term; wider slabs (tiny
// grids whose absorbers meet) read their coefficients from global memory.
constexpr int kCoefSlots = 32;
// Absorber cells off the domain faces take a dedicated branch with psi fetched
// ahead of use when this is set.
constexpr bool kCpmlAhead = false;

template <int NW, int R>
struct TmaTile {
  static constexpr int TX = 32, TY = NW * R, NT = 32 * NW;
  static constexpr int BX = TX + 8;            // staged row: x from i0-4 to i0+TX+3
  static constexpr int EH = TY + 2;            // E rows j0-1 .. j0+TY
  static constexpr int HH = TY + 1;            // H rows j0-1 .. j0+TY-1
  static constexpr int VX = TX + 16;           // voxel row bytes: x from i0-16
  static constexpr int HW = TX + 1;            // H/eps region columns i0-1 .. i0+TX-1
  static constexpr int EBOX = ((EH * BX + 31) / 32) * 32;  // floats, 128 B multiples
  static constexpr int HBOX = ((HH * BX + 31) / 32) * 32;
  static constexpr int VBOX = ((HH * VX + 127) / 128) * 128;  // bytes
  struct Smem {
    float e[3 * 3][EBOX];  // E ring: 3 planes x 3 components
    float h[2 * 3][HBOX];  // H(old) ring: 2 planes x 3 components
    uint8_t v[2][VBOX];    // voxel ring: 2 planes
    float hn[2][3][HH][HW];
    float eps[3][HH][HW];
    float table[256];
    float amp[kMaxFusedSources];
    float4 coef[12][kCoefSlots];  // CPML (a, b, 1/kappa) per term (H 0-5, E 6-11) and slot
    unsigned long long bar[2];
  };
};

struct TmaMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
  CUtensorMap vox;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_expect(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool bar_try(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait: gives up after 200 ms of device time, far beyond any plane's
// copy latency, so a broken copy ends the kernel instead of hanging the GPU.
__device__ __forceinline__ bool bar_wait(unsigned long long* b, unsigned parity) {
  if (bar_try(b, parity)) return true;
  const unsigned long long start = global_ns();
  for (;;) {
    for (int n = 0; n < 64; ++n)
      if (bar_try(b, parity)) return true;
    if (global_ns() - start > 200000000ull) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(b))
      : "memory");
}

// Issue bundle q: E(q+1) (and E(q) when `first`), H(q), voxels(clip(q)).
template <class T>
__device__ __forceinline__ void issue_bundle(typename T::Smem& sm, const TmaMaps& maps, int q, int Z, int j0, int i0,
                                             int slot, bool first) {
  unsigned bytes = 0;
  const int ne = (first ? 1 : 0) + (q + 1 <= Z ? 1 : 0);
  bytes += ne * 3 * T::EH * T::BX * 4;
  bytes += 3 * T::HH * T::BX * 4;
  bytes += T::HH * T::VX;
  unsigned long long* b = &sm.bar[slot];
  bar_expect(b, bytes);
  if (first) {
    for (int c = 0; c < 3; ++c) tma_load_3d(sm.e[(q % 3) * 3 + c], &maps.e[c], i0 - 4, j0 - 1, q, b);
  }
  if (q + 1 <= Z) {
    for (int c = 0; c < 3; ++c) tma_load_3d(sm.e[((q + 1) % 3) * 3 + c], &maps.e[c], i0 - 4, j0 - 1, q + 1, b);
  }
  for (int c = 0; c < 3; ++c) tma_load_3d(sm.h[(q % 2) * 3 + c], &maps.h[c], i0 - 4, j0 - 1, q, b);
  const int kv = q < 0 ? 0 : (q > Z - 1 ? Z - 1 : q);
  tma_load_3d(sm.v[q % 2], &maps.vox, i0 - 16, j0 - 1, kv, b);
}

__device__ __forceinline__ float ghost(float center, float below, bool at_low, bool at_high, bool low_wall,
                                       bool high_wall, float res, float inv_res) {
  // beamz/lattice.py:523-551: zero beyond a metallic wall, else a copy of the
  // edge sample so that the edge derivative vanishes.
  if (at_low) return low_wall ? div_rn(center - 0.0f, res, inv_res) : 0.0f;
  if (at_high) return high_wall ? div_rn(0.0f - below, res, inv_res) : 0.0f;
  return div_rn(center - below, res, inv_res);
}

// A CPML recurrence split in two so that the operand loads of every term of a
// cell are in flight together: fetch (slot, psi, a, b, 1/kappa), then apply.
struct CpmlOp {
  int slot = -1;
  int64_t off = 0;
  float psi = 0.0f, a = 0.0f, b = 0.0f, k = 1.0f;
};

template <int Axis>
__device__ __forceinline__ CpmlOp cpml_fetch(const CpmlTermDev& t, int k, int j, int i) {
  CpmlOp op;
  const int coord = Axis == 0 ? k : (Axis == 1 ? j : i);
  op.slot = cpml_slot(t, coord);
  if (op.slot >= 0) {
    const int pk = Axis == 0 ? op.slot : k;
    const int pj = Axis == 1 ? op.slot : j;
    const int pi = Axis == 2 ? op.slot : i;
    op.off = (static_cast<int64_t>(pk) * t.pdy + pj) * static_cast<int64_t>(t.pdx) + pi;
    op.psi = t.psi_in[op.off];
    op.a = __ldg(t.a + op.slot);
    op.b = __ldg(t.b + op.slot);
    op.k = __ldg(t.k + op.slot);
  }
  return op;
}

// psi <- b psi + a d; returns d / kappa + psi (beamz/simulation/kernels.py:257-264).
__device__ __forceinline__ float cpml_apply(const CpmlTermDev& t, const CpmlOp& op, float d, bool write) {
  if (op.slot < 0) return d;
  const float psi = op.b * op.psi + op.a * d;
  if (write) t.psi_out[op.off] = psi;
  return d * op.k + psi;
}

template <int Axis>
__device__ __forceinline__ int64_t psi_offset(const CpmlTermDev& t, int slot, int k, int j, int i) {
  const int pk = Axis == 0 ? slot : k, pj = Axis == 1 ? slot : j, pi = Axis == 2 ? slot : i;
  return (static_cast<int64_t>(pk) * t.pdy + pj) * static_cast<int64_t>(t.pdx) + pi;
}

// Corrected derivative with the psi value already in hand (coefficients from
// shared memory when the slab fits): psi <- b psi + a d, d' = d / kappa + psi.
__device__ __forceinline__ float cpml_use(const CpmlTermDev& t, const float4* coef, bool coef_smem, int slot,
                                          float psi_old, float d, float* psi_out, int64_t off) {
  if (slot < 0) return d;
  float a, b, kk;
  if (coef_smem) {
    const float4 c = coef[slot];
    a = c.x;
    b = c.y;
    kk = c.z;
  } else {
    a = __ldg(t.a + slot);
    b = __ldg(t.b + slot);
    kk = __ldg(t.k + slot);
  }
  const float psi = b * psi_old + a * d;
  psi_out[off] = psi;
  return d * kk + psi;
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

__device__ __forceinline__ bool sources_hit(const Step3D& p, int k, int jlo, int jhi, int ilo, int ihi) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    if (k >= src.z0 && k < src.z0 + src.ez && jhi >= src.y0 && jlo < src.y0 + src.ey && ihi >= src.x0 &&
        ilo < src.x0 + src.ex)
      return true;
  }
  return false;
}

template <int NW, int R, bool Cpml>
__global__ void __launch_bounds__(32 * NW, 1024 / (32 * NW)) tma_step_kernel(const __grid_constant__ TmaMaps maps, Step3D p) {
  using T = TmaTile<NW, R>;
  using S = typename T::Smem;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);
  const int lane = threadIdx.x, warp = threadIdx.y;
  const int tid = warp * 32 + lane;
  const int i0 = blockIdx.x * T::TX, j0 = blockIdx.y * T::TY;
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int k0 = blockIdx.z * p.z_chunk;
  const int k1 = min(k0 + p.z_chunk, Z + 1);
  const int kstart = k0 > 0 ? k0 - 1 : 0;
  const float res = p.res, inv_res = p.inv_res, dto = p.dt_over_eps;
  const int P = p.pitch, PL = (Y + 1) * p.pitch;

  if (tid == 0) {
    bar_init(&sm.bar[0], 1);
    bar_init(&sm.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int e = tid; e < 256; e += T::NT) sm.table[e] = p.em.eps_table[e];
  bool coef_smem = true;
  if (Cpml) {
#pragma unroll
    for (int t = 0; t < 12; ++t) {
      const CpmlTermDev& d = t < 6 ? p.ht[t] : p.et[t - 6];
      const int w = d.low + d.high;
      coef_smem = coef_smem && w <= kCoefSlots;
      for (int e = tid; e < w && e < kCoefSlots; e += T::NT)
        sm.coef[t][e] = make_float4(d.a[e], d.b[e], d.k[e], 0.0f);
    }
  }
  if (tid < p.n_hsrc) sm.amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);
  __syncthreads();
  // Bundle kstart now; bundle k+1 is issued at plane k (a three-plane E ring
  // and two-plane H/voxel rings hold planes k, k+1 and the one in flight).
  if (tid == 0) issue_bundle<T>(sm, maps, kstart, Z, j0, i0, 0, true);

  // ---- per-thread constants --------------------------------------------------
  const bool wz0 = wall(p.metallic, 0, false), wz1 = wall(p.metallic, 0, true);
  const bool wy0 = wall(p.metallic, 1, false), wy1 = wall(p.metallic, 1, true);
  const bool wx0 = wall(p.metallic, 2, false), wx1 = wall(p.metallic, 2, true);
  // The pitched layout carries uniform H coefficients (validated on the host).
  const float hdec0 = p.hm.decay[0][0], hdec1 = p.hm.decay[1][0], hdec2 = p.hm.decay[2][0];
  const float hsrc0 = p.hm.source[0][0], hsrc1 = p.hm.source[1][0], hsrc2 = p.hm.source[2][0];
  const int i = i0 + lane;
  const int zin0 = Cpml ? max(1, p.cpml_inner[0][0]) : 1, zin1 = Cpml ? min(Z, p.cpml_inner[0][1]) : Z;
  const int yin0 = Cpml ? max(1, p.cpml_inner[1][0]) : 1, yin1 = Cpml ? min(Y, p.cpml_inner[1][1]) : Y;
  const int xin0 = Cpml ? max(1, p.cpml_inner[2][0]) : 1, xin1 = Cpml ? min(X, p.cpml_inner[2][1]) : X;
  // Own cells away from every face and absorber take the straight-line path.
  const bool col_fast = i >= xin0 && i < xin1;
  bool row_fast[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + warp * R + r;
    row_fast[r] = j >= yin0 && j < yin1;
  }
  const bool cpml_xy = Cpml && !(i0 - 1 >= p.cpml_inner[2][0] && i0 + T::TX < p.cpml_inner[2][1] &&
                                 j0 - 1 >= p.cpml_inner[1][0] && j0 + T::TY < p.cpml_inner[1][1]);
  // Own cells off every domain face (ghost-, PEC- and validity-free).
  const bool col_face_free = i >= 1 && i < X;
  bool row_face_free[R];
  int syh[R], sye[R];  // y slots: H terms (Hxy, Hzy; extent Y), E terms (Exy, Ezy; extent Y+1)
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + warp * R + r;
    row_face_free[r] = j >= 1 && j < Y;
    syh[r] = Cpml ? cpml_slot(p.ht[0], j) : -1;
    sye[r] = Cpml ? cpml_slot(p.et[0], j) : -1;
  }
  const int sxh = Cpml ? cpml_slot(p.ht[3], i) : -1;  // x slots: Hyx, Hzx (extent X)
  const int sxe = Cpml ? cpml_slot(p.et[3], i) : -1;  //          Eyx, Ezx (extent X+1)
  // psi of the H terms for the own cells of the next plane, fetched a plane ahead.
  float nph[R][6];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int t = 0; t < 6; ++t) nph[r][t] = 0.0f;
  auto fetch_h_psi = [&](int q, float (&dst)[R][6]) {
    const int szh = cpml_slot(p.ht[1], q);  // Hxz, Hyz (extent Z)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + warp * R + r;
      if (!(col_face_free && row_face_free[r] && q >= 1 && q < Z)) continue;
      if (syh[r] >= 0) {
        dst[r][0] = p.ht[0].psi_in[psi_offset<1>(p.ht[0], syh[r], q, j, i)];
        dst[r][5] = p.ht[5].psi_in[psi_offset<1>(p.ht[5], syh[r], q, j, i)];
      }
      if (szh >= 0) {
        dst[r][1] = p.ht[1].psi_in[psi_offset<0>(p.ht[1], szh, q, j, i)];
        dst[r][2] = p.ht[2].psi_in[psi_offset<0>(p.ht[2], szh, q, j, i)];
      }
      if (sxh >= 0) {
        dst[r][3] = p.ht[3].psi_in[psi_offset<2>(p.ht[3], sxh, q, j, i)];
        dst[r][4] = p.ht[4].psi_in[psi_offset<2>(p.ht[4], sxh, q, j, i)];
      }
    }
  };
  if (Cpml && kCpmlAhead && k0 < k1) fetch_h_psi(kstart, nph);

  for (int k = kstart; k < k1; ++k) {
    const int n = k - kstart;
    const bool emit = k >= k0;
    const bool arrived = bar_wait(&sm.bar[n & 1], (n >> 1) & 1);
    if (__syncthreads_or(!arrived)) {  // CTA-uniform: every thread leaves together
      if (tid == 0 && p.status) atomicExch(p.status, 1);
      return;
    }
    if (tid == 0 && k + 1 < k1) {
      // Plane k-1's generic reads of these buffers precede the TMA writes.
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue_bundle<T>(sm, maps, k + 1, Z, j0, i0, (n + 1) & 1, false);
    }

    const float* E0x = sm.e[(k % 3) * 3 + 0];
    const float* E0y = sm.e[(k % 3) * 3 + 1];
    const float* E0z = sm.e[(k % 3) * 3 + 2];
    const float* E1x = sm.e[((k + 1) % 3) * 3 + 0];
    const float* E1y = sm.e[((k + 1) % 3) * 3 + 1];
    const float* HOx = sm.h[(k % 2) * 3 + 0];
    const float* HOy = sm.h[(k % 2) * 3 + 1];
    const float* HOz = sm.h[(k % 2) * 3 + 2];
    const int hb = k & 1;
    const bool zZ = k < Z;
    const bool cpml = Cpml && (cpml_xy || !(k >= p.cpml_inner[0][0] && k < p.cpml_inner[0][1]));
    const bool src = p.n_hsrc > 0 && sources_hit(p, k, j0 - 1, j0 + T::TY, i0 - 1, i0 + T::TX);
    const bool plane_fast = k >= zin0 && k < zin1 && !src;
    const bool plane_face_free = k >= 1 && k < Z && !src;
    const int szh = Cpml ? cpml_slot(p.ht[1], k) : -1, sze = Cpml ? cpml_slot(p.et[1], k) : -1;
    float ph[R][6], pe[R][6];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        ph[r][t] = nph[r][t];
        pe[r][t] = 0.0f;
      }
    if (Cpml && kCpmlAhead && cpml && emit) {
      // psi of the E terms at this plane: in flight while H is computed.
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + warp * R + r;
        if (!(plane_face_free && row_face_free[r] && col_face_free)) continue;
        if (sye[r] >= 0) {
          pe[r][0] = p.et[0].psi_in[psi_offset<1>(p.et[0], sye[r], k, j, i)];
          pe[r][5] = p.et[5].psi_in[psi_offset<1>(p.et[5], sye[r], k, j, i)];
        }
        if (sze >= 0) {
          pe[r][1] = p.et[1].psi_in[psi_offset<0>(p.et[1], sze, k, j, i)];
          pe[r][2] = p.et[2].psi_in[psi_offset<0>(p.et[2], sze, k, j, i)];
        }
        if (sxe >= 0) {
          pe[r][3] = p.et[3].psi_in[psi_offset<2>(p.et[3], sxe, k, j, i)];
          pe[r][4] = p.et[4].psi_in[psi_offset<2>(p.et[4], sxe, k, j, i)];
        }
      }
    }
    if (Cpml && kCpmlAhead && k + 1 < k1) fetch_h_psi(k + 1, nph);

    // Voxel ids -> permittivity for plane clip(k) (and clip(k-1) == clip(k) at k = 0).
    {
      const uint8_t* vb = sm.v[k % 2];
      for (int e = tid; e < T::HH * T::HW; e += T::NT) {
        const int ly = e / T::HW, lx = e - ly * T::HW;
        const float v = sm.table[vb[ly * T::VX + lx + 15]];
        sm.eps[k % 3][ly][lx] = v;
        if (k == 0) sm.eps[2][ly][lx] = v;
      }
    }

    // ---- H(k), general form: region (ly, lx) = lattice (k, j0-1+ly, i0-1+lx),
    // box column bx = lx + 3.  `which`: bit 0 Hx, 1 Hy, 2 Hz.
    auto h_general = [&](int ly, int lx, bool own, int which) {
      const int j = j0 - 1 + ly, ii = i0 - 1 + lx, bx = lx + 3, b = ly * T::BX + bx;
      const int o = k * PL + j * P + ii;
      const bool yY = j >= 0 && j < Y, yY1 = j >= 0 && j <= Y;
      const bool iX = ii >= 0 && ii < X, iX1 = ii >= 0 && ii <= X;
      const bool okx = (which & 1) && zZ && yY && iX1;
      const bool oky = (which & 2) && zZ && yY1 && iX;
      const bool okz = (which & 4) && yY && iX;
      // Each component fetches both of its CPML operands before using either.
      const float ez = E0z[b], ey = E0y[b], ex = E0x[b];
      if (which & 1) {  // Hx: dEz/dy - dEy/dz
        CpmlOp cx0, cx1;
        if (cpml && okx) { cx0 = cpml_fetch<1>(p.ht[0], k, j, ii); cx1 = cpml_fetch<0>(p.ht[1], k, j, ii); }
        float d0 = div_rn(E0z[b + T::BX] - ez, res, inv_res);
        float d1 = div_rn(E1y[b] - ey, res, inv_res);
        if (cpml && okx) {
          d0 = cpml_apply(p.ht[0], cx0, d0, own);
          d1 = cpml_apply(p.ht[1], cx1, d1, own);
        }
        float h = hdec0 * HOx[b] - hsrc0 * (d0 - d1);
        if (src) h = h_sources(p, sm.amp, 3, k, j, ii, h);
        if ((ii == 0 && wx0) || (ii == X && wx1)) h = 0.0f;
        sm.hn[hb][0][ly][lx] = h;
        if (own && okx) p.hout[0][o] = h;
      }
      if (which & 2) {  // Hy: dEx/dz - dEz/dx
        CpmlOp cy0, cy1;
        if (cpml && oky) { cy0 = cpml_fetch<0>(p.ht[2], k, j, ii); cy1 = cpml_fetch<2>(p.ht[3], k, j, ii); }
        float d0 = div_rn(E1x[b] - ex, res, inv_res);
        float d1 = div_rn(E0z[b + 1] - ez, res, inv_res);
        if (cpml && oky) {
          d0 = cpml_apply(p.ht[2], cy0, d0, own);
          d1 = cpml_apply(p.ht[3], cy1, d1, own);
        }
        float h = hdec1 * HOy[b] - hsrc1 * (d0 - d1);
        if (src) h = h_sources(p, sm.amp, 4, k, j, ii, h);
        if ((j == 0 && wy0) || (j == Y && wy1)) h = 0.0f;
        sm.hn[hb][1][ly][lx] = h;
        if (own && oky) p.hout[1][o] = h;
      }
      if (which & 4) {  // Hz: dEy/dx - dEx/dy
        CpmlOp cz0, cz1;
        if (cpml && okz) { cz0 = cpml_fetch<2>(p.ht[4], k, j, ii); cz1 = cpml_fetch<1>(p.ht[5], k, j, ii); }
        float d0 = div_rn(E0y[b + 1] - ey, res, inv_res);
        float d1 = div_rn(E0x[b + T::BX] - ex, res, inv_res);
        if (cpml && okz) {
          d0 = cpml_apply(p.ht[4], cz0, d0, own);
          d1 = cpml_apply(p.ht[5], cz1, d1, own);
        }
        float h = hdec2 * HOz[b] - hsrc2 * (d0 - d1);
        if (src) h = h_sources(p, sm.amp, 5, k, j, ii, h);
        if ((k == 0 && wz0) || (k == Z && wz1)) h = 0.0f;
        sm.hn[hb][2][ly][lx] = h;
        if (own && okz) p.hout[2][o] = h;
      }
    };
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int ly = 1 + warp * R + r, lx = 1 + lane;
      if (plane_fast && row_fast[r] && col_fast) {
        // Interior, absorber-free, source-free: every H component exists here.
        const int b = ly * T::BX + lane + 4;
        const int o = k * PL + (j0 + ly - 1) * P + i;
        const float ez = E0z[b], ey = E0y[b], ex = E0x[b];
        const float hx = hdec0 * HOx[b] - hsrc0 * (div_rn(E0z[b + T::BX] - ez, res, inv_res) -
                                                   div_rn(E1y[b] - ey, res, inv_res));
        const float hy = hdec1 * HOy[b] - hsrc1 * (div_rn(E1x[b] - ex, res, inv_res) -
                                                   div_rn(E0z[b + 1] - ez, res, inv_res));
        const float hz = hdec2 * HOz[b] - hsrc2 * (div_rn(E0y[b + 1] - ey, res, inv_res) -
                                                   div_rn(E0x[b + T::BX] - ex, res, inv_res));
        sm.hn[hb][0][ly][lx] = hx;
        sm.hn[hb][1][ly][lx] = hy;
        sm.hn[hb][2][ly][lx] = hz;
        if (emit) {
          p.hout[0][o] = hx;
          p.hout[1][o] = hy;
          p.hout[2][o] = hz;
        }
      } else if (Cpml && kCpmlAhead && plane_face_free && row_face_free[r] && col_face_free) {
        // Off every face but inside an absorber: raw derivatives, then the
        // active recurrences with psi fetched a plane ahead.
        const int j = j0 + ly - 1;
        const int b = ly * T::BX + lane + 4;
        const int o = k * PL + j * P + i;
        const float ez = E0z[b], ey = E0y[b], ex = E0x[b];
        float dx0 = div_rn(E0z[b + T::BX] - ez, res, inv_res), dx1 = div_rn(E1y[b] - ey, res, inv_res);
        float dy0 = div_rn(E1x[b] - ex, res, inv_res), dy1 = div_rn(E0z[b + 1] - ez, res, inv_res);
        float dz0 = div_rn(E0y[b + 1] - ey, res, inv_res), dz1 = div_rn(E0x[b + T::BX] - ex, res, inv_res);
        if (emit) {
          dx0 = cpml_use(p.ht[0], sm.coef[0], coef_smem, syh[r], ph[r][0], dx0, p.ht[0].psi_out,
                         syh[r] >= 0 ? psi_offset<1>(p.ht[0], syh[r], k, j, i) : 0);
          dx1 = cpml_use(p.ht[1], sm.coef[1], coef_smem, szh, ph[r][1], dx1, p.ht[1].psi_out,
                         szh >= 0 ? psi_offset<0>(p.ht[1], szh, k, j, i) : 0);
          dy0 = cpml_use(p.ht[2], sm.coef[2], coef_smem, szh, ph[r][2], dy0, p.ht[2].psi_out,
                         szh >= 0 ? psi_offset<0>(p.ht[2], szh, k, j, i) : 0);
          dy1 = cpml_use(p.ht[3], sm.coef[3], coef_smem, sxh, ph[r][3], dy1, p.ht[3].psi_out,
                         sxh >= 0 ? psi_offset<2>(p.ht[3], sxh, k, j, i) : 0);
          dz0 = cpml_use(p.ht[4], sm.coef[4], coef_smem, sxh, ph[r][4], dz0, p.ht[4].psi_out,
                         sxh >= 0 ? psi_offset<2>(p.ht[4], sxh, k, j, i) : 0);
          dz1 = cpml_use(p.ht[5], sm.coef[5], coef_smem, syh[r], ph[r][5], dz1, p.ht[5].psi_out,
                         syh[r] >= 0 ? psi_offset<1>(p.ht[5], syh[r], k, j, i) : 0);
        } else {
          h_general(ly, lx, false, 7);  // chunk prologue plane: values only
          continue;
        }
        const float hx = hdec0 * HOx[b] - hsrc0 * (dx0 - dx1);
        const float hy = hdec1 * HOy[b] - hsrc1 * (dy0 - dy1);
        const float hz = hdec2 * HOz[b] - hsrc2 * (dz0 - dz1);
        sm.hn[hb][0][ly][lx] = hx;
        sm.hn[hb][1][ly][lx] = hy;
        sm.hn[hb][2][ly][lx] = hz;
        p.hout[0][o] = hx;
        p.hout[1][o] = hy;
        p.hout[2][o] = hz;
      } else {
        h_general(ly, lx, emit, 7);
      }
    }
    if (warp == 0) h_general(0, 1 + lane, false, 1 | 4);                       // y halo row: Hx, Hz
    if (warp == 1 && lane < T::TY) h_general(1 + lane, 0, false, 2 | 4);       // x halo column: Hy, Hz
    __syncthreads();

    // ---- E(k) ----------------------------------------------------------------
    if (emit) {
      const int pb = hb ^ 1;
      const int v0 = (k + 2) % 3, v1 = k % 3;  // permittivity planes clip(k-1), clip(k)
      const bool zlo = k == 0, zhi = k == Z;
      const bool xlo = i == 0, xhi = i == X;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int ly = 1 + warp * R + r, lx = 1 + lane, b = ly * T::BX + lane + 4;
        const int j = j0 + ly - 1;
        const int o = k * PL + j * P + i;
        const float hx = sm.hn[hb][0][ly][lx], hy = sm.hn[hb][1][ly][lx], hz = sm.hn[hb][2][ly][lx];
        const float hz_y = sm.hn[hb][2][ly - 1][lx], hz_x = sm.hn[hb][2][ly][lx - 1];
        const float hy_z = sm.hn[pb][1][ly][lx], hy_x = sm.hn[hb][1][ly][lx - 1];
        const float hx_z = sm.hn[pb][0][ly][lx], hx_y = sm.hn[hb][0][ly - 1][lx];
        if (plane_fast && row_fast[r] && col_fast) {
          // Interior, absorber-free: every component exists, no ghost planes, no PEC.
          const float dx0 = div_rn(hz - hz_y, res, inv_res), dx1 = div_rn(hy - hy_z, res, inv_res);
          const float dy0 = div_rn(hx - hx_z, res, inv_res), dy1 = div_rn(hz - hz_x, res, inv_res);
          const float dz0 = div_rn(hy - hy_x, res, inv_res), dz1 = div_rn(hx - hx_y, res, inv_res);
          const float a00 = sm.eps[v0][ly - 1][lx - 1], a01 = sm.eps[v0][ly - 1][lx];
          const float a10 = sm.eps[v0][ly][lx - 1], a11 = sm.eps[v0][ly][lx];
          const float b00 = sm.eps[v1][ly - 1][lx - 1], b01 = sm.eps[v1][ly - 1][lx];
          const float b10 = sm.eps[v1][ly][lx - 1], b11 = sm.eps[v1][ly][lx];
          // beamz/lattice.py:732-786: average z, then y (Ex) / x (Ey); Ez: y then x.
          const float ex_eps = 0.5f * (0.5f * (a01 + b01) + 0.5f * (a11 + b11));
          const float ey_eps = 0.5f * (0.5f * (a10 + b10) + 0.5f * (a11 + b11));
          const float ez_eps = 0.5f * (0.5f * (b00 + b10) + 0.5f * (b01 + b11));
          p.eout[0][o] = E0x[b] + (dto * __frcp_rn(ex_eps)) * (dx0 - dx1);
          p.eout[1][o] = E0y[b] + (dto * __frcp_rn(ey_eps)) * (dy0 - dy1);
          p.eout[2][o] = E0z[b] + (dto * __frcp_rn(ez_eps)) * (dz0 - dz1);
        } else if (Cpml && kCpmlAhead && plane_face_free && row_face_free[r] && col_face_free) {
          // Off every face, inside an absorber.
          float dx0 = div_rn(hz - hz_y, res, inv_res), dx1 = div_rn(hy - hy_z, res, inv_res);
          float dy0 = div_rn(hx - hx_z, res, inv_res), dy1 = div_rn(hz - hz_x, res, inv_res);
          float dz0 = div_rn(hy - hy_x, res, inv_res), dz1 = div_rn(hx - hx_y, res, inv_res);
          dx0 = cpml_use(p.et[0], sm.coef[6], coef_smem, sye[r], pe[r][0], dx0, p.et[0].psi_out,
                         sye[r] >= 0 ? psi_offset<1>(p.et[0], sye[r], k, j, i) : 0);
          dx1 = cpml_use(p.et[1], sm.coef[7], coef_smem, sze, pe[r][1], dx1, p.et[1].psi_out,
                         sze >= 0 ? psi_offset<0>(p.et[1], sze, k, j, i) : 0);
          dy0 = cpml_use(p.et[2], sm.coef[8], coef_smem, sze, pe[r][2], dy0, p.et[2].psi_out,
                         sze >= 0 ? psi_offset<0>(p.et[2], sze, k, j, i) : 0);
          dy1 = cpml_use(p.et[3], sm.coef[9], coef_smem, sxe, pe[r][3], dy1, p.et[3].psi_out,
                         sxe >= 0 ? psi_offset<2>(p.et[3], sxe, k, j, i) : 0);
          dz0 = cpml_use(p.et[4], sm.coef[10], coef_smem, sxe, pe[r][4], dz0, p.et[4].psi_out,
                         sxe >= 0 ? psi_offset<2>(p.et[4], sxe, k, j, i) : 0);
          dz1 = cpml_use(p.et[5], sm.coef[11], coef_smem, sye[r], pe[r][5], dz1, p.et[5].psi_out,
                         sye[r] >= 0 ? psi_offset<1>(p.et[5], sye[r], k, j, i) : 0);
          const float a00 = sm.eps[v0][ly - 1][lx - 1], a01 = sm.eps[v0][ly - 1][lx];
          const float a10 = sm.eps[v0][ly][lx - 1], a11 = sm.eps[v0][ly][lx];
          const float b00 = sm.eps[v1][ly - 1][lx - 1], b01 = sm.eps[v1][ly - 1][lx];
          const float b10 = sm.eps[v1][ly][lx - 1], b11 = sm.eps[v1][ly][lx];
          const float ex_eps = 0.5f * (0.5f * (a01 + b01) + 0.5f * (a11 + b11));
          const float ey_eps = 0.5f * (0.5f * (a10 + b10) + 0.5f * (a11 + b11));
          const float ez_eps = 0.5f * (0.5f * (b00 + b10) + 0.5f * (b01 + b11));
          p.eout[0][o] = E0x[b] + (dto * __frcp_rn(ex_eps)) * (dx0 - dx1);
          p.eout[1][o] = E0y[b] + (dto * __frcp_rn(ey_eps)) * (dy0 - dy1);
          p.eout[2][o] = E0z[b] + (dto * __frcp_rn(ez_eps)) * (dz0 - dz1);
        } else if (j <= Y && i <= X) {
          // Faces, absorbers: ghost planes, clamped voxel sampling, PEC, CPML.
          const bool ylo = j == 0, yhi = j == Y;
          const int ry0 = ylo ? ly : ly - 1, ry1 = yhi ? ly - 1 : ly;  // rows clip(j-1), clip(j)
          const int cx0 = xlo ? lx : lx - 1, cx1 = xhi ? lx - 1 : lx;  // cols clip(i-1), clip(i)
          const bool okx = i < X, oky = j < Y, okz = zZ;
          if (okx) {  // Ex: dHz/dy - dHy/dz
            CpmlOp cx0p, cx1p;
            if (cpml) { cx0p = cpml_fetch<1>(p.et[0], k, j, i); cx1p = cpml_fetch<0>(p.et[1], k, j, i); }
            float d0 = ghost(hz, hz_y, ylo, yhi, wy0, wy1, res, inv_res);
            float d1 = ghost(hy, hy_z, zlo, zhi, wz0, wz1, res, inv_res);
            if (cpml) {
              d0 = cpml_apply(p.et[0], cx0p, d0, true);
              d1 = cpml_apply(p.et[1], cx1p, d1, true);
            }
            const float eps = 0.5f * (0.5f * (sm.eps[v0][ry0][lx] + sm.eps[v1][ry0][lx]) +
                                      0.5f * (sm.eps[v0][ry1][lx] + sm.eps[v1][ry1][lx]));
            float e = E0x[b] + (dto * __frcp_rn(eps)) * (d0 - d1);
            if ((zlo && wz0) || (zhi && wz1) || (ylo && wy0) || (yhi && wy1)) e = 0.0f;
            p.eout[0][o] = e;
          }
          if (oky) {  // Ey: dHx/dz - dHz/dx
            CpmlOp cy0p, cy1p;
            if (cpml) { cy0p = cpml_fetch<0>(p.et[2], k, j, i); cy1p = cpml_fetch<2>(p.et[3], k, j, i); }
            float d0 = ghost(hx, hx_z, zlo, zhi, wz0, wz1, res, inv_res);
            float d1 = ghost(hz, hz_x, xlo, xhi, wx0, wx1, res, inv_res);
            if (cpml) {
              d0 = cpml_apply(p.et[2], cy0p, d0, true);
              d1 = cpml_apply(p.et[3], cy1p, d1, true);
            }
            const float eps = 0.5f * (0.5f * (sm.eps[v0][ly][cx0] + sm.eps[v1][ly][cx0]) +
                                      0.5f * (sm.eps[v0][ly][cx1] + sm.eps[v1][ly][cx1]));
            float e = E0y[b] + (dto * __frcp_rn(eps)) * (d0 - d1);
            if ((zlo && wz0) || (zhi && wz1) || (xlo && wx0) || (xhi && wx1)) e = 0.0f;
            p.eout[1][o] = e;
          }
          if (okz) {  // Ez: dHy/dx - dHx/dy
            CpmlOp cz0p, cz1p;
            if (cpml) { cz0p = cpml_fetch<2>(p.et[4], k, j, i); cz1p = cpml_fetch<1>(p.et[5], k, j, i); }
            float d0 = ghost(hy, hy_x, xlo, xhi, wx0, wx1, res, inv_res);
            float d1 = ghost(hx, hx_y, ylo, yhi, wy0, wy1, res, inv_res);
            if (cpml) {
              d0 = cpml_apply(p.et[4], cz0p, d0, true);
              d1 = cpml_apply(p.et[5], cz1p, d1, true);
            }
            const float eps = 0.5f * (0.5f * (sm.eps[v1][ry0][cx0] + sm.eps[v1][ry1][cx0]) +
                                      0.5f * (sm.eps[v1][ry0][cx1] + sm.eps[v1][ry1][cx1]));
            float e = E0z[b] + (dto * __frcp_rn(eps)) * (d0 - d1);
            if ((ylo && wy0) || (yhi && wy1) || (xlo && wx0) || (xhi && wx1)) e = 0.0f;
            p.eout[2][o] = e;
          }
        }
      }
    }
  }
}

template <int NW, int R, bool Cpml>
cudaError_t launch_tma_t(cudaStream_t s, const TmaMaps& maps, const Step3D& p) {
  using T = TmaTile<NW, R>;
  const size_t smem = sizeof(typename T::Smem) + 128;
  auto kern = tma_step_kernel<NW, R, Cpml>;
  static bool configured = false;
  if (!configured) {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    configured = true;
  }
  const int kmax = p.Z + 1;
  const int zc = p.z_chunk > 0 ? p.z_chunk : kmax;
  const dim3 grid((p.X + 1 + T::TX - 1) / T::TX, (p.Y + 1 + T::TY - 1) / T::TY, (kmax + zc - 1) / zc);
  Step3D q = p;
  q.z_chunk = zc;
  kern<<<grid, dim3(32, NW, 1), smem, s>>>(maps, q);
  return cudaPeekAtLastError();
}

// ---- tensor maps -------------------------------------------------------------
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder() {
  static EncodeFn fn = nullptr;
  if (fn == nullptr) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &ptr, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    fn = reinterpret_cast<EncodeFn>(ptr);
  }
  return fn;
}

bool encode(CUtensorMap* map, CUtensorMapDataType type, const void* base, int elem, int64_t dx, int64_t dy,
            int64_t dz, int64_t row_bytes, int64_t plane_bytes, int bx, int by) {
  EncodeFn fn = encoder();
  if (fn == nullptr) return false;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(dx), static_cast<cuuint64_t>(dy), static_cast<cuuint64_t>(dz)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(row_bytes), static_cast<cuuint64_t>(plane_bytes)};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(bx), static_cast<cuuint32_t>(by), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  (void)elem;
  return fn(map, type, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int NW, int R>
cudaError_t launch_tma_shape(cudaStream_t s, const Step3D& p) {
  using T = TmaTile<NW, R>;
  TmaMaps maps;
  const int64_t P = p.pitch, rowb = P * 4, planeb = static_cast<int64_t>(p.Y + 1) * P * 4;
  for (int c = 0; c < 3; ++c) {
    const Dims de = component_dims(c, p.Z, p.Y, p.X), dh = component_dims(c + 3, p.Z, p.Y, p.X);
    if (!encode(&maps.e[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.ein[c], 4, de.x, de.y, de.z, rowb, planeb, T::BX,
                T::EH) ||
        !encode(&maps.h[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.hin[c], 4, dh.x, dh.y, dh.z, rowb, planeb, T::BX,
                T::HH))
      return cudaErrorInvalidValue;
  }
  if (!encode(&maps.vox, CU_TENSOR_MAP_DATA_TYPE_UINT8, p.em.voxels, 1, p.X, p.Y, p.Z, p.voxel_pitch,
              static_cast<int64_t>(p.Y) * p.voxel_pitch, T::VX, T::HH))
    return cudaErrorInvalidValue;
  return p.cpml ? launch_tma_t<NW, R, true>(s, maps, p) : launch_tma_t<NW, R, false>(s, maps, p);
}

}  // namespace

// tile_y selects the CTA shape: y rows = warps x rows per thread.
cudaError_t launch_fused_tma(cudaStream_t s, const Step3D& p, int tile_y) {
  switch (tile_y) {
    case 4: return launch_tma_shape<4, 1>(s, p);
    case 16: return launch_tma_shape<8, 2>(s, p);
    case 108: return launch_tma_shape<4, 2>(s, p);  // 8 rows, two per thread
    case 116: return launch_tma_shape<4, 4>(s, p);  // 16 rows, four per thread
    default: return launch_tma_shape<8, 1>(s, p);
  }
}

}  // namespace fdtd
