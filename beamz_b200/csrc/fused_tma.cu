// One-kernel 3D leapfrog step on the pitched field layout, staged by TMA.
//
// Pitched layout: every field component is a (Z+1, Y+1, P) float array with
// the same 16-byte-multiple row pitch P >= X+1 (the component's own extent is
// its corner (dz, dy, dx) block).  The electric material is a codebook: one
// 32-bit word per lattice point on the same pitch holds the 8-bit ids of the
// Ex, Ey and Ez update coefficients fl(fl(dt)/fl(eps0) * fl(1/eps_site)),
// looked up in three 256-entry tables (beamz packs its lossless E material the
// same way, beamz/simulation/compile.py:146-187).  One element offset
// (k*(Y+1) + j)*P + i addresses a lattice point in all of these arrays, and
// each plane of each array is a legal TMA box.
//
// A CTA of NW warps owns a 32 x (NW*R) tile of (y, x) lattice points and a
// chunk of z planes.  Per plane k:
//   1. wait on the mbarrier of bundle k = {E(k+1), H(k), site ids(k)} (one TMA
//      box per array), then one CTA barrier;
//   2. thread 0 issues bundle k+1 into the buffers plane k-1 released;
//   3. H(k) on the own cells (R per thread), the y-halo row (warp 0: Hx, Hz)
//      and the x-halo column (warp 1: Hy, Hz) -- recomputed, so no CTA waits
//      on another; barrier;
//   4. E(k) on the own cells from H(k) and H(k-1) (double-buffered in shared
//      memory).
// A tile-plane clear of the high domain faces and of H sources runs one of six
// straight-line bodies (by the absorber axes it touches); all others run the
// general one (ghost planes, PEC, CPML with both operands of a component
// fetched before use, H sources, validity).
// TMA zero-fills outside each array's extent.  Fields and the H-term CPML
// memories are double-banked (read A, write B); E-term memories stay in
// place.  Every mbarrier wait is bounded: on expiry the kernel records an
// error word, drains its copy in flight (bounded again) and returns.
//
// Arithmetic follows beamz/simulation/kernels.py:458-626 operation for
// operation (rounding contract in fdtd_common.cuh); PEC, CPML and H-timing
// sources follow beamz/simulation/execute.py:467-522.

#include <cuda.h>

#include <type_traits>

#include "kernels.cuh"
#include "tma_util.cuh"

namespace fdtd {

namespace {

using tma::bar_expect;
using tma::bar_init;
using tma::bar_wait;
using tma::encode;
using tma::smem_u32;

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* b) {
  tma::load_3d(dst, map, x, y, z, b);
}

constexpr int kCoefSlots = 32;  // CPML coefficient slots staged per term

template <int NW, int R>
struct TmaTile {
  static constexpr int TX = 32, TY = NW * R, NT = 32 * NW;
  static constexpr int BX = TX + 8;  // staged row: x from i0-4 to i0+TX+3
  static constexpr int EH = TY + 2;  // E rows j0-1 .. j0+TY
  static constexpr int HH = TY + 1;  // H rows j0-1 .. j0+TY-1
  static constexpr int HW = TX + 2;  // H-region columns i0-1 .. i0+TX (the last: column X of the last tile)
  static constexpr int EBOX = ((EH * BX + 31) / 32) * 32;  // floats; boxes start on 128 B
  static constexpr int HBOX = ((HH * BX + 31) / 32) * 32;
  static constexpr int IBOX = TY * TX;  // site-id words, rows j0 .. j0+TY-1
  struct Smem {
    float e[3 * 3][EBOX];  // E ring: 3 planes x 3 components
    float h[2 * 3][HBOX];  // H(old) ring: 2 planes x 3 components
    uint32_t ids[2][IBOX];
    float hn[2][3][HH][HW];
    float coef[3][256];
    float4 cc[12][kCoefSlots];  // CPML (a, b, 1/kappa): H terms 0-5, E terms 6-11
    float amp[kMaxFusedSources];
    unsigned long long bar[2];
  };
};

struct TmaMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
  CUtensorMap ids;
};

// Issue bundle q: E(q+1) (and E(q) when `first`), H(q), site ids(q).  Every x
// coordinate is i0 - 4 or i0 (i0 a multiple of 32): 16-byte aligned.
template <class T>
__device__ __forceinline__ void issue_bundle(typename T::Smem& sm, const TmaMaps& maps, int q, int Z, int j0, int i0,
                                             int slot, bool first) {
  const int ne = (first ? 1 : 0) + (q + 1 <= Z ? 1 : 0);
  const unsigned bytes = ne * 3 * T::EH * T::BX * 4 + 3 * T::HH * T::BX * 4 + T::IBOX * 4;
  unsigned long long* b = &sm.bar[slot];
  bar_expect(b, bytes);
  if (first)
    for (int c = 0; c < 3; ++c) tma_load_3d(sm.e[(q % 3) * 3 + c], &maps.e[c], i0 - 4, j0 - 1, q, b);
  if (q + 1 <= Z)
    for (int c = 0; c < 3; ++c) tma_load_3d(sm.e[((q + 1) % 3) * 3 + c], &maps.e[c], i0 - 4, j0 - 1, q + 1, b);
  for (int c = 0; c < 3; ++c) tma_load_3d(sm.h[(q % 2) * 3 + c], &maps.h[c], i0 - 4, j0 - 1, q, b);
  tma_load_3d(sm.ids[q % 2], &maps.ids, i0, j0, q, b);
}

__device__ __forceinline__ float ghost(float center, float below, bool at_low, bool at_high, bool low_wall,
                                       bool high_wall, float res, float inv_res) {
  // beamz/lattice.py:523-551: zero beyond a metallic wall, else a copy of the
  // edge sample so that the edge derivative vanishes.
  if (at_low) return low_wall ? div_rn(center - 0.0f, res, inv_res) : 0.0f;
  if (at_high) return high_wall ? div_rn(0.0f - below, res, inv_res) : 0.0f;
  return div_rn(center - below, res, inv_res);
}

// A CPML recurrence split in two so that both operands' loads of a component
// are in flight together: fetch (slot, psi, a, b, 1/kappa), then apply.
struct CpmlOp {
  int slot = -1;
  int off = 0;
  float psi = 0.0f;
  float4 c = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
};

template <int Axis>
__device__ __forceinline__ CpmlOp cpml_fetch(const CpmlTermDev& t, const float4* cc, bool cc_smem, int k, int j,
                                             int i) {
  CpmlOp op;
  const int coord = Axis == 0 ? k : (Axis == 1 ? j : i);
  op.slot = cpml_slot(t, coord);
  if (op.slot >= 0) {
    const int pk = Axis == 0 ? op.slot : k;
    const int pj = Axis == 1 ? op.slot : j;
    const int pi = Axis == 2 ? op.slot : i;
    op.off = (pk * t.pdy + pj) * t.pdx + pi;  // psi slabs hold < 2^31 elements (validated)
    op.psi = t.psi_in[op.off];
    op.c = cc_smem ? cc[op.slot]
                   : make_float4(__ldg(t.a + op.slot), __ldg(t.b + op.slot), __ldg(t.k + op.slot), 0.0f);
  }
  return op;
}

// psi <- b psi + a d; returns d / kappa + psi (beamz/simulation/kernels.py:257-264).
__device__ __forceinline__ float cpml_apply(const CpmlTermDev& t, const CpmlOp& op, float d, bool write) {
  if (op.slot < 0) return d;
  const float psi = op.c.y * op.psi + op.c.x * d;
  if (write) t.psi_out[op.off] = psi;
  return d * op.c.z + psi;
}

// CPML halves for the straight-line paths: every term of a cell is fetched
// (slot, offset, psi) before any is applied, so the loads are in flight
// together; apply runs psi <- b psi + a d and returns d / kappa + psi with
// (a, b, 1/kappa) staged in shared memory.
struct Psi {
  int slot = -1;
  int off = 0;
  float v = 0.0f;
};

template <int Axis>
__device__ __forceinline__ int psi_offset(const CpmlTermDev& t, int slot, int k, int j, int i) {
  const int pk = Axis == 0 ? slot : k;
  const int pj = Axis == 1 ? slot : j;
  const int pi = Axis == 2 ? slot : i;
  return (pk * t.pdy + pj) * t.pdx + pi;
}

template <int Axis>
__device__ __forceinline__ Psi psi_fetch(const CpmlTermDev& t, int slot, int k, int j, int i) {
  Psi q;
  q.slot = slot;
  if (slot >= 0) {
    q.off = psi_offset<Axis>(t, slot, k, j, i);
    q.v = t.psi_in[q.off];
  }
  return q;
}

__device__ __forceinline__ float psi_apply(const CpmlTermDev& t, const float4* cc, const Psi& q, float d,
                                           bool write) {
  if (q.slot < 0) return d;
  const float4 c = cc[q.slot];
  const float next = c.y * q.v + c.x * d;
  if (write) t.psi_out[q.off] = next;
  return d * c.z + next;
}

// Paired FP32 arithmetic (sm_100 f32x2 instructions): each lane of the pair is
// rounded exactly as the scalar operation, so paired and scalar code agree
// bit for bit; the pair halves the instructions issued.  The operations are
// PTX with an explicit rounding mode, and the pairs are packed and unpacked
// with mov.b64 (no type punning).  A paired add or subtract fed by a paired
// multiply was measured to come out fused into one rounding (about a fifth of
// the lanes differ), so the final multiply-adds of the H and E updates stay
// scalar.
__device__ __forceinline__ unsigned long long f2pack(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};\n" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}

__device__ __forceinline__ float2 f2unpack(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;\n" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}

__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;\n" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)));
  return f2unpack(r);
}

__device__ __forceinline__ float2 f2mul(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;\n" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)));
  return f2unpack(r);
}

__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;\n" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)), "l"(f2pack(c)));
  return f2unpack(r);
}

// div_rn on a pair (fdtd_common.cuh): r2 = (rs, rs), nb2 = (-bs, -bs).
__device__ __forceinline__ float2 f2div(float2 a, float2 r2, float2 nb2) {
  const float2 as = f2mul(a, make_float2(kDivScale, kDivScale));
  const float2 q = f2mul(as, r2);
  const float2 e = f2fma(q, nb2, as);
  return f2fma(e, r2, q);
}

using kOff = std::integral_constant<bool, false>;
using kOn = std::integral_constant<bool, true>;

__device__ __forceinline__ float h_sources(const Step3D& p, const float* amp, int c, int k, int j, int i, float h) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    const int z = k - src.z0, y = j - src.y0, x = i - src.x0;
    if (src.component != c || z < 0 || y < 0 || x < 0 || z >= src.ez || y >= src.ey || x >= src.ex) continue;
    h = h + src.coeff[(static_cast<int64_t>(z) * src.ey + y) * src.ex + x] * amp[s];
  }
  return h;
}

// Does any H source touch plane k of the region rows [jlo, jhi] x cols [ilo, ihi]?
__device__ __forceinline__ bool sources_hit(const Step3D& p, int k, int jlo, int jhi, int ilo, int ihi) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    if (k >= src.z0 && k < src.z0 + src.ez && jhi >= src.y0 && jlo < src.y0 + src.ey && ihi >= src.x0 &&
        ilo < src.x0 + src.ex)
      return true;
  }
  return false;
}

// Straight-line H of one cell from the staged E planes (box index b).
struct HFast {
  float dec0, dec1, dec2, src0, src1, src2, res, inv_res;
  template <int BX>
  __device__ __forceinline__ float hx(const float* E0z, const float* E0y, const float* E1y, const float* HOx,
                                     int b) const {
    return dec0 * HOx[b] - src0 * (div_rn(E0z[b + BX] - E0z[b], res, inv_res) - div_rn(E1y[b] - E0y[b], res, inv_res));
  }
  template <int BX>
  __device__ __forceinline__ float hy(const float* E0x, const float* E0z, const float* E1x, const float* HOy,
                                     int b) const {
    return dec1 * HOy[b] - src1 * (div_rn(E1x[b] - E0x[b], res, inv_res) - div_rn(E0z[b + 1] - E0z[b], res, inv_res));
  }
  template <int BX>
  __device__ __forceinline__ float hz(const float* E0y, const float* E0x, const float* HOz, int b) const {
    return dec2 * HOz[b] - src2 * (div_rn(E0y[b + 1] - E0y[b], res, inv_res) - div_rn(E0x[b + BX] - E0x[b], res, inv_res));
  }
};

// 8-warp, one-row CTAs are capped at 48 registers (5 resident CTAs, the
// shared-memory limit too); the CPML body still fits without spills.
template <int NW, int R, bool Cpml>
__global__ void __launch_bounds__(32 * NW, NW == 8 && R == 1 ? 5 : 1024 / (32 * NW))
    tma_step_kernel(const __grid_constant__ TmaMaps maps, Step3D p) {
  using T = TmaTile<NW, R>;
  using S = typename T::Smem;
  constexpr int BX = T::BX;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);
  const int lane = threadIdx.x, warp = threadIdx.y;
  const int tid = warp * 32 + lane;
  const int i0 = blockIdx.x * T::TX, j0 = blockIdx.y * T::TY;
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int k0 = blockIdx.z * p.z_chunk;
  const int k1 = min(k0 + p.z_chunk, Z + 1);
  const int kstart = k0 > 0 ? k0 - 1 : 0;
  const float res = p.div_bs, inv_res = p.div_rs;  // div_rn's scaled cell size and reciprocal
  const int P = p.pitch, PL = (Y + 1) * p.pitch;

  if (tid == 0) {
    bar_init(&sm.bar[0], 1);
    bar_init(&sm.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    // Bundle kstart goes out first, so its latency overlaps the table staging;
    // bundle k+1 is issued at plane k (the three-plane E ring and two-plane
    // H / id rings hold planes k, k+1 and the one in flight).
    issue_bundle<T>(sm, maps, kstart, Z, j0, i0, 0, true);
  }
  for (int e = tid; e < 3 * 256; e += T::NT) (&sm.coef[0][0])[e] = p.em.site_coef[e];
  bool cc_smem = true;
  if (Cpml) {
#pragma unroll
    for (int t = 0; t < 12; ++t) {
      const CpmlTermDev& d = t < 6 ? p.ht[t] : p.et[t - 6];
      const int w = d.low + d.high;
      cc_smem = cc_smem && w <= kCoefSlots;
      for (int e = tid; e < w && e < kCoefSlots; e += T::NT) sm.cc[t][e] = make_float4(d.a[e], d.b[e], d.k[e], 0.0f);
    }
  }
  if (tid < p.n_hsrc) sm.amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);
  __syncthreads();

  // ---- per-CTA / per-thread constants -------------------------------------
  const bool wz0 = wall(p.metallic, 0, false), wz1 = wall(p.metallic, 0, true);
  const bool wy0 = wall(p.metallic, 1, false), wy1 = wall(p.metallic, 1, true);
  const bool wx0 = wall(p.metallic, 2, false), wx1 = wall(p.metallic, 2, true);
  // The pitched layout carries uniform H coefficients (validated on the host).
  const HFast hf{p.hm.decay[0][0], p.hm.decay[1][0], p.hm.decay[2][0], p.hm.source[0][0], p.hm.source[1][0],
                 p.hm.source[2][0], res, inv_res};
  const int i = i0 + lane;
  // When X is a multiple of the tile width, the last tile also owns the
  // face column i = X (Hx, Ey, Ez there), computed by its last warp, so no
  // CTA is spent on a single column.
  const bool xcol = X % T::TX == 0 && i0 + T::TX == X;
  const int xe = xcol ? 1 : 0;
  const bool cpml_xy = Cpml && !(i0 - 1 >= p.cpml_inner[2][0] && i0 + T::TX + xe <= p.cpml_inner[2][1] &&
                                 j0 - 1 >= p.cpml_inner[1][0] && j0 + T::TY <= p.cpml_inner[1][1]);
  // Straight-line tiles: below the y-high face and left of the x-high face
  // (the low faces x = 0 and y = 0 by per-lane / per-row selects, column X
  // by the last warp), with every CPML coefficient staged in shared memory.
  const bool mid_ok = j0 + T::TY <= Y && i0 + T::TX <= X && cc_smem;
  const bool xface = i0 == 0, yface = j0 == 0;
  // Axes whose absorber slabs the tile (own cells and halos) touches.
  const bool ax = Cpml && !(i0 - 1 >= p.cpml_inner[2][0] && i0 + T::TX + xe <= p.cpml_inner[2][1]);
  const bool ay = Cpml && !(j0 - 1 >= p.cpml_inner[1][0] && j0 + T::TY <= p.cpml_inner[1][1]);

  int e0 = kstart % 3, e1 = (kstart + 1) % 3, hs = kstart & 1;
  for (int k = kstart; k < k1; ++k) {
    const int n = k - kstart;
    const bool emit = k >= k0;
    const bool arrived = bar_wait(&sm.bar[n & 1], (n >> 1) & 1);
    if (__syncthreads_or(!arrived)) {  // CTA-uniform: every thread leaves together
      if (tid == 0) {
        if (p.status) atomicExch(p.status, 1);
        bar_wait(&sm.bar[n & 1], (n >> 1) & 1);  // the only bundle in flight
      }
      __syncthreads();
      return;
    }
    if (tid == 0 && k + 1 < k1) {
      // Plane k-1's generic reads of these buffers precede the TMA writes.
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue_bundle<T>(sm, maps, k + 1, Z, j0, i0, (n + 1) & 1, false);
    }
    const float* E0x = sm.e[e0 * 3 + 0];
    const float* E0y = sm.e[e0 * 3 + 1];
    const float* E0z = sm.e[e0 * 3 + 2];
    const float* E1x = sm.e[e1 * 3 + 0];
    const float* E1y = sm.e[e1 * 3 + 1];
    const float* HOx = sm.h[hs * 3 + 0];
    const float* HOy = sm.h[hs * 3 + 1];
    const float* HOz = sm.h[hs * 3 + 2];
    const uint32_t* IDS = sm.ids[hs];
    const int hb = k & 1, pb = hb ^ 1;
    const bool src = p.n_hsrc > 0 && sources_hit(p, k, j0 - 1, j0 + T::TY, i0 - 1, i0 + T::TX);

    if (mid_ok && !src && k >= 1 && k < Z) {
      // ---- straight-line tile-plane --------------------------------------
      // Every own and halo cell is a valid site of all six components; the
      // faces x = 0 (i0 == 0) and y = 0 (j0 == 0) drop their halo and take the
      // ghost value by select; column X (xcol) is the last warp's extra work.
      // CPML terms run only for the axes whose slabs the tile-plane touches,
      // chosen at compile time: AX, AY, AZ.
      auto body = [&](auto axc, auto ayc, auto azc, auto fc) {
        constexpr bool AX = decltype(axc)::value, AY = decltype(ayc)::value, AZ = decltype(azc)::value;
        // FC: the tile may touch the faces x = 0 / y = 0 (else their selects drop).
        constexpr bool FC = decltype(fc)::value;
        const bool at_x0 = FC && xface, at_y0 = FC && yface;
        int zh1 = -1, zh2 = -1, ze1 = -1, ze2 = -1;  // plane-uniform z slots
        if constexpr (AZ) {
          zh1 = cpml_slot(p.ht[1], k);
          zh2 = cpml_slot(p.ht[2], k);
          ze1 = cpml_slot(p.et[1], k);
          ze2 = cpml_slot(p.et[2], k);
        }
        // H at box index b, lattice (k, j, ii); W: 1 Hx, 2 Hy, 4 Hz.
        auto h_cell = [&](auto wc, int b, int j, int ii, bool own, float* hv) {
          constexpr int W = decltype(wc)::value;
          Psi q0, q1, q2, q3, q4, q5;
          if constexpr ((W & 1) && AY) q0 = psi_fetch<1>(p.ht[0], cpml_slot(p.ht[0], j), k, j, ii);
          if constexpr ((W & 1) && AZ) q1 = psi_fetch<0>(p.ht[1], zh1, k, j, ii);
          if constexpr ((W & 2) && AZ) q2 = psi_fetch<0>(p.ht[2], zh2, k, j, ii);
          if constexpr ((W & 2) && AX) q3 = psi_fetch<2>(p.ht[3], cpml_slot(p.ht[3], ii), k, j, ii);
          if constexpr ((W & 4) && AX) q4 = psi_fetch<2>(p.ht[4], cpml_slot(p.ht[4], ii), k, j, ii);
          if constexpr ((W & 4) && AY) q5 = psi_fetch<1>(p.ht[5], cpml_slot(p.ht[5], j), k, j, ii);
          if constexpr ((W & 1) != 0) {  // Hx: dEz/dy - dEy/dz
            float d0 = div_rn(E0z[b + BX] - E0z[b], res, inv_res);
            float d1 = div_rn(E1y[b] - E0y[b], res, inv_res);
            if constexpr (AY) d0 = psi_apply(p.ht[0], sm.cc[0], q0, d0, own);
            if constexpr (AZ) d1 = psi_apply(p.ht[1], sm.cc[1], q1, d1, own);
            const float h = hf.dec0 * HOx[b] - hf.src0 * (d0 - d1);
            hv[0] = ((at_x0 && ii == 0 && wx0) || (ii == X && wx1)) ? 0.0f : h;
          }
          if constexpr ((W & 2) != 0) {  // Hy: dEx/dz - dEz/dx
            float d0 = div_rn(E1x[b] - E0x[b], res, inv_res);
            float d1 = div_rn(E0z[b + 1] - E0z[b], res, inv_res);
            if constexpr (AZ) d0 = psi_apply(p.ht[2], sm.cc[2], q2, d0, own);
            if constexpr (AX) d1 = psi_apply(p.ht[3], sm.cc[3], q3, d1, own);
            const float h = hf.dec1 * HOy[b] - hf.src1 * (d0 - d1);
            hv[1] = (at_y0 && j == 0 && wy0) ? 0.0f : h;
          }
          if constexpr ((W & 4) != 0) {  // Hz: dEy/dx - dEx/dy
            float d0 = div_rn(E0y[b + 1] - E0y[b], res, inv_res);
            float d1 = div_rn(E0x[b + BX] - E0x[b], res, inv_res);
            if constexpr (AX) d0 = psi_apply(p.ht[4], sm.cc[4], q4, d0, own);
            if constexpr (AY) d1 = psi_apply(p.ht[5], sm.cc[5], q5, d1, own);
            hv[2] = hf.dec2 * HOz[b] - hf.src2 * (d0 - d1);
          }
        };
        using W1 = std::integral_constant<int, 1>;
        using W7 = std::integral_constant<int, 7>;
        using W5 = std::integral_constant<int, 5>;
        using W6 = std::integral_constant<int, 6>;
        const float2 r2 = make_float2(inv_res, inv_res), nb2 = make_float2(-res, -res);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int ly = 1 + warp * R + r, lx = 1 + lane, b = ly * BX + lane + 4;
          float hv[3];
          if constexpr (!AX && !AY && !AZ) {  // Hx and Hy as a pair, Hz alone
            const int j = j0 + ly - 1;
            const float2 d0 = f2div(f2sub(make_float2(E0z[b + BX], E1x[b]), make_float2(E0z[b], E0x[b])), r2, nb2);
            const float2 d1 = f2div(f2sub(make_float2(E1y[b], E0z[b + 1]), make_float2(E0y[b], E0z[b])), r2, nb2);
            const float2 cd = f2sub(d0, d1);
            const float hx = hf.dec0 * HOx[b] - hf.src0 * cd.x, hy = hf.dec1 * HOy[b] - hf.src1 * cd.y;
            hv[0] = (at_x0 && i == 0 && wx0) ? 0.0f : hx;
            hv[1] = (at_y0 && j == 0 && wy0) ? 0.0f : hy;
            hv[2] = hf.dec2 * HOz[b] - hf.src2 * (div_rn(E0y[b + 1] - E0y[b], res, inv_res) -
                                                  div_rn(E0x[b + BX] - E0x[b], res, inv_res));
          } else {
            h_cell(W7{}, b, j0 + ly - 1, i, emit, hv);
          }
          sm.hn[hb][0][ly][lx] = hv[0];
          sm.hn[hb][1][ly][lx] = hv[1];
          sm.hn[hb][2][ly][lx] = hv[2];
          if (emit) {
            const int o = k * PL + (j0 + ly - 1) * P + i;
            p.hout[0][o] = hv[0];
            p.hout[1][o] = hv[1];
            p.hout[2][o] = hv[2];
          }
        }
        if (warp == 0) {  // y-halo row: Hx, Hz
          if (!at_y0) {
            float hv[3];
            h_cell(W5{}, lane + 4, j0 - 1, i, false, hv);
            sm.hn[hb][0][0][1 + lane] = hv[0];
            sm.hn[hb][2][0][1 + lane] = hv[2];
          }
        } else if (warp == 1 && lane < T::TY && !at_x0) {  // x-halo column: Hy, Hz
          float hv[3];
          h_cell(W6{}, (1 + lane) * BX + 3, j0 + lane, i0 - 1, false, hv);
          sm.hn[hb][1][1 + lane][0] = hv[1];
          sm.hn[hb][2][1 + lane][0] = hv[2];
        }
        if (xcol && warp == NW - 1 && lane <= T::TY && !(at_y0 && lane == 0)) {  // Hx on column X
          float hv[3];
          const int j = j0 - 1 + lane;
          h_cell(W1{}, lane * BX + T::TX + 4, j, X, emit && lane >= 1, hv);
          sm.hn[hb][0][lane][T::TX + 1] = hv[0];
          if (emit && lane >= 1) p.hout[0][k * PL + j * P + X] = hv[0];
        }
        __syncthreads();
        if (!emit) return;
        if (xcol && warp == NW - 1 && lane < T::TY) {  // Ey, Ez on column X
          const int ly = 1 + lane, j = j0 + lane, b = ly * BX + T::TX + 4;
          const float hx = sm.hn[hb][0][ly][T::TX + 1], hx_z = sm.hn[pb][0][ly][T::TX + 1];
          float hx_y = sm.hn[hb][0][ly - 1][T::TX + 1];
          const float hz_x = sm.hn[hb][2][ly][T::TX], hy_x = sm.hn[hb][1][ly][T::TX];
          // Ghost beyond x = X: zero on a metallic wall, else the edge value.
          const float hz = wx1 ? 0.0f : hz_x, hy = wx1 ? 0.0f : hy_x;
          const bool y0 = at_y0 && j == 0;
          if (y0) hx_y = wy0 ? 0.0f : hx;
          Psi q2, q3, q4, q5;
          if constexpr (AZ) q2 = psi_fetch<0>(p.et[2], ze2, k, j, X);
          if constexpr (AX) q3 = psi_fetch<2>(p.et[3], cpml_slot(p.et[3], X), k, j, X);
          if constexpr (AX) q4 = psi_fetch<2>(p.et[4], cpml_slot(p.et[4], X), k, j, X);
          if constexpr (AY) q5 = psi_fetch<1>(p.et[5], cpml_slot(p.et[5], j), k, j, X);
          const int o = k * PL + j * P + X;
          const uint32_t id = p.em.site_ids[o];
          {  // Ey: dHx/dz - dHz/dx
            float d0 = div_rn(hx - hx_z, res, inv_res), d1 = div_rn(hz - hz_x, res, inv_res);
            if constexpr (AZ) d0 = psi_apply(p.et[2], sm.cc[8], q2, d0, true);
            if constexpr (AX) d1 = psi_apply(p.et[3], sm.cc[9], q3, d1, true);
            const float e = E0y[b] + sm.coef[1][(id >> 8) & 0xffu] * (d0 - d1);
            p.eout[1][o] = wx1 ? 0.0f : e;
          }
          {  // Ez: dHy/dx - dHx/dy
            float d0 = div_rn(hy - hy_x, res, inv_res), d1 = div_rn(hx - hx_y, res, inv_res);
            if constexpr (AX) d0 = psi_apply(p.et[4], sm.cc[10], q4, d0, true);
            if constexpr (AY) d1 = psi_apply(p.et[5], sm.cc[11], q5, d1, true);
            const float e = E0z[b] + sm.coef[2][(id >> 16) & 0xffu] * (d0 - d1);
            p.eout[2][o] = (wx1 || (y0 && wy0)) ? 0.0f : e;
          }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int ly = 1 + warp * R + r, lx = 1 + lane, b = ly * BX + lane + 4;
          const int j = j0 + ly - 1;
          const float hx = sm.hn[hb][0][ly][lx], hy = sm.hn[hb][1][ly][lx], hz = sm.hn[hb][2][ly][lx];
          const float hy_z = sm.hn[pb][1][ly][lx], hx_z = sm.hn[pb][0][ly][lx];
          float hz_x = sm.hn[hb][2][ly][lx - 1], hy_x = sm.hn[hb][1][ly][lx - 1];
          float hz_y = sm.hn[hb][2][ly - 1][lx], hx_y = sm.hn[hb][0][ly - 1][lx];
          const bool x0 = at_x0 && i == 0, y0 = at_y0 && j == 0;
          if (x0) {  // ghost beyond x = 0: zero on a metallic wall, else the edge value
            hz_x = wx0 ? 0.0f : hz;
            hy_x = wx0 ? 0.0f : hy;
          }
          if (y0) {  // ghost beyond y = 0
            hz_y = wy0 ? 0.0f : hz;
            hx_y = wy0 ? 0.0f : hx;
          }
          Psi q0, q1, q2, q3, q4, q5;
          if constexpr (AY) q0 = psi_fetch<1>(p.et[0], cpml_slot(p.et[0], j), k, j, i);
          if constexpr (AZ) q1 = psi_fetch<0>(p.et[1], ze1, k, j, i);
          if constexpr (AZ) q2 = psi_fetch<0>(p.et[2], ze2, k, j, i);
          if constexpr (AX) q3 = psi_fetch<2>(p.et[3], cpml_slot(p.et[3], i), k, j, i);
          if constexpr (AX) q4 = psi_fetch<2>(p.et[4], cpml_slot(p.et[4], i), k, j, i);
          if constexpr (AY) q5 = psi_fetch<1>(p.et[5], cpml_slot(p.et[5], j), k, j, i);
          const uint32_t id = IDS[(ly - 1) * T::TX + lane];
          const int o = k * PL + j * P + i;
          if constexpr (!AX && !AY && !AZ) {  // Ex and Ey as a pair, Ez alone
            const float2 d0 = f2div(f2sub(make_float2(hz, hx), make_float2(hz_y, hx_z)), r2, nb2);
            const float2 d1 = f2div(f2sub(make_float2(hy, hz), make_float2(hy_z, hz_x)), r2, nb2);
            const float2 cd = f2sub(d0, d1);
            const float2 e = make_float2(E0x[b] + sm.coef[0][id & 0xffu] * cd.x,
                                         E0y[b] + sm.coef[1][(id >> 8) & 0xffu] * cd.y);
            p.eout[0][o] = (y0 && wy0) ? 0.0f : e.x;
            p.eout[1][o] = (x0 && wx0) ? 0.0f : e.y;
            const float ez = E0z[b] + sm.coef[2][(id >> 16) & 0xffu] *
                                          (div_rn(hy - hy_x, res, inv_res) - div_rn(hx - hx_y, res, inv_res));
            p.eout[2][o] = ((x0 && wx0) || (y0 && wy0)) ? 0.0f : ez;
            continue;
          }
          {  // Ex: dHz/dy - dHy/dz
            float d0 = div_rn(hz - hz_y, res, inv_res), d1 = div_rn(hy - hy_z, res, inv_res);
            if constexpr (AY) d0 = psi_apply(p.et[0], sm.cc[6], q0, d0, true);
            if constexpr (AZ) d1 = psi_apply(p.et[1], sm.cc[7], q1, d1, true);
            const float e = E0x[b] + sm.coef[0][id & 0xffu] * (d0 - d1);
            p.eout[0][o] = (y0 && wy0) ? 0.0f : e;
          }
          {  // Ey: dHx/dz - dHz/dx
            float d0 = div_rn(hx - hx_z, res, inv_res), d1 = div_rn(hz - hz_x, res, inv_res);
            if constexpr (AZ) d0 = psi_apply(p.et[2], sm.cc[8], q2, d0, true);
            if constexpr (AX) d1 = psi_apply(p.et[3], sm.cc[9], q3, d1, true);
            const float e = E0y[b] + sm.coef[1][(id >> 8) & 0xffu] * (d0 - d1);
            p.eout[1][o] = (x0 && wx0) ? 0.0f : e;
          }
          {  // Ez: dHy/dx - dHx/dy
            float d0 = div_rn(hy - hy_x, res, inv_res), d1 = div_rn(hx - hx_y, res, inv_res);
            if constexpr (AX) d0 = psi_apply(p.et[4], sm.cc[10], q4, d0, true);
            if constexpr (AY) d1 = psi_apply(p.et[5], sm.cc[11], q5, d1, true);
            const float e = E0z[b] + sm.coef[2][(id >> 16) & 0xffu] * (d0 - d1);
            p.eout[2][o] = ((x0 && wx0) || (y0 && wy0)) ? 0.0f : e;
          }
        }
      };
      // Six straight variants, each inlined once: the interior with and
      // without the low faces, one absorbing axis (x, y or z), and every
      // tile-plane whose slabs span two or three axes (rare: edges and
      // corners) through the all-axes body; fewer bodies keep the hot code
      // small for the instruction cache.
      if constexpr (!Cpml) {
        if (xface || yface) body(kOff{}, kOff{}, kOff{}, kOn{});
        else body(kOff{}, kOff{}, kOff{}, kOff{});
      } else {
        const bool az = !(k >= p.cpml_inner[0][0] && k < p.cpml_inner[0][1]);
        const int v = (ax ? 4 : 0) | (ay ? 2 : 0) | (az ? 1 : 0);
        switch (v == 3 || v == 5 || v == 6 ? 7 : (v == 0 && !(xface || yface) ? 8 : v)) {
          case 8: body(kOff{}, kOff{}, kOff{}, kOff{}); break;
          case 0: body(kOff{}, kOff{}, kOff{}, kOn{}); break;
          case 1: body(kOff{}, kOff{}, kOn{}, kOn{}); break;
          case 2: body(kOff{}, kOn{}, kOff{}, kOn{}); break;
          case 4: body(kOn{}, kOff{}, kOff{}, kOn{}); break;
          default: body(kOn{}, kOn{}, kOn{}, kOn{}); break;
        }
      }
    } else {
      // ---- general tile ---------------------------------------------------
      const bool zZ = k < Z;
      const bool cpml = Cpml && (cpml_xy || !(k >= p.cpml_inner[0][0] && k < p.cpml_inner[0][1]));
      // One H cell at region (ly, lx) = lattice (k, j0-1+ly, i0-1+lx), box
      // column lx + 3.  `which`: bit 0 Hx, 1 Hy, 2 Hz.
      auto h_general = [&](int ly, int lx, bool own, int which) {
        const int j = j0 - 1 + ly, ii = i0 - 1 + lx, b = ly * BX + lx + 3;
        const int o = k * PL + j * P + ii;
        const bool yY = j >= 0 && j < Y, yY1 = j >= 0 && j <= Y;
        const bool iX = ii >= 0 && ii < X, iX1 = ii >= 0 && ii <= X;
        const float ez = E0z[b], ey = E0y[b], ex = E0x[b];
        if (which & 1) {  // Hx: dEz/dy - dEy/dz
          const bool ok = zZ && yY && iX1;
          CpmlOp c0, c1;
          if (cpml && ok) {
            c0 = cpml_fetch<1>(p.ht[0], sm.cc[0], cc_smem, k, j, ii);
            c1 = cpml_fetch<0>(p.ht[1], sm.cc[1], cc_smem, k, j, ii);
          }
          const float d0 = cpml_apply(p.ht[0], c0, div_rn(E0z[b + BX] - ez, res, inv_res), own);
          const float d1 = cpml_apply(p.ht[1], c1, div_rn(E1y[b] - ey, res, inv_res), own);
          float h = hf.dec0 * HOx[b] - hf.src0 * (d0 - d1);
          if (src) h = h_sources(p, sm.amp, 3, k, j, ii, h);
          if ((ii == 0 && wx0) || (ii == X && wx1)) h = 0.0f;
          sm.hn[hb][0][ly][lx] = h;
          if (own && ok) p.hout[0][o] = h;
        }
        if (which & 2) {  // Hy: dEx/dz - dEz/dx
          const bool ok = zZ && yY1 && iX;
          CpmlOp c0, c1;
          if (cpml && ok) {
            c0 = cpml_fetch<0>(p.ht[2], sm.cc[2], cc_smem, k, j, ii);
            c1 = cpml_fetch<2>(p.ht[3], sm.cc[3], cc_smem, k, j, ii);
          }
          const float d0 = cpml_apply(p.ht[2], c0, div_rn(E1x[b] - ex, res, inv_res), own);
          const float d1 = cpml_apply(p.ht[3], c1, div_rn(E0z[b + 1] - ez, res, inv_res), own);
          float h = hf.dec1 * HOy[b] - hf.src1 * (d0 - d1);
          if (src) h = h_sources(p, sm.amp, 4, k, j, ii, h);
          if ((j == 0 && wy0) || (j == Y && wy1)) h = 0.0f;
          sm.hn[hb][1][ly][lx] = h;
          if (own && ok) p.hout[1][o] = h;
        }
        if (which & 4) {  // Hz: dEy/dx - dEx/dy
          const bool ok = yY && iX;
          CpmlOp c0, c1;
          if (cpml && ok) {
            c0 = cpml_fetch<2>(p.ht[4], sm.cc[4], cc_smem, k, j, ii);
            c1 = cpml_fetch<1>(p.ht[5], sm.cc[5], cc_smem, k, j, ii);
          }
          const float d0 = cpml_apply(p.ht[4], c0, div_rn(E0y[b + 1] - ey, res, inv_res), own);
          const float d1 = cpml_apply(p.ht[5], c1, div_rn(E0x[b + BX] - ex, res, inv_res), own);
          float h = hf.dec2 * HOz[b] - hf.src2 * (d0 - d1);
          if (src) h = h_sources(p, sm.amp, 5, k, j, ii, h);
          if ((k == 0 && wz0) || (k == Z && wz1)) h = 0.0f;
          sm.hn[hb][2][ly][lx] = h;
          if (own && ok) p.hout[2][o] = h;
        }
      };
#pragma unroll
      for (int r = 0; r < R; ++r) h_general(1 + warp * R + r, 1 + lane, emit, 7);
      if (warp == 0) h_general(0, 1 + lane, false, 1 | 4);
      if (warp == 1 && lane < T::TY) h_general(1 + lane, 0, false, 2 | 4);
      if (xcol && warp == NW - 1 && lane <= T::TY) h_general(lane, T::TX + 1, emit && lane >= 1, 1);
      __syncthreads();
      // E of one cell at region (ly, lx) = lattice (k, j0-1+ly, i0-1+lx).
      auto e_general = [&](int ly, int lx, bool from_box) {
        const int j = j0 + ly - 1, i = i0 - 1 + lx, b = ly * BX + lx + 3;
        if (j > Y || i > X) return;
        const bool zlo = k == 0, zhi = k == Z;
        const bool xlo = i == 0, xhi = i == X;
        const int o = k * PL + j * P + i;
        const bool ylo = j == 0, yhi = j == Y;
          const float hx = sm.hn[hb][0][ly][lx], hy = sm.hn[hb][1][ly][lx], hz = sm.hn[hb][2][ly][lx];
          const float hz_y = sm.hn[hb][2][ly - 1][lx], hz_x = sm.hn[hb][2][ly][lx - 1];
          const float hy_z = sm.hn[pb][1][ly][lx], hy_x = sm.hn[hb][1][ly][lx - 1];
          const float hx_z = sm.hn[pb][0][ly][lx], hx_y = sm.hn[hb][0][ly - 1][lx];
          const uint32_t id = from_box ? IDS[(ly - 1) * T::TX + lx - 1] : p.em.site_ids[o];
          if (i < X) {  // Ex: dHz/dy - dHy/dz
            CpmlOp c0, c1;
            if (cpml) {
              c0 = cpml_fetch<1>(p.et[0], sm.cc[6], cc_smem, k, j, i);
              c1 = cpml_fetch<0>(p.et[1], sm.cc[7], cc_smem, k, j, i);
            }
            const float d0 = cpml_apply(p.et[0], c0, ghost(hz, hz_y, ylo, yhi, wy0, wy1, res, inv_res), true);
            const float d1 = cpml_apply(p.et[1], c1, ghost(hy, hy_z, zlo, zhi, wz0, wz1, res, inv_res), true);
            float e = E0x[b] + sm.coef[0][id & 0xffu] * (d0 - d1);
            if ((zlo && wz0) || (zhi && wz1) || (ylo && wy0) || (yhi && wy1)) e = 0.0f;
            p.eout[0][o] = e;
          }
          if (j < Y) {  // Ey: dHx/dz - dHz/dx
            CpmlOp c0, c1;
            if (cpml) {
              c0 = cpml_fetch<0>(p.et[2], sm.cc[8], cc_smem, k, j, i);
              c1 = cpml_fetch<2>(p.et[3], sm.cc[9], cc_smem, k, j, i);
            }
            const float d0 = cpml_apply(p.et[2], c0, ghost(hx, hx_z, zlo, zhi, wz0, wz1, res, inv_res), true);
            const float d1 = cpml_apply(p.et[3], c1, ghost(hz, hz_x, xlo, xhi, wx0, wx1, res, inv_res), true);
            float e = E0y[b] + sm.coef[1][(id >> 8) & 0xffu] * (d0 - d1);
            if ((zlo && wz0) || (zhi && wz1) || (xlo && wx0) || (xhi && wx1)) e = 0.0f;
            p.eout[1][o] = e;
          }
          if (zZ) {  // Ez: dHy/dx - dHx/dy
            CpmlOp c0, c1;
            if (cpml) {
              c0 = cpml_fetch<2>(p.et[4], sm.cc[10], cc_smem, k, j, i);
              c1 = cpml_fetch<1>(p.et[5], sm.cc[11], cc_smem, k, j, i);
            }
            const float d0 = cpml_apply(p.et[4], c0, ghost(hy, hy_x, xlo, xhi, wx0, wx1, res, inv_res), true);
            const float d1 = cpml_apply(p.et[5], c1, ghost(hx, hx_y, ylo, yhi, wy0, wy1, res, inv_res), true);
            float e = E0z[b] + sm.coef[2][(id >> 16) & 0xffu] * (d0 - d1);
            if ((ylo && wy0) || (yhi && wy1) || (xlo && wx0) || (xhi && wx1)) e = 0.0f;
            p.eout[2][o] = e;
          }
      };
      if (emit) {
#pragma unroll
        for (int r = 0; r < R; ++r) e_general(1 + warp * R + r, 1 + lane, true);
        if (xcol && warp == NW - 1 && lane < T::TY) e_general(1 + lane, T::TX + 1, false);
      }
    }
    e0 = e1;
    e1 = e1 == 2 ? 0 : e1 + 1;
    hs ^= 1;
  }
}

template <int NW, int R, bool Cpml>
cudaError_t launch_tma_t(cudaStream_t s, const TmaMaps& maps, const Step3D& p) {
  using T = TmaTile<NW, R>;
  const size_t smem = sizeof(typename T::Smem);
  auto kern = tma_step_kernel<NW, R, Cpml>;
  // The dynamic shared-memory limit is a per-device function attribute: set it
  // on every launch (cheap) rather than once per process.
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  const int kmax = p.Z + 1;
  const int zc = p.z_chunk > 0 ? p.z_chunk : kmax;
  // A multiple-of-32 X leaves column X to the last full tile (xcol).
  const int gx = p.X % T::TX == 0 ? p.X / T::TX : (p.X + T::TX) / T::TX;
  const dim3 grid(gx, (p.Y + 1 + T::TY - 1) / T::TY, (kmax + zc - 1) / zc);
  Step3D q = p;
  q.z_chunk = zc;
  kern<<<grid, dim3(32, NW, 1), smem, s>>>(maps, q);
  return cudaPeekAtLastError();
}

template <int NW, int R>
cudaError_t launch_tma_shape(cudaStream_t s, const Step3D& p) {
  using T = TmaTile<NW, R>;
  TmaMaps maps;
  const int64_t P = p.pitch, rowb = P * 4, planeb = static_cast<int64_t>(p.Y + 1) * P * 4;
  for (int c = 0; c < 3; ++c) {
    const Dims de = component_dims(c, p.Z, p.Y, p.X), dh = component_dims(c + 3, p.Z, p.Y, p.X);
    if (!encode(&maps.e[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.ein[c], de.x, de.y, de.z, rowb, planeb, T::BX, T::EH) ||
        !encode(&maps.h[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.hin[c], dh.x, dh.y, dh.z, rowb, planeb, T::BX, T::HH))
      return cudaErrorInvalidValue;
  }
  if (!encode(&maps.ids, CU_TENSOR_MAP_DATA_TYPE_UINT32, p.em.site_ids, p.X + 1, p.Y + 1, p.Z + 1, rowb, planeb,
              T::TX, T::TY))
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
    default: return launch_tma_shape<8, 1>(s, p);
  }
}

}  // namespace fdtd
