// The class step: one launch per 3D leapfrog step on the pitched field layout,
// with the E material as one uint8 class per lattice point
// (FDTD_FLAG_CLASSES).  The engine's 3D hot path.
//
// Same schedule as the codebook kernel in fused_tma.cu (z-marching CTAs,
// TMA-staged planes on an mbarrier ring, a recomputed H halo so that no CTA
// waits on another), re-shaped so that a thread updates four cells per plane
// instead of one:
//
//  * a CTA of NW warps owns a 128 x NW tile of (x, y) lattice points; lane l of
//    warp w owns x = i0 + 4l .. 4l + 3 on row j = j0 + w, so every shared and
//    global access of a cell group is one 16-byte vector;
//  * x neighbours come from the adjacent lane by shuffle (the tile edges from
//    the staged box); the y neighbour of the H update is the next staged row,
//    that of the E update the row above in the new-H plane; H of the previous
//    plane stays in registers;
//  * the E material is one uint8 class id per lattice point (a class is one
//    (Ex, Ey, Ez) coefficient triple of the codebook), 1 byte per cell instead
//    of a 4-byte codebook word, with the class table in shared memory;
//  * the CPML recurrences of a row's x-slab cells are shared by the row's warp
//    (one cell per lane) instead of falling on the few lanes that own them;
//    their psi rows ride in the plane's TMA bundle (a 16-slot window per x
//    term), so an x-slab tile never waits on a psi load; the y / z terms' psi
//    loads of a plane are all issued at its top;
//  * CTAs are dispatched longest first (absorber tile rows, then absorber z
//    chunks, then the interior), so that the last wave is not absorber-heavy.
//
// Arithmetic: beamz's float32 order bit for bit (every difference divided by
// the cell size with a correctly rounded quotient, every product and sum
// rounded separately; this file is compiled with -fmad=false).  With
// FDTD_FLAG_FAST_MATH instead the tolerance form: 1/dx folded into the
// coefficients (dt/(mu0 dx) for H, dt/(eps0 eps dx) per class for E, a/dx for
// the CPML) and explicit fused multiply-adds.
//
// The tiles end at x = X - 1 (a partial last tile masks its stores past X)
// and the lattice column x = X is a small column kernel's, run before the
// step.  Tile-planes that touch a z face or an H source run a general
// per-cell path with every validity, ghost and PEC rule; the rest run
// a straight body compiled for their case: the interior, the x = 0 / y = 0
// faces, the x-slab tiles (about half of them on a 512-wide grid), the other
// absorber tiles (axes as plane-uniform run-time flags), and the last tile
// row, shifted down to end at row Y (where Hx, Hz and Ey do not exist and the
// y = Y ghost applies) with its rows below the tile row before computed but
// not stored.  The H-term CPML memories are double-banked (the halo
// recomputation reads them), the E-term ones updated in place.
//
// Operation order follows beamz/simulation/kernels.py:458-626 (H from E with
// CPML, H sources, H PEC; E from ghost-padded H with CPML, E PEC) and
// beamz/simulation/execute.py:467-522.

#include <cuda.h>

#include <algorithm>
#include <type_traits>

#include "kernels.cuh"
#include "tma_util.cuh"

namespace fdtd {

namespace {

constexpr int kSlots = 32;  // CPML coefficient slots staged per term
constexpr unsigned kFull = 0xffffffffu;

// Lossy: conductive material (FDTD_FLAG_LOSSY) -- per-class (decay, source)
// pairs for E and H classes, the H classes staged with the halo; no x-psi
// staging (its room holds the H classes).
template <int NW, bool Lossy = false>
struct ClassTile {
  static constexpr int TX = 128, TY = NW, NT = 32 * NW;
  static constexpr int BX = TX + 8;  // staged row: x from i0-4 to i0+131 (16-byte aligned start)
  static constexpr int EH = TY + 2;  // E rows j0-1 .. j0+TY
  static constexpr int HH = TY + 1;  // H rows j0-1 .. j0+TY-1
  static constexpr int EBOX = ((EH * BX + 31) / 32) * 32;  // floats; every box starts on 128 B
  static constexpr int HBOX = ((HH * BX + 31) / 32) * 32;
  static constexpr int IBOX = TY * TX;  // class ids (bytes), rows j0 .. j0+TY-1, x i0 .. i0+127
  static constexpr int XW = 16;         // staged x-psi window (slots)
  static constexpr int XPS = ((HH * XW + 31) / 32) * 32;
  // Lossy: H-class box, rows j0-1 .. j0+TY-1, x from i0-16 (a 16-byte
  // coordinate for 1-byte elements) to i0+127: the own cells and the halo.
  static constexpr int HW = TX + 16;
  static constexpr int HIBYTES = HH * HW;
  static constexpr int HIBOX = ((HIBYTES + 127) / 128) * 128;
  struct Smem {
    alignas(128) float e[3][3][EBOX];  // E ring: plane slot, component (TMA boxes start on 128 B)
    alignas(128) float h[2][3][HBOX];  // H (old) ring
    alignas(128) uint8_t ids[2][IBOX];
    alignas(16) float hn[3][HH][BX];   // H (new) of this plane: own rows + halo row, own columns + halo column
    float4 cls[256];  // per class: dt/(eps0 eps dx) of Ex, Ey, Ez; Lossy: [128][4] (decay, source) float2
    float4 cc[12][kSlots];  // CPML (a, b, 1/kappa) (a/dx in the tolerance form): H terms 0-5, E terms 6-11
    float xd[2][TY][32];    // corrected x differences of a row's x-slab cells by slot (compact x work)
    // x-term psi (Hyx, Hzx, Eyx, Ezx) of the bundle's plane, staged with it:
    // rows j0-1 .. j0+TY-1, a 16-slot window of the tile's slab run.
    alignas(128) float xps[Lossy ? 1 : 2][4][Lossy ? 32 : XPS];
    alignas(128) uint8_t hids[Lossy ? 2 : 1][Lossy ? HIBOX : 128];  // Lossy: H classes by plane parity
    float2 hcls[Lossy ? 64 * 4 : 1];  // Lossy: [64][4] (decay, source) of Hx, Hy, Hz
    int xwin[4];            // each term's window start (slot)
    int xst[8][32];         // per lane: x-slab masks xs3, xs4, xe3, xe4 and compact items h0, h1, e0, e1
    float hcoef[6];         // uniform H decay (Hx, Hy, Hz) and source (over dx in the tolerance form)
    float amp[kMaxFusedSources];
    unsigned long long bar[2];
  };
  // Every TMA destination starts on 128 bytes; two 8-warp CTAs fit an SM
  // (228 KB less 1 KB reserved per CTA).
  static_assert((EBOX * 4) % 128 == 0 && (HBOX * 4) % 128 == 0 && IBOX % 128 == 0 && (XPS * 4) % 128 == 0 &&
                    HIBOX % 128 == 0,
                "TMA ring slots keep 128-byte alignment");
  static_assert(NW != 8 || sizeof(Smem) <= 233472 / 2 - 1024, "8-warp class step: two CTAs per SM");
};

struct ClassMaps {
  CUtensorMap e[3];
  CUtensorMap h[3];
  CUtensorMap ids;
  CUtensorMap hids;  // Lossy: H classes
  CUtensorMap xpsi[4];  // x-term psi slabs (Hyx, Hzx, Eyx, Ezx), when Step3D::xstage
};

// CTA dispatch order, longest first: the CTAs of the absorber tile rows (every
// z chunk), then the absorber z chunks of the other rows, then the rest, each
// group x fastest.  Absorber CTAs take two to three times as long as interior
// ones, so in launch order the last wave would otherwise be absorber-heavy
// (the high z slab's chunks) and leave SMs idle at the end of the step.
struct TileIdx {
  int x, y, z;
};
__device__ __forceinline__ TileIdx tile_of(int L, int gx, int gy, int gz, const int* ord) {
  const int ylo = ord[0], yhi = ord[1], zlo = ord[2], zhi = ord[3];
  const int nys = ylo + (gy - yhi), nzs = zlo + (gz - zhi), nyi = gy - nys;
  TileIdx t;
  t.x = L % gx;
  int q = L / gx;
  auto row = [&](int r, bool shell) { return shell ? (r < ylo ? r : yhi + r - ylo) : ylo + r; };
  auto chunk = [&](int c, bool shell) { return shell ? (c < zlo ? c : zhi + c - zlo) : zlo + c; };
  if (q < nys * gz) {
    t.y = row(q % nys, true);
    t.z = q / nys;
    return t;
  }
  q -= nys * gz;
  if (q < nyi * nzs) {
    t.y = row(q % nyi, false);
    t.z = chunk(q / nyi, true);
    return t;
  }
  q -= nyi * nzs;
  t.y = row(q % nyi, false);
  t.z = chunk(q / nyi, false);
  return t;
}

// ---- float4 helpers ----------------------------------------------------------
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
// The first `nv` of four cells (all four: one 16-byte store).
__device__ __forceinline__ void st4m(float* p, float4 v, int nv) {
  if (nv >= 4) {
    st4(p, v);
    return;
  }
  if (nv > 0) p[0] = v.x;
  if (nv > 1) p[1] = v.y;
  if (nv > 2) p[2] = v.z;
}
__device__ __forceinline__ float4 sub4(float4 a, float4 b) {
  return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
// (v.y, v.z, v.w, n): the x+1 neighbours of a lane's four cells.
__device__ __forceinline__ float4 next4(float4 v, float n) { return make_float4(v.y, v.z, v.w, n); }
// (p, v.x, v.y, v.z): the x-1 neighbours.
__device__ __forceinline__ float4 prev4(float p, float4 v) { return make_float4(p, v.x, v.y, v.z); }
__device__ __forceinline__ float get(const float4& v, int q) { return q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w)); }

// ---- arithmetic ------------------------------------------------------------
// Exact: beamz's float32 order (kernels.py:458-626): every difference divided
// by the cell size (correctly rounded, div_rn), every product and sum rounded
// separately (this file is compiled with -fmad=false).  Otherwise the
// tolerance form: differences left unscaled (1/dx folded into the
// coefficients) and explicit fused multiply-adds.
template <bool Exact>
__device__ __forceinline__ float dv(float diff, float bs, float rs) {
  if constexpr (Exact) return div_rn(diff, bs, rs);
  return diff;
}

template <bool Exact>
__device__ __forceinline__ float4 dv4(float4 d, float bs, float rs) {
  return make_float4(dv<Exact>(d.x, bs, rs), dv<Exact>(d.y, bs, rs), dv<Exact>(d.z, bs, rs), dv<Exact>(d.w, bs, rs));
}

// H <- dec H - s (d0 - d1).
template <bool Exact>
__device__ __forceinline__ float h1(float h, float dec, float s, float d0, float d1) {
  if constexpr (Exact) return dec * h - s * (d0 - d1);
  return fmaf(-s, d0 - d1, dec * h);
}

template <bool Exact>
__device__ __forceinline__ float4 h4(float4 h, float dec, float s, float4 d0, float4 d1) {
  return make_float4(h1<Exact>(h.x, dec, s, d0.x, d1.x), h1<Exact>(h.y, dec, s, d0.y, d1.y),
                     h1<Exact>(h.z, dec, s, d0.z, d1.z), h1<Exact>(h.w, dec, s, d0.w, d1.w));
}

// E <- E + c (d0 - d1).
template <bool Exact>
__device__ __forceinline__ float e_upd(float e, float c, float d0, float d1) {
  if constexpr (Exact) return e + c * (d0 - d1);
  return fmaf(c, d0 - d1, e);
}

// Conductive material (FDTD_FLAG_LOSSY): per-class (decay, source) pairs,
// tab[class * 4 + component].  E <- decay E + source (d0 - d1), beamz's
// per-site form (the dense kernels' e_update); H as h1.
template <bool Exact>
__device__ __forceinline__ float e_loss(float e, float2 c, float d0, float d1) {
  if constexpr (Exact) return c.x * e + c.y * (d0 - d1);
  return fmaf(c.y, d0 - d1, c.x * e);
}

// Four cells whose classes are the bytes of `ids4`, component n.
// E classes are at most 128, H classes at most 64 (the ids are masked so that
// no byte can read past a table).
constexpr unsigned kEClassMask = 127u, kHClassMask = 63u;

template <bool Exact>
__device__ __forceinline__ float4 e4_loss(float4 e, const float2* tab, uint32_t ids4, int n, float4 d0, float4 d1) {
  return make_float4(e_loss<Exact>(e.x, tab[(ids4 & kEClassMask) * 4 + n], d0.x, d1.x),
                     e_loss<Exact>(e.y, tab[((ids4 >> 8) & kEClassMask) * 4 + n], d0.y, d1.y),
                     e_loss<Exact>(e.z, tab[((ids4 >> 16) & kEClassMask) * 4 + n], d0.z, d1.z),
                     e_loss<Exact>(e.w, tab[((ids4 >> 24) & kEClassMask) * 4 + n], d0.w, d1.w));
}

template <bool Exact>
__device__ __forceinline__ float4 h4_loss(float4 h, const float2* tab, uint32_t ids4, int n, float4 d0, float4 d1) {
  const float2 c0 = tab[(ids4 & kHClassMask) * 4 + n], c1 = tab[((ids4 >> 8) & kHClassMask) * 4 + n];
  const float2 c2 = tab[((ids4 >> 16) & kHClassMask) * 4 + n], c3 = tab[((ids4 >> 24) & kHClassMask) * 4 + n];
  return make_float4(h1<Exact>(h.x, c0.x, c0.y, d0.x, d1.x), h1<Exact>(h.y, c1.x, c1.y, d0.y, d1.y),
                     h1<Exact>(h.z, c2.x, c2.y, d0.z, d1.z), h1<Exact>(h.w, c3.x, c3.y, d0.w, d1.w));
}

// ---- CPML --------------------------------------------------------------------
// psi <- b psi + a d and the corrected derivative d' = d / kappa + psi
// (beamz/simulation/kernels.py:257-264), c = (a, b, 1/kappa).  In the
// tolerance form d is the raw difference D = d dx, `a` is staged as a/dx and
// the result is scaled by dx (D' = D/kappa + dx psi), so the update's
// coefficient over dx applies to D' as to a plain difference.
template <bool Exact>
__device__ __forceinline__ float cpml_d(float4 c, float res, float psi_old, float d, float* psi_new) {
  if constexpr (Exact) {
    const float psi = c.y * psi_old + c.x * d;
    *psi_new = psi;
    return d * c.z + psi;
  }
  const float psi = fmaf(c.y, psi_old, c.x * d);
  *psi_new = psi;
  return fmaf(c.z, d, res * psi);
}

// Packed slab coordinate, -1 outside (fdtd_common.cuh's cpml_slot).
__device__ __forceinline__ int slot_of(const CpmlTermDev& t, int coord) { return cpml_slot(t, coord); }

// Offset of (k, j, i) in a term's packed slab, with the term axis coordinate
// replaced by `slot`.
template <int Axis>
__device__ __forceinline__ int psi_off(const CpmlTermDev& t, int slot, int k, int j, int i) {
  const int pk = Axis == 0 ? slot : k;
  const int pj = Axis == 1 ? slot : j;
  const int pi = Axis == 2 ? slot : i;
  return (pk * t.pdy + pj) * t.pdx + pi;  // slabs hold < 2^31 elements (validated)
}

// A term whose slot is uniform over a lane's four cells (y terms on a row, z
// terms on a plane): psi of the four cells is fetched ahead of its use (the
// offset is recomputed when applying, to keep registers free).
// `nv`: how many of the lane's four cells lie before x = X (a partial last
// tile stores nothing, and loads no psi, past it).
template <int Axis>
__device__ __forceinline__ float4 psi4_fetch(const CpmlTermDev& t, int slot, int k, int j, int i, int nv) {
  if (slot < 0) return make_float4(0.f, 0.f, 0.f, 0.f);
  const float* s = t.psi_in + psi_off<Axis>(t, slot, k, j, i);
  if (nv >= 4) return make_float4(s[0], s[1], s[2], s[3]);
  return make_float4(nv > 0 ? s[0] : 0.f, nv > 1 ? s[1] : 0.f, nv > 2 ? s[2] : 0.f, 0.f);
}

template <bool Exact, int Axis>
__device__ __forceinline__ float4 psi4_apply(const CpmlTermDev& t, const float4* cc, int slot, float4 v, int k, int j,
                                             int i, float res, float4 d, bool write, int nv) {
  if (slot < 0) return d;
  const float4 c = cc[slot];
  float4 n;
  float4 r;
  r.x = cpml_d<Exact>(c, res, v.x, d.x, &n.x);
  r.y = cpml_d<Exact>(c, res, v.y, d.y, &n.y);
  r.z = cpml_d<Exact>(c, res, v.z, d.z, &n.z);
  r.w = cpml_d<Exact>(c, res, v.w, d.w, &n.w);
  if (write) {
    float* o = t.psi_out + psi_off<Axis>(t, slot, k, j, i);
    if (nv > 0) o[0] = n.x;
    if (nv > 1) o[1] = n.y;
    if (nv > 2) o[2] = n.z;
    if (nv > 3) o[3] = n.w;
  }
  return r;
}

// An x term on a lane's four cells: which cells lie in the term's slab (bits
// 0-3) and the slot of cell 0, packed as mask | slot0 << 4; the slots of a
// contiguous slab are consecutive.  Tile-constant, so computed once per CTA.
__device__ __forceinline__ int xslab_of(const CpmlTermDev& t, int i) {
  int mask = 0, base = 0;
#pragma unroll
  for (int c = 3; c >= 0; --c) {
    const int slot = slot_of(t, i + c);
    if (slot >= 0) {
      mask |= 1 << c;
      base = slot - c;
    }
  }
  return mask | (base << 4);
}

// psi of an x term on the own cells of row (k, j): the row offset of slot 0.
__device__ __forceinline__ int xrow(const CpmlTermDev& t, int xs, int k, int j) {
  return (k * t.pdy + j) * t.pdx + (xs >> 4);
}

__device__ __forceinline__ float4 psix_fetch(const CpmlTermDev& t, int xs, int k, int j) {
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  if (xs & 15) {
    const float* row = t.psi_in + xrow(t, xs, k, j);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (xs & (1 << c)) v[c] = row[c];
  }
  return make_float4(v[0], v[1], v[2], v[3]);
}

template <bool Exact>
__device__ __forceinline__ float4 psix_apply(const CpmlTermDev& t, const float4* cc, int xs, float4 v, int k, int j,
                                             float res, float4 d, bool write) {
  if (!(xs & 15)) return d;
  float r[4] = {d.x, d.y, d.z, d.w};
  const float pv[4] = {v.x, v.y, v.z, v.w};
  const int base = xs >> 4;
  float* row = t.psi_out + xrow(t, xs, k, j);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (!(xs & (1 << c))) continue;
    float n;
    r[c] = cpml_d<Exact>(cc[base + c], res, pv[c], r[c], &n);
    if (write) row[c] = n;
  }
  return make_float4(r[0], r[1], r[2], r[3]);
}

// The own cells' x differences with the slab cells replaced by their corrected
// values from the compact x work (`slots`: the row's corrected differences by
// slab slot; the slots of the own cells are consecutive from xs >> 4).
__device__ __forceinline__ float4 xtake(float4 d, int xs, const float* slots) {
  if (!(xs & 15)) return d;
  float r[4] = {d.x, d.y, d.z, d.w};
  const int base = xs >> 4;
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (xs & (1 << c)) r[c] = slots[base + c];
  return make_float4(r[0], r[1], r[2], r[3]);
}

// The compact x work's items of one x term in a tile: its slab slots whose x
// lies in [i0, i1) (at most two runs: the low and the high slab).  Item q maps
// to a slot and an x; returns false past the last item.
struct XItems {
  int lo_n, hi_s, hi_n, hi_x;  // low run: slots [0.., lo_n) at x = slot + lo_x0
  int lo_s, lo_x;
  __device__ __forceinline__ bool item(int q, int* slot, int* x) const {
    if (q < lo_n) {
      *slot = lo_s + q;
      *x = lo_x + q;
      return true;
    }
    q -= lo_n;
    if (q < hi_n) {
      *slot = hi_s + q;
      *x = hi_x + q;
      return true;
    }
    return false;
  }
};

__device__ __forceinline__ XItems x_items(const CpmlTermDev& t, int i0, int i1) {
  XItems r{};
  // low slab: x = slot in [0, low)
  const int lb = max(0, i0), le = min(t.low, i1);
  r.lo_n = max(0, le - lb);
  r.lo_s = lb;
  r.lo_x = lb;
  // high slab: x in [n - high, n), slot = low + x - (n - high)
  const int hx0 = t.n_axis - t.high;
  const int hb = max(hx0, i0), he = min(t.n_axis, i1);
  r.hi_n = t.high > 0 ? max(0, he - hb) : 0;
  r.hi_s = t.low + hb - hx0;
  r.hi_x = hb;
  return r;
}

// One scalar cell of a term: psi fetched ahead (0 outside the slab), then applied.
template <int Axis>
__device__ __forceinline__ float psi1_fetch(const CpmlTermDev& t, int k, int j, int i) {
  const int slot = slot_of(t, Axis == 0 ? k : (Axis == 1 ? j : i));
  return slot >= 0 ? t.psi_in[psi_off<Axis>(t, slot, k, j, i)] : 0.0f;
}

template <bool Exact, int Axis>
__device__ __forceinline__ float psi1_apply(const CpmlTermDev& t, const float4* cc, float v, int k, int j, int i,
                                            float res, float d, bool write) {
  const int slot = slot_of(t, Axis == 0 ? k : (Axis == 1 ? j : i));
  if (slot < 0) return d;
  float n;
  const float r = cpml_d<Exact>(cc[slot], res, v, d, &n);
  if (write) t.psi_out[psi_off<Axis>(t, slot, k, j, i)] = n;
  return r;
}

// One scalar cell of a term fetched and applied at once (general path).
template <bool Exact, int Axis>
__device__ __forceinline__ float cpml1(const CpmlTermDev& t, const float4* cc, bool cc_smem, float res, int k, int j,
                                       int i, float d, bool write) {
  const int coord = Axis == 0 ? k : (Axis == 1 ? j : i);
  const int slot = slot_of(t, coord);
  if (slot < 0) return d;
  const int off = psi_off<Axis>(t, slot, k, j, i);
  const float a = Exact ? __ldg(t.a + slot) : __ldg(t.a + slot) * (1.0f / res);
  const float4 c = cc_smem ? cc[slot] : make_float4(a, __ldg(t.b + slot), __ldg(t.k + slot), 0.0f);
  float n;
  const float r = cpml_d<Exact>(c, res, t.psi_in[off], d, &n);
  if (write) t.psi_out[off] = n;
  return r;
}

__device__ __forceinline__ float h_sources_at(const Step3D& p, const float* amp, int c, int k, int j, int i, float h) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    const int z = k - src.z0, y = j - src.y0, x = i - src.x0;
    if (src.component != c || z < 0 || y < 0 || x < 0 || z >= src.ez || y >= src.ey || x >= src.ex) continue;
    h = h + src.coeff[(static_cast<int64_t>(z) * src.ey + y) * src.ex + x] * amp[s];
  }
  return h;
}

__device__ __forceinline__ bool sources_touch(const Step3D& p, int k, int jlo, int jhi, int ilo, int ihi) {
  for (int s = 0; s < p.n_hsrc; ++s) {
    const SourceDev& src = p.hsrc[s];
    if (k >= src.z0 && k < src.z0 + src.ez && jhi >= src.y0 && jlo < src.y0 + src.ey && ihi >= src.x0 &&
        ilo < src.x0 + src.ex)
      return true;
  }
  return false;
}

// Ghost-padded backward difference along one axis at E coordinate v of an
// axis with n H samples (beamz/lattice.py:523-551): beyond a metallic wall the
// ghost is zero, else a copy of the edge sample (the difference vanishes).
__device__ __forceinline__ float ghost_diff(float center, float below, int v, int n, bool low_wall, bool high_wall) {
  if (v == 0) return low_wall ? center : 0.0f;
  if (v == n) return high_wall ? 0.0f - below : 0.0f;
  return center - below;
}

// 8-warp CTAs: two per SM (shared memory), 128 registers; 4-warp CTAs: four.
// Partial: X is not a multiple of 128 (the last tile is partial); only then
// do the run-time bodies carry the per-lane store masks.
template <int NW, bool Cpml, bool Exact, bool Lossy, bool Partial, bool Metric>
__global__ void __launch_bounds__(32 * NW, NW == 8 ? 2 : 4)
    class_step_kernel(const __grid_constant__ ClassMaps maps, const __grid_constant__ Step3D p) {
  using T = ClassTile<NW, Lossy>;
  using S = typename T::Smem;
  constexpr int BX = T::BX, TX = T::TX, TY = T::TY;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S& sm = *reinterpret_cast<S*>(smem_raw);
  const int lane = threadIdx.x, warp = threadIdx.y;
  const int tid = warp * 32 + lane;
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int gx = (X + TX - 1) / TX, gy = (Y + TY) / TY, gz = (Z + p.z_chunk) / p.z_chunk;
  const TileIdx tile = tile_of(blockIdx.x, gx, gy, gz, p.order);
  // The last tile row, when it would hold rows past Y, is shifted down to
  // end at row Y (j0 = Y + 1 - TY) so that it runs a straight body; its rows
  // below jown belong to the tile row before and are computed, not stored.
  const int jown = tile.y * TY;
  const bool ylast = jown + TY > Y && Y + 1 >= TY;
  const int i0 = tile.x * TX, j0 = ylast ? Y + 1 - TY : jown;
  const int k0 = tile.z * p.z_chunk;
  const int k1 = min(k0 + p.z_chunk, Z + 1);
  const int kstart = k0 > 0 ? k0 - 1 : 0;
  const int P = p.pitch, PL = (Y + 1) * p.pitch;
  const float res = p.res, inv_res = p.inv_res;
  const unsigned long long wait_ns = p.wait_ns;

  // The tiles end at x = X - 1 -- the last one partial when X is not a
  // multiple of 128, its lanes past X storing nothing (nv below) -- and column
  // X (Hx, Ey, Ez there) is the column kernel's, launched before this one.
  const int i1 = min(i0 + TX, X);  // the tile's columns end here (a partial last tile before i0 + 128)
  const bool ax = Cpml && !(i0 - 1 >= p.cpml_inner[2][0] && i1 <= p.cpml_inner[2][1]);
  // Compact x work: in a tile that touches an x slab, the recurrences of a
  // row's x-slab cells are shared by the row's warp -- each lane takes items
  // lane and lane + 32 of the row's (term, slot) list, the first x term's
  // slots (Hyx, Eyx), then the second's (Hzx, Ezx) -- instead of falling on
  // the few lanes that own slab cells; the corrected differences reach the
  // owners through shared memory.  It covers slabs of at most 32 slots per
  // term (wider ones take the general path).
  const bool xcompact = ax && p.ht[3].low + p.ht[3].high <= 32 && p.ht[4].low + p.ht[4].high <= 32 &&
                        p.et[3].low + p.et[3].high <= 32 && p.et[4].low + p.et[4].high <= 32;
  // The x terms' psi rides in the plane's bundle when each term's run of
  // slots in this tile fits one 16-slot window starting on a multiple of 4
  // (16-byte TMA coordinate); otherwise the x work loads it directly.
  int xwin[4] = {0, 0, 0, 0};
  bool xstage = xcompact && p.xstage && !Lossy;
  if (xstage) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const XItems a = x_items(t < 2 ? p.ht[3 + t] : p.et[1 + t], i0, i1);
      if (a.lo_n + a.hi_n == 0) continue;
      const int first = a.lo_n > 0 ? a.lo_s : a.hi_s;
      const int last = a.hi_n > 0 ? a.hi_s + a.hi_n - 1 : a.lo_s + a.lo_n - 1;
      xwin[t] = first & ~3;
      if (last - xwin[t] >= T::XW) xstage = false;
    }
  }

  // Bundle q: E(q+1) (and E(q) when `first`), H(q), class ids(q), and the x
  // terms' psi of plane q.  x starts at i0 - 4 (fields), i0 (ids) or a
  // multiple of 4 (psi): 16-byte aligned.
  auto issue = [&](int q, int slot, bool first) {
    const int ne = (first ? 1 : 0) + (q + 1 <= Z ? 1 : 0);
    const unsigned bytes =
        ne * 3 * T::EH * BX * 4 + 3 * T::HH * BX * 4 + T::IBOX + (xstage ? 4 * T::XW * T::HH * 4 : 0) +
        (Lossy ? T::HIBYTES : 0);
    unsigned long long* b = &sm.bar[slot];
    tma::bar_expect(b, bytes);
    if (p.test_stall) return;  // test-only: the barrier is armed, no copy is issued, nothing is in flight
    if (first)
      for (int c = 0; c < 3; ++c) tma::load_3d(sm.e[q % 3][c], &maps.e[c], i0 - 4, j0 - 1, q, b);
    if (q + 1 <= Z)
      for (int c = 0; c < 3; ++c) tma::load_3d(sm.e[(q + 1) % 3][c], &maps.e[c], i0 - 4, j0 - 1, q + 1, b);
    for (int c = 0; c < 3; ++c) tma::load_3d(sm.h[q % 2][c], &maps.h[c], i0 - 4, j0 - 1, q, b);
    tma::load_3d(sm.ids[q % 2], &maps.ids, i0, j0, q, b);
    if constexpr (Lossy) tma::load_3d(sm.hids[q % 2], &maps.hids, i0 - 16, j0 - 1, q, b);
    if (xstage) {
#pragma unroll
      for (int t = 0; t < 4; ++t) tma::load_3d(sm.xps[q % 2][t], &maps.xpsi[t], xwin[t], j0 - 1, q, b);
    }
  };

  if (tid == 0) {
#pragma unroll
    for (int t = 0; t < 4; ++t) sm.xwin[t] = xwin[t];
    tma::bar_init(&sm.bar[0], 1);
    tma::bar_init(&sm.bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    issue(kstart, 0, true);
  }
  for (int e = tid; e < 256; e += T::NT) sm.cls[e] = p.class_coef[e];
  if constexpr (Lossy)
    for (int e = tid; e < 64 * 4; e += T::NT) sm.hcls[e] = p.h_class_coef[e];
  bool cc_smem = true;
  if (Cpml) {
#pragma unroll
    for (int t = 0; t < 12; ++t) {
      const CpmlTermDev& d = t < 6 ? p.ht[t] : p.et[t - 6];
      const int w = d.low + d.high;
      cc_smem = cc_smem && w <= kSlots;
      for (int e = tid; e < w && e < kSlots; e += T::NT)
        sm.cc[t][e] = make_float4(Exact ? d.a[e] : d.a[e] * inv_res, d.b[e], d.k[e], 0.0f);
    }
  }
  if (tid < p.n_hsrc) sm.amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);
  // The uniform H coefficients live in shared memory (read where used) rather
  // than in six registers for the whole kernel.  The tolerance form folds 1/dx
  // into the source (the class table carries E's).
  if (tid < 3) {
    sm.hcoef[tid] = p.hm.decay[tid][0];
    sm.hcoef[3 + tid] = p.hm.source[tid][0] * (Exact ? 1.0f : inv_res);
  }
  __syncthreads();

  const bool wz0 = wall(p.metallic, 0, false), wz1 = wall(p.metallic, 0, true);
  const bool wy0 = wall(p.metallic, 1, false), wy1 = wall(p.metallic, 1, true);
  const bool wx0 = wall(p.metallic, 2, false), wx1 = wall(p.metallic, 2, true);
  // Uniform H coefficients (the pitched layout carries no per-site H).

  const float dbs = p.div_bs, drs = p.div_rs;  // div_rn's scaled cell size and reciprocal
  auto D1 = [&](float v) { return dv<Exact>(v, dbs, drs); };
  auto D4 = [&](float4 v) { return dv4<Exact>(v, dbs, drs); };
  // Derivatives along an axis at a coordinate: with Metric (axis-uniform and
  // rectilinear grids, 3D: every axis carries one) the difference times the
  // inverse distance there (beamz/simulation/kernels.py:164-176, 293-323),
  // forward differences (feeding H) on metric_h at 0..n-1, backward ones
  // (feeding E) on metric_e at 0..n; halo coordinates that are never stored
  // are clamped into the arrays.  Otherwise D1 / D4.  MH4 / ME4 take four
  // cells on one coordinate (z or y), MH4x / ME4x the four x cells from c.
  auto MH = [&](float v, int axis, int c) -> float {
    if constexpr (Metric) return v * p.metric_h[axis][clampi(c, axis_cells(p, axis) - 1)];
    else return D1(v);
  };
  auto ME = [&](float v, int axis, int c) -> float {
    if constexpr (Metric) return v * p.metric_e[axis][clampi(c, axis_cells(p, axis))];
    else return D1(v);
  };
  auto MH4 = [&](float4 v, int axis, int c) -> float4 {
    if constexpr (Metric) {
      const float m = p.metric_h[axis][clampi(c, axis_cells(p, axis) - 1)];
      return make_float4(v.x * m, v.y * m, v.z * m, v.w * m);
    } else {
      return D4(v);
    }
  };
  auto ME4 = [&](float4 v, int axis, int c) -> float4 {
    if constexpr (Metric) {
      const float m = p.metric_e[axis][clampi(c, axis_cells(p, axis))];
      return make_float4(v.x * m, v.y * m, v.z * m, v.w * m);
    } else {
      return D4(v);
    }
  };
  auto MH4x = [&](float4 v, int c) -> float4 {
    if constexpr (Metric) {
      const float* m = p.metric_h[2];
      const int hi = X - 1;
      return make_float4(v.x * m[clampi(c, hi)], v.y * m[clampi(c + 1, hi)], v.z * m[clampi(c + 2, hi)],
                         v.w * m[clampi(c + 3, hi)]);
    } else {
      return D4(v);
    }
  };
  auto ME4x = [&](float4 v, int c) -> float4 {
    if constexpr (Metric) {
      const float* m = p.metric_e[2];
      return make_float4(v.x * m[clampi(c, X)], v.y * m[clampi(c + 1, X)], v.z * m[clampi(c + 2, X)],
                         v.w * m[clampi(c + 3, X)]);
    } else {
      return D4(v);
    }
  };

  const int r = 1 + warp;              // own row in the staged boxes and hn
  const int j = j0 + warp;             // its lattice row
  const int c0 = 4 + 4 * lane;         // own first column in the boxes and hn
  const int i = i0 + 4 * lane;         // its lattice x
  const int rc = r * BX + c0;
  const bool fast_ok0 = (j0 + TY <= Y || ylast) && cc_smem;
  const int nv = min(max(X - i, 0), 4);  // own cells before x = X (a partial last tile)
  const bool own = j >= jown;  // this warp's row is the tile's to store
  const bool xface = i0 == 0, yface = j0 == 0;
  const bool ay = Cpml && !(j0 - 1 >= p.cpml_inner[1][0] && j0 + TY <= p.cpml_inner[1][1]);
  const bool fast_ok = fast_ok0 && (!ax || xcompact);
  const bool shell_x = ax, shell_y = ay;  // the tile's absorber axes (z is per plane)

  // Tile-constant x state per lane, in shared memory so that it holds no
  // register outside the x work: the x-slab masks of the own cells for Hyx,
  // Hzx, Eyx, Ezx (xslab_of) and the lane's compact items, packed as valid |
  // second term << 1 | slot << 2 | (x - i0) << 8 (items lane and lane + 32 of
  // the H terms' list, then of the E terms').  The items stop at the tile's
  // last column (column X is the column kernel's).
  if (xcompact && warp == 0) {
    auto pack = [&](const CpmlTermDev& t3, const CpmlTermDev& t4, int q) {
      const XItems a3 = x_items(t3, i0, i1), a4 = x_items(t4, i0, i1);
      const int n3 = a3.lo_n + a3.hi_n;
      const bool second = q >= n3;
      int slot = 0, x = 0;
      if (!(second ? a4 : a3).item(second ? q - n3 : q, &slot, &x)) return 0;
      return 1 | (second ? 2 : 0) | (slot << 2) | ((x - i0) << 8);
    };
    sm.xst[0][lane] = xslab_of(p.ht[3], i);
    sm.xst[1][lane] = xslab_of(p.ht[4], i);
    sm.xst[2][lane] = xslab_of(p.et[3], i);
    sm.xst[3][lane] = xslab_of(p.et[4], i);
    sm.xst[4][lane] = pack(p.ht[3], p.ht[4], lane);
    sm.xst[5][lane] = pack(p.ht[3], p.ht[4], lane + 32);
    sm.xst[6][lane] = pack(p.et[3], p.et[4], lane);
    sm.xst[7][lane] = pack(p.et[3], p.et[4], lane + 32);
  }
  if (xcompact) __syncthreads();  // CTA-uniform
  bool shell_z = false;

  // H of the previous plane on the own cells (the z-backward differences of E).
  float4 hxp = make_float4(0.f, 0.f, 0.f, 0.f), hyp = hxp;

  int e0 = kstart % 3, e1 = (kstart + 1) % 3, hs = kstart & 1;
  for (int k = kstart; k < k1; ++k) {
    const int n = k - kstart;
    const bool emit = k >= k0;
    const bool arrived = tma::bar_wait(&sm.bar[n & 1], (n >> 1) & 1, wait_ns);
    if (__syncthreads_or(!arrived)) {  // CTA-uniform: every thread leaves together
      if (tid == 0) {
        if (p.status) atomicExch(p.status, 1);
        if (!p.test_stall) tma::bar_wait(&sm.bar[n & 1], (n >> 1) & 1, wait_ns);  // the bundle in flight
      }
      __syncthreads();
      return;
    }
    if (tid == 0 && k + 1 < k1) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue(k + 1, (n + 1) & 1, false);
    }
    const float* E0x = sm.e[e0][0];
    const float* E0y = sm.e[e0][1];
    const float* E0z = sm.e[e0][2];
    const float* E1x = sm.e[e1][0];
    const float* E1y = sm.e[e1][1];
    const float* HOx = sm.h[hs][0];
    const float* HOy = sm.h[hs][1];
    const float* HOz = sm.h[hs][2];
    const uint8_t* IDS = sm.ids[hs];
    const uint8_t* HIDS = sm.hids[Lossy ? hs : 0];  // Lossy: H classes, box column = x - i0 + 16
    const bool src = p.n_hsrc > 0 && sources_touch(p, k, j0 - 1, j0 + TY, i0 - 1, i0 + TX);

    if (fast_ok && !src && k >= 1 && k < Z) {
      // ---- straight tile-plane: every own and halo cell valid ----------------
      auto body = [&](auto mode) {
        // The body's CPML axes (bits 0-2: x, y, z) and whether the tile may
        // touch x = 0 / y = 0 (bit 3) are compile-time, so that a tile-plane
        // runs code holding only its own absorber work; with bit 4 the axes
        // are upper bounds and the plane's own flags decide at run time (the
        // rare combinations share that body).
        constexpr int M = decltype(mode)::value;
        constexpr bool SX = M & 1, SY = M & 2, SZ = M & 4, FC = M & 8, RT = M & 16;
        // Bit 5, or the run-time body on the last tile row: own rows from
        // jown, row Y in warp TY-1 (Hx, Hz and Ey do not exist there and the
        // y = Y ghost applies).
        constexpr bool LY = M & 32;
        // The run-time and last-row bodies also take the partial last tile:
        // stores and psi accesses stop at x = X (nv); the others handle all
        // four cells of every lane with no test.
        const int nvv = Partial && (RT || LY) ? nv : 4;
        const bool lyr = LY || (RT && ylast);
        const bool st = !lyr || own;       // this row is stored
        const bool rowY = lyr && j == Y;   // row Y: Hx, Hz, Ey absent
        const bool AX = SX && (!RT || shell_x), AY = SY && (!RT || shell_y), AZ = SZ && (!RT || shell_z);
        const bool at_x0 = FC && xface, at_y0 = FC && yface;
        const int jh = j0 - 1, ih = i0 - 1;  // the halo row and column
        // Which warps recompute a halo this plane (never on a pre-plane).
        const bool halo_row_x = emit && warp == 0 && !at_y0;              // Hx on row j0-1
        const bool halo_row_z = emit && warp == 1 && !at_y0;              // Hz on row j0-1
        const bool halo_col = emit && warp == 2 && lane < TY && !at_x0;   // Hy, Hz on column i0-1
        const int jc = j0 + lane;                                         // halo_col's row
        // ---- every global load of the plane goes out first ----
        // psi of the H terms: own cells and halos.
        float4 qh0, qh1, qh2, qh5;
        if (AY && !rowY) {
          qh0 = psi4_fetch<1>(p.ht[0], slot_of(p.ht[0], j), k, j, i, nvv);
          qh5 = psi4_fetch<1>(p.ht[5], slot_of(p.ht[5], j), k, j, i, nvv);
        }
        if (AZ) {
          if (!rowY) qh1 = psi4_fetch<0>(p.ht[1], slot_of(p.ht[1], k), k, j, i, nvv);
          qh2 = psi4_fetch<0>(p.ht[2], slot_of(p.ht[2], k), k, j, i, nvv);
        }
        // psi of the E terms too: in flight through the whole H phase.
        float4 qe0, qe1, qe2, qe5;
        if (emit) {
          if (AY) {
            qe0 = psi4_fetch<1>(p.et[0], slot_of(p.et[0], j), k, j, i, nvv);
            qe5 = psi4_fetch<1>(p.et[5], slot_of(p.et[5], j), k, j, i, nvv);
          }
          if (AZ) {
            qe1 = psi4_fetch<0>(p.et[1], slot_of(p.et[1], k), k, j, i, nvv);
            if (!rowY) qe2 = psi4_fetch<0>(p.et[2], slot_of(p.et[2], k), k, j, i, nvv);
          }
        }
        // ---- compact x work of the H terms (Hyx, Hzx) on this warp's row ----
        if (AX) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int w = sm.xst[4 + h][lane];
            if ((w & 1) && !(rowY && (w & 2))) {
              const bool second = w & 2;  // Hzx (dEy/dx), else Hyx (dEz/dx)
              const int slot = (w >> 2) & 63, xo = w >> 8;
              const CpmlTermDev& d = second ? p.ht[4] : p.ht[3];
              const float* Erow = second ? E0y : E0z;
              const int b = r * BX + 4 + xo;
              const int off = (k * d.pdy + j) * d.pdx + slot;
              const int t = second ? 1 : 0;
              const float psi = xstage ? sm.xps[hs][t][r * T::XW + slot - sm.xwin[t]] : d.psi_in[off];
              float nv;
              const float dp = cpml_d<Exact>(sm.cc[second ? 4 : 3][slot], res, psi, MH(Erow[b + 1] - Erow[b], 2, i0 + xo), &nv);
              if (emit && st) d.psi_out[off] = nv;
              sm.xd[second ? 1 : 0][warp][slot] = dp;
            }
          }
          __syncwarp();
        }
        // ---- H on the own row ----
        float4 dx0, dx1, dy0, dy1, dz0, dz1;
        {
          const float4 ez = ld4(E0z + rc), ey = ld4(E0y + rc), ex = ld4(E0x + rc);
          float ez4 = __shfl_down_sync(kFull, ez.x, 1), ey4 = __shfl_down_sync(kFull, ey.x, 1);
          if (lane == 31) {
            ez4 = E0z[rc + 4];
            ey4 = E0y[rc + 4];
          }
          dx0 = MH4(sub4(ld4(E0z + rc + BX), ez), 1, j), dx1 = MH4(sub4(ld4(E1y + rc), ey), 0, k);  // Hx: dEz/dy, dEy/dz
          dy0 = MH4(sub4(ld4(E1x + rc), ex), 0, k), dy1 = MH4x(sub4(next4(ez, ez4), ez), i);       // Hy: dEx/dz, dEz/dx
          dz0 = MH4x(sub4(next4(ey, ey4), ey), i), dz1 = MH4(sub4(ld4(E0x + rc + BX), ex), 1, j);  // Hz: dEy/dx, dEx/dy
        }
        if (AY && !rowY) {
          dx0 = psi4_apply<Exact, 1>(p.ht[0], sm.cc[0], slot_of(p.ht[0], j), qh0, k, j, i, res, dx0, emit && st, nvv);
          dz1 = psi4_apply<Exact, 1>(p.ht[5], sm.cc[5], slot_of(p.ht[5], j), qh5, k, j, i, res, dz1, emit && st, nvv);
        }
        if (AZ) {
          if (!rowY)
            dx1 = psi4_apply<Exact, 0>(p.ht[1], sm.cc[1], slot_of(p.ht[1], k), qh1, k, j, i, res, dx1, emit && st, nvv);
          dy0 = psi4_apply<Exact, 0>(p.ht[2], sm.cc[2], slot_of(p.ht[2], k), qh2, k, j, i, res, dy0, emit && st, nvv);
        }
        if (AX) {
          dy1 = xtake(dy1, sm.xst[0][lane], sm.xd[0][warp]);
          dz0 = xtake(dz0, sm.xst[1][lane], sm.xd[1][warp]);
        }
        float4 hx, hy, hz;
        if constexpr (Lossy) {
          const uint32_t hw4 = *reinterpret_cast<const uint32_t*>(HIDS + r * T::HW + 16 + 4 * lane);
          hx = h4_loss<Exact>(ld4(HOx + rc), sm.hcls, hw4, 0, dx0, dx1);
          hy = h4_loss<Exact>(ld4(HOy + rc), sm.hcls, hw4, 1, dy0, dy1);
          hz = h4_loss<Exact>(ld4(HOz + rc), sm.hcls, hw4, 2, dz0, dz1);
        } else {
          hx = h4<Exact>(ld4(HOx + rc), sm.hcoef[0], sm.hcoef[3], dx0, dx1);
          hy = h4<Exact>(ld4(HOy + rc), sm.hcoef[1], sm.hcoef[4], dy0, dy1);
          hz = h4<Exact>(ld4(HOz + rc), sm.hcoef[2], sm.hcoef[5], dz0, dz1);
        }
        if (at_x0 && lane == 0 && wx0) hx.x = 0.0f;  // PEC: normal H on the x = 0 wall
        if (at_y0 && warp == 0 && wy0) hy = make_float4(0.f, 0.f, 0.f, 0.f);
        if (rowY && wy1) hy = make_float4(0.f, 0.f, 0.f, 0.f);  // PEC: normal H on the y = Y wall
        st4(&sm.hn[0][r][c0], hx);
        st4(&sm.hn[1][r][c0], hy);
        st4(&sm.hn[2][r][c0], hz);
        const int o = k * PL + j * P + i;
        if (emit && st) {
          if (!rowY) st4m(p.hout[0] + o, hx, nvv);
          st4m(p.hout[1] + o, hy, nvv);
          if (!rowY) st4m(p.hout[2] + o, hz, nvv);
        }
        // ---- recomputed halo: row j0-1 (Hx by warp 0, Hz by warp 1) and
        //      column i0-1 (Hy, Hz by warp 2), read-only on psi ----
        if (halo_row_x) {
          const int b = c0;
          float4 qa, qb;
          if (AY) qa = psi4_fetch<1>(p.ht[0], slot_of(p.ht[0], jh), k, jh, i, nvv);
          if (AZ) qb = psi4_fetch<0>(p.ht[1], slot_of(p.ht[1], k), k, jh, i, nvv);
          float4 d0 = MH4(sub4(ld4(E0z + b + BX), ld4(E0z + b)), 1, jh), d1 = MH4(sub4(ld4(E1y + b), ld4(E0y + b)), 0, k);
          if (AY) d0 = psi4_apply<Exact, 1>(p.ht[0], sm.cc[0], slot_of(p.ht[0], jh), qa, k, jh, i, res, d0, false, nvv);
          if (AZ) d1 = psi4_apply<Exact, 0>(p.ht[1], sm.cc[1], slot_of(p.ht[1], k), qb, k, jh, i, res, d1, false, nvv);
          float4 h;
          if constexpr (Lossy)
            h = h4_loss<Exact>(ld4(HOx + b), sm.hcls, *reinterpret_cast<const uint32_t*>(HIDS + 16 + 4 * lane), 0,
                               d0, d1);
          else
            h = h4<Exact>(ld4(HOx + b), sm.hcoef[0], sm.hcoef[3], d0, d1);
          if (at_x0 && lane == 0 && wx0) h.x = 0.0f;
          st4(&sm.hn[0][0][b], h);
        } else if (halo_row_z) {
          const int b = c0;
          float4 qa, qb;
          const int xs4 = AX ? sm.xst[1][lane] : 0;
          if (AX) {
            if (xstage) {  // row j0-1 of the staged Hzx box (cells outside the slab are not read)
              const float* q = &sm.xps[hs][1][(xs4 >> 4) - sm.xwin[1]];
              qa = make_float4(q[0], q[1], q[2], q[3]);
            } else {
              qa = psix_fetch(p.ht[4], xs4, k, jh);
            }
          }
          if (AY) qb = psi4_fetch<1>(p.ht[5], slot_of(p.ht[5], jh), k, jh, i, nvv);
          const float4 eyh = ld4(E0y + b);
          float e4 = __shfl_down_sync(kFull, eyh.x, 1);
          if (lane == 31) e4 = E0y[b + 4];
          float4 d0 = MH4x(sub4(next4(eyh, e4), eyh), i), d1 = MH4(sub4(ld4(E0x + b + BX), ld4(E0x + b)), 1, jh);
          if (AX) d0 = psix_apply<Exact>(p.ht[4], sm.cc[4], xs4, qa, k, jh, res, d0, false);
          if (AY) d1 = psi4_apply<Exact, 1>(p.ht[5], sm.cc[5], slot_of(p.ht[5], jh), qb, k, jh, i, res, d1, false, nvv);
          if constexpr (Lossy)
            st4(&sm.hn[2][0][b], h4_loss<Exact>(ld4(HOz + b), sm.hcls,
                                                *reinterpret_cast<const uint32_t*>(HIDS + 16 + 4 * lane), 2, d0, d1));
          else
            st4(&sm.hn[2][0][b], h4<Exact>(ld4(HOz + b), sm.hcoef[2], sm.hcoef[5], d0, d1));
        } else if (halo_col) {
          const int rr = 1 + lane, b = rr * BX + 3;
          const bool hz_ok = !(lyr && jc == Y);  // Hz has no row Y
          float qc0 = 0.f, qc1 = 0.f, qc2 = 0.f, qc3 = 0.f;
          if (AZ) qc0 = psi1_fetch<0>(p.ht[2], k, jc, ih);
          if (AX) qc1 = psi1_fetch<2>(p.ht[3], k, jc, ih);
          if (AX && hz_ok) qc2 = psi1_fetch<2>(p.ht[4], k, jc, ih);
          if (AY && hz_ok) qc3 = psi1_fetch<1>(p.ht[5], k, jc, ih);
          float d0 = MH(E1x[b] - E0x[b], 0, k), d1 = MH(E0z[b + 1] - E0z[b], 2, ih);  // Hy: dEx/dz, dEz/dx
          if (AZ) d0 = psi1_apply<Exact, 0>(p.ht[2], sm.cc[2], qc0, k, jc, ih, res, d0, false);
          if (AX) d1 = psi1_apply<Exact, 2>(p.ht[3], sm.cc[3], qc1, k, jc, ih, res, d1, false);
          const int hc = Lossy ? (HIDS[rr * T::HW + 15] & kHClassMask) : 0;  // the halo column's H class
          const float2 cy = Lossy ? sm.hcls[hc * 4 + 1] : make_float2(sm.hcoef[1], sm.hcoef[4]);
          const float2 cz = Lossy ? sm.hcls[hc * 4 + 2] : make_float2(sm.hcoef[2], sm.hcoef[5]);
          float hyv = h1<Exact>(HOy[b], cy.x, cy.y, d0, d1);
          if (at_y0 && jc == 0 && wy0) hyv = 0.0f;
          float f0 = MH(E0y[b + 1] - E0y[b], 2, ih), f1 = MH(E0x[b + BX] - E0x[b], 1, jc);  // Hz: dEy/dx, dEx/dy
          if (AX && hz_ok) f0 = psi1_apply<Exact, 2>(p.ht[4], sm.cc[4], qc2, k, jc, ih, res, f0, false);
          if (AY && hz_ok) f1 = psi1_apply<Exact, 1>(p.ht[5], sm.cc[5], qc3, k, jc, ih, res, f1, false);
          sm.hn[1][rr][3] = hyv;
          sm.hn[2][rr][3] = h1<Exact>(HOz[b], cz.x, cz.y, f0, f1);
        }
        __syncthreads();
        if (!emit) {
          hxp = hx;
          hyp = hy;
          return;
        }
        // ---- compact x work of the E terms (Eyx, Ezx) on this warp's row ----
        if (AX) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int w = sm.xst[6 + h][lane];
            if ((w & 1) && !(rowY && !(w & 2))) {
              const bool second = w & 2;  // Ezx (dHy/dx), else Eyx (dHz/dx)
              const int slot = (w >> 2) & 63, xo = w >> 8;
              const CpmlTermDev& d = second ? p.et[4] : p.et[3];
              const float* Hrow = second ? sm.hn[1][r] : sm.hn[2][r];
              const int c = 4 + xo;
              // Beyond x = 0 the ghost: zero on a metallic wall, else the edge value.
              const float dv = (at_x0 && xo == 0) ? (wx0 ? Hrow[c] : 0.0f) : Hrow[c] - Hrow[c - 1];
              const int off = (k * d.pdy + j) * d.pdx + slot;
              const int t = second ? 3 : 2;
              const float psi = xstage ? sm.xps[hs][t][r * T::XW + slot - sm.xwin[t]] : d.psi_in[off];
              float nv;
              const float dp = cpml_d<Exact>(sm.cc[second ? 10 : 9][slot], res, psi, ME(dv, 2, i0 + xo), &nv);
              if (st) d.psi_out[off] = nv;
              sm.xd[second ? 1 : 0][warp][slot] = dp;
            }
          }
          __syncwarp();
        }
        // ---- E on the own row ----
        float4 hzy = ld4(&sm.hn[2][r - 1][c0]), hxy = ld4(&sm.hn[0][r - 1][c0]);
        float hzl = __shfl_up_sync(kFull, hz.w, 1), hyl = __shfl_up_sync(kFull, hy.w, 1);
        if (lane == 0) {
          hzl = sm.hn[2][r][3];
          hyl = sm.hn[1][r][3];
          if (at_x0) {  // ghost beyond x = 0: zero on a metallic wall, else the edge value
            hzl = wx0 ? 0.0f : hz.x;
            hyl = wx0 ? 0.0f : hy.x;
          }
        }
        if (at_y0 && warp == 0) {  // ghost beyond y = 0
          hzy = wy0 ? make_float4(0.f, 0.f, 0.f, 0.f) : hz;
          hxy = wy0 ? make_float4(0.f, 0.f, 0.f, 0.f) : hx;
        }
        float4 fx0 = ME4(sub4(hz, hzy), 1, j), fx1 = ME4(sub4(hy, hyp), 0, k);        // Ex: dHz/dy, dHy/dz
        float4 fy0 = ME4(sub4(hx, hxp), 0, k), fy1 = ME4x(sub4(hz, prev4(hzl, hz)), i);  // Ey: dHx/dz, dHz/dx
        float4 fz0 = ME4x(sub4(hy, prev4(hyl, hy)), i), fz1 = ME4(sub4(hx, hxy), 1, j);  // Ez: dHy/dx, dHx/dy
        if (rowY) {  // ghost beyond y = Y: zero on a metallic wall, else the edge value
          const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
          fx0 = ME4(wy1 ? sub4(z4, hzy) : z4, 1, j);
          fz1 = ME4(wy1 ? sub4(z4, hxy) : z4, 1, j);
        }
        if (AY) {
          fx0 = psi4_apply<Exact, 1>(p.et[0], sm.cc[6], slot_of(p.et[0], j), qe0, k, j, i, res, fx0, st, nvv);
          fz1 = psi4_apply<Exact, 1>(p.et[5], sm.cc[11], slot_of(p.et[5], j), qe5, k, j, i, res, fz1, st, nvv);
        }
        if (AZ) {
          fx1 = psi4_apply<Exact, 0>(p.et[1], sm.cc[7], slot_of(p.et[1], k), qe1, k, j, i, res, fx1, st, nvv);
          if (!rowY)
            fy0 = psi4_apply<Exact, 0>(p.et[2], sm.cc[8], slot_of(p.et[2], k), qe2, k, j, i, res, fy0, st, nvv);
        }
        if (AX) {
          fy1 = xtake(fy1, sm.xst[2][lane], sm.xd[0][warp]);
          fz0 = xtake(fz0, sm.xst[3][lane], sm.xd[1][warp]);
        }
        const float4 ex = ld4(E0x + rc), ey = ld4(E0y + rc), ez = ld4(E0z + rc);  // E(k) of the own cells
        const uint32_t w4 = *reinterpret_cast<const uint32_t*>(IDS + warp * TX + 4 * lane);
        float4 nx, ny, nz;
        if constexpr (Lossy) {
          const float2* ec = reinterpret_cast<const float2*>(sm.cls);
          nx = e4_loss<Exact>(ex, ec, w4, 0, fx0, fx1);
          ny = e4_loss<Exact>(ey, ec, w4, 1, fy0, fy1);
          nz = e4_loss<Exact>(ez, ec, w4, 2, fz0, fz1);
        } else {
          const float4 t0 = sm.cls[w4 & 0xffu], t1 = sm.cls[(w4 >> 8) & 0xffu];
          const float4 t2 = sm.cls[(w4 >> 16) & 0xffu], t3 = sm.cls[w4 >> 24];
          nx = make_float4(e_upd<Exact>(ex.x, t0.x, fx0.x, fx1.x), e_upd<Exact>(ex.y, t1.x, fx0.y, fx1.y),
                           e_upd<Exact>(ex.z, t2.x, fx0.z, fx1.z), e_upd<Exact>(ex.w, t3.x, fx0.w, fx1.w));
          ny = make_float4(e_upd<Exact>(ey.x, t0.y, fy0.x, fy1.x), e_upd<Exact>(ey.y, t1.y, fy0.y, fy1.y),
                           e_upd<Exact>(ey.z, t2.y, fy0.z, fy1.z), e_upd<Exact>(ey.w, t3.y, fy0.w, fy1.w));
          nz = make_float4(e_upd<Exact>(ez.x, t0.z, fz0.x, fz1.x), e_upd<Exact>(ez.y, t1.z, fz0.y, fz1.y),
                           e_upd<Exact>(ez.z, t2.z, fz0.z, fz1.z), e_upd<Exact>(ez.w, t3.z, fz0.w, fz1.w));
        }
        if (at_y0 && warp == 0 && wy0) {  // PEC: Ex, Ez on the y = 0 wall
          nx = make_float4(0.f, 0.f, 0.f, 0.f);
          nz = nx;
        }
        if (at_x0 && lane == 0 && wx0) {  // Ey, Ez on the x = 0 wall
          ny.x = 0.0f;
          nz.x = 0.0f;
        }
        if (rowY && wy1) {  // Ex, Ez on the y = Y wall
          nx = make_float4(0.f, 0.f, 0.f, 0.f);
          nz = nx;
        }
        if (st) {
          st4m(p.eout[0] + o, nx, nvv);
          if (!rowY) st4m(p.eout[1] + o, ny, nvv);
          st4m(p.eout[2] + o, nz, nvv);
        }
        hxp = hx;
        hyp = hy;
      };
      using std::integral_constant;
      if constexpr (!Cpml) {
        if (ylast || i0 + TX > X) body(integral_constant<int, 32 | 8>{});  // last row, partial last tile
        else if (xface || yface) body(integral_constant<int, 8>{});
        else body(integral_constant<int, 0>{});
      } else {
        shell_z = !(k >= p.cpml_inner[0][0] && k < p.cpml_inner[0][1]);
        if (ylast || shell_y || shell_z || i0 + TX > X)
          body(integral_constant<int, 16 | 8 | 7>{});  // last row, y / z slabs, partial last tile
        else if (shell_x) body(integral_constant<int, 8 | 1>{});           // x slab tiles (about half)
        else if (xface || yface) body(integral_constant<int, 8>{});
        else body(integral_constant<int, 0>{});
      }
    } else {
      // ---- general tile-plane: per cell, every validity / ghost / PEC rule ---
      const bool cpml = Cpml;
      // H of one lattice point at box (rr, cc) = (j0-1+rr, i0-4+cc); `which`
      // bit 0 Hx, 1 Hy, 2 Hz; `own` stores it (and its psi).
      auto h_cell = [&](int rr, int cc, int which, bool own) {
        const int jj = j0 - 1 + rr, ii = i0 - 4 + cc, b = rr * BX + cc;
        own = own && ii < X;  // column X: the column kernel
        const int o = k * PL + jj * P + ii;
        // H coefficients: uniform, or (Lossy) the point's H class (box column
        // of x = ii: cc + 12).
        auto hco = [&](int n) {
          if constexpr (Lossy) return sm.hcls[(HIDS[rr * T::HW + cc + 12] & kHClassMask) * 4 + n];
          return make_float2(sm.hcoef[n], sm.hcoef[3 + n]);
        };
        const bool zZ = k < Z, yY = jj >= 0 && jj < Y, yY1 = jj >= 0 && jj <= Y;
        const bool iX = ii >= 0 && ii < X, iX1 = ii >= 0 && ii <= X;
        if ((which & 1) && zZ && yY && iX1) {  // Hx: dEz/dy - dEy/dz
          float d0 = MH(E0z[b + BX] - E0z[b], 1, jj), d1 = MH(E1y[b] - E0y[b], 0, k);
          if (cpml) {
            d0 = cpml1<Exact, 1>(p.ht[0], sm.cc[0], cc_smem, res, k, jj, ii, d0, own);
            d1 = cpml1<Exact, 0>(p.ht[1], sm.cc[1], cc_smem, res, k, jj, ii, d1, own);
          }
          const float2 c = hco(0);
          float h = h1<Exact>(HOx[b], c.x, c.y, d0, d1);
          if (src) h = h_sources_at(p, sm.amp, 3, k, jj, ii, h);
          if ((ii == 0 && wx0) || (ii == X && wx1)) h = 0.0f;
          sm.hn[0][rr][cc] = h;
          if (own) p.hout[0][o] = h;
        }
        if ((which & 2) && zZ && yY1 && iX) {  // Hy: dEx/dz - dEz/dx
          float d0 = MH(E1x[b] - E0x[b], 0, k), d1 = MH(E0z[b + 1] - E0z[b], 2, ii);
          if (cpml) {
            d0 = cpml1<Exact, 0>(p.ht[2], sm.cc[2], cc_smem, res, k, jj, ii, d0, own);
            d1 = cpml1<Exact, 2>(p.ht[3], sm.cc[3], cc_smem, res, k, jj, ii, d1, own);
          }
          const float2 c = hco(1);
          float h = h1<Exact>(HOy[b], c.x, c.y, d0, d1);
          if (src) h = h_sources_at(p, sm.amp, 4, k, jj, ii, h);
          if ((jj == 0 && wy0) || (jj == Y && wy1)) h = 0.0f;
          sm.hn[1][rr][cc] = h;
          if (own) p.hout[1][o] = h;
        }
        if ((which & 4) && yY && iX) {  // Hz: dEy/dx - dEx/dy
          float d0 = MH(E0y[b + 1] - E0y[b], 2, ii), d1 = MH(E0x[b + BX] - E0x[b], 1, jj);
          if (cpml) {
            d0 = cpml1<Exact, 2>(p.ht[4], sm.cc[4], cc_smem, res, k, jj, ii, d0, own);
            d1 = cpml1<Exact, 1>(p.ht[5], sm.cc[5], cc_smem, res, k, jj, ii, d1, own);
          }
          const float2 c = hco(2);
          float h = h1<Exact>(HOz[b], c.x, c.y, d0, d1);
          if (src) h = h_sources_at(p, sm.amp, 5, k, jj, ii, h);
          if ((k == 0 && wz0) || (k == Z && wz1)) h = 0.0f;
          sm.hn[2][rr][cc] = h;
          if (own) p.hout[2][o] = h;
        }
      };
      // E of one own lattice point at box (rr, cc), with H of the previous
      // plane there (hxz, hyz).
      auto e_cell = [&](int rr, int cc, float hxz, float hyz) {
        const int jj = j0 - 1 + rr, ii = i0 - 4 + cc, b = rr * BX + cc;
        if (jj > Y || ii >= X) return;  // column X: the column kernel
        const int o = k * PL + jj * P + ii;
        const float hx = sm.hn[0][rr][cc], hy = sm.hn[1][rr][cc], hz = sm.hn[2][rr][cc];
        const float hz_y = sm.hn[2][rr - 1][cc], hx_y = sm.hn[0][rr - 1][cc];
        const float hz_x = sm.hn[2][rr][cc - 1], hy_x = sm.hn[1][rr][cc - 1];
        const bool in_box = cc >= 4 && cc < 4 + TX && rr >= 1 && rr <= TY;
        const int cid = in_box ? IDS[(rr - 1) * TX + cc - 4] : p.site_class[(k * (Y + 1) + jj) * p.pitch8 + ii];
        const float4 t = sm.cls[Lossy ? 0 : cid];
        // E <- E + t.c (d0 - d1), or (Lossy) decay E + source (d0 - d1).
        auto eup = [&](float e, int n, float d0, float d1) {
          if constexpr (Lossy)
            return e_loss<Exact>(e, reinterpret_cast<const float2*>(sm.cls)[(cid & kEClassMask) * 4 + n], d0, d1);
          return e_upd<Exact>(e, n == 0 ? t.x : (n == 1 ? t.y : t.z), d0, d1);
        };
        if (ii < X) {  // Ex: dHz/dy - dHy/dz
          float d0 = ME(ghost_diff(hz, hz_y, jj, Y, wy0, wy1), 1, jj), d1 = ME(ghost_diff(hy, hyz, k, Z, wz0, wz1), 0, k);
          if (cpml) {
            d0 = cpml1<Exact, 1>(p.et[0], sm.cc[6], cc_smem, res, k, jj, ii, d0, true);
            d1 = cpml1<Exact, 0>(p.et[1], sm.cc[7], cc_smem, res, k, jj, ii, d1, true);
          }
          float e = eup(E0x[b], 0, d0, d1);
          if ((k == 0 && wz0) || (k == Z && wz1) || (jj == 0 && wy0) || (jj == Y && wy1)) e = 0.0f;
          p.eout[0][o] = e;
        }
        if (jj < Y) {  // Ey: dHx/dz - dHz/dx
          float d0 = ME(ghost_diff(hx, hxz, k, Z, wz0, wz1), 0, k), d1 = ME(ghost_diff(hz, hz_x, ii, X, wx0, wx1), 2, ii);
          if (cpml) {
            d0 = cpml1<Exact, 0>(p.et[2], sm.cc[8], cc_smem, res, k, jj, ii, d0, true);
            d1 = cpml1<Exact, 2>(p.et[3], sm.cc[9], cc_smem, res, k, jj, ii, d1, true);
          }
          float e = eup(E0y[b], 1, d0, d1);
          if ((k == 0 && wz0) || (k == Z && wz1) || (ii == 0 && wx0) || (ii == X && wx1)) e = 0.0f;
          p.eout[1][o] = e;
        }
        if (k < Z) {  // Ez: dHy/dx - dHx/dy
          float d0 = ME(ghost_diff(hy, hy_x, ii, X, wx0, wx1), 2, ii), d1 = ME(ghost_diff(hx, hx_y, jj, Y, wy0, wy1), 1, jj);
          if (cpml) {
            d0 = cpml1<Exact, 2>(p.et[4], sm.cc[10], cc_smem, res, k, jj, ii, d0, true);
            d1 = cpml1<Exact, 1>(p.et[5], sm.cc[11], cc_smem, res, k, jj, ii, d1, true);
          }
          float e = eup(E0z[b], 2, d0, d1);
          if ((jj == 0 && wy0) || (jj == Y && wy1) || (ii == 0 && wx0) || (ii == X && wx1)) e = 0.0f;
          p.eout[2][o] = e;
        }
      };
#pragma unroll 1
      for (int q = 0; q < 4; ++q) h_cell(r, c0 + q, 7, emit && own);
      if (emit) {
        if (warp == 0 && j0 > 0) {
#pragma unroll 1
          for (int q = 0; q < 4; ++q) h_cell(0, c0 + q, 1 | 4, false);
        } else if (warp == 2 && lane < TY && i0 > 0) {
          h_cell(1 + lane, 3, 2 | 4, false);
        }
      }
      __syncthreads();
      if (emit && own) {
#pragma unroll 1
        for (int q = 0; q < 4; ++q) e_cell(r, c0 + q, get(hxp, q), get(hyp, q));
      }
      hxp = ld4(&sm.hn[0][r][c0]);
      hyp = ld4(&sm.hn[1][r][c0]);
    }
    e0 = e1;
    e1 = e1 == 2 ? 0 : e1 + 1;
    hs ^= 1;
  }
}



// ---- column x = X ------------------------------------------------------------
// The class step's tiles end at x = X - 1 and this kernel, run before it on
// the same stream, updates the lattice column x = X:
// Hx there, then Ey and Ez, with the general path's per-cell rules (ghosts,
// PEC, CPML, H sources).  It reads only the step's inputs, so it depends on no
// other launch of the step: the H of x = X - 1 that Ey and Ez see through the
// ghost beyond x = X counts only with a metallic x = X wall, and is then
// recomputed here from the same inputs with the class step's arithmetic.  A
// block covers 32 rows x 8 planes and recomputes the Hx of the row before and
// of the plane before read-only; every load of a thread goes out before the
// first use, so the column costs about one memory round trip.  (Done inside
// the tiles, by one lane or one warp, the column put its psi latency on the
// critical path of a quarter of the CTAs: 12-15 % of the 512 x 512 x 256 step.)
constexpr int kColJ = 32, kColK = 8;

// One CPML term at a cell of the column: psi <- b psi + a d, d' = d / kappa +
// psi, with the coefficients as the class step stages them.
template <bool Exact, int Axis>
__device__ __forceinline__ float col_cpml(const CpmlTermDev& t, float res, float inv_res, float psi_old, int k, int j,
                                          int x, float d, bool write) {
  const int slot = slot_of(t, Axis == 0 ? k : (Axis == 1 ? j : x));
  if (slot < 0) return d;
  const float4 c = make_float4(Exact ? __ldg(t.a + slot) : __ldg(t.a + slot) * inv_res, __ldg(t.b + slot),
                               __ldg(t.k + slot), 0.0f);
  float n;
  const float r = cpml_d<Exact>(c, res, psi_old, d, &n);
  if (write) t.psi_out[psi_off<Axis>(t, slot, k, j, x)] = n;
  return r;
}

// psi of a term at a cell, 0 outside its slab.
template <int Axis>
__device__ __forceinline__ float col_psi(const CpmlTermDev& t, int k, int j, int x) {
  const int slot = slot_of(t, Axis == 0 ? k : (Axis == 1 ? j : x));
  return slot >= 0 ? t.psi_in[psi_off<Axis>(t, slot, k, j, x)] : 0.0f;
}

template <bool Cpml, bool Exact, bool Lossy, bool Metric>
__global__ void __launch_bounds__(kColJ * kColK) class_column_kernel(const __grid_constant__ Step3D p) {
  __shared__ float hx[kColK + 1][kColJ + 1];  // new Hx at (k0 - 1 + a, j0 - 1 + b, X)
  __shared__ float amp[kMaxFusedSources];
  const int Z = p.Z, Y = p.Y, X = p.X;
  const int j0 = blockIdx.x * kColJ, k0 = blockIdx.y * kColK;
  const int tid = threadIdx.y * kColJ + threadIdx.x;
  const int P = p.pitch, PL = (Y + 1) * p.pitch;  // element offsets < 2^31 (validated)
  const float res = p.res, inv_res = p.inv_res;
  const float dbs = p.div_bs, drs = p.div_rs;
  const bool wz0 = wall(p.metallic, 0, false), wz1 = wall(p.metallic, 0, true);
  const bool wy0 = wall(p.metallic, 1, false), wy1 = wall(p.metallic, 1, true);
  const bool wx0 = wall(p.metallic, 2, false), wx1 = wall(p.metallic, 2, true);
  auto D1 = [&](float v) { return dv<Exact>(v, dbs, drs); };
  // Forward (H) and backward (E) derivatives along an axis at a coordinate:
  // the difference times the metric's inverse distance there, or D1.
  auto MH = [&](float v, int axis, int c) -> float {
    if constexpr (Metric) return v * p.metric_h[axis][clampi(c, axis_cells(p, axis) - 1)];
    else return D1(v);
  };
  auto ME = [&](float v, int axis, int c) -> float {
    if constexpr (Metric) return v * p.metric_e[axis][clampi(c, axis_cells(p, axis))];
    else return D1(v);
  };
  // This thread's E cell (k, j, X): its inputs are loaded first.
  const int k = k0 + threadIdx.y, j = j0 + threadIdx.x;
  const bool live = k <= Z && j <= Y;
  const bool ey_ok = live && j < Y, ez_ok = live && k < Z;
  const int o = live ? k * PL + j * P + X : 0;
  const float ey0 = ey_ok ? p.ein[1][o] : 0.0f, ez0 = ez_ok ? p.ein[2][o] : 0.0f;
  const int cid = live ? p.site_class[(static_cast<int64_t>(k) * (Y + 1) + j) * p.pitch8 + X] : 0;
  const float4 t = Lossy ? make_float4(0.f, 0.f, 0.f, 0.f) : p.class_coef[cid];
  const float2* ec = reinterpret_cast<const float2*>(p.class_coef);  // Lossy: [128][4] (decay, source)
  // Lossy: the (decay, source) of H component n at lattice point (kk, jj, x).
  auto hco = [&](int kk, int jj, int x, int n) {
    return p.h_class_coef[(p.h_class[(static_cast<int64_t>(kk) * (Y + 1) + jj) * p.pitch8 + x] & kHClassMask) * 4 + n];
  };
  float q_eyz = 0.f, q_eyx = 0.f, q_ezx = 0.f, q_ezy = 0.f;
  if (Cpml) {
    if (ey_ok) {
      q_eyz = col_psi<0>(p.et[2], k, j, X);
      q_eyx = col_psi<2>(p.et[3], k, j, X);
    }
    if (ez_ok) {
      q_ezx = col_psi<2>(p.et[4], k, j, X);
      q_ezy = col_psi<1>(p.et[5], k, j, X);
    }
  }
  if (tid < p.n_hsrc) amp[tid] = source_amplitude(p.hsrc[tid], p.step_counter[0] + p.step_offset);
  __syncthreads();
  const float hdec = p.hm.decay[0][0], hsrc = p.hm.source[0][0] * (Exact ? 1.0f : inv_res);
  // Hx (storage (Z, Y, X + 1)): dEz/dy - dEy/dz.
  for (int q = tid; q < (kColK + 1) * (kColJ + 1); q += kColJ * kColK) {
    const int a = q / (kColJ + 1), b = q % (kColJ + 1);
    const int kk = k0 - 1 + a, jj = j0 - 1 + b;
    float h = 0.0f;
    if (kk >= 0 && kk < Z && jj >= 0 && jj < Y) {
      const bool own = a > 0 && b > 0;
      const int oh = kk * PL + jj * P + X;
      float qy = 0.f, qz = 0.f;
      if (Cpml) {
        qy = col_psi<1>(p.ht[0], kk, jj, X);
        qz = col_psi<0>(p.ht[1], kk, jj, X);
      }
      float d0 = MH(p.ein[2][oh + P] - p.ein[2][oh], 1, jj);
      float d1 = MH(p.ein[1][oh + PL] - p.ein[1][oh], 0, kk);
      if (Cpml) {
        d0 = col_cpml<Exact, 1>(p.ht[0], res, inv_res, qy, kk, jj, X, d0, own);
        d1 = col_cpml<Exact, 0>(p.ht[1], res, inv_res, qz, kk, jj, X, d1, own);
      }
      const float2 c = Lossy ? hco(kk, jj, X, 0) : make_float2(hdec, hsrc);
      h = h1<Exact>(p.hin[0][oh], c.x, c.y, d0, d1);
      if (p.n_hsrc > 0) h = h_sources_at(p, amp, 3, kk, jj, X, h);
      if (wx1) h = 0.0f;  // PEC: normal H on the x = X wall
      if (own) p.hout[0][oh] = h;
    }
    hx[a][b] = h;
  }
  __syncthreads();
  if (!live) return;
  const int a = threadIdx.y + 1, b = threadIdx.x + 1;
  // Hz, Hy at x = X - 1 (only a metallic x = X wall makes the ghost use them),
  // as the class step computes them: read-only on psi.
  float hz_w = 0.0f, hy_w = 0.0f;
  if (wx1) {
    const int ow = o - 1;
    if (ey_ok) {  // Hz(k, j, X - 1): dEy/dx - dEx/dy
      float d0 = MH(p.ein[1][ow + 1] - p.ein[1][ow], 2, X - 1), d1 = MH(p.ein[0][ow + P] - p.ein[0][ow], 1, j);
      if (Cpml) {
        d0 = col_cpml<Exact, 2>(p.ht[4], res, inv_res, col_psi<2>(p.ht[4], k, j, X - 1), k, j, X - 1, d0, false);
        d1 = col_cpml<Exact, 1>(p.ht[5], res, inv_res, col_psi<1>(p.ht[5], k, j, X - 1), k, j, X - 1, d1, false);
      }
      const float2 c = Lossy ? hco(k, j, X - 1, 2)
                             : make_float2(p.hm.decay[2][0], p.hm.source[2][0] * (Exact ? 1.0f : inv_res));
      hz_w = h1<Exact>(p.hin[2][ow], c.x, c.y, d0, d1);
      if (p.n_hsrc > 0) hz_w = h_sources_at(p, amp, 5, k, j, X - 1, hz_w);
      if ((k == 0 && wz0) || (k == Z && wz1)) hz_w = 0.0f;
    }
    if (ez_ok) {  // Hy(k, j, X - 1): dEx/dz - dEz/dx
      float d0 = MH(p.ein[0][ow + PL] - p.ein[0][ow], 0, k), d1 = MH(p.ein[2][ow + 1] - p.ein[2][ow], 2, X - 1);
      if (Cpml) {
        d0 = col_cpml<Exact, 0>(p.ht[2], res, inv_res, col_psi<0>(p.ht[2], k, j, X - 1), k, j, X - 1, d0, false);
        d1 = col_cpml<Exact, 2>(p.ht[3], res, inv_res, col_psi<2>(p.ht[3], k, j, X - 1), k, j, X - 1, d1, false);
      }
      const float2 c = Lossy ? hco(k, j, X - 1, 1)
                             : make_float2(p.hm.decay[1][0], p.hm.source[1][0] * (Exact ? 1.0f : inv_res));
      hy_w = h1<Exact>(p.hin[1][ow], c.x, c.y, d0, d1);
      if (p.n_hsrc > 0) hy_w = h_sources_at(p, amp, 4, k, j, X - 1, hy_w);
      if ((j == 0 && wy0) || (j == Y && wy1)) hy_w = 0.0f;
    }
  }
  if (ey_ok) {  // Ey: dHx/dz - dHz/dx, the Hz ghost beyond x = X
    float d0 = ME(ghost_diff(hx[a][b], hx[a - 1][b], k, Z, wz0, wz1), 0, k);
    float d1 = ME(ghost_diff(0.0f, hz_w, X, X, wx0, wx1), 2, X);
    if (Cpml) {
      d0 = col_cpml<Exact, 0>(p.et[2], res, inv_res, q_eyz, k, j, X, d0, true);
      d1 = col_cpml<Exact, 2>(p.et[3], res, inv_res, q_eyx, k, j, X, d1, true);
    }
    float e = Lossy ? e_loss<Exact>(ey0, ec[(cid & kEClassMask) * 4 + 1], d0, d1) : e_upd<Exact>(ey0, t.y, d0, d1);
    if ((k == 0 && wz0) || (k == Z && wz1) || wx1) e = 0.0f;
    p.eout[1][o] = e;
  }
  if (ez_ok) {  // Ez: dHy/dx - dHx/dy, the Hy ghost beyond x = X
    float d0 = ME(ghost_diff(0.0f, hy_w, X, X, wx0, wx1), 2, X);
    float d1 = ME(ghost_diff(hx[a][b], hx[a][b - 1], j, Y, wy0, wy1), 1, j);
    if (Cpml) {
      d0 = col_cpml<Exact, 2>(p.et[4], res, inv_res, q_ezx, k, j, X, d0, true);
      d1 = col_cpml<Exact, 1>(p.et[5], res, inv_res, q_ezy, k, j, X, d1, true);
    }
    float e = Lossy ? e_loss<Exact>(ez0, ec[(cid & kEClassMask) * 4 + 2], d0, d1) : e_upd<Exact>(ez0, t.z, d0, d1);
    if ((j == 0 && wy0) || (j == Y && wy1) || wx1) e = 0.0f;
    p.eout[2][o] = e;
  }
}

template <int NW, bool Cpml, bool Exact, bool Lossy, bool Partial, bool Metric>
cudaError_t launch_class_p(cudaStream_t s, const ClassMaps& maps, const Step3D& p);

template <int NW, bool Cpml, bool Exact, bool Lossy = false, bool Metric = false>
cudaError_t launch_class_t(cudaStream_t s, const ClassMaps& maps, const Step3D& p) {
  if (p.X % ClassTile<NW, Lossy>::TX != 0) return launch_class_p<NW, Cpml, Exact, Lossy, true, Metric>(s, maps, p);
  return launch_class_p<NW, Cpml, Exact, Lossy, false, Metric>(s, maps, p);
}

template <int NW, bool Cpml, bool Exact, bool Lossy, bool Partial, bool Metric>
cudaError_t launch_class_p(cudaStream_t s, const ClassMaps& maps, const Step3D& p) {
  using T = ClassTile<NW, Lossy>;
  const size_t smem = sizeof(typename T::Smem);
  auto kern = class_step_kernel<NW, Cpml, Exact, Lossy, Partial, Metric>;
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return err;
  // The dynamic shared-memory limit is a per-device function attribute: set it
  // on every launch (cheap) rather than once per process.
  err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (err != cudaSuccess) return err;
  const int kmax = p.Z + 1;
  const int zc = p.z_chunk > 0 ? p.z_chunk : kmax;
  const int gx = (p.X + T::TX - 1) / T::TX;  // the tiles end at x = X - 1: column X is the column kernel's
  const int gy = (p.Y + 1 + T::TY - 1) / T::TY, gz = (kmax + zc - 1) / zc;
  Step3D q = p;
  q.z_chunk = zc;
  // Absorber rows and chunks at both ends (the tile test of the kernel's ay
  // and per-plane shell_z): dispatched first.
  auto row_shell = [&](int b) {
    const int j0 = b * T::TY;
    return p.cpml && !(j0 - 1 >= p.cpml_inner[1][0] && j0 + T::TY <= p.cpml_inner[1][1]);
  };
  auto chunk_shell = [&](int c) {
    const int k0 = c * zc, k1 = std::min(k0 + zc, kmax);
    return p.cpml && (k0 < p.cpml_inner[0][0] || k1 > p.cpml_inner[0][1]);
  };
  int ylo = 0, yhi = gy, zlo = 0, zhi = gz;
  while (ylo < gy && row_shell(ylo)) ++ylo;
  while (yhi > ylo && row_shell(yhi - 1)) --yhi;
  while (zlo < gz && chunk_shell(zlo)) ++zlo;
  while (zhi > zlo && chunk_shell(zhi - 1)) --zhi;
  q.order[0] = ylo;
  q.order[1] = yhi;
  q.order[2] = zlo;
  q.order[3] = zhi;
  const long long ctas = static_cast<long long>(gx) * gy * gz;
  if (ctas > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  {  // column X first: it reads only the step's inputs
    const dim3 cgrid((p.Y + 1 + kColJ - 1) / kColJ, (p.Z + 1 + kColK - 1) / kColK, 1);
    class_column_kernel<Cpml, Exact, Lossy, Metric><<<cgrid, dim3(kColJ, kColK, 1), 0, s>>>(q);
    err = cudaPeekAtLastError();
    if (err != cudaSuccess) return err;
  }
  kern<<<dim3(static_cast<unsigned>(ctas), 1, 1), dim3(32, NW, 1), smem, s>>>(maps, q);
  return cudaPeekAtLastError();
}

template <int NW>
cudaError_t launch_class_shape(cudaStream_t s, const Step3D& p) {
  using T = ClassTile<NW>;
  ClassMaps maps;
  const int64_t P = p.pitch, rowb = P * 4, planeb = static_cast<int64_t>(p.Y + 1) * P * 4;
  for (int c = 0; c < 3; ++c) {
    const Dims de = component_dims(c, p.Z, p.Y, p.X), dh = component_dims(c + 3, p.Z, p.Y, p.X);
    if (!tma::encode(&maps.e[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.ein[c], de.x, de.y, de.z, rowb, planeb, T::BX,
                     T::EH) ||
        !tma::encode(&maps.h[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, p.hin[c], dh.x, dh.y, dh.z, rowb, planeb, T::BX,
                     T::HH))
      return cudaErrorInvalidValue;
  }
  const int64_t P8 = p.pitch8;
  if (!tma::encode(&maps.ids, CU_TENSOR_MAP_DATA_TYPE_UINT8, p.site_class, p.X + 1, p.Y + 1, p.Z + 1, P8,
                   P8 * (p.Y + 1), T::TX, T::TY))
    return cudaErrorInvalidValue;
  // Conductive material: the H classes, rows j0-1 .. and x from i0-16 (a
  // 16-byte coordinate for 1-byte elements), 144 bytes wide.
  if (p.lossy && !tma::encode(&maps.hids, CU_TENSOR_MAP_DATA_TYPE_UINT8, p.h_class, p.X + 1, p.Y + 1, p.Z + 1, P8,
                              P8 * (p.Y + 1), ClassTile<NW, true>::HW, T::HH))
    return cudaErrorInvalidValue;
  // x-term psi slabs (Hyx, Hzx, Eyx, Ezx): (plane, row, slot) with rows of
  // low + high slots.  Staged only when every row is a multiple of 16 bytes
  // and every slab 16-byte aligned (TMA's stride and base rules).
  Step3D q = p;
  q.xstage = 0;
  if (p.cpml) {
    const CpmlTermDev* xt[4] = {&p.ht[3], &p.ht[4], &p.et[3], &p.et[4]};
    const int comp[4] = {4, 5, 1, 2};  // Hy, Hz, Ey, Ez
    bool ok = true;
    for (int t = 0; t < 4 && ok; ++t) {
      const CpmlTermDev& d = *xt[t];
      const int w = d.low + d.high;
      const Dims dc = component_dims(comp[t], p.Z, p.Y, p.X);
      ok = w > 0 && w % 4 == 0 && d.pdx == w && (reinterpret_cast<uintptr_t>(d.psi_in) & 15) == 0 &&
           tma::encode(&maps.xpsi[t], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d.psi_in, w, d.pdy, dc.z, int64_t(w) * 4,
                       int64_t(w) * 4 * d.pdy, T::XW, T::HH);
    }
    q.xstage = ok ? 1 : 0;
  }
  if constexpr (NW == 8) {
    // Derivative metrics (axis-uniform / rectilinear grids): exact arithmetic
    // on lossless classes only (validated), 128 x 8 tiles.
    if (has_metric(q))
      return q.cpml ? launch_class_t<8, true, true, false, true>(s, maps, q)
                    : launch_class_t<8, false, true, false, true>(s, maps, q);
  }
  if (q.lossy)  // exact arithmetic only (validated)
    return q.cpml ? launch_class_t<NW, true, true, true>(s, maps, q) : launch_class_t<NW, false, true, true>(s, maps, q);
  if (q.fast_math) return q.cpml ? launch_class_t<NW, true, false>(s, maps, q) : launch_class_t<NW, false, false>(s, maps, q);
  return q.cpml ? launch_class_t<NW, true, true>(s, maps, q) : launch_class_t<NW, false, true>(s, maps, q);
}

}  // namespace

// tile_y: 8 (8 warps, 128 x 8 tiles) or 4 (4 warps, 128 x 4 tiles; programs
// with derivative metrics always take 8).
cudaError_t launch_class_step(cudaStream_t s, const Step3D& p, int tile_y) {
  return tile_y == 4 && !has_metric(p) ? launch_class_shape<4>(s, p) : launch_class_shape<8>(s, p);
}

}  // namespace fdtd
