/*
 * fdtd_cpu.c -- C restatement of the beamz leapfrog step on host memory.
 *
 * TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py and a second
 * CPU checker; nothing in the product links or loads it.  It consumes the same
 * FdtdProgram description as the CUDA library (include/fdtd_b200.h) with
 * HOST pointers and advances program->nsteps steps in beamz's phase order
 * (beamz/simulation/execute.py:467-541): pre-E sources, H with CPML
 * (kernels.py:458-503), H sources, H PEC, E with ghost planes and CPML
 * (kernels.py:554-626, lattice.py:523-575), E sources, E PEC, DFT
 * (observe.py:529-585).  Compile with -ffp-contract=off so that every float
 * operation rounds in source order, like the reference's float32 path.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../include/fdtd_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define EPS0_F 8.8541878128e-12f

typedef struct {
  int z, y, x;
} dims_t;

static dims_t cdims(int c, int Z, int Y, int X) {
  dims_t d;
  switch (c) {
    case 0: d.z = Z + 1; d.y = Y + 1; d.x = X; break;
    case 1: d.z = Z + 1; d.y = Y; d.x = X + 1; break;
    case 2: d.z = Z; d.y = Y + 1; d.x = X + 1; break;
    case 3: d.z = Z; d.y = Y; d.x = X + 1; break;
    case 4: d.z = Z; d.y = Y + 1; d.x = X; break;
    default: d.z = Z + 1; d.y = Y; d.x = X; break;
  }
  return d;
}

static inline int64_t L(dims_t d, int k, int j, int i) { return ((int64_t)k * d.y + j) * (int64_t)d.x + i; }
static inline int wall(int m, int axis, int high) { return (m >> (2 * axis + high)) & 1; }
static inline int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }
static int64_t nel(const FdtdBuffer* b) {
  int64_t n = 1;
  for (int a = 0; a < b->rank; ++a) n *= b->dims[a];
  return n;
}

typedef struct {
  int Z, Y, X, active, metallic, mat;
  float res;
  float dto;
  float* f[6];
  const FdtdProgram* p;
  /* term slot -> program term (3D identity, 2D mapped) */
  const FdtdCpmlTerm* ht[6];
  const FdtdCpmlTerm* et[6];
} ctx_t;

/* Derivative axis of each term slot (Hxy Hxz Hyz Hyx Hzx Hzy / Exy ... Ezy). */
static const int H_AXIS[6] = {1, 0, 0, 2, 2, 1};
static const int E_AXIS[6] = {1, 0, 0, 2, 2, 1};

static int slot_of(int ndim, int pol, int h, int t) {
  if (ndim == 3) return t;
  if (pol == 0) return h ? (t == 0 ? 0 : 3) : (t == 0 ? 4 : 5);
  return h ? (t == 0 ? 4 : 5) : (t == 0 ? 0 : 3);
}

/* d' = d / kappa + psi with psi <- b psi + a d inside the packed slabs. */
static inline float cpml(const FdtdCpmlTerm* t, dims_t target, int axis, float d, int k, int j, int i) {
  if (!t || t->low + t->high == 0) return d;
  const int n = axis == 0 ? target.z : (axis == 1 ? target.y : target.x);
  const int c = axis == 0 ? k : (axis == 1 ? j : i);
  int s = -1;
  if (c < t->low) s = c;
  else if (t->high > 0 && c >= n - t->high) s = t->low + c - (n - t->high);
  if (s < 0) return d;
  dims_t pd = target;
  const int w = t->low + t->high;
  if (axis == 0) pd.z = w;
  if (axis == 1) pd.y = w;
  if (axis == 2) pd.x = w;
  const int pk = axis == 0 ? s : k, pj = axis == 1 ? s : j, pi = axis == 2 ? s : i;
  float* psi = (float*)t->psi.data;
  const float* a = (const float*)t->a.data;
  const float* b = (const float*)t->b.data;
  const float* kk = (const float*)t->inv_kappa.data;
  const int64_t o = L(pd, pk, pj, pi);
  const float v = b[s] * psi[o] + a[s] * d;
  psi[o] = v;
  return d * kk[s] + v;
}

static inline float coef(const FdtdBuffer* b, int64_t o) {
  const float* p = (const float*)b->data;
  return nel(b) > 1 ? p[o] : p[0];
}

static inline float get(const ctx_t* x, int c, int k, int j, int i) {
  if (!((x->active >> c) & 1)) return 0.0f;
  return x->f[c][L(cdims(c, x->Z, x->Y, x->X), k, j, i)];
}

static inline float fd(const ctx_t* x, int c, int axis, int k, int j, int i) {
  if (!((x->active >> c) & 1)) return 0.0f;
  const float lo = get(x, c, k, j, i);
  const float hi = get(x, c, k + (axis == 0), j + (axis == 1), i + (axis == 2));
  return (hi - lo) / x->res;
}

static inline float bd(const ctx_t* x, int c, int axis, int k, int j, int i) {
  if (!((x->active >> c) & 1)) return 0.0f;
  const dims_t d = cdims(c, x->Z, x->Y, x->X);
  const int n = axis == 0 ? d.z : (axis == 1 ? d.y : d.x);
  const int co = axis == 0 ? k : (axis == 1 ? j : i);
  if (n == 0) return 0.0f;
  if (co == 0) return wall(x->metallic, axis, 0) ? (get(x, c, k, j, i) - 0.0f) / x->res : 0.0f;
  if (co == n)
    return wall(x->metallic, axis, 1)
               ? (0.0f - get(x, c, k - (axis == 0), j - (axis == 1), i - (axis == 2))) / x->res
               : 0.0f;
  return (get(x, c, k, j, i) - get(x, c, k - (axis == 0), j - (axis == 1), i - (axis == 2))) / x->res;
}

static inline float vox(const ctx_t* x, int k, int j, int i) {
  const uint8_t* v = (const uint8_t*)x->p->voxels.data;
  const float* t = (const float*)x->p->eps_table.data;
  k = clampi(k, x->Z - 1);
  j = clampi(j, x->Y - 1);
  i = clampi(i, x->X - 1);
  return t[v[((int64_t)k * x->Y + j) * x->X + i]];
}

static float site_eps(const ctx_t* x, int c, int k, int j, int i) {
  float a, b;
  if (c == 0) {
    a = 0.5f * (vox(x, k - 1, j - 1, i) + vox(x, k, j - 1, i));
    b = 0.5f * (vox(x, k - 1, j, i) + vox(x, k, j, i));
  } else if (c == 1) {
    a = 0.5f * (vox(x, k - 1, j, i - 1) + vox(x, k, j, i - 1));
    b = 0.5f * (vox(x, k - 1, j, i) + vox(x, k, j, i));
  } else {
    a = 0.5f * (vox(x, k, j - 1, i - 1) + vox(x, k, j, i - 1));
    b = 0.5f * (vox(x, k, j - 1, i) + vox(x, k, j, i));
  }
  return 0.5f * (a + b);
}

static void phase_h(const ctx_t* x) {
  static const int src0[3] = {2, 0, 1}, ax0[3] = {1, 0, 2};
  static const int src1[3] = {1, 2, 0}, ax1[3] = {0, 2, 1};
  for (int h = 0; h < 3; ++h) {
    const int c = 3 + h;
    if (!((x->active >> c) & 1)) continue;
    const dims_t d = cdims(c, x->Z, x->Y, x->X);
    const int normal = 2 - h;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < d.z; ++k)
      for (int j = 0; j < d.y; ++j)
        for (int i = 0; i < d.x; ++i) {
          float d0 = fd(x, src0[h], ax0[h], k, j, i);
          float d1 = fd(x, src1[h], ax1[h], k, j, i);
          d0 = cpml(x->ht[2 * h], d, H_AXIS[2 * h], d0, k, j, i);
          d1 = cpml(x->ht[2 * h + 1], d, H_AXIS[2 * h + 1], d1, k, j, i);
          const int64_t o = L(d, k, j, i);
          float v = coef(&x->p->h_decay[h], o) * x->f[c][o] - coef(&x->p->h_source_site[h], o) * (d0 - d1);
          const int co = normal == 0 ? k : (normal == 1 ? j : i);
          const int n = normal == 0 ? d.z : (normal == 1 ? d.y : d.x);
          if ((co == 0 && wall(x->metallic, normal, 0)) || (co == n - 1 && wall(x->metallic, normal, 1))) v = 0.0f;
          x->f[c][o] = v;
        }
  }
}

static void phase_e(const ctx_t* x) {
  static const int src0[3] = {5, 3, 4}, ax0[3] = {1, 0, 2};
  static const int src1[3] = {4, 5, 3}, ax1[3] = {0, 2, 1};
  for (int c = 0; c < 3; ++c) {
    if (!((x->active >> c) & 1)) continue;
    const dims_t d = cdims(c, x->Z, x->Y, x->X);
    const int normal = 2 - c;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < d.z; ++k)
      for (int j = 0; j < d.y; ++j)
        for (int i = 0; i < d.x; ++i) {
          float d0 = bd(x, src0[c], ax0[c], k, j, i);
          float d1 = bd(x, src1[c], ax1[c], k, j, i);
          d0 = cpml(x->et[2 * c], d, E_AXIS[2 * c], d0, k, j, i);
          d1 = cpml(x->et[2 * c + 1], d, E_AXIS[2 * c + 1], d1, k, j, i);
          const int64_t o = L(d, k, j, i);
          float v;
          if (x->mat == FDTD_MATERIAL_VOXEL) {
            const float inv = 1.0f / site_eps(x, c, k, j, i);
            v = x->f[c][o] + (x->dto * inv) * (d0 - d1);
          } else {
            v = coef(&x->p->e_decay[c], o) * x->f[c][o] + coef(&x->p->e_source[c], o) * (d0 - d1);
          }
          const int co[3] = {k, j, i};
          const int nn[3] = {d.z, d.y, d.x};
          for (int a = 0; a < 3; ++a) {
            if (a == normal) continue;
            if ((co[a] == 0 && wall(x->metallic, a, 0)) || (co[a] == nn[a] - 1 && wall(x->metallic, a, 1))) v = 0.0f;
          }
          x->f[c][o] = v;
        }
  }
}

static void sources(const ctx_t* x, int timing, int step) {
  const FdtdProgram* p = x->p;
  for (int s = 0; s < p->source_count; ++s) {
    const FdtdSource* src = &p->sources[s];
    if (src->timing != timing) continue;
    const int c = src->component;
    const dims_t d = cdims(c, x->Z, x->Y, x->X);
    int64_t ext[3] = {1, 1, 1};
    for (int a = 0; a < src->coeff.rank; ++a) ext[3 - src->coeff.rank + a] = src->coeff.dims[a];
    const int64_t wl = nel(&src->waveform);
    int w = step < 0 ? 0 : step;
    w = w >= wl ? (int)wl - 1 : w;
    const float amp = ((const float*)src->waveform.data)[w];
    const float* co = (const float*)src->coeff.data;
    for (int z = 0; z < ext[0]; ++z)
      for (int y = 0; y < ext[1]; ++y)
        for (int xx = 0; xx < ext[2]; ++xx) {
          const int k = src->start[0] + z, j = src->start[1] + y, i = src->start[2] + xx;
          const int64_t o = L(d, k, j, i);
          x->f[c][o] = x->f[c][o] + co[((int64_t)z * ext[1] + y) * ext[2] + xx] * amp;
        }
  }
}

static void zero_pec(const ctx_t* x, int electric) {
  /* Re-applies the masks after E/H-timing injections (execute.py:506-522). */
  for (int c = electric ? 0 : 3; c < (electric ? 3 : 6); ++c) {
    if (!((x->active >> c) & 1)) continue;
    const dims_t d = cdims(c, x->Z, x->Y, x->X);
    const int normal = electric ? 2 - c : 2 - (c - 3);
    for (int k = 0; k < d.z; ++k)
      for (int j = 0; j < d.y; ++j)
        for (int i = 0; i < d.x; ++i) {
          const int co[3] = {k, j, i};
          const int nn[3] = {d.z, d.y, d.x};
          int hit = 0;
          for (int a = 0; a < 3; ++a) {
            if (electric ? a == normal : a != normal) continue;
            if ((co[a] == 0 && wall(x->metallic, a, 0)) || (co[a] == nn[a] - 1 && wall(x->metallic, a, 1))) hit = 1;
          }
          if (hit) x->f[c][L(d, k, j, i)] = 0.0f;
        }
  }
}

static void dft(const ctx_t* x, int step) {
  const FdtdDft* m = &x->p->dft;
  if (m->monitor_count <= 0) return;
  const int K = (int)m->indices.dims[2], P = (int)m->indices.dims[3], F = (int)m->freqs.dims[1];
  const int* counts = (const int*)m->counts.data;
  const int* codes = (const int*)m->codes.data;
  const float* win = (const float*)m->windows.data;
  const float* st = (const float*)x->p->step_time.data;
  const int64_t stl = nel(&x->p->step_time);
  const float t = st[step < stl ? step : stl - 1];
  for (int mi = 0; mi < m->monitor_count; ++mi) {
    const int nf = counts[5 * mi], np = counts[5 * mi + 1];
    const int interval = counts[5 * mi + 2] > 0 ? counts[5 * mi + 2] : 1;
    const int voff = counts[5 * mi + 3], woff = counts[5 * mi + 4];
    const float t0 = win[3 * mi], t1 = win[3 * mi + 1], unit = win[3 * mi + 2];
    if (step % interval != 0 || !(t >= t0 && t <= t1)) continue;
    float window = 1.0f;
    if (codes[2 * mi] == 1 && isfinite(t1) && t1 > t0) {
      const float span = fmaxf(t1 - t0, 1e-30f);
      const float tau = fminf(fmaxf((t - t0) / span, 0.0f), 1.0f);
      window = 0.5f * (1.0f - cosf(6.2831855f * tau));
    }
    float scale = fmaxf(window, 0.0f);
    if (codes[2 * mi + 1] == 1) scale = scale * ((((x->p->dt * (float)interval) * 299792458.0f) / unit) / sqrtf(6.2831855f));
    float cs[64], sn[64];
    for (int f = 0; f < nf; ++f) {
      const float th = (6.2831855f * ((const float*)m->freqs.data)[mi * F + f]) * t;
      cs[f] = cosf(th);
      sn[f] = sinf(th);
    }
    float* ws = (float*)m->weight_sum.data;
    for (int f = 0; f < nf; ++f) ws[woff + f] += window;
    const float* masks = (const float*)m->masks.data;
    for (int c = 0; c < 6; ++c) {
      const float mk = masks[mi * 6 + c];
      if (mk == 0.0f) continue;
      const int* idx = (const int*)m->indices.data;
      const float* w = (const float*)m->weights.data;
      const float sm = scale * mk;
#pragma omp parallel for schedule(static)
      for (int pp = 0; pp < np; ++pp) {
        const int64_t base = (((int64_t)mi * 6 + c) * K) * P + pp;  /* neighbour-major */
        float v = 0.0f;
        for (int n = 0; n < K; ++n)
          if (w[base + (int64_t)n * P] != 0.0f) v = v + x->f[c][idx[base + (int64_t)n * P]] * w[base + (int64_t)n * P];
        const int64_t out = voff + (int64_t)c * nf * np + pp;
        for (int f = 0; f < nf; ++f) {
          ((float*)m->re.data)[out + (int64_t)f * np] += sm * (cs[f] * v);
          ((float*)m->im.data)[out + (int64_t)f * np] += sm * (sn[f] * v);
        }
      }
    }
  }
}

/* Advance program->nsteps steps on host memory; returns 0.  `threads` <= 0
 * keeps the OpenMP default.  step_counter (S32, host) is advanced. */
int fdtd_cpu_run(const FdtdProgram* p, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  ctx_t x;
  memset(&x, 0, sizeof(x));
  x.p = p;
  if (p->ndim == 3) {
    x.Z = (int)p->cells[0];
    x.Y = (int)p->cells[1];
    x.X = (int)p->cells[2];
    x.active = 0x3F;
    x.metallic = p->metallic_edges;
  } else {
    x.Z = p->polarization == 0 ? 1 : 0;
    x.Y = (int)p->cells[1];
    x.X = (int)p->cells[2];
    x.active = p->polarization == 0 ? 0x1C : 0x23;
    x.metallic = p->metallic_edges & ~3;
  }
  x.mat = p->material_kind;
  x.res = p->resolution;
  x.dto = p->dt_over_eps;
  for (int c = 0; c < 6; ++c) x.f[c] = (float*)p->fields[c].data;
  if (p->cpml) {
    const int nt = p->ndim == 3 ? 6 : 2;
    for (int t = 0; t < nt; ++t) {
      x.ht[slot_of(p->ndim, p->polarization, 1, t)] = &p->h_terms[t];
      x.et[slot_of(p->ndim, p->polarization, 0, t)] = &p->e_terms[t];
    }
  }
  int* counter = (int*)p->step_counter.data;
  for (int s = 0; s < p->nsteps; ++s) {
    const int step = counter[0];
    sources(&x, FDTD_TIMING_PRE_E, step);
    phase_h(&x);
    sources(&x, FDTD_TIMING_H, step);
    zero_pec(&x, 0);
    phase_e(&x);
    sources(&x, FDTD_TIMING_E, step);
    zero_pec(&x, 1);
    dft(&x, step);
    counter[0] = step + 1;
  }
  return 0;
}

int fdtd_cpu_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
