// C ABI: validation, parameter packing, step schedules and the CUDA-graph cache.
//
// beamz counterparts: program validation and schedules in cuda/src/program.cu
// (110-354), phase validation in cuda/src/update.cu (47-146) and the graph
// cache in cuda/src/graph.cu (11-154).

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>

#include "kernels.cuh"

namespace fdtd {
namespace {

constexpr int kInvalid = static_cast<int>(cudaErrorInvalidValue);

int64_t elements(const FdtdBuffer& b) {
  if (b.rank < 0 || b.rank > 4) return -1;
  int64_t n = 1;
  for (int a = 0; a < b.rank; ++a) {
    if (b.dims[a] < 0) return -1;
    n *= b.dims[a];
  }
  return n;
}

bool is_f32(const FdtdBuffer& b) { return b.element_type == FDTD_F32; }

struct Layout {
  int Z, Y, X;  // internal 3D cell extents (2D TM: Z = 1, 2D TE: Z = 0)
  int active;
};

bool layout_of(const FdtdProgram& p, Layout* out) {
  if (p.ndim == 3) {
    if (p.cells[0] < 1 || p.cells[1] < 1 || p.cells[2] < 1) return false;
    *out = {static_cast<int>(p.cells[0]), static_cast<int>(p.cells[1]), static_cast<int>(p.cells[2]), kActive3D};
  } else if (p.ndim == 2) {
    if (p.cells[1] < 1 || p.cells[2] < 1) return false;
    if (p.polarization == 0) {
      *out = {1, static_cast<int>(p.cells[1]), static_cast<int>(p.cells[2]), kActiveTM};
    } else if (p.polarization == 1) {
      *out = {0, static_cast<int>(p.cells[1]), static_cast<int>(p.cells[2]), kActiveTE};
    } else {
      return false;
    }
  } else {
    return false;
  }
  // The step kernels use 32-bit element offsets: every component array must
  // hold fewer than 2^31 elements.
  for (int c = 0; c < 6; ++c) {
    const Dims d = component_dims(c, out->Z, out->Y, out->X);
    if (static_cast<int64_t>(d.z) * d.y * d.x >= (int64_t{1} << 31)) return false;
  }
  return true;
}

int64_t dims_count(const Dims& d) { return static_cast<int64_t>(d.z) * d.y * d.x; }

// 2D programs name CPML axes in (y, x) storage terms and use two terms per
// phase; they land in the 3D term slots that carry the same derivative.
int term_slot(int ndim, int pol, bool h, int t) {
  if (ndim == 3) return t;
  if (pol == 0) return h ? (t == 0 ? 0 : 3) : (t == 0 ? 4 : 5);
  return h ? (t == 0 ? 4 : 5) : (t == 0 ? 0 : 3);
}

// Target component and derivative axis of each 3D term slot.
constexpr int kHTermComp[6] = {3, 3, 4, 4, 5, 5};
constexpr int kHTermAxis[6] = {1, 0, 0, 2, 2, 1};
constexpr int kETermComp[6] = {0, 0, 1, 1, 2, 2};
constexpr int kETermAxis[6] = {1, 0, 0, 2, 2, 1};

bool check_coeff(const FdtdBuffer& b, int64_t full) {
  if (!is_f32(b) || b.data == nullptr) return false;
  const int64_t n = elements(b);
  return n == 1 || n == full;
}

bool has_metric(const FdtdProgram& p) {
  for (int a = 0; a < 3; ++a)
    if (p.metric_h[a].data != nullptr || p.metric_e[a].data != nullptr) return true;
  return false;
}

int validate(const FdtdProgram& p) {
  if (p.abi_version != FDTD_ABI_VERSION) return kInvalid;
  Layout L;
  if (!layout_of(p, &L)) return kInvalid;
  if (p.schedule != FDTD_SCHEDULE_PHASES && p.schedule != FDTD_SCHEDULE_FUSED) return kInvalid;
  if (p.schedule == FDTD_SCHEDULE_PHASES && p.layout != FDTD_LAYOUT_DENSE) return kInvalid;
  if (p.material_kind != FDTD_MATERIAL_SITE && p.material_kind != FDTD_MATERIAL_VOXEL &&
      p.material_kind != FDTD_MATERIAL_CODEBOOK)
    return kInvalid;
  if (p.material_kind == FDTD_MATERIAL_VOXEL && p.ndim != 3) return kInvalid;
  if (p.nsteps < 0 || p.source_count < 0 || p.source_count > FDTD_MAX_SOURCES) return kInvalid;
  if (!(p.resolution > 0.0f) || !(p.inv_resolution > 0.0f)) return kInvalid;
  if (p.metallic_edges & ~0x3F) return kInvalid;
  const bool pitched = p.layout == FDTD_LAYOUT_PITCHED;
  if (p.layout != FDTD_LAYOUT_DENSE && !pitched) return kInvalid;
  if (pitched) {
    // 3D codebook programs with uniform H coefficients; 16-byte-aligned rows.
    if (p.ndim != 3 || p.material_kind != FDTD_MATERIAL_CODEBOOK) return kInvalid;
    if (p.pitch < L.X + 1 || p.pitch % 4 != 0) return kInvalid;
    if (static_cast<int64_t>(L.Z + 1) * (L.Y + 1) * p.pitch >= (int64_t{1} << 31)) return kInvalid;
  } else if (p.material_kind == FDTD_MATERIAL_CODEBOOK) {
    return kInvalid;  // the codebook shares the pitched field layout
  }
  auto field_ok = [&](const FdtdBuffer& b, int64_t n) {
    if (!is_f32(b)) return false;
    if (!pitched) return elements(b) == n && (n == 0 || b.data != nullptr);
    return b.rank == 3 && b.dims[0] == L.Z + 1 && b.dims[1] == L.Y + 1 && b.dims[2] == p.pitch &&
           b.data != nullptr && (reinterpret_cast<uintptr_t>(b.data) & 15) == 0;
  };
  for (int c = 0; c < 6; ++c) {
    if (!((L.active >> c) & 1)) continue;
    const int64_t n = dims_count(component_dims(c, L.Z, L.Y, L.X));
    if (!field_ok(p.fields[c], n)) return kInvalid;
    if (p.schedule == FDTD_SCHEDULE_FUSED && !field_ok(p.fields_alt[c], n)) return kInvalid;
    if (pitched && (elements(p.h_decay[c % 3]) != 1 || elements(p.h_source_site[c % 3]) != 1)) return kInvalid;
    if (c < 3) {
      if (p.material_kind == FDTD_MATERIAL_SITE &&
          (!check_coeff(p.e_decay[c], n) || !check_coeff(p.e_source[c], n)))
        return kInvalid;
    } else {
      if (!check_coeff(p.h_decay[c - 3], n) || !check_coeff(p.h_source_site[c - 3], n)) return kInvalid;
    }
  }
  if (has_metric(p)) {
    // On the pitched layout, only the class step carries metrics, in exact
    // arithmetic on lossless classes.
    if (pitched && (!(p.flags & FDTD_FLAG_CLASSES) || (p.flags & (FDTD_FLAG_FAST_MATH | FDTD_FLAG_LOSSY))))
      return kInvalid;
    for (int a = 0; a < 3; ++a) {
      const int n = a == 0 ? L.Z : (a == 1 ? L.Y : L.X);
      const FdtdBuffer &mh = p.metric_h[a], &me = p.metric_e[a];
      if (p.ndim == 2 && a == 0) {
        if (mh.data != nullptr || me.data != nullptr) return kInvalid;
        continue;
      }
      if (!is_f32(mh) || mh.rank != 1 || mh.dims[0] != n || mh.data == nullptr) return kInvalid;
      if (!is_f32(me) || me.rank != 1 || me.dims[0] != n + 1 || me.data == nullptr) return kInvalid;
    }
  }
  if (p.material_kind == FDTD_MATERIAL_VOXEL) {
    if (p.voxels.element_type != FDTD_U8 || p.voxels.data == nullptr) return kInvalid;
    if (elements(p.voxels) != static_cast<int64_t>(L.Z) * L.Y * L.X) return kInvalid;
    if (!is_f32(p.eps_table) || elements(p.eps_table) != 256 || p.eps_table.data == nullptr) return kInvalid;
  }
  if (p.material_kind == FDTD_MATERIAL_CODEBOOK) {
    const FdtdBuffer& ids = p.site_ids;
    if (ids.element_type != FDTD_S32 || ids.rank != 3 || ids.dims[0] != L.Z + 1 || ids.dims[1] != L.Y + 1 ||
        ids.dims[2] != p.pitch || ids.data == nullptr || (reinterpret_cast<uintptr_t>(ids.data) & 15) != 0)
      return kInvalid;
    if (!is_f32(p.site_coef) || elements(p.site_coef) != 3 * 256 || p.site_coef.data == nullptr) return kInvalid;
  }
  if (p.flags & FDTD_FLAG_CLASSES) {
    // The class step: uint8 classes on 16-byte rows, a
    // 256-entry class table.
    if (!pitched) return kInvalid;
    const FdtdBuffer& cls = p.site_class;
    if (cls.element_type != FDTD_U8 || cls.rank != 3 || cls.dims[0] != L.Z + 1 || cls.dims[1] != L.Y + 1 ||
        cls.dims[2] < L.X + 1 || cls.dims[2] % 16 != 0 || cls.data == nullptr ||
        (reinterpret_cast<uintptr_t>(cls.data) & 15) != 0)
      return kInvalid;
    if (static_cast<int64_t>(L.Z + 1) * (L.Y + 1) * cls.dims[2] >= (int64_t{1} << 31)) return kInvalid;
    if (!is_f32(p.class_coef) || elements(p.class_coef) != 4 * 256 || p.class_coef.data == nullptr ||
        (reinterpret_cast<uintptr_t>(p.class_coef.data) & 15) != 0)
      return kInvalid;
  }
  if ((p.flags & FDTD_FLAG_FAST_MATH) && !(p.flags & FDTD_FLAG_CLASSES)) return kInvalid;
  if (p.flags & FDTD_FLAG_LOSSY) {
    // Conductive classes: exact arithmetic, H classes on the E classes' rows.
    if (!(p.flags & FDTD_FLAG_CLASSES) || (p.flags & FDTD_FLAG_FAST_MATH)) return kInvalid;
    const FdtdBuffer &cls = p.site_class, &hc = p.h_class;
    if (hc.element_type != FDTD_U8 || hc.rank != 3 || hc.data == nullptr ||
        (reinterpret_cast<uintptr_t>(hc.data) & 15) != 0)
      return kInvalid;
    for (int a = 0; a < 3; ++a)
      if (hc.dims[a] != cls.dims[a]) return kInvalid;
    if (!is_f32(p.h_class_coef) || elements(p.h_class_coef) != 64 * 4 * 2 || p.h_class_coef.data == nullptr)
      return kInvalid;
  }
  if ((p.flags & FDTD_FLAG_TEST_STALL) && !pitched) return kInvalid;
  if (p.wait_limit_ns < 0) return kInvalid;
  if (p.cpml) {
    const int nterms = p.ndim == 3 ? 6 : 2;
    for (int h = 0; h < 2; ++h) {
      for (int t = 0; t < nterms; ++t) {
        const FdtdCpmlTerm& term = h ? p.h_terms[t] : p.e_terms[t];
        const int slot = term_slot(p.ndim, p.polarization, h, t);
        const int comp = h ? kHTermComp[slot] : kETermComp[slot];
        const int axis = h ? kHTermAxis[slot] : kETermAxis[slot];
        const int given_axis = p.ndim == 3 ? term.axis : term.axis + 1;
        if (given_axis != axis) return kInvalid;
        const Dims d = component_dims(comp, L.Z, L.Y, L.X);
        const int n_axis = axis == 0 ? d.z : (axis == 1 ? d.y : d.x);
        if (term.low < 0 || term.high < 0 || term.low + term.high > n_axis) return kInvalid;
        const int w = term.low + term.high;
        if (w == 0) continue;
        for (const FdtdBuffer* b : {&term.a, &term.b, &term.inv_kappa}) {
          if (!is_f32(*b) || elements(*b) < w || b->data == nullptr) return kInvalid;
        }
        Dims pd = d;
        if (axis == 0) pd.z = w;
        if (axis == 1) pd.y = w;
        if (axis == 2) pd.x = w;
        if (!is_f32(term.psi) || elements(term.psi) != dims_count(pd) || term.psi.data == nullptr) return kInvalid;
        if (h && p.schedule == FDTD_SCHEDULE_FUSED &&
            (!is_f32(term.psi_alt) || elements(term.psi_alt) != dims_count(pd) || term.psi_alt.data == nullptr))
          return kInvalid;
      }
    }
  }
  for (int s = 0; s < p.source_count; ++s) {
    const FdtdSource& src = p.sources[s];
    if (src.component < 0 || src.component > 5 || !((L.active >> src.component) & 1)) return kInvalid;
    if (src.timing < FDTD_TIMING_PRE_E || src.timing > FDTD_TIMING_E) return kInvalid;
    const bool is_h = src.component >= 3;
    if ((src.timing == FDTD_TIMING_H) != is_h) return kInvalid;
    if (!is_f32(src.coeff) || src.coeff.data == nullptr || src.coeff.rank < 1 || src.coeff.rank > 3) return kInvalid;
    if (!is_f32(src.waveform) || src.waveform.data == nullptr || elements(src.waveform) < 1) return kInvalid;
    const Dims d = component_dims(src.component, L.Z, L.Y, L.X);
    int64_t ext[3] = {1, 1, 1};
    for (int a = 0; a < src.coeff.rank; ++a) ext[3 - src.coeff.rank + a] = src.coeff.dims[a];
    const int64_t lo[3] = {src.start[0], src.start[1], src.start[2]};
    const int64_t hi[3] = {d.z, d.y, d.x};
    for (int a = 0; a < 3; ++a) {
      if (ext[a] < 1 || lo[a] < 0 || lo[a] + ext[a] > hi[a]) return kInvalid;
    }
  }
  if (p.step_counter.element_type != FDTD_S32 || elements(p.step_counter) < 1 || p.step_counter.data == nullptr)
    return kInvalid;
  if (p.status.data != nullptr && (p.status.element_type != FDTD_S32 || elements(p.status) < 1)) return kInvalid;
  if (p.dft.monitor_count < 0 || p.dft.monitor_count > FDTD_MAX_MONITORS) return kInvalid;
  if (p.dft.monitor_count > 0) {
    const FdtdDft& d = p.dft;
    const int M = d.monitor_count;
    if (d.indices.element_type != FDTD_S32 || d.indices.rank != 4 || d.indices.dims[0] != M || d.indices.dims[1] != 6)
      return kInvalid;
    if (!is_f32(d.weights) || d.weights.rank != 4) return kInvalid;
    for (int a = 0; a < 4; ++a)
      if (d.weights.dims[a] != d.indices.dims[a]) return kInvalid;
    if (!is_f32(d.freqs) || d.freqs.rank != 2 || d.freqs.dims[0] != M || d.freqs.dims[1] > 64) return kInvalid;
    if (!is_f32(d.masks) || elements(d.masks) != 6 * M) return kInvalid;
    if (d.counts.element_type != FDTD_S32 || elements(d.counts) != 5 * M) return kInvalid;
    if (d.codes.element_type != FDTD_S32 || elements(d.codes) != 2 * M) return kInvalid;
    if (!is_f32(d.windows) || elements(d.windows) != 3 * M) return kInvalid;
    if (!is_f32(d.re) || !is_f32(d.im) || elements(d.re) != elements(d.im) || !is_f32(d.weight_sum)) return kInvalid;
    if (!is_f32(p.step_time) || elements(p.step_time) < 1 || p.step_time.data == nullptr) return kInvalid;
    for (const FdtdBuffer* b : {&d.indices, &d.weights, &d.freqs, &d.masks, &d.counts, &d.codes, &d.windows, &d.re,
                                &d.im, &d.weight_sum})
      if (b->data == nullptr && elements(*b) > 0) return kInvalid;
    if (d.batch < 0 || d.batch > 16) return kInvalid;
    if (d.affine.data != nullptr && (d.affine.element_type != FDTD_S32 || elements(d.affine) != 24 * 6 * M))
      return kInvalid;
    if (d.samples.data != nullptr &&
        (!is_f32(d.samples) || elements(d.samples) != static_cast<int64_t>(d.batch) * M * 6 * d.indices.dims[3]))
      return kInvalid;
  }
  if (p.recorder_count < 0 || p.recorder_count > FDTD_MAX_RECORDERS) return kInvalid;
  if (p.recorder_count > 0 && (!is_f32(p.step_time) || elements(p.step_time) < 1 || p.step_time.data == nullptr))
    return kInvalid;
  for (int r = 0; r < p.recorder_count; ++r) {
    const FdtdRecorder& rec = p.recorders[r];
    if (rec.interval < 1 || rec.capacity < 0 || rec.component_count < 1 || rec.component_count > 6) return kInvalid;
    const int64_t cap = rec.capacity;
    if (rec.steps.element_type != FDTD_S32 || elements(rec.steps) != cap || (cap > 0 && rec.steps.data == nullptr))
      return kInvalid;
    if (!is_f32(rec.times) || elements(rec.times) != cap || (cap > 0 && rec.times.data == nullptr)) return kInvalid;
    if (rec.count.element_type != FDTD_S32 || elements(rec.count) != 2 || rec.count.data == nullptr) return kInvalid;
    for (int q = 0; q < rec.component_count; ++q) {
      const int c = rec.components[q];
      if (c < 0 || c > 5 || !((L.active >> c) & 1)) return kInvalid;
      const FdtdBuffer &ix = rec.indices[q], &w = rec.weights[q];
      int64_t V;
      if (ix.data == nullptr && w.data == nullptr) {
        V = dims_count(component_dims(c, L.Z, L.Y, L.X));
      } else {
        if (ix.element_type != FDTD_S32 || !is_f32(w) || ix.rank != 2 || w.rank != 2 || ix.data == nullptr ||
            w.data == nullptr || ix.dims[0] != w.dims[0] || ix.dims[1] != w.dims[1] || ix.dims[0] < 1 ||
            ix.dims[0] > 32)
          return kInvalid;
        V = ix.dims[1];
      }
      if (!is_f32(rec.values[q]) || elements(rec.values[q]) != cap * V || (cap * V > 0 && rec.values[q].data == nullptr))
        return kInvalid;
    }
  }
  return 0;
}

// Device view of recorder r reading the component arrays of `bank`.
RecorderDev recorder_dev(const FdtdProgram& p, const Layout& L, int r, const FdtdBuffer* bank) {
  const FdtdRecorder& rec = p.recorders[r];
  RecorderDev d;
  d.interval = rec.interval;
  d.capacity = rec.capacity;
  d.ncomp = rec.component_count;
  const bool pitched = p.layout == FDTD_LAYOUT_PITCHED;
  for (int q = 0; q < d.ncomp; ++q) {
    const int c = rec.components[q];
    const Dims cd = component_dims(c, L.Z, L.Y, L.X);
    d.sign[q] = rec.signs[q];
    d.field[q] = static_cast<const float*>(bank[c].data);
    d.field_len[q] = elements(bank[c]);
    d.dy[q] = cd.y;
    d.dx[q] = cd.x;
    d.row[q] = pitched ? p.pitch : cd.x;
    d.plane[q] = pitched ? p.pitch * (L.Y + 1) : static_cast<int64_t>(cd.y) * cd.x;
    int64_t V;
    if (rec.indices[q].data == nullptr) {
      V = dims_count(cd);
    } else {
      d.slots[q] = static_cast<int>(rec.indices[q].dims[0]);
      d.idx[q] = static_cast<const int*>(rec.indices[q].data);
      d.w[q] = static_cast<const float*>(rec.weights[q].data);
      V = rec.indices[q].dims[1];
    }
    d.values[q] = static_cast<float*>(rec.values[q].data);
    d.start[q + 1] = d.start[q] + V;
  }
  d.steps = static_cast<int*>(rec.steps.data);
  d.times = static_cast<float*>(rec.times.data);
  d.count = static_cast<int*>(rec.count.data);
  d.step_time = static_cast<const float*>(p.step_time.data);
  d.step_time_len = static_cast<int>(elements(p.step_time));
  return d;
}

CpmlTermDev term_dev(const FdtdCpmlTerm& t, const Dims& target, int axis, bool alt_in, bool alt_out) {
  CpmlTermDev d{};
  d.low = t.low;
  d.high = t.high;
  // An empty term keeps its true axis extent so that no coordinate maps into it.
  d.n_axis = axis == 0 ? target.z : (axis == 1 ? target.y : target.x);
  if (t.low + t.high == 0) return d;
  d.a = static_cast<const float*>(t.a.data);
  d.b = static_cast<const float*>(t.b.data);
  d.k = static_cast<const float*>(t.inv_kappa.data);
  d.psi_in = static_cast<const float*>(alt_in ? t.psi_alt.data : t.psi.data);
  d.psi_out = static_cast<float*>(alt_out ? t.psi_alt.data : t.psi.data);
  const int w = t.low + t.high;
  d.pdy = axis == 1 ? w : target.y;
  d.pdx = axis == 2 ? w : target.x;
  return d;
}

// Kernel parameters for one step.  `bank` selects which field bank is the input
// (0 = fields, 1 = fields_alt); for the one-bank schedule input == output.
Step3D make_step(const FdtdProgram& p, const Layout& L, int bank, bool fused, int step_offset) {
  Step3D s{};
  s.Z = L.Z;
  s.Y = L.Y;
  s.X = L.X;
  const FdtdBuffer* in = bank == 0 ? p.fields : p.fields_alt;
  const FdtdBuffer* out = fused ? (bank == 0 ? p.fields_alt : p.fields) : in;
  for (int c = 0; c < 3; ++c) {
    s.ein[c] = static_cast<const float*>(in[c].data);
    s.eout[c] = static_cast<float*>(out[c].data);
    s.hin[c] = static_cast<const float*>(in[c + 3].data);
    s.hout[c] = static_cast<float*>(out[c + 3].data);
  }
  s.res = p.resolution;
  s.inv_res = p.inv_resolution;
  s.div_bs = p.resolution * kDivScale;
  s.div_rs = p.inv_resolution * kDivUnscale;
  s.dt_over_eps = p.dt_over_eps;
  s.metallic = p.metallic_edges;
  if (p.ndim == 2) s.metallic &= ~(FDTD_EDGE_FRONT | FDTD_EDGE_BACK);
  s.cpml = p.cpml;
  for (int c = 0; c < 3; ++c) {
    const bool ea = (L.active >> c) & 1, ha = (L.active >> (c + 3)) & 1;
    if (ea && p.material_kind == FDTD_MATERIAL_SITE) {
      s.em.decay[c] = static_cast<const float*>(p.e_decay[c].data);
      s.em.source[c] = static_cast<const float*>(p.e_source[c].data);
      s.em.decay_full[c] = elements(p.e_decay[c]) > 1;
      s.em.source_full[c] = elements(p.e_source[c]) > 1;
    }
    if (ha) {
      s.hm.decay[c] = static_cast<const float*>(p.h_decay[c].data);
      s.hm.source[c] = static_cast<const float*>(p.h_source_site[c].data);
      s.hm.decay_full[c] = elements(p.h_decay[c]) > 1;
      s.hm.source_full[c] = elements(p.h_source_site[c]) > 1;
    }
  }
  if (p.material_kind == FDTD_MATERIAL_VOXEL) {
    s.em.voxels = static_cast<const uint8_t*>(p.voxels.data);
    s.em.eps_table = static_cast<const float*>(p.eps_table.data);
  }
  if (p.material_kind == FDTD_MATERIAL_CODEBOOK) {
    s.em.site_ids = static_cast<const uint32_t*>(p.site_ids.data);
    s.em.site_coef = static_cast<const float*>(p.site_coef.data);
  }
  if (p.cpml) {
    const int nterms = p.ndim == 3 ? 6 : 2;
    for (int t = 0; t < nterms; ++t) {
      const int hs = term_slot(p.ndim, p.polarization, true, t);
      const int es = term_slot(p.ndim, p.polarization, false, t);
      const Dims hd = component_dims(kHTermComp[hs], L.Z, L.Y, L.X);
      const Dims ed = component_dims(kETermComp[es], L.Z, L.Y, L.X);
      // H memories are double-banked under the fused schedule.
      s.ht[hs] = term_dev(p.h_terms[t], hd, kHTermAxis[hs], fused && bank == 1, fused && bank == 0);
      s.et[es] = term_dev(p.e_terms[t], ed, kETermAxis[es], false, false);
    }
  }
  s.step_counter = static_cast<const int*>(p.step_counter.data);
  s.step_offset = step_offset;
  s.z_chunk = p.z_chunk;
  s.pitch = static_cast<int>(p.pitch);
  s.status = static_cast<int*>(p.status.data);
  s.wait_ns = p.wait_limit_ns > 0 ? static_cast<unsigned long long>(p.wait_limit_ns) : 200000000ull;
  s.test_stall = (p.flags & FDTD_FLAG_TEST_STALL) ? 1 : 0;
  if (p.flags & FDTD_FLAG_CLASSES) {
    s.fast_math = (p.flags & FDTD_FLAG_FAST_MATH) ? 1 : 0;
    s.site_class = static_cast<const uint8_t*>(p.site_class.data);
    s.pitch8 = static_cast<int>(p.site_class.dims[2]);
    s.class_coef = static_cast<const float4*>(p.class_coef.data);
    s.lossy = (p.flags & FDTD_FLAG_LOSSY) ? 1 : 0;
    s.h_class = static_cast<const uint8_t*>(p.h_class.data);
    s.h_class_coef = static_cast<const float2*>(p.h_class_coef.data);
  }
  for (int a = 0; a < 3; ++a) {
    s.metric_h[a] = static_cast<const float*>(p.metric_h[a].data);
    s.metric_e[a] = static_cast<const float*>(p.metric_e[a].data);
  }
  // An axis without absorber terms has no slab anywhere, the faces included.
  for (int a = 0; a < 3; ++a) {
    s.cpml_inner[a][0] = -(1 << 30);
    s.cpml_inner[a][1] = 1 << 30;
  }
  if (p.cpml) {
    for (int t = 0; t < 6; ++t) {
      for (const CpmlTermDev* d : {&s.ht[t], &s.et[t]}) {
        const int a = (d == &s.ht[t] ? kHTermAxis : kETermAxis)[t];
        if (d->low + d->high == 0) continue;
        s.cpml_inner[a][0] = d->low > s.cpml_inner[a][0] ? d->low : s.cpml_inner[a][0];
        if (s.cpml_inner[a][0] < 0) s.cpml_inner[a][0] = 0;
        const int hi = d->n_axis - d->high;
        s.cpml_inner[a][1] = hi < s.cpml_inner[a][1] ? hi : s.cpml_inner[a][1];
      }
    }
  }
  return s;
}

SourceDev source_dev(const FdtdSource& src) {
  SourceDev d{};
  d.coeff = static_cast<const float*>(src.coeff.data);
  d.waveform = static_cast<const float*>(src.waveform.data);
  d.wave_len = static_cast<int>(elements(src.waveform));
  d.component = src.component;
  d.z0 = src.start[0];
  d.y0 = src.start[1];
  d.x0 = src.start[2];
  int64_t ext[3] = {1, 1, 1};
  for (int a = 0; a < src.coeff.rank; ++a) ext[3 - src.coeff.rank + a] = src.coeff.dims[a];
  d.ez = static_cast<int>(ext[0]);
  d.ey = static_cast<int>(ext[1]);
  d.ex = static_cast<int>(ext[2]);
  return d;
}

cudaError_t enqueue_sources(cudaStream_t s, const FdtdProgram& p, const Layout& L, const FdtdBuffer* bank_fields,
                            int timing, int step_offset) {
  const int metallic = p.ndim == 2 ? (p.metallic_edges & ~(FDTD_EDGE_FRONT | FDTD_EDGE_BACK)) : p.metallic_edges;
  for (int i = 0; i < p.source_count; ++i) {
    const FdtdSource& src = p.sources[i];
    if (src.timing != timing) continue;
    const Dims td = component_dims(src.component, L.Z, L.Y, L.X);
    const bool pitched = p.layout == FDTD_LAYOUT_PITCHED;
    const int64_t row = pitched ? p.pitch : td.x;
    const int64_t plane = pitched ? (L.Y + 1) * p.pitch : static_cast<int64_t>(td.y) * td.x;
    cudaError_t err = launch_source(s, source_dev(src), static_cast<float*>(bank_fields[src.component].data), td, row,
                                    plane, timing, metallic, static_cast<const int*>(p.step_counter.data), step_offset);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

DftDev make_dft(const FdtdProgram& p, const FdtdBuffer* bank_fields) {
  DftDev d{};
  const FdtdDft& m = p.dft;
  d.monitor_count = m.monitor_count;
  if (m.monitor_count == 0) return d;
  d.max_points = static_cast<int>(m.indices.dims[3]);
  d.neighbors = static_cast<int>(m.indices.dims[2]);
  d.max_freqs = static_cast<int>(m.freqs.dims[1]);
  d.indices = static_cast<const int*>(m.indices.data);
  d.weights = static_cast<const float*>(m.weights.data);
  d.freqs = static_cast<const float*>(m.freqs.data);
  d.masks = static_cast<const float*>(m.masks.data);
  d.counts = static_cast<const int*>(m.counts.data);
  d.codes = static_cast<const int*>(m.codes.data);
  d.windows = static_cast<const float*>(m.windows.data);
  d.re = static_cast<float*>(m.re.data);
  d.im = static_cast<float*>(m.im.data);
  d.weight_sum = static_cast<float*>(m.weight_sum.data);
  d.arena_len = elements(m.re);
  d.weight_len = elements(m.weight_sum);
  for (int c = 0; c < 6; ++c) {
    d.fields[c] = static_cast<const float*>(bank_fields[c].data);
    d.field_len[c] = elements(bank_fields[c]);
  }
  d.step_time = static_cast<const float*>(p.step_time.data);
  d.step_time_len = static_cast<int>(elements(p.step_time));
  d.dt = p.dt;
  d.affine = static_cast<const int*>(m.affine.data);
  return d;
}

// ---- DFT sampling beside the next step --------------------------------------
// With FDTD_FLAG_DFT_OVERLAP, step n's sample runs on a side stream while step
// n+1 (which only reads that bank) runs on the caller's stream; step n+2, which
// overwrites the bank, waits for it, and every call joins the side stream
// before the step counter advances.  One side stream (higher priority, so its
// small blocks take the SM room the step kernel leaves) and its events per
// (device, caller stream), created outside any capture and kept until exit.
struct SideStream {
  cudaStream_t side = nullptr;
  cudaEvent_t step_done = nullptr;
  cudaEvent_t sample_done[2] = {nullptr, nullptr};
  cudaEvent_t joined = nullptr;
};

std::mutex& side_mutex() {
  static std::mutex* m = new std::mutex();
  return *m;
}

std::map<std::pair<int, cudaStream_t>, SideStream>& side_table() {
  static auto* t = new std::map<std::pair<int, cudaStream_t>, SideStream>();
  return *t;
}

// The side stream of `s`, created when `create` (never while `s` captures);
// nullptr when absent.
cudaError_t side_stream_of(cudaStream_t s, bool create, SideStream** out) {
  *out = nullptr;
  int device = 0;
  cudaError_t err = cudaGetDevice(&device);
  if (err != cudaSuccess) return err;
  std::lock_guard<std::mutex> lock(side_mutex());
  auto& table = side_table();
  const auto key = std::make_pair(device, s);
  auto it = table.find(key);
  if (it != table.end()) {
    *out = &it->second;
    return cudaSuccess;
  }
  if (!create) return cudaSuccess;
  SideStream ss;
  int least = 0, greatest = 0;
  err = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (err == cudaSuccess) err = cudaStreamCreateWithPriority(&ss.side, cudaStreamNonBlocking, greatest);
  cudaEvent_t* events[4] = {&ss.step_done, &ss.sample_done[0], &ss.sample_done[1], &ss.joined};
  for (cudaEvent_t* e : events)
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(e, cudaEventDisableTiming);
  if (err != cudaSuccess) {
    for (cudaEvent_t* e : events)
      if (*e) cudaEventDestroy(*e);
    if (ss.side) cudaStreamDestroy(ss.side);
    return err;
  }
  *out = &table.emplace(key, ss).first->second;
  return cudaSuccess;
}

bool wants_side_stream(const FdtdProgram& p) {
  return (p.flags & FDTD_FLAG_DFT_OVERLAP) != 0 && p.schedule == FDTD_SCHEDULE_FUSED && p.dft.monitor_count > 0 &&
         p.dft.batch > 1 && p.dft.samples.data != nullptr;
}

// Enqueue `nsteps` steps.  Under the fused schedule step s reads bank (s & 1).
cudaError_t enqueue_program(cudaStream_t s, const FdtdProgram& p) {
  Layout L;
  layout_of(p, &L);
  const bool fused = p.schedule == FDTD_SCHEDULE_FUSED;
  const int* counter = static_cast<const int*>(p.step_counter.data);
  // Sources of H timing ride inside the fused kernel.
  int n_hsrc = 0;
  SourceDev hsrc[kMaxFusedSources];
  for (int i = 0; i < p.source_count; ++i)
    if (p.sources[i].timing == FDTD_TIMING_H) hsrc[n_hsrc++] = source_dev(p.sources[i]);
  // ... and, for 2D programs, the pre-E sources (added to the staged E planes,
  // so the bank itself is never written before the step).
  const bool fuse_pre_e = fused && p.layout == FDTD_LAYOUT_DENSE && L.active != kActive3D;
  int n_esrc = 0;
  SourceDev esrc[kMaxFusedSources];
  if (fuse_pre_e)
    for (int i = 0; i < p.source_count; ++i)
      if (p.sources[i].timing == FDTD_TIMING_PRE_E) esrc[n_esrc++] = source_dev(p.sources[i]);
  // DFT step batching (validated: batch <= 16, samples sized [batch, M, 6, P]).
  const bool batched = p.dft.monitor_count > 0 && p.dft.batch > 1 && p.dft.samples.data != nullptr;
  float* samples = static_cast<float*>(p.dft.samples.data);
  int batch_start = 0;
  // Side stream for the samples (FDTD_FLAG_DFT_OVERLAP); while `s` captures, an
  // absent one is not created and the samples stay on `s`.
  SideStream* ss = nullptr;
  if (wants_side_stream(p)) {
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(s, &status);
    if (err != cudaSuccess) return err;
    err = side_stream_of(s, status == cudaStreamCaptureStatusNone, &ss);
    if (err != cudaSuccess) return err;
  }
  const cudaStream_t ds = ss ? ss->side : s;
  for (int step = 0; step < p.nsteps; ++step) {
    const int bank = fused ? (step & 1) : 0;
    const FdtdBuffer* a = bank == 0 ? p.fields : p.fields_alt;
    const FdtdBuffer* b = fused ? (bank == 0 ? p.fields_alt : p.fields) : a;
    cudaError_t err = fuse_pre_e ? cudaSuccess : enqueue_sources(s, p, L, a, FDTD_TIMING_PRE_E, step);
    if (err != cudaSuccess) return err;
    Step3D sp = make_step(p, L, bank, fused, step);
    if (ss && step >= 2) {  // step `step` overwrites the bank that sample step-2 reads
      err = cudaStreamWaitEvent(s, ss->sample_done[step & 1], 0);
      if (err != cudaSuccess) return err;
    }
    if (fused) {
      sp.n_hsrc = n_hsrc;
      for (int i = 0; i < n_hsrc; ++i) sp.hsrc[i] = hsrc[i];
      sp.n_esrc = n_esrc;
      for (int i = 0; i < n_esrc; ++i) sp.esrc[i] = esrc[i];
      if (p.layout == FDTD_LAYOUT_PITCHED && (p.flags & FDTD_FLAG_CLASSES)) {
        err = launch_class_step(s, sp, p.tile_y);
      } else if (p.layout == FDTD_LAYOUT_PITCHED) {
        err = launch_fused_tma(s, sp, p.tile_y);
      } else if (L.active == kActive3D) {
        err = launch_fused_lean(s, sp, p.material_kind, p.tile_y);
      } else {
        err = launch_fused(s, sp, p.material_kind, L.active, p.tile_x, p.tile_y);
      }
      if (err != cudaSuccess) return err;
    } else {
      err = launch_phase(s, sp, 0, p.material_kind, L.active);
      if (err != cudaSuccess) return err;
      err = enqueue_sources(s, p, L, a, FDTD_TIMING_H, step);
      if (err != cudaSuccess) return err;
      err = launch_phase(s, sp, 1, p.material_kind, L.active);
      if (err != cudaSuccess) return err;
    }
    err = enqueue_sources(s, p, L, b, FDTD_TIMING_E, step);
    if (err != cudaSuccess) return err;
    if (p.dft.monitor_count > 0 && batched) {
      const DftDev dd = make_dft(p, b);
      if (ss) {
        err = cudaEventRecord(ss->step_done, s);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(ds, ss->step_done, 0);
        if (err != cudaSuccess) return err;
      }
      err = launch_dft_sample(ds, dd, samples, step - batch_start);
      if (err != cudaSuccess) return err;
      if (ss) {
        err = cudaEventRecord(ss->sample_done[step & 1], ds);
        if (err != cudaSuccess) return err;
      }
      if (step - batch_start + 1 == p.dft.batch || step == p.nsteps - 1) {
        err = launch_dft_flush(ds, dd, samples, counter, batch_start, step - batch_start + 1);
        if (err != cudaSuccess) return err;
        batch_start = step + 1;
      }
    } else if (p.dft.monitor_count > 0) {
      err = launch_dft(s, make_dft(p, b), counter, step);
      if (err != cudaSuccess) return err;
    }
    for (int r = 0; r < p.recorder_count; ++r) {
      err = launch_record(s, recorder_dev(p, L, r, b), counter, step);
      if (err != cudaSuccess) return err;
    }
  }
  if (ss) {  // join: the flush reads the step counter, and callers read the arena
    cudaError_t err = cudaEventRecord(ss->joined, ds);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s, ss->joined, 0);
    if (err != cudaSuccess) return err;
  }
  if (p.nsteps > 0) return launch_counter_advance(s, static_cast<int*>(p.step_counter.data), p.nsteps);
  return cudaSuccess;
}

// ---- graph cache (beamz: cuda/src/graph.cu:84-154) -------------------------
struct GraphCache {
  std::mutex mu;
  std::unordered_map<std::string, cudaGraphExec_t> graphs;
};

GraphCache& cache() {
  static GraphCache* c = new GraphCache();
  return *c;
}

constexpr size_t kMaxGraphs = 32;

std::string graph_key(const FdtdProgram& p, cudaStream_t s) {
  int device = 0;
  cudaGetDevice(&device);
  std::string key(reinterpret_cast<const char*>(&p), sizeof(FdtdProgram));
  key.append(reinterpret_cast<const char*>(&s), sizeof(s));
  key.append(reinterpret_cast<const char*>(&device), sizeof(device));
  return key;
}

cudaError_t launch_with_graph(cudaStream_t s, const FdtdProgram& p) {
  cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
  cudaError_t err = cudaStreamIsCapturing(s, &status);
  if (err != cudaSuccess) return err;
  if (status != cudaStreamCaptureStatusNone || s == nullptr) return enqueue_program(s, p);
  if (wants_side_stream(p)) {
    SideStream* ss = nullptr;
    err = side_stream_of(s, true, &ss);
    if (err != cudaSuccess) return err;
  }
  const std::string key = graph_key(p, s);
  GraphCache& gc = cache();
  std::lock_guard<std::mutex> lock(gc.mu);
  auto it = gc.graphs.find(key);
  if (it == gc.graphs.end()) {
    err = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) {
      cudaGetLastError();
      return enqueue_program(s, p);
    }
    cudaError_t enq = enqueue_program(s, p);
    cudaGraph_t graph = nullptr;
    err = cudaStreamEndCapture(s, &graph);
    if (enq != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return enq;
    }
    if (err != cudaSuccess) return err;
    cudaGraphExec_t exec = nullptr;
    err = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) return err;
    if (gc.graphs.size() >= kMaxGraphs) {
      for (auto& kv : gc.graphs) cudaGraphExecDestroy(kv.second);
      gc.graphs.clear();
    }
    it = gc.graphs.emplace(key, exec).first;
  }
  return cudaGraphLaunch(it->second, s);
}

// Capture one program into a caller-owned executable graph.
cudaError_t capture_program(cudaStream_t s, const FdtdProgram& p, cudaGraphExec_t* out) {
  if (wants_side_stream(p)) {
    SideStream* ss = nullptr;
    const cudaError_t e = side_stream_of(s, true, &ss);
    if (e != cudaSuccess) return e;
  }
  cudaError_t err = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return err;
  const cudaError_t enq = enqueue_program(s, p);
  cudaGraph_t graph = nullptr;
  err = cudaStreamEndCapture(s, &graph);
  if (enq != cudaSuccess || err != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return enq != cudaSuccess ? enq : err;
  }
  err = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  return err;
}

}  // namespace
}  // namespace fdtd

extern "C" {

int fdtd_abi_version(void) { return FDTD_ABI_VERSION; }

int64_t fdtd_program_size(void) { return static_cast<int64_t>(sizeof(FdtdProgram)); }

int fdtd_validate(const FdtdProgram* program) {
  if (program == nullptr) return fdtd::kInvalid;
  return fdtd::validate(*program);
}

int fdtd_launch_phase(void* stream, const FdtdProgram* program, int32_t phase) {
  if (program == nullptr || (phase != 0 && phase != 1)) return fdtd::kInvalid;
  if (program->layout != FDTD_LAYOUT_DENSE) return fdtd::kInvalid;
  FdtdProgram p = *program;
  p.schedule = FDTD_SCHEDULE_PHASES;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  const fdtd::Step3D sp = fdtd::make_step(p, L, 0, false, 0);
  return static_cast<int>(
      fdtd::launch_phase(static_cast<cudaStream_t>(stream), sp, phase, p.material_kind, L.active));
}

int fdtd_launch_program(void* stream, const FdtdProgram* program) {
  if (program == nullptr) return fdtd::kInvalid;
  const int v = fdtd::validate(*program);
  if (v != 0) return v;
  if (program->nsteps == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (program->flags & FDTD_FLAG_GRAPH_CACHE) return static_cast<int>(fdtd::launch_with_graph(s, *program));
  return static_cast<int>(fdtd::enqueue_program(s, *program));
}

int fdtd_apply_sources(void* stream, const FdtdProgram* program, int32_t timing, int32_t step_offset) {
  if (program == nullptr) return fdtd::kInvalid;
  FdtdProgram p = *program;
  p.schedule = FDTD_SCHEDULE_PHASES;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  if (timing < FDTD_TIMING_PRE_E || timing > FDTD_TIMING_E) return fdtd::kInvalid;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  return static_cast<int>(
      fdtd::enqueue_sources(static_cast<cudaStream_t>(stream), p, L, p.fields, timing, step_offset));
}

int fdtd_accumulate_dft(void* stream, const FdtdProgram* program, int32_t step_offset) {
  if (program == nullptr) return fdtd::kInvalid;
  FdtdProgram p = *program;
  p.schedule = FDTD_SCHEDULE_PHASES;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  if (p.dft.monitor_count == 0) return 0;
  return static_cast<int>(fdtd::launch_dft(static_cast<cudaStream_t>(stream), fdtd::make_dft(p, p.fields),
                                           static_cast<const int*>(p.step_counter.data), step_offset));
}

int fdtd_record_fields(void* stream, const FdtdProgram* program, int32_t step_offset) {
  if (program == nullptr) return fdtd::kInvalid;
  FdtdProgram p = *program;
  p.schedule = FDTD_SCHEDULE_PHASES;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  for (int r = 0; r < p.recorder_count; ++r) {
    const cudaError_t err = fdtd::launch_record(static_cast<cudaStream_t>(stream), fdtd::recorder_dev(p, L, r, p.fields),
                                                static_cast<const int*>(p.step_counter.data), step_offset);
    if (err != cudaSuccess) return static_cast<int>(err);
  }
  return 0;
}

int fdtd_copy_component(void* stream, const FdtdBuffer* src, const FdtdBuffer* dst, const int64_t* extent) {
  if (src == nullptr || dst == nullptr || extent == nullptr) return fdtd::kInvalid;
  if (src->element_type != FDTD_F32 || dst->element_type != FDTD_F32 || src->rank != 3 || dst->rank != 3)
    return fdtd::kInvalid;
  for (int a = 0; a < 3; ++a)
    if (extent[a] < 0 || extent[a] > src->dims[a] || extent[a] > dst->dims[a]) return fdtd::kInvalid;
  if (extent[0] * extent[1] * extent[2] == 0) return 0;
  if (src->data == nullptr || dst->data == nullptr) return fdtd::kInvalid;
  return static_cast<int>(fdtd::launch_copy3d(static_cast<cudaStream_t>(stream), static_cast<const float*>(src->data),
                                              src->dims[2], src->dims[1] * src->dims[2],
                                              static_cast<float*>(dst->data), dst->dims[2],
                                              dst->dims[1] * dst->dims[2], extent[0], extent[1], extent[2]));
}

namespace fdtd {
namespace {

bool f32_sized(const FdtdBuffer& b, int64_t n) { return is_f32(b) && b.data != nullptr && elements(b) == n; }

// Shared checks of an adjoint call: a valid dense phase program and a box
// whose curl needs no ghost, wall or CPML handling.
int check_adjoint(const FdtdProgram& p, const FdtdAdjointStep& a, const Layout& L, bool need_box) {
  if (a.abi_version != FDTD_ABI_VERSION) return kInvalid;
  if (p.layout != FDTD_LAYOUT_DENSE) return kInvalid;
  const int64_t bz = a.box_hi[0] - a.box_lo[0], by = a.box_hi[1] - a.box_lo[1], bx = a.box_hi[2] - a.box_lo[2];
  bool any_box = false;
  for (int c = 0; c < 3; ++c) any_box = any_box || a.curl[c].data != nullptr || a.grad[c].data != nullptr;
  if (!any_box) return need_box ? kInvalid : 0;
  if (bz <= 0 || by <= 0 || bx <= 0) return kInvalid;
  const int lo[3] = {a.box_lo[0], a.box_lo[1], a.box_lo[2]}, hi[3] = {a.box_hi[0], a.box_hi[1], a.box_hi[2]};
  const int ext[3] = {L.Z, L.Y, L.X};
  for (int c = 0; c < 3; ++c) {
    if (!((L.active >> c) & 1)) {
      if (a.curl[c].data != nullptr || a.grad[c].data != nullptr) return kInvalid;
      continue;
    }
    if ((a.curl[c].data != nullptr && !f32_sized(a.curl[c], bz * by * bx)) ||
        (a.grad[c].data != nullptr && !f32_sized(a.grad[c], bz * by * bx)))
      return kInvalid;
    if (a.grad[c].data != nullptr && a.curl[c].data == nullptr) return kInvalid;
    // Axes the component is differentiated along need a lower neighbour and
    // stay below the H extent; its own axis spans the E extent.
    for (int ax = 0; ax < 3; ++ax) {
      const bool derived = ax != 2 - c;
      const int need_lo = derived ? 1 : 0;
      const int need_hi = derived ? ext[ax] : ext[ax];
      if (lo[ax] < need_lo || hi[ax] > need_hi) return kInvalid;
    }
    if (p.cpml) {
      for (int t = 2 * c; t < 2 * c + 2; ++t) {
        const int ax = kETermAxis[t];
        for (int s = 0; s < (p.ndim == 3 ? 6 : 2); ++s) {
          if (term_slot(p.ndim, p.polarization, false, s) != t) continue;
          const FdtdCpmlTerm& term = p.e_terms[s];
          const Dims d = component_dims(c, L.Z, L.Y, L.X);
          const int n = ax == 0 ? d.z : (ax == 1 ? d.y : d.x);
          if (lo[ax] < term.low || hi[ax] > n - term.high) return kInvalid;
        }
      }
    }
  }
  return 0;
}

// Elements of each derivative term's adjoint scratch (0 for a term between
// inactive components): an E term's target E component, an H term's target H
// component.  Both adjoint entry points size their scratch from this.
void adjoint_term_lengths(const Layout& L, int64_t e_len[6], int64_t h_len[6]) {
  for (int t = 0; t < 6; ++t) {
    const int ec = kETermComp[t], hsrc = (t == 0 || t == 3) ? 5 : ((t == 1 || t == 4) ? 4 : 3);
    e_len[t] = ((L.active >> ec) & 1) && ((L.active >> hsrc) & 1)
                   ? dims_count(component_dims(ec, L.Z, L.Y, L.X))
                   : 0;
    const int hc = kHTermComp[t], esrc = (t == 0 || t == 3) ? 2 : ((t == 1 || t == 4) ? 1 : 0);
    h_len[t] = ((L.active >> hc) & 1) && ((L.active >> esrc) & 1)
                   ? dims_count(component_dims(hc, L.Z, L.Y, L.X))
                   : 0;
  }
}

AdjDev adjoint_dev(const FdtdProgram& p, const FdtdAdjointStep& a) {
  AdjDev d{};
  for (int c = 0; c < 6; ++c) d.lam[c] = static_cast<float*>(p.fields[c].data);
  for (int t = 0; t < 6; ++t) {
    d.scratch_e[t] = static_cast<float*>(a.scratch_e[t].data);
    d.scratch_h[t] = static_cast<float*>(a.scratch_h[t].data);
  }
  d.dft_grad_re = static_cast<const float*>(a.dft_grad_re.data);
  d.dft_grad_im = static_cast<const float*>(a.dft_grad_im.data);
  for (int c = 0; c < 3; ++c) {
    d.curl[c] = static_cast<float*>(a.curl[c].data);
    d.grad[c] = static_cast<float*>(a.grad[c].data);
    d.box_lo[c] = a.box_lo[c];
    d.box_hi[c] = a.box_hi[c];
  }
  return d;
}

}  // namespace
}  // namespace fdtd

int fdtd_adjoint_step(void* stream, const FdtdProgram* adjoint, const FdtdAdjointStep* a) {
  if (adjoint == nullptr || a == nullptr) return fdtd::kInvalid;
  FdtdProgram p = *adjoint;
  p.schedule = FDTD_SCHEDULE_PHASES;
  if (p.material_kind != FDTD_MATERIAL_SITE) return fdtd::kInvalid;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  const int b = fdtd::check_adjoint(p, *a, L, false);
  if (b != 0) return b;
  // Every derivative term between two active components needs its scratch.
  int64_t e_len[6], h_len[6];
  fdtd::adjoint_term_lengths(L, e_len, h_len);
  for (int t = 0; t < 6; ++t) {
    if (e_len[t] > 0 ? !fdtd::f32_sized(a->scratch_e[t], e_len[t]) : a->scratch_e[t].data != nullptr)
      return fdtd::kInvalid;
    if (h_len[t] > 0 ? !fdtd::f32_sized(a->scratch_h[t], h_len[t]) : a->scratch_h[t].data != nullptr)
      return fdtd::kInvalid;
  }
  const bool dft = p.dft.monitor_count > 0 && a->dft_grad_re.data != nullptr;
  fdtd::DftDev dd{};
  if (dft) {
    dd = fdtd::make_dft(p, p.fields);
    if (!fdtd::f32_sized(a->dft_grad_re, dd.arena_len) || !fdtd::f32_sized(a->dft_grad_im, dd.arena_len))
      return fdtd::kInvalid;
  }
  const fdtd::Step3D sp = fdtd::make_step(p, L, 0, false, 0);
  return static_cast<int>(fdtd::launch_adjoint_step(static_cast<cudaStream_t>(stream), sp, dft ? &dd : nullptr,
                                                    fdtd::adjoint_dev(p, *a), L.active, a->step));
}

int fdtd_adjoint_step_noalloc(void* stream, const FdtdProgram* adjoint, const FdtdAdjointStep* a) {
  if (adjoint == nullptr || a == nullptr) return fdtd::kInvalid;
  FdtdProgram p = *adjoint;
  p.schedule = FDTD_SCHEDULE_PHASES;
  if (p.material_kind != FDTD_MATERIAL_SITE) return fdtd::kInvalid;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  const int b = fdtd::check_adjoint(p, *a, L, false);
  if (b != 0) return b;
  int64_t e_len[6], h_len[6];
  fdtd::adjoint_term_lengths(L, e_len, h_len);
  for (int t = 0; t < 6; ++t)
    if (a->scratch_e[t].data != nullptr || a->scratch_h[t].data != nullptr) return fdtd::kInvalid;
  // The scratch bound is checked once, by the launcher, before any work is enqueued.
  const bool dft = p.dft.monitor_count > 0 && a->dft_grad_re.data != nullptr;
  fdtd::DftDev dd{};
  if (dft) {
    dd = fdtd::make_dft(p, p.fields);
    if (!fdtd::f32_sized(a->dft_grad_re, dd.arena_len) || !fdtd::f32_sized(a->dft_grad_im, dd.arena_len))
      return fdtd::kInvalid;
  }
  const fdtd::Step3D sp = fdtd::make_step(p, L, 0, false, 0);
  return static_cast<int>(fdtd::launch_adjoint_step_noalloc(static_cast<cudaStream_t>(stream), sp,
                                                            dft ? &dd : nullptr, fdtd::adjoint_dev(p, *a), L.active,
                                                            a->step, e_len, h_len));
}

int fdtd_adjoint_curl(void* stream, const FdtdProgram* forward, const FdtdAdjointStep* a) {
  if (forward == nullptr || a == nullptr) return fdtd::kInvalid;
  FdtdProgram p = *forward;
  p.schedule = FDTD_SCHEDULE_PHASES;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  const int b = fdtd::check_adjoint(p, *a, L, true);
  if (b != 0) return b;
  const fdtd::Step3D sp = fdtd::make_step(p, L, 0, false, 0);
  return static_cast<int>(
      fdtd::launch_adjoint_curl(static_cast<cudaStream_t>(stream), sp, fdtd::adjoint_dev(p, *a), L.active));
}

int fdtd_field_diagnostics(void* stream, const FdtdProgram* program, const FdtdDiagnostics* d) {
  if (program == nullptr || d == nullptr) return fdtd::kInvalid;
  const FdtdProgram& p = *program;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  fdtd::Layout L;
  fdtd::layout_of(p, &L);
  auto f64_at_least = [](const FdtdBuffer& b, int64_t n) {
    return b.element_type == FDTD_F64 && b.data != nullptr && fdtd::elements(b) >= n;
  };
  if (!f64_at_least(d->partials, int64_t{6} * FDTD_DIAG_BLOCKS * 3) || !f64_at_least(d->out, 18))
    return fdtd::kInvalid;
  const bool pitched = p.layout == FDTD_LAYOUT_PITCHED;
  const bool codebook = p.material_kind == FDTD_MATERIAL_CODEBOOK;
  if (codebook && (!fdtd::is_f32(d->site_eps_table) || d->site_eps_table.data == nullptr ||
                   fdtd::elements(d->site_eps_table) != 3 * 256))
    return fdtd::kInvalid;
  fdtd::DiagArgs a;
  a.active = L.active;
  a.partials = static_cast<double*>(d->partials.data);
  for (int c = 0; c < 6; ++c) {
    if (!((L.active >> c) & 1)) continue;
    fdtd::DiagComp& q = a.comp[c];
    q.field = static_cast<const float*>(p.fields[c].data);
    q.d = fdtd::component_dims(c, L.Z, L.Y, L.X);
    q.row = pitched ? p.pitch : q.d.x;
    q.plane = pitched ? static_cast<int64_t>(L.Y + 1) * p.pitch : static_cast<int64_t>(q.d.y) * q.d.x;
    q.integrate_z = p.ndim == 3 ? 1 : 0;
    q.edge_z = q.d.z == L.Z + 1 ? 1 : 0;
    q.edge_y = q.d.y == L.Y + 1 ? 1 : 0;
    q.edge_x = q.d.x == L.X + 1 ? 1 : 0;
    if (c >= 3) continue;  // non-magnetic: mu_r = 1
    if (codebook) {
      q.ids = static_cast<const uint32_t*>(p.site_ids.data);
      q.shift = 8 * c;
      q.table = static_cast<const float*>(d->site_eps_table.data) + 256 * c;
    } else if (d->site_eps[c].data != nullptr) {
      const int64_t n = static_cast<int64_t>(q.d.z) * q.d.y * q.d.x;
      if (!fdtd::is_f32(d->site_eps[c]) || d->site_eps[c].data == nullptr || fdtd::elements(d->site_eps[c]) != n)
        return fdtd::kInvalid;
      q.eps = static_cast<const float*>(d->site_eps[c].data);
    }
  }
  return static_cast<int>(
      fdtd::launch_field_diagnostics(static_cast<cudaStream_t>(stream), a, static_cast<double*>(d->out.data)));
}

int fdtd_dft_change(void* stream, const FdtdProgram* program, const FdtdDftChange* c) {
  if (program == nullptr || c == nullptr) return fdtd::kInvalid;
  const FdtdProgram& p = *program;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  if (p.dft.monitor_count <= 0) return fdtd::kInvalid;
  const int64_t arena = fdtd::elements(p.dft.re);
  for (const FdtdBuffer* b : {&c->prev_re, &c->prev_im})
    if (!fdtd::is_f32(*b) || b->data == nullptr || fdtd::elements(*b) != arena) return fdtd::kInvalid;
  const fdtd::DftDev dd = fdtd::make_dft(p, p.fields);
  const int64_t keys = static_cast<int64_t>(dd.monitor_count) * 6 * dd.max_freqs;
  if (c->out.element_type != FDTD_F64 || c->out.data == nullptr || fdtd::elements(c->out) < keys * 3)
    return fdtd::kInvalid;
  return static_cast<int>(fdtd::launch_dft_change(static_cast<cudaStream_t>(stream), dd,
                                                  static_cast<float*>(c->prev_re.data),
                                                  static_cast<float*>(c->prev_im.data),
                                                  static_cast<double*>(c->out.data)));
}

int fdtd_monitor_reduce(void* stream, const FdtdProgram* program, const FdtdMonitorReduce* r) {
  if (program == nullptr || r == nullptr) return fdtd::kInvalid;
  const FdtdProgram& p = *program;
  const int v = fdtd::validate(p);
  if (v != 0) return v;
  if (r->abi_version != FDTD_ABI_VERSION || p.dft.monitor_count <= 0) return fdtd::kInvalid;
  const int64_t arena = fdtd::elements(p.dft.re);
  const int64_t F = r->freq_count, P = r->point_count;
  if (F < 1 || P < 0 || r->value_offset < 0 || r->rows < 0 || r->value_offset + 6 * F * P > arena)
    return fdtd::kInvalid;
  for (int q = 0; q < 2; ++q)
    if (r->e[q] < 0 || r->e[q] > 2 || r->h[q] < 3 || r->h[q] > 5) return fdtd::kInvalid;
  auto f64 = [](const FdtdBuffer& b, int64_t n) {
    return b.element_type == FDTD_F64 && fdtd::elements(b) == n && (n == 0 || b.data != nullptr);
  };
  const int64_t rows = r->rows > 0 ? r->rows : 1;
  if (!f64(r->scale, F * 3) || !f64(r->weights, 2 * P) || !f64(r->out, rows * F * 4)) return fdtd::kInvalid;
  if (r->rows > 0 && (!f64(r->profile_re, rows * F * 4 * P) || !f64(r->profile_im, rows * F * 4 * P)))
    return fdtd::kInvalid;
  fdtd::MonitorReduceDev d;
  d.re = static_cast<const float*>(p.dft.re.data);
  d.im = static_cast<const float*>(p.dft.im.data);
  d.value_offset = r->value_offset;
  d.points = P;
  d.freqs = static_cast<int>(F);
  d.rows = r->rows;
  for (int q = 0; q < 2; ++q) {
    d.e[q] = r->e[q];
    d.h[q] = r->h[q];
  }
  d.scale = static_cast<const double*>(r->scale.data);
  d.weights = static_cast<const double*>(r->weights.data);
  d.prof_re = static_cast<const double*>(r->profile_re.data);
  d.prof_im = static_cast<const double*>(r->profile_im.data);
  d.out = static_cast<double*>(r->out.data);
  return static_cast<int>(fdtd::launch_monitor_reduce(static_cast<cudaStream_t>(stream), d));
}

int fdtd_pack_gather(void* stream, const FdtdGatherPack* g) {
  if (g == nullptr) return fdtd::kInvalid;
  const FdtdBuffer &ii = g->indices_in, &wi = g->weights_in, &io = g->indices_out, &wo = g->weights_out;
  if (ii.element_type != FDTD_S32 || !fdtd::is_f32(wi) || io.element_type != FDTD_S32 || !fdtd::is_f32(wo))
    return fdtd::kInvalid;
  if (ii.rank != 2 || wi.rank != 2 || io.rank != 2 || wo.rank != 2) return fdtd::kInvalid;
  if (wi.dims[0] != ii.dims[0] || wi.dims[1] != ii.dims[1] || wo.dims[0] != io.dims[0] || wo.dims[1] != io.dims[1])
    return fdtd::kInvalid;
  const int64_t points = ii.dims[0], slots = ii.dims[1], K = io.dims[0], pmax = io.dims[1];
  if (K < 1 || points > pmax || slots > 32 || pmax >= (int64_t{1} << 31)) return fdtd::kInvalid;
  if (g->dims[0] < 1 || g->dims[1] < 1 || g->dims[2] < 1 || g->row < g->dims[2] ||
      g->plane < g->row * static_cast<int64_t>(g->dims[1]) ||
      static_cast<int64_t>(g->dims[0]) * g->plane >= (int64_t{1} << 31))
    return fdtd::kInvalid;
  if (points > 0 && (ii.data == nullptr || wi.data == nullptr || io.data == nullptr || wo.data == nullptr))
    return fdtd::kInvalid;
  fdtd::GatherPackDev d;
  d.idx_in = static_cast<const int*>(ii.data);
  d.w_in = static_cast<const float*>(wi.data);
  d.idx_out = static_cast<int*>(io.data);
  d.w_out = static_cast<float*>(wo.data);
  d.points = static_cast<int>(points);
  d.slots_in = static_cast<int>(slots);
  d.pmax = static_cast<int>(pmax);
  d.rows = static_cast<int>(K < slots ? K : slots);
  d.dz = g->dims[0];
  d.dy = g->dims[1];
  d.dx = g->dims[2];
  d.row = g->row;
  d.plane = g->plane;
  return static_cast<int>(fdtd::launch_gather_pack(static_cast<cudaStream_t>(stream), d));
}

int fdtd_voxel_histogram(void* stream, const FdtdBuffer* voxels, const FdtdBuffer* counts) {
  if (voxels == nullptr || counts == nullptr) return fdtd::kInvalid;
  if (voxels->element_type != FDTD_U8 || counts->element_type != FDTD_S32 || fdtd::elements(*counts) != 256 ||
      counts->data == nullptr)
    return fdtd::kInvalid;
  const int64_t n = fdtd::elements(*voxels);
  if (n < 0 || (n > 0 && voxels->data == nullptr)) return fdtd::kInvalid;
  return static_cast<int>(fdtd::launch_voxel_histogram(static_cast<cudaStream_t>(stream),
                                                       static_cast<const uint8_t*>(voxels->data), n,
                                                       static_cast<int*>(counts->data)));
}

int fdtd_graph_create(void* stream, const FdtdProgram* program, void** graph) {
  if (program == nullptr || graph == nullptr || stream == nullptr || program->nsteps < 1) return fdtd::kInvalid;
  *graph = nullptr;
  const int v = fdtd::validate(*program);
  if (v != 0) return v;
  cudaGraphExec_t exec = nullptr;
  const cudaError_t err = fdtd::capture_program(static_cast<cudaStream_t>(stream), *program, &exec);
  if (err != cudaSuccess) return static_cast<int>(err);
  *graph = static_cast<void*>(exec);
  return 0;
}

int fdtd_graph_launch(void* stream, void* graph) {
  if (graph == nullptr) return fdtd::kInvalid;
  return static_cast<int>(cudaGraphLaunch(static_cast<cudaGraphExec_t>(graph), static_cast<cudaStream_t>(stream)));
}

int fdtd_graph_destroy(void* graph) {
  if (graph == nullptr) return 0;
  return static_cast<int>(cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph)));
}

void fdtd_clear_graph_cache(void) {
  fdtd::GraphCache& gc = fdtd::cache();
  std::lock_guard<std::mutex> lock(gc.mu);
  for (auto& kv : gc.graphs) cudaGraphExecDestroy(kv.second);
  gc.graphs.clear();
}

const char* fdtd_error_string(int code) { return cudaGetErrorString(static_cast<cudaError_t>(code)); }

const FdtdRegistration* fdtd_registrations(int32_t* count) {
  static const FdtdRegistration table[] = {
      {"fdtd_phase", reinterpret_cast<void*>(&fdtd_launch_phase)},
      {"fdtd_program", reinterpret_cast<void*>(&fdtd_launch_program)},
  };
  if (count != nullptr) *count = static_cast<int32_t>(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // extern "C"
