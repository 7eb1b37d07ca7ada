// Device helpers shared by the phase and fused step kernels, and the host
// launcher declarations.
#pragma once

#include "params.cuh"

namespace fdtd {

// Active-component masks (bit c = component c, order Ex Ey Ez Hx Hy Hz).
constexpr int kActive3D = 0x3F;
constexpr int kActiveTM = (1 << 2) | (1 << 3) | (1 << 4);  // Ez Hx Hy
constexpr int kActiveTE = (1 << 0) | (1 << 1) | (1 << 5);  // Ex Ey Hz

// H <- decay * H - source * curl (beamz: cuda/src/update.cu:402-409; with
// decay == 1 and source == fl(dt)/fl(mu0) this is kernels.py:497-500 exactly).
__device__ __forceinline__ float h_update(const HMaterial& m, int c, int64_t o, float h, float curl) {
  const float dec = m.decay[c][m.decay_full[c] ? o : 0];
  const float src = m.source[c][m.source_full[c] ? o : 0];
  return dec * h - src * curl;
}

__device__ __forceinline__ int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

__device__ __forceinline__ int axis_cells(const Step3D& p, int axis) { return axis == 0 ? p.Z : (axis == 1 ? p.Y : p.X); }

// Does the program carry derivative metrics (FdtdProgram.metric_h/_e)?
__host__ __device__ inline bool has_metric(const Step3D& p) {
  return p.metric_h[0] != nullptr || p.metric_h[1] != nullptr || p.metric_h[2] != nullptr;
}

// A forward difference of E along `axis` at H coordinate `c`, as a derivative:
// divided by the cell size (kernels.py:477-488), or with Metric times the
// inverse distance of a metric grid (beamz/simulation/kernels.py:164-176,
// 293-323; cuda/src/update.cu:172-203).  Kernels are instantiated per Metric
// so the isotropic step carries no metric test.  Coordinates of halo cells
// that are never stored are clamped into the metric; an axis without one (z
// of a 2D program, whose z differences are of inactive components) divides.
template <bool Metric>
__device__ __forceinline__ float dh(const Step3D& p, int axis, int c, float diff) {
  if constexpr (Metric) {
    const float* m = p.metric_h[axis];
    if (m != nullptr) return diff * m[clampi(c, axis_cells(p, axis) - 1)];
  }
  return div_rn(diff, p.div_bs, p.div_rs);
}

// dh / de with the coordinate's inverse distance already loaded (kernels that
// hoist the metric out of their loops), or divided by the cell size.
template <bool Metric>
__device__ __forceinline__ float dm(const Step3D& p, float diff, float m) {
  if constexpr (Metric) return diff * m;
  return div_rn(diff, p.div_bs, p.div_rs);
}

// A backward difference of H along `axis` at E coordinate `c` (0..n_axis).
template <bool Metric>
__device__ __forceinline__ float de(const Step3D& p, int axis, int c, float diff) {
  if constexpr (Metric) {
    const float* m = p.metric_e[axis];
    if (m != nullptr) return diff * m[clampi(c, axis_cells(p, axis))];
  }
  return div_rn(diff, p.div_bs, p.div_rs);
}

__device__ __forceinline__ float vox_eps(const EMaterial& m, int Z, int Y, int X, int k, int j, int i) {
  k = clampi(k, Z - 1);
  j = clampi(j, Y - 1);
  i = clampi(i, X - 1);
  return m.eps_table[m.voxels[(static_cast<int64_t>(k) * Y + j) * X + i]];
}

// Centered E-site permittivity from the voxel grid, in the averaging order of
// beamz/lattice.py:732-786 (axes z, y, x; 0.5 * (lo + hi) on face-aligned axes).
__device__ __forceinline__ float site_eps(const Step3D& p, int c, int k, int j, int i) {
  const EMaterial& m = p.em;
  const int Z = p.Z, Y = p.Y, X = p.X;
  if (c == 0) {  // Ex: average z, then y; x owned.
    const float a = 0.5f * (vox_eps(m, Z, Y, X, k - 1, j - 1, i) + vox_eps(m, Z, Y, X, k, j - 1, i));
    const float b = 0.5f * (vox_eps(m, Z, Y, X, k - 1, j, i) + vox_eps(m, Z, Y, X, k, j, i));
    return 0.5f * (a + b);
  }
  if (c == 1) {  // Ey: average z, then x; y owned.
    const float a = 0.5f * (vox_eps(m, Z, Y, X, k - 1, j, i - 1) + vox_eps(m, Z, Y, X, k, j, i - 1));
    const float b = 0.5f * (vox_eps(m, Z, Y, X, k - 1, j, i) + vox_eps(m, Z, Y, X, k, j, i));
    return 0.5f * (a + b);
  }
  // Ez: average y, then x; z owned.
  const float a = 0.5f * (vox_eps(m, Z, Y, X, k, j - 1, i - 1) + vox_eps(m, Z, Y, X, k, j, i - 1));
  const float b = 0.5f * (vox_eps(m, Z, Y, X, k, j - 1, i) + vox_eps(m, Z, Y, X, k, j, i));
  return 0.5f * (a + b);
}

// E <- E + (dt/eps0 * 1/eps) * curl for voxel materials (kernels.py:612-623 with
// zero conductivity), or decay * E + source * curl for per-site coefficients.
template <int Mat>
__device__ __forceinline__ float e_update(const Step3D& p, int c, int64_t o, int k, int j, int i, float e,
                                          float curl) {
  if (Mat == FDTD_MATERIAL_VOXEL) {
    const float inv = __frcp_rn(site_eps(p, c, k, j, i));
    return e + (p.dt_over_eps * inv) * curl;
  } else {
    const float dec = p.em.decay[c][p.em.decay_full[c] ? o : 0];
    const float src = p.em.source[c][p.em.source_full[c] ? o : 0];
    return dec * e + src * curl;
  }
}

// PEC: an E component is constrained on a metallic wall normal to either of
// its two transverse axes (beamz/devices/_boundary_compile.py:129-136).
__device__ __forceinline__ bool e_constrained(int metallic, int c, const Dims& d, int k, int j, int i) {
  const int normal = 2 - c;
  const int coord[3] = {k, j, i};
  const int n[3] = {d.z, d.y, d.x};
  for (int a = 0; a < 3; ++a) {
    if (a == normal) continue;
    if ((coord[a] == 0 && wall(metallic, a, false)) || (coord[a] == n[a] - 1 && wall(metallic, a, true)))
      return true;
  }
  return false;
}

// H components are constrained only on walls normal to themselves.
__device__ __forceinline__ bool h_constrained(int metallic, int c, const Dims& d, int k, int j, int i) {
  const int normal = 2 - (c - 3);
  const int coord = normal == 0 ? k : (normal == 1 ? j : i);
  const int n = normal == 0 ? d.z : (normal == 1 ? d.y : d.x);
  return (coord == 0 && wall(metallic, normal, false)) || (coord == n - 1 && wall(metallic, normal, true));
}

// ---- host launchers -------------------------------------------------------
cudaError_t launch_phase(cudaStream_t s, const Step3D& p, int phase, int mat, int active_mask);
cudaError_t launch_fused(cudaStream_t s, const Step3D& p, int mat, int active_mask, int tile_x, int tile_y);
cudaError_t launch_fused_lean(cudaStream_t s, const Step3D& p, int mat, int tile_y);
cudaError_t launch_fused_tma(cudaStream_t s, const Step3D& p, int tile_y);
cudaError_t launch_class_step(cudaStream_t s, const Step3D& p, int tile_y);
// `row`/`plane` are the target's element pitches (dense: dx and dy*dx).
cudaError_t launch_source(cudaStream_t s, const SourceDev& src, float* target, Dims td, int64_t row,
                          int64_t plane, int timing, int metallic, const int* counter, int step_offset);
cudaError_t launch_copy3d(cudaStream_t s, const float* src, int64_t src_row, int64_t src_plane, float* dst,
                          int64_t dst_row, int64_t dst_plane, int64_t nz, int64_t ny, int64_t nx);
struct DftDev;
cudaError_t launch_dft(cudaStream_t s, const DftDev& dft, const int* counter, int step_offset);
cudaError_t launch_counter_advance(cudaStream_t s, int* counter, int nsteps);
cudaError_t launch_dft_sample(cudaStream_t s, const DftDev& dft, float* samples, int slot);
cudaError_t launch_dft_flush(cudaStream_t s, const DftDev& dft, const float* samples, const int* counter, int first,
                             int count);

// Adjoint step buffers (see FdtdAdjointStep in fdtd_b200.h).
struct AdjDev {
  float* lam[6];           // adjoint fields, dense component shapes
  float* scratch_e[6];     // per E term: lam_d at E sites
  float* scratch_h[6];     // per H term: lam_d at H sites
  const float* dft_grad_re;
  const float* dft_grad_im;
  float* curl[3];          // forward curl over the design box
  float* grad[3];          // accumulated dJ/dc over the design box
  int box_lo[3], box_hi[3];
};
cudaError_t launch_adjoint_step(cudaStream_t s, const Step3D& p, const DftDev* dft, const AdjDev& a, int active,
                                int step);
cudaError_t launch_adjoint_curl(cudaStream_t s, const Step3D& p, const AdjDev& a, int active);
int64_t adjoint_noalloc_span(int64_t floats);
cudaError_t launch_adjoint_step_noalloc(cudaStream_t s, const Step3D& p, const DftDev* dft, AdjDev a, int active,
                                        int step, const int64_t e_len[6], const int64_t h_len[6]);

// DFT arena view (see FdtdDft in fdtd_b200.h).
struct DftDev {
  int monitor_count;
  int max_points, neighbors, max_freqs;
  const int* indices;
  const float* weights;
  const float* freqs;
  const float* masks;
  const int* counts;
  const int* codes;
  const float* windows;
  float* re;
  float* im;
  float* weight_sum;
  int64_t arena_len;   // elements of re / im
  int64_t weight_len;  // elements of weight_sum
  const float* fields[6];
  int64_t field_len[6];
  const float* step_time;
  int step_time_len;
  float dt;
  const int* affine;  // [M, 6, 24] affine plans (FdtdDft::affine), or null
};

// Monitor-plane reduction (analysis.cu); see FdtdMonitorReduce.
struct MonitorReduceDev {
  const float* re = nullptr;
  const float* im = nullptr;
  int64_t value_offset = 0, points = 0;
  int freqs = 0, rows = 0;
  int e[2] = {0, 0}, h[2] = {0, 0};
  const double* scale = nullptr;    // [F, 3]
  const double* weights = nullptr;  // [2, P]
  const double* prof_re = nullptr;  // [rows, F, 4, P]
  const double* prof_im = nullptr;
  double* out = nullptr;            // [max(rows, 1), F, 2, 2]
};
cudaError_t launch_monitor_reduce(cudaStream_t s, const MonitorReduceDev& r);

// One field recorder for one step (recorder.cu); see FdtdRecorder.
struct RecorderDev {
  int interval = 1, capacity = 0, ncomp = 0;
  int64_t start[7] = {0, 0, 0, 0, 0, 0, 0};  // prefix sums of the value counts
  float sign[6] = {1, 1, 1, 1, 1, 1};
  int slots[6] = {0, 0, 0, 0, 0, 0};          // gather slots K; 0 = whole component
  const int* idx[6] = {};
  const float* w[6] = {};
  float* values[6] = {};
  const float* field[6] = {};                 // the component in the step's output bank
  int64_t field_len[6] = {};
  int64_t dy[6] = {}, dx[6] = {};             // component extents (whole recorders)
  int64_t row[6] = {}, plane[6] = {};         // device-layout strides
  int* steps = nullptr;
  float* times = nullptr;
  int* count = nullptr;
  const float* step_time = nullptr;
  int step_time_len = 0;
};
cudaError_t launch_record(cudaStream_t s, const RecorderDev& r, const int* counter, int step_offset);

// Gather-plan packing (planner.cu): one (monitor, component) plan.
struct GatherPackDev {
  const int* idx_in = nullptr;    // [points, slots_in]
  const float* w_in = nullptr;
  int* idx_out = nullptr;         // [K, pmax]
  float* w_out = nullptr;
  int points = 0, slots_in = 0, pmax = 0, rows = 0;  // rows: K of the output
  int dz = 0, dy = 0, dx = 0;     // component extents
  int64_t row = 0, plane = 0;     // device layout strides
};

cudaError_t launch_gather_pack(cudaStream_t s, const GatherPackDev& g);
cudaError_t launch_voxel_histogram(cudaStream_t s, const uint8_t* v, int64_t n, int* counts);

// Field diagnostics (diag.cu): one component's view.
struct DiagComp {
  const float* field = nullptr;   // stored array (dense, or pitched rows)
  Dims d{};                       // stored extents (z, y, x)
  int64_t row = 0, plane = 0;     // element strides of the field and of ids
  int edge_z = 0, edge_y = 0, edge_x = 0;  // axis extent n + 1: its end sites weigh 1/2
  int integrate_z = 0;            // 3D: the z axis is integrated
  const uint32_t* ids = nullptr;  // codebook words (pitched); id byte at `shift`
  int shift = 0;
  const float* table = nullptr;   // 256 relative permittivities of the ids
  const float* eps = nullptr;     // per-site relative permittivity, dense over d
};

struct DiagArgs {
  DiagComp comp[6];
  int active = 0;                 // bit c: component c is reduced
  double* partials = nullptr;     // [6][FDTD_DIAG_BLOCKS][3]
};

cudaError_t launch_field_diagnostics(cudaStream_t s, const DiagArgs& a, double* out);
cudaError_t launch_dft_change(cudaStream_t s, const DftDev& d, float* prev_re, float* prev_im, double* out);

}  // namespace fdtd
