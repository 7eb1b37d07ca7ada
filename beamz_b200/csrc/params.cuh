// Kernel parameter blocks built from an FdtdProgram by the host code.
#pragma once

#include "fdtd_common.cuh"

namespace fdtd {

// Electric material for the E update.
struct EMaterial {
  // FDTD_MATERIAL_SITE: per-site (stride 1) or uniform (stride 0) decay/source.
  const float* decay[3];
  const float* source[3];
  int decay_full[3];
  int source_full[3];
  // FDTD_MATERIAL_VOXEL: voxel ids [Z, Y, X] and permittivity table [256].
  const uint8_t* voxels;
  const float* eps_table;
  // FDTD_MATERIAL_CODEBOOK: one word per lattice point (Ex, Ey, Ez ids in
  // bytes 0-2) on the field pitch, and three 256-entry coefficient tables.
  const uint32_t* site_ids;
  const float* site_coef;
};

// Magnetic update coefficients (uniform or per-site).
struct HMaterial {
  const float* decay[3];
  const float* source[3];
  int decay_full[3];
  int source_full[3];
};

// Everything a 3D step/phase kernel reads.
struct Step3D {
  int Z, Y, X;
  const float* ein[3];
  const float* hin[3];
  float* eout[3];
  float* hout[3];
  float res, inv_res;
  float div_bs, div_rs;  // res 2^50 and inv_res 2^-50: div_rn's operands
  float dt_over_eps;
  int metallic;
  int cpml;
  EMaterial em;
  HMaterial hm;
  CpmlTermDev ht[6];
  CpmlTermDev et[6];
  // h-timing sources fused into the step kernel (FDTD_SCHEDULE_FUSED).
  int n_hsrc;
  SourceDev hsrc[kMaxFusedSources];
  int n_esrc;  // pre-E sources applied inside the 2D fused kernel (else 0)
  SourceDev esrc[kMaxFusedSources];
  const int* step_counter;
  int step_offset;
  int z_chunk;
  // Per axis (z, y, x): coordinates [lo, hi) where no CPML term of that axis
  // is active for any component; lets tiles and planes skip slot tests.
  int cpml_inner[3][2];
  // FDTD_LAYOUT_PITCHED: floats per row of every field and site-id array.
  int pitch;
  int* status;  // optional error word for expired bounded waits
  unsigned long long wait_ns;  // bound of every mbarrier wait (device time)
  int test_stall;              // test-only: arm the first bundle's barrier without issuing its copies
  // FDTD_FLAG_FAST pitched step: uint8 material class per lattice point
  // (rows of pitch8 bytes) and the class table (Ex, Ey, Ez coefficients over dx).
  const uint8_t* site_class;
  int pitch8;
  const float4* class_coef;
  int fast_math;  // tolerance arithmetic in the class step (1/dx folded, fused multiply-adds)
  // Class step dispatch order (longest first): tile rows [0, order[0]) and
  // [order[1], rows) and z chunks [0, order[2]) and [order[3], chunks) hold
  // absorber cells; their CTAs are dispatched before the others.
  int order[4];
  int xstage;  // class step: the x-term psi slabs have tensor maps (staged with each plane's bundle)
  // FDTD_FLAG_LOSSY class step: class_coef holds (decay, source) pairs per E
  // class and component ([128][4] float2), h_class / h_class_coef the H ones.
  int lossy;
  const uint8_t* h_class;
  const float2* h_class_coef;
  // Derivative metrics per axis (z, y, x), or null (isotropic: divide by res).
  const float* metric_h[3];  // [n_axis]: forward differences feeding H
  const float* metric_e[3];  // [n_axis + 1]: backward differences feeding E
};

// 2D (canonical xy plane) step/phase parameters; z extent is 1.
struct Step2D {
  int Y, X, pol;
  const float* fin[6];
  float* fout[6];
  float res, inv_res;
  int metallic;
  int cpml;
  EMaterial em;
  HMaterial hm;
  CpmlTermDev ht[2];
  CpmlTermDev et[2];
};

}  // namespace fdtd
