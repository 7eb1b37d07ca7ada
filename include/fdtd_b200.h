/*
 * fdtd_b200.h -- C ABI of the B200 FDTD leapfrog engine (sm_100a).
 *
 * This is the drop-in boundary for beamz's native step path.  beamz's Python
 * runtime hands non-owning device buffers to a native library and receives a
 * CUDA error code back (beamz: cuda/src/launch.h:12-82,
 * beamz/simulation/cuda/runtime.py:80-86, cuda/src/ffi_handler.cc:666-708).
 * Here the same contract is a plain C ABI: every pointer is a device pointer
 * owned by the caller (in practice PyTorch tensors), every call enqueues work
 * on the caller's CUDA stream and returns 0 or a cudaError_t code.  No torch
 * or JAX type appears in any signature.
 *
 * Storage order is (z, y, x), row-major and contiguous, with the complete Yee
 * supports of beamz/lattice.py:32-45 (3D) and 789-813 (2D).  Component slots
 * are always ordered Ex, Ey, Ez, Hx, Hy, Hz.
 */
#ifndef FDTD_B200_H_
#define FDTD_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Bumped whenever a struct below changes layout (beamz: abi_layout.json "abi_version"). */
#define FDTD_ABI_VERSION 13

/* Element types (beamz: cuda/src/launch.h:6-10, plus U8 for voxel ids and F64
 * for reduction results). */
enum {
  FDTD_F32 = 0,
  FDTD_S32 = 1,
  FDTD_BF16 = 2,
  FDTD_U8 = 3,
  FDTD_F64 = 4,
};

/* Flags (beamz: abi_layout.json "flags"; bit 7 keeps its meaning). */
#define FDTD_FLAG_GRAPH_CACHE (1 << 7) /* capture multi-step programs into CUDA graphs */
/* Batched DFT sampling of step n runs on a side stream, beside step n+1 (no
 * counterpart in beamz).  Set it only when no pre-E source cell is gathered by
 * a monitor: a pre-E source writes the bank that the previous step's sample
 * reads.  One host thread per caller stream. */
#define FDTD_FLAG_DFT_OVERLAP (1 << 16)
/* Class step (no counterpart in beamz): the 3D step of a PITCHED program reads
 * its E material as one uint8 class per lattice point (site_class /
 * class_coef below, 1 byte per cell instead of a 4-byte codebook word) and
 * runs 128-wide tiles with four cells per thread.  Its arithmetic is beamz's
 * float32 order, bit for bit, unless FDTD_FLAG_FAST_MATH is set too. */
#define FDTD_FLAG_CLASSES (1 << 17)
/* Tolerance arithmetic in the class step: 1/dx folded into the coefficients
 * (class_coef then holds dt / (eps0 eps dx)), products contracted into fused
 * multiply-adds.  Each step rounds within a few ulp of beamz's float32 path;
 * after long runs whose fields decay (absorbed pulses) the difference grows
 * to the float32 noise floor of the run itself (that of float32 against
 * float64), so parity with the float32 path is a tolerance, not equality. */
#define FDTD_FLAG_FAST_MATH (1 << 19)
/* With FDTD_FLAG_CLASSES: conductive (lossy) material on the class step.
 * class_coef then holds F32 [128, 4, 2] -- per E class and component (Ex, Ey,
 * Ez, unused) the (decay, source) pair of E <- decay E + source curl -- and
 * h_class / h_class_coef give each lattice point an H class (at most 64) with
 * F32 [64, 4, 2] (decay, source) pairs of H <- decay H - source curl
 * (beamz: compile.py:563-640 per-site coefficients).  Exact arithmetic only. */
#define FDTD_FLAG_LOSSY (1 << 20)
/* Test only: the pitched step arms its first copy barrier without issuing the
 * copies, so its bounded wait runs out after wait_limit_ns with nothing in
 * flight, and the kernel returns after setting `status` -- the expiry path,
 * exercised without a fault or a hang. */
#define FDTD_FLAG_TEST_STALL (1 << 18)

/* Step schedules. */
enum {
  FDTD_SCHEDULE_PHASES = 0, /* in place: H kernel, then E kernel (one field bank) */
  FDTD_SCHEDULE_FUSED = 1,  /* one z-marching kernel per step, bank A -> bank B  */
};

/* Field storage layouts.
 * DENSE:   each component is its own contiguous (dz, dy, dx) array -- beamz's
 *          complete Yee supports, exactly as the reference stores them.
 * PITCHED: each component is a (Z+1, Y+1, pitch) float array, pitch a multiple
 *          of 4 and >= X+1, holding the component in its (dz, dy, dx) corner.
 *          All rows are 16-byte aligned, which lets the fused 3D step stage
 *          planes with TMA.  3D, FDTD_MATERIAL_CODEBOOK and uniform H
 *          coefficients only; fdtd_copy_component converts between layouts. */
enum {
  FDTD_LAYOUT_DENSE = 0,
  FDTD_LAYOUT_PITCHED = 1,
};

/* Material encodings for the electric update. */
enum {
  FDTD_MATERIAL_SITE = 0,  /* per-site (or scalar) decay/source arrays, E = d*E + s*curl      */
  FDTD_MATERIAL_VOXEL = 1, /* uint8 voxel ids + eps table; E-site eps averaged on the fly     */
  FDTD_MATERIAL_CODEBOOK = 2, /* per-site uint8 ids of E coefficients (pitched layout)        */
};

/* Source timings (beamz/simulation/execute.py:48-52). */
enum {
  FDTD_TIMING_PRE_E = 0, /* added to E before the H update               */
  FDTD_TIMING_H = 1,     /* added to H after the H update, before PEC     */
  FDTD_TIMING_E = 2,     /* added to E after the E update, before PEC     */
};

/* Metallic (PEC) walls bitmask, order (front, back, bottom, top, left, right)
 * = (z low, z high, y low, y high, x low, x high)
 * (beamz/simulation/cuda/runtime.py:38-40). */
#define FDTD_EDGE_FRONT (1 << 0)
#define FDTD_EDGE_BACK (1 << 1)
#define FDTD_EDGE_BOTTOM (1 << 2)
#define FDTD_EDGE_TOP (1 << 3)
#define FDTD_EDGE_LEFT (1 << 4)
#define FDTD_EDGE_RIGHT (1 << 5)

#define FDTD_MAX_SOURCES 16
#define FDTD_MAX_MONITORS 16

/* Non-owning buffer (replaces BeamzBuffer, beamz: cuda/src/launch.h:12-17).
 * rank 0 = scalar; dims beyond rank are ignored. */
typedef struct FdtdBuffer {
  void* data;
  int32_t rank;
  int32_t element_type;
  int64_t dims[4];
} FdtdBuffer;

/* One packed CPML recurrence (beamz/simulation/model.py:306-324,
 * beamz/simulation/kernels.py:238-264).  a/b/inv_kappa are 1-D of length
 * low + high along `axis` (0 = z, 1 = y, 2 = x of the target component);
 * psi has the target component's shape with that axis replaced by low + high.
 * psi_alt is the second psi bank used by FDTD_SCHEDULE_FUSED for H terms. */
typedef struct FdtdCpmlTerm {
  int32_t axis;
  int32_t low;
  int32_t high;
  int32_t reserved;
  FdtdBuffer a;
  FdtdBuffer b;
  FdtdBuffer inv_kappa;
  FdtdBuffer psi;
  FdtdBuffer psi_alt;
} FdtdCpmlTerm;

/* One slab injection field[start + idx] += coeff[idx] * waveform[clamp(step)]
 * (beamz/devices/sources/compiler.py:116-129, beamz/simulation/execute.py:374-433,
 * cuda/src/io.cu:122-168).  coeff has rank 3 (extent z, y, x); waveform rank 1. */
typedef struct FdtdSource {
  int32_t component; /* 0..5 = Ex..Hz */
  int32_t timing;    /* FDTD_TIMING_* */
  int32_t start[3];  /* z, y, x (2D: z = 0) */
  int32_t reserved;
  FdtdBuffer coeff;
  FdtdBuffer waveform;
} FdtdSource;

/* Vector-DFT monitor arena (beamz: cuda/src/launch.h:47-61, observe.py:529-585).
 *  indices  S32 [M, 6, K, P]  flat offsets into each component, neighbour-major
 *  weights  F32 [M, 6, K, P]  (per point, the nonzero weights come first: a
 *                             zero weight ends that point's gather)
 *  freqs    F32 [M, F]
 *  masks    F32 [M, 6]
 *  counts   S32 [M, 5]: freq_count, point_count, interval, value_offset, weight_offset
 *  codes    S32 [M, 2]: window code (1 = Hann), normalization code (1 = physical)
 *  windows  F32 [M, 3]: t_start, t_end, length_unit
 *  re, im   F32 arena, accumulated at value_offset + (c * F + f) * P + p
 *  weight_sum F32 arena, accumulated at weight_offset + f
 *  samples  F32 [batch, M, 6, P] (optional step batching)                      */
typedef struct FdtdDft {
  int32_t monitor_count;
  int32_t batch;           /* > 1 with `samples`: accumulate every `batch` steps (below) */
  FdtdBuffer indices;
  FdtdBuffer weights;
  FdtdBuffer freqs;
  FdtdBuffer masks;
  FdtdBuffer counts;
  FdtdBuffer codes;
  FdtdBuffer windows;
  FdtdBuffer re;
  FdtdBuffer im;
  FdtdBuffer weight_sum;
  /* F32 [batch, M, 6, P], optional.  With it, fdtd_launch_program stores each
   * step's gathered samples and adds a batch of them to re/im/weight_sum in
   * one pass every `batch` steps and at the end of the call -- in step order,
   * so the arena is bit-identical to per-step accumulation, with the arena
   * read and written once per batch instead of once per step. */
  FdtdBuffer samples;
  /* S32 [M, 6, 24], optional: per (monitor, component) the affine form of its
   * gather plan, which the batched sampling then uses instead of indices /
   * weights (no plan read per point).  Word 0 = 1 marks it: every point
   * p = a * nb + b (a < na, b < nb) sums slot s < k at index
   * base + a * sa + b * sb + delta[s] with weight w[s], in slot order, as the
   * packed plan does (k <= 4).  Words: 0 flag, 1 na, 2 nb, 3 base, 4 sa, 5 sb, 6 k,
   * 8..15 delta[8], 16..23 w[8] (float bits).  The runtime derives it from the
   * packed plan only where the plan has exactly that form (plane monitors on
   * uniform coordinates do). */
  FdtdBuffer affine;
} FdtdDft;

/* A time-domain field recorder (beamz: FieldRecorder, compiled by
 * devices/monitors/compiler.py:286-412 and updated each step by
 * simulation/observe.py:588-646 _record_fields).  After every step s with
 * (s + 1) % interval == 0, while fewer than `capacity` records exist, record
 * n = count writes, for each recorded component q:
 *   values[q][n, v] = sign[q] * field value v,
 * where field value v is, with indices/weights null, element v of the
 * component in its own (z, y, x) order (a "domain" recorder), else the sum
 * over slots k of field[indices[k, v]] * weights[k, v] in slot order, up to
 * the first zero weight (plans packed by fdtd_pack_gather); steps[n] = s + 1
 * and times[n] = step_time[s].  `count` holds the number of records twice,
 * double-buffered by step parity (read count[s & 1], write count[(s+1) & 1]),
 * and starts as {0, 0}. */
#define FDTD_MAX_RECORDERS 4
typedef struct FdtdRecorder {
  int32_t interval;
  int32_t capacity;
  int32_t component_count;  /* 1..6 */
  int32_t components[6];    /* component index of each value set */
  float signs[6];
  FdtdBuffer indices[6];    /* S32 [K, V] device-layout offsets, or null */
  FdtdBuffer weights[6];    /* F32 [K, V], or null */
  FdtdBuffer values[6];     /* F32 [capacity, V] */
  FdtdBuffer steps;         /* S32 [capacity] */
  FdtdBuffer times;         /* F32 [capacity] */
  FdtdBuffer count;         /* S32 [2] */
} FdtdRecorder;

/* A complete step program (replaces BeamzLaunch + BeamzProgramLaunch,
 * beamz: cuda/src/launch.h:19-77). */
typedef struct FdtdProgram {
  int32_t abi_version;    /* FDTD_ABI_VERSION */
  int32_t flags;          /* FDTD_FLAG_* */
  int32_t ndim;           /* 2 or 3 */
  int32_t polarization;   /* 2D: 0 = TM (Ez, Hx, Hy), 1 = TE (Ex, Ey, Hz) */
  int32_t schedule;       /* FDTD_SCHEDULE_* */
  int32_t material_kind;  /* FDTD_MATERIAL_* */
  int32_t metallic_edges; /* FDTD_EDGE_* bitmask */
  int32_t cpml;           /* 0, or 1 when h_terms/e_terms are populated */
  int32_t nsteps;         /* steps enqueued by fdtd_launch_program */
  int32_t source_count;
  int64_t cells[3];       /* nz, ny, nx material cells (2D: 1, ny, nx) */
  float dt;
  float resolution;
  float inv_resolution;
  float dt_over_eps;      /* fl32(dt) / fl32(EPS_0) */
  float dt_over_mu;       /* fl32(dt) / fl32(MU_0) */
  float h_source;         /* 2D and scalar-H: fl32(dt / MU_0) */
  int32_t tile_x;         /* fused-kernel tile (0 = default) */
  int32_t tile_y;
  int32_t z_chunk;        /* fused-kernel z planes per CTA (0 = whole axis) */
  int32_t layout;         /* FDTD_LAYOUT_* */
  int64_t pitch;          /* PITCHED: floats per row of every field array */
  int64_t wait_limit_ns;  /* bound of every device-side wait of the pitched step (0 = 200 ms) */
  FdtdBuffer fields[6];     /* bank A (in/out) */
  FdtdBuffer fields_alt[6]; /* bank B (FDTD_SCHEDULE_FUSED only) */
  /* FDTD_MATERIAL_SITE: e_decay[c], e_source[c] are rank-0 or full E-component
   * arrays; h_decay/h_source likewise for H (rank 0 = uniform). */
  FdtdBuffer e_decay[3];
  FdtdBuffer e_source[3];
  FdtdBuffer h_decay[3];
  FdtdBuffer h_source_site[3];
  /* FDTD_MATERIAL_VOXEL: U8 [nz, ny, nx] ids and F32 [256] permittivity table. */
  FdtdBuffer voxels;
  FdtdBuffer eps_table;
  /* FDTD_MATERIAL_CODEBOOK: S32 [Z+1, Y+1, pitch] words whose bytes 0, 1, 2 are
   * the ids of the Ex, Ey, Ez coefficient fl(fl(dt)/fl(eps0) * fl(1/eps_site))
   * at that lattice point (beamz: compile.py:146-187 packs its lossless E
   * material the same way), and the F32 [3, 256] coefficient tables. */
  FdtdBuffer site_ids;
  FdtdBuffer site_coef;
  FdtdCpmlTerm h_terms[6]; /* 3D: Hxy Hxz Hyz Hyx Hzx Hzy; 2D: first 2 */
  FdtdCpmlTerm e_terms[6]; /* 3D: Exy Exz Eyz Eyx Ezx Ezy; 2D: first 2 */
  FdtdSource sources[FDTD_MAX_SOURCES];
  FdtdDft dft;
  FdtdBuffer step_counter; /* S32 [1]: absolute step of the next step, advanced on device */
  FdtdBuffer step_time;    /* F32 [T]: t + dt after absolute step s (FP32-accumulated clock) */
  FdtdBuffer status;       /* S32 [1], optional: set nonzero when a bounded device wait expired */
  /* Derivative metrics of an axis-uniform or rectilinear grid (beamz:
   * DerivativeMetricPlan, model.py:290-303; BeamzLaunch metric_kind/metrics,
   * cuda/src/launch.h:24-33).  All null: the isotropic grid, each difference
   * divided by `resolution`.  Otherwise, for every axis a of the grid (z, y, x;
   * 2D: y, x, with z null), metric_h[a] is F32 [n_a] (n_a = cells along a):
   * the inverse distances that multiply the forward differences of the H
   * update at each H coordinate; metric_e[a] is F32 [n_a + 1], those of the
   * backward differences of the E update at each E coordinate (an axis-uniform
   * grid repeats one value).  FDTD_LAYOUT_DENSE, or FDTD_LAYOUT_PITCHED with
   * FDTD_FLAG_CLASSES and neither FDTD_FLAG_FAST_MATH nor FDTD_FLAG_LOSSY (the
   * class step, 128 x 8 tiles whatever tile_y asks).  The adjoint entry points
   * take them on FDTD_LAYOUT_DENSE. */
  FdtdBuffer metric_h[3];
  FdtdBuffer metric_e[3];
  /* Field recorders, run after each step's DFT sample (see FdtdRecorder). */
  int32_t recorder_count;
  int32_t reserved_recorders;
  FdtdRecorder recorders[FDTD_MAX_RECORDERS];
  /* FDTD_FLAG_CLASSES with FDTD_MATERIAL_CODEBOOK: U8 [Z+1, Y+1, pitch8]
   * material class of every lattice point (pitch8 = dims[2], a multiple of 16
   * >= X+1) and F32 [256, 4] per class the Ex, Ey, Ez update coefficients
   * fl(fl(dt)/fl(eps0) * fl(1/eps_site)) -- over dx with FDTD_FLAG_FAST_MATH
   * -- (the fourth column unused).  A class is one distinct (Ex, Ey, Ez)
   * coefficient triple of the codebook. */
  FdtdBuffer site_class;
  FdtdBuffer class_coef;
  /* FDTD_FLAG_LOSSY: U8 [Z+1, Y+1, pitch8] H class of every lattice point and
   * its F32 [64, 4, 2] (decay, source) table (see FDTD_FLAG_LOSSY). */
  FdtdBuffer h_class;
  FdtdBuffer h_class_coef;
} FdtdProgram;

/* ABI version of the loaded library (beamz: cuda/src/extension.cc __abi_version__). */
int fdtd_abi_version(void);

/* sizeof(FdtdProgram) as compiled into the library, so a binding can check its
 * struct mirror before the first call (beamz: backend.py:139-157 validates the
 * extension manifest the same way). */
int64_t fdtd_program_size(void);

/* Validate a program without enqueueing work; 0 or cudaErrorInvalidValue (1).
 * (beamz: cuda/src/program.cu:110-170, update.cu:66-146) */
int fdtd_validate(const FdtdProgram* program);

/* One in-place half step: phase 0 = H from E, phase 1 = E from H, including
 * CPML psi and PEC zeroing of constrained cells (beamz: BeamzLaunchStreamed,
 * cuda/src/update.cu:919-971; beamz/simulation/cuda/runtime.py:184/234). */
int fdtd_launch_phase(void* stream, const FdtdProgram* program, int32_t phase);

/* Enqueue program->nsteps complete leapfrog steps -- sources at their three
 * timings, H, E, PEC, DFT monitors, step counter -- on `stream`
 * (beamz: BeamzLaunchProgram, cuda/src/program.cu:339-354;
 * beamz/simulation/cuda/runtime.py:496/621/685).  With FDTD_SCHEDULE_FUSED
 * an odd step count leaves the result in fields_alt / psi_alt (the caller
 * swaps its handles); an even count leaves it in fields / psi. */
int fdtd_launch_program(void* stream, const FdtdProgram* program);

/* Add every source of `timing` for absolute step counter[0] + step_offset to
 * its target field in `program->fields` (beamz: cuda/src/io.cu:250-286). */
int fdtd_apply_sources(void* stream, const FdtdProgram* program, int32_t timing, int32_t step_offset);

/* Accumulate the DFT monitors once from `program->fields` for absolute step
 * counter[0] + step_offset (beamz: cuda/src/io.cu:381-401). */
int fdtd_accumulate_dft(void* stream, const FdtdProgram* program, int32_t step_offset);

/* Record every field recorder once from `program->fields` for absolute step
 * counter[0] + step_offset (as fdtd_launch_program does after each step;
 * beamz: observe.py:588-646). */
int fdtd_record_fields(void* stream, const FdtdProgram* program, int32_t step_offset);

/* Copy the (extent[0], extent[1], extent[2]) corner block between two rank-3
 * F32 buffers whose own dims give their row and plane pitches (dense <->
 * pitched field layouts).  No beamz counterpart: beamz keeps one layout. */
int fdtd_copy_component(void* stream, const FdtdBuffer* src, const FdtdBuffer* dst, const int64_t* extent);

/* Capture program->nsteps complete steps, exactly as fdtd_launch_program
 * enqueues them, into a CUDA graph owned by the caller; *graph receives the
 * executable graph.  The graph holds every pointer of `program`: each replay
 * advances that same state by nsteps steps (the step counter and clock live on
 * the device).  `stream` must be a created stream (capture source).
 * No beamz counterpart: beamz keeps graphs only in its process-global cache
 * (cuda/src/graph.cu:84-154); a serving loop that keeps many simulations
 * resident owns one graph per simulation instead. */
int fdtd_graph_create(void* stream, const FdtdProgram* program, void** graph);

/* Replay a graph from fdtd_graph_create on `stream`. */
int fdtd_graph_launch(void* stream, void* graph);

/* Release a graph from fdtd_graph_create (null is a no-op). */
int fdtd_graph_destroy(void* graph);

/* One adjoint (time-reversed, transposed) step.  No beamz counterpart: beamz
 * differentiates its JAX path with JAX; this is the hand-written discrete
 * adjoint of the step fdtd_launch_program runs (dense layout, per-site E
 * material, phase schedule).  The FdtdProgram passed with it is the ADJOINT
 * program: the forward program's coefficients, CPML terms, walls and
 * monitors, with `fields` holding the adjoint fields and each term's `psi`
 * the adjoint memory. */
typedef struct FdtdAdjointStep {
  int32_t abi_version;
  int32_t step;              /* absolute step n whose transpose is applied */
  FdtdBuffer scratch_e[6];   /* F32, per E term: that E component's shape */
  FdtdBuffer scratch_h[6];   /* F32, per H term: that H component's shape */
  FdtdBuffer dft_grad_re;    /* F32 [arena], optional: dJ/d(dft re) */
  FdtdBuffer dft_grad_im;    /* F32 [arena], optional: dJ/d(dft im) */
  FdtdBuffer curl[3];        /* F32 [box], optional: forward curl of Ex/Ey/Ez over the box */
  FdtdBuffer grad[3];        /* F32 [box], optional: accumulated dJ/dc of Ex/Ey/Ez */
  int32_t box_lo[3];         /* design box of E sites (z, y, x), interior and */
  int32_t box_hi[3];         /* clear of every absorber slab */
} FdtdAdjointStep;

/* Apply the transpose of step `a->step` to the adjoint state in `adjoint`:
 * the DFT adjoint source of that step's sample (when dft_grad_* are given),
 * the E update's transpose with gradient accumulation grad += mu * curl over
 * the box (when grad/curl are given), then the H update's transpose. */
int fdtd_adjoint_step(void* stream, const FdtdProgram* adjoint, const FdtdAdjointStep* a);

/* Floats in the device scratch array of fdtd_adjoint_step_noalloc (16 MiB). */
#define FDTD_ADJOINT_NOALLOC_MAX_FLOATS (4 * 1024 * 1024)

/* fdtd_adjoint_step without caller scratch: the per-term scratch arrays are
 * carved from one device array of FDTD_ADJOINT_NOALLOC_MAX_FLOATS floats
 * inside this library, so the call allocates no device memory.  It is for
 * callers that cannot allocate device memory where they step the adjoint: a
 * host program that links only this C library and owns no device allocator
 * for temporaries, or one held to a fixed device-memory budget.
 * No counterpart in the reference (beamz differentiates through JAX).
 * a->scratch_e and a->scratch_h must be empty.  A program whose live
 * derivative terms need more scratch than the maximum (each term's array
 * rounded up to 64 floats; 2D TM up to about 1000 x 1000, 3D up to about
 * 330 000 lattice points) is rejected with cudaErrorInvalidValue (1) before
 * any work is enqueued.  Every call shares the one array: calls that overlap
 * on the GPU (two streams, or two host threads) race and corrupt each
 * other's results, so serialize them.  Nothing in it needs to start at
 * zero: each call writes every scratch element it reads first. */
int fdtd_adjoint_step_noalloc(void* stream, const FdtdProgram* adjoint, const FdtdAdjointStep* a);

/* Write the forward curl of each active E component over `a`'s box into
 * a->curl from `forward`'s current H fields (call after a forward step). */
int fdtd_adjoint_curl(void* stream, const FdtdProgram* forward, const FdtdAdjointStep* a);

/* ---- Field diagnostics and monitor change (automatic termination) ---------
 * beamz checks a chunked run for convergence, divergence and non-finite
 * fields between chunks (beamz/simulation/execute.py:1312-1484): integrated
 * electromagnetic energy, the largest |field| and finiteness of every active
 * component (_field_diagnostics, execute.py:184-222) and the relative change
 * of each monitor's DFT vectors (_relative_monitor_change, 294-316).  beamz
 * reduces with jnp; these two entry points are the device reductions, each
 * deterministic (fixed block partition, fixed summation order). */

/* Reduction blocks per component of fdtd_field_diagnostics. */
#define FDTD_DIAG_BLOCKS 592

typedef struct FdtdDiagnostics {
  FdtdBuffer site_eps_table; /* F32 [3, 256]: relative permittivity per codebook id (codebook programs) */
  FdtdBuffer site_eps[3];    /* F32 per E component over its stored shape (other programs); empty = 1 */
  FdtdBuffer partials;       /* F64 scratch of >= 6 * FDTD_DIAG_BLOCKS * 3 elements */
  FdtdBuffer out;            /* F64 [6, 3]: per component sum(eps * v^2 * h), max |v|, non-finite count */
} FdtdDiagnostics;

/* Reduce the program's current fields (`fields`).  For every active component
 * c: S_c = sum over its stored sites of eps_r * v^2 * h, where h is the
 * product over the integrated axes (x, y and, in 3D, z) of 1/2 at the two ends
 * of an edge-aligned axis (extent n + 1) and 1 elsewhere: beamz's control
 * volumes (_axis_integration_weights, execute.py:75-92) divided by the cell
 * size.  eps_r is 1 for H components.  Non-finite values are counted and left
 * out of the sum and the maximum.  The caller forms the energy
 * sum_c 0.5 * const_c * S_c * res^ndim (const = eps0 for E, mu0 for H). */
int fdtd_field_diagnostics(void* stream, const FdtdProgram* program, const FdtdDiagnostics* d);

typedef struct FdtdDftChange {
  FdtdBuffer prev_re;  /* F32 [arena]: the arena at the previous check (updated to the current one) */
  FdtdBuffer prev_im;
  FdtdBuffer out;      /* F64 [M, 6, F, 3]: |cur - prev|^2, |cur|^2, |prev|^2 per (monitor, component, frequency) */
} FdtdDftChange;

/* Squared norms of each (monitor, component, frequency) DFT vector's change
 * since the previous check, of the vector and of its previous value; then
 * copies the arena into prev_re / prev_im.  Masked-off components and
 * frequencies beyond a monitor's count report zeros. */
int fdtd_dft_change(void* stream, const FdtdProgram* program, const FdtdDftChange* c);

/* ---- On-device planning -------------------------------------------------
 * beamz packs monitor gather plans and compacts voxel materials on the host
 * (beamz/simulation/cuda/runtime.py:530-618, compile.py:146-187); these move
 * the per-element part of that work to the device. */

/* One (monitor, component) gather plan and where its packed form goes. */
typedef struct FdtdGatherPack {
  FdtdBuffer indices_in;   /* S32 [P, Kc]: dense flat offsets into the component */
  FdtdBuffer weights_in;   /* F32 [P, Kc] */
  FdtdBuffer indices_out;  /* S32 [K, Pmax] (P <= Pmax): the program's [M, 6, K, Pmax] slice */
  FdtdBuffer weights_out;  /* F32 [K, Pmax] */
  int32_t dims[3];         /* the component's stored extents (z, y, x) */
  int64_t row, plane;      /* element strides of the device layout (dense: x, y*x; pitched: P, (Y+1)*P) */
} FdtdGatherPack;

/* Per point p < P: the slots with a nonzero weight first, then the others,
 * each group in slot order, into rows 0..min(Kc, K)-1 of column p (a K below
 * Kc drops trailing slots, so it must cover every point's nonzero count; the
 * runtime sizes K that way); each offset
 * (k, j, i) = unravel(flat, dims) becomes k*plane + j*row + i, an offset
 * outside the component becomes -1 (never gathered).  Rows Kc..K-1 and
 * columns P..Pmax-1 are left as they are (zero in a fresh plan).  No beamz
 * counterpart (its runtime packs on the host). */
int fdtd_pack_gather(void* stream, const FdtdGatherPack* g);

/* counts[v] = number of voxels with id v (U8 voxels, S32 [256] counts, set
 * to zero first): the materials a program uses, for the codebook's compact
 * material indices (beamz compacts on the host, compile.py:146-187). */
int fdtd_voxel_histogram(void* stream, const FdtdBuffer* voxels, const FdtdBuffer* counts);

/* ---- Monitor-plane reductions --------------------------------------------
 * The sums behind beamz's DFT flux through a monitor (observe.py:166-234
 * monitor_dft_component, _flux_component, monitor_dft_flux) and its modal
 * overlaps with mode profiles (devices/modes/fields.py:76-129 _modal_overlap),
 * evaluated on the device arena instead of a host copy of it. */
typedef struct FdtdMonitorReduce {
  int32_t abi_version;     /* FDTD_ABI_VERSION */
  int32_t freq_count;      /* F of the monitor */
  int64_t value_offset;    /* the monitor's first element in program->dft.re/im */
  int64_t point_count;     /* P of the monitor */
  int32_t e[2];            /* E component (0..2) of each (E, H) pair */
  int32_t h[2];            /* H component (3..5) of each pair */
  int32_t rows;            /* mode profile rows; 0 = field products (flux) */
  int32_t reserved;
  FdtdBuffer scale;        /* F64 [F, 3]: alpha_f, phase_f (re, im) */
  FdtdBuffer weights;      /* F64 [2, P]: point weights of pair 0 and pair 1 */
  FdtdBuffer profile_re;   /* F64 [rows, F, 4, P]: each row's e0, e1, h0, h1 (rows > 0) */
  FdtdBuffer profile_im;
  FdtdBuffer out;          /* F64 [max(rows, 1), F, 2, 2]: per pair q the complex sum */
} FdtdMonitorReduce;

/* With E_q = alpha_f v(e[q]) and H_q = (alpha_f v(h[q])) phase_f, v(c) the
 * arena value re + i im of component c at value_offset + (c F + f) P + p:
 *   rows == 0:  out[0, f, q] = sum_p weights[q, p] E_q conj(H_q)
 *   rows > 0:   out[r, f, q] = sum_p weights[q, p] (E_q conj(G_{2+q}) + conj(G_q) H_q)
 * where G_k = profile_re + i profile_im [r, f, k, p].  Each term is formed in
 * double with numpy's complex operand order; the sums run in a fixed order.
 * No beamz counterpart (beamz copies the arena to the host and sums there). */
int fdtd_monitor_reduce(void* stream, const FdtdProgram* program, const FdtdMonitorReduce* r);

/* Drop every cached CUDA graph (beamz: cuda/src/graph.cu cache reset). */
void fdtd_clear_graph_cache(void);

/* Human-readable name of a returned error code. */
const char* fdtd_error_string(int code);

/* One launch entry point by target name. */
typedef struct FdtdRegistration {
  const char* name;
  void* fn;
} FdtdRegistration;

/* The launch entry points keyed by target name, as beamz's extension module
 * lists its FFI targets (beamz: cuda/src/extension.cc:13-21 registrations()):
 * "fdtd_phase" -> fdtd_launch_phase, "fdtd_program" -> fdtd_launch_program.
 * Writes the entry count to *count (when non-null); the table is static. */
const FdtdRegistration* fdtd_registrations(int32_t* count);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_B200_H_ */
