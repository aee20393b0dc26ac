/*
 * psr_b200 — C ABI of the B200-native screened-Poisson reconstruction library.
 *
 * Every entry point returns an int status (PSR_OK = 0).  Pointers named "device" are CUDA
 * device pointers (torch tensors, Warp arrays or anything exposing
 * __cuda_array_interface__); sizes are element counts; `stream` is a cudaStream_t (NULL =
 * legacy default stream).  Work is stream-ordered; the only host synchronisations are the
 * element-count reads that size data-dependent buffers, as in the reference.  A result is
 * thread-compatible, not thread-safe.  psr_last_error() returns the calling thread's last
 * message.
 *
 * Interfaces replaced (warp-psr, file:line):
 *   psr_reconstruct       <- warp_psr.reconstruct            src/warp_psr/reconstruction.py:137-349
 *   psr_result_info       <- Reconstruction.iso_value/.metadata reconstruction.py:119-134,303-344
 *   psr_result_arrays     <- LevelField keys/coefficients/cumulative  src/warp_psr/field.py:122-148
 *   psr_evaluate          <- Reconstruction.evaluate / LevelField.evaluate  field.py:150-184,395-421
 *   psr_device_field      <- Reconstruction.device_field / _device_field  device_field.py:19-28,115-142
 *   psr_free              <- (Python garbage collection of the Reconstruction)
 *   psr_relax_sliced      <- relaxation.relax_sliced         src/warp_psr/relaxation.py:189-210
 *   psr_isovalue          <- reconstruction._compute_isovalue src/warp_psr/reconstruction.py:101-116
 *   psr_backward          <- reconstruct_differentiable backward  src/warp_psr/reconstruction_adjoint.py:99-172
 *   psr_evaluate_backward <- DifferentiableField.evaluate VJP  field_adjoint.py:34-45,246-288; field.py:214-284
 *   psr_mc_*, psr_mesh_*  <- extract_isosurface (sparse/dense) meshing.py:150-281, Warp's marching cubes
 *   psr_extract_mesh      <- extract_mesh                     meshing.py:284-346
 */
#ifndef PSR_B200_H
#define PSR_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PSR_OK = 0,
  PSR_EINVAL = 1,      /* invalid argument (raised before any allocation, like the reference's ValueError) */
  PSR_ECUDA = 2,       /* CUDA runtime error */
  PSR_EDATA = 3,       /* degenerate input: nonfinite positions, zero extent, no accepted samples */
  PSR_ETIMEOUT = 4,    /* a bounded device-side wait gave up (dependency scheduler) */
  PSR_ENOMEM = 5
};

enum { PSR_FLOAT32 = 0, PSR_FLOAT64 = 1 };

/* Solve precision.  PSR_PRECISION_INPUT follows the input dtype exactly like the reference
 * (float32 in, float32 solve; float64 in, float64 solve).  PSR_PRECISION_MIXED keeps
 * float32 operator storage and runs the vector arithmetic of the ordered relaxation in
 * float64: coefficients are float64, the relaxation reads half the operator bytes. */
enum { PSR_PRECISION_INPUT = 0, PSR_PRECISION_MIXED = 1 };

/* reconstruct() keyword arguments (reconstruction.py:137-153); all fields required. */
typedef struct psr_params {
  int32_t depth, full_depth, base_depth, solve_depth, kernel_depth;
  double samples_per_node, scale, point_weight, cg_accuracy;
  int32_t exact_interpolation, iters, base_v_cycles;
  int32_t precision;
  int32_t keep_stages; /* nonzero: keep intermediate stage arrays for psr_result_stage (tests) */
  int32_t differentiable; /* nonzero: keep the reverse-pass tape for psr_backward */
} psr_params;

typedef struct psr_result psr_result;

/* Summary of one reconstruction. */
typedef struct psr_info {
  int32_t dtype;            /* PSR_FLOAT32 / PSR_FLOAT64 of coefficients and queries */
  int32_t depth;
  int64_t total;            /* coefficients over all levels */
  int64_t groups;           /* accepted leaf sample groups */
  int64_t basis_counts[16]; /* active basis functions per depth (0 beyond depth) */
  int64_t support_counts[16];
  double iso_value;
  double cube_to_model[16]; /* row-major 4x4 (transforms.py:55-79, first matrix) */
  double model_to_cube[16]; /* row-major 4x4 (second matrix) */
  double stage_ms[8];       /* samples, density, normal_field, tree, assembly_and_solve, field, isovalue, total */
  double relax_ms;          /* device time of the ordered sliced relaxation kernels (CUDA events) */
  int64_t relax_row_visits; /* rows x sweeps relaxed by those kernels */
  int64_t relax_launches;
  double relax_finest_ms;            /* the finest level's launch alone (the dominant one) */
  int64_t relax_finest_row_visits;
  double normalization[5];  /* sample transform [1/width, t0, t1, t2, normal scale] (samples.py:54-88) */
  double backward_ms[8];    /* last psr_backward, device ms: field, mirrored operators, reverse sweeps, operator
                               adjoints, base multigrid, point constraints, normal loads, splats+density+samples */
} psr_info;

/* Device arrays owned by the result (valid until psr_free). */
typedef struct psr_arrays {
  const int64_t* keys;          /* d<<48 | x<<32 | y<<16 | z, sorted, all levels */
  const void* coefficients;     /* per-level corrections, dtype */
  const void* cumulative;       /* cumulative coefficients (field.py:187-210), dtype */
  const int64_t* level_offsets; /* host array, depth+2 entries */
  const int64_t* support_keys[16]; /* signed tree keys of each depth's non-ghost support (device) */
} psr_arrays;

/* Zero-copy handle mirroring warp-psr's DeviceField struct (device_field.py:19-28), passed
 * by value to CUDA kernels that evaluate the field with psr_evaluate_field (psr_field.cuh). */
typedef struct psr_field_handle {
  const int64_t* keys;      /* sorted basis keys of all levels (device) */
  const void* coefficients; /* per-level corrections, dtype (device) */
  const void* cumulative;   /* cumulative coefficients, dtype (device); NULL = direct evaluation */
  int64_t count;            /* keys */
  double linear[9];         /* model -> unit cube, row-major */
  double translation[3];
  int32_t depth;
  int32_t dtype;
  double iso_value;
  const void* hash_slots;   /* open-addressing table of {int64 key, int64 index} slots, key -1 = empty
                               (device); NULL = binary search of keys */
  uint64_t hash_mask;       /* slots - 1 (a power of two minus one) */
} psr_field_handle;

int psr_reconstruct(const void* positions, const void* normals, int64_t n, int32_t dtype, const psr_params* params,
                    void* stream, psr_result** out);
int psr_result_info(const psr_result* result, psr_info* info);
int psr_result_arrays(const psr_result* result, psr_arrays* arrays);
int psr_evaluate(const psr_result* result, const void* queries, int64_t nq, void* values, void* gradients,
                 int32_t* valid, void* stream);
int psr_device_field(const psr_result* result, psr_field_handle* handle);
int psr_free(psr_result* result);
int psr_last_error(char* buffer, size_t length);

/* Number of this library's own kernel launches since it was loaded (library sorts and
 * scans from CUB are not counted). */
int psr_kernel_launches(int64_t* count);

/* Device time of the library's main kernels for a per-kernel roofline (a diagnostic, no
 * counterpart in the reference).  Launches issued while the environment variable
 * PSR_KERNEL_CLOCKS=1 is set are bracketed by CUDA events; this call waits for them and
 * reports, per kernel, the launches, summed device ms, summed algorithmic bytes (what the
 * launch must read and write once) and summed units (rows, row visits, points), then clears
 * the totals.  Up to `capacity` entries are written; *count receives how many kernels have
 * totals.  While nobody reads them, at most 4096 launches' events are held: beyond that the
 * older half is folded into the totals (waiting for those launches). */
typedef struct psr_kernel_clock {
  const char* kernel;
  const char* unit;
  int64_t launches;
  double ms;
  double bytes;
  double units;
} psr_kernel_clock;
int psr_kernel_clocks(psr_kernel_clock* out, int32_t capacity, int32_t* count);

/* Ordered sliced Gauss-Seidel of one level on a caller-supplied CSR operator (device
 * pointers; rows = basis keys of `depth`).  Result bitwise identical to the reference's
 * sequential slice/colour order. */
int psr_relax_sliced(int32_t dtype, const int64_t* keys, int64_t n, int32_t depth, const int32_t* offsets,
                     const int32_t* columns, const void* values, const void* b, void* x, int32_t iters, void* stream);

/* Device pointer, element count and element size of an intermediate array kept when
 * params.keep_stages was set (names: group_keys, group_sums, group_normal_sums,
 * group_weights, group_first, transform, depths_and_weights, normal_keys, normal_values,
 * normal_average, normal_load_<d>, rhs_<d>, centroid_values).  *count = -1 if absent. */
int psr_result_stage(const psr_result* result, const char* name, const void** data, int64_t* count, int32_t* elem);

/* Weighted mean sum(v*w)/sum(w) with float64 accumulation, written to out[0] (dtype). */
int psr_isovalue(int32_t dtype, const void* values, const void* weights, int64_t n, void* out, void* stream);

/* psr_isovalue without any device allocation: no counterpart in the reference.  For callers
 * that cannot allocate device memory while they run (code embedded in a framework whose own
 * pool already holds the device memory, real-time loops that must not allocate).  Its
 * scratch is a fixed 64 KiB array in the library's device image, held by every GPU that
 * loads the library until the process exits; n is limited to 4,194,304 values (PSR_EINVAL
 * beyond).  Every call looks up that array's address in the current context (no
 * allocation); the first call on a device also loads the library's module, so make it
 * before any stream capture.  All calls share the array, so calls that overlap on the GPU
 * (e.g. on different streams) race; results are stream-ordered, no synchronisation. */
int psr_isovalue_static(int32_t dtype, const void* values, const void* weights, int64_t n, void* out, void* stream);

/* Reverse pass of a reconstruction made with params.differentiable (warp-psr
 * reconstruction_adjoint.py:99-172): the vector-Jacobian product of the finite algorithm
 * the forward ran, with its discrete choices fixed (groups, tree, bins, schedules, CG
 * stopping points).  Seeds (device pointers, result dtype; NULL = zero): g_coefficients and
 * g_cumulative (total values each), g_iso (one value), g_normalization (5, the adjoint of
 * psr_info.normalization).
 * positions/normals are the forward's inputs (unchanged since), n points of input dtype
 * `dtype`; g_positions and g_normals (n x 3, input dtype) are written, stream-ordered on
 * `stream` (the call returns without waiting for the device; psr_result_info waits for the
 * pass when it reports backward_ms).  The tape stays, so the pass can be repeated with other
 * seeds. */
int psr_backward(psr_result* result, const void* positions, const void* normals, int64_t n, int32_t dtype,
                 const void* g_coefficients, const void* g_cumulative, const void* g_iso, const void* g_normalization,
                 void* g_positions, void* g_normals, void* stream);

/* psr_evaluate reversed: seeds g_values (nq) and g_gradients (nq x 3, NULL = zero), result
 * dtype.  g_coefficients and g_cumulative (total values) accumulate; g_queries (nq x 3, may
 * be NULL) is written; g_normalization (5, may be NULL) accumulates the adjoint of the model
 * to cube transform, expressed on psr_info.normalization. */
int psr_evaluate_backward(const psr_result* result, const void* queries, int64_t nq, const void* g_values,
                          const void* g_gradients, void* g_coefficients, void* g_cumulative, void* g_queries,
                          void* g_normalization, void* stream);

/* ---- Sparse marching cubes: the field's mesh consumer (warp-psr meshing.py:150-346) ----
 * Grid: shape[0..2] >= 2 nodes per axis spanning [lower, upper] in model space, the spacing
 * step = (upper - lower) / (shape - 1) computed in float32 as the reference does; node
 * (i, j, k) sits at min(max(lower + step * (i, j, k), lower), upper), node index
 * (i * ny + j) * nz + k, cell index (i * (ny - 1) + j) * (nz - 1) + k.  Values are centred
 * (field - isovalue) in dtype; a node is inside when its value is >= 0 and a cell is kept when
 * its corners are neither all inside nor all outside.  Triangles are oriented with normals
 * pointing from inside to outside; one vertex per crossing grid edge, at pa + t (pb - pa),
 * t = fa / (fa - fb), on the edge's lower node a and upper node b. */
typedef struct psr_mesh psr_mesh;

/* Model positions (count x 3, dtype) of the nodes of x-planes start.. (cells == NULL: count =
 * (planes) * ny * nz) or of the eight corners of each listed cell (count = 8 * cells). */
int psr_mc_points(int32_t dtype, const int64_t shape[3], const double lower[3], const double upper[3],
                  const int64_t* cells, int64_t start, int64_t count, void* points, void* stream);
/* Sets the mask bit (uint32 words over all cells) of every crossing cell of the x-slab
 * [start, start + width) from the values of its (width + 1) * ny * nz nodes; status[0] |= 1
 * if a value is not finite (meshing.py:45-60). */
int psr_mc_mark(int32_t dtype, const void* values, const int64_t shape[3], int64_t start, int64_t width,
                uint32_t* mask, int32_t* status, void* stream);
/* Number of marked cells (*count, a host read) and, when cells != NULL, their indices in
 * ascending order (meshing.py:63-85). */
int psr_mc_cells(const uint32_t* mask, int64_t words, int64_t* cells, int64_t capacity, int64_t* count, void* stream);
/* Triangles of the listed cells from their corner values (count x 8, corner order 000, 100,
 * 110, 010, 001, 101, 111, 011). */
int psr_mc_triangulate(int32_t dtype, const int64_t shape[3], const double lower[3], const double upper[3],
                       const int64_t* cells, const void* corner_values, int64_t count, psr_mesh** out, void* stream);
/* The whole extraction on a reconstruction's own field (extract_mesh, meshing.py:284-346):
 * slabs of `slab` x-planes classified with the library's evaluator, then the kept cells'
 * corners evaluated and triangulated; *retained = kept cells.  PSR_EDATA if a grid node lies
 * outside the reconstruction cube (nonfinite field value). */
int psr_extract_mesh(const psr_result* result, const int64_t shape[3], const double lower[3], const double upper[3],
                     double iso, int64_t slab, int64_t* retained, psr_mesh** out, void* stream);
int psr_mesh_info(const psr_mesh* mesh, int32_t* dtype, int64_t* vertices, int64_t* triangles, int64_t* cells);
/* vertices (x 3, dtype), indices (triangles x 3, int32), the crossing edge of each vertex
 * ((lower node index) * 3 + axis), its two corner values (cell * 8 + corner, flat indices
 * into the corner values), and the kept cells (psr_extract_mesh; NULL otherwise). */
int psr_mesh_arrays(const psr_mesh* mesh, const void** vertices, const int32_t** indices, const int64_t** edges,
                    const int64_t** ends, const int64_t** cells);
int psr_mesh_free(psr_mesh* mesh);

#ifdef __cplusplus
}
#endif
#endif
