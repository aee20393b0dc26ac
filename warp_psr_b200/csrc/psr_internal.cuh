// Internal stage interfaces of the screened-Poisson pipeline.  Each stage runs on one
// stream; data-dependent sizes are read back with read_scalar (a handful per stage).
#pragma once
#include "psr_common.cuh"

#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace psr {

struct Params {
  int depth, full_depth, base_depth, solve_depth, kernel_depth;
  double samples_per_node, scale, point_weight, cg_accuracy;
  int exact, iters, base_v_cycles, precision;
  int differentiable = 0;
};

// Optional copies of intermediate arrays, kept for stage-by-stage parity checks.
struct StageSink {
  struct Entry {
    DBuf<char> data;
    int64_t count = 0;
    int elem = 0;
  };
  bool on = false;
  std::map<std::string, Entry> entries;
  template <class V>
  void put(const std::string& name, const V* src, int64_t count, cudaStream_t s) {
    if (!on) return;
    Entry e;
    e.count = count;
    e.elem = int(sizeof(V));
    e.data.alloc(count * int64_t(sizeof(V)), s);
    if (count > 0) PSR_CUDA(cudaMemcpyAsync(e.data.p, src, count * sizeof(V), cudaMemcpyDeviceToDevice, s));
    entries[name] = std::move(e);
  }
};

// Stream-ordered stage timer: mark(k) closes the interval since the previous mark and adds
// its device time to slot k (read after the stream has synchronised).
struct EventMarks {
  std::vector<std::pair<int, cudaEvent_t>> marks;
  cudaEvent_t start = nullptr;
  void begin(cudaStream_t s) {
    PSR_CUDA(cudaEventCreate(&start));
    PSR_CUDA(cudaEventRecord(start, s));
  }
  void mark(int slot, cudaStream_t s) {
    cudaEvent_t e;
    PSR_CUDA(cudaEventCreate(&e));
    PSR_CUDA(cudaEventRecord(e, s));
    marks.emplace_back(slot, e);
  }
  bool pending() const { return start != nullptr; }
  void collect(double* out, int slots) {  // waits for the last mark
    if (!marks.empty()) cudaEventSynchronize(marks.back().second);
    for (int i = 0; i < slots; ++i) out[i] = 0;
    cudaEvent_t prev = start;
    for (auto& m : marks) {
      float ms = 0;
      if (prev && cudaEventElapsedTime(&ms, prev, m.second) == cudaSuccess && m.first < slots) out[m.first] += ms;
      prev = m.second;
    }
    for (auto& m : marks) cudaEventDestroy(m.second);
    if (start) cudaEventDestroy(start);
    marks.clear();
    start = nullptr;
  }
  EventMarks() = default;
  EventMarks(const EventMarks&) = delete;
  EventMarks& operator=(const EventMarks&) = delete;
  ~EventMarks() {
    for (auto& m : marks) cudaEventDestroy(m.second);
    if (start) cudaEventDestroy(start);
  }
};
// Process-wide device time of selected kernels, for the per-kernel roofline: a diagnostic,
// off unless PSR_KERNEL_CLOCKS=1 when the launch is issued.  A KernelClock brackets one
// launch with events; `bytes` is the launch's algorithmic traffic (what it must read and
// write once), `units` the rows, points or row visits it processes.  psr_kernel_clocks()
// waits for the events, reports the totals per kernel and clears them.
enum ClockKind {
  kClkAssembleSliced,
  kClkCrossApply,
  kClkNormalStencil,
  kClkBaseRelax,
  kClkStripForward,
  kClkStripReverse,
  kClkNormalStencilReverse,
  kClkLevelRowsReverse,
  kClkScreeningReverse,
  kClkKinds
};
bool kernel_clocks_on();
void kernel_clock_push(int kind, double bytes, double units, cudaEvent_t a, cudaEvent_t b);
struct KernelClock {
  int kind;
  double bytes, units;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  KernelClock(int kind_, double bytes_, double units_, cudaStream_t s_)
      : kind(kind_), bytes(bytes_), units(units_), s(s_) {
    if (kernel_clocks_on() && cudaEventCreate(&a) == cudaSuccess) cudaEventRecord(a, s);
  }
  void stop() {  // closes the interval (at scope end if not called)
    cudaEvent_t b = nullptr;
    if (a && cudaEventCreate(&b) == cudaSuccess && cudaEventRecord(b, s) == cudaSuccess)
      kernel_clock_push(kind, bytes, units, a, b);
    else if (a)
      cudaEventDestroy(a);
    a = nullptr;
  }
  ~KernelClock() { stop(); }
  KernelClock(const KernelClock&) = delete;
  KernelClock& operator=(const KernelClock&) = delete;
};

enum { kBwField, kBwMirror, kBwSweep, kBwOperator, kBwBase, kBwPoints, kBwNormalLoads, kBwSamples, kBwSlots };

// Sets the message psr_last_error returns on this thread.
void set_last_error(const std::string& message);

// ---------------------------------------------------------------- A1 samples.py
template <class T>
struct SampleGroups {
  int64_t count = 0;          // G accepted leaf groups
  DBuf<int64_t> keys;         // basis keys at `depth`, sorted
  DBuf<T> sums, normal_sums;  // 3 per group (positions / unit normals, unit-cube frame)
  DBuf<T> weights;            // sample count per group
  DBuf<int32_t> first;        // smallest input index of the group
  DBuf<T> transform;          // [inv, t0, t1, t2, normal_scale]
  // Kept for the adjoint only (`keep`): group of every input point (-1 when rejected), the
  // bounding box [lo xyz, hi xyz] and, per bound, the lowest input index attaining it.
  DBuf<int32_t> input_group;
  DBuf<T> bounds;
  DBuf<int32_t> bound_owner;
};
template <class T>
SampleGroups<T> prepare_samples(const T* pos, const T* nrm, int64_t n, int depth, double scale, cudaStream_t s,
                                bool keep = false);

// ---------------------------------------------------------------- A2 density.py
template <class T>
struct DensityData {
  std::vector<DBuf<int64_t>> agg_keys;  // per depth, sorted basis keys of occupied cells
  std::vector<DBuf<T>> agg_values;      // 4 per record: position sum xyz, weight
  std::vector<int64_t> agg_count;
  DBuf<T> dw;                           // 2 per group: raw splat depth, splat weight
  T scale;
  // Kept for the adjoint only (`keep`):
  std::vector<DBuf<int32_t>> parent_of;   // [d]: aggregate index at d-1 of each record at d
  std::vector<DBuf<int32_t>> splat_order; // [d]: morton order of the depth-d aggregates
  std::vector<DBuf<int32_t>> splat_slot;  // [d]: unique level value of splat record 27*i+k, or -1
  std::vector<DBuf<T>> level_values;      // [d]: reduced density splat values
  std::vector<HashMap> level_hash;        // [d]: their keys
  DBuf<T> densities;                      // G x (kernel_depth+1) density at each group centroid
};
template <class T>
DensityData<T> build_density(const SampleGroups<T>& g, int depth, int kernel_depth, double spn, cudaStream_t s,
                             bool keep = false);
template <class T>
T density_scale();

// ---------------------------------------------------------------- A3 normals.py
template <class T>
struct NormalData {
  int64_t count = 0;
  DBuf<int64_t> keys;               // sorted basis keys of every level
  DBuf<T> values;                   // 4 per record (negated normal coefficients, 4th = -0)
  std::vector<int64_t> offsets;     // per depth, depth+2 entries
  DBuf<T> average;                  // [mean depth, mean weight, total weight]
  // Kept for the adjoint only (`keep`): groups in first-index order and the unique record
  // of every splat record 54*i+k (-1 when the record was not emitted).
  DBuf<int32_t> group_order;
  DBuf<int32_t> record_slot;
};
template <class T>
NormalData<T> build_normals(const SampleGroups<T>& g, const DensityData<T>& D, int minimum, int maximum,
                            cudaStream_t s, bool keep = false);

// ---------------------------------------------------------------- A4 tree.py
struct TreeData {
  std::vector<DBuf<int64_t>> support;  // signed tree keys per depth (non-ghost support)
  std::vector<DBuf<int64_t>> basis;    // basis keys per depth
  std::vector<int64_t> support_count, basis_count;
};
template <class T>
TreeData build_tree(const NormalData<T>& N, int depth, int full_depth, int base_depth, cudaStream_t s);

// ---------------------------------------------------------------- A5-A10 solver.py
struct RelaxDeferred {
  int* error = nullptr;                                                // device word, zeroed before the first launch
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* events = nullptr;  // created by the launch, owned by the caller
};
void throw_relax_error(int err);  // nonzero relaxation error code -> Error

struct SolveStats {
  double relax_ms = 0;       // ordered relaxation kernels (sum over levels)
  int64_t row_visits = 0;    // rows x sweeps relaxed by the sliced kernels
  int64_t launches = 0;
  std::vector<double> level_relax_ms;
  int64_t finest_row_visits = 0;  // rows x sweeps of the last (finest) sliced level
  // Read back once, after the caller's stream synchronisation (finish), not per level.
  DBuf<int> relax_error;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> relax_events;
  RelaxDeferred defer(cudaStream_t s) {
    if (!relax_error.p) {
      relax_error.alloc(1, s);
      relax_error.zero();
    }
    return RelaxDeferred{relax_error.p, &relax_events};
  }
  // The stream has synchronised: throws the first relaxation error, else fills the timings.
  void finish() {
    int err = 0;
    if (relax_error.p) PSR_CUDA(cudaMemcpy(&err, relax_error.p, sizeof(int), cudaMemcpyDeviceToHost));
    for (auto& e : relax_events) {
      float ms = 0;
      if (!err) PSR_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
      relax_ms += ms;
      level_relax_ms.push_back(ms);
    }
    release();
    throw_relax_error(err);
  }
  void release() {
    for (auto& e : relax_events) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    relax_events.clear();
  }
  SolveStats() = default;
  SolveStats(const SolveStats&) = delete;
  SolveStats& operator=(const SolveStats&) = delete;
  ~SolveStats() { release(); }
};
// With `tape_out` the solve keeps what its adjoint needs (an opaque SolveTape<T>).
template <class T>
void solve_levels(const TreeData& tree, const DensityData<T>& D, const NormalData<T>& N,
                  const std::vector<int64_t>& level_offsets, const int64_t* all_keys, const HashMap& all_hash,
                  const Params& p, T* coefficients, cudaStream_t s, SolveStats* stats, StageSink* sink,
                  std::shared_ptr<void>* tape_out = nullptr);

// Reverse pass of solve_levels over its tape: from the adjoint of the per-level coefficients
// (all levels, key order) to the adjoints of the density aggregates (g_agg[d], 4 per record,
// accumulated), of the normal average (3, accumulated) and of the normal coefficients
// (4 per record, accumulated).
template <class T>
void solve_backward(void* tape, const TreeData& tree, const DensityData<T>& D, const NormalData<T>& N,
                    const std::vector<int64_t>& level_offsets, const int64_t* all_keys, const HashMap& all_hash,
                    const Params& p, const T* g_coef, std::vector<DBuf<T>>& g_agg, T* g_average, T* g_nvals,
                    cudaStream_t s, EventMarks* marks = nullptr);

// Index rows of the schedule-order operator: 32 slots (0..26 neighbours, 27 own index); the
// padding slots 28..31 carry 1 / A_ii in the vector precision (write_inv_diag).
// An absent neighbour in those index rows is the most negative index: its footprint position
// (index + a non-negative offset below 2^15 for 16-bit rows, below 2^31 for 32-bit, taken
// unsigned) always lies past the footprint's end, where the relaxation keeps a +0 entry.
template <class I>
__host__ __device__ constexpr I idx_absent() {
  return sizeof(I) == 2 ? I(-32768) : I(-2147483647 - 1);
}
template <class V, class I>
__host__ __device__ __forceinline__ void write_inv_diag(I* row, V inv) {
  static_assert(4 * sizeof(I) >= sizeof(V), "index padding too small for the reciprocal");
  memcpy(reinterpret_cast<char*>(row + 28), &inv, sizeof(V));
}

// Stored index rows keep their 16-byte chunks permuted by schedule position: logical chunk q
// of row p sits at chunk q ^ idx_swizzle<I>(p).  Any eight consecutive rows then hold a given
// logical chunk in eight different groups of four shared-memory banks (64-byte rows of 16-bit
// indices: two rows per 128 bytes, four chunks; 128-byte rows of 32-bit indices: eight
// chunks), so a warp reading one chunk of 32 consecutive staged rows takes the minimum of four
// wavefronts instead of sixteen (thirty-two for 32-bit rows), at any offset of the rows in
// shared memory.  Rows are written and read whole through store_idx_row / load_idx_row.
template <class I>
__host__ __device__ constexpr int idx_chunks() {
  return 32 * int(sizeof(I)) / 16;
}
template <class I>
__host__ __device__ __forceinline__ int idx_swizzle(int64_t p) {
  return int(p / (8 / idx_chunks<I>())) & (idx_chunks<I>() - 1);
}
// Position of logical slot k in the stored row of schedule position p.
template <class I>
__host__ __device__ __forceinline__ int idx_slot(int64_t p, int k) {
  constexpr int E = 16 / int(sizeof(I));
  return ((k / E) ^ idx_swizzle<I>(p)) * E + k % E;
}
// Logical row (32 slots, 16-byte aligned) of schedule position p from its stored row.
template <class I>
__device__ __forceinline__ void load_idx_row(const I* stored, int64_t p, I* out) {
  const int g = idx_swizzle<I>(p);
  const int4* src = reinterpret_cast<const int4*>(stored);
  int4* dst = reinterpret_cast<int4*>(out);
#pragma unroll
  for (int q = 0; q < idx_chunks<I>(); ++q) dst[q] = src[q ^ g];
}
template <class I>
__device__ __forceinline__ void load_idx_row_ldg(const I* stored, int64_t p, I* out) {
  const int g = idx_swizzle<I>(p);
  const int4* src = reinterpret_cast<const int4*>(stored);
  int4* dst = reinterpret_cast<int4*>(out);
#pragma unroll
  for (int q = 0; q < idx_chunks<I>(); ++q) dst[q] = __ldg(src + (q ^ g));
}
template <class I>
__device__ __forceinline__ void store_idx_row(I* stored, int64_t p, const I* in) {
  const int g = idx_swizzle<I>(p);
  int4* dst = reinterpret_cast<int4*>(stored);
  const int4* src = reinterpret_cast<const int4*>(in);
#pragma unroll
  for (int q = 0; q < idx_chunks<I>(); ++q) dst[q ^ g] = src[q];
}

// Schedule order of a sliced level: rows sorted by (slice, colour), key order inside a group.
struct StripSchedule {
  int64_t rows = 0;
  int depth = 0;
  bool wide = false;          // a (slice, colour) group too large for 16-bit neighbour indices
  DBuf<int32_t> perm, inv;    // schedule position -> key-order row, and back
  DBuf<int32_t> off;          // 4*(2^depth+1)+1 group offsets
  DBuf<int64_t> skeys;        // keys in schedule order
};
void build_strip_schedule(const int64_t* keys, int64_t rows, int depth, StripSchedule& S, cudaStream_t s);

// Strip-scheduled relaxation of operator rows already in schedule order: values T[28] and
// group-relative neighbour indices I[32] per row, b with 16 bytes of slack; x in key order
// holds the initial guess and receives the result.
//
// `hist` (optional, rows x iters in schedule order: row p, visit t at p * iters + t) receives
// per visit the new x of every row, or with `record_increment` the update r / A_ii.  `rev`
// runs the exact reverse of the forward sequential order over the same schedule-order rows:
// slices 2^d .. 0 (logical slice z is stored slice 2^d - z) and the colours of a slice in the
// order 3, 2, 1, 0 (used by the adjoint on the transposed operator).
// With `defer`, a launch merges its error code into defer->error (the first nonzero code wins,
// on the device) and appends its start/end events to defer->events instead of reading either
// back, so a stage that relaxes several levels synchronises once rather than once per level.
template <class T, class V, class I>
void relax_strips_scheduled(const StripSchedule& S, const T* svals, const I* sidx, const V* sb, V* x, int iters,
                            cudaStream_t s, float* ms, V* hist = nullptr, bool rev = false,
                            bool record_increment = false, RelaxDeferred* defer = nullptr);

// Strip-scheduled ordered relaxation (psr_relax.cu): slot-ELL rows in key order, x in key
// order holds the initial guess and receives the result.
template <class T, class V>
void relax_sliced_strips(const int64_t* keys, int64_t rows, int depth, const int32_t* cols, const T* vals,
                         const V* b, V* x, int iters, cudaStream_t s, float* ms);

// ---------------------------------------------------------------- A11/A12 field.py, reconstruction.py
template <class T>
void cumulative_coefficients(const int64_t* keys, const std::vector<int64_t>& offsets, const HashView& h,
                             const T* coeff, T* cumulative, int depth, cudaStream_t s);
template <class T>
void evaluate_queries(const int64_t* keys, const HashView& h, const T* coeff, const T* cumulative, const T* queries,
                      int64_t nq, const T* linear, const T* translation, int depth, T* values, T* gradients,
                      int32_t* valid, bool cube_frame, const T* group_sums, const T* group_weights, cudaStream_t s);
template <class T>
void isovalue(const T* values, const T* weights, int64_t n, T* out, cudaStream_t s);
template <class T>
void evaluation_transforms(const T* normalization, T* transforms /* 32 */, cudaStream_t s);

// ---------------------------------------------------------------- A13 reverse passes
// Isovalue (seed g_iso) through the centroid evaluation, then the cumulative coefficients:
// g_coeff and g_cum (in/out) end as the adjoint of the per-level coefficients; g_sums (3 per
// group, accumulated) receives the centroids' share.
template <class T>
void field_backward(const int64_t* keys, const std::vector<int64_t>& offsets, const HashView& h, const T* coeff,
                    const T* cumulative, int depth, const T* gsums, const T* gweights, int64_t groups, const T* g_iso,
                    T* g_coeff, T* g_cum, T* g_sums, cudaStream_t s);
// Model-frame query evaluation reversed: g_coeff, g_cum accumulate; g_queries is written;
// g_ltr (12 float64: L row-major, then tr) accumulates.
template <class T>
void evaluate_backward(const HashView& h, const T* coeff, const T* cumulative, const T* queries, int64_t nq,
                       const T* linear, const T* translation, int depth, const T* g_values, const T* g_gradients,
                       T* g_coeff, T* g_cum, T* g_queries, double* g_ltr, cudaStream_t s);
// Normal splat, splat depths, density and sample preparation reversed onto the inputs.
template <class T>
void samples_backward(const SampleGroups<T>& G, const DensityData<T>& D, const NormalData<T>& N, int depth,
                      int kernel_depth, int base_depth, double samples_per_node, double scale,
                      std::vector<DBuf<T>>& g_agg, const T* g_average, const T* g_nvals, T* g_sums,
                      const T* g_transform, const T* pos, const T* nrm, int64_t n, T* g_pos, T* g_nrm,
                      cudaStream_t s);

}  // namespace psr
