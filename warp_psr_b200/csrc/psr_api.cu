// C ABI of libpsr_b200 (declared in include/psr_b200.h): argument validation, stage
// orchestration on the caller's stream, result ownership and the stage-level entry points.
#include "../../include/psr_b200.h"
#include "psr_internal.cuh"

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

using namespace psr;

static thread_local std::string g_error;

namespace psr {
std::atomic<long long> g_kernel_launches{0};

void set_last_error(const std::string& message) { g_error = message; }

namespace clocks {
struct ClockTotals {
  long long launches = 0;
  double ms = 0, bytes = 0, units = 0;
};
struct PendingClock {
  int kind;
  double bytes, units;
  cudaEvent_t a, b;
};
std::mutex g_clock_mutex;
std::vector<PendingClock> g_clock_pending;
ClockTotals g_clock_totals[kClkKinds];
const char* const kClockNames[kClkKinds] = {
    "assemble_sliced_kernel",        "cross_apply_kernel",        "normal_stencil_dense_kernel",
    "relax_colors_shared_kernel",    "strip_gs_kernel (forward)", "strip_gs_kernel (reverse)",
    "normal_stencil_reverse_kernel", "level_rows_reverse_kernel", "screening_points_reverse_kernel"};
const char* const kClockUnits[kClkKinds] = {"row", "row", "row", "row visit", "row visit",
                                            "row visit", "normal record", "row", "point"};
}  // namespace clocks
using namespace clocks;

bool kernel_clocks_on() {
  const char* v = std::getenv("PSR_KERNEL_CLOCKS");
  return v && v[0] == '1';
}

void kernel_clock_push(int kind, double bytes, double units, cudaEvent_t a, cudaEvent_t b) {
  std::lock_guard<std::mutex> lock(clocks::g_clock_mutex);
  clocks::g_clock_pending.push_back(PendingClock{kind, bytes, units, a, b});
  // Bound the events held while nobody reads the clocks: fold the older half into the
  // totals (waiting for those launches; a diagnostic mode only).
  if (clocks::g_clock_pending.size() >= 4096) {
    const size_t half = clocks::g_clock_pending.size() / 2;
    for (size_t i = 0; i < half; ++i) {
      PendingClock& c = clocks::g_clock_pending[i];
      float ms = 0;
      if (cudaEventSynchronize(c.b) == cudaSuccess && cudaEventElapsedTime(&ms, c.a, c.b) == cudaSuccess) {
        clocks::ClockTotals& t = clocks::g_clock_totals[c.kind];
        t.launches += 1;
        t.ms += ms;
        t.bytes += c.bytes;
        t.units += c.units;
      }
      cudaEventDestroy(c.a);
      cudaEventDestroy(c.b);
    }
    clocks::g_clock_pending.erase(clocks::g_clock_pending.begin(), clocks::g_clock_pending.begin() + half);
  }
}

__global__ void hash_insert_kernel(const int64_t* __restrict__ src, int64_t n, longlong2* slots, uint64_t mask,
                                   int32_t value_offset) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int64_t key = src[i];
  uint64_t h = HashView::mix(uint64_t(key)) & mask;
  while (true) {
    unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&slots[h].x), ~0ULL,
                                        static_cast<unsigned long long>(key));
    if (prev == ~0ULL || prev == static_cast<unsigned long long>(key)) {
      slots[h].y = int64_t(int32_t(i) + value_offset);
      return;
    }
    h = (h + 1) & mask;
  }
}

__global__ void hash_insert_counted_kernel(const int64_t* __restrict__ src, int64_t n_max, const int32_t* count,
                                           longlong2* slots, uint64_t mask) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n_max || i >= int64_t(*count)) return;
  int64_t key = src[i];
  uint64_t h = HashView::mix(uint64_t(key)) & mask;
  while (true) {  // the table holds more than twice n_max slots: a free one is always found
    unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&slots[h].x), ~0ULL,
                                        static_cast<unsigned long long>(key));
    if (prev == ~0ULL || prev == static_cast<unsigned long long>(key)) {
      slots[h].y = i;
      return;
    }
    h = (h + 1) & mask;
  }
}

// Column heads of sorted keys: (depth, x, y) changes.
__global__ void column_insert_kernel(const int64_t* __restrict__ keys, int64_t n, longlong2* slots, uint64_t mask) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int64_t k = keys[i];
  if (i > 0 && (keys[i - 1] >> 16) == (k >> 16)) return;
  int64_t key = (k >> 16) << 16;
  uint64_t h = HashView::mix(uint64_t(key)) & mask;
  while (true) {
    unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&slots[h].x), ~0ULL,
                                        static_cast<unsigned long long>(key));
    if (prev == ~0ULL || prev == static_cast<unsigned long long>(key)) {
      slots[h].y = int64_t(i);
      return;
    }
    h = (h + 1) & mask;
  }
}

__global__ void dense_column_kernel(const int64_t* __restrict__ keys, int64_t n, int2* dense, int32_t* error) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int64_t k = keys[i];
  if (i > 0 && (keys[i - 1] >> 16) == (k >> 16)) return;
  int c[3];
  key_coords(k, c);
  const int d = int(k >> 48), side = (1 << d) + 1;
  if (d > kDenseColumnDepth || unsigned(c[0]) >= unsigned(side) || unsigned(c[1]) >= unsigned(side)) {
    atomicExch(error, 1);
    return;
  }
  dense[dense_column_base(d) + int64_t(c[0]) * side + c[1]] = make_int2(int32_t(i), 0);
}

// Second pass: the last key of each column stores the column's length.
__global__ void dense_count_kernel(const int64_t* __restrict__ keys, int64_t n, int2* dense) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int64_t k = keys[i];
  if (i + 1 < n && (keys[i + 1] >> 16) == (k >> 16)) return;
  int c[3];
  key_coords(k, c);
  const int d = int(k >> 48), side = (1 << d) + 1;
  if (d > kDenseColumnDepth || unsigned(c[0]) >= unsigned(side) || unsigned(c[1]) >= unsigned(side)) return;
  int2* e = dense + dense_column_base(d) + int64_t(c[0]) * side + c[1];
  e->y = int32_t(i + 1) - e->x;
}
}  // namespace psr

struct psr_result {
  int dtype = 0;
  int depth = 0;
  Params params{};
  int64_t groups = 0;
  std::vector<int64_t> level_offsets;
  std::vector<int64_t> support_count;
  DBuf<int64_t> keys;
  DBuf<char> coefficients, cumulative, transforms;
  std::vector<DBuf<int64_t>> support;
  HashMap hash;
  double iso = 0;
  double host_transforms[32] = {0};
  double normalization[5] = {0};
  std::shared_ptr<void> tape;  // psr::Tape<T> of a differentiable reconstruction
  double stage_ms[8] = {0};
  SolveStats stats;
  StageSink sink;
  // last reverse pass, per stage (psr_info.backward_ms): its event marks are read when the
  // info is asked for, so the pass itself ends without a host synchronisation
  mutable double backward_ms[8] = {0};
  mutable psr::EventMarks bw_marks;
};

namespace psr {
// Everything the reverse pass needs, kept by a differentiable reconstruction.
template <class T>
struct Tape {
  SampleGroups<T> G;
  DensityData<T> D;
  NormalData<T> N;
  TreeData tree;
  std::shared_ptr<void> solve;
  int64_t n_input = 0;
};
}  // namespace psr

namespace {

int fail(const Error& e) {
  g_error = e.what();
  return e.code;
}

void validate(const psr_params* p) {
  if (!p) throw Error(PSR_EINVAL, "params must not be NULL");
  // reconstruction.py:160-203
  if (!(0 <= p->base_depth && p->base_depth <= p->full_depth && p->full_depth <= p->solve_depth &&
        p->solve_depth <= p->depth && p->depth <= 15) ||
      p->depth < 1 || !(0 <= p->kernel_depth && p->kernel_depth <= p->depth))
    throw Error(PSR_EINVAL,
                "Require 0 <= base_depth <= full_depth <= solve_depth <= depth <= 15, depth >= 1, and 0 <= "
                "kernel_depth <= depth");
  if (p->iters < 1 || p->base_v_cycles < 1) throw Error(PSR_EINVAL, "iters and base_v_cycles must be positive integers");
  if (!std::isfinite(p->point_weight) || p->point_weight < 0 || !std::isfinite(p->cg_accuracy) || p->cg_accuracy <= 0)
    throw Error(PSR_EINVAL, "Require finite nonnegative point_weight and positive cg_accuracy");
  if (!std::isfinite(p->samples_per_node) || p->samples_per_node <= 0 || !std::isfinite(p->scale) || p->scale <= 1)
    throw Error(PSR_EINVAL, "Require finite positive samples_per_node and scale > 1");
  if (p->precision != PSR_PRECISION_INPUT && p->precision != PSR_PRECISION_MIXED)
    throw Error(PSR_EINVAL, "precision must be PSR_PRECISION_INPUT or PSR_PRECISION_MIXED");
}

void tune_pool() {  // once per device: each device has its own default pool
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  PSR_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = dev < 64 ? uint64_t(1) << dev : 0;
  if (bit && (done.load() & bit)) return;
  cudaMemPool_t pool;
  PSR_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t threshold = ~uint64_t(0);
  PSR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  done.fetch_or(bit);
}

__global__ void upcast_kernel(const float* in, int64_t n, double* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = double(in[i]);
}


template <class T>
void run(const T* pos, const T* nrm, int64_t n, const Params& prm, cudaStream_t s, psr_result* R) {
  cudaEvent_t ev[8];
  for (auto& e : ev) PSR_CUDA(cudaEventCreate(&e));
  PSR_CUDA(cudaEventRecord(ev[0], s));
  const bool keep = prm.differentiable != 0;
  SampleGroups<T> G = prepare_samples<T>(pos, nrm, n, prm.depth, prm.scale, s, keep);
  PSR_CUDA(cudaEventRecord(ev[1], s));
  DensityData<T> D = build_density<T>(G, prm.depth, prm.kernel_depth, prm.samples_per_node, s, keep);
  PSR_CUDA(cudaEventRecord(ev[2], s));
  NormalData<T> N = build_normals<T>(G, D, prm.base_depth, prm.depth, s, keep);
  StageSink& sink = R->sink;
  sink.put("group_keys", G.keys.p, G.count, s);
  sink.put("group_sums", G.sums.p, 3 * G.count, s);
  sink.put("group_normal_sums", G.normal_sums.p, 3 * G.count, s);
  sink.put("group_weights", G.weights.p, G.count, s);
  sink.put("group_first", G.first.p, G.count, s);
  sink.put("transform", G.transform.p, 5, s);
  sink.put("depths_and_weights", D.dw.p, 2 * G.count, s);
  sink.put("normal_keys", N.keys.p, N.count, s);
  sink.put("normal_values", N.values.p, 4 * N.count, s);
  sink.put("normal_average", N.average.p, 3, s);
  PSR_CUDA(cudaEventRecord(ev[3], s));
  TreeData tree = build_tree<T>(N, prm.depth, prm.full_depth, prm.base_depth, s);
  PSR_CUDA(cudaEventRecord(ev[4], s));
  // Concatenated basis keys of every level (reconstruction.py:260-267).
  R->level_offsets.assign(prm.depth + 2, 0);
  for (int d = 0; d <= prm.depth; ++d) R->level_offsets[d + 1] = R->level_offsets[d] + tree.basis_count[d];
  int64_t total = R->level_offsets[prm.depth + 1];
  R->keys.alloc(total, s);
  for (int d = 0; d <= prm.depth; ++d)
    if (tree.basis_count[d])
      PSR_CUDA(cudaMemcpyAsync(R->keys.p + R->level_offsets[d], tree.basis[d].p, tree.basis_count[d] * sizeof(int64_t),
                               cudaMemcpyDeviceToDevice, s));
  R->hash.build(R->keys.p, total, s);
  R->coefficients.alloc(total * int64_t(sizeof(T)), s);
  R->coefficients.zero();
  T* coeff = reinterpret_cast<T*>(R->coefficients.p);
  std::shared_ptr<void> solve_tape;
  solve_levels<T>(tree, D, N, R->level_offsets, R->keys.p, R->hash, prm, coeff, s, &R->stats, &sink,
                  keep ? &solve_tape : nullptr);
  PSR_CUDA(cudaEventRecord(ev[5], s));
  R->cumulative.alloc(total * int64_t(sizeof(T)), s);
  T* cum = reinterpret_cast<T*>(R->cumulative.p);
  HashView hv = R->hash.view();
  cumulative_coefficients<T>(R->keys.p, R->level_offsets, hv, coeff, cum, prm.depth, s);
  DBuf<T> values(G.count, s);
  evaluate_queries<T>(R->keys.p, hv, coeff, cum, nullptr, G.count, nullptr, nullptr, prm.depth, values.p, nullptr,
                      nullptr, true, G.sums.p, G.weights.p, s);
  PSR_CUDA(cudaEventRecord(ev[6], s));
  sink.put("centroid_values", values.p, G.count, s);
  DBuf<T> iso(1, s);
  isovalue<T>(values.p, G.weights.p, G.count, iso.p, s);
  R->transforms.alloc(32 * int64_t(sizeof(T)), s);
  evaluation_transforms<T>(G.transform.p, reinterpret_cast<T*>(R->transforms.p), s);
  PSR_CUDA(cudaEventRecord(ev[7], s));
  T host_iso;
  T host_tr[32];
  T host_norm[5];
  PSR_CUDA(cudaMemcpyAsync(&host_iso, iso.p, sizeof(T), cudaMemcpyDeviceToHost, s));
  PSR_CUDA(cudaMemcpyAsync(host_tr, R->transforms.p, 32 * sizeof(T), cudaMemcpyDeviceToHost, s));
  PSR_CUDA(cudaMemcpyAsync(host_norm, G.transform.p, 5 * sizeof(T), cudaMemcpyDeviceToHost, s));
  PSR_CUDA(cudaStreamSynchronize(s));
  R->stats.finish();
  R->iso = double(host_iso);
  for (int i = 0; i < 32; ++i) R->host_transforms[i] = double(host_tr[i]);
  for (int i = 0; i < 5; ++i) R->normalization[i] = double(host_norm[i]);
  for (int i = 0; i < 7; ++i) {
    float ms = 0;
    PSR_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
    R->stage_ms[i] = ms;
  }
  float all = 0;
  PSR_CUDA(cudaEventElapsedTime(&all, ev[0], ev[7]));
  R->stage_ms[7] = all;
  for (auto& e : ev) cudaEventDestroy(e);
  R->groups = G.count;
  R->support_count = tree.support_count;
  R->support = std::move(tree.support);
  if (keep) {
    auto tape = std::make_shared<Tape<T>>();
    tape->G = std::move(G);
    tape->D = std::move(D);
    tape->N = std::move(N);
    tape->tree = std::move(tree);
    tape->solve = std::move(solve_tape);
    tape->n_input = n;
    R->tape = tape;
  }
}

template <class T>
__global__ void cast_kernel_t(const void* in, int in_double, int64_t n, T* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  out[i] = in_double ? T(static_cast<const double*>(in)[i]) : T(static_cast<const float*>(in)[i]);
}

// Reverse pass: field (isovalue, cumulative) -> solve -> splats, density -> inputs.
template <class T>
void backward(psr_result* R, const T* pos, const T* nrm, int64_t n, const T* g_coef_in, const T* g_cum_in,
              const T* g_iso, const T* g_norm, T* g_pos, T* g_nrm, cudaStream_t s) {
  Tape<T>& tp = *static_cast<Tape<T>*>(R->tape.get());
  const Params& prm = R->params;
  const int64_t total = R->level_offsets.back();
  DBuf<T> g_coef(total, s), g_cum(total, s), g_sums(3 * tp.G.count, s);
  if (g_coef_in)
    PSR_CUDA(cudaMemcpyAsync(g_coef.p, g_coef_in, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
  else
    g_coef.zero();
  if (g_cum_in)
    PSR_CUDA(cudaMemcpyAsync(g_cum.p, g_cum_in, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
  else
    g_cum.zero();
  g_sums.zero();
  HashView hv = R->hash.view();
  EventMarks& marks = R->bw_marks;
  if (marks.pending()) marks.collect(R->backward_ms, kBwSlots);
  marks.begin(s);
  field_backward<T>(R->keys.p, R->level_offsets, hv, reinterpret_cast<const T*>(R->coefficients.p),
                    reinterpret_cast<const T*>(R->cumulative.p), prm.depth, tp.G.sums.p, tp.G.weights.p, tp.G.count,
                    g_iso, g_coef.p, g_cum.p, g_sums.p, s);
  marks.mark(kBwField, s);
  std::vector<DBuf<T>> g_agg(prm.depth + 1);
  for (int d = 0; d <= prm.depth; ++d) {
    g_agg[d].alloc(4 * tp.D.agg_count[d], s);
    g_agg[d].zero();
  }
  DBuf<T> g_avg(3, s), g_nvals(4 * tp.N.count, s);
  g_avg.zero();
  g_nvals.zero();
  solve_backward<T>(tp.solve.get(), tp.tree, tp.D, tp.N, R->level_offsets, R->keys.p, R->hash, prm, g_coef.p, g_agg,
                    g_avg.p, g_nvals.p, s, &marks);
  samples_backward<T>(tp.G, tp.D, tp.N, prm.depth, prm.kernel_depth, prm.base_depth, prm.samples_per_node, prm.scale,
                      g_agg, g_avg.p, g_nvals.p, g_sums.p, g_norm, pos, nrm, n, g_pos, g_nrm, s);
  marks.mark(kBwSamples, s);
}


}  // namespace

namespace {
template <class T>
__global__ void ltr_to_normalization_kernel(const double* g_ltr, T* g_norm) {
  if (threadIdx.x != 0) return;
  // model -> cube is [[0,s,0,t0],[0,0,s,t1],[s,0,0,t2]] (transforms.py:55-70)
  g_norm[0] = g_norm[0] + T(g_ltr[1] + g_ltr[5] + g_ltr[6]);
  for (int a = 0; a < 3; ++a) g_norm[1 + a] = g_norm[1 + a] + T(g_ltr[9 + a]);
}

template <class T>
static void evaluate_backward_typed(const psr_result* R, const T* q, int64_t nq, const T* gv, const T* gg, T* gc,
                                    T* gcum, T* gq, T* gnorm, cudaStream_t s) {
  DBuf<T> lt(12, s);
  T h[12];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) h[3 * r + c] = T(R->host_transforms[16 + 4 * r + c]);
    h[9 + r] = T(R->host_transforms[16 + 4 * r + 3]);
  }
  PSR_CUDA(cudaMemcpyAsync(lt.p, h, sizeof(h), cudaMemcpyHostToDevice, s));
  DBuf<double> ltr(12, s);
  ltr.zero();
  evaluate_backward<T>(R->hash.view(), reinterpret_cast<const T*>(R->coefficients.p),
                       reinterpret_cast<const T*>(R->cumulative.p), q, nq, lt.p, lt.p + 9, R->depth, gv, gg, gc, gcum,
                       gq, gnorm ? ltr.p : nullptr, s);
  if (gnorm) {
    ltr_to_normalization_kernel<T><<<1, 32, 0, s>>>(ltr.p, gnorm);
    PSR_LAUNCH_CHECK();
  }
  PSR_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

int psr_reconstruct(const void* positions, const void* normals, int64_t n, int32_t dtype, const psr_params* params,
                    void* stream, psr_result** out) {
  try {
    if (!out) throw Error(PSR_EINVAL, "out must not be NULL");
    *out = nullptr;
    validate(params);
    if (dtype != PSR_FLOAT32 && dtype != PSR_FLOAT64)
      throw Error(PSR_EINVAL, "Reconstruction requires matching float32/float64 3D vectors on the same CUDA device");
    if (!positions || !normals || n <= 0) throw Error(PSR_EINVAL, "points and normals must have equal nonempty 1D shapes");
    if (n > int64_t(INT32_MAX) / 54) throw Error(PSR_EINVAL, "too many points for 32-bit record indices");
    cudaStream_t s = (cudaStream_t)stream;
    tune_pool();
    Params prm{params->depth, params->full_depth, params->base_depth, params->solve_depth, params->kernel_depth,
               params->samples_per_node, params->scale, params->point_weight, params->cg_accuracy,
               params->exact_interpolation, params->iters, params->base_v_cycles, params->precision};
    prm.differentiable = params->differentiable != 0;
    std::unique_ptr<psr_result> R(new psr_result());
    R->sink.on = params->keep_stages != 0;
    R->depth = prm.depth;
    R->params = prm;
    if (prm.precision == PSR_PRECISION_MIXED || dtype == PSR_FLOAT64) {
      R->dtype = PSR_FLOAT64;
      if (dtype == PSR_FLOAT32) {
        DBuf<double> p64(3 * n, s), n64(3 * n, s);
        upcast_kernel<<<blocks_for(3 * n), kThreads, 0, s>>>((const float*)positions, 3 * n, p64.p);
        PSR_LAUNCH_CHECK();
        upcast_kernel<<<blocks_for(3 * n), kThreads, 0, s>>>((const float*)normals, 3 * n, n64.p);
        PSR_LAUNCH_CHECK();
        run<double>(p64.p, n64.p, n, prm, s, R.get());
      } else {
        run<double>((const double*)positions, (const double*)normals, n, prm, s, R.get());
      }
    } else {
      R->dtype = PSR_FLOAT32;
      run<float>((const float*)positions, (const float*)normals, n, prm, s, R.get());
    }
    *out = R.release();
    return PSR_OK;
  } catch (const Error& e) {
    return fail(e);
  } catch (const std::exception& e) {
    g_error = e.what();
    return PSR_ECUDA;
  }
}

int psr_result_info(const psr_result* R, psr_info* info) {
  if (!R || !info) {
    g_error = "NULL argument";
    return PSR_EINVAL;
  }
  std::memset(info, 0, sizeof(*info));
  info->dtype = R->dtype;
  info->depth = R->depth;
  info->total = R->level_offsets.back();
  info->groups = R->groups;
  for (int d = 0; d <= R->depth && d < 16; ++d) {
    info->basis_counts[d] = R->level_offsets[d + 1] - R->level_offsets[d];
    info->support_counts[d] = R->support_count[d];
  }
  info->iso_value = R->iso;
  for (int i = 0; i < 16; ++i) {
    info->cube_to_model[i] = R->host_transforms[i];
    info->model_to_cube[i] = R->host_transforms[16 + i];
  }
  for (int i = 0; i < 8; ++i) info->stage_ms[i] = R->stage_ms[i];
  info->relax_ms = R->stats.relax_ms;
  info->relax_row_visits = R->stats.row_visits;
  info->relax_launches = R->stats.launches;
  info->relax_finest_ms = R->stats.level_relax_ms.empty() ? 0.0 : R->stats.level_relax_ms.back();
  info->relax_finest_row_visits = R->stats.finest_row_visits;
  for (int i = 0; i < 5; ++i) info->normalization[i] = R->normalization[i];
  if (R->bw_marks.pending()) R->bw_marks.collect(R->backward_ms, kBwSlots);
  for (int i = 0; i < 8; ++i) info->backward_ms[i] = R->backward_ms[i];
  return PSR_OK;
}

int psr_result_arrays(const psr_result* R, psr_arrays* a) {
  if (!R || !a) {
    g_error = "NULL argument";
    return PSR_EINVAL;
  }
  std::memset(a, 0, sizeof(*a));
  a->keys = R->keys.p;
  a->coefficients = R->coefficients.p;
  a->cumulative = R->cumulative.p;
  a->level_offsets = R->level_offsets.data();
  for (int d = 0; d <= R->depth && d < 16; ++d) a->support_keys[d] = R->support[d].p;
  return PSR_OK;
}

int psr_evaluate(const psr_result* R, const void* queries, int64_t nq, void* values, void* gradients, int32_t* valid,
                 void* stream) {
  try {
    if (!R) throw Error(PSR_EINVAL, "result must not be NULL");
    if (nq < 0 || (nq > 0 && (!queries || !values))) throw Error(PSR_EINVAL, "queries and values are required");
    cudaStream_t s = (cudaStream_t)stream;
    if (nq == 0) return PSR_OK;
    if (R->dtype == PSR_FLOAT64) {
      DBuf<double> lt(12, s);
      double h[12];
      for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) h[3 * r + c] = R->host_transforms[16 + 4 * r + c];
        h[9 + r] = R->host_transforms[16 + 4 * r + 3];
      }
      PSR_CUDA(cudaMemcpyAsync(lt.p, h, sizeof(h), cudaMemcpyHostToDevice, s));
      evaluate_queries<double>(R->keys.p, R->hash.view(), (const double*)R->coefficients.p,
                               (const double*)R->cumulative.p, (const double*)queries, nq, lt.p, lt.p + 9, R->depth,
                               (double*)values, (double*)gradients, valid, false, nullptr, nullptr, s);
    } else {
      DBuf<float> lt(12, s);
      float h[12];
      for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) h[3 * r + c] = float(R->host_transforms[16 + 4 * r + c]);
        h[9 + r] = float(R->host_transforms[16 + 4 * r + 3]);
      }
      PSR_CUDA(cudaMemcpyAsync(lt.p, h, sizeof(h), cudaMemcpyHostToDevice, s));
      evaluate_queries<float>(R->keys.p, R->hash.view(), (const float*)R->coefficients.p, (const float*)R->cumulative.p,
                              (const float*)queries, nq, lt.p, lt.p + 9, R->depth, (float*)values, (float*)gradients,
                              valid, false, nullptr, nullptr, s);
    }
    PSR_CUDA(cudaStreamSynchronize(s));
    return PSR_OK;
  } catch (const Error& e) {
    return fail(e);
  }
}

int psr_backward(psr_result* R, const void* positions, const void* normals, int64_t n, int32_t dtype,
                 const void* g_coefficients, const void* g_cumulative, const void* g_iso, const void* g_normalization,
                 void* g_positions, void* g_normals, void* stream) {
  try {
    if (!R) throw Error(PSR_EINVAL, "result must not be NULL");
    if (!R->tape) throw Error(PSR_EINVAL, "the reconstruction was not made differentiable (params.differentiable)");
    if (dtype != PSR_FLOAT32 && dtype != PSR_FLOAT64) throw Error(PSR_EINVAL, "dtype must be float32 or float64");
    if (!positions || !normals || !g_positions || !g_normals) throw Error(PSR_EINVAL, "inputs and outputs are required");
    cudaStream_t s = (cudaStream_t)stream;
    if (R->dtype == PSR_FLOAT64) {
      const int64_t want = static_cast<Tape<double>*>(R->tape.get())->n_input;
      if (n != want) throw Error(PSR_EINVAL, "n differs from the forward's point count");
      if (dtype == PSR_FLOAT64) {
        backward<double>(R, (const double*)positions, (const double*)normals, n, (const double*)g_coefficients,
                         (const double*)g_cumulative, (const double*)g_iso, (const double*)g_normalization, (double*)g_positions,
                         (double*)g_normals, s);
      } else {
        DBuf<double> p64(3 * n, s), n64(3 * n, s), gp(3 * n, s), gn(3 * n, s);
        cast_kernel_t<double><<<blocks_for(3 * n), kThreads, 0, s>>>(positions, 0, 3 * n, p64.p);
        PSR_LAUNCH_CHECK();
        cast_kernel_t<double><<<blocks_for(3 * n), kThreads, 0, s>>>(normals, 0, 3 * n, n64.p);
        PSR_LAUNCH_CHECK();
        backward<double>(R, p64.p, n64.p, n, (const double*)g_coefficients, (const double*)g_cumulative, (const double*)g_iso,
                         (const double*)g_normalization, gp.p, gn.p, s);
        cast_kernel_t<float><<<blocks_for(3 * n), kThreads, 0, s>>>(gp.p, 1, 3 * n, (float*)g_positions);
        PSR_LAUNCH_CHECK();
        cast_kernel_t<float><<<blocks_for(3 * n), kThreads, 0, s>>>(gn.p, 1, 3 * n, (float*)g_normals);
        PSR_LAUNCH_CHECK();
      }
    } else {
      if (dtype != PSR_FLOAT32) throw Error(PSR_EINVAL, "inputs must have the forward's dtype");
      const int64_t want = static_cast<Tape<float>*>(R->tape.get())->n_input;
      if (n != want) throw Error(PSR_EINVAL, "n differs from the forward's point count");
      backward<float>(R, (const float*)positions, (const float*)normals, n, (const float*)g_coefficients,
                      (const float*)g_cumulative, (const float*)g_iso, (const float*)g_normalization, (float*)g_positions,
                      (float*)g_normals, s);
    }
    return PSR_OK;
  } catch (const Error& e) {
    return fail(e);
  }
}

int psr_evaluate_backward(const psr_result* R, const void* queries, int64_t nq, const void* g_values,
                          const void* g_gradients, void* g_coefficients, void* g_cumulative, void* g_queries,
                          void* g_normalization, void* stream) {
  try {
    if (!R) throw Error(PSR_EINVAL, "result must not be NULL");
    if (nq < 0 || (nq > 0 && !queries)) throw Error(PSR_EINVAL, "queries are required");
    if (!g_coefficients || !g_cumulative) throw Error(PSR_EINVAL, "coefficient adjoints are required");
    if (nq == 0) return PSR_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (R->dtype == PSR_FLOAT64)
      evaluate_backward_typed<double>(R, (const double*)queries, nq, (const double*)g_values,
                                      (const double*)g_gradients, (double*)g_coefficients, (double*)g_cumulative,
                                      (double*)g_queries, (double*)g_normalization, s);
    else
      evaluate_backward_typed<float>(R, (const float*)queries, nq, (const float*)g_values, (const float*)g_gradients,
                                     (float*)g_coefficients, (float*)g_cumulative, (float*)g_queries,
                                     (float*)g_normalization, s);
    return PSR_OK;
  } catch (const Error& e) {
    return fail(e);
  }
}

int psr_device_field(const psr_result* R, psr_field_handle* h) {
  if (!R || !h) {
    g_error = "NULL argument";
    return PSR_EINVAL;
  }
  std::memset(h, 0, sizeof(*h));
  h->keys = R->keys.p;
  h->coefficients = R->coefficients.p;
  h->cumulative = R->cumulative.p;
  h->count = R->level_offsets.back();
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) h->linear[3 * r + c] = R->host_transforms[16 + 4 * r + c];
    h->translation[r] = R->host_transforms[16 + 4 * r + 3];
  }
  h->depth = R->depth;
  h->dtype = R->dtype;
  h->iso_value = R->iso;
  const HashView hv = R->hash.view();
  h->hash_slots = hv.slots;
  h->hash_mask = hv.mask;
  return PSR_OK;
}

int psr_free(psr_result* R) {
  if (!R) return PSR_OK;
  cudaDeviceSynchronize();
  delete R;
  return PSR_OK;
}

namespace {
// CSR rows (columns ascending) -> 28-slot rows where slot k holds the k-th lexicographic
// neighbour; error 1: an entry is not within the 27-neighbourhood or columns not ascending.
__global__ void csr_to_slots_kernel(const int64_t* keys, const int32_t* offsets, const int32_t* columns,
                                    const char* values, int elem, int64_t n, int32_t* cols, char* vals, int* error) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  for (int k = 0; k < 28; ++k) {
    cols[i * 28 + k] = -1;
    for (int q = 0; q < elem; ++q) vals[(i * 28 + k) * elem + q] = 0;
  }
  int b = offsets[i], e = offsets[i + 1];
  if (e < b || e - b > 27) {
    atomicExch(error, 1);
    return;
  }
  int c[3];
  key_coords(keys[i], c);
  int last = -1;
  for (int j = b; j < e; ++j) {
    int col = columns[j];
    if (col < 0 || col >= n) {
      atomicExch(error, 3);
      return;
    }
    int q[3];
    key_coords(keys[col], q);
    int dx = q[0] - c[0], dy = q[1] - c[1], dz = q[2] - c[2];
    if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1 || (keys[col] >> 48) != (keys[i] >> 48)) {
      atomicExch(error, 1);
      return;
    }
    int k = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
    if (k <= last) {
      atomicExch(error, 1);
      return;
    }
    last = k;
    cols[i * 28 + k] = col;
    for (int q2 = 0; q2 < elem; ++q2) vals[(i * 28 + k) * elem + q2] = values[int64_t(j) * elem + q2];
  }
}

__global__ void sliced_group_kernel(const int64_t* keys, int64_t n, int depth, uint32_t* groups, int32_t* ids,
                                    int* error) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  if (c[0] > (1 << depth) || c[1] > (1 << depth) || c[2] > (1 << depth) || int(keys[i] >> 48) != depth)
    atomicExch(error, 2);
  if (groups) groups[i] = uint32_t((c[0] & 1) + 2 * (c[1] & 1) + 4 * min(c[2], 1 << depth));
  if (ids) ids[i] = int32_t(i);
}

__global__ void offsets_kernel(const uint32_t* sorted, int64_t n, int count, int32_t* off) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g > count) return;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (sorted[mid] < uint32_t(g))
      lo = mid + 1;
    else
      hi = mid;
  }
  off[g] = int32_t(lo);
}
}  // namespace

int psr_relax_sliced(int32_t dtype, const int64_t* keys, int64_t n, int32_t depth, const int32_t* offsets,
                     const int32_t* columns, const void* values, const void* b, void* x, int32_t iters, void* stream) {
  try {
    if (dtype != PSR_FLOAT32 && dtype != PSR_FLOAT64) throw Error(PSR_EINVAL, "dtype must be float32 or float64");
    if (depth < 0 || depth > 15 || iters < 0 || n < 0) throw Error(PSR_EINVAL, "invalid depth, iters or size");
    if (n == 0 || iters == 0) return PSR_OK;
    if (!keys || !offsets || !columns || !values || !b || !x) throw Error(PSR_EINVAL, "NULL array");
    cudaStream_t s = (cudaStream_t)stream;
    int elem = dtype == PSR_FLOAT64 ? 8 : 4;
    DBuf<int32_t> cols(28 * n, s);
    DBuf<char> vals(28 * n * elem, s);
    DBuf<int> error(1, s);
    error.zero();
    sliced_group_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, n, depth, nullptr, nullptr, error.p);
    PSR_LAUNCH_CHECK();
    csr_to_slots_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, offsets, columns, (const char*)values, elem, n,
                                                          cols.p, vals.p, error.p);
    PSR_LAUNCH_CHECK();
    int err = read_scalar(error.p, s);
    if (err == 1) throw Error(PSR_EINVAL, "every row needs at most 27 entries, ascending, within its 27-neighbourhood");
    if (err == 2) throw Error(PSR_EINVAL, "keys must be basis keys of `depth`");
    if (err == 3) throw Error(PSR_EINVAL, "column index out of range");
    if (dtype == PSR_FLOAT64)
      relax_sliced_strips<double, double>(keys, n, depth, cols.p, (const double*)vals.p, (const double*)b, (double*)x,
                                          iters, s, nullptr);
    else
      relax_sliced_strips<float, float>(keys, n, depth, cols.p, (const float*)vals.p, (const float*)b, (float*)x,
                                        iters, s, nullptr);
    PSR_CUDA(cudaStreamSynchronize(s));
    return PSR_OK;
  } catch (const Error& e) {
    return fail(e);
  }
}

int psr_isovalue(int32_t dtype, const void* values, const void* weights, int64_t n, void* out, void* stream) {
  try {
    if (dtype != PSR_FLOAT32 && dtype != PSR_FLOAT64) throw Error(PSR_EINVAL, "dtype must be float32 or float64");
    if (n <= 0 || !values || !weights || !out) throw Error(PSR_EINVAL, "nonempty values and weights are required");
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PSR_FLOAT64)
      isovalue<double>((const double*)values, (const double*)weights, n, (double*)out, s);
    else
      isovalue<float>((const float*)values, (const float*)weights, n, (float*)out, s);
    PSR_CUDA(cudaStreamSynchronize(s));
    return PSR_OK;
  } catch (const Error& e) {
    return fail(e);
  }
}

int psr_result_stage(const psr_result* R, const char* name, const void** data, int64_t* count, int32_t* elem) {
  if (!R || !name || !data || !count || !elem) {
    g_error = "NULL argument";
    return PSR_EINVAL;
  }
  auto it = R->sink.entries.find(name);
  if (it == R->sink.entries.end()) {
    *data = nullptr;
    *count = -1;
    *elem = 0;
    return PSR_OK;
  }
  *data = it->second.data.p;
  *count = it->second.count;
  *elem = it->second.elem;
  return PSR_OK;
}

int psr_kernel_clocks(psr_kernel_clock* out, int32_t capacity, int32_t* count) {
  if (!count || (capacity > 0 && !out)) return PSR_EINVAL;
  try {
    using namespace psr::clocks;
    std::lock_guard<std::mutex> lock(g_clock_mutex);
    for (PendingClock& c : g_clock_pending) {
      float ms = 0;
      PSR_CUDA(cudaEventSynchronize(c.b));
      PSR_CUDA(cudaEventElapsedTime(&ms, c.a, c.b));
      ClockTotals& t = g_clock_totals[c.kind];
      t.launches += 1;
      t.ms += ms;
      t.bytes += c.bytes;
      t.units += c.units;
      cudaEventDestroy(c.a);
      cudaEventDestroy(c.b);
    }
    g_clock_pending.clear();
    int n = 0;
    for (int k = 0; k < kClkKinds; ++k) {
      const ClockTotals& t = g_clock_totals[k];
      if (!t.launches) continue;
      if (n < capacity) out[n] = psr_kernel_clock{kClockNames[k], kClockUnits[k], t.launches, t.ms, t.bytes, t.units};
      ++n;
      g_clock_totals[k] = ClockTotals();
    }
    *count = n;
    return PSR_OK;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return PSR_ECUDA;
  }
}

int psr_kernel_launches(int64_t* count) {
  if (!count) return PSR_EINVAL;
  *count = int64_t(g_kernel_launches.load());
  return PSR_OK;
}

int psr_last_error(char* buffer, size_t length) {
  if (!buffer || !length) return PSR_EINVAL;
  std::strncpy(buffer, g_error.c_str(), length - 1);
  buffer[length - 1] = 0;
  return PSR_OK;
}

}  // extern "C"
