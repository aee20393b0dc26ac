// CPU oracle for the screened-Poisson reconstruction path.  TEST INFRASTRUCTURE ONLY:
// only tests, the smoke check and the bench's CPU-baseline leg may load it, as the
// checker.  The product path (warp_psr_b200 + libpsr_b200.so) never links or calls it.
//
// A plain C++17 restatement of warp-psr's degree-1, Neumann, confidence-off PSR/SPSR
// forward algorithm (which itself restates PoissonRecon 262b0f5), templated on the
// input precision.  Every function cites the reference file:line it follows.  Built with
// -ffp-contract=off, mirroring the reference's `fuse_fp: False` module option, so every
// scalar operation rounds exactly where the reference's does.
//
// Deliberate restatements (the reference's result is the same function, the floating
// point summation order differs and is documented beside each):
//  * base-level and small-level operators (Warp-FEM quadrature in solver.py:365-398) are
//    assembled with the analytic stencils (stiffness.py, screening_stencils.py);
//  * the float32 base-depth-0 "ordered" normal loads (ordered_normal_loads.py:263) use the
//    float64 stencil loads (normal_loads.py:114-190) like every other profile;
//  * Galerkin products (warp.sparse.bsr_mm) and root CG dot products use a fixed
//    sequential order;
//  * the normal average (normals.py:132-163) and the isovalue (reconstruction.py:77-93)
//    use the fixed blocked orders that the CUDA kernels use (see `blocked_*` below).
#include <algorithm>
#include <array>
#include <type_traits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int64_t kInvalid = std::numeric_limits<int64_t>::max();

struct Params {
  int depth, full_depth, base_depth, solve_depth, kernel_depth;
  double samples_per_node, scale, point_weight, cg_accuracy;
  int exact, iters, base_v_cycles;
};

// ---------------------------------------------------------------- keys (field.py:13-32, tree.py:16-28)
inline int64_t basis_key(int d, int x, int y, int z) {
  return (int64_t(d) << 48) | (int64_t(x) << 32) | (int64_t(y) << 16) | int64_t(z);
}
inline void coords(int64_t k, int c[3]) {
  c[0] = int((k >> 32) & 65535);
  c[1] = int((k >> 16) & 65535);
  c[2] = int(k & 65535);
}
inline int key_depth(int64_t k) { return int(k >> 48); }
inline int64_t tree_key(int x, int y, int z) {
  return (int64_t(x + 524288) << 40) | (int64_t(y + 524288) << 20) | int64_t(z + 524288);
}
inline void tree_coords(int64_t k, int c[3]) {
  c[0] = int((k >> 40) & 1048575) - 524288;
  c[1] = int((k >> 20) & 1048575) - 524288;
  c[2] = int(k & 1048575) - 524288;
}
// tree.py:26-28 floor(c / 2) for signed coordinates
inline int parent_coord(int c) { return c >> 1; }

inline int64_t find_key(const std::vector<int64_t>& keys, int64_t key) {
  auto it = std::lower_bound(keys.begin(), keys.end(), key);
  if (it != keys.end() && *it == key) return int64_t(it - keys.begin());
  return -1;
}

// keyed.py:23-30
inline int64_t morton(const int c[3], int depth) {
  int64_t m = 0;
  for (int bit = 0; bit < depth; ++bit)
    for (int a = 0; a < 3; ++a) m |= int64_t((c[a] >> bit) & 1) << (3 * bit + a);
  return m;
}

// Stable order of `keys` (a stable radix sort in the reference, keyed.py:102-108,122-124).
std::vector<int64_t> stable_order(const std::vector<int64_t>& keys) {
  std::vector<int64_t> ids(keys.size());
  std::iota(ids.begin(), ids.end(), 0);
  std::stable_sort(ids.begin(), ids.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
  return ids;
}

// keyed.py:66-94,111-142 — sort records by key (stable), sum each key's values in record order.
template <class T>
void reduce_records(const std::vector<int64_t>& keys, const std::vector<T>& values /* 4 per record */,
                    std::vector<int64_t>& out_keys, std::vector<T>& out_values) {
  auto ids = stable_order(keys);
  out_keys.clear();
  out_values.clear();
  size_t n = ids.size();
  size_t i = 0;
  while (i < n) {
    int64_t k = keys[ids[i]];
    if (k == kInvalid) break;
    T acc[4] = {T(0), T(0), T(0), T(0)};
    size_t j = i;
    while (j < n && keys[ids[j]] == k) {
      for (int a = 0; a < 4; ++a) acc[a] = acc[a] + values[4 * ids[j] + a];
      ++j;
    }
    out_keys.push_back(k);
    for (int a = 0; a < 4; ++a) out_values.push_back(acc[a]);
    i = j;
  }
}

std::vector<int64_t> unique_sorted(std::vector<int64_t> keys) {
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  while (!keys.empty() && keys.back() == kInvalid) keys.pop_back();
  return keys;
}

// density.py:14-22 degree-2 B-spline values, float64
inline void quadratic(double x, double b[3]) {
  double one = 1.0, half = 0.5;
  b[0] = (one - x) * (one - x) * half;
  b[1] = ((one - x) * (x + one) + x * (2.0 - x)) * half;
  b[2] = x * x * half;
}

template <class T>
inline int ceil_cell(T p, int n) {  // max(0, int(ceil(p*n)) - 1)
  int c = int(std::ceil(p * T(n))) - 1;
  return c < 0 ? 0 : c;
}

// ---------------------------------------------------------------- stage data
template <class T>
struct Samples {
  T transform[5];
  std::vector<int64_t> keys;                // unique leaf keys (sorted)
  std::vector<T> sums, normal_sums;         // 3 per group
  std::vector<T> weights;                   // per group
  std::vector<int32_t> first;               // first input index per group
  std::vector<T> q;                         // transformed positions (3 per input)
};

template <class T>
struct Density {
  std::vector<std::vector<int64_t>> agg_keys;  // per depth
  std::vector<std::vector<T>> agg_values;      // 4 per record
  std::vector<std::vector<int64_t>> level_keys;
  std::vector<std::vector<T>> level_values;    // 4 per record (density in [0])
  std::vector<T> dw;                           // 2 per group (raw depth, weight)
  T scale;
};

template <class T>
struct Normals {
  std::vector<int64_t> keys;  // all records, sorted
  std::vector<T> values;      // 4 per record
  std::vector<size_t> offsets;  // per depth, size max+2
  T average[3];
};

struct Tree {
  std::vector<std::vector<int64_t>> support;  // signed tree keys per depth
  std::vector<std::vector<int64_t>> basis;    // field keys per depth
};

template <class T>
struct Csr {
  int64_t rows = 0, cols = 0;
  std::vector<int32_t> offsets, columns;
  std::vector<T> values;
};

struct StageArray {
  std::vector<char> bytes;
  int64_t count = 0;
  int elem = 0;
};

struct ResultBase {
  int dtype = 0;
  int depth = 0;
  std::vector<std::vector<int64_t>> basis, support;
  std::vector<int64_t> all_keys;
  std::vector<int64_t> level_offsets;
  std::map<std::string, StageArray> stages;
  std::string error;
  virtual ~ResultBase() {}
};

template <class T>
struct Result : ResultBase {
  std::vector<T> coefficients, cumulative;
  T iso = T(0);
  T transforms[2][16];
};

template <class V>
void put_stage(ResultBase& r, const std::string& name, const std::vector<V>& v) {
  StageArray s;
  s.elem = sizeof(V);
  s.count = int64_t(v.size());
  s.bytes.resize(v.size() * sizeof(V));
  if (!v.empty()) std::memcpy(s.bytes.data(), v.data(), s.bytes.size());
  r.stages[name] = std::move(s);
}

// ---------------------------------------------------------------- A1 samples (samples.py:34-188,219-311)
template <class T>
Samples<T> prepare_samples(const T* pos, const T* nrm, int64_t count, int depth, double scale_arg) {
  Samples<T> s;
  T lo[3] = {std::numeric_limits<T>::infinity(), std::numeric_limits<T>::infinity(),
             std::numeric_limits<T>::infinity()};
  T hi[3] = {-lo[0], -lo[1], -lo[2]};
  int64_t bad = 0;
  for (int64_t i = 0; i < count; ++i) {  // samples.py:40-52
    const T* p = pos + 3 * i;
    if (std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2])) {
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], p[a]);
        hi[a] = std::max(hi[a], p[a]);
      }
    } else {
      ++bad;
    }
  }
  // samples.py:54-88
  T scale = T(scale_arg);
  T width = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2])) * scale;
  if (bad || !std::isfinite(width) || width <= T(0))
    throw std::runtime_error("Nonfinite positions or degenerate/overflowing bounding cube");
  T inv = T(1.0 / double(width));
  s.transform[0] = inv;
  T determinant = inv * (inv * inv);
  s.transform[4] = inv * inv / determinant * T(std::pow(double(determinant), 1.0 / 3.0));
  for (int a = 0; a < 3; ++a) {
    int axis = (a + 1) % 3;
    T origin = (hi[axis] + lo[axis]) / T(2.0) - width / T(2.0);
    s.transform[a + 1] = -origin * inv;
  }
  // samples.py:90-134
  std::vector<int64_t> keys(count, kInvalid);
  std::vector<T> un(3 * count, T(0));
  s.q.resize(3 * count);
  for (int64_t i = 0; i < count; ++i) {
    const T* p = pos + 3 * i;
    const T* n = nrm + 3 * i;
    T q[3] = {p[1] * inv + s.transform[1], p[2] * inv + s.transform[2], p[0] * inv + s.transform[3]};
    T m[3] = {n[1] * s.transform[4], n[2] * s.transform[4], n[0] * s.transform[4]};
    T length2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
    for (int a = 0; a < 3; ++a) s.q[3 * i + a] = q[a];
    if (length2 > T(0) && std::isfinite(length2) && std::min(q[0], std::min(q[1], q[2])) >= T(0) &&
        std::max(q[0], std::max(q[1], q[2])) <= T(1)) {
      T len = std::sqrt(length2);
      for (int a = 0; a < 3; ++a) un[3 * i + a] = m[a] / len;
      int res = 1 << depth;
      keys[i] = basis_key(depth, ceil_cell(q[0], res), ceil_cell(q[1], res), ceil_cell(q[2], res));
    }
  }
  // samples.py:136-188 (stable sort, group sums in input order)
  auto order = stable_order(keys);
  size_t i = 0;
  while (i < order.size()) {
    int64_t k = keys[order[i]];
    if (k == kInvalid) break;
    T ps[3] = {T(0), T(0), T(0)}, ns[3] = {T(0), T(0), T(0)}, w = T(0);
    size_t j = i;
    while (j < order.size() && keys[order[j]] == k) {
      for (int a = 0; a < 3; ++a) {
        ps[a] = ps[a] + s.q[3 * order[j] + a];
        ns[a] = ns[a] + un[3 * order[j] + a];
      }
      w = w + T(1.0);
      ++j;
    }
    s.keys.push_back(k);
    for (int a = 0; a < 3; ++a) {
      s.sums.push_back(ps[a]);
      s.normal_sums.push_back(ns[a]);
    }
    s.weights.push_back(w);
    s.first.push_back(int32_t(order[i]));
    i = j;
  }
  if (s.keys.empty()) throw std::runtime_error("No accepted samples with finite nonzero normals");
  return s;
}

// ---------------------------------------------------------------- A2 density (density.py:25-279)
template <class T>
T density_scale() {  // density.py:37-50
  T total = T(0);
  T dx = T(0.1);
  for (int x = 0; x < 10; ++x) {
    T p = dx / T(2.0) + dx * T(x);
    double b[3];
    quadratic(double(p), b);
    T sc = T(1.0 / (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]));
    for (int y = 0; y < 100; ++y) total = total + sc;
  }
  return total / T(1000.0);
}

template <class T>
std::vector<int64_t> morton_order(const std::vector<int64_t>& keys, int d) {
  std::vector<int64_t> codes(keys.size());
  for (size_t i = 0; i < keys.size(); ++i) {
    int c[3];
    coords(keys[i], c);
    codes[i] = morton(c, d);
  }
  return stable_order(codes);
}

template <class T>
T density_value(const std::vector<int64_t>& keys, const std::vector<T>& values, const T p[3], int depth) {
  int n = 1 << depth;  // density.py:108-136
  int c[3] = {ceil_cell(p[0], n), ceil_cell(p[1], n), ceil_cell(p[2], n)};
  T h = T(1.0) / T(n);
  double b[3][3];
  for (int a = 0; a < 3; ++a) quadratic(double((p[a] - T(c[a]) * h) / h), b[a]);
  T value = T(0);
  for (int k = 0; k < 27; ++k) {
    int x = k / 9, y = k / 3 % 3, z = k % 3;
    int t[3] = {c[0] + x - 1, c[1] + y - 1, c[2] + z - 1};
    if (std::min(t[0], std::min(t[1], t[2])) >= 0 && std::max(t[0], std::max(t[1], t[2])) < n) {
      int64_t idx = find_key(keys, basis_key(depth, t[0], t[1], t[2]));
      if (idx >= 0) value = value + T(b[0][x] * b[1][y] * b[2][z] * double(values[4 * idx]));
    }
  }
  return value;
}

template <class T>
Density<T> build_density(const Samples<T>& s, int depth, int kernel_depth, double spn) {
  Density<T> D;
  size_t count = s.keys.size();
  D.agg_keys.resize(depth + 1);
  D.agg_values.resize(depth + 1);
  D.agg_keys[depth] = s.keys;
  D.agg_values[depth].resize(4 * count);
  for (size_t i = 0; i < count; ++i) {  // density.py:52-57
    for (int a = 0; a < 3; ++a) D.agg_values[depth][4 * i + a] = s.sums[3 * i + a];
    D.agg_values[depth][4 * i + 3] = s.weights[i];
  }
  for (int d = depth; d > 0; --d) {  // density.py:228-240
    const auto& keys = D.agg_keys[d];
    const auto& vals = D.agg_values[d];
    auto order = morton_order<T>(keys, d);
    std::vector<int64_t> pk(keys.size());
    std::vector<T> pv(vals.size());
    for (size_t i = 0; i < keys.size(); ++i) {
      int c[3];
      coords(keys[order[i]], c);
      pk[i] = basis_key(d - 1, c[0] / 2, c[1] / 2, c[2] / 2);
      for (int a = 0; a < 4; ++a) pv[4 * i + a] = vals[4 * order[i] + a];
    }
    reduce_records(pk, pv, D.agg_keys[d - 1], D.agg_values[d - 1]);
  }
  D.scale = density_scale<T>();
  D.level_keys.resize(kernel_depth + 1);
  D.level_values.resize(kernel_depth + 1);
  std::vector<T> dens(count * (kernel_depth + 1));
  for (int d = 0; d <= kernel_depth; ++d) {  // density.py:74-107,245-271
    const auto& keys = D.agg_keys[d];
    const auto& vals = D.agg_values[d];
    auto order = morton_order<T>(keys, d);
    size_t m = keys.size();
    std::vector<int64_t> rk(27 * m, kInvalid);
    std::vector<T> rv(4 * 27 * m, T(0));
    int n = 1 << d;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(m); ++i) {
      int64_t j = order[i];
      int c[3];
      coords(keys[j], c);
      const T* v = &vals[4 * j];
      T p[3] = {v[0] / v[3], v[1] / v[3], v[2] / v[3]};
      T h = T(1.0) / T(n);
      double b[3][3];
      for (int a = 0; a < 3; ++a) quadratic(double((p[a] - T(c[a]) * h) / h), b[a]);
      T weight = v[3] * D.scale;
      for (int k = 0; k < 27; ++k) {
        int x = k / 9, y = k / 3 % 3, z = k % 3;
        int t[3] = {c[0] + x - 1, c[1] + y - 1, c[2] + z - 1};
        if (std::min(t[0], std::min(t[1], t[2])) >= 0 && std::max(t[0], std::max(t[1], t[2])) < n) {
          rk[27 * i + k] = basis_key(d, t[0], t[1], t[2]);
          rv[4 * (27 * i + k)] = T(double(weight) * b[0][x] * b[1][y] * b[2][z]);
        }
      }
    }
    reduce_records(rk, rv, D.level_keys[d], D.level_values[d]);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(count); ++i) {  // density.py:138-150
      T p[3] = {s.sums[3 * i] / s.weights[i], s.sums[3 * i + 1] / s.weights[i], s.sums[3 * i + 2] / s.weights[i]};
      dens[i * (kernel_depth + 1) + d] = density_value(D.level_keys[d], D.level_values[d], p, d);
    }
  }
  D.dw.resize(2 * count);
  T target = T(spn);
  auto real_log = [](T v) { return T(std::log(double(v))); };
  for (size_t i = 0; i < count; ++i) {  // density.py:152-182
    int d = kernel_depth;
    T density = dens[i * (kernel_depth + 1) + d];
    T raw;
    if (density >= target) {
      raw = T(double(d) + double(real_log(density / target)) / (std::log(2.0) * 2.0));
    } else {
      T fine = density;
      while (density < target && d > 0) {
        fine = density;
        d -= 1;
        density = dens[i * (kernel_depth + 1) + d];
      }
      raw = T(T(d) + real_log(density / target) / real_log(density / fine));
    }
    T h = T(1.0) / T(1 << d);
    D.dw[2 * i] = raw;
    D.dw[2 * i + 1] = h * h / density;
  }
  return D;
}

// ---------------------------------------------------------------- A3 normals (normals.py:33-245)
// Fixed blocked order shared with the CUDA kernel: blocks of 1024 contributions summed
// serially (in T, input order) inside a block, then the block totals serially.
template <class T>
void blocked_sum3(const std::vector<T>& contrib /*3 per item*/, T out[3]) {
  size_t n = contrib.size() / 3;
  T total[3] = {T(0), T(0), T(0)};
  for (size_t b = 0; b < n; b += 1024) {
    T part[3] = {T(0), T(0), T(0)};
    for (size_t j = b; j < std::min(n, b + 1024); ++j)
      if (contrib[3 * j + 2] > T(0))
        for (int a = 0; a < 3; ++a) part[a] = part[a] + contrib[3 * j + a];
    for (int a = 0; a < 3; ++a) total[a] = total[a] + part[a];
  }
  for (int a = 0; a < 3; ++a) out[a] = total[a];
}

template <class T>
Normals<T> build_normal_field(const Samples<T>& s, const Density<T>& D, int minimum, int maximum) {
  Normals<T> N;
  size_t n = s.keys.size();
  std::vector<int64_t> fk(s.first.begin(), s.first.end());
  auto order = stable_order(fk);  // normals.py:36-43,192-202
  std::vector<int64_t> rk(54 * n, kInvalid);
  std::vector<T> rv(4 * 54 * n, T(0));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(n); ++i) {  // normals.py:46-104
    int64_t src = order[i];
    T w = s.weights[src];
    T nm[3] = {s.normal_sums[3 * src] / w, s.normal_sums[3 * src + 1] / w, s.normal_sums[3 * src + 2] / w};
    T length = std::sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
    if (!(length > T(0))) continue;
    for (int a = 0; a < 3; ++a) nm[a] = nm[a] / length * w;
    T p[3] = {s.sums[3 * src] / w, s.sums[3 * src + 1] / w, s.sums[3 * src + 2] / w};
    T depth = std::min(std::max(D.dw[2 * src], T(minimum)), T(maximum));
    int top = int(std::ceil(depth));
    T dx = T(1.0) - (T(top) - depth);
    if (top <= minimum) {
      top = minimum;
      dx = T(1.0);
    }
    if (top > maximum) {
      top = maximum;
      dx = T(1.0);
    }
    int nn = 1 << top;
    T h = T(1.0) / T(nn);
    int c[3] = {ceil_cell(p[0], nn), ceil_cell(p[1], nn), ceil_cell(p[2], nn)};
    double b[3][3];
    for (int a = 0; a < 3; ++a) quadratic(double((p[a] - T(c[a]) * h) / h), b[a]);
    bool second = std::abs(1.0 - double(dx)) > 1e-06;
    for (int k = 0; k < 54; ++k) {
      if (k >= 27 && !second) break;
      T fraction = k < 27 ? dx : T(1.0) - dx;
      int q = k % 27;
      int x = q / 9, y = q / 3 % 3, z = q % 3;
      int t[3] = {c[0] + x - 1, c[1] + y - 1, c[2] + z - 1};
      if (std::min(t[0], std::min(t[1], t[2])) >= 0 && std::max(t[0], std::max(t[1], t[2])) < nn) {
        T bw = T(b[0][x] * b[1][y] * b[2][z]);
        size_t dst = 54 * i + k;
        rk[dst] = basis_key(top, t[0], t[1], t[2]);
        for (int a = 0; a < 3; ++a) rv[4 * dst + a] = nm[a] * D.dw[2 * src + 1] / (h * h * h) * fraction * bw;
      }
    }
  }
  reduce_records(rk, rv, N.keys, N.values);
  for (auto& v : N.values) v = -v;  // normals.py:106-110,219-221
  std::vector<T> contrib(3 * n, T(0));  // normals.py:132-147
  for (size_t i = 0; i < n; ++i) {
    int64_t src = order[i];
    T w = s.weights[src];
    T nm[3] = {s.normal_sums[3 * src] / w, s.normal_sums[3 * src + 1] / w, s.normal_sums[3 * src + 2] / w};
    if (std::sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]) > T(0)) {
      contrib[3 * i] = D.dw[2 * src] * w;
      contrib[3 * i + 1] = D.dw[2 * src + 1] * w;
      contrib[3 * i + 2] = w;
    }
  }
  T total[3];
  blocked_sum3(contrib, total);
  N.average[0] = N.average[1] = N.average[2] = T(0);
  if (total[2] > T(0)) {
    N.average[0] = total[0] / total[2];
    N.average[1] = total[1] / total[2];
    N.average[2] = total[2];
  }
  N.offsets.resize(maximum + 2);  // normals.py:17-31,228-232
  for (int d = 0; d <= maximum + 1; ++d)
    N.offsets[d] = size_t(std::lower_bound(N.keys.begin(), N.keys.end(), int64_t(d) << 48) - N.keys.begin());
  return N;
}

// ---------------------------------------------------------------- A4 tree (tree.py:152-201)
template <class T>
Tree build_tree(const Normals<T>& N, int depth, int full_depth, int base_depth) {
  Tree tree;
  tree.support.resize(depth + 1);
  tree.basis.resize(depth + 1);
  std::vector<int64_t> broods;  // unique sorted brood keys of the previous (finer) level
  bool have_broods = false;
  std::vector<int64_t> requests;
  bool have_requests = false;
  for (int d = depth; d >= 0; --d) {
    std::vector<int64_t> parents = have_broods ? broods : std::vector<int64_t>();
    if (d > base_depth) {
      requests = parents;
      have_requests = true;
    } else if (have_requests) {
      std::vector<int64_t> rk;
      for (int64_t r : requests) {
        int c[3];
        tree_coords(r, c);
        rk.push_back(tree_key(parent_coord(c[0]), parent_coord(c[1]), parent_coord(c[2])));
      }
      requests = unique_sorted(rk);
    } else {
      requests = parents;
      have_requests = true;
    }
    std::vector<int64_t> keys;
    for (size_t r = N.offsets[d]; r < N.offsets[d + 1]; ++r) {  // tree.py:41-50
      const T* v = &N.values[4 * r];
      T l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
      if (double(l2) > 0.0) {
        int c[3];
        coords(N.keys[r], c);
        keys.push_back(tree_key(parent_coord(c[0]), parent_coord(c[1]), parent_coord(c[2])));
      }
    }
    int cc = d <= full_depth ? (d == 0 ? 2 : (1 << (d - 1)) + 2) : 0;  // tree.py:30-34,183
    for (int i = 0; i < cc * cc * cc; ++i) keys.push_back(tree_key(i / (cc * cc) - 1, (i / cc) % cc - 1, i % cc - 1));
    int n = 1 << d;
    auto support = [&](const std::vector<int64_t>& src, int radius) {  // tree.py:52-64
      int width = 2 * radius + 1;
      for (int64_t f : src) {
        int c[3];
        tree_coords(f, c);
        int p[3] = {parent_coord(c[0]), parent_coord(c[1]), parent_coord(c[2])};
        for (int j = 0; j < width * width * width; ++j) {
          int q[3] = {p[0] + j / (width * width) - radius, p[1] + (j / width) % width - radius, p[2] + j % width - radius};
          if (std::min(q[0], std::min(q[1], q[2])) >= -n && std::max(q[0], std::max(q[1], q[2])) < n)
            keys.push_back(tree_key(q[0], q[1], q[2]));
        }
      }
    };
    support(requests, 1);
    support(parents, 0);
    broods = unique_sorted(keys);
    have_broods = true;
    std::vector<int64_t> children;  // tree.py:78-103
    children.reserve(8 * broods.size());
    for (int64_t b : broods) {
      int c[3];
      tree_coords(b, c);
      for (int k = 0; k < 8; ++k)
        children.push_back(tree_key(2 * c[0] + ((k >> 2) & 1), 2 * c[1] + ((k >> 1) & 1), 2 * c[2] + (k & 1)));
    }
    std::sort(children.begin(), children.end());
    tree.support[d] = children;
    for (int64_t k : children) {  // tree.py:105-143
      int c[3];
      tree_coords(k, c);
      if (std::min(c[0], std::min(c[1], c[2])) >= 0 && std::max(c[0], std::max(c[1], c[2])) <= n)
        tree.basis[d].push_back(basis_key(d, c[0], c[1], c[2]));
    }
  }
  return tree;
}

// ---------------------------------------------------------------- A5 operators
// stiffness.py:14-36 1-D hat mass/stiffness integrals (float64)
void hat_integrals(int depth, int index, int trial_depth, int trial_index, double out[2]) {
  int resolution = 1 << depth;
  int ratio = 1 << (depth - trial_depth);
  int first = std::max(0, std::max(index - 1, (trial_index - 1) * ratio));
  int end = std::min(resolution, std::min(index + 1, (trial_index + 1) * ratio));
  out[0] = out[1] = 0.0;
  for (int cell = first; cell < end; ++cell) {
    double t0 = double(cell - index);
    double c0 = double(cell) / double(ratio) - double(trial_index);
    double ts = cell >= index ? -1.0 : 1.0;
    double cs = 1.0 / double(ratio);
    if (cell >= trial_index * ratio) cs = -cs;
    double tv = 1.0 - std::abs(t0);
    double cv = 1.0 - std::abs(c0);
    out[0] += (tv * cv + (tv * cs + ts * cv) * 0.5 + ts * cs / 3.0) / double(resolution);
    out[1] += ts * cs * double(resolution);
  }
}

// stiffness.py:38-108 — CSR rows in lexicographic neighbour order, float64 values.
Csr<double> level_stiffness(const std::vector<int64_t>& rows, const std::vector<int64_t>& cols, int depth,
                            int trial_depth) {
  Csr<double> A;
  A.rows = int64_t(rows.size());
  A.cols = int64_t(cols.size());
  int shift = depth - trial_depth;
  int res = 1 << depth;
  std::vector<double> table(size_t(res + 1) * 3 * 2);
  for (int i = 0; i <= res; ++i)
    for (int k = 0; k < 3; ++k) hat_integrals(depth, i, trial_depth, (i >> shift) + k - 1, &table[(i * 3 + k) * 2]);
  A.offsets.assign(rows.size() + 1, 0);
  std::vector<std::array<int32_t, 27>> cand(rows.size());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(rows.size()); ++i) {
    int c[3];
    coords(rows[i], c);
    int ctr[3] = {c[0] >> shift, c[1] >> shift, c[2] >> shift};
    int count = 0;
    for (int k = 0; k < 27; ++k) {
      int q[3] = {ctr[0] + k / 9 - 1, ctr[1] + (k / 3) % 3 - 1, ctr[2] + k % 3 - 1};
      int64_t idx = -1;
      if (std::min(q[0], std::min(q[1], q[2])) >= 0 && std::max(q[0], std::max(q[1], q[2])) <= (1 << trial_depth))
        idx = find_key(cols, basis_key(trial_depth, q[0], q[1], q[2]));
      cand[i][k] = int32_t(idx);
      if (idx >= 0) ++count;
    }
    A.offsets[i + 1] = count;
  }
  for (size_t i = 0; i < rows.size(); ++i) A.offsets[i + 1] += A.offsets[i];
  A.columns.resize(A.offsets.back());
  A.values.resize(A.offsets.back());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(rows.size()); ++i) {
    int c[3];
    coords(rows[i], c);
    int out = A.offsets[i];
    for (int k = 0; k < 27; ++k) {
      if (cand[i][k] < 0) continue;
      const double* x = &table[(c[0] * 3 + k / 9) * 2];
      const double* y = &table[(c[1] * 3 + (k / 3) % 3) * 2];
      const double* z = &table[(c[2] * 3 + k % 3) * 2];
      A.values[out] = x[1] * y[0] * z[0] + x[0] * y[1] * z[0] + x[0] * y[0] * z[1];
      A.columns[out] = cand[i][k];
      ++out;
    }
  }
  return A;
}

template <class T>
struct Points {
  std::vector<T> positions;  // 3 per point
  std::vector<T> weights;
  std::vector<int64_t> bin_keys;  // sorted
  std::vector<int64_t> bin_ids;
};

// constraints.py:20-84
template <class T>
Points<T> point_constraints(const Density<T>& D, const Normals<T>& N, const Tree& tree, int depth, double pw,
                            bool exact) {
  Points<T> P;
  const auto& keys = D.agg_keys[depth];
  const auto& vals = D.agg_values[depth];
  size_t m = keys.size();
  P.positions.resize(3 * m);
  P.weights.resize(m);
  for (size_t i = 0; i < m; ++i) {
    const T* v = &vals[4 * i];
    for (int a = 0; a < 3; ++a) P.positions[3 * i + a] = v[a] / v[3];
    int c[3];
    coords(keys[i], c);
    T w = v[3] * T(1 << depth);
    w = w * (T(pw) * N.average[1]);
    if (depth == 0 || find_key(tree.support[depth], tree_key(c[0], c[1], c[2])) < 0) w = T(0);
    P.weights[i] = exact ? T(0) : w;
  }
  // screening_stencils.py:17-26,80-88 floor bins, stable sorted
  int n = 1 << depth;
  std::vector<int64_t> bk(m);
  for (size_t i = 0; i < m; ++i) {
    int c[3];
    for (int a = 0; a < 3; ++a) {
      int f = int(std::floor(P.positions[3 * i + a] * T(n)));
      c[a] = std::min(std::max(f, 0), n - 1);
    }
    bk[i] = basis_key(depth, c[0], c[1], c[2]);
  }
  auto ids = stable_order(bk);
  P.bin_keys.resize(m);
  P.bin_ids.resize(m);
  for (size_t i = 0; i < m; ++i) {
    P.bin_keys[i] = bk[ids[i]];
    P.bin_ids[i] = ids[i];
  }
  return P;
}

template <class T>
inline T hat3(const T p[3], const int c[3], int depth) {  // screening_stencils.py:28-32
  T h[3];
  for (int a = 0; a < 3; ++a) {
    T t = p[a] * T(1 << depth) - T(c[a]);
    h[a] = std::max(T(1.0) - std::abs(t), T(0.0));
  }
  return h[0] * h[1] * h[2];
}

// screening_stencils.py:34-101 — adds Σ w φ_i φ_j to the existing entries; returns Σ w φ_i.
template <class T>
std::vector<double> add_screening(Csr<double>& A, const std::vector<int64_t>& rows, const std::vector<int64_t>& cols,
                                  const Points<T>& P, int depth, int trial_depth) {
  std::vector<double> load(rows.size());
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < int64_t(rows.size()); ++i) {
    int c[3];
    coords(rows[i], c);
    double acc[27] = {0};
    double rhs = 0.0;
    int begin = A.offsets[i], end = A.offsets[i + 1];
    for (int k = 0; k < 8; ++k) {
      int cell[3] = {c[0] - k / 4, c[1] - (k / 2) % 2, c[2] - k % 2};
      if (std::min(cell[0], std::min(cell[1], cell[2])) < 0 ||
          std::max(cell[0], std::max(cell[1], cell[2])) >= (1 << depth))
        continue;
      int64_t key = basis_key(depth, cell[0], cell[1], cell[2]);
      int64_t j = find_key(P.bin_keys, key);
      if (j < 0) continue;
      for (; j < int64_t(P.bin_keys.size()) && P.bin_keys[j] == key; ++j) {
        int64_t index = P.bin_ids[j];
        const T* p = &P.positions[3 * index];
        T weight = P.weights[index];
        if (weight == T(0)) continue;
        T phi = hat3(p, c, depth);
        rhs += double(phi * weight);
        for (int e = begin; e < end; ++e) {
          int q[3];
          coords(cols[A.columns[e]], q);
          T trial = hat3(p, q, trial_depth);
          acc[e - begin] += double(phi * trial * weight);
        }
      }
    }
    load[i] = rhs;
    for (int e = begin; e < end; ++e) A.values[e] += acc[e - begin];
  }
  return load;
}

// ---------------------------------------------------------------- A9 transfers (transfer_stencils.py:12-66)
template <class T>
Csr<T> prolongation(const std::vector<int64_t>& coarse, const std::vector<int64_t>& fine, int depth) {
  Csr<T> P;
  P.rows = int64_t(fine.size());
  P.cols = int64_t(coarse.size());
  P.offsets.assign(fine.size() + 1, 0);
  std::vector<std::array<int32_t, 8>> col(fine.size());
  std::vector<std::array<T, 8>> val(fine.size());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(fine.size()); ++i) {
    int f[3];
    coords(fine[i], f);
    int count = 0;
    for (int k = 0; k < 8; ++k) {
      int c[3] = {f[0] / 2 + k / 4, f[1] / 2 + (k / 2) % 2, f[2] / 2 + k % 2};
      T h[3];
      for (int a = 0; a < 3; ++a) h[a] = T(1.0) - std::abs(T(f[a]) * T(0.5) - T(c[a]));
      T weight = h[0] * h[1] * h[2];
      int64_t column = -1;
      if (weight > T(0)) column = find_key(coarse, basis_key(depth - 1, c[0], c[1], c[2]));
      if (column >= 0) {
        col[i][count] = int32_t(column);
        val[i][count] = weight;
        ++count;
      }
    }
    P.offsets[i + 1] = count;
  }
  for (size_t i = 0; i < fine.size(); ++i) P.offsets[i + 1] += P.offsets[i];
  P.columns.resize(P.offsets.back());
  P.values.resize(P.offsets.back());
  for (size_t i = 0; i < fine.size(); ++i)
    for (int e = P.offsets[i]; e < P.offsets[i + 1]; ++e) {
      P.columns[e] = col[i][e - P.offsets[i]];
      P.values[e] = val[i][e - P.offsets[i]];
    }
  return P;
}

template <class T>
Csr<T> transposed(const Csr<T>& A) {  // CSR transpose, rows of the result in ascending source order
  Csr<T> R;
  R.rows = A.cols;
  R.cols = A.rows;
  R.offsets.assign(A.cols + 1, 0);
  for (int32_t c : A.columns) R.offsets[c + 1]++;
  for (int64_t i = 0; i < A.cols; ++i) R.offsets[i + 1] += R.offsets[i];
  R.columns.resize(A.columns.size());
  R.values.resize(A.values.size());
  std::vector<int32_t> fill(R.offsets.begin(), R.offsets.end() - 1);
  for (int64_t i = 0; i < A.rows; ++i)
    for (int e = A.offsets[i]; e < A.offsets[i + 1]; ++e) {
      int p = fill[A.columns[e]]++;
      R.columns[p] = int32_t(i);
      R.values[p] = A.values[e];
    }
  return R;
}

// y = alpha*A x + beta*y with alpha, beta in {-1, 0, 1}: row sums in CSR order.
template <class T, class S>
void spmv(const Csr<S>& A, const std::vector<T>& x, std::vector<T>& y, int alpha, int beta) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.rows; ++i) {
    T s = T(0);
    for (int e = A.offsets[i]; e < A.offsets[i + 1]; ++e) s = s + T(A.values[e]) * x[A.columns[e]];
    T a = alpha == 1 ? s : (alpha == -1 ? -s : T(0));
    y[i] = beta == 0 ? a : (beta == 1 ? a + y[i] : a - y[i]);
  }
}

// ---------------------------------------------------------------- A6 normal loads (normal_loads.py, normal_stencils.py)
inline void quadratic_piece(double t0, double step, int offset, double b[3]) {  // ordered_normal_loads.py:15-34
  b[0] = b[1] = b[2] = 0.0;
  if (offset == -1) {
    b[0] = 0.5 * (1.0 - t0) * (1.0 - t0);
    b[1] = -(1.0 - t0) * step;
    b[2] = 0.5 * step * step;
  } else if (offset == 0) {
    b[0] = 0.5 + t0 - t0 * t0;
    b[1] = (1.0 - 2.0 * t0) * step;
    b[2] = -step * step;
  } else if (offset == 1) {
    b[0] = 0.5 * t0 * t0;
    b[1] = t0 * step;
    b[2] = 0.5 * step * step;
  }
}

// ordered_normal_loads.py:37-84
void normal_integral(int test_depth, int test_index, int normal_depth, int normal_index, double out[2]) {
  int nt = 1 << test_depth, nn = 1 << normal_depth;
  int resolution = std::max(nt, nn);
  double test_step = double(nt) / double(resolution);
  double normal_step = double(nn) / double(resolution);
  int first = std::max(0, std::max((test_index - 1) * (resolution / nt), (normal_index - 1) * (resolution / nn)));
  int end = std::min(resolution, std::min((test_index + 1) * (resolution / nt), (normal_index + 2) * (resolution / nn)));
  out[0] = out[1] = 0.0;
  for (int cell = first; cell < end; ++cell) {
    double tx = double(cell) * test_step - double(test_index);
    double sign = -1.0;
    if (tx + 0.5 * test_step < 0.0) sign = 1.0;
    double h0 = 1.0 + sign * tx;
    double h1 = sign * test_step;
    int normal_cell = int(std::floor((double(cell) + 0.5) * normal_step));
    double t0 = double(cell) * normal_step - double(normal_cell);
    double b[3], r[3];
    quadratic_piece(t0, normal_step, normal_index - normal_cell, b);
    quadratic_piece(t0, normal_step, -1 - normal_index - normal_cell, r);
    for (int a = 0; a < 3; ++a) b[a] -= r[a];
    quadratic_piece(t0, normal_step, 2 * nn - 1 - normal_index - normal_cell, r);
    for (int a = 0; a < 3; ++a) b[a] -= r[a];
    out[0] += (h0 * b[0] + (h0 * b[1] + h1 * b[0]) * 0.5 + (h0 * b[2] + h1 * b[1]) / 3.0 + h1 * b[2] * 0.25) /
              double(resolution);
    out[1] += (b[0] + b[1] * 0.5 + b[2] / 3.0) * sign * test_step;
  }
}

inline int normal_center(int index, int test_depth, int normal_depth) {  // normal_stencils.py:11-18
  if (test_depth > normal_depth) return index >> 1;
  if (test_depth < normal_depth) return index << 1;
  return index;
}

// normal_stencils.py:11-70
template <class T>
std::vector<double> normal_stencil(const std::vector<int64_t>& keys, const int64_t* nkeys, const T* nvals, size_t nrec,
                                   int test_depth, int normal_depth) {
  std::vector<double> out(keys.size(), 0.0);
  if (!nrec) return out;
  int width = test_depth < normal_depth ? 6 : 4;
  int first = test_depth < normal_depth ? -3 : -2;
  int res = 1 << test_depth;
  std::vector<double> table(size_t(res + 1) * width * 2);
  for (int i = 0; i <= res; ++i)
    for (int k = 0; k < width; ++k)
      normal_integral(test_depth, i, normal_depth, normal_center(i, test_depth, normal_depth) + first + k,
                      &table[(i * width + k) * 2]);
  std::vector<int64_t> nk(nkeys, nkeys + nrec);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(keys.size()); ++i) {
    int c[3];
    coords(keys[i], c);
    int ctr[3] = {normal_center(c[0], test_depth, normal_depth), normal_center(c[1], test_depth, normal_depth),
                  normal_center(c[2], test_depth, normal_depth)};
    double value = 0.0;
    for (int k = 0; k < width * width * width; ++k) {
      int x = k / (width * width), y = (k / width) % width, z = k % width;
      int n[3] = {ctr[0] + x + first, ctr[1] + y + first, ctr[2] + z + first};
      if (std::min(n[0], std::min(n[1], n[2])) < 0 || std::max(n[0], std::max(n[1], n[2])) >= (1 << normal_depth))
        continue;
      int64_t j = find_key(nk, basis_key(normal_depth, n[0], n[1], n[2]));
      if (j < 0) continue;
      const double* ix = &table[(c[0] * width + x) * 2];
      const double* iy = &table[(c[1] * width + y) * 2];
      const double* iz = &table[(c[2] * width + z) * 2];
      const T* v = nvals + 4 * j;
      value += double(v[0]) * ix[1] * iy[0] * iz[0];
      value += double(v[1]) * ix[0] * iy[1] * iz[0];
      value += double(v[2]) * ix[0] * iy[0] * iz[1];
    }
    out[i] = value;
  }
  return out;
}

// normal_loads.py:27-63 — degree-1 prolongation of the normal coefficients (issue #35).
template <class T>
std::vector<T> prolong_normals(const std::vector<int64_t>& keys, const std::vector<int64_t>& prev_keys,
                               const std::vector<T>& prev, const int64_t* own_keys, const T* own, size_t nown,
                               int depth) {
  std::vector<T> out(4 * keys.size(), T(0));
  std::vector<int64_t> ok(own_keys, own_keys + nown);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(keys.size()); ++i) {
    int c[3];
    coords(keys[i], c);
    T value[4] = {T(0), T(0), T(0), T(0)};
    int64_t j = find_key(ok, keys[i]);
    if (j >= 0)
      for (int a = 0; a < 4; ++a) value[a] = own[4 * j + a];
    if (depth > 0) {
      for (int corner = 0; corner < 8; ++corner) {
        int p[3] = {c[0] / 2, c[1] / 2, c[2] / 2};
        T weight = T(1.0);
        for (int axis = 0; axis < 3; ++axis) {
          if ((corner >> axis) & 1) p[axis] += 1;
          weight = weight * (T(1.0) - std::abs(T(c[axis]) * T(0.5) - T(p[axis])));
        }
        if (weight > T(0)) {
          int64_t q = find_key(prev_keys, basis_key(depth - 1, p[0], p[1], p[2]));
          if (q >= 0)
            for (int a = 0; a < 4; ++a) value[a] = value[a] + prev[4 * q + a] * weight;
        }
      }
    }
    for (int a = 0; a < 4; ++a) out[4 * i + a] = value[a];
  }
  return out;
}

// normal_loads.py:66-190 (stencil route)
template <class T>
std::vector<std::vector<double>> normal_loads(const Tree& tree, const Normals<T>& N, int max_depth, int base_depth,
                                              const std::vector<Csr<T>>& transfers) {
  std::vector<std::vector<double>> same(max_depth + 1), from_child(max_depth + 1), from_parent(max_depth + 1);
  std::vector<int64_t> prev_keys;
  std::vector<T> prev;
  bool has_cumulative = false;
  for (int d = 0; d <= max_depth; ++d) {
    const int64_t* rk = N.keys.data() + N.offsets[d];
    const T* rv = N.values.data() + 4 * N.offsets[d];
    size_t nr = N.offsets[d + 1] - N.offsets[d];
    has_cumulative = has_cumulative || nr > 0;
    if (d >= base_depth) {
      same[d] = normal_stencil(tree.basis[d], rk, rv, nr, d, d);
      if (d > base_depth) from_child[d - 1] = normal_stencil(tree.basis[d - 1], rk, rv, nr, d - 1, d);
    }
    if (d < max_depth) {
      const auto& keys = tree.basis[d];
      auto cumulative = prolong_normals(keys, prev_keys, prev, rk, rv, nr, d);
      if (d >= base_depth && has_cumulative)
        from_parent[d + 1] = normal_stencil(tree.basis[d + 1], keys.data(), cumulative.data(), keys.size(), d + 1, d);
      prev_keys = keys;
      prev = std::move(cumulative);
    }
  }
  std::vector<std::vector<double>> loads(max_depth + 1);
  std::vector<double> finer(tree.basis[max_depth].size(), 0.0);
  for (int d = max_depth; d >= base_depth; --d) {
    std::vector<double> load = same[d];
    for (size_t i = 0; i < load.size(); ++i) load[i] = finer[i] + load[i];
    if (!from_parent[d].empty())
      for (size_t i = 0; i < load.size(); ++i) load[i] = from_parent[d][i] + load[i];
    loads[d] = std::move(load);
    if (d > base_depth) {
      std::vector<double> next = from_child[d - 1];
      Csr<double> P;
      const Csr<T>& Pt = transfers[d - 1];
      P.rows = Pt.rows;
      P.cols = Pt.cols;
      P.offsets = Pt.offsets;
      P.columns = Pt.columns;
      P.values.assign(Pt.values.begin(), Pt.values.end());
      Csr<double> R = transposed(P);
      spmv(R, finer, next, 1, 1);
      finer = std::move(next);
    }
  }
  return loads;
}

// ---------------------------------------------------------------- A8 relaxation (relaxation.py)
template <class T>
inline void gs_row(const Csr<T>& A, const std::vector<T>& b, std::vector<T>& x, int64_t i) {  // relaxation.py:51-62
  T r = b[i];
  T diagonal = T(0);
  for (int e = A.offsets[i]; e < A.offsets[i + 1]; ++e) {
    int col = A.columns[e];
    r = r - x[col] * A.values[e];
    if (col == i) diagonal = A.values[e];
  }
  if (diagonal != T(0)) x[i] = x[i] + r * (T(1.0) / diagonal);
}

// groups[g] lists the rows of group g in ascending row order (relaxation.py:14-29,221-238).
std::vector<std::vector<int64_t>> row_groups(const std::vector<int64_t>& keys, int depth, bool sliced) {
  int count = sliced ? 4 * ((1 << depth) + 1) : 8;
  std::vector<std::vector<int64_t>> groups(count);
  for (size_t i = 0; i < keys.size(); ++i) {
    int c[3];
    coords(keys[i], c);
    int g = sliced ? (c[0] & 1) + 2 * (c[1] & 1) + 4 * c[2] : (c[0] & 1) + 2 * (c[1] & 1) + 4 * (c[2] & 1);
    groups[g].push_back(int64_t(i));
  }
  return groups;
}

template <class T>
void relax_group(const Csr<T>& A, const std::vector<T>& b, std::vector<T>& x, const std::vector<int64_t>& rows) {
#pragma omp parallel for schedule(static) if (rows.size() > 4096)
  for (int64_t j = 0; j < int64_t(rows.size()); ++j) gs_row(A, b, x, rows[j]);
}

// relaxation.py:121-126 sequential definition of the sliced order
template <class T>
void relax_sliced(const Csr<T>& A, const std::vector<T>& b, std::vector<T>& x,
                  const std::vector<std::vector<int64_t>>& groups, int depth, int iters) {
  int n = 1 << depth;
  for (int front = n; front > -iters; --front)
    for (int z = std::max(front, 0); z < std::min(front + iters, n + 1); ++z)
      for (int color = 0; color < 4; ++color) relax_group(A, b, x, groups[z * 4 + color]);
}

// relaxation.py:261-271
template <class T>
void relax_scheduled(const Csr<T>& A, const std::vector<T>& b, std::vector<T>& x,
                     const std::vector<std::vector<int64_t>>& groups, int iters, bool forward) {
  for (int it = 0; it < iters; ++it)
    for (int k = 0; k < 8; ++k) relax_group(A, b, x, groups[forward ? k : 7 - k]);
}

// ---------------------------------------------------------------- A10 base solve (solver.py:167-317)
// Galerkin product R (A P) with R = P^T, both products summed in a fixed row order.
template <class T>
Csr<T> spgemm(const Csr<T>& A, const Csr<T>& B) {
  Csr<T> C;
  C.rows = A.rows;
  C.cols = B.cols;
  C.offsets.assign(A.rows + 1, 0);
  std::vector<std::vector<std::pair<int32_t, T>>> rows(A.rows);
  std::vector<T> acc(B.cols, T(0));
  std::vector<char> used(B.cols, 0);
  for (int64_t i = 0; i < A.rows; ++i) {
    std::vector<int32_t> touched;
    for (int e = A.offsets[i]; e < A.offsets[i + 1]; ++e) {
      int k = A.columns[e];
      for (int f = B.offsets[k]; f < B.offsets[k + 1]; ++f) {
        int j = B.columns[f];
        if (!used[j]) {
          used[j] = 1;
          acc[j] = T(0);
          touched.push_back(j);
        }
        acc[j] = acc[j] + A.values[e] * B.values[f];
      }
    }
    std::sort(touched.begin(), touched.end());
    for (int j : touched) {
      rows[i].push_back({j, acc[j]});
      used[j] = 0;
    }
    C.offsets[i + 1] = C.offsets[i] + int32_t(touched.size());
  }
  for (auto& r : rows)
    for (auto& e : r) {
      C.columns.push_back(e.first);
      C.values.push_back(e.second);
    }
  return C;
}

template <class T>
T dot(const std::vector<T>& a, const std::vector<T>& b) {
  T s = T(0);
  for (size_t i = 0; i < a.size(); ++i) s = s + a[i] * b[i];
  return s;
}

inline int root_row(int64_t key) {  // solver.py:30-33
  int c[3];
  coords(key, c);
  for (int a = 0; a < 3; ++a) c[a] += 2;
  return c[2] * 16 + (c[0] & 1) + 2 * (c[1] & 1) + 2 * (c[0] & 2) + 4 * (c[1] & 2);
}

template <class T>
struct RootOp {
  const Csr<T>* K;
  bool dc;
  // z = alpha*(K x) + beta*y (+ alpha*mean(x) with the constant-mode term, solver.py:128-180)
  void apply(const std::vector<T>& x, const std::vector<T>& y, std::vector<T>& z, int alpha, int beta) const {
    std::vector<T> out(y);
    spmv(*K, x, out, alpha, beta);
    if (dc) {
      T mean = T(0);
      for (T v : x) mean = mean + v;
      mean = mean / T(x.size());
      for (auto& v : out) v = v + T(alpha) * mean;
    }
    z = out;
  }
};

// Conjugate gradients with the stopping rule of warp.optim.linear.cg (absolute tolerance
// max(atol, tol*|b|, eps^(9/4)), residual checked before every iteration).
template <class T>
void root_cg(const RootOp<T>& A, const std::vector<T>& b, std::vector<T>& x, double tol, double atol, int maxiter) {
  double eps = double(std::numeric_limits<T>::epsilon());
  double bnorm = std::sqrt(double(dot(b, b)));
  double abs_tol = std::max(std::max(atol, tol * bnorm), std::pow(eps, 9.0 / 4.0));
  double atol_sq = abs_tol * abs_tol;
  T gate = T(atol_sq);
  std::vector<T> r(b.size()), Ap(b.size());
  A.apply(x, b, r, -1, 1);
  T rr = dot(r, r);
  std::vector<T> p = r;
  for (int it = 0; it < maxiter; ++it) {
    if (double(rr) <= atol_sq) break;
    A.apply(p, Ap, Ap, 1, 0);
    T pAp = dot(p, Ap);
    T alpha = rr > gate ? rr / pAp : T(0);
    for (size_t i = 0; i < x.size(); ++i) {
      x[i] = x[i] + alpha * p[i];
      r[i] = r[i] - alpha * Ap[i];
    }
    T rr_new = dot(r, r);
    T beta = rr_new > gate ? rr_new / rr : T(0);
    for (size_t i = 0; i < p.size(); ++i) p[i] = r[i] + beta * p[i];
    rr = rr_new;
  }
}

template <class T>
std::vector<T> regular_multigrid(const Csr<T>& A, const std::vector<T>& b, const std::vector<std::vector<int64_t>>& keys,
                                 const std::vector<Csr<T>>& transfers, int iters, int cycles, double cg_accuracy,
                                 bool dc) {
  int base = int(keys.size()) - 1;
  std::vector<Csr<T>> mats(base + 1), restr(base);
  mats[base] = A;
  for (int d = 0; d < base; ++d) restr[d] = transposed(transfers[d]);
  for (int d = base; d > 0; --d) mats[d - 1] = spgemm(spgemm(restr[d - 1], mats[d]), transfers[d - 1]);
  std::vector<std::vector<T>> rhs(base + 1), x(base + 1);
  for (int d = 0; d <= base; ++d) {
    rhs[d].assign(keys[d].size(), T(0));
    x[d].assign(keys[d].size(), T(0));
  }
  rhs[base] = b;
  std::vector<std::vector<std::vector<int64_t>>> groups(base + 1);
  for (int d = 0; d <= base; ++d) groups[d] = row_groups(keys[d], d, false);
  Csr<T> padded;
  RootOp<T> op{&mats[0], false};
  std::vector<T> root_rhs, root_x;
  bool embed = dc;
  if (embed) {  // solver.py:183-202
    const Csr<T>& K = mats[0];
    std::vector<std::pair<std::pair<int, int>, T>> trip;
    for (int64_t i = 0; i < K.rows; ++i)
      for (int e = K.offsets[i]; e < K.offsets[i + 1]; ++e)
        trip.push_back({{root_row(keys[0][i]), root_row(keys[0][K.columns[e]])}, K.values[e]});
    std::stable_sort(trip.begin(), trip.end(), [](auto& a, auto& b) { return a.first < b.first; });
    padded.rows = padded.cols = 64;
    padded.offsets.assign(65, 0);
    for (size_t t = 0; t < trip.size();) {
      size_t u = t;
      T v = T(0);
      while (u < trip.size() && trip[u].first == trip[t].first) v = v + trip[u++].second;
      padded.columns.push_back(trip[t].first.second);
      padded.values.push_back(v);
      padded.offsets[trip[t].first.first + 1]++;
      t = u;
    }
    for (int i = 0; i < 64; ++i) padded.offsets[i + 1] += padded.offsets[i];
    op = RootOp<T>{&padded, true};
    root_x.assign(64, T(0));
  }
  for (int cycle = 0; cycle < cycles; ++cycle) {
    for (int d = base; d > 0; --d) {
      relax_scheduled(mats[d], rhs[d], x[d], groups[d], iters, true);
      std::vector<T> residual = rhs[d];
      spmv(mats[d], x[d], residual, -1, 1);
      spmv(restr[d - 1], residual, rhs[d - 1], 1, 0);
      std::fill(x[d - 1].begin(), x[d - 1].end(), T(0));
    }
    if (embed) {
      root_rhs.assign(64, T(0));
      for (size_t i = 0; i < keys[0].size(); ++i) root_rhs[root_row(keys[0][i])] = rhs[0][i];
    } else {
      root_rhs = rhs[0];
      root_x = x[0];
    }
    std::vector<T> residual = root_rhs;
    if (base == 0 && cycle > 0) op.apply(root_x, root_rhs, residual, -1, 1);
    T nsq = dot(residual, residual);
    if (double(nsq) > cg_accuracy * cg_accuracy)
      root_cg(op, root_rhs, root_x, base == 0 ? 0.0 : cg_accuracy,
              base == 0 ? cg_accuracy * std::sqrt(double(nsq)) : 0.0, int(keys[0].size()));
    if (embed) {
      for (size_t i = 0; i < keys[0].size(); ++i) x[0][i] = root_x[root_row(keys[0][i])];
    } else {
      x[0] = root_x;
    }
    for (int d = 1; d <= base; ++d) {
      spmv(transfers[d - 1], x[d - 1], x[d], 1, 1);
      std::fill(x[d - 1].begin(), x[d - 1].end(), T(0));
      if (embed && d == 1) std::fill(root_x.begin(), root_x.end(), T(0));
      relax_scheduled(mats[d], rhs[d], x[d], groups[d], iters, false);
    }
  }
  return x[base];
}

template <class T>
Csr<T> cast_csr(const Csr<double>& A) {
  Csr<T> B;
  B.rows = A.rows;
  B.cols = A.cols;
  B.offsets = A.offsets;
  B.columns = A.columns;
  B.values.resize(A.values.size());
  for (size_t i = 0; i < A.values.size(); ++i) B.values[i] = T(A.values[i]);
  return B;
}

// ---------------------------------------------------------------- A11/A12 field (field.py:187-421, transforms.py)
template <class T>
void add_level(const std::vector<int64_t>& keys, const T* coeff, const T p[3], int d, T result[4]) {
  int n = 1 << d;  // field.py:370-393
  T t[3];
  int cell[3], base[3];
  T f[3];
  for (int a = 0; a < 3; ++a) {
    t[a] = p[a] * T(n);
    cell[a] = std::min(std::max(int(std::ceil(t[a])) - 1, 0), n - 1);
    base[a] = int(std::floor(t[a]));
    f[a] = t[a] - T(base[a]);
  }
  for (int corner = 0; corner < 8; ++corner) {
    int node[3] = {cell[0] + corner / 4, cell[1] + (corner / 2) % 2, cell[2] + corner % 2};
    if (std::min(node[0] - base[0], std::min(node[1] - base[1], node[2] - base[2])) < 0) continue;
    int64_t idx = find_key(keys, basis_key(d, node[0], node[1], node[2]));
    if (idx < 0) continue;
    T h[3], s[3];
    for (int a = 0; a < 3; ++a) {
      h[a] = T(1) - f[a];
      s[a] = T(-1);
      if (node[a] > base[a]) {
        h[a] = f[a];
        s[a] = T(1);
      }
    }
    T c = coeff[idx];
    result[0] = result[0] + c * h[0] * h[1] * h[2];
    result[1] = result[1] + c * T(n) * s[0] * h[1] * h[2];
    result[2] = result[2] + c * T(n) * h[0] * s[1] * h[2];
    result[3] = result[3] + c * T(n) * h[0] * h[1] * s[2];
  }
}

template <class T>
void evaluate_query(const std::vector<int64_t>& keys, const T* coeff, const T* cumulative, const T q[3],
                    const T L[9], const T tr[3], int depth, T& value, T grad[3], int& valid) {
  T p[3];  // field.py:395-421
  for (int r = 0; r < 3; ++r) p[r] = L[3 * r] * q[0] + L[3 * r + 1] * q[1] + L[3 * r + 2] * q[2] + tr[r];
  bool ok = std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]) &&
            std::min(p[0], std::min(p[1], p[2])) >= T(0) && std::max(p[0], std::max(p[1], p[2])) <= T(1);
  valid = ok;
  if (!ok) {
    value = grad[0] = grad[1] = grad[2] = std::numeric_limits<T>::quiet_NaN();
    return;
  }
  int leaf = 0;
  for (int d = depth; d >= 0; --d) {
    int n = 1 << d;
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = std::min(std::max(int(std::ceil(p[a] * T(n))) - 1, 0), n - 1);
    if (find_key(keys, basis_key(d, c[0], c[1], c[2])) >= 0) {
      leaf = d;
      break;
    }
  }
  for (int a = 0; a < 3; ++a) {
    if (p[a] == T(0))
      p[a] = T(1e-6);
    else if (p[a] == T(1))
      p[a] = T(1.0 - 1e-6);
  }
  T r[4] = {T(0), T(0), T(0), T(0)};
  add_level(keys, coeff, p, leaf, r);
  if (leaf > 0) {
    T s[4] = {T(0), T(0), T(0), T(0)};
    add_level(keys, cumulative, p, leaf - 1, s);
    for (int a = 0; a < 4; ++a) r[a] = r[a] + s[a];
  }
  if (leaf < depth) {
    T s[4] = {T(0), T(0), T(0), T(0)};
    add_level(keys, coeff, p, leaf + 1, s);
    for (int a = 0; a < 4; ++a) r[a] = r[a] + s[a];
  }
  value = r[0];
  for (int a = 0; a < 3; ++a) grad[a] = L[a] * r[1] + L[3 + a] * r[2] + L[6 + a] * r[3];
}

template <class T>
T det3(const T m[9]) {  // transforms.py:16-22
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
template <class T>
T minor4(const T m[16], int row, int col) {
  T out[9];
  int rr = 0;
  for (int r = 0; r < 4; ++r) {
    if (r == row) continue;
    int cc = 0;
    for (int c = 0; c < 4; ++c) {
      if (c == col) continue;
      out[rr * 3 + cc] = m[r * 4 + c];
      ++cc;
    }
    ++rr;
  }
  return det3(out);
}
template <class T>
void reference_inverse(const T m[16], T out[16]) {  // transforms.py:38-53
  T det = T(0);
  for (int c = 0; c < 4; ++c) {
    if (c % 2 == 0)
      det = det + m[c] * minor4(m, 0, c);
    else
      det = det - m[c] * minor4(m, 0, c);
  }
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      T v = minor4(m, r, c);
      if ((r + c) % 2 != 0) v = -v;
      out[c * 4 + r] = v / det;
    }
}

// Fixed blocked order shared with the CUDA isovalue kernel: 1024-value blocks; inside a
// block, 256 lanes each sum 4 strided values serially in float64, then a pairwise tree
// over lanes (stride 128, 64, ..., 1); block totals are summed serially.
template <class T>
void blocked_isovalue(const std::vector<T>& values, const std::vector<T>& weights, double& total, double& mass) {
  size_t n = values.size();
  total = 0.0;
  mass = 0.0;
  for (size_t b = 0; b < n; b += 1024) {
    double tv[256], tw[256];
    for (int l = 0; l < 256; ++l) {
      tv[l] = 0.0;
      tw[l] = 0.0;
      for (int j = 0; j < 4; ++j) {
        size_t i = b + size_t(l) + 256 * size_t(j);
        if (i < n) {
          tv[l] += double(values[i] * weights[i]);
          tw[l] += double(weights[i]);
        }
      }
    }
    for (int stride = 128; stride >= 1; stride /= 2)
      for (int l = 0; l < stride; ++l) {
        tv[l] = tv[l] + tv[l + stride];
        tw[l] = tw[l] + tw[l + stride];
      }
    total += tv[0];
    mass += tw[0];
  }
}

// ---------------------------------------------------------------- driver (reconstruction.py:137-349, solver.py:320-466)
// tree_only: stop after the tree (stages up to A4, basis and support keys; no solve).
template <class T>
Result<T>* reconstruct(const T* pos, const T* nrm, int64_t count, const Params& prm, bool tree_only = false) {
  auto R = std::make_unique<Result<T>>();
  R->dtype = sizeof(T) == 8 ? 1 : 0;
  R->depth = prm.depth;
  Samples<T> S = prepare_samples(pos, nrm, count, prm.depth, prm.scale);
  put_stage(*R, "group_keys", S.keys);
  put_stage(*R, "group_sums", S.sums);
  put_stage(*R, "group_normal_sums", S.normal_sums);
  put_stage(*R, "group_weights", S.weights);
  put_stage(*R, "group_first", S.first);
  put_stage(*R, "transform", std::vector<T>(S.transform, S.transform + 5));
  Density<T> D = build_density(S, prm.depth, prm.kernel_depth, prm.samples_per_node);
  put_stage(*R, "depths_and_weights", D.dw);
  for (int d = 0; d <= prm.depth; ++d) {
    put_stage(*R, "aggregate_keys_" + std::to_string(d), D.agg_keys[d]);
    put_stage(*R, "aggregate_values_" + std::to_string(d), D.agg_values[d]);
  }
  for (int d = 0; d <= prm.kernel_depth; ++d) {
    put_stage(*R, "density_keys_" + std::to_string(d), D.level_keys[d]);
    put_stage(*R, "density_values_" + std::to_string(d), D.level_values[d]);
  }
  Normals<T> N = build_normal_field(S, D, prm.base_depth, prm.depth);
  put_stage(*R, "normal_keys", N.keys);
  put_stage(*R, "normal_values", N.values);
  put_stage(*R, "normal_average", std::vector<T>(N.average, N.average + 3));
  Tree tree = build_tree(N, prm.depth, prm.full_depth, prm.base_depth);
  R->basis = tree.basis;
  R->support = tree.support;
  if (tree_only) {
    for (int d = 0; d <= prm.depth; ++d) {
      R->level_offsets.push_back(int64_t(R->all_keys.size()));
      R->all_keys.insert(R->all_keys.end(), tree.basis[d].begin(), tree.basis[d].end());
    }
    R->level_offsets.push_back(int64_t(R->all_keys.size()));
    return R.release();
  }
  int finest = prm.depth;
  const auto& keys = tree.basis;
  std::vector<Csr<T>> transfers(finest);
  for (int d = 1; d <= finest; ++d) transfers[d - 1] = prolongation<T>(keys[d - 1], keys[d], d);
  std::vector<std::vector<T>> corrections(finest + 1);
  for (int d = 0; d <= finest; ++d) corrections[d].assign(keys[d].size(), T(0));
  auto loads = normal_loads(tree, N, finest, prm.base_depth, transfers);
  bool screened = prm.point_weight > 0 && !prm.exact;
  std::vector<T> cumulative;
  for (int d = prm.base_depth; d <= prm.solve_depth; ++d) {
    if (keys[d].empty()) break;
    put_stage(*R, "normal_load_" + std::to_string(d), loads[d]);
    Csr<double> A64 = level_stiffness(keys[d], keys[d], d, d);
    std::vector<double> point_load(keys[d].size(), 0.0);
    Points<T> P;
    if (screened) {
      P = point_constraints(D, N, tree, d, prm.point_weight, prm.exact);
      point_load = add_screening(A64, keys[d], keys[d], P, d, d);
    }
    std::vector<T> b(keys[d].size());
    for (size_t i = 0; i < b.size(); ++i) b[i] = T(loads[d][i]) + T(0.5) * T(point_load[i]);  // solver.py:119-126
    Csr<T> A = cast_csr<T>(A64);
    put_stage(*R, "matrix_offsets_" + std::to_string(d), A.offsets);
    put_stage(*R, "matrix_columns_" + std::to_string(d), A.columns);
    put_stage(*R, "matrix_values_" + std::to_string(d), A.values);
    if (d == prm.base_depth) {
      std::vector<std::vector<int64_t>> lk(keys.begin(), keys.begin() + d + 1);
      std::vector<Csr<T>> tr(transfers.begin(), transfers.begin() + d);
      put_stage(*R, "rhs_" + std::to_string(d), b);
      corrections[d] = regular_multigrid(A, b, lk, tr, prm.iters, prm.base_v_cycles, prm.cg_accuracy,
                                         prm.base_depth == 0 && prm.point_weight == 0);
      cumulative = corrections[d];
    } else {
      Csr<double> C64 = level_stiffness(keys[d], keys[d - 1], d, d - 1);
      if (screened) add_screening(C64, keys[d], keys[d - 1], P, d, d - 1);
      Csr<T> C = cast_csr<T>(C64);
      spmv(C, cumulative, b, -1, 1);
      put_stage(*R, "rhs_" + std::to_string(d), b);
      auto groups = row_groups(keys[d], d, true);
      relax_sliced(A, b, corrections[d], groups, d, prm.iters);
      std::vector<T> next = corrections[d];
      spmv(transfers[d - 1], cumulative, next, 1, 1);
      cumulative = std::move(next);
    }
  }
  // reconstruction.py:260-281
  for (int d = 0; d <= finest; ++d) {
    R->level_offsets.push_back(int64_t(R->all_keys.size()));
    R->all_keys.insert(R->all_keys.end(), keys[d].begin(), keys[d].end());
    R->coefficients.insert(R->coefficients.end(), corrections[d].begin(), corrections[d].end());
  }
  R->level_offsets.push_back(int64_t(R->all_keys.size()));
  R->cumulative = R->coefficients;  // field.py:187-210
  for (int d = 1; d <= finest; ++d) {
    for (int64_t i = R->level_offsets[d]; i < R->level_offsets[d + 1]; ++i) {
      int c[3];
      coords(R->all_keys[i], c);
      T value = T(0);
      for (int corner = 0; corner < 8; ++corner) {
        int p[3] = {c[0] / 2 + corner / 4, c[1] / 2 + (corner / 2) % 2, c[2] / 2 + corner % 2};
        T h = (T(1) - std::abs(T(c[0]) * T(.5) - T(p[0]))) * (T(1) - std::abs(T(c[1]) * T(.5) - T(p[1]))) *
              (T(1) - std::abs(T(c[2]) * T(.5) - T(p[2])));
        if (h > T(0)) {
          int64_t idx = find_key(R->all_keys, basis_key(d - 1, p[0], p[1], p[2]));
          if (idx >= 0) value = value + R->cumulative[idx] * h;
        }
      }
      R->cumulative[i] = value + R->coefficients[i];
    }
  }
  size_t G = S.keys.size();
  std::vector<T> values(G);
  T L[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, tr[3] = {0, 0, 0};
#pragma omp parallel for schedule(static)
  for (int64_t g = 0; g < int64_t(G); ++g) {
    T q[3] = {S.sums[3 * g] / S.weights[g], S.sums[3 * g + 1] / S.weights[g], S.sums[3 * g + 2] / S.weights[g]};
    T grad[3];
    int valid;
    evaluate_query(R->all_keys, R->coefficients.data(), R->cumulative.data(), q, L, tr, prm.depth, values[g], grad,
                   valid);
  }
  put_stage(*R, "centroid_values", values);
  double total, mass;
  blocked_isovalue(values, S.weights, total, mass);
  R->iso = T(total / mass);
  T s = S.transform[0];  // transforms.py:55-79
  T m[16] = {T(0), s, T(0), S.transform[1], T(0), T(0), s, S.transform[2], s, T(0), T(0), S.transform[3],
             T(0), T(0), T(0), T(1)};
  reference_inverse(m, R->transforms[0]);
  reference_inverse(R->transforms[0], R->transforms[1]);
  return R.release();
}

}  // namespace

// ---------------------------------------------------------------- C interface (ctypes)
extern "C" {

struct oracle_params {
  int32_t depth, full_depth, base_depth, solve_depth, kernel_depth;
  double samples_per_node, scale, point_weight, cg_accuracy;
  int32_t exact, iters, base_v_cycles;
};

static thread_local std::string g_error;

void* oracle_reconstruct(const void* pos, const void* nrm, int64_t n, int32_t dtype, const oracle_params* p) {
  Params prm{p->depth, p->full_depth, p->base_depth, p->solve_depth, p->kernel_depth, p->samples_per_node,
             p->scale, p->point_weight, p->cg_accuracy, p->exact, p->iters, p->base_v_cycles};
  try {
    if (dtype == 1) return reconstruct<double>((const double*)pos, (const double*)nrm, n, prm);
    return reconstruct<float>((const float*)pos, (const float*)nrm, n, prm);
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

// The stages up to the tree only (samples, density, normal field, tree): keys, no solve.
void* oracle_tree(const void* pos, const void* nrm, int64_t n, int32_t dtype, const oracle_params* p) {
  Params prm{p->depth, p->full_depth, p->base_depth, p->solve_depth, p->kernel_depth, p->samples_per_node,
             p->scale, p->point_weight, p->cg_accuracy, p->exact, p->iters, p->base_v_cycles};
  try {
    if (dtype == 1) return reconstruct<double>((const double*)pos, (const double*)nrm, n, prm, true);
    return reconstruct<float>((const float*)pos, (const float*)nrm, n, prm, true);
  } catch (const std::exception& e) {
    g_error = e.what();
    return nullptr;
  }
}

const char* oracle_last_error() { return g_error.c_str(); }

void oracle_free(void* h) { delete (ResultBase*)h; }

int64_t oracle_level_count(void* h, int32_t d, int32_t support) {
  auto* r = (ResultBase*)h;
  return int64_t(support ? r->support[d].size() : r->basis[d].size());
}
const int64_t* oracle_level_keys(void* h, int32_t d, int32_t support) {
  auto* r = (ResultBase*)h;
  return support ? r->support[d].data() : r->basis[d].data();
}
int64_t oracle_total(void* h) { return int64_t(((ResultBase*)h)->all_keys.size()); }
const int64_t* oracle_keys(void* h) { return ((ResultBase*)h)->all_keys.data(); }
const void* oracle_coefficients(void* h) {
  auto* r = (ResultBase*)h;
  if (r->dtype == 1) return ((Result<double>*)r)->coefficients.data();
  return ((Result<float>*)r)->coefficients.data();
}
const void* oracle_cumulative(void* h) {
  auto* r = (ResultBase*)h;
  if (r->dtype == 1) return ((Result<double>*)r)->cumulative.data();
  return ((Result<float>*)r)->cumulative.data();
}
double oracle_iso(void* h) {
  auto* r = (ResultBase*)h;
  if (r->dtype == 1) return ((Result<double>*)r)->iso;
  return ((Result<float>*)r)->iso;
}
void oracle_transforms(void* h, double* out) {
  auto* r = (ResultBase*)h;
  for (int t = 0; t < 2; ++t)
    for (int i = 0; i < 16; ++i)
      out[16 * t + i] = r->dtype == 1 ? ((Result<double>*)r)->transforms[t][i] : ((Result<float>*)r)->transforms[t][i];
}
const void* oracle_stage(void* h, const char* name, int64_t* count, int32_t* elem) {
  auto* r = (ResultBase*)h;
  auto it = r->stages.find(name);
  if (it == r->stages.end()) {
    *count = -1;
    return nullptr;
  }
  *count = it->second.count;
  *elem = it->second.elem;
  return it->second.bytes.data();
}

// Field evaluation in model coordinates (Reconstruction.evaluate, field.py:150-184).
void oracle_evaluate(void* h, const void* queries, int64_t nq, void* values, void* grads, int32_t* valid) {
  auto* r = (ResultBase*)h;
  auto run = [&](auto* res) {
    using T = std::remove_reference_t<decltype(res->coefficients[0])>;
    const T* q = (const T*)queries;
    T* v = (T*)values;
    T* g = (T*)grads;
    T L[9], tr[3];
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) L[3 * i + j] = res->transforms[1][4 * i + j];
      tr[i] = res->transforms[1][4 * i + 3];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nq; ++i) {
      int ok;
      evaluate_query(res->all_keys, res->coefficients.data(), res->cumulative.data(), q + 3 * i, L, tr, res->depth,
                     v[i], g + 3 * i, ok);
      valid[i] = ok;
    }
  };
  if (r->dtype == 1)
    run((Result<double>*)r);
  else
    run((Result<float>*)r);
}

// Sequential sliced Gauss-Seidel on a caller-supplied CSR level (relaxation.py:121-126).
int32_t oracle_relax_sliced(int32_t dtype, const int64_t* keys, int64_t n, int32_t depth, const int32_t* offsets,
                            const int32_t* columns, const void* values, const void* b, void* x, int32_t iters) {
  std::vector<int64_t> k(keys, keys + n);
  auto groups = row_groups(k, depth, true);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    Csr<T> A;
    A.rows = A.cols = n;
    A.offsets.assign(offsets, offsets + n + 1);
    A.columns.assign(columns, columns + offsets[n]);
    A.values.assign((const T*)values, (const T*)values + offsets[n]);
    std::vector<T> bb((const T*)b, (const T*)b + n), xx((T*)x, (T*)x + n);
    relax_sliced(A, bb, xx, groups, depth, iters);
    std::copy(xx.begin(), xx.end(), (T*)x);
  };
  if (dtype == 1)
    run(double());
  else
    run(float());
  return 0;
}

int32_t oracle_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
}
