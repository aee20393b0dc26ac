// A5-A10: matrix-free level assembly, normal loads, ordered Gauss-Seidel, transfers and
// the cascadic schedule (warp-psr solver.py:320-466 and the modules it calls).
//
// Operators are stored as 28-slot ELL rows (slot k < 27 = k-th lexicographic neighbour,
// the reference's CSR column order; -1 = absent; slot 27 = padding for 16-byte vector
// loads).  Stiffness values come from 1-D hat-integral tables (float64), the point
// screening is accumulated in float64 per row exactly as screening_stencils.py:34-71, and
// the result is rounded once to the solve precision.
#include <atomic>
#include "psr_internal.cuh"

#include <algorithm>
#include <cmath>

namespace psr {

constexpr int kSlots = 28;

// ------------------------------------------------------------------ 1-D integral tables
// stiffness.py:14-36 — mass (.x) and stiffness (.y) integrals of Neumann hats.
__device__ void hat_integrals(int depth, int index, int trial_depth, int trial_index, double out[2]) {
  int resolution = 1 << depth;
  int ratio = 1 << (depth - trial_depth);
  int first = max(0, max(index - 1, (trial_index - 1) * ratio));
  int end = min(resolution, min(index + 1, (trial_index + 1) * ratio));
  out[0] = out[1] = 0.0;
  for (int cell = first; cell < end; ++cell) {
    double t0 = double(cell - index);
    double c0 = double(cell) / double(ratio) - double(trial_index);
    double ts = cell >= index ? -1.0 : 1.0;
    double cs = 1.0 / double(ratio);
    if (cell >= trial_index * ratio) cs = -cs;
    double tv = 1.0 - fabs(t0);
    double cv = 1.0 - fabs(c0);
    out[0] += (tv * cv + (tv * cs + ts * cv) * 0.5 + ts * cs / 3.0) / double(resolution);
    out[1] += ts * cs * double(resolution);
  }
}

__global__ void stiffness_table_kernel(int depth, int trial_depth, double* table) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > (1 << depth)) return;
  for (int k = 0; k < 3; ++k) hat_integrals(depth, i, trial_depth, (i >> (depth - trial_depth)) + k - 1, table + (i * 3 + k) * 2);
}

// ordered_normal_loads.py:15-84 — Neumann hat (and derivative) against a Dirichlet B2.
__device__ void quadratic_piece(double t0, double step, int offset, double b[3]) {
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

__device__ void normal_integral(int test_depth, int test_index, int normal_depth, int normal_index, double out[2]) {
  int nt = 1 << test_depth, nn = 1 << normal_depth;
  int resolution = max(nt, nn);
  double test_step = double(nt) / double(resolution);
  double normal_step = double(nn) / double(resolution);
  int first = max(0, max((test_index - 1) * (resolution / nt), (normal_index - 1) * (resolution / nn)));
  int end = min(resolution, min((test_index + 1) * (resolution / nt), (normal_index + 2) * (resolution / nn)));
  out[0] = out[1] = 0.0;
  for (int cell = first; cell < end; ++cell) {
    double tx = double(cell) * test_step - double(test_index);
    double sign = -1.0;
    if (tx + 0.5 * test_step < 0.0) sign = 1.0;
    double h0 = 1.0 + sign * tx;
    double h1 = sign * test_step;
    int normal_cell = int(floor((double(cell) + 0.5) * normal_step));
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

__device__ __forceinline__ int normal_center(int index, int test_depth, int normal_depth) {
  if (test_depth > normal_depth) return index >> 1;
  if (test_depth < normal_depth) return index << 1;
  return index;
}

__global__ void normal_table_kernel(int test_depth, int normal_depth, int first, int width, double* table) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > (1 << test_depth)) return;
  for (int k = 0; k < width; ++k)
    normal_integral(test_depth, i, normal_depth, normal_center(i, test_depth, normal_depth) + first + k,
                    table + (i * width + k) * 2);
}

// Columns of the 27 neighbours q = ctr + (dx, dy, dz) at depth d (slot order), found with
// one column probe per (dx, dy) and a scan over three consecutive z (any column index).
__device__ __forceinline__ uint32_t neighbours27_scan(const ColumnView& cv, int d, const int ctr[3], int64_t off,
                                                 int32_t col[27]) {
  const int lim = 1 << d;
  uint32_t present = 0;
#pragma unroll
  for (int k = 0; k < 27; ++k) col[k] = -1;
  for (int dx = 0; dx < 3; ++dx) {
    int qx = ctr[0] + dx - 1;
    if (qx < 0 || qx > lim) continue;
    for (int dy = 0; dy < 3; ++dy) {
      int qy = ctr[1] + dy - 1;
      if (qy < 0 || qy > lim) continue;
      int32_t count;
      const int32_t j0 = cv.column_range(d, qx, qy, count);
      if (j0 < 0) continue;
      const int64_t colk = ColumnView::column_key(d, qx, qy) >> 16;
      const int z0 = ctr[2] - 1;
      const int64_t end = count == INT32_MAX ? cv.n : int64_t(j0) + count;
      int32_t j = cv.lower_z(j0, count, colk, z0);
      // the keys of z0, z0 + 1, z0 + 2 (those present) follow each other from j
#pragma unroll
      for (int dz = 0; dz < 3; ++dz) {
        if (j >= end) break;
        const int64_t key = __ldg(cv.keys + j);
        if ((key >> 16) != colk) break;
        if (int(key & 65535) != z0 + dz) continue;
        const int k = dx * 9 + dy * 3 + dz;
        col[k] = int32_t(j - off);
        present |= 1u << k;
        ++j;
      }
    }
  }
  return present;
}

// The same with the dense column table (depth <= 12): the nine column ranges are read
// together and their lower bounds of z = ctr_z - 1 advance in lock step, so each step's nine
// loads are in flight at once (the row's dependent-load chain is one binary search long, not
// nine); then the up to three keys after each bound are matched to dz.  Same result.
__device__ __forceinline__ uint32_t neighbours27(const ColumnView& cv, int d, const int ctr[3], int64_t off,
                                                 int32_t col[27]) {
  if (!cv.dense) return neighbours27_scan(cv, d, ctr, off, col);
  const int lim = 1 << d;
  const int side = lim + 1;
  const int z0 = ctr[2] - 1;
  const int2* dense = cv.dense + dense_column_base(d);
  int32_t lo[9], hi[9], end[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const int qx = ctr[0] + c / 3 - 1, qy = ctr[1] + c % 3 - 1;
    lo[c] = 0;
    end[c] = 0;
    if (unsigned(qx) <= unsigned(lim) && unsigned(qy) <= unsigned(lim)) {
      const int2 e = __ldg(dense + int64_t(qx) * side + qy);
      if (e.x >= 0) {
        lo[c] = e.x;
        end[c] = e.x + e.y;
      }
    }
    hi[c] = end[c];
  }
  for (int step = 0; step < 32; ++step) {
    bool active = false;
#pragma unroll
    for (int c = 0; c < 9; ++c) active |= lo[c] < hi[c];
    if (!active) break;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      if (lo[c] < hi[c]) {
        const int32_t mid = (lo[c] + hi[c]) >> 1;
        if (int(__ldg(cv.keys + mid) & 65535) < z0)
          lo[c] = mid + 1;
        else
          hi[c] = mid;
      }
    }
  }
  uint32_t present = 0;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    constexpr int kNone = -0x40000000;  // below every z0 + dz
    int zs[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) zs[e] = lo[c] + e < end[c] ? int(__ldg(cv.keys + lo[c] + e) & 65535) : kNone;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz) {
      int32_t found = -1;
#pragma unroll
      for (int e = 0; e < 3; ++e)
        if (zs[e] == z0 + dz) found = int32_t(lo[c] + e - off);
      col[c * 3 + dz] = found;
      if (found >= 0) present |= 1u << (c * 3 + dz);
    }
  }
  return present;
}

// ------------------------------------------------------------------ A6 normal loads (normal_stencils.py:11-70)
// `nvals` are 4-wide normal coefficients indexed by (hash result - noff).
template <class T>
__global__ void __launch_bounds__(256, 6) normal_stencil_kernel(const int64_t* keys, int64_t n, int test_depth, int normal_depth, ColumnView cv,
                                      int64_t noff, const T* nvals, const double* table, int width, int first,
                                      double* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  int ctr[3] = {normal_center(c[0], test_depth, normal_depth), normal_center(c[1], test_depth, normal_depth),
                normal_center(c[2], test_depth, normal_depth)};
  int lim = 1 << normal_depth;
  int z0 = ctr[2] + first;
  double value = 0.0;
  for (int x = 0; x < width; ++x) {
    int nx = ctr[0] + x + first;
    if (nx < 0 || nx >= lim) continue;
    const double* ix = table + (c[0] * width + x) * 2;
    for (int y = 0; y < width; ++y) {
      int ny = ctr[1] + y + first;
      if (ny < 0 || ny >= lim) continue;
      int32_t count;
      const int32_t j0 = cv.column_range(normal_depth, nx, ny, count);
      if (j0 < 0) continue;
      const double* iy = table + (c[1] * width + y) * 2;
      const int64_t colk = ColumnView::column_key(normal_depth, nx, ny) >> 16;
      const int64_t end = count == INT32_MAX ? cv.n : int64_t(j0) + count;
      int32_t j = cv.lower_z(j0, count, colk, z0);
      // ascending z inside the window: the reference's innermost loop order
      for (int z = 0; z < width; ++z) {
        if (j >= end) break;
        const int64_t key = __ldg(cv.keys + j);
        if ((key >> 16) != colk) break;
        const int kz = int(key & 65535);
        if (kz != z0 + z) continue;
        ++j;
        if (kz >= lim) continue;
        const double* iz = table + (c[2] * width + z) * 2;
        const T* v = nvals + 4 * (int64_t(j - 1) - noff);
        value += double(v[0]) * ix[1] * iy[0] * iz[0];
        value += double(v[1]) * ix[0] * iy[1] * iz[0];
        value += double(v[2]) * ix[0] * iy[0] * iz[1];
      }
    }
  }
  out[i] = value;
}

// The first three components of a normal record (4 values, 16- or 32-byte aligned) with
// one vector load and one scalar load (double) or one vector load (float).
__device__ __forceinline__ void load_normal3(const double* v, double& a, double& b, double& c) {
  const double2 ab = __ldg(reinterpret_cast<const double2*>(v));
  a = ab.x;
  b = ab.y;
  c = __ldg(v + 2);
}
__device__ __forceinline__ void load_normal3(const float* v, float& a, float& b, float& c) {
  const float4 r = __ldg(reinterpret_cast<const float4*>(v));
  a = r.x;
  b = r.y;
  c = r.z;
}

// The same with the dense column table and a compile-time window W: for each x the W
// columns' ranges are read together and their lower bounds of z0 advance in lock step, and
// the up to W keys after each bound (increasing z, so in the z-loop's order) are loaded
// together.  The row's 1-D integrals along y and z (2 W table entries each) are loaded once
// into registers; a column's normals in the window become a bit mask over the W z offsets
// (keys ascend, so the t-th set bit is the t-th key after the bound), which keeps every
// register index a constant.  The kernel is bound by L1 throughput (scattered 8-byte loads),
// so fewer loads per row is what counts.  The additions run in the same (x, y, z) order with
// the same products: same result.
template <class T, int W>
__global__ void __launch_bounds__(256, W == 4 ? 4 : 3) normal_stencil_dense_kernel(const int64_t* keys, int64_t n, int test_depth,
                                                                      int normal_depth, ColumnView cv, int64_t noff,
                                                                      const T* nvals, const double* table, int first,
                                                                      double* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  const int ctr[3] = {normal_center(c[0], test_depth, normal_depth), normal_center(c[1], test_depth, normal_depth),
                      normal_center(c[2], test_depth, normal_depth)};
  const int lim = 1 << normal_depth;
  const int side = lim + 1;
  const int z0 = ctr[2] + first;
  const int2* dense = cv.dense + dense_column_base(normal_depth);
  const double2* tab = reinterpret_cast<const double2*>(table);  // entry (coordinate * W + offset)
  // W = 6 keeps only z's entries in registers (y's are read per window column): with both,
  // the wide window needs more registers than 3 blocks per SM allow.
  constexpr int WY = W <= 4 ? W : 1;
  double2 ty[WY], tz[W];
#pragma unroll
  for (int o = 0; o < W; ++o) {
    if (W <= 4) ty[o < WY ? o : 0] = __ldg(tab + c[1] * W + o);
    tz[o] = __ldg(tab + c[2] * W + o);
  }
  double value = 0.0;
  for (int x = 0; x < W; ++x) {
    const int nx = ctr[0] + x + first;
    if (nx < 0 || nx >= lim) continue;
    const double2 tx = __ldg(tab + c[0] * W + x);
    int32_t lo[W], hi[W], end[W];
#pragma unroll
    for (int y = 0; y < W; ++y) {
      const int ny = ctr[1] + y + first;
      lo[y] = 0;
      end[y] = 0;
      if (ny >= 0 && ny < lim) {
        const int2 e = __ldg(dense + int64_t(nx) * side + ny);
        if (e.x >= 0) {
          lo[y] = e.x;
          end[y] = e.x + e.y;
        }
      }
      hi[y] = end[y];
    }
    for (int step = 0; step < 32; ++step) {
      bool active = false;
#pragma unroll
      for (int y = 0; y < W; ++y) active |= lo[y] < hi[y];
      if (!active) break;
#pragma unroll
      for (int y = 0; y < W; ++y) {
        if (lo[y] < hi[y]) {
          const int32_t mid = (lo[y] + hi[y]) >> 1;
          if (int(__ldg(cv.keys + mid) & 65535) < z0)
            lo[y] = mid + 1;
          else
            hi[y] = mid;
        }
      }
    }
#pragma unroll
    for (int y = 0; y < W; ++y) {
      const double2 tyy = W <= 4 ? ty[y < WY ? y : 0] : __ldg(tab + c[1] * W + y);
      uint32_t mask = 0;  // bit t: a normal at z0 + t (keys after lo[y] ascend in z)
#pragma unroll
      for (int e = 0; e < W; ++e) {
        const int dz = lo[y] + e < end[y] ? int(__ldg(cv.keys + lo[y] + e) & 65535) - z0 : W;
        if (dz < W) mask |= 1u << dz;
      }
#pragma unroll
      for (int t = 0; t < W; ++t) {
        if (!((mask >> t) & 1u)) continue;
        if (z0 + t >= lim) continue;
        const int64_t idx = int64_t(lo[y]) + __popc(mask & ((1u << t) - 1u));
        T v0, v1, v2;
        load_normal3(nvals + 4 * (idx - noff), v0, v1, v2);
        value += double(v0) * tx.y * tyy.x * tz[t].x;
        value += double(v1) * tx.x * tyy.y * tz[t].x;
        value += double(v2) * tx.x * tyy.x * tz[t].y;
      }
    }
  }
  out[i] = value;
}

// normal_loads.py:27-63 — degree-1 prolongation of normal coefficients (issue #35).
template <class T>
__global__ void prolong_normals_kernel(const int64_t* keys, int64_t n, int d, HashView nh, const T* nvals,
                                       HashView bh, int64_t prev_off, const T* prev, T* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  T value[4] = {T(0), T(0), T(0), T(0)};
  // the own record's and the parents' first hash probes issued together, collisions after
  uint64_t hj = 0;
  int32_t j = nh.first_probe(keys[i], hj);
  T wk[8];
  int64_t key8[8];
  uint64_t h8[8];
  int32_t q8[8];
#pragma unroll
  for (int corner = 0; corner < 8; ++corner) {
    int p[3] = {c[0] / 2, c[1] / 2, c[2] / 2};
    T weight = T(1.0);
    for (int axis = 0; axis < 3; ++axis) {
      if ((corner >> axis) & 1) p[axis] += 1;
      weight = weight * (T(1.0) - fabs(T(c[axis]) * T(0.5) - T(p[axis])));
    }
    wk[corner] = weight;
    key8[corner] = basis_key(d - 1, p[0], p[1], p[2]);
    h8[corner] = 0;
    q8[corner] = (d > 0 && weight > T(0)) ? bh.first_probe(key8[corner], h8[corner]) : -1;
  }
  if (j == -2) j = nh.find_from(keys[i], hj);
#pragma unroll
  for (int corner = 0; corner < 8; ++corner)
    if (q8[corner] == -2) q8[corner] = bh.find_from(key8[corner], h8[corner]);
  if (j >= 0)
    for (int a = 0; a < 4; ++a) value[a] = nvals[4 * int64_t(j) + a];
  if (d > 0) {
    for (int corner = 0; corner < 8; ++corner) {
      const T weight = wk[corner];
      if (weight > T(0)) {
        const int32_t q = q8[corner];
        if (q >= 0) {
          const T* pv = prev + 4 * (int64_t(q) - prev_off);
          for (int a = 0; a < 4; ++a) value[a] = value[a] + pv[a] * weight;
        }
      }
    }
  }
  for (int a = 0; a < 4; ++a) out[4 * i + a] = value[a];
}

// next[i] = (P^T finer)[i] + next[i] over the 27 fine neighbours 2c+{-1,0,1}^3 (the
// transposed trilinear prolongation, ascending fine index), with weights rounded in T.
template <class T, class V>
__global__ void restrict_add_kernel(const int64_t* coarse_keys, int64_t n, int d /*fine depth*/, ColumnView cv,
                                    int64_t fine_off, const V* finer, V* next, bool accumulate) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(coarse_keys[i], c);
  int ctr[3] = {2 * c[0], 2 * c[1], 2 * c[2]};
  int32_t col[27];
  uint32_t present = neighbours27(cv, d, ctr, fine_off, col);
  V s = V(0);
  for (int k = 0; k < 27; ++k) {
    if (!((present >> k) & 1)) continue;
    int f[3] = {ctr[0] + k / 9 - 1, ctr[1] + (k / 3) % 3 - 1, ctr[2] + k % 3 - 1};
    T h[3];
    for (int a = 0; a < 3; ++a) h[a] = T(1.0) - fabs(T(f[a]) * T(0.5) - T(c[a]));
    T w = h[0] * h[1] * h[2];
    s = s + V(w) * finer[col[k]];
  }
  next[i] = accumulate ? s + next[i] : s;
}

__global__ void add3_kernel(const double* same, const double* finer, const double* parent, int64_t n, double* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  double v = finer[i] + same[i];
  out[i] = parent ? parent[i] + v : v;
}

// ------------------------------------------------------------------ A5 point constraints (constraints.py:20-84)
template <class T>
__global__ void points_kernel(const int64_t* keys, const T* vals, int64_t m, int d, T pw, const T* average,
                              HashView support, bool exact, T* pos, T* w, uint64_t* bin_keys, int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  const T* v = vals + 4 * i;
  T p[3] = {v[0] / v[3], v[1] / v[3], v[2] / v[3]};
  for (int a = 0; a < 3; ++a) pos[3 * i + a] = p[a];
  int c[3];
  key_coords(keys[i], c);
  T wt = v[3] * T(1 << d);
  wt = wt * (pw * average[1]);
  if (d == 0 || support.find(tree_key(c[0], c[1], c[2])) < 0) wt = T(0);
  w[i] = exact ? T(0) : wt;
  int n = 1 << d, D = d > 0 ? d : 1;  // screening_stencils.py:17-26 floor bins
  int b[3];
  for (int a = 0; a < 3; ++a) b[a] = min(max(int(floor(p[a] * T(n))), 0), n - 1);
  bin_keys[i] = (uint64_t(b[0]) << (2 * D)) | (uint64_t(b[1]) << D) | uint64_t(b[2]);
  ids[i] = int32_t(i);
}

__global__ void bin_heads_kernel(const uint64_t* keys, int64_t n, int32_t* heads) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) heads[i] = (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void bin_fill_kernel(const uint64_t* keys, const int32_t* heads, const int32_t* prefix, int64_t n, int d,
                                int64_t* bkeys, int32_t* bstart) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i > n) return;
  if (i == n) {
    if (n > 0) bstart[prefix[n - 1]] = int32_t(n);
    return;
  }
  if (!heads[i]) return;
  int D = d > 0 ? d : 1;
  uint64_t mask = (uint64_t(1) << D) - 1, k = keys[i];
  int64_t u = prefix[i] - 1;
  bkeys[u] = basis_key(d, int((k >> (2 * D)) & mask), int((k >> D) & mask), int(k & mask));
  bstart[u] = int32_t(i);
}

// Point positions and weights gathered into bin order, so the points of a bin are read
// without the id indirection.
template <class T>
__global__ void bin_order_points_kernel(const int32_t* ids, int64_t m, const T* pos, const T* w, T* spos, T* sw) {
  int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (j >= m) return;
  const int64_t i = ids[j];
  for (int a = 0; a < 3; ++a) spos[3 * j + a] = pos[3 * i + a];
  sw[j] = w[i];
}

template <class T>
struct PointsView {
  const T* pos = nullptr;
  const T* w = nullptr;
  const T* spos = nullptr;          // pos and w in bin order (spos[3j + a] = pos[3 ids[j] + a])
  const T* sw = nullptr;
  const int32_t* ids = nullptr;     // point ids sorted by bin (stable)
  const int32_t* bstart = nullptr;  // per unique bin, start into ids; count+1 entries
  HashView bins;                    // basis key of a bin cell -> unique bin index
};

template <class T>
struct PointsData {
  int64_t m = 0, nbins = 0;
  DBuf<T> pos, w, spos, sw;
  DBuf<int32_t> ids, bstart;
  DBuf<int64_t> bkeys;
  HashMap bins;
  PointsView<T> view() const {
    PointsView<T> v;
    v.pos = pos.p;
    v.w = w.p;
    v.spos = spos.p;
    v.sw = sw.p;
    v.ids = ids.p;
    v.bstart = bstart.p;
    v.bins = bins.view();
    return v;
  }
};

template <class T>
__device__ __forceinline__ T hat3(const T p[3], const int c[3], int depth) {  // screening_stencils.py:28-32
  T h[3];
  for (int a = 0; a < 3; ++a) {
    T t = p[a] * T(1 << depth) - T(c[a]);
    h[a] = dmax(T(1.0) - fabs(t), T(0.0));
  }
  return h[0] * h[1] * h[2];
}

// Float64 screening sums of one row (screening_stencils.py:34-71): acc[k] for the row's
// present slots (slot k = trial function q0 + (k/9, (k/3)%3, k%3)), and the point load.
// Only the eight corners of the point's cell at the trial depth can have a nonzero trial
// hat; every other slot would receive exactly +0.0, so skipping them leaves each
// accumulator's sequence of nonzero additions, and hence its value, unchanged.
template <class T>
// `rin` (optional): the eight cells' point ranges found by an earlier pass over the same row
// (the sliced assembly hands them to the cross term); `rout` (optional) receives them.
__device__ __forceinline__ double screening_row(const PointsView<T>& P, const int c[3], int d, int trial_depth,
                                                const int q0[3], uint32_t present, double acc[27],
                                                const int2* rin = nullptr, int2* rout = nullptr) {
  double rhs = 0.0;
  const int nt = 1 << trial_depth;
  for (int k8 = 0; k8 < 8; ++k8) {
    int2 range = make_int2(0, 0);
    if (rin) {
      range = rin[k8];
    } else {
      int cell[3] = {c[0] - k8 / 4, c[1] - (k8 / 2) % 2, c[2] - k8 % 2};
      if (dmin(cell[0], dmin(cell[1], cell[2])) >= 0 && dmax(cell[0], dmax(cell[1], cell[2])) < (1 << d)) {
        int32_t u = P.bins.find(basis_key(d, cell[0], cell[1], cell[2]));
        if (u >= 0) range = make_int2(P.bstart[u], P.bstart[u + 1]);
      }
      if (rout) rout[k8] = range;
    }
    for (int32_t j = range.x; j < range.y; ++j) {
      T p[3] = {P.spos[3 * j], P.spos[3 * j + 1], P.spos[3 * j + 2]};
      T weight = P.sw[j];
      if (weight == T(0)) continue;
      T phi = hat3(p, c, d);
      rhs += double(phi * weight);
      int f[3];
      for (int a = 0; a < 3; ++a) f[a] = min(max(int(floor(p[a] * T(nt))), 0), nt - 1) - q0[a];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        int s0 = f[0] + e / 4, s1 = f[1] + (e / 2) % 2, s2 = f[2] + e % 2;
        if (s0 < 0 || s0 > 2 || s1 < 0 || s1 > 2 || s2 < 0 || s2 > 2) continue;
        int k = s0 * 9 + s1 * 3 + s2;
        if (!((present >> k) & 1)) continue;
        int q[3] = {q0[0] + s0, q0[1] + s1, q0[2] + s2};
        T trial = hat3(p, q, trial_depth);
        acc[k] += double(phi * trial * weight);
      }
    }
  }
  return rhs;
}

// screening_row for trial functions at the row's own depth, with compile-time slots.  A
// point of the row's k8-th support cell c - o (o = (k8/4, k8/2%2, k8%2)) lies in that cell's
// floor bin (points_kernel bins with the same clamp(floor(p 2^d)) as screening_row), so
// screening_row's f is 1 - o for every such point and its eight trial functions are the
// slots (1 - o) + e, all inside the 3x3x3 window.  With both loops unrolled every acc index is
// a constant and acc stays in registers instead of local memory.  Same contributions, same
// order, same arithmetic as screening_row.
template <class T>
__device__ __forceinline__ double screening_row_same(const PointsView<T>& P, const int c[3], int d, uint32_t present,
                                                     double acc[27], int2* rout) {
  double rhs = 0.0;
#pragma unroll
  for (int k8 = 0; k8 < 8; ++k8) {
    const int o0 = k8 / 4, o1 = (k8 / 2) % 2, o2 = k8 % 2;
    int2 range = make_int2(0, 0);
    const int cell[3] = {c[0] - o0, c[1] - o1, c[2] - o2};
    if (dmin(cell[0], dmin(cell[1], cell[2])) >= 0 && dmax(cell[0], dmax(cell[1], cell[2])) < (1 << d)) {
      int32_t u = P.bins.find(basis_key(d, cell[0], cell[1], cell[2]));
      if (u >= 0) range = make_int2(P.bstart[u], P.bstart[u + 1]);
    }
    if (rout) rout[k8] = range;
    for (int32_t j = range.x; j < range.y; ++j) {
      T p[3] = {P.spos[3 * j], P.spos[3 * j + 1], P.spos[3 * j + 2]};
      T weight = P.sw[j];
      if (weight == T(0)) continue;
      T phi = hat3(p, c, d);
      rhs += double(phi * weight);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int s0 = 1 - o0 + e / 4, s1 = 1 - o1 + (e / 2) % 2, s2 = 1 - o2 + e % 2;
        const int k = s0 * 9 + s1 * 3 + s2;
        if (!((present >> k) & 1)) continue;
        const int q[3] = {c[0] - 1 + s0, c[1] - 1 + s1, c[2] - 1 + s2};
        T trial = hat3(p, q, d);
        acc[k] += double(phi * trial * weight);
      }
    }
  }
  return rhs;
}

// ------------------------------------------------------------------ A5/A7 level assembly
// Same-level operator rows (stiffness.py:38-108 + screening) and b = T(load) + 0.5*T(point load).
template <class T, bool SCREEN>
__global__ void assemble_level_kernel(const int64_t* keys, int64_t n, int d, ColumnView cv, int64_t off,
                                      const double* table, PointsView<T> P, const double* load, int32_t* cols,
                                      T* vals, T* b) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  int32_t col[27];
  uint32_t present = neighbours27(cv, d, c, off, col);
  double acc[27];
  for (int k = 0; k < 27; ++k) acc[k] = 0.0;
  double pl = 0.0;
  if (SCREEN) pl = screening_row_same(P, c, d, present, acc, nullptr);
  for (int k = 0; k < 27; ++k) {
    T v = T(0);
    if (col[k] >= 0) {
      const double* x = table + (c[0] * 3 + k / 9) * 2;
      const double* y = table + (c[1] * 3 + (k / 3) % 3) * 2;
      const double* z = table + (c[2] * 3 + k % 3) * 2;
      double stiff = x[1] * y[0] * z[0] + x[0] * y[1] * z[0] + x[0] * y[0] * z[1];
      v = T(SCREEN ? stiff + acc[k] : stiff);
    }
    cols[i * kSlots + k] = col[k];
    vals[i * kSlots + k] = v;
  }
  cols[i * kSlots + 27] = -1;
  vals[i * kSlots + 27] = T(0);
  b[i] = T(load[i]) + T(0.5) * T(pl);
}

// Same-level operator rows of a sliced level written straight into schedule order: values
// rounded to T then stored as S (float32 storage in the mixed precision), neighbours as
// indices inside their (slice, colour) group (slot 27 = the row's own index), and
// b = T(load) + 0.5*T(point load).
template <class T, class S, class I, bool SCREEN>
__global__ void __launch_bounds__(128, 5) assemble_sliced_kernel(const int64_t* keys, int64_t n, int d, ColumnView cv, int64_t off,
                                       const double* table, PointsView<T> P, const double* load, const int32_t* inv,
                                       const int32_t* group_off, S* svals, I* sidx, T* sb,
                                       int2* ranges_out = nullptr) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  // The neighbours' schedule indices first: the 27 columns are then dead before the
  // screening loop, which needs the registers for its 27 sums (present bit k <=> col[k] >= 0).
  __align__(16) I idx[32];
  uint32_t present;
  {
    int32_t col[27];
    present = neighbours27(cv, d, c, off, col);
#pragma unroll
    for (int k = 0; k < 27; ++k) {
      idx[k] = idx_absent<I>();
      if (col[k] >= 0) {
        int g = 4 * (c[2] + k % 3 - 1) + ((c[0] + k / 9 - 1) & 1) + 2 * ((c[1] + (k / 3) % 3 - 1) & 1);
        idx[k] = I(inv[col[k]] - group_off[g]);
      }
    }
  }
  double acc[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) acc[k] = 0.0;
  double pl = 0.0;
  if (SCREEN) pl = screening_row_same(P, c, d, present, acc, ranges_out ? ranges_out + 8 * i : nullptr);
  const int64_t p = inv[i];
  __align__(16) S v[28];  // written to global memory as 16-byte vectors
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    v[k] = S(0);
    if ((present >> k) & 1) {
      const double* x = table + (c[0] * 3 + k / 9) * 2;
      const double* y = table + (c[1] * 3 + (k / 3) % 3) * 2;
      const double* z = table + (c[2] * 3 + k % 3) * 2;
      double stiff = x[1] * y[0] * z[0] + x[0] * y[1] * z[0] + x[0] * y[0] * z[1];
      v[k] = S(T(SCREEN ? stiff + acc[k] : stiff));
    }
  }
  v[27] = S(0);
  idx[27] = I(p - group_off[4 * c[2] + (c[0] & 1) + 2 * (c[1] & 1)]);
  for (int k = 28; k < 32; ++k) idx[k] = I(-1);
  write_inv_diag<T>(idx, v[13] != S(0) ? T(1.0) / T(v[13]) : T(0));
  int4* vd = reinterpret_cast<int4*>(svals + p * 28);
  const int4* vs = reinterpret_cast<const int4*>(v);
  for (int q = 0; q < 28 * int(sizeof(S)) / 16; ++q) vd[q] = vs[q];
  store_idx_row(sidx + p * 32, p, idx);
  sb[p] = T(load[i]) + T(0.5) * T(pl);
}

// screening_row for the cross term (trial functions at depth d-1), with the sums of the
// current cell kept in registers.  A point of the row's k8-th support cell c - o lies in
// depth-d bin c - o (points_kernel's clamp(floor(p 2^d))) and so in depth-(d-1) bin
// (c - o) >> 1 (p 2^d = 2 (p 2^(d-1)) exactly, floor(2x) >> 1 = floor(x), clamps included):
// screening_row's f is ((c - o) >> 1) - (c >> 1) + 1 for every point of the cell, and the
// cell's points add into the same eight slots f + e.  Those eight running sums are read from
// acc into registers when the cell starts and written back when it ends, so each sum still
// receives the same additions in the same order (same result), and the 27 sums' local memory
// is touched 16 times per cell instead of 8 times per point.
template <class T>
__device__ __forceinline__ void screening_row_cross(const PointsView<T>& P, const int c[3], int d, uint32_t present,
                                                    double acc[27], const int2* rin) {
  const int q0[3] = {(c[0] >> 1) - 1, (c[1] >> 1) - 1, (c[2] >> 1) - 1};
  for (int k8 = 0; k8 < 8; ++k8) {
    const int o[3] = {k8 / 4, (k8 / 2) % 2, k8 % 2};
    int2 range = make_int2(0, 0);
    if (rin) {
      range = rin[k8];
    } else {
      const int cell[3] = {c[0] - o[0], c[1] - o[1], c[2] - o[2]};
      if (dmin(cell[0], dmin(cell[1], cell[2])) >= 0 && dmax(cell[0], dmax(cell[1], cell[2])) < (1 << d)) {
        int32_t u = P.bins.find(basis_key(d, cell[0], cell[1], cell[2]));
        if (u >= 0) range = make_int2(P.bstart[u], P.bstart[u + 1]);
      }
    }
    if (range.x >= range.y) continue;
    int f[3];
    for (int a = 0; a < 3; ++a) f[a] = ((c[a] - o[a]) >> 1) - (c[a] >> 1) + 1;
    int ks[8];
    uint32_t live = 0;
    double r[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int k = (f[0] + e / 4) * 9 + (f[1] + (e / 2) % 2) * 3 + f[2] + e % 2;
      ks[e] = k;
      if ((present >> k) & 1) live |= 1u << e;
      r[e] = acc[k];
    }
    for (int32_t j = range.x; j < range.y; ++j) {
      T p[3] = {P.spos[3 * j], P.spos[3 * j + 1], P.spos[3 * j + 2]};
      T weight = P.sw[j];
      if (weight == T(0)) continue;
      T phi = hat3(p, c, d);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        if (!((live >> e) & 1)) continue;
        const int q[3] = {q0[0] + f[0] + e / 4, q0[1] + f[1] + (e / 2) % 2, q0[2] + f[2] + e % 2};
        T trial = hat3(p, q, d - 1);
        r[e] += double(phi * trial * weight);
      }
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) acc[ks[e]] = r[e];
  }
}

// Cross operator (rows at d, trial functions at d-1; stiffness + screening, rounded to T)
// applied to the coarser cumulative solution: b = b - C cumulative (solver.py:428-446).
// With ccols_out / cvals_out (adjoint tape) the row's cross operator is kept (28 slots).
template <class T, bool SCREEN>
__global__ void __launch_bounds__(128, 6) cross_apply_kernel(const int64_t* keys, int64_t n, int d, ColumnView cv, int64_t coff,
                                   const double* table, PointsView<T> P, const T* cumulative, T* b,
                                   const int32_t* inv, int32_t* ccols_out = nullptr, T* cvals_out = nullptr,
                                   const int2* ranges_in = nullptr) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  int ctr[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
  int32_t col[27];
  uint32_t present = neighbours27(cv, d - 1, ctr, coff, col);
  double acc[27];
  for (int k = 0; k < 27; ++k) acc[k] = 0.0;
  if (SCREEN) screening_row_cross(P, c, d, present, acc, ranges_in ? ranges_in + 8 * i : nullptr);
  T s = T(0);
  for (int k = 0; k < 27; ++k) {
    if (col[k] < 0) {
      if (cvals_out) cvals_out[i * kSlots + k] = T(0);
      continue;
    }
    const double* x = table + (c[0] * 3 + k / 9) * 2;
    const double* y = table + (c[1] * 3 + (k / 3) % 3) * 2;
    const double* z = table + (c[2] * 3 + k % 3) * 2;
    double stiff = x[1] * y[0] * z[0] + x[0] * y[1] * z[0] + x[0] * y[0] * z[1];
    T v = T(SCREEN ? stiff + acc[k] : stiff);
    s = s + v * cumulative[col[k]];
    if (cvals_out) cvals_out[i * kSlots + k] = v;
  }
  if (ccols_out)
    for (int k = 0; k < kSlots; ++k) ccols_out[i * kSlots + k] = k < 27 ? col[k] : -1;
  if (cvals_out) cvals_out[i * kSlots + 27] = T(0);
  const int64_t p = inv ? inv[i] : i;
  b[p] = -s + b[p];
}

// ------------------------------------------------------------------ A9 transfers (transfer_stencils.py:12-66)
template <class T>
__global__ void prolongation_kernel(const int64_t* fine, int64_t n, int d, HashView bh, int64_t coff, int32_t* pcol,
                                    T* pval) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int f[3];
  key_coords(fine[i], f);
  // the parents' weights, then their first hash probes together, collisions after
  T wk[8];
  int64_t key8[8];
  uint64_t h8[8];
  int32_t g8[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int c[3] = {f[0] / 2 + k / 4, f[1] / 2 + (k / 2) % 2, f[2] / 2 + k % 2};
    T h[3];
    for (int a = 0; a < 3; ++a) h[a] = T(1.0) - fabs(T(f[a]) * T(0.5) - T(c[a]));
    wk[k] = h[0] * h[1] * h[2];
    key8[k] = basis_key(d - 1, c[0], c[1], c[2]);
    h8[k] = 0;
    g8[k] = wk[k] > T(0) ? bh.first_probe(key8[k], h8[k]) : -1;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (g8[k] == -2) g8[k] = bh.find_from(key8[k], h8[k]);
  int out = 0;
  for (int k = 0; k < 8; ++k) {
    const T weight = wk[k];
    const int32_t column = g8[k] >= 0 ? int32_t(g8[k] - coff) : -1;
    if (column >= 0) {
      pcol[i * 8 + out] = column;
      pval[i * 8 + out] = weight;
      ++out;
    }
  }
  for (; out < 8; ++out) {
    pcol[i * 8 + out] = -1;
    pval[i * 8 + out] = T(0);
  }
}

// y[i] = (P x)[i] + y[i]  (warp.sparse.bsr_mv with beta = 1)
template <class T>
__global__ void prolong_add_kernel(const int32_t* pcol, const T* pval, int64_t n, const T* x, T* y) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  T s = T(0);
  for (int e = 0; e < 8; ++e) {
    int32_t c = pcol[i * 8 + e];
    if (c < 0) break;
    s = s + pval[i * 8 + e] * x[c];
  }
  y[i] = s + y[i];
}

// ------------------------------------------------------------------ A8 ordered relaxation (relaxation.py)
template <class V>
__device__ __forceinline__ V ld_x(const V* x, int64_t i) { return __ldcg(x + i); }
template <class V>
__device__ __forceinline__ void st_x(V* x, int64_t i, V v) { __stcg(x + i, v); }

// relaxation.py:51-62, one row: r = b_i - sum_k x[c_k] A_k (slot order); x_i += r / A_ii.
// With `rec` (adjoint tape) the row's old x and residual r are stored at rec[0], rec[1].
template <class T, class V>
__device__ __forceinline__ void gs_row(const int32_t* __restrict__ cols, const T* __restrict__ vals,
                                       const V* __restrict__ b, V* x, int32_t row, V* rec = nullptr) {
  const int4* cr = reinterpret_cast<const int4*>(cols + int64_t(row) * kSlots);
  int cc[kSlots];
#pragma unroll
  for (int q = 0; q < kSlots / 4; ++q) {
    int4 v = __ldg(cr + q);
    cc[4 * q] = v.x;
    cc[4 * q + 1] = v.y;
    cc[4 * q + 2] = v.z;
    cc[4 * q + 3] = v.w;
  }
  T aa[kSlots];
  const T* vr = vals + int64_t(row) * kSlots;
#pragma unroll
  for (int q = 0; q < kSlots; ++q) aa[q] = __ldg(vr + q);
  V xs[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) xs[k] = cc[k] >= 0 ? ld_x(x, cc[k]) : V(0);
  V r = b[row];
  T diagonal = T(0);
  V xi = V(0);
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    if (cc[k] < 0) continue;
    r = r - xs[k] * V(aa[k]);
    if (cc[k] == row) {
      diagonal = aa[k];
      xi = xs[k];
    }
  }
  if (rec) {
    rec[0] = xi;
    rec[1] = r;
  }
  if (diagonal != T(0)) st_x(x, row, xi + r * (V(1.0) / V(diagonal)));
}

// One colour phase of the base levels' eight-colour relaxation (relaxation.py:261-271), spread
// over the whole GPU: the rows of colour group g (positions group_off[g] .. group_off[g + 1] of the colour-ordered
// list), one per thread, x in global memory.  Rows of one colour are never each other's
// neighbours, so they update independently, exactly as the threads of
// relax_colors_shared_kernel do between two of its barriers; consecutive launches order the
// phases.  With `hist` (adjoint tape) visit `it` of row i stores (old x, r) at
// hist[2 * (it * n + i)].  The grid covers all n rows (a group never has more), threads past the
// group return at once.
template <class T>
__global__ void relax_phase_kernel(const int32_t* cols, const T* vals, const T* b, T* x, const int32_t* rows,
                                   const int32_t* group_off, int g, int it, T* hist, int64_t n) {
  const int64_t j = group_off[g] + blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (j >= group_off[g + 1]) return;
  const int32_t row = rows[j];
  gs_row(cols, vals, b, x, row, hist ? hist + 2 * (int64_t(it) * n + row) : nullptr);
}

// The same relaxation with x held in shared memory for the whole call (levels whose x fits):
// identical arithmetic and order, without a round trip to L2 per neighbour read.  Every slot
// takes part in the sum: an absent slot (column -1, value +0) reads the +0 entry kept at
// xs_sh[n], and r - (+0 * +0) = r exactly, so the result is bitwise that of skipping it; the
// rows hold their k-th neighbour in slot k, so the diagonal is slot 13.  The unsigned clamp
// keeps every read inside the n + 1 entries.
template <class T>
__device__ __forceinline__ void gs_row_shared(const int32_t* __restrict__ cols, const T* __restrict__ vals,
                                              const T* __restrict__ b, T* xs_sh, int32_t row, T* rec, unsigned n) {
  const int4* cr = reinterpret_cast<const int4*>(cols + int64_t(row) * kSlots);
  __align__(16) int cc[kSlots];
#pragma unroll
  for (int q = 0; q < kSlots / 4; ++q) reinterpret_cast<int4*>(cc)[q] = __ldg(cr + q);
  __align__(16) T aa[kSlots];
  const int4* vr = reinterpret_cast<const int4*>(vals + int64_t(row) * kSlots);
#pragma unroll
  for (int q = 0; q < kSlots * int(sizeof(T)) / 16; ++q) reinterpret_cast<int4*>(aa)[q] = __ldg(vr + q);
  T xs[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) xs[k] = xs_sh[min(unsigned(cc[k]), n)];
  T r = b[row];
#pragma unroll
  for (int k = 0; k < 27; ++k) r = r - xs[k] * T(aa[k]);
  T diagonal = T(0);
  T xi = T(0);
  if (cc[13] == row) {
    diagonal = aa[13];
    xi = xs[13];
  }
  if (rec) {
    rec[0] = xi;
    rec[1] = r;
  }
  if (diagonal != T(0)) xs_sh[row] = xi + r * (T(1.0) / T(diagonal));
}

// The row of schedule position j from a slot-major copy of the operator (slot k of position
// j at k * stride): 27 values v, 27 columns c already clamped to n (absent -> the +0 entry of
// x), and b.  Consecutive threads take consecutive positions, so each slot is one coalesced
// (global) or conflict-free (shared) access per warp.  Same arithmetic and order as
// gs_row_shared.
template <class T>
__device__ __forceinline__ void gs_row_slots(const T* v, const uint16_t* c, int64_t stride, T bj, T* xs_sh, int32_t row,
                                             T* rec) {
  T xv[27], a[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    a[k] = v[k * stride];
    xv[k] = xs_sh[c[k * stride]];
  }
  T r = bj;
#pragma unroll
  for (int k = 0; k < 27; ++k) r = r - xv[k] * a[k];
  T diagonal = T(0);
  T xi = T(0);
  if (c[13 * stride] == unsigned(row)) {
    diagonal = a[13];
    xi = xv[13];
  }
  if (rec) {
    rec[0] = xi;
    rec[1] = r;
  }
  if (diagonal != T(0)) xs_sh[row] = xi + r * (T(1.0) / T(diagonal));
}

// Slot-major copy of a base level's operator in colour order (v[k n + j], c[k n + j] with the
// column clamped to n, bj[j] = b[rows[j]]) for relax_colors_shared_kernel<T, false>.
template <class T>
__global__ void base_slots_kernel(const int32_t* cols, const T* vals, const T* b, const int32_t* rows, int64_t n, T* v,
                                  uint16_t* c, T* bj) {
  const int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (e >= 27 * n) return;
  const int64_t j = e / 27, k = e - 27 * j;
  const int64_t src = int64_t(rows[j]) * kSlots + k;
  v[k * n + j] = vals[src];
  c[k * n + j] = uint16_t(min(unsigned(cols[src]), unsigned(n)));
  if (k == 0) bj[j] = b[rows[j]];
}

// Shared-memory layout of relax_colors_shared_kernel<T, STAGED> for n rows.
template <class T, bool STAGED>
struct BaseRelaxLayout {
  static constexpr size_t bytes(int64_t n) {
    return size_t(n + 1) * sizeof(T) + (STAGED ? size_t(28 * n) * sizeof(T) : 0) + size_t(n + 9) * sizeof(int32_t) +
           (STAGED ? size_t(27 * n) * sizeof(uint16_t) : 0);
  }
};

// One CTA relaxes the whole level for `iters` sweeps over the 8 colours.  Shared memory holds
// x (n + 1 entries, the last a +0 for absent slots), the colour-ordered row list and the 9
// group offsets, so a colour phase starts with one shared-memory read instead of two
// dependent global loads (offsets, then row).  The operator comes slot-major in colour order
// (base_slots_kernel: vT, cT, bT), so the phase's loads are coalesced -- one SM's L1 serves
// them all, and row-major rows cost a wavefront per lane.  STAGED (levels whose operator fits,
// up to ~790 float64 rows) copies every slot into shared memory first, so the 8 x iters phases
// read no global memory; it builds that copy from the row-major operator itself.
template <class T, bool STAGED>
__global__ void __launch_bounds__(1024) relax_colors_shared_kernel(const int32_t* cols, const T* vals, const T* b,
                                                                   const T* vT, const uint16_t* cT, const T* bT, T* x,
                                                                   const int32_t* rows, const int32_t* group_off,
                                                                   int iters, int forward, T* hist, int64_t n) {
  extern __shared__ __align__(16) unsigned char relax_smem[];
  T* xs = reinterpret_cast<T*>(relax_smem);
  T* vs = xs + n + 1;                  // STAGED: 27 n values, slot-major
  T* bs = vs + (STAGED ? 27 * n : 0);  // STAGED: n right-hand sides
  int32_t* rows_s = reinterpret_cast<int32_t*>(bs + (STAGED ? n : 0));
  int32_t* off_s = rows_s + n;
  uint16_t* cs = reinterpret_cast<uint16_t*>(off_s + 9);  // STAGED: 27 n columns, slot-major
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    xs[i] = x[i];
    rows_s[i] = rows[i];
    if (STAGED) bs[i] = b[rows[i]];
  }
  if (STAGED)
    for (int64_t e = threadIdx.x; e < 27 * n; e += blockDim.x) {
      const int64_t j = e / 27, k = e - 27 * j;
      const int64_t src = int64_t(rows[j]) * kSlots + k;
      vs[k * n + j] = vals[src];
      cs[k * n + j] = uint16_t(min(unsigned(cols[src]), unsigned(n)));
    }
  if (threadIdx.x <= 8) off_s[threadIdx.x] = group_off[threadIdx.x];
  if (threadIdx.x == 0) xs[n] = T(0);  // the entry absent slots read
  __syncthreads();
  for (int it = 0; it < iters; ++it)
    for (int cc = 0; cc < 8; ++cc) {
      int g = forward ? cc : 7 - cc;
      for (int j = off_s[g] + threadIdx.x; j < off_s[g + 1]; j += blockDim.x) {
        T* rec = hist ? hist + 2 * (int64_t(it) * n + rows_s[j]) : nullptr;
        if (STAGED)
          gs_row_slots(vs + j, cs + j, n, bs[j], xs, rows_s[j], rec);
        else
          gs_row_slots(vT + j, cT + j, n, __ldg(bT + j), xs, rows_s[j], rec);
      }
      __syncthreads();
    }
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) x[i] = xs[i];
}

constexpr size_t kRelaxSharedBytes = 227 * 1024;  // the opt-in limit of one CTA

// One colour-relaxation call on a small level: shared-memory x when it fits.  1024 threads
// (41 registers each): a depth-4 colour group of ~600 rows is one pass instead of two.
template <class T>
static void relax_colors(const int32_t* cols, const T* vals, const T* b, T* x, const int32_t* rows,
                         const int32_t* group_off, int iters, int forward, T* hist, int64_t n, cudaStream_t s) {
  const size_t bytes = BaseRelaxLayout<T, false>::bytes(n), staged_bytes = BaseRelaxLayout<T, true>::bytes(n);
  // PSR_BASE_RELAX=global keeps x in global memory at any size, =shared never stages the
  // operator rows (test overrides: the paths of larger base levels, on small cases).
  const char* mode = std::getenv("PSR_BASE_RELAX");
  const bool force_global = mode && mode[0] == 'g';
  const bool allow_staged = !(mode && mode[0] == 's');
  // per row visit: 27 columns and values, b, x read and written, row id, and the tape record
  const double visits = double(n) * iters;
  KernelClock clock(kClkBaseRelax, visits * (27.0 * (4 + sizeof(T)) + 3 * sizeof(T) + 4 + (hist ? 2 * sizeof(T) : 0)),
                    visits, s);
  static std::atomic<uint64_t> configured{0};  // per device: the attribute is set per device
  int dev = 0;
  PSR_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = dev < 64 ? uint64_t(1) << dev : 0;
  if (!bit || !(configured.load() & bit)) {
    PSR_CUDA(cudaFuncSetAttribute(relax_colors_shared_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kRelaxSharedBytes)));
    PSR_CUDA(cudaFuncSetAttribute(relax_colors_shared_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kRelaxSharedBytes)));
    configured.fetch_or(bit);
  }
  if (n > 0 && n < 65535 && staged_bytes <= kRelaxSharedBytes && !force_global && allow_staged) {
    relax_colors_shared_kernel<T, true><<<1, 1024, staged_bytes, s>>>(cols, vals, b, nullptr, nullptr, nullptr, x,
                                                                      rows, group_off, iters, forward, hist, n);
  } else if (n > 0 && n < 65535 && bytes <= kRelaxSharedBytes && !force_global) {
    DBuf<T> vT(27 * n, s), bT(n, s);
    DBuf<uint16_t> cT(27 * n, s);
    base_slots_kernel<T><<<blocks_for(27 * n), kThreads, 0, s>>>(cols, vals, b, rows, n, vT.p, cT.p, bT.p);
    PSR_LAUNCH_CHECK();
    relax_colors_shared_kernel<T, false><<<1, 1024, bytes, s>>>(cols, vals, b, vT.p, cT.p, bT.p, x, rows, group_off,
                                                                iters, forward, hist, n);
  } else if (n > 0) {
    // x does not fit one CTA's shared memory: one launch per colour phase, each spread over
    // the GPU (a single CTA would pull every row of the level through one SM's L1).
    for (int it = 0; it < iters; ++it)
      for (int cc = 0; cc < 8; ++cc) {
        relax_phase_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(cols, vals, b, x, rows, group_off,
                                                                 forward ? cc : 7 - cc, it, hist, n);
        PSR_LAUNCH_CHECK();
      }
  }
  PSR_LAUNCH_CHECK();
}

// r = rhs - A x  (bsr_mv alpha=-1, beta=1)
template <class T>
__global__ void residual_kernel(const int32_t* cols, const T* vals, const T* rhs, const T* x, int64_t n, T* r) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  T s = T(0);
  for (int k = 0; k < 27; ++k) {
    int32_t c = cols[i * kSlots + k];
    if (c < 0) continue;
    s = s + vals[i * kSlots + k] * x[c];
  }
  r[i] = -s + rhs[i];
}

// ------------------------------------------------------------------ schedules
__global__ void group_kernel(const int64_t* keys, int64_t n, int sliced, uint32_t* groups, int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  groups[i] = uint32_t(sliced ? (c[0] & 1) + 2 * (c[1] & 1) + 4 * c[2] : (c[0] & 1) + 2 * (c[1] & 1) + 4 * (c[2] & 1));
  ids[i] = int32_t(i);
}

__global__ void group_offsets_kernel(const uint32_t* sorted, int64_t n, int count, int32_t* off) {
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

struct Schedule {
  DBuf<int32_t> rows, off;
  int groups = 0;
};

static Schedule make_schedule(const int64_t* keys, int64_t n, int depth, bool sliced, cudaStream_t s) {
  Schedule S;
  S.groups = sliced ? 4 * ((1 << depth) + 1) : 8;
  DBuf<uint32_t> g(n, s), sg(n, s);
  DBuf<int32_t> ids(n, s);
  S.rows.alloc(n, s);
  S.off.alloc(S.groups + 1, s);
  if (n > 0) {
    group_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, n, sliced, g.p, ids.p);
    PSR_LAUNCH_CHECK();
    sort_pairs(g.p, sg.p, ids.p, S.rows.p, n, bits_for(uint64_t(S.groups)), s);
  }
  group_offsets_kernel<<<blocks_for(S.groups + 1), kThreads, 0, s>>>(sg.p, n, S.groups, S.off.p);
  PSR_LAUNCH_CHECK();
  return S;
}

// ------------------------------------------------------------------ A10 base solve (solver.py:241-317)
// Galerkin R A P on a complete regular level (all nodes of [0, 2^d]^3 present), products
// summed in the fixed order of the oracle's sparse product.
// One 128-thread block per coarse row: the 27 fine rows of R^T are found once (one thread
// each); each of the 125 sums over the fine neighbourhood is one thread (its contributions
// arrive in fine-row order k); each of the 27 coarse slots is one thread summing over the
// fine neighbourhood in order o.
template <class T>
__global__ void __launch_bounds__(128) galerkin_block_kernel(const int64_t* coarse_keys, int64_t nc, int d /*fine*/,
                                                             HashView bh, int64_t foff, int64_t coff,
                                                             const int32_t* fcols, const T* fvals, int32_t* ccols,
                                                             T* cvals) {
  const int64_t i = blockIdx.x;
  if (i >= nc) return;
  __shared__ int64_t s_fr[27];
  __shared__ T s_r[27];
  __shared__ T s_acc[125];
  __shared__ int s_touched[125];
  int c[3];
  key_coords(coarse_keys[i], c);
  const int lim = 1 << d;
  const int tid = threadIdx.x;
  if (tid < 27) {  // rows of R = columns of P: fine nodes 2c + {-1,0,1}^3
    const int k = tid;
    const int f[3] = {2 * c[0] + k / 9 - 1, 2 * c[1] + (k / 3) % 3 - 1, 2 * c[2] + k % 3 - 1};
    int64_t fr = -1;
    T r = T(0);
    if (!(dmin(f[0], dmin(f[1], f[2])) < 0 || dmax(f[0], dmax(f[1], f[2])) > lim)) {
      const int32_t g = bh.find(basis_key(d, f[0], f[1], f[2]));
      if (g >= 0) {
        fr = int64_t(g) - foff;
        T h[3];
        for (int a = 0; a < 3; ++a) h[a] = T(1.0) - fabs(T(f[a]) * T(0.5) - T(c[a]));
        r = h[0] * h[1] * h[2];
      }
    }
    s_fr[k] = fr;
    s_r[k] = r;
  }
  __syncthreads();
  if (tid < 125) {  // fine neighbour j = 2c - 2 + (o / 25, o / 5 % 5, o % 5)
    const int o = tid;
    T a = T(0);
    int touched = 0;
    for (int k = 0; k < 27; ++k) {
      const int64_t fr = s_fr[k];
      if (fr < 0) continue;
      const int ex = o / 25 - k / 9, ey = (o / 5) % 5 - (k / 3) % 3, ez = o % 5 - k % 3;
      if (ex < 0 || ex > 2 || ey < 0 || ey > 2 || ez < 0 || ez > 2) continue;
      const int e = ex * 9 + ey * 3 + ez;
      if (fcols[fr * kSlots + e] < 0) continue;
      a = a + s_r[k] * fvals[fr * kSlots + e];
      touched = 1;
    }
    s_acc[o] = a;
    s_touched[o] = touched;
  }
  __syncthreads();
  if (tid < 27) {  // coarse slot
    const int sk = tid;
    T cs = T(0);
    bool ct = false;
    for (int o = 0; o < 125; ++o) {
      if (!s_touched[o]) continue;
      const int j[3] = {2 * c[0] - 2 + o / 25, 2 * c[1] - 2 + (o / 5) % 5, 2 * c[2] - 2 + o % 5};
      for (int k = 0; k < 8; ++k) {
        const int jj[3] = {j[0] / 2 + k / 4, j[1] / 2 + (k / 2) % 2, j[2] / 2 + k % 2};
        const int sl = (jj[0] - c[0] + 1) * 9 + (jj[1] - c[1] + 1) * 3 + (jj[2] - c[2] + 1);
        if (sl != sk) continue;
        T h[3];
        for (int a = 0; a < 3; ++a) h[a] = T(1.0) - fabs(T(j[a]) * T(0.5) - T(jj[a]));
        const T w = h[0] * h[1] * h[2];
        if (!(w > T(0))) continue;
        if (dmax(jj[0], dmax(jj[1], jj[2])) > (lim >> 1)) continue;
        cs = cs + s_acc[o] * w;
        ct = true;
      }
    }
    int32_t col = -1;
    if (ct) {
      const int q[3] = {c[0] + sk / 9 - 1, c[1] + (sk / 3) % 3 - 1, c[2] + sk % 3 - 1};
      const int32_t g = bh.find(basis_key(d - 1, q[0], q[1], q[2]));
      col = g >= 0 ? int32_t(g - coff) : -1;
    }
    ccols[i * kSlots + sk] = col;
    cvals[i * kSlots + sk] = col >= 0 ? cs : T(0);
  } else if (tid == 27) {
    ccols[i * kSlots + 27] = -1;
    cvals[i * kSlots + 27] = T(0);
  }
}

__device__ __forceinline__ int root_row(int64_t key) {  // solver.py:30-33
  int c[3];
  key_coords(key, c);
  for (int a = 0; a < 3; ++a) c[a] += 2;
  return c[2] * 16 + (c[0] & 1) + 2 * (c[1] & 1) + 2 * (c[0] & 2) + 4 * (c[1] & 2);
}

// Root conjugate gradients (warp.optim.linear.cg stopping rule) on the 8-row depth-0
// system, or on the 64-row padded system with the constant-mode term (solver.py:167-202).
// One thread; dot products sequential in T.
template <class T>
__global__ void root_solve_kernel(const int64_t* keys, int nk, const int32_t* cols, const T* vals, const T* rhs, T* x,
                                  T* root_state, int dc, double cg_accuracy, int base, int cycle) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int N = dc ? 64 : nk;
  T K[64][64];
  unsigned char has[64][64];
  T bb[64], xx[64], r[64], p[64], Ap[64];
  for (int a = 0; a < N; ++a) {
    bb[a] = T(0);
    xx[a] = T(0);
    for (int q = 0; q < N; ++q) {
      K[a][q] = T(0);
      has[a][q] = 0;
    }
  }
  if (dc)
    for (int a = 0; a < N; ++a) xx[a] = root_state[a];
  for (int i = 0; i < nk; ++i) {
    int ri = dc ? root_row(keys[i]) : i;
    bb[ri] = rhs[i];
    if (!dc) xx[ri] = x[i];
    for (int k = 0; k < 27; ++k) {
      int32_t c = cols[i * kSlots + k];
      if (c < 0) continue;
      int rc = dc ? root_row(keys[c]) : c;
      K[ri][rc] = vals[i * kSlots + k];
      has[ri][rc] = 1;
    }
  }
  auto apply = [&](const T* in, const T* y, T* out, int alpha, int beta) {
    T mean = T(0);
    if (dc) {
      for (int a = 0; a < N; ++a) mean = mean + in[a];
      mean = mean / T(N);
    }
    for (int a = 0; a < N; ++a) {
      T s = T(0);
      for (int q = 0; q < N; ++q)
        if (has[a][q]) s = s + K[a][q] * in[q];
      T v = alpha == 1 ? s : -s;
      v = beta == 0 ? v : v + y[a];
      if (dc) v = v + T(alpha) * mean;
      out[a] = v;
    }
  };
  auto dot = [&](const T* u, const T* v) {
    T s = T(0);
    for (int a = 0; a < N; ++a) s = s + u[a] * v[a];
    return s;
  };
  T residual[64];
  for (int a = 0; a < N; ++a) residual[a] = bb[a];
  if (base == 0 && cycle > 0) apply(xx, bb, residual, -1, 1);
  T nsq = dot(residual, residual);
  if (double(nsq) > cg_accuracy * cg_accuracy) {
    double tol = base == 0 ? 0.0 : cg_accuracy;
    double atol = base == 0 ? cg_accuracy * sqrt(double(nsq)) : 0.0;
    double eps = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    double bnorm = sqrt(double(dot(bb, bb)));
    double abs_tol = dmax(dmax(atol, tol * bnorm), pow(eps, 9.0 / 4.0));
    double atol_sq = abs_tol * abs_tol;
    T gate = T(atol_sq);
    apply(xx, bb, r, -1, 1);
    T rr = dot(r, r);
    for (int a = 0; a < N; ++a) p[a] = r[a];
    for (int it = 0; it < nk; ++it) {
      if (double(rr) <= atol_sq) break;
      apply(p, Ap, Ap, 1, 0);
      T pAp = dot(p, Ap);
      T alpha = rr > gate ? rr / pAp : T(0);
      for (int a = 0; a < N; ++a) {
        xx[a] = xx[a] + alpha * p[a];
        r[a] = r[a] - alpha * Ap[a];
      }
      T rr_new = dot(r, r);
      T beta = rr_new > gate ? rr_new / rr : T(0);
      for (int a = 0; a < N; ++a) p[a] = r[a] + beta * p[a];
      rr = rr_new;
    }
  }
  if (dc)
    for (int a = 0; a < N; ++a) root_state[a] = xx[a];
  for (int i = 0; i < nk; ++i) x[i] = xx[dc ? root_row(keys[i]) : i];
}

template <class T>
__global__ void unpermute_kernel(const int32_t* perm, int64_t n, const T* in, T* out) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) out[perm[p]] = in[p];
}

// ------------------------------------------------------------------ adjoint tape of the solve
// What the reverse pass needs from the forward solve, kept only when a reconstruction is
// differentiable.  Everything is in the forward's own layout.
template <class T>
struct SlicedTape {
  bool on = false;
  StripSchedule sched;
  DBuf<char> svals, sidx;  // schedule-order operator rows (float32 values in the mixed precision)
  DBuf<T> b;               // schedule-order right-hand side after the cross term
  DBuf<T> hist;            // n x iters (schedule order): x after each visit
  DBuf<int32_t> ccols;     // cross operator (rows at d, columns at d-1), key order, 28 slots
  DBuf<T> cvals;
};

template <class T>
struct SolveTape {
  int base = 0, top = -1;  // solved depths base..top
  bool screened = false, mixed = false, dc = false;
  std::vector<PointsData<T>> points;        // per depth (screened levels)
  std::vector<DBuf<int32_t>> pcol;          // per depth: prolongation from d-1 (8 slots per fine row)
  std::vector<DBuf<T>> pval;
  std::vector<DBuf<T>> cum;                 // cumulative solution after solving depth d (key order)
  std::vector<SlicedTape<T>> sliced;        // per depth > base
  // base multigrid: level operators (index base = the assembled level, below = Galerkin)
  std::vector<DBuf<int32_t>> mcols;
  std::vector<DBuf<T>> mvals;
  std::vector<Schedule> msched;
  DBuf<T> base_b;
  std::vector<DBuf<T>> relax_hist;          // per colour-relaxation call, in call order
  std::vector<DBuf<T>> resid_x;             // per residual call: x of that level at the time
  std::vector<DBuf<T>> root_x0, root_b;     // per cycle: root CG starting point (64) and right-hand side
};

// ------------------------------------------------------------------ orchestration
struct LevelOp {
  DBuf<int32_t> cols;
  DBuf<char> vals;  // T
};

template <class T>
static PointsData<T> make_points(const DensityData<T>& D, const NormalData<T>& N, const TreeData& tree, int d,
                                 double pw, bool exact, cudaStream_t s) {
  PointsData<T> P;
  int64_t m = D.agg_count[d];
  P.m = m;
  P.pos.alloc(3 * m, s);
  P.w.alloc(m, s);
  HashMap support;
  support.build(tree.support[d].p, tree.support_count[d], s);
  DBuf<uint64_t> bk(m, s), sbk(m, s);
  DBuf<int32_t> ids(m, s);
  P.ids.alloc(m, s);
  if (m) {
    points_kernel<T><<<blocks_for(m), kThreads, 0, s>>>(D.agg_keys[d].p, D.agg_values[d].p, m, d, T(pw), N.average.p,
                                                        support.view(), exact, P.pos.p, P.w.p, bk.p, ids.p);
    PSR_LAUNCH_CHECK();
    int Db = d > 0 ? d : 1;
    sort_pairs(bk.p, sbk.p, ids.p, P.ids.p, m, 3 * Db, s);
  }
  P.spos.alloc(3 * m, s);
  P.sw.alloc(m, s);
  if (m) {
    bin_order_points_kernel<T><<<blocks_for(m), kThreads, 0, s>>>(P.ids.p, m, P.pos.p, P.w.p, P.spos.p, P.sw.p);
    PSR_LAUNCH_CHECK();
  }
  // Unique bins: at most m.  The arrays and the bin hash are sized for m and the hash takes
  // the count from the device, so the count is never read back (a host synchronisation).
  DBuf<int32_t> heads(m, s), prefix(m, s);
  if (m) {
    bin_heads_kernel<<<blocks_for(m), kThreads, 0, s>>>(sbk.p, m, heads.p);
    PSR_LAUNCH_CHECK();
    inclusive_sum(heads.p, prefix.p, m, s);
  }
  P.nbins = m;  // an upper bound; the bins are the first prefix[m - 1] entries
  P.bkeys.alloc(m, s);
  P.bstart.alloc(m + 1, s);
  if (m) {
    bin_fill_kernel<<<blocks_for(m + 1), kThreads, 0, s>>>(sbk.p, heads.p, prefix.p, m, d, P.bkeys.p, P.bstart.p);
    PSR_LAUNCH_CHECK();
    P.bins.build_counted(P.bkeys.p, m, prefix.p + m - 1, s);
  } else {
    P.bins.build(P.bkeys.p, 0, s);
  }
  return P;
}

template <class T>
void solve_levels(const TreeData& tree, const DensityData<T>& D, const NormalData<T>& N,
                  const std::vector<int64_t>& level_offsets, const int64_t* all_keys, const HashMap& all_hash,
                  const Params& p, T* coefficients, cudaStream_t s, SolveStats* stats, StageSink* sink,
                  std::shared_ptr<void>* tape_out) {
  const int finest = p.depth, base = p.base_depth;
  std::shared_ptr<SolveTape<T>> tape_holder;
  SolveTape<T>* tp = nullptr;
  if (tape_out) {
    tape_holder = std::make_shared<SolveTape<T>>();
    tp = tape_holder.get();
    *tape_out = tape_holder;
    tp->base = base;
    tp->points.resize(finest + 1);
    tp->cum.resize(finest + 1);
    tp->sliced.resize(finest + 1);
    tp->mcols.resize(base + 1);
    tp->mvals.resize(base + 1);
  }
  HashView bh = all_hash.view();
  auto keys_at = [&](int d) { return all_keys + level_offsets[d]; };
  auto count_at = [&](int d) { return level_offsets[d + 1] - level_offsets[d]; };
  HashMap nhash;
  nhash.build(N.keys.p, N.count, s);
  HashView nh = nhash.view();
  ColumnIndex ncols, bcols;
  ncols.build(N.keys.p, N.count, finest, s);
  bcols.build(all_keys, level_offsets.back(), finest, s);
  const ColumnView ncv = ncols.view(), bcv = bcols.view();

  // ---- A6 normal loads through the finest depth (normal_loads.py:66-190)
  std::vector<DBuf<double>> same(finest + 1), from_child(finest + 1), from_parent(finest + 1);
  auto stencil = [&](int test_d, int normal_d, const ColumnView& h, int64_t noff, const T* nvals, int64_t nrec,
                     DBuf<double>& out) {
    int64_t n = count_at(test_d);
    out.alloc(n, s);
    out.zero();
    if (!nrec || !n) return;
    int width = test_d < normal_d ? 6 : 4, first = test_d < normal_d ? -3 : -2;
    int res = 1 << test_d;
    DBuf<double> table(int64_t(res + 1) * width * 2, s);
    normal_table_kernel<<<blocks_for(res + 1), kThreads, 0, s>>>(test_d, normal_d, first, width, table.p);
    PSR_LAUNCH_CHECK();
    // test key and load per row; key and 4 values per normal record
    KernelClock clock(kClkNormalStencil, n * 16.0 + nrec * (8.0 + 4 * sizeof(T)), double(n), s);
    if (h.dense && width == 4)
      normal_stencil_dense_kernel<T, 4><<<blocks_for(n), kThreads, 0, s>>>(keys_at(test_d), n, test_d, normal_d, h,
                                                                          noff, nvals, table.p, first, out.p);
    else if (h.dense && width == 6)
      normal_stencil_dense_kernel<T, 6><<<blocks_for(n), kThreads, 0, s>>>(keys_at(test_d), n, test_d, normal_d, h,
                                                                          noff, nvals, table.p, first, out.p);
    else
      normal_stencil_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(keys_at(test_d), n, test_d, normal_d, h, noff,
                                                                  nvals, table.p, width, first, out.p);
    PSR_LAUNCH_CHECK();
  };
  DBuf<T> prev;
  bool has_cumulative = false;
  for (int d = 0; d <= finest; ++d) {
    int64_t nrec = N.offsets[d + 1] - N.offsets[d];
    has_cumulative = has_cumulative || nrec > 0;
    if (d >= base) {
      stencil(d, d, ncv, 0, N.values.p, nrec, same[d]);
      if (d > base) stencil(d - 1, d, ncv, 0, N.values.p, nrec, from_child[d - 1]);
    }
    if (d < finest) {
      int64_t n = count_at(d);
      DBuf<T> cum(4 * n, s);
      if (n) {
        prolong_normals_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(keys_at(d), n, d, nh, N.values.p, bh,
                                                                     d > 0 ? level_offsets[d - 1] : 0, prev.p, cum.p);
        PSR_LAUNCH_CHECK();
      }
      if (d >= base && has_cumulative) stencil(d + 1, d, bcv, level_offsets[d], cum.p, n, from_parent[d + 1]);
      prev = std::move(cum);
    }
  }
  std::vector<DBuf<double>> loads(finest + 1);
  {
    DBuf<double> finer(count_at(finest), s);
    finer.zero();
    for (int d = finest; d >= base; --d) {
      int64_t n = count_at(d);
      loads[d].alloc(n, s);
      if (n) {
        add3_kernel<<<blocks_for(n), kThreads, 0, s>>>(same[d].p, finer.p, from_parent[d].p ? from_parent[d].p : nullptr,
                                                       n, loads[d].p);
        PSR_LAUNCH_CHECK();
      }
      if (d > base) {
        int64_t nc = count_at(d - 1);
        DBuf<double> next(nc, s);
        if (nc) {
          PSR_CUDA(cudaMemcpyAsync(next.p, from_child[d - 1].p, nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
          restrict_add_kernel<T, double><<<blocks_for(nc), kThreads, 0, s>>>(keys_at(d - 1), nc, d, bcv, level_offsets[d],
                                                                             finer.p, next.p, true);
          PSR_LAUNCH_CHECK();
        }
        finer = std::move(next);
      }
    }
  }
  same.clear();
  from_child.clear();
  from_parent.clear();
  prev.release();

  // ---- transfers (solver.py:339-342)
  std::vector<DBuf<int32_t>> pcol(finest + 1);
  std::vector<DBuf<T>> pval(finest + 1);
  for (int d = 1; d <= std::min(finest, p.solve_depth); ++d) {
    int64_t n = count_at(d);
    pcol[d].alloc(8 * n, s);
    pval[d].alloc(8 * n, s);
    if (n) {
      prolongation_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(keys_at(d), n, d, bh, level_offsets[d - 1], pcol[d].p,
                                                                pval[d].p);
      PSR_LAUNCH_CHECK();
    }
  }

  const bool screened = p.point_weight > 0 && !p.exact;
  if (tp) {
    tp->screened = screened;
    tp->mixed = sizeof(T) == 8 && p.precision == 1;
  }
  DBuf<T> cumulative;
  for (int d = base; d <= p.solve_depth; ++d) {
    int64_t n = count_at(d);
    if (!n) break;
    if (tp) tp->top = d;
    PointsData<T> P;
    if (screened) P = make_points(D, N, tree, d, p.point_weight, bool(p.exact), s);
    PointsView<T> pv = screened ? P.view() : PointsView<T>();
    int res = 1 << d;
    DBuf<double> table(int64_t(res + 1) * 6, s);
    stiffness_table_kernel<<<blocks_for(res + 1), kThreads, 0, s>>>(d, d, table.p);
    PSR_LAUNCH_CHECK();
    // The base level keeps key-order rows for its multigrid; finer levels are assembled
    // straight into the schedule order of the strip-scheduled relaxation.
    const bool sliced = d > base;
    const bool mixed = sizeof(T) == 8 && p.precision == 1;
    DBuf<int32_t> cols;
    DBuf<T> vals, b;
    StripSchedule sched;
    DBuf<char> svals, sidx;
    DBuf<int2> cell_ranges;  // the screening cells' point ranges of each row, assembly -> cross term
    if (!sliced) {
      cols.alloc(kSlots * n, s);
      vals.alloc(kSlots * n, s);
      b.alloc(n, s);
      if (screened)
        assemble_level_kernel<T, true><<<blocks_for(n, 128), 128, 0, s>>>(keys_at(d), n, d, bcv, level_offsets[d],
                                                                           table.p, pv, loads[d].p, cols.p, vals.p,
                                                                           b.p);
      else
        assemble_level_kernel<T, false><<<blocks_for(n, 128), 128, 0, s>>>(keys_at(d), n, d, bcv, level_offsets[d],
                                                                            table.p, pv, loads[d].p, cols.p, vals.p,
                                                                            b.p);
      PSR_LAUNCH_CHECK();
    } else {
      build_strip_schedule(keys_at(d), n, d, sched, s);
      if (screened) cell_ranges.alloc(8 * n, s);
      const int sbytes = mixed ? 4 : int(sizeof(T));
      const int ibytes = sched.wide ? 4 : 2;
      svals.alloc(kSlots * n * sbytes, s);
      sidx.alloc(32 * n * ibytes, s);
      b.alloc(n + 4, s);
      b.zero();
      auto launch = [&](auto s_tag, auto i_tag) {
        using S = decltype(s_tag);
        using I = decltype(i_tag);
        S* sv = reinterpret_cast<S*>(svals.p);
        I* si = reinterpret_cast<I*>(sidx.p);
        // key, float64 load, schedule position, operator row, index row, b, screening cell ranges
        const double row_bytes = 8 + 8 + 4 + kSlots * sizeof(S) + 32 * sizeof(I) + sizeof(T) + (screened ? 64 : 0);
        KernelClock clock(kClkAssembleSliced, n * row_bytes + (screened ? P.m * 4.0 * sizeof(T) : 0.0), double(n), s);
        if (screened)
          assemble_sliced_kernel<T, S, I, true><<<blocks_for(n, 128), 128, 0, s>>>(
              keys_at(d), n, d, bcv, level_offsets[d], table.p, pv, loads[d].p, sched.inv.p, sched.off.p, sv, si, b.p,
              cell_ranges.p);
        else
          assemble_sliced_kernel<T, S, I, false><<<blocks_for(n, 128), 128, 0, s>>>(
              keys_at(d), n, d, bcv, level_offsets[d], table.p, pv, loads[d].p, sched.inv.p, sched.off.p, sv, si, b.p);
        PSR_LAUNCH_CHECK();
      };
      if (mixed) {
        if (sched.wide)
          launch(float(), int32_t());
        else
          launch(float(), int16_t());
      } else {
        if (sched.wide)
          launch(T(), int32_t());
        else
          launch(T(), int16_t());
      }
    }
    T* x = coefficients + level_offsets[d];
    PSR_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
    if (sink) sink->put("normal_load_" + std::to_string(d), loads[d].p, n, s);
    if (d == base) {
      // ---- regular multigrid at the base depth (solver.py:241-317)
      std::vector<DBuf<int32_t>> mc(base + 1);
      std::vector<DBuf<T>> mv(base + 1), rhs(base + 1), xs(base + 1);
      std::vector<Schedule> sched(base + 1);
      for (int l = base - 1; l >= 0; --l) {
        int64_t nl = count_at(l);
        mc[l].alloc(kSlots * nl, s);
        mv[l].alloc(kSlots * nl, s);
        const int32_t* fc = l + 1 == base ? cols.p : mc[l + 1].p;
        const T* fv = l + 1 == base ? vals.p : mv[l + 1].p;
        if (nl > 0)
          galerkin_block_kernel<T><<<unsigned(nl), 128, 0, s>>>(keys_at(l), nl, l + 1, bh, level_offsets[l + 1],
                                                                level_offsets[l], fc, fv, mc[l].p, mv[l].p);
        PSR_LAUNCH_CHECK();
      }
      for (int l = 0; l <= base; ++l) {
        int64_t nl = count_at(l);
        sched[l] = make_schedule(keys_at(l), nl, l, false, s);
        if (l < base) {
          rhs[l].alloc(nl, s);
          rhs[l].zero();
          xs[l].alloc(nl, s);
          xs[l].zero();
        }
      }
      auto Cl = [&](int l) { return l == base ? cols.p : mc[l].p; };
      auto Vl = [&](int l) { return l == base ? vals.p : mv[l].p; };
      auto Rl = [&](int l) { return l == base ? b.p : rhs[l].p; };
      auto Xl = [&](int l) { return l == base ? x : xs[l].p; };
      bool dc = base == 0 && p.point_weight == 0;
      DBuf<T> root_state(64, s);
      root_state.zero();
      // Adjoint tape: (old x, r) of every colour-relaxation visit, x at every residual, and
      // the root solve's inputs.
      auto relax_hist = [&](int l) -> T* {
        if (!tp) return nullptr;
        tp->relax_hist.emplace_back(2 * int64_t(p.iters) * count_at(l), s);
        return tp->relax_hist.back().p;
      };
      for (int cycle = 0; cycle < p.base_v_cycles; ++cycle) {
        for (int l = base; l > 0; --l) {
          int64_t nl = count_at(l);
          T* rh = relax_hist(l);
          relax_colors<T>(Cl(l), Vl(l), Rl(l), Xl(l), sched[l].rows.p, sched[l].off.p, p.iters, 1, rh, nl, s);
          if (tp) {
            tp->resid_x.emplace_back(nl, s);
            PSR_CUDA(cudaMemcpyAsync(tp->resid_x.back().p, Xl(l), nl * sizeof(T), cudaMemcpyDeviceToDevice, s));
          }
          DBuf<T> r(nl, s);
          residual_kernel<T><<<blocks_for(nl), kThreads, 0, s>>>(Cl(l), Vl(l), Rl(l), Xl(l), nl, r.p);
          PSR_LAUNCH_CHECK();
          int64_t nc = count_at(l - 1);
          restrict_add_kernel<T, T><<<blocks_for(nc), kThreads, 0, s>>>(keys_at(l - 1), nc, l, bcv, level_offsets[l], r.p,
                                                                        rhs[l - 1].p, false);
          PSR_LAUNCH_CHECK();
          PSR_CUDA(cudaMemsetAsync(xs[l - 1].p, 0, nc * sizeof(T), s));
        }
        if (tp) {
          const int64_t n0 = count_at(0);
          tp->root_b.emplace_back(n0, s);
          PSR_CUDA(cudaMemcpyAsync(tp->root_b.back().p, Rl(0), n0 * sizeof(T), cudaMemcpyDeviceToDevice, s));
          tp->root_x0.emplace_back(64, s);
          tp->root_x0.back().zero();
          if (dc)
            PSR_CUDA(cudaMemcpyAsync(tp->root_x0.back().p, root_state.p, 64 * sizeof(T), cudaMemcpyDeviceToDevice, s));
          else
            PSR_CUDA(cudaMemcpyAsync(tp->root_x0.back().p, Xl(0), n0 * sizeof(T), cudaMemcpyDeviceToDevice, s));
        }
        root_solve_kernel<T><<<1, 32, 0, s>>>(keys_at(0), int(count_at(0)), Cl(0), Vl(0), Rl(0), Xl(0), root_state.p,
                                              dc, p.cg_accuracy, base, cycle);
        PSR_LAUNCH_CHECK();
        for (int l = 1; l <= base; ++l) {
          int64_t nl = count_at(l);
          prolong_add_kernel<T><<<blocks_for(nl), kThreads, 0, s>>>(pcol[l].p, pval[l].p, nl, Xl(l - 1), Xl(l));
          PSR_LAUNCH_CHECK();
          PSR_CUDA(cudaMemsetAsync(xs[l - 1].p, 0, count_at(l - 1) * sizeof(T), s));
          T* rh = relax_hist(l);
          relax_colors<T>(Cl(l), Vl(l), Rl(l), Xl(l), sched[l].rows.p, sched[l].off.p, p.iters, 0, rh, nl, s);
        }
      }
      if (tp) {
        tp->dc = dc;
        tp->mcols[base] = std::move(cols);
        tp->mvals[base] = std::move(vals);
        tp->base_b = std::move(b);
        for (int l = 0; l < base; ++l) {
          tp->mcols[l] = std::move(mc[l]);
          tp->mvals[l] = std::move(mv[l]);
        }
        tp->msched = std::move(sched);
      }
      cumulative.alloc(n, s);
      PSR_CUDA(cudaMemcpyAsync(cumulative.p, x, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
      if (sink) sink->put("rhs_" + std::to_string(d), tp ? tp->base_b.p : b.p, n, s);
    } else {
      DBuf<double> ctable(int64_t(res + 1) * 6, s);
      stiffness_table_kernel<<<blocks_for(res + 1), kThreads, 0, s>>>(d, d - 1, ctable.p);
      PSR_LAUNCH_CHECK();
      DBuf<int32_t> ccols;
      DBuf<T> cvals;
      if (tp) {
        ccols.alloc(kSlots * n, s);
        cvals.alloc(kSlots * n, s);  // every slot written by the cross kernel
      }
      // key, schedule position, b read and written, screening cell ranges, tape row (columns,
      // values), the binned points and the coarser cumulative solution
      KernelClock cross_clock(kClkCrossApply,
                              n * (8.0 + 4 + 2 * sizeof(T) + (screened ? 64 : 0) + (tp ? kSlots * (4.0 + sizeof(T)) : 0)) +
                                  (screened ? P.m * 4.0 * sizeof(T) : 0.0) + count_at(d - 1) * double(sizeof(T)),
                              double(n), s);
      if (screened)
        cross_apply_kernel<T, true><<<blocks_for(n, 128), 128, 0, s>>>(keys_at(d), n, d, bcv, level_offsets[d - 1],
                                                                        ctable.p, pv, cumulative.p, b.p, sched.inv.p,
                                                                        ccols.p, cvals.p, cell_ranges.p);
      else
        cross_apply_kernel<T, false><<<blocks_for(n, 128), 128, 0, s>>>(keys_at(d), n, d, bcv, level_offsets[d - 1],
                                                                         ctable.p, pv, cumulative.p, b.p,
                                                                         sched.inv.p, ccols.p, cvals.p);
      if (tp) {
        tp->sliced[d].ccols = std::move(ccols);
        tp->sliced[d].cvals = std::move(cvals);
      }
      PSR_LAUNCH_CHECK();
      cross_clock.stop();
      if (sink && sink->on) {  // kept in key order, like every other stage
        DBuf<T> kb(n, s);
        unpermute_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(sched.perm.p, n, b.p, kb.p);
        PSR_LAUNCH_CHECK();
        sink->put("rhs_" + std::to_string(d), kb.p, n, s);
      }
      RelaxDeferred deferred;
      RelaxDeferred* dp = nullptr;
      if (stats) {
        deferred = stats->defer(s);
        dp = &deferred;
      }
      float* msp = nullptr;
      DBuf<T> hist;
      if (tp) hist.alloc(int64_t(p.iters) * n, s);
      if (mixed) {
        if (sched.wide)
          relax_strips_scheduled<float, T, int32_t>(sched, reinterpret_cast<const float*>(svals.p),
                                                    reinterpret_cast<const int32_t*>(sidx.p), b.p, x, p.iters, s, msp,
                                                    hist.p, false, false, dp);
        else
          relax_strips_scheduled<float, T, int16_t>(sched, reinterpret_cast<const float*>(svals.p),
                                                    reinterpret_cast<const int16_t*>(sidx.p), b.p, x, p.iters, s, msp,
                                                    hist.p, false, false, dp);
      } else {
        if (sched.wide)
          relax_strips_scheduled<T, T, int32_t>(sched, reinterpret_cast<const T*>(svals.p),
                                                reinterpret_cast<const int32_t*>(sidx.p), b.p, x, p.iters, s, msp,
                                                hist.p, false, false, dp);
        else
          relax_strips_scheduled<T, T, int16_t>(sched, reinterpret_cast<const T*>(svals.p),
                                                reinterpret_cast<const int16_t*>(sidx.p), b.p, x, p.iters, s, msp,
                                                hist.p, false, false, dp);
      }
      if (stats) {  // relax_ms and level_relax_ms are filled by stats->finish()
        stats->row_visits += n * p.iters;
        stats->finest_row_visits = n * p.iters;
        stats->launches += 1;
      }
      DBuf<T> next(n, s);
      PSR_CUDA(cudaMemcpyAsync(next.p, x, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
      prolong_add_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(pcol[d].p, pval[d].p, n, cumulative.p, next.p);
      PSR_LAUNCH_CHECK();
      cumulative = std::move(next);
      if (tp) {
        SlicedTape<T>& st = tp->sliced[d];
        st.on = true;
        st.sched = std::move(sched);
        st.svals = std::move(svals);
        st.sidx = std::move(sidx);
        st.b = std::move(b);
        st.hist = std::move(hist);
      }
    }
    if (tp) {
      tp->cum[d].alloc(n, s);
      PSR_CUDA(cudaMemcpyAsync(tp->cum[d].p, cumulative.p, n * sizeof(T), cudaMemcpyDeviceToDevice, s));
      if (screened) tp->points[d] = std::move(P);
    }
  }
  if (tp) {
    tp->pcol = std::move(pcol);
    tp->pval = std::move(pval);
  }
}

template void solve_levels<float>(const TreeData&, const DensityData<float>&, const NormalData<float>&,
                                  const std::vector<int64_t>&, const int64_t*, const HashMap&, const Params&, float*,
                                  cudaStream_t, SolveStats*, StageSink*, std::shared_ptr<void>*);
template void solve_levels<double>(const TreeData&, const DensityData<double>&, const NormalData<double>&,
                                   const std::vector<int64_t>&, const int64_t*, const HashMap&, const Params&, double*,
                                   cudaStream_t, SolveStats*, StageSink*, std::shared_ptr<void>*);
#include "psr_solve_adjoint.cuh"


}  // namespace psr
