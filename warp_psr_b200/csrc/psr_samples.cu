// A1-A3: sample normalisation and grouping (warp-psr samples.py), degree-2 density and
// splat depths (density.py), normal splat and weighted average (normals.py, keyed.py).
//
// Order-sensitive float sums follow the reference's record order exactly: records are
// grouped with a stable radix sort and every segment is summed serially in record order
// by one thread.  Keys are sorted in a compact form (coordinates packed at `depth` bits)
// that has the same order as the reference's 64-bit keys but needs fewer radix passes.
#include "psr_internal.cuh"

#include <cmath>
#include <limits>

namespace psr {

// ------------------------------------------------------------------ A1 samples.py:34-188
template <class T>
__global__ void bounds_partial_kernel(const T* __restrict__ pos, int64_t n, T* partial, int* status) {
  __shared__ T lo[3][kThreads], hi[3][kThreads];
  T l[3] = {T(INFINITY), T(INFINITY), T(INFINITY)}, h[3] = {T(-INFINITY), T(-INFINITY), T(-INFINITY)};
  int bad = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    T p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    if (isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2])) {
      for (int a = 0; a < 3; ++a) {
        l[a] = dmin(l[a], p[a]);
        h[a] = dmax(h[a], p[a]);
      }
    } else {
      ++bad;
    }
  }
  if (bad) atomicAdd(status, bad);
  for (int a = 0; a < 3; ++a) {
    lo[a][threadIdx.x] = l[a];
    hi[a][threadIdx.x] = h[a];
  }
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int a = 0; a < 3; ++a) {
        lo[a][threadIdx.x] = dmin(lo[a][threadIdx.x], lo[a][threadIdx.x + st]);
        hi[a][threadIdx.x] = dmax(hi[a][threadIdx.x], hi[a][threadIdx.x + st]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int a = 0; a < 3; ++a) {
      partial[6 * blockIdx.x + a] = lo[a][0];
      partial[6 * blockIdx.x + 3 + a] = hi[a][0];
    }
}

// samples.py:54-88 — bounding cube, scale and the cofactor normal scale.
// Bounds over the per-block partials, reduced by one block of kBoundsThreads threads (min and
// max are exact in any grouping, as in the per-block reduction that made the partials).
constexpr int kBoundsThreads = 256;
template <class T>
__device__ void reduce_partials(const T* partial, int blocks, T lo[3], T hi[3]) {
  __shared__ T s_lo[3][kBoundsThreads], s_hi[3][kBoundsThreads];
  T l[3] = {T(INFINITY), T(INFINITY), T(INFINITY)}, h[3] = {T(-INFINITY), T(-INFINITY), T(-INFINITY)};
  for (int b = threadIdx.x; b < blocks; b += blockDim.x)
    for (int a = 0; a < 3; ++a) {
      l[a] = dmin(l[a], partial[6 * b + a]);
      h[a] = dmax(h[a], partial[6 * b + 3 + a]);
    }
  for (int a = 0; a < 3; ++a) {
    s_lo[a][threadIdx.x] = l[a];
    s_hi[a][threadIdx.x] = h[a];
  }
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int a = 0; a < 3; ++a) {
        s_lo[a][threadIdx.x] = dmin(s_lo[a][threadIdx.x], s_lo[a][threadIdx.x + st]);
        s_hi[a][threadIdx.x] = dmax(s_hi[a][threadIdx.x], s_hi[a][threadIdx.x + st]);
      }
    __syncthreads();
  }
  for (int a = 0; a < 3; ++a) {
    lo[a] = s_lo[a][0];
    hi[a] = s_hi[a][0];
  }
}

template <class T>
__global__ void __launch_bounds__(kBoundsThreads) transform_kernel(const T* partial, int blocks, T scale, T* transform,
                                                                   int* status) {
  T lo[3], hi[3];
  reduce_partials(partial, blocks, lo, hi);
  if (threadIdx.x != 0) return;
  T width = dmax(hi[0] - lo[0], dmax(hi[1] - lo[1], hi[2] - lo[2])) * scale;
  if (!isfinite(width) || width <= T(0)) {
    status[0] += 1;
    return;
  }
  T inv = T(1.0 / double(width));
  transform[0] = inv;
  T determinant = inv * (inv * inv);
  transform[4] = inv * inv / determinant * T(pow(double(determinant), 1.0 / 3.0));
  for (int a = 0; a < 3; ++a) {
    int axis = (a + 1) % 3;
    T origin = (hi[axis] + lo[axis]) / T(2.0) - width / T(2.0);
    transform[a + 1] = -origin * inv;
  }
}

// samples.py:90-134 — cyclic axis permutation, unit normals, left-owned leaf cell.
template <class T>
__global__ void classify_kernel(const T* __restrict__ pos, const T* __restrict__ nrm, int64_t n,
                                const T* __restrict__ transform, int depth, T* q, T* un, uint64_t* keys,
                                int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  T inv = transform[0], ns = transform[4];
  const T* p = pos + 3 * i;
  const T* m = nrm + 3 * i;
  T qq[3] = {p[1] * inv + transform[1], p[2] * inv + transform[2], p[0] * inv + transform[3]};
  T mm[3] = {m[1] * ns, m[2] * ns, m[0] * ns};
  T length2 = mm[0] * mm[0] + mm[1] * mm[1] + mm[2] * mm[2];
  for (int a = 0; a < 3; ++a) q[3 * i + a] = qq[a];
  ids[i] = int32_t(i);
  uint64_t key = uint64_t(1) << (3 * depth);
  T u[3] = {T(0), T(0), T(0)};
  if (length2 > T(0) && isfinite(length2) && dmin(qq[0], dmin(qq[1], qq[2])) >= T(0) &&
      dmax(qq[0], dmax(qq[1], qq[2])) <= T(1)) {
    T len = sqrt(length2);
    for (int a = 0; a < 3; ++a) u[a] = mm[a] / len;
    int res = 1 << depth;
    key = (uint64_t(ceil_cell(qq[0], res)) << (2 * depth)) | (uint64_t(ceil_cell(qq[1], res)) << depth) |
          uint64_t(ceil_cell(qq[2], res));
  }
  for (int a = 0; a < 3; ++a) un[3 * i + a] = u[a];
  keys[i] = key;
}

// head[i] = 1 where a new valid segment of `keys >> shift` starts (32- or 64-bit keys).
template <class K>
__global__ void heads_kernel(const K* __restrict__ keys, int64_t n, uint64_t sentinel, int shift, int32_t* heads) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = uint64_t(keys[i]) >> shift;
  heads[i] = (uint64_t(keys[i]) < sentinel && (i == 0 || (uint64_t(keys[i - 1]) >> shift) != k)) ? 1 : 0;
}

template <class T>
__global__ void groups_kernel(const uint64_t* __restrict__ keys, const int32_t* __restrict__ order,
                              const int32_t* __restrict__ heads, const int32_t* __restrict__ prefix, int64_t n,
                              const T* __restrict__ q, const T* __restrict__ un, int depth, int64_t* gkeys,
                              T* sums, T* nsums, T* weights, int32_t* first) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n || !heads[i]) return;
  int64_t g = prefix[i] - 1;
  uint64_t k = keys[i];
  T p[3] = {T(0), T(0), T(0)}, m[3] = {T(0), T(0), T(0)}, w = T(0);
  for (int64_t j = i; j < n && keys[j] == k; ++j) {
    int64_t o = order[j];
    for (int a = 0; a < 3; ++a) {
      p[a] = p[a] + q[3 * o + a];
      m[a] = m[a] + un[3 * o + a];
    }
    w = w + T(1.0);
  }
  uint64_t mask = (uint64_t(1) << depth) - 1;
  gkeys[g] = basis_key(depth, int((k >> (2 * depth)) & mask), int((k >> depth) & mask), int(k & mask));
  for (int a = 0; a < 3; ++a) {
    sums[3 * g + a] = p[a];
    nsums[3 * g + a] = m[a];
  }
  weights[g] = w;
  first[g] = order[i];
}

// Adjoint bookkeeping: bounding box and the lowest input index attaining each bound.
template <class T>
__global__ void __launch_bounds__(kBoundsThreads) bounds_final_kernel(const T* partial, int blocks, T* bounds) {
  T lo[3], hi[3];
  reduce_partials(partial, blocks, lo, hi);
  if (threadIdx.x != 0) return;
  for (int a = 0; a < 3; ++a) {
    bounds[a] = lo[a];
    bounds[3 + a] = hi[a];
  }
}

template <class T>
__global__ void bound_owner_kernel(const T* __restrict__ pos, int64_t n, const T* bounds, int32_t* owner) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  T p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  if (!(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]))) return;
  for (int a = 0; a < 3; ++a) {
    if (p[a] == bounds[a]) atomicMin(owner + a, int32_t(i));
    if (p[a] == bounds[3 + a]) atomicMin(owner + 3 + a, int32_t(i));
  }
}

// Group of every input point (-1 for points rejected by the classification).
__global__ void input_group_kernel(const uint64_t* __restrict__ keys, const int32_t* __restrict__ order,
                                   const int32_t* __restrict__ prefix, int64_t n, uint64_t sentinel, int32_t* group) {
  int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (j >= n) return;
  group[order[j]] = keys[j] < sentinel ? prefix[j] - 1 : -1;
}

// Marks segment heads of sorted keys and returns the number of segments.
template <class K>
static int64_t segment_heads(const K* keys, int64_t n, uint64_t sentinel, int shift, DBuf<int32_t>& heads,
                             DBuf<int32_t>& prefix, cudaStream_t s) {
  heads.alloc(n, s);
  prefix.alloc(n, s);
  if (n == 0) return 0;
  heads_kernel<K><<<blocks_for(n), kThreads, 0, s>>>(keys, n, sentinel, shift, heads.p);
  PSR_LAUNCH_CHECK();
  inclusive_sum(heads.p, prefix.p, n, s);
  return read_scalar(prefix.p + n - 1, s);
}

template <class T>
SampleGroups<T> prepare_samples(const T* pos, const T* nrm, int64_t n, int depth, double scale, cudaStream_t s,
                                bool keep) {
  SampleGroups<T> G;
  int blocks = int(blocks_for(n) < 592 ? blocks_for(n) : 592);
  DBuf<T> partial(6 * blocks, s);
  DBuf<int> status(1, s);
  status.zero();
  G.transform.alloc(5, s);
  G.transform.zero();
  bounds_partial_kernel<T><<<blocks, kThreads, 0, s>>>(pos, n, partial.p, status.p);
  PSR_LAUNCH_CHECK();
  transform_kernel<T><<<1, kBoundsThreads, 0, s>>>(partial.p, blocks, T(scale), G.transform.p, status.p);
  PSR_LAUNCH_CHECK();
  if (read_scalar(status.p, s)) throw Error(3, "Nonfinite positions or degenerate/overflowing bounding cube");
  if (keep) {
    G.bounds.alloc(6, s);
    bounds_final_kernel<T><<<1, kBoundsThreads, 0, s>>>(partial.p, blocks, G.bounds.p);
    PSR_LAUNCH_CHECK();
    G.bound_owner.alloc(6, s);
    PSR_CUDA(cudaMemsetAsync(G.bound_owner.p, 0x7f, 6 * sizeof(int32_t), s));
    bound_owner_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(pos, n, G.bounds.p, G.bound_owner.p);
    PSR_LAUNCH_CHECK();
  }
  DBuf<T> q(3 * n, s), un(3 * n, s);
  DBuf<uint64_t> keys(n, s), skeys(n, s);
  DBuf<int32_t> ids(n, s), order(n, s);
  classify_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(pos, nrm, n, G.transform.p, depth, q.p, un.p, keys.p, ids.p);
  PSR_LAUNCH_CHECK();
  sort_pairs(keys.p, skeys.p, ids.p, order.p, n, 3 * depth + 1, s);
  DBuf<int32_t> heads, prefix;
  uint64_t sentinel = uint64_t(1) << (3 * depth);
  int64_t count = segment_heads(skeys.p, n, sentinel, 0, heads, prefix, s);
  if (!count) throw Error(3, "No accepted samples with finite nonzero normals");
  G.count = count;
  G.keys.alloc(count, s);
  G.sums.alloc(3 * count, s);
  G.normal_sums.alloc(3 * count, s);
  G.weights.alloc(count, s);
  G.first.alloc(count, s);
  groups_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(skeys.p, order.p, heads.p, prefix.p, n, q.p, un.p, depth,
                                                      G.keys.p, G.sums.p, G.normal_sums.p, G.weights.p, G.first.p);
  PSR_LAUNCH_CHECK();
  if (keep) {
    G.input_group.alloc(n, s);
    input_group_kernel<<<blocks_for(n), kThreads, 0, s>>>(skeys.p, order.p, prefix.p, n, sentinel, G.input_group.p);
    PSR_LAUNCH_CHECK();
  }
  return G;
}

// ------------------------------------------------------------------ A2 density.py:25-279
template <class T>
T density_scale() {  // density.py:37-50 (a constant of the precision)
  T total = T(0);
  T dx = T(0.1);
  for (int x = 0; x < 10; ++x) {
    T p = dx / T(2.0) + dx * T(x);
    double xd = double(p);
    double b0 = (1.0 - xd) * (1.0 - xd) * 0.5;
    double b1 = ((1.0 - xd) * (xd + 1.0) + xd * (2.0 - xd)) * 0.5;
    double b2 = xd * xd * 0.5;
    T sc = T(1.0 / (b0 * b0 + b1 * b1 + b2 * b2));
    for (int y = 0; y < 100; ++y) total = total + sc;
  }
  return total / T(1000.0);
}

template <class T>
__global__ void leaf_values_kernel(const T* sums, const T* weights, int64_t n, T* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  for (int a = 0; a < 3; ++a) out[4 * i + a] = sums[3 * i + a];
  out[4 * i + 3] = weights[i];
}

// Children of depth d sorted by (parent cell, morton child index): the order in which
// density.py:228-240 (morton order, then a stable sort by parent key) sums them.
__global__ void parent_composite_kernel(const int64_t* keys, int64_t n, int d, uint64_t* comp, int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  int D = d - 1;
  uint64_t parent = (uint64_t(c[0] >> 1) << (2 * D)) | (uint64_t(c[1] >> 1) << D) | uint64_t(c[2] >> 1);
  comp[i] = (parent << 3) | uint64_t((c[0] & 1) | ((c[1] & 1) << 1) | ((c[2] & 1) << 2));
  ids[i] = int32_t(i);
}

template <class T>
__global__ void parent_reduce_kernel(const uint64_t* comp, const int32_t* order, const int32_t* heads,
                                     const int32_t* prefix, int64_t n, const T* values, int d, int64_t* out_keys,
                                     T* out_values) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n || !heads[i]) return;
  int64_t g = prefix[i] - 1;
  uint64_t parent = comp[i] >> 3;
  T acc[4] = {T(0), T(0), T(0), T(0)};
  for (int64_t j = i; j < n && (comp[j] >> 3) == parent; ++j)
    for (int a = 0; a < 4; ++a) acc[a] = acc[a] + values[4 * int64_t(order[j]) + a];
  int D = d - 1;
  uint64_t mask = (uint64_t(1) << D) - 1;
  out_keys[g] = basis_key(D, int((parent >> (2 * D)) & mask), int((parent >> D) & mask), int(parent & mask));
  for (int a = 0; a < 4; ++a) out_values[4 * g + a] = acc[a];
}

__global__ void morton_kernel(const int64_t* keys, int64_t n, int d, uint64_t* codes, int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  uint64_t m = 0;  // keyed.py:23-30
  for (int bit = 0; bit < d; ++bit)
    for (int a = 0; a < 3; ++a) m |= uint64_t((c[a] >> bit) & 1) << (3 * bit + a);
  codes[i] = m;
  ids[i] = int32_t(i);
}

// density.py:74-107 — 27 degree-2 splat records per occupied cell, in morton order.
template <class T, class K>
__global__ void density_splat_kernel(const int64_t* keys, const T* values, const int32_t* order, int64_t m, int d,
                                     T scale, K* rkeys, int32_t* rids, T* rvals) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  int64_t j = order[i];
  int c[3];
  key_coords(keys[j], c);
  const T* v = values + 4 * j;
  int n = 1 << d;
  T p[3] = {v[0] / v[3], v[1] / v[3], v[2] / v[3]};
  T h = T(1.0) / T(n);
  double b[3][3];
  for (int a = 0; a < 3; ++a) quadratic(double((p[a] - T(c[a]) * h) / h), b[a]);
  T weight = v[3] * scale;
  int D = d > 0 ? d : 1;
  uint64_t sentinel = uint64_t(1) << (3 * D);
  for (int k = 0; k < 27; ++k) {
    int x = k / 9, y = k / 3 % 3, z = k % 3;
    int t[3] = {c[0] + x - 1, c[1] + y - 1, c[2] + z - 1};
    int64_t r = 27 * i + k;
    rids[r] = int32_t(r);
    if (dmin(t[0], dmin(t[1], t[2])) >= 0 && dmax(t[0], dmax(t[1], t[2])) < n) {
      rkeys[r] = K((uint64_t(t[0]) << (2 * D)) | (uint64_t(t[1]) << D) | uint64_t(t[2]));
      rvals[r] = T(double(weight) * b[0][x] * b[1][y] * b[2][z]);
    } else {
      rkeys[r] = K(sentinel);
      rvals[r] = T(0);
    }
  }
}

template <class T, class K>
__global__ void scalar_reduce_kernel(const K* keys, const int32_t* order, const int32_t* heads,
                                     const int32_t* prefix, int64_t n, const T* values, int d, int D,
                                     int64_t* out_keys, T* out_values) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n || !heads[i]) return;
  int64_t g = prefix[i] - 1;
  const K k = keys[i];
  T acc = T(0);
  for (int64_t j = i; j < n && keys[j] == k; ++j) acc = acc + values[order[j]];
  uint64_t mask = (uint64_t(1) << D) - 1;
  out_keys[g] = basis_key(d, int((k >> (2 * D)) & mask), int((k >> D) & mask), int(k & mask));
  out_values[g] = acc;
}

// density.py:108-150 — density at every group centroid for level d.
template <class T>
__global__ void density_eval_kernel(HashView h, const T* lvals, const T* sums, const T* weights, int64_t G, int d,
                                    int stride, T* dens) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= G) return;
  T w = weights[i];
  T p[3] = {sums[3 * i] / w, sums[3 * i + 1] / w, sums[3 * i + 2] / w};
  int n = 1 << d;
  int c[3] = {ceil_cell(p[0], n), ceil_cell(p[1], n), ceil_cell(p[2], n)};
  T hh = T(1.0) / T(n);
  double b[3][3];
  for (int a = 0; a < 3; ++a) quadratic(double((p[a] - T(c[a]) * hh) / hh), b[a]);
  T value = T(0);
  // per x-plane, the nine first hash probes issued together (collisions resolved after); the
  // sum still runs in slot order
  for (int x = 0; x < 3; ++x) {
    int64_t key9[9];
    uint64_t h9[9];
    int32_t idx9[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const int y = q / 3, z = q % 3;
      const int t[3] = {c[0] + x - 1, c[1] + y - 1, c[2] + z - 1};
      const bool inside = dmin(t[0], dmin(t[1], t[2])) >= 0 && dmax(t[0], dmax(t[1], t[2])) < n;
      key9[q] = basis_key(d, t[0], t[1], t[2]);
      h9[q] = 0;
      idx9[q] = inside ? h.first_probe(key9[q], h9[q]) : -1;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q)
      if (idx9[q] == -2) idx9[q] = h.find_from(key9[q], h9[q]);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const int y = q / 3, z = q % 3;
      if (idx9[q] >= 0) value = value + T(b[0][x] * b[1][y] * b[2][z] * double(lvals[idx9[q]]));
    }
  }
  dens[i * stride + d] = value;
}

// density.py:152-182 — raw splat depth and weight.
template <class T>
__global__ void depths_kernel(const T* dens, int64_t G, int kernel_depth, T target, T* dw) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= G) return;
  int stride = kernel_depth + 1;
  int d = kernel_depth;
  T density = dens[i * stride + d];
  T raw;
  if (density >= target) {
    raw = T(double(d) + double(T(log(double(density / target)))) / (log(2.0) * 2.0));
  } else {
    T fine = density;
    while (density < target && d > 0) {
      fine = density;
      d -= 1;
      density = dens[i * stride + d];
    }
    raw = T(T(d) + T(log(double(density / target))) / T(log(double(density / fine))));
  }
  T h = T(1.0) / T(1 << d);
  dw[2 * i] = raw;
  dw[2 * i + 1] = h * h / density;
}

// Adjoint bookkeeping: map every sorted record to its segment (unique key) index.
template <class K>
__global__ void segment_slot_kernel(const int32_t* order, const int32_t* prefix, const K* skeys, int64_t n,
                                    uint64_t sentinel, int shift, int32_t* slot) {
  int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (j >= n) return;
  slot[order[j]] = (uint64_t(skeys[j]) >> shift) < (sentinel >> shift) ? prefix[j] - 1 : -1;
}

template <class T>
DensityData<T> build_density(const SampleGroups<T>& g, int depth, int kernel_depth, double spn, cudaStream_t s,
                             bool keep) {
  DensityData<T> D;
  if (keep) {
    D.parent_of.resize(depth + 1);
    D.splat_order.resize(kernel_depth + 1);
    D.splat_slot.resize(kernel_depth + 1);
    D.level_values.resize(kernel_depth + 1);
    D.level_hash.resize(kernel_depth + 1);
  }
  int64_t G = g.count;
  D.agg_keys.resize(depth + 1);
  D.agg_values.resize(depth + 1);
  D.agg_count.assign(depth + 1, 0);
  D.agg_keys[depth].alloc(G, s);
  PSR_CUDA(cudaMemcpyAsync(D.agg_keys[depth].p, g.keys.p, G * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
  D.agg_values[depth].alloc(4 * G, s);
  D.agg_count[depth] = G;
  leaf_values_kernel<T><<<blocks_for(G), kThreads, 0, s>>>(g.sums.p, g.weights.p, G, D.agg_values[depth].p);
  PSR_LAUNCH_CHECK();
  for (int d = depth; d > 0; --d) {
    int64_t n = D.agg_count[d];
    DBuf<uint64_t> comp(n, s), scomp(n, s);
    DBuf<int32_t> ids(n, s), order(n, s);
    parent_composite_kernel<<<blocks_for(n), kThreads, 0, s>>>(D.agg_keys[d].p, n, d, comp.p, ids.p);
    PSR_LAUNCH_CHECK();
    sort_pairs(comp.p, scomp.p, ids.p, order.p, n, 3 * d, s);
    DBuf<int32_t> heads, prefix;
    int64_t m = segment_heads(scomp.p, n, ~uint64_t(0), 3, heads, prefix, s);
    D.agg_count[d - 1] = m;
    D.agg_keys[d - 1].alloc(m, s);
    D.agg_values[d - 1].alloc(4 * m, s);
    parent_reduce_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(scomp.p, order.p, heads.p, prefix.p, n,
                                                               D.agg_values[d].p, d, D.agg_keys[d - 1].p,
                                                               D.agg_values[d - 1].p);
    PSR_LAUNCH_CHECK();
    if (keep) {
      D.parent_of[d].alloc(n, s);
      segment_slot_kernel<<<blocks_for(n), kThreads, 0, s>>>(order.p, prefix.p, scomp.p, n, ~uint64_t(0), 0,
                                                             D.parent_of[d].p);
      PSR_LAUNCH_CHECK();
    }
  }
  D.scale = density_scale<T>();
  DBuf<T> dens(G * (kernel_depth + 1), s);
  for (int d = 0; d <= kernel_depth; ++d) {
    int64_t m = D.agg_count[d];
    DBuf<uint64_t> codes(m, s), scodes(m, s);
    DBuf<int32_t> ids(m, s), order(m, s);
    morton_kernel<<<blocks_for(m), kThreads, 0, s>>>(D.agg_keys[d].p, m, d, codes.p, ids.p);
    PSR_LAUNCH_CHECK();
    sort_pairs(codes.p, scodes.p, ids.p, order.p, m, d > 0 ? 3 * d : 1, s);
    int64_t r = 27 * m;
    DBuf<int32_t> rids(r, s), rorder(r, s);
    DBuf<T> rvals(r, s);
    int Db = d > 0 ? d : 1;
    DBuf<int32_t> heads, prefix;
    DBuf<int64_t> lkeys;
    DBuf<T> lvals;
    int64_t u = 0;
    // Record keys of 3 Db + 1 bits: 32-bit keys while they fit (a third less data through the
    // sort's passes), else 64-bit.  Same keys, same stable order either way.
    auto splat_reduce = [&](auto key_tag) {
      using K = decltype(key_tag);
      DBuf<K> rkeys(r, s), skeys(r, s);
      density_splat_kernel<T, K><<<blocks_for(m), kThreads, 0, s>>>(D.agg_keys[d].p, D.agg_values[d].p, order.p, m,
                                                                    d, D.scale, rkeys.p, rids.p, rvals.p);
      PSR_LAUNCH_CHECK();
      sort_pairs(rkeys.p, skeys.p, rids.p, rorder.p, r, 3 * Db + 1, s);
      u = segment_heads(skeys.p, r, uint64_t(1) << (3 * Db), 0, heads, prefix, s);
      lkeys.alloc(u, s);
      lvals.alloc(u, s);
      scalar_reduce_kernel<T, K><<<blocks_for(r), kThreads, 0, s>>>(skeys.p, rorder.p, heads.p, prefix.p, r, rvals.p,
                                                                    d, Db, lkeys.p, lvals.p);
      PSR_LAUNCH_CHECK();
      if (keep) {
        D.splat_slot[d].alloc(r, s);
        segment_slot_kernel<<<blocks_for(r), kThreads, 0, s>>>(rorder.p, prefix.p, skeys.p, r,
                                                               uint64_t(1) << (3 * Db), 0, D.splat_slot[d].p);
        PSR_LAUNCH_CHECK();
      }
    };
    if (3 * Db + 1 <= 32)
      splat_reduce(uint32_t());
    else
      splat_reduce(uint64_t());
    HashMap hm;
    hm.build(lkeys.p, u, s);
    density_eval_kernel<T><<<blocks_for(G), kThreads, 0, s>>>(hm.view(), lvals.p, g.sums.p, g.weights.p, G, d,
                                                              kernel_depth + 1, dens.p);
    PSR_LAUNCH_CHECK();
    if (keep) {
      D.splat_order[d] = std::move(order);
      D.level_values[d] = std::move(lvals);
      D.level_hash[d] = std::move(hm);
    }
  }
  D.dw.alloc(2 * G, s);
  depths_kernel<T><<<blocks_for(G), kThreads, 0, s>>>(dens.p, G, kernel_depth, T(spn), D.dw.p);
  PSR_LAUNCH_CHECK();
  if (keep) D.densities = std::move(dens);
  return D;
}

// ------------------------------------------------------------------ A3 normals.py:33-245
__global__ void first_keys_kernel(const int32_t* first, int64_t n, uint32_t* keys, int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  keys[i] = uint32_t(first[i]);
  ids[i] = int32_t(i);
}

// normals.py:46-104 — 54 records per group: two 27-node degree-2 splats on the same
// node `top` (issue #12), weighted by dx and 1-dx.
// The per-group part of the normal splat: the unit normal times the weight, the splat depth
// and its two fractions, the cell and the 3 x 3 quadratic B-spline weights.
template <class T>
struct SplatGroup {
  T nm[3], dx, h, sw;
  double b[3][3];
  int c[3], top, nn, valid, second;
};

// One thread per record (54 per sample): neighbouring threads write neighbouring records.  A
// block's records span at most six samples; their per-sample values (two divisions and a
// square root per component, the B-spline weights) are computed once per sample by the
// block's first threads into shared memory instead of once per record.  Same arithmetic:
// same records.
template <class T, class K>
__global__ void __launch_bounds__(kThreads) normal_splat_kernel(const int32_t* order, int64_t n, const T* sums,
                                                                const T* nsums, const T* weights, const T* dw,
                                                                int minimum, int maximum, K* rkeys, int32_t* rids,
                                                                T* rvals) {
  constexpr int kGroups = (kThreads + 53) / 54 + 1;  // samples a block's records can touch
  __shared__ SplatGroup<T> sg[kGroups];
  const int64_t r0 = blockIdx.x * int64_t(blockDim.x);
  const int64_t i0 = r0 / 54;
  if (threadIdx.x < kGroups) {
    const int64_t i = i0 + threadIdx.x;
    SplatGroup<T>& G = sg[threadIdx.x];
    G.valid = 0;
    if (i < n && i * 54 < r0 + blockDim.x) {
      int64_t src = order[i];
      T w = weights[src];
      T nm[3] = {nsums[3 * src] / w, nsums[3 * src + 1] / w, nsums[3 * src + 2] / w};
      T length = sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
      if (length > T(0)) {
        for (int a = 0; a < 3; ++a) G.nm[a] = nm[a] / length * w;
        T p[3] = {sums[3 * src] / w, sums[3 * src + 1] / w, sums[3 * src + 2] / w};
        T depth = dmin(dmax(dw[2 * src], T(minimum)), T(maximum));
        int top = int(ceil(depth));
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
        for (int a = 0; a < 3; ++a) {
          G.c[a] = ceil_cell(p[a], nn);
          quadratic(double((p[a] - T(G.c[a]) * h) / h), G.b[a]);
        }
        G.top = top;
        G.nn = nn;
        G.dx = dx;
        G.h = h;
        G.second = fabs(1.0 - double(dx)) > 1e-06;
        G.sw = dw[2 * src + 1];
        G.valid = 1;
      }
    }
  }
  __syncthreads();
  const int64_t r = r0 + threadIdx.x;
  if (r >= 54 * n) return;
  const int64_t i = r / 54;
  const int k = int(r % 54);
  int D = maximum > 0 ? maximum : 1;
  uint64_t sentinel = uint64_t(1) << (3 * D + 4);
  rkeys[r] = K(sentinel);
  rids[r] = int32_t(r);
  const SplatGroup<T>& G = sg[i - i0];
  if (!G.valid) return;
  if (k >= 27 && !G.second) return;
  T fraction = k < 27 ? G.dx : T(1.0) - G.dx;
  int q = k % 27;
  int x = q / 9, y = q / 3 % 3, z = q % 3;
  int t[3] = {G.c[0] + x - 1, G.c[1] + y - 1, G.c[2] + z - 1};
  if (dmin(t[0], dmin(t[1], t[2])) >= 0 && dmax(t[0], dmax(t[1], t[2])) < G.nn) {
    T bw = T(G.b[0][x] * G.b[1][y] * G.b[2][z]);
    const T h = G.h;
    rkeys[r] = K((uint64_t(G.top) << (3 * D)) | (uint64_t(t[0]) << (2 * D)) | (uint64_t(t[1]) << D) | uint64_t(t[2]));
    for (int a = 0; a < 3; ++a) rvals[3 * r + a] = G.nm[a] * G.sw / (h * h * h) * fraction * bw;
  }
}

template <class T, class K>
__global__ void normal_reduce_kernel(const K* keys, const int32_t* order, const int32_t* heads,
                                     const int32_t* prefix, int64_t n, const T* values, int D, int64_t* out_keys,
                                     T* out_values) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n || !heads[i]) return;
  int64_t g = prefix[i] - 1;
  const uint64_t k = keys[i];
  T acc[3] = {T(0), T(0), T(0)};
  for (int64_t j = i; j < n && keys[j] == k; ++j) {
    int64_t r = order[j];
    for (int a = 0; a < 3; ++a) acc[a] = acc[a] + values[3 * r + a];
  }
  uint64_t mask = (uint64_t(1) << D) - 1;
  out_keys[g] = basis_key(int(k >> (3 * D)), int((k >> (2 * D)) & mask), int((k >> D) & mask), int(k & mask));
  for (int a = 0; a < 3; ++a) out_values[4 * g + a] = -acc[a];  // normals.py:106-110,219-221
  out_values[4 * g + 3] = -T(0);
}

// normals.py:132-147 contributions (raw depth * w, splat weight * w, w) in first-index
// order; zero for groups whose mean normal vanishes.
template <class T>
__global__ void average_contrib_kernel(const int32_t* order, int64_t n, const T* nsums, const T* weights, const T* dw,
                                       T* contrib) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int64_t src = order[i];
  T w = weights[src];
  T nm[3] = {nsums[3 * src] / w, nsums[3 * src + 1] / w, nsums[3 * src + 2] / w};
  bool ok = sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]) > T(0);
  contrib[3 * i] = ok ? dw[2 * src] * w : T(0);
  contrib[3 * i + 1] = ok ? dw[2 * src + 1] * w : T(0);
  contrib[3 * i + 2] = ok ? w : T(0);
}

// Fixed 1024-item chunks summed serially (in T, input order) — the order the oracle
// restates — then the chunk totals serially.  One block per chunk copies the chunk's 3 x 1024
// values into shared memory with coalesced loads, then one thread adds them in order (a
// serial loop over global memory waits an L2 round trip per item).
constexpr int kAverageChunk = 1024, kAverageThreads = 128;
template <class T>
__global__ void __launch_bounds__(kAverageThreads) average_chunks_kernel(const T* contrib, int64_t n, T* partial) {
  __shared__ T s_c[3 * kAverageChunk];
  const int64_t chunk = blockIdx.x;
  const int64_t begin = chunk * kAverageChunk;
  if (begin >= n) return;
  const int count = int(begin + kAverageChunk < n ? kAverageChunk : n - begin);
  for (int e = threadIdx.x; e < 3 * count; e += blockDim.x) s_c[e] = contrib[3 * begin + e];
  __syncthreads();
  if (threadIdx.x != 0) return;
  T part[3] = {T(0), T(0), T(0)};
  for (int i = 0; i < count; ++i) {
    T c2 = s_c[3 * i + 2];
    if (c2 > T(0)) {
      part[0] = part[0] + s_c[3 * i];
      part[1] = part[1] + s_c[3 * i + 1];
      part[2] = part[2] + c2;
    }
  }
  for (int a = 0; a < 3; ++a) partial[3 * chunk + a] = part[a];
}

template <class T>
__global__ void __launch_bounds__(kAverageThreads) average_finish_kernel(const T* partial, int64_t chunks, T* average) {
  __shared__ T s_p[3 * kAverageChunk];
  T total[3] = {T(0), T(0), T(0)};
  for (int64_t c0 = 0; c0 < chunks; c0 += kAverageChunk) {  // tiles of chunk totals, in order
    const int count = int(c0 + kAverageChunk < chunks ? kAverageChunk : chunks - c0);
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * count; e += blockDim.x) s_p[e] = partial[3 * c0 + e];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int c = 0; c < count; ++c)
        for (int a = 0; a < 3; ++a) total[a] = total[a] + s_p[3 * c + a];
  }
  if (threadIdx.x != 0) return;
  average[0] = average[1] = average[2] = T(0);
  if (total[2] > T(0)) {
    average[0] = total[0] / total[2];
    average[1] = total[1] / total[2];
    average[2] = total[2];
  }
}

__global__ void depth_offsets_kernel(const int64_t* keys, int64_t n, int levels, int64_t* offsets) {
  int d = threadIdx.x;
  if (d >= levels) return;
  int64_t target = int64_t(d) << 48, lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (keys[mid] < target)
      lo = mid + 1;
    else
      hi = mid;
  }
  offsets[d] = lo;
}

template <class T>
NormalData<T> build_normals(const SampleGroups<T>& g, const DensityData<T>& D, int minimum, int maximum,
                            cudaStream_t s, bool keep) {
  NormalData<T> N;
  int64_t n = g.count;
  DBuf<uint32_t> fk(n, s), sfk(n, s);
  DBuf<int32_t> ids(n, s), order(n, s);
  first_keys_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.first.p, n, fk.p, ids.p);
  PSR_LAUNCH_CHECK();
  sort_pairs(fk.p, sfk.p, ids.p, order.p, n, 32, s);
  int64_t r = 54 * n;
  int Db = maximum > 0 ? maximum : 1;
  {
    DBuf<int32_t> rids(r, s), rorder(r, s);
    DBuf<T> rvals(3 * r, s);
    // Record keys of 3 Db + 5 bits: 32-bit keys up to depth 9 (a third less data through the
    // sort's passes), else 64-bit.  Same keys, same stable order either way.
    auto splat_reduce = [&](auto key_tag) {
      using K = decltype(key_tag);
      DBuf<K> rkeys(r, s), skeys(r, s);
      normal_splat_kernel<T, K><<<blocks_for(54 * n), kThreads, 0, s>>>(order.p, n, g.sums.p, g.normal_sums.p,
                                                                        g.weights.p, D.dw.p, minimum, maximum,
                                                                        rkeys.p, rids.p, rvals.p);
      PSR_LAUNCH_CHECK();
      sort_pairs(rkeys.p, skeys.p, rids.p, rorder.p, r, 3 * Db + 5, s);
      DBuf<int32_t> heads, prefix;
      int64_t u = segment_heads(skeys.p, r, uint64_t(1) << (3 * Db + 4), 0, heads, prefix, s);
      N.count = u;
      N.keys.alloc(u, s);
      N.values.alloc(4 * u, s);
      normal_reduce_kernel<T, K><<<blocks_for(r), kThreads, 0, s>>>(skeys.p, rorder.p, heads.p, prefix.p, r,
                                                                    rvals.p, Db, N.keys.p, N.values.p);
      PSR_LAUNCH_CHECK();
      if (keep) {
        N.record_slot.alloc(r, s);
        segment_slot_kernel<<<blocks_for(r), kThreads, 0, s>>>(rorder.p, prefix.p, skeys.p, r,
                                                               uint64_t(1) << (3 * Db + 4), 0, N.record_slot.p);
        PSR_LAUNCH_CHECK();
      }
    };
    if (3 * Db + 5 <= 32)
      splat_reduce(uint32_t());
    else
      splat_reduce(uint64_t());
  }
  int64_t chunks = (n + kAverageChunk - 1) / kAverageChunk;
  DBuf<T> partial(3 * chunks, s), contrib(3 * n, s);
  average_contrib_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(order.p, n, g.normal_sums.p, g.weights.p, D.dw.p,
                                                               contrib.p);
  PSR_LAUNCH_CHECK();
  if (chunks) average_chunks_kernel<T><<<unsigned(chunks), kAverageThreads, 0, s>>>(contrib.p, n, partial.p);
  PSR_LAUNCH_CHECK();
  N.average.alloc(3, s);
  average_finish_kernel<T><<<1, kAverageThreads, 0, s>>>(partial.p, chunks, N.average.p);
  PSR_LAUNCH_CHECK();
  DBuf<int64_t> off(maximum + 2, s);
  depth_offsets_kernel<<<1, 32, 0, s>>>(N.keys.p, N.count, maximum + 2, off.p);
  PSR_LAUNCH_CHECK();
  N.offsets = read_vector(off.p, maximum + 2, s);
  if (keep) N.group_order = std::move(order);
  return N;
}

template SampleGroups<float> prepare_samples<float>(const float*, const float*, int64_t, int, double, cudaStream_t,
                                                   bool);
template SampleGroups<double> prepare_samples<double>(const double*, const double*, int64_t, int, double,
                                                     cudaStream_t, bool);
template DensityData<float> build_density<float>(const SampleGroups<float>&, int, int, double, cudaStream_t, bool);
template DensityData<double> build_density<double>(const SampleGroups<double>&, int, int, double, cudaStream_t, bool);
template NormalData<float> build_normals<float>(const SampleGroups<float>&, const DensityData<float>&, int, int,
                                                cudaStream_t, bool);
template NormalData<double> build_normals<double>(const SampleGroups<double>&, const DensityData<double>&, int, int,
                                                  cudaStream_t, bool);
template float density_scale<float>();
template double density_scale<double>();

#include "psr_samples_adjoint.cuh"

}  // namespace psr
