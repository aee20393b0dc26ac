/*
 * psr_field.cuh -- header-only evaluation of a reconstructed field inside CUDA kernels.
 *
 * Replaces warp-psr's `evaluate_field(field, point) -> (value, gradient, valid)`, the inline
 * @wp.func that application kernels call on the handle returned by `result.device_field()`
 * (src/warp_psr/device_field.py:91-112; the query it wraps: device_field.py:15-41, and the
 * reference and direct evaluators field.py:36-81, 365-421).
 *
 * Usage, in a user kernel compiled for sm_100a:
 *
 *   #include "psr_field.cuh"
 *   __global__ void k(psr_field_handle f, const float* q, float* v, int n) {
 *     int i = blockIdx.x * blockDim.x + threadIdx.x;
 *     if (i < n) v[i] = psr_evaluate_field(f, q[3*i], q[3*i+1], q[3*i+2]).value;
 *   }
 *
 * The handle (psr_device_field / Reconstruction.device_field().handle) is a POD of device
 * pointers owned by the result; pass it by value.  Its dtype selects the overload: the
 * float overload for PSR_FLOAT32 fields, the double overload for PSR_FLOAT64.
 *
 * Contract (the reference's): the point is in the reconstruction's input coordinates;
 * the result is the raw implicit value, its gradient in input coordinates and valid = 1,
 * or NaN value and gradient with valid = 0 when the point maps outside the unit cube or is
 * not finite.  The surface is value == handle.iso_value.
 *
 * Every product and sum is a round-to-nearest intrinsic (__fmul_rn / __fadd_rn and the
 * double forms), which the compiler never contracts into a fused multiply-add, so a user
 * kernel built with the default --fmad=true returns bit for bit what psr_evaluate returns.
 *
 * Lookups: with hash_slots set (every handle the library returns) a key is found by linear
 * probing of 16-byte {key, index} slots; a handle built by hand with hash_slots = NULL
 * binary-searches the sorted keys like the reference's find_key (field.py:19-32).  With
 * cumulative = NULL the field is evaluated the direct way, every level summed
 * (field.py:36-81); otherwise the reference way: the leaf level, the cumulative field one
 * level up and the coefficients one level down (field.py:365-421).
 */
#ifndef PSR_FIELD_CUH
#define PSR_FIELD_CUH

#include <stdint.h>

#include "psr_b200.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>

namespace psr_field {

// Mixer of the open-addressing tables (the library builds its tables with the same one).
__host__ __device__ __forceinline__ uint64_t hash_mix(uint64_t x) {
  x ^= x >> 31;
  x *= 0x7fb5d329728ea185ULL;
  x ^= x >> 27;
  x *= 0x81dadef4bc2dd44dULL;
  x ^= x >> 33;
  return x;
}

__host__ __device__ __forceinline__ int64_t basis_key(int d, int x, int y, int z) {
  return (int64_t(d) << 48) | (int64_t(x) << 32) | (int64_t(y) << 16) | int64_t(z);
}

// Uncontracted arithmetic.
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// What one evaluation needs, in the field's precision T.
template <class T>
struct View {
  const int64_t* keys;
  const T* coefficients;
  const T* cumulative;  // NULL: direct evaluation
  int64_t count;
  const longlong2* slots;  // NULL: binary search of keys
  uint64_t mask;
  int depth;
};

template <class T>
__device__ __forceinline__ View<T> view(const psr_field_handle& h) {
  View<T> v;
  v.keys = h.keys;
  v.coefficients = static_cast<const T*>(h.coefficients);
  v.cumulative = static_cast<const T*>(h.cumulative);
  v.count = h.count;
  v.slots = static_cast<const longlong2*>(h.hash_slots);
  v.mask = h.hash_mask;
  v.depth = h.depth;
  return v;
}

// Index of `key` among the field's keys, or -1.
template <class T>
__device__ __forceinline__ int64_t find(const View<T>& f, int64_t key) {
  if (f.slots) {
    uint64_t s = hash_mix(uint64_t(key)) & f.mask;
    while (true) {
      const longlong2 e = __ldg(f.slots + s);
      if (e.x == key) return e.y;
      if (e.x == -1) return -1;
      s = (s + 1) & f.mask;
    }
  }
  int64_t lo = 0, hi = f.count;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(f.keys + mid) < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < f.count && __ldg(f.keys + lo) == key) ? lo : -1;
}

// One level of the reference evaluator (field.py:370-393): the eight corners of the
// left-owned cell, the polynomial piece on the right-owned side of each corner.
// r = {value, d/dx, d/dy, d/dz} in the cube frame, accumulated in place.
template <class T>
__device__ __forceinline__ void add_level(const View<T>& f, const T* coeff, const T p[3], int d, T r[4]) {
  const int n = 1 << d;
  const T nn = T(n);
  T t[3], fr[3];
  int cell[3], base[3];
  for (int a = 0; a < 3; ++a) {
    t[a] = mul(p[a], nn);
    cell[a] = min(max(int(ceil(t[a])) - 1, 0), n - 1);
    base[a] = int(floor(t[a]));
    fr[a] = sub(t[a], T(base[a]));
  }
  for (int corner = 0; corner < 8; ++corner) {
    const int node[3] = {cell[0] + corner / 4, cell[1] + (corner / 2) % 2, cell[2] + corner % 2};
    if (min(node[0] - base[0], min(node[1] - base[1], node[2] - base[2])) < 0) continue;
    const int64_t idx = find(f, basis_key(d, node[0], node[1], node[2]));
    if (idx < 0) continue;
    T hh[3], sg[3];
    for (int a = 0; a < 3; ++a) {
      hh[a] = sub(T(1), fr[a]);
      sg[a] = T(-1);
      if (node[a] > base[a]) {
        hh[a] = fr[a];
        sg[a] = T(1);
      }
    }
    const T c = coeff[idx];
    r[0] = add(r[0], mul(mul(mul(c, hh[0]), hh[1]), hh[2]));
    r[1] = add(r[1], mul(mul(mul(mul(c, nn), sg[0]), hh[1]), hh[2]));
    r[2] = add(r[2], mul(mul(mul(mul(c, nn), hh[0]), sg[1]), hh[2]));
    r[3] = add(r[3], mul(mul(mul(mul(c, nn), hh[0]), hh[1]), sg[2]));
  }
}

// One level of the direct evaluator (field.py:50-73): the eight corners of the left-owned
// cell, the piece of that cell.
template <class T>
__device__ __forceinline__ void add_level_direct(const View<T>& f, const T p[3], int d, T r[4]) {
  const int n = 1 << d;
  const T nn = T(n);
  T fr[3];
  int cell[3];
  for (int a = 0; a < 3; ++a) {
    const T t = mul(p[a], nn);
    cell[a] = min(max(int(ceil(t)) - 1, 0), n - 1);
    fr[a] = sub(t, T(cell[a]));
  }
  for (int corner = 0; corner < 8; ++corner) {
    const int cc[3] = {corner / 4, (corner / 2) % 2, corner % 2};
    const int64_t idx = find(f, basis_key(d, cell[0] + cc[0], cell[1] + cc[1], cell[2] + cc[2]));
    if (idx < 0) continue;
    T hh[3], sg[3];
    for (int a = 0; a < 3; ++a) {
      hh[a] = sub(T(1), fr[a]);
      sg[a] = T(-1);
      if (cc[a] != 0) {
        hh[a] = fr[a];
        sg[a] = T(1);
      }
    }
    const T c = f.coefficients[idx];
    r[0] = add(r[0], mul(mul(mul(c, hh[0]), hh[1]), hh[2]));
    const T cn = mul(c, nn);
    r[1] = add(r[1], mul(cn, mul(mul(sg[0], hh[1]), hh[2])));
    r[2] = add(r[2], mul(cn, mul(mul(hh[0], sg[1]), hh[2])));
    r[3] = add(r[3], mul(cn, mul(mul(hh[0], hh[1]), sg[2])));
  }
}

// Value and cube-frame gradient r at a point p of the unit cube (finite, 0 <= p <= 1).
template <class T>
__device__ __forceinline__ void evaluate_cube(const View<T>& f, T p[3], T r[4]) {
  r[0] = r[1] = r[2] = r[3] = T(0);
  if (!f.cumulative) {
    for (int d = 0; d <= f.depth; ++d) add_level_direct(f, p, d, r);
    return;
  }
  // leaf: the deepest level with an active key at the point's left-owned cell (field.py:406-412)
  int leaf = 0;
  for (int d = f.depth; d >= 0; --d) {
    const int n = 1 << d;
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = min(max(int(ceil(mul(p[a], T(n)))) - 1, 0), n - 1);
    if (find(f, basis_key(d, c[0], c[1], c[2])) >= 0) {
      leaf = d;
      break;
    }
  }
  // points on the cube's faces move inside (field.py:413-415)
  for (int a = 0; a < 3; ++a) {
    if (p[a] == T(0))
      p[a] = T(1e-6);
    else if (p[a] == T(1))
      p[a] = T(1.0 - 1e-6);
  }
  add_level(f, f.coefficients, p, leaf, r);
  if (leaf > 0) {
    T s[4] = {T(0), T(0), T(0), T(0)};
    add_level(f, f.cumulative, p, leaf - 1, s);
    for (int a = 0; a < 4; ++a) r[a] = add(r[a], s[a]);
  }
  if (leaf < f.depth) {
    T s[4] = {T(0), T(0), T(0), T(0)};
    add_level(f, f.coefficients, p, leaf + 1, s);
    for (int a = 0; a < 4; ++a) r[a] = add(r[a], s[a]);
  }
}

// p = L q + t (row-major L), in the order the reference's mat-vec takes.
template <class T>
__device__ __forceinline__ void to_cube(const T L[9], const T tr[3], const T q[3], T p[3]) {
  for (int r = 0; r < 3; ++r)
    p[r] = add(add(add(mul(L[3 * r], q[0]), mul(L[3 * r + 1], q[1])), mul(L[3 * r + 2], q[2])), tr[r]);
}

template <class T>
__device__ __forceinline__ bool inside(const T p[3]) {
  const T lo = (p[1] < p[0]) ? ((p[2] < p[1]) ? p[2] : p[1]) : ((p[2] < p[0]) ? p[2] : p[0]);
  const T hi = (p[0] < p[1]) ? ((p[1] < p[2]) ? p[2] : p[1]) : ((p[0] < p[2]) ? p[2] : p[0]);
  return isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) && lo >= T(0) && hi <= T(1);
}

template <class T>
struct Result {
  T value;
  T gradient[3];
  int valid;
};

// The full query: model point -> cube, evaluation, gradient back to the model frame
// (L^T r), NaN and valid = 0 outside.
template <class T>
__device__ __forceinline__ Result<T> evaluate(const View<T>& f, const T L[9], const T tr[3], const T q[3]) {
  Result<T> out;
  T p[3];
  to_cube(L, tr, q, p);
  out.valid = inside(p) ? 1 : 0;
  if (!out.valid) {
    const T nan = T(NAN);
    out.value = nan;
    out.gradient[0] = out.gradient[1] = out.gradient[2] = nan;
    return out;
  }
  T r[4];
  evaluate_cube(f, p, r);
  out.value = r[0];
  for (int a = 0; a < 3; ++a) out.gradient[a] = add(add(mul(L[a], r[1]), mul(L[3 + a], r[2])), mul(L[6 + a], r[3]));
  return out;
}

template <class T>
__device__ __forceinline__ Result<T> evaluate(const psr_field_handle& h, T x, T y, T z) {
  T L[9], tr[3];
  for (int a = 0; a < 9; ++a) L[a] = T(h.linear[a]);
  for (int a = 0; a < 3; ++a) tr[a] = T(h.translation[a]);
  const T q[3] = {x, y, z};
  return evaluate(view<T>(h), L, tr, q);
}

}  // namespace psr_field

// warp-psr evaluate_field(field: Field, point: vec3) for PSR_FLOAT32 handles.
__device__ __forceinline__ psr_field::Result<float> psr_evaluate_field(const psr_field_handle& h, float x, float y,
                                                                       float z) {
  return psr_field::evaluate<float>(h, x, y, z);
}
// warp-psr evaluate_field(field: Field64, point: vec3d) for PSR_FLOAT64 handles.
__device__ __forceinline__ psr_field::Result<double> psr_evaluate_field(const psr_field_handle& h, double x, double y,
                                                                        double z) {
  return psr_field::evaluate<double>(h, x, y, z);
}

#endif  // __CUDACC__
#endif  // PSR_FIELD_CUH
