// A11/A12: cumulative coefficients, field evaluation, isovalue and evaluation transforms
// (warp-psr field.py:187-421, reconstruction.py:18-116, transforms.py:11-86).
#include "../../include/psr_b200.h"
#include "psr_internal.cuh"

#include <algorithm>
#include <exception>

namespace psr {

// field.py:187-203 — cumulative[i] = sum_h cumulative[parent]*h + coefficients[i], one depth per launch.
template <class T>
__global__ void cumulative_kernel(const int64_t* keys, int64_t begin, int64_t end, int d, HashView h, const T* coeff,
                                  T* cum) {
  int64_t i = begin + blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= end) return;
  int c[3];
  key_coords(keys[i], c);
  T value = T(0);
  for (int corner = 0; corner < 8; ++corner) {
    int p[3] = {c[0] / 2 + corner / 4, c[1] / 2 + (corner / 2) % 2, c[2] / 2 + corner % 2};
    T hw = (T(1) - fabs(T(c[0]) * T(.5) - T(p[0]))) * (T(1) - fabs(T(c[1]) * T(.5) - T(p[1]))) *
           (T(1) - fabs(T(c[2]) * T(.5) - T(p[2])));
    if (hw > T(0)) {
      int32_t idx = h.find(basis_key(d - 1, p[0], p[1], p[2]));
      if (idx >= 0) value = value + cum[idx] * hw;
    }
  }
  cum[i] = value + coeff[i];
}

template <class T>
void cumulative_coefficients(const int64_t* keys, const std::vector<int64_t>& offsets, const HashView& h,
                             const T* coeff, T* cumulative, int depth, cudaStream_t s) {
  int64_t total = offsets[depth + 1];
  PSR_CUDA(cudaMemcpyAsync(cumulative, coeff, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
  for (int d = 1; d <= depth; ++d) {
    int64_t n = offsets[d + 1] - offsets[d];
    if (!n) continue;
    cumulative_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(keys, offsets[d], offsets[d + 1], d, h, coeff, cumulative);
    PSR_LAUNCH_CHECK();
  }
}

// The per-query evaluation (field.py:365-421) is psr_field.cuh's, the same code user
// kernels include, so psr_evaluate and psr_evaluate_field agree bit for bit.
template <class T>
__device__ __forceinline__ psr_field::View<T> field_view(const HashView& h, const int64_t* keys, const T* coeff,
                                                        const T* cumulative, int depth) {
  return psr_field::View<T>{keys, coeff, cumulative, 0, h.slots, h.mask, depth};
}

template <class T>
__device__ __forceinline__ void add_level(const HashView& h, const T* coeff, const T p[3], int d, T r[4]) {
  psr_field::add_level(field_view<T>(h, nullptr, coeff, coeff, d), coeff, p, d, r);
}

// Model-frame queries, or (cube_frame) the centroids of the isovalue, q = sums / weights
// with the identity transform (reconstruction.py:273-280).
template <class T>
__global__ void evaluate_kernel(const HashView h, const int64_t* keys, const T* coeff, const T* cumulative,
                                const T* queries, int64_t nq, const T* linear, const T* translation, int depth,
                                T* values, T* gradients, int32_t* valid, int cube_frame, const T* gsums,
                                const T* gweights) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nq) return;
  T L[9], tr[3], q[3];
  if (cube_frame) {
    for (int a = 0; a < 9; ++a) L[a] = (a % 4 == 0) ? T(1) : T(0);
    tr[0] = tr[1] = tr[2] = T(0);
    T w = gweights[i];
    for (int a = 0; a < 3; ++a) q[a] = gsums[3 * i + a] / w;
  } else {
    for (int a = 0; a < 9; ++a) L[a] = linear[a];
    for (int a = 0; a < 3; ++a) tr[a] = translation[a];
    for (int a = 0; a < 3; ++a) q[a] = queries[3 * i + a];
  }
  const psr_field::Result<T> r = psr_field::evaluate(field_view<T>(h, keys, coeff, cumulative, depth), L, tr, q);
  if (valid) valid[i] = r.valid;
  values[i] = r.value;
  if (gradients)
    for (int a = 0; a < 3; ++a) gradients[3 * i + a] = r.gradient[a];
}

template <class T>
void evaluate_queries(const int64_t* keys, const HashView& h, const T* coeff, const T* cumulative, const T* queries,
                      int64_t nq, const T* linear, const T* translation, int depth, T* values, T* gradients,
                      int32_t* valid, bool cube_frame, const T* group_sums, const T* group_weights, cudaStream_t s) {
  if (nq <= 0) return;
  evaluate_kernel<T><<<blocks_for(nq, 128), 128, 0, s>>>(h, keys, coeff, cumulative, queries, nq, linear, translation,
                                                         depth, values, gradients, valid, cube_frame ? 1 : 0,
                                                         group_sums, group_weights);
  PSR_LAUNCH_CHECK();
}

// Weighted mean in a fixed order: 1024-value blocks, 256 lanes x 4 strided values summed
// in float64, pairwise tree over lanes, block totals summed serially.  Products stay in
// the input precision before the float64 accumulation (reconstruction.py:63-66).
template <class T>
__global__ void isovalue_blocks_kernel(const T* values, const T* weights, int64_t n, double* partial) {
  __shared__ double tv[256], tw[256];
  int l = threadIdx.x;
  int64_t b = blockIdx.x * int64_t(1024);
  double v = 0.0, w = 0.0;
  for (int j = 0; j < 4; ++j) {
    int64_t i = b + l + 256 * j;
    if (i < n) {
      v += double(values[i] * weights[i]);
      w += double(weights[i]);
    }
  }
  tv[l] = v;
  tw[l] = w;
  __syncthreads();
  // pairwise tree, stride 128 .. 1: element l takes l + stride.  Strides 128..32 in shared
  // memory, 16..1 inside warp 0 with shuffles (the same additions in the same order).
  for (int stride = 128; stride >= 32; stride >>= 1) {
    if (l < stride) {
      tv[l] = tv[l] + tv[l + stride];
      tw[l] = tw[l] + tw[l + stride];
    }
    __syncthreads();
  }
  if (l < 32) {
    v = tv[l];
    w = tw[l];
#pragma unroll
    for (int stride = 16; stride >= 1; stride >>= 1) {
      v = v + __shfl_down_sync(0xffffffffu, v, stride);
      w = w + __shfl_down_sync(0xffffffffu, w, stride);
    }
    if (l == 0) {
      partial[2 * blockIdx.x] = v;
      partial[2 * blockIdx.x + 1] = w;
    }
  }
}

template <class T>
__global__ void __launch_bounds__(128) isovalue_finish_kernel(const double* partial, int64_t blocks, T* out) {
  // block totals summed serially in order by one thread, from tiles staged in shared memory
  // with coalesced loads (a loop over global memory waits an L2 round trip per total)
  constexpr int kTile = 1024;
  __shared__ double s_p[2 * kTile];
  double total = 0.0, mass = 0.0;
  for (int64_t b0 = 0; b0 < blocks; b0 += kTile) {
    const int count = int(b0 + kTile < blocks ? kTile : blocks - b0);
    __syncthreads();
    for (int e = threadIdx.x; e < 2 * count; e += blockDim.x) s_p[e] = partial[2 * b0 + e];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int b = 0; b < count; ++b) {
        total += s_p[2 * b];
        mass += s_p[2 * b + 1];
      }
  }
  if (threadIdx.x == 0) out[0] = T(total / mass);
}

template <class T>
void isovalue(const T* values, const T* weights, int64_t n, T* out, cudaStream_t s) {
  int64_t blocks = (n + 1023) / 1024;
  DBuf<double> partial(2 * (blocks > 0 ? blocks : 1), s);
  if (blocks) {
    isovalue_blocks_kernel<T><<<unsigned(blocks), 256, 0, s>>>(values, weights, n, partial.p);
    PSR_LAUNCH_CHECK();
  }
  isovalue_finish_kernel<T><<<1, 128, 0, s>>>(partial.p, blocks, out);
  PSR_LAUNCH_CHECK();
}

// transforms.py:16-79 — cofactor inverse of the cube->model matrix, applied twice.
template <class T>
__device__ T det3(const T m[9]) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
template <class T>
__device__ T minor4(const T m[16], int row, int col) {
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
__device__ void reference_inverse(const T m[16], T out[16]) {
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

template <class T>
__global__ void transforms_kernel(const T* nz, T* out) {
  if (threadIdx.x != 0) return;
  T s = nz[0];
  T m[16] = {T(0), s, T(0), nz[1], T(0), T(0), s, nz[2], s, T(0), T(0), nz[3], T(0), T(0), T(0), T(1)};
  reference_inverse(m, out);
  reference_inverse(out, out + 16);
}

template <class T>
void evaluation_transforms(const T* normalization, T* transforms, cudaStream_t s) {
  transforms_kernel<T><<<1, 32, 0, s>>>(normalization, transforms);
  PSR_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ allocation-free isovalue
// Some callers cannot allocate device memory while they run: code embedded in a host
// framework that has already claimed the device memory through its own pool (a renderer, a
// deep-learning framework's caching allocator), or a real-time loop that must not take the
// implicit synchronisation or failure modes of an allocation.  psr_isovalue_static serves
// them: the per-block partial sums live in this file-scope array instead of a buffer from
// the stream-ordered allocator.  Every GPU that loads the library keeps the array (64 KiB)
// until the process exits.
constexpr int64_t kStaticIsoBlocks = 4096;  // at most 4096 * 1024 = 4,194,304 values per call
static __device__ __align__(256) double g_iso_scratch[2 * kStaticIsoBlocks];

// Device address of g_iso_scratch in the current context.  The host-side name is only a
// stand-in for the device array and must not be passed to kernels.  The address belongs to
// the context that loaded this library's module, so it is looked up on every call (no
// allocation): a cached address would go stale after cudaDeviceReset or under a context the
// caller made current itself.  The first call on a device also loads the module.
static double* static_iso_scratch() {
  void* p = nullptr;
  PSR_CUDA(cudaGetSymbolAddress(&p, g_iso_scratch));
  return static_cast<double*>(p);
}

template <class T>
static void isovalue_static(const T* values, const T* weights, int64_t n, T* out, cudaStream_t s) {
  const int64_t blocks = (n + 1023) / 1024;
  if (blocks > kStaticIsoBlocks)
    throw Error(PSR_EINVAL, "psr_isovalue_static: at most 4,194,304 values per call (use psr_isovalue beyond that)");
  double* partial = static_iso_scratch();
  // Each block writes its own two partial sums before the finishing kernel reads exactly
  // `blocks` of them, so no slot has to start at zero.
  isovalue_blocks_kernel<T><<<unsigned(blocks), 256, 0, s>>>(values, weights, n, partial);
  PSR_LAUNCH_CHECK();
  isovalue_finish_kernel<T><<<1, 128, 0, s>>>(partial, blocks, out);
  PSR_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ A13 field reverse (field_adjoint.py, field.py:214-284)
// One level of evaluate_kernel reversed: coefficient adjoints (atomic) and the cube-frame
// position adjoint.  gv seeds the value, gg (cube frame) the spatial gradient r[1..3].
template <class T>
__device__ __forceinline__ void add_level_reverse(const HashView& h, const T* coeff, const T p[3], int d, T gv,
                                                  const T gg[3], T* g_coeff, T qp[3]) {
  int n = 1 << d;
  T t[3], f[3];
  int cell[3], base[3];
  for (int a = 0; a < 3; ++a) {
    t[a] = p[a] * T(n);
    cell[a] = min(max(int(ceil(t[a])) - 1, 0), n - 1);
    base[a] = int(floor(t[a]));
    f[a] = t[a] - T(base[a]);
  }
  for (int corner = 0; corner < 8; ++corner) {
    int node[3] = {cell[0] + corner / 4, cell[1] + (corner / 2) % 2, cell[2] + corner % 2};
    if (min(node[0] - base[0], min(node[1] - base[1], node[2] - base[2])) < 0) continue;
    int32_t idx = h.find(basis_key(d, node[0], node[1], node[2]));
    if (idx < 0) continue;
    T hh[3], sg[3];
    for (int a = 0; a < 3; ++a) {
      hh[a] = T(1) - f[a];
      sg[a] = T(-1);
      if (node[a] > base[a]) {
        hh[a] = f[a];
        sg[a] = T(1);
      }
    }
    const T nn = T(n);
    const T bgrad[3] = {nn * sg[0] * hh[1] * hh[2], nn * hh[0] * sg[1] * hh[2], nn * hh[0] * hh[1] * sg[2]};
    const T gc = gv * hh[0] * hh[1] * hh[2] + gg[0] * bgrad[0] + gg[1] * bgrad[1] + gg[2] * bgrad[2];
    if (gc != T(0)) atomicAdd(g_coeff + idx, gc);
    const T c = coeff[idx];
    const T xy = c * nn * nn * sg[0] * sg[1] * hh[2];
    const T xz = c * nn * nn * sg[0] * hh[1] * sg[2];
    const T yz = c * nn * nn * hh[0] * sg[1] * sg[2];
    qp[0] = qp[0] + gv * c * bgrad[0] + gg[1] * xy + gg[2] * xz;
    qp[1] = qp[1] + gv * c * bgrad[1] + gg[0] * xy + gg[2] * yz;
    qp[2] = qp[2] + gv * c * bgrad[2] + gg[0] * xz + gg[1] * yz;
  }
}

// evaluate_kernel reversed.  Model frame: p = L q + tr, model gradient = L^T r[1..3]; the
// adjoints of q (g_q, written), of L and tr (g_ltr: 12 float64 sums, atomic) are produced.
// Cube frame (isovalue centroids q = sums / w): g_q is the adjoint of the group sums.
template <class T>
__global__ void evaluate_reverse_kernel(const HashView h, const T* coeff, const T* cumulative, const T* queries,
                                        int64_t nq, const T* linear, const T* translation, int depth, const T* g_values,
                                        const T* g_gradients, T* g_coeff, T* g_cum, T* g_q, double* g_ltr,
                                        int cube_frame, const T* gsums, const T* gweights) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nq) return;
  T L[9], tr[3], q[3];
  if (cube_frame) {
    for (int a = 0; a < 9; ++a) L[a] = (a % 4 == 0) ? T(1) : T(0);
    tr[0] = tr[1] = tr[2] = T(0);
    T w = gweights[i];
    for (int a = 0; a < 3; ++a) q[a] = gsums[3 * i + a] / w;
  } else {
    for (int a = 0; a < 9; ++a) L[a] = linear[a];
    for (int a = 0; a < 3; ++a) tr[a] = translation[a];
    for (int a = 0; a < 3; ++a) q[a] = queries[3 * i + a];
  }
  const T gv = g_values ? g_values[i] : T(0);
  T gm[3] = {T(0), T(0), T(0)};
  if (g_gradients)
    for (int a = 0; a < 3; ++a) gm[a] = g_gradients[3 * i + a];
  T gq[3] = {T(0), T(0), T(0)};
  T p[3];
  for (int r = 0; r < 3; ++r) p[r] = L[3 * r] * q[0] + L[3 * r + 1] * q[1] + L[3 * r + 2] * q[2] + tr[r];
  bool ok = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]) && dmin(p[0], dmin(p[1], p[2])) >= T(0) &&
            dmax(p[0], dmax(p[1], p[2])) <= T(1);
  if (ok && (gv != T(0) || gm[0] != T(0) || gm[1] != T(0) || gm[2] != T(0))) {
    const T orig[3] = {p[0], p[1], p[2]};
    int leaf = 0;
    for (int d = depth; d >= 0; --d) {
      int n = 1 << d;
      int c[3];
      for (int a = 0; a < 3; ++a) c[a] = min(max(int(ceil(p[a] * T(n))) - 1, 0), n - 1);
      if (h.find(basis_key(d, c[0], c[1], c[2])) >= 0) {
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
    // cube-frame spatial seed: model gradient = L^T r  =>  g_r = L g_model
    const T gg[3] = {L[0] * gm[0] + L[1] * gm[1] + L[2] * gm[2], L[3] * gm[0] + L[4] * gm[1] + L[5] * gm[2],
                     L[6] * gm[0] + L[7] * gm[1] + L[8] * gm[2]};
    T qp[3] = {T(0), T(0), T(0)};
    add_level_reverse(h, coeff, p, leaf, gv, gg, g_coeff, qp);
    if (leaf > 0) add_level_reverse(h, cumulative, p, leaf - 1, gv, gg, g_cum, qp);
    if (leaf < depth) add_level_reverse(h, coeff, p, leaf + 1, gv, gg, g_coeff, qp);
    for (int a = 0; a < 3; ++a)
      if (orig[a] == T(0) || orig[a] == T(1)) qp[a] = T(0);
    for (int c = 0; c < 3; ++c) gq[c] = L[c] * qp[0] + L[3 + c] * qp[1] + L[6 + c] * qp[2];
    if (g_ltr && !cube_frame) {
      // r[1..3] of the forward, needed for the adjoint of L through the model gradient
      T r[4] = {T(0), T(0), T(0), T(0)};
      add_level(h, coeff, p, leaf, r);
      if (leaf > 0) {
        T sl[4] = {T(0), T(0), T(0), T(0)};
        add_level(h, cumulative, p, leaf - 1, sl);
        for (int a = 0; a < 4; ++a) r[a] = r[a] + sl[a];
      }
      if (leaf < depth) {
        T sl[4] = {T(0), T(0), T(0), T(0)};
        add_level(h, coeff, p, leaf + 1, sl);
        for (int a = 0; a < 4; ++a) r[a] = r[a] + sl[a];
      }
      for (int rr = 0; rr < 3; ++rr)
        for (int c = 0; c < 3; ++c) {
          const double g = double(qp[rr]) * double(q[c]) + double(r[1 + rr]) * double(gm[c]);
          if (g != 0.0) atomicAdd(g_ltr + 3 * rr + c, g);
        }
      for (int rr = 0; rr < 3; ++rr)
        if (qp[rr] != T(0)) atomicAdd(g_ltr + 9 + rr, double(qp[rr]));
    }
  }
  if (g_q) {
    if (cube_frame) {
      const T w = gweights[i];
      for (int a = 0; a < 3; ++a) g_q[3 * i + a] = g_q[3 * i + a] + gq[a] / w;
    } else {
      for (int a = 0; a < 3; ++a) g_q[3 * i + a] = gq[a];
    }
  }
}

// Isovalue reversed (field_adjoint.py:144-152): each centroid value's adjoint is
// T(g_iso / total weight) * w, the seed g_iso read from device memory (no host round trip).
template <class T>
__global__ void isovalue_reverse_kernel(const T* weights, int64_t n, const T* g_iso, const double* mass, T* g_values) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) g_values[i] = T(double(g_iso[0]) / mass[0]) * weights[i];
}

// Total sample weight (float64), block sums added atomically (mass must start at zero).
template <class T>
__global__ void mass_kernel(const T* weights, int64_t n, double* mass) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    acc += double(weights[i]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(mass, red[0]);
}

// cumulative_kernel reversed for one depth: g_coeff += g_cum; parents receive h * g_cum.
template <class T>
__global__ void cumulative_reverse_kernel(const int64_t* keys, int64_t begin, int64_t end, int d, HashView h, T* g_cum,
                                          T* g_coeff) {
  int64_t i = begin + blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= end) return;
  const T g = g_cum[i];
  g_coeff[i] = g_coeff[i] + g;
  if (d == 0 || g == T(0)) return;
  int c[3];
  key_coords(keys[i], c);
  for (int corner = 0; corner < 8; ++corner) {
    int p[3] = {c[0] / 2 + corner / 4, c[1] / 2 + (corner / 2) % 2, c[2] / 2 + corner % 2};
    T hw = (T(1) - fabs(T(c[0]) * T(.5) - T(p[0]))) * (T(1) - fabs(T(c[1]) * T(.5) - T(p[1]))) *
           (T(1) - fabs(T(c[2]) * T(.5) - T(p[2])));
    if (hw > T(0)) {
      int32_t idx = h.find(basis_key(d - 1, p[0], p[1], p[2]));
      if (idx >= 0) atomicAdd(g_cum + idx, g * hw);
    }
  }
}

template <class T>
void field_backward(const int64_t* keys, const std::vector<int64_t>& offsets, const HashView& h, const T* coeff,
                    const T* cumulative, int depth, const T* gsums, const T* gweights, int64_t groups, const T* g_iso,
                    T* g_coeff, T* g_cum, T* g_sums, cudaStream_t s) {
  if (g_iso && groups > 0) {
    DBuf<double> mass(1, s);
    mass.zero();
    mass_kernel<T><<<std::min<int64_t>(blocks_for(groups), 592), 256, 0, s>>>(gweights, groups, mass.p);
    PSR_LAUNCH_CHECK();
    DBuf<T> gv(groups, s);
    isovalue_reverse_kernel<T><<<blocks_for(groups), kThreads, 0, s>>>(gweights, groups, g_iso, mass.p, gv.p);
    PSR_LAUNCH_CHECK();
    evaluate_reverse_kernel<T><<<blocks_for(groups, 128), 128, 0, s>>>(h, coeff, cumulative, nullptr, groups, nullptr,
                                                                       nullptr, depth, gv.p, nullptr, g_coeff, g_cum,
                                                                       g_sums, nullptr, 1, gsums, gweights);
    PSR_LAUNCH_CHECK();
  }
  for (int d = depth; d >= 0; --d) {
    int64_t n = offsets[d + 1] - offsets[d];
    if (!n) continue;
    cumulative_reverse_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(keys, offsets[d], offsets[d + 1], d, h, g_cum,
                                                                    g_coeff);
    PSR_LAUNCH_CHECK();
  }
}

template <class T>
void evaluate_backward(const HashView& h, const T* coeff, const T* cumulative, const T* queries, int64_t nq,
                       const T* linear, const T* translation, int depth, const T* g_values, const T* g_gradients,
                       T* g_coeff, T* g_cum, T* g_queries, double* g_ltr, cudaStream_t s) {
  if (nq <= 0) return;
  evaluate_reverse_kernel<T><<<blocks_for(nq, 128), 128, 0, s>>>(h, coeff, cumulative, queries, nq, linear,
                                                                 translation, depth, g_values, g_gradients, g_coeff,
                                                                 g_cum, g_queries, g_ltr, 0, nullptr, nullptr);
  PSR_LAUNCH_CHECK();
}

#define INSTANTIATE(T)                                                                                               \
  template void field_backward<T>(const int64_t*, const std::vector<int64_t>&, const HashView&, const T*, const T*, \
                                  int, const T*, const T*, int64_t, const T*, T*, T*, T*, cudaStream_t);             \
  template void evaluate_backward<T>(const HashView&, const T*, const T*, const T*, int64_t, const T*, const T*,     \
                                     int, const T*, const T*, T*, T*, T*, double*, cudaStream_t);                    \
  template void cumulative_coefficients<T>(const int64_t*, const std::vector<int64_t>&, const HashView&, const T*,  \
                                           T*, int, cudaStream_t);                                                   \
  template void evaluate_queries<T>(const int64_t*, const HashView&, const T*, const T*, const T*, int64_t,         \
                                    const T*, const T*, int, T*, T*, int32_t*, bool, const T*, const T*,            \
                                    cudaStream_t);                                                                   \
  template void isovalue<T>(const T*, const T*, int64_t, T*, cudaStream_t);                                         \
  template void evaluation_transforms<T>(const T*, T*, cudaStream_t);
INSTANTIATE(float)
INSTANTIATE(double)

}  // namespace psr

extern "C" int psr_isovalue_static(int32_t dtype, const void* values, const void* weights, int64_t n, void* out,
                                   void* stream) {
  try {
    if (dtype != PSR_FLOAT32 && dtype != PSR_FLOAT64) throw psr::Error(PSR_EINVAL, "dtype must be float32 or float64");
    if (n <= 0 || !values || !weights || !out) throw psr::Error(PSR_EINVAL, "nonempty values and weights are required");
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PSR_FLOAT64)
      psr::isovalue_static<double>((const double*)values, (const double*)weights, n, (double*)out, s);
    else
      psr::isovalue_static<float>((const float*)values, (const float*)weights, n, (float*)out, s);
    return PSR_OK;
  } catch (const psr::Error& e) {
    psr::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    psr::set_last_error(e.what());
    return PSR_ECUDA;
  }
}
