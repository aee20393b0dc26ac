// Shared device/host helpers of the B200 screened-Poisson library: error handling,
// stream-ordered buffers, key packing, GPU hash maps (the replacement of warp-psr's
// binary-search `find_key`, field.py:19-32) and thin CUB wrappers for radix sort / scan.
#pragma once
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include "../../include/psr_field.cuh"

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace psr {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PSR_CUDA(call)                                                                              \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      throw ::psr::Error(2, std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + \
                                ":" + std::to_string(__LINE__) + ")");                              \
  } while (0)

// Every launch of this library's kernels is followed by PSR_LAUNCH_CHECK(), which also
// counts it (psr_kernel_launches).
extern std::atomic<long long> g_kernel_launches;
#define PSR_LAUNCH_CHECK()                                           \
  do {                                                               \
    ::psr::g_kernel_launches.fetch_add(1, std::memory_order_relaxed); \
    PSR_CUDA(cudaGetLastError());                                    \
  } while (0)

constexpr int64_t kInvalidKey = 0x7fffffffffffffffLL;
constexpr int kThreads = 256;

inline unsigned blocks_for(int64_t n, int threads = kThreads) {
  int64_t b = (n + threads - 1) / threads;
  return unsigned(b < 1 ? 1 : b);
}

// ------------------------------------------------------------------ stream-ordered buffers
struct Stream {
  cudaStream_t s;
};

template <class T>
struct DBuf {
  T* p = nullptr;
  int64_t n = 0;
  cudaStream_t s = nullptr;
  DBuf() = default;
  DBuf(int64_t count, cudaStream_t stream) { alloc(count, stream); }
  void alloc(int64_t count, cudaStream_t stream) {
    release();
    s = stream;
    n = count;
    if (count > 0) PSR_CUDA(cudaMallocAsync((void**)&p, size_t(count) * sizeof(T), stream));
  }
  void zero() {
    if (n > 0) PSR_CUDA(cudaMemsetAsync(p, 0, size_t(n) * sizeof(T), s));
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      s = o.s;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  T* get() const { return p; }
  int64_t size() const { return n; }
};

// Reads one device scalar (a count) synchronously — the analogue of the reference's
// small status/count reads (samples.py:254,276; keyed.py:132,174; tree.py:139).
template <class T>
T read_scalar(const T* dptr, cudaStream_t s) {
  T v;
  PSR_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(T), cudaMemcpyDeviceToHost, s));
  PSR_CUDA(cudaStreamSynchronize(s));
  return v;
}

template <class T>
std::vector<T> read_vector(const T* dptr, int64_t n, cudaStream_t s) {
  std::vector<T> v(size_t(n > 0 ? n : 0));
  if (n > 0) {
    PSR_CUDA(cudaMemcpyAsync(v.data(), dptr, size_t(n) * sizeof(T), cudaMemcpyDeviceToHost, s));
    PSR_CUDA(cudaStreamSynchronize(s));
  }
  return v;
}

// ------------------------------------------------------------------ arithmetic helpers
// Same NaN behaviour as std::min / std::max in the oracle.
template <class T>
__host__ __device__ __forceinline__ T dmin(T a, T b) { return (b < a) ? b : a; }
template <class T>
__host__ __device__ __forceinline__ T dmax(T a, T b) { return (a < b) ? b : a; }

// density.py:14-22 degree-2 B-spline values (float64).
__device__ __forceinline__ void quadratic(double x, double b[3]) {
  b[0] = (1.0 - x) * (1.0 - x) * 0.5;
  b[1] = ((1.0 - x) * (x + 1.0) + x * (2.0 - x)) * 0.5;
  b[2] = x * x * 0.5;
}

template <class T>
__device__ __forceinline__ int ceil_cell(T p, int n) {  // max(0, int(ceil(p*n)) - 1)
  int c = int(ceil(p * T(n))) - 1;
  return c < 0 ? 0 : c;
}

// ------------------------------------------------------------------ keys (field.py:13-16, tree.py:16-24)
__host__ __device__ __forceinline__ int64_t basis_key(int d, int x, int y, int z) {
  return (int64_t(d) << 48) | (int64_t(x) << 32) | (int64_t(y) << 16) | int64_t(z);
}
__host__ __device__ __forceinline__ void key_coords(int64_t k, int c[3]) {
  c[0] = int((k >> 32) & 65535);
  c[1] = int((k >> 16) & 65535);
  c[2] = int(k & 65535);
}
__host__ __device__ __forceinline__ int64_t tree_key(int x, int y, int z) {
  return (int64_t(x + 524288) << 40) | (int64_t(y + 524288) << 20) | int64_t(z + 524288);
}
__host__ __device__ __forceinline__ void tree_coords(int64_t k, int c[3]) {
  c[0] = int((k >> 40) & 1048575) - 524288;
  c[1] = int((k >> 20) & 1048575) - 524288;
  c[2] = int(k & 1048575) - 524288;
}

// ------------------------------------------------------------------ GPU hash map: int64 key -> int32 index
// Open addressing with linear probing over a power-of-two table at most half full.  A
// lookup returns exactly the index the reference's binary search over the sorted key
// array returns (or -1), so it can replace find_key anywhere.
// Open-addressing table of 16-byte slots {key, value} (key -1 = empty): a probe is one
// 16-byte load that brings the value with the key.
struct HashView {
  const longlong2* slots = nullptr;
  uint64_t mask = 0;
  __device__ __forceinline__ int32_t find(int64_t key) const {
    if (!slots) return -1;
    uint64_t h = mix(uint64_t(key)) & mask;
    while (true) {
      const longlong2 e = __ldg(slots + h);
      if (e.x == key) return int32_t(e.y);
      if (e.x == -1) return -1;
      h = (h + 1) & mask;
    }
  }
  // First probe only: the value, -1 (absent) or -2 (slot taken by another key: continue
  // with find_from(key, h)).  Lets a caller put several first probes in flight together.
  __device__ __forceinline__ int32_t first_probe(int64_t key, uint64_t& h) const {
    if (!slots) return -1;
    h = mix(uint64_t(key)) & mask;
    const longlong2 e = __ldg(slots + h);
    if (e.x == key) return int32_t(e.y);
    return e.x == -1 ? -1 : -2;
  }
  __device__ __forceinline__ int32_t find_from(int64_t key, uint64_t h) const {
    while (true) {
      h = (h + 1) & mask;
      const longlong2 e = __ldg(slots + h);
      if (e.x == key) return int32_t(e.y);
      if (e.x == -1) return -1;
    }
  }
  // the mixer of psr_field.cuh, so kernels outside the library probe the same tables
  __host__ __device__ static __forceinline__ uint64_t mix(uint64_t x) { return psr_field::hash_mix(x); }
};

__global__ void hash_insert_kernel(const int64_t* __restrict__ src, int64_t n, longlong2* slots, uint64_t mask,
                                   int32_t value_offset);
// hash_insert_kernel over the first *count keys (a device count, at most n_max).
__global__ void hash_insert_counted_kernel(const int64_t* __restrict__ src, int64_t n_max, const int32_t* count,
                                           longlong2* slots, uint64_t mask);

struct HashMap {
  DBuf<longlong2> slots;
  uint64_t mask = 0;
  int64_t count = 0;
  // Build from n unique keys; key i maps to value_offset + i.
  void build(const int64_t* src, int64_t n, cudaStream_t s, int32_t value_offset = 0) {
    count = n;
    uint64_t cap = 16;
    while (cap < uint64_t(2 * n + 1)) cap <<= 1;
    mask = cap - 1;
    slots.alloc(int64_t(cap), s);
    PSR_CUDA(cudaMemsetAsync(slots.p, 0xff, cap * sizeof(longlong2), s));
    if (n > 0) {
      hash_insert_kernel<<<blocks_for(n), kThreads, 0, s>>>(src, n, slots.p, mask, value_offset);
      PSR_LAUNCH_CHECK();
    }
  }
  // Build from the first *d_count keys of src, a count known only on the device (at most
  // n_max): the table is sized for n_max, so the count needs no host read-back.  Key i maps
  // to i.
  void build_counted(const int64_t* src, int64_t n_max, const int32_t* d_count, cudaStream_t s) {
    count = n_max;
    uint64_t cap = 16;
    while (cap < uint64_t(2 * n_max + 1)) cap <<= 1;
    mask = cap - 1;
    slots.alloc(int64_t(cap), s);
    PSR_CUDA(cudaMemsetAsync(slots.p, 0xff, cap * sizeof(longlong2), s));
    if (n_max > 0) {
      hash_insert_counted_kernel<<<blocks_for(n_max), kThreads, 0, s>>>(src, n_max, d_count, slots.p, mask);
      PSR_LAUNCH_CHECK();
    }
  }
  HashView view() const {
    HashView v;
    if (count > 0) {
      v.slots = slots.p;
      v.mask = mask;
    }
    return v;
  }
};

// ------------------------------------------------------------------ column index over sorted keys
// Keys sorted by (depth, x, y, z) form contiguous z-runs per (depth, x, y) column.  The
// column index maps a column to the position of its first key, so a box of neighbours costs
// one probe per (x, y) column plus a short scan in z instead of one probe per key.
// Column index of sorted basis keys: (d, x, y) -> index of the first key of that z-run.
// Up to kDenseColumnDepth it is a dense table per depth ((2^d + 1)^2 int32 entries, 1.4 MB
// through depth 9, so it stays in L2 and a probe is one load); deeper trees use a hash.
constexpr int kDenseColumnDepth = 12;

__host__ __device__ __forceinline__ int64_t dense_column_base(int d) {
  // sum over e < d of (2^e + 1)^2
  return ((int64_t(1) << (2 * d)) - 1) / 3 + 2 * ((int64_t(1) << d) - 1) + d;
}

struct ColumnView {
  HashView h;
  const int2* dense = nullptr;  // {first index, length} per column, start -1 when empty
  const int64_t* keys = nullptr;
  int64_t n = 0;
  __host__ __device__ static __forceinline__ int64_t column_key(int d, int x, int y) { return basis_key(d, x, y, 0); }
  // Index of the first key of column (d, x, y), or -1.
  __device__ __forceinline__ int32_t column(int d, int x, int y) const {
    int32_t count;
    return column_range(d, x, y, count);
  }
  // First index and length of column (d, x, y) (-1 when absent).  Without the dense table
  // the length is unknown and reported as INT32_MAX: the caller stops at the column's end.
  __device__ __forceinline__ int32_t column_range(int d, int x, int y, int32_t& count) const {
    if (dense) {
      const int side = (1 << d) + 1;
      count = 0;
      if (unsigned(x) >= unsigned(side) || unsigned(y) >= unsigned(side)) return -1;
      const int2 e = __ldg(dense + dense_column_base(d) + int64_t(x) * side + y);
      count = e.y;
      return e.x;
    }
    count = INT32_MAX;
    return h.find(column_key(d, x, y));
  }
  // First index in [start, start + count) of column `colk` (= key >> 16) whose z >= z0.
  __device__ __forceinline__ int32_t lower_z(int32_t start, int32_t count, int64_t colk, int z0) const {
    if (count != INT32_MAX) {
      int32_t lo = start, hi = start + count;
      while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (int(__ldg(keys + mid) & 65535) < z0)
          lo = mid + 1;
        else
          hi = mid;
      }
      return lo;
    }
    int32_t j = start;
    while (j < n) {
      const int64_t k = __ldg(keys + j);
      if ((k >> 16) != colk || int(k & 65535) >= z0) break;
      ++j;
    }
    return j;
  }
  // Index of the key (d, x, y, z), or -1.
  __device__ __forceinline__ int32_t find(int d, int x, int y, int z) const {
    int32_t count;
    const int32_t j0 = column_range(d, x, y, count);
    if (j0 < 0) return -1;
    const int64_t col = column_key(d, x, y) >> 16;
    const int32_t j = lower_z(j0, count, col, z);
    if (j >= n || (count != INT32_MAX && j >= j0 + count)) return -1;
    return __ldg(keys + j) == basis_key(d, x, y, z) ? j : -1;
  }
};

__global__ void column_insert_kernel(const int64_t* __restrict__ keys, int64_t n, longlong2* slots, uint64_t mask);
__global__ void dense_column_kernel(const int64_t* __restrict__ keys, int64_t n, int2* dense, int32_t* error);
__global__ void dense_count_kernel(const int64_t* __restrict__ keys, int64_t n, int2* dense);

struct ColumnIndex {
  HashMap map;
  DBuf<int2> table;
  ColumnView view_;
  // `max_depth` bounds the depth of every key (coordinates within [0, 2^d]).
  void build(const int64_t* keys, int64_t n, int max_depth, cudaStream_t s) {
    view_ = ColumnView();
    // PSR_COLUMN_INDEX=hash takes the hashed column index at any depth (test override: the
    // path of depths beyond the dense tables on small cases).
    const char* mode = std::getenv("PSR_COLUMN_INDEX");
    const bool force_hash = mode && mode[0] == 'h';
    if (max_depth <= kDenseColumnDepth && !force_hash) {
      const int64_t size = dense_column_base(max_depth + 1);
      table.alloc(size, s);
      PSR_CUDA(cudaMemsetAsync(table.p, 0xff, size * sizeof(int2), s));
      if (n > 0) {
        DBuf<int32_t> err(1, s);
        err.zero();
        dense_column_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, n, table.p, err.p);
        PSR_LAUNCH_CHECK();
        dense_count_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, n, table.p);
        PSR_LAUNCH_CHECK();
        if (read_scalar(err.p, s)) throw std::runtime_error("column index: key outside its depth's grid");
      }
      view_.dense = table.p;
    } else {
      map.count = n;
      uint64_t cap = 16;
      while (cap < uint64_t(2 * n + 1)) cap <<= 1;
      map.mask = cap - 1;
      map.slots.alloc(int64_t(cap), s);
      PSR_CUDA(cudaMemsetAsync(map.slots.p, 0xff, cap * sizeof(longlong2), s));
      if (n > 0) {
        column_insert_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys, n, map.slots.p, map.mask);
        PSR_LAUNCH_CHECK();
      }
      view_.h = map.view();
    }
    view_.keys = keys;
    view_.n = n;
  }
  ColumnView view() const { return view_; }
};

// ------------------------------------------------------------------ CUB wrappers
// Stable LSD radix sort of (key, value) pairs on key bits [0, end_bit).
template <class K, class V>
void sort_pairs(const K* kin, K* kout, const V* vin, V* vout, int64_t n, int end_bit, cudaStream_t s) {
  if (n <= 0) return;
  size_t temp = 0;
  PSR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, kin, kout, vin, vout, n, 0, end_bit, s));
  DBuf<char> t(int64_t(temp), s);
  PSR_CUDA(cub::DeviceRadixSort::SortPairs(t.p, temp, kin, kout, vin, vout, n, 0, end_bit, s));
}

template <class T>
void exclusive_sum(const T* in, T* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  size_t temp = 0;
  PSR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, in, out, n, s));
  DBuf<char> t(int64_t(temp), s);
  PSR_CUDA(cub::DeviceScan::ExclusiveSum(t.p, temp, in, out, n, s));
}

template <class T>
void inclusive_sum(const T* in, T* out, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  size_t temp = 0;
  PSR_CUDA(cub::DeviceScan::InclusiveSum(nullptr, temp, in, out, n, s));
  DBuf<char> t(int64_t(temp), s);
  PSR_CUDA(cub::DeviceScan::InclusiveSum(t.p, temp, in, out, n, s));
}

inline int bits_for(uint64_t maxval) {
  int b = 1;
  while (b < 64 && (maxval >> b)) ++b;
  return b;
}

}  // namespace psr
