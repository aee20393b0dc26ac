// A8: ordered sliced Gauss-Seidel (warp-psr relaxation.py:121-210) as a persistent,
// dependency-scheduled kernel over x-strips of each slice.
//
// Sequential definition: for front = 2^d .. -iters+1, for z in [max(front,0),
// min(front+iters, 2^d+1)), for colour 0..3 (colour = (x&1) + 2(y&1)): update every row of
// slice z with that colour (rows of one colour in one slice never couple).  Visit t of slice
// z needs visit t of z+1 and visit t-1 of z-1 (relaxation.py:128-135).
//
// B200 mapping:
//  * each slice-visit (z, t) is split into NS x-strips; strip tasks run on independent CTAs;
//  * a strip recomputes a halo of width 3-c around itself in colour phase c, so the four
//    colour phases need no synchronisation with neighbouring strips (the halo values are
//    the same arithmetic on the same inputs, hence bit-identical to the neighbour's);
//  * the strip's x footprint (three slices, x within 4 of the strip) is staged in shared
//    memory once the dependencies are met; the phases then run on shared memory only;
//  * x is double-buffered by visit parity: visit t of a slice is written to buffer t&1, so a
//    strip never overwrites values another strip of the same visit still reads.  The slice
//    dependency edges order every reader of buffer t&1's previous contents before the write;
//  * rows are permuted into schedule order (slice, colour, x, y), so every footprint is 12
//    contiguous position ranges, found through a per-(slice, colour) x-start table.
// Waits are bounded; a timeout sets an error word and every CTA exits.
#include "psr_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace psr {

constexpr int kSlotsR = 28;
constexpr int kPad = 32;

struct StripLevel {
  int n;          // 2^depth (slices 0..n)
  int strips;     // NS (per slice; boundaries balance the rows)
  const int32_t* bounds;     // [(n+1)*(NS+1)] x boundaries of the strips of each slice
  int iters;
  int cap;        // footprint capacity (elements) per CTA
  int use_scratch;
  int row_cap;    // update rows staged in shared memory per task (0: read rows from global)
  const int32_t* cols;       // schedule positions, slot k = lexicographic neighbour k, -1 absent
  const void* vals;          // T[rows*28]
  const void* b;             // V[rows]
  void* xb0;                 // V[rows]  even visits
  void* xb1;                 // V[rows]  odd visits (holds the initial x)
  const int64_t* keys;       // schedule order
  const int32_t* xstart;     // [(n+1)*4][n+2]: first position of group (z,c) with x >= X
  const int2* visits;        // slice-visits (z, t) in the sequential order
  int nvisits;
  int* done;                 // completed strip tasks of slice z at done[z * kPad] (one 128-byte line each)
  long long* trace;          // optional: 8 timestamps per task (PSR_RELAX_TRACE_FILE)
  int* counter;
  int* error;
  void* scratch;             // V[grid*cap] when use_scratch
};

__device__ __forceinline__ long long globaltimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire_r(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool wait_at_least(const int* p, int v, const int* error) {
  for (long long it = 0; it < (1LL << 26); ++it) {
    if (ld_acquire_r(p) >= v) return true;
    if ((it & 63) == 63 && *(volatile const int*)error) return false;
    __nanosleep(it < 512 ? 32 : 256);
  }
  return false;
}

// All 28 slots of a row with 16-byte loads (rows are 16-byte aligned: 28 * 4 or 28 * 8 bytes).
__device__ __forceinline__ void load_row(const float* src, float out[kSlotsR]) {
  const float4* v = reinterpret_cast<const float4*>(src);
#pragma unroll
  for (int q = 0; q < kSlotsR / 4; ++q) {
    float4 w = __ldg(v + q);
    out[4 * q] = w.x;
    out[4 * q + 1] = w.y;
    out[4 * q + 2] = w.z;
    out[4 * q + 3] = w.w;
  }
}
__device__ __forceinline__ void load_row(const double* src, double out[kSlotsR]) {
  const double2* v = reinterpret_cast<const double2*>(src);
#pragma unroll
  for (int q = 0; q < kSlotsR / 2; ++q) {
    double2 w = __ldg(v + q);
    out[2 * q] = w.x;
    out[2 * q + 1] = w.y;
  }
}

// Range r of a flattened index i (bases ascending, count entries + a final total).
__device__ __forceinline__ int range_of(const int* base, int count, int i) {
  int r = 0;
  while (r + 1 < count && base[r + 1] <= i) ++r;
  return r;
}

template <class T, class V>
__global__ void __launch_bounds__(256) strip_gs_kernel(StripLevel L) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // Per task: footprint ranges (j = slice z-1+j, colour c), update ranges (colour c, halo
  // 3-c) and own ranges (colour c, no halo), all as schedule positions.
  __shared__ int s_task, s_fail, s_total, s_rows;
  __shared__ int s_lo[12], s_hi[12], s_base[13];
  __shared__ int s_p0[4], s_p1[4], s_rbase[5], s_o0[4], s_o1[4], s_obase[5];
  const T* __restrict__ vals = reinterpret_cast<const T*>(L.vals);
  const V* __restrict__ b = reinterpret_cast<const V*>(L.b);
  V* xb0 = reinterpret_cast<V*>(L.xb0);
  V* xb1 = reinterpret_cast<V*>(L.xb1);
  V* foot = L.use_scratch ? reinterpret_cast<V*>(L.scratch) + int64_t(blockIdx.x) * L.cap
                          : reinterpret_cast<V*>(smem_raw);
  // Staged rows (tasks with at most L.row_cap update rows): operator values, footprint
  // indices of the 27 neighbours (-1 absent), b and the row's own footprint index.
  unsigned char* rows_raw = smem_raw + (L.use_scratch ? 0 : ((int64_t(L.cap) * sizeof(V) + 15) & ~int64_t(15)));
  // Layout (every part 16-byte aligned): values T[28] per row (112 or 224 bytes), footprint
  // indices int16[32] per row (64 bytes: slots 0..26, the row itself at 27, padding), b.
  T* r_vals = reinterpret_cast<T*>(rows_raw);
  int16_t* r_fidx = reinterpret_cast<int16_t*>(rows_raw + int64_t(L.row_cap) * kSlotsR * sizeof(T));
  V* r_b = reinterpret_cast<V*>(rows_raw + int64_t(L.row_cap) * (kSlotsR * sizeof(T) + 64));
  const int nx = L.n + 2;
  const int total_tasks = L.nvisits * L.strips;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) {
      s_task = atomicAdd(L.counter, 1);
      s_fail = 0;
    }
    __syncthreads();
    const int task = s_task;
    if (task >= total_tasks) return;
    long long* tr = (L.trace && threadIdx.x == 0) ? L.trace + int64_t(task) * 8 : nullptr;
    if (tr) {
      tr[0] = globaltimer();
      tr[7] = blockIdx.x;
    }
    const int2 zt = L.visits[task / L.strips];
    const int z = zt.x, t = zt.y, s = task % L.strips;
    const int x0 = L.bounds[z * (L.strips + 1) + s], x1 = L.bounds[z * (L.strips + 1) + s + 1];
    // All range lookups in one round: 24 footprint bounds, 8 update bounds, 8 own bounds.
    if (threadIdx.x < 40) {
      int i = threadIdx.x;
      if (i < 24) {
        int r = i >> 1, j = r >> 2, c = r & 3, zz = z + j - 1;
        int v = 0;
        if (zz >= 0 && zz <= L.n) {
          int X = (i & 1) ? min(x1 + 4, L.n + 1) : max(x0 - 4, 0);
          v = L.xstart[int64_t(zz * 4 + c) * nx + X];
        }
        if (i & 1)
          s_hi[r] = v;
        else
          s_lo[r] = v;
      } else {
        int k = i - 24, c = (k >> 1) & 3, own = k >= 8, h = own ? 0 : 3 - c;
        int X = (k & 1) ? min(x1 + h, L.n + 1) : max(min(x0 - h, L.n + 1), 0);
        int v = L.xstart[int64_t(z * 4 + c) * nx + X];
        if (own) {
          if (k & 1)
            s_o1[c] = v;
          else
            s_o0[c] = v;
        } else {
          if (k & 1)
            s_p1[c] = v;
          else
            s_p0[c] = v;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int total = 0;
      for (int r = 0; r < 12; ++r) {
        s_base[r] = total;
        total += s_hi[r] - s_lo[r];
      }
      s_base[12] = total;
      s_total = total;
      int rows = 0, owns = 0;
      for (int c = 0; c < 4; ++c) {
        s_rbase[c] = rows;
        rows += s_p1[c] - s_p0[c];
        s_obase[c] = owns;
        owns += s_o1[c] - s_o0[c];
      }
      s_rbase[4] = rows;
      s_obase[4] = owns;
      s_rows = rows;
      if (total > L.cap) {
        atomicExch(L.error, 2);
        s_fail = 1;
      }
    }
    __syncthreads();
    if (s_fail) return;
    // Stage the update rows' data before waiting (it does not depend on x) when it fits.
    const bool staged = s_rows <= L.row_cap && s_total < 32768;
    if (staged) {
      for (int i = threadIdx.x; i < s_rows; i += blockDim.x) {
        int c = range_of(s_rbase, 4, i);
        int p = s_p0[c] + (i - s_rbase[c]);
        const int4* vs = reinterpret_cast<const int4*>(vals + int64_t(p) * kSlotsR);
        int4* vd = reinterpret_cast<int4*>(r_vals + int64_t(i) * kSlotsR);
#pragma unroll
        for (int q = 0; q < kSlotsR * int(sizeof(T)) / 16; ++q) vd[q] = __ldg(vs + q);
        r_b[i] = __ldg(b + p);
        int64_t key = __ldg(L.keys + p);
        int px = int((key >> 32) & 65535), py = int((key >> 16) & 65535);
        const int4* cr = reinterpret_cast<const int4*>(L.cols + int64_t(p) * kSlotsR);
        int cw[kSlotsR];
#pragma unroll
        for (int q = 0; q < kSlotsR / 4; ++q) {
          int4 w = __ldg(cr + q);
          cw[4 * q] = w.x;
          cw[4 * q + 1] = w.y;
          cw[4 * q + 2] = w.z;
          cw[4 * q + 3] = w.w;
        }
        int16_t f[32];
        bool bad = false;
#pragma unroll
        for (int k = 0; k < 27; ++k) {
          int fi = -1;
          if (cw[k] >= 0) {
            int rr = (k % 3) * 4 + ((px + k / 9 - 1) & 1) + 2 * ((py + (k / 3) % 3 - 1) & 1);
            fi = s_base[rr] + (cw[k] - s_lo[rr]);
            if (fi < 0 || fi >= s_base[12]) {  // not the k-th neighbour: malformed operator
              bad = true;
              fi = -1;
            }
          }
          f[k] = int16_t(fi);
        }
        f[27] = int16_t(s_base[4 + c] + (p - s_lo[4 + c]));  // the row itself
        f[28] = f[29] = f[30] = f[31] = -1;
        int4* fd = reinterpret_cast<int4*>(r_fidx + int64_t(i) * 32);
        const int4* fs = reinterpret_cast<const int4*>(f);
#pragma unroll
        for (int q = 0; q < 4; ++q) fd[q] = fs[q];
        if (bad) atomicExch(L.error, 3);
      }
    }
    if (tr) tr[1] = globaltimer();
    if (threadIdx.x == 0) {
      bool ok = true;
      if (z + 1 <= L.n) ok = wait_at_least(L.done + (z + 1) * kPad, (t + 1) * L.strips, L.error);
      if (ok && z > 0) ok = wait_at_least(L.done + (z - 1) * kPad, t * L.strips, L.error);
      if (ok) ok = wait_at_least(L.done + z * kPad, t * L.strips, L.error);
      if (!ok) {
        atomicCAS(L.error, 0, 1);
        s_fail = 1;
      }
      if (tr) tr[2] = globaltimer();
    }
    __syncthreads();
    if (s_fail) return;
    if (tr) tr[3] = globaltimer();
    // Stage the footprint: slice z+1 after visit t, slices z and z-1 after visit t-1.
    // One warp per contiguous range.
    {
      const V* cur = (t & 1) ? xb1 : xb0;
      const V* prev = (t & 1) ? xb0 : xb1;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
      for (int r = warp; r < 12; r += nwarps) {
        const V* src = ((r >> 2) == 2 ? cur : prev) + s_lo[r];
        V* dst = foot + s_base[r];
        const int cnt = s_hi[r] - s_lo[r];
        for (int i0 = lane; i0 < cnt; i0 += 128) {
          V v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (i0 + 32 * u < cnt) v[u] = __ldcg(src + i0 + 32 * u);
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (i0 + 32 * u < cnt) dst[i0 + 32 * u] = v[u];
        }
      }
    }
    __syncthreads();
    if (tr) tr[4] = globaltimer();
    // Colour phases on the staged footprint (halo 3-c).
    for (int c = 0; c < 4; ++c) {
      const int p0 = s_p0[c], p1 = s_p1[c], rb = s_rbase[c];
      for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        T diagonal = T(0);
        V xi = V(0);
        int self;
        if (staged) {
          // Staged row: 27 independent shared-memory loads, then the ordered subtraction.
          int i = rb + (p - p0);
          int16_t fd[32];
          {
            const int4* fs = reinterpret_cast<const int4*>(r_fidx + int64_t(i) * 32);
            int4* fl = reinterpret_cast<int4*>(fd);
#pragma unroll
            for (int q = 0; q < 4; ++q) fl[q] = fs[q];
          }
          T aa[kSlotsR];
          {
            const int4* vs = reinterpret_cast<const int4*>(r_vals + int64_t(i) * kSlotsR);
            int4* vl = reinterpret_cast<int4*>(aa);
#pragma unroll
            for (int q = 0; q < kSlotsR * int(sizeof(T)) / 16; ++q) vl[q] = vs[q];
          }
          V xs[27];
#pragma unroll
          for (int k = 0; k < 27; ++k) {
            int fi = fd[k];
            xs[k] = fi >= 0 ? foot[fi] : V(0);
          }
          V r = r_b[i];
#pragma unroll
          for (int k = 0; k < 27; ++k)
            if (fd[k] >= 0) r = r - xs[k] * V(aa[k]);
          if (fd[13] >= 0) {
            diagonal = aa[13];
            xi = xs[13];
          }
          self = fd[27];
          if (diagonal != T(0)) foot[self] = xi + r * (V(1.0) / V(diagonal));
          continue;
        }
        int cc[kSlotsR];
        T aa[kSlotsR];
        V r;
        int px, py;
        {
          const int4* cr = reinterpret_cast<const int4*>(L.cols + int64_t(p) * kSlotsR);
#pragma unroll
          for (int q = 0; q < kSlotsR / 4; ++q) {
            int4 w = __ldg(cr + q);
            cc[4 * q] = w.x;
            cc[4 * q + 1] = w.y;
            cc[4 * q + 2] = w.z;
            cc[4 * q + 3] = w.w;
          }
          load_row(vals + int64_t(p) * kSlotsR, aa);
          r = __ldg(b + p);
          int64_t key = __ldg(L.keys + p);
          px = int((key >> 32) & 65535);
          py = int((key >> 16) & 65535);
        }
        self = s_base[4 + c] + (p - s_lo[4 + c]);
#pragma unroll
        for (int k = 0; k < 27; ++k) {
          if (cc[k] < 0) continue;
          int dx = k / 9 - 1, dy = (k / 3) % 3 - 1, j = k % 3;
          int cn = ((px + dx) & 1) + 2 * ((py + dy) & 1);
          int rr = j * 4 + cn;
          int fi = s_base[rr] + (cc[k] - s_lo[rr]);
          if (fi < 0 || fi >= s_total) {  // not the k-th neighbour: malformed operator
            atomicExch(L.error, 3);
            continue;
          }
          V xn = foot[fi];
          T a = aa[k];
          r = r - xn * V(a);
          if (k == 13) {
            diagonal = a;
            xi = xn;
          }
        }
        if (diagonal != T(0)) foot[self] = xi + r * (V(1.0) / V(diagonal));
      }
      __syncthreads();
    }
    if (tr) tr[5] = globaltimer();
    // Publish the strip's own rows (x in [x0, x1)) as visit t.
    {
      V* out = (t & 1) ? xb1 : xb0;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
      for (int c = warp; c < 4; c += nwarps) {
        const int o0 = s_o0[c], o1 = s_o1[c], base = s_base[4 + c] - s_lo[4 + c];
        for (int p = o0 + lane; p < o1; p += 32) __stcg(out + p, foot[base + p]);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(L.done + z * kPad, 1);
      if (tr) tr[6] = globaltimer();
    }
  }
}

// ------------------------------------------------------------------ level preparation
// xstart[(z*4+c)*(n+2) + X] = first schedule position of group 4z+c whose x >= X.
__global__ void xstart_kernel(const int64_t* skeys, const int32_t* group_off, int n, int32_t* xstart) {
  int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  int nx = n + 2;
  int64_t total = int64_t(n + 1) * 4 * nx;
  if (idx >= total) return;
  int X = int(idx % nx);
  int g = int(idx / nx);
  int lo = group_off[g], hi = group_off[g + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    int x = int((skeys[mid] >> 32) & 65535);
    if (x < X)
      lo = mid + 1;
    else
      hi = mid;
  }
  xstart[idx] = lo;
}

// Row-balanced strip boundaries: slice z's rows split into NS runs of x of about equal size.
__global__ void strip_bounds_kernel(const int32_t* xstart, int n, int strips, int32_t* bounds) {
  int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z > n) return;
  int nx = n + 2;
  const int32_t* xs = xstart + int64_t(z * 4) * nx;
  int total = 0;
  for (int c = 0; c < 4; ++c) total += xs[c * nx + n + 1] - xs[c * nx];
  int32_t* out = bounds + int64_t(z) * (strips + 1);
  out[0] = 0;
  int k = 1, below = 0;
  for (int X = 0; X <= n && k < strips; ++X) {
    for (int c = 0; c < 4; ++c) below += xs[c * nx + X + 1] - xs[c * nx + X];
    while (k < strips && int64_t(below) * strips >= int64_t(k) * total) out[k++] = X + 1;
  }
  while (k < strips) out[k++] = n + 1;
  out[strips] = n + 1;
}

__global__ void footprint_kernel(const int32_t* xstart, const int32_t* bounds, int n, int strips, int* maxfp) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (n + 1) * strips) return;
  int z = idx / strips, s = idx % strips, nx = n + 2;
  int x0 = bounds[z * (strips + 1) + s], x1 = bounds[z * (strips + 1) + s + 1];
  int rows = 0;
  for (int c = 0; c < 4; ++c) {
    const int32_t* xs = xstart + int64_t(z * 4 + c) * nx;
    int h = 3 - c;
    rows += xs[min(x1 + h, n + 1)] - xs[max(min(x0 - h, n + 1), 0)];
  }
  atomicMax(maxfp + 1, rows);
  int total = 0;
  for (int j = -1; j <= 1; ++j) {
    int zz = z + j;
    if (zz < 0 || zz > n) continue;
    for (int c = 0; c < 4; ++c) {
      const int32_t* xs = xstart + int64_t(zz * 4 + c) * nx;
      total += xs[min(x1 + 4, n + 1)] - xs[max(x0 - 4, 0)];
    }
  }
  atomicMax(maxfp, total);
}

__global__ void inverse_kernel(const int32_t* perm, int64_t n, int32_t* inv) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) inv[perm[p]] = int32_t(p);
}

// Gathers an ELL operator (key order) into schedule order, columns as schedule positions.
template <class T, class V>
__global__ void reorder_kernel(const int32_t* perm, const int32_t* inv, int64_t n, const int32_t* cols, const T* vals,
                               const V* b, const V* x, const int64_t* keys, int32_t* scols, T* svals, V* sb, V* sx,
                               int64_t* skeys) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  int64_t row = perm[p];
  for (int k = 0; k < kSlotsR; ++k) {
    int32_t c = cols[row * kSlotsR + k];
    scols[p * kSlotsR + k] = c >= 0 ? inv[c] : -1;
    svals[p * kSlotsR + k] = vals[row * kSlotsR + k];
  }
  sb[p] = b[row];
  sx[p] = x[row];
  skeys[p] = keys[row];
}

template <class V>
__global__ void scatter_back_kernel(const int32_t* perm, int64_t n, const V* sx, V* x) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) x[perm[p]] = sx[p];
}

__global__ void slice_groups_kernel(const int64_t* keys, int64_t n, uint32_t* groups, int32_t* ids) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  key_coords(keys[i], c);
  groups[i] = uint32_t((c[0] & 1) + 2 * (c[1] & 1) + 4 * c[2]);
  ids[i] = int32_t(i);
}

__global__ void group_bounds_kernel(const uint32_t* sorted, int64_t n, int count, int32_t* off) {
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

static int device_sms() {
  static int count = 0;
  if (!count) {
    int dev = 0;
    PSR_CUDA(cudaGetDevice(&dev));
    PSR_CUDA(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev));
  }
  return count;
}

// Ordered sliced relaxation of one level given as slot-ELL rows in key order.  x (key
// order) holds the initial guess and receives the result.
template <class T, class V>
void relax_sliced_strips(const int64_t* keys, int64_t rows, int depth, const int32_t* cols, const T* vals,
                         const V* b, V* x, int iters, cudaStream_t s, float* ms) {
  if (iters <= 0 || rows <= 0) return;
  const int n = 1 << depth;
  const int groups = 4 * (n + 1);
  // Schedule order: stable sort by group (slice, colour); rows of a group stay in key order.
  DBuf<uint32_t> g(rows, s), sg(rows, s);
  DBuf<int32_t> ids(rows, s), perm(rows, s), inv(rows, s), off(groups + 1, s);
  slice_groups_kernel<<<blocks_for(rows), kThreads, 0, s>>>(keys, rows, g.p, ids.p);
  PSR_LAUNCH_CHECK();
  sort_pairs(g.p, sg.p, ids.p, perm.p, rows, bits_for(uint64_t(groups)), s);
  group_bounds_kernel<<<blocks_for(groups + 1), kThreads, 0, s>>>(sg.p, rows, groups, off.p);
  PSR_LAUNCH_CHECK();
  inverse_kernel<<<blocks_for(rows), kThreads, 0, s>>>(perm.p, rows, inv.p);
  PSR_LAUNCH_CHECK();
  DBuf<int32_t> scols(kSlotsR * rows, s);
  DBuf<T> svals(kSlotsR * rows, s);
  DBuf<V> sb(rows, s), x0(rows, s), x1(rows, s);
  DBuf<int64_t> skeys(rows, s);
  reorder_kernel<T, V><<<blocks_for(rows), kThreads, 0, s>>>(perm.p, inv.p, rows, cols, vals, b, x, keys, scols.p,
                                                            svals.p, sb.p, x1.p, skeys.p);
  PSR_LAUNCH_CHECK();
  const int nx = n + 2;
  DBuf<int32_t> xstart(int64_t(n + 1) * 4 * nx, s);
  xstart_kernel<<<blocks_for(int64_t(n + 1) * 4 * nx), kThreads, 0, s>>>(skeys.p, off.p, n, xstart.p);
  PSR_LAUNCH_CHECK();
  // Strips per slice: enough tasks per wave (iters x strips) to fill the persistent grid,
  // at least ~96 rows per strip.
  int strips = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(2 * device_sms() + iters - 1) / iters,
                                                          rows / (int64_t(n + 1) * 96))));
  DBuf<int32_t> bounds(int64_t(n + 1) * (strips + 1), s);
  strip_bounds_kernel<<<blocks_for(n + 1), kThreads, 0, s>>>(xstart.p, n, strips, bounds.p);
  PSR_LAUNCH_CHECK();
  const int64_t pad_end = int64_t(n + 1) * kPad;
  DBuf<int> flags(pad_end + 4 * kPad, s);
  flags.zero();
  int* counter = flags.p + pad_end;
  int* error = flags.p + pad_end + kPad;
  int* caps_dev = flags.p + pad_end + 2 * kPad;
  footprint_kernel<<<blocks_for((n + 1) * strips), kThreads, 0, s>>>(xstart.p, bounds.p, n, strips, caps_dev);
  PSR_LAUNCH_CHECK();
  std::vector<int> caps = read_vector(caps_dev, 2, s);
  int maxfp = caps[0], maxrows = caps[1];
  // Slice-visits in wave order (relaxation.py:128-143): wave q = 2t + n - z holds slices two
  // apart; every dependency of a wave-q task lies in wave q-1 or q-2, so dequeuing by wave
  // is deadlock-free and keeps a whole wave (up to `iters` slice-visits) in flight.
  std::vector<int2> visits;
  for (int q = 0; q <= n + 2 * (iters - 1); ++q) {
    int first = std::max(0, (q - n + 1) / 2), last = std::min(iters - 1, q / 2);
    for (int t = first; t <= last; ++t) visits.push_back(make_int2(n - q + 2 * t, t));
  }
  DBuf<int2> dvisits(int64_t(visits.size()), s);
  PSR_CUDA(cudaMemcpyAsync(dvisits.p, visits.data(), visits.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
  const int smem_cap_bytes = 110 * 1024;  // two CTAs per SM
  StripLevel L{};
  L.n = n;
  L.strips = strips;
  L.bounds = bounds.p;
  L.iters = iters;
  L.cols = scols.p;
  L.vals = svals.p;
  L.b = sb.p;
  L.xb0 = x0.p;
  L.xb1 = x1.p;
  L.keys = skeys.p;
  L.xstart = xstart.p;
  L.visits = dvisits.p;
  L.nvisits = int(visits.size());
  L.done = flags.p;
  L.counter = counter;
  L.error = error;
  // Shared memory: the x footprint, plus the update rows' operator data of tasks whose rows
  // fit (other tasks read their rows from global memory).
  const int64_t per_row = kSlotsR * int64_t(sizeof(T)) + 64 + int64_t(sizeof(V));
  int64_t fp_bytes = (int64_t(maxfp) * int64_t(sizeof(V)) + 15) & ~int64_t(15);
  int64_t smem = 0;
  L.cap = std::max(maxfp, 1);
  L.use_scratch = fp_bytes > smem_cap_bytes;
  L.row_cap = 0;
  if (!L.use_scratch) {
    L.row_cap = int(std::min<int64_t>(maxrows, (smem_cap_bytes - fp_bytes) / per_row));
    smem = std::max<int64_t>(fp_bytes + L.row_cap * per_row, 16);
  }
  auto kernel = strip_gs_kernel<T, V>;
  PSR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap_bytes));
  int per_sm = 0;
  PSR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, int(smem)));
  int64_t total_tasks = int64_t(visits.size()) * strips;
  int grid = int(std::min<int64_t>(total_tasks, int64_t(std::max(per_sm, 1)) * device_sms()));
  const char* trace_file = std::getenv("PSR_RELAX_TRACE_FILE");
  DBuf<long long> trace;
  if (trace_file) {
    trace.alloc(total_tasks * 8, s);
    trace.zero();
    L.trace = trace.p;
  }
  DBuf<V> scratch;
  if (L.use_scratch) {
    scratch.alloc(int64_t(grid) * L.cap, s);
    L.scratch = scratch.p;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms) {
    PSR_CUDA(cudaEventCreate(&e0));
    PSR_CUDA(cudaEventCreate(&e1));
    PSR_CUDA(cudaEventRecord(e0, s));
  }
  kernel<<<grid, 256, size_t(smem), s>>>(L);
  PSR_LAUNCH_CHECK();
  if (ms) PSR_CUDA(cudaEventRecord(e1, s));
  scatter_back_kernel<V><<<blocks_for(rows), kThreads, 0, s>>>(perm.p, rows, ((iters - 1) & 1) ? x1.p : x0.p, x);
  PSR_LAUNCH_CHECK();
  int err = read_scalar(L.error, s);
  if (ms) {
    PSR_CUDA(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (trace_file) {
    std::vector<long long> h = read_vector(trace.p, total_tasks * 8, s);
    if (FILE* f = std::fopen(trace_file, "ab")) {
      long long header[6] = {depth, n, strips, L.row_cap, grid, total_tasks};
      std::fwrite(header, sizeof(header), 1, f);
      std::fwrite(visits.data(), sizeof(int2), visits.size(), f);
      std::fwrite(h.data(), sizeof(long long), h.size(), f);
      std::fclose(f);
    }
  }
  if (err == 2) throw Error(4, "ordered relaxation: footprint exceeds its capacity");
  if (err == 3) throw Error(1, "ordered relaxation: an operator column is not its slot's neighbour");
  if (err) throw Error(4, "ordered relaxation: a dependency wait timed out");
}

template void relax_sliced_strips<float, float>(const int64_t*, int64_t, int, const int32_t*, const float*,
                                                const float*, float*, int, cudaStream_t, float*);
template void relax_sliced_strips<double, double>(const int64_t*, int64_t, int, const int32_t*, const double*,
                                                  const double*, double*, int, cudaStream_t, float*);
template void relax_sliced_strips<float, double>(const int64_t*, int64_t, int, const int32_t*, const float*,
                                                 const double*, double*, int, cudaStream_t, float*);

}  // namespace psr
