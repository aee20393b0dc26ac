// A8: ordered sliced Gauss-Seidel (warp-psr relaxation.py:121-210) as a persistent,
// dependency-scheduled kernel over x-strips of each slice.
//
// Sequential definition: for front = 2^d .. -iters+1, for z in [max(front,0),
// min(front+iters, 2^d+1)), for colour 0..3 (colour = (x&1) + 2(y&1)): update every row of
// slice z with that colour (rows of one colour in one slice never couple).  Visit t of slice
// z needs visit t of z+1 and visit t-1 of z-1 (relaxation.py:128-135).  Any execution that
// honours those edges is bitwise identical to the sequential order.
//
// B200 mapping:
//  * rows are permuted into schedule order (slice, colour, x, y): the rows of one slice and
//    colour within an x-window are one contiguous position range;
//  * each slice-visit (z, t) is split into row-balanced x-strips; a strip task runs on one
//    CTA (one CTA per SM, persistent), tasks are taken in wave order (wave q = 2t + 2^d - z);
//  * a strip recomputes a halo of width 3-c around itself in colour phase c, so the four
//    colour phases need no synchronisation with neighbouring strips (the halo values are the
//    same arithmetic on the same inputs, hence bit-identical to the neighbour's);
//  * right after a task is taken, one thread issues bulk copies (cp.async.bulk, completion on
//    an mbarrier) of the task's operator rows, neighbour indices and right-hand side into
//    shared memory; they land while the task waits for its dependencies;
//  * once the dependencies are met the x footprint (three slices, x within 4 of the strip)
//    is staged in shared memory and the four phases run on shared memory only;
//  * neighbours are addressed by their index inside their (slice, colour) group; since the
//    colour of a phase is fixed, the footprint range of slot k is a compile-time function of
//    (colour, k) and a neighbour's footprint index is one addition;
//  * x is double-buffered by visit parity: visit t of a slice is written to buffer t&1, so a
//    strip never overwrites values another strip of the same visit still reads.  The slice
//    dependency edges order every reader of buffer t&1's previous contents before the write.
// Every wait is bounded; a timeout sets an error word, waits (bounded) for its own copies in
// flight, and every CTA exits.
#include "psr_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>

namespace psr {

constexpr int kSlotsR = 28;
constexpr int kIdxSlots = 32;  // neighbour index rows: slots 0..26, own index at 27, then 1 / A_ii

// The padding of an index row (slots 28..31, 8 bytes or more) carries the row's reciprocal
// diagonal 1 / A_ii in the vector precision, computed exactly as the update would
// (V(1) / V(A_ii)), so the sweep multiplies instead of dividing on its critical path.
template <class V, class I>
__host__ __device__ __forceinline__ void put_inv_diag(I* row, V inv) {
  static_assert(4 * sizeof(I) >= sizeof(V), "index padding too small for the reciprocal");
  memcpy(reinterpret_cast<char*>(row + 28), &inv, sizeof(V));
}
template <class V, class I>
__host__ __device__ __forceinline__ V get_inv_diag(const I* row) {
  V inv;
  memcpy(&inv, reinterpret_cast<const char*>(row + 28), sizeof(V));
  return inv;
}
constexpr int kFlagPad = 8;    // one 32-byte sector per strip flag
constexpr int kTraceSlots = 16;
constexpr int kRelaxThreads = 512;
// Resident CTAs per SM.  Measured at depth 9 (mixed, 16 strips): one 512-thread CTA per SM
// 3.01 ms, two 256-thread CTAs per SM with half the shared memory each 5.2 ms (tasks that no
// longer fit shared memory read their rows from global memory).
constexpr int kRelaxCtasPerSm = 1;
constexpr int kMetaInts = 96;

// One task description per (logical slice z, strip s), shared by the iters visits of that
// strip; built once per launch by strip_meta_kernel.  Footprint range r = 4j + c is colour
// c of logical slice z - 1 + j, x within 4 of the strip.
struct __align__(16) StripMeta {
  int lo[12], hi[12];        // schedule positions [lo, hi) of each footprint range
  int base[13];              // footprint offset of each range; base[12] = footprint size
  int delta[12];             // footprint index of a group-relative neighbour index i: i + delta[r]
  int p0[4], p1[4];          // rows updated in colour phase c: own rows plus a halo of width 3 - c
  int rbase[5];              // staged row offset of each colour's rows; rbase[4] = staged rows
  int bshift[4];             // staged right-hand-side offset of each colour's first row
  int o0[4], o1[4];          // own rows (x in [x0, x1)): published and recorded
  int staged;                // rows and right-hand sides fit shared memory (bulk copies)
  uint32_t bytes;            // bytes of those copies
  int dep_lo[3], dep_hi[3];  // strips of slices z-1, z, z+1 whose x range meets the footprint window
  int pad[14];
};
static_assert(sizeof(StripMeta) == kMetaInts * 4, "StripMeta is loaded as kMetaInts ints");

struct StripLevel {
  int n;                 // 2^depth (slices 0..n)
  int strips;            // strips per slice
  int nvisits;
  int cap;               // footprint capacity (elements) per CTA
  int row_cap;           // staged update rows per task
  int b_cap;             // staged right-hand-side elements per task
  const StripMeta* meta;     // [(n+1) * strips] by logical slice, then strip
  const void* vals;          // T[rows*28]   schedule order
  const void* nidx;          // I[rows*32]   neighbour index within its group, -1 absent; [27] = own
  const void* b;             // V[rows + slack]
  void* xb0;                 // V[rows]  even visits
  void* xb1;                 // V[rows]  odd visits (holds the initial x)
  const int2* visits;        // slice-visits (z, t) in wave order
  int* done;                 // visits completed by strip s of logical slice z at done[(z*strips + s) * kFlagPad]
  int* counter;
  int* error;
  long long* trace;          // optional, kTraceSlots per task: [0] start (globaltimer ns); [1..11] SM cycles from
                             // the start to: copies issued, own-slice wait done, first barrier, newest-slice wait
                             // done, second barrier, phases start, end of phase 0, 1, 2, 3, published; [15] CTA
  void* hist;                // optional V[rows * iters]: row p's record of visit t at p * iters + t
  int64_t rows;              // rows of the level
  int iters;                 // visits per slice
  int record_increment;      // hist holds the update r / A_ii (else the new x)
  int poll_log2;             // a dependency wait gives up after 2^poll_log2 polls
  int stall;                 // test override: the newest-slice wait targets a count nothing reaches
};

__device__ __forceinline__ long long globaltimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool wait_at_least(const int* p, int v, const int* error, int poll_log2) {
  const long long limit = 1LL << poll_log2;
  for (long long it = 0; it < limit; ++it) {
    if (ld_acquire(p) >= v) return true;
    if ((it & 63) == 63 && *(volatile const int*)error) return false;
    __nanosleep(it < 512 ? 32 : 256);
  }
  return false;
}

// The lanes of one warp wait together until strips [slo, shi] of logical slice zz have
// completed v visits (one strip per lane); false if any wait gave up.
__device__ __forceinline__ bool wait_strips(const StripLevel& L, int zz, int slo, int shi, int v, int lane) {
  bool ok = true;
  for (int sp = slo + lane; sp <= shi; sp += 32)
    ok = ok && wait_at_least(L.done + (int64_t(zz) * L.strips + sp) * kFlagPad, v, L.error, L.poll_log2);
  return __all_sync(0xffffffffu, ok);
}

// ---- mbarrier and 1-D bulk copy (global -> shared), no multicast
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long it = 0; it < (1LL << 26); ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Footprint range (j * 4 + colour) of slot k for a row of colour C: slice z-1+(k%3),
// colour of (x + k/9 - 1, y + (k/3)%3 - 1).
template <int C, bool M = false>
__device__ __forceinline__ constexpr int slot_range(int k) {
  return (M ? 2 - k % 3 : k % 3) * 4 + (((C & 1) + k / 9 + 1) & 1) + 2 * (((C >> 1) + (k / 3) % 3 + 1) & 1);
}

template <class T>
__device__ __forceinline__ void load_vals(const T* src, T out[kSlotsR]) {
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(out);
#pragma unroll
  for (int q = 0; q < kSlotsR * int(sizeof(T)) / 16; ++q) d[q] = s[q];
}

// One row of colour C: r = b - sum_k x_k A_k in slot order; x_self += r / A_self.
// Every slot takes part in the sum: an absent slot (value +0, index idx_absent) reads the +0
// entry kept at foot[total], and r - (+0 * +0) = r exactly, so the result is bitwise that of
// skipping it.  A present slot holds its k-th neighbour (checked where the rows are built),
// which lies in the footprint by construction; the unsigned clamp keeps every read inside
// the footprint whatever the rows hold.  Measured ~2x fewer instructions per slot than
// testing each slot's presence and range.  An own row (out != nullptr) is published to
// global memory as soon as it is computed: later phases of the strip do not change it.
template <int C, bool M, class T, class V, class I>
__device__ __forceinline__ void update_row(const I* nrow, int p, const T* arow, V bv, V* foot, const int* delta,
                                           unsigned total, int* error, V* rec, bool record_increment, V* out,
                                           V* out2 = nullptr) {
  __align__(16) I n[kIdxSlots];  // filled with 16-byte vector loads (stored row of position p)
  load_idx_row(nrow, p, n);
  __align__(16) T a[kSlotsR];
  load_vals(arow, a);
  V xs[27];
#pragma unroll
  for (int k = 0; k < 27; ++k)
    xs[k] = foot[min(unsigned(int(n[k])) + unsigned(delta[slot_range<C, M>(k)]), total)];
  V r = bv;
#pragma unroll
  for (int k = 0; k < 27; ++k) r = r - xs[k] * V(a[k]);
  const unsigned self = unsigned(int(n[27]) + delta[4 + C]);
  if (self >= total) {
    atomicExch(error, 3);
    return;
  }
  V inc = V(0), xn;
  if (n[13] >= 0 && a[13] != T(0)) {
    inc = r * get_inv_diag<V>(n);
    xn = xs[13] + inc;
    foot[self] = xn;
  } else {
    xn = foot[self];
  }
  if (out) __stcg(out, xn);
  if (out2) *out2 = xn;
  if (rec) *rec = record_increment ? inc : xn;
}

// `hist` (optional) points at this visit's record column (row p records at hist[p * iters]);
// only the strip's own rows [o0, o1) write it and are published to `out` (halo rows are
// recomputed by the neighbouring strip, which owns them).
template <int C, bool M, class T, class V, class I>
__device__ __forceinline__ void phase(const StripLevel& L, const StripMeta& m, bool staged, const I* s_idx,
                                      const T* s_vals, const V* s_b, V* foot, V* hist, V* out) {
  const I* gidx = reinterpret_cast<const I*>(L.nidx);
  const T* gvals = reinterpret_cast<const T*>(L.vals);
  const V* gb = reinterpret_cast<const V*>(L.b);
  const bool inc = L.record_increment != 0;
  const int p0 = m.p0[C], p1 = m.p1[C], o0 = m.o0[C], o1 = m.o1[C], rbase = m.rbase[C], bshift = m.bshift[C];
  const unsigned total = unsigned(m.base[12]);
  int dreg[12];  // footprint offsets in registers (measured ~1% faster than shared-memory reads)
#pragma unroll
  for (int r = 0; r < 12; ++r) dreg[r] = m.delta[r];
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    const bool own = p >= o0 && p < o1;
    V* rec = (hist && own) ? hist + int64_t(p) * L.iters : nullptr;
    if (staged) {
      int i = rbase + (p - p0);
      update_row<C, M>(s_idx + int64_t(i) * kIdxSlots, p, s_vals + int64_t(i) * kSlotsR, s_b[bshift + (p - p0)],
                       foot, dreg, total, L.error, rec, inc, own ? out + p : nullptr);
    } else {
      update_row<C, M>(gidx + int64_t(p) * kIdxSlots, p, gvals + int64_t(p) * kSlotsR, gb[p], foot, dreg, total,
                       L.error, rec, inc, own ? out + p : nullptr);
    }
  }
}

// REV false: colours 0..3 in the stored slice order (the forward sweep).  REV true: the exact
// reverse of that sweep on the same layout -- logical slice z is stored slice n - z (so slot
// k's neighbour lies in logical slice z + 1 - k % 3) and the colours run 3..0.  One
// instantiation per order keeps each kernel's body to its own four phases.
//
// Task (z, t, s) -- visit t of strip s of logical slice z -- waits for the strips whose x
// range meets its footprint window: of slice z after visit t-1 (early, while its operator
// rows are copied), then of slice z+1 after visit t and of slice z-1 after visit t-1.  Those
// waits also order every earlier reader of the x buffer it overwrites (visit t-2 of slice z,
// read by tasks (z, t-1), (z+1, t-1) and (z-1, t-2) of strips within 4 of its rows) before
// its first write: each of them is, or was waited for by, a strip this task waits for.  A
// strip publishes the number of its completed visits with a release (atomicMax, so the count
// only grows).
template <class T, class V, class I, bool REV>
__global__ void __launch_bounds__(kRelaxThreads, kRelaxCtasPerSm) strip_gs_kernel(StripLevel L) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_task[2], s_fail;
  __shared__ int2 s_zt[2];
  __shared__ __align__(16) StripMeta s_meta[2];
  // Shared layout (each part 16-byte aligned): footprint V[cap + 1] | values T[row_cap*28] |
  // neighbour indices I[row_cap*32] | right-hand side V[b_cap].
  V* foot = reinterpret_cast<V*>(smem_raw);
  const int64_t fp_bytes = (int64_t(L.cap + 1) * sizeof(V) + 15) & ~int64_t(15);
  T* s_vals = reinterpret_cast<T*>(smem_raw + fp_bytes);
  I* s_idx = reinterpret_cast<I*>(smem_raw + fp_bytes + int64_t(L.row_cap) * kSlotsR * sizeof(T));
  V* s_b = reinterpret_cast<V*>(smem_raw + fp_bytes +
                                int64_t(L.row_cap) * (kSlotsR * sizeof(T) + kIdxSlots * sizeof(I)));
  const T* gvals = reinterpret_cast<const T*>(L.vals);
  const I* gidx = reinterpret_cast<const I*>(L.nidx);
  const V* gb = reinterpret_cast<const V*>(L.b);
  V* xb0 = reinterpret_cast<V*>(L.xb0);
  V* xb1 = reinterpret_cast<V*>(L.xb1);
  const int total_tasks = L.nvisits * L.strips;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  uint32_t parity = 0;
  // Takes the next task and loads its description into s_task[b], s_meta[b] (one warp).
  auto fetch = [&](int b) {
    int task = 0;
    if (lane == 0) task = atomicAdd(L.counter, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (lane == 0) s_task[b] = task;
    if (task < total_tasks) {
      const int2 zt = L.visits[task / L.strips];
      if (lane == 0) s_zt[b] = zt;
      static_assert(kMetaInts / 4 <= 32, "one 16-byte load per lane");
      const int4* src = reinterpret_cast<const int4*>(L.meta + int64_t(zt.x) * L.strips + task % L.strips);
      if (lane < kMetaInts / 4) reinterpret_cast<int4*>(&s_meta[b])[lane] = __ldg(src + lane);
    }
  };
  if (threadIdx.x == 0) mbar_init(&s_bar);
  if (warp == 0) fetch(0);
  __syncthreads();
  for (int buf = 0;; buf ^= 1) {
    const int task = s_task[buf];
    if (task >= total_tasks) return;
    const StripMeta& m = s_meta[buf];
    long long* tr = (L.trace && threadIdx.x == 0) ? L.trace + int64_t(task) * kTraceSlots : nullptr;
    long long* trc = (L.trace && threadIdx.x == 32) ? L.trace + int64_t(task) * kTraceSlots : nullptr;
    const long long g0 = tr ? globaltimer() : 0;
    const long long c0 = (tr || trc) ? clock64() : 0;
    if (tr) {
      tr[0] = g0;
      tr[15] = blockIdx.x;
    }
    const int2 zt = s_zt[buf];
    const int z = zt.x, t = zt.y, s = task % L.strips;
    const bool staged = m.staged != 0;
    const int total = m.base[12];
    if (warp == 0) {
      if (lane == 0) {
        s_fail = 0;
        if (total > L.cap) {
          atomicExch(L.error, 2);
          s_fail = 1;
        }
      }
      __syncwarp();
      // slice z after visit t-1 (two waves back); the newer dependencies are awaited below
      // while this slice is staged
      if (!s_fail && !wait_strips(L, z, m.dep_lo[1], m.dep_hi[1], t, lane) && lane == 0) {
        atomicCAS(L.error, 0, 1);
        s_fail = 1;
      }
      if (tr && threadIdx.x == 0) tr[2] = clock64() - c0;
    } else if (warp == 1) {
      // Operator rows do not depend on x: one bulk copy per lane (values, indices and
      // right-hand side of each colour's rows) lands them while warp 0 waits for the
      // dependencies.  Issuing the copies takes ~0.8 us, so they are not on warp 0's path.
      if (staged && total <= L.cap) {
        if (lane == 0) mbar_expect_tx(&s_bar, m.bytes);
        __syncwarp();
        if (lane < 12) {
          constexpr int per16 = 16 / int(sizeof(V));
          const int c = lane / 3, kind = lane % 3;
          const int p0 = m.p0[c], cnt = m.p1[c] - p0;
          if (cnt > 0) {
            fence_proxy_async();
            if (kind == 0) {
              bulk_copy(s_vals + int64_t(m.rbase[c]) * kSlotsR, gvals + int64_t(p0) * kSlotsR,
                        uint32_t(cnt) * kSlotsR * sizeof(T), &s_bar);
            } else if (kind == 1) {
              bulk_copy(s_idx + int64_t(m.rbase[c]) * kIdxSlots, gidx + int64_t(p0) * kIdxSlots,
                        uint32_t(cnt) * kIdxSlots * sizeof(I), &s_bar);
            } else {
              const int a0 = p0 - p0 % per16, a1 = (m.p1[c] + per16 - 1) / per16 * per16;
              bulk_copy(s_b + (m.bshift[c] - p0 % per16), gb + a0, uint32_t(a1 - a0) * sizeof(V), &s_bar);
            }
          }
        }
      }
      if (trc) trc[1] = clock64() - c0;
    } else if (warp == nwarps - 1) {
      // The last warp takes the next task and loads its description meanwhile (the other
      // warps are idle until the barrier below).
      fetch(buf ^ 1);
    }
    __syncthreads();
    if (s_fail) {
      if (staged && total <= L.cap) mbar_wait(&s_bar, parity);  // never leave with copies in flight
      return;
    }
    if (tr && threadIdx.x == 0) tr[3] = clock64() - c0;
    // Stage the footprint: slice z+1 after visit t, slices z and z-1 after visit t-1.  Warp 0
    // waits for slices z+1 and z-1 while the other warps stage slice z, then all stage the rest.
    {
      const V* cur = (t & 1) ? xb1 : xb0;
      const V* prev = (t & 1) ? xb0 : xb1;
      // range r staged by `parts` warps, part `part` of them (4 loads in flight per lane)
      auto stage_range = [&](int r, int part, int parts) {
        const V* src = ((r >> 2) == 2 ? cur : prev) + m.lo[r];
        V* dst = foot + m.base[r];
        const int cnt = m.hi[r] - m.lo[r];
        for (int i0 = part * 128 + lane; i0 < cnt; i0 += 128 * parts) {
          V v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (i0 + 32 * u < cnt) v[u] = __ldcg(src + i0 + 32 * u);
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (i0 + 32 * u < cnt) dst[i0 + 32 * u] = v[u];
        }
      };
      if (warp == 0) {
        bool ok = true;
        if (z + 1 <= L.n)
          ok = wait_strips(L, z + 1, m.dep_lo[2], m.dep_hi[2], t + 1 + (L.stall ? (1 << 30) : 0), lane);
        if (ok && z > 0) ok = wait_strips(L, z - 1, m.dep_lo[0], m.dep_hi[0], t, lane);
        if (!ok && lane == 0) {
          atomicCAS(L.error, 0, 1);
          s_fail = 1;
        }
        if (tr && threadIdx.x == 0) tr[4] = clock64() - c0;
      } else {
        // slice z: 4 ranges over the other warps
        const int parts = max(1, (nwarps - 1) / 4);
        for (int q = warp - 1; q < 4 * parts; q += nwarps - 1) stage_range(4 + q / parts, q % parts, parts);
      }
      __syncthreads();
      if (tr && threadIdx.x == 0) tr[5] = clock64() - c0;
      if (s_fail) {
        if (staged) mbar_wait(&s_bar, parity);
        return;
      }
      {  // slices z-1 and z+1: 8 ranges over all warps
        const int parts = max(1, nwarps / 8);
        for (int q = warp; q < 8 * parts; q += nwarps) {
          const int rr = q / parts;
          stage_range(rr < 4 ? rr : rr + 4, q % parts, parts);
        }
      }
    }
    if (threadIdx.x == 0) foot[total] = V(0);  // the entry absent slots read
    if (staged && !mbar_wait(&s_bar, parity)) {
      if (threadIdx.x == 0) atomicExch(L.error, 4);
      return;
    }
    if (staged) parity ^= 1;
    __syncthreads();
    if (tr && threadIdx.x == 0) tr[6] = clock64() - c0;
    {
      V* hv = L.hist ? reinterpret_cast<V*>(L.hist) + t : nullptr;
      V* out = (t & 1) ? xb1 : xb0;
#define PSR_PHASE(C, M, K)                                                \
  phase<C, M, T, V, I>(L, m, staged, s_idx, s_vals, s_b, foot, hv, out); \
  __syncthreads();                                                        \
  if (tr && threadIdx.x == 0) tr[7 + K] = clock64() - c0;
      if (!REV) {
        PSR_PHASE(0, false, 0) PSR_PHASE(1, false, 1) PSR_PHASE(2, false, 2) PSR_PHASE(3, false, 3)
      } else {
        PSR_PHASE(3, true, 0) PSR_PHASE(2, true, 1) PSR_PHASE(1, true, 2) PSR_PHASE(0, true, 3)
      }
#undef PSR_PHASE
    }
    // The strip's own rows were published in their phases: release visit t.  (Measured: from
    // another warp, overlapping the next task's bulk copies, the release takes longer and the
    // launch is ~7% slower.)
    if (threadIdx.x == 0) {
      __threadfence();
      atomicMax(L.done + (int64_t(z) * L.strips + s) * kFlagPad, t + 1);
      if (tr) tr[11] = clock64() - c0;
    }
  }
}

// Task descriptions of one launch: one thread per (logical slice z, strip s).  Error 2: a
// footprint exceeds the capacity (the kernel then stops before staging it).
template <bool REV>
__global__ void strip_meta_kernel(const int32_t* xstart, const int32_t* bounds, const int32_t* group_off, int n,
                                  int strips, int per16, int cap, int row_cap, int b_cap, int row_bytes,
                                  int vbytes, StripMeta* meta) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (n + 1) * strips) return;
  const int z = idx / strips, s = idx % strips, nx = n + 2;
  auto phys = [&](int zz) { return REV ? n - zz : zz; };
  const int32_t* bz = bounds + int64_t(phys(z)) * (strips + 1);
  const int x0 = bz[s], x1 = bz[s + 1];
  const int xa = max(x0 - 4, 0), xb = min(x1 + 4, n + 1);
  StripMeta m;
  int total = 0;
  for (int r = 0; r < 12; ++r) {
    const int j = r >> 2, c = r & 3, zz = z + j - 1;
    int lo = 0, hi = 0, gstart = 0;
    if (zz >= 0 && zz <= n) {
      const int32_t* xs = xstart + int64_t(phys(zz) * 4 + c) * nx;
      lo = xs[xa];
      hi = xs[xb];
      gstart = group_off[phys(zz) * 4 + c];
    }
    m.lo[r] = lo;
    m.hi[r] = hi;
    m.base[r] = total;
    m.delta[r] = total + gstart - lo;
    total += hi - lo;
  }
  m.base[12] = total;
  int rows = 0, bsum = 0;
  uint32_t bytes = 0;
  for (int c = 0; c < 4; ++c) {
    const int32_t* xs = xstart + int64_t(phys(z) * 4 + c) * nx;
    const int h = REV ? c : 3 - c;
    const int p0 = xs[max(min(x0 - h, n + 1), 0)], p1 = xs[min(x1 + h, n + 1)];
    m.p0[c] = p0;
    m.p1[c] = p1;
    m.o0[c] = xs[x0];
    m.o1[c] = xs[min(x1, n + 1)];
    m.rbase[c] = rows;
    rows += p1 - p0;
    const int a0 = p0 - p0 % per16, a1 = (p1 + per16 - 1) / per16 * per16;
    m.bshift[c] = bsum + (p0 - a0);
    if (p1 > p0) {
      bsum += a1 - a0;
      bytes += uint32_t(p1 - p0) * uint32_t(row_bytes) + uint32_t(a1 - a0) * uint32_t(vbytes);
    }
  }
  m.rbase[4] = rows;
  m.staged = total <= cap && rows <= row_cap && bsum <= b_cap;
  m.bytes = bytes;
  for (int j = 0; j < 3; ++j) {
    const int zz = z + j - 1;
    int lo = strips, hi = -1;
    if (zz >= 0 && zz <= n) {
      const int32_t* bb = bounds + int64_t(phys(zz)) * (strips + 1);
      for (int sp = 0; sp < strips; ++sp)
        if (bb[sp] < bb[sp + 1] && bb[sp] < xb && bb[sp + 1] > xa) {
          lo = min(lo, sp);
          hi = max(hi, sp);
        }
    }
    m.dep_lo[j] = lo;
    m.dep_hi[j] = hi;
  }
  for (int i = 0; i < 14; ++i) m.pad[i] = 0;
  meta[idx] = m;
}

// ------------------------------------------------------------------ cluster pipelines
// The same order run as one pipeline per visit.  Visit t's pipeline is one cluster of
// kPipeCtas CTAs (strip s = rank) that relaxes slices z = 2^d .. 0 in turn (step = 2^d - z),
// which is the order in which the sequential sweep gives visit t to the slices.  Visit t of
// slice z needs:
//  * slice z+1 after visit t -- the previous step of the same pipeline: each CTA keeps its
//    own rows' new values of every step in an export buffer in shared memory, and the CTAs
//    read their neighbours' through distributed shared memory after a cluster barrier;
//  * slices z and z-1 after visit t-1 -- pipeline t-1, one and two steps earlier: through
//    global memory (x buffer of visit parity t-1) and per-strip completion counts, as in the
//    dynamic scheduler above, staged by helper warps during the previous step.
// So a step costs its four colour phases, one cluster barrier and the neighbour exchange in
// shared memory; the global-memory hand-off between pipelines is paid once per visit (the
// pipelines run staggered), not once per slice.  Operator rows are brought in per colour phase
// by bulk copies into two alternating regions, issued two phases ahead; a phase with more rows
// than a region holds (polar slices: the few largest tasks) reads its rows from global memory.
//
// Warps 0..11 update rows; warp 12 loads the next step's task description and issues the bulk
// copies and the release of each step; warps 13..15 stage the next step's global ranges.  Every
// wait is bounded; after an error the CTAs keep taking part in the barriers (skipping the work)
// until the loop ends, so no barrier is left waiting, and drain their copies before exiting.
constexpr int kPipeCtas = 8;
constexpr int kPipeRowThreads = 384;
constexpr int kPipeRegions = 2;
constexpr int kMaxPeerSegs = 40;

struct PeerSeg {
  int rank, src, dst, count;  // values [src, src+count) of CTA `rank`'s export -> footprint [dst, dst+count)
};
struct PipeMeta {
  StripMeta m;   // footprint layout padded: every range starts where its first element's
                 // offset from a 16-byte boundary matches the x buffers' (bulk copies)
  int ebase[5];  // export offset of each colour's own rows (colour-major); ebase[4] = own rows
  int nseg, overflow, npush;
  PeerSeg seg[kMaxPeerSegs];      // the slice z+1 footprint ranges, by owner (pulled: rank = owner)
  PeerSeg push[kMaxPeerSegs];     // this task's exports pushed into the next step's footprints
                                  // (rank = receiving CTA, dst = its footprint offset)
  int pushoff[kMaxPeerSegs + 4];  // values before each push segment; pushoff[npush] = all of them
};
constexpr int kPipeMetaInts = int(sizeof(PipeMeta) / 4);
static_assert(sizeof(PipeMeta) % 16 == 0, "PipeMeta is copied as ints into 16-byte aligned shared memory");

struct PipeLevel {
  StripLevel L;  // n, strips (= kPipeCtas), vals, nidx, b, xb0, xb1, done, error, hist, iters, ...
  const PipeMeta* meta;
  int cap;       // footprint elements
  int rcap;      // rows per region
  int bcap;      // right-hand-side elements per region
  int ecap;      // exported values per step
  int64_t off_foot[2], off_vals[kPipeRegions], off_idx[kPipeRegions], off_b[kPipeRegions], off_exp[2], off_meta[2];
};

__device__ __forceinline__ void bar_named(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
// Cluster barrier in two halves (each warp, converged): arrive releases this thread's writes
// (shared memory of any CTA of the cluster, global memory); wait acquires the others'.
__device__ __forceinline__ void cluster_arrive() {
  __syncwarp();
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  __syncwarp();
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

template <int C, bool M, class T, class V, class I>
__device__ __forceinline__ void pipe_phase(const StripLevel& L, const StripMeta& m, const int* ebase, const I* r_idx,
                                           const T* r_vals, const V* r_b, V* foot, V* hist, V* out, V* expo,
                                           int rcap, int bcap) {
  constexpr int per16 = 16 / int(sizeof(V));
  const bool inc = L.record_increment != 0;
  const int p0 = m.p0[C], p1 = m.p1[C], o0 = m.o0[C], o1 = m.o1[C];
  int bshift = p0 % per16;
  const int a1 = (p1 + per16 - 1) / per16 * per16;
  if (p1 - p0 > rcap || a1 - (p0 - bshift) > bcap) {  // not staged: the rows in global memory
    r_idx = reinterpret_cast<const I*>(L.nidx) + int64_t(p0) * kIdxSlots;
    r_vals = reinterpret_cast<const T*>(L.vals) + int64_t(p0) * kSlotsR;
    r_b = reinterpret_cast<const V*>(L.b) + p0;
    bshift = 0;
  }
  const unsigned total = unsigned(m.base[12]);
  int dreg[12];
#pragma unroll
  for (int r = 0; r < 12; ++r) dreg[r] = m.delta[r];
  for (int p = p0 + int(threadIdx.x); p < p1; p += kPipeRowThreads) {
    const bool own = p >= o0 && p < o1;
    V* rec = (hist && own) ? hist + int64_t(p) * L.iters : nullptr;
    const int i = p - p0;
    update_row<C, M>(r_idx + int64_t(i) * kIdxSlots, p, r_vals + int64_t(i) * kSlotsR, r_b[bshift + i], foot, dreg,
                     total, L.error, rec, inc, own ? out + p : nullptr, own ? expo + ebase[C] + (p - o0) : nullptr);
  }
}

template <class T, class V, class I, bool REV>
__global__ void __launch_bounds__(kRelaxThreads, 1) pipeline_gs_kernel(PipeLevel P) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_full[kPipeRegions];   // rows of the region's phase have landed
  __shared__ uint64_t s_empty[kPipeRegions];  // the region's phase is done with them
  __shared__ uint64_t s_gfull[2];             // foot[b]'s slices from the previous visit have landed
  __shared__ int s_err;
  const StripLevel& L = P.L;
  const int t = int(blockIdx.x) / kPipeCtas;
  const int s = int(cluster.block_rank());
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsteps = L.n + 1, nphases = 4 * nsteps;
  V* foot[2] = {reinterpret_cast<V*>(smem_raw + P.off_foot[0]), reinterpret_cast<V*>(smem_raw + P.off_foot[1])};
  V* expo[2] = {reinterpret_cast<V*>(smem_raw + P.off_exp[0]), reinterpret_cast<V*>(smem_raw + P.off_exp[1])};
  PipeMeta* sm[2] = {reinterpret_cast<PipeMeta*>(smem_raw + P.off_meta[0]),
                     reinterpret_cast<PipeMeta*>(smem_raw + P.off_meta[1])};
  const T* gvals = reinterpret_cast<const T*>(L.vals);
  const I* gidx = reinterpret_cast<const I*>(L.nidx);
  const V* gb = reinterpret_cast<const V*>(L.b);
  V* xout = reinterpret_cast<V*>((t & 1) ? L.xb1 : L.xb0);         // x after visit t
  const V* xprev = reinterpret_cast<const V*>((t & 1) ? L.xb0 : L.xb1);  // after visit t-1 (t = 0: initial x)
  V* hv = L.hist ? reinterpret_cast<V*>(L.hist) + t : nullptr;
  if (threadIdx.x == 0) {
    for (int r = 0; r < kPipeRegions; ++r) {
      mbar_init(&s_full[r]);
      mbar_init(&s_empty[r]);
    }
    mbar_init(&s_gfull[0]);
    mbar_init(&s_gfull[1]);
    s_err = 0;
  }
  auto fail = [&](int code) {
    atomicCAS(L.error, 0, code);
    s_err = 1;
  };
  // warp 12: the task description of a step into sm[step & 1] -- every 16-byte load issued
  // before the first store (a load/store loop serialises on the loads' latency)
  auto load_meta = [&](int step) {
    constexpr int kVecs = int(sizeof(PipeMeta) / 16), kPer = (kVecs + 31) / 32;
    const int z = L.n - step;
    const int4* src = reinterpret_cast<const int4*>(P.meta + (int64_t(z) * kPipeCtas + s));
    int4* dst = reinterpret_cast<int4*>(sm[step & 1]);
    int4 v[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u)
      if (lane + 32 * u < kVecs) v[u] = __ldg(src + lane + 32 * u);
#pragma unroll
    for (int u = 0; u < kPer; ++u)
      if (lane + 32 * u < kVecs) dst[lane + 32 * u] = v[u];
  };
  int last_issued[kPipeRegions];  // thread 384: the last phase issued into each region
  for (int r = 0; r < kPipeRegions; ++r) last_issued[r] = -1;
  // thread 384: bulk copies of phase k's rows into region k % kPipeRegions (phases with no rows,
  // or more than a region holds, only arrive)
  auto issue = [&](int k) {
    last_issued[k % kPipeRegions] = k;
    constexpr int per16 = 16 / int(sizeof(V));
    const int step = k / 4, col = REV ? 3 - k % 4 : k % 4, r = k % kPipeRegions;
    const StripMeta& m = sm[step & 1]->m;
    const int p0 = m.p0[col], cnt = m.p1[col] - p0;
    const int a0 = p0 - p0 % per16, a1 = (m.p1[col] + per16 - 1) / per16 * per16;
    const bool ok = cnt > 0 && cnt <= P.rcap && a1 - a0 <= P.bcap;  // else the phase reads global rows
    const uint32_t bytes =
        ok ? uint32_t(cnt) * (kSlotsR * sizeof(T) + kIdxSlots * sizeof(I)) + uint32_t(a1 - a0) * sizeof(V) : 0;
    fence_proxy_async();
    mbar_expect_tx(&s_full[r], bytes);
    if (ok) {
      bulk_copy(smem_raw + P.off_vals[r], gvals + int64_t(p0) * kSlotsR, uint32_t(cnt) * kSlotsR * sizeof(T),
                &s_full[r]);
      bulk_copy(smem_raw + P.off_idx[r], gidx + int64_t(p0) * kIdxSlots, uint32_t(cnt) * kIdxSlots * sizeof(I),
                &s_full[r]);
      bulk_copy(smem_raw + P.off_b[r], gb + a0, uint32_t(a1 - a0) * sizeof(V), &s_full[r]);
    }
  };
  // warp 13: footprint ranges of slices z and z-1 after visit t-1 for a step, into
  // foot[step & 1] by bulk copies (completion on s_gfull[step & 1]), once pipeline t-1 has
  // published them.  The flag reads are generic-proxy acquires; the proxy fence orders the
  // copies' async-proxy reads of the released values after them.
  int gissued[2] = {-1, -1};  // warp 13 lane 0: the last step whose copies went into each buffer
  auto stage_global = [&](int step) {
    const StripMeta& m = sm[step & 1]->m;
    const int z = L.n - step;
    bool ok = !s_err;
    if (ok) ok = wait_strips(L, z, m.dep_lo[1], m.dep_hi[1], t, lane);
    if (ok && z > 0) ok = wait_strips(L, z - 1, m.dep_lo[0], m.dep_hi[0], t, lane);
    if (!ok && lane == 0 && !s_err) fail(1);
    if (lane == 0) {
      constexpr int per16 = 16 / int(sizeof(V));
      uint32_t bytes = 0;
      if (ok)
        for (int r = 0; r < 8; ++r)
          if (m.hi[r] > m.lo[r])
            bytes += uint32_t((m.hi[r] + per16 - 1) / per16 * per16 - (m.lo[r] - m.lo[r] % per16)) * sizeof(V);
      asm volatile("fence.proxy.async.global;" ::: "memory");
      fence_proxy_async();
      gissued[step & 1] = step;
      mbar_expect_tx(&s_gfull[step & 1], bytes);
      if (ok) {
        V* f = foot[step & 1];
        for (int r = 0; r < 8; ++r) {
          if (m.hi[r] <= m.lo[r]) continue;
          const int lo = m.lo[r] - m.lo[r] % per16, hi = (m.hi[r] + per16 - 1) / per16 * per16;
          bulk_copy(f + (m.base[r] - m.lo[r] % per16), xprev + lo, uint32_t(hi - lo) * sizeof(V), &s_gfull[step & 1]);
        }
      }
    }
    __syncwarp();
  };
  __syncthreads();
  // prologue: step 0's description, its first phases' rows, its global ranges
  if (warp == 12) load_meta(0);
  __syncthreads();
  if (threadIdx.x == 12 * 32)
    for (int k = 0; k < kPipeRegions && k < nphases; ++k) issue(k);
  if (warp == 13) stage_global(0);
  __syncthreads();
  cluster.sync();  // every CTA of the cluster has initialised its shared memory
  for (int step = 0; step < nsteps; ++step) {
    const int z = L.n - step, fb = step & 1;
    const PipeMeta& pm = *sm[fb];
    const StripMeta& m = pm.m;
    // trace (optional): per (visit, strip, step) 16 values: [0] step start (globaltimer ns);
    // [1..6] SM cycles from then to the phases' start, the end of phase 0..3 and the cluster
    // barrier's end; [7] the global ranges of the next step staged (globaltimer ns); [8..11]
    // SM cycles to each phase's rows being in place; [12..15] (copy thread) SM cycles to the
    // copies of phase k + 2 being issued
    long long* tr = L.trace ? L.trace + ((int64_t(t) * kPipeCtas + s) * nsteps + step) * 16 : nullptr;
    const long long c0 = (tr && (threadIdx.x == 0 || threadIdx.x == 12 * 32)) ? clock64() : 0;
    if (tr && threadIdx.x == 0) tr[0] = globaltimer();
    // slices z and z-1 after visit t-1 (copied in during the previous step); slice z+1 after
    // visit t was pushed into foot[fb] by the peers before the cluster barrier
    if (warp < 12 && !s_err && !mbar_wait(&s_gfull[fb], uint32_t(step >> 1) & 1)) fail(4);
    if (threadIdx.x == 0) foot[fb][m.base[12]] = V(0);
    __syncthreads();
    if (tr && threadIdx.x == 0) tr[1] = clock64() - c0;
    if (warp < 12) {
#define PSR_PIPE_PHASE(CI)                                                                                         \
  {                                                                                                                \
    const int k = 4 * step + CI;                                                                                   \
    constexpr int col = REV ? 3 - CI : CI;                                                                         \
    const int r = k % kPipeRegions;                                                                                \
    if (!s_err && !mbar_wait(&s_full[r], uint32_t(k / kPipeRegions) & 1)) fail(4);                              \
    if (tr && threadIdx.x == 0) tr[8 + CI] = clock64() - c0;                                                       \
    if (!s_err)                                                                                                    \
      pipe_phase<col, REV, T, V, I>(L, m, pm.ebase, reinterpret_cast<const I*>(smem_raw + P.off_idx[r]),          \
                                    reinterpret_cast<const T*>(smem_raw + P.off_vals[r]),                          \
                                    reinterpret_cast<const V*>(smem_raw + P.off_b[r]), foot[fb], hv, xout,         \
                                    expo[fb], P.rcap, P.bcap);                                                     \
    bar_named(1, kPipeRowThreads);                                                                                 \
    if (threadIdx.x == 0) mbar_arrive(&s_empty[r]);                                                                \
    if (tr && threadIdx.x == 0) tr[2 + CI] = clock64() - c0;                                                       \
  }
      PSR_PIPE_PHASE(0) PSR_PIPE_PHASE(1) PSR_PIPE_PHASE(2) PSR_PIPE_PHASE(3)
#undef PSR_PIPE_PHASE
      // push this step's new values of slice z into the peers' next footprints (remote
      // stores; the cluster barrier makes them visible)
      if (step + 1 < nsteps && !s_err) {
        const int total = pm.pushoff[min(pm.npush, kMaxPeerSegs)];
        int g = 0;
        for (int e = threadIdx.x; e < total; e += kPipeRowThreads) {
          while (pm.pushoff[g + 1] <= e) ++g;
          const PeerSeg& sg = pm.push[g];
          V* remote = cluster.map_shared_rank(foot[(step + 1) & 1], sg.rank);
          remote[sg.dst + (e - pm.pushoff[g])] = expo[fb][sg.src + (e - pm.pushoff[g])];
        }
      }
      cluster_arrive();
    } else if (warp == 12) {
      if (step + 1 < nsteps) load_meta(step + 1);
      __syncwarp();
      bar_named(2, 128);  // the next step's description is in place for warps 13..15
      if (lane == 0) {
        for (int ci = 0; ci < 4; ++ci) {
          // the region of phase k is free once phase k is done; then the copies of phase
          // k + kPipeRegions go in.  (One full and one empty barrier per region: neither can run
          // a phase ahead of the other, so a parity wait never confuses two phases.)
          const int k = 4 * step + ci;
          if (!mbar_wait(&s_empty[k % kPipeRegions], uint32_t(k / kPipeRegions) & 1) && !s_err) fail(4);
          if (k + kPipeRegions < nphases && !s_err) issue(k + kPipeRegions);
          if (tr) tr[12 + ci] = clock64() - c0;  // copies of phase k + 2 issued (cycles from this thread's step start)
        }
      }
      __syncwarp();
      cluster_arrive();  // this warp's part of the step is done; the release below overlaps the barrier
      if (lane == 0 && !s_err) {  // release slice z after visit t to pipeline t+1
        __threadfence();
        atomicMax(L.done + (int64_t(z) * L.strips + s) * kFlagPad, t + 1);
      }
      __syncwarp();
    } else {
      bar_named(2, 128);
      cluster_arrive();  // the next step's staging (bulk copies) overlaps the barrier
      if (warp == 13 && step + 1 < nsteps) stage_global(step + 1);
      if (tr && threadIdx.x == 13 * 32) tr[7] = globaltimer();
    }
    cluster_wait();
    if (tr && threadIdx.x == 0) tr[6] = clock64() - c0;
  }
  // never leave with copies in flight (after an error some were not consumed)
  if (threadIdx.x == 12 * 32)
    for (int r = 0; r < kPipeRegions; ++r)
      if (last_issued[r] >= 0) mbar_wait(&s_full[r], uint32_t(last_issued[r] / kPipeRegions) & 1);
  if (threadIdx.x == 13 * 32)
    for (int b = 0; b < 2; ++b)
      if (gissued[b] >= 0) mbar_wait(&s_gfull[b], uint32_t(gissued[b] >> 1) & 1);
  __syncthreads();
}

// Padded footprint layout, peer segments and export offsets of the cluster pipelines, one
// thread per (logical slice z, strip s); strip_meta holds the StripMeta of the same tasks.
template <bool REV>
__global__ void pipe_meta_kernel(const StripMeta* strip_meta, const int32_t* xstart, const int32_t* bounds,
                                 const int32_t* group_off, int n, int per16, PipeMeta* meta, int* caps) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (n + 1) * kPipeCtas) return;
  const int z = idx / kPipeCtas, nx = n + 2;
  auto phys = [&](int zz) { return REV ? n - zz : zz; };
  PipeMeta pm;
  pm.m = strip_meta[idx];
  StripMeta& m = pm.m;
  // range r starts at base[r] with base[r] = lo[r] (mod per16), after the previous range's
  // 16-byte-rounded end, so that a bulk copy of [lo rounded down, hi rounded up) lands in place
  int tot = 0;
  for (int r = 0; r < 12; ++r) {
    const int j = r >> 2, c = r & 3, zz = z + j - 1;
    const int gstart = (zz >= 0 && zz <= n) ? group_off[phys(zz) * 4 + c] : 0;
    const int start = (tot + per16 - 1) / per16 * per16;
    m.base[r] = start + m.lo[r] % per16;
    m.delta[r] = m.base[r] + gstart - m.lo[r];
    tot = m.base[r] + (m.hi[r] - m.lo[r]) + ((m.hi[r] + per16 - 1) / per16 * per16 - m.hi[r]);
  }
  m.base[12] = tot;
  int e = 0;
  for (int c = 0; c < 4; ++c) {
    pm.ebase[c] = e;
    e += m.o1[c] - m.o0[c];
  }
  pm.ebase[4] = e;
  pm.nseg = 0;
  pm.overflow = 0;
  pm.npush = 0;
  const int zz = z + 1;
  if (zz <= n) {
    const int32_t* bb = bounds + int64_t(phys(zz)) * (kPipeCtas + 1);
    for (int sp = m.dep_lo[2]; sp <= m.dep_hi[2]; ++sp) {
      int ob[4], o0s[4], o1s[4], acc = 0;
      for (int c = 0; c < 4; ++c) {
        const int32_t* xs = xstart + int64_t(phys(zz) * 4 + c) * nx;
        o0s[c] = xs[bb[sp]];
        o1s[c] = xs[bb[sp + 1]];
        ob[c] = acc;
        acc += o1s[c] - o0s[c];
      }
      for (int c = 0; c < 4; ++c) {
        const int r = 8 + c;
        const int a = max(m.lo[r], o0s[c]), b = min(m.hi[r], o1s[c]);
        if (a >= b) continue;
        if (pm.nseg < kMaxPeerSegs) {
          pm.seg[pm.nseg] = PeerSeg{sp, ob[c] + (a - o0s[c]), m.base[r] + (a - m.lo[r]), b - a};
          ++pm.nseg;
        } else {
          pm.overflow = 1;
        }
      }
    }
  }
  for (int g = pm.nseg; g < kMaxPeerSegs; ++g) pm.seg[g] = PeerSeg{0, 0, 0, 0};
  for (int g = 0; g < kMaxPeerSegs; ++g) pm.push[g] = PeerSeg{0, 0, 0, 0};
  for (int g = 0; g < kMaxPeerSegs + 4; ++g) pm.pushoff[g] = 0;
  meta[idx] = pm;
  // capacities: footprint, rows per colour, exported values, overflow (right-hand-side spans:
  // pipe_bspan_kernel)
  atomicMax(caps + 0, tot + per16);
  for (int c = 0; c < 4; ++c) atomicMax(caps + 1, m.p1[c] - m.p0[c]);
  atomicMax(caps + 3, e);
  if (pm.overflow) atomicMax(caps + 4, 1);
}

// Inverts the pull segments: the segment of consumer (z, s') reading owner rank s of slice
// z+1 becomes a push segment of task (z+1, s), with the consumer's rank and footprint offset.
__global__ void pipe_push_kernel(PipeMeta* meta, int n, int* caps) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * kPipeCtas) return;  // consumers z = 0 .. n-1
  const int z = idx / kPipeCtas, sc = idx % kPipeCtas;
  const PipeMeta& cm = meta[idx];
  for (int g = 0; g < cm.nseg; ++g) {
    const PeerSeg sg = cm.seg[g];
    PipeMeta& pr = meta[(z + 1) * kPipeCtas + sg.rank];
    const int slot = atomicAdd(&pr.npush, 1);
    if (slot < kMaxPeerSegs)
      pr.push[slot] = PeerSeg{sc, sg.src, sg.dst, sg.count};
    else
      atomicMax(caps + 4, 1);
  }
}

__global__ void pipe_pushoff_kernel(PipeMeta* meta, int count) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= count) return;
  PipeMeta& pm = meta[idx];
  const int np = min(pm.npush, kMaxPeerSegs);
  int acc = 0;
  for (int g = 0; g < kMaxPeerSegs + 4; ++g) {
    pm.pushoff[g] = acc;
    if (g < np) acc += pm.push[g].count;
  }
}

__global__ void pipe_bspan_kernel(const PipeMeta* meta, int count, int per16, int* caps) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= count) return;
  const StripMeta& m = meta[idx].m;
  for (int c = 0; c < 4; ++c) {
    if (m.p1[c] <= m.p0[c]) continue;
    const int a0 = m.p0[c] - m.p0[c] % per16, a1 = (m.p1[c] + per16 - 1) / per16 * per16;
    atomicMax(caps + 2, a1 - a0);
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

// Row-balanced strip boundaries: slice z's rows split into `strips` runs of x of about equal size.
__global__ void strip_bounds_kernel(const int32_t* xstart, int n, int strips, int32_t* bounds) {
  // One thread per (slice z, boundary k): boundary k is the smallest Y in [1, n+1] with
  // rows(x < Y) * strips >= k * rows(slice), found by binary search (rows(x < Y) grows with Y).
  const int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (idx >= int64_t(n + 1) * (strips + 1)) return;
  const int z = int(idx / (strips + 1)), k = int(idx % (strips + 1));
  int32_t* out = bounds + int64_t(z) * (strips + 1);
  if (k == 0) {
    out[0] = 0;
    return;
  }
  if (k == strips) {
    out[strips] = n + 1;
    return;
  }
  const int nx = n + 2;
  const int32_t* xs = xstart + int64_t(z * 4) * nx;
  auto rows_below = [&](int Y) {
    int r = 0;
    for (int c = 0; c < 4; ++c) r += xs[c * nx + Y] - xs[c * nx];
    return r;
  };
  const int64_t total = rows_below(n + 1);
  int lo = 1, hi = n + 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (int64_t(rows_below(mid)) * strips >= int64_t(k) * total)
      hi = mid;
    else
      lo = mid + 1;
  }
  out[k] = lo;
}

// Largest footprint, update-row count and staged right-hand-side span over all tasks.
__global__ void footprint_kernel(const int32_t* xstart, const int32_t* bounds, int n, int strips, int per16, int rev,
                                 int* caps) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (n + 1) * strips) return;
  int z = idx / strips, s = idx % strips, nx = n + 2;
  int x0 = bounds[z * (strips + 1) + s], x1 = bounds[z * (strips + 1) + s + 1];
  int rows = 0, bspan = 0;
  for (int c = 0; c < 4; ++c) {
    const int32_t* xs = xstart + int64_t(z * 4 + c) * nx;
    int h = rev ? c : 3 - c;
    int p0 = xs[max(min(x0 - h, n + 1), 0)], p1 = xs[min(x1 + h, n + 1)];
    rows += p1 - p0;
    if (p1 > p0) bspan += (p1 + per16 - 1) / per16 * per16 - (p0 - p0 % per16);
  }
  atomicMax(caps + 1, rows);
  atomicMax(caps + 2, bspan);
  int total = 0;
  for (int j = -1; j <= 1; ++j) {
    int zz = z + j;
    if (zz < 0 || zz > n) continue;
    for (int c = 0; c < 4; ++c) {
      const int32_t* xs = xstart + int64_t(zz * 4 + c) * nx;
      total += xs[min(x1 + 4, n + 1)] - xs[max(x0 - 4, 0)];
    }
  }
  atomicMax(caps, total);
}

// Tasks whose update rows or right-hand sides exceed the staging capacity (they read their
// rows from global memory), added to caps[3].  The capacity follows from footprint_kernel's
// caps[0..2] as the launch computes it: rows of row_bytes + vbytes that fit `budget` beside a
// footprint of caps[0] elements (and its +0 entry).
__global__ void unstaged_kernel(const int32_t* xstart, const int32_t* bounds, int n, int strips, int per16, int rev,
                                int64_t budget, int row_bytes, int vbytes, int* caps) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (n + 1) * strips) return;
  const int64_t fp_bytes = (int64_t(max(caps[0], 1) + 1) * vbytes + 15) & ~int64_t(15);
  const int64_t rc = max(int64_t(0), min(int64_t(caps[1]), (budget - fp_bytes - 4 * 16) / (row_bytes + vbytes)));
  const int row_cap = int(rc);
  const int b_cap = int(min(int64_t(caps[2]), rc + 4 * per16) / per16 * per16);
  int* count = caps + 3;
  int z = idx / strips, s = idx % strips, nx = n + 2;
  int x0 = bounds[z * (strips + 1) + s], x1 = bounds[z * (strips + 1) + s + 1];
  int rows = 0, bspan = 0;
  for (int c = 0; c < 4; ++c) {
    const int32_t* xs = xstart + int64_t(z * 4 + c) * nx;
    int h = rev ? c : 3 - c;
    int p0 = xs[max(min(x0 - h, n + 1), 0)], p1 = xs[min(x1 + h, n + 1)];
    rows += p1 - p0;
    if (p1 > p0) bspan += (p1 + per16 - 1) / per16 * per16 - (p0 - p0 % per16);
  }
  if (rows > row_cap || bspan > b_cap) atomicAdd(count, 1);
}

__global__ void inverse_kernel(const int32_t* perm, int64_t n, int32_t* inv) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) inv[perm[p]] = int32_t(p);
}

__device__ __forceinline__ int group_of(int64_t key) {
  int c[3];
  key_coords(key, c);
  return 4 * c[2] + (c[0] & 1) + 2 * (c[1] & 1);
}

// Gathers a slot-ELL operator (key order) into schedule order; neighbours become indices
// inside their (slice, colour) group.
template <class T, class V, class I>
__global__ void reorder_kernel(const int32_t* perm, const int32_t* inv, const int32_t* group_off, int64_t n,
                               const int32_t* cols, const T* vals, const V* b, const V* x, const int64_t* keys,
                               I* sidx, T* svals, V* sb, V* sx, int64_t* skeys) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  int64_t row = perm[p];
  __align__(16) I idx[kIdxSlots];
  for (int k = 0; k < kSlotsR; ++k) {
    int32_t c = k < 27 ? cols[row * kSlotsR + k] : -1;
    idx[k] = idx_absent<I>();
    if (c >= 0) idx[k] = I(inv[c] - group_off[group_of(keys[c])]);
    svals[p * kSlotsR + k] = k < 27 ? vals[row * kSlotsR + k] : T(0);
  }
  idx[27] = I(p - group_off[group_of(keys[row])]);
  for (int k = 28; k < kIdxSlots; ++k) idx[k] = I(-1);
  const T diag = vals[row * kSlotsR + 13];
  put_inv_diag<V>(idx, diag != T(0) ? V(1.0) / V(diag) : V(0));
  store_idx_row(sidx + p * kIdxSlots, p, idx);
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
  groups[i] = uint32_t(group_of(keys[i]));
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

__global__ void permute_keys_kernel(const int32_t* perm, int64_t n, const int64_t* keys, int64_t* skeys) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) skeys[p] = keys[perm[p]];
}

__global__ void max_group_kernel(const int32_t* off, int count, int* out) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < count) atomicMax(out, off[g + 1] - off[g]);
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

static int device_smem_optin() {
  static int bytes = 0;
  if (!bytes) {
    int dev = 0;
    PSR_CUDA(cudaGetDevice(&dev));
    PSR_CUDA(cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  }
  return bytes;
}

static int device_smem_per_sm() {
  static int bytes = 0;
  if (!bytes) {
    int dev = 0;
    PSR_CUDA(cudaGetDevice(&dev));
    PSR_CUDA(cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  }
  return bytes;
}

template <class V>
__global__ void gather_x_kernel(const int32_t* perm, int64_t n, const V* x, V* sx) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) sx[p] = x[perm[p]];
}

// The first nonzero error word of a launch into the stage's deferred word.
__global__ void merge_error_kernel(const int* launch_error, int* stage_error) {
  if (threadIdx.x == 0 && *launch_error) atomicCAS(stage_error, 0, *launch_error);
}

void throw_relax_error(int err) {
  if (err == 2) throw Error(4, "ordered relaxation: footprint exceeds its capacity");
  if (err == 3) throw Error(1, "ordered relaxation: an operator column is not its slot's neighbour");
  if (err == 4) throw Error(4, "ordered relaxation: a bulk copy or a phase did not complete");
  if (err) throw Error(4, "ordered relaxation: a dependency wait timed out");
}

// The cluster pipelines for one level, when they apply: every task's rows fit a region and
// its footprint, peer segments and exports fit shared memory, and `iters` clusters of
// kPipeCtas CTAs can be resident at once.  Returns false (nothing launched) otherwise.
// PSR_RELAX_KERNEL=strip keeps the dynamic scheduler; =pipeline asks for the pipelines even
// when a test override of the dynamic scheduler is set.
template <class T, class V, class I>
static bool relax_pipeline(const StripSchedule& S, const T* svals, const I* sidx, const V* sb, const int32_t* xstart,
                           V* xb0, V* xb1, int iters, cudaStream_t s, float* ms, V* hist, bool rev,
                           bool record_increment, RelaxDeferred* defer) {
  const char* mode = std::getenv("PSR_RELAX_KERNEL");
  const bool forced = mode && std::string(mode) == "pipeline";
  if (!forced) return false;  // opt-in: measured slower than the dynamic scheduler
  const int depth = S.depth, n = 1 << depth, strips = kPipeCtas;
  const int per16 = 16 / int(sizeof(V));
  if (int64_t(iters) * kPipeCtas > device_sms()) return false;
  const int ntasks = (n + 1) * strips;
  DBuf<int32_t> bounds(int64_t(n + 1) * (strips + 1), s);
  strip_bounds_kernel<<<blocks_for(int64_t(n + 1) * (strips + 1)), kThreads, 0, s>>>(xstart, n, strips, bounds.p);
  PSR_LAUNCH_CHECK();
  DBuf<int> caps(8, s);
  caps.zero();
  footprint_kernel<<<blocks_for(ntasks), kThreads, 0, s>>>(xstart, bounds.p, n, strips, per16, rev ? 1 : 0, caps.p);
  PSR_LAUNCH_CHECK();
  std::vector<int> fcap = read_vector(caps.p, 3, s);
  if (sizeof(I) == 2 && fcap[0] > 32767) return false;
  const int big = 1 << 30;
  DBuf<StripMeta> smeta(ntasks, s);
  auto mk = rev ? strip_meta_kernel<true> : strip_meta_kernel<false>;
  mk<<<blocks_for(ntasks, 128), 128, 0, s>>>(xstart, bounds.p, S.off.p, n, strips, per16, big, big, big,
                                             kSlotsR * int(sizeof(T)) + kIdxSlots * int(sizeof(I)), int(sizeof(V)),
                                             smeta.p);
  PSR_LAUNCH_CHECK();
  DBuf<PipeMeta> meta(ntasks, s);
  caps.zero();
  auto pk = rev ? pipe_meta_kernel<true> : pipe_meta_kernel<false>;
  pk<<<blocks_for(ntasks, 64), 64, 0, s>>>(smeta.p, xstart, bounds.p, S.off.p, n, per16, meta.p, caps.p);
  PSR_LAUNCH_CHECK();
  pipe_push_kernel<<<blocks_for(int64_t(n) * kPipeCtas, 64), 64, 0, s>>>(meta.p, n, caps.p);
  PSR_LAUNCH_CHECK();
  pipe_pushoff_kernel<<<blocks_for(ntasks, 64), 64, 0, s>>>(meta.p, ntasks);
  PSR_LAUNCH_CHECK();
  pipe_bspan_kernel<<<blocks_for(ntasks), kThreads, 0, s>>>(meta.p, ntasks, per16, caps.p);
  PSR_LAUNCH_CHECK();
  std::vector<int> c = read_vector(caps.p, 5, s);
  if (c[4]) return false;  // more peer segments than a task description holds
  PipeLevel P{};
  P.cap = std::max(c[0], 1);
  P.ecap = std::max(c[3], 1);
  auto al = [](int64_t b) { return (b + 127) & ~int64_t(127); };
  const int64_t budget = int64_t(device_smem_optin()) - 2048;  // static shared memory of the kernel
  {  // rows per region: all of them if they fit, else as many as fit beside the rest
    const int64_t fixed = 2 * al(int64_t(P.cap + 1) * int64_t(sizeof(V))) + 2 * al(int64_t(P.ecap) * int64_t(sizeof(V))) +
                          2 * al(int64_t(sizeof(PipeMeta))) + kPipeRegions * 3 * 128;
    const int64_t per_row = kSlotsR * int64_t(sizeof(T)) + kIdxSlots * int64_t(sizeof(I)) + int64_t(sizeof(V));
    const int64_t fit = (budget - fixed - kPipeRegions * 2 * per16 * int64_t(sizeof(V))) / (kPipeRegions * per_row);
    P.rcap = int(std::min<int64_t>(std::max(c[1], 1), fit));
    P.bcap = std::min(std::max(c[2], per16), (P.rcap + 2 * per16) / per16 * per16);
    // below a quarter of the median task's rows the pipelines would read most rows from global memory
    if (P.rcap < 64) return false;
  }
  int64_t off = 0;
  for (int f = 0; f < 2; ++f) {
    P.off_foot[f] = off;
    off += al(int64_t(P.cap + 1) * int64_t(sizeof(V)));
  }
  for (int r = 0; r < kPipeRegions; ++r) {
    P.off_vals[r] = off;
    off += al(int64_t(P.rcap) * kSlotsR * int64_t(sizeof(T)));
    P.off_idx[r] = off;
    off += al(int64_t(P.rcap) * kIdxSlots * int64_t(sizeof(I)));
    P.off_b[r] = off;
    off += al(int64_t(P.bcap) * int64_t(sizeof(V)));
  }
  for (int f = 0; f < 2; ++f) {
    P.off_exp[f] = off;
    off += al(int64_t(P.ecap) * int64_t(sizeof(V)));
  }
  for (int f = 0; f < 2; ++f) {
    P.off_meta[f] = off;
    off += al(int64_t(sizeof(PipeMeta)));
  }
  if (std::getenv("PSR_RELAX_DEBUG")) {
    std::vector<PipeMeta> hm = read_vector(meta.p, ntasks, s);
    std::vector<int> rows, fps;
    for (const PipeMeta& q : hm) {
      for (int cc = 0; cc < 4; ++cc) rows.push_back(q.m.p1[cc] - q.m.p0[cc]);
      fps.push_back(q.m.base[12]);
    }
    std::sort(rows.begin(), rows.end());
    std::sort(fps.begin(), fps.end());
    auto pct = [](const std::vector<int>& v, double f) { return v.empty() ? 0 : v[size_t(f * (v.size() - 1))]; };
    std::fprintf(stderr, "pipeline depth %d: cap %d rcap %d bcap %d ecap %d smem %lld budget %lld; rows/colour p50 %d "
                 "p90 %d p99 %d max %d; footprint p50 %d p90 %d p99 %d max %d\n", depth, P.cap, P.rcap, P.bcap, P.ecap,
                 (long long)off, (long long)budget, pct(rows, .5), pct(rows, .9), pct(rows, .99), pct(rows, 1.0),
                 pct(fps, .5), pct(fps, .9), pct(fps, .99), pct(fps, 1.0));
  }
  if (off > budget) return false;
  auto kernel = rev ? pipeline_gs_kernel<T, V, I, true> : pipeline_gs_kernel<T, V, I, false>;
  PSR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(off)));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kPipeCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(unsigned(iters * kPipeCtas));
  cfg.blockDim = dim3(kRelaxThreads);
  cfg.dynamicSmemBytes = size_t(off);
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (clusters < iters) return false;
  DBuf<int> ctrl(64, s);  // error word
  ctrl.zero();
  DBuf<int> done(int64_t(ntasks) * kFlagPad, s);
  done.zero();
  StripLevel& L = P.L;
  L.n = n;
  L.strips = strips;
  L.vals = svals;
  L.nidx = sidx;
  L.b = sb;
  L.xb0 = xb0;
  L.xb1 = xb1;
  L.done = done.p;
  L.error = ctrl.p;
  L.hist = hist;
  L.rows = S.rows;
  L.iters = iters;
  L.record_increment = record_increment ? 1 : 0;
  L.poll_log2 = 26;
  L.cap = P.cap;
  P.meta = meta.p;
  const char* trace_file = std::getenv("PSR_RELAX_TRACE_FILE");
  DBuf<long long> trace;
  const int64_t trace_count = int64_t(iters) * kPipeCtas * (n + 1) * 16;
  if (trace_file) {
    trace.alloc(trace_count, s);
    trace.zero();
    L.trace = trace.p;
  }
  const bool timed = ms || (defer && defer->events);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (timed) {
    PSR_CUDA(cudaEventCreate(&e0));
    PSR_CUDA(cudaEventCreate(&e1));
    PSR_CUDA(cudaEventRecord(e0, s));
  }
  PSR_CUDA(cudaLaunchKernelEx(&cfg, kernel, P));
  PSR_LAUNCH_CHECK();
  if (timed) PSR_CUDA(cudaEventRecord(e1, s));
  if (defer && defer->error && !trace_file) {
    merge_error_kernel<<<1, 32, 0, s>>>(L.error, defer->error);
    PSR_LAUNCH_CHECK();
    if (timed) defer->events->emplace_back(e0, e1);
    return true;
  }
  const int err = read_scalar(L.error, s);
  if (timed) {
    if (ms) PSR_CUDA(cudaEventElapsedTime(ms, e0, e1));
    if (defer && defer->events)
      defer->events->emplace_back(e0, e1);
    else {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
  }
  if (trace_file) {
    std::vector<long long> h = read_vector(trace.p, trace_count, s);
    if (FILE* f = std::fopen(trace_file, "ab")) {
      long long header[8] = {depth, n, kPipeCtas, iters, -1, trace_count, 0, 16};  // -1: pipeline trace
      std::fwrite(header, sizeof(header), 1, f);
      std::fwrite(h.data(), sizeof(long long), h.size(), f);
      std::fclose(f);
    }
  }
  throw_relax_error(err);
  return true;
}

template <class T, class V, class I>
void relax_strips_scheduled(const StripSchedule& S, const T* svals, const I* sidx, const V* sb, V* x, int iters,
                            cudaStream_t s, float* ms, V* hist, bool rev, bool record_increment, RelaxDeferred* defer) {
  const int64_t rows = S.rows;
  if (iters <= 0 || rows <= 0) return;
  const int depth = S.depth;
  const int n = 1 << depth;
  const int nx = n + 2;
  const int per16 = 16 / int(sizeof(V));
  const int32_t* perm = S.perm.p;
  const int32_t* off = S.off.p;
  DBuf<V> x0(rows + 16, s), x1(rows + 16, s);  // slack: 16-byte copies may read past the last row
  gather_x_kernel<V><<<blocks_for(rows), kThreads, 0, s>>>(perm, rows, x, x1.p);
  PSR_LAUNCH_CHECK();
  const int64_t* skeys_p = S.skeys.p;
  DBuf<int32_t> xstart(int64_t(n + 1) * 4 * nx, s);
  xstart_kernel<<<blocks_for(int64_t(n + 1) * 4 * nx), kThreads, 0, s>>>(skeys_p, off, n, xstart.p);
  PSR_LAUNCH_CHECK();
  if (relax_pipeline<T, V, I>(S, svals, sidx, sb, xstart.p, x0.p, x1.p, iters, s, ms, hist, rev, record_increment,
                              defer)) {
    scatter_back_kernel<V><<<blocks_for(rows), kThreads, 0, s>>>(perm, rows, ((iters - 1) & 1) ? x1.p : x0.p, x);
    PSR_LAUNCH_CHECK();
    return;
  }
  // Strips per slice: a wave (iters x strips tasks) fills about seven eighths of the persistent
  // grid, leaving CTAs that take the next wave's tasks early and prefetch their operator rows;
  // at least ~128 rows per strip.  More strips are taken (up to twice as many) while more than
  // 5% of the tasks would not fit their rows in shared memory.  Measured at depth 9, 8 sweeps,
  // 148 SMs (finest level, ms): mixed 12/14/16/18/20/24 strips 3.28/3.04/3.01/3.15/3.40/3.99;
  // float64 (wider rows) 12/16/20/24 strips 9.40/5.83/4.38/4.48.
  const int sms = device_sms();
  const int ctas = kRelaxCtasPerSm * sms;
  int strips = int(std::max<int64_t>(
      1, std::min<int64_t>(std::max(1, (7 * ctas) / (8 * iters)), rows / (int64_t(n + 1) * 128))));
  // Tuning override of the strips per slice (sweeps; the default above is the measured choice).
  bool forced_strips = false;
  if (const char* env = std::getenv("PSR_RELAX_STRIPS")) {
    const int forced = std::atoi(env);
    if (forced >= 1 && forced <= 256) {
      strips = forced;
      forced_strips = true;
    }
  }
  const int base_strips = strips;
  DBuf<int> ctrl(3 * 32, s);  // task counter, error word, capacities: one 128-byte line each
  int* counter = ctrl.p;
  int* error = ctrl.p + 32;
  int* caps_dev = ctrl.p + 64;
  DBuf<int32_t> bounds;
  std::vector<int> caps;
  // 16-bit index rows reach the footprint through offsets below 2^15 (idx_absent).
  // PSR_RELAX_FOOTPRINT_LIMIT lowers that bound (test override: the strip narrowing below,
  // which only very large levels need, on small levels).
  int fp_limit = 32767;
  if (const char* env = std::getenv("PSR_RELAX_FOOTPRINT_LIMIT")) {
    const int forced = std::atoi(env);
    if (forced >= 1 && forced < fp_limit) fp_limit = forced;
  }
  // Shared memory of one CTA: the footprint (and its +0 entry), the staged rows and their
  // right-hand sides.
  const int64_t budget = std::min<int64_t>(device_smem_optin(), device_smem_per_sm() / kRelaxCtasPerSm) - 4096;
  const int64_t row_bytes = kSlotsR * int64_t(sizeof(T)) + kIdxSlots * int64_t(sizeof(I));
  auto fp_bytes_of = [&](int fp) { return (int64_t(std::max(fp, 1) + 1) * int64_t(sizeof(V)) + 15) & ~int64_t(15); };
  // staged rows and right-hand-side elements that fit beside a footprint of fp elements
  auto row_capacity = [&](int fp, int maxrows, int maxb) {
    int64_t rc = std::max<int64_t>(0, std::min<int64_t>(maxrows, (budget - fp_bytes_of(fp) - 4 * 16) /
                                                                       (row_bytes + int64_t(sizeof(V)))));
    return std::make_pair(rc, std::min<int64_t>(maxb, rc + 4 * per16) / per16 * per16);
  };
  while (true) {
    bounds.alloc(int64_t(n + 1) * (strips + 1), s);
    strip_bounds_kernel<<<blocks_for(int64_t(n + 1) * (strips + 1)), kThreads, 0, s>>>(xstart.p, n, strips,
                                                                                        bounds.p);
    PSR_LAUNCH_CHECK();
    ctrl.zero();
    footprint_kernel<<<blocks_for((n + 1) * strips), kThreads, 0, s>>>(xstart.p, bounds.p, n, strips, per16,
                                                                        rev ? 1 : 0, caps_dev);
    PSR_LAUNCH_CHECK();
    unstaged_kernel<<<blocks_for((n + 1) * strips), kThreads, 0, s>>>(xstart.p, bounds.p, n, strips, per16,
                                                                       rev ? 1 : 0, budget, int(row_bytes),
                                                                       int(sizeof(V)), caps_dev);
    PSR_LAUNCH_CHECK();
    caps = read_vector(caps_dev, 4, s);  // footprint, rows, right-hand side, unstaged tasks
    // narrow the strips until the largest footprint fits the 16-bit offsets
    if (!(sizeof(I) == 4 || caps[0] <= fp_limit) && strips < 256) {
      strips = std::min(256, 2 * strips);
      continue;
    }
    // then while more than 5% of the tasks would run unstaged (wide rows: float64 values)
    if (!forced_strips && int64_t(caps[3]) * 20 > int64_t(n + 1) * strips && strips < std::min(256, 2 * base_strips)) {
      strips = std::min({256, 2 * base_strips, strips + std::max(1, strips / 4)});
      continue;
    }
    break;
  }
  if (sizeof(I) == 2 && caps[0] > fp_limit)
    throw Error(4, "ordered relaxation: a strip footprint exceeds the 16-bit index range");
  const int maxfp = caps[0], maxrows = caps[1], maxb = caps[2];
  // Slice-visits in wave order (relaxation.py:128-143): wave q = 2t + n - z holds slices two
  // apart; every dependency of a wave-q task lies in wave q-1 or q-2, so dequeuing by wave is
  // deadlock-free and keeps whole waves in flight.
  std::vector<int2> visits;
  for (int q = 0; q <= n + 2 * (iters - 1); ++q) {
    int first = std::max(0, (q - n + 1) / 2), last = std::min(iters - 1, q / 2);
    for (int t = first; t <= last; ++t) visits.push_back(make_int2(n - q + 2 * t, t));
  }
  DBuf<int2> dvisits(int64_t(visits.size()), s);
  PSR_CUDA(cudaMemcpyAsync(dvisits.p, visits.data(), visits.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
  StripLevel L{};
  L.n = n;
  L.strips = strips;
  L.nvisits = int(visits.size());
  L.vals = svals;
  L.nidx = sidx;
  L.b = sb;
  L.xb0 = x0.p;
  L.xb1 = x1.p;
  L.visits = dvisits.p;
  DBuf<int> done(int64_t(n + 1) * strips * kFlagPad, s);
  done.zero();
  L.done = done.p;
  L.counter = counter;
  L.error = error;
  L.hist = hist;
  L.rows = rows;
  L.iters = iters;
  L.record_increment = record_increment ? 1 : 0;
  L.poll_log2 = 26;
  // PSR_RELAX_STALL_TEST=1 (tests of the timeout path): every wait on the newest slice waits
  // for a count that no task publishes and gives up after 4096 polls, so the launch ends with
  // PSR_ETIMEOUT without a fault and the context stays usable.
  if (const char* env = std::getenv("PSR_RELAX_STALL_TEST"))
    if (std::atoi(env) == 1) {
      L.stall = 1;
      L.poll_log2 = 12;
    }
  // Shared memory: the footprint, plus the staged rows of tasks that fit.
  const int64_t fp_bytes = fp_bytes_of(maxfp);
  if (fp_bytes > budget) throw Error(4, "ordered relaxation: a strip footprint exceeds shared memory");
  L.cap = std::max(maxfp, 1);
  int64_t rc = row_capacity(maxfp, maxrows, maxb).first;
  // PSR_RELAX_ROW_CAP caps the staged rows per task (test override: 0 sends every task down
  // the global-memory row path that only tasks too large for shared memory take).
  if (const char* env = std::getenv("PSR_RELAX_ROW_CAP")) {
    const int forced = std::atoi(env);
    if (forced >= 0) rc = std::min<int64_t>(rc, forced);
  }
  L.row_cap = int(rc);
  L.b_cap = int(std::min<int64_t>(maxb, rc + 4 * per16) / per16 * per16);
  int64_t smem = fp_bytes + rc * (kSlotsR * int64_t(sizeof(T)) + kIdxSlots * int64_t(sizeof(I))) +
                 ((int64_t(L.b_cap) * int64_t(sizeof(V)) + 15) & ~int64_t(15));
  smem = std::max<int64_t>(smem, 16);
  DBuf<StripMeta> meta(int64_t(n + 1) * strips, s);
  {
    auto mk = rev ? strip_meta_kernel<true> : strip_meta_kernel<false>;
    mk<<<blocks_for(int64_t(n + 1) * strips, 128), 128, 0, s>>>(xstart.p, bounds.p, off, n, strips, per16, L.cap,
                                                                 L.row_cap, L.b_cap, int(row_bytes), int(sizeof(V)),
                                                                 meta.p);
    PSR_LAUNCH_CHECK();
  }
  L.meta = meta.p;
  auto kernel = rev ? strip_gs_kernel<T, V, I, true> : strip_gs_kernel<T, V, I, false>;
  PSR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const int64_t total_tasks = int64_t(visits.size()) * strips;
  const int grid = int(std::min<int64_t>(total_tasks, ctas));
  const char* trace_file = std::getenv("PSR_RELAX_TRACE_FILE");
  DBuf<long long> trace;
  if (trace_file) {
    trace.alloc(total_tasks * kTraceSlots, s);
    trace.zero();
    L.trace = trace.p;
  }
  const bool timed = ms || (defer && defer->events);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (timed) {
    PSR_CUDA(cudaEventCreate(&e0));
    PSR_CUDA(cudaEventCreate(&e1));
    PSR_CUDA(cudaEventRecord(e0, s));
  }
  {
    // per row visit: 27 operator values (S), b, x read and written (V), row id, visit record
    const double visits = double(rows) * iters;
    KernelClock clock(rev ? kClkStripReverse : kClkStripForward,
                      visits * (27.0 * sizeof(T) + 3 * sizeof(V) + 4 + (hist ? sizeof(V) : 0)), visits, s);
    kernel<<<grid, kRelaxThreads, size_t(smem), s>>>(L);
    PSR_LAUNCH_CHECK();
  }
  if (timed) PSR_CUDA(cudaEventRecord(e1, s));
  scatter_back_kernel<V><<<blocks_for(rows), kThreads, 0, s>>>(perm, rows, ((iters - 1) & 1) ? x1.p : x0.p, x);
  PSR_LAUNCH_CHECK();
  if (defer && defer->error && !trace_file) {
    merge_error_kernel<<<1, 32, 0, s>>>(L.error, defer->error);
    PSR_LAUNCH_CHECK();
    if (timed) defer->events->emplace_back(e0, e1);
    return;
  }
  int err = read_scalar(L.error, s);
  if (timed) {
    if (ms) PSR_CUDA(cudaEventElapsedTime(ms, e0, e1));
    if (defer && defer->events)
      defer->events->emplace_back(e0, e1);
    else {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
  }
  if (trace_file) {
    std::vector<long long> h = read_vector(trace.p, total_tasks * kTraceSlots, s);
    if (FILE* f = std::fopen(trace_file, "ab")) {
      long long header[8] = {depth, n, strips, L.row_cap, grid, total_tasks, caps[3], kTraceSlots};
      std::fwrite(header, sizeof(header), 1, f);
      std::fwrite(visits.data(), sizeof(int2), visits.size(), f);
      std::fwrite(h.data(), sizeof(long long), h.size(), f);
      std::fclose(f);
    }
  }
  throw_relax_error(err);
}

void build_strip_schedule(const int64_t* keys, int64_t rows, int depth, StripSchedule& S, cudaStream_t s) {
  const int n = 1 << depth;
  const int groups = 4 * (n + 1);
  S.rows = rows;
  S.depth = depth;
  // Schedule order: stable sort by group (slice, colour); rows of a group stay in key order.
  DBuf<uint32_t> g(rows, s), sg(rows, s);
  DBuf<int32_t> ids(rows, s);
  S.perm.alloc(rows, s);
  S.inv.alloc(rows, s);
  S.off.alloc(groups + 1, s);
  S.skeys.alloc(rows, s);
  slice_groups_kernel<<<blocks_for(rows), kThreads, 0, s>>>(keys, rows, g.p, ids.p);
  PSR_LAUNCH_CHECK();
  sort_pairs(g.p, sg.p, ids.p, S.perm.p, rows, bits_for(uint64_t(groups)), s);
  group_bounds_kernel<<<blocks_for(groups + 1), kThreads, 0, s>>>(sg.p, rows, groups, S.off.p);
  PSR_LAUNCH_CHECK();
  inverse_kernel<<<blocks_for(rows), kThreads, 0, s>>>(S.perm.p, rows, S.inv.p);
  PSR_LAUNCH_CHECK();
  permute_keys_kernel<<<blocks_for(rows), kThreads, 0, s>>>(S.perm.p, rows, keys, S.skeys.p);
  PSR_LAUNCH_CHECK();
  // Group-relative neighbour indices fit 16 bits unless a (slice, colour) group is huge.  A
  // group holds one x and one y parity of a slice, at most (2^(d-1) + 1)^2 rows (and never
  // more than the level), so below depth 9 the bound settles it without reading the largest
  // group back (a host synchronisation).  PSR_INDEX_WIDTH=32 takes the 32-bit rows regardless
  // (test override: the huge-group path on small levels).
  const int64_t side = (int64_t(1) << std::max(depth - 1, 0)) + 1;
  if (std::min<int64_t>(rows, side * side) < 32767) {
    S.wide = false;
  } else {
    DBuf<int> gmax(1, s);
    gmax.zero();
    max_group_kernel<<<blocks_for(groups), kThreads, 0, s>>>(S.off.p, groups, gmax.p);
    PSR_LAUNCH_CHECK();
    S.wide = read_scalar(gmax.p, s) >= 32767;
  }
  if (const char* env = std::getenv("PSR_INDEX_WIDTH"))
    if (std::atoi(env) == 32) S.wide = true;
}

template <class T, class V, class I>
static void reorder_and_relax(const StripSchedule& S, const int64_t* keys, const int32_t* cols, const T* vals,
                              const V* b, V* x, int iters, cudaStream_t s, float* ms) {
  const int64_t rows = S.rows;
  const int per16 = 16 / int(sizeof(V));
  DBuf<I> sidx(kIdxSlots * rows, s);
  DBuf<T> svals(kSlotsR * rows, s);
  DBuf<V> sb(rows + 2 * per16, s), sx(rows, s);
  DBuf<int64_t> skeys(rows, s);
  sb.zero();
  reorder_kernel<T, V, I><<<blocks_for(rows), kThreads, 0, s>>>(S.perm.p, S.inv.p, S.off.p, rows, cols, vals, b, x,
                                                               keys, sidx.p, svals.p, sb.p, sx.p, skeys.p);
  PSR_LAUNCH_CHECK();
  relax_strips_scheduled<T, V, I>(S, svals.p, sidx.p, sb.p, x, iters, s, ms);
}

// Ordered sliced relaxation of one level given as slot-ELL rows in key order.  x (key
// order) holds the initial guess and receives the result.
template <class T, class V>
void relax_sliced_strips(const int64_t* keys, int64_t rows, int depth, const int32_t* cols, const T* vals,
                         const V* b, V* x, int iters, cudaStream_t s, float* ms) {
  if (iters <= 0 || rows <= 0) return;
  StripSchedule S;
  build_strip_schedule(keys, rows, depth, S, s);
  if (!S.wide)
    reorder_and_relax<T, V, int16_t>(S, keys, cols, vals, b, x, iters, s, ms);
  else
    reorder_and_relax<T, V, int32_t>(S, keys, cols, vals, b, x, iters, s, ms);
}

template void relax_sliced_strips<float, float>(const int64_t*, int64_t, int, const int32_t*, const float*,
                                                const float*, float*, int, cudaStream_t, float*);
template void relax_sliced_strips<double, double>(const int64_t*, int64_t, int, const int32_t*, const double*,
                                                  const double*, double*, int, cudaStream_t, float*);
template void relax_sliced_strips<float, double>(const int64_t*, int64_t, int, const int32_t*, const float*,
                                                 const double*, double*, int, cudaStream_t, float*);

}  // namespace psr

namespace psr {
#define PSR_SCHED(T, V, I)                                                                                       \
  template void relax_strips_scheduled<T, V, I>(const StripSchedule&, const T*, const I*, const V*, V*, int,  \
                                                cudaStream_t, float*, V*, bool, bool, RelaxDeferred*);
PSR_SCHED(float, float, int16_t)
PSR_SCHED(float, float, int32_t)
PSR_SCHED(double, double, int16_t)
PSR_SCHED(double, double, int32_t)
PSR_SCHED(float, double, int16_t)
PSR_SCHED(float, double, int32_t)
}  // namespace psr
