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
constexpr int kPad = 32;       // one 128-byte line per slice counter
constexpr int kRelaxThreads = 512;

struct StripLevel {
  int n;                 // 2^depth (slices 0..n)
  int strips;            // strips per slice
  int nvisits;
  int cap;               // footprint capacity (elements) per CTA
  int row_cap;           // staged update rows per task
  int b_cap;             // staged right-hand-side elements per task
  const int32_t* bounds;     // [(n+1)*(strips+1)] x boundaries of the strips of each slice
  const int32_t* group_off;  // [4(n+1)+1] schedule position of each (slice, colour) group
  const void* vals;          // T[rows*28]   schedule order
  const void* nidx;          // I[rows*32]   neighbour index within its group, -1 absent; [27] = own
  const void* b;             // V[rows + slack]
  void* xb0;                 // V[rows]  even visits
  void* xb1;                 // V[rows]  odd visits (holds the initial x)
  const int32_t* xstart;     // [(n+1)*4][n+2]: first position of group (z,c) with x >= X
  const int2* visits;        // slice-visits (z, t) in wave order
  int* done;                 // completed strip tasks of slice z at done[z * kPad]
  int* counter;
  int* error;
  long long* trace;          // optional: 8 timestamps per task
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
template <class I>
__device__ __forceinline__ void load_idx(const I* src, I out[kIdxSlots]) {
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(out);
#pragma unroll
  for (int q = 0; q < kIdxSlots * int(sizeof(I)) / 16; ++q) d[q] = s[q];
}

// One row of colour C: r = b - sum_k x_k A_k in slot order; x_self += r / A_self.
// Every slot takes part in the sum: an absent slot (value +0, index idx_absent) reads the +0
// entry kept at foot[total], and r - (+0 * +0) = r exactly, so the result is bitwise that of
// skipping it.  A present slot holds its k-th neighbour (checked where the rows are built),
// which lies in the footprint by construction; the unsigned clamp keeps every read inside
// the footprint whatever the rows hold.  Measured ~2x fewer instructions per slot than
// testing each slot's presence and range.
template <int C, bool M, class T, class V, class I>
__device__ __forceinline__ void update_row(const I* nrow, const T* arow, V bv, V* foot, const int* delta,
                                           unsigned total, int* error, V* rec, bool record_increment) {
  __align__(16) I n[kIdxSlots];  // filled with 16-byte vector loads
  load_idx(nrow, n);
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
  V inc = V(0);
  if (n[13] >= 0 && a[13] != T(0)) {
    inc = r * get_inv_diag<V>(n);
    foot[self] = xs[13] + inc;
  }
  if (rec) *rec = record_increment ? inc : foot[self];
}

// `hist` (optional) points at this visit's record column (row p records at hist[p * iters]);
// only the strip's own rows [o0, o1) write it (halo rows are recomputed by the neighbouring
// strip, which owns them).
template <int C, bool M, class T, class V, class I>
__device__ __forceinline__ void phase(const StripLevel& L, bool staged, int p0, int p1, int rbase, int bshift,
                                      const I* s_idx, const T* s_vals, const V* s_b, V* foot, const int* delta,
                                      unsigned total, V* hist, int o0, int o1) {
  const I* gidx = reinterpret_cast<const I*>(L.nidx);
  const T* gvals = reinterpret_cast<const T*>(L.vals);
  const V* gb = reinterpret_cast<const V*>(L.b);
  const bool inc = L.record_increment != 0;
  int dreg[12];  // footprint offsets in registers (measured ~1% faster than shared-memory reads)
#pragma unroll
  for (int r = 0; r < 12; ++r) dreg[r] = delta[r];
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    V* rec = (hist && p >= o0 && p < o1) ? hist + int64_t(p) * L.iters : nullptr;
    if (staged) {
      int i = rbase + (p - p0);
      update_row<C, M>(s_idx + int64_t(i) * kIdxSlots, s_vals + int64_t(i) * kSlotsR, s_b[bshift + (p - p0)], foot,
                       dreg, total, L.error, rec, inc);
    } else {
      update_row<C, M>(gidx + int64_t(p) * kIdxSlots, gvals + int64_t(p) * kSlotsR, gb[p], foot, dreg, total,
                       L.error, rec, inc);
    }
  }
}

// REV false: colours 0..3 in the stored slice order (the forward sweep).  REV true: the exact
// reverse of that sweep on the same layout -- logical slice z is stored slice n - z (so slot
// k's neighbour lies in logical slice z + 1 - k % 3) and the colours run 3..0.  One
// instantiation per order keeps each kernel's body to its own four phases.
template <class T, class V, class I, bool REV>
__global__ void __launch_bounds__(kRelaxThreads, 1) strip_gs_kernel(StripLevel L) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_bar;
  __shared__ int s_task, s_fail, s_total, s_rows, s_staged;
  __shared__ int s_lo[12], s_hi[12], s_base[13], s_delta[12];
  __shared__ int s_p0[4], s_p1[4], s_rbase[5], s_bshift[4], s_o0[4], s_o1[4];
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
  const int nx = L.n + 2;
  const int total_tasks = L.nvisits * L.strips;
  constexpr int per16 = 16 / int(sizeof(V));  // right-hand-side elements per 16 bytes
  uint32_t parity = 0;
  if (threadIdx.x == 0) mbar_init(&s_bar);
  __syncthreads();
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
    // stored slice of a logical slice (the mirrored sweep reads the forward layout)
    auto phys = [&](int zz) { return REV ? L.n - zz : zz; };
    const int x0 = L.bounds[phys(z) * (L.strips + 1) + s], x1 = L.bounds[phys(z) * (L.strips + 1) + s + 1];
    // All range lookups in one round: 24 footprint bounds, 8 update bounds, 8 own bounds.
    if (threadIdx.x < 40) {
      int i = threadIdx.x;
      if (i < 24) {
        int r = i >> 1, j = r >> 2, c = r & 3, zz = z + j - 1;
        int v = 0;
        if (zz >= 0 && zz <= L.n) {
          int X = (i & 1) ? min(x1 + 4, L.n + 1) : max(x0 - 4, 0);
          v = L.xstart[int64_t(phys(zz) * 4 + c) * nx + X];
        }
        if (i & 1)
          s_hi[r] = v;
        else
          s_lo[r] = v;
      } else {
        int k = i - 24, c = (k >> 1) & 3, own = k >= 8, h = own ? 0 : (REV ? c : 3 - c);
        int X = (k & 1) ? min(x1 + h, L.n + 1) : max(min(x0 - h, L.n + 1), 0);
        int v = L.xstart[int64_t(phys(z) * 4 + c) * nx + X];
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
        int j = r >> 2, c = r & 3, zz = z + j - 1;
        int gstart = (zz >= 0 && zz <= L.n) ? L.group_off[phys(zz) * 4 + c] : 0;
        s_delta[r] = s_base[r] + gstart - s_lo[r];
      }
      s_base[12] = total;
      s_total = total;
      int rows = 0, bsum = 0;
      for (int c = 0; c < 4; ++c) {
        s_rbase[c] = rows;
        rows += s_p1[c] - s_p0[c];
        int a0 = s_p0[c] - s_p0[c] % per16, a1 = (s_p1[c] + per16 - 1) / per16 * per16;
        s_bshift[c] = bsum + (s_p0[c] - a0);
        bsum += s_p1[c] > s_p0[c] ? a1 - a0 : 0;
      }
      s_rbase[4] = rows;
      s_rows = rows;
      if (total > L.cap) {
        atomicExch(L.error, 2);
        s_fail = 1;
      }
      s_staged = !s_fail && rows <= L.row_cap && bsum <= L.b_cap;
      if (s_staged) {
        // Operator rows do not depend on x: copy them while the dependencies are pending.
        fence_proxy_async();
        uint32_t bytes = 0;
        for (int c = 0; c < 4; ++c) {
          int cnt = s_p1[c] - s_p0[c];
          if (cnt <= 0) continue;
          bytes += uint32_t(cnt) * (kSlotsR * sizeof(T) + kIdxSlots * sizeof(I));
          int a0 = s_p0[c] - s_p0[c] % per16, a1 = (s_p1[c] + per16 - 1) / per16 * per16;
          bytes += uint32_t(a1 - a0) * sizeof(V);
        }
        mbar_expect_tx(&s_bar, bytes);
        int bpos = 0;
        for (int c = 0; c < 4; ++c) {
          int cnt = s_p1[c] - s_p0[c];
          if (cnt <= 0) continue;
          int p0 = s_p0[c];
          bulk_copy(s_vals + int64_t(s_rbase[c]) * kSlotsR, gvals + int64_t(p0) * kSlotsR,
                    uint32_t(cnt) * kSlotsR * sizeof(T), &s_bar);
          bulk_copy(s_idx + int64_t(s_rbase[c]) * kIdxSlots, gidx + int64_t(p0) * kIdxSlots,
                    uint32_t(cnt) * kIdxSlots * sizeof(I), &s_bar);
          int a0 = p0 - p0 % per16, a1 = (s_p1[c] + per16 - 1) / per16 * per16;
          bulk_copy(s_b + bpos, gb + a0, uint32_t(a1 - a0) * sizeof(V), &s_bar);
          bpos += a1 - a0;
        }
      }
      if (tr) tr[1] = globaltimer();
      // slice z after visit t-1 (two waves back); the newer dependencies are awaited below
      // while this slice is staged
      bool ok = !s_fail;
      if (ok) ok = wait_at_least(L.done + z * kPad, t * L.strips, L.error, L.poll_log2);
      if (!ok) {
        atomicCAS(L.error, 0, 1);
        s_fail = 1;
      }
      if (tr) tr[2] = globaltimer();
    }
    __syncthreads();
    const bool staged = s_staged;
    if (s_fail) {
      if (staged) mbar_wait(&s_bar, parity);  // never leave with copies in flight
      return;
    }
    if (tr) tr[3] = globaltimer();
    // Stage the footprint: slice z+1 after visit t, slices z and z-1 after visit t-1.  Warp 0
    // waits for slices z+1 and z-1 while the other warps stage slice z, then all stage the rest.
    {
      const V* cur = (t & 1) ? xb1 : xb0;
      const V* prev = (t & 1) ? xb0 : xb1;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
      // range r staged by `parts` warps, part `part` of them (4 loads in flight per lane)
      auto stage_range = [&](int r, int part, int parts) {
        const V* src = ((r >> 2) == 2 ? cur : prev) + s_lo[r];
        V* dst = foot + s_base[r];
        const int cnt = s_hi[r] - s_lo[r];
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
        if (lane == 0) {
          bool ok = true;
          if (z + 1 <= L.n)
            ok = wait_at_least(L.done + (z + 1) * kPad, (t + 1) * L.strips + (L.stall ? (1 << 30) : 0), L.error,
                               L.poll_log2);
          if (ok && z > 0) ok = wait_at_least(L.done + (z - 1) * kPad, t * L.strips, L.error, L.poll_log2);
          if (!ok) {
            atomicCAS(L.error, 0, 1);
            s_fail = 1;
          }
        }
        __syncwarp();
      } else {
        // slice z: 4 ranges over the other warps
        const int parts = max(1, (nwarps - 1) / 4);
        for (int q = warp - 1; q < 4 * parts; q += nwarps - 1) stage_range(4 + q / parts, q % parts, parts);
      }
      __syncthreads();
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
    if (threadIdx.x == 0) foot[s_total] = V(0);  // the entry absent slots read
    if (staged && !mbar_wait(&s_bar, parity)) {
      if (threadIdx.x == 0) atomicExch(L.error, 4);
      return;
    }
    if (staged) parity ^= 1;
    __syncthreads();
    if (tr) tr[4] = globaltimer();
    {
      V* hv = L.hist ? reinterpret_cast<V*>(L.hist) + t : nullptr;
#define PSR_PHASE(C, M)                                                                                          \
  phase<C, M, T, V, I>(L, staged, s_p0[C], s_p1[C], s_rbase[C], s_bshift[C], s_idx, s_vals, s_b, foot, s_delta, \
                       unsigned(s_total), hv, s_o0[C], s_o1[C]);                                               \
  __syncthreads();
      if (!REV) {
        PSR_PHASE(0, false) PSR_PHASE(1, false) PSR_PHASE(2, false) PSR_PHASE(3, false)
      } else {
        PSR_PHASE(3, true) PSR_PHASE(2, true) PSR_PHASE(1, true) PSR_PHASE(0, true)
      }
#undef PSR_PHASE
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
  for (int k = 0; k < kSlotsR; ++k) {
    int32_t c = k < 27 ? cols[row * kSlotsR + k] : -1;
    I idx = idx_absent<I>();
    if (c >= 0) idx = I(inv[c] - group_off[group_of(keys[c])]);
    svals[p * kSlotsR + k] = k < 27 ? vals[row * kSlotsR + k] : T(0);
    sidx[p * kIdxSlots + k] = idx;
  }
  sidx[p * kIdxSlots + 27] = I(p - group_off[group_of(keys[row])]);
  for (int k = 28; k < kIdxSlots; ++k) sidx[p * kIdxSlots + k] = I(-1);
  const T diag = vals[row * kSlotsR + 13];
  put_inv_diag<V>(sidx + p * kIdxSlots, diag != T(0) ? V(1.0) / V(diag) : V(0));
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

template <class V>
__global__ void gather_x_kernel(const int32_t* perm, int64_t n, const V* x, V* sx) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) sx[p] = x[perm[p]];
}

template <class T, class V, class I>
void relax_strips_scheduled(const StripSchedule& S, const T* svals, const I* sidx, const V* sb, V* x, int iters,
                            cudaStream_t s, float* ms, V* hist, bool rev, bool record_increment) {
  const int64_t rows = S.rows;
  if (iters <= 0 || rows <= 0) return;
  const int depth = S.depth;
  const int n = 1 << depth;
  const int nx = n + 2;
  const int per16 = 16 / int(sizeof(V));
  const int32_t* perm = S.perm.p;
  const int32_t* off = S.off.p;
  DBuf<V> x0(rows, s), x1(rows, s);
  gather_x_kernel<V><<<blocks_for(rows), kThreads, 0, s>>>(perm, rows, x, x1.p);
  PSR_LAUNCH_CHECK();
  const int64_t* skeys_p = S.skeys.p;
  DBuf<int32_t> xstart(int64_t(n + 1) * 4 * nx, s);
  xstart_kernel<<<blocks_for(int64_t(n + 1) * 4 * nx), kThreads, 0, s>>>(skeys_p, off, n, xstart.p);
  PSR_LAUNCH_CHECK();
  // Strips per slice: a wave (iters x strips tasks) fills about two thirds of the persistent
  // grid, leaving CTAs that take the next wave's tasks early and prefetch their operator rows;
  // at least ~128 rows per strip.  (Measured at depth 9, 8 sweeps, 148 SMs: 12 strips 4.4 ms,
  // 9 strips 7.0 ms, 18 strips 4.6 ms, 24 strips 5.9 ms.)
  const int sms = device_sms();
  int strips = int(std::max<int64_t>(
      1, std::min<int64_t>(std::max(1, (2 * sms) / (3 * iters)), rows / (int64_t(n + 1) * 128))));
  // Tuning override of the strips per slice (sweeps; the default above is the measured choice).
  if (const char* env = std::getenv("PSR_RELAX_STRIPS")) {
    const int forced = std::atoi(env);
    if (forced >= 1 && forced <= 256) strips = forced;
  }
  const int64_t pad_end = int64_t(n + 1) * kPad;
  DBuf<int> flags(pad_end + 4 * kPad, s);
  int* counter = flags.p + pad_end;
  int* error = flags.p + pad_end + kPad;
  int* caps_dev = flags.p + pad_end + 2 * kPad;
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
  while (true) {
    bounds.alloc(int64_t(n + 1) * (strips + 1), s);
    strip_bounds_kernel<<<blocks_for(int64_t(n + 1) * (strips + 1)), kThreads, 0, s>>>(xstart.p, n, strips,
                                                                                        bounds.p);
    PSR_LAUNCH_CHECK();
    flags.zero();
    footprint_kernel<<<blocks_for((n + 1) * strips), kThreads, 0, s>>>(xstart.p, bounds.p, n, strips, per16,
                                                                        rev ? 1 : 0, caps_dev);
    PSR_LAUNCH_CHECK();
    caps = read_vector(caps_dev, 3, s);
    // narrow the strips until the largest footprint fits the 16-bit offsets
    if (sizeof(I) == 4 || caps[0] <= fp_limit || strips >= 256) break;
    strips = std::min(256, 2 * strips);
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
  L.bounds = bounds.p;
  L.group_off = off;
  L.vals = svals;
  L.nidx = sidx;
  L.b = sb;
  L.xb0 = x0.p;
  L.xb1 = x1.p;
  L.xstart = xstart.p;
  L.visits = dvisits.p;
  L.done = flags.p;
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
  const int64_t budget = std::min<int64_t>(device_smem_optin() - 4096, 220 * 1024);
  // the footprint plus its +0 entry at index `total`
  const int64_t fp_bytes = (int64_t(std::max(maxfp, 1) + 1) * int64_t(sizeof(V)) + 15) & ~int64_t(15);
  if (fp_bytes > budget) throw Error(4, "ordered relaxation: a strip footprint exceeds shared memory");
  const int64_t per_row = kSlotsR * int64_t(sizeof(T)) + kIdxSlots * int64_t(sizeof(I)) + int64_t(sizeof(V));
  L.cap = std::max(maxfp, 1);
  int64_t rc = std::min<int64_t>(maxrows, (budget - fp_bytes - 4 * 16) / per_row);
  rc = std::max<int64_t>(rc, 0);
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
  auto kernel = rev ? strip_gs_kernel<T, V, I, true> : strip_gs_kernel<T, V, I, false>;
  PSR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const int64_t total_tasks = int64_t(visits.size()) * strips;
  const int grid = int(std::min<int64_t>(total_tasks, sms));
  const char* trace_file = std::getenv("PSR_RELAX_TRACE_FILE");
  DBuf<long long> trace;
  if (trace_file) {
    trace.alloc(total_tasks * 8, s);
    trace.zero();
    L.trace = trace.p;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms) {
    PSR_CUDA(cudaEventCreate(&e0));
    PSR_CUDA(cudaEventCreate(&e1));
    PSR_CUDA(cudaEventRecord(e0, s));
  }
  kernel<<<grid, kRelaxThreads, size_t(smem), s>>>(L);
  PSR_LAUNCH_CHECK();
  if (ms) PSR_CUDA(cudaEventRecord(e1, s));
  scatter_back_kernel<V><<<blocks_for(rows), kThreads, 0, s>>>(perm, rows, ((iters - 1) & 1) ? x1.p : x0.p, x);
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
  if (err == 4) throw Error(4, "ordered relaxation: a bulk copy did not complete");
  if (err) throw Error(4, "ordered relaxation: a dependency wait timed out");
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
  DBuf<int> gmax(1, s);
  gmax.zero();
  max_group_kernel<<<blocks_for(groups), kThreads, 0, s>>>(S.off.p, groups, gmax.p);
  PSR_LAUNCH_CHECK();
  // Group-relative neighbour indices fit 16 bits unless a (slice, colour) group is huge.
  // PSR_INDEX_WIDTH=32 takes the 32-bit rows regardless (test override: the huge-group path
  // on small levels).
  S.wide = read_scalar(gmax.p, s) >= 32767;
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
                                                cudaStream_t, float*, V*, bool, bool);
PSR_SCHED(float, float, int16_t)
PSR_SCHED(float, float, int32_t)
PSR_SCHED(double, double, int16_t)
PSR_SCHED(double, double, int32_t)
PSR_SCHED(float, double, int16_t)
PSR_SCHED(float, double, int32_t)
}  // namespace psr
