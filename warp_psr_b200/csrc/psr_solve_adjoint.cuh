// A13: reverse pass of the solve (warp-psr cascadic_adjoint.py:76-104, relaxation_adjoint.py:159-264,
// assembly_adjoint.py:69-116, solver_adjoint.py:106-196, multigrid_adjoint.py:118-174,
// normal_load_adjoint.py:123-161).  Included at the end of psr_solve.cu (same translation unit:
// it reuses the forward's device helpers and the SolveTape layout).
//
// The derivative is that of the finite algorithm the forward ran, with its discrete choices
// (tree, bins, schedules, CG stopping points) held fixed.
//
// Ordered relaxation.  Forward, row i's visit t is x_i += (b_i - sum_k A_ik x_k) / A_ii.  With
// lambda the adjoint of x, reversing the visits in the exact reverse order gives
//   mu = lambda_i / A_ii,  b-adjoint += mu,  lambda_k -= mu A_ik (k = i included),
//   A-adjoint_ik -= mu x_k(at that visit),   A-adjoint_ii -= mu x_i(after the visit).
// Writing M_k for the sum of the mu of row k so far, lambda_i = seed_i - sum_k A_ki M_k, so the
// reverse sweep is itself a Gauss-Seidel sweep: M_i += (seed_i - sum_k A^T_ik M_k) / A_ii over the
// reversed visit order.  The reversed order of the sliced schedule is the forward order of the
// z-mirrored level with the colours run 3..0, so the reverse sweep runs on the same strip kernel
// (mirrored, transposed operator; increments recorded per visit).  The b-adjoint is M after the
// last reversed visit.  The operator adjoint then needs, per visit, mu and the forward x the row
// saw; the forward kept x after every visit, and which visit of a neighbour a row saw follows
// from the sequential order (neighbours in slice z+1 or earlier colours of the same slice: this
// visit; slice z-1 or later colours: the previous one).

// ------------------------------------------------------------------ small helpers
constexpr int kIdxSlots = 32;  // schedule-order neighbour index rows (psr_relax.cu layout)

template <class T>
__global__ void axpy_kernel(const T* a, const T* b, int64_t n, T* out) {  // out = a + b (b may be null)
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = b ? a[i] + b[i] : a[i];
}

template <class T>
__global__ void to_double_kernel(const T* a, int64_t n, double* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = double(a[i]);
}

// d/dp of the degree-1 hat at node c (screening_stencils.py:28-32; assembly_adjoint.py:39-49):
// zero derivative where |t| >= 1 or exactly at the node.
template <class T>
__device__ __forceinline__ T hat3_grad(const T p[3], const int c[3], int depth, T g[3]) {
  const T n = T(1 << depth);
  T h[3], dh[3];
  for (int a = 0; a < 3; ++a) {
    T t = p[a] * n - T(c[a]);
    h[a] = dmax(T(1.0) - fabs(t), T(0.0));
    dh[a] = (fabs(t) < T(1) && t != T(0)) ? (t > T(0) ? -n : n) : T(0);
  }
  g[0] = dh[0] * h[1] * h[2];
  g[1] = h[0] * dh[1] * h[2];
  g[2] = h[0] * h[1] * dh[2];
  return h[0] * h[1] * h[2];
}

// Schedule group of a key at sliced depth (slice z, colour (x&1) + 2(y&1)).
__device__ __forceinline__ int sched_group(const int c[3]) { return 4 * c[2] + (c[0] & 1) + 2 * (c[1] & 1); }

// ------------------------------------------------------------------ mirrored, transposed operator
// Transposed operator in the forward schedule layout: slot k of row p holds A_{nbr, row}, the
// neighbour's entry at the opposite offset (slot 26 - k); the index rows are the forward's.
template <class S, class I>
__global__ void transpose_values_kernel(int64_t n, const int64_t* skeys, const int32_t* off, const S* svals,
                                        const I* sidx, S* tvals) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  int c[3];
  key_coords(skeys[p], c);
  const I* row = sidx + p * kIdxSlots;
  __align__(16) S v[kSlots];
  for (int k = 0; k < 27; ++k) {
    const I idx = row[idx_slot<I>(p, k)];
    S a = S(0);
    if (idx >= 0) {
      int q[3] = {c[0] + k / 9 - 1, c[1] + (k / 3) % 3 - 1, c[2] + k % 3 - 1};
      const int64_t pn = off[sched_group(q)] + int64_t(idx);
      a = svals[pn * kSlots + (26 - k)];
    }
    v[k] = a;
  }
  v[27] = S(0);
  int4* dst = reinterpret_cast<int4*>(tvals + p * kSlots);
  const int4* src = reinterpret_cast<const int4*>(v);
  for (int q = 0; q < kSlots * int(sizeof(S)) / 16; ++q) dst[q] = src[q];
}

template <class T>
__global__ void gather_seed_kernel(const int32_t* perm, int64_t n, const T* seed, T* out) {
  int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p < n) out[p] = seed[perm[p]];
}

// ------------------------------------------------------------------ fused level reverse kernel
// One row per thread (key order).  Operator adjoint of the row (from the visit records, or
// given explicitly for the base level), cross term C^T g_b into the coarser cumulative
// adjoint, and the screening VJP of every point in the row's eight cells
// (assembly_adjoint.py:69-100) for the same-depth and the cross operator.
template <class T, class S, class I>
struct LevelReverse {
  // rows
  const int64_t* keys = nullptr;
  int64_t n = 0;
  int d = 0, iters = 0;
  ColumnView cv;
  int64_t coff = 0;            // key offset of depth d-1 in the global key array
  const T* g_b = nullptr;      // rhs adjoint, key order
  // sliced operator (schedule order) and visit records
  const int32_t* inv = nullptr;
  const int32_t* off = nullptr;
  const I* sidx = nullptr;
  const T* xhist = nullptr;    // n x iters forward x after each visit (schedule order)
  const T* mu = nullptr;       // n x iters increments of the reversed sweep (schedule order)
  // base level: explicit operator adjoint (28 slots, key order)
  const T* g_A = nullptr;
  // cross
  bool cross = false;
  const int32_t* ccols = nullptr;  // forward's cross operator (28 slots, key order); else recomputed
  const T* cvals = nullptr;
  const double* ctable = nullptr;
  const T* cum_prev = nullptr;
  T* g_cum_prev = nullptr;
  // points
  bool screened = false;
  PointsView<T> P;
  T* g_pos = nullptr;
  T* g_w = nullptr;
  // when set, the row's operator adjoint is written here (27 per row, key order) and the
  // screening VJP is left to screening_points_reverse_kernel
  T* row_gA = nullptr;
};

template <class T, class S, class I, bool SLICED, int ITERS = 0>
__global__ void level_reverse_kernel(LevelReverse<T, S, I> L) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= L.n) return;
  int c[3];
  key_coords(L.keys[i], c);
  const T gb = L.g_b[i];
  // operator adjoint of the row
  T gA[27];
  for (int k = 0; k < 27; ++k) gA[k] = T(0);
  if (SLICED) {
    const int64_t p = L.inv[i];
    const int own = (c[0] & 1) + 2 * (c[1] & 1);
    // the row's index record (vector loads) and its increments of every visit, loaded once
    __align__(16) I row[kIdxSlots];
    load_idx_row_ldg(L.sidx + p * kIdxSlots, p, row);
    const int iters = ITERS > 0 ? ITERS : L.iters;
    const T* mrow = L.mu + p * iters;
    // fixed visit count (the common 8): records in registers, vector loads
    T mu[ITERS > 0 ? ITERS : 1];
    if constexpr (ITERS > 0) {
#pragma unroll
      for (int u = 0; u < ITERS; ++u) mu[u] = __ldg(mrow + u);  // mirrored visit u = forward visit ITERS-1-u
    }
    for (int k = 0; k < 27; ++k) {
      const I idx = row[k];
      if (idx < 0) continue;
      int q[3] = {c[0] + k / 9 - 1, c[1] + (k / 3) % 3 - 1, c[2] + k % 3 - 1};
      const int64_t pk = L.off[sched_group(q)] + int64_t(idx);
      const int qc = (q[0] & 1) + 2 * (q[1] & 1);
      // 0: the neighbour's value after this visit, 1: after the previous visit
      const bool delayed = !(k == 13 || q[2] > c[2] || (q[2] == c[2] && qc < own));
      T acc = T(0);
      const T* xrow = L.xhist + pk * iters;
      if constexpr (ITERS > 0) {
        T xv[ITERS];
#pragma unroll
        for (int t = 0; t < ITERS; ++t) xv[t] = __ldg(xrow + t);
#pragma unroll
        for (int t = 0; t < ITERS; ++t) {
          const T x_now = xv[t];
          const T x_prev = t > 0 ? xv[t > 0 ? t - 1 : 0] : T(0);
          acc = acc - mu[ITERS - 1 - t] * (delayed ? x_prev : x_now);
        }
      } else {
        for (int t = 0; t < iters; ++t) {
          const T m = mrow[iters - 1 - t];
          const int tv = delayed ? t - 1 : t;
          const T xv = tv >= 0 ? xrow[tv] : T(0);
          acc = acc - m * xv;
        }
      }
      gA[k] = acc;
    }
  } else {
    for (int k = 0; k < 27; ++k) gA[k] = L.g_A[i * kSlots + k];
  }
  // cross operator: rows at d, trial functions at d-1
  int32_t ccol[27];
  uint32_t cpresent = 0;
  T gC[27];
  double cacc[27];
  int q0c[3] = {0, 0, 0};
  if (L.cross && L.ccols) {
    int ctr[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
    for (int a = 0; a < 3; ++a) q0c[a] = ctr[a] - 1;
    __align__(16) int32_t ccr[kSlots];
    {
      const int4* src = reinterpret_cast<const int4*>(L.ccols + i * kSlots);
      int4* dst = reinterpret_cast<int4*>(ccr);
#pragma unroll
      for (int q = 0; q < kSlots / 4; ++q) dst[q] = __ldg(src + q);
    }
    for (int k = 0; k < 27; ++k) {
      gC[k] = T(0);
      const int32_t col = ccr[k];
      if (col < 0) continue;
      cpresent |= 1u << k;
      const T v = L.cvals[i * kSlots + k];
      if (gb != T(0)) atomicAdd(L.g_cum_prev + col, -(v * gb));
      if (!L.row_gA) gC[k] = -(gb * L.cum_prev[col]);
    }
  } else if (L.cross) {
    int ctr[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
    cpresent = neighbours27(L.cv, L.d - 1, ctr, L.coff, ccol);
    for (int k = 0; k < 27; ++k) cacc[k] = 0.0;
    for (int a = 0; a < 3; ++a) q0c[a] = ctr[a] - 1;
    if (L.screened) screening_row(L.P, c, L.d, L.d - 1, q0c, cpresent, cacc);
    for (int k = 0; k < 27; ++k) {
      gC[k] = T(0);
      if (ccol[k] < 0) continue;
      const double* x = L.ctable + (c[0] * 3 + k / 9) * 2;
      const double* y = L.ctable + (c[1] * 3 + (k / 3) % 3) * 2;
      const double* z = L.ctable + (c[2] * 3 + k % 3) * 2;
      double stiff = x[1] * y[0] * z[0] + x[0] * y[1] * z[0] + x[0] * y[0] * z[1];
      T v = T(L.screened ? stiff + cacc[k] : stiff);
      if (gb != T(0)) atomicAdd(L.g_cum_prev + ccol[k], -(v * gb));
      gC[k] = -(gb * L.cum_prev[ccol[k]]);
    }
  }
  if (!L.screened) return;
  if (L.row_gA) {
    for (int k = 0; k < 27; ++k) L.row_gA[i * 27 + k] = gA[k];
    return;
  }
  // screening VJP (point load: b = T(load) + T(0.5) T(point load))
  const T gl = T(0.5) * gb;
  const int nt = 1 << L.d, ntc = 1 << (L.d > 0 ? L.d - 1 : 0);
  uint32_t present = 0;
  for (int k = 0; k < 27; ++k)
    if (gA[k] != T(0)) present |= 1u << k;
  const int q0[3] = {c[0] - 1, c[1] - 1, c[2] - 1};
  for (int k8 = 0; k8 < 8; ++k8) {
    int cell[3] = {c[0] - k8 / 4, c[1] - (k8 / 2) % 2, c[2] - k8 % 2};
    if (dmin(cell[0], dmin(cell[1], cell[2])) < 0 || dmax(cell[0], dmax(cell[1], cell[2])) >= nt) continue;
    int32_t u = L.P.bins.find(basis_key(L.d, cell[0], cell[1], cell[2]));
    if (u < 0) continue;
    for (int32_t j = L.P.bstart[u]; j < L.P.bstart[u + 1]; ++j) {
      const T p[3] = {L.P.spos[3 * j], L.P.spos[3 * j + 1], L.P.spos[3 * j + 2]};
      const T w = L.P.sw[j];
      if (w == T(0)) continue;
      T dphi[3];
      const T phi = hat3_grad(p, c, L.d, dphi);
      T gp[3] = {gl * w * dphi[0], gl * w * dphi[1], gl * w * dphi[2]};
      T gw = gl * phi;
      int f[3];
      for (int a = 0; a < 3; ++a) f[a] = min(max(int(floor(p[a] * T(nt))), 0), nt - 1) - q0[a];
      for (int e = 0; e < 8; ++e) {
        int s0 = f[0] + e / 4, s1 = f[1] + (e / 2) % 2, s2 = f[2] + e % 2;
        if (s0 < 0 || s0 > 2 || s1 < 0 || s1 > 2 || s2 < 0 || s2 > 2) continue;
        int k = s0 * 9 + s1 * 3 + s2;
        if (!((present >> k) & 1)) continue;
        int q[3] = {q0[0] + s0, q0[1] + s1, q0[2] + s2};
        T dtr[3];
        const T tr = hat3_grad(p, q, L.d, dtr);
        const T g = gA[k], gwp = g * w;
        gw = gw + g * (phi * tr);
        for (int a = 0; a < 3; ++a) gp[a] = gp[a] + (gwp * tr) * dphi[a] + (gwp * phi) * dtr[a];
      }
      if (L.cross) {
        for (int a = 0; a < 3; ++a) f[a] = min(max(int(floor(p[a] * T(ntc))), 0), ntc - 1) - q0c[a];
        for (int e = 0; e < 8; ++e) {
          int s0 = f[0] + e / 4, s1 = f[1] + (e / 2) % 2, s2 = f[2] + e % 2;
          if (s0 < 0 || s0 > 2 || s1 < 0 || s1 > 2 || s2 < 0 || s2 > 2) continue;
          int k = s0 * 9 + s1 * 3 + s2;
          if (!((cpresent >> k) & 1)) continue;
          int q[3] = {q0c[0] + s0, q0c[1] + s1, q0c[2] + s2};
          T dtr[3];
          const T tr = hat3_grad(p, q, L.d - 1, dtr);
          const T g = gC[k], gwp = g * w;
          gw = gw + g * (phi * tr);
          for (int a = 0; a < 3; ++a) gp[a] = gp[a] + (gwp * tr) * dphi[a] + (gwp * phi) * dtr[a];
        }
      }
      const int32_t index = L.P.ids[j];
      for (int a = 0; a < 3; ++a)
        if (gp[a] != T(0)) atomicAdd(L.g_pos + 3 * index + a, gp[a]);
      if (gw != T(0)) atomicAdd(L.g_w + index, gw);
    }
  }
}

// The per-row pass of a sliced level with the stored cross operator, unrolled so that every
// per-slot quantity stays in registers: the operator adjoint of the row (written to row_gA,
// 27 per row, for the per-point screening pass) and -C^T g_b into the coarser cumulative.
template <class T, class I, int ITERS>
__global__ void __launch_bounds__(128) level_rows_reverse_kernel(const int64_t* __restrict__ skeys, int64_t n,
                                                                 const int32_t* __restrict__ perm,
                                                                 const int32_t* __restrict__ off,
                                                                 const I* __restrict__ sidx,
                                                                 const T* __restrict__ xhist,
                                                                 const T* __restrict__ mu_hist,
                                                                 const T* __restrict__ g_b,
                                                                 const int32_t* __restrict__ ccols,
                                                                 const T* __restrict__ cvals, T* g_cum_prev,
                                                                 T* row_gA) {
  // one thread per schedule position: consecutive threads are neighbours in one (slice,
  // colour) group, so their neighbours' visit records are read together
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  int c[3];
  key_coords(skeys[p], c);
  const int64_t i = perm[p];
  const int own = (c[0] & 1) + 2 * (c[1] & 1);
  __align__(16) I row[kIdxSlots];
  load_idx_row_ldg(sidx + p * kIdxSlots, p, row);
  // visit records as 16-byte vector loads (a row's ITERS values are contiguous and aligned)
  static_assert(ITERS * sizeof(T) % 16 == 0, "visit records in 16-byte vectors");
  __align__(16) T mu[ITERS];  // reverse visit u
#pragma unroll
  for (int q = 0; q < ITERS * int(sizeof(T)) / 16; ++q)
    reinterpret_cast<int4*>(mu)[q] = __ldg(reinterpret_cast<const int4*>(mu_hist + p * ITERS) + q);
  T* out = row_gA ? row_gA + i * 27 : nullptr;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const I idx = row[k];
    T acc = T(0);
    if (idx >= 0) {
      const int q[3] = {c[0] + k / 9 - 1, c[1] + (k / 3) % 3 - 1, c[2] + k % 3 - 1};
      const int64_t pk = __ldg(off + sched_group(q)) + int64_t(idx);
      const int qc = (q[0] & 1) + 2 * (q[1] & 1);
      const bool delayed = !(k == 13 || k % 3 == 2 || (k % 3 == 1 && qc < own));
      const int4* xrow = reinterpret_cast<const int4*>(xhist + pk * ITERS);
      __align__(16) T xv[ITERS];
#pragma unroll
      for (int q = 0; q < ITERS * int(sizeof(T)) / 16; ++q) reinterpret_cast<int4*>(xv)[q] = __ldg(xrow + q);
#pragma unroll
      for (int t = 0; t < ITERS; ++t) {
        const T x_prev = t > 0 ? xv[t > 0 ? t - 1 : 0] : T(0);
        acc = acc - mu[ITERS - 1 - t] * (delayed ? x_prev : xv[t]);
      }
    }
    if (out) out[k] = acc;
  }
  const T gb = g_b[i];
  if (gb == T(0)) return;
  __align__(16) int32_t cc[kSlots];
  {
    const int4* src = reinterpret_cast<const int4*>(ccols + i * kSlots);
    int4* dst = reinterpret_cast<int4*>(cc);
#pragma unroll
    for (int q = 0; q < kSlots / 4; ++q) dst[q] = __ldg(src + q);
  }
#pragma unroll
  for (int k = 0; k < 27; ++k)
    if (cc[k] >= 0) atomicAdd(g_cum_prev + cc[k], -(__ldg(cvals + i * kSlots + k) * gb));
}

// Screening VJP per point (assembly_adjoint.py:69-100, gathered): a point of bin cell b
// (floor bins at depth d) enters the rows at the eight corners b + {0,1}^3 that exist; for
// each, the point-load term, the same-depth trial functions (the corners of b) and, with a
// cross operator, the depth d-1 trial functions (the corners of the point's depth d-1 bin).
// Row adjoints come from level_reverse_kernel (gA, gC: 27 per row; gA may use a 28-slot
// stride).  One thread per point, no atomics.
template <class T>
__global__ void screening_points_reverse_kernel(PointsView<T> P, int64_t m, int d, ColumnView cv, int64_t row_off,
                                                const T* g_b, const T* gA, int gA_stride, const T* cum_prev,
                                                int64_t coff, T* g_pos, T* g_w) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  const T w = P.w[i];
  if (w == T(0)) return;
  const T p[3] = {P.pos[3 * i], P.pos[3 * i + 1], P.pos[3 * i + 2]};
  const int nt = 1 << d, ntc = 1 << (d > 0 ? d - 1 : 0);
  int b[3], bc[3];
  for (int a = 0; a < 3; ++a) {
    b[a] = min(max(int(floor(p[a] * T(nt))), 0), nt - 1);
    bc[a] = min(max(int(floor(p[a] * T(ntc))), 0), ntc - 1);
  }
  // cross trial functions: the corners of the point's depth d-1 bin, with the coarser
  // cumulative solution there (the cross operator's adjoint is -g_b(row) * cumulative(q))
  T cq[8];
  if (cum_prev) {
    for (int e = 0; e < 8; ++e) {
      const int q[3] = {bc[0] + e / 4, bc[1] + (e / 2) % 2, bc[2] + e % 2};
      const int32_t j = cv.find(d - 1, q[0], q[1], q[2]);
      cq[e] = j >= 0 ? cum_prev[int64_t(j) - coff] : T(0);
    }
  }
  T gp[3] = {T(0), T(0), T(0)};
  T gw = T(0);
  for (int ex = 0; ex < 2; ++ex)
    for (int ey = 0; ey < 2; ++ey) {
      int32_t count;
      const int rx = b[0] + ex, ry = b[1] + ey;
      const int32_t j0 = cv.column_range(d, rx, ry, count);
      if (j0 < 0) continue;
      const int64_t colk = ColumnView::column_key(d, rx, ry) >> 16;
      const int64_t end = count == INT32_MAX ? cv.n : int64_t(j0) + count;
      int32_t j = cv.lower_z(j0, count, colk, b[2]);
      for (int ez = 0; ez < 2; ++ez) {
        if (j >= end) break;
        const int64_t key = __ldg(cv.keys + j);
        if ((key >> 16) != colk) break;
        const int rz = int(key & 65535);
        if (rz != b[2] + ez) continue;
        const int64_t row = int64_t(j) - row_off;
        ++j;
        const int r[3] = {rx, ry, rz};
        T dphi[3];
        const T phi = hat3_grad(p, r, d, dphi);
        const T gl = T(0.5) * g_b[row];
        gw = gw + gl * phi;
        for (int a = 0; a < 3; ++a) gp[a] = gp[a] + gl * w * dphi[a];
        const T* ga = gA + row * gA_stride;
        for (int e = 0; e < 8; ++e) {
          const int q[3] = {b[0] + e / 4, b[1] + (e / 2) % 2, b[2] + e % 2};
          const int k = (q[0] - r[0] + 1) * 9 + (q[1] - r[1] + 1) * 3 + (q[2] - r[2] + 1);
          const T g = ga[k];
          if (g == T(0)) continue;
          T dtr[3];
          const T tr = hat3_grad(p, q, d, dtr);
          const T gwp = g * w;
          gw = gw + g * (phi * tr);
          for (int a = 0; a < 3; ++a) gp[a] = gp[a] + (gwp * tr) * dphi[a] + (gwp * phi) * dtr[a];
        }
        if (cum_prev) {
          const T gbr = g_b[row];
          for (int e = 0; e < 8; ++e) {
            const int q[3] = {bc[0] + e / 4, bc[1] + (e / 2) % 2, bc[2] + e % 2};
            const T g = -(gbr * cq[e]);
            if (g == T(0)) continue;
            T dtr[3];
            const T tr = hat3_grad(p, q, d - 1, dtr);
            const T gwp = g * w;
            gw = gw + g * (phi * tr);
            for (int a = 0; a < 3; ++a) gp[a] = gp[a] + (gwp * tr) * dphi[a] + (gwp * phi) * dtr[a];
          }
        }
      }
    }
  for (int a = 0; a < 3; ++a) g_pos[3 * i + a] = g_pos[3 * i + a] + gp[a];
  g_w[i] = g_w[i] + gw;
}

// g_coarse[parent] += w * g_fine[i] over the prolongation stencil (transpose of prolong_add).
template <class T>
__global__ void prolong_transpose_kernel(const int32_t* pcol, const T* pval, int64_t n, const T* g_fine, T* g_coarse) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const T g = g_fine[i];
  if (g == T(0)) return;
  for (int e = 0; e < 8; ++e) {
    int32_t c = pcol[i * 8 + e];
    if (c < 0) break;
    atomicAdd(g_coarse + c, pval[i * 8 + e] * g);
  }
}

// g_fine[i] += sum_e w_e g_coarse[pcol_e] (the prolongation applied to an adjoint).
template <class T, class V>
__global__ void prolong_apply_kernel(const int32_t* pcol, const T* pval, int64_t n, const V* g_coarse, V* g_fine) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  V s = V(0);
  for (int e = 0; e < 8; ++e) {
    int32_t c = pcol[i * 8 + e];
    if (c < 0) break;
    s = s + V(pval[i * 8 + e]) * g_coarse[c];
  }
  g_fine[i] = g_fine[i] + s;
}

// ------------------------------------------------------------------ base multigrid reverse
// ---- colour relaxation reversed as a Gauss-Seidel sweep on A^T (no atomics)
// Transposed operator in the same 28-slot layout: slot k of row i holds A_{col, i}, the
// neighbour's entry at the opposite offset (slot 26 - k).
template <class T>
__global__ void transpose_slots_kernel(const int32_t* cols, const T* vals, int64_t n, T* vals_t) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  for (int k = 0; k < kSlots; ++k) {
    const int32_t c = k < 27 ? cols[i * kSlots + k] : -1;
    vals_t[i * kSlots + k] = c >= 0 ? vals[int64_t(c) * kSlots + (26 - k)] : T(0);
  }
}

// lambda -= A^T M  (the adjoint leaving the call), and g_b += M.
template <class T>
__global__ void adjoint_out_kernel(const int32_t* cols, const T* vals_t, const T* M, int64_t n, T* lambda, T* g_b) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  T s = T(0);
  for (int k = 0; k < 27; ++k) {
    const int32_t c = cols[i * kSlots + k];
    if (c < 0) continue;
    s = s + vals_t[i * kSlots + k] * M[c];
  }
  lambda[i] = lambda[i] - s;
  g_b[i] = g_b[i] + M[i];
}

__device__ __forceinline__ int colour8(const int c[3]) { return (c[0] & 1) + 2 * (c[1] & 1) + 4 * (c[2] & 1); }

// Operator adjoint of one colour-relaxation call: g_A_ik -= sum_t mu_i(t) x_k(seen at visit t),
// mu from the transposed sweep's records, x from the forward call's records.
template <class T>
__global__ void relax_operator_adjoint_kernel(const int64_t* keys, const int32_t* cols, const T* vals, int64_t n,
                                              int iters, int forward, const T* hist_fwd, const T* hist_rev, T* g_A) {
  // one thread per (row, slot)
  const int64_t t0 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (t0 >= 27 * n) return;
  const int64_t i = t0 / 27;
  const int k = int(t0 % 27);
  int ci[3];
  key_coords(keys[i], ci);
  const int pos_i = forward ? colour8(ci) : 7 - colour8(ci);
  // the rows hold their k-th neighbour in slot k, so a row's own column is slot 13
  const T diag_i = cols[i * kSlots + 13] == int32_t(i) ? vals[i * kSlots + 13] : T(0);
  if (diag_i == T(0)) return;
  const T inv_i = T(1.0) / diag_i;
  {
    const int32_t c = cols[i * kSlots + k];
    if (c < 0) return;
    int ck[3];
    key_coords(keys[c], ck);
    const int pos_k = forward ? colour8(ck) : 7 - colour8(ck);
    T diag_k = T(0);
    if ((c == int32_t(i) || pos_k < pos_i) && cols[int64_t(c) * kSlots + 13] == c)
      diag_k = vals[int64_t(c) * kSlots + 13];
    T acc = T(0);
    for (int t = 0; t < iters; ++t) {
      const T mu = hist_rev[2 * (int64_t(iters - 1 - t) * n + i) + 1] * inv_i;
      T xv;
      if (c == int32_t(i) || pos_k < pos_i) {  // seen after its own visit t
        const T* rec = hist_fwd + 2 * (int64_t(t) * n + c);
        xv = diag_k != T(0) ? rec[0] + rec[1] * (T(1.0) / diag_k) : rec[0];
      } else {  // seen before its visit t
        xv = hist_fwd[2 * (int64_t(t) * n + c)];
      }
      acc = acc - mu * xv;
    }
    g_A[i * kSlots + k] = g_A[i * kSlots + k] + acc;
  }
}

template <class T>
struct BaseTranspose {
  std::vector<DBuf<T>> vals_t;
};

// Reverse of one relax_colors call (forward flag `forward`): lambda (in/out) is the adjoint
// of x, g_b and g_A accumulate.
template <class T>
static void relax_colors_adjoint(const int64_t* keys, const int32_t* cols, const T* vals, const T* vals_t,
                                 const int32_t* rows, const int32_t* group_off, int iters, int forward,
                                 const T* hist_fwd, int64_t n, T* lambda, T* g_b, T* g_A, cudaStream_t s) {
  if (n <= 0) return;
  DBuf<T> M(n, s), hist_rev(2 * int64_t(iters) * n, s);
  M.zero();
  relax_colors<T>(cols, vals_t, lambda, M.p, rows, group_off, iters, forward ? 0 : 1, hist_rev.p, n, s);
  relax_operator_adjoint_kernel<T><<<blocks_for(27 * n), kThreads, 0, s>>>(keys, cols, vals, n, iters, forward, hist_fwd,
                                                                       hist_rev.p, g_A);
  PSR_LAUNCH_CHECK();
  adjoint_out_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(cols, vals_t, M.p, n, lambda, g_b);
  PSR_LAUNCH_CHECK();
}

// r = rhs - A x reversed: g_rhs += g_r, g_x -= A^T g_r, g_A_ik -= g_r_i x_k.
template <class T>
__global__ void residual_reverse_kernel(const int32_t* cols, const T* vals, const T* x, const T* g_r, int64_t n,
                                        T* g_rhs, T* g_x, T* g_A) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const T g = g_r[i];
  if (g == T(0)) return;
  g_rhs[i] = g_rhs[i] + g;
  for (int k = 0; k < 27; ++k) {
    const int32_t c = cols[i * kSlots + k];
    if (c < 0) continue;
    atomicAdd(g_x + c, -(vals[i * kSlots + k] * g));
    g_A[i * kSlots + k] = g_A[i * kSlots + k] - g * x[c];
  }
}

// A_c = P^T A_f P reversed (multigrid_adjoint.py:36-48): for each fine entry (a, b),
// g_A_f[a][b] += sum_{i in P(a), j in P(b)} P_ai g_A_c[i][j] P_bj.
template <class T>
__global__ void galerkin_reverse_kernel(const int64_t* fine_keys, int64_t nf, const int32_t* fcols,
                                        const int32_t* pcol, const T* pval, const int64_t* coarse_keys,
                                        const int32_t* ccols, const T* g_Ac, T* g_Af) {
  // one thread per (fine row, slot): 27x the threads of a row loop, same sums
  const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (t >= 27 * nf) return;
  const int64_t a = t / 27;
  const int e = int(t % 27);
  {
    const int32_t b = fcols[a * kSlots + e];
    if (b < 0) return;
    T total = T(0);
    for (int u = 0; u < 8; ++u) {
      const int32_t ci = pcol[a * 8 + u];
      if (ci < 0) break;
      int cc[3];
      key_coords(coarse_keys[ci], cc);
      for (int v = 0; v < 8; ++v) {
        const int32_t cj = pcol[int64_t(b) * 8 + v];
        if (cj < 0) break;
        int cd[3];
        key_coords(coarse_keys[cj], cd);
        int dx = cd[0] - cc[0] + 1, dy = cd[1] - cc[1] + 1, dz = cd[2] - cc[2] + 1;
        if (dx < 0 || dx > 2 || dy < 0 || dy > 2 || dz < 0 || dz > 2) continue;
        const int slot = dx * 9 + dy * 3 + dz;
        if (ccols[int64_t(ci) * kSlots + slot] != cj) continue;
        total = total + pval[a * 8 + u] * g_Ac[int64_t(ci) * kSlots + slot] * pval[int64_t(b) * 8 + v];
      }
    }
    g_Af[a * kSlots + e] = g_Af[a * kSlots + e] + total;
  }
}

// Root CG reversed (solver_adjoint.py:135-196): replays the forward CG of root_solve_kernel
// with its stopping decisions and reverses it.  One thread; 64 x 64 at most, at most nk steps.
template <class T>
__global__ void root_reverse_kernel(const int64_t* keys, int nk, const int32_t* cols, const T* vals, const T* rhs,
                                    const T* x0in, int dc, double cg_accuracy, int base, int cycle, const T* g_out,
                                    const T* g_state_out, T* g_rhs, T* g_x0, T* g_state_in, T* g_A, T* work) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int N = dc ? 64 : nk;
  // work layout: K[64*64] has[64*64] | per step p, Ap (nk+1 steps) | scalars
  T* K = work;
  T* has = K + 64 * 64;
  T* P = has + 64 * 64;             // (nk + 1) x 64
  T* AP = P + 65 * 64;              // nk x 64
  T* R = AP + 64 * 64;              // (nk + 1) x 64 residuals
  T* X = R + 65 * 64;               // x after each step (unused in reverse but kept for clarity)
  T* sc = X + 65 * 64;              // per step: rr, pAp, alpha, rrn, beta (5 x 64)
  for (int a = 0; a < N * 64; ++a) K[a] = has[a] = T(0);
  T bb[64], xx[64];
  for (int a = 0; a < N; ++a) {
    bb[a] = T(0);
    xx[a] = dc ? x0in[a] : T(0);
  }
  for (int i = 0; i < nk; ++i) {
    int ri = dc ? root_row(keys[i]) : i;
    bb[ri] = rhs[i];
    if (!dc) xx[ri] = x0in[i];
    for (int k = 0; k < 27; ++k) {
      int32_t c = cols[i * kSlots + k];
      if (c < 0) continue;
      int rc = dc ? root_row(keys[c]) : c;
      K[ri * 64 + rc] = vals[i * kSlots + k];
      has[ri * 64 + rc] = T(1);
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
        if (has[a * 64 + q] != T(0)) s = s + K[a * 64 + q] * in[q];
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
  // forward replay
  T residual[64];
  for (int a = 0; a < N; ++a) residual[a] = bb[a];
  if (base == 0 && cycle > 0) apply(xx, bb, residual, -1, 1);
  T nsq = dot(residual, residual);
  int steps = 0;
  bool ran = double(nsq) > cg_accuracy * cg_accuracy;
  T gate = T(0);
  if (ran) {
    double tol = base == 0 ? 0.0 : cg_accuracy;
    double atol = base == 0 ? cg_accuracy * sqrt(double(nsq)) : 0.0;
    double eps = sizeof(T) == 8 ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    double bnorm = sqrt(double(dot(bb, bb)));
    double abs_tol = dmax(dmax(atol, tol * bnorm), pow(eps, 9.0 / 4.0));
    double atol_sq = abs_tol * abs_tol;
    gate = T(atol_sq);
    apply(xx, bb, R, -1, 1);
    T rr = dot(R, R);
    for (int a = 0; a < N; ++a) P[a] = R[a];
    for (int it = 0; it < nk; ++it) {
      if (double(rr) <= atol_sq) break;
      T* p = P + it * 64;
      T* ap = AP + it * 64;
      T* r = R + it * 64;
      T* rn = R + (it + 1) * 64;
      apply(p, ap, ap, 1, 0);
      T pAp = dot(p, ap);
      T alpha = rr > gate ? rr / pAp : T(0);
      for (int a = 0; a < N; ++a) {
        xx[a] = xx[a] + alpha * p[a];
        rn[a] = r[a] - alpha * ap[a];
      }
      T rr_new = dot(rn, rn);
      T beta = rr_new > gate ? rr_new / rr : T(0);
      T* pn = P + (it + 1) * 64;
      for (int a = 0; a < N; ++a) pn[a] = rn[a] + beta * p[a];
      sc[0 * 64 + it] = rr;
      sc[1 * 64 + it] = pAp;
      sc[2 * 64 + it] = alpha;
      sc[3 * 64 + it] = rr_new;
      sc[4 * 64 + it] = beta;
      rr = rr_new;
      ++steps;
    }
  }
  // reverse
  T gx[64], gr[64], gp[64], gK_unused = T(0);
  (void)gK_unused;
  for (int a = 0; a < N; ++a) {
    gx[a] = dc ? g_state_out[a] : T(0);
    gr[a] = T(0);
    gp[a] = T(0);
  }
  for (int i = 0; i < nk; ++i) {
    int ri = dc ? root_row(keys[i]) : i;
    gx[ri] = gx[ri] + g_out[i];
  }
  T gbb[64], gxx0[64];
  for (int a = 0; a < N; ++a) {
    gbb[a] = T(0);
    gxx0[a] = gx[a];
  }
  auto add_gK = [&](const T* gv, const T* v, T sign) {  // g_K[a][q] += sign * gv[a] * v[q]
    for (int i = 0; i < nk; ++i) {
      int ri = dc ? root_row(keys[i]) : i;
      if (gv[ri] == T(0)) continue;
      for (int k = 0; k < 27; ++k) {
        int32_t c = cols[i * kSlots + k];
        if (c < 0) continue;
        int rc = dc ? root_row(keys[c]) : c;
        g_A[i * kSlots + k] = g_A[i * kSlots + k] + sign * gv[ri] * v[rc];
      }
    }
  };
  // K^T g (+ dc: constant mode) into out
  auto apply_t = [&](const T* g, T* out, T sign) {
    T mean = T(0);
    if (dc) {
      for (int a = 0; a < N; ++a) mean = mean + g[a];
      mean = mean / T(N);
    }
    for (int q = 0; q < N; ++q) {
      T s = T(0);
      for (int a = 0; a < N; ++a)
        if (has[a * 64 + q] != T(0)) s = s + K[a * 64 + q] * g[a];
      if (dc) s = s + mean;
      out[q] = out[q] + sign * s;
    }
  };
  if (ran) {
    T grr = T(0);
    for (int it = steps - 1; it >= 0; --it) {
      const T* p = P + it * 64;
      const T* ap = AP + it * 64;
      const T* rn = R + (it + 1) * 64;
      const T rr = sc[it], pAp = sc[64 + it], alpha = sc[128 + it], rr_new = sc[192 + it], beta = sc[256 + it];
      // p_next = rn + beta p
      T gbeta = T(0);
      T gpn[64];
      for (int a = 0; a < N; ++a) {
        gpn[a] = gp[a];
        gbeta = gbeta + gp[a] * p[a];
      }
      T grn[64];
      for (int a = 0; a < N; ++a) grn[a] = gr[a] + gpn[a];
      T gp_it[64];
      for (int a = 0; a < N; ++a) gp_it[a] = beta * gpn[a];
      T grr_new = grr;  // rr carried to the next step is rr_new
      T grr_it = T(0);
      if (rr_new > gate) {
        grr_new = grr_new + gbeta / rr;
        grr_it = grr_it - gbeta * rr_new / (rr * rr);
      }
      for (int a = 0; a < N; ++a) grn[a] = grn[a] + T(2) * grr_new * rn[a];
      // rn = r - alpha ap ; x_next = x + alpha p
      T galpha = T(0);
      T gap[64];
      for (int a = 0; a < N; ++a) {
        galpha = galpha - grn[a] * ap[a] + gx[a] * p[a];
        gap[a] = -alpha * grn[a];
        gp_it[a] = gp_it[a] + alpha * gx[a];
      }
      if (rr > gate) {
        grr_it = grr_it + galpha / pAp;
        const T gpAp = -galpha * rr / (pAp * pAp);
        for (int a = 0; a < N; ++a) {
          gp_it[a] = gp_it[a] + gpAp * ap[a];
          gap[a] = gap[a] + gpAp * p[a];
        }
      }
      // ap = K p (+ mean)
      apply_t(gap, gp_it, T(1));
      add_gK(gap, p, T(1));
      for (int a = 0; a < N; ++a) {
        gp[a] = gp_it[a];
        gr[a] = grn[a];
      }
      grr = grr_it;
    }
    // p0 = r0, rr0 = r0.r0, r0 = bb - K xx0 (- mean)
    const T* r0 = R;
    T gr0[64];
    for (int a = 0; a < N; ++a) gr0[a] = gr[a] + gp[a] + T(2) * grr * r0[a];
    for (int a = 0; a < N; ++a) gbb[a] = gbb[a] + gr0[a];
    T xin[64];
    for (int a = 0; a < N; ++a) xin[a] = dc ? x0in[a] : T(0);
    if (!dc)
      for (int i = 0; i < nk; ++i) xin[i] = x0in[i];
    apply_t(gr0, gxx0, T(-1));
    add_gK(gr0, xin, T(-1));
  }
  for (int i = 0; i < nk; ++i) {
    int ri = dc ? root_row(keys[i]) : i;
    g_rhs[i] = g_rhs[i] + gbb[ri];
    if (!dc) g_x0[i] = gxx0[ri];
  }
  if (dc)
    for (int a = 0; a < N; ++a) g_state_in[a] = gxx0[a];
}

// ------------------------------------------------------------------ point constraints reversed
// points_kernel: p = v.xyz / v.w, w = v.w 2^d (pw avg[1]) (zero without support / exact).
template <class T>
__global__ void points_reverse_kernel(const int64_t* keys, const T* vals, int64_t m, int d, T pw, const T* average,
                                      const T* w_out, const T* g_pos, const T* g_w, T* g_vals, T* g_average) {
  int64_t i0 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int64_t i = i0 < m ? i0 : m - 1;  // every thread reaches the block reduction
  const bool live = i0 < m;
  const T* v = vals + 4 * i;
  T gv[4] = {T(0), T(0), T(0), T(0)};
  for (int a = 0; a < 3; ++a) {
    const T g = g_pos[3 * i + a];
    gv[a] = gv[a] + g / v[3];
    gv[3] = gv[3] - g * (v[a] / v[3]) / v[3];
  }
  T gavg = T(0);
  if (live && w_out[i] != T(0)) {
    const T g = g_w[i];
    const T scale = T(1 << d);
    gv[3] = gv[3] + g * scale * (pw * average[1]);
    gavg = g * v[3] * scale * pw;
  }
  if (live)
    for (int a = 0; a < 4; ++a) g_vals[4 * i + a] = g_vals[4 * i + a] + gv[a];
  // the mean-weight adjoint: block sum, one atomic per block
  __shared__ T red[kThreads];
  red[threadIdx.x] = gavg;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0 && red[0] != T(0)) atomicAdd(g_average + 1, red[0]);
}

// ------------------------------------------------------------------ normal loads reversed
// Transpose of normal_stencil_kernel: for each normal coefficient j (at normal_depth) gather
// sum_i g_i * (x', y', z' integrals) over the test rows i whose window covers j.
template <class T>
__global__ void __launch_bounds__(256, 5) normal_stencil_reverse_kernel(const int64_t* nkeys, int64_t m, int test_depth, int normal_depth,
                                              ColumnView tcv, int64_t toff, const double* g_test, const double* table,
                                              int width, int first, T* g_vals) {
  int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (j >= m) return;
  int a[3];
  key_coords(nkeys[j], a);
  const int tl = 1 << test_depth;
  int lo[3], hi[3];
  for (int ax = 0; ax < 3; ++ax) {
    if (test_depth == normal_depth) {
      lo[ax] = a[ax] - width - first + 1;
      hi[ax] = a[ax] - first;
    } else if (test_depth < normal_depth) {  // centre 2i
      lo[ax] = (a[ax] - first - width + 1 + 1) >> 1;
      hi[ax] = (a[ax] - first) >> 1;
      if (2 * lo[ax] < a[ax] - first - width + 1) ++lo[ax];
    } else {  // centre i >> 1
      lo[ax] = 2 * (a[ax] - first - width + 1);
      hi[ax] = 2 * (a[ax] - first) + 1;
    }
    lo[ax] = max(lo[ax], 0);
    hi[ax] = min(hi[ax], tl);
  }
  double acc[3] = {0.0, 0.0, 0.0};
  for (int xi = lo[0]; xi <= hi[0]; ++xi) {
    const int cx = normal_center(xi, test_depth, normal_depth);
    const int ox = a[0] - cx - first;
    if (ox < 0 || ox >= width) continue;
    const double* ix = table + (xi * width + ox) * 2;
    for (int yi = lo[1]; yi <= hi[1]; ++yi) {
      const int cy = normal_center(yi, test_depth, normal_depth);
      const int oy = a[1] - cy - first;
      if (oy < 0 || oy >= width) continue;
      int32_t count;
      const int32_t r0 = tcv.column_range(test_depth, xi, yi, count);
      if (r0 < 0) continue;
      const double* iy = table + (yi * width + oy) * 2;
      const int64_t colk = ColumnView::column_key(test_depth, xi, yi) >> 16;
      const int64_t end = count == INT32_MAX ? tcv.n : int64_t(r0) + count;
      for (int32_t r = tcv.lower_z(r0, count, colk, lo[2]); r < end; ++r) {
        const int64_t key = __ldg(tcv.keys + r);
        if ((key >> 16) != colk) break;
        const int zi = int(key & 65535);
        if (zi > hi[2]) break;
        const int cz = normal_center(zi, test_depth, normal_depth);
        const int oz = a[2] - cz - first;
        if (oz < 0 || oz >= width) continue;
        const double* iz = table + (zi * width + oz) * 2;
        const double g = g_test[int64_t(r) - toff];
        acc[0] += g * ix[1] * iy[0] * iz[0];
        acc[1] += g * ix[0] * iy[1] * iz[0];
        acc[2] += g * ix[0] * iy[0] * iz[1];
      }
    }
  }
  for (int ax = 0; ax < 3; ++ax) g_vals[4 * j + ax] = g_vals[4 * j + ax] + T(acc[ax]);
}

// normal_stencil_reverse_kernel with the dense column table and a compile-time window, for
// test functions at the normals' own depth (MODE 0: W = 4, K = 4), one depth coarser
// (MODE 1: W = 6, centre 2i, K = 3) or one depth finer (MODE 2: W = 4, centre i >> 1,
// K = 8).  The test functions whose window holds normal a are w0 + [0, K)^3, with w0 =
// a - first - W + 1, ceil((a - first - W + 1) / 2) or 2 (a - first - W + 1); the one at
// window index u along an axis (coordinate i = w0 + u) uses table entry (i W + a -
// centre(i) - first), so the K entries along z (and y, for K <= 4) are loaded once into
// registers.  Per x the K columns' lower bounds advance in lock step (as in the forward
// stencil), and a column's test functions in the window become a bit mask over the K z
// offsets (keys ascend).  Additions in the same (x, y, z) order with the same products as
// normal_stencil_reverse_kernel: same result.
template <class T, int W, int K, int MODE>
__global__ void __launch_bounds__(256, 3) normal_stencil_reverse_window_kernel(const int64_t* nkeys, int64_t m,
                                                                               int test_depth, ColumnView tcv,
                                                                               int64_t toff, const double* g_test,
                                                                               const double* table, int first,
                                                                               T* g_vals) {
  const int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (j >= m) return;
  int a[3];
  key_coords(nkeys[j], a);
  const int tl = 1 << test_depth, side = tl + 1;
  int w0[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax)
    w0[ax] = MODE == 1 ? (a[ax] - first - W + 2) >> 1 : MODE == 2 ? 2 * (a[ax] - first - W + 1) : a[ax] - first - W + 1;
  const int zlo = max(w0[2], 0);
  const double2* tab = reinterpret_cast<const double2*>(table);
  // table entry of window index u along axis ax (zero when the coordinate is outside the grid)
  auto entry = [&](int ax, int u) {
    const int i = w0[ax] + u;
    const int off = a[ax] - (MODE == 1 ? 2 * i : MODE == 2 ? i >> 1 : i) - first;
    return i >= 0 && i <= tl ? __ldg(tab + i * W + off) : make_double2(0.0, 0.0);
  };
  constexpr int KY = K <= 4 ? K : 1;  // y entries in registers only for narrow windows
  double2 ty[KY], tz[K];
#pragma unroll
  for (int u = 0; u < K; ++u) {
    if (K <= 4) ty[u < KY ? u : 0] = entry(1, u);
    tz[u] = entry(2, u);
  }
  const int2* dense = tcv.dense + dense_column_base(test_depth);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int u = 0; u < K; ++u) {
    const int xi = w0[0] + u;
    if (xi < 0 || xi > tl) continue;
    const double2 tx = entry(0, u);
    int32_t lo[K], hi[K], end[K];
#pragma unroll
    for (int v = 0; v < K; ++v) {
      const int yi = w0[1] + v;
      lo[v] = 0;
      end[v] = 0;
      if (yi >= 0 && yi <= tl) {
        const int2 e = __ldg(dense + int64_t(xi) * side + yi);
        if (e.x >= 0) {
          lo[v] = e.x;
          end[v] = e.x + e.y;
        }
      }
      hi[v] = end[v];
    }
    for (int step = 0; step < 32; ++step) {
      bool active = false;
#pragma unroll
      for (int v = 0; v < K; ++v) active |= lo[v] < hi[v];
      if (!active) break;
#pragma unroll
      for (int v = 0; v < K; ++v) {
        if (lo[v] < hi[v]) {
          const int32_t mid = (lo[v] + hi[v]) >> 1;
          if (int(__ldg(tcv.keys + mid) & 65535) < zlo)
            lo[v] = mid + 1;
          else
            hi[v] = mid;
        }
      }
    }
#pragma unroll
    for (int v = 0; v < K; ++v) {
      const double2 tyv = K <= 4 ? ty[v < KY ? v : 0] : entry(1, v);
      uint32_t mask = 0;  // bit t: a test function at w0[2] + t
#pragma unroll
      for (int e = 0; e < K; ++e) {
        const int dz = lo[v] + e < end[v] ? int(__ldg(tcv.keys + lo[v] + e) & 65535) - w0[2] : K;
        if (dz < K) mask |= 1u << dz;
      }
#pragma unroll
      for (int t = 0; t < K; ++t) {
        if (!((mask >> t) & 1u)) continue;
        const int64_t r = int64_t(lo[v]) + __popc(mask & ((1u << t) - 1u));
        const double g = __ldg(g_test + (r - toff));
        acc[0] += g * tx.y * tyv.x * tz[t].x;
        acc[1] += g * tx.x * tyv.y * tz[t].x;
        acc[2] += g * tx.x * tyv.x * tz[t].y;
      }
    }
  }
  for (int ax = 0; ax < 3; ++ax) g_vals[4 * j + ax] = g_vals[4 * j + ax] + T(acc[ax]);
}

// Transpose of prolong_normals_kernel: own record and the 8 coarse parents.
template <class T>
__global__ void prolong_normals_reverse_kernel(const int64_t* keys, int64_t n, int d, HashView nh, HashView bh,
                                               int64_t prev_off, const T* g_cum, T* g_nvals, T* g_prev) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const T* g = g_cum + 4 * i;
  if (g[0] == T(0) && g[1] == T(0) && g[2] == T(0) && g[3] == T(0)) return;
  int c[3];
  key_coords(keys[i], c);
  int32_t j = nh.find(keys[i]);
  if (j >= 0)
    for (int a = 0; a < 4; ++a) atomicAdd(g_nvals + 4 * int64_t(j) + a, g[a]);
  if (d > 0) {
    for (int corner = 0; corner < 8; ++corner) {
      int p[3] = {c[0] / 2, c[1] / 2, c[2] / 2};
      T weight = T(1.0);
      for (int axis = 0; axis < 3; ++axis) {
        if ((corner >> axis) & 1) p[axis] += 1;
        weight = weight * (T(1.0) - fabs(T(c[axis]) * T(0.5) - T(p[axis])));
      }
      if (weight > T(0)) {
        int32_t q = bh.find(basis_key(d - 1, p[0], p[1], p[2]));
        if (q >= 0)
          for (int a = 0; a < 4; ++a) atomicAdd(g_prev + 4 * (int64_t(q) - prev_off) + a, g[a] * weight);
      }
    }
  }
}

// ------------------------------------------------------------------ orchestration
template <class T>
void solve_backward(void* tape_ptr, const TreeData& tree, const DensityData<T>& D, const NormalData<T>& N,
                    const std::vector<int64_t>& level_offsets, const int64_t* all_keys, const HashMap& all_hash,
                    const Params& p, const T* g_coef, std::vector<DBuf<T>>& g_agg, T* g_average, T* g_nvals,
                    cudaStream_t s, EventMarks* marks) {
  SolveTape<T>& tp = *static_cast<SolveTape<T>*>(tape_ptr);
  auto mark = [&](int slot) {
    if (marks) marks->mark(slot, s);
  };
  const int finest = p.depth, base = p.base_depth;
  HashView bh = all_hash.view();
  auto keys_at = [&](int d) { return all_keys + level_offsets[d]; };
  auto count_at = [&](int d) { return level_offsets[d + 1] - level_offsets[d]; };
  ColumnIndex bcols;
  bcols.build(all_keys, level_offsets.back(), finest, s);
  const ColumnView bcv = bcols.view();

  std::vector<DBuf<T>> g_cum(finest + 1);
  std::vector<DBuf<double>> g_load(finest + 1);
  for (int d = 0; d <= finest; ++d) {
    g_cum[d].alloc(count_at(d), s);
    g_cum[d].zero();
    g_load[d].alloc(count_at(d), s);
    g_load[d].zero();
  }
  std::vector<DBuf<T>> g_pos(finest + 1), g_w(finest + 1);
  auto point_grads = [&](int d) {
    if (!tp.screened) return;
    const PointsData<T>& P = tp.points[d];
    g_pos[d].alloc(3 * P.m, s);
    g_pos[d].zero();
    g_w[d].alloc(P.m, s);
    g_w[d].zero();
  };

  const int top = tp.top;
  // The reverse sweeps' error codes merge into one device word, read once after the sliced
  // levels (one host synchronisation for all of them).
  DBuf<int> relax_error(1, s);
  relax_error.zero();
  RelaxDeferred deferred{relax_error.p, nullptr};
  // ---- sliced levels, finest first
  for (int d = top; d > base; --d) {
    const int64_t n = count_at(d);
    SlicedTape<T>& st = tp.sliced[d];
    if (!st.on) throw Error(1, "adjoint: missing tape of a sliced level");
    point_grads(d);
    DBuf<T> seed(n, s);
    axpy_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(g_coef + level_offsets[d], g_cum[d].p, n, seed.p);
    PSR_LAUNCH_CHECK();
    // The reverse sweep runs on the forward schedule in mirrored slice order over the
    // transposed operator; its increments are recorded at the forward positions.
    DBuf<T> sb(n + 4, s), M(n, s), mu(int64_t(p.iters) * n, s);
    sb.zero();
    M.zero();
    gather_seed_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(st.sched.perm.p, n, seed.p, sb.p);
    PSR_LAUNCH_CHECK();
    mark(kBwMirror);
    auto reverse_sweep = [&](auto s_tag, auto i_tag) {
      using S = decltype(s_tag);
      using I = decltype(i_tag);
      DBuf<S> tv(kSlots * n, s);
      transpose_values_kernel<S, I><<<blocks_for(n), kThreads, 0, s>>>(n, st.sched.skeys.p, st.sched.off.p,
                                                                       reinterpret_cast<const S*>(st.svals.p),
                                                                       reinterpret_cast<const I*>(st.sidx.p), tv.p);
      PSR_LAUNCH_CHECK();
      mark(kBwMirror);
      relax_strips_scheduled<S, T, I>(st.sched, tv.p, reinterpret_cast<const I*>(st.sidx.p), sb.p, M.p, p.iters, s,
                                      nullptr, mu.p, true, true, &deferred);
      mark(kBwSweep);
    };
    if (tp.mixed) {
      if (st.sched.wide)
        reverse_sweep(float(), int32_t());
      else
        reverse_sweep(float(), int16_t());
    } else {
      if (st.sched.wide)
        reverse_sweep(T(), int32_t());
      else
        reverse_sweep(T(), int16_t());
    }
    // M (forward key order): the rhs adjoint
    DBuf<T>& g_b = M;
    // operator, cross and screening adjoints
    const int res = 1 << d;
    DBuf<double> ctable(int64_t(res + 1) * 6, s);
    stiffness_table_kernel<<<blocks_for(res + 1), kThreads, 0, s>>>(d, d - 1, ctable.p);
    PSR_LAUNCH_CHECK();
    auto fused = [&](auto s_tag, auto i_tag) {
      using S = decltype(s_tag);
      using I = decltype(i_tag);
      LevelReverse<T, S, I> L;
      L.keys = keys_at(d);
      L.n = n;
      L.d = d;
      L.iters = p.iters;
      L.cv = bcv;
      L.coff = level_offsets[d - 1];
      L.g_b = g_b.p;
      L.inv = st.sched.inv.p;
      L.off = st.sched.off.p;
      L.sidx = reinterpret_cast<const I*>(st.sidx.p);
      L.xhist = st.hist.p;
      L.mu = mu.p;
      L.cross = true;
      L.ccols = st.ccols.p;
      L.cvals = st.cvals.p;
      L.ctable = ctable.p;
      L.cum_prev = tp.cum[d - 1].p;
      L.g_cum_prev = g_cum[d - 1].p;
      L.screened = tp.screened;
      DBuf<T> rA;
      if (tp.screened) {
        L.P = tp.points[d].view();
        L.g_pos = g_pos[d].p;
        L.g_w = g_w[d].p;
        rA.alloc(27 * n, s);
        L.row_gA = rA.p;
      }
      // per row: sorted key, permutation, index row, reverse and forward visit records, g_b,
      // the 27 operator adjoints, the cross tape row; the coarser cumulative adjoint read and
      // written
      KernelClock rows_clock(kClkLevelRowsReverse,
                             n * (8.0 + 4 + 32 * sizeof(I) + 2.0 * p.iters * sizeof(T) + sizeof(T) +
                                  (tp.screened ? 27 * sizeof(T) : 0) + kSlots * (4.0 + sizeof(T))) +
                                 2.0 * count_at(d - 1) * sizeof(T),
                             double(n), s);
      if (p.iters == 8 && L.ccols) {
        level_rows_reverse_kernel<T, I, 8><<<blocks_for(n, 128), 128, 0, s>>>(
            st.sched.skeys.p, n, st.sched.perm.p, L.off, L.sidx, L.xhist, L.mu, L.g_b, L.ccols, L.cvals,
            L.g_cum_prev, tp.screened ? rA.p : nullptr);
      } else {
        level_reverse_kernel<T, S, I, true, 0><<<blocks_for(n, 128), 128, 0, s>>>(L);
      }
      PSR_LAUNCH_CHECK();
      rows_clock.stop();
      if (tp.screened && tp.points[d].m) {
        const int64_t m = tp.points[d].m;
        // per point: position and weight read, their adjoints written; per row: g_b and the
        // 27 operator adjoints; the coarser cumulative solution
        KernelClock points_clock(kClkScreeningReverse,
                                 m * 8.0 * sizeof(T) + n * 28.0 * sizeof(T) + count_at(d - 1) * double(sizeof(T)),
                                 double(m), s);
        screening_points_reverse_kernel<T><<<blocks_for(m, 128), 128, 0, s>>>(
            L.P, m, d, bcv, level_offsets[d], g_b.p, rA.p, 27, tp.cum[d - 1].p, level_offsets[d - 1], g_pos[d].p,
            g_w[d].p);
        PSR_LAUNCH_CHECK();
      }
    };
    if (st.sched.wide)
      fused(T(), int32_t());
    else
      fused(T(), int16_t());
    // cumulative_d = x_d + P cumulative_{d-1}
    prolong_transpose_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(tp.pcol[d].p, tp.pval[d].p, n, g_cum[d].p,
                                                                   g_cum[d - 1].p);
    PSR_LAUNCH_CHECK();
    to_double_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(g_b.p, n, g_load[d].p);
    PSR_LAUNCH_CHECK();
    mark(kBwOperator);
  }
  throw_relax_error(read_scalar(relax_error.p, s));

  // ---- base multigrid
  {
    const int64_t nb = count_at(base);
    point_grads(base);
    std::vector<DBuf<T>> gx(base + 1), grhs(base + 1), gA(base + 1);
    for (int l = 0; l <= base; ++l) {
      const int64_t nl = count_at(l);
      gx[l].alloc(nl, s);
      gx[l].zero();
      grhs[l].alloc(nl, s);
      grhs[l].zero();
      gA[l].alloc(kSlots * nl, s);
      gA[l].zero();
    }
    axpy_kernel<T><<<blocks_for(nb), kThreads, 0, s>>>(g_coef + level_offsets[base], g_cum[base].p, nb, gx[base].p);
    PSR_LAUNCH_CHECK();
    std::vector<DBuf<T>> vt(base + 1);  // transposed level operators
    for (int l = 1; l <= base; ++l) {
      const int64_t nl = count_at(l);
      vt[l].alloc(kSlots * nl, s);
      if (nl) {
        transpose_slots_kernel<T><<<blocks_for(nl), kThreads, 0, s>>>(tp.mcols[l].p, tp.mvals[l].p, nl, vt[l].p);
        PSR_LAUNCH_CHECK();
      }
    }
    auto Rl = [&](int l) { return l == base ? tp.base_b.p : nullptr; };
    (void)Rl;
    const int cycles = p.base_v_cycles;
    int h = int(tp.relax_hist.size()) - 1;
    int rx = int(tp.resid_x.size()) - 1;
    DBuf<T> g_state(64, s), g_state_in(64, s);
    g_state.zero();
    g_state_in.zero();
    DBuf<T> root_work(64 * 64 * 2 + 65 * 64 * 3 + 64 * 64 + 5 * 64, s);
    DBuf<T> g_x0(count_at(0), s);
    for (int cycle = cycles - 1; cycle >= 0; --cycle) {
      for (int l = base; l >= 1; --l) {  // reverse of the upward pass
        const int64_t nl = count_at(l);
        relax_colors_adjoint<T>(keys_at(l), tp.mcols[l].p, tp.mvals[l].p, vt[l].p, tp.msched[l].rows.p,
                                tp.msched[l].off.p, p.iters, 0, tp.relax_hist[h--].p, nl, gx[l].p, grhs[l].p,
                                gA[l].p, s);
        // x_l += P x_{l-1}, then x_{l-1} = 0
        gx[l - 1].zero();
        prolong_transpose_kernel<T><<<blocks_for(nl), kThreads, 0, s>>>(tp.pcol[l].p, tp.pval[l].p, nl, gx[l].p,
                                                                       gx[l - 1].p);
        PSR_LAUNCH_CHECK();
      }
      // root solve
      {
        const int64_t n0 = count_at(0);
        g_x0.zero();
        root_reverse_kernel<T><<<1, 32, 0, s>>>(keys_at(0), int(n0), tp.mcols[0].p, tp.mvals[0].p,
                                                tp.root_b[cycle].p, tp.root_x0[cycle].p, tp.dc ? 1 : 0,
                                                p.cg_accuracy, base, cycle, gx[0].p, g_state.p, grhs[0].p, g_x0.p,
                                                g_state_in.p, gA[0].p, root_work.p);
        PSR_LAUNCH_CHECK();
        if (tp.dc) {
          PSR_CUDA(cudaMemcpyAsync(g_state.p, g_state_in.p, 64 * sizeof(T), cudaMemcpyDeviceToDevice, s));
          gx[0].zero();
        } else {
          PSR_CUDA(cudaMemcpyAsync(gx[0].p, g_x0.p, n0 * sizeof(T), cudaMemcpyDeviceToDevice, s));
        }
      }
      for (int l = 1; l <= base; ++l) {  // reverse of the downward pass
        const int64_t nl = count_at(l), nc = count_at(l - 1);
        gx[l - 1].zero();  // x_{l-1} = 0 after the restriction
        // rhs_{l-1} = P^T r_l
        DBuf<T> g_r(nl, s);
        g_r.zero();
        prolong_apply_kernel<T, T><<<blocks_for(nl), kThreads, 0, s>>>(tp.pcol[l].p, tp.pval[l].p, nl, grhs[l - 1].p,
                                                                        g_r.p);
        PSR_LAUNCH_CHECK();
        grhs[l - 1].zero();
        (void)nc;
        residual_reverse_kernel<T><<<blocks_for(nl), kThreads, 0, s>>>(tp.mcols[l].p, tp.mvals[l].p,
                                                                       tp.resid_x[rx--].p, g_r.p, nl, grhs[l].p,
                                                                       gx[l].p, gA[l].p);
        PSR_LAUNCH_CHECK();
        relax_colors_adjoint<T>(keys_at(l), tp.mcols[l].p, tp.mvals[l].p, vt[l].p, tp.msched[l].rows.p,
                                tp.msched[l].off.p, p.iters, 1, tp.relax_hist[h--].p, nl, gx[l].p, grhs[l].p,
                                gA[l].p, s);
      }
    }
    // Galerkin products, coarsest first
    for (int l = 0; l < base; ++l) {
      const int64_t nf = count_at(l + 1);
      galerkin_reverse_kernel<T><<<blocks_for(27 * nf), kThreads, 0, s>>>(keys_at(l + 1), nf, tp.mcols[l + 1].p,
                                                                     tp.pcol[l + 1].p, tp.pval[l + 1].p, keys_at(l),
                                                                     tp.mcols[l].p, gA[l].p, gA[l + 1].p);
      PSR_LAUNCH_CHECK();
    }
    // screening of the base level (no cross operator)
    LevelReverse<T, T, int32_t> L;
    L.keys = keys_at(base);
    L.n = nb;
    L.d = base;
    L.iters = p.iters;
    L.cv = bcv;
    L.g_b = grhs[base].p;
    L.g_A = gA[base].p;
    L.cross = false;
    L.screened = tp.screened;
    if (tp.screened) {
      L.P = tp.points[base].view();
      L.g_pos = g_pos[base].p;
      L.g_w = g_w[base].p;
    }
    if (nb) {
      if (tp.screened && tp.points[base].m) {
        const int64_t m = tp.points[base].m;
        screening_points_reverse_kernel<T><<<blocks_for(m, 128), 128, 0, s>>>(
            L.P, m, base, bcv, level_offsets[base], grhs[base].p, gA[base].p, kSlots, nullptr, 0, g_pos[base].p,
            g_w[base].p);
        PSR_LAUNCH_CHECK();
      }
      to_double_kernel<T><<<blocks_for(nb), kThreads, 0, s>>>(grhs[base].p, nb, g_load[base].p);
      PSR_LAUNCH_CHECK();
    }
  }

  mark(kBwBase);
  // ---- point constraints -> density aggregates and the mean splat weight
  if (tp.screened) {
    for (int d = base; d <= top; ++d) {
      const PointsData<T>& P = tp.points[d];
      const int64_t m = P.m;
      if (!m) continue;
      points_reverse_kernel<T><<<blocks_for(m), kThreads, 0, s>>>(D.agg_keys[d].p, D.agg_values[d].p, m, d,
                                                                  T(p.point_weight), N.average.p, P.w.p, g_pos[d].p,
                                                                  g_w[d].p, g_agg[d].p, g_average);
      PSR_LAUNCH_CHECK();
    }
  }

  mark(kBwPoints);
  // ---- normal loads (normal_load_adjoint.py:123-161)
  {
    HashMap nhash;
    nhash.build(N.keys.p, N.count, s);
    HashView nh = nhash.view();
    auto stencil_t = [&](int test_d, int normal_d, const int64_t* nkeys, int64_t m, const double* g_test,
                         T* g_vals) {
      const int64_t nt = count_at(test_d);
      if (!m || !nt) return;
      int width = test_d < normal_d ? 6 : 4, first = test_d < normal_d ? -3 : -2;
      int res = 1 << test_d;
      DBuf<double> table(int64_t(res + 1) * width * 2, s);
      normal_table_kernel<<<blocks_for(res + 1), kThreads, 0, s>>>(test_d, normal_d, first, width, table.p);
      PSR_LAUNCH_CHECK();
      // per normal record: key, 3 value adjoints read and written; per test function: its adjoint
      KernelClock clock(kClkNormalStencilReverse, m * (8.0 + 6 * sizeof(T)) + nt * 8.0, double(m), s);
      // PSR_NORMAL_REVERSE=generic: the generic kernel for every window (test override: the
      // window kernels must give its result bit for bit)
      const char* mode = std::getenv("PSR_NORMAL_REVERSE");
      const bool generic = mode && mode[0] == 'g';
      if (!generic && test_d == normal_d && width == 4 && first == -2 && bcv.dense)
        normal_stencil_reverse_window_kernel<T, 4, 4, 0><<<blocks_for(m), kThreads, 0, s>>>(
            nkeys, m, test_d, bcv, level_offsets[test_d], g_test, table.p, first, g_vals);
      else if (!generic && test_d + 1 == normal_d && width == 6 && first == -3 && bcv.dense)
        normal_stencil_reverse_window_kernel<T, 6, 3, 1><<<blocks_for(m), kThreads, 0, s>>>(
            nkeys, m, test_d, bcv, level_offsets[test_d], g_test, table.p, first, g_vals);
      else if (!generic && test_d == normal_d + 1 && width == 4 && first == -2 && bcv.dense)
        normal_stencil_reverse_window_kernel<T, 4, 8, 2><<<blocks_for(m), kThreads, 0, s>>>(
            nkeys, m, test_d, bcv, level_offsets[test_d], g_test, table.p, first, g_vals);
      else
        normal_stencil_reverse_kernel<T><<<blocks_for(m), kThreads, 0, s>>>(
            nkeys, m, test_d, normal_d, bcv, level_offsets[test_d], g_test, table.p, width, first, g_vals);
      PSR_LAUNCH_CHECK();
    };
    // finer chain: loads[d] = same[d] + finer_d + parent[d], finer_{d-1} = child[d-1] + P^T finer_d
    std::vector<DBuf<double>> g_finer(finest + 1);
    for (int d = base; d <= finest; ++d) {
      const int64_t n = count_at(d);
      g_finer[d].alloc(n, s);
      PSR_CUDA(cudaMemcpyAsync(g_finer[d].p, g_load[d].p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      if (d > base && n) {
        DBuf<int32_t> pc;
        DBuf<T> pv;
        const int32_t* pcp = nullptr;
        const T* pvp = nullptr;
        if (d < int(tp.pcol.size()) && tp.pcol[d].p) {
          pcp = tp.pcol[d].p;
          pvp = tp.pval[d].p;
        } else {
          pc.alloc(8 * n, s);
          pv.alloc(8 * n, s);
          prolongation_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(keys_at(d), n, d, bh, level_offsets[d - 1], pc.p,
                                                                    pv.p);
          PSR_LAUNCH_CHECK();
          pcp = pc.p;
          pvp = pv.p;
        }
        prolong_apply_kernel<T, double><<<blocks_for(n), kThreads, 0, s>>>(pcp, pvp, n, g_finer[d - 1].p,
                                                                            g_finer[d].p);
        PSR_LAUNCH_CHECK();
      }
    }
    // stencils of the normal coefficients of each depth
    std::vector<DBuf<T>> g_prolonged(finest + 1);
    bool has_cumulative = false;
    std::vector<char> has_cum(finest + 1, 0);
    for (int d = 0; d <= finest; ++d) {
      has_cumulative = has_cumulative || (N.offsets[d + 1] - N.offsets[d]) > 0;
      has_cum[d] = has_cumulative;
    }
    for (int d = 0; d <= finest; ++d) {
      const int64_t nrec = N.offsets[d + 1] - N.offsets[d];
      const int64_t* nk = N.keys.p + N.offsets[d];
      T* gv = g_nvals + 4 * N.offsets[d];
      if (d >= base) {
        stencil_t(d, d, nk, nrec, g_load[d].p, gv);
        if (d > base) stencil_t(d - 1, d, nk, nrec, g_finer[d - 1].p, gv);
      }
      if (d < finest) {
        g_prolonged[d].alloc(4 * count_at(d), s);
        g_prolonged[d].zero();
        if (d >= base && has_cum[d])
          stencil_t(d + 1, d, keys_at(d), count_at(d), g_load[d + 1].p, g_prolonged[d].p);
      }
    }
    for (int d = finest - 1; d >= 0; --d) {
      const int64_t n = count_at(d);
      if (!n) continue;
      prolong_normals_reverse_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(
          keys_at(d), n, d, nh, bh, d > 0 ? level_offsets[d - 1] : 0, g_prolonged[d].p, g_nvals,
          d > 0 ? g_prolonged[d - 1].p : nullptr);
      PSR_LAUNCH_CHECK();
    }
  }
  mark(kBwNormalLoads);
}

template void solve_backward<float>(void*, const TreeData&, const DensityData<float>&, const NormalData<float>&,
                                    const std::vector<int64_t>&, const int64_t*, const HashMap&, const Params&,
                                    const float*, std::vector<DBuf<float>>&, float*, float*, cudaStream_t,
                                    EventMarks*);
template void solve_backward<double>(void*, const TreeData&, const DensityData<double>&, const NormalData<double>&,
                                     const std::vector<int64_t>&, const int64_t*, const HashMap&, const Params&,
                                     const double*, std::vector<DBuf<double>>&, double*, double*, cudaStream_t,
                                     EventMarks*);
