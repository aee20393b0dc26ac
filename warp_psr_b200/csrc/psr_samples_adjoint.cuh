// A13: reverse pass of the sample, density and normal stages (warp-psr splat_adjoint.py:105-188,
// sample_adjoint.py:62-102).  Included at the end of psr_samples.cu.  Every layout (groups,
// records, unique keys, splat depths) is the forward's; only continuous values are reversed.

// d b / d u of the degree-2 B-spline pieces of quadratic().
__device__ __forceinline__ void quadratic_grad(double x, double g[3]) {
  g[0] = -(1.0 - x);
  g[1] = 1.0 - 2.0 * x;
  g[2] = x;
}

// Normal splat (normal_splat_kernel) and the weighted average (average_contrib_kernel /
// average_finish_kernel) reversed, one group per thread in first-index order.
template <class T>
__global__ void normal_splat_reverse_kernel(const int32_t* order, int64_t n, const T* sums, const T* nsums,
                                            const T* weights, const T* dw, int minimum, int maximum,
                                            const int32_t* record_slot, const T* g_nvals, const T* average,
                                            const T* g_average, T* g_sums, T* g_nsums, T* g_dw) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const int64_t src = order[i];
  const T w = weights[src];
  T nm[3] = {nsums[3 * src] / w, nsums[3 * src + 1] / w, nsums[3 * src + 2] / w};
  const T length = sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
  if (!(length > T(0))) return;
  T unit[3], nmw[3];
  for (int a = 0; a < 3; ++a) {
    unit[a] = nm[a] / length;
    nmw[a] = nm[a] / length * w;
  }
  // average contributions (raw depth * w, splat weight * w, w)
  T g_raw = T(0), g_sw = T(0);
  if (average[2] > T(0)) {
    g_raw = g_raw + g_average[0] / average[2] * w;
    g_sw = g_sw + g_average[1] / average[2] * w;
  }
  const T p[3] = {sums[3 * src] / w, sums[3 * src + 1] / w, sums[3 * src + 2] / w};
  const T raw = dw[2 * src];
  const T depth = dmin(dmax(raw, T(minimum)), T(maximum));
  int top = int(ceil(depth));
  T dx = T(1.0) - (T(top) - depth);
  bool free_dx = true;
  if (top <= minimum) {
    top = minimum;
    dx = T(1.0);
    free_dx = false;
  }
  if (top > maximum) {
    top = maximum;
    dx = T(1.0);
    free_dx = false;
  }
  const int nn = 1 << top;
  const T h = T(1.0) / T(nn);
  const int c[3] = {ceil_cell(p[0], nn), ceil_cell(p[1], nn), ceil_cell(p[2], nn)};
  double b[3][3], bg[3][3];
  for (int a = 0; a < 3; ++a) {
    const double u = double((p[a] - T(c[a]) * h) / h);
    quadratic(u, b[a]);
    quadratic_grad(u, bg[a]);
  }
  const bool second = fabs(1.0 - double(dx)) > 1e-06;
  const T sw = dw[2 * src + 1];
  const T inv_h3 = T(1) / (h * h * h);
  T g_nmw[3] = {T(0), T(0), T(0)}, g_p[3] = {T(0), T(0), T(0)}, g_dx = T(0);
  for (int k = 0; k < 54; ++k) {
    if (k >= 27 && !second) break;
    const int32_t slot = record_slot[54 * i + k];
    if (slot < 0) continue;
    const T fraction = k < 27 ? dx : T(1.0) - dx;
    const int q = k % 27, x = q / 9, y = q / 3 % 3, z = q % 3;
    const T bw = T(b[0][x] * b[1][y] * b[2][z]);
    // records are negated when reduced (normals.py:106-110,219-221)
    const T gr[3] = {-g_nvals[4 * int64_t(slot)], -g_nvals[4 * int64_t(slot) + 1], -g_nvals[4 * int64_t(slot) + 2]};
    const T G = gr[0] * nmw[0] + gr[1] * nmw[1] + gr[2] * nmw[2];
    for (int a = 0; a < 3; ++a) g_nmw[a] = g_nmw[a] + gr[a] * sw * inv_h3 * fraction * bw;
    g_sw = g_sw + G * inv_h3 * fraction * bw;
    const T gfrac = G * sw * inv_h3 * bw;
    g_dx = g_dx + (k < 27 ? gfrac : -gfrac);
    const T gbw = G * sw * inv_h3 * fraction;
    const double db[3] = {bg[0][x] * b[1][y] * b[2][z], b[0][x] * bg[1][y] * b[2][z], b[0][x] * b[1][y] * bg[2][z]};
    for (int a = 0; a < 3; ++a) g_p[a] = g_p[a] + gbw * T(db[a]) / h;
  }
  if (free_dx && raw > T(minimum) && raw < T(maximum)) g_raw = g_raw + g_dx;
  // nmw = u / |u| * w with u = nsums / w
  const T ug = unit[0] * g_nmw[0] + unit[1] * g_nmw[1] + unit[2] * g_nmw[2];
  for (int a = 0; a < 3; ++a) {
    g_nsums[3 * src + a] = g_nsums[3 * src + a] + (g_nmw[a] - unit[a] * ug) / length;
    g_sums[3 * src + a] = g_sums[3 * src + a] + g_p[a] / w;
  }
  g_dw[2 * src] = g_dw[2 * src] + g_raw;
  g_dw[2 * src + 1] = g_dw[2 * src + 1] + g_sw;
}

// depths_kernel reversed: density adjoints at the selected depth (and the finer one when the
// depth was interpolated).
template <class T>
__global__ void depths_reverse_kernel(const T* dens, int64_t G, int kernel_depth, T target, const T* g_dw, T* g_dens) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= G) return;
  const int stride = kernel_depth + 1;
  int d = kernel_depth;
  T density = dens[i * stride + d];
  const T graw = g_dw[2 * i], gsw = g_dw[2 * i + 1];
  if (density >= target) {
    const T h = T(1.0) / T(1 << d);
    T g = graw / (density * T(2.0 * log(2.0)));
    g = g - gsw * h * h / (density * density);
    g_dens[i * stride + d] = g_dens[i * stride + d] + g;
    return;
  }
  T fine = density;
  while (density < target && d > 0) {
    fine = density;
    d -= 1;
    density = dens[i * stride + d];
  }
  const T h = T(1.0) / T(1 << d);
  const T la = T(log(double(density / target))), lb = T(log(double(density / fine)));
  T gD = graw * (lb - la) / (density * lb * lb) - gsw * h * h / (density * density);
  T gF = graw * la / (lb * lb * fine);
  g_dens[i * stride + d] = g_dens[i * stride + d] + gD;
  if (d + 1 <= kernel_depth) g_dens[i * stride + d + 1] = g_dens[i * stride + d + 1] + gF;
}

// density_eval_kernel reversed: level-value adjoints (atomic) and the centroid's position.
template <class T>
__global__ void density_eval_reverse_kernel(HashView h, const T* lvals, const T* sums, const T* weights, int64_t G,
                                            int d, int stride, const T* g_dens, T* g_lvals, T* g_sums) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= G) return;
  const T gv = g_dens[i * stride + d];
  if (gv == T(0)) return;
  const T w = weights[i];
  const T p[3] = {sums[3 * i] / w, sums[3 * i + 1] / w, sums[3 * i + 2] / w};
  const int n = 1 << d;
  const int c[3] = {ceil_cell(p[0], n), ceil_cell(p[1], n), ceil_cell(p[2], n)};
  const T hh = T(1.0) / T(n);
  double b[3][3], bg[3][3];
  for (int a = 0; a < 3; ++a) {
    const double u = double((p[a] - T(c[a]) * hh) / hh);
    quadratic(u, b[a]);
    quadratic_grad(u, bg[a]);
  }
  T gp[3] = {T(0), T(0), T(0)};
  for (int k = 0; k < 27; ++k) {
    const int x = k / 9, y = k / 3 % 3, z = k % 3;
    const int t[3] = {c[0] + x - 1, c[1] + y - 1, c[2] + z - 1};
    if (dmin(t[0], dmin(t[1], t[2])) < 0 || dmax(t[0], dmax(t[1], t[2])) >= n) continue;
    const int32_t idx = h.find(basis_key(d, t[0], t[1], t[2]));
    if (idx < 0) continue;
    atomicAdd(g_lvals + idx, gv * T(b[0][x] * b[1][y] * b[2][z]));
    const double lv = double(lvals[idx]);
    gp[0] = gp[0] + gv * T(bg[0][x] * b[1][y] * b[2][z] * lv) / hh;
    gp[1] = gp[1] + gv * T(b[0][x] * bg[1][y] * b[2][z] * lv) / hh;
    gp[2] = gp[2] + gv * T(b[0][x] * b[1][y] * bg[2][z] * lv) / hh;
  }
  for (int a = 0; a < 3; ++a) g_sums[3 * i + a] = g_sums[3 * i + a] + gp[a] / w;
}

// density_splat_kernel reversed: one aggregate per thread (records 27 i + k, i in morton order).
template <class T>
__global__ void density_splat_reverse_kernel(const int64_t* keys, const T* values, const int32_t* order, int64_t m,
                                             int d, T scale, const int32_t* slot, const T* g_lvals, T* g_values) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= m) return;
  const int64_t j = order[i];
  int c[3];
  key_coords(keys[j], c);
  const T* v = values + 4 * j;
  const int n = 1 << d;
  const T p[3] = {v[0] / v[3], v[1] / v[3], v[2] / v[3]};
  const T h = T(1.0) / T(n);
  double b[3][3], bg[3][3];
  for (int a = 0; a < 3; ++a) {
    const double u = double((p[a] - T(c[a]) * h) / h);
    quadratic(u, b[a]);
    quadratic_grad(u, bg[a]);
  }
  const T weight = v[3] * scale;
  T gweight = T(0), gp[3] = {T(0), T(0), T(0)};
  for (int k = 0; k < 27; ++k) {
    const int32_t u = slot[27 * i + k];
    if (u < 0) continue;
    const T g = g_lvals[u];
    if (g == T(0)) continue;
    const int x = k / 9, y = k / 3 % 3, z = k % 3;
    gweight = gweight + g * T(b[0][x] * b[1][y] * b[2][z]);
    gp[0] = gp[0] + g * T(double(weight) * bg[0][x] * b[1][y] * b[2][z]) / h;
    gp[1] = gp[1] + g * T(double(weight) * b[0][x] * bg[1][y] * b[2][z]) / h;
    gp[2] = gp[2] + g * T(double(weight) * b[0][x] * b[1][y] * bg[2][z]) / h;
  }
  T* gv = g_values + 4 * j;
  for (int a = 0; a < 3; ++a) {
    gv[a] = gv[a] + gp[a] / v[3];
    gv[3] = gv[3] - gp[a] * p[a] / v[3];
  }
  gv[3] = gv[3] + gweight * scale;
}

// Aggregates: a parent's adjoint reaches each of its children.
template <class T>
__global__ void parent_broadcast_kernel(const int32_t* parent_of, int64_t n, const T* g_parent, T* g_child) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const int32_t q = parent_of[i];
  for (int a = 0; a < 4; ++a) g_child[4 * i + a] = g_child[4 * i + a] + g_parent[4 * int64_t(q) + a];
}

template <class T>
__global__ void leaf_reverse_kernel(const T* g_leaf, int64_t G, T* g_sums) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= G) return;
  for (int a = 0; a < 3; ++a) g_sums[3 * i + a] = g_sums[3 * i + a] + g_leaf[4 * i + a];
}

// classify_kernel + groups_kernel reversed for every input point; the transform adjoint
// (sum of q-adjoint * point for the scale, sum of q-adjoints for the translations) is
// reduced per block and added atomically in float64.
template <class T>
__global__ void samples_reverse_kernel(const T* __restrict__ pos, const T* __restrict__ nrm, int64_t n,
                                       const T* transform, const int32_t* input_group, const T* g_sums,
                                       const T* g_nsums, T* g_pos, T* g_nrm, double* g_tr) {
  __shared__ double red[4][kThreads];
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < n) {
    T gp[3] = {T(0), T(0), T(0)}, gn[3] = {T(0), T(0), T(0)};
    const int32_t g = input_group[i];
    if (g >= 0) {
      const T inv = transform[0], ns = transform[4];
      const T* p = pos + 3 * i;
      const T gq[3] = {g_sums[3 * g], g_sums[3 * g + 1], g_sums[3 * g + 2]};
      gp[1] = gq[0] * inv;
      gp[2] = gq[1] * inv;
      gp[0] = gq[2] * inv;
      acc[0] = double(gq[0]) * double(p[1]) + double(gq[1]) * double(p[2]) + double(gq[2]) * double(p[0]);
      for (int a = 0; a < 3; ++a) acc[1 + a] = double(gq[a]);
      const T* m = nrm + 3 * i;
      const T mm[3] = {m[1] * ns, m[2] * ns, m[0] * ns};
      const T len = sqrt(mm[0] * mm[0] + mm[1] * mm[1] + mm[2] * mm[2]);
      const T u[3] = {mm[0] / len, mm[1] / len, mm[2] / len};
      const T gu[3] = {g_nsums[3 * g], g_nsums[3 * g + 1], g_nsums[3 * g + 2]};
      const T ug = u[0] * gu[0] + u[1] * gu[1] + u[2] * gu[2];
      T gmm[3];
      for (int a = 0; a < 3; ++a) gmm[a] = (gu[a] - u[a] * ug) / len;
      gn[1] = gmm[0] * ns;
      gn[2] = gmm[1] * ns;
      gn[0] = gmm[2] * ns;
    }
    for (int a = 0; a < 3; ++a) {
      g_pos[3 * i + a] = gp[a];
      g_nrm[3 * i + a] = gn[a];
    }
  }
  for (int a = 0; a < 4; ++a) red[a][threadIdx.x] = acc[a];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int a = 0; a < 4; ++a) red[a][threadIdx.x] += red[a][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int a = 0; a < 4; ++a)
      if (red[a][0] != 0.0) atomicAdd(g_tr + a, red[a][0]);
}

// transform_kernel reversed onto the bounding-box extremes (their lowest-index owners).
template <class T>
__global__ void transform_reverse_kernel(const T* bounds, const int32_t* owner, T scale, const T* transform,
                                         const double* g_tr_acc, const T* g_transform, T* g_pos) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const T* lo = bounds;
  const T* hi = bounds + 3;
  const T e[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  const T width = dmax(e[0], dmax(e[1], e[2])) * scale;
  const T inv = transform[0];
  double g_inv = g_tr_acc[0] + (g_transform ? double(g_transform[0]) : 0.0);
  double g_lo[3] = {0, 0, 0}, g_hi[3] = {0, 0, 0}, g_width = 0;
  for (int a = 0; a < 3; ++a) {
    const int axis = (a + 1) % 3;
    const double g_t = g_tr_acc[1 + a] + (g_transform ? double(g_transform[1 + a]) : 0.0);
    const T origin = (hi[axis] + lo[axis]) / T(2.0) - width / T(2.0);
    const double g_origin = -g_t * double(inv);
    g_inv += -g_t * double(origin);
    g_hi[axis] += g_origin / 2;
    g_lo[axis] += g_origin / 2;
    g_width += -g_origin / 2;
  }
  g_width += -g_inv / (double(width) * double(width));
  // width = max extent * scale (dmax keeps the first argument on ties)
  const int a12 = e[1] >= e[2] ? 1 : 2;
  const int A = e[0] >= e[a12] ? 0 : a12;
  g_hi[A] += g_width * double(scale);
  g_lo[A] -= g_width * double(scale);
  for (int a = 0; a < 3; ++a) {
    g_pos[3 * int64_t(owner[a]) + a] = g_pos[3 * int64_t(owner[a]) + a] + T(g_lo[a]);
    g_pos[3 * int64_t(owner[3 + a]) + a] = g_pos[3 * int64_t(owner[3 + a]) + a] + T(g_hi[a]);
  }
}

template <class T>
void samples_backward(const SampleGroups<T>& G, const DensityData<T>& D, const NormalData<T>& N, int depth,
                      int kernel_depth, int base_depth, double samples_per_node, double scale,
                      std::vector<DBuf<T>>& g_agg, const T* g_average, const T* g_nvals, T* g_sums,
                      const T* g_transform, const T* pos, const T* nrm, int64_t n, T* g_pos, T* g_nrm,
                      cudaStream_t s) {
  const int64_t count = G.count;
  DBuf<T> g_nsums(3 * count, s), g_dw(2 * count, s);
  g_nsums.zero();
  g_dw.zero();
  // normal splat and average
  normal_splat_reverse_kernel<T><<<blocks_for(count), kThreads, 0, s>>>(
      N.group_order.p, count, G.sums.p, G.normal_sums.p, G.weights.p, D.dw.p, base_depth, depth, N.record_slot.p,
      g_nvals, N.average.p, g_average, g_sums, g_nsums.p, g_dw.p);
  PSR_LAUNCH_CHECK();
  // splat depths -> densities at the centroids
  const int stride = kernel_depth + 1;
  DBuf<T> g_dens(count * stride, s);
  g_dens.zero();
  depths_reverse_kernel<T><<<blocks_for(count), kThreads, 0, s>>>(D.densities.p, count, kernel_depth,
                                                                  T(samples_per_node), g_dw.p, g_dens.p);
  PSR_LAUNCH_CHECK();
  // densities -> level values -> splat records -> aggregates
  for (int d = 0; d <= kernel_depth; ++d) {
    const int64_t u = D.level_hash[d].count;
    DBuf<T> g_lvals(u, s);
    g_lvals.zero();
    density_eval_reverse_kernel<T><<<blocks_for(count), kThreads, 0, s>>>(D.level_hash[d].view(), D.level_values[d].p,
                                                                          G.sums.p, G.weights.p, count, d, stride,
                                                                          g_dens.p, g_lvals.p, g_sums);
    PSR_LAUNCH_CHECK();
    const int64_t m = D.agg_count[d];
    if (m) {
      density_splat_reverse_kernel<T><<<blocks_for(m), kThreads, 0, s>>>(D.agg_keys[d].p, D.agg_values[d].p,
                                                                         D.splat_order[d].p, m, d, D.scale,
                                                                         D.splat_slot[d].p, g_lvals.p, g_agg[d].p);
      PSR_LAUNCH_CHECK();
    }
  }
  for (int d = 1; d <= depth; ++d) {
    const int64_t m = D.agg_count[d];
    if (!m) continue;
    parent_broadcast_kernel<T><<<blocks_for(m), kThreads, 0, s>>>(D.parent_of[d].p, m, g_agg[d - 1].p, g_agg[d].p);
    PSR_LAUNCH_CHECK();
  }
  leaf_reverse_kernel<T><<<blocks_for(count), kThreads, 0, s>>>(g_agg[depth].p, count, g_sums);
  PSR_LAUNCH_CHECK();
  // inputs
  DBuf<double> g_tr(4, s);
  g_tr.zero();
  samples_reverse_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(pos, nrm, n, G.transform.p, G.input_group.p, g_sums,
                                                               g_nsums.p, g_pos, g_nrm, g_tr.p);
  PSR_LAUNCH_CHECK();
  transform_reverse_kernel<T><<<1, 32, 0, s>>>(G.bounds.p, G.bound_owner.p, T(scale), G.transform.p, g_tr.p,
                                               g_transform, g_pos);
  PSR_LAUNCH_CHECK();
}

template void samples_backward<float>(const SampleGroups<float>&, const DensityData<float>&, const NormalData<float>&,
                                      int, int, int, double, double, std::vector<DBuf<float>>&, const float*,
                                      const float*, float*, const float*, const float*, const float*, int64_t, float*,
                                      float*, cudaStream_t);
template void samples_backward<double>(const SampleGroups<double>&, const DensityData<double>&,
                                       const NormalData<double>&, int, int, int, double, double,
                                       std::vector<DBuf<double>>&, const double*, const double*, double*,
                                       const double*, const double*, const double*, int64_t, double*, double*,
                                       cudaStream_t);
