// A4: sparse tree completion (warp-psr tree.py:152-201).  Integer only; keys must match
// the reference bit for bit.  Brood keys are sorted in a compact form: at level d every
// candidate brood coordinate lies in [-2^d, 2^d), so (c + 2^d) packs into d+1 bits per
// axis with the same lexicographic order as the reference's 20-bit signed tree keys.
#include "psr_internal.cuh"

namespace psr {

__device__ __forceinline__ uint64_t pack_brood(const int c[3], int d) {
  int n = 1 << d, D = d + 1;
  return (uint64_t(c[0] + n) << (2 * D)) | (uint64_t(c[1] + n) << D) | uint64_t(c[2] + n);
}
__device__ __forceinline__ void unpack_brood(uint64_t k, int d, int c[3]) {
  int n = 1 << d, D = d + 1;
  uint64_t mask = (uint64_t(1) << D) - 1;
  c[0] = int((k >> (2 * D)) & mask) - n;
  c[1] = int((k >> D) & mask) - n;
  c[2] = int(k & mask) - n;
}

// tree.py:41-50 — broods of this level's normal records with nonzero coefficients.
template <class T>
__global__ void seed_kernel(const int64_t* nkeys, const T* nvals, int64_t count, int d, uint64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  const T* v = nvals + 4 * i;
  T l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
  uint64_t key = uint64_t(1) << (3 * (d + 1));
  if (double(l2) > 0.0) {
    int c[3];
    key_coords(nkeys[i], c);
    int p[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
    key = pack_brood(p, d);
  }
  out[i] = key;
}

// tree.py:30-34 — the full-depth coarse region, starting at -1.
__global__ void coarse_kernel(int d, int count, uint64_t* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count * count * count) return;
  int c[3] = {i / (count * count) - 1, (i / count) % count - 1, i % count - 1};
  out[i] = pack_brood(c, d);
}

// tree.py:52-64 — (2r+1)^3 broods around the parent of every source node.
__global__ void support_kernel(const int64_t* src, int64_t count, int radius, int d, uint64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  int w = 2 * radius + 1;
  int c[3];
  tree_coords(src[i], c);
  int p[3] = {c[0] >> 1, c[1] >> 1, c[2] >> 1};
  int n = 1 << d;
  uint64_t sentinel = uint64_t(1) << (3 * (d + 1));
  for (int j = 0; j < w * w * w; ++j) {
    int q[3] = {p[0] + j / (w * w) - radius, p[1] + (j / w) % w - radius, p[2] + j % w - radius};
    bool ok = dmin(q[0], dmin(q[1], q[2])) >= -n && dmax(q[0], dmax(q[1], q[2])) < n;
    out[i * w * w * w + j] = ok ? pack_brood(q, d) : sentinel;
  }
}

template <class K>
__global__ void unique_heads_kernel(const K* keys, int64_t n, uint64_t sentinel, int32_t* heads) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  heads[i] = uint64_t(keys[i]) < sentinel && (i == 0 || keys[i] != keys[i - 1]);
}

template <class K>
__global__ void compact_kernel(const K* keys, const int32_t* heads, const int32_t* prefix, int64_t n,
                               uint64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n && heads[i]) out[prefix[i] - 1] = uint64_t(keys[i]);
}

// 64-bit keys below 2^32 narrowed to 32 bits for the sort.
__global__ void narrow_keys_kernel(const uint64_t* keys, int64_t n, uint32_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = uint32_t(keys[i]);
}

__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t* a, int64_t n, uint64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// tree.py:78-97 — eight children per sorted unique brood, written directly in sorted order.
__global__ void expand_kernel(const uint64_t* broods, int64_t n, int d, int64_t* children, int32_t* basis_mark) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int D = d + 1;
  uint64_t key = broods[i];
  uint64_t x = (key >> (2 * D)) << (2 * D);
  uint64_t xy = (key >> D) << D;
  int64_t x0 = lower_bound_u64(broods, n, x), x1 = lower_bound_u64(broods, n, x + (uint64_t(1) << (2 * D)));
  int64_t xy0 = lower_bound_u64(broods, n, xy), xy1 = lower_bound_u64(broods, n, xy + (uint64_t(1) << D));
  int c[3];
  unpack_brood(key, d, c);
  int res = 1 << d;
  for (int k = 0; k < 8; ++k) {
    int ox = (k >> 2) & 1, oy = (k >> 1) & 1, oz = k & 1;
    int64_t dest = 8 * x0 + 4 * ox * (x1 - x0) + 4 * (xy0 - x0) + 2 * oy * (xy1 - xy0) + 2 * (i - xy0) + oz;
    int q[3] = {2 * c[0] + ox, 2 * c[1] + oy, 2 * c[2] + oz};
    children[dest] = tree_key(q[0], q[1], q[2]);
    basis_mark[dest] = dmin(q[0], dmin(q[1], q[2])) >= 0 && dmax(q[0], dmax(q[1], q[2])) <= res;
  }
}

__global__ void basis_fill_kernel(const int64_t* children, const int32_t* mark, const int32_t* prefix, int64_t n,
                                  int d, int64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n || !mark[i]) return;
  int c[3];
  tree_coords(children[i], c);
  out[prefix[i] - 1] = basis_key(d, c[0], c[1], c[2]);
}

__global__ void parent_tree_keys_kernel(const int64_t* src, int64_t n, uint64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  tree_coords(src[i], c);
  out[i] = uint64_t(tree_key(c[0] >> 1, c[1] >> 1, c[2] >> 1));
}

__global__ void u64_to_i64_kernel(const uint64_t* in, int64_t n, int64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) out[i] = int64_t(in[i]);
}

__global__ void broods_to_tree_keys_kernel(const uint64_t* in, int64_t n, int d, int64_t* out) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  int c[3];
  unpack_brood(in[i], d, c);
  out[i] = tree_key(c[0], c[1], c[2]);
}

// Sort + unique of n keys below `sentinel`; returns the count and the unique keys.
static int64_t sort_unique(DBuf<uint64_t>& keys, int64_t n, int end_bit, uint64_t sentinel, DBuf<uint64_t>& out,
                           cudaStream_t s) {
  if (n == 0) {
    out.alloc(0, s);
    return 0;
  }
  // Keys of at most 32 bits (depth <= 9 here) are sorted as 32-bit keys: half the data
  // through every pass for one narrowing copy.  Same order, same unique keys.
  DBuf<int32_t> heads(n, s), prefix(n, s);
  int64_t u = 0;
  auto run = [&](auto key_tag, const decltype(key_tag)* in) {
    using K = decltype(key_tag);
    DBuf<K> sorted(n, s);
    size_t temp = 0;
    PSR_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, temp, in, sorted.p, n, 0, end_bit, s));
    {
      DBuf<char> t(int64_t(temp), s);
      PSR_CUDA(cub::DeviceRadixSort::SortKeys(t.p, temp, in, sorted.p, n, 0, end_bit, s));
    }
    unique_heads_kernel<K><<<blocks_for(n), kThreads, 0, s>>>(sorted.p, n, sentinel, heads.p);
    PSR_LAUNCH_CHECK();
    inclusive_sum(heads.p, prefix.p, n, s);
    u = read_scalar(prefix.p + n - 1, s);
    out.alloc(u, s);
    compact_kernel<K><<<blocks_for(n), kThreads, 0, s>>>(sorted.p, heads.p, prefix.p, n, out.p);
    PSR_LAUNCH_CHECK();
  };
  if (end_bit <= 32) {
    DBuf<uint32_t> narrow(n, s);
    narrow_keys_kernel<<<blocks_for(n), kThreads, 0, s>>>(keys.p, n, narrow.p);
    PSR_LAUNCH_CHECK();
    run(uint32_t(), narrow.p);
  } else {
    run(uint64_t(), keys.p);
  }
  return u;
}

template <class T>
TreeData build_tree(const NormalData<T>& N, int depth, int full_depth, int base_depth, cudaStream_t s) {
  TreeData tree;
  tree.support.resize(depth + 1);
  tree.basis.resize(depth + 1);
  tree.support_count.assign(depth + 1, 0);
  tree.basis_count.assign(depth + 1, 0);
  DBuf<int64_t> broods;  // tree keys of the previous (finer) level's broods = this level's refined nodes
  int64_t nbroods = 0;
  DBuf<int64_t> requests;
  int64_t nrequests = 0;
  bool have_requests = false;
  for (int d = depth; d >= 0; --d) {
    // tree.py:171-182
    const int64_t* parents = broods.p;
    int64_t nparents = nbroods;
    DBuf<int64_t> req_storage;
    const int64_t* req = nullptr;
    if (d > base_depth || !have_requests) {
      req = parents;
      nrequests = nparents;
      have_requests = true;
    } else {
      DBuf<uint64_t> pk(nrequests, s), upk;
      if (nrequests) {
        parent_tree_keys_kernel<<<blocks_for(nrequests), kThreads, 0, s>>>(requests.p, nrequests, pk.p);
        PSR_LAUNCH_CHECK();
      }
      int64_t u = sort_unique(pk, nrequests, 62, ~uint64_t(0), upk, s);
      req_storage.alloc(u, s);
      if (u) {
        u64_to_i64_kernel<<<blocks_for(u), kThreads, 0, s>>>(upk.p, u, req_storage.p);
        PSR_LAUNCH_CHECK();
      }
      nrequests = u;
      req = req_storage.p;
    }
    int64_t nseed = N.offsets[d + 1] - N.offsets[d];
    int cc = d <= full_depth ? (d == 0 ? 2 : (1 << (d - 1)) + 2) : 0;
    int64_t nc = int64_t(cc) * cc * cc;
    int64_t total = nseed + nc + 27 * nrequests + nparents;
    DBuf<uint64_t> cand(total, s);
    int64_t off = 0;
    if (nseed) {
      seed_kernel<T><<<blocks_for(nseed), kThreads, 0, s>>>(N.keys.p + N.offsets[d], N.values.p + 4 * N.offsets[d],
                                                            nseed, d, cand.p);
      PSR_LAUNCH_CHECK();
    }
    off += nseed;
    if (nc) {
      coarse_kernel<<<blocks_for(nc), kThreads, 0, s>>>(d, cc, cand.p + off);
      PSR_LAUNCH_CHECK();
    }
    off += nc;
    if (nrequests) {
      support_kernel<<<blocks_for(nrequests), kThreads, 0, s>>>(req, nrequests, 1, d, cand.p + off);
      PSR_LAUNCH_CHECK();
    }
    off += 27 * nrequests;
    if (nparents) {
      support_kernel<<<blocks_for(nparents), kThreads, 0, s>>>(parents, nparents, 0, d, cand.p + off);
      PSR_LAUNCH_CHECK();
    }
    // Keep the refined-node requests alive for the next (coarser) level.
    DBuf<int64_t> next_requests;
    if (d <= base_depth || true) {
      next_requests.alloc(nrequests, s);
      if (nrequests)
        PSR_CUDA(cudaMemcpyAsync(next_requests.p, req, nrequests * sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    }
    uint64_t sentinel = uint64_t(1) << (3 * (d + 1));
    DBuf<uint64_t> ub;
    int64_t u = sort_unique(cand, total, 3 * (d + 1) + 1, sentinel, ub, s);
    // tree.py:196-199: expand into sorted children, compact the basis.
    int64_t nch = 8 * u;
    tree.support[d].alloc(nch, s);
    tree.support_count[d] = nch;
    DBuf<int32_t> mark(nch, s), prefix(nch, s);
    if (u) {
      expand_kernel<<<blocks_for(u), kThreads, 0, s>>>(ub.p, u, d, tree.support[d].p, mark.p);
      PSR_LAUNCH_CHECK();
      inclusive_sum(mark.p, prefix.p, nch, s);
      int64_t nb = read_scalar(prefix.p + nch - 1, s);
      tree.basis[d].alloc(nb, s);
      tree.basis_count[d] = nb;
      basis_fill_kernel<<<blocks_for(nch), kThreads, 0, s>>>(tree.support[d].p, mark.p, prefix.p, nch, d,
                                                             tree.basis[d].p);
      PSR_LAUNCH_CHECK();
    }
    DBuf<int64_t> nb_keys(u, s);
    if (u) {
      broods_to_tree_keys_kernel<<<blocks_for(u), kThreads, 0, s>>>(ub.p, u, d, nb_keys.p);
      PSR_LAUNCH_CHECK();
    }
    requests = std::move(next_requests);
    broods = std::move(nb_keys);
    nbroods = u;
  }
  return tree;
}

template TreeData build_tree<float>(const NormalData<float>&, int, int, int, cudaStream_t);
template TreeData build_tree<double>(const NormalData<double>&, int, int, int, cudaStream_t);

}  // namespace psr
