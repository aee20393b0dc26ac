// Sparse marching cubes over a regular grid of field values: the consumer of the field that
// warp-psr ships as extract_isosurface / extract_mesh (meshing.py:150-346).
//
// Grid: nx x ny x nz nodes spanning [lower, upper] in model space, node (i, j, k) at
// min(max(lower + step * (i, j, k), lower), upper), step = (upper - lower) / (n - 1) per axis;
// node index (i * ny + j) * nz + k, cell index (i * (ny - 1) + j) * (nz - 1) + k.  Values are
// centred (field - isovalue); a corner is inside when its value is >= 0 and a cell crosses
// the surface when its corners are neither all inside nor all outside (meshing.py:45-60).
//
// Steps (each a kernel or a library scan/sort, all on the caller's stream):
//  1. mark: one bit per crossing cell, from node values of an x-slab (the grid is classified
//     slab by slab so no full-grid value array is needed);
//  2. cells: popcount + scan of the mask words, then the crossing cells' indices in order;
//  3. triangulate: the eight corner values of each crossing cell -> triangles from the case
//     table; a vertex per crossing grid edge, shared by the triangles of every cell around it
//     (sort + unique of the 64-bit edge ids), placed at pa + t (pb - pa), t = fa / (fa - fb),
//     on the edge's lower (a) and upper (b) node.
//
// Case table.  Built at compile time from the cube's faces instead of a stored list: on each
// face, walking its corners counter-clockwise as seen from outside, every maximal run of
// inside corners gives one contour segment from the edge entering the run to the edge leaving
// it (a face whose inside corners are diagonal gets two segments: the inside corners are kept
// apart).  The segment of a face depends only on that face's four corner signs, so the two
// cells sharing a face cut it identically and the mesh has no cracks.  Segments chain into
// closed loops (an edge left on one face is entered on the other face holding it); each loop
// is a fan of triangles, oriented with their normals pointing from the inside (>= iso)
// toward the outside -- outward for the reconstructed indicator, which is larger inside.
#include "../../include/psr_b200.h"
#include "psr_internal.cuh"

#include <cmath>
#include <cstring>
#include <memory>
#include <string>

namespace psr {
namespace mc {

// Corner c of a cell at offset (x, y, z) (meshing.py:31-35 order: 000,100,110,010,001,...).
constexpr int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
// Edge e joins corners kEdge[e][0] (lower node along the edge's axis) and kEdge[e][1].
constexpr int kEdge[12][2] = {{0, 1}, {3, 2}, {0, 3}, {1, 2}, {4, 5}, {7, 6}, {4, 7}, {5, 6},
                              {0, 4}, {1, 5}, {3, 7}, {2, 6}};
// Faces, corners counter-clockwise as seen from outside the cell.
constexpr int kFace[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {3, 7, 6, 2}, {0, 4, 7, 3}, {1, 2, 6, 5}};
constexpr int kMaxTriangles = 8;

struct Tables {
  int8_t tri[256][3 * kMaxTriangles];  // edges of each triangle
  uint8_t count[256];                  // triangles per case
  int max_count;
  int8_t corner[8][3];                 // kCorner and kEdge for device code
  int8_t edge[12][2];
};

constexpr int edge_of(int a, int b) {
  for (int e = 0; e < 12; ++e)
    if ((kEdge[e][0] == a && kEdge[e][1] == b) || (kEdge[e][0] == b && kEdge[e][1] == a)) return e;
  return -1;
}

// Loops of one case as edge sequences; returns the loop count.
constexpr int case_loops(int code, int loops[6][13], int lengths[6]) {
  int entry[24] = {}, exit_[24] = {}, ns = 0;
  for (int f = 0; f < 6; ++f)
    for (int i = 0; i < 4; ++i) {
      const int c = kFace[f][i], prev = kFace[f][(i + 3) % 4];
      if (!((code >> c) & 1) || ((code >> prev) & 1)) continue;  // not the first corner of an inside run
      int j = i;
      while ((code >> kFace[f][(j + 1) % 4]) & 1) j = (j + 1) % 4;
      entry[ns] = edge_of(prev, c);
      exit_[ns] = edge_of(kFace[f][j], kFace[f][(j + 1) % 4]);
      ++ns;
    }
  bool used[24] = {};
  int nl = 0;
  for (int s = 0; s < ns; ++s) {
    if (used[s]) continue;
    int len = 0, cur = s;
    loops[nl][len++] = entry[s];
    while (true) {
      used[cur] = true;
      const int e = exit_[cur];
      if (e == loops[nl][0]) break;
      loops[nl][len++] = e;
      int next = -1;
      for (int t = 0; t < ns; ++t)
        if (!used[t] && entry[t] == e) next = t;
      if (next < 0) break;  // unreachable: every exit edge is some face's entry edge
      cur = next;
    }
    lengths[nl++] = len;
  }
  return nl;
}

constexpr double edge_mid(int e, int axis) {
  return 0.5 * (kCorner[kEdge[e][0]][axis] + kCorner[kEdge[e][1]][axis]);
}

constexpr Tables build_tables() {
  Tables t = {};
  for (int c = 0; c < 8; ++c)
    for (int a = 0; a < 3; ++a) t.corner[c][a] = int8_t(kCorner[c][a]);
  for (int e = 0; e < 12; ++e)
    for (int k = 0; k < 2; ++k) t.edge[e][k] = int8_t(kEdge[e][k]);
  // Orientation: the fan of case 1 (corner 0 inside) must face away from corner 0.
  bool flip = false;
  {
    int loops[6][13] = {}, lengths[6] = {};
    case_loops(1, loops, lengths);
    double a[3] = {}, b[3] = {}, c[3] = {};
    for (int k = 0; k < 3; ++k) {
      a[k] = edge_mid(loops[0][0], k);
      b[k] = edge_mid(loops[0][1], k);
      c[k] = edge_mid(loops[0][2], k);
    }
    const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const double n[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    flip = n[0] + n[1] + n[2] < 0.0;  // away from corner 0 = toward +x+y+z
  }
  t.max_count = 0;
  for (int code = 0; code < 256; ++code) {
    for (int i = 0; i < 3 * kMaxTriangles; ++i) t.tri[code][i] = -1;
    int loops[6][13] = {}, lengths[6] = {};
    const int nl = case_loops(code, loops, lengths);
    int n = 0;
    for (int l = 0; l < nl; ++l)
      for (int k = 1; k + 1 < lengths[l]; ++k) {
        if (n < kMaxTriangles) {
          t.tri[code][3 * n] = int8_t(loops[l][0]);
          t.tri[code][3 * n + 1] = int8_t(loops[l][flip ? k + 1 : k]);
          t.tri[code][3 * n + 2] = int8_t(loops[l][flip ? k : k + 1]);
        }
        ++n;
      }
    t.count[code] = uint8_t(n);
    if (n > t.max_count) t.max_count = n;
  }
  return t;
}

constexpr Tables kTables = build_tables();
static_assert(kTables.max_count <= kMaxTriangles, "a case has more triangles than the table holds");
static_assert(kTables.count[0] == 0 && kTables.count[255] == 0 && kTables.count[1] == 1, "case table");
__constant__ Tables c_tables = kTables;

struct Grid {
  int64_t nx, ny, nz;
  double lower[3], upper[3], step[3];
};

// Model-space position of node (i, j, k) in the field's precision (meshing.py:38-42,88-94).
template <class T>
__device__ __forceinline__ void node_point(const Grid& g, int64_t i, int64_t j, int64_t k, T p[3]) {
  const int64_t c[3] = {i, j, k};
  for (int a = 0; a < 3; ++a) {
    const T lo = T(g.lower[a]), hi = T(g.upper[a]);
    const T v = lo + T(g.step[a]) * T(c[a]);
    p[a] = v < lo ? lo : (v > hi ? hi : v);
  }
}

__device__ __forceinline__ void cell_coords(const Grid& g, int64_t cell, int64_t c[3]) {
  c[2] = cell % (g.nz - 1);
  c[1] = (cell / (g.nz - 1)) % (g.ny - 1);
  c[0] = cell / ((g.nz - 1) * (g.ny - 1));
}

// Nodes of x-planes [start, start + width] (slab) or the eight corners of each listed cell:
// their model positions (for a caller's field callback).
template <class T>
__global__ void points_kernel(Grid g, const int64_t* cells, int64_t start, int64_t count, T* points) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  int64_t c[3];
  if (cells) {
    cell_coords(g, cells[i / 8], c);
    for (int a = 0; a < 3; ++a) c[a] += c_tables.corner[i % 8][a];
  } else {
    c[0] = start + i / (g.ny * g.nz);
    c[1] = (i / g.nz) % g.ny;
    c[2] = i % g.nz;
  }
  node_point(g, c[0], c[1], c[2], points + 3 * i);
}

// The same points evaluated on the library's own field, centred: value - iso (meshing.py:114-118).
template <class T>
__global__ void field_values_kernel(psr_field_handle h, Grid g, const int64_t* cells, int64_t start, int64_t count,
                                    T iso, T* values) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  int64_t c[3];
  if (cells) {
    cell_coords(g, cells[i / 8], c);
    for (int a = 0; a < 3; ++a) c[a] += c_tables.corner[i % 8][a];
  } else {
    c[0] = start + i / (g.ny * g.nz);
    c[1] = (i / g.nz) % g.ny;
    c[2] = i % g.nz;
  }
  T p[3];
  node_point(g, c[0], c[1], c[2], p);
  values[i] = psr_field::evaluate<T>(h, p[0], p[1], p[2]).value - iso;
}

// Crossing cells of the slab [start, start + width) from its nodes' values (meshing.py:45-60).
template <class T>
__global__ void mark_kernel(const T* values, Grid g, int64_t start, int64_t width, uint32_t* mask, int* status) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int64_t ny = g.ny, nz = g.nz;
  if (i >= width * (ny - 1) * (nz - 1)) return;
  const int64_t x = i / ((ny - 1) * (nz - 1)), y = (i / (nz - 1)) % (ny - 1), z = i % (nz - 1);
  int code = 0;
  for (int c = 0; c < 8; ++c) {
    const T v = values[((x + c_tables.corner[c][0]) * ny + y + c_tables.corner[c][1]) * nz + z + c_tables.corner[c][2]];
    if (!isfinite(v)) atomicOr(status, 1);
    if (v >= T(0)) code |= 1 << c;
  }
  if (code != 0 && code != 255) {
    const int64_t index = ((start + x) * (ny - 1) + y) * (nz - 1) + z;
    atomicOr(mask + index / 32, 1u << (index % 32));
  }
}

__global__ void popc_kernel(const uint32_t* mask, int64_t words, int64_t* counts) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < words) counts[i] = __popc(mask[i]);
}

// Crossing cell indices in ascending order (inclusive word offsets).
__global__ void emit_cells_kernel(const uint32_t* mask, const int64_t* inclusive, int64_t words, int64_t* cells) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= words) return;
  uint32_t bits = mask[i];
  int64_t out = inclusive[i] - __popc(bits);
  while (bits) {
    const int b = __ffs(bits) - 1;
    cells[out++] = i * 32 + b;
    bits &= bits - 1;
  }
}

template <class T>
__device__ __forceinline__ int cube_code(const T* v) {
  int code = 0;
  for (int c = 0; c < 8; ++c)
    if (v[c] >= T(0)) code |= 1 << c;
  return code;
}

template <class T>
__global__ void triangle_count_kernel(const T* corner_values, int64_t count, int64_t* triangles) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < count) triangles[i] = c_tables.count[cube_code(corner_values + 8 * i)];
}

// Triangle corners of every crossing cell: the global id of the crossing edge, (node index of
// its lower node) * 3 + axis, and the flat corner-value indices of the edge's two nodes.
template <class T>
__global__ void triangle_emit_kernel(Grid g, const int64_t* cells, const T* corner_values, int64_t count,
                                     const int64_t* first, int64_t* edge_ids, int64_t* record_ids, int64_t* ends) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= count) return;
  const int code = cube_code(corner_values + 8 * i);
  int64_t c[3];
  cell_coords(g, cells[i], c);
  const int n = c_tables.count[code];
  for (int k = 0; k < 3 * n; ++k) {
    const int e = c_tables.tri[code][k];
    const int a = c_tables.edge[e][0], b = c_tables.edge[e][1];
    int axis = 0;
    while (c_tables.corner[a][axis] == c_tables.corner[b][axis]) ++axis;
    const int64_t node = ((c[0] + c_tables.corner[a][0]) * g.ny + c[1] + c_tables.corner[a][1]) * g.nz + c[2] + c_tables.corner[a][2];
    const int64_t r = 3 * first[i] + k;
    edge_ids[r] = node * 3 + axis;
    record_ids[r] = r;
    ends[2 * r] = 8 * i + a;
    ends[2 * r + 1] = 8 * i + b;
  }
}

// Sorted triangle corners -> vertex number of each (0-based, by first occurrence in edge order).
__global__ void vertex_flags_kernel(const int64_t* sorted_edges, int64_t n, int64_t* flags) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i < n) flags[i] = (i == 0 || sorted_edges[i] != sorted_edges[i - 1]) ? 1 : 0;
}

// One vertex per crossing edge at pa + t (pb - pa), t = fa / (fa - fb); triangle indices.
template <class T>
__global__ void vertex_kernel(Grid g, const int64_t* sorted_edges, const int64_t* sorted_records, const int64_t* number,
                              int64_t n, const int64_t* ends, const T* corner_values, T* vertices, int64_t* vertex_edges,
                              int64_t* vertex_ends, int32_t* indices) {
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const int64_t v = number[i] - 1;
  const int64_t r = sorted_records[i];
  indices[r] = int32_t(v);
  if (i != 0 && sorted_edges[i] == sorted_edges[i - 1]) return;
  const int64_t edge = sorted_edges[i], node = edge / 3;
  const int axis = int(edge % 3);
  int64_t c[3] = {node / (g.ny * g.nz), (node / g.nz) % g.ny, node % g.nz};
  T pa[3], pb[3];
  node_point(g, c[0], c[1], c[2], pa);
  c[axis] += 1;
  node_point(g, c[0], c[1], c[2], pb);
  const T fa = corner_values[ends[2 * r]], fb = corner_values[ends[2 * r + 1]];
  const T t = fa / (fa - fb);
  for (int a = 0; a < 3; ++a) vertices[3 * v + a] = pa[a] + t * (pb[a] - pa[a]);
  vertex_edges[v] = edge;
  vertex_ends[2 * v] = ends[2 * r];
  vertex_ends[2 * v + 1] = ends[2 * r + 1];
}

}  // namespace mc
}  // namespace psr

// ------------------------------------------------------------------ C ABI
struct psr_mesh {
  int32_t dtype = PSR_FLOAT32;
  int64_t vertices = 0, triangles = 0, cells = 0;
  psr::DBuf<int64_t> cell_ids;     // crossing cells (ascending), psr_extract_mesh only
  psr::DBuf<char> positions;       // vertices x 3 (dtype)
  psr::DBuf<int32_t> indices;      // triangles x 3
  psr::DBuf<int64_t> edges;        // vertices: crossing grid edge of each vertex
  psr::DBuf<int64_t> ends;         // vertices x 2: corner values (flat cell*8 + corner) at its two nodes
};

namespace {
using namespace psr;

mc::Grid make_grid(const int64_t shape[3], const double lower[3], const double upper[3]) {
  if (!shape || !lower || !upper) throw Error(PSR_EINVAL, "shape, lower and upper are required");
  mc::Grid g{};
  g.nx = shape[0];
  g.ny = shape[1];
  g.nz = shape[2];
  for (int a = 0; a < 3; ++a) {
    if (shape[a] < 2) throw Error(PSR_EINVAL, "resolution must be an integer or three integers >= 2");
    if (!std::isfinite(lower[a]) || !std::isfinite(upper[a]) || !(lower[a] < upper[a]))
      throw Error(PSR_EINVAL, "bounds must be finite with lower < upper on every axis");
    g.lower[a] = lower[a];
    g.upper[a] = upper[a];
  }
  // float32 spacing of the grid, as the reference computes it (meshing.py:145-147); float64
  // fields use the same spacing rounded to float64 from it
  for (int a = 0; a < 3; ++a) {
    const float step = (float(upper[a]) - float(lower[a])) / float(shape[a] - 1);
    if (!std::isfinite(step) || !(step > 0.f)) throw Error(PSR_EINVAL, "bounds/spacing must be representable in float32");
    g.step[a] = double(step);
    g.lower[a] = double(float(lower[a]));
    g.upper[a] = double(float(upper[a]));
  }
  if ((g.nx - 1) * (g.ny - 1) * (g.nz - 1) > int64_t(2147483647))
    throw Error(PSR_EINVAL, "extraction cell count exceeds int32 indexing");
  if (g.nx * g.ny * g.nz > int64_t(2147483647)) throw Error(PSR_EINVAL, "grid node count exceeds int32 sampling indices");
  return g;
}

int mesh_fail(const std::exception& e, int code) {
  set_last_error(e.what());
  return code;
}

template <class T>
psr_mesh* triangulate(const mc::Grid& g, const int64_t* cells, const T* cv, int64_t count, cudaStream_t s) {
  auto M = std::make_unique<psr_mesh>();
  M->dtype = sizeof(T) == 8 ? PSR_FLOAT64 : PSR_FLOAT32;
  if (count <= 0) return M.release();
  DBuf<int64_t> tc(count, s), first(count, s);
  mc::triangle_count_kernel<T><<<blocks_for(count), kThreads, 0, s>>>(cv, count, tc.p);
  PSR_LAUNCH_CHECK();
  exclusive_sum(tc.p, first.p, count, s);
  const int64_t tris = read_scalar(first.p + count - 1, s) + read_scalar(tc.p + count - 1, s);
  if (3 * tris > int64_t(2147483647)) throw Error(PSR_EINVAL, "triangle count exceeds int32 indexing");
  M->triangles = tris;
  if (!tris) return M.release();
  const int64_t n = 3 * tris;
  DBuf<int64_t> eid(n, s), rid(n, s), ends(2 * n, s), seid(n, s), srid(n, s), number(n, s);
  mc::triangle_emit_kernel<T><<<blocks_for(count), kThreads, 0, s>>>(g, cells, cv, count, first.p, eid.p, rid.p,
                                                                      ends.p);
  PSR_LAUNCH_CHECK();
  sort_pairs(eid.p, seid.p, rid.p, srid.p, n, bits_for(uint64_t(3 * g.nx * g.ny * g.nz)), s);
  mc::vertex_flags_kernel<<<blocks_for(n), kThreads, 0, s>>>(seid.p, n, number.p);
  PSR_LAUNCH_CHECK();
  inclusive_sum(number.p, number.p, n, s);
  const int64_t nv = read_scalar(number.p + n - 1, s);
  M->vertices = nv;
  M->positions.alloc(3 * nv * int64_t(sizeof(T)), s);
  M->indices.alloc(n, s);
  M->edges.alloc(nv, s);
  M->ends.alloc(2 * nv, s);
  mc::vertex_kernel<T><<<blocks_for(n), kThreads, 0, s>>>(g, seid.p, srid.p, number.p, n, ends.p, cv,
                                                          reinterpret_cast<T*>(M->positions.p), M->edges.p, M->ends.p,
                                                          M->indices.p);
  PSR_LAUNCH_CHECK();
  return M.release();
}

template <class T>
void slab_values(const psr_field_handle& h, const mc::Grid& g, int64_t start, int64_t width, double iso, T* values,
                 cudaStream_t s) {
  const int64_t count = (width + 1) * g.ny * g.nz;
  mc::field_values_kernel<T><<<blocks_for(count, 128), 128, 0, s>>>(h, g, nullptr, start, count, T(iso), values);
  PSR_LAUNCH_CHECK();
}

template <class T>
psr_mesh* extract(const psr_field_handle& h, const mc::Grid& g, double iso, int64_t slab, cudaStream_t s,
                  int64_t* retained) {
  const int64_t cells_total = (g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  const int64_t words = (cells_total + 31) / 32;
  DBuf<uint32_t> mask(words, s);
  mask.zero();
  DBuf<int> status(1, s);
  status.zero();
  DBuf<T> values((std::min(slab, g.nx - 1) + 1) * g.ny * g.nz, s);
  for (int64_t start = 0; start < g.nx - 1; start += slab) {
    const int64_t width = std::min(slab, g.nx - 1 - start);
    slab_values<T>(h, g, start, width, iso, values.p, s);
    mc::mark_kernel<T><<<blocks_for(width * (g.ny - 1) * (g.nz - 1)), kThreads, 0, s>>>(values.p, g, start, width,
                                                                                        mask.p, status.p);
    PSR_LAUNCH_CHECK();
  }
  values.release();
  DBuf<int64_t> counts(words, s);
  mc::popc_kernel<<<blocks_for(words), kThreads, 0, s>>>(mask.p, words, counts.p);
  PSR_LAUNCH_CHECK();
  inclusive_sum(counts.p, counts.p, words, s);
  const int64_t count = read_scalar(counts.p + words - 1, s);
  if (read_scalar(status.p, s)) throw Error(PSR_EDATA, "field returned nonfinite values inside extraction bounds");
  *retained = count;
  DBuf<int64_t> cells(count, s);
  DBuf<T> cv(8 * count, s);
  if (count) {
    mc::emit_cells_kernel<<<blocks_for(words), kThreads, 0, s>>>(mask.p, counts.p, words, cells.p);
    PSR_LAUNCH_CHECK();
    mc::field_values_kernel<T><<<blocks_for(8 * count, 128), 128, 0, s>>>(h, g, cells.p, 0, 8 * count, T(iso), cv.p);
    PSR_LAUNCH_CHECK();
  }
  psr_mesh* M = triangulate<T>(g, cells.p, cv.p, count, s);
  M->cells = count;
  M->cell_ids = std::move(cells);
  return M;
}
}  // namespace

extern "C" {

int psr_mc_points(int32_t dtype, const int64_t shape[3], const double lower[3], const double upper[3],
                  const int64_t* cells, int64_t start, int64_t count, void* points, void* stream) {
  try {
    const mc::Grid g = make_grid(shape, lower, upper);
    if (count < 0 || (count > 0 && !points)) throw Error(PSR_EINVAL, "points are required");
    if (count == 0) return PSR_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PSR_FLOAT64)
      mc::points_kernel<double><<<blocks_for(count), kThreads, 0, s>>>(g, cells, start, count, (double*)points);
    else if (dtype == PSR_FLOAT32)
      mc::points_kernel<float><<<blocks_for(count), kThreads, 0, s>>>(g, cells, start, count, (float*)points);
    else
      throw Error(PSR_EINVAL, "dtype must be float32 or float64");
    PSR_LAUNCH_CHECK();
    return PSR_OK;
  } catch (const Error& e) {
    return mesh_fail(e, e.code);
  } catch (const std::exception& e) {
    return mesh_fail(e, PSR_ECUDA);
  }
}

int psr_mc_mark(int32_t dtype, const void* values, const int64_t shape[3], int64_t start, int64_t width,
                uint32_t* mask, int32_t* status, void* stream) {
  try {
    if (!values || !shape || !mask || !status) throw Error(PSR_EINVAL, "values, shape, mask and status are required");
    mc::Grid g{};
    g.nx = shape[0];
    g.ny = shape[1];
    g.nz = shape[2];
    if (g.nx < 2 || g.ny < 2 || g.nz < 2 || start < 0 || width < 1 || start + width > g.nx - 1)
      throw Error(PSR_EINVAL, "slab outside the grid");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t cells = width * (g.ny - 1) * (g.nz - 1);
    if (dtype == PSR_FLOAT64)
      mc::mark_kernel<double><<<blocks_for(cells), kThreads, 0, s>>>((const double*)values, g, start, width, mask,
                                                                     status);
    else if (dtype == PSR_FLOAT32)
      mc::mark_kernel<float><<<blocks_for(cells), kThreads, 0, s>>>((const float*)values, g, start, width, mask,
                                                                    status);
    else
      throw Error(PSR_EINVAL, "dtype must be float32 or float64");
    PSR_LAUNCH_CHECK();
    return PSR_OK;
  } catch (const Error& e) {
    return mesh_fail(e, e.code);
  } catch (const std::exception& e) {
    return mesh_fail(e, PSR_ECUDA);
  }
}

int psr_mc_cells(const uint32_t* mask, int64_t words, int64_t* cells, int64_t capacity, int64_t* count, void* stream) {
  try {
    if (!mask || !count || words < 0) throw Error(PSR_EINVAL, "mask and count are required");
    cudaStream_t s = (cudaStream_t)stream;
    *count = 0;
    if (!words) return PSR_OK;
    DBuf<int64_t> counts(words, s);
    mc::popc_kernel<<<blocks_for(words), kThreads, 0, s>>>(mask, words, counts.p);
    PSR_LAUNCH_CHECK();
    inclusive_sum(counts.p, counts.p, words, s);
    *count = read_scalar(counts.p + words - 1, s);
    if (cells && *count) {
      if (capacity < *count) throw Error(PSR_EINVAL, "cells capacity is smaller than the crossing cell count");
      mc::emit_cells_kernel<<<blocks_for(words), kThreads, 0, s>>>(mask, counts.p, words, cells);
      PSR_LAUNCH_CHECK();
    }
    return PSR_OK;
  } catch (const Error& e) {
    return mesh_fail(e, e.code);
  } catch (const std::exception& e) {
    return mesh_fail(e, PSR_ECUDA);
  }
}

int psr_mc_triangulate(int32_t dtype, const int64_t shape[3], const double lower[3], const double upper[3],
                       const int64_t* cells, const void* corner_values, int64_t count, psr_mesh** out, void* stream) {
  try {
    if (!out) throw Error(PSR_EINVAL, "out must not be NULL");
    *out = nullptr;
    const mc::Grid g = make_grid(shape, lower, upper);
    if (count < 0 || (count > 0 && (!cells || !corner_values))) throw Error(PSR_EINVAL, "cells and values are required");
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PSR_FLOAT64)
      *out = triangulate<double>(g, cells, (const double*)corner_values, count, s);
    else if (dtype == PSR_FLOAT32)
      *out = triangulate<float>(g, cells, (const float*)corner_values, count, s);
    else
      throw Error(PSR_EINVAL, "dtype must be float32 or float64");
    return PSR_OK;
  } catch (const Error& e) {
    return mesh_fail(e, e.code);
  } catch (const std::exception& e) {
    return mesh_fail(e, PSR_ECUDA);
  }
}

int psr_extract_mesh(const psr_result* result, const int64_t shape[3], const double lower[3], const double upper[3],
                     double iso, int64_t slab, int64_t* retained, psr_mesh** out, void* stream) {
  try {
    if (!result || !out || !retained) throw Error(PSR_EINVAL, "result, retained and out are required");
    *out = nullptr;
    if (!std::isfinite(iso)) throw Error(PSR_EINVAL, "iso_value must be finite");
    if (slab < 1) throw Error(PSR_EINVAL, "slab_size must be a positive integer");
    const mc::Grid g = make_grid(shape, lower, upper);
    psr_field_handle h;
    int rc = psr_device_field(result, &h);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (h.dtype == PSR_FLOAT64)
      *out = extract<double>(h, g, iso, slab, s, retained);
    else
      *out = extract<float>(h, g, iso, slab, s, retained);
    return PSR_OK;
  } catch (const Error& e) {
    return mesh_fail(e, e.code);
  } catch (const std::exception& e) {
    return mesh_fail(e, PSR_ECUDA);
  }
}

int psr_mesh_info(const psr_mesh* mesh, int32_t* dtype, int64_t* vertices, int64_t* triangles, int64_t* cells) {
  if (!mesh || !dtype || !vertices || !triangles || !cells) {
    set_last_error("NULL argument");
    return PSR_EINVAL;
  }
  *dtype = mesh->dtype;
  *vertices = mesh->vertices;
  *triangles = mesh->triangles;
  *cells = mesh->cell_ids.p ? mesh->cells : 0;
  return PSR_OK;
}

int psr_mesh_arrays(const psr_mesh* mesh, const void** vertices, const int32_t** indices, const int64_t** edges,
                    const int64_t** ends, const int64_t** cells) {
  if (!mesh || !vertices || !indices || !edges || !ends || !cells) {
    set_last_error("NULL argument");
    return PSR_EINVAL;
  }
  *vertices = mesh->positions.p;
  *indices = mesh->indices.p;
  *edges = mesh->edges.p;
  *ends = mesh->ends.p;
  *cells = mesh->cell_ids.p;
  return PSR_OK;
}

int psr_mesh_free(psr_mesh* mesh) {
  if (!mesh) return PSR_OK;
  cudaDeviceSynchronize();
  delete mesh;
  return PSR_OK;
}

}  // extern "C"
