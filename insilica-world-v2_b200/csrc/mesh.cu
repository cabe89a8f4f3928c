// The icosahedral Voronoi mesh with TRiSK C-grid tables, built from scratch: icosphere, Lloyd/SCVT smoothing (CPU, or a
// CUDA kernel per iteration for large levels), cell geometry, the edge list, the 3-D Hilbert renumbering, the TRiSK
// weights and the gather tables. It restates the reference's grid construction:
//   icosphere            src/insilica/grid/icosa.py:101-140     _adjacency :167-178   _sorted_ring :156-164
//   circumcenter         icosa.py:83-98   sph_tri_area :68-80   angle_between :62-65   _tangent_frame :143-153
//   lloyd_scvt           icosa.py:194-223   build_grid :227-277   edge_list :280-287
//   hilbert_order        icosa.py:290-338   reorder :341-353
//   build_trisk          src/insilica/grid/trisk.py:15-113   gather_tables :116-142
// Floating-point expressions keep NumPy's operation order (host code compiled without FMA contraction), so given the
// same Lloyd positions the integer tables (numbering, neighbours, edges, vertices, CSR, gather orders) are the
// reference's bit for bit; geometry that goes through atan2/asin/cos/sin may differ from NumPy's in the last bit.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace isw {
namespace mesh {

constexpr double R_PLANET = 6.371e6;
constexpr double PI = 3.141592653589793;
constexpr double OMEGA = 2 * PI / 86400;
constexpr double LLOYD_TOL = 1e-11;

struct V3 {
  double x, y, z;
};

__host__ __device__ inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline V3 add3(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ inline double norm(V3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
__host__ __device__ inline V3 scale(V3 v, double s) { return {v.x * s, v.y * s, v.z * s}; }
__host__ __device__ inline V3 divs(V3 v, double s) { return {v.x / s, v.y / s, v.z / s}; }

// tangent basis at a: e1 = a x axis (axis the coordinate least aligned with a, first on ties), normalised; e2 = a x e1
__host__ __device__ inline void tangent_basis(V3 a, V3 &e1, V3 &e2) {
  const double ax = fabs(a.x), ay = fabs(a.y), az = fabs(a.z);
  int k = 0;
  double m = ax;
  if (ay < m) { k = 1; m = ay; }
  if (az < m) { k = 2; }
  const V3 axis = {k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0};
  e1 = cross(a, axis);
  e1 = divs(e1, norm(e1));
  e2 = cross(a, e1);
}

// area of the spherical triangle (a, b, c) (Van Oosterom & Strackee, in a's tangent frame)
__host__ __device__ inline double sph_tri_area(V3 a, V3 b, V3 c) {
  const V3 u = sub(b, a), v = sub(c, a);
  V3 e1, e2;
  tangent_basis(a, e1, e2);
  const double u1 = dot(u, e1), u2 = dot(u, e2);
  const double v1 = dot(v, e1), v2 = dot(v, e2);
  const double triple = u1 * v2 - u2 * v1;
  const V3 w = sub(c, b);
  const double den = 4 - 0.5 * (dot(u, u) + dot(w, w) + dot(v, v));
  return 2 * atan2(fabs(triple), den);
}

// circumcenter of (a, b, c) on the unit sphere, computed in a's tangent frame from chords
__host__ __device__ inline V3 circumcenter(V3 pa, V3 pb, V3 pc) {
  V3 e1, e2;
  tangent_basis(pa, e1, e2);
  const V3 u = sub(pb, pa), v = sub(pc, pa);
  const double u1 = dot(u, e1), u2 = dot(u, e2), u3 = -0.5 * dot(u, u);
  const double v1 = dot(v, e1), v2 = dot(v, e2), v3 = -0.5 * dot(v, v);
  const double w1 = u2 * v3 - u3 * v2;
  const double w2 = u3 * v1 - u1 * v3;
  const double w3 = u1 * v2 - u2 * v1;
  const double t1 = w1 / w3, t2 = w2 / w3;
  const V3 p = add3(add3(pa, scale(e1, t1)), scale(e2, t2));
  return divs(p, norm(p));
}

inline double angle_between(V3 a, V3 b) {
  const double h = 0.5 * norm(sub(b, a));
  return 2 * std::asin(h < 1.0 ? h : 1.0);
}

// One Jacobi Lloyd update of cell i (icosa.py:208-219): the centroid of its Voronoi polygon's fan triangles.
// ring: 6 neighbours with pads replaced by slot 0's; nxt: next slot (pads point at themselves); m = degree.
__host__ __device__ inline V3 lloyd_cell(const V3 *V, const int *ring, const int *nxt, int m, int i) {
  const V3 p = V[i];
  V3 C[6];
  for (int k = 0; k < 6; k++) C[k] = circumcenter(p, V[ring[i * 6 + k]], V[ring[i * 6 + nxt[i * 6 + k]]]);
  V3 s = {0.0, 0.0, 0.0};
  for (int k = 0; k < 6; k++) {
    if (k >= m) continue;
    const V3 c0 = C[k], c1 = C[nxt[i * 6 + k]];
    const double a = sph_tri_area(p, c0, c1);
    s = add3(s, scale(add3(add3(p, c0), c1), a));
  }
  return divs(s, norm(s));
}

__global__ void k_lloyd(const V3 *__restrict__ Vin, V3 *__restrict__ Vout, const int *__restrict__ ring, const int *__restrict__ nxt,
                        const unsigned char *__restrict__ deg, int N, const int *done, unsigned long long *moved_bits) {
  if (*done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (i == 0 || i == 11) {                 // the poles stay pinned
    Vout[i] = Vin[i];
    return;
  }
  const V3 q = lloyd_cell(Vin, ring, nxt, deg[i], i);
  Vout[i] = q;
  const double d = norm(sub(q, Vin[i]));
  atomicMax(moved_bits, (unsigned long long)__double_as_longlong(d));
}

// after iteration `it`: stop once the largest move is below the tolerance (the iteration's update stays, as in the reference)
__global__ void k_lloyd_check(int it, double tol, int *done, int *last, unsigned long long *moved_bits, double *moved) {
  if (*done) return;
  const double m = __longlong_as_double((long long)*moved_bits);
  *moved = m;
  *last = it;
  if (m < tol) *done = 1;
  *moved_bits = 0ull;
}

struct Mesh {
  int n = 0, N = 0, E = 0, NV = 0;
  int lloydIters = 0;
  double lloydMoved = 0, totalArea = 0;
  std::vector<V3> pos, east, north, corners, edgeDir, xe, ne, vPos, xm;   // corners, edgeDir: N x 6
  std::vector<double> lat, lon, area, dist, edgeLen, de, le, kite, areaCell, areaV, fV, w;
  std::vector<int32_t> nbr, perm, eI, eJ, cornerV, cellEdge, ev1, ev2, eoeStart, eoe, cellEdgeAsc, vEdge, vCell;
  std::vector<uint8_t> deg, eKi, eKj;
  std::vector<int8_t> cellSign, circ1, circ2, vEdgeSign, vSlot;
};

// ---- icosphere (icosa.py:101-140) ----
static void icosphere(int n, std::vector<V3> &V, std::vector<std::array<int, 3>> &faces) {
  V.clear();
  auto addv = [&](double x, double y, double z) {
    const double r = std::sqrt(x * x + y * y + z * z);
    V.push_back({x / r, y / r, z / r});
    return (int)V.size() - 1;
  };
  addv(0.0, 0.0, 1.0);
  const double ring_lat = std::atan(0.5);
  for (int k = 0; k < 5; k++) {
    const double lo = (double)(k * 2) * PI / 5;
    addv(std::cos(ring_lat) * std::cos(lo), std::cos(ring_lat) * std::sin(lo), std::sin(ring_lat));
  }
  for (int k = 0; k < 5; k++) {
    const double lo = (k + 0.5) * 2 * PI / 5;
    addv(std::cos(ring_lat) * std::cos(lo), std::cos(ring_lat) * std::sin(lo), -std::sin(ring_lat));
  }
  addv(0.0, 0.0, -1.0);
  faces.clear();
  for (int k = 0; k < 5; k++) {
    const int u0 = 1 + k, u1 = 1 + (k + 1) % 5, l0 = 6 + k, l1 = 6 + (k + 1) % 5;
    faces.push_back({0, u0, u1});
    faces.push_back({u0, l0, u1});
    faces.push_back({u1, l0, l1});
    faces.push_back({11, l1, l0});
  }
  for (int s = 0; s < n; s++) {
    std::unordered_map<uint64_t, int> mid;
    auto midpoint = [&](int a, int b) {
      const uint64_t key = a < b ? ((uint64_t)a << 32 | (uint32_t)b) : ((uint64_t)b << 32 | (uint32_t)a);
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      const V3 va = V[a], vb = V[b];
      const int m = addv(va.x + vb.x, va.y + vb.y, va.z + vb.z);
      mid[key] = m;
      return m;
    };
    std::vector<std::array<int, 3>> nf;
    nf.reserve(faces.size() * 4);
    for (auto &f : faces) {
      const int a = f[0], b = f[1], c = f[2];
      const int ab = midpoint(a, b);
      const int bc = midpoint(b, c);
      const int ca = midpoint(c, a);
      nf.push_back({a, ab, ca});
      nf.push_back({b, bc, ab});
      nf.push_back({c, ca, bc});
      nf.push_back({ab, bc, ca});
    }
    faces.swap(nf);
  }
}

// neighbours of each cell in ascending index order (icosa.py:167-178)
static void adjacency(const std::vector<std::array<int, 3>> &faces, int N, std::vector<int32_t> &adj, std::vector<uint8_t> &deg) {
  std::vector<std::vector<int>> nb(N);
  for (auto &f : faces)
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++)
        if (p != q) nb[f[p]].push_back(f[q]);
  adj.assign((size_t)N * 6, -1);
  deg.assign(N, 0);
  for (int i = 0; i < N; i++) {
    std::sort(nb[i].begin(), nb[i].end());
    nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
    if (nb[i].size() > 6) fail(ISW_EINVAL, "mesh: a vertex with more than 6 neighbours");
    deg[i] = (uint8_t)nb[i].size();
    for (size_t k = 0; k < nb[i].size(); k++) adj[(size_t)i * 6 + k] = nb[i][k];
  }
}

static void tangent_frame(const std::vector<V3> &P, std::vector<V3> &east, std::vector<V3> &north) {
  const size_t N = P.size();
  east.resize(N);
  north.resize(N);
  for (size_t i = 0; i < N; i++) {
    double ex = -P[i].y, ey = P[i].x;
    double er = std::sqrt(ex * ex + ey * ey);
    if (er < 1e-12) { ex = 0.0; ey = 1.0; er = 1.0; }
    east[i] = {ex / er, ey / er, 0.0};
    north[i] = cross(P[i], east[i]);
  }
}

// neighbours sorted counterclockwise from east (icosa.py:156-164); pads stay last
static void sorted_ring(const std::vector<V3> &P, const std::vector<int32_t> &adj, std::vector<int32_t> &ring) {
  const size_t N = P.size();
  std::vector<V3> east, north;
  tangent_frame(P, east, north);
  ring.assign(N * 6, -1);
  for (size_t i = 0; i < N; i++) {
    double ang[6];
    int order[6];
    for (int k = 0; k < 6; k++) {
      const int a = adj[i * 6 + k];
      const V3 q = P[a > 0 ? a : 0];
      ang[k] = a < 0 ? INFINITY : std::atan2(dot(q, north[i]), dot(q, east[i]));
      order[k] = k;
    }
    std::stable_sort(order, order + 6, [&](int x, int y) { return ang[x] < ang[y]; });
    for (int k = 0; k < 6; k++) ring[i * 6 + k] = adj[i * 6 + order[k]];
  }
}

static inline int next_slot(int k, int m) { return k < m ? (k + 1) % m : k; }
static inline int prev_slot(int k, int m) { return k < m ? (k + m - 1) % m : k; }

// Lloyd/SCVT (icosa.py:194-223): Jacobi updates until the largest move is below tol, on the GPU (device >= 0) or host
static void lloyd(std::vector<V3> &V, const std::vector<int32_t> &ring, const std::vector<uint8_t> &deg, int max_iters, int device,
                  int &iters, double &moved) {
  const int N = (int)V.size();
  std::vector<int> ring_d((size_t)N * 6), nxt((size_t)N * 6);
  for (int i = 0; i < N; i++)
    for (int k = 0; k < 6; k++) {
      const int r = ring[(size_t)i * 6 + k];
      ring_d[(size_t)i * 6 + k] = r < 0 ? ring[(size_t)i * 6] : r;
      nxt[(size_t)i * 6 + k] = next_slot(k, deg[i]);
    }
  iters = 0;
  moved = INFINITY;
  if (max_iters <= 0) return;
  if (device < 0) {
    std::vector<V3> out(N);
    for (int it = 1; it <= max_iters; it++) {
      double mv = 0;
#pragma omp parallel for reduction(max : mv) schedule(static)
      for (int i = 0; i < N; i++) {
        if (i == 0 || i == 11) { out[i] = V[i]; continue; }
        const V3 q = lloyd_cell(V.data(), ring_d.data(), nxt.data(), deg[i], i);
        out[i] = q;
        const double d = norm(sub(q, V[i]));
        mv = d > mv ? d : mv;
      }
      V.swap(out);
      iters = it;
      moved = mv;
      if (mv < LLOYD_TOL) break;
    }
    return;
  }
  ISW_CUDA(cudaSetDevice(device));
  V3 *dV[2] = {nullptr, nullptr};
  int *dring = nullptr, *dnxt = nullptr, *ddone = nullptr, *dlast = nullptr;
  unsigned char *ddeg = nullptr;
  unsigned long long *dbits = nullptr;
  double *dmoved = nullptr;
  auto cleanup = [&] {
    cudaFree(dV[0]); cudaFree(dV[1]); cudaFree(dring); cudaFree(dnxt); cudaFree(ddeg); cudaFree(ddone); cudaFree(dlast);
    cudaFree(dbits); cudaFree(dmoved);
  };
  try {
    ISW_CUDA(cudaMalloc(&dV[0], sizeof(V3) * N));
    ISW_CUDA(cudaMalloc(&dV[1], sizeof(V3) * N));
    ISW_CUDA(cudaMalloc(&dring, sizeof(int) * N * 6));
    ISW_CUDA(cudaMalloc(&dnxt, sizeof(int) * N * 6));
    ISW_CUDA(cudaMalloc(&ddeg, N));
    ISW_CUDA(cudaMalloc(&ddone, sizeof(int)));
    ISW_CUDA(cudaMalloc(&dlast, sizeof(int)));
    ISW_CUDA(cudaMalloc(&dbits, sizeof(unsigned long long)));
    ISW_CUDA(cudaMalloc(&dmoved, sizeof(double)));
    ISW_CUDA(cudaMemcpy(dV[0], V.data(), sizeof(V3) * N, cudaMemcpyHostToDevice));
    ISW_CUDA(cudaMemcpy(dring, ring_d.data(), sizeof(int) * N * 6, cudaMemcpyHostToDevice));
    ISW_CUDA(cudaMemcpy(dnxt, nxt.data(), sizeof(int) * N * 6, cudaMemcpyHostToDevice));
    ISW_CUDA(cudaMemcpy(ddeg, deg.data(), N, cudaMemcpyHostToDevice));
    ISW_CUDA(cudaMemset(ddone, 0, sizeof(int)));
    ISW_CUDA(cudaMemset(dlast, 0, sizeof(int)));
    ISW_CUDA(cudaMemset(dbits, 0, sizeof(unsigned long long)));
    const int threads = 128, blocks = (N + threads - 1) / threads;
    const int chunk = 256;                   // iterations queued between host checks of the stop flag
    int done = 0;
    for (int it0 = 1; it0 <= max_iters && !done; it0 += chunk) {
      for (int it = it0; it < it0 + chunk && it <= max_iters; it++) {
        const int src = (it - 1) & 1;
        k_lloyd<<<blocks, threads>>>(dV[src], dV[src ^ 1], dring, dnxt, ddeg, N, ddone, dbits);
        k_lloyd_check<<<1, 1>>>(it, LLOYD_TOL, ddone, dlast, dbits, dmoved);
      }
      ISW_CUDA(cudaGetLastError());
      ISW_CUDA(cudaMemcpy(&done, ddone, sizeof(int), cudaMemcpyDeviceToHost));
    }
    ISW_CUDA(cudaMemcpy(&iters, dlast, sizeof(int), cudaMemcpyDeviceToHost));
    ISW_CUDA(cudaMemcpy(&moved, dmoved, sizeof(double), cudaMemcpyDeviceToHost));
    // iteration `iters` read buffer (iters - 1) & 1 and wrote the other one
    ISW_CUDA(cudaMemcpy(V.data(), dV[((iters - 1) & 1) ^ 1], sizeof(V3) * N, cudaMemcpyDeviceToHost));
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
}

// unique sorted triple key of corner (i, k): its cell and the two neighbours it sits between
static inline int64_t tri_key(int64_t a, int64_t b, int64_t c, int64_t N) {
  int64_t t[3] = {a, b, c};
  std::sort(t, t + 3);
  return (t[0] * N + t[1]) * N + t[2];
}

// first-occurrence table: for every valid (cell, slot) in row-major order, the flat index of the first (cell, slot) with
// the same key (np.unique(..., return_index) semantics), and the rank of each key by first appearance
static void first_occurrence(const std::vector<int64_t> &key, const std::vector<int> &flat, std::vector<int> &first_of,
                             std::vector<int> &rank_of) {
  std::unordered_map<int64_t, int> first;
  first.reserve(flat.size());
  first_of.resize(flat.size());
  rank_of.resize(flat.size());
  std::unordered_map<int64_t, int> rank;
  rank.reserve(flat.size());
  for (size_t q = 0; q < flat.size(); q++) {
    const int64_t k = key[flat[q]];
    auto it = first.find(k);
    if (it == first.end()) {
      first.emplace(k, flat[q]);
      rank.emplace(k, (int)rank.size());
      first_of[q] = flat[q];
      rank_of[q] = (int)rank.size() - 1;
    } else {
      first_of[q] = it->second;
      rank_of[q] = rank[k];
    }
  }
}

// geometry of the smoothed mesh (icosa.py:235-277)
static void build_geometry(Mesh &g, const std::vector<int32_t> &adj) {
  const int N = g.N;
  g.lat.resize(N);
  g.lon.resize(N);
  for (int i = 0; i < N; i++) {
    const double z = g.pos[i].z;
    g.lat[i] = std::asin(z < -1 ? -1 : (z > 1 ? 1 : z));
    g.lon[i] = std::atan2(g.pos[i].y, g.pos[i].x);
  }
  tangent_frame(g.pos, g.east, g.north);
  sorted_ring(g.pos, adj, g.nbr);
  std::vector<int> nb((size_t)N * 6);
  for (int i = 0; i < N; i++)
    for (int k = 0; k < 6; k++) {
      const bool valid = k < g.deg[i];
      if (!valid) g.nbr[(size_t)i * 6 + k] = -1;
      nb[(size_t)i * 6 + k] = valid ? g.nbr[(size_t)i * 6 + k] : g.nbr[(size_t)i * 6];
    }
  g.corners.assign((size_t)N * 6, {0.0, 0.0, 0.0});
  std::vector<int64_t> key((size_t)N * 6, 0);
  std::vector<int> flat;
  for (int i = 0; i < N; i++)
    for (int k = 0; k < g.deg[i]; k++) {
      const int j = nb[(size_t)i * 6 + k], j2 = nb[(size_t)i * 6 + next_slot(k, g.deg[i])];
      g.corners[(size_t)i * 6 + k] = circumcenter(g.pos[i], g.pos[j], g.pos[j2]);
      key[(size_t)i * 6 + k] = tri_key(i, j, j2, N);
      flat.push_back(i * 6 + k);
    }
  std::vector<int> first_of, rank_of;
  first_occurrence(key, flat, first_of, rank_of);
  std::vector<V3> shared(g.corners);
  for (size_t q = 0; q < flat.size(); q++) shared[flat[q]] = g.corners[first_of[q]];
  g.corners.swap(shared);
  g.dist.assign((size_t)N * 6, 0.0);
  g.edgeLen.assign((size_t)N * 6, 0.0);
  g.edgeDir.assign((size_t)N * 6, {0.0, 0.0, 0.0});
  g.area.assign(N, 0.0);
  for (int i = 0; i < N; i++) {
    const int m = g.deg[i];
    const V3 P = g.pos[i];
    double area = 0.0;
    for (int k = 0; k < 6; k++) {
      if (k >= m) continue;
      const V3 ca = g.corners[(size_t)i * 6 + prev_slot(k, m)], cb = g.corners[(size_t)i * 6 + k];
      const V3 q = g.pos[nb[(size_t)i * 6 + k]];
      g.dist[(size_t)i * 6 + k] = R_PLANET * angle_between(P, q);
      g.edgeLen[(size_t)i * 6 + k] = R_PLANET * angle_between(ca, cb);
      const V3 e = sub(cb, ca);
      V3 t = cross(e, P);
      const double tp = dot(t, P);
      t = sub(t, scale(P, tp));
      if (dot(t, sub(q, P)) < 0) t = {-t.x, -t.y, -t.z};
      g.edgeDir[(size_t)i * 6 + k] = divs(t, norm(t));
      const V3 c1 = g.corners[(size_t)i * 6 + next_slot(k, m)];
      area = area + sph_tri_area(P, cb, c1);
    }
    g.area[i] = area * R_PLANET * R_PLANET;
  }
  double tot = 0;
  for (int i = 0; i < N; i++) tot += g.area[i];
  g.totalArea = tot;
}

// edges (i < j) by i, then slot (icosa.py:280-287)
static void edge_list(Mesh &g) {
  g.eI.clear(); g.eJ.clear(); g.eKi.clear(); g.eKj.clear();
  for (int i = 0; i < g.N; i++)
    for (int k = 0; k < g.deg[i]; k++) {
      const int j = g.nbr[(size_t)i * 6 + k];
      if (j > i) {
        int kj = 0;
        for (int s = 0; s < 6; s++)
          if (g.nbr[(size_t)j * 6 + s] == i) { kj = s; break; }
        g.eI.push_back(i); g.eJ.push_back(j); g.eKi.push_back((uint8_t)k); g.eKj.push_back((uint8_t)kj);
      }
    }
  g.E = (int)g.eI.size();
}

// 3-D Hilbert order of the unit positions (icosa.py:290-338; Skilling 2004): quantise to 21 bits, transpose, Gray code,
// interleave the bits into one key, stable sort
void hilbert_order(const std::vector<V3> &pos, std::vector<int32_t> &perm) {
  const int bits = 21;
  const size_t N = pos.size();
  const uint64_t maxq = (1ull << bits) - 1;
  std::vector<uint64_t> key(N);
  for (size_t n = 0; n < N; n++) {
    const double c[3] = {pos[n].x, pos[n].y, pos[n].z};
    uint64_t X[3];
    for (int i = 0; i < 3; i++) {
      const double f = (c[i] + 1) * 0.5 * (double)maxq;
      uint64_t q = (uint64_t)f;
      X[i] = q > maxq ? maxq : q;
    }
    for (uint64_t Q = 1ull << (bits - 1); Q > 1; Q >>= 1) {
      const uint64_t P = Q - 1;
      for (int i = 0; i < 3; i++) {
        const bool hit = (X[i] & Q) != 0;
        const uint64_t t = (X[0] ^ X[i]) & P;
        const uint64_t X0 = hit ? X[0] ^ P : X[0] ^ t;
        const uint64_t Xi = hit ? X[i] : X[i] ^ t;
        X[0] = X0;
        if (i) X[i] = Xi;
      }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    uint64_t t = 0;
    for (uint64_t Q = 1ull << (bits - 1); Q > 1; Q >>= 1)
      if (X[2] & Q) t ^= Q - 1;
    for (int i = 0; i < 3; i++) X[i] ^= t;
    uint64_t k = 0;
    for (int b = bits - 1; b >= 0; b--)
      for (int i = 0; i < 3; i++) k = (k << 1) | ((X[i] >> b) & 1ull);
    key[n] = k;
  }
  perm.resize(N);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
}

// renumber cells: new cell k is old cell perm[k]; edges follow by their lower cell (icosa.py:341-353)
static void reorder(Mesh &g, const std::vector<int32_t> &perm) {
  const int N = g.N;
  std::vector<int32_t> inv(N);
  for (int k = 0; k < N; k++) inv[perm[k]] = k;
  auto pc = [&](auto &a, int width) {
    auto b = a;
    for (int k = 0; k < N; k++)
      for (int s = 0; s < width; s++) b[(size_t)k * width + s] = a[(size_t)perm[k] * width + s];
    a.swap(b);
  };
  pc(g.pos, 1); pc(g.lat, 1); pc(g.lon, 1); pc(g.area, 1); pc(g.east, 1); pc(g.north, 1); pc(g.deg, 1);
  pc(g.dist, 6); pc(g.edgeLen, 6); pc(g.edgeDir, 6); pc(g.corners, 6);
  std::vector<int32_t> nbr((size_t)N * 6);
  for (int k = 0; k < N; k++)
    for (int s = 0; s < 6; s++) {
      const int v = g.nbr[(size_t)perm[k] * 6 + s];
      nbr[(size_t)k * 6 + s] = v >= 0 ? inv[v] : -1;
    }
  g.nbr.swap(nbr);
  edge_list(g);
  g.perm = perm;
}

// TRiSK geometry and tables (trisk.py:15-113) and the gather tables (trisk.py:116-142)
static void build_trisk(Mesh &g) {
  const int N = g.N, E = g.E;
  // vertices: one per triangle, numbered by first appearance of its sorted cell triple
  std::vector<int64_t> key((size_t)N * 6, 0);
  std::vector<int> flat;
  for (int i = 0; i < N; i++) {
    const int m = g.deg[i];
    for (int k = 0; k < m; k++) {
      const int j = g.nbr[(size_t)i * 6 + k], j2 = g.nbr[(size_t)i * 6 + next_slot(k, m)];
      key[(size_t)i * 6 + k] = tri_key(i, j, j2, N);
      flat.push_back(i * 6 + k);
    }
  }
  std::vector<int> first_of, rank_of;
  first_occurrence(key, flat, first_of, rank_of);
  int NV = 0;
  for (int r : rank_of) NV = r + 1 > NV ? r + 1 : NV;
  g.NV = NV;
  g.cornerV.assign((size_t)N * 6, -1);
  g.vPos.assign(NV, {0.0, 0.0, 0.0});
  for (size_t q = 0; q < flat.size(); q++) {
    g.cornerV[flat[q]] = rank_of[q];
    if (first_of[q] == flat[q]) g.vPos[rank_of[q]] = g.corners[flat[q]];
  }
  g.cellEdge.assign((size_t)N * 6, -1);
  g.cellSign.assign((size_t)N * 6, 0);
  for (int e = 0; e < E; e++) {
    g.cellEdge[(size_t)g.eI[e] * 6 + g.eKi[e]] = e;
    g.cellSign[(size_t)g.eI[e] * 6 + g.eKi[e]] = 1;
    g.cellEdge[(size_t)g.eJ[e] * 6 + g.eKj[e]] = e;
    g.cellSign[(size_t)g.eJ[e] * 6 + g.eKj[e]] = -1;
  }
  g.ev1.resize(E); g.ev2.resize(E); g.de.resize(E); g.le.resize(E); g.xe.resize(E); g.ne.resize(E);
  for (int e = 0; e < E; e++) {
    const int i = g.eI[e], ki = g.eKi[e], mi = g.deg[i];
    g.ev1[e] = g.cornerV[(size_t)i * 6 + (ki + mi - 1) % mi];
    g.ev2[e] = g.cornerV[(size_t)i * 6 + ki];
    g.de[e] = g.dist[(size_t)i * 6 + ki];
    g.le[e] = g.edgeLen[(size_t)i * 6 + ki];
    const V3 pi = g.pos[i], pj = g.pos[g.eJ[e]];
    const V3 s = add3(pi, pj);
    const V3 xe = divs(s, norm(s));
    V3 d = sub(pj, pi);
    d = sub(d, scale(xe, dot(d, xe)));
    g.xe[e] = xe;
    g.ne[e] = divs(d, norm(d));
  }
  // kites: cell i and the triangle at corner k (xi, edge k's xe, the vertex, edge k+1's xe)
  g.kite.assign((size_t)N * 6, 0.0);
  g.areaCell.assign(N, 0.0);
  for (int i = 0; i < N; i++) {
    const int m = g.deg[i];
    const V3 P = g.pos[i];
    for (int k = 0; k < m; k++) {
      const int e0 = g.cellEdge[(size_t)i * 6 + k], e1 = g.cellEdge[(size_t)i * 6 + next_slot(k, m)];
      const V3 vp = g.vPos[g.cornerV[(size_t)i * 6 + k]];
      g.kite[(size_t)i * 6 + k] = (sph_tri_area(P, g.xe[e0], vp) + sph_tri_area(P, vp, g.xe[e1])) * R_PLANET * R_PLANET;
    }
    double a = 0.0;
    for (int k = 0; k < 6; k++) a = a + g.kite[(size_t)i * 6 + k];
    g.areaCell[i] = a;
  }
  g.areaV.assign(NV, 0.0);
  for (int i = 0; i < N; i++)
    for (int k = 0; k < g.deg[i]; k++) g.areaV[g.cornerV[(size_t)i * 6 + k]] += g.kite[(size_t)i * 6 + k];
  auto circ = [&](int e, int vi) -> int8_t {
    const V3 dd = sub(g.xe[e], g.vPos[vi]);
    const double x = dot(g.ne[e], cross(g.xe[e], dd));
    return (int8_t)(x > 0 ? 1 : (x < 0 ? -1 : 0));
  };
  g.circ1.resize(E); g.circ2.resize(E);
  for (int e = 0; e < E; e++) { g.circ1[e] = circ(e, g.ev1[e]); g.circ2[e] = circ(e, g.ev2[e]); }
  // tangential weights, CSR in the reference's order: eI's edges (steps 1..deg-1), then eJ's
  g.eoeStart.assign((size_t)E + 1, 0);
  g.eoe.clear();
  g.w.clear();
  for (int e = 0; e < E; e++) {
    for (int side = 0; side < 2; side++) {
      const int c = side == 0 ? g.eI[e] : g.eJ[e], kc = side == 0 ? g.eKi[e] : g.eKj[e];
      const double se = side == 0 ? 1.0 : -1.0;
      const int m = g.deg[c];
      double rsum = 0.0;
      for (int step = 1; step <= 5; step++) {
        const bool ok = step < m;
        const int k = (kc + step) % m, kv = (k + m - 1) % m;
        rsum = rsum + (ok ? g.kite[(size_t)c * 6 + kv] / g.areaCell[c] : 0.0);
        if (!ok) continue;
        const int e2 = g.cellEdge[(size_t)c * 6 + k];
        const double wt = se * (0.5 - rsum) * (double)g.cellSign[(size_t)c * 6 + k] * g.le[e2] / g.de[e];
        g.eoe.push_back(e2);
        g.w.push_back(wt);
      }
    }
    g.eoeStart[(size_t)e + 1] = (int32_t)g.eoe.size();
  }
  g.fV.resize(NV);
  g.xm.resize(E);
  for (int v = 0; v < NV; v++) g.fV[v] = 2 * OMEGA * g.vPos[v].z;
  for (int e = 0; e < E; e++) {
    const V3 s = add3(g.vPos[g.ev1[e]], g.vPos[g.ev2[e]]);
    g.xm[e] = divs(s, norm(s));
  }
  // gather tables
  g.cellEdgeAsc.assign((size_t)N * 6, -1);
  for (int i = 0; i < N; i++) {
    int order[6];
    for (int k = 0; k < 6; k++) order[k] = k;
    const int32_t *ce = &g.cellEdge[(size_t)i * 6];
    std::stable_sort(order, order + 6, [&](int a, int b) {
      const int64_t ka = ce[a] < 0 ? INT64_MAX : ce[a], kb = ce[b] < 0 ? INT64_MAX : ce[b];
      return ka < kb;
    });
    for (int k = 0; k < 6; k++) g.cellEdgeAsc[(size_t)i * 6 + k] = ce[order[k]];
  }
  std::vector<std::vector<std::pair<int, int8_t>>> ve(NV);
  for (int e = 0; e < E; e++) {
    ve[g.ev1[e]].push_back({e, g.circ1[e]});
    ve[g.ev2[e]].push_back({e, g.circ2[e]});
  }
  g.vEdge.assign((size_t)NV * 3, 0);
  g.vEdgeSign.assign((size_t)NV * 3, 0);
  for (int v = 0; v < NV; v++) {
    auto &l = ve[v];
    if (l.size() != 3) fail(ISW_EINVAL, "mesh: a vertex without exactly three edges");
    std::stable_sort(l.begin(), l.end(), [](const std::pair<int, int8_t> &a, const std::pair<int, int8_t> &b) { return a.first < b.first; });
    for (int s = 0; s < 3; s++) { g.vEdge[(size_t)v * 3 + s] = l[s].first; g.vEdgeSign[(size_t)v * 3 + s] = l[s].second; }
  }
  std::vector<std::vector<std::pair<int, int>>> vc(NV);
  for (int i = 0; i < N; i++)
    for (int k = 0; k < g.deg[i]; k++) vc[g.cornerV[(size_t)i * 6 + k]].push_back({i, k});
  g.vCell.assign((size_t)NV * 3, 0);
  g.vSlot.assign((size_t)NV * 3, 0);
  for (int v = 0; v < NV; v++) {
    auto &l = vc[v];
    if (l.size() != 3) fail(ISW_EINVAL, "mesh: a vertex not shared by exactly three cells");
    std::stable_sort(l.begin(), l.end(), [](const std::pair<int, int> &a, const std::pair<int, int> &b) { return a.first < b.first; });
    for (int s = 0; s < 3; s++) { g.vCell[(size_t)v * 3 + s] = l[s].first; g.vSlot[(size_t)v * 3 + s] = (int8_t)l[s].second; }
  }
}

}  // namespace mesh
}  // namespace isw

using namespace isw;
using namespace isw::mesh;

struct isw_mesh {
  Mesh m;
};

namespace {

isw_mesh *mesh_build(int n, int hilbert, int max_iters, int device, const double *pos_v1) {
  if (n < 0 || n > 9) fail(ISW_EINVAL, "mesh: level n outside 0..9");
  auto *out = new isw_mesh();
  Mesh &g = out->m;
  try {
    std::vector<std::array<int, 3>> faces;
    icosphere(n, g.pos, faces);
    g.n = n;
    g.N = (int)g.pos.size();
    std::vector<int32_t> adj;
    adjacency(faces, g.N, adj, g.deg);
    if (pos_v1) {
      for (int i = 0; i < g.N; i++) g.pos[i] = {pos_v1[3 * i], pos_v1[3 * i + 1], pos_v1[3 * i + 2]};
      g.lloydIters = 0;
      g.lloydMoved = 0;
    } else {
      std::vector<int32_t> ring;
      sorted_ring(g.pos, adj, ring);
      lloyd(g.pos, ring, g.deg, max_iters, device, g.lloydIters, g.lloydMoved);
    }
    build_geometry(g, adj);
    edge_list(g);
    if (hilbert) {
      std::vector<int32_t> perm;
      hilbert_order(g.pos, perm);
      reorder(g, perm);
    }
    build_trisk(g);
  } catch (...) {
    delete out;
    throw;
  }
  return out;
}

template <class T>
void put(const std::vector<T> &v, const void **data, int64_t *count) {
  *data = v.data();
  *count = (int64_t)v.size();
}

}  // namespace

extern "C" {

int isw_mesh_build(int n, int hilbert, int max_iters, int device, const double *pos_v1, isw_mesh **out) {
  try {
    if (!out) fail(ISW_EINVAL, "mesh: null output handle");
    *out = mesh_build(n, hilbert, max_iters, device, pos_v1);
    return ISW_OK;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("mesh: host allocation failed");
    return ISW_ENOMEM;
  }
}

int isw_mesh_destroy(isw_mesh *m) {
  delete m;
  return ISW_OK;
}

// kinds: 0 float64 (count = values), 1 int32, 2 int8, 3 uint8, 4 float64 x3 vectors (count = vectors)
int isw_mesh_get(const isw_mesh *mp, const char *name, const void **data, int64_t *count, int *kind) {
  try {
    if (!mp || !name || !data || !count || !kind) fail(ISW_EINVAL, "mesh_get: null argument");
    const Mesh &g = mp->m;
    const std::string s(name);
    static thread_local int64_t scalar_i;
    static thread_local double scalar_d;
    *kind = 0;
#define F64(n) if (s == #n) { put(g.n, data, count); *kind = 0; return ISW_OK; }
#define I32(n) if (s == #n) { put(g.n, data, count); *kind = 1; return ISW_OK; }
#define I8(n) if (s == #n) { put(g.n, data, count); *kind = 2; return ISW_OK; }
#define U8(n) if (s == #n) { put(g.n, data, count); *kind = 3; return ISW_OK; }
#define VEC(n) if (s == #n) { put(g.n, data, count); *kind = 4; return ISW_OK; }
    F64(lat) F64(lon) F64(area) F64(dist) F64(edgeLen) F64(de) F64(le) F64(kite) F64(areaCell) F64(areaV) F64(fV) F64(w)
    I32(nbr) I32(perm) I32(eI) I32(eJ) I32(cornerV) I32(cellEdge) I32(ev1) I32(ev2) I32(eoeStart) I32(eoe) I32(cellEdgeAsc)
    I32(vEdge) I32(vCell)
    U8(deg) U8(eKi) U8(eKj)
    I8(cellSign) I8(circ1) I8(circ2) I8(vEdgeSign) I8(vSlot)
    VEC(pos) VEC(east) VEC(north) VEC(corners) VEC(edgeDir) VEC(xe) VEC(ne) VEC(vPos) VEC(xm)
#undef F64
#undef I32
#undef I8
#undef U8
#undef VEC
    if (s == "n" || s == "N" || s == "E" || s == "NV" || s == "lloydIters") {
      scalar_i = s == "n" ? g.n : s == "N" ? g.N : s == "E" ? g.E : s == "NV" ? g.NV : g.lloydIters;
      *data = &scalar_i;
      *count = 1;
      *kind = 5;           // int64 scalar
      return ISW_OK;
    }
    if (s == "lloydMoved" || s == "totalArea") {
      scalar_d = s == "lloydMoved" ? g.lloydMoved : g.totalArea;
      *data = &scalar_d;
      *count = 1;
      *kind = 6;           // float64 scalar
      return ISW_OK;
    }
    fail(ISW_EINVAL, "mesh_get: no array named " + s);
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  }
  return ISW_EINVAL;
}

}  // extern "C"
