// Host-side construction of the fast-loop tiles (see tiles.cuh).
#include <algorithm>
#include <numeric>
#include <unordered_map>

#include "common.cuh"
#include "tiles.cuh"

namespace isw {

TileSetHost build_tiles(int N, int E, const int32_t *nbr, const int32_t *cellEdge, const int32_t *eI, const int32_t *eJ, int P,
                        int k) {
  if (P < 1 || k < 1) fail(ISW_EINVAL, "tiles: P and k must be positive");
  TileSetHost t;
  t.P = P;
  t.k = k;
  t.cell_off.push_back(0);
  t.edge_off.push_back(0);
  std::vector<int> ring(N, -1);
  std::vector<int> touched;
  for (int p = 0; p < P; p++) {
    const int c0 = (int)((int64_t)N * p / P), c1 = (int)((int64_t)N * (p + 1) / P);
    // rings by breadth-first search from the owned range
    std::vector<int> order;
    for (int c = c0; c < c1; c++) { ring[c] = 0; order.push_back(c); touched.push_back(c); }
    size_t head = 0;
    std::vector<int> ring_end(k + 1, 0);
    ring_end[0] = (int)order.size();
    for (int r = 1; r <= k; r++) {
      const size_t stop = order.size();
      for (; head < stop; head++) {
        const int c = order[head];
        for (int s = 0; s < 6; s++) {
          const int j = nbr[(size_t)c * 6 + s];
          if (j < 0 || ring[j] >= 0) continue;
          ring[j] = r;
          order.push_back(j);
          touched.push_back(j);
        }
      }
      ring_end[r] = (int)order.size();
    }
    // ring order, ascending global id within a ring
    for (int r = 0; r <= k; r++) {
      const int a = r == 0 ? 0 : ring_end[r - 1], b = ring_end[r];
      std::sort(order.begin() + a, order.begin() + b);
    }
    std::unordered_map<int, int> lc;
    lc.reserve(order.size() * 2);
    for (size_t q = 0; q < order.size(); q++) lc[order[q]] = (int)q;
    // edges of the local cells, keyed by the ring of their nearer cell
    std::vector<std::pair<int, int>> ev;     // (ring, edge)
    std::unordered_map<int, int> seen;
    seen.reserve(order.size() * 4);
    for (int c : order)
      for (int s = 0; s < 6; s++) {
        const int e = cellEdge[(size_t)c * 6 + s];
        if (e < 0 || seen.count(e)) continue;
        seen[e] = 1;
        const int ra = ring[eI[e]] >= 0 ? ring[eI[e]] : k + 1, rb = ring[eJ[e]] >= 0 ? ring[eJ[e]] : k + 1;
        ev.push_back({std::min(ra, rb), e});
      }
    std::sort(ev.begin(), ev.end());
    std::unordered_map<int, int> le;
    le.reserve(ev.size() * 2);
    for (size_t q = 0; q < ev.size(); q++) le[ev[q].second] = (int)q;
    if (order.size() > 32767 || ev.size() > 32767) fail(ISW_EINVAL, "tiles: a tile outgrows 16-bit local ids");
    for (int r = 0; r <= k; r++) {
      t.ncnt.push_back(ring_end[r]);
      int ne = 0;
      while (ne < (int)ev.size() && ev[ne].first <= r) ne++;
      t.ecnt.push_back(ne);
    }
    for (int c : order) {
      t.cells.push_back(c);
      for (int s = 0; s < 6; s++) {
        const int e = cellEdge[(size_t)c * 6 + s];
        t.cedge.push_back(e < 0 ? (int16_t)-1 : (int16_t)le.at(e));
      }
    }
    for (auto &pr : ev) {
      const int e = pr.second;
      t.edges.push_back(e);
      auto a = lc.find(eI[e]), b = lc.find(eJ[e]);
      t.eIl.push_back(a == lc.end() ? (int16_t)-1 : (int16_t)a->second);
      t.eJl.push_back(b == lc.end() ? (int16_t)-1 : (int16_t)b->second);
    }
    t.cell_off.push_back((int32_t)t.cells.size());
    t.edge_off.push_back((int32_t)t.edges.size());
    t.smem = std::max(t.smem, tile_smem_bytes(order.size(), ev.size()));
    for (int c : touched) ring[c] = -1;
    touched.clear();
  }
  return t;
}

}  // namespace isw
