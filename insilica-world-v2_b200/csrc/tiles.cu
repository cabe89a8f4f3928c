// Host-side construction of the fast-loop tiles (see tiles.cuh).
#include <algorithm>
#include <deque>
#include <queue>
#include <unordered_map>

#include "common.cuh"
#include "tiles.cuh"

namespace isw {

std::vector<int32_t> partition_cells(int N, const int32_t *nbr, int P) {
  if (P < 1 || P > N) fail(ISW_EINVAL, "tiles: P outside 1..N");
  std::vector<int32_t> owner(N, -1);
  std::vector<std::deque<int>> frontier(P);
  std::vector<int> size(P, 0);
  // seeds spread along the cell numbering (Hilbert order: spread over the sphere)
  for (int p = 0; p < P; p++) frontier[p].push_back((int)(((int64_t)p * N + N / 2) / P));
  // grow the smallest region first (ties: the lower region id), one cell at a time, breadth-first within a region
  using Item = std::pair<int, int>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  for (int p = 0; p < P; p++) heap.push({0, p});
  while (!heap.empty()) {
    const int p = heap.top().second;
    heap.pop();
    auto &q = frontier[p];
    while (!q.empty() && owner[q.front()] >= 0) q.pop_front();
    if (q.empty()) continue;
    const int c = q.front();
    q.pop_front();
    owner[c] = p;
    size[p]++;
    for (int s = 0; s < 6; s++) {
      const int j = nbr[(size_t)c * 6 + s];
      if (j >= 0 && owner[j] < 0) q.push_back(j);
    }
    heap.push({size[p], p});
  }
  for (int c = 0; c < N; c++)
    if (owner[c] < 0) fail(ISW_EINVAL, "tiles: a cell no region reached");
  return owner;
}

TileSetHost build_tiles(int N, int E, const int32_t *nbr, const int32_t *cellEdge, const int8_t *cellSign, const int32_t *eI,
                        const int32_t *eJ, const std::vector<int32_t> &owner, int P, int k) {
  if (P < 1 || k < 1) fail(ISW_EINVAL, "tiles: P and k must be positive");
  TileSetHost t;
  t.P = P;
  t.k = k;
  t.cell_off.push_back(0);
  t.edge_off.push_back(0);
  std::vector<std::vector<int>> own(P);
  for (int c = 0; c < N; c++) own[owner[c]].push_back(c);
  std::vector<int> ring(N, -1);
  std::vector<int> touched;
  for (int p = 0; p < P; p++) {
    std::vector<int> order = own[p];
    for (int c : order) { ring[c] = 0; touched.push_back(c); }
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
    for (int r = 0; r <= k; r++) {
      const int a = r == 0 ? 0 : ring_end[r - 1], b = ring_end[r];
      std::sort(order.begin() + a, order.begin() + b);
    }
    std::unordered_map<int, int> lc;
    lc.reserve(order.size() * 2);
    for (size_t q = 0; q < order.size(); q++) lc[order[q]] = (int)q;
    // edges of the local cells, keyed by (ring of the nearer cell, not owned, id): owned edges first within ring 0
    std::vector<std::tuple<int, int, int>> ev;
    std::unordered_map<int, int> seen;
    seen.reserve(order.size() * 4);
    int eown = 0;
    for (int c : order)
      for (int s = 0; s < 6; s++) {
        const int e = cellEdge[(size_t)c * 6 + s];
        if (e < 0 || seen.count(e)) continue;
        seen[e] = 1;
        const int ra = ring[eI[e]] >= 0 ? ring[eI[e]] : k + 1, rb = ring[eJ[e]] >= 0 ? ring[eJ[e]] : k + 1;
        const int owned = owner[eI[e]] == p ? 0 : 1;
        if (!owned) eown++;
        ev.push_back(std::make_tuple(std::min(ra, rb), owned, e));
      }
    std::sort(ev.begin(), ev.end());
    std::unordered_map<int, int> le;
    le.reserve(ev.size() * 2);
    for (size_t q = 0; q < ev.size(); q++) le[std::get<2>(ev[q])] = (int)q;
    if (order.size() > 32000 || ev.size() > 32000) fail(ISW_EINVAL, "tiles: a tile outgrows 16-bit local ids");
    for (int r = 0; r <= k; r++) {
      t.ncnt.push_back(ring_end[r]);
      int ne = 0;
      while (ne < (int)ev.size() && std::get<0>(ev[ne]) <= r) ne++;
      t.ecnt.push_back(ne);
    }
    t.eown.push_back(eown);
    for (int c : order) {
      t.cells.push_back(c);
      for (int s = 0; s < 6; s++) {
        const int e = cellEdge[(size_t)c * 6 + s];
        const int v = e < 0 ? 0 : le.at(e) + 1;
        t.cedge.push_back((int16_t)(cellSign[(size_t)c * 6 + s] < 0 ? -v : v));
      }
      t.cedge.push_back(0);                    // two pads: a cell's slots are one 16-byte word
      t.cedge.push_back(0);
    }
    for (auto &tu : ev) {
      const int e = std::get<2>(tu);
      t.edges.push_back(e);
      auto a = lc.find(eI[e]), b = lc.find(eJ[e]);
      t.eIl.push_back(a == lc.end() ? (int16_t)-1 : (int16_t)a->second);
      t.eJl.push_back(b == lc.end() ? (int16_t)-1 : (int16_t)b->second);
    }
    t.cell_off.push_back((int32_t)t.cells.size());
    t.edge_off.push_back((int32_t)t.edges.size());
    t.smem = std::max(t.smem, tile_smem_bytes(order.size(), ev.size(), eown));
    for (int c : touched) ring[c] = -1;
    touched.clear();
  }
  return t;
}

}  // namespace isw
