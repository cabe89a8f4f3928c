// Grid upload (reference src/insilica/gpu.py:55-83, DeviceGrid) and the 3rd-order transport stencil (gpu.py:86-108).
//
// Every index table is validated on the host before it reaches the device: each entry is in range (or a -1 pad where
// the reference pads), so the kernels may gather through them without bounds checks.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <sstream>

#include "common.cuh"

namespace isw {

static thread_local std::string g_last_error;

void set_last_error(const std::string &m) { g_last_error = m; }

void fail(int status, const std::string &m) { throw Error{status, m}; }

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << what << ": " << cudaGetErrorString(e);
    fail(e == cudaErrorMemoryAllocation ? ISW_ENOMEM : ISW_ECUDA, s.str());
  }
}

const char *last_error() { return g_last_error.c_str(); }

namespace {

template <class T>
void need(const T *p, const char *name) {
  if (!p) fail(ISW_EINVAL, std::string("grid: missing array ") + name);
}

void check_range(const int32_t *a, size_t n, int lo, int hi, bool pads, const char *name) {
  for (size_t i = 0; i < n; i++) {
    const int v = a[i];
    if (v == -1 && pads) continue;
    if (v < lo || v >= hi) {
      std::ostringstream s;
      s << "grid: " << name << "[" << i << "] = " << v << " outside [" << lo << ", " << hi << ")";
      fail(ISW_EINVAL, s.str());
    }
  }
}

// Padded per-cell tables: valid slots first, then -1 only (the kernels stop at the first pad).
void check_padded_rows(const int32_t *a, int rows, int width, int hi, const char *name) {
  check_range(a, (size_t)rows * width, 0, hi, true, name);
  for (int r = 0; r < rows; r++) {
    bool pad = false;
    for (int k = 0; k < width; k++) {
      const int v = a[(size_t)r * width + k];
      if (v < 0) pad = true;
      else if (pad) fail(ISW_EINVAL, std::string("grid: ") + name + " has an entry after a pad");
    }
    if (a[(size_t)r * width] < 0) fail(ISW_EINVAL, std::string("grid: ") + name + " has an empty row");
  }
}

template <class T>
T *upload(isw_grid *g, const T *host, size_t n) {
  void *p = nullptr;
  ISW_CUDA(cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)));
  g->allocs.push_back(p);
  if (n) ISW_CUDA(cudaMemcpy(p, host, sizeof(T) * n, cudaMemcpyHostToDevice));
  return (T *)p;
}

template <class T>
float *upload_f32(isw_grid *g, const T *host, size_t n) {
  std::vector<float> v(n);
  for (size_t i = 0; i < n; i++) v[i] = (float)host[i];
  return upload(g, v.data(), n);
}

}  // namespace

// The reference's d2_stencil (gpu.py:86-108): per edge end (eI side, then eJ side), four cells (c, j, o1, o2) and their
// weights for the second derivative along the line to the neighbour, scaled by d_e^2 / 12. The operations and their
// order follow the NumPy expression, so the FP64 weights are the reference's bit for bit.
void d2_stencil(const isw_grid_host &h, std::vector<int32_t> &idx, std::vector<double> &wt) {
  const int E = h.E;
  idx.assign((size_t)E * 8, 0);
  wt.assign((size_t)E * 8, 0.0);
  for (int e = 0; e < E; e++)
    for (int side = 0; side < 2; side++) {
      const int c = side == 0 ? h.eI[e] : h.eJ[e];
      const int k = side == 0 ? h.eKi[e] : h.eKj[e];
      const int m = h.deg[c];
      const int j = h.nbr[c * 6 + k];
      const double d1 = h.dist[c * 6 + k];
      const bool hexa = m == 6;
      const int ka = hexa ? (k + 3) % 6 : (k + 2) % m;
      const int kb = hexa ? (k + 3) % 6 : (k + 3) % m;
      const int o1 = h.nbr[c * 6 + ka], o2 = h.nbr[c * 6 + kb];
      const double d2v = hexa ? h.dist[c * 6 + (k + 3) % 6] : 0.5 * (h.dist[c * 6 + ka] + h.dist[c * 6 + kb]);
      const double s = 2 / (d1 + d2v) * h.de[e] * h.de[e] / 12;
      int32_t *I = &idx[(size_t)e * 8 + side * 4];
      double *W = &wt[(size_t)e * 8 + side * 4];
      I[0] = c; I[1] = j; I[2] = o1; I[3] = o2;
      W[0] = -s * (1 / d1 + 1 / d2v);
      W[1] = s / d1;
      W[2] = 0.5 * s / d2v;
      W[3] = 0.5 * s / d2v;
    }
}

}  // namespace isw

using namespace isw;

static isw_grid *grid_create(const isw_grid_host *h, int device) {
  if (!h) fail(ISW_EINVAL, "grid: null descriptor");
  const int N = h->N, E = h->E, NV = h->NV;
  if (N <= 0 || E <= 0 || NV <= 0) fail(ISW_EINVAL, "grid: N, E and NV must be positive");
  need(h->eI, "eI"); need(h->eJ, "eJ"); need(h->nbr, "nbr"); need(h->cellEdge, "cellEdge"); need(h->cellEdgeAsc, "cellEdgeAsc");
  need(h->cellSign, "cellSign"); need(h->ev1, "ev1"); need(h->ev2, "ev2"); need(h->vEdge, "vEdge"); need(h->vCell, "vCell");
  need(h->vEdgeSign, "vEdgeSign"); need(h->vSlot, "vSlot"); need(h->eoeStart, "eoeStart"); need(h->eoe, "eoe");
  need(h->le, "le"); need(h->de, "de"); need(h->areaCell, "areaCell"); need(h->areaV, "areaV"); need(h->fV, "fV");
  need(h->kite, "kite"); need(h->w, "w"); need(h->deg, "deg"); need(h->dist, "dist"); need(h->eKi, "eKi"); need(h->eKj, "eKj");
  check_range(h->eI, E, 0, N, false, "eI");
  check_range(h->eJ, E, 0, N, false, "eJ");
  check_padded_rows(h->nbr, N, 6, N, "nbr");
  check_padded_rows(h->cellEdge, N, 6, E, "cellEdge");
  check_padded_rows(h->cellEdgeAsc, N, 6, E, "cellEdgeAsc");
  check_range(h->ev1, E, 0, NV, false, "ev1");
  check_range(h->ev2, E, 0, NV, false, "ev2");
  check_range(h->vEdge, (size_t)NV * 3, 0, E, false, "vEdge");
  check_range(h->vCell, (size_t)NV * 3, 0, N, false, "vCell");
  for (size_t i = 0; i < (size_t)NV * 3; i++)
    if (h->vSlot[i] < 0 || h->vSlot[i] >= 6) fail(ISW_EINVAL, "grid: vSlot outside [0, 6)");
  if (h->eoeStart[0] != 0) fail(ISW_EINVAL, "grid: eoeStart[0] != 0");
  for (int e = 0; e < E; e++)
    if (h->eoeStart[e + 1] < h->eoeStart[e]) fail(ISW_EINVAL, "grid: eoeStart not ascending");
  for (int e = 0; e < E; e++)
    if (h->eoeStart[e + 1] - h->eoeStart[e] > EOE_MAX) fail(ISW_EINVAL, "grid: a TRiSK row (eoe) longer than 10 edges");
  const int nE2 = h->eoeStart[E];
  check_range(h->eoe, nE2, 0, E, false, "eoe");
  for (int i = 0; i < N; i++)
    if (h->deg[i] < 3 || h->deg[i] > 6) fail(ISW_EINVAL, "grid: deg outside [3, 6]");
  for (int e = 0; e < E; e++) {
    if (h->eKi[e] >= h->deg[h->eI[e]] || h->eKj[e] >= h->deg[h->eJ[e]]) fail(ISW_EINVAL, "grid: eKi/eKj outside the cell's slots");
    // each edge sits at its cells' slots eKi, eKj (the transport stencil relies on it: [eI, eJ, ... | eJ, eI, ...])
    if (h->nbr[h->eI[e] * 6 + h->eKi[e]] != h->eJ[e] || h->nbr[h->eJ[e] * 6 + h->eKj[e]] != h->eI[e])
      fail(ISW_EINVAL, "grid: nbr at eKi/eKj does not name the edge's other cell");
  }
  for (int i = 0; i < N; i++)     // the stencil reads nbr at slots < deg
    for (int k = 0; k < h->deg[i]; k++)
      if (h->nbr[i * 6 + k] < 0) fail(ISW_EINVAL, "grid: nbr pad inside deg");

  std::vector<int32_t> d2i;
  std::vector<double> d2w;
  d2_stencil(*h, d2i, d2w);

  int ndev = 0;
  ISW_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) fail(ISW_EINVAL, "grid: no such CUDA device");
  ISW_CUDA(cudaSetDevice(device));

  isw_grid *g = new isw_grid();
  g->device = device;
  g->n = h->n;
  try {
    GridDev &d = g->d;
    d.N = N; d.E = E; d.NV = NV; d.nE2 = nE2;
    d.eI = upload(g, h->eI, E); d.eJ = upload(g, h->eJ, E);
    {
      std::vector<int32_t> eij((size_t)E * 2);
      for (int e = 0; e < E; e++) { eij[2 * (size_t)e] = h->eI[e]; eij[2 * (size_t)e + 1] = h->eJ[e]; }
      d.eIJ = reinterpret_cast<const int2 *>(upload(g, eij.data(), eij.size()));
    }
    d.nbr = upload(g, h->nbr, (size_t)N * 6);
    d.cellEdge = upload(g, h->cellEdge, (size_t)N * 6);
    d.cellEdgeAsc = upload(g, h->cellEdgeAsc, (size_t)N * 6);
    d.cellSign = upload(g, h->cellSign, (size_t)N * 6);
    d.ev1 = upload(g, h->ev1, E); d.ev2 = upload(g, h->ev2, E);
    d.vEdge = upload(g, h->vEdge, (size_t)NV * 3); d.vCell = upload(g, h->vCell, (size_t)NV * 3);
    d.vEdgeSign = upload(g, h->vEdgeSign, (size_t)NV * 3); d.vSlot = upload(g, h->vSlot, (size_t)NV * 3);
    d.eoeStart = upload(g, h->eoeStart, (size_t)E + 1); d.eoe = upload(g, h->eoe, nE2);
    d.d2idx = upload(g, d2i.data(), d2i.size());
    d.le = upload(g, h->le, E); d.de = upload(g, h->de, E);
    d.areaCell = upload(g, h->areaCell, N); d.areaV = upload(g, h->areaV, NV); d.fV = upload(g, h->fV, NV);
    d.kite = upload(g, h->kite, (size_t)N * 6); d.w = upload(g, h->w, nE2);
    d.d2wt = upload(g, d2w.data(), d2w.size());
    std::vector<double> rA(N), rde(E), rAV(NV);
    for (int i = 0; i < N; i++) rA[i] = 1.0 / h->areaCell[i];
    for (int e = 0; e < E; e++) rde[e] = 1.0 / h->de[e];
    for (int v = 0; v < NV; v++) rAV[v] = 1.0 / h->areaV[v];
    d.rA = upload(g, rA.data(), N); d.rde = upload(g, rde.data(), E); d.rAV = upload(g, rAV.data(), NV);
    d.w32 = upload_f32(g, h->w, nE2); d.d2wt32 = upload_f32(g, d2w.data(), d2w.size());
    d.le32 = upload_f32(g, h->le, E); d.de32 = upload_f32(g, h->de, E); d.rde32 = upload_f32(g, rde.data(), E);
    d.rA32 = upload_f32(g, rA.data(), N); d.rAV32 = upload_f32(g, rAV.data(), NV);
    std::vector<double> rle(E);
    for (int e = 0; e < E; e++) rle[e] = 1.0 / h->le[e];
    d.rle32 = upload_f32(g, rle.data(), E);
    d.kite32 = upload_f32(g, h->kite, (size_t)N * 6);
    // the TRiSK rows padded to EOE_MAX entries per edge (pads: edge 0, weight 0, never summed): rows start on 8-byte
    // (ids, FP32 weights) and 16-byte (FP64 weights) boundaries, so the slow tendency reads them as vectors
    std::vector<int32_t> eoeP((size_t)E * EOE_MAX, 0);
    std::vector<double> wP((size_t)E * EOE_MAX, 0.0);
    for (int e = 0; e < E; e++)
      for (int t = h->eoeStart[e]; t < h->eoeStart[e + 1]; t++) {
        eoeP[(size_t)e * EOE_MAX + (t - h->eoeStart[e])] = h->eoe[t];
        wP[(size_t)e * EOE_MAX + (t - h->eoeStart[e])] = h->w[t];
      }
    d.eoeP = upload(g, eoeP.data(), eoeP.size());
    d.wP = upload(g, wP.data(), wP.size());
    d.wP32 = upload_f32(g, wP.data(), wP.size());
    // the slow tendency's neighbour staging: for each block of THREADS consecutive edges, the distinct edges its TRiSK
    // rows name (ascending), and per edge the position of each row entry in its block's list (pads 0, never read)
    {
      const int nch = (E + THREADS - 1) / THREADS;
      std::vector<int32_t> off(nch + 1, 0), list;
      std::vector<int16_t> loc((size_t)E * EOE_MAX, 0);
      std::vector<int32_t> ids;
      int smax = 0;
      for (int c = 0; c < nch; c++) {
        const int e0 = c * THREADS, e1 = std::min(E, e0 + THREADS);
        ids.assign(eoeP.begin() + (size_t)e0 * EOE_MAX, eoeP.begin() + (size_t)e1 * EOE_MAX);
        std::sort(ids.begin(), ids.end());
        ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
        for (int e = e0; e < e1; e++)
          for (int t = 0; t < h->eoeStart[e + 1] - h->eoeStart[e]; t++)
            loc[(size_t)e * EOE_MAX + t] = (int16_t)(std::lower_bound(ids.begin(), ids.end(), eoeP[(size_t)e * EOE_MAX + t]) - ids.begin());
        list.insert(list.end(), ids.begin(), ids.end());
        off[c + 1] = (int32_t)list.size();
        smax = std::max(smax, (int)ids.size());
      }
      if (smax > 32767) fail(ISW_EINVAL, "grid.create: a block's TRiSK neighbours exceed the staging table's range");
      d.sOff = upload(g, off.data(), off.size());
      d.sList = upload(g, list.data(), list.size());
      d.sLoc = upload(g, loc.data(), loc.size());
      d.sMax = smax;
    }
    g->h_nbr.assign(h->nbr, h->nbr + (size_t)N * 6);
    g->h_cellEdge.assign(h->cellEdge, h->cellEdge + (size_t)N * 6);
    g->h_cellSign.assign(h->cellSign, h->cellSign + (size_t)N * 6);
    g->h_de.assign(h->de, h->de + E);
    g->h_le.assign(h->le, h->le + E);
    g->h_areaCell.assign(h->areaCell, h->areaCell + N);
    g->h_eI.assign(h->eI, h->eI + E);
    g->h_eJ.assign(h->eJ, h->eJ + E);
    double dmin = h->de[0];
    for (int e = 1; e < E; e++) dmin = h->de[e] < dmin ? h->de[e] : dmin;
    g->dmin = dmin;
  } catch (...) {
    for (void *p : g->allocs) cudaFree(p);
    delete g;
    throw;
  }
  return g;
}

extern "C" {

const char *isw_last_error(void) { return isw::last_error(); }

int isw_version(void) { return 100; }

int isw_grid_create(const isw_grid_host *g, int device, isw_grid **out) {
  try {
    if (!out) fail(ISW_EINVAL, "grid: null output handle");
    *out = grid_create(g, device);
    return ISW_OK;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("grid: host allocation failed");
    return ISW_ENOMEM;
  }
}

int isw_grid_destroy(isw_grid *g) {
  if (!g) return ISW_OK;
  cudaSetDevice(g->device);
  for (void *p : g->allocs) cudaFree(p);
  delete g;
  (void)cudaGetLastError();         // a failure while freeing must not surface in the caller's next call
  return ISW_OK;
}

}  // extern "C"
