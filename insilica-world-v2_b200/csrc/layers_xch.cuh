// The between-step exchange hook (reference layers.py:214-232, Layers.exchange; kernels/layers.cu:452-545).
//
// A column (a cell, or an edge with the mean of its two cells) exchanges thickness across its L - 1 interfaces:
// v[k] > 0 moves v[k] up across the interface below layer k (layer k + 1 gives, layer k receives), v[k] < 0 moves it
// down. What the moved thickness carries is the donor's: tracer concentration in cells, wind on edges. Everything is
// a transfer between two neighbouring layers, so the column totals (volume, tracer mass, momentum) are exact.
//
// Two orders of the transfers:
//  - all at once (cells, seq = 0): every transfer carries its donor's value from before the exchange; a layer's change
//    is the transfer through its floor minus the transfer through its ceiling (flux form);
//  - in flow order (cells with seq = 1, and always on edges): rising transfers from the deepest interface up, then
//    sinking transfers from the top interface down, each carrying its donor's value as the earlier transfers left it, so
//    thickness that passes through a layer carries what it picked up on the way.
// Edges also hand back the kinetic energy the momentum mixing removes (plus the step's nabla^4 loss when asked), and
// for air a nearly empty layer is pulled toward its neighbours' wind. Plain FP64 compiled with -fmad=false; every
// rounding is the reference's own, so results are bit-identical to it.
#pragma once
#include "common.cuh"

namespace isw {
namespace fp64 {
namespace xch {

// The interfaces of a column in flow order: rising transfers bottom-up, then sinking ones top-down. Interfaces that
// move nothing (v == 0, or NaN) are skipped.
template <int L, class Visit>
__device__ __forceinline__ void in_flow_order(const double (&v)[L], Visit &&visit) {
  for (int k = L - 2; k >= 0; k--)
    if (v[k] > 0) visit(k);
  for (int k = 0; k + 1 < L; k++)
    if (v[k] < 0) visit(k);
}

// Layer k + 1 is the donor of a rising transfer across interface k, layer k of a sinking one.
__device__ __forceinline__ int donor(double v, int k) { return v > 0 ? k + 1 : k; }

// Net gain of layer j from the transfers through its ceiling (interface j - 1) and floor (interface j), given per
// interface: the floor's transfer adds, the ceiling's subtracts; the top and bottom layers have one interface.
template <int L>
__device__ __forceinline__ double net_gain(const double (&through)[L], int j) {
  const double ceiling = j > 0 ? through[j - 1] : 0.0;
  const double floor_in = j + 1 < L ? through[j] : 0.0;
  return (0.0 - ceiling) + floor_in;
}

}  // namespace xch

// One cell: thickness h, mass M and the tracer psi of every layer, moved by wx (L - 1 rows of N).
template <int L>
__device__ __forceinline__ void xch_cell(const LayersDev &M, const double *__restrict__ wx, double *__restrict__ h,
                                         double *__restrict__ Mm, double *__restrict__ psi, int seq, int i) {
  const int N = M.g.N;
  const double area = M.g.areaCell[i];
  double v[L], mass0[L], conc0[L];
#pragma unroll
  for (int k = 0; k < L; k++) {
    v[k] = k + 1 < L ? wx[(size_t)k * N + i] : 0.0;
    mass0[k] = Mm[(size_t)k * N + i];
    conc0[k] = psi[(size_t)k * N + i];
  }
  if (!seq) {
    // every transfer at its donor's concentration from before: per interface the volume and tracer mass moved
    double vol[L], load[L];
#pragma unroll
    for (int k = 0; k + 1 < L; k++) {
      vol[k] = v[k] * area;
      load[k] = vol[k] * conc0[xch::donor(v[k], k)];
    }
#pragma unroll
    for (int j = 0; j < L; j++) {
      const size_t o = (size_t)j * N + i;
      const double dmass = xch::net_gain<L>(vol, j), dload = xch::net_gain<L>(load, j);
      const double mass1 = mass0[j] + dmass;
      psi[o] = (mass0[j] * conc0[j] + dload) / mass1;
      Mm[o] = mass1;
      h[o] = h[o] + dmass / area;
    }
    return;
  }
  // flow order: mass and tracer mass per layer, each transfer at the donor's concentration as it stands
  double mass[L], tracer[L];
#pragma unroll
  for (int k = 0; k < L; k++) {
    mass[k] = mass0[k];
    tracer[k] = mass0[k] * conc0[k];
  }
  xch::in_flow_order<L>(v, [&](int k) {
    const int d = xch::donor(v[k], k);
    const double vol = v[k] * area, c = tracer[d] / mass[d];
    mass[k] += vol;
    mass[k + 1] -= vol;
    tracer[k] += vol * c;
    tracer[k + 1] -= vol * c;
  });
#pragma unroll
  for (int j = 0; j < L; j++) {
    const size_t o = (size_t)j * N + i;
    h[o] = h[o] + (mass[j] - mass0[j]) / area;
    Mm[o] = mass[j];
    psi[o] = tracer[j] / mass[j];
  }
}

// One edge: every layer's wind u, with the edge thicknesses from before the exchange (hold, the mean of the two cells)
// and the moves wx averaged onto the edge; column momentum sum h_e u is conserved. diss (or null) receives the
// kinetic energy removed, 0.5 sum h_e u^2 before minus after, plus nu4dt sum h_e u lap4 when lap4 is given. hthin > 0
// (air): a layer whose thinner cell holds less than hthin takes part of its neighbours' mass-weighted wind.
template <int L>
__device__ __forceinline__ void xch_edge(const LayersDev &M, const double *__restrict__ wx, const double *__restrict__ hold,
                                         double *__restrict__ u, double *__restrict__ diss, const double *__restrict__ lap4,
                                         double nu4dt, double hthin, int e) {
  const GridDev &g = M.g;
  const int N = g.N, E = g.E;
  const size_t a = g.eI[e], b = g.eJ[e];
  const double hfloor = M.floor_;
  double thick[L], mom[L], wind0[L], hmin[L], v[L];
  double ke_before = 0, visc = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    const double ha = hold[(size_t)k * N + a], hb = hold[(size_t)k * N + b];
    wind0[k] = u[(size_t)k * E + e];
    thick[k] = 0.5 * (ha + hb);
    hmin[k] = fmin(ha, hb);
    mom[k] = thick[k] * wind0[k];
    ke_before += mom[k] * wind0[k];
    if (lap4) visc += mom[k] * lap4[(size_t)k * E + e];
    v[k] = k + 1 < L ? 0.5 * (wx[(size_t)k * N + a] + wx[(size_t)k * N + b]) : 0.0;
  }
  // a donor's wind is its momentum over its thickness while it holds more than the floor, else its wind from before
  xch::in_flow_order<L>(v, [&](int k) {
    const int d = xch::donor(v[k], k);
    const double carried = v[k] * (thick[d] > hfloor ? mom[d] / thick[d] : wind0[d]);
    mom[k] += carried;
    mom[k + 1] -= carried;
    thick[k] += v[k];
    thick[k + 1] -= v[k];
  });
  double wind[L];
#pragma unroll
  for (int k = 0; k < L; k++) wind[k] = mom[k] / thick[k];
  if (hthin > 0) {
    // a nearly empty layer: pull its wind toward the neighbours' mass-weighted wind, by how far it is below hthin (all
    // the way at the floor), at most to the mean of it and its neighbours; the neighbours pay its momentum change
    for (int k = 0; k < L; k++) {
      if (hmin[k] >= hthin) continue;
      const bool up = k > 0, down = k + 1 < L;
      double nthick = 0.0, nmom = 0.0;          // the neighbours' thickness and momentum, the layer above first
      if (up) {
        nthick += thick[k - 1];
        nmom += thick[k - 1] * wind[k - 1];
      }
      if (down) {
        nthick += thick[k + 1];
        nmom += thick[k + 1] * wind[k + 1];
      }
      if (nthick <= 0) continue;
      const double reach = (hthin - hmin[k]) / (hthin - hfloor);
      const double pull = fmin(reach > 1 ? 1.0 : reach, nthick / (thick[k] + nthick));
      const double dwind = pull * (nmom / nthick - wind[k]);
      wind[k] += dwind;
      const double back = thick[k] * dwind / nthick;
      if (up) wind[k - 1] -= back;
      if (down) wind[k + 1] -= back;
    }
  }
  const bool closed = M.wall && M.wall[e] == 0;    // thin walls: the wind across a closed edge stays zero
  double ke_after = 0;
#pragma unroll
  for (int k = 0; k < L; k++) {
    u[(size_t)k * E + e] = closed ? 0.0 : wind[k];
    ke_after += thick[k] * wind[k] * wind[k];
  }
  if (diss) diss[e] = 0.5 * (ke_before - ke_after) + nu4dt * visc;
}

}  // namespace fp64
}  // namespace isw
