// Shared-memory tiles for the barotropic fast loop.
//
// The fast loop (reference layers.cu:366-388, driven by layers.py:168-175) alternates a cell pass (eta) and an edge pass
// (ubar) ceil(c nfast) times per stage. Each tile owns a compact region of cells (grown breadth-first from a seed, the
// smallest region growing first, so regions are compact and within a few cells of equal size) and the edges whose eI
// cell it owns; it stages in shared memory its cells out to k rings (ring 0 = owned) and every edge of those cells. It
// can then advance k sub-steps with no grid-wide sync: sub-step m (1..k) updates eta on cells of ring <= k - m + 1
// and ubar on edges whose nearer cell has ring <= k - m, which is exactly what the owned values after k sub-steps
// depend on. Tiles exchange owned eta and ubar through global memory every k sub-steps (double-buffered, one grid
// barrier per exchange). Arithmetic is the reference's, per cell and edge, in the same gather order.
//
// Local numbering: cells in ring order, edges in order of their nearer cell's ring with the owned edges first, so
// "ring <= r" is a prefix and the owned edges are [0, eown).
#pragma once
#include <stdint.h>

#include <vector>

namespace isw {

struct TileSetHost {
  int P = 0, k = 0;
  size_t smem = 0;                             // dynamic shared memory of the largest tile
  std::vector<int32_t> cell_off, edge_off;     // P + 1 offsets
  std::vector<int32_t> cells, edges;           // global ids, tile by tile, local order
  std::vector<int32_t> ncnt, ecnt;             // per tile k + 1 prefix counts: cells of ring <= r, edges of ring <= r
  std::vector<int32_t> eown;                   // per tile: owned edges (eI owned), the first of the local edges
  std::vector<int16_t> cedge;                  // per local cell 8 slots: +-(local edge + 1), sign = cellSign; 0 pads
  std::vector<int16_t> eIl, eJl;               // per local edge its local cells (-1 outside the tile)
};

// Per-tile shared-memory bytes. FP64 form: per cell eta, Y = Gc (eta + gamma (eta - eta_prev)), area, Gc (8 B each) and
// its 8 signed local edge ids (16 B); per edge (l_e H_e, ubar) and (G, d_e) (16 B each) and its two local cell ids
// (4 B); per owned edge the sub-step sum acc (8 B); 64 B of alignment slack.
inline size_t tile_smem_bytes(size_t nc, size_t ne, size_t nown) { return nc * (4 * 8 + 16) + ne * (2 * 16 + 4) + nown * 8 + 64; }
// The mixed form's tile: per cell deta, Y, 1/area, Gc, c0 (4 B each) and the edge ids (16 B); per edge dub, its flux,
// l_e H_e, G', 1/d_e (4 B each) and the cell ids (4 B); the owned edges' sums live in registers.
inline size_t tile_smem_bytes_mixed(size_t nc, size_t ne, size_t) { return nc * (5 * 4 + 16) + ne * (5 * 4 + 4) + 64; }

// Compact balanced partition of the N cells into P regions (owner per cell).
std::vector<int32_t> partition_cells(int N, const int32_t *nbr, int P);

// Build the tiles of a partition over a grid (neighbour table nbr (N x 6, pads -1), cellEdge and cellSign (N x 6),
// eI, eJ (E)).
TileSetHost build_tiles(int N, int E, const int32_t *nbr, const int32_t *cellEdge, const int8_t *cellSign, const int32_t *eI,
                        const int32_t *eJ, const std::vector<int32_t> &owner, int P, int k);

}  // namespace isw
