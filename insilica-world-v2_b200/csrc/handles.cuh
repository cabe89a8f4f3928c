// Library-side definitions of the Layers and Transport handles (shared by the per-call path and the batched step).
#pragma once
#include <list>
#include <vector>

#include "common.cuh"
#include "transport_fp64.cuh"

struct GraphEntry {
  const double *h, *u, *Fm;
  double dt;
  int nfast;
  cudaGraphExec_t exec;
};

struct isw_layers {
  isw_grid *grid;
  isw::LayersDev d;
  std::vector<void *> allocs;
  cudaStream_t cap;                 // private stream the step graphs are captured on
  std::list<GraphEntry> graphs;     // most recent first
  int colmax_blocks;
  int *nonfinite;
};

struct isw_transport {
  isw_grid *grid;
  isw::TransportDev d;
  int L, T, precision;
  double beta;
  std::vector<void *> allocs;
};
