// Library-side definitions of the Layers and Transport handles (shared by the per-call path and the batched step).
#pragma once
#include <list>
#include <vector>

#include "common.cuh"
#include "transport_fp64.cuh"

struct GraphEntry {
  const double *h, *u, *Fm, *theta;
  double dt;
  int nfast;
  cudaGraphExec_t exec;
};

struct isw_batch;

struct isw_layers {
  isw_grid *grid;
  int device = 0;                   // the grid's device (kept here so that destroy reads nothing of the grid)
  isw::LayersDev d;
  std::vector<void *> allocs;
  cudaStream_t cap;                 // private stream the step graphs are captured on
  std::list<GraphEntry> graphs;     // most recent first
  int colmax_blocks;
  int *nonfinite;
  double nu4dt = 0;                 // nu4 dt of the last step (the exchange books the step's nabla^4 loss as heat)
  int version = 0;                  // bumped when an option is set: batches holding the stack rebuild its descriptor
  bool percall = false;             // FP64: step with the per-call kernels instead of the private batch
  // the mixed form steps call by call through a private one-stack batch (its step graph and tiles)
  isw_batch *solo = nullptr;
  int solo_slot = -1;
  GraphEntry solo_key{};
  double *solo_Fm = nullptr;        // Fm when the caller passes none
};

struct isw_transport {
  isw_grid *grid;
  int device = 0;                   // the grid's device (kept here so that destroy reads nothing of the grid)
  isw::TransportDev d;
  int L, T, precision;
  double beta;
  std::vector<void *> allocs;
};
