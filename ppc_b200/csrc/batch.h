// Batched propagation: thousands of events with uneven photon counts in one persistent,
// work-stealing launch, replayed from a CUDA graph, with per-event hit regions sized from
// an upper-bound estimate and an autotuned launch shape.  No counterpart in the reference,
// which runs one source per eout() (gpu/f2k.cxx:536-541, gpu/ppc.cu:432-469).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace ppcb {

struct BatchResult {
  std::vector<uint32_t> produced;   // hits produced per event
  std::vector<uint64_t> offset;     // per event: first hit in `hits` (events x+1)
  std::vector<ppcb_hit> hits;       // kept hits, grouped by event
  uint64_t photons = 0, steps = 0;
  uint32_t overflowed = 0;          // events whose region was too small
  float device_ms = 0;              // propagation kernel
  float graph_ms = 0;               // whole graph: uploads, kernel, compaction, downloads
};

struct TuneResult {
  int threads = 256, blocks_per_sm = 3, refill_below = 0;
  double photons_per_s = 0;
  std::vector<std::string> log;
};

class Batch {
 public:
  Batch(Engine& e, int device, uint32_t max_events, uint32_t max_bunches, uint64_t hit_capacity);
  ~Batch();
  // Bunch .q fields are event indices in [0, events).  `hits_per_photon` is the upper
  // bound used to size each event's hit region (plus `hit_slack` slots).
  void run(const ppcb_bunch* b, int nb, uint32_t events, BatchResult& out, double hits_per_photon,
           uint32_t hit_slack = 64);
  // Times the candidate launch shapes on a sample of the batch and keeps the fastest.
  TuneResult autotune(const ppcb_bunch* b, int nb, uint32_t events, uint64_t sample_photons);
  bool use_graph = true;

 private:
  void capture();
  void release_graph();
  Engine& eng_;
  int d_;
  int cuda_dev_ = -1;  // the CUDA device of the buffers (frees them without the engine)
  uint32_t maxE_, maxB_;
  uint64_t hcap_;
  cudaStream_t st_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  cudaEvent_t k0_ = nullptr, k1_ = nullptr, g0_ = nullptr, g1_ = nullptr;
  // device
  ppcb_bunch* bunches_ = nullptr;
  uint64_t* bstart_ = nullptr;
  uint64_t* ev_off_ = nullptr;
  uint32_t* ev_cap_ = nullptr;
  unsigned int* ev_cnt_ = nullptr;
  uint64_t* dyn_ = nullptr;          // num, nb, events
  ppcb_hit* hits_ = nullptr;
  ppcb_hit* out_ = nullptr;
  uint64_t* out_off_ = nullptr;
  ppcb_ctrl* ctrl_ = nullptr;
  // pinned host
  ppcb_bunch* h_bunches_ = nullptr;
  uint64_t* h_bstart_ = nullptr;
  uint64_t* h_ev_off_ = nullptr;
  uint32_t* h_ev_cap_ = nullptr;
  unsigned int* h_ev_cnt_ = nullptr;
  uint64_t* h_dyn_ = nullptr;
  uint64_t* h_out_off_ = nullptr;
  ppcb_ctrl* h_ctrl_ = nullptr;
};

}  // namespace ppcb
