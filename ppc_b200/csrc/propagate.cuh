// Kernel-facing declarations shared by the launch code and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ppcb_types.h"
#include "strgrid.h"

namespace ppcb {

// Per-launch arguments, passed as a __grid_constant__ kernel parameter (constant bank).
struct KArgs {
  ppcb_params p;
  // read-only tables in HBM
  const float2* absca;       // [WNUM][size] (abs, sca)
  const ppcb_wmeta* wmeta;   // [WNUM]
  const float2* lp;          // [LMAX][LYRS] tilt maps
  const ppcb_dom* oms;       // [gsize]
  const ppcb_aniz* az;       // [size]        -> shared memory
  const ppcb_line* sc;       // [nstr]        -> shared memory
  const float* lr;           // [LMAX]        -> shared memory
  const uint16_t* ls;        // [NSTR]        -> shared memory
  const uint16_t* is;        // [CX*CY]       -> shared memory
  const int8_t* mcol;        // [CTX*CTY]     -> shared memory
  const float4* bfrt;        // [BFR_TAB+1]   -> shared memory
  StrGridParams sg;          // string-proximity table (strgrid.h); sg.on = 0: no strings
  const StrGroup* sg_groups; // [sg_ngroups]  -> shared memory
  int sg_ngroups;
  const uint16_t* sg_cells;  // [nx*ny]       -> shared memory (dynamic)
  // work
  const ppcb_bunch* bunches; // [nb]
  const uint64_t* bstart;    // [nb+1] first photon index of each bunch (exclusive prefix sum)
  int nb;
  uint64_t num;              // photons in this launch
  // random streams, one per thread slot
  uint64_t* rs;              // [threads] MWC state
  const uint32_t* rm;        // [threads] multipliers
  // output
  ppcb_hit* hits;
  uint64_t hcap;
  ppcb_ctrl* ctrl;
  // options
  int deterministic;         // 0: dynamic photon order; 1: photon i runs on thread i % threads
                             // (static order); 2: dynamic, photon i draws from its own stream (seed, i)
  uint32_t seed;             // per-photon stream seed
  uint32_t max_steps;        // 0: unlimited; else photons stopped after this many steps
  int refill_below;          // photon pool: the warp also resamples when fewer than this are left
  // batched launches (optional, all null otherwise)
  const uint64_t* dyn;       // {num, nb} read by the kernel at start (graph replays)
  const uint64_t* ev_off;    // per event: first slot of its hit region in `hits`
  const uint32_t* ev_cap;    // per event: slots in its region
  unsigned int* ev_cnt;      // per event: hits produced (may exceed ev_cap)
  // gradient (optional): recording pass writes 64-byte provenance records here, one per hit slot
  void* prov;
};

// Launch shape chosen by the host.
struct LaunchShape {
  int blocks;
  int threads;
};

// Kernel entry points (defined in propagate.cu).
cudaError_t launch_propagate(const KArgs& a, LaunchShape s, cudaStream_t st);
cudaError_t launch_generate(const KArgs& a, LaunchShape s, void* pbuf_out, cudaStream_t st);
cudaError_t launch_index_probe(const KArgs& a, const float4* pos, int n, int32_t* out_i, float* out_f,
                               cudaStream_t st);
// Charges are binned per DOM, or with events > 0 per (event, DOM), the event being the
// hit's segment id (bin = event * gsize + DOM; hits of segments >= events are left out).
// With nh_dev (a device pointer to the recording pass's hit count) the kernels read how many
// hits there are at run time, up to nh: a graph replay then needs no host round trip.
cudaError_t launch_adjoint(const KArgs& a, const ppcb_hit* hits, const void* prov, uint64_t nh, uint32_t events,
                           const float* wdom, const float2* wgrad, double* g_out, unsigned int* stats, int blocks,
                           cudaStream_t st, const unsigned long long* nh_dev = nullptr);
cudaError_t launch_dom_hist(const ppcb_hit* hits, uint64_t nh, unsigned int* counts, uint32_t events, int gsize,
                            cudaStream_t st, const unsigned long long* nh_dev = nullptr);
cudaError_t adjoint_prepare();  // the replay's launch attribute on the current device (before a capture)
constexpr size_t kProvBytes = 64;  // provenance record per hit slot of the gradient's recording pass
cudaError_t propagate_attributes(int* regs, int* max_threads, size_t* smem, size_t* local);
int propagate_max_blocks_per_sm(int threads);
int propagate_rec_blocks_per_sm(int threads, int deterministic);

}  // namespace ppcb
