// Device runtime: per-GPU table image in HBM, random streams, double-buffered launch
// slots, hit collection.  Replaces the reference's `struct gpu` and kernel()
// (gpu/ppc.cu:102-321, :432-469) with a depth-2 pipeline: batch k is queued before the
// host waits for batch k-1, so the GPU is never idle between batches.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <deque>
#include <memory>
#include <string>
#include <functional>
#include <vector>

#include "config.h"
#include "propagate.cuh"

namespace ppcb {

struct RunInfo {
  uint64_t photons = 0;
  uint64_t hits = 0;        // produced by the kernel (may exceed what was kept)
  uint64_t kept = 0;        // stored (bounded by the hit-buffer capacity)
  uint64_t steps = 0;
  uint32_t nan_steps = 0;
  uint32_t capped = 0;
  float device_ms = 0;
  bool overflow = false;
};

struct BackendTables;  // the device back end's sensor tables (backend.cu)
struct FrontScratch;   // the device front end's per-source buffers (frontend.cu)

struct DeviceCtx {
  int dev = -1;
  cudaDeviceProp prop{};
  cudaStream_t st = nullptr, cp = nullptr;
  LaunchShape shape{0, 0};
  int T = 0;                      // threads in flight (= random streams)
  // table image
  float2* absca = nullptr;
  ppcb_wmeta* wmeta = nullptr;
  float2* lp = nullptr;
  ppcb_dom* oms = nullptr;
  ppcb_aniz* az = nullptr;
  ppcb_line* sc = nullptr;
  float* lr = nullptr;
  uint16_t* ls = nullptr;
  uint16_t* is = nullptr;
  int8_t* mcol = nullptr;
  float4* bfrt = nullptr;
  StrGroup* sg_groups = nullptr;   // string-proximity table (strgrid.h)
  uint16_t* sg_cells = nullptr;
  uint64_t* rs = nullptr;
  uint32_t* rm = nullptr;
  struct Slot {
    ppcb_bunch* bunches = nullptr;   // device
    uint64_t* bstart = nullptr;      // device
    ppcb_bunch* hb = nullptr;        // pinned staging
    uint64_t* hbstart = nullptr;     // pinned staging
    ppcb_hit* hits = nullptr;        // device
    ppcb_ctrl* ctrl = nullptr;       // device
    ppcb_ctrl* hctrl = nullptr;      // pinned
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    uint64_t num = 0;
    int nb = 0;
    bool busy = false;
    long tag = 0;
  } slot[2];
  int next_slot = 0;
  uint64_t bcap = 0, hcap = 0;
  double device_ms = 0;
  ppcb_hit* hhits = nullptr;       // pinned, grows
  uint64_t hhits_cap = 0;
  std::shared_ptr<BackendTables> back;  // built on the first device back-end call
  std::shared_ptr<FrontScratch> front;  // grows to the largest device front-end call
};

struct GradScratch;  // the gradient's device buffers (gradient.cu), kept between calls

class Engine {
 public:
  ~Engine();
  Config cfg;
  unsigned int sv = 0;             // seed: MWC stream start and host rand_r state
  int deterministic = 0;           // 0 dynamic order, 1 static order (thread streams), 2 dynamic + per-photon streams
  uint32_t max_steps = 1000000;     // per-photon step cap (typical photons take 20-100 steps)
  std::vector<DeviceCtx> devs;
  uint64_t pmax = 0, pmxo = 0;     // photons / bunches per launch
  unsigned int hquo = 1;
  int blocks_per_sm = 0;           // 0: occupancy maximum
  int threads_per_block = 864;     // 128, 256, 768 or 864 (compiled shapes of the kernel)
  int refill_below = 0;            // photon pool refill threshold (0: refill on demand)

  void initialize(const std::string& dir, float enh);
  void choose(int device);         // -1: every visible device
  void ini();
  void fin();
  bool ready() const { return inited_; }

  // Queue one batch (bunch list with photon counts) on every device; the photon range
  // is split across devices in proportion to capacity (gpu/ppc.cu:313-320, :450-457).
  long submit(const ppcb_bunch* b, int nb, uint64_t num);
  // Wait for the oldest queued batch; append its kept hits.  False if none queued.
  bool collect(std::vector<ppcb_hit>& out, RunInfo& info, long* tag = nullptr);
  // The same, handing each device's kept hits to `sink` straight from the pinned staging
  // buffer (valid during the call only).
  bool collect(const std::function<void(const ppcb_hit*, uint64_t)>& sink, RunInfo& info, long* tag = nullptr);
  int in_flight() const { return (int)queue_.size(); }

  // Device-pointer entry point: one launch on device `d` over caller buffers.
  void launch_device(int d, const ppcb_bunch* dbunch, const uint64_t* dbstart, int nb, uint64_t num,
                     ppcb_hit* dhits, uint64_t hcap, ppcb_ctrl* dctrl, cudaStream_t st);
  void reset_streams();            // re-seed every stream (reference rs_ini, gpu/ini.cxx:556-571)
  // New per-layer be/ba (file order, null keeps): rebuilds and re-uploads the ice table.
  void set_ice(const float* be, const float* ba);

  struct Grad {
    double ll = 0;                   // Poisson log-likelihood sum_d (k_d log mu_d - mu_d) over DOMs with mu_d > 0
    std::vector<uint32_t> counts;    // simulated hits per charge bin
    std::vector<double> g_be, g_ba;  // d/d be_j, d/d ba_j in file order (icemodel.dat rows)
    uint64_t photons = 0, hits = 0, replayed = 0, unmatched = 0, steps = 0;
    float forward_ms = 0, backward_ms = 0;
  };
  // Gradient of sum_d w_d mu_d, mu_d = scale x (simulated hits in charge bin d), with respect
  // to the 2 x size ice coefficients.  The bins are the DOMs (events = 0) or the (event, DOM)
  // pairs, event = hit segment id < events.  With `observed` (per bin) w_d = dLL/dmu_d of the
  // Poisson log-likelihood; otherwise `weights` (per bin) are used as given.  One recording
  // forward launch over the bunches (device 0) and one replay of the recorded hits.
  Grad gradient(const ppcb_bunch* b, int nb, uint32_t events, const float* observed, const float* weights,
                double scale, uint64_t hit_cap);
  // Hit back end on device `d` (gpu/f2k.cxx:247-363 acceptance, one random stream per hit):
  // accepted hits of dhits[0..n) written to dout in input order, their number to *dcount
  // (device pointer), on stream st.  Standard sensors only.
  void accept(int d, const ppcb_hit* dhits, uint64_t n, uint32_t seed, ppcb_acc_hit* dout,
              unsigned long long* dcount, cudaStream_t st);
  // Device front end on device `d`: sources to bunches (gpu/f2k.cxx:17-167, 377-528),
  // one random stream per source; counts[0..1] (device) receive bunches needed and photons.
  void sources(int d, const ppcb_source* dsrc, uint64_t ns, uint32_t seed, ppcb_bunch* dout, uint64_t* dbstart,
               uint64_t cap, uint64_t* dcounts, cudaStream_t st);
  int front_errors(int d);  // sources whose sampling failed, since ini (synchronises)
  // The back end's tables on device `d` (built from the configuration on first use).
  BackendTables& backend_tables(int d);
  double total_device_ms() const;
  KArgs args_for(int d) const;

 private:
  void free_device(DeviceCtx& g);
  std::shared_ptr<GradScratch> gs_;  // grows to the largest gradient call; freed by fin()
  bool inited_ = false;
  bool initialized_ = false;
  std::deque<long> queue_;
  long tag_ = 0;
};

void check(cudaError_t e, const char* what);

// One ice-fit iteration as a CUDA graph (gradient.cu): the recording forward pass, the charge
// histogram, the Poisson weights and log-likelihood, and the replay of the detected photons
// over fixed bunches and observed charges, captured once on device 0 and replayed per call
// with new ice coefficients.  Hit counts stay on the device between the steps.
struct GradGraphState;
class GradGraph {
 public:
  GradGraph(Engine& e, const ppcb_bunch* b, int nb, uint32_t events, const float* observed, double scale,
            uint64_t hit_cap);
  ~GradGraph();
  // New be/ba (file order; null keeps), then one replay: LL, gradient, charges, timings.
  Engine::Grad run(const float* be, const float* ba, bool counts = true);
  GradGraph(const GradGraph&) = delete;
  GradGraph& operator=(const GradGraph&) = delete;

 private:
  Engine& e_;
  std::unique_ptr<GradGraphState> s_;
};

}  // namespace ppcb
