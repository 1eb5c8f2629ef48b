// DirectFit's likelihood of simulated against observed DOM pulses (llh/llh.cxx:419-662,
// 1075-1082): the observed side is prepared once per event on the host (llh.cpp), the
// simulated side is accepted, binned and reduced on the GPU (llh.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "../../include/ppc_b200.h"

namespace ppcb {

class Engine;

// One DOM that enters the likelihood (dat::in(), llh/llh.cxx:664-666), after dat::prep and
// dat::optimize (llh/llh.cxx:436-450, 516-612).
struct LlhDom {
  int32_t str, om;
  int32_t n1, n2;    // bins [n1, n2) take part
  int32_t block0;    // its first block in the block list
  int32_t nblock;
  int32_t bin0;      // offset of its bin n1 in the bin -> block table
  int32_t win0;      // its excluded windows
  int32_t nwin;
  int32_t pad_;
  double dtot;       // observed charge in bins [0, 200) outside the windows
};

struct LlhDevice;  // device buffers (llh.cu)
struct LlhDeviceFree {
  void operator()(LlhDevice* p) const;  // frees the buffers (llh.cu)
};

class Likelihood {
 public:
  static constexpr int kBins = 200;     // num (llh/llh.cxx:43)
  static constexpr double kBin = 25.0;  // bin (llh/llh.cxx:46)

  Likelihood(Engine& e, int device, const ppcb_llh_hit* data, uint64_t n, const ppcb_llh_window* win,
             uint64_t nwin, const int32_t* bad, uint64_t nbad, const ppcb_llh_opts& o);
  ~Likelihood();

  // out[j] = fllh(dts[j], nsim) over the accepted hits among dhits[0..n) (device pointers;
  // dout receives ndt doubles), on stream st
  void eval_device(const ppcb_hit* dhits, uint64_t n, uint32_t seed, const double* dts, int ndt, double nsim,
                   double* dout, cudaStream_t st);
  int errors();  // llf evaluations that left their domain, since creation (synchronises)
  void require_device();  // throws (status 6) before ppcb_ini(); uploads the tables

  ppcb_llh_opts opts;
  double lbin = 0, t0 = 0;
  int ndof = 1;
  std::vector<LlhDom> doms;              // in (str, om) order
  std::vector<ppcb_llh_block> blocks;    // each DOM's blocks from its last bin backwards
  std::vector<int32_t> block_dom;        // block -> index into doms
  std::vector<int32_t> bin_block;        // per DOM, per bin in [n1, n2): block index
  std::vector<double> win;               // (ti, tf) pairs of the DOMs' windows
  std::vector<int32_t> dom_slot;         // per sensor index: index into doms; -1 no observed
                                         // pulses (the no-hit term); -2 left out

 private:
  Engine& eng_;
  int dev_;
  int cuda_dev_ = -1;  // the CUDA device the tables live on (frees them without the engine)
  std::unique_ptr<LlhDevice, LlhDeviceFree> d_;
  void upload();
};

}  // namespace ppcb
