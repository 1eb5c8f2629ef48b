// Ice-model gradient (Engine::gradient, Engine::set_ice).  No counterpart in the reference:
// llh/DirectFit fits the ice by repeated forward runs (llh/llh.cxx:1435-1634); here the
// gradient of the likelihood with respect to all 2 x 171 per-layer coefficients comes from
// one recording forward pass and a replay of the detected photons (propagate.cu, AdjHook).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "engine.h"

namespace ppcb {

void Engine::set_ice(const float* be, const float* ba) {
  cfg.set_ice(be, ba);
  if (!inited_) return;
  for (auto& g : devs) {
    check(cudaSetDevice(g.dev), "cudaSetDevice");
    check(cudaMemcpy(g.absca, cfg.absca.data(), cfg.absca.size() * sizeof(float), cudaMemcpyHostToDevice),
          "ice table");
  }
}

namespace {
// device buffer that keeps its memory between calls and grows when a call needs more
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  void need(size_t n) {
    n = std::max<size_t>(n, 1);
    if (n <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    check(cudaMalloc((void**)&p, n * sizeof(T)), "gradient buffer");
    cap = n;
  }
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { if (p) cudaFree(p); }
};
}  // namespace

struct GradScratch {
  DBuf<ppcb_bunch> bunches;
  DBuf<uint64_t> bstart;
  DBuf<ppcb_hit> hits;
  DBuf<unsigned char> prov;
  DBuf<ppcb_ctrl> ctrl;
  DBuf<unsigned int> counts;
  DBuf<float> weights;
  DBuf<float2> wgrad;
  DBuf<double> g;
  DBuf<unsigned int> stats;
  cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
  GradScratch() {
    for (auto& x : e) check(cudaEventCreate(&x), "event");
  }
  ~GradScratch() {
    for (auto& x : e) if (x) cudaEventDestroy(x);
  }
};

Engine::Grad Engine::gradient(const ppcb_bunch* b, int nb, uint32_t events, const float* observed,
                              const float* weights, double scale, uint64_t hit_cap) {
  if (!inited_) throw Error("ini() must come before the gradient", 6);
  if (nb <= 0) throw Error("no bunches", 7);
  if (!observed && !weights) throw Error("gradient: observed counts or DOM weights required", 7);
  DeviceCtx& g = devs[0];
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  const int gsize = cfg.p.gsize, size = cfg.p.size;
  const size_t nbins = (size_t)gsize * (events ? events : 1);  // charge bins: DOM, or (event, DOM)
  std::vector<uint64_t> bs(nb + 1, 0);
  for (int k = 0; k < nb; k++) bs[k + 1] = bs[k] + b[k].num;
  if (!gs_) gs_ = std::make_shared<GradScratch>();
  GradScratch& X = *gs_;
  X.bunches.need(nb);
  X.bstart.need(nb + 1);
  X.hits.need(hit_cap);
  X.prov.need(hit_cap * kProvBytes);
  X.ctrl.need(1);
  X.counts.need(nbins);
  X.weights.need(nbins);
  X.wgrad.need(PPCB_WNUM);
  X.g.need(2 * PPCB_MAXLYS);
  X.stats.need(2);
  auto& db = X.bunches;
  auto& dbs = X.bstart;
  auto& dh = X.hits;
  auto& dprov = X.prov;
  auto& dctrl = X.ctrl;
  auto& dcnt = X.counts;
  auto& dw = X.weights;
  auto& dwg = X.wgrad;
  auto& dgo = X.g;
  auto& dstat = X.stats;
  cudaStream_t st = g.st;
  check(cudaMemcpyAsync(db.p, b, nb * sizeof(ppcb_bunch), cudaMemcpyHostToDevice, st), "H2D bunches");
  check(cudaMemcpyAsync(dbs.p, bs.data(), (nb + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "H2D offsets");
  check(cudaMemcpyAsync(dwg.p, cfg.wgrad.data(), PPCB_WNUM * sizeof(float2), cudaMemcpyHostToDevice, st), "H2D");
  check(cudaMemsetAsync(dctrl.p, 0, sizeof(ppcb_ctrl), st), "memset");
  check(cudaMemsetAsync(dcnt.p, 0, nbins * sizeof(unsigned int), st), "memset");
  check(cudaMemsetAsync(dgo.p, 0, 2 * PPCB_MAXLYS * sizeof(double), st), "memset");
  check(cudaMemsetAsync(dstat.p, 0, 2 * sizeof(unsigned int), st), "memset");
  cudaEvent_t e0 = X.e[0], e1 = X.e[1], e2 = X.e[2];
  // recording forward pass
  KArgs a = args_for(0);
  a.bunches = db.p; a.bstart = dbs.p; a.nb = nb; a.num = bs[nb];
  a.hits = dh.p; a.hcap = hit_cap; a.ctrl = dctrl.p; a.prov = dprov.p;
  check(cudaEventRecord(e0, st), "event");
  // the recording kernel's shape: the engine's block size (864 threads, one block per SM, or
  // 256 threads, three per SM), all blocks resident at once (a static photon order must not
  // leave a second wave of blocks), and no more threads than streams
  // (the 864-thread shape falls back to 256 threads when it cannot be resident)
  int tpb = threads_per_block == 864 ? 864 : 256;
  int per_sm = propagate_rec_blocks_per_sm(tpb, a.deterministic);
  if (tpb == 864 && (per_sm < 1 || g.T / 864 < 1)) {
    tpb = 256;
    per_sm = propagate_rec_blocks_per_sm(tpb, a.deterministic);
  }
  if (per_sm < 1 || g.T / tpb < 1) throw Error("gradient: the recording kernel does not fit on this device", 2);
  const int rec_blocks = std::min(g.prop.multiProcessorCount * per_sm, g.T / tpb);
  check(launch_propagate(a, LaunchShape{rec_blocks, tpb}, st), "recording launch");
  check(cudaEventRecord(e1, st), "event");
  ppcb_ctrl c;
  check(cudaMemcpyAsync(&c, dctrl.p, sizeof(c), cudaMemcpyDeviceToHost, st), "D2H ctrl");
  check(cudaStreamSynchronize(st), "recording pass");
  const uint64_t nh = std::min<uint64_t>(c.hidx, hit_cap);
  if (c.hidx > hit_cap) throw Error("gradient: hit capacity too small (" + std::to_string(c.hidx) + " hits)", 7);
  check(launch_dom_hist(dh.p, nh, dcnt.p, events, gsize, st), "histogram");
  Grad out;
  out.counts.resize(nbins);
  check(cudaMemcpyAsync(out.counts.data(), dcnt.p, nbins * sizeof(unsigned int), cudaMemcpyDeviceToHost, st), "D2H");
  check(cudaStreamSynchronize(st), "histogram");
  // per-bin weights: dLL/dmu_d = k_d/mu_d - 1 (times d mu_d / d count = scale)
  std::vector<float> w(nbins, 0.f);
  double ll = 0;
  for (size_t d = 0; d < nbins; d++) {
    const double mu = scale * out.counts[d];
    if (observed) {
      if (mu > 0) {
        ll += observed[d] * std::log(mu) - mu;
        w[d] = (float)(scale * (observed[d] / mu - 1.0));
      }
    } else w[d] = (float)(scale * weights[d]);
  }
  out.ll = ll;
  check(cudaMemcpyAsync(dw.p, w.data(), nbins * sizeof(float), cudaMemcpyHostToDevice, st), "H2D weights");
  // replay of the detected photons
  KArgs r = args_for(0);
  r.ctrl = dctrl.p;
  check(launch_adjoint(r, dh.p, dprov.p, nh, events, dw.p, dwg.p, dgo.p, dstat.p, g.prop.multiProcessorCount * 4, st),
        "replay launch");
  check(cudaEventRecord(e2, st), "event");
  std::vector<double> go(2 * PPCB_MAXLYS);
  unsigned int stat[2];
  check(cudaMemcpyAsync(go.data(), dgo.p, go.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H gradient");
  check(cudaMemcpyAsync(stat, dstat.p, sizeof(stat), cudaMemcpyDeviceToHost, st), "D2H stats");
  check(cudaStreamSynchronize(st), "replay");
  check(cudaEventElapsedTime(&out.forward_ms, e0, e1), "elapsed");
  check(cudaEventElapsedTime(&out.backward_ms, e1, e2), "elapsed");
  // kernel layers run from the deepest row of icemodel.dat (layer i <-> row size-1-i)
  out.g_be.assign(size, 0.0);
  out.g_ba.assign(size, 0.0);
  for (int i = 0; i < size; i++) {
    out.g_be[size - 1 - i] = go[i];
    out.g_ba[size - 1 - i] = go[PPCB_MAXLYS + i];
  }
  out.photons = bs[nb];
  out.hits = nh;
  out.steps = c.steps;
  out.replayed = stat[0];
  out.unmatched = stat[1];
  g.device_ms += out.forward_ms + out.backward_ms;
  return out;
}

// ---------------------------------------------------------------- one fit iteration as a graph
namespace {

constexpr int kWBlocks = 592, kWThreads = 256;

// Poisson weights w_d = scale (k_d / mu_d - 1) and the log-likelihood terms k_d log mu_d - mu_d
// of the bins with mu_d = scale x simulated count > 0 (as Engine::gradient forms them on the
// host), summed per block in a fixed order (strided per thread, then a tree).
__global__ void __launch_bounds__(kWThreads) k_weights(const unsigned int* __restrict__ counts,
                                                       const float* __restrict__ observed, uint64_t nbins,
                                                       double scale, float* w, double* part) {
  __shared__ double red[kWThreads];
  double ll = 0;
  for (uint64_t d = blockIdx.x * (uint64_t)kWThreads + threadIdx.x; d < nbins; d += (uint64_t)gridDim.x * kWThreads) {
    const double mu = scale * counts[d];
    float wd = 0.f;
    if (mu > 0) {
      ll += observed[d] * log(mu) - mu;
      wd = (float)(scale * (observed[d] / mu - 1.0));
    }
    w[d] = wd;
  }
  red[threadIdx.x] = ll;
  __syncthreads();
  for (int o = kWThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// The block sums in block order.
__global__ void k_ll_sum(const double* part, int n, double* ll) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0;
    for (int k = 0; k < n; k++) s += part[k];
    *ll = s;
  }
}

template <class T>
struct Pinned {
  T* p = nullptr;
  void need(size_t n) { check(cudaMallocHost((void**)&p, std::max<size_t>(n, 1) * sizeof(T)), "pinned"); }
  ~Pinned() { if (p) cudaFreeHost(p); }
};

}  // namespace

struct GradGraphState {
  int dev = 0;
  cudaStream_t st = nullptr;
  uint32_t events = 0;
  size_t nbins = 0;
  uint64_t photons = 0, hit_cap = 0;
  DBuf<ppcb_bunch> bunches;
  DBuf<uint64_t> bstart;
  DBuf<ppcb_hit> hits;
  DBuf<unsigned char> prov;
  DBuf<ppcb_ctrl> ctrl;
  DBuf<unsigned int> counts;
  DBuf<float> observed, weights;
  DBuf<float2> wgrad;
  DBuf<double> g, part, ll;
  DBuf<unsigned int> stats;
  Pinned<float> absca;          // staging of the ice table the graph uploads first
  Pinned<double> hg, hll;
  Pinned<unsigned int> hstats, hcounts;
  Pinned<ppcb_ctrl> hctrl;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~GradGraphState() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto& x : ev) if (x) cudaEventDestroy(x);
  }
};

GradGraph::GradGraph(Engine& e, const ppcb_bunch* b, int nb, uint32_t events, const float* observed, double scale,
                     uint64_t hit_cap)
    : e_(e), s_(new GradGraphState) {
  if (!e.ready()) throw Error("ini() must come before the gradient", 6);
  if (nb <= 0 || !b || !observed) throw Error("gradient graph: bunches and observed counts required", 7);
  DeviceCtx& g = e.devs[0];
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  GradGraphState& S = *s_;
  S.dev = g.dev;
  S.st = g.st;
  S.events = events;
  S.nbins = (size_t)e.cfg.p.gsize * (events ? events : 1);
  S.hit_cap = hit_cap;
  std::vector<uint64_t> bs(nb + 1, 0);
  for (int k = 0; k < nb; k++) bs[k + 1] = bs[k] + b[k].num;
  S.photons = bs[nb];
  S.bunches.need(nb); S.bstart.need(nb + 1);
  S.hits.need(hit_cap); S.prov.need(hit_cap * kProvBytes); S.ctrl.need(1);
  S.counts.need(S.nbins); S.observed.need(S.nbins); S.weights.need(S.nbins);
  S.wgrad.need(PPCB_WNUM); S.g.need(2 * PPCB_MAXLYS); S.part.need(kWBlocks); S.ll.need(1); S.stats.need(2);
  S.absca.need(e.cfg.absca.size());
  S.hg.need(2 * PPCB_MAXLYS); S.hll.need(1); S.hstats.need(2); S.hcounts.need(S.nbins); S.hctrl.need(1);
  for (auto& x : S.ev) check(cudaEventCreate(&x), "event");
  cudaStream_t st = S.st;
  check(cudaMemcpyAsync(S.bunches.p, b, nb * sizeof(ppcb_bunch), cudaMemcpyHostToDevice, st), "H2D bunches");
  check(cudaMemcpyAsync(S.bstart.p, bs.data(), (nb + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "H2D");
  check(cudaMemcpyAsync(S.observed.p, observed, S.nbins * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
  check(cudaMemcpyAsync(S.wgrad.p, e.cfg.wgrad.data(), PPCB_WNUM * sizeof(float2), cudaMemcpyHostToDevice, st),
        "H2D");
  check(cudaStreamSynchronize(st), "gradient graph set-up");

  // the recording kernel's shape (as Engine::gradient picks it); the occupancy queries also
  // set the kernels' shared-memory attributes, which must happen before the capture
  KArgs a = e.args_for(0);
  a.bunches = S.bunches.p; a.bstart = S.bstart.p; a.nb = nb; a.num = S.photons;
  a.hits = S.hits.p; a.hcap = hit_cap; a.ctrl = S.ctrl.p; a.prov = S.prov.p;
  int tpb = e.threads_per_block == 864 ? 864 : 256;
  int per_sm = propagate_rec_blocks_per_sm(tpb, a.deterministic);
  if (tpb == 864 && (per_sm < 1 || g.T / 864 < 1)) {
    tpb = 256;
    per_sm = propagate_rec_blocks_per_sm(tpb, a.deterministic);
  }
  if (per_sm < 1 || g.T / tpb < 1) throw Error("gradient: the recording kernel does not fit on this device", 2);
  const LaunchShape shape{std::min(g.prop.multiProcessorCount * per_sm, g.T / tpb), tpb};
  KArgs r = e.args_for(0);
  r.ctrl = S.ctrl.p;
  const unsigned long long* nh_dev = &S.ctrl.p->hidx;
  check(adjoint_prepare(), "replay attribute");

  // the timing events are recorded as external event nodes, so that a replay records them
  check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t err = cudaSuccess;
  auto q = [&](cudaError_t x) { if (err == cudaSuccess) err = x; };
  q(cudaMemcpyAsync(g.absca, S.absca.p, e.cfg.absca.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  q(cudaMemsetAsync(S.ctrl.p, 0, sizeof(ppcb_ctrl), st));
  q(cudaMemsetAsync(S.counts.p, 0, S.nbins * sizeof(unsigned int), st));
  q(cudaMemsetAsync(S.g.p, 0, 2 * PPCB_MAXLYS * sizeof(double), st));
  q(cudaMemsetAsync(S.stats.p, 0, 2 * sizeof(unsigned int), st));
  q(cudaEventRecordWithFlags(S.ev[0], st, cudaEventRecordExternal));
  q(launch_propagate(a, shape, st));
  q(cudaEventRecordWithFlags(S.ev[1], st, cudaEventRecordExternal));
  q(launch_dom_hist(S.hits.p, hit_cap, S.counts.p, events, e.cfg.p.gsize, st, nh_dev));
  k_weights<<<kWBlocks, kWThreads, 0, st>>>(S.counts.p, S.observed.p, S.nbins, scale, S.weights.p, S.part.p);
  q(cudaGetLastError());
  k_ll_sum<<<1, 32, 0, st>>>(S.part.p, kWBlocks, S.ll.p);
  q(cudaGetLastError());
  q(launch_adjoint(r, S.hits.p, S.prov.p, hit_cap, events, S.weights.p, S.wgrad.p, S.g.p, S.stats.p,
                   g.prop.multiProcessorCount * 4, st, nh_dev));
  q(cudaEventRecordWithFlags(S.ev[2], st, cudaEventRecordExternal));
  q(cudaMemcpyAsync(S.hg.p, S.g.p, 2 * PPCB_MAXLYS * sizeof(double), cudaMemcpyDeviceToHost, st));
  q(cudaMemcpyAsync(S.hll.p, S.ll.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  q(cudaMemcpyAsync(S.hstats.p, S.stats.p, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  q(cudaMemcpyAsync(S.hctrl.p, S.ctrl.p, sizeof(ppcb_ctrl), cudaMemcpyDeviceToHost, st));
  q(cudaMemcpyAsync(S.hcounts.p, S.counts.p, S.nbins * sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(st, &graph);
  S.graph = graph;
  check(err, "gradient graph capture");
  check(ec, "end capture");
  check(cudaGraphInstantiate(&S.exec, S.graph, 0), "graph instantiate");
}

GradGraph::~GradGraph() = default;

Engine::Grad GradGraph::run(const float* be, const float* ba, bool counts) {
  GradGraphState& S = *s_;
  check(cudaSetDevice(S.dev), "cudaSetDevice");
  e_.cfg.set_ice(be, ba);  // the table the graph uploads, then every other device's copy
  memcpy(S.absca.p, e_.cfg.absca.data(), e_.cfg.absca.size() * sizeof(float));
  check(cudaGraphLaunch(S.exec, S.st), "graph launch");
  check(cudaStreamSynchronize(S.st), "gradient graph");
  for (size_t k = 1; k < e_.devs.size(); k++) {
    check(cudaSetDevice(e_.devs[k].dev), "cudaSetDevice");
    check(cudaMemcpy(e_.devs[k].absca, S.absca.p, e_.cfg.absca.size() * sizeof(float), cudaMemcpyHostToDevice),
          "ice table");
  }
  check(cudaSetDevice(S.dev), "cudaSetDevice");
  const ppcb_ctrl c = *S.hctrl.p;
  if (c.hidx > S.hit_cap) throw Error("gradient: hit capacity too small (" + std::to_string(c.hidx) + " hits)", 7);
  Engine::Grad out;
  out.ll = *S.hll.p;
  if (counts) out.counts.assign(S.hcounts.p, S.hcounts.p + S.nbins);
  const int size = e_.cfg.p.size;
  out.g_be.assign(size, 0.0);
  out.g_ba.assign(size, 0.0);
  for (int i = 0; i < size; i++) {  // kernel layer i <-> icemodel.dat row size-1-i
    out.g_be[size - 1 - i] = S.hg.p[i];
    out.g_ba[size - 1 - i] = S.hg.p[PPCB_MAXLYS + i];
  }
  check(cudaEventElapsedTime(&out.forward_ms, S.ev[0], S.ev[1]), "elapsed");
  check(cudaEventElapsedTime(&out.backward_ms, S.ev[1], S.ev[2]), "elapsed");
  out.photons = S.photons;
  out.hits = c.hidx;
  out.steps = c.steps;
  out.replayed = S.hstats.p[0];
  out.unmatched = S.hstats.p[1];
  e_.devs[0].device_ms += out.forward_ms + out.backward_ms;
  return out;
}

}  // namespace ppcb
