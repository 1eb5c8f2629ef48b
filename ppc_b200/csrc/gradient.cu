// Ice-model gradient (Engine::gradient, Engine::set_ice).  No counterpart in the reference:
// llh/DirectFit fits the ice by repeated forward runs (llh/llh.cxx:1435-1634); here the
// gradient of the likelihood with respect to all 2 x 171 per-layer coefficients comes from
// one recording forward pass and a replay of the detected photons (propagate.cu, AdjHook).
#include <algorithm>
#include <cmath>

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

}  // namespace ppcb
