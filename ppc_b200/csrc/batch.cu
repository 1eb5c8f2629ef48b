// Batched propagation (see batch.h).
#include "batch.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ppcb {

template <class T>
static T* dmalloc(size_t n) {
  void* p = nullptr;
  check(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "batch buffer");
  return (T*)p;
}

template <class T>
static T* hmalloc(size_t n) {
  void* p = nullptr;
  check(cudaMallocHost(&p, std::max<size_t>(n, 1) * sizeof(T)), "batch pinned buffer");
  return (T*)p;
}

// Exclusive prefix of the kept hits per event, min(produced, capacity); one block.
__global__ void k_compact_scan(const unsigned int* cnt, const uint32_t* cap, const uint64_t* dyn, uint64_t* out_off) {
  __shared__ unsigned long long part[1024];
  const int E = (int)dyn[2];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (E + nt - 1) / nt;
  const int lo = t * per, hi = min(E, lo + per);
  unsigned long long s = 0;
  for (int e = lo; e < hi; e++) s += min(cnt[e], cap[e]);
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {
    unsigned long long v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  unsigned long long acc = part[t] - s;
  for (int e = lo; e < hi; e++) {
    out_off[e] = acc;
    acc += min(cnt[e], cap[e]);
  }
  if (t == nt - 1) out_off[E] = part[t];
}

// One warp per event: copy its kept hits into the compact output.
__global__ void k_compact_gather(const ppcb_hit* __restrict__ hits, const uint64_t* __restrict__ ev_off,
                                 const uint64_t* __restrict__ out_off, const uint64_t* dyn, ppcb_hit* out) {
  const int E = (int)dyn[2];
  const int e = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (e >= E) return;
  const uint64_t n = out_off[e + 1] - out_off[e];
  const uint4* src = reinterpret_cast<const uint4*>(hits + ev_off[e]);
  uint4* dst = reinterpret_cast<uint4*>(out + out_off[e]);
  for (uint64_t k = threadIdx.x & 31; k < 2 * n; k += 32) dst[k] = src[k];
}

Batch::Batch(Engine& e, int device, uint32_t max_events, uint32_t max_bunches, uint64_t hit_capacity)
    : eng_(e), d_(device), maxE_(max_events), maxB_(max_bunches), hcap_(hit_capacity) {
  if (!e.ready()) throw Error("ini() must come before creating a batch", 6);
  if (device < 0 || device >= (int)e.devs.size()) throw Error("bad device index", 7);
  if (max_events == 0 || max_bunches == 0) throw Error("empty batch capacity", 7);
  cuda_dev_ = e.devs[d_].dev;
  check(cudaSetDevice(cuda_dev_), "cudaSetDevice");
  check(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "stream");
  for (cudaEvent_t* ev : {&k0_, &k1_, &g0_, &g1_}) check(cudaEventCreate(ev), "event");
  bunches_ = dmalloc<ppcb_bunch>(maxB_);
  bstart_ = dmalloc<uint64_t>(maxB_ + 1);
  ev_off_ = dmalloc<uint64_t>(maxE_);
  ev_cap_ = dmalloc<uint32_t>(maxE_);
  ev_cnt_ = dmalloc<unsigned int>(maxE_);
  dyn_ = dmalloc<uint64_t>(4);
  hits_ = dmalloc<ppcb_hit>(hcap_);
  out_ = dmalloc<ppcb_hit>(hcap_);
  out_off_ = dmalloc<uint64_t>(maxE_ + 1);
  ctrl_ = dmalloc<ppcb_ctrl>(1);
  h_bunches_ = hmalloc<ppcb_bunch>(maxB_);
  h_bstart_ = hmalloc<uint64_t>(maxB_ + 1);
  h_ev_off_ = hmalloc<uint64_t>(maxE_);
  h_ev_cap_ = hmalloc<uint32_t>(maxE_);
  h_ev_cnt_ = hmalloc<unsigned int>(maxE_);
  h_dyn_ = hmalloc<uint64_t>(4);
  h_out_off_ = hmalloc<uint64_t>(maxE_ + 1);
  h_ctrl_ = hmalloc<ppcb_ctrl>(1);
  memset(h_bunches_, 0, sizeof(ppcb_bunch) * maxB_);
  memset(h_bstart_, 0, sizeof(uint64_t) * (maxB_ + 1));
  memset(h_ev_off_, 0, sizeof(uint64_t) * maxE_);
  memset(h_ev_cap_, 0, sizeof(uint32_t) * maxE_);
  memset(h_dyn_, 0, sizeof(uint64_t) * 4);
}

Batch::~Batch() {
  cudaSetDevice(cuda_dev_);
  if (st_) cudaStreamSynchronize(st_);
  release_graph();
  void* d[] = {bunches_, bstart_, ev_off_, ev_cap_, ev_cnt_, dyn_, hits_, out_, out_off_, ctrl_};
  for (void* p : d) if (p) cudaFree(p);
  void* h[] = {h_bunches_, h_bstart_, h_ev_off_, h_ev_cap_, h_ev_cnt_, h_dyn_, h_out_off_, h_ctrl_};
  for (void* p : h) if (p) cudaFreeHost(p);
  for (cudaEvent_t ev : {k0_, k1_, g0_, g1_}) if (ev) cudaEventDestroy(ev);
  if (st_) cudaStreamDestroy(st_);
}

void Batch::release_graph() {
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
}

// The work of one batch.  Every size is fixed at construction, so the same sequence
// replays from a graph; the kernels read the batch's own sizes from `dyn`.
static void enqueue(Engine& eng, int d, cudaStream_t st, uint32_t maxE, uint32_t maxB, uint64_t hcap,
                    ppcb_bunch* bunches, uint64_t* bstart, uint64_t* ev_off, uint32_t* ev_cap, unsigned int* ev_cnt,
                    uint64_t* dyn, ppcb_hit* hits, ppcb_hit* out, uint64_t* out_off, ppcb_ctrl* ctrl,
                    const ppcb_bunch* h_b, const uint64_t* h_bs, const uint64_t* h_eo, const uint32_t* h_ec,
                    const uint64_t* h_dyn, unsigned int* h_cnt, uint64_t* h_oo, ppcb_ctrl* h_ctrl, cudaEvent_t g0,
                    cudaEvent_t k0, cudaEvent_t k1, cudaEvent_t g1) {
  // events are recorded only on direct launches: inside a captured graph they become
  // nodes whose times cannot be read back (graph replays are timed from outside)
  if (g0) check(cudaEventRecord(g0, st), "event");
  check(cudaMemcpyAsync(bunches, h_b, maxB * sizeof(ppcb_bunch), cudaMemcpyHostToDevice, st), "H2D bunches");
  check(cudaMemcpyAsync(bstart, h_bs, (maxB + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "H2D offsets");
  check(cudaMemcpyAsync(ev_off, h_eo, maxE * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "H2D regions");
  check(cudaMemcpyAsync(ev_cap, h_ec, maxE * sizeof(uint32_t), cudaMemcpyHostToDevice, st), "H2D capacities");
  check(cudaMemcpyAsync(dyn, h_dyn, 4 * sizeof(uint64_t), cudaMemcpyHostToDevice, st), "H2D sizes");
  check(cudaMemsetAsync(ev_cnt, 0, maxE * sizeof(unsigned int), st), "memset counters");
  check(cudaMemsetAsync(ctrl, 0, sizeof(ppcb_ctrl), st), "memset ctrl");
  KArgs a = eng.args_for(d);
  a.bunches = bunches; a.bstart = bstart; a.dyn = dyn;
  a.ev_off = ev_off; a.ev_cap = ev_cap; a.ev_cnt = ev_cnt;
  a.hits = hits; a.hcap = hcap; a.ctrl = ctrl;
  if (k0) check(cudaEventRecord(k0, st), "event");
  check(launch_propagate(a, eng.devs[d].shape, st), "propagate launch");
  if (k1) check(cudaEventRecord(k1, st), "event");
  k_compact_scan<<<1, 1024, 0, st>>>(ev_cnt, ev_cap, dyn, out_off);
  check(cudaGetLastError(), "compact scan");
  k_compact_gather<<<(maxE + 7) / 8, 256, 0, st>>>(hits, ev_off, out_off, dyn, out);
  check(cudaGetLastError(), "compact gather");
  check(cudaMemcpyAsync(h_cnt, ev_cnt, maxE * sizeof(unsigned int), cudaMemcpyDeviceToHost, st), "D2H counts");
  check(cudaMemcpyAsync(h_oo, out_off, (maxE + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st), "D2H offsets");
  check(cudaMemcpyAsync(h_ctrl, ctrl, sizeof(ppcb_ctrl), cudaMemcpyDeviceToHost, st), "D2H ctrl");
  if (g1) check(cudaEventRecord(g1, st), "event");
}

void Batch::capture() {
  release_graph();
  cudaGraph_t g;
  check(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "begin capture");
  enqueue(eng_, d_, st_, maxE_, maxB_, hcap_, bunches_, bstart_, ev_off_, ev_cap_, ev_cnt_, dyn_, hits_, out_,
          out_off_, ctrl_, h_bunches_, h_bstart_, h_ev_off_, h_ev_cap_, h_dyn_, h_ev_cnt_, h_out_off_, h_ctrl_, nullptr,
          nullptr, nullptr, nullptr);
  check(cudaStreamEndCapture(st_, &g), "end capture");
  cudaError_t e = cudaGraphInstantiate(&exec_, g, 0);
  cudaGraphDestroy(g);
  check(e, "graph instantiate");
}

void Batch::run(const ppcb_bunch* b, int nb, uint32_t events, BatchResult& out, double hits_per_photon,
                uint32_t hit_slack) {
  if (nb <= 0 || (uint32_t)nb > maxB_) throw Error("batch: bunch count outside 1.." + std::to_string(maxB_), 7);
  if (events == 0 || events > maxE_) throw Error("batch: event count outside 1.." + std::to_string(maxE_), 7);
  check(cudaSetDevice(eng_.devs[d_].dev), "cudaSetDevice");
  std::vector<uint64_t> ph(events, 0);
  uint64_t num = 0;
  for (int k = 0; k < nb; k++) {
    if (b[k].q >= events) throw Error("batch: bunch event index out of range", 7);
    h_bstart_[k] = num;
    num += b[k].num;
    ph[b[k].q] += b[k].num;
  }
  h_bstart_[nb] = num;
  memcpy(h_bunches_, b, nb * sizeof(ppcb_bunch));
  uint64_t off = 0;
  for (uint32_t e = 0; e < events; e++) {
    double c = std::ceil(ph[e] * hits_per_photon) + hit_slack;
    uint32_t cap = (uint32_t)std::min<double>(c, 4.0e9);
    h_ev_off_[e] = off;
    h_ev_cap_[e] = cap;
    off += cap;
  }
  if (off > hcap_) throw Error("batch: per-event hit regions (" + std::to_string(off) + ") exceed the capacity " +
                               std::to_string(hcap_), 7);
  h_dyn_[0] = num;
  h_dyn_[1] = (uint64_t)nb;
  h_dyn_[2] = events;
  if (use_graph) {
    if (!exec_) capture();
    check(cudaEventRecord(g0_, st_), "event");
    check(cudaGraphLaunch(exec_, st_), "graph launch");
    check(cudaEventRecord(g1_, st_), "event");
  } else {
    enqueue(eng_, d_, st_, maxE_, maxB_, hcap_, bunches_, bstart_, ev_off_, ev_cap_, ev_cnt_, dyn_, hits_, out_,
            out_off_, ctrl_, h_bunches_, h_bstart_, h_ev_off_, h_ev_cap_, h_dyn_, h_ev_cnt_, h_out_off_, h_ctrl_, g0_,
            k0_, k1_, g1_);
  }
  check(cudaStreamSynchronize(st_), "batch");
  out.produced.assign(h_ev_cnt_, h_ev_cnt_ + events);
  out.offset.assign(h_out_off_, h_out_off_ + events + 1);
  out.overflowed = 0;
  for (uint32_t e = 0; e < events; e++) if (h_ev_cnt_[e] > h_ev_cap_[e]) out.overflowed++;
  const uint64_t kept = h_out_off_[events];
  out.hits.resize(kept);
  if (kept) check(cudaMemcpy(out.hits.data(), out_, kept * sizeof(ppcb_hit), cudaMemcpyDeviceToHost), "D2H hits");
  out.photons = num;
  out.steps = h_ctrl_->steps;
  check(cudaEventElapsedTime(&out.graph_ms, g0_, g1_), "elapsed");
  // a replayed graph is timed as a whole; the kernel dominates it
  if (use_graph) out.device_ms = out.graph_ms;
  else check(cudaEventElapsedTime(&out.device_ms, k0_, k1_), "elapsed");
  eng_.devs[d_].device_ms += out.device_ms;
}

TuneResult Batch::autotune(const ppcb_bunch* b, int nb, uint32_t events, uint64_t sample_photons) {
  // a scaled-down copy of the batch: every bunch keeps its share of the photons
  uint64_t total = 0;
  for (int k = 0; k < nb; k++) total += b[k].num;
  std::vector<ppcb_bunch> s(b, b + nb);
  const double f = total > sample_photons ? (double)sample_photons / total : 1.0;
  for (auto& x : s) x.num = (uint32_t)std::max<double>(1.0, std::floor(x.num * f));
  DeviceCtx& g = eng_.devs[d_];
  const LaunchShape keep = g.shape;
  const int keep_refill = eng_.refill_below;
  const int Tmax = g.T;
  struct Cand { int threads, per_sm, refill; };
  const Cand cands[] = {{256, 3, 0}, {128, 6, 0}, {768, 1, 0}, {864, 1, 0}, {256, 3, 8},
                        {768, 1, 8}, {128, 6, 8}, {256, 2, 0}, {256, 3, 16}};
  TuneResult best;
  BatchResult r;
  const bool graph = use_graph;
  use_graph = false;
  for (const Cand& c : cands) {
    const int blocks = g.prop.multiProcessorCount * c.per_sm;
    if (blocks * c.threads > Tmax) continue;  // one random stream per thread
    if (propagate_max_blocks_per_sm(c.threads) < c.per_sm) continue;
    g.shape = LaunchShape{blocks, c.threads};
    eng_.refill_below = c.refill;
    run(s.data(), nb, events, r, 0.05);  // warm
    run(s.data(), nb, events, r, 0.05);
    const double rate = r.photons / (r.device_ms * 1e-3);
    best.log.push_back(std::to_string(c.threads) + "x" + std::to_string(c.per_sm) + " refill " +
                       std::to_string(c.refill) + ": " + std::to_string(rate) + " photons/s");
    if (rate > best.photons_per_s) {
      best.photons_per_s = rate;
      best.threads = c.threads;
      best.blocks_per_sm = c.per_sm;
      best.refill_below = c.refill;
    }
  }
  use_graph = graph;
  if (best.photons_per_s > 0) {
    g.shape = LaunchShape{g.prop.multiProcessorCount * best.blocks_per_sm, best.threads};
    eng_.refill_below = best.refill_below;
  } else {
    g.shape = keep;
    eng_.refill_below = keep_refill;
  }
  release_graph();  // kernel parameters changed: capture again on the next run
  return best;
}

}  // namespace ppcb
