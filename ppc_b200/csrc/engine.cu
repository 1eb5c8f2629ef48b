// Device runtime (see engine.h).
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>

namespace ppcb {

static const int kOver = 128;   // minimum photons per bunch slot (gpu/ini.cxx:18)
static const int kNpho = 1024;  // photons per thread per launch (gpu/ini.cxx:21)

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e), 2);
}

template <class T>
static T* dalloc(size_t n, const char* what) {
  void* p = nullptr;
  check(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), what);
  return (T*)p;
}

template <class T>
static void upload(T* d, const T* h, size_t n, const char* what) {
  if (n) check(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), what);
}

Engine::~Engine() {
  try { fin(); } catch (...) {}
}

void Engine::initialize(const std::string& dir, float enh) {
  cfg.load(dir);
  cfg.eff *= enh;
  initialized_ = true;
}

static int env_int(const std::string& name, int def) {
  const char* v = getenv(name.c_str());
  return (v && *v) ? atoi(v) : def;
}

void Engine::choose(int device) {
  int count = 0;
  check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
  std::vector<int> list;
  if (device < 0) for (int d = 0; d < count; d++) list.push_back(d);
  else {
    if (device >= count) throw Error("No active GPU(s) selected!", 5);
    sv += device;
    list.push_back(device);
  }
  devs.clear();
  for (int d : list) {
    std::ostringstream o;
    o << "NPHO_" << d;
    int npho = env_int(o.str(), env_int("NPHO", kNpho));
    if (npho <= 0) continue;  // device switched off (gpu/ppc.cu:120-131)
    DeviceCtx g;
    g.dev = d;
    check(cudaGetDeviceProperties(&g.prop, d), "cudaGetDeviceProperties");
    g.T = npho;  // provisional: photons per thread, resolved in ini()
    devs.push_back(g);
  }
  if (devs.empty()) throw Error("No active GPU(s) selected!", 5);
}

void Engine::ini() {
  if (!initialized_) throw Error("initialize() must come before ini()");
  if (devs.empty()) choose(0);
  fin();
  hquo = std::max(1, env_int("HQUO", 1));
  pmax = 0;
  pmxo = 0;
  for (size_t k = 0; k < devs.size(); k++) {
    DeviceCtx& g = devs[k];
    int npho = g.T;
    check(cudaSetDevice(g.dev), "cudaSetDevice");
    int kBlock = threads_per_block;
    if (const char* t = getenv("PPCB_THREADS_PER_BLOCK")) if (atoi(t) > 0) kBlock = atoi(t);
    if (kBlock != 128 && kBlock != 256 && kBlock != 768 && kBlock != 864) kBlock = 256;
    int per_sm = blocks_per_sm > 0 ? blocks_per_sm : propagate_max_blocks_per_sm(kBlock);
    if (const char* b = getenv("PPCB_BLOCKS_PER_SM")) if (atoi(b) > 0) per_sm = atoi(b);
    if (per_sm <= 0) per_sm = 1;
    int blocks = g.prop.multiProcessorCount * per_sm;
    // one distinct MWC multiplier per thread: never reuse a stream
    int maxb = cfg.p.rsize / kBlock;
    if (maxb < 1) throw Error("not enough random multipliers in rnd.txt (need at least 256)");
    if (blocks > maxb) blocks = maxb;
    g.shape = LaunchShape{blocks, kBlock};
    g.T = blocks * kBlock;
    // capacities, halved until they fit (gpu/ppc.cu:170-186)
    size_t freeb = 0, totb = 0;
    check(cudaMemGetInfo(&freeb, &totb), "cudaMemGetInfo");
    uint64_t pm = 0, po = 0, hc = 0;
    while (npho > 0) {
      pm = (uint64_t)g.T * npho;
      po = pm / kOver;
      pm = po * kOver;
      hc = pm / hquo;
      uint64_t need = 2 * (po * (sizeof(ppcb_bunch) + 8) + hc * sizeof(ppcb_hit)) + (8 << 20);
      if (need > freeb * 0.9) npho /= 2;
      else break;
    }
    if (npho <= 0) throw Error("not enough device memory");
    g.bcap = po;
    g.hcap = hc;
    pmax += pm;
    if (pmxo == 0 || pmxo > po) pmxo = po;

    check(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking), "stream");
    check(cudaStreamCreateWithFlags(&g.cp, cudaStreamNonBlocking), "stream");
    const ppcb_params& p = cfg.p;
    g.absca = dalloc<float2>((size_t)PPCB_WNUM * p.size, "absca");
    upload(g.absca, (const float2*)cfg.absca.data(), (size_t)PPCB_WNUM * p.size, "absca");
    g.wmeta = dalloc<ppcb_wmeta>(PPCB_WNUM, "wmeta");
    upload(g.wmeta, cfg.wmeta.data(), PPCB_WNUM, "wmeta");
    g.lp = dalloc<float2>((size_t)PPCB_LMAX * PPCB_LYRS, "lp");
    upload(g.lp, (const float2*)cfg.lp.data(), (size_t)PPCB_LMAX * PPCB_LYRS, "lp");
    g.oms = dalloc<ppcb_dom>(p.gsize, "oms");
    upload(g.oms, cfg.oms.data(), p.gsize, "oms");
    g.az = dalloc<ppcb_aniz>(p.size, "az");
    upload(g.az, cfg.az.data(), p.size, "az");
    g.sc = dalloc<ppcb_line>(PPCB_NSTR, "sc");
    upload(g.sc, cfg.sc.data(), PPCB_NSTR, "sc");
    g.lr = dalloc<float>(PPCB_LMAX, "lr");
    upload(g.lr, cfg.lr.data(), PPCB_LMAX, "lr");
    g.ls = dalloc<uint16_t>(PPCB_NSTR, "ls");
    upload(g.ls, cfg.ls.data(), PPCB_NSTR, "ls");
    g.is = dalloc<uint16_t>(PPCB_CX * PPCB_CY, "is");
    upload(g.is, cfg.is.data(), PPCB_CX * PPCB_CY, "is");
    g.mcol = dalloc<int8_t>(PPCB_CTX * PPCB_CTY, "mcol");
    upload(g.mcol, cfg.mcol.data(), PPCB_CTX * PPCB_CTY, "mcol");
    g.bfrt = dalloc<float4>(PPCB_BFR_TAB + 1, "bfrt");
    upload(g.bfrt, (const float4*)cfg.bfrt.data(), PPCB_BFR_TAB + 1, "bfrt");
    if (cfg.sg.on) {
      g.sg_groups = dalloc<StrGroup>(cfg.sg_groups.size(), "sg_groups");
      upload(g.sg_groups, cfg.sg_groups.data(), cfg.sg_groups.size(), "sg_groups");
      g.sg_cells = dalloc<uint16_t>(cfg.sg_cells.size(), "sg_cells");
      upload(g.sg_cells, cfg.sg_cells.data(), cfg.sg_cells.size(), "sg_cells");
    }
    g.rs = dalloc<uint64_t>(g.T, "rs");
    g.rm = dalloc<uint32_t>(g.T, "rm");
    upload(g.rm, cfg.rm.data(), g.T, "rm");
    for (int s = 0; s < 2; s++) {
      auto& S = g.slot[s];
      S.bunches = dalloc<ppcb_bunch>(g.bcap, "bunches");
      S.bstart = dalloc<uint64_t>(g.bcap + 1, "bstart");
      S.hits = dalloc<ppcb_hit>(g.hcap, "hits");
      S.ctrl = dalloc<ppcb_ctrl>(1, "ctrl");
      check(cudaMallocHost((void**)&S.hb, g.bcap * sizeof(ppcb_bunch)), "pinned bunches");
      check(cudaMallocHost((void**)&S.hbstart, (g.bcap + 1) * sizeof(uint64_t)), "pinned bstart");
      check(cudaMallocHost((void**)&S.hctrl, sizeof(ppcb_ctrl)), "pinned ctrl");
      check(cudaEventCreate(&S.t0), "event");
      check(cudaEventCreate(&S.t1), "event");
      S.busy = false;
    }
    g.hhits_cap = 1 << 16;
    check(cudaMallocHost((void**)&g.hhits, g.hhits_cap * sizeof(ppcb_hit)), "pinned hits");
  }
  inited_ = true;
  reset_streams();
  for (auto& g : devs) check(cudaStreamSynchronize(g.st), "sync");
}

void Engine::reset_streams() {
  // every stream starts at (362436069 + sv, 1234567); streams differ by multiplier
  // (gpu/ini.cxx:556-571); each further device gets sv+1 (gpu/ppc.cu:339)
  unsigned int s = sv;
  for (auto& g : devs) {
    check(cudaSetDevice(g.dev), "cudaSetDevice");
    uint64_t v = (uint64_t)(362436069u + s) | ((uint64_t)1234567u << 32);
    std::vector<uint64_t> h(g.T, v);
    upload(g.rs, h.data(), g.T, "rs");
    if (devs.size() > 1) s++;
  }
}

void Engine::free_device(DeviceCtx& g) {
  cudaSetDevice(g.dev);
  g.back.reset();
  g.front.reset();
  if (g.st) cudaStreamSynchronize(g.st);
  if (g.cp) cudaStreamSynchronize(g.cp);
  void* ptrs[] = {g.absca, g.wmeta, g.lp, g.oms, g.az, g.sc, g.lr, g.ls, g.is, g.mcol, g.bfrt, g.sg_groups, g.sg_cells,
                  g.rs, g.rm};
  for (void* p : ptrs) if (p) cudaFree(p);
  g.absca = nullptr; g.wmeta = nullptr; g.lp = nullptr; g.oms = nullptr; g.az = nullptr; g.sc = nullptr;
  g.bfrt = nullptr; g.sg_groups = nullptr; g.sg_cells = nullptr;
  g.lr = nullptr; g.ls = nullptr; g.is = nullptr; g.mcol = nullptr; g.rs = nullptr; g.rm = nullptr;
  for (auto& S : g.slot) {
    if (S.bunches) cudaFree(S.bunches);
    if (S.bstart) cudaFree(S.bstart);
    if (S.hits) cudaFree(S.hits);
    if (S.ctrl) cudaFree(S.ctrl);
    if (S.hb) cudaFreeHost(S.hb);
    if (S.hbstart) cudaFreeHost(S.hbstart);
    if (S.hctrl) cudaFreeHost(S.hctrl);
    if (S.t0) cudaEventDestroy(S.t0);
    if (S.t1) cudaEventDestroy(S.t1);
    S = DeviceCtx::Slot();
  }
  if (g.hhits) cudaFreeHost(g.hhits);
  g.hhits = nullptr;
  g.hhits_cap = 0;
  if (g.st) cudaStreamDestroy(g.st);
  if (g.cp) cudaStreamDestroy(g.cp);
  g.st = nullptr; g.cp = nullptr;
}

void Engine::fin() {
  if (!inited_) return;
  if (!devs.empty()) cudaSetDevice(devs[0].dev);
  gs_.reset();
  for (auto& g : devs) free_device(g);
  queue_.clear();
  inited_ = false;
}

KArgs Engine::args_for(int d) const {
  const DeviceCtx& g = devs[d];
  KArgs a;
  memset(&a, 0, sizeof(a));
  a.p = cfg.p;
  a.absca = g.absca; a.wmeta = g.wmeta; a.lp = g.lp; a.oms = g.oms; a.az = g.az; a.sc = g.sc;
  a.lr = g.lr; a.ls = g.ls; a.is = g.is; a.mcol = g.mcol; a.bfrt = g.bfrt;
  a.sg = cfg.sg; a.sg_groups = g.sg_groups; a.sg_ngroups = (int)cfg.sg_groups.size(); a.sg_cells = g.sg_cells;
  if (!a.sg_cells) a.sg.on = 0;
  a.rs = g.rs; a.rm = g.rm;
  a.deterministic = deterministic;
  a.seed = sv;
  a.max_steps = max_steps;
  a.refill_below = refill_below;
  return a;
}

long Engine::submit(const ppcb_bunch* b, int nb, uint64_t num) {
  if (!inited_) throw Error("ini() must come before propagation");
  long tag = ++tag_;
  // split [0, num) across devices in proportion to capacity
  uint64_t total_cap = 0;
  for (auto& g : devs) total_cap += g.bcap * kOver;
  uint64_t lo = 0;
  std::vector<uint64_t> bs(nb + 1, 0);
  for (int k = 0; k < nb; k++) bs[k + 1] = bs[k] + b[k].num;
  if (bs[nb] < num) throw Error("bunch photon counts do not cover the launch");
  for (size_t d = 0; d < devs.size(); d++) {
    DeviceCtx& g = devs[d];
    uint64_t share = d + 1 == devs.size() ? num - lo : num * (g.bcap * kOver) / total_cap;
    uint64_t hi = lo + share;
    auto& S = g.slot[g.next_slot];
    if (S.busy) throw Error("internal: launch slot still in flight");
    // bunches overlapping [lo, hi), trimmed
    int k0 = (int)(std::upper_bound(bs.begin(), bs.end(), lo) - bs.begin()) - 1;
    int n = 0;
    uint64_t acc = 0;
    for (int k = std::max(k0, 0); k < nb && bs[k] < hi; k++) {
      if ((uint64_t)n >= g.bcap) throw Error("too many bunches for one launch");
      uint64_t a0 = std::max(bs[k], lo), a1 = std::min(bs[k + 1], hi);
      if (a1 <= a0) continue;
      S.hb[n] = b[k];
      S.hb[n].num = (uint32_t)(a1 - a0);
      S.hbstart[n] = acc;
      acc += a1 - a0;
      n++;
    }
    S.hbstart[n] = acc;
    S.num = acc;
    S.nb = n;
    S.tag = tag;
    check(cudaSetDevice(g.dev), "cudaSetDevice");
    check(cudaEventRecord(S.t0, g.st), "event");
    if (n > 0) {
      check(cudaMemcpyAsync(S.bunches, S.hb, n * sizeof(ppcb_bunch), cudaMemcpyHostToDevice, g.st), "H2D bunches");
      check(cudaMemcpyAsync(S.bstart, S.hbstart, (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, g.st), "H2D bstart");
    }
    check(cudaMemsetAsync(S.ctrl, 0, sizeof(ppcb_ctrl), g.st), "memset ctrl");
    if (acc > 0) {
      KArgs a = args_for((int)d);
      a.bunches = S.bunches; a.bstart = S.bstart; a.nb = n; a.num = acc;
      a.hits = S.hits; a.hcap = g.hcap; a.ctrl = S.ctrl;
      check(launch_propagate(a, g.shape, g.st), "propagate launch");
    }
    check(cudaMemcpyAsync(S.hctrl, S.ctrl, sizeof(ppcb_ctrl), cudaMemcpyDeviceToHost, g.st), "D2H ctrl");
    check(cudaEventRecord(S.t1, g.st), "event");
    S.busy = true;
    g.next_slot ^= 1;
    lo = hi;
  }
  queue_.push_back(tag);
  return tag;
}

bool Engine::collect(std::vector<ppcb_hit>& out, RunInfo& info, long* tagp) {
  return collect([&](const ppcb_hit* h, uint64_t n) { out.insert(out.end(), h, h + n); }, info, tagp);
}

bool Engine::collect(const std::function<void(const ppcb_hit*, uint64_t)>& sink, RunInfo& info, long* tagp) {
  if (queue_.empty()) return false;
  long tag = queue_.front();
  queue_.pop_front();
  info = RunInfo();
  for (auto& g : devs) {
    DeviceCtx::Slot* S = nullptr;
    for (auto& s : g.slot) if (s.busy && s.tag == tag) S = &s;
    if (!S) continue;
    check(cudaSetDevice(g.dev), "cudaSetDevice");
    check(cudaEventSynchronize(S->t1), "kernel");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, S->t0, S->t1), "elapsed");
    g.device_ms += ms;
    info.device_ms += ms;
    const ppcb_ctrl c = *S->hctrl;
    uint64_t kept = std::min<uint64_t>(c.hidx, g.hcap);
    if (c.hidx > g.hcap) info.overflow = true;
    if (kept > g.hhits_cap) {
      cudaFreeHost(g.hhits);
      g.hhits_cap = std::max<uint64_t>(kept, g.hhits_cap * 2);
      check(cudaMallocHost((void**)&g.hhits, g.hhits_cap * sizeof(ppcb_hit)), "pinned hits");
    }
    if (kept) {
      check(cudaMemcpyAsync(g.hhits, S->hits, kept * sizeof(ppcb_hit), cudaMemcpyDeviceToHost, g.cp), "D2H hits");
      check(cudaStreamSynchronize(g.cp), "D2H hits");
      sink(g.hhits, kept);
    }
    info.photons += S->num;
    info.hits += c.hidx;
    info.kept += kept;
    info.steps += c.steps;
    info.nan_steps += c.nan_steps;
    info.capped += c.capped;
    S->busy = false;
  }
  if (tagp) *tagp = tag;
  return true;
}

void Engine::launch_device(int d, const ppcb_bunch* dbunch, const uint64_t* dbstart, int nb, uint64_t num,
                           ppcb_hit* dhits, uint64_t hcap, ppcb_ctrl* dctrl, cudaStream_t st) {
  if (!inited_) throw Error("ini() must come before propagation");
  DeviceCtx& g = devs.at(d);
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  KArgs a = args_for(d);
  a.bunches = dbunch; a.bstart = dbstart; a.nb = nb; a.num = num;
  a.hits = dhits; a.hcap = hcap; a.ctrl = dctrl;
  if (num > 0 && nb > 0) check(launch_propagate(a, g.shape, st), "propagate launch");
}

double Engine::total_device_ms() const {
  double t = 0;
  for (auto& g : devs) t += g.device_ms;
  return t;
}

}  // namespace ppcb
