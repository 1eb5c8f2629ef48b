// C ABI over Session / Engine (declarations and reference citations: include/ppc_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <string>

#include "../../include/ppc_b200.h"
#include "ctx.h"

static thread_local std::string g_err;

template <class F>
static int guard(F&& f) {
  try {
    f();
    return PPCB_OK;
  } catch (const ppcb::Error& e) {
    g_err = e.what();
    return e.code ? e.code : PPCB_ECONFIG;
  } catch (const std::exception& e) {
    g_err = e.what();
    return PPCB_EARG;
  }
}

#define CTX_OR_FAIL(c) \
  if (!(c)) { g_err = "null context"; return PPCB_EARG; }

extern "C" {

const char* ppcb_last_error(void) { return g_err.c_str(); }

int ppcb_create(ppcb_ctx** out) {
  if (!out) { g_err = "null output"; return PPCB_EARG; }
  return guard([&] {
    cudaSetDeviceFlags(cudaDeviceBlockingSync);
    cudaGetLastError();
    *out = new ppcb_ctx();
  });
}

int ppcb_destroy(ppcb_ctx* c) {
  CTX_OR_FAIL(c);
  int r = guard([&] { c->s.fin(); });
  delete c;
  return r;
}

int ppcb_initialize(ppcb_ctx* c, const char* dir, float enh) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.initialize(dir ? std::string(dir) : std::string(), enh); });
}

int ppcb_choose(ppcb_ctx* c, int device) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.choose(device); });
}

int ppcb_set_seed(ppcb_ctx* c, uint32_t seed) {
  CTX_OR_FAIL(c);
  return guard([&] {
    c->s.eng.sv = seed;
    if (c->s.eng.ready()) c->s.eng.reset_streams();
  });
}

int ppcb_set_options(ppcb_ctx* c, int deterministic, uint32_t max_steps, int blocks_per_sm) {
  CTX_OR_FAIL(c);
  return guard([&] {
    if (deterministic < 0 || deterministic > 2) throw ppcb::Error("deterministic: 0, 1 or 2", PPCB_EARG);
    c->s.eng.deterministic = deterministic;
    c->s.eng.max_steps = max_steps;
    c->s.eng.blocks_per_sm = blocks_per_sm;
  });
}

int ppcb_ini(ppcb_ctx* c) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.ini(); });
}

int ppcb_fin(ppcb_ctx* c) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.fin(); });
}

int ppcb_get_info(ppcb_ctx* c, ppcb_info* o) {
  CTX_OR_FAIL(c);
  if (!o) { g_err = "null output"; return PPCB_EARG; }
  return guard([&] {
    memset(o, 0, sizeof(*o));
    const ppcb::Engine& e = c->s.eng;
    o->max_bunch_size = e.pmxo;
    o->workgroup_size = e.devs.empty() ? 0 : e.devs[0].shape.threads;
    o->total_device_ms = e.total_device_ms();
    o->max_photons = e.pmax;
    o->hit_capacity = e.devs.empty() ? 0 : e.devs[0].hcap;
    o->devices = (int32_t)e.devs.size();
    o->threads = e.devs.empty() ? 0 : e.devs[0].T;
    o->blocks = e.devs.empty() ? 0 : e.devs[0].shape.blocks;
    if (e.ready()) {
      int regs = 0, mt = 0;
      size_t sm = 0, lm = 0;
      if (ppcb::propagate_attributes(&regs, &mt, &sm, &lm) == cudaSuccess) o->regs = regs;
    }
    o->gsize = e.cfg.p.gsize;
    o->size = e.cfg.p.size;
    o->nstr = e.cfg.p.nstr;
    o->rsize = e.cfg.p.rsize;
    o->eff = e.cfg.eff;
    o->ovr = e.cfg.ovr;
    o->seed = e.sv;
    o->nextgen = e.cfg.nextgen ? 1 : 0;
  });
}

int ppcb_flset(ppcb_ctx* c, int str, int om, ppcb_dom* out) {
  CTX_OR_FAIL(c);
  return guard([&] {
    const ppcb_dom& d = c->s.flset(str, om);
    if (out) *out = d;
  });
}

int ppcb_fldir(ppcb_ctx* c, float dir[3]) {
  CTX_OR_FAIL(c);
  return guard([&] {
    const float* d = c->s.fldir();
    for (int i = 0; i < 3; i++) dir[i] = d[i];
  });
}

int ppcb_flshift(ppcb_ctx* c, float m[3], float n[3], float* r) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.flshift(m, n, r); });
}

int ppcb_sett(ppcb_ctx* c, float nx, float ny, float nz, int32_t a, uint64_t b, int32_t frame, double t0) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.sett(nx, ny, nz, std::make_pair((int)a, (unsigned long long)b), frame, t0); });
}

int ppcb_addp(ppcb_ctx* c, float x, float y, float z, float t, float E, float dr, int32_t type, float scale) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.addp(x, y, z, t, E, dr, type, scale); });
}

int ppcb_addp_clst(ppcb_ctx* c, float x, float y, float z, float t, uint64_t n, float dr, float beta) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.addp_clst(x, y, z, t, n, dr, beta); });
}

int ppcb_addp_mopo(ppcb_ctx* c, float x, float y, float z, float t, float light, float length, float beta,
                   float tau, float fr) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.addp_mopo(x, y, z, t, light, length, beta, tau, fr); });
}

int ppcb_flone(ppcb_ctx* c, uint64_t num) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.flone(num); });
}

int ppcb_eout(ppcb_ctx* c) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.eout(); });
}

int ppcb_back_end(ppcb_ctx* c, const ppcb_hit* hits, uint64_t n) {
  CTX_OR_FAIL(c);
  if (n > 0 && !hits) { g_err = "null argument"; return PPCB_EARG; }
  return guard([&] {
    std::vector<ppcb_hit> v(hits, hits + n);
    c->s.print(v, c->s.flne);
  });
}

int ppcb_efin(ppcb_ctx* c) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.efin(); });
}

int ppcb_set_res(ppcb_ctx* c, float t, float cz) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.set_res(t, cz); });
}

float ppcb_xrnd(ppcb_ctx* c) { return c ? c->s.xrnd() : 0.f; }

int ppcb_hitz_count(ppcb_ctx* c, uint64_t* n) {
  CTX_OR_FAIL(c);
  return guard([&] {
    uint64_t k = 0;
    for (auto& e : *c->s.hitz) k += e.second.size();
    *n = k;
  });
}

int ppcb_hitz_copy(ppcb_ctx* c, ppcb_hitz_rec* out, uint64_t cap, uint64_t* written) {
  CTX_OR_FAIL(c);
  return guard([&] {
    uint64_t k = 0;
    for (auto& e : *c->s.hitz)
      for (auto& po : e.second) {
        if (k < cap) {
          ppcb_hitz_rec& r = out[k];
          r.track_first = e.first.track.first;
          r.track_second = e.first.track.second;
          r.frame = e.first.track.frame;
          r.t0 = e.first.track.t0;
          r.str = e.first.omkey.str;
          r.om = e.first.omkey.dom;
          r.pmt = e.first.pmt;
          r.dir = e.first.dir;
          r.time = e.first.time;
          memcpy(r.r, po.r, sizeof(r.r));
          memcpy(r.n, po.n, sizeof(r.n));
        }
        k++;
      }
    if (written) *written = k < cap ? k : cap;
  });
}

int ppcb_keep_raw(ppcb_ctx* c, int keep) {
  CTX_OR_FAIL(c);
  c->s.keep_raw = keep != 0;
  return PPCB_OK;
}

int ppcb_raw_count(ppcb_ctx* c, uint64_t* n) {
  CTX_OR_FAIL(c);
  *n = c->s.raw_.size();
  return PPCB_OK;
}

int ppcb_raw_copy(ppcb_ctx* c, ppcb_hit* out, uint64_t cap, uint64_t* written) {
  CTX_OR_FAIL(c);
  uint64_t k = std::min<uint64_t>(cap, c->s.raw_.size());
  if (k) memcpy(out, c->s.raw_.data(), k * sizeof(ppcb_hit));
  if (written) *written = k;
  return PPCB_OK;
}

static void to_c(const ppcb::RunInfo& r, ppcb_run_info* o) {
  o->photons = r.photons;
  o->hits = r.hits;
  o->kept = r.kept;
  o->steps = r.steps;
  o->nan_steps = r.nan_steps;
  o->capped = r.capped;
  o->device_ms = r.device_ms;
}

int ppcb_last_run(ppcb_ctx* c, ppcb_run_info* last, ppcb_run_info* total) {
  CTX_OR_FAIL(c);
  if (last) to_c(c->s.last, last);
  if (total) to_c(c->s.total, total);
  return PPCB_OK;
}

int ppcb_propagate(ppcb_ctx* c, const ppcb_bunch* bunches, int32_t nb, ppcb_hit* hits, uint64_t cap,
                   uint64_t* nhits, ppcb_run_info* info) {
  CTX_OR_FAIL(c);
  if (nb < 0 || (nb > 0 && !bunches)) { g_err = "bad bunch list"; return PPCB_EARG; }
  return guard([&] {
    ppcb::Engine& e = c->s.eng;
    if (!e.ready()) throw ppcb::Error("ppcb_ini() must come before propagation", PPCB_ESTATE);
    ppcb::RunInfo tot;
    uint64_t produced = 0, stored = 0;
    // kept hits go from the pinned staging buffer straight into the caller's array
    auto sink = [&](const ppcb_hit* h, uint64_t n) {
      if (hits && stored < cap) std::memcpy(hits + stored, h, std::min<uint64_t>(n, cap - stored) * sizeof(ppcb_hit));
      stored += n;
    };
    auto drain_one = [&]() {
      ppcb::RunInfo ri;
      e.collect(sink, ri);
      tot.photons += ri.photons; tot.hits += ri.hits; tot.kept += ri.kept; tot.steps += ri.steps;
      tot.nan_steps += ri.nan_steps; tot.capped += ri.capped; tot.device_ms += ri.device_ms;
      produced += ri.hits;
    };
    // batches of at most pmax photons and pmxo bunches (gpu/f2k.cxx:377-385)
    std::vector<ppcb_bunch> batch;
    uint64_t pn = 0;
    auto flush = [&]() {
      if (pn == 0) { batch.clear(); return; }
      if (e.in_flight() >= 2) drain_one();
      e.submit(batch.data(), (int)batch.size(), pn);
      batch.clear();
      pn = 0;
    };
    for (int k = 0; k < nb; k++) {
      uint64_t left = bunches[k].num;
      do {
        ppcb_bunch b = bunches[k];
        b.num = (uint32_t)std::min<uint64_t>(e.pmax - pn, left);
        left -= b.num;
        pn += b.num;
        batch.push_back(b);
        if (pn == e.pmax || batch.size() == e.pmxo) flush();
      } while (left > 0);
    }
    flush();
    while (e.in_flight() > 0) drain_one();
    if (nhits) *nhits = produced;
    if (info) to_c(tot, info);
  });
}

int ppcb_propagate_device(ppcb_ctx* c, int device, const ppcb_bunch* bunches, const uint64_t* bstart, int32_t nb,
                          uint64_t num, ppcb_hit* hits, uint64_t hcap, ppcb_ctrl* ctrl, void* stream) {
  CTX_OR_FAIL(c);
  if (!ctrl || (num > 0 && (!bunches || !bstart || nb <= 0))) { g_err = "bad arguments"; return PPCB_EARG; }
  return guard([&] {
    if (!c->s.eng.ready()) throw ppcb::Error("ppcb_ini() must come before propagation", PPCB_ESTATE);
    if (device < 0 || device >= (int)c->s.eng.devs.size()) throw ppcb::Error("bad device index", PPCB_EARG);
    c->s.eng.launch_device(device, bunches, bstart, nb, num, hits, hcap, ctrl, (cudaStream_t)stream);
  });
}

int ppcb_rng_get(ppcb_ctx* c, int device, uint64_t* rs, uint64_t n) {
  CTX_OR_FAIL(c);
  return guard([&] {
    auto& g = c->s.eng.devs.at(device);
    if (n > (uint64_t)g.T) n = g.T;
    ppcb::check(cudaSetDevice(g.dev), "cudaSetDevice");
    ppcb::check(cudaMemcpy(rs, g.rs, n * 8, cudaMemcpyDeviceToHost), "rng get");
  });
}

int ppcb_rng_set(ppcb_ctx* c, int device, const uint64_t* rs, uint64_t n) {
  CTX_OR_FAIL(c);
  return guard([&] {
    auto& g = c->s.eng.devs.at(device);
    if (n > (uint64_t)g.T) n = g.T;
    ppcb::check(cudaSetDevice(g.dev), "cudaSetDevice");
    ppcb::check(cudaMemcpy(g.rs, rs, n * 8, cudaMemcpyHostToDevice), "rng set");
  });
}

int ppcb_rng_reset(ppcb_ctx* c) {
  CTX_OR_FAIL(c);
  return guard([&] { c->s.eng.reset_streams(); });
}

int ppcb_table(ppcb_ctx* c, const char* name, const void** ptr, uint64_t* bytes) {
  CTX_OR_FAIL(c);
  return guard([&] {
    const ppcb::Config& f = c->s.eng.cfg;
    std::string n(name);
    const void* p = nullptr;
    uint64_t b = 0;
#define T(nm, vec) else if (n == nm) { p = f.vec.data(); b = f.vec.size() * sizeof(f.vec[0]); }
    if (n == "params") { p = &f.p; b = sizeof(f.p); }
    T("az", az) T("lr", lr) T("ls", ls) T("is", is) T("mcol", mcol) T("sc", sc) T("lp", lp) T("absca", absca)
    T("wmeta", wmeta) T("oms", oms) T("rm", rm) T("wvs", wvs) T("bfrt", bfrt)
    else if (n == "eff") { p = &f.eff; b = sizeof(f.eff); }
    else throw ppcb::Error("unknown table " + n, PPCB_EARG);
#undef T
    *ptr = p;
    *bytes = b;
  });
}

int ppcb_generate_device(ppcb_ctx* c, int device, const ppcb_bunch* bunches, const uint64_t* bstart, int32_t nb,
                         uint64_t num, void* out, void* stream) {
  CTX_OR_FAIL(c);
  return guard([&] {
    auto& e = c->s.eng;
    if (!e.ready()) throw ppcb::Error("ppcb_ini() must come before propagation", PPCB_ESTATE);
    auto& g = e.devs.at(device);
    if (num > (uint64_t)g.T) throw ppcb::Error("generate: at most one photon per thread", PPCB_EARG);
    ppcb::check(cudaSetDevice(g.dev), "cudaSetDevice");
    ppcb::KArgs a = e.args_for(device);
    a.bunches = bunches; a.bstart = bstart; a.nb = nb; a.num = num;
    ppcb::check(ppcb::launch_generate(a, g.shape, out, (cudaStream_t)stream), "generate launch");
  });
}

int ppcb_index_probe_device(ppcb_ctx* c, int device, const void* pos, int32_t n, int32_t* out_i, float* out_f,
                            void* stream) {
  CTX_OR_FAIL(c);
  return guard([&] {
    auto& e = c->s.eng;
    if (!e.ready()) throw ppcb::Error("ppcb_ini() must come before propagation", PPCB_ESTATE);
    auto& g = e.devs.at(device);
    ppcb::check(cudaSetDevice(g.dev), "cudaSetDevice");
    ppcb::KArgs a = e.args_for(device);
    ppcb::check(ppcb::launch_index_probe(a, (const float4*)pos, n, out_i, out_f, (cudaStream_t)stream),
                "index probe launch");
  });
}

int ppcb_string_grid_probe(ppcb_ctx* c, const void* pos, int32_t n, int32_t* out) {
  CTX_OR_FAIL(c);
  if (n < 0 || (n > 0 && (!pos || !out))) { g_err = "bad arguments"; return PPCB_EARG; }
  return guard([&] {
    const ppcb::Config& f = c->s.eng.cfg;
    struct HostTab {
      const ppcb::Config& f;
      uint32_t cell(int k) const { return f.sg_cells[k]; }
      const ppcb::StrGroup& group(int m) const { return f.sg_groups[m]; }
    } t{f};
    const float* p = static_cast<const float*>(pos);
    for (int32_t k = 0; k < n; k++) {
      const float* r = p + 8 * k;
      out[k] = ppcb::sg_may_reach(f.sg, t, r[0], r[1], r[4], r[5], r[6], r[7]) ? 1 : 0;
    }
  });
}

}  // extern "C"

void ppcb_internal_set_error(const std::string& msg) { g_err = msg; }
