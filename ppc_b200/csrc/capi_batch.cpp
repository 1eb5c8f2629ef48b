// C ABI of the batched launch (declarations: include/ppc_b200.h, "batched events").
#include <algorithm>
#include <cstring>
#include <memory>
#include <exception>
#include <string>

#include "../../include/ppc_b200.h"
#include "batch.h"
#include "ctx.h"
#include "session.h"

struct ppcb_batch {
  ppcb::Batch* b = nullptr;
  ppcb::BatchResult last;
  uint32_t events = 0;
};

template <class F>
static int bguard(F&& f) {
  try {
    f();
    return PPCB_OK;
  } catch (const ppcb::Error& e) {
    ppcb_internal_set_error(e.what());
    return e.code ? e.code : PPCB_ECONFIG;
  } catch (const std::exception& e) {
    ppcb_internal_set_error(e.what());
    return PPCB_EARG;
  }
}

extern "C" {

int ppcb_batch_create(ppcb_ctx* c, int device, uint32_t max_events, uint32_t max_bunches, uint64_t hit_capacity,
                      ppcb_batch** out) {
  if (!c || !out) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    ppcb_batch* x = new ppcb_batch();
    try {
      x->b = new ppcb::Batch(c->s.eng, device, max_events, max_bunches, hit_capacity);
    } catch (...) {
      delete x;
      throw;
    }
    *out = x;
  });
}

int ppcb_batch_destroy(ppcb_batch* x) {
  if (!x) return PPCB_OK;
  int r = bguard([&] { delete x->b; });
  delete x;
  return r;
}

int ppcb_batch_set_graph(ppcb_batch* x, int use_graph) {
  if (!x) { ppcb_internal_set_error("null batch"); return PPCB_EARG; }
  x->b->use_graph = use_graph != 0;
  return PPCB_OK;
}

int ppcb_batch_run(ppcb_batch* x, const ppcb_bunch* bunches, int32_t nb, uint32_t events, double hits_per_photon,
                   ppcb_batch_info* info) {
  if (!x || !bunches) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    x->b->run(bunches, nb, events, x->last, hits_per_photon);
    x->events = events;
    if (info) {
      memset(info, 0, sizeof(*info));
      info->photons = x->last.photons;
      info->steps = x->last.steps;
      info->kept = x->last.hits.size();
      uint64_t produced = 0;
      for (uint32_t v : x->last.produced) produced += v;
      info->hits = produced;
      info->overflowed = x->last.overflowed;
      info->device_ms = x->last.device_ms;
      info->graph_ms = x->last.graph_ms;
    }
  });
}

int ppcb_batch_counts(ppcb_batch* x, uint32_t* produced, uint64_t* offsets) {
  if (!x) { ppcb_internal_set_error("null batch"); return PPCB_EARG; }
  if (produced) memcpy(produced, x->last.produced.data(), x->events * sizeof(uint32_t));
  if (offsets) memcpy(offsets, x->last.offset.data(), (x->events + 1) * sizeof(uint64_t));
  return PPCB_OK;
}

int ppcb_batch_hits(ppcb_batch* x, ppcb_hit* out, uint64_t cap, uint64_t* n) {
  if (!x) { ppcb_internal_set_error("null batch"); return PPCB_EARG; }
  uint64_t k = std::min<uint64_t>(cap, x->last.hits.size());
  if (k && out) memcpy(out, x->last.hits.data(), k * sizeof(ppcb_hit));
  if (n) *n = x->last.hits.size();
  return PPCB_OK;
}

int ppcb_batch_autotune(ppcb_batch* x, const ppcb_bunch* bunches, int32_t nb, uint32_t events, uint64_t sample_photons,
                        ppcb_tune_info* out) {
  if (!x || !bunches) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    ppcb::TuneResult t = x->b->autotune(bunches, nb, events, sample_photons);
    if (out) {
      out->threads = t.threads;
      out->blocks_per_sm = t.blocks_per_sm;
      out->refill_below = t.refill_below;
      out->photons_per_s = t.photons_per_s;
    }
  });
}

int ppcb_set_ice(ppcb_ctx* c, const float* be, const float* ba) {
  if (!c) { ppcb_internal_set_error("null context"); return PPCB_EARG; }
  return bguard([&] { c->s.eng.set_ice(be, ba); });
}

int ppcb_get_ice(ppcb_ctx* c, float* be, float* ba, int32_t* size) {
  if (!c) { ppcb_internal_set_error("null context"); return PPCB_EARG; }
  return bguard([&] {
    const ppcb::Config& f = c->s.eng.cfg;
    if (size) *size = f.p.size;
    for (int j = 0; j < f.p.size; j++) {
      if (be) be[j] = f.be[j];
      if (ba) ba[j] = f.ba[j];
    }
  });
}

int ppcb_gradient(ppcb_ctx* c, const ppcb_bunch* bunches, int32_t nb, uint32_t events, const float* observed,
                  const float* weights, double scale, uint64_t hit_cap, uint32_t* counts, double* g_be, double* g_ba,
                  ppcb_grad_info* info) {
  if (!c || !bunches) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    ppcb::Engine::Grad r = c->s.eng.gradient(bunches, nb, events, observed, weights, scale, hit_cap);
    const int size = c->s.eng.cfg.p.size;
    if (counts) memcpy(counts, r.counts.data(), r.counts.size() * sizeof(uint32_t));
    if (g_be) memcpy(g_be, r.g_be.data(), size * sizeof(double));
    if (g_ba) memcpy(g_ba, r.g_ba.data(), size * sizeof(double));
    if (info) {
      info->ll = r.ll;
      info->photons = r.photons;
      info->hits = r.hits;
      info->replayed = r.replayed;
      info->unmatched = r.unmatched;
      info->steps = r.steps;
      info->forward_ms = r.forward_ms;
      info->backward_ms = r.backward_ms;
    }
  });
}

struct ppcb_gradgraph {
  ppcb_ctx* c;
  std::unique_ptr<ppcb::GradGraph> g;
};

int ppcb_gradgraph_create(ppcb_ctx* c, const ppcb_bunch* bunches, int32_t nb, uint32_t events, const float* observed,
                          double scale, uint64_t hit_cap, ppcb_gradgraph** out) {
  if (!c || !bunches || !observed || !out) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    std::unique_ptr<ppcb_gradgraph> h(new ppcb_gradgraph{c, nullptr});
    h->g.reset(new ppcb::GradGraph(c->s.eng, bunches, nb, events, observed, scale, hit_cap));
    *out = h.release();
  });
}

int ppcb_gradgraph_run(ppcb_gradgraph* g, const float* be, const float* ba, uint32_t* counts, double* g_be,
                       double* g_ba, ppcb_grad_info* info) {
  if (!g) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    ppcb::Engine::Grad r = g->g->run(be, ba, counts != nullptr);
    const int size = g->c->s.eng.cfg.p.size;
    if (counts) memcpy(counts, r.counts.data(), r.counts.size() * sizeof(uint32_t));
    if (g_be) memcpy(g_be, r.g_be.data(), size * sizeof(double));
    if (g_ba) memcpy(g_ba, r.g_ba.data(), size * sizeof(double));
    if (info) {
      info->ll = r.ll;
      info->photons = r.photons;
      info->hits = r.hits;
      info->replayed = r.replayed;
      info->unmatched = r.unmatched;
      info->steps = r.steps;
      info->forward_ms = r.forward_ms;
      info->backward_ms = r.backward_ms;
    }
  });
}

int ppcb_gradgraph_destroy(ppcb_gradgraph* g) {
  if (!g) return PPCB_OK;
  return bguard([&] { delete g; });
}

}  // extern "C"

extern "C" {

int ppcb_accept_device(ppcb_ctx* c, int device, const ppcb_hit* hits, uint64_t n, uint32_t seed, ppcb_acc_hit* out,
                       unsigned long long* count, void* stream) {
  if (!c || (n > 0 && (!hits || !out)) || !count) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    if (device < 0 || device >= (int)c->s.eng.devs.size()) throw ppcb::Error("bad device index", PPCB_EARG);
    c->s.eng.accept(device, hits, n, seed, out, count, static_cast<cudaStream_t>(stream));
  });
}

int ppcb_accept(ppcb_ctx* c, const ppcb_hit* hits, uint64_t n, uint32_t seed, ppcb_acc_hit* out, uint64_t cap,
                uint64_t* nout) {
  if (!c || (n > 0 && !hits) || !nout) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return bguard([&] {
    ppcb::Engine& e = c->s.eng;
    if (!e.ready()) throw ppcb::Error("ppcb_ini() must come before the back end", PPCB_ESTATE);
    ppcb::check(cudaSetDevice(e.devs[0].dev), "cudaSetDevice");
    ppcb_hit* dh = nullptr;
    ppcb_acc_hit* dout = nullptr;
    unsigned long long* dcnt = nullptr;
    auto release = [&]() {
      if (dh) cudaFree(dh);
      if (dout) cudaFree(dout);
      if (dcnt) cudaFree(dcnt);
    };
    try {
      ppcb::check(cudaMalloc((void**)&dh, std::max<uint64_t>(n, 1) * sizeof(ppcb_hit)), "back end input");
      ppcb::check(cudaMalloc((void**)&dout, std::max<uint64_t>(n, 1) * sizeof(ppcb_acc_hit)), "back end output");
      ppcb::check(cudaMalloc((void**)&dcnt, sizeof(unsigned long long)), "back end count");
      if (n) ppcb::check(cudaMemcpy(dh, hits, n * sizeof(ppcb_hit), cudaMemcpyHostToDevice), "H2D hits");
      e.accept(0, dh, n, seed, dout, dcnt, 0);
      unsigned long long k = 0;
      ppcb::check(cudaMemcpy(&k, dcnt, sizeof(k), cudaMemcpyDeviceToHost), "D2H count");
      const uint64_t w = std::min<uint64_t>(k, cap);
      if (w && out) ppcb::check(cudaMemcpy(out, dout, w * sizeof(ppcb_acc_hit), cudaMemcpyDeviceToHost), "D2H");
      *nout = k;
    } catch (...) {
      release();
      throw;
    }
    release();
  });
}

}  // extern "C"

extern "C" {

int ppcb_sources_device(ppcb_ctx* c, int device, const ppcb_source* src, uint64_t ns, uint32_t seed,
                        ppcb_bunch* out, uint64_t* bstart, uint64_t cap, uint64_t* counts, void* stream) {
  if (!c || (ns > 0 && !src) || (cap > 0 && !out) || !bstart || !counts) {
    ppcb_internal_set_error("null argument");
    return PPCB_EARG;
  }
  return bguard([&] {
    if (device < 0 || device >= (int)c->s.eng.devs.size()) throw ppcb::Error("bad device index", PPCB_EARG);
    c->s.eng.sources(device, src, ns, seed, out, bstart, cap, counts, static_cast<cudaStream_t>(stream));
  });
}

int ppcb_sources(ppcb_ctx* c, const ppcb_source* src, uint64_t ns, uint32_t seed, ppcb_bunch* out, uint64_t* bstart,
                 uint64_t cap, uint64_t* nb, uint64_t* num) {
  if (!c || (ns > 0 && !src) || (cap > 0 && (!out || !bstart)) || !nb || !num) {
    ppcb_internal_set_error("null argument");
    return PPCB_EARG;
  }
  return bguard([&] {
    ppcb::Engine& e = c->s.eng;
    if (!e.ready()) throw ppcb::Error("ppcb_ini() must come before the front end", PPCB_ESTATE);
    ppcb::check(cudaSetDevice(e.devs[0].dev), "cudaSetDevice");
    const int before = e.front_errors(0);
    ppcb_source* ds = nullptr;
    ppcb_bunch* dout = nullptr;
    uint64_t* dbs = nullptr;
    uint64_t* dcnt = nullptr;
    auto release = [&]() {
      for (void* p : {(void*)ds, (void*)dout, (void*)dbs, (void*)dcnt})
        if (p) cudaFree(p);
    };
    try {
      ppcb::check(cudaMalloc((void**)&ds, std::max<uint64_t>(ns, 1) * sizeof(ppcb_source)), "front end input");
      ppcb::check(cudaMalloc((void**)&dout, std::max<uint64_t>(cap, 1) * sizeof(ppcb_bunch)), "front end output");
      ppcb::check(cudaMalloc((void**)&dbs, (cap + 1) * sizeof(uint64_t)), "front end output");
      ppcb::check(cudaMalloc((void**)&dcnt, 2 * sizeof(uint64_t)), "front end counts");
      if (ns) ppcb::check(cudaMemcpy(ds, src, ns * sizeof(ppcb_source), cudaMemcpyHostToDevice), "H2D sources");
      e.sources(0, ds, ns, seed, dout, dbs, cap, dcnt, 0);
      uint64_t cnt[2];
      ppcb::check(cudaMemcpy(cnt, dcnt, sizeof(cnt), cudaMemcpyDeviceToHost), "D2H counts");
      const uint64_t w = std::min<uint64_t>(cnt[0], cap);
      if (w) ppcb::check(cudaMemcpy(out, dout, w * sizeof(ppcb_bunch), cudaMemcpyDeviceToHost), "D2H bunches");
      if (cap > 0 || cnt[0] == 0)
        if (bstart)
          ppcb::check(cudaMemcpy(bstart, dbs, (w + (cnt[0] <= cap ? 1 : 0)) * sizeof(uint64_t),
                                 cudaMemcpyDeviceToHost), "D2H bunch starts");
      *nb = cnt[0];
      *num = cnt[1];
    } catch (...) {
      release();
      throw;
    }
    release();
    if (e.front_errors(0) != before)
      throw ppcb::Error("front end: a source's sampling failed (negative type, bad count or no convergence)",
                        PPCB_EARG);
  });
}

int ppcb_f2k_sources(const char* text, uint64_t len, uint32_t first_segment, ppcb_source* out, uint64_t cap,
                     uint64_t* n, uint64_t* lines) {
  if ((len > 0 && !text) || (cap > 0 && !out) || !n || !lines) {
    ppcb_internal_set_error("null argument");
    return PPCB_EARG;
  }
  return bguard([&] {
    uint64_t k = 0, line = 0, pos = 0;
    while (pos < len) {
      uint64_t end = pos;
      while (end < len && text[end] != '\n') end++;
      const std::string in(text + pos, end - pos);
      pos = end + 1;
      const uint32_t seg = first_segment + (uint32_t)line++;
      ppcb::F2kTrack tr;
      if (!ppcb::parse_f2k_track(in, tr) || tr.type == -1) continue;
      if (k < cap) {
        ppcb_source s;
        std::memset(&s, 0, sizeof(s));
        s.r[0] = tr.x; s.r[1] = tr.y; s.r[2] = tr.z; s.r[3] = tr.t;
        s.n[0] = tr.n[0]; s.n[1] = tr.n[1]; s.n[2] = tr.n[2];
        s.q = seg;
        if (tr.type == -2) {
          s.kind = PPCB_SRC_POINT;
          s.amount = (double)(unsigned long long)tr.E;
        } else {
          s.kind = PPCB_SRC_PARTICLE;
          s.type = tr.type;
          s.amount = tr.E;
          s.dr = tr.l;
          s.scale = 1;
        }
        out[k] = s;
      }
      k++;
    }
    *n = k;
    *lines = line;
  });
}

}  // extern "C"
