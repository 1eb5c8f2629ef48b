// C ABI of the DirectFit likelihood (declarations: include/ppc_b200.h, "DirectFit
// likelihood on the device").
#include <algorithm>
#include <cmath>
#include <exception>
#include <string>

#include "../../include/ppc_b200.h"
#include "ctx.h"
#include "llh.h"

struct ppcb_llh {
  ppcb::Likelihood* l = nullptr;
};

template <class F>
static int lguard(F&& f) {
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

int ppcb_llh_default_opts(ppcb_llh_opts* o) {
  if (!o) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  *o = ppcb_llh_opts{};
  o->lbin = 0;
  o->sig = 0.10;
  o->qmin = 0.1;
  o->qsat = 500;
  o->drep = 1;
  o->fsep = 1;
  return PPCB_OK;
}

int ppcb_llh_create(ppcb_ctx* c, int device, const ppcb_llh_hit* data, uint64_t n, const ppcb_llh_window* windows,
                    uint64_t nwin, const int32_t* bad, uint64_t nbad, const ppcb_llh_opts* opts, ppcb_llh** out) {
  if (!c || !out || !opts || (n > 0 && !data) || (nwin > 0 && !windows) || (nbad > 0 && !bad)) {
    ppcb_internal_set_error("null argument");
    return PPCB_EARG;
  }
  *out = nullptr;
  return lguard([&] {
    ppcb_llh* h = new ppcb_llh;
    try {
      h->l = new ppcb::Likelihood(c->s.eng, device, data, n, windows, nwin, bad, nbad, *opts);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int ppcb_llh_destroy(ppcb_llh* l) {
  if (!l) return PPCB_OK;
  int r = lguard([&] { delete l->l; });
  delete l;
  return r;
}

int ppcb_llh_get_info(ppcb_llh* l, ppcb_llh_info* info) {
  if (!l || !info) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return lguard([&] {
    ppcb::Likelihood& L = *l->l;
    info->lbin = L.lbin;
    info->t0 = L.t0;
    info->ndof = L.ndof;
    info->doms = (int32_t)L.doms.size();
    info->blocks = (int32_t)L.blocks.size();
    info->errors = L.errors();
  });
}

int ppcb_llh_blocks(ppcb_llh* l, ppcb_llh_block* out, uint64_t cap, uint64_t* n) {
  if (!l || !n || (cap > 0 && !out)) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  const auto& b = l->l->blocks;
  const uint64_t w = std::min<uint64_t>(cap, b.size());
  std::copy(b.begin(), b.begin() + w, out);
  *n = b.size();
  return PPCB_OK;
}

int ppcb_llh_eval_device(ppcb_llh* l, const ppcb_hit* hits, uint64_t n, uint32_t seed, const double* dts, int32_t ndt,
                         double nsim, double* out, void* stream) {
  if (!l || !dts || !out || (n > 0 && !hits)) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return lguard([&] { l->l->eval_device(hits, n, seed, dts, ndt, nsim, out, static_cast<cudaStream_t>(stream)); });
}

int ppcb_llh_eval(ppcb_llh* l, const ppcb_hit* hits, uint64_t n, uint32_t seed, const double* dts, int32_t ndt,
                  double nsim, double* out) {
  if (!l || !dts || !out || (n > 0 && !hits)) { ppcb_internal_set_error("null argument"); return PPCB_EARG; }
  return lguard([&] {
    ppcb::Likelihood& L = *l->l;
    if (ndt < 1 || ndt > PPCB_LLH_MAX_SHIFTS) throw ppcb::Error("likelihood: 1 to 64 time shifts per evaluation", 7);
    L.require_device();
    const int before = L.errors();
    ppcb_hit* dh = nullptr;
    double* dout = nullptr;
    auto release = [&]() {
      if (dh) cudaFree(dh);
      if (dout) cudaFree(dout);
    };
    try {
      ppcb::check(cudaMalloc((void**)&dh, std::max<uint64_t>(n, 1) * sizeof(ppcb_hit)), "likelihood input");
      ppcb::check(cudaMalloc((void**)&dout, ndt * sizeof(double)), "likelihood output");
      if (n) ppcb::check(cudaMemcpy(dh, hits, n * sizeof(ppcb_hit), cudaMemcpyHostToDevice), "H2D hits");
      L.eval_device(dh, n, seed, dts, ndt, nsim, dout, 0);
      ppcb::check(cudaMemcpy(out, dout, ndt * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    } catch (...) {
      release();
      throw;
    }
    release();
    if (L.errors() != before)
      throw ppcb::Error("llf: the Newton iteration left its domain (llh/llh.cxx:649-650)", PPCB_ECONFIG);
  });
}

}  // extern "C"
