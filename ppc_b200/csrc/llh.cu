// Simulated side of DirectFit's likelihood on the GPU, three kernels per evaluation:
//   k_llh_fill    one thread per kernel-level hit: the back end's acceptance (backend.cuh,
//                 the same per-hit streams as Engine::accept), then for each time shift the
//                 hit's bin round((t + dt - t0) / lbin) and, when it lies in the DOM's
//                 window and outside its errata windows, +1 on that bin's block (dat::fill,
//                 dat::join, llh/llh.cxx:469-482, 614-621).  Simulated hits on DOMs without
//                 observed pulses count toward the no-hit total (cascade::ppc,
//                 llh/llh.cxx:1694-1700).
//   k_llh_terms   one thread per (shift, block): llf (llh/llh.cxx:637-662) in FP64, a
//                 fixed-order tree sum per CTA.
//   k_llh_final   one CTA per shift: the CTA sums in a fixed order, the no-hit term and the
//                 division by ndof (fllh, llh/llh.cxx:1075-1082).
// Counts are integers (one per accepted hit), so the binning is exact; every sum runs in a
// fixed order, so an evaluation is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "backend.cuh"
#include "engine.h"
#include "llh.h"

namespace ppcb {

struct LlhDevice {
  int32_t* dom_slot = nullptr;
  LlhDom* doms = nullptr;
  int32_t* bin_block = nullptr;
  double* block_dat = nullptr;
  int32_t* block_dom = nullptr;
  double2* win = nullptr;
  unsigned int* simc = nullptr;      // [shift][block] simulated counts
  unsigned int* stot = nullptr;      // [shift][DOM] simulated counts in the DOM's window
  unsigned long long* nohit = nullptr;
  double* partial = nullptr;         // [shift][CTA] sums of llf terms
  int* errors = nullptr;
  int ndt_cap = 0;
  ~LlhDevice() {
    for (void* p : {(void*)dom_slot, (void*)doms, (void*)bin_block, (void*)block_dat, (void*)block_dom, (void*)win,
                    (void*)simc, (void*)stot, (void*)nohit, (void*)partial, (void*)errors})
      if (p) cudaFree(p);
  }
};

void LlhDeviceFree::operator()(LlhDevice* p) const { delete p; }

namespace {

constexpr int kThreads = 256;
constexpr int kMaxNewton = 200;

struct FillArgs {
  BackArgs A;
  const int32_t* dom_slot;
  const LlhDom* doms;
  const int32_t* bin_block;
  const double2* win;
  unsigned int* simc;
  unsigned int* stot;
  unsigned long long* nohit;
  double t0, lbin;
  int nblocks, ndom, ndt, unh, norm;
  double dt[PPCB_LLH_MAX_SHIFTS];
};

__global__ void __launch_bounds__(kThreads) k_llh_fill(FillArgs F) {
  __shared__ unsigned int s_nohit;
  if (threadIdx.x == 0) s_nohit = 0;
  __syncthreads();
  const uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  ppcb_acc_hit o;
  if (k < F.A.n && accept_one(F.A, k, o)) {
    const int slot = F.dom_slot[o.i];
    if (slot == -1) {
      if (F.unh) atomicAdd(&s_nohit, 1u);
    } else if (slot >= 0) {
      const LlhDom D = F.doms[slot];
      for (int j = 0; j < F.ndt; j++) {
        const double t = (double)o.t + F.dt[j];
        bool ok = true;
        for (int w = 0; w < D.nwin; w++) {
          const double2 x = F.win[D.win0 + w];
          if (x.x <= t && t < x.y) ok = false;
        }
        if (!ok) continue;
        const double b = round((t - F.t0) / F.lbin);
        if (!(b >= D.n1 && b < D.n2)) continue;  // also drops NaN times
        const int blk = F.bin_block[D.bin0 + (int)b - D.n1];
        atomicAdd(&F.simc[(size_t)j * F.nblocks + blk], 1u);
        if (F.norm) atomicAdd(&F.stot[(size_t)j * F.ndom + slot], 1u);  // only norm reads it
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_nohit) atomicAdd(F.nohit, (unsigned long long)s_nohit);
}

// llf of llh/llh.cxx:637-662: the saturated likelihood of s simulated (nsim repetitions)
// against d observed (ndat repetitions) with a log-normal model error sig; the common rate
// is found by Newton's method.  A step that leaves the domain (the reference stops the
// program there) or that has not converged in kMaxNewton steps gives NaN and sets `err`.
__device__ double llf(double s, double d, double nsim, double ndat, double sig, bool& err) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  if (s < 0 || d < 0) {
    err = true;
    return nan;
  }
  if (s == 0 && d == 0) return 0;
  const double s2 = sig * sig, tol = 1.e-8;
  const double sd = s + d, ntot = ndat + nsim;
  double ls = sd / ntot, ld = ls, llx = 0;
  if (sig > 0) {
    double dls;
    int it = 0;
    do {
      const double f = nsim * ls - s - log(ld / ls) / s2;
      const double df = 1 + (1 / (ndat * ld) + 1 / (nsim * ls)) / s2;
      dls = -f / (nsim * df);
      ls += dls;
      ld = (sd - nsim * ls) / ndat;
      if (ls < 0 || ld < 0 || ++it > kMaxNewton) {
        err = true;
        return nan;
      }
    } while (fabs(dls) > tol * ls);
    const double lr = log(ld / ls);
    llx = lr * lr / (2 * s2);
  }
  double lls = 0, lld = 0;
  if (s > 0) lls = s * log((s / nsim) / ls);
  if (d > 0) lld = d * log((d / ndat) / ld);
  return llx + lls + lld;
}

__device__ double cta_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  return sh[0];
}

struct TermArgs {
  const unsigned int* simc;
  const unsigned int* stot;
  const double* block_dat;
  const int32_t* block_dom;
  const LlhDom* doms;
  double* partial;
  int* errors;
  double nsim, ndat, sig;
  int nblocks, ndom, norm;
};

__global__ void __launch_bounds__(kThreads) k_llh_terms(TermArgs T) {
  __shared__ double sh[kThreads];
  const int b = blockIdx.x * kThreads + threadIdx.x, j = blockIdx.y;
  double v = 0;
  bool err = false;
  if (b < T.nblocks) {
    const double s = T.simc[(size_t)j * T.nblocks + b];
    double nsim = T.nsim;
    bool use = true;
    if (T.norm) {
      const int slot = T.block_dom[b];
      const double st = T.stot[(size_t)j * T.ndom + slot];
      if (st > 0) nsim = st * T.ndat / T.doms[slot].dtot;
      else use = false;  // dat::llh returns 0 for a DOM without simulated hits
    }
    if (use) v = llf(s, T.block_dat[b], nsim, T.ndat, T.sig, err);
  }
  if (err) atomicAdd(T.errors, 1);
  const double total = cta_sum(v, sh);
  if (threadIdx.x == 0) T.partial[(size_t)j * gridDim.x + blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads) k_llh_final(const double* partial, int nparts,
                                                        const unsigned long long* nohit, int norm, double nsim,
                                                        double ndat, double sig, int ndof, int* errors, double* out) {
  __shared__ double sh[kThreads];
  const int j = blockIdx.x;
  double v = 0;
  for (int c = threadIdx.x; c < nparts; c += kThreads) v += partial[(size_t)j * nparts + c];
  const double total = cta_sum(v, sh);
  if (threadIdx.x == 0) {
    double nh = 0;
    bool err = false;
    if (!norm) nh = llf((double)*nohit, 0, nsim, ndat, sig, err);
    if (err) atomicAdd(errors, 1);
    out[j] = (nh + total) / ndof;
  }
}

template <class T>
T* upload_vec(const std::vector<T>& v, const char* what) {
  T* p = nullptr;
  const size_t n = std::max<size_t>(1, v.size());
  check(cudaMalloc((void**)&p, n * sizeof(T)), what);
  if (!v.empty()) check(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
  return p;
}

}  // namespace

void Likelihood::upload() {
  cuda_dev_ = eng_.devs.at(dev_).dev;
  check(cudaSetDevice(cuda_dev_), "cudaSetDevice");
  d_.reset(new LlhDevice);
  LlhDevice& D = *d_;
  std::vector<double> dat(blocks.size());
  for (size_t k = 0; k < blocks.size(); k++) dat[k] = blocks[k].dat;
  D.dom_slot = upload_vec(dom_slot, "likelihood tables");
  D.doms = upload_vec(doms, "likelihood tables");
  D.bin_block = upload_vec(bin_block, "likelihood tables");
  D.block_dat = upload_vec(dat, "likelihood tables");
  D.block_dom = upload_vec(block_dom, "likelihood tables");
  std::vector<double2> w(win.size() / 2);
  for (size_t k = 0; k < w.size(); k++) w[k] = make_double2(win[2 * k], win[2 * k + 1]);
  D.win = upload_vec(w, "likelihood tables");
  check(cudaMalloc((void**)&D.nohit, sizeof(unsigned long long)), "likelihood scratch");
  check(cudaMalloc((void**)&D.errors, sizeof(int)), "likelihood scratch");
  check(cudaMemset(D.errors, 0, sizeof(int)), "likelihood scratch");
}

Likelihood::~Likelihood() {
  if (d_) {
    cudaSetDevice(cuda_dev_);
    d_.reset();
  }
}

void Likelihood::eval_device(const ppcb_hit* dhits, uint64_t n, uint32_t seed, const double* dts, int ndt,
                             double nsim, double* dout, cudaStream_t st) {
  if (ndt < 1 || ndt > PPCB_LLH_MAX_SHIFTS) throw Error("likelihood: 1 to 64 time shifts per evaluation", 7);
  if (n > 0 && !dhits) throw Error("likelihood: null hits", 7);
  if (!(nsim > 0)) throw Error("likelihood: nsim must be positive", 7);
  require_device();
  check(cudaSetDevice(eng_.devs.at(dev_).dev), "cudaSetDevice");
  LlhDevice& D = *d_;
  const int nblocks = (int)blocks.size(), ndom = (int)doms.size();
  const int parts = std::max(1, (nblocks + kThreads - 1) / kThreads);
  if (ndt > D.ndt_cap) {
    for (void** p : {(void**)&D.simc, (void**)&D.stot, (void**)&D.partial})
      if (*p) {
        cudaFree(*p);
        *p = nullptr;
      }
    D.ndt_cap = 0;
    check(cudaMalloc((void**)&D.simc, (size_t)ndt * std::max(1, nblocks) * sizeof(unsigned int)), "likelihood scratch");
    check(cudaMalloc((void**)&D.stot, (size_t)ndt * std::max(1, ndom) * sizeof(unsigned int)), "likelihood scratch");
    check(cudaMalloc((void**)&D.partial, (size_t)ndt * parts * sizeof(double)), "likelihood scratch");
    D.ndt_cap = ndt;
  }
  check(cudaMemsetAsync(D.simc, 0, (size_t)ndt * std::max(1, nblocks) * sizeof(unsigned int), st), "memset");
  check(cudaMemsetAsync(D.stot, 0, (size_t)ndt * std::max(1, ndom) * sizeof(unsigned int), st), "memset");
  check(cudaMemsetAsync(D.nohit, 0, sizeof(unsigned long long), st), "memset");
  if (n > 0) {
    const uint64_t grid = (n + kThreads - 1) / kThreads;
    if (grid > 0x7fffffffull) throw Error("likelihood: too many hits in one call", 7);
    FillArgs F;
    F.A = back_args(eng_, dev_, dhits, n, seed);
    F.dom_slot = D.dom_slot;
    F.doms = D.doms;
    F.bin_block = D.bin_block;
    F.win = D.win;
    F.simc = D.simc;
    F.stot = D.stot;
    F.nohit = D.nohit;
    F.t0 = t0;
    F.lbin = lbin;
    F.nblocks = nblocks;
    F.ndom = ndom;
    F.ndt = ndt;
    F.unh = opts.unh;
    F.norm = opts.norm;
    for (int j = 0; j < PPCB_LLH_MAX_SHIFTS; j++) F.dt[j] = j < ndt ? dts[j] : 0.0;
    k_llh_fill<<<(unsigned int)grid, kThreads, 0, st>>>(F);
    check(cudaGetLastError(), "likelihood fill");
  }
  TermArgs T;
  T.simc = D.simc;
  T.stot = D.stot;
  T.block_dat = D.block_dat;
  T.block_dom = D.block_dom;
  T.doms = D.doms;
  T.partial = D.partial;
  T.errors = D.errors;
  T.nsim = nsim;
  T.ndat = opts.drep;
  T.sig = opts.sig;
  T.nblocks = nblocks;
  T.ndom = ndom;
  T.norm = opts.norm;
  k_llh_terms<<<dim3(parts, ndt), kThreads, 0, st>>>(T);
  check(cudaGetLastError(), "likelihood terms");
  k_llh_final<<<ndt, kThreads, 0, st>>>(D.partial, parts, D.nohit, opts.norm, nsim, opts.drep, opts.sig, ndof,
                                        D.errors, dout);
  check(cudaGetLastError(), "likelihood sum");
}

void Likelihood::require_device() {
  if (d_) return;
  if (!eng_.ready()) throw Error("ppcb_ini() must come before a likelihood evaluation", 6);
  if (dev_ >= (int)eng_.devs.size()) throw Error("bad device index", 7);
  upload();
}

int Likelihood::errors() {
  if (!d_) return 0;
  check(cudaSetDevice(eng_.devs.at(dev_).dev), "cudaSetDevice");
  int e = 0;
  check(cudaMemcpy(&e, d_->errors, sizeof(int), cudaMemcpyDeviceToHost), "likelihood errors");
  return e;
}

}  // namespace ppcb
