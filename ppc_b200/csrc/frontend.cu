// Source front end on the device (Engine::sources): the library's sources become photon
// bunches on the GPU, as the host front end makes them:
//   light yield per particle type       gpu/f2k.cxx:17-167 (muon segments, EM and hadronic
//                                        cascades with the hadronic light fluctuation)
//   Poisson photon count                gpu/f2k.cxx:387-433 (poidev)
//   addp / addp_clst / addp_mopo / ph   gpu/f2k.cxx:478-528
//   bunching                            gpu/f2k.cxx:377-385 (addh)
// Three kernels: k_src_count (one thread per source: its bunch template, the light
// fluctuation and the Poisson count, from the source's own random stream; bunch and photon
// totals per block of 256 sources), k_src_scan (offsets of the blocks), k_src_write (offsets
// within the block by a CTA scan; the bunches and their first-photon indices).  A source
// makes ceil(count / 2^31) bunches.  This file is compiled without fast-math and without
// contraction, so the bunch templates follow the host front end's float arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "backend.cuh"
#include "engine.h"

namespace ppcb {

struct FrontScratch {
  unsigned long long* num = nullptr;      // photons per source
  unsigned long long* blk_rec = nullptr;  // bunches per block of kThreads sources
  unsigned long long* blk_ph = nullptr;   // photons per block
  unsigned long long* rec_off = nullptr;  // [blocks + 1] first bunch of each block
  unsigned long long* ph_off = nullptr;   // [blocks + 1] first photon of each block
  int* errors = nullptr;
  uint64_t cap = 0;
  ~FrontScratch() {
    for (void* p : {(void*)num, (void*)blk_rec, (void*)blk_ph, (void*)rec_off, (void*)ph_off, (void*)errors})
      if (p) cudaFree(p);
  }
};

namespace {

constexpr int kThreads = 256;
constexpr unsigned long long kMaxBunch = 1ull << 31;  // photons per bunch record
constexpr int kMaxTries = 100000;                     // bound on every rejection loop
constexpr float kRho = 0.9216f;                       // density of ice [mwe]
constexpr float kM0 = 0.105658389f;                   // muon rest mass [GeV]

struct SrcRng {
  uint32_t x, y, a;
  __device__ float u() { return bxrnd(x, y, a); }  // (0, 1]
};

// the source's stream: a SplitMix64 hash (Steele, Lea, Flood 2014) of (seed, k) seeds an
// MWC generator with one of the configuration's multipliers
__device__ SrcRng src_stream(uint32_t seed, uint64_t k, const uint32_t* rm, uint32_t nmul) {
  uint64_t z = ((uint64_t)seed << 32 | 0x3c6ef372u) + (k + 1) * 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  SrcRng r;
  r.a = rm[k % nmul];
  r.x = (uint32_t)z;
  r.y = __umulhi((uint32_t)(z >> 32), r.a);
  return r;
}

__device__ float src_grnd(SrcRng& r) {  // gpu/f2k.cxx:8-10
  const float a = sqrtf(-2 * logf(r.u()));
  return a * sinf(2 * PPCB_FPI * r.u());
}

// log Gamma(xx) by the Lanczos series the reference uses (gpu/f2k.cxx:387-400)
__device__ double src_gammln(double xx) {
  const double stp = 2.5066282746310005;
  const double cof[6] = {76.18009172947146, -86.50532032941677, 24.01409824083091,
                         -1.231739572450155, 0.1208650973866179e-2, -0.5395239384953e-5};
  double ser = 1, x = xx - 1;
  double tmp = x + 5.5;
  tmp -= (x + 0.5) * log(tmp);
  for (int j = 0; j <= 5; j++) {
    x++;
    ser += cof[j] / x;
  }
  return -tmp + log(stp * ser);
}

// Poisson sample of mean xm (gpu/f2k.cxx:402-433): multiplication of uniforms below 12,
// rejection from a Lorentzian above
__device__ unsigned long long src_poisson(double xm, SrcRng& r, bool& err) {
  if (isnan(xm)) {
    err = true;
    return 0;
  }
  if (xm < 12) {
    const double g = exp(-xm);
    unsigned long long um = 0;
    double t = r.u();
    for (int it = 0; t > g; it++) {
      if (it >= kMaxTries) {
        err = true;
        break;
      }
      um++;
      t *= r.u();
    }
    return um;
  }
  const double sq = sqrt(2 * xm), alxm = log(xm), g = xm * alxm - src_gammln(xm + 1);
  for (int it = 0; it < kMaxTries; it++) {
    double y, em;
    int k = 0;
    do {
      y = tan((double)(PPCB_FPI * r.u()));
      em = sq * y + xm;
    } while (em < 0 && ++k < kMaxTries);
    if (em < 0) break;
    const double um = floor(em);
    const double t = 0.9 * (1 + y * y) * exp(um * alxm - src_gammln(um + 1) - g);
    if (!(r.u() > t)) return (unsigned long long)um;
  }
  err = true;
  return (unsigned long long)floor(xm + 0.5);
}

// The bunch template of a source (everything but its count).  Returns the mean photon
// count, or -1 for an exact count (`amount`).  `r` (null: template only) draws the
// hadronic light fluctuation.
__device__ double src_bunch(const ppcb_source& s, float eff, float ovr, ppcb_bunch& p, SrcRng* r, bool& err) {
  for (int i = 0; i < 4; i++) p.u.c[i] = 0;
  p.r[0] = s.r[0];
  p.r[1] = s.r[1];
  p.r[2] = s.r[2];
  p.r[3] = s.r[3];
  p.n[0] = s.n[0];
  p.n[1] = s.n[1];
  p.n[2] = s.n[2];
  p.n[3] = 0;
  p.q = s.q;
  p.num = 0;
  p.f = 0;
  switch (s.kind) {
    case PPCB_SRC_PARTICLE: {
      const int type = s.type;
      const float E = (float)s.amount, dr = s.dr;
      p.type = -type;
      p.u.p.beta = 1;
      p.u.p.tau = 0;
      p.n[3] = dr;
      if (type < 0) {
        err = true;
        return 0;
      }
      float nph;
      const float logE = logf(fmaxf(kM0, E));
      if (type < 10) {  // bare muon (0) or its end point (1)
        const float extr = 1 + fmaxf(0.0f, 0.1880f + 0.0206f * (logE - type)) * 0.910f / kRho;
        nph = dr > 0 ? dr * extr : 0;
        p.f = 1 / extr;
        p.u.p.a = 0;
        p.u.p.b = 0;
      } else {  // cascades
        const float Lrad = 0.39652 * 0.910f / kRho;
        const float em = 5.321 * 0.910f / kRho;
        nph = em * E;
        if (type < 100) {
          switch (type) {
            default:
            case 10: case 11: case 12:
              p.u.p.a = 2.01849f + 0.63176f * logE; p.u.p.b = Lrad / 0.63207f; break;
            case 13:
              p.u.p.a = 2.00035f + 0.63190f * logE; p.u.p.b = Lrad / 0.63008f; break;
            case 14:
              p.u.p.a = 2.83923f + 0.58209f * logE; p.u.p.b = Lrad / 0.64526f; break;
          }
        } else {
          float E0, m, f0, rms0, gamma;
          switch (type) {
            default:
            case 101: case 102:
              p.u.p.a = 1.58357292f + 0.41886807f * logE; p.u.p.b = Lrad / 0.33833116f;
              E0 = 0.18791678f; m = 0.16267529f; f0 = 0.30974123f; rms0 = 0.95899551f; gamma = 1.35589541f; break;
            case 103:
              p.u.p.a = 1.69176636f + 0.40803489f * logE; p.u.p.b = Lrad / 0.34108075f;
              E0 = 0.19826506f; m = 0.16218006f; f0 = 0.31859323f; rms0 = 0.94033488f; gamma = 1.35070162f; break;
            case 104:
              p.u.p.a = 1.95948974f + 0.34934666f * logE; p.u.p.b = Lrad / 0.34535151f;
              E0 = 0.21687243f; m = 0.16861530f; f0 = 0.27724987f; rms0 = 1.00318874f; gamma = 1.37528605f; break;
            case 105:
              p.u.p.a = 1.47495778f + 0.40450398f * logE; p.u.p.b = Lrad / 0.35226706f;
              E0 = 0.29579368f; m = 0.19373018f; f0 = 0.02455403f; rms0 = 1.01619344f; gamma = 1.45477346f; break;
            case 106:
              p.u.p.a = 1.57739060f + 0.40631102f * logE; p.u.p.b = Lrad / 0.35269455f;
              E0 = 0.66725124f; m = 0.19263595f; f0 = 0.17559033f; rms0 = 1.01414337f; gamma = 1.45086895f; break;
            case 107:
              p.u.p.a = 1.92249171f + 0.33701751f * logE; p.u.p.b = Lrad / 0.34969748f;
              E0 = 0.29579368f; m = 0.19373018f; f0 = 0.02455403f; rms0 = 1.01094637f; gamma = 1.50438415f; break;
          }
          if (r) {  // hadronic light-yield fluctuation, truncated to [0, 1.1]
            const float e = fmaxf(2.71828183f, E);
            const float F = 1 - powf(e / E0, -m) * (1 - f0);
            const float dF = F * rms0 * powf(logf(e), -gamma);
            float f;
            int it = 0;
            do f = F + dF * src_grnd(*r);
            while ((f < 0 || 1.1 < f) && ++it < kMaxTries);
            if (f < 0 || 1.1 < f) err = true;
            nph *= f;
          }
        }
        p.f = 0;
        if (dr > 0) {
          p.u.p.a = 0;
          p.u.p.b = 0;
        }
      }
      const float y = eff * nph;
      return (double)(s.scale * y / ovr);
    }
    case PPCB_SRC_CLST:
      p.type = 0;
      p.n[3] = s.dr;
      p.f = 1.f;
      p.u.p.beta = s.beta;
      return -1;
    case PPCB_SRC_MOPO:
      p.type = 0;
      p.n[3] = s.dr;
      p.f = s.fr;
      p.u.p.beta = s.beta;
      p.u.p.tau = s.tau;
      return (double)((float)s.amount * eff / ovr);
    case PPCB_SRC_POINT:
      p.type = 1;
      p.u.l.ka = 0;
      p.u.l.up = 0;
      p.u.l.fldr = -1;
      p.u.l.fla = -1;
      p.u.l.ofla = -1;
      p.n[3] = 1;
      return -1;
    default:
      err = true;
      return 0;
  }
}

struct SrcArgs {
  const ppcb_source* src;
  uint64_t n;
  const uint32_t* rm;
  uint32_t nmul, seed;
  float eff, ovr;
  unsigned long long* num;
  unsigned long long* blk_rec;
  unsigned long long* blk_ph;
  int* errors;
};

// Exclusive prefix sums over the CTA of two per-thread values (warp shuffles, then the warp
// totals); returns the CTA totals in *ta, *tb.
__device__ void cta_scan2(unsigned long long& a, unsigned long long& b, unsigned long long* ta,
                          unsigned long long* tb) {
  __shared__ unsigned long long wa[kThreads / 32], wb[kThreads / 32];
  const unsigned int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long ia = a, ib = b;
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long xa = __shfl_up_sync(0xffffffffu, ia, d), xb = __shfl_up_sync(0xffffffffu, ib, d);
    if ((int)lane >= d) {
      ia += xa;
      ib += xb;
    }
  }
  if (lane == 31) {
    wa[w] = ia;
    wb[w] = ib;
  }
  __syncthreads();
  unsigned long long oa = 0, ob = 0, sa = 0, sb = 0;
  for (int j = 0; j < kThreads / 32; j++) {
    if (j < (int)w) {
      oa += wa[j];
      ob += wb[j];
    }
    sa += wa[j];
    sb += wb[j];
  }
  a = oa + ia - a;
  b = ob + ib - b;
  *ta = sa;
  *tb = sb;
}

__device__ __forceinline__ unsigned long long src_bunches(unsigned long long num) {
  return (num + kMaxBunch - 1) / kMaxBunch;
}

__global__ void __launch_bounds__(kThreads) k_src_count(SrcArgs A) {
  const uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  unsigned long long num = 0;
  if (k < A.n) {
    const ppcb_source s = A.src[k];
    SrcRng r = src_stream(A.seed, k, A.rm, A.nmul);
    ppcb_bunch p;
    bool err = false;
    const double mean = src_bunch(s, A.eff, A.ovr, p, &r, err);
    if (mean < 0) {  // exact count
      if (!(s.amount >= 0) || s.amount >= 1.8e19) err = true;
      else num = (unsigned long long)s.amount;
    } else {
      num = src_poisson(mean, r, err);
    }
    A.num[k] = num;
    if (err) atomicAdd(A.errors, 1);
  }
  unsigned long long nr = src_bunches(num), np = num, tr, tp;
  cta_scan2(nr, np, &tr, &tp);
  if (threadIdx.x == 0) {
    A.blk_rec[blockIdx.x] = tr;
    A.blk_ph[blockIdx.x] = tp;
  }
}

// exclusive scans of the blocks' bunch and photon totals (one block, a contiguous chunk of
// blocks per thread)
__global__ void k_src_scan(const unsigned long long* nrec, const unsigned long long* num, uint64_t n,
                           unsigned long long* rec_off, unsigned long long* ph_off, uint64_t* counts) {
  __shared__ unsigned long long pr[1024], pp[1024];
  const uint64_t t = threadIdx.x, nt = blockDim.x;
  const uint64_t per = (n + nt - 1) / nt;
  const uint64_t lo = min(n, t * per), hi = min(n, lo + per);
  unsigned long long sr = 0, sp = 0;
  for (uint64_t k = lo; k < hi; k++) {
    sr += nrec[k];
    sp += num[k];
  }
  pr[t] = sr;
  pp[t] = sp;
  __syncthreads();
  for (unsigned int d = 1; d < nt; d <<= 1) {
    const unsigned long long vr = t >= d ? pr[t - d] : 0, vp = t >= d ? pp[t - d] : 0;
    __syncthreads();
    pr[t] += vr;
    pp[t] += vp;
    __syncthreads();
  }
  unsigned long long ar = pr[t] - sr, ap = pp[t] - sp;
  for (uint64_t k = lo; k < hi; k++) {
    rec_off[k] = ar;
    ph_off[k] = ap;
    ar += nrec[k];
    ap += num[k];
  }
  if (t == nt - 1) {
    rec_off[n] = pr[t];
    ph_off[n] = pp[t];
    counts[0] = pr[t];
    counts[1] = pp[t];
  }
}

__global__ void __launch_bounds__(kThreads) k_src_write(SrcArgs A, const unsigned long long* rec_off,
                                                        const unsigned long long* ph_off, uint64_t nblk,
                                                        ppcb_bunch* out, uint64_t* bstart, uint64_t cap) {
  const uint64_t k = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
  const unsigned long long num = k < A.n ? A.num[k] : 0, nrec = src_bunches(num);
  unsigned long long b0 = nrec, ph0 = num, tr, tp;
  cta_scan2(b0, ph0, &tr, &tp);
  if (k >= A.n) return;
  b0 += rec_off[blockIdx.x];
  ph0 += ph_off[blockIdx.x];
  if (nrec > 0) {
    const ppcb_source s = A.src[k];
    ppcb_bunch p;
    bool err = false;
    src_bunch(s, A.eff, A.ovr, p, nullptr, err);
    for (unsigned long long j = 0; j < nrec; j++) {
      const unsigned long long b = b0 + j;
      if (b >= cap) break;
      const unsigned long long left = num - j * kMaxBunch;
      p.num = (uint32_t)(left < kMaxBunch ? left : kMaxBunch);
      out[b] = p;
      bstart[b] = ph0 + j * kMaxBunch;
    }
  }
  if (k == A.n - 1 && rec_off[nblk] <= cap) bstart[rec_off[nblk]] = ph_off[nblk];
}

}  // namespace

void Engine::sources(int d, const ppcb_source* dsrc, uint64_t ns, uint32_t seed, ppcb_bunch* dout, uint64_t* dbstart,
                     uint64_t cap, uint64_t* dcounts, cudaStream_t st) {
  if (!inited_) throw Error("ini() must come before the front end", 6);
  DeviceCtx& g = devs.at(d);
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  if (ns == 0) {
    check(cudaMemsetAsync(dcounts, 0, 2 * sizeof(uint64_t), st), "memset");
    check(cudaMemsetAsync(dbstart, 0, sizeof(uint64_t), st), "memset");
    return;
  }
  const uint64_t grid = (ns + kThreads - 1) / kThreads;
  if (grid > 0x7fffffffull) throw Error("front end: too many sources in one call", 7);
  if (!g.front) {
    g.front = std::make_shared<FrontScratch>();
    check(cudaMalloc((void**)&g.front->errors, sizeof(int)), "front end scratch");
    check(cudaMemset(g.front->errors, 0, sizeof(int)), "front end scratch");
  }
  FrontScratch& F = *g.front;
  if (ns > F.cap) {
    for (void** p : {(void**)&F.num, (void**)&F.blk_rec, (void**)&F.blk_ph, (void**)&F.rec_off, (void**)&F.ph_off})
      if (*p) {
        cudaFree(*p);
        *p = nullptr;
      }
    F.cap = 0;
    check(cudaMalloc((void**)&F.num, ns * sizeof(unsigned long long)), "front end scratch");
    check(cudaMalloc((void**)&F.blk_rec, grid * sizeof(unsigned long long)), "front end scratch");
    check(cudaMalloc((void**)&F.blk_ph, grid * sizeof(unsigned long long)), "front end scratch");
    check(cudaMalloc((void**)&F.rec_off, (grid + 1) * sizeof(unsigned long long)), "front end scratch");
    check(cudaMalloc((void**)&F.ph_off, (grid + 1) * sizeof(unsigned long long)), "front end scratch");
    F.cap = ns;
  }
  SrcArgs A;
  A.src = dsrc;
  A.n = ns;
  A.rm = g.rm;
  A.nmul = (uint32_t)std::max(1, std::min(g.T, 1024));
  A.seed = seed;
  A.eff = cfg.eff;
  A.ovr = cfg.ovr;
  A.num = F.num;
  A.blk_rec = F.blk_rec;
  A.blk_ph = F.blk_ph;
  A.errors = F.errors;
  k_src_count<<<(unsigned int)grid, kThreads, 0, st>>>(A);
  check(cudaGetLastError(), "front end count");
  k_src_scan<<<1, 1024, 0, st>>>(F.blk_rec, F.blk_ph, grid, F.rec_off, F.ph_off, dcounts);
  check(cudaGetLastError(), "front end scan");
  k_src_write<<<(unsigned int)grid, kThreads, 0, st>>>(A, F.rec_off, F.ph_off, grid, dout, dbstart, cap);
  check(cudaGetLastError(), "front end write");
}

int Engine::front_errors(int d) {
  DeviceCtx& g = devs.at(d);
  if (!g.front) return 0;
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  int e = 0;
  check(cudaMemcpy(&e, g.front->errors, sizeof(int), cudaMemcpyDeviceToHost), "front end errors");
  return e;
}

}  // namespace ppcb
