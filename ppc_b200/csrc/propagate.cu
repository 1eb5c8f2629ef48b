// Photon propagation kernels for sm_100a.
//
// Physics restated from the reference kernel gpu/pro.cu:287-904 (phase 1: source
// sampling :334-477, phase 2: stepping :486-889); the helpers cite their lines below.
// B200-specific structure (not in the reference):
//   * one persistent launch; phase 1 is fused into phase 2 -- a thread samples a new
//     photon only when its previous one is absorbed, so the 48-byte per-photon phase-1
//     record never round-trips through HBM;
//   * photon indices are handed out by one warp-aggregated atomic per refill (one
//     global counter, 64-bit, so a launch may cover more than 2^32 photons), or
//     statically (photon i on thread i mod T) in deterministic mode;
//   * the photon -> bunch map is a binary search over an exclusive prefix sum, so a
//     launch may hold thousands of bunches/events;
//   * the small tables (per-layer anisotropy/BFR, strings, cell index, tilt radii) sit
//     in shared memory; the per-wavelength ice table, tilt maps and DOMs are read
//     through the read-only cache from HBM (they are L2-resident: < 1 MB);
//   * hits are appended with one atomic per coalesced group of hitting lanes;
//   * paired components ((x, y) of a direction, (absorption, scattering) of a layer) go
//     through sm_100's two-lane FP32 instructions (__ffma2_rn and the like), one issue slot
//     for two operations in a kernel whose limit is instruction issue;
//   * the index helpers (tilt shift, layer, cell range, DOM window) use explicit
//     round-to-nearest operations without contraction, so for identical positions they
//     are bit-identical to the IEEE CPU restatement; the rest of the physics uses the
//     same fast-math intrinsics as the reference's GPU build (--use_fast_math).
#include <cooperative_groups.h>

#include <atomic>
#include <type_traits>

#include "propagate.cuh"
#include "tilt.h"

namespace cg = cooperative_groups;

namespace ppcb {

#define XXX PPCB_XXX
#define FPI PPCB_FPI
#define OMR PPCB_OMR
#define WNUM PPCB_WNUM

__device__ __constant__ float kFcv = PPCB_FPI / 180.f;

struct SmemTables {
  ppcb_aniz az[PPCB_MAXLYS];
  ppcb_line sc[PPCB_NSTR];
  float lr[PPCB_LMAX];
  uint16_t ls[PPCB_NSTR];
  uint16_t is[PPCB_CX * PPCB_CY];
  int8_t mcol[PPCB_CTX * PPCB_CTY];
  StrGroup sgg[PPCB_NSTR + 1];    // string-proximity table: string axes and the sentinel (strgrid.h)
  float4 azr[PPCB_MAXLYS];        // per layer 1/k1, 1/k2, 1/(k1 k2): the scattering's frame divisions
  float4 scat[2][2];              // bulk [0] / hole ice [1]: (sf, g, gr, 1/(1-sf)), (1-g^2, (1-g)^2, 1/(2g), 1/sf)
};

// ---------------------------------------------------------------- IEEE helpers
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ int imin(int a, int b) { return b < a ? b : a; }
__device__ __forceinline__ int imax(int a, int b) { return a < b ? b : a; }

struct Rng {
  uint32_t x, y, a;
};

// gpu/pro.cu:47-57: 64-bit multiply-with-carry, (0,1]
__device__ __forceinline__ float xrnd(Rng& s) {
  unsigned long long sda = (unsigned long long)s.a * s.x + s.y;
  s.x = (uint32_t)sda;
  s.y = (uint32_t)(sda >> 32);
  return 2.f - __uint_as_float((s.x >> 9) | 0x3f800000u);
}

// Per-photon stream (no counterpart in the reference): the MWC state of photon i is a
// SplitMix64 hash (Steele, Lea, Flood, OOPSLA 2014) of (seed, i), the carry mapped into
// [0, a) of the thread's multiplier; the photon's random numbers then depend only on
// (seed, i, thread multiplier) and not on what the thread simulated before.
__device__ __forceinline__ void photon_stream(Rng& s, uint64_t i, uint32_t seed) {
  uint64_t z = ((uint64_t)seed << 32 | 0x2545f491u) + (i + 1) * 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  s.x = (uint32_t)z;
  s.y = __umulhi((uint32_t)(z >> 32), s.a);
}

// gpu/pro.cu:59-85
__device__ float mrnd(float k, Rng& s) {
  float x;
  if (k < 1) {
    float c = 1 / k;
    float d = (1 - k) * powf(k, 1 / (c - 1));
    float z, e;
    int guard = 0;  // bounded rejection loop (only degenerate shape parameters reach the bound)
    do {
      z = -logf(xrnd(s));
      e = -logf(xrnd(s));
      x = powf(z, c);
    } while (z + e < d + x && ++guard < 100000);
  } else {
    float b = k - logf(4.0f);
    float l = sqrtf(2 * k - 1);
    float c = 1 + logf(4.5f);
    float u, v, y, z, r;
    int guard = 0;
    do {
      u = xrnd(s);
      v = xrnd(s);
      y = -logf(1 / v - 1) / l;
      x = k * expf(y);
      z = u * v * v;
      r = b + (k + l) * y - x;
    } while (r < 4.5f * z - c && r < logf(z) && ++guard < 100000);
  }
  return x;
}

// 2 pi xrnd(s) as one FMA on the generator's [1, 2) float f: xrnd = 2 - f exactly (Sterbenz),
// and 4 pi, 2 pi differ by a power of two, so the product 2 pi (2 - f) rounds the same way.
__device__ __forceinline__ float xrnd_angle(Rng& s) {
  unsigned long long sda = (unsigned long long)s.a * s.x + s.y;
  s.x = (uint32_t)sda;
  s.y = (uint32_t)(sda >> 32);
  const float f = __uint_as_float((s.x >> 9) | 0x3f800000u);
  return fmaf(-2 * FPI, f, 4 * FPI);
}

// gpu/pro.cu:87-95
__device__ __forceinline__ float grnd(Rng& s) {
  float a = sqrtf(-2 * logf(xrnd(s)));
  return a * sinf(xrnd_angle(s));
}

__device__ __forceinline__ float2 grnd2(Rng& s) {
  float r = sqrtf(-2 * logf(xrnd(s)));
  float2 p;
  sincosf(xrnd_angle(s), &p.y, &p.x);
  return __fmul2_rn(p, make_float2(r, r));
}

__device__ __forceinline__ void swp(float& a, float& b) { float t = a; a = b; b = t; }

// gpu/pro.cu:111-153: rotate n by polar angle (cs = 1-cos, si = sin), uniform azimuth
__device__ __forceinline__ void rotate(float cs, float si, float4& n, Rng& s) {
  float3 p1, p2;
  int i = 0;
  {
    float3 r;
    r.x = n.x * n.x; r.y = n.y * n.y; r.z = n.z * n.z;
    if (r.y > r.z) {
      if (r.y > r.x) { swp(n.x, n.y); swp(r.x, r.y); i = 1; }
    } else {
      if (r.z > r.x) { swp(n.x, n.z); swp(r.x, r.z); i = 2; }
    }
    r.y = rsqrtf(r.x + r.y); p1.x = -n.y * r.y; p1.y = n.x * r.y; p1.z = 0;
    r.z = rsqrtf(r.x + r.z); p2.x = -n.z * r.z; p2.y = 0; p2.z = n.x * r.z;
  }
  {
    float3 q1;
    q1.x = p1.x - p2.x; q1.y = p1.y - p2.y; q1.z = p1.z - p2.z;
    p2.x += p1.x; p2.y += p1.y; p2.z += p1.z;
    float w = rsqrtf(q1.x * q1.x + q1.y * q1.y + q1.z * q1.z);
    p1.x = q1.x * w; p1.y = q1.y * w; p1.z = q1.z * w;
    w = rsqrtf(p2.x * p2.x + p2.y * p2.y + p2.z * p2.z);
    p2.x *= w; p2.y *= w; p2.z *= w;
  }
  {
    float2 p;
    float xi = xrnd_angle(s);
    sincosf(xi, &p.y, &p.x);
    n.x -= cs * n.x - si * (p.x * p1.x + p.y * p2.x);
    n.y -= cs * n.y - si * (p.x * p1.y + p.y * p2.y);
    n.z -= cs * n.z - si * (p.x * p1.z + p.y * p2.z);
    float r = rsqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    n.x *= r; n.y *= r; n.z *= r;
    if (i == 1) swp(n.x, n.y);
    else if (i == 2) swp(n.x, n.z);
  }
}

__device__ __forceinline__ void normalize3(float4& n) {
  float r = rsqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
  n.x *= r; n.y *= r; n.z *= r;
}

// ---------------------------------------------------------------- index helpers
// tilt tables as seen by the kernel: radii and map columns in shared memory, the
// depth maps through the read-only cache
struct DevTilt {
  const SmemTables& S;
  const ppcb_params& d;
  const float2* __restrict__ lpg;
  __device__ __forceinline__ float lr(int i) const { return S.lr[i]; }
  __device__ __forceinline__ int mcol(int x, int y) const {
    return x >= 0 && x < d.mnum[0] && y >= 0 && y < d.mnum[1] ? S.mcol[x * PPCB_CTY + y] : -1;
  }
  __device__ __forceinline__ float2 lp(int i, int k) const { return __ldg(&lpg[i * PPCB_LYRS + k]); }
};

__device__ __forceinline__ float zshift(const ppcb_params& d, const SmemTables& S, const float2* __restrict__ lp,
                                        float rx, float ry, float rz, float& dz) {
  DevTilt t{S, d, lp};
  return zshift_t(d, t, rx, ry, rz, dz);
}

// gpu/pro.cu:507-515: tilt-corrected depth in layer units and the current layer.
__device__ __forceinline__ int layer_of(const ppcb_params& d, float rz, float zs, float& z) {
  z = fm(fs(fs(rz, zs), d.hmin), d.rdh);
  return imin(imax(__float2int_rn(z), 0), d.size - 1);
}

// gpu/pro.cu:580-594: range of search cells covered by a segment (plus margin rx).
__device__ __forceinline__ void cell_range(const ppcb_params& d, float rx0, float ry0, float rx1, float ry1,
                                           int& xlx, int& xhx, int& xly, int& xhy) {
  float pix = fa(fm(d.cb[0][0], rx0), fm(d.cb[1][0], ry0));
  float piy = fa(fm(d.cb[0][1], rx0), fm(d.cb[1][1], ry0));
  float pfx = fa(fm(d.cb[0][0], rx1), fm(d.cb[1][0], ry1));
  float pfy = fa(fm(d.cb[0][1], rx1), fm(d.cb[1][1], ry1));
  float lx = fs(fminf(pix, pfx), d.rx), hx = fa(fmaxf(pix, pfx), d.rx);
  float ly = fs(fminf(piy, pfy), d.rx), hy = fa(fmaxf(piy, pfy), d.rx);
  xlx = imin(imax(__float2int_rn(fm(fs(lx, d.cl[0]), d.crst[0])), 0), d.cn[0]);
  xhx = imax(imin(__float2int_rn(fm(fs(hx, d.cl[0]), d.crst[0])), d.cn[0] - 1), -1);
  xly = imin(imax(__float2int_rn(fm(fs(ly, d.cl[1]), d.crst[1])), 0), d.cn[1]);
  xhy = imax(imin(__float2int_rn(fm(fs(hy, d.cl[1]), d.crst[1])), d.cn[1] - 1), -1);
}

// gpu/pro.cu:623-626: DOMs of one string whose depth window overlaps [zl, zh].
__device__ __forceinline__ void dom_window(const ppcb_line& s, float zl, float zh, int& n1, int& n2) {
  const int omin = 0, omax = s.max;
  n1 = s.n - omin + imin(omax + 1, imax(omin, __float2int_ru(fs((float)omin, fm(fs(fs(zh, s.dl), s.h), s.d)))));
  n2 = s.n - omin + imax(omin - 1, imin(omax, __float2int_rd(fs((float)omin, fm(fs(fs(zl, s.dh), s.h), s.d)))));
}

// ---------------------------------------------------------------- photon state
struct Photon {
  float4 r, n;     // position/time, direction/(1/group velocity)
  float TOT, SCA;  // remaining absorption / scattering optical depths
  int wl;          // wavelength bin
  uint32_t niw;    // segment id
  int old;         // DOM excluded from the search (last hit / flasher)
  int ofla;        // DOM that absorbs without registering (flasher), or <-1 veto code
  int om0;         // flasher DOM on the first step, -1 afterwards
  uint32_t steps;
  int nhit;        // hits registered so far (ordinal of the next one)
};

__device__ __forceinline__ int find_bunch(const KArgs& a, int nb, uint64_t i, int hint) {
  // exclusive prefix sums: bunch k holds photons [bstart[k], bstart[k+1])
  if (hint >= 0 && hint < nb && __ldg(&a.bstart[hint]) <= i && i < __ldg(&a.bstart[hint + 1])) return hint;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(&a.bstart[mid]) <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// gpu/pro.cu:335-476: phase-1 source sampling of one photon of bunch p.
__device__ __forceinline__ void generate(const KArgs& a, const ppcb_bunch& p, Rng& s, Photon& ph) {
  const ppcb_params& e = a.p;
  float4 r, n;
  int j = imin(__float2int_rd(WNUM * xrnd(s)), WNUM - 1);
  const ppcb_wmeta w = a.wmeta[j];
  n.w = w.ocm;
  r = make_float4(p.r[0], p.r[1], p.r[2], p.r[3]);
  n.x = p.n[0]; n.y = p.n[1]; n.z = p.n[2];
  float l = p.n[3];
  int fla, ofla;
  if (p.type > 0) {
    const float ka = p.u.l.ka, up = p.u.l.up, fldr = p.u.l.fldr;
    fla = p.u.l.fla; ofla = p.u.l.ofla;
    if (l == 0) {  // N-fold / cylindrical LED pattern
      float xi = xrnd(s);
      if (fldr < 0) xi *= 2 * FPI;
      else {
        int rr = __float2int_rd(fldr / 360) + 1;
        int ss = __float2int_rd(xi * rr);
        xi = (fldr + ss * 360 / rr) * kFcv;
      }
      sincosf(xi, &r.y, &r.x);
      sincosf(up, &n.z, &xi);
      n.x = xi * r.x; n.y = xi * r.y;
    }
    if (ka != 0) {
      float xi;
      if (ka > 999.f) {  // lab-measured beam profile
        xi = xrnd(s);
        float s1 = 0.0191329f, s2 = 0.0686944f, C1 = 0.583583f, C2 = 0.967762f;
        switch (p.type) {
          case 1: s1 = 0.0196242f; s2 = 0.0750278f; C1 = 0.606833f; C2 = 0.960863f; break;
          case 2: s1 = 0.0185603f; s2 = 0.0624481f; C1 = 0.553192f; C2 = 0.974129f; break;
        }
        xi = xi < C1 ? s1 * fabsf(grnd(s)) : xi < C2 ? -s2 * logf(xrnd(s)) : 2.f;
        if (xi >= 2.f) xi = 2 * (1 - sqrtf(xrnd(s)));
      } else if (ka > 0) xi = fminf(-ka * logf(1 - (1 - xrnd(s)) * (1 - expf(-2 / ka))), 2.f);
      else if (ka == -1) xi = 2 * (1 - xrnd(s));
      else xi = 2 * (1 - sqrtf(xrnd(s)));
      rotate(xi, sqrtf(xi * (2 - xi)), n, s);
    }
    if (ka > 999.f) {  // start on the DOM surface; harness and cable vetoes
      const float FLZ = 0.07735f, FLR = 0.119f - 0.008f, FLB = 0.03396f;
      if (l == 0) { r.x *= FLR; r.y *= FLR; r.z = FLZ; r.w = 0; }
      float b = r.x * n.x + r.y * n.y + r.z * n.z;
      float c = FLZ * FLZ + FLR * FLR - OMR * OMR;
      float t = sqrtf(b * b - c) - b;
      r.x += t * n.x; r.y += t * n.y; r.z += t * n.z; r.w += t * e.ocv;
      if (fabsf(r.z) < FLB) ofla = -2;
      else if (l == 0 && r.z < 0 && xrnd(s) < 0.9f) ofla = -3;
      if (ka > 1050.f) {
        const float rc = 0.023f;
        const float dc = OMR + rc;
        float ph = (ka - 1080.f) * kFcv;
        float drx = r.x - dc * cosf(ph);
        float dry = r.y - dc * sinf(ph);
        float aa = n.x * n.x + n.y * n.y;
        if (aa > 0) {
          float bb = n.x * drx + n.y * dry;
          float cc = drx * drx + dry * dry - rc * rc;
          float D = bb * bb - aa * cc;
          if (D >= 0) {
            float h1 = (-bb + sqrtf(D)) / aa;
            if (h1 > 0) ofla = -4;
          }
        }
      }
      if (l == 0) { r.x += p.r[0]; r.y += p.r[1]; r.z += p.r[2]; r.w += p.r[3]; }
      else {
        const ppcb_dom dom = a.oms[(unsigned)fla < (unsigned)e.gsize ? fla : 0];  // invalid input: no out-of-bounds read
        r.x += dom.r[0]; r.y += dom.r[1]; r.z += dom.r[2]; r.w += p.r[3];
      }
    } else if (fla >= 0) {
      const float t = OMR;
      r.x = t * n.x; r.y = t * n.y; r.z = t * n.z; r.w = t * e.ocv;
      r.x += p.r[0]; r.y += p.r[1]; r.z += p.r[2]; r.w += p.r[3];
    } else {
      r = make_float4(p.r[0], p.r[1], p.r[2], p.r[3]);
    }
  } else {
    const float pa = p.u.p.a, pb = p.u.p.b, beta0 = p.u.p.beta, tau = p.u.p.tau;
    fla = -1; ofla = -1;
    if (l > 0) l *= xrnd(s);
    else l = pb * mrnd(pa, s);
    if (l > 0) {
      r.x += l * n.x; r.y += l * n.y; r.z += l * n.z;
      r.w += l * e.ocv / beta0;
    }
    if (tau > 0) {  // isotropic delayed emission
      r.w -= tau * logf(xrnd(s));
      float xi = 1 - xrnd(s);
      rotate(xi, sqrtf(xi * (2 - xi)), n, s);
    } else {
      float cs = w.coschr, si = w.sinchr;
      if (p.f < xrnd(s)) {  // cascade secondary directions
        const float aa = 0.39f, bb = 2.61f;
        const float I = 1 - expf(-bb * exp2f(aa));
        float xi = fminf(powf(-logf(1 - xrnd(s) * I) / bb, 1 / aa), 2.f);
        rotate(xi, sqrtf(xi * (2 - xi)), n, s);
      } else {
        float beta = beta0;
        if (p.type < 0) {  // muon slowing down near its end point
          const float ar = 0.26f * 0.9216f / 0.105658389f;
          float dx = ar * (p.n[3] - l);
          beta = sqrtf(dx * (2 + dx)) / (1 + dx);
          if (beta >= cs) r.w -= e.ocv * (sqrtf(dx * dx + 1) - asinhf(1 / dx) - dx) / ar;
        }
        if (beta < 1) {
          float xi = cs / beta;
          if (xi <= 1) {
            float sx = sqrtf(1 - xi * xi);
            if (p.type < 0 && sx < xrnd(s) * si) ofla = -3;
            cs = xi; si = sx;
          } else ofla = -2;
        }
      }
      rotate(1 - cs, si, n, s);  // Cherenkov cone
    }
  }
  ph.r = r; ph.n = n;
  ph.wl = j; ph.niw = p.q; ph.om0 = fla; ph.ofla = ofla;
}

// The two rare branches of the photon loop, sampling (once per photon) and the hit record
// (about once per 2e4 steps), are compiled out of line: inlined, their code (source
// types, Cherenkov cone, acos/atan2) would share the instruction cache with the step.
struct Sampled {
  Photon ph;
  uint32_t x, y;  // stream state after the draws
};

__device__ __noinline__ Sampled sample_photon(const KArgs& a, int bunch, uint32_t sx, uint32_t sy, uint32_t sa) {
  Rng s;
  s.x = sx; s.y = sy; s.a = sa;
  Sampled out;
  const ppcb_bunch p = a.bunches[bunch];
  generate(a, p, s, out.ph);
  out.x = s.x; out.y = s.y;
  return out;
}

// gpu/pro.cu:734-745: the hit record (photon and DOM-surface angles)
__device__ __noinline__ ppcb_hit hit_record(const KArgs& a, int om, float4 r, float4 n, float sqd, uint32_t niw,
                                           int wl) {
  const ppcb_params& e = a.p;
  ppcb_hit h;
  h.i = om; h.t = r.w; h.n = niw; h.z = a.wmeta[wl].wvl;
  h.pth = acosf(n.z); h.pph = atan2f(n.y, n.x);
  sqd *= e.xR - 1;
  const ppcb_dom dom = a.oms[om];
  float dx = dom.r[0] - r.x + sqd * n.x;
  float dy = dom.r[1] - r.y + sqd * n.y;
  float dz = dom.r[2] - r.z + sqd * n.z;
  h.dth = acosf(fminf(fmaxf(dz / (e.xR * dom.R * dom.F), -1.f), 1.f));
  h.dph = atan2f(dy, dx);
  return h;
}

__device__ __forceinline__ float2 ice(const float2* __restrict__ t, int J) { return __ldg(&t[J]); }

__device__ __forceinline__ unsigned long long emit_hit(const KArgs& a, const ppcb_hit& h) {
  if (a.ev_cnt) {  // batched launch: the event's own region, sized from an upper bound
    const unsigned int e = h.n;
    const unsigned int slot = atomicAdd(&a.ev_cnt[e], 1u);
    if (slot < __ldg(&a.ev_cap[e])) {
      uint4* dst = reinterpret_cast<uint4*>(&a.hits[__ldg(&a.ev_off[e]) + slot]);
      const uint4* src = reinterpret_cast<const uint4*>(&h);
      dst[0] = src[0];
      dst[1] = src[1];
    }
    return ~0ull;
  }
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(&a.ctrl->hidx, (unsigned long long)g.size());
  base = g.shfl(base, 0) + g.thread_rank();
  if (base < a.hcap) {
    uint4* dst = reinterpret_cast<uint4*>(&a.hits[base]);
    const uint4* src = reinterpret_cast<const uint4*>(&h);
    dst[0] = src[0];
    dst[1] = src[1];
  }
  return base;
}

// the plain kernel's hit append, out of line (about one step in 2e4 registers a hit)
__device__ __noinline__ void emit_hit_cold(const KArgs& a, ppcb_hit h) { emit_hit(a, h); }

// ---------------------------------------------------------------- step hooks
// The plain propagation: hits are appended, nothing else is observed.
struct NoHook {
  __device__ __forceinline__ bool active() const { return false; }
  __device__ __forceinline__ void segment(int, float, int, float, float, float, float, float, int) {}
  __device__ __forceinline__ void scatter(int, float) {}
  __device__ __forceinline__ void hit(const KArgs& a, const ppcb_hit& h, Photon&) { emit_hit_cold(a, h); }
};

// Provenance of a hit, enough to replay its photon: the sampled photon, the stream state
// of the propagating thread before its first draw, that thread, and the hit's ordinal
// among the photon's hits.  64 bytes, stored at the hit's slot.
struct Prov {
  float4 r, n;
  int4 m;    // wavelength bin, segment, flasher DOM, veto code
  uint4 s;   // stream x, stream y, thread, hit ordinal
};

// Gradient hook.  In the recording forward pass it writes each hit's provenance; in the
// replay it accumulates, for the photon's path up to the recorded hit, the derivatives of
// that hit's weight with respect to the per-layer scattering (be) and absorption (ba)
// coefficients of the ice model:
//   absorption (pathwise): d/dba_j = -D l_k(lambda) nr L_j      (survival exp(-sum abs nr L))
//   scattering (score):    d/dbe_j = l_a(lambda)/(1-g) (n_j/sca_j - L_j)
// with L_j the path length in layer j (split as the reference splits overburdens,
// gpu/pro.cu:678-696) and n_j the scatterings in layer j.  Sums go to FP64 shared memory.
struct AdjHook {
  bool replay;
  int target;          // replay: ordinal of the hit to stop at
  uint32_t target_i;   // replay: its DOM
  float target_t;      // replay: its time
  bool done, matched;
  float w_be, w_ba;    // hit weight x dsca/dbe, x dabs/dba (per wavelength)
  double* g_be;
  double* g_ba;
  Prov* prov_out;      // recording: provenance array, indexed like the hits
  Prov* start;         // recording: this thread's current photon (a shared-memory slot)
  __device__ __forceinline__ bool active() const { return replay && !done; }
  // path length `del` from layer coordinate z (layer I), direction sign/anz, layer step edh.
  // The hook's arithmetic is in explicitly rounded intrinsics, which the compiler neither
  // contracts nor shares with the step's own expressions: the step compiles to the same
  // floating-point operations whether the hook is live (replay) or not (recording).
  __device__ __forceinline__ void segment(int I, float z, int sign, float anz, float edh, float nr, float del,
                                          float nz, int size) {
    if (!active() || !(del > 0)) return;
    const float y = __fadd_rn(z, __fdiv_rn(__fmul_rn(nz, del), edh));
    const int J = min(max(__float2int_rn(y), 0), size - 1);
    if (I == J) { add(I, del, nr); return; }
    const float f = __fdiv_rn(edh, anz);
    const float s = (float)sign;
    add(I, __fmul_rn(__fsub_rn(0.5f, __fmul_rn(s, __fsub_rn(z, (float)I))), f), nr);
    add(J, __fmul_rn(__fadd_rn(0.5f, __fmul_rn(s, __fsub_rn(y, (float)J))), f), nr);
    for (int i = I + sign; i != J && (unsigned)i < (unsigned)size; i += sign) add(i, f, nr);
  }
  __device__ __forceinline__ void add(int j, float len, float nr) {
    if (!(len > 0)) return;
    atomicAdd(&g_be[j], -(double)w_be * len);
    atomicAdd(&g_ba[j], -(double)w_ba * nr * len);
  }
  __device__ __forceinline__ void scatter(int J, float scaJ) {
    if (active()) atomicAdd(&g_be[J], (double)w_be / scaJ);
  }
  __device__ __forceinline__ void hit(const KArgs& a, const ppcb_hit& h, Photon& ph) {
    if (replay) {
      if (!done && ph.nhit == target) {
        done = true;
        matched = h.i == target_i && __float_as_uint(h.t) == __float_as_uint(target_t);
      }
      ph.nhit++;
      return;
    }
    const unsigned long long slot = emit_hit(a, h);
    if (prov_out && slot < a.hcap) {
      Prov p = *start;
      p.s.w = (unsigned)ph.nhit;
      prov_out[slot] = p;
    }
    ph.nhit++;
  }
};

// Rare parts of the step, compiled out of line so that the step loop stays small in the
// instruction cache.

// gpu/pro.cu:655-669: entry and exit of the segment in the hole-ice column of a string
// (radius hr), given the string's closest-approach terms b, c and np = 1 - nz^2; returns
// the updated (hi, hf).
__device__ __noinline__ float2 hole_column(const ppcb_params& e, float b, float c, float np, float sca, float hi,
                                           float hf) {
  float DH = b * b - (c - e.hr2) * np;
  if (DH > 0) {
    DH = sqrtf(DH);
    float h1 = b - DH, h2 = b + DH;
    if (h2 >= 0 && h1 <= sca * np) {
      if (np > XXX) {
        h1 /= np; h2 /= np;
        if (h1 < 0) h1 = 0;
        if (h2 > sca) h2 = sca;
      } else { h1 = 0; h2 = sca; }
      if (h1 < hi && h2 > sqrtf(XXX) * e.hr) { hi = h1; hf = h2; }
    }
  }
  return make_float2(hi, hf);
}

struct Truncated {
  float SCA, TOT, del;
  int om, J;
};

// gpu/pro.cu:677-717: a step cut short at fin (DOM hit or hole-ice entry): the optical
// depths used over the bulk-ice part by layers, then the hole-ice part.
__device__ __noinline__ Truncated truncated_step(const ppcb_params& e, const float2* __restrict__ wz, float z, float nz,
                                                 float fin, float edh, int I, int sign, float anz, float SCA,
                                                 float TOT, float nr, float hi, float hf, float del, float sca,
                                                 int om) {
  Truncated t;
  {
    float xs = 0, xa = 0;
    float y = z + nz * fin / edh;
    const int J = imin(imax(__float2int_rn(y), 0), e.size - 1);
    t.J = J;
    if (I == J) { float2 c = ice(wz, I); xs = fin * c.y; xa = fin * c.x; }
    else {
      float h = 0.5f - sign * (z - I);
      float g = 0.5f + sign * (y - J);
      float2 ci = ice(wz, I), cj = ice(wz, J);
      xs = h * ci.y + g * cj.y;
      xa = h * ci.x + g * cj.x;
      for (int i = I + sign; i != J && (unsigned)i < (unsigned)e.size; i += sign) { float2 c = ice(wz, i); xs += c.y; xa += c.x; }
      float f = edh / anz;
      xs *= f; xa *= f;
    }
    if (xs < 0) xs = 0;
    if (xa < 0) xa = 0;
    SCA -= xs; TOT -= xa;
  }
  TOT *= nr;
  if (hi < del) {
    float fin2 = fminf(hi + fminf(SCA / e.hs, TOT / e.ha), hf);
    if (om != -1) { if (fin2 < del) { del = fin2; om = -1; } }
    else {
      if (fin2 < del) del = fin2;
      else del = fminf(fin2, sca);
    }
    fin2 = del - hi;
    SCA -= fin2 * e.hs; TOT -= fin2 * e.ha;
  }
  t.SCA = SCA; t.TOT = TOT; t.del = del; t.om = om;
  return t;
}

// gpu/pro.cu:728: a step with a non-finite optical depth is counted (and the first four SMs
// where it happened recorded); the photon is then dropped by the caller
__device__ __noinline__ void record_nan_step(const KArgs& a) {
  unsigned int k = atomicAdd(&a.ctrl->nan_steps, 1u);
  if (k < 4) { unsigned int sm; asm volatile("mov.u32 %0, %%smid;" : "=r"(sm)); a.ctrl->bad_sm[k] = sm; }
}

// Tables in dynamic shared memory (load_dyn): the string-proximity cells and the
// birefringence angular functions per interval.
constexpr size_t kBfrBytes = PPCB_BFR_TAB * (sizeof(float4) + sizeof(float2));
struct DynTabs {
  const uint16_t* cells;
  const float4* bfr0;
  const float2* bfr1;
};

// String-proximity table as the kernel reads it: cell entries in dynamic shared memory,
// string axes in the static tables.
struct SgTab {
  const SmemTables& S;
  const uint16_t* cells;
  __device__ __forceinline__ uint32_t cell(int k) const { return cells[k]; }
  __device__ __forceinline__ const StrGroup& group(int m) const { return S.sgg[m]; }
};

// Result of the DOM search: the hit DOM (or -1) and its distance, the hole-ice column
// entry and exit, and sqd of the last DOM whose quadratic had a root (gpu/pro.cu:644).
struct Found {
  int om;
  float del, hi, hf, sqd;
};

// gpu/pro.cu:577-672: the DOM search through the search-cell grid, in the reference's
// order (cells, then the strings of each cell, then the DOM window of each string).  It
// runs only for the steps the string-proximity table cannot rule out.  Inlined: as a call
// it would make the step save and restore its live registers around the call site.
__device__ __forceinline__ Found dom_search(const KArgs& a, const SmemTables& S, float4 r, float4 n, float sca, int old,
                                         int ofla) {
  const ppcb_params& e = a.p;
  int om = -1;
  float del = sca, hi = sca, hf = 0, sqd = 0;
  {  // DOM search, gpu/pro.cu:577-672
    int xlx, xhx, xly, xhy;
    cell_range(e, r.x, r.y, fa(r.x, fm(sca, n.x)), fa(r.y, fm(sca, n.y)), xlx, xhx, xly, xhy);
    const bool hole_on = e.hr > 0 && (e.hifl == 0 || (e.hifl < 0 && r.w < -e.hifl) || (e.hifl > 0 && r.w > e.hifl));
    for (int i = xlx, j = xly; i <= xhx && j <= xhy; (++j <= xhy) ? 0 : (j = xly, i++)) {
      for (unsigned int k = S.is[i * PPCB_CY + j]; k != 0x8000;) {
        unsigned int m = S.ls[k];
        const ppcb_line& sl = S.sc[m & 0x7fff];
        k = (m & 0x8000) ? 0x8000 : k + 1;
        float b = 0, c = 0, dr;
        dr = sl.x - r.x; b += n.x * dr; c += dr * dr;
        dr = sl.y - r.y; b += n.y * dr; c += dr * dr;
        float np = 1 - n.z * n.z;
        float D = b * b - (c - sl.r * sl.r) * np;
        if (D >= 0) {
          D = sqrtf(D);
          float h1 = b - D, h2 = b + D;
          if (h2 >= 0 && h1 <= sca * np) {
            if (np > XXX) {
              h1 /= np; h2 /= np;
              if (h1 < 0) h1 = 0;
              if (h2 > sca) h2 = sca;
            } else { h1 = 0; h2 = sca; }
            h1 = r.z + n.z * h1; h2 = r.z + n.z * h2;
            float zl, zh;
            if (n.z > 0) { zl = h1; zh = h2; }
            else { zl = h2; zh = h1; }
            int n1, n2;
            dom_window(sl, zl, zh, n1, n2);
            for (int l = n1; l <= n2; l++) if (l != old) {
              const ppcb_dom dom = a.oms[l];
              float aa = 0, bb = 0, cc = 0, dd;
              float fq = dom.F > 0 ? (1 / dom.F) * (1 / dom.F) : 0;
              dd = dom.r[0] - r.x; aa += n.x * n.x; bb += n.x * dd; cc += dd * dd;
              dd = dom.r[1] - r.y; aa += n.y * n.y; bb += n.y * dd; cc += dd * dd;
              dd = dom.r[2] - r.z; aa += fq * n.z * n.z; bb += fq * n.z * dd; cc += fq * dd * dd;
              if (aa > 0) {
                bb /= aa;
                float xR = (l == ofla ? 1 : e.xR);
                float DD = bb * bb - (cc - (xR * dom.R) * (xR * dom.R)) / aa;
                if (DD >= 0) {
                  sqd = sqrtf(DD);
                  float h = bb - sqd;
                  if (dom.F > 0 || fabsf(dd - n.z * h) < -xR * dom.F * dom.R) {
                    sqd /= xR; h = bb - sqd;
                    if (h > 0 && h <= del) { om = l; del = h; }
                  }
                }
              }
            }
          }
        }
        if (hole_on) {  // hole-ice column around the string
          const float2 h = hole_column(e, b, c, np, sca, hi, hf);
          hi = h.x; hf = h.y;
        }
      }
    }
  }

  return Found{om, del, hi, hf, sqd};
}

// gpu/pro.cu:499-888: one propagation step (one scattering segment).  Returns with
// ph.TOT == 0 once the photon is absorbed or registered.
template <class HOOK>
__device__ __forceinline__ void step(const KArgs& a, const SmemTables& S, const DynTabs& dt, Photon& ph, Rng& s,
                                     unsigned int& nan_steps, HOOK& hk) {
  const ppcb_params& e = a.p;
  const float2* __restrict__ wz = a.absca + (size_t)ph.wl * e.size;
  float4 r = ph.r, n = ph.n;
  float TOT = ph.TOT, SCA = ph.SCA;
  int om = ph.om0;
  float sqd = 0;
  if (SCA == 0) { SCA = -logf(xrnd(s)); ph.old = om; }
  const int old = ph.old;
  float sca, tot;
  int sign = n.z < 0 ? -1 : 1;
  float anz = sign * n.z;
  float edh = e.dh;
  float zs = zshift(e, S, a.lp, r.x, r.y, r.z, edh);
  float z;
  int I = layer_of(e, r.z, zs, z);
  int J;
  float nr = 1.f;
  {
    if (TOT > 0) {  // absorption anisotropy, gpu/pro.cu:517-544
      float2 n12 = __ffma2_rn(make_float2(e.azx, -e.azy), make_float2(n.x, n.x),
                              __fmul2_rn(make_float2(e.azy, e.azx), make_float2(n.y, n.y)));
      float n1 = n12.x, n2 = n12.y;
      float n3 = n.z;
      if (e.fr != 0) {
        float k1 = S.az[I].k1, k2 = S.az[I].k2;
        float kz = 1 / (k1 * k2);
        float s1 = n1 * n1, l1 = k1 * k1;
        float s2 = n2 * n2, l2 = k2 * k2;
        float s3 = n3 * n3, l3 = kz * kz;
        float B2 = nr / l1 + nr / l2 + nr / l3;
        float nB = s1 / l1 + s2 / l2 + s3 / l3;
        float An = s1 * l1 + s2 * l2 + s3 * l3;
        nr = powf((B2 - nB) * An / 2, e.fr);
      }
      n12 = __fmul2_rn(n12, make_float2(e.k1, e.k2));
      n1 = n12.x; n2 = n12.y; n3 *= e.kz;
      nr *= rsqrtf(n1 * n1 + n2 * n2 + n3 * n3);
      TOT /= nr;
    }
    float ahx = edh * (0.5f - sign * (z - I));
    J = I;  // layer stepping, gpu/pro.cu:548-571
    // (absorption, scattering) pairs in two-lane FP32 operations, as the table stores them
    float2 ts = make_float2(0.f, 0.f);   // (tot, sca)
    float2 aa = make_float2(TOT, SCA);   // (aia, ais)
    float2 c = ice(wz, J);
    while (true) {
      float dsca = aa.y / c.y, dtot = aa.x / c.x;
      float dist = fminf(dsca, dtot) * anz;
      if ((sign < 0 ? J > 0 : J < e.size - 1) && dist > ahx) {
        float del = ahx / anz;
        ts = __fadd2_rn(ts, make_float2(del, del));
        aa = __ffma2_rn(c, make_float2(-del, -del), aa);
        ahx = edh;
        J += sign;
        c = ice(wz, J);
      } else {
        ts = __fadd2_rn(ts, make_float2(dtot, dsca));
        break;
      }
    }
    tot = ts.x; sca = ts.y;
    if (sca < 0) sca = 0;
    if (tot < 0) tot = 0;
    if (tot < sca) { sca = tot; tot = 0; }
    else tot = (tot - sca) * c.x;
  }

  om = -1;
  float del = sca;
  float hi = sca, hf = 0;
  // DOM search, gpu/pro.cu:577-672: only for the steps that may reach a string's cylinder
  // (strgrid.h; on the full detector about 0.2% of them); for the others it would find
  // nothing and leave om, del, hi, hf and sqd as they are
  if (sg_may_reach(a.sg, SgTab{S, dt.cells}, r.x, r.y, n.x, n.y, n.z, sca)) {
    const Found f = dom_search(a, S, r, n, sca, old, ph.ofla);
    om = f.om; del = f.del; hi = f.hi; hf = f.hf; sqd = f.sqd;
  }

  float fin = fminf(del, hi);
  bool hole = fin < sca;
  if (hole) {  // truncated step (a DOM or the hole-ice column ends it first): rare, out of line
    const Truncated t = truncated_step(e, wz, z, n.z, fin, edh, I, sign, anz, SCA, TOT, nr, hi, hf, del, sca, om);
    SCA = t.SCA; TOT = t.TOT; del = t.del; om = t.om; J = t.J;
  } else { SCA = 0; TOT = tot * nr; }

  hk.segment(I, z, sign, anz, edh, nr, fin, n.z, e.size);  // bulk-ice part of the step (the rest is hole ice)
  {
    const float2 d2 = make_float2(del, del);
    const float2 rxy = __ffma2_rn(d2, make_float2(n.x, n.y), make_float2(r.x, r.y));
    const float2 rzw = __ffma2_rn(d2, make_float2(n.z, n.w), make_float2(r.z, r.w));
    r = make_float4(rxy.x, rxy.y, rzw.x, rzw.y);
  }

  if (!isfinite(TOT) || !isfinite(SCA)) {  // gpu/pro.cu:728
    record_nan_step(a);
    TOT = 0; om = -1;
    nan_steps++;
  }

  if (om != -1) {  // DOM hit, gpu/pro.cu:731-753
    if (om == ph.ofla) TOT = 0;
    else {
      const ppcb_hit h = hit_record(a, om, r, n, sqd, ph.niw, ph.wl);
      hk.hit(a, h, ph);
      if (e.xR == 1) TOT = 0;
      else ph.old = om;
    }
  }

  if (TOT < XXX) TOT = 0;
  else {
    if (e.sum > 0 && fin > 0) {  // birefringence diffusion, gpu/pro.cu:757-836
      float ra, rb;
      if (I == J) {
        const float2 q = __fmul2_rn(make_float2(fin, fin), make_float2(S.az[I].ra, S.az[I].rb));
        ra = q.x; rb = q.y;
      }
      else {
        float y = z + n.z * fin / edh;
        float h = 0.5f - sign * (z - I);
        float g = 0.5f + sign * (y - J);
        ra = h * S.az[I].ra + g * S.az[J].ra;
        rb = h * S.az[I].rb + g * S.az[J].rb;
        for (int i = I + sign; i != J && (unsigned)i < (unsigned)e.size; i += sign) { ra += S.az[i].ra; rb += S.az[i].rb; }
        float f = edh / anz;
        ra *= f; rb *= f;
      }
      if (ra < 0) ra = 0;
      if (rb < 0) rb = 0;
      // The (x, y) components go through the two-lane FP32 operations (__ffma2_rn,
      // __fmul2_rn, __fadd2_rn: one instruction for two operations), the z component alone.
      const float2 nxy = make_float2(n.x, n.y);
      float dot = e.azx * n.x + e.azy * n.y;
      // angular diffusion functions of gpu/pro.cu:784-786, tabulated on the host in
      // v = sqrt(1 - |dot|) (smooth in v at both ends) and interpolated linearly
      float2 sxy;
      float mx;
      {
        const float v = sqrtf(fmaxf(0.f, 1.f - fabsf(dot))) * PPCB_BFR_TAB;
        const int iv = min((int)v, PPCB_BFR_TAB - 1);
        const float fv = v - iv;
        const float4 t0 = dt.bfr0[iv];
        const float2 d01 = dt.bfr1[iv];
        const float sra = sqrtf(ra);
        sxy = __fmul2_rn(make_float2(sra, sra), __ffma2_rn(make_float2(fv, fv), d01, make_float2(t0.x, t0.y)));
        mx = rb * fmaf(fv, t0.w, t0.z);
      }
      const float sg = dot < 0 ? -1.f : 1.f;
      float2 qxy = __fmul2_rn(__ffma2_rn(make_float2(-dot, -dot), nxy, make_float2(e.azx, e.azy)), make_float2(sg, sg));
      float qz = -dot * n.z * sg;
      float qn = qxy.x * qxy.x + qxy.y * qxy.y + qz * qz;
      if (qn > 0) {
        float f = rsqrtf(qn);
        qxy = __fmul2_rn(qxy, make_float2(f, f)); qz *= f;
      } else { qxy = make_float2(0.f, 0.f); qz = 1; }
      const float2 pxy = __ffma2_rn(make_float2(n.y, n.z), make_float2(qz, qxy.x),
                                    __fmul2_rn(make_float2(-n.z, -n.x), make_float2(qxy.y, qz)));
      const float pz = n.x * qxy.y - n.y * qxy.x;
      float2 rnd = grnd2(s);
      float2 dn = __ffma2_rn(sxy, rnd, make_float2(mx, 0.f));
      if (del <= hi) {  // curved path within the segment
        rnd = grnd2(s);
        float2 vn = __fmul2_rn(__ffma2_rn(__fmul2_rn(sxy, rnd), make_float2(rsqrtf(3.f), rsqrtf(3.f)), dn),
                               make_float2(0.5f, 0.5f));
        float den = vn.x * vn.x + vn.y * vn.y;
        float dnz = -den;
        den = 2 / (1 + den);
        vn = __fmul2_rn(vn, make_float2(den, den)); dnz *= den;
        float2 mxy = __ffma2_rn(nxy, make_float2(dnz, dnz),
                                __ffma2_rn(pxy, make_float2(vn.y, vn.y), __ffma2_rn(qxy, make_float2(vn.x, vn.x), nxy)));
        float4 m;
        m.x = mxy.x; m.y = mxy.y;
        m.z = n.z + qz * vn.x + pz * vn.y + n.z * dnz;
        normalize3(m);
        del -= fin / 2;
        const float2 rxy = __ffma2_rn(make_float2(del, del), __fadd2_rn(make_float2(m.x, m.y), make_float2(-n.x, -n.y)),
                                      make_float2(r.x, r.y));
        r.x = rxy.x; r.y = rxy.y;
        r.z += del * (m.z - n.z);
      }
      dn = __fmul2_rn(dn, make_float2(0.5f, 0.5f));
      float den = dn.x * dn.x + dn.y * dn.y;
      float dnz = -den;
      den = 2 / (1 + den);
      dn = __fmul2_rn(dn, make_float2(den, den)); dnz *= den;
      const float2 nn = __ffma2_rn(nxy, make_float2(dnz, dnz),
                                   __ffma2_rn(pxy, make_float2(dn.y, dn.y), __ffma2_rn(qxy, make_float2(dn.x, dn.x), nxy)));
      n.z += qz * dn.x + pz * dn.y + n.z * dnz;
      n.x = nn.x; n.y = nn.y;
      normalize3(n);
    }
    if (SCA < XXX) {  // scattering, gpu/pro.cu:838-887
      if (!hole) hk.scatter(J, ice(wz, J).y);
      SCA = 0;
      const float4 c0 = S.scat[hole][0], c1 = S.scat[hole][1];
      float xi = xrnd(s);
      if (xi > c0.x) {
        xi = (1 - xi) * c0.w;
        xi = 2 * xi - 1;
        if (c0.y != 0) {
          float ga = c1.x / (1 + c0.y * xi);
          xi = (ga * ga - c1.y) * c1.z;
        }
      } else {
        xi *= c1.w;
        xi = 2 * (1 - powf(xi, c0.z));
      }
      if (xi < 0) xi = 0;
      else if (xi > 2) xi = 2;
      const float k1 = S.az[J].k1, k2 = S.az[J].k2;
      const float okz = k1 * k2;
      if (!hole) {  // stretch into the anisotropic frame
        float n1 = (e.azx * n.x + e.azy * n.y) * k1;
        float n2 = (-e.azy * n.x + e.azx * n.y) * k2;
        n.x = n1 * e.azx - n2 * e.azy;
        n.y = n1 * e.azy + n2 * e.azx;
        n.z *= S.azr[J].z;
        normalize3(n);
      }
      rotate(xi, sqrtf(xi * (2 - xi)), n, s);
      if (!hole) {
        float n1 = (e.azx * n.x + e.azy * n.y) * S.azr[J].x;
        float n2 = (-e.azy * n.x + e.azx * n.y) * S.azr[J].y;
        n.x = n1 * e.azx - n2 * e.azy;
        n.y = n1 * e.azy + n2 * e.azx;
        n.z *= okz;
        normalize3(n);
      }
    }
  }
  ph.r = r; ph.n = n; ph.TOT = TOT; ph.SCA = SCA; ph.om0 = -1;
}

__device__ __forceinline__ void load_tables(const KArgs& a, SmemTables& S) {
  const int nt = blockDim.x, t = threadIdx.x;
  for (int i = t; i < a.p.size; i += nt) S.az[i] = a.az[i];
  for (int i = t; i < a.p.nstr; i += nt) S.sc[i] = a.sc[i];
  for (int i = t; i < PPCB_LMAX; i += nt) S.lr[i] = a.lr[i];
  for (int i = t; i < PPCB_NSTR; i += nt) S.ls[i] = a.ls[i];
  for (int i = t; i < PPCB_CX * PPCB_CY; i += nt) S.is[i] = a.is[i];
  for (int i = t; i < PPCB_CTX * PPCB_CTY; i += nt) S.mcol[i] = a.mcol[i];
  for (int i = t; i < a.sg_ngroups; i += nt) S.sgg[i] = a.sg_groups[i];
  if (t < 2) {
    const float sf = t ? a.p.SF : a.p.sf, g = t ? a.p.G : a.p.g, gr = t ? a.p.GR : a.p.gr;
    S.scat[t][0] = make_float4(sf, g, gr, __fdiv_rn(1.f, __fsub_rn(1.f, sf)));
    S.scat[t][1] = make_float4(__fsub_rn(1.f, __fmul_rn(g, g)), __fmul_rn(__fsub_rn(1.f, g), __fsub_rn(1.f, g)),
                               __fdiv_rn(1.f, __fmul_rn(2.f, g)), __fdiv_rn(1.f, sf));
  }
  for (int i = t; i < a.p.size; i += nt) {
    const ppcb_aniz z = a.az[i];
    S.azr[i] = make_float4(__fdividef(1.f, z.k1), __fdividef(1.f, z.k2), __fdividef(1.f, z.k1 * z.k2), 0.f);
  }
  __syncthreads();
}

// The string-proximity cell entries into (dynamic) shared memory; bytes they take there.
__host__ __device__ __forceinline__ size_t sg_cells_bytes(const KArgs& a) {
  return a.sg.on ? (((size_t)a.sg.nx * a.sg.ny * sizeof(uint16_t) + 15) & ~(size_t)15) : 0;
}
__device__ __forceinline__ void load_cells(const KArgs& a, uint16_t* cells) {
  const int n = a.sg.on ? a.sg.nx * a.sg.ny : 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) cells[i] = a.sg_cells[i];
  __syncthreads();
}

// Tables in dynamic shared memory: the string-proximity cells, then the birefringence
// angular functions per interval as (sx, sy, mx, next mx - mx) and (next sx - sx,
// next sy - sy): one 16-byte and one 8-byte load per step, and the differences the
// interpolation needs rounded once here instead of every step (the same floats).
__device__ __forceinline__ DynTabs load_dyn(const KArgs& a, unsigned char* base) {
  uint16_t* cells = reinterpret_cast<uint16_t*>(base);
  float4* b0 = reinterpret_cast<float4*>(base + sg_cells_bytes(a));
  float2* b1 = reinterpret_cast<float2*>(base + sg_cells_bytes(a) + PPCB_BFR_TAB * sizeof(float4));
  for (int i = threadIdx.x; i < PPCB_BFR_TAB; i += blockDim.x) {
    const float4 t0 = a.bfrt[i], t1 = a.bfrt[i + 1];
    b0[i] = make_float4(t0.x, t0.y, t0.z, __fsub_rn(t1.z, t0.z));
    b1[i] = make_float2(__fsub_rn(t1.x, t0.x), __fsub_rn(t1.y, t0.y));
  }
  load_cells(a, cells);
  return DynTabs{cells, b0, b1};
}

#define PPCB_BLOCK 256

// Per-warp pool of sampled photons (photon regrouping by state).  Sampling a photon is
// long and branchy (source type, gamma profile, Cherenkov cone); done by the one or two
// lanes whose photon just died it runs at 1/32 SIMT efficiency.  Instead the whole warp
// samples up to 32 photons at once into the pool, and lanes whose photon died take one
// from the pool (three 16-byte shared-memory loads).  With per-photon streams the pool
// also carries each photon's stream state.
template <bool STREAMS>
struct PhotonPool {
  float4 r[32];
  float4 n[32];
  int4 m[32];                   // wavelength bin, segment, flasher DOM, veto code
  uint4 st[STREAMS ? 32 : 1];   // per-photon streams: state x, y and multiplier index
};

// Random streams.  Thread streams (STREAMS = false, the reference's scheme): each thread
// owns one MWC stream that runs on from photon to photon and from launch to launch.
// Per-photon streams (STREAMS = true): photon i starts from photon_stream(seed, i) with
// multiplier rm[i mod min(T, 1024)], and its state travels with it through the pool, so
// its random numbers do not depend on which lane samples or propagates it or on what ran
// before -- two launches that differ only in the ice see the same numbers per photon.
// Dynamic shared memory of a block: the warps' photon pools, then (recording pass) one
// provenance slot per thread.
template <int BLOCK, bool REC, bool STREAMS>
__host__ __device__ constexpr size_t dyn_smem() {
  return (BLOCK / 32) * sizeof(PhotonPool<STREAMS>) + (REC ? BLOCK * sizeof(Prov) : 0);
}

template <int BLOCK, int MINB, bool REC, bool STREAMS>
__global__ void __launch_bounds__(BLOCK, MINB) k_propagate(const __grid_constant__ KArgs a) {
  __shared__ SmemTables S;
  extern __shared__ __align__(16) unsigned char dsm[];
  PhotonPool<STREAMS>* pools = reinterpret_cast<PhotonPool<STREAMS>*>(dsm);
  Prov* snaps = reinterpret_cast<Prov*>(dsm + (BLOCK / 32) * sizeof(PhotonPool<STREAMS>));
  __shared__ unsigned long long bsteps;  // the block's propagation steps
  if (threadIdx.x == 0) bsteps = 0;
  load_tables(a, S);
  const DynTabs dt = load_dyn(a, dsm + dyn_smem<BLOCK, REC, STREAMS>());
  // launch sizes: from the parameters, or from device memory for replayed graphs
  const uint64_t num = a.dyn ? a.dyn[0] : a.num;
  const int nb = a.dyn ? (int)a.dyn[1] : a.nb;
  const uint32_t T = gridDim.x * blockDim.x;
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nmul = T < 1024u ? T : 1024u;  // multipliers used by per-photon streams
  const unsigned int lane = threadIdx.x & 31;
  const unsigned int FULL = 0xffffffffu;
  PhotonPool<STREAMS>& P = pools[threadIdx.x >> 5];
  Rng s;
  uint32_t mi = gt;  // multiplier index of the stream in s
  {
    uint64_t st = a.rs[gt];
    s.x = (uint32_t)st; s.y = (uint32_t)(st >> 32); s.a = a.rm[gt];
  }
  Photon ph;
  bool alive = false;
  bool exhausted = false;   // warp-uniform: no photons left to sample
  int have = 0;             // warp-uniform: photons in the pool
  // rarely used per-thread state in shared memory instead of registers: the next photon
  // index in the static order and the last bunch found
  __shared__ uint64_t s_sidx[BLOCK];
  __shared__ int s_hint[BLOCK];
  s_sidx[threadIdx.x] = gt;
  s_hint[threadIdx.x] = 0;
  unsigned int nan_steps = 0;
  // REC: the gradient's recording pass (same step code as the replay, see AdjHook)
  typename std::conditional<REC, AdjHook, NoHook>::type hk;
  if constexpr (REC) {
    hk.replay = false;
    hk.done = false;
    hk.prov_out = static_cast<Prov*>(a.prov);
    hk.start = &snaps[threadIdx.x];
  }
  // every lane of the warp stays in this loop until the warp is done, so the warp-wide
  // operations below always see all 32 lanes
  while (true) {
    const unsigned int dead = __ballot_sync(FULL, !alive);
    if (dead && !(exhausted && have == 0)) {
      // --- sample: each generating lane produces one photon
      bool gen = false;
      uint64_t gidx = 0;
      unsigned long long base = 0;
      int ngen = 0;
      if (a.deterministic == 1) {  // photon i on thread i mod T, as the oracle sequences it
        gen = !alive && s_sidx[threadIdx.x] < num;
        gidx = s_sidx[threadIdx.x];
        if (!alive) s_sidx[threadIdx.x] += T;
      } else if ((have < __popc(dead) || have < a.refill_below) && !exhausted) {
        ngen = 32 - have;
        if (lane == 0) base = atomicAdd(&a.ctrl->next, (unsigned long long)ngen);
        base = __shfl_sync(FULL, base, 0);
        gidx = base + lane;
        gen = (int)lane < ngen && gidx < num;
        if (base + ngen >= num) exhausted = true;
      }
      Photon g;
      uint4 gst = make_uint4(0, 0, 0, 0);
      if (gen) {
        const int hint = find_bunch(a, nb, gidx, s_hint[threadIdx.x]);
        s_hint[threadIdx.x] = hint;
        if constexpr (STREAMS) {  // the photon's own stream; the lane's s is left alone
          Rng sg;
          const uint32_t m = (uint32_t)(gidx % nmul);
          sg.a = a.rm[m];
          photon_stream(sg, gidx, a.seed);
          const Sampled smp = sample_photon(a, hint, sg.x, sg.y, sg.a);
          g = smp.ph;
          gst = make_uint4(smp.x, smp.y, m, 0);
        } else {
          const Sampled smp = sample_photon(a, hint, s.x, s.y, s.a);
          g = smp.ph;
          s.x = smp.x; s.y = smp.y;
        }
      }
      if (a.deterministic == 1) {
        if (gen) {
          ph = g;
          alive = true;
          if constexpr (STREAMS) { s.x = gst.x; s.y = gst.y; mi = gst.z; s.a = a.rm[mi]; }
        }
        exhausted = __all_sync(FULL, s_sidx[threadIdx.x] >= num);
      } else {
        if (gen) {
          const int slot = have + lane;
          P.r[slot] = g.r;
          P.n[slot] = g.n;
          P.m[slot] = make_int4(g.wl, (int)g.niw, g.om0, g.ofla);
          if constexpr (STREAMS) P.st[slot] = gst;
        }
        have += __popc(__ballot_sync(FULL, gen));
        __syncwarp();
        // --- hand out: the k-th dead lane takes the k-th photon from the top of the pool
        const int rank = __popc(dead & ((1u << lane) - 1u));
        if (!alive && rank < have) {
          const int slot = have - 1 - rank;
          ph.r = P.r[slot];
          ph.n = P.n[slot];
          const int4 m = P.m[slot];
          ph.wl = m.x; ph.niw = (uint32_t)m.y; ph.om0 = m.z; ph.ofla = m.w;
          if constexpr (STREAMS) {
            const uint4 t = P.st[slot];
            s.x = t.x; s.y = t.y; mi = t.z; s.a = a.rm[mi];
          }
          alive = true;
        }
        have -= min(have, __popc(dead));
        __syncwarp();
      }
      if (alive && (dead >> lane & 1u)) {  // a fresh photon: absorption depth, gpu/pro.cu:496-497
        ph.nhit = 0;
        if constexpr (REC) {
          hk.start->r = ph.r;
          hk.start->n = ph.n;
          hk.start->m = make_int4(ph.wl, (int)ph.niw, ph.om0, ph.ofla);
          hk.start->s = make_uint4(s.x, s.y, mi, 0);
        }
        ph.TOT = -logf(xrnd(s));
        ph.SCA = 0;
        ph.old = -1;
        ph.steps = 0;
        if (ph.ofla < -1) ph.TOT = 0;
      }
    }
    if (!__any_sync(FULL, alive)) {
      if (exhausted && have == 0) break;
      continue;
    }
    if (alive) {
      step(a, S, dt, ph, s, nan_steps, hk);
      ph.steps++;
      if (a.max_steps && ph.steps >= a.max_steps && ph.TOT != 0) {  // the step cap (rare)
        ph.TOT = 0;
        atomicAdd(&a.ctrl->capped, 1u);
      }
      if (ph.TOT == 0) {  // the photon's steps go to the block's count
        alive = false;
        atomicAdd(&bsteps, (unsigned long long)ph.steps);
      }
    }
  }
  if constexpr (!STREAMS) a.rs[gt] = (uint64_t)s.x | ((uint64_t)s.y << 32);
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(&a.ctrl->steps, bsteps);
}

// Charge bin of a hit: its DOM, or with `events` > 0 (event, DOM) with the event taken
// from the hit's segment id; -1 for a segment id outside [0, events).
__device__ __forceinline__ long long charge_bin(const ppcb_hit& h, uint32_t events, int gsize) {
  if (!events) return h.i;
  return h.n < events ? (long long)h.n * gsize + h.i : -1;
}

// Gradient replay: one thread per recorded hit.  The photon is restarted from its
// provenance (sampled state, stream state, thread multiplier) and stepped with the same
// step<AdjHook> code as the recording pass, so it retraces the same path; the hook sums
// the path's per-layer derivative terms, weighted by the hit's DOM weight, until the
// recorded hit is reached again.  A replay that does not end on the recorded hit (same
// DOM, same time bits) is counted in stats[1].
__global__ void __launch_bounds__(256, 3) k_adjoint(const __grid_constant__ KArgs a, const ppcb_hit* __restrict__ hits,
                                                 const Prov* __restrict__ prov, uint64_t cap,
                                                 const unsigned long long* nh_dev, uint32_t events,
                                                 const float* __restrict__ wdom, const float2* __restrict__ wgrad,
                                                 double* g_out, unsigned int* stats) {
  // hits to replay: `cap`, or the recording pass's count from device memory (graph replays)
  const uint64_t nh = nh_dev ? (*nh_dev < cap ? *nh_dev : cap) : cap;
  __shared__ SmemTables S;
  __shared__ double gbe[PPCB_MAXLYS], gba[PPCB_MAXLYS];
  extern __shared__ __align__(16) unsigned char dsm[];
  for (int i = threadIdx.x; i < PPCB_MAXLYS; i += blockDim.x) { gbe[i] = 0; gba[i] = 0; }
  load_tables(a, S);
  const DynTabs dt = load_dyn(a, dsm);
  unsigned int nan_steps = 0, replayed = 0, unmatched = 0;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nh; k += (uint64_t)gridDim.x * blockDim.x) {
    const ppcb_hit h = hits[k];
    const long long bin = charge_bin(h, events, a.p.gsize);
    const float w = bin >= 0 ? wdom[bin] : 0.f;
    if (w == 0) continue;
    const Prov P = prov[k];
    Rng s;
    s.x = P.s.x; s.y = P.s.y; s.a = a.rm[P.s.z];
    Photon ph;
    ph.r = P.r; ph.n = P.n;
    ph.wl = P.m.x; ph.niw = (uint32_t)P.m.y; ph.om0 = P.m.z; ph.ofla = P.m.w;
    ph.nhit = 0;
    ph.TOT = -logf(xrnd(s));  // as at pick-up in the recording pass
    ph.SCA = 0;
    ph.old = -1;
    ph.steps = 0;
    if (ph.ofla < -1) ph.TOT = 0;
    AdjHook hk;
    hk.replay = true;
    hk.target = (int)P.s.w;
    hk.target_i = h.i;
    hk.target_t = h.t;
    hk.done = false;
    hk.matched = false;
    const float2 c = wgrad[ph.wl];
    hk.w_be = w * c.x;
    hk.w_ba = w * c.y;
    hk.g_be = gbe;
    hk.g_ba = gba;
    hk.prov_out = nullptr;
    hk.start = nullptr;
    while (!hk.done && ph.TOT != 0 && ph.steps < a.max_steps) {
      step(a, S, dt, ph, s, nan_steps, hk);
      ph.steps++;
    }
    replayed++;
    if (!hk.matched) unmatched++;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < a.p.size; i += blockDim.x) {
    if (gbe[i] != 0) atomicAdd(&g_out[i], gbe[i]);
    if (gba[i] != 0) atomicAdd(&g_out[PPCB_MAXLYS + i], gba[i]);
  }
  if (replayed) atomicAdd(&stats[0], replayed);
  if (unmatched) atomicAdd(&stats[1], unmatched);
}

__global__ void k_dom_hist(const ppcb_hit* __restrict__ hits, uint64_t cap, const unsigned long long* nh_dev,
                           unsigned int* counts, uint32_t events, int gsize) {
  const uint64_t nh = nh_dev ? (*nh_dev < cap ? *nh_dev : cap) : cap;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nh; k += (uint64_t)gridDim.x * blockDim.x) {
    const long long b = charge_bin(hits[k], events, gsize);
    if (b >= 0) atomicAdd(&counts[b], 1u);
  }
}

// The replay's static shared memory plus the string-proximity table exceed the default
// 48 KiB of dynamic shared memory: allow the largest table, once per device (before any
// stream capture that launches the replay there).
cudaError_t adjoint_prepare() {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!(done.load() & (1ull << (dev & 63)))) {
    e = cudaFuncSetAttribute(k_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kSgMaxCells * sizeof(uint16_t) + kBfrBytes));
    if (e != cudaSuccess) return e;
    done.fetch_or(1ull << (dev & 63));
  }
  return cudaSuccess;
}

cudaError_t launch_adjoint(const KArgs& a, const ppcb_hit* hits, const void* prov, uint64_t nh, uint32_t events,
                           const float* wdom, const float2* wgrad, double* g_out, unsigned int* stats, int blocks,
                           cudaStream_t st, const unsigned long long* nh_dev) {
  if (nh == 0) return cudaSuccess;
  const cudaError_t e = adjoint_prepare();
  if (e != cudaSuccess) return e;
  k_adjoint<<<blocks, 256, sg_cells_bytes(a) + kBfrBytes, st>>>(a, hits, static_cast<const Prov*>(prov), nh, nh_dev, events,
                                                   wdom, wgrad, g_out, stats);
  return cudaGetLastError();
}

cudaError_t launch_dom_hist(const ppcb_hit* hits, uint64_t nh, unsigned int* counts, uint32_t events, int gsize,
                            cudaStream_t st, const unsigned long long* nh_dev) {
  if (nh == 0) return cudaSuccess;
  k_dom_hist<<<592, 256, 0, st>>>(hits, nh, nh_dev, counts, events, gsize);
  return cudaGetLastError();
}

// Phase-1 only: thread t samples photon t with stream t (test entry point).
__global__ void __launch_bounds__(PPCB_BLOCK) k_generate(const __grid_constant__ KArgs a, float4* out) {
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt >= a.num) return;
  Rng s;
  uint64_t st = a.rs[gt];
  s.x = (uint32_t)st; s.y = (uint32_t)(st >> 32); s.a = a.rm[gt];
  int b = find_bunch(a, a.nb, gt, 0);
  const ppcb_bunch p = a.bunches[b];
  Photon ph;
  generate(a, p, s, ph);
  float4* o = out + 3 * (size_t)gt;
  o[0] = ph.r;
  o[1] = ph.n;
  o[2] = make_float4(__int_as_float(ph.wl), __int_as_float((int)ph.niw), __int_as_float(ph.om0),
                     __int_as_float(ph.ofla));
  a.rs[gt] = (uint64_t)s.x | ((uint64_t)s.y << 32);
}

// Index helpers at given points (test entry point).  pos[2k] = (x,y,z,t) start,
// pos[2k+1] = (nx,ny,nz,len) direction and segment length.  Outputs per point:
// ints  [layer, xlx, xhx, xly, xhy, n1, n2, string]   floats [zshift, dz]
__global__ void k_index_probe(const __grid_constant__ KArgs a, const float4* pos, int np, int32_t* oi, float* of) {
  __shared__ SmemTables S;
  load_tables(a, S);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const float4 r = pos[2 * k], n = pos[2 * k + 1];
  float dz = a.p.dh;
  float zs = zshift(a.p, S, a.lp, r.x, r.y, r.z, dz);
  float z;
  int I = layer_of(a.p, r.z, zs, z);
  int xlx, xhx, xly, xhy;
  cell_range(a.p, r.x, r.y, fa(r.x, fm(n.w, n.x)), fa(r.y, fm(n.w, n.y)), xlx, xhx, xly, xhy);
  const int m = k % (a.p.nstr > 0 ? a.p.nstr : 1);
  int n1 = 0, n2 = -1;
  if (a.p.nstr > 0) {
    float z1 = r.z, z2 = fa(r.z, fm(n.w, n.z));
    dom_window(S.sc[m], fminf(z1, z2), fmaxf(z1, z2), n1, n2);
  }
  int32_t* o = oi + 8 * k;
  o[0] = I; o[1] = xlx; o[2] = xhx; o[3] = xly; o[4] = xhy; o[5] = n1; o[6] = n2; o[7] = m;
  of[2 * k] = zs;
  of[2 * k + 1] = dz;
}

// Compiled shapes: 256 threads x 3 blocks per SM, 128 x 6 and 768 x 1 (768 threads per SM
// at 80 registers), and 864 x 1 (27 warps at 72 registers); the autotuner picks one.  With
// one block per SM the shared tables are held once instead of three times, which leaves
// that memory to the L1 cache.  Per-photon streams run with
// deterministic = 2, and in the gradient's recording pass unless the photon order is
// static (deterministic = 1: thread streams, photon i on thread i mod T, nothing interleaves).
// The dynamic shared-memory limit is a per-device function attribute: set it once on each
// device (before any stream capture that launches the kernel there).
// Dynamic shared memory: the photon pools (and provenance slots), then the
// string-proximity cell entries; the attribute allows the largest table.
template <int BLOCK, int MINB, bool REC, bool STREAMS>
static cudaError_t launch_one(const KArgs& a, int blocks, cudaStream_t st) {
  constexpr size_t dmax = dyn_smem<BLOCK, REC, STREAMS>() + kSgMaxCells * sizeof(uint16_t) + kBfrBytes;
  const size_t dyn = dyn_smem<BLOCK, REC, STREAMS>() + sg_cells_bytes(a) + kBfrBytes;
  if (dyn > dmax) return cudaErrorInvalidValue;
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(done.load() & bit)) {
    e = cudaFuncSetAttribute(k_propagate<BLOCK, MINB, REC, STREAMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dmax);
    if (e != cudaSuccess) return e;
    done.fetch_or(bit);
  }
  k_propagate<BLOCK, MINB, REC, STREAMS><<<blocks, BLOCK, dyn, st>>>(a);
  return cudaGetLastError();
}

template <bool REC, bool STREAMS>
static cudaError_t launch_shape(const KArgs& a, LaunchShape sh, cudaStream_t st) {
  if constexpr (REC) {
    switch (sh.threads) {
      case 256: return launch_one<256, 3, true, STREAMS>(a, sh.blocks, st);
      case 864: return launch_one<864, 1, true, STREAMS>(a, sh.blocks, st);
      default: return cudaErrorInvalidConfiguration;
    }
  } else {
    switch (sh.threads) {
      case 256: return launch_one<256, 3, false, STREAMS>(a, sh.blocks, st);
      case 128: return launch_one<128, 6, false, STREAMS>(a, sh.blocks, st);
      case 768: return launch_one<768, 1, false, STREAMS>(a, sh.blocks, st);
      case 864: return launch_one<864, 1, false, STREAMS>(a, sh.blocks, st);
      default: return cudaErrorInvalidConfiguration;
    }
  }
}

cudaError_t launch_propagate(const KArgs& a, LaunchShape sh, cudaStream_t st) {
  if (a.deterministic < 0 || a.deterministic > 2) return cudaErrorInvalidValue;
  if (a.prov) {
    return a.deterministic == 1 ? launch_shape<true, false>(a, sh, st) : launch_shape<true, true>(a, sh, st);
  }
  return a.deterministic == 2 ? launch_shape<false, true>(a, sh, st) : launch_shape<false, false>(a, sh, st);
}

cudaError_t launch_generate(const KArgs& a, LaunchShape, void* pbuf_out, cudaStream_t st) {
  int blocks = (int)((a.num + PPCB_BLOCK - 1) / PPCB_BLOCK);
  if (blocks == 0) return cudaSuccess;
  k_generate<<<blocks, PPCB_BLOCK, 0, st>>>(a, (float4*)pbuf_out);
  return cudaGetLastError();
}

cudaError_t launch_index_probe(const KArgs& a, const float4* pos, int n, int32_t* out_i, float* out_f,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_index_probe<<<(n + 255) / 256, 256, 0, st>>>(a, pos, n, out_i, out_f);
  return cudaGetLastError();
}

cudaError_t propagate_attributes(int* regs, int* max_threads, size_t* smem, size_t* local) {
  cudaFuncAttributes at;
  cudaError_t e = cudaFuncGetAttributes(&at, k_propagate<256, 3, false, false>);
  if (e != cudaSuccess) return e;
  *regs = at.numRegs;
  *max_threads = at.maxThreadsPerBlock;
  *smem = at.sharedSizeBytes;
  *local = at.localSizeBytes;
  return cudaSuccess;
}

template <int BLOCK, int MINB>
static int max_blocks(int* nb) {
  // the larger pool (per-photon streams) and the largest string-proximity table
  constexpr size_t dyn = dyn_smem<BLOCK, false, true>() + kSgMaxCells * sizeof(uint16_t) + kBfrBytes;
  cudaError_t e = cudaFuncSetAttribute(k_propagate<BLOCK, MINB, false, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_propagate<BLOCK, MINB, false, false>, BLOCK, dyn);
  return e == cudaSuccess ? *nb : 0;
}

// Resident blocks per SM of the gradient's recording kernel (its provenance slots and the
// largest string-proximity table included); 0 when the shape does not fit.
template <int BLOCK, int MINB, bool STREAMS>
static int rec_blocks(int* nb) {
  constexpr size_t dyn = dyn_smem<BLOCK, true, STREAMS>() + kSgMaxCells * sizeof(uint16_t) + kBfrBytes;
  cudaError_t e = cudaFuncSetAttribute(k_propagate<BLOCK, MINB, true, STREAMS>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(nb, k_propagate<BLOCK, MINB, true, STREAMS>, BLOCK, dyn);
  if (e != cudaSuccess) { cudaGetLastError(); return 0; }
  return *nb;
}

int propagate_rec_blocks_per_sm(int threads, int deterministic) {
  int nb = 0;
  const bool streams = deterministic != 1;
  switch (threads) {
    case 256: return streams ? rec_blocks<256, 3, true>(&nb) : rec_blocks<256, 3, false>(&nb);
    case 864: return streams ? rec_blocks<864, 1, true>(&nb) : rec_blocks<864, 1, false>(&nb);
    default: return 0;
  }
}

int propagate_max_blocks_per_sm(int threads) {
  int nb = 0;
  switch (threads) {
    case 128: return max_blocks<128, 6>(&nb);
    case 256: return max_blocks<256, 3>(&nb);
    case 768: return max_blocks<768, 1>(&nb);
    case 864: return max_blocks<864, 1>(&nb);
    default: return 0;
  }
}

}  // namespace ppcb
