// Per-hit acceptance of the device back end (gpu/f2k.cxx:247-363), shared by the back end
// (backend.cu) and the likelihood (llh.cu), and the per-device tables it reads.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "ppcb_types.h"

namespace ppcb {

constexpr int kMaxPoly = 16;

struct BackDom {
  float tilt[3];
  float azi;        // cable azimuth [deg], < 0: none
  float R, F;       // radius and spheroid factor
  float scale;      // rde / rmax
  int acc;          // acceptance table, -1: never registers (no HV, no table, rde = 0)
  int sensor;       // sensor type, -1: none
  int str, om;
};

struct BackSensor {
  float mas;        // > 0: polynomial acceptance; <= 0: threshold on the impact height
  int ns;
  float s[kMaxPoly];
};

__device__ __forceinline__ float bxrnd(uint32_t& x, uint32_t& y, uint32_t a) {
  unsigned long long sda = (unsigned long long)a * x + y;
  x = (uint32_t)sda;
  y = (uint32_t)(sda >> 32);
  return 2.f - __uint_as_float((x >> 9) | 0x3f800000u);
}

struct BackArgs {
  const ppcb_hit* hits;
  uint64_t n;
  const BackDom* doms;
  const BackSensor* sensors;
  const float* rat;     // [acceptance tables][WNUM]
  const float2* wvs;    // [WNUM] bin edges (i, f)
  const uint32_t* rm;
  uint32_t nmul, seed, gsize;
};

// decides hit k; fills `o` when accepted
__device__ __forceinline__ bool accept_one(const BackArgs& A, uint64_t k, ppcb_acc_hit& o) {
  const ppcb_hit h = A.hits[k];
  if (h.i >= A.gsize || h.z >= PPCB_WNUM) return false;
  const BackDom D = A.doms[h.i];
  if (D.acc < 0) return false;
  // the hit's stream: a SplitMix64 hash (Steele, Lea, Flood 2014) of (seed, k)
  uint64_t z = ((uint64_t)A.seed << 32 | 0x6a09e667u) + (k + 1) * 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  const uint32_t a = A.rm[k % A.nmul];
  uint32_t sx = (uint32_t)z, sy = __umulhi((uint32_t)(z >> 32), a);
  if (!(bxrnd(sx, sy, a) < A.rat[(size_t)D.acc * PPCB_WNUM + h.z] * D.scale)) return false;
  float ptc, pts, ppc, pps, dpc, dps;
  sincosf(h.pth, &pts, &ptc);
  sincosf(h.pph, &pps, &ppc);
  sincosf(h.dph, &dps, &dpc);
  const float dtc = D.F * cosf(h.dth);
  const float dts = D.F < 0 ? 1.f : sinf(h.dth);
  const float rx = dts * dpc, ry = dts * dps, rz = dtc;
  const float nx = pts * ppc, ny = pts * pps, nz = ptc;
  if (D.sensor < 0) return false;
  const BackSensor& S = A.sensors[D.sensor];
  const float u = bxrnd(sx, sy, a);
  bool flag;
  if (S.mas > 0) {
    const float x = nx * D.tilt[0] + ny * D.tilt[1] + nz * D.tilt[2];
    float y = 1, sum = S.s[0];
    for (int i = 1; i < S.ns; i++) { y *= x; sum += S.s[i] * y; }
    flag = S.mas * u < sum;
  } else {
    flag = rx * D.tilt[0] + ry * D.tilt[1] + rz * D.tilt[2] > S.s[0];
  }
  if (!flag) return false;
  if (D.azi >= 0) {  // cable shadow
    const float rc = 0.023f, dc = D.R + rc;
    float sp, cp;
    sincosf(D.azi * (PPCB_FPI / 180.f), &sp, &cp);
    const float drx = -D.R * rx - dc * cp, dry = -D.R * ry - dc * sp;
    const float aa = nx * nx + ny * ny;
    if (aa > 0) {
      const float b = -2 * (nx * drx + ny * dry);
      const float cc = drx * drx + dry * dry - rc * rc;
      const float Dd = b * b - 4 * aa * cc;
      if (Dd >= 0 && (-b + sqrtf(Dd)) / (2 * aa) > 0) return false;
    }
  }
  const float2 w = A.wvs[h.z];
  o.i = h.i; o.n = h.n; o.hit = (uint32_t)k;
  o.str = D.str; o.om = D.om; o.pmt = 0;
  o.t = h.t;
  o.wv = w.x + (w.y - w.x) * bxrnd(sx, sy, a);
  o.r[0] = -D.R * rx; o.r[1] = -D.R * ry; o.r[2] = -D.R * rz;
  o.d[0] = nx; o.d[1] = ny; o.d[2] = nz;
  return true;
}

struct BackendTables {
  BackDom* doms = nullptr;
  BackSensor* sensors = nullptr;
  float* rat = nullptr;
  float2* wvs = nullptr;
  unsigned int* block_cnt = nullptr;
  unsigned long long* block_off = nullptr;
  uint64_t blocks_cap = 0;
  ~BackendTables() {
    for (void* p : {(void*)doms, (void*)sensors, (void*)rat, (void*)wvs, (void*)block_cnt, (void*)block_off})
      if (p) cudaFree(p);
  }
};

class Engine;
// The acceptance arguments for n kernel-level hits (device pointer) on device `d`.
BackArgs back_args(Engine& e, int d, const ppcb_hit* dhits, uint64_t n, uint32_t seed);

}  // namespace ppcb
