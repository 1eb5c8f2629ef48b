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

// Sensor kinds of getPMT (gpu/ini.cxx:210-280)
constexpr int kSensorStandard = 0;  // one PMT: angular polynomial or impact-height threshold
constexpr int kSensorMultiPMT = 1;  // PMT axes with an angular response each (mDOM, D-Egg)
constexpr int kSensorTube = 2;      // wavelength-shifting tube read out at both ends (beta = -2)

struct BackSensor {
  int kind;
  float mas;        // standard: > 0 polynomial acceptance; <= 0 threshold on the impact height
  int ns;
  float s[kMaxPoly];
  float beta;       // multi-PMT: the PMTs' angular response parameter
  float fx;         // multi-PMT: maximum of (summed PMT response) / (cross-sectional area)
  float Rr, Rz;     // sensor radius and half height (Rz < 0: a cylinder)
  float cable;      // azimuth of the cable in the sensor's frame [deg]
  int dir0, ndir;   // multi-PMT: its PMT axes in the axis table
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
  const float3* dirs;   // PMT axes of the multi-PMT sensors
  const float2* wvs;    // [WNUM] bin edges (i, f)
  const uint32_t* rm;
  uint32_t nmul, seed, gsize;
};

// angular response of one PMT to light arriving at cos(angle) x off its axis (itype::f,
// gpu/ini.cxx:173-187): the projected area of a disc behind a sphere segment of opening beta
__device__ __forceinline__ float pmt_response(float beta, float x) {
  if (beta < -1) return sqrtf(1 - x * x);
  float sum = x > 0 ? x : 0;
  if (beta < 1) {
    float y = sqrtf(1 - x * x) / beta;
    if (y > 1) {
      y = 1 / y;
      const float c = 1 - beta * beta;
      const float a1 = acosf(y), a2 = acosf(y * fabsf(x) / sqrtf(c));
      sum += ((a1 - sinf(2 * a1) / 2) / c - (a2 - sinf(2 * a2) / 2) * fabsf(x)) / PPCB_FPI;
    }
  }
  return sum;
}

// cross-sectional area of the sensor seen along a direction with z component dot
// (itype::xarea, gpu/ini.cxx:189-191)
__device__ __forceinline__ float sensor_xarea(const BackSensor& S, float dot) {
  return S.Rz > 0 ? PPCB_FPI * S.Rr * sqrtf(S.Rz * S.Rz - dot * dot * (S.Rz * S.Rz - S.Rr * S.Rr))
                  : -4 * S.Rr * S.Rz * sqrtf(1 - dot * dot);
}

// multi-PMT branch of getPMT (gpu/ini.cxx:262-279): the photon direction is turned by the
// cable azimuth into the sensor's frame, then PMT k takes the hit with probability
// response_k / (fx x cross-section); -1 when none does
__device__ __forceinline__ int multi_pmt(const BackArgs& A, const BackSensor& S, float azi, float nx, float ny, float nz,
                                         float u) {
  if (azi >= 0) {
    float sp, cp;
    sincosf((azi - S.cable) * (PPCB_FPI / 180.f), &sp, &cp);
    const float x = nx * cp + ny * sp, y = ny * cp - nx * sp;
    nx = x;
    ny = y;
  }
  const float crx = S.fx * sensor_xarea(S, nz);
  float tot = 0;
  for (int k = 0; k < S.ndir; k++) {
    const float3 d = A.dirs[S.dir0 + k];
    tot += pmt_response(S.beta, -(nx * d.x + ny * d.y + nz * d.z)) / crx;
    if (tot > u) return k;
  }
  return -1;
}

// wavelength-shifting tube branch of getPMT (gpu/ini.cxx:211-237): the end that detects the
// photon, chosen from the impact height, and the transit delay to it (a King-function
// spread, absorption in the tube, paint re-emission) added to the hit time
__device__ __forceinline__ int tube_pmt(const BackSensor& S, float rz, float u, float& t, uint32_t& sx, uint32_t& sy,
                                        uint32_t a) {
  const float cn = 0.299792458f / 1.46f, absl = 3.0f / cn, att = 0.678f, cut = 0.01f, tau = 1.6f, h = 0.76f;
  const float ea = h / (1 - expf(-h / att));
  float z = S.Rr * rz;
  z *= h / fabsf(2 * S.Rz);
  const int i = u - 0.5f < z / (2 * ea) ? 1 : 0;
  z = i > 0 ? h / 2 - z : h / 2 + z;
  const float d = (z / h) * (1 - z / (2 * ea)) / (1 - h / (2 * ea));
  z = -att * logf(1 - d * (1 - expf(-h / att)));
  if (z < cut) z = cut;
  const float x = logf(z);
  const float s = expf(((0.0034112f * x + 0.041727f) * x + 0.45550f) * x - 1.9188f);
  const float g = expf(((0.0012658f * x + 0.017228f) * x - 0.012750f) * x + 0.20924f);
  float dt;
  for (int it = 0; it < 10000; it++) {  // rejection of photons absorbed on the way
    dt = s * sqrtf(2 * g * powf(1 - bxrnd(sx, sy, a), 1 / (1 - g)) - 1);
    if (!(dt > -absl * logf(bxrnd(sx, sy, a)))) break;
  }
  dt += z / cn - tau * logf(bxrnd(sx, sy, a));
  t += dt;
  return i;
}

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
  int pmt = 0;
  float t = h.t;
  if (S.kind == kSensorStandard) {
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
  } else if (S.kind == kSensorMultiPMT) {
    pmt = multi_pmt(A, S, D.azi, nx, ny, nz, u);
    if (pmt < 0) return false;
  } else {
    pmt = tube_pmt(S, rz, u, t, sx, sy, a);
  }
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
  o.str = D.str; o.om = D.om; o.pmt = pmt;
  o.t = t;
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
  float3* dirs = nullptr;
  unsigned int* block_cnt = nullptr;
  unsigned long long* block_off = nullptr;
  uint64_t blocks_cap = 0;
  ~BackendTables() {
    for (void* p : {(void*)doms, (void*)sensors, (void*)rat, (void*)wvs, (void*)dirs, (void*)block_cnt,
                    (void*)block_off})
      if (p) cudaFree(p);
  }
};

class Engine;
// The acceptance arguments for n kernel-level hits (device pointer) on device `d`.
BackArgs back_args(Engine& e, int d, const ppcb_hit* dhits, uint64_t n, uint32_t seed);

}  // namespace ppcb
