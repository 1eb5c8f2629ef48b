// Hit back end on the device (Engine::accept): the acceptance of gpu/f2k.cxx:247-363 applied
// to kernel-level hits on the GPU.  For every hit, in the reference's order of decisions:
//   1. wavelength x RDE acceptance: a DOM with high voltage and an acceptance table for its
//      (module type, variant) keeps the hit with probability rat[z] x rde / rmax;
//   2. sensor angular acceptance (standard sensors, gpu/ini.cxx:237-247): polynomial in the
//      cosine between the photon direction and the sensor axis against mas x u, or the
//      impact point's height along the axis against a threshold;
//   3. cable shadow (gpu/f2k.cxx:314-335);
//   4. wavelength sampled uniformly in the hit's wavelength bin.
// The reference draws the three uniform numbers from one host stream in hit order; here
// every hit has its own stream keyed by (seed, hit index), so the decisions are the same in
// distribution, not hit by hit.  Output is in input order (a block-level scan of the
// accept flags), so a call is deterministic for a given seed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "engine.h"

namespace ppcb {

namespace {

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
__device__ bool accept_one(const BackArgs& A, uint64_t k, ppcb_acc_hit& o) {
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

constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) k_accept_count(BackArgs A, unsigned int* block_cnt) {
  const uint64_t k = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  ppcb_acc_hit o;
  const bool f = k < A.n && accept_one(A, k, o);
  const int c = __syncthreads_count(f);
  if (threadIdx.x == 0) block_cnt[blockIdx.x] = c;
}

// exclusive scan of the block counts (one block; each thread scans a contiguous chunk)
__global__ void k_accept_scan(const unsigned int* cnt, uint64_t nb, unsigned long long* off) {
  __shared__ unsigned long long part[1024];
  const uint64_t t = threadIdx.x, nt = blockDim.x;
  const uint64_t per = (nb + nt - 1) / nt;
  const uint64_t lo = min(nb, t * per), hi = min(nb, lo + per);
  unsigned long long s = 0;
  for (uint64_t b = lo; b < hi; b++) s += cnt[b];
  part[t] = s;
  __syncthreads();
  for (unsigned int d = 1; d < nt; d <<= 1) {
    const unsigned long long v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  unsigned long long acc = part[t] - s;
  for (uint64_t b = lo; b < hi; b++) {
    off[b] = acc;
    acc += cnt[b];
  }
  if (t == nt - 1) off[nb] = part[t];
}

__global__ void __launch_bounds__(kBlock) k_accept_write(BackArgs A, const unsigned long long* off,
                                                         ppcb_acc_hit* out) {
  __shared__ unsigned int warp_cnt[kBlock / 32];
  const uint64_t k = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  ppcb_acc_hit o;
  const bool f = k < A.n && accept_one(A, k, o);
  const unsigned int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned int bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) warp_cnt[w] = __popc(bal);
  __syncthreads();
  unsigned int before = 0;
  for (unsigned int j = 0; j < w; j++) before += warp_cnt[j];
  if (f) out[off[blockIdx.x] + before + __popc(bal & ((1u << lane) - 1u))] = o;
}

}  // namespace

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

void Engine::accept_tables(int d) {
  DeviceCtx& g = devs.at(d);
  if (g.back) return;
  const Config& c = cfg;
  std::vector<BackDom> doms(c.p.gsize);
  std::vector<BackSensor> sensors;
  std::map<int, int> sensor_index;
  std::vector<float> rat;
  std::map<std::pair<int, int>, int> acc_index;
  for (int k = 0; k < c.p.gsize; k++) {
    const OMName& n = c.names[k];
    BackDom& D = doms[k];
    for (int j = 0; j < 3; j++) D.tilt[j] = n.tilt[j];
    D.azi = n.azi;
    D.R = c.oms[k].R;
    D.F = c.oms[k].F;
    D.str = n.k.str;
    D.om = n.k.dom;
    D.acc = -1;
    D.sensor = -1;
    D.scale = 0;
    if (n.hv > 0) {
      auto it = c.irdes.find(std::make_pair(n.omt, n.type));
      if (it != c.irdes.end() && it->second.rde > 0) {
        auto ai = acc_index.find(it->first);
        if (ai == acc_index.end()) {
          ai = acc_index.insert(std::make_pair(it->first, (int)acc_index.size())).first;
          std::vector<float> r(PPCB_WNUM, 0.f);
          for (int z = 0; z < PPCB_WNUM && z < (int)it->second.rat.size(); z++) r[z] = it->second.rat[z];
          rat.insert(rat.end(), r.begin(), r.end());
        }
        D.acc = ai->second;
        D.scale = n.rde / it->second.rmax;
      }
    }
    auto ti = c.types.find(n.omt);
    if (ti != c.types.end()) {
      const SensorType& T = ti->second;
      if (T.beta == -2 || !T.def || (int)T.s.size() > kMaxPoly)
        throw Error("the device back end handles standard sensors only (module type " + std::to_string(n.omt) +
                    " is not one); use the host back end (eout)", 7);
      auto si = sensor_index.find(n.omt);
      if (si == sensor_index.end()) {
        si = sensor_index.insert(std::make_pair(n.omt, (int)sensors.size())).first;
        BackSensor S{};
        S.mas = T.mas;
        S.ns = (int)T.s.size();
        for (int i = 0; i < S.ns; i++) S.s[i] = T.s[i];
        if (S.ns == 0) { S.ns = 1; S.s[0] = T.mas > 0 ? 0.f : 1.f; }
        sensors.push_back(S);
      }
      D.sensor = si->second;
    }
  }
  if (rat.empty()) rat.assign(PPCB_WNUM, 0.f);
  if (sensors.empty()) sensors.push_back(BackSensor{});
  std::vector<float2> wvs(PPCB_WNUM);
  for (int z = 0; z < PPCB_WNUM; z++) wvs[z] = make_float2(c.wvs[z].i, c.wvs[z].f);
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  auto T = std::make_shared<BackendTables>();
  check(cudaMalloc((void**)&T->doms, doms.size() * sizeof(BackDom)), "back end tables");
  check(cudaMalloc((void**)&T->sensors, sensors.size() * sizeof(BackSensor)), "back end tables");
  check(cudaMalloc((void**)&T->rat, rat.size() * sizeof(float)), "back end tables");
  check(cudaMalloc((void**)&T->wvs, wvs.size() * sizeof(float2)), "back end tables");
  check(cudaMemcpy(T->doms, doms.data(), doms.size() * sizeof(BackDom), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->sensors, sensors.data(), sensors.size() * sizeof(BackSensor), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->rat, rat.data(), rat.size() * sizeof(float), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->wvs, wvs.data(), wvs.size() * sizeof(float2), cudaMemcpyHostToDevice), "H2D");
  g.back = T;
}

void Engine::accept(int d, const ppcb_hit* dhits, uint64_t n, uint32_t seed, ppcb_acc_hit* dout,
                    unsigned long long* dcount, cudaStream_t st) {
  if (!inited_) throw Error("ini() must come before the back end", 6);
  accept_tables(d);
  DeviceCtx& g = devs.at(d);
  check(cudaSetDevice(g.dev), "cudaSetDevice");
  BackendTables& T = *g.back;
  if (n == 0) {
    check(cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), st), "memset");
    return;
  }
  const uint64_t nb = (n + kBlock - 1) / kBlock;
  if (nb > 0x7fffffffull) throw Error("back end: too many hits in one call", 7);
  if (nb > T.blocks_cap) {
    if (T.block_cnt) cudaFree(T.block_cnt);
    if (T.block_off) cudaFree(T.block_off);
    T.block_cnt = nullptr;
    T.block_off = nullptr;
    T.blocks_cap = 0;
    check(cudaMalloc((void**)&T.block_cnt, nb * sizeof(unsigned int)), "back end scratch");
    check(cudaMalloc((void**)&T.block_off, (nb + 1) * sizeof(unsigned long long)), "back end scratch");
    T.blocks_cap = nb;
  }
  BackArgs A;
  A.hits = dhits; A.n = n; A.doms = T.doms; A.sensors = T.sensors; A.rat = T.rat; A.wvs = T.wvs;
  A.rm = g.rm; A.nmul = (uint32_t)std::max(1, std::min(g.T, 1024)); A.seed = seed; A.gsize = cfg.p.gsize;
  k_accept_count<<<(unsigned int)nb, kBlock, 0, st>>>(A, T.block_cnt);
  check(cudaGetLastError(), "back end count");
  k_accept_scan<<<1, 1024, 0, st>>>(T.block_cnt, nb, T.block_off);
  check(cudaGetLastError(), "back end scan");
  k_accept_write<<<(unsigned int)nb, kBlock, 0, st>>>(A, T.block_off, dout);
  check(cudaGetLastError(), "back end write");
  check(cudaMemcpyAsync(dcount, T.block_off + nb, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st), "count");
}

}  // namespace ppcb
