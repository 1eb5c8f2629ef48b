// Hit back end on the device (Engine::accept): the acceptance of gpu/f2k.cxx:247-363 applied
// to kernel-level hits on the GPU.  For every hit, in the reference's order of decisions:
//   1. wavelength x RDE acceptance: a DOM with high voltage and an acceptance table for its
//      (module type, variant) keeps the hit with probability rat[z] x rde / rmax;
//   2. the sensor's PMT choice (getPMT, gpu/ini.cxx:210-280): for a standard DOM a
//      polynomial in the cosine between the photon direction and the sensor axis against
//      mas x u, or the impact point's height along the axis against a threshold; for a
//      multi-PMT module one PMT by its angular response; for a wavelength-shifting tube the
//      readout end and its transit delay (backend.cuh);
//   3. cable shadow (gpu/f2k.cxx:314-335);
//   4. wavelength sampled uniformly in the hit's wavelength bin.
// The reference draws the three uniform numbers from one host stream in hit order; here
// every hit has its own stream keyed by (seed, hit index), so the decisions are the same in
// distribution, not hit by hit.  Output is in input order (a block-level scan of the
// accept flags), so a call is deterministic for a given seed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "backend.cuh"
#include "engine.h"

namespace ppcb {

namespace {

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

// The block's accepted records are compacted in shared memory, then copied out as one
// contiguous run with coalesced 4-byte stores (a record is 14 words; the caller's buffer
// needs only the record's own 4-byte alignment).
__global__ void __launch_bounds__(kBlock) k_accept_write(BackArgs A, const unsigned long long* off,
                                                         ppcb_acc_hit* out) {
  static_assert(sizeof(ppcb_acc_hit) == 56, "record of 14 words of 4 bytes");
  constexpr int kWords = 14;
  __shared__ unsigned int warp_cnt[kBlock / 32];
  __shared__ uint32_t stage[kBlock * kWords];
  const uint64_t k = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
  ppcb_acc_hit o;
  const bool f = k < A.n && accept_one(A, k, o);
  const unsigned int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned int bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) warp_cnt[w] = __popc(bal);
  __syncthreads();
  unsigned int before = 0, total = 0;
  for (unsigned int j = 0; j < kBlock / 32; j++) {
    if (j < w) before += warp_cnt[j];
    total += warp_cnt[j];
  }
  if (f) {
    const unsigned int pos = before + __popc(bal & ((1u << lane) - 1u));
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&o);
    for (int q = 0; q < kWords; q++) stage[pos * kWords + q] = src[q];
  }
  __syncthreads();
  uint32_t* dst = reinterpret_cast<uint32_t*>(out + off[blockIdx.x]);
  for (unsigned int q = threadIdx.x; q < total * kWords; q += kBlock) dst[q] = stage[q];
}

}  // namespace


BackArgs back_args(Engine& e, int d, const ppcb_hit* dhits, uint64_t n, uint32_t seed) {
  BackendTables& T = e.backend_tables(d);
  const DeviceCtx& g = e.devs.at(d);
  BackArgs A;
  A.hits = dhits; A.n = n; A.doms = T.doms; A.sensors = T.sensors; A.rat = T.rat; A.wvs = T.wvs; A.dirs = T.dirs;
  A.rm = g.rm; A.nmul = (uint32_t)std::max(1, std::min(g.T, 1024)); A.seed = seed; A.gsize = e.cfg.p.gsize;
  return A;
}

BackendTables& Engine::backend_tables(int d) {
  DeviceCtx& g = devs.at(d);
  if (g.back) return *g.back;
  const Config& c = cfg;
  std::vector<BackDom> doms(c.p.gsize);
  std::vector<BackSensor> sensors;
  std::vector<float3> pmt_dirs;
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
      auto si = sensor_index.find(n.omt);
      if (si == sensor_index.end()) {
        si = sensor_index.insert(std::make_pair(n.omt, (int)sensors.size())).first;
        BackSensor S{};
        S.beta = T.beta;
        S.fx = T.fx;
        S.Rr = T.Rr;
        S.Rz = T.Rz;
        S.cable = T.cable;
        if (T.beta == -2) {  // the getPMT branches in the reference's order (gpu/ini.cxx:210-280)
          S.kind = kSensorTube;
        } else if (T.def) {
          if ((int)T.s.size() > kMaxPoly)
            throw Error("the device back end takes angular polynomials of at most 16 coefficients", 7);
          S.kind = kSensorStandard;
          S.mas = T.mas;
          S.ns = (int)T.s.size();
          for (int i = 0; i < S.ns; i++) S.s[i] = T.s[i];
          if (S.ns == 0) { S.ns = 1; S.s[0] = T.mas > 0 ? 0.f : 1.f; }
        } else {
          S.kind = kSensorMultiPMT;
          S.dir0 = (int)pmt_dirs.size();
          S.ndir = (int)T.dirs.size();
          for (const Vec3& v : T.dirs) pmt_dirs.push_back(make_float3(v[0], v[1], v[2]));
        }
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
  if (pmt_dirs.empty()) pmt_dirs.push_back(make_float3(0, 0, 1));
  check(cudaMalloc((void**)&T->dirs, pmt_dirs.size() * sizeof(float3)), "back end tables");
  check(cudaMemcpy(T->dirs, pmt_dirs.data(), pmt_dirs.size() * sizeof(float3), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->doms, doms.data(), doms.size() * sizeof(BackDom), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->sensors, sensors.data(), sensors.size() * sizeof(BackSensor), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->rat, rat.data(), rat.size() * sizeof(float), cudaMemcpyHostToDevice), "H2D");
  check(cudaMemcpy(T->wvs, wvs.data(), wvs.size() * sizeof(float2), cudaMemcpyHostToDevice), "H2D");
  g.back = T;
  return *g.back;
}

void Engine::accept(int d, const ppcb_hit* dhits, uint64_t n, uint32_t seed, ppcb_acc_hit* dout,
                    unsigned long long* dcount, cudaStream_t st) {
  if (!inited_) throw Error("ini() must come before the back end", 6);
  BackendTables& T = backend_tables(d);
  DeviceCtx& g = devs.at(d);
  check(cudaSetDevice(g.dev), "cudaSetDevice");
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
  const BackArgs A = back_args(*this, d, dhits, n, seed);
  k_accept_count<<<(unsigned int)nb, kBlock, 0, st>>>(A, T.block_cnt);
  check(cudaGetLastError(), "back end count");
  k_accept_scan<<<1, 1024, 0, st>>>(T.block_cnt, nb, T.block_off);
  check(cudaGetLastError(), "back end scan");
  k_accept_write<<<(unsigned int)nb, kBlock, 0, st>>>(A, T.block_off, dout);
  check(cudaGetLastError(), "back end write");
  check(cudaMemcpyAsync(dcount, T.block_off + nb, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st), "count");
}

}  // namespace ppcb
