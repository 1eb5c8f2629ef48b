// ppcb_propagate_noalloc: the propagation launch for callers that must not allocate
// device memory while they run.  Examples are host frameworks that reserve the GPU's
// memory for their own pool at start-up and forbid further driver allocations during
// event processing, and steady-state loops where a cudaMalloc/cudaFree would implicitly
// synchronise the device and stall the other streams.
//
// The scratch this launch needs -- the photon work counter, the hit counter and the
// per-bunch photon offsets -- lives in one file-scope static device array below instead
// of memory the caller or the library allocates.  Inputs (the bunches) and outputs (the
// hit records and the hit count) are still the caller's.
#include <cuda_runtime.h>

#include <string>

#include "../../include/ppc_b200.h"
#include "ctx.h"

namespace {

// Scratch layout: one control block (counters), then the exclusive prefix sums of the
// bunch photon counts, PPCB_NOALLOC_MAX_BUNCHES + 1 entries.  64 B + 512 KiB in total,
// held by every GPU that loads the library until the process exits.
constexpr int kCtrlWords = 8;  // ppcb_ctrl (56 B) rounded up to 64 B
static_assert(sizeof(ppcb_ctrl) <= kCtrlWords * sizeof(unsigned long long), "control block does not fit");
constexpr size_t kScratchWords = kCtrlWords + PPCB_NOALLOC_MAX_BUNCHES + 1;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchWords];

// Device address of g_noalloc_scratch per device ordinal.  In host code the symbol is
// only a host-side stand-in, never a device address, so it is looked up once per device
// with that device current.
constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices] = {nullptr};

// Exclusive prefix sum of bunch photon counts into the scratch (one block).
__global__ void k_bunch_offsets(const ppcb_bunch* __restrict__ b, int nb, unsigned long long* bstart) {
  __shared__ unsigned long long part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (nb + nt - 1) / nt;
  const int lo = t * per, hi = min(nb, lo + per);
  unsigned long long s = 0;
  for (int k = lo; k < hi; k++) s += b[k].num;
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < nt; off <<= 1) {  // inclusive scan of the per-thread sums
    unsigned long long v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  unsigned long long acc = part[t] - s;
  for (int k = lo; k < hi; k++) {
    bstart[k] = acc;
    acc += b[k].num;
  }
  if (t == nt - 1) bstart[nb] = part[t];
}

}  // namespace

extern "C" int ppcb_propagate_noalloc(ppcb_ctx* c, int device, const ppcb_bunch* bunches, int32_t nb, uint64_t num,
                                      ppcb_hit* hits, uint64_t hcap, uint64_t* nhits, void* stream) {
  if (!c) { ppcb_internal_set_error("null context"); return PPCB_EARG; }
  if (nb <= 0 || !bunches || !nhits || (hcap > 0 && !hits)) {
    ppcb_internal_set_error("ppcb_propagate_noalloc: bunches, a hit-count output and a hit buffer are required");
    return PPCB_EARG;
  }
  if (nb > PPCB_NOALLOC_MAX_BUNCHES) {
    ppcb_internal_set_error("ppcb_propagate_noalloc: " + std::to_string(nb) + " bunches exceed the maximum of " +
                            std::to_string(PPCB_NOALLOC_MAX_BUNCHES) + " held in its static scratch");
    return PPCB_EARG;
  }
  ppcb::Engine& e = c->s.eng;
  if (!e.ready()) { ppcb_internal_set_error("ppcb_ini() must come before propagation"); return PPCB_ESTATE; }
  if (device < 0 || device >= (int)e.devs.size()) { ppcb_internal_set_error("bad device index"); return PPCB_EARG; }
  const ppcb::DeviceCtx& g = e.devs[device];
  if (g.dev < 0 || g.dev >= kMaxDevices) { ppcb_internal_set_error("device ordinal out of range"); return PPCB_EARG; }
  cudaError_t err = cudaSetDevice(g.dev);
  if (err != cudaSuccess) { ppcb_internal_set_error(cudaGetErrorString(err)); return PPCB_ECUDA; }
  if (!g_scratch_addr[g.dev]) {  // set-up, once per device, with that device current
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess || !p) {
      ppcb_internal_set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
      return PPCB_ECUDA;
    }
    g_scratch_addr[g.dev] = p;
  }
  unsigned long long* scratch = (unsigned long long*)g_scratch_addr[g.dev];
  ppcb_ctrl* ctrl = (ppcb_ctrl*)scratch;
  unsigned long long* bstart = scratch + kCtrlWords;
  cudaStream_t st = (cudaStream_t)stream;
  // the array keeps the previous call's contents: the counters must start at zero
  err = cudaMemsetAsync(ctrl, 0, kCtrlWords * sizeof(unsigned long long), st);
  if (err == cudaSuccess) {
    k_bunch_offsets<<<1, 1024, 0, st>>>(bunches, nb, bstart);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess && num > 0) {
    ppcb::KArgs a = e.args_for(device);
    a.bunches = bunches; a.bstart = (const uint64_t*)bstart; a.nb = nb; a.num = num;
    a.hits = hits; a.hcap = hcap; a.ctrl = ctrl;
    err = ppcb::launch_propagate(a, g.shape, st);
  }
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(nhits, &ctrl->hidx, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
  if (err != cudaSuccess) { ppcb_internal_set_error(cudaGetErrorString(err)); return PPCB_ECUDA; }
  return PPCB_OK;
}
