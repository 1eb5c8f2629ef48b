// ppcb_propagate_noalloc: the propagation launch for callers that must not allocate
// device memory while they run.  Examples are host frameworks that reserve the GPU's
// memory for their own pool at start-up and forbid further driver allocations during
// event processing, and steady-state loops where a cudaMalloc/cudaFree would implicitly
// synchronise the device and stall the other streams.
//
// The scratch this launch needs -- the photon work counter, the hit counter, the launch
// sizes and the per-bunch photon offsets -- lives in one file-scope static device array
// below instead of memory the caller or the library allocates.  Inputs (the bunches) and
// outputs (the hit records and the hit count) are still the caller's.
#include <cuda_runtime.h>

#include <exception>
#include <string>

#include "../../include/ppc_b200.h"
#include "ctx.h"

namespace {

// Scratch layout, in 64-bit words: one control block (counters, 8 words), the launch
// sizes the kernel reads at start ({photons, bunches}, padded to 8 words), then the
// exclusive prefix sums of the bunch photon counts, PPCB_NOALLOC_MAX_BUNCHES + 1 entries.
// 128 B + 512 KiB in total, held by every GPU that loads the library until the process exits.
constexpr int kCtrlWords = 8;  // ppcb_ctrl (56 B) rounded up to 64 B
constexpr int kDynWords = 8;
static_assert(sizeof(ppcb_ctrl) <= kCtrlWords * sizeof(unsigned long long), "control block does not fit");
constexpr size_t kScratchWords = kCtrlWords + kDynWords + PPCB_NOALLOC_MAX_BUNCHES + 1;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kScratchWords];

// Exclusive prefix sum of bunch photon counts into the scratch (one block), and the launch
// sizes: the photons are clamped to the bunches' total, so a `num` above it produces no
// photon beyond the last bunch.
__global__ void k_bunch_offsets(const ppcb_bunch* __restrict__ b, int nb, unsigned long long num,
                                unsigned long long* bstart, unsigned long long* dyn) {
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
  if (t == nt - 1) {
    bstart[nb] = part[t];
    dyn[0] = num < part[t] ? num : part[t];
    dyn[1] = (unsigned long long)nb;
  }
}

// The caller's current device, put back on every return path.
struct DeviceRestore {
  int dev = -1;
  DeviceRestore() { if (cudaGetDevice(&dev) != cudaSuccess) { dev = -1; cudaGetLastError(); } }
  ~DeviceRestore() { if (dev >= 0) cudaSetDevice(dev); }
};

int fail(int code, const char* msg) {
  ppcb_internal_set_error(msg);
  return code;
}

int propagate_noalloc(ppcb_ctx* c, int device, const ppcb_bunch* bunches, int32_t nb, uint64_t num, ppcb_hit* hits,
                      uint64_t hcap, uint64_t* nhits, void* stream) {
  if (!c) return fail(PPCB_EARG, "null context");
  if (nb <= 0 || !bunches || !nhits || (hcap > 0 && !hits))
    return fail(PPCB_EARG, "ppcb_propagate_noalloc: bunches, a hit-count output and a hit buffer are required");
  if (nb > PPCB_NOALLOC_MAX_BUNCHES)
    return fail(PPCB_EARG, ("ppcb_propagate_noalloc: " + std::to_string(nb) + " bunches exceed the maximum of " +
                            std::to_string(PPCB_NOALLOC_MAX_BUNCHES) + " held in its static scratch").c_str());
  ppcb::Engine& e = c->s.eng;
  if (!e.ready()) return fail(PPCB_ESTATE, "ppcb_ini() must come before propagation");
  if (device < 0 || device >= (int)e.devs.size()) return fail(PPCB_EARG, "bad device index");
  const ppcb::DeviceCtx& g = e.devs[device];
  DeviceRestore restore;
  cudaError_t err = cudaSetDevice(g.dev);
  if (err != cudaSuccess) return fail(PPCB_ECUDA, cudaGetErrorString(err));
  // The array's device address, looked up with the device current: in host code the
  // symbol is only a host-side stand-in.  The lookup is a host-side table read that
  // allocates nothing; the first one on a device may load the library's device code.
  void* p = nullptr;
  err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (err != cudaSuccess || !p)
    return fail(PPCB_ECUDA, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err)).c_str());
  unsigned long long* scratch = static_cast<unsigned long long*>(p);
  ppcb_ctrl* ctrl = reinterpret_cast<ppcb_ctrl*>(scratch);
  unsigned long long* dyn = scratch + kCtrlWords;
  unsigned long long* bstart = scratch + kCtrlWords + kDynWords;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: the counters must start at zero
  err = cudaMemsetAsync(ctrl, 0, kCtrlWords * sizeof(unsigned long long), st);
  if (err == cudaSuccess) {
    k_bunch_offsets<<<1, 1024, 0, st>>>(bunches, nb, num, bstart, dyn);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess && num > 0) {
    ppcb::KArgs a = e.args_for(device);
    a.bunches = bunches; a.bstart = reinterpret_cast<const uint64_t*>(bstart); a.nb = nb; a.num = num;
    a.dyn = reinterpret_cast<const uint64_t*>(dyn);  // sizes as clamped on the device
    a.hits = hits; a.hcap = hcap; a.ctrl = ctrl;
    err = ppcb::launch_propagate(a, g.shape, st);
  }
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(nhits, &ctrl->hidx, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
  if (err != cudaSuccess) return fail(PPCB_ECUDA, cudaGetErrorString(err));
  return PPCB_OK;
}

}  // namespace

extern "C" int ppcb_propagate_noalloc(ppcb_ctx* c, int device, const ppcb_bunch* bunches, int32_t nb, uint64_t num,
                                      ppcb_hit* hits, uint64_t hcap, uint64_t* nhits, void* stream) {
  try {  // nothing may cross the C boundary as an exception (e.g. a failed string allocation)
    return propagate_noalloc(c, device, bunches, nb, num, hits, hcap, nhits, stream);
  } catch (const std::exception& x) {
    ppcb_internal_set_error(x.what());
    return PPCB_EARG;
  } catch (...) {
    ppcb_internal_set_error("ppcb_propagate_noalloc: unexpected exception");
    return PPCB_EARG;
  }
}
