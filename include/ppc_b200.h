/* C ABI of the B200 photon propagator (libppcb.so).
 *
 * Plain pointers and sizes only.  Every call returns 0 on success or a nonzero status
 * (PPCB_E*) with a message from ppcb_last_error(); where the reference calls exit(n)
 * (gpu/ini.cxx passim, gpu/ppc.cu:98, :266, :505, gpu/f2k.cxx:533) the status is n.
 *
 * The functions mirror the reference's library interface, the xppc:: namespace of
 * llh/ppc.h (defined in gpu/ppc.cu and gpu/f2k.cxx under -DXLIB); each cites the
 * reference entry point it replaces.  A context holds what the reference keeps in
 * globals (tables, device buffers, pending bunches, segment list, hit map), so several
 * contexts may coexist in one process; one context must not be used from two host
 * threads at once.  The record types are in ppc_b200/csrc/ppcb_types.h.
 */
#ifndef PPC_B200_H
#define PPC_B200_H
#include <stddef.h>
#include <stdint.h>

#include "../ppc_b200/csrc/ppcb_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PPCB_OK 0
#define PPCB_ECONFIG 1    /* bad or missing input file (reference: exit(1)) */
#define PPCB_ECUDA 2      /* CUDA runtime error (reference: exit(2)) */
#define PPCB_ESEGMENT 3   /* too many event segments (reference: exit(3)) */
#define PPCB_ESTATE 6     /* call out of order (e.g. propagation before ppcb_ini) */
#define PPCB_EARG 7       /* invalid argument */
#define PPCB_ENODEV 5     /* no usable GPU (reference: exit(5)) */

typedef struct ppcb_ctx ppcb_ctx;

/* One entry of the binned hit map (reference `hitz`, gpu/f2k.cxx:183-221), flattened:
 * key fields (track, module, pmt, direction bin, time bin) followed by the photon. */
typedef struct ppcb_hitz_rec {
  int32_t track_first;
  int32_t frame;
  uint64_t track_second;
  double t0;
  int32_t str, om, pmt;
  float dir, time;
  float r[4], n[4];
} ppcb_hitz_rec;

typedef struct ppcb_run_info {
  uint64_t photons;     /* photons propagated */
  uint64_t hits;        /* kernel-level hits produced */
  uint64_t kept;        /* hits stored (bounded by capacity) */
  uint64_t steps;       /* propagation steps (scattering segments) */
  uint32_t nan_steps;   /* steps with non-finite optical depth, photon dropped */
  uint32_t capped;      /* photons stopped by the step cap */
  double device_ms;     /* device time of the launches */
} ppcb_run_info;

typedef struct ppcb_info {
  uint64_t max_bunch_size;   /* getMaxBunchSize(), gpu/ppc.cu:368 */
  uint64_t workgroup_size;   /* getWorkgroupSize(), gpu/ppc.cu:370-386 */
  double total_device_ms;    /* getTotalDeviceTime(), gpu/ppc.cu:388-395 */
  uint64_t max_photons;      /* photons per launch (pmax) */
  uint64_t hit_capacity;     /* hits per launch and device */
  int32_t devices;
  int32_t threads;           /* threads (= random streams) per device */
  int32_t blocks;
  int32_t regs;              /* registers per thread of the propagation kernel */
  int32_t gsize, size, nstr, rsize;
  float eff;                 /* photons per metre after acceptance (ppm) */
  uint32_t ovr;              /* oversize area factor xR^2 */
  uint32_t seed;
  int32_t nextgen;
} ppcb_info;

const char* ppcb_last_error(void);

/* ---- lifecycle ---- */
int ppcb_create(ppcb_ctx** out);                                     /* start(), gpu/ppc.cu:481-483 */
int ppcb_destroy(ppcb_ctx* c);                                       /* stop(), gpu/ppc.cu:485-488 */
int ppcb_initialize(ppcb_ctx* c, const char* tables_dir, float enh); /* initialize(), gpu/ppc.cu:36; dir NULL: PPCTABLESDIR */
int ppcb_choose(ppcb_ctx* c, int device);                            /* choose(), gpu/ppc.cu:490-508 */
int ppcb_set_seed(ppcb_ctx* c, uint32_t seed);                       /* fixed seed instead of the clock (gpu/ini.cxx:792-795, DTMN) */
/* deterministic: 0 photons taken dynamically, one random stream per thread (fastest);
 * 1 photon i on thread i mod T with the thread streams, the reference's order; 2 photons taken
 * dynamically, each drawing from its own stream keyed by (seed, i), so two runs that differ
 * only in the ice share every photon's random numbers (common random numbers for finite
 * differences and fits).  Mode 2 has no counterpart in the reference. */
int ppcb_set_options(ppcb_ctx* c, int deterministic, uint32_t max_steps, int blocks_per_sm);
int ppcb_ini(ppcb_ctx* c);                                           /* ini(), gpu/ppc.cu:330-361 */
int ppcb_fin(ppcb_ctx* c);                                           /* fin(), gpu/ppc.cu:398-402 */
int ppcb_get_info(ppcb_ctx* c, ppcb_info* out);

/* ---- sources ---- */
int ppcb_flset(ppcb_ctx* c, int str, int om, ppcb_dom* out);         /* flset(), gpu/f2k.cxx:630-759 */
int ppcb_fldir(ppcb_ctx* c, float dir[3]);                           /* fldir(), gpu/f2k.cxx:762-765 */
int ppcb_flshift(ppcb_ctx* c, float m[3], float n[3], float* r);     /* flshift(), gpu/f2k.cxx:590-628; r may be NULL */
int ppcb_sett(ppcb_ctx* c, float nx, float ny, float nz, int32_t id_first, uint64_t id_second, int32_t frame,
              double t0);                                            /* sett(), gpu/f2k.cxx:548-552 */
int ppcb_addp(ppcb_ctx* c, float x, float y, float z, float t, float E, float dr, int32_t type,
              float scale);                                          /* addp(), gpu/f2k.cxx:484-504 */
int ppcb_addp_clst(ppcb_ctx* c, float x, float y, float z, float t, uint64_t n, float dr,
                   float beta);                                      /* addp_clst(), gpu/f2k.cxx:507-518 */
int ppcb_addp_mopo(ppcb_ctx* c, float x, float y, float z, float t, float light, float length, float beta,
                   float tau, float fr);                             /* addp_mopo(), gpu/f2k.cxx:520-528 */
int ppcb_flone(ppcb_ctx* c, uint64_t num);                           /* flone(), gpu/f2k.cxx:586-588 */
int ppcb_eout(ppcb_ctx* c);                                          /* eout(), gpu/f2k.cxx:536-541 */
int ppcb_efin(ppcb_ctx* c);                                          /* efin(), gpu/f2k.cxx:544-546 */
/* The host back end (print(), gpu/f2k.cxx:247-363) over kernel-level hits computed elsewhere,
 * e.g. by ppcb_propagate_device: hits of the segments started with sett (segment ids in .n)
 * go through acceptance, PMT choice and cable shadow into hitz.  Hits come in segment
 * order: hits of a segment before the newest one already seen are dropped with the
 * reference's "Internal Error" message.  No counterpart in the reference's API. */
int ppcb_back_end(ppcb_ctx* c, const ppcb_hit* hits, uint64_t n);
int ppcb_set_res(ppcb_ctx* c, float t, float cz);                    /* set_res(), gpu/f2k.cxx:202-210 */
float ppcb_xrnd(ppcb_ctx* c);                                        /* xrnd(), gpu/f2k.cxx:1-6 */

/* ---- results ---- */
int ppcb_hitz_count(ppcb_ctx* c, uint64_t* records);                 /* hitz, gpu/f2k.cxx:221 */
int ppcb_hitz_copy(ppcb_ctx* c, ppcb_hitz_rec* out, uint64_t cap, uint64_t* written);
int ppcb_keep_raw(ppcb_ctx* c, int keep);                            /* also keep kernel-level hits */
int ppcb_raw_count(ppcb_ctx* c, uint64_t* n);
int ppcb_raw_copy(ppcb_ctx* c, ppcb_hit* out, uint64_t cap, uint64_t* written);
int ppcb_last_run(ppcb_ctx* c, ppcb_run_info* last, ppcb_run_info* total);

/* ---- the hot path, called directly ----
 * ppcb_propagate: host buffers in and out (copies included).  Propagates the photons of
 * `nb` bunches (photon counts in .num, segment ids in .q), in launches of at most
 * max_photons, and writes kernel-level hits to `hits` (at most `cap`; *nhits receives
 * the number produced, which may be larger).  Replaces the reference's kernel()
 * (gpu/ppc.cu:432-469) with the front and back ends left out. */
int ppcb_propagate(ppcb_ctx* c, const ppcb_bunch* bunches, int32_t nb, ppcb_hit* hits, uint64_t cap,
                   uint64_t* nhits, ppcb_run_info* info);
/* ppcb_propagate_device: one asynchronous launch on device `device` (index into the
 * chosen devices) over caller-owned device memory, on `stream` (a cudaStream_t, NULL for
 * the default stream).  bstart[k] is the first photon index of bunch k, bstart[nb] = num.
 * `ctrl` must be zeroed before the launch; afterwards ctrl->hidx is the number of hits
 * produced (only the first hcap are stored).  Replaces the main propagate launch,
 * gpu/ppc.cu:293-306. */
int ppcb_propagate_device(ppcb_ctx* c, int device, const ppcb_bunch* bunches, const uint64_t* bstart, int32_t nb,
                          uint64_t num, ppcb_hit* hits, uint64_t hcap, ppcb_ctrl* ctrl, void* stream);
/* Random stream state per thread (the reference keeps it in datz.rs, gpu/pro.cu:891-892):
 * read or restore it, e.g. to checkpoint and resume a run.  n = threads of the device. */
int ppcb_rng_get(ppcb_ctx* c, int device, uint64_t* rs, uint64_t n);
int ppcb_rng_set(ppcb_ctx* c, int device, const uint64_t* rs, uint64_t n);
int ppcb_rng_reset(ppcb_ctx* c);                                     /* rs_ini(), gpu/ini.cxx:556-571 */

/* ---- inspection (tests, tools) ---- */
/* Host copy of a named table (params, az, lr, ls, is, mcol, sc, lp, absca, wmeta, oms, rm,
 * wvs, eff): pointer valid until the next ppcb_initialize / ppcb_destroy. */
int ppcb_table(ppcb_ctx* c, const char* name, const void** ptr, uint64_t* bytes);
/* Phase-1 sampling only: thread t samples photon t (t < num) with its own stream;
 * out[3t..3t+2] = position, direction, (wavelength bin, segment, fla, ofla) as int bits. */
int ppcb_generate_device(ppcb_ctx* c, int device, const ppcb_bunch* bunches, const uint64_t* bstart, int32_t nb,
                         uint64_t num, void* out, void* stream);
/* Index helpers at points: pos[2k] = (x,y,z,t), pos[2k+1] = (nx,ny,nz,length).
 * out_i[8k..] = layer, cell x lo/hi, cell y lo/hi, DOM window lo/hi, string; out_f[2k..] =
 * tilt shift, layer thickness (gpu/pro.cu:168-264, :507-515, :580-594, :623-626). */
int ppcb_index_probe_device(ppcb_ctx* c, int device, const void* pos, int32_t n, int32_t* out_i, float* out_f,
                            void* stream);
/* The kernel's string-proximity pre-test of the DOM search, on the host (same code): for
 * segments pos[2k] = (x,y,z,t), pos[2k+1] = (nx,ny,nz,length), out[k] = 1 when the
 * segment may reach a string's cylinder (the reference's search, gpu/pro.cu:577-672, then
 * runs), 0 when that search would find nothing.  Needs ppcb_initialize only. */
int ppcb_string_grid_probe(ppcb_ctx* c, const void* pos, int32_t n, int32_t* out);

/* ---- batched events ----
 * No counterpart in the reference, which propagates one source per eout()
 * (gpu/f2k.cxx:536-541).  Thousands of events with uneven photon counts run in one
 * persistent, work-stealing launch, replayed from a CUDA graph; each event's hits go to
 * its own region of the hit buffer, sized as photons x hits_per_photon + 64 slots (an
 * upper bound: hits beyond it are counted in `overflowed`, not stored).  Bunch .q is the
 * event index in [0, events).  The buffers are sized once at creation. */
typedef struct ppcb_batch ppcb_batch;
typedef struct ppcb_batch_info {
  uint64_t photons, steps;
  uint64_t hits;        /* produced */
  uint64_t kept;        /* stored */
  uint32_t overflowed;  /* events whose region was too small */
  uint32_t pad_;
  double device_ms;     /* the propagation kernel */
  double graph_ms;      /* uploads, kernel, compaction and downloads */
} ppcb_batch_info;
typedef struct ppcb_tune_info {
  int32_t threads, blocks_per_sm, refill_below, pad_;
  double photons_per_s;
} ppcb_tune_info;
int ppcb_batch_create(ppcb_ctx* c, int device, uint32_t max_events, uint32_t max_bunches, uint64_t hit_capacity,
                      ppcb_batch** out);
/* every ppcb_batch is destroyed before the ppcb_ctx it was created with */
int ppcb_batch_destroy(ppcb_batch* b);
int ppcb_batch_set_graph(ppcb_batch* b, int use_graph);
int ppcb_batch_run(ppcb_batch* b, const ppcb_bunch* bunches, int32_t nb, uint32_t events, double hits_per_photon,
                   ppcb_batch_info* info);
/* per event of the last run: hits produced, and offsets (events+1) into the kept hits */
int ppcb_batch_counts(ppcb_batch* b, uint32_t* produced, uint64_t* offsets);
int ppcb_batch_hits(ppcb_batch* b, ppcb_hit* out, uint64_t cap, uint64_t* n);
/* Times the kernel's launch shapes (threads per block, blocks per SM, photon-pool refill
 * threshold) on a scaled-down copy of the batch and keeps the fastest for this context. */
int ppcb_batch_autotune(ppcb_batch* b, const ppcb_bunch* bunches, int32_t nb, uint32_t events, uint64_t sample_photons,
                        ppcb_tune_info* out);

/* ---- ice-model gradient ----
 * No counterpart in the reference (llh/DirectFit fits the ice by repeated forward runs,
 * llh/llh.cxx:1435-1634).  ppcb_set_ice replaces the per-layer scattering (be) and
 * absorption (ba) coefficients at 400 nm (icemodel.dat columns 2-3, file order, `size`
 * values each; NULL keeps) and rebuilds the wavelength table.  ppcb_gradient propagates
 * the bunches once while recording each hit's provenance, then replays only the detected
 * photons to form d/d be_j and d/d ba_j (FP64, file order) of
 *   LL = sum_d (k_d log mu_d - mu_d)   with `observed` k_d (DOMs with mu_d = 0 left out), or
 *   sum_d w_d mu_d                     with `weights` w_d when observed is NULL,
 * where mu_d = scale x (simulated hits in charge bin d).  The charge bins are the DOMs
 * (events = 0; observed/weights/counts hold gsize values) or, with events > 0, the
 * (event, DOM) pairs, the event being the hit's segment id (the bunch's q): bin =
 * event x gsize + DOM, events x gsize values, hits of segments >= events left out.
 * Absorption terms are pathwise
 * (-nr L_j dabs/dba), scattering terms score-function ((n_j/sca_j - L_j) dsca/dbe). */
typedef struct ppcb_grad_info {
  double ll;
  uint64_t photons, hits, replayed, unmatched, steps;
  double forward_ms, backward_ms;
} ppcb_grad_info;
int ppcb_set_ice(ppcb_ctx* c, const float* be, const float* ba);
int ppcb_get_ice(ppcb_ctx* c, float* be, float* ba, int32_t* size);
int ppcb_gradient(ppcb_ctx* c, const ppcb_bunch* bunches, int32_t nb, uint32_t events, const float* observed,
                  const float* weights, double scale, uint64_t hit_cap, uint32_t* counts, double* g_be, double* g_ba,
                  ppcb_grad_info* info);
/* One ice-fit iteration as a CUDA graph: the bunches and observed charges are fixed at
 * creation; each ppcb_gradgraph_run sets new be/ba (NULL keeps), uploads the rebuilt table
 * and replays the recording pass, histogram, Poisson weights and log-likelihood, and the
 * replay of the detected photons, with the hit count kept on the device between them.
 * Same results as ppcb_gradient with `observed` (the log-likelihood summed in another
 * order).  Destroy it before its context. */
typedef struct ppcb_gradgraph ppcb_gradgraph;
int ppcb_gradgraph_create(ppcb_ctx* c, const ppcb_bunch* bunches, int32_t nb, uint32_t events, const float* observed,
                          double scale, uint64_t hit_cap, ppcb_gradgraph** out);
int ppcb_gradgraph_run(ppcb_gradgraph* g, const float* be, const float* ba, uint32_t* counts, double* g_be,
                       double* g_ba, ppcb_grad_info* info);
int ppcb_gradgraph_destroy(ppcb_gradgraph* g);

/* ---- propagation that allocates nothing ----
 * No counterpart in the reference.  For callers that may not allocate device memory while
 * they run: frameworks that reserve the GPU's memory for their own pool at start-up, and
 * steady-state loops where a cudaMalloc/cudaFree would synchronise the device.  Same
 * launch as ppcb_propagate_device, but its scratch (photon work counter, hit counter,
 * launch sizes and per-bunch photon offsets) is a static device array of fixed size inside
 * the library: at most PPCB_NOALLOC_MAX_BUNCHES bunches per call (larger lists are rejected
 * with PPCB_EARG).  The caller passes the bunches (device memory), the hit buffer and
 * `nhits`, a device pointer that receives the number of hits produced; when that number
 * exceeds hcap only the first hcap records are stored.  `num` is the sum of
 * bunches[k].num: a smaller value propagates the first `num` photons, a larger one is
 * clamped to the sum on the device.  The call allocates nothing; the context's tables come
 * from an earlier ppcb_ini.  The caller's current device is left as it was.
 * Each call looks up the array's device address with the device current (a host-side
 * lookup, no allocation); the first call on a device may also load the library's device
 * code (the runtime's module loading, not an allocation by this library).  All calls on a
 * device share the one
 * array and it keeps the last call's contents (each call clears its counters first): calls
 * whose work overlaps on the GPU race, so order them (one stream, or events). */
#define PPCB_NOALLOC_MAX_BUNCHES 65536
int ppcb_propagate_noalloc(ppcb_ctx* c, int device, const ppcb_bunch* bunches, int32_t nb, uint64_t num,
                           ppcb_hit* hits, uint64_t hcap, uint64_t* nhits, void* stream);

/* ---- hit back end on the device ----
 * The reference's back end runs on the host inside eout() (gpu/f2k.cxx:247-363); these
 * apply the same acceptance to kernel-level hits on the GPU: the wavelength x RDE
 * acceptance of the DOM's (module type, variant), the sensor's PMT choice (getPMT: standard
 * DOMs, multi-PMT modules, wavelength-shifting tubes with their transit delay added to the
 * time), the cable shadow, and a wavelength sampled in the hit's bin.  Each hit draws from its own random stream keyed by (seed, hit index)
 * instead of the host's shared sequence: the same decisions in distribution, not hit by
 * hit.  Accepted hits are written in input order.
 * ppcb_accept_device: device pointers on `stream`; *count (a device pointer) receives the
 * number accepted; `out` must hold n records.  ppcb_accept: host buffers, device 0; at most
 * `cap` records written, *nout receives the number accepted. */
int ppcb_accept_device(ppcb_ctx* c, int device, const ppcb_hit* hits, uint64_t n, uint32_t seed, ppcb_acc_hit* out,
                       unsigned long long* count, void* stream);
int ppcb_accept(ppcb_ctx* c, const ppcb_hit* hits, uint64_t n, uint32_t seed, ppcb_acc_hit* out, uint64_t cap,
                uint64_t* nout);

/* ---- source front end on the device ----
 * The library's sources (addp with particle types, addp_clst, addp_mopo; f2k "ph" records)
 * become photon bunches on the GPU, as the host front end makes them (gpu/f2k.cxx:17-167,
 * 377-528):
 *   - light yield per particle type: muon segments, EM cascades, hadronic cascades with
 *     their charge fluctuation;
 *   - times the efficiency, over the DOM oversize factor;
 *   - a Poisson-sampled photon count (exact counts for clst and "ph").
 * A source makes one bunch, or several of at most 2^31 photons each.  Each source draws
 * from its own random stream keyed by (seed, source index), so the counts match the host
 * front end in distribution, not source for source.  The bunches feed
 * ppcb_propagate_device directly: bstart[k] is the first photon of bunch k and bstart[nb]
 * the total. */
/* src: device pointer, ns sources; out: room for cap bunches; bstart: cap + 1 entries;
 * counts (device, 2 x uint64): bunches needed and photons.  When counts[0] > cap only the
 * first cap bunches are written (call again with more room).  Asynchronous on `stream`. */
int ppcb_sources_device(ppcb_ctx* c, int device, const ppcb_source* src, uint64_t ns, uint32_t seed,
                        ppcb_bunch* out, uint64_t* bstart, uint64_t cap, uint64_t* counts, void* stream);
/* host buffers, device 0; *nb and *num receive the bunches needed and the photons */
int ppcb_sources(ppcb_ctx* c, const ppcb_source* src, uint64_t ns, uint32_t seed, ppcb_bunch* out, uint64_t* bstart,
                 uint64_t cap, uint64_t* nb, uint64_t* num);
/* f2k text (TR records, one segment per line, gpu/f2k.cxx:555-583) to sources; the first
 * line is segment first_segment.  *n receives the number of sources, at most cap written;
 * *lines the number of lines (segments) read. */
int ppcb_f2k_sources(const char* text, uint64_t len, uint32_t first_segment, ppcb_source* out, uint64_t cap,
                     uint64_t* n, uint64_t* lines);

/* ---- DirectFit likelihood on the device ----
 * The saturated Poisson likelihood with model error that DirectFit fits with
 * (llh/llh.cxx:419-662, 1075-1082), with the simulation side on the GPU.  ppcb_llh_create
 * prepares the observed side once per event on the host, as dat::prep/optimize do:
 *   - observed hits binned per DOM in 200 bins of lbin ns from the earliest hit;
 *   - DOMs selected by total charge (qmin < q/drep < qsat) and flasher distance;
 *   - each DOM's bins outside its window around the peak (500 ns before, 1000 ns after)
 *     dropped;
 *   - the remaining bins merged into blocks by the Bayesian-blocks partition of the
 *     observed charge.
 * ppcb_llh_eval_device then takes kernel-level hits and, in one pass over them, applies the
 * back end's acceptance (the same per-hit streams as ppcb_accept with the same seed).  It
 * bins the accepted hits of every DOM into its blocks for each of ndt time shifts and sums
 * llf(simulated, observed, nsim, drep) over all blocks:
 *   out[j] = (llf(nohit, 0, nsim, drep) [unless norm] + sum_DOM sum_block llf(...)) / ndof,
 * as fllh(dts[j], nsim) does.  Hit times are on the observed hits' clock; a shift dt moves
 * every simulated hit by +dt.  Simulated hits count 1 each (DirectFit without SPE charge
 * sampling).  As in the reference, with norm a DOM that enters with all of its observed
 * charge outside the 200 bins (dtot = 0) makes the result NaN.
 * A good-DOM list (DirectFit's `set` file) enters as bad DOMs: those with observed pulses
 * that are not on it, which is what llh/llh.cxx:785-792 does with it; `unh` stays the
 * caller's choice, as the list does not set it there.
 * Not supported: multi-PMT keys, the charge-unfolding variants. */
typedef struct ppcb_llh ppcb_llh;
typedef struct ppcb_llh_hit {        /* one observed pulse: the columns of DirectFit's dat file */
  int32_t str, om;
  double t, q;
} ppcb_llh_hit;
typedef struct ppcb_llh_window {     /* pulses of (str, om) with ti <= t < tf are ignored (ert) */
  int32_t str, om;
  double ti, tf;
} ppcb_llh_window;
typedef struct ppcb_llh_opts {
  double lbin;    /* time bin [ns]; <= 0: max(25, (tmax - tmin + 1) / 200) (llh/llh.cxx:799) */
  double sig;     /* model error of the saturated likelihood (LSSL::SIG, 0.10); 0: plain Poisson */
  double qmin;    /* a DOM enters when qmin * drep < its charge < qsat * drep (0.1, 500) */
  double qsat;
  double drep;    /* repetitions of the observed data (1) */
  int32_t peak;   /* window from the monotone-blocks fit instead of the highest bin (0) */
  int32_t mono;   /* blocks rise to the peak and fall after it (0) */
  int32_t norm;   /* normalise each DOM's simulation to its observed charge (0) */
  int32_t unh;    /* count simulated hits on DOMs without data ("no-hit" term); DirectFit sets
                     it when it reads a bad-DOM list (0) */
  int32_t flasher, fla_str, fla_om, fsep; /* flasher run: leave out DOMs within fsep of it */
} ppcb_llh_opts;
typedef struct ppcb_llh_info {
  double lbin, t0;  /* bin width and the time of bin 0 (earliest observed pulse) */
  int32_t ndof;     /* 1 + blocks of the DOMs that enter */
  int32_t doms;     /* DOMs that enter */
  int32_t blocks;
  int32_t errors;   /* llf evaluations whose Newton iteration left the domain (the reference
                       stops there; here the term is NaN), summed since creation */
} ppcb_llh_info;
typedef struct ppcb_llh_block {      /* one block of one DOM: bins [first, last] and its charge */
  int32_t str, om, first, last;
  double dat;
} ppcb_llh_block;
#define PPCB_LLH_MAX_SHIFTS 64
/* DirectFit's defaults (llh/llh.cxx:27-55, lssl.cxx:4) */
int ppcb_llh_default_opts(ppcb_llh_opts* o);
/* observed pulses (host), excluded windows and bad DOMs (str, om pairs; both may be null);
 * device: the device of the ppcb_ctx whose acceptance and hits are used */
int ppcb_llh_create(ppcb_ctx* c, int device, const ppcb_llh_hit* data, uint64_t n, const ppcb_llh_window* windows,
                    uint64_t nwin, const int32_t* bad, uint64_t nbad, const ppcb_llh_opts* opts, ppcb_llh** out);
/* every ppcb_llh is destroyed before the ppcb_ctx it was created with */
int ppcb_llh_destroy(ppcb_llh* l);
int ppcb_llh_get_info(ppcb_llh* l, ppcb_llh_info* info);
/* blocks in DOM order, each DOM's from its last bin backwards (the order llh() sums them) */
int ppcb_llh_blocks(ppcb_llh* l, ppcb_llh_block* out, uint64_t cap, uint64_t* n);
/* hits: kernel-level hits in device memory; dts (host, ndt <= PPCB_LLH_MAX_SHIFTS); out: ndt
 * doubles in device memory, written on `stream` */
int ppcb_llh_eval_device(ppcb_llh* l, const ppcb_hit* hits, uint64_t n, uint32_t seed, const double* dts, int32_t ndt,
                         double nsim, double* out, void* stream);
/* the same with host buffers (copies included); fails with status 1 when an llf evaluation
 * left its domain, as the reference exits */
int ppcb_llh_eval(ppcb_llh* l, const ppcb_hit* hits, uint64_t n, uint32_t seed, const double* dts, int32_t ndt,
                  double nsim, double* out);

/* ---- measurement ----
 * No counterpart in the reference.  FP32 FMA throughput of `device` (TFLOP/s, best of
 * `repeats` launches of an FFMA loop over every SM): the FP32 side of the propagation
 * kernel's FP32/SFU issue roofline. */
int ppcb_fp32_peak(int device, int repeats, double* tflops, double* ms);
/* special-function-unit throughput (reciprocal square roots) of `device` in tera-operations
 * per second, measured the same way: the SFU side of the kernel's FP32/SFU issue roofline.
 * No counterpart in the reference. */
int ppcb_sfu_peak(int device, int repeats, double* tops, double* ms);

#ifdef __cplusplus
}
#endif
#endif
