/* TEST INFRASTRUCTURE ONLY -- the oracle.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product never links or calls it.
 *
 * A plain-C restatement of the reference's photon propagation (gpu/pro.cu), fed with
 * the same table image the product builds (ppc_b200/csrc/ppcb_types.h).  Parity is
 * pinned against the reference itself: tests/test_oracle_pin.py runs the reference's
 * own CPU build (oracle/_ref/ref_harness, built from the reference sources by
 * oracle/Makefile) and the committed golden vectors in tests/golden/.
 */
#ifndef PPC_ORACLE_H
#define PPC_ORACLE_H
#include <stdint.h>

#include "../ppc_b200/csrc/ppcb_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ppco_tables {
  const ppcb_params* p;
  const ppcb_aniz* az;      /* [size] */
  const float* lr;          /* [LMAX] */
  const uint16_t* ls;       /* [NSTR] */
  const uint16_t* is;       /* [CX*CY] */
  const int8_t* mcol;       /* [CTX*CTY] */
  const ppcb_line* sc;      /* [NSTR] */
  const float* lp;          /* [LMAX*LYRS*2] */
  const float* absca;       /* [WNUM*size*2] */
  const ppcb_wmeta* wmeta;  /* [WNUM] */
  const ppcb_dom* oms;      /* [gsize] */
} ppco_tables;

/* MWC stream: x,y state words, a multiplier (gpu/pro.cu:47-57) */
typedef struct ppco_rng { uint32_t x, y, a; } ppco_rng;

/* Events counted by ppco_propagate since the last ppco_counts_reset. */
typedef struct ppco_counts {
  uint64_t photons, steps, sca_draws, crossings;
  uint64_t strings_tested, strings_passed, doms_tested, hits, truncated;
  uint64_t bfr, bfr_curved, bfr_layers, scatter_hg, scatter_sam;
} ppco_counts;
void ppco_counts_reset(void);
void ppco_counts_get(ppco_counts* out);
/* step trace: each step's DOM-search segment (r.xyzw, n.xyz, sca), at most cap steps */
void ppco_trace_steps(float* buf, uint64_t cap);
uint64_t ppco_trace_count(void);

/* phase-1 photon record (gpu/ini.cxx:391-397) */
typedef struct ppco_pbuf {
  float r[4], n[4];
  uint32_t q, i;
  int32_t fla, ofla;
} ppco_pbuf;

float ppco_xrnd(ppco_rng* s);
float ppco_zshift(const ppco_tables* t, const float r[4], float* dz);

/* Source sampling of one photon from bunch b (gpu/pro.cu:335-476). */
void ppco_generate(const ppco_tables* t, const ppcb_bunch* b, ppco_rng* s, ppco_pbuf* out);

/* Propagates one photon from its phase-1 record until absorbed (gpu/pro.cu:486-889).
 * Hits go to hits[*nh] while *nh < cap; *nh counts every hit.  Returns the steps. */
uint64_t ppco_propagate(const ppco_tables* t, const ppco_pbuf* f, ppco_rng* s, ppcb_hit* hits,
                        uint64_t* nh, uint64_t cap);

/* Reference CPU-build sequencing (gpu/ppc.cu:439-440 with XCPU): nthr pseudo-threads
 * share one stream; each runs phase 1 for photons t, t+nthr, ... then phase 2 for them.
 * pbuf_out (optional) receives the phase-1 records by photon index. */
uint64_t ppco_run_reference_order(const ppco_tables* t, const ppcb_bunch* b, int nb, uint32_t num,
                                  uint32_t nthr, ppco_rng* stream, ppcb_hit* hits, uint64_t cap,
                                  ppco_pbuf* pbuf_out);

/* Per-thread fused sequencing (the CUDA kernel's deterministic mode): thread t owns
 * stream (rs[t], rm[t]) and handles photons t, t+nthr, ... each generated then propagated. */
uint64_t ppco_run_fused(const ppco_tables* t, const ppcb_bunch* b, int nb, uint64_t num, uint32_t nthr,
                        uint64_t* rs, const uint32_t* rm, ppcb_hit* hits, uint64_t cap, uint64_t* steps);

/* Index helpers at points (the product's ppcb_index_probe_device counterpart):
 * pos[8k..] = x,y,z,t, nx,ny,nz,length; out as there. */
void ppco_index_probe(const ppco_tables* t, const float* pos, int n, int32_t* out_i, float* out_f);
void ppco_string_pass(const ppco_tables* t, const float* pos, int n, int32_t* out);

#ifdef __cplusplus
}
#endif
#endif
