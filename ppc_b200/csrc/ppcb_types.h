// Plain-old-data records shared by the host library, the CUDA kernels and the C ABI.
//
// Capacities and record layouts follow the reference's data model so that files and
// output records stay interchangeable:
//   capacities            gpu/ini.cxx:1-26
//   DOM {R,F,r[3]}        gpu/ini.cxx:42-45   (20 B, one per optical module)
//   hit                   gpu/ini.cxx:367-371 (32 B kernel-level hit record)
//   photon (bunch)        gpu/ini.cxx:399-419 (64 B source record, one per photon bunch)
//   line (string)         gpu/ini.cxx:438-443
//   aniz (per layer)      gpu/ini.cxx:431-436
// Everything else (the table image that goes to HBM, the kernel parameter block) is
// this library's own layout.
#pragma once
#include <stdint.h>

#define PPCB_LMAX 80        // dust-logger maps for the tilt model
#define PPCB_LYRS 172       // tilt depth points
#define PPCB_CTX 11         // 2-d tilt grid
#define PPCB_CTY 10
#define PPCB_CX 21          // DOM-search cell grid
#define PPCB_CY 19
#define PPCB_NSTR 240       // strings
#define PPCB_WNUM 512       // wavelength bins
#define PPCB_MAXLYS 172     // ice layers
#define PPCB_MAXGEO 16384   // optical modules
#define PPCB_MAXRND 131072  // MWC multipliers (one random stream per GPU thread)

#define PPCB_BFR_TAB 1024   // intervals of the tabulated birefringence angular functions

#define PPCB_XXX 1.e-5f
#define PPCB_FPI 3.141592653589793f
#define PPCB_OMR 0.16510f   // DOM radius [m]
#define PPCB_DIR1 9.3f      // cell / tilt grid axes [deg]
#define PPCB_DIR2 129.3f

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ppcb_dom {
  float R, F;     // radius, spheroid flattening (F<0: cylinder)
  float r[3];     // position
} ppcb_dom;

typedef struct ppcb_hit {
  uint32_t i;     // DOM index (sorted geometry order)
  uint32_t n;     // segment (event) id
  uint32_t z;     // wavelength bin
  float t;        // time [ns]
  float pth, pph; // photon direction at impact
  float dth, dph; // impact point direction seen from the DOM centre
} ppcb_hit;

// A hit accepted by the back end (gpu/f2k.cxx:247-363): the sensor and PMT it registers
// on, its time and sampled wavelength, and the two vectors of the reference's hit map
// record (pout): the impact point relative to the sensor centre and the photon direction.
typedef struct ppcb_acc_hit {
  uint32_t i;      // DOM index
  uint32_t n;      // segment (event) id
  uint32_t hit;    // index of the kernel-level hit it came from
  int32_t str, om, pmt;
  float t;         // time [ns]
  float wv;        // wavelength [nm]
  float r[3];      // impact point [m], relative to the sensor centre
  float d[3];      // photon direction
} ppcb_acc_hit;

// One photon bunch: `num` photons sharing a source description.
// type>0: flasher/LED (ka,up,fldr,fla,ofla valid); type<=0: particle (a,b,beta,tau valid).
typedef struct ppcb_bunch {
  float r[4];     // position, time
  float n[4];     // direction, track length (n[3])
  uint32_t q;     // segment id echoed in hits
  uint32_t num;   // photons in this bunch
  int32_t type;   // source type
  float f;        // fraction of light from the bare muon
  union {
    struct { float a, b, beta, tau; } p;                   // particle
    struct { float ka, up, fldr; int16_t fla, ofla; } l;   // LED
    uint32_t c[4];
  } u;
} ppcb_bunch;

// A light source for the device front end: one addp (particle type), addp_clst,
// addp_mopo or f2k "ph" record with its segment's direction and id.
typedef struct ppcb_source {
  float r[4];      // x, y, z [m], t [ns]
  float n[3];      // direction (the segment's direction, as sett sets it)
  int32_t kind;    // PPCB_SRC_*
  double amount;   // PARTICLE: energy [GeV]; CLST, POINT: photons; MOPO: light
  float dr;        // PARTICLE, CLST: track length [m]; MOPO: length
  int32_t type;    // PARTICLE: 0 muon, 1 muon end point, 10-14 EM, 101-107 hadron (addp)
  float scale;     // PARTICLE: light scale (addp)
  float beta;      // CLST, MOPO
  float tau, fr;   // MOPO
  uint32_t q;      // segment id echoed in the hits
  uint32_t pad_;
} ppcb_source;
#define PPCB_SRC_PARTICLE 0  // addp, type >= 0 (gpu/f2k.cxx:484-504)
#define PPCB_SRC_CLST 1      // addp_clst (gpu/f2k.cxx:507-518)
#define PPCB_SRC_MOPO 2      // addp_mopo (gpu/f2k.cxx:520-528)
#define PPCB_SRC_POINT 3     // f2k "ph": exact count at a point (gpu/f2k.cxx:478-482)

typedef struct ppcb_line {
  int16_t n, max; // first DOM index, last DOM offset
  float x, y, r;  // string centre and search radius
  float h, d;     // top DOM depth, 1/spacing
  float dl, dh;   // depth tolerance below / above
} ppcb_line;

typedef struct ppcb_aniz { float k1, k2, ra, rb; } ppcb_aniz;

// Per-wavelength optical constants (bin index, 1/group velocity, Cherenkov cos/sin).
typedef struct ppcb_wmeta { float ocm, coschr, sinchr; int32_t wvl; } ppcb_wmeta;

// Scalar ice/geometry parameters consumed by the kernel (the scalar part of the
// reference's `dats`, gpu/ini.cxx:452-518).
typedef struct ppcb_params {
  int32_t size;               // ice layers
  float dh, rdh, hmin;        // layer step, 1/step, lowest layer centre depth
  float ocv;                  // 1/c in vacuum
  float sf, g, gr;            // scattering function mix and shape
  float xR;                   // DOM oversize
  float SF, G, GR;            // hole-ice scattering function
  float hr, hr2, hs, ha;      // hole-ice radius and coefficients
  float azx, azy;             // anisotropy axis
  int32_t cn[2];
  float cl[2], crst[2];
  float cb[2][2];
  int32_t tmod, vthk;         // tilt model, variable layer thickness
  int32_t lnum, lpts, l0;
  float lmin, lrdz, r0;
  float lnx, lny;
  float mmin[2], mstp[2];
  int32_t mnum[2], mcut[2];
  float k1, k2, kz, fr;       // absorption anisotropy
  float sum;                  // BFR strength
  float bfr[12];
  float rx;                   // cell-search safety margin
  float hifl;                 // hole-ice time window
  int32_t gsize;              // DOMs
  int32_t nstr;               // strings in use
  int32_t rsize;              // MWC multipliers
  int32_t pad_;
} ppcb_params;

// Device-side control block: counters written by the kernel, read back by the host.
typedef struct ppcb_ctrl {
  unsigned long long next;    // photon work counter (work stealing)
  unsigned long long hidx;    // hits produced (may exceed capacity: overflow)
  unsigned int nan_steps;     // steps with a non-finite TOT/SCA (photon killed)
  unsigned int capped;        // photons stopped by the per-photon step cap
  unsigned long long steps;   // total propagation steps (when counting is enabled)
  unsigned int bad_sm[4];     // SM ids of the first non-finite steps
  unsigned int pad_[2];
} ppcb_ctrl;

#ifdef __cplusplus
}
#endif
