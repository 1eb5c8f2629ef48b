/* TEST INFRASTRUCTURE -- the oracle of DirectFit's likelihood (llh_oracle.c).  The records
 * have the layouts of the product's ppcb_llh_hit / _window / _opts / _block. */
#pragma once
#include <stdint.h>

typedef struct { int32_t str, om; double t, q; } llho_hit;
typedef struct { int32_t str, om; double ti, tf; } llho_window;
typedef struct {
  double lbin, sig, qmin, qsat, drep;
  int32_t peak, mono, norm, unh, flasher, fla_str, fla_om, fsep;
} llho_opts;
typedef struct { int32_t str, om, first, last; double dat; } llho_block;
typedef struct { int32_t str, om; float t; } llho_sim;  /* one accepted simulated hit */

double llho_llf(double s, double d, double nsim, double ndat, double sig, int* err);
/* 0, or -1 where the product reports an error (no pulses, empty bin window) */
int llho_setup(const llho_hit* data, long n, const llho_window* w, long nw, const int32_t* bad, long nbad,
               const llho_opts* o, llho_block* out, long cap, long* nblocks, double* lbin, double* t0, int* ndof);
int llho_fllh(const llho_hit* data, long n, const llho_window* w, long nw, const int32_t* bad, long nbad,
              const llho_opts* o, const llho_sim* sim, long ns, const double* dts, int ndt, double nsim, double* out,
              int* errors);
