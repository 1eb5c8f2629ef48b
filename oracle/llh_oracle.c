/* TEST INFRASTRUCTURE -- never part of the product.
 *
 * Plain-C restatement of DirectFit's likelihood (llh/llh.cxx), the checker for the GPU
 * likelihood (ppcb_llh_*).  It follows the reference's own structure: one `dat` record per
 * DOM with its 200 bins (llh/llh.cxx:419-435), prep (:436-450), optimize (:516-612),
 * fill/join (:469-482, :614-621), llh (:484-492), llf (:637-662), in (:664-666) and fllh
 * (:1075-1082); the pulses are read as in cascade::ini (:739-806) and the simulated hits
 * are sorted into DOMs as in cascade::ppc (:1694-1700).
 *
 * Parity unpinned: the reference's llh.cxx needs GSL (gsl_sf_lnfact, minimisers), which is
 * not installed, so it cannot be compiled here and has no fixtures for this path.  The
 * tests pin this restatement by properties instead: llf's closed form without model error,
 * the Newton solution's stationarity with it, and the block partition against an
 * exhaustive search.  log L! is lgamma(L + 1) (the reference: gsl_sf_lnfact).
 */
#include "llh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NUM 200     /* llh/llh.cxx:43 */
#define BIN 25.0    /* llh/llh.cxx:46 */

typedef struct { float t, q; } pulse;

typedef struct {
  int str, om;
  pulse* draw; long ndraw, cdraw;
  double (*ert)[2]; long nert, cert;
  float* sraw; long nsraw, csraw;  /* simulated hit times */
  double dbin[NUM], sbin[NUM], dtot, stot, qtot;
  int n1, n2, ntop, htop;
  double opt[NUM], val[NUM];
  int lastchange[NUM];
  double dat[NUM], sim[NUM];
  int fnum;
} dat_t;

typedef struct {
  dat_t* d; long n, cap;
} all_t;

static int key_cmp(int s1, int o1, int s2, int o2) { return s1 != s2 ? (s1 < s2 ? -1 : 1) : (o1 < o2 ? -1 : o1 > o2); }

/* the DOM record for (str, om), created in key order if absent */
static dat_t* find(all_t* a, int str, int om, int create) {
  long lo = 0, hi = a->n;
  while (lo < hi) {
    long m = (lo + hi) / 2;
    int c = key_cmp(a->d[m].str, a->d[m].om, str, om);
    if (c == 0) return &a->d[m];
    if (c < 0) lo = m + 1; else hi = m;
  }
  if (!create) return NULL;
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 64;
    a->d = (dat_t*)realloc(a->d, a->cap * sizeof(dat_t));
  }
  memmove(&a->d[lo + 1], &a->d[lo], (a->n - lo) * sizeof(dat_t));
  memset(&a->d[lo], 0, sizeof(dat_t));
  a->d[lo].str = str; a->d[lo].om = om;
  a->n++;
  return &a->d[lo];
}

static void all_free(all_t* a) {
  for (long k = 0; k < a->n; k++) { free(a->d[k].draw); free(a->d[k].ert); free(a->d[k].sraw); }
  free(a->d);
}

static int isok_t(const dat_t* d, double t) {  /* llh/llh.cxx:426-429 */
  for (long i = 0; i < d->nert; i++) if (d->ert[i][0] <= t && t < d->ert[i][1]) return 0;
  return 1;
}

static double G(double L, double D) { /* llh/llh.cxx:500-505 with prior 0 */
  double R = D <= 0 ? 0 : D * log(D / L);
  double Q = lgamma(L + 1);
  return R + Q;
}

static int bad_has(const int32_t* bad, long nbad, int str, int om) {
  for (long k = 0; k < nbad; k++) if (bad[2 * k] == str && bad[2 * k + 1] == om) return 1;
  return 0;
}

static int isinice(int str, int om) { return str > 86 || (str > 0 && om >= 1 && om <= 60); }  /* llh/ppc.h:39 */

/* dat::optimize (llh/llh.cxx:516-612, keep = false) */
static int optimize(dat_t* d, const llho_opts* o, double lbin) {
  int htop;
  if (o->peak) {
    double opt1[NUM], val1[NUM], opt2[NUM], val2[NUM];
    int ntop = NUM;
    const double* dtop = d->dbin;
    for (int n = 0; n < ntop; n++) {
      double sD = 0, mxo = 0, sat = 0;
      int mxj = -1;
      for (int j = n; j >= 0; j--) {
        sD += dtop[j];
        int len = n - j + 1;
        double aux = G(len, sD), rat = sD / len;
        if (j > 0) aux += opt1[j - 1];
        if (j == 0 || val1[j - 1] < rat) if (mxj == -1 || aux > mxo) { mxo = aux; sat = rat; mxj = j; }
      }
      opt1[n] = mxo; val1[n] = sat;
    }
    for (int n = ntop - 1; n >= 0; n--) {
      double sD = 0, mxo = 0, sat = 0;
      int mxj = -1;
      for (int j = n; j < ntop; j++) {
        sD += dtop[j];
        int len = j - n + 1;
        double aux = G(len, sD), rat = sD / len;
        if (j < ntop - 1) aux += opt2[j + 1];
        if (j == ntop - 1 || val2[j + 1] < rat) if (mxj == -1 || aux > mxo) { mxo = aux; sat = rat; mxj = j; }
      }
      opt2[n] = mxo; val2[n] = sat;
    }
    {
      int m = -2;
      double sum = 0;
      for (int n = -1; n < ntop; n++) {
        double aux = (n >= 0 ? opt1[n] : 0) + (n < ntop - 1 ? opt2[n + 1] : 0);
        if (m == -2 || aux > sum) m = n, sum = aux;
      }
      if (m == -1 || (m < ntop - 1 && val2[m + 1] > val1[m])) m++;
      d->n1 = m - (int)round(500 / lbin); if (d->n1 < 0) d->n1 = 0;
      htop = m;
    }
    {
      int m = ntop + 1;
      double sum = 0;
      for (int n = ntop; n >= 0; n--) {
        double aux = (n < ntop ? opt2[n] : 0) + (n > 0 ? opt1[n - 1] : 0);
        if (m == ntop + 1 || aux > sum) m = n, sum = aux;
      }
      if (m == ntop || (m > 0 && val2[m] < val1[m - 1])) m--;
      d->n2 = m + (int)round(1000 / lbin); if (d->n2 > NUM) d->n2 = NUM;
      htop = (m + htop) / 2;
    }
  } else {
    int dmax = 0;
    double vmax = 0;
    for (int i = 0; i < NUM; i++) if (d->dbin[i] > vmax) vmax = d->dbin[i], dmax = i;
    d->n1 = dmax - (int)round(500 / lbin); if (d->n1 < 0) d->n1 = 0;
    htop = dmax;
    for (int i = NUM - 1; i > dmax; i--) if (d->dbin[i] == vmax) { dmax = i; break; }
    d->n2 = dmax + (int)round(1000 / lbin); if (d->n2 > NUM) d->n2 = NUM;
    htop = (dmax + htop) / 2;
  }
  const double* dtop = &d->dbin[d->n1];
  d->ntop = d->n2 - d->n1;
  htop -= d->n1;
  d->htop = htop;
  if (d->ntop <= 0) return -1;
  for (int n = 0; n < d->ntop; n++) {
    double sD = 0, mxo = 0, sat = 0;
    int mxj = -1;
    for (int j = n; j >= 0; j--) {
      sD += dtop[j];
      int len = n - j + 1;
      double aux = G(len, sD), rat = sD / len;
      if (j > 0) aux += d->opt[j - 1];
      if (!o->mono || j == 0 || (d->val[j - 1] - rat) * (j - 0.5 - htop) > 0)
        if (mxj == -1 || aux > mxo) { mxo = aux; sat = rat; mxj = j; }
    }
    d->opt[n] = mxo; d->val[n] = sat; d->lastchange[n] = mxj;
  }
  int f = d->ntop - 1;
  d->fnum = 0;
  for (int k = d->lastchange[f];; k = d->lastchange[f]) {
    double s = 0;
    for (; f >= k; f--) s += dtop[f];
    d->dat[d->fnum++] = s;
    if (k == 0) break;
  }
  return 0;
}

/* dat::prep (llh/llh.cxx:436-450) */
static int prep(dat_t* d, double t0, double lbin, const llho_opts* o) {
  for (int k = 0; k < NUM; k++) d->dbin[k] = 0;
  d->dtot = 0; d->qtot = 0;
  for (long j = 0; j < d->ndraw; j++) {
    d->qtot += d->draw[j].q;
    if (isok_t(d, d->draw[j].t)) {
      double t = round((d->draw[j].t - t0) / lbin), q = d->draw[j].q;
      if (t < 0 || t >= NUM) q = 0;
      if (t < 0) t = 0; else if (t >= NUM) t = NUM - 1;
      d->dbin[(int)t] += q; d->dtot += q;
    }
  }
  return optimize(d, o, lbin);
}

static int in(const dat_t* d, const llho_opts* o) {  /* dat::in (llh/llh.cxx:664-666) */
  return d->qtot < o->qsat * o->drep && d->qtot > o->qmin * o->drep &&
         (!o->flasher || d->str != abs(o->fla_str) || abs(d->om - o->fla_om) > o->fsep);
}

double llho_llf(double s, double d, double nsim, double ndat, double sig, int* err) {
  if (s < 0 || d < 0) { *err = 1; return NAN; }
  if (s == 0 && d == 0) return 0;
  double s2 = sig * sig, tol = 1.e-8;
  double sd = s + d, ntot = ndat + nsim;
  double ls = sd / ntot, ld = ls, llx;
  if (sig > 0) {
    double dls;
    int it = 0;
    do {
      double f = nsim * ls - s - log(ld / ls) / s2;
      double df = 1 + (1 / (ndat * ld) + 1 / (nsim * ls)) / s2;
      dls = -f / (nsim * df); ls += dls; ld = (sd - nsim * ls) / ndat;
      if (ls < 0 || ld < 0 || ++it > 200) { *err = 1; return NAN; }  /* the reference exits */
    } while (fabs(dls) > tol * ls);
    llx = log(ld / ls) * log(ld / ls) / (2 * s2);
  } else llx = 0;
  double lls = 0; if (s > 0) lls += s * log((s / nsim) / ls);
  double lld = 0; if (d > 0) lld += d * log((d / ndat) / ld);
  return llx + lls + lld;
}

/* cascade::ini's reading of the pulses and the preparation of every DOM */
static int setup(all_t* a, const llho_hit* data, long n, const llho_window* w, long nw, const int32_t* bad, long nbad,
                 const llho_opts* o, double* lbin, double* t0, int* ndof) {
  for (long k = 0; k < nw; k++) {
    dat_t* d = find(a, w[k].str, w[k].om, 1);
    if (d->nert == d->cert) { d->cert = d->cert ? 2 * d->cert : 4; d->ert = realloc(d->ert, d->cert * sizeof(*d->ert)); }
    d->ert[d->nert][0] = w[k].ti; d->ert[d->nert][1] = w[k].tf; d->nert++;
  }
  double tmin = NAN, tx = NAN;
  for (long k = 0; k < n; k++) {
    if (!isinice(data[k].str, data[k].om) || bad_has(bad, nbad, data[k].str, data[k].om)) continue;
    double t = data[k].t;
    if (isnan(tmin) || t < tmin) tmin = t;
    if (isnan(tx) || t > tx) tx = t;
    double q = data[k].q * o->drep;
    if (q > 0) {
      dat_t* d = find(a, data[k].str, data[k].om, 1);
      if (d->ndraw == d->cdraw) { d->cdraw = d->cdraw ? 2 * d->cdraw : 16; d->draw = realloc(d->draw, d->cdraw * sizeof(pulse)); }
      d->draw[d->ndraw].t = (float)t; d->draw[d->ndraw].q = (float)q; d->ndraw++;
    }
  }
  if (isnan(tmin)) return -1;
  if (o->lbin > 0) *lbin = o->lbin;
  else { double aux = (tx - tmin + 1) / NUM; *lbin = aux > BIN ? aux : BIN; }
  if (round(1000 / *lbin) < 1) return -1;
  *t0 = tmin;
  *ndof = 1;
  for (long k = 0; k < a->n; k++) {
    dat_t* d = &a->d[k];
    if (prep(d, *t0, *lbin, o) && in(d, o)) return -1;
    if (in(d, o)) *ndof += d->fnum;
  }
  return 0;
}

int llho_setup(const llho_hit* data, long n, const llho_window* w, long nw, const int32_t* bad, long nbad,
               const llho_opts* o, llho_block* out, long cap, long* nblocks, double* lbin, double* t0, int* ndof) {
  all_t a = {0};
  if (setup(&a, data, n, w, nw, bad, nbad, o, lbin, t0, ndof)) { all_free(&a); return -1; }
  long nb = 0;
  for (long k = 0; k < a.n; k++) {
    dat_t* d = &a.d[k];
    if (!in(d, o)) continue;
    int f = d->ntop - 1;
    for (int b = 0; b < d->fnum; b++) {
      int first = d->lastchange[f];
      if (nb < cap) {
        out[nb].str = d->str; out[nb].om = d->om;
        out[nb].first = d->n1 + first; out[nb].last = d->n1 + f;
        out[nb].dat = d->dat[b];
      }
      nb++;
      f = first - 1;
    }
  }
  *nblocks = nb;
  all_free(&a);
  return 0;
}

int llho_fllh(const llho_hit* data, long n, const llho_window* w, long nw, const int32_t* bad, long nbad,
              const llho_opts* o, const llho_sim* sim, long ns, const double* dts, int ndt, double nsim, double* out,
              int* errors) {
  all_t a = {0};
  double lbin, t0;
  int ndof;
  if (setup(&a, data, n, w, nw, bad, nbad, o, &lbin, &t0, &ndof)) { all_free(&a); return -1; }
  double nohit = 0;
  for (long k = 0; k < ns; k++) {  /* cascade::ppc (llh/llh.cxx:1686-1703), one charge per hit */
    if (bad_has(bad, nbad, sim[k].str, sim[k].om)) continue;
    dat_t* d = find(&a, sim[k].str, sim[k].om, 0);
    if (!d) { if (o->unh) nohit += 1; continue; }
    if (d->nsraw == d->csraw) { d->csraw = d->csraw ? 2 * d->csraw : 16; d->sraw = realloc(d->sraw, d->csraw * sizeof(float)); }
    d->sraw[d->nsraw++] = sim[k].t;
  }
  *errors = 0;
  for (int j = 0; j < ndt; j++) {
    const double dt = dts[j];
    int err = 0;
    double llh = o->norm ? 0 : llho_llf(nohit, 0, nsim, o->drep, o->sig, &err);
    *errors += err;
    for (long k = 0; k < a.n; k++) {
      dat_t* d = &a.d[k];
      if (!in(d, o)) continue;
      /* dat::fill: the simulated time on the observed clock is t + dt */
      for (int b = d->n1; b < d->n2; b++) d->sbin[b] = 0;
      d->stot = 0;
      for (long i = 0; i < d->nsraw; i++) {
        double ta = (double)d->sraw[i] + dt;
        if (!isok_t(d, ta)) continue;
        double t = round((ta - t0) / lbin), q = 1;
        if (t < 0 || t >= NUM) q = 0;
        if (d->n1 <= t && t < d->n2) { d->sbin[(int)t] += q; d->stot += q; }
      }
      { /* dat::join */
        const double* stop = &d->sbin[d->n1];
        int f = d->ntop - 1, fnum = 0;
        for (int k2 = d->lastchange[f];; k2 = d->lastchange[f]) {
          double s = 0;
          for (; f >= k2; f--) s += stop[f];
          d->sim[fnum++] = s;
          if (k2 == 0) break;
        }
      }
      /* dat::llh */
      double ns_ = nsim, r = 0;
      if (o->norm) {
        if (d->stot > 0) ns_ = d->stot * o->drep / d->dtot;
        else continue;
      }
      for (int b = 0; b < d->fnum; b++) { err = 0; r += llho_llf(d->sim[b], d->dat[b], ns_, o->drep, o->sig, &err); *errors += err; }
      llh += r;
    }
    out[j] = llh / ndof;
  }
  all_free(&a);
  return 0;
}
