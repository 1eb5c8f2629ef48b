/* TEST INFRASTRUCTURE ONLY -- the oracle (see ppc_oracle.h).
 *
 * Plain-C restatement of the reference's propagation kernel, gpu/pro.cu, in the form the
 * reference's CPU build executes it (XCPU shims gpu/pro.cu:1-45: rsqrtf = 1/sqrtf,
 * __float2int_rn = lroundf, _ru = ceilf, _rd = floorf).  Compiled with IEEE float
 * semantics (-O2, no fast-math); the reference compiled the same way (oracle/Makefile,
 * _ref/ref_harness) produces bit-identical photons, hits and random streams.  Each
 * function cites the lines it follows.
 */
#define _GNU_SOURCE
#include "ppc_oracle.h"

#include <math.h>
#include <string.h>

#define WNUM PPCB_WNUM
#define XXX PPCB_XXX
#define FPI PPCB_FPI
#define OMR PPCB_OMR
static const float fcv = FPI / 180.f;

/* Event counters of ppco_propagate (the algorithmic work of the propagation: steps, layer
 * crossings, string and DOM tests, hits, birefringence and scattering evaluations). */
static ppco_counts g_cnt;
void ppco_counts_reset(void) { memset(&g_cnt, 0, sizeof(g_cnt)); }
void ppco_counts_get(ppco_counts* out) { *out = g_cnt; }

/* Optional step trace: the segment each step hands to the DOM search (position, direction,
 * geometric length), 8 floats per step, in the layout ppco_string_pass reads. */
static float* g_trace;
static uint64_t g_trace_cap, g_trace_n;
void ppco_trace_steps(float* buf, uint64_t cap) { g_trace = buf; g_trace_cap = cap; g_trace_n = 0; }
uint64_t ppco_trace_count(void) { return g_trace_n; }

/* std::min / std::max argument-order semantics */
static inline float mnf(float a, float b) { return b < a ? b : a; }
static inline float mxf(float a, float b) { return a < b ? b : a; }
static inline int mni(int a, int b) { return b < a ? b : a; }
static inline int mxi(int a, int b) { return a < b ? b : a; }
static inline int rn(float x) { return (int)lroundf(x); }
static inline int rd(float x) { return (int)floorf(x); }
static inline int ru(float x) { return (int)ceilf(x); }
static inline float sq(float x) { return x * x; }

typedef struct { float x, y, z, w; } f4;

/* gpu/pro.cu:47-57: 64-bit multiply-with-carry, result in (0,1] */
float ppco_xrnd(ppco_rng* s) {
  uint64_t sda = s->y;
  sda += (uint64_t)s->a * (uint64_t)s->x;
  s->x = (uint32_t)sda;
  s->y = (uint32_t)(sda >> 32);
  uint32_t tmp = (s->x >> 9) | 0x3f800000u;
  float f;
  memcpy(&f, &tmp, 4);
  return 2.f - f;
}

/* gpu/pro.cu:59-85: gamma-distributed sample (Weibull rejection for k<1, Cheng for k>=1) */
static float mrnd(float k, ppco_rng* s) {
  float x;
  if (k < 1) {
    float c = 1 / k;
    float d = (1 - k) * powf(k, 1 / (c - 1));
    float z, e;
    do {
      z = -logf(ppco_xrnd(s));
      e = -logf(ppco_xrnd(s));
      x = powf(z, c);
    } while (z + e < d + x);
  } else {
    float b = k - logf(4.0f);
    float l = sqrtf(2 * k - 1);
    float c = 1 + logf(4.5f);
    float u, v, y, z, r;
    do {
      u = ppco_xrnd(s);
      v = ppco_xrnd(s);
      y = -logf(1 / v - 1) / l;
      x = k * expf(y);
      z = u * v * v;
      r = b + (k + l) * y - x;
    } while (r < 4.5f * z - c && r < logf(z));
  }
  return x;
}

/* gpu/pro.cu:87-95: Box-Muller */
static float grnd(ppco_rng* s) {
  float a = sqrtf(-2 * logf(ppco_xrnd(s)));
  return a * sinf(2 * FPI * ppco_xrnd(s));
}

static void grnd2(float* px, float* py, ppco_rng* s) {
  float r = sqrtf(-2 * logf(ppco_xrnd(s)));
  sincosf(2 * FPI * ppco_xrnd(s), py, px);
  *px *= r;
  *py *= r;
}

static void swp(float* a, float* b) { float t = *a; *a = *b; *b = t; }

/* gpu/pro.cu:111-153: rotate n by polar angle (cs = 1-cos, si = sin), uniform azimuth */
static void rotate(float cs, float si, f4* n, ppco_rng* s) {
  float p1x, p1y, p1z, p2x, p2y, p2z;
  int i = 0;
  {
    float rx = n->x * n->x, ry = n->y * n->y, rz = n->z * n->z;
    if (ry > rz) {
      if (ry > rx) { swp(&n->x, &n->y); swp(&rx, &ry); i = 1; }
    } else {
      if (rz > rx) { swp(&n->x, &n->z); swp(&rx, &rz); i = 2; }
    }
    ry = 1 / sqrtf(rx + ry); p1x = -n->y * ry; p1y = n->x * ry; p1z = 0;
    rz = 1 / sqrtf(rx + rz); p2x = -n->z * rz; p2y = 0; p2z = n->x * rz;
  }
  {
    float q1x = p1x - p2x, q1y = p1y - p2y, q1z = p1z - p2z;
    p2x += p1x; p2y += p1y; p2z += p1z;
    float q1w = 1 / sqrtf(q1x * q1x + q1y * q1y + q1z * q1z);
    p1x = q1x * q1w; p1y = q1y * q1w; p1z = q1z * q1w;
    q1w = 1 / sqrtf(p2x * p2x + p2y * p2y + p2z * p2z);
    p2x *= q1w; p2y *= q1w; p2z *= q1w;
  }
  {
    float px, py;
    float xi = 2 * FPI * ppco_xrnd(s);
    sincosf(xi, &py, &px);
    n->x -= cs * n->x - si * (px * p1x + py * p2x);
    n->y -= cs * n->y - si * (px * p1y + py * p2y);
    n->z -= cs * n->z - si * (px * p1z + py * p2z);
    float r = 1 / sqrtf(n->x * n->x + n->y * n->y + n->z * n->z);
    n->x *= r; n->y *= r; n->z *= r;
    if (i == 1) swp(&n->x, &n->y);
    else if (i == 2) swp(&n->x, &n->z);
  }
}

static inline int findcol(const ppco_tables* t, int x, int y) {
  const ppcb_params* d = t->p;
  return x >= 0 && x < d->mnum[0] && y >= 0 && y < d->mnum[1] ? t->mcol[x * PPCB_CTY + y] : -1;
}

static inline void lpv(const ppco_tables* t, int i, int k, float* x, float* y) {
  *x = t->lp[(i * PPCB_LYRS + k) * 2];
  *y = t->lp[(i * PPCB_LYRS + k) * 2 + 1];
}

/* gpu/pro.cu:168-264: depth shift of the layer isochrons (1-d and 2-d tilt models) */
float ppco_zshift(const ppco_tables* t, const float* r, float* dz) {
  const ppcb_params* d = t->p;
  if (d->tmod == 1) {
    float nr = d->lnx * r[0] + d->lny * r[1] - d->r0;
    int j = 1;
    for (; j < PPCB_LMAX; j++) if (nr < t->lr[j] || j == d->lnum - 1) break;
    float z = (r[2] - d->lmin) * d->lrdz;
    int i = j - 1, k = mni(mxi(rd(z), 0), d->lpts);
    float pix, piy, pjx, pjy;
    lpv(t, i, k, &pix, &piy);
    lpv(t, j, k, &pjx, &pjy);
    float dw = t->lr[j] - t->lr[i];
    float wx = (nr - t->lr[i]) / dw;
    float wy = (t->lr[j] - nr) / dw;
    float qx = pjx * wx + pix * wy;
    float qy = pjy * wx + piy * wy;
    float rr = qx + qy * (z - k);
    if (d->vthk != 0) *dz /= 1 - d->lrdz * qy;
    return rr;
  } else if (d->tmod == 2) {
    float qx = d->cb[0][0] * r[0] + d->cb[1][0] * r[1];
    float qy = d->cb[0][1] * r[0] + d->cb[1][1] * r[1];
    qx = (qx - d->mmin[0]) / d->mstp[0];
    qy = (qy - d->mmin[1]) / d->mstp[1];
    {
      float x = qx, y = qy, xy;
      int n0 = d->mnum[0] - 1, n1 = d->mnum[1] - 1, c0 = d->mcut[0] - 1, c1 = d->mcut[1] - 1;
      if (y < 0) if (x - y > 0 && x <= c0) { x = (x - y) * c0 / (c0 - y); y = 0; }
      if (x < 0) if (y - x >= 0 && y < c1) { y = (y - x) * c1 / (c1 - x); x = 0; }
      if (y > n1) if (x >= n1 - c1 && y - x > n1 - n0) { x = n1 - c1 + (n0 - (n1 - c1)) * (x - (n1 - c1)) / (y - (n1 - n0) - (n1 - c1)); y = n1; }
      if (x > n0) if (y > n0 - c0 && y - x <= n1 - n0) { y = n0 - c0 + (n1 - (n0 - c0)) * (y - (n0 - c0)) / (x - (n0 - n1) - (n0 - c0)); x = n0; }
      if (y - x > c1) if (y >= c1 && x < n1 - c1) { xy = y - x - c1; xy = c1 + (x + y - c1 + xy) * (n1 - c1) / (n1 - c1 + xy); x = (xy - c1) / 2; y = (xy + c1) / 2; }
      if (x - y > c0) if (x > c0 && y <= n0 - c0) { xy = x - y - c0; xy = c0 + (x + y - c0 + xy) * (n0 - c0) / (n0 - c0 + xy); x = (xy + c0) / 2; y = (xy - c0) / 2; }
      qx = x; qy = y;
    }
    int qnx0 = mni(mxi(rd(qx), 0), d->mnum[0]);
    int qny0 = mni(mxi(rd(qy), 0), d->mnum[1]);
    float qrx0 = qx - qnx0, qry0 = qy - qny0;
    float qrx, qry;
    int qnx, qny;
    if (qrx0 > qry0) { qrx = qrx0; qry = qry0; qnx = qnx0 + 1; qny = qny0; }
    else { qrx = qry0; qry = qrx0; qnx = qnx0; qny = qny0 + 1; }
    int cx = findcol(t, qnx0, qny0);
    int cy = findcol(t, qnx, qny);
    int cz = findcol(t, qnx0 + 1, qny0 + 1);
    float wx = 1 - qrx, wy = qrx - qry, wz = qry;
    float z = (r[2] - d->lmin) * d->lrdz;
    int k = mni(mxi(rd(z), 0), d->lpts);
    float ax = 0, ay = 0;
    float px, py;
    if (cx >= 0) { lpv(t, cx, k, &px, &py); ax += px * wx; ay += py * wx; }
    if (cy >= 0) { lpv(t, cy, k, &px, &py); ax += px * wy; ay += py * wy; }
    if (cz >= 0) { lpv(t, cz, k, &px, &py); ax += px * wz; ay += py * wz; }
    float rr = ax + ay * (z - k);
    if (d->vthk != 0) *dz /= 1 - d->lrdz * ay;
    return rr;
  }
  return 0;
}

/* gpu/pro.cu:580-594: search cells covered by the segment r -> r + sca*n (plus margin rx) */
static void cell_range(const ppcb_params* e, float rx0, float ry0, float rx1, float ry1, int* xlx, int* xhx,
                       int* xly, int* xhy) {
  float pix = e->cb[0][0] * rx0 + e->cb[1][0] * ry0;
  float piy = e->cb[0][1] * rx0 + e->cb[1][1] * ry0;
  float pfx = e->cb[0][0] * rx1 + e->cb[1][0] * ry1;
  float pfy = e->cb[0][1] * rx1 + e->cb[1][1] * ry1;
  float lx = mnf(pix, pfx) - e->rx, hx = mxf(pix, pfx) + e->rx;
  float ly = mnf(piy, pfy) - e->rx, hy = mxf(piy, pfy) + e->rx;
  *xlx = mni(mxi(rn((lx - e->cl[0]) * e->crst[0]), 0), e->cn[0]);
  *xhx = mxi(mni(rn((hx - e->cl[0]) * e->crst[0]), e->cn[0] - 1), -1);
  *xly = mni(mxi(rn((ly - e->cl[1]) * e->crst[1]), 0), e->cn[1]);
  *xhy = mxi(mni(rn((hy - e->cl[1]) * e->crst[1]), e->cn[1] - 1), -1);
}

/* gpu/pro.cu:623-626: DOM index window of one string for the depth range [zl, zh] */
static void dom_window(const ppcb_line* sl, float zl, float zh, int* n1, int* n2) {
  int omin = 0, omax = sl->max;
  *n1 = sl->n - omin + mni(omax + 1, mxi(omin, ru(omin - (zh - sl->dl - sl->h) * sl->d)));
  *n2 = sl->n - omin + mxi(omin - 1, mni(omax, rd(omin - (zl - sl->dh - sl->h) * sl->d)));
}

static inline float wabs(const ppco_tables* t, uint32_t w, int J) { return t->absca[((size_t)w * t->p->size + J) * 2]; }
static inline float wsca(const ppco_tables* t, uint32_t w, int J) { return t->absca[((size_t)w * t->p->size + J) * 2 + 1]; }

/* gpu/pro.cu:335-476: one photon from its bunch */
void ppco_generate(const ppco_tables* t, const ppcb_bunch* pp, ppco_rng* s, ppco_pbuf* out) {
  const ppcb_params* e = t->p;
  const ppcb_bunch p = *pp;
  f4 r, n;
  unsigned int j = (unsigned int)mni(rd(WNUM * ppco_xrnd(s)), WNUM - 1);
  const ppcb_wmeta* w = &t->wmeta[j];
  n.w = w->ocm;
  r.x = p.r[0]; r.y = p.r[1]; r.z = p.r[2]; r.w = p.r[3];
  n.x = p.n[0]; n.y = p.n[1]; n.z = p.n[2];
  float l = p.n[3];
  int fla, ofla;
  if (p.type > 0) {
    fla = p.u.l.fla; ofla = p.u.l.ofla;
    if (l == 0) {  /* N-fold / cylindrical LED pattern */
      float xi = ppco_xrnd(s);
      if (p.u.l.fldr < 0) xi *= 2 * FPI;
      else {
        int rr = rd(p.u.l.fldr / 360) + 1;
        int ss = rd(xi * rr);
        xi = (p.u.l.fldr + ss * 360 / rr) * fcv;
      }
      sincosf(xi, &r.y, &r.x);
      sincosf(p.u.l.up, &n.z, &xi);
      n.x = xi * r.x; n.y = xi * r.y;
    }
    if (p.u.l.ka != 0) {
      float xi;
      if (p.u.l.ka > 999.f) {  /* lab-measured beam profile */
        xi = ppco_xrnd(s);
        float s1 = 0.0191329f, s2 = 0.0686944f, C1 = 0.583583f, C2 = 0.967762f;
        switch (p.type) {
          case 1: s1 = 0.0196242f; s2 = 0.0750278f; C1 = 0.606833f; C2 = 0.960863f; break;
          case 2: s1 = 0.0185603f; s2 = 0.0624481f; C1 = 0.553192f; C2 = 0.974129f; break;
        }
        xi = xi < C1 ? s1 * fabsf(grnd(s)) : xi < C2 ? -s2 * logf(ppco_xrnd(s)) : 2.f;
        if (xi >= 2.f) xi = 2 * (1 - sqrtf(ppco_xrnd(s)));
      } else if (p.u.l.ka > 0) xi = mnf(-p.u.l.ka * logf(1 - (1 - ppco_xrnd(s)) * (1 - expf(-2 / p.u.l.ka))), 2.f);
      else if (p.u.l.ka == -1) xi = 2 * (1 - ppco_xrnd(s));
      else xi = 2 * (1 - sqrtf(ppco_xrnd(s)));
      rotate(xi, sqrtf(xi * (2 - xi)), &n, s);
    }
    if (p.u.l.ka > 999.f) {  /* start on the DOM surface; harness and cable veto */
      const float FLZ = 0.07735f, FLR = 0.119f - 0.008f, FLB = 0.03396f;
      if (l == 0) { r.x *= FLR; r.y *= FLR; r.z = FLZ; r.w = 0; }
      float b = r.x * n.x + r.y * n.y + r.z * n.z;
      float c = FLZ * FLZ + FLR * FLR - OMR * OMR;
      float tt = sqrtf(b * b - c) - b;
      r.x += tt * n.x; r.y += tt * n.y; r.z += tt * n.z; r.w += tt * e->ocv;
      if (fabsf(r.z) < FLB) ofla = -2;
      else if (l == 0 && r.z < 0 && ppco_xrnd(s) < 0.9f) ofla = -3;
      if (p.u.l.ka > 1050.f) {
        const float rc = 0.023f;
        const float dc = OMR + rc;
        float ph = (p.u.l.ka - 1080.f) * fcv;
        float drx = r.x - dc * cosf(ph);
        float dry = r.y - dc * sinf(ph);
        float a = n.x * n.x + n.y * n.y;
        if (a > 0) {
          float bb = n.x * drx + n.y * dry;
          float cc = drx * drx + dry * dry - rc * rc;
          float D = bb * bb - a * cc;
          if (D >= 0) {
            float h1 = (-bb + sqrtf(D)) / a;
            if (h1 > 0) ofla = -4;
          }
        }
      }
      if (l == 0) { r.x += p.r[0]; r.y += p.r[1]; r.z += p.r[2]; r.w += p.r[3]; }
      else {
        const ppcb_dom* dom = &t->oms[fla];
        r.x += dom->r[0]; r.y += dom->r[1]; r.z += dom->r[2]; r.w += p.r[3];
      }
    } else if (fla >= 0) {
      const float tt = OMR;
      r.x = tt * n.x; r.y = tt * n.y; r.z = tt * n.z; r.w = tt * e->ocv;
      r.x += p.r[0]; r.y += p.r[1]; r.z += p.r[2]; r.w += p.r[3];
    } else {
      r.x = p.r[0]; r.y = p.r[1]; r.z = p.r[2]; r.w = p.r[3];
    }
  } else {
    fla = -1; ofla = -1;
    if (l > 0) l *= ppco_xrnd(s);
    else l = p.u.p.b * mrnd(p.u.p.a, s);
    if (l > 0) {
      r.x += l * n.x; r.y += l * n.y; r.z += l * n.z;
      r.w += l * e->ocv / p.u.p.beta;
    }
    if (p.u.p.tau > 0) {  /* isotropic delayed emission */
      r.w -= p.u.p.tau * logf(ppco_xrnd(s));
      float xi = 1 - ppco_xrnd(s);
      rotate(xi, sqrtf(xi * (2 - xi)), &n, s);
    } else {
      float cs = w->coschr, si = w->sinchr;
      if (p.f < ppco_xrnd(s)) {  /* cascade secondary directions */
        const float a = 0.39f, b = 2.61f;
        const float I = 1 - expf(-b * exp2f(a));
        float xi = mnf(powf(-logf(1 - ppco_xrnd(s) * I) / b, 1 / a), 2.f);
        rotate(xi, sqrtf(xi * (2 - xi)), &n, s);
      } else {
        float beta = p.u.p.beta;
        if (p.type < 0) {  /* muon slowing down near its end point */
          const float ar = 0.26f * 0.9216f / 0.105658389f;
          float dx = ar * (p.n[3] - l);
          beta = sqrtf(dx * (2 + dx)) / (1 + dx);
          if (beta >= cs) r.w -= e->ocv * (sqrtf(dx * dx + 1) - asinhf(1 / dx) - dx) / ar;
        }
        if (beta < 1) {
          float xi = cs / beta;
          if (xi <= 1) {
            float sx = sqrtf(1 - xi * xi);
            if (p.type < 0 && sx < ppco_xrnd(s) * si) ofla = -3;
            cs = xi; si = sx;
          } else ofla = -2;
        }
      }
      rotate(1 - cs, si, &n, s);  /* Cherenkov cone */
    }
  }
  out->r[0] = r.x; out->r[1] = r.y; out->r[2] = r.z; out->r[3] = r.w;
  out->n[0] = n.x; out->n[1] = n.y; out->n[2] = n.z; out->n[3] = n.w;
  out->q = j; out->i = p.q; out->fla = fla; out->ofla = ofla;
}

/* gpu/pro.cu:486-889, one photon from initialisation until TOT==0 */
uint64_t ppco_propagate(const ppco_tables* t, const ppco_pbuf* f, ppco_rng* s, ppcb_hit* hits,
                        uint64_t* nhit, uint64_t cap) {
  const ppcb_params* e = t->p;
  f4 r, n;
  r.x = f->r[0]; r.y = f->r[1]; r.z = f->r[2]; r.w = f->r[3];
  n.x = f->n[0]; n.y = f->n[1]; n.z = f->n[2]; n.w = f->n[3];
  const uint32_t wl = f->q;
  const uint32_t niw = f->i;
  int om = f->fla;
  const int ofla = f->ofla;
  g_cnt.photons++;
  int old = -1;
  float TOT = -logf(ppco_xrnd(s)), SCA = 0;
  if (ofla < -1) TOT = 0;
  uint64_t steps = 0;
  for (;;) {
    steps++;
    g_cnt.steps++;
    float sqd = 0;
    if (SCA == 0) { SCA = -logf(ppco_xrnd(s)); old = om; g_cnt.sca_draws++; }
    float sca, tot;
    int sign = n.z < 0 ? -1 : 1;
    float anz = sign * n.z;
    float edh = e->dh;
    float rr[4] = {r.x, r.y, r.z, r.w};
    float z = r.z - ppco_zshift(t, rr, &edh);
    float nr = 1.f;
    int I, J;
    {
      z = (z - e->hmin) * e->rdh;
      I = mni(mxi(rn(z), 0), e->size - 1);
      if (TOT > 0) {  /* absorption anisotropy, gpu/pro.cu:517-544 */
        float n1 = e->azx * n.x + e->azy * n.y;
        float n2 = -e->azy * n.x + e->azx * n.y;
        float n3 = n.z;
        if (e->fr != 0) {
          float k1 = t->az[I].k1, k2 = t->az[I].k2;
          float kz = 1 / (k1 * k2);
          float s1 = n1 * n1, l1 = k1 * k1;
          float s2 = n2 * n2, l2 = k2 * k2;
          float s3 = n3 * n3, l3 = kz * kz;
          float B2 = nr / l1 + nr / l2 + nr / l3;
          float nB = s1 / l1 + s2 / l2 + s3 / l3;
          float An = s1 * l1 + s2 * l2 + s3 * l3;
          nr = powf((B2 - nB) * An / 2, e->fr);
        }
        n1 *= e->k1; n2 *= e->k2; n3 *= e->kz;
        nr *= 1 / sqrtf(n1 * n1 + n2 * n2 + n3 * n3);
        TOT /= nr;
      }
      float ahx = edh * (0.5f - sign * (z - I));
      J = I;  /* layer stepping, gpu/pro.cu:548-571 */
      sca = 0; tot = 0;
      float ais = SCA, aia = TOT;
      for (;;) {
        float dsca = ais / wsca(t, wl, J), dtot = aia / wabs(t, wl, J);
        float dist = mnf(dsca, dtot) * anz;
        if ((sign < 0 ? J > 0 : J < e->size - 1) && dist > ahx) {
          float del = ahx / anz;
          sca += del; tot += del;
          ais -= wsca(t, wl, J) * del; aia -= wabs(t, wl, J) * del;
          ahx = edh;
          J += sign;
          g_cnt.crossings++;
        } else {
          sca += dsca; tot += dtot;
          break;
        }
      }
      if (sca < 0) sca = 0;
      if (tot < 0) tot = 0;
      if (tot < sca) { sca = tot; tot = 0; }
      else tot = (tot - sca) * wabs(t, wl, J);
    }

    om = -1;
    float del = sca;
    float hi = sca, hf = 0;
    if (g_trace && g_trace_n < g_trace_cap) {
      float* q = g_trace + 8 * g_trace_n++;
      q[0] = r.x; q[1] = r.y; q[2] = r.z; q[3] = r.w; q[4] = n.x; q[5] = n.y; q[6] = n.z; q[7] = sca;
    }
    {  /* DOM search through the cell grid, gpu/pro.cu:577-672 */
      int xlx, xhx, xly, xhy;
      cell_range(e, r.x, r.y, r.x + sca * n.x, r.y + sca * n.y, &xlx, &xhx, &xly, &xhy);
      for (int i = xlx, j = xly; i <= xhx && j <= xhy; (++j <= xhy) ? 0 : (j = xly, i++)) {
        for (unsigned short k = t->is[i * PPCB_CY + j]; k != 0x8000;) {
          unsigned short m = t->ls[k];
          const ppcb_line* sl = &t->sc[m & 0x7fff];
          k = (m & 0x8000) ? 0x8000 : k + 1;
          g_cnt.strings_tested++;
          float b = 0, c = 0, dr;
          dr = sl->x - r.x; b += n.x * dr; c += dr * dr;
          dr = sl->y - r.y; b += n.y * dr; c += dr * dr;
          float np = 1 - n.z * n.z;
          float D = b * b - (c - sl->r * sl->r) * np;
          if (D >= 0) {
            D = sqrtf(D);
            float h1 = b - D, h2 = b + D;
            if (h2 >= 0 && h1 <= sca * np) {
              if (np > XXX) {
                h1 /= np; h2 /= np;
                if (h1 < 0) h1 = 0;
                if (h2 > sca) h2 = sca;
              } else { h1 = 0; h2 = sca; }
              h1 = r.z + n.z * h1; h2 = r.z + n.z * h2;
              float zl, zh;
              if (n.z > 0) { zl = h1; zh = h2; }
              else { zl = h2; zh = h1; }
              int n1, n2;
              dom_window(sl, zl, zh, &n1, &n2);
              g_cnt.strings_passed++;
              for (int l = n1; l <= n2; l++) if (l != old) {
                g_cnt.doms_tested++;
                const ppcb_dom* dom = &t->oms[l];
                float a = 0, bb = 0, cc = 0, dd;
                float fq = dom->F > 0 ? sq(1 / dom->F) : 0;
                dd = dom->r[0] - r.x; a += n.x * n.x; bb += n.x * dd; cc += dd * dd;
                dd = dom->r[1] - r.y; a += n.y * n.y; bb += n.y * dd; cc += dd * dd;
                dd = dom->r[2] - r.z; a += fq * n.z * n.z; bb += fq * n.z * dd; cc += fq * dd * dd;
                if (a > 0) {
                  bb /= a;
                  float xR = (l == ofla ? 1 : e->xR);
                  float DD = bb * bb - (cc - sq(xR * dom->R)) / a;
                  if (DD >= 0) {
                    sqd = sqrtf(DD);
                    float h = bb - sqd;
                    if (dom->F > 0 || fabsf(dd - n.z * h) < -xR * dom->F * dom->R) {
                      sqd /= xR; h = bb - sqd;
                      if (h > 0 && h <= del) { om = l; del = h; }
                    }
                  }
                }
              }
            }
          }
          if (e->hr > 0 && (e->hifl == 0 || (e->hifl < 0 && r.w < -e->hifl) || (e->hifl > 0 && r.w > e->hifl))) {
            float DH = b * b - (c - e->hr2) * np;
            if (DH > 0) {
              DH = sqrtf(DH);
              float h1 = b - DH, h2 = b + DH;
              if (h2 >= 0 && h1 <= sca * np) {
                if (np > XXX) {
                  h1 /= np; h2 /= np;
                  if (h1 < 0) h1 = 0;
                  if (h2 > sca) h2 = sca;
                } else { h1 = 0; h2 = sca; }
                if (h1 < hi && h2 > sqrtf(XXX) * e->hr) { hi = h1; hf = h2; }
              }
            }
          }
        }
      }
    }

    float fin = mnf(del, hi);
    int hole = fin < sca;
    if (hole) {  /* truncated step: overburden by layers, hole-ice column, gpu/pro.cu:677-717 */
      g_cnt.truncated++;
      {
        float xs = 0, xa = 0;
        float y = z + n.z * fin / edh;
        J = mni(mxi(rn(y), 0), e->size - 1);
        if (I == J) { xs = fin * wsca(t, wl, I); xa = fin * wabs(t, wl, I); }
        else {
          float h = 0.5f - sign * (z - I);
          float g = 0.5f + sign * (y - J);
          xs = h * wsca(t, wl, I) + g * wsca(t, wl, J);
          xa = h * wabs(t, wl, I) + g * wabs(t, wl, J);
          for (int i = I + sign; i != J; i += sign) { xs += wsca(t, wl, i); xa += wabs(t, wl, i); }
          float ff = edh / anz;
          xs *= ff; xa *= ff;
        }
        if (xs < 0) xs = 0;
        if (xa < 0) xa = 0;
        SCA -= xs; TOT -= xa;
      }
      TOT *= nr;
      if (hi < del) {
        float fin2 = mnf(hi + mnf(SCA / e->hs, TOT / e->ha), hf);
        if (om != -1) { if (fin2 < del) { del = fin2; om = -1; } }
        else {
          if (fin2 < del) del = fin2;
          else del = mnf(fin2, sca);
        }
        fin2 = del - hi;
        SCA -= fin2 * e->hs; TOT -= fin2 * e->ha;
      }
    } else { SCA = 0; TOT = tot * nr; }

    r.x += del * n.x; r.y += del * n.y; r.z += del * n.z; r.w += del * n.w;

    if (om != -1) {  /* DOM hit, gpu/pro.cu:731-753 */
      if (om == ofla) TOT = 0;
      else {
        ppcb_hit h;
        h.i = om; h.t = r.w; h.n = niw; h.z = t->wmeta[wl].wvl;
        h.pth = acosf(n.z); h.pph = atan2f(n.y, n.x);
        sqd *= e->xR - 1;
        const ppcb_dom* dom = &t->oms[om];
        float dx = dom->r[0] - r.x + sqd * n.x;
        float dy = dom->r[1] - r.y + sqd * n.y;
        float dz = dom->r[2] - r.z + sqd * n.z;
        h.dth = acosf(mnf(mxf(dz / (e->xR * dom->R * dom->F), -1.f), 1.f));
        h.dph = atan2f(dy, dx);
        uint64_t jh = (*nhit)++;
        g_cnt.hits++;
        if (jh < cap) hits[jh] = h;
        if (e->xR == 1) TOT = 0;
        else old = om;
      }
    }

    if (TOT < XXX) TOT = 0;
    else {
      if (e->sum > 0 && fin > 0) {  /* birefringence diffusion, gpu/pro.cu:757-836 */
        g_cnt.bfr++;
        float ra, rb;
        if (I == J) { ra = fin * t->az[I].ra; rb = fin * t->az[I].rb; }
        else {
          float y = z + n.z * fin / edh;
          float h = 0.5f - sign * (z - I);
          float g = 0.5f + sign * (y - J);
          ra = h * t->az[I].ra + g * t->az[J].ra;
          rb = h * t->az[I].rb + g * t->az[J].rb;
          for (int i = I + sign; i != J; i += sign) { ra += t->az[i].ra; rb += t->az[i].rb; g_cnt.bfr_layers++; }
          float ff = edh / anz;
          ra *= ff; rb *= ff;
        }
        if (ra < 0) ra = 0;
        if (rb < 0) rb = 0;
        float dot = e->azx * n.x + e->azy * n.y;
        float sdt = sqrtf(1 - dot * dot);
        float cdt = fabsf(dot);
        const float* bf = e->bfr;
        float sx = sqrtf(ra) * mxf(0.f, bf[0] * expf(-bf[1] * powf(atanf(bf[3] * sdt), bf[2])));
        float sy = sqrtf(ra) * mxf(0.f, bf[4] * expf(-bf[5] * powf(atanf(bf[7] * sdt), bf[6])));
        float mx = rb * mxf(0.f, bf[8] * atanf(bf[11] * sdt * cdt) * expf(-bf[9] * sdt + bf[10] * cdt));
        float qx = e->azx - dot * n.x, qy = e->azy - dot * n.y, qz = -dot * n.z;
        if (dot < 0) { qx = -qx; qy = -qy; qz = -qz; }
        float qn = qx * qx + qy * qy + qz * qz;
        if (qn > 0) {
          float ff = 1 / sqrtf(qn);
          qx *= ff; qy *= ff; qz *= ff;
        } else { qx = 0; qy = 0; qz = 1; }
        float px = n.y * qz - n.z * qy, py = n.z * qx - n.x * qz, pz = n.x * qy - n.y * qx;
        float g1, g2;
        grnd2(&g1, &g2, s);
        float dnx = sx * g1 + mx;
        float dny = sy * g2;
        if (del <= hi) {  /* curved path within the segment */
          g_cnt.bfr_curved++;
          grnd2(&g1, &g2, s);
          /* the CPU build's rsqrtf is the textual macro 1/sqrtf (gpu/pro.cu:6), so this
             product becomes a division there: keep that rounding */
          float vnx = dnx + sx * g1 * 1 / sqrtf(3.f);
          float vny = dny + sy * g2 * 1 / sqrtf(3.f);
          vnx /= 2; vny /= 2;
          float den = vnx * vnx + vny * vny;
          float dnz = -den;
          den = 2 / (1 + den);
          vnx *= den; vny *= den; dnz *= den;
          float mxx = n.x + qx * vnx + px * vny + n.x * dnz;
          float myy = n.y + qy * vnx + py * vny + n.y * dnz;
          float mzz = n.z + qz * vnx + pz * vny + n.z * dnz;
          float rq = 1 / sqrtf(mxx * mxx + myy * myy + mzz * mzz);
          mxx *= rq; myy *= rq; mzz *= rq;
          del -= fin / 2;
          r.x += del * (mxx - n.x);
          r.y += del * (myy - n.y);
          r.z += del * (mzz - n.z);
        }
        dnx /= 2; dny /= 2;
        float den = dnx * dnx + dny * dny;
        float dnz = -den;
        den = 2 / (1 + den);
        dnx *= den; dny *= den; dnz *= den;
        n.x += qx * dnx + px * dny + n.x * dnz;
        n.y += qy * dnx + py * dny + n.y * dnz;
        n.z += qz * dnx + pz * dny + n.z * dnz;
        float rq = 1 / sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
        n.x *= rq; n.y *= rq; n.z *= rq;
      }
      if (SCA < XXX) {  /* scattering, gpu/pro.cu:838-887 */
        SCA = 0;
        float sf, g, gr;
        if (hole) { sf = e->SF; g = e->G; gr = e->GR; }
        else { sf = e->sf; g = e->g; gr = e->gr; }
        float xi = ppco_xrnd(s);
        if (xi > sf) {
          g_cnt.scatter_hg++;
          xi = (1 - xi) / (1 - sf);
          xi = 2 * xi - 1;
          if (g != 0) {
            float ga = (1 - g * g) / (1 + g * xi);
            xi = (ga * ga - sq(1 - g)) / (2 * g);
          }
        } else {
          g_cnt.scatter_sam++;
          xi /= sf;
          xi = 2 * (1 - powf(xi, gr));
        }
        if (xi < 0) xi = 0;
        else if (xi > 2) xi = 2;
        float k1 = t->az[J].k1, k2 = t->az[J].k2;
        float okz = k1 * k2;
        if (!hole) {
          float n1 = (e->azx * n.x + e->azy * n.y) * k1;
          float n2 = (-e->azy * n.x + e->azx * n.y) * k2;
          n.x = n1 * e->azx - n2 * e->azy;
          n.y = n1 * e->azy + n2 * e->azx;
          n.z /= okz;
          float rq = 1 / sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
          n.x *= rq; n.y *= rq; n.z *= rq;
        }
        rotate(xi, sqrtf(xi * (2 - xi)), &n, s);
        if (!hole) {
          float n1 = (e->azx * n.x + e->azy * n.y) / k1;
          float n2 = (-e->azy * n.x + e->azx * n.y) / k2;
          n.x = n1 * e->azx - n2 * e->azy;
          n.y = n1 * e->azy + n2 * e->azx;
          n.z *= okz;
          float rq = 1 / sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
          n.x *= rq; n.y *= rq; n.z *= rq;
        }
      }
    }
    if (TOT == 0) break;
    om = -1;
  }
  return steps;
}

/* photon index -> bunch (gpu/pro.cu:335 restated as a forward scan) */
static int find_bunch(const ppcb_bunch* b, int nb, uint64_t i, int* pj, uint64_t* pn) {
  while (i >= *pn && *pj + 1 < nb) { (*pj)++; *pn += b[*pj].num; }
  return *pj;
}

uint64_t ppco_run_reference_order(const ppco_tables* t, const ppcb_bunch* b, int nb, uint32_t num,
                                  uint32_t nthr, ppco_rng* stream, ppcb_hit* hits, uint64_t cap,
                                  ppco_pbuf* pbuf_out) {
  uint64_t nh = 0;
  ppco_pbuf f;
  for (uint32_t th = 0; th < nthr; th++) {
    int pj = -1;
    uint64_t pn = 0;
    for (uint32_t i = th; i < num; i += nthr) {
      find_bunch(b, nb, i, &pj, &pn);
      ppco_generate(t, &b[pj], stream, pbuf_out ? &pbuf_out[i] : &f);
    }
    for (uint32_t i = th; i < num; i += nthr) {
      if (!pbuf_out) return nh; /* reference order needs the phase-1 buffer */
      ppco_propagate(t, &pbuf_out[i], stream, hits, &nh, cap);
    }
  }
  return nh;
}

uint64_t ppco_run_fused(const ppco_tables* t, const ppcb_bunch* b, int nb, uint64_t num, uint32_t nthr,
                        uint64_t* rs, const uint32_t* rm, ppcb_hit* hits, uint64_t cap, uint64_t* steps) {
  uint64_t nh = 0, st = 0;
  for (uint32_t th = 0; th < nthr; th++) {
    ppco_rng s;
    s.x = (uint32_t)rs[th]; s.y = (uint32_t)(rs[th] >> 32); s.a = rm[th];
    int pj = -1;
    uint64_t pn = 0;
    for (uint64_t i = th; i < num; i += nthr) {
      ppco_pbuf f;
      find_bunch(b, nb, i, &pj, &pn);
      ppco_generate(t, &b[pj], &s, &f);
      st += ppco_propagate(t, &f, &s, hits, &nh, cap);
    }
    rs[th] = (uint64_t)s.x | ((uint64_t)s.y << 32);
  }
  if (steps) *steps = st;
  return nh;
}

void ppco_index_probe(const ppco_tables* t, const float* pos, int n, int32_t* oi, float* of) {
  const ppcb_params* e = t->p;
  for (int k = 0; k < n; k++) {
    const float* r = pos + 8 * k;
    const float* d = r + 4;
    float dz = e->dh;
    float zs = ppco_zshift(t, r, &dz);
    float z = r[2] - zs;
    z = (z - e->hmin) * e->rdh;
    int I = mni(mxi(rn(z), 0), e->size - 1);
    int xlx, xhx, xly, xhy;
    cell_range(e, r[0], r[1], r[0] + d[3] * d[0], r[1] + d[3] * d[1], &xlx, &xhx, &xly, &xhy);
    int m = k % (e->nstr > 0 ? e->nstr : 1), n1 = 0, n2 = -1;
    if (e->nstr > 0) {
      float z1 = r[2], z2 = r[2] + d[3] * d[2];
      dom_window(&t->sc[m], mnf(z1, z2), mxf(z1, z2), &n1, &n2);
    }
    int32_t* o = oi + 8 * k;
    o[0] = I; o[1] = xlx; o[2] = xhx; o[3] = xly; o[4] = xhy; o[5] = n1; o[6] = n2; o[7] = m;
    of[2 * k] = zs;
    of[2 * k + 1] = dz;
  }
}

/* The string loop of the DOM search (gpu/pro.cu:577-672) for one segment per row of `pos`
 * (x, y, z, t, nx, ny, nz, length): out[2k] counts the strings of the visited search cells
 * whose cylinder test passes (gpu/pro.cu:601-607), out[2k+1] those whose hole-ice column
 * test passes (gpu/pro.cu:655-660, taken as if hole ice were on at every time). */
void ppco_string_pass(const ppco_tables* t, const float* pos, int n, int32_t* out) {
  const ppcb_params* e = t->p;
  for (int k = 0; k < n; k++) {
    const float* r = pos + 8 * k;
    const float* d = r + 4;
    const float sca = d[3];
    int pass = 0, hole = 0;
    int xlx, xhx, xly, xhy;
    cell_range(e, r[0], r[1], r[0] + sca * d[0], r[1] + sca * d[1], &xlx, &xhx, &xly, &xhy);
    for (int i = xlx, j = xly; i <= xhx && j <= xhy; (++j <= xhy) ? 0 : (j = xly, i++)) {
      for (unsigned short q = t->is[i * PPCB_CY + j]; q != 0x8000;) {
        unsigned short m = t->ls[q];
        const ppcb_line* sl = &t->sc[m & 0x7fff];
        q = (m & 0x8000) ? 0x8000 : q + 1;
        float b = 0, c = 0, dr;
        dr = sl->x - r[0]; b += d[0] * dr; c += dr * dr;
        dr = sl->y - r[1]; b += d[1] * dr; c += dr * dr;
        float np = 1 - d[2] * d[2];
        float D = b * b - (c - sl->r * sl->r) * np;
        if (D >= 0) {
          D = sqrtf(D);
          if (b + D >= 0 && b - D <= sca * np) pass++;
        }
        if (e->hr > 0) {
          float DH = b * b - (c - e->hr2) * np;
          if (DH > 0) {
            DH = sqrtf(DH);
            if (b + DH >= 0 && b - DH <= sca * np) hole++;
          }
        }
      }
    }
    out[2 * k] = pass;
    out[2 * k + 1] = hole;
  }
}

