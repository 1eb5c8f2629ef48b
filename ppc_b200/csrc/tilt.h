// Ice-layer tilt: depth shift of the layer isochrons at (x, y, z), gpu/pro.cu:168-264.
// One implementation for the kernel and the host tools.  Every operation is an IEEE
// round-to-nearest step without contraction (explicit intrinsics on the device; the host
// code is compiled with -ffp-contract=off), so the device and the host agree bit for bit
// and the result matches an IEEE build of the reference for identical positions.
//
// `Tab` supplies lr(i) (1-d map radii), mcol(x, y) (2-d map column, -1 = none) and
// lp(i, k) (shift and slope of map i at depth point k, as float2).
#pragma once
#include <vector_types.h>

#include "ppcb_types.h"

#if defined(__CUDACC__)
#define PPCB_HD __host__ __device__ __forceinline__
#else
#define PPCB_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define PPCB_ADD(a, b) __fadd_rn((a), (b))
#define PPCB_SUB(a, b) __fsub_rn((a), (b))
#define PPCB_MUL(a, b) __fmul_rn((a), (b))
#define PPCB_DIV(a, b) __fdiv_rn((a), (b))
#define PPCB_FLOOR_I(x) __float2int_rd(x)
#else
#include <cmath>
#define PPCB_ADD(a, b) ((a) + (b))
#define PPCB_SUB(a, b) ((a) - (b))
#define PPCB_MUL(a, b) ((a) * (b))
#define PPCB_DIV(a, b) ((a) / (b))
#define PPCB_FLOOR_I(x) ((int)floorf(x))
#endif

namespace ppcb {

PPCB_HD int tmin(int a, int b) { return b < a ? b : a; }
PPCB_HD int tmax(int a, int b) { return a < b ? b : a; }

// 1-d: interpolate between the two maps bracketing the distance along 225 deg
template <class Tab>
PPCB_HD float zshift_1d_t(const ppcb_params& d, const Tab& t, float rx, float ry, float rz, float& dz) {
  {
    float nr = PPCB_SUB(PPCB_ADD(PPCB_MUL(d.lnx, rx), PPCB_MUL(d.lny, ry)), d.r0);
    // first j >= 1 with nr < lr[j], or j = lnum-1.  The radii are non-decreasing (checked
    // when loaded), so that is 1 + #{k in [1, lnum-2] : !(nr < lr[k])}: a loop with the same
    // trip count for every thread (NaN counts as "not below", as in the search loop).
    int j = 1;
    if (d.lnum >= 2) {
      for (int k = 1; k < d.lnum - 1; k++) j += !(nr < t.lr(k));
    } else {
      for (; j < PPCB_LMAX; j++) if (nr < t.lr(j)) break;
      if (j >= PPCB_LMAX) j = PPCB_LMAX - 1;  // a single-map table would run off the end
    }
    float z = PPCB_MUL(PPCB_SUB(rz, d.lmin), d.lrdz);
    int i = j - 1, k = tmin(tmax(PPCB_FLOOR_I(z), 0), d.lpts);
    const float2 pi = t.lp(i, k), pj = t.lp(j, k);
    float dw = PPCB_SUB(t.lr(j), t.lr(i));
    float wx = PPCB_DIV(PPCB_SUB(nr, t.lr(i)), dw);
    float wy = PPCB_DIV(PPCB_SUB(t.lr(j), nr), dw);
    float qx = PPCB_ADD(PPCB_MUL(pj.x, wx), PPCB_MUL(pi.x, wy));
    float qy = PPCB_ADD(PPCB_MUL(pj.y, wx), PPCB_MUL(pi.y, wy));
    float r = PPCB_ADD(qx, PPCB_MUL(qy, PPCB_SUB(z, (float)k)));
    if (d.vthk != 0) dz = PPCB_DIV(dz, PPCB_SUB(1.f, PPCB_MUL(d.lrdz, qy)));
    return r;
  }
}

// 2-d: barycentric interpolation on the skewed map grid
template <class Tab>
PPCB_HD float zshift_2d_t(const ppcb_params& d, const Tab& t, float rx, float ry, float rz, float& dz) {
  {
    float qx = PPCB_ADD(PPCB_MUL(d.cb[0][0], rx), PPCB_MUL(d.cb[1][0], ry));
    float qy = PPCB_ADD(PPCB_MUL(d.cb[0][1], rx), PPCB_MUL(d.cb[1][1], ry));
    qx = PPCB_DIV(PPCB_SUB(qx, d.mmin[0]), d.mstp[0]);
    qy = PPCB_DIV(PPCB_SUB(qy, d.mmin[1]), d.mstp[1]);
    {  // extrapolation beyond the map edges, gpu/pro.cu:200-214
      float x = qx, y = qy, xy;
      const int n0 = d.mnum[0] - 1, n1 = d.mnum[1] - 1, c0 = d.mcut[0] - 1, c1 = d.mcut[1] - 1;
      const float N0 = n0, N1 = n1, C0 = c0, C1 = c1;
      if (y < 0) if (PPCB_SUB(x, y) > 0 && x <= C0) { x = PPCB_DIV(PPCB_MUL(PPCB_SUB(x, y), C0), PPCB_SUB(C0, y)); y = 0; }
      if (x < 0) if (PPCB_SUB(y, x) >= 0 && y < C1) { y = PPCB_DIV(PPCB_MUL(PPCB_SUB(y, x), C1), PPCB_SUB(C1, x)); x = 0; }
      if (y > N1) if (x >= (float)(n1 - c1) && PPCB_SUB(y, x) > (float)(n1 - n0)) {
        x = PPCB_ADD((float)(n1 - c1), PPCB_DIV(PPCB_MUL((float)(n0 - (n1 - c1)), PPCB_SUB(x, (float)(n1 - c1))),
                                                PPCB_SUB(PPCB_SUB(y, (float)(n1 - n0)), (float)(n1 - c1))));
        y = N1;
      }
      if (x > N0) if (y > (float)(n0 - c0) && PPCB_SUB(y, x) <= (float)(n1 - n0)) {
        y = PPCB_ADD((float)(n0 - c0), PPCB_DIV(PPCB_MUL((float)(n1 - (n0 - c0)), PPCB_SUB(y, (float)(n0 - c0))),
                                                PPCB_SUB(PPCB_SUB(x, (float)(n0 - n1)), (float)(n0 - c0))));
        x = N0;
      }
      if (PPCB_SUB(y, x) > C1) if (y >= C1 && x < (float)(n1 - c1)) {
        xy = PPCB_SUB(PPCB_SUB(y, x), C1);
        xy = PPCB_ADD(C1, PPCB_DIV(PPCB_MUL(PPCB_ADD(PPCB_SUB(PPCB_ADD(x, y), C1), xy), (float)(n1 - c1)),
                                   PPCB_ADD((float)(n1 - c1), xy)));
        x = PPCB_SUB(xy, C1) / 2; y = PPCB_ADD(xy, C1) / 2;
      }
      if (PPCB_SUB(x, y) > C0) if (x > C0 && y <= (float)(n0 - c0)) {
        xy = PPCB_SUB(PPCB_SUB(x, y), C0);
        xy = PPCB_ADD(C0, PPCB_DIV(PPCB_MUL(PPCB_ADD(PPCB_SUB(PPCB_ADD(x, y), C0), xy), (float)(n0 - c0)),
                                   PPCB_ADD((float)(n0 - c0), xy)));
        x = PPCB_ADD(xy, C0) / 2; y = PPCB_SUB(xy, C0) / 2;
      }
      qx = x; qy = y;
    }
    int qnx0 = tmin(tmax(PPCB_FLOOR_I(qx), 0), d.mnum[0]);
    int qny0 = tmin(tmax(PPCB_FLOOR_I(qy), 0), d.mnum[1]);
    float qrx0 = PPCB_SUB(qx, (float)qnx0), qry0 = PPCB_SUB(qy, (float)qny0);
    float qrx, qry;
    int qnx, qny;
    if (qrx0 > qry0) { qrx = qrx0; qry = qry0; qnx = qnx0 + 1; qny = qny0; }
    else { qrx = qry0; qry = qrx0; qnx = qnx0; qny = qny0 + 1; }
    int cx = t.mcol(qnx0, qny0);
    int cy = t.mcol(qnx, qny);
    int cz = t.mcol(qnx0 + 1, qny0 + 1);
    float wx = PPCB_SUB(1.f, qrx), wy = PPCB_SUB(qrx, qry), wz = qry;
    float z = PPCB_MUL(PPCB_SUB(rz, d.lmin), d.lrdz);
    int k = tmin(tmax(PPCB_FLOOR_I(z), 0), d.lpts);
    float ax = 0, ay = 0;
    if (cx >= 0) { const float2 p = t.lp(cx, k); ax = PPCB_ADD(ax, PPCB_MUL(p.x, wx)); ay = PPCB_ADD(ay, PPCB_MUL(p.y, wx)); }
    if (cy >= 0) { const float2 p = t.lp(cy, k); ax = PPCB_ADD(ax, PPCB_MUL(p.x, wy)); ay = PPCB_ADD(ay, PPCB_MUL(p.y, wy)); }
    if (cz >= 0) { const float2 p = t.lp(cz, k); ax = PPCB_ADD(ax, PPCB_MUL(p.x, wz)); ay = PPCB_ADD(ay, PPCB_MUL(p.y, wz)); }
    float r = PPCB_ADD(ax, PPCB_MUL(ay, PPCB_SUB(z, (float)k)));
    if (d.vthk != 0) dz = PPCB_DIV(dz, PPCB_SUB(1.f, PPCB_MUL(d.lrdz, ay)));
    return r;
  }
}

template <class Tab>
PPCB_HD float zshift_t(const ppcb_params& d, const Tab& t, float rx, float ry, float rz, float& dz) {
  if (d.tmod == 1) return zshift_1d_t(d, t, rx, ry, rz, dz);
  if (d.tmod == 2) return zshift_2d_t(d, t, rx, ry, rz, dz);
  return 0;
}

}  // namespace ppcb
