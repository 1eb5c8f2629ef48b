// String-proximity table: an exact, conservative pre-test for the DOM search.
//
// The reference's DOM search (gpu/pro.cu:577-672) visits, for every propagation step, the
// strings of the skewed search cells (about 62 m wide) that the step's horizontal extent
// touches and tests each string's cylinder against the step's segment.  On the full
// detector that is about two strings per step, while fewer than 0.2% of steps pass a
// cylinder test at all.  This table lets a step prove, with one shared-memory load and a
// distance test (a cylinder test near a string), that the search would find nothing:
//
//   * lines that share an axis (a string split into several lines, axes equal up to
//     rounding) form a group, whose disc covers each line's search disc (the search radius
//     already includes the hole-ice radius);
//   * a square grid covers the groups' horizontal footprint plus `margin` on every side;
//     each cell holds the group nearest to it and a lower bound, in units of kSgClearUnit
//     metres, on the distance from any point of the cell to the widened disc
//     (radius + kReachPad) of every OTHER group.
//
// A step from r, of length sca along n, reaches horizontally no farther than
// L = sca sqrt(1 - nz^2) from r.  If L is below the cell's clearance no other group can be
// reached.  The nearest group is then out of reach when r lies farther than rw + sca from
// its axis (a ball test, no square root); otherwise it is tested with the reference's
// cylinder arithmetic on the widened radius.  A string that the reference's test accepts is within its radius of the
// segment, so the widened test accepts it too: the widening changes the test's
// discriminant by 0.09 np m^2, against a rounding of at most 1e-3 np m^2 for strings
// within 120 m of the segment.  When nothing can be reached the reference's search would
// find nothing -- no DOM candidate, no hole-ice column -- so skipping it leaves the step
// bit for bit unchanged.  Otherwise (and for near-vertical or non-finite steps) the
// reference's search runs in full, in its own order.
#pragma once
#include <stdint.h>
#if !defined(__CUDA_ARCH__)
#include <cmath>
#endif

#include "ppcb_types.h"

#if defined(__CUDACC__)
#define PPCB_SG_HD __host__ __device__ __forceinline__
#else
#define PPCB_SG_HD inline
#endif

namespace ppcb {

constexpr float kReachPad = 0.05f;      // [m] added to every group's radius
constexpr float kSgClearUnit = 0.5f;    // [m] clearance quantum of a cell entry (8 bits)
constexpr int kSgMaxCells = 16384;      // cells (two bytes each): 32 KiB of shared memory
constexpr float kSgMinNp = 1e-4f;       // 1 - nz^2 below this: full search

// Table geometry (a kernel parameter).  Point (x, y) lies in cell
// (floor(x inv + ou), floor(y inv + ov)), whose square on the host is widened by a
// millimetre on every side to cover the rounding of that product.  A point outside the
// grid is at least sqrt(margin2) from every group's widened disc.
struct StrGridParams {
  float ou, ov, inv, margin2;  // -origin / cell size, 1 / cell size, squared distance bound outside the grid
  int32_t nx, ny, on, pad_;    // cells per row, rows; on = 0: no strings (nothing to search)
};

// One group as the pre-test reads it: axis and widened radius.  After the groups the
// table holds a sentinel (an axis at 1e30 m, never within reach), the entry of a cell
// that has no nearest group.
struct StrGroup {
  float x, y, rw, pad_;
};

// The reference's cylinder test (gpu/pro.cu:601-607) on the widened radius: true when the
// segment from (rx, ry) along (nx, ny) (np = 1 - nz^2 >= kSgMinNp) of length sca may meet
// the group's cylinder.
PPCB_SG_HD bool sg_group_near(const StrGroup& G, float rx, float ry, float nx, float ny, float np, float sca) {
  const float dx = G.x - rx, dy = G.y - ry;
  const float c = dx * dx + dy * dy;
  const float b = nx * dx + ny * dy;
  const float D = b * b - (c - G.rw * G.rw) * np;
  if (!(D >= 0)) return !(D < 0);  // NaN: may reach
  const float q = sqrtf(D);
  return b + q >= -0.01f && b - q <= sca * np + 0.01f;
}

// Whether the step may reach a string's cylinder (the full search must run).  `Tab`
// supplies cell(k) (the 16-bit cell entry: group in the low byte, clearance in the high
// byte) and group(m).  Host and device evaluate it with the same IEEE operations.
template <class Tab>
PPCB_SG_HD bool sg_may_reach(const StrGridParams& g, const Tab& t, float rx, float ry, float nx, float ny, float nz,
                             float sca) {
  if (!g.on) return false;
  // Near-vertical steps go to the full search: there 1 - nz^2 rounds to (nearly) zero and
  // the reference's cylinder test accepts strings at any distance (its discriminant is
  // b^2 - (c - r^2) np), which matters when hole ice is on (gpu/pro.cu:655-669).  About
  // one step in 2e4 of an isotropic photon is that steep.
  const float np = 1 - nz * nz;
  if (!(np >= kSgMinNp)) return true;
  const float L2 = sca * sca * np;  // squared horizontal reach of the step
#if defined(__CUDA_ARCH__)
  const int iu = __float2int_rd(fmaf(rx, g.inv, g.ou)), iv = __float2int_rd(fmaf(ry, g.inv, g.ov));
#else
  const float fu = std::floor(std::fma(rx, g.inv, g.ou)), fv = std::floor(std::fma(ry, g.inv, g.ov));
  const int iu = fu >= 0 && fu < (float)g.nx ? (int)fu : -1, iv = fv >= 0 && fv < (float)g.ny ? (int)fv : -1;
#endif
  if (!((unsigned)iu < (unsigned)g.nx && (unsigned)iv < (unsigned)g.ny))  // outside the grid (or NaN)
    return !(L2 < g.margin2);
  const uint32_t e = t.cell(iv * g.nx + iu);
  const float clear = (float)(e >> 8) * kSgClearUnit;
  if (!(L2 < clear * clear)) return true;  // another group may be within reach
  const StrGroup& G = t.group((int)(e & 0xff));
  const float dx = G.x - rx, dy = G.y - ry, w = G.rw + sca;
  if (dx * dx + dy * dy > w * w) return false;  // the nearest axis is farther than rw + sca
  return sg_group_near(G, rx, ry, nx, ny, np, sca);
}

}  // namespace ppcb
