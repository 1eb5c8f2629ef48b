// Drop-in C++ API of the photon propagator, namespace xppc.
//
// This is the interface llh/DirectFit links against (the reference declares it in
// llh/ppc.h:1-113 and defines it in gpu/ppc.cu + gpu/f2k.cxx under -DXLIB).  Names,
// signatures, record layouts and ordering operators are kept identical so that a
// program compiled against the reference header links against libxppc.so from this
// package unchanged.  Each declaration cites the reference
// definition it replaces.
#ifndef PPC_B200_XPPC_H
#define PPC_B200_XPPC_H

#include <cmath>
#include <cstddef>
#include <map>
#include <utility>
#include <vector>

namespace xppc {

float xrnd();                       // host uniform (0,1], gpu/f2k.cxx:1-6
float grnd();                       // host Gaussian, gpu/f2k.cxx:8-10

void start();                       // gpu/ppc.cu:481-483
void stop();                        // gpu/ppc.cu:485-488
void choose(int);                   // gpu/ppc.cu:490-508 (-1: every GPU)
void ini();                         // gpu/ppc.cu:330-361
void fin();                         // gpu/ppc.cu:398-402
void eout();                        // gpu/f2k.cxx:536-541

void flone(unsigned long long);     // gpu/f2k.cxx:586-588

size_t getMaxBunchSize();           // gpu/ppc.cu:368
size_t getWorkgroupSize();          // gpu/ppc.cu:370-386
float getTotalDeviceTime();         // gpu/ppc.cu:388-395

// track identity echoed with every hit, gpu/f2k.cxx:170-181
struct mcid : std::pair<int, unsigned long long> {
  int frame;
  double t0;
  bool operator<(const mcid& o) const {
    if (frame != o.frame) return frame < o.frame;
    if (first != o.first) return first < o.first;
    if (second != o.second) return second < o.second;
    return t0 < o.t0;
  }
};

// optical module: radius, flattening, position (gpu/ini.cxx:42-45)
struct DOM {
  float R, F;
  float r[3];
};

// string / module key (gpu/ini.cxx:47-61)
struct ikey {
  int str, dom;
  bool isinice() const { return str > 86 || (str > 0 && dom >= 1 && dom <= 60); }
  bool operator<(const ikey& o) const { return str == o.str ? dom < o.dom : str < o.str; }
  bool operator!=(const ikey& o) const { return str != o.str || dom != o.dom; }
};

// per-module geometry record used by llh (llh/ppc.h:52-64)
struct xgeo {
  int num;
  int type;
  float r[3];
  float hv, rde;
  xgeo() : num(0), type(0), hv(NAN), rde(NAN) { r[0] = r[1] = r[2] = 0; }
};

struct OM : DOM, ikey {};
extern std::vector<OM> i3oms;                                   // gpu/ini.cxx:63-64

extern std::map<ikey, int> omts;                                // gpu/ini.cxx:357
extern std::map<ikey, float> hvs;                               // gpu/ini.cxx:362
extern std::map<ikey, std::pair<float, int> > rdes;             // gpu/ini.cxx:363

void initialize(float);                                         // gpu/ppc.cu:36
const DOM& flset(int, int);                                     // gpu/f2k.cxx:630-759
const float* fldir();                                           // gpu/f2k.cxx:762-765
void flshift(float[], float[], float* = NULL);                  // gpu/f2k.cxx:590-628

// binned hit key, gpu/f2k.cxx:183-198
struct ihit {
  mcid track;
  ikey omkey;
  int pmt;
  float dir;
  float time;
  bool operator<(const ihit& o) const {
    // like the reference, tracks are told apart by their (first, second) pair only
    // (std::pair's !=); frame and t0 order tracks that differ in the pair
    const std::pair<int, unsigned long long>& a = track;
    const std::pair<int, unsigned long long>& b = o.track;
    if (a != b) return track < o.track;
    if (omkey != o.omkey) return omkey < o.omkey;
    if (pmt != o.pmt) return pmt < o.pmt;
    if (dir != o.dir) return dir < o.dir;
    return time < o.time;
  }
};

void set_res(float);                                            // gpu/f2k.cxx:202-204
void set_res(float, float);                                     // gpu/f2k.cxx:208-210

// photon at the module surface, gpu/f2k.cxx:218-220
struct pout {
  float r[4], n[4];
};

typedef std::map<ihit, std::vector<pout> > outz;
extern outz hitz;                                               // gpu/f2k.cxx:221
extern bool nextgen;                                            // gpu/ini.cxx:120

void efin();                                                    // gpu/f2k.cxx:544-546

void sett(float, float, float, std::pair<int, unsigned long long>, int, double = 0);  // gpu/f2k.cxx:548-552
void addp(float, float, float, float, float, float, int, float = 1);                   // gpu/f2k.cxx:484-504

void addp_clst(float, float, float, float, unsigned long long, float, float);          // gpu/f2k.cxx:507-518
void addp_mopo(float, float, float, float, float, float, float, float, float);         // gpu/f2k.cxx:520-528

}  // namespace xppc

#endif
