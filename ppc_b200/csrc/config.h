// Ice / geometry / wavelength configuration: parses the reference's input files
// (cfg.txt, icemodel.dat/.par/.bbl, geo-f2k, tilt.*, wv.*, rnd.txt, as.dat, om.*,
// eff-f2k, hvs-f2k, str-f2k, cx.dat, dx.dat) and builds the tables the propagation
// kernel reads.  Semantics follow gpu/ini.cxx:578-1700 (`ini::set`), including the
// environment overrides (OVSZ, BFRA/BFRB, HIFL, GECO, VTHK, WFLA, FLWL, ABSM, BFRM and
// the *DIR variables).  Errors throw ppcb::Error instead of calling exit().
#pragma once
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ppcb_types.h"
#include "strgrid.h"

namespace ppcb {

struct Error : std::runtime_error {
  int code;
  explicit Error(const std::string& m, int c = 1) : std::runtime_error(m), code(c) {}
};

struct Vec3 {
  float x[3];
  Vec3() { x[0] = 0; x[1] = 0; x[2] = 1; }
  float& operator[](int i) { return x[i]; }
  float operator[](int i) const { return x[i]; }
  float dot(const Vec3& q) const {
    float s = 0;
    for (int i = 0; i < 3; i++) s += x[i] * q.x[i];
    return s;
  }
};

struct OMKey {
  int str, dom;
  bool isinice() const { return str > 86 || (str > 0 && dom >= 1 && dom <= 60); }
  bool operator<(const OMKey& o) const { return str == o.str ? dom < o.dom : str < o.str; }
  bool operator!=(const OMKey& o) const { return str != o.str || dom != o.dom; }
};

// One geometry entry as read from geo-f2k.
struct GeoOM {
  ppcb_dom d;
  OMKey k;
  bool operator<(const GeoOM& o) const { return k < o.k; }
};

// Per-DOM host attributes used by the hit back end (gpu/ini.cxx:86-98).
struct OMName {
  OMKey k;
  int omt;     // module type (om.map), -1 = standard DOM
  int type;    // wavelength-acceptance variant (eff-f2k column 4)
  float rde, hv;
  float azi;   // cable azimuth (dx.dat), <0 unset
  Vec3 tilt;   // DOM axis (cx.dat)
};

// Sensor type: angular sensitivity and multi-PMT layout (gpu/ini.cxx:122-281).
struct SensorType {
  float area = 0, beta = 0, rde = 0, fx = 0, Rr = 0, Rz = 0, cable = 0;
  std::vector<Vec3> dirs;
  bool def = false;
  float ave = 0, mas = 0;
  std::vector<float> s;

  void load_angsens(const std::string& file);
  void add_dir(float th, float ph);
  float aS(float x) const;
  float f(float x) const;
  float xarea(float dot) const;
  void fraq(const std::vector<Vec3>& ico);
  // Returns the PMT index or -1; may add a transit-time delay to ht.
  int getPMT(Vec3 dir, Vec3 pos, Vec3 tilt, float rnd, float& ht, float ph,
             const std::function<float()>& xrnd) const;
};

// Wavelength acceptance of one (type, variant) class (gpu/ini.cxx:319-355).
struct WaveAcc {
  float rde = 0;
  std::vector<float> dat, sum, rat;
  int oms = 0;
  float rmax = 0;
  void addr(float r) { if (r > rmax) rmax = r; oms++; }
  float binf(float p) const;
};

// Wavelength grid (gpu/ini.cxx:283-317).
struct WaveGrid {
  bool swv = false;
  int num = 450;
  float bin, wmin = 250.f, wmax = 700.f;
  WaveGrid() { bin = (wmax - wmin) / num; }
  void ssw(float wva) { swv = true; num = 10; wmin = wva - 5.f; wmax = wva + 5.f; bin = (wmax - wmin) / num; }
  float wav(float i) const { return wmin + bin * i; }
  float np(float wv, float* ng = nullptr) const;
  float cherenkov(float wva) const;
  void read(WaveAcc& a, const std::vector<float>& qw, const std::vector<float>& qf,
            float blo = -1.f, float bhi = -1.f) const;
};

struct WaveSample { float w, i, f; };

class Config {
 public:
  // Loads everything.  `tables_dir` overrides PPCTABLESDIR when non-empty.
  void load(const std::string& tables_dir = "");
  // New per-layer be / ba (icemodel.dat columns 2-3, file order; null keeps): rebuilds absca.
  void set_ice(const float* be_new, const float* ba_new);

  // ---- kernel-facing tables (device image) ----
  ppcb_params p{};
  std::vector<ppcb_aniz> az;               // [size]
  std::vector<float> lr;                   // [LMAX]
  std::vector<uint16_t> ls;                // [NSTR]
  std::vector<uint16_t> is;                // [CX*CY]
  std::vector<int8_t> mcol;                // [CTX*CTY]
  std::vector<ppcb_line> sc;               // [NSTR]
  std::vector<float> lp;                   // [LMAX*LYRS*2]  (x = shift, y = slope)
  std::vector<float> absca;                // [WNUM*size*2]  (abs, sca) per wavelength, per layer
  std::vector<ppcb_wmeta> wmeta;           // [WNUM]
  std::vector<ppcb_dom> oms;               // [gsize]
  std::vector<uint32_t> rm;                // [rsize]
  std::vector<float> bfrt;                 // [(BFR_TAB+1)*4] birefringence functions of v = sqrt(1-|cos|)
  std::vector<float> wgrad;                // [WNUM*2] d sca/d be, d abs/d ba per wavelength bin
  // string-proximity table over sc (strgrid.h): geometry, groups, cell entries [nx*ny]
  StrGridParams sg{};
  std::vector<StrGroup> sg_groups;
  std::vector<uint16_t> sg_cells;

  // ---- host-side tables ----
  std::vector<OMName> names;               // [gsize]
  std::vector<GeoOM> i3oms;                // all entries of geo-f2k, sorted
  std::map<OMKey, int> omts;
  std::map<OMKey, float> hvs;
  std::map<OMKey, std::pair<float, int> > rdes;
  std::map<OMKey, Vec3> cx;
  std::map<OMKey, float> dx;
  std::map<int, std::pair<float, float> > strs;
  std::map<int, SensorType> types;
  std::map<std::pair<int, int>, WaveAcc> irdes;
  WaveAcc env;
  WaveGrid qwv;
  std::vector<Vec3> ico;
  std::vector<WaveSample> wvs;             // [WNUM]
  float eff = 1;                           // photons per metre ratio (ppm after load)
  unsigned int ovr = 1;                    // oversize area factor xR^2
  bool nextgen = false;

  // raw per-layer ice inputs (needed by the gradient path), original file order
  std::vector<float> dp, be, ba, td, k1v, k2v, rav, rbv;
  float ice_a = 0, ice_k = 0, ice_A = 0, ice_B = 0, ice_D = 0, ice_E = 0;
  float bble = 0, bblz = 0, bbly = 0;
  float arf = 0, srw = 0, srf = 1;

  std::string ppcdir, omdir, icedir, tiltdir, holeice;

 private:
  void fill_ice(int n, float wva);
  void build_strgrid();
  unsigned short sname(int n);
  std::map<int, unsigned short> sname_overflow_;
  unsigned short sname_next_ = 86 + 10 + 1;
};

}  // namespace ppcb
