// Configuration loader.  Each block names the part of gpu/ini.cxx it restates; the
// arithmetic keeps the reference's float/double promotions so that the tables come
// out bit-identical to the reference's host code compiled the same way (IEEE float:
// -O2 -ffp-contract=off, no fast-math, on both sides).
#include "config.h"

#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>

// The reference brings std:: into scope (gpu/ppc.cu:26), so cos(float), exp(float), ...
// resolve to the float overloads; the same lookup is kept here.
using namespace std;

namespace ppcb {

static const float kDoma = PPCB_FPI * PPCB_OMR * PPCB_OMR;  // DOM cross-section [m^2]
static const float kOmav = 0.335822;                        // average DOM angular sensitivity
static const float kDppm = 2450.08;                         // photons per metre, nominal DOM
static const float kFcv = PPCB_FPI / 180.f;
static const float kZoff = 1948.07;

static std::string env_str(const char* name) {
  const char* v = getenv(name);
  return v ? std::string(v) : std::string();
}

static void note(const std::string& s) {
  if (!getenv("PPCB_QUIET")) std::cerr << s << std::endl;
}

// ---------------------------------------------------------------- sensor types
// gpu/ini.cxx:133-159 (angular sensitivity file, e.g. as.dat)
void SensorType::load_angsens(const std::string& file) {
  def = true; mas = 1; ave = 0;
  area = 1; beta = 0.33f; Rr = PPCB_OMR; Rz = PPCB_OMR; cable = 0;
  std::ifstream in(file.c_str());
  if (in.fail()) throw Error("Could not open file " + file);
  float aux;
  if (in >> aux) mas = aux;
  while (in >> aux) s.push_back(aux);
  if (s.empty()) s.push_back(1.f);
  if (mas > 0) {
    ave = s[0];
    for (unsigned int i = 2; i < s.size(); i += 2) ave += s[i] / i;
  } else {
    ave = (1 - s[0]) / 2;
  }
  if (!(ave > 0)) throw Error("File " + file + " did not contain valid data");
  ave = kOmav;  // the reference keeps the nominal average for compatibility
  rde = (mas > 0 ? mas : 1.f) / (kDoma * ave);
}

// gpu/ini.cxx:161-167
void SensorType::add_dir(float th, float ph) {
  float ct = cos(th * kFcv), st = sin(th * kFcv);
  float cp = cos(ph * kFcv), sp = sin(ph * kFcv);
  Vec3 d;
  d[0] = st * cp; d[1] = st * sp; d[2] = ct;
  dirs.push_back(d);
}

// gpu/ini.cxx:169-188
float SensorType::aS(float x) const {
  float al = acos(x);
  return al - sin(2 * al) / 2;
}

float SensorType::f(float x) const {
  if (beta < -1) return sqrt(1 - x * x);
  float sum = x > 0 ? x : 0;
  if (beta < 1) {
    float y = sqrt(1 - x * x) / beta;
    if (y > 1) {
      y = 1 / y;
      float c = 1 - beta * beta;
      sum += (aS(y) / c - aS(y * fabs(x) / sqrt(c)) * fabs(x)) / PPCB_FPI;
    }
  }
  return sum;
}

// gpu/ini.cxx:190-192
float SensorType::xarea(float dot) const {
  return Rz > 0 ? PPCB_FPI * Rr * sqrt(Rz * Rz - dot * dot * (Rz * Rz - Rr * Rr))
                : -4 * Rr * Rz * sqrt(1 - dot * dot);
}

// gpu/ini.cxx:194-208
void SensorType::fraq(const std::vector<Vec3>& icod) {
  if (def) return;
  float fr_flat = 0, sum_ave = 0;
  for (const Vec3& i : icod) {
    float tot = 0;
    for (const Vec3& j : dirs) tot += f(i.dot(j));
    float fra = xarea(i[2]);
    fra = fra > 0 ? tot / fra : 0;
    if (fr_flat < fra) fr_flat = fra;
    sum_ave += tot;
  }
  sum_ave /= icod.size();
  fx = fr_flat;
  rde = area * fr_flat / sum_ave;
}

// gpu/ini.cxx:210-280
int SensorType::getPMT(Vec3 dir, Vec3 pos, Vec3 tilt, float rnd, float& ht, float ph,
                       const std::function<float()>& xrnd) const {
  if (beta == -2) {  // wavelength-shifting tube: PMT at either end, with transit delay
    const float cn = 0.299792458 / 1.46;
    const float absl = 3.0 / cn;
    const float att = 0.678;
    const float cut = 0.01;
    const float tau = 1.6;
    const float h = 0.76;
    const float a = h / (1 - exp(-h / att));
    float z = Rr * pos[2];
    z *= h / fabs(2 * Rz);
    int i = rnd - 0.5 < z / (2 * a) ? 1 : 0;
    z = i > 0 ? h / 2 - z : h / 2 + z;
    float d = (z / h) * (1 - z / (2 * a)) / (1 - h / (2 * a));
    z = -att * log(1 - d * (1 - exp(-h / att)));
    if (z < cut) z = cut;
    float x = log(z), dt;
    float s = exp(((0.0034112 * x + 0.041727) * x + 0.45550) * x - 1.9188);
    float g = exp(((0.0012658 * x + 0.017228) * x - 0.012750) * x + 0.20924);
    do {
      dt = s * sqrt(2 * g * pow(1 - xrnd(), 1 / (1 - g)) - 1);
    } while (dt > -absl * log(xrnd()));
    dt += z / cn - tau * log(xrnd());
    ht += dt;
    return i;
  } else if (def) {
    bool flag;
    if (mas > 0) {
      float sum;
      {
        float x = dir.dot(tilt);
        float y = 1;
        sum = s[0];
        for (unsigned int i = 1; i < s.size(); i++) { y *= x; sum += s[i] * y; }
      }
      flag = mas * rnd < sum;
    } else {
      flag = pos.dot(tilt) > s[0];
    }
    return flag ? 0 : -1;
  } else {
    if (ph >= 0) {
      ph -= cable;
      float cp = cos(kFcv * ph);
      float sp = sin(kFcv * ph);
      float nx = dir[0] * cp + dir[1] * sp;
      float ny = dir[1] * cp - dir[0] * sp;
      dir[0] = nx; dir[1] = ny;
    }
    float crx = fx * xarea(dir[2]);
    unsigned int k = 0;
    float tot = 0;
    for (auto j = dirs.begin(); j != dirs.end(); ++j, k++) {
      tot += f(-dir.dot(*j)) / crx;
      if (tot > rnd) break;
    }
    return k < dirs.size() ? (int)k : -1;
  }
}

// ---------------------------------------------------------------- wavelengths
// gpu/ini.cxx:333-336: inverse of the cumulative acceptance, in wavelength-bin units
float WaveAcc::binf(float pv) const {
  int i, j = 0;
  while (sum[++j] <= 0) {}
  j--;
  while (sum[++j] < pv) {}
  i = j - 1;
  return i + (sum[j] > sum[i] ? (pv - sum[i]) / (sum[j] - sum[i]) : 0);
}

// gpu/ini.cxx:301-305 (phase and group refractive index of ice)
float WaveGrid::np(float wv, float* ng) const {
  float npv = 1.55749 - wv * (1.57988 - wv * (3.99993 - wv * (4.68271 - 2.09354 * wv)));
  if (ng != nullptr) *ng = npv * (1 + 0.227106 - wv * (0.954648 - wv * (1.42568 - 0.711832 * wv)));
  return npv;
}

// gpu/ini.cxx:307-316
float WaveGrid::cherenkov(float wva) const {
  if (swv) return 1 / (wmax - wmin);
  const float c = PPCB_FPI * 0.2 / 137.03599911;
  float wv = wva * 1.e-3, n = np(wv);
  return c * (1 - 1 / (n * n)) / (wv * wv);
}

// gpu/ini.cxx:338-354: resample (qw, qf) onto the wavelength grid
void WaveGrid::read(WaveAcc& a, const std::vector<float>& qw, const std::vector<float>& qf,
                    float blo, float bhi) const {
  a.dat.clear();
  int k = 0, n = qw.size();
  float wlo = qw[0] - (blo < 0 ? qw[1] - qw[0] : blo);
  float whi = qw[n - 1] + (bhi < 0 ? qw[n - 1] - qw[n - 2] : bhi);
  float w1 = wlo, w2 = qw[0], f1 = 0, f2 = qf[0];
  for (float w = wmin + bin / 2; w < wmax; w += bin) {
    while (k < n && qw[k] < w) {
      w1 = w2; f1 = f2; k++;
      if (k < n) { w2 = qw[k]; f2 = qf[k]; }
      else { w2 = whi; f2 = 0; }
    }
    a.dat.push_back(wlo < w && w < whi ? (f1 * (w2 - w) + f2 * (w - w1)) / (w2 - w1) : 0);
  }
}

// gpu/ini.cxx:1677-1691: absorption and scattering of wavelength bin n in every layer,
// plus the derivatives the gradient needs: d sca / d be = l_a / (1 - g) and
// d abs / d ba = D l_k (per wavelength; the same for every layer).
void Config::fill_ice(int n, float wva) {
  const float wv0 = 400;
  const float a = ice_a, k = ice_k, A = ice_A, B = ice_B, D = ice_D, E = ice_E;
  const int size = p.size;
  float l_a = pow(wva / wv0, -a);
  float l_k = pow(wva / wv0, -k);
  float AB0 = A * exp(-B / wv0);
  float ABl = A * exp(-B / wva);
  for (int i = 0; i < size; i++) {
    int j = size - 1 - i;
    float bbl = bble > 0 ? dp[j] < bblz && dp[j] < bbly ? bble * (1 - dp[j] / bblz) * (1 - dp[j] / bbly) : 0 : 0;
    float sca = (bbl + be[j] * l_a - rav[j] * p.sum * (srf + srw * l_a)) / (1 - p.g);
    float abs = (D * ba[j] + E) * l_k + (ABl - arf * AB0 * l_k) * (1 + 0.01 * td[j]);
    if (sca > 0 && abs > 0) {
      absca[((size_t)n * size + i) * 2 + 0] = abs;
      absca[((size_t)n * size + i) * 2 + 1] = sca;
    } else throw Error("Invalid value of ice parameter, cannot proceed");
  }
  wgrad[n * 2 + 0] = l_a / (1 - p.g);
  wgrad[n * 2 + 1] = D * l_k;
}

// New per-layer scattering (be) and absorption (ba) coefficients at 400 nm, file order
// (icemodel.dat rows); null keeps the current values.  Rebuilds the per-wavelength table.
void Config::set_ice(const float* be_new, const float* ba_new) {
  const int size = p.size;
  std::vector<float> be0 = be, ba0 = ba;
  for (int j = 0; j < size; j++) {
    if (be_new) be[j] = be_new[j];
    if (ba_new) ba[j] = ba_new[j];
  }
  try {
    for (int n = 0; n < PPCB_WNUM; n++) fill_ice(n, wvs[n].w);
  } catch (...) {
    be = be0; ba = ba0;
    for (int n = 0; n < PPCB_WNUM; n++) fill_ice(n, wvs[n].w);
    throw;
  }
}

// gpu/ini.cxx:538-551: string label, DeepCore strings split at DOM 10
unsigned short Config::sname(int n) {
  const OMName& s = names[n];
  if (s.k.str > 86) {
    auto it = sname_overflow_.find(s.k.str);
    if (it == sname_overflow_.end()) {
      if (sname_next_ >= 0x8000) throw Error("Number of string labels exceeds capacity of 32768");
      sname_overflow_.insert(std::make_pair(s.k.str, sname_next_++));
    }
    return sname_overflow_[s.k.str];
  }
  return (unsigned short)((s.k.str > 78 && s.k.dom > 10) ? s.k.str + 10 : s.k.str);
}

// Reads "depth v1 .. vN" records (possibly several per line), gpu/ini.cxx:1212-1222.
static void read_depth_table(std::ifstream& in, int lnum, std::vector<float>& ds,
                             std::vector<std::vector<float> >& lp) {
  std::vector<float> pts(lnum);
  lp.assign(lnum, std::vector<float>());
  std::string line;
  while (getline(in, line)) {
    std::stringstream str(line);
    float depth;
    while (str >> depth) {
      int i = 0;
      while (str >> pts[i++]) if (i >= lnum) break;
      if (i != lnum) break;
      ds.push_back(depth);
      for (i = 0; i < lnum; i++) lp[i].push_back(pts[i]);
    }
  }
}

void Config::load(const std::string& tables_dir) {
  *this = Config();
  p.hifl = 0;

  // directories, gpu/ini.cxx:584-625
  {
    const char* e = getenv("PPCTABLESDIR");
    if (!tables_dir.empty()) ppcdir = tables_dir + "/";
    else if (e) ppcdir = std::string(e) + "/";
    else if ((e = getenv("I3_SRC"))) ppcdir = std::string(e) + "/ppc/resources/ice/";
    note("Configuring ppc in \"" + ppcdir + "\"");
    omdir = getenv("NEXTGENDIR") ? env_str("NEXTGENDIR") + "/" : ppcdir;
    icedir = getenv("ICEMODELDIR") ? env_str("ICEMODELDIR") + "/" : ppcdir;
    tiltdir = getenv("TILTMODELDIR") ? env_str("TILTMODELDIR") + "/" : icedir;
    holeice = getenv("PPCHOLEICE") ? env_str("PPCHOLEICE") : ppcdir + "as.dat";
  }

  float dk1, dk2, dkz;
  // cfg.txt, gpu/ini.cxx:629-729
  {
    std::ifstream in((icedir + "cfg.txt").c_str());
    if (in.fail()) throw Error("Could not open file cfg.txt");
    std::string line;
    float aux;
    std::vector<float> v;
    while (getline(in, line)) if (sscanf(line.c_str(), "%f", &aux) == 1) v.push_back(aux);
    if (getenv("OVSZ")) {
      float ovsz = atof(getenv("OVSZ"));
      if (v.size() >= 1) v[0] = ovsz;
    }
    if (v.size() < 4) throw Error("File cfg.txt did not contain valid data");
    int xR = lroundf(v[0]);
    p.xR = xR; ovr *= xR * xR;
    eff = v[1]; p.sf = v[2]; p.g = v[3]; p.gr = (1 - p.g) / (1 + p.g);
    if (v.size() < 12) { p.SF = p.sf; p.G = p.g; p.GR = p.gr; }
    else { p.SF = v[10]; p.G = v[11]; p.GR = (1 - p.G) / (1 + p.G); }
    if (v.size() >= 10) {
      float xH = v[7], hS = v[8], hA = v[9];
      p.hr = PPCB_OMR * xH; p.hr2 = p.hr * p.hr; p.hs = 1 / (hS * (1 - p.G)); p.ha = 1 / hA;
    } else { p.hr = 0; p.hr2 = 0; p.hs = 0; p.ha = 0; }
    if (v.size() >= 7) {
      const float thx = v[4];
      p.azx = cos(kFcv * thx); p.azy = sin(kFcv * thx);
      dk1 = exp(v[5]); dk2 = exp(v[6]); dkz = 1 / (dk1 * dk2);
    } else { dk1 = 1; dk2 = 1; dkz = 1; p.azx = 1; p.azy = 0; }
    (void)dkz;
    if (v.size() >= 15) {
      p.k1 = exp(v[12]); p.k2 = exp(v[13]); p.kz = exp(v[14]);
      if (p.k1 >= p.k2 && p.k2 == p.kz) {
        float r = p.k1 / p.k2;
        float s = sqrt(r * r - 1);
        r = (s > PPCB_XXX ? log(r + s) / s : 1 + s / 2) / p.k2;
        p.k1 *= r; p.k2 *= r; p.kz *= r;
      }
    } else { p.k1 = 1; p.k2 = 1; p.kz = 1; }
    p.fr = v.size() >= 16 ? v[15] : 1;
    if (v.size() >= 28) {
      for (int i = 0; i < 12; i++) p.bfr[i] = v[16 + i];
      const char* A = getenv("BFRA");
      float bfra = A == nullptr ? 1.0 : atof(A);
      const char* B = getenv("BFRB");
      float bfrb = B == nullptr ? 1.0 : atof(B);
      for (int i = 0; i < 12; i += 4) p.bfr[i] *= i < 8 ? sqrt(bfra) : bfra * bfrb;
      float step = 0.01, sum = 0;
      for (float x = step / 2; x < 1; x += step) {
        float y = sqrt(1 - x * x);
        float sx = std::max(0.f, p.bfr[0] * exp(-p.bfr[1] * pow(atan(p.bfr[3] * y), p.bfr[2])));
        float sy = std::max(0.f, p.bfr[4] * exp(-p.bfr[5] * pow(atan(p.bfr[7] * y), p.bfr[6])));
        float mx = std::max(0.f, p.bfr[8] * atan(p.bfr[11] * y * x) * exp(-p.bfr[9] * y + p.bfr[10] * x));
        sum += sx * sx + sy * sy + mx * mx;
      }
      sum *= step / 2;
      p.sum = sum;
    } else {
      p.sum = 0;
      for (int i = 0; i < 12; i++) p.bfr[i] = i % 4 < 1 ? 0 : 1;
    }
  }

  // multi-PMT sensor types, gpu/ini.cxx:731-761
  {
    std::ifstream in((omdir + "om.conf").c_str());
    if (!in.fail()) {
      std::string line;
      while (getline(in, line)) {
        int m;
        unsigned int n;
        SensorType t;
        float th, ph, other;
        int read = sscanf(line.c_str(), "%*s %d %f %f %f %f %d %f %f %f", &m, &t.area, &t.beta, &t.Rr,
                          &t.Rz, (int*)&n, &th, &ph, &other);
        t.cable = read >= 9 ? other : 0;
        if (read >= 8) {
          t.add_dir(th, ph);
          for (unsigned int i = 1; i < n && getline(in, line); i++)
            if (2 == sscanf(line.c_str(), "%f %f %f", &th, &ph, &other)) t.add_dir(th, ph);
          if (t.dirs.size() == n) types.insert(std::make_pair(m, t));
        }
      }
    }
    if (!types.empty()) {
      std::ifstream di((omdir + "om.dirs").c_str());
      if (!di.fail()) {
        std::string line;
        while (getline(di, line)) {
          Vec3 d;
          if (3 == sscanf(line.c_str(), "%*d %f %f %f", &d[0], &d[1], &d[2])) ico.push_back(d);
        }
      }
      if (ico.size() < 1) throw Error("Error: could not initialize an array of directions");
      nextgen = true;
      for (auto& j : types) j.second.fraq(ico);
    }
  }
  if (types.find(-1) == types.end()) types[-1].load_angsens(holeice);

  // random multipliers, gpu/ini.cxx:767-799
  {
    std::ifstream in((ppcdir + "rnd.txt").c_str());
    if (in.fail()) throw Error("Could not open file rnd.txt");
    std::vector<unsigned int> rx;
    std::string line;
    while (getline(in, line)) {
      std::stringstream str(line);
      unsigned int a;
      if (str >> a) rx.push_back(a);
    }
    if (rx.size() < 1) throw Error("File rnd.txt did not contain valid data");
    int size = rx.size();
    if (size > PPCB_MAXRND) size = PPCB_MAXRND;
    p.rsize = size;
    rm.assign(rx.begin(), rx.begin() + size);
  }

  // geometry, gpu/ini.cxx:801-818
  {
    std::ifstream in((ppcdir + "geo-f2k").c_str());
    if (!in.fail()) {
      GeoOM om;
      std::string mbid;
      unsigned long long omid;
      while (in >> mbid >> std::hex >> omid >> std::dec >> om.d.r[0] >> om.d.r[1] >> om.d.r[2] >> om.k.str >>
             om.k.dom) {
        om.d.R = PPCB_OMR; om.d.F = 1;
        om.d.r[2] += kZoff;
        i3oms.push_back(om);
      }
    }
  }
  {
    const char* h = getenv("HIFL");
    p.hifl = h == nullptr ? 0.f : atof(h);
  }
  // per-DOM position correction, gpu/ini.cxx:826-855
  {
    std::map<OMKey, std::pair<float, float> > geco;
    const char* bmp = getenv("GECO");
    if (bmp != nullptr) {
      OMKey om;
      float x, y, xH, hS;
      int num = sscanf(bmp, "%d %d %f %f %f %f", &om.str, &om.dom, &x, &y, &xH, &hS);
      if (num >= 4) geco[om] = std::make_pair(PPCB_OMR * x, PPCB_OMR * y);
      if (num >= 5) { p.hr = PPCB_OMR * xH; p.hr2 = p.hr * p.hr; }
      if (num >= 6) p.hs = 1 / (hS * (1 - p.G));
    }
    for (auto& i : i3oms) {
      auto j = geco.find(i.k);
      if (j != geco.end()) { i.d.r[0] += j->second.first; i.d.r[1] += j->second.second; }
    }
  }
  {
    std::ifstream in((ppcdir + "str-f2k").c_str());
    if (!in.fail()) {
      int str;
      float x, y;
      while (in >> str >> x >> y) strs[str] = std::make_pair(x, y);
    }
  }
  {
    std::ifstream in((ppcdir + "eff-f2k").c_str());
    if (!in.fail()) {
      int typ;
      OMKey om;
      float e;
      std::string line;
      while (getline(in, line)) {
        int num = sscanf(line.c_str(), "%d %d %f %d", &om.str, &om.dom, &e, &typ);
        if (num < 4) typ = 0;
        if (num >= 3 && om.isinice()) rdes.insert(std::make_pair(om, std::make_pair(e, typ)));
      }
    }
  }
  {
    std::ifstream in((omdir + "om.map").c_str());
    if (!in.fail()) {
      OMKey om;
      int m;
      while (in >> om.str >> om.dom >> m) if (om.isinice()) omts.insert(std::make_pair(om, m));
    }
  }
  {
    std::ifstream in((ppcdir + "hvs-f2k").c_str());
    if (!in.fail()) {
      OMKey om;
      float hv;
      while (in >> om.str >> om.dom >> hv) if (om.isinice()) hvs.insert(std::make_pair(om, hv));
    }
  }
  {
    std::ifstream in((ppcdir + "cx.dat").c_str());
    if (!in.fail()) {
      OMKey om;
      Vec3 d;
      float r;
      while (in >> om.str >> om.dom >> d[0] >> d[1] >> d[2] >> r) cx[om] = d;
      if (cx.empty()) throw Error("File cx.dat did not contain valid data");
    }
  }
  {
    std::ifstream in((ppcdir + "dx.dat").c_str());
    if (!in.fail()) {
      OMKey om;
      float d, r;
      while (in >> om.str >> om.dom >> d >> r) {
        while (d < 0) d += 360.f;
        dx[om] = d;
      }
      if (dx.empty()) throw Error("File dx.dat did not contain valid data");
    }
  }

  float Rr = 0, Rz = 0;
  // in-ice DOM list, gpu/ini.cxx:945-1017
  {
    std::sort(i3oms.begin(), i3oms.end());
    for (auto& i : i3oms) {
      if (!i.k.isinice()) continue;
      OMKey om = i.k;
      int m, t;
      float r, h;
      Vec3 tilt;
      float azi = -1.f;
      if (omts.empty()) m = -1;
      else {
        auto j = omts.find(om);
        m = j == omts.end() ? -1 : j->second;
        if (types.find(m) == types.end()) m = -1;
        auto it = types.find(m);
        if (it != types.end()) { i.d.R = it->second.Rr; i.d.F = it->second.Rz / it->second.Rr; }
      }
      Rr = std::max(Rr, i.d.R); Rz = std::max(Rz, i.d.R * fabsf(i.d.F));
      oms.push_back(i.d);
      {
        auto j = rdes.find(om);
        if (j != rdes.end()) { r = j->second.first; t = j->second.second; }
        else { r = 1; t = 0; }
        irdes[std::make_pair(m, t)].addr(r);
      }
      if (hvs.empty()) h = 1200;
      else { auto j = hvs.find(om); h = j == hvs.end() ? 0 : j->second; }
      {
        auto ci = cx.find(om);
        if (ci != cx.end()) tilt = ci->second;
        auto di = dx.find(om);
        if (di != dx.end()) azi = di->second;
      }
      OMName nm;
      nm.k = om; nm.omt = m; nm.type = t; nm.rde = r; nm.hv = h; nm.tilt = tilt; nm.azi = azi;
      names.push_back(nm);
    }
    int gsize = oms.size();
    if (gsize > PPCB_MAXGEO) gsize = PPCB_MAXGEO;
    oms.resize(gsize); names.resize(gsize);
    p.gsize = gsize;
  }
  Rr *= p.xR; Rz *= p.xR;

  // strings, gpu/ini.cxx:1021-1081
  sc.assign(PPCB_NSTR, ppcb_line());
  std::map<unsigned short, short> num;
  {
    std::map<unsigned short, float> l;
    std::map<unsigned short, ppcb_line> scm;
    for (int n = 0; n < p.gsize; n++) {
      unsigned short str = sname(n);
      ppcb_line& s = scm[str];
      const ppcb_dom& om = oms[n];
      if (num.find(str) == num.end()) { l[str] = om.r[2]; s.h = om.r[2]; s.n = n; }
      else {
        if (l[str] > om.r[2]) l[str] = om.r[2];
        if (s.h < om.r[2]) s.h = om.r[2];
        if (s.n > n) s.n = n;
      }
      num[str]++; s.x += om.r[0]; s.y += om.r[1];
    }
    if (scm.size() > PPCB_NSTR) throw Error("Number of strings exceeds capacity of 240");
    for (auto& i : num) {
      unsigned short str = i.first, n = i.second;
      ppcb_line& s = scm[str];
      float d = s.h - l[str];
      if (n > 1 && d <= 0) throw Error("Cannot estimate the spacing along string " + std::to_string(str));
      s.x /= n; s.y /= n; s.r = 0; s.d = n > 1 ? (n - 1) / d : 0; s.dl = 0; s.dh = 0;
      auto j = strs.find(str);
      if (j != strs.end()) { s.x = j->second.first; s.y = j->second.second; }
    }
    for (int n = 0; n < p.gsize; n++) {
      ppcb_line& s = scm[sname(n)];
      const ppcb_dom& om = oms[n];
      float dx = s.x - om.r[0], dy = s.y - om.r[1];
      float dr = dx * dx + dy * dy;
      if (dr > s.r) s.r = dr;
      if (s.d > 0) {
        float dz = om.r[2] - (s.h + (s.n - n) / s.d);
        if (s.dl > dz) s.dl = dz;
        if (s.dh < dz) s.dh = dz;
      }
    }
    p.rx = 0;
    int n = 0;
    for (auto i = num.begin(); i != num.end(); ++i, n++) {
      ppcb_line& s = scm[i->first];
      s.max = i->second - 1;
      i->second = n;
      s.r = Rr + sqrt(s.r);
      if (p.hr > s.r) s.r = p.hr;
      if (p.rx < s.r) p.rx = s.r;
      s.dl -= Rz; s.dh += Rz;
      sc[n] = s;
    }
    p.nstr = n;
  }

  // skewed cell basis, gpu/ini.cxx:1083-1101
  float sin12 = 0;
  {
    float bv[2][2];
    bv[0][0] = cos(kFcv * PPCB_DIR1);
    bv[0][1] = sin(kFcv * PPCB_DIR1);
    bv[1][0] = cos(kFcv * PPCB_DIR2);
    bv[1][1] = sin(kFcv * PPCB_DIR2);
    float det = bv[0][0] * bv[1][1] - bv[0][1] * bv[1][0];
    p.cb[0][0] = bv[1][1] / det;
    p.cb[0][1] = -bv[0][1] / det;
    p.cb[1][0] = -bv[1][0] / det;
    p.cb[1][1] = bv[0][0] / det;
    for (int i = 0; i < 2; i++) sin12 += bv[0][i] * bv[1][i];
    sin12 = sqrt(1 - sin12 * sin12);
    p.rx /= sin12;
  }

  // DOM-search cell grid, gpu/ini.cxx:1103-1174
  std::vector<std::map<unsigned short, int> > cells(PPCB_CX * PPCB_CY);
  {
    auto ctr = [&](const ppcb_line& s, int m) { return p.cb[0][m] * s.x + p.cb[1][m] * s.y; };
    float cl[2] = {0, 0}, ch[2] = {0, 0}, crst[2];
    int n = 0;
    for (auto i = num.begin(); i != num.end(); ++i, n++) {
      const ppcb_line& s = sc[i->second];
      for (int m = 0; m < 2; m++) {
        if (n == 0 || ctr(s, m) < cl[m]) cl[m] = ctr(s, m);
        if (n == 0 || ctr(s, m) > ch[m]) ch[m] = ctr(s, m);
      }
    }
    p.cn[0] = PPCB_CX; p.cn[1] = PPCB_CY;
    for (int m = 0; m < 2; m++) {
      float diff = ch[m] - cl[m];
      p.cn[m] = std::min(p.cn[m], 1 + 2 * (int)lroundf(diff / 125));
      if (p.cn[m] <= 1) {
        ch[m] = cl[m] = (cl[m] + ch[m]) / 2;
        crst[m] = 1 / (p.rx * (2 + PPCB_XXX) + diff);
      } else {
        float s = Rr * (p.cn[m] - 1);
        if (diff < 2 * s) {
          float ave = (cl[m] + ch[m]) / 2;
          cl[m] = ave - s; ch[m] = ave + s; diff = 2 * s;
        }
        crst[m] = (p.cn[m] - 1) / diff;
      }
    }
    bool flag = true;
    for (auto i = num.begin(); i != num.end(); ++i) {
      const ppcb_line& s = sc[i->second];
      int nn[2];
      for (int m = 0; m < 2; m++) {
        nn[m] = lroundf((ctr(s, m) - cl[m]) * crst[m]);
        if (nn[m] < 0 || nn[m] >= p.cn[m]) throw Error("Error in cell initialization");
        float d1 = fabs(ctr(s, m) - (cl[m] + (nn[m] - 0.5f) / crst[m]));
        float d2 = fabs(ctr(s, m) - (cl[m] + (nn[m] + 0.5f) / crst[m]));
        float d = std::min(d1, d2) * sin12 - s.r;
        if (d < 0) flag = false;
      }
      cells[nn[0] * PPCB_CY + nn[1]][i->first]++;
    }
    if (flag) p.rx = 0;
    for (int m = 0; m < 2; m++) { p.cl[m] = cl[m]; p.crst[m] = crst[m]; }
  }
  ls.assign(PPCB_NSTR, 0);
  is.assign(PPCB_CX * PPCB_CY, 0x8000);
  {
    unsigned int pos = 0;
    for (int i = 0; i < p.cn[0]; i++)
      for (int j = 0; j < p.cn[1]; j++) {
        auto& c = cells[i * PPCB_CY + j];
        if (!c.empty()) {
          is[i * PPCB_CY + j] = pos;
          for (auto& n : c) {
            if (pos == PPCB_NSTR) throw Error("Number of string cells exceeds capacity of 240");
            ls[pos++] = num[n.first];
          }
          ls[pos - 1] |= 0x8000;
        } else is[i * PPCB_CY + j] = 0x8000;
      }
  }

  build_strgrid();

  // ice layer tilt, gpu/ini.cxx:1178-1319
  p.tmod = 0;
  lr.assign(PPCB_LMAX, 0.f);
  lp.assign(PPCB_LMAX * PPCB_LYRS * 2, 0.f);
  mcol.assign(PPCB_CTX * PPCB_CTY, 0);
  p.lnum = 0;
  {
    std::ifstream in((tiltdir + "tilt.set").c_str());
    if (!in.fail()) {
      float mdir[2];
      int n = 0;
      std::string line;
      while (getline(in, line)) {
        int tot = sscanf(line.c_str(), "%f %f %f %d %d", &mdir[n], &p.mmin[n], &p.mstp[n], &p.mnum[n], &p.mcut[n]);
        if (tot == 5) n++;
        if (n >= 2) break;
      }
      if (n < 2) throw Error("File tilt.set found, but is corrupt");
      if (mdir[0] != PPCB_DIR1 || mdir[1] != PPCB_DIR2) throw Error("Unsupported tilt grid configuration");
      int size = 0;
      for (int j = 0; j < p.mnum[1]; j++)
        for (int i = 0; i < p.mnum[0]; i++)
          if (i < j + p.mcut[0] && j < i + p.mcut[1]) size++;
      if (size > PPCB_LMAX) throw Error("File tilt.set defines too many dust maps");
      if (p.mnum[0] > PPCB_CTX || p.mnum[1] > PPCB_CTY) throw Error("Error: tilt map configuration exceeds buffer");
      if (p.mstp[0] <= 0 || p.mstp[1] <= 0) throw Error("Tilt map does not use increasing range order");
      for (int m = 0, j = 0; j < p.mnum[1]; j++)
        for (int i = 0; i < p.mnum[0]; i++)
          mcol[i * PPCB_CTY + j] = (i < j + p.mcut[0] && j < i + p.mcut[1]) ? m++ : -1;
      std::ifstream mi((tiltdir + "tilt.map").c_str());
      if (!mi.fail()) {
        p.lnum = size;
        std::vector<float> ds;
        std::vector<std::vector<float> > lpv;
        read_depth_table(mi, p.lnum, ds, lpv);
        int sz = ds.size();
        if (sz - 1 > PPCB_LYRS) throw Error("File tilt.map defines too many map points");
        for (int i = 1; i < sz; i++) if (ds[i] < ds[i - 1]) throw Error("Tilt map does not use increasing depth order");
        for (int i = 0; i < p.lnum; i++)
          for (int j = 0; j < sz - 1; j++) {
            lp[(i * PPCB_LYRS + j) * 2 + 0] = lpv[i][sz - 1 - j];
            lp[(i * PPCB_LYRS + j) * 2 + 1] = lpv[i][sz - 2 - j] - lpv[i][sz - 1 - j];
          }
        p.lpts = sz - 2;
        if (sz < 2) p.lnum = 0;
        else {
          float lmin = ds[0], lmax = ds[sz - 1];
          p.lmin = kZoff - lmax; p.lrdz = (sz - 1) / (lmax - lmin);
        }
        if (p.lnum > 0) p.tmod = 2;
      }
    }
  }
  if (p.lnum <= 0) {
    p.lnum = 0; p.l0 = 0; p.r0 = 0;
    const float thx = 225;
    p.lnx = cos(kFcv * thx); p.lny = sin(kFcv * thx);
    std::ifstream in((tiltdir + "tilt.par").c_str());
    if (!in.fail()) {
      int str;
      float aux;
      std::vector<float> lrv;
      while (in >> str >> aux) { if (aux == 0) p.l0 = str; lrv.push_back(aux); }
      int size = lrv.size();
      if (size > PPCB_LMAX) throw Error("File tilt.par defines too many dust maps");
      for (int i = 1; i < size; i++) if (lrv[i] < lrv[i - 1]) throw Error("Tilt map does not use increasing range order");
      for (int i = 0; i < size; i++) lr[i] = lrv[i];
      std::ifstream di((tiltdir + "tilt.dat").c_str());
      if (!di.fail()) {
        p.lnum = size;
        std::vector<float> ds;
        std::vector<std::vector<float> > lpv;
        read_depth_table(di, p.lnum, ds, lpv);
        int sz = ds.size();
        if (sz - 1 > PPCB_LYRS) throw Error("File tilt.dat defines too many map points");
        for (int i = 1; i < sz; i++) if (ds[i] < ds[i - 1]) throw Error("Tilt map does not use increasing depth order");
        for (int i = 0; i < p.lnum; i++)
          for (int j = 0; j < sz - 1; j++) {
            lp[(i * PPCB_LYRS + j) * 2 + 0] = lpv[i][sz - 1 - j];
            lp[(i * PPCB_LYRS + j) * 2 + 1] = lpv[i][sz - 2 - j] - lpv[i][sz - 1 - j];
          }
        p.lpts = sz - 2;
        if (sz < 2) p.lnum = 0;
        else {
          float lmin = ds[0], lmax = ds[sz - 1];
          p.lmin = kZoff - lmax; p.lrdz = (sz - 1) / (lmax - lmin);
        }
        if (p.lnum > 0) p.tmod = 1;
      }
    }
  }
  {  // reference string of the 1-d tilt, gpu/ini.cxx:1307-1319
    int nr = 0;
    float r0 = 0;
    for (int n = 0; n < p.gsize; n++)
      if (names[n].k.str == p.l0) { nr++; r0 += p.lnx * oms[n].r[0] + p.lny * oms[n].r[1]; }
    if (nr > 0) p.r0 = r0 / nr;
  }
  {
    const char* v = getenv("VTHK");
    p.vthk = v == nullptr ? 0 : atoi(v);
  }

  // wavelength sampling and acceptance, gpu/ini.cxx:1342-1492
  {
    std::vector<float> wx, wy, wz;
    bool rdef = false;
    const char* W = getenv("WFLA");
    float wfla = W == nullptr ? 0 : atof(W);
    if (wfla > 0) {
      for (float x = 0.f; x < 1.f + PPCB_XXX; x += 0.1f) {
        wx.push_back(3 * x * x - 2 * x * x * x);
        wy.push_back(wfla + 10.f * (2 * x - 1));
      }
      qwv.ssw(wfla);
    } else {
      std::string flwl("dat");
      if (getenv("FLWL")) flwl = env_str("FLWL");
      flwl = "wv." + flwl;
      std::ifstream in((ppcdir + flwl).c_str());
      if (in.fail()) throw Error("Could not open file " + flwl);
      bool flag = true;
      int n = 0;
      float xa, ya, xo = 0, yo = 0;
      while (in >> xa >> ya) {
        if ((xa < 0 || 1 < xa) || (n == 0 && xa != 0) || (n > 0 && (xa <= xo || ya <= yo))) { flag = false; break; }
        wx.push_back(xa); wy.push_back(ya);
        xo = xa; yo = ya; n++;
      }
      if (xo != 1 || wx.size() < 2) flag = false;
      if (!flag) throw Error("File " + flwl + " did not contain valid data");
    }
    std::vector<float> qx, qy;
    {
      std::ifstream in((ppcdir + "wv.rde").c_str());
      if (!in.fail()) {
        int n = 0;
        bool flag = true;
        float xa, ya, yo = 0;
        while (in >> ya >> xa) {
          if (xa < 0 || (n > 0 && ya <= yo)) { flag = false; break; }
          qx.push_back(xa); qy.push_back(ya);
          yo = ya; n++;
        }
        if (qx.size() < 2) flag = false;
        if (!flag) throw Error("File wv.rde did not contain valid data");
        rdef = flag;
      }
    }
    if (rdef) {
      int k = 0, n = qy.size();
      for (float w : wy) {
        float r;
        for (; k < n; k++) if (qy[k] > w) break;
        if (k == 0) r = qx[0];
        else if (k == n) r = qx[n - 1];
        else {
          r = ((w - qy[k - 1]) * qx[k] + (qy[k] - w) * qx[k - 1]) / (qy[k] - qy[k - 1]);
          k--;
        }
        wz.push_back(r);
      }
    }
    {
      std::vector<float> qw, qf, qz;
      float qo = 0, wo = wy[0];
      unsigned int n = wx.size();
      for (unsigned int i = 1; i < n; i++) {
        float qv = wx[i], wv = wy[i];
        float bin = wv - wo;
        float wva = wv - bin / 2;
        float val = kDppm * kDoma * kOmav * (qv - qo) / bin;
        qw.push_back(wva);
        qf.push_back(val);
        if (rdef) qz.push_back(val * (wz[i] + wz[i - 1]) / 2);
        qo = qv; wo = wv;
      }
      float blo = wy[1] - wy[0], bhi = wy[n - 1] - wy[n - 2];
      qwv.read(irdes[std::make_pair(-1, 0)], qw, qf, blo, bhi);
      if (rdef) qwv.read(irdes[std::make_pair(-1, 1)], qw, qz, blo, bhi);
    }
  }
  for (auto& i : irdes) {
    const std::pair<int, int>& m = i.first;
    if (m.first < 0) continue;
    std::stringstream fn;
    fn << omdir << "om.wv_" << m.first << "." << m.second;
    std::ifstream in(fn.str().c_str());
    bool flag = false;
    std::vector<float> qw, qf;
    if (!in.fail()) {
      int n = 0;
      flag = true;
      float w, f, u = 0;
      while (in >> w >> f) {
        if (f < 0 || (n > 0 && w <= u)) { flag = false; break; }
        qf.push_back(f * qwv.cherenkov(w)); qw.push_back(w);
        u = w; n++;
      }
      if (qf.size() < 2) flag = false;
      if (!flag) throw Error("File " + fn.str() + " did not contain valid data");
    }
    if (flag) qwv.read(i.second, qw, qf);
  }
  {
    float sum = 0;
    int k = 0;
    for (float w = qwv.wmin + qwv.bin / 2; w < qwv.wmax; w += qwv.bin, k++) {
      float val = 0;
      for (auto& i : irdes) {
        WaveAcc& mt = i.second;
        if (!mt.dat.empty()) {
          float ri = mt.dat[k] * types[i.first.first].rde * mt.rmax * qwv.bin;
          mt.rde += ri; mt.sum.push_back(mt.rde); mt.dat[k] = ri;
          if (val < ri) val = ri;
        }
      }
      sum += val;
      env.dat.push_back(val);
      env.sum.push_back(sum);
    }
    env.rde = sum; eff *= sum;
    for (int i = 0; i < k; i++) env.sum[i] /= sum;
  }

  // Birefringence angular functions of gpu/pro.cu:784-786 (without the sqrt(ra), rb
  // factors), tabulated in double precision against v = sqrt(1 - |cos|) of the angle to
  // the anisotropy axis: with cos = 1 - v^2 and sin = v*sqrt(2 - v^2) all three are smooth
  // in v, so linear interpolation on 512 intervals is accurate to ~1e-7 relative.
  bfrt.assign((PPCB_BFR_TAB + 1) * 4, 0.f);
  for (int k = 0; k <= PPCB_BFR_TAB; k++) {
    const double v = (double)k / PPCB_BFR_TAB, c = 1 - v * v, s = v * std::sqrt(2 - v * v);
    const float* b = p.bfr;
    double sx = std::max(0.0, b[0] * std::exp(-b[1] * std::pow(std::atan(b[3] * s), (double)b[2])));
    double sy = std::max(0.0, b[4] * std::exp(-b[5] * std::pow(std::atan(b[7] * s), (double)b[6])));
    double mx = std::max(0.0, b[8] * std::atan(b[11] * s * c) * std::exp(-b[9] * s + b[10] * c));
    bfrt[k * 4 + 0] = (float)sx;
    bfrt[k * 4 + 1] = (float)sy;
    bfrt[k * 4 + 2] = (float)mx;
  }

  // ice optical properties, gpu/ini.cxx:1494-1696
  const float wv0 = 400;
  float A, B, D, E, a, k;
  {
    std::ifstream in((icedir + "icemodel.par").c_str());
    if (in.fail()) throw Error("File icemodel.par was not found");
    float ae, ke, Ae, Be, De, Ee;
    bool flag = true;
    if (flag) flag = (bool)(in >> a >> ae);
    if (flag) flag = (bool)(in >> k >> ke);
    if (flag) flag = (bool)(in >> A >> Ae);
    if (flag) flag = (bool)(in >> B >> Be);
    bool fail = !flag;
    if (flag) flag = (bool)(in >> D >> De);
    D = flag ? D / pow(wv0, k) : 1;
    if (flag) flag = (bool)(in >> E >> Ee);
    E = flag ? E / pow(wv0, k) : 0;
    if (fail) throw Error("File icemodel.par found, but is corrupt");
  }
  ice_a = a; ice_k = k; ice_A = A; ice_B = B; ice_D = D; ice_E = E;
  int size = 0;
  {
    std::ifstream in((icedir + "icemodel.dat").c_str());
    if (in.fail()) throw Error("File icemodel.dat was not found");
    float dpa, bea, baa, tda, k1a, k2a, bfra, bfrb;
    std::string line;
    while (getline(in, line)) {
      int n = sscanf(line.c_str(), "%f %f %f %f %f %f %f %f", &dpa, &bea, &baa, &tda, &k1a, &k2a, &bfra, &bfrb);
      if (n >= 4) {
        dp.push_back(dpa); be.push_back(bea); ba.push_back(baa); td.push_back(tda);
        k1v.push_back(n >= 5 ? exp(k1a) : dk1);
        k2v.push_back(n >= 6 ? exp(k2a) : dk2);
        rav.push_back(n >= 7 ? bfra : 1);
        rbv.push_back(n >= 8 ? bfrb : 1);
        size++;
      }
    }
    if (size < 1) throw Error("File icemodel.dat found, but is corrupt");
  }
  float dh = size > 1 ? (dp[size - 1] - dp[0]) / (size - 1) : 100.f;
  if (dh <= 0) throw Error("Ice table does not use increasing depth spacing");
  for (int i = 1; i < size; i++)
    if (fabs(dp[i] - dp[i - 1] - dh) > dh * PPCB_XXX) throw Error("Ice table does not use uniform depth spacing");
  if (size > PPCB_MAXLYS) size = PPCB_MAXLYS;
  p.size = size; p.dh = dh; p.rdh = 1 / dh; p.hmin = kZoff - dp[size - 1];
  {
    std::ifstream in((icedir + "icemodel.bbl").c_str());
    if (!in.fail()) { if (!(in >> bble >> bblz >> bbly)) bble = 0; }
  }
  az.assign(size, ppcb_aniz());
  for (int i = 0; i < size; i++) {
    int j = size - 1 - i;
    az[i].k1 = k1v[j]; az[i].k2 = k2v[j];
    az[i].ra = rav[j]; az[i].rb = rav[j] * rbv[j];
  }
  arf = 0; srw = 0; srf = 1;
  {
    std::ifstream in((icedir + "version").c_str());
    int version = 0;
    if (!in.fail()) { if (!(in >> version)) version = 0; }
    switch (version) {
      case 10: arf = 0; srw = 0; srf = 0; break;
      case 20: arf = 1; srw = 1; srf = 0; break;
    }
  }
  if (const char* absm = getenv("ABSM")) {
    switch (atoi(absm)) { case 0: arf = 0; break; case 1: arf = 1; break; }
  }
  if (const char* bfrm = getenv("BFRM")) {
    switch (atoi(bfrm)) {
      case 0: srw = 0; srf = 1; break;
      case 1: srw = 1; srf = 0; break;
      case 2: srw = 0; srf = 0; break;
    }
  }
  wvs.assign(PPCB_WNUM, WaveSample());
  wmeta.assign(PPCB_WNUM, ppcb_wmeta());
  absca.assign((size_t)PPCB_WNUM * size * 2, 0.f);
  wgrad.assign(PPCB_WNUM * 2, 0.f);
  for (int n = 0; n < PPCB_WNUM; n++) {
    float wvi = env.binf((n + 0.f) / PPCB_WNUM);
    int mi = std::min(std::max((int)floor(wvi), 0), qwv.num - 1);
    float wvf = env.binf((n + 1.f) / PPCB_WNUM);
    int mf = std::min(std::max((int)floor(wvf), 0), qwv.num - 1);
    float wva = qwv.wav(env.binf((n + 0.5f) / PPCB_WNUM));
    wvs[n].w = wva; wvs[n].i = qwv.wav(wvi); wvs[n].f = qwv.wav(wvf);
    for (auto& i : irdes) {
      WaveAcc& mt = i.second;
      if (mt.rde > 0) {
        const std::vector<float>& wy = mt.dat;
        float rde;
        if (mf == mi) rde = wy[mi] * (wvf - wvi);
        else {
          rde = (mi + 1 - wvi) * wy[mi] + (wvf - mf) * wy[mf];
          for (int ii = mi + 1; ii < mf; ii++) rde += wy[ii];
        }
        rde /= env.rde / PPCB_WNUM;
        mt.rat.push_back(rde);
      }
    }
    fill_ice(n, wva);
    float ng, npv = qwv.np(wva * 1.e-3, &ng);
    float c = 0.299792458;
    p.ocv = 1 / c;
    wmeta[n].wvl = n; wmeta[n].ocm = ng / c;
    wmeta[n].coschr = 1 / npv; wmeta[n].sinchr = sqrt(1 - wmeta[n].coschr * wmeta[n].coschr);
  }
}

// String-proximity table (strgrid.h).  Lines on the same axis form a group (its disc covers
// theirs, widened by kReachPad); a square grid over the groups' footprint plus a
// 64 m margin, with cells as small as kSgMaxCells allows (from 8 m up), stores per cell the
// nearest group and a lower bound on the distance from the cell to every other group's
// widened disc (exact on the cell square, rounded down to kSgClearUnit).  Not part of the
// reference's tables: it only decides when the reference's DOM search can be skipped.
void Config::build_strgrid() {
  sg = StrGridParams{};
  sg_groups.clear();
  sg_cells.clear();
  if (p.nstr <= 0) return;
  // lines whose axes are within a metre of a group's axis join it (a string split into
  // lines has the same axis up to rounding); the group's disc covers each line's disc
  for (int m = 0; m < p.nstr; m++) {
    bool merged = false;
    for (auto& g : sg_groups) {
      const double d = std::hypot((double)sc[m].x - g.x, (double)sc[m].y - g.y);
      if (d < 1) {
        g.rw = std::max(g.rw, (float)(d + sc[m].r + kReachPad) * (1 + 1e-6f));
        merged = true;
        break;
      }
    }
    if (!merged) sg_groups.push_back(StrGroup{sc[m].x, sc[m].y, sc[m].r + kReachPad, 0});
  }
  if (sg_groups.size() >= 255) throw Error("string-proximity table: too many string axes");
  const int ng = (int)sg_groups.size();
  const double margin = 64;
  double x0 = 1e30, x1 = -1e30, y0 = 1e30, y1 = -1e30;
  for (auto& g : sg_groups) {
    x0 = std::min(x0, (double)g.x - g.rw); x1 = std::max(x1, (double)g.x + g.rw);
    y0 = std::min(y0, (double)g.y - g.rw); y1 = std::max(y1, (double)g.y + g.rw);
  }
  double cell = 8;
  int nx = 0, ny = 0;
  for (;;) {
    nx = (int)std::ceil((x1 - x0 + 2 * margin) / cell);
    ny = (int)std::ceil((y1 - y0 + 2 * margin) / cell);
    if ((long)nx * ny <= kSgMaxCells) break;
    cell *= 1.25;
  }
  const double ox = x0 - margin, oy = y0 - margin;
  sg.inv = (float)(1 / cell);
  sg.ou = (float)(-ox / cell);
  sg.ov = (float)(-oy / cell);
  sg.margin2 = (float)(margin * margin);
  sg.nx = nx; sg.ny = ny; sg.on = 1;
  sg_cells.assign((size_t)nx * ny, 0);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      // the cell of the device's index arithmetic, widened by a millimetre on each side
      // (the index is computed in single precision from the origin and the cell size)
      const double xa = ox + i * cell - 1e-3, xb = ox + (i + 1) * cell + 1e-3;
      const double ya = oy + j * cell - 1e-3, yb = oy + (j + 1) * cell + 1e-3;
      int best = -1;
      double d1 = 1e30, d2 = 1e30;  // nearest and second-nearest disc distance
      for (int k = 0; k < ng; k++) {
        const double gx = sg_groups[k].x, gy = sg_groups[k].y;
        const double qx = gx - std::min(std::max(gx, xa), xb), qy = gy - std::min(std::max(gy, ya), yb);
        const double d = std::max(0.0, std::sqrt(qx * qx + qy * qy) - (double)sg_groups[k].rw);
        if (d < d1) { d2 = d1; d1 = d; best = k; }
        else if (d < d2) d2 = d;
      }
      const double q = std::floor(d2 / kSgClearUnit);
      const unsigned int clear = q > 255 ? 255u : (unsigned int)q;
      sg_cells[(size_t)j * nx + i] = (uint16_t)((clear << 8) | (unsigned int)(best < 0 ? ng : best));
    }
  sg_groups.push_back(StrGroup{1e30f, 1e30f, 0, 0});  // the sentinel: no group within reach
}

}  // namespace ppcb
