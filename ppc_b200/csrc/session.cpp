// Session: front end, batching pipeline and hit back end (see session.h).
// Compiled with IEEE float semantics, like config.cpp.
#include "session.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>

// float overloads of the math functions, as in the reference (gpu/ppc.cu:26)
using namespace std;

namespace ppcb {

static const float kFcv = PPCB_FPI / 180.f;
static const float kDppm = 2450.08;
static const float kRho = 0.9216f;          // density of ice [mwe]
static const float kM0 = 0.105658389f;      // muon rest mass [GeV]

static bool quiet() { return getenv("PPCB_QUIET") != nullptr; }

void Session::initialize(const std::string& dir, float enh) { eng.initialize(dir, enh); }

void Session::ini() {
  eng.ini();
  pz_.clear();
  pz_.reserve(eng.pmxo);
  pn_ = 0;
  total = RunInfo();
}

void Session::fin() {
  eng.fin();
}

// gpu/f2k.cxx:1-10
float Session::xrnd() {
  unsigned int rnd;
  do rnd = rand_r(&eng.sv); while (rnd == 0);
  const float a = 1.0f / (1ll + RAND_MAX);
  return a * rnd;
}

float Session::grnd() {
  float a = sqrtf(-2 * logf(xrnd()));
  return a * sinf(2 * PPCB_FPI * xrnd());
}

// gpu/f2k.cxx:559-582: direction from the zenith and azimuth of the track (pointing back to
// where it comes from), particle names to light-yield types
bool parse_f2k_track(const std::string& line, F2kTrack& tr) {
  char name[32];
  int gens, igen;
  float th, ph;
  if (sscanf(line.c_str(), "TR %d %d %31s %f %f %f %f %f %f %f %f", &gens, &igen, name, &tr.x, &tr.y, &tr.z, &th,
             &ph, &tr.l, &tr.E, &tr.t) != 11)
    return false;
  const float fcv = PPCB_FPI / 180.f;
  th = fcv * (180 - th);
  ph = fcv * (ph < 180 ? ph + 180 : ph - 180);
  const float costh = cosf(th), sinth = sinf(th), cosph = cosf(ph), sinph = sinf(ph);
  tr.n[0] = sinth * cosph;
  tr.n[1] = sinth * sinph;
  tr.n[2] = costh;
  tr.type = -1;
  if (!strcmp(name, "amu+") || !strcmp(name, "amu-") || !strcmp(name, "amu")) tr.type = 0;
  else if (!strcmp(name, "delta") || !strcmp(name, "brems") || !strcmp(name, "epair") || !strcmp(name, "e"))
    tr.type = 11;
  else if (!strcmp(name, "e-")) tr.type = 12;
  else if (!strcmp(name, "e+")) tr.type = 13;
  else if (!strcmp(name, "munu") || !strcmp(name, "hadr")) tr.type = 101;
  else if (!strcmp(name, "ph")) tr.type = -2;
  return true;
}

// gpu/f2k.cxx:17-167: photons per bunch template for a source of energy E
float Session::yield(float E, float dr, int type) {
  p.n[3] = dr;
  float nph = 0;
  if (type < 0) {
    nph = E / kDppm;
  } else {
    float logE = logf(std::max(kM0, E));
    if (type < 10) {  // bare muon (0) or its end point (1)
      float extr = 1 + std::max(0.0f, 0.1880f + 0.0206f * (logE - type)) * 0.910f / kRho;
      nph = dr > 0 ? dr * extr : 0;
      p.f = 1 / extr;
      p.u.p.a = 0; p.u.p.b = 0;
    } else {  // cascades
      const float Lrad = 0.39652 * 0.910f / kRho;
      const float em = 5.321 * 0.910f / kRho;
      nph = em * E;
      if (type < 100) {
        switch (type) {
          default:
          case 10: case 11: case 12:
            p.u.p.a = 2.01849f + 0.63176f * logE; p.u.p.b = Lrad / 0.63207f; break;
          case 13:
            p.u.p.a = 2.00035f + 0.63190f * logE; p.u.p.b = Lrad / 0.63008f; break;
          case 14:
            p.u.p.a = 2.83923f + 0.58209f * logE; p.u.p.b = Lrad / 0.64526f; break;
        }
      } else {
        float E0, m, f0, rms0, gamma;
        switch (type) {
          default:
          case 101: case 102:
            p.u.p.a = 1.58357292f + 0.41886807f * logE; p.u.p.b = Lrad / 0.33833116f;
            E0 = 0.18791678f; m = 0.16267529f; f0 = 0.30974123f; rms0 = 0.95899551f; gamma = 1.35589541f; break;
          case 103:
            p.u.p.a = 1.69176636f + 0.40803489f * logE; p.u.p.b = Lrad / 0.34108075f;
            E0 = 0.19826506f; m = 0.16218006f; f0 = 0.31859323f; rms0 = 0.94033488f; gamma = 1.35070162f; break;
          case 104:
            p.u.p.a = 1.95948974f + 0.34934666f * logE; p.u.p.b = Lrad / 0.34535151f;
            E0 = 0.21687243f; m = 0.16861530f; f0 = 0.27724987f; rms0 = 1.00318874f; gamma = 1.37528605f; break;
          case 105:
            p.u.p.a = 1.47495778f + 0.40450398f * logE; p.u.p.b = Lrad / 0.35226706f;
            E0 = 0.29579368f; m = 0.19373018f; f0 = 0.02455403f; rms0 = 1.01619344f; gamma = 1.45477346f; break;
          case 106:
            p.u.p.a = 1.57739060f + 0.40631102f * logE; p.u.p.b = Lrad / 0.35269455f;
            E0 = 0.66725124f; m = 0.19263595f; f0 = 0.17559033f; rms0 = 1.01414337f; gamma = 1.45086895f; break;
          case 107:
            p.u.p.a = 1.92249171f + 0.33701751f * logE; p.u.p.b = Lrad / 0.34969748f;
            E0 = 0.29579368f; m = 0.19373018f; f0 = 0.02455403f; rms0 = 1.01094637f; gamma = 1.50438415f; break;
        }
        {  // hadronic light-yield fluctuation
          float e = std::max(2.71828183f, E), f;
          float F = 1 - powf(e / E0, -m) * (1 - f0);
          float dF = F * rms0 * powf(logf(e), -gamma);
          do f = F + dF * grnd(); while (f < 0 || 1.1 < f);
          nph *= f;
        }
      }
      p.f = 0;
      if (dr > 0) { p.u.p.a = 0; p.u.p.b = 0; }
    }
  }
  return eng.cfg.eff * nph;
}

// gpu/f2k.cxx:387-433
static double gammln(double xx) {
  static const double stp = 2.5066282746310005;
  static const double cof[6] = {76.18009172947146, -86.50532032941677, 24.01409824083091,
                                -1.231739572450155, 0.1208650973866179e-2, -0.5395239384953e-5};
  double ser = 1, x = xx - 1;
  double tmp = x + 5.5;
  tmp -= (x + 0.5) * log(tmp);
  for (int j = 0; j <= 5; j++) { x++; ser += cof[j] / x; }
  return -tmp + log(stp * ser);
}

unsigned long long Session::poidev(double xm) {
  double sq, alxm, g, t, y;
  unsigned long long um;
  if (xm < 12) {
    g = exp(-xm);
    um = -1ULL;
    t = 1;
    do { um++; t *= xrnd(); } while (t > g);
  } else {
    sq = sqrt(2 * xm);
    alxm = log(xm);
    g = xm * alxm - gammln(xm + 1);
    do {
      double em;
      do {
        y = tan(PPCB_FPI * xrnd());
        em = sq * y + xm;
      } while (em < 0);
      um = floor(em);
      t = 0.9 * (1 + y * y) * exp(um * alxm - gammln(um + 1) - g);
    } while (xrnd() > t);
  }
  return um;
}

// gpu/f2k.cxx:435-476
unsigned long long Session::bnldev(unsigned long long n, double pp) {
  unsigned long long j, bnl;
  double am, em, g, angle, pv, sq, t, y;
  double pc, plog, pclog, en, oldg;
  pv = (pp <= 0.5 ? pp : 1 - pp);
  am = n * pv;
  if (n < 25) {
    bnl = 0;
    for (j = 1; j <= n; j++) if (xrnd() < pv) bnl++;
  } else if (am < 1) {
    g = exp(-am);
    t = 1;
    for (j = 0; j <= n; j++) { t *= xrnd(); if (t < g) break; }
    bnl = (j <= n ? j : n);
  } else {
    en = n;
    oldg = gammln(en + 1);
    pc = 1 - pv;
    plog = log(pv);
    pclog = log(pc);
    sq = sqrt(2 * am * pc);
    do {
      do {
        angle = PPCB_FPI * xrnd();
        y = tan(angle);
        em = sq * y + am;
      } while (em < 0 || em >= (en + 1));
      em = floor(em);
      t = 1.2 * sq * (1 + y * y) * exp(oldg - gammln(em + 1) - gammln(en - em + 1) + em * plog + (en - em) * pclog);
    } while (xrnd() > t);
    bnl = em;
  }
  if (pv != pp) bnl = n - bnl;
  return bnl;
}

// gpu/f2k.cxx:377-385: split a source into bunches, flushing full batches
void Session::addh(unsigned long long num) {
  if (!eng.ready()) throw Error("ini() must come before adding sources");
  do {
    p.num = (uint32_t)std::min<unsigned long long>(eng.pmax - pn_, num);
    num -= p.num;
    pn_ += p.num;
    pz_.push_back(p);
    if (pn_ == eng.pmax || pz_.size() == eng.pmxo) output();
  } while (num > 0);
  if (pn_ > 0 && pz_.empty()) pz_.push_back(p);
}

// gpu/f2k.cxx:478-482 (f2k "ph" record: exact photon count at a point)
void Session::addf(float rx, float ry, float rz, float t, unsigned long long num) {
  p.r[0] = rx; p.r[1] = ry; p.r[2] = rz; p.r[3] = t; p.type = 1;
  p.u.l.ka = 0; p.u.l.up = 0; p.u.l.fldr = -1; p.u.l.fla = -1; p.u.l.ofla = -1;
  p.n[3] = 1;
  addh(num);
}

// gpu/f2k.cxx:484-504
void Session::addp(float rx, float ry, float rz, float t, float E, float dr, int type, float scale) {
  p.r[0] = rx; p.r[1] = ry; p.r[2] = rz; p.r[3] = t;
  if (type < 0) {
    memcpy(p.u.c, pfl.u.c, sizeof(p.u.c));
    switch (type) {
      case -1: dr = 0; p.u.l.ka = -2; break;  // linear cone around n
      case -2: dr = 0; break;                 // 2-d gaussian around n
      case -3: dr = 0; p.u.l.ka = -1; break;  // isotropic
      case -4:
      default:
        dr = pfl.n[3];
        p.type = pfl.type;
        memcpy(p.r, pfl.r, sizeof(p.r));
        memcpy(p.n, pfl.n, sizeof(p.n));
    }
  } else {
    p.type = -type;
    p.u.p.beta = 1; p.u.p.tau = 0;
  }
  unsigned long long num = poidev(scale * yield(E, dr, type) / eng.cfg.ovr);
  addh(num);
}

// gpu/f2k.cxx:507-518
void Session::addp_clst(float rx, float ry, float rz, float t, unsigned long long n, float dr, float beta) {
  p.type = 0;
  p.r[3] = t; p.r[0] = rx; p.r[1] = ry; p.r[2] = rz;
  p.n[3] = dr; p.f = 1.f; p.u.p.a = 0; p.u.p.b = 0;
  p.u.p.beta = beta; p.u.p.tau = 0;
  float qmas = 1.f;
  unsigned long long num = qmas > 0 && qmas < 1 ? bnldev(n, qmas) : n;
  addh(num);
}

// gpu/f2k.cxx:520-528
void Session::addp_mopo(float rx, float ry, float rz, float t, float light, float length, float beta, float tau,
                        float fr) {
  p.type = 0;
  p.r[3] = t; p.r[0] = rx; p.r[1] = ry; p.r[2] = rz;
  p.n[3] = length; p.f = fr; p.u.p.a = 0; p.u.p.b = 0;
  p.u.p.beta = beta; p.u.p.tau = tau;
  unsigned long long num = poidev(light * eng.cfg.eff / eng.cfg.ovr);
  addh(num);
}

// gpu/f2k.cxx:586-588
void Session::flone(unsigned long long num) {
  addh(num * (eng.cfg.eff / kDppm) / eng.cfg.ovr);
}

// gpu/f2k.cxx:590-628: rotate the LED frame from vertical to the DOM tilt m
void Session::flshift(float m[], float n[], float* r) {
  if (std::isnan(n[2])) {
    float xi;
    sincosf(p.u.l.up, &n[2], &xi);
    n[0] *= xi; n[1] *= xi;
  }
  float q[3], o[3] = {0, 0, 1};
  q[0] = m[1] * o[2] - m[2] * o[1];
  q[1] = m[2] * o[0] - m[0] * o[2];
  q[2] = m[0] * o[1] - m[1] * o[0];
  float norm = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
  if (norm > 0) {
    float cs = 0;
    for (int i = 0; i < 3; i++) { q[i] /= norm; cs += o[i] * m[i]; }
    float sn = sin(acos(cs));
    float R[3][3] = {{0}};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        R[i][j] = (i == j ? cs : sn * q[3 - i - j] * ((j - i + 3) % 3 == 1 ? 1 : -1)) + (1 - cs) * q[i] * q[j];
    for (int i = 0; i < 3; i++) {
      q[i] = 0;
      for (int j = 0; j < 3; j++) q[i] += R[i][j] * n[j];
    }
    for (int i = 0; i < 3; i++) n[i] = q[i];
    if (r != nullptr) {
      for (int i = 0; i < 3; i++) {
        q[i] = 0;
        for (int j = 0; j < 3; j++) q[i] += R[i][j] * r[j];
      }
      for (int i = 0; i < 3; i++) r[i] = q[i];
    }
  }
}

// gpu/f2k.cxx:630-759: flasher / standard candle at (str, dom), configured from the
// environment (FZCR, ELEV, OFLA, FLDR, FWID, FTLT)
const ppcb_dom& Session::flset(int str, int dom) {
  const Config& c = eng.cfg;
  p.u.l.fla = -1; p.u.l.ofla = -1;
  p.u.l.ka = 0; p.u.l.up = 0; p.u.l.fldr = -1;
  p.n[0] = 0; p.n[1] = 0; p.n[2] = 1; p.n[3] = 0;
  int type = 1;
  {
    float r[3] = {0, 0, 0};
    if (str < 0) { type = 2; str = -str; }
    if (str == 0) {
      switch (dom) {  // standard candles
        case 1: type = 3; r[0] = 544.07; r[1] = 55.89; r[2] = 136.86; break;
        case 2: type = 4; r[0] = 11.87; r[1] = 179.19; r[2] = -205.64; break;
      }
    } else {
      for (int n = 0; n < c.p.gsize; n++)
        if (c.names[n].k.str == str && c.names[n].k.dom == dom) {
          p.u.l.fla = n;
          for (int m = 0; m < 3; m++) r[m] = c.oms[n].r[m];
          break;
        }
    }
    if (!quiet()) std::cerr << "Flasher configured at " << r[0] << ", " << r[1] << ", " << r[2] << std::endl;
    p.type = type;
    p.r[0] = r[0]; p.r[1] = r[1]; p.r[2] = r[2]; p.r[3] = 0;
    for (int m = 0; m < 3; m++) flom_.r[m] = r[m];
  }
  float fzcr = 0.f;
  if (const char* v = getenv("FZCR")) fzcr = atof(v);
  switch (type) {
    case 1: p.u.l.up = (-0.2f + fzcr) * kFcv; break;
    case 2: p.u.l.up = (48.1f + fzcr) * kFcv; break;
    case 3: p.u.l.up = (90.0f - 41.13f) * kFcv; break;
    case 4: p.u.l.up = (41.13f - 90.0f) * kFcv; break;
  }
  if (const char* v = getenv("ELEV")) p.u.l.up = atof(v) * kFcv;
  p.u.l.ofla = p.u.l.fla;
  if (const char* v = getenv("OFLA")) if (*v != 0 && atoi(v) == 0) p.u.l.ofla = -1;
  {
    const char* v = getenv("FLDR");
    p.u.l.fldr = v == nullptr ? -1 : atof(v);
  }
  float vx, vy;
  {
    float xi = p.u.l.fldr * kFcv;
    sincosf(xi, &vy, &vx);
    sincosf(p.u.l.up, &p.n[2], &xi);
    p.n[0] = xi * vx; p.n[1] = xi * vy;
  }
  float fwid = 9.7f;
  if (const char* v = getenv("FWID")) fwid = atof(v);
  if (fwid > 999.f) {
    p.u.l.ka = fwid;
    if (p.u.l.fla >= 0 && p.u.l.fldr >= 0 && p.u.l.fldr < 360) {
      if (const char* bmp = getenv("FTLT")) {
        float m[3] = {0, 0, 1};
        float nx, ny, nz;
        int num = sscanf(bmp, "%f %f %f", &nx, &ny, &nz);
        if (num == 3) { m[0] = nx; m[1] = ny; m[2] = nz; }
        else {
          OMKey om{str, dom};
          auto it = c.cx.find(om);
          if (it != c.cx.end()) for (int i = 0; i < 3; i++) m[i] = it->second[i];
        }
        p.n[3] = 1;
        const float FLZ = 0.07735f, FLR = 0.119f - 0.008f;
        p.r[0] = FLR * vx; p.r[1] = FLR * vy; p.r[2] = FLZ;
        float n[3] = {p.n[0], p.n[1], p.n[2]};
        float r[3] = {p.r[0], p.r[1], p.r[2]};
        flshift(m, n, r);
        p.r[0] = r[0]; p.r[1] = r[1]; p.r[2] = r[2];
        p.n[0] = n[0]; p.n[1] = n[1]; p.n[2] = n[2];
      }
    }
  } else if (fwid > 0) p.u.l.ka = (kFcv * fwid) * (kFcv * fwid);
  else p.u.l.ka = fwid;
  pfl = p;
  return flom_;
}

// gpu/f2k.cxx:762-765 (the direction is captured on the first call, as there)
const float* Session::fldir() {
  if (!fldir_set_) {
    fldir_[0] = pfl.n[0]; fldir_[1] = pfl.n[1]; fldir_[2] = pfl.n[2];
    fldir_set_ = true;
  }
  return fldir_;
}

// gpu/f2k.cxx:531-534
void Session::finc() {
  flne++;
  if ((int)(flne - flnb) < 0) throw Error("Error: too many event segments", 3);
}

// gpu/f2k.cxx:548-552
void Session::sett(float nx, float ny, float nz, std::pair<int, unsigned long long> id, int frame, double t0) {
  Seg s;
  s.is_line = false;
  s.id.first = id.first; s.id.second = id.second; s.id.frame = frame; s.id.t0 = t0;
  flnz_.push_back(s);
  finc();
  p.q = flne; p.n[0] = nx; p.n[1] = ny; p.n[2] = nz;
}

void Session::sett_line(const std::string& line) {
  Seg s;
  s.is_line = true;
  s.line = line;
  flnz_.push_back(s);
  finc();
}

// gpu/f2k.cxx:365-375
void Session::output() {
  kernel(pn_);
  pn_ = 0;
  pz_.clear();
}

// gpu/ppc.cu:432-469, restated as a depth-2 pipeline: queue this batch first, then
// collect and post-process the previous one while this one runs.  A call without
// photons drains the pipeline (the reference's second output() in eout()).
void Session::kernel(uint64_t num) {
  if (num > 0) {
    if (eng.in_flight() >= 2) collect_one();
    eng.submit(pz_.data(), (int)pz_.size(), num);
    flnd_q_.push_back(flne);
    if (eng.in_flight() >= 2) collect_one();
  } else {
    while (eng.in_flight() > 0) collect_one();
  }
}

void Session::collect_one() {
  std::vector<ppcb_hit> hits;
  RunInfo info;
  if (!eng.collect(hits, info)) return;
  unsigned int flnd = flnd_q_.front();
  flnd_q_.pop_front();
  last = info;
  total.photons += info.photons;
  total.hits += info.hits;
  total.kept += info.kept;
  total.steps += info.steps;
  total.nan_steps += info.nan_steps;
  total.capped += info.capped;
  total.device_ms += info.device_ms;
  if (info.nan_steps > 0)
    std::cerr << "Error: TOT was a nan or an inf " << info.nan_steps << " times!" << std::endl;
  if (info.overflow)
    std::cerr << "Error: data buffer overflow occurred: " << info.hits << ">" << info.kept << "!" << std::endl;
  if (!quiet()) std::cerr << "photons: " << info.photons << "  hits: " << info.kept << std::endl;
  if (keep_raw) raw_.insert(raw_.end(), hits.begin(), hits.end());
  print(hits, flnd);
}

// gpu/f2k.cxx:536-541: flush everything, blocking
void Session::eout() {
  output();
  output();
}

static float res(float val, float bin) { return bin > 0 ? (floor(val / bin) + 0.5) * bin : val; }

// gpu/f2k.cxx:247-363: per-hit acceptance and output
void Session::print(std::vector<ppcb_hit>& hits, unsigned int flnd) {
  const Config& c = eng.cfg;
  if ((int)(flnb - flnd) < 0)
    std::stable_sort(hits.begin(), hits.end(), [](const ppcb_hit& a, const ppcb_hit& b) { return (int)(a.n - b.n) < 0; });
  auto pop = [&]() {
    Seg& s = flnz_.front();
    if (s.is_line) { if (hit_out) fprintf(hit_out, "%s\n", s.line.c_str()); }
    else tmph_.track = s.id;
    flnz_.pop_front();
  };
  for (ppcb_hit& h : hits) {
    if ((int)(h.n - flnb) < 0 || (int)(h.n - flnd) > 0) {
      std::cerr << "Internal Error: " << h.n << " is not between " << flnb << " " << flnd << " " << flne << std::endl;
      continue;
    }
    for (; (int)(flnb - h.n) < 0; flnb++) pop();
    const OMName& n = c.names[h.i];
    bool flag = n.hv > 0;
    if (flag) {
      auto it = c.irdes.find(std::make_pair(n.omt, n.type));
      if (it == c.irdes.end()) flag = false;
      else {
        const WaveAcc& mt = it->second;
        flag = mt.rde > 0 && xrnd() < mt.rat[h.z] * n.rde / mt.rmax;
      }
    }
    float nx = 0, ny = 0, nz = 0, rx = 0, ry = 0, rz = 0;
    if (flag) {
      float F = c.oms[h.i].F;
      float ptc = cosf(h.pth), pts = sinf(h.pth), ppc = cosf(h.pph), pps = sinf(h.pph);
      float dtc = F * cosf(h.dth), dts = F < 0 ? 1 : sinf(h.dth), dpc = cosf(h.dph), dps = sinf(h.dph);
      rx = dts * dpc; ry = dts * dps; rz = dtc;
      nx = pts * ppc; ny = pts * pps; nz = ptc;
    }
    int pmt = 0;
    if (flag) {
      auto it = c.types.find(n.omt);
      if (it != c.types.end()) {
        Vec3 dir, pos;
        dir[0] = nx; dir[1] = ny; dir[2] = nz;
        pos[0] = rx; pos[1] = ry; pos[2] = rz;
        float rnd = xrnd();
        pmt = it->second.getPMT(dir, pos, n.tilt, rnd, h.t, n.azi, [this]() { return xrnd(); });
        flag = pmt >= 0;
      } else flag = false;
    }
    if (flag) {  // cable shadow
      float omr = c.oms[h.i].R;
      float rc = 0.023f;
      float dc = omr + rc;
      float ph = n.azi;
      if (ph >= 0) {
        float drx = -omr * rx - dc * cos(kFcv * ph);
        float dry = -omr * ry - dc * sin(kFcv * ph);
        float a = nx * nx + ny * ny;
        if (a > 0) {
          float b = -2 * (nx * drx + ny * dry);
          float cc = drx * drx + dry * dry - rc * rc;
          float D = b * b - 4 * a * cc;
          if (D >= 0) {
            float h1 = (-b + sqrt(D)) / (2 * a);
            if (h1 > 0) flag = false;
          }
        }
      }
    }
    if (flag) {
      const WaveSample& ws = c.wvs[h.z];
      float wv = ws.i + (ws.f - ws.i) * xrnd();
      if (hit_out) {
        if (c.nextgen)
          fprintf(hit_out, "HIT %d %d_%d %f %f %f %f %f %f\n", n.k.str, n.k.dom, pmt, h.t, wv, h.pth, h.pph, h.dth, h.dph);
        else
          fprintf(hit_out, "HIT %d %d %f %f %f %f %f %f\n", n.k.str, n.k.dom, h.t, wv, h.pth, h.pph, h.dth, h.dph);
      } else {
        tmph_.omkey.str = n.k.str; tmph_.omkey.dom = n.k.dom;
        tmph_.pmt = pmt;
        tmph_.time = res(h.t, trz_);
        tmph_.dir = res(1 + cos(h.pth), crz_) - 1;
        xppc::pout po;
        float omr = c.oms[h.i].R;
        po.r[0] = -omr * rx; po.r[1] = -omr * ry; po.r[2] = -omr * rz; po.r[3] = h.t;
        po.n[0] = nx; po.n[1] = ny; po.n[2] = nz; po.n[3] = wv;
        (*hitz)[tmph_].push_back(po);
      }
    }
  }
  for (; (int)(flnb - flnd) < 0; flnb++) pop();
}

}  // namespace ppcb
