// Drop-in definitions of the xppc:: API (include/xppc.h) over one process-wide Session.
// Error behaviour follows the reference: configuration and device errors print a
// message and exit with the reference's status code.
#include <cstdlib>
#include <iostream>

#include "../../include/xppc.h"
#include "session.h"

namespace xppc {

std::vector<OM> i3oms;
std::map<ikey, int> omts;
std::map<ikey, float> hvs;
std::map<ikey, std::pair<float, int> > rdes;
outz hitz;
bool nextgen = false;

static ppcb::Session& S() {
  static ppcb::Session* s = [] {
    ppcb::Session* x = new ppcb::Session();
    x->hitz = &xppc::hitz;
    return x;
  }();
  return *s;
}

template <class F>
static void run(F&& f) {
  try {
    f();
  } catch (const ppcb::Error& e) {
    std::cerr << e.what() << std::endl;
    exit(e.code ? e.code : 1);
  }
}

static ikey K(const ppcb::OMKey& k) {
  ikey o;
  o.str = k.str;
  o.dom = k.dom;
  return o;
}

// refresh the exported geometry tables after a (re)load
static void publish() {
  const ppcb::Config& c = S().eng.cfg;
  i3oms.clear();
  for (const ppcb::GeoOM& g : c.i3oms) {
    OM om;
    om.R = g.d.R; om.F = g.d.F;
    om.r[0] = g.d.r[0]; om.r[1] = g.d.r[1]; om.r[2] = g.d.r[2];
    om.str = g.k.str; om.dom = g.k.dom;
    i3oms.push_back(om);
  }
  omts.clear();
  for (auto& e : c.omts) omts[K(e.first)] = e.second;
  hvs.clear();
  for (auto& e : c.hvs) hvs[K(e.first)] = e.second;
  rdes.clear();
  for (auto& e : c.rdes) rdes[K(e.first)] = e.second;
  nextgen = c.nextgen;
}

float xrnd() { return S().xrnd(); }
float grnd() { return S().grnd(); }

void start() {}

void stop() {
  std::cerr << "Device time: " << S().eng.total_device_ms() << " [ms]" << std::endl;
}

void choose(int device) { run([&] { S().choose(device); }); }
void ini() { run([&] { S().ini(); }); }
void fin() { run([&] { S().fin(); }); }
void eout() { run([&] { S().eout(); }); }
void flone(unsigned long long num) { run([&] { S().flone(num); }); }

size_t getMaxBunchSize() { return S().eng.pmxo; }
size_t getWorkgroupSize() { return S().eng.devs.empty() ? 0 : S().eng.devs[0].shape.threads; }
float getTotalDeviceTime() { return (float)S().eng.total_device_ms(); }

void initialize(float enh) {
  run([&] {
    S().initialize("", enh);
    publish();
  });
}

const DOM& flset(int str, int dom) {
  static DOM d;
  run([&] {
    const ppcb_dom& x = S().flset(str, dom);
    d.R = x.R; d.F = x.F;
    d.r[0] = x.r[0]; d.r[1] = x.r[1]; d.r[2] = x.r[2];
  });
  return d;
}

const float* fldir() { return S().fldir(); }
void flshift(float m[], float n[], float* r) { S().flshift(m, n, r); }
void set_res(float t) { S().set_res(t); }
void set_res(float t, float c) { S().set_res(t, c); }
void efin() { S().efin(); }

void sett(float nx, float ny, float nz, std::pair<int, unsigned long long> id, int frame, double t0) {
  run([&] { S().sett(nx, ny, nz, id, frame, t0); });
}

void addp(float x, float y, float z, float t, float E, float dr, int type, float scale) {
  run([&] { S().addp(x, y, z, t, E, dr, type, scale); });
}

void addp_clst(float x, float y, float z, float t, unsigned long long n, float dr, float beta) {
  run([&] { S().addp_clst(x, y, z, t, n, dr, beta); });
}

void addp_mopo(float x, float y, float z, float t, float light, float length, float beta, float tau, float fr) {
  run([&] { S().addp_mopo(x, y, z, t, light, length, beta, tau, fr); });
}

}  // namespace xppc
