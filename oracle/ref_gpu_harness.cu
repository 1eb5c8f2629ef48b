// MEASUREMENT INFRASTRUCTURE ONLY -- never linked into the product.
//
// The reference's own CUDA build: gpu/ppc.cu (with gpu/ini.cxx, gpu/pro.cu, gpu/f2k.cxx)
// compiled by nvcc with the reference's flags (gpu/Makefile:7-8: -O2 --use_fast_math
// --maxrregcount=64) for sm_100a, in library mode (-DXLIB).  This is the "plain kernel"
// baseline: the reference's propagate() on a B200, driven by its own kernel()
// (gpu/ppc.cu:432-469) exactly as eout() does, one source per launch.  Build recipe:
// oracle/Makefile (target ref_gpu); output in oracle/_ref/.
//
// usage: ref_gpu_harness <spec> <photons-per-event> <events> [seed]
//   spec as in ref_harness.cxx ("cascade:x:y:z:E:nx:ny:nz:type", "flasher:str:om", "point:x:y:z")
// prints one JSON line: photons, hits, device milliseconds (the reference's own CUDA-event
// timing of its launches, gpu/ppc.cu:296-304), wall seconds.
#include "ppc.cu"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace xppc;

int main(int argc, char** argv) {
  if (argc < 4) { fprintf(stderr, "usage: ref_gpu_harness spec photons events [seed]\n"); return 2; }
  std::string spec = argv[1];
  unsigned long long photons = strtoull(argv[2], 0, 10);
  int events = atoi(argv[3]);
  if (argc > 4) sv = strtoul(argv[4], 0, 10);
  start();
  initialize(1.f);
  choose(0);
  ini();
  std::vector<std::string> tok;
  {
    size_t a = 0, b;
    while ((b = spec.find(':', a)) != std::string::npos) { tok.push_back(spec.substr(a, b - a)); a = b + 1; }
    tok.push_back(spec.substr(a));
  }
  if (tok[0] == "flasher") flset(atoi(tok[1].c_str()), atoi(tok[2].c_str()));
  else if (tok[0] == "point") {
    flset(0, 0);
    p.r.x = atof(tok[1].c_str()); p.r.y = atof(tok[2].c_str()); p.r.z = atof(tok[3].c_str());
  }
  auto t0 = std::chrono::steady_clock::now();
  unsigned long long done = 0, nhits = 0;
  if (tok[0] == "file") {
    // one event per line: "F <str> <om> <photons>" (flasher set up by flset from FLDR/ELEV)
    // or "C <x> <y> <z> <E> <nx> <ny> <nz> <photons>" (EM cascade)
    FILE* f = fopen(tok[1].c_str(), "r");
    if (!f) { perror(tok[1].c_str()); return 2; }
    char kind[4];
    int ev = 0;
    while (fscanf(f, "%3s", kind) == 1) {
      unsigned long long n = 0;
      if (kind[0] == 'F') {
        int str, om;
        if (fscanf(f, "%d %d %llu", &str, &om, &n) != 3) break;
        flset(str, om);
      } else {
        float x, y, zz, E, nx, ny, nz;
        if (fscanf(f, "%f %f %f %f %f %f %f %llu", &x, &y, &zz, &E, &nx, &ny, &nz, &n) != 8) break;
        p.r.x = x; p.r.y = y; p.r.z = zz; p.r.w = 0;
        p.n.x = nx; p.n.y = ny; p.n.z = nz;
        p.type = -11; p.beta = 1; p.tau = 0;
        yield(E, 0, 11);
      }
      mcid id; id.first = ev; id.second = 0; id.frame = 0; id.t0 = 0;
      flnz.push_back(id); finc(); p.q = flne;
      addh(n);
      eout();
      for (auto i = hitz.begin(); i != hitz.end(); ++i) nhits += i->second.size();
      efin();
      done += n;
      ev++;
    }
    fclose(f);
    events = ev;
  }
  for (int ev = 0; ev < events && tok[0] != "file"; ev++) {
    if (tok[0] == "cascade") {
      p.r.x = atof(tok[1].c_str()); p.r.y = atof(tok[2].c_str()); p.r.z = atof(tok[3].c_str()); p.r.w = 0;
      p.n.x = atof(tok[5].c_str()); p.n.y = atof(tok[6].c_str()); p.n.z = atof(tok[7].c_str());
      int type = atoi(tok[8].c_str());
      p.type = -type; p.beta = 1; p.tau = 0;
      yield(atof(tok[4].c_str()), 0, type);
    }
    // one segment per event (gpu/f2k.cxx:548-552) and exactly `photons` photons
    mcid id; id.first = ev; id.second = 0; id.frame = 0; id.t0 = 0;
    flnz.push_back(id); finc(); p.q = flne;
    addh(photons);
    eout();
    for (auto i = hitz.begin(); i != hitz.end(); ++i) nhits += i->second.size();
    efin();
    done += photons;
  }
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("{\"photons\": %llu, \"events\": %d, \"accepted_hits\": %llu, \"device_ms\": %.3f, \"wall_s\": %.6f}\n",
         done, events, nhits, getTotalDeviceTime(), wall);
  fin();
  return 0;
}
