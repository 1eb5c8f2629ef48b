// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// Harness around the reference's own DirectFit likelihood: llh/llh.cxx (with its
// llh/lssl.cxx and llh/nnls.cxx) compiled unmodified, against the GSL stand-in of
// oracle/gsl_shim (GSL is not installed here) and the reference's CPU library gpu/ppc.cu
// built with -DXLIB, as llh/Makefile's `cpu` target links it.  Its main() is renamed; this
// one drives the reference's own code:
//   * xyz::ini (llh/llh.cxx:739-877) reads the observed pulses ("dat"), the errata windows
//     ("ert") and the bad-DOM list ("bad") from the working directory and prepares every
//     DOM (dat::prep, dat::optimize: binning and the Bayesian-blocks partition);
//   * simulated hits are added to the DOMs as cascade::ppc does (llh/llh.cxx:1686-1703), one
//     unit of charge each, their times relative to the event's time origin;
//   * fllh (llh/llh.cxx:1075-1082) is evaluated at the given time shifts.
//
// usage: llh_harness <dir> <sim> <nsim> <dt,dt,...> [norm] [mono] [peak] [qsat=X] [drep=N]
//                    [sig=X] [flasher=STR:OM:FSEP]
//   <sim>: lines "str om t" (t on the observed clock).  Prints one JSON object: lbin, t0,
//   ndof, the blocks of every DOM in the fit (str, om, first bin, last bin, observed charge)
//   in the reference's order, and fllh at each shift.
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define main llh_reference_main
#include "llh.cxx"
#undef main

int main(int argc, char** argv) {
  if (argc < 5) { fprintf(stderr, "usage: see header\n"); return 2; }
  const char* dir = argv[1];
  const char* simf = argv[2];
  const double nsim = atof(argv[3]);
  std::vector<double> dts;
  for (char* p = strtok(argv[4], ","); p; p = strtok(NULL, ",")) dts.push_back(atof(p));
  for (int k = 5; k < argc; k++) {
    std::string a = argv[k];
    if (a == "norm") norm = true;
    else if (a == "mono") mono = true;
    else if (a == "peak") peak = true;
    else if (a.rfind("qsat=", 0) == 0) qsat = atof(a.c_str() + 5);
    else if (a.rfind("drep=", 0) == 0) drep = atoi(a.c_str() + 5);
    else if (a.rfind("sig=", 0) == 0) LSSL::SIG = atof(a.c_str() + 4);
    else if (a.rfind("flasher=", 0) == 0) {
      int s, o, f;
      if (sscanf(a.c_str() + 8, "%d:%d:%d", &s, &o, &f) != 3) { fprintf(stderr, "bad flasher\n"); return 2; }
      flasher = true; fla = make_pair(s, o); fsep = f;
    } else { fprintf(stderr, "bad option %s\n", a.c_str()); return 2; }
  }
  xppc::initialize(1.f);  // geometry and high voltages (xppc::i3oms, hvs) for ini()
  if (chdir(dir) != 0) { perror(dir); return 2; }
  xyz ev;
  ev.ini();
  {
    FILE* f = fopen(simf, "r");
    if (!f) { perror(simf); return 2; }
    int str, om;
    double t;
    while (fscanf(f, "%d %d %lf", &str, &om, &t) == 3) {
      xkey k(make_pair(str, om), 0);
      if (!isok(k)) continue;
      map<xkey, dat>::iterator i = all.find(k);
      if (i == all.end()) { if (unh) nohit += 1; }
      else i->second.sraw.push_back(hix((float)(t - tshift), 1.f, NAN));
    }
    fclose(f);
  }
  printf("{\"lbin\": %.17g, \"t0\": %.17g, \"ndof\": %u, \"blocks\": [", lbin, tshift, ndof);
  bool first = true;
  for (map<xkey, dat>::iterator i = all.begin(); i != all.end(); ++i) {
    dat& d = i->second;
    if (!d.in()) continue;
    int f = d.ntop - 1;
    for (int b = 0; b < d.fnum; b++) {
      const int k = d.lastchange[f];
      printf("%s[%d, %d, %d, %d, %.17g]", first ? "" : ", ", i->first.first, i->first.second, d.n1 + k, d.n1 + f,
             d.dat[b]);
      first = false;
      f = k - 1;
    }
  }
  printf("], \"fllh\": [");
  for (size_t j = 0; j < dts.size(); j++) printf("%s%.17g", j ? ", " : "", fllh(dts[j], nsim));
  printf("]}\n");
  return 0;
}
