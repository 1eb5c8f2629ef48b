// Command-line program with the reference's modes and output (gpu/ppc.cu:524-598,
// doc/index.rst "Command-line parameters"):
//   ppc                         list devices and usage
//   ppc - [x y]                 ice table at the middle wavelength bin
//   ppc =                       read "x y z" lines, append tilt shift and layer thickness
//   ppc _                       tilt surface grid
//   ppc <dev>                   f2k particles from stdin, HIT lines to stdout
//   ppc <str> <om> <num[*n]> <dev>   flasher / standard candle
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "session.h"
#include "tilt.h"

using namespace ppcb;

namespace {

struct HostTilt {
  const Config& c;
  float lr(int i) const { return c.lr[i]; }
  int mcol(int x, int y) const {
    return x >= 0 && x < c.p.mnum[0] && y >= 0 && y < c.p.mnum[1] ? c.mcol[x * PPCB_CTY + y] : -1;
  }
  float2 lp(int i, int k) const {
    float2 v;
    v.x = c.lp[(i * PPCB_LYRS + k) * 2];
    v.y = c.lp[(i * PPCB_LYRS + k) * 2 + 1];
    return v;
  }
};

float zshift_host(const Config& c, float x, float y, float z, float& dz) {
  HostTilt t{c};
  dz = c.p.dh;
  return zshift_t(c.p, t, x, y, z, dz);
}

void list_devices() {
  int n = 0, drv = 0, rt = 0;
  cudaGetDeviceCount(&n);
  cudaDriverGetVersion(&drv);
  cudaRuntimeGetVersion(&rt);
  fprintf(stderr, "Found %d devices, driver %d, runtime %d\n", n, drv, rt);
  for (int d = 0; d < n; d++) {
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, d);
    fprintf(stderr, "%d(%d.%d): %s G(%lu) S(%lu) M(%d)\n", d, p.major, p.minor, p.name,
            (unsigned long)p.totalGlobalMem, (unsigned long)p.sharedMemPerBlock, p.multiProcessorCount);
  }
  fprintf(stderr, "\n");
}

// f2k reader: one segment per input line, TR records become sources (gpu/f2k.cxx:555-583)
void f2k(Session& s) {
  std::string in;
  while (std::getline(std::cin, in)) {
    s.sett_line(in);
    F2kTrack tr;
    if (parse_f2k_track(in, tr)) {
      s.p.q = s.flne;
      s.p.n[0] = tr.n[0]; s.p.n[1] = tr.n[1]; s.p.n[2] = tr.n[2];
      if (tr.type == -2) s.addf(tr.x, tr.y, tr.z, tr.t, (unsigned long long)tr.E);
      else if (tr.type >= 0) s.addp(tr.x, tr.y, tr.z, tr.t, tr.E, tr.l, tr.type);
    }
  }
  s.eout();
}

// gpu/f2k.cxx:768-783
void flasher(Session& s, int str, int dom, unsigned long long num, int itr) {
  s.flset(str, dom);
  for (int j = 0; j < std::max(1, itr); j++) {
    s.p.q = s.flne;
    s.flone(num);
    if (itr > 0) s.sett_line("");
  }
  s.eout();
}

}  // namespace

int main(int argc, char** argv) {
  Session s;
  s.hit_out = stdout;
  try {
    if (argc <= 1) {
      list_devices();
      fprintf(stderr, "Use: %s [device] (f2k muons)\n     %s [str] [om] [num] [device] (flasher)\n", argv[0], argv[0]);
    } else if (!strcmp(argv[1], "-")) {
      s.initialize("", 1.f);
      const Config& c = s.eng.cfg;
      const int w = PPCB_WNUM / 2;
      const ppcb_wmeta& m = c.wmeta[w];
      std::cerr << "For wavelength=" << c.wvs[m.wvl].w << " [nm]  np=" << (1 / m.coschr) << "  cm=" << 1 / m.ocm
                << " [m/ns]" << std::endl;
      float x = 0, y = 0;
      if (argc == 4) { x = atof(argv[2]); y = atof(argv[3]); }
      for (int i = 0; i < c.p.size; i++) {
        float z = c.p.hmin + c.p.dh * i, dz;
        float rz = z;
        for (int j = 0; j < 10; j++) rz = z + zshift_host(c, x, y, rz, dz);
        z = rz;
        const float* ab = &c.absca[((size_t)w * c.p.size + i) * 2];
        std::cout << z << " " << ab[0] << " " << ab[1] * (1 - c.p.g) << " " << c.az[i].ra * c.p.sum << std::endl;
      }
    } else if (!strcmp(argv[1], "=")) {
      s.initialize("", 1.f);
      const Config& c = s.eng.cfg;
      std::string in;
      while (std::getline(std::cin, in)) {
        float x, y, z, dz;
        if (3 == sscanf(in.c_str(), "%f %f %f", &x, &y, &z)) {
          float v = zshift_host(c, x, y, z, dz);
          std::cout << in << " " << v << " " << dz << std::endl;
        }
      }
    } else if (!strcmp(argv[1], "_")) {
      s.initialize("", 1.f);
      const Config& c = s.eng.cfg;
      for (float x = -750.f; x < 751.f; x += 3.f)
        for (float y = -750.f; y < 751.f; y += 3.f)
          for (float z = -750.f; z < 751.f; z += 6.f) {
            float rz = z, dz;
            for (int j = 0; j < 10; j++) rz = z + zshift_host(c, x, y, rz, dz);
            std::cout << z << " " << x << " " << y << " " << (rz - z) << std::endl;
          }
    } else if (argc <= 2) {
      int device = atoi(argv[1]);
      s.initialize("", 1.f);
      s.choose(device);
      fprintf(stderr, "Processing f2k muons from stdin on device %d\n", device);
      s.ini();
      f2k(s);
      s.fin();
    } else {
      int str = atoi(argv[1]), dom = argc > 2 ? atoi(argv[2]) : 0, device = 0, itr = 0;
      unsigned long long num = 1000000ULL;
      if (argc > 3) {
        num = (unsigned long long)atof(argv[3]);
        const char* sub = strchr(argv[3], '*');
        if (sub != nullptr) itr = (int)atof(++sub);
      }
      if (argc > 4) device = atoi(argv[4]);
      s.initialize("", 1.f);
      s.choose(device);
      fprintf(stderr, "Running flasher simulation on device %d\n", device);
      s.ini();
      flasher(s, str, dom, num, itr);
      s.fin();
    }
    fprintf(stderr, "\nDevice time: %2.1f [ms]\n", s.eng.total_device_ms());
  } catch (const Error& e) {
    std::cerr << e.what() << std::endl;
    return e.code ? e.code : 1;
  }
  return 0;
}
