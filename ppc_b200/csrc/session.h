// Session: everything between the caller's sources and the device runtime.
//   front end  -- light yield, Poisson sampling, LED/flasher set-up, bunch packing
//                 (gpu/f2k.cxx:17-167, :377-385, :403-528, :586-759)
//   pipeline   -- batches of at most pmax photons / pmxo bunches, double buffered
//                 (gpu/ppc.cu:432-469, gpu/f2k.cxx:365-375, :536-541)
//   back end   -- per-hit acceptance (wavelength x RDE), PMT choice, cable shadow,
//                 then HIT lines or the binned `hitz` map (gpu/f2k.cxx:237-363)
#pragma once
#include <cstdio>
#include <deque>
#include <string>
#include <vector>

#include "../../include/xppc.h"
#include "engine.h"

namespace ppcb {

// One TR record of an f2k line (gpu/f2k.cxx:559-582): the source it makes (type >= 0 a
// particle for addp, -2 an exact photon count "ph" for addf, -1 none), its position, time,
// direction, length and energy.
struct F2kTrack {
  int type = -1;
  float x = 0, y = 0, z = 0, t = 0, l = 0, E = 0;
  float n[3] = {0, 0, 0};
};
// False when the line is not a TR record.
bool parse_f2k_track(const std::string& line, F2kTrack& tr);

class Session {
 public:
  Engine eng;

  // ---- lifecycle
  void initialize(const std::string& dir, float enh);
  void choose(int device) { eng.choose(device); }
  void ini();
  void fin();

  // ---- sources (reference semantics)
  float yield(float E, float dr, int type);
  void addh(unsigned long long num);
  void addf(float rx, float ry, float rz, float t, unsigned long long num);
  void addp(float rx, float ry, float rz, float t, float E, float dr, int type, float scale = 1);
  void addp_clst(float rx, float ry, float rz, float t, unsigned long long n, float dr, float beta);
  void addp_mopo(float rx, float ry, float rz, float t, float light, float length, float beta, float tau, float fr);
  void flone(unsigned long long num);
  const ppcb_dom& flset(int str, int dom);
  const float* fldir();
  void flshift(float m[], float n[], float* r = nullptr);
  void sett(float nx, float ny, float nz, std::pair<int, unsigned long long> id, int frame, double t0 = 0);
  void sett_line(const std::string& line);   // CLI f2k: the echoed input line is the segment id
  void finc();
  void eout();
  void efin() { hitz->clear(); raw_.clear(); }
  void set_res(float t) { trz_ = t; }
  void set_res(float t, float c) { trz_ = t; crz_ = c; }

  // ---- host random numbers (rand_r on the shared seed, gpu/f2k.cxx:1-10)
  float xrnd();
  float grnd();
  unsigned long long poidev(double xm);
  unsigned long long bnldev(unsigned long long n, double pp);

  // ---- results
  xppc::outz own_hitz;
  xppc::outz* hitz = &own_hitz;      // library mode: binned hits (xppc::hitz for the drop-in)
  FILE* hit_out = nullptr;           // CLI mode: HIT lines (and echoed segments) here
  bool keep_raw = false;             // also keep kernel-level hits (C ABI)
  std::vector<ppcb_hit> raw_;        // kernel-level hits, segment id in .n
  RunInfo last;                      // totals of the last collected batch
  RunInfo total;                     // totals since ini()

  // back end on an explicit hit list (also used by tests)
  void print(std::vector<ppcb_hit>& hits, unsigned int flnd);

  ppcb_bunch p{}, pfl{};
  unsigned int flnb = 0, flne = 0;

 private:
  void output();
  void kernel(uint64_t num);
  void collect_one();
  struct Seg {
    bool is_line;
    std::string line;
    xppc::mcid id;
  };
  std::deque<Seg> flnz_;
  std::deque<unsigned int> flnd_q_;  // flne at submission, per batch in flight
  std::vector<ppcb_bunch> pz_;       // pending bunches of the next batch
  uint64_t pn_ = 0;                  // pending photons
  float trz_ = 0, crz_ = 0;
  xppc::ihit tmph_{};
  ppcb_dom flom_{};
  float fldir_[3] = {0, 0, 0};
  bool fldir_set_ = false;
};

}  // namespace ppcb
