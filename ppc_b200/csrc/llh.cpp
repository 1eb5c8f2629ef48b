// Observed side of DirectFit's likelihood, prepared on the host once per event:
//   reading the pulses      llh/llh.cxx:739-796 (bad DOMs, errata windows, drep scaling)
//   bin width and origin    llh/llh.cxx:798-806
//   dat::prep               llh/llh.cxx:436-450 (200 bins, end bins cut)
//   dat::optimize           llh/llh.cxx:516-612 (peak window, Bayesian-blocks partition)
//   dat::in                 llh/llh.cxx:664-666 (charge and flasher selection)
// The simulated side runs on the GPU (llh.cu).
#include "llh.h"

#include <cmath>
#include <cstdlib>
#include <limits>
#include <map>
#include <set>
#include <string>
#include <utility>

#include "engine.h"

namespace ppcb {

namespace {

constexpr int N = Likelihood::kBins;

typedef std::pair<int, int> Key;

struct Pulse {
  float t, q;  // the reference keeps pulses as float (llh/llh.cxx:378-385)
};

struct Observed {
  std::vector<Pulse> pulses;
  std::vector<std::pair<double, double>> windows;

  bool outside_windows(double t) const {
    for (const auto& w : windows)
      if (w.first <= t && t < w.second) return false;
    return true;
  }
};

// log L! as lgamma(L + 1); the reference calls GSL's gsl_sf_lnfact
double lnfact(int L) { return std::lgamma(L + 1.0); }

// the score of one block of L bins holding charge D (dat::G with the flat prior)
double block_score(int L, double D) { return (D <= 0 ? 0.0 : D * std::log(D / L)) + lnfact(L); }

// Best partition of x[0..n) into blocks by dynamic programming over the last block's start.
// With `rising`, a block is allowed only if its rate is above the previous block's (peak
// search); `mono` (with top >= 0) makes rates rise before bin `top` and fall after it.
// Fills score[], rate[] and start[] per end bin.
void partition(const double* x, int n, bool rising, bool mono, int top, double* score, double* rate, int* start) {
  for (int e = 0; e < n; e++) {
    double sum = 0, best = 0, best_rate = 0;
    int best_start = -1;
    for (int b = e; b >= 0; b--) {
      sum += x[b];
      const int len = e - b + 1;
      double s = block_score(len, sum);
      const double r = sum / len;
      if (b > 0) s += score[b - 1];
      bool allowed = true;
      if (rising) allowed = b == 0 || rate[b - 1] < r;
      else if (mono) allowed = b == 0 || (rate[b - 1] - r) * (b - 0.5 - top) > 0;
      if (allowed && (best_start == -1 || s > best)) {
        best = s;
        best_rate = r;
        best_start = b;
      }
    }
    score[e] = best;
    rate[e] = best_rate;
    if (start) start[e] = best_start;
  }
}

// The same from the right: blocks of x[e..n) with rates above the next block's.
void partition_falling(const double* x, int n, double* score, double* rate) {
  for (int e = n - 1; e >= 0; e--) {
    double sum = 0, best = 0, best_rate = 0;
    int best_end = -1;
    for (int b = e; b < n; b++) {
      sum += x[b];
      const int len = b - e + 1;
      double s = block_score(len, sum);
      const double r = sum / len;
      if (b < n - 1) s += score[b + 1];
      if ((b == n - 1 || rate[b + 1] < r) && (best_end == -1 || s > best)) {
        best = s;
        best_rate = r;
        best_end = b;
      }
    }
    score[e] = best;
    rate[e] = best_rate;
  }
}

struct Window {
  int n1, n2, top;
};

// The bins that take part (dat::optimize's first half): around the highest bin, or with
// `peak` around the split of the best rising-then-falling blocks.
Window choose_window(const double* bins, double lbin, bool peak) {
  const int before = (int)std::round(500 / lbin), after = (int)std::round(1000 / lbin);
  Window w;
  if (peak) {
    double s1[N], r1[N], s2[N], r2[N];
    partition(bins, N, true, false, -1, s1, r1, nullptr);
    partition_falling(bins, N, s2, r2);
    int m = -2;
    double best = 0;
    for (int n = -1; n < N; n++) {
      const double v = (n >= 0 ? s1[n] : 0) + (n < N - 1 ? s2[n + 1] : 0);
      if (m == -2 || v > best) m = n, best = v;
    }
    if (m == -1 || (m < N - 1 && r2[m + 1] > r1[m])) m++;
    w.n1 = std::max(0, m - before);
    int top = m;
    m = N + 1;
    best = 0;
    for (int n = N; n >= 0; n--) {
      const double v = (n < N ? s2[n] : 0) + (n > 0 ? s1[n - 1] : 0);
      if (m == N + 1 || v > best) m = n, best = v;
    }
    if (m == N || (m > 0 && r2[m] < r1[m - 1])) m--;
    w.n2 = std::min(m + after, N);
    w.top = (m + top) / 2;
  } else {
    int hi = 0;
    double vmax = 0;
    for (int i = 0; i < N; i++)
      if (bins[i] > vmax) vmax = bins[i], hi = i;
    w.n1 = std::max(0, hi - before);
    int top = hi;
    for (int i = N - 1; i > hi; i--)
      if (bins[i] == vmax) {
        hi = i;
        break;
      }
    w.n2 = std::min(hi + after, N);
    w.top = (hi + top) / 2;
  }
  return w;
}

}  // namespace

Likelihood::Likelihood(Engine& e, int device, const ppcb_llh_hit* data, uint64_t n, const ppcb_llh_window* wins,
                       uint64_t nwin, const int32_t* bad, uint64_t nbad, const ppcb_llh_opts& o)
    : opts(o), eng_(e), dev_(device) {
  if (e.cfg.p.gsize <= 0) throw Error("ppcb_initialize() must come before the likelihood", 6);
  if (device < 0 || (e.ready() && device >= (int)e.devs.size())) throw Error("bad device index", 7);
  if (!(o.drep > 0) || !(o.sig >= 0)) throw Error("likelihood options: drep > 0 and sig >= 0 are required", 7);
  std::set<Key> badset;
  for (uint64_t k = 0; k < nbad; k++) badset.insert(Key(bad[2 * k], bad[2 * k + 1]));
  std::map<Key, Observed> all;
  for (uint64_t k = 0; k < nwin; k++) all[Key(wins[k].str, wins[k].om)].windows.push_back({wins[k].ti, wins[k].tf});
  double tmin = std::numeric_limits<double>::quiet_NaN(), tmax = tmin;
  for (uint64_t k = 0; k < n; k++) {
    const ppcb_llh_hit& h = data[k];
    OMKey om{h.str, h.om};
    if (!om.isinice() || badset.count(Key(h.str, h.om))) continue;
    if (std::isnan(tmin) || h.t < tmin) tmin = h.t;
    if (std::isnan(tmax) || h.t > tmax) tmax = h.t;
    const double q = h.q * o.drep;
    if (q > 0) all[Key(h.str, h.om)].pulses.push_back({(float)h.t, (float)q});
  }
  if (std::isnan(tmin)) throw Error("likelihood: no observed pulses on in-ice DOMs", 7);
  if (o.lbin > 0) lbin = o.lbin;
  else {
    const double span = (tmax - tmin + 1) / N;
    lbin = span > kBin ? span : kBin;
  }
  if (std::round(1000 / lbin) < 1)
    throw Error("likelihood: time bins wider than 2000 ns leave no bins after the peak", 7);
  t0 = tmin;

  ndof = 1;
  for (const auto& kv : all) {
    const Observed& ob = kv.second;
    double bins[N] = {0};
    double dtot = 0, qtot = 0;
    for (const Pulse& p : ob.pulses) {  // dat::prep
      qtot += p.q;
      if (!ob.outside_windows(p.t)) continue;
      double k = std::round((p.t - t0) / lbin), q = p.q;
      if (k < 0 || k >= N) q = 0;
      if (k < 0) k = 0;
      else if (k >= N) k = N - 1;
      bins[(int)k] += q;
      dtot += q;
    }
    const bool in = qtot < o.qsat * o.drep && qtot > o.qmin * o.drep &&
                    (!o.flasher || kv.first.first != std::abs(o.fla_str) ||
                     std::abs(kv.first.second - o.fla_om) > o.fsep);
    if (!in) continue;
    const Window w = choose_window(bins, lbin, o.peak != 0);
    const int ntop = w.n2 - w.n1;
    if (ntop <= 0)
      throw Error("likelihood: empty bin window on DOM " + std::to_string(kv.first.first) + "-" +
                  std::to_string(kv.first.second), 7);
    double score[N], rate[N];
    int start[N];
    partition(bins + w.n1, ntop, false, o.mono != 0, w.top - w.n1, score, rate, start);
    LlhDom D{};
    D.str = kv.first.first;
    D.om = kv.first.second;
    D.n1 = w.n1;
    D.n2 = w.n2;
    D.block0 = (int32_t)blocks.size();
    D.bin0 = (int32_t)bin_block.size();
    D.win0 = (int32_t)(win.size() / 2);
    D.nwin = (int32_t)ob.windows.size();
    D.dtot = dtot;
    for (const auto& x : ob.windows) win.push_back(x.first), win.push_back(x.second);
    bin_block.resize(bin_block.size() + ntop);
    for (int f = ntop - 1;;) {  // blocks from the last bin backwards (dat::optimize's tail)
      const int k = start[f];
      double d = 0;
      ppcb_llh_block B;
      B.str = D.str;
      B.om = D.om;
      B.first = w.n1 + k;
      B.last = w.n1 + f;
      for (; f >= k; f--) {
        d += bins[w.n1 + f];
        bin_block[D.bin0 + f] = (int32_t)blocks.size();
      }
      B.dat = d;
      block_dom.push_back((int32_t)doms.size());
      blocks.push_back(B);
      if (k == 0) break;
    }
    D.nblock = (int32_t)blocks.size() - D.block0;
    ndof += D.nblock;
    doms.push_back(D);
  }

  // where each sensor's simulated hits go
  std::map<Key, int> slot;
  for (size_t k = 0; k < doms.size(); k++) slot[Key(doms[k].str, doms[k].om)] = (int)k;
  const Config& c = e.cfg;
  dom_slot.assign(c.p.gsize, -2);
  for (int i = 0; i < c.p.gsize; i++) {
    const Key k(c.names[i].k.str, c.names[i].k.dom);
    if (badset.count(k)) continue;
    auto s = slot.find(k);
    if (s != slot.end()) dom_slot[i] = s->second;
    else if (!all.count(k)) dom_slot[i] = -1;
  }
  if (e.ready()) upload();  // otherwise on the first evaluation after ppcb_ini()
}

}  // namespace ppcb
