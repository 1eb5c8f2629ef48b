// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// Harness around the reference implementation itself: this file is compiled together
// with the reference's unmodified gpu/ppc.cu (which pulls in gpu/ini.cxx, gpu/pro.cu and
// gpu/f2k.cxx), as the reference's CPU build (`$(CXX) -x c++ ppc.cu -O2 --fast-math`,
// gpu/Makefile:10) with -DXLIB (library mode, gpu/Makefile:12-13) and -DDTMN
// (deterministic seeding, gpu/ini.cxx:28,792-795).  Build recipe: oracle/Makefile;
// output goes to oracle/_ref/ only.
//
// It exposes what the reference computes but does not print: the table image built by
// ini::set (gpu/ini.cxx:578-1700), zshift (gpu/pro.cu:168-264) at given points, the
// phase-1 photon records and the kernel-level hit records of propagate
// (gpu/pro.cu:287-904) driven exactly as the CPU build's kernel() does
// (gpu/ppc.cu:432-442), and a timing mode used as the CPU baseline.
//
// usage:
//   ref_harness tables <out.bin>
//   ref_harness zshift <in.f32x4> <out.f32x3>
//   ref_harness yield <in> <out>
//      in: (f32 E, f32 dr, i32 type, f32 scale) per source; out: (f32 mean, f32 f, f32 a,
//      f32 b, f32 length, f32 yield) per source -- the bunch template addp() makes and the
//      Poisson mean it samples (gpu/f2k.cxx:17-167, 484-504)
//   ref_harness backend <hits> <seed> <out>
//      the reference's own back end (print, gpu/f2k.cxx:247-363) over kernel-level hit
//      records of one segment (n = 1, sett id (3, 9)), with the host random state sv = seed;
//      out: the hit map, one 80-byte record per photon (track, str, om, pmt, dir, time,
//      r[4], n[4]) in the map's order
//   ref_harness frontend <sources> <seed>
//      times the reference's own front end (addp: yield, poidev, addh; gpu/f2k.cxx:17-167,
//      377-504) over (f32 x, y, z, t, E, dr, i32 type) per source; the bunches are dropped
//      before a batch fills, so no propagation runs.  Prints photons and seconds.
//   ref_harness run <spec> <photons> <seed> <out-prefix> [nodump | hits]
//      writes <out-prefix>.hits, .pbuf and .bunch; "nodump" writes nothing (timing),
//      "hits" only the kernel-level hit records (high-statistics runs)
//      spec = "flasher:<str>:<om>" | "cascade:<x>:<y>:<z>:<E>:<nx>:<ny>:<nz>:<type>"
//           | "point:<x>:<y>:<z>"   (isotropic point source, FWID=-1 style, at x,y,z)
#include "ppc.cu"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace xppc;

static FILE* xopen(const char* path, const char* mode) {
  FILE* f = fopen(path, mode);
  if (!f) { perror(path); exit(2); }
  return f;
}

// record: name[32] | elem size u32 | count u64 | bytes
static void put(FILE* f, const char* name, const void* p, unsigned int esz, unsigned long long n) {
  char nm[32] = {0};
  strncpy(nm, name, 31);
  fwrite(nm, 1, 32, f);
  fwrite(&esz, 4, 1, f);
  fwrite(&n, 8, 1, f);
  fwrite(p, esz, n, f);
}

static void dump_tables(const char* out) {
  FILE* f = xopen(out, "wb");
#define S(field) put(f, #field, &d.field, sizeof(d.field), 1)
  S(size); S(dh); S(rdh); S(hmin); S(ocv); S(sf); S(g); S(gr); S(xR); S(SF); S(G); S(GR);
  S(hr); S(hr2); S(hs); S(ha); S(azx); S(azy); S(tmod); S(vthk); S(lnum); S(lpts); S(l0);
  S(lmin); S(lrdz); S(r0); S(lnx); S(lny); S(k1); S(k2); S(kz); S(fr); S(sum); S(rx); S(hifl);
  S(gsize); S(rsize);
#undef S
  put(f, "cn", d.cn, 4, 2); put(f, "cl", d.cl, 4, 2); put(f, "crst", d.crst, 4, 2);
  put(f, "cb", d.cb, 4, 4); put(f, "mmin", d.mmin, 4, 2); put(f, "mstp", d.mstp, 4, 2);
  put(f, "mnum", d.mnum, 4, 2); put(f, "mcut", d.mcut, 4, 2); put(f, "bfr", d.bfr, 4, 12);
  put(f, "az", d.az, sizeof(aniz), d.size);
  put(f, "lr", d.lr, 4, LMAX);
  put(f, "ls", d.ls, 2, NSTR);
  put(f, "is", d.is, 2, CX * CY);
  put(f, "mcol", d.mcol, 1, CTX * CTY);
  put(f, "sc", d.sc, sizeof(line), NSTR);
  put(f, "lp", z.lp, 8, LMAX * LYRS);
  {
    std::vector<float> absca((size_t)WNUM * d.size * 2);
    std::vector<float> meta((size_t)WNUM * 4);
    for (int n = 0; n < WNUM; n++) {
      for (int i = 0; i < d.size; i++) {
        absca[((size_t)n * d.size + i) * 2] = z.w[n].z[i].abs;
        absca[((size_t)n * d.size + i) * 2 + 1] = z.w[n].z[i].sca;
      }
      meta[n * 4 + 0] = z.w[n].ocm;
      meta[n * 4 + 1] = z.w[n].coschr;
      meta[n * 4 + 2] = z.w[n].sinchr;
      memcpy(&meta[n * 4 + 3], &z.w[n].wvl, 4);
    }
    put(f, "absca", absca.data(), 4, absca.size());
    put(f, "wmeta", meta.data(), 4, meta.size());
  }
  put(f, "oms", q.oms, sizeof(DOM), d.gsize);
  put(f, "rm", z.rm, 4, d.rsize);
  {
    std::vector<float> w((size_t)WNUM * 3);
    for (int n = 0; n < WNUM; n++) { w[n * 3] = q.wvs[n].w; w[n * 3 + 1] = q.wvs[n].i; w[n * 3 + 2] = q.wvs[n].f; }
    put(f, "wvs", w.data(), 4, w.size());
  }
  put(f, "eff", &q.eff, 4, 1);
  fclose(f);
}

static void do_zshift(const char* in, const char* out) {
  FILE* fi = xopen(in, "rb");
  FILE* fo = xopen(out, "wb");
  float v[4];
  while (fread(v, 4, 4, fi) == 4) {
    float4 r;
    r.x = v[0]; r.y = v[1]; r.z = v[2]; r.w = v[3];
    float dz = d.dh;
    float s = zshift(d, r, dz);
    float o[3] = {s, dz, 0};
    fwrite(o, 4, 3, fo);
  }
  fclose(fi);
  fclose(fo);
}

// Drive propagate() exactly like the CPU build's kernel() (gpu/ppc.cu:436-442), but keep
// the raw hit records instead of handing them to print().
static unsigned long long launch(unsigned int num, std::vector<hit>& hits, std::vector<pbuf>* bufs) {
  d.hidx = 0;
  for (d.blockIdx = 0, d.gridDim = nblk, blockDim.x = nthr; d.blockIdx < d.gridDim; d.blockIdx++)
    for (threadIdx.x = 0; threadIdx.x < blockDim.x; threadIdx.x++) propagate(e, num);
  unsigned long long nh = d.hidx;
  unsigned int keep = d.hidx > d.hnum ? d.hnum : d.hidx;
  hits.insert(hits.end(), q.hits, q.hits + keep);
  if (bufs) bufs->insert(bufs->end(), d.bf, d.bf + num);
  return nh;
}

int main(int argc, char** argv) {
  if (argc < 2) { fprintf(stderr, "usage: see header\n"); return 2; }
  std::string mode = argv[1];
  if (mode == "tables" && argc >= 3) {
    initialize();
    dump_tables(argv[2]);
    return 0;
  }
  if (mode == "zshift" && argc >= 4) {
    initialize();
    do_zshift(argv[2], argv[3]);
    return 0;
  }
  if (mode == "yield" && argc >= 4) {
    initialize();
    FILE* f = xopen(argv[2], "rb");
    std::vector<float> out;
    struct { float E, dr; int type; float scale; } src;
    while (fread(&src, sizeof(src), 1, f) == 1) {
      p = photon();
      const float y = yield(src.E, src.dr, src.type);
      const float mean = src.scale * y / ovr;
      const float rec[6] = {mean, p.f, p.a, p.b, p.n.w, y};
      out.insert(out.end(), rec, rec + 6);
    }
    fclose(f);
    f = xopen(argv[3], "wb");
    fwrite(out.data(), sizeof(float), out.size(), f);
    fclose(f);
    return 0;
  }
  if (mode == "frontend" && argc >= 4) {
    struct { float x, y, z, t, E, dr; int type; } src;
    std::vector<decltype(src)> in;
    {
      FILE* f = xopen(argv[2], "rb");
      while (fread(&src, sizeof(src), 1, f) == 1) in.push_back(src);
      fclose(f);
    }
    initialize();
    choose(0);
    ini();
    sv = strtoul(argv[3], 0, 10);
    sett(0.3f, 0.4f, 0.8660254f, std::make_pair(1, 1ULL), 0);
    unsigned long long photons = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (size_t k = 0; k < in.size(); k++) {
      addp(in[k].x, in[k].y, in[k].z, in[k].t, in[k].E, in[k].dr, in[k].type);
      for (unsigned int j = 0; j < pk; j++) photons += q.pz[j].num;
      pn = 0;  // drop the bunches: only the front end is timed
      pk = 0;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("{\"sources\": %zu, \"photons\": %llu, \"seconds\": %.6f}\n", in.size(), photons, secs);
    return 0;
  }
  if (mode == "backend" && argc >= 5) {
    std::vector<hit> in;
    {
      FILE* f = xopen(argv[2], "rb");
      hit h;
      while (fread(&h, sizeof(hit), 1, f) == 1) in.push_back(h);
      fclose(f);
    }
    initialize();
    choose(0);
    ini();
    sv = strtoul(argv[3], 0, 10);
    sett(0, 0, 1, std::make_pair(3, 9ULL), 0);
    if (in.size() > d.hnum) { fprintf(stderr, "too many hits for one batch\n"); return 2; }
    std::copy(in.begin(), in.end(), q.hits);
    d.hidx = in.size();
    auto t0 = std::chrono::steady_clock::now();
    print();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("{\"hits\": %zu, \"seconds\": %.6f}\n", in.size(), secs);
    struct {
      int first, frame;
      unsigned long long second;
      double t0;
      int str, dom, pmt;
      float dir, time, r[4], n[4];
      unsigned int pad;
    } rec;
    FILE* f = xopen(argv[4], "wb");
    for (std::map<ihit, std::vector<pout> >::const_iterator i = hitz.begin(); i != hitz.end(); ++i)
      for (std::vector<pout>::const_iterator j = i->second.begin(); j != i->second.end(); ++j) {
        memset(&rec, 0, sizeof(rec));
        rec.first = i->first.track.first;
        rec.second = i->first.track.second;
        rec.frame = i->first.track.frame;
        rec.t0 = i->first.track.t0;
        rec.str = i->first.omkey.str;
        rec.dom = i->first.omkey.dom;
        rec.pmt = i->first.pmt;
        rec.dir = i->first.dir;
        rec.time = i->first.time;
        for (int k = 0; k < 4; k++) rec.r[k] = j->r[k], rec.n[k] = j->n[k];
        fwrite(&rec, sizeof(rec), 1, f);
      }
    fclose(f);
    fin();
    return 0;
  }
  if (mode == "run" && argc >= 6) {
    std::string spec = argv[2];
    unsigned long long total = strtoull(argv[3], 0, 10);
    unsigned int seedv = strtoul(argv[4], 0, 10);
    std::string outp = argv[5];
    const std::string opt = argc >= 7 ? argv[6] : "";
    const bool dump = opt != "nodump" && opt != "hits";
    const bool keep_hits = opt != "nodump";
    initialize();
    sv = seedv;      // DTMN leaves sv at 0; the caller picks the stream start
    choose(0);
    ini();
    // build the bunch template p
    std::vector<std::string> tok;
    {
      size_t a = 0, b;
      while ((b = spec.find(':', a)) != std::string::npos) { tok.push_back(spec.substr(a, b - a)); a = b + 1; }
      tok.push_back(spec.substr(a));
    }
    if (tok[0] == "flasher") {
      flset(atoi(tok[1].c_str()), atoi(tok[2].c_str()));
    } else if (tok[0] == "point") {
      flset(0, 0);  // str=0, om=0: point at the origin, FWID from the environment
      p.r.x = atof(tok[1].c_str()); p.r.y = atof(tok[2].c_str()); p.r.z = atof(tok[3].c_str());
    } else if (tok[0] == "cascade") {
      p.r.x = atof(tok[1].c_str()); p.r.y = atof(tok[2].c_str()); p.r.z = atof(tok[3].c_str()); p.r.w = 0;
      float E = atof(tok[4].c_str());
      p.n.x = atof(tok[5].c_str()); p.n.y = atof(tok[6].c_str()); p.n.z = atof(tok[7].c_str());
      int type = atoi(tok[8].c_str());
      p.type = -type; p.beta = 1; p.tau = 0;
      yield(E, 0, type);
    } else { fprintf(stderr, "bad spec\n"); return 2; }
    p.q = 1;
    std::vector<hit> hits;
    std::vector<pbuf> bufs;
    std::vector<photon> bunches;
    unsigned long long produced = 0, done = 0;
    double secs = 0;
    while (done < total) {
      unsigned int num = (unsigned int)std::min<unsigned long long>(pmax, total - done);
      // one bunch per launch, as addh() does for a single source (gpu/f2k.cxx:377-385)
      p.num = num;
      q.pz[0] = p;
      if (dump) bunches.push_back(p);
      auto t0 = std::chrono::steady_clock::now();
      produced += launch(num, hits, dump ? &bufs : nullptr);
      if (!keep_hits) hits.clear();
      secs += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      done += num;
    }
    if (keep_hits) {
      FILE* f = xopen((outp + ".hits").c_str(), "wb");
      fwrite(hits.data(), sizeof(hit), hits.size(), f);
      fclose(f);
    }
    if (dump) {
      FILE* f = xopen((outp + ".pbuf").c_str(), "wb");
      fwrite(bufs.data(), sizeof(pbuf), bufs.size(), f);
      fclose(f);
      f = xopen((outp + ".bunch").c_str(), "wb");
      fwrite(bunches.data(), sizeof(photon), bunches.size(), f);
      fclose(f);
    }
    printf("{\"photons\": %llu, \"hits\": %llu, \"seconds\": %.6f, \"rs\": %llu}\n", done, produced, secs,
           (unsigned long long)z.rs[seed % d.rsize]);
    return 0;
  }
  fprintf(stderr, "bad arguments\n");
  return 2;
}
