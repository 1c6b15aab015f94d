// lce_main.cpp -- the reference driver f/main.f restated in C++ over the C ABI.
//
// Reads the same 20-line inputfile (f/paraminit.f:82-101), starts the lattice
// as f/confget.f does (init 0..4), runs the thermalisation and the sweep loop
// of f/main.f:20-83 on the GPU, and writes the reference's measurement files
// with their names and formats (f/measinit.f, f/meas1.f, f/meas2a.f,
// f/correlator.f, f/polyakov.f, f/scalarcorr.f).  At the end it saves the
// configuration (f/confsave.f format) and rewrites the inputfile the way
// f/finalize.f does.
//
//   lce_main [--input FILE] [--dir DIR] [--precision f32|f64] [--seed N]
//            [--corr-flag 1|2|3] [--therm N] [--max-gf-iters N]
//            [--gf-angle acos|atan2] [--device N] [--agauge-hits 1|3]
//            [--gauge-fix plain|warm|fourier|fourier-cg|it] [--it-step S]
//
// --agauge-hits 3 runs the 3-hit link update of f/agauge1.f (the reference
// picks agauge.f or agauge1.f at build time).  --gauge-fix: plain is
// f/landau_gauge.f (copy, overrelaxation from G = 1); warm starts every
// measurement after the first from the previous converged transform; fourier
// uses the Fourier-accelerated iteration (power-of-two extents) from that warm
// start, fourier-cg its conjugate-gradient form; it is f/landau_gauge.f with the reference's iterative form
// f/it_gauge_fixing.f in place of the overrelaxation, component corrected and
// ascending, step --it-step (default 0.3; the reference's alpha diverges).
// All stop at theta <= limit_or.
//
// Deviations: init = 0 is a Haar hot start on the device (the reference's
// randomconf is not Haar distributed, f/confget.f:115-149); the per-site
// random numbers are Philox (the reference uses gfortran random_number);
// saved configurations use the lower-case names oldconf reads.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "lceqcd_gpu.h"

namespace {

struct Input {
  int n_lattice[3], dimproc[3], nproc, init, rand, save, confstart;
  double beta, x, y, lambda, alpha, limit_or, limit_it;
  int inorm, nsweep_flag, ntime, nsweep, imeas, imode;
};

[[noreturn]] void die(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::fprintf(stderr, "lce_main: ");
  std::vfprintf(stderr, fmt, ap);
  std::fprintf(stderr, "\n");
  va_end(ap);
  std::exit(1);
}

void check(lce_ctx* ctx, int rc, const char* what) {
  if (rc < 0) die("%s: %s (%s)", what, lce_strerror(rc), lce_last_error(ctx));
}

// list-directed read of the leading values of each of the 20 lines
Input read_input(const std::string& path) {
  std::ifstream f(path);
  if (!f) die("cannot open inputfile %s", path.c_str());
  std::vector<std::string> lines;
  std::string s;
  while (std::getline(f, s)) lines.push_back(s);
  if (lines.size() < 20) die("break: data input (inputfile has %zu lines, needs 20)", lines.size());
  auto nums = [&](int i, int n) {
    std::string t = lines[i];
    for (char& ch : t)
      if (ch == ',') ch = ' ';
    std::istringstream is(t);
    std::vector<double> v;
    for (int k = 0; k < n; ++k) {
      std::string tok;
      if (!(is >> tok)) die("break: data input (line %d)", i + 1);
      for (char& ch : tok)
        if (ch == 'd' || ch == 'D') ch = 'e';
      char* end = nullptr;
      double d = std::strtod(tok.c_str(), &end);
      if (end == tok.c_str()) die("break: data input (line %d: '%s')", i + 1, tok.c_str());
      v.push_back(d);
    }
    return v;
  };
  Input in;
  auto a = nums(0, 3), b = nums(1, 3);
  for (int i = 0; i < 3; ++i) {
    in.n_lattice[i] = (int)a[i];
    in.dimproc[i] = (int)b[i];
  }
  in.nproc = (int)nums(2, 1)[0];
  in.init = (int)nums(3, 1)[0];
  in.rand = (int)nums(4, 1)[0];
  in.save = (int)nums(5, 1)[0];
  in.confstart = (int)nums(6, 1)[0];
  in.beta = nums(7, 1)[0];
  in.x = nums(8, 1)[0];
  in.y = nums(9, 1)[0];
  in.lambda = nums(10, 1)[0];
  in.alpha = nums(11, 1)[0];
  in.limit_or = nums(12, 1)[0];
  in.limit_it = nums(13, 1)[0];
  in.inorm = (int)nums(14, 1)[0];
  in.nsweep_flag = (int)nums(15, 1)[0];
  in.ntime = (int)nums(16, 1)[0];
  in.nsweep = (int)nums(17, 1)[0];
  in.imeas = (int)nums(18, 1)[0];
  in.imode = (int)nums(19, 1)[0];
  if (in.imeas <= 0) die("imeas must be positive");
  return in;
}

// Fortran Ew.d: 0.ddddE+xx, right-justified in w; the optional leading zero
// is dropped when the field is too narrow, as gfortran does
std::string fe(double v, int w, int d) {
  char m[64];
  std::string body;
  if (v == 0.0 || !std::isfinite(v)) {
    if (!std::isfinite(v)) body = std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity");
    else body = "0." + std::string(d, '0') + "E+00";
  } else {
    std::snprintf(m, sizeof m, "%.*e", d - 1, std::fabs(v));  // d significant digits: x.xxxe+yy
    std::string t(m);
    const size_t e = t.find('e');
    std::string digits = t.substr(0, 1) + t.substr(2, e - 2);
    const int ex = std::atoi(t.c_str() + e + 1) + 1;
    char eb[16];
    std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    body = "0." + digits + eb;
    if (v < 0) body = "-" + body;
  }
  if ((int)body.size() > w) {
    const size_t z = body.find("0.");
    if (z != std::string::npos && (z == 0 || (z == 1 && body[0] == '-'))) body.erase(z, 1);
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

std::string fi(long v, int w, int m) {  // Iw.m
  char b[64];
  std::snprintf(b, sizeof b, "%0*ld", m, v);
  std::string s(b);
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

std::string name(const char* prefix, const Input& in, int number) {
  char buf[256];
  lce_conf_filename(buf, sizeof buf, prefix, in.n_lattice[2], in.beta, in.x, in.y, number);
  return buf;
}

void append(const std::string& path, const std::string& text) {
  FILE* f = std::fopen(path.c_str(), "a");
  if (!f) die("cannot append to %s", path.c_str());
  std::fputs(text.c_str(), f);
  std::fclose(f);
}

// f/measinit.f:234-238 header
std::string header(const Input& in) {
  char b[256];
  std::snprintf(b, sizeof b, "# %02d %02d %02d \n# %7.4f %7.4f %7.4f \n# %05d\n", in.n_lattice[0], in.n_lattice[1],
                in.n_lattice[2], in.beta, in.x, in.y, in.nsweep);
  return b;
}

}  // namespace

int main(int argc, char** argv) {
  std::string input = "inputfile", dir = ".";
  int prec = LCE_PREC_F32, corr_flag = 1, therm = 100, device = 0, max_gf = 0, gf_angle = LCE_GF_ATAN2;
  int agauge_hits = 1;
  std::string gauge_fix = "plain";
  double it_step = 0.3;
  unsigned long long seed = 314159;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) die("missing value for %s", a.c_str());
      return argv[++i];
    };
    if (a == "--input") input = next();
    else if (a == "--dir") dir = next();
    else if (a == "--precision") prec = next() == "f64" ? LCE_PREC_F64 : LCE_PREC_F32;
    else if (a == "--seed") seed = std::strtoull(next().c_str(), nullptr, 10);
    else if (a == "--corr-flag") corr_flag = std::atoi(next().c_str());
    else if (a == "--therm") therm = std::atoi(next().c_str());
    else if (a == "--device") device = std::atoi(next().c_str());
    else if (a == "--max-gf-iters") max_gf = std::atoi(next().c_str());
    else if (a == "--gf-angle") gf_angle = next() == "acos" ? LCE_GF_ACOS : LCE_GF_ATAN2;
    else if (a == "--agauge-hits") agauge_hits = std::atoi(next().c_str());
    else if (a == "--gauge-fix") gauge_fix = next();
    else if (a == "--it-step") it_step = std::atof(next().c_str());
    else die("unknown option %s", a.c_str());
  }
  const Input in = read_input(input);
  std::printf("Adjoint Higgs Modell on a %d X %d X %d lattice (one GPU)\n", in.n_lattice[0], in.n_lattice[1],
              in.n_lattice[2]);
  std::printf(" beta %g x %g y %g lambda %g alpha %g limit_or %g nsweep %d imeas %d imode %d init %d\n", in.beta,
              in.x, in.y, in.lambda, in.alpha, in.limit_or, in.nsweep, in.imeas, in.imode, in.init);

  lce_params p;
  lce_default_params(&p);
  for (int i = 0; i < 3; ++i) p.L[i] = in.n_lattice[i];
  p.beta = in.beta;
  p.x = in.x;
  p.y = in.y;
  p.lambda = in.lambda;
  p.alpha = in.alpha;
  p.limit_or = in.limit_or;
  p.imode = in.imode;
  p.precision = prec;
  p.seed = seed;
  p.device = device;
  p.gf_angle = gf_angle;
  p.agauge_hits = agauge_hits;
  if (gauge_fix != "plain" && gauge_fix != "warm" && gauge_fix != "fourier" && gauge_fix != "fourier-cg" &&
      gauge_fix != "it")
    die("unknown --gauge-fix %s", gauge_fix.c_str());
  lce_ctx* ctx = lce_create(&p);
  if (!ctx) die("lce_create: %s", lce_last_error(nullptr));

  const int L1 = in.n_lattice[0], L2 = in.n_lattice[1], L3 = in.n_lattice[2];
  const long nh = (long)L1 * L2 * L3 / 2;
  const std::string d = dir + "/";
  const std::string f_action = d + name("action", in, in.confstart), f_joblog = d + name("joblog", in, in.confstart),
                    f_correl = d + name("correl", in, in.confstart), f_afield = d + name("afield", in, in.confstart),
                    f_checkp = d + name("checkp", in, in.confstart), f_polyak = d + name("polyak", in, in.confstart),
                    f_corra2 = d + name("corra2", in, in.confstart);
  for (const std::string* f : {&f_action, &f_joblog, &f_correl, &f_afield, &f_checkp, &f_polyak, &f_corra2})
    append(*f, header(in));

  // ---- f/confget.f:51-59
  const float twopi = 2.0f * (2.0f * std::acos(0.0f));
  std::mt19937_64 host_rng(seed);
  std::uniform_real_distribution<float> unif(0.0f, 1.0f);
  if (in.init == 0) {
    check(ctx, lce_init_hot(ctx, seed), "init 0 (hot start)");
  } else if (in.init == 1 || in.init == 4) {
    std::vector<float> u((size_t)24 * nh), a((size_t)6 * nh);
    if (in.init == 1) {  // onerandconf f/confget.f:166-264: one SU(2) matrix and one A everywhere
      float x1 = 2.0f * unif(host_rng) - 1.0f, s1 = std::sqrt(1.0f - x1 * x1);
      float s2 = 2.0f * unif(host_rng) - 1.0f, x2 = s1 * s2, s3 = std::sqrt(1.0f - s2 * s2), s4 = s1 * s3;
      float s5 = twopi * unif(host_rng), x4 = s4 * std::cos(s5), x3 = s4 * std::sin(s5);
      float a3 = 2.0f * unif(host_rng) - 1.0f, t1 = std::sqrt(1.0f - a3 * a3), t2 = twopi * unif(host_rng);
      for (long i = 0; i < 6 * nh; ++i) {
        u[i * 4 + 0] = x1;
        u[i * 4 + 1] = x2;
        u[i * 4 + 2] = x3;
        u[i * 4 + 3] = x4;
      }
      for (long i = 0; i < 2 * nh; ++i) {
        a[i * 3 + 0] = t1 * std::cos(t2);
        a[i * 3 + 1] = t1 * std::sin(s3);  // the reference's sin(s3) (f/confget.f:147 pattern)
        a[i * 3 + 2] = a3;
      }
    } else {  // testconf f/confget.f:528-575
      const long nxy = (long)L1 * L2 / 2;
      for (int mu = 0; mu < 3; ++mu)
        for (int eo = 0; eo < 2; ++eo)
          for (long s = 0; s < nh; ++s) {
            float* q = &u[(((size_t)(mu * 2 + eo)) * nh + s) * 4];
            const float z = (float)(s / nxy);
            q[0] = 0.0f;
            q[1] = (float)(mu + 1) * z;
            q[2] = 0.0f;
            q[3] = (float)(mu + 1) * z;
          }
      const float r3 = 1.0f / std::sqrt(3.0f);
      for (long i = 0; i < 6 * nh; ++i) a[i] = r3;
    }
    check(ctx, lce_upload(ctx, 0, LCE_FIELDS, u.data(), a.data(), nh), "upload");
  } else if (in.init == 2) {
    check(ctx, lce_init_unit(ctx, 1.0), "init 2 (unitconf)");
  } else if (in.init == 3) {
    const std::string fu = d + name("u_conf", in, in.confstart), fa = d + name("a_conf", in, in.confstart);
    check(ctx, lce_confget(ctx, 0, fu.c_str(), fa.c_str()), "init 3 (oldconf)");
  } else {
    die("init must be 0..4");
  }

  // ---- thermalisation f/main.f:20-25
  check(ctx, lce_sweeps(ctx, therm, 0), "thermalisation");

  // ---- f/main.f:28-83
  double acco = 0, acch = 0, accg = 0, da = 0;
  long iter_or = 0;
  int meas = 0;
  const int mstart = in.confstart / in.imeas;
  const int nmeas = in.nsweep / in.imeas;
  std::vector<double> ca(L3), cu(L3), c3(L3), sl(L3), co(L3);
  for (int isweep = 1; isweep <= in.nsweep; ++isweep) {
    lce_meas m;
    check(ctx, lce_sweep(ctx, 1, &m), "sweep");
    acco += m.acc_or;
    acch += m.acc_hb;
    accg += m.acc_gauge;
    // meas1 f/meas1.f:86-95
    append(f_action, fi(isweep + in.confstart, 5, 1) + " " + fe(m.plaq, 23, 16) + " " + fe(m.akin, 23, 16) + " " +
                         fe(m.a2, 23, 16) + " " + fe(m.a4, 23, 16) + " \n");
    if (isweep == in.nsweep) {
      append(f_joblog, std::string("Overrelaxation acceptance : ") + fe(acco / in.nsweep, 10, 5) + "\n" +
                           "heat-bath acceptance :  " + fe(acch / in.nsweep, 10, 5) + "\n" +
                           "Gauge  acceptance    :  " + fe(accg / in.nsweep, 10, 5) + "\n");
    }
    if (isweep % in.imeas != 0) continue;
    ++meas;
    if (corr_flag == 1 || corr_flag == 3) {
      double theta = 0;
      int iters = 0;
      int rc;
      const int start = meas > 1 ? LCE_GF_START_TRANSFORM : LCE_GF_START_IDENTITY;
      if (gauge_fix == "warm") {
        rc = lce_landau_gauge_from(ctx, 0, start, nullptr, &theta, &iters, max_gf);
      } else if (gauge_fix == "fourier") {
        int it_plain = 0;
        rc = lce_landau_gauge_fourier(ctx, 0, start, 0.0, 0.0, &theta, &iters, &it_plain, max_gf);
        iters += it_plain;
      } else if (gauge_fix == "fourier-cg") {
        int it_plain = 0;
        rc = lce_landau_gauge_fourier_cg(ctx, 0, start, 0.0, &theta, &iters, &it_plain, max_gf);
        iters += it_plain;
      } else if (gauge_fix == "it") {
        rc = lce_it_landau_gauge(ctx, 0, it_step, LCE_ITGF_FIX_COMPONENT | LCE_ITGF_ASCEND, &theta, &iters, max_gf);
      } else {
        rc = lce_landau_gauge(ctx, 0, &theta, &iters, max_gf);
      }
      if (rc == LCE_ERR_GF_NOT_CONVERGED)
        std::fprintf(stderr, "lce_main: gauge fixing stopped at the cap (theta %g after %d iterations)\n", theta, iters);
      else
        check(ctx, rc, "landau_gauge");
      da += theta;
      iter_or += iters;
      double af[3];
      check(ctx, lce_correlator(ctx, 0, ca.data(), cu.data(), c3.data(), af), "correlator");
      // f/correlator.f:168-181
      std::string t = fi(mstart + meas, 3, 3) + "\n", t3 = t;
      for (int z = 0; z < L3; ++z) {
        t += fe(ca[z], 23, 16) + " " + fe(cu[z], 23, 16) + " \n";
        t3 += fe(c3[z], 23, 16) + "\n";
      }
      append(f_correl, t);
      append(f_checkp, t3);
      // f/meas2a.f:77-99
      if (meas == nmeas) {
        const long itg = nmeas > 0 ? iter_or / nmeas : 0;
        append(f_joblog, std::string("number of iteration for or. gauge fixing : ") + fi(itg, 20, 1) + "\n" +
                             "precision of the condition |d_mu A_mu|^2=0 : " + fe(da / nmeas, 20, 10) + "\n");
      }
      append(f_afield, fi(meas + mstart, 5, 5) + " " + fe(af[0], 23, 16) + " " + fe(af[1], 23, 16) + " " +
                           fe(af[2], 23, 16) + " \n");
    }
    if (corr_flag == 2 || corr_flag == 3) {
      double mean2 = 0, mean = 0;
      check(ctx, lce_polyakov(ctx, 0, sl.data(), co.data(), &mean2), "polyakov");
      std::string t = fi(mstart + meas, 5, 5) + "\n" + fe(mean2, 23, 16) + "\n";
      for (int z = 0; z < L3; ++z) t += fe(co[z], 23, 16) + "\n";
      append(f_polyak, t);
      if (corr_flag == 2) {
        check(ctx, lce_scalarcorr(ctx, 0, sl.data(), co.data(), &mean), "scalarcorr");
        std::string s2 = fi(mstart + meas, 5, 5) + "\n" + fe(mean, 23, 16) + "\n";
        for (int z = 0; z < L3; ++z) s2 += fe(co[z], 23, 16) + "\n";
        append(f_corra2, s2);
      }
    }
  }

  // ---- finalize f/finalize.f:39-161
  const int last = in.confstart + in.nsweep;
  const std::string fu = d + name("u_conf", in, last), fa = d + name("a_conf", in, last);
  check(ctx, lce_confsave(ctx, 0, fu.c_str(), fa.c_str()), "confsave");
  {
    char b[256];
    std::snprintf(b, sizeof b, "%slastconfig_s%02d_be%05ld_x%05ld_y%05ld", d.c_str(), L3, std::lround(1000 * in.beta),
                  std::lround(10000 * in.x), std::lround(10000 * in.y));
    FILE* f = std::fopen(b, "w");
    if (f) {
      std::fprintf(f, "%06d\n", last);
      std::fclose(f);
    }
  }
  {
    Input o = in;
    if (o.save == 1) {
      o.init = 3;
      o.rand = 1;
    }
    FILE* f = std::fopen(input.c_str(), "w");
    if (!f) die("break: data input (cannot rewrite %s)", input.c_str());
    std::fprintf(f, "%02d %02d %02d    !nx/ny/nz global lattice size\n", o.n_lattice[0], o.n_lattice[1], o.n_lattice[2]);
    std::fprintf(f, "%02d %02d %02d    !dimproc     numbers of processes in every dimension mu = 1-3\n",
                 o.dimproc[0], o.dimproc[1], o.dimproc[2]);
    std::fprintf(f, "%03d         !nproc       total numbers of processes\n", o.nproc);
    std::fprintf(f, "%1d           !init        init for gaugefields 0=rand,1=onerand,2=unit,3=old\n", o.init);
    std::fprintf(f, "%1d           !rand        old(=1) or new(=0) random numbers\n", o.rand);
    std::fprintf(f, "%1d           !save        save on disc yes or no (1,0)\n", o.save);
    std::fprintf(f, "%06d      !confstart   starting configuration\n", last);
    std::fprintf(f, "%6.3f      !beta\n", o.beta);
    std::fprintf(f, "%6.4f      !x\n", o.x);
    std::fprintf(f, "%6.4f      !y\n", o.y);
    std::fprintf(f, "%6.4f      !lambda overrelaxation parameter\n", o.lambda);
    std::fprintf(f, "%8.6f    !gauge transformation parameter\n", o.alpha);
    std::fprintf(f, "%s   !limit_or precision of the condition d_mu A_mu=0\n", fe(o.limit_or, 9, 3).c_str());
    std::fprintf(f, "%s   !limit_it precision of the condition d_mu A_mu=0\n", fe(o.limit_it, 9, 3).c_str());
    std::fprintf(f, "%03d         !inorm   number of iteration  followed by norm. \n", o.inorm);
    std::fprintf(f, "%1d           !nsweep_flag  (0=number of sweeps 1=max time in min) \n", o.nsweep_flag);
    std::fprintf(f, "%03d         !ntime       maximal time for the program in minuntes \n", o.ntime);
    std::fprintf(f, "%05d       !nsweeps       number of sweeps \n", o.nsweep);
    std::fprintf(f, "%05d       !imeas  number of sweeps followed by measurement\n", o.imeas);
    std::fprintf(f, "%03d         !imode  mode for the heatbath algorithm\n", o.imode);
    std::fclose(f);
  }
  lce_destroy(ctx);
  std::printf("done: %d sweeps, %d measurements\n", in.nsweep, meas);
  return 0;
}
