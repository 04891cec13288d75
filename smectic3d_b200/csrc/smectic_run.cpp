// smectic_run: the reference's main() around the B200 time loop.
//
// Restates the driver part of periodicFFT/pf3d.cpp (and the cos variants):
//  - compile-time constants become command-line flags;
//  - the initial condition is one of the reference's ICs or a psi text file
//    (psiIC.dat layout: N^3 values, i, j, k with k fastest);
//  - the loop runs while L1 > limit, evaluating L1 every --l1-every steps
//    (pf3d.cpp:390-518);
//  - L1 values are appended to L1.dat and psi is written to psi.dat, in the
//    reference's text formats (one value per line, "\n " separators,
//    pf3d.cpp:510-546).
// The time loop itself is the C-ABI of libsmectic_b200.so.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/smectic_b200.h"

namespace {

struct Opts {
  int n = 64, nw = 16, l1_every = 100, save_every = 100, surface_every = 0, amp_nw = 0;
  double sub_sigma = 0.0, sub_z0 = 1e-4;
  bool alternate = false;
  long long max_steps = -1;
  double dt = 0.001, eps = -0.7, beta = 2.0, gamma = 1.0, alpha = 1.0, q0 = 1.0, eta = 1.0, rho = 1.0, w_mid = 0.0;
  double l1_limit = 1e-6;
  std::string boundary = "periodic", precision = "fp64", ic = "lamellae", out = ".", curvature = "difference";
  bool advection = false;
};

void usage() {
  std::puts(
      "usage: smectic_run [--n N] [--nw Nw] [--dt dt] [--eps e] [--beta b] [--gamma g] [--alpha a] [--q0 q]\n"
      "                   [--eta h] [--rho r] [--w-mid w] [--boundary periodic|neumann] [--advection]\n"
      "                   [--precision fp64|fp32|fp32_u64] [--ic lamellae|torus|hyperboloid|load:FILE]\n"
      "                   [--curvature difference|spectral]\n"
      "                   [--l1-limit x] [--l1-every k] [--save-every m] [--max-steps s] [--out DIR]\n"
      "                   [--sub-sigma s] [--sub-z0 z0] [--surface-every m] [--amp-nw Nw]\n"
      "  --surface-every m  every m-th L1 evaluation, end the block with the surface pass and append\n"
      "                     surfPsi.dat, velSurf.dat, curvH.dat, curvK.dat (Neumann: all columns, keeping\n"
      "                     the last value where no crossing is found; periodic: surfTrack, crossings only)\n"
      "  --amp-nw Nw        at the end, write the local-amplitude map psiAvg.dat (morphSurfAmp)\n"
      "  --alternate        saves alternate between psi.dat and psiB.dat and append the y = N/2\n"
      "                     slice of psi to psiMid.dat (cosNoAdvMorphCurv.cpp:980-1045)");
}

bool parse(int argc, char** argv, Opts& o) {
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto need = [&](const char* name) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", name);
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--help" || a == "-h") {
      usage();
      std::exit(0);
    } else if (a == "--n") o.n = std::atoi(need("--n"));
    else if (a == "--nw") o.nw = std::atoi(need("--nw"));
    else if (a == "--dt") o.dt = std::atof(need("--dt"));
    else if (a == "--eps") o.eps = std::atof(need("--eps"));
    else if (a == "--beta") o.beta = std::atof(need("--beta"));
    else if (a == "--gamma") o.gamma = std::atof(need("--gamma"));
    else if (a == "--alpha") o.alpha = std::atof(need("--alpha"));
    else if (a == "--q0") o.q0 = std::atof(need("--q0"));
    else if (a == "--eta") o.eta = std::atof(need("--eta"));
    else if (a == "--rho") o.rho = std::atof(need("--rho"));
    else if (a == "--w-mid") o.w_mid = std::atof(need("--w-mid"));
    else if (a == "--boundary") o.boundary = need("--boundary");
    else if (a == "--advection") o.advection = true;
    else if (a == "--precision") o.precision = need("--precision");
    else if (a == "--ic") o.ic = need("--ic");
    else if (a == "--l1-limit") o.l1_limit = std::atof(need("--l1-limit"));
    else if (a == "--l1-every") o.l1_every = std::atoi(need("--l1-every"));
    else if (a == "--save-every") o.save_every = std::atoi(need("--save-every"));
    else if (a == "--max-steps") o.max_steps = std::atoll(need("--max-steps"));
    else if (a == "--out") o.out = need("--out");
    else if (a == "--sub-sigma") o.sub_sigma = std::atof(need("--sub-sigma"));
    else if (a == "--sub-z0") o.sub_z0 = std::atof(need("--sub-z0"));
    else if (a == "--surface-every") o.surface_every = std::atoi(need("--surface-every"));
    else if (a == "--amp-nw") o.amp_nw = std::atoi(need("--amp-nw"));
    else if (a == "--alternate") o.alternate = true;
    else if (a == "--curvature") o.curvature = need("--curvature");
    else {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      usage();
      return false;
    }
  }
  return true;
}

// Initial conditions of the reference, scaled from the N at which the
// reference sets them (dz = dx = 2 pi / (q0 Nw)).
void make_ic(const Opts& o, double dx, std::vector<double>& psi) {
  const int n = o.n;
  psi.assign(size_t(n) * n * n, 0.0);
  auto at = [&](int i, int j, int k) -> double& { return psi[(size_t(i) * n + j) * n + k]; };
  if (o.ic == "lamellae") {
    // periodicFFT/pf3d.cpp:302-324 (24 < k < 232 at N = 256)
    const double amp = 1.2441, qi = 0.5;
    const double kmin = 24.0 * n / 256, kmax = 232.0 * n / 256;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k)
          if (k > kmin && k < kmax)
            at(i, j, k) = amp * std::cos(o.q0 * k * dx) +
                          amp * 0.1 * std::sin(o.q0 * k * dx) * (std::cos(qi * i * dx) + std::cos(qi * j * dx));
  } else if (o.ic == "torus" || o.ic == "hyperboloid") {
    // periodicFFT/pf3dMorph.cpp:331-376 (torus, centred) and
    // cosFFT/mesabi/cosNoAdvMorph.cpp:289-331 (on the k = 0 wall)
    const bool torus = o.ic == "torus";
    const double amp = 1.328, mid = n / 2;
    const double ae = (torus ? 245.0 : 312.0) * n / 512, be = (torus ? 180.0 : 376.0) * n / 512;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k) {
          if (torus ? !(k > 62.0 * n / 512 && k < 450.0 * n / 512) : !(k < be + 1)) continue;
          const double xs = i - mid, ys = j - mid, zs = torus ? k - mid : k;
          const double ds = std::sqrt(xs * xs + ys * ys);
          double v = 0.0;
          if (ds < mid) {
            if (std::sqrt(std::pow((ds - mid) / ae, 2) + std::pow(zs / be, 2)) <= 1)
              v = amp * std::cos(o.q0 * dx * std::sqrt(std::pow((be / ae) * (ds - mid), 2) + zs * zs));
          } else if (std::fabs(zs) < be) {
            v = amp * std::cos(o.q0 * zs * dx);
          }
          at(i, j, k) = v;
        }
  } else if (o.ic.rfind("load:", 0) == 0) {
    std::ifstream f(o.ic.substr(5));
    if (!f) {
      std::fprintf(stderr, "cannot open %s\n", o.ic.c_str() + 5);
      std::exit(1);
    }
    for (auto& v : psi)
      if (!(f >> v)) {
        std::fprintf(stderr, "%s holds fewer than N^3 values\n", o.ic.c_str() + 5);
        std::exit(1);
      }
  } else {
    std::fprintf(stderr, "unknown --ic %s\n", o.ic.c_str());
    std::exit(2);
  }
}

void write_psi(const std::string& path, const std::vector<double>& psi) {
  std::ofstream f(path);
  for (double v : psi) f << v << "\n ";
}

}  // namespace

int main(int argc, char** argv) {
  Opts o;
  if (!parse(argc, argv, o)) return 2;
  sh_params p;
  sh_default_params(&p);
  p.n = o.n;
  p.dx = 2.0 * M_PI / (o.q0 * o.nw);
  p.dt = o.dt;
  p.eps = o.eps;
  p.beta = o.beta;
  p.gamma = o.gamma;
  p.alpha = o.alpha;
  p.q0 = o.q0;
  p.eta = o.eta;
  p.rho = o.rho;
  p.w_mid = o.w_mid;
  p.boundary = o.boundary == "neumann" ? SH_NEUMANN : SH_PERIODIC;
  p.advection = o.advection ? 1 : 0;
  p.precision = o.precision == "fp32" ? SH_FP32 : (o.precision == "fp32_u64" ? SH_FP32_UPDATE64 : SH_FP64);
  p.curvature = o.curvature == "spectral" ? SH_CURV_SPECTRAL : SH_CURV_DIFFERENCE;
  p.l1_interval = o.l1_every;
  p.sub_sigma = o.sub_sigma;
  p.sub_z0 = o.sub_z0;
  sh_handle* h = nullptr;
  if (sh_create(&p, &h) != SH_OK) {
    std::fprintf(stderr, "sh_create: %s\n", sh_last_error(nullptr));
    return 1;
  }
  std::vector<double> psi;
  make_ic(o, p.dx, psi);
  write_psi(o.out + "/psiIC.dat", psi);
  if (sh_set_psi(h, psi.data(), SH_LAYOUT_DENSE) != SH_OK) {
    std::fprintf(stderr, "sh_set_psi: %s\n", sh_last_error(h));
    return 1;
  }
  std::ofstream(o.out + "/L1.dat").close();
  const size_t nc = size_t(o.n) * o.n;
  std::vector<int> zc(nc);
  std::vector<double> vn(nc), hh(nc), kk(nc), zs(nc, 0.0), vs(nc, 0.0), hs(nc, 0.0), ks(nc, 0.0);
  if (o.surface_every > 0)
    for (const char* f : {"/surfPsi.dat", "/velSurf.dat", "/curvH.dat", "/curvK.dat"}) std::ofstream(o.out + f).close();
  double l1 = 1.0;
  long long steps = 0;
  int count_save = 0, count_surf = 0;
  long long saves = 0;
  if (o.alternate) std::ofstream(o.out + "/psiMid.dat").close();
  while (l1 > o.l1_limit && (o.max_steps < 0 || steps < o.max_steps)) {
    const int k = o.max_steps < 0 ? o.l1_every : int(std::min<long long>(o.l1_every, o.max_steps - steps));
    const bool surf = o.surface_every > 0 && k == o.l1_every && ++count_surf == o.surface_every;
    if (sh_step(h, surf ? k - 1 : k) != SH_OK) {
      std::fprintf(stderr, "sh_step: %s\n", sh_last_error(h));
      return 1;
    }
    if (surf) {  // the last step of the block goes through the surface pass
      count_surf = 0;
      if (sh_surface_step(h, zc.data(), vn.data(), hh.data(), kk.data()) != SH_OK) {
        std::fprintf(stderr, "sh_surface_step: %s\n", sh_last_error(h));
        return 1;
      }
      std::ofstream fz(o.out + "/surfPsi.dat", std::ios_base::app), fv(o.out + "/velSurf.dat", std::ios_base::app),
          fh(o.out + "/curvH.dat", std::ios_base::app), fk(o.out + "/curvK.dat", std::ios_base::app);
      for (size_t c = 0; c < nc; ++c) {
        if (p.boundary == SH_NEUMANN) {
          // cosNoAdvMorphCurv.cpp:995-1013: every column; a column without a crossing keeps its value
          if (zc[c] >= 0) {
            zs[c] = zc[c];
            vs[c] = vn[c];
            hs[c] = hh[c];
            ks[c] = kk[c];
          }
          fz << zs[c] << "\n";
          fv << vs[c] << "\n ";
          fh << hs[c] << "\n ";
          fk << ks[c] << "\n ";
        } else if (zc[c] >= 0) {  // surfTrack.cpp:787-799: the columns with a crossing
          fz << zc[c] << "\n ";
          fv << vn[c] << "\n ";
          fh << hh[c] << "\n ";
          fk << kk[c] << "\n ";
        }
      }
    }
    steps += k;
    if (k < o.l1_every) break;  // partial last block: no L1 evaluation
    int cnt = 0;
    sh_l1(h, &l1, &cnt);
    std::ofstream(o.out + "/L1.dat", std::ios_base::app) << l1 << "\n";
    if (++count_save == o.save_every) {
      sh_get_psi(h, psi.data(), SH_LAYOUT_DENSE);
      if (o.alternate) {
        // psiMid.dat: the y = N/2 plane, i then k, "\n" separated; psi.dat and psiB.dat in turn
        std::ofstream mid(o.out + "/psiMid.dat", std::ios_base::app);
        for (int i = 0; i < o.n; ++i)
          for (int k = 0; k < o.n; ++k) mid << psi[(size_t(i) * o.n + o.n / 2) * o.n + k] << "\n";
        write_psi(o.out + (saves % 2 == 0 ? "/psi.dat" : "/psiB.dat"), psi);
        ++saves;
      } else {
        write_psi(o.out + "/psi.dat", psi);
      }
      count_save = 0;
    }
  }
  sh_get_psi(h, psi.data(), SH_LAYOUT_DENSE);
  write_psi(o.out + "/psi.dat", psi);
  if (o.amp_nw > 0) {
    std::vector<double> amp(psi.size());
    if (sh_local_amplitude(h, o.amp_nw, amp.data()) != SH_OK) {
      std::fprintf(stderr, "sh_local_amplitude: %s\n", sh_last_error(h));
      return 1;
    }
    write_psi(o.out + "/psiAvg.dat", amp);  // morphSurfAmp.cpp:1113-1122
  }
  std::printf("steps %lld  L1 %.6g\n", steps, l1);
  sh_destroy(h);
  return 0;
}
