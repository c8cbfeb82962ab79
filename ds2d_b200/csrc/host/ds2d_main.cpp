// ds2d_elsrtm: C++ host driver of the B200 DS2D path, the single-process replacement of the
// reference's GPU2DDS (main.cpp:1326-1504 set-up, :788-1217 lsrtm_all_iteration).
//
//   ds2d_elsrtm parameters [max_shots=N] [device=D] [strips=f32|f16|bf16] [adjoint_born=0|1]
//
// Reads the reference's 9-line parameters file (main.cpp:1349-1359), indexes the vz / vx SU
// files, reads every shot gather ONCE (the reference re-reads them each iteration), and runs
// maxiter iterations of reference-mode ELSRTM with all shots batched on one GPU, followed by
// the Adam-like image update of main.cpp:1092-1131.  Output files keep the reference's names
// (main.cpp:1134-1186): sum_bgrad2_{pp,ps}_<iter>_<allnx>_<allnz>.dat,
// all_grad_{pp,ps}_..., sum_image_{pp,ps}_... and misfit.txt in the image directory.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../../include/ds2d.h"
#include "su.hpp"

using namespace ds2d_host;

namespace {

struct Params {
  float dx = 0, dz = 0;
  int pml = 0, allnx = 0, allnz = 0, minshot = 0, maxshot = 0;
  std::string fvp, fvs, fvz, fvx, imagedir;
  float f0 = 0;
  int maxiter = 0, sy = 0, gy = 0;
  int light = 0, rbc = 0, cpu_mem = 0, iointerval = 0;
};

bool read_params(const std::string &path, Params &p, std::string &err) {
  std::ifstream in(path);
  if (!in) {
    err = "cannot open " + path;
    return false;
  }
  // main.cpp:1349-1359
  if (!(in >> p.dx >> p.dz >> p.pml >> p.allnx >> p.allnz >> p.minshot >> p.maxshot >> p.fvp >>
        p.fvs >> p.fvz >> p.fvx >> p.imagedir >> p.f0 >> p.maxiter >> p.sy >> p.gy >> p.light >>
        p.rbc >> p.cpu_mem >> p.iointerval)) {
    err = path + ": expected the 9-line parameters format";
    return false;
  }
  return true;
}

// Relative paths in the parameters file are relative to the directory the driver runs in, as
// for the reference.
bool read_model(const std::string &path, int allnx, int allnz, std::vector<float> &v,
                std::string &err) {
  v.assign((size_t)allnx * allnz, 0.f);
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp) {
    err = "cannot open " + path;
    return false;
  }
  const size_t got = std::fread(v.data(), 4, v.size(), fp);
  std::fclose(fp);
  if (got != v.size()) {
    err = path + ": expected " + std::to_string(v.size()) + " floats";
    return false;
  }
  return true;
}

void ricker1(int nt, float f, float dt, float *s) {  // main.cpp:461-473
  float pi = 3.14159265358979f;
  float t0 = 1 / f;
  int kt = (int)(t0 / dt);
  for (int i = 0; i < nt; i++) {
    float tt = i * dt - kt * dt;
    float sp = pi * f * tt;
    s[i] = (float)(1.0 * std::exp((double)(-sp * sp)) * (1. - 2. * sp * sp));
  }
}

bool write_dat(const std::string &path, const std::vector<float> &v) {
  FILE *fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  const bool ok = std::fwrite(v.data(), 4, v.size(), fp) == v.size();
  std::fclose(fp);
  return ok;
}

int die(const std::string &msg) {
  std::fprintf(stderr, "ds2d_elsrtm: %s\n", msg.c_str());
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) return die("usage: ds2d_elsrtm parameters [max_shots=N] [device=D] [strips=f32|f16|bf16] [adjoint_born=0|1]");
  int max_shots = 64, device = 0, strips = DS2D_STRIPS_F32, adjoint_born = 0;
  for (int i = 2; i < argc; i++) {
    std::string a(argv[i]);
    const size_t eq = a.find('=');
    if (eq == std::string::npos) return die("bad option " + a);
    const std::string k = a.substr(0, eq), v = a.substr(eq + 1);
    if (k == "max_shots") max_shots = std::atoi(v.c_str());
    else if (k == "device") device = std::atoi(v.c_str());
    else if (k == "adjoint_born") adjoint_born = std::atoi(v.c_str());
    else if (k == "strips") strips = v == "f16" ? DS2D_STRIPS_F16 : (v == "bf16" ? DS2D_STRIPS_BF16 : DS2D_STRIPS_F32);
    else return die("unknown option " + k);
  }
  Params P;
  std::string err;
  if (!read_params(argv[1], P, err)) return die(err);
  int nt = 0;
  float dt = 0;
  std::vector<ShotIndex> table, table_x;
  if (!su_index(P.fvz, &nt, &dt, table, err)) return die(err);
  if (!su_index(P.fvx, &nt, &dt, table_x, err)) return die(err);
  if (table_x.size() != table.size()) return die("vz and vx files hold different shots");
  // main.cpp:1414-1442: leftmost aperture, window width of the first shot, nz = allnz.
  int all_left = table[0].xmin;
  for (const ShotIndex &s : table) all_left = std::min(all_left, s.xmin);
  const int nx = (int)(table[0].xmax / P.dx + 0.5) - (int)(table[0].xmin / P.dx + 0.5) + 1;
  std::vector<float> vp, vs;
  if (!read_model(P.fvp, P.allnx, P.allnz, vp, err) || !read_model(P.fvs, P.allnx, P.allnz, vs, err))
    return die(err);
  std::vector<float> wav(nt);
  ricker1(nt, P.f0, dt, wav.data());

  // All selected shots are read once and kept in host memory.
  std::vector<ds2d_shot> shots;
  std::vector<std::vector<int>> igx;
  std::vector<float> obs_z, obs_x;
  int max_ntr = 1;
  for (const ShotIndex &s : table) {
    if (s.sno < P.minshot || s.sno > P.maxshot) continue;
    std::vector<float> dz((size_t)s.ntr * nt), dxv((size_t)s.ntr * nt);
    std::vector<int> gx(s.ntr), gx2(s.ntr);
    if (!su_read_gather(P.fvz, s.pos, s.ntr, nt, dz.data(), gx.data(), err) ||
        !su_read_gather(P.fvx, s.pos, s.ntr, nt, dxv.data(), gx2.data(), err))
      return die(err);
    const int ngx_left = s.xmin;
    const int delta_left = (int)((ngx_left - all_left) / P.dx);  // main.cpp:988
    std::vector<int> cells(s.ntr);
    for (int t = 0; t < s.ntr; t++)  // FD2DGPU.cu:3097
      cells[t] = P.pml + (int)((float)(gx[t] - ngx_left) / P.dx);
    igx.push_back(cells);
    ds2d_shot d{};
    d.win_left = delta_left;  // + record_left_in_v = 0 (main.cpp:1496)
    d.isx = P.pml + (int)((s.sx - ngx_left) / P.dx);
    d.isz = P.pml + P.sy;
    d.igz = P.pml + P.gy;
    d.ntr = s.ntr;
    d.nx = 0;
    shots.push_back(d);
    obs_z.insert(obs_z.end(), dz.begin(), dz.end());
    obs_x.insert(obs_x.end(), dxv.begin(), dxv.end());
    max_ntr = std::max(max_ntr, s.ntr);
  }
  for (size_t i = 0; i < shots.size(); i++) shots[i].igx = igx[i].data();
  if (shots.empty()) return die("no shot in [minshot, maxshot]");
  std::printf("ds2d_elsrtm: %zu shots, nt = %d, dt = %g s, window nx = %d, nz = %d, pml = %d\n",
              shots.size(), nt, dt, nx, P.allnz, P.pml);

  ds2d_grid grid{P.allnx, P.allnz, nx, P.pml, nt, P.dx, P.dz, dt};
  ds2d_opts opts{P.rbc ? DS2D_BOUNDARY_RANDOM : DS2D_BOUNDARY_PML, strips,
                 std::min<int>(max_shots, (int)shots.size()), max_ntr, 1234ULL, device};
  ds2d_ctx *ctx = nullptr;
  if (ds2d_create(&grid, &opts, &ctx)) return die(ds2d_last_error(nullptr));
  auto check = [&](int rc) {
    if (rc) {
      std::fprintf(stderr, "ds2d_elsrtm: %s\n", ds2d_last_error(ctx));
      ds2d_destroy(ctx);
      std::exit(1);
    }
  };
  check(ds2d_set_models(ctx, vp.data(), vs.data(), nullptr));
  check(ds2d_set_wavelet(ctx, wav.data()));
  check(ds2d_set_option(ctx, "adjoint_born", adjoint_born));
  mkdir(P.imagedir.c_str(), 0755);

  const size_t N = (size_t)P.allnx * P.allnz;
  std::vector<float> image_pp(N, 0.f), image_ps(N, 0.f);
  std::vector<float> g[7];
  for (auto &x : g) x.assign(N, 0.f);
  std::vector<float> s_k0_p(N, 0.f), s_k0_s(N, 0.f), r_k0_p(N, 0.f), r_k0_s(N, 0.f);
  std::vector<float> sum_pp(N), sum_ps(N);
  // main.cpp:869-876
  const float beta1 = 0.8f, beta2 = 0.999f, alpha = 3e-5f, epsilon = 5e8f, gama = 0.99f;
  std::vector<float> rms(P.maxiter);
  for (int iter = 0; iter < P.maxiter; iter++) {
    check(ds2d_set_image(ctx, image_pp.data(), image_ps.data()));
    double misfit = 0;
    check(ds2d_elsrtm(ctx, shots.data(), (int)shots.size(), obs_z.data(), obs_x.data(), iter,
                      &misfit, nullptr, nullptr, nullptr, nullptr));
    float *img[7];
    for (int a = 0; a < 7; a++) img[a] = g[a].data();
    check(ds2d_read_images(ctx, img, 1));
    if (iter == 0) misfit = 0.0f;  // main.cpp:1065-1067
    rms[iter] = 1.0f - std::fabs((1.0f / table.size()) * misfit);
    std::printf("iter = %d  misfit = %g  rmsmisfit = %g\n", iter, misfit, rms[iter]);
    // Adam-like update, main.cpp:1092-1131 (float arrays, double powers as in the reference).
    const float alpha_k = iter == 0 ? alpha : (alpha / 2) * std::pow(gama, iter);
    const int k = iter + 1;
    for (size_t i = 0; i < N; i++) {
      sum_pp[i] = g[0][i] + g[3][i] + g[5][i];
      sum_ps[i] = g[1][i] + g[4][i] + g[6][i];
      const float s_k_p = beta1 * s_k0_p[i] + (1 - beta1) * sum_pp[i];
      const float s_k_s = beta1 * s_k0_s[i] + (1 - beta1) * sum_ps[i];
      const float r_k_p = beta2 * r_k0_p[i] + (1 - beta2) * (sum_pp[i] * sum_pp[i]);
      const float r_k_s = beta2 * r_k0_s[i] + (1 - beta2) * (sum_ps[i] * sum_ps[i]);
      const float s_kmod_p = s_k_p / (1 - std::pow(beta1, k));
      const float s_kmod_s = s_k_s / (1 - std::pow(beta1, k));
      const float r_kmod_p = r_k_p / (1 - std::pow(beta2, k));
      const float r_kmod_s = r_k_s / (1 - std::pow(beta2, k));
      image_pp[i] -= alpha_k * (s_kmod_p / (std::sqrt(r_kmod_p) + epsilon));
      image_ps[i] -= alpha_k * (s_kmod_s / (std::sqrt(r_kmod_s) + epsilon));
      s_k0_p[i] = s_k_p;
      s_k0_s[i] = s_k_s;
      r_k0_p[i] = r_k_p;
      r_k0_s[i] = r_k_s;
    }
    char suffix[128];
    std::snprintf(suffix, sizeof suffix, "_%d_%d_%d.dat", iter, P.allnx, P.allnz);
    const std::string dir = P.imagedir + "/";
    bool ok = write_dat(dir + "sum_bgrad2_pp" + suffix, g[5]) &&
              write_dat(dir + "sum_bgrad2_ps" + suffix, g[6]) &&
              write_dat(dir + "all_grad_pp" + suffix, sum_pp) &&
              write_dat(dir + "all_grad_ps" + suffix, sum_ps) &&
              write_dat(dir + "sum_image_pp" + suffix, image_pp) &&
              write_dat(dir + "sum_image_ps" + suffix, image_ps);
    if (!ok) {
      ds2d_destroy(ctx);
      return die("cannot write images into " + P.imagedir);
    }
  }
  FILE *fp = std::fopen((P.imagedir + "/misfit.txt").c_str(), "w");  // main.cpp:1178-1185
  if (fp) {
    for (int i = 0; i < P.maxiter; i++)
      std::fprintf(fp, "i = %d,misfit = %e,rms_misfit = %f\n", i, rms[i], rms[i]);
    std::fclose(fp);
  }
  ds2d_destroy(ctx);
  return 0;
}
