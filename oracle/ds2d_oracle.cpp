// CPU oracle for the DS2D time-stepping path -- TEST INFRASTRUCTURE ONLY (see ds2d_oracle.h).
//
// Each "kernel" below restates one __global__ function of the reference, with the same bounds,
// the same stencil index pattern and the same operand order; citations are file:line into the
// reference project.  Loops are hazard-free exactly like the reference kernels: a kernel only
// writes arrays that it reads at its own cell.
#include "ds2d_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// 8th-order staggered coefficients, FD2DGPU.cuh:16 (stored as float constants by the reference).
const float kCoef[5] = {0.f, 1225.0f / 1024.0f, -245.0f / 3072.0f, 49.0f / 5120.0f,
                        -5.0f / 7168.0f};

template <class R>
struct Geo {
  int nx, nz;  // padded window (nxpml, nzpml)
  int pml, nop;
  R dx, dz, dt;
  size_t n;
  int wnx, wnz;  // interior window (nx, nz of the reference)
  R c[5];
  explicit Geo(const orc_grid *g)
      : nx(g->nxpml), nz(g->nzpml), pml(g->pml), nop(g->nop), dx(g->dx), dz(g->dz), dt(g->dt) {
    n = (size_t)nx * nz;
    wnx = nx - 2 * pml;
    wnz = nz - 2 * pml;
    for (int i = 0; i < 5; i++) c[i] = (R)kCoef[i];
  }
  inline size_t I(int ix, int iz) const { return (size_t)ix * nz + iz; }
};

template <class R>
using Vec = std::vector<R>;

// One wavefield set: the five sums and the ten split memory variables (FD2DGPU.cuh:124-422).
template <class R>
struct Wave {
  Vec<R> vx, vz, txx, tzz, txz, vx_x, vx_z, vz_x, vz_z, txx_x, txx_z, tzz_x, tzz_z, txz_x, txz_z;
  explicit Wave(size_t n) {
    for (Vec<R> *v : {&vx, &vz, &txx, &tzz, &txz, &vx_x, &vx_z, &vz_x, &vz_z, &txx_x, &txx_z,
                      &tzz_x, &tzz_z, &txz_x, &txz_z})
      v->assign(n, (R)0);
  }
};

template <class R>
struct Strain {
  Vec<R> gx_vx, gz_vz, gz_vx, gx_vz;  // vx_gx, vz_gz, vx_gz, vz_gx of the reference
  explicit Strain(size_t n) {
    for (Vec<R> *v : {&gx_vx, &gz_vz, &gz_vx, &gx_vz}) v->assign(n, (R)0);
  }
};

template <class R>
struct Model {
  Vec<R> vp, vs, rho, lam, mu, dampx, dampz, dmp, dms;
};

template <class R>
Model<R> load_model(const Geo<R> &g, const float *const m[7], const float *dmp, const float *dms) {
  Model<R> M;
  Vec<R> *dst[7] = {&M.vp, &M.vs, &M.rho, &M.lam, &M.mu, &M.dampx, &M.dampz};
  for (int a = 0; a < 7; a++) dst[a]->assign(m[a], m[a] + g.n);
  if (dmp) M.dmp.assign(dmp, dmp + g.n); else M.dmp.assign(g.n, (R)0);
  if (dms) M.dms.assign(dms, dms + g.n); else M.dms.assign(g.n, (R)0);
  return M;
}

#define FOR_CELLS(lo_x, hi_x, lo_z, hi_z)           \
  _Pragma("omp parallel for schedule(static)")      \
  for (int ix = (lo_x); ix < (hi_x); ix++)          \
    for (int iz = (lo_z); iz < (hi_z); iz++)

// born.cu:215-247 update_vx; FD2DGPU.cu:903-945 GPUcalculate_elastic_vx (same math, bounds lo..n-lo).
template <class R>
void k_update_vx(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir, int lo) {
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_txx = 0, tmp_txz = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_txx += g.c[i] * (w.txx[g.I(ix + i, iz)] - w.txx[g.I(ix - i + 1, iz)]);
      tmp_txz += g.c[i] * (w.txz[g.I(ix, iz + i - 1)] - w.txz[g.I(ix, iz - i)]);
    }
    w.vx_x[k] = (damp1 * w.vx_x[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dx) * tmp_txx) / damp2;
    w.vx_z[k] = (damp3 * w.vx_z[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dz) * tmp_txz) / damp4;
    w.vx[k] = w.vx_x[k] + w.vx_z[k];
  }
}

// born.cu:249-279 update_vz; FD2DGPU.cu:948-990 GPUcalculate_elastic_vz.
template <class R>
void k_update_vz(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir, int lo) {
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_tzz = 0, tmp_txz = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_tzz += g.c[i] * (w.tzz[g.I(ix, iz + i)] - w.tzz[g.I(ix, iz - i + 1)]);
      tmp_txz += g.c[i] * (w.txz[g.I(ix + i - 1, iz)] - w.txz[g.I(ix - i, iz)]);
    }
    w.vz_x[k] = (damp1 * w.vz_x[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dx) * tmp_txz) / damp2;
    w.vz_z[k] = (damp3 * w.vz_z[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dz) * tmp_tzz) / damp4;
    w.vz[k] = w.vz_x[k] + w.vz_z[k];
  }
}

// born.cu:282-315 update_txx_tzz; FD2DGPU.cu:993-1037 _txx_tzz_grad (strains when st != NULL).
template <class R>
void k_update_txx_tzz(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir, int lo,
                      Strain<R> *st) {
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_vx = 0, tmp_vz = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_vx += g.c[i] * (w.vx[g.I(ix + i - 1, iz)] - w.vx[g.I(ix - i, iz)]);
      tmp_vz += g.c[i] * (w.vz[g.I(ix, iz + i - 1)] - w.vz[g.I(ix, iz - i)]);
    }
    R l2m = M.lam[k] + 2 * M.mu[k];
    w.txx_x[k] = (damp1 * w.txx_x[k] + dir * l2m * (g.dt / g.dx) * tmp_vx) / damp2;
    w.txx_z[k] = (damp3 * w.txx_z[k] + dir * M.lam[k] * (g.dt / g.dz) * tmp_vz) / damp4;
    w.tzz_x[k] = (damp1 * w.tzz_x[k] + dir * M.lam[k] * (g.dt / g.dx) * tmp_vx) / damp2;
    w.tzz_z[k] = (damp3 * w.tzz_z[k] + dir * l2m * (g.dt / g.dz) * tmp_vz) / damp4;
    w.txx[k] = w.txx_x[k] + w.txx_z[k];
    w.tzz[k] = w.tzz_x[k] + w.tzz_z[k];
    if (st) {
      st->gx_vx[k] = tmp_vx / g.dx;
      st->gz_vz[k] = tmp_vz / g.dz;
    }
  }
}

// born.cu:318-349 update_txz; FD2DGPU.cu:1040-1081 _txz_grad (strains when st != NULL).
template <class R>
void k_update_txz(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir, int lo,
                  Strain<R> *st) {
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_vx = 0, tmp_vz = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_vx += g.c[i] * (w.vx[g.I(ix, iz + i)] - w.vx[g.I(ix, iz - i + 1)]);
      tmp_vz += g.c[i] * (w.vz[g.I(ix + i, iz)] - w.vz[g.I(ix - i + 1, iz)]);
    }
    w.txz_x[k] = (damp1 * w.txz_x[k] + dir * (g.dt / g.dx) * M.mu[k] * tmp_vz) / damp2;
    w.txz_z[k] = (damp3 * w.txz_z[k] + dir * (g.dt / g.dz) * M.mu[k] * tmp_vx) / damp4;
    w.txz[k] = w.txz_x[k] + w.txz_z[k];
    if (st) {
      st->gz_vx[k] = tmp_vx / g.dz;
      st->gx_vz[k] = tmp_vz / g.dx;
    }
  }
}

// FD2DGPU.cu:725-761 GPUcalculate_elastic_txx_tzz: adjoint "strain" update without moduli,
// txx = txx_x only, tzz = tzz_z only.  Bounds [nop, n-nop).
template <class R>
void k_adj_txx_tzz(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir) {
  int lo = g.nop;
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_vx = 0, tmp_vz = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_vx += g.c[i] * (w.vx[g.I(ix + i - 1, iz)] - w.vx[g.I(ix - i, iz)]);
      tmp_vz += g.c[i] * (w.vz[g.I(ix, iz + i - 1)] - w.vz[g.I(ix, iz - i)]);
    }
    w.txx_x[k] = (damp1 * w.txx_x[k] + dir * (g.dt / g.dx) * tmp_vx) / damp2;
    w.tzz_z[k] = (damp3 * w.tzz_z[k] + dir * (g.dt / g.dz) * tmp_vz) / damp4;
    w.txx[k] = w.txx_x[k];
    w.tzz[k] = w.tzz_z[k];
  }
}

// FD2DGPU.cu:860-895 GPUcalculate_elastic_txz: adjoint shear update without mu.
template <class R>
void k_adj_txz(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir) {
  int lo = g.nop;
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_vx = 0, tmp_vz = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_vx += g.c[i] * (w.vx[g.I(ix, iz + i)] - w.vx[g.I(ix, iz - i + 1)]);
      tmp_vz += g.c[i] * (w.vz[g.I(ix + i, iz)] - w.vz[g.I(ix - i + 1, iz)]);
    }
    w.txz_x[k] = (damp1 * w.txz_x[k] + dir * (g.dt / g.dx) * tmp_vz) / damp2;
    w.txz_z[k] = (damp3 * w.txz_z[k] + dir * (g.dt / g.dz) * tmp_vx) / damp4;
    w.txz[k] = w.txz_x[k] + w.txz_z[k];
  }
}

// FD2DGPU.cu:591-635 GPUcalculate_elastic_vx_back: moduli inside the divergence.
template <class R>
void k_adj_vx(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir) {
  int lo = g.nop;
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_txx = 0, tmp_txz = 0, tmp_tzz = 0;
    for (int i = 1; i <= 4; i++) {
      size_t p = g.I(ix + i, iz), q = g.I(ix - i + 1, iz);
      size_t pz = g.I(ix, iz + i - 1), qz = g.I(ix, iz - i);
      tmp_txx += g.c[i] * ((M.lam[p] + 2 * M.mu[p]) * w.txx[p] - (M.lam[q] + 2 * M.mu[q]) * w.txx[q]);
      tmp_txz += g.c[i] * (M.mu[pz] * w.txz[pz] - M.mu[qz] * w.txz[qz]);
      tmp_tzz += g.c[i] * ((M.lam[p]) * w.tzz[p] - (M.lam[q]) * w.tzz[q]);
    }
    w.vx_x[k] = (damp1 * w.vx_x[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dx) * tmp_txx +
                 dir * (1.0 / M.rho[k]) * (g.dt / g.dx) * tmp_tzz) / damp2;
    w.vx_z[k] = (damp3 * w.vx_z[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dz) * tmp_txz) / damp4;
    w.vx[k] = w.vx_x[k] + w.vx_z[k];
  }
}

// FD2DGPU.cu:638-682 GPUcalculate_elastic_vz_back.
template <class R>
void k_adj_vz(const Geo<R> &g, Wave<R> &w, const Model<R> &M, int dir) {
  int lo = g.nop;
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R damp1 = 1 - g.dt * M.dampx[k] / 2, damp2 = 1 + g.dt * M.dampx[k] / 2;
    R damp3 = 1 - g.dt * M.dampz[k] / 2, damp4 = 1 + g.dt * M.dampz[k] / 2;
    R tmp_tzz = 0, tmp_txz = 0, tmp_txx = 0;
    for (int i = 1; i <= 4; i++) {
      size_t p = g.I(ix, iz + i), q = g.I(ix, iz - i + 1);
      size_t px = g.I(ix + i - 1, iz), qx = g.I(ix - i, iz);
      tmp_tzz += g.c[i] * ((M.lam[p] + 2 * M.mu[p]) * w.tzz[p] - (M.lam[q] + 2 * M.mu[q]) * w.tzz[q]);
      tmp_txz += g.c[i] * (M.mu[px] * w.txz[px] - M.mu[qx] * w.txz[qx]);
      tmp_txx += g.c[i] * ((M.lam[p]) * w.txx[p] - (M.lam[q]) * w.txx[q]);
    }
    w.vz_x[k] = (damp1 * w.vz_x[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dx) * tmp_txz) / damp2;
    w.vz_z[k] = (damp3 * w.vz_z[k] + dir * (1.0 / M.rho[k]) * (g.dt / g.dz) * tmp_tzz +
                 dir * (1.0 / M.rho[k]) * (g.dt / g.dz) * tmp_txx) / damp4;
    w.vz[k] = w.vz_x[k] + w.vz_z[k];
  }
}

// born.cu:351-405 add_born_source: virtual source from the velocities of `src` into the stresses
// of `dst`, interior [pml, n-pml) only.  `direction` multiplies only the first addend of the
// txx / tzz lines (operator precedence in the reference).
template <class R>
void k_born_source(const Geo<R> &g, const Wave<R> &src, Wave<R> &dst, const Model<R> &M,
                   int dir) {
  int lo = g.pml;
  const R scale = 1.0f;
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R tmp_vx_x = 0, tmp_vz_z = 0, tmp_vx_z = 0, tmp_vz_x = 0;
    for (int i = 1; i <= 4; i++) {
      tmp_vx_x += g.c[i] * (src.vx[g.I(ix + i - 1, iz)] - src.vx[g.I(ix - i, iz)]);
      tmp_vz_z += g.c[i] * (src.vz[g.I(ix, iz + i - 1)] - src.vz[g.I(ix, iz - i)]);
      tmp_vx_z += g.c[i] * (src.vx[g.I(ix, iz + i)] - src.vx[g.I(ix, iz - i + 1)]);
      tmp_vz_x += g.c[i] * (src.vz[g.I(ix + i, iz)] - src.vz[g.I(ix - i + 1, iz)]);
    }
    R lam = M.lam[k], mu = M.mu[k], dmp = M.dmp[k], dms = M.dms[k];
    dst.txx[k] = dst.txx[k] + dir * scale * 2 * (lam + 2 * mu) * (-dmp) * (tmp_vx_x) / g.dx +
                 2 * ((lam + 2 * mu) * (-dmp) - 2 * mu * (-dms)) * (tmp_vz_z) / g.dz;
    dst.tzz[k] = dst.tzz[k] + dir * scale * 2 * ((lam + 2 * mu) * (-dmp) - 2 * mu * (-dms)) * (tmp_vx_x) / g.dx +
                 2 * (lam + 2 * mu) * (-dmp) * (tmp_vz_z) / g.dz;
    dst.txz[k] = dst.txz[k] + dir * scale * 2 * mu * (-dms) * ((tmp_vz_x) / g.dx + (tmp_vx_z) / g.dz);
  }
}

// born.cu:408-527 add_born_source_adjoint: from the adjoint stresses of `src` into the
// velocities of `dst`.  The txz x-term weights both samples with the modulus at ix+i-1
// (born.cu:514-515).
template <class R>
void k_born_source_adjoint(const Geo<R> &g, const Wave<R> &src, Wave<R> &dst, const Model<R> &M,
                           int dir) {
  int lo = g.pml;
  auto P = [&](size_t q) { return 2 * (M.lam[q] + 2 * M.mu[q]) * (-M.dmp[q]); };
  auto Q = [&](size_t q) {
    return 2 * ((M.lam[q] + 2 * M.mu[q]) * (-M.dmp[q]) - 2 * M.mu[q] * (-M.dms[q]));
  };
  auto S = [&](size_t q) { return 2 * M.mu[q] * (-M.dms[q]); };
  FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
    size_t k = g.I(ix, iz);
    R txx_x = 0, txx_z = 0, tzz_x = 0, tzz_z = 0, txz_x = 0, txz_z = 0;
    for (int i = 1; i <= 4; i++) {
      size_t xp = g.I(ix + i, iz), xq = g.I(ix - i + 1, iz);
      size_t zp = g.I(ix, iz + i), zq = g.I(ix, iz - i + 1);
      size_t xa = g.I(ix + i - 1, iz), xb = g.I(ix - i, iz);
      size_t za = g.I(ix, iz + i - 1), zb = g.I(ix, iz - i);
      txx_x += g.c[i] * (P(xp) * src.txx[xp] - P(xq) * src.txx[xq]);
      txx_z += g.c[i] * (Q(zp) * src.txx[zp] - Q(zq) * src.txx[zq]);
      tzz_x += g.c[i] * (Q(xp) * src.tzz[xp] - Q(xq) * src.tzz[xq]);
      tzz_z += g.c[i] * (P(zp) * src.tzz[zp] - P(zq) * src.tzz[zq]);
      txz_x += g.c[i] * (S(xa) * src.txz[xa] - S(xa) * src.txz[xb]);
      txz_z += g.c[i] * (S(za) * src.txz[za] - S(zb) * src.txz[zb]);
    }
    dst.vx[k] = dst.vx[k] + dir * (1.0 / M.rho[k]) * (txx_x / g.dx + tzz_x / g.dx + txz_z / g.dz);
    dst.vz[k] = dst.vz[k] + dir * (1.0 / M.rho[k]) * (tzz_z / g.dz + txx_z / g.dz + txz_x / g.dx);
  }
}

// FD2DGPU.cu:3093-3101 GPUrecord_scatterwavefield: rec[tr*nt + it] = v[igx, igz].
template <class R>
void k_record(const Geo<R> &g, const orc_shot *s, int nt, int it, const Vec<R> &vz,
              const Vec<R> &vx, Vec<R> &rz, Vec<R> &rx) {
  for (int tr = 0; tr < s->ntr; tr++) {
    size_t k = g.I(s->igx[tr], s->igz);
    rz[(size_t)tr * nt + it] = vz[k];
    rx[(size_t)tr * nt + it] = vx[k];
  }
}

// FD2DGPU.cu:3306-3322 GPUapplysource_backward_from_record with stack = true.
template <class R>
void k_inject(const Geo<R> &g, const orc_shot *s, int nt, int it, Wave<R> &w, const Vec<R> &rz,
              const Vec<R> &rx) {
  for (int tr = 0; tr < s->ntr; tr++) {
    size_t k = g.I(s->igx[tr], s->igz);
    w.vz[k] += rz[(size_t)tr * nt + it];
    w.vx[k] += rx[(size_t)tr * nt + it];
  }
}

// Boundary strips of vx, vz: 2N-wide bands on each side of the interior/PML interface,
// FD2DGPU.cu:3674-3731 (2-field record_edge_wavefield / load_edge_wavefield), N = nop.
template <class R>
struct Strips {
  int N, nx, nz;  // nx, nz: interior window
  Vec<R> up_x, up_z, dn_x, dn_z, lf_x, lf_z, rt_x, rt_z;
  Strips(const Geo<R> &g, int nt) : N(g.nop), nx(g.wnx), nz(g.wnz) {
    size_t a = (size_t)nt * nx * 2 * N, b = (size_t)nt * 2 * N * nz;
    up_x.assign(a, 0); up_z.assign(a, 0); dn_x.assign(a, 0); dn_z.assign(a, 0);
    lf_x.assign(b, 0); lf_z.assign(b, 0); rt_x.assign(b, 0); rt_z.assign(b, 0);
  }
  template <bool kSave>
  void move(const Geo<R> &g, Vec<R> &vx, Vec<R> &vz, int it) {
    int pml = g.pml;
    for (int ix = pml; ix < g.nx - pml; ix++)
      for (int iz = pml - N; iz < pml + N; iz++) {
        size_t o = (size_t)it * nx * 2 * N + (size_t)(ix - pml) * 2 * N + (iz - (pml - N));
        xfer<kSave>(vx[g.I(ix, iz)], up_x[o]);
        xfer<kSave>(vz[g.I(ix, iz)], up_z[o]);
      }
    for (int ix = pml; ix < g.nx - pml; ix++)
      for (int iz = g.nz - pml - N; iz < g.nz - pml + N; iz++) {
        size_t o = (size_t)it * nx * 2 * N + (size_t)(ix - pml) * 2 * N + (iz - (g.nz - pml - N));
        xfer<kSave>(vx[g.I(ix, iz)], dn_x[o]);
        xfer<kSave>(vz[g.I(ix, iz)], dn_z[o]);
      }
    for (int ix = pml - N; ix < pml + N; ix++)
      for (int iz = pml; iz < g.nz - pml; iz++) {
        size_t o = (size_t)it * 2 * N * nz + (size_t)(ix - (pml - N)) * nz + (iz - pml);
        xfer<kSave>(vx[g.I(ix, iz)], lf_x[o]);
        xfer<kSave>(vz[g.I(ix, iz)], lf_z[o]);
      }
    for (int ix = g.nx - pml - N; ix < g.nx - pml + N; ix++)
      for (int iz = pml; iz < g.nz - pml; iz++) {
        size_t o = (size_t)it * 2 * N * nz + (size_t)(ix - (g.nx - pml - N)) * nz + (iz - pml);
        xfer<kSave>(vx[g.I(ix, iz)], rt_x[o]);
        xfer<kSave>(vz[g.I(ix, iz)], rt_z[o]);
      }
  }
  template <bool kSave>
  static void xfer(R &field, R &store) {
    if (kSave) store = field; else field = store;
  }
};

// FD2DGPU.cu:3245-3263 doimage_gradient into a window image [wnx][wnz].
template <class R>
void k_image(const Geo<R> &g, const Model<R> &M, const Strain<R> &e, const Wave<R> &adj,
             Vec<R> &pp, Vec<R> &ps) {
  const R scale = 1.0f;
#pragma omp parallel for schedule(static)
  for (int ix = 0; ix < g.wnx; ix++)
    for (int iz = 0; iz < g.wnz; iz++) {
      size_t k = g.I(ix + g.pml, iz + g.pml);
      R lamda_grad = (e.gx_vx[k] + e.gz_vz[k]) * (adj.txx[k] + adj.tzz[k]);
      R miu_grad = -2 * (e.gx_vx[k] * adj.tzz[k] + e.gz_vz[k] * adj.txx[k]) +
                   (e.gz_vx[k] + e.gx_vz[k]) * adj.txz[k];
      R cpp = -2 * M.vp[k] * M.vp[k] * M.rho[k] * lamda_grad;
      R cps = -2 * M.vs[k] * M.vs[k] * M.rho[k] * miu_grad;
      size_t o = (size_t)ix * g.wnz + iz;
      pp[o] += scale * cpp;
      ps[o] += scale * cps;
    }
}

// FD2DGPU.cu:3235-3242 doimage_illum.
template <class R>
void k_illum(const Geo<R> &g, const Wave<R> &w, Vec<R> &il) {
  const R scale = 1.0f;
#pragma omp parallel for schedule(static)
  for (int ix = 0; ix < g.wnx; ix++)
    for (int iz = 0; iz < g.wnz; iz++) {
      size_t k = g.I(ix + g.pml, iz + g.pml);
      R illumination = w.vx[k] * w.vx[k] + w.vz[k] * w.vz[k];
      il[(size_t)ix * g.wnz + iz] += scale * illumination;
    }
}

template <class R>
void fwd_background_step(const Geo<R> &g, Wave<R> &w, const Model<R> &M, const float *wav,
                         const orc_shot *s, int it) {
  // FD2DGPU.cu:2039-2049 elastic_rotation_addS_for: txx, tzz += s[it] before the update.
  size_t ks = g.I(s->isx, s->isz);
  w.txx[ks] += (R)wav[it];
  w.tzz[ks] += (R)wav[it];
  // FD2DGPU.cu:1839-1844 born_modeling mode 0.
  k_update_vx(g, w, M, 1, g.nop);
  k_update_vz(g, w, M, 1, g.nop);
  k_update_txx_tzz(g, w, M, 1, g.nop, (Strain<R> *)nullptr);
  k_update_txz(g, w, M, 1, g.nop, (Strain<R> *)nullptr);
}

template <class R>
int forward_impl(const orc_grid *gg, const float *const model[7], const float *wav, int nt,
                 const orc_shot *s, double *rec_vz, double *rec_vx) {
  Geo<R> g(gg);
  Model<R> M = load_model(g, model, nullptr, nullptr);
  Wave<R> w(g.n);
  Vec<R> rz((size_t)s->ntr * nt), rx((size_t)s->ntr * nt);
  for (int it = 0; it < nt; it++) {
    fwd_background_step(g, w, M, wav, s, it);
    k_record(g, s, nt, it, w.vz, w.vx, rz, rx);
  }
  for (size_t i = 0; i < rz.size(); i++) {
    rec_vz[i] = rz[i];
    rec_vx[i] = rx[i];
  }
  return 0;
}

// First-order Born modelling, FD2DGPU.cu:1820-1831 (born_modeling mode 1) after the explosive
// source: background step, add_born_source of the new background velocities into the scattered
// stresses (born.cu:351-405), scattered step; the scattered velocities are recorded.  With
// vs = 0 (mu = 0) this is the acoustic Born operator of the elastic scheme.
template <class R>
int born_impl(const orc_grid *gg, const float *const model[7], const float *dmp,
              const float *dms, const float *wav, int nt, const orc_shot *s, double *rec_vz,
              double *rec_vx) {
  Geo<R> g(gg);
  Model<R> M = load_model(g, model, dmp, dms);
  Wave<R> w(g.n), b(g.n);
  Vec<R> rz((size_t)s->ntr * nt), rx((size_t)s->ntr * nt);
  for (int it = 0; it < nt; it++) {
    fwd_background_step(g, w, M, wav, s, it);
    k_born_source(g, w, b, M, 1);
    k_update_vx(g, b, M, 1, g.nop);
    k_update_vz(g, b, M, 1, g.nop);
    k_update_txx_tzz(g, b, M, 1, g.nop, (Strain<R> *)nullptr);
    k_update_txz(g, b, M, 1, g.nop, (Strain<R> *)nullptr);
    k_record(g, s, nt, it, b.vz, b.vx, rz, rx);
  }
  for (size_t i = 0; i < rz.size(); i++) {
    rec_vz[i] = rz[i];
    rec_vx[i] = rx[i];
  }
  return 0;
}

// FD2DGPU.cu:4556-4664: NCC adjoint source (double host arithmetic).
void ncc_residual(int ntr, int nt, const std::vector<double> &sz, const std::vector<double> &sx,
                  const float *dz_obs, const float *dx_obs, int iter, std::vector<double> &rz,
                  std::vector<double> &rx, double *misfit) {
  rz.assign((size_t)ntr * nt, 0.0);
  rx.assign((size_t)ntr * nt, 0.0);
  for (int i = 0; i < ntr; i++) {
    double dx = 0, Dx = 0, dDx = 0, dz = 0, Dz = 0, dDz = 0;
    for (int j = 0; j < nt; j++) {
      size_t q = (size_t)i * nt + j;
      double ox = dx_obs[q], oz = dz_obs[q];
      Dx += ox * ox;
      Dz += oz * oz;
      if (iter != 0) {
        dx += sx[q] * sx[q];
        dz += sz[q] * sz[q];
        dDx += sx[q] * ox;
        dDz += sz[q] * oz;
      }
    }
    if (iter == 0) {
      // FD2DGPU.cu:4567-4572: r = 1/(sqrt(D)*sqrt(D)) * (0 - d)
      for (int j = 0; j < nt; j++) {
        size_t q = (size_t)i * nt + j;
        rx[q] = 1 / (std::sqrt(Dx) * std::sqrt(Dx)) * (0.0f - dx_obs[q]);
        rz[q] = 1 / (std::sqrt(Dz) * std::sqrt(Dz)) * (0.0f - dz_obs[q]);
      }
    } else {
      // FD2DGPU.cu:4615-4623
      if (misfit)
        *misfit -= (1.0f / (2 * ntr)) *
                   (dDx / (std::sqrt(dx) * std::sqrt(Dx)) + dDz / (std::sqrt(dz) * std::sqrt(Dz)));
      for (int j = 0; j < nt; j++) {
        size_t q = (size_t)i * nt + j;
        rx[q] = 1 / (std::sqrt(dx) * std::sqrt(Dx)) * ((dDx / dx) * sx[q] - dx_obs[q]);
        rz[q] = 1 / (std::sqrt(dz) * std::sqrt(Dz)) * ((dDz / dz) * sz[q] - dz_obs[q]);
      }
    }
  }
}

template <class R>
int elsrtm_impl(const orc_grid *gg, const float *const model[7], const float *dmp,
                const float *dms, const float *wav, int nt, const orc_shot *s,
                const float *obs_vz, const float *obs_vx, int iter, int rbc, int adjoint_born,
                   double *lm_vz,
                double *lm_vx, double *res_vz, double *res_vx, double *const img[7],
                double *misfit) {
  Geo<R> g(gg);
  Model<R> M = load_model(g, model, dmp, dms);
  Wave<R> w(g.n), b(g.n), b2(g.n), wbk(g.n), bbk(g.n);
  Strain<R> e(g.n), be(g.n);
  size_t nrec = (size_t)s->ntr * nt;
  Vec<R> sz(nrec), sx(nrec), s2z(nrec), s2x(nrec);
  Strips<R> *st = nullptr, *st2 = nullptr;
  if (!rbc) {
    st = new Strips<R>(g, nt);
    st2 = new Strips<R>(g, nt);
  }
  // Forward pass, FD2DGPU.cu:4396-4478.
  for (int it = 0; it < nt; it++) {
    fwd_background_step(g, w, M, wav, s, it);                        // addS + mode 0
    k_born_source(g, w, b, M, 1);                                     // mode 3
    k_update_vx(g, b, M, 1, g.nop);
    k_update_vz(g, b, M, 1, g.nop);
    k_update_txx_tzz(g, b, M, 1, g.nop, (Strain<R> *)nullptr);       // mode 4
    k_update_txz(g, b, M, 1, g.nop, (Strain<R> *)nullptr);
    k_born_source(g, b, b2, M, 1);                                    // mode 5
    k_update_vx(g, b2, M, 1, g.nop);
    k_update_vz(g, b2, M, 1, g.nop);
    k_update_txx_tzz(g, b2, M, 1, g.nop, (Strain<R> *)nullptr);
    k_update_txz(g, b2, M, 1, g.nop, (Strain<R> *)nullptr);
    k_record(g, s, nt, it, b.vz, b.vx, sz, sx);                       // record_scatter(it, true)
    k_record(g, s, nt, it, b2.vz, b2.vx, s2z, s2x);
    if (!rbc) {
      st->template move<true>(g, w.vx, w.vz, it);
      st2->template move<true>(g, b.vx, b.vz, it);
    }
  }
  // scatter_add(1.0): Lm + Lm2 (FD2DGPU.cu:3119-3132, alpha = 1).
  std::vector<double> lz(nrec), lx(nrec);
  for (size_t q = 0; q < nrec; q++) {
    sz[q] = (R)1.0f * sz[q] + s2z[q];
    sx[q] = (R)1.0f * sx[q] + s2x[q];
    lz[q] = sz[q];
    lx[q] = sx[q];
  }
  if (lm_vz) std::copy(lz.begin(), lz.end(), lm_vz);
  if (lm_vx) std::copy(lx.begin(), lx.end(), lm_vx);
  std::vector<double> rzd, rxd;
  ncc_residual(s->ntr, nt, lz, lx, obs_vz, obs_vx, iter, rzd, rxd, misfit);
  // The residual is stored as float on the device (FD2DGPU.cu:4663-4664).
  Vec<R> rz(nrec), rx(nrec);
  for (size_t q = 0; q < nrec; q++) {
    rz[q] = (R)(float)rzd[q];
    rx[q] = (R)(float)rxd[q];
  }
  if (res_vz) for (size_t q = 0; q < nrec; q++) res_vz[q] = rz[q];
  if (res_vx) for (size_t q = 0; q < nrec; q++) res_vx[q] = rx[q];
  size_t wn = (size_t)g.wnx * g.wnz;
  Vec<R> im[7];
  for (int a = 0; a < 7; a++) im[a].assign(wn, 0);
  // Backward pass, FD2DGPU.cu:4685-4807.
  for (int it = nt - 1; it >= 0; --it) {
    if (!rbc) {
      st->template move<false>(g, w.vx, w.vz, it);
      st2->template move<false>(g, b.vx, b.vz, it);
    }
    k_update_txz(g, w, M, -1, g.pml, &e);                  // calculateTxz(-1, forward)
    k_update_txx_tzz(g, w, M, -1, g.pml, &e);              // calculateTxxzz(-1, forward)
    k_update_vz(g, w, M, -1, g.pml);                       // calculateVz
    k_update_vx(g, w, M, -1, g.pml);                       // calculateVx
    // pure_born_reconstruct_backward(-1, forward), FD2DGPU.cu:1864-1874
    k_update_txx_tzz(g, b, M, -1, g.pml, &be);
    k_update_txz(g, b, M, -1, g.pml, &be);
    k_born_source(g, w, b, M, 1);
    k_update_vx(g, b, M, -1, g.pml);
    k_update_vz(g, b, M, -1, g.pml);
    k_inject(g, s, nt, it, wbk, rz, rx);                    // elastic_rotation_addS_bac(stack)
    k_adj_txz(g, wbk, M, -1);                               // calculateTxz(-1, backward)
    k_adj_txx_tzz(g, wbk, M, -1);
    k_adj_vz(g, wbk, M, -1);
    k_adj_vx(g, wbk, M, -1);
    // pure_born_reconstruct_backward(-1, backward), FD2DGPU.cu:1881-1889.  On a GPU the
    // reference's add_born_source_adjoint launch fails (96 registers x 1024 threads per block >
    // 65,536; the error is never checked), so its runs leave the scattered adjoint at zero:
    // adjoint_born = 0 reproduces that, 1 evaluates the term as written.
    if (adjoint_born) {
      k_adj_vz(g, bbk, M, -1);
      k_adj_vx(g, bbk, M, -1);
      k_born_source_adjoint(g, wbk, bbk, M, -1);
      k_adj_txx_tzz(g, bbk, M, -1);
      k_adj_txz(g, bbk, M, -1);
    }
    // image_gradient, FD2DGPU.cu:3333-3342
    k_image(g, M, e, wbk, im[0], im[1]);
    k_image(g, M, be, wbk, im[3], im[4]);
    k_image(g, M, e, bbk, im[5], im[6]);
    k_illum(g, w, im[2]);
  }
  for (int a = 0; a < 7; a++)
    if (img && img[a])
      for (size_t q = 0; q < wn; q++) img[a][q] = im[a][q];
  delete st;
  delete st2;
  return 0;
}

template <class R>
int rtm_impl(const orc_grid *gg, const float *const model[7], const float *wav, int nt,
             const orc_shot *s, const float *adj_vz, const float *adj_vx, int rbc,
             double *const img[3]) {
  Geo<R> g(gg);
  Model<R> M = load_model(g, model, nullptr, nullptr);
  Wave<R> w(g.n), wbk(g.n);
  Strain<R> e(g.n);
  Strips<R> *st = rbc ? nullptr : new Strips<R>(g, nt);
  for (int it = 0; it < nt; it++) {
    fwd_background_step(g, w, M, wav, s, it);
    if (st) st->template move<true>(g, w.vx, w.vz, it);
  }
  size_t nrec = (size_t)s->ntr * nt;
  Vec<R> rz(adj_vz, adj_vz + nrec), rx(adj_vx, adj_vx + nrec);
  size_t wn = (size_t)g.wnx * g.wnz;
  Vec<R> pp(wn, 0), ps(wn, 0), il(wn, 0);
  for (int it = nt - 1; it >= 0; --it) {
    if (st) st->template move<false>(g, w.vx, w.vz, it);
    k_update_txz(g, w, M, -1, g.pml, &e);
    k_update_txx_tzz(g, w, M, -1, g.pml, &e);
    k_update_vz(g, w, M, -1, g.pml);
    k_update_vx(g, w, M, -1, g.pml);
    k_inject(g, s, nt, it, wbk, rz, rx);
    k_adj_txz(g, wbk, M, -1);
    k_adj_txx_tzz(g, wbk, M, -1);
    k_adj_vz(g, wbk, M, -1);
    k_adj_vx(g, wbk, M, -1);
    k_image(g, M, e, wbk, pp, ps);
    k_illum(g, w, il);
  }
  for (size_t q = 0; q < wn; q++) {
    if (img[0]) img[0][q] = pp[q];
    if (img[1]) img[1][q] = ps[q];
    if (img[2]) img[2][q] = il[q];
  }
  delete st;
  return 0;
}

// ---- acoustic Born operator pair (exact discrete adjoint), FP64 -----------------------------
// Fields vx, vz, s (s = txx = tzz of the mu = 0 elastic scheme).  U = [nop, n-nop)^2 is the
// updated set, I = [pml, n-pml)^2 the interior carrying the Born source.  With a PML (non-zero
// damping) the update is the reference's split form with mu = 0 (born.cu:215-349): vx is damped
// in x only and vz in z only (their z / x parts are driven by txz = 0), and s = s_x + s_z with
// s_x <- (d1x s_x + lam dt/dx Dx- vx) / d2x, s_z likewise in z, d1 = 1 - dt d / 2, d2 = 1 + dt d / 2.
// PML cells are those of the geometric PML (ix < pml, ix > nx - pml, likewise in z) and carry
// s_x, s_z; the other cells carry only s.  Without damping (random band) no cell is split.
struct AcOp {
  Geo<double> g;
  Vec<double> b, lam, d1x, d2x, d1z, d2z;
  Vec<char> split;
  bool has_pml = false;
  double cx, cz;  // dt/dx, dt/dz
  explicit AcOp(const orc_grid *gg, const float *const model[7]) : g(gg) {
    b.resize(g.n);
    lam.resize(g.n);
    d1x.resize(g.n); d2x.resize(g.n); d1z.resize(g.n); d2z.resize(g.n);
    split.assign(g.n, 0);
    for (size_t k = 0; k < g.n; k++) {
      b[k] = 1.0 / (double)model[2][k];
      lam[k] = model[3][k];
      const double hx = g.dt * (double)model[5][k] * 0.5, hz = g.dt * (double)model[6][k] * 0.5;
      d1x[k] = 1.0 - hx; d2x[k] = 1.0 + hx; d1z[k] = 1.0 - hz; d2z[k] = 1.0 + hz;
      if (model[5][k] != 0.f || model[6][k] != 0.f) has_pml = true;
    }
    if (has_pml)
      for (int ix = 0; ix < g.nx; ix++)
        for (int iz = 0; iz < g.nz; iz++)
          split[I(ix, iz)] = ix < g.pml || ix > g.nx - g.pml || iz < g.pml || iz > g.nz - g.pml;
    cx = g.dt / g.dx;
    cz = g.dt / g.dz;
  }
  size_t I(int ix, int iz) const { return g.I(ix, iz); }
  // Dx+ f = sum c_i (f[x+i] - f[x-i+1]); Dx- f = sum c_i (f[x+i-1] - f[x-i]); same in z.
  template <class F> double dxp(F f, int ix, int iz) const {
    double t = 0;
    for (int i = 1; i <= 4; i++) t += g.c[i] * (f(I(ix + i, iz)) - f(I(ix - i + 1, iz)));
    return t;
  }
  template <class F> double dxm(F f, int ix, int iz) const {
    double t = 0;
    for (int i = 1; i <= 4; i++) t += g.c[i] * (f(I(ix + i - 1, iz)) - f(I(ix - i, iz)));
    return t;
  }
  template <class F> double dzp(F f, int ix, int iz) const {
    double t = 0;
    for (int i = 1; i <= 4; i++) t += g.c[i] * (f(I(ix, iz + i)) - f(I(ix, iz - i + 1)));
    return t;
  }
  template <class F> double dzm(F f, int ix, int iz) const {
    double t = 0;
    for (int i = 1; i <= 4; i++) t += g.c[i] * (f(I(ix, iz + i - 1)) - f(I(ix, iz - i)));
    return t;
  }
  // One step: v += b dt/d D+ (s + e + source), then s += lam (dt/dx Dx- vx + dt/dz Dz- vz);
  // split (damped) in PML cells.  dir = -1 undoes a dir = +1 step exactly (stress first, then
  // velocities) on a grid without damping.
  void step(Vec<double> &vx, Vec<double> &vz, Vec<double> &s, Vec<double> &sx, Vec<double> &sz,
            const Vec<double> *e, long ksrc, double sval, int dir) const {
    const int lo = g.nop;
    auto S = [&](size_t q) {
      double v = s[q];
      if (e) v += (*e)[q];
      if ((long)q == ksrc) v += sval;
      return v;
    };
    auto vstage = [&]() {
      FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
        size_t k = I(ix, iz);
        if (split[k]) {
          vx[k] = (d1x[k] * vx[k] + b[k] * cx * dxp(S, ix, iz)) / d2x[k];
          vz[k] = (d1z[k] * vz[k] + b[k] * cz * dzp(S, ix, iz)) / d2z[k];
        } else {
          vx[k] += dir * b[k] * cx * dxp(S, ix, iz);
          vz[k] += dir * b[k] * cz * dzp(S, ix, iz);
        }
      }
    };
    auto sstage = [&]() {
      auto VX = [&](size_t q) { return vx[q]; };
      auto VZ = [&](size_t q) { return vz[q]; };
      FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
        size_t k = I(ix, iz);
        if (split[k]) {
          sx[k] = (d1x[k] * sx[k] + lam[k] * cx * dxm(VX, ix, iz)) / d2x[k];
          sz[k] = (d1z[k] * sz[k] + lam[k] * cz * dzm(VZ, ix, iz)) / d2z[k];
          s[k] = sx[k] + sz[k];
        } else {
          s[k] += dir * lam[k] * (cx * dxm(VX, ix, iz) + cz * dzm(VZ, ix, iz));
        }
      }
    };
    if (dir > 0) { vstage(); sstage(); } else { sstage(); vstage(); }
  }
  // Born source e = -2 lam m (Dx- vx / dx + Dz- vz / dz) on I.
  void born(const Vec<double> &vx, const Vec<double> &vz, const double *m, Vec<double> &e) const {
    auto VX = [&](size_t q) { return vx[q]; };
    auto VZ = [&](size_t q) { return vz[q]; };
    FOR_CELLS(g.pml, g.nx - g.pml, g.pml, g.nz - g.pml) {
      size_t k = I(ix, iz);
      e[k] = -2.0 * lam[k] * m[k] * (dxm(VX, ix, iz) / g.dx + dzm(VZ, ix, iz) / g.dz);
    }
  }
  // Transpose of one dir = +1 step acting on the adjoint state (y_s on unsplit cells, y_sx / y_sz
  // on split ones); returns the gradient with respect to the injected e in ge (on U).
  // Stress stage v' -> s': y_v' -= D+(lam dt/d y_s' [/ d2]), y_sx <- d1x / d2x y_sx'.
  // Velocity stage (v, S) -> v': y_S = -Dx-(b dt/dx y_vx' [/ d2x]) - Dz-(...), y_v <- d1/d2 y_v',
  // and S = s + e adds y_S to y_s (both parts on split cells) and to ge.
  void adj_step(Vec<double> &yx, Vec<double> &yz, Vec<double> &ys, Vec<double> &ysx,
                Vec<double> &ysz, Vec<double> &ge) const {
    const int lo = g.nop;
    Vec<double> wx(g.n, 0.0), wz(g.n, 0.0), ux(g.n, 0.0), uz(g.n, 0.0);
    FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
      size_t k = I(ix, iz);
      if (split[k]) {
        wx[k] = lam[k] * cx * ysx[k] / d2x[k];
        wz[k] = lam[k] * cz * ysz[k] / d2z[k];
      } else {
        wx[k] = lam[k] * cx * ys[k];
        wz[k] = lam[k] * cz * ys[k];
      }
    }
    auto WX = [&](size_t q) { return wx[q]; };
    auto WZ = [&](size_t q) { return wz[q]; };
    FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {  // transpose of the stress stage
      size_t k = I(ix, iz);
      yx[k] -= dxp(WX, ix, iz);
      yz[k] -= dzp(WZ, ix, iz);
      if (split[k]) {
        ysx[k] *= d1x[k] / d2x[k];
        ysz[k] *= d1z[k] / d2z[k];
      }
    }
    FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {
      size_t k = I(ix, iz);
      ux[k] = b[k] * cx * yx[k] / (split[k] ? d2x[k] : 1.0);
      uz[k] = b[k] * cz * yz[k] / (split[k] ? d2z[k] : 1.0);
    }
    auto UX = [&](size_t q) { return ux[q]; };
    auto UZ = [&](size_t q) { return uz[q]; };
    FOR_CELLS(lo, g.nx - lo, lo, g.nz - lo) {  // transpose of the velocity stage
      size_t k = I(ix, iz);
      const double gs = -dxm(UX, ix, iz) - dzm(UZ, ix, iz);
      if (split[k]) {
        ysx[k] += gs;
        ysz[k] += gs;
        yx[k] *= d1x[k] / d2x[k];
        yz[k] *= d1z[k] / d2z[k];
      } else {
        ys[k] += gs;
      }
      ge[k] = gs;
    }
  }
};

int ac_born(const orc_grid *gg, const float *const model[7], const float *wav, int nt,
            const orc_shot *s, const double *m, double *rz, double *rx) {
  AcOp op(gg, model);
  const Geo<double> &g = op.g;
  Vec<double> vx(g.n, 0), vz(g.n, 0), sg(g.n, 0), sgx(g.n, 0), sgz(g.n, 0);
  Vec<double> dvx(g.n, 0), dvz(g.n, 0), ds(g.n, 0), dsx(g.n, 0), dsz(g.n, 0), e(g.n, 0);
  const long ks = (long)g.I(s->isx, s->isz);
  for (int it = 0; it < nt; it++) {
    op.step(vx, vz, sg, sgx, sgz, nullptr, ks, wav[it], 1);
    op.born(vx, vz, m, e);
    op.step(dvx, dvz, ds, dsx, dsz, &e, -1, 0.0, 1);
    for (int tr = 0; tr < s->ntr; tr++) {
      size_t k = g.I(s->igx[tr], s->igz);
      rz[(size_t)tr * nt + it] = dvz[k];
      rx[(size_t)tr * nt + it] = dvx[k];
    }
  }
  return 0;
}

// Exact transpose of ac_born.  The background at each step comes from exact time reversal
// without damping, and from the stored forward history with a PML (damping cannot be reversed).
int ac_born_adj(const orc_grid *gg, const float *const model[7], const float *wav, int nt,
                const orc_shot *s, const double *rz, const double *rx, double *grad) {
  AcOp op(gg, model);
  const Geo<double> &g = op.g;
  Vec<double> vx(g.n, 0), vz(g.n, 0), sg(g.n, 0), sgx(g.n, 0), sgz(g.n, 0);
  Vec<double> yx(g.n, 0), yz(g.n, 0), ys(g.n, 0), ysx(g.n, 0), ysz(g.n, 0), ge(g.n, 0);
  const long ks = (long)g.I(s->isx, s->isz);
  std::vector<Vec<double>> hist;  // background velocities after each step (PML only)
  for (int it = 0; it < nt; it++) {
    op.step(vx, vz, sg, sgx, sgz, nullptr, ks, wav[it], 1);
    if (op.has_pml) {
      hist.push_back(vx);
      hist.push_back(vz);
    }
  }
  std::fill(grad, grad + g.n, 0.0);
  for (int it = nt - 1; it >= 0; --it) {
    for (int tr = 0; tr < s->ntr; tr++) {  // transpose of the recording after step it
      size_t k = g.I(s->igx[tr], s->igz);
      yz[k] += rz[(size_t)tr * nt + it];
      yx[k] += rx[(size_t)tr * nt + it];
    }
    op.adj_step(yx, yz, ys, ysx, ysz, ge);
    const Vec<double> &bx = op.has_pml ? hist[2 * it] : vx;
    const Vec<double> &bz = op.has_pml ? hist[2 * it + 1] : vz;
    auto VX = [&](size_t q) { return bx[q]; };
    auto VZ = [&](size_t q) { return bz[q]; };
    for (int ix = g.pml; ix < g.nx - g.pml; ix++)  // transpose of the Born source at step it
      for (int iz = g.pml; iz < g.nz - g.pml; iz++) {
        size_t k = g.I(ix, iz);
        grad[k] += -2.0 * op.lam[k] * (op.dxm(VX, ix, iz) / g.dx + op.dzm(VZ, ix, iz) / g.dz) * ge[k];
      }
    if (!op.has_pml) op.step(vx, vz, sg, sgx, sgz, nullptr, ks, wav[it], -1);  // back to it-1
  }
  return 0;
}

inline uint64_t splitmix64(uint64_t z) {
  // SplitMix64 finalizer (Steele, Lea, Flood 2014).
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

float orc_random_band_factor(uint64_t seed, int shot_id, int ix, int iz) {
  uint64_t h = splitmix64(seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(uint32_t)(shot_id + 1)));
  h = splitmix64(h ^ (((uint64_t)(uint32_t)ix << 32) | (uint32_t)iz));
  float u = (float)(h >> 40) * (1.0f / 16777216.0f);
  return std::fmaf(0.4f, u, 0.6f);
}

int orc_build_model(const orc_grid *g, int allnx, int allnz, const float *vp_all,
                    const float *vs_all, const float *rho_all, int win_left, int rbc,
                    uint64_t seed, int shot_id, float *vp, float *vs, float *rho, float *lam,
                    float *mu, float *dampx, float *dampz) {
  int nxp = g->nxpml, nzp = g->nzpml, pml = g->pml;
  int nx = nxp - 2 * pml, nz = nzp - 2 * pml;
  if (nz != allnz || win_left < 0 || win_left + nx > allnx) return -1;
  // log10(1/rr) with rr = 0.001f (FD2DGPU.cu:1299), profile ((pml - i)/pml)^4 (:444-494).
  const float rr = 0.001f;
  const double L = std::log10((double)(1.0f / rr));
  for (int ix = 0; ix < nxp; ix++)
    for (int iz = 0; iz < nzp; iz++) {
      int jx = std::min(std::max(ix - pml, 0), nx - 1);
      int jz = std::min(std::max(iz - pml, 0), nz - 1);
      size_t src = (size_t)(win_left + jx) * allnz + jz, k = (size_t)ix * nzp + iz;
      float p = vp_all[src], sv = vs_all[src];
      bool band = ix < pml || ix >= nxp - pml || iz < pml || iz >= nzp - pml;
      if (rbc && band) {
        float f = orc_random_band_factor(seed, shot_id, ix, iz);
        p = p * f;
        sv = sv * f;
      }
      float r = rho_all ? rho_all[src] : 2000.0f;
      vp[k] = p;
      vs[k] = sv;
      rho[k] = r;
      // FD2DGPU.cu:1117-1125 GPUcalculate_elastic_rho_C (float arithmetic, no contraction).
      float vp2 = p * p, vs2 = sv * sv;
      float twovs2 = 2.0f * vs2;
      float diff = vp2 - twovs2;
      lam[k] = r * diff;
      mu[k] = r * vs2;
      double dx = 0, dz = 0;
      if (!rbc) {
        double c = L * ((5.0 * (double)p) / (2.0 * pml));
        if (ix < pml) dx = c * std::pow((double)(pml - ix) / pml, 4.0);
        if (ix > nxp - pml) dx = c * std::pow((double)(ix - (nxp - pml)) / pml, 4.0);
        if (iz < pml) dz = c * std::pow((double)(pml - iz) / pml, 4.0);
        if (iz > nzp - pml) dz = c * std::pow((double)(iz - (nzp - pml)) / pml, 4.0);
      }
      dampx[k] = (float)dx;
      dampz[k] = (float)dz;
    }
  return 0;
}

int orc_window_image(const orc_grid *g, int allnx, int allnz, const float *img_all,
                     int win_left, float *img_pad) {
  int nxp = g->nxpml, nzp = g->nzpml, pml = g->pml;
  int nx = nxp - 2 * pml, nz = nzp - 2 * pml;
  if (nz != allnz || win_left < 0 || win_left + nx > allnx) return -1;
  for (int ix = 0; ix < nxp; ix++)
    for (int iz = 0; iz < nzp; iz++) {
      int jx = std::min(std::max(ix - pml, 0), nx - 1);
      int jz = std::min(std::max(iz - pml, 0), nz - 1);
      img_pad[(size_t)ix * nzp + iz] = img_all[(size_t)(win_left + jx) * allnz + jz];
    }
  return 0;
}

void orc_ricker(int nt, float f, float dt, float *s) {
  // main.cpp:461-473
  float pi = 3.14159265358979f;
  float t0 = 1 / f;
  int kt = (int)(t0 / dt);
  for (int i = 0; i < nt; i++) {
    float tt = i * dt - kt * dt;
    float sp = pi * f * tt;
    s[i] = (float)(1.0 * std::exp((double)(-sp * sp)) * (1. - 2. * sp * sp));
  }
}

int orc_forward_f64(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                    const orc_shot *s, double *rec_vz, double *rec_vx) {
  return forward_impl<double>(g, model, wavelet, nt, s, rec_vz, rec_vx);
}
int orc_forward_f32(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                    const orc_shot *s, double *rec_vz, double *rec_vx) {
  return forward_impl<float>(g, model, wavelet, nt, s, rec_vz, rec_vx);
}
int orc_born_f64(const orc_grid *g, const float *const model[7], const float *dm_p,
                 const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                 double *rec_vz, double *rec_vx) {
  return born_impl<double>(g, model, dm_p, dm_s, wavelet, nt, s, rec_vz, rec_vx);
}
int orc_born_f32(const orc_grid *g, const float *const model[7], const float *dm_p,
                 const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                 double *rec_vz, double *rec_vx) {
  return born_impl<float>(g, model, dm_p, dm_s, wavelet, nt, s, rec_vz, rec_vx);
}

int orc_elsrtm_f64(const orc_grid *g, const float *const model[7], const float *dm_p,
                   const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                   const float *obs_vz, const float *obs_vx, int iter, int rbc, int adjoint_born,
                   double *lm_vz,
                   double *lm_vx, double *res_vz, double *res_vx, double *const img[7],
                   double *misfit) {
  return elsrtm_impl<double>(g, model, dm_p, dm_s, wavelet, nt, s, obs_vz, obs_vx, iter, rbc,
                             adjoint_born, lm_vz, lm_vx, res_vz, res_vx, img, misfit);
}
int orc_elsrtm_f32(const orc_grid *g, const float *const model[7], const float *dm_p,
                   const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                   const float *obs_vz, const float *obs_vx, int iter, int rbc, int adjoint_born,
                   double *lm_vz,
                   double *lm_vx, double *res_vz, double *res_vx, double *const img[7],
                   double *misfit) {
  return elsrtm_impl<float>(g, model, dm_p, dm_s, wavelet, nt, s, obs_vz, obs_vx, iter, rbc,
                            adjoint_born, lm_vz, lm_vx, res_vz, res_vx, img, misfit);
}

int orc_rtm_f64(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                const orc_shot *s, const float *adj_vz, const float *adj_vx, int rbc,
                double *const img[3]) {
  return rtm_impl<double>(g, model, wavelet, nt, s, adj_vz, adj_vx, rbc, img);
}
int orc_rtm_f32(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                const orc_shot *s, const float *adj_vz, const float *adj_vx, int rbc,
                double *const img[3]) {
  return rtm_impl<float>(g, model, wavelet, nt, s, adj_vz, adj_vx, rbc, img);
}

int orc_ac_born(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                const orc_shot *s, const double *m, double *rec_vz, double *rec_vx) {
  return ac_born(g, model, wavelet, nt, s, m, rec_vz, rec_vx);
}

int orc_ac_born_adj(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                    const orc_shot *s, const double *rec_vz, const double *rec_vx, double *grad) {
  return ac_born_adj(g, model, wavelet, nt, s, rec_vz, rec_vx, grad);
}

void orc_ncc_residual(int ntr, int nt, const float *syn_vz, const float *syn_vx,
                      const float *obs_vz, const float *obs_vx, int iter, double *res_vz,
                      double *res_vx, double *misfit) {
  size_t n = (size_t)ntr * nt;
  std::vector<double> sz(syn_vz, syn_vz + n), sx(syn_vx, syn_vx + n), rz, rx;
  ncc_residual(ntr, nt, sz, sx, obs_vz, obs_vx, iter, rz, rx, misfit);
  std::copy(rz.begin(), rz.end(), res_vz);
  std::copy(rx.begin(), rx.end(), res_vx);
}

void orc_adam_update(int n, int iter, const float *const grads[6], float *image_pp,
                     float *image_ps, double *s_p, double *s_s, double *r_p, double *r_s) {
  // main.cpp:869-876 hyper-parameters, :1092-1131 update.
  const double beta1 = 0.8f, beta2 = 0.999f, alpha = 3e-5f, epsilon = 5e8f, gama = 0.99f;
  double alpha_k = iter == 0 ? alpha : (alpha / 2) * std::pow(gama, iter);
  int k = iter + 1;
  for (int i = 0; i < n; i++) {
    double gp = (double)grads[0][i] + grads[2][i] + grads[4][i];
    double gs = (double)grads[1][i] + grads[3][i] + grads[5][i];
    s_p[i] = beta1 * s_p[i] + (1 - beta1) * gp;
    s_s[i] = beta1 * s_s[i] + (1 - beta1) * gs;
    r_p[i] = beta2 * r_p[i] + (1 - beta2) * (gp * gp);
    r_s[i] = beta2 * r_s[i] + (1 - beta2) * (gs * gs);
    double mp = s_p[i] / (1 - std::pow(beta1, k)), ms = s_s[i] / (1 - std::pow(beta1, k));
    double vp = r_p[i] / (1 - std::pow(beta2, k)), vs = r_s[i] / (1 - std::pow(beta2, k));
    image_pp[i] = (float)(image_pp[i] - alpha_k * (mp / (std::sqrt(vp) + epsilon)));
    image_ps[i] = (float)(image_ps[i] - alpha_k * (ms / (std::sqrt(vs) + epsilon)));
  }
}

}  // extern "C"
