// Half-step kernels of the elastic velocity-stress scheme (reference born.cu:215-349 forward,
// FD2DGPU.cu:903-1082 reconstruction, FD2DGPU.cu:591-895 adjoint), one launch per half step for
// all resident shots (blockIdx.z = slot), plus the Born sources, strips, imaging and the NCC
// residual.  Each kernel updates arrays in place and only reads, at other cells, arrays it does
// not write -- the same hazard discipline as the reference kernels.
#pragma once
#include "ds2d_kernels.cuh"

namespace ds2d {

constexpr int kBX = 32;  // cells along z per block (one warp, coalesced)
constexpr int kBY = 8;   // cells along x per block

struct VelArgs {
  Dims d;
  Wave w;
  Par p;
  const float *ov_txx, *ov_tzz, *ov_txz;  // additive read overlays (Born source), or null
  const ShotDev *shots;
  const float *wavelet;
  int it;
  int src_on;            // explosive source on txx / tzz (FD2DGPU.cu:2039-2049)
  const int *rmap;       // [slot][nxp] receiver index or -1
  float *rec_vz, *rec_vx;  // [slot][max_ntr][nt]
  int rec_on;
  Strips st;
  int strips_outer;      // reconstruction: reload the strip cells outside the interior
};

template <int MODE>
__global__ void __launch_bounds__(kBX *kBY) k_vel(VelArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * kBX + threadIdx.x;
  const int ix = blockIdx.y * kBY + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp) return;
  const int lo = (MODE == kRev) ? d.pml : d.nop;
  const long long base = d.slot * s;
  const long long k = base + (long long)ix * d.ld + iz;
  if (ix < lo || ix >= d.nxp - lo || iz < lo || iz >= d.nzp - lo) {
    if (MODE == kRev && a.strips_outer) {
      const int bo = band_offset(d, ix, iz);
      if (bo >= 0) {
        a.w.vx[k] = strip_get(a.st, d, s, a.it, 0, bo);
        a.w.vz[k] = strip_get(a.st, d, s, a.it, 1, bo);
      }
    }
    return;
  }
  const int ld = d.ld;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float dir = (MODE == kFwd) ? 1.0f : -1.0f;
  const float bb = a.p.b[k];
  const float cbx = bb * dtdx, cbz = bb * dtdz;
  float ux_x, ux_z, uz_x, uz_z;  // increments of vx, vz; x- and z-parts kept apart for the PML
  if (MODE != kAdj) {
    const float *txx = a.w.txx, *tzz = a.w.tzz, *txz = a.w.txz;
    const float *oxx = a.ov_txx, *ozz = a.ov_tzz, *oxz = a.ov_txz;
    long long ksrc = -1;
    float sval = 0.f;
    if (a.src_on) {
      const ShotDev sh = a.shots[s];
      ksrc = base + (long long)sh.isx * ld + sh.isz;
      sval = a.wavelet[a.it];
    }
    auto rd = [&](const float *arr, const float *ov, long long q, bool srcf) {
      float v = __ldg(arr + q);
      if (ov) v += __ldg(ov + q);
      if (srcf && q == ksrc) v += sval;
      return v;
    };
    // born.cu:235-245 / 265-275
    const float ax = stencil4([&](int i) {
      return rd(txx, oxx, k + (long long)i * ld, true) - rd(txx, oxx, k + (long long)(1 - i) * ld, true);
    });
    const float bz = stencil4([&](int i) { return rd(txz, oxz, k + i - 1, false) - rd(txz, oxz, k - i, false); });
    const float fx = stencil4([&](int i) {
      return rd(txz, oxz, k + (long long)(i - 1) * ld, false) - rd(txz, oxz, k - (long long)i * ld, false);
    });
    const float ez = stencil4([&](int i) { return rd(tzz, ozz, k + i, true) - rd(tzz, ozz, k - i + 1, true); });
    ux_x = dir * cbx * ax;
    ux_z = dir * cbz * bz;
    uz_x = dir * cbx * fx;
    uz_z = dir * cbz * ez;
  } else {
    // FD2DGPU.cu:591-682: moduli inside the divergence.
    const float *txx = a.w.txx, *tzz = a.w.tzz, *txz = a.w.txz;
    const float *lam = a.p.lam, *mu = a.p.mu;
    auto l2m = [&](long long q) { return __ldg(lam + q) + 2.0f * __ldg(mu + q); };
    const float t_xx = stencil4([&](int i) {
      long long p = k + (long long)i * ld, q = k + (long long)(1 - i) * ld;
      return l2m(p) * __ldg(txx + p) - l2m(q) * __ldg(txx + q);
    });
    const float t_xz = stencil4([&](int i) {
      long long p = k + i - 1, q = k - i;
      return __ldg(mu + p) * __ldg(txz + p) - __ldg(mu + q) * __ldg(txz + q);
    });
    const float t_zx = stencil4([&](int i) {
      long long p = k + (long long)i * ld, q = k + (long long)(1 - i) * ld;
      return __ldg(lam + p) * __ldg(tzz + p) - __ldg(lam + q) * __ldg(tzz + q);
    });
    const float s_zz = stencil4([&](int i) {
      long long p = k + i, q = k - i + 1;
      return l2m(p) * __ldg(tzz + p) - l2m(q) * __ldg(tzz + q);
    });
    const float s_xz = stencil4([&](int i) {
      long long p = k + (long long)(i - 1) * ld, q = k - (long long)i * ld;
      return __ldg(mu + p) * __ldg(txz + p) - __ldg(mu + q) * __ldg(txz + q);
    });
    const float s_xx = stencil4([&](int i) {
      long long p = k + i, q = k - i + 1;
      return __ldg(lam + p) * __ldg(txx + p) - __ldg(lam + q) * __ldg(txx + q);
    });
    ux_x = fmaf(dir * cbx, t_zx, dir * cbx * t_xx);
    ux_z = dir * cbz * t_xz;
    uz_x = dir * cbx * s_xz;
    uz_z = fmaf(dir * cbz, s_xx, dir * cbz * s_zz);
  }
  float vx, vz;
  if (pml_cell(d, ix, iz)) {
    const float ddx = a.p.dampx[k] * d.dt * 0.5f, ddz = a.p.dampz[k] * d.dt * 0.5f;
    const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
    // (d1 v + u) / (1 + dt d / 2) as a multiply by the rounded reciprocal: a division takes its
    // slow path for the tiny amplitudes ahead of a wavefront
    const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);
    const float vxx = fmaf(d1, a.w.vx_x[k], ux_x) * i2;
    const float vxz = fmaf(d3, a.w.vx_z[k], ux_z) * i4;
    const float vzx = fmaf(d1, a.w.vz_x[k], uz_x) * i2;
    const float vzz = fmaf(d3, a.w.vz_z[k], uz_z) * i4;
    a.w.vx_x[k] = vxx;
    a.w.vx_z[k] = vxz;
    a.w.vz_x[k] = vzx;
    a.w.vz_z[k] = vzz;
    vx = vxx + vxz;
    vz = vzx + vzz;
  } else {
    vx = a.w.vx[k] + (ux_x + ux_z);
    vz = a.w.vz[k] + (uz_x + uz_z);
  }
  a.w.vx[k] = vx;
  a.w.vz[k] = vz;
  if (a.rec_on && iz == a.shots[s].igz) {
    const int tr = a.rmap[(long long)s * d.nxp_max + ix];
    if (tr >= 0) {
      const long long r = ((long long)s * d.max_ntr + tr) * d.nt + a.it;
      a.rec_vz[r] = vz;
      a.rec_vx[r] = vx;
    }
  }
}

struct StrArgs {
  Dims d;
  Wave w;
  Par p;
  Strain e;              // strains (reconstruction), gx_vx null = none
  Strips st;
  int strips_on;         // reconstruction: velocities of strip cells come from the strips
  int it;
  const ShotDev *shots;
  const int *rmap;
  const float *res_vz, *res_vx;  // [slot][max_ntr][nt] adjoint source, injected at the receivers
  int res_on;
  const float *ov_vx, *ov_vz;    // additive read overlays (adjoint Born source), or null
};

template <int MODE>
__global__ void __launch_bounds__(kBX *kBY) k_str(StrArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * kBX + threadIdx.x;
  const int ix = blockIdx.y * kBY + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp) return;
  const int lo = (MODE == kRev) ? d.pml : d.nop;
  if (ix < lo || ix >= d.nxp - lo || iz < lo || iz >= d.nzp - lo) return;
  const int ld = d.ld;
  const long long base = d.slot * s;
  const long long k = base + (long long)ix * ld + iz;
  const float *vxa = a.w.vx, *vza = a.w.vz;
  // Whether this block's stencil footprint can touch a strip band (warp-uniform).
  bool near_band = false;
  if (MODE == kRev && a.strips_on) {
    const int N = d.nop, pml = d.pml;
    const int x0 = blockIdx.y * kBY - 4, x1 = blockIdx.y * kBY + kBY + 3;
    const int z0 = blockIdx.x * kBX - 4, z1 = blockIdx.x * kBX + kBX + 3;
    near_band = x0 < pml + N || x1 >= d.nxp - pml - N || z0 < pml + N || z1 >= d.nzp - pml - N;
  }
  int igz = -1;
  const float *rz = nullptr, *rx = nullptr;
  const int *rmap = nullptr;
  if (a.res_on) {
    igz = a.shots[s].igz;
    rz = a.res_vz + (long long)s * d.max_ntr * d.nt + a.it;
    rx = a.res_vx + (long long)s * d.max_ntr * d.nt + a.it;
    rmap = a.rmap + (long long)s * d.nxp_max;
  }
  auto rv = [&](int comp, int qx, int qz) {
    if (MODE == kRev && near_band) {
      const int bo = band_offset(d, qx, qz);
      if (bo >= 0) return strip_get(a.st, d, s, a.it, comp, bo);
    }
    const long long q = base + (long long)qx * ld + qz;
    float v = __ldg((comp ? vza : vxa) + q);
    const float *ov = comp ? a.ov_vz : a.ov_vx;
    if (ov) v += __ldg(ov + q);
    if (qz == igz) {
      const int tr = rmap[qx];
      if (tr >= 0) v += comp ? rz[(long long)tr * d.nt] : rx[(long long)tr * d.nt];
    }
    return v;
  };
  // born.cu:300-304 / 336-340
  const float sa = stencil4([&](int i) { return rv(0, ix + i - 1, iz) - rv(0, ix - i, iz); });
  const float sb = stencil4([&](int i) { return rv(1, ix, iz + i - 1) - rv(1, ix, iz - i); });
  const float se = stencil4([&](int i) { return rv(0, ix, iz + i) - rv(0, ix, iz - i + 1); });
  const float sf = stencil4([&](int i) { return rv(1, ix + i, iz) - rv(1, ix - i + 1, iz); });
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float dir = (MODE == kFwd) ? 1.0f : -1.0f;
  const bool pml = pml_cell(d, ix, iz);
  float d1 = 1.f, i2 = 1.f, d3 = 1.f, i4 = 1.f;  // damping factors; i2, i4 = 1 / (1 + dt d / 2)
  if (pml) {
    const float ddx = a.p.dampx[k] * d.dt * 0.5f, ddz = a.p.dampz[k] * d.dt * 0.5f;
    d1 = 1.0f - ddx; i2 = __frcp_rn(1.0f + ddx); d3 = 1.0f - ddz; i4 = __frcp_rn(1.0f + ddz);
  }
  if (MODE != kAdj) {
    const float lam = a.p.lam[k], mu = a.p.mu[k];
    const float l2m = lam + 2.0f * mu;
    const float xx_x = dir * l2m * dtdx * sa, xx_z = dir * lam * dtdz * sb;
    const float zz_x = dir * lam * dtdx * sa, zz_z = dir * l2m * dtdz * sb;
    // operand order of update_txz (born.cu:344-345) forward, of _txz_grad (FD2DGPU.cu:1067-1068)
    // in reconstruction
    const float xz_x = MODE == kRev ? dir * mu * dtdx * sf : dir * dtdx * mu * sf;
    const float xz_z = MODE == kRev ? dir * mu * dtdz * se : dir * dtdz * mu * se;
    if (pml) {
      const float a1 = fmaf(d1, a.w.txx_x[k], xx_x) * i2;
      const float a2 = fmaf(d3, a.w.txx_z[k], xx_z) * i4;
      const float b1 = fmaf(d1, a.w.tzz_x[k], zz_x) * i2;
      const float b2 = fmaf(d3, a.w.tzz_z[k], zz_z) * i4;
      const float c1 = fmaf(d1, a.w.txz_x[k], xz_x) * i2;
      const float c2 = fmaf(d3, a.w.txz_z[k], xz_z) * i4;
      a.w.txx_x[k] = a1; a.w.txx_z[k] = a2;
      a.w.tzz_x[k] = b1; a.w.tzz_z[k] = b2;
      a.w.txz_x[k] = c1; a.w.txz_z[k] = c2;
      a.w.txx[k] = a1 + a2;
      a.w.tzz[k] = b1 + b2;
      a.w.txz[k] = c1 + c2;
    } else {
      a.w.txx[k] = a.w.txx[k] + (xx_x + xx_z);
      a.w.tzz[k] = a.w.tzz[k] + (zz_x + zz_z);
      a.w.txz[k] = a.w.txz[k] + (xz_x + xz_z);
    }
    if (MODE == kRev && a.e.gx_vx) {
      const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;  // reciprocal multiplies, as above
      a.e.gx_vx[k] = sa * rdx;
      a.e.gz_vz[k] = sb * rdz;
      a.e.gz_vx[k] = se * rdz;
      a.e.gx_vz[k] = sf * rdx;
    }
  } else {
    // FD2DGPU.cu:725-761, 860-895: no moduli; txx is txx_x, tzz is tzz_z.
    const float xx = dir * dtdx * sa, zz = dir * dtdz * sb;
    const float xz_x = dir * dtdx * sf, xz_z = dir * dtdz * se;
    if (pml) {
      a.w.txx[k] = fmaf(d1, a.w.txx[k], xx) * i2;
      a.w.tzz[k] = fmaf(d3, a.w.tzz[k], zz) * i4;
      const float c1 = fmaf(d1, a.w.txz_x[k], xz_x) * i2;
      const float c2 = fmaf(d3, a.w.txz_z[k], xz_z) * i4;
      a.w.txz_x[k] = c1; a.w.txz_z[k] = c2;
      a.w.txz[k] = c1 + c2;
    } else {
      a.w.txx[k] = a.w.txx[k] + xx;
      a.w.tzz[k] = a.w.tzz[k] + zz;
      a.w.txz[k] = a.w.txz[k] + (xz_x + xz_z);
    }
  }
}

// born.cu:351-405 add_born_source, written into read overlays of the scattered set's stresses
// (interior cells only; the overlays stay zero elsewhere).
struct BornArgs {
  Dims d;
  const ShotDev *shots;
  const float *vx, *vz;  // source-side velocities
  Par p;
  float *ov_txx, *ov_tzz, *ov_txz;
};

__global__ void __launch_bounds__(kBX *kBY) k_born(BornArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * kBX + threadIdx.x;
  const int ix = blockIdx.y * kBY + threadIdx.y;
  const int lo = d.pml;
  if (ix < lo || ix >= d.nxp - lo || iz < lo || iz >= d.nzp - lo) return;
  const int ld = d.ld;
  const long long k = d.slot * s + (long long)ix * ld + iz;
  const float *vx = a.vx, *vz = a.vz;
  const float vx_x = stencil4([&](int i) { return __ldg(vx + k + (long long)(i - 1) * ld) - __ldg(vx + k - (long long)i * ld); });
  const float vz_z = stencil4([&](int i) { return __ldg(vz + k + i - 1) - __ldg(vz + k - i); });
  const float vx_z = stencil4([&](int i) { return __ldg(vx + k + i) - __ldg(vx + k - i + 1); });
  const float vz_x = stencil4([&](int i) { return __ldg(vz + k + (long long)i * ld) - __ldg(vz + k + (long long)(1 - i) * ld); });
  const float lam = a.p.lam[k], mu = a.p.mu[k], dmp = a.p.dmp[k], dms = a.p.dms[k];
  const float l2m = lam + 2.0f * mu;
  const float P = 2.0f * l2m * (-dmp);
  const float Q = 2.0f * (l2m * (-dmp) - 2.0f * mu * (-dms));
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;  // reciprocal multiplies (no divide slow path)
  a.ov_txx[k] = P * vx_x * rdx + Q * vz_z * rdz;
  a.ov_tzz[k] = Q * vx_x * rdx + P * vz_z * rdz;
  a.ov_txz[k] = 2.0f * mu * (-dms) * (vz_x * rdx + vx_z * rdz);
}

// born.cu:408-527 add_born_source_adjoint into read overlays of the scattered adjoint
// velocities.  The txz x-term weights both samples with the modulus at ix+i-1 (born.cu:514).
struct BornAdjArgs {
  Dims d;
  const ShotDev *shots;
  const float *txx, *tzz, *txz;  // adjoint stresses of the background adjoint set
  Par p;
  float *ov_vx, *ov_vz;
};

__global__ void __launch_bounds__(kBX *kBY) k_born_adj(BornAdjArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * kBX + threadIdx.x;
  const int ix = blockIdx.y * kBY + threadIdx.y;
  const int lo = d.pml;
  if (ix < lo || ix >= d.nxp - lo || iz < lo || iz >= d.nzp - lo) return;
  const int ld = d.ld;
  const long long k = d.slot * s + (long long)ix * ld + iz;
  const float *lam = a.p.lam, *mu = a.p.mu, *dmp = a.p.dmp, *dms = a.p.dms;
  auto P = [&](long long q) { return 2.0f * (__ldg(lam + q) + 2.0f * __ldg(mu + q)) * (-__ldg(dmp + q)); };
  auto Q = [&](long long q) {
    return 2.0f * ((__ldg(lam + q) + 2.0f * __ldg(mu + q)) * (-__ldg(dmp + q)) - 2.0f * __ldg(mu + q) * (-__ldg(dms + q)));
  };
  auto S = [&](long long q) { return 2.0f * __ldg(mu + q) * (-__ldg(dms + q)); };
  const float *txx = a.txx, *tzz = a.tzz, *txz = a.txz;
  const float txx_x = stencil4([&](int i) {
    long long p = k + (long long)i * ld, q = k + (long long)(1 - i) * ld;
    return P(p) * __ldg(txx + p) - P(q) * __ldg(txx + q);
  });
  const float txx_z = stencil4([&](int i) {
    long long p = k + i, q = k - i + 1;
    return Q(p) * __ldg(txx + p) - Q(q) * __ldg(txx + q);
  });
  const float tzz_x = stencil4([&](int i) {
    long long p = k + (long long)i * ld, q = k + (long long)(1 - i) * ld;
    return Q(p) * __ldg(tzz + p) - Q(q) * __ldg(tzz + q);
  });
  const float tzz_z = stencil4([&](int i) {
    long long p = k + i, q = k - i + 1;
    return P(p) * __ldg(tzz + p) - P(q) * __ldg(tzz + q);
  });
  const float txz_x = stencil4([&](int i) {
    long long p = k + (long long)(i - 1) * ld, q = k - (long long)i * ld;
    return S(p) * __ldg(txz + p) - S(p) * __ldg(txz + q);
  });
  const float txz_z = stencil4([&](int i) {
    long long p = k + i - 1, q = k - i;
    return S(p) * __ldg(txz + p) - S(q) * __ldg(txz + q);
  });
  const float bb = -a.p.b[k];  // direction -1 (FD2DGPU.cu:1886)
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;  // reciprocal multiplies (no divide slow path)
  a.ov_vx[k] = bb * (txx_x * rdx + tzz_x * rdx + txz_z * rdz);
  a.ov_vz[k] = bb * (tzz_z * rdz + txx_z * rdz + txz_x * rdx);
}

// Saves the strip cells of (vx, vz) after forward step `it` (FD2DGPU.cu:4419-4444).  One warp
// per 32-element segment; 16-bit formats store q = v / scale with scale = segment max / 2^15.
struct StripSaveArgs {
  Dims d;
  const ShotDev *shots;
  const float *vx, *vz;
  Strips st;
  int it;
};

__global__ void __launch_bounds__(256) k_strip_save(StripSaveArgs a) {
  const int s = blockIdx.z, comp = blockIdx.y;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int bo = blockIdx.x * 256 + threadIdx.x;
  const bool valid = bo < d.lb;
  float v = 0.f;
  if (valid) {
    int ix, iz;
    band_cell(d, bo, ix, iz);
    v = (comp ? a.vz : a.vx)[d.slot * s + (long long)ix * d.ld + iz];
  }
  const long long row = ((long long)s * d.nt + a.it) * 2 + comp;
  const long long e = row * d.lb_max + bo;
  if (a.st.prec == 0) {
    if (valid) ((float *)a.st.data)[e] = v;
    return;
  }
  float m = fabsf(v);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  // Leading wavefront tails reach subnormal magnitudes, where m / 2^15 would underflow to 0;
  // clamping the scale at FLT_MIN keeps |q| <= 2^15 inside the fp16 range.
  const float sc = m > 0.f ? fmaxf(m * (1.0f / 32768.0f), 1.17549435e-38f) : 1.0f;
  if ((threadIdx.x & 31) == 0 && bo < d.lb) a.st.scale[row * d.nseg_max + (bo >> 5)] = sc;
  if (!valid) return;
  const float q = v / sc;
  if (a.st.prec == 1) ((__half *)a.st.data)[e] = __float2half_rn(q);
  else ((__nv_bfloat16 *)a.st.data)[e] = __float2bfloat16_rn(q);
}

// Zero-lag imaging, FD2DGPU.cu:3245-3263 doimage_gradient (x3 in reference mode) and
// :3235-3242 doimage_illum, accumulated per slot over the interior window [wnx][wnz].
struct ImgArgs {
  Dims d;
  const ShotDev *shots;
  Par p;
  Strain e, be;
  const float *atxx, *atzz, *atxz;   // adjoint stresses
  const float *btxx, *btzz, *btxz;   // scattered adjoint stresses (reference mode) or null
  const float *vx, *vz;              // reconstructed source velocities (illumination)
  float *img;                        // [7][slot][wnx][wnz]
  long long img_plane;               // slots * wnx * wnz
  int full;  // 0: pp, ps, illum; 1: + scattered-strain images; 2: + scattered-adjoint images
};

__device__ __forceinline__ void image_pair(const float *e0, const float *e1, const float *e2,
                                           const float *e3, const float *txx, const float *tzz,
                                           const float *txz, long long k, float kpp, float kps,
                                           float &pp, float &ps) {
  const float gx_vx = e0[k], gz_vz = e1[k], gz_vx = e2[k], gx_vz = e3[k];
  const float sxx = txx[k], szz = tzz[k], sxz = txz[k];
  const float lamda_grad = (gx_vx + gz_vz) * (sxx + szz);
  const float miu_grad = -2.0f * (gx_vx * szz + gz_vz * sxx) + (gz_vx + gx_vz) * sxz;
  pp = kpp * lamda_grad;
  ps = kps * miu_grad;
}

__global__ void __launch_bounds__(kBX *kBY) k_image(ImgArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * kBX + threadIdx.x;
  const int ix = blockIdx.y * kBY + threadIdx.y;
  if (ix >= d.wnx || iz >= d.wnz) return;
  const long long k = d.slot * s + (long long)(ix + d.pml) * d.ld + iz + d.pml;
  const long long o = ((long long)s * d.wnx_max + ix) * d.ild + (iz + d.pml);
  const float kpp = a.p.kpp[k], kps = a.p.kps[k];
  float pp, ps;
  image_pair(a.e.gx_vx, a.e.gz_vz, a.e.gz_vx, a.e.gx_vz, a.atxx, a.atzz, a.atxz, k, kpp, kps, pp, ps);
  a.img[o] += pp;
  a.img[a.img_plane + o] += ps;
  const float vx = a.vx[k], vz = a.vz[k];
  a.img[2 * a.img_plane + o] += vx * vx + vz * vz;
  if (a.full >= 1) {
    image_pair(a.be.gx_vx, a.be.gz_vz, a.be.gz_vx, a.be.gx_vz, a.atxx, a.atzz, a.atxz, k, kpp, kps, pp, ps);
    a.img[3 * a.img_plane + o] += pp;
    a.img[4 * a.img_plane + o] += ps;
  }
  if (a.full >= 2) {
    image_pair(a.e.gx_vx, a.e.gz_vz, a.e.gz_vx, a.e.gx_vz, a.btxx, a.btzz, a.btxz, k, kpp, kps, pp, ps);
    a.img[5 * a.img_plane + o] += pp;
    a.img[6 * a.img_plane + o] += ps;
  }
}

// Adds the per-slot window images into the model-size images (slot order, deterministic):
// the reference accumulates every shot into the same full image at column delta_left + ix
// (FD2DGPU.cu:3261-3262).
__global__ void k_image_reduce(Dims d, const float *img, long long img_plane, int nimg,
                               int nslots, const ShotDev *shots, float *full, long long full_plane) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = blockIdx.y;
  if (iz >= d.allnz) return;
  for (int a = 0; a < nimg; a++) {
    float acc = full[a * full_plane + (long long)col * d.allnz + iz];
    for (int s = 0; s < nslots; s++) {
      const int c = col - shots[s].win_left;
      if (c >= 0 && c < shots[s].wnx)
        acc += img[a * img_plane + ((long long)s * d.wnx_max + c) * d.ild + (iz + d.pml)];
    }
    full[a * full_plane + (long long)col * d.allnz + iz] = acc;
  }
}

// scatter_add(1.0): Lm + Lm2 (FD2DGPU.cu:3119-3132 GPU_add with alpha = 1).
__global__ void k_lm_add(float *sz, float *sx, const float *s2z, const float *s2x, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  sz[i] = 1.0f * sz[i] + s2z[i];
  sx[i] = 1.0f * sx[i] + s2x[i];
}

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  const int nw = blockDim.x >> 5;
  for (int i = 0; i < nw; i++) t += sh[i];
  return t;
}

// NCC adjoint source and per-trace misfit term (FD2DGPU.cu:4556-4664), one block per
// (trace, slot), FP64 sums of float products as the reference's host loops.
__global__ void __launch_bounds__(256) k_ncc(Dims d, const ShotDev *shots, const float *syn_z,
                                             const float *syn_x, const float *obs_z,
                                             const float *obs_x, float *res_z, float *res_x,
                                             double *mis_terms, int iter) {
  __shared__ double sh[8];
  const int tr = blockIdx.x, s = blockIdx.y;
  if (tr >= shots[s].ntr) return;
  const long long off = ((long long)s * d.max_ntr + tr) * d.nt;
  double dx = 0, Dx = 0, dDx = 0, dz = 0, Dz = 0, dDz = 0;
  for (int j = threadIdx.x; j < d.nt; j += blockDim.x) {
    const float ox = obs_x[off + j], oz = obs_z[off + j];
    const float sx = syn_x[off + j], sz = syn_z[off + j];
    Dx += (double)__fmul_rn(ox, ox);
    Dz += (double)__fmul_rn(oz, oz);
    dx += (double)__fmul_rn(sx, sx);
    dz += (double)__fmul_rn(sz, sz);
    dDx += (double)__fmul_rn(sx, ox);
    dDz += (double)__fmul_rn(sz, oz);
  }
  Dx = block_sum(Dx, sh); Dz = block_sum(Dz, sh);
  dx = block_sum(dx, sh); dz = block_sum(dz, sh);
  dDx = block_sum(dDx, sh); dDz = block_sum(dDz, sh);
  if (iter == 0) {
    const double cx = 1 / (sqrt(Dx) * sqrt(Dx)), cz = 1 / (sqrt(Dz) * sqrt(Dz));
    for (int j = threadIdx.x; j < d.nt; j += blockDim.x) {
      res_x[off + j] = (float)(cx * (double)(0.0f - obs_x[off + j]));
      res_z[off + j] = (float)(cz * (double)(0.0f - obs_z[off + j]));
    }
    if (threadIdx.x == 0) mis_terms[(long long)s * d.max_ntr + tr] = 0.0;
  } else {
    const double cx = 1 / (sqrt(dx) * sqrt(Dx)), cz = 1 / (sqrt(dz) * sqrt(Dz));
    const double ax = dDx / dx, az = dDz / dz;
    for (int j = threadIdx.x; j < d.nt; j += blockDim.x) {
      res_x[off + j] = (float)(cx * (ax * (double)syn_x[off + j] - (double)obs_x[off + j]));
      res_z[off + j] = (float)(cz * (az * (double)syn_z[off + j] - (double)obs_z[off + j]));
    }
    if (threadIdx.x == 0)
      mis_terms[(long long)s * d.max_ntr + tr] =
          (double)(1.0f / (float)(2 * shots[s].ntr)) *
          (dDx / (sqrt(dx) * sqrt(Dx)) + dDz / (sqrt(dz) * sqrt(Dz)));
  }
}

}  // namespace ds2d
