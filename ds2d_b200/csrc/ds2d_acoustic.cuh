// Acoustic Born operator pair for CG-LSRTM on sm_100a.
//
// The acoustic scheme is the reference's elastic one with mu = 0 (txx = tzz = s, txz = 0;
// born.cu:215-349 with miu = 0) and its Born source is add_born_source with mu = 0
// (born.cu:394-400): e = -2 lam m (Dx- vx / dx + Dz- vz / dz) on the interior, applied as a
// transient read overlay of the scattered stress.  L m records the scattered vz, vx after every
// step; L^T is its exact discrete transpose (no reference counterpart: the reference's adjoint is
// not the transpose of its Born modelling and its CG helpers, main.cpp:1224-1320, are unused).
// With the random band (no damping) the background field is rebuilt by exact time reversal of the
// whole grid (source included).  With a PML the update is the reference's split form with mu = 0
// (vx damped in x only, vz in z only, s = s_x + s_z split in the PML cells, born.cu:215-349), L^T
// is the exact transpose of that damped scheme, and the background is rebuilt backward on the
// interior from boundary strips of vx, vz saved during a forward replay (the reference's
// reconstruction, FD2DGPU.cu:3674-3731, 4769-4772), in FP32, FP16 or BF16.
#pragma once
#include "ds2d_kernels.cuh"

namespace ds2d {

struct AcArgs {
  Dims d;
  const ShotDev *shots;
  Par p;
  float *vx, *vz, *s;      // state updated in place
  float *sx, *sz;          // split stress of the PML cells (null without a PML)
  int interior;            // update only the interior [pml, n - pml)^2 (reconstruction)
  const float *e;          // additive stress overlay (Born source) or null
  const float *wavelet;
  int it;
  int src_on;              // explosive source overlay on s
  float dir;               // +1 forward, -1 exact reversal
  const int *rmap;
  float *rec_vz, *rec_vx;  // [slot][max_ntr][nt]
  int rec_on;
};

__device__ __forceinline__ bool in_upd(const Dims &d, int ix, int iz) {
  return ix >= d.nop && ix < d.nxp - d.nop && iz >= d.nop && iz < d.nzp - d.nop;
}
__device__ __forceinline__ bool in_int(const Dims &d, int ix, int iz) {
  return ix >= d.pml && ix < d.nxp - d.pml && iz >= d.pml && iz < d.nzp - d.pml;
}
// Damping factors of a PML cell: d1 = 1 - dt d / 2 and 1 / d2 = 1 / (1 + dt d / 2).
struct AcDamp {
  float d1x, r2x, d1z, r2z;
};
__device__ __forceinline__ AcDamp ac_damp(const Dims &d, const Par &p, long long k) {
  const float hx = p.dampx[k] * d.dt * 0.5f, hz = p.dampz[k] * d.dt * 0.5f;
  return AcDamp{1.0f - hx, __frcp_rn(1.0f + hx), 1.0f - hz, __frcp_rn(1.0f + hz)};
}

// v += dir * b dt/d * D+(s + e + source)
__global__ void __launch_bounds__(256) k_ac_vel(AcArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp || !in_upd(d, ix, iz)) return;
  if (a.interior && !in_int(d, ix, iz)) return;
  const int ld = d.ld;
  const long long base = d.slot * s, k = base + (long long)ix * ld + iz;
  long long ksrc = -1;
  float sval = 0.f;
  if (a.src_on) {
    const ShotDev sh = a.shots[s];
    ksrc = base + (long long)sh.isx * ld + sh.isz;
    sval = a.wavelet[a.it];
  }
  const float *S = a.s, *E = a.e;
  auto rd = [&](long long q) {
    float v = __ldg(S + q);
    if (E) v += __ldg(E + q);
    if (q == ksrc) v += sval;
    return v;
  };
  const float ax = stencil4([&](int i) { return rd(k + (long long)i * ld) - rd(k + (long long)(1 - i) * ld); });
  const float az = stencil4([&](int i) { return rd(k + i) - rd(k - i + 1); });
  const float bb = a.p.b[k];
  float vx, vz;
  if (a.sx && pml_cell(d, ix, iz)) {  // damped (forward only): (d1 v + b dt/d D+ S) / d2
    const AcDamp q = ac_damp(d, a.p, k);
    vx = fmaf(q.d1x, a.vx[k], bb * (d.dt / d.dx) * ax) * q.r2x;
    vz = fmaf(q.d1z, a.vz[k], bb * (d.dt / d.dz) * az) * q.r2z;
  } else {
    vx = a.vx[k] + a.dir * (bb * (d.dt / d.dx)) * ax;
    vz = a.vz[k] + a.dir * (bb * (d.dt / d.dz)) * az;
  }
  a.vx[k] = vx;
  a.vz[k] = vz;
  if (a.rec_on && iz == a.shots[s].igz) {
    const int tr = a.rmap[(long long)s * d.nxp_max + ix];
    if (tr >= 0) {
      const long long r = ((long long)s * d.max_ntr + tr) * d.nt + a.it;
      a.rec_vz[r] = vz;
      a.rec_vx[r] = vx;
    }
  }
}

// s += dir * lam (dt/dx Dx- vx + dt/dz Dz- vz)
__global__ void __launch_bounds__(256) k_ac_str(AcArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp || !in_upd(d, ix, iz)) return;
  if (a.interior && !in_int(d, ix, iz)) return;
  const int ld = d.ld;
  const long long k = d.slot * s + (long long)ix * ld + iz;
  const float *VX = a.vx, *VZ = a.vz;
  const float sx = stencil4([&](int i) { return __ldg(VX + k + (long long)(i - 1) * ld) - __ldg(VX + k - (long long)i * ld); });
  const float sz = stencil4([&](int i) { return __ldg(VZ + k + i - 1) - __ldg(VZ + k - i); });
  if (a.sx && pml_cell(d, ix, iz)) {  // split and damped (forward only)
    const AcDamp q = ac_damp(d, a.p, k);
    const float lam = a.p.lam[k];
    const float nx = fmaf(q.d1x, a.sx[k], lam * (d.dt / d.dx) * sx) * q.r2x;
    const float nz = fmaf(q.d1z, a.sz[k], lam * (d.dt / d.dz) * sz) * q.r2z;
    a.sx[k] = nx;
    a.sz[k] = nz;
    a.s[k] = nx + nz;
    return;
  }
  a.s[k] = a.s[k] + a.dir * a.p.lam[k] * ((d.dt / d.dx) * sx + (d.dt / d.dz) * sz);
}

// Interior reconstruction of the background with a PML: the band of vx, vz around the PML edge
// (the 2-field strips of FD2DGPU.cu:3674-3731) restored from the step's saved strips.
struct AcStripArgs {
  Dims d;
  const ShotDev *shots;
  float *vx, *vz;
  Strips st;
  int it;
};
__global__ void __launch_bounds__(256) k_ac_strip_load(AcStripArgs a) {
  const int s = blockIdx.z, comp = blockIdx.y;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int bo = blockIdx.x * 256 + threadIdx.x;
  if (bo >= d.lb) return;
  int ix, iz;
  band_cell(d, bo, ix, iz);
  (comp ? a.vz : a.vx)[d.slot * s + (long long)ix * d.ld + iz] = strip_get(a.st, d, s, a.it, comp, bo);
}

// ---- background checkpoints of the PML L^T --------------------------------------------------
// With option "ac_ckpt" = K the forward replay of L^T keeps, instead of every step's boundary
// strips, a snapshot of the whole background state (vx, vz, s and the PML split stress sx, sz)
// every K steps, stored in the context's strip precision with one FP32 scale per field, shot and
// snapshot (scale = max|f| / 2^15 as for the strips, so FP16 stays in range; BF16 takes the same
// scale).  The reverse pass then works segment by segment from the last: decode the segment's
// snapshot, replay its steps saving their strips (a K-step strip buffer), reverse through them.
constexpr int kCkptFields = 5;
struct CkptArgs {
  long long slot;          // floats per shot slot
  const float *f[kCkptFields];
  float *fw[kCkptFields];  // the same arrays, written by the decode
  void *data;              // this snapshot: [kCkptFields][B][slot] elements
  float *scale;            // this snapshot: [kCkptFields][B]
  unsigned *amax;          // scratch [kCkptFields][B]: max |f| as float bits (non-negative)
  int prec, B;
};

__global__ void __launch_bounds__(256) k_ckpt_absmax(CkptArgs a) {
  const int s = blockIdx.z, f = blockIdx.y;
  const float *src = a.f[f] + a.slot * s;
  float m = 0.f;
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < a.slot;
       i += (long long)gridDim.x * 256)
    m = fmaxf(m, fabsf(src[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  // non-negative floats order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(&a.amax[f * a.B + s], __float_as_uint(m));
}

__device__ __forceinline__ float ckpt_scale(unsigned bits) {
  const float m = __uint_as_float(bits);
  return m > 0.f ? fmaxf(m * (1.0f / 32768.0f), 1.17549435e-38f) : 1.0f;
}

__global__ void __launch_bounds__(256) k_ckpt_encode(CkptArgs a) {
  const int s = blockIdx.z, f = blockIdx.y;
  const float *src = a.f[f] + a.slot * s;
  const long long base = ((long long)f * a.B + s) * a.slot;
  const float sc = a.prec == 0 ? 1.0f : ckpt_scale(a.amax[f * a.B + s]);
  if (a.prec != 0 && blockIdx.x == 0 && threadIdx.x == 0) a.scale[f * a.B + s] = sc;
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < a.slot;
       i += (long long)gridDim.x * 256) {
    const float v = src[i];
    if (a.prec == 0) ((float *)a.data)[base + i] = v;
    else if (a.prec == 1) ((__half *)a.data)[base + i] = __float2half_rn(v / sc);
    else ((__nv_bfloat16 *)a.data)[base + i] = __float2bfloat16_rn(v / sc);
  }
}

__global__ void __launch_bounds__(256) k_ckpt_decode(CkptArgs a) {
  const int s = blockIdx.z, f = blockIdx.y;
  float *dst = a.fw[f] + a.slot * s;
  const long long base = ((long long)f * a.B + s) * a.slot;
  const float sc = a.prec == 0 ? 1.0f : a.scale[f * a.B + s];
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < a.slot;
       i += (long long)gridDim.x * 256) {
    if (a.prec == 0) dst[i] = ((const float *)a.data)[base + i];
    else if (a.prec == 1) dst[i] = __half2float(((const __half *)a.data)[base + i]) * sc;
    else dst[i] = __bfloat162float(((const __nv_bfloat16 *)a.data)[base + i]) * sc;
  }
}

// e = -2 lam m (Dx- vx / dx + Dz- vz / dz) on the interior (m = the windowed model in p.dmp).
__global__ void __launch_bounds__(256) k_ac_born(Dims d0, const ShotDev *shots, Par p,
                                                 const float *vx, const float *vz, float *e) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(d0, shots[s]);
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp || !in_int(d, ix, iz)) return;
  const int ld = d.ld;
  const long long k = d.slot * s + (long long)ix * ld + iz;
  const float sx = stencil4([&](int i) { return __ldg(vx + k + (long long)(i - 1) * ld) - __ldg(vx + k - (long long)i * ld); });
  const float sz = stencil4([&](int i) { return __ldg(vz + k + i - 1) - __ldg(vz + k - i); });
  // reciprocal multiplies (same form as the transpose in k_ac_adj_s); a division would take its
  // slow path for the tiny amplitudes ahead of a wavefront
  e[k] = -2.0f * p.lam[k] * p.dmp[k] * (sx * (1.0f / d.dx) + sz * (1.0f / d.dz));
}

// Adjoint, part 1 (transpose of the stress stage) with the transpose of the recording:
// y_v += r (receivers), yx -= dt/dx Dx+(lam ys), yz -= dt/dz Dz+(lam ys).
struct AcAdjArgs {
  Dims d;
  const ShotDev *shots;
  Par p;
  float *yx, *yz, *ys;
  const int *rmap;
  const float *res_vz, *res_vx;  // [slot][max_ntr][nt]
  int it;
  const float *bvx, *bvz;        // background velocities at this step (gradient)
  float *grad;                   // [slot][wnx][ild] (wnx_max stride)
  float *ysx, *ysz;              // adjoint of the split stress of the PML cells (null: none)
};

__global__ void __launch_bounds__(256) k_ac_adj_v(AcAdjArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp || !in_upd(d, ix, iz)) return;
  const int ld = d.ld;
  const long long k = d.slot * s + (long long)ix * ld + iz;
  const float *lam = a.p.lam, *ys = a.ys;
  float tx, tz;
  float yx = a.yx[k], yz = a.yz[k];
  if (a.ysx) {
    // With a PML: the stress stage's transpose reads y_sx / d2x (x part) and y_sz / d2z (z part)
    // on split cells, and the velocity decay d1/d2 of the previous reverse step's velocity-stage
    // transpose is applied here, where y_v is read only at its own cell.
    const float *ysx = a.ysx, *ysz = a.ysz, *dpx = a.p.dampx, *dpz = a.p.dampz;
    auto wx = [&](long long q, int qx, int qz) {
      if (!pml_cell(d, qx, qz)) return __ldg(lam + q) * __ldg(ys + q);
      return __ldg(lam + q) * __ldg(ysx + q) * __frcp_rn(1.0f + __ldg(dpx + q) * d.dt * 0.5f);
    };
    auto wz = [&](long long q, int qx, int qz) {
      if (!pml_cell(d, qx, qz)) return __ldg(lam + q) * __ldg(ys + q);
      return __ldg(lam + q) * __ldg(ysz + q) * __frcp_rn(1.0f + __ldg(dpz + q) * d.dt * 0.5f);
    };
    tx = stencil4([&](int i) { return wx(k + (long long)i * ld, ix + i, iz) - wx(k + (long long)(1 - i) * ld, ix + 1 - i, iz); });
    tz = stencil4([&](int i) { return wz(k + i, ix, iz + i) - wz(k - i + 1, ix, iz - i + 1); });
    if (pml_cell(d, ix, iz)) {
      const AcDamp q = ac_damp(d, a.p, k);
      yx *= q.d1x * q.r2x;
      yz *= q.d1z * q.r2z;
    }
  } else {
    auto w = [&](long long q) { return __ldg(lam + q) * __ldg(ys + q); };
    tx = stencil4([&](int i) { return w(k + (long long)i * ld) - w(k + (long long)(1 - i) * ld); });
    tz = stencil4([&](int i) { return w(k + i) - w(k - i + 1); });
  }
  if (iz == a.shots[s].igz) {
    const int tr = a.rmap[(long long)s * d.nxp_max + ix];
    if (tr >= 0) {
      const long long r = ((long long)s * d.max_ntr + tr) * d.nt + a.it;
      yz += a.res_vz[r];
      yx += a.res_vx[r];
    }
  }
  a.yx[k] = yx - (d.dt / d.dx) * tx;
  a.yz[k] = yz - (d.dt / d.dz) * tz;
}

// Adjoint, part 2 (transpose of the velocity stage): gs = -Dx-(b dt/dx yx) - Dz-(b dt/dz yz),
// ys += gs, and the transpose of the Born source: grad += -2 lam (Dx- vx/dx + Dz- vz/dz) gs.
__global__ void __launch_bounds__(256) k_ac_adj_s(AcAdjArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * 32 + threadIdx.x, ix = blockIdx.y * 8 + threadIdx.y;
  if (ix >= d.nxp || iz >= d.nzp || !in_upd(d, ix, iz)) return;
  const int ld = d.ld;
  const long long k = d.slot * s + (long long)ix * ld + iz;
  const float *b = a.p.b, *yx = a.yx, *yz = a.yz;
  const float cx = d.dt / d.dx, cz = d.dt / d.dz;
  float gx, gz;
  if (a.ysx) {  // velocity-stage transpose with the PML's 1 / d2 on split cells
    const float *dpx = a.p.dampx, *dpz = a.p.dampz;
    auto ux = [&](long long q, int qx, int qz) {
      const float u = __ldg(b + q) * cx * __ldg(yx + q);
      return pml_cell(d, qx, qz) ? u * __frcp_rn(1.0f + __ldg(dpx + q) * d.dt * 0.5f) : u;
    };
    auto uz = [&](long long q, int qx, int qz) {
      const float u = __ldg(b + q) * cz * __ldg(yz + q);
      return pml_cell(d, qx, qz) ? u * __frcp_rn(1.0f + __ldg(dpz + q) * d.dt * 0.5f) : u;
    };
    gx = stencil4([&](int i) { return ux(k + (long long)(i - 1) * ld, ix + i - 1, iz) - ux(k - (long long)i * ld, ix - i, iz); });
    gz = stencil4([&](int i) { return uz(k + i - 1, ix, iz + i - 1) - uz(k - i, ix, iz - i); });
  } else {
    auto ux = [&](long long q) { return __ldg(b + q) * cx * __ldg(yx + q); };
    auto uz = [&](long long q) { return __ldg(b + q) * cz * __ldg(yz + q); };
    gx = stencil4([&](int i) { return ux(k + (long long)(i - 1) * ld) - ux(k - (long long)i * ld); });
    gz = stencil4([&](int i) { return uz(k + i - 1) - uz(k - i); });
  }
  const float gs = -gx - gz;
  if (a.ysx && pml_cell(d, ix, iz)) {  // S = s_x + s_z: y_S reaches both split parts
    const AcDamp q = ac_damp(d, a.p, k);
    a.ysx[k] = fmaf(q.d1x * q.r2x, a.ysx[k], gs);
    a.ysz[k] = fmaf(q.d1z * q.r2z, a.ysz[k], gs);
  } else {
    a.ys[k] = a.ys[k] + gs;
  }
  if (in_int(d, ix, iz)) {
    const float *VX = a.bvx, *VZ = a.bvz;
    const float sx = stencil4([&](int i) { return __ldg(VX + k + (long long)(i - 1) * ld) - __ldg(VX + k - (long long)i * ld); });
    const float sz = stencil4([&](int i) { return __ldg(VZ + k + i - 1) - __ldg(VZ + k - i); });
    const long long o = ((long long)s * d.wnx_max + (ix - d.pml)) * d.ild + iz;
    a.grad[o] += -2.0f * a.p.lam[k] * (sx * (1.0f / d.dx) + sz * (1.0f / d.dz)) * gs;
  }
}

// FP64 inner product <a, b> over n floats: per-block partial sums (scratch), then one block adds
// the partials in a fixed order (deterministic).  Warp shuffles for the in-block reduction.
constexpr int kDotBlocks = 592;  // 4 x 148 SMs
constexpr int kDotThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kDotThreads) k_dot_partial(const float *a, const float *b,
                                                             long long n, double *partial) {
  __shared__ double sh[kDotThreads / 32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * kDotThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kDotThreads)
    acc = fma((double)a[i], (double)b[i], acc);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < kDotThreads / 32 ? sh[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(32) k_dot_final(const double *partial, int np, double *out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += 32) v += partial[i];
  v = warp_sum(v);
  if (threadIdx.x == 0) *out = v;
}

// y = alpha * x + y and y = x + beta * y on float vectors with FP64 scalars (CG updates).
__global__ void k_axpy(long long n, double alpha, const float *x, float *y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = (float)((double)y[i] + alpha * (double)x[i]);
}
__global__ void k_xpby(long long n, const float *x, double beta, float *y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = (float)((double)x[i] + beta * (double)y[i]);
}

}  // namespace ds2d
