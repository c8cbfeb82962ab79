// Fused single-pass elastic time step for sm_100a: one launch advances the velocities AND the
// stresses of every resident shot by one step (reference update_vx, update_vz, update_txx_tzz,
// update_txz, born.cu:215-349, four launches per step there).
//
// Shape: each CTA owns a z-strip of tz <= 112 output columns (128 threads: one thread per column
// of the strip plus an 8-column halo on each side) and marches along x over xr output rows.  At
// row step r it
//   1. loads the old stresses of row r (coalesced rows of 128 floats),
//   2. computes the new velocities of row r-4 for the strip plus a 4-column halo,
//   3. computes the new stresses of row r-8 for the strip.
// The 8-tap x-derivatives come from per-thread register windows of the last 9 rows; the z-taps of
// the current row come from one shared-memory row per field.  State ping-pongs between two
// buffers (a -> b), so neighbouring CTAs never see a half-updated halo.  DRAM traffic per cell is
// the algorithmic 52 bytes (5 fields read + written, b, lam, mu read); halo re-reads hit L2.
//
// Injections keep the reference's transient semantics (see ds2d_kernels.cuh): the explosive
// source is added to the stress values that enter the stencil windows; the one cell that carries
// it reloads its own old state from memory for the stress update.
#pragma once
#include "ds2d_kernels.cuh"

namespace ds2d {

// Row steps per iteration of the ring kernels' x-march (compile-time tuning knob).  Two steps
// per iteration let the compiler rename half of the window shifts away (60-shot RTM at
// 1201x401 on a B200: forward 669 -> 643 us, backward 1596 -> 1572 us per launch); three or
// four spill registers or overflow the instruction cache.
#ifndef DS2D_RING_UNROLL_FWD
#define DS2D_RING_UNROLL_FWD 2
#endif
#ifndef DS2D_RING_UNROLL_BWD
#define DS2D_RING_UNROLL_BWD 2
#endif
constexpr int kRingUnrollFwd = DS2D_RING_UNROLL_FWD;
constexpr int kRingUnrollBwd = DS2D_RING_UNROLL_BWD;

constexpr int kFB = 128;        // threads per CTA
constexpr int kFTZ = kFB - 16;  // max output columns of one strip

struct FwdFusedArgs {
  Dims d;
  Wave a, b;  // state at t-1 (read) and t (written)
  Par p;
  const ShotDev *shots;
  const float *wavelet;
  int it;
  int tz, xr;  // output columns per strip, output rows per CTA
  const int *rmap;
  float *rec_vz, *rec_vx;
  int rec_on;
  // Born modelling sets (ring kernel modes 1-3): read overlay of the stresses (the Born source
  // of the previous set, added to the stencil values only) and the Born source written from the
  // new velocities for the next set.
  const float *ovi_txx, *ovi_tzz, *ovi_txz;
  float *ovo_txx, *ovo_tzz, *ovo_txz;
  int *err;  // device error word of the pair kernels' bounded waits (null: none)
};

template <int N>
__device__ __forceinline__ void push(float (&w)[N], float v) {
#pragma unroll
  for (int i = 0; i < N - 1; i++) w[i] = w[i + 1];
  w[N - 1] = v;
}

// Window of 9 rows, w[8] = newest row q0; row q sits at index 8 - (q0 - q).
// Dx+ at row q0 - 4 (taps q+i, q-i+1) and Dx- at row q0 - 4 (taps q+i-1, q-i).
__device__ __forceinline__ float dxp_mid(const float (&w)[9]) {
  return stencil4([&](int i) { return w[4 + i] - w[5 - i]; });
}
__device__ __forceinline__ float dxm_mid(const float (&w)[9]) {
  return stencil4([&](int i) { return w[3 + i] - w[4 - i]; });
}

template <bool kPML>
__global__ void __launch_bounds__(kFB) k_fwd_fused(FwdFusedArgs a) {
  __shared__ float s_txz[kFB], s_tzz[kFB], s_vx[kFB], s_vz[kFB];
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int z = blockIdx.x * a.tz - 8 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const long long base = d.slot * s;
  const int ld = d.ld;
  const bool zin = z >= 0 && z < d.nzp;
  const bool zupd = z >= d.nop && z < d.nzp - d.nop;
  const bool vcol = t >= 4 && t < a.tz + 12 && zupd;
  const bool scol = t >= 8 && t < a.tz + 8 && zupd;
  const ShotDev sh = a.shots[s];
  const float sval = a.wavelet[a.it];
  const bool src_col = z == sh.isz;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float *Atxx = a.a.txx, *Atzz = a.a.tzz, *Atxz = a.a.txz;

  float w_txx[9], w_tzz[9], w_txz[9], w_vx[9], w_vz[9];
#pragma unroll
  for (int i = 0; i < 9; i++) w_txx[i] = w_tzz[i] = w_txz[i] = w_vx[i] = w_vz[i] = 0.f;

  float n_txx = 0.f, n_tzz = 0.f, n_txz = 0.f;
  auto load_s = [&](int r) {
    n_txx = n_tzz = n_txz = 0.f;
    if (r >= 0 && r < d.nxp && zin) {
      const long long k = base + (long long)r * ld + z;
      n_txx = __ldg(Atxx + k);
      n_tzz = __ldg(Atzz + k);
      n_txz = __ldg(Atxz + k);
      if (src_col && r == sh.isx) {  // FD2DGPU.cu:2039-2049 (transient)
        n_txx += sval;
        n_tzz += sval;
      }
    }
  };
  load_s(x0 - 8);
  for (int r = x0 - 8; r < x1 + 8; r++) {
    push(w_txx, n_txx);
    push(w_tzz, n_tzz);
    push(w_txz, n_txz);
    load_s(r + 1);
    // ---- velocities of row rv = r - 4 --------------------------------------------------
    const int rv = r - 4;
    s_txz[t] = w_txz[4];
    s_tzz[t] = w_tzz[4];
    __syncthreads();
    float vxn = 0.f, vzn = 0.f;
    if (vcol && r >= x0 && rv >= d.nop && rv < d.nxp - d.nop) {
      const long long k = base + (long long)rv * ld + z;
      const float ax = dxp_mid(w_txx);
      const float fx = dxm_mid(w_txz);
      const float bz = stencil4([&](int i) { return s_txz[t + i - 1] - s_txz[t - i]; });
      const float ez = stencil4([&](int i) { return s_tzz[t + i] - s_tzz[t - i + 1]; });
      const float bb = __ldg(a.p.b + k);
      const float cbx = bb * dtdx, cbz = bb * dtdz;
      const float ux_x = cbx * ax, ux_z = cbz * bz, uz_x = cbx * fx, uz_z = cbz * ez;
      const bool own = rv >= x0 && rv < x1 && t >= 8 && t < a.tz + 8;
      if (kPML && pml_cell(d, rv, z)) {
        const float ddx = a.p.dampx[k] * d.dt * 0.5f, ddz = a.p.dampz[k] * d.dt * 0.5f;
        const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
        const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
        const float vxx = fmaf(d1, a.a.vx_x[k], ux_x) * i2;
        const float vxz = fmaf(d3, a.a.vx_z[k], ux_z) * i4;
        const float vzx = fmaf(d1, a.a.vz_x[k], uz_x) * i2;
        const float vzz = fmaf(d3, a.a.vz_z[k], uz_z) * i4;
        if (own) {
          a.b.vx_x[k] = vxx; a.b.vx_z[k] = vxz; a.b.vz_x[k] = vzx; a.b.vz_z[k] = vzz;
        }
        vxn = vxx + vxz;
        vzn = vzx + vzz;
      } else {
        vxn = __ldg(a.a.vx + k) + (ux_x + ux_z);
        vzn = __ldg(a.a.vz + k) + (uz_x + uz_z);
      }
      if (own) {
        a.b.vx[k] = vxn;
        a.b.vz[k] = vzn;
        if (a.rec_on && z == sh.igz) {
          const int tr = a.rmap[(long long)s * d.nxp_max + rv];
          if (tr >= 0) {
            const long long q = ((long long)s * d.max_ntr + tr) * d.nt + a.it;
            a.rec_vz[q] = vzn;
            a.rec_vx[q] = vxn;
          }
        }
      }
    }
    push(w_vx, vxn);
    push(w_vz, vzn);
    // ---- stresses of row rs = r - 8 -----------------------------------------------------
    const int rs = r - 8;
    s_vx[t] = w_vx[4];
    s_vz[t] = w_vz[4];
    __syncthreads();
    if (scol && rs >= x0 && rs < x1 && rs >= d.nop && rs < d.nxp - d.nop) {
      const long long k = base + (long long)rs * ld + z;
      const float sa = dxm_mid(w_vx);
      const float sf = dxp_mid(w_vz);
      const float sb = stencil4([&](int i) { return s_vz[t + i - 1] - s_vz[t - i]; });
      const float se = stencil4([&](int i) { return s_vx[t + i] - s_vx[t - i + 1]; });
      const float lam = __ldg(a.p.lam + k), mu = __ldg(a.p.mu + k);
      const float l2m = lam + 2.0f * mu;
      const float xx_x = l2m * dtdx * sa, xx_z = lam * dtdz * sb;
      const float zz_x = lam * dtdx * sa, zz_z = l2m * dtdz * sb;
      const float xz_x = dtdx * mu * sf, xz_z = dtdz * mu * se;
      if (kPML && pml_cell(d, rs, z)) {
        const float ddx = a.p.dampx[k] * d.dt * 0.5f, ddz = a.p.dampz[k] * d.dt * 0.5f;
        const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
        const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
        const float a1 = fmaf(d1, a.a.txx_x[k], xx_x) * i2;
        const float a2 = fmaf(d3, a.a.txx_z[k], xx_z) * i4;
        const float b1 = fmaf(d1, a.a.tzz_x[k], zz_x) * i2;
        const float b2 = fmaf(d3, a.a.tzz_z[k], zz_z) * i4;
        const float c1 = fmaf(d1, a.a.txz_x[k], xz_x) * i2;
        const float c2 = fmaf(d3, a.a.txz_z[k], xz_z) * i4;
        a.b.txx_x[k] = a1; a.b.txx_z[k] = a2;
        a.b.tzz_x[k] = b1; a.b.tzz_z[k] = b2;
        a.b.txz_x[k] = c1; a.b.txz_z[k] = c2;
        a.b.txx[k] = a1 + a2;
        a.b.tzz[k] = b1 + b2;
        a.b.txz[k] = c1 + c2;
      } else {
        float oxx = w_txx[0], ozz = w_tzz[0];
        if (src_col && rs == sh.isx) {  // the injected cell: state without the source
          oxx = __ldg(Atxx + k);
          ozz = __ldg(Atzz + k);
        }
        a.b.txx[k] = oxx + (xx_x + xx_z);
        a.b.tzz[k] = ozz + (zz_x + zz_z);
        a.b.txz[k] = w_txz[0] + (xz_x + xz_z);
      }
    }
    // No third barrier: the next step writes s_txz / s_tzz only after every thread has passed
    // this step's second barrier (V stage done) and s_vx / s_vz only after its first barrier.
  }
}

// ---------------------------------------------------------------------------------------------
// Asynchronous row prefetch for the row-marching kernels.  Every per-row operand of a thread's
// column is copied global -> shared with cp.async (LDGSTS) kD - 1 row steps before it is used
// (kD = ring depth, a power of two, a template parameter of the kernels).  Ring slot q (q mod kD)
// holds everything row step q consumes: the stage-1 stencil inputs of row q, the stage-1
// own-cell operands of row q-4 and the stage-2 operands of row q-8, issued together as one commit
// group at step q - (kD - 1), into the slot row step q - 1 has just finished with.  A thread only
// ever reads ring entries it copied itself, so cp.async.wait_group alone orders them (no
// barrier), and kD slots suffice however long the lags are.  The prefetch distance needed is a
// few microseconds of DRAM latency; one row step of a CTA takes about as long, so a shallow ring
// (kD = 4) hides it while leaving shared memory for more resident CTAs.

__device__ __forceinline__ void cp_async4(float *smem, const float *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Forward step fed by the ring: same arithmetic as k_fwd_fused.  Fields of ring slot q:
// 0 txx, 1 tzz, 2 txz of row q (stencil windows); 3 vx, 4 vz, 5 b of row q-4 (velocity stage);
// 6 lam, 7 mu of row q-8 (stress stage).  With PML the split operands of a PML cell come through
// the ring too (a PML cell does not read its own vx, vz, so slots 3-4 carry vx_x, vx_z):
// 8 vz_x, 9 vz_z, 10 dampx, 11 dampz of row q-4; 12 dampx, 13 dampz, 14 txx_x, 15 txx_z,
// 16 tzz_x, 17 tzz_z, 18 txz_x, 19 txz_z of row q-8.
//
// Modes (the reference's born_modeling sequence, FD2DGPU.cu:1817-1862 with add_born_source,
// born.cu:351-405, after each set):
//   0  background step with the explosive source (modelling, RTM);
//   1  background step that also writes the Born source of its new velocities (interior cells)
//      into ovo_* for the first-order scattered set;
//   2  scattered step without source, ovi_* added to the stress stencil values, Born source of
//      its own new velocities written into ovo_* for the second-order set;
//   3  scattered step with the ovi_* overlay only.
// An overlay mode reads each cell's own stresses for the stress update from extra ring fields
// (the windows hold stress + overlay), and a Born-source mode reads dmp, dms:
//   NF0 + 0..2 ovi txx, tzz, txz of row q; NF0 + 3..5 txx, tzz, txz of row q-8 (overlay modes);
//   then dmp, dms of row q-8 (Born-source modes), NF0 = fwd_ring_fields(kPML).
constexpr int kFwdRingFields = 8;
constexpr int kFwdRingFieldsPml = 20;
__host__ __device__ constexpr int fwd_ring_fields(bool pml) {
  return pml ? kFwdRingFieldsPml : kFwdRingFields;
}
__host__ __device__ constexpr int fwd_ring_fields(bool pml, int mode) {
  return fwd_ring_fields(pml) + (mode >= 2 ? 6 : 0) + (mode == 1 || mode == 2 ? 2 : 0);
}

template <bool kPML, int kD, int kMinB, int kT = kFB, int kMode = 0>
__global__ void __launch_bounds__(kT, kMinB) k_fwd_ring(FwdFusedArgs a) {
  static_assert(kD >= 2 && kD <= 8 && (kD & (kD - 1)) == 0, "ring depth: 2, 4 or 8");
  constexpr bool kOvIn = kMode >= 2, kBornOut = kMode == 1 || kMode == 2, kSrc = kMode < 2;
  constexpr int NF0 = fwd_ring_fields(kPML);
  constexpr int NF = fwd_ring_fields(kPML, kMode);
  constexpr int FOV = NF0, FOWN = NF0 + 3, FBORN = NF0 + (kOvIn ? 6 : 0);
  extern __shared__ float ring[];  // [kD][NF][kT]
  __shared__ float s_txz[kT], s_tzz[kT], s_vx[kT], s_vz[kT];
  __shared__ int s_tr[16];  // receiver column: trace index of velocity row mod 16, 8 rows ahead
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int z = blockIdx.x * a.tz - 8 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const int base = (int)(d.slot * s);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld;
  const bool zin = z >= 0 && z < d.nzp;
  const bool zupd = z >= d.nop && z < d.nzp - d.nop;
  const bool vcol = t >= 4 && t < a.tz + 12 && zupd;
  const bool scol = t >= 8 && t < a.tz + 8 && zupd;
  const ShotDev sh = a.shots[s];
  const float sval = a.wavelet[a.it];
  const bool src_col = kSrc && z == sh.isz;
  const bool rec_col = a.rec_on && z == sh.igz;
  const bool z_int = z >= d.pml && z < d.nzp - d.pml;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  // R(q, f): field f of ring slot q (row q for f < 3, row q-4 for f < 6, row q-8 otherwise)
  auto R = [&](int q, int f) -> float & { return ring[((q & (kD - 1)) * NF + f) * kT + t]; };
  auto issue = [&](int q) {
    const int r0 = q, r4 = q - 4, r8 = q - 8;
    const bool in0 = r0 >= 0 && r0 < d.nxp && zin;
    const bool in4 = r4 >= 0 && r4 < d.nxp && zin;
    const bool in8 = r8 >= 0 && r8 < d.nxp && zin;
    const int o0 = base + r0 * ld + z, o4 = base + r4 * ld + z, o8 = base + r8 * ld + z;
    const bool pml4 = kPML && in4 && pml_cell(d, r4, z);
    const bool pml8 = kPML && in8 && pml_cell(d, r8, z);
    if (in0) {
      cp_async4(&R(q, 0), a.a.txx + o0);
      cp_async4(&R(q, 1), a.a.tzz + o0);
      cp_async4(&R(q, 2), a.a.txz + o0);
    } else {
      R(q, 0) = R(q, 1) = R(q, 2) = 0.f;
    }
    if (in4) {
      cp_async4(&R(q, 3), (pml4 ? a.a.vx_x : a.a.vx) + o4);
      cp_async4(&R(q, 4), (pml4 ? a.a.vx_z : a.a.vz) + o4);
      cp_async4(&R(q, 5), a.p.b + o4);
    } else {
      R(q, 3) = R(q, 4) = R(q, 5) = 0.f;
    }
    if (in8) {
      cp_async4(&R(q, 6), a.p.lam + o8);
      cp_async4(&R(q, 7), a.p.mu + o8);
    } else {
      R(q, 6) = R(q, 7) = 0.f;
    }
    if (kPML && pml4) {
      cp_async4(&R(q, 8), a.a.vz_x + o4);
      cp_async4(&R(q, 9), a.a.vz_z + o4);
      cp_async4(&R(q, 10), a.p.dampx + o4);
      cp_async4(&R(q, 11), a.p.dampz + o4);
    }
    if (kPML && pml8) {
      cp_async4(&R(q, 12), a.p.dampx + o8);
      cp_async4(&R(q, 13), a.p.dampz + o8);
      cp_async4(&R(q, 14), a.a.txx_x + o8);
      cp_async4(&R(q, 15), a.a.txx_z + o8);
      cp_async4(&R(q, 16), a.a.tzz_x + o8);
      cp_async4(&R(q, 17), a.a.tzz_z + o8);
      cp_async4(&R(q, 18), a.a.txz_x + o8);
      cp_async4(&R(q, 19), a.a.txz_z + o8);
    }
    if (kOvIn) {
      if (in0) {
        cp_async4(&R(q, FOV), a.ovi_txx + o0);
        cp_async4(&R(q, FOV + 1), a.ovi_tzz + o0);
        cp_async4(&R(q, FOV + 2), a.ovi_txz + o0);
      } else {
        R(q, FOV) = R(q, FOV + 1) = R(q, FOV + 2) = 0.f;
      }
      if (in8 && !pml8) {
        cp_async4(&R(q, FOWN), a.a.txx + o8);
        cp_async4(&R(q, FOWN + 1), a.a.tzz + o8);
        cp_async4(&R(q, FOWN + 2), a.a.txz + o8);
      }
    }
    if (kBornOut && in8 && r8 >= d.pml && r8 < d.nxp - d.pml && z_int) {
      cp_async4(&R(q, FBORN), a.p.dmp + o8);
      cp_async4(&R(q, FBORN + 1), a.p.dms + o8);
    }
    cp_async_commit();
  };

  float w_txx[9], w_tzz[9], w_txz[9], w_vx[9], w_vz[9];
#pragma unroll
  for (int i = 0; i < 9; i++) w_txx[i] = w_tzz[i] = w_txz[i] = w_vx[i] = w_vz[i] = 0.f;

#pragma unroll
  for (int j = 0; j < kD - 1; j++) issue(x0 - 8 + j);
#pragma unroll kRingUnrollFwd
  for (int r = x0 - 8; r < x1 + 8; r++) {
    cp_async_wait<kD - 2>();  // row r has landed (this thread's copies)
    if (rec_col) {  // trace index of velocity row r + 4 (read 8 steps on, landed by then)
      const int q = r + 4;
      if (q >= 0 && q < d.nxp)
        cp_async4((float *)&s_tr[q & 15], (const float *)(rmap + q));
      else
        s_tr[q & 15] = -1;
    }
    float n_txx = R(r, 0), n_tzz = R(r, 1), n_txz = R(r, 2);
    if (kOvIn) {  // Born source of the previous set (read overlay, as k_vel)
      n_txx += R(r, FOV);
      n_tzz += R(r, FOV + 1);
      n_txz += R(r, FOV + 2);
    }
    if (src_col && r == sh.isx) {  // FD2DGPU.cu:2039-2049 (transient)
      n_txx += sval;
      n_tzz += sval;
    }
    push(w_txx, n_txx);
    push(w_tzz, n_tzz);
    push(w_txz, n_txz);
    issue(r + kD - 1);  // into the slot of row r - 1 (mod kD), finished last step
    // ---- velocities of row rv = r - 4 --------------------------------------------------
    const int rv = r - 4;
    s_txz[t] = w_txz[4];
    s_tzz[t] = w_tzz[4];
    __syncthreads();
    float vxn = 0.f, vzn = 0.f;
    if (vcol && r >= x0 && rv >= d.nop && rv < d.nxp - d.nop) {
      const int k = base + rv * ld + z;
      const float ax = dxp_mid(w_txx);
      const float fx = dxm_mid(w_txz);
      const float bz = stencil4([&](int i) { return s_txz[t + i - 1] - s_txz[t - i]; });
      const float ez = stencil4([&](int i) { return s_tzz[t + i] - s_tzz[t - i + 1]; });
      const float bb = R(r, 5);
      const float cbx = bb * dtdx, cbz = bb * dtdz;
      const float ux_x = cbx * ax, ux_z = cbz * bz, uz_x = cbx * fx, uz_z = cbz * ez;
      const bool own = rv >= x0 && rv < x1 && t >= 8 && t < a.tz + 8;
      if (kPML && pml_cell(d, rv, z)) {
        const float ddx = R(r, 10) * d.dt * 0.5f, ddz = R(r, 11) * d.dt * 0.5f;
        const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
        const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
        const float vxx = fmaf(d1, R(r, 3), ux_x) * i2;
        const float vxz = fmaf(d3, R(r, 4), ux_z) * i4;
        const float vzx = fmaf(d1, R(r, 8), uz_x) * i2;
        const float vzz = fmaf(d3, R(r, 9), uz_z) * i4;
        if (own) {
          a.b.vx_x[k] = vxx; a.b.vx_z[k] = vxz; a.b.vz_x[k] = vzx; a.b.vz_z[k] = vzz;
        }
        vxn = vxx + vxz;
        vzn = vzx + vzz;
      } else {
        vxn = R(r, 3) + (ux_x + ux_z);
        vzn = R(r, 4) + (uz_x + uz_z);
      }
      if (own) {
        a.b.vx[k] = vxn;
        a.b.vz[k] = vzn;
        if (rec_col) {
          const int tr = s_tr[rv & 15];
          if (tr >= 0) {
            const long long q = ((long long)s * d.max_ntr + tr) * d.nt + a.it;
            a.rec_vz[q] = vzn;
            a.rec_vx[q] = vxn;
          }
        }
      }
    }
    push(w_vx, vxn);
    push(w_vz, vzn);
    // ---- stresses of row rs = r - 8 -----------------------------------------------------
    const int rs = r - 8;
    s_vx[t] = w_vx[4];
    s_vz[t] = w_vz[4];
    __syncthreads();
    if (scol && rs >= x0 && rs < x1 && rs >= d.nop && rs < d.nxp - d.nop) {
      const int k = base + rs * ld + z;
      const float sa = dxm_mid(w_vx);
      const float sf = dxp_mid(w_vz);
      const float sb = stencil4([&](int i) { return s_vz[t + i - 1] - s_vz[t - i]; });
      const float se = stencil4([&](int i) { return s_vx[t + i] - s_vx[t - i + 1]; });
      const float lam = R(r, 6), mu = R(r, 7);
      const float l2m = lam + 2.0f * mu;
      const float xx_x = l2m * dtdx * sa, xx_z = lam * dtdz * sb;
      const float zz_x = lam * dtdx * sa, zz_z = l2m * dtdz * sb;
      const float xz_x = dtdx * mu * sf, xz_z = dtdz * mu * se;
      if (kPML && pml_cell(d, rs, z)) {
        const float ddx = R(r, 12) * d.dt * 0.5f, ddz = R(r, 13) * d.dt * 0.5f;
        const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
        const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
        const float a1 = fmaf(d1, R(r, 14), xx_x) * i2;
        const float a2 = fmaf(d3, R(r, 15), xx_z) * i4;
        const float b1 = fmaf(d1, R(r, 16), zz_x) * i2;
        const float b2 = fmaf(d3, R(r, 17), zz_z) * i4;
        const float c1 = fmaf(d1, R(r, 18), xz_x) * i2;
        const float c2 = fmaf(d3, R(r, 19), xz_z) * i4;
        a.b.txx_x[k] = a1; a.b.txx_z[k] = a2;
        a.b.tzz_x[k] = b1; a.b.tzz_z[k] = b2;
        a.b.txz_x[k] = c1; a.b.txz_z[k] = c2;
        a.b.txx[k] = a1 + a2;
        a.b.tzz[k] = b1 + b2;
        a.b.txz[k] = c1 + c2;
      } else {
        float oxx = w_txx[0], ozz = w_tzz[0], oxz = w_txz[0];
        if (kOvIn) {  // the windows carry the overlay: own state from the ring
          oxx = R(r, FOWN);
          ozz = R(r, FOWN + 1);
          oxz = R(r, FOWN + 2);
        }
        if (src_col && rs == sh.isx) {  // the injected cell: state without the source
          oxx = __ldg(a.a.txx + k);
          ozz = __ldg(a.a.tzz + k);
        }
        a.b.txx[k] = oxx + (xx_x + xx_z);
        a.b.tzz[k] = ozz + (zz_x + zz_z);
        a.b.txz[k] = oxz + (xz_x + xz_z);
      }
      if (kBornOut && rs >= d.pml && rs < d.nxp - d.pml && z_int) {
        // add_born_source of the new velocities (k_born): sa, sb, se, sf are Dx- vx, Dz- vz,
        // Dz+ vx, Dx+ vz of this row
        const float dmp = R(r, FBORN), dms = R(r, FBORN + 1);
        const float P = 2.0f * l2m * (-dmp);
        const float Q = 2.0f * (l2m * (-dmp) - 2.0f * mu * (-dms));
        const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
        a.ovo_txx[k] = P * sa * rdx + Q * sb * rdz;
        a.ovo_tzz[k] = Q * sa * rdx + P * sb * rdz;
        a.ovo_txz[k] = 2.0f * mu * (-dms) * (sf * rdx + se * rdz);
      }
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Fused backward RTM step: interior reconstruction of the source wavefield (stress then
// velocity, direction -1, FD2DGPU.cu:903-1082 via calculateTxz/Txxzz/Vz/Vx at :4769-4772), the
// adjoint step (modulus-free stresses, moduli inside the velocity divergence, FD2DGPU.cu:591-895
// via :4775-4778) with the receiver-side injection (:3306-3322), and the imaging condition
// (doimage_gradient :3245, doimage_illum :3235) in one pass.  Same strip/row-march shape as
// k_fwd_fused; both field sets ping-pong a -> b.  At row step r: stage 1 updates the stresses of
// row r-4 (strip + 4-column halo) and images them, stage 2 updates the velocities of row r-8.
// Strains never leave registers.  Strip values (PML mode) enter only the stage-1 windows; the
// inner-band cells reload their own state, as the reference's split update recomputes them.
struct BwdFusedArgs {
  Dims d;
  Wave ra, rb;   // reconstructed source field: state at t (read), t-1 (written)
  Wave aa, ab;   // adjoint field
  Par p;
  const ShotDev *shots;
  const int *rmap;
  const float *res_vz, *res_vx;  // [slot][max_ntr][nt]
  Strips st;
  int strips_on;
  int it;
  int tz, xr;
  float *img;        // [3][slot][wnx][ild]: pp, ps, illumination
  long long img_plane;
  int *err;          // device error word of the pair kernels' bounded waits (null: none)
};

template <bool kPML>
__global__ void __launch_bounds__(kFB) k_bwd_fused(BwdFusedArgs a) {
  __shared__ float s_bvx[kFB], s_bvz[kFB], s_avx[kFB], s_avz[kFB];          // stage-1 z-taps
  __shared__ float s_btxz[kFB], s_btzz[kFB], s_m[kFB], s_pz[kFB], s_lx[kFB];  // stage-2 z-taps
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int z = blockIdx.x * a.tz - 8 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const long long base = d.slot * s;
  const int ld = d.ld, pml = d.pml;
  const bool zin = z >= 0 && z < d.nzp;
  const bool c1 = t >= 4 && t < a.tz + 12;  // stage-1 columns (strip + halo)
  const bool c2 = t >= 8 && t < a.tz + 8;   // stage-2 / output columns
  const bool z_int = z >= pml && z < d.nzp - pml;
  const bool z_upd = z >= d.nop && z < d.nzp - d.nop;
  const ShotDev sh = a.shots[s];
  const bool rec_col = z == sh.igz;
  const float *res_z = a.res_vz + (long long)s * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)s * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;

  // stage-1 inputs (velocities at t, rows r-8..r)
  float w_bvx[9], w_bvz[9], w_avx[9], w_avz[9];
  // stage-2 inputs (stresses at t-1 and adjoint products, rows r-12..r-4 / r-8..r-4)
  float w_btxx[9], w_btxz[9], w_btzz[5], w_P[9], w_L[9], w_M[9], w_Pz[5], w_Lx[5];
#pragma unroll
  for (int i = 0; i < 9; i++)
    w_bvx[i] = w_bvz[i] = w_avx[i] = w_avz[i] = w_btxx[i] = w_btxz[i] = w_P[i] = w_L[i] = w_M[i] = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) w_btzz[i] = w_Pz[i] = w_Lx[i] = 0.f;

  float n_bvx = 0.f, n_bvz = 0.f, n_avx = 0.f, n_avz = 0.f;
  auto load_v = [&](int r) {
    n_bvx = n_bvz = n_avx = n_avz = 0.f;
    if (r < 0 || r >= d.nxp || !zin) return;
    const long long k = base + (long long)r * ld + z;
    int bo = -1;
    if (a.strips_on) bo = band_offset(d, r, z);
    if (bo >= 0) {
      n_bvx = strip_get(a.st, d, s, a.it, 0, bo);
      n_bvz = strip_get(a.st, d, s, a.it, 1, bo);
    } else {
      n_bvx = __ldg(a.ra.vx + k);
      n_bvz = __ldg(a.ra.vz + k);
    }
    n_avx = __ldg(a.aa.vx + k);
    n_avz = __ldg(a.aa.vz + k);
    if (rec_col) {
      const int tr = rmap[r];
      if (tr >= 0) {
        n_avz += res_z[(long long)tr * d.nt];
        n_avx += res_x[(long long)tr * d.nt];
      }
    }
  };
  load_v(x0 - 8);
  for (int r = x0 - 8; r < x1 + 8; r++) {
    push(w_bvx, n_bvx);
    push(w_bvz, n_bvz);
    push(w_avx, n_avx);
    push(w_avz, n_avz);
    load_v(r + 1);
    // ---- stage 1: stresses of row r1 = r - 4 -----------------------------------------------
    const int r1 = r - 4;
    s_bvx[t] = w_bvx[4];
    s_bvz[t] = w_bvz[4];
    s_avx[t] = w_avx[4];
    s_avz[t] = w_avz[4];
    __syncthreads();
    float btxx = 0.f, btzz = 0.f, btxz = 0.f, P = 0.f, L = 0.f, M = 0.f, Pz = 0.f, Lx = 0.f;
    if (c1 && zin && r >= x0 && r1 >= 0 && r1 < d.nxp) {
      const long long k = base + (long long)r1 * ld + z;
      const bool own = c2 && r1 >= x0 && r1 < x1;
      btxx = __ldg(a.ra.txx + k);
      btzz = __ldg(a.ra.tzz + k);
      btxz = __ldg(a.ra.txz + k);
      const bool x_int = r1 >= pml && r1 < d.nxp - pml;
      float gx_vx = 0.f, gz_vz = 0.f, gz_vx = 0.f, gx_vz = 0.f;
      const float lam = __ldg(a.p.lam + k), mu = __ldg(a.p.mu + k);
      if (x_int && z_int) {
        const float sa = dxm_mid(w_bvx);
        const float sf = dxp_mid(w_bvz);
        const float sb = stencil4([&](int i) { return s_bvz[t + i - 1] - s_bvz[t - i]; });
        const float se = stencil4([&](int i) { return s_bvx[t + i] - s_bvx[t - i + 1]; });
        const float l2m = lam + 2.0f * mu;
        const float dir = -1.0f;
        btxx = btxx + (dir * l2m * dtdx * sa + dir * lam * dtdz * sb);
        btzz = btzz + (dir * lam * dtdx * sa + dir * l2m * dtdz * sb);
        btxz = btxz + (dir * mu * dtdx * sf + dir * mu * dtdz * se);
        gx_vx = sa * rdx;  // strains; reciprocal multiply (the division's slow path is taken
        gz_vz = sb * rdz;  // for the tiny amplitudes ahead of a wavefront)
        gz_vx = se * rdz;
        gx_vz = sf * rdx;
        if (own) {
          a.rb.txx[k] = btxx;
          a.rb.tzz[k] = btzz;
          a.rb.txz[k] = btxz;
        }
      }
      // adjoint stresses (modulus-free; txx is txx_x, tzz is tzz_z)
      float atxx = 0.f, atzz = 0.f, atxz = 0.f;
      if (r1 >= d.nop && r1 < d.nxp - d.nop && z_upd) {
        const float sa = dxm_mid(w_avx);
        const float sf = dxp_mid(w_avz);
        const float sb = stencil4([&](int i) { return s_avz[t + i - 1] - s_avz[t - i]; });
        const float se = stencil4([&](int i) { return s_avx[t + i] - s_avx[t - i + 1]; });
        const float xx = -dtdx * sa, zz = -dtdz * sb, xz_x = -dtdx * sf, xz_z = -dtdz * se;
        const float oxx = __ldg(a.aa.txx + k), ozz = __ldg(a.aa.tzz + k);
        if (kPML && pml_cell(d, r1, z)) {
          const float ddx = a.p.dampx[k] * d.dt * 0.5f, ddz = a.p.dampz[k] * d.dt * 0.5f;
          const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
          const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
          atxx = fmaf(d1, oxx, xx) * i2;
          atzz = fmaf(d3, ozz, zz) * i4;
          const float q1 = fmaf(d1, a.aa.txz_x[k], xz_x) * i2;
          const float q2 = fmaf(d3, a.aa.txz_z[k], xz_z) * i4;
          if (own) {
            a.ab.txz_x[k] = q1;
            a.ab.txz_z[k] = q2;
          }
          atxz = q1 + q2;
        } else {
          atxx = oxx + xx;
          atzz = ozz + zz;
          atxz = __ldg(a.aa.txz + k) + (xz_x + xz_z);
        }
        if (own) {
          a.ab.txx[k] = atxx;
          a.ab.tzz[k] = atzz;
          a.ab.txz[k] = atxz;
        }
      }
      const float l2m = lam + 2.0f * mu;
      P = l2m * atxx;
      L = lam * atzz;
      M = mu * atxz;
      Pz = l2m * atzz;
      Lx = lam * atxx;
      if (own && x_int && z_int) {
        const long long o = ((long long)s * d.wnx_max + (r1 - pml)) * d.ild + z;
        const float kpp = __ldg(a.p.kpp + k), kps = __ldg(a.p.kps + k);
        const float lamda_grad = (gx_vx + gz_vz) * (atxx + atzz);
        const float miu_grad = -2.0f * (gx_vx * atzz + gz_vz * atxx) + (gz_vx + gx_vz) * atxz;
        a.img[o] += kpp * lamda_grad;
        a.img[a.img_plane + o] += kps * miu_grad;
      }
    }
    push(w_btxx, btxx);
    push(w_btxz, btxz);
    push(w_btzz, btzz);
    push(w_P, P);
    push(w_L, L);
    push(w_M, M);
    push(w_Pz, Pz);
    push(w_Lx, Lx);
    // ---- stage 2: velocities of row r2 = r - 8 ---------------------------------------------
    const int r2 = r - 8;
    s_btxz[t] = w_btxz[4];
    s_btzz[t] = w_btzz[0];
    s_m[t] = w_M[4];
    s_pz[t] = w_Pz[0];
    s_lx[t] = w_Lx[0];
    __syncthreads();
    if (c2 && zin && r2 >= x0 && r2 < x1) {
      const long long k = base + (long long)r2 * ld + z;
      const bool x_int = r2 >= pml && r2 < d.nxp - pml;
      const float bb = __ldg(a.p.b + k);
      const float cbx = bb * dtdx, cbz = bb * dtdz;
      if (x_int && z_int) {
        const float ax = dxp_mid(w_btxx);
        const float fx = dxm_mid(w_btxz);
        const float bz = stencil4([&](int i) { return s_btxz[t + i - 1] - s_btxz[t - i]; });
        const float ez = stencil4([&](int i) { return s_btzz[t + i] - s_btzz[t - i + 1]; });
        float ovx = w_bvx[0], ovz = w_bvz[0];
        if (a.strips_on && band_offset(d, r2, z) >= 0) {  // inner band: own state, not the strip
          ovx = __ldg(a.ra.vx + k);
          ovz = __ldg(a.ra.vz + k);
        }
        const float vx = ovx + (-cbx * ax + -cbz * bz);
        const float vz = ovz + (-cbx * fx + -cbz * ez);
        a.rb.vx[k] = vx;
        a.rb.vz[k] = vz;
        const long long o = ((long long)s * d.wnx_max + (r2 - pml)) * d.ild + z;
        a.img[2 * a.img_plane + o] += vx * vx + vz * vz;
      }
      if (r2 >= d.nop && r2 < d.nxp - d.nop && z_upd) {
        const float t_xx = dxp_mid(w_P);
        const float t_zx = dxp_mid(w_L);
        const float s_xz = dxm_mid(w_M);
        const float t_xz = stencil4([&](int i) { return s_m[t + i - 1] - s_m[t - i]; });
        const float s_zz = stencil4([&](int i) { return s_pz[t + i] - s_pz[t - i + 1]; });
        const float s_xx = stencil4([&](int i) { return s_lx[t + i] - s_lx[t - i + 1]; });
        const float ux_x = fmaf(-cbx, t_zx, -cbx * t_xx), ux_z = -cbz * t_xz;
        const float uz_x = -cbx * s_xz, uz_z = fmaf(-cbz, s_xx, -cbz * s_zz);
        float vx, vz;
        if (kPML && pml_cell(d, r2, z)) {
          const float ddx = a.p.dampx[k] * d.dt * 0.5f, ddz = a.p.dampz[k] * d.dt * 0.5f;
          const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
          const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
          const float vxx = fmaf(d1, a.aa.vx_x[k], ux_x) * i2;
          const float vxz = fmaf(d3, a.aa.vx_z[k], ux_z) * i4;
          const float vzx = fmaf(d1, a.aa.vz_x[k], uz_x) * i2;
          const float vzz = fmaf(d3, a.aa.vz_z[k], uz_z) * i4;
          a.ab.vx_x[k] = vxx; a.ab.vx_z[k] = vxz; a.ab.vz_x[k] = vzx; a.ab.vz_z[k] = vzz;
          vx = vxx + vxz;
          vz = vzx + vzz;
        } else {
          float ovx = w_avx[0], ovz = w_avz[0];
          if (rec_col && rmap[r2] >= 0) {  // injected cell: state without the residual
            ovx = __ldg(a.aa.vx + k);
            ovz = __ldg(a.aa.vz + k);
          }
          vx = ovx + (ux_x + ux_z);
          vz = ovz + (uz_x + uz_z);
        }
        a.ab.vx[k] = vx;
        a.ab.vz[k] = vz;
      }
    }
  }
}

// Backward RTM step fed by the ring (same arithmetic as k_bwd_fused).  Fields of ring slot q:
//  0-3   bvx, bvz, avx, avz of row q            (stage-1 stencil windows)
//  4-15  btxx, btzz, btxz, atxx, atzz, atxz, lam, mu, kpp, kps, img pp, img ps of row q-4
//  16-17 b, img illumination of row q-8          (stage 2)
// With PML and strips every operand that a cell of the band reads is prefetched the same way, so
// no load waits inside the march.  A PML cell is never an imaging cell and never reads its own
// atxz, so for it the slots of atxz, kpp, kps, img pp (row q-4) carry atxz_x, atxz_z, dampx,
// dampz, and the slot of the illumination (row q-8) carries dampx; a strip-band cell takes its
// velocities from the strips, so slots 0-1 carry the strip words of its row.  Extra fields:
//  18-22 dampz, avx_x, avx_z, avz_x, avz_z of row q-8  (PML cells, stage 2)
//  23-24 bvx, bvz of row q-8   (inner strip-band cells: their own state, stage 2)
//  25-26 the FP32 scales of the two strip words of row q  (FP16 / BF16 strips)
constexpr int kBwdRingFields = 18;
constexpr int kBwdRingFieldsPml = 27;
__host__ __device__ constexpr int bwd_ring_fields(bool pml) {
  return pml ? kBwdRingFieldsPml : kBwdRingFields;
}

// Band value of strip element e from its ring copy: the FP32 element itself, or the aligned
// 32-bit word holding the FP16 / BF16 element (upper half for odd e) times its segment's scale.
// Same result as strip_get.
__device__ __forceinline__ float strip_unpack(int prec, long long e, float word, float sc) {
  if (prec == 0) return word;
  const unsigned u = __float_as_uint(word);
  const unsigned short h = (unsigned short)((e & 1) ? (u >> 16) : (u & 0xffffu));
  if (prec == 1) return __half2float(__ushort_as_half(h)) * sc;
  return __bfloat162float(__ushort_as_bfloat16(h)) * sc;
}

// kOne: one barrier per row step instead of two.  Every z-tap row of a step
// exists at its top -- stage 1's rows are this step's inputs at row r - 4, stage 2's are stage-1
// outputs of row r - 8, computed four steps earlier -- so all eight are published there, into one
// of two buffers (a thread running ahead writes the other), and the two stages then run without
// a barrier between them.
template <bool kPML, int kD, int kMinB, int kT = kFB, bool kOne = false>
__global__ void __launch_bounds__(kT, kMinB) k_bwd_ring(BwdFusedArgs a) {
  static_assert(kD >= 2 && kD <= 8 && (kD & (kD - 1)) == 0, "ring depth: 2, 4 or 8");
  constexpr int NF = bwd_ring_fields(kPML);
  extern __shared__ float ring[];  // [kD][NF][kT]
  // z-tap rows: bvx bvz avx avz (stage 1), btxz btzz M PzLx (stage 2); two buffers with kOne
  __shared__ float s_zt[kOne ? 2 : 1][8][kT];
  // Receiver column (one thread of the CTA, if any): per row mod 16, the trace index (fetched 16
  // rows ahead), whether a trace sits there and its residual at this step (fetched 8 rows ahead)
  // and the cell's state without the residual (kept 8 rows for stage 2).
  __shared__ int s_tr[16], s_has[16];
  __shared__ float s_rz[16], s_rx[16], s_ownx[16], s_ownz[16];
  // PML variants: per ring slot and thread, the predicates issue(q) derives for the rows slot q's
  // step consumes -- the strip-band offset of row q, and bits 1 / 2 / 4 = PML cell at row q-4,
  // PML cell at row q-8, inner strip-band cell at row q-8 -- so the march does not derive them
  // again (same thread, written kD - 1 steps before the read).
  __shared__ int s_bo[kPML ? kD * kT : 1], s_fl[kPML ? kD * kT : 1];
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int z = blockIdx.x * a.tz - 8 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const int base = (int)(d.slot * s);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld, pml = d.pml;
  const bool zin = z >= 0 && z < d.nzp;
  const bool c1 = t >= 4 && t < a.tz + 12;
  const bool c2 = t >= 8 && t < a.tz + 8;
  const bool z_int = z >= pml && z < d.nzp - pml;
  const bool z_upd = z >= d.nop && z < d.nzp - d.nop;
  const ShotDev sh = a.shots[s];
  const bool rec_col = z == sh.igz;
  const bool strips = kPML && a.strips_on;
  const float *res_z = a.res_vz + (long long)s * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)s * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  const int img_row = s * d.wnx_max;  // image row of model row r: img_row + r - pml
  float *img_pp = a.img, *img_ps = a.img + a.img_plane, *img_il = a.img + 2 * a.img_plane;
  const long long strip_row0 = ((long long)s * d.nt + a.it) * 2;  // strip row of component 0
  const float *grid_src[15] = {a.ra.vx,  a.ra.vz,  a.aa.vx,  a.aa.vz,  a.ra.txx,
                               a.ra.tzz, a.ra.txz, a.aa.txx, a.aa.tzz, a.aa.txz,
                               a.p.lam,  a.p.mu,   a.p.kpp,  a.p.kps,  a.p.b};
  auto R = [&](int q, int f) -> float & { return ring[((q & (kD - 1)) * NF + f) * kT + t]; };
  auto strip_elem = [&](int comp, int bo) { return (strip_row0 + comp) * d.lb_max + bo; };
  // band_offset with this thread's column terms hoisted, as selects
  const int N = d.nop;
  const bool zb_up = z >= pml - N && z < pml + N, zb_dn = z >= d.nzp - pml - N && z < d.nzp - pml + N;
  const int zb_off = zb_up ? z - (pml - N) : d.wnx * 2 * N + z - (d.nzp - pml - N);
  const bool zP = z < pml || z > d.nzp - pml;
  auto band_row = [&](int ix) {
    const bool xint = ix >= pml && ix < d.nxp - pml;
    const bool xl = ix >= pml - N && ix < pml + N, xr = ix >= d.nxp - pml - N && ix < d.nxp - pml + N;
    const int a1 = (ix - pml) * 2 * N + zb_off;
    const int a2 = 4 * N * d.wnx + (xl ? ix - (pml - N) : 2 * N + ix - (d.nxp - pml - N)) * d.wnz + (z - pml);
    return (xint && (zb_up || zb_dn)) ? a1 : ((z_int && (xl || xr)) ? a2 : -1);
  };
  auto pml_row = [&](int ix) { return zP || ix < pml || ix > d.nxp - pml; };
  auto issue = [&](int q) {
    const int r0 = q, r4 = q - 4, r8 = q - 8;
    const bool in0 = r0 >= 0 && r0 < d.nxp && zin;
    const bool in4 = r4 >= 0 && r4 < d.nxp && zin;
    const bool in8 = r8 >= 0 && r8 < d.nxp && zin;
    const int o0 = base + r0 * ld + z, o4 = base + r4 * ld + z, o8 = base + r8 * ld + z;
    const bool int4 = in4 && r4 >= pml && r4 < d.nxp - pml && z_int;
    const bool int8 = in8 && r8 >= pml && r8 < d.nxp - pml && z_int;
    const bool pml4 = kPML && in4 && pml_row(r4);
    const bool pml8 = kPML && in8 && pml_row(r8);
    const int bo0 = strips && in0 ? band_row(r0) : -1;
    const bool own8 = strips && int8 && band_row(r8) >= 0;
    if (kPML) {
      s_bo[(q & (kD - 1)) * kT + t] = bo0;
      s_fl[(q & (kD - 1)) * kT + t] = (pml4 ? 1 : 0) | (pml8 ? 2 : 0) | (own8 ? 4 : 0);
    }
    // lag 0: stencil inputs (strip words in the band)
#pragma unroll
    for (int f = 0; f < 4; f++) {
      float *dst = &R(q, f);
      if (!in0) {
        *dst = 0.f;
      } else if (kPML && f < 2 && bo0 >= 0) {
        const long long e = strip_elem(f, bo0);
        if (a.st.prec == 0) {
          cp_async4(dst, (const float *)a.st.data + e);
        } else {
          cp_async4(dst, (const float *)((const char *)a.st.data + ((e * 2) & ~3LL)));
          cp_async4(&R(q, 25 + f), a.st.scale + (strip_row0 + f) * d.nseg_max + (bo0 >> 5));
        }
      } else {
        cp_async4(dst, grid_src[f] + o0);
      }
    }
    // lag 4: stage-1 own-cell operands
#pragma unroll
    for (int f = 4; f < 16; f++) {
      float *dst = &R(q, f);
      if (kPML && pml4 && (f == 9 || (f >= 12 && f <= 15))) {
        if (f == 9) cp_async4(dst, a.aa.txz_x + o4);
        if (f == 12) cp_async4(dst, a.aa.txz_z + o4);
        if (f == 13) cp_async4(dst, a.p.dampx + o4);
        if (f == 14) cp_async4(dst, a.p.dampz + o4);
      } else if (f == 14 || f == 15) {
        if (int4)
          cp_async4(dst, (f == 14 ? img_pp : img_ps) + ((img_row + r4 - pml) * d.ild + z));
        else
          *dst = 0.f;
      } else if (in4) {
        cp_async4(dst, grid_src[f] + o4);
      } else {
        *dst = 0.f;
      }
    }
    // lag 8: stage-2 own-cell operands
    if (in8) cp_async4(&R(q, 16), a.p.b + o8); else R(q, 16) = 0.f;
    if (kPML && pml8) {
      cp_async4(&R(q, 17), a.p.dampx + o8);
      cp_async4(&R(q, 18), a.p.dampz + o8);
      cp_async4(&R(q, 19), a.aa.vx_x + o8);
      cp_async4(&R(q, 20), a.aa.vx_z + o8);
      cp_async4(&R(q, 21), a.aa.vz_x + o8);
      cp_async4(&R(q, 22), a.aa.vz_z + o8);
    } else if (int8) {
      cp_async4(&R(q, 17), img_il + ((img_row + r8 - pml) * d.ild + z));
      if (own8) {
        cp_async4(&R(q, 23), a.ra.vx + o8);
        cp_async4(&R(q, 24), a.ra.vz + o8);
      }
    } else {
      R(q, 17) = 0.f;
    }
    cp_async_commit();
  };

  float w_bvx[9], w_bvz[9], w_avx[9], w_avz[9];
  // Adjoint-velocity operands: the stage-2 update needs Dx+((l+2m) atxx) + Dx+(l atzz) and
  // Dz+((l+2m) atzz) + Dz+(l atxx); by linearity each pair is one derivative of the summed
  // product, so stage 1 keeps PL = (l+2m) atxx + l atzz and PzLx = (l+2m) atzz + l atxx.
  float w_btxx[9], w_btxz[9], w_btzz[5], w_PL[9], w_M[9], w_PzLx[5];
#pragma unroll
  for (int i = 0; i < 9; i++)
    w_bvx[i] = w_bvz[i] = w_avx[i] = w_avz[i] = w_btxx[i] = w_btxz[i] = w_PL[i] = w_M[i] = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) w_btzz[i] = w_PzLx[i] = 0.f;

#pragma unroll
  for (int j = 0; j < kD - 1; j++) issue(x0 - 8 + j);
  if (rec_col) {  // trace indexes of the first 16 rows, residuals of the first 8 (direct loads)
    for (int q = x0 - 8; q < x0 + 8; q++) s_tr[q & 15] = (q >= 0 && q < d.nxp) ? rmap[q] : -1;
    for (int q = x0 - 8; q < x0; q++) {
      const int tr = s_tr[q & 15];
      s_has[q & 15] = tr >= 0;
      if (tr >= 0) {
        s_rz[q & 15] = res_z[(long long)tr * d.nt];
        s_rx[q & 15] = res_x[(long long)tr * d.nt];
      }
    }
  }
#pragma unroll kRingUnrollBwd
  for (int r = x0 - 8; r < x1 + 8; r++) {
    cp_async_wait<kD - 2>();  // slot r has landed (this thread's copies)
    if (rec_col) {
      // Residual of row r + 8 and trace index of row r + 16, copied asynchronously with this
      // step's commit group (landed kD - 1 <= 7 steps later, before either is read).
      const int q8 = r + 8, q16 = r + 16;
      const int tr8 = s_tr[q8 & 15];
      s_has[q8 & 15] = tr8 >= 0;
      if (tr8 >= 0) {
        cp_async4(&s_rz[q8 & 15], res_z + (long long)tr8 * d.nt);
        cp_async4(&s_rx[q8 & 15], res_x + (long long)tr8 * d.nt);
      }
      if (q16 < d.nxp)
        cp_async4((float *)&s_tr[q16 & 15], (const float *)(rmap + q16));
      else
        s_tr[q16 & 15] = -1;
    }
    const int pfl = kPML ? s_fl[(r & (kD - 1)) * kT + t] : 0;  // cached predicates of slot r
    {
      float n_bvx = R(r, 0), n_bvz = R(r, 1), n_avx = R(r, 2), n_avz = R(r, 3);
      if (r >= 0 && r < d.nxp && zin) {
        if (strips) {
          const int bo = s_bo[(r & (kD - 1)) * kT + t];
          if (bo >= 0) {
            n_bvx = strip_unpack(a.st.prec, strip_elem(0, bo), n_bvx, R(r, 25));
            n_bvz = strip_unpack(a.st.prec, strip_elem(1, bo), n_bvz, R(r, 26));
          }
        }
        if (rec_col) {
          s_ownx[r & 15] = n_avx;
          s_ownz[r & 15] = n_avz;
          if (s_has[r & 15]) {
            n_avz += s_rz[r & 15];
            n_avx += s_rx[r & 15];
          }
        }
      }
      push(w_bvx, n_bvx);
      push(w_bvz, n_bvz);
      push(w_avx, n_avx);
      push(w_avz, n_avz);
    }
    // Refill the slot of row r - 1 (mod kD) with row r + kD - 1; only slot r is read below.
    issue(r + kD - 1);
    // ---- stage 1: stresses of row r1 = r - 4 -----------------------------------------------
    const int r1 = r - 4;
    float *const s_bvx = s_zt[kOne ? (r & 1) : 0][0], *const s_bvz = s_zt[kOne ? (r & 1) : 0][1];
    float *const s_avx = s_zt[kOne ? (r & 1) : 0][2], *const s_avz = s_zt[kOne ? (r & 1) : 0][3];
    float *const s_btxz = s_zt[kOne ? (r & 1) : 0][4], *const s_btzz = s_zt[kOne ? (r & 1) : 0][5];
    float *const s_m = s_zt[kOne ? (r & 1) : 0][6], *const s_pzlx = s_zt[kOne ? (r & 1) : 0][7];
    s_bvx[t] = w_bvx[4];
    s_bvz[t] = w_bvz[4];
    s_avx[t] = w_avx[4];
    s_avz[t] = w_avz[4];
    if (kOne) {  // stage-2 rows of row r - 8 (before this step's stage-1 push: index 5 / 1)
      s_btxz[t] = w_btxz[5];
      s_btzz[t] = w_btzz[1];
      s_m[t] = w_M[5];
      s_pzlx[t] = w_PzLx[1];
    }
    __syncthreads();
    float btxx = 0.f, btzz = 0.f, btxz = 0.f, PL = 0.f, M = 0.f, PzLx = 0.f;
    if (c1 && zin && r >= x0 && r1 >= 0 && r1 < d.nxp) {
      const int k = base + r1 * ld + z;
      const bool own = c2 && r1 >= x0 && r1 < x1;
      btxx = R(r, 4);
      btzz = R(r, 5);
      btxz = R(r, 6);
      const bool x_int = r1 >= pml && r1 < d.nxp - pml;
      float gx_vx = 0.f, gz_vz = 0.f, gz_vx = 0.f, gx_vz = 0.f;
      const float lam = R(r, 10), mu = R(r, 11);
      if (x_int && z_int) {
        const float sa = dxm_mid(w_bvx);
        const float sf = dxp_mid(w_bvz);
        const float sb = stencil4([&](int i) { return s_bvz[t + i - 1] - s_bvz[t - i]; });
        const float se = stencil4([&](int i) { return s_bvx[t + i] - s_bvx[t - i + 1]; });
        const float l2m = lam + 2.0f * mu;
        const float dir = -1.0f;
        btxx = btxx + (dir * l2m * dtdx * sa + dir * lam * dtdz * sb);
        btzz = btzz + (dir * lam * dtdx * sa + dir * l2m * dtdz * sb);
        btxz = btxz + (dir * mu * dtdx * sf + dir * mu * dtdz * se);
        gx_vx = sa * rdx;  // strains; reciprocal multiply (the division's slow path is taken
        gz_vz = sb * rdz;  // for the tiny amplitudes ahead of a wavefront)
        gz_vx = se * rdz;
        gx_vz = sf * rdx;
        if (own) {
          a.rb.txx[k] = btxx;
          a.rb.tzz[k] = btzz;
          a.rb.txz[k] = btxz;
        }
      }
      float atxx = 0.f, atzz = 0.f, atxz = 0.f;
      if (r1 >= d.nop && r1 < d.nxp - d.nop && z_upd) {
        const float sa = dxm_mid(w_avx);
        const float sf = dxp_mid(w_avz);
        const float sb = stencil4([&](int i) { return s_avz[t + i - 1] - s_avz[t - i]; });
        const float se = stencil4([&](int i) { return s_avx[t + i] - s_avx[t - i + 1]; });
        const float xx = -dtdx * sa, zz = -dtdz * sb, xz_x = -dtdx * sf, xz_z = -dtdz * se;
        const float oxx = R(r, 7), ozz = R(r, 8);
        if (kPML && (pfl & 1)) {
          // ring slots 9, 12, 13, 14 of a PML cell: atxz_x, atxz_z, dampx, dampz
          const float ddx = R(r, 13) * d.dt * 0.5f, ddz = R(r, 14) * d.dt * 0.5f;
          const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
          const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
          atxx = fmaf(d1, oxx, xx) * i2;
          atzz = fmaf(d3, ozz, zz) * i4;
          const float q1 = fmaf(d1, R(r, 9), xz_x) * i2;
          const float q2 = fmaf(d3, R(r, 12), xz_z) * i4;
          if (own) {
            a.ab.txz_x[k] = q1;
            a.ab.txz_z[k] = q2;
          }
          atxz = q1 + q2;
        } else {
          atxx = oxx + xx;
          atzz = ozz + zz;
          atxz = R(r, 9) + (xz_x + xz_z);
        }
        if (own) {
          a.ab.txx[k] = atxx;
          a.ab.tzz[k] = atzz;
          a.ab.txz[k] = atxz;
        }
      }
      const float l2m = lam + 2.0f * mu;
      PL = l2m * atxx + lam * atzz;
      M = mu * atxz;
      PzLx = l2m * atzz + lam * atxx;
      if (own && x_int && z_int) {
        const int o = (img_row + (r1 - pml)) * d.ild + z;
        const float kpp = R(r, 12), kps = R(r, 13);
        const float lamda_grad = (gx_vx + gz_vz) * (atxx + atzz);
        const float miu_grad = -2.0f * (gx_vx * atzz + gz_vz * atxx) + (gz_vx + gx_vz) * atxz;
        img_pp[o] = R(r, 14) + kpp * lamda_grad;
        img_ps[o] = R(r, 15) + kps * miu_grad;
      }
    }
    push(w_btxx, btxx);
    push(w_btxz, btxz);
    push(w_btzz, btzz);
    push(w_PL, PL);
    push(w_M, M);
    push(w_PzLx, PzLx);
    // ---- stage 2: velocities of row r2 = r - 8 ---------------------------------------------
    const int r2 = r - 8;
    if (!kOne) {
      s_btxz[t] = w_btxz[4];
      s_btzz[t] = w_btzz[0];
      s_m[t] = w_M[4];
      s_pzlx[t] = w_PzLx[0];
      __syncthreads();
    }
    if (c2 && zin && r2 >= x0 && r2 < x1) {
      const int k = base + r2 * ld + z;
      const bool x_int = r2 >= pml && r2 < d.nxp - pml;
      const float bb = R(r, 16);
      const float cbx = bb * dtdx, cbz = bb * dtdz;
      if (x_int && z_int) {
        const float ax = dxp_mid(w_btxx);
        const float fx = dxm_mid(w_btxz);
        const float bz = stencil4([&](int i) { return s_btxz[t + i - 1] - s_btxz[t - i]; });
        const float ez = stencil4([&](int i) { return s_btzz[t + i] - s_btzz[t - i + 1]; });
        float ovx = w_bvx[0], ovz = w_bvz[0];
        if (strips && (pfl & 4)) {  // inner band: own state, not the strip
          ovx = R(r, 23);
          ovz = R(r, 24);
        }
        const float vx = ovx + (-cbx * ax + -cbz * bz);
        const float vz = ovz + (-cbx * fx + -cbz * ez);
        a.rb.vx[k] = vx;
        a.rb.vz[k] = vz;
        const int o = (img_row + (r2 - pml)) * d.ild + z;
        img_il[o] = R(r, 17) + (vx * vx + vz * vz);
      }
      if (r2 >= d.nop && r2 < d.nxp - d.nop && z_upd) {
        const float t_x = dxp_mid(w_PL);
        const float s_xz = dxm_mid(w_M);
        const float t_xz = stencil4([&](int i) { return s_m[t + i - 1] - s_m[t - i]; });
        const float s_z = stencil4([&](int i) { return s_pzlx[t + i] - s_pzlx[t - i + 1]; });
        const float ux_x = -cbx * t_x, ux_z = -cbz * t_xz;
        const float uz_x = -cbx * s_xz, uz_z = -cbz * s_z;
        float vx, vz;
        if (kPML && (pfl & 2)) {
          // ring slots 17-22 of a PML cell: dampx, dampz, avx_x, avx_z, avz_x, avz_z
          const float ddx = R(r, 17) * d.dt * 0.5f, ddz = R(r, 18) * d.dt * 0.5f;
          const float d1 = 1.0f - ddx, d3 = 1.0f - ddz;
          const float i2 = __frcp_rn(1.0f + ddx), i4 = __frcp_rn(1.0f + ddz);  // no divide slow path
          const float vxx = fmaf(d1, R(r, 19), ux_x) * i2;
          const float vxz = fmaf(d3, R(r, 20), ux_z) * i4;
          const float vzx = fmaf(d1, R(r, 21), uz_x) * i2;
          const float vzz = fmaf(d3, R(r, 22), uz_z) * i4;
          a.ab.vx_x[k] = vxx; a.ab.vx_z[k] = vxz; a.ab.vz_x[k] = vzx; a.ab.vz_z[k] = vzz;
          vx = vxx + vxz;
          vz = vzx + vzz;
        } else {
          float ovx = w_avx[0], ovz = w_avz[0];
          if (rec_col) {  // receiver column: the state without the residual
            ovx = s_ownx[r2 & 15];
            ovz = s_ownz[r2 & 15];
          }
          vx = ovx + (ux_x + ux_z);
          vz = ovz + (uz_x + uz_z);
        }
        a.ab.vx[k] = vx;
        a.ab.vz[k] = vz;
      }
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Reverse step of the first-order scattered set of reference-mode ELSRTM (FD2DGPU.cu:4685-4807),
// fed by the ring: interior reconstruction of b1 (stress then velocity, direction -1; strips st_b
// in the band, as k_str<kRev> / k_vel<kRev>), with the Born source of the background's
// reconstructed velocities (ov_*, written by k_born after k_bwd_ring) added to the stress stencil
// values of the velocity stage, and the imaging condition of b1's strains with the adjoint
// stresses of the same step into images 3 and 4 (k_image, b_pp / b_ps).  Same x-march as
// k_bwd_ring: stage 1 updates the stresses of row r-4 and images them, stage 2 the velocities of
// row r-8.  Fields of ring slot q:
//  0-1   bvx, bvz of row q (strip words in the band)
//  2-6   btxx, btzz, btxz, lam, mu of row q-4
//  7-16  kpp, kps, image 3, image 4, atxx, atzz, atxz, ov txx, ov tzz, ov txz of row q-4 (interior)
//  17    b of row q-8; 18-19 bvx, bvz of row q-8 (inner strip-band cells: their own state)
//  20-21 the FP32 scales of the two strip words of row q (FP16 / BF16 strips)
struct BwdScatArgs {
  Dims d;
  Wave ra, rb;                            // b1 state at t (read), t-1 (written)
  const float *atxx, *atzz, *atxz;        // adjoint stresses of this step
  const float *ov_txx, *ov_tzz, *ov_txz;  // Born source of the background's velocities
  Par p;
  const ShotDev *shots;
  Strips st;
  int strips_on;
  int it;
  int tz, xr;
  float *img;  // [7][slot][wnx][wnz]; planes 3 and 4 are accumulated
  long long img_plane;
};
constexpr int kBwdScatRingFields = 22;

template <bool kPML, int kD, int kMinB>
__global__ void __launch_bounds__(kFB, kMinB) k_bwd_scat_ring(BwdScatArgs a) {
  static_assert(kD >= 2 && kD <= 8 && (kD & (kD - 1)) == 0, "ring depth: 2, 4 or 8");
  constexpr int NF = kBwdScatRingFields;
  extern __shared__ float ring[];  // [kD][NF][kFB]
  __shared__ float s_bvx[kFB], s_bvz[kFB], s_btxz[kFB], s_btzz[kFB];
  // strips: per ring slot and thread, the band offset of row q and whether row q-8 is an inner
  // band cell (derived once by issue(q), read by the same thread kD - 1 steps later)
  __shared__ int s_bo[kPML ? kD * kFB : 1], s_fl[kPML ? kD * kFB : 1];
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int z = blockIdx.x * a.tz - 8 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const int base = (int)(d.slot * s);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld, pml = d.pml;
  const bool zin = z >= 0 && z < d.nzp;
  const bool c1 = t >= 4 && t < a.tz + 12;
  const bool c2 = t >= 8 && t < a.tz + 8;
  const bool z_int = z >= pml && z < d.nzp - pml;
  const bool strips = kPML && a.strips_on;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  const int img_row = s * d.wnx_max;  // image row of model row r: img_row + r - pml
  float *img_b = a.img + 3 * a.img_plane, *img_bs = a.img + 4 * a.img_plane;
  const long long strip_row0 = ((long long)s * d.nt + a.it) * 2;
  auto R = [&](int q, int f) -> float & { return ring[((q & (kD - 1)) * NF + f) * kFB + t]; };
  auto strip_elem = [&](int comp, int bo) { return (strip_row0 + comp) * d.lb_max + bo; };
  auto issue = [&](int q) {
    const int r0 = q, r4 = q - 4, r8 = q - 8;
    const bool in0 = r0 >= 0 && r0 < d.nxp && zin;
    const bool in4 = r4 >= 0 && r4 < d.nxp && zin;
    const bool in8 = r8 >= 0 && r8 < d.nxp && zin;
    const int o0 = base + r0 * ld + z, o4 = base + r4 * ld + z, o8 = base + r8 * ld + z;
    const bool int4 = in4 && r4 >= pml && r4 < d.nxp - pml && z_int;
    const bool int8 = in8 && r8 >= pml && r8 < d.nxp - pml && z_int;
    const int bo0 = strips && in0 ? band_offset(d, r0, z) : -1;
    const bool own8 = strips && int8 && band_offset(d, r8, z) >= 0;
    if (kPML) {
      s_bo[(q & (kD - 1)) * kFB + t] = bo0;
      s_fl[(q & (kD - 1)) * kFB + t] = own8 ? 1 : 0;
    }
#pragma unroll
    for (int f = 0; f < 2; f++) {
      float *dst = &R(q, f);
      if (!in0) {
        *dst = 0.f;
      } else if (kPML && bo0 >= 0) {
        const long long e = strip_elem(f, bo0);
        if (a.st.prec == 0) {
          cp_async4(dst, (const float *)a.st.data + e);
        } else {
          cp_async4(dst, (const float *)((const char *)a.st.data + ((e * 2) & ~3LL)));
          cp_async4(&R(q, 20 + f), a.st.scale + (strip_row0 + f) * d.nseg_max + (bo0 >> 5));
        }
      } else {
        cp_async4(dst, (f == 0 ? a.ra.vx : a.ra.vz) + o0);
      }
    }
    if (in4) {
      cp_async4(&R(q, 2), a.ra.txx + o4);
      cp_async4(&R(q, 3), a.ra.tzz + o4);
      cp_async4(&R(q, 4), a.ra.txz + o4);
      cp_async4(&R(q, 5), a.p.lam + o4);
      cp_async4(&R(q, 6), a.p.mu + o4);
    } else {
      R(q, 2) = R(q, 3) = R(q, 4) = R(q, 5) = R(q, 6) = 0.f;
    }
    if (int4) {
      const int io = (img_row + r4 - pml) * d.ild + z;
      cp_async4(&R(q, 7), a.p.kpp + o4);
      cp_async4(&R(q, 8), a.p.kps + o4);
      cp_async4(&R(q, 9), img_b + io);
      cp_async4(&R(q, 10), img_bs + io);
      cp_async4(&R(q, 11), a.atxx + o4);
      cp_async4(&R(q, 12), a.atzz + o4);
      cp_async4(&R(q, 13), a.atxz + o4);
      cp_async4(&R(q, 14), a.ov_txx + o4);
      cp_async4(&R(q, 15), a.ov_tzz + o4);
      cp_async4(&R(q, 16), a.ov_txz + o4);
    } else {
      R(q, 14) = R(q, 15) = R(q, 16) = 0.f;  // the Born source is zero outside the interior
    }
    if (in8) cp_async4(&R(q, 17), a.p.b + o8); else R(q, 17) = 0.f;
    if (own8) {
      cp_async4(&R(q, 18), a.ra.vx + o8);
      cp_async4(&R(q, 19), a.ra.vz + o8);
    }
    cp_async_commit();
  };

  float w_bvx[9], w_bvz[9], w_btxx[9], w_btxz[9], w_btzz[5];
#pragma unroll
  for (int i = 0; i < 9; i++) w_bvx[i] = w_bvz[i] = w_btxx[i] = w_btxz[i] = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) w_btzz[i] = 0.f;

#pragma unroll
  for (int j = 0; j < kD - 1; j++) issue(x0 - 8 + j);
#pragma unroll kRingUnrollBwd
  for (int r = x0 - 8; r < x1 + 8; r++) {
    cp_async_wait<kD - 2>();  // slot r has landed (this thread's copies)
    {
      float n_bvx = R(r, 0), n_bvz = R(r, 1);
      if (strips && r >= 0 && r < d.nxp && zin) {
        const int bo = s_bo[(r & (kD - 1)) * kFB + t];
        if (bo >= 0) {
          n_bvx = strip_unpack(a.st.prec, strip_elem(0, bo), n_bvx, R(r, 20));
          n_bvz = strip_unpack(a.st.prec, strip_elem(1, bo), n_bvz, R(r, 21));
        }
      }
      push(w_bvx, n_bvx);
      push(w_bvz, n_bvz);
    }
    issue(r + kD - 1);
    // ---- stage 1: stresses of row r1 = r - 4, strains, images 3 and 4 -------------------------
    const int r1 = r - 4;
    s_bvx[t] = w_bvx[4];
    s_bvz[t] = w_bvz[4];
    __syncthreads();
    float pxx = 0.f, pzz = 0.f, pxz = 0.f;  // stress + Born source: the velocity stage's operand
    if (c1 && zin && r >= x0 && r1 >= 0 && r1 < d.nxp) {
      const int k = base + r1 * ld + z;
      const bool own = c2 && r1 >= x0 && r1 < x1;
      float btxx = R(r, 2), btzz = R(r, 3), btxz = R(r, 4);
      if (r1 >= pml && r1 < d.nxp - pml && z_int) {
        const float sa = dxm_mid(w_bvx);
        const float sf = dxp_mid(w_bvz);
        const float sb = stencil4([&](int i) { return s_bvz[t + i - 1] - s_bvz[t - i]; });
        const float se = stencil4([&](int i) { return s_bvx[t + i] - s_bvx[t - i + 1]; });
        const float lam = R(r, 5), mu = R(r, 6);
        const float l2m = lam + 2.0f * mu;
        const float dir = -1.0f;
        btxx = btxx + (dir * l2m * dtdx * sa + dir * lam * dtdz * sb);
        btzz = btzz + (dir * lam * dtdx * sa + dir * l2m * dtdz * sb);
        btxz = btxz + (dir * mu * dtdx * sf + dir * mu * dtdz * se);
        if (own) {
          a.rb.txx[k] = btxx;
          a.rb.tzz[k] = btzz;
          a.rb.txz[k] = btxz;
          const float gx_vx = sa * rdx, gz_vz = sb * rdz, gz_vx = se * rdz, gx_vz = sf * rdx;
          const float atxx = R(r, 11), atzz = R(r, 12), atxz = R(r, 13);
          const float lamda_grad = (gx_vx + gz_vz) * (atxx + atzz);
          const float miu_grad = -2.0f * (gx_vx * atzz + gz_vz * atxx) + (gz_vx + gx_vz) * atxz;
          const int o = (img_row + (r1 - pml)) * d.ild + z;
          img_b[o] = R(r, 9) + R(r, 7) * lamda_grad;
          img_bs[o] = R(r, 10) + R(r, 8) * miu_grad;
        }
      }
      pxx = btxx + R(r, 14);
      pzz = btzz + R(r, 15);
      pxz = btxz + R(r, 16);
    }
    push(w_btxx, pxx);
    push(w_btxz, pxz);
    push(w_btzz, pzz);
    // ---- stage 2: velocities of row r2 = r - 8 ---------------------------------------------
    const int r2 = r - 8;
    s_btxz[t] = w_btxz[4];
    s_btzz[t] = w_btzz[0];
    __syncthreads();
    if (c2 && zin && r2 >= x0 && r2 < x1 && r2 >= pml && r2 < d.nxp - pml && z_int) {
      const int k = base + r2 * ld + z;
      const float bb = R(r, 17);
      const float cbx = bb * dtdx, cbz = bb * dtdz;
      const float ax = dxp_mid(w_btxx);
      const float fx = dxm_mid(w_btxz);
      const float bz = stencil4([&](int i) { return s_btxz[t + i - 1] - s_btxz[t - i]; });
      const float ez = stencil4([&](int i) { return s_btzz[t + i] - s_btzz[t - i + 1]; });
      float ovx = w_bvx[0], ovz = w_bvz[0];
      if (strips && s_fl[(r & (kD - 1)) * kFB + t]) {  // inner band: own state, not the strip
        ovx = R(r, 18);
        ovz = R(r, 19);
      }
      a.rb.vx[k] = ovx + (-cbx * ax + -cbz * bz);
      a.rb.vz[k] = ovz + (-cbx * fx + -cbz * ez);
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Acoustic forward step fed by the ring (vs = 0: the stress is one field s = txx = tzz, txz = 0),
// the fused counterpart of k_ac_vel + k_ac_str (+ k_ac_born).  Same x-march as k_fwd_ring: at row
// step r the velocities of row r - 4 (from the window of S = s + overlay) and the stress of row
// r - 8 (from the new velocities) are updated, state ping-pongs between two buffers.
//   kMode 0 (background): the explosive source is the overlay on s; with `e` set, the stress
//           stage also writes the Born source e = -2 lam m (Dx- vx / dx + Dz- vz / dz) of the new
//           velocities on the interior (the k_ac_born of the same step).
//   kMode 1 (scattered): the Born source e of the same step is the overlay on s; the new
//           velocities are recorded at the receivers.
// Ring fields of slot q: 0 s and 1 e (overlay, mode 1) of row q; 2 vx, 3 vz, 4 b of row q - 4;
// 5 s (own state), 6 lam, 7 m of row q - 8.
// ---------------------------------------------------------------------------------------------
constexpr int kAcRingFields = 8;

struct AcRingArgs {
  Dims d;
  const ShotDev *shots;
  const float *vx, *vz, *s;  // state at t-1 (read)
  float *vx_n, *vz_n, *s_n;  // state at t (written)
  const float *b, *lam, *m;
  const float *e_in;         // mode 1: Born source overlay
  float *e_out;              // mode 0: Born source written (or null)
  const float *wavelet;
  int it, tz, xr;
  const int *rmap;
  float *rec_vz, *rec_vx;    // mode 1: records [slot][max_ntr][nt]
  int *err;                  // pair kernels: error word (a ring wait that gave up)
};

template <int kMode, int kD>
__global__ void __launch_bounds__(kFB, 6) k_ac_ring(AcRingArgs a) {
  static_assert(kD >= 2 && (kD & (kD - 1)) == 0, "ring depth: a power of two");
  extern __shared__ float ring[];  // [kD][kAcRingFields][kFB]
  __shared__ float s_S[kFB], s_vz[kFB];
  const int sl = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[sl]);
  const int z = blockIdx.x * a.tz - 8 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const int base = (int)(d.slot * sl);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld;
  const bool zin = z >= 0 && z < d.nzp;
  const bool zupd = z >= d.nop && z < d.nzp - d.nop;
  const bool z_int = z >= d.pml && z < d.nzp - d.pml;
  const bool vcol = t >= 4 && t < a.tz + 12 && zupd;
  const bool scol = t >= 8 && t < a.tz + 8 && zupd;
  const ShotDev sh = a.shots[sl];
  const float sval = kMode == 0 ? a.wavelet[a.it] : 0.f;
  const bool src_col = kMode == 0 && z == sh.isz;
  const float cx = d.dt / d.dx, cz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  const float *src[kAcRingFields] = {a.s, a.e_in, a.vx, a.vz, a.b, a.s, a.lam, a.m};
  auto R = [&](int q, int f) -> float & {
    return ring[((q & (kD - 1)) * kAcRingFields + f) * kFB + t];
  };
  auto used = [&](int f) {
    return !(f == 1 && kMode != 1) && !(f == 7 && (kMode != 0 || !a.e_out));
  };
  auto issue = [&](int q) {
#pragma unroll
    for (int f = 0; f < kAcRingFields; f++) {
      const int row = q - (f < 2 ? 0 : (f < 5 ? 4 : 8));
      if (!used(f)) continue;
      if (row >= 0 && row < d.nxp && zin)
        cp_async4(&R(q, f), src[f] + (base + row * ld + z));
      else
        R(q, f) = 0.f;
    }
    cp_async_commit();
  };

  float w_S[9], w_vx[9], w_vz[9];
#pragma unroll
  for (int i = 0; i < 9; i++) w_S[i] = w_vx[i] = w_vz[i] = 0.f;

#pragma unroll
  for (int j = 0; j < kD - 1; j++) issue(x0 - 8 + j);
  for (int r = x0 - 8; r < x1 + 8; r++) {
    cp_async_wait<kD - 2>();  // row r has landed (this thread's copies)
    float nS = R(r, 0);
    if (kMode == 1) nS += R(r, 1);
    if (src_col && r == sh.isx) nS += sval;  // FD2DGPU.cu:2039-2049 (transient)
    push(w_S, nS);
    issue(r + kD - 1);  // into the slot of row r - 1 (mod kD), finished last step
    // ---- velocities of row rv = r - 4 ----------------------------------------------------
    const int rv = r - 4;
    s_S[t] = w_S[4];
    __syncthreads();
    float vxn = 0.f, vzn = 0.f;
    if (vcol && r >= x0 && rv >= d.nop && rv < d.nxp - d.nop) {
      const int k = base + rv * ld + z;
      const float ax = dxp_mid(w_S);
      const float az = stencil4([&](int i) { return s_S[t + i] - s_S[t - i + 1]; });
      const float bb = R(r, 4);
      vxn = R(r, 2) + 1.0f * (bb * cx) * ax;  // k_ac_vel: v + dir (b dt/d) D+ S, dir = +1
      vzn = R(r, 3) + 1.0f * (bb * cz) * az;
      if (rv >= x0 && rv < x1 && t >= 8 && t < a.tz + 8) {
        a.vx_n[k] = vxn;
        a.vz_n[k] = vzn;
        if (kMode == 1 && z == sh.igz) {
          const int tr = a.rmap[(long long)sl * d.nxp_max + rv];
          if (tr >= 0) {
            const long long q = ((long long)sl * d.max_ntr + tr) * d.nt + a.it;
            a.rec_vz[q] = vzn;
            a.rec_vx[q] = vxn;
          }
        }
      }
    }
    push(w_vx, vxn);
    push(w_vz, vzn);
    // ---- stress of row rs = r - 8 --------------------------------------------------------
    const int rs = r - 8;
    s_vz[t] = w_vz[4];
    __syncthreads();
    if (scol && rs >= x0 && rs < x1 && rs >= d.nop && rs < d.nxp - d.nop) {
      const int k = base + rs * ld + z;
      const float sx = dxm_mid(w_vx);
      const float sz = stencil4([&](int i) { return s_vz[t + i - 1] - s_vz[t - i]; });
      const float lam = R(r, 6);
      a.s_n[k] = R(r, 5) + 1.0f * lam * (cx * sx + cz * sz);  // k_ac_str, dir = +1
      if (kMode == 0 && a.e_out && rs >= d.pml && rs < d.nxp - d.pml && z_int)
        a.e_out[k] = -2.0f * lam * R(r, 7) * (sx * rdx + sz * rdz);  // k_ac_born
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Reverse step of the acoustic L^T fed by the ring: the adjoint pair with the gradient and the
// exact reversal of the background, the fused counterpart of k_ac_adj_v, k_ac_adj_s, k_ac_str and
// k_ac_vel (direction -1) in that order, with the same arithmetic.  At row step r it
//   A. (row r-4)  y_v += residual; yx -= dt/dx Dx+(lam ys), yz -= dt/dz Dz+(lam ys);
//   B. (row r-8)  gs = -Dx-(b dt/dx yx) - Dz-(b dt/dz yz), ys += gs,
//                 grad += -2 lam (Dx- bvx / dx + Dz- bvz / dz) gs (interior),
//                 s -= lam (dt/dx Dx- bvx + dt/dz Dz- bvz)  (the same two derivatives);
//   C. (row r-12) v -= b dt/d D+(s + source)  with the reversed s of stage B.
// The three chained z-stencils need a 12-column halo on each side (kAcRevTZ output columns of
// 128 threads) and the rows a 10-row lead; both state sets ping-pong between two buffers.
// Ring fields of slot q: 0 ys, 1 lam of row q; 2 yx, 3 yz, 4 b, 5 bvx, 6 bvz of row q-4;
// 7 ys, 8 bs, 9 lam, 10 grad of row q-8; 11 b of row q-12.
// ---------------------------------------------------------------------------------------------
constexpr int kAcRevRingFields = 12;
constexpr int kAcRevTZ = kFB - 24;

struct AcRevArgs {
  Dims d;
  const ShotDev *shots;
  const float *yx, *yz, *ys;     // adjoint state (read)
  float *yx_n, *yz_n, *ys_n;     // adjoint state one step back (written)
  const float *vx, *vz, *s;      // background at step it (read)
  float *vx_n, *vz_n, *s_n;      // background at step it - 1 (written)
  const float *b, *lam;
  float *grad;                   // [slot][wnx][wnz] (wnx_max stride), accumulated
  const float *wavelet;
  int it, tz, xr;
  const int *rmap;
  const float *res_vz, *res_vx;  // [slot][max_ntr][nt]
  int *err;                      // pair kernel: error word (a ring wait that gave up)
};

template <int kD>
__global__ void __launch_bounds__(kFB, 4) k_ac_rev_ring(AcRevArgs a) {
  static_assert(kD >= 2 && kD <= 8 && (kD & (kD - 1)) == 0, "ring depth: 2, 4 or 8");
  constexpr int NF = kAcRevRingFields;
  extern __shared__ float ring[];  // [kD][NF][kFB]
  __shared__ float s_w[kFB], s_uz[kFB], s_bvz[kFB], s_S[kFB];
  // receiver column: trace index (16 stage-A rows ahead), residual (8 ahead) per row mod 16
  __shared__ int s_tr[16], s_has[16];
  __shared__ float s_rz[16], s_rx[16];
  const int sl = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[sl]);
  const int z = blockIdx.x * a.tz - 12 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  const int base = (int)(d.slot * sl);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld, pml = d.pml;
  const bool zin = z >= 0 && z < d.nzp;
  const bool zupd = z >= d.nop && z < d.nzp - d.nop;
  const bool z_int = z >= pml && z < d.nzp - pml;
  const bool colA = t >= 5 && t < a.tz + 19 && zupd;   // stage A: rows of the B halo
  const bool colB = t >= 9 && t < a.tz + 16 && zupd;   // stage B: the C halo
  const bool colC = t >= 12 && t < a.tz + 12 && zupd;  // stage C: own columns
  const bool ownB = t >= 12 && t < a.tz + 12;
  const ShotDev sh = a.shots[sl];
  const bool rec_col = z == sh.igz;
  const bool src_col = z == sh.isz;
  const float sval = a.wavelet[a.it];
  const float *res_z = a.res_vz + (long long)sl * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)sl * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)sl * d.nxp_max;
  const float cx = d.dt / d.dx, cz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  auto R = [&](int q, int f) -> float & { return ring[((q & (kD - 1)) * NF + f) * kFB + t]; };
  auto issue = [&](int q) {
    const int r0 = q, r4 = q - 4, r8 = q - 8, r12 = q - 12;
    const bool in0 = r0 >= 0 && r0 < d.nxp && zin;
    const bool in4 = r4 >= 0 && r4 < d.nxp && zin;
    const bool in8 = r8 >= 0 && r8 < d.nxp && zin;
    const bool in12 = r12 >= 0 && r12 < d.nxp && zin;
    const int o0 = base + r0 * ld + z, o4 = base + r4 * ld + z, o8 = base + r8 * ld + z;
    if (in0) {
      cp_async4(&R(q, 0), a.ys + o0);
      cp_async4(&R(q, 1), a.lam + o0);
    } else {
      R(q, 0) = R(q, 1) = 0.f;
    }
    if (in4) {
      cp_async4(&R(q, 2), a.yx + o4);
      cp_async4(&R(q, 3), a.yz + o4);
      cp_async4(&R(q, 4), a.b + o4);
      cp_async4(&R(q, 5), a.vx + o4);
      cp_async4(&R(q, 6), a.vz + o4);
    } else {
      R(q, 2) = R(q, 3) = R(q, 4) = R(q, 5) = R(q, 6) = 0.f;
    }
    if (in8) {
      cp_async4(&R(q, 7), a.ys + o8);
      cp_async4(&R(q, 8), a.s + o8);
      cp_async4(&R(q, 9), a.lam + o8);
      if (r8 >= pml && r8 < d.nxp - pml && z_int)
        cp_async4(&R(q, 10), a.grad + ((sl * d.wnx_max + (r8 - pml)) * d.ild + z));
    } else {
      R(q, 7) = R(q, 8) = R(q, 9) = 0.f;
    }
    if (in12) cp_async4(&R(q, 11), a.b + (base + r12 * ld + z)); else R(q, 11) = 0.f;
    cp_async_commit();
  };

  float w_w[9], w_ux[9], w_uz[5], w_bvx[9], w_bvz[9], w_S[9];
#pragma unroll
  for (int i = 0; i < 9; i++) w_w[i] = w_ux[i] = w_bvx[i] = w_bvz[i] = w_S[i] = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) w_uz[i] = 0.f;

  const int r_first = x0 - 10, r_last = x1 + 12;
#pragma unroll
  for (int j = 0; j < kD - 1; j++) issue(r_first + j);
  if (rec_col) {  // stage-A rows a = r - 4: trace indexes of the first 16, residuals of the first 8
    const int a0 = r_first - 4;
    for (int q = a0; q < a0 + 16; q++) s_tr[q & 15] = (q >= 0 && q < d.nxp) ? rmap[q] : -1;
    for (int q = a0; q < a0 + 8; q++) {
      const int tr = s_tr[q & 15];
      s_has[q & 15] = tr >= 0;
      if (tr >= 0) {
        s_rz[q & 15] = res_z[(long long)tr * d.nt];
        s_rx[q & 15] = res_x[(long long)tr * d.nt];
      }
    }
  }
  for (int r = r_first; r < r_last; r++) {
    cp_async_wait<kD - 2>();  // slot r has landed (this thread's copies)
    const int rA = r - 4, rB = r - 8, rC = r - 12;
    if (rec_col) {  // residual of stage-A row rA + 8, trace index of rA + 16 (landed in time)
      const int q8 = rA + 8, q16 = rA + 16;
      const int tr8 = s_tr[q8 & 15];
      s_has[q8 & 15] = tr8 >= 0;
      if (tr8 >= 0) {
        cp_async4(&s_rz[q8 & 15], res_z + (long long)tr8 * d.nt);
        cp_async4(&s_rx[q8 & 15], res_x + (long long)tr8 * d.nt);
      }
      if (q16 >= 0 && q16 < d.nxp)
        cp_async4((float *)&s_tr[q16 & 15], (const float *)(rmap + q16));
      else
        s_tr[q16 & 15] = -1;
    }
    push(w_w, R(r, 0) * R(r, 1));  // ys * lam  (k_ac_adj_v: lam[q] * ys[q])
    push(w_bvx, R(r, 5));           // background velocities of row rA (stage B window)
    push(w_bvz, R(r, 6));
    issue(r + kD - 1);
    // ---- A: adjoint velocities of row rA -------------------------------------------------------
    s_w[t] = w_w[4];
    __syncthreads();
    float uxn = 0.f, uzn = 0.f;
    if (rA >= 0 && rA < d.nxp && zin) {
      float yx = R(r, 2), yz = R(r, 3);
      if (colA && rA >= d.nop && rA < d.nxp - d.nop) {
        const float tx = dxp_mid(w_w);
        const float tzv = stencil4([&](int i) { return s_w[t + i] - s_w[t - i + 1]; });
        if (rec_col && s_has[rA & 15]) {
          yz += s_rz[rA & 15];
          yx += s_rx[rA & 15];
        }
        yx = yx - cx * tx;
        yz = yz - cz * tzv;
        if (ownB && rA >= x0 && rA < x1) {
          const int k = base + rA * ld + z;
          a.yx_n[k] = yx;
          a.yz_n[k] = yz;
        }
      }
      const float bb = R(r, 4);
      uxn = bb * cx * yx;  // k_ac_adj_s: b[q] * cx * yx[q]
      uzn = bb * cz * yz;
    }
    push(w_ux, uxn);
    push(w_uz, uzn);
    // ---- B: ys, gradient and the background stress of row rB ---------------------------------
    s_uz[t] = w_uz[0];  // 5-deep window: row rB is its oldest entry
    s_bvz[t] = w_bvz[4];
    __syncthreads();
    float Sn = 0.f;
    if (rB >= 0 && rB < d.nxp && zin) {
      float bs = R(r, 8);
      if (colB && rB >= d.nop && rB < d.nxp - d.nop) {
        const int k = base + rB * ld + z;
        const bool own = ownB && rB >= x0 && rB < x1;
        const float gx = dxm_mid(w_ux);
        const float gz = stencil4([&](int i) { return s_uz[t + i - 1] - s_uz[t - i]; });
        const float gs = -gx - gz;
        const float sx = dxm_mid(w_bvx);
        const float sz = stencil4([&](int i) { return s_bvz[t + i - 1] - s_bvz[t - i]; });
        const float lam = R(r, 9);
        if (own) {
          a.ys_n[k] = R(r, 7) + gs;
          if (rB >= pml && rB < d.nxp - pml && z_int) {
            const int o = (sl * d.wnx_max + (rB - pml)) * d.ild + z;
            a.grad[o] = R(r, 10) + -2.0f * lam * (sx * rdx + sz * rdz) * gs;
          }
        }
        bs = bs + -1.0f * lam * (cx * sx + cz * sz);  // k_ac_str, dir = -1
        if (own) a.s_n[k] = bs;
      }
      Sn = bs;
      if (src_col && rB == sh.isx) Sn += sval;  // the source overlay of k_ac_vel (transient)
    }
    push(w_S, Sn);
    // ---- C: background velocities of row rC ----------------------------------------------------
    s_S[t] = w_S[4];
    __syncthreads();
    if (colC && rC >= x0 && rC < x1 && rC >= d.nop && rC < d.nxp - d.nop) {
      const int k = base + rC * ld + z;
      const float ax = dxp_mid(w_S);
      const float az = stencil4([&](int i) { return s_S[t + i] - s_S[t - i + 1]; });
      const float bb = R(r, 11);
      a.vx_n[k] = w_bvx[0] + -1.0f * (bb * cx) * ax;  // k_ac_vel, dir = -1
      a.vz_n[k] = w_bvz[0] + -1.0f * (bb * cz) * az;
    }
  }
  cp_async_wait<0>();
}

}  // namespace ds2d
