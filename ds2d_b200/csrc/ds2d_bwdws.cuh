// Warp-specialised backward RTM step for sm_100a (random boundary): the computation of k_bwd_ring
// (interior reconstruction of the source wavefield, adjoint step with the receiver residual, and
// the imaging condition, FD2DGPU.cu:591-1082, 3235-3263, 3306-3322) with each wavefield given to
// its own warps.
//
// k_bwd_ring holds both wavefields' register windows (10 windows, 82 registers) in every thread,
// which limits it to 12 warps per SM, and its stalls are latency (fixed-latency dependencies and
// barriers), not DRAM.  Here a CTA of 2 kT threads marches the same z-strip with two roles: the
// first kT threads (the reconstruction warps) own the source field's windows, its ring fields
// and the illumination; the other kT threads (the adjoint warps) own the adjoint field's, the
// receiver staging and the two images.  Each thread carries half the windows, so twice the warps
// fit on an SM for the same register file, and each role copies only its own operands.  The one
// product that needs both fields -- the imaging condition at row r - 4, from the reconstruction's
// strains of its input state and the adjoint's new stresses -- goes through shared memory: the
// reconstruction warps store the four strains of the row before the step's second barrier, the
// adjoint warps read them after it.  Arithmetic per cell is k_bwd_ring's, expression for
// expression.
#pragma once
#include "ds2d_fused.cuh"

namespace ds2d {

// Ring fields per role (row q of ring slot q):
//   reconstruction: 0 vx(q) 1 vz(q) | 2 txx 3 tzz 4 txz 5 lam 6 mu (q-4) | 7 b 8 illumination (q-8)
//   adjoint:        0 vx(q) 1 vz(q) | 2 txx 3 tzz 4 txz 5 lam 6 mu 7 kpp 8 kps 9 img pp
//                   10 img ps (q-4) | 11 b (q-8)
constexpr int kWsFields = 12;  // per role (the reconstruction uses 9)
constexpr int kWsRing = 4;
__host__ __device__ constexpr size_t ws_smem(int kT) {
  return sizeof(float) * (size_t)kWsRing * 2 * kWsFields * kT;
}

template <int kT, int kMinB>
__global__ void __launch_bounds__(2 * kT, kMinB) k_bwd_ws(BwdFusedArgs a) {
  constexpr int kD = kWsRing, NF = kWsFields;
  extern __shared__ float ring[];  // [kD][2 roles][NF][kT]
  __shared__ float s_vx[kT], s_vz[kT];     // stage-1 z-tap rows of this role's velocities (r-4)
  __shared__ float s_avx[kT], s_avz[kT];
  __shared__ float s_t1[kT], s_t2[kT];     // stage-2 z-tap rows: btxz, btzz (reconstruction)
  __shared__ float s_m[kT], s_pzlx[kT];    //                     M, PzLx (adjoint)
  __shared__ float s_eps[4][kT];           // strains of row r-4: gx_vx, gz_vz, gz_vx, gx_vz
  __shared__ int s_tr[16], s_has[16];
  __shared__ float s_rz[16], s_rx[16], s_ownx[16], s_ownz[16];
  const int s = blockIdx.z;
  const bool adj = threadIdx.x >= kT;  // warp-uniform role
  const int t = adj ? threadIdx.x - kT : threadIdx.x;
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
  const bool rec_col = adj && z == sh.igz;
  const float *res_z = a.res_vz + (long long)s * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)s * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  const int img_row = s * d.wnx_max;  // image row of model row r: img_row + r - pml
  float *img_pp = a.img, *img_ps = a.img + a.img_plane, *img_il = a.img + 2 * a.img_plane;
  const Wave &src = adj ? a.aa : a.ra;
  auto R = [&](int q, int f) -> float & {
    return ring[(((q & (kD - 1)) * 2 + (adj ? 1 : 0)) * NF + f) * kT + t];
  };
  auto issue = [&](int q) {
    const int r0 = q, r4 = q - 4, r8 = q - 8;
    const bool in0 = r0 >= 0 && r0 < d.nxp && zin;
    const bool in4 = r4 >= 0 && r4 < d.nxp && zin;
    const bool in8 = r8 >= 0 && r8 < d.nxp && zin;
    const int o0 = base + r0 * ld + z, o4 = base + r4 * ld + z, o8 = base + r8 * ld + z;
    const bool int4 = in4 && r4 >= pml && r4 < d.nxp - pml && z_int;
    const bool int8 = in8 && r8 >= pml && r8 < d.nxp - pml && z_int;
    if (in0) {
      cp_async4(&R(q, 0), src.vx + o0);
      cp_async4(&R(q, 1), src.vz + o0);
    } else {
      R(q, 0) = R(q, 1) = 0.f;
    }
    if (in4) {
      cp_async4(&R(q, 2), src.txx + o4);
      cp_async4(&R(q, 3), src.tzz + o4);
      cp_async4(&R(q, 4), src.txz + o4);
      cp_async4(&R(q, 5), a.p.lam + o4);
      cp_async4(&R(q, 6), a.p.mu + o4);
      if (adj) {
        cp_async4(&R(q, 7), a.p.kpp + o4);
        cp_async4(&R(q, 8), a.p.kps + o4);
      }
    } else {
      R(q, 2) = R(q, 3) = R(q, 4) = R(q, 5) = R(q, 6) = 0.f;
    }
    if (adj) {
      if (int4) {
        const int io = (img_row + r4 - pml) * d.ild + z;
        cp_async4(&R(q, 9), img_pp + io);
        cp_async4(&R(q, 10), img_ps + io);
      } else {
        R(q, 9) = R(q, 10) = 0.f;
      }
      if (in8) cp_async4(&R(q, 11), a.p.b + o8); else R(q, 11) = 0.f;
    } else {
      if (in8) cp_async4(&R(q, 7), a.p.b + o8); else R(q, 7) = 0.f;
      if (int8)
        cp_async4(&R(q, 8), img_il + ((img_row + r8 - pml) * d.ild + z));
      else
        R(q, 8) = 0.f;
    }
    cp_async_commit();
  };

  // Windows of this role.  Reconstruction: w_v = vx, w_u = vz of the input state; w_a = txx,
  // w_b = txz, w_c (5) = tzz of its new stresses.  Adjoint: w_v = vx, w_u = vz; w_a = PL, w_b = M,
  // w_c (5) = PzLx (the adjoint velocity update's operands, see k_bwd_ring).
  float w_v[9], w_u[9], w_a[9], w_b[9], w_c[5];
#pragma unroll
  for (int i = 0; i < 9; i++) w_v[i] = w_u[i] = w_a[i] = w_b[i] = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) w_c[i] = 0.f;

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
      // residual of row r + 8 and trace index of row r + 16, copied with this step's group
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
    {
      float n_vx = R(r, 0), n_vz = R(r, 1);
      if (rec_col && r >= 0 && r < d.nxp && zin) {
        s_ownx[r & 15] = n_vx;
        s_ownz[r & 15] = n_vz;
        if (s_has[r & 15]) {
          n_vz += s_rz[r & 15];
          n_vx += s_rx[r & 15];
        }
      }
      push(w_v, n_vx);
      push(w_u, n_vz);
    }
    issue(r + kD - 1);  // refill the slot of row r - 1 (mod kD) with row r + kD - 1
    // ---- stage 1: stresses of row r1 = r - 4 -----------------------------------------------
    const int r1 = r - 4;
    if (adj) {
      s_avx[t] = w_v[4];
      s_avz[t] = w_u[4];
    } else {
      s_vx[t] = w_v[4];
      s_vz[t] = w_u[4];
    }
    __syncthreads();
    float o_a = 0.f, o_b = 0.f, o_c = 0.f;  // windows' new entries
    float atxx = 0.f, atzz = 0.f, atxz = 0.f;
    const bool st1 = c1 && zin && r >= x0 && r1 >= 0 && r1 < d.nxp;
    const bool own1 = c2 && r1 >= x0 && r1 < x1;
    const bool x_int1 = r1 >= pml && r1 < d.nxp - pml;
    if (!adj) {
      float btxx = 0.f, btzz = 0.f, btxz = 0.f;
      float gx_vx = 0.f, gz_vz = 0.f, gz_vx = 0.f, gx_vz = 0.f;
      if (st1) {
        const int k = base + r1 * ld + z;
        btxx = R(r, 2);
        btzz = R(r, 3);
        btxz = R(r, 4);
        const float lam = R(r, 5), mu = R(r, 6);
        if (x_int1 && z_int) {
          const float sa = dxm_mid(w_v);
          const float sf = dxp_mid(w_u);
          const float sb = stencil4([&](int i) { return s_vz[t + i - 1] - s_vz[t - i]; });
          const float se = stencil4([&](int i) { return s_vx[t + i] - s_vx[t - i + 1]; });
          const float l2m = lam + 2.0f * mu;
          const float dir = -1.0f;
          btxx = btxx + (dir * l2m * dtdx * sa + dir * lam * dtdz * sb);
          btzz = btzz + (dir * lam * dtdx * sa + dir * l2m * dtdz * sb);
          btxz = btxz + (dir * mu * dtdx * sf + dir * mu * dtdz * se);
          gx_vx = sa * rdx;
          gz_vz = sb * rdz;
          gz_vx = se * rdz;
          gx_vz = sf * rdx;
          if (own1) {
            a.rb.txx[k] = btxx;
            a.rb.tzz[k] = btzz;
            a.rb.txz[k] = btxz;
          }
        }
      }
      s_eps[0][t] = gx_vx;
      s_eps[1][t] = gz_vz;
      s_eps[2][t] = gz_vx;
      s_eps[3][t] = gx_vz;
      o_a = btxx;
      o_b = btxz;
      o_c = btzz;
    } else if (st1) {
      const int k = base + r1 * ld + z;
      const float lam = R(r, 5), mu = R(r, 6);
      if (r1 >= d.nop && r1 < d.nxp - d.nop && z_upd) {
        const float sa = dxm_mid(w_v);
        const float sf = dxp_mid(w_u);
        const float sb = stencil4([&](int i) { return s_avz[t + i - 1] - s_avz[t - i]; });
        const float se = stencil4([&](int i) { return s_avx[t + i] - s_avx[t - i + 1]; });
        const float xx = -dtdx * sa, zz = -dtdz * sb, xz_x = -dtdx * sf, xz_z = -dtdz * se;
        atxx = R(r, 2) + xx;
        atzz = R(r, 3) + zz;
        atxz = R(r, 4) + (xz_x + xz_z);
        if (own1) {
          a.ab.txx[k] = atxx;
          a.ab.tzz[k] = atzz;
          a.ab.txz[k] = atxz;
        }
      }
      const float l2m = lam + 2.0f * mu;
      o_a = l2m * atxx + lam * atzz;  // PL
      o_b = mu * atxz;                // M
      o_c = l2m * atzz + lam * atxx;  // PzLx
    }
    push(w_a, o_a);
    push(w_b, o_b);
    push(w_c, o_c);
    // ---- stage 2: velocities of row r2 = r - 8 ---------------------------------------------
    const int r2 = r - 8;
    if (adj) {
      s_m[t] = w_b[4];
      s_pzlx[t] = w_c[0];
    } else {
      s_t1[t] = w_b[4];
      s_t2[t] = w_c[0];
    }
    __syncthreads();
    if (adj && st1 && own1 && x_int1 && z_int) {
      // imaging condition of row r1 (doimage_gradient, FD2DGPU.cu:3245): the reconstruction's
      // strains of its input state with the new adjoint stresses
      const int o = (img_row + (r1 - pml)) * d.ild + z;
      const float gx_vx = s_eps[0][t], gz_vz = s_eps[1][t], gz_vx = s_eps[2][t],
                  gx_vz = s_eps[3][t];
      const float kpp = R(r, 7), kps = R(r, 8);
      const float lamda_grad = (gx_vx + gz_vz) * (atxx + atzz);
      const float miu_grad = -2.0f * (gx_vx * atzz + gz_vz * atxx) + (gz_vx + gx_vz) * atxz;
      img_pp[o] = R(r, 9) + kpp * lamda_grad;
      img_ps[o] = R(r, 10) + kps * miu_grad;
    }
    if (c2 && zin && r2 >= x0 && r2 < x1) {
      const int k = base + r2 * ld + z;
      if (!adj) {
        const bool x_int = r2 >= pml && r2 < d.nxp - pml;
        const float bb = R(r, 7);
        const float cbx = bb * dtdx, cbz = bb * dtdz;
        if (x_int && z_int) {
          const float ax = dxp_mid(w_a);
          const float fx = dxm_mid(w_b);
          const float bz = stencil4([&](int i) { return s_t1[t + i - 1] - s_t1[t - i]; });
          const float ez = stencil4([&](int i) { return s_t2[t + i] - s_t2[t - i + 1]; });
          const float vx = w_v[0] + (-cbx * ax + -cbz * bz);
          const float vz = w_u[0] + (-cbx * fx + -cbz * ez);
          a.rb.vx[k] = vx;
          a.rb.vz[k] = vz;
          const int o = (img_row + (r2 - pml)) * d.ild + z;
          img_il[o] = R(r, 8) + (vx * vx + vz * vz);
        }
      } else if (r2 >= d.nop && r2 < d.nxp - d.nop && z_upd) {
        const float bb = R(r, 11);
        const float cbx = bb * dtdx, cbz = bb * dtdz;
        const float t_x = dxp_mid(w_a);
        const float s_xz = dxm_mid(w_b);
        const float t_xz = stencil4([&](int i) { return s_m[t + i - 1] - s_m[t - i]; });
        const float s_z = stencil4([&](int i) { return s_pzlx[t + i] - s_pzlx[t - i + 1]; });
        const float ux_x = -cbx * t_x, ux_z = -cbz * t_xz;
        const float uz_x = -cbx * s_xz, uz_z = -cbz * s_z;
        float ovx = w_v[0], ovz = w_u[0];
        if (rec_col) {  // receiver column: the state without the residual
          ovx = s_ownx[r2 & 15];
          ovz = s_ownz[r2 & 15];
        }
        a.ab.vx[k] = ovx + (ux_x + ux_z);
        a.ab.vz[k] = ovz + (uz_x + uz_z);
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace ds2d
