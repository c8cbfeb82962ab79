// Backward RTM step of k_bwd_ring (random boundary) with its operand rows fed by bulk copies.
//
// The one-column backward step executes most of its instructions on per-row work rather than on
// the stencils: every thread issues its own 18 cp.async copies a row step (addresses, range
// predicates, zero stores for rows outside the window) and waits on its own commit groups.  Here
// one cp.async.bulk per field row copies it for the whole CTA (global -> shared, completion
// counted on the ring slot's mbarrier), as in the pair kernels of ds2d_pair.cuh, and every
// thread waits on the slot's phase (bounded by device time; a wait that gives up raises the error word and the CTA leaves the
// march together).  The ring layout, the stages and the arithmetic are k_bwd_ring's, expression
// for expression; rows outside the window are skipped rather than zeroed, because no update
// reads them (the stencils of updated rows stay inside the grid, and imaging rows inside the
// interior).  kOne: one barrier per row step (all eight z-tap rows published at the top of the
// step, into one of two buffers), as k_bwd_ring's kOne.  The copies of a slot are spread over
// all warps of the CTA (warp w issues the fields f with f mod W = w, W warps; every warp arrives
// on the slot's barrier with its own bytes), so no warp carries a step's whole copy issue.
//
// z-strips: strip j owns columns [zs, zs + tz), zs = j tz; its CTA's threads cover them plus the
// 8 halo columns of each side that borders another strip (none at the grid's edges, where the
// columns beyond are zero), from c0 = zs - 8 (or 0 for the first strip).  tz is a multiple of 4,
// so every copy row starts on a 16-byte boundary (copies are clipped to the row's allocation
// [0, ld)).  Without halo columns at the edges, 2 strips of 256 threads cover a 481-deep grid
// (512 threads for 481 columns, 128 registers: 16 warps per SM).
#pragma once
#include "ds2d_pair.cuh"

namespace ds2d {

constexpr int kBulkRing = 4;
constexpr int kBwdBulkFields = 18;
__host__ __device__ constexpr size_t bwd_bulk_smem(int kT) {
  return sizeof(float) * (size_t)kBulkRing * kBwdBulkFields * kT + 8 * kBulkRing;
}

// Copies of one ring slot for one-column CTAs, by one warp: its lane owning ring field f (row
// q - lag of its array if that row lies in [lo, hi)) copies it; the CTA's columns
// [c0, c0 + kT) map to ring floats 0 .. kT, clipped to [0, ld).  Lane 0 arrives on the slot's
// barrier with the bytes of the warp's copies before any is issued.
template <int kT>
__device__ __forceinline__ void issue_slot_col(const RingField &fd, float *slot_base, int f,
                                               unsigned long long *bar, int q, int ld, int c0,
                                               int lane) {
  const int glo = max(0, c0), ghi = min(ld, c0 + kT);
  const unsigned bytes = (unsigned)(ghi - glo) * 4u;
  const int row = q - fd.lag;
  const bool mine = fd.src != nullptr && row >= fd.lo && row < fd.hi;
  const unsigned n = __popc(__ballot_sync(0xffffffffu, mine));
  if (lane == 0) mbar_arrive_tx(bar, n * bytes);
  __syncwarp();
  if (mine)
    bulk_g2s(slot_base + f * kT + (glo - c0), fd.src + (long long)row * ld + glo, bytes, bar);
}

template <int kT, int kMinB, bool kOne>
__global__ void __launch_bounds__(kT, kMinB) k_bwd_bulk(BwdFusedArgs a) {
  constexpr int kD = kBulkRing, NF = kBwdBulkFields;
  extern __shared__ __align__(16) float ring[];  // [kD][NF][kT], then the slot barriers
  unsigned long long *bars = (unsigned long long *)(ring + (size_t)kD * NF * kT);
  // z-tap rows: bvx bvz avx avz (stage 1), btxz btzz M PzLx (stage 2); two buffers with kOne
  __shared__ float s_zt[kOne ? 2 : 1][8][kT];
  __shared__ int s_tr[16], s_has[16];
  __shared__ float s_rz[16], s_rx[16], s_ownx[16], s_ownz[16];
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int zs = blockIdx.x * a.tz;
  const int c0 = zs > 0 ? zs - 8 : 0;  // first column of the CTA: 8 halo columns inside the grid
  const int z = c0 + t;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  if (__syncthreads_or(t == 0 && pair_err_raised(a.err))) return;  // whole CTA
  const int base = (int)(d.slot * s);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld, pml = d.pml;
  const bool zin = z >= 0 && z < d.nzp;
  const bool c1 = z >= zs - 4 && z < zs + a.tz + 4;  // stage-1 columns: the strip and 4 each side
  const bool c2 = z >= zs && z < zs + a.tz;          // stage-2 columns: the strip
  const bool z_int = z >= pml && z < d.nzp - pml;
  const bool z_upd = z >= d.nop && z < d.nzp - d.nop;
  const ShotDev sh = a.shots[s];
  const bool rec_col = z == sh.igz;
  const float *res_z = a.res_vz + (long long)s * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)s * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  const int img_row = s * d.wnx_max;  // image row of model row r: img_row + r - pml
  float *img_pp = a.img, *img_ps = a.img + a.img_plane, *img_il = a.img + 2 * a.img_plane;

  // ring field of this lane: warp w, lane l owns field f = w + W l (W warps); the per-slot images
  // share the wavefields' row stride (ild == ld), model row x at image row x - pml
  constexpr int W = kT / 32;
  const int lane = t & 31;
  const int my_f = (t >> 5) + W * lane;
  RingField fd{nullptr, 0, 0, d.nxp};
  {
    const long long fbase = d.slot * s;
    const long long ibase = (long long)s * d.wnx_max * d.ild - (long long)pml * ld;
    const float *src[NF] = {a.ra.vx,  a.ra.vz,  a.aa.vx,  a.aa.vz,  a.ra.txx, a.ra.tzz,
                            a.ra.txz, a.aa.txx, a.aa.tzz, a.aa.txz, a.p.lam,  a.p.mu,
                            a.p.kpp,  a.p.kps,  img_pp,   img_ps,   a.p.b,    img_il};
#pragma unroll
    for (int f = 0; f < NF; f++)
      if (my_f == f) {
        const bool img = f == 14 || f == 15 || f == 17;
        fd.src = src[f] + (img ? ibase : fbase);
        fd.lag = f < 4 ? 0 : (f < 16 ? 4 : 8);
        fd.lo = img ? pml : 0;
        fd.hi = img ? d.nxp - pml : d.nxp;
      }
  }
  if (t == 0) {
    for (int k = 0; k < kD; k++) mbar_init(&bars[k], W);  // one arrival per warp and phase
    mbar_fence_init();
  }
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
  __syncthreads();
  const int rs0 = x0 - 8;
  for (int j = 0; j < kD - 1; j++)
    issue_slot_col<kT>(fd, ring + (size_t)j * NF * kT, my_f, &bars[j], rs0 + j, ld, c0, lane);

  float w_bvx[9], w_bvz[9], w_avx[9], w_avz[9];
  // adjoint-velocity operands, as k_bwd_ring: PL = (l+2m) atxx + l atzz, PzLx = (l+2m) atzz + l atxx
  float w_btxx[9], w_btxz[9], w_btzz[5], w_PL[9], w_M[9], w_PzLx[5];
#pragma unroll
  for (int i = 0; i < 9; i++)
    w_bvx[i] = w_bvz[i] = w_avx[i] = w_avz[i] = w_btxx[i] = w_btxz[i] = w_PL[i] = w_M[i] = 0.f;
#pragma unroll
  for (int i = 0; i < 5; i++) w_btzz[i] = w_PzLx[i] = 0.f;

  RingCursor<kD> cur;
  bool ok = true, aborted = false;
#pragma unroll kRingUnrollBwd
  for (int r = rs0; r < x1 + 8; r++) {
    // A wait that gives up skips the step's reads; the barrier below is a vote, so every thread
    // leaves the march together.
    ok = mbar_wait(&bars[cur.slot], cur.phase);
    const float *S = ring + (size_t)cur.slot * NF * kT + t;
    if (rec_col) {
      // residual of row r + 8 and trace index of row r + 16, one commit group per step (landed
      // before either is read, cp_async_wait<7> at the end of each step)
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
      cp_async_commit();
    }
    {
      float n_bvx = 0.f, n_bvz = 0.f, n_avx = 0.f, n_avz = 0.f;
      if (ok) {
        n_bvx = S[0 * kT];
        n_bvz = S[1 * kT];
        n_avx = S[2 * kT];
        n_avz = S[3 * kT];
      }
      if (rec_col && r >= 0 && r < d.nxp && zin) {
        s_ownx[r & 15] = n_avx;
        s_ownz[r & 15] = n_avz;
        if (s_has[r & 15]) {
          n_avz += s_rz[r & 15];
          n_avx += s_rx[r & 15];
        }
      }
      push(w_bvx, n_bvx);
      push(w_bvz, n_bvz);
      push(w_avx, n_avx);
      push(w_avz, n_avz);
    }
    const int r1 = r - 4;
    float *const zb = s_zt[kOne ? (r & 1) : 0][0];
    float *const s_bvx = zb, *const s_bvz = zb + kT, *const s_avx = zb + 2 * kT;
    float *const s_avz = zb + 3 * kT, *const s_btxz = zb + 4 * kT, *const s_btzz = zb + 5 * kT;
    float *const s_m = zb + 6 * kT, *const s_pzlx = zb + 7 * kT;
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
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    // every thread is done with the previous slot: refill it kD - 1 steps ahead
    {
      const int ps = cur.slot == 0 ? kD - 1 : cur.slot - 1;
      issue_slot_col<kT>(fd, ring + (size_t)ps * NF * kT, my_f, &bars[ps], r + kD - 1, ld, c0,
                         lane);
    }
    // ---- stage 1: stresses of row r1 = r - 4 -----------------------------------------------
    float btxx = 0.f, btzz = 0.f, btxz = 0.f, PL = 0.f, M = 0.f, PzLx = 0.f;
    if (c1 && zin && r >= x0 && r1 >= 0 && r1 < d.nxp) {
      const int k = base + r1 * ld + z;
      const bool own = c2 && r1 >= x0 && r1 < x1;
      btxx = S[4 * kT];
      btzz = S[5 * kT];
      btxz = S[6 * kT];
      const bool x_int = r1 >= pml && r1 < d.nxp - pml;
      float gx_vx = 0.f, gz_vz = 0.f, gz_vx = 0.f, gx_vz = 0.f;
      const float lam = S[10 * kT], mu = S[11 * kT];
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
        gx_vx = sa * rdx;  // strains; reciprocal multiply
        gz_vz = sb * rdz;
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
        atxx = S[7 * kT] + xx;
        atzz = S[8 * kT] + zz;
        atxz = S[9 * kT] + (xz_x + xz_z);
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
        const float kpp = S[12 * kT], kps = S[13 * kT];
        const float lamda_grad = (gx_vx + gz_vz) * (atxx + atzz);
        const float miu_grad = -2.0f * (gx_vx * atzz + gz_vz * atxx) + (gz_vx + gx_vz) * atxz;
        img_pp[o] = S[14 * kT] + kpp * lamda_grad;
        img_ps[o] = S[15 * kT] + kps * miu_grad;
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
      const float bb = S[16 * kT];
      const float cbx = bb * dtdx, cbz = bb * dtdz;
      if (x_int && z_int) {
        const float ax = dxp_mid(w_btxx);
        const float fx = dxm_mid(w_btxz);
        const float bz = stencil4([&](int i) { return s_btxz[t + i - 1] - s_btxz[t - i]; });
        const float ez = stencil4([&](int i) { return s_btzz[t + i] - s_btzz[t - i + 1]; });
        const float vx = w_bvx[0] + (-cbx * ax + -cbz * bz);
        const float vz = w_bvz[0] + (-cbx * fx + -cbz * ez);
        a.rb.vx[k] = vx;
        a.rb.vz[k] = vz;
        const int o = (img_row + (r2 - pml)) * d.ild + z;
        img_il[o] = S[17 * kT] + (vx * vx + vz * vz);
      }
      if (r2 >= d.nop && r2 < d.nxp - d.nop && z_upd) {
        const float t_x = dxp_mid(w_PL);
        const float s_xz = dxm_mid(w_M);
        const float t_xz = stencil4([&](int i) { return s_m[t + i - 1] - s_m[t - i]; });
        const float s_z = stencil4([&](int i) { return s_pzlx[t + i] - s_pzlx[t - i + 1]; });
        const float ux_x = -cbx * t_x, ux_z = -cbz * t_xz;
        const float uz_x = -cbx * s_xz, uz_z = -cbz * s_z;
        float ovx = w_avx[0], ovz = w_avz[0];
        if (rec_col) {  // receiver column: the state without the residual
          ovx = s_ownx[r2 & 15];
          ovz = s_ownz[r2 & 15];
        }
        a.ab.vx[k] = ovx + (ux_x + ux_z);
        a.ab.vz[k] = ovz + (uz_x + uz_z);
      }
    }
    if (rec_col) cp_async_wait<7>();
    cur.advance();
  }
  pair_exit<kD>(bars, cur, aborted, ok, a.err);
  cp_async_wait<0>();
}

}  // namespace ds2d
