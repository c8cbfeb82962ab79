// Time-blocked forward step for sm_100a: one launch advances every resident shot by kK time
// steps (random boundary: no PML cells, no strips).
//
// Same x-march as k_fwd_ring (a CTA owns a z-strip, walks its rows along x, operands prefetched
// global -> shared by a per-thread cp.async ring), with the stages of kK time steps chained in
// one pass: at row step r, stage V_k updates the velocities of row r - 4 - 8k to time t + k + 1
// and stage S_k the stresses of row r - 8 - 8k.  V_0 reads the stresses of time t from memory;
// every later stage reads the output rows of the stage before it from per-thread register
// windows (x-taps) and from shared z-tap rows, so the intermediate time levels never leave the
// SM.  Only the state of time t + kK is written (ping-pong a -> b), and every parameter row is
// read from L2 once per stage.  DRAM bytes per cell-update fall from 52 to 52 / kK; the price is
// a halo that grows with kK (8 kK rows at each end of a CTA's x-range, 8 kK columns at each
// inner edge of a z-strip, recomputed) and kK sets of windows (45 registers each).
//
// Every z-tap row a step needs was computed at least four row steps earlier (V_k's taps at row
// r - 4 - 8k come from S_{k-1}'s output of step r - 4, S_k's at row r - 8 - 8k from V_k's of
// step r - 4), so all of them are copied into shared memory at the top of the step, into one of
// two buffers, and ONE barrier per row step publishes them (double buffering keeps a thread that
// runs ahead from overwriting rows another thread still reads).  Within a step the stages depend
// on one another only through the newest window entries (registers of the same thread).
//
// Strip geometry: z-strip j owns columns [j tz, j tz + tz); its threads cover those plus 8 kK
// halo columns on each side that borders another strip (none at the grid's edges, where the
// columns beyond are zero), so a kT-thread CTA owns up to kT - 16 kK columns (kT - 8 kK at an
// edge, kT when one strip covers the whole depth).
//
// kBulk: the operand rows arrive by bulk copy instead of per-thread cp.async -- one
// cp.async.bulk per field row for the whole CTA into the same ring layout, the copies of a slot
// spread over all warps (warp w issues the fields f with f mod W = w and arrives on the slot's
// mbarrier with its own bytes), every thread waiting (bounded) on the slot's phase, the slot of
// step r - 1 refilled after the step's barrier.  Rows outside the window are skipped, not
// zeroed: no updated row reads them.  A strip's first column is then a multiple of 4 (16-byte
// aligned copy rows).
//
// Injections are the one-step kernels': the explosive source of time t + k (FD2DGPU.cu:2039-2049)
// is added to the stress values that enter V_k (window entry and z-tap copy); the injected cell
// keeps its un-injected stresses in registers for S_k.  Receivers record the V_k output of rows
// and columns the CTA owns at time index it + k.  Results are bit-identical to kK launches of
// k_fwd_ring.
#pragma once
#include "ds2d_pair.cuh"

namespace ds2d {

// Ring fields of row step q: 0 txx, 1 tzz, 2 txz of row q; 3 vx, 4 vz of row q - 4; then b of
// row q - 4 - 8k (k < kK) and lam, mu of row q - 8 - 8k (k < kK).
__host__ __device__ constexpr int tb_fields(int K) { return 5 + 3 * K; }
constexpr int kTbRing = 4;   // ring depth
constexpr int kTbPad = 4;    // zero floats on each side of a shared z-tap row
__host__ __device__ constexpr int tb_row(int kT) { return kT + 2 * kTbPad; }
// Dynamic shared memory: the ring, two buffers of 4 kK z-tap rows, the trace indexes of the
// CTA's rows (xr ints).
__host__ __device__ constexpr size_t tb_smem(int K, int kT, int xr) {
  return sizeof(float) * ((size_t)kTbRing * tb_fields(K) * kT + 2 * 4 * K * tb_row(kT)) +
         (sizeof(int) * (size_t)xr + 7) / 8 * 8 + 8 * kTbRing;  // + the slot barriers (kBulk)
}

// One warp's share of the bulk copies of a ring slot: the lane owning ring field f copies row
// q - lag of its array (if that row lies in [lo, hi)) over the strip columns [c0, c0 + kT),
// clipped to the row's allocation [0, ld), into ring floats 0 .. kT; lane 0 arrives on the
// slot's barrier with the bytes of the warp's copies first.
template <int kT>
__device__ __forceinline__ void tb_issue_warp(const RingField &fd, float *slot_base, int f,
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

template <int K>
struct TbWin {
  float txx[K][9], tzz[K][9], txz[K][9];  // stresses entering V_k (k = 0: time t from memory)
  float vx[K][9], vz[K][9];               // V_k outputs entering S_k
};

template <int kK, int kT, int kMinB, bool kBulk = false>
__global__ void __launch_bounds__(kT, kMinB) k_fwd_tb(FwdFusedArgs a) {
  constexpr int kD = kTbRing, NF = tb_fields(kK), ROW = tb_row(kT);
  constexpr int H = 8 * kK;  // halo columns at an inner strip edge, halo rows at each x end
  extern __shared__ __align__(16) float smem[];
  float *ring = smem;                          // [kD][NF][kT]
  float *ztap = ring + (size_t)kD * NF * kT;   // [2][4 kK][ROW]
  int *s_tr = (int *)(ztap + 2 * 4 * kK * ROW);  // [xr] trace index of row x0 + i, or -1
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(  // [kD] slot barriers (kBulk)
      (char *)smem + ((size_t)((char *)(s_tr + a.xr) - (char *)smem) + 7) / 8 * 8);
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int zs = blockIdx.x * a.tz, ze = min(zs + a.tz, d.nzp);
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  if (kBulk && __syncthreads_or(t == 0 && pair_err_raised(a.err))) return;  // whole CTA
  const int hl = zs > 0 ? H : 0;
  const int z = zs - hl + t;
  const int base = (int)(d.slot * s);  // cell offsets fit 32 bits (checked on the host)
  const int ld = d.ld, nop = d.nop;
  const bool zin = z >= 0 && z < d.nzp;
  const bool zupd = z >= nop && z < d.nzp - nop;
  const bool zown = z >= zs && z < ze;
  const ShotDev sh = a.shots[s];
  const bool src_col = z == sh.isz;
  const bool rec_col = a.rec_on && zown && z == sh.igz;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  // z-range of stage V_k / S_k (columns whose outputs a later stage or the owner needs)
  auto vcol = [&](int k) {
    const int h = 4 + 8 * (kK - 1 - k);
    return zupd && z >= zs - h && z < ze + h;
  };
  auto scol = [&](int k) {
    const int h = 8 * (kK - 1 - k);
    return zupd && z >= zs - h && z < ze + h;
  };
  auto R = [&](int q, int f) -> float & { return ring[((q & (kD - 1)) * NF + f) * kT + t]; };
  auto issue = [&](int q) {
    const int o = base + z;
    if (zin && q >= 0 && q < d.nxp) {
      cp_async4(&R(q, 0), a.a.txx + o + q * ld);
      cp_async4(&R(q, 1), a.a.tzz + o + q * ld);
      cp_async4(&R(q, 2), a.a.txz + o + q * ld);
    } else {
      R(q, 0) = R(q, 1) = R(q, 2) = 0.f;
    }
    const int r4 = q - 4;
    if (zin && r4 >= 0 && r4 < d.nxp) {
      cp_async4(&R(q, 3), a.a.vx + o + r4 * ld);
      cp_async4(&R(q, 4), a.a.vz + o + r4 * ld);
    } else {
      R(q, 3) = R(q, 4) = 0.f;
    }
#pragma unroll
    for (int k = 0; k < kK; k++) {
      const int rb = q - 4 - 8 * k, rl = q - 8 - 8 * k;
      if (zin && rb >= 0 && rb < d.nxp) cp_async4(&R(q, 5 + k), a.p.b + o + rb * ld);
      if (zin && rl >= 0 && rl < d.nxp) {
        cp_async4(&R(q, 5 + kK + 2 * k), a.p.lam + o + rl * ld);
        cp_async4(&R(q, 6 + kK + 2 * k), a.p.mu + o + rl * ld);
      }
    }
    cp_async_commit();
  };
  // kBulk: ring field of this thread (warp w, lane l owns field w + W l) and the slot barriers
  const int lane = t & 31;
  const int my_f = (t >> 5) + (kT / 32) * lane;
  RingField fd{nullptr, 0, 0, d.nxp};
  if (kBulk) {
    const long long fbase = d.slot * s;
#pragma unroll
    for (int f = 0; f < NF; f++)
      if (my_f == f) {
        const float *src = f == 0 ? a.a.txx : f == 1 ? a.a.tzz : f == 2 ? a.a.txz
                         : f == 3 ? a.a.vx : f == 4 ? a.a.vz
                         : f < 5 + kK ? a.p.b : ((f - 5 - kK) & 1) ? a.p.mu : a.p.lam;
        fd.src = src + fbase;
        fd.lag = f < 3 ? 0 : f < 5 ? 4 : f < 5 + kK ? 4 + 8 * (f - 5) : 8 + 8 * ((f - 5 - kK) >> 1);
      }
    if (t == 0) {
      for (int k = 0; k < kD; k++) mbar_init(&bars[k], kT / 32);  // one arrival per warp
      mbar_fence_init();
    }
  }
  const int c0 = zs - hl;  // first column of the CTA (a multiple of 4 with kBulk)

  // trace indexes of the CTA's own rows (receiver column only reads them; everyone copies)
  if (a.rec_on) {
    const int *rmap = a.rmap + (long long)s * d.nxp_max;
    for (int i = t; i < x1 - x0; i += kT) s_tr[i] = rmap[x0 + i];
  }
  // zero the pads of the z-tap rows (read only by columns that are never updated)
  for (int i = t; i < 2 * 4 * kK; i += kT) {
#pragma unroll
    for (int p = 0; p < kTbPad; p++) {
      ztap[i * ROW + p] = 0.f;
      ztap[i * ROW + kTbPad + kT + p] = 0.f;
    }
  }

  TbWin<kK> w;
#pragma unroll
  for (int k = 0; k < kK; k++)
#pragma unroll
    for (int i = 0; i < 9; i++)
      w.txx[k][i] = w.tzz[k][i] = w.txz[k][i] = w.vx[k][i] = w.vz[k][i] = 0.f;
  // un-injected stresses of the source cell, per stage (the windows carry the source)
  float own_txx[kK], own_tzz[kK];
#pragma unroll
  for (int k = 0; k < kK; k++) own_txx[k] = own_tzz[k] = 0.f;
  __syncthreads();

  const int r_begin = x0 - H, r_end = x1 + H;
  if (kBulk) {
    for (int j = 0; j < kD - 1; j++)
      tb_issue_warp<kT>(fd, ring + (size_t)j * NF * kT, my_f, &bars[j], r_begin + j, ld, c0, lane);
  } else {
#pragma unroll
    for (int j = 0; j < kD - 1; j++) issue(r_begin + j);
  }
  RingCursor<kD> cur;  // kBulk: slot and phase of the step being consumed
  bool ok = true, aborted = false;
  // two row steps per iteration let the compiler rename half of the window shifts away
  constexpr int kUnroll = kK <= 2 ? 2 : 1;
#pragma unroll kUnroll
  for (int r = r_begin; r < r_end; r++) {
    // row step r has landed: this thread's copies, or (kBulk) the slot's phase, bounded
    if (kBulk)
      ok = mbar_wait(&bars[cur.slot], cur.phase);
    else
      cp_async_wait<kD - 2>();
    const float *S = ring + (size_t)(kBulk ? cur.slot : (r & (kD - 1))) * NF * kT + t;
    {
      float n_txx = S[0], n_tzz = S[kT];
      const float n_txz = S[2 * kT];
      if (src_col && r == sh.isx) {  // FD2DGPU.cu:2039-2049 (transient)
        own_txx[0] = n_txx;
        own_tzz[0] = n_tzz;
        const float sv = a.wavelet[a.it];
        n_txx += sv;
        n_tzz += sv;
      }
      push(w.txx[0], n_txx);
      push(w.tzz[0], n_tzz);
      push(w.txz[0], n_txz);
    }
    // own operands of this step (read before the refill below can reuse ring slots)
    const float ovx0 = S[3 * kT], ovz0 = S[4 * kT];
    float bb[kK], lam[kK], mu[kK];
#pragma unroll
    for (int k = 0; k < kK; k++) {
      bb[k] = S[(5 + k) * kT];
      lam[k] = S[(5 + kK + 2 * k) * kT];
      mu[k] = S[(6 + kK + 2 * k) * kT];
    }
    if (!kBulk) issue(r + kD - 1);  // into the slot of row step r - 1 (mod kD), finished last step
    // ---- publish this step's z-tap rows -----------------------------------------------------
    float *zb = ztap + (r & 1) * 4 * kK * ROW + kTbPad;
#pragma unroll
    for (int k = 0; k < kK; k++) {
      // V_k taps: txz, tzz of row r - 4 - 8k (index 4 of window 0 after this step's push,
      // index 5 of the later windows, whose push comes below)
      const int iv = k == 0 ? 4 : 5;
      zb[(4 * k + 0) * ROW + t] = w.txz[k][iv];
      zb[(4 * k + 1) * ROW + t] = w.tzz[k][iv];
      // S_k taps: vx, vz of row r - 8 - 8k (index 5 before this step's V_k push)
      zb[(4 * k + 2) * ROW + t] = w.vx[k][5];
      zb[(4 * k + 3) * ROW + t] = w.vz[k][5];
    }
    if (kBulk) {
      // a wait that gave up ends the march for the whole CTA (the barrier is a vote); otherwise
      // every thread is done with slot r - 1: refill it kD - 1 steps ahead
      if (__syncthreads_or(!ok)) {
        aborted = true;
        break;
      }
      const int ps = cur.slot == 0 ? kD - 1 : cur.slot - 1;
      tb_issue_warp<kT>(fd, ring + (size_t)ps * NF * kT, my_f, &bars[ps], r + kD - 1, ld, c0, lane);
      cur.advance();
    } else {
      __syncthreads();
    }
#pragma unroll
    for (int k = 0; k < kK; k++) {
      const float *zt_txz = zb + (4 * k + 0) * ROW + t;
      const float *zt_tzz = zb + (4 * k + 1) * ROW + t;
      const float *zt_vx = zb + (4 * k + 2) * ROW + t;
      const float *zt_vz = zb + (4 * k + 3) * ROW + t;
      // ---- V_k: velocities of row rv = r - 4 - 8k to time t + k + 1 ------------------------
      const int rv = r - 4 - 8 * k;
      const int hv = 4 + 8 * (kK - 1 - k);
      float vxn = 0.f, vzn = 0.f;
      if (vcol(k) && rv >= x0 - hv && rv < x1 + hv && rv >= nop && rv < d.nxp - nop) {
        const float ax = dxp_mid(w.txx[k]);
        const float fx = dxm_mid(w.txz[k]);
        const float bz = stencil4([&](int i) { return zt_txz[i - 1] - zt_txz[-i]; });
        const float ez = stencil4([&](int i) { return zt_tzz[i] - zt_tzz[-i + 1]; });
        const float cbx = bb[k] * dtdx, cbz = bb[k] * dtdz;
        const float ux_x = cbx * ax, ux_z = cbz * bz, uz_x = cbx * fx, uz_z = cbz * ez;
        const float ovx = k == 0 ? ovx0 : w.vx[k == 0 ? 0 : k - 1][0];
        const float ovz = k == 0 ? ovz0 : w.vz[k == 0 ? 0 : k - 1][0];
        vxn = ovx + (ux_x + ux_z);
        vzn = ovz + (uz_x + uz_z);
        if (zown && rv >= x0 && rv < x1) {
          if (k == kK - 1) {
            const int o = base + rv * ld + z;
            a.b.vx[o] = vxn;
            a.b.vz[o] = vzn;
          }
          if (rec_col) {
            const int tr = s_tr[rv - x0];
            if (tr >= 0) {
              const long long q = ((long long)s * d.max_ntr + tr) * d.nt + a.it + k;
              a.rec_vz[q] = vzn;
              a.rec_vx[q] = vxn;
            }
          }
        }
      }
      push(w.vx[k], vxn);
      push(w.vz[k], vzn);
      // ---- S_k: stresses of row rs = r - 8 - 8k to time t + k + 1 ---------------------------
      const int rs = r - 8 - 8 * k;
      const int hs = 8 * (kK - 1 - k);
      float nxx = 0.f, nzz = 0.f, nxz = 0.f;
      const bool s_on = scol(k) && rs >= x0 - hs && rs < x1 + hs && rs >= nop && rs < d.nxp - nop;
      if (s_on) {
        const float sa = dxm_mid(w.vx[k]);
        const float sf = dxp_mid(w.vz[k]);
        const float sb = stencil4([&](int i) { return zt_vz[i - 1] - zt_vz[-i]; });
        const float se = stencil4([&](int i) { return zt_vx[i] - zt_vx[-i + 1]; });
        const float l2m = lam[k] + 2.0f * mu[k];
        const float xx_x = l2m * dtdx * sa, xx_z = lam[k] * dtdz * sb;
        const float zz_x = lam[k] * dtdx * sa, zz_z = l2m * dtdz * sb;
        const float xz_x = dtdx * mu[k] * sf, xz_z = dtdz * mu[k] * se;
        float oxx = w.txx[k][0], ozz = w.tzz[k][0];
        const float oxz = w.txz[k][0];
        if (src_col && rs == sh.isx) {  // the injected cell: its stresses without the source
          oxx = own_txx[k];
          ozz = own_tzz[k];
        }
        nxx = oxx + (xx_x + xx_z);
        nzz = ozz + (zz_x + zz_z);
        nxz = oxz + (xz_x + xz_z);
      }
      if (k == kK - 1) {
        if (s_on && zown && rs >= x0 && rs < x1) {
          const int o = base + rs * ld + z;
          a.b.txx[o] = nxx;
          a.b.tzz[o] = nzz;
          a.b.txz[o] = nxz;
        }
      } else {
        // into the windows of V_{k+1}, with the source of time t + k + 1 at its cell
        // (a cell no stage updates keeps its state, zero: the grid's edge rows and columns)
        const int kn = k + 1 < kK ? k + 1 : 0;
        if (src_col && rs == sh.isx) {
          own_txx[kn] = nxx;
          own_tzz[kn] = nzz;
          const float sv = a.wavelet[a.it + k + 1];
          nxx += sv;
          nzz += sv;
        }
        push(w.txx[kn], nxx);
        push(w.tzz[kn], nzz);
        push(w.txz[kn], nxz);
      }
    }
  }
  if (kBulk) pair_exit<kD>(bars, cur, aborted, ok, a.err);
  cp_async_wait<0>();
}

}  // namespace ds2d
