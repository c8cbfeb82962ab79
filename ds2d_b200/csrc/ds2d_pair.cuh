// Pair-blocked, bulk-copy-fed ring kernels of the random-boundary elastic RTM step for sm_100a.
//
// Same x-march as the ring kernels of ds2d_fused.cuh (a CTA owns a z-strip, walks xr rows along
// x, stage 1 runs 4 rows behind the newest loaded row and stage 2 8 rows behind, both half steps
// of a time step in one pass), with three changes that cut the instructions per cell:
//
//  * Two cells per thread.  Thread t owns the adjacent columns z0 = zs - 8 + 2t and z0 + 1 and
//    moves them as float2.  An 8-tap z-derivative of both cells needs the 10 columns z0-4..z0+5:
//    five 8-byte shared loads (the thread's own pair and two pairs either side) instead of the
//    sixteen 4-byte loads two one-column threads issue, and every per-row cost (loop, indexes,
//    predicates, barrier) is paid once per two cells.
//  * Rows arrive by bulk copy.  Each ring slot holds, for one row step, every row segment the
//    step consumes (the newest stencil rows, the z-tap rows of stage 1 and the own-cell operands
//    of both stages).  One cp.async.bulk per field row (global -> shared, completion counted on
//    the slot's mbarrier) fills it kD - 1 steps ahead; the copies are spread over all warps of
//    the CTA (warp w issues the fields f with f mod W = w, and every warp arrives on the slot's
//    barrier with its own bytes), so no warp carries a step's whole copy issue to the next
//    barrier.  Every thread waits on the barrier's phase before it reads the slot.  Stage-1 z-taps are read straight from the ring, so a step has a
//    single CTA barrier (before the stage-2 z-taps, whose rows are computed in registers).
//  * Injections on the stencil values only.  The explosive source (forward) and the receiver
//    residual (adjoint) act on the stencil values, not on the stored state (the reference adds
//    them to the summed arrays, which its split update recomputes, FD2DGPU.cu:2039-2049,
//    :3306-3322).  The owner of the injected column adds the value to its x-window entry; the
//    threads whose z-taps read that column add it to their copy of the tap (the source, so the
//    sum rounds as in the one-column kernels) or add c_i * value to the derivative (the
//    residual).  The own-cell operands come from the ring, i.e. from memory, without it.
//
// Scope: random boundary (no PML cells, no strips), RTM forward (optional receiver recording)
// and backward steps.  The PML / strip / Born variants stay on the one-column ring kernels.
#pragma once
#include "ds2d_fused.cuh"

namespace ds2d {

// ---- bulk-copy ring primitives (PTX ISA 8.x, sm_90 and later) ------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// One arrival that also raises the transaction count the phase waits for by `bytes`.
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// One bounded poll: the thread may be suspended for up to kSuspendNs while the phase is open, so
// a waiting warp sleeps instead of re-issuing the poll.
constexpr unsigned kSuspendNs = 200000;
__device__ __forceinline__ bool mbar_test(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "n"(kSuspendNs)
      : "memory");
  return ok != 0;
}
// Global -> shared bulk copy (no multicast); `bytes` and both addresses multiples of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// A wait gives up once kRingWaitNs of device time have passed with the phase still open (read
// from %globaltimer, so the bound holds whatever the suspend hint does): far beyond any copy's
// latency, short of a hang.  A kernel that gives up raises the error word (code kErrRingWait)
// and leaves its march; the host turns the word into an error.
constexpr unsigned long long kRingWaitNs = 2000000000ull;
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr int kErrRingWait = 1;
// True once a pair kernel of this context has given up a wait: later launches return at once, so
// a failed step does not cost every later step its own wait bound before the host sees the word.
__device__ __forceinline__ bool pair_err_raised(const int *err) {
  return err && *(const volatile int *)err != 0;
}
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_test(bar, parity))
    if (global_ns() - t0 > kRingWaitNs) return false;
  return true;
}

// Floats per ring row of a kT-thread CTA: two columns per thread plus two pairs of padding on
// each side, so the z-taps of the edge threads stay inside the row.
__host__ __device__ constexpr int pair_row(int kT) { return 2 * kT + 8; }

// c_k of the 8th-order staggered stencil for k = 1..4, 0 otherwise (injection corrections).
__device__ __forceinline__ float coef_or0(int k) {
  return k == 1 ? kC1 : k == 2 ? kC2 : k == 3 ? kC3 : k == 4 ? kC4 : 0.0f;
}

// The ten columns z0-4 .. z0+5 around a thread's pair, v[k + 4] = column z0 + k, from a ring row
// (float2 index i of the thread's own pair).
struct Z10 {
  float v[10];
};
__device__ __forceinline__ Z10 z10(const float2 *row, int i) {
  const float2 a = row[i - 2], b = row[i - 1], c = row[i], e = row[i + 1], f = row[i + 2];
  return Z10{{a.x, a.y, b.x, b.y, c.x, c.y, e.x, e.y, f.x, f.y}};
}
// Dz+ f = sum c_i (f[z+i] - f[z-i+1]) and Dz- f = sum c_i (f[z+i-1] - f[z-i]) at column z0 + e.
template <int e>
__device__ __forceinline__ float dzp(const Z10 &z) {
  return stencil4([&](int i) { return z.v[4 + e + i] - z.v[5 + e - i]; });
}
template <int e>
__device__ __forceinline__ float dzm(const Z10 &z) {
  return stencil4([&](int i) { return z.v[3 + e + i] - z.v[4 + e - i]; });
}

// x-windows of float2 pairs: w[j] = row (newest - (N-1) + j).  Dx taps at the row 4 below the
// window's top, in the index pattern both staggered forms share here: sum c_i (w[3+i] - w[4-i]).
template <int N>
__device__ __forceinline__ void push2(float2 (&w)[N], float2 v) {
#pragma unroll
  for (int i = 0; i < N - 1; i++) w[i] = w[i + 1];
  w[N - 1] = v;
}
template <int N>
__device__ __forceinline__ float dxw_x(const float2 (&w)[N]) {
  return stencil4([&](int i) { return w[3 + i].x - w[4 - i].x; });
}
template <int N>
__device__ __forceinline__ float dxw_y(const float2 (&w)[N]) {
  return stencil4([&](int i) { return w[3 + i].y - w[4 - i].y; });
}

// Per-step ring bookkeeping shared by the pair kernels: slot / phase of the step being consumed
// and of the step being refilled (kD - 1 ahead).
template <int kD>
struct RingCursor {
  int slot = 0;
  unsigned phase = 0;
  __device__ __forceinline__ void advance() {
    if (++slot == kD) {
      slot = 0;
      phase ^= 1u;
    }
  }
};

// End of a pair kernel's march.  No bulk copy may still be landing in shared memory when the CTA
// exits, so every thread waits (bounded) for the phases still in flight: after a normal march,
// the kD - 1 slots issued beyond its last step; after an aborted one (some wait gave up), both
// phases of every slot.  A thread whose own wait gave up raises the error word.
template <int kD>
__device__ __forceinline__ void pair_exit(unsigned long long *bars, RingCursor<kD> cur,
                                          bool aborted, bool ok, int *err) {
  if (!aborted) {
    for (int j = 0; j < kD - 1; j++) {
      mbar_wait(&bars[cur.slot], cur.phase);
      cur.advance();
    }
    return;
  }
  if (!ok && err) atomicExch(err, kErrRingWait);
  for (int k = 0; k < kD; k++) {
    mbar_wait(&bars[k], 0);
    mbar_wait(&bars[k], 1);
  }
}

// One warp's share of the copies of a ring slot: the lane owning ring field f reads row
// (q - lag) of an array whose rows are ld floats apart (wavefields, parameters and the per-slot
// images alike) if that row lies in [lo, hi).  The strip's columns [zs - 8, zs - 8 + 2 kT) map to
// ring floats 4 .. 2 kT + 4; the copy is clipped to [0, ld) (the row's own allocation).  Lane 0
// arrives on the slot's barrier (one arrival per warp) with the bytes of the warp's copies
// (counted by ballot) before any is issued, so the phase cannot complete early.
struct RingField {
  const float *src;  // this lane's field: array row x starts at src + x * ld (0 for lanes >= NF)
  int lag, lo, hi;
};

template <int kT, int kHalo = 8>
__device__ __forceinline__ void issue_slot_warp(const RingField &fd, float *slot_base, int f,
                                                unsigned long long *bar, int q, int ld, int zs,
                                                int lane) {
  // (strips with a kHalo-column halo: columns [zs - kHalo, zs - kHalo + 2 kT))
  const int glo = max(0, zs - kHalo), ghi = min(ld, zs - kHalo + 2 * kT);
  const unsigned bytes = (unsigned)(ghi - glo) * 4u;
  const int row = q - fd.lag;
  const bool mine = fd.src != nullptr && row >= fd.lo && row < fd.hi;
  const unsigned n = __popc(__ballot_sync(0xffffffffu, mine));
  if (lane == 0) mbar_arrive_tx(bar, n * bytes);
  __syncwarp();
  if (mine)
    bulk_g2s(slot_base + f * pair_row(kT) + (glo - (zs - kHalo) + 4),
             fd.src + (long long)row * ld + glo, bytes, bar);
}

// Shared-memory bytes of a pair kernel: the ring, `rows` rows of stage-2 z-taps, the slot
// barriers and the receiver staging.
__host__ __device__ constexpr size_t pair_smem(int kT, int kD, int NF, int rows) {
  return sizeof(float) * ((size_t)kD * NF + rows) * pair_row(kT) + 8 * 8 + 6 * 16 * 4;
}

// ---------------------------------------------------------------------------------------------
// Forward step (background modelling, RTM source side): velocities of row r-4 and stresses of
// row r-8 at row step r; optional receiver recording.  Ring fields of step r:
//   0 txx(r)  1 txz(r-1)        x-window inputs (Dx+ txx over rows r-7..r, Dx- txz over r-8..r-1)
//   2 txz(r-4)  3 tzz(r-4)      stage-1 z-tap rows
//   4 vx(r-4)  5 vz(r-4)  6 b(r-4)            stage-1 own cells
//   7 txx(r-8)  8 tzz(r-8)  9 lam(r-8)  10 mu(r-8)   stage-2 own cells (txz(r-8) is w_txz[0])
constexpr int kFwdPairFields = 11;
constexpr int kFwdPairZ2 = 2;  // stage-2 z-tap rows: vx, vz of row r-8
constexpr int kFwdPairZ2Rows = 2 * kFwdPairZ2;  // double-buffered

template <int kT, int kD, int kMinB>
__global__ void __launch_bounds__(kT, kMinB) k_fwd_pair(FwdFusedArgs a) {
  constexpr int NF = kFwdPairFields, ROW = pair_row(kT);
  extern __shared__ __align__(16) float smem[];
  float *ring = smem;                               // [kD][NF][ROW]
  float *z2 = ring + (size_t)kD * NF * ROW;         // [2][kFwdPairZ2][ROW]
  unsigned long long *bars = (unsigned long long *)(z2 + kFwdPairZ2Rows * ROW);
  int *s_tr = (int *)(bars + 8);                    // receiver staging [16]
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int zs = blockIdx.x * a.tz;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  if (__syncthreads_or(t == 0 && pair_err_raised(a.err))) return;  // whole CTA
  const int ld = d.ld, nop = d.nop;
  const long long fbase = d.slot * s;
  const int z0 = zs - 8 + 2 * t;
  const int pi = t + 2;  // float2 index of the own pair in a ring row
  // column predicates of the pair: stage-1 columns, stage-2 (owned) columns, update masks
  const bool c1 = z0 >= zs - 4 && z0 < zs + a.tz + 4;
  const bool c2 = z0 >= zs && z0 < zs + a.tz && z0 < d.nzp;
  const bool u0 = z0 >= nop && z0 < d.nzp - nop, u1 = z0 + 1 >= nop && z0 + 1 < d.nzp - nop;
  const ShotDev sh = a.shots[s];
  const float sval = a.wavelet[a.it];
  const int se = sh.isz - z0;  // source column relative to the pair (0 / 1: owned here)
  const bool src_near = se >= -4 && se <= 5;
  const bool rec_col = a.rec_on && (sh.igz - z0 == 0 || sh.igz - z0 == 1);
  const int rec_e = sh.igz - z0;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;

  // ring fields (the thread owning field f issues its row copies)
  const int lane = t & 31;
  // ring field of this thread: warp w, lane l owns field w + W l (W warps), so every warp issues
  // a share of a slot's copies
  const int my_f = (t >> 5) + (kT / 32) * lane;
  RingField fd{nullptr, 0, 0, d.nxp};
  {
    const float *src[NF] = {a.a.txx, a.a.txz, a.a.txz, a.a.tzz, a.a.vx, a.a.vz,
                            a.p.b,   a.a.txx, a.a.tzz, a.p.lam, a.p.mu};
    const int lag[NF] = {0, 1, 4, 4, 4, 4, 4, 8, 8, 8, 8};
#pragma unroll
    for (int f = 0; f < NF; f++)
      if (my_f == f) {
        fd.src = src[f] + fbase;
        fd.lag = lag[f];
      }
  }
  if (t == 0) {
    for (int k = 0; k < kD; k++) mbar_init(&bars[k], kT / 32);  // one arrival per warp
    mbar_fence_init();
  }
  __syncthreads();
  const int rs0 = x0 - 8;
  for (int j = 0; j < kD - 1; j++)
    issue_slot_warp<kT>(fd, ring + (size_t)j * NF * ROW, my_f, &bars[j], rs0 + j, ld, zs, lane);

  float2 w_txx[8], w_txz[8], w_vx[9], w_vz[8];
#pragma unroll
  for (int i = 0; i < 8; i++) w_txx[i] = w_txz[i] = w_vz[i] = make_float2(0.f, 0.f);
#pragma unroll
  for (int i = 0; i < 9; i++) w_vx[i] = make_float2(0.f, 0.f);

  RingCursor<kD> cur;
  bool ok = true, aborted = false;
#pragma unroll 2
  for (int r = rs0; r < x1 + 8; r++) {
    // A wait that gives up skips the step's work; the barrier below is a vote, so every thread
    // leaves the march together (none is left waiting at a barrier).
    ok = mbar_wait(&bars[cur.slot], cur.phase);
    const float *S = ring + (size_t)cur.slot * NF * ROW;
    auto F2 = [&](int f) -> float2 { return reinterpret_cast<const float2 *>(S + f * ROW)[pi]; };
    // trace index of velocity row r + 4 (recorded at step r + 8, one commit group per step)
    if (rec_col && r + 4 < d.nxp && r + 4 >= 0)
      cp_async4((float *)&s_tr[(r + 4) & 15], (const float *)(rmap + r + 4));
    if (ok) {
      float2 n_txx = F2(0);
      if (r == sh.isx && (se == 0 || se == 1)) {  // FD2DGPU.cu:2039-2049 (transient)
        if (se == 0) n_txx.x += sval; else n_txx.y += sval;
      }
      push2(w_txx, n_txx);
      push2(w_txz, F2(1));
    }
    // ---- stage 1: velocities of row rv = r - 4 ------------------------------------------
    const int rv = r - 4;
    float2 vn = make_float2(0.f, 0.f), vzn = make_float2(0.f, 0.f);
    if (ok && c1 && r >= x0 && rv >= nop && rv < d.nxp - nop) {
      const Z10 zxz = z10(reinterpret_cast<const float2 *>(S + 2 * ROW), pi);
      Z10 zzz = z10(reinterpret_cast<const float2 *>(S + 3 * ROW), pi);
      if (rv == sh.isx && src_near) zzz.v[se + 4] += sval;  // tzz + source, as the ring kernel
      const float ez0 = dzp<0>(zzz), ez1 = dzp<1>(zzz);
      const float2 bb = F2(6), ovx = F2(4), ovz = F2(5);
      const float ax0 = dxw_x(w_txx), ax1 = dxw_y(w_txx);
      const float fx0 = dxw_x(w_txz), fx1 = dxw_y(w_txz);
      const float bz0 = dzm<0>(zxz), bz1 = dzm<1>(zxz);
      {
        const float cbx = bb.x * dtdx, cbz = bb.x * dtdz;
        if (u0) {
          vn.x = ovx.x + (cbx * ax0 + cbz * bz0);
          vzn.x = ovz.x + (cbx * fx0 + cbz * ez0);
        }
      }
      {
        const float cbx = bb.y * dtdx, cbz = bb.y * dtdz;
        if (u1) {
          vn.y = ovx.y + (cbx * ax1 + cbz * bz1);
          vzn.y = ovz.y + (cbx * fx1 + cbz * ez1);
        }
      }
      if (c2 && rv >= x0 && rv < x1) {
        const long long k = fbase + (long long)rv * ld + z0;
        *reinterpret_cast<float2 *>(a.b.vx + k) = vn;
        *reinterpret_cast<float2 *>(a.b.vz + k) = vzn;
        if (rec_col) {
          const int tr = s_tr[rv & 15];
          if (tr >= 0) {
            const long long q = ((long long)s * d.max_ntr + tr) * d.nt + a.it;
            a.rec_vz[q] = rec_e == 0 ? vzn.x : vzn.y;
            a.rec_vx[q] = rec_e == 0 ? vn.x : vn.y;
          }
        }
      }
    }
    push2(w_vx, vn);
    push2(w_vz, vzn);
    // ---- stage-2 z-tap rows (vx, vz of row r - 8), then the step's only barrier --------------
    float *zb = z2 + (r & 1) * kFwdPairZ2 * ROW;
    reinterpret_cast<float2 *>(zb)[pi] = w_vx[4];
    reinterpret_cast<float2 *>(zb + ROW)[pi] = w_vz[3];
    if (rec_col) cp_async_commit();
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    // every thread is done with the previous slot: refill it kD - 1 steps ahead
    {  // every warp issues its share of the slot's copies
      const int ps = cur.slot == 0 ? kD - 1 : cur.slot - 1;
      issue_slot_warp<kT>(fd, ring + (size_t)ps * NF * ROW, my_f, &bars[ps], r + kD - 1, ld, zs,
                          lane);
    }
    // ---- stage 2: stresses of row rs = r - 8 ------------------------------------------------
    const int rs = r - 8;
    if (c2 && rs >= x0 && rs < x1 && rs >= nop && rs < d.nxp - nop) {
      const Z10 zvx = z10(reinterpret_cast<const float2 *>(zb), pi);
      const Z10 zvz = z10(reinterpret_cast<const float2 *>(zb + ROW), pi);
      const float2 lam = F2(9), mu = F2(10), oxx = F2(7), ozz = F2(8), oxz = w_txz[0];
      float2 nxx = oxx, nzz = ozz, nxz = oxz;
      {
        const float sa = stencil4([&](int i) { return w_vx[3 + i].x - w_vx[4 - i].x; });
        const float sf = stencil4([&](int i) { return w_vz[3 + i].x - w_vz[4 - i].x; });
        const float sb = dzm<0>(zvz), sev = dzp<0>(zvx);
        const float l2m = lam.x + 2.0f * mu.x;
        if (u0) {
          nxx.x = oxx.x + (l2m * dtdx * sa + lam.x * dtdz * sb);
          nzz.x = ozz.x + (lam.x * dtdx * sa + l2m * dtdz * sb);
          nxz.x = oxz.x + (dtdx * mu.x * sf + dtdz * mu.x * sev);
        }
      }
      {
        const float sa = stencil4([&](int i) { return w_vx[3 + i].y - w_vx[4 - i].y; });
        const float sf = stencil4([&](int i) { return w_vz[3 + i].y - w_vz[4 - i].y; });
        const float sb = dzm<1>(zvz), sev = dzp<1>(zvx);
        const float l2m = lam.y + 2.0f * mu.y;
        if (u1) {
          nxx.y = oxx.y + (l2m * dtdx * sa + lam.y * dtdz * sb);
          nzz.y = ozz.y + (lam.y * dtdx * sa + l2m * dtdz * sb);
          nxz.y = oxz.y + (dtdx * mu.y * sf + dtdz * mu.y * sev);
        }
      }
      const long long k = fbase + (long long)rs * ld + z0;
      *reinterpret_cast<float2 *>(a.b.txx + k) = nxx;
      *reinterpret_cast<float2 *>(a.b.tzz + k) = nzz;
      *reinterpret_cast<float2 *>(a.b.txz + k) = nxz;
    }
    if (rec_col) cp_async_wait<7>();
    cur.advance();
  }
  pair_exit<kD>(bars, cur, aborted, ok, a.err);
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Acoustic forward step (vs = 0: one stress s), pair-blocked: the counterpart of k_ac_ring with
// the same arithmetic per cell (its modes, its overlay and source, its Born source and records).
// At row step r the velocities of row r - 4 and the stress of row r - 8 are updated.  Ring fields
// of step r:
//   0 s(r)  1 e(r)                   x-window of S = s (+ e, mode 1)
//   2 s(r-4)  3 e(r-4)               stage-1 z-tap rows of S
//   4 vx(r-4)  5 vz(r-4)  6 b(r-4)   stage-1 own cells
//   7 s(r-8)  8 lam(r-8)  9 m(r-8)   stage-2 own cells (m: mode 0 with the Born source written)
// The e rows (mode 1) and m (mode 0 without a Born source) are not copied.  In mode 1 the z-taps
// of S add the s and e rows column by column, so S is rounded as in k_ac_ring; in mode 0 the
// source enters the x-window at its row and the z-tap copies of the columns within 4 of it.
// ---------------------------------------------------------------------------------------------
constexpr int kAcPairFields = 10;
constexpr int kAcPairZ2Rows = 2;  // stage-2 z-tap row (vz of row r-8), double-buffered
constexpr int kAcPairD = 4;
__host__ __device__ constexpr size_t ac_pair_smem(int kT) {
  return pair_smem(kT, kAcPairD, kAcPairFields, kAcPairZ2Rows);
}

template <int kMode, int kT, int kMinB>
__global__ void __launch_bounds__(kT, kMinB) k_ac_pair(AcRingArgs a) {
  constexpr int kD = kAcPairD, NF = kAcPairFields, ROW = pair_row(kT);
  extern __shared__ __align__(16) float smem[];
  float *ring = smem;                               // [kD][NF][ROW]
  float *z2 = ring + (size_t)kD * NF * ROW;         // [2][ROW]
  unsigned long long *bars = (unsigned long long *)(z2 + kAcPairZ2Rows * ROW);
  int *s_tr = (int *)(bars + 8);                    // receiver staging [16]
  const int sl = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[sl]);
  const int zs = blockIdx.x * a.tz;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  if (__syncthreads_or(t == 0 && pair_err_raised(a.err))) return;  // whole CTA
  const int ld = d.ld, nop = d.nop, pml = d.pml;
  const long long fbase = d.slot * sl;
  const int z0 = zs - 8 + 2 * t;
  const int pi = t + 2;  // float2 index of the own pair in a ring row
  const bool c1 = z0 >= zs - 4 && z0 < zs + a.tz + 4;
  const bool c2 = z0 >= zs && z0 < zs + a.tz && z0 < d.nzp;
  const bool u0 = z0 >= nop && z0 < d.nzp - nop, u1 = z0 + 1 >= nop && z0 + 1 < d.nzp - nop;
  const bool zi0 = z0 >= pml && z0 < d.nzp - pml, zi1 = z0 + 1 >= pml && z0 + 1 < d.nzp - pml;
  const ShotDev sh = a.shots[sl];
  const float sval = kMode == 0 ? a.wavelet[a.it] : 0.f;
  const int se = sh.isz - z0;  // source column relative to the pair (0 / 1: owned here)
  const bool src_near = kMode == 0 && se >= -4 && se <= 5;
  const bool rec_col = kMode == 1 && a.rec_vz && (sh.igz - z0 == 0 || sh.igz - z0 == 1);
  const int rec_e = sh.igz - z0;
  const int *rmap = a.rmap + (long long)sl * d.nxp_max;
  const float cx = d.dt / d.dx, cz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  const bool born_out = kMode == 0 && a.e_out != nullptr;

  const int lane = t & 31;
  // ring field of this thread: warp w, lane l owns field w + W l (W warps), so every warp issues
  // a share of a slot's copies
  const int my_f = (t >> 5) + (kT / 32) * lane;
  RingField fd{nullptr, 0, 0, d.nxp};
  {
    const float *src[NF] = {a.s, kMode == 1 ? a.e_in : nullptr, a.s, kMode == 1 ? a.e_in : nullptr,
                            a.vx, a.vz, a.b, a.s, a.lam, born_out ? a.m : nullptr};
    const int lag[NF] = {0, 0, 4, 4, 4, 4, 4, 8, 8, 8};
#pragma unroll
    for (int f = 0; f < NF; f++)
      if (my_f == f && src[f]) {
        fd.src = src[f] + fbase;
        fd.lag = lag[f];
      }
  }
  if (t == 0) {
    for (int k = 0; k < kD; k++) mbar_init(&bars[k], kT / 32);  // one arrival per warp
    mbar_fence_init();
  }
  __syncthreads();
  const int rs0 = x0 - 8;
  for (int j = 0; j < kD - 1; j++)
    issue_slot_warp<kT>(fd, ring + (size_t)j * NF * ROW, my_f, &bars[j], rs0 + j, ld, zs, lane);

  float2 w_S[8], w_vx[9], w_vz[8];
#pragma unroll
  for (int i = 0; i < 8; i++) w_S[i] = w_vz[i] = make_float2(0.f, 0.f);
#pragma unroll
  for (int i = 0; i < 9; i++) w_vx[i] = make_float2(0.f, 0.f);

  RingCursor<kD> cur;
  bool ok = true, aborted = false;
#pragma unroll 2
  for (int r = rs0; r < x1 + 8; r++) {
    ok = mbar_wait(&bars[cur.slot], cur.phase);
    const float *S = ring + (size_t)cur.slot * NF * ROW;
    auto F2 = [&](int f) -> float2 { return reinterpret_cast<const float2 *>(S + f * ROW)[pi]; };
    if (rec_col && r + 4 < d.nxp && r + 4 >= 0)
      cp_async4((float *)&s_tr[(r + 4) & 15], (const float *)(rmap + r + 4));
    if (ok) {
      float2 nS = F2(0);
      if (kMode == 1) {
        const float2 e = F2(1);
        nS.x += e.x;
        nS.y += e.y;
      }
      if (kMode == 0 && r == sh.isx && (se == 0 || se == 1)) {  // FD2DGPU.cu:2039-2049
        if (se == 0) nS.x += sval; else nS.y += sval;
      }
      push2(w_S, nS);
    }
    // ---- stage 1: velocities of row rv = r - 4 ------------------------------------------
    const int rv = r - 4;
    float2 vxn = make_float2(0.f, 0.f), vzn = make_float2(0.f, 0.f);
    if (ok && c1 && r >= x0 && rv >= nop && rv < d.nxp - nop) {
      Z10 zS = z10(reinterpret_cast<const float2 *>(S + 2 * ROW), pi);
      if (kMode == 1) {
        const Z10 zE = z10(reinterpret_cast<const float2 *>(S + 3 * ROW), pi);
#pragma unroll
        for (int k = 0; k < 10; k++) zS.v[k] += zE.v[k];
      }
      if (kMode == 0 && rv == sh.isx && src_near) zS.v[se + 4] += sval;  // S + source
      const float az0 = dzp<0>(zS), az1 = dzp<1>(zS);
      const float2 bb = F2(6), ovx = F2(4), ovz = F2(5);
      const float ax0 = dxw_x(w_S), ax1 = dxw_y(w_S);
      if (u0) {  // k_ac_vel: v + dir (b dt/d) D+ S, dir = +1
        vxn.x = ovx.x + (bb.x * cx) * ax0;
        vzn.x = ovz.x + (bb.x * cz) * az0;
      }
      if (u1) {
        vxn.y = ovx.y + (bb.y * cx) * ax1;
        vzn.y = ovz.y + (bb.y * cz) * az1;
      }
      if (c2 && rv >= x0 && rv < x1) {
        const long long k = fbase + (long long)rv * ld + z0;
        *reinterpret_cast<float2 *>(a.vx_n + k) = vxn;
        *reinterpret_cast<float2 *>(a.vz_n + k) = vzn;
        if (rec_col) {
          const int tr = s_tr[rv & 15];
          if (tr >= 0) {
            const long long q = ((long long)sl * d.max_ntr + tr) * d.nt + a.it;
            a.rec_vz[q] = rec_e == 0 ? vzn.x : vzn.y;
            a.rec_vx[q] = rec_e == 0 ? vxn.x : vxn.y;
          }
        }
      }
    }
    push2(w_vx, vxn);
    push2(w_vz, vzn);
    // ---- stage-2 z-tap row (vz of row r - 8), then the step's only barrier ------------------
    float *zb = z2 + (r & 1) * ROW;
    reinterpret_cast<float2 *>(zb)[pi] = w_vz[3];
    if (rec_col) cp_async_commit();
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    {  // every warp issues its share of the slot's copies
      const int ps = cur.slot == 0 ? kD - 1 : cur.slot - 1;
      issue_slot_warp<kT>(fd, ring + (size_t)ps * NF * ROW, my_f, &bars[ps], r + kD - 1, ld, zs,
                          lane);
    }
    // ---- stage 2: stress of row rs = r - 8 --------------------------------------------------
    const int rs = r - 8;
    if (c2 && rs >= x0 && rs < x1 && rs >= nop && rs < d.nxp - nop) {
      const Z10 zvz = z10(reinterpret_cast<const float2 *>(zb), pi);
      const float2 lam = F2(8), os = F2(7);
      const float sx0 = stencil4([&](int i) { return w_vx[3 + i].x - w_vx[4 - i].x; });
      const float sx1 = stencil4([&](int i) { return w_vx[3 + i].y - w_vx[4 - i].y; });
      const float sz0 = dzm<0>(zvz), sz1 = dzm<1>(zvz);
      float2 ns = os;
      if (u0) ns.x = os.x + lam.x * (cx * sx0 + cz * sz0);  // k_ac_str, dir = +1
      if (u1) ns.y = os.y + lam.y * (cx * sx1 + cz * sz1);
      const long long k = fbase + (long long)rs * ld + z0;
      *reinterpret_cast<float2 *>(a.s_n + k) = ns;
      if (born_out && rs >= pml && rs < d.nxp - pml && (zi0 || zi1)) {
        const float2 mm = F2(9);
        float2 e = make_float2(0.f, 0.f);  // the band's cells stay zero (k_ac_born)
        if (zi0) e.x = -2.0f * lam.x * mm.x * (sx0 * rdx + sz0 * rdz);
        if (zi1) e.y = -2.0f * lam.y * mm.y * (sx1 * rdx + sz1 * rdz);
        *reinterpret_cast<float2 *>(a.e_out + k) = e;
      }
    }
    if (rec_col) cp_async_wait<7>();
    cur.advance();
  }
  pair_exit<kD>(bars, cur, aborted, ok, a.err);
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Reverse step of the acoustic L^T, pair-blocked: the counterpart of k_ac_rev_ring, with the same
// three chained stages and the same arithmetic per cell,
//   A. (row r-4)  y_v += residual; yx -= dt/dx Dx+(lam ys), yz -= dt/dz Dz+(lam ys);
//   B. (row r-8)  gs = -Dx-(b dt/dx yx) - Dz-(b dt/dz yz), ys += gs, the gradient, and
//                 s -= lam (dt/dx Dx- bvx + dt/dz Dz- bvz);
//   C. (row r-12) v -= b dt/d D+(s + source),
// on strips with a 12-column halo (stage A runs on the halo of B, B on the halo of C).  Ring
// fields of step r:
//   0 ys(r)  1 lam(r)                  x-window of w = ys lam
//   2 ys(r-4)  3 lam(r-4)              stage-A z-taps of w (the products formed per tap)
//   4 yx(r-4)  5 yz(r-4)  6 b(r-4)     stage-A own cells
//   7 vx(r-4)  8 vz(r-4)               background velocities (x-window of vx; vz kept 8 rows)
//   9 vz(r-8)                          stage-B z-taps of the background vz
//   10 ys(r-8)  11 s(r-8)  12 lam(r-8)  13 gradient(r-8)   stage-B own cells
//   14 b(r-12)                         stage-C own cells
// The stage-B z-taps of b dt/dz yz and the stage-C z-taps of s + source are values the kernel
// computed 4 row steps earlier (stages A and B); they go through two circular row buffers in
// shared memory, written at step r and read at step r + 4, so one barrier per step suffices
// (k_ac_rev_ring needs three).  The residual enters stage A's own cells (as in k_ac_rev_ring),
// the source stage B's computed S values, so neither needs a z-tap correction.
// ---------------------------------------------------------------------------------------------
constexpr int kAcRevPairFields = 15;
constexpr int kAcRevPairD = 3;
constexpr int kAcRevPairZ = 8;  // rows of each z-tap buffer (written at r, read at r + 4)
constexpr int kAcRevHalo = 12;
__host__ __device__ constexpr size_t ac_rev_pair_smem(int kT) {
  return pair_smem(kT, kAcRevPairD, kAcRevPairFields, 2 * kAcRevPairZ);
}

template <int kT, int kMinB>
__global__ void __launch_bounds__(kT, kMinB) k_ac_rev_pair(AcRevArgs a) {
  constexpr int kD = kAcRevPairD, NF = kAcRevPairFields, ROW = pair_row(kT), ZD = kAcRevPairZ;
  extern __shared__ __align__(16) float smem[];
  float *ring = smem;                               // [kD][NF][ROW]
  float *zu = ring + (size_t)kD * NF * ROW;         // [ZD][ROW]  b dt/dz yz of stage A
  float *zS = zu + (size_t)ZD * ROW;                // [ZD][ROW]  s + source of stage B
  unsigned long long *bars = (unsigned long long *)(zS + (size_t)ZD * ROW);
  int *s_tr = (int *)(bars + 8), *s_has = s_tr + 16;  // receiver staging [16] each
  float *s_rz = (float *)(s_has + 16), *s_rx = s_rz + 16;
  const int sl = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[sl]);
  const int zs = blockIdx.x * a.tz;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;  // beyond this slot's window (uneven batches), whole CTA
  if (__syncthreads_or(t == 0 && pair_err_raised(a.err))) return;  // whole CTA
  const int ld = d.ld, nop = d.nop, pml = d.pml;
  const long long fbase = d.slot * sl;
  const long long ibase = (long long)sl * d.wnx_max * d.ild;
  const int z0 = zs - kAcRevHalo + 2 * t;
  const int pi = t + 2;  // float2 index of the own pair in a ring row
  const bool cA = z0 >= zs - 8 && z0 < zs + a.tz + 8;
  const bool cB = z0 >= zs - 4 && z0 < zs + a.tz + 4;
  const bool cC = z0 >= zs && z0 < zs + a.tz && z0 < d.nzp;
  const bool u0 = z0 >= nop && z0 < d.nzp - nop, u1 = z0 + 1 >= nop && z0 + 1 < d.nzp - nop;
  const bool i0 = z0 >= pml && z0 < d.nzp - pml, i1 = z0 + 1 >= pml && z0 + 1 < d.nzp - pml;
  const ShotDev sh = a.shots[sl];
  const int re = sh.igz - z0, se = sh.isz - z0;
  const bool rec_col = re == 0 || re == 1;
  const float sval = a.wavelet[a.it];
  const float *res_z = a.res_vz + (long long)sl * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)sl * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)sl * d.nxp_max;
  const float cx = d.dt / d.dx, cz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;

  const int lane = t & 31;
  // ring field of this thread: warp w, lane l owns field w + W l (W warps), so every warp issues
  // a share of a slot's copies
  const int my_f = (t >> 5) + (kT / 32) * lane;
  RingField fd{nullptr, 0, 0, d.nxp};
  {
    const float *src[NF] = {a.ys, a.lam, a.ys, a.lam, a.yx, a.yz, a.b, a.vx,
                            a.vz, a.vz,  a.ys, a.s,   a.lam, a.grad, a.b};
    const int lag[NF] = {0, 0, 4, 4, 4, 4, 4, 4, 4, 8, 8, 8, 8, 8, 12};
#pragma unroll
    for (int f = 0; f < NF; f++)
      if (my_f == f) {
        // gradient rows: grid row x is image row x - pml of the slot's plane
        fd.src = f == 13 ? src[f] + ibase - (long long)pml * ld : src[f] + fbase;
        fd.lag = lag[f];
        fd.lo = f == 13 ? pml : 0;
        fd.hi = f == 13 ? d.nxp - pml : d.nxp;
      }
  }
  const int r_first = x0 - 10, r_last = x1 + 12;
  if (t == 0) {
    for (int k = 0; k < kD; k++) mbar_init(&bars[k], kT / 32);  // one arrival per warp
    mbar_fence_init();
  }
  if (rec_col) {  // stage-A rows r_first-4 ..: residuals of the first 8 rows and trace indexes
                  // of the 8 after them (direct; the march fetches the rest ahead)
    const int a0 = r_first - 4;
    for (int q = a0; q < a0 + 8; q++) {
      const int tr = (q >= 0 && q < d.nxp) ? rmap[q] : -1;
      s_has[q & 15] = tr >= 0;
      if (tr >= 0) {
        s_rz[q & 15] = res_z[(long long)tr * d.nt];
        s_rx[q & 15] = res_x[(long long)tr * d.nt];
      }
    }
    for (int q = a0 + 8; q < a0 + 16; q++) s_tr[q & 15] = (q >= 0 && q < d.nxp) ? rmap[q] : -1;
  }
  __syncthreads();
  for (int j = 0; j < kD - 1; j++)
    issue_slot_warp<kT, kAcRevHalo>(fd, ring + (size_t)j * NF * ROW, my_f, &bars[j], r_first + j,
                                      ld, zs, lane);

  const float2 zero2 = make_float2(0.f, 0.f);
  float2 w_w[8], w_ux[9], w_bvx[9], w_bvz[9], w_S[8];
#pragma unroll
  for (int i = 0; i < 8; i++) w_w[i] = w_S[i] = zero2;
#pragma unroll
  for (int i = 0; i < 9; i++) w_ux[i] = w_bvx[i] = w_bvz[i] = zero2;

  RingCursor<kD> cur;
  bool ok = true, aborted = false;
  for (int r = r_first; r < r_last; r++) {
    ok = mbar_wait(&bars[cur.slot], cur.phase);
    const float *S = ring + (size_t)cur.slot * NF * ROW;
    auto F2 = [&](int f) -> float2 { return reinterpret_cast<const float2 *>(S + f * ROW)[pi]; };
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
      cp_async_commit();
    }
    if (ok) {
      const float2 ys = F2(0), lam = F2(1);
      push2(w_w, make_float2(ys.x * lam.x, ys.y * lam.y));  // k_ac_adj_v: lam[q] * ys[q]
      push2(w_bvx, F2(7));
      push2(w_bvz, F2(8));
    }
    // ---- A: adjoint velocities of row rA -------------------------------------------------------
    float2 uxn = zero2, uzn = zero2;
    if (ok && cA && rA >= 0 && rA < d.nxp) {
      float2 yx = F2(4), yz = F2(5);
      if (rA >= nop && rA < d.nxp - nop) {
        const Z10 zy = z10(reinterpret_cast<const float2 *>(S + 2 * ROW), pi);
        const Z10 zl = z10(reinterpret_cast<const float2 *>(S + 3 * ROW), pi);
        Z10 zw;
#pragma unroll
        for (int k = 0; k < 10; k++) zw.v[k] = zy.v[k] * zl.v[k];
        if (rec_col && s_has[rA & 15]) {
          if (re == 0) {
            yz.x += s_rz[rA & 15];
            yx.x += s_rx[rA & 15];
          } else {
            yz.y += s_rz[rA & 15];
            yx.y += s_rx[rA & 15];
          }
        }
        if (u0) {
          yx.x = yx.x - cx * dxw_x(w_w);
          yz.x = yz.x - cz * dzp<0>(zw);
        }
        if (u1) {
          yx.y = yx.y - cx * dxw_y(w_w);
          yz.y = yz.y - cz * dzp<1>(zw);
        }
        if (cC && rA >= x0 && rA < x1) {
          const long long k = fbase + (long long)rA * ld + z0;
          *reinterpret_cast<float2 *>(a.yx_n + k) = yx;
          *reinterpret_cast<float2 *>(a.yz_n + k) = yz;
        }
      }
      const float2 bb = F2(6);
      uxn = make_float2(bb.x * cx * yx.x, bb.y * cx * yx.y);  // k_ac_adj_s: b[q] * cx * yx[q]
      uzn = make_float2(bb.x * cz * yz.x, bb.y * cz * yz.y);
    }
    push2(w_ux, uxn);
    reinterpret_cast<float2 *>(zu + ((r + 16) & (ZD - 1)) * ROW)[pi] = uzn;
    // ---- B: ys, gradient and the background stress of row rB ---------------------------------
    float2 Sn = zero2;
    if (ok && cB && rB >= 0 && rB < d.nxp) {
      float2 bs = F2(11);
      if (rB >= nop && rB < d.nxp - nop) {
        const Z10 zuz = z10(reinterpret_cast<const float2 *>(zu + ((r + 12) & (ZD - 1)) * ROW), pi);
        const Z10 zbv = z10(reinterpret_cast<const float2 *>(S + 9 * ROW), pi);
        const float2 lam = F2(12), ys_o = F2(10);
        float2 ys_n = ys_o, gr = zero2;
        const bool own = cC && rB >= x0 && rB < x1;
        if (own && rB >= pml && rB < d.nxp - pml) gr = F2(13);
        const float2 g_o = gr;
        {
          const float gx = stencil4([&](int i) { return w_ux[3 + i].x - w_ux[4 - i].x; });
          const float gs = -gx - dzm<0>(zuz);
          const float sx = stencil4([&](int i) { return w_bvx[3 + i].x - w_bvx[4 - i].x; });
          const float sz = dzm<0>(zbv);
          if (u0) {
            ys_n.x = ys_o.x + gs;
            if (i0) gr.x = g_o.x + -2.0f * lam.x * (sx * rdx + sz * rdz) * gs;
            bs.x = bs.x + -1.0f * lam.x * (cx * sx + cz * sz);  // k_ac_str, dir = -1
          }
        }
        {
          const float gx = stencil4([&](int i) { return w_ux[3 + i].y - w_ux[4 - i].y; });
          const float gs = -gx - dzm<1>(zuz);
          const float sx = stencil4([&](int i) { return w_bvx[3 + i].y - w_bvx[4 - i].y; });
          const float sz = dzm<1>(zbv);
          if (u1) {
            ys_n.y = ys_o.y + gs;
            if (i1) gr.y = g_o.y + -2.0f * lam.y * (sx * rdx + sz * rdz) * gs;
            bs.y = bs.y + -1.0f * lam.y * (cx * sx + cz * sz);
          }
        }
        if (own) {
          const long long k = fbase + (long long)rB * ld + z0;
          *reinterpret_cast<float2 *>(a.ys_n + k) = ys_n;
          *reinterpret_cast<float2 *>(a.s_n + k) = bs;
          if (rB >= pml && rB < d.nxp - pml && (i0 || i1))
            *reinterpret_cast<float2 *>(a.grad + ibase + (long long)(rB - pml) * d.ild + z0) = gr;
        }
      }
      Sn = bs;
      if (rB == sh.isx) {  // the source overlay of k_ac_vel (transient)
        if (se == 0) Sn.x += sval;
        if (se == 1) Sn.y += sval;
      }
    }
    push2(w_S, Sn);
    reinterpret_cast<float2 *>(zS + ((r + 16) & (ZD - 1)) * ROW)[pi] = Sn;
    // ---- C: background velocities of row rC ----------------------------------------------------
    if (ok && cC && rC >= x0 && rC < x1 && rC >= nop && rC < d.nxp - nop) {
      const Z10 zsn = z10(reinterpret_cast<const float2 *>(zS + ((r + 12) & (ZD - 1)) * ROW), pi);
      const float2 bb = F2(14), ovx = w_bvx[0], ovz = w_bvz[0];
      float2 vx = ovx, vz = ovz;
      if (u0) {
        vx.x = ovx.x + -1.0f * (bb.x * cx) * dxw_x(w_S);  // k_ac_vel, dir = -1
        vz.x = ovz.x + -1.0f * (bb.x * cz) * dzp<0>(zsn);
      }
      if (u1) {
        vx.y = ovx.y + -1.0f * (bb.y * cx) * dxw_y(w_S);
        vz.y = ovz.y + -1.0f * (bb.y * cz) * dzp<1>(zsn);
      }
      const long long k = fbase + (long long)rC * ld + z0;
      *reinterpret_cast<float2 *>(a.vx_n + k) = vx;
      *reinterpret_cast<float2 *>(a.vz_n + k) = vz;
    }
    // one barrier per step: the z-tap rows written above are read 4 steps on; the ring slot of
    // the previous step is free once every thread has passed it
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    {  // every warp issues its share of the slot's copies
      const int ps = cur.slot == 0 ? kD - 1 : cur.slot - 1;
      issue_slot_warp<kT, kAcRevHalo>(fd, ring + (size_t)ps * NF * ROW, my_f, &bars[ps],
                                      r + kD - 1, ld, zs, lane);
    }
    if (rec_col) cp_async_wait<7>();
    cur.advance();
  }
  pair_exit<kD>(bars, cur, aborted, ok, a.err);
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// Backward RTM step (random boundary): interior reconstruction of the source field (direction
// -1, FD2DGPU.cu:903-1082 via :4769-4772), the adjoint step with the receiver residual
// (FD2DGPU.cu:591-895, :3306-3322) and the imaging condition (doimage_gradient :3245,
// doimage_illum :3235).  Stage 1 (stresses and images) at row r-4, stage 2 (velocities and
// illumination) at row r-8.
//
// kPart selects what one launch does: 0 everything (one pass, 124 B per cell), 1 the
// reconstruction and the illumination (60 B), 2 the adjoint and the imaging, the latter with the
// strains of the reconstruction's input state (t), which part 1 does not change (84 B).  Parts 1
// and 2 of a step are independent; split, each needs far fewer registers than the fused pass, so
// more CTAs stay resident per SM.
//
// Ring fields of step r (the rows each stage consumes), by part:
//   x-windows:  bvx(r-1) bvz(r) [0, 1, 2]   avx(r-1) avz(r) [0, 2]
//   stage-1 z-tap rows (r-4): bvx bvz [0, 1, 2]   avx avz [0, 2]
//   stage-1 own (r-4): btxx btzz btxz [0, 1]  atxx atzz atxz [0, 2]  lam mu [all]
//                      kpp kps, images pp ps [0, 2]
//   stage-2 own (r-8): b [all]  bvz, illumination [0, 1]  avx avz [0, 2]
// (bvx(r-8) is w_bvx[0]; the adjoint own velocities come from the ring because the windows carry
// the residual.)
template <int P>
struct BwdPairLayout;
template <>
struct BwdPairLayout<0> {
  enum : int { BVXW = 0, BVZW, AVXW, AVZW, BVX4, BVZ4, AVX4, AVZ4, BTXX, BTZZ, BTXZ, ATXX, ATZZ,
               ATXZ, LAM, MU, KPP, KPS, IPP, IPS, B8, BVZ8, AVX8, AVZ8, IL8, NF };
};
template <>
struct BwdPairLayout<1> {
  enum : int { BVXW = 0, BVZW, BVX4, BVZ4, BTXX, BTZZ, BTXZ, LAM, MU, B8, BVZ8, IL8, NF,
               AVXW = -1, AVZW = -1, AVX4 = -1, AVZ4 = -1, ATXX = -1, ATZZ = -1, ATXZ = -1,
               KPP = -1, KPS = -1, IPP = -1, IPS = -1, AVX8 = -1, AVZ8 = -1 };
};
template <>
struct BwdPairLayout<2> {
  enum : int { AVXW = 0, AVZW, BVXW, BVZW, AVX4, AVZ4, BVX4, BVZ4, ATXX, ATZZ, ATXZ, LAM, MU, KPP,
               KPS, IPP, IPS, B8, AVX8, AVZ8, NF, BTXX = -1, BTZZ = -1, BTXZ = -1, BVZ8 = -1,
               IL8 = -1 };
};
__host__ __device__ constexpr int bwd_pair_fields(int part) {
  return part == 0 ? (int)BwdPairLayout<0>::NF
                   : part == 1 ? (int)BwdPairLayout<1>::NF : (int)BwdPairLayout<2>::NF;
}
constexpr int kBwdPairFields = BwdPairLayout<0>::NF;
// Stage-2 z-tap rows (btxz, btzz of the reconstruction; M, PzLx of the adjoint), written by stage
// 1 for its row and read by stage 2 four steps later: a circular buffer of 6 rows (rows r-9 ..
// r-4 are distinct slots, so the write of step r never meets a read of step r-1 still in flight).
constexpr int kBwdPairZDepth = 6;
__host__ __device__ constexpr int bwd_pair_z2(int part) { return part == 0 ? 4 : 2; }
__host__ __device__ constexpr int bwd_pair_z2_rows(int part) {
  return bwd_pair_z2(part) * kBwdPairZDepth;
}

template <int kT, int kD, int kMinB, int kPart = 0>
__global__ void __launch_bounds__(kT, kMinB) k_bwd_pair(BwdFusedArgs a) {
  using L = BwdPairLayout<kPart>;
  constexpr bool kRec = kPart != 2, kAdj = kPart != 1;
  constexpr int NF = L::NF, ROW = pair_row(kT), NZ2 = bwd_pair_z2(kPart);
  // z-tap rows of the circular buffer: reconstruction at 0-1, adjoint after them
  constexpr int ZR = 0, ZA = kRec ? 2 : 0;
  extern __shared__ __align__(16) float smem[];
  float *ring = smem;
  float *zc = ring + (size_t)kD * NF * ROW;  // [kBwdPairZDepth][NZ2][ROW]
  unsigned long long *bars = (unsigned long long *)(zc + NZ2 * kBwdPairZDepth * ROW);
  int *s_tr = (int *)(bars + 8);
  int *s_has = s_tr + 16;
  float *s_rz = (float *)(s_has + 16), *s_rx = s_rz + 16;
  const int s = blockIdx.z, t = threadIdx.x;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int zs = blockIdx.x * a.tz;
  const int x0 = blockIdx.y * a.xr, x1 = min(x0 + a.xr, d.nxp);
  if (x0 >= d.nxp) return;
  if (__syncthreads_or(t == 0 && pair_err_raised(a.err))) return;  // whole CTA
  const int ld = d.ld, nop = d.nop, pml = d.pml;
  const long long fbase = d.slot * s;
  const long long ibase = (long long)s * d.wnx_max * d.ild;
  const int z0 = zs - 8 + 2 * t;
  const int pi = t + 2;
  const bool c1 = z0 >= zs - 4 && z0 < zs + a.tz + 4;
  const bool c2 = z0 >= zs && z0 < zs + a.tz && z0 < d.nzp;
  const bool u0 = z0 >= nop && z0 < d.nzp - nop, u1 = z0 + 1 >= nop && z0 + 1 < d.nzp - nop;
  const bool i0 = z0 >= pml && z0 < d.nzp - pml, i1 = z0 + 1 >= pml && z0 + 1 < d.nzp - pml;
  const ShotDev sh = a.shots[s];
  const int re = sh.igz - z0;  // receiver column relative to the pair
  const bool rec_col = kAdj && (re == 0 || re == 1);
  const bool rec_near = kAdj && re >= -4 && re <= 5;
  const float *res_z = a.res_vz + (long long)s * d.max_ntr * d.nt + a.it;
  const float *res_x = a.res_vx + (long long)s * d.max_ntr * d.nt + a.it;
  const int *rmap = a.rmap + (long long)s * d.nxp_max;
  const float dtdx = d.dt / d.dx, dtdz = d.dt / d.dz;
  const float rdx = 1.0f / d.dx, rdz = 1.0f / d.dz;
  float *img_pp = a.img, *img_ps = a.img + a.img_plane, *img_il = a.img + 2 * a.img_plane;

  // ring fields (the thread owning field f issues its row copies)
  const int lane = t & 31;
  // ring field of this thread: warp w, lane l owns field w + W l (W warps), so every warp issues
  // a share of a slot's copies
  const int my_f = (t >> 5) + (kT / 32) * lane;
  RingField fd{nullptr, 0, 0, d.nxp};
  {
    struct Src {
      int f;
      const float *p;
      int lag;
      bool img;
    };
    const Src tab[25] = {{L::BVXW, a.ra.vx, 1, false},  {L::BVZW, a.ra.vz, 0, false},
                         {L::AVXW, a.aa.vx, 1, false},  {L::AVZW, a.aa.vz, 0, false},
                         {L::BVX4, a.ra.vx, 4, false},  {L::BVZ4, a.ra.vz, 4, false},
                         {L::AVX4, a.aa.vx, 4, false},  {L::AVZ4, a.aa.vz, 4, false},
                         {L::BTXX, a.ra.txx, 4, false}, {L::BTZZ, a.ra.tzz, 4, false},
                         {L::BTXZ, a.ra.txz, 4, false}, {L::ATXX, a.aa.txx, 4, false},
                         {L::ATZZ, a.aa.tzz, 4, false}, {L::ATXZ, a.aa.txz, 4, false},
                         {L::LAM, a.p.lam, 4, false},   {L::MU, a.p.mu, 4, false},
                         {L::KPP, a.p.kpp, 4, false},   {L::KPS, a.p.kps, 4, false},
                         {L::IPP, img_pp, 4, true},     {L::IPS, img_ps, 4, true},
                         {L::B8, a.p.b, 8, false},      {L::BVZ8, a.ra.vz, 8, false},
                         {L::AVX8, a.aa.vx, 8, false},  {L::AVZ8, a.aa.vz, 8, false},
                         {L::IL8, img_il, 8, true}};
#pragma unroll
    for (int q = 0; q < 25; q++)
      if (tab[q].f >= 0 && my_f == tab[q].f) {
        // image rows: grid row x is image row x - pml of the slot's plane
        fd.src = tab[q].img ? tab[q].p + ibase - (long long)pml * ld : tab[q].p + fbase;
        fd.lag = tab[q].lag;
        fd.lo = tab[q].img ? pml : 0;
        fd.hi = tab[q].img ? d.nxp - pml : d.nxp;
      }
  }
  if (t == 0) {
    for (int k = 0; k < kD; k++) mbar_init(&bars[k], kT / 32);  // one arrival per warp
    mbar_fence_init();
  }
  if (rec_col) {  // residuals of rows x0-9 .. x0-1 and trace indexes of rows x0 .. x0+7 (direct;
                  // the march fetches the rest ahead)
    for (int q = x0 - 9; q < x0; q++) {
      const int tr = (q >= 0 && q < d.nxp) ? rmap[q] : -1;
      s_has[q & 15] = tr >= 0;
      if (tr >= 0) {
        s_rz[q & 15] = res_z[(long long)tr * d.nt];
        s_rx[q & 15] = res_x[(long long)tr * d.nt];
      }
    }
    for (int q = x0; q < x0 + 8; q++) s_tr[q & 15] = (q >= 0 && q < d.nxp) ? rmap[q] : -1;
  }
  __syncthreads();
  const int rs0 = x0 - 8;
  for (int j = 0; j < kD - 1; j++)
    issue_slot_warp<kT>(fd, ring + (size_t)j * NF * ROW, my_f, &bars[j], rs0 + j, ld, zs, lane);

  const float2 zero2 = make_float2(0.f, 0.f);
  float2 w_bvx[8], w_bvz[8];               // stage-1 x-windows (strains / reconstruction)
  float2 w_avx[kAdj ? 8 : 1], w_avz[kAdj ? 8 : 1];
  float2 w_btxx[kRec ? 8 : 1], w_btxz[kRec ? 9 : 1];  // stage-2 x-windows
  float2 w_PL[kAdj ? 8 : 1], w_M[kAdj ? 9 : 1];
#pragma unroll
  for (int i = 0; i < 8; i++) w_bvx[i] = w_bvz[i] = zero2;
  if constexpr (kAdj) {
#pragma unroll
    for (int i = 0; i < 8; i++) w_avx[i] = w_avz[i] = w_PL[i] = zero2;
#pragma unroll
    for (int i = 0; i < 9; i++) w_M[i] = zero2;
  }
  if constexpr (kRec) {
#pragma unroll
    for (int i = 0; i < 8; i++) w_btxx[i] = zero2;
#pragma unroll
    for (int i = 0; i < 9; i++) w_btxz[i] = zero2;
  }
  // circular z-tap slot of stage 1's row r-4 (stage 2 reads row r-8, two slots further on)
  int zw = ((rs0 - 4) % kBwdPairZDepth + kBwdPairZDepth) % kBwdPairZDepth;

  RingCursor<kD> cur;
  bool ok = true, aborted = false;
  // Two row steps per loop iteration let the compiler rename half of the window shifts away
  // where the registers allow it (the split parts); the fused pass is at its register limit.
  constexpr int kUnroll = kPart == 0 ? 1 : 2;
#pragma unroll kUnroll
  for (int r = rs0; r < x1 + 8; r++) {
    // A wait that gives up skips the step's work; the barrier below is a vote, so every thread
    // leaves the march together (none is left waiting at a barrier).
    ok = mbar_wait(&bars[cur.slot], cur.phase);
    const float *S = ring + (size_t)cur.slot * NF * ROW;
    auto F2 = [&](int f) -> float2 { return reinterpret_cast<const float2 *>(S + f * ROW)[pi]; };
    auto ROWP = [&](int f) { return reinterpret_cast<const float2 *>(S + f * ROW); };
    if (rec_col) {
      // residual of row r + 8 (its trace index landed 8 steps ago), trace index of row r + 16;
      // one commit group per step, waited for 7 steps later
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
    if (ok) {
      push2(w_bvx, F2(L::BVXW));
      push2(w_bvz, F2(L::BVZW));
      if constexpr (kAdj) {
        float2 n_avx = F2(L::AVXW), n_avz = F2(L::AVZW);
        if (rec_col) {  // the residual enters the stencil values of the receiver column
          const int qa = r - 1, qz = r;
          if (qa >= 0 && qa < d.nxp && s_has[qa & 15]) {
            if (re == 0) n_avx.x += s_rx[qa & 15]; else n_avx.y += s_rx[qa & 15];
          }
          if (qz >= 0 && qz < d.nxp && s_has[qz & 15]) {
            if (re == 0) n_avz.x += s_rz[qz & 15]; else n_avz.y += s_rz[qz & 15];
          }
        }
        push2(w_avx, n_avx);
        push2(w_avz, n_avz);
      }
    }
    // ---- stage 1: stresses of row r1 = r - 4, images ----------------------------------------
    const int r1 = r - 4;
    float2 btxx = zero2, btzz = zero2, btxz = zero2, PL = zero2, M = zero2, PzLx = zero2;
    if (ok && c1 && r >= x0 && r1 >= 0 && r1 < d.nxp) {
      const bool own = c2 && r1 >= x0 && r1 < x1;
      const bool x_int = r1 >= pml && r1 < d.nxp - pml;
      const float2 lam = F2(L::LAM), mu = F2(L::MU);
      if constexpr (kRec) {
        btxx = F2(L::BTXX);
        btzz = F2(L::BTZZ);
        btxz = F2(L::BTXZ);
      }
      float2 gxx = zero2, gzz = zero2, gsh = zero2;  // strains: Dx vx, Dz vz, Dz vx + Dx vz
      if (x_int) {
        const Z10 zbx = z10(ROWP(L::BVX4), pi);
        const Z10 zbz = z10(ROWP(L::BVZ4), pi);
        const float sa0 = dxw_x(w_bvx), sa1 = dxw_y(w_bvx);
        const float sf0 = dxw_x(w_bvz), sf1 = dxw_y(w_bvz);
        const float sb0 = dzm<0>(zbz), sb1 = dzm<1>(zbz);
        const float se0 = dzp<0>(zbx), se1 = dzp<1>(zbx);
        if constexpr (kRec) {
          const float dir = -1.0f;
          if (i0) {
            const float l2m = lam.x + 2.0f * mu.x;
            btxx.x = btxx.x + (dir * l2m * dtdx * sa0 + dir * lam.x * dtdz * sb0);
            btzz.x = btzz.x + (dir * lam.x * dtdx * sa0 + dir * l2m * dtdz * sb0);
            btxz.x = btxz.x + (dir * mu.x * dtdx * sf0 + dir * mu.x * dtdz * se0);
          }
          if (i1) {
            const float l2m = lam.y + 2.0f * mu.y;
            btxx.y = btxx.y + (dir * l2m * dtdx * sa1 + dir * lam.y * dtdz * sb1);
            btzz.y = btzz.y + (dir * lam.y * dtdx * sa1 + dir * l2m * dtdz * sb1);
            btxz.y = btxz.y + (dir * mu.y * dtdx * sf1 + dir * mu.y * dtdz * se1);
          }
          if (own) {
            const long long k = fbase + (long long)r1 * ld + z0;
            *reinterpret_cast<float2 *>(a.rb.txx + k) = btxx;
            *reinterpret_cast<float2 *>(a.rb.tzz + k) = btzz;
            *reinterpret_cast<float2 *>(a.rb.txz + k) = btxz;
          }
        }
        if constexpr (kAdj) {
          if (i0) {
            gxx.x = sa0 * rdx;
            gzz.x = sb0 * rdz;
            gsh.x = se0 * rdz + sf0 * rdx;
          }
          if (i1) {
            gxx.y = sa1 * rdx;
            gzz.y = sb1 * rdz;
            gsh.y = se1 * rdz + sf1 * rdx;
          }
        }
      }
      if constexpr (kAdj) {
        float2 atxx = zero2, atzz = zero2, atxz = zero2;
        if (r1 >= nop && r1 < d.nxp - nop) {
          const Z10 zax = z10(ROWP(L::AVX4), pi);
          const Z10 zaz = z10(ROWP(L::AVZ4), pi);
          float sb0 = dzm<0>(zaz), sb1 = dzm<1>(zaz);
          float se0 = dzp<0>(zax), se1 = dzp<1>(zax);
          if (rec_near && s_has[r1 & 15]) {  // residual of the receiver cell in the z-taps
            const float rz = s_rz[r1 & 15], rx = s_rx[r1 & 15];
            sb0 += rz * (coef_or0(re + 1) - coef_or0(-re));
            sb1 += rz * (coef_or0(re) - coef_or0(1 - re));
            se0 += rx * (coef_or0(re) - coef_or0(1 - re));
            se1 += rx * (coef_or0(re - 1) - coef_or0(2 - re));
          }
          const float sa0 = dxw_x(w_avx), sa1 = dxw_y(w_avx);
          const float sf0 = dxw_x(w_avz), sf1 = dxw_y(w_avz);
          const float2 oxx = F2(L::ATXX), ozz = F2(L::ATZZ), oxz = F2(L::ATXZ);
          if (u0) {
            atxx.x = oxx.x + -dtdx * sa0;
            atzz.x = ozz.x + -dtdz * sb0;
            atxz.x = oxz.x + (-dtdx * sf0 + -dtdz * se0);
          }
          if (u1) {
            atxx.y = oxx.y + -dtdx * sa1;
            atzz.y = ozz.y + -dtdz * sb1;
            atxz.y = oxz.y + (-dtdx * sf1 + -dtdz * se1);
          }
          if (own) {
            const long long k = fbase + (long long)r1 * ld + z0;
            *reinterpret_cast<float2 *>(a.ab.txx + k) = atxx;
            *reinterpret_cast<float2 *>(a.ab.tzz + k) = atzz;
            *reinterpret_cast<float2 *>(a.ab.txz + k) = atxz;
          }
        }
        {
          const float l2m0 = lam.x + 2.0f * mu.x, l2m1 = lam.y + 2.0f * mu.y;
          PL = make_float2(l2m0 * atxx.x + lam.x * atzz.x, l2m1 * atxx.y + lam.y * atzz.y);
          M = make_float2(mu.x * atxz.x, mu.y * atxz.y);
          PzLx = make_float2(l2m0 * atzz.x + lam.x * atxx.x, l2m1 * atzz.y + lam.y * atxx.y);
        }
        if (own && x_int) {  // doimage_gradient, FD2DGPU.cu:3245-3263
          const float2 kpp = F2(L::KPP), kps = F2(L::KPS), ipp = F2(L::IPP), ips = F2(L::IPS);
          float2 npp = ipp, nps = ips;
          if (i0) {
            npp.x = ipp.x + kpp.x * ((gxx.x + gzz.x) * (atxx.x + atzz.x));
            nps.x = ips.x + kps.x * (-2.0f * (gxx.x * atzz.x + gzz.x * atxx.x) + gsh.x * atxz.x);
          }
          if (i1) {
            npp.y = ipp.y + kpp.y * ((gxx.y + gzz.y) * (atxx.y + atzz.y));
            nps.y = ips.y + kps.y * (-2.0f * (gxx.y * atzz.y + gzz.y * atxx.y) + gsh.y * atxz.y);
          }
          const long long o = ibase + (long long)(r1 - pml) * d.ild + z0;
          *reinterpret_cast<float2 *>(img_pp + o) = npp;
          *reinterpret_cast<float2 *>(img_ps + o) = nps;
        }
      }
    }
    if constexpr (kRec) {
      push2(w_btxx, btxx);
      push2(w_btxz, btxz);
    }
    if constexpr (kAdj) {
      push2(w_PL, PL);
      push2(w_M, M);
    }
    {  // z-tap rows of row r - 4 for stage 2 four steps on
      float *zwb = zc + zw * NZ2 * ROW;
      if constexpr (kRec) {
        reinterpret_cast<float2 *>(zwb + ZR * ROW)[pi] = btxz;
        reinterpret_cast<float2 *>(zwb + (ZR + 1) * ROW)[pi] = btzz;
      }
      if constexpr (kAdj) {
        reinterpret_cast<float2 *>(zwb + ZA * ROW)[pi] = M;
        reinterpret_cast<float2 *>(zwb + (ZA + 1) * ROW)[pi] = PzLx;
      }
    }
    const float *zb =
        zc + (zw >= kBwdPairZDepth - 2 ? zw - (kBwdPairZDepth - 2) : zw + 2) * NZ2 * ROW;
    zw = zw == kBwdPairZDepth - 1 ? 0 : zw + 1;
    // ---- the step's barrier, the refill -------------------------------------------------------
    if (__syncthreads_or(!ok)) {
      aborted = true;
      break;
    }
    {  // every warp issues its share of the slot's copies
      const int ps = cur.slot == 0 ? kD - 1 : cur.slot - 1;
      issue_slot_warp<kT>(fd, ring + (size_t)ps * NF * ROW, my_f, &bars[ps], r + kD - 1, ld, zs,
                          lane);
    }
    // ---- stage 2: velocities of row r2 = r - 8, illumination ---------------------------------
    const int r2 = r - 8;
    if (c2 && r2 >= x0 && r2 < x1) {
      const long long k = fbase + (long long)r2 * ld + z0;
      const float2 bb = F2(L::B8);
      if constexpr (kRec) {
        if (r2 >= pml && r2 < d.nxp - pml) {
          const Z10 ztxz = z10(reinterpret_cast<const float2 *>(zb + ZR * ROW), pi);
          const Z10 ztzz = z10(reinterpret_cast<const float2 *>(zb + (ZR + 1) * ROW), pi);
          const float2 ovx = w_bvx[0], ovz = F2(L::BVZ8), il = F2(L::IL8);
          float2 vx = ovx, vz = ovz, nil = il;
          if (i0) {
            const float cbx = bb.x * dtdx, cbz = bb.x * dtdz;
            const float ax = dxw_x(w_btxx), fx = dxw_x(w_btxz);
            const float bz = dzm<0>(ztxz), ez = dzp<0>(ztzz);
            vx.x = ovx.x + (-cbx * ax + -cbz * bz);
            vz.x = ovz.x + (-cbx * fx + -cbz * ez);
            nil.x = il.x + (vx.x * vx.x + vz.x * vz.x);
          }
          if (i1) {
            const float cbx = bb.y * dtdx, cbz = bb.y * dtdz;
            const float ax = dxw_y(w_btxx), fx = dxw_y(w_btxz);
            const float bz = dzm<1>(ztxz), ez = dzp<1>(ztzz);
            vx.y = ovx.y + (-cbx * ax + -cbz * bz);
            vz.y = ovz.y + (-cbx * fx + -cbz * ez);
            nil.y = il.y + (vx.y * vx.y + vz.y * vz.y);
          }
          *reinterpret_cast<float2 *>(a.rb.vx + k) = vx;
          *reinterpret_cast<float2 *>(a.rb.vz + k) = vz;
          *reinterpret_cast<float2 *>(img_il + ibase + (long long)(r2 - pml) * d.ild + z0) = nil;
        }
      }
      if constexpr (kAdj) {
        if (r2 >= nop && r2 < d.nxp - nop) {
          const Z10 zm = z10(reinterpret_cast<const float2 *>(zb + ZA * ROW), pi);
          const Z10 zp = z10(reinterpret_cast<const float2 *>(zb + (ZA + 1) * ROW), pi);
          float2 vx = zero2, vz = zero2;
          const float2 ovx = F2(L::AVX8), ovz = F2(L::AVZ8);
          if (u0) {
            const float cbx = bb.x * dtdx, cbz = bb.x * dtdz;
            const float t_x = dxw_x(w_PL), s_xz = dxw_x(w_M);
            const float t_xz = dzm<0>(zm), s_z = dzp<0>(zp);
            vx.x = ovx.x + (-cbx * t_x + -cbz * t_xz);
            vz.x = ovz.x + (-cbx * s_xz + -cbz * s_z);
          }
          if (u1) {
            const float cbx = bb.y * dtdx, cbz = bb.y * dtdz;
            const float t_x = dxw_y(w_PL), s_xz = dxw_y(w_M);
            const float t_xz = dzm<1>(zm), s_z = dzp<1>(zp);
            vx.y = ovx.y + (-cbx * t_x + -cbz * t_xz);
            vz.y = ovz.y + (-cbx * s_xz + -cbz * s_z);
          }
          *reinterpret_cast<float2 *>(a.ab.vx + k) = vx;
          *reinterpret_cast<float2 *>(a.ab.vz + k) = vz;
        }
      }
    }
    if (rec_col) cp_async_wait<6>();
    cur.advance();
  }
  pair_exit<kD>(bars, cur, aborted, ok, a.err);
  cp_async_wait<0>();
}

}  // namespace ds2d
