// Host engine and C ABI (include/ds2d.h) of the B200 DS2D time-stepping path.
//
// The engine owns all device memory of a run: the full models and images, and a batch of
// "slots" (one per resident shot) with the shot's padded parameters, wavefields, strips and
// window images.  One call (ds2d_forward / ds2d_elsrtm / ds2d_rtm) processes its shots in
// batches of opts.max_shots; every kernel launch covers all shots of the batch.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ds2d.h"
#include "ds2d_acoustic.cuh"
#include "ds2d_filter.cuh"
#include "ds2d_fused.cuh"
#include "ds2d_pair.cuh"
#include "ds2d_step.cuh"
#include "ds2d_tblock.cuh"
#include "ds2d_bwdws.cuh"
#include "ds2d_bwdbulk.cuh"

using namespace ds2d;

namespace {

// Ring depths the fused kernels are instantiated for, and the default (option "ring").
constexpr int kRingDepths[3] = {2, 4, 8};
constexpr int kDefaultRing = 4;

using FwdFn = void (*)(FwdFusedArgs);
using BwdFn = void (*)(BwdFusedArgs);

// Fused ring kernels by boundary, ring depth and occupancy target (option "occ": 0 = registers
// for 6 forward / 3 backward CTAs per SM, 1 = capped for 8 forward / 4 backward CTAs per SM).
template <int kD, int kF, int kB>
FwdFn fwd_pick(bool rbc) { return rbc ? k_fwd_ring<false, kD, kF> : k_fwd_ring<true, kD, kF>; }
template <int kD, int kF, int kB>
BwdFn bwd_pick(bool rbc) { return rbc ? k_bwd_ring<false, kD, kB> : k_bwd_ring<true, kD, kB>; }

// Wider CTAs (option "cta"): 192 threads = 176 output columns per z-strip, instantiated for the
// default ring depth and occupancy target only (4 forward / 2 backward CTAs per SM, the same
// warps per SM as 128-thread CTAs at 6 / 3).
constexpr int kWideCta = 192;

FwdFn fwd_ring_fn(bool rbc, int depth, int occ = 0, int cta = kFB) {
  if (cta == kWideCta && depth == 4 && occ == 0)
    return rbc ? k_fwd_ring<false, 4, 4, kWideCta> : k_fwd_ring<true, 4, 4, kWideCta>;
  switch (depth * 2 + (occ ? 1 : 0)) {
    case 4: return fwd_pick<2, 6, 3>(rbc);
    case 5: return fwd_pick<2, 8, 4>(rbc);
    case 8: return fwd_pick<4, 6, 3>(rbc);
    case 9: return fwd_pick<4, 8, 4>(rbc);
    case 17: return fwd_pick<8, 8, 4>(rbc);
    default: return fwd_pick<8, 6, 3>(rbc);
  }
}

// Born-modelling modes of the forward ring kernel (1 background + Born source, 2 first-order
// scattered set, 3 second-order set), default ring depth and CTA width; their larger rings allow
// 3-4 CTAs per SM, so the register budget is set for 4.
#ifndef DS2D_BORN_RING
#define DS2D_BORN_RING 4
#endif
constexpr int kBornRing = DS2D_BORN_RING;  // ring depth of the Born-modelling modes

FwdFn fwd_mode_fn(bool rbc, int mode) {
  switch (mode) {
    case 1: return rbc ? k_fwd_ring<false, kBornRing, 4, kFB, 1> : k_fwd_ring<true, kBornRing, 4, kFB, 1>;
    case 2: return rbc ? k_fwd_ring<false, kBornRing, 4, kFB, 2> : k_fwd_ring<true, kBornRing, 4, kFB, 2>;
    default: return rbc ? k_fwd_ring<false, kBornRing, 4, kFB, 3> : k_fwd_ring<true, kBornRing, 4, kFB, 3>;
  }
}

using ScatFn = void (*)(BwdScatArgs);
ScatFn bwd_scat_fn(bool rbc) { return rbc ? k_bwd_scat_ring<false, 4, 4> : k_bwd_scat_ring<true, 4, 4>; }

BwdFn bwd_ring_fn(bool rbc, int depth, int occ = 0, int cta = kFB, bool one = false) {
  if (one && depth == 4 && occ == 0) {  // one barrier per row step
    if (rbc)
      return cta == kWideCta ? k_bwd_ring<false, 4, 2, kWideCta, true> : k_bwd_ring<false, 4, 3, kFB, true>;
    return cta == kWideCta ? k_bwd_ring<true, 4, 2, kWideCta, true> : k_bwd_ring<true, 4, 3, kFB, true>;
  }
  if (cta == kWideCta && depth == 4 && occ == 0)
    return rbc ? k_bwd_ring<false, 4, 2, kWideCta> : k_bwd_ring<true, 4, 2, kWideCta>;
  switch (depth * 2 + (occ ? 1 : 0)) {
    case 4: return bwd_pick<2, 6, 3>(rbc);
    case 5: return bwd_pick<2, 8, 4>(rbc);
    case 8: return bwd_pick<4, 6, 3>(rbc);
    case 9: return bwd_pick<4, 8, 4>(rbc);
    case 17: return bwd_pick<8, 8, 4>(rbc);
    default: return bwd_pick<8, 6, 3>(rbc);
  }
}

// Setup of one batch of slots: window of the full model with edge replication
// (FD2DGPU.cu:122-138, :234-250), optional project random band, PML damping (:444-494, profile
// ((pml-i)/pml)^4 scaled by log10(1/rr) * 5 vp / (2 pml)), moduli with the reference's rho
// (:1117-1125), imaging weights -2 vp^2 rho and -2 vs^2 rho (:3257-3258), image windows
// (:1324-1333).
struct SetupArgs {
  Dims d;
  const float *vp_all, *vs_all, *rho_all, *pp_all, *ps_all;
  const ShotDev *shots;
  float *b, *lam, *mu, *dampx, *dampz, *kpp, *kps, *dmp, *dms;
  double L;  // log10(1/rr)
  unsigned long long seed;
  int shot_base;
};

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  // SplitMix64 finalizer (Steele, Lea, Flood 2014).
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float band_factor(unsigned long long seed, int shot, int ix, int iz) {
  unsigned long long h =
      splitmix64(seed ^ (0xD1B54A32D192ED03ull * (unsigned long long)(unsigned)(shot + 1)));
  h = splitmix64(h ^ (((unsigned long long)(unsigned)ix << 32) | (unsigned)iz));
  const float u = (float)(h >> 40) * (1.0f / 16777216.0f);
  return fmaf(0.4f, u, 0.6f);
}

__global__ void k_setup(SetupArgs a) {
  const int s = blockIdx.z;
  const Dims d = slot_dims(a.d, a.shots[s]);
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = blockIdx.y;
  if (iz >= d.ld) return;
  const long long k = d.slot * s + (long long)ix * d.ld + iz;
  if (iz >= d.nzp || ix >= d.nxp) {  // row padding, or beyond this slot's (narrower) window
    a.b[k] = 0.f; a.lam[k] = 0.f; a.mu[k] = 0.f;
    if (a.dampx) { a.dampx[k] = 0.f; a.dampz[k] = 0.f; }
    a.kpp[k] = 0.f; a.kps[k] = 0.f;
    if (a.dmp) { a.dmp[k] = 0.f; a.dms[k] = 0.f; }
    return;
  }
  const int pml = d.pml;
  const int jx = min(max(ix - pml, 0), d.wnx - 1), jz = min(max(iz - pml, 0), d.wnz - 1);
  const long long src = (long long)(a.shots[s].win_left + jx) * d.allnz + jz;
  float p = a.vp_all[src], sv = a.vs_all[src];
  const bool band = ix < pml || ix >= d.nxp - pml || iz < pml || iz >= d.nzp - pml;
  if (d.rbc && band) {
    const float f = band_factor(a.seed, a.shot_base + s, ix, iz);
    p = __fmul_rn(p, f);
    sv = __fmul_rn(sv, f);
  }
  const float r = a.rho_all ? a.rho_all[src] : 2000.0f;
  const float vp2 = __fmul_rn(p, p), vs2 = __fmul_rn(sv, sv);
  const float lam = __fmul_rn(r, __fsub_rn(vp2, __fmul_rn(2.0f, vs2)));
  const float mu = __fmul_rn(r, vs2);
  a.b[k] = (float)(1.0 / (double)r);
  a.lam[k] = lam;
  a.mu[k] = mu;
  a.kpp[k] = __fmul_rn(__fmul_rn(__fmul_rn(-2.0f, p), p), r);
  a.kps[k] = __fmul_rn(__fmul_rn(__fmul_rn(-2.0f, sv), sv), r);
  if (a.dampx) {
    double dx = 0, dz = 0;
    if (!d.rbc) {
      const double c = __dmul_rn(a.L, __ddiv_rn(__dmul_rn(5.0, (double)p), 2.0 * pml));
      auto prof = [&](int n) {
        const double t = (double)n / pml;
        const double t2 = __dmul_rn(t, t);
        return __dmul_rn(c, __dmul_rn(t2, t2));
      };
      if (ix < pml) dx = prof(pml - ix);
      if (ix > d.nxp - pml) dx = prof(ix - (d.nxp - pml));
      if (iz < pml) dz = prof(pml - iz);
      if (iz > d.nzp - pml) dz = prof(iz - (d.nzp - pml));
    }
    a.dampx[k] = (float)dx;
    a.dampz[k] = (float)dz;
  }
  if (a.dmp) {
    a.dmp[k] = a.pp_all[src];
    a.dms[k] = a.ps_all[src];
  }
}

struct Arena {
  std::vector<void *> ptrs;
  ~Arena() { release(); }
  void release() {
    for (void *p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

// Per-launch device timing (profiling mode): one event pair per launch, folded per kernel name.
struct ProfRec {
  const char *name;
  int ev;
  double bytes;
};

struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  std::vector<ProfRec> recs;
  int used = 0;
  ~Profiler() {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
  int take() {
    if (used + 2 > (int)pool.size()) {
      for (int i = 0; i < 256; i++) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        pool.push_back(e);
      }
    }
    used += 2;
    return used - 2;
  }
};

}  // namespace

struct ds2d_ctx {
  ds2d_grid g{};
  ds2d_opts o{};
  Dims d{};
  int B = 1;
  cudaStream_t own = nullptr, stream = nullptr;
  std::string err;
  double last_updates = 0;
  long long last_launches = 0;

  // full-size arrays
  float *vp_all = nullptr, *vs_all = nullptr, *rho_all = nullptr;
  float *pp_all = nullptr, *ps_all = nullptr, *wavelet = nullptr;
  float *images = nullptr;  // [7][allnx][allnz]
  bool models_set = false, wavelet_set = false, image_set = false;

  // per-slot arrays
  Par par{};
  float *p_b = nullptr, *p_lam = nullptr, *p_mu = nullptr, *p_dampx = nullptr, *p_dampz = nullptr;
  float *p_kpp = nullptr, *p_kps = nullptr, *p_dmp = nullptr, *p_dms = nullptr;
  Wave fw{}, b1{}, b2{}, abk{}, bbk{};
  Strain e{}, be{};
  float *ov_s[3] = {nullptr, nullptr, nullptr}, *ov_v[2] = {nullptr, nullptr};
  Strips st_a{}, st_b{};
  int st_a_steps = 0, st_b_steps = 0;  // time steps the strip buffers hold
  // background checkpoints of the PML L^T (option "ac_ckpt")
  int opt_ac_ckpt = 0;
  void *ckpt = nullptr;
  float *ckpt_scale = nullptr;
  unsigned *ckpt_amax = nullptr;
  size_t ckpt_bytes = 0;
  ShotDev *d_shots = nullptr;
  int *d_rmap = nullptr;
  float *rec[8] = {};          // obs/adj z,x | scattered z,x | scattered2 z,x | residual z,x
  float *img_slot = nullptr;   // [7][B][wnx][wnz]
  double *d_mis = nullptr;
  bool have_elsrtm = false, have_rtm = false;
  // Tuning knobs (ds2d_set_option): fused single-pass forward step, rows per CTA of the fused
  // kernels.
  int opt_fused = 1, opt_xr = 128;
  int opt_adjoint_born = 0;  // scattered adjoint of ELSRTM (off = the reference's observed runs)
  int opt_ring = kDefaultRing;  // cp.async ring depth of the fused kernels (0 = no ring)
  int opt_occ = 0;           // occupancy target of the ring kernels (see fwd_ring_fn)
  int opt_cta = 0;           // threads per CTA of the ring kernels: 0 auto, 128 or 192
  bool ring_ok = true;       // batch arrays fit the ring kernels' 32-bit offsets
  // Pair-blocked bulk-copy kernels of the random-boundary RTM step (ds2d_pair.cuh): option
  // "pair" (2 forward only: the default; 1 forward and backward; 0 off), "pair_cta" (backward CTA
  // width: 0 auto, 256 or 160), "pair_xr" (rows per CTA: 0 = chosen to fill whole waves).
  int opt_pair = 2, opt_pair_cta = 0, opt_pair_fcta = 0, opt_pair_xr = 0, opt_pair_split = 0;
  int opt_ac_pair = 1, opt_ac_pair_cta = 0;  // acoustic steps on k_ac_pair / k_ac_rev_pair
  // Time-blocked forward launches (ds2d_tblock.cuh, random boundary): option "tb" = time steps
  // per launch (0 off, 1-4; default 2), "tb_cta" = threads per CTA (0 automatic, 256 or 512).
  int opt_tb = 2, opt_tb_cta = 0;
  int opt_tb_bulk = 1;       // option "tb_bulk": depth 1-2 rows by bulk copy (0 = per-thread cp.async)
  int occ_tb_bulk[2][2] = {};  // resident CTAs per SM of k_fwd_tb with bulk copies [256 / 512][depth - 1]
  // Warp-specialised backward step (ds2d_bwdws.cuh, random boundary): option "bwd_ws" = threads
  // per role (0 off, 96, 128 or 192; a CTA holds both roles).
  int opt_bwd_ws = 0;
  int opt_bwd_1b = 1;        // option "bwd_1b": one barrier per row step in k_bwd_ring / k_bwd_bulk
                             // (PML and random boundary)
  int opt_bwd_bulk = 1;      // option "bwd_bulk": k_bwd_bulk, operand rows by bulk copy (random
                             // boundary; the default, 0 = the per-thread cp.async ring of k_bwd_ring)
  int opt_bwd_cta = 0;       // option "bwd_cta": threads per CTA of k_bwd_bulk (0 automatic, 128 / 192 / 256)
  int occ_bulk[6] = {};      // resident CTAs per SM of k_bwd_bulk: [128 / 192 / 256 threads][one barrier]
  int occ_ws[3] = {};        // resident CTAs per SM of k_bwd_ws, 96 / 128 / 192 threads per role
  int occ_tb[2][4] = {};     // resident CTAs per SM of k_fwd_tb, [256 / 512 threads][depth - 1]
  // split backward: the two launches of a step as parallel branches (second stream, fork / join
  // events; parallel nodes in a captured graph)
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int *d_err = nullptr;      // error word raised by a pair kernel's bounded wait
  int num_sms = 148;
  // resident CTAs per SM: forward 256 / 64, backward 256 / 160 / 64, split parts 1 / 2
  int occ_pair[7] = {0, 0, 0, 0, 0, 0, 0};
  int occ_ac_pair[3] = {0, 0, 0};  // k_ac_pair, 256 / 192 / 128 threads
  int occ_ac_rev[2] = {0, 0};      // k_ac_rev_pair, 192 / 128 threads
  std::vector<int> h_nxp;    // padded window rows of each slot of the current batch
  int opt_pcg_switch = 970;  // ds2d_lsrtm_pcg: per-mille residual ratio that ends the network phase
  int opt_pcg_m = 8;         // ds2d_lsrtm_pcg: directions kept for explicit conjugation
  // Acoustic Born pair (LSRTM): background, scattered and adjoint states, Born overlay.
  float *ac[10] = {};        // bvx bvz bs | dvx dvz ds | yx yz ys | e
  float *ac_split[6] = {};   // with a PML: split stress s_x, s_z of background | scattered | adjoint
  float *ac2[6] = {};        // second (ping-pong) buffers of bvx bvz bs | dvx dvz ds (fused steps)
  double *dot_part = nullptr, *dot_out = nullptr;  // FP64 inner-product scratch
  // Work vectors of the LSRTM solver (model- and data-space), grown on demand.
  struct Vec {
    float *p = nullptr;
    size_t n = 0;
  };
  Vec vecs[64];  // 0-11 solver vectors, 16+ the flexible-CG direction window
  Wave fw2{}, abk2{};  // ping-pong partners of fw / abk for the fused kernels
  Wave b1_2{}, b2_2{};  // ping-pong partners of the scattered sets (fused ELSRTM forward)
  float *ov_s2[3] = {nullptr, nullptr, nullptr};  // Born source of b1 for b2 (fused forward)
  Wave *fw_cur = nullptr;  // buffer holding the latest forward state
  double batch_cells = 0, batch_wcells = 0;  // padded / interior cells of the current batch
  // CUDA graphs of whole batches (time loops included), keyed by everything baked into them.
  int opt_graph = 1;
  struct GraphEntry {
    long long key[6];
    cudaGraphExec_t exec;
    long long launches;
  };
  std::vector<GraphEntry> graphs;
  Profiler prof;
  Arena arena;
};

namespace {

thread_local std::string g_create_err = "";  // reported by ds2d_last_error(NULL)

int fail(ds2d_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(c, DS2D_E_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),  \
                  __FILE__, __LINE__);                                                     \
  } while (0)

int alloc(ds2d_ctx *c, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(c, DS2D_E_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  }
  c->arena.ptrs.push_back(*p);
  return DS2D_OK;
}

int alloc_slots(ds2d_ctx *c, float **p) {
  return alloc(c, (void **)p, sizeof(float) * (size_t)c->d.slot * c->B);
}

int alloc_wave(ds2d_ctx *c, Wave &w, bool adjoint) {
  int rc;
  float **sums[5] = {&w.vx, &w.vz, &w.txx, &w.tzz, &w.txz};
  for (float **p : sums)
    if ((rc = alloc_slots(c, p))) return rc;
  if (c->d.rbc) return DS2D_OK;
  // Split memory variables (only PML cells are touched).  The adjoint's txx / tzz are single
  // variables (FD2DGPU.cu:754-755 txx = txx_x, tzz = tzz_z).
  float **split_f[10] = {&w.vx_x, &w.vx_z, &w.vz_x, &w.vz_z, &w.txx_x,
                         &w.txx_z, &w.tzz_x, &w.tzz_z, &w.txz_x, &w.txz_z};
  float **split_a[6] = {&w.vx_x, &w.vx_z, &w.vz_x, &w.vz_z, &w.txz_x, &w.txz_z};
  if (adjoint) {
    for (float **p : split_a)
      if ((rc = alloc_slots(c, p))) return rc;
  } else {
    for (float **p : split_f)
      if ((rc = alloc_slots(c, p))) return rc;
  }
  return DS2D_OK;
}

int zero_wave(ds2d_ctx *c, const Wave &w, int nslots) {
  size_t bytes = sizeof(float) * (size_t)c->d.slot * nslots;
  const float *all[15] = {w.vx, w.vz, w.txx, w.tzz, w.txz, w.vx_x, w.vx_z, w.vz_x,
                          w.vz_z, w.txx_x, w.txx_z, w.tzz_x, w.tzz_z, w.txz_x, w.txz_z};
  for (const float *p : all)
    if (p) CK(cudaMemsetAsync((void *)p, 0, bytes, c->stream));
  return DS2D_OK;
}

int alloc_strips(ds2d_ctx *c, Strips &st, int steps) {
  int rc;
  st.prec = c->o.strip_precision;
  size_t elems = (size_t)c->B * steps * 2 * c->d.lb;
  size_t esz = st.prec == DS2D_STRIPS_F32 ? 4 : 2;
  if ((rc = alloc(c, &st.data, elems * esz))) return rc;
  if (st.prec != DS2D_STRIPS_F32) {
    size_t ns = (size_t)c->B * steps * 2 * c->d.nseg;
    if ((rc = alloc(c, (void **)&st.scale, ns * sizeof(float)))) return rc;
  }
  return DS2D_OK;
}

// Frees one arena allocation before the context's end (buffers whose size follows an option).
void release(ds2d_ctx *c, void *p) {
  if (!p) return;
  cudaFree(p);
  auto &v = c->arena.ptrs;
  v.erase(std::remove(v.begin(), v.end(), p), v.end());
}

// A strip buffer holding at least `steps` time steps (strips are indexed by the step within the
// buffer, so a larger one serves a shorter use).
int ensure_strips(ds2d_ctx *c, Strips &st, int &have, int steps) {
  if (st.data && have >= steps) return DS2D_OK;
  release(c, st.data);
  release(c, st.scale);
  st.data = nullptr;
  st.scale = nullptr;
  have = 0;
  int rc;
  if ((rc = alloc_strips(c, st, steps))) return rc;
  have = steps;
  return DS2D_OK;
}

int ensure_common(ds2d_ctx *c) {
  if (c->p_b) return DS2D_OK;
  int rc;
  float **ps[5] = {&c->p_b, &c->p_lam, &c->p_mu, &c->p_kpp, &c->p_kps};
  for (float **p : ps)
    if ((rc = alloc_slots(c, p))) return rc;
  if (!c->d.rbc) {
    if ((rc = alloc_slots(c, &c->p_dampx))) return rc;
    if ((rc = alloc_slots(c, &c->p_dampz))) return rc;
  }
  if ((rc = alloc_wave(c, c->fw, false))) return rc;
  if ((rc = alloc(c, (void **)&c->d_shots, sizeof(ShotDev) * c->B))) return rc;
  if ((rc = alloc(c, (void **)&c->d_rmap, sizeof(int) * (size_t)c->B * c->d.nxp))) return rc;
  size_t nrec = (size_t)c->B * c->d.max_ntr * c->d.nt;
  for (int i = 0; i < 2; i++)
    if ((rc = alloc(c, (void **)&c->rec[i], nrec * sizeof(float)))) return rc;
  c->par.b = c->p_b; c->par.lam = c->p_lam; c->par.mu = c->p_mu;
  c->par.dampx = c->p_dampx; c->par.dampz = c->p_dampz;
  c->par.kpp = c->p_kpp; c->par.kps = c->p_kps;
  return DS2D_OK;
}

int ensure_rtm(ds2d_ctx *c) {
  int rc;
  if ((rc = ensure_common(c))) return rc;
  if (c->have_rtm) return DS2D_OK;
  if ((rc = alloc_wave(c, c->abk, true))) return rc;
  float **es[4] = {&c->e.gx_vx, &c->e.gz_vz, &c->e.gz_vx, &c->e.gx_vz};
  for (float **p : es)
    if ((rc = alloc_slots(c, p))) return rc;
  if (!c->d.rbc && (rc = ensure_strips(c, c->st_a, c->st_a_steps, c->d.nt))) return rc;
  if (!c->img_slot) {
    size_t n = (size_t)7 * c->B * c->d.wnx * c->d.ild;
    if ((rc = alloc(c, (void **)&c->img_slot, n * sizeof(float)))) return rc;
  }
  c->have_rtm = true;
  return DS2D_OK;
}

int ensure_elsrtm(ds2d_ctx *c) {
  int rc;
  if ((rc = ensure_rtm(c))) return rc;
  if (c->have_elsrtm) return DS2D_OK;
  if ((rc = alloc_slots(c, &c->p_dmp))) return rc;
  if ((rc = alloc_slots(c, &c->p_dms))) return rc;
  c->par.dmp = c->p_dmp;
  c->par.dms = c->p_dms;
  if ((rc = alloc_wave(c, c->b1, false))) return rc;
  if ((rc = alloc_wave(c, c->b2, false))) return rc;
  if ((rc = alloc_wave(c, c->bbk, true))) return rc;
  float **es[4] = {&c->be.gx_vx, &c->be.gz_vz, &c->be.gz_vx, &c->be.gx_vz};
  for (float **p : es)
    if ((rc = alloc_slots(c, p))) return rc;
  for (int i = 0; i < 3; i++)
    if ((rc = alloc_slots(c, &c->ov_s[i]))) return rc;
  for (int i = 0; i < 2; i++)
    if ((rc = alloc_slots(c, &c->ov_v[i]))) return rc;
  if (!c->d.rbc && (rc = ensure_strips(c, c->st_b, c->st_b_steps, c->d.nt))) return rc;
  size_t nrec = (size_t)c->B * c->d.max_ntr * c->d.nt;
  for (int i = 2; i < 8; i++)
    if ((rc = alloc(c, (void **)&c->rec[i], nrec * sizeof(float)))) return rc;
  if ((rc = alloc(c, (void **)&c->d_mis, sizeof(double) * (size_t)c->B * c->d.max_ntr))) return rc;
  c->have_elsrtm = true;
  return DS2D_OK;
}

// Validates shots [first, first + n) and uploads their descriptors and receiver maps.
int upload_batch(ds2d_ctx *c, const ds2d_shot *shots, int n) {
  const Dims &d = c->d;
  std::vector<ShotDev> sd(n);
  std::vector<int> rmap((size_t)n * d.nxp, -1);
  for (int s = 0; s < n; s++) {
    const ds2d_shot &sh = shots[s];
    const int wnx = sh.nx > 0 ? sh.nx : d.wnx;
    const int nxp = wnx + 2 * d.pml;
    if (wnx > d.wnx)
      return fail(c, DS2D_E_ARG, "shot %d: window width %d exceeds grid.nx = %d", s, wnx, d.wnx);
    if (sh.win_left < 0 || sh.win_left + wnx > d.allnx)
      return fail(c, DS2D_E_ARG, "shot %d: window [%d, %d) outside the model (allnx = %d)", s,
                  sh.win_left, sh.win_left + wnx, d.allnx);
    if (sh.isx < d.nop || sh.isx >= nxp - d.nop || sh.isz < d.nop || sh.isz >= d.nzp - d.nop)
      return fail(c, DS2D_E_ARG, "shot %d: source cell (%d, %d) outside the updated grid", s,
                  sh.isx, sh.isz);
    if (sh.ntr < 0 || sh.ntr > d.max_ntr || (sh.ntr > 0 && !sh.igx))
      return fail(c, DS2D_E_ARG, "shot %d: ntr = %d (max_ntr = %d)", s, sh.ntr, d.max_ntr);
    if (sh.ntr > 0 && (sh.igz < d.pml || sh.igz >= d.nzp - d.pml))
      return fail(c, DS2D_E_ARG, "shot %d: receiver row %d outside the interior", s, sh.igz);
    for (int t = 0; t < sh.ntr; t++) {
      int gx = sh.igx[t];
      if (gx < d.pml || gx >= nxp - d.pml)
        return fail(c, DS2D_E_ARG, "shot %d trace %d: receiver column %d outside the interior", s,
                    t, gx);
      int &slot = rmap[(size_t)s * d.nxp + gx];
      if (slot >= 0)
        return fail(c, DS2D_E_ARG, "shot %d: receivers %d and %d share column %d", s, slot, t, gx);
      slot = t;
    }
    sd[s] = ShotDev{sh.win_left, sh.isx, sh.isz, sh.igz, sh.ntr, nxp, wnx,
                    4 * d.nop * (wnx + d.wnz)};
  }
  c->batch_cells = c->batch_wcells = 0;
  c->h_nxp.assign(n, 0);
  for (int s = 0; s < n; s++) c->h_nxp[s] = sd[s].nxp;
  for (const ShotDev &x : sd) {
    c->batch_cells += (double)x.nxp * d.nzp;
    c->batch_wcells += (double)x.wnx * d.wnz;
  }
  CK(cudaMemcpyAsync(c->d_shots, sd.data(), sizeof(ShotDev) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_rmap, rmap.data(), sizeof(int) * rmap.size(), cudaMemcpyHostToDevice,
                     c->stream));
  return DS2D_OK;
}

int setup_batch(ds2d_ctx *c, int n, int shot_base, bool with_image) {
  SetupArgs a{};
  a.d = c->d;
  a.vp_all = c->vp_all; a.vs_all = c->vs_all; a.rho_all = c->rho_all;
  a.pp_all = c->pp_all; a.ps_all = c->ps_all;
  a.shots = c->d_shots;
  a.b = c->p_b; a.lam = c->p_lam; a.mu = c->p_mu; a.dampx = c->p_dampx; a.dampz = c->p_dampz;
  a.kpp = c->p_kpp; a.kps = c->p_kps;
  a.dmp = with_image ? c->p_dmp : nullptr;
  a.dms = with_image ? c->p_dms : nullptr;
  a.L = std::log10((double)(1.0f / 0.001f));  // rr = 0.001 (FD2DGPU.cu:1299)
  a.seed = c->o.seed;
  a.shot_base = shot_base;
  dim3 grid((c->d.ld + 127) / 128, c->d.nxp, n);
  k_setup<<<grid, 128, 0, c->stream>>>(a);
  CK(cudaGetLastError());
  c->last_launches++;
  return DS2D_OK;
}

dim3 cell_grid(const Dims &d, int n) { return dim3((d.nzp + kBX - 1) / kBX, (d.nxp + kBY - 1) / kBY, n); }

VelArgs vel_args(ds2d_ctx *c, const Wave &w, int it) {
  VelArgs v{};
  v.d = c->d; v.w = w; v.p = c->par; v.shots = c->d_shots; v.wavelet = c->wavelet; v.it = it;
  v.rmap = c->d_rmap;
  return v;
}

StrArgs str_args(ds2d_ctx *c, const Wave &w, int it) {
  StrArgs s{};
  s.d = c->d; s.w = w; s.p = c->par; s.it = it; s.shots = c->d_shots; s.rmap = c->d_rmap;
  return s;
}

// Launch on the context stream; in profiling mode bracket it with an event pair and record the
// launch's algorithmic bytes (cells * bytes per cell of that kernel).
#define LAUNCHP(pname, pbytes, kernel, grid, block, args)                       \
  do {                                                                          \
    int ev_ = -1;                                                               \
    if (c->prof.on) {                                                           \
      ev_ = c->prof.take();                                                     \
      cudaEventRecord(c->prof.pool[ev_], c->stream);                            \
    }                                                                           \
    kernel<<<grid, block, 0, c->stream>>>(args);                                \
    c->last_launches++;                                                         \
    if (ev_ >= 0) {                                                             \
      cudaEventRecord(c->prof.pool[ev_ + 1], c->stream);                        \
      c->prof.recs.push_back(ProfRec{pname, ev_, (double)(pbytes)});           \
    }                                                                           \
  } while (0)

// Algorithmic bytes per padded cell of each half-step kernel (FP32): every array the update
// needs read once and every array it produces written once.
constexpr double kBytesVel = 32;     // S (12) + V (8) + b (4) read, V (8) written
constexpr double kBytesStr = 40;     // V (8) + S (12) + lam, mu (8) read, S (12) written
constexpr double kBytesStrRev = 56;  // + four strains written
constexpr double kBytesVelAdj = 40;  // S (12) + lam, mu (8) + b (4) + V (8) read, V written
constexpr double kBytesStrAdj = 32;  // V (8) + S (12) read, S (12) written
constexpr double kBytesImage = 68;   // strains 16 + S 12 + weights 8 + V 8 read, 3 images r/w 24
constexpr double kBytesFused = 52;   // one fused elastic step: 5 fields r/w + b, lam, mu read
// Fused Born-modelling steps (ring modes 1-3): the elastic step plus the overlay read (12), the
// Born source written (12) and dmp, dms read (8) where the mode has them.
constexpr double kBytesBornMode[4] = {52, 72, 84, 64};
// Reverse step of the first-order scattered set (k_bwd_scat_ring): its 5 fields read and written,
// b, lam, mu, kpp, kps, the adjoint stresses and the Born source read, images 3 and 4 updated.
constexpr double kBytesBwdScat = 100;
// Fused acoustic reverse step (k_ac_rev_ring): adjoint state and background, 3 fields each read
// and written, b and lam read, the gradient updated on the interior.
constexpr double kBytesAcRev = 64;
// Fused backward RTM step per padded cell: source and adjoint fields r/w (2 x 40), b, lam, mu
// (12), imaging weights (8) and three image accumulators r/w (24).
constexpr double kBytesBwdFused = 124;
#define CELLS(n) (c->batch_cells)
#define WCELLS(n) (c->batch_wcells)
#define LAUNCH(kernel, grid, block, args) LAUNCHP(#kernel, 0, kernel, grid, block, args)
// Same with dynamic shared memory.
#define LAUNCHS(pname, pbytes, kernel, grid, block, smem, args)                 \
  do {                                                                          \
    int ev_ = -1;                                                               \
    if (c->prof.on) {                                                           \
      ev_ = c->prof.take();                                                     \
      cudaEventRecord(c->prof.pool[ev_], c->stream);                            \
    }                                                                           \
    kernel<<<grid, block, smem, c->stream>>>(args);                             \
    c->last_launches++;                                                         \
    if (ev_ >= 0) {                                                             \
      cudaEventRecord(c->prof.pool[ev_ + 1], c->stream);                        \
      c->prof.recs.push_back(ProfRec{pname, ev_, (double)(pbytes)});           \
    }                                                                           \
  } while (0)

int strip_save(ds2d_ctx *c, const Wave &w, Strips &st, int it, int n) {
  StripSaveArgs a{c->d, c->d_shots, w.vx, w.vz, st, it};
  dim3 grid((c->d.lb + 255) / 256, 2, n);
  LAUNCH(k_strip_save, grid, 256, a);
  return DS2D_OK;
}

// Threads per CTA of the fused elastic launches.  A CTA computes (threads - 16) columns of a
// z-strip; the strips split nzp evenly, so the share of working threads depends on nzp (481:
// 97 of 128 or 161 of 192; 441: 111 of 128 or 147 of 192).  Automatic choice: the wider CTA
// when its share of working threads is at least 5 % higher.  Only the ring kernels at the default
// depth and occupancy have the wide variant.
int fused_cta(const ds2d_ctx *c) {
  if (!(c->opt_ring && c->ring_ok) || c->opt_ring != 4 || c->opt_occ != 0) return kFB;
  if (c->opt_cta) return c->opt_cta;
  auto share = [&](int cta) {
    const int ns = (c->d.nzp + cta - 17) / (cta - 16);
    return (double)((c->d.nzp + ns - 1) / ns) / cta;
  };
  return share(kWideCta) > 1.05 * share(kFB) ? kWideCta : kFB;
}

// z-strip split of the fused launches for CTAs of `cta` threads: (strips, columns per strip).
void strip_split(const Dims &d, int cta, int *nstrips, int *tz) {
  *nstrips = (d.nzp + cta - 17) / (cta - 16);
  *tz = (d.nzp + *nstrips - 1) / *nstrips;
}

// ---- pair-blocked kernels (random boundary) ------------------------------------------------
// CTA widths: 256 threads cover a whole 481-deep column (no z-halo recomputed) at 2 forward / 1
// backward CTAs per SM; 64 threads (z-strips of 100 columns) give 8 forward / 4 backward CTAs per
// SM, each barrier syncing two warps; 160 threads: two strips of a 481-deep column.
constexpr int kPairFwdD = 4;  // forward ring: 4 slots
constexpr int kPairBwdD = 3;  // backward ring: 3 slots
using PairFwdFn = void (*)(FwdFusedArgs);
using PairBwdFn = void (*)(BwdFusedArgs);
PairFwdFn pair_fwd_fn(int cta) {
  return cta == 64 ? k_fwd_pair<64, kPairFwdD, 8> : k_fwd_pair<256, kPairFwdD, 2>;
}
PairBwdFn pair_bwd_fn(int cta) {
  return cta == 64    ? k_bwd_pair<64, kPairBwdD, 4>
         : cta == 160 ? k_bwd_pair<160, kPairBwdD, 2>
                      : k_bwd_pair<256, kPairBwdD, 1>;
}
// The backward step split in two launches (option "pair_split"): reconstruction + illumination,
// then adjoint + imaging, both on 64-thread strips.
constexpr int kPairSplitT = 64;
PairBwdFn pair_split_fn(int part) {
  return part == 1 ? k_bwd_pair<kPairSplitT, kPairBwdD, 8, 1> : k_bwd_pair<kPairSplitT, kPairBwdD, 5, 2>;
}
constexpr size_t pair_split_smem(int part) {
  return pair_smem(kPairSplitT, kPairBwdD, bwd_pair_fields(part), bwd_pair_z2_rows(part));
}
// Algorithmic bytes per padded cell of the two parts: reconstruction 5 fields r/w + b, lam, mu +
// illumination r/w (60); adjoint 5 fields r/w + b, lam, mu + the reconstruction's input
// velocities + imaging weights + two images r/w (84).
constexpr double kBytesBwdRec = 60, kBytesBwdAdj = 84;
constexpr size_t pair_fwd_smem(int cta) {
  return pair_smem(cta, kPairFwdD, kFwdPairFields, kFwdPairZ2Rows);
}
constexpr size_t pair_bwd_smem(int cta) {
  return pair_smem(cta, kPairBwdD, kBwdPairFields, bwd_pair_z2_rows(0));
}

bool pair_ok(const ds2d_ctx *c) {
  return c->opt_fused && c->ring_ok && c->d.rbc && c->d.nop == 4 && c->d.ild == c->d.ld &&
         c->d_err && c->occ_pair[0] > 0;
}
// option "pair": 0 none, 1 forward and backward, 2 forward only (the backward stays on the
// one-column ring kernel)
bool pair_fwd_on(const ds2d_ctx *c) { return c->opt_pair && pair_ok(c); }
bool pair_bwd_on(const ds2d_ctx *c) { return c->opt_pair == 1 && pair_ok(c); }
// CTA widths (options "pair_cta" backward, "pair_fcta" forward; 0 = automatic): narrow 64-thread
// strips by default (more CTAs per SM, barriers of two warps).
int pair_bwd_cta(const ds2d_ctx *c) { return c->opt_pair_cta ? c->opt_pair_cta : 64; }
int pair_fwd_cta(const ds2d_ctx *c) { return c->opt_pair_fcta ? c->opt_pair_fcta : 256; }
// resident CTAs per SM of each variant (queried at create)
int pair_occ(const ds2d_ctx *c, bool fwd, int cta) {
  if (fwd) return cta == 64 ? c->occ_pair[1] : c->occ_pair[0];
  return cta == 64 ? c->occ_pair[4] : cta == 160 ? c->occ_pair[3] : c->occ_pair[2];
}
// z-strips of a pair launch: each CTA computes tz (a multiple of 4) columns, 2 kT - 16 at most.
void pair_split(const Dims &d, int kT, int *nstrips, int *tz) {
  const int w = 2 * kT - 16;
  *nstrips = (d.nzp + w - 1) / w;
  const int t = (d.nzp + *nstrips - 1) / *nstrips;
  *tz = (t + 3) / 4 * 4;
}
// Rows per CTA: a CTA's time grows with xr + 12 (16 halo steps, 8 of them loads only), and the
// launch takes as many waves as its CTAs fill; xr minimises waves x (xr + 12) over the batch's
// own window widths.
int pair_xr(const ds2d_ctx *c, int nstrips, int per_sm) {
  if (c->opt_pair_xr > 0) return std::max(8, c->opt_pair_xr);
  const long long slots = (long long)c->num_sms * std::max(1, per_sm);
  long long best = -1;
  int best_xr = 128;
  for (int xr = 48; xr <= 256; xr++) {
    long long ctas = 0;
    for (int nx : c->h_nxp) ctas += (long long)nstrips * ((nx + xr - 1) / xr);
    const long long cost = (ctas + slots - 1) / slots * (xr + 12);
    if (best < 0 || cost <= best) {
      best = cost;
      best_xr = xr;
    }
  }
  return best_xr;
}

// Reads and clears the error word of the pair kernels (after the stream has been synchronised).
int check_pair_err(ds2d_ctx *c) {
  if (!c->d_err) return DS2D_OK;
  int h = 0;
  CK(cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    CK(cudaMemset(c->d_err, 0, sizeof(int)));
    return fail(c, DS2D_E_CUDA, "a pair kernel's ring wait gave up (error word %d)", h);
  }
  return DS2D_OK;
}

// ---- time-blocked forward kernels (random boundary) ----------------------------------------
// k_fwd_tb<depth, threads>: 256 threads at any depth (register budget for 3 / 2 / 1 / 1 CTAs per
// SM at depth 1 / 2 / 3 / 4), or 512 threads at depth 1-2 (one CTA per SM: a single strip covers
// a grid up to 512 deep with no z-halo, e.g. 481 rows, which 256-thread strips split in three
// once the depth-2 halo of 16 columns is added).
constexpr int kTbCtas[2] = {256, 512};
constexpr int kTbMaxXr = 512;  // rows per CTA (bounds the trace-index staging in shared memory)
using TbFn = void (*)(FwdFusedArgs);
template <int kT>
TbFn tb_fn_t(int depth) {
  switch (depth) {
    case 1: return k_fwd_tb<1, kT, 3>;
    case 2: return k_fwd_tb<2, kT, 2>;
    case 3: return k_fwd_tb<3, kT, 1>;
    default: return k_fwd_tb<4, kT, 1>;
  }
}
TbFn tb_fn(int depth, int cta, bool bulk = false) {
  if (bulk && depth <= 2) {  // operand rows by bulk copy (depth 1-2)
    if (cta == 512) return depth == 1 ? k_fwd_tb<1, 512, 1, true> : k_fwd_tb<2, 512, 1, true>;
    return depth == 1 ? k_fwd_tb<1, 256, 3, true> : k_fwd_tb<2, 256, 2, true>;
  }
  if (cta == 512) return depth == 1 ? k_fwd_tb<1, 512, 1> : k_fwd_tb<2, 512, 1>;
  return tb_fn_t<256>(depth);
}
int tb_idx(int cta) { return cta == 512 ? 1 : 0; }
// z-strips of a time-blocked launch of depth K: a strip owns tz columns, its CTA covers them plus
// 8K halo columns at each inner edge (one strip: the whole depth; two: one halo each; more: the
// inner strips carry two).  Returns false when kT threads cannot cover a strip.
bool tb_split(const Dims &d, int kT, int K, int *nstrips, int *tz) {
  const int H = 8 * K;
  for (int ns = 1; ns <= 64; ns++) {
    // several strips: widths a multiple of 4, so every strip starts on a 16-byte boundary
    const int t = ns == 1 ? d.nzp : ((d.nzp + ns - 1) / ns + 3) / 4 * 4;
    const int cap = ns == 1 ? kT : ns == 2 ? kT - H : kT - 2 * H;
    if (t <= cap) {
      *nstrips = ns;
      *tz = t;
      return true;
    }
  }
  return false;
}
// CTA width: option "tb_cta", else the width with the fewest threads per grid row.
int tb_cta(const ds2d_ctx *c, int K) {
  if (c->opt_tb_cta) return K > 2 ? 256 : c->opt_tb_cta;
  int best = 256;
  long long best_thr = 1LL << 40;
  for (int cta : kTbCtas) {
    int ns, tz;
    if ((cta == 512 && K > 2) || !tb_split(c->d, cta, K, &ns, &tz)) continue;
    if ((long long)ns * cta < best_thr) {
      best_thr = (long long)ns * cta;
      best = cta;
    }
  }
  return best;
}
// Rows per CTA: a CTA marches xr + 16K row steps; xr minimises waves x (xr + 12K) over the
// batch's window widths (the halo steps at the start only load and fill windows).
int tb_xr(const ds2d_ctx *c, int nstrips, int per_sm, int K) {
  if (c->opt_pair_xr > 0) return std::min(kTbMaxXr, std::max(8, c->opt_pair_xr));
  const long long slots = (long long)c->num_sms * std::max(1, per_sm);
  long long best = -1;
  int best_xr = 128;
  for (int xr = 48; xr <= kTbMaxXr; xr++) {
    long long ctas = 0;
    for (int nx : c->h_nxp) ctas += (long long)nstrips * ((nx + xr - 1) / xr);
    const long long cost = (ctas + slots - 1) / slots * (xr + 12 * K);
    if (best < 0 || cost <= best) {
      best = cost;
      best_xr = xr;
    }
  }
  return best_xr;
}
// ---- warp-specialised backward (random boundary) ------------------------------------------
constexpr int kWsRoles[3] = {96, 128, 192};
BwdFn ws_fn(int kt) {
  return kt == 96 ? k_bwd_ws<96, 4> : kt == 128 ? k_bwd_ws<128, 3> : k_bwd_ws<192, 2>;
}
int ws_idx(int kt) { return kt == 96 ? 0 : kt == 128 ? 1 : 2; }
// ---- bulk-copy-fed one-column backward (random boundary) ------------------------------------
// 128 threads at 4 CTAs per SM and 256 at 2 (128 registers, 16 warps per SM), 192 at 2 (12).
constexpr int kBulkCtas[3] = {128, 192, 256};
BwdFn bulk_fn(int cta, bool one) {
  if (cta == 256) return one ? k_bwd_bulk<256, 2, true> : k_bwd_bulk<256, 2, false>;
  if (cta == kWideCta) return one ? k_bwd_bulk<kWideCta, 2, true> : k_bwd_bulk<kWideCta, 2, false>;
  return one ? k_bwd_bulk<kFB, 4, true> : k_bwd_bulk<kFB, 4, false>;
}
int bulk_idx(int cta, bool one) { return (cta == 256 ? 4 : cta == kWideCta ? 2 : 0) + (one ? 1 : 0); }

// CTA width of k_bwd_bulk: option "bwd_cta", else the width with the fewest threads per grid row
// (edge-aware strips), the wider on a tie.
int bulk_cta(const ds2d_ctx *c) {
  if (c->opt_bwd_cta) return c->opt_bwd_cta;
  int best = kWideCta;
  long long best_thr = 1LL << 40;
  for (int cta : kBulkCtas) {
    int ns, tz;
    if (!tb_split(c->d, cta, 1, &ns, &tz)) continue;
    if ((long long)ns * cta <= best_thr) {
      best_thr = (long long)ns * cta;
      best = cta;
    }
  }
  return best;
}

bool ws_on(const ds2d_ctx *c) {
  return c->opt_bwd_ws > 0 && c->opt_fused && c->ring_ok && c->d.rbc &&
         c->occ_ws[ws_idx(c->opt_bwd_ws)] > 0;
}

bool tb_on(const ds2d_ctx *c) {
  if (!(c->opt_tb > 0 && c->opt_fused && c->ring_ok && c->d.rbc && c->d.nop == 4)) return false;
  const int cta = tb_cta(c, c->opt_tb);
  int ns, tz;
  return tb_split(c->d, cta, c->opt_tb, &ns, &tz) && c->occ_tb[tb_idx(cta)][c->opt_tb - 1] > 0;
}

// Acoustic pair kernels (k_ac_pair): 256 / 192 / 128 threads at 2 / 3 / 4 CTAs per SM.
constexpr int kAcPairCtas[3] = {256, 192, 128};
using AcPairFn = void (*)(AcRingArgs);
AcPairFn ac_pair_fn(int mode, int cta) {
  if (cta == 256) return mode ? k_ac_pair<1, 256, 2> : k_ac_pair<0, 256, 2>;
  if (cta == 192) return mode ? k_ac_pair<1, 192, 3> : k_ac_pair<0, 192, 3>;
  return mode ? k_ac_pair<1, 128, 4> : k_ac_pair<0, 128, 4>;
}
int ac_pair_idx(int cta) { return cta == 256 ? 0 : cta == 192 ? 1 : 2; }
// CTA width: option "ac_pair_cta", else the width with the fewest threads per grid row (z-strips
// x threads; the wider on a tie), so the z-halo recomputed and the idle columns stay small.
int ac_pair_cta(const ds2d_ctx *c) {
  if (c->opt_ac_pair_cta) return c->opt_ac_pair_cta;
  int best = 256, best_thr = 1 << 30;
  for (int cta : kAcPairCtas) {
    int ns, tz;
    pair_split(c->d, cta, &ns, &tz);
    if (ns * cta < best_thr) {
      best_thr = ns * cta;
      best = cta;
    }
  }
  return best;
}
bool ac_pair_on(const ds2d_ctx *c) {
  return c->opt_ac_pair && pair_ok(c) && c->occ_ac_pair[ac_pair_idx(ac_pair_cta(c))] > 0;
}
// Reverse step (k_ac_rev_pair): 192 / 128 threads at 2 / 3 CTAs per SM, strips with a
// 12-column halo (each CTA computes tz <= 2 kT - 24 columns); the width with the fewest threads
// per grid row, the wider on a tie.
constexpr int kAcRevCtas[2] = {192, 128};
using AcRevFn = void (*)(AcRevArgs);
AcRevFn ac_rev_fn(int cta) { return cta == 192 ? k_ac_rev_pair<192, 2> : k_ac_rev_pair<128, 3>; }
void ac_rev_split(const Dims &d, int kT, int *nstrips, int *tz) {
  const int w = 2 * kT - 2 * kAcRevHalo;
  *nstrips = (d.nzp + w - 1) / w;
  const int t = (d.nzp + *nstrips - 1) / *nstrips;
  *tz = (t + 3) / 4 * 4;
}
int ac_rev_cta(const ds2d_ctx *c) {
  int best = 192, best_thr = 1 << 30;
  for (int cta : kAcRevCtas) {
    int ns, tz;
    ac_rev_split(c->d, cta, &ns, &tz);
    if (ns * cta < best_thr) {
      best_thr = ns * cta;
      best = cta;
    }
  }
  return best;
}
bool ac_rev_pair_on(const ds2d_ctx *c) {
  return ac_pair_on(c) && c->occ_ac_rev[ac_rev_cta(c) == 192 ? 0 : 1] > 0;
}

// Fused forward pass: one k_fwd_fused launch per step, ping-ponging fw <-> fw2.
int run_forward_fused(ds2d_ctx *c, int n, bool record, bool strips) {
  const Dims &d = c->d;
  int rc;
  if (!c->fw2.vx && (rc = alloc_wave(c, c->fw2, false))) return rc;
  if ((rc = zero_wave(c, c->fw2, n))) return rc;
  const int cta = fused_cta(c);
  int nstrips, tz;
  strip_split(d, cta, &nstrips, &tz);
  const int xr = std::max(8, c->opt_xr);
  dim3 grid(nstrips, (d.nxp + xr - 1) / xr, n);
  Wave *cur = &c->fw, *nxt = &c->fw2;
  if (!strips && tb_on(c)) {
    // time blocks of opt_tb steps, one launch each (the last block takes what is left)
    for (int it = 0; it < d.nt;) {
      const int K = std::min(c->opt_tb, d.nt - it);
      const int tc = tb_cta(c, c->opt_tb);
      int ns, tz;
      if (!tb_split(d, tc, K, &ns, &tz))
        return fail(c, DS2D_E_ARG, "time-blocked strips do not fit %d threads", tc);
      const int txr = tb_xr(c, ns, c->occ_tb[tb_idx(tc)][K - 1], K);
      FwdFusedArgs a{};
      a.d = d; a.a = *cur; a.b = *nxt; a.p = c->par; a.shots = c->d_shots; a.wavelet = c->wavelet;
      a.it = it; a.tz = tz; a.xr = txr; a.rmap = c->d_rmap; a.err = c->d_err;
      if (record) { a.rec_on = 1; a.rec_vz = c->rec[0]; a.rec_vx = c->rec[1]; }
      dim3 tgrid(ns, (d.nxp + txr - 1) / txr, n);
      const bool bulk = c->opt_tb_bulk && K <= 2 && c->d_err && d.ild == d.ld &&
                        c->occ_tb_bulk[tb_idx(tc)][K - 1] > 0;
      LAUNCHS("fwd_tb", kBytesFused * CELLS(n), tb_fn(K, tc, bulk), tgrid, tc, tb_smem(K, tc, txr),
              a);
      std::swap(cur, nxt);
      it += K;
    }
    c->fw_cur = cur;
    CK(cudaGetLastError());
    return DS2D_OK;
  }
  for (int it = 0; it < d.nt; it++) {
    FwdFusedArgs a{};
    a.d = d; a.a = *cur; a.b = *nxt; a.p = c->par; a.shots = c->d_shots; a.wavelet = c->wavelet;
    a.it = it; a.tz = tz; a.xr = xr; a.rmap = c->d_rmap;
    if (record) { a.rec_on = 1; a.rec_vz = c->rec[0]; a.rec_vx = c->rec[1]; }
    if (pair_fwd_on(c)) {
      const int pc = pair_fwd_cta(c);
      int pns, ptz;
      pair_split(d, pc, &pns, &ptz);
      const int pxr = pair_xr(c, pns, pair_occ(c, true, pc));
      a.tz = ptz; a.xr = pxr; a.err = c->d_err;
      dim3 pgrid(pns, (d.nxp + pxr - 1) / pxr, n);
      LAUNCHS("fwd_pair", kBytesFused * CELLS(n), pair_fwd_fn(pc), pgrid, pc, pair_fwd_smem(pc), a);
    } else if (c->opt_ring && c->ring_ok) {
      const size_t sm = sizeof(float) * c->opt_ring * fwd_ring_fields(!d.rbc) * cta;
      FwdFn kfn = fwd_ring_fn(d.rbc != 0, c->opt_ring, c->opt_occ, cta);
      LAUNCHS("fwd_fused", kBytesFused * CELLS(n), kfn, grid, cta, sm, a);
    } else if (d.rbc) {
      LAUNCHP("fwd_fused", kBytesFused * CELLS(n), k_fwd_fused<false>, grid, kFB, a);
    } else {
      LAUNCHP("fwd_fused", kBytesFused * CELLS(n), k_fwd_fused<true>, grid, kFB, a);
    }
    if (strips) strip_save(c, *nxt, c->st_a, it, n);
    std::swap(cur, nxt);
  }
  c->fw_cur = cur;
  CK(cudaGetLastError());
  return DS2D_OK;
}

// Background forward pass with optional recording and strip saving.
int run_forward_pass(ds2d_ctx *c, int n, bool record, bool strips) {
  if (c->opt_fused) return run_forward_fused(c, n, record, strips);
  const Dims &d = c->d;
  c->fw_cur = &c->fw;
  dim3 grid = cell_grid(d, n), blk(kBX, kBY);
  for (int it = 0; it < d.nt; it++) {
    VelArgs v = vel_args(c, c->fw, it);
    v.src_on = 1;
    if (record) { v.rec_on = 1; v.rec_vz = c->rec[0]; v.rec_vx = c->rec[1]; }
    LAUNCHP("vel_fwd", kBytesVel * CELLS(n), k_vel<kFwd>, grid, blk, v);
    StrArgs s = str_args(c, c->fw, it);
    LAUNCHP("str_fwd", kBytesStr * CELLS(n), k_str<kFwd>, grid, blk, s);
    if (strips) strip_save(c, c->fw, c->st_a, it, n);
  }
  CK(cudaGetLastError());
  return DS2D_OK;
}

int reduce_images(ds2d_ctx *c, int n, int nimg) {
  const Dims &d = c->d;
  dim3 grid((d.allnz + 255) / 256, d.allnx);
  long long plane = (long long)c->B * d.wnx * d.ild;
  k_image_reduce<<<grid, 256, 0, c->stream>>>(d, c->img_slot, plane, nimg, n, c->d_shots, c->images,
                                              (long long)d.allnx * d.allnz);
  c->last_launches++;
  CK(cudaGetLastError());
  return DS2D_OK;
}

int check_ready(ds2d_ctx *c, bool need_image) {
  if (!c) return DS2D_E_ARG;
  if (!c->models_set) return fail(c, DS2D_E_STATE, "models not set (ds2d_set_models)");
  if (!c->wavelet_set) return fail(c, DS2D_E_STATE, "wavelet not set (ds2d_set_wavelet)");
  if (need_image && !c->image_set) return fail(c, DS2D_E_STATE, "image not set (ds2d_set_image)");
  return DS2D_OK;
}

int copy_records_in(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *src_z,
                    const float *src_x, long long trace_base, float *dz, float *dx,
                    cudaMemcpyKind kind) {
  const Dims &d = c->d;
  size_t nrec = (size_t)n * d.max_ntr * d.nt;
  CK(cudaMemsetAsync(dz, 0, nrec * sizeof(float), c->stream));
  CK(cudaMemsetAsync(dx, 0, nrec * sizeof(float), c->stream));
  long long tb = trace_base;
  for (int s = 0; s < n; s++) {
    size_t cnt = (size_t)shots[s].ntr * d.nt;
    size_t dst = (size_t)s * d.max_ntr * d.nt;
    if (cnt) {
      CK(cudaMemcpyAsync(dz + dst, src_z + tb * d.nt, cnt * sizeof(float), kind, c->stream));
      CK(cudaMemcpyAsync(dx + dst, src_x + tb * d.nt, cnt * sizeof(float), kind, c->stream));
    }
    tb += shots[s].ntr;
  }
  return DS2D_OK;
}

int copy_records_out(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *sz,
                     const float *sx, long long trace_base, float *out_z, float *out_x) {
  const Dims &d = c->d;
  long long tb = trace_base;
  for (int s = 0; s < n; s++) {
    size_t cnt = (size_t)shots[s].ntr * d.nt;
    size_t src = (size_t)s * d.max_ntr * d.nt;
    if (cnt) {
      if (out_z) CK(cudaMemcpyAsync(out_z + tb * d.nt, sz + src, cnt * 4, cudaMemcpyDeviceToHost, c->stream));
      if (out_x) CK(cudaMemcpyAsync(out_x + tb * d.nt, sx + src, cnt * 4, cudaMemcpyDeviceToHost, c->stream));
    }
    tb += shots[s].ntr;
  }
  return DS2D_OK;
}

int rtm_batch_body(ds2d_ctx *c, const ds2d_shot *shots, int n, int shot_base);

// Runs `body` (device work only: launches, async device copies and memsets on c->stream) as a
// CUDA graph: captured on first use for `key`, replayed afterwards.  Direct launches when
// graphs are off, when profiling, or on the legacy default stream (which cannot be captured).
template <class F>
int run_graph(ds2d_ctx *c, const long long (&key)[6], F &&body) {
  if (!c->opt_graph || c->prof.on || c->stream == nullptr) return body();
  for (const auto &g : c->graphs)
    if (std::equal(key, key + 6, g.key)) {
      CK(cudaGraphLaunch(g.exec, c->stream));
      c->last_launches += g.launches;
      return DS2D_OK;
    }
  const long long before = c->last_launches;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = body();
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  CK(e);
  ds2d_ctx::GraphEntry g{};
  std::copy(key, key + 6, g.key);
  const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  CK(ie);
  g.launches = c->last_launches - before;
  c->graphs.push_back(g);
  CK(cudaGraphLaunch(g.exec, c->stream));
  return DS2D_OK;
}

int rtm_batch(ds2d_ctx *c, const ds2d_shot *shots, int n, int shot_base) {
  int rc;
  if (c->opt_fused) {  // allocations must precede any graph capture
    if (!c->fw2.vx && (rc = alloc_wave(c, c->fw2, false))) return rc;
    if (!c->abk2.vx && (rc = alloc_wave(c, c->abk2, true))) return rc;
  }
  const long long key[6] = {2, n, shot_base, c->opt_fused + 2 * c->opt_ring + 32 * c->opt_occ + 64 * c->opt_cta, c->opt_xr + 1000LL * c->opt_pair_xr + 1000000LL * c->opt_pair_cta + 100000000LL * (c->opt_pair_fcta / 64 + 5 * c->opt_pair_split) + 1000000000LL * c->opt_pair + 10000000000LL * (c->opt_tb + 5 * (c->opt_tb_cta / 32)) + 1000000000000LL * (c->opt_bwd_ws / 32 + 8 * c->opt_bwd_1b + 16 * c->opt_bwd_bulk + 32 * c->opt_tb_bulk + 64 * (c->opt_bwd_cta / 64)), (long long)(size_t)c->stream};
  return run_graph(c, key, [&]() { return rtm_batch_body(c, shots, n, shot_base); });
}

int rtm_batch_body(ds2d_ctx *c, const ds2d_shot *shots, int n, int shot_base) {
  const Dims &d = c->d;
  int rc;
  if ((rc = setup_batch(c, n, shot_base, false))) return rc;
  if ((rc = zero_wave(c, c->fw, n))) return rc;
  if ((rc = zero_wave(c, c->abk, n))) return rc;
  size_t plane = (size_t)c->B * d.wnx * d.ild;
  CK(cudaMemsetAsync(c->img_slot, 0, 7 * plane * sizeof(float), c->stream));
  const bool strips = !d.rbc;
  if ((rc = run_forward_pass(c, n, false, strips))) return rc;
  if (c->opt_fused) {
    // Both buffers of the source field start from the final forward state, so the cells the
    // interior reconstruction never updates (PML / random band) stay frozen in both.
    Wave *cur = c->fw_cur, *nxt = (cur == &c->fw) ? &c->fw2 : &c->fw;
    size_t bytes = sizeof(float) * (size_t)d.slot * n;
    const float *src[5] = {cur->vx, cur->vz, cur->txx, cur->tzz, cur->txz};
    float *dst[5] = {nxt->vx, nxt->vz, nxt->txx, nxt->tzz, nxt->txz};
    for (int i = 0; i < 5; i++)
      CK(cudaMemcpyAsync(dst[i], src[i], bytes, cudaMemcpyDeviceToDevice, c->stream));
    if (!c->abk2.vx && (rc = alloc_wave(c, c->abk2, true))) return rc;
    if ((rc = zero_wave(c, c->abk2, n))) return rc;
    Wave *acur = &c->abk, *anxt = &c->abk2;
    const int cta = fused_cta(c);
    int nstrips, tz;
    strip_split(d, cta, &nstrips, &tz);
    const int xr = std::max(8, c->opt_xr);
    dim3 fgrid(nstrips, (d.nxp + xr - 1) / xr, n);
    for (int it = d.nt - 1; it >= 0; --it) {
      BwdFusedArgs a{};
      a.d = d; a.ra = *cur; a.rb = *nxt; a.aa = *acur; a.ab = *anxt; a.p = c->par;
      a.shots = c->d_shots; a.rmap = c->d_rmap; a.res_vz = c->rec[0]; a.res_vx = c->rec[1];
      a.st = c->st_a; a.strips_on = strips; a.it = it; a.tz = tz; a.xr = xr;
      a.img = c->img_slot; a.img_plane = (long long)plane;
      if (pair_bwd_on(c) && c->opt_pair_split) {
        int pns, ptz;
        pair_split(d, kPairSplitT, &pns, &ptz);
        const int pxr = pair_xr(c, pns, std::min(c->occ_pair[5], c->occ_pair[6]));
        a.tz = ptz; a.xr = pxr; a.err = c->d_err;
        dim3 pgrid(pns, (d.nxp + pxr - 1) / pxr, n);
        // independent launches (both read the step's input states, write their own buffers):
        // the adjoint part runs on the second stream between a fork and a join event
        CK(cudaEventRecord(c->ev_fork, c->stream));
        CK(cudaStreamWaitEvent(c->aux, c->ev_fork, 0));
        LAUNCHS("bwd_rec", kBytesBwdRec * CELLS(n), pair_split_fn(1), pgrid, kPairSplitT,
                pair_split_smem(1), a);
        {
          cudaStream_t main = c->stream;
          c->stream = c->aux;
          LAUNCHS("bwd_adj", kBytesBwdAdj * CELLS(n), pair_split_fn(2), pgrid, kPairSplitT,
                  pair_split_smem(2), a);
          c->stream = main;
        }
        CK(cudaEventRecord(c->ev_join, c->aux));
        CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
      } else if (c->opt_bwd_bulk && pair_ok(c) &&
                 c->occ_bulk[bulk_idx(bulk_cta(c), c->opt_bwd_1b != 0)] > 0) {
        const int bc = bulk_cta(c);
        int bns, btz;
        tb_split(d, bc, 1, &bns, &btz);  // edge-aware strips, widths a multiple of 4
        // rows per CTA: option "pair_xr", else the count that fills the SMs' waves best
        const int bxr = pair_xr(c, bns, c->occ_bulk[bulk_idx(bc, c->opt_bwd_1b != 0)]);
        a.tz = btz; a.xr = bxr; a.err = c->d_err;
        dim3 bgrid(bns, (d.nxp + bxr - 1) / bxr, n);
        LAUNCHS("bwd_fused", kBytesBwdFused * CELLS(n), bulk_fn(bc, c->opt_bwd_1b != 0), bgrid,
                bc, bwd_bulk_smem(bc), a);
      } else if (ws_on(c)) {
        const int kt = c->opt_bwd_ws;
        int wns, wtz;
        strip_split(d, kt, &wns, &wtz);
        a.tz = wtz;
        dim3 wgrid(wns, (d.nxp + xr - 1) / xr, n);
        LAUNCHS("bwd_ws", kBytesBwdFused * CELLS(n), ws_fn(kt), wgrid, 2 * kt, ws_smem(kt), a);
      } else if (pair_bwd_on(c)) {
        const int pc = pair_bwd_cta(c);
        int pns, ptz;
        pair_split(d, pc, &pns, &ptz);
        const int pxr = pair_xr(c, pns, pair_occ(c, false, pc));
        a.tz = ptz; a.xr = pxr; a.err = c->d_err;
        dim3 pgrid(pns, (d.nxp + pxr - 1) / pxr, n);
        LAUNCHS("bwd_pair", kBytesBwdFused * CELLS(n), pair_bwd_fn(pc), pgrid, pc,
                pair_bwd_smem(pc), a);
      } else if (c->opt_ring && c->ring_ok) {
        const size_t sm = sizeof(float) * c->opt_ring * bwd_ring_fields(!d.rbc) * cta;
        BwdFn kfn = bwd_ring_fn(d.rbc != 0, c->opt_ring, c->opt_occ, cta, c->opt_bwd_1b != 0);
        LAUNCHS("bwd_fused", kBytesBwdFused * CELLS(n), kfn, fgrid, cta, sm, a);
      } else if (d.rbc) {
        LAUNCHP("bwd_fused", kBytesBwdFused * CELLS(n), k_bwd_fused<false>, fgrid, kFB, a);
      } else {
        LAUNCHP("bwd_fused", kBytesBwdFused * CELLS(n), k_bwd_fused<true>, fgrid, kFB, a);
      }
      std::swap(cur, nxt);
      std::swap(acur, anxt);
    }
    CK(cudaGetLastError());
    return reduce_images(c, n, 3);
  }
  dim3 grid = cell_grid(d, n), blk(kBX, kBY);
  dim3 igrid((d.wnz + kBX - 1) / kBX, (d.wnx + kBY - 1) / kBY, n);
  for (int it = d.nt - 1; it >= 0; --it) {
    StrArgs sr = str_args(c, *c->fw_cur, it);
    sr.e = c->e;
    sr.st = c->st_a;
    sr.strips_on = strips;
    LAUNCHP("str_rev", kBytesStrRev * CELLS(n), k_str<kRev>, grid, blk, sr);
    VelArgs vr = vel_args(c, *c->fw_cur, it);
    vr.st = c->st_a;
    vr.strips_outer = strips;
    LAUNCHP("vel_rev", kBytesVel * CELLS(n), k_vel<kRev>, grid, blk, vr);
    StrArgs sa = str_args(c, c->abk, it);
    sa.res_on = 1; sa.res_vz = c->rec[0]; sa.res_vx = c->rec[1];
    LAUNCHP("str_adj", kBytesStrAdj * CELLS(n), k_str<kAdj>, grid, blk, sa);
    VelArgs va = vel_args(c, c->abk, it);
    LAUNCHP("vel_adj", kBytesVelAdj * CELLS(n), k_vel<kAdj>, grid, blk, va);
    ImgArgs im{};
    im.d = d; im.shots = c->d_shots; im.p = c->par; im.e = c->e;
    im.atxx = c->abk.txx; im.atzz = c->abk.tzz; im.atxz = c->abk.txz;
    im.vx = c->fw_cur->vx; im.vz = c->fw_cur->vz;
    im.img = c->img_slot; im.img_plane = (long long)plane; im.full = 0;
    LAUNCHP("image", kBytesImage * WCELLS(n), k_image, igrid, blk, im);
  }
  CK(cudaGetLastError());
  return reduce_images(c, n, 3);
}

// ELSRTM forward pass on the ring kernels (FD2DGPU.cu:4396-4478): per step one launch per
// wavefield set -- the background writing its Born source, the first-order set reading it as an
// overlay, recording and writing its own Born source, the second-order set reading that and
// recording -- each set ping-ponging between two buffers, then the strips of the background and
// the first-order set.  The final states are copied back into fw, b1, b2 where the half-step
// pass leaves them.
int elsrtm_forward_fused(ds2d_ctx *c, int n, bool strips) {
  const Dims &d = c->d;
  int rc;
  if (!c->fw2.vx && (rc = alloc_wave(c, c->fw2, false))) return rc;
  if (!c->b1_2.vx && (rc = alloc_wave(c, c->b1_2, false))) return rc;
  if (!c->b2_2.vx && (rc = alloc_wave(c, c->b2_2, false))) return rc;
  for (int i = 0; i < 3; i++)
    if (!c->ov_s2[i] && (rc = alloc_slots(c, &c->ov_s2[i]))) return rc;
  for (const Wave *w : {&c->fw2, &c->b1_2, &c->b2_2})
    if ((rc = zero_wave(c, *w, n))) return rc;
  const size_t bytes = sizeof(float) * (size_t)d.slot * n;
  for (int i = 0; i < 3; i++) CK(cudaMemsetAsync(c->ov_s2[i], 0, bytes, c->stream));
  int nstrips, tz;
  strip_split(d, kFB, &nstrips, &tz);
  const int xr = std::max(8, c->opt_xr);
  dim3 grid(nstrips, (d.nxp + xr - 1) / xr, n);
  Wave *set[3][2] = {{&c->fw, &c->fw2}, {&c->b1, &c->b1_2}, {&c->b2, &c->b2_2}};
  float *const *ov[2] = {c->ov_s, c->ov_s2};  // Born source of the background / of b1
  int cur = 0;
  for (int it = 0; it < d.nt; it++, cur ^= 1) {
    for (int m = 0; m < 3; m++) {
      FwdFusedArgs a{};
      a.d = d; a.a = *set[m][cur]; a.b = *set[m][cur ^ 1]; a.p = c->par; a.shots = c->d_shots;
      a.wavelet = c->wavelet; a.it = it; a.tz = tz; a.xr = xr; a.rmap = c->d_rmap;
      if (m > 0) {
        a.rec_on = 1; a.rec_vz = c->rec[2 * m]; a.rec_vx = c->rec[2 * m + 1];
        a.ovi_txx = ov[m - 1][0]; a.ovi_tzz = ov[m - 1][1]; a.ovi_txz = ov[m - 1][2];
      }
      if (m < 2) { a.ovo_txx = ov[m][0]; a.ovo_tzz = ov[m][1]; a.ovo_txz = ov[m][2]; }
      const int mode = m + 1;
      const size_t sm = sizeof(float) * kBornRing * fwd_ring_fields(!d.rbc, mode) * kFB;
      FwdFn kfn = fwd_mode_fn(d.rbc != 0, mode);
      LAUNCHS("fwd_born", kBytesBornMode[mode] * CELLS(n), kfn, grid, kFB, sm, a);
    }
    if (strips) {
      strip_save(c, *set[0][cur ^ 1], c->st_a, it, n);
      strip_save(c, *set[1][cur ^ 1], c->st_b, it, n);
    }
  }
  if (cur == 1)
    for (int m = 0; m < 3; m++) {
      const Wave &src = *set[m][1], &dst = *set[m][0];
      const float *from[5] = {src.vx, src.vz, src.txx, src.tzz, src.txz};
      float *to[5] = {dst.vx, dst.vz, dst.txx, dst.tzz, dst.txz};
      for (int i = 0; i < 5; i++)
        CK(cudaMemcpyAsync(to[i], from[i], bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
  CK(cudaGetLastError());
  return DS2D_OK;
}

// ELSRTM backward pass on the ring kernels (FD2DGPU.cu:4685-4807): per step k_bwd_ring
// (background reconstruction, adjoint with the NCC source, images 0-2), k_born of the
// background's reconstructed velocities, then k_bwd_scat_ring (first-order set reconstruction
// with that Born source, images 3-4).  Each set ping-pongs between two buffers that both start
// from its final forward state, so the cells the interior reconstruction never updates stay
// frozen in both.
int elsrtm_backward_fused(ds2d_ctx *c, int n, bool strips) {
  const Dims &d = c->d;
  int rc;
  if (!c->abk2.vx && (rc = alloc_wave(c, c->abk2, true))) return rc;
  if ((rc = zero_wave(c, c->abk2, n))) return rc;
  const size_t bytes = sizeof(float) * (size_t)d.slot * n;
  for (int m = 0; m < 2; m++) {
    const Wave &src = m ? c->b1 : c->fw, &dst = m ? c->b1_2 : c->fw2;
    const float *from[5] = {src.vx, src.vz, src.txx, src.tzz, src.txz};
    float *to[5] = {dst.vx, dst.vz, dst.txx, dst.tzz, dst.txz};
    for (int i = 0; i < 5; i++)
      CK(cudaMemcpyAsync(to[i], from[i], bytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  int nstrips, tz;
  strip_split(d, kFB, &nstrips, &tz);
  const int xr = std::max(8, c->opt_xr);
  dim3 grid(nstrips, (d.nxp + xr - 1) / xr, n);
  dim3 bgrid = cell_grid(d, n), blk(kBX, kBY);
  const long long plane = (long long)c->B * d.wnx * d.ild;
  Wave *fc = &c->fw, *fn = &c->fw2, *ac = &c->abk, *an = &c->abk2, *bc = &c->b1, *bn = &c->b1_2;
  const size_t sm = sizeof(float) * 4 * bwd_ring_fields(!d.rbc) * kFB;
  const size_t sm2 = sizeof(float) * 4 * kBwdScatRingFields * kFB;
  for (int it = d.nt - 1; it >= 0; --it) {
    BwdFusedArgs a{};
    a.d = d; a.ra = *fc; a.rb = *fn; a.aa = *ac; a.ab = *an; a.p = c->par;
    a.shots = c->d_shots; a.rmap = c->d_rmap; a.res_vz = c->rec[6]; a.res_vx = c->rec[7];
    a.st = c->st_a; a.strips_on = strips; a.it = it; a.tz = tz; a.xr = xr;
    a.img = c->img_slot; a.img_plane = plane;
    BwdFn kfn = bwd_ring_fn(d.rbc != 0, 4, 0, kFB, c->opt_bwd_1b != 0);
    LAUNCHS("bwd_fused", kBytesBwdFused * CELLS(n), kfn, grid, kFB, sm, a);
    BornArgs bs{d, c->d_shots, fn->vx, fn->vz, c->par, c->ov_s[0], c->ov_s[1], c->ov_s[2]};
    LAUNCH(k_born, bgrid, blk, bs);
    BwdScatArgs b{};
    b.d = d; b.ra = *bc; b.rb = *bn; b.atxx = an->txx; b.atzz = an->tzz; b.atxz = an->txz;
    b.ov_txx = c->ov_s[0]; b.ov_tzz = c->ov_s[1]; b.ov_txz = c->ov_s[2]; b.p = c->par;
    b.shots = c->d_shots; b.st = c->st_b; b.strips_on = strips; b.it = it; b.tz = tz; b.xr = xr;
    b.img = c->img_slot; b.img_plane = plane;
    ScatFn kfn2 = bwd_scat_fn(d.rbc != 0);
    LAUNCHS("bwd_scat", kBytesBwdScat * CELLS(n), kfn2, grid, kFB, sm2, b);
    std::swap(fc, fn);
    std::swap(ac, an);
    std::swap(bc, bn);
  }
  CK(cudaGetLastError());
  return DS2D_OK;
}

int elsrtm_batch(ds2d_ctx *c, const ds2d_shot *shots, int n, int shot_base, int iter,
                 double *mis_host) {
  const Dims &d = c->d;
  int rc;
  if ((rc = setup_batch(c, n, shot_base, true))) return rc;
  for (const Wave *w : {&c->fw, &c->b1, &c->b2, &c->abk, &c->bbk})
    if ((rc = zero_wave(c, *w, n))) return rc;
  size_t bytes = sizeof(float) * (size_t)d.slot * n;
  for (int i = 0; i < 3; i++) CK(cudaMemsetAsync(c->ov_s[i], 0, bytes, c->stream));
  for (int i = 0; i < 2; i++) CK(cudaMemsetAsync(c->ov_v[i], 0, bytes, c->stream));
  size_t plane = (size_t)c->B * d.wnx * d.ild;
  CK(cudaMemsetAsync(c->img_slot, 0, 7 * plane * sizeof(float), c->stream));
  size_t nrec = (size_t)n * d.max_ntr * d.nt;
  for (int i = 2; i < 6; i++) CK(cudaMemsetAsync(c->rec[i], 0, nrec * sizeof(float), c->stream));
  const bool strips = !d.rbc;
  dim3 grid = cell_grid(d, n), blk(kBX, kBY);
  // Forward pass, FD2DGPU.cu:4396-4478: background, first- and second-order scattered sets.
  // The ring kernels compute the Born source from the new velocities inside their stress stage;
  // that needs every interior cell inside the updated band (pml >= nop).
  const bool fused_fwd = c->opt_fused && c->opt_ring == 4 && c->ring_ok && d.pml >= d.nop;
  if (fused_fwd && (rc = elsrtm_forward_fused(c, n, strips))) return rc;
  for (int it = 0; it < d.nt && !fused_fwd; it++) {
    VelArgs v = vel_args(c, c->fw, it);
    v.src_on = 1;
    LAUNCH(k_vel<kFwd>, grid, blk, v);
    StrArgs s = str_args(c, c->fw, it);
    LAUNCH(k_str<kFwd>, grid, blk, s);
    BornArgs bs{d, c->d_shots, c->fw.vx, c->fw.vz, c->par, c->ov_s[0], c->ov_s[1], c->ov_s[2]};
    LAUNCH(k_born, grid, blk, bs);
    VelArgs v1 = vel_args(c, c->b1, it);
    v1.ov_txx = c->ov_s[0]; v1.ov_tzz = c->ov_s[1]; v1.ov_txz = c->ov_s[2];
    v1.rec_on = 1; v1.rec_vz = c->rec[2]; v1.rec_vx = c->rec[3];
    LAUNCH(k_vel<kFwd>, grid, blk, v1);
    StrArgs s1 = str_args(c, c->b1, it);
    LAUNCH(k_str<kFwd>, grid, blk, s1);
    BornArgs bs2{d, c->d_shots, c->b1.vx, c->b1.vz, c->par, c->ov_s[0], c->ov_s[1], c->ov_s[2]};
    LAUNCH(k_born, grid, blk, bs2);
    VelArgs v2 = vel_args(c, c->b2, it);
    v2.ov_txx = c->ov_s[0]; v2.ov_tzz = c->ov_s[1]; v2.ov_txz = c->ov_s[2];
    v2.rec_on = 1; v2.rec_vz = c->rec[4]; v2.rec_vx = c->rec[5];
    LAUNCH(k_vel<kFwd>, grid, blk, v2);
    StrArgs s2 = str_args(c, c->b2, it);
    LAUNCH(k_str<kFwd>, grid, blk, s2);
    if (strips) {
      strip_save(c, c->fw, c->st_a, it, n);
      strip_save(c, c->b1, c->st_b, it, n);
    }
  }
  // Lm + Lm2 and the NCC adjoint source (FD2DGPU.cu:4532, 4556-4664).
  k_lm_add<<<(unsigned)((nrec + 255) / 256), 256, 0, c->stream>>>(c->rec[2], c->rec[3], c->rec[4],
                                                                   c->rec[5], (long long)nrec);
  c->last_launches++;
  k_ncc<<<dim3(d.max_ntr, n), 256, 0, c->stream>>>(d, c->d_shots, c->rec[2], c->rec[3], c->rec[0],
                                                   c->rec[1], c->rec[6], c->rec[7], c->d_mis, iter);
  c->last_launches++;
  CK(cudaGetLastError());
  dim3 igrid((d.wnz + kBX - 1) / kBX, (d.wnx + kBY - 1) / kBY, n);
  // Backward pass, FD2DGPU.cu:4685-4807 (the fused path has no scattered-adjoint term).
  const bool fused_bwd = fused_fwd && !c->opt_adjoint_born;
  if (fused_bwd && (rc = elsrtm_backward_fused(c, n, strips))) return rc;
  for (int it = d.nt - 1; it >= 0 && !fused_bwd; --it) {
    StrArgs sr = str_args(c, c->fw, it);
    sr.e = c->e; sr.st = c->st_a; sr.strips_on = strips;
    LAUNCH(k_str<kRev>, grid, blk, sr);
    VelArgs vr = vel_args(c, c->fw, it);
    vr.st = c->st_a; vr.strips_outer = strips;
    LAUNCH(k_vel<kRev>, grid, blk, vr);
    StrArgs sb = str_args(c, c->b1, it);
    sb.e = c->be; sb.st = c->st_b; sb.strips_on = strips;
    LAUNCH(k_str<kRev>, grid, blk, sb);
    BornArgs bs{d, c->d_shots, c->fw.vx, c->fw.vz, c->par, c->ov_s[0], c->ov_s[1], c->ov_s[2]};
    LAUNCH(k_born, grid, blk, bs);
    VelArgs vb = vel_args(c, c->b1, it);
    vb.ov_txx = c->ov_s[0]; vb.ov_tzz = c->ov_s[1]; vb.ov_txz = c->ov_s[2];
    vb.st = c->st_b; vb.strips_outer = strips;
    LAUNCH(k_vel<kRev>, grid, blk, vb);
    StrArgs sa = str_args(c, c->abk, it);
    sa.res_on = 1; sa.res_vz = c->rec[6]; sa.res_vx = c->rec[7];
    LAUNCH(k_str<kAdj>, grid, blk, sa);
    VelArgs va = vel_args(c, c->abk, it);
    LAUNCH(k_vel<kAdj>, grid, blk, va);
    if (c->opt_adjoint_born) {
      // pure_born_reconstruct_backward(-1, backward), FD2DGPU.cu:1881-1889, as written.  In the
      // reference's own runs add_born_source_adjoint never executes (96 registers x 1024-thread
      // blocks exceeds the 65,536-register limit and the launch error is never checked), so
      // the scattered adjoint stays zero; that observed behaviour is the default.
      VelArgs vbb = vel_args(c, c->bbk, it);
      LAUNCH(k_vel<kAdj>, grid, blk, vbb);
      BornAdjArgs ba{d, c->d_shots, c->abk.txx, c->abk.tzz, c->abk.txz, c->par, c->ov_v[0], c->ov_v[1]};
      LAUNCH(k_born_adj, grid, blk, ba);
      StrArgs sbb = str_args(c, c->bbk, it);
      sbb.ov_vx = c->ov_v[0]; sbb.ov_vz = c->ov_v[1];
      LAUNCH(k_str<kAdj>, grid, blk, sbb);
    }
    ImgArgs im{};
    im.d = d; im.shots = c->d_shots; im.p = c->par; im.e = c->e; im.be = c->be;
    im.atxx = c->abk.txx; im.atzz = c->abk.tzz; im.atxz = c->abk.txz;
    im.btxx = c->bbk.txx; im.btzz = c->bbk.tzz; im.btxz = c->bbk.txz;
    im.vx = c->fw.vx; im.vz = c->fw.vz;
    im.img = c->img_slot; im.img_plane = (long long)plane; im.full = c->opt_adjoint_born ? 2 : 1;
    LAUNCH(k_image, igrid, blk, im);
  }
  CK(cudaGetLastError());
  if ((rc = reduce_images(c, n, 7))) return rc;
  std::vector<double> terms((size_t)n * d.max_ntr);
  CK(cudaMemcpyAsync(terms.data(), c->d_mis, terms.size() * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (mis_host && iter != 0)
    for (int s = 0; s < n; s++)
      for (int t = 0; t < shots[s].ntr; t++) *mis_host -= terms[(size_t)s * d.max_ntr + t];
  return DS2D_OK;
}

// ---- acoustic Born pair and CG-LSRTM ---------------------------------------------------------

int ensure_acoustic(ds2d_ctx *c) {
  int rc;
  if ((rc = ensure_common(c))) return rc;
  if (!c->d.rbc) {  // PML: split stress in the damped cells, background strips for L^T
    for (float *&p : c->ac_split)
      if (!p && (rc = alloc_slots(c, &p))) return rc;
    // the L^T replay saves the strips of every step, or with checkpoints of one segment
    const int k = c->opt_ac_ckpt;
    const int steps = k > 0 && k < c->d.nt ? k : c->d.nt;
    if ((rc = ensure_strips(c, c->st_a, c->st_a_steps, steps))) return rc;
  }
  if (!c->p_dmp) {
    if ((rc = alloc_slots(c, &c->p_dmp))) return rc;
    if ((rc = alloc_slots(c, &c->p_dms))) return rc;
    c->par.dmp = c->p_dmp;
    c->par.dms = c->p_dms;
  }
  for (float *&p : c->ac)
    if (!p && (rc = alloc_slots(c, &p))) return rc;
  if (c->opt_fused && c->ring_ok)
    for (float *&p : c->ac2)
      if (!p && (rc = alloc_slots(c, &p))) return rc;
  if (!c->img_slot) {  // per-shot gradient planes (same 7-plane size as the RTM images)
    size_t n = (size_t)7 * c->B * c->d.wnx * c->d.ild;
    if ((rc = alloc(c, (void **)&c->img_slot, n * sizeof(float)))) return rc;
  }
  if (!c->dot_part) {
    if ((rc = alloc(c, (void **)&c->dot_part, sizeof(double) * kDotBlocks))) return rc;
    if ((rc = alloc(c, (void **)&c->dot_out, sizeof(double)))) return rc;
  }
  return DS2D_OK;
}

AcArgs ac_args(ds2d_ctx *c, int set, int it, float dir) {
  AcArgs a{};
  a.d = c->d; a.shots = c->d_shots; a.p = c->par;
  a.vx = c->ac[3 * set]; a.vz = c->ac[3 * set + 1]; a.s = c->ac[3 * set + 2];
  if (!c->d.rbc && set < 2) {
    a.sx = c->ac_split[2 * set];
    a.sz = c->ac_split[2 * set + 1];
  }
  a.wavelet = c->wavelet; a.it = it; a.dir = dir; a.rmap = c->d_rmap;
  return a;
}

// One fused acoustic forward step (k_ac_ring) of the buffer pair `set` (0 background, 1
// scattered) from ping-pong side `cur` to 1 - cur.
int ac_ring_step(ds2d_ctx *c, int n, int set, int cur, int it, bool born_out, bool record) {
  const Dims &d = c->d;
  const int nstrips = (d.nzp + kFTZ - 1) / kFTZ;
  const int tz = (d.nzp + nstrips - 1) / nstrips;
  const int xr = std::max(8, c->opt_xr);
  dim3 grid(nstrips, (d.nxp + xr - 1) / xr, n);
  float *side[2][3] = {{c->ac[3 * set], c->ac[3 * set + 1], c->ac[3 * set + 2]},
                       {c->ac2[3 * set], c->ac2[3 * set + 1], c->ac2[3 * set + 2]}};
  AcRingArgs a{};
  a.d = d; a.shots = c->d_shots;
  a.vx = side[cur][0]; a.vz = side[cur][1]; a.s = side[cur][2];
  a.vx_n = side[1 - cur][0]; a.vz_n = side[1 - cur][1]; a.s_n = side[1 - cur][2];
  a.b = c->par.b; a.lam = c->par.lam; a.m = c->par.dmp;
  a.wavelet = c->wavelet; a.it = it; a.tz = tz; a.xr = xr; a.rmap = c->d_rmap;
  if (set == 0) {
    a.e_out = born_out ? c->ac[9] : nullptr;
  } else {
    a.e_in = c->ac[9];
    if (record) { a.rec_vz = c->rec[0]; a.rec_vx = c->rec[1]; }
  }
  if (ac_pair_on(c)) {
    const int pc = ac_pair_cta(c);
    int pns, ptz;
    pair_split(d, pc, &pns, &ptz);
    const int pxr = pair_xr(c, pns, c->occ_ac_pair[ac_pair_idx(pc)]);
    a.tz = ptz; a.xr = pxr; a.err = c->d_err;
    dim3 pgrid(pns, (d.nxp + pxr - 1) / pxr, n);
    LAUNCHS("ac_pair", 0, ac_pair_fn(set, pc), pgrid, pc, ac_pair_smem(pc), a);
    return DS2D_OK;
  }
  const size_t sm = sizeof(float) * 4 * kAcRingFields * kFB;
  void (*kfn)(AcRingArgs) = set == 0 ? k_ac_ring<0, 4> : k_ac_ring<1, 4>;
  LAUNCHS("ac_ring", 0, kfn, grid, kFB, sm, a);
  return DS2D_OK;
}

// L m for the uploaded batch: scattered vz / vx into rec[0] / rec[1] (m = the window p_dmp).
int ac_L_batch(ds2d_ctx *c, int n) {
  const Dims &d = c->d;
  size_t bytes = sizeof(float) * (size_t)d.slot * n;
  if (!d.rbc)
    for (float *p : c->ac_split) CK(cudaMemsetAsync(p, 0, bytes, c->stream));
  if (d.rbc && c->opt_fused && c->ring_ok && c->ac2[0]) {
    // fused: per step one background launch (Born source out) and one scattered launch
    for (int i = 0; i < 10; i++)
      if (i < 6 || i == 9) CK(cudaMemsetAsync(c->ac[i], 0, bytes, c->stream));
    for (float *p : c->ac2) CK(cudaMemsetAsync(p, 0, bytes, c->stream));
    size_t nrec = (size_t)n * d.max_ntr * d.nt;
    CK(cudaMemsetAsync(c->rec[0], 0, nrec * 4, c->stream));
    CK(cudaMemsetAsync(c->rec[1], 0, nrec * 4, c->stream));
    int rc;
    for (int it = 0, cur = 0; it < d.nt; it++, cur ^= 1) {
      if ((rc = ac_ring_step(c, n, 0, cur, it, true, false))) return rc;
      if ((rc = ac_ring_step(c, n, 1, cur, it, false, true))) return rc;
    }
    CK(cudaGetLastError());
    return DS2D_OK;
  }
  for (int i = 0; i < 10; i++)
    if (i < 6 || i == 9) CK(cudaMemsetAsync(c->ac[i], 0, bytes, c->stream));
  size_t nrec = (size_t)n * d.max_ntr * d.nt;
  CK(cudaMemsetAsync(c->rec[0], 0, nrec * 4, c->stream));
  CK(cudaMemsetAsync(c->rec[1], 0, nrec * 4, c->stream));
  dim3 grid = cell_grid(d, n), blk(32, 8);
  for (int it = 0; it < d.nt; it++) {
    AcArgs b = ac_args(c, 0, it, 1.f);
    b.src_on = 1;
    LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, b);
    LAUNCHP("ac_str", 0, k_ac_str, grid, blk, b);
    k_ac_born<<<grid, blk, 0, c->stream>>>(d, c->d_shots, c->par, c->ac[0], c->ac[1], c->ac[9]);
    c->last_launches++;
    AcArgs s = ac_args(c, 1, it, 1.f);
    s.e = c->ac[9];
    s.rec_on = 1; s.rec_vz = c->rec[0]; s.rec_vx = c->rec[1];
    LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, s);
    LAUNCHP("ac_str", 0, k_ac_str, grid, blk, s);
  }
  CK(cudaGetLastError());
  return DS2D_OK;
}

// L^T r with a PML (half steps): forward replay of the background (damped) saving the strips of
// vx, vz each step, then per step in reverse: the step's strips restored into the band, the
// transpose of the damped scattered step (records injected, gradient with the background
// velocities after the step), and the interior reconstruction of the background one step back.
// Saves (save) or restores background snapshot `snap` of the PML L^T: vx, vz, s and the split
// stress sx, sz of every slot, in the strip precision with per-field, per-shot FP32 scales.
int ac_ckpt_io(ds2d_ctx *c, int n, int snap, bool save) {
  const Dims &d = c->d;
  CkptArgs a{};
  a.slot = (long long)d.slot;
  a.prec = c->o.strip_precision;
  a.B = c->B;
  float *f[kCkptFields] = {c->ac[0], c->ac[1], c->ac[2], c->ac_split[0], c->ac_split[1]};
  for (int i = 0; i < kCkptFields; i++) {
    a.f[i] = f[i];
    a.fw[i] = f[i];
  }
  const size_t esz = a.prec == DS2D_STRIPS_F32 ? 4 : 2;
  const size_t per = (size_t)kCkptFields * c->B * d.slot;
  a.data = (char *)c->ckpt + (size_t)snap * per * esz;
  a.scale = c->ckpt_scale + (size_t)snap * kCkptFields * c->B;
  a.amax = c->ckpt_amax;
  dim3 grid((unsigned)std::min<long long>(((long long)d.slot + 255) / 256, 64), kCkptFields, n);
  if (save) {
    if (a.prec != DS2D_STRIPS_F32) {
      CK(cudaMemsetAsync(c->ckpt_amax, 0, sizeof(unsigned) * kCkptFields * c->B, c->stream));
      LAUNCH(k_ckpt_absmax, grid, 256, a);
    }
    LAUNCH(k_ckpt_encode, grid, 256, a);
  } else {
    LAUNCH(k_ckpt_decode, grid, 256, a);
  }
  return DS2D_OK;
}

// One reverse step of the PML L^T: the band of the background from the strips (row `srow` of
// the strip buffer described by `ds`), the adjoint step with the gradient, the interior of the
// background one step back.
void ac_LT_pml_reverse_step(ds2d_ctx *c, int n, const Dims &ds, int srow, int it) {
  const Dims &d = c->d;
  dim3 grid = cell_grid(d, n), blk(32, 8);
  AcStripArgs ld{ds, c->d_shots, c->ac[0], c->ac[1], c->st_a, srow};
  LAUNCH(k_ac_strip_load, dim3((d.lb + 255) / 256, 2, n), 256, ld);
  AcAdjArgs y{};
  y.d = d; y.shots = c->d_shots; y.p = c->par;
  y.yx = c->ac[6]; y.yz = c->ac[7]; y.ys = c->ac[8];
  y.ysx = c->ac_split[4]; y.ysz = c->ac_split[5];
  y.rmap = c->d_rmap; y.res_vz = c->rec[0]; y.res_vx = c->rec[1]; y.it = it;
  y.bvx = c->ac[0]; y.bvz = c->ac[1]; y.grad = c->img_slot;
  LAUNCHP("ac_adj_v", 0, k_ac_adj_v, grid, blk, y);
  LAUNCHP("ac_adj_s", 0, k_ac_adj_s, grid, blk, y);
  AcArgs b = ac_args(c, 0, it, -1.f);  // background back to step it-1 on the interior
  b.src_on = 1;
  b.interior = 1;
  b.sx = b.sz = nullptr;
  LAUNCHP("ac_str", 0, k_ac_str, grid, blk, b);
  LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, b);
}

// PML L^T with background checkpoints every K steps (option "ac_ckpt"): a forward pass keeps
// snapshots 0 .. nseg-2 (the state before steps 0, K, 2K, ...); then, from the last segment to the
// first, the segment's start state (the exact state for the last, a decoded snapshot for the
// others) is replayed over its steps saving their strips into a K-step buffer, and the segment is
// reversed with them.  Forward work: (nseg - 1) K + nt steps instead of nt.
int ac_LT_batch_pml_ckpt(ds2d_ctx *c, int n, int K) {
  const Dims &d = c->d;
  const int nseg = (d.nt + K - 1) / K;
  const size_t esz = c->o.strip_precision == DS2D_STRIPS_F32 ? 4 : 2;
  const int nsnap = std::max(1, nseg - 1);
  const size_t need = (size_t)nsnap * kCkptFields * c->B * d.slot * esz;
  int rc;
  if (c->ckpt_bytes < need) {
    release(c, c->ckpt);
    release(c, c->ckpt_scale);
    c->ckpt = nullptr;
    c->ckpt_scale = nullptr;
    c->ckpt_bytes = 0;
    if ((rc = alloc(c, &c->ckpt, need))) return rc;
    if ((rc = alloc(c, (void **)&c->ckpt_scale, sizeof(float) * nsnap * kCkptFields * c->B)))
      return rc;
    c->ckpt_bytes = need;
  }
  if (!c->ckpt_amax &&
      (rc = alloc(c, (void **)&c->ckpt_amax, sizeof(unsigned) * kCkptFields * c->B)))
    return rc;
  dim3 grid = cell_grid(d, n), blk(32, 8);
  auto fwd_step = [&](int it) {
    AcArgs b = ac_args(c, 0, it, 1.f);
    b.src_on = 1;
    LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, b);
    LAUNCHP("ac_str", 0, k_ac_str, grid, blk, b);
  };
  for (int it = 0; it < (nseg - 1) * K; it++) {
    if (it % K == 0 && (rc = ac_ckpt_io(c, n, it / K, true))) return rc;
    fwd_step(it);
  }
  Dims dk = d;
  dk.nt = K;  // strip rows of one segment
  for (int j = nseg - 1; j >= 0; --j) {
    const int t0 = j * K, t1 = std::min(d.nt, t0 + K);
    if (j < nseg - 1 && (rc = ac_ckpt_io(c, n, j, false))) return rc;
    for (int it = t0; it < t1; it++) {
      fwd_step(it);
      StripSaveArgs sv{dk, c->d_shots, c->ac[0], c->ac[1], c->st_a, it - t0};
      LAUNCH(k_strip_save, dim3((d.lb + 255) / 256, 2, n), 256, sv);
    }
    for (int it = t1 - 1; it >= t0; --it) ac_LT_pml_reverse_step(c, n, dk, it - t0, it);
  }
  CK(cudaGetLastError());
  return reduce_images(c, n, 1);
}

int ac_LT_batch_pml(ds2d_ctx *c, int n) {
  const Dims &d = c->d;
  size_t bytes = sizeof(float) * (size_t)d.slot * n;
  for (float *p : c->ac_split) CK(cudaMemsetAsync(p, 0, bytes, c->stream));
  if (c->opt_ac_ckpt > 0 && c->opt_ac_ckpt < d.nt) return ac_LT_batch_pml_ckpt(c, n, c->opt_ac_ckpt);
  dim3 grid = cell_grid(d, n), blk(32, 8);
  for (int it = 0; it < d.nt; it++) {
    AcArgs b = ac_args(c, 0, it, 1.f);
    b.src_on = 1;
    LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, b);
    LAUNCHP("ac_str", 0, k_ac_str, grid, blk, b);
    StripSaveArgs sv{d, c->d_shots, c->ac[0], c->ac[1], c->st_a, it};
    LAUNCH(k_strip_save, dim3((d.lb + 255) / 256, 2, n), 256, sv);
  }
  for (int it = d.nt - 1; it >= 0; --it) ac_LT_pml_reverse_step(c, n, d, it, it);
  CK(cudaGetLastError());
  return reduce_images(c, n, 1);
}

// L^T r for the uploaded batch (r in rec[0] / rec[1]); the windowed gradients are added into
// the model-size image 0.
int ac_LT_batch(ds2d_ctx *c, int n) {
  const Dims &d = c->d;
  size_t bytes = sizeof(float) * (size_t)d.slot * n;
  for (int i = 0; i < 9; i++)
    if (i < 3 || i >= 6) CK(cudaMemsetAsync(c->ac[i], 0, bytes, c->stream));
  size_t plane = (size_t)c->B * d.wnx * d.ild;
  CK(cudaMemsetAsync(c->img_slot, 0, plane * sizeof(float), c->stream));
  dim3 grid = cell_grid(d, n), blk(32, 8);
  if (!d.rbc) return ac_LT_batch_pml(c, n);
  const bool fused = c->opt_fused && c->ring_ok && c->ac2[0];
  if (fused) {
    // fused forward replay of the background, final state left in ac[0..2]
    for (int i = 0; i < 3; i++) CK(cudaMemsetAsync(c->ac2[i], 0, bytes, c->stream));
    int rc, cur = 0;
    for (int it = 0; it < d.nt; it++, cur ^= 1)
      if ((rc = ac_ring_step(c, n, 0, cur, it, false, false))) return rc;
    if (cur == 1)
      for (int i = 0; i < 3; i++)
        CK(cudaMemcpyAsync(c->ac[i], c->ac2[i], bytes, cudaMemcpyDeviceToDevice, c->stream));
    // fused reversal: one k_ac_rev_ring launch per step; the background ping-pongs between
    // ac[0..2] and ac2[0..2], the adjoint state between ac[6..8] and ac2[3..5] (both start at
    // zero; cells outside the updated band are never written in either)
    for (int i = 3; i < 6; i++) CK(cudaMemsetAsync(c->ac2[i], 0, bytes, c->stream));
    if (ac_rev_pair_on(c)) {
      const int pc = ac_rev_cta(c);
      int pns, ptz;
      ac_rev_split(d, pc, &pns, &ptz);
      const int pxr = pair_xr(c, pns, c->occ_ac_rev[pc == 192 ? 0 : 1]);
      dim3 pgrid(pns, (d.nxp + pxr - 1) / pxr, n);
      float *bk[2][3] = {{c->ac[0], c->ac[1], c->ac[2]}, {c->ac2[0], c->ac2[1], c->ac2[2]}};
      float *yk[2][3] = {{c->ac[6], c->ac[7], c->ac[8]}, {c->ac2[3], c->ac2[4], c->ac2[5]}};
      cur = 0;
      for (int it = d.nt - 1; it >= 0; --it, cur ^= 1) {
        AcRevArgs a{};
        a.d = d; a.shots = c->d_shots;
        a.yx = yk[cur][0]; a.yz = yk[cur][1]; a.ys = yk[cur][2];
        a.yx_n = yk[cur ^ 1][0]; a.yz_n = yk[cur ^ 1][1]; a.ys_n = yk[cur ^ 1][2];
        a.vx = bk[cur][0]; a.vz = bk[cur][1]; a.s = bk[cur][2];
        a.vx_n = bk[cur ^ 1][0]; a.vz_n = bk[cur ^ 1][1]; a.s_n = bk[cur ^ 1][2];
        a.b = c->par.b; a.lam = c->par.lam; a.grad = c->img_slot; a.wavelet = c->wavelet;
        a.it = it; a.tz = ptz; a.xr = pxr; a.rmap = c->d_rmap;
        a.res_vz = c->rec[0]; a.res_vx = c->rec[1]; a.err = c->d_err;
        LAUNCHS("ac_rev_pair", kBytesAcRev * CELLS(n), ac_rev_fn(pc), pgrid, pc,
                ac_rev_pair_smem(pc), a);
      }
      CK(cudaGetLastError());
      return reduce_images(c, n, 1);
    }
    const int nstrips = (d.nzp + kAcRevTZ - 1) / kAcRevTZ;
    const int tz = (d.nzp + nstrips - 1) / nstrips;
    const int xr = std::max(8, c->opt_xr);
    dim3 rgrid(nstrips, (d.nxp + xr - 1) / xr, n);
    float *bk[2][3] = {{c->ac[0], c->ac[1], c->ac[2]}, {c->ac2[0], c->ac2[1], c->ac2[2]}};
    float *yk[2][3] = {{c->ac[6], c->ac[7], c->ac[8]}, {c->ac2[3], c->ac2[4], c->ac2[5]}};
    const size_t sm = sizeof(float) * 4 * kAcRevRingFields * kFB;
    cur = 0;
    for (int it = d.nt - 1; it >= 0; --it, cur ^= 1) {
      AcRevArgs a{};
      a.d = d; a.shots = c->d_shots;
      a.yx = yk[cur][0]; a.yz = yk[cur][1]; a.ys = yk[cur][2];
      a.yx_n = yk[cur ^ 1][0]; a.yz_n = yk[cur ^ 1][1]; a.ys_n = yk[cur ^ 1][2];
      a.vx = bk[cur][0]; a.vz = bk[cur][1]; a.s = bk[cur][2];
      a.vx_n = bk[cur ^ 1][0]; a.vz_n = bk[cur ^ 1][1]; a.s_n = bk[cur ^ 1][2];
      a.b = c->par.b; a.lam = c->par.lam; a.grad = c->img_slot; a.wavelet = c->wavelet;
      a.it = it; a.tz = tz; a.xr = xr; a.rmap = c->d_rmap;
      a.res_vz = c->rec[0]; a.res_vx = c->rec[1];
      void (*kfn)(AcRevArgs) = k_ac_rev_ring<4>;
      LAUNCHS("ac_rev", kBytesAcRev * CELLS(n), kfn, rgrid, kFB, sm, a);
    }
    CK(cudaGetLastError());
    return reduce_images(c, n, 1);
  } else {
    for (int it = 0; it < d.nt; it++) {
      AcArgs b = ac_args(c, 0, it, 1.f);
      b.src_on = 1;
      LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, b);
      LAUNCHP("ac_str", 0, k_ac_str, grid, blk, b);
    }
  }
  for (int it = d.nt - 1; it >= 0; --it) {
    AcAdjArgs y{};
    y.d = d; y.shots = c->d_shots; y.p = c->par;
    y.yx = c->ac[6]; y.yz = c->ac[7]; y.ys = c->ac[8];
    y.rmap = c->d_rmap; y.res_vz = c->rec[0]; y.res_vx = c->rec[1]; y.it = it;
    y.bvx = c->ac[0]; y.bvz = c->ac[1]; y.grad = c->img_slot;
    LAUNCHP("ac_adj_v", 0, k_ac_adj_v, grid, blk, y);
    LAUNCHP("ac_adj_s", 0, k_ac_adj_s, grid, blk, y);
    AcArgs b = ac_args(c, 0, it, -1.f);  // background back to step it-1: stress, then velocity
    b.src_on = 1;
    LAUNCHP("ac_str", 0, k_ac_str, grid, blk, b);
    LAUNCHP("ac_vel", 0, k_ac_vel, grid, blk, b);
  }
  CK(cudaGetLastError());
  return reduce_images(c, n, 1);
}

// Applies L (m_dev -> data vector [n][max_ntr][nt] x {z, x}) or L^T (data -> grad_dev) over all
// shots in batches.  m_dev / grad_dev are model-size device arrays.
int ac_apply(ds2d_ctx *c, const ds2d_shot *shots, int n, bool adjoint, const float *m_dev,
             float *dz, float *dx, float *grad_dev) {
  const Dims &d = c->d;
  int rc;
  size_t nall = (size_t)d.allnx * d.allnz;
  if (!adjoint) CK(cudaMemcpyAsync(c->pp_all, m_dev, nall * 4, cudaMemcpyDeviceToDevice, c->stream));
  else CK(cudaMemsetAsync(c->images, 0, nall * 4, c->stream));
  const size_t per = (size_t)d.max_ntr * d.nt;
  for (int f = 0; f < n; f += c->B) {
    const int m = std::min(c->B, n - f);
    if ((rc = upload_batch(c, shots + f, m))) return rc;
    if ((rc = setup_batch(c, m, f, !adjoint))) return rc;
    if (!adjoint) {
      if ((rc = ac_L_batch(c, m))) return rc;
      CK(cudaMemcpyAsync(dz + f * per, c->rec[0], m * per * 4, cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(dx + f * per, c->rec[1], m * per * 4, cudaMemcpyDeviceToDevice, c->stream));
    } else {
      CK(cudaMemcpyAsync(c->rec[0], dz + f * per, m * per * 4, cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(c->rec[1], dx + f * per, m * per * 4, cudaMemcpyDeviceToDevice, c->stream));
      if ((rc = ac_LT_batch(c, m))) return rc;
    }
    // upload_batch of the next batch overwrites d_shots / rmap: finish this batch first.
    CK(cudaStreamSynchronize(c->stream));
    c->last_updates += 2.0 * c->batch_cells * d.nt;
  }
  if (adjoint) CK(cudaMemcpyAsync(grad_dev, c->images, nall * 4, cudaMemcpyDeviceToDevice, c->stream));
  return DS2D_OK;
}

// Work vector `i` with room for n floats (zeroed when (re)allocated).
int work_vec(ds2d_ctx *c, int i, size_t n, float **out) {
  ds2d_ctx::Vec &v = c->vecs[i];
  if (v.n < n) {
    if (v.p) cudaFree(v.p);
    v.p = nullptr;
    v.n = 0;
    cudaError_t e = cudaMalloc(&v.p, n * sizeof(float));
    if (e != cudaSuccess) {
      cudaGetLastError();
      v.p = nullptr;
      return fail(c, DS2D_E_NOMEM, "cudaMalloc(%zu floats) for a solver vector: %s", n,
                  cudaGetErrorString(e));
    }
    v.n = n;
    CK(cudaMemsetAsync(v.p, 0, n * sizeof(float), c->stream));
  }
  *out = v.p;
  return DS2D_OK;
}

// FP64 <a, b> over n floats (device), result on the host.
int dot64(ds2d_ctx *c, const float *a, const float *b, long long n, double *out) {
  k_dot_partial<<<kDotBlocks, kDotThreads, 0, c->stream>>>(a, b, n, c->dot_part);
  k_dot_final<<<1, 32, 0, c->stream>>>(c->dot_part, kDotBlocks, c->dot_out);
  c->last_launches += 2;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->dot_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DS2D_OK;
}

}  // namespace

extern "C" {

int ds2d_create(const ds2d_grid *grid, const ds2d_opts *opts, ds2d_ctx **out) {
  if (!grid || !opts || !out) return DS2D_E_ARG;
  *out = nullptr;
  ds2d_ctx *c = new ds2d_ctx();
  c->g = *grid;
  c->o = *opts;
  const ds2d_grid &g = *grid;
  const int nop = 4;
  auto bad = [&](const char *m) {
    g_create_err = m;
    delete c;
    return DS2D_E_ARG;
  };
  if (g.allnx <= 0 || g.allnz <= 0 || g.nx <= 0 || g.nx > g.allnx || g.nt <= 0)
    return bad("grid sizes must be positive with nx <= allnx");
  if (g.pml < 2 * nop) return bad("pml must be at least 8 cells (2 * nop) for the strip bands");
  if (!(g.dx > 0 && g.dz > 0 && g.dt > 0)) return bad("dx, dz, dt must be positive");
  if (opts->max_shots <= 0 || opts->max_shots > 65535) return bad("max_shots out of range");
  if (opts->max_ntr < 0) return bad("max_ntr must be >= 0");
  if (opts->strip_precision < 0 || opts->strip_precision > 2) return bad("strip_precision");
  if (opts->boundary != DS2D_BOUNDARY_PML && opts->boundary != DS2D_BOUNDARY_RANDOM)
    return bad("boundary");
  cudaError_t e = cudaSetDevice(opts->device);
  if (e != cudaSuccess) {
    g_create_err = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
    delete c;
    return DS2D_E_CUDA;
  }
  Dims &d = c->d;
  d.nxp = g.nx + 2 * g.pml;
  d.nzp = g.allnz + 2 * g.pml;
  d.ld = (d.nzp + 31) / 32 * 32;
  d.pml = g.pml;
  d.nop = nop;
  d.wnx = g.nx;
  d.wnz = g.allnz;
  d.ild = d.ld;
  d.nt = g.nt;
  d.allnx = g.allnx;
  d.allnz = g.allnz;
  d.slot = (long long)d.nxp * d.ld;
  d.dx = g.dx; d.dz = g.dz; d.dt = g.dt;
  d.rbc = opts->boundary == DS2D_BOUNDARY_RANDOM;
  d.lb = 4 * nop * (d.wnx + d.wnz);
  d.nseg = (d.lb + 31) / 32;
  d.max_ntr = std::max(opts->max_ntr, 1);
  d.nxp_max = d.nxp;
  d.wnx_max = d.wnx;
  d.lb_max = d.lb;
  d.nseg_max = d.nseg;
  c->B = opts->max_shots;
  // The ring-fed kernels index cells and image pixels with 32-bit offsets; batches whose arrays
  // exceed 2^31 elements fall back to the 64-bit fused kernels.
  c->ring_ok = (long long)c->B * d.slot < (1LL << 31) &&
               (long long)c->B * d.wnx * d.ild < (1LL << 31);
  {
    // Ring-fed kernels may use more than the default 48 KB of dynamic shared memory.
    cudaError_t e = cudaSuccess;
    for (int depth : kRingDepths) {
      for (bool rbc : {false, true})
        for (int occ : {0, 1}) {
          const int fwd_sm = (int)(sizeof(float) * depth * fwd_ring_fields(!rbc) * kFB);
          const int bwd_sm = (int)(sizeof(float) * depth * bwd_ring_fields(!rbc) * kFB);
          if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fwd_ring_fn(rbc, depth, occ),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, fwd_sm);
          if (e == cudaSuccess)
            e = cudaFuncSetAttribute(bwd_ring_fn(rbc, depth, occ),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bwd_sm);
          if (depth == 4 && occ == 0) {
            // shared memory scales with the CTA width
            if (e == cudaSuccess)
              e = cudaFuncSetAttribute(fwd_ring_fn(rbc, depth, occ, kWideCta),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       fwd_sm / kFB * kWideCta);
            if (e == cudaSuccess)
              e = cudaFuncSetAttribute(bwd_ring_fn(rbc, depth, occ, kWideCta),
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       bwd_sm / kFB * kWideCta);
            for (int cta : {kFB, kWideCta})
              if (e == cudaSuccess)
                e = cudaFuncSetAttribute(bwd_ring_fn(rbc, depth, occ, cta, true),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         bwd_sm / kFB * cta);
          }
        }
    }
    {
      const int fctas[2] = {256, 64}, bctas[3] = {256, 160, 64};
      for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        e = cudaFuncSetAttribute(pair_fwd_fn(fctas[i]), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_fwd_smem(fctas[i]));
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_pair[i], pair_fwd_fn(fctas[i]),
                                                            fctas[i], pair_fwd_smem(fctas[i]));
      }
      for (int i = 0; i < 3 && e == cudaSuccess; i++) {
        const int cta = kAcPairCtas[i];
        for (int mode = 0; mode < 2 && e == cudaSuccess; mode++)
          e = cudaFuncSetAttribute(ac_pair_fn(mode, cta),
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)ac_pair_smem(cta));
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_ac_pair[i], ac_pair_fn(1, cta),
                                                            cta, ac_pair_smem(cta));
      }
      for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        const int cta = kAcRevCtas[i];
        e = cudaFuncSetAttribute(ac_rev_fn(cta), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ac_rev_pair_smem(cta));
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_ac_rev[i], ac_rev_fn(cta), cta,
                                                            ac_rev_pair_smem(cta));
      }
      for (int part = 1; part <= 2 && e == cudaSuccess; part++) {
        e = cudaFuncSetAttribute(pair_split_fn(part), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_split_smem(part));
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_pair[4 + part],
                                                            pair_split_fn(part), kPairSplitT,
                                                            pair_split_smem(part));
      }
      for (int i = 0; i < 3 && e == cudaSuccess; i++) {
        e = cudaFuncSetAttribute(pair_bwd_fn(bctas[i]), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_bwd_smem(bctas[i]));
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_pair[2 + i],
                                                            pair_bwd_fn(bctas[i]), bctas[i],
                                                            pair_bwd_smem(bctas[i]));
      }
    }
    for (int i = 0; i < 6 && e == cudaSuccess; i++) {
      const int cta = kBulkCtas[i / 2];
      const bool one = (i & 1) != 0;
      e = cudaFuncSetAttribute(bulk_fn(cta, one), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)bwd_bulk_smem(cta));
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_bulk[bulk_idx(cta, one)],
                                                          bulk_fn(cta, one), cta,
                                                          bwd_bulk_smem(cta));
    }
    for (int i = 0; i < 3 && e == cudaSuccess; i++) {
      const int kt = kWsRoles[i];
      e = cudaFuncSetAttribute(ws_fn(kt), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)ws_smem(kt));
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_ws[i], ws_fn(kt), 2 * kt,
                                                          ws_smem(kt));
    }
    for (int i = 0; i < 2 && e == cudaSuccess; i++)
      for (int K = 1; K <= (i ? 2 : 4) && e == cudaSuccess; K++) {
        const int cta = kTbCtas[i];
        const size_t sm = tb_smem(K, cta, kTbMaxXr);
        e = cudaFuncSetAttribute(tb_fn(K, cta), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_tb[i][K - 1], tb_fn(K, cta),
                                                            cta, sm);
        if (K <= 2 && e == cudaSuccess)
          e = cudaFuncSetAttribute(tb_fn(K, cta, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sm);
        if (K <= 2 && e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c->occ_tb_bulk[i][K - 1],
                                                            tb_fn(K, cta, true), cta, sm);
      }
    int dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
    for (bool rbc : {false, true})
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(bwd_scat_fn(rbc), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(float) * 4 * kBwdScatRingFields * kFB));
    for (bool rbc : {false, true})
      for (int mode = 1; mode <= 3 && e == cudaSuccess; mode++)
        e = cudaFuncSetAttribute(fwd_mode_fn(rbc, mode), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(float) * kBornRing * fwd_ring_fields(!rbc, mode) * kFB));
    if (e != cudaSuccess) {
      g_create_err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
      delete c;
      return DS2D_E_CUDA;
    }
  }
  if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
    fail(c, DS2D_E_CUDA, "cudaStreamCreate failed");
    delete c;
    return DS2D_E_CUDA;
  }
  c->stream = c->own;
  if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    fail(c, DS2D_E_CUDA, "cudaStreamCreate / cudaEventCreate failed");
    ds2d_destroy(c);
    return DS2D_E_CUDA;
  }
  size_t nall = (size_t)g.allnx * g.allnz;
  int rc = 0;
  if ((rc = alloc(c, (void **)&c->vp_all, nall * 4)) || (rc = alloc(c, (void **)&c->vs_all, nall * 4)) ||
      (rc = alloc(c, (void **)&c->pp_all, nall * 4)) || (rc = alloc(c, (void **)&c->ps_all, nall * 4)) ||
      (rc = alloc(c, (void **)&c->images, 7 * nall * 4)) ||
      (rc = alloc(c, (void **)&c->wavelet, (size_t)g.nt * 4)) ||
      (rc = alloc(c, (void **)&c->d_err, sizeof(int)))) {
    ds2d_destroy(c);
    return rc;
  }
  if (cudaMemsetAsync(c->images, 0, 7 * nall * 4, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    ds2d_destroy(c);
    return DS2D_E_CUDA;
  }
  *out = c;
  return DS2D_OK;
}

int ds2d_destroy(ds2d_ctx *c) {
  if (!c) return DS2D_OK;
  if (c->own) cudaStreamSynchronize(c->own);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->aux) cudaStreamSynchronize(c->aux);
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.exec);
  c->graphs.clear();
  for (auto &v : c->vecs)
    if (v.p) cudaFree(v.p);
  c->arena.release();
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->aux) cudaStreamDestroy(c->aux);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return DS2D_OK;
}

const char *ds2d_last_error(const ds2d_ctx *c) { return c ? c->err.c_str() : g_create_err.c_str(); }

int ds2d_set_stream(ds2d_ctx *c, void *stream) {
  if (!c) return DS2D_E_ARG;
  c->stream = stream ? (cudaStream_t)stream : c->own;
  return DS2D_OK;
}

int ds2d_set_models(ds2d_ctx *c, const float *vp, const float *vs, const float *rho) {
  if (!c || !vp || !vs) return DS2D_E_ARG;
  size_t n = (size_t)c->g.allnx * c->g.allnz;
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(vp[i]) || !std::isfinite(vs[i]) || vp[i] <= 0.f || vs[i] < 0.f)
      return fail(c, DS2D_E_ARG, "model value at %zu is not a valid velocity (vp %g, vs %g)", i,
                  vp[i], vs[i]);
  CK(cudaMemcpyAsync(c->vp_all, vp, n * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->vs_all, vs, n * 4, cudaMemcpyHostToDevice, c->stream));
  if (rho) {
    for (size_t i = 0; i < n; i++)
      if (!std::isfinite(rho[i]) || rho[i] <= 0.f)
        return fail(c, DS2D_E_ARG, "density at %zu is not positive", i);
    if (!c->rho_all) {
      int rc = alloc(c, (void **)&c->rho_all, n * 4);
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(c->rho_all, rho, n * 4, cudaMemcpyHostToDevice, c->stream));
  } else {
    c->rho_all = nullptr;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->models_set = true;
  return DS2D_OK;
}

int ds2d_set_wavelet(ds2d_ctx *c, const float *w) {
  if (!c || !w) return DS2D_E_ARG;
  CK(cudaMemcpyAsync(c->wavelet, w, (size_t)c->g.nt * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->wavelet_set = true;
  return DS2D_OK;
}

int ds2d_set_image(ds2d_ctx *c, const float *pp, const float *ps) {
  if (!c || !pp || !ps) return DS2D_E_ARG;
  size_t n = (size_t)c->g.allnx * c->g.allnz;
  CK(cudaMemcpyAsync(c->pp_all, pp, n * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->ps_all, ps, n * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->image_set = true;
  return DS2D_OK;
}

int ds2d_forward(ds2d_ctx *c, const ds2d_shot *shots, int n, float *rec_vz, float *rec_vx) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n < 0 || (n > 0 && (!shots || !rec_vz || !rec_vx))) return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_common(c))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  long long tb = 0;
  for (int f = 0; f < n; f += c->B) {
    int m = std::min(c->B, n - f);
    if ((rc = upload_batch(c, shots + f, m))) return rc;
    if (c->opt_fused && !c->fw2.vx && (rc = alloc_wave(c, c->fw2, false))) return rc;
    const long long key[6] = {1, m, f, c->opt_fused + 2 * c->opt_ring + 32 * c->opt_occ + 64 * c->opt_cta, c->opt_xr + 1000LL * c->opt_pair_xr + 1000000LL * c->opt_pair_cta + 100000000LL * (c->opt_pair_fcta / 64 + 5 * c->opt_pair_split) + 1000000000LL * c->opt_pair + 10000000000LL * (c->opt_tb + 5 * (c->opt_tb_cta / 32)) + 1000000000000LL * (c->opt_bwd_ws / 32 + 8 * c->opt_bwd_1b + 16 * c->opt_bwd_bulk + 32 * c->opt_tb_bulk + 64 * (c->opt_bwd_cta / 64)), (long long)(size_t)c->stream};
    rc = run_graph(c, key, [&]() {
      int r;
      if ((r = setup_batch(c, m, f, false))) return r;
      if ((r = zero_wave(c, c->fw, m))) return r;
      size_t nrec = (size_t)m * c->d.max_ntr * c->d.nt;
      CK(cudaMemsetAsync(c->rec[0], 0, nrec * 4, c->stream));
      CK(cudaMemsetAsync(c->rec[1], 0, nrec * 4, c->stream));
      return run_forward_pass(c, m, true, false);
    });
    if (rc) return rc;
    if ((rc = copy_records_out(c, shots + f, m, c->rec[0], c->rec[1], tb, rec_vz, rec_vx))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < m; s++) tb += shots[f + s].ntr;
    c->last_updates += c->batch_cells * c->d.nt;
  }
  return check_pair_err(c);
}

static int rtm_common(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *az,
                      const float *ax, cudaMemcpyKind kind) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n < 0 || (n > 0 && (!shots || !az || !ax))) return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_rtm(c))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  long long tb = 0;
  for (int f = 0; f < n; f += c->B) {
    int m = std::min(c->B, n - f);
    if ((rc = upload_batch(c, shots + f, m))) return rc;
    if ((rc = copy_records_in(c, shots + f, m, az, ax, tb, c->rec[0], c->rec[1], kind))) return rc;
    if ((rc = rtm_batch(c, shots + f, m, f))) return rc;
    for (int s = 0; s < m; s++) tb += shots[f + s].ntr;
    c->last_updates += 3.0 * c->batch_cells * c->d.nt;
  }
  CK(cudaStreamSynchronize(c->stream));
  return check_pair_err(c);
}

int ds2d_rtm(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *adj_vz, const float *adj_vx) {
  return rtm_common(c, shots, n, adj_vz, adj_vx, cudaMemcpyHostToDevice);
}

int ds2d_rtm_device(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *adj_vz,
                    const float *adj_vx) {
  return rtm_common(c, shots, n, adj_vz, adj_vx, cudaMemcpyDeviceToDevice);
}

int ds2d_elsrtm(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *obs_vz,
                const float *obs_vx, int iter, double *misfit, float *lm_vz, float *lm_vx,
                float *res_vz, float *res_vx) {
  int rc;
  if ((rc = check_ready(c, true))) return rc;
  if (n < 0 || (n > 0 && (!shots || !obs_vz || !obs_vx))) return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_elsrtm(c))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  long long tb = 0;
  for (int f = 0; f < n; f += c->B) {
    int m = std::min(c->B, n - f);
    if ((rc = upload_batch(c, shots + f, m))) return rc;
    if ((rc = copy_records_in(c, shots + f, m, obs_vz, obs_vx, tb, c->rec[0], c->rec[1],
                              cudaMemcpyDefault)))
      return rc;
    if ((rc = elsrtm_batch(c, shots + f, m, f, iter, misfit))) return rc;
    if (lm_vz || lm_vx)
      if ((rc = copy_records_out(c, shots + f, m, c->rec[2], c->rec[3], tb, lm_vz, lm_vx))) return rc;
    if (res_vz || res_vx)
      if ((rc = copy_records_out(c, shots + f, m, c->rec[6], c->rec[7], tb, res_vz, res_vx))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    for (int s = 0; s < m; s++) tb += shots[f + s].ntr;
    c->last_updates += (c->opt_adjoint_born ? 7.0 : 6.0) * c->batch_cells * c->d.nt;
  }
  return DS2D_OK;
}

int ds2d_read_images(ds2d_ctx *c, float *const images[7], int reset) {
  if (!c || !images) return DS2D_E_ARG;
  size_t n = (size_t)c->g.allnx * c->g.allnz;
  for (int a = 0; a < 7; a++)
    if (images[a])
      CK(cudaMemcpyAsync(images[a], c->images + a * n, n * 4, cudaMemcpyDeviceToHost, c->stream));
  if (reset) CK(cudaMemsetAsync(c->images, 0, 7 * n * 4, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DS2D_OK;
}

int ds2d_read_images_device(ds2d_ctx *c, float *const images[7], int reset) {
  if (!c || !images) return DS2D_E_ARG;
  size_t n = (size_t)c->g.allnx * c->g.allnz;
  for (int a = 0; a < 7; a++)
    if (images[a])
      CK(cudaMemcpyAsync(images[a], c->images + a * n, n * 4, cudaMemcpyDeviceToDevice, c->stream));
  if (reset) CK(cudaMemsetAsync(c->images, 0, 7 * n * 4, c->stream));
  return DS2D_OK;
}

static int data_io(ds2d_ctx *c, const ds2d_shot *shots, int n, float *dev, float *host,
                   bool to_dev) {
  const size_t per = (size_t)c->d.max_ntr * c->d.nt;
  long long tb = 0;
  for (int s = 0; s < n; s++) {
    const size_t cnt = (size_t)shots[s].ntr * c->d.nt;
    if (cnt) {
      // cudaMemcpyDefault: the caller's records may live in host or device memory
      if (to_dev)
        CK(cudaMemcpyAsync(dev + s * per, host + tb * c->d.nt, cnt * 4, cudaMemcpyDefault, c->stream));
      else
        CK(cudaMemcpyAsync(host + tb * c->d.nt, dev + s * per, cnt * 4, cudaMemcpyDefault, c->stream));
    }
    tb += shots[s].ntr;
  }
  return DS2D_OK;
}

static int check_shots(ds2d_ctx *c, const ds2d_shot *shots, int n) {
  for (int s = 0; s < n; s++)
    if (shots[s].ntr > c->d.max_ntr) return fail(c, DS2D_E_ARG, "shot %d: ntr > max_ntr", s);
  return DS2D_OK;
}

int ds2d_ac_born(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *m, float *rec_vz,
                 float *rec_vx) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n <= 0 || !shots || !m || !rec_vz || !rec_vx) return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_acoustic(c)) || (rc = check_shots(c, shots, n))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  const size_t nall = (size_t)c->d.allnx * c->d.allnz, nd = (size_t)n * c->d.max_ntr * c->d.nt;
  float *mv, *dz, *dx;
  if ((rc = work_vec(c, 0, nall, &mv)) || (rc = work_vec(c, 7, nd, &dz)) || (rc = work_vec(c, 8, nd, &dx)))
    return rc;
  CK(cudaMemcpyAsync(mv, m, nall * 4, cudaMemcpyDefault, c->stream));
  if ((rc = ac_apply(c, shots, n, false, mv, dz, dx, nullptr))) return rc;
  if ((rc = data_io(c, shots, n, dz, rec_vz, false)) || (rc = data_io(c, shots, n, dx, rec_vx, false)))
    return rc;
  CK(cudaStreamSynchronize(c->stream));
  return check_pair_err(c);
}

int ds2d_ac_born_adj(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *rec_vz,
                     const float *rec_vx, float *grad) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n <= 0 || !shots || !grad || !rec_vz || !rec_vx) return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_acoustic(c)) || (rc = check_shots(c, shots, n))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  const size_t nall = (size_t)c->d.allnx * c->d.allnz, nd = (size_t)n * c->d.max_ntr * c->d.nt;
  float *gv, *dz, *dx;
  if ((rc = work_vec(c, 1, nall, &gv)) || (rc = work_vec(c, 5, nd, &dz)) || (rc = work_vec(c, 6, nd, &dx)))
    return rc;
  CK(cudaMemsetAsync(dz, 0, nd * 4, c->stream));
  CK(cudaMemsetAsync(dx, 0, nd * 4, c->stream));
  if ((rc = data_io(c, shots, n, dz, (float *)rec_vz, true)) ||
      (rc = data_io(c, shots, n, dx, (float *)rec_vx, true)))
    return rc;
  if ((rc = ac_apply(c, shots, n, true, nullptr, dz, dx, gv))) return rc;
  CK(cudaMemcpyAsync(grad, gv, nall * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_pair_err(c);
}

int ds2d_lsrtm(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *obs_vz,
               const float *obs_vx, int niter, double target, float *m_out, double *resid,
               int *iters_done) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n <= 0 || !shots || !obs_vz || !obs_vx || !m_out || niter < 0)
    return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_acoustic(c)) || (rc = check_shots(c, shots, n))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  const size_t nall = (size_t)c->d.allnx * c->d.allnz, nd = (size_t)n * c->d.max_ntr * c->d.nt;
  float *m, *sv, *p, *rz, *rx, *qz, *qx;
  if ((rc = work_vec(c, 0, nall, &m)) || (rc = work_vec(c, 1, nall, &sv)) ||
      (rc = work_vec(c, 2, nall, &p)) || (rc = work_vec(c, 5, nd, &rz)) ||
      (rc = work_vec(c, 6, nd, &rx)) || (rc = work_vec(c, 7, nd, &qz)) ||
      (rc = work_vec(c, 8, nd, &qx)))
    return rc;
  CK(cudaMemsetAsync(m, 0, nall * 4, c->stream));
  CK(cudaMemsetAsync(rz, 0, nd * 4, c->stream));
  CK(cudaMemsetAsync(rx, 0, nd * 4, c->stream));
  if ((rc = data_io(c, shots, n, rz, (float *)obs_vz, true)) ||
      (rc = data_io(c, shots, n, rx, (float *)obs_vx, true)))
    return rc;
  // CGLS on || L m - d ||^2 with m0 = 0: r = d, s = L^T r, p = s (FP64 scalars throughout).
  double dd, tz, tx;
  if ((rc = dot64(c, rz, rz, nd, &tz)) || (rc = dot64(c, rx, rx, nd, &tx))) return rc;
  dd = tz + tx;
  if (!(dd > 0)) return fail(c, DS2D_E_NUMERIC, "observed data are zero or not finite");
  if ((rc = ac_apply(c, shots, n, true, nullptr, rz, rx, sv))) return rc;
  CK(cudaMemcpyAsync(p, sv, nall * 4, cudaMemcpyDeviceToDevice, c->stream));
  double gamma;
  if ((rc = dot64(c, sv, sv, nall, &gamma))) return rc;
  const int nb = 4 * 148;
  int k = 0;
  for (; k < niter; k++) {
    if ((rc = ac_apply(c, shots, n, false, p, qz, qx, nullptr))) return rc;
    if ((rc = dot64(c, qz, qz, nd, &tz)) || (rc = dot64(c, qx, qx, nd, &tx))) return rc;
    const double delta = tz + tx;
    if (!(delta > 0) || !std::isfinite(gamma)) return fail(c, DS2D_E_NUMERIC, "CG breakdown at %d", k);
    const double alpha = gamma / delta;
    k_axpy<<<nb, 256, 0, c->stream>>>((long long)nall, alpha, p, m);
    k_axpy<<<nb, 256, 0, c->stream>>>((long long)nd, -alpha, qz, rz);
    k_axpy<<<nb, 256, 0, c->stream>>>((long long)nd, -alpha, qx, rx);
    c->last_launches += 3;
    if ((rc = dot64(c, rz, rz, nd, &tz)) || (rc = dot64(c, rx, rx, nd, &tx))) return rc;
    const double rel = std::sqrt((tz + tx) / dd);
    if (resid) resid[k] = rel;
    if (rel <= target) {
      k++;
      break;
    }
    if ((rc = ac_apply(c, shots, n, true, nullptr, rz, rx, sv))) return rc;
    double gnew;
    if ((rc = dot64(c, sv, sv, nall, &gnew))) return rc;
    const double beta = gnew / gamma;
    gamma = gnew;
    k_xpby<<<nb, 256, 0, c->stream>>>((long long)nall, sv, beta, p);
    c->last_launches++;
  }
  if (iters_done) *iters_done = k;
  CK(cudaMemcpyAsync(m_out, m, nall * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_pair_err(c);
}

int ds2d_ac_normal(ds2d_ctx *c, const ds2d_shot *shots, int n, const float *m, float *img) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n <= 0 || !shots || !m || !img) return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_acoustic(c)) || (rc = check_shots(c, shots, n))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  const size_t nall = (size_t)c->d.allnx * c->d.allnz, nd = (size_t)n * c->d.max_ntr * c->d.nt;
  float *mv, *gv, *dz, *dx;
  if ((rc = work_vec(c, 0, nall, &mv)) || (rc = work_vec(c, 1, nall, &gv)) ||
      (rc = work_vec(c, 7, nd, &dz)) || (rc = work_vec(c, 8, nd, &dx)))
    return rc;
  CK(cudaMemcpyAsync(mv, m, nall * 4, cudaMemcpyDefault, c->stream));
  if ((rc = ac_apply(c, shots, n, false, mv, dz, dx, nullptr))) return rc;
  if ((rc = ac_apply(c, shots, n, true, nullptr, dz, dx, gv))) return rc;
  CK(cudaMemcpyAsync(img, gv, nall * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_pair_err(c);
}

}  // extern "C"

namespace {

__global__ void k_scale_f(long long n, float s, float *x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= s;
}

// z = P(g): the U-Net applied to g / rms(g) on the model grid zero-padded to multiples of 8
// (images [allnx][allnz] are the network's [h][w]); z = g without a network.
int precondition(ds2d_ctx *c, ds2d_unet *net, const float *g, float *z) {
  const Dims &d = c->d;
  const size_t nall = (size_t)d.allnx * d.allnz;
  if (!net) {
    CK(cudaMemcpyAsync(z, g, nall * 4, cudaMemcpyDeviceToDevice, c->stream));
    return DS2D_OK;
  }
  const int hp = (d.allnx + 7) / 8 * 8, wp = (d.allnz + 7) / 8 * 8;
  int rc;
  float *xin, *xout;
  if ((rc = work_vec(c, 9, (size_t)hp * wp, &xin)) || (rc = work_vec(c, 10, (size_t)hp * wp, &xout)))
    return rc;
  double gg;
  if ((rc = dot64(c, g, g, (long long)nall, &gg))) return rc;
  if (!(gg > 0)) {
    CK(cudaMemsetAsync(z, 0, nall * 4, c->stream));
    return DS2D_OK;
  }
  CK(cudaMemsetAsync(xin, 0, (size_t)hp * wp * 4, c->stream));
  CK(cudaMemcpy2DAsync(xin, (size_t)wp * 4, g, (size_t)d.allnz * 4, (size_t)d.allnz * 4, d.allnx,
                       cudaMemcpyDeviceToDevice, c->stream));
  k_scale_f<<<4 * 148, 256, 0, c->stream>>>((long long)hp * wp, (float)(1.0 / std::sqrt(gg / nall)), xin);
  c->last_launches++;
  if (ds2d_unet_set_stream(net, c->stream) || ds2d_unet_forward(net, xin, xout, 1, hp, wp))
    return fail(c, DS2D_E_CUDA, "preconditioner: %s", ds2d_unet_last_error(net));
  CK(cudaMemcpy2DAsync(z, (size_t)d.allnz * 4, xout, (size_t)wp * 4, (size_t)d.allnz * 4, d.allnx,
                       cudaMemcpyDeviceToDevice, c->stream));
  return DS2D_OK;
}

}  // namespace

extern "C" {

int ds2d_lsrtm_pcg(ds2d_ctx *c, ds2d_unet *net, const ds2d_shot *shots, int n, const float *obs_vz,
                   const float *obs_vx, int niter, double target, float *m_out, double *resid,
                   double *elapsed_ms, int *iters_done) {
  int rc;
  if ((rc = check_ready(c, false))) return rc;
  if (n <= 0 || !shots || !obs_vz || !obs_vx || !m_out || niter < 0)
    return fail(c, DS2D_E_ARG, "bad arguments");
  if ((rc = ensure_acoustic(c)) || (rc = check_shots(c, shots, n))) return rc;
  c->last_launches = 0;
  c->last_updates = 0;
  const auto t0 = std::chrono::steady_clock::now();
  const size_t nall = (size_t)c->d.allnx * c->d.allnz, nd = (size_t)n * c->d.max_ntr * c->d.nt;
  const int M = std::max(1, std::min(c->opt_pcg_m, 15));
  float *m, *g, *z, *rz, *rx, *wz, *wx;
  if ((rc = work_vec(c, 0, nall, &m)) || (rc = work_vec(c, 1, nall, &g)) ||
      (rc = work_vec(c, 4, nall, &z)) || (rc = work_vec(c, 5, nd, &rz)) ||
      (rc = work_vec(c, 6, nd, &rx)) || (rc = work_vec(c, 7, nd, &wz)) ||
      (rc = work_vec(c, 8, nd, &wx)))
    return rc;
  // direction window: p_j (model space) and q_j = L p_j (data space, two components)
  std::vector<float *> P(M), QZ(M), QX(M);
  std::vector<double> sig(M, 0.0);
  for (int j = 0; j < M; j++)
    if ((rc = work_vec(c, 16 + 3 * j, nall, &P[j])) || (rc = work_vec(c, 17 + 3 * j, nd, &QZ[j])) ||
        (rc = work_vec(c, 18 + 3 * j, nd, &QX[j])))
      return rc;
  CK(cudaMemsetAsync(m, 0, nall * 4, c->stream));
  CK(cudaMemsetAsync(rz, 0, nd * 4, c->stream));
  CK(cudaMemsetAsync(rx, 0, nd * 4, c->stream));
  if ((rc = data_io(c, shots, n, rz, (float *)obs_vz, true)) ||
      (rc = data_io(c, shots, n, rx, (float *)obs_vx, true)))
    return rc;
  // Flexible CG with truncated explicit conjugation (Notay's FCG(M)) on || d - L m ||^2 from
  // m = 0, FP64 scalars.  Each iteration: g = L^T r, z = P(g), w = L z, then z and w are made
  // L^T L-conjugate to the last M directions (z -= beta_j p_j, w -= beta_j q_j with
  // beta_j = <w, q_j> / <q_j, q_j>), and the exact step alpha = <r, q> / <q, q> is taken along
  // p = z, q = w.  With P = I this is CG; with the network the explicit conjugation keeps its
  // directions from undoing one another (an inexact, non-linear P breaks the short recurrence).
  // When an iteration with the network reduces the residual by less than the "pcg_switch"
  // ratio, the network phase ends and the solver continues with P = I and a fresh window.
  double dd, tz, tx;
  if ((rc = dot64(c, rz, rz, nd, &tz)) || (rc = dot64(c, rx, rx, nd, &tx))) return rc;
  dd = tz + tx;
  if (!(dd > 0)) return fail(c, DS2D_E_NUMERIC, "observed data are zero or not finite");
  if ((rc = ac_apply(c, shots, n, true, nullptr, rz, rx, g))) return rc;
  const int nb = 4 * 148;
  int k = 0, nwin = 0, head = 0;  // window: nwin entries, next slot `head`
  double prev_rel = 1.0;
  for (; k < niter; k++) {
    if ((rc = precondition(c, net, g, z))) return rc;
    if ((rc = ac_apply(c, shots, n, false, z, wz, wx, nullptr))) return rc;
    for (int i = 0; i < nwin; i++) {
      const int j = (head - 1 - i + M) % M;
      double bz, bx;
      if ((rc = dot64(c, wz, QZ[j], nd, &bz)) || (rc = dot64(c, wx, QX[j], nd, &bx))) return rc;
      const double beta = (bz + bx) / sig[j];
      k_axpy<<<nb, 256, 0, c->stream>>>((long long)nall, -beta, P[j], z);
      k_axpy<<<nb, 256, 0, c->stream>>>((long long)nd, -beta, QZ[j], wz);
      k_axpy<<<nb, 256, 0, c->stream>>>((long long)nd, -beta, QX[j], wx);
      c->last_launches += 3;
    }
    double rq_z, rq_x;
    if ((rc = dot64(c, wz, wz, nd, &tz)) || (rc = dot64(c, wx, wx, nd, &tx)) ||
        (rc = dot64(c, rz, wz, nd, &rq_z)) || (rc = dot64(c, rx, wx, nd, &rq_x)))
      return rc;
    const double qq = tz + tx;
    if (!(qq > 0) || !std::isfinite(rq_z + rq_x))
      return fail(c, DS2D_E_NUMERIC, "PCG breakdown at %d", k);
    const double alpha = (rq_z + rq_x) / qq;
    k_axpy<<<nb, 256, 0, c->stream>>>((long long)nall, alpha, z, m);
    k_axpy<<<nb, 256, 0, c->stream>>>((long long)nd, -alpha, wz, rz);
    k_axpy<<<nb, 256, 0, c->stream>>>((long long)nd, -alpha, wx, rx);
    c->last_launches += 3;
    // keep (p, q) = (z, w) in the window
    CK(cudaMemcpyAsync(P[head], z, nall * 4, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(QZ[head], wz, nd * 4, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(QX[head], wx, nd * 4, cudaMemcpyDeviceToDevice, c->stream));
    sig[head] = qq;
    head = (head + 1) % M;
    nwin = std::min(nwin + 1, M);
    if ((rc = dot64(c, rz, rz, nd, &tz)) || (rc = dot64(c, rx, rx, nd, &tx))) return rc;
    const double rel = std::sqrt((tz + tx) / dd);
    if (resid) resid[k] = rel;
    if (elapsed_ms)
      elapsed_ms[k] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (rel <= target || k + 1 == niter) {
      k++;
      break;
    }
    if (net && c->opt_pcg_switch > 0 && rel > prev_rel * (c->opt_pcg_switch / 1000.0)) {
      net = nullptr;  // network phase over: plain CG from the current iterate
      nwin = 0;
    }
    prev_rel = rel;
    if ((rc = ac_apply(c, shots, n, true, nullptr, rz, rx, g))) return rc;
  }
  if (iters_done) *iters_done = k;
  CK(cudaMemcpyAsync(m_out, m, nall * 4, cudaMemcpyDefault, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_pair_err(c);
}

int ds2d_dot_f64(ds2d_ctx *c, const float *a, const float *b, long long n, double *result) {
  if (!c || !a || !b || !result || n < 0) return DS2D_E_ARG;
  if (!c->dot_part) {
    int rc;
    if ((rc = alloc(c, (void **)&c->dot_part, sizeof(double) * kDotBlocks))) return rc;
    if ((rc = alloc(c, (void **)&c->dot_out, sizeof(double)))) return rc;
  }
  return dot64(c, a, b, n, result);
}

int ds2d_set_option(ds2d_ctx *c, const char *key, long long value) {
  if (!c || !key) return DS2D_E_ARG;
  std::string k(key);
  if (k == "fused") {
    c->opt_fused = value != 0;
  } else if (k == "adjoint_born") {
    c->opt_adjoint_born = value != 0;
  } else if (k == "graph") {
    c->opt_graph = value != 0;
  } else if (k == "ring") {
    if (value == 1) value = kDefaultRing;
    if (value != 0 && value != 2 && value != 4 && value != 8)
      return fail(c, DS2D_E_ARG, "ring must be 0 (off), 1 (default depth) or a depth of 2, 4 or 8");
    c->opt_ring = (int)value;
  } else if (k == "pcg_m") {
    if (value < 1 || value > 15) return fail(c, DS2D_E_ARG, "pcg_m must be in [1, 15]");
    c->opt_pcg_m = (int)value;
  } else if (k == "pcg_switch") {
    if (value < 0 || value > 1000) return fail(c, DS2D_E_ARG, "pcg_switch must be in [0, 1000]");
    c->opt_pcg_switch = (int)value;
  } else if (k == "occ") {
    if (value != 0 && value != 1) return fail(c, DS2D_E_ARG, "occ must be 0 or 1");
    c->opt_occ = (int)value;
  } else if (k == "cta") {
    if (value != 0 && value != kFB && value != kWideCta)
      return fail(c, DS2D_E_ARG, "cta must be 0 (automatic), 128 or 192");
    c->opt_cta = (int)value;
  } else if (k == "pair") {
    if (value < 0 || value > 2)
      return fail(c, DS2D_E_ARG, "pair must be 0, 1 (forward and backward) or 2 (forward only)");
    c->opt_pair = (int)value;
  } else if (k == "pair_cta") {
    if (value != 0 && value != 64 && value != 160 && value != 256)
      return fail(c, DS2D_E_ARG, "pair_cta must be 0 (automatic), 64, 160 or 256");
    c->opt_pair_cta = (int)value;
  } else if (k == "ac_ckpt") {
    if (value < 0 || value > (1 << 30)) return fail(c, DS2D_E_ARG, "ac_ckpt must be >= 0");
    c->opt_ac_ckpt = (int)value;
  } else if (k == "ac_pair") {
    if (value != 0 && value != 1) return fail(c, DS2D_E_ARG, "ac_pair must be 0 or 1");
    c->opt_ac_pair = (int)value;
  } else if (k == "ac_pair_cta") {
    if (value != 0 && value != 128 && value != 192 && value != 256)
      return fail(c, DS2D_E_ARG, "ac_pair_cta must be 0 (automatic), 128, 192 or 256");
    c->opt_ac_pair_cta = (int)value;
  } else if (k == "pair_split") {
    if (value != 0 && value != 1) return fail(c, DS2D_E_ARG, "pair_split must be 0 or 1");
    c->opt_pair_split = (int)value;
  } else if (k == "pair_fcta") {
    if (value != 0 && value != 64 && value != 256)
      return fail(c, DS2D_E_ARG, "pair_fcta must be 0 (automatic), 64 or 256");
    c->opt_pair_fcta = (int)value;
  } else if (k == "pair_xr") {
    if (value != 0 && (value < 8 || value > 4096))
      return fail(c, DS2D_E_ARG, "pair_xr must be 0 (automatic) or in [8, 4096]");
    c->opt_pair_xr = (int)value;
  } else if (k == "tb") {
    if (value < 0 || value > 4) return fail(c, DS2D_E_ARG, "tb must be 0 (off) or 1-4");
    c->opt_tb = (int)value;
  } else if (k == "bwd_bulk") {
    if (value != 0 && value != 1) return fail(c, DS2D_E_ARG, "bwd_bulk must be 0 or 1");
    c->opt_bwd_bulk = (int)value;
  } else if (k == "bwd_cta") {
    if (value != 0 && value != 128 && value != 192 && value != 256)
      return fail(c, DS2D_E_ARG, "bwd_cta must be 0 (automatic), 128, 192 or 256");
    c->opt_bwd_cta = (int)value;
  } else if (k == "bwd_1b") {
    if (value != 0 && value != 1) return fail(c, DS2D_E_ARG, "bwd_1b must be 0 or 1");
    c->opt_bwd_1b = (int)value;
  } else if (k == "bwd_ws") {
    if (value != 0 && value != 96 && value != 128 && value != 192)
      return fail(c, DS2D_E_ARG, "bwd_ws must be 0 (off) or 96, 128, 192 threads per role");
    c->opt_bwd_ws = (int)value;
  } else if (k == "tb_bulk") {
    if (value != 0 && value != 1) return fail(c, DS2D_E_ARG, "tb_bulk must be 0 or 1");
    c->opt_tb_bulk = (int)value;
  } else if (k == "tb_cta") {
    if (value != 0 && value != 256 && value != 512)
      return fail(c, DS2D_E_ARG, "tb_cta must be 0 (automatic), 256 or 512 (depth 1-2)");
    c->opt_tb_cta = (int)value;
  } else if (k == "xr") {
    if (value < 8 || value > 4096) return fail(c, DS2D_E_ARG, "xr must be in [8, 4096]");
    c->opt_xr = (int)value;
  } else {
    return fail(c, DS2D_E_ARG, "unknown option '%s'", key);
  }
  return DS2D_OK;
}

int ds2d_profile(ds2d_ctx *c, int enable) {
  if (!c) return DS2D_E_ARG;
  CK(cudaStreamSynchronize(c->stream));
  c->prof.on = enable != 0;
  c->prof.recs.clear();
  c->prof.used = 0;
  return DS2D_OK;
}

int ds2d_profile_report(ds2d_ctx *c, char *buf, int len) {
  if (!c || !buf || len <= 0) return DS2D_E_ARG;
  CK(cudaStreamSynchronize(c->stream));
  struct Agg {
    std::string name;
    long long n = 0;
    double ms = 0, bytes = 0;
  };
  std::vector<Agg> agg;
  for (const ProfRec &r : c->prof.recs) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->prof.pool[r.ev], c->prof.pool[r.ev + 1]));
    Agg *a = nullptr;
    for (Agg &x : agg)
      if (x.name == r.name) a = &x;
    if (!a) {
      agg.push_back(Agg{r.name});
      a = &agg.back();
    }
    a->n++;
    a->ms += ms;
    a->bytes += r.bytes;
  }
  std::string out;
  for (const Agg &a : agg) {
    char line[256];
    snprintf(line, sizeof line, "%s %lld %.6f %.6e\n", a.name.c_str(), a.n, a.ms, a.bytes);
    out += line;
  }
  snprintf(buf, len, "%s", out.c_str());
  c->prof.recs.clear();
  c->prof.used = 0;
  return (int)out.size() < len ? DS2D_OK : DS2D_E_ARG;
}

double ds2d_last_cell_updates(const ds2d_ctx *c) { return c ? c->last_updates : 0.0; }
long long ds2d_last_launches(const ds2d_ctx *c) { return c ? c->last_launches : 0; }

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// FP64 inner product that allocates nothing.
//
// ds2d_dot_f64 keeps its per-block partial sums in scratch that the context allocates on first
// use, and a context itself allocates the whole wavefield arena when it is created.  Some
// callers cannot allocate device memory at the moment they need a dot product:
//  - a host framework that owns the device memory budget and hands libraries only the buffers
//    they work on (a pool that is already at its limit, or a policy that forbids a library
//    from calling cudaMalloc behind its back);
//  - a caller that has no ds2d context at all (a CG or convergence check on the host
//    application's own vectors), for which creating one would allocate hundreds of MB;
//  - a caller running when the HBM is full, e.g. between batches that sized the arena to what
//    was left, where any new allocation fails with out-of-memory.
// For them the scratch lives in this module's static device memory: the CUDA runtime reserves
// it when it loads the module, so a call makes no allocation.  The price is that the scratch is
// shared by every call on a device: calls on the same device that overlap in time (two host
// threads, or two streams whose work runs concurrently) race on it and return wrong sums.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int kNaPerThread = 64;                               // elements per thread
constexpr long long kNaChunk = (long long)kDotThreads * kNaPerThread;  // 16384 per block
constexpr int kNaMaxPartials = 32768;                          // 256 KiB of partial sums
constexpr long long kNaMaxElems = kNaChunk * kNaMaxPartials;   // 2^29 = 536,870,912 elements
constexpr int kNaMaxDevices = 64;

// Partial sums [0, kNaMaxPartials) and the result slot [kNaMaxPartials].  Nothing here has to
// start at zero: a call writes every partial it later reads, and the result before reading it.
static __device__ __align__(256) double g_na_scratch[kNaMaxPartials + 1];

// Same per-block reduction as k_dot_partial, but each block owns one contiguous chunk of
// kNaChunk elements instead of a grid stride, so the block count (and the scratch a call needs)
// follows n and is bounded by the static array.
__global__ void __launch_bounds__(kDotThreads) k_dot_chunk(const float *a, const float *b,
                                                           long long n, double *partial) {
  __shared__ double sh[kDotThreads / 32];
  const long long lo = (long long)blockIdx.x * kNaChunk;
  const long long hi = lo + kNaChunk < n ? lo + kNaChunk : n;
  double acc = 0.0;
  for (long long i = lo + threadIdx.x; i < hi; i += kDotThreads)
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

std::mutex g_na_mu;
struct NaSlot {
  CUcontext ctx;  // context the address below belongs to
  double *ptr;
};
NaSlot g_na_slot[kNaMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry point (no link against libcuda).
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CtxGetCurrentFn na_ctx_fn() {
  static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// Device address of g_na_scratch in the current context.  It is looked up (with the device
// current, as cudaGetSymbolAddress requires) on the first call in a context and cached per
// device together with the context it belongs to; a call from another context of the same
// device (a non-primary context, or the primary context re-created after cudaDeviceReset under
// a new handle) looks it up again.  The first call in a context may load this module there, so
// it should come before any stream capture on that device.
int na_scratch(double **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_create_err = std::string("ds2d_dot_f64_noalloc: cudaGetDevice: ") + cudaGetErrorString(e);
    return DS2D_E_CUDA;
  }
  if (dev < 0 || dev >= kNaMaxDevices) {
    g_create_err = "ds2d_dot_f64_noalloc: device ordinal " + std::to_string(dev) +
                   " is beyond the table of " + std::to_string(kNaMaxDevices) + " devices";
    return DS2D_E_ARG;
  }
  // cudaFree(0) makes the runtime bind (or create) the device's primary context when the
  // calling thread has none yet; it allocates nothing.
  CUcontext ctx = nullptr;
  CtxGetCurrentFn get = na_ctx_fn();
  if (get && get(&ctx) == CUDA_SUCCESS && !ctx && cudaFree(nullptr) == cudaSuccess) get(&ctx);
  std::lock_guard<std::mutex> lock(g_na_mu);
  NaSlot &slot = g_na_slot[dev];
  if (!slot.ptr || slot.ctx != ctx || !ctx) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p) {
      g_create_err = std::string("ds2d_dot_f64_noalloc: cudaGetSymbolAddress: ") +
                     cudaGetErrorString(e);
      slot = NaSlot{};
      return DS2D_E_CUDA;
    }
    slot = NaSlot{ctx, static_cast<double *>(p)};
  }
  *out = slot.ptr;
  return DS2D_OK;
}

}  // namespace

extern "C" int ds2d_dot_f64_noalloc(const float *a, const float *b, long long n, void *stream,
                                    double *result) {
  if (!a || !b || !result || n < 0) {
    g_create_err = "ds2d_dot_f64_noalloc: null vector/result pointer or negative length";
    return DS2D_E_ARG;
  }
  if (n > kNaMaxElems) {
    g_create_err = "ds2d_dot_f64_noalloc: n = " + std::to_string(n) +
                   " exceeds the static scratch limit of " + std::to_string(kNaMaxElems) +
                   " elements (" + std::to_string(kNaMaxPartials) + " partial sums of " +
                   std::to_string(kNaChunk) + " elements); use ds2d_dot_f64";
    return DS2D_E_ARG;
  }
  double *scratch = nullptr;
  int rc = na_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = n == 0 ? 1 : (int)((n + kNaChunk - 1) / kNaChunk);
  k_dot_chunk<<<nb, kDotThreads, 0, st>>>(a, b, n, scratch);
  k_dot_final<<<1, 32, 0, st>>>(scratch, nb, scratch + kNaMaxPartials);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(result, scratch + kNaMaxPartials, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    g_create_err = std::string("ds2d_dot_f64_noalloc: ") + cudaGetErrorString(e);
    return DS2D_E_CUDA;
  }
  return DS2D_OK;
}

// ---------------------------------------------------------------------------------------------
// Gradient band-pass filter (reference bandpass_filter, FD2DGPU.cu:4125-4182; see
// ds2d_filter.cuh for the arithmetic it reproduces).
namespace {

struct BandpassScratch {
  double2 *wz = nullptr, *wzi = nullptr, *wx = nullptr, *wxi = nullptr, *t1 = nullptr,
          *t2 = nullptr;
  float *filt = nullptr;
  std::vector<void *> all;
  ~BandpassScratch() {
    for (void *p : all) cudaFree(p);
  }
  cudaError_t get(void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) all.push_back(*p);
    return e;
  }
};

int bandpass_images(int nx, int nz, int z1, int z2, float *const imgs[2], cudaStream_t st) {
  auto err = [&](const char *what, cudaError_t e) {
    g_create_err = std::string("ds2d_bandpass_filter: ") + what + ": " + cudaGetErrorString(e);
    return DS2D_E_CUDA;
  };
  BandpassScratch sc;
  const size_t ncell = (size_t)nx * nz;
  cudaError_t e = cudaSuccess;
  if ((e = sc.get((void **)&sc.wz, sizeof(double2) * nz * nz)) ||
      (e = sc.get((void **)&sc.wzi, sizeof(double2) * nz * nz)) ||
      (e = sc.get((void **)&sc.wx, sizeof(double2) * nx * nx)) ||
      (e = sc.get((void **)&sc.wxi, sizeof(double2) * nx * nx)) ||
      (e = sc.get((void **)&sc.t1, sizeof(double2) * ncell)) ||
      (e = sc.get((void **)&sc.t2, sizeof(double2) * ncell)) ||
      (e = sc.get((void **)&sc.filt, sizeof(float) * ncell)))
    return err("cudaMalloc", e);
  // filter in natural frequency order: k'(j) = k(S(j))
  const std::vector<float> k = gaussian_bandpass(nx, nz, z1, z2);
  std::vector<float> kp(ncell);
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) kp[(size_t)ix * nz + iz] = k[quadrant_swap(nx, nz, ix, iz)];
  const std::vector<double2> wz = dft_matrix(nz, -1), wzi = dft_matrix(nz, 1);
  const std::vector<double2> wx = dft_matrix(nx, -1), wxi = dft_matrix(nx, 1);
  if ((e = cudaMemcpyAsync(sc.wz, wz.data(), sizeof(double2) * wz.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(sc.wzi, wzi.data(), sizeof(double2) * wzi.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(sc.wx, wx.data(), sizeof(double2) * wx.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(sc.wxi, wxi.data(), sizeof(double2) * wxi.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(sc.filt, kp.data(), sizeof(float) * ncell, cudaMemcpyHostToDevice, st)))
    return err("cudaMemcpyAsync", e);
  auto gemm = [&](DftArgs a) {
    dim3 grid((a.N + kDftTile - 1) / kDftTile, (a.M + kDftTile - 1) / kDftTile);
    k_dft_gemm<<<grid, kDftTile * kDftTile, 0, st>>>(a);
  };
  for (int i = 0; i < 2; i++) {
    if (!imgs[i]) continue;
    DftArgs a{};
    // forward along z: t1[x][kz] = sum_z f[x][z] Wz[z][kz]
    a = DftArgs{};
    a.M = nx; a.N = nz; a.K = nz; a.a_real = imgs[i]; a.lda = nz; a.b = sc.wz; a.ldb = nz;
    a.c = sc.t1; a.ldc = nz;
    gemm(a);
    // forward along x, times (k', k'): t2[kx][kz] = (k', k') * sum_x Wx[kx][x] t1[x][kz]
    a = DftArgs{};
    a.M = nx; a.N = nz; a.K = nx; a.a = sc.wx; a.lda = nx; a.b = sc.t1; a.ldb = nz;
    a.c = sc.t2; a.ldc = nz; a.filt = sc.filt; a.ldf = nz;
    gemm(a);
    // inverse along x: t1[x][kz] = sum_kx Wx*[x][kx] t2[kx][kz]
    a = DftArgs{};
    a.M = nx; a.N = nz; a.K = nx; a.a = sc.wxi; a.lda = nx; a.b = sc.t2; a.ldb = nz;
    a.c = sc.t1; a.ldc = nz;
    gemm(a);
    // inverse along z, real part / (nx nz) into the image
    a = DftArgs{};
    a.M = nx; a.N = nz; a.K = nz; a.a = sc.t1; a.lda = nz; a.b = sc.wzi; a.ldb = nz;
    a.out_real = imgs[i]; a.ldo = nz; a.scale = (double)(nx * nz);
    gemm(a);
  }
  if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(st))) return err("launch", e);
  return DS2D_OK;
}

int bandpass_check(int nx, int nz, int z1, int z2) {
  if (nx < 2 || nz < 2 || z2 <= 0 || z1 < 0) {
    g_create_err = "ds2d_bandpass_filter: need nx, nz >= 2, high cut-off z2 > 0, low cut-off z1 >= 0";
    return DS2D_E_ARG;
  }
  return DS2D_OK;
}

}  // namespace

extern "C" int ds2d_bandpass_filter_device(int nx, int nz, int x1, int x2, int z1, int z2,
                                           float *grad_pp, float *grad_ps, void *stream) {
  (void)x1;
  (void)x2;  // accepted for the reference's signature; its live filter uses z1, z2 only
  int rc = bandpass_check(nx, nz, z1, z2);
  if (rc) return rc;
  float *imgs[2] = {grad_pp, grad_ps};
  return bandpass_images(nx, nz, z1, z2, imgs, static_cast<cudaStream_t>(stream));
}

extern "C" int ds2d_bandpass_filter(int nx, int nz, int x1, int x2, int z1, int z2,
                                    float *grad_pp, float *grad_ps) {
  int rc = bandpass_check(nx, nz, z1, z2);
  if (rc) return rc;
  const size_t bytes = sizeof(float) * (size_t)nx * nz;
  float *d[2] = {nullptr, nullptr};
  float *h[2] = {grad_pp, grad_ps};
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 2 && e == cudaSuccess; i++)
    if (h[i] && (e = cudaMalloc(&d[i], bytes)) == cudaSuccess)
      e = cudaMemcpy(d[i], h[i], bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = bandpass_images(nx, nz, z1, z2, d, nullptr);
    for (int i = 0; i < 2 && rc == DS2D_OK && e == cudaSuccess; i++)
      if (h[i]) e = cudaMemcpy(h[i], d[i], bytes, cudaMemcpyDeviceToHost);
  }
  for (float *p : d)
    if (p) cudaFree(p);
  if (e != cudaSuccess) {
    g_create_err = std::string("ds2d_bandpass_filter: ") + cudaGetErrorString(e);
    return DS2D_E_CUDA;
  }
  return rc;
}
