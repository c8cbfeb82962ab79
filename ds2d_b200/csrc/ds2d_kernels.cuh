// Device side of the B200 DS2D time-stepping path: data layout, stencil helpers, kernels.
//
// Data layout in HBM (one "slot" per resident shot, all slots of a batch in one allocation):
//   field / parameter arrays  [slot][nxpml][ld], ld = nzpml rounded up to 32 floats (128-byte
//   rows, z fastest: the reference's idx = ix*nzpml + iz with a padded row), slot stride
//   nxpml*ld floats.
// PML split memory variables are touched only where the reference's damping is non-zero (the
// geometric PML of dampX/dampZ, FD2DGPU.cu:444-494); interior cells carry the unsplit sums,
// which is the reference's split update with damp1 = damp2 = 1.  Additive injections
// (explosive source FD2DGPU.cu:2039, Born sources born.cu:351 / born.cu:408, receiver-side
// residual FD2DGPU.cu:3306, strip reloads FD2DGPU.cu:3705) are applied as read overlays: the
// reference adds them to the summed array, which its next split update recomputes from the
// split variables, so each acts on exactly one stencil evaluation and never enters the state.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace ds2d {

// FD2DGPU.cuh:16 coeff2: double expressions stored as float.
constexpr float kC1 = (float)(1225.0 / 1024.0);
constexpr float kC2 = (float)(-245.0 / 3072.0);
constexpr float kC3 = (float)(49.0 / 5120.0);
constexpr float kC4 = (float)(-5.0 / 7168.0);

// Grid of a batch.  nxp / wnx / lb / nseg describe ONE slot (kernels narrow them to the slot's
// own window with slot_dims); the *_max fields are the allocation strides shared by all slots.
struct Dims {
  int nxp, nzp, ld;  // padded window, leading dimension
  int pml, nop;
  int wnx, wnz;      // interior window (reference nx, nz)
  int ild;           // row stride of the per-slot window images [slot][wnx][ild]; window
                     // column iz - pml sits at iz, so rows align like the wavefield rows
  int nt;
  int allnx, allnz;
  long long slot;    // floats per slot of one array (nxp_max * ld)
  float dx, dz, dt;
  int rbc;           // random boundary: no PML cells, no strips
  int lb;            // strip band cells per component per step
  int nseg;          // 32-cell scale segments per component per step
  int max_ntr;
  int nxp_max, wnx_max, lb_max, nseg_max;  // strides
};

struct ShotDev {
  int win_left, isx, isz, igz, ntr, nxp, wnx, lb;
};

__host__ __device__ __forceinline__ Dims slot_dims(const Dims &d, const ShotDev &sh) {
  Dims r = d;
  r.nxp = sh.nxp;
  r.wnx = sh.wnx;
  r.lb = sh.lb;
  r.nseg = (sh.lb + 31) / 32;
  return r;
}

// One wavefield set (base pointers of slot 0).  Split arrays are null without a PML.
struct Wave {
  float *vx, *vz, *txx, *tzz, *txz;
  float *vx_x, *vx_z, *vz_x, *vz_z, *txx_x, *txx_z, *tzz_x, *tzz_z, *txz_x, *txz_z;
};

struct Strain {
  float *gx_vx, *gz_vz, *gz_vx, *gx_vz;  // reference vx_gx, vz_gz, vx_gz, vz_gx
};

struct Par {
  const float *b, *lam, *mu, *dampx, *dampz, *kpp, *kps, *dmp, *dms;
};

// Saved boundary strips of one wavefield set: [slot][it][component][lb] elements in `prec`
// (0 fp32, 1 fp16, 2 bf16) and, for the 16-bit formats, one fp32 scale per
// [slot][it][component][32-element segment].
struct Strips {
  void *data;
  float *scale;
  int prec;
};

// Kernel families: forward (born.cu:215-349), interior reconstruction (FD2DGPU.cu:903-1082)
// and adjoint (FD2DGPU.cu:591-895).
enum Mode { kFwd = 0, kRev = 1, kAdj = 2 };

template <class F>
__device__ __forceinline__ float stencil4(F f) {
  float t = kC1 * f(1);
  t = fmaf(kC2, f(2), t);
  t = fmaf(kC3, f(3), t);
  t = fmaf(kC4, f(4), t);
  return t;
}

__device__ __forceinline__ bool pml_cell(const Dims &d, int ix, int iz) {
  return !d.rbc && (ix < d.pml || ix > d.nxp - d.pml || iz < d.pml || iz > d.nzp - d.pml);
}

// Offset of (ix, iz) inside the band vector of one step, or -1 (geometry of the 2-field
// record_edge_wavefield, FD2DGPU.cu:3674-3700: up / down bands 2N wide in z over the interior
// columns, then left / right bands 2N wide in x over the interior rows).
__device__ __forceinline__ int band_offset(const Dims &d, int ix, int iz) {
  const int N = d.nop, pml = d.pml;
  if (ix >= pml && ix < d.nxp - pml) {
    if (iz >= pml - N && iz < pml + N) return (ix - pml) * 2 * N + (iz - (pml - N));
    if (iz >= d.nzp - pml - N && iz < d.nzp - pml + N)
      return d.wnx * 2 * N + (ix - pml) * 2 * N + (iz - (d.nzp - pml - N));
  }
  if (iz >= pml && iz < d.nzp - pml) {
    if (ix >= pml - N && ix < pml + N)
      return 4 * N * d.wnx + (ix - (pml - N)) * d.wnz + (iz - pml);
    if (ix >= d.nxp - pml - N && ix < d.nxp - pml + N)
      return 4 * N * d.wnx + 2 * N * d.wnz + (ix - (d.nxp - pml - N)) * d.wnz + (iz - pml);
  }
  return -1;
}

// Inverse of band_offset.
__device__ __forceinline__ void band_cell(const Dims &d, int bo, int &ix, int &iz) {
  const int N = d.nop, pml = d.pml, ud = 2 * N * d.wnx;
  if (bo < ud) {
    ix = pml + bo / (2 * N);
    iz = pml - N + bo % (2 * N);
  } else if (bo < 2 * ud) {
    int b = bo - ud;
    ix = pml + b / (2 * N);
    iz = d.nzp - pml - N + b % (2 * N);
  } else if (bo < 2 * ud + 2 * N * d.wnz) {
    int b = bo - 2 * ud;
    ix = pml - N + b / d.wnz;
    iz = pml + b % d.wnz;
  } else {
    int b = bo - 2 * ud - 2 * N * d.wnz;
    ix = d.nxp - pml - N + b / d.wnz;
    iz = pml + b % d.wnz;
  }
}

__device__ __forceinline__ float strip_get(const Strips &st, const Dims &d, int s, int it,
                                           int comp, int bo) {
  long long row = ((long long)s * d.nt + it) * 2 + comp;
  long long e = row * d.lb_max + bo;
  if (st.prec == 0) return ((const float *)st.data)[e];
  float sc = st.scale[row * d.nseg_max + (bo >> 5)];
  if (st.prec == 1) return __half2float(((const __half *)st.data)[e]) * sc;
  return __bfloat162float(((const __nv_bfloat16 *)st.data)[e]) * sc;
}

}  // namespace ds2d
