// Gradient band-pass filter (reference bandpass_filter, FD2DGPU.cu:4125-4182, with the Gaussian
// filter of construct_gaussian_bandpass_filter, FD2DGPU.cu:4038-4077, as the reference calls it
// at :4135).  Off the time-stepping path: the reference applies it, when enabled, once per LSRTM
// iteration to the summed gradients (main.cpp:1074-1089, commented out in the shipped loop).
//
// What the reference computes for one image f [nx][nz] (z fastest):
//   F = FFT2(f) in double complex (cuFFT Z2Z, unnormalised), quadrant swap S, multiply every
//   element by the complex number (k, k) (GPU_lowpass builds make_cuDoubleComplex(k, k), not
//   (k, 0)), quadrant swap S again, inverse FFT2, divide by nx*nz, keep the real part.
// S exchanges quadrant (y, x) with (y + nx/2, x + nz/2) and (y, x + nz/2) with (y + nx/2, x) for
// y < nx/2, x < nz/2 (fft_shift / ifft_shift); for odd sizes the last row / column stay put.  S is
// an involution and the multiply is elementwise, so S (k F) S-swapped equals k(S(j)) F(j): the
// filter simply acts in natural frequency order as k' = k o S.  The result is therefore
//   out = Re(IFFT2((1 + i) k' F)) / (nx nz) = (Re g - Im g) / (nx nz),  g = IFFT2(k' F).
//
// Here the two 2D transforms are four dense complex DFT products in FP64 (along z, along x, the
// filter fused into the second, inverse along x, inverse along z) on shared-memory tiles: exact
// for any size (the benchmark grids are odd, 1201 x 401), no library FFT, and a few milliseconds
// per image on a B200, against the seconds of an RTM step the filter follows.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

namespace ds2d {

constexpr int kDftTile = 16;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ void cmac(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}

// Operand / result access of one DFT product C[m][n] = sum_k A[m][k] B[k][n].
struct DftArgs {
  int M, N, K;
  // A: real float [M][K] (lda), or complex [M][K] (lda); B: complex [K][N] (ldb)
  const float *a_real;
  const double2 *a, *b;
  long long lda, ldb;
  // epilogue: complex C [M][N] (ldc), optionally times (k, k) with k = filt[m][n] (ldf);
  // or the real part of C / scale as float into out_real [M][N] (ldo)
  double2 *c;
  long long ldc;
  const float *filt;
  long long ldf;
  float *out_real;
  long long ldo;
  double scale;
};

__global__ void __launch_bounds__(kDftTile *kDftTile) k_dft_gemm(DftArgs p) {
  __shared__ double2 As[kDftTile][kDftTile + 1], Bs[kDftTile][kDftTile + 1];
  const int tx = threadIdx.x % kDftTile, ty = threadIdx.x / kDftTile;
  const int m = blockIdx.y * kDftTile + ty, n = blockIdx.x * kDftTile + tx;
  double2 acc = make_double2(0.0, 0.0);
  for (int k0 = 0; k0 < p.K; k0 += kDftTile) {
    const int ka = k0 + tx, kb = k0 + ty;
    double2 av = make_double2(0.0, 0.0), bv = make_double2(0.0, 0.0);
    if (m < p.M && ka < p.K)
      av = p.a_real ? make_double2((double)p.a_real[(long long)m * p.lda + ka], 0.0)
                    : p.a[(long long)m * p.lda + ka];
    if (kb < p.K && n < p.N) bv = p.b[(long long)kb * p.ldb + n];
    As[ty][tx] = av;
    Bs[ty][tx] = bv;
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kDftTile; kk++) cmac(acc, As[ty][kk], Bs[kk][tx]);
    __syncthreads();
  }
  if (m >= p.M || n >= p.N) return;
  if (p.out_real) {  // GPU_divide then Z2R: real part / (nx nz), as float
    p.out_real[(long long)m * p.ldo + n] = (float)(acc.x / p.scale);
    return;
  }
  if (p.filt) {
    const double k = (double)p.filt[(long long)m * p.ldf + n];
    acc = cmul(acc, make_double2(k, k));
  }
  p.c[(long long)m * p.ldc + n] = acc;
}

// Host side -----------------------------------------------------------------------------------

// construct_gaussian_bandpass_filter(filter, width = nz, height = nx, low, high) in the
// reference's own arithmetic (FD2DGPU.cu:4038-4077): float distance, double exponentials stored
// as float, negative values clamped to 0, normalised to a maximum of 1; low == 0 gives the
// low-pass form.  Indexed [ix][iz] like the images.
inline std::vector<float> gaussian_bandpass(int nx, int nz, int low, int high) {
  std::vector<float> f((size_t)nx * nz);
  const int cx = nz / 2, cy = nx / 2;
  float maxv = 0.0f;
  for (int y = 0; y < nx; y++)
    for (int x = 0; x < nz; x++) {
      const int dx = x - cx, dy = y - cy;
      const float scale = float(nz) / nx;
      const float dist = std::sqrt((float)(dx * dx) + (scale * dy) * (scale * dy));
      const float d2 = -dist * dist;
      float g;
      if (low == 0)
        g = (float)std::exp(d2 / (2.0 * high * high));
      else
        g = (float)(std::exp(d2 / (2.0 * high * high)) - std::exp(d2 / (2.0 * low * low)));
      if (g < 0) g = 0;
      f[(size_t)y * nz + x] = g;
      if (g > maxv) maxv = g;
    }
  for (float &v : f) v /= maxv;
  return f;
}

// The quadrant swap S of fft_shift / ifft_shift (FD2DGPU.cu:3922-3965) as an index map on
// [ix][iz] (an involution; for odd sizes the last row and column map to themselves).
inline size_t quadrant_swap(int nx, int nz, int ix, int iz) {
  const int hx = nx / 2, hz = nz / 2;
  if (ix < 2 * hx && iz < 2 * hz) {
    const int jx = ix < hx ? ix + hx : ix - hx;
    const int jz = iz < hz ? iz + hz : iz - hz;
    return (size_t)jx * nz + jz;
  }
  return (size_t)ix * nz + iz;
}

// DFT matrix W[j][k] = exp(sign 2 pi i (j k mod n) / n) in FP64.
inline std::vector<double2> dft_matrix(int n, int sign) {
  std::vector<double2> w((size_t)n * n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int j = 0; j < n; j++)
    for (int k = 0; k < n; k++) {
      const long long m = ((long long)j * k) % n;
      const double a = sign * two_pi * (double)m / n;
      w[(size_t)j * n + k] = make_double2(std::cos(a), std::sin(a));
    }
  return w;
}

}  // namespace ds2d
