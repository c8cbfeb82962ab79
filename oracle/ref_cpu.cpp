// The reference's own CPU acoustic stepper -- TEST INFRASTRUCTURE ONLY (the acoustic CPU
// baseline of the benchmark).  main.cpp is compiled where it lies in the reference tree (included
// here with its main renamed, against the stub oracle/stub/mpi.h; nothing is copied) and its
// staggered_grid_extrapolation_2d_pml (main.cpp:602-727, OpenMP, 8th order, PML) is driven for
// nt steps.  The reference never calls the stepper itself, so the driver below supplies the
// explosive source at (isx, isz) before every step, half into each split part px, pz (the stepper
// recomputes p = px + pz from them, so a source added to p alone would be lost).
#define main ref_main
#include "main.cpp"
#undef main

#include <chrono>

extern "C" int ref_cpu_acoustic(int nxpml, int nzpml, int nt, float dt, float dx, float dz,
                                const float *vp, const float *rho, const float *damp, int isx,
                                int isz, const float *wavelet, float *p_out, double *seconds) {
  float **p = alloc2float(nzpml, nxpml), **px = alloc2float(nzpml, nxpml);
  float **pz = alloc2float(nzpml, nxpml), **vx = alloc2float(nzpml, nxpml);
  float **vz = alloc2float(nzpml, nxpml), **dmp = alloc2float(nzpml, nxpml);
  float **rh = alloc2float(nzpml, nxpml), **k = alloc2float(nzpml, nxpml);
  for (int ix = 0; ix < nxpml; ix++)
    for (int iz = 0; iz < nzpml; iz++) {
      const size_t q = (size_t)ix * nzpml + iz;
      p[ix][iz] = px[ix][iz] = pz[ix][iz] = vx[ix][iz] = vz[ix][iz] = 0.f;
      dmp[ix][iz] = damp[q];
      rh[ix][iz] = rho[q];
      k[ix][iz] = rho[q] * vp[q] * vp[q];
    }
  const auto t0 = std::chrono::steady_clock::now();
  for (int it = 0; it < nt; it++) {
    px[isx][isz] += 0.5f * wavelet[it];
    pz[isx][isz] += 0.5f * wavelet[it];
    staggered_grid_extrapolation_2d_pml(p, px, pz, vx, vz, dmp, rh, k, dt, nzpml, nxpml, dz, dx,
                                        8);
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (p_out)
    for (int ix = 0; ix < nxpml; ix++)
      for (int iz = 0; iz < nzpml; iz++) p_out[(size_t)ix * nzpml + iz] = p[ix][iz];
  for (float **a : {p, px, pz, vx, vz, dmp, rh, k}) free2float(a);
  return 0;
}
