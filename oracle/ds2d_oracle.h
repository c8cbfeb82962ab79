/*
 * CPU oracle for the DS2D time-stepping path -- TEST INFRASTRUCTURE ONLY.
 *
 * A line-by-line restatement, on the host, of the reference's elastic staggered-grid scheme
 * (born.cu, FD2DGPU.cu, main.cpp of 285639863/DS2D).  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference legs may load it, and only as the checker.
 *
 * Every entry point exists in two precisions: *_f64 (ground truth) and *_f32 (the same code in
 * float, which also serves as the timed CPU baseline).  Inputs are float (the same arrays the
 * GPU path receives); outputs are double.
 *
 * Parity pin: the restatement is checked against outputs of the reference's own CUDA build
 * (oracle/ref_harness.cu, built into oracle/_ref/) run on the B200; the committed fixtures in
 * tests/golden/ hold those outputs.
 *
 * Layout conventions (reference: FD2DGPU.cu, idx = ix*nzpml + iz everywhere):
 *   padded window  [nxpml][nzpml], nxpml = nx + 2*pml, nzpml = allnz + 2*pml
 *   records        [ntr][nt]
 *   window images  [nx][nz] with nz = allnz (placed at model column win_left by the caller)
 */
#ifndef DS2D_ORACLE_H
#define DS2D_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nxpml, nzpml; /* padded window */
  int pml;          /* PML or random-band width (cells) */
  int nop;          /* stencil half width, 4 (main.cpp:1490) */
  float dx, dz, dt;
} orc_grid;

typedef struct {
  int isx, isz;     /* source cell, padded window coordinates */
  int igz;          /* receiver row */
  int ntr;          /* number of receivers */
  const int *igx;   /* receiver columns */
} orc_shot;

/* Padded per-shot model (FD2DGPU.cu:122-138 window + edge replication, :444-494 PML profile,
 * :1117-1125 moduli).  rbc = 1 replaces the PML by the project random band
 * (uniform [0.6, 1.0] * vp, vs scaled alike, seeded) and leaves the damping at zero.
 * rho_all may be NULL: the reference hard-wires rho = 2000 (FD2DGPU.cu:1121).
 * Outputs are [nxpml][nzpml] float arrays: vp, vs, rho, lam, mu, dampx, dampz. */
int orc_build_model(const orc_grid *g, int allnx, int allnz, const float *vp_all,
                    const float *vs_all, const float *rho_all, int win_left, int rbc,
                    uint64_t seed, int shot_id, float *vp, float *vs, float *rho, float *lam,
                    float *mu, float *dampx, float *dampz);

/* Windowed, edge-replicated image (FD2DGPU.cu:1324-1333 buffer_image_extrapolation). */
int orc_window_image(const orc_grid *g, int allnx, int allnz, const float *img_all,
                     int win_left, float *img_pad);

/* Ricker wavelet exactly as main.cpp:461-473 ricker1. */
void orc_ricker(int nt, float f0, float dt, float *s);

/* Background forward modeling, one shot: source on txx/tzz, the four update_* kernels per step
 * (FD2DGPU.cu:4398-4400, born.cu:215-349); records the background vz / vx at the receivers
 * after every step.  rec_* are [ntr][nt]. */
int orc_forward_f64(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                    const orc_shot *s, double *rec_vz, double *rec_vx);
int orc_forward_f32(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                    const orc_shot *s, double *rec_vz, double *rec_vx);

/* Reference-mode ELSRTM, one shot (FD2DGPU.cu:4184-4879 ELSRTM_ROT_EXP_IMAGE_SINGLESHOT with
 * cpu_mem = 0).  dm_p / dm_s are the padded image windows (orc_window_image).  obs_* [ntr][nt].
 * Outputs (any may be NULL):
 *   lm_vz / lm_vx      Lm + Lm2 recorded in the forward pass (before the residual overwrites it)
 *   res_vz / res_vx    adjoint source injected in the backward pass
 *   img[7]             window images [nx][nz] in imagebuffer_resettozero order:
 *                      pp_grad, ps_grad, illumination, b_pp, b_ps, b_pp2, b_ps2
 *   misfit             accumulated exactly as FD2DGPU.cu:4615-4618 (iter > 0 only) */
/* First-order Born records (scattered vz, vx) of born_modeling mode 1 (FD2DGPU.cu:1820-1831). */
int orc_born_f64(const orc_grid *g, const float *const model[7], const float *dm_p,
                 const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                 double *rec_vz, double *rec_vx);
int orc_born_f32(const orc_grid *g, const float *const model[7], const float *dm_p,
                 const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                 double *rec_vz, double *rec_vx);
int orc_elsrtm_f64(const orc_grid *g, const float *const model[7], const float *dm_p,
                   const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                   const float *obs_vz, const float *obs_vx, int iter, int rbc, int adjoint_born,
                   double *lm_vz,
                   double *lm_vx, double *res_vz, double *res_vx, double *const img[7],
                   double *misfit);
int orc_elsrtm_f32(const orc_grid *g, const float *const model[7], const float *dm_p,
                   const float *dm_s, const float *wavelet, int nt, const orc_shot *s,
                   const float *obs_vz, const float *obs_vx, int iter, int rbc, int adjoint_born,
                   double *lm_vz,
                   double *lm_vx, double *res_vz, double *res_vx, double *const img[7],
                   double *misfit);

/* Elastic RTM, one shot: background forward pass (strips saved unless rbc), then per backward
 * step the interior reconstruction (FD2DGPU.cu:4769-4772), injection of adj_* at the receivers
 * (:3306, stack = true), the adjoint step (:4775-4778) and the zero-lag imaging condition
 * (:3245 doimage_gradient, :3235 doimage_illum).  img[3] = pp, ps, illumination [nx][nz]. */
int orc_rtm_f64(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                const orc_shot *s, const float *adj_vz, const float *adj_vx, int rbc,
                double *const img[3]);
int orc_rtm_f32(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                const orc_shot *s, const float *adj_vz, const float *adj_vx, int rbc,
                double *const img[3]);

/* NCC adjoint source and misfit on one shot (FD2DGPU.cu:4556-4664), in double. */
void orc_ncc_residual(int ntr, int nt, const float *syn_vz, const float *syn_vx,
                      const float *obs_vz, const float *obs_vx, int iter, double *res_vz,
                      double *res_vx, double *misfit);

/* Adam-like image update of main.cpp:1092-1131 (one call = one iteration on rank 1). State arrays
 * s_p, s_s, r_p, r_s carry the first / second moments between calls ([allnx*allnz] each). */
void orc_adam_update(int n, int iter, const float *const grads[6], float *image_pp,
                     float *image_ps, double *s_p, double *s_s, double *r_p, double *r_s);

/* Acoustic Born operator pair for CG-LSRTM (no reference counterpart: the reference's CG
 * helpers, main.cpp:1224-1320, are never called and its adjoint is not the transpose of its
 * Born modelling).  The acoustic scheme is the elastic one with mu = 0 (txx = tzz = sigma,
 * txz = 0; born.cu:282-349 with miu = 0); the Born source is add_born_source with mu = 0
 * (born.cu:394-400: sigma += -2 lam m (Dx- vx / dx + Dz- vz / dz), interior only, transient).
 * Boundary: random band (model as built by orc_build_model with rbc = 1) and NO damping, so the
 * background field is reconstructed by exact time reversal over the whole grid (source
 * included).  model[] = vp, vs(unused), rho, lam, mu(unused), dampx, dampz (unused).
 *   orc_ac_born:  m (padded [nxpml][nzpml], zero outside the interior) -> rec_vz, rec_vx [ntr][nt]
 *   orc_ac_born_adj: rec_vz, rec_vx -> g (padded), the exact transpose of orc_ac_born. */
int orc_ac_born(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                const orc_shot *s, const double *m, double *rec_vz, double *rec_vx);
int orc_ac_born_adj(const orc_grid *g, const float *const model[7], const float *wavelet, int nt,
                    const orc_shot *s, const double *rec_vz, const double *rec_vx, double *grad);

/* Project random-band factor in [0.6, 1.0): shared bit-for-bit with the CUDA setup kernel. */
float orc_random_band_factor(uint64_t seed, int shot_id, int ix, int iz);

#ifdef __cplusplus
}
#endif
#endif
