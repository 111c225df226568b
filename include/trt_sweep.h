/*
 * trt_sweep.h -- C ABI of the B200 SCB transport sweep library (libtrt_sweep.so).
 *
 * Drop-in for the hot path of jmc9/2D_TRT_ROM_System: MODULE TRANSPORT_SOLVES
 * (MainSrc/TRANSPORT_SOLVES.f08) and the QD-factor routines of MODULE MLOQD_SOLVES / GLOQD_SOLVES
 * that consume its output.  Two layers:
 *
 *  1. Reference-signature entry points (trt_transport_scb, trt_collapse_intensities, ...): the same
 *     arguments, in the same order and the same Fortran column-major layouts, as the Fortran
 *     subroutine each one replaces, plus the array extents that Fortran's assumed-shape arrays carry
 *     implicitly.  All arrays are host memory owned by the caller.  A Fortran shim module with
 *     BIND(C) interfaces re-exposes them under the original subroutine names.
 *  2. A resident-state handle (trt_create ... trt_destroy): the corner intensities I_crn and the
 *     boundary intensities stay in device memory between calls; only materials go in and moments,
 *     QD factors and boundary factors come out.
 *
 * Conventions: every array argument is a plain pointer to doubles (REAL*8) or ints (INTEGER), in the
 * reference's layout; indices inside arrays follow Fortran order (first index fastest).  Every
 * function returns 0 on success or a negative TRT_ERR_* code (the reference STOPs; a shim STOPs
 * with trt_strerror(code)).  A handle is single-threaded and not re-entrant; it owns one CUDA stream.
 * Functions that return data to host memory synchronise that stream.  There is no CPU fallback: with
 * no usable CUDA device every call returns TRT_ERR_NODEV.
 */
#ifndef TRT_SWEEP_H
#define TRT_SWEEP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TRT_OK 0
#define TRT_ERR_ARG (-1)          /* invalid argument or extent */
#define TRT_ERR_CUDA (-2)         /* CUDA runtime error */
#define TRT_ERR_NOMEM (-3)        /* device or pinned allocation failed */
#define TRT_ERR_BUDGET (-4)       /* request exceeds the handle's device-memory budget */
#define TRT_ERR_TIMEOUT (-5)      /* a bounded device-side wait gave up; the handle stays usable */
#define TRT_ERR_STATE (-6)        /* call order: e.g. trt_sweep before trt_set_material */
#define TRT_ERR_NODEV (-7)        /* no CUDA device */
#define TRT_ERR_UNSUPPORTED (-8)  /* shape outside the compiled kernel set (N_m/4 > 64) */
#define TRT_ERR_SCRATCH (-9)      /* problem larger than the fixed scratch of trt_transport_residual_noalloc */
#define TRT_ERR_NOCONV (-10)      /* the low-order linear solve of a group stopped without converging */

#define TRT_PREC_FP64 0   /* plain: FP64 state and arithmetic throughout */
#define TRT_PREC_FP32 1   /* mixed: FP32 state and sweep, FP64 moment combination and QD factors */
/* OR-ed into trt_create's precision: lay the handle out with one (in-place) state buffer from the start, as
 * trt_set_inplace(ctx, 1) would, without ever allocating the second one. */
#define TRT_CREATE_INPLACE 0x10

/* trt_sweep flags */
#define TRT_ROLL_STATE 1u  /* I_crn_old = I_crn before sweeping (start of a time step, ALGORITHMS.f08:397) */
#define TRT_MOMENTS 2u     /* combine moments, fg, Cg, incoming E/F and group sums after the sweep */
#define TRT_RES_CALC 4u    /* corner-balance residual norms (TRANSPORT_SOLVES.f08:249-323) */

/* ---------------------------------------------------------------------------------------------
 * Layer 1: reference-signature entry points.
 * ------------------------------------------------------------------------------------------- */

/* Replaces SUBROUTINE TRANSPORT_SCB, MainSrc/TRANSPORT_SOLVES.f08:14-27 (body :28-327).
 * I_avg(n_x,n_y,n_m,n_g), I_edgV(n_x+1,n_y,n_m,n_g), I_edgH(n_x,n_y+1,n_m,n_g): out (entries on inflow
 * faces are left as the caller had them, as in the reference); I_crn(2n_x,2n_y,n_m,n_g): out;
 * Ic_edgV(n_x+1,2n_y,n_m,n_g), Ic_edgH(2n_x,n_y+1,n_m,n_g): in (inflow faces) / out;
 * A(n_x,n_y); KapE_in(n_x,n_y,n_g); Src_in, I_crn_old (2n_x,2n_y,n_m,n_g);
 * RT_Residual(4,n_g,5), RT_ResLoc_x/y(4,n_g,5): written when Res_Calc != 0.
 * Open_Threads is accepted for signature compatibility and ignored. */
int trt_transport_scb(int n_x, int n_y, int n_m, int n_g, double* I_avg, double* I_edgV, double* I_edgH,
                      double* I_crn, double* Ic_edgV, double* Ic_edgH, const double* Omega_x,
                      const double* Omega_y, const double* Delx, const double* Dely, const double* A,
                      const double* KapE_in, const double* Src_in, const double* I_crn_old, double c,
                      double Delt, int Open_Threads, double* RT_Residual, int* RT_ResLoc_x, int* RT_ResLoc_y,
                      int Res_Calc);

/* Replaces SUBROUTINE COLLAPSE_INTENSITIES, MainSrc/TRANSPORT_SOLVES.f08:381-397 (body :398-511).
 * Group-resolved outputs are (n_x[+1], n_y[+1], n_g), totals (n_x[+1], n_y[+1]). */
int trt_collapse_intensities(int n_x, int n_y, int n_m, int n_g, int Open_Threads, const double* I_avg,
                             const double* I_edgV, const double* I_edgH, const double* Omega_x,
                             const double* Omega_y, const double* quad_weight, double Comp_Unit,
                             double* Hg_avg_xx, double* Hg_avg_yy, double* Hg_avg_xy, double* Hg_edgV_xx,
                             double* Hg_edgV_xy, double* Hg_edgH_yy, double* Hg_edgH_xy, double* Eg_edgV,
                             double* Eg_edgH, double* Eg_avg, double* Fxg_edgV, double* Fyg_edgH,
                             double* E_edgV, double* E_edgH, double* E_avg, double* Fx_edgV, double* Fy_edgH);

/* Replaces SUBROUTINE fg_Calc, MainSrc/MLOQD_SOLVES.f08:619-621 (body :622-678). */
int trt_fg_calc(int n_x, int n_y, int n_g, double* fg_avg_xx, double* fg_avg_yy, double* fg_avg_xy,
                double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy, double* fg_edgH_xy,
                const double* Hg_avg_xx, const double* Hg_avg_yy, const double* Hg_avg_xy,
                const double* Hg_edgV_xx, const double* Hg_edgV_xy, const double* Hg_edgH_yy,
                const double* Hg_edgH_xy, const double* HO_Eg_avg, const double* HO_Eg_edgV,
                const double* HO_Eg_edgH, double c, int Open_Threads);

/* Replaces SUBROUTINE Cg_Calc, MainSrc/MLOQD_SOLVES.f08:367 (body :368-488).
 * Cg_L/Cg_R(n_y,n_g), Cg_B/Cg_T(n_x,n_g); BC_Type(4) = L, B, R, T. */
int trt_cg_calc(int n_x, int n_y, int n_m, int n_g, double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T,
                const double* I_edgV, const double* I_edgH, const double* Omega_x, const double* Omega_y,
                const double* quad_weight, double Comp_Unit, const int* BC_Type, int Open_Threads);

/* Replaces SUBROUTINE MGQD_In_Calc, MainSrc/MLOQD_SOLVES.f08:493-494 (body :495-614). */
int trt_mgqd_in_calc(int n_x, int n_y, int n_m, int n_g, double* Eg_in_L, double* Eg_in_B, double* Eg_in_R,
                     double* Eg_in_T, double* Fg_in_L, double* Fg_in_B, double* Fg_in_R, double* Fg_in_T,
                     const double* I_edgV, const double* I_edgH, const double* Omega_x, const double* Omega_y,
                     const double* quad_weight, double c, double Comp_Unit, const int* BC_Type,
                     int Open_Threads);

/* Replaces SUBROUTINE GQD_In_Calc, MainSrc/GLOQD_SOLVES.f08:263-264 (body :265-290). */
int trt_gqd_in_calc(int n_x, int n_y, int n_g, double* E_in_L, double* E_in_B, double* E_in_R, double* E_in_T,
                    double* F_in_L, double* F_in_B, double* F_in_R, double* F_in_T, const double* Eg_in_L,
                    const double* Eg_in_B, const double* Eg_in_R, const double* Eg_in_T, const double* Fg_in_L,
                    const double* Fg_in_B, const double* Fg_in_R, const double* Fg_in_T);

/* Replaces SUBROUTINE RT_BC_UPDATE, MainSrc/UPDATES.f08:12 (body :13-105). Nu_g has n_g+1 edges. */
int trt_rt_bc_update(int n_x, int n_y, int n_m, int n_g, const int* BC_Type, double bcT_left, double bcT_lower,
                     double bcT_right, double bcT_upper, double Comp_Unit, const double* Nu_g, double* I_edgV,
                     double* I_edgH, double* Ic_edgV, double* Ic_edgH);

/* Bg_planck_calc, MainSrc/TEMP_FUNCTIONS.f08:90-108 (host evaluation, used for boundary values). */
double trt_bg_planck(double T, double nu_low, double nu_high, double Comp_Unit);

/* Replaces SUBROUTINE OLD_MGQD_COEFS, MainSrc/MLOQD_SOLVES.f08:12-14 (body :15-73).  Cell arrays
 * (n_x,n_y,n_g), vertical-edge arrays (n_x+1,n_y,n_g), horizontal-edge arrays (n_x,n_y+1,n_g); outputs
 * G_old, Pold_L/B/R/T (n_x,n_y,n_g). */
int trt_old_mgqd_coefs(int n_x, int n_y, int n_g, const double* Eg_avg_old, const double* Eg_edgV_old,
                       const double* Eg_edgH_old, const double* Fxg_edgV_old, const double* Fyg_edgH_old,
                       const double* fg_avg_xx_old, const double* fg_avg_yy_old, const double* fg_edgV_xx_old,
                       const double* fg_edgV_xy_old, const double* fg_edgH_yy_old, const double* fg_edgH_xy_old,
                       const double* KapE_old, const double* KapR_old, const double* Src_old, const double* Delx,
                       const double* Dely, const double* A, double c, double Delt, double Theta, double* G_old,
                       double* Pold_L, double* Pold_B, double* Pold_R, double* Pold_T, int Open_Threads);

/* Replaces SUBROUTINE MLOQD_FV, MainSrc/MLOQD_SOLVES.f08:78-82 (body :83-362), including its linear
 * solver QD_FV (MainSrc/QD_SOLVERS.f08:40-538).  Eg_avg(n_x,n_y,n_g), Eg_edgV(n_x+1,n_y,n_g),
 * Eg_edgH(n_x,n_y+1,n_g): in (initial guess) / out; Fxg_edgV(n_x+1,n_y,n_g), Fyg_edgH(n_x,n_y+1,n_g): out;
 * QD factors in the shapes of fg_Calc's outputs; Cg_L/R, Eg_in_L/R, Fg_in_L/R (n_y,n_g); Cg_B/T,
 * Eg_in_B/T, Fg_in_B/T (n_x,n_g); MGQD_Residual(n_g,5,5) and MGQD_BC_Residual(n_g,4): out when
 * Res_Calc != 0; MGQD_Kits(n_g): matrix-vector products per group (as SPARSKIT's ipar(7) counts them),
 * negated for a group that stopped without converging, in which case the call returns TRT_ERR_NOCONV
 * with the last iterate in the outputs.  All groups are solved on the device at once (FP64 BiCGSTAB,
 * right-preconditioned like the reference, with an edge-elimination + multigrid preconditioner), to a
 * Jacobi-scaled residual of at most tol * max|E| per group (trt_mgqd_set_tolerance; default 1e-13). */
int trt_mloqd_fv(int n_x, int n_y, int n_g, double* Eg_avg, double* Eg_edgV, double* Eg_edgH, double* Fxg_edgV,
                 double* Fyg_edgH, const double* fg_avg_xx, const double* fg_avg_yy, const double* fg_edgV_xx,
                 const double* fg_edgV_xy, const double* fg_edgH_yy, const double* fg_edgH_xy, const double* Cg_L,
                 const double* Cg_B, const double* Cg_R, const double* Cg_T, const double* Eg_in_L,
                 const double* Eg_in_B, const double* Eg_in_R, const double* Eg_in_T, const double* Fg_in_L,
                 const double* Fg_in_B, const double* Fg_in_R, const double* Fg_in_T, const double* Src,
                 const double* KapE, const double* KapR, const double* Delx, const double* Dely, const double* A,
                 double c, double Delt, double Theta, int Open_Threads, int Res_Calc, double* MGQD_Residual,
                 double* MGQD_BC_Residual, const double* G_old, const double* Pold_L, const double* Pold_B,
                 const double* Pold_R, const double* Pold_T, const double* Eg_avg_old, const double* Fxg_edgV_old,
                 const double* Fyg_edgH_old, int* MGQD_Kits, double Fdt_Weight, double Fin_Weight,
                 double Ein_Weight);

/* Replaces SUBROUTINE COLLAPSE_MG_EF, MainSrc/MLOQD_SOLVES.f08:687 (body :688-730): group sums of the
 * multigroup E and F into the grey E_avg(n_x,n_y), E_edgV/Fx_edgV(n_x+1,n_y), E_edgH/Fy_edgH(n_x,n_y+1). */
int trt_collapse_mg_ef(int n_x, int n_y, int n_g, const double* Eg_avg, const double* Eg_edgV, const double* Eg_edgH,
                       const double* Fxg_edgV, const double* Fyg_edgH, int Open_Threads, double* E_avg, double* E_edgV,
                       double* E_edgH, double* Fx_edgV, double* Fy_edgH);

/* Replaces SUBROUTINE Cbar_Calc, MainSrc/GLOQD_SOLVES.f08:177 (body :178-231). Cb_L/Cb_R (n_y), Cb_B/Cb_T
 * (n_x); Cg_* and Eg_in_* in the multigroup boundary shapes. */
int trt_cbar_calc(int n_x, int n_y, int n_g, double* Cb_L, double* Cb_B, double* Cb_R, double* Cb_T, const double* Cg_L,
                  const double* Cg_B, const double* Cg_R, const double* Cg_T, const double* Eg_avg,
                  const double* Eg_edgV, const double* Eg_edgH, const double* Eg_in_L, const double* Eg_in_B,
                  const double* Eg_in_R, const double* Eg_in_T);

/* Replaces SUBROUTINE OLD_GREY_COEFS, MainSrc/GLOQD_SOLVES.f08:12 (body :13-42). Gold(n_x,n_y,n_g);
 * the other arrays (n_x,n_y). */
int trt_old_grey_coefs(int n_x, int n_y, int n_g, double c, double Delt, double Theta, double cv, const double* A,
                       const double* Gold, const double* Temp_old, const double* KapE_bar_old, const double* E_avg_old,
                       const double* GQD_Src_old, double* Gold_Hat, double* Rhat_old);

/* Replaces SUBROUTINE GREY_COEFS, MainSrc/GLOQD_SOLVES.f08:47-49 (body :50-146), argument order as the
 * subroutine (Pold_L, Pold_R, Pold_B, Pold_T in; KapE_Bar, the D's and PL, PR, PB, PT out, (n_x,n_y)). */
int trt_grey_coefs(int n_x, int n_y, int n_g, const double* Eg_avg, const double* Eg_edgV, const double* Eg_edgH,
                   const double* Fxg_edgV_old, const double* Fyg_edgH_old, const double* fg_avg_xx,
                   const double* fg_avg_yy, const double* fg_edgV_xx, const double* fg_edgV_xy, const double* fg_edgH_yy,
                   const double* fg_edgH_xy, const double* KapE, const double* KapR, const double* A, double c,
                   double Delt, double Theta, const double* Pold_L, const double* Pold_R, const double* Pold_B,
                   const double* Pold_T, double* KapE_Bar, double* DC_xx, double* DL_xx, double* DR_xx, double* DC_yy,
                   double* DB_yy, double* DT_yy, double* DL_xy, double* DR_xy, double* DB_xy, double* DT_xy,
                   double* PL, double* PR, double* PB, double* PT, double Fdt_Weight);

/* Replaces SUBROUTINE EGP_FV_NEWT, MainSrc/GLOQD_SOLVES.f08:305-309 (body :310-860): Newton iterations of the
 * effective grey problem, each linear solve on the device (the solver of trt_mloqd_fv, one system).
 * E_avg/Temp/KapE_Bar (n_x,n_y), E_edgV/Fx_edgV (n_x+1,n_y), E_edgH/Fy_edgH (n_x,n_y+1): in/out; Q_bar,
 * KapE_Bar_dT (n_x,n_y): out; Its: Newton iterations; GQD_Kits(Maxits): matrix-vector products of each
 * iteration's solve (negated if it did not converge, and the call then returns TRT_ERR_NOCONV after
 * finishing the iterations).  Deltas and dresiduals are (Maxits,6) buffers whose first Its rows are filled
 * when Res_Calc != 0 (the reference allocates them (Its,6)).  Logical arguments are 0/1.  The safety
 * search makes one pass (the reference's loop at :646-755 has no exit; one pass is the state it reaches). */
int trt_egp_fv_newt(int n_x, int n_y, double* E_avg, double* E_edgV, double* E_edgH, double* Temp, double* KapE_Bar,
                    double* Fx_edgV, double* Fy_edgH, double* Q_bar, double* KapE_Bar_dT, int* Its, double* Deltas,
                    double* dresiduals, const double* Temp_Mold, const double* KapE_bar_Mold, double Theta, double Delt,
                    const double* Delx, const double* Dely, const double* A, const double* Cb_L, const double* Cb_B,
                    const double* Cb_R, const double* Cb_T, const double* E_in_L, const double* E_in_B,
                    const double* E_in_R, const double* E_in_T, const double* F_in_L, const double* F_in_B,
                    const double* F_in_R, const double* F_in_T, const double* DC_xx, const double* DL_xx,
                    const double* DR_xx, const double* DC_yy, const double* DB_yy, const double* DT_yy,
                    const double* DL_xy, const double* DR_xy, const double* DB_xy, const double* DT_xy,
                    const double* PL, const double* PR, const double* PB, const double* PT, const double* Gold_Hat,
                    const double* Rhat_old, double Kap0, double cv, double Comp_Unit, double Chi, double line_src,
                    double E_Bound_Low, double T_Bound_Low, double Eps1, double Eps2, int Maxits, int MGQD_It,
                    int Use_Line_Search, int Use_Safety_Search, int Res_Calc, int kapE_dT_flag, int* GQD_Kits,
                    double Fin_Weight, double Ein_Weight);

/* Convergence settings of trt_mloqd_fv (process-wide): tol > 0, maxit >= 1 iterations per group. */
int trt_mgqd_set_tolerance(double tol, int maxit);
/* No counterpart in the reference.  The low-order BiCGSTAB solves (MLOQD_FV, the EGP Newton steps, the mlqd
 * time step) replay each block of iterations between two host convergence checks as one CUDA graph (on, the
 * default) or launch its kernels one by one (0); the kernels and their order are the same either way. */
int trt_mgqd_set_graphs(int on);
/* No counterpart in the reference.  The multigrid preconditioner of those solves runs each fine level's
 * pre-smoothing and restriction, and its prolongation and post-smoothing, as one kernel over tiles with a halo
 * (on, the default) or as one kernel per half-sweep (0); the cell arithmetic and its order are the same, so the
 * results are identical. */
int trt_mgqd_set_fused_levels(int on);
/* No counterpart in the reference.  The multigrid levels of at most 64 x 64 cells run in one kernel per group
 * that keeps them in shared memory (on, the default, where they fit in 200 KB) or the levels above 32 x 32 in
 * the tiled level passes and the rest in a one-CTA kernel over global memory (0); the cell arithmetic and its
 * order are the same, so the results are identical. */
int trt_mgqd_set_smem_vcycle(int on);

/* Of the last trt_mloqd_fv call: device time (ms, events around the solve, excluding host<->device
 * copies), the largest iteration count, and the device time of its first matrix-vector product (ms;
 * 0 when the initial guess had already converged).  Any pointer may be NULL. */
int trt_mgqd_last_stats(double* device_ms, int* max_iterations, double* matvec_ms);

/* ---------------------------------------------------------------------------------------------
 * Layer 2: resident-state handle.  Replaces the state hand-off of ALGORITHMS.f08:397 and the call
 * sequence TRANSPORT_SCB -> COLLAPSE_INTENSITIES -> [RT_BC_UPDATE, MGQD_In_Calc] -> fg_Calc ->
 * Cg_Calc of ALGORITHMS.f08:541-572 and :1045-1095.
 * ------------------------------------------------------------------------------------------- */
typedef struct trt_ctx trt_ctx;

/* Host destinations for trt_moments; any NULL field is skipped.  Shapes as in the reference
 * (RT_INIT/MGQD_INIT, MainSrc/INITIALIZERS.f08:51-76,193-230).  Fyg_edgH/Fy_edgH are weighted
 * by Omega_x as COLLAPSE_INTENSITIES writes them (TRANSPORT_SOLVES.f08:469); Fyg_edgH_true/
 * Fy_edgH_true are the Omega_y-weighted fluxes. */
typedef struct trt_moments_host {
  double *Hg_avg_xx, *Hg_avg_yy, *Hg_avg_xy, *Hg_edgV_xx, *Hg_edgV_xy, *Hg_edgH_yy, *Hg_edgH_xy;
  double *Eg_avg, *Eg_edgV, *Eg_edgH, *Fxg_edgV, *Fyg_edgH;
  double *fg_avg_xx, *fg_avg_yy, *fg_avg_xy, *fg_edgV_xx, *fg_edgV_xy, *fg_edgH_yy, *fg_edgH_xy;
  double *Cg_L, *Cg_B, *Cg_R, *Cg_T;
  double *Eg_in_L, *Eg_in_B, *Eg_in_R, *Eg_in_T, *Fg_in_L, *Fg_in_B, *Fg_in_R, *Fg_in_T;
  double *E_avg, *E_edgV, *E_edgH, *Fx_edgV, *Fy_edgH;
  double *E_in_L, *E_in_B, *E_in_R, *E_in_T, *F_in_L, *F_in_B, *F_in_R, *F_in_T;
  double *Fyg_edgH_true, *Fy_edgH_true;
} trt_moments_host;

/* Create a handle for an n_x x n_y grid, n_m directions (n_m % 4 == 0, quadrant-ordered as
 * INPUT_QUAD builds them, INPUTS.f08:1658-1669) and n_g groups.  precision = TRT_PREC_*.
 * hbm_budget = bytes of device memory the handle may allocate (0 = no limit).  *status receives 0 or
 * a TRT_ERR_* code; NULL is returned on failure. */
trt_ctx* trt_create(int n_x, int n_y, int n_m, int n_g, const double* Omega_x, const double* Omega_y,
                    const double* quad_weight, const double* Delx, const double* Dely, int precision,
                    size_t hbm_budget, int* status);
void trt_destroy(trt_ctx* ctx);

/* Device bytes a handle of this shape would allocate with the default tiling (for admission against
 * a budget).  A full corner source (trt_set_source_full, TRANSPORT_SCB) adds one more state-sized array. */
size_t trt_required_bytes(int n_x, int n_y, int n_m, int n_g, int precision);

/* Kernel tiling: warps per CTA (1..16), direction slices per warp (1,2,4,8,16,32), TMA pipeline
 * stages (1..4) and direction splits per quadrant (CTAs per (group, quadrant), 1..n_m/4); 0 selects
 * the default for each.  Re-lays out the resident state (zeroed: put it again afterwards).  Sweep
 * results do not depend on warps, slices or stages; the moment sums are added in a different order
 * when the number of splits changes (last-bit differences). */
int trt_set_tiling(trt_ctx* ctx, int warps_per_cta, int slices, int stages, int splits);
int trt_get_tiling(const trt_ctx* ctx, int* warps_per_cta, int* slices, int* dirs_per_lane, int* stages,
                   int* splits);

/* Spatial tiles of the sweep: the rounds (row tiles of warps x rows-per-warp rows) of every (group,
 * quadrant, split) sweep are dealt round-robin to `bands` CTAs (1..8) that run as one thread-block
 * cluster, each a row tile behind the one below on a tile-diagonal wavefront; a round's bottom inflow is
 * the round below's top outflow, handed over through an L2-resident buffer with a cluster-scope
 * release/acquire progress count per step (bounded waits; a wait that runs out sets the timeout error).
 * 0 or 1 = one CTA sweeps every round.  Capped at the number of rounds.  Results are bit-identical for
 * every band count.  Re-lays out (zeroes) the state.  trt_get_bands returns the count in use.
 * (TRANSPORT_SOLVES.f08:54-242 sweeps each (m, g) over the whole grid in one thread.) */
int trt_set_bands(trt_ctx* ctx, int bands);
int trt_get_bands(const trt_ctx* ctx);

/* In-place state (on = 1): one corner-state buffer instead of two.  The sweep reads each cell's I_crn_old
 * from the skewed layout before it writes I_crn to the same place, so the state takes half the device
 * memory (the 1024^2 x 64-group x S16 instance fits in FP32 only this way).  A sweep then consumes
 * I_crn_old: after a sweep, the next one must roll (TRT_ROLL_STATE, a new time step), TRT_RES_CALC is
 * refused, and trt_tstep / trt_mlqd_step allow a single outer iteration per step (TRT_ERR_STATE otherwise).
 * Re-lays out (zeroes) the state.  (The reference keeps I_crn and I_crn_old, ALGORITHMS.f08:397.) */
int trt_set_inplace(trt_ctx* ctx, int on);
/* Bytes of the handle's corner state in its current layout (one buffer). */
size_t trt_state_bytes(const trt_ctx* ctx);
/* In-place handles only: use caller-provided device memory (at least trt_state_bytes, 128-byte aligned) for
 * the state, so that a host driver can stream group slabs of a state larger than the device through a few
 * device buffers (the bytes are the handle's private layout; copy them whole).  The handle's own buffer is
 * released; the binding ends with the next re-layout.  The bound state must be put (trt_put_state,
 * trt_init_state or raw bytes copied in by the caller, then trt_state_written) before the next sweep. */
int trt_bind_state(trt_ctx* ctx, void* device_state, size_t bytes);
/* The bound or own state holds a valid I_crn_old (after the caller copied raw state bytes in). */
int trt_state_written(trt_ctx* ctx);
/* Snapshot of groups g0 .. g0+n_groups-1 of the cell-average angular intensity (as trt_snapshot_angular,
 * FP32, (n_x, n_y, n_m, n_groups) Fortran order) into a caller's device store, on the handle's stream. */
int trt_snapshot_angular_groups(trt_ctx* ctx, int g0, int n_groups, float* I_avg_device);

/* Register budget of the sweep kernel.  Each configuration is compiled at three levels: 0 for any CTA
 * size (at most 128 registers per thread), 1 for CTAs of at most 128 threads with 3 per SM (up to 170),
 * 2 for CTAs of at most 128 threads with 2 per SM (up to 255).  mode -1 (the default) uses the highest
 * level whose variant keeps the whole grid resident at once; mode 0..2 caps the level.  Re-lays out
 * (zeroes) the state.  trt_get_register_mode returns the level in use. */
int trt_set_register_mode(trt_ctx* ctx, int mode);
int trt_get_register_mode(const trt_ctx* ctx);

/* Autotuner: times one sweep of this handle's problem for each (direction splits 1..4) x (warps per CTA
 * 2, 3, 4, 5, 6, 8) x (bands 1, 2, 4) tiling whose CTAs are all resident at once (CUDA occupancy query),
 * with the default slices per warp, and keeps the fastest.  Uses the handle's material if set, else a zero
 * material.  Call before trt_init_state / trt_put_state: it re-lays out (and zeroes) the state.
 * Outputs (each may be NULL): the chosen warps, slices, splits and its sweep time in ms. */
int trt_autotune(trt_ctx* ctx, int* warps_per_cta, int* slices, int* splits, float* sweep_ms);

/* Material for the next sweeps: KapE_in(n_x,n_y,n_g) (the opacity before the 1/(c*Delt) term of
 * TRANSPORT_SOLVES.f08:47) and the isotropic corner source src_iso(n_x,n_y,n_g) = KapB*Bg
 * (UPDATES.f08:141-150).  c and Delt as passed to TRANSPORT_SCB; Comp_Unit as passed to
 * COLLAPSE_INTENSITIES (eps = 1e-25/Comp_Unit). */
int trt_set_material(trt_ctx* ctx, const double* KapE_in, const double* src_iso, double c, double Delt,
                     double Comp_Unit);
/* Same with device pointers (FP64, same layouts), stream-ordered on the handle's stream. */
int trt_set_material_device(trt_ctx* ctx, const double* d_KapE_in, const double* d_src_iso, double c,
                            double Delt, double Comp_Unit);
/* Anisotropic per-corner source Src_in(2n_x,2n_y,n_m,n_g) instead of src_iso (NULL reverts). */
int trt_set_source_full(trt_ctx* ctx, const double* Src_in);

/* Boundary corner-edge intensities on the inflow faces, taken from full reference arrays
 * Ic_edgV(n_x+1,2n_y,n_m,n_g) and Ic_edgH(2n_x,n_y+1,n_m,n_g); BC_Type(4) = L, B, R, T selects
 * Planck/vacuum (0) or reflective (1) sides for the moment combination. */
int trt_set_boundary(trt_ctx* ctx, const double* Ic_edgV, const double* Ic_edgH, const int* BC_Type);
/* RT_BC_UPDATE (UPDATES.f08:12-105) applied to the resident boundary intensities. */
int trt_bc_update(trt_ctx* ctx, const int* BC_Type, double bcT_left, double bcT_lower, double bcT_right,
                  double bcT_upper, double Comp_Unit, const double* Nu_g);

/* RT_INIT (INITIALIZERS.f08:84-107): I_crn = I_crn_old = Bg(Tini) per group, then the Planck
 * inflow faces of RT_BC_UPDATE((/0,0,0,0/), ...). */
int trt_init_state(trt_ctx* ctx, double Tini, double bcT_left, double bcT_lower, double bcT_right,
                   double bcT_upper, double Comp_Unit, const double* Nu_g);
/* I_crn_old <- I_crn(2n_x,2n_y,n_m,n_g) (restart input). */
int trt_put_state(trt_ctx* ctx, const double* I_crn);
/* I_crn(2n_x,2n_y,n_m,n_g) of the latest sweep (restart output / state hand-off). */
int trt_get_state(trt_ctx* ctx, double* I_crn);

/* One sweep of all directions and groups, enqueued on the handle's stream (flags: TRT_*). */
int trt_sweep(trt_ctx* ctx, unsigned flags);
/* Wait for the handle's stream; returns the first error a device-side check reported. */
int trt_sync(trt_ctx* ctx);
/* Copy the combined moments / factors of the latest TRT_MOMENTS sweep to host memory. */
int trt_moments(trt_ctx* ctx, const trt_moments_host* out);
/* Pipelined stepping (no counterpart in the reference, whose calls are synchronous).  For a caller that
 * streams many materials through one handle (snapshot generation, parametric runs):
 *   trt_set_material_async: enqueues the host-to-device copy of KapE_in and src_iso (as trt_set_material) on
 *     a copy stream into a staging pair, so that it overlaps the sweep already queued; the handle's stream
 *     takes the new material over in order, before the next trt_sweep.
 *   trt_moments_async: enqueues the device-to-host copies of the latest TRT_MOMENTS sweep's outputs (as
 *     trt_moments) on a second copy stream, so that they overlap the next sweep; that sweep's moment
 *     epilogue waits for them before it overwrites the outputs.
 * Host buffers should be pinned (pageable ones make the copies synchronous); inputs must stay unchanged and
 * outputs unread until trt_sync returns, which waits for both copy streams.  A step is then
 *   trt_set_material_async -> trt_sweep(TRT_ROLL_STATE | TRT_MOMENTS) -> trt_moments_async. */
int trt_set_material_async(trt_ctx* ctx, const double* KapE_in, const double* src_iso, double c, double Delt,
                           double Comp_Unit);
int trt_moments_async(trt_ctx* ctx, const trt_moments_host* out);
/* Angular intensities of the latest sweep in the reference layouts (any pointer may be NULL). */
int trt_get_angular(trt_ctx* ctx, double* I_avg, double* I_edgV, double* I_edgH, double* Ic_edgV,
                    double* Ic_edgH);
/* Snapshot output on the device (the I_out / fg / Cg writes of a snapshot-generating run, Tgen_QDf,
 * MainSrc/ALGORITHMS.f08:1046-1095, into a caller's device store instead of a netCDF file):
 * trt_snapshot_angular writes the latest I_avg(n_x,n_y,n_m,n_g) (mean of the corner intensities) as 4-byte
 * floats to I_avg_device; trt_snapshot_output copies a combined output (name as in trt_moments_host) of the
 * latest TRT_MOMENTS sweep to dst_device.  Both are enqueued on the handle's stream (trt_sync to wait) and
 * allocate nothing; a time-last store (snapshot t at offset t * size) is the layout trt_pod_calc_device reads. */
int trt_snapshot_angular(trt_ctx* ctx, float* I_avg_device);
int trt_snapshot_output(trt_ctx* ctx, const char* name, double* dst_device);
/* Residual norms of the latest TRT_RES_CALC sweep: RT_Residual(4,n_g,5), RT_ResLoc_x/y(4,n_g,5). */
int trt_get_residual(trt_ctx* ctx, double* RT_Residual, int* RT_ResLoc_x, int* RT_ResLoc_y);

/* The handle's cudaStream_t (as void*), for callers that order their own work after a sweep. */
void* trt_stream(trt_ctx* ctx);
/* Device pointer of a combined output (name as in trt_moments_host, e.g. "fg_avg_xx"), or NULL. */
const double* trt_device_output(trt_ctx* ctx, const char* name);

/* Bound on the polls of each device-side wait of the sweep (0 = default).  The failure path of a
 * wait that never completes is exercised with trt_set_wait_limit_zero: every wait gives up at once,
 * the kernel drains its outstanding copies, sets its error word and returns; trt_sync then reports
 * TRT_ERR_TIMEOUT and the handle stays usable. */
int trt_set_wait_limit(trt_ctx* ctx, unsigned polls);
int trt_set_wait_limit_zero(trt_ctx* ctx);

/* No counterpart in the reference.  Residual norms RT_Residual(4,n_g,5), RT_ResLoc_x/y(4,n_g,5) of
 * TRANSPORT_SCB's corner-balance equations (the Res_Calc block of TRANSPORT_SOLVES.f08:249-323) for
 * callers that cannot allocate device memory: a host code that owns a fixed, pre-sized device arena,
 * or a loop that must not pay the device synchronisation of cudaMalloc/cudaFree.  Every pointer is a
 * DEVICE pointer to the caller's array in the reference's Fortran layout (the I_crn, Ic_edgV, Ic_edgH
 * that TRANSPORT_SCB produced, and its inputs); the work is enqueued on `stream` (NULL = default
 * stream) and the outputs are valid once that stream has synchronised.  Nothing is allocated: the
 * per-(direction, group) scratch is a fixed device array of the library (3 MiB, held by every GPU that
 * loads the library until exit), which limits n_m*n_g to 65536 (TRT_ERR_SCRATCH beyond).  The first
 * call on a device looks up that array's address (with the device current); make that first call
 * before any stream capture.  All calls share the array and it keeps the last call's contents; calls
 * whose kernels overlap on the GPU race on it, so serialise them (one stream, or synchronise). */
int trt_transport_residual_noalloc(int n_x, int n_y, int n_m, int n_g, const double* I_crn, const double* Ic_edgV,
                                   const double* Ic_edgH, const double* Omega_x, const double* Omega_y,
                                   const double* Delx, const double* Dely, const double* A, const double* KapE_in,
                                   const double* Src_in, const double* I_crn_old, double c, double Delt,
                                   double* RT_Residual, int* RT_ResLoc_x, int* RT_ResLoc_y, void* stream);

/* ---- Transport-only time step on the device (the reference's run_type 'tr_no_qd') ----------------
 * Replaces, for one handle, the time loop of TRT_MLQD_ALGORITHM with HO_Form 0 and no low-order
 * solve (MainSrc/ALGORITHMS.f08:389-421 and 524-572, 662-668, 816-836): per time step
 * Temp_old <- Temp, I_crn_old <- I_crn, then outer iterations of
 *   TRANSPORT_SCB + COLLAPSE_INTENSITIES + fg_Calc + Cg_Calc  (the fused sweep and epilogue),
 *   RT_BC_UPDATE when a side is reflective,
 *   MEB_SOLVE(Temp, HO_Eg_avg, ...)           (UPDATES.f08:185-230),
 *   MATERIAL_UPDATE(Temp)                      (UPDATES.f08:110-152; KapE = kapB_calc * Kappa_Mult),
 *   CONVERGENCE on Temp and HO_E_avg           (CONVERGENCE_CHECKS.f08:7-44),
 * until both converge or maxit_rte iterations.  Temperatures and Nu_g are in eV, as in the reference.
 * trt_tstep_setup: Nu_g (n_g+1) group edges; kappa_mult (n_x,n_y) = Kappa_Mult(Mat(i,j)); cV (n_x,n_y)
 * heat capacity per cell (the reference's scalar cV broadcast); Temp (n_x,n_y) initial temperature;
 * Kap0, Comp_Unit, c, Delt as in the reference; BC_Type[4] and bcT[4] (L, B, R, T) for the reflective
 * boundary update.  It computes the initial material (INITIALIZERS.f08:137); the angular state comes
 * from trt_init_state or trt_put_state.  trt_tstep returns the outer-iteration count and the last T
 * and E norms. */
int trt_tstep_setup(trt_ctx* ctx, const double* Nu_g, const double* kappa_mult, const double* cV, const double* Temp,
                    double Kap0, double Comp_Unit, double c, double Delt, const int* BC_Type, const double* bcT,
                    int conv_type, double conv_ho, int maxit_rte);
int trt_tstep(trt_ctx* ctx, int* rt_its, double* T_norm, double* E_norm);
/* The same time step with the groups split over several handles (the ranks of a multi-GPU run, each with
 * its own group range, or group slabs of one instance streamed through one device).  The only coupling
 * between groups is in the energy balance (MEB_SOLVE, UPDATES.f08:185-230, or its T^4-linearised form) and
 * in the convergence test on the transport E (ALGORITHMS.f08:816-818), both per-cell sums over groups.
 * Per outer iteration its = 1, 2, ... every handle runs
 *   trt_tstep_sweep(its)        sweep (rolling I_crn_old <- I_crn when its == 1) + moments + RT_BC_UPDATE;
 *   trt_tstep_partials(part)    its group sums, 3 n_x n_y doubles in device memory, on the handle's stream;
 * the caller adds the partials of all handles (an all-reduce across ranks), and every handle then runs
 *   trt_tstep_finish(sum, its, &converged, &T_norm, &E_norm)
 * which forms the temperature from the sums (identical on every handle), the material of its own groups
 * and the convergence test; E_avg becomes the summed transport E.  trt_tstep_begin starts a step
 * (Temp_old <- Temp).  With one handle holding every group, this is trt_tstep. */
int trt_tstep_begin(trt_ctx* ctx);
int trt_tstep_sweep(trt_ctx* ctx, int its);
int trt_tstep_partials(trt_ctx* ctx, double* part_device);
int trt_tstep_finish(trt_ctx* ctx, const double* sum_device, int its, int* converged, double* T_norm,
                     double* E_norm);
/* Material law of the time loops (trt_tstep, trt_batch_tstep, trt_mlqd_step).
 *   TRT_LAW_FLECK_CUMMINGS (default): the reference's material, KapE = kapB_calc(T) * Kappa_Mult
 *     (TEMP_FUNCTIONS.f08:11-32, UPDATES.f08:130-150) and MEB_SOLVE (UPDATES.f08:185-230).
 *   TRT_LAW_CONFIG: the synthetic configurations' opacity law in place of kapB_calc,
 *     KapE = kappa0(i,j) (1 - exp(-nu_g/T)) / (nu_g^3 sqrt(T)), nu_g = sqrt(Nu_g(g) Nu_g(g+1)), T and nu in
 *     keV (the arguments stay in eV), with kappa0 passed as trt_tstep_setup's kappa_mult; MEB_SOLVE is
 *     replaced by the backward-Euler balance cv (T - T_old)/Delt = sum_g KapE_g (c Eg - 4 pi Bg(T)) with
 *     the emission linearised about the current iterate (one Newton step per outer iteration); Kap0 is
 *     unused.  The reference has no such material (it is not expressible in its input); MATERIAL_UPDATE
 *     is the template.
 * May be called before or after trt_tstep_setup; after it, the material is recomputed at once. */
#define TRT_LAW_FLECK_CUMMINGS 0
#define TRT_LAW_CONFIG 1
int trt_tstep_set_law(trt_ctx* ctx, int law);
int trt_get_temperature(trt_ctx* ctx, double* Temp);
/* Replace the device temperature and recompute the material from it (MATERIAL_UPDATE). */
int trt_put_temperature(trt_ctx* ctx, const double* Temp);

/* ---- The mlqd time step on the device (the reference's run_type 'mlqd', use_grey = 1) -------------
 * Replaces, for one handle, the time loop of TRT_MLQD_ALGORITHM with HO_Form 0, RT_start_Its 2 and
 * Fdt/Fin/Ein weights 1 (MainSrc/ALGORITHMS.f08:294-302, 389-416, 518-572, 670-836).  Per time step:
 * the _old copies (:395-413), OLD_MGQD_COEFS and OLD_GREY_COEFS, then outer iterations, each (from the
 * second on) one sweep with the fused COLLAPSE_INTENSITIES, fg_Calc and Cg_Calc (RT_BC_UPDATE on reflective
 * sides), followed by MGQD iterations of
 *   MLOQD_FV                (the device BiCGSTAB + multigrid solve of trt_mloqd_fv, FP64),
 *   COLLAPSE_MG_EF, Cbar_Calc, GREY_COEFS,
 *   EGP_FV_NEWT             (the Newton iteration of trt_egp_fv_newt, FP64),
 *   MATERIAL_UPDATE and CONVERGENCE(conv_lo) on T and the MGQD E,
 * and CONVERGENCE(conv_ho) on T and the transport E.  The sweep runs in the handle's precision; every
 * low-order field, the material and the convergence data are FP64 and stay on the device.
 * Call order: trt_create -> trt_init_state (RT_INIT) -> trt_tstep_setup (material model, Temp, Delt,
 * BC_Type, bcT, conv_type, conv_ho, maxit_rte) -> trt_mlqd_setup -> trt_mlqd_step per time step.
 * trt_mlqd_setup sets the initial low-order state of MGQD_INIT and GQD_INIT (INITIALIZERS.f08:159-427)
 * at Tini; KapE_Bar and GQD_Src, which the reference leaves unset, start at zero.  The heat capacity is
 * the per-cell cV of trt_tstep_setup (the reference's scalar cv broadcast). */
typedef struct trt_mlqd_params {
  double conv_lo;              /* MGQD-iteration tolerance */
  double conv_gr1, conv_gr2;   /* EGP Newton tolerances (Eps1 relative, Eps2 absolute) */
  int maxit_mloqd, maxit_gloqd;
  double chi, line_src;        /* KapE_Bar_dT bound factor; line-search factor (> 1) */
  double E_bound_low, T_bound_low;
  int use_line_search, use_safety_search, kapE_dT_flag;
  double theta;                /* time-integration weight (1 = backward Euler) */
  int ho_form;                 /* 0: the sweep supplies fg and Cg (run_type 'mlqd', RT_start_Its 2); 1: fg and
                                  Cg are held as the caller last set them with trt_mlqd_put, no sweep runs
                                  (HO_Form 1/3/4 with RT_start_Its 1: the POD / DMD / file-driven runs) */
} trt_mlqd_params;
typedef struct trt_mlqd_stats {
  int rt_its;          /* outer iterations of the step */
  int sweeps;          /* sweeps run (the first outer iteration of a step has none) */
  int mgqd_its;        /* MGQD iterations, summed over the outer iterations */
  int egp_its;         /* EGP Newton iterations, summed over the MGQD iterations */
  int mgqd_nonconv;    /* group solves of MLOQD_FV that stopped at the iteration limit (the step goes on
                          with that iterate; the reference falls back to a direct solve there) */
  int egp_nonconv;     /* EGP Newton linear solves that stopped at the iteration limit (likewise) */
  int mgqd_krylov_max; /* most BiCGSTAB iterations of a group solve of MLOQD_FV in the step */
  int egp_krylov_max;  /* most BiCGSTAB iterations of an EGP Newton linear solve in the step */
  double T_norm, E_norm;   /* norms of the last outer iteration */
  double sweep_ms, low_order_ms;   /* device time of the sweeps and of everything else in the step */
  double mgqd_solve_ms, egp_ms;    /* of low_order_ms: the MLOQD_FV solves and the EGP Newton iterations */
  long long mgqd_krylov_sum;       /* BiCGSTAB iterations of the MLOQD_FV solves (slowest group of each) */
  long long egp_krylov_sum;        /* BiCGSTAB iterations of the EGP Newton linear solves */
} trt_mlqd_stats;
int trt_mlqd_setup(trt_ctx* ctx, double Tini, const trt_mlqd_params* params);
int trt_mlqd_step(trt_ctx* ctx, trt_mlqd_stats* stats);
/* Groups split over handles (the ranks of a multi-GPU run; no counterpart in the reference, whose only
 * parallelism is the OpenMP loop over groups, TRANSPORT_SOLVES.f08:50-53).  The groups of the mlqd algorithm
 * meet only in group sums: OLD_GREY_COEFS's sum of G_old once per step, the transport E of the outer
 * convergence test once per outer iteration, and per MGQD iteration the sums of COLLAPSE_MG_EF
 * (MLOQD_SOLVES.f08:687-730), Cbar_Calc and GREY_COEFS (GLOQD_SOLVES.f08:89-229).
 * trt_mlqd_setup_range: the handle holds groups g_first .. g_first + n_g - 1 of an instance of ng_total groups
 * with edges nu_total (ng_total + 1 values, the handle's own edges a sub-range of them); the initial grey
 * fields and incoming energies are the sums over every group.  A time step is then, on every handle with the
 * same arguments:
 *   trt_mlqd_step_begin(part); [add the parts over the handles into tot]; trt_mlqd_step_begin_finish(tot);
 *   for rt = 1, 2, ... (at most maxit_rte):
 *     trt_mlqd_outer_begin(rt, part); [add]; trt_mlqd_outer_begin_finish(tot);
 *     for mg = 1, 2, ... (at most maxit_mloqd):
 *       trt_mlqd_mgqd_local(part); [add]; trt_mlqd_mgqd_finish(mg, tot, &converged); stop when converged
 *     trt_mlqd_outer_end(rt, &converged); stop when converged
 *   trt_mlqd_step_end(stats);
 * `part` and `tot` are device buffers of trt_mlqd_exchange_size doubles (the sums of one exchange: 16 n_x n_y
 * + 2 (n_x+1) n_y + 2 n_x (n_y+1) + 4 (n_x + n_y) at most); each *_begin / *_local call has written its part when
 * it returns, and `tot` must hold the sum over the handles when the next call starts.  The grey Newton solve
 * runs on every handle with the same totals, so every handle takes the same iterations.  With one handle
 * holding every group, `tot` = `part` gives trt_mlqd_step bit for bit (trt_mlqd_step is this sequence). */
int trt_mlqd_setup_range(trt_ctx* ctx, double Tini, const trt_mlqd_params* params, int ng_total, int g_first,
                         const double* nu_total);
long long trt_mlqd_exchange_size(trt_ctx* ctx);
int trt_mlqd_step_begin(trt_ctx* ctx, double* part);
int trt_mlqd_step_begin_finish(trt_ctx* ctx, const double* tot);
int trt_mlqd_outer_begin(trt_ctx* ctx, int rt, double* part);
int trt_mlqd_outer_begin_finish(trt_ctx* ctx, const double* tot);
int trt_mlqd_mgqd_local(trt_ctx* ctx, double* part);
int trt_mlqd_mgqd_finish(trt_ctx* ctx, int mg, const double* tot, int* converged);
int trt_mlqd_outer_end(trt_ctx* ctx, int rt, int* converged);
int trt_mlqd_step_end(trt_ctx* ctx, trt_mlqd_stats* stats);
/* Iteration counts of the last step: MGQD iterations of each outer iteration (n_outer values) and EGP
 * iterations of each MGQD iteration (n_mgqd values), each copied up to its capacity. */
int trt_mlqd_counts(trt_ctx* ctx, int* mgqd_per_outer, int cap_outer, int* egp_per_mgqd, int cap_mgqd,
                    int* n_outer, int* n_mgqd);
/* Copy a device field of the mlqd state to host memory, Fortran layout: "Temp", the grey "E_avg",
 * "E_edgV", "E_edgH", "Fx_edgV", "Fy_edgH", "KapE_Bar", "KapE_Bar_dT", "GQD_Src", "Cb_L/B/R/T", the
 * multigroup "Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH", "MGQD_Src", "MGQD_E_avg", and the
 * transport "HO_E_avg" (summed over every group; "HO_E_avg_own": over the handle's groups).  `count` is the number of doubles the caller provides (checked). */
int trt_mlqd_get(trt_ctx* ctx, const char* name, double* host, long long count);
/* Overwrite a QD-factor or boundary-factor field of the handle ("fg_avg_xx", "fg_avg_yy", "fg_edgV_xx",
 * "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy", "Cg_L", "Cg_B", "Cg_R", "Cg_T"; Fortran layout, `count` values)
 * from host memory (on_device = 0) or device memory (1): the factors a ROM reconstructs (POD_RECONSTRUCT_fg,
 * POD_RECONSTRUCT_BCg, MainSrc/POD_ROUTINES.f08:28-353) before an ho_form = 1 step. */
int trt_mlqd_put(trt_ctx* ctx, const char* name, const double* src, long long count, int on_device);

/* ---- Reduced-order model: POD of QD-factor snapshots and its reconstruction ----------------------
 * trt_pod_calc replaces the offline decomposer's POD_Calc with SVD_Calc_Cntr
 * (Decomposer/DecompSrc/POD_ROUTINES.c:75-120, LA_ROUTINES.c:50-170): data(clen, n_g, n_t) in the decomposer's
 * layout (one snapshot of n_g blocks of clen values per time level; n_g = 0 for a single block), the POD of
 * block g (0-based): center(clen) = mean over t, and the thin SVD of the centred (clen x n_t) matrix,
 * umat(clen, k), sig(k) descending, vtmat(k, n_t) = V^T, k = min(clen, n_t).  The SVD is cuSOLVER's gesvd
 * (LAPACK's dgesvd in the reference); singular vectors are unique up to sign.  Returns TRT_ERR_NOCONV when the
 * SVD does not converge.  trt_pod_calc_device takes device pointers (data resident in HBM, e.g. snapshots
 * stored by a time loop) and enqueues on `stream`. */
int trt_pod_calc(const double* data, long long n_t, long long n_g, long long clen, long long g, double* center,
                 double* umat, double* sig, double* vtmat);
int trt_pod_calc_device(const double* data, long long n_t, long long n_g, long long clen, long long g, double* center,
                        double* umat, double* sig, double* vtmat, void* stream);
/* Replaces SUBROUTINE POD_RECONSTRUCT, MainSrc/POD_ROUTINES.f08:372-432 (argument order as the subroutine;
 * t is 1-based): dat(len) = C + sum_r S U V^T(., t), groupwise (PODgsum = 0: N_g blocks of len/N_g values,
 * block g with rank(g) modes packed after the earlier blocks' in S, U and V) or over the whole vector
 * (PODgsum = 1, rank(1) modes).  trt_pod_reconstruct_device takes device pointers and the per-block mode
 * offsets (sum of the earlier ranks), for a caller that keeps the basis on the device. */
int trt_pod_reconstruct(double* dat, const double* C, const double* S, const double* U, const double* V,
                        const int* rank, int len, int N_g, int N_t, int t, int PODgsum);
int trt_pod_reconstruct_device(double* dat, const double* C, const double* S, const double* U, const double* V,
                               const int* rank, const long long* offsets, int len, int n_blocks, int N_t, int t,
                               void* stream);
/* Replaces the offline decomposer's DMD of one block (DMD_Calc, Coef_Calc and Omega_Calc,
 * Decomposer/DecompSrc/DMD_ROUTINES.c:100-470): from data(clen, n_g, n_t) (layout as trt_pod_calc), the base
 * vector cvec (the last snapshot when base_subtract, else zero), X and Y = the snapshots 0..n-1 and 1..n less
 * cvec (n = N_t - 1, or N_t - 2 when base_subtract), the thin SVD X = U S V^T truncated to xr modes (all when
 * svd_eps < 0, else SVD_Rank_Calc's tail-energy rule), A~ = U^T Y V S^-1, its eigenpairs (lambda, W~), the
 * modes wmat = Y V S^-1 W~ / lambda and wmat_proj = U W~, the amplitudes b solving W~ b = U^T a0 (a0 the first
 * snapshot, less cvec only for an undivided data set, as the reference does) and omega = log(lambda) / delt
 * with Omega_Calc's branches.  Complex outputs are interleaved (re, im); the caller sizes them for
 * k = min(clen, n) modes: lambda, omega, b (2k), wmat, wmat_proj (2 clen k), umat (clen k), wmat_tild (2 k k),
 * cvec (clen); N_modes gets xr.  SVD by cuSOLVER gesvd, products by cuBLAS, eigenpairs by cuSOLVER's geev in
 * complex arithmetic (the reference: LAPACK dgeev); eigenvectors have unit norm, unique up to a phase. */
int trt_dmd_calc(const double* data, long long N_t, long long N_g, long long clen, long long g, int base_subtract,
                 double svd_eps, double delt, long long* N_modes, double* lambda, double* omega, double* b,
                 double* wmat, double* wmat_proj, double* umat, double* wmat_tild, double* cvec);
/* Replaces SUBROUTINE FMAP, MainSrc/GRID_FUNCTIONS.f08:14-44 (with BILINEAR_INTERPOLATE, :366-401): data f1 on grid 1
 * (flen1 values, blocks of Glen1) to grid 2 (f2, flen2 values, blocks of Glen2) by bilinear interpolation.
 * Grid1 / Grid2 hold (x, y) pairs; VMap(4, Glen2) names the four grid-1 values (1-based within a block) and
 * GMap(4, Glen2) the 1-based x index of the corner coordinates, as GENERATE_GRIDS builds them.  Map entries out
 * of range are rejected (TRT_ERR_ARG) before anything runs. */
int trt_fmap(const double* f1, double* f2, const double* Grid1, const double* Grid2, const int* GMap, const int* VMap,
             int Glen1, int Glen2, int flen1, int flen2);
/* Replace SUBROUTINEs GRIDMAP_GEN_AVG (kind 0), GRIDMAP_GEN_EDGV (1) and GRIDMAP_GEN_EDGH (2),
 * MainSrc/GRID_FUNCTIONS.f08:49-133: the (x, y) pairs of an N_x by N_y set of points (cell centres; vertical edges;
 * horizontal edges) from the cell widths Delx, Dely, into GridMap(2 N_x N_y).  Host code. */
int trt_gridmap_gen(int kind, const double* Delx, const double* Dely, int N_x, int N_y, double* GridMap);
/* Replaces SUBROUTINE MAP_GRIDS, MainSrc/GRID_FUNCTIONS.f08:222-327: for every point of Grid2 (len2 = twice its point
 * count) the four bracketing points of Grid1 (len1; xlen1 = twice the points of a grid-1 row), as 1-based x indices
 * into Grid1 (Map(4 len2/2), FMAP's GMap), and, when Vec_Locs is given, as point indices (FMAP's VMap).  The
 * nearest point is searched with the reference's distance.  A bracket that would reach outside Grid1's arrays is
 * rejected with TRT_ERR_ARG (the reference would read past them); like the reference, the caller keeps grid 2's
 * points inside grid 1's extent.  Host code. */
int trt_map_grids(int* Map, const double* Grid1, const double* Grid2, int len1, int len2, int xlen1, int* Vec_Locs);
/* Replace SUBROUTINEs GRIDMAP_GEN_LR_BND (side 0) and GRIDMAP_GEN_BT_BND (side 1), MainSrc/GRID_FUNCTIONS.f08:158-200:
 * the N points of a domain side, at x = pos (side 0, y at the midpoints of Del) or y = pos (side 1, x at the
 * midpoints of Del), into GridMap(2 N).  Host code. */
int trt_gridmap_gen_bnd(int side, const double* Del, double pos, int N, double* GridMap);
/* Replaces SUBROUTINE GENERATE_GRIDS_XY, MainSrc/GRID_FUNCTIONS.f08:689-749: the simulation grid's point sets
 * (cell centres 2 N_x N_y, vertical edges 2 (N_x+1) N_y, horizontal edges 2 N_x (N_y+1), boundaries 4 (N_x+N_y):
 * left, bottom, right at x = ylen, top at y = xlen, the reference's placement), the data grid's point sets on its
 * cells padded with a zero-width cell on each side (2 (dN_x+2)(dN_y+2), 2 (dN_x+1)(dN_y+2), 2 (dN_x+2)(dN_y+1),
 * 4 (dN_x+dN_y)+16), and MAP_GRIDS of each pair (GMap_/VMap_ with twice the simulation set's values).  Each
 * boundary map uses its own side's counts, which equals the reference's calls on its square grids (it passes
 * the left side's counts for all four sides).  Host code. */
int trt_generate_grids_xy(const double* Delx_d, const double* Dely_d, const double* Delx, const double* Dely,
                          double xlen_d, double ylen_d, double xlen, double ylen, int dN_x, int dN_y, int N_x, int N_y,
                          double* Sim_Grid_Avg, double* Sim_Grid_EdgV, double* Sim_Grid_EdgH, double* Sim_Grid_Bnds,
                          double* Dat_Grid_Avg, double* Dat_Grid_EdgV, double* Dat_Grid_EdgH, double* Dat_Grid_Bnds,
                          int* GMap_xyAvg, int* GMap_xyEdgV, int* GMap_xyEdgH, int* GMap_xyBnds, int* VMap_xyAvg,
                          int* VMap_xyEdgV, int* VMap_xyEdgH, int* VMap_xyBnds);
/* Replace SUBROUTINEs POD_RECONSTRUCT_fg and POD_RECONSTRUCT_BCg, MainSrc/POD_ROUTINES.f08:28-353, and
 * DMD_RECONSTRUCT_fg and DMD_RECONSTRUCT_BCg, MainSrc/DMD_ROUTINES.f08:131-424 (arguments in the reference's order,
 * without Open_Threads; COMPLEX*16 arrays as interleaved (re, im) doubles).  Each field is reconstructed on the data
 * grid (POD: at data level TMap(2t-1), and when TMap(2t) differs also there with LINEAR_INTERPOLATION between them;
 * DMD: at Time), padded as the reference pads it for the mapping (EXTND_BT_BND for the vertical-edge factors,
 * EXTND_LR_BND for the horizontal-edge ones, AVG_APND_BND for the cell averages with the left/right values of
 * fg_edgV_xx and the bottom/top values of fg_edgH_yy, each boundary factor side with its end values repeated) and
 * mapped to the simulation grid by FMAP with the point sets and maps of trt_generate_grids_xy and the time map of
 * trt_generate_grids_t.  Host arrays in and out; the work runs on the device.  N_g must equal dN_g; the maps are
 * checked on the host before any launch. */
int trt_pod_reconstruct_fg(
    double* fg_avg_xx, double* fg_avg_yy, double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy,
    double* fg_edgH_xy, const double* C_fg_avg_xx, const double* S_fg_avg_xx, const double* U_fg_avg_xx,
    const double* V_fg_avg_xx, const double* C_fg_edgV_xx, const double* S_fg_edgV_xx, const double* U_fg_edgV_xx,
    const double* V_fg_edgV_xx, const double* C_fg_avg_yy, const double* S_fg_avg_yy, const double* U_fg_avg_yy,
    const double* V_fg_avg_yy, const double* C_fg_edgH_yy, const double* S_fg_edgH_yy, const double* U_fg_edgH_yy,
    const double* V_fg_edgH_yy, const double* C_fg_edgV_xy, const double* S_fg_edgV_xy, const double* U_fg_edgV_xy,
    const double* V_fg_edgV_xy, const double* C_fg_edgH_xy, const double* S_fg_edgH_xy, const double* U_fg_edgH_xy,
    const double* V_fg_edgH_xy, const int* rrank_fg_avg_xx, const int* rrank_fg_edgV_xx, const int* rrank_fg_avg_yy,
    const int* rrank_fg_edgH_yy, const int* rrank_fg_edgV_xy, const int* rrank_fg_edgH_xy, int dN_x, int dN_y,
    int dN_g, int dN_t, int N_x, int N_y, int N_g, int N_t, int t, int PODgsum, const double* Sim_Grid_Avg,
    const double* Sim_Grid_EdgV, const double* Sim_Grid_EdgH, const double* Dat_Grid_Avg, const double* Dat_Grid_EdgV,
    const double* Dat_Grid_EdgH, const double* Sim_TGrid, const double* Dat_TGrid, const int* GMap_xyAvg,
    const int* GMap_xyEdgV, const int* GMap_xyEdgH, const int* VMap_xyAvg, const int* VMap_xyEdgV,
    const int* VMap_xyEdgH, const int* TMap);
int trt_pod_reconstruct_bcg(double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T, const double* C_BCg,
                            const double* S_BCg, const double* U_BCg, const double* V_BCg, const int* rrank_BCg,
                            int dN_x, int dN_y, int dN_g, int dN_t, int N_x, int N_y, int N_g, int N_t, int t,
                            int PODgsum, const double* Sim_Grid_Bnds, const double* Dat_Grid_Bnds,
                            const double* Sim_TGrid, const double* Dat_TGrid, const int* GMap_xyBnds,
                            const int* VMap_xyBnds, const int* TMap);
int trt_dmd_reconstruct_fg(
    double* fg_avg_xx, double* fg_avg_yy, double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy,
    double* fg_edgH_xy, const double* L_fg_avg_xx, const double* B_fg_avg_xx, const double* W_fg_avg_xx,
    const double* C_fg_avg_xx, const double* L_fg_edgV_xx, const double* B_fg_edgV_xx, const double* W_fg_edgV_xx,
    const double* C_fg_edgV_xx, const double* L_fg_avg_yy, const double* B_fg_avg_yy, const double* W_fg_avg_yy,
    const double* C_fg_avg_yy, const double* L_fg_edgH_yy, const double* B_fg_edgH_yy, const double* W_fg_edgH_yy,
    const double* C_fg_edgH_yy, const double* L_fg_edgV_xy, const double* B_fg_edgV_xy, const double* W_fg_edgV_xy,
    const double* C_fg_edgV_xy, const double* L_fg_edgH_xy, const double* B_fg_edgH_xy, const double* W_fg_edgH_xy,
    const double* C_fg_edgH_xy, const int* rrank_fg_avg_xx, const int* rrank_fg_edgV_xx, const int* rrank_fg_avg_yy,
    const int* rrank_fg_edgH_yy, const int* rrank_fg_edgV_xy, const int* rrank_fg_edgH_xy, int dN_x, int dN_y,
    int dN_g, int N_x, int N_y, int N_g, double Time, int DMDgsum, const double* Sim_Grid_Avg,
    const double* Sim_Grid_EdgV, const double* Sim_Grid_EdgH, const double* Dat_Grid_Avg, const double* Dat_Grid_EdgV,
    const double* Dat_Grid_EdgH, const int* GMap_xyAvg, const int* GMap_xyEdgV, const int* GMap_xyEdgH,
    const int* VMap_xyAvg, const int* VMap_xyEdgV, const int* VMap_xyEdgH);
int trt_dmd_reconstruct_bcg(double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T, const double* L_BCg,
                            const double* B_BCg, const double* W_BCg, const double* C_BCg, const int* rrank_BCg,
                            int dN_x, int dN_y, int dN_g, int N_x, int N_y, int N_g, double Time, int DMDgsum,
                            const double* Sim_Grid_Bnds, const double* Dat_Grid_Bnds, const int* GMap_xyBnds,
                            const int* VMap_xyBnds);
/* Device-resident forms of trt_pod_reconstruct_fg / trt_pod_reconstruct_bcg for a caller that keeps the
 * decomposition in HBM (an online ROM run): the outputs, the decomposition arrays (C, S, U, V), the point sets and
 * the maps are device arrays; the ranks, the time grids and TMap are host arrays.  The maps are checked on the
 * device before any mapping reads through them; the work runs on the given stream and is complete on return. */
int trt_pod_reconstruct_fg_device(
    double* fg_avg_xx, double* fg_avg_yy, double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy,
    double* fg_edgH_xy, const double* C_fg_avg_xx, const double* S_fg_avg_xx, const double* U_fg_avg_xx,
    const double* V_fg_avg_xx, const double* C_fg_edgV_xx, const double* S_fg_edgV_xx, const double* U_fg_edgV_xx,
    const double* V_fg_edgV_xx, const double* C_fg_avg_yy, const double* S_fg_avg_yy, const double* U_fg_avg_yy,
    const double* V_fg_avg_yy, const double* C_fg_edgH_yy, const double* S_fg_edgH_yy, const double* U_fg_edgH_yy,
    const double* V_fg_edgH_yy, const double* C_fg_edgV_xy, const double* S_fg_edgV_xy, const double* U_fg_edgV_xy,
    const double* V_fg_edgV_xy, const double* C_fg_edgH_xy, const double* S_fg_edgH_xy, const double* U_fg_edgH_xy,
    const double* V_fg_edgH_xy, const int* rrank_fg_avg_xx, const int* rrank_fg_edgV_xx, const int* rrank_fg_avg_yy,
    const int* rrank_fg_edgH_yy, const int* rrank_fg_edgV_xy, const int* rrank_fg_edgH_xy, int dN_x, int dN_y,
    int dN_g, int dN_t, int N_x, int N_y, int N_g, int N_t, int t, int PODgsum, const double* Sim_Grid_Avg,
    const double* Sim_Grid_EdgV, const double* Sim_Grid_EdgH, const double* Dat_Grid_Avg, const double* Dat_Grid_EdgV,
    const double* Dat_Grid_EdgH, const double* Sim_TGrid, const double* Dat_TGrid, const int* GMap_xyAvg,
    const int* GMap_xyEdgV, const int* GMap_xyEdgH, const int* VMap_xyAvg, const int* VMap_xyEdgV,
    const int* VMap_xyEdgH, const int* TMap, void* stream);
int trt_pod_reconstruct_bcg_device(double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T, const double* C_BCg,
                                   const double* S_BCg, const double* U_BCg, const double* V_BCg,
                                   const int* rrank_BCg, int dN_x, int dN_y, int dN_g, int dN_t, int N_x, int N_y,
                                   int N_g, int N_t, int t, int PODgsum, const double* Sim_Grid_Bnds,
                                   const double* Dat_Grid_Bnds, const double* Sim_TGrid, const double* Dat_TGrid,
                                   const int* GMap_xyBnds, const int* VMap_xyBnds, const int* TMap, void* stream);
/* Replaces SUBROUTINE RRANK_CALC, MainSrc/POD_ROUTINES.f08:791-819: the smallest rank whose discarded singular
 * values sig(rank+1:len) have a norm at most eps times the norm of all of them (len when none qualifies before
 * the last), the truncation READ_POD_FULL / READ_POD_GPART apply to a stored decomposition.  Host code. */
int trt_rrank_calc(const double* sig, double eps, int len, int* rank);
/* Replaces SUBROUTINE GENERATE_GRIDS_T, MainSrc/GRID_FUNCTIONS.f08:754-814: the data and simulation time levels and
 * TMap(2, N_t), for every simulation level the two data levels (1-based) that bracket it (equal when it coincides
 * with one within 1e-14 relative, or lies outside the data range).  Host code. */
int trt_generate_grids_t(double Delt_d, double Delt, double Start_Time_d, double Start_Time, int dN_t, int N_t,
                         double* Sim_TGrid, double* Dat_TGrid, int* TMap);
/* Replace the boundary helpers of the ROM reconstruction, MainSrc/GRID_FUNCTIONS.f08:406-656 (each with the
 * reference's arguments and value order; blocks of N_y rows of N_x values, N_g blocks): COLLECT_LR_BND (first and
 * last value of every row), COLLECT_BT_BND (first and last row), COLLECT_CRN_BND (the four corners),
 * EXTND_BT_BND (first and last row repeated below and above), EXTND_LR_BND (first and last value repeated left
 * and right), AVG_APND_BND (a field framed by given edge and corner values).  Host code. */
int trt_collect_lr_bnd(double* bnd, const double* f, int N_g, int N_y, int N_x);
int trt_collect_bt_bnd(double* bnd, const double* f, int N_g, int N_y, int N_x);
int trt_collect_crn_bnd(double* bnd, const double* f, int N_g, int N_y, int N_x);
int trt_extnd_bt_bnd(double* f_out, const double* f_in, int N_g, int N_y, int N_x);
int trt_extnd_lr_bnd(double* f_out, const double* f_in, int N_g, int N_y, int N_x);
int trt_avg_apnd_bnd(double* f_out, const double* f_in, const double* LR_Bnd, const double* BT_Bnd,
                     const double* Crn_Bnd, int N_g, int N_y, int N_x);
/* Replaces SUBROUTINE LINEAR_INTERPOLATION, MainSrc/GRID_FUNCTIONS.f08:819-829 (LINEAR_INTERPOLATE, :831-836):
 * v1 = v1 + (xm - x1) (v2 - v1) / (x2 - x1), the time interpolation between two reconstructed data levels. */
int trt_linear_interpolation(double* v1, const double* v2, double xm, double x1, double x2, int len);
/* Replaces SUBROUTINE DMD_RECONSTRUCT, MainSrc/DMD_ROUTINES.f08:28-109 (argument order as the subroutine;
 * the COMPLEX*16 arrays L (eigenvalue exponents), B (mode amplitudes) and W (modes) as interleaved (re, im)
 * doubles): dat(len) = Re(sum_r B(r) W(., r) exp(L(r) Time)) + C, groupwise (DMDgsum = 0: N_g blocks, block g
 * with rank(g) modes packed after the earlier blocks') or over the whole vector (DMDgsum = 1). */
int trt_dmd_reconstruct(double* dat, const double* L, const double* B, const double* W, const double* C,
                        const int* rank, int len, int N_g, int DMDgsum, double Time);

/* ---- Batched instances ---------------------------------------------------------------------------
 * Many independent handles (different grids, groups, quadratures, precisions) stepped together: the
 * sweeps of all handles that share a tiling class (precision, slices, directions per lane, warps per
 * CTA, stages) run as ONE kernel launch whose CTAs are the (handle, group, quadrant, direction split)
 * sweeps of every member, largest first; different classes run concurrently.  Config 2's batched
 * solve (and the serving loop's stepping) drives this instead of one launch per handle.  Every
 * handle's results are bit-identical to stepping it alone.  A batch does not own its handles; it
 * orders itself after each handle's earlier calls and each handle's later calls after it.
 *   trt_batch_sweep: trt_sweep of every handle with the same flags (asynchronous; trt_batch_sync).
 *   trt_batch_tstep: trt_tstep of every handle (set up with trt_tstep_setup); handles that converge
 *   stop sweeping while the others iterate; rt_its / T_norms / E_norms receive n values each. */
typedef struct trt_batch trt_batch;
trt_batch* trt_batch_create(trt_ctx* const* handles, int n, int* status);
void trt_batch_destroy(trt_batch* batch);
int trt_batch_sweep(trt_batch* batch, unsigned flags);
int trt_batch_sync(trt_batch* batch);
/* Launch form of the batched sweep.  on = 1 (default): for each tiling class without band CTAs, one
 * persistent launch of at most one wave of resident CTAs that take (instance, group, quadrant, split)
 * sweeps from a device work queue, largest instances first, until it is empty.  on = 0: one CTA per sweep,
 * drained by the block scheduler.  Results are bit-identical either way. */
int trt_batch_set_persistent(trt_batch* batch, int on);
int trt_batch_tstep(trt_batch* batch, int* rt_its, double* T_norms, double* E_norms);

/* Message for a TRT_ERR_* code. */
const char* trt_strerror(int code);
/* Number of kernels this library has launched in this process (instrumentation). */
unsigned long long trt_kernel_launches(void);

#ifdef __cplusplus
}
#endif

#endif /* TRT_SWEEP_H */
