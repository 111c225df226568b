// CPU oracle for the SCB transport sweep and its angular moments.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, its C-ABI or the Python
// package) links, loads or calls this file; only tests/, the smoke check and the CPU-baseline leg of
// bench.py do, as the checker.
//
// This is a restatement, in C++17 with the reference's Fortran column-major layouts and loop
// orders, of the hot path of jmc9/2D_TRT_ROM_System (MainSrc, Fortran 2008):
//   TRANSPORT_SCB            MainSrc/TRANSPORT_SOLVES.f08:14-327   -> oracle_transport_scb
//   SCB_BGEN                 MainSrc/TRANSPORT_SOLVES.f08:332-371  -> scb_bgen
//   COLLAPSE_INTENSITIES     MainSrc/TRANSPORT_SOLVES.f08:381-511  -> oracle_collapse_intensities
//   Cg_Calc                  MainSrc/MLOQD_SOLVES.f08:367-488      -> oracle_cg_calc
//   MGQD_In_Calc             MainSrc/MLOQD_SOLVES.f08:493-614      -> oracle_mgqd_in_calc
//   fg_Calc                  MainSrc/MLOQD_SOLVES.f08:619-678      -> oracle_fg_calc
//   GQD_In_Calc              MainSrc/GLOQD_SOLVES.f08:263-290      -> oracle_gqd_in_calc
//   RT_BC_UPDATE             MainSrc/UPDATES.f08:12-105            -> oracle_rt_bc_update
//   Bg_planck_calc, sigint   MainSrc/TEMP_FUNCTIONS.f08:90-141     -> oracle_bg_planck, oracle_sigint
//   kapB_calc                MainSrc/TEMP_FUNCTIONS.f08:11-32      -> oracle_kapb
//   MATERIAL_UPDATE          MainSrc/UPDATES.f08:110-152           -> oracle_material_update
//   MEB_SOLVE                MainSrc/UPDATES.f08:185-230           -> oracle_meb_solve
//   (the configurations' opacity law and T^4-linearised energy balance, in place of kapB_calc and
//    MEB_SOLVE)                                                  -> oracle_material_update_law,
//                                                                   oracle_meb_solve_law
//   CONVERGENCE              MainSrc/CONVERGENCE_CHECKS.f08:7-44   -> oracle_convergence
//
// Third-party arithmetic: the reference solves each 4x4 corner system with GAUSS_COMPLETE from the
// un-vendored library LA_TOOLS ("libjmcmath", no source and no version in the reference tree).  The
// oracle restates the published algorithm its name denotes, Gaussian elimination with complete
// pivoting (Golub & Van Loan, Matrix Computations, Alg. 3.4.2), ties resolved by the first maximum
// in column-major order.  The linear interpolation used by sigint on z in (1.95, 2.05]
// (INTERPOLATORS, also un-vendored) is restated as y1 + (y2-y1)*(z-x1)/(x2-x1).
//
// Parity status: UNPINNED.  The reference ships no tests, no golden vectors and no fixtures for this
// path, and it cannot be compiled here (no Fortran compiler, un-vendored LA_TOOLS).  The oracle is
// pinned instead by known-answer tests derived from the discrete equations and by exact rational
// solutions of small sweeps (tests/golden/).
//
// Build: -O2 -fopenmp -ffp-contract=off (the reference builds with -O2 -fopenmp; contraction is
// disabled so every operation rounds once, as written).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "scb_cell.h"

namespace {

constexpr double kC = 2.99792458e2;      // cm/sh (TRANSPORT_SOLVES.f08:403, TEMP_FUNCTIONS.f08:95)
constexpr double kErg = 6.24150934e11;   // eV/erg (TEMP_FUNCTIONS.f08:96)
constexpr double kH = 6.62613e-19;       // erg*sh (TEMP_FUNCTIONS.f08:97)

// Fortran column-major index, 0-based.
struct F2 {
  long n1;
  long operator()(long i, long j) const { return i + n1 * j; }
};
struct F3 {
  long n1, n2;
  long operator()(long i, long j, long k) const { return i + n1 * (j + n2 * k); }
};
struct F4 {
  long n1, n2, n3;
  long operator()(long i, long j, long k, long l) const { return i + n1 * (j + n2 * (k + n3 * l)); }
};

int team(int open_threads, int ng) {
  int t = open_threads;
  if (t > ng) t = ng;
  if (t < 1) t = 1;
  return t;
}

// SCB_BGEN (TRANSPORT_SOLVES.f08:332-371).  B is 4x4 column-major.
void scb_bgen(double* B, double Omega_x, double Omega_y, double Delx, double Dely, double KapE) {
  double A = Delx * Dely;
  double gamma = (std::fabs(Omega_x) * Dely + std::fabs(Omega_y) * Delx + KapE * A) / 4.0;
  double Del_Omx = Omega_x * Dely / 4.0;
  double Del_Omy = Omega_y * Delx / 4.0;
  for (int k = 0; k < 16; ++k) B[k] = 0.0;
  auto b = [&](int r, int c) -> double& { return B[(r - 1) + 4 * (c - 1)]; };
  b(1, 1) = gamma;
  b(2, 2) = gamma;
  b(3, 3) = gamma;
  b(4, 4) = gamma;
  b(1, 2) = Del_Omx;
  b(2, 3) = Del_Omy;
  b(3, 4) = -Del_Omx;
  b(1, 4) = Del_Omy;
  b(2, 1) = -Del_Omx;
  b(3, 2) = -Del_Omy;
  b(4, 3) = Del_Omx;
  b(4, 1) = -Del_Omy;
}

// Gaussian elimination with complete pivoting on a 4x4 column-major matrix; Q <- B^-1 Q.
void gauss_complete(double* Bin, double* Q) {
  double B[16];
  std::memcpy(B, Bin, sizeof(B));
  int colperm[4] = {0, 1, 2, 3};
  auto b = [&](int r, int c) -> double& { return B[r + 4 * c]; };
  for (int k = 0; k < 4; ++k) {
    int pr = k, pc = k;
    double best = -1.0;
    for (int c = k; c < 4; ++c)
      for (int r = k; r < 4; ++r)
        if (std::fabs(b(r, c)) > best) {
          best = std::fabs(b(r, c));
          pr = r;
          pc = c;
        }
    if (pr != k) {
      for (int c = 0; c < 4; ++c) std::swap(b(k, c), b(pr, c));
      std::swap(Q[k], Q[pr]);
    }
    if (pc != k) {
      for (int r = 0; r < 4; ++r) std::swap(b(r, k), b(r, pc));
      std::swap(colperm[k], colperm[pc]);
    }
    for (int r = k + 1; r < 4; ++r) {
      double f = b(r, k) / b(k, k);
      b(r, k) = 0.0;
      for (int c = k + 1; c < 4; ++c) b(r, c) = b(r, c) - f * b(k, c);
      Q[r] = Q[r] - f * Q[k];
    }
  }
  double y[4];
  for (int k = 3; k >= 0; --k) {
    double s = Q[k];
    for (int c = k + 1; c < 4; ++c) s = s - b(k, c) * y[c];
    y[k] = s / b(k, k);
  }
  for (int k = 0; k < 4; ++k) Q[colperm[k]] = y[k];
}

// sigint (TEMP_FUNCTIONS.f08:114-141).
double sigint(double z) {
  const double pi = 4.0 * std::atan(1.0);
  const double pi4 = (pi * pi) * (pi * pi);
  if (z <= 1.95) {
    return ((z * z) * z) * (1.0 / 3.0 - z / 8.0 + (z * z) / 62.4);
  } else if (z > 2.05) {
    return pi4 / 15.0 - std::exp(-z) * (((z * z) * z) + 3.0 * (z * z) + 6.0 * z + 7.28);
  } else {
    double x1 = 1.95, x2 = 2.05;
    double y1 = ((x1 * x1) * x1) * (1.0 / 3.0 - x1 / 8.0 + (x1 * x1) / 62.4);
    double y2 = pi4 / 15.0 - std::exp(-x2) * (((x2 * x2) * x2) + 3.0 * (x2 * x2) + 6.0 * x2 + 7.28);
    return y1 + (y2 - y1) * (z - x1) / (x2 - x1);
  }
}

// Bg_planck_calc (TEMP_FUNCTIONS.f08:90-108).
double bg_planck(double Tin, double nu_low, double nu_high, double comp_unit) {
  if (Tin <= 1e-15) return 0.0;
  double sig = sigint(nu_high / Tin) - sigint(nu_low / Tin);
  double h3 = (kH * kH) * kH;
  double c2 = kC * kC;
  double e2 = kErg * kErg;
  double e4 = e2 * e2;
  sig = sig / (((h3 * c2) * e4) * comp_unit);
  double t2 = Tin * Tin;
  return (2.0 * (t2 * t2)) * sig;
}

}  // namespace

extern "C" {

double oracle_sigint(double z) { return sigint(z); }

double oracle_bg_planck(double T, double nu_low, double nu_high, double comp_unit) {
  return bg_planck(T, nu_low, nu_high, comp_unit);
}

// kapB_calc (TEMP_FUNCTIONS.f08:11-32).
double oracle_kapb(double Temp, double nu_low, double nu_high) {
  const double sig0 = 27.0 * 1e9;
  double z1 = nu_high / Temp;
  double z2 = nu_low / Temp;
  double sig;
  double t3 = (Temp * Temp) * Temp;
  if (z2 > 10.0) {
    sig = -std::exp(-(z1 - z2)) * (((z1 * z1) * z1) + 3.0 * (z1 * z1) + 6.0 * z1 + 7.28) +
          (((z2 * z2) * z2) + 3.0 * (z2 * z2) + 6.0 * z2 + 7.28);
    return sig0 * (1.0 - std::exp(-(nu_high - nu_low) / Temp)) / (t3 * sig);
  }
  sig = sigint(z1) - sigint(z2);
  return sig0 * (std::exp(-nu_low / Temp) - std::exp(-nu_high / Temp)) / (t3 * sig);
}

// Solve one 4x4 SCB system (test hook).  solver 0: SCB_BGEN + Gaussian elimination with complete
// pivoting, physical frame, signed direction cosines; Q (4) is overwritten with the solution.
void oracle_scb_cell_ge(double omx, double omy, double dx, double dy, double kapE, double* Q) {
  double B[16];
  scb_bgen(B, omx, omy, dx, dy, kapE);
  gauss_complete(B, Q);
}

// TRANSPORT_SCB (TRANSPORT_SOLVES.f08:14-327).  Arrays are Fortran column-major:
//   I_avg(nx,ny,nm,ng) I_edgV(nx+1,ny,nm,ng) I_edgH(nx,ny+1,nm,ng) I_crn(2nx,2ny,nm,ng)
//   Ic_edgV(nx+1,2ny,nm,ng) Ic_edgH(2nx,ny+1,nm,ng) A(nx,ny) KapE_in(nx,ny,ng)
//   Src_in, I_crn_old (2nx,2ny,nm,ng); RT_Residual(4,ng,5), RT_ResLoc_x/y(4,ng,5).
// Ic_edgV/Ic_edgH are in/out (their inflow faces are read).  solver 0 follows the reference
// (SCB_BGEN + GAUSS_COMPLETE, Src_in + I_crn_old/(c*Delt)); solver 1 uses the closed-form cell
// solve of scb_cell.h with Src = fma(I_crn_old, 1/(c*Delt), Src_in), the arithmetic of the device.
int oracle_transport_scb(int nx, int ny, int nm, int ng, double* I_avg, double* I_edgV, double* I_edgH,
                         double* I_crn, double* Ic_edgV, double* Ic_edgH, const double* Omega_x,
                         const double* Omega_y, const double* Delx, const double* Dely, const double* A,
                         const double* KapE_in, const double* Src_in, const double* I_crn_old, double c,
                         double Delt, int open_threads, double* RT_Residual, int* RT_ResLoc_x,
                         int* RT_ResLoc_y, int res_calc, int solver) {
  if (nx < 1 || ny < 1 || ng < 1 || nm < 4 || nm % 4) return -1;
  const F4 ic{2L * nx, 2L * ny, nm};       // corner arrays
  const F4 ia{nx, ny, nm};                  // I_avg
  const F4 iv{nx + 1L, ny, nm};             // I_edgV
  const F4 ih{nx, ny + 1L, nm};             // I_edgH
  const F4 icv{nx + 1L, 2L * ny, nm};       // Ic_edgV
  const F4 ich{2L * nx, ny + 1L, nm};       // Ic_edgH
  const F3 i3{nx, ny};
  const F2 i2{nx};
  const long ncrn = 4L * nx * ny * nm * ng;

  // KapE = KapE_in + 1/(c*Delt); Src = Src_in + I_crn_old/(c*Delt)   (:45-48)
  std::vector<double> KapE((size_t)nx * ny * ng), Src((size_t)ncrn);
  const double rcdt = 1.0 / (c * Delt);
  for (size_t k = 0; k < KapE.size(); ++k) KapE[k] = KapE_in[k] + rcdt;
  if (solver == 0) {
    for (long k = 0; k < ncrn; ++k) Src[k] = Src_in[k] + I_crn_old[k] / (c * Delt);
  } else {
    for (long k = 0; k < ncrn; ++k) Src[k] = trt::tfma(I_crn_old[k], rcdt, Src_in[k]);
  }

  const int mq = nm / 4;
  const int threads = team(open_threads, ng);

#pragma omp parallel for num_threads(threads) schedule(static)
  for (int g = 0; g < ng; ++g) {
    double B[16], Q[4];
    for (int quad = 0; quad < 4; ++quad) {
      // quadrant order and sweep directions of :58-241
      const bool fx = (quad == 1 || quad == 2);   // Omega_x < 0: i runs N_x..1
      const bool fy = (quad == 2 || quad == 3);   // Omega_y < 0: j runs N_y..1
      for (int m = quad * mq; m < (quad + 1) * mq; ++m) {
        const double Ox = Omega_x[m], Oy = Omega_y[m];
        for (int jj = 0; jj < ny; ++jj) {
          const int j = fy ? ny - 1 - jj : jj;
          for (int ii = 0; ii < nx; ++ii) {
            const int i = fx ? nx - 1 - ii : ii;
            const int left = 2 * i, right = 2 * i + 1, bot = 2 * j, top = 2 * j + 1;
            const double Aij = A[i2(i, j)];
            const double kap = KapE[i3(i, j, g)];
            auto S = [&](int cx, int cy) { return Src[ic(cx, cy, m, g)]; };
            if (solver == 0) {
              scb_bgen(B, Ox, Oy, Delx[i], Dely[j], kap);
              if (quad == 0) {          // :72-76
                Q[0] = Aij * S(left, bot) / 4.0 + Ox * Dely[j] * Ic_edgV[icv(i, bot, m, g)] / 2.0 +
                       Oy * Delx[i] * Ic_edgH[ich(left, j, m, g)] / 2.0;
                Q[1] = Aij * S(right, bot) / 4.0 + Oy * Delx[i] * Ic_edgH[ich(right, j, m, g)] / 2.0;
                Q[2] = Aij * S(right, top) / 4.0;
                Q[3] = Aij * S(left, top) / 4.0 + Ox * Dely[j] * Ic_edgV[icv(i, top, m, g)] / 2.0;
              } else if (quad == 1) {   // :119-123
                Q[0] = Aij * S(left, bot) / 4.0 + Oy * Delx[i] * Ic_edgH[ich(left, j, m, g)] / 2.0;
                Q[1] = Aij * S(right, bot) / 4.0 - Ox * Dely[j] * Ic_edgV[icv(i + 1, bot, m, g)] / 2.0 +
                       Oy * Delx[i] * Ic_edgH[ich(right, j, m, g)] / 2.0;
                Q[2] = Aij * S(right, top) / 4.0 - Ox * Dely[j] * Ic_edgV[icv(i + 1, top, m, g)] / 2.0;
                Q[3] = Aij * S(left, top) / 4.0;
              } else if (quad == 2) {   // :166-170
                Q[0] = Aij * S(left, bot) / 4.0;
                Q[1] = Aij * S(right, bot) / 4.0 - Ox * Dely[j] * Ic_edgV[icv(i + 1, bot, m, g)] / 2.0;
                Q[2] = Aij * S(right, top) / 4.0 - Ox * Dely[j] * Ic_edgV[icv(i + 1, top, m, g)] / 2.0 -
                       Oy * Delx[i] * Ic_edgH[ich(right, j + 1, m, g)] / 2.0;
                Q[3] = Aij * S(left, top) / 4.0 - Oy * Delx[i] * Ic_edgH[ich(left, j + 1, m, g)] / 2.0;
              } else {                  // :213-217
                Q[0] = Aij * S(left, bot) / 4.0 + Ox * Dely[j] * Ic_edgV[icv(i, bot, m, g)] / 2.0;
                Q[1] = Aij * S(right, bot) / 4.0;
                Q[2] = Aij * S(right, top) / 4.0 - Oy * Delx[i] * Ic_edgH[ich(right, j + 1, m, g)] / 2.0;
                Q[3] = Aij * S(left, top) / 4.0 + Ox * Dely[j] * Ic_edgV[icv(i, top, m, g)] / 2.0 -
                       Oy * Delx[i] * Ic_edgH[ich(left, j + 1, m, g)] / 2.0;
              }
              gauss_complete(B, Q);
            } else {
              // sweep frame: mirror x when fx, y when fy (see scb_cell.h)
              const int sl = fx ? right : left, sr = fx ? left : right;
              const int sb = fy ? top : bot, st = fy ? bot : top;
              const int vface = fx ? i + 1 : i;   // inflow vertical face
              const int hface = fy ? j + 1 : j;   // inflow horizontal face
              const double ax = std::fabs(Ox), ay = std::fabs(Oy);
              trt::ScbGeom<double> G = trt::scb_geom(ax * 0.25, ay * 0.25, Delx[i], Dely[j]);
              double gam = trt::scb_gamma(G, trt::scb_kA4(Delx[i], Dely[j], kap));
              double s[4] = {S(sl, sb), S(sr, sb), S(sr, st), S(sl, st)};
              double x[4];
              trt::scb_solve(G, gam, Aij * 0.25, s, Ic_edgV[icv(vface, sb, m, g)],
                             Ic_edgV[icv(vface, st, m, g)], Ic_edgH[ich(sl, hface, m, g)],
                             Ic_edgH[ich(sr, hface, m, g)], x);
              // back to physical corners lb, rb, rt, lt
              auto put = [&](int cx, int cy, double v) {
                int k = (cx == left) ? (cy == bot ? 0 : 3) : (cy == bot ? 1 : 2);
                Q[k] = v;
              };
              put(sl, sb, x[0]);
              put(sr, sb, x[1]);
              put(sr, st, x[2]);
              put(sl, st, x[3]);
            }
            I_crn[ic(left, bot, m, g)] = Q[0];
            I_crn[ic(right, bot, m, g)] = Q[1];
            I_crn[ic(right, top, m, g)] = Q[2];
            I_crn[ic(left, top, m, g)] = Q[3];
            if (quad == 0) {            // :86-96
              Ic_edgV[icv(i + 1, bot, m, g)] = I_crn[ic(right, bot, m, g)];
              Ic_edgV[icv(i + 1, top, m, g)] = I_crn[ic(right, top, m, g)];
              Ic_edgH[ich(right, j + 1, m, g)] = I_crn[ic(right, top, m, g)];
              Ic_edgH[ich(left, j + 1, m, g)] = I_crn[ic(left, top, m, g)];
              I_edgV[iv(i + 1, j, m, g)] = (Ic_edgV[icv(i + 1, bot, m, g)] + Ic_edgV[icv(i + 1, top, m, g)]) / 2.0;
              I_edgH[ih(i, j + 1, m, g)] = (Ic_edgH[ich(left, j + 1, m, g)] + Ic_edgH[ich(right, j + 1, m, g)]) / 2.0;
            } else if (quad == 1) {     // :133-140
              Ic_edgV[icv(i, bot, m, g)] = I_crn[ic(left, bot, m, g)];
              Ic_edgV[icv(i, top, m, g)] = I_crn[ic(left, top, m, g)];
              Ic_edgH[ich(left, j + 1, m, g)] = I_crn[ic(left, top, m, g)];
              Ic_edgH[ich(right, j + 1, m, g)] = I_crn[ic(right, top, m, g)];
              I_edgV[iv(i, j, m, g)] = (Ic_edgV[icv(i, bot, m, g)] + Ic_edgV[icv(i, top, m, g)]) / 2.0;
              I_edgH[ih(i, j + 1, m, g)] = (Ic_edgH[ich(left, j + 1, m, g)] + Ic_edgH[ich(right, j + 1, m, g)]) / 2.0;
            } else if (quad == 2) {     // :180-187
              Ic_edgV[icv(i, top, m, g)] = I_crn[ic(left, top, m, g)];
              Ic_edgV[icv(i, bot, m, g)] = I_crn[ic(left, bot, m, g)];
              Ic_edgH[ich(left, j, m, g)] = I_crn[ic(left, bot, m, g)];
              Ic_edgH[ich(right, j, m, g)] = I_crn[ic(right, bot, m, g)];
              I_edgV[iv(i, j, m, g)] = (Ic_edgV[icv(i, bot, m, g)] + Ic_edgV[icv(i, top, m, g)]) / 2.0;
              I_edgH[ih(i, j, m, g)] = (Ic_edgH[ich(left, j, m, g)] + Ic_edgH[ich(right, j, m, g)]) / 2.0;
            } else {                    // :227-234
              Ic_edgV[icv(i + 1, top, m, g)] = I_crn[ic(right, top, m, g)];
              Ic_edgV[icv(i + 1, bot, m, g)] = I_crn[ic(right, bot, m, g)];
              Ic_edgH[ich(right, j, m, g)] = I_crn[ic(right, bot, m, g)];
              Ic_edgH[ich(left, j, m, g)] = I_crn[ic(left, bot, m, g)];
              I_edgV[iv(i + 1, j, m, g)] = (Ic_edgV[icv(i + 1, bot, m, g)] + Ic_edgV[icv(i + 1, top, m, g)]) / 2.0;
              I_edgH[ih(i, j, m, g)] = (Ic_edgH[ich(left, j, m, g)] + Ic_edgH[ich(right, j, m, g)]) / 2.0;
            }
            I_avg[ia(i, j, m, g)] = (I_crn[ic(left, bot, m, g)] + I_crn[ic(right, bot, m, g)] +
                                     I_crn[ic(right, top, m, g)] + I_crn[ic(left, top, m, g)]) / 4.0;
          }
        }
      }
    }
  }

  if (res_calc) {
    // Residual norms (:249-323).  KapE and Src are the prepared arrays of :47-48.
    const F3 r3{4, ng};
    for (long k = 0; k < 4L * ng * 5; ++k) RT_Residual[k] = 0.0;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int g = 0; g < ng; ++g) {
      for (int m = 0; m < nm; ++m) {
        const int m2 = (4 * m) / nm;   // 1 + INT(4*(m-1)/N_m), 0-based
        double sums[4] = {0.0, 0.0, 0.0, 0.0};
        const double Ox = Omega_x[m], Oy = Omega_y[m];
        for (int j = 0; j < ny; ++j) {
          for (int i = 0; i < nx; ++i) {
            const int left = 2 * i, right = 2 * i + 1, bot = 2 * j, top = 2 * j + 1;
            const double Aij = A[i2(i, j)], kap = KapE[i3(i, j, g)];
            const double dx = Delx[i], dy = Dely[j];
            auto I = [&](int cx, int cy) { return I_crn[ic(cx, cy, m, g)]; };
            auto S = [&](int cx, int cy) { return Src[ic(cx, cy, m, g)]; };
            double res[4];
            res[0] = std::fabs((Ox * dy + Oy * dx + kap * Aij) * I(left, bot) / 4.0 +
                               Ox * dy * I(right, bot) / 4.0 + Oy * dx * I(left, top) / 4.0 -
                               Ox * dy * Ic_edgV[icv(i, bot, m, g)] / 2.0 -
                               Oy * dx * Ic_edgH[ich(left, j, m, g)] / 2.0 - Aij * S(left, bot) / 4.0);
            res[1] = std::fabs((-Ox * dy + Oy * dx + kap * Aij) * I(right, bot) / 4.0 -
                               Ox * dy * I(left, bot) / 4.0 + Oy * dx * I(right, top) / 4.0 +
                               Ox * dy * Ic_edgV[icv(i + 1, bot, m, g)] / 2.0 -
                               Oy * dx * Ic_edgH[ich(right, j, m, g)] / 2.0 - Aij * S(right, bot) / 4.0);
            res[2] = std::fabs((-Ox * dy - Oy * dx + kap * Aij) * I(right, top) / 4.0 -
                               Ox * dy * I(left, top) / 4.0 - Oy * dx * I(right, bot) / 4.0 +
                               Ox * dy * Ic_edgV[icv(i + 1, top, m, g)] / 2.0 +
                               Oy * dx * Ic_edgH[ich(right, j + 1, m, g)] / 2.0 - Aij * S(right, top) / 4.0);
            res[3] = std::fabs((Ox * dy - Oy * dx + kap * Aij) * I(left, top) / 4.0 +
                               Ox * dy * I(right, top) / 4.0 - Oy * dx * I(left, bot) / 4.0 -
                               Ox * dy * Ic_edgV[icv(i, top, m, g)] / 2.0 +
                               Oy * dx * Ic_edgH[ich(left, j + 1, m, g)] / 2.0 - Aij * S(left, top) / 4.0);
            for (int k = 0; k < 4; ++k) {
              if (res[k] > RT_Residual[r3(m2, g, 0)]) {
                RT_Residual[r3(m2, g, 0)] = res[k];
                RT_ResLoc_x[r3(m2, g, 0)] = i + 1;
                RT_ResLoc_y[r3(m2, g, 0)] = j + 1;
              }
              sums[0] = sums[0] + res[k];
              sums[1] = sums[1] + res[k] * res[k];
              sums[2] = sums[2] + Aij * res[k] / 4.0;
              sums[3] = sums[3] + Aij * (res[k] * res[k]) / 4.0;
            }
          }
        }
        // the reference records the DO-loop exit values i = N_x+1, j = N_y+1 here (:311-317)
        for (int k = 0; k < 4; ++k) {
          if (sums[k] > RT_Residual[r3(m2, g, k + 1)]) {
            RT_Residual[r3(m2, g, k + 1)] = sums[k];
            RT_ResLoc_x[r3(m2, g, k + 1)] = nx + 1;
            RT_ResLoc_y[r3(m2, g, k + 1)] = ny + 1;
          }
        }
      }
    }
  }
  return 0;
}

// COLLAPSE_INTENSITIES (TRANSPORT_SOLVES.f08:381-511), same argument order.
int oracle_collapse_intensities(int nx, int ny, int nm, int ng, int open_threads, const double* I_avg,
                                const double* I_edgV, const double* I_edgH, const double* Omega_x,
                                const double* Omega_y, const double* quad_weight, double Comp_Unit,
                                double* Hg_avg_xx, double* Hg_avg_yy, double* Hg_avg_xy, double* Hg_edgV_xx,
                                double* Hg_edgV_xy, double* Hg_edgH_yy, double* Hg_edgH_xy, double* Eg_edgV,
                                double* Eg_edgH, double* Eg_avg, double* Fxg_edgV, double* Fyg_edgH,
                                double* E_edgV, double* E_edgH, double* E_avg, double* Fx_edgV, double* Fy_edgH) {
  const double c = kC;
  double eps = 1e-25;
  eps = eps / Comp_Unit;
  const F4 ia{nx, ny, nm}, iv{nx + 1L, ny, nm}, ih{nx, ny + 1L, nm};
  const F3 a3{nx, ny}, v3{nx + 1L, ny}, h3{nx, ny + 1L};
  const long na = (long)nx * ny, nv = (long)(nx + 1) * ny, nh = (long)nx * (ny + 1);
  for (long k = 0; k < na * ng; ++k) Hg_avg_xx[k] = Hg_avg_yy[k] = Hg_avg_xy[k] = Eg_avg[k] = 0.0;
  for (long k = 0; k < nv * ng; ++k) Hg_edgV_xx[k] = Hg_edgV_xy[k] = Eg_edgV[k] = Fxg_edgV[k] = 0.0;
  for (long k = 0; k < nh * ng; ++k) Hg_edgH_yy[k] = Hg_edgH_xy[k] = Eg_edgH[k] = Fyg_edgH[k] = 0.0;
  const int threads = team(open_threads, ng);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int g = 0; g < ng; ++g) {
    for (int m = 0; m < nm; ++m) {
      const double Ox = Omega_x[m], Oy = Omega_y[m], w = quad_weight[m];
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double I = I_avg[ia(i, j, m, g)] + eps;
          const long k = a3(i, j, g);
          Hg_avg_xx[k] = Hg_avg_xx[k] + (Ox * Ox) * w * I;
          Hg_avg_yy[k] = Hg_avg_yy[k] + (Oy * Oy) * w * I;
          Hg_avg_xy[k] = Hg_avg_xy[k] + Ox * Oy * w * I;
          Eg_avg[k] = Eg_avg[k] + w * I;
        }
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx + 1; ++i) {
          const double I = I_edgV[iv(i, j, m, g)] + eps;
          const long k = v3(i, j, g);
          Hg_edgV_xx[k] = Hg_edgV_xx[k] + (Ox * Ox) * w * I;
          Hg_edgV_xy[k] = Hg_edgV_xy[k] + Ox * Oy * w * I;
          Fxg_edgV[k] = Fxg_edgV[k] + Ox * w * I;
          Eg_edgV[k] = Eg_edgV[k] + w * I;
        }
      for (int j = 0; j < ny + 1; ++j)
        for (int i = 0; i < nx; ++i) {
          const double I = I_edgH[ih(i, j, m, g)] + eps;
          const long k = h3(i, j, g);
          Hg_edgH_yy[k] = Hg_edgH_yy[k] + (Oy * Oy) * w * I;
          Hg_edgH_xy[k] = Hg_edgH_xy[k] + Ox * Oy * w * I;
          Fyg_edgH[k] = Fyg_edgH[k] + Ox * w * I;   // Omega_x, as written at :469
          Eg_edgH[k] = Eg_edgH[k] + w * I;
        }
    }
    for (long k = 0; k < na; ++k) Eg_avg[k + na * g] = Eg_avg[k + na * g] / c;
    for (long k = 0; k < nv; ++k) Eg_edgV[k + nv * g] = Eg_edgV[k + nv * g] / c;
    for (long k = 0; k < nh; ++k) Eg_edgH[k + nh * g] = Eg_edgH[k + nh * g] / c;
  }
  for (long k = 0; k < na; ++k) {
    double s = 0.0;
    for (int g = 0; g < ng; ++g) s = s + Eg_avg[k + na * g];
    E_avg[k] = s;
  }
  for (long k = 0; k < nv; ++k) {
    double s = 0.0, f = 0.0;
    for (int g = 0; g < ng; ++g) {
      s = s + Eg_edgV[k + nv * g];
      f = f + Fxg_edgV[k + nv * g];
    }
    E_edgV[k] = s;
    Fx_edgV[k] = f;
  }
  for (long k = 0; k < nh; ++k) {
    double s = 0.0, f = 0.0;
    for (int g = 0; g < ng; ++g) {
      s = s + Eg_edgH[k + nh * g];
      f = f + Fyg_edgH[k + nh * g];
    }
    E_edgH[k] = s;
    Fy_edgH[k] = f;
  }
  return 0;
}

// fg_Calc (MLOQD_SOLVES.f08:619-678).
int oracle_fg_calc(int nx, int ny, int ng, double* fg_avg_xx, double* fg_avg_yy, double* fg_avg_xy,
                   double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy, double* fg_edgH_xy,
                   const double* Hg_avg_xx, const double* Hg_avg_yy, const double* Hg_avg_xy,
                   const double* Hg_edgV_xx, const double* Hg_edgV_xy, const double* Hg_edgH_yy,
                   const double* Hg_edgH_xy, const double* HO_Eg_avg, const double* HO_Eg_edgV,
                   const double* HO_Eg_edgH, double c, int open_threads) {
  const long na = (long)nx * ny, nv = (long)(nx + 1) * ny, nh = (long)nx * (ny + 1);
  const int threads = team(open_threads, ng);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int g = 0; g < ng; ++g) {
    for (long k = na * g; k < na * (g + 1); ++k) {
      fg_avg_xx[k] = Hg_avg_xx[k] / (c * HO_Eg_avg[k]);
      fg_avg_yy[k] = Hg_avg_yy[k] / (c * HO_Eg_avg[k]);
      fg_avg_xy[k] = Hg_avg_xy[k] / (c * HO_Eg_avg[k]);
    }
    for (long k = nv * g; k < nv * (g + 1); ++k) {
      fg_edgV_xx[k] = Hg_edgV_xx[k] / (c * HO_Eg_edgV[k]);
      fg_edgV_xy[k] = Hg_edgV_xy[k] / (c * HO_Eg_edgV[k]);
    }
    for (long k = nh * g; k < nh * (g + 1); ++k) {
      fg_edgH_yy[k] = Hg_edgH_yy[k] / (c * HO_Eg_edgH[k]);
      fg_edgH_xy[k] = Hg_edgH_xy[k] / (c * HO_Eg_edgH[k]);
    }
  }
  return 0;
}

// Cg_Calc (MLOQD_SOLVES.f08:367-488).  Cg_L/R(ny,ng), Cg_B/T(nx,ng).
int oracle_cg_calc(int nx, int ny, int nm, int ng, double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T,
                   const double* I_edgV, const double* I_edgH, const double* Omega_x, const double* Omega_y,
                   const double* quad_weight, double Comp_Unit, const int* BC_Type, int open_threads) {
  double eps = 1e-25;
  eps = eps / Comp_Unit;
  const F4 iv{nx + 1L, ny, nm}, ih{nx, ny + 1L, nm};
  const int threads = team(open_threads, ng);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int g = 0; g < ng; ++g) {
    for (int i = 0; i < ny; ++i) Cg_L[i + (long)ny * g] = Cg_R[i + (long)ny * g] = 0.0;
    for (int i = 0; i < nx; ++i) Cg_B[i + (long)nx * g] = Cg_T[i + (long)nx * g] = 0.0;
    if (BC_Type[0] == 0) {
      for (int i = 0; i < ny; ++i) {
        double sum = 0.0, &C = Cg_L[i + (long)ny * g];
        for (int m = nm / 4; m < 3 * nm / 4; ++m) {
          C = C + Omega_x[m] * quad_weight[m] * (I_edgV[iv(0, i, m, g)] + eps);
          sum = sum + quad_weight[m] * (I_edgV[iv(0, i, m, g)] + eps);
        }
        C = C / sum;
      }
    }
    if (BC_Type[1] == 0) {
      for (int i = 0; i < nx; ++i) {
        double sum = 0.0, &C = Cg_B[i + (long)nx * g];
        for (int m = nm / 2; m < nm; ++m) {
          C = C + Omega_y[m] * quad_weight[m] * (I_edgH[ih(i, 0, m, g)] + eps);
          sum = sum + quad_weight[m] * (I_edgH[ih(i, 0, m, g)] + eps);
        }
        C = C / sum;
      }
    }
    if (BC_Type[2] == 0) {
      for (int i = 0; i < ny; ++i) {
        double sum = 0.0, &C = Cg_R[i + (long)ny * g];
        for (int m = 0; m < nm / 4; ++m) {
          C = C + Omega_x[m] * quad_weight[m] * (I_edgV[iv(nx, i, m, g)] + eps);
          sum = sum + quad_weight[m] * (I_edgV[iv(nx, i, m, g)] + eps);
        }
        for (int m = 3 * nm / 4; m < nm; ++m) {
          C = C + Omega_x[m] * quad_weight[m] * (I_edgV[iv(nx, i, m, g)] + eps);
          sum = sum + quad_weight[m] * (I_edgV[iv(nx, i, m, g)] + eps);
        }
        C = C / sum;
      }
    }
    if (BC_Type[3] == 0) {
      for (int i = 0; i < nx; ++i) {
        double sum = 0.0, &C = Cg_T[i + (long)nx * g];
        for (int m = 0; m < nm / 2; ++m) {
          C = C + Omega_y[m] * quad_weight[m] * (I_edgH[ih(i, ny, m, g)] + eps);
          sum = sum + quad_weight[m] * (I_edgH[ih(i, ny, m, g)] + eps);
        }
        C = C / sum;
      }
    }
  }
  return 0;
}

// MGQD_In_Calc (MLOQD_SOLVES.f08:493-614).  Eg_in_L/R, Fg_in_L/R (ny,ng); Eg_in_B/T, Fg_in_B/T (nx,ng).
int oracle_mgqd_in_calc(int nx, int ny, int nm, int ng, double* Eg_in_L, double* Eg_in_B, double* Eg_in_R,
                        double* Eg_in_T, double* Fg_in_L, double* Fg_in_B, double* Fg_in_R, double* Fg_in_T,
                        const double* I_edgV, const double* I_edgH, const double* Omega_x,
                        const double* Omega_y, const double* quad_weight, double c, double Comp_Unit,
                        const int* BC_Type, int open_threads) {
  (void)Comp_Unit;
  const F4 iv{nx + 1L, ny, nm}, ih{nx, ny + 1L, nm};
  const int threads = team(open_threads, ng);
#pragma omp parallel for num_threads(threads) schedule(static)
  for (int g = 0; g < ng; ++g) {
    const long oy = (long)ny * g, ox = (long)nx * g;
    for (int i = 0; i < ny; ++i) Eg_in_L[i + oy] = Fg_in_L[i + oy] = Eg_in_R[i + oy] = Fg_in_R[i + oy] = 0.0;
    for (int i = 0; i < nx; ++i) Eg_in_B[i + ox] = Fg_in_B[i + ox] = Eg_in_T[i + ox] = Fg_in_T[i + ox] = 0.0;
    if (BC_Type[0] == 0) {
      for (int i = 0; i < ny; ++i) {
        for (int m = 0; m < nm / 4; ++m) {
          Fg_in_L[i + oy] = Fg_in_L[i + oy] + Omega_x[m] * quad_weight[m] * I_edgV[iv(0, i, m, g)];
          Eg_in_L[i + oy] = Eg_in_L[i + oy] + quad_weight[m] * I_edgV[iv(0, i, m, g)];
        }
        for (int m = 3 * nm / 4; m < nm; ++m) {
          Fg_in_L[i + oy] = Fg_in_L[i + oy] + Omega_x[m] * quad_weight[m] * I_edgV[iv(0, i, m, g)];
          Eg_in_L[i + oy] = Eg_in_L[i + oy] + quad_weight[m] * I_edgV[iv(0, i, m, g)];
        }
      }
    }
    if (BC_Type[1] == 0) {
      for (int i = 0; i < nx; ++i)
        for (int m = 0; m < nm / 2; ++m) {
          Fg_in_B[i + ox] = Fg_in_B[i + ox] + Omega_y[m] * quad_weight[m] * I_edgH[ih(i, 0, m, g)];
          Eg_in_B[i + ox] = Eg_in_B[i + ox] + quad_weight[m] * I_edgH[ih(i, 0, m, g)];
        }
    }
    if (BC_Type[2] == 0) {
      for (int i = 0; i < ny; ++i)
        for (int m = nm / 4; m < 3 * nm / 4; ++m) {
          Fg_in_R[i + oy] = Fg_in_R[i + oy] + Omega_x[m] * quad_weight[m] * I_edgV[iv(nx, i, m, g)];
          Eg_in_R[i + oy] = Eg_in_R[i + oy] + quad_weight[m] * I_edgV[iv(nx, i, m, g)];
        }
    }
    if (BC_Type[3] == 0) {
      for (int i = 0; i < nx; ++i)
        for (int m = nm / 2; m < nm; ++m) {
          Fg_in_T[i + ox] = Fg_in_T[i + ox] + Omega_y[m] * quad_weight[m] * I_edgH[ih(i, ny, m, g)];
          Eg_in_T[i + ox] = Eg_in_T[i + ox] + quad_weight[m] * I_edgH[ih(i, ny, m, g)];
        }
    }
    for (int i = 0; i < ny; ++i) {
      Eg_in_L[i + oy] = Eg_in_L[i + oy] / c;
      Eg_in_R[i + oy] = Eg_in_R[i + oy] / c;
    }
    for (int i = 0; i < nx; ++i) {
      Eg_in_B[i + ox] = Eg_in_B[i + ox] / c;
      Eg_in_T[i + ox] = Eg_in_T[i + ox] / c;
    }
  }
  return 0;
}

// GQD_In_Calc (GLOQD_SOLVES.f08:263-290).
int oracle_gqd_in_calc(int nx, int ny, int ng, double* E_in_L, double* E_in_B, double* E_in_R, double* E_in_T,
                       double* F_in_L, double* F_in_B, double* F_in_R, double* F_in_T, const double* Eg_in_L,
                       const double* Eg_in_B, const double* Eg_in_R, const double* Eg_in_T,
                       const double* Fg_in_L, const double* Fg_in_B, const double* Fg_in_R,
                       const double* Fg_in_T) {
  for (int i = 0; i < ny; ++i) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int g = 0; g < ng; ++g) {
      a = a + Eg_in_L[i + (long)ny * g];
      b = b + Eg_in_R[i + (long)ny * g];
      c = c + Fg_in_L[i + (long)ny * g];
      d = d + Fg_in_R[i + (long)ny * g];
    }
    E_in_L[i] = a;
    E_in_R[i] = b;
    F_in_L[i] = c;
    F_in_R[i] = d;
  }
  for (int i = 0; i < nx; ++i) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int g = 0; g < ng; ++g) {
      a = a + Eg_in_B[i + (long)nx * g];
      b = b + Eg_in_T[i + (long)nx * g];
      c = c + Fg_in_B[i + (long)nx * g];
      d = d + Fg_in_T[i + (long)nx * g];
    }
    E_in_B[i] = a;
    E_in_T[i] = b;
    F_in_B[i] = c;
    F_in_T[i] = d;
  }
  return 0;
}

// RT_BC_UPDATE (UPDATES.f08:12-105).  Nu_g has ng+1 edges.
int oracle_rt_bc_update(int nx, int ny, int nm, int ng, const int* BC_Type, double bcT_left, double bcT_lower,
                        double bcT_right, double bcT_upper, double Comp_Unit, const double* Nu_g,
                        double* I_edgV, double* I_edgH, double* Ic_edgV, double* Ic_edgH) {
  const F4 iv{nx + 1L, ny, nm}, ih{nx, ny + 1L, nm}, icv{nx + 1L, 2L * ny, nm}, ich{2L * nx, ny + 1L, nm};
  const int q = nm / 4;
  for (int g = 0; g < ng; ++g) {
    if (BC_Type[0] == 0) {
      double B = bg_planck(bcT_left, Nu_g[g], Nu_g[g + 1], Comp_Unit);
      for (int m = 0; m < nm; ++m) {
        if (!(m < q || m >= 3 * q)) continue;
        for (int j = 0; j < ny; ++j) I_edgV[iv(0, j, m, g)] = B;
        for (int j = 0; j < 2 * ny; ++j) Ic_edgV[icv(0, j, m, g)] = B;
      }
    } else if (BC_Type[0] == 1) {
      for (int m = 0; m < q; ++m) {
        for (int j = 0; j < ny; ++j) I_edgV[iv(0, j, m, g)] = I_edgV[iv(0, j, m + q, g)];
        for (int j = 0; j < 2 * ny; ++j) Ic_edgV[icv(0, j, m, g)] = Ic_edgV[icv(0, j, m + q, g)];
      }
      for (int m = 3 * q; m < nm; ++m) {
        for (int j = 0; j < ny; ++j) I_edgV[iv(0, j, m, g)] = I_edgV[iv(0, j, m - q, g)];
        for (int j = 0; j < 2 * ny; ++j) Ic_edgV[icv(0, j, m, g)] = Ic_edgV[icv(0, j, m - q, g)];
      }
    }
  }
  for (int g = 0; g < ng; ++g) {
    if (BC_Type[1] == 0) {
      double B = bg_planck(bcT_lower, Nu_g[g], Nu_g[g + 1], Comp_Unit);
      for (int m = 0; m < 2 * q; ++m) {
        for (int i = 0; i < nx; ++i) I_edgH[ih(i, 0, m, g)] = B;
        for (int i = 0; i < 2 * nx; ++i) Ic_edgH[ich(i, 0, m, g)] = B;
      }
    } else if (BC_Type[1] == 1) {
      for (int m = 0; m < q; ++m) {
        for (int i = 0; i < nx; ++i) I_edgH[ih(i, 0, m, g)] = I_edgH[ih(i, 0, m + 3 * q, g)];
        for (int i = 0; i < 2 * nx; ++i) Ic_edgH[ich(i, 0, m, g)] = Ic_edgH[ich(i, 0, m + 3 * q, g)];
      }
      for (int m = q; m < 2 * q; ++m) {
        for (int i = 0; i < nx; ++i) I_edgH[ih(i, 0, m, g)] = I_edgH[ih(i, 0, m + q, g)];
        for (int i = 0; i < 2 * nx; ++i) Ic_edgH[ich(i, 0, m, g)] = Ic_edgH[ich(i, 0, m + q, g)];
      }
    }
  }
  for (int g = 0; g < ng; ++g) {
    if (BC_Type[2] == 0) {
      double B = bg_planck(bcT_right, Nu_g[g], Nu_g[g + 1], Comp_Unit);
      for (int m = q; m < 3 * q; ++m) {
        for (int j = 0; j < ny; ++j) I_edgV[iv(nx, j, m, g)] = B;
        for (int j = 0; j < 2 * ny; ++j) Ic_edgV[icv(nx, j, m, g)] = B;
      }
    } else if (BC_Type[2] == 1) {
      for (int m = q; m < 2 * q; ++m) {
        for (int j = 0; j < ny; ++j) I_edgV[iv(nx, j, m, g)] = I_edgV[iv(nx, j, m - q, g)];
        for (int j = 0; j < 2 * ny; ++j) Ic_edgV[icv(nx, j, m, g)] = Ic_edgV[icv(nx, j, m - q, g)];
      }
      for (int m = 2 * q; m < 3 * q; ++m) {
        for (int j = 0; j < ny; ++j) I_edgV[iv(nx, j, m, g)] = I_edgV[iv(nx, j, m + q, g)];
        for (int j = 0; j < 2 * ny; ++j) Ic_edgV[icv(nx, j, m, g)] = Ic_edgV[icv(nx, j, m + q, g)];
      }
    }
  }
  for (int g = 0; g < ng; ++g) {
    if (BC_Type[3] == 0) {
      double B = bg_planck(bcT_upper, Nu_g[g], Nu_g[g + 1], Comp_Unit);
      for (int m = 2 * q; m < nm; ++m) {
        for (int i = 0; i < nx; ++i) I_edgH[ih(i, ny, m, g)] = B;
        for (int i = 0; i < 2 * nx; ++i) Ic_edgH[ich(i, ny, m, g)] = B;
      }
    } else if (BC_Type[3] == 1) {
      for (int m = 2 * q; m < 3 * q; ++m) {
        for (int i = 0; i < nx; ++i) I_edgH[ih(i, ny, m, g)] = I_edgH[ih(i, ny, m - q, g)];
        for (int i = 0; i < 2 * nx; ++i) Ic_edgH[ich(i, ny, m, g)] = Ic_edgH[ich(i, ny, m - q, g)];
      }
      for (int m = 3 * q; m < nm; ++m) {
        for (int i = 0; i < nx; ++i) I_edgH[ih(i, ny, m, g)] = I_edgH[ih(i, ny, m - 3 * q, g)];
        for (int i = 0; i < 2 * nx; ++i) Ic_edgH[ich(i, ny, m, g)] = Ic_edgH[ich(i, ny, m - 3 * q, g)];
      }
    }
  }
  return 0;
}

// MATERIAL_UPDATE (UPDATES.f08:110-152), the arrays the sweep and MEB_SOLVE read: per (i, j, g)
// Bg = Bg_planck_calc(T, nu_g, nu_g+1), KapE = KapB = kapB_calc(T, nu_g, nu_g+1) * kappa_mult(i,j)
// (kappa_mult = Kappa_Mult(Mat(i,j))) and the isotropic corner source src = KapB * Bg (RT_Src holds
// this value at every corner and direction).  Temp(nx,ny), Nu_g(ng+1); outputs (nx,ny,ng).
int oracle_material_update(int nx, int ny, int ng, const double* Temp, const double* Nu_g, const double* kappa_mult,
                           double Comp_Unit, double* KapE, double* src, double* Bg) {
  for (int g = 0; g < ng; ++g)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t c = (size_t)i + (size_t)nx * j, k = c + (size_t)nx * ny * g;
        const double B = bg_planck(Temp[c], Nu_g[g], Nu_g[g + 1], Comp_Unit);
        const double kB = oracle_kapb(Temp[c], Nu_g[g], Nu_g[g + 1]) * kappa_mult[c];
        if (Bg) Bg[k] = B;
        KapE[k] = kB;
        src[k] = kB * B;
      }
  return 0;
}

// MEB_SOLVE (UPDATES.f08:185-230) with cV per cell (the reference passes one value):
//   E = sum_g Eg_HO, KapE_Bar = (sum_g KapE*Eg_HO)/E,
//   Temp = c**2*h**3/(c**2*h**3*cv*Comp_Unit + 8*pi*Delt*Kap0/erg**4)*(Delt*c*KapE_Bar*E + cv*Temp_old)*Comp_Unit.
int oracle_meb_solve(int nx, int ny, int ng, double* Temp, const double* Eg_HO, const double* KapE,
                     const double* Temp_old, double Delt, const double* cV, double Kap0, double Comp_Unit) {
  const double pi = 4.0 * std::atan(1.0);
  const double c2h3 = (kC * kC) * ((kH * kH) * kH);
  const double e2 = kErg * kErg;
  const double lin = (((8.0 * pi) * Delt) * Kap0) / (e2 * e2);
  const size_t nxy = (size_t)nx * ny;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t c = (size_t)i + (size_t)nx * j;
      double E = 0.0, kb = 0.0;
      for (int g = 0; g < ng; ++g) {
        E = E + Eg_HO[c + nxy * g];
        kb = kb + KapE[c + nxy * g] * Eg_HO[c + nxy * g];
      }
      kb = kb / E;
      const double coef = c2h3 / (((c2h3 * cV[c]) * Comp_Unit) + lin);
      Temp[c] = (coef * ((((Delt * kC) * kb) * E) + cV[c] * Temp_old[c])) * Comp_Unit;
    }
  return 0;
}

// ---- Material of the synthetic configurations (not the reference's material) ---------------------
// The configurations replace kapB_calc with the opacity law
//   kappa_g(T) = kappa0(i,j) (1 - exp(-nu_g/T)) / (nu_g^3 sqrt(T)),  nu_g = sqrt(Nu_g(g) Nu_g(g+1)),
// T and nu in keV (Temp and Nu_g are passed in eV, as everywhere else), and the Fleck-Cummings
// MEB_SOLVE with a backward-Euler energy balance per cell,
//   cv (T - T_old)/Delt = sum_g KapE_g (c Eg - 4 pi Bg(T)),
// whose emission is linearised about the current iterate T* (one Newton step per outer iteration):
//   T = (cv T_old/Delt + sum_g KapE_g (c Eg - 4 pi Bg(T*) + 4 pi Bg'(T*) T*)) / (cv/Delt + 4 pi sum_g KapE_g Bg'(T*)).
// MATERIAL_UPDATE (UPDATES.f08:130-150) is the template: KapE = KapB, src = KapB * Bg.
double law_kappa(double Temp, double nu_low, double nu_high, double kappa0) {
  const double nb = std::sqrt(nu_low * nu_high) * 1e-3;
  const double tk = Temp * 1e-3;
  return kappa0 * (-std::expm1(-nb / tk)) / (((nb * nb) * nb) * std::sqrt(tk));
}

// dBg/dT of Bg_planck_calc: Bg = 2 T^4 (sigint(nu_h/T) - sigint(nu_l/T)) / K, with the exact derivative
// of the Planck integral, d sigint(z)/dz = z^3/(e^z - 1):
//   dBg/dT = 2 T^3 (4 (sigint(z_h) - sigint(z_l)) - z_h^4/(e^z_h - 1) + z_l^4/(e^z_l - 1)) / K.
double bg_planck_dT(double Tin, double nu_low, double nu_high, double comp_unit) {
  if (Tin <= 1e-15) return 0.0;
  const double zh = nu_high / Tin, zl = nu_low / Tin;
  const double s = sigint(zh) - sigint(zl);
  const double ph = zh > 700.0 ? 0.0 : (((zh * zh) * (zh * zh)) / std::expm1(zh));
  const double pl = zl > 700.0 ? 0.0 : (((zl * zl) * (zl * zl)) / std::expm1(zl));
  const double h3 = (kH * kH) * kH, c2 = kC * kC, e2 = kErg * kErg;
  const double K = ((h3 * c2) * (e2 * e2)) * comp_unit;
  const double t3 = (Tin * Tin) * Tin;
  return ((2.0 * t3) * (((4.0 * s) - ph) + pl)) / K;
}

int oracle_material_update_law(int nx, int ny, int ng, const double* Temp, const double* Nu_g, const double* kappa0,
                               double Comp_Unit, double* KapE, double* src, double* Bg) {
  for (int g = 0; g < ng; ++g)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t c = (size_t)i + (size_t)nx * j, k = c + (size_t)nx * ny * g;
        const double B = bg_planck(Temp[c], Nu_g[g], Nu_g[g + 1], Comp_Unit);
        const double kB = law_kappa(Temp[c], Nu_g[g], Nu_g[g + 1], kappa0[c]);
        if (Bg) Bg[k] = B;
        KapE[k] = kB;
        src[k] = kB * B;
      }
  return 0;
}

// Temp holds the current iterate T* on entry and the new temperature on return.
int oracle_meb_solve_law(int nx, int ny, int ng, double* Temp, const double* Eg_HO, const double* KapE,
                         const double* Temp_old, double Delt, const double* cV, const double* Nu_g, double Comp_Unit,
                         double c) {
  const double fp = 4.0 * (4.0 * std::atan(1.0));
  const size_t nxy = (size_t)nx * ny;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t k = (size_t)i + (size_t)nx * j;
      const double ts = Temp[k];
      double num = 0.0, den = 0.0;
      for (int g = 0; g < ng; ++g) {
        const double kap = KapE[k + nxy * g];
        const double B = bg_planck(ts, Nu_g[g], Nu_g[g + 1], Comp_Unit);
        const double dB = bg_planck_dT(ts, Nu_g[g], Nu_g[g + 1], Comp_Unit);
        num = num + kap * (((c * Eg_HO[k + nxy * g]) - (fp * B)) + ((fp * dB) * ts));
        den = den + (fp * kap) * dB;
      }
      Temp[k] = (((cV[k] * Temp_old[k]) / Delt) + num) / ((cV[k] / Delt) + den);
    }
  return 0;
}

// The energy balances split over group ranges (the device's trt_tstep_partials / trt_tstep_finish):
// per cell the group sums over groups [g0, g1) of the arrays (nx, ny, ng) ...
//   law 0 (MEB_SOLVE): {sum KapE Eg, sum Eg, sum Eg};  law 1: {sum KapE (c Eg - 4 pi Bg + 4 pi Bg' T*),
//   sum 4 pi KapE Bg', sum Eg}   -> part (3, nx, ny)
// ... and the temperature from the sums over all ranges (and E_avg = the summed transport E).
int oracle_meb_partial(int nx, int ny, int ng, int g0, int g1, int law, const double* Eg_HO, const double* KapE,
                       const double* Temp, const double* Nu_g, double Comp_Unit, double c, double* part) {
  (void)ng;
  const double fp = 4.0 * (4.0 * std::atan(1.0));
  const size_t nxy = (size_t)nx * ny;
  for (size_t k = 0; k < nxy; ++k) {
    double p0 = 0.0, p1 = 0.0, p2 = 0.0;
    const double ts = Temp[k];
    for (int g = g0; g < g1; ++g) {
      const double e = Eg_HO[k + nxy * g], kap = KapE[k + nxy * g];
      if (law == 1) {
        const double B = bg_planck(ts, Nu_g[g], Nu_g[g + 1], Comp_Unit);
        const double dB = bg_planck_dT(ts, Nu_g[g], Nu_g[g + 1], Comp_Unit);
        p0 = p0 + kap * (((c * e) - (fp * B)) + ((fp * dB) * ts));
        p1 = p1 + (fp * kap) * dB;
      } else {
        p0 = p0 + kap * e;
        p1 = p1 + e;
      }
      p2 = p2 + e;
    }
    part[k] = p0;
    part[k + nxy] = p1;
    part[k + 2 * nxy] = p2;
  }
  return 0;
}

int oracle_meb_finish(int nx, int ny, int law, const double* sum, const double* Temp_old, const double* cV,
                      double Delt, double Kap0, double Comp_Unit, double* Temp, double* E_avg) {
  const double pi = 4.0 * std::atan(1.0);
  const double c2h3 = (kC * kC) * ((kH * kH) * kH);
  const double e2 = kErg * kErg;
  const double lin = (((8.0 * pi) * Delt) * Kap0) / (e2 * e2);
  const size_t nxy = (size_t)nx * ny;
  for (size_t k = 0; k < nxy; ++k) {
    const double p0 = sum[k], p1 = sum[k + nxy];
    if (law == 1) {
      Temp[k] = (((cV[k] * Temp_old[k]) / Delt) + p0) / ((cV[k] / Delt) + p1);
    } else {
      const double kb = p0 / p1;
      const double coef = c2h3 / (((c2h3 * cV[k]) * Comp_Unit) + lin);
      Temp[k] = (coef * ((((Delt * kC) * kb) * p1) + cV[k] * Temp_old[k])) * Comp_Unit;
    }
    E_avg[k] = sum[k + 2 * nxy];
  }
  return 0;
}

// CONVERGENCE (CONVERGENCE_CHECKS.f08:7-44) of a field of n values; returns 1 when converged.
int oracle_convergence(int conv_type, double eps, const double* x, const double* x_old, const double* x_old2, int n,
                       int its, double* norm, double* rho) {
  double d0 = 0.0, d1 = 0.0, mx = 0.0, mn = HUGE_VAL, r2 = 0.0;
  for (int k = 0; k < n; ++k) {
    d0 = std::max(d0, std::fabs(x[k] - x_old[k]));
    d1 = std::max(d1, std::fabs(x_old[k] - x_old2[k]));
    mx = std::max(mx, std::fabs(x[k]));
    mn = std::min(mn, std::fabs(x[k]));
    r2 = std::max(r2, std::fabs(1.0 - x_old[k] / x[k]));
  }
  const double r = its > 1 ? d0 / d1 : 2.0;
  double nrm;
  if (conv_type == 1) nrm = d0 / mx;
  else if (conv_type == 2) nrm = r2;
  else nrm = d0 / mn;
  if (norm) *norm = nrm;
  if (rho) *rho = r;
  const double new_eps = std::fabs(1.0 / r - 1.0) * eps;
  return nrm > new_eps ? 0 : 1;
}

int oracle_openmp_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
