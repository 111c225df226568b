// CPU oracle for the multigroup low-order quasidiffusion (MGQD) solve.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, its C-ABI or the Python
// package) links, loads or calls this file; only tests/ and the CPU-baseline leg of bench.py do, as
// the checker.
//
// Restates, in C++17 with the reference's Fortran column-major layouts and loop orders:
//   OLD_MGQD_COEFS   MainSrc/MLOQD_SOLVES.f08:12-73     -> oracle_old_mgqd_coefs
//   MLOQD_FV         MainSrc/MLOQD_SOLVES.f08:78-362    -> oracle_mloqd_fv
//   QD_FV equations  MainSrc/QD_SOLVERS.f08:40-386      -> assemble_group (rows of the reduced system)
//
// Linear solve.  The reference assembles the reduced system of each group in CSR (QD_SOLVERS.f08:66-386)
// and solves it with SPARSKIT2's ILUT(fill 3, drop 1e-6) preconditioned BiCGSTAB, relative tolerance
// 1e-13 and absolute 1e-15 (QD_SOLVERS.f08:415-470), falling back to dense GAUSS_COMPLETE when the
// iteration fails (:489-497).  SPARSKIT2 is not vendored in the reference tree.  The oracle solves the
// same equations directly, by banded LU with partial pivoting over a row-by-row numbering of the
// unknowns (its own numbering: the solution does not depend on it), and so returns the discrete
// solution that the reference's iteration converges to.  MGQD_Kits is -1 for every group, the value
// the reference records when it solves directly.
//
// Parity status: UNPINNED (no reference outputs exist for this path).  The oracle is checked instead
// through the reference's own residual formulas (MLOQD_SOLVES.f08:277-345), which are written on the
// un-reduced equations and so test the reduction, the assembly and the flux recovery together.
#include <algorithm>
#include <cmath>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct Idx2 {
  long n1;
  long operator()(long i, long j) const { return i + n1 * j; }
};
struct Idx3 {
  long n1, n2;
  long operator()(long i, long j, long k) const { return i + n1 * (j + n2 * k); }
};

// Band matrix with partial-pivoting room: row r stores columns r-kl .. r+kl+ku.
struct Band {
  long n, kl, ku, w;
  std::vector<double> a;
  Band(long n_, long kl_, long ku_) : n(n_), kl(kl_), ku(ku_), w(2 * kl_ + ku_ + 1), a((size_t)n_ * w, 0.0) {}
  double& at(long r, long c) { return a[(size_t)r * w + (c - r + kl)]; }
};

// Gaussian elimination with partial (row) pivoting on the band, then back substitution; b is
// overwritten with the solution.  Returns false on a zero pivot.
bool band_solve(Band& B, std::vector<double>& b) {
  const long n = B.n, kl = B.kl, ku = B.ku;
  for (long k = 0; k < n; ++k) {
    const long last = std::min(n - 1, k + kl);
    long p = k;
    double best = std::fabs(B.at(k, k));
    for (long r = k + 1; r <= last; ++r)
      if (std::fabs(B.at(r, k)) > best) {
        best = std::fabs(B.at(r, k));
        p = r;
      }
    if (best == 0.0) return false;
    const long cend = std::min(n - 1, k + kl + ku);
    if (p != k) {
      for (long c = k; c <= cend; ++c) std::swap(B.at(k, c), B.at(p, c));
      std::swap(b[k], b[p]);
    }
    const double piv = B.at(k, k);
    for (long r = k + 1; r <= last; ++r) {
      const double l = B.at(r, k) / piv;
      if (l == 0.0) continue;
      B.at(r, k) = 0.0;
      for (long c = k + 1; c <= cend; ++c) B.at(r, c) -= l * B.at(k, c);
      b[r] -= l * b[k];
    }
  }
  for (long k = n - 1; k >= 0; --k) {
    double s = b[k];
    const long cend = std::min(n - 1, k + kl + ku);
    for (long c = k + 1; c <= cend; ++c) s -= B.at(k, c) * b[c];
    b[k] = s / B.at(k, k);
  }
  return true;
}

// Unknown numbering of one group: row block j (0..ny-1) holds the bottom edges E_edgH(0..nx-1, j),
// then E_edgV(0, j), and per cell i the pair E_avg(i, j), E_edgV(i+1, j); the top edges
// E_edgH(0..nx-1, ny) close the vector.  Equation rows use the same numbers (energy balance on the
// cell's number, x-momentum/boundary condition on the vertical edge's, y-momentum/boundary condition on
// the horizontal edge's).
struct Numbering {
  long nx, ny, blk;
  Numbering(long nx_, long ny_) : nx(nx_), ny(ny_), blk(3 * nx_ + 1) {}
  long n() const { return ny * blk + nx; }
  long H(long i, long j) const { return j * blk + i; }
  long V(long i, long j) const { return j * blk + nx + 2 * i; }
  long C(long i, long j) const { return j * blk + nx + 2 * i + 1; }
};

}  // namespace

extern "C" {

// OLD_MGQD_COEFS (MLOQD_SOLVES.f08:12-73).  Cell arrays (nx,ny,ng); V-edge arrays (nx+1,ny,ng);
// H-edge arrays (nx,ny+1,ng).
int oracle_old_mgqd_coefs(int nx, int ny, int ng, const double* Eg_avg_old, const double* Eg_edgV_old,
                          const double* Eg_edgH_old, const double* Fxg_edgV_old, const double* Fyg_edgH_old,
                          const double* fg_avg_xx_old, const double* fg_avg_yy_old, const double* fg_edgV_xx_old,
                          const double* fg_edgV_xy_old, const double* fg_edgH_yy_old, const double* fg_edgH_xy_old,
                          const double* KapE_old, const double* KapR_old, const double* Src_old, const double* Delx,
                          const double* Dely, const double* A, double c, double Delt, double Theta, double* G_old,
                          double* Pold_L, double* Pold_B, double* Pold_R, double* Pold_T) {
  (void)Delt;
  if (nx < 1 || ny < 1 || ng < 1) return -1;
  const Idx3 C{nx, ny}, V{nx + 1, ny}, H{nx, ny + 1};
  const Idx2 A2{nx};
  const double w = (Theta - 1.0) / Theta;
#pragma omp parallel for schedule(static)
  for (int g = 0; g < ng; ++g)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = C(i, j, g);
        G_old[k] = w * (Dely[j] * (Fxg_edgV_old[V(i + 1, j, g)] - Fxg_edgV_old[V(i, j, g)]) +
                        Delx[i] * (Fyg_edgH_old[H(i, j + 1, g)] - Fyg_edgH_old[H(i, j, g)]) +
                        A[A2(i, j)] * (c * KapE_old[k] * Eg_avg_old[k] - Src_old[k]));
        Pold_L[k] = w * (c * Dely[j] *
                             (fg_avg_xx_old[k] * Eg_avg_old[k] - fg_edgV_xx_old[V(i, j, g)] * Eg_edgV_old[V(i, j, g)]) +
                         c * Delx[i] *
                             (fg_edgH_xy_old[H(i, j + 1, g)] * Eg_edgH_old[H(i, j + 1, g)] -
                              fg_edgH_xy_old[H(i, j, g)] * Eg_edgH_old[H(i, j, g)]) / 2.0 +
                         A[A2(i, j)] * (KapR_old[k] * Fxg_edgV_old[V(i, j, g)]) / 2.0);
        Pold_B[k] = w * (c * Delx[i] *
                             (fg_avg_yy_old[k] * Eg_avg_old[k] - fg_edgH_yy_old[H(i, j, g)] * Eg_edgH_old[H(i, j, g)]) +
                         c * Dely[j] *
                             (fg_edgV_xy_old[V(i + 1, j, g)] * Eg_edgV_old[V(i + 1, j, g)] -
                              fg_edgV_xy_old[V(i, j, g)] * Eg_edgV_old[V(i, j, g)]) / 2.0 +
                         A[A2(i, j)] * (KapR_old[k] * Fyg_edgH_old[H(i, j, g)]) / 2.0);
        Pold_R[k] = w * (c * Dely[j] *
                             (fg_edgV_xx_old[V(i + 1, j, g)] * Eg_edgV_old[V(i + 1, j, g)] - fg_avg_xx_old[k] * Eg_avg_old[k]) +
                         c * Delx[i] *
                             (fg_edgH_xy_old[H(i, j + 1, g)] * Eg_edgH_old[H(i, j + 1, g)] -
                              fg_edgH_xy_old[H(i, j, g)] * Eg_edgH_old[H(i, j, g)]) / 2.0 +
                         A[A2(i, j)] * (KapR_old[k] * Fxg_edgV_old[V(i + 1, j, g)]) / 2.0);
        Pold_T[k] = w * (c * Delx[i] *
                             (fg_edgH_yy_old[H(i, j + 1, g)] * Eg_edgH_old[H(i, j + 1, g)] - fg_avg_yy_old[k] * Eg_avg_old[k]) +
                         c * Dely[j] *
                             (fg_edgV_xy_old[V(i + 1, j, g)] * Eg_edgV_old[V(i + 1, j, g)] -
                              fg_edgV_xy_old[V(i, j, g)] * Eg_edgV_old[V(i, j, g)]) / 2.0 +
                         A[A2(i, j)] * (KapR_old[k] * Fyg_edgH_old[H(i, j + 1, g)]) / 2.0);
      }
  return 0;
}

// MLOQD_FV (MLOQD_SOLVES.f08:78-362), arguments in the subroutine's order after the extents.
// Boundary arrays: Cg_L/Cg_R, Eg_in_L/R, Fg_in_L/R (ny,ng); Cg_B/Cg_T, Eg_in_B/T, Fg_in_B/T (nx,ng).
// MGQD_Residual(ng,5,5), MGQD_BC_Residual(ng,4), MGQD_Kits(ng).  Eg_avg/Eg_edgV/Eg_edgH are in/out (the
// reference uses them as the initial guess; a direct solve does not need one).  Returns 0, or -2 when
// a group's system is singular.
int oracle_mloqd_fv(int nx, int ny, int ng, double* Eg_avg, double* Eg_edgV, double* Eg_edgH, double* Fxg_edgV,
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
                    double Ein_Weight) {
  if (nx < 1 || ny < 1 || ng < 1) return -1;
  const Idx3 C{nx, ny}, V{nx + 1, ny}, H{nx, ny + 1};
  const Idx2 A2{nx}, P2{nx}, Bx{nx}, By{ny};
  int threads = Open_Threads > 0 ? std::min(Open_Threads, ng) : 1;
  int bad = 0;
#pragma omp parallel for schedule(dynamic) num_threads(threads) reduction(+ : bad)
  for (int g = 0; g < ng; ++g) {
    const size_t ncell = (size_t)nx * ny;
    std::vector<double> Xi(ncell), Ghat(ncell), PhL(ncell), PhB(ncell), PhR(ncell), PhT(ncell);
    std::vector<double> EBL(ncell), EBB(ncell), EBC(ncell), EBR(ncell), EBT(ncell);
    std::vector<double> MxC(ncell), MxT(ncell), MxB(ncell), MyC(ncell), MyR(ncell), MyL(ncell);
    std::vector<double> MxR(ncell), MyT(ncell), MxRHS(ncell), MyRHS(ncell);
    std::vector<double> CpL(ny), CpR(ny), BCL(ny), BCR(ny), CpB(nx), CpT(nx), BCB(nx), BCT(nx);
    // coefficients, MLOQD_SOLVES.f08:148-220
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = P2(i, j), kg = C(i, j, g);
        const double a = A[A2(i, j)];
        Xi[k] = a * (Fdt_Weight / (Theta * c * Delt) + KapR[kg]) / 2.0;
        PhL[k] = (Fdt_Weight * a * Fxg_edgV_old[V(i, j, g)] / (2.0 * Theta * c * Delt) + Pold_L[kg]) / Xi[k];
        PhB[k] = (Fdt_Weight * a * Fyg_edgH_old[H(i, j, g)] / (2.0 * Theta * c * Delt) + Pold_B[kg]) / Xi[k];
        PhR[k] = (Fdt_Weight * a * Fxg_edgV_old[V(i + 1, j, g)] / (2.0 * Theta * c * Delt) + Pold_R[kg]) / Xi[k];
        PhT[k] = (Fdt_Weight * a * Fyg_edgH_old[H(i, j + 1, g)] / (2.0 * Theta * c * Delt) + Pold_T[kg]) / Xi[k];
        Ghat[k] = a * Src[kg] + a * Eg_avg_old[kg] / (Theta * Delt) + G_old[kg] + Dely[j] * (PhL[k] - PhR[k]) +
                  Delx[i] * (PhB[k] - PhT[k]);
      }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = P2(i, j), kg = C(i, j, g);
        const double a = A[A2(i, j)], dx = Delx[i], dy = Dely[j];
        EBC[k] = (a * (1.0 / (Theta * Delt) + c * KapE[kg]) + 2.0 * c * (dy * dy) * fg_avg_xx[kg] / Xi[k] +
                  2.0 * c * (dx * dx) * fg_avg_yy[kg] / Xi[k]);
        EBR[k] = -c * (dy * dy) * fg_edgV_xx[V(i + 1, j, g)] / Xi[k];
        EBL[k] = -c * (dy * dy) * fg_edgV_xx[V(i, j, g)] / Xi[k];
        EBT[k] = -c * (dx * dx) * fg_edgH_yy[H(i, j + 1, g)] / Xi[k];
        EBB[k] = -c * (dx * dx) * fg_edgH_yy[H(i, j, g)] / Xi[k];
        MxC[k] = c * dy * fg_avg_xx[kg] / Xi[k];
        MxT[k] = -c * dx * fg_edgH_xy[H(i, j + 1, g)] / (2.0 * Xi[k]);
        MxB[k] = c * dx * fg_edgH_xy[H(i, j, g)] / (2.0 * Xi[k]);
        MyC[k] = c * dx * fg_avg_yy[kg] / Xi[k];
        MyR[k] = -c * dy * fg_edgV_xy[V(i + 1, j, g)] / (2.0 * Xi[k]);
        MyL[k] = c * dy * fg_edgV_xy[V(i, j, g)] / (2.0 * Xi[k]);
      }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i + 1 < nx; ++i)
        MxR[P2(i, j)] = -(c * Dely[j] / Xi[P2(i, j)] + c * Dely[j] / Xi[P2(i + 1, j)]) * fg_edgV_xx[V(i + 1, j, g)];
    for (int j = 0; j + 1 < ny; ++j)
      for (int i = 0; i < nx; ++i)
        MyT[P2(i, j)] = -(c * Delx[i] / Xi[P2(i, j)] + c * Delx[i] / Xi[P2(i, j + 1)]) * fg_edgH_yy[H(i, j + 1, g)];
    for (int j = 0; j < ny; ++j) {
      CpL[j] = c * Cg_L[By(j, g)] - c * Dely[j] * fg_edgV_xx[V(0, j, g)] / Xi[P2(0, j)];
      CpR[j] = c * Cg_R[By(j, g)] + c * Dely[j] * fg_edgV_xx[V(nx, j, g)] / Xi[P2(nx - 1, j)];
      BCL[j] = Ein_Weight * c * Cg_L[By(j, g)] * Eg_in_L[By(j, g)] - Fin_Weight * Fg_in_L[By(j, g)] + PhL[P2(0, j)];
      BCR[j] = Ein_Weight * c * Cg_R[By(j, g)] * Eg_in_R[By(j, g)] - Fin_Weight * Fg_in_R[By(j, g)] +
               PhR[P2(nx - 1, j)];
    }
    for (int i = 0; i < nx; ++i) {
      CpB[i] = c * Cg_B[Bx(i, g)] - c * Delx[i] * fg_edgH_yy[H(i, 0, g)] / Xi[P2(i, 0)];
      CpT[i] = c * Cg_T[Bx(i, g)] + c * Delx[i] * fg_edgH_yy[H(i, ny, g)] / Xi[P2(i, ny - 1)];
      BCB[i] = Ein_Weight * c * Cg_B[Bx(i, g)] * Eg_in_B[Bx(i, g)] - Fin_Weight * Fg_in_B[Bx(i, g)] + PhB[P2(i, 0)];
      BCT[i] = Ein_Weight * c * Cg_T[Bx(i, g)] * Eg_in_T[Bx(i, g)] - Fin_Weight * Fg_in_T[Bx(i, g)] +
               PhT[P2(i, ny - 1)];
    }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (i != nx - 1) MxRHS[P2(i, j)] = PhL[P2(i + 1, j)] - PhR[P2(i, j)];
        if (j != ny - 1) MyRHS[P2(i, j)] = PhB[P2(i, j + 1)] - PhT[P2(i, j)];
      }

    // the reduced system (QD_SOLVERS.f08:66-386), one row per unknown
    const Numbering N(nx, ny);
    const long n = N.n();
    struct Ent {
      long r, c;
      double v;
    };
    std::vector<Ent> ent;
    ent.reserve((size_t)19 * nx * ny + nx + ny);
    std::vector<double> rhs(n, 0.0);
    auto put = [&](long r, long col, double v) {
      if (v != 0.0) ent.push_back({r, col, v});
    };
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = P2(i, j);
        // radiation energy balance
        long r = N.C(i, j);
        rhs[r] = Ghat[k];
        put(r, N.V(i, j), EBL[k]);
        put(r, N.H(i, j), EBB[k]);
        put(r, N.C(i, j), EBC[k]);
        put(r, N.V(i + 1, j), EBR[k]);
        put(r, N.H(i, j + 1), EBT[k]);
        // left boundary condition
        if (i == 0) {
          r = N.V(0, j);
          rhs[r] = BCL[j];
          put(r, N.V(0, j), CpL[j]);
          put(r, N.H(0, j), -MxB[k]);
          put(r, N.C(0, j), MxC[k]);
          put(r, N.H(0, j + 1), -MxT[k]);
        }
        // x-momentum balance across the right edge, or the right boundary condition
        r = N.V(i + 1, j);
        if (i != nx - 1) {
          const long kr = P2(i + 1, j);
          rhs[r] = MxRHS[k];
          put(r, N.H(i, j), MxB[k]);
          put(r, N.C(i, j), MxC[k]);
          put(r, N.V(i + 1, j), MxR[k]);
          put(r, N.H(i, j + 1), MxT[k]);
          put(r, N.H(i + 1, j), -MxB[kr]);
          put(r, N.C(i + 1, j), MxC[kr]);
          put(r, N.H(i + 1, j + 1), -MxT[kr]);
        } else {
          rhs[r] = BCR[j];
          put(r, N.H(i, j), -MxB[k]);
          put(r, N.C(i, j), -MxC[k]);
          put(r, N.V(i + 1, j), CpR[j]);
          put(r, N.H(i, j + 1), -MxT[k]);
        }
        // bottom boundary condition
        if (j == 0) {
          r = N.H(i, 0);
          rhs[r] = BCB[i];
          put(r, N.V(i, 0), -MyL[k]);
          put(r, N.H(i, 0), CpB[i]);
          put(r, N.C(i, 0), MyC[k]);
          put(r, N.V(i + 1, 0), -MyR[k]);
        }
        // y-momentum balance across the top edge, or the top boundary condition
        r = N.H(i, j + 1);
        if (j != ny - 1) {
          const long kt = P2(i, j + 1);
          rhs[r] = MyRHS[k];
          put(r, N.V(i, j), MyL[k]);
          put(r, N.C(i, j), MyC[k]);
          put(r, N.V(i + 1, j), MyR[k]);
          put(r, N.H(i, j + 1), MyT[k]);
          put(r, N.V(i, j + 1), -MyL[kt]);
          put(r, N.C(i, j + 1), MyC[kt]);
          put(r, N.V(i + 1, j + 1), -MyR[kt]);
        } else {
          rhs[r] = BCT[i];
          put(r, N.V(i, j), -MyL[k]);
          put(r, N.C(i, j), -MyC[k]);
          put(r, N.V(i + 1, j), -MyR[k]);
          put(r, N.H(i, j + 1), CpT[i]);
        }
      }
    long kl = 0, ku = 0;
    for (const Ent& e : ent) {
      kl = std::max(kl, e.r - e.c);
      ku = std::max(ku, e.c - e.r);
    }
    Band B(n, kl, ku);
    for (const Ent& e : ent) B.at(e.r, e.c) += e.v;
    if (!band_solve(B, rhs)) {
      bad += 1;
      continue;
    }
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        Eg_avg[C(i, j, g)] = rhs[N.C(i, j)];
        Eg_edgH[H(i, j, g)] = rhs[N.H(i, j)];
      }
      for (int i = 0; i <= nx; ++i) Eg_edgV[V(i, j, g)] = rhs[N.V(i, j)];
    }
    for (int i = 0; i < nx; ++i) Eg_edgH[H(i, ny, g)] = rhs[N.H(i, ny)];
    MGQD_Kits[g] = -1;

    // fluxes from the auxiliary equations, MLOQD_SOLVES.f08:244-268
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        const long k = P2(i, j), kg = C(i, j, g);
        Fxg_edgV[V(i, j, g)] =
            -(c * Dely[j] / (Xi[k])) * (fg_avg_xx[kg] * Eg_avg[kg] - fg_edgV_xx[V(i, j, g)] * Eg_edgV[V(i, j, g)]) -
            (c * Delx[i] / (2.0 * Xi[k])) *
                (fg_edgH_xy[H(i, j + 1, g)] * Eg_edgH[H(i, j + 1, g)] - fg_edgH_xy[H(i, j, g)] * Eg_edgH[H(i, j, g)]) +
            PhL[k];
        Fyg_edgH[H(i, j, g)] =
            -(c * Delx[i] / (Xi[k])) * (fg_avg_yy[kg] * Eg_avg[kg] - fg_edgH_yy[H(i, j, g)] * Eg_edgH[H(i, j, g)]) -
            (c * Dely[j] / (2.0 * Xi[k])) *
                (fg_edgV_xy[V(i + 1, j, g)] * Eg_edgV[V(i + 1, j, g)] - fg_edgV_xy[V(i, j, g)] * Eg_edgV[V(i, j, g)]) +
            PhB[k];
      }
      const int i = nx - 1;
      const long k = P2(i, j), kg = C(i, j, g);
      Fxg_edgV[V(nx, j, g)] =
          -(c * Dely[j] / (Xi[k])) * (fg_edgV_xx[V(nx, j, g)] * Eg_edgV[V(nx, j, g)] - fg_avg_xx[kg] * Eg_avg[kg]) -
          (c * Delx[i] / (2.0 * Xi[k])) *
              (fg_edgH_xy[H(i, j + 1, g)] * Eg_edgH[H(i, j + 1, g)] - fg_edgH_xy[H(i, j, g)] * Eg_edgH[H(i, j, g)]) +
          PhR[k];
    }
    for (int i = 0; i < nx; ++i) {
      const int j = ny - 1;
      const long k = P2(i, j), kg = C(i, j, g);
      Fyg_edgH[H(i, ny, g)] =
          -(c * Delx[i] / (Xi[k])) * (fg_edgH_yy[H(i, ny, g)] * Eg_edgH[H(i, ny, g)] - fg_avg_yy[kg] * Eg_avg[kg]) -
          (c * Dely[j] / (2.0 * Xi[k])) *
              (fg_edgV_xy[V(i + 1, j, g)] * Eg_edgV[V(i + 1, j, g)] - fg_edgV_xy[V(i, j, g)] * Eg_edgV[V(i, j, g)]) +
          PhT[k];
    }
  }
  if (bad) return -2;

  // residuals, MLOQD_SOLVES.f08:277-345: MGQD_Residual(g,k,m) and MGQD_BC_Residual(g,side)
  if (Res_Calc) {
    const Idx3 R{ng, 5};
    const Idx2 RB{ng};
    for (long q = 0; q < (long)ng * 25; ++q) MGQD_Residual[q] = 0.0;
    for (long q = 0; q < (long)ng * 4; ++q) MGQD_BC_Residual[q] = 0.0;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int g = 0; g < ng; ++g) {
      double res[5];
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const long kg = C(i, j, g);
          const double a = A[A2(i, j)];
          res[0] = std::fabs(a * (1.0 / (Theta * Delt) + c * KapE[kg]) * Eg_avg[kg] +
                             Dely[j] * (Fxg_edgV[V(i + 1, j, g)] - Fxg_edgV[V(i, j, g)]) +
                             Delx[i] * (Fyg_edgH[H(i, j + 1, g)] - Fyg_edgH[H(i, j, g)]) -
                             (a * Src[kg] + a * Eg_avg_old[kg] / (Theta * Delt) + G_old[kg]));
          res[1] = std::fabs(a * (1.0 / (Theta * c * Delt) + KapR[kg]) * Fxg_edgV[V(i, j, g)] / 2.0 +
                             c * Dely[j] * (fg_avg_xx[kg] * Eg_avg[kg] - fg_edgV_xx[V(i, j, g)] * Eg_edgV[V(i, j, g)]) +
                             c * Delx[i] *
                                 (fg_edgH_xy[H(i, j + 1, g)] * Eg_edgH[H(i, j + 1, g)] -
                                  fg_edgH_xy[H(i, j, g)] * Eg_edgH[H(i, j, g)]) / 2.0 -
                             (a * Fxg_edgV_old[V(i, j, g)] / (2.0 * Theta * c * Delt) + Pold_L[kg]));
          res[2] = std::fabs(a * (1.0 / (Theta * c * Delt) + KapR[kg]) * Fyg_edgH[H(i, j, g)] / 2.0 +
                             c * Delx[i] * (fg_avg_yy[kg] * Eg_avg[kg] - fg_edgH_yy[H(i, j, g)] * Eg_edgH[H(i, j, g)]) +
                             c * Dely[j] *
                                 (fg_edgV_xy[V(i + 1, j, g)] * Eg_edgV[V(i + 1, j, g)] -
                                  fg_edgV_xy[V(i, j, g)] * Eg_edgV[V(i, j, g)]) / 2.0 -
                             (a * Fyg_edgH_old[H(i, j, g)] / (2.0 * Theta * c * Delt) + Pold_B[kg]));
          res[3] = std::fabs(a * (1.0 / (Theta * c * Delt) + KapR[kg]) * Fxg_edgV[V(i + 1, j, g)] / 2.0 +
                             c * Dely[j] *
                                 (fg_edgV_xx[V(i + 1, j, g)] * Eg_edgV[V(i + 1, j, g)] - fg_avg_xx[kg] * Eg_avg[kg]) +
                             c * Delx[i] *
                                 (fg_edgH_xy[H(i, j + 1, g)] * Eg_edgH[H(i, j + 1, g)] -
                                  fg_edgH_xy[H(i, j, g)] * Eg_edgH[H(i, j, g)]) / 2.0 -
                             (a * Fxg_edgV_old[V(i + 1, j, g)] / (2.0 * Theta * c * Delt) + Pold_R[kg]));
          res[4] = std::fabs(a * (1.0 / (Theta * c * Delt) + KapR[kg]) * Fyg_edgH[H(i, j + 1, g)] / 2.0 +
                             c * Delx[i] *
                                 (fg_edgH_yy[H(i, j + 1, g)] * Eg_edgH[H(i, j + 1, g)] - fg_avg_yy[kg] * Eg_avg[kg]) +
                             c * Dely[j] *
                                 (fg_edgV_xy[V(i + 1, j, g)] * Eg_edgV[V(i + 1, j, g)] -
                                  fg_edgV_xy[V(i, j, g)] * Eg_edgV[V(i, j, g)]) / 2.0 -
                             (a * Fyg_edgH_old[H(i, j + 1, g)] / (2.0 * Theta * c * Delt) + Pold_T[kg]));
          for (int k = 0; k < 5; ++k) {
            if (res[k] > MGQD_Residual[R(g, k, 0)]) MGQD_Residual[R(g, k, 0)] = res[k];
            MGQD_Residual[R(g, k, 1)] += res[k];
            MGQD_Residual[R(g, k, 2)] += res[k] * res[k];
            MGQD_Residual[R(g, k, 3)] += a * res[k];
            MGQD_Residual[R(g, k, 4)] += a * (res[k] * res[k]);
          }
        }
      for (int k = 0; k < 5; ++k) {
        MGQD_Residual[R(g, k, 2)] = std::sqrt(MGQD_Residual[R(g, k, 2)]);
        MGQD_Residual[R(g, k, 4)] = std::sqrt(MGQD_Residual[R(g, k, 4)]);
      }
      for (int j = 0; j < ny; ++j) {
        double r1 = std::fabs(Fxg_edgV[V(0, j, g)] - c * Cg_L[By(j, g)] * (Eg_edgV[V(0, j, g)] - Eg_in_L[By(j, g)]) -
                              Fg_in_L[By(j, g)]);
        if (r1 > MGQD_BC_Residual[RB(g, 0)]) MGQD_BC_Residual[RB(g, 0)] = r1;
        r1 = std::fabs(Fxg_edgV[V(nx, j, g)] - c * Cg_R[By(j, g)] * (Eg_edgV[V(nx, j, g)] - Eg_in_R[By(j, g)]) -
                       Fg_in_R[By(j, g)]);
        if (r1 > MGQD_BC_Residual[RB(g, 2)]) MGQD_BC_Residual[RB(g, 2)] = r1;
      }
      for (int i = 0; i < nx; ++i) {
        double r1 = std::fabs(Fyg_edgH[H(i, 0, g)] - c * Cg_B[Bx(i, g)] * (Eg_edgH[H(i, 0, g)] - Eg_in_B[Bx(i, g)]) -
                              Fg_in_B[Bx(i, g)]);
        if (r1 > MGQD_BC_Residual[RB(g, 1)]) MGQD_BC_Residual[RB(g, 1)] = r1;
        r1 = std::fabs(Fyg_edgH[H(i, ny, g)] - c * Cg_T[Bx(i, g)] * (Eg_edgH[H(i, ny, g)] - Eg_in_T[Bx(i, g)]) -
                       Fg_in_T[Bx(i, g)]);
        if (r1 > MGQD_BC_Residual[RB(g, 3)]) MGQD_BC_Residual[RB(g, 3)] = r1;
      }
    }
  }
  return 0;
}

}  // extern "C"
