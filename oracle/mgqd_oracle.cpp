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
// iteration fails (:489-497).  SPARSKIT2 is not vendored in the reference tree.  Two solvers:
//   solver 0 (oracle_mloqd_fv, the checker): the same equations solved directly, by banded LU with
//     partial pivoting over a row-by-row numbering of the unknowns (its own numbering: the solution
//     does not depend on it); this is the discrete solution the reference's iteration converges to.
//     MGQD_Kits is -1 for every group, the value the reference records when it solves directly.
//   solver 1 (oracle_mloqd_fv_solver(1, ...), the CPU baseline): the reference's own procedure, in the
//     reference's unknown numbering (QD_SOLVERS.f08:66-77,162-171,219-233) and with its initial guess
//     (:447-470): ILUT with dual threshold (Saad, "ILUT: a dual threshold incomplete LU
//     factorization", 1994, as SPARSKIT2 implements it: drop below droptol times the row's mean
//     absolute value, keep the lfil largest entries of each L and U row besides the diagonal), then
//     right-preconditioned BiCGSTAB (van der Vorst 1992) stopped on the SPARSKIT criterion ipar(3) = -1
//     as documented there, ||x_k - x_{k-1}|| <= rtol ||x_k|| + atol, at most 2000 matrix-vector
//     products, falling back to the direct solve.  MGQD_Kits counts matrix-vector products.
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
  bool ref;   // the reference's numbering (QD_SOLVERS.f08:66-77, 162-171, 219-233), 0-based
  Numbering(long nx_, long ny_, bool ref_ = false) : nx(nx_), ny(ny_), blk(3 * nx_ + 1), ref(ref_) {}
  long n() const { return ny * blk + nx; }
  // reference: row j = 0 holds [E_edgV(0,0), per cell (bottom, centre, right, top)] (4 nx + 1 unknowns),
  // every later row [E_edgV(0,j), per cell (centre, right, top)] (3 nx + 1)
  long rstart(long j) const { return 4 * nx + 1 + (j - 1) * (3 * nx + 1); }
  long H(long i, long j) const {
    if (!ref) return j * blk + i;
    if (j == 0) return 4 * i + 1;
    if (j == 1) return 4 * i + 4;
    return rstart(j - 1) + 3 * i + 3;
  }
  long V(long i, long j) const {
    if (!ref) return j * blk + nx + 2 * i;
    if (j == 0) return i == 0 ? 0 : 4 * i - 1;
    return i == 0 ? rstart(j) : rstart(j) + 3 * i - 1;
  }
  long C(long i, long j) const {
    if (!ref) return j * blk + nx + 2 * i + 1;
    return j == 0 ? 4 * i + 2 : rstart(j) + 3 * i + 1;
  }
};

// Compressed sparse rows, entries of a row in insertion order.
struct Csr {
  long n = 0;
  std::vector<long> ia, ja;
  std::vector<double> a;
  void matvec(const double* x, double* y) const {
    for (long r = 0; r < n; ++r) {
      double s = 0.0;
      for (long p = ia[r]; p < ia[r + 1]; ++p) s += a[p] * x[ja[p]];
      y[r] = s;
    }
  }
};

// ILUT factors: L strictly lower (unit diagonal implied), U upper with the diagonal first in each row.
struct Ilu {
  std::vector<long> lia, lja, uia, uja;
  std::vector<double> la, ua;
  void solve(const double* x, double* y, long n) const {
    for (long r = 0; r < n; ++r) {
      double s = x[r];
      for (long p = lia[r]; p < lia[r + 1]; ++p) s -= la[p] * y[lja[p]];
      y[r] = s;
    }
    for (long r = n - 1; r >= 0; --r) {
      double s = y[r];
      for (long p = uia[r] + 1; p < uia[r + 1]; ++p) s -= ua[p] * y[uja[p]];
      y[r] = s / ua[uia[r]];
    }
  }
};

// Dual-threshold incomplete LU (Saad 1994): row-wise elimination in increasing column order on a dense
// work row, dropping multipliers and entries below droptol * mean|a_r|, keeping the lfil largest of
// each of the L and U parts of a row (the diagonal always; a zero diagonal becomes
// (1e-4 + droptol) * mean|a_r|).
void ilut(const Csr& A, int lfil, double droptol, Ilu& F) {
  const long n = A.n;
  std::vector<double> w(n, 0.0);
  std::vector<char> used(n, 0);
  std::vector<long> lidx, uidx;
  F.lia.assign(1, 0);
  F.uia.assign(1, 0);
  for (long r = 0; r < n; ++r) {
    double tnorm = 0.0;
    const long len = A.ia[r + 1] - A.ia[r];
    lidx.clear();
    uidx.clear();
    for (long p = A.ia[r]; p < A.ia[r + 1]; ++p) {
      const long c = A.ja[p];
      tnorm += std::fabs(A.a[p]);
      if (!used[c]) {
        used[c] = 1;
        (c < r ? lidx : uidx).push_back(c);
      }
      w[c] += A.a[p];
    }
    tnorm = len > 0 ? tnorm / (double)len : 1.0;
    const double thr = droptol * tnorm;
    if (!used[r]) {
      used[r] = 1;
      uidx.push_back(r);
    }
    // eliminate the lower part in increasing column order
    std::vector<long> lkept;
    size_t done = 0;
    while (done < lidx.size()) {
      size_t m = done;
      for (size_t q = done + 1; q < lidx.size(); ++q)
        if (lidx[q] < lidx[m]) m = q;
      std::swap(lidx[done], lidx[m]);
      const long k = lidx[done++];
      const double fact = w[k] / F.ua[F.uia[k]];
      if (std::fabs(fact) <= thr) {
        w[k] = 0.0;
        continue;
      }
      w[k] = fact;
      lkept.push_back(k);
      for (long p = F.uia[k] + 1; p < F.uia[k + 1]; ++p) {
        const long c = F.uja[p];
        if (!used[c]) {
          used[c] = 1;
          (c < r ? lidx : uidx).push_back(c);
        }
        w[c] -= fact * F.ua[p];
      }
    }
    // keep the lfil largest of L and of the off-diagonal U
    auto keep_largest = [&](std::vector<long>& idx) {
      std::vector<long> out;
      for (long c : idx)
        if (std::fabs(w[c]) > thr) out.push_back(c);
      if ((long)out.size() > lfil) {
        std::partial_sort(out.begin(), out.begin() + lfil, out.end(),
                          [&](long x, long y) { return std::fabs(w[x]) > std::fabs(w[y]); });
        out.resize(lfil);
      }
      std::sort(out.begin(), out.end());
      return out;
    };
    std::vector<long> lsel = keep_largest(lkept);
    std::vector<long> uoff;
    for (long c : uidx)
      if (c != r) uoff.push_back(c);
    std::vector<long> usel = keep_largest(uoff);
    for (long c : lsel) {
      F.lja.push_back(c);
      F.la.push_back(w[c]);
    }
    F.lia.push_back((long)F.lja.size());
    double diag = w[r];
    if (diag == 0.0) diag = (1e-4 + droptol) * tnorm;
    F.uja.push_back(r);
    F.ua.push_back(diag);
    for (long c : usel) {
      F.uja.push_back(c);
      F.ua.push_back(w[c]);
    }
    F.uia.push_back((long)F.uja.size());
    // clear the work row
    for (long c : lidx) {
      w[c] = 0.0;
      used[c] = 0;
    }
    for (long c : uidx) {
      w[c] = 0.0;
      used[c] = 0;
    }
  }
}

// Right-preconditioned BiCGSTAB; stops when ||x_k - x_{k-1}||_2 <= rtol ||x_k||_2 + atol.  Returns the
// matrix-vector products used (initial residual included), or -1 on breakdown / after max_mv products.
long bicgstab(const Csr& A, const Ilu& M, const std::vector<double>& b, std::vector<double>& x, double rtol,
              double atol, long max_mv) {
  const long n = A.n;
  std::vector<double> r(n), rh(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
    double z = 0.0;
    for (long k = 0; k < n; ++k) z += a[k] * c[k];
    return z;
  };
  A.matvec(x.data(), r.data());
  long nmv = 1;
  for (long k = 0; k < n; ++k) r[k] = b[k] - r[k];
  rh = r;
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  for (;;) {
    const double rho1 = dot(rh, r);
    if (rho1 == 0.0) return nmv;   // exact residual zero
    const double beta = (rho1 / rho) * (alpha / omega);
    rho = rho1;
    for (long k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - omega * v[k]);
    M.solve(p.data(), ph.data(), n);
    A.matvec(ph.data(), v.data());
    ++nmv;
    const double rv = dot(rh, v);
    if (rv == 0.0) return -1;
    alpha = rho / rv;
    for (long k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
    M.solve(s.data(), sh.data(), n);
    A.matvec(sh.data(), t.data());
    ++nmv;
    const double tt = dot(t, t);
    omega = tt != 0.0 ? dot(t, s) / tt : 0.0;
    double dx2 = 0.0, x2 = 0.0;
    for (long k = 0; k < n; ++k) {
      const double dx = alpha * ph[k] + omega * sh[k];
      x[k] += dx;
      r[k] = s[k] - omega * t[k];
      dx2 += dx * dx;
      x2 += x[k] * x[k];
    }
    if (std::sqrt(dx2) <= rtol * std::sqrt(x2) + atol) return nmv;
    if (omega == 0.0 || nmv >= max_mv) return -1;
  }
}

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
int oracle_mloqd_fv_solver(int solver, int nx, int ny, int ng, double* Eg_avg, double* Eg_edgV, double* Eg_edgH,
                           double* Fxg_edgV,
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
    const Numbering N(nx, ny, solver == 1);
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
    long kits = -1;
    if (solver == 1) {
      // QD_SOLVERS.f08:386-497: CSR in row order, ILUT(3, 1e-6), BiCGSTAB from the current E
      Csr A;
      A.n = n;
      std::vector<long> cnt(n + 1, 0);
      for (const Ent& e : ent) cnt[e.r + 1] += 1;
      for (long r = 0; r < n; ++r) cnt[r + 1] += cnt[r];
      A.ia = cnt;
      A.ja.resize(ent.size());
      A.a.resize(ent.size());
      for (const Ent& e : ent) {
        const long q = cnt[e.r]++;
        A.ja[q] = e.c;
        A.a[q] = e.v;
      }
      Ilu M;
      ilut(A, 3, 1e-6, M);
      std::vector<double> x(n);
      for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
          x[N.C(i, j)] = Eg_avg[C(i, j, g)];
          x[N.H(i, j)] = Eg_edgH[H(i, j, g)];
        }
        for (int i = 0; i <= nx; ++i) x[N.V(i, j)] = Eg_edgV[V(i, j, g)];
      }
      for (int i = 0; i < nx; ++i) x[N.H(i, ny)] = Eg_edgH[H(i, ny, g)];
      kits = bicgstab(A, M, rhs, x, 1e-13, 1e-15, 2000);
      if (kits > 0) rhs = x;
    }
    if (kits < 0) {
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
    }
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        Eg_avg[C(i, j, g)] = rhs[N.C(i, j)];
        Eg_edgH[H(i, j, g)] = rhs[N.H(i, j)];
      }
      for (int i = 0; i <= nx; ++i) Eg_edgV[V(i, j, g)] = rhs[N.V(i, j)];
    }
    for (int i = 0; i < nx; ++i) Eg_edgH[H(i, ny, g)] = rhs[N.H(i, ny)];
    MGQD_Kits[g] = (int)kits;

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
  return oracle_mloqd_fv_solver(0, nx, ny, ng, Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV, Fyg_edgH, fg_avg_xx, fg_avg_yy,
                                fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy, Cg_L, Cg_B, Cg_R, Cg_T, Eg_in_L,
                                Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T, Src, KapE, KapR, Delx,
                                Dely, A, c, Delt, Theta, Open_Threads, Res_Calc, MGQD_Residual, MGQD_BC_Residual,
                                G_old, Pold_L, Pold_B, Pold_R, Pold_T, Eg_avg_old, Fxg_edgV_old, Fyg_edgH_old,
                                MGQD_Kits, Fdt_Weight, Fin_Weight, Ein_Weight);
}

}  // extern "C"
