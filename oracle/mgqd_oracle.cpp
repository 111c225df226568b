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

// Coefficients of the reduced system of QD_FV (QD_SOLVERS.f08:40-52), one group: cell planes (nx,ny);
// MxR valid for i < nx-1, MyT for j < ny-1, MxRHS/MyRHS likewise; boundary vectors.
struct QdSystem {
  int nx, ny;
  const double *EBL, *EBB, *EBC, *EBR, *EBT, *MxC, *MxR, *MxB, *MxT, *MyC, *MyT, *MyL, *MyR;
  const double *rhsC, *MxRHS, *MyRHS, *CpL, *CpB, *CpR, *CpT, *BCL, *BCB, *BCR, *BCT;
};

// QD_FV (QD_SOLVERS.f08:40-538): assemble the reduced system and solve it; E (nx,ny), EV (nx+1,ny), EH
// (nx,ny+1) hold the initial guess and receive the solution.  solver 0: direct; solver 1: the reference's
// ILUT + BiCGSTAB, falling back to the direct solve.  Returns the matrix-vector products of the
// iteration, -1 for a direct solve, -2 for a singular system.
long qd_fv(const QdSystem& S, int solver, double* E, double* EV, double* EH) {
  const int nx = S.nx, ny = S.ny;
  const Idx2 P2{nx};
  const double *EBL = S.EBL, *EBB = S.EBB, *EBC = S.EBC, *EBR = S.EBR, *EBT = S.EBT, *MxC = S.MxC, *MxR = S.MxR;
  const double *MxB = S.MxB, *MxT = S.MxT, *MyC = S.MyC, *MyT = S.MyT, *MyL = S.MyL, *MyR = S.MyR, *Ghat = S.rhsC;
  const double *MxRHS = S.MxRHS, *MyRHS = S.MyRHS, *CpL = S.CpL, *CpB = S.CpB, *CpR = S.CpR, *CpT = S.CpT;
  const double *BCL = S.BCL, *BCB = S.BCB, *BCR = S.BCR, *BCT = S.BCT;
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
        x[N.C(i, j)] = E[i + (long)nx * j];
        x[N.H(i, j)] = EH[i + (long)nx * j];
      }
      for (int i = 0; i <= nx; ++i) x[N.V(i, j)] = EV[i + (long)(nx + 1) * j];
    }
    for (int i = 0; i < nx; ++i) x[N.H(i, ny)] = EH[i + (long)nx * ny];
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
    if (!band_solve(B, rhs)) return -2;
  }
  for (int j = 0; j < ny; ++j) {
    for (int i = 0; i < nx; ++i) {
      E[i + (long)nx * j] = rhs[N.C(i, j)];
      EH[i + (long)nx * j] = rhs[N.H(i, j)];
    }
    for (int i = 0; i <= nx; ++i) EV[i + (long)(nx + 1) * j] = rhs[N.V(i, j)];
  }
  for (int i = 0; i < nx; ++i) EH[i + (long)nx * ny] = rhs[N.H(i, ny)];
  return kits;
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

    // the reduced system (QD_SOLVERS.f08:66-386) and its solve
    const QdSystem sys{nx, ny, EBL.data(), EBB.data(), EBC.data(), EBR.data(), EBT.data(), MxC.data(), MxR.data(),
                       MxB.data(), MxT.data(), MyC.data(), MyT.data(), MyL.data(), MyR.data(), Ghat.data(),
                       MxRHS.data(), MyRHS.data(), CpL.data(), CpB.data(), CpR.data(), CpT.data(), BCL.data(),
                       BCB.data(), BCR.data(), BCT.data()};
    const long kits = qd_fv(sys, solver, Eg_avg + C(0, 0, g), Eg_edgV + V(0, 0, g), Eg_edgH + H(0, 0, g));
    if (kits == -2) {
      bad += 1;
      continue;
    }
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

// ------------------------------------------------------------------------------------------------
// Grey low-order side (MainSrc/GLOQD_SOLVES.f08, MLOQD_SOLVES.f08:687-730)
// ------------------------------------------------------------------------------------------------
extern "C" {

// COLLAPSE_MG_EF (MLOQD_SOLVES.f08:687-730): group sums in group order.
int oracle_collapse_mg_ef(int nx, int ny, int ng, const double* Eg_avg, const double* Eg_edgV, const double* Eg_edgH,
                          const double* Fxg_edgV, const double* Fyg_edgH, int Open_Threads, double* E_avg,
                          double* E_edgV, double* E_edgH, double* Fx_edgV, double* Fy_edgH) {
  (void)Open_Threads;
  const long nC = (long)nx * ny, nV = (long)(nx + 1) * ny, nH = (long)nx * (ny + 1);
  for (long k = 0; k < nC; ++k) {
    double s = 0.0;
    for (int g = 0; g < ng; ++g) s += Eg_avg[k + nC * g];
    E_avg[k] = s;
  }
  for (long k = 0; k < nV; ++k) {
    double s = 0.0, f = 0.0;
    for (int g = 0; g < ng; ++g) {
      s += Eg_edgV[k + nV * g];
      f += Fxg_edgV[k + nV * g];
    }
    E_edgV[k] = s;
    Fx_edgV[k] = f;
  }
  for (long k = 0; k < nH; ++k) {
    double s = 0.0, f = 0.0;
    for (int g = 0; g < ng; ++g) {
      s += Eg_edgH[k + nH * g];
      f += Fyg_edgH[k + nH * g];
    }
    E_edgH[k] = s;
    Fy_edgH[k] = f;
  }
  return 0;
}

// Cbar_Calc (GLOQD_SOLVES.f08:177-231).
int oracle_cbar_calc(int nx, int ny, int ng, double* Cb_L, double* Cb_B, double* Cb_R, double* Cb_T, const double* Cg_L,
                     const double* Cg_B, const double* Cg_R, const double* Cg_T, const double* Eg_avg,
                     const double* Eg_edgV, const double* Eg_edgH, const double* Eg_in_L, const double* Eg_in_B,
                     const double* Eg_in_R, const double* Eg_in_T) {
  (void)Eg_avg;
  const long nV = (long)(nx + 1) * ny, nH = (long)nx * (ny + 1);
  for (int j = 0; j < ny; ++j) {
    double l = 0.0, r = 0.0, s1 = 0.0, s2 = 0.0;
    for (int g = 0; g < ng; ++g) {
      double q = Eg_edgV[0 + (long)(nx + 1) * j + nV * g] - Eg_in_L[j + (long)ny * g];
      l = l + Cg_L[j + (long)ny * g] * q;
      s1 = s1 + q;
      q = Eg_edgV[nx + (long)(nx + 1) * j + nV * g] - Eg_in_R[j + (long)ny * g];
      r = r + Cg_R[j + (long)ny * g] * q;
      s2 = s2 + q;
    }
    Cb_L[j] = l / s1;
    Cb_R[j] = r / s2;
  }
  for (int i = 0; i < nx; ++i) {
    double b = 0.0, t = 0.0, s1 = 0.0, s2 = 0.0;
    for (int g = 0; g < ng; ++g) {
      double q = Eg_edgH[i + nH * g] - Eg_in_B[i + (long)nx * g];
      b = b + Cg_B[i + (long)nx * g] * q;
      s1 = s1 + q;
      q = Eg_edgH[i + (long)nx * ny + nH * g] - Eg_in_T[i + (long)nx * g];
      t = t + Cg_T[i + (long)nx * g] * q;
      s2 = s2 + q;
    }
    Cb_B[i] = b / s1;
    Cb_T[i] = t / s2;
  }
  return 0;
}

// OLD_GREY_COEFS (GLOQD_SOLVES.f08:12-42).
// cv_cells: heat capacity per cell (the reference passes one value, cv; nullptr means that value).
int oracle_old_grey_coefs_cells(int nx, int ny, int ng, double c, double Delt, double Theta, double cv,
                                const double* A, const double* Gold, const double* Temp_old,
                                const double* KapE_bar_old, const double* E_avg_old, const double* GQD_Src_old,
                                double* Gold_Hat, double* Rhat_old, const double* cv_cells) {
  const long nC = (long)nx * ny;
  for (long k = 0; k < nC; ++k) Gold_Hat[k] = 0.0;
  for (int g = 0; g < ng; ++g)
    for (long k = 0; k < nC; ++k) Gold_Hat[k] = Gold_Hat[k] + Gold[k + nC * g];
  for (long k = 0; k < nC; ++k) {
    Gold_Hat[k] = Gold_Hat[k] + A[k] * E_avg_old[k] / (Theta * Delt);
    const double cvk = cv_cells ? cv_cells[k] : cv;
    Rhat_old[k] = cvk / (Theta * Delt) * Temp_old[k] +
                  ((1.0 - Theta) / Theta) * (c * KapE_bar_old[k] * E_avg_old[k] - GQD_Src_old[k]);
  }
  return 0;
}

int oracle_old_grey_coefs(int nx, int ny, int ng, double c, double Delt, double Theta, double cv, const double* A,
                          const double* Gold, const double* Temp_old, const double* KapE_bar_old,
                          const double* E_avg_old, const double* GQD_Src_old, double* Gold_Hat, double* Rhat_old) {
  return oracle_old_grey_coefs_cells(nx, ny, ng, c, Delt, Theta, cv, A, Gold, Temp_old, KapE_bar_old, E_avg_old,
                                     GQD_Src_old, Gold_Hat, Rhat_old, nullptr);
}

// GREY_COEFS (GLOQD_SOLVES.f08:47-146); argument order as the subroutine (Pold_L, Pold_R, Pold_B, Pold_T).
int oracle_grey_coefs(int nx, int ny, int ng, const double* Eg_avg, const double* Eg_edgV, const double* Eg_edgH,
                      const double* Fxg_edgV_old, const double* Fyg_edgH_old, const double* fg_avg_xx,
                      const double* fg_avg_yy, const double* fg_edgV_xx, const double* fg_edgV_xy,
                      const double* fg_edgH_yy, const double* fg_edgH_xy, const double* KapE, const double* KapR,
                      const double* A, double c, double Delt, double Theta, const double* Pold_L, const double* Pold_R,
                      const double* Pold_B, const double* Pold_T, double* KapE_Bar, double* DC_xx, double* DL_xx,
                      double* DR_xx, double* DC_yy, double* DB_yy, double* DT_yy, double* DL_xy, double* DR_xy,
                      double* DB_xy, double* DT_xy, double* PL, double* PR, double* PB, double* PT, double Fdt_Weight) {
  const long nC = (long)nx * ny, nV = (long)(nx + 1) * ny, nH = (long)nx * (ny + 1);
  double* outs[] = {KapE_Bar, DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy, PL, PR, PB, PT};
  for (double* o : outs)
    for (long k = 0; k < nC; ++k) o[k] = 0.0;
  for (int g = 0; g < ng; ++g)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = i + (long)nx * j, kg = k + nC * g;
        const long vL = i + (long)(nx + 1) * j + nV * g, vR = vL + 1;
        const long hB = i + (long)nx * j + nH * g, hT = hB + nx;
        const double tk = KapR[kg] + Fdt_Weight / (Theta * c * Delt);
        KapE_Bar[k] = KapE_Bar[k] + KapE[kg] * Eg_avg[kg];
        DC_xx[k] = DC_xx[k] + fg_avg_xx[kg] * Eg_avg[kg] / tk;
        DL_xx[k] = DL_xx[k] + fg_edgV_xx[vL] * Eg_edgV[vL] / tk;
        DR_xx[k] = DR_xx[k] + fg_edgV_xx[vR] * Eg_edgV[vR] / tk;
        DC_yy[k] = DC_yy[k] + fg_avg_yy[kg] * Eg_avg[kg] / tk;
        DB_yy[k] = DB_yy[k] + fg_edgH_yy[hB] * Eg_edgH[hB] / tk;
        DT_yy[k] = DT_yy[k] + fg_edgH_yy[hT] * Eg_edgH[hT] / tk;
        DL_xy[k] = DL_xy[k] + fg_edgV_xy[vL] * Eg_edgV[vL] / tk;
        DR_xy[k] = DR_xy[k] + fg_edgV_xy[vR] * Eg_edgV[vR] / tk;
        DB_xy[k] = DB_xy[k] + fg_edgH_xy[hB] * Eg_edgH[hB] / tk;
        DT_xy[k] = DT_xy[k] + fg_edgH_xy[hT] * Eg_edgH[hT] / tk;
        PL[k] = PL[k] + (Fdt_Weight * A[k] / (2.0 * Theta * c * Delt) * Fxg_edgV_old[vL] + Pold_L[kg]) / tk;
        PR[k] = PR[k] + (Fdt_Weight * A[k] / (2.0 * Theta * c * Delt) * Fxg_edgV_old[vR] + Pold_R[kg]) / tk;
        PB[k] = PB[k] + (Fdt_Weight * A[k] / (2.0 * Theta * c * Delt) * Fyg_edgH_old[hB] + Pold_B[kg]) / tk;
        PT[k] = PT[k] + (Fdt_Weight * A[k] / (2.0 * Theta * c * Delt) * Fyg_edgH_old[hT] + Pold_T[kg]) / tk;
      }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const long k = i + (long)nx * j;
      double s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, s5 = 0.0;
      for (int g = 0; g < ng; ++g) {
        s1 += Eg_avg[k + nC * g];
        s2 += Eg_edgV[i + (long)(nx + 1) * j + nV * g];
        s3 += Eg_edgV[i + 1 + (long)(nx + 1) * j + nV * g];
        s4 += Eg_edgH[i + (long)nx * j + nH * g];
        s5 += Eg_edgH[i + (long)nx * (j + 1) + nH * g];
      }
      KapE_Bar[k] = KapE_Bar[k] / s1;
      DC_xx[k] = DC_xx[k] / s1;
      DL_xx[k] = DL_xx[k] / s2;
      DR_xx[k] = DR_xx[k] / s3;
      DC_yy[k] = DC_yy[k] / s1;
      DB_yy[k] = DB_yy[k] / s4;
      DT_yy[k] = DT_yy[k] / s5;
      DL_xy[k] = DL_xy[k] / s2;
      DR_xy[k] = DR_xy[k] / s3;
      DB_xy[k] = DB_xy[k] / s4;
      DT_xy[k] = DT_xy[k] / s5;
    }
  return 0;
}

// EGP_FV_NEWT (GLOQD_SOLVES.f08:305-860), the grey problem's Newton iteration.  Deltas and dresiduals
// are (Maxits, 6) buffers (the reference allocates (Its, 6)); the first Its rows are filled when
// Res_Calc.  The linear solve of each iteration is QD_FV solved directly.  The safety search
// (:646-755) loops without an exit in the reference; this restatement makes the single pass that
// leaves every bounded value at or above its bound, which is the state that loop reaches.
int oracle_egp_fv_newt_cells(int nx, int ny, double* E_avg, double* E_edgV, double* E_edgH, double* Temp, double* KapE_Bar,
                       double* Fx_edgV, double* Fy_edgH, double* Q_bar, double* KapE_Bar_dT, int* Its,
                       double* Deltas, double* dresiduals, const double* Temp_Mold, const double* KapE_bar_Mold,
                       double Theta, double Delt, const double* Delx, const double* Dely, const double* A,
                       const double* Cb_L, const double* Cb_B, const double* Cb_R, const double* Cb_T,
                       const double* E_in_L, const double* E_in_B, const double* E_in_R, const double* E_in_T,
                       const double* F_in_L, const double* F_in_B, const double* F_in_R, const double* F_in_T,
                       const double* DC_xx, const double* DL_xx, const double* DR_xx, const double* DC_yy,
                       const double* DB_yy, const double* DT_yy, const double* DL_xy, const double* DR_xy,
                       const double* DB_xy, const double* DT_xy, const double* PL, const double* PR, const double* PB,
                       const double* PT, const double* Gold_Hat, const double* Rhat_old, double Kap0, double cv,
                       double Comp_Unit, double Chi, double line_src, double E_Bound_Low, double T_Bound_Low,
                       double Eps1, double Eps2, int Maxits, int MGQD_It, int Use_Line_Search, int Use_Safety_Search,
                       int Res_Calc, int kapE_dT_flag, int* GQD_Kits, double Fin_Weight, double Ein_Weight,
                       const double* cv_cells) {
  auto CV = [&](long k) { return cv_cells ? cv_cells[k] : cv; };
  const double h = 6.62613e-19, c = 2.99792458e2, pi = 4.0 * std::atan(1.0), erg = 6.24150934e11;
  const double sig_R = 2.0 * std::pow(pi, 5) / (15.0 * (c * c) * (h * h * h) * std::pow(erg, 4) * Comp_Unit);
  const double aR = 4.0 * sig_R / c;
  const long nC = (long)nx * ny, nV = (long)(nx + 1) * ny, nH = (long)nx * (ny + 1);
  auto Ci = [&](int i, int j) { return i + (long)nx * j; };
  auto Vi = [&](int i, int j) { return i + (long)(nx + 1) * j; };
  auto Hi = [&](int i, int j) { return i + (long)nx * j; };
  std::vector<double> dT(nC, 0.0), dE(nC, 0.0), dEV(nV, 0.0), dEH(nH, 0.0), dFx(nV, 0.0), dFy(nH, 0.0);
  std::vector<double> oT, oE, oEV, oEH, oFx, oFy, Qdt(nC), Org(nC), W(nC);
  std::vector<double> drB(nC), drT(nC), drML(nC), drMB(nC), drMR(nC), drMT(nC), drG(nC);
  std::vector<double> EBL(nC), EBB(nC), EBC(nC), EBR(nC), EBT(nC), MxC(nC), MxR(nC), MxB(nC), MxT(nC);
  std::vector<double> MyC(nC), MyT(nC), MyL(nC), MyR(nC), MxRHS(nC), MyRHS(nC);
  std::vector<double> CpL(ny), CpR(ny), BCL(ny), BCR(ny), CpB(nx), CpT(nx), BCB(nx), BCT(nx);
  const double p4 = std::pow(pi, 4);

  if (MGQD_It > 1 && kapE_dT_flag) {
    for (long k = 0; k < nC; ++k)
      KapE_Bar_dT[k] = (std::fabs(Temp[k] - Temp_Mold[k]) < 1e-15) ? 0.0
                                                                     : (KapE_Bar[k] - KapE_bar_Mold[k]) / (Temp[k] - Temp_Mold[k]);
    Org.assign(KapE_Bar_dT, KapE_Bar_dT + nC);
  } else {
    for (long k = 0; k < nC; ++k) KapE_Bar_dT[k] = 0.0;
  }
  bool converged = false;
  int its = 0;
  while (!converged && its < Maxits) {
    its += 1;
    oT = dT; oE = dE; oEV = dEV; oEH = dEH; oFx = dFx; oFy = dFy;
    for (long k = 0; k < nC; ++k) {
      Q_bar[k] = 15.0 * Kap0 * c * aR * Temp[k] / p4;
      Qdt[k] = 15.0 * Kap0 * c * aR / p4;
    }
    if (MGQD_It > 1 && kapE_dT_flag) {
      for (long k = 0; k < nC; ++k) {
        KapE_Bar_dT[k] = Org[k];
        const double bound = (CV(k) / (Theta * Delt) + Qdt[k]) / (c * E_avg[k]);
        if (KapE_Bar_dT[k] > Chi * bound) KapE_Bar_dT[k] = Chi * bound;
      }
    }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = Ci(i, j);
        const double a = A[k], dx = Delx[i], dy = Dely[j];
        drT[k] = CV(k) / (Theta * Delt) * Temp[k] + Q_bar[k] - c * KapE_Bar[k] * E_avg[k] - Rhat_old[k];
        drB[k] = a * (1.0 / (Theta * Delt) + c * KapE_Bar[k]) * E_avg[k] + dy * (Fx_edgV[Vi(i + 1, j)] - Fx_edgV[Vi(i, j)]) +
                 dx * (Fy_edgH[Hi(i, j + 1)] - Fy_edgH[Hi(i, j)]) - a * Q_bar[k] - Gold_Hat[k];
        drML[k] = a * Fx_edgV[Vi(i, j)] / 2.0 + c * dy * (DC_xx[k] * E_avg[k] - DL_xx[k] * E_edgV[Vi(i, j)]) +
                  c * dx * (DT_xy[k] * E_edgH[Hi(i, j + 1)] - DB_xy[k] * E_edgH[Hi(i, j)]) / 2.0 - PL[k];
        drMR[k] = a * Fx_edgV[Vi(i + 1, j)] / 2.0 + c * dy * (DR_xx[k] * E_edgV[Vi(i + 1, j)] - DC_xx[k] * E_avg[k]) +
                  c * dx * (DT_xy[k] * E_edgH[Hi(i, j + 1)] - DB_xy[k] * E_edgH[Hi(i, j)]) / 2.0 - PR[k];
        drMB[k] = a * Fy_edgH[Hi(i, j)] / 2.0 + c * dx * (DC_yy[k] * E_avg[k] - DB_yy[k] * E_edgH[Hi(i, j)]) +
                  c * dy * (DR_xy[k] * E_edgV[Vi(i + 1, j)] - DL_xy[k] * E_edgV[Vi(i, j)]) / 2.0 - PB[k];
        drMT[k] = a * Fy_edgH[Hi(i, j + 1)] / 2.0 + c * dx * (DT_yy[k] * E_edgH[Hi(i, j + 1)] - DC_yy[k] * E_avg[k]) +
                  c * dy * (DR_xy[k] * E_edgV[Vi(i + 1, j)] - DL_xy[k] * E_edgV[Vi(i, j)]) / 2.0 - PT[k];
        W[k] = CV(k) / (Theta * Delt) + Qdt[k] - c * KapE_Bar_dT[k] * E_avg[k];
        drG[k] = -drB[k] + drT[k] * (a / W[k]) * (c * KapE_Bar_dT[k] * E_avg[k] - Qdt[k]) +
                 2.0 * dy * (drMR[k] - drML[k]) / a + 2.0 * dx * (drMT[k] - drMB[k]) / a;
        EBC[k] = a * (1.0 / (Theta * Delt) + c * KapE_Bar[k] * (1.0 + (c * KapE_Bar_dT[k] * E_avg[k] - Qdt[k]) / W[k])) +
                 4.0 * c * (dy * dy) * DC_xx[k] / a + 4.0 * c * (dx * dx) * DC_yy[k] / a;
        EBL[k] = -2.0 * c * (dy * dy) * DL_xx[k] / a;
        EBR[k] = -2.0 * c * (dy * dy) * DR_xx[k] / a;
        EBB[k] = -2.0 * c * (dx * dx) * DB_yy[k] / a;
        EBT[k] = -2.0 * c * (dx * dx) * DT_yy[k] / a;
        MxC[k] = 2.0 * c * dy * DC_xx[k] / a;
        MxT[k] = -c * dx * DT_xy[k] / a;
        MxB[k] = c * dx * DB_xy[k] / a;
        MyC[k] = 2.0 * c * dx * DC_yy[k] / a;
        MyR[k] = -c * dy * DR_xy[k] / a;
        MyL[k] = c * dy * DL_xy[k] / a;
      }
    for (int j = 0; j + 1 < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long k = Ci(i, j), kt = Ci(i, j + 1);
        MyT[k] = -2.0 * c * Delx[i] * (DT_yy[k] / A[k] + DB_yy[kt] / A[kt]);
        MyRHS[k] = 2.0 * drMT[k] / A[k] - 2.0 * drMB[kt] / A[kt];
      }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i + 1 < nx; ++i) {
        const long k = Ci(i, j), kr = Ci(i + 1, j);
        MxR[k] = -2.0 * c * Dely[j] * (DR_xx[k] / A[k] + DL_xx[kr] / A[kr]);
        MxRHS[k] = 2.0 * drMR[k] / A[k] - 2.0 * drML[kr] / A[kr];
      }
    for (int j = 0; j < ny; ++j) {
      const long kl = Ci(0, j), kr = Ci(nx - 1, j);
      CpL[j] = c * Cb_L[j] - 2.0 * c * Dely[j] * DL_xx[kl] / A[kl];
      CpR[j] = c * Cb_R[j] + 2.0 * c * Dely[j] * DR_xx[kr] / A[kr];
      BCL[j] = c * Cb_L[j] * (Ein_Weight * E_in_L[j] - E_edgV[Vi(0, j)]) + Fx_edgV[Vi(0, j)] - Fin_Weight * F_in_L[j] -
               2.0 * drML[kl] / A[kl];
      BCR[j] = c * Cb_R[j] * (Ein_Weight * E_in_R[j] - E_edgV[Vi(nx, j)]) + Fx_edgV[Vi(nx, j)] - Fin_Weight * F_in_R[j] -
               2.0 * drMR[kr] / A[kr];
    }
    for (int i = 0; i < nx; ++i) {
      const long kb = Ci(i, 0), kt = Ci(i, ny - 1);
      CpB[i] = c * Cb_B[i] - 2.0 * c * Delx[i] * DB_yy[kb] / A[kb];
      CpT[i] = c * Cb_T[i] + 2.0 * c * Delx[i] * DT_yy[kt] / A[kt];
      BCB[i] = c * Cb_B[i] * (Ein_Weight * E_in_B[i] - E_edgH[Hi(i, 0)]) + Fy_edgH[Hi(i, 0)] - Fin_Weight * F_in_B[i] -
               2.0 * drMB[kb] / A[kb];
      BCT[i] = c * Cb_T[i] * (Ein_Weight * E_in_T[i] - E_edgH[Hi(i, ny)]) + Fy_edgH[Hi(i, ny)] - Fin_Weight * F_in_T[i] -
               2.0 * drMT[kt] / A[kt];
    }
    const QdSystem sys{nx, ny, EBL.data(), EBB.data(), EBC.data(), EBR.data(), EBT.data(), MxC.data(), MxR.data(),
                       MxB.data(), MxT.data(), MyC.data(), MyT.data(), MyL.data(), MyR.data(), drG.data(),
                       MxRHS.data(), MyRHS.data(), CpL.data(), CpB.data(), CpR.data(), CpT.data(), BCL.data(),
                       BCB.data(), BCR.data(), BCT.data()};
    const long kits = qd_fv(sys, 0, dE.data(), dEV.data(), dEH.data());
    if (kits == -2) return -2;
    GQD_Kits[its - 1] = (int)kits;
    // Delta T and Delta F from Delta E (:580-598, with the reference's DT_xy in both cross terms of dFx)
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        const long k = Ci(i, j);
        const double a = A[k];
        dT[k] = (c * KapE_Bar[k] * dE[k] - drT[k]) / W[k];
        dFx[Vi(i, j)] = -2.0 * c * Dely[j] * (DC_xx[k] * dE[k] - DL_xx[k] * dEV[Vi(i, j)]) / a -
                        c * Delx[i] * (DT_xy[k] * dEH[Hi(i, j + 1)] - DT_xy[k] * dEH[Hi(i, j)]) / a - 2.0 * drML[k] / a;
        dFy[Hi(i, j)] = -2.0 * c * Delx[i] * (DC_yy[k] * dE[k] - DB_yy[k] * dEH[Hi(i, j)]) / a -
                        c * Dely[j] * (DR_xy[k] * dEV[Vi(i + 1, j)] - DL_xy[k] * dEV[Vi(i, j)]) / a - 2.0 * drMB[k] / a;
      }
      const int i = nx - 1;
      const long k = Ci(i, j);
      const double a = A[k];
      dFx[Vi(nx, j)] = -2.0 * c * Dely[j] * (DR_xx[k] * dEV[Vi(nx, j)] - DC_xx[k] * dE[k]) / a -
                       c * Delx[i] * (DT_xy[k] * dEH[Hi(i, j + 1)] - DT_xy[k] * dEH[Hi(i, j)]) / a - 2.0 * drMR[k] / a;
    }
    for (int i = 0; i < nx; ++i) {
      const int j = ny - 1;
      const long k = Ci(i, j);
      const double a = A[k];
      dFy[Hi(i, ny)] = -2.0 * c * Delx[i] * (DT_yy[k] * dEH[Hi(i, ny)] - DC_yy[k] * dE[k]) / a -
                       c * Dely[j] * (DR_xy[k] * dEV[Vi(i + 1, j)] - DL_xy[k] * dEV[Vi(i, j)]) / a - 2.0 * drMT[k] / a;
    }
    auto scale_all = [&](double LS) {
      for (auto* v : {&dT, &dE, &dEV, &dEH, &dFx, &dFy})
        for (double& x : *v) x = x / LS;
    };
    auto norm2 = [](const std::vector<double>& v) {
      double s = 0.0;
      for (double x : v) s += x * x;
      return std::sqrt(s);
    };
    // line search (:604-636)
    if (Use_Line_Search && its > 1) {
      const std::vector<double>* cur[6] = {&dT, &dE, &dEV, &dEH, &dFx, &dFy};
      const std::vector<double>* old[6] = {&oT, &oE, &oEV, &oEH, &oFx, &oFy};
      for (int q = 0; q < 6; ++q) {
        const double nrm = norm2(*cur[q]), nrm_old = norm2(*old[q]);
        double LS = 1.0;
        int ls_its = 0;
        while (ls_its < 10) {
          ls_its += 1;
          if (nrm / LS > nrm_old) LS = LS * line_src;
          else break;
        }
        if (LS > 1.0) scale_all(LS);
      }
    }
    // safety search, one pass (:642-755)
    if (Use_Safety_Search) {
      auto guard = [&](double value, const double& delta, double bound) {
        double LS = 1.0;
        for (int n = 0; n < 64 && value + delta / LS < bound; ++n) LS = LS * line_src;
        if (LS > 1.0) scale_all(LS);
      };
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          guard(Temp[Ci(i, j)], dT[Ci(i, j)], T_Bound_Low);
          guard(E_avg[Ci(i, j)], dE[Ci(i, j)], E_Bound_Low);
        }
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) guard(E_edgV[Vi(i, j)], dEV[Vi(i, j)], E_Bound_Low);
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) guard(E_edgH[Hi(i, j)], dEH[Hi(i, j)], E_Bound_Low);
    }
    // new iterate (:757-766)
    for (long k = 0; k < nC; ++k) {
      Temp[k] = Temp[k] + dT[k];
      E_avg[k] = E_avg[k] + dE[k];
    }
    for (long k = 0; k < nH; ++k) E_edgH[k] = E_edgH[k] + dEH[k];
    for (long k = 0; k < nV; ++k) E_edgV[k] = E_edgV[k] + dEV[k];
    for (long k = 0; k < nV; ++k) Fx_edgV[k] = Fx_edgV[k] + dFx[k];
    for (long k = 0; k < nH; ++k) Fy_edgH[k] = Fy_edgH[k] + dFy[k];
    for (long k = 0; k < nC; ++k) {
      KapE_Bar[k] = KapE_Bar[k] + KapE_Bar_dT[k] * dT[k];
      Q_bar[k] = 15.0 * Kap0 * c * aR * Temp[k] / p4;
    }
    // convergence (:771-798)
    auto amax = [](const double* v, long n) {
      double m = 0.0;
      for (long k = 0; k < n; ++k) m = std::max(m, std::fabs(v[k]));
      return m;
    };
    const double nrm[6] = {amax(dT.data(), nC), amax(dE.data(), nC), amax(dEV.data(), nV),
                           amax(dEH.data(), nH), amax(dFx.data(), nV), amax(dFy.data(), nH)};
    const double eps[6] = {Eps1 * amax(Temp, nC) + Eps2, Eps1 * amax(E_avg, nC) + Eps2, Eps1 * amax(E_edgV, nV) + Eps2,
                           Eps1 * amax(E_edgH, nH) + Eps2, Eps1 * amax(Fx_edgV, nV) + Eps2, Eps1 * amax(Fy_edgH, nH) + Eps2};
    converged = true;
    for (int q = 0; q < 6; ++q)
      if (nrm[q] > eps[q]) converged = false;
    if (Res_Calc) {
      const double dr[6] = {amax(drT.data(), nC), amax(drB.data(), nC), amax(drML.data(), nC),
                            amax(drMB.data(), nC), amax(drMR.data(), nC), amax(drMT.data(), nC)};
      for (int q = 0; q < 6; ++q) {
        Deltas[(its - 1) + (long)Maxits * q] = nrm[q];
        dresiduals[(its - 1) + (long)Maxits * q] = dr[q];
      }
    }
  }
  *Its = its;
  return 0;
}

int oracle_egp_fv_newt(int nx, int ny, double* E_avg, double* E_edgV, double* E_edgH, double* Temp, double* KapE_Bar,
                       double* Fx_edgV, double* Fy_edgH, double* Q_bar, double* KapE_Bar_dT, int* Its,
                       double* Deltas, double* dresiduals, const double* Temp_Mold, const double* KapE_bar_Mold,
                       double Theta, double Delt, const double* Delx, const double* Dely, const double* A,
                       const double* Cb_L, const double* Cb_B, const double* Cb_R, const double* Cb_T,
                       const double* E_in_L, const double* E_in_B, const double* E_in_R, const double* E_in_T,
                       const double* F_in_L, const double* F_in_B, const double* F_in_R, const double* F_in_T,
                       const double* DC_xx, const double* DL_xx, const double* DR_xx, const double* DC_yy,
                       const double* DB_yy, const double* DT_yy, const double* DL_xy, const double* DR_xy,
                       const double* DB_xy, const double* DT_xy, const double* PL, const double* PR, const double* PB,
                       const double* PT, const double* Gold_Hat, const double* Rhat_old, double Kap0, double cv,
                       double Comp_Unit, double Chi, double line_src, double E_Bound_Low, double T_Bound_Low,
                       double Eps1, double Eps2, int Maxits, int MGQD_It, int Use_Line_Search, int Use_Safety_Search,
                       int Res_Calc, int kapE_dT_flag, int* GQD_Kits, double Fin_Weight, double Ein_Weight) {
  return oracle_egp_fv_newt_cells(nx, ny, E_avg, E_edgV, E_edgH, Temp, KapE_Bar, Fx_edgV, Fy_edgH, Q_bar, KapE_Bar_dT,
                                  Its, Deltas, dresiduals, Temp_Mold, KapE_bar_Mold, Theta, Delt, Delx, Dely, A, Cb_L,
                                  Cb_B, Cb_R, Cb_T, E_in_L, E_in_B, E_in_R, E_in_T, F_in_L, F_in_B, F_in_R, F_in_T,
                                  DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy, PL, PR, PB, PT,
                                  Gold_Hat, Rhat_old, Kap0, cv, Comp_Unit, Chi, line_src, E_Bound_Low, T_Bound_Low,
                                  Eps1, Eps2, Maxits, MGQD_It, Use_Line_Search, Use_Safety_Search, Res_Calc,
                                  kapE_dT_flag, GQD_Kits, Fin_Weight, Ein_Weight, nullptr);
}

}  // extern "C"
