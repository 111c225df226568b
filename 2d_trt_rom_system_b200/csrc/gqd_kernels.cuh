// Grey low-order side on the device, FP64 (sm_100a): COLLAPSE_MG_EF (MainSrc/MLOQD_SOLVES.f08:687-730),
// Cbar_Calc, OLD_GREY_COEFS, GREY_COEFS and the Newton iteration EGP_FV_NEWT of the effective grey
// problem (MainSrc/GLOQD_SOLVES.f08:12-231, 305-996).
//
// The grey Newton system has the structure of QD_FV's reduced system (GLOQD_SOLVES.f08:565), so its
// linear solve is the multigroup solver of mgqd_kernels.cuh run on one "group": egp_coef_kernel fills the
// same coefficient planes from the grey residuals and D/P coefficients.  Group sums run in group order
// (one thread per cell or boundary point), as the reference's loops do.
#pragma once

#include <cuda_runtime.h>

#include "mgqd_kernels.cuh"

namespace trt_gqd {

using trt_mgqd::Coefs;
using trt_mgqd::Dims;

// ------------------------------------------------------------------------------------------------
// group sums
// ------------------------------------------------------------------------------------------------

// COLLAPSE_MG_EF: one thread per position (cell, vertical edge, horizontal edge it owns).
__global__ void collapse_kernel(const Dims d, const double* __restrict__ Eg, const double* __restrict__ EgV,
                                const double* __restrict__ EgH, const double* __restrict__ FgV,
                                const double* __restrict__ FgH, double* E, double* EV, double* EH, double* FV,
                                double* FH) {
  const long pos = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (pos >= d.npos()) return;
  int i, j;
  trt_mgqd::pos_ij(pos, d.nx, i, j);
  if (i < d.nx && j < d.ny) {
    const long k = i + (long)d.nx * j;
    double s = 0.0;
    for (int g = 0; g < d.ng; ++g) s += Eg[k + d.nC * g];
    E[k] = s;
  }
  if (j < d.ny) {
    const long k = i + (long)(d.nx + 1) * j;
    double s = 0.0, f = 0.0;
    for (int g = 0; g < d.ng; ++g) {
      s += EgV[k + d.nV * g];
      f += FgV[k + d.nV * g];
    }
    EV[k] = s;
    FV[k] = f;
  }
  if (i < d.nx) {
    const long k = i + (long)d.nx * j;
    double s = 0.0, f = 0.0;
    for (int g = 0; g < d.ng; ++g) {
      s += EgH[k + d.nH * g];
      f += FgH[k + d.nH * g];
    }
    EH[k] = s;
    FH[k] = f;
  }
}

// Cbar_Calc: threads 0..ny-1 the left/right boundary points, ny..ny+nx-1 the bottom/top ones.
struct CbarArgs {
  const double *CgL, *CgB, *CgR, *CgT, *EgV, *EgH, *EinL, *EinB, *EinR, *EinT;
  double *CbL, *CbB, *CbR, *CbT;
};
__global__ void cbar_kernel(const Dims d, const CbarArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = d.nx, ny = d.ny;
  if (t < ny) {
    const int j = t;
    double l = 0.0, r = 0.0, s1 = 0.0, s2 = 0.0;
    for (int g = 0; g < d.ng; ++g) {
      double q = a.EgV[(long)(nx + 1) * j + d.nV * g] - a.EinL[j + (long)ny * g];
      l = l + a.CgL[j + (long)ny * g] * q;
      s1 = s1 + q;
      q = a.EgV[nx + (long)(nx + 1) * j + d.nV * g] - a.EinR[j + (long)ny * g];
      r = r + a.CgR[j + (long)ny * g] * q;
      s2 = s2 + q;
    }
    a.CbL[j] = l / s1;
    a.CbR[j] = r / s2;
  } else if (t < ny + nx) {
    const int i = t - ny;
    double b = 0.0, tt = 0.0, s1 = 0.0, s2 = 0.0;
    for (int g = 0; g < d.ng; ++g) {
      double q = a.EgH[i + d.nH * g] - a.EinB[i + (long)nx * g];
      b = b + a.CgB[i + (long)nx * g] * q;
      s1 = s1 + q;
      q = a.EgH[i + (long)nx * ny + d.nH * g] - a.EinT[i + (long)nx * g];
      tt = tt + a.CgT[i + (long)nx * g] * q;
      s2 = s2 + q;
    }
    a.CbB[i] = b / s1;
    a.CbT[i] = tt / s2;
  }
}

// OLD_GREY_COEFS: one thread per cell.
// cvc: heat capacity per cell, or nullptr for the reference's single value cv.
__global__ void old_grey_kernel(const Dims d, double c, double Delt, double Theta, double cv,
                                const double* __restrict__ A, const double* __restrict__ Gold,
                                const double* __restrict__ Told, const double* __restrict__ Kbold,
                                const double* __restrict__ Eold, const double* __restrict__ Qold, double* Gh,
                                double* Rh, const double* __restrict__ cvc) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= d.nC) return;
  double s = 0.0;
  for (int g = 0; g < d.ng; ++g) s = s + Gold[k + d.nC * g];
  Gh[k] = s + A[k] * Eold[k] / (Theta * Delt);
  const double cvk = cvc ? cvc[k] : cv;
  Rh[k] = cvk / (Theta * Delt) * Told[k] + ((1.0 - Theta) / Theta) * (c * Kbold[k] * Eold[k] - Qold[k]);
}

// GREY_COEFS: one thread per cell, groups in order.
struct GreyIn {
  const double *Eg, *EgV, *EgH, *FxOld, *FyOld, *fxx, *fyy, *fVxx, *fVxy, *fHyy, *fHxy, *KapE, *KapR, *A;
  const double *PoldL, *PoldR, *PoldB, *PoldT;
  double c, Delt, Theta, Fdt;
};
struct GreyOut {
  double *Kb, *DCxx, *DLxx, *DRxx, *DCyy, *DByy, *DTyy, *DLxy, *DRxy, *DBxy, *DTxy, *PL, *PR, *PB, *PT;
};
__global__ void grey_coefs_kernel(const Dims d, const GreyIn in, const GreyOut o) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= d.nC) return;
  const int nx = d.nx;
  const int i = (int)(k % nx), j = (int)(k / nx);
  double Kb = 0, DCxx = 0, DLxx = 0, DRxx = 0, DCyy = 0, DByy = 0, DTyy = 0, DLxy = 0, DRxy = 0, DBxy = 0, DTxy = 0;
  double PL = 0, PR = 0, PB = 0, PT = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
  const double a = in.A[k];
  for (int g = 0; g < d.ng; ++g) {
    const long kg = k + d.nC * g;
    const long vL = i + (long)(nx + 1) * j + d.nV * g, vR = vL + 1;
    const long hB = k + d.nH * g, hT = hB + nx;
    const double tk = in.KapR[kg] + in.Fdt / (in.Theta * in.c * in.Delt);
    Kb = Kb + in.KapE[kg] * in.Eg[kg];
    DCxx = DCxx + in.fxx[kg] * in.Eg[kg] / tk;
    DLxx = DLxx + in.fVxx[vL] * in.EgV[vL] / tk;
    DRxx = DRxx + in.fVxx[vR] * in.EgV[vR] / tk;
    DCyy = DCyy + in.fyy[kg] * in.Eg[kg] / tk;
    DByy = DByy + in.fHyy[hB] * in.EgH[hB] / tk;
    DTyy = DTyy + in.fHyy[hT] * in.EgH[hT] / tk;
    DLxy = DLxy + in.fVxy[vL] * in.EgV[vL] / tk;
    DRxy = DRxy + in.fVxy[vR] * in.EgV[vR] / tk;
    DBxy = DBxy + in.fHxy[hB] * in.EgH[hB] / tk;
    DTxy = DTxy + in.fHxy[hT] * in.EgH[hT] / tk;
    const double w = in.Fdt * a / (2.0 * in.Theta * in.c * in.Delt);
    PL = PL + (w * in.FxOld[vL] + in.PoldL[kg]) / tk;
    PR = PR + (w * in.FxOld[vR] + in.PoldR[kg]) / tk;
    PB = PB + (w * in.FyOld[hB] + in.PoldB[kg]) / tk;
    PT = PT + (w * in.FyOld[hT] + in.PoldT[kg]) / tk;
  }
  for (int g = 0; g < d.ng; ++g) {
    s1 += in.Eg[k + d.nC * g];
    s2 += in.EgV[i + (long)(nx + 1) * j + d.nV * g];
    s3 += in.EgV[i + 1 + (long)(nx + 1) * j + d.nV * g];
    s4 += in.EgH[k + d.nH * g];
    s5 += in.EgH[k + nx + d.nH * g];
  }
  o.Kb[k] = Kb / s1;
  o.DCxx[k] = DCxx / s1;
  o.DLxx[k] = DLxx / s2;
  o.DRxx[k] = DRxx / s3;
  o.DCyy[k] = DCyy / s1;
  o.DByy[k] = DByy / s4;
  o.DTyy[k] = DTyy / s5;
  o.DLxy[k] = DLxy / s2;
  o.DRxy[k] = DRxy / s3;
  o.DBxy[k] = DBxy / s4;
  o.DTxy[k] = DTxy / s5;
  o.PL[k] = PL;
  o.PR[k] = PR;
  o.PB[k] = PB;
  o.PT[k] = PT;
}

// ------------------------------------------------------------------------------------------------
// The same group sums split in two, for groups held in several ranges (ranks of a multi-GPU run): each range
// forms its partial sums (the loops above over its own groups, in order), the partials are added across the
// ranges (one all-reduce), and the finish kernels form the ratios.  With one range the results are
// bit-identical to the kernels above: the sums run over the same groups in the same order, and the E, EV, EH
// sums that GREY_COEFS divides by are the collapse sums themselves (same loops, same order).
// ------------------------------------------------------------------------------------------------

// Offsets of the per-MGQD-iteration partial sums in one exchange buffer: the collapse sums (E, EV, EH, FV, FH),
// the boundary sums of Cbar_Calc (per left/right point j: l, s1, r, s2; per bottom/top point i: b, s1, t, s2),
// and the 15 numerators of GREY_COEFS per cell.
struct GreyX {
  long E, EV, EH, FV, FH, cbLR, cbBT, grey, size;
};
__host__ __device__ inline GreyX greyx_of(const Dims& d) {
  GreyX x;
  x.E = 0;
  x.EV = x.E + d.nC;
  x.EH = x.EV + d.nV;
  x.FV = x.EH + d.nH;
  x.FH = x.FV + d.nV;
  x.cbLR = x.FH + d.nH;
  x.cbBT = x.cbLR + 4L * d.ny;
  x.grey = x.cbBT + 4L * d.nx;
  x.size = x.grey + 15L * d.nC;
  return x;
}

// OLD_GREY_COEFS's group sum of G_old (partial: this range's groups).
__global__ void gold_sum_kernel(const Dims d, const double* __restrict__ Gold, double* out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= d.nC) return;
  double s = 0.0;
  for (int g = 0; g < d.ng; ++g) s = s + Gold[k + d.nC * g];
  out[k] = s;
}

// OLD_GREY_COEFS from the total group sum of G_old.
__global__ void old_grey_from_sum_kernel(const Dims d, double c, double Delt, double Theta, double cv,
                                         const double* __restrict__ A, const double* __restrict__ Gsum,
                                         const double* __restrict__ Told, const double* __restrict__ Kbold,
                                         const double* __restrict__ Eold, const double* __restrict__ Qold, double* Gh,
                                         double* Rh, const double* __restrict__ cvc) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= d.nC) return;
  Gh[k] = Gsum[k] + A[k] * Eold[k] / (Theta * Delt);
  const double cvk = cvc ? cvc[k] : cv;
  Rh[k] = cvk / (Theta * Delt) * Told[k] + ((1.0 - Theta) / Theta) * (c * Kbold[k] * Eold[k] - Qold[k]);
}

// Cbar_Calc's numerators and weights (partial).
__global__ void cbar_partial_kernel(const Dims d, const CbarArgs a, double* lr, double* bt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = d.nx, ny = d.ny;
  if (t < ny) {
    const int j = t;
    double l = 0.0, r = 0.0, s1 = 0.0, s2 = 0.0;
    for (int g = 0; g < d.ng; ++g) {
      double q = a.EgV[(long)(nx + 1) * j + d.nV * g] - a.EinL[j + (long)ny * g];
      l = l + a.CgL[j + (long)ny * g] * q;
      s1 = s1 + q;
      q = a.EgV[nx + (long)(nx + 1) * j + d.nV * g] - a.EinR[j + (long)ny * g];
      r = r + a.CgR[j + (long)ny * g] * q;
      s2 = s2 + q;
    }
    lr[4 * j] = l;
    lr[4 * j + 1] = s1;
    lr[4 * j + 2] = r;
    lr[4 * j + 3] = s2;
  } else if (t < ny + nx) {
    const int i = t - ny;
    double b = 0.0, tt = 0.0, s1 = 0.0, s2 = 0.0;
    for (int g = 0; g < d.ng; ++g) {
      double q = a.EgH[i + d.nH * g] - a.EinB[i + (long)nx * g];
      b = b + a.CgB[i + (long)nx * g] * q;
      s1 = s1 + q;
      q = a.EgH[i + (long)nx * ny + d.nH * g] - a.EinT[i + (long)nx * g];
      tt = tt + a.CgT[i + (long)nx * g] * q;
      s2 = s2 + q;
    }
    bt[4 * i] = b;
    bt[4 * i + 1] = s1;
    bt[4 * i + 2] = tt;
    bt[4 * i + 3] = s2;
  }
}

__global__ void cbar_finish_kernel(const Dims d, const double* __restrict__ lr, const double* __restrict__ bt,
                                   double* CbL, double* CbB, double* CbR, double* CbT) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < d.ny) {
    CbL[t] = lr[4 * t] / lr[4 * t + 1];
    CbR[t] = lr[4 * t + 2] / lr[4 * t + 3];
  } else if (t < d.ny + d.nx) {
    const int i = t - d.ny;
    CbB[i] = bt[4 * i] / bt[4 * i + 1];
    CbT[i] = bt[4 * i + 2] / bt[4 * i + 3];
  }
}

// GREY_COEFS's 15 numerators per cell (partial), planes k + nC * v in the order Kb, DCxx, DLxx, DRxx, DCyy, DByy,
// DTyy, DLxy, DRxy, DBxy, DTxy, PL, PR, PB, PT.
__global__ void grey_partial_kernel(const Dims d, const GreyIn in, double* out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= d.nC) return;
  const int nx = d.nx;
  const int i = (int)(k % nx), j = (int)(k / nx);
  double v[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double a = in.A[k];
  for (int g = 0; g < d.ng; ++g) {
    const long kg = k + d.nC * g;
    const long vL = i + (long)(nx + 1) * j + d.nV * g, vR = vL + 1;
    const long hB = k + d.nH * g, hT = hB + nx;
    const double tk = in.KapR[kg] + in.Fdt / (in.Theta * in.c * in.Delt);
    v[0] = v[0] + in.KapE[kg] * in.Eg[kg];
    v[1] = v[1] + in.fxx[kg] * in.Eg[kg] / tk;
    v[2] = v[2] + in.fVxx[vL] * in.EgV[vL] / tk;
    v[3] = v[3] + in.fVxx[vR] * in.EgV[vR] / tk;
    v[4] = v[4] + in.fyy[kg] * in.Eg[kg] / tk;
    v[5] = v[5] + in.fHyy[hB] * in.EgH[hB] / tk;
    v[6] = v[6] + in.fHyy[hT] * in.EgH[hT] / tk;
    v[7] = v[7] + in.fVxy[vL] * in.EgV[vL] / tk;
    v[8] = v[8] + in.fVxy[vR] * in.EgV[vR] / tk;
    v[9] = v[9] + in.fHxy[hB] * in.EgH[hB] / tk;
    v[10] = v[10] + in.fHxy[hT] * in.EgH[hT] / tk;
    const double w = in.Fdt * a / (2.0 * in.Theta * in.c * in.Delt);
    v[11] = v[11] + (w * in.FxOld[vL] + in.PoldL[kg]) / tk;
    v[12] = v[12] + (w * in.FxOld[vR] + in.PoldR[kg]) / tk;
    v[13] = v[13] + (w * in.FyOld[hB] + in.PoldB[kg]) / tk;
    v[14] = v[14] + (w * in.FyOld[hT] + in.PoldT[kg]) / tk;
  }
#pragma unroll
  for (int q = 0; q < 15; ++q) out[k + d.nC * q] = v[q];
}

// GREY_COEFS's ratios from the total numerators and the total group sums of E, EV, EH.
__global__ void grey_finish_kernel(const Dims d, const double* __restrict__ num, const double* __restrict__ E,
                                   const double* __restrict__ EV, const double* __restrict__ EH, const GreyOut o) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= d.nC) return;
  const int nx = d.nx;
  const int i = (int)(k % nx), j = (int)(k / nx);
  const double s1 = E[k], s2 = EV[i + (long)(nx + 1) * j], s3 = EV[i + 1 + (long)(nx + 1) * j], s4 = EH[k],
               s5 = EH[k + nx];
  auto n = [&](int q) { return num[k + d.nC * q]; };
  o.Kb[k] = n(0) / s1;
  o.DCxx[k] = n(1) / s1;
  o.DLxx[k] = n(2) / s2;
  o.DRxx[k] = n(3) / s3;
  o.DCyy[k] = n(4) / s1;
  o.DByy[k] = n(5) / s4;
  o.DTyy[k] = n(6) / s5;
  o.DLxy[k] = n(7) / s2;
  o.DRxy[k] = n(8) / s3;
  o.DBxy[k] = n(9) / s4;
  o.DTxy[k] = n(10) / s5;
  o.PL[k] = n(11);
  o.PR[k] = n(12);
  o.PB[k] = n(13);
  o.PT[k] = n(14);
}

// ------------------------------------------------------------------------------------------------
// EGP_FV_NEWT
// ------------------------------------------------------------------------------------------------

constexpr double kEgpC = 2.99792458e2;   // the routine's own PARAMETER c (GLOQD_SOLVES.f08:360)

struct Egp {
  int nx, ny;
  // state (in/out)
  double *E, *EV, *EH, *T, *Kb, *Fx, *Fy, *Q, *Kdt, *Korg;
  // inputs
  const double *Tm, *Kbm, *Delx, *Dely, *A, *CbL, *CbB, *CbR, *CbT, *EinL, *EinB, *EinR, *EinT, *FinL, *FinB, *FinR,
      *FinT;
  const double *DCxx, *DLxx, *DRxx, *DCyy, *DByy, *DTyy, *DLxy, *DRxy, *DBxy, *DTxy, *PL, *PR, *PB, *PT, *Gh, *Rh;
  // per-iteration work
  double *drT, *W, *dT, *dFx, *dFy;
  unsigned long long* maxbuf;   // [0..5] max |dr_*|; [6..11] max |Delta|; [12..17] max |value|
  int* kreq;                    // safety search: steps of line_src required
  double Theta, Delt, Kap0, cv, aR, Chi, Fin, Ein;
  const double* cvc;            // heat capacity per cell, or nullptr for the single value cv
  int damp;                     // MGQD_It > 1 and kapE_dT_flag
};

__device__ __forceinline__ double egp_cv(const Egp& e, long k) { return e.cvc ? e.cvc[k] : e.cv; }

__device__ __forceinline__ void atomic_max_abs(unsigned long long* p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(fabs(v)));
}

// dr_ML / dr_MR / dr_MB / dr_MT of cell (i, j) (GLOQD_SOLVES.f08:941-996)
__device__ __forceinline__ double egp_drML(const Egp& e, int i, int j) {
  const long k = i + (long)e.nx * j, vL = i + (long)(e.nx + 1) * j, hB = k, hT = k + e.nx;
  const double c = kEgpC;
  return e.A[k] * e.Fx[vL] / 2.0 + c * e.Dely[j] * (e.DCxx[k] * e.E[k] - e.DLxx[k] * e.EV[vL]) +
         c * e.Delx[i] * (e.DTxy[k] * e.EH[hT] - e.DBxy[k] * e.EH[hB]) / 2.0 - e.PL[k];
}
__device__ __forceinline__ double egp_drMR(const Egp& e, int i, int j) {
  const long k = i + (long)e.nx * j, vR = i + 1 + (long)(e.nx + 1) * j, hB = k, hT = k + e.nx;
  const double c = kEgpC;
  return e.A[k] * e.Fx[vR] / 2.0 + c * e.Dely[j] * (e.DRxx[k] * e.EV[vR] - e.DCxx[k] * e.E[k]) +
         c * e.Delx[i] * (e.DTxy[k] * e.EH[hT] - e.DBxy[k] * e.EH[hB]) / 2.0 - e.PR[k];
}
__device__ __forceinline__ double egp_drMB(const Egp& e, int i, int j) {
  const long k = i + (long)e.nx * j, vL = i + (long)(e.nx + 1) * j, hB = k;
  const double c = kEgpC;
  return e.A[k] * e.Fy[hB] / 2.0 + c * e.Delx[i] * (e.DCyy[k] * e.E[k] - e.DByy[k] * e.EH[hB]) +
         c * e.Dely[j] * (e.DRxy[k] * e.EV[vL + 1] - e.DLxy[k] * e.EV[vL]) / 2.0 - e.PB[k];
}
__device__ __forceinline__ double egp_drMT(const Egp& e, int i, int j) {
  const long k = i + (long)e.nx * j, vL = i + (long)(e.nx + 1) * j, hT = k + e.nx;
  const double c = kEgpC;
  return e.A[k] * e.Fy[hT] / 2.0 + c * e.Delx[i] * (e.DTyy[k] * e.EH[hT] - e.DCyy[k] * e.E[k]) +
         c * e.Dely[j] * (e.DRxy[k] * e.EV[vL + 1] - e.DLxy[k] * e.EV[vL]) / 2.0 - e.PT[k];
}

// KapE_Bar_dT before the iterations (GLOQD_SOLVES.f08:398-414).
__global__ void egp_dtinit_kernel(const Egp e) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= (long)e.nx * e.ny) return;
  double v = 0.0;
  if (e.damp) v = (fabs(e.T[k] - e.Tm[k]) < 1e-15) ? 0.0 : (e.Kb[k] - e.Kbm[k]) / (e.T[k] - e.Tm[k]);
  e.Kdt[k] = v;
  e.Korg[k] = v;
}

// Residuals and the coefficients of the Newton system (GLOQD_SOLVES.f08:435-560) into the solver's planes.
__global__ void egp_coef_kernel(const Egp e, const Dims d, const Coefs cf) {
  const long pos = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (pos >= d.npos()) return;
  const int nx = e.nx, ny = e.ny;
  int i, j;
  trt_mgqd::pos_ij(pos, nx, i, j);
  const double c = kEgpC, pi4 = 97.40909103400243723644033268870511;   // pi^4
  const double Qdt = 15.0 * e.Kap0 * c * e.aR / pi4;
  if (i < nx && j < ny) {
    const long k = i + (long)nx * j;
    const double a = e.A[k], dx = e.Delx[i], dy = e.Dely[j];
    const double Q = 15.0 * e.Kap0 * c * e.aR * e.T[k] / pi4;
    e.Q[k] = Q;
    double kdt = e.Kdt[k];
    if (e.damp) {
      kdt = e.Korg[k];
      const double bound = (egp_cv(e, k) / (e.Theta * e.Delt) + Qdt) / (c * e.E[k]);
      if (kdt > e.Chi * bound) kdt = e.Chi * bound;
      e.Kdt[k] = kdt;
    }
    const long vL = i + (long)(nx + 1) * j, hB = k;
    const double drT = egp_cv(e, k) / (e.Theta * e.Delt) * e.T[k] + Q - c * e.Kb[k] * e.E[k] - e.Rh[k];
    const double drB = a * (1.0 / (e.Theta * e.Delt) + c * e.Kb[k]) * e.E[k] + dy * (e.Fx[vL + 1] - e.Fx[vL]) +
                       dx * (e.Fy[hB + nx] - e.Fy[hB]) - a * Q - e.Gh[k];
    const double drML = egp_drML(e, i, j), drMR = egp_drMR(e, i, j), drMB = egp_drMB(e, i, j),
                 drMT = egp_drMT(e, i, j);
    const double W = egp_cv(e, k) / (e.Theta * e.Delt) + Qdt - c * kdt * e.E[k];
    e.drT[k] = drT;
    e.W[k] = W;
    atomic_max_abs(&e.maxbuf[0], drT);
    atomic_max_abs(&e.maxbuf[1], drB);
    atomic_max_abs(&e.maxbuf[2], drML);
    atomic_max_abs(&e.maxbuf[3], drMB);
    atomic_max_abs(&e.maxbuf[4], drMR);
    atomic_max_abs(&e.maxbuf[5], drMT);
    cf.b[k] = -drB + drT * (a / W) * (c * kdt * e.E[k] - Qdt) + 2.0 * dy * (drMR - drML) / a +
              2.0 * dx * (drMT - drMB) / a;
    cf.EBC[k] = a * (1.0 / (e.Theta * e.Delt) + c * e.Kb[k] * (1.0 + (c * kdt * e.E[k] - Qdt) / W)) +
                4.0 * c * (dy * dy) * e.DCxx[k] / a + 4.0 * c * (dx * dx) * e.DCyy[k] / a;
    cf.EBL[k] = -2.0 * c * (dy * dy) * e.DLxx[k] / a;
    cf.EBR[k] = -2.0 * c * (dy * dy) * e.DRxx[k] / a;
    cf.EBB[k] = -2.0 * c * (dx * dx) * e.DByy[k] / a;
    cf.EBT[k] = -2.0 * c * (dx * dx) * e.DTyy[k] / a;
    cf.MXC[k] = 2.0 * c * dy * e.DCxx[k] / a;
    cf.MXT[k] = -c * dx * e.DTxy[k] / a;
    cf.MXB[k] = c * dx * e.DBxy[k] / a;
    cf.MYC[k] = 2.0 * c * dx * e.DCyy[k] / a;
    cf.MYR[k] = -c * dy * e.DRxy[k] / a;
    cf.MYL[k] = c * dy * e.DLxy[k] / a;
  }
  if (j < ny) {   // vertical edge (i, j): x-momentum across it or the boundary condition
    const double dy = e.Dely[j];
    const long ev = i + (long)(nx + 1) * j;
    double dv, bv;
    if (i == 0) {
      const long k = (long)nx * j;
      dv = c * e.CbL[j] - 2.0 * c * dy * e.DLxx[k] / e.A[k];
      bv = c * e.CbL[j] * (e.Ein * e.EinL[j] - e.EV[ev]) + e.Fx[ev] - e.Fin * e.FinL[j] - 2.0 * egp_drML(e, 0, j) / e.A[k];
    } else if (i == nx) {
      const long k = nx - 1 + (long)nx * j;
      dv = c * e.CbR[j] + 2.0 * c * dy * e.DRxx[k] / e.A[k];
      bv = c * e.CbR[j] * (e.Ein * e.EinR[j] - e.EV[ev]) + e.Fx[ev] - e.Fin * e.FinR[j] -
           2.0 * egp_drMR(e, nx - 1, j) / e.A[k];
    } else {
      const long kl = i - 1 + (long)nx * j, kr = kl + 1;
      dv = -2.0 * c * dy * (e.DRxx[kl] / e.A[kl] + e.DLxx[kr] / e.A[kr]);
      bv = 2.0 * egp_drMR(e, i - 1, j) / e.A[kl] - 2.0 * egp_drML(e, i, j) / e.A[kr];
    }
    cf.dV[ev] = dv;
    cf.b[d.oV() + ev] = bv;
  }
  if (i < nx) {   // horizontal edge (i, j)
    const double dx = e.Delx[i];
    const long eh = i + (long)nx * j;
    double dh, bh;
    if (j == 0) {
      const long k = i;
      dh = c * e.CbB[i] - 2.0 * c * dx * e.DByy[k] / e.A[k];
      bh = c * e.CbB[i] * (e.Ein * e.EinB[i] - e.EH[eh]) + e.Fy[eh] - e.Fin * e.FinB[i] - 2.0 * egp_drMB(e, i, 0) / e.A[k];
    } else if (j == ny) {
      const long k = i + (long)nx * (ny - 1);
      dh = c * e.CbT[i] + 2.0 * c * dx * e.DTyy[k] / e.A[k];
      bh = c * e.CbT[i] * (e.Ein * e.EinT[i] - e.EH[eh]) + e.Fy[eh] - e.Fin * e.FinT[i] -
           2.0 * egp_drMT(e, i, ny - 1) / e.A[k];
    } else {
      const long kb = i + (long)nx * (j - 1), kt = kb + nx;
      dh = -2.0 * c * dx * (e.DTyy[kb] / e.A[kb] + e.DByy[kt] / e.A[kt]);
      bh = 2.0 * egp_drMT(e, i, j - 1) / e.A[kb] - 2.0 * egp_drMB(e, i, j) / e.A[kt];
    }
    cf.dH[eh] = dh;
    cf.b[d.oH() + eh] = bh;
  }
}

// Delta T and Delta F from Delta E (GLOQD_SOLVES.f08:572-598, with the reference's DT_xy in both cross
// terms of Delta Fx); partial sums of squares of the six deltas for the line search.
__global__ void __launch_bounds__(trt_mgqd::kRedBlock) egp_delta_kernel(const Egp e, const Dims d,
                                                                        const double* __restrict__ x, double* part) {
  const long pos = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  const int nx = e.nx, ny = e.ny;
  if (pos < d.npos()) {
    int i, j;
    trt_mgqd::pos_ij(pos, nx, i, j);
    const double c = kEgpC;
    const double* dE = x;
    const double* dEV = x + d.oV();
    const double* dEH = x + d.oH();
    if (i < nx && j < ny) {
      const long k = i + (long)nx * j;
      const double t = (c * e.Kb[k] * dE[k] - e.drT[k]) / e.W[k];
      e.dT[k] = t;
      v[0] = t * t;
      v[1] = dE[k] * dE[k];
    }
    if (j < ny) {
      const long ev = i + (long)(nx + 1) * j;
      const bool last = (i == nx);
      const int ic = last ? nx - 1 : i;
      const long k = ic + (long)nx * j;
      const double a = e.A[k];
      const long hB = k, hT = k + nx;
      const double cross = c * e.Delx[ic] * (e.DTxy[k] * dEH[hT] - e.DTxy[k] * dEH[hB]) / a;
      double f;
      if (!last)
        f = -2.0 * c * e.Dely[j] * (e.DCxx[k] * dE[k] - e.DLxx[k] * dEV[ev]) / a - cross - 2.0 * egp_drML(e, i, j) / a;
      else
        f = -2.0 * c * e.Dely[j] * (e.DRxx[k] * dEV[ev] - e.DCxx[k] * dE[k]) / a - cross - 2.0 * egp_drMR(e, ic, j) / a;
      e.dFx[ev] = f;
      v[2] = dEV[ev] * dEV[ev];
      v[4] = f * f;
    }
    if (i < nx) {
      const long eh = i + (long)nx * j;
      const bool last = (j == ny);
      const int jc = last ? ny - 1 : j;
      const long k = i + (long)nx * jc;
      const double a = e.A[k];
      const long vL = i + (long)(nx + 1) * jc;
      const double cross = c * e.Dely[jc] * (e.DRxy[k] * dEV[vL + 1] - e.DLxy[k] * dEV[vL]) / a;
      double f;
      if (!last)
        f = -2.0 * c * e.Delx[i] * (e.DCyy[k] * dE[k] - e.DByy[k] * dEH[eh]) / a - cross - 2.0 * egp_drMB(e, i, j) / a;
      else
        f = -2.0 * c * e.Delx[i] * (e.DTyy[k] * dEH[eh] - e.DCyy[k] * dE[k]) / a - cross - 2.0 * egp_drMT(e, i, jc) / a;
      e.dFy[eh] = f;
      v[3] = dEH[eh] * dEH[eh];
      v[5] = f * f;
    }
  }
  const int kind[6] = {0, 0, 0, 0, 0, 0};
  trt_mgqd::block_reduce<6>(v, kind, part, 0);
}

__global__ void egp_norm_finish_kernel(const double* part, int nblk, double* out) {
  const int kind[6] = {0, 0, 0, 0, 0, 0};
  double o[6];
  trt_mgqd::warp_finish<6>(part, nblk, 0, kind, o);
  if (threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) out[q] = o[q];
}

// Safety search (GLOQD_SOLVES.f08:642-755): the number of line_src steps each bounded value needs so
// that value + Delta / (scale * line_src^k) stays at or above its bound; the maximum is the pass's step.
__device__ __forceinline__ int safety_steps(double value, double delta, double bound, double scale, double ls) {
  double LS = 1.0;
  int k = 0;
  while (k < 64 && value + delta / (scale * LS) < bound) {
    LS = LS * ls;
    ++k;
  }
  return k;
}
__global__ void egp_safety_kernel(const Egp e, const Dims d, const double* __restrict__ x, double scale, double ls,
                                  double Tlow, double Elow) {
  const long pos = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (pos >= d.npos()) return;
  const int nx = e.nx, ny = e.ny;
  int i, j;
  trt_mgqd::pos_ij(pos, nx, i, j);
  int k = 0;
  if (i < nx && j < ny) {
    const long c = i + (long)nx * j;
    k = max(k, safety_steps(e.T[c], e.dT[c], Tlow, scale, ls));
    k = max(k, safety_steps(e.E[c], x[c], Elow, scale, ls));
  }
  if (j < ny) {
    const long ev = i + (long)(nx + 1) * j;
    k = max(k, safety_steps(e.EV[ev], x[d.oV() + ev], Elow, scale, ls));
  }
  if (i < nx) {
    const long eh = i + (long)nx * j;
    k = max(k, safety_steps(e.EH[eh], x[d.oH() + eh], Elow, scale, ls));
  }
  if (k > 0) atomicMax(e.kreq, k);
}

// New iterate with the deltas divided by `scale` (GLOQD_SOLVES.f08:757-766); the scaled Delta E stays in
// x as the next iteration's initial guess; maxima for the convergence test (:771-798).
__global__ void egp_update_kernel(const Egp e, const Dims d, double* x, double scale) {
  const long pos = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (pos >= d.npos()) return;
  const int nx = e.nx, ny = e.ny;
  int i, j;
  trt_mgqd::pos_ij(pos, nx, i, j);
  const double c = kEgpC, pi4 = 97.40909103400243723644033268870511;
  if (i < nx && j < ny) {
    const long k = i + (long)nx * j;
    const double dt = e.dT[k] / scale, de = x[k] / scale;
    const double t = e.T[k] + dt, en = e.E[k] + de;
    e.T[k] = t;
    e.E[k] = en;
    x[k] = de;
    e.Kb[k] = e.Kb[k] + e.Kdt[k] * dt;
    e.Q[k] = 15.0 * e.Kap0 * c * e.aR * t / pi4;
    atomic_max_abs(&e.maxbuf[6], dt);
    atomic_max_abs(&e.maxbuf[7], de);
    atomic_max_abs(&e.maxbuf[12], t);
    atomic_max_abs(&e.maxbuf[13], en);
  }
  if (j < ny) {
    const long ev = i + (long)(nx + 1) * j;
    const double de = x[d.oV() + ev] / scale, df = e.dFx[ev] / scale;
    const double en = e.EV[ev] + de, fn = e.Fx[ev] + df;
    e.EV[ev] = en;
    e.Fx[ev] = fn;
    x[d.oV() + ev] = de;
    atomic_max_abs(&e.maxbuf[8], de);
    atomic_max_abs(&e.maxbuf[10], df);
    atomic_max_abs(&e.maxbuf[14], en);
    atomic_max_abs(&e.maxbuf[16], fn);
  }
  if (i < nx) {
    const long eh = i + (long)nx * j;
    const double de = x[d.oH() + eh] / scale, df = e.dFy[eh] / scale;
    const double en = e.EH[eh] + de, fn = e.Fy[eh] + df;
    e.EH[eh] = en;
    e.Fy[eh] = fn;
    x[d.oH() + eh] = de;
    atomic_max_abs(&e.maxbuf[9], de);
    atomic_max_abs(&e.maxbuf[11], df);
    atomic_max_abs(&e.maxbuf[15], en);
    atomic_max_abs(&e.maxbuf[17], fn);
  }
}

}  // namespace trt_gqd
