// Kernels behind the reference-signature entry points that take the angular arrays themselves
// (Fortran layouts) rather than the resident sweep state.  One thread per output point walks the
// directions in the reference's order with the reference's operation order, so with --fmad=false
// the results are bit-identical to a sequential evaluation of the Fortran.
#pragma once

#include <cuda_runtime.h>

namespace trt {

// COLLAPSE_INTENSITIES, TRANSPORT_SOLVES.f08:441-478 (the group totals of :488-509 are
// group_sum_kernel).
__global__ void collapse_dropin_kernel(int nx, int ny, int nm, int ng, const double* __restrict__ I_avg,
                                       const double* __restrict__ I_edgV, const double* __restrict__ I_edgH,
                                       const double* __restrict__ Ox, const double* __restrict__ Oy,
                                       const double* __restrict__ w, double eps, double* Hg_avg_xx,
                                       double* Hg_avg_yy, double* Hg_avg_xy, double* Hg_edgV_xx, double* Hg_edgV_xy,
                                       double* Hg_edgH_yy, double* Hg_edgH_xy, double* Eg_edgV, double* Eg_edgH,
                                       double* Eg_avg, double* Fxg_edgV, double* Fyg_edgH) {
  const double c = 2.99792458e2;
  const long long nA = (long long)nx * ny, nV = (long long)(nx + 1) * ny, nH = (long long)nx * (ny + 1);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long k = k0; k < nA * ng; k += stride) {
    const long long p = k % nA, g = k / nA;
    double xx = 0, yy = 0, xy = 0, e = 0;
    for (int m = 0; m < nm; ++m) {
      const double I = I_avg[p + nA * (m + (long long)nm * g)] + eps;
      xx = xx + (Ox[m] * Ox[m]) * w[m] * I;
      yy = yy + (Oy[m] * Oy[m]) * w[m] * I;
      xy = xy + Ox[m] * Oy[m] * w[m] * I;
      e = e + w[m] * I;
    }
    Hg_avg_xx[k] = xx; Hg_avg_yy[k] = yy; Hg_avg_xy[k] = xy; Eg_avg[k] = e / c;
  }
  for (long long k = k0; k < nV * ng; k += stride) {
    const long long p = k % nV, g = k / nV;
    double xx = 0, xy = 0, fx = 0, e = 0;
    for (int m = 0; m < nm; ++m) {
      const double I = I_edgV[p + nV * (m + (long long)nm * g)] + eps;
      xx = xx + (Ox[m] * Ox[m]) * w[m] * I;
      xy = xy + Ox[m] * Oy[m] * w[m] * I;
      fx = fx + Ox[m] * w[m] * I;
      e = e + w[m] * I;
    }
    Hg_edgV_xx[k] = xx; Hg_edgV_xy[k] = xy; Fxg_edgV[k] = fx; Eg_edgV[k] = e / c;
  }
  for (long long k = k0; k < nH * ng; k += stride) {
    const long long p = k % nH, g = k / nH;
    double yy = 0, xy = 0, fy = 0, e = 0;
    for (int m = 0; m < nm; ++m) {
      const double I = I_edgH[p + nH * (m + (long long)nm * g)] + eps;
      yy = yy + (Oy[m] * Oy[m]) * w[m] * I;
      xy = xy + Ox[m] * Oy[m] * w[m] * I;
      fy = fy + Ox[m] * w[m] * I;   // Omega_x, as written at :469
      e = e + w[m] * I;
    }
    Hg_edgH_yy[k] = yy; Hg_edgH_xy[k] = xy; Fyg_edgH[k] = fy; Eg_edgH[k] = e / c;
  }
}

// fg_Calc, MLOQD_SOLVES.f08:646-674.
__global__ void fg_dropin_kernel(long long nA, long long nV, long long nH, double c, const double* Hxx,
                                 const double* Hyy, const double* Hxy, const double* HVxx, const double* HVxy,
                                 const double* HHyy, const double* HHxy, const double* Ea, const double* EV,
                                 const double* EH, double* fxx, double* fyy, double* fxy, double* fVxx, double* fVxy,
                                 double* fHyy, double* fHxy) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long k = k0; k < nA; k += stride) {
    fxx[k] = Hxx[k] / (c * Ea[k]);
    fyy[k] = Hyy[k] / (c * Ea[k]);
    fxy[k] = Hxy[k] / (c * Ea[k]);
  }
  for (long long k = k0; k < nV; k += stride) {
    fVxx[k] = HVxx[k] / (c * EV[k]);
    fVxy[k] = HVxy[k] / (c * EV[k]);
  }
  for (long long k = k0; k < nH; k += stride) {
    fHyy[k] = HHyy[k] / (c * EH[k]);
    fHxy[k] = HHxy[k] / (c * EH[k]);
  }
}

// Cg_Calc (MLOQD_SOLVES.f08:392-484) and MGQD_In_Calc (:517-610) on the boundary faces of
// I_edgV/I_edgH.  mode 0 = Cg, mode 1 = incoming E and F.
__global__ void boundary_dropin_kernel(int nx, int ny, int nm, int ng, int mode, int4 bc, const double* I_edgV,
                                       const double* I_edgH, const double* Ox, const double* Oy, const double* w,
                                       double eps, double c, double* L, double* B, double* Rr, double* T,
                                       double* FL, double* FB, double* FR, double* FT) {
  const long long nV = (long long)(nx + 1) * ny, nH = (long long)nx * (ny + 1);
  const int q = nm / 4;
  const long long total = 2LL * ny * ng + 2LL * nx * ng;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += stride) {
    int side, pos, g;   // side 0 L, 1 R, 2 B, 3 T
    long long r = k;
    if (r < 2LL * ny * ng) {
      side = (int)(r / ((long long)ny * ng));
      r %= (long long)ny * ng;
      pos = (int)(r % ny);
      g = (int)(r / ny);
    } else {
      r -= 2LL * ny * ng;
      side = 2 + (int)(r / ((long long)nx * ng));
      r %= (long long)nx * ng;
      pos = (int)(r % nx);
      g = (int)(r / nx);
    }
    const int bctype = side == 0 ? bc.x : side == 1 ? bc.z : side == 2 ? bc.y : bc.w;
    const bool vert = side < 2;
    const double* Ia = vert ? I_edgV : I_edgH;
    const long long base = vert ? (side == 0 ? (long long)pos * (nx + 1) : (long long)pos * (nx + 1) + nx)
                                : (side == 2 ? (long long)pos : (long long)pos + (long long)ny * nx);
    const long long pstride = vert ? nV : nH;
    const double* Om = vert ? Ox : Oy;
    const long long oi = vert ? (long long)pos + (long long)ny * g : (long long)pos + (long long)nx * g;
    double* out = side == 0 ? L : side == 1 ? Rr : side == 2 ? B : T;
    double* fout = side == 0 ? FL : side == 1 ? FR : side == 2 ? FB : FT;
    // direction ranges of the reference, in its order
    int r1a, r1b, r2a, r2b;
    if (mode == 0) {   // outgoing
      if (side == 0) { r1a = q; r1b = 3 * q; r2a = r2b = 0; }
      else if (side == 2) { r1a = 2 * q; r1b = 4 * q; r2a = r2b = 0; }
      else if (side == 1) { r1a = 0; r1b = q; r2a = 3 * q; r2b = 4 * q; }
      else { r1a = 0; r1b = 2 * q; r2a = r2b = 0; }
    } else {           // incoming
      if (side == 0) { r1a = 0; r1b = q; r2a = 3 * q; r2b = 4 * q; }
      else if (side == 2) { r1a = 0; r1b = 2 * q; r2a = r2b = 0; }
      else if (side == 1) { r1a = q; r1b = 3 * q; r2a = r2b = 0; }
      else { r1a = 2 * q; r1b = 4 * q; r2a = r2b = 0; }
    }
    if (mode == 0) {
      double C = 0.0, sum = 0.0;
      if (bctype == 0) {
        for (int pass = 0; pass < 2; ++pass) {
          const int a0 = pass ? r2a : r1a, a1 = pass ? r2b : r1b;
          for (int m = a0; m < a1; ++m) {
            const double I = Ia[base + pstride * (m + (long long)nm * g)];
            C = C + Om[m] * w[m] * (I + eps);
            sum = sum + w[m] * (I + eps);
          }
        }
        C = C / sum;
      }
      out[oi] = C;
    } else {
      double E = 0.0, F = 0.0;
      if (bctype == 0) {
        for (int pass = 0; pass < 2; ++pass) {
          const int a0 = pass ? r2a : r1a, a1 = pass ? r2b : r1b;
          for (int m = a0; m < a1; ++m) {
            const double I = Ia[base + pstride * (m + (long long)nm * g)];
            F = F + Om[m] * w[m] * I;
            E = E + w[m] * I;
          }
        }
      }
      out[oi] = E / c;
      fout[oi] = F;
    }
  }
}

}  // namespace trt
