// Device kernels of the transport-only time step (the reference's run_type 'tr_no_qd',
// MainSrc/ALGORITHMS.f08:541-572, 662-668, 816-836): the material update from the temperature,
// the material energy balance that gives the temperature from the sweep's group energies, and the
// outer-iteration convergence norms.  Each function cites the reference routine it restates; the
// operation order follows the Fortran expressions (all files are built with --fmad=false).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace trt {

// Physical constants of TEMP_FUNCTIONS.f08:95-97 and UPDATES.f08:191-195.
constexpr double kTsH = 6.62613e-19;       // erg*sh
constexpr double kTsC = 2.99792458e2;      // cm/sh
constexpr double kTsErg = 6.24150934e11;   // eV/erg

// sigint (TEMP_FUNCTIONS.f08:114-141): the integral of z^3/(e^z - 1) by its two series, blended
// linearly on (1.95, 2.05] (the INTERPOLATORS call).
__device__ __forceinline__ double ts_sigint(double z) {
  const double pi = 3.141592653589793;
  const double pi4 = (pi * pi) * (pi * pi);
  if (z <= 1.95) return ((z * z) * z) * (1.0 / 3.0 - z / 8.0 + (z * z) / 62.4);
  if (z > 2.05) return pi4 / 15.0 - exp(-z) * (((z * z) * z) + 3.0 * (z * z) + 6.0 * z + 7.28);
  const double x1 = 1.95, x2 = 2.05;
  const double y1 = ((x1 * x1) * x1) * (1.0 / 3.0 - x1 / 8.0 + (x1 * x1) / 62.4);
  const double y2 = pi4 / 15.0 - exp(-x2) * (((x2 * x2) * x2) + 3.0 * (x2 * x2) + 6.0 * x2 + 7.28);
  return y1 + (y2 - y1) * (z - x1) / (x2 - x1);
}

// Bg_planck_calc (TEMP_FUNCTIONS.f08:90-108).
__device__ __forceinline__ double ts_bg_planck(double T, double nu_low, double nu_high, double comp_unit) {
  if (T <= 1e-15) return 0.0;
  double sig = ts_sigint(nu_high / T) - ts_sigint(nu_low / T);
  const double h3 = (kTsH * kTsH) * kTsH, c2 = kTsC * kTsC, e2 = kTsErg * kTsErg;
  sig = sig / (((h3 * c2) * (e2 * e2)) * comp_unit);
  const double t2 = T * T;
  return (2.0 * (t2 * t2)) * sig;
}

// kapB_calc (TEMP_FUNCTIONS.f08:11-32): group Planck-mean opacity of the Fleck-Cummings material.
__device__ __forceinline__ double ts_kapb(double T, double nu_low, double nu_high) {
  const double sig0 = 27.0 * 1e9;
  const double z1 = nu_high / T, z2 = nu_low / T;
  const double t3 = (T * T) * T;
  if (z2 > 10.0) {
    const double sig = -exp(-(z1 - z2)) * (((z1 * z1) * z1) + 3.0 * (z1 * z1) + 6.0 * z1 + 7.28) +
                       (((z2 * z2) * z2) + 3.0 * (z2 * z2) + 6.0 * z2 + 7.28);
    return sig0 * (1.0 - exp(-(nu_high - nu_low) / T)) / (t3 * sig);
  }
  const double sig = ts_sigint(z1) - ts_sigint(z2);
  return sig0 * (exp(-nu_low / T) - exp(-nu_high / T)) / (t3 * sig);
}

// Opacity law of the synthetic configurations, in place of kapB_calc:
//   kappa_g(T) = kappa0 (1 - exp(-nu_g/T)) / (nu_g^3 sqrt(T)),  nu_g = sqrt(nu_low nu_high),
// T and nu in keV (the arguments are in eV, as everywhere else).
__device__ __forceinline__ double ts_law_kappa(double T, double nu_low, double nu_high, double kappa0) {
  const double nb = sqrt(nu_low * nu_high) * 1e-3;
  const double tk = T * 1e-3;
  return kappa0 * (-expm1(-nb / tk)) / (((nb * nb) * nb) * sqrt(tk));
}

// dBg/dT of Bg_planck_calc, Bg = 2 T^4 (sigint(nu_high/T) - sigint(nu_low/T)) / K, with the exact
// derivative of the Planck integral, d sigint(z)/dz = z^3/(e^z - 1):
//   dBg/dT = 2 T^3 (4 (sigint(z_h) - sigint(z_l)) - z_h^4/(e^z_h - 1) + z_l^4/(e^z_l - 1)) / K.
__device__ __forceinline__ double ts_bg_planck_dT(double T, double nu_low, double nu_high, double comp_unit) {
  if (T <= 1e-15) return 0.0;
  const double zh = nu_high / T, zl = nu_low / T;
  const double s = ts_sigint(zh) - ts_sigint(zl);
  const double ph = zh > 700.0 ? 0.0 : (((zh * zh) * (zh * zh)) / expm1(zh));
  const double pl = zl > 700.0 ? 0.0 : (((zl * zl) * (zl * zl)) / expm1(zl));
  const double h3 = (kTsH * kTsH) * kTsH, c2 = kTsC * kTsC, e2 = kTsErg * kTsErg;
  const double K = ((h3 * c2) * (e2 * e2)) * comp_unit;
  const double t3 = (T * T) * T;
  return ((2.0 * t3) * (((4.0 * s) - ph) + pl)) / K;
}

// Material laws of the time loops: the reference's Fleck-Cummings opacity with MEB_SOLVE, or the
// configurations' opacity law with the T^4-linearised energy balance (meb_law_kernel).
enum MaterialLaw { kLawFleckCummings = 0, kLawConfig = 1 };

// MATERIAL_UPDATE (UPDATES.f08:110-152) for the sweep: KapE = KapB = kapB_calc(T, nu_g, nu_g+1) *
// Kappa_Mult(Mat(i,j)) and the isotropic corner source RT_Src = KapB * Bg, one value per (cell, g)
// (the reference stores it for all 4 corners and N_m directions).  kmult(i,j) = Kappa_Mult(Mat(i,j)),
// or kappa0(i,j) of the configurations' law (law = kLawConfig).
// Writes the FP64 copies and the sweep's Real copies; with mgsrc set, also the low-order source
// MGQD_Src = 4 pi KapB Bg (UPDATES.f08:141).
template <class Real>
__global__ void material_update_kernel(int nx, int ny, int ng, const double* __restrict__ T,
                                       const double* __restrict__ nu, const double* __restrict__ kmult,
                                       double comp_unit, double* __restrict__ kap64, double* __restrict__ q64,
                                       Real* __restrict__ kap, Real* __restrict__ q, double* __restrict__ mgsrc,
                                       int law) {
  const long long nxy = (long long)nx * ny, n = nxy * ng;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long cell = k % nxy;
    const int g = (int)(k / nxy);
    const double Tc = T[cell];
    const double Bg = ts_bg_planck(Tc, nu[g], nu[g + 1], comp_unit);
    const double kB = law == kLawConfig ? ts_law_kappa(Tc, nu[g], nu[g + 1], kmult[cell])
                                        : ts_kapb(Tc, nu[g], nu[g + 1]) * kmult[cell];
    const double src = kB * Bg;
    kap64[k] = kB;
    q64[k] = src;
    kap[k] = (Real)kB;
    q[k] = (Real)src;
    if (mgsrc) mgsrc[k] = ((4.0 * 3.141592653589793) * kB) * Bg;
  }
}

// MEB_SOLVE (UPDATES.f08:185-230): the linearised material energy balance of the Fleck-Cummings
// problem, with the transport group energies Eg (HO_Eg_avg):
//   E = sum_g Eg,  KapE_Bar = sum_g KapE_g Eg / E,
//   T = c^2 h^3 / (c^2 h^3 cv CU + 8 pi Delt Kap0 / erg^4) * (Delt c KapE_Bar E + cv T_old) * CU.
// cv may vary per cell (the reference passes one value).
__global__ void meb_kernel(int nx, int ny, int ng, const double* __restrict__ Eg, const double* __restrict__ kapE,
                           const double* __restrict__ T_old, const double* __restrict__ cv, double Delt, double Kap0,
                           double comp_unit, double* __restrict__ T) {
  const long long nxy = (long long)nx * ny;
  const double pi = 3.141592653589793;
  const double c2h3 = (kTsC * kTsC) * ((kTsH * kTsH) * kTsH);
  const double e2 = kTsErg * kTsErg;
  const double lin = (((8.0 * pi) * Delt) * Kap0) / (e2 * e2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nxy; k += (long long)gridDim.x * blockDim.x) {
    double E = 0.0, kb = 0.0;
    for (int g = 0; g < ng; ++g) {
      const double e = Eg[k + nxy * g];
      E = E + e;
      kb = kb + kapE[k + nxy * g] * e;
    }
    kb = kb / E;
    const double cvk = cv[k];
    const double coef = c2h3 / (((c2h3 * cvk) * comp_unit) + lin);
    T[k] = (coef * ((((Delt * kTsC) * kb) * E) + cvk * T_old[k])) * comp_unit;
  }
}

// Energy balance of the configurations' material (in place of MEB_SOLVE), backward Euler per cell,
//   cv (T - T_old)/Delt = sum_g KapE_g (c Eg - 4 pi Bg(T)),
// with the emission linearised about the current iterate T* (one Newton step per outer iteration):
//   T = (cv T_old/Delt + sum_g KapE_g (c Eg - 4 pi Bg(T*) + 4 pi Bg'(T*) T*)) / (cv/Delt + 4 pi sum_g KapE_g Bg'(T*)).
// T holds T* on entry.  Eg are the transport group energies (HO_Eg_avg), KapE the material at T*.
__global__ void meb_law_kernel(int nx, int ny, int ng, const double* __restrict__ Eg, const double* __restrict__ kapE,
                               const double* __restrict__ T_old, const double* __restrict__ cv,
                               const double* __restrict__ nu, double Delt, double comp_unit, double c,
                               double* __restrict__ T) {
  const long long nxy = (long long)nx * ny;
  const double fp = 4.0 * 3.141592653589793;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nxy; k += (long long)gridDim.x * blockDim.x) {
    const double ts = T[k];
    double num = 0.0, den = 0.0;
    for (int g = 0; g < ng; ++g) {
      const double kap = kapE[k + nxy * g];
      const double B = ts_bg_planck(ts, nu[g], nu[g + 1], comp_unit);
      const double dB = ts_bg_planck_dT(ts, nu[g], nu[g + 1], comp_unit);
      num = num + kap * (((c * Eg[k + nxy * g]) - (fp * B)) + ((fp * dB) * ts));
      den = den + (fp * kap) * dB;
    }
    T[k] = (((cv[k] * T_old[k]) / Delt) + num) / ((cv[k] / Delt) + den);
  }
}

// Group-partial form of the energy balances, for time loops whose groups are split over several handles
// (ranks of a multi-GPU run, or group slabs streamed through one device): per cell the group sums each
// balance needs, over this handle's groups, into part[0..2][cell]; the sums over all handles then give the
// new temperature in meb_finish_kernel.  Fleck-Cummings (MEB_SOLVE): {sum KapE Eg, sum Eg, sum Eg};
// configurations' law: {sum KapE (c Eg - 4 pi Bg + 4 pi Bg' T*), sum 4 pi KapE Bg', sum Eg}.  The third is
// the handle's part of the transport E (HO_E_avg), whose sum the convergence test reads.
__global__ void meb_partial_kernel(int nx, int ny, int ng, int law, const double* __restrict__ Eg,
                                   const double* __restrict__ kapE, const double* __restrict__ T,
                                   const double* __restrict__ nu, double comp_unit, double c,
                                   double* __restrict__ part) {
  const long long nxy = (long long)nx * ny;
  const double fp = 4.0 * 3.141592653589793;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nxy; k += (long long)gridDim.x * blockDim.x) {
    double p0 = 0.0, p1 = 0.0, p2 = 0.0;
    const double ts = T[k];
    for (int g = 0; g < ng; ++g) {
      const double e = Eg[k + nxy * g];
      const double kap = kapE[k + nxy * g];
      if (law == kLawConfig) {
        const double B = ts_bg_planck(ts, nu[g], nu[g + 1], comp_unit);
        const double dB = ts_bg_planck_dT(ts, nu[g], nu[g + 1], comp_unit);
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
}

// The new temperature from the group sums over all handles (the expressions of meb_kernel and
// meb_law_kernel with their group sums replaced by the totals), and E_avg = the summed transport E.
__global__ void meb_finish_kernel(int nx, int ny, int law, const double* __restrict__ sum,
                                  const double* __restrict__ T_old, const double* __restrict__ cv, double Delt,
                                  double Kap0, double comp_unit, double* __restrict__ T, double* __restrict__ E_avg) {
  const long long nxy = (long long)nx * ny;
  const double pi = 3.141592653589793;
  const double c2h3 = (kTsC * kTsC) * ((kTsH * kTsH) * kTsH);
  const double e2 = kTsErg * kTsErg;
  const double lin = (((8.0 * pi) * Delt) * Kap0) / (e2 * e2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nxy; k += (long long)gridDim.x * blockDim.x) {
    const double p0 = sum[k], p1 = sum[k + nxy];
    if (law == kLawConfig) {
      T[k] = (((cv[k] * T_old[k]) / Delt) + p0) / ((cv[k] / Delt) + p1);
    } else {
      const double kb = p0 / p1;
      const double cvk = cv[k];
      const double coef = c2h3 / (((c2h3 * cvk) * comp_unit) + lin);
      T[k] = (coef * ((((Delt * kTsC) * kb) * p1) + cvk * T_old[k])) * comp_unit;
    }
    E_avg[k] = sum[k + 2 * nxy];
  }
}

// Outer-iteration convergence data of CONVERGENCE (CONVERGENCE_CHECKS.f08:7-44) for one field x
// with its last two iterates: out[0] = max|x - x_old|, out[1] = max|x_old - x_old2|, out[2] = max|x|,
// out[3] = min|x|, out[4] = max|1 - x_old/x|.  Maxima and minima of non-negative doubles are exact and
// order-independent, so they are combined with integer atomics on the bit patterns (deterministic).
// out must hold {0, 0, 0, +inf, 0} before the launch.
__global__ void conv_reduce_kernel(long long n, const double* __restrict__ x, const double* __restrict__ xo,
                                   const double* __restrict__ xo2, unsigned long long* out) {
  double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = __longlong_as_double(0x7ff0000000000000LL), v4 = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double a = x[k], b = xo[k], c = xo2[k];
    v0 = fmax(v0, fabs(a - b));
    v1 = fmax(v1, fabs(b - c));
    v2 = fmax(v2, fabs(a));
    v3 = fmin(v3, fabs(a));
    v4 = fmax(v4, fabs(1.0 - b / a));
  }
  for (int o = 16; o > 0; o >>= 1) {
    v0 = fmax(v0, __shfl_xor_sync(0xffffffffu, v0, o));
    v1 = fmax(v1, __shfl_xor_sync(0xffffffffu, v1, o));
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
    v3 = fmin(v3, __shfl_xor_sync(0xffffffffu, v3, o));
    v4 = fmax(v4, __shfl_xor_sync(0xffffffffu, v4, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(v0));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(v1));
    atomicMax(&out[2], (unsigned long long)__double_as_longlong(v2));
    atomicMin(&out[3], (unsigned long long)__double_as_longlong(v3));
    atomicMax(&out[4], (unsigned long long)__double_as_longlong(v4));
  }
}

}  // namespace trt
