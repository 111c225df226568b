// Device kernels around the sweep: layout conversion, angular exports, moment combination,
// group sums, boundary updates and residual norms.  Each one cites the reference routine whose
// result it produces.  All files are built with --fmad=false: operations written as separate
// multiply and add round twice, as in the reference Fortran.
#pragma once

#include <cuda_runtime.h>

#include "layout.cuh"
#include "sweep_kernel.cuh"

namespace trt {

constexpr double kCLight = 2.99792458e2;   // cm/sh, TRANSPORT_SOLVES.f08:403

// ---------------------------------------------------------------------------------------------
// State layout conversion: Fortran I_crn(2nx, 2ny, nm, ng) (double) <-> skewed (Real).
// ---------------------------------------------------------------------------------------------
struct Geo {
  int nx, ny, nm, ng, mq;
  Tiling t;
  long long blk;
};

template <class Real>
__device__ __forceinline__ long long state_index(const Geo& G, int i, int j, int cx, int cy, int m, int g) {
  constexpr int NV = 16 / (int)sizeof(Real);
  const int q = m / G.mq, mlq = m % G.mq;
  // split h holds quadrant-local directions [split_first(h), split_first(h) + split_count(h))
  const int NH = G.t.NH, base = G.mq / NH, rem = G.mq % NH;
  const int h = mlq < rem * (base + 1) ? mlq / (base + 1) : rem + (mlq - rem * (base + 1)) / base;
  const int ml = mlq - split_first(G.mq, NH, h);
  const SweepPos p = sweep_pos(G.nx, G.ny, G.t, q, i, j);
  const int c = frame_corner(q, cx, cy);
  return ((long long)(g * 4 + q) * NH + h) * G.blk + skew_offset<NV>(G.t, p.T, p.w, ml, p.r, c);
}

template <class Real>
__global__ void pack_state_kernel(Geo G, const double* __restrict__ fort, Real* __restrict__ skew) {
  const long long n = 4LL * G.nx * G.ny * G.nm * G.ng;
  const long long nxx = 2LL * G.nx, nyy = 2LL * G.ny;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    long long r = k;
    const int ix = (int)(r % nxx); r /= nxx;
    const int iy = (int)(r % nyy); r /= nyy;
    const int m = (int)(r % G.nm); r /= G.nm;
    const int g = (int)r;
    skew[state_index<Real>(G, ix >> 1, iy >> 1, ix & 1, iy & 1, m, g)] = (Real)fort[k];
  }
}

template <class Real>
__global__ void unpack_state_kernel(Geo G, const Real* __restrict__ skew, double* __restrict__ fort) {
  const long long n = 4LL * G.nx * G.ny * G.nm * G.ng;
  const long long nxx = 2LL * G.nx, nyy = 2LL * G.ny;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    long long r = k;
    const int ix = (int)(r % nxx); r /= nxx;
    const int iy = (int)(r % nyy); r /= nyy;
    const int m = (int)(r % G.nm); r /= G.nm;
    const int g = (int)r;
    fort[k] = (double)skew[state_index<Real>(G, ix >> 1, iy >> 1, ix & 1, iy & 1, m, g)];
  }
}

// Fill a whole skewed state with one value per group (used to initialise the state to B_g(T_ini) as
// RT_INIT does, INITIALIZERS.f08:84-92).  The (g, q, h) blocks of group g are contiguous, so this is a
// streaming store; slots that hold no (cell, direction) get the value too, which is harmless because
// the sweep never uses them as data.
template <class Real>
__global__ void fill_groups_kernel(long long per_group, int ng, const double* __restrict__ per_g,
                                   Real* __restrict__ skew) {
  const long long n = per_group * ng;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    skew[k] = (Real)per_g[k / per_group];
}

// ---------------------------------------------------------------------------------------------
// Corner-edge value Ic on a vertical face f (0..nx) at corner-edge row iy (0..2ny-1) for direction m:
// the upwind cell's corner (TRANSPORT_SOLVES.f08:86-87,133-134,180-181,227-228) or the boundary
// array on the inflow face.  Horizontal faces likewise (:88-89,135-136,182-183,229-230).
// ---------------------------------------------------------------------------------------------
template <class Real>
__device__ __forceinline__ Real icV_value(const Geo& G, const Real* st, const Real* bndV, int f, int iy, int m, int g) {
  const int q = m / G.mq;
  const bool xpos = (q == 0 || q == 3);   // Omega_x > 0
  if (xpos) {
    if (f == 0) return bndV[((size_t)(0 * G.ng + g) * G.nm + m) * 2 * G.ny + iy];
    return st[state_index<Real>(G, f - 1, iy >> 1, 1, iy & 1, m, g)];
  } else {
    if (f == G.nx) return bndV[((size_t)(1 * G.ng + g) * G.nm + m) * 2 * G.ny + iy];
    return st[state_index<Real>(G, f, iy >> 1, 0, iy & 1, m, g)];
  }
}

template <class Real>
__device__ __forceinline__ Real icH_value(const Geo& G, const Real* st, const Real* bndH, int ix, int f, int m, int g) {
  const int q = m / G.mq;
  const bool ypos = (q == 0 || q == 1);   // Omega_y > 0
  if (ypos) {
    if (f == 0) return bndH[((size_t)(0 * G.ng + g) * G.nm + m) * 2 * G.nx + ix];
    return st[state_index<Real>(G, ix >> 1, f - 1, ix & 1, 1, m, g)];
  } else {
    if (f == G.ny) return bndH[((size_t)(1 * G.ng + g) * G.nm + m) * 2 * G.nx + ix];
    return st[state_index<Real>(G, ix >> 1, f, ix & 1, 0, m, g)];
  }
}

// Angular exports in the reference layouts: I_avg(nx,ny,nm,ng) (TRANSPORT_SOLVES.f08:96),
// I_edgV(nx+1,ny,nm,ng) (:92), I_edgH(nx,ny+1,nm,ng) (:93), Ic_edgV(nx+1,2ny,nm,ng),
// Ic_edgH(2nx,ny+1,nm,ng).  Any output pointer may be null.  Values on inflow faces are the boundary
// arrays (the reference keeps the caller's values there; the host layer restores them).
// Snapshot of the cell-average angular intensity I_avg(nx, ny, nm, ng) = mean of the four corner values
// (TRANSPORT_SOLVES.f08 forms I_avg so), written as 4-byte floats into a caller's device store.
// Groups g0 .. g0+ngs-1 only (out holds those groups, group-slowest).
template <class Real>
__global__ void snapshot_avg_kernel(Geo G, const Real* __restrict__ st, float* __restrict__ out, int g0, int ngs) {
  const long long nA = (long long)G.nx * G.ny * G.nm * ngs;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nA; k += (long long)gridDim.x * blockDim.x) {
    long long r = k;
    const int i = (int)(r % G.nx); r /= G.nx;
    const int j = (int)(r % G.ny); r /= G.ny;
    const int m = (int)(r % G.nm);
    const int g = g0 + (int)(r / G.nm);
    const double lb = (double)st[state_index<Real>(G, i, j, 0, 0, m, g)];
    const double rb = (double)st[state_index<Real>(G, i, j, 1, 0, m, g)];
    const double rt = (double)st[state_index<Real>(G, i, j, 1, 1, m, g)];
    const double lt = (double)st[state_index<Real>(G, i, j, 0, 1, m, g)];
    out[k] = (float)((lb + rb + rt + lt) / 4.0);
  }
}

template <class Real>
__global__ void export_angular_kernel(Geo G, const Real* __restrict__ st, const Real* __restrict__ bndV,
                                      const Real* __restrict__ bndH, double* I_avg, double* I_edgV, double* I_edgH,
                                      double* Ic_edgV, double* Ic_edgH) {
  const int nx = G.nx, ny = G.ny, nm = G.nm, ng = G.ng;
  const long long nA = (long long)nx * ny * nm * ng;
  const long long nV = (long long)(nx + 1) * ny * nm * ng;
  const long long nH = (long long)nx * (ny + 1) * nm * ng;
  const long long ncV = (long long)(nx + 1) * 2 * ny * nm * ng;
  const long long ncH = (long long)2 * nx * (ny + 1) * nm * ng;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (I_avg)
    for (long long k = k0; k < nA; k += stride) {
      long long r = k;
      const int i = (int)(r % nx); r /= nx;
      const int j = (int)(r % ny); r /= ny;
      const int m = (int)(r % nm);
      const int g = (int)(r / nm);
      const double lb = (double)st[state_index<Real>(G, i, j, 0, 0, m, g)];
      const double rb = (double)st[state_index<Real>(G, i, j, 1, 0, m, g)];
      const double rt = (double)st[state_index<Real>(G, i, j, 1, 1, m, g)];
      const double lt = (double)st[state_index<Real>(G, i, j, 0, 1, m, g)];
      I_avg[k] = (lb + rb + rt + lt) / 4.0;
    }
  if (I_edgV)
    for (long long k = k0; k < nV; k += stride) {
      long long r = k;
      const int f = (int)(r % (nx + 1)); r /= (nx + 1);
      const int j = (int)(r % ny); r /= ny;
      const int m = (int)(r % nm);
      const int g = (int)(r / nm);
      const double b = (double)icV_value<Real>(G, st, bndV, f, 2 * j, m, g);
      const double t = (double)icV_value<Real>(G, st, bndV, f, 2 * j + 1, m, g);
      I_edgV[k] = (b + t) / 2.0;
    }
  if (I_edgH)
    for (long long k = k0; k < nH; k += stride) {
      long long r = k;
      const int i = (int)(r % nx); r /= nx;
      const int f = (int)(r % (ny + 1)); r /= (ny + 1);
      const int m = (int)(r % nm);
      const int g = (int)(r / nm);
      const double l = (double)icH_value<Real>(G, st, bndH, 2 * i, f, m, g);
      const double rr = (double)icH_value<Real>(G, st, bndH, 2 * i + 1, f, m, g);
      I_edgH[k] = (l + rr) / 2.0;
    }
  if (Ic_edgV)
    for (long long k = k0; k < ncV; k += stride) {
      long long r = k;
      const int f = (int)(r % (nx + 1)); r /= (nx + 1);
      const int iy = (int)(r % (2 * ny)); r /= (2 * ny);
      const int m = (int)(r % nm);
      const int g = (int)(r / nm);
      Ic_edgV[k] = (double)icV_value<Real>(G, st, bndV, f, iy, m, g);
    }
  if (Ic_edgH)
    for (long long k = k0; k < ncH; k += stride) {
      long long r = k;
      const int ix = (int)(r % (2 * nx)); r /= (2 * nx);
      const int f = (int)(r % (ny + 1)); r /= (ny + 1);
      const int m = (int)(r % nm);
      const int g = (int)(r / nm);
      Ic_edgH[k] = (double)icH_value<Real>(G, st, bndH, ix, f, m, g);
    }
}

// ---------------------------------------------------------------------------------------------
// Combination of the quadrant partials into the reference's low-order inputs.
//   COLLAPSE_INTENSITIES  TRANSPORT_SOLVES.f08:441-478  (Hg_*, HO_Eg_*, HO_Fxg_edgV, HO_Fyg_edgH)
//   fg_Calc               MLOQD_SOLVES.f08:646-674
//   Cg_Calc               MLOQD_SOLVES.f08:392-484
//   MGQD_In_Calc          MLOQD_SOLVES.f08:517-610
// The reference adds eps = 1e-25/Comp_Unit to every intensity in the moment and C_g sums; here the
// sums of the intensities are taken first and eps times the matching sum of weights is added in
// FP64 (the same value up to rounding, and finite where FP32 intensities underflow).
// ---------------------------------------------------------------------------------------------
struct MomentOut {
  double *Hg_avg_xx, *Hg_avg_yy, *Hg_avg_xy, *Hg_edgV_xx, *Hg_edgV_xy, *Hg_edgH_yy, *Hg_edgH_xy;
  double *Eg_avg, *Eg_edgV, *Eg_edgH, *Fxg_edgV, *Fyg_edgH;
  double *fg_avg_xx, *fg_avg_yy, *fg_avg_xy, *fg_edgV_xx, *fg_edgV_xy, *fg_edgH_yy, *fg_edgH_xy;
  double *Cg_L, *Cg_B, *Cg_R, *Cg_T;
  double *Eg_in_L, *Eg_in_B, *Eg_in_R, *Eg_in_T, *Fg_in_L, *Fg_in_B, *Fg_in_R, *Fg_in_T;
  double *E_avg, *E_edgV, *E_edgH, *Fx_edgV, *Fy_edgH;
  double *E_in_L, *E_in_B, *E_in_R, *E_in_T, *F_in_L, *F_in_B, *F_in_R, *F_in_T;
  double *Fyg_edgH_true, *Fy_edgH_true;   // Omega_y-weighted horizontal-face flux (physics reporting)
};

// Per-quadrant weight sums for the analytic eps terms: [q][kNDirRow] over the mq directions.
struct WeightSums {
  double s[4][kNDirRow];
};

struct CombineArgs {
  int nx, ny, nm, ng, mq;
  double eps;          // 1e-25 / Comp_Unit
  double c;            // speed of light used by fg_Calc (passed in by the reference's caller)
  int bc[4];           // BC_Type L, B, R, T
  int nh;              // direction splits per quadrant (partials per quadrant)
  WeightSums ws;
  const void* part;    // [4*nh][ng][ny][nx][part_rec<Real>()] partial records (Real = state precision)
  const double* dir;   // [kNDirRow][nm] full direction table (physical), double
};

// Sum over the directions of quadrant q of w*f(Omega)*(Ic_bot + Ic_top)/2 on an inflow face.
template <class Real>
__device__ __forceinline__ void inflow_face_sums(const CombineArgs& A, const Real* bnd, int side, int g, int q,
                                                 int pos, int len2, double* out /*[kNDirRow]*/) {
  for (int v = 0; v < kNDirRow; ++v) out[v] = 0.0;
  for (int ml = 0; ml < A.mq; ++ml) {
    const int m = q * A.mq + ml;
    const Real* b = bnd + ((size_t)(side * A.ng + g) * A.nm + m) * len2;
    const double I = ((double)b[2 * pos] + (double)b[2 * pos + 1]) / 2.0;
    for (int v = kW; v < kNDirRow; ++v) out[v] += A.dir[v * A.nm + m] * I;
  }
}

// Moment epilogue, interior part.  A CTA takes a tile of kCombTX x kCombTY cells of one group; for
// each (quadrant q, split h) in turn it stages the tile's partial records, plus the column on its
// left (q = 0, 3) or the row below it (q = 0, 1) where a face needs them, into shared memory with
// coalesced 16-byte cp.async copies (double-buffered: the copies of the next (q, h) fly while this
// one is added), then every thread adds the record slots of its cell (i, j) to
//   * the cell-centre moments (COLLAPSE_INTENSITIES :446-449, fg_Calc :63-65),
//   * the vertical face f = i when i >= 1 (:450-452, :458; fg_Calc :66-67),
//   * the horizontal face f = j when j >= 1 (:453-455, :469; fg_Calc :68-69).
// The boundary faces (f = 0, nx and f = 0, ny) are left to combine_boundary_kernel.  Each sum adds
// the quadrant partials in the order q = 0..3, split h = 0..NH-1 inside, then the analytic eps term.
constexpr int kCombTX = 32, kCombTY = 8;
constexpr int kCombRow = kCombTX + 1;                                 // records per staged row
// Staged record stride in shared memory: 112-byte FP64 records are conflict-free for 16-byte loads
// as they are; 64-byte FP32 records are padded to 80 bytes (8 consecutive records then cover all
// 32 banks).
template <class P>
__host__ __device__ constexpr int comb_rec_stride() { return sizeof(P) == 4 ? 20 : 14; }
template <class P>
__host__ __device__ constexpr size_t comb_smem() {   // two staging buffers of records of type P
  return 2 * (size_t)(kCombTY + 1) * kCombRow * comb_rec_stride<P>() * sizeof(P);
}

// Slots a..a+3 (a a multiple of 4) of a staged record as doubles.
__device__ __forceinline__ void rec4(const double* p, int a, double (&v)[4]) {
  const double2 x = *reinterpret_cast<const double2*>(p + a), y = *reinterpret_cast<const double2*>(p + a + 2);
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
__device__ __forceinline__ void rec4(const float* p, int a, double (&v)[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p + a);
  v[0] = (double)x.x; v[1] = (double)x.y; v[2] = (double)x.z; v[3] = (double)x.w;
}

template <class P>
__global__ void __launch_bounds__(kCombTX * kCombTY) combine_cells_kernel(CombineArgs A, MomentOut O) {
  // two staging buffers [kCombTY + 1][kCombRow][kRecS]; row 0 / column 0 = halo
  extern __shared__ __align__(16) unsigned char comb_smem_raw[];
  P* rec = reinterpret_cast<P*>(comb_smem_raw);
  constexpr int kRec = part_rec<P>(), kRecS = comb_rec_stride<P>();
  constexpr int kPerVec = 16 / (int)sizeof(P);          // values per 16-byte vector
  const int nx = A.nx, ny = A.ny, ng = A.ng, NH = A.nh;
  const int tx = threadIdx.x % kCombTX, ty = threadIdx.x / kCombTX;
  const int i0 = blockIdx.x * kCombTX, j0 = blockIdx.y * kCombTY, g = blockIdx.z;
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i < nx && j < ny;
  const int ncol = min(kCombTX, nx - i0), nrow = min(kCombTY, ny - j0);
  const double eps = A.eps, c = A.c;
  auto wsum = [&](int v) { return A.ws.s[0][v] + A.ws.s[1][v] + A.ws.s[2][v] + A.ws.s[3][v]; };
  constexpr int kV2 = kRec * (int)sizeof(P) / 16;     // 16-byte vectors per record
  constexpr size_t kBuf = (size_t)(kCombTY + 1) * kCombRow * kRecS;

  // issue the copies of (q, h) = qh into buffer b (asynchronous, one commit group)
  auto stage = [&](int qh, int b) {
    const int q = qh / NH;
    const bool left_halo = (q == 0 || q == 3) && i0 > 0;   // vertical faces take cell i - 1
    const bool low_halo = (q == 0 || q == 1) && j0 > 0;    // horizontal faces take cell j - 1
    const int c0 = left_halo ? 0 : 1, r0 = low_halo ? 0 : 1;
    const int rowlen = (ncol + 1 - c0) * kV2;              // vectors per staged row
    const int nvec = (nrow + 1 - r0) * rowlen;
    const uint4* src = reinterpret_cast<const uint4*>(static_cast<const P*>(A.part) + ((size_t)(qh * ng + g) * ny * nx) * kRec);
    P* dst = rec + b * kBuf;
    for (int v = threadIdx.x; v < nvec; v += kCombTX * kCombTY) {
      const int rr = r0 + v / rowlen, e = v % rowlen;      // staged row, vector within the row
      const int rc = c0 + e / kV2, part = e % kV2;          // staged record (column), vector within it
      cp_async16(dst + (rr * kCombRow + rc) * kRecS + part * kPerVec,
                 src + ((size_t)(j0 - 1 + rr) * nx + (i0 - 1 + c0)) * kV2 + e);
    }
    cp_async_commit();
  };

  double cxx = 0, cyy = 0, cxy = 0, ce = 0;            // centre
  double vxx = 0, vxy = 0, vx = 0, ve = 0;             // vertical face f = i
  double hyy = 0, hxy = 0, hy = 0, hx = 0, he = 0;     // horizontal face f = j
  const int nqh = 4 * NH;
  stage(0, 0);
  for (int qh = 0; qh < nqh; ++qh) {
    const int q = qh / NH;
    if (qh + 1 < nqh) {
      stage(qh + 1, (qh + 1) & 1);   // that buffer was released by the barrier ending step qh - 1
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (in) {
      const P* own = rec + (qh & 1) * kBuf + ((size_t)(ty + 1) * kCombRow + tx + 1) * kRecS;
      double u[4];
      rec4(own, kCxx, u);
      cxx += u[0]; cyy += u[1]; cxy += u[2]; ce += u[3];
      const P* pv = (q == 0 || q == 3) ? own - kRecS : own;
      rec4(pv, kVxx, u);
      vxx += u[0]; vxy += u[1]; vx += u[2]; ve += u[3];
      const P* ph = (q == 0 || q == 1) ? own - (size_t)kCombRow * kRecS : own;
      rec4(ph, kHyy, u);
      hyy += u[0]; hxy += u[1]; hy += u[2]; hx += u[3]; he += (double)ph[kHe];
    }
    __syncthreads();   // buffer qh & 1 is consumed
  }
  if (!in) return;
  const long long k = i + (long long)nx * (j + (long long)ny * g);
  {
    cxx += eps * wsum(kWxx); cyy += eps * wsum(kWyy); cxy += eps * wsum(kWxy); ce += eps * wsum(kW);
    const double Eg = ce / kCLight;
    if (O.Hg_avg_xx) { O.Hg_avg_xx[k] = cxx; O.Hg_avg_yy[k] = cyy; O.Hg_avg_xy[k] = cxy; }
    if (O.Eg_avg) O.Eg_avg[k] = Eg;
    if (O.fg_avg_xx) {
      O.fg_avg_xx[k] = cxx / (c * Eg);
      O.fg_avg_yy[k] = cyy / (c * Eg);
      O.fg_avg_xy[k] = cxy / (c * Eg);
    }
  }
  if (i >= 1) {
    vxx += eps * wsum(kWxx); vxy += eps * wsum(kWxy); vx += eps * wsum(kWx); ve += eps * wsum(kW);
    const double Eg = ve / kCLight;
    const long long kv = i + (long long)(nx + 1) * (j + (long long)ny * g);
    if (O.Hg_edgV_xx) { O.Hg_edgV_xx[kv] = vxx; O.Hg_edgV_xy[kv] = vxy; }
    if (O.Eg_edgV) O.Eg_edgV[kv] = Eg;
    if (O.Fxg_edgV) O.Fxg_edgV[kv] = vx;
    if (O.fg_edgV_xx) { O.fg_edgV_xx[kv] = vxx / (c * Eg); O.fg_edgV_xy[kv] = vxy / (c * Eg); }
  }
  if (j >= 1) {
    hyy += eps * wsum(kWyy); hxy += eps * wsum(kWxy); hy += eps * wsum(kWy); hx += eps * wsum(kWx);
    he += eps * wsum(kW);
    const double Eg = he / kCLight;
    const long long kh = i + (long long)nx * (j + (long long)(ny + 1) * g);
    if (O.Hg_edgH_yy) { O.Hg_edgH_yy[kh] = hyy; O.Hg_edgH_xy[kh] = hxy; }
    if (O.Eg_edgH) O.Eg_edgH[kh] = Eg;
    if (O.Fyg_edgH) O.Fyg_edgH[kh] = hx;           // Omega_x weighted, as TRANSPORT_SOLVES.f08:469
    if (O.Fyg_edgH_true) O.Fyg_edgH_true[kh] = hy;
    if (O.fg_edgH_yy) { O.fg_edgH_yy[kh] = hyy / (c * Eg); O.fg_edgH_xy[kh] = hxy / (c * Eg); }
  }
}

// Moment epilogue, boundary faces: one thread per face of the four domain edges (vertical faces
// f = 0, nx; horizontal faces f = 0, ny).  Outgoing quadrants add their partials (and give Cg,
// Cg_Calc :156-203); incoming quadrants add the caller's boundary intensity, Ic averaged over the
// face's two corner values (and give E_in/F_in, MGQD_In_Calc :125-178).
template <class Real>
__global__ void combine_boundary_kernel(CombineArgs A, const Real* __restrict__ bndV, const Real* __restrict__ bndH,
                                        MomentOut O) {
  const int nx = A.nx, ny = A.ny, ng = A.ng;
  const long long nVb = 2LL * ny * ng, nHb = 2LL * nx * ng;
  const long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const double eps = A.eps, c = A.c;
  const int NH = A.nh;
  // partial slot v of (q, h) = qh at cell (i, j) of group g
  auto P = [&](int qh, int g, int i, int j, int v) {
    return (double)static_cast<const Real*>(A.part)[(((size_t)(qh * ng + g) * ny + j) * nx + i) * part_rec<Real>() + v];
  };
  auto wsum = [&](int v) { return A.ws.s[0][v] + A.ws.s[1][v] + A.ws.s[2][v] + A.ws.s[3][v]; };

  for (long long t = k0; t < nVb + nHb; t += stride) {
    if (t < nVb) {
      // vertical boundary face: t = j + ny*(g + ng*side), f = 0 (side 0) or nx (side 1)
      const int j = (int)(t % ny), g = (int)((t / ny) % ng), side = (int)(t / ((long long)ny * ng));
      const int f = side ? nx : 0;
      const long long k = f + (long long)(nx + 1) * (j + (long long)ny * g);
      double xx = 0, xy = 0, fxs = 0, e = 0;
      double outF = 0, outE = 0;     // outgoing sums on the face (Cg)
      double inF = 0, inE = 0;       // incoming sums on the face (MGQD_In_Calc)
      for (int q = 0; q < 4; ++q) {
        const bool xpos = (q == 0 || q == 3);
        const int cell = xpos ? f - 1 : f;     // upwind cell of this face for quadrant q
        if (cell >= 0 && cell < nx) {
          for (int h = 0; h < NH; ++h) {
            const int qh = q * NH + h;
            const double vx = P(qh, g, cell, j, kVx), ve = P(qh, g, cell, j, kVe);
            xx += P(qh, g, cell, j, kVxx); xy += P(qh, g, cell, j, kVxy); fxs += vx; e += ve;
            outF += vx; outE += ve;
          }
        } else {
          double sm[kNDirRow];
          inflow_face_sums<Real>(A, bndV, side, g, q, j, 2 * ny, sm);
          xx += sm[kWxx]; xy += sm[kWxy]; fxs += sm[kWx]; e += sm[kW];
          inF += sm[kWx]; inE += sm[kW];
        }
      }
      xx += eps * wsum(kWxx); xy += eps * wsum(kWxy); fxs += eps * wsum(kWx); e += eps * wsum(kW);
      const double Eg = e / kCLight;
      if (O.Hg_edgV_xx) { O.Hg_edgV_xx[k] = xx; O.Hg_edgV_xy[k] = xy; }
      if (O.Eg_edgV) O.Eg_edgV[k] = Eg;
      if (O.Fxg_edgV) O.Fxg_edgV[k] = fxs;
      if (O.fg_edgV_xx) { O.fg_edgV_xx[k] = xx / (c * Eg); O.fg_edgV_xy[k] = xy / (c * Eg); }
      const int bside = side ? 2 : 0;   // BC_Type index: L = 0, R = 2
      // outgoing quadrants of this face: left face -> q 1,2 ; right face -> q 0,3
      const int qa = side ? 0 : 1, qb = side ? 3 : 2;
      const long long bi = (long long)j + (long long)ny * g;
      double* Cg = side ? O.Cg_R : O.Cg_L;
      double* Ein = side ? O.Eg_in_R : O.Eg_in_L;
      double* Fin = side ? O.Fg_in_R : O.Fg_in_L;
      if (Cg) {
        if (A.bc[bside] == 0) {
          const double num = outF + eps * (A.ws.s[qa][kWx] + A.ws.s[qb][kWx]);
          const double den = outE + eps * (A.ws.s[qa][kW] + A.ws.s[qb][kW]);
          Cg[bi] = num / den;
        } else {
          Cg[bi] = 0.0;
        }
      }
      if (Ein) {
        if (A.bc[bside] == 0) { Ein[bi] = inE / kCLight; Fin[bi] = inF; }
        else { Ein[bi] = 0.0; Fin[bi] = 0.0; }
      }
    } else {
      // horizontal boundary face: t - nVb = i + nx*(g + ng*side), f = 0 (side 0) or ny (side 1)
      const long long u = t - nVb;
      const int i = (int)(u % nx), g = (int)((u / nx) % ng), side = (int)(u / ((long long)nx * ng));
      const int f = side ? ny : 0;
      const long long k = i + (long long)nx * (f + (long long)(ny + 1) * g);
      double yy = 0, xy = 0, fys = 0, fxq = 0, e = 0;
      double outF = 0, outE = 0, inF = 0, inE = 0;
      for (int q = 0; q < 4; ++q) {
        const bool ypos = (q == 0 || q == 1);
        const int cell = ypos ? f - 1 : f;
        if (cell >= 0 && cell < ny) {
          for (int h = 0; h < NH; ++h) {
            const int qh = q * NH + h;
            const double hy = P(qh, g, i, cell, kHy), he = P(qh, g, i, cell, kHe);
            yy += P(qh, g, i, cell, kHyy); xy += P(qh, g, i, cell, kHxy); fys += hy; fxq += P(qh, g, i, cell, kHx);
            e += he;
            outF += hy; outE += he;
          }
        } else {
          double sm[kNDirRow];
          inflow_face_sums<Real>(A, bndH, side, g, q, i, 2 * nx, sm);
          yy += sm[kWyy]; xy += sm[kWxy]; fys += sm[kWy]; fxq += sm[kWx]; e += sm[kW];
          inF += sm[kWy]; inE += sm[kW];
        }
      }
      yy += eps * wsum(kWyy); xy += eps * wsum(kWxy); fys += eps * wsum(kWy); fxq += eps * wsum(kWx);
      e += eps * wsum(kW);
      const double Eg = e / kCLight;
      if (O.Hg_edgH_yy) { O.Hg_edgH_yy[k] = yy; O.Hg_edgH_xy[k] = xy; }
      if (O.Eg_edgH) O.Eg_edgH[k] = Eg;
      if (O.Fyg_edgH) O.Fyg_edgH[k] = fxq;           // Omega_x weighted, as TRANSPORT_SOLVES.f08:469
      if (O.Fyg_edgH_true) O.Fyg_edgH_true[k] = fys;
      if (O.fg_edgH_yy) { O.fg_edgH_yy[k] = yy / (c * Eg); O.fg_edgH_xy[k] = xy / (c * Eg); }
      const int bside = side ? 3 : 1;   // BC_Type index: B = 1, T = 3
      // outgoing quadrants: bottom face -> q 2,3 ; top face -> q 0,1
      const int qa = side ? 0 : 2, qb = side ? 1 : 3;
      const long long bi = (long long)i + (long long)nx * g;
      double* Cg = side ? O.Cg_T : O.Cg_B;
      double* Ein = side ? O.Eg_in_T : O.Eg_in_B;
      double* Fin = side ? O.Fg_in_T : O.Fg_in_B;
      if (Cg) {
        if (A.bc[bside] == 0) {
          const double num = outF + eps * (A.ws.s[qa][kWy] + A.ws.s[qb][kWy]);
          const double den = outE + eps * (A.ws.s[qa][kW] + A.ws.s[qb][kW]);
          Cg[bi] = num / den;
        } else {
          Cg[bi] = 0.0;
        }
      }
      if (Ein) {
        if (A.bc[bside] == 0) { Ein[bi] = inE / kCLight; Fin[bi] = inF; }
        else { Ein[bi] = 0.0; Fin[bi] = 0.0; }
      }
    }
  }
}

// Group sums: COLLAPSE_INTENSITIES totals (TRANSPORT_SOLVES.f08:488-509, sequential in g) and
// GQD_In_Calc (GLOQD_SOLVES.f08:276-288).  One thread per (output array, point), groups added in
// the order g = 0..ng-1.  Work items: E_avg (nx*ny), E_edgV and Fx_edgV ((nx+1)*ny each), E_edgH,
// Fy_edgH, Fy_edgH_true (nx*(ny+1) each), E_in/F_in on L and R (ny each) and on B and T (nx each).
__host__ __device__ inline long long group_sum_items(int nx, int ny) {
  return (long long)nx * ny + 2LL * (nx + 1) * ny + 3LL * nx * (ny + 1) + 4LL * ny + 4LL * nx;
}

__global__ void group_sum_kernel(int nx, int ny, int ng, MomentOut O) {
  const long long nA = (long long)nx * ny, nV = (long long)(nx + 1) * ny, nH = (long long)nx * (ny + 1);
  const long long seg_n[14] = {nA, nV, nV, nH, nH, nH, ny, ny, ny, ny, nx, nx, nx, nx};
  const double* src[14] = {O.Eg_avg, O.Eg_edgV, O.Fxg_edgV, O.Eg_edgH, O.Fyg_edgH, O.Fyg_edgH_true,
                           O.Eg_in_L, O.Eg_in_R, O.Fg_in_L, O.Fg_in_R, O.Eg_in_B, O.Eg_in_T, O.Fg_in_B, O.Fg_in_T};
  double* dst[14] = {O.E_avg, O.E_edgV, O.Fx_edgV, O.E_edgH, O.Fy_edgH, O.Fy_edgH_true,
                     O.E_in_L, O.E_in_R, O.F_in_L, O.F_in_R, O.E_in_B, O.E_in_T, O.F_in_B, O.F_in_T};
  const long long total = group_sum_items(nx, ny);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
    long long p = t;
    int a = 0;
    while (p >= seg_n[a]) p -= seg_n[a++];
    if (!src[a] || !dst[a]) continue;
    const double* x = src[a] + p;
    const long long n = seg_n[a];
    double s = 0.0;
    int g = 0;
    for (; g + 8 <= ng; g += 8) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = x[n * (g + u)];
#pragma unroll
      for (int u = 0; u < 8; ++u) s = s + v[u];
    }
    for (; g < ng; ++g) s = s + x[n * g];
    dst[a][p] = s;
  }
}

// ---------------------------------------------------------------------------------------------
// Boundary arrays (RT_BC_UPDATE, UPDATES.f08:12-105).  Planck sides (type 0) get one value per
// (side, g) on the inflow directions; reflective sides (type 1) copy the mirrored outflow direction.
// bndV[side][g][m][2ny] holds Ic_edgV on x = 0 (side 0) and x = nx (side 1); bndH likewise.
// ---------------------------------------------------------------------------------------------
template <class Real>
__global__ void bc_update_kernel(int nx, int ny, int nm, int ng, int4 bc, const double* __restrict__ bval /*[4][ng]*/,
                                 Real* bndV, Real* bndH) {
  const int q = nm / 4;
  const long long nVtot = 2LL * ng * nm * 2 * ny, nHtot = 2LL * ng * nm * 2 * nx;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long k = k0; k < nVtot; k += stride) {
    const int iy = (int)(k % (2 * ny));
    const int m = (int)((k / (2 * ny)) % nm);
    const int g = (int)((k / (2LL * ny * nm)) % ng);
    const int side = (int)(k / (2LL * ny * nm * ng));
    const int type = side == 0 ? bc.x : bc.z;
    const bool inflow = side == 0 ? (m < q || m >= 3 * q) : (m >= q && m < 3 * q);
    if (!inflow) continue;
    if (type == 0) {
      bndV[k] = (Real)bval[(side == 0 ? 0 : 2) * ng + g];
    } else if (type == 1) {
      int src;
      if (side == 0) src = (m < q) ? m + q : m - q;        // :36-43
      else src = (m < 2 * q) ? m - q : m + q;              // :74-81
      bndV[k] = bndV[k + (long long)(src - m) * 2 * ny];
    }
  }
  for (long long k = k0; k < nHtot; k += stride) {
    const int ix = (int)(k % (2 * nx));
    const int m = (int)((k / (2 * nx)) % nm);
    const int g = (int)((k / (2LL * nx * nm)) % ng);
    const int side = (int)(k / (2LL * nx * nm * ng));
    (void)ix; (void)g;
    const int type = side == 0 ? bc.y : bc.w;
    const bool inflow = side == 0 ? (m < 2 * q) : (m >= 2 * q);
    if (!inflow) continue;
    if (type == 0) {
      bndH[k] = (Real)bval[(side == 0 ? 1 : 3) * ng + g];
    } else if (type == 1) {
      int src;
      if (side == 0) src = (m < q) ? m + 3 * q : m + q;     // :55-62
      else src = (m < 3 * q) ? m - q : m - 3 * q;           // :93-100
      bndH[k] = bndH[k + (long long)(src - m) * 2 * nx];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Residual norms of the corner balance equations, TRANSPORT_SOLVES.f08:249-323, same operation
// order and the same loop order per (quadrant, group), so results agree bit for bit with a
// sequential evaluation on identical inputs.  One thread per (m, g); a second pass takes the
// maxima over the directions of each quadrant in direction order.
// ---------------------------------------------------------------------------------------------
template <class Real>
struct ResidualArgs {
  Geo G;
  const double* omx; const double* omy;
  const double* dx; const double* dy; const double* area;
  const double* kap;            // KapE_in (nx,ny,ng), double
  double rcdt;
  const Real* Inew; const Real* Iold;
  const Real* qiso;             // isotropic source (nx,ny,ng) or null
  const Real* srcfull;          // skewed full source or null
  const Real* bndV; const Real* bndH;
  double* per_m;                // [ng][nm][5]  max, L1, L2, area-L1, area-L2 per direction
  int* per_m_loc;               // [ng][nm][2]  (i, j) of the max, 1-based; 0 when no residual > 0
};

template <class Real>
__global__ void residual_kernel(ResidualArgs<Real> a) {
  const Geo& G = a.G;
  const int nx = G.nx, ny = G.ny, nm = G.nm, ng = G.ng;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nm * ng) return;
  const int m = k % nm, g = k / nm;
  const double Ox = a.omx[m], Oy = a.omy[m];
  double vmax = 0.0, sums[4] = {0.0, 0.0, 0.0, 0.0};
  int li = 0, lj = 0;
  for (int j = 0; j < ny; ++j) {
    for (int i = 0; i < nx; ++i) {
      const double Aij = a.area[i + (long long)nx * j];
      const double kp = a.kap[i + (long long)nx * (j + (long long)ny * g)] + a.rcdt;
      const double dxx = a.dx[i], dyy = a.dy[j];
      double I[2][2], Sr[2][2];
      for (int cx = 0; cx < 2; ++cx)
        for (int cy = 0; cy < 2; ++cy) {
          const long long si = state_index<Real>(G, i, j, cx, cy, m, g);
          I[cx][cy] = (double)a.Inew[si];
          const double io = (double)a.Iold[si];
          const double sv = a.srcfull ? (double)a.srcfull[si] : (double)a.qiso[i + (long long)nx * (j + (long long)ny * g)];
          Sr[cx][cy] = fma(io, a.rcdt, sv);
        }
      const double vL_b = (double)icV_value<Real>(G, a.Inew, a.bndV, i, 2 * j, m, g);
      const double vL_t = (double)icV_value<Real>(G, a.Inew, a.bndV, i, 2 * j + 1, m, g);
      const double vR_b = (double)icV_value<Real>(G, a.Inew, a.bndV, i + 1, 2 * j, m, g);
      const double vR_t = (double)icV_value<Real>(G, a.Inew, a.bndV, i + 1, 2 * j + 1, m, g);
      const double hB_l = (double)icH_value<Real>(G, a.Inew, a.bndH, 2 * i, j, m, g);
      const double hB_r = (double)icH_value<Real>(G, a.Inew, a.bndH, 2 * i + 1, j, m, g);
      const double hT_l = (double)icH_value<Real>(G, a.Inew, a.bndH, 2 * i, j + 1, m, g);
      const double hT_r = (double)icH_value<Real>(G, a.Inew, a.bndH, 2 * i + 1, j + 1, m, g);
      double res[4];
      res[0] = fabs((Ox * dyy + Oy * dxx + kp * Aij) * I[0][0] / 4.0 + Ox * dyy * I[1][0] / 4.0 +
                    Oy * dxx * I[0][1] / 4.0 - Ox * dyy * vL_b / 2.0 - Oy * dxx * hB_l / 2.0 - Aij * Sr[0][0] / 4.0);
      res[1] = fabs((-Ox * dyy + Oy * dxx + kp * Aij) * I[1][0] / 4.0 - Ox * dyy * I[0][0] / 4.0 +
                    Oy * dxx * I[1][1] / 4.0 + Ox * dyy * vR_b / 2.0 - Oy * dxx * hB_r / 2.0 - Aij * Sr[1][0] / 4.0);
      res[2] = fabs((-Ox * dyy - Oy * dxx + kp * Aij) * I[1][1] / 4.0 - Ox * dyy * I[0][1] / 4.0 -
                    Oy * dxx * I[1][0] / 4.0 + Ox * dyy * vR_t / 2.0 + Oy * dxx * hT_r / 2.0 - Aij * Sr[1][1] / 4.0);
      res[3] = fabs((Ox * dyy - Oy * dxx + kp * Aij) * I[0][1] / 4.0 + Ox * dyy * I[1][1] / 4.0 -
                    Oy * dxx * I[0][0] / 4.0 - Ox * dyy * vL_t / 2.0 + Oy * dxx * hT_l / 2.0 - Aij * Sr[0][1] / 4.0);
      for (int kk = 0; kk < 4; ++kk) {
        if (res[kk] > vmax) { vmax = res[kk]; li = i + 1; lj = j + 1; }
        sums[0] = sums[0] + res[kk];
        sums[1] = sums[1] + res[kk] * res[kk];
        sums[2] = sums[2] + Aij * res[kk] / 4.0;
        sums[3] = sums[3] + Aij * (res[kk] * res[kk]) / 4.0;
      }
    }
  }
  double* o = a.per_m + ((size_t)g * nm + m) * 5;
  o[0] = vmax; o[1] = sums[0]; o[2] = sums[1]; o[3] = sums[2]; o[4] = sums[3];
  int* l = a.per_m_loc + ((size_t)g * nm + m) * 2;
  l[0] = li; l[1] = lj;
}

// RT_Residual(4, ng, 5), RT_ResLoc_x/y(4, ng, 5): maxima over the directions of each quadrant in
// direction order, strictly greater replaces (TRANSPORT_SOLVES.f08:297-317).  The location of a sum
// norm is the DO-loop exit value (N_x+1, N_y+1), as in the reference.
__global__ void residual_reduce_kernel(int nx, int ny, int nm, int ng, const double* per_m, const int* per_m_loc,
                                       double* res, int* locx, int* locy) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 4 * ng) return;
  const int q = k % 4, g = k / 4;
  const int mq = nm / 4;
  double best[5] = {0, 0, 0, 0, 0};
  for (int ml = 0; ml < mq; ++ml) {
    const int m = q * mq + ml;
    const double* o = per_m + ((size_t)g * nm + m) * 5;
    const int* l = per_m_loc + ((size_t)g * nm + m) * 2;
    if (o[0] > best[0]) {
      best[0] = o[0];
      locx[q + 4 * g] = l[0];
      locy[q + 4 * g] = l[1];
    }
    for (int v = 1; v < 5; ++v)
      if (o[v] > best[v]) {
        best[v] = o[v];
        locx[q + 4 * (g + ng * v)] = nx + 1;
        locy[q + 4 * (g + ng * v)] = ny + 1;
      }
  }
  for (int v = 0; v < 5; ++v) res[q + 4 * (g + ng * v)] = best[v];
}

}  // namespace trt
