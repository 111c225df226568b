// SCB transport sweep with fused angular-moment epilogue (sm_100a).
//
// Replaces the per-group OpenMP loop of TRANSPORT_SCB (MainSrc/TRANSPORT_SOLVES.f08:50-244) and the
// angular sums of COLLAPSE_INTENSITIES (TRANSPORT_SOLVES.f08:441-478).  Layout and work
// decomposition: layout.cuh.  Per CTA step every lane solves its cell for D directions:
//
//   * I_crn_old for the whole CTA step is one contiguous run of the skewed state, staged into
//     shared memory by a TMA bulk copy `stages` steps ahead (mbarrier completion);
//   * the left inflow of a cell is the right outflow the same lane produced one step earlier
//     (registers); the bottom inflow is the top outflow of the row below one step earlier:
//     a warp shuffle inside a warp, a shared-memory handoff between warps, an L2-resident wrap
//     buffer between rounds, and the boundary arrays on the inflow faces;
//   * the 13 moment products of a cell are accumulated over the lane's D directions, reduced over
//     the S slices of the row with xor-shuffles (fixed order), and written once per (cell, g,
//     quadrant) as a partial; quadrant partials are combined in a fixed order afterwards, so results
//     are bit-reproducible run to run;
//   * the new corner intensities are written straight back in the same skewed layout.
//
// Every wait is bounded: a TMA phase that does not complete sets the error word and the CTA leaves
// the loop together (the per-step barrier is a __syncthreads_or on the timeout flag) after a bounded
// drain of its outstanding copies.
#pragma once

#include <cuda_runtime.h>

#include "layout.cuh"
#include "ptx.cuh"
#include "scb_cell.h"

namespace trt {

template <class Real>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};

// Direction-table rows (per quadrant, mq entries each), physical signs for the moment weights.
enum DirRow { kAx = 0, kAy, kW, kWxx, kWyy, kWxy, kWx, kWy, kNDirRow };

template <class Real>
struct SweepArgs {
  int nx, ny, nm, ng, mq;
  Tiling t;
  int stages;
  long long chunk;          // elements per (T, w) chunk
  long long blk;            // elements per (g, q) block
  Real rcdt;                // 1 / (c * dt)
  const Real* dx;           // (nx)
  const Real* dy;           // (ny)
  const Real* area;         // (nx, ny)
  const Real* kap;          // (nx, ny, ng): KapE_in (without 1/(c dt))
  const Real* qiso;         // (nx, ny, ng): isotropic corner source, or null with srcfull
  const Real* srcfull;      // skewed layout, anisotropic per-corner source (drop-in path), or null
  const Real* dirtab;       // [4][kNDirRow][mq]
  const double* dir64;      // [kNDirRow][nm] FP64 direction table (moment weights)
  const Real* Iold;         // skewed
  Real* Inew;               // skewed
  Real* bndV;               // [2][ng][nm][2 ny]  Ic_edgV on faces x=0 (side 0) and x=nx (side 1)
  Real* bndH;               // [2][ng][nm][2 nx]  Ic_edgH on faces y=0 (side 0) and y=ny (side 1)
  Real* wrap;               // [4 ng][nx][mq][2]  top outflow of the last row of a round
  Real* part;               // [4*NH][ng][ny][nx][part_rec<Real>()]  moment partial records (physical cells)
  int* err;                 // error word (bit 0: TMA wait timed out)
  unsigned max_polls;       // bound on mbarrier polls per wait of the sweep
  unsigned drain_polls;     // bound on the polls that drain outstanding copies after a timeout
};

constexpr int kErrTmaTimeout = 1;

// Dynamic shared memory of one sweep CTA: the TMA ring, its mbarriers, the row handoff, the direction
// table and the moment-weight table (FP32 sweep: float2 pairs of direction slots, 6 rows).
template <class Real>
__host__ __device__ inline size_t sweep_smem_bytes(int W, long long chunk, int stages, int mqc, int D, int S) {
  (void)mqc;
  size_t ring = (size_t)stages * W * chunk * sizeof(Real);
  size_t bars = (size_t)stages * sizeof(uint64_t);
  size_t hand = (size_t)2 * W * mqc * 2 * sizeof(Real);
  size_t dtab = (size_t)kNDirRow * D * S * sizeof(Real);
  size_t wtab = (size_t)6 * ((D + 1) / 2) * S * sizeof(float2) + 16;
  return ring + bars + hand + dtab + wtab + 32;
}

// Reduce-scatter of the 16 moment slots over the S slices of a row (xor partners R, 2R, ..., 16):
// after log2(S) levels every lane holds 16/S consecutive slots summed over the slices, in a fixed
// order.  Returns the index of the first slot this lane holds.
// With S = 32 the last level is a plain pairwise sum and only the lower lane of the pair owns the
// slot (*owner = false for the other).
template <int S, int R>
__device__ __forceinline__ int slice_reduce_scatter(double (&v)[16], int s, bool* owner) {
  int base = 0;
  int width = 16;
  *owner = true;
#pragma unroll
  for (int o = 16; o >= R; o >>= 1) {
    if (o >= R * S) continue;   // lane bits above the slice bits: not a slice partner
    const bool upper = (s & (o / R)) != 0;
    if (width == 1) {
      v[0] = v[0] + __shfl_xor_sync(0xffffffffu, v[0], o);
      if (upper) *owner = false;
      continue;
    }
    const int half = width / 2;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < half) {
        const double send = upper ? v[k] : v[k + half];
        const double keep = upper ? v[k + half] : v[k];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
    if (upper) base += half;
    width = half;
  }
  return base;
}

// Both precisions accumulate the per-lane moment sums in FP64: the FP32 ("mixed") sweep's
// intensities are converted exactly and multiplied by FP64 weights on the otherwise idle FP64 pipe,
// so the sums carry no FP32 rounding at all (stronger than a Kahan-compensated FP32 sum, and cheaper
// on this part: measured 7.2 ms with Kahan vs the FP64-accumulating kernel on C1).  Sums over
// slices, quadrants and groups are FP64 as well.
// Two variants of the step body, chosen by precision (measured on C1, each the faster for its type):
//  * FP32: every lane computes every direction slot and the bottom-inflow shuffle runs inline (no
//    per-direction top-face registers);
//  * FP64: only live slots compute, top faces kept in registers and shuffled after the direction loop.
// Both take the inflows that come from global memory (boundary faces, the wrap buffer) and the next cell's
// material one step ahead, so that no step waits on a global load: the per-step barrier would make the
// whole CTA wait for the slowest warp's load.
// The sweep of one CTA: (group, quadrant, direction split) number `bid` of the instance described by
// `a` (blockIdx.x for a single-instance launch; the instance-local number in a batched launch).
template <class Real, int S, int D, bool SRC_FULL>
__device__ __forceinline__ bool scb_sweep_body(const SweepArgs<Real>& a, const int bid) {
  constexpr bool kLeanFP32 = sizeof(Real) == 4;
  constexpr int R = 32 / S;
  constexpr int NV = 16 / (int)sizeof(Real);
  constexpr int NSLOT = S >= 16 ? 1 : 16 / S;   // moment slots a lane holds after the reduce-scatter
  constexpr int DS = D * S;                      // row stride of the direction table

  const Tiling t = a.t;
  const int W = t.W;
  const int nx = a.nx, ny = a.ny, nm = a.nm, ng = a.ng, mq = a.mq;
  // band CTAs of one (g, q, h) sweep are consecutive blocks (one cluster); band = rank in the cluster
  const int NB = t.NB;
  const int band = NB > 1 ? bid % NB : 0;
  const int gqh = NB > 1 ? bid / NB : bid;
  const int prod = (band + NB - 1) % NB;   // the band CTA that sweeps the round below each of ours
  const int h = gqh % t.NH, g = (gqh / t.NH) >> 2, q = (gqh / t.NH) & 3;
  const int mqc = t.mqc;                           // chunk width (directions of the largest split)
  const int mo = split_first(mq, t.NH, h);         // first quadrant-local direction of this split
  const int mq_h = split_count(mq, t.NH, h);       // directions of this split
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = lane / R, r = lane % R;
  const int rho = warp * R + r;
  const bool fx = (q == 1 || q == 2), fy = (q >= 2);
  const int stages = a.stages;
  const int chunk = (int)a.chunk;
  const uint32_t stage_bytes = (uint32_t)(W * chunk * (int)sizeof(Real));
  // slices of the last direction block that hold a direction (all slices of the earlier blocks do)
  const int s_last = mq_h - (D - 1) * S;
  const int nl_last = R * (mqc - (D - 1) * S);

  extern __shared__ __align__(128) unsigned char smem[];
  Real* ring = reinterpret_cast<Real*>(smem);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + (size_t)stages * stage_bytes);
  Real* hand = reinterpret_cast<Real*>(mbar + stages);
  Real* dtab = hand + 2 * W * mqc * 2;
  // FP32 moment weights w, w Ox^2, w Oy^2, w Ox Oy, w Ox, w Oy as float2 pairs: row k, pair p, slice s holds
  // the weights of the lane's direction slots 2p (.x) and 2p+1 (.y); slots without a direction hold 0
  constexpr int NP = (D + 1) / 2;
  float2* wt2 = reinterpret_cast<float2*>(
      (reinterpret_cast<uintptr_t>(dtab + kNDirRow * DS) + 15) & ~static_cast<uintptr_t>(15));

  // direction table of this split: row k of split-local direction ml at dtab[k * DS + ml] (a compile-time row
  // stride, so that every table read is a constant offset from one per-lane base)
  for (int k = threadIdx.x; k < kNDirRow * DS; k += blockDim.x) {
    const int row = k / DS, col = k % DS;
    Real v = col < mq_h ? a.dirtab[((size_t)q * kNDirRow + row) * mq + mo + col] : Real(0);
    if (row < 2) v = v * Real(0.25);   // |Omega| / 4 for the corner-matrix geometry
    dtab[k] = v;
  }
  if constexpr (kLeanFP32) {
    for (int k = threadIdx.x; k < 6 * NP * S; k += blockDim.x) {
      const int row = k / (NP * S), p = (k / S) % NP, sl = k % S;
      const int m0 = (2 * p) * S + sl, m1 = (2 * p + 1) * S + sl;   // split-local directions of the two slots
      const double* wr = a.dir64 + (size_t)(kW + row) * nm + q * mq + mo;
      wt2[k] = make_float2(2 * p < D && m0 < mq_h ? (float)wr[m0] : 0.0f,
                           2 * p + 1 < D && m1 < mq_h ? (float)wr[m1] : 0.0f);
    }
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < stages; ++k) mbar_init(&mbar[k], 1);
    fence_mbar_init();
  }
  // Band handoff (NB > 1): band_prog holds the local steps the producer band has completed; the producer
  // writes it into this CTA's shared memory with a cluster-scope release after each step that the
  // rounds above it still need (publication stops once the last of those steps is out, so no CTA writes
  // into a CTA that may have left).  Every CTA initialises its slot before any CTA publishes.
  __shared__ int band_prog;
  if (NB > 1 && threadIdx.x == 0) band_prog = 0;
  __syncthreads();
  if (NB > 1) cluster_sync_all();

  // this band's steps inside the (g, q, h) block of the skewed state
  const long long blk_off = (long long)gqh * a.blk + (long long)band * t.Tb * W * chunk;
  const Real* gold = a.Iold + blk_off;
  Real* gnew = a.Inew + blk_off;
  const int Tsteps = band_steps(t, nx, band);

  // the TMA copies are issued by lane 0 of the last warp, whose rows take no inflow from global memory (the
  // first warp's first row does, and a copy issued behind those loads would wait for them)
  const bool tma_thread = threadIdx.x == 32 * (W - 1);
  if (tma_thread) {
    for (int k = 0; k < stages && k < Tsteps; ++k) {
      mbar_arrive_expect_tx(&mbar[k], stage_bytes);
      tma_bulk_g2s(ring + (size_t)k * W * chunk, gold + (long long)k * W * chunk, stage_bytes, &mbar[k]);
    }
  }

  const Real rcdt = a.rcdt;
  const int nxy = nx * ny;
  Real* wrapc = a.wrap + (size_t)gqh * nx * mqc * 2;
  constexpr int kRec = part_rec<Real>();
  Real* partg = a.part + ((size_t)((q * t.NH + h) * ng + g) * nxy) * kRec;
  const int sideVin = fx ? 1 : 0, sideVout = fx ? 0 : 1;
  const int sideHin = fy ? 1 : 0, sideHout = fy ? 0 : 1;
  const Real* bVin = a.bndV + ((size_t)(sideVin * ng + g) * nm + q * mq + mo) * (2 * ny);
  Real* bVout = a.bndV + ((size_t)(sideVout * ng + g) * nm + q * mq + mo) * (2 * ny);
  const Real* bHin = a.bndH + ((size_t)(sideHin * ng + g) * nm + q * mq + mo) * (2 * nx);
  Real* bHout = a.bndH + ((size_t)(sideHout * ng + g) * nm + q * mq + mo) * (2 * nx);
  const Real* kapg = a.kap + (size_t)nxy * g;
  const Real* qisog = SRC_FULL ? nullptr : a.qiso + (size_t)nxy * g;
  const int byo = fy ? 1 : 0;   // physical corner-edge offset of the frame's bottom corner
  const int bxo = fx ? 1 : 0;   // ... of the frame's left corner

  Real vb[D], vt[D], hl[D], hr[D];
#pragma unroll
  for (int d = 0; d < D; ++d) vb[d] = vt[d] = hl[d] = hr[d] = Real(0);

  // lane position: column ip of round n (ip < 0 before the lane starts); advanced incrementally
  int ip = -rho, n = band;
  bool timed_out = false;
  // Producer side: publish after every local step up to the end of the last round that has a round
  // above it (round band + ks*NB <= nr - 2, its top row done with column nx-1).
  const int ks = (t.nr - 2 - band) >= 0 ? (t.nr - 2 - band) / NB : -1;
  const int pub_stop = ks >= 0 ? ks * t.P + nx + t.H - 1 : 0;
  const uint32_t prog_remote = NB > 1 ? cluster_map(&band_prog, (uint32_t)((band + 1) % NB)) : 0u;
  // Consumer side (warp 0, whose first row reads the wrap buffer): before the first row of round nn > 0
  // takes the bottom inflow of column ipn, the producer must have finished that column in round nn - 1
  // (its local round (nn-1-prod)/NB), i.e. completed local step k'P + ipn + H - 1.  Bounded wait: false
  // when the producer did not get there within max_polls polls.
  // Called by every lane of warp 0 with its own position; lane 0 is row 0 of the band (the lanes that read
  // the wrap buffer are the slices of that row, at the same position), so its position decides.
  int seen = 0;
  auto band_wait = [&](int ipn, int nn) -> bool {
    if (NB == 1) return true;
    int ok = 1;
    if (lane == 0 && nn > 0 && nn < t.nr && ipn >= 0 && ipn < nx) {
      const int need = ((nn - 1 - prod) / NB) * t.P + ipn + t.H;
      for (unsigned k = 0; seen < need; ++k) {
        seen = ld_acquire_cluster(&band_prog);
        if (seen >= need) break;
        if (k >= a.max_polls) {
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
  };
  // material of the lane's cell at the current step (m*) and at the next one (n*): the next cell's loads are
  // issued at the top of a step and only consumed (scaled by 1/4, 1/(c dt) added) after its solve, so that
  // their latency hides behind the step; arithmetic on a loaded value right after the load would stall the
  // warp there (measured on C1: 1700 of 8200 cycles per warp step)
  Real mdx = Real(0), mdy = Real(0), mA4 = Real(0), mkp = Real(0), mqs = Real(0);
  Real ndx = Real(0), ndy = Real(0), nA4 = Real(0), nkp = Real(0), nqs = Real(0);
  auto fetch_material = [&](int ipn, int nn) {
    const int jpn = nn * t.H + rho;
    if (ipn >= 0 && ipn < nx && nn < t.nr && jpn < ny) {
      const int i = fx ? nx - 1 - ipn : ipn;
      const int j = fy ? ny - 1 - jpn : jpn;
      const int cell = i + nx * j;
      ndx = a.dx[i];
      ndy = a.dy[j];
      nA4 = a.area[cell];
      nkp = kapg[cell];
      if (!SRC_FULL) nqs = qisog[cell];
    }
  };
  auto take_material = [&]() {
    mdx = ndx;
    mdy = ndy;
    mA4 = nA4 * Real(0.25);
    mkp = nkp + rcdt;
    mqs = nqs;
  };
  // Inflows that come from global memory, loaded one step ahead into the inflow registers: the
  // sweep-left boundary face at the start of a round, and for the CTA's first row the sweep-bottom
  // boundary face (round 0) or the wrap buffer (later rounds).  The wrap entry for column ip of
  // round n was written at step (n-1)P + ip + H - 1, before the barrier that precedes this prefetch
  // (P > H).
  auto load_inflow = [&](int ipn, int nn) {
    const int jpn = nn * t.H + rho;
    if (!(ipn >= 0 && ipn < nx && nn < t.nr && jpn < ny)) return;
    const int in = fx ? nx - 1 - ipn : ipn;
    const int jn = fy ? ny - 1 - jpn : jpn;
    if (ipn == 0) {
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const int ml = d * S + s;
        if (d < D - 1 || s < s_last) {
          vb[d] = bVin[ml * 2 * ny + 2 * jn + byo];
          vt[d] = bVin[ml * 2 * ny + 2 * jn + 1 - byo];
        }
      }
    }
    if (rho == 0) {
#pragma unroll
      for (int d = 0; d < D; ++d) {
        const int ml = d * S + s;
        if (d < D - 1 || s < s_last) {
          if (nn == 0) {
            hl[d] = bHin[ml * 2 * nx + 2 * in + bxo];
            hr[d] = bHin[ml * 2 * nx + 2 * in + 1 - bxo];
          } else {   // written by another band CTA (or this one): read through L2
            hl[d] = __ldcg(wrapc + (ipn * mqc + ml) * 2 + 0);
            hr[d] = __ldcg(wrapc + (ipn * mqc + ml) * 2 + 1);
          }
        }
      }
    }
  };
  fetch_material(ip, n);
  take_material();
  if (warp == 0 && !band_wait(ip, n)) timed_out = true;
  load_inflow(ip, n);

  int stage = 0;
  uint32_t phase = 0;
  int T_break = Tsteps;
  for (int T = 0; T < Tsteps; ++T) {
    {   // the next cell's material (the lane's position one step on)
      const bool wrap_round = ip + 1 == t.P;
      fetch_material(wrap_round ? 0 : ip + 1, wrap_round ? n + NB : n);
    }
    if (!mbar_wait_bounded(&mbar[stage], phase, a.max_polls)) timed_out = true;
    const Real* sm = ring + (size_t)stage * W * chunk + (size_t)warp * chunk;
    const int gchunk = (T * W + warp) * chunk;

    int i, j;
    bool active;
    double acc[13];
    if constexpr (!kLeanFP32) {
      const int jp = n * t.H + rho;
      active = !timed_out && ip >= 0 && ip < nx && n < t.nr && jp < ny;
      i = fx ? nx - 1 - ip : ip;
      j = fy ? ny - 1 - jp : jp;

      Real topL[D], topR[D];
  #pragma unroll
      for (int v = 0; v < 13; ++v) acc[v] = 0.0;
  #pragma unroll
      for (int d = 0; d < D; ++d) topL[d] = topR[d] = Real(0);

      if (active) {
        const Real dx = mdx, dy = mdy, A4 = mA4, kp = mkp, qs = mqs;
        if (r == 0 && warp > 0) {
  #pragma unroll
          for (int d = 0; d < D; ++d) {
            const int ml = d * S + s;
            if (d < D - 1 || s < s_last) {
              const Real* src = hand + ((((T - 1) & 1) * W + (warp - 1)) * mqc + ml) * 2;
              hl[d] = src[0];
              hr[d] = src[1];
            }
          }
        }

        const Real kA4 = scb_kA4(dx, dy, kp);
  #pragma unroll
        for (int d = 0; d < D; ++d) {
          const int ml = d * S + s;
          if (d < D - 1 || s < s_last) {
            const int nl = (d < D - 1) ? 32 : nl_last;
            const Real* sb = sm + d * 128;
            Real io[4];
            if (NV == 2) {
              const double2 p0 = *reinterpret_cast<const double2*>(sb + lane * 2);
              const double2 p1 = *reinterpret_cast<const double2*>(sb + nl * 2 + lane * 2);
              io[0] = (Real)p0.x; io[1] = (Real)p0.y; io[2] = (Real)p1.x; io[3] = (Real)p1.y;
            } else {
              const float4 p0 = *reinterpret_cast<const float4*>(sb + lane * 4);
              io[0] = (Real)p0.x; io[1] = (Real)p0.y; io[2] = (Real)p0.z; io[3] = (Real)p0.w;
            }
            Real src[4];
            if (SRC_FULL) {
              const Real* gs = a.srcfull + blk_off + gchunk + d * 128;
  #pragma unroll
              for (int c = 0; c < 4; ++c)
                src[c] = tfma(io[c], rcdt, gs[(c / NV) * nl * NV + lane * NV + (c % NV)]);
            } else {
  #pragma unroll
              for (int c = 0; c < 4; ++c) src[c] = tfma(io[c], rcdt, qs);
            }
            const ScbGeom<Real> G = scb_geom(dtab[kAx * DS + ml], dtab[kAy * DS + ml], dx, dy);
            const Real gam = scb_gamma(G, kA4);
            Real x[4];
            scb_solve(G, gam, A4, src, vb[d], vt[d], hl[d], hr[d], x);

            Real* gb = gnew + gchunk + d * 128;
            if (NV == 2) {
              *reinterpret_cast<double2*>(gb + lane * 2) = make_double2((double)x[0], (double)x[1]);
              *reinterpret_cast<double2*>(gb + nl * 2 + lane * 2) = make_double2((double)x[2], (double)x[3]);
            } else {
              *reinterpret_cast<float4*>(gb + lane * 4) = make_float4((float)x[0], (float)x[1], (float)x[2], (float)x[3]);
            }
            // outflow: right face feeds the next column of this lane, top face the next row
            vb[d] = x[1];
            vt[d] = x[2];
            topL[d] = x[3];
            topR[d] = x[2];

            const Real Iavg = ((x[0] + x[1]) + (x[2] + x[3])) * Real(0.25);
            const Real Iv = (x[1] + x[2]) * Real(0.5);
            const Real Ih = (x[3] + x[2]) * Real(0.5);
            const Real wxx = dtab[kWxx * DS + ml], wyy = dtab[kWyy * DS + ml], wxy = dtab[kWxy * DS + ml];
            const Real ww = dtab[kW * DS + ml], wx = dtab[kWx * DS + ml], wy = dtab[kWy * DS + ml];
            {
              acc[kCxx] = tfma(wxx, Iavg, acc[kCxx]);
              acc[kCyy] = tfma(wyy, Iavg, acc[kCyy]);
              acc[kCxy] = tfma(wxy, Iavg, acc[kCxy]);
              acc[kCe] = tfma(ww, Iavg, acc[kCe]);
              acc[kVxx] = tfma(wxx, Iv, acc[kVxx]);
              acc[kVxy] = tfma(wxy, Iv, acc[kVxy]);
              acc[kVx] = tfma(wx, Iv, acc[kVx]);
              acc[kVe] = tfma(ww, Iv, acc[kVe]);
              acc[kHyy] = tfma(wyy, Ih, acc[kHyy]);
              acc[kHxy] = tfma(wxy, Ih, acc[kHxy]);
              acc[kHy] = tfma(wy, Ih, acc[kHy]);
              acc[kHx] = tfma(wx, Ih, acc[kHx]);
              acc[kHe] = tfma(ww, Ih, acc[kHe]);
            }
          }
        }

        // outflow boundary faces and the handoff of the warp's last row
        const bool right_edge = (ip == nx - 1), top_edge = (jp == ny - 1), last_row = (r == R - 1);
        if (right_edge || top_edge || last_row) {
  #pragma unroll
          for (int d = 0; d < D; ++d) {
            const int ml = d * S + s;
            if (d < D - 1 || s < s_last) {
              if (right_edge) {
                bVout[ml * 2 * ny + 2 * j + byo] = vb[d];
                bVout[ml * 2 * ny + 2 * j + 1 - byo] = vt[d];
              }
              if (top_edge) {
                bHout[ml * 2 * nx + 2 * i + bxo] = topL[d];
                bHout[ml * 2 * nx + 2 * i + 1 - bxo] = topR[d];
              }
              if (last_row) {
                Real* dst = (warp < W - 1) ? hand + (((T & 1) * W + warp) * mqc + ml) * 2
                                           : wrapc + (ip * mqc + ml) * 2;
                if (warp < W - 1 || t.nr > 1) {
                  dst[0] = topL[d];
                  dst[1] = topR[d];
                }
              }
            }
          }
        }
      }

      // bottom inflow of rows r >= 1 for the next step (rows r == 0 reload it)
  #pragma unroll
      for (int d = 0; d < D; ++d) {
        hl[d] = __shfl_up_sync(0xffffffffu, topL[d], 1);
        hr[d] = __shfl_up_sync(0xffffffffu, topR[d], 1);
      }

    } else {
      const int jp = n * t.H + rho;
      active = !timed_out && ip >= 0 && ip < nx && n < t.nr && jp < ny;
      i = fx ? nx - 1 - ip : ip;
      j = fy ? ny - 1 - jp : jp;
      const Real dx = mdx, dy = mdy, A4 = mA4, kp = mkp, qs = mqs;

      // bottom inflow of a warp's first row from the warp below (shared memory, written last step)
      if (active && r == 0 && warp > 0) {
  #pragma unroll
        for (int d = 0; d < D; ++d) {
          const int ml = d * S + s;
          if (d < D - 1 || s < s_last) {
            const Real* src = hand + ((((T - 1) & 1) * W + (warp - 1)) * mqc + ml) * 2;
            hl[d] = src[0];
            hr[d] = src[1];
          }
        }
      }

      const bool right_edge = active && (ip == nx - 1);
      const bool top_edge = active && (jp == ny - 1);
      const bool last_row = active && (r == R - 1) && (warp < W - 1 || t.nr > 1);
      Real* hand_dst = (warp < W - 1) ? hand + ((T & 1) * W + warp) * mqc * 2 : wrapc + ip * mqc * 2;

      // FP32 moment lane sums: acc2[v].x sums the lane's even direction slots, .y its odd ones (at most
      // ceil(D/2) terms each, one FP32 rounding per fused multiply-add); the two are added in FP64 at the
      // end of the step, before the slice reduction, so each lane sum carries a relative error of at most
      // ceil(D/2) units of FP32 rounding.
      float2 acc2[13];
  #pragma unroll
      for (int v = 0; v < 13; ++v) acc2[v] = make_float2(0.0f, 0.0f);
      Real topL[kLeanFP32 ? 1 : D], topR[kLeanFP32 ? 1 : D];
      const Real kA4 = scb_kA4(dx, dy, kp);

      // moment products of the direction slots 2p (.x) and 2p+1 (.y) of the lane, packed FP32x2
      auto add_moments2 = [&](int p, float2 x0, float2 x1, float2 x2, float2 x3) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
        const float2 Iavg = __fmul2_rn(__fadd2_rn(__fadd2_rn(x0, x1), __fadd2_rn(x2, x3)), f2(0.25f));
        const float2 Iv = __fmul2_rn(__fadd2_rn(x1, x2), f2(0.5f));
        const float2 Ih = __fmul2_rn(__fadd2_rn(x3, x2), f2(0.5f));
        const float2* wp = wt2 + p * S + s;
        const float2 ww = wp[0 * NP * S], wxx = wp[1 * NP * S], wyy = wp[2 * NP * S];
        const float2 wxy = wp[3 * NP * S], wx = wp[4 * NP * S], wy = wp[5 * NP * S];
        acc2[kCxx] = __ffma2_rn(wxx, Iavg, acc2[kCxx]);
        acc2[kCyy] = __ffma2_rn(wyy, Iavg, acc2[kCyy]);
        acc2[kCxy] = __ffma2_rn(wxy, Iavg, acc2[kCxy]);
        acc2[kCe] = __ffma2_rn(ww, Iavg, acc2[kCe]);
        acc2[kVxx] = __ffma2_rn(wxx, Iv, acc2[kVxx]);
        acc2[kVxy] = __ffma2_rn(wxy, Iv, acc2[kVxy]);
        acc2[kVx] = __ffma2_rn(wx, Iv, acc2[kVx]);
        acc2[kVe] = __ffma2_rn(ww, Iv, acc2[kVe]);
        acc2[kHyy] = __ffma2_rn(wyy, Ih, acc2[kHyy]);
        acc2[kHxy] = __ffma2_rn(wxy, Ih, acc2[kHxy]);
        acc2[kHy] = __ffma2_rn(wy, Ih, acc2[kHy]);
        acc2[kHx] = __ffma2_rn(wx, Ih, acc2[kHx]);
        acc2[kHe] = __ffma2_rn(ww, Ih, acc2[kHe]);
#endif
      };
      // moment products of one direction slot d (component d & 1 of pair d / 2)
      auto add_moments = [&](int d, float x0, float x1, float x2, float x3) {
        const float Iavg = ((x0 + x1) + (x2 + x3)) * 0.25f;
        const float Iv = (x1 + x2) * 0.5f;
        const float Ih = (x3 + x2) * 0.5f;
        const float2* wp = wt2 + (d / 2) * S + s;
        const bool hi = (d & 1) != 0;
        auto w = [&](int row) { const float2 v = wp[row * NP * S]; return hi ? v.y : v.x; };
        auto acc = [&](int k, float wv, float I) {
          if (hi) acc2[k].y = fmaf(wv, I, acc2[k].y);
          else acc2[k].x = fmaf(wv, I, acc2[k].x);
        };
        acc(kCxx, w(1), Iavg);
        acc(kCyy, w(2), Iavg);
        acc(kCxy, w(3), Iavg);
        acc(kCe, w(0), Iavg);
        acc(kVxx, w(1), Iv);
        acc(kVxy, w(3), Iv);
        acc(kVx, w(4), Iv);
        acc(kVe, w(0), Iv);
        acc(kHyy, w(2), Ih);
        acc(kHxy, w(3), Ih);
        acc(kHy, w(5), Ih);
        acc(kHx, w(4), Ih);
        acc(kHe, w(0), Ih);
      };
      // FP32 outputs of one live direction slot: corner state, outflow boundary faces, row handoff
      auto store_slot = [&](int d, int ml, Real x0, Real x1, Real x2, Real x3) {
        Real* gb = gnew + gchunk + d * 128;
        *reinterpret_cast<float4*>(gb + lane * 4) = make_float4((float)x0, (float)x1, (float)x2, (float)x3);
        if (right_edge) {
          bVout[ml * 2 * ny + 2 * j + byo] = x1;
          bVout[ml * 2 * ny + 2 * j + 1 - byo] = x2;
        }
        if (top_edge) {
          bHout[ml * 2 * nx + 2 * i + bxo] = x3;
          bHout[ml * 2 * nx + 2 * i + 1 - bxo] = x2;
        }
        if (last_row) {
          hand_dst[ml * 2 + 0] = x3;
          hand_dst[ml * 2 + 1] = x2;
        }
      };

#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
      // FP32: directions d and d+1 of the lane solved together on the packed FP32x2 pipe (bit-identical
      // to two scalar solves); every lane computes (idle slots and inactive lanes on valid addresses,
      // results discarded) so the bottom-inflow shuffles run inline.
      auto pair = [&](int d) {
        const bool valid1 = (d + 1 < D - 1) || (s < s_last);
        const int ml0 = d * S + s, ml1 = valid1 ? (d + 1) * S + s : 0;
        const int ln1 = valid1 ? lane : 0;
        const bool live1 = active && valid1;
        const float4 p0 = *reinterpret_cast<const float4*>(sm + d * 128 + lane * 4);
        const float4 p1 = *reinterpret_cast<const float4*>(sm + (d + 1) * 128 + ln1 * 4);
        const float2 io[4] = {make_float2(p0.x, p1.x), make_float2(p0.y, p1.y), make_float2(p0.z, p1.z),
                              make_float2(p0.w, p1.w)};
        float2 src[4];
        if (SRC_FULL) {
          const Real* gs0 = a.srcfull + blk_off + gchunk + d * 128 + lane * 4;
          const Real* gs1 = a.srcfull + blk_off + gchunk + (d + 1) * 128 + ln1 * 4;
  #pragma unroll
          for (int c = 0; c < 4; ++c)
            src[c] = __ffma2_rn(io[c], f2(rcdt), make_float2(active ? gs0[c] : 0.0f, live1 ? gs1[c] : 0.0f));
        } else {
  #pragma unroll
          for (int c = 0; c < 4; ++c) src[c] = __ffma2_rn(io[c], f2(rcdt), f2(qs));
        }
        const ScbGeom2 G2 = scb_geom2(make_float2(dtab[kAx * DS + ml0], dtab[kAx * DS + ml1]),
                                      make_float2(dtab[kAy * DS + ml0], dtab[kAy * DS + ml1]), dx, dy);
        const float2 gam = scb_gamma2(G2, kA4);
        float2 x[4];
        scb_solve2(G2, gam, A4, src, make_float2(vb[d], vb[d + 1]), make_float2(vt[d], vt[d + 1]),
                   make_float2(hl[d], hl[d + 1]), make_float2(hr[d], hr[d + 1]), x);
        vb[d] = x[1].x;
        vb[d + 1] = x[1].y;
        vt[d] = x[2].x;
        vt[d + 1] = x[2].y;
        hl[d] = __shfl_up_sync(0xffffffffu, x[3].x, 1);
        hl[d + 1] = __shfl_up_sync(0xffffffffu, x[3].y, 1);
        hr[d] = __shfl_up_sync(0xffffffffu, x[2].x, 1);
        hr[d + 1] = __shfl_up_sync(0xffffffffu, x[2].y, 1);
        if (active) store_slot(d, ml0, x[0].x, x[1].x, x[2].x, x[3].x);
        if (live1) store_slot(d + 1, ml1, x[0].y, x[1].y, x[2].y, x[3].y);
        if (live1) add_moments2(d / 2, x[0], x[1], x[2], x[3]);
        else if (active) add_moments(d, x[0].x, x[1].x, x[2].x, x[3].x);
      };
#endif

      // a warp none of whose lanes has a cell at this step (wavefront fill and drain) skips the solve:
      // a row that starts at the next step takes its inflows from the boundary, the wrap buffer or the
      // handoff, never from the shuffles of this step
      const bool warp_live = __any_sync(0xffffffffu, active);
  #pragma unroll
      for (int d = 0; d < D; ++d) {
        if (!warp_live) break;
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
        if constexpr (kLeanFP32) {
          if (d % 2 == 0 && d + 1 < D) {
            pair(d);
            continue;
          }
          if (d % 2 == 1) continue;   // second direction of a pair
        }
#endif
        const bool valid = (d < D - 1) || (s < s_last);
        // FP32: every lane computes every slot (idle slots and inactive lanes on valid addresses, results
        // discarded) so the bottom-inflow shuffle runs inline; FP64: only live slots compute.
        if (!kLeanFP32 && !(active && valid)) continue;
        const int ml = valid ? d * S + s : 0;
        const int ln = valid ? lane : 0;
        const bool live = active && valid;
        const int nl = (d < D - 1) ? 32 : nl_last;
        const Real* sb = sm + d * 128;
        Real io[4];
        if (NV == 2) {
          const double2 p0 = *reinterpret_cast<const double2*>(sb + ln * 2);
          const double2 p1 = *reinterpret_cast<const double2*>(sb + nl * 2 + ln * 2);
          io[0] = (Real)p0.x; io[1] = (Real)p0.y; io[2] = (Real)p1.x; io[3] = (Real)p1.y;
        } else {
          const float4 p0 = *reinterpret_cast<const float4*>(sb + ln * 4);
          io[0] = (Real)p0.x; io[1] = (Real)p0.y; io[2] = (Real)p0.z; io[3] = (Real)p0.w;
        }
        Real src[4];
        if (SRC_FULL) {
          const Real* gs = a.srcfull + blk_off + gchunk + d * 128;
  #pragma unroll
          for (int c = 0; c < 4; ++c)
            src[c] = tfma(io[c], rcdt, live ? gs[(c / NV) * nl * NV + ln * NV + (c % NV)] : Real(0));
        } else {
  #pragma unroll
          for (int c = 0; c < 4; ++c) src[c] = tfma(io[c], rcdt, qs);
        }
        const ScbGeom<Real> G = scb_geom(dtab[kAx * DS + ml], dtab[kAy * DS + ml], dx, dy);
        const Real gam = scb_gamma(G, kA4);
        Real x[4];
        scb_solve(G, gam, A4, src, vb[d], vt[d], hl[d], hr[d], x);

        // outflow: right face feeds this lane's next column, top face the next row
        vb[d] = x[1];
        vt[d] = x[2];
        if (kLeanFP32) {
          hl[d] = __shfl_up_sync(0xffffffffu, x[3], 1);
          hr[d] = __shfl_up_sync(0xffffffffu, x[2], 1);
        } else {
          topL[kLeanFP32 ? 0 : d] = x[3];
          topR[kLeanFP32 ? 0 : d] = x[2];
        }

        if (live) {
          Real* gb = gnew + gchunk + d * 128;
          if (NV == 2) {
            *reinterpret_cast<double2*>(gb + lane * 2) = make_double2((double)x[0], (double)x[1]);
            *reinterpret_cast<double2*>(gb + nl * 2 + lane * 2) = make_double2((double)x[2], (double)x[3]);
          } else {
            *reinterpret_cast<float4*>(gb + lane * 4) = make_float4((float)x[0], (float)x[1], (float)x[2], (float)x[3]);
          }
          if (kLeanFP32) {
            if (right_edge) {
              bVout[ml * 2 * ny + 2 * j + byo] = x[1];
              bVout[ml * 2 * ny + 2 * j + 1 - byo] = x[2];
            }
            if (top_edge) {
              bHout[ml * 2 * nx + 2 * i + bxo] = x[3];
              bHout[ml * 2 * nx + 2 * i + 1 - bxo] = x[2];
            }
            if (last_row) {
              hand_dst[ml * 2 + 0] = x[3];
              hand_dst[ml * 2 + 1] = x[2];
            }
          }
          add_moments(d, (float)x[0], (float)x[1], (float)x[2], (float)x[3]);
        }
      }

      if (!kLeanFP32) {
        // FP64: outflow boundary faces, the handoff of the warp's last row and the bottom-inflow
        // shuffle, after the direction loop
        if (right_edge || top_edge || last_row) {
  #pragma unroll
          for (int d = 0; d < D; ++d) {
            const int ml = d * S + s;
            if (d < D - 1 || s < s_last) {
              if (right_edge) {
                bVout[ml * 2 * ny + 2 * j + byo] = vb[d];
                bVout[ml * 2 * ny + 2 * j + 1 - byo] = vt[d];
              }
              if (top_edge) {
                bHout[ml * 2 * nx + 2 * i + bxo] = topL[kLeanFP32 ? 0 : d];
                bHout[ml * 2 * nx + 2 * i + 1 - bxo] = topR[kLeanFP32 ? 0 : d];
              }
              if (last_row) {
                hand_dst[ml * 2 + 0] = topL[kLeanFP32 ? 0 : d];
                hand_dst[ml * 2 + 1] = topR[kLeanFP32 ? 0 : d];
              }
            }
          }
        }
  #pragma unroll
        for (int d = 0; d < D; ++d) {
          hl[d] = __shfl_up_sync(0xffffffffu, topL[kLeanFP32 ? 0 : d], 1);
          hr[d] = __shfl_up_sync(0xffffffffu, topR[kLeanFP32 ? 0 : d], 1);
        }
      }
  #pragma unroll
      for (int v = 0; v < 13; ++v) acc[v] = (double)acc2[v].x + (double)acc2[v].y;
    }

    // moments: reduce-scatter over the S slices of each row, then each lane writes its slots
    double mv[16];
#pragma unroll
    for (int v = 0; v < 13; ++v) mv[v] = acc[v];
    mv[13] = mv[14] = mv[15] = 0.0;
    bool owner;
    const int base = slice_reduce_scatter<S, R>(mv, s, &owner);
    if (active && owner) {
      Real* pc = partg + (size_t)(j * nx + i) * kRec;
      if constexpr (sizeof(Real) == 8) {
#pragma unroll
        for (int k = 0; k < NSLOT; k += 2) {
          if (NSLOT == 1) {
            if (base < kRec) pc[base] = mv[0];
          } else if (base + k < kRec) {
            *reinterpret_cast<double2*>(pc + base + k) = make_double2(mv[k], mv[k + 1]);
          }
        }
      } else {
        // 16-float record: every slot exists (13..15 are zero pads)
        if constexpr (NSLOT >= 4) {
#pragma unroll
          for (int k = 0; k < NSLOT; k += 4)
            *reinterpret_cast<float4*>(pc + base + k) =
                make_float4((float)mv[k], (float)mv[k + 1], (float)mv[k + 2], (float)mv[k + 3]);
        } else if constexpr (NSLOT == 2) {
          *reinterpret_cast<float2*>(pc + base) = make_float2((float)mv[0], (float)mv[1]);
        } else {
          pc[base] = (float)mv[0];
        }
      }
    }

    // advance the lane and prefetch the material and the global-memory inflows of its next cell
    ++ip;
    if (ip == t.P) {
      ip = 0;
      n += NB;
    }
    take_material();
    if (warp == 0 && !band_wait(ip, n)) timed_out = true;
    load_inflow(ip, n);

    const int any_timeout = __syncthreads_or(timed_out ? 1 : 0);
    if (any_timeout) {
      timed_out = true;
      T_break = T;
      break;
    }
    // the step's wrap-buffer writes (top rows, before the barrier) go out with the progress count
    if (NB > 1 && threadIdx.x == 0 && T + 1 <= pub_stop) st_release_cluster(prog_remote, T + 1);
    if (tma_thread && T + stages < Tsteps) {
      mbar_arrive_expect_tx(&mbar[stage], stage_bytes);
      tma_bulk_g2s(ring + (size_t)stage * W * chunk, gold + (long long)(T + stages) * W * chunk, stage_bytes,
                   &mbar[stage]);
    }
    if (++stage == stages) {
      stage = 0;
      phase ^= 1u;
    }
  }

  if (timed_out) {
    if (threadIdx.x == 0) {
      atomicOr(a.err, kErrTmaTimeout);
      // drain: the copies of steps T_break .. T_break+stages-1 were issued and may be in flight; the
      // CTA must not exit before they land in its shared memory.  Waits are bounded.
      for (int s2 = T_break; s2 < T_break + stages && s2 < Tsteps; ++s2)
        (void)mbar_wait_bounded(&mbar[s2 % stages], (uint32_t)((s2 / stages) & 1), a.drain_polls);
    }
    __syncthreads();
  }
  // no band CTA leaves while another may still write into its shared memory
  if (NB > 1) cluster_sync_all();
  // every copy has landed (or the bounded drain gave up): the barriers can be set up again by a next task
  if (threadIdx.x == 0 && !timed_out)
    for (int k = 0; k < stages; ++k) mbar_inval(&mbar[k]);
  __syncthreads();
  return timed_out;
}

// MAXT/MINB: 512/1 fits every tiling (at most 128 registers per thread); 128/3 and 128/2 are the
// variants for CTAs of at most 4 warps when 3 or 2 of them per SM keep the whole grid resident: up to
// 170 or 255 registers per thread, which the solve uses for more independent directions in flight.
template <class Real, int S, int D, bool SRC_FULL, int MAXT = 512, int MINB = 1>
__global__ void __launch_bounds__(MAXT, MINB) scb_sweep_kernel(const SweepArgs<Real> a) {
  scb_sweep_body<Real, S, D, SRC_FULL>(a, blockIdx.x);
}

// Persistent form of the batched sweep: a grid of at most one wave of resident CTAs drains the queue of
// (instance, group, quadrant, split) sweeps, each CTA taking the next task from a global counter (reset
// before the launch) until none is left; tasks are ordered as the first-CTA table orders the instances
// (largest sweeps first).  One CTA per task (no band CTAs).  A CTA whose sweep timed out stops.
template <class Real, int S, int D, bool SRC_FULL, int MAXT = 512, int MINB = 1>
__global__ void __launch_bounds__(MAXT, MINB) scb_sweep_queue_kernel(const SweepArgs<Real>* __restrict__ args,
                                                              const int* __restrict__ first, int n, int total,
                                                              int* queue) {
  __shared__ SweepArgs<Real> sa;
  __shared__ int sbid, stask;
  for (;;) {
    if (threadIdx.x == 0) {
      stask = atomicAdd(queue, 1);
      if (stask < total) {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (first[mid] <= stask) lo = mid;
          else hi = mid - 1;
        }
        sa = args[lo];
        sbid = stask - first[lo];
      }
    }
    __syncthreads();
    if (stask >= total) break;
    if (scb_sweep_body<Real, S, D, SRC_FULL>(sa, sbid)) break;
  }
}

// One launch over the CTAs of several instances (same precision, slices, directions per lane, warps
// per CTA and stages): instance k owns CTAs [first[k], first[k+1]).  Its arguments are copied to
// shared memory once; the block scheduler then drains the (instance, group, quadrant, split) CTAs.
template <class Real, int S, int D, bool SRC_FULL, int MAXT = 512, int MINB = 1>
__global__ void __launch_bounds__(MAXT, MINB) scb_sweep_batch_kernel(const SweepArgs<Real>* __restrict__ args,
                                                              const int* __restrict__ first, int n) {
  __shared__ SweepArgs<Real> sa;
  __shared__ int sbid;
  if (threadIdx.x == 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (first[mid] <= (int)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    sa = args[lo];
    sbid = (int)blockIdx.x - first[lo];
  }
  __syncthreads();
  scb_sweep_body<Real, S, D, SRC_FULL>(sa, sbid);
}

}  // namespace trt
