// Device data layout of one sweep instance (host and device code).
//
// Reference arrays (MainSrc/INITIALIZERS.f08:41-49) are Fortran column-major, e.g.
// I_crn(2*N_x, 2*N_y, N_m, N_g).  On the device the angular state I_crn is stored in a private
// "skewed" layout built for the wavefront sweep; every other array keeps the reference layout.
//
// Sweep frame.  Quadrant q (0..3 = directions m in [q*mq, (q+1)*mq), ordered (+,+), (-,+), (-,-),
// (+,-) as INPUT_QUAD builds them, MainSrc/INPUTS.f08:1658-1669) is swept in the frame where x is
// mirrored when Omega_x < 0 (fx) and y when Omega_y < 0 (fy): i' = fx ? nx-1-i : i, j' likewise.
// In that frame every quadrant sweeps i' and j' upward, which is the loop order of
// TRANSPORT_SOLVES.f08:58-241 mirrored.  Corners of a cell are numbered in the frame: 0 = lb,
// 1 = rb, 2 = rt, 3 = lt.
//
// Work decomposition.  One CTA sweeps one (group, quadrant, direction split): the mq directions of
// a quadrant are split into NH contiguous parts of floor/ceil(mq/NH) directions (more CTAs than
// (group, quadrant) pairs balance the SMs).  A CTA has W warps; a warp holds R rows x S direction
// slices (R*S = 32, lane = s*R + r).  Lane (s, r) of warp w owns the directions d*S + s (d < D) of
// its split and the row rho = w*R + r of a band of H = W*R rows.
// Bands ("rounds") n = 0..nr-1 cover j' = n*H + rho.  Step T of the CTA puts every lane on the
// anti-diagonal cell i' = T - rho - n*P (P = period, nx <= P, H < P), so lane rows form a wavefront:
// a cell's left inflow comes from the same lane one step earlier, its bottom inflow from the row
// below one step earlier.
//
// Spatial tiles.  With NB > 1 the rounds of one (g, q, h) sweep are dealt round-robin to NB CTAs
// (one thread-block cluster): CTA b sweeps rounds n = b, b + NB, b + 2 NB, ... one after the other
// (local round k = n / NB starts at local step k*P), and round n's first row takes its bottom inflow
// from round n-1's top outflow, written by the neighbouring CTA of the cluster into the L2-resident
// wrap buffer.  The CTAs run as a pipeline of row tiles on a tile-diagonal wavefront, each about H
// steps behind the one below.  Every step index below is local to a CTA: cell (i', j') of round n
// sits at step T = (n % NB) * Tb + (n / NB) * P + i' + rho of its (g, q, h) block, where Tb (steps
// per band) is the local step count of the band with the most rounds.
//
// Skewed state layout.  For each (g, q, h) a block of Tsteps*W chunks; chunk (T, w) holds the cells
// the lanes of warp w touch at step T, as D sub-blocks (one per d) of nl_d lanes
// (nl_d = R*min(S, mqc - d*S), mqc = ceil(mq/NH)); a lane's 4 corners are stored as 16-byte vectors ("pairs" for
// FP64, one vector for FP32), vector-major inside a sub-block so that a warp's load of one vector
// is one contiguous 16*nl_d-byte run.  A whole CTA step is W contiguous chunks, which one TMA
// bulk copy stages into shared memory.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define TRT_LHD __host__ __device__ __forceinline__
#else
#define TRT_LHD inline
#endif

namespace trt {

struct Tiling {
  int W;       // warps per CTA
  int S;       // direction slices per warp (power of two)
  int R;       // rows per warp = 32 / S
  int NH;      // direction splits per quadrant (CTAs per (group, quadrant))
  int mqc;     // directions of the largest split = ceil(mq / NH) (chunk width)
  int D;       // directions per lane = ceil(mqc / S)
  int H;       // rows per round = W * R
  int P;       // period = max(nx, H + 1)
  int nr;      // rounds = ceil(ny / H)
  int NB;      // band CTAs per (g, q, h) sweep (rounds dealt round-robin); 1 = one CTA sweeps every round
  int Tb;      // local steps of a band CTA with the most rounds = (ceil(nr/NB)-1)*P + nx + H - 1
  int Tsteps;  // steps of one (g, q, h) block = NB * Tb
};

TRT_LHD int ceil_div(int a, int b) { return (a + b - 1) / b; }

TRT_LHD Tiling make_tiling(int nx, int ny, int mq, int W, int S, int NH, int NB = 1) {
  Tiling t;
  t.W = W;
  t.S = S;
  t.R = 32 / S;
  t.NH = NH;
  t.mqc = ceil_div(mq, NH);
  t.D = ceil_div(t.mqc, S);
  t.H = W * t.R;
  t.P = nx > t.H ? nx : t.H + 1;   // P > H: a round's wrap entry is written a step before it is prefetched
  t.nr = ceil_div(ny, t.H);
  t.NB = NB < 1 ? 1 : (NB > t.nr ? t.nr : NB);
  t.Tb = (ceil_div(t.nr, t.NB) - 1) * t.P + nx + t.H - 1;
  t.Tsteps = t.NB * t.Tb;
  return t;
}

// Rounds of band b (n = b, b + NB, ...) and its local step count.
TRT_LHD int band_rounds(const Tiling& t, int b) { return ceil_div(t.nr - b, t.NB); }
TRT_LHD int band_steps(const Tiling& t, int nx, int b) { return (band_rounds(t, b) - 1) * t.P + nx + t.H - 1; }

// Direction split h of a quadrant: first quadrant-local direction and count (floor/ceil(mq/NH)).
TRT_LHD int split_first(int mq, int NH, int h) { return h * (mq / NH) + (h < mq % NH ? h : mq % NH); }
TRT_LHD int split_count(int mq, int NH, int h) { return mq / NH + (h < mq % NH ? 1 : 0); }

// Elements per chunk (T, w): mqc directions x R rows x 4 corners.
TRT_LHD long long chunk_elems(const Tiling& t) { return (long long)t.mqc * t.R * 4; }
// Elements per (g, q, h) block.
TRT_LHD long long block_elems(const Tiling& t) { return (long long)t.Tsteps * t.W * chunk_elems(t); }

// Offset of corner c (frame numbering) of split-local direction mloc of lane (s, r) of warp w at
// step T, inside one (g, q, h) block.  NV = 16 / sizeof(Real) values per 16-byte vector.
template <int NV>
TRT_LHD long long skew_offset(const Tiling& t, int T, int w, int mloc, int r, int c) {
  const int d = mloc / t.S;
  const int s = mloc % t.S;
  const int nslice = (t.mqc - d * t.S) < t.S ? (t.mqc - d * t.S) : t.S;
  const int nl = t.R * nslice;
  const int lane = s * t.R + r;
  long long off = ((long long)T * t.W + w) * chunk_elems(t);
  off += (long long)d * 128;              // all earlier sub-blocks are full (32 lanes x 4)
  off += (long long)(c / NV) * nl * NV + (long long)lane * NV + (c % NV);
  return off;
}

// Map a physical cell (i, j) of quadrant q to (T, w, r) of the sweep.
struct SweepPos {
  int T, w, r;
};
TRT_LHD SweepPos sweep_pos(int nx, int ny, const Tiling& t, int q, int i, int j) {
  const bool fx = (q == 1 || q == 2), fy = (q >= 2);
  const int ip = fx ? nx - 1 - i : i;
  const int jp = fy ? ny - 1 - j : j;
  const int n = jp / t.H, rho = jp % t.H;
  SweepPos p;
  p.T = (n % t.NB) * t.Tb + (n / t.NB) * t.P + ip + rho;
  p.w = rho / t.R;
  p.r = rho % t.R;
  return p;
}

// Physical corner (cx: 0 left / 1 right, cy: 0 bottom / 1 top) -> frame corner number.
TRT_LHD int frame_corner(int q, int cx, int cy) {
  const int fx = (q == 1 || q == 2), fy = (q >= 2);
  const int sx = cx ^ fx, sy = cy ^ fy;
  return sy ? (sx ? 2 : 3) : (sx ? 1 : 0);
}

// Moment partial record of one (cell, quadrant, split): 13 values, padded to whole 16-byte vectors.
// Records hold the state's precision: 14 doubles (112 B) for FP64, 16 floats (64 B) for FP32 (the
// FP32 sweep's lane sums are FP64 and are rounded once, when the record is written).
constexpr int kNPartUsed = 13;
template <class P>
TRT_LHD constexpr int part_rec() { return sizeof(P) == 4 ? 16 : 14; }
// Partial value slots.  Signs are physical (Omega as given by the caller).
enum PartSlot {
  kCxx = 0, kCyy, kCxy, kCe,        // cell centre: w Ox^2, w Oy^2, w Ox Oy, w       (x I_avg)
  kVxx, kVxy, kVx, kVe,             // downwind vertical face: w Ox^2, w Ox Oy, w Ox, w  (x I_edgV)
  kHyy, kHxy, kHy, kHx, kHe         // downwind horizontal face: w Oy^2, w Ox Oy, w Oy, w Ox, w (x I_edgH)
};

}  // namespace trt
