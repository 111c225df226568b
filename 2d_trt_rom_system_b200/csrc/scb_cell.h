// Per-cell Simple Corner Balance (SCB) solve, shared by the CUDA sweep and the CPU oracle.
//
// The reference builds the 4x4 corner matrix in SCB_BGEN (MainSrc/TRANSPORT_SOLVES.f08:332-371) and
// solves it with the un-vendored LA_TOOLS routine GAUSS_COMPLETE (called at TRANSPORT_SOLVES.f08:79,
// 126,173,220).  Here the system is solved in closed form.  In the "sweep frame" of a quadrant
// (x and/or y mirrored so that both direction cosines are non-negative, corners ordered
// lb, rb, rt, lt of the mirrored cell) the matrix is
//
//     B = g*I + a*P + b*R,     g = (|Ox| dy + |Oy| dx + kapE dx dy)/4,  a = |Ox| dy/4,  b = |Oy| dx/4
//
// with P, R the two commuting signed permutations of SCB_BGEN (P^2 = R^2 = -I).  With S = P R
// (S^2 = I):  B (g I - a P - b R) = c I - d S,  c = g^2 + a^2 + b^2,  d = 2ab,  and
// (c I - d S)(c I + d S) = (c^2 - d^2) I, so
//
//     B^-1 = (g I - a P - b R)(c I + d S) / det,   det = (g^2 + (a-b)^2)(g^2 + (a+b)^2) > 0.
//
// Because g >= a + b both factors have condition number <= 2, so the formula is as accurate as
// Gaussian elimination on this matrix (a few ulp normwise).
//
// Every multiply-add below is an explicit fused multiply-add and every other operation is a single
// IEEE operation, so a build without automatic FMA contraction (nvcc --fmad=false, g++
// -ffp-contract=off) gives bit-identical results on the host and on the device.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define TRT_HD __host__ __device__ __forceinline__
#else
#define TRT_HD inline
#endif

namespace trt {

TRT_HD double tfma(double x, double y, double z) { return fma(x, y, z); }
TRT_HD float tfma(float x, float y, float z) { return fmaf(x, y, z); }

// Per-(cell, direction) geometry of the corner matrix, sweep frame.  ax4 = |Omega_x|/4 and
// ay4 = |Omega_y|/4 are per-direction constants; scaling by powers of two is exact, so
// a = ax4*dy equals (|Ox| dy)/4 of SCB_BGEN bit for bit.
template <class R>
struct ScbGeom {
  R a, b;      // |Ox| dy / 4, |Oy| dx / 4
  R hx, hy;    // |Ox| dy / 2, |Oy| dx / 2  (inflow face weights)
};

template <class R>
TRT_HD ScbGeom<R> scb_geom(R ax4, R ay4, R dx, R dy) {
  ScbGeom<R> G;
  G.a = ax4 * dy;
  G.b = ay4 * dx;
  G.hx = G.a + G.a;
  G.hy = G.b + G.b;
  return G;
}

// kA4 = (kapE * dx*dy) / 4, shared by every direction of a cell.
template <class R>
TRT_HD R scb_kA4(R dx, R dy, R kapE) {
  return (kapE * (dx * dy)) * R(0.25);
}

// gamma of SCB_BGEN, (|Ox| dy + |Oy| dx + kapE dx dy) / 4: the same sum with every term scaled by
// the exact factor 1/4 first.
template <class R>
TRT_HD R scb_gamma(const ScbGeom<R>& G, R kA4) {
  return (G.a + G.b) + kA4;
}

// Solve one cell.  s[k] = total corner source (isotropic/anisotropic source plus I_old/(c dt)),
// A4 = cell area / 4, vb/vt = inflow corner-edge values on the sweep-left face (bottom, top corner),
// hl/hr = inflow corner-edge values on the sweep-bottom face (left, right corner).
// x[] receives the corner intensities lb, rb, rt, lt of the sweep frame.
template <class R>
TRT_HD void scb_solve(const ScbGeom<R>& G, R gamma, R A4, const R s[4], R vb, R vt, R hl, R hr, R x[4]) {
  // right-hand side (TRANSPORT_SOLVES.f08:72-76 in the sweep frame)
  R Q1 = tfma(G.hy, hl, tfma(G.hx, vb, A4 * s[0]));
  R Q2 = tfma(G.hy, hr, A4 * s[1]);
  R Q3 = A4 * s[2];
  R Q4 = tfma(G.hx, vt, A4 * s[3]);

  const R a = G.a, b = G.b, g = gamma;
  R g2 = g * g;
  R c = tfma(g, g, tfma(a, a, b * b));
  R d = (a + a) * b;
  R amb = a - b;
  R apb = a + b;
  R det = tfma(amb, amb, g2) * tfma(apb, apb, g2);
  R inv = R(1) / det;

  R y1 = tfma(d, Q3, c * Q1);
  R y2 = tfma(-d, Q4, c * Q2);
  R y3 = tfma(d, Q1, c * Q3);
  R y4 = tfma(-d, Q2, c * Q4);

  x[0] = tfma(-b, y4, tfma(-a, y2, g * y1)) * inv;
  x[1] = tfma(-b, y3, tfma(a, y1, g * y2)) * inv;
  x[2] = tfma(b, y2, tfma(a, y4, g * y3)) * inv;
  x[3] = tfma(b, y1, tfma(-a, y3, g * y4)) * inv;
}

// Same solve for FP32 state ("mixed" precision).  det ~ gamma^4 overflows FP32 in optically thick
// cells (kappa*dx ~ 1e11 gives gamma ~ 1e10), so the system is scaled by 1/gamma first:
// B/gamma = I + a'P + b'R with a' = a/gamma, b' = b/gamma <= 1, whose inverse factors have
// determinant det' in [1, 5]; x = (I - a'P - b'R)(c'I + d'S) Q / (gamma det').
TRT_HD float frcp(float v) {
#if defined(__CUDA_ARCH__)
  return __fdividef(1.0f, v);
#else
  return 1.0f / v;
#endif
}

TRT_HD void scb_solve(const ScbGeom<float>& G, float gamma, float A4, const float s[4], float vb, float vt, float hl,
                      float hr, float x[4]) {
  float Q1 = tfma(G.hy, hl, tfma(G.hx, vb, A4 * s[0]));
  float Q2 = tfma(G.hy, hr, A4 * s[1]);
  float Q3 = A4 * s[2];
  float Q4 = tfma(G.hx, vt, A4 * s[3]);

  const float r = frcp(gamma);
  const float a = G.a * r, b = G.b * r;
  const float c = tfma(a, a, tfma(b, b, 1.0f));
  const float d = (a + a) * b;
  const float amb = a - b, apb = a + b;
  const float det = tfma(amb, amb, 1.0f) * tfma(apb, apb, 1.0f);
  const float inv = r * frcp(det);

  const float y1 = tfma(d, Q3, c * Q1);
  const float y2 = tfma(-d, Q4, c * Q2);
  const float y3 = tfma(d, Q1, c * Q3);
  const float y4 = tfma(-d, Q2, c * Q4);

  x[0] = tfma(-b, y4, tfma(-a, y2, y1)) * inv;
  x[1] = tfma(-b, y3, tfma(a, y1, y2)) * inv;
  x[2] = tfma(b, y2, tfma(a, y4, y3)) * inv;
  x[3] = tfma(b, y1, tfma(-a, y3, y4)) * inv;
}

#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
// Two directions at once on the packed FP32x2 pipe of sm_100 (component .x = one direction, .y =
// another): the FP32 solve above, operation for operation.  Each packed operation rounds each
// component as the scalar one does, and negations are multiplications by -1 (exact), so both
// components are bit-identical to two calls of the scalar solve.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 frcp2(float2 v) { return make_float2(frcp(v.x), frcp(v.y)); }

struct ScbGeom2 {
  float2 a, b, hx, hy;
};

__device__ __forceinline__ ScbGeom2 scb_geom2(float2 ax4, float2 ay4, float dx, float dy) {
  ScbGeom2 G;
  G.a = __fmul2_rn(ax4, f2(dy));
  G.b = __fmul2_rn(ay4, f2(dx));
  G.hx = __fadd2_rn(G.a, G.a);
  G.hy = __fadd2_rn(G.b, G.b);
  return G;
}

__device__ __forceinline__ float2 scb_gamma2(const ScbGeom2& G, float kA4) {
  return __fadd2_rn(__fadd2_rn(G.a, G.b), f2(kA4));
}

__device__ __forceinline__ void scb_solve2(const ScbGeom2& G, float2 gamma, float A4, const float2 s[4], float2 vb,
                                           float2 vt, float2 hl, float2 hr, float2 x[4]) {
  const float2 A = f2(A4), one = f2(1.0f), m1 = f2(-1.0f);
  const float2 Q1 = __ffma2_rn(G.hy, hl, __ffma2_rn(G.hx, vb, __fmul2_rn(A, s[0])));
  const float2 Q2 = __ffma2_rn(G.hy, hr, __fmul2_rn(A, s[1]));
  const float2 Q3 = __fmul2_rn(A, s[2]);
  const float2 Q4 = __ffma2_rn(G.hx, vt, __fmul2_rn(A, s[3]));

  const float2 r = frcp2(gamma);
  const float2 a = __fmul2_rn(G.a, r), b = __fmul2_rn(G.b, r);
  const float2 c = __ffma2_rn(a, a, __ffma2_rn(b, b, one));
  const float2 d = __fmul2_rn(__fadd2_rn(a, a), b);
  const float2 amb = __ffma2_rn(b, m1, a), apb = __fadd2_rn(a, b);
  const float2 det = __fmul2_rn(__ffma2_rn(amb, amb, one), __ffma2_rn(apb, apb, one));
  const float2 inv = __fmul2_rn(r, frcp2(det));
  const float2 nd = __fmul2_rn(d, m1), na = __fmul2_rn(a, m1), nb = __fmul2_rn(b, m1);

  const float2 y1 = __ffma2_rn(d, Q3, __fmul2_rn(c, Q1));
  const float2 y2 = __ffma2_rn(nd, Q4, __fmul2_rn(c, Q2));
  const float2 y3 = __ffma2_rn(d, Q1, __fmul2_rn(c, Q3));
  const float2 y4 = __ffma2_rn(nd, Q2, __fmul2_rn(c, Q4));

  x[0] = __fmul2_rn(__ffma2_rn(nb, y4, __ffma2_rn(na, y2, y1)), inv);
  x[1] = __fmul2_rn(__ffma2_rn(nb, y3, __ffma2_rn(a, y1, y2)), inv);
  x[2] = __fmul2_rn(__ffma2_rn(b, y2, __ffma2_rn(a, y4, y3)), inv);
  x[3] = __fmul2_rn(__ffma2_rn(b, y1, __ffma2_rn(na, y3, y4)), inv);
}
#endif

}  // namespace trt
