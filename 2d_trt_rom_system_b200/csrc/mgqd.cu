// Host side of the device MGQD solve: trt_mloqd_fv and trt_old_mgqd_coefs (include/trt_sweep.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "trt_sweep.h"
#include "mgqd_kernels.cuh"

namespace trt_host {
void add_launches(unsigned long long n);   // library-wide launch counter (trt_api.cu)
}

namespace {

using namespace trt_mgqd;

#define MG_CUDA(expr)                                   \
  do {                                                  \
    cudaError_t e_ = (expr);                            \
    if (e_ != cudaSuccess) {                            \
      if (e_ == cudaErrorMemoryAllocation) {            \
        cudaGetLastError();                             \
        return TRT_ERR_NOMEM;                           \
      }                                                 \
      return TRT_ERR_CUDA;                              \
    }                                                   \
  } while (0)

// after each launch: count it and surface a launch error
#define MG_LAUNCHED()                  \
  do {                                 \
    trt_host::add_launches(1);         \
    MG_CUDA(cudaGetLastError());       \
  } while (0)

constexpr int kSmallCells = 1024;   // levels at or below this many cells run in the one-CTA kernel
constexpr int kNu1 = 2, kNu2 = 2, kCoarseSweeps = 16;
constexpr int kCheckEvery = 4;      // iterations between host checks of the convergence flags

struct Settings {
  double tol = 1e-13;
  int maxit = 1000;
};
Settings g_settings;

// Device buffers of one (nx, ny, ng) shape, reused across calls.
struct Solver {
  Dims d{};
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr, m0 = nullptr, m1 = nullptr;   // solve; first matrix-vector product
  std::vector<void*> bufs;
  Inputs in{};
  Coefs cf{};
  Krylov K{};
  LevelSet ls{};
  int k0 = 0;
  double *Fx = nullptr, *Fy = nullptr, *rpart = nullptr, *res = nullptr, *bcres = nullptr;
  int* h_done = nullptr;
  Scal* h_scal = nullptr;
  float last_ms = 0.f, last_matvec_ms = 0.f;
  bool matvec_timed = false;
  int last_its = 0;

  ~Solver() {
    for (void* p : bufs) cudaFree(p);
    if (h_done) cudaFreeHost(h_done);
    if (h_scal) cudaFreeHost(h_scal);
    for (cudaEvent_t e : {e0, e1, m0, m1})
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }
  template <class T>
  int alloc(T** p, size_t n) {
    if (cudaMalloc(p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      *p = nullptr;
      return TRT_ERR_NOMEM;
    }
    bufs.push_back(*p);
    return TRT_OK;
  }
  int init(int nx, int ny, int ng);
  int solve(cudaStream_t s);
  int pos_blocks() const { return (int)((d.npos() + kRedBlock - 1) / kRedBlock); }
};

int Solver::init(int nx, int ny, int ng) {
  d.nx = nx;
  d.ny = ny;
  d.ng = ng;
  d.nC = (long)nx * ny;
  d.nV = (long)(nx + 1) * ny;
  d.nH = (long)nx * (ny + 1);
  d.nU = d.nC + d.nV + d.nH;
  MG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  MG_CUDA(cudaEventCreate(&e0));
  MG_CUDA(cudaEventCreate(&e1));
  MG_CUDA(cudaEventCreate(&m0));
  MG_CUDA(cudaEventCreate(&m1));
  const size_t C = (size_t)d.nC * ng, V = (size_t)d.nV * ng, H = (size_t)d.nH * ng, U = (size_t)d.nU * ng;
  int rc = TRT_OK;
  auto A = [&](const double** p, size_t n) {
    double* q = nullptr;
    if (!rc) rc = alloc(&q, n);
    *p = q;
  };
  auto M = [&](auto** p, size_t n) {
    if (!rc) rc = alloc(p, n);
  };
  // inputs
  A(&in.fxx, C); A(&in.fyy, C); A(&in.fVxx, V); A(&in.fVxy, V); A(&in.fHyy, H); A(&in.fHxy, H);
  A(&in.CgL, (size_t)ny * ng); A(&in.CgB, (size_t)nx * ng); A(&in.CgR, (size_t)ny * ng); A(&in.CgT, (size_t)nx * ng);
  A(&in.EinL, (size_t)ny * ng); A(&in.EinB, (size_t)nx * ng); A(&in.EinR, (size_t)ny * ng); A(&in.EinT, (size_t)nx * ng);
  A(&in.FinL, (size_t)ny * ng); A(&in.FinB, (size_t)nx * ng); A(&in.FinR, (size_t)ny * ng); A(&in.FinT, (size_t)nx * ng);
  A(&in.Src, C); A(&in.KapE, C); A(&in.KapR, C); A(&in.Delx, nx); A(&in.Dely, ny); A(&in.A, d.nC);
  A(&in.Gold, C); A(&in.PoldL, C); A(&in.PoldB, C); A(&in.PoldR, C); A(&in.PoldT, C);
  A(&in.Eold, C); A(&in.Fxold, V); A(&in.Fyold, H);
  // coefficients
  M(&cf.Xi, C); M(&cf.PhL, C); M(&cf.PhB, C); M(&cf.PhR, C); M(&cf.PhT, C);
  M(&cf.EBL, C); M(&cf.EBB, C); M(&cf.EBC, C); M(&cf.EBR, C); M(&cf.EBT, C);
  M(&cf.MXB, C); M(&cf.MXC, C); M(&cf.MXT, C); M(&cf.MYL, C); M(&cf.MYC, C); M(&cf.MYR, C);
  M(&cf.dV, V); M(&cf.dH, H); M(&cf.b, U);
  M(&cf.aV, V); M(&cf.blV, V); M(&cf.brV, V); M(&cf.aH, H); M(&cf.bbH, H); M(&cf.btH, H);
  // Krylov vectors
  M(&K.x, U); M(&K.r, U); M(&K.rh, U); M(&K.p0, U); M(&K.p1, U); M(&K.v, U); M(&K.s, U); M(&K.t, U);
  M(&K.ph, U); M(&K.sh, U);
  const int nblk = pos_blocks();
  M(&K.part, (size_t)ng * nblk * 4);
  M(&rpart, (size_t)ng * nblk * kNRes);
  M(&Fx, V); M(&Fy, H); M(&res, (size_t)ng * 25); M(&bcres, (size_t)ng * 4);
  double* sc = nullptr;
  M(&sc, (sizeof(Scal) * ng + sizeof(double) - 1) / sizeof(double));
  double* dn = nullptr;
  M(&dn, ((size_t)ng * sizeof(int) + sizeof(double) - 1) / sizeof(double));
  if (rc) return rc;
  K.sc = reinterpret_cast<Scal*>(sc);
  K.done = reinterpret_cast<int*>(dn);
  // multigrid levels: halve (rounding up) until both extents are at most 2
  int mx = nx, my = ny;
  ls.n = 0;
  for (;;) {
    if (ls.n == kMaxLevels) return TRT_ERR_UNSUPPORTED;
    Level& L = ls.L[ls.n++];
    L.mx = mx;
    L.my = my;
    L.n = (long)mx * my;
    M(&L.sC, (size_t)L.n * ng); M(&L.sW, (size_t)L.n * ng); M(&L.sE, (size_t)L.n * ng);
    M(&L.sS, (size_t)L.n * ng); M(&L.sN, (size_t)L.n * ng); M(&L.x, (size_t)L.n * ng); M(&L.b, (size_t)L.n * ng);
    if (rc) return rc;
    if (mx <= 2 && my <= 2) break;
    mx = (mx + 1) / 2;
    my = (my + 1) / 2;
  }
  k0 = 0;
  while (ls.L[k0].n > kSmallCells) ++k0;
  MG_CUDA(cudaMallocHost(&h_done, sizeof(int) * ng));
  MG_CUDA(cudaMallocHost(&h_scal, sizeof(Scal) * ng));
  return TRT_OK;
}

int grid1(long n) { return (int)((n + 255) / 256); }

// Right-preconditioned BiCGSTAB over all groups; inputs and the initial guess (K.x) already on the device.
int Solver::solve(cudaStream_t s) {
  const int ng = d.ng;
  const dim3 gpos(pos_blocks(), ng);
  const int nblk = pos_blocks();
  matvec_timed = false;
  K.tol = g_settings.tol;
  K.maxit = g_settings.maxit;
  coef_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, cf);
  MG_LAUNCHED();
  prec_coef_kernel<<<gpos, kRedBlock, 0, s>>>(d, cf, ls.L[0]);
  MG_LAUNCHED();
  for (int k = 0; k + 1 < ls.n; ++k) {
    coarse_op_kernel<<<dim3(grid1(ls.L[k + 1].n), ng), 256, 0, s>>>(ls.L[k], ls.L[k + 1]);
    MG_LAUNCHED();
  }
  init_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K);
  MG_LAUNCHED();
  init_finish_kernel<<<ng, 32, 0, s>>>(K, nblk);
  MG_LAUNCHED();

  auto vcycle = [&]() -> int {
    for (int k = 0; k < k0; ++k) {
      const Level& L = ls.L[k];
      const dim3 gl(grid1(L.n), ng);
      for (int sw = 0; sw < kNu1; ++sw) {
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 0, sw == 0 ? 1 : 0);
        MG_LAUNCHED();
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 1, 0);
        MG_LAUNCHED();
      }
      restrict_kernel<<<dim3(grid1(ls.L[k + 1].n), ng), 256, 0, s>>>(L, ls.L[k + 1], K.done);
      MG_LAUNCHED();
    }
    small_vcycle_kernel<<<ng, 256, 0, s>>>(ls, k0, kNu1, kNu2, kCoarseSweeps, K.done);
    MG_LAUNCHED();
    for (int k = k0 - 1; k >= 0; --k) {
      const Level& L = ls.L[k];
      const dim3 gl(grid1(L.n), ng);
      prolong_kernel<<<gl, 256, 0, s>>>(L, ls.L[k + 1], K.done);
      MG_LAUNCHED();
      for (int sw = 0; sw < kNu2; ++sw) {
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 0, 0);
        MG_LAUNCHED();
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 1, 0);
        MG_LAUNCHED();
      }
    }
    return TRT_OK;
  };

  int rc;
  for (int it = 0; it < K.maxit; ++it) {
    if (it % kCheckEvery == 0) {
      MG_CUDA(cudaMemcpyAsync(h_done, K.done, sizeof(int) * ng, cudaMemcpyDeviceToHost, s));
      MG_CUDA(cudaStreamSynchronize(s));
      bool all = true;
      for (int g = 0; g < ng; ++g) all = all && h_done[g] != 0;
      if (all) break;
    }
    double* pold = (it & 1) ? K.p1 : K.p0;
    double* pnew = (it & 1) ? K.p0 : K.p1;
    elim_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], pold, pnew, 0);
    MG_LAUNCHED();
    if ((rc = vcycle())) return rc;
    backsub_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], pnew, K.ph);
    MG_LAUNCHED();
    matvec_timed = matvec_timed || it == 0;
    if (it == 0) MG_CUDA(cudaEventRecord(m0, s));
    matvec_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, K.ph, K.v, 0);
    MG_LAUNCHED();
    if (it == 0) MG_CUDA(cudaEventRecord(m1, s));
    scalar_finish_kernel<<<ng, 32, 0, s>>>(K, nblk, 0);
    MG_LAUNCHED();
    elim_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], nullptr, K.s, 1);
    MG_LAUNCHED();
    if ((rc = vcycle())) return rc;
    backsub_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], K.s, K.sh);
    MG_LAUNCHED();
    matvec_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, K.sh, K.t, 1);
    MG_LAUNCHED();
    scalar_finish_kernel<<<ng, 32, 0, s>>>(K, nblk, 1);
    MG_LAUNCHED();
    update_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K);
    MG_LAUNCHED();
    update_finish_kernel<<<ng, 32, 0, s>>>(K, nblk);
    MG_LAUNCHED();
  }
  const Outputs out{Fx, Fy};
  flux_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, cf, K.x, out);
  MG_LAUNCHED();
  residual_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, K.x, out, rpart);
  MG_LAUNCHED();
  residual_finish_kernel<<<ng, 32, 0, s>>>(rpart, nblk, ng, res, bcres);
  MG_LAUNCHED();
  return TRT_OK;
}

struct Cache {
  std::mutex mu;
  std::unique_ptr<Solver> s;
};
Cache g_cache;

int device_ok() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    cudaGetLastError();
    return TRT_ERR_NODEV;
  }
  return TRT_OK;
}

int get_solver(int nx, int ny, int ng, Solver** out) {
  Solver* s = g_cache.s.get();
  if (!s || s->d.nx != nx || s->d.ny != ny || s->d.ng != ng) {
    g_cache.s.reset();
    auto fresh = std::make_unique<Solver>();
    const int rc = fresh->init(nx, ny, ng);
    if (rc) return rc;
    g_cache.s = std::move(fresh);
  }
  *out = g_cache.s.get();
  return TRT_OK;
}

int put(cudaStream_t st, const double* dst, const double* src, size_t n) {
  MG_CUDA(cudaMemcpyAsync(const_cast<double*>(dst), src, n * sizeof(double), cudaMemcpyHostToDevice, st));
  return TRT_OK;
}

}  // namespace

extern "C" {

int trt_mgqd_set_tolerance(double tol, int maxit) {
  if (!(tol > 0.0) || maxit < 1) return TRT_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_cache.mu);
  g_settings.tol = tol;
  g_settings.maxit = maxit;
  return TRT_OK;
}

int trt_mgqd_last_stats(double* device_ms, int* max_iterations, double* matvec_ms) {
  std::lock_guard<std::mutex> lk(g_cache.mu);
  if (!g_cache.s) return TRT_ERR_STATE;
  if (device_ms) *device_ms = g_cache.s->last_ms;
  if (max_iterations) *max_iterations = g_cache.s->last_its;
  if (matvec_ms) *matvec_ms = g_cache.s->last_matvec_ms;
  return TRT_OK;
}

int trt_mloqd_fv(int n_x, int n_y, int n_g, double* Eg_avg, double* Eg_edgV, double* Eg_edgH, double* Fxg_edgV,
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
  (void)Open_Threads;
  const double* ins[] = {fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy, Cg_L, Cg_B, Cg_R,
                         Cg_T, Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T, Src, KapE,
                         KapR, Delx, Dely, A, G_old, Pold_L, Pold_B, Pold_R, Pold_T, Eg_avg_old, Fxg_edgV_old,
                         Fyg_edgH_old};
  if (n_x < 1 || n_y < 1 || n_g < 1 || n_g > 65535 || !Eg_avg || !Eg_edgV || !Eg_edgH || !Fxg_edgV || !Fyg_edgH ||
      !MGQD_Kits || (Res_Calc && (!MGQD_Residual || !MGQD_BC_Residual)) || !(Theta != 0.0) || !(Delt > 0.0) ||
      !(c > 0.0))
    return TRT_ERR_ARG;
  for (const double* p : ins)
    if (!p) return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_cache.mu);
  Solver* S = nullptr;
  if ((rc = get_solver(n_x, n_y, n_g, &S))) return rc;
  const Dims& d = S->d;
  Inputs& in = S->in;
  const size_t C = (size_t)d.nC * n_g, V = (size_t)d.nV * n_g, H = (size_t)d.nH * n_g;
  const size_t by = (size_t)n_y * n_g, bx = (size_t)n_x * n_g;
  cudaStream_t st = S->st;
  const struct {
    const double* dst;
    const double* src;
    size_t n;
  } up[] = {{in.fxx, fg_avg_xx, C},   {in.fyy, fg_avg_yy, C},     {in.fVxx, fg_edgV_xx, V}, {in.fVxy, fg_edgV_xy, V},
            {in.fHyy, fg_edgH_yy, H}, {in.fHxy, fg_edgH_xy, H},   {in.CgL, Cg_L, by},       {in.CgB, Cg_B, bx},
            {in.CgR, Cg_R, by},       {in.CgT, Cg_T, bx},         {in.EinL, Eg_in_L, by},   {in.EinB, Eg_in_B, bx},
            {in.EinR, Eg_in_R, by},   {in.EinT, Eg_in_T, bx},     {in.FinL, Fg_in_L, by},   {in.FinB, Fg_in_B, bx},
            {in.FinR, Fg_in_R, by},   {in.FinT, Fg_in_T, bx},     {in.Src, Src, C},         {in.KapE, KapE, C},
            {in.KapR, KapR, C},       {in.Delx, Delx, (size_t)n_x}, {in.Dely, Dely, (size_t)n_y},
            {in.A, A, (size_t)d.nC},  {in.Gold, G_old, C},        {in.PoldL, Pold_L, C},    {in.PoldB, Pold_B, C},
            {in.PoldR, Pold_R, C},    {in.PoldT, Pold_T, C},      {in.Eold, Eg_avg_old, C}, {in.Fxold, Fxg_edgV_old, V},
            {in.Fyold, Fyg_edgH_old, H}};
  for (const auto& u : up)
    if ((rc = put(st, u.dst, u.src, u.n))) return rc;
  in.c = c;
  in.Delt = Delt;
  in.Theta = Theta;
  in.Fdt = Fdt_Weight;
  in.Fin = Fin_Weight;
  in.Ein = Ein_Weight;
  // initial guess: the E fields passed in, into the unknown layout
  const size_t pitch = (size_t)d.nU * sizeof(double);
  MG_CUDA(cudaMemcpy2DAsync(S->K.x, pitch, Eg_avg, d.nC * sizeof(double), d.nC * sizeof(double), n_g,
                            cudaMemcpyHostToDevice, st));
  MG_CUDA(cudaMemcpy2DAsync(S->K.x + d.oV(), pitch, Eg_edgV, d.nV * sizeof(double), d.nV * sizeof(double), n_g,
                            cudaMemcpyHostToDevice, st));
  MG_CUDA(cudaMemcpy2DAsync(S->K.x + d.oH(), pitch, Eg_edgH, d.nH * sizeof(double), d.nH * sizeof(double), n_g,
                            cudaMemcpyHostToDevice, st));
  MG_CUDA(cudaEventRecord(S->e0, st));
  if ((rc = S->solve(st))) return rc;
  MG_CUDA(cudaEventRecord(S->e1, st));
  MG_CUDA(cudaMemcpy2DAsync(Eg_avg, d.nC * sizeof(double), S->K.x, pitch, d.nC * sizeof(double), n_g,
                            cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpy2DAsync(Eg_edgV, d.nV * sizeof(double), S->K.x + d.oV(), pitch, d.nV * sizeof(double), n_g,
                            cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpy2DAsync(Eg_edgH, d.nH * sizeof(double), S->K.x + d.oH(), pitch, d.nH * sizeof(double), n_g,
                            cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpyAsync(Fxg_edgV, S->Fx, V * sizeof(double), cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpyAsync(Fyg_edgH, S->Fy, H * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (Res_Calc) {
    MG_CUDA(cudaMemcpyAsync(MGQD_Residual, S->res, (size_t)n_g * 25 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaMemcpyAsync(MGQD_BC_Residual, S->bcres, (size_t)n_g * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  MG_CUDA(cudaMemcpyAsync(S->h_scal, S->K.sc, sizeof(Scal) * n_g, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  MG_CUDA(cudaEventElapsedTime(&S->last_ms, S->e0, S->e1));
  S->last_matvec_ms = 0.f;
  if (S->matvec_timed && cudaEventElapsedTime(&S->last_matvec_ms, S->m0, S->m1) != cudaSuccess) {
    cudaGetLastError();
    S->last_matvec_ms = 0.f;
  }
  bool conv = true;
  S->last_its = 0;
  for (int g = 0; g < n_g; ++g) {
    const Scal& sc = S->h_scal[g];
    S->last_its = std::max(S->last_its, sc.its);
    // matrix-vector products, as the reference counts them (ipar(7)): one for the initial residual
    // and two per iteration
    MGQD_Kits[g] = 1 + 2 * sc.its;
    if (sc.done != 1) {
      conv = false;
      MGQD_Kits[g] = -MGQD_Kits[g];
    }
  }
  return conv ? TRT_OK : TRT_ERR_NOCONV;
}

int trt_old_mgqd_coefs(int n_x, int n_y, int n_g, const double* Eg_avg_old, const double* Eg_edgV_old,
                       const double* Eg_edgH_old, const double* Fxg_edgV_old, const double* Fyg_edgH_old,
                       const double* fg_avg_xx_old, const double* fg_avg_yy_old, const double* fg_edgV_xx_old,
                       const double* fg_edgV_xy_old, const double* fg_edgH_yy_old, const double* fg_edgH_xy_old,
                       const double* KapE_old, const double* KapR_old, const double* Src_old, const double* Delx,
                       const double* Dely, const double* A, double c, double Delt, double Theta, double* G_old,
                       double* Pold_L, double* Pold_B, double* Pold_R, double* Pold_T, int Open_Threads) {
  (void)Open_Threads;
  (void)Delt;
  const double* ins[] = {Eg_avg_old,     Eg_edgV_old,    Eg_edgH_old,    Fxg_edgV_old,   Fyg_edgH_old, fg_avg_xx_old,
                         fg_avg_yy_old,  fg_edgV_xx_old, fg_edgV_xy_old, fg_edgH_yy_old, fg_edgH_xy_old, KapE_old,
                         KapR_old,       Src_old,        Delx,           Dely,           A};
  double* outs[] = {G_old, Pold_L, Pold_B, Pold_R, Pold_T};
  if (n_x < 1 || n_y < 1 || n_g < 1 || n_g > 65535 || !(Theta != 0.0)) return TRT_ERR_ARG;
  for (const double* p : ins)
    if (!p) return TRT_ERR_ARG;
  for (double* p : outs)
    if (!p) return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  Dims d{};
  d.nx = n_x;
  d.ny = n_y;
  d.ng = n_g;
  d.nC = (long)n_x * n_y;
  d.nV = (long)(n_x + 1) * n_y;
  d.nH = (long)n_x * (n_y + 1);
  d.nU = d.nC + d.nV + d.nH;
  const size_t C = (size_t)d.nC * n_g, V = (size_t)d.nV * n_g, H = (size_t)d.nH * n_g;
  const size_t sz[17] = {C, V, H, V, H, C, C, V, V, H, H, C, C, C, (size_t)n_x, (size_t)n_y, (size_t)d.nC};
  std::vector<double*> dev(22, nullptr);
  auto release = [&]() {
    for (double* p : dev)
      if (p) cudaFree(p);
  };
  for (int k = 0; k < 22; ++k) {
    const size_t n = k < 17 ? sz[k] : C;
    if (cudaMalloc(&dev[k], n * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      release();
      return TRT_ERR_NOMEM;
    }
    if (k < 17 && cudaMemcpy(dev[k], ins[k], n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      release();
      return TRT_ERR_CUDA;
    }
  }
  const OldIn oi{dev[0], dev[1], dev[2],  dev[3],  dev[4],  dev[5],  dev[6],  dev[7], dev[8],
                 dev[9], dev[10], dev[11], dev[12], dev[13], dev[14], dev[15], dev[16], c, Theta};
  const OldOut oo{dev[17], dev[18], dev[19], dev[20], dev[21]};
  old_coefs_kernel<<<dim3(grid1(d.nC), n_g), 256>>>(oi, d, oo);
  trt_host::add_launches(1);
  rc = cudaGetLastError() == cudaSuccess ? TRT_OK : TRT_ERR_CUDA;
  for (int k = 0; k < 5 && !rc; ++k)
    if (cudaMemcpy(outs[k], dev[17 + k], C * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) rc = TRT_ERR_CUDA;
  release();
  return rc;
}

}  // extern "C"
