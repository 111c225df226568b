// Host side of the device MGQD solve: trt_mloqd_fv and trt_old_mgqd_coefs (include/trt_sweep.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "trt_sweep.h"
#include "gqd_kernels.cuh"
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
  int solve(cudaStream_t s);    // MLOQD_FV: coefficients, Krylov solve, fluxes, residuals
  int krylov(cudaStream_t s);   // the solve of whatever system the coefficient planes hold
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

// MLOQD_FV on the device; inputs and the initial guess (K.x) already uploaded.
int Solver::solve(cudaStream_t s) {
  const dim3 gpos(pos_blocks(), d.ng);
  const int nblk = pos_blocks();
  coef_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, cf);
  MG_LAUNCHED();
  const int rc = krylov(s);
  if (rc) return rc;
  const Outputs out{Fx, Fy};
  flux_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, cf, K.x, out);
  MG_LAUNCHED();
  residual_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, K.x, out, rpart);
  MG_LAUNCHED();
  residual_finish_kernel<<<d.ng, 32, 0, s>>>(rpart, nblk, d.ng, res, bcres);
  MG_LAUNCHED();
  return TRT_OK;
}

// Right-preconditioned BiCGSTAB over all groups of the system in cf (coefficients, edge diagonals and
// right-hand side set), from the initial guess in K.x.
int Solver::krylov(cudaStream_t s) {
  const int ng = d.ng;
  const dim3 gpos(pos_blocks(), ng);
  const int nblk = pos_blocks();
  matvec_timed = false;
  K.tol = g_settings.tol;
  K.maxit = g_settings.maxit;
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
  return TRT_OK;
}

struct Cache {
  std::mutex mu;
  std::unique_ptr<Solver> s;       // multigroup shape
  std::unique_ptr<Solver> grey;    // one-group shape of the grey Newton system
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

int get_solver(int nx, int ny, int ng, Solver** out, std::unique_ptr<Solver>& slot = g_cache.s) {
  Solver* s = slot.get();
  if (!s || s->d.nx != nx || s->d.ny != ny || s->d.ng != ng) {
    slot.reset();
    auto fresh = std::make_unique<Solver>();
    const int rc = fresh->init(nx, ny, ng);
    if (rc) return rc;
    slot = std::move(fresh);
  }
  *out = slot.get();
  return TRT_OK;
}

// One device allocation carved into 256-byte aligned pieces (the stateless grey entry points).
struct Arena {
  char* base = nullptr;
  size_t used = 0, cap = 0;
  ~Arena() {
    if (base) cudaFree(base);
  }
  int reserve(size_t bytes) {
    cap = bytes;
    if (cudaMalloc(&base, std::max<size_t>(bytes, 256)) != cudaSuccess) {
      cudaGetLastError();
      base = nullptr;
      return TRT_ERR_NOMEM;
    }
    return TRT_OK;
  }
  template <class T>
  T* take(size_t n) {
    const size_t b = (n * sizeof(T) + 255) & ~(size_t)255;
    T* p = reinterpret_cast<T*>(base + used);
    used += b;
    return p;
  }
  static size_t need(size_t n, size_t esz) { return (n * esz + 255) & ~(size_t)255; }
};

Dims dims_of(int nx, int ny, int ng) {
  Dims d{};
  d.nx = nx;
  d.ny = ny;
  d.ng = ng;
  d.nC = (long)nx * ny;
  d.nV = (long)(nx + 1) * ny;
  d.nH = (long)nx * (ny + 1);
  d.nU = d.nC + d.nV + d.nH;
  return d;
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

// ------------------------------------------------------------------------------------------------
// Grey low-order side
// ------------------------------------------------------------------------------------------------

namespace {

// Host arrays to device pieces of one arena, and device pieces back.
struct HostIn {
  const double* h;
  size_t n;
  const double** d;
};
struct HostOut {
  double* h;
  size_t n;
  double** d;
};
int stage(Arena& ar, std::initializer_list<HostIn> ins, std::initializer_list<HostOut> outs, size_t extra,
          cudaStream_t st) {
  size_t bytes = extra;
  for (const auto& u : ins) bytes += Arena::need(u.n, sizeof(double));
  for (const auto& u : outs) bytes += Arena::need(u.n, sizeof(double));
  int rc = ar.reserve(bytes);
  if (rc) return rc;
  for (const auto& u : ins) {
    double* p = ar.take<double>(u.n);
    *u.d = p;
    MG_CUDA(cudaMemcpyAsync(p, u.h, u.n * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  for (const auto& u : outs) *u.d = ar.take<double>(u.n);
  return TRT_OK;
}
int fetch(std::initializer_list<HostOut> outs, cudaStream_t st) {
  for (const auto& u : outs) MG_CUDA(cudaMemcpyAsync(u.h, *u.d, u.n * sizeof(double), cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

}  // namespace

extern "C" {

int trt_collapse_mg_ef(int n_x, int n_y, int n_g, const double* Eg_avg, const double* Eg_edgV, const double* Eg_edgH,
                       const double* Fxg_edgV, const double* Fyg_edgH, int Open_Threads, double* E_avg, double* E_edgV,
                       double* E_edgH, double* Fx_edgV, double* Fy_edgH) {
  (void)Open_Threads;
  if (n_x < 1 || n_y < 1 || n_g < 1 || !Eg_avg || !Eg_edgV || !Eg_edgH || !Fxg_edgV || !Fyg_edgH || !E_avg ||
      !E_edgV || !E_edgH || !Fx_edgV || !Fy_edgH)
    return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  const Dims d = dims_of(n_x, n_y, n_g);
  Arena ar;
  const double *a, *b, *c, *e, *f;
  double *o1, *o2, *o3, *o4, *o5;
  if ((rc = stage(ar, {{Eg_avg, (size_t)d.nC * n_g, &a}, {Eg_edgV, (size_t)d.nV * n_g, &b},
                       {Eg_edgH, (size_t)d.nH * n_g, &c}, {Fxg_edgV, (size_t)d.nV * n_g, &e},
                       {Fyg_edgH, (size_t)d.nH * n_g, &f}},
                  {{E_avg, (size_t)d.nC, &o1}, {E_edgV, (size_t)d.nV, &o2}, {E_edgH, (size_t)d.nH, &o3},
                   {Fx_edgV, (size_t)d.nV, &o4}, {Fy_edgH, (size_t)d.nH, &o5}},
                  0, nullptr)))
    return rc;
  trt_gqd::collapse_kernel<<<grid1(d.npos()), 256>>>(d, a, b, c, e, f, o1, o2, o3, o4, o5);
  MG_LAUNCHED();
  return fetch({{E_avg, (size_t)d.nC, &o1}, {E_edgV, (size_t)d.nV, &o2}, {E_edgH, (size_t)d.nH, &o3},
                {Fx_edgV, (size_t)d.nV, &o4}, {Fy_edgH, (size_t)d.nH, &o5}},
               nullptr);
}

int trt_cbar_calc(int n_x, int n_y, int n_g, double* Cb_L, double* Cb_B, double* Cb_R, double* Cb_T, const double* Cg_L,
                  const double* Cg_B, const double* Cg_R, const double* Cg_T, const double* Eg_avg,
                  const double* Eg_edgV, const double* Eg_edgH, const double* Eg_in_L, const double* Eg_in_B,
                  const double* Eg_in_R, const double* Eg_in_T) {
  (void)Eg_avg;
  if (n_x < 1 || n_y < 1 || n_g < 1 || !Cb_L || !Cb_B || !Cb_R || !Cb_T || !Cg_L || !Cg_B || !Cg_R || !Cg_T ||
      !Eg_edgV || !Eg_edgH || !Eg_in_L || !Eg_in_B || !Eg_in_R || !Eg_in_T)
    return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  const Dims d = dims_of(n_x, n_y, n_g);
  const size_t by = (size_t)n_y * n_g, bx = (size_t)n_x * n_g;
  Arena ar;
  trt_gqd::CbarArgs a{};
  if ((rc = stage(ar, {{Cg_L, by, &a.CgL}, {Cg_B, bx, &a.CgB}, {Cg_R, by, &a.CgR}, {Cg_T, bx, &a.CgT},
                       {Eg_edgV, (size_t)d.nV * n_g, &a.EgV}, {Eg_edgH, (size_t)d.nH * n_g, &a.EgH},
                       {Eg_in_L, by, &a.EinL}, {Eg_in_B, bx, &a.EinB}, {Eg_in_R, by, &a.EinR}, {Eg_in_T, bx, &a.EinT}},
                  {{Cb_L, (size_t)n_y, &a.CbL}, {Cb_B, (size_t)n_x, &a.CbB}, {Cb_R, (size_t)n_y, &a.CbR},
                   {Cb_T, (size_t)n_x, &a.CbT}},
                  0, nullptr)))
    return rc;
  trt_gqd::cbar_kernel<<<grid1(n_x + n_y), 256>>>(d, a);
  MG_LAUNCHED();
  return fetch({{Cb_L, (size_t)n_y, &a.CbL}, {Cb_B, (size_t)n_x, &a.CbB}, {Cb_R, (size_t)n_y, &a.CbR},
                {Cb_T, (size_t)n_x, &a.CbT}},
               nullptr);
}

int trt_old_grey_coefs(int n_x, int n_y, int n_g, double c, double Delt, double Theta, double cv, const double* A,
                       const double* Gold, const double* Temp_old, const double* KapE_bar_old, const double* E_avg_old,
                       const double* GQD_Src_old, double* Gold_Hat, double* Rhat_old) {
  if (n_x < 1 || n_y < 1 || n_g < 1 || !A || !Gold || !Temp_old || !KapE_bar_old || !E_avg_old || !GQD_Src_old ||
      !Gold_Hat || !Rhat_old || !(Theta != 0.0) || !(Delt > 0.0))
    return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  const Dims d = dims_of(n_x, n_y, n_g);
  const size_t C = (size_t)d.nC;
  Arena ar;
  const double *a, *g, *t, *k, *e, *q;
  double *gh, *rh;
  if ((rc = stage(ar, {{A, C, &a}, {Gold, C * n_g, &g}, {Temp_old, C, &t}, {KapE_bar_old, C, &k}, {E_avg_old, C, &e},
                       {GQD_Src_old, C, &q}},
                  {{Gold_Hat, C, &gh}, {Rhat_old, C, &rh}}, 0, nullptr)))
    return rc;
  trt_gqd::old_grey_kernel<<<grid1(d.nC), 256>>>(d, c, Delt, Theta, cv, a, g, t, k, e, q, gh, rh);
  MG_LAUNCHED();
  return fetch({{Gold_Hat, C, &gh}, {Rhat_old, C, &rh}}, nullptr);
}

int trt_grey_coefs(int n_x, int n_y, int n_g, const double* Eg_avg, const double* Eg_edgV, const double* Eg_edgH,
                   const double* Fxg_edgV_old, const double* Fyg_edgH_old, const double* fg_avg_xx,
                   const double* fg_avg_yy, const double* fg_edgV_xx, const double* fg_edgV_xy, const double* fg_edgH_yy,
                   const double* fg_edgH_xy, const double* KapE, const double* KapR, const double* A, double c,
                   double Delt, double Theta, const double* Pold_L, const double* Pold_R, const double* Pold_B,
                   const double* Pold_T, double* KapE_Bar, double* DC_xx, double* DL_xx, double* DR_xx, double* DC_yy,
                   double* DB_yy, double* DT_yy, double* DL_xy, double* DR_xy, double* DB_xy, double* DT_xy,
                   double* PL, double* PR, double* PB, double* PT, double Fdt_Weight) {
  const double* ins[] = {Eg_avg, Eg_edgV, Eg_edgH, Fxg_edgV_old, Fyg_edgH_old, fg_avg_xx, fg_avg_yy, fg_edgV_xx,
                         fg_edgV_xy, fg_edgH_yy, fg_edgH_xy, KapE, KapR, A, Pold_L, Pold_R, Pold_B, Pold_T};
  double* outs[] = {KapE_Bar, DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy, DR_xy, DB_xy, DT_xy, PL, PR, PB, PT};
  if (n_x < 1 || n_y < 1 || n_g < 1 || !(Theta != 0.0) || !(Delt > 0.0) || !(c > 0.0)) return TRT_ERR_ARG;
  for (const double* p : ins)
    if (!p) return TRT_ERR_ARG;
  for (double* p : outs)
    if (!p) return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  const Dims d = dims_of(n_x, n_y, n_g);
  const size_t C = (size_t)d.nC * n_g, V = (size_t)d.nV * n_g, H = (size_t)d.nH * n_g, c1 = (size_t)d.nC;
  Arena ar;
  trt_gqd::GreyIn in{};
  trt_gqd::GreyOut o{};
  if ((rc = stage(ar, {{Eg_avg, C, &in.Eg}, {Eg_edgV, V, &in.EgV}, {Eg_edgH, H, &in.EgH}, {Fxg_edgV_old, V, &in.FxOld},
                       {Fyg_edgH_old, H, &in.FyOld}, {fg_avg_xx, C, &in.fxx}, {fg_avg_yy, C, &in.fyy},
                       {fg_edgV_xx, V, &in.fVxx}, {fg_edgV_xy, V, &in.fVxy}, {fg_edgH_yy, H, &in.fHyy},
                       {fg_edgH_xy, H, &in.fHxy}, {KapE, C, &in.KapE}, {KapR, C, &in.KapR}, {A, c1, &in.A},
                       {Pold_L, C, &in.PoldL}, {Pold_R, C, &in.PoldR}, {Pold_B, C, &in.PoldB}, {Pold_T, C, &in.PoldT}},
                  {{KapE_Bar, c1, &o.Kb}, {DC_xx, c1, &o.DCxx}, {DL_xx, c1, &o.DLxx}, {DR_xx, c1, &o.DRxx},
                   {DC_yy, c1, &o.DCyy}, {DB_yy, c1, &o.DByy}, {DT_yy, c1, &o.DTyy}, {DL_xy, c1, &o.DLxy},
                   {DR_xy, c1, &o.DRxy}, {DB_xy, c1, &o.DBxy}, {DT_xy, c1, &o.DTxy}, {PL, c1, &o.PL}, {PR, c1, &o.PR},
                   {PB, c1, &o.PB}, {PT, c1, &o.PT}},
                  0, nullptr)))
    return rc;
  in.c = c;
  in.Delt = Delt;
  in.Theta = Theta;
  in.Fdt = Fdt_Weight;
  trt_gqd::grey_coefs_kernel<<<grid1(d.nC), 256>>>(d, in, o);
  MG_LAUNCHED();
  return fetch({{KapE_Bar, c1, &o.Kb}, {DC_xx, c1, &o.DCxx}, {DL_xx, c1, &o.DLxx}, {DR_xx, c1, &o.DRxx},
                {DC_yy, c1, &o.DCyy}, {DB_yy, c1, &o.DByy}, {DT_yy, c1, &o.DTyy}, {DL_xy, c1, &o.DLxy},
                {DR_xy, c1, &o.DRxy}, {DB_xy, c1, &o.DBxy}, {DT_xy, c1, &o.DTxy}, {PL, c1, &o.PL}, {PR, c1, &o.PR},
                {PB, c1, &o.PB}, {PT, c1, &o.PT}},
               nullptr);
}

int trt_egp_fv_newt(int n_x, int n_y, double* E_avg, double* E_edgV, double* E_edgH, double* Temp, double* KapE_Bar,
                    double* Fx_edgV, double* Fy_edgH, double* Q_bar, double* KapE_Bar_dT, int* Its, double* Deltas,
                    double* dresiduals, const double* Temp_Mold, const double* KapE_bar_Mold, double Theta, double Delt,
                    const double* Delx, const double* Dely, const double* A, const double* Cb_L, const double* Cb_B,
                    const double* Cb_R, const double* Cb_T, const double* E_in_L, const double* E_in_B,
                    const double* E_in_R, const double* E_in_T, const double* F_in_L, const double* F_in_B,
                    const double* F_in_R, const double* F_in_T, const double* DC_xx, const double* DL_xx,
                    const double* DR_xx, const double* DC_yy, const double* DB_yy, const double* DT_yy,
                    const double* DL_xy, const double* DR_xy, const double* DB_xy, const double* DT_xy,
                    const double* PL, const double* PR, const double* PB, const double* PT, const double* Gold_Hat,
                    const double* Rhat_old, double Kap0, double cv, double Comp_Unit, double Chi, double line_src,
                    double E_Bound_Low, double T_Bound_Low, double Eps1, double Eps2, int Maxits, int MGQD_It,
                    int Use_Line_Search, int Use_Safety_Search, int Res_Calc, int kapE_dT_flag, int* GQD_Kits,
                    double Fin_Weight, double Ein_Weight) {
  const double* ins[] = {Temp_Mold, KapE_bar_Mold, Delx, Dely, A, Cb_L, Cb_B, Cb_R, Cb_T, E_in_L, E_in_B, E_in_R,
                         E_in_T, F_in_L, F_in_B, F_in_R, F_in_T, DC_xx, DL_xx, DR_xx, DC_yy, DB_yy, DT_yy, DL_xy,
                         DR_xy, DB_xy, DT_xy, PL, PR, PB, PT, Gold_Hat, Rhat_old};
  double* io[] = {E_avg, E_edgV, E_edgH, Temp, KapE_Bar, Fx_edgV, Fy_edgH, Q_bar, KapE_Bar_dT};
  if (n_x < 1 || n_y < 1 || Maxits < 1 || !Its || !GQD_Kits || (Res_Calc && (!Deltas || !dresiduals)) ||
      !(Theta != 0.0) || !(Delt > 0.0) || !(Comp_Unit > 0.0) || (Use_Line_Search && !(line_src > 1.0)) ||
      (Use_Safety_Search && !(line_src > 1.0)))
    return TRT_ERR_ARG;
  for (const double* p : ins)
    if (!p) return TRT_ERR_ARG;
  for (double* p : io)
    if (!p) return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_cache.mu);
  Solver* G = nullptr;
  if ((rc = get_solver(n_x, n_y, 1, &G, g_cache.grey))) return rc;
  const Dims d = G->d;
  cudaStream_t st = G->st;
  const size_t C = (size_t)d.nC, V = (size_t)d.nV, H = (size_t)d.nH;
  const int nblk = G->pos_blocks();
  trt_gqd::Egp e{};
  e.nx = n_x;
  e.ny = n_y;
  Arena ar;
  const double *cE, *cEV, *cEH, *cT, *cKb, *cFx, *cFy;
  const size_t extra = Arena::need(C, 8) * 2 + Arena::need(C, 8) * 5 + Arena::need(V, 8) + Arena::need(H, 8) +
                       Arena::need((size_t)nblk * 6, 8) + Arena::need(8, 8) + Arena::need(18, 8) + 256;
  if ((rc = stage(ar,
                  {{E_avg, C, &cE}, {E_edgV, V, &cEV}, {E_edgH, H, &cEH}, {Temp, C, &cT}, {KapE_Bar, C, &cKb},
                   {Fx_edgV, V, &cFx}, {Fy_edgH, H, &cFy}, {Temp_Mold, C, &e.Tm}, {KapE_bar_Mold, C, &e.Kbm},
                   {Delx, (size_t)n_x, &e.Delx}, {Dely, (size_t)n_y, &e.Dely}, {A, C, &e.A}, {Cb_L, (size_t)n_y, &e.CbL},
                   {Cb_B, (size_t)n_x, &e.CbB}, {Cb_R, (size_t)n_y, &e.CbR}, {Cb_T, (size_t)n_x, &e.CbT},
                   {E_in_L, (size_t)n_y, &e.EinL}, {E_in_B, (size_t)n_x, &e.EinB}, {E_in_R, (size_t)n_y, &e.EinR},
                   {E_in_T, (size_t)n_x, &e.EinT}, {F_in_L, (size_t)n_y, &e.FinL}, {F_in_B, (size_t)n_x, &e.FinB},
                   {F_in_R, (size_t)n_y, &e.FinR}, {F_in_T, (size_t)n_x, &e.FinT}, {DC_xx, C, &e.DCxx},
                   {DL_xx, C, &e.DLxx}, {DR_xx, C, &e.DRxx}, {DC_yy, C, &e.DCyy}, {DB_yy, C, &e.DByy},
                   {DT_yy, C, &e.DTyy}, {DL_xy, C, &e.DLxy}, {DR_xy, C, &e.DRxy}, {DB_xy, C, &e.DBxy},
                   {DT_xy, C, &e.DTxy}, {PL, C, &e.PL}, {PR, C, &e.PR}, {PB, C, &e.PB}, {PT, C, &e.PT},
                   {Gold_Hat, C, &e.Gh}, {Rhat_old, C, &e.Rh}},
                  {}, extra, st)))
    return rc;
  e.E = const_cast<double*>(cE);
  e.EV = const_cast<double*>(cEV);
  e.EH = const_cast<double*>(cEH);
  e.T = const_cast<double*>(cT);
  e.Kb = const_cast<double*>(cKb);
  e.Fx = const_cast<double*>(cFx);
  e.Fy = const_cast<double*>(cFy);
  e.Q = ar.take<double>(C);
  e.Kdt = ar.take<double>(C);
  e.Korg = ar.take<double>(C);
  e.drT = ar.take<double>(C);
  e.W = ar.take<double>(C);
  e.dT = ar.take<double>(C);
  e.dFx = ar.take<double>(V);
  e.dFy = ar.take<double>(H);
  double* part = ar.take<double>((size_t)nblk * 6);
  double* norms = ar.take<double>(8);
  e.maxbuf = ar.take<unsigned long long>(18);
  e.kreq = ar.take<int>(8);
  if (ar.used > ar.cap + 256) return TRT_ERR_NOMEM;
  const double h = 6.62613e-19, c = 2.99792458e2, pi = 4.0 * std::atan(1.0), erg = 6.24150934e11;
  const double sig_R = 2.0 * std::pow(pi, 5) / (15.0 * (c * c) * (h * h * h) * std::pow(erg, 4) * Comp_Unit);
  e.aR = 4.0 * sig_R / c;
  e.Theta = Theta;
  e.Delt = Delt;
  e.Kap0 = Kap0;
  e.cv = cv;
  e.Chi = Chi;
  e.Fin = Fin_Weight;
  e.Ein = Ein_Weight;
  e.damp = (MGQD_It > 1 && kapE_dT_flag) ? 1 : 0;

  const int gp = G->pos_blocks();
  trt_gqd::egp_dtinit_kernel<<<grid1(d.nC), 256, 0, st>>>(e);
  MG_LAUNCHED();
  MG_CUDA(cudaMemsetAsync(G->K.x, 0, sizeof(double) * d.nU, st));   // Delta E of "iteration 0"
  double hbuf[18];
  double hn[8];
  double prev[6] = {0, 0, 0, 0, 0, 0};
  bool converged = false, noconv = false;
  int its = 0;
  while (!converged && its < Maxits) {
    its += 1;
    MG_CUDA(cudaMemsetAsync(e.maxbuf, 0, sizeof(unsigned long long) * 18, st));
    MG_CUDA(cudaMemsetAsync(e.kreq, 0, sizeof(int), st));
    trt_gqd::egp_coef_kernel<<<gp, kRedBlock, 0, st>>>(e, d, G->cf);
    MG_LAUNCHED();
    if ((rc = G->krylov(st))) return rc;
    trt_gqd::egp_delta_kernel<<<gp, kRedBlock, 0, st>>>(e, d, G->K.x, part);
    MG_LAUNCHED();
    trt_gqd::egp_norm_finish_kernel<<<1, 32, 0, st>>>(part, nblk, norms);
    MG_LAUNCHED();
    MG_CUDA(cudaMemcpyAsync(hn, norms, sizeof(double) * 6, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaMemcpyAsync(G->h_scal, G->K.sc, sizeof(Scal), cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    GQD_Kits[its - 1] = (G->h_scal[0].done == 1 ? 1 : -1) * (1 + 2 * G->h_scal[0].its);
    if (G->h_scal[0].done != 1) noconv = true;
    // line search (GLOQD_SOLVES.f08:604-636): the six quantities in order, each on the deltas as the
    // earlier ones left them; the deltas are scaled uniformly, so one cumulative factor carries it
    double S = 1.0;
    double nrm[6];
    for (int q = 0; q < 6; ++q) nrm[q] = std::sqrt(hn[q]);
    if (Use_Line_Search && its > 1) {
      for (int q = 0; q < 6; ++q) {
        double LS = 1.0;
        for (int k = 0; k < 10; ++k) {
          if (nrm[q] / S / LS > prev[q]) LS = LS * line_src;
          else break;
        }
        if (LS > 1.0) S = S * LS;
      }
    }
    if (Use_Safety_Search) {
      trt_gqd::egp_safety_kernel<<<gp, kRedBlock, 0, st>>>(e, d, G->K.x, S, line_src, T_Bound_Low, E_Bound_Low);
      MG_LAUNCHED();
      int kq = 0;
      MG_CUDA(cudaMemcpyAsync(&kq, e.kreq, sizeof(int), cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaStreamSynchronize(st));
      for (int k = 0; k < kq; ++k) S = S * line_src;
    }
    trt_gqd::egp_update_kernel<<<gp, kRedBlock, 0, st>>>(e, d, G->K.x, S);
    MG_LAUNCHED();
    MG_CUDA(cudaMemcpyAsync(hbuf, e.maxbuf, sizeof(double) * 18, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < 6; ++q) prev[q] = nrm[q] / S;
    converged = true;
    for (int q = 0; q < 6; ++q)
      if (hbuf[6 + q] > Eps1 * hbuf[12 + q] + Eps2) converged = false;
    if (Res_Calc)
      for (int q = 0; q < 6; ++q) {
        Deltas[(its - 1) + (long)Maxits * q] = hbuf[6 + q];
        dresiduals[(its - 1) + (long)Maxits * q] = hbuf[q];
      }
  }
  *Its = its;
  if ((rc = fetch({{E_avg, C, &e.E}, {E_edgV, V, &e.EV}, {E_edgH, H, &e.EH}, {Temp, C, &e.T}, {KapE_Bar, C, &e.Kb},
                   {Fx_edgV, V, &e.Fx}, {Fy_edgH, H, &e.Fy}, {Q_bar, C, &e.Q}, {KapE_Bar_dT, C, &e.Kdt}},
                  st)))
    return rc;
  return noconv ? TRT_ERR_NOCONV : TRT_OK;
}

}  // extern "C"

