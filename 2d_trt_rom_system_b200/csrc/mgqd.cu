// Host side of the device MGQD solve: trt_mloqd_fv and trt_old_mgqd_coefs (include/trt_sweep.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "trt_sweep.h"
#include "gqd_kernels.cuh"
#include "handle_hooks.h"
#include "mgqd_kernels.cuh"

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
// ... or, when every level from the first of at most kSmallCellsSmem cells on fits in kSmemMax bytes of shared
// memory, in the one-CTA kernel that keeps them in shared memory (64^2 and below on the configurations' grids)
constexpr int kSmallCellsSmem = 4096;
constexpr size_t kSmemMax = 200 * 1024;
constexpr int kNu1 = 2, kNu2 = 2, kCoarseSweeps = 16;
constexpr int kCheckEvery = 4;      // iterations between host checks of the convergence flags

struct Settings {
  double tol = 1e-13;
  int maxit = 1000;
  bool graphs = true;   // replay BiCGSTAB iteration blocks as CUDA graphs
  bool fused = true;    // one tiled kernel per level and direction of the V-cycle (else one per half-sweep)
  bool smem_vcycle = true;    // levels of at most 64^2 cells in small_vcycle_smem_kernel where they fit
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
  int k0 = 0;                 // first level of the one-CTA kernel in use (kS or kG)
  int kS = 0, kG = 0;         // first level of small_vcycle_smem_kernel / of small_vcycle_kernel
  bool vsmem = false;         // the levels from k0 on run in small_vcycle_smem_kernel
  bool vsmem_ok = false;      // they fit in shared memory
  size_t vsmem_bytes = 0;
  double *Fx = nullptr, *Fy = nullptr, *rpart = nullptr, *res = nullptr, *bcres = nullptr;
  int* h_done = nullptr;
  Scal* h_scal = nullptr;
  float last_ms = 0.f, last_matvec_ms = 0.f;
  bool matvec_timed = false;
  bool time_matvec = true;          // time the first iteration's matrix-vector product (trt_mgqd_last_stats)
  bool use_graphs = true;           // replay iteration blocks as a CUDA graph
  bool use_fused = true;            // fused tiled level passes in the V-cycle
  bool g_fused = true, g_vsmem = true;   // the forms the recorded graph was made with
  bool update_test = false;         // SPARSKIT's solution-update stopping test (Krylov::update_test)
  cudaGraphExec_t gexec = nullptr;  // kCheckEvery iterations, recorded on first use
  int g_nodes = 0, g_maxit = -1, g_rel = -1;
  double g_tol = -1.0;
  int last_its = 0;

  ~Solver() {
    if (gexec) cudaGraphExecDestroy(gexec);
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
  int init(int nx, int ny, int ng, bool own_inputs = true);   // own_inputs: allocate the Inputs planes
  // MLOQD_FV: coefficients, Krylov solve, fluxes, and the residual norms when residuals is set (the reference
  // forms them under Res_Calc only, as diagnostics)
  int solve(cudaStream_t s, bool residuals = true);
  int krylov(cudaStream_t s);   // the solve of whatever system the coefficient planes hold
  int pos_blocks() const { return (int)((d.npos() + kRedBlock - 1) / kRedBlock); }
};

int Solver::init(int nx, int ny, int ng, bool own_inputs) {
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
  // inputs (a caller that points them at its own device fields skips them)
  if (own_inputs) {
    A(&in.fxx, C); A(&in.fyy, C); A(&in.fVxx, V); A(&in.fVxy, V); A(&in.fHyy, H); A(&in.fHxy, H);
    A(&in.CgL, (size_t)ny * ng); A(&in.CgB, (size_t)nx * ng); A(&in.CgR, (size_t)ny * ng); A(&in.CgT, (size_t)nx * ng);
    A(&in.EinL, (size_t)ny * ng); A(&in.EinB, (size_t)nx * ng); A(&in.EinR, (size_t)ny * ng); A(&in.EinT, (size_t)nx * ng);
    A(&in.FinL, (size_t)ny * ng); A(&in.FinB, (size_t)nx * ng); A(&in.FinR, (size_t)ny * ng); A(&in.FinT, (size_t)nx * ng);
    A(&in.Src, C); A(&in.KapE, C); A(&in.KapR, C); A(&in.Delx, nx); A(&in.Dely, ny); A(&in.A, d.nC);
    A(&in.Gold, C); A(&in.PoldL, C); A(&in.PoldB, C); A(&in.PoldR, C); A(&in.PoldT, C);
    A(&in.Eold, C); A(&in.Fxold, V); A(&in.Fyold, H);
  }
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
  M(&K.part, (size_t)ng * nblk * 5);
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
    M(&L.xd, (size_t)L.n * ng);
    if (rc) return rc;
    if (mx <= 2 && my <= 2) break;
    mx = (mx + 1) / 2;
    my = (my + 1) / 2;
  }
  kS = 0;
  while (ls.L[kS].n > kSmallCellsSmem) ++kS;
  kG = 0;
  while (ls.L[kG].n > kSmallCells) ++kG;
  vsmem_bytes = small_vcycle_smem_bytes(ls, kS);
  vsmem_ok = vsmem_bytes <= kSmemMax &&
          cudaFuncSetAttribute(small_vcycle_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kSmemMax) == cudaSuccess;   // one bound for every solver's launches
  if (!vsmem_ok) cudaGetLastError();
  vsmem = vsmem_ok;
  k0 = vsmem ? kS : kG;
  MG_CUDA(cudaMallocHost(&h_done, sizeof(int) * ng));
  MG_CUDA(cudaMallocHost(&h_scal, sizeof(Scal) * ng));
  return TRT_OK;
}

int grid1(long n) { return (int)((n + 255) / 256); }

// MLOQD_FV on the device; inputs and the initial guess (K.x) already uploaded.
int Solver::solve(cudaStream_t s, bool residuals) {
  const dim3 gpos(pos_blocks(), d.ng);
  const int nblk = pos_blocks();
  coef_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, cf);
  MG_LAUNCHED();
  const int rc = krylov(s);
  if (rc) return rc;
  const Outputs out{Fx, Fy};
  flux_kernel<<<gpos, kRedBlock, 0, s>>>(in, d, cf, K.x, out);
  MG_LAUNCHED();
  if (!residuals) return TRT_OK;
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
  K.update_test = update_test ? 1 : 0;
  K.atol = 1e-15;   // fpar(2) of QD_SOLVERS.f08:445
  use_graphs = g_settings.graphs;
  use_fused = g_settings.fused;
  vsmem = vsmem_ok && g_settings.smem_vcycle;
  k0 = vsmem ? kS : kG;
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

  // Launch bookkeeping: a direct launch is counted at once; a launch recorded into the iteration graph is
  // counted each time the graph is replayed.
  int recorded = 0;
  bool capturing = false;
  auto launched = [&]() -> int {
    if (capturing) ++recorded;
    else trt_host::add_launches(1);
    MG_CUDA(cudaGetLastError());
    return TRT_OK;
  };
  static_assert(2 * kNu1 <= kTH && 2 * kNu2 <= kTH, "the tile halo covers the level's half-sweeps");
  auto vcycle = [&]() -> int {
    int rc;
    for (int k = 0; k < k0; ++k) {
      const Level& L = ls.L[k];
      if (use_fused) {
        smooth_restrict_tile_kernel<<<dim3(level_tiles(L), ng), kTileThreads, 0, s>>>(L, ls.L[k + 1], K.done, kNu1);
        if ((rc = launched())) return rc;
        continue;
      }
      const dim3 gl(grid1(L.n), ng);
      for (int sw = 0; sw < kNu1; ++sw) {
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 0, sw == 0 ? 1 : 0);
        if ((rc = launched())) return rc;
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 1, 0);
        if ((rc = launched())) return rc;
      }
      restrict_kernel<<<dim3(grid1(ls.L[k + 1].n), ng), 256, 0, s>>>(L, ls.L[k + 1], K.done);
      if ((rc = launched())) return rc;
    }
    if (vsmem)
      small_vcycle_smem_kernel<<<ng, 1024, vsmem_bytes, s>>>(ls, k0, kNu1, kNu2, kCoarseSweeps, K.done);
    else
      small_vcycle_kernel<<<ng, 256, 0, s>>>(ls, k0, kNu1, kNu2, kCoarseSweeps, K.done);
    if ((rc = launched())) return rc;
    for (int k = k0 - 1; k >= 0; --k) {
      const Level& L = ls.L[k];
      if (use_fused) {
        prolong_smooth_tile_kernel<<<dim3(level_tiles(L), ng), kTileThreads, 0, s>>>(L, ls.L[k + 1], K.done, kNu2);
        if ((rc = launched())) return rc;
        continue;
      }
      const dim3 gl(grid1(L.n), ng);
      prolong_kernel<<<gl, 256, 0, s>>>(L, ls.L[k + 1], K.done);
      if ((rc = launched())) return rc;
      for (int sw = 0; sw < kNu2; ++sw) {
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 0, 0);
        if ((rc = launched())) return rc;
        smooth_kernel<<<gl, 256, 0, s>>>(L, K.done, 1, 0);
        if ((rc = launched())) return rc;
      }
    }
    return TRT_OK;
  };
  // One BiCGSTAB iteration; the p vectors alternate with the iteration's parity.  Groups that have
  // converged (or stopped) skip every kernel, so iterations run past the end leave the result unchanged.
  auto iteration = [&](int it, bool timed) -> int {
    int rc;
    double* pold = (it & 1) ? K.p1 : K.p0;
    double* pnew = (it & 1) ? K.p0 : K.p1;
    elim_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], pold, pnew, 0);
    if ((rc = launched())) return rc;
    if ((rc = vcycle())) return rc;
    backsub_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], pnew, K.ph);
    if ((rc = launched())) return rc;
    if (timed) MG_CUDA(cudaEventRecord(m0, s));
    matvec_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, K.ph, K.v, 0);
    if ((rc = launched())) return rc;
    if (timed) MG_CUDA(cudaEventRecord(m1, s));
    scalar_finish_kernel<<<ng, 32, 0, s>>>(K, nblk, 0);
    if ((rc = launched())) return rc;
    elim_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], nullptr, K.s, 1);
    if ((rc = launched())) return rc;
    if ((rc = vcycle())) return rc;
    backsub_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, ls.L[0], K.s, K.sh);
    if ((rc = launched())) return rc;
    matvec_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K, K.sh, K.t, 1);
    if ((rc = launched())) return rc;
    scalar_finish_kernel<<<ng, 32, 0, s>>>(K, nblk, 1);
    if ((rc = launched())) return rc;
    update_kernel<<<gpos, kRedBlock, 0, s>>>(cf, d, K);
    if ((rc = launched())) return rc;
    update_finish_kernel<<<ng, 32, 0, s>>>(K, nblk);
    return launched();
  };
  // kCheckEvery iterations (an even count, so the parity pattern repeats) recorded once as a CUDA graph and
  // replayed between the host's convergence checks: the same kernels in the same order, one launch.  The
  // kernels take the solver's fixed buffers and K by value, so the graph is recorded again only when the
  // tolerance or the iteration limit in K changes.
  auto block = [&]() -> int {
    if (!gexec || g_tol != K.tol || g_maxit != K.maxit || g_rel != K.update_test || g_fused != use_fused ||
        g_vsmem != vsmem) {
      if (gexec) {
        cudaGraphExecDestroy(gexec);
        gexec = nullptr;
      }
      cudaGraph_t g = nullptr;
      MG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      capturing = true;
      recorded = 0;
      int rc = TRT_OK;
      for (int k = 0; k < kCheckEvery && !rc; ++k) rc = iteration(k, false);
      capturing = false;
      const cudaError_t e = cudaStreamEndCapture(s, &g);
      if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc ? rc : TRT_ERR_CUDA;
      }
      const cudaError_t ei = cudaGraphInstantiate(&gexec, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) {
        gexec = nullptr;
        cudaGetLastError();
        return TRT_ERR_CUDA;
      }
      g_nodes = recorded;
      g_tol = K.tol;
      g_maxit = K.maxit;
      g_rel = K.update_test;
      g_fused = use_fused;
      g_vsmem = vsmem;
    }
    MG_CUDA(cudaGraphLaunch(gexec, s));
    trt_host::add_launches((unsigned long long)g_nodes);
    return TRT_OK;
  };

  static_assert(kCheckEvery % 2 == 0, "graph blocks must keep the parity of the p vectors");
  int rc;
  for (int it = 0; it < K.maxit; ++it) {
    if (it % kCheckEvery == 0) {
      MG_CUDA(cudaMemcpyAsync(h_done, K.done, sizeof(int) * ng, cudaMemcpyDeviceToHost, s));
      MG_CUDA(cudaStreamSynchronize(s));
      bool all = true;
      for (int g = 0; g < ng; ++g) all = all && h_done[g] != 0;
      if (all) break;
      const bool timed_block = it == 0 && time_matvec;
      if (use_graphs && !timed_block && it + kCheckEvery <= K.maxit) {
        if ((rc = block())) return rc;
        it += kCheckEvery - 1;
        continue;
      }
    }
    if ((rc = iteration(it, it == 0 && time_matvec))) return rc;
    matvec_timed = matvec_timed || (it == 0 && time_matvec);
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

int trt_mgqd_set_graphs(int on) {
  std::lock_guard<std::mutex> lk(g_cache.mu);
  g_settings.graphs = on != 0;
  return TRT_OK;
}

int trt_mgqd_set_fused_levels(int on) {
  std::lock_guard<std::mutex> lk(g_cache.mu);
  g_settings.fused = on != 0;
  return TRT_OK;
}

int trt_mgqd_set_smem_vcycle(int on) {
  std::lock_guard<std::mutex> lk(g_cache.mu);
  g_settings.smem_vcycle = on != 0;
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
  if ((rc = S->solve(st, Res_Calc != 0))) return rc;
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

// Options of EGP_FV_NEWT's iteration (GLOQD_SOLVES.f08:305-309).
struct EgpOpts {
  double line_src, T_Bound_Low, E_Bound_Low, Eps1, Eps2;
  int Maxits, Use_Line_Search, Use_Safety_Search, Res_Calc;
};

// The Newton iterations of EGP_FV_NEWT (GLOQD_SOLVES.f08:393-860) on the device state of e, each linear
// solve by G's preconditioned BiCGSTAB (one system).  part: nblk*6 doubles, norms: 8 doubles (device).
// GQD_Kits gets the matrix-vector products of each iteration (negative where the solve did not
// converge); Deltas / dresiduals (Maxits, 6) when Res_Calc.
int egp_newton(Solver* G, cudaStream_t st, trt_gqd::Egp& e, const EgpOpts& o, double* part, double* norms,
               int* its_out, int* GQD_Kits, double* Deltas, double* dresiduals, bool* noconv_out) {
  const Dims d = G->d;
  const int nblk = G->pos_blocks();
  int rc;
  const int gp = G->pos_blocks();
  trt_gqd::egp_dtinit_kernel<<<grid1(d.nC), 256, 0, st>>>(e);
  MG_LAUNCHED();
  MG_CUDA(cudaMemsetAsync(G->K.x, 0, sizeof(double) * d.nU, st));   // Delta E of "iteration 0"
  double hbuf[18];
  double hn[8];
  double prev[6] = {0, 0, 0, 0, 0, 0};
  bool converged = false, noconv = false;
  int its = 0;
  while (!converged && its < o.Maxits) {
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
    if (o.Use_Line_Search && its > 1) {
      for (int q = 0; q < 6; ++q) {
        double LS = 1.0;
        for (int k = 0; k < 10; ++k) {
          if (nrm[q] / S / LS > prev[q]) LS = LS * o.line_src;
          else break;
        }
        if (LS > 1.0) S = S * LS;
      }
    }
    if (o.Use_Safety_Search) {
      trt_gqd::egp_safety_kernel<<<gp, kRedBlock, 0, st>>>(e, d, G->K.x, S, o.line_src, o.T_Bound_Low, o.E_Bound_Low);
      MG_LAUNCHED();
      int kq = 0;
      MG_CUDA(cudaMemcpyAsync(&kq, e.kreq, sizeof(int), cudaMemcpyDeviceToHost, st));
      MG_CUDA(cudaStreamSynchronize(st));
      for (int k = 0; k < kq; ++k) S = S * o.line_src;
    }
    trt_gqd::egp_update_kernel<<<gp, kRedBlock, 0, st>>>(e, d, G->K.x, S);
    MG_LAUNCHED();
    MG_CUDA(cudaMemcpyAsync(hbuf, e.maxbuf, sizeof(double) * 18, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < 6; ++q) prev[q] = nrm[q] / S;
    converged = true;
    for (int q = 0; q < 6; ++q)
      if (hbuf[6 + q] > o.Eps1 * hbuf[12 + q] + o.Eps2) converged = false;
    if (o.Res_Calc)
      for (int q = 0; q < 6; ++q) {
        Deltas[(its - 1) + (long)o.Maxits * q] = hbuf[6 + q];
        dresiduals[(its - 1) + (long)o.Maxits * q] = hbuf[q];
      }
  }
  *its_out = its;
  *noconv_out = noconv;
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
  trt_gqd::old_grey_kernel<<<grid1(d.nC), 256>>>(d, c, Delt, Theta, cv, a, g, t, k, e, q, gh, rh, nullptr);
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

  const EgpOpts opt{line_src, T_Bound_Low, E_Bound_Low, Eps1, Eps2, Maxits, Use_Line_Search, Use_Safety_Search,
                    Res_Calc};
  bool noconv = false;
  if ((rc = egp_newton(G, st, e, opt, part, norms, Its, GQD_Kits, Deltas, dresiduals, &noconv))) return rc;
  if ((rc = fetch({{E_avg, C, &e.E}, {E_edgV, V, &e.EV}, {E_edgH, H, &e.EH}, {Temp, C, &e.T}, {KapE_Bar, C, &e.Kb},
                   {Fx_edgV, V, &e.Fx}, {Fy_edgH, H, &e.Fy}, {Q_bar, C, &e.Q}, {KapE_Bar_dT, C, &e.Kdt}},
                  st)))
    return rc;
  return noconv ? TRT_ERR_NOCONV : TRT_OK;
}

}  // extern "C"


// ------------------------------------------------------------------------------------------------
// The mlqd time step on the device: TRT_MLQD_ALGORITHM with run_type 'mlqd', use_grey = 1, HO_Form 0,
// RT_start_Its 2 and Fdt/Fin/Ein weights 1 (MainSrc/ALGORITHMS.f08:294-302, 389-416, 518-572, 670-836).
// The handle supplies the sweep, the material and the temperature; everything else lives here.
// ------------------------------------------------------------------------------------------------

namespace {

struct Mlqd {
  trt_ctx* h = nullptr;
  trt_host::HandleView v{};
  trt_mlqd_params p{};
  Dims d{};
  std::unique_ptr<Solver> MG, GR;   // multigroup system (n_g groups) and the grey Newton system
  Arena ar;
  cudaEvent_t ev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  unsigned long long* h_conv = nullptr;   // pinned, 10 convergence values
  // multigroup fields, Fortran layouts.  The current solution lives in MG->K.x (unknown layout) and
  // MG->Fx / MG->Fy; Eg/EgV/EgH are its copies in the reference layout.
  double *Eg, *EgV, *EgH, *EgO, *EgVO, *EgHO, *FxO, *FyO, *fO[6], *KapO, *Src, *SrcO;
  double *Gold, *Pold[4];                               // G_old, Pold_L, Pold_B, Pold_R, Pold_T
  double *EinG[4], *FinG[4];                            // Eg_in_*, Fg_in_* (n_g per boundary point)
  // grey fields
  double *E, *EV, *EH, *Fx, *Fy, *MGE, *MGEV, *MGEH, *MGFx, *MGFy, *Eo;
  double *Kb, *KbO, *KbM, *Kdt, *Korg, *Q, *QO, *Gh, *Rh, *Dc[10], *Pc[4], *Cb[4], *Ein[4], *Fin[4];
  double *Tm1, *Tm2, *Em1, *Em2, *Tr1, *Tr2, *Er1, *Er2, *Told;
  double *drT, *W, *dT, *dFx, *dFy, *part, *norms;
  unsigned long long *maxbuf, *conv;
  int* kreq;
  const double* f[6];        // the handle's fg fields (avg_xx, avg_yy, edgV_xx, edgV_xy, edgH_yy, edgH_xy)
  const double* Cg[4];       // the handle's Cg fields
  const double* HOE;         // the handle's transport E_avg (the sum over this handle's groups)
  double* HOEt = nullptr;    // the transport E_avg summed over every group (= HOE when the handle holds them all)
  double* xbuf = nullptr;    // group sums of one exchange (trt_gqd::greyx_of), when the caller passes none
  int ng_total = 0, g_first = 0;   // the groups of the instance and the first one this handle holds
  std::vector<int> mg_counts, egp_counts, kits;
  // state of the step in progress (the phases below)
  trt_mlqd_stats S{};
  float sweep_ms = 0.f;
  bool swept = false;
  int mg_cur = 0, rt_cur = 0;
  double tn = 0.0, en = 0.0;

  ~Mlqd() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (h_conv) cudaFreeHost(h_conv);
  }
};

void mlqd_release(void* p) { delete static_cast<Mlqd*>(p); }

// Device copies of the time step run on the SMs: a device-to-device cudaMemcpy(2D)Async goes to a copy engine,
// which moves a few hundred GB/s and adds its own latency to each of the step's many small copies.
__global__ void copy_kernel(double* __restrict__ dst, const double* __restrict__ src, long n) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) dst[k] = src[k];
}

// The three fields of every group between the solver's unknown layout (one [E_avg | E_edgV | E_edgH] segment of
// nU values per group) and the reference layouts (group-major planes of nC, nV, nH values); to_fields picks the
// direction.
__global__ void unknowns_fields_kernel(const Dims d, double* __restrict__ x, double* __restrict__ Eg,
                                       double* __restrict__ EgV, double* __restrict__ EgH, int to_fields) {
  const int g = blockIdx.y;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < d.nU; k += (long)gridDim.x * blockDim.x) {
    double* f = k < d.nC ? Eg + d.nC * g + k
                         : (k < d.nC + d.nV ? EgV + d.nV * g + (k - d.nC) : EgH + d.nH * g + (k - d.nC - d.nV));
    double* u = x + d.nU * g + k;
    if (to_fields) *f = *u;
    else *u = *f;
  }
}

int copy_grid(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 8); }

int d2d(double* dst, const double* src, size_t n, cudaStream_t st) {
  if (n == 0) return TRT_OK;
  copy_kernel<<<copy_grid((long)n), 256, 0, st>>>(dst, src, (long)n);
  MG_LAUNCHED();
  return TRT_OK;
}

int h2d(double* dst, const std::vector<double>& src, cudaStream_t st) {
  MG_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  return TRT_OK;
}

// MLOQD_FV's solution in the unknown layout <-> the reference layouts (one strided copy per field).
int unknowns_fields(const Mlqd& m, cudaStream_t st, int to_fields) {
  const Dims& d = m.d;
  const int per_group = (int)std::max<long>(1, std::min<long>((d.nU + 255) / 256, (148L * 8 + d.ng - 1) / d.ng));
  unknowns_fields_kernel<<<dim3(per_group, d.ng), 256, 0, st>>>(d, m.MG->K.x, m.Eg, m.EgV, m.EgH, to_fields);
  MG_LAUNCHED();
  return TRT_OK;
}

int unknowns_to_fields(const Mlqd& m, cudaStream_t st) { return unknowns_fields(m, st, 1); }

int fields_to_unknowns(const Mlqd& m, cudaStream_t st) { return unknowns_fields(m, st, 0); }

// ng_total > 0: the handle holds groups g_first .. g_first + ng - 1 of an instance of ng_total groups whose
// group edges are nu_total (ng_total + 1 values); the initial grey fields and incoming energies are the sums
// over every group, the handle's own transport E the sum over its groups.
int mlqd_setup_impl(trt_ctx* h, double Tini, const trt_mlqd_params& prm, int ng_total, int g_first,
                    const double* nu_total) {
  auto m = std::make_unique<Mlqd>();
  int rc = trt_host::handle_view(h, &m->v);
  if (rc) return rc;
  const trt_host::HandleView& v = m->v;
  if (v.law != TRT_LAW_FLECK_CUMMINGS) return TRT_ERR_ARG;   // the grey emission below is the reference's
  m->h = h;
  m->p = prm;
  const int nx = v.nx, ny = v.ny, ng = v.ng;
  if (ng_total <= 0) {
    ng_total = ng;
    g_first = 0;
    nu_total = v.nu;
  }
  if (!nu_total || g_first < 0 || g_first + ng > ng_total) return TRT_ERR_ARG;
  for (int g = 0; g <= ng; ++g)
    if (nu_total[g_first + g] != v.nu[g]) return TRT_ERR_ARG;   // the handle's groups are that range
  m->ng_total = ng_total;
  m->g_first = g_first;
  m->d = dims_of(nx, ny, ng);
  const Dims& d = m->d;
  cudaStream_t st = v.stream;
  m->MG = std::make_unique<Solver>();
  if ((rc = m->MG->init(nx, ny, ng, false))) return rc;
  m->GR = std::make_unique<Solver>();
  if ((rc = m->GR->init(nx, ny, 1, false))) return rc;
  m->MG->time_matvec = false;   // every iteration block of the time loop's solves runs as a graph
  m->GR->time_matvec = false;
  m->GR->update_test = true;    // Newton corrections: the reference's stopping test (ipar(3) = -1)
  const size_t C = (size_t)d.nC * ng, V = (size_t)d.nV * ng, H = (size_t)d.nH * ng;
  const size_t c1 = d.nC, v1 = d.nV, hh1 = d.nH;
  const size_t side[4] = {(size_t)ny, (size_t)nx, (size_t)ny, (size_t)nx};   // L, B, R, T
  const int nblk = m->GR->pos_blocks();
  // one arena for every field: sizes in the order they are taken below
  std::vector<std::pair<double**, size_t>> plan = {
      {&m->Eg, C},    {&m->EgV, V},   {&m->EgH, H},   {&m->EgO, C},   {&m->EgVO, V},  {&m->EgHO, H},
      {&m->FxO, V},   {&m->FyO, H},   {&m->fO[0], C}, {&m->fO[1], C}, {&m->fO[2], V}, {&m->fO[3], V},
      {&m->fO[4], H}, {&m->fO[5], H}, {&m->KapO, C},  {&m->Src, C},   {&m->SrcO, C},  {&m->Gold, C},
      {&m->Pold[0], C}, {&m->Pold[1], C}, {&m->Pold[2], C}, {&m->Pold[3], C},
      {&m->E, c1},    {&m->EV, v1},   {&m->EH, hh1},  {&m->Fx, v1},   {&m->Fy, hh1},  {&m->MGE, c1},
      {&m->MGEV, v1}, {&m->MGEH, hh1}, {&m->MGFx, v1}, {&m->MGFy, hh1}, {&m->Eo, c1},  {&m->Kb, c1},
      {&m->KbO, c1},  {&m->KbM, c1},  {&m->Kdt, c1},  {&m->Korg, c1}, {&m->Q, c1},    {&m->QO, c1},
      {&m->Gh, c1},   {&m->Rh, c1},   {&m->Tm1, c1},  {&m->Tm2, c1},  {&m->Em1, c1},  {&m->Em2, c1},
      {&m->Tr1, c1},  {&m->Tr2, c1},  {&m->Er1, c1},  {&m->Er2, c1},  {&m->Told, c1}, {&m->drT, c1},
      {&m->W, c1},    {&m->dT, c1},   {&m->dFx, v1},  {&m->dFy, hh1}, {&m->part, (size_t)nblk * 6},
      {&m->norms, 8}, {&m->HOEt, c1}, {&m->xbuf, (size_t)trt_gqd::greyx_of(m->d).size}};
  for (int k = 0; k < 10; ++k) plan.push_back({&m->Dc[k], c1});
  for (int k = 0; k < 4; ++k) {
    plan.push_back({&m->Pc[k], c1});
    plan.push_back({&m->Cb[k], side[k]});
    plan.push_back({&m->Ein[k], side[k]});
    plan.push_back({&m->Fin[k], side[k]});
    plan.push_back({&m->EinG[k], side[k] * ng});
    plan.push_back({&m->FinG[k], side[k] * ng});
  }
  size_t bytes = Arena::need(18, 8) + Arena::need(8, 4) + Arena::need(10, 8);
  for (const auto& q : plan) bytes += Arena::need(q.second, sizeof(double));
  if ((rc = m->ar.reserve(bytes))) return rc;
  for (const auto& q : plan) *q.first = m->ar.take<double>(q.second);
  m->maxbuf = m->ar.take<unsigned long long>(18);
  m->kreq = m->ar.take<int>(8);
  m->conv = m->ar.take<unsigned long long>(10);
  for (cudaEvent_t& e : m->ev) MG_CUDA(cudaEventCreate(&e));
  MG_CUDA(cudaMallocHost(&m->h_conv, 10 * sizeof(unsigned long long)));
  static const char* fnames[6] = {"fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy"};
  static const char* cnames[4] = {"Cg_L", "Cg_B", "Cg_R", "Cg_T"};
  for (int k = 0; k < 6; ++k)
    if (!(m->f[k] = trt_device_output(h, fnames[k]))) return TRT_ERR_STATE;
  for (int k = 0; k < 4; ++k)
    if (!(m->Cg[k] = trt_device_output(h, cnames[k]))) return TRT_ERR_STATE;
  if (!(m->HOE = trt_device_output(h, "E_avg"))) return TRT_ERR_STATE;

  // --- initial state at Tini ---
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> eg_all(ng_total);
  for (int g = 0; g < ng_total; ++g)
    eg_all[g] = 4.0 * pi * trt_bg_planck(Tini, nu_total[g], nu_total[g + 1], v.comp_unit) / v.c;
  const std::vector<double> eg(eg_all.begin() + g_first, eg_all.begin() + g_first + ng);
  double Esum = 0.0;   // the group sum as MGQD_INIT / GQD_INIT / RT_INIT accumulate it
  for (int g = 0; g < ng_total; ++g) Esum = Esum + eg_all[g];
  double Esum_own = 0.0;   // over this handle's groups (= Esum when it holds them all)
  for (int g = 0; g < ng; ++g) Esum_own = Esum_own + eg[g];
  auto per_group = [&](size_t plane) {
    std::vector<double> x(plane * ng);
    for (int g = 0; g < ng; ++g) std::fill(x.begin() + plane * g, x.begin() + plane * (g + 1), eg[g]);
    return x;
  };
  if ((rc = h2d(m->Eg, per_group(d.nC), st)) || (rc = h2d(m->EgV, per_group(d.nV), st)) ||
      (rc = h2d(m->EgH, per_group(d.nH), st)))
    return rc;
  if ((rc = fields_to_unknowns(*m, st))) return rc;
  MG_CUDA(cudaMemsetAsync(m->MG->Fx, 0, V * sizeof(double), st));
  MG_CUDA(cudaMemsetAsync(m->MG->Fy, 0, H * sizeof(double), st));
  // QD factors of an isotropic field and the vacuum / reflective boundary factors (MGQD_INIT)
  const double third = 1.0 / 3.0;
  const size_t fsz[6] = {C, C, V, V, H, H};
  const double fval[6] = {third, third, third, 0.0, third, 0.0};
  for (int k = 0; k < 6; ++k)
    if ((rc = h2d(const_cast<double*>(m->f[k]), std::vector<double>(fsz[k], fval[k]), st))) return rc;
  const double cval[4] = {-0.5, -0.5, 0.5, 0.5};
  for (int k = 0; k < 4; ++k) {
    const double cv0 = v.bc[k] == 0 ? cval[k] : 0.0;
    if ((rc = h2d(const_cast<double*>(m->Cg[k]), std::vector<double>(side[k] * ng, cv0), st))) return rc;
    if ((rc = h2d(m->Cb[k], std::vector<double>(side[k], cv0), st))) return rc;
  }
  // transport E of RT_INIT: the handle's own groups, and all of them
  if ((rc = h2d(const_cast<double*>(m->HOE), std::vector<double>(c1, Esum_own), st)) ||
      (rc = h2d(m->HOEt, std::vector<double>(c1, Esum), st)))
    return rc;
  // grey E, F of GQD_INIT
  if ((rc = h2d(m->E, std::vector<double>(c1, Esum), st)) || (rc = h2d(m->EV, std::vector<double>(v1, Esum), st)) ||
      (rc = h2d(m->EH, std::vector<double>(hh1, Esum), st)))
    return rc;
  MG_CUDA(cudaMemsetAsync(m->Fx, 0, v1 * sizeof(double), st));
  MG_CUDA(cudaMemsetAsync(m->Fy, 0, hh1 * sizeof(double), st));
  for (double* z : {m->Kb, m->Q, m->Kdt})
    MG_CUDA(cudaMemsetAsync(z, 0, c1 * sizeof(double), st));
  // MGQD_In_Calc (MLOQD_SOLVES.f08:493-614) on the inflow faces that RT_INIT's RT_BC_UPDATE leaves at
  // Bg(bcT of the side); reflective sides have none.  These faces keep those values at every later
  // RT_BC_UPDATE, so the incoming E and F never change.  GQD_In_Calc (GLOQD_SOLVES.f08:263-290) sums
  // them over groups.
  const int nm = v.nm;
  const int range[4][4] = {{0, nm / 4, 3 * nm / 4, nm},   // L: Omega_x > 0
                           {0, nm / 2, 0, 0},             // B: Omega_y > 0
                           {nm / 4, 3 * nm / 4, 0, 0},    // R: Omega_x < 0
                           {nm / 2, nm, 0, 0}};           // T: Omega_y < 0
  for (int s = 0; s < 4; ++s) {
    // every group of the instance (the grey sums); the handle keeps its own range
    std::vector<double> Eg_in(side[s] * ng_total, 0.0), Fg_in(side[s] * ng_total, 0.0), E_in(side[s], 0.0),
        F_in(side[s], 0.0);
    for (int g = 0; g < ng_total; ++g) {
      const double I = v.bc[s] == 0 ? trt_bg_planck(v.Tb[s], nu_total[g], nu_total[g + 1], v.comp_unit) : 0.0;
      for (size_t i = 0; i < side[s] && v.bc[s] == 0; ++i) {
        double e = 0.0, f = 0.0;
        for (int r = 0; r < 2; ++r)
          for (int mm = range[s][2 * r]; mm < range[s][2 * r + 1]; ++mm) {
            const double om = (s == 0 || s == 2) ? v.omx[mm] : v.omy[mm];
            f = f + om * v.w[mm] * I;
            e = e + v.w[mm] * I;
          }
        Fg_in[i + side[s] * g] = f;
        Eg_in[i + side[s] * g] = e / v.c;
      }
    }
    for (size_t i = 0; i < side[s]; ++i)
      for (int g = 0; g < ng_total; ++g) {
        E_in[i] = E_in[i] + Eg_in[i + side[s] * g];
        F_in[i] = F_in[i] + Fg_in[i + side[s] * g];
      }
    const std::vector<double> own_E(Eg_in.begin() + side[s] * g_first, Eg_in.begin() + side[s] * (g_first + ng));
    const std::vector<double> own_F(Fg_in.begin() + side[s] * g_first, Fg_in.begin() + side[s] * (g_first + ng));
    if ((rc = h2d(m->EinG[s], own_E, st)) || (rc = h2d(m->FinG[s], own_F, st)) || (rc = h2d(m->Ein[s], E_in, st)) ||
        (rc = h2d(m->Fin[s], F_in, st)))
      return rc;
  }
  // the material of TEMP_INIT with the low-order source
  if ((rc = trt_host::handle_material(h, m->Src))) return rc;
  // MLOQD_FV's inputs point at the live fields
  Inputs& in = m->MG->in;
  in.fxx = m->f[0]; in.fyy = m->f[1]; in.fVxx = m->f[2]; in.fVxy = m->f[3]; in.fHyy = m->f[4]; in.fHxy = m->f[5];
  in.CgL = m->Cg[0]; in.CgB = m->Cg[1]; in.CgR = m->Cg[2]; in.CgT = m->Cg[3];
  in.EinL = m->EinG[0]; in.EinB = m->EinG[1]; in.EinR = m->EinG[2]; in.EinT = m->EinG[3];
  in.FinL = m->FinG[0]; in.FinB = m->FinG[1]; in.FinR = m->FinG[2]; in.FinT = m->FinG[3];
  in.Src = m->Src; in.KapE = v.kap64; in.KapR = v.kap64; in.Delx = v.dx; in.Dely = v.dy; in.A = v.area;
  in.Gold = m->Gold; in.PoldL = m->Pold[0]; in.PoldB = m->Pold[1]; in.PoldR = m->Pold[2]; in.PoldT = m->Pold[3];
  in.Eold = m->EgO; in.Fxold = m->FxO; in.Fyold = m->FyO;
  in.c = v.c; in.Delt = v.dt; in.Theta = prm.theta; in.Fdt = 1.0; in.Fin = 1.0; in.Ein = 1.0;
  MG_CUDA(cudaStreamSynchronize(st));
  trt_host::handle_attach(h, m.release(), mlqd_release);
  return TRT_OK;
}

// Convergence data of (x vs xo, xo2) and (y vs yo, yo2) to the host; CONVERGENCE of both.
int conv_pair(Mlqd& m, const double* x, const double* xo, const double* xo2, const double* y, const double* yo,
              const double* yo2, double eps, int its, double* xn, double* yn, bool* both) {
  const long long n = m.d.nC;
  int rc;
  if ((rc = trt_host::handle_conv_reduce(m.h, n, x, xo, xo2, m.conv))) return rc;
  if ((rc = trt_host::handle_conv_reduce(m.h, n, y, yo, yo2, m.conv + 5))) return rc;
  MG_CUDA(cudaMemcpyAsync(m.h_conv, m.conv, 10 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, m.v.stream));
  MG_CUDA(cudaStreamSynchronize(m.v.stream));
  double r[10];
  std::memcpy(r, m.h_conv, sizeof(r));
  const bool a = trt_host::handle_convergence(m.v.conv_type, eps, r, its, xn);
  const bool b = trt_host::handle_convergence(m.v.conv_type, eps, r + 5, its, yn);
  *both = a && b;
  return TRT_OK;
}

// ---- the mlqd time step in phases -------------------------------------------------------------------
// A step is: step_begin / step_begin_finish; per outer iteration outer_begin / outer_begin_finish, the MGQD
// iterations (mgqd_local / mgqd_finish) and outer_end; step_end.  Each *_begin / *_local phase writes the
// group sums this handle contributes into `part` (a device buffer of greyx_of(d).size doubles), and the next
// phase reads the sums over every group's handle from `tot`: with one handle holding every group the two are
// the same buffer (trt_mlqd_step below); with the groups split over handles (ranks) the caller adds the
// partial buffers (one all-reduce) in between.  The exchanges are the sums behind OLD_GREY_COEFS, the
// transport E of the convergence test, and per MGQD iteration COLLAPSE_MG_EF, Cbar_Calc and GREY_COEFS; the
// grey Newton solve then runs on every handle with the same inputs (replicated), and each handle updates the
// material of its own groups.

trt_gqd::Egp egp_state(Mlqd& m) {
  const trt_host::HandleView& v = m.v;
  trt_gqd::Egp e{};
  e.nx = m.d.nx;
  e.ny = m.d.ny;
  e.E = m.E; e.EV = m.EV; e.EH = m.EH; e.T = v.T; e.Kb = m.Kb; e.Fx = m.Fx; e.Fy = m.Fy; e.Q = m.Q;
  e.Kdt = m.Kdt; e.Korg = m.Korg;
  e.Kbm = m.KbM; e.Delx = v.dx; e.Dely = v.dy; e.A = v.area;
  e.CbL = m.Cb[0]; e.CbB = m.Cb[1]; e.CbR = m.Cb[2]; e.CbT = m.Cb[3];
  e.EinL = m.Ein[0]; e.EinB = m.Ein[1]; e.EinR = m.Ein[2]; e.EinT = m.Ein[3];
  e.FinL = m.Fin[0]; e.FinB = m.Fin[1]; e.FinR = m.Fin[2]; e.FinT = m.Fin[3];
  e.DCxx = m.Dc[0]; e.DLxx = m.Dc[1]; e.DRxx = m.Dc[2]; e.DCyy = m.Dc[3]; e.DByy = m.Dc[4]; e.DTyy = m.Dc[5];
  e.DLxy = m.Dc[6]; e.DRxy = m.Dc[7]; e.DBxy = m.Dc[8]; e.DTxy = m.Dc[9];
  e.PL = m.Pc[0]; e.PR = m.Pc[1]; e.PB = m.Pc[2]; e.PT = m.Pc[3];
  e.Gh = m.Gh; e.Rh = m.Rh;
  e.drT = m.drT; e.W = m.W; e.dT = m.dT; e.dFx = m.dFx; e.dFy = m.dFy; e.maxbuf = m.maxbuf; e.kreq = m.kreq;
  {
    const double hP = 6.62613e-19, cL = 2.99792458e2, pi = 4.0 * std::atan(1.0), erg = 6.24150934e11;
    const double sig_R = 2.0 * std::pow(pi, 5) / (15.0 * (cL * cL) * (hP * hP * hP) * std::pow(erg, 4) * v.comp_unit);
    e.aR = 4.0 * sig_R / cL;
  }
  e.Theta = m.p.theta; e.Delt = v.dt; e.Kap0 = v.Kap0; e.cv = 0.0; e.cvc = v.cv; e.Chi = m.p.chi;
  e.Fin = 1.0; e.Ein = 1.0;
  return e;
}

// The last time step's data -> _old (ALGORITHMS.f08:395-413), OLD_MGQD_COEFS; part[0, nC) = the group sum of
// G_old over this handle's groups (OLD_GREY_COEFS).
int ph_step_begin(Mlqd& m, double* part) {
  const trt_host::HandleView& v = m.v;
  const Dims& d = m.d;
  const int ng = d.ng;
  cudaStream_t st = v.stream;
  const size_t C = (size_t)d.nC * ng, V = (size_t)d.nV * ng, H = (size_t)d.nH * ng;
  const size_t c1 = d.nC;
  int rc;
  m.S = trt_mlqd_stats{};
  m.sweep_ms = 0.f;
  m.rt_cur = m.mg_cur = 0;
  m.tn = m.en = 0.0;
  m.mg_counts.clear();
  m.egp_counts.clear();
  m.kits.assign((size_t)std::max(m.p.maxit_gloqd, 1), 0);
  MG_CUDA(cudaEventRecord(m.ev[0], st));
  const size_t fsz[6] = {C, C, V, V, H, H};
  if ((rc = d2d(m.Told, v.T, c1, st)) || (rc = d2d(m.EgO, m.Eg, C, st)) || (rc = d2d(m.EgVO, m.EgV, V, st)) ||
      (rc = d2d(m.EgHO, m.EgH, H, st)) || (rc = d2d(m.FxO, m.MG->Fx, V, st)) || (rc = d2d(m.FyO, m.MG->Fy, H, st)) ||
      (rc = d2d(m.KapO, v.kap64, C, st)) || (rc = d2d(m.SrcO, m.Src, C, st)) || (rc = d2d(m.Eo, m.E, c1, st)) ||
      (rc = d2d(m.KbO, m.Kb, c1, st)) || (rc = d2d(m.QO, m.Q, c1, st)))
    return rc;
  for (int k = 0; k < 6; ++k)
    if ((rc = d2d(m.fO[k], m.f[k], fsz[k], st))) return rc;
  // OLD_MGQD_COEFS (KapR_old = KapE_old: MATERIAL_UPDATE sets both to KapB)
  const OldIn oi{m.EgO, m.EgVO, m.EgHO, m.FxO, m.FyO, m.fO[0], m.fO[1], m.fO[2], m.fO[3], m.fO[4], m.fO[5],
                 m.KapO, m.KapO, m.SrcO, v.dx, v.dy, v.area, v.c, m.p.theta};
  const OldOut oo{m.Gold, m.Pold[0], m.Pold[1], m.Pold[2], m.Pold[3]};
  old_coefs_kernel<<<dim3(grid1(d.nC), ng), 256, 0, st>>>(oi, d, oo);
  MG_LAUNCHED();
  trt_gqd::gold_sum_kernel<<<grid1(d.nC), 256, 0, st>>>(d, m.Gold, part);
  MG_LAUNCHED();
  MG_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

// OLD_GREY_COEFS from the total group sum of G_old in tot[0, nC).
int ph_step_begin_finish(Mlqd& m, const double* tot) {
  const trt_host::HandleView& v = m.v;
  const Dims& d = m.d;
  cudaStream_t st = v.stream;
  trt_gqd::old_grey_from_sum_kernel<<<grid1(d.nC), 256, 0, st>>>(d, v.c, v.dt, m.p.theta, 0.0, v.area, tot, m.Told,
                                                                 m.KbO, m.Eo, m.QO, m.Gh, m.Rh, v.cv);
  MG_LAUNCHED();
  for (double* z : {m.Tr1, m.Tr2, m.Er1, m.Er2}) MG_CUDA(cudaMemsetAsync(z, 0, d.nC * sizeof(double), st));
  return TRT_OK;
}

// Outer iteration rt: the sweep (from the second on, RT_start_Its = 2; none with ho_form 1); part[0, nC) = the
// transport E over this handle's groups.
int ph_outer_begin(Mlqd& m, int rt, double* part) {
  cudaStream_t st = m.v.stream;
  int rc;
  m.swept = false;
  m.rt_cur = rt;
  if (m.p.ho_form == 0 && rt >= 2) {
    MG_CUDA(cudaEventRecord(m.ev[2], st));
    if ((rc = trt_host::handle_outer_sweep(m.h, rt == 2))) return rc;
    MG_CUDA(cudaEventRecord(m.ev[3], st));
    ++m.S.sweeps;
    m.swept = true;
  }
  if ((rc = d2d(part, m.HOE, m.d.nC, st))) return rc;
  MG_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

// The transport E over every group; the MGQD iterations start (:675-810).
int ph_outer_begin_finish(Mlqd& m, const double* tot) {
  cudaStream_t st = m.v.stream;
  const size_t c1 = m.d.nC;
  int rc;
  if ((rc = d2d(m.HOEt, tot, c1, st)) || (rc = d2d(m.Em1, m.HOEt, c1, st)) || (rc = d2d(m.Tm1, m.v.T, c1, st)))
    return rc;
  MG_CUDA(cudaMemsetAsync(m.Em2, 0, c1 * sizeof(double), st));
  MG_CUDA(cudaMemsetAsync(m.Tm2, 0, c1 * sizeof(double), st));
  m.mg_cur = 0;
  return TRT_OK;
}

// MGQD iteration, this handle's part: MLOQD_FV from the previous solution, and the group sums of
// COLLAPSE_MG_EF, Cbar_Calc and GREY_COEFS over its groups into part (greyx_of layout).
int ph_mgqd_local(Mlqd& m, double* part) {
  const trt_host::HandleView& v = m.v;
  const Dims& d = m.d;
  const int ng = d.ng;
  cudaStream_t st = v.stream;
  int rc;
  MG_CUDA(cudaEventRecord(m.ev[4], st));
  if ((rc = m.MG->solve(st, false))) return rc;   // the time step reports no MGQD residuals
  MG_CUDA(cudaEventRecord(m.ev[5], st));
  MG_CUDA(cudaMemcpyAsync(m.MG->h_scal, m.MG->K.sc, sizeof(Scal) * ng, cudaMemcpyDeviceToHost, st));
  if ((rc = unknowns_to_fields(m, st))) return rc;
  const trt_gqd::GreyX x = trt_gqd::greyx_of(d);
  trt_gqd::collapse_kernel<<<grid1(d.npos()), 256, 0, st>>>(d, m.Eg, m.EgV, m.EgH, m.MG->Fx, m.MG->Fy, part + x.E,
                                                            part + x.EV, part + x.EH, part + x.FV, part + x.FH);
  MG_LAUNCHED();
  const trt_gqd::CbarArgs ca{m.Cg[0], m.Cg[1], m.Cg[2], m.Cg[3], m.EgV, m.EgH, m.EinG[0], m.EinG[1], m.EinG[2],
                             m.EinG[3], m.Cb[0], m.Cb[1], m.Cb[2], m.Cb[3]};
  trt_gqd::cbar_partial_kernel<<<grid1(d.nx + d.ny), 256, 0, st>>>(d, ca, part + x.cbLR, part + x.cbBT);
  MG_LAUNCHED();
  trt_gqd::GreyIn gi{};
  gi.Eg = m.Eg; gi.EgV = m.EgV; gi.EgH = m.EgH; gi.FxOld = m.FxO; gi.FyOld = m.FyO;
  gi.fxx = m.f[0]; gi.fyy = m.f[1]; gi.fVxx = m.f[2]; gi.fVxy = m.f[3]; gi.fHyy = m.f[4]; gi.fHxy = m.f[5];
  gi.KapE = v.kap64; gi.KapR = v.kap64; gi.A = v.area;
  gi.PoldL = m.Pold[0]; gi.PoldR = m.Pold[2]; gi.PoldB = m.Pold[1]; gi.PoldT = m.Pold[3];
  gi.c = v.c; gi.Delt = v.dt; gi.Theta = m.p.theta; gi.Fdt = 1.0;
  trt_gqd::grey_partial_kernel<<<grid1(d.nC), 256, 0, st>>>(d, gi, part + x.grey);
  MG_LAUNCHED();
  MG_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

// MGQD iteration mg, from the sums over every group in tot: the grey fields, boundary factors and
// coefficients, EGP_FV_NEWT, MATERIAL_UPDATE of this handle's groups, CONVERGENCE(conv_lo) on T and the MGQD E.
int ph_mgqd_finish(Mlqd& m, int mg, const double* tot, bool* mg_conv) {
  const trt_host::HandleView& v = m.v;
  const Dims& d = m.d;
  const int ng = d.ng;
  cudaStream_t st = v.stream;
  const size_t c1 = d.nC, v1 = d.nV, hh1 = d.nH;
  int rc;
  m.mg_cur = mg;
  const trt_gqd::GreyX x = trt_gqd::greyx_of(d);
  if ((rc = d2d(m.MGE, tot + x.E, c1, st)) || (rc = d2d(m.MGEV, tot + x.EV, v1, st)) ||
      (rc = d2d(m.MGEH, tot + x.EH, hh1, st)) || (rc = d2d(m.MGFx, tot + x.FV, v1, st)) ||
      (rc = d2d(m.MGFy, tot + x.FH, hh1, st)))
    return rc;
  trt_gqd::cbar_finish_kernel<<<grid1(d.nx + d.ny), 256, 0, st>>>(d, tot + x.cbLR, tot + x.cbBT, m.Cb[0], m.Cb[1],
                                                                   m.Cb[2], m.Cb[3]);
  MG_LAUNCHED();
  if ((rc = d2d(m.KbM, m.Kb, c1, st))) return rc;   // KapE_bar_MGQDold = KapE_bar
  const trt_gqd::GreyOut go{m.Kb,    m.Dc[0], m.Dc[1], m.Dc[2], m.Dc[3], m.Dc[4], m.Dc[5], m.Dc[6],
                            m.Dc[7], m.Dc[8], m.Dc[9], m.Pc[0], m.Pc[1], m.Pc[2], m.Pc[3]};
  trt_gqd::grey_finish_kernel<<<grid1(d.nC), 256, 0, st>>>(d, tot + x.grey, m.MGE, m.MGEV, m.MGEH, go);
  MG_LAUNCHED();
  if ((rc = d2d(m.E, m.MGE, c1, st)) || (rc = d2d(m.EV, m.MGEV, v1, st)) || (rc = d2d(m.EH, m.MGEH, hh1, st)) ||
      (rc = d2d(m.Fx, m.MGFx, v1, st)) || (rc = d2d(m.Fy, m.MGFy, hh1, st)))
    return rc;
  trt_gqd::Egp e = egp_state(m);
  e.Tm = m.Tm2;   // Temp_MGQDold2
  e.damp = (mg > 1 && m.p.kapE_dT_flag) ? 1 : 0;
  const EgpOpts eo{m.p.line_src, m.p.T_bound_low, m.p.E_bound_low, m.p.conv_gr1, m.p.conv_gr2, m.p.maxit_gloqd,
                   m.p.use_line_search, m.p.use_safety_search, 0};
  int its = 0;
  bool noconv = false;
  MG_CUDA(cudaEventRecord(m.ev[6], st));
  if ((rc = egp_newton(m.GR.get(), st, e, eo, m.part, m.norms, &its, m.kits.data(), nullptr, nullptr, &noconv)))
    return rc;
  MG_CUDA(cudaEventRecord(m.ev[7], st));
  trt_mlqd_stats& S = m.S;
  int slowest = 0;
  for (int g = 0; g < ng; ++g) {   // h_scal was read before the Newton iteration's synchronisations
    if (m.MG->h_scal[g].done != 1) ++S.mgqd_nonconv;
    slowest = std::max(slowest, m.MG->h_scal[g].its);
  }
  S.mgqd_krylov_max = std::max(S.mgqd_krylov_max, slowest);
  S.mgqd_krylov_sum += slowest;
  for (int k = 0; k < its; ++k) {
    if (m.kits[k] < 0) ++S.egp_nonconv;
    const int ki = (std::abs(m.kits[k]) - 1) / 2;
    S.egp_krylov_max = std::max(S.egp_krylov_max, ki);
    S.egp_krylov_sum += ki;
  }
  m.egp_counts.push_back(its);
  S.egp_its += its;
  if ((rc = trt_host::handle_material(m.h, m.Src))) return rc;   // MATERIAL_UPDATE(Temp)
  double a = 0.0, b = 0.0;
  if ((rc = conv_pair(m, v.T, m.Tm1, m.Tm2, m.MGE, m.Em1, m.Em2, m.p.conv_lo, mg, &a, &b, mg_conv))) return rc;
  {   // the stream has synchronised: both intervals are complete
    float t1 = 0.f, t2 = 0.f;
    MG_CUDA(cudaEventElapsedTime(&t1, m.ev[4], m.ev[5]));
    MG_CUDA(cudaEventElapsedTime(&t2, m.ev[6], m.ev[7]));
    S.mgqd_solve_ms += t1;
    S.egp_ms += t2;
  }
  std::swap(m.Em1, m.Em2);
  std::swap(m.Tm1, m.Tm2);
  if ((rc = d2d(m.Em1, m.MGE, c1, st)) || (rc = d2d(m.Tm1, v.T, c1, st))) return rc;
  return TRT_OK;
}

// End of outer iteration rt: CONVERGENCE(conv_ho) on T and the transport E (over every group).
int ph_outer_end(Mlqd& m, int rt, bool* rt_conv) {
  const trt_host::HandleView& v = m.v;
  cudaStream_t st = v.stream;
  const size_t c1 = m.d.nC;
  int rc;
  m.mg_counts.push_back(m.mg_cur);
  m.S.mgqd_its += m.mg_cur;
  if (m.swept) {
    float ms = 0.f;
    MG_CUDA(cudaEventSynchronize(m.ev[3]));
    MG_CUDA(cudaEventElapsedTime(&ms, m.ev[2], m.ev[3]));
    m.sweep_ms += ms;
  }
  if ((rc = conv_pair(m, v.T, m.Tr1, m.Tr2, m.HOEt, m.Er1, m.Er2, v.conv_ho, rt, &m.tn, &m.en, rt_conv))) return rc;
  std::swap(m.Er1, m.Er2);
  std::swap(m.Tr1, m.Tr2);
  if ((rc = d2d(m.Er1, m.HOEt, c1, st)) || (rc = d2d(m.Tr1, v.T, c1, st))) return rc;
  return TRT_OK;
}

int ph_step_end(Mlqd& m, trt_mlqd_stats* out) {
  cudaStream_t st = m.v.stream;
  int rc;
  MG_CUDA(cudaEventRecord(m.ev[1], st));
  if ((rc = trt_host::handle_check(m.h))) return rc;
  MG_CUDA(cudaEventSynchronize(m.ev[1]));
  float total = 0.f;
  MG_CUDA(cudaEventElapsedTime(&total, m.ev[0], m.ev[1]));
  m.S.rt_its = m.rt_cur;
  m.S.T_norm = m.tn;
  m.S.E_norm = m.en;
  m.S.sweep_ms = m.sweep_ms;
  m.S.low_order_ms = total - m.sweep_ms;
  if (out) *out = m.S;
  return TRT_OK;
}

// One time step with every group on this handle: the phases with the exchange buffer as both the partial
// and the total sums.
int mlqd_step_impl(Mlqd& m, trt_mlqd_stats* out) {
  double* x = m.xbuf;
  int rc;
  if ((rc = ph_step_begin(m, x)) || (rc = ph_step_begin_finish(m, x))) return rc;
  int rt = 0;
  bool rt_conv = false;
  while (!rt_conv && rt < m.v.maxit_rte) {
    ++rt;
    if ((rc = ph_outer_begin(m, rt, x)) || (rc = ph_outer_begin_finish(m, x))) return rc;
    int mg = 0;
    bool mg_conv = false;
    while (!mg_conv && mg < m.p.maxit_mloqd) {
      ++mg;
      if ((rc = ph_mgqd_local(m, x)) || (rc = ph_mgqd_finish(m, mg, x, &mg_conv))) return rc;
    }
    if ((rc = ph_outer_end(m, rt, &rt_conv))) return rc;
  }
  return ph_step_end(m, out);
}

}  // namespace

extern "C" {

int trt_mlqd_setup_range(trt_ctx* ctx, double Tini, const trt_mlqd_params* p, int ng_total, int g_first,
                         const double* nu_total) {
  if (!ctx || !p || !(Tini >= 0.0) || p->maxit_mloqd < 1 || p->maxit_gloqd < 1 || !(p->conv_lo >= 0.0) ||
      (p->ho_form != 0 && p->ho_form != 1) ||
      !(p->conv_gr1 >= 0.0) || !(p->conv_gr2 >= 0.0) || !(p->theta > 0.0) ||
      ((p->use_line_search || p->use_safety_search) && !(p->line_src > 1.0)) || ng_total < 0 ||
      (ng_total > 0 && !nu_total))
    return TRT_ERR_ARG;
  int rc = device_ok();
  if (rc) return rc;
  return mlqd_setup_impl(ctx, Tini, *p, ng_total, g_first, nu_total);
}

int trt_mlqd_setup(trt_ctx* ctx, double Tini, const trt_mlqd_params* p) {
  return trt_mlqd_setup_range(ctx, Tini, p, 0, 0, nullptr);
}

int trt_mlqd_step(trt_ctx* ctx, trt_mlqd_stats* stats) {
  if (!ctx) return TRT_ERR_ARG;
  Mlqd* m = static_cast<Mlqd*>(trt_host::handle_attached(ctx));
  if (!m) return TRT_ERR_STATE;
  return mlqd_step_impl(*m, stats);
}

long long trt_mlqd_exchange_size(trt_ctx* ctx) {
  if (!ctx) return TRT_ERR_ARG;
  const Mlqd* m = static_cast<const Mlqd*>(trt_host::handle_attached(ctx));
  if (!m) return TRT_ERR_STATE;
  return trt_gqd::greyx_of(m->d).size;
}

// The phases of a step (see ph_step_begin ... ph_step_end); buffers are device pointers of
// trt_mlqd_exchange_size doubles, `part` complete when the call returns.
static Mlqd* mlqd_of(trt_ctx* ctx) { return ctx ? static_cast<Mlqd*>(trt_host::handle_attached(ctx)) : nullptr; }

int trt_mlqd_step_begin(trt_ctx* ctx, double* part) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  return part ? ph_step_begin(*m, part) : TRT_ERR_ARG;
}
int trt_mlqd_step_begin_finish(trt_ctx* ctx, const double* tot) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  return tot ? ph_step_begin_finish(*m, tot) : TRT_ERR_ARG;
}
int trt_mlqd_outer_begin(trt_ctx* ctx, int rt, double* part) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  return part && rt >= 1 ? ph_outer_begin(*m, rt, part) : TRT_ERR_ARG;
}
int trt_mlqd_outer_begin_finish(trt_ctx* ctx, const double* tot) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  return tot ? ph_outer_begin_finish(*m, tot) : TRT_ERR_ARG;
}
int trt_mlqd_mgqd_local(trt_ctx* ctx, double* part) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  return part ? ph_mgqd_local(*m, part) : TRT_ERR_ARG;
}
int trt_mlqd_mgqd_finish(trt_ctx* ctx, int mg, const double* tot, int* converged) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  if (!tot || !converged || mg < 1) return TRT_ERR_ARG;
  bool c = false;
  const int rc = ph_mgqd_finish(*m, mg, tot, &c);
  *converged = c ? 1 : 0;
  return rc;
}
int trt_mlqd_outer_end(trt_ctx* ctx, int rt, int* converged) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  if (!converged || rt < 1) return TRT_ERR_ARG;
  bool c = false;
  const int rc = ph_outer_end(*m, rt, &c);
  *converged = c ? 1 : 0;
  return rc;
}
int trt_mlqd_step_end(trt_ctx* ctx, trt_mlqd_stats* stats) {
  Mlqd* m = mlqd_of(ctx);
  if (!m) return ctx ? TRT_ERR_STATE : TRT_ERR_ARG;
  return ph_step_end(*m, stats);
}

int trt_mlqd_counts(trt_ctx* ctx, int* mgqd_per_outer, int cap_outer, int* egp_per_mgqd, int cap_mgqd, int* n_outer,
                    int* n_mgqd) {
  if (!ctx) return TRT_ERR_ARG;
  const Mlqd* m = static_cast<const Mlqd*>(trt_host::handle_attached(ctx));
  if (!m) return TRT_ERR_STATE;
  for (int k = 0; k < cap_outer && k < (int)m->mg_counts.size() && mgqd_per_outer; ++k)
    mgqd_per_outer[k] = m->mg_counts[k];
  for (int k = 0; k < cap_mgqd && k < (int)m->egp_counts.size() && egp_per_mgqd; ++k)
    egp_per_mgqd[k] = m->egp_counts[k];
  if (n_outer) *n_outer = (int)m->mg_counts.size();
  if (n_mgqd) *n_mgqd = (int)m->egp_counts.size();
  return TRT_OK;
}

int trt_mlqd_put(trt_ctx* ctx, const char* name, const double* src, long long count, int on_device) {
  if (!ctx || !name || !src) return TRT_ERR_ARG;
  Mlqd* m = static_cast<Mlqd*>(trt_host::handle_attached(ctx));
  if (!m) return TRT_ERR_STATE;
  const Dims& d = m->d;
  const long long ng = d.ng;
  static const char* names[10] = {"fg_avg_xx", "fg_avg_yy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy",
                                  "fg_edgH_xy", "Cg_L",      "Cg_B",       "Cg_R",       "Cg_T"};
  const long long sizes[10] = {d.nC * ng, d.nC * ng, d.nV * ng, d.nV * ng, d.nH * ng,
                               d.nH * ng, d.ny * ng, d.nx * ng, d.ny * ng, d.nx * ng};
  for (int k = 0; k < 10; ++k)
    if (std::strcmp(names[k], name) == 0) {
      if (count != sizes[k]) return TRT_ERR_ARG;
      double* dst = const_cast<double*>(k < 6 ? m->f[k] : m->Cg[k - 6]);
      MG_CUDA(cudaMemcpyAsync(dst, src, (size_t)count * sizeof(double),
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, m->v.stream));
      MG_CUDA(cudaStreamSynchronize(m->v.stream));
      return TRT_OK;
    }
  return TRT_ERR_ARG;
}

int trt_mlqd_get(trt_ctx* ctx, const char* name, double* host, long long count) {
  if (!ctx || !name || !host) return TRT_ERR_ARG;
  Mlqd* m = static_cast<Mlqd*>(trt_host::handle_attached(ctx));
  if (!m) return TRT_ERR_STATE;
  const Dims& d = m->d;
  const long long ng = d.ng, C = d.nC, V = d.nV, H = d.nH, nx = d.nx, ny = d.ny;
  const struct {
    const char* n;
    const double* p;
    long long sz;
  } tab[] = {{"Temp", m->v.T, C},          {"E_avg", m->E, C},          {"E_edgV", m->EV, V},
             {"E_edgH", m->EH, H},         {"Fx_edgV", m->Fx, V},       {"Fy_edgH", m->Fy, H},
             {"KapE_Bar", m->Kb, C},       {"KapE_Bar_dT", m->Kdt, C},  {"GQD_Src", m->Q, C},
             {"Cb_L", m->Cb[0], ny},       {"Cb_B", m->Cb[1], nx},      {"Cb_R", m->Cb[2], ny},
             {"Cb_T", m->Cb[3], nx},       {"Eg_avg", m->Eg, C * ng},   {"Eg_edgV", m->EgV, V * ng},
             {"Eg_edgH", m->EgH, H * ng},  {"Fxg_edgV", m->MG->Fx, V * ng}, {"Fyg_edgH", m->MG->Fy, H * ng},
             {"MGQD_Src", m->Src, C * ng}, {"MGQD_E_avg", m->MGE, C}, {"HO_E_avg", m->HOEt, C},
             {"HO_E_avg_own", m->HOE, C}};
  for (const auto& t : tab)
    if (std::strcmp(t.n, name) == 0) {
      if (count < t.sz) return TRT_ERR_ARG;
      MG_CUDA(cudaMemcpyAsync(host, t.p, (size_t)t.sz * sizeof(double), cudaMemcpyDeviceToHost, m->v.stream));
      MG_CUDA(cudaStreamSynchronize(m->v.stream));
      return TRT_OK;
    }
  return TRT_ERR_ARG;
}

}  // extern "C"
