// C-ABI of libtrt_sweep.so (declarations and contracts: include/trt_sweep.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "trt_sweep.h"
#include "aux_kernels.cuh"
#include "handle_hooks.h"
#include "dropin_kernels.cuh"
#include "sweep_kernel.cuh"
#include "tstep_kernels.cuh"

namespace {

std::atomic<unsigned long long> g_launches{0};

#define TRT_CUDA(expr)                                  \
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

#define TRT_LAUNCHED() g_launches.fetch_add(1, std::memory_order_relaxed)

int device_check() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    cudaGetLastError();
    return TRT_ERR_NODEV;
  }
  return TRT_OK;
}

int grid_for(long long n, int block = 256) {
  long long b = (n + block - 1) / block;
  if (b < 1) b = 1;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)b;
}

// Bg_planck_calc and sigint, MainSrc/TEMP_FUNCTIONS.f08:90-141 (host evaluation).
double sigint_h(double z) {
  const double pi = 4.0 * std::atan(1.0);
  const double pi4 = (pi * pi) * (pi * pi);
  auto low = [](double x) { return ((x * x) * x) * (1.0 / 3.0 - x / 8.0 + (x * x) / 62.4); };
  auto high = [&](double x) { return pi4 / 15.0 - std::exp(-x) * (((x * x) * x) + 3.0 * (x * x) + 6.0 * x + 7.28); };
  if (z <= 1.95) return low(z);
  if (z > 2.05) return high(z);
  const double y1 = low(1.95), y2 = high(2.05);
  return y1 + (y2 - y1) * (z - 1.95) / (2.05 - 1.95);
}

double bg_planck_h(double T, double nl, double nh, double cu) {
  if (T <= 1e-15) return 0.0;
  const double c = 2.99792458e2, erg = 6.24150934e11, h = 6.62613e-19;
  double sig = sigint_h(nh / T) - sigint_h(nl / T);
  const double e2 = erg * erg;
  sig = sig / ((((h * h) * h) * (c * c)) * (e2 * e2) * cu);
  const double t2 = T * T;
  return (2.0 * (t2 * t2)) * sig;
}

struct Shape {
  int nx, ny, nm, ng, mq;
};

bool valid_shape(int nx, int ny, int nm, int ng) {
  return nx >= 1 && ny >= 1 && ng >= 1 && nm >= 4 && nm % 4 == 0 && nx < (1 << 20) && ny < (1 << 20);
}

// Compiled (slices, directions per lane) pairs of the sweep kernel; D is exact (ceil(ndir / S)) for
// the ndir directions of a split.
struct KernelCfg {
  int S, D;
};
const KernelCfg kCfgs[] = {{1, 2}, {1, 4}, {2, 2}, {2, 3}, {2, 5}, {2, 9}, {4, 1}, {4, 2}, {4, 3}, {4, 5},
                           {4, 6}, {4, 9}, {8, 1}, {8, 2}, {8, 3}, {8, 4}, {8, 5}, {16, 1}, {16, 2}, {16, 3},
                           {32, 1}, {32, 2}};

bool pick_cfg(int ndir, int prec, int S_req, KernelCfg* out) {
  bool found = false;
  KernelCfg best{0, 0};
  long best_key = 0;
  for (const KernelCfg& k : kCfgs) {
    if (S_req && k.S != S_req) continue;
    if ((ndir + k.S - 1) / k.S != k.D) continue;
    const int waste = k.S * k.D - ndir;
    // FP64 keeps D <= 5 (registers); then least idle slots; then fewer slices (fewer shuffles)
    const int dpen = (prec == TRT_PREC_FP64 && k.D > 5) ? 1 : 0;
    const long key = (long)dpen * 1000000 + waste * 1000 + k.S;
    if (!found || key < best_key) {
      found = true;
      best = k;
      best_key = key;
    }
  }
  if (found) *out = best;
  return found;
}

template <class Real>
using SweepKernel = void (*)(trt::SweepArgs<Real>);

// The compiled sweep kernel of a (slices, directions per lane) configuration (null if none).  Register
// level 0: any CTA size, at most 128 registers per thread; 1: at most 128 threads and 3 CTAs per SM (up to
// 170 registers); 2: at most 128 threads and 2 CTAs per SM (up to 255 registers).
template <class Real>
SweepKernel<Real> sweep_kernel_for(const KernelCfg& kc, bool src_full, int level = 0) {
#define TRT_SWEEP_CASE(S_, D_)                                                                         \
  if (kc.S == S_ && kc.D == D_)                                                                        \
    return src_full ? trt::scb_sweep_kernel<Real, S_, D_, true>                                        \
                    : (level == 2 ? trt::scb_sweep_kernel<Real, S_, D_, false, 128, 2>                 \
                                  : (level == 1 ? trt::scb_sweep_kernel<Real, S_, D_, false, 128, 3>     \
                                                : trt::scb_sweep_kernel<Real, S_, D_, false>));
  TRT_SWEEP_CASE(1, 2)
  TRT_SWEEP_CASE(1, 4)
  TRT_SWEEP_CASE(2, 2)
  TRT_SWEEP_CASE(2, 3)
  TRT_SWEEP_CASE(2, 5)
  TRT_SWEEP_CASE(2, 9)
  TRT_SWEEP_CASE(4, 1)
  TRT_SWEEP_CASE(4, 2)
  TRT_SWEEP_CASE(4, 3)
  TRT_SWEEP_CASE(4, 5)
  TRT_SWEEP_CASE(4, 6)
  TRT_SWEEP_CASE(4, 9)
  TRT_SWEEP_CASE(8, 1)
  TRT_SWEEP_CASE(8, 2)
  TRT_SWEEP_CASE(8, 3)
  TRT_SWEEP_CASE(8, 4)
  TRT_SWEEP_CASE(8, 5)
  TRT_SWEEP_CASE(16, 1)
  TRT_SWEEP_CASE(16, 2)
  TRT_SWEEP_CASE(16, 3)
  TRT_SWEEP_CASE(32, 1)
  TRT_SWEEP_CASE(32, 2)
#undef TRT_SWEEP_CASE
  return nullptr;
}

template <class Real>
using SweepBatchKernel = void (*)(const trt::SweepArgs<Real>*, const int*, int);

// The batched sweep kernel of a configuration (null if none); level 1 as for sweep_kernel_for.
template <class Real>
SweepBatchKernel<Real> sweep_batch_kernel_for(const KernelCfg& kc, bool src_full, int level = 0) {
#define TRT_SWEEP_CASE(S_, D_)                                                                         \
  if (kc.S == S_ && kc.D == D_)                                                                        \
    return src_full ? trt::scb_sweep_batch_kernel<Real, S_, D_, true>                                  \
                    : (level == 1 ? trt::scb_sweep_batch_kernel<Real, S_, D_, false, 128, 3>           \
                                  : trt::scb_sweep_batch_kernel<Real, S_, D_, false>);
  TRT_SWEEP_CASE(1, 2)
  TRT_SWEEP_CASE(1, 4)
  TRT_SWEEP_CASE(2, 2)
  TRT_SWEEP_CASE(2, 3)
  TRT_SWEEP_CASE(2, 5)
  TRT_SWEEP_CASE(2, 9)
  TRT_SWEEP_CASE(4, 1)
  TRT_SWEEP_CASE(4, 2)
  TRT_SWEEP_CASE(4, 3)
  TRT_SWEEP_CASE(4, 5)
  TRT_SWEEP_CASE(4, 6)
  TRT_SWEEP_CASE(4, 9)
  TRT_SWEEP_CASE(8, 1)
  TRT_SWEEP_CASE(8, 2)
  TRT_SWEEP_CASE(8, 3)
  TRT_SWEEP_CASE(8, 4)
  TRT_SWEEP_CASE(8, 5)
  TRT_SWEEP_CASE(16, 1)
  TRT_SWEEP_CASE(16, 2)
  TRT_SWEEP_CASE(16, 3)
  TRT_SWEEP_CASE(32, 1)
  TRT_SWEEP_CASE(32, 2)
#undef TRT_SWEEP_CASE
  return nullptr;
}

// Launch a sweep kernel; with NB band CTAs per (group, quadrant, split) sweep, every NB consecutive CTAs
// form one thread-block cluster (co-scheduled, so a band never waits for a CTA that is not running).
template <class K, class... Args>
cudaError_t launch_banded(K k, int NB, int grid, int block, size_t smem, cudaStream_t st, Args... args) {
  if (NB <= 1) {
    k<<<grid, block, smem, st>>>(args...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3((unsigned)block, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)NB;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

template <class Real>
using SweepQueueKernel = void (*)(const trt::SweepArgs<Real>*, const int*, int, int, int*);

// The persistent (work-queue) batched sweep of a configuration (null if none); level 1 as above.
template <class Real>
SweepQueueKernel<Real> sweep_queue_kernel_for(const KernelCfg& kc, bool src_full, int level = 0) {
#define TRT_SWEEP_CASE(S_, D_)                                                                         \
  if (kc.S == S_ && kc.D == D_)                                                                        \
    return src_full ? trt::scb_sweep_queue_kernel<Real, S_, D_, true>                                  \
                    : (level == 1 ? trt::scb_sweep_queue_kernel<Real, S_, D_, false, 128, 3>           \
                                  : trt::scb_sweep_queue_kernel<Real, S_, D_, false>);
  TRT_SWEEP_CASE(1, 2)
  TRT_SWEEP_CASE(1, 4)
  TRT_SWEEP_CASE(2, 2)
  TRT_SWEEP_CASE(2, 3)
  TRT_SWEEP_CASE(2, 5)
  TRT_SWEEP_CASE(2, 9)
  TRT_SWEEP_CASE(4, 1)
  TRT_SWEEP_CASE(4, 2)
  TRT_SWEEP_CASE(4, 3)
  TRT_SWEEP_CASE(4, 5)
  TRT_SWEEP_CASE(4, 6)
  TRT_SWEEP_CASE(4, 9)
  TRT_SWEEP_CASE(8, 1)
  TRT_SWEEP_CASE(8, 2)
  TRT_SWEEP_CASE(8, 3)
  TRT_SWEEP_CASE(8, 4)
  TRT_SWEEP_CASE(8, 5)
  TRT_SWEEP_CASE(16, 1)
  TRT_SWEEP_CASE(16, 2)
  TRT_SWEEP_CASE(16, 3)
  TRT_SWEEP_CASE(32, 1)
  TRT_SWEEP_CASE(32, 2)
#undef TRT_SWEEP_CASE
  return nullptr;
}

template <class Real>
cudaError_t launch_sweep(const KernelCfg& kc, bool src_full, int level, int grid, int block, size_t smem,
                         cudaStream_t st, const trt::SweepArgs<Real>& a) {
  SweepKernel<Real> k = sweep_kernel_for<Real>(kc, src_full, level);
  if (!k) return cudaErrorInvalidValue;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return launch_banded(k, a.t.NB, grid, block, smem, st, a);
}

// CTAs of a sweep configuration that are resident on one SM at once (0 on failure).
template <class Real>
int sweep_ctas_per_sm(const KernelCfg& kc, int block, size_t smem, int level = 0) {
  SweepKernel<Real> k = sweep_kernel_for<Real>(kc, false, level);
  int n = 0;
  if (!k) return 0;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, block, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

}  // namespace

constexpr unsigned kDefaultWaitPolls = 1u << 22;

struct trt_ctx {
  int nx = 0, ny = 0, nm = 0, ng = 0, mq = 0, prec = 0;
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;
  int Wreq = 0, Sreq = 0, NHreq = 0, NBreq = 0, stages = 2;   // NBreq: band CTAs per sweep (0: default)
  int regs = 0;                      // register level of the sweep kernel in use (set by setup_layout)
  int regs_req = -1;                 // -1: the highest level that keeps the grid resident; 0..2: at most that
  KernelCfg kc{8, 5};
  trt::Tiling t{};
  long long chunk = 0, blk = 0;
  std::vector<double> omx, omy, w, dx, dy;
  trt::WeightSums ws{};
  // device memory
  std::vector<void*> allocs;
  double* d_dir = nullptr;      // [kNDirRow][nm]
  void* d_dirtab = nullptr;     // [4][kNDirRow][mq] Real
  double *d_dx = nullptr, *d_dy = nullptr, *d_area = nullptr;
  void *d_dxr = nullptr, *d_dyr = nullptr, *d_arear = nullptr;
  double *d_kap64 = nullptr, *d_q64 = nullptr;
  void *d_kap = nullptr, *d_q = nullptr;
  void* d_state[2] = {nullptr, nullptr};
  int cur = 0;                  // d_state[cur] = I_crn_old, d_state[1-cur] = I_crn
  bool inplace = false;         // one state buffer, swept in place (each sweep consumes I_crn_old)
  void* ext_state = nullptr;    // caller-provided device memory holding the in-place state (trt_bind_state)
  void* d_srcfull = nullptr;
  bool use_srcfull = false;
  void *d_bndV = nullptr, *d_bndH = nullptr;
  void* d_wrap = nullptr;
  void* d_part = nullptr;        // moment partial records (state precision)
  int* d_err = nullptr;
  double* d_outs = nullptr;
  trt::MomentOut dout{};
  double *d_res_m = nullptr, *d_res = nullptr;
  int *d_res_loc = nullptr, *d_resx = nullptr, *d_resy = nullptr;
  double* d_stage = nullptr;    // per-group staging slab (double, 4*nx*ny*nm)
  double* d_bval = nullptr;     // [4][ng] Planck boundary values
  double c = 2.99792458e2, dt = 1.0, comp_unit = 1.0;
  int bc[4] = {0, 0, 0, 0};
  bool have_material = false, have_state = false, swept = false, have_moments = false, have_res = false;
  unsigned wait_polls = kDefaultWaitPolls;
  // transport-only time step (run_type 'tr_no_qd'): temperature and material model on the device
  bool ts_ready = false;
  double *d_T = nullptr, *d_Told = nullptr, *d_Trt1 = nullptr, *d_Trt2 = nullptr;
  double *d_Ert1 = nullptr, *d_Ert2 = nullptr, *d_nu = nullptr, *d_kmult = nullptr, *d_cv = nullptr;
  unsigned long long* d_conv = nullptr;   // [2][5] convergence reductions (T, E)
  double ts_Kap0 = 0.0, ts_conv_ho = 0.0, ts_Tb[4] = {0, 0, 0, 0};
  int ts_conv_type = 1, ts_maxit = 1, ts_bc[4] = {0, 0, 0, 0};
  int ts_law = trt::kLawFleckCummings;   // material law of the time loops (trt_tstep_set_law)
  std::vector<double> ts_nu;
  // pipelined stepping (trt_set_material_async / trt_moments_async): a copy stream for each direction,
  // a staging pair for the next material, and the events that order them against the handle's stream
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_staged = nullptr, ev_stage_free = nullptr, ev_epi = nullptr, ev_out = nullptr;
  double *d_kap_in = nullptr, *d_q_in = nullptr;
  bool out_pending = false;
  // low-order (mlqd) state attached by the MGQD side of the library, released with the handle
  void* lo = nullptr;
  void (*lo_free)(void*) = nullptr;

  size_t esz() const { return prec == TRT_PREC_FP64 ? sizeof(double) : sizeof(float); }
  long long state_elems() const { return 4LL * ng * t.NH * blk; }
  trt::Geo geo() const { return trt::Geo{nx, ny, nm, ng, mq, t, blk}; }

  int dalloc(void** p, size_t bytes) {
    if (budget && used + bytes > budget) return TRT_ERR_BUDGET;
    void* q = nullptr;
    if (cudaMalloc(&q, bytes ? bytes : 16) != cudaSuccess) {
      cudaGetLastError();
      return TRT_ERR_NOMEM;
    }
    allocs.push_back(q);
    used += bytes;
    *p = q;
    return TRT_OK;
  }
  void dfree(void* p, size_t bytes) {
    if (!p) return;
    cudaFree(p);
    allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
    used -= std::min(used, bytes);
  }
};

namespace {

template <class T>
int alloc_t(trt_ctx* c, T** p, size_t n) {
  void* q = nullptr;
  int rc = c->dalloc(&q, n * sizeof(T));
  *p = static_cast<T*>(q);
  return rc;
}

// Sizes (elements) of the combined outputs, in MomentOut field order.
void output_sizes(int nx, int ny, int ng, long long* sz) {
  const long long A = (long long)nx * ny, V = (long long)(nx + 1) * ny, H = (long long)nx * (ny + 1);
  long long s[] = {A * ng, A * ng, A * ng, V * ng, V * ng, H * ng, H * ng,   // Hg
                   A * ng, V * ng, H * ng, V * ng, H * ng,                   // Eg, Fg
                   A * ng, A * ng, A * ng, V * ng, V * ng, H * ng, H * ng,   // fg
                   (long long)ny * ng, (long long)nx * ng, (long long)ny * ng, (long long)nx * ng,   // Cg L B R T
                   (long long)ny * ng, (long long)nx * ng, (long long)ny * ng, (long long)nx * ng,   // Eg_in
                   (long long)ny * ng, (long long)nx * ng, (long long)ny * ng, (long long)nx * ng,   // Fg_in
                   A, V, H, V, H,                                                 // E, F totals
                   ny, nx, ny, nx, ny, nx, ny, nx,                                // E_in, F_in totals
                   H * ng, H};                                                    // Fy true
  for (int k = 0; k < (int)(sizeof(s) / sizeof(s[0])); ++k) sz[k] = s[k];
}
constexpr int kNOut = 46;
static_assert(sizeof(trt::MomentOut) == kNOut * sizeof(double*), "MomentOut layout");
static_assert(sizeof(trt_moments_host) == kNOut * sizeof(double*), "trt_moments_host layout");

const char* kOutNames[kNOut] = {
    "Hg_avg_xx", "Hg_avg_yy", "Hg_avg_xy", "Hg_edgV_xx", "Hg_edgV_xy", "Hg_edgH_yy", "Hg_edgH_xy",
    "Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH",
    "fg_avg_xx", "fg_avg_yy", "fg_avg_xy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy",
    "Cg_L", "Cg_B", "Cg_R", "Cg_T",
    "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B", "Fg_in_R", "Fg_in_T",
    "E_avg", "E_edgV", "E_edgH", "Fx_edgV", "Fy_edgH",
    "E_in_L", "E_in_B", "E_in_R", "E_in_T", "F_in_L", "F_in_B", "F_in_R", "F_in_T",
    "Fyg_edgH_true", "Fy_edgH_true"};

size_t layout_state_bytes(int nx, int ny, int mq, int ng, int W, int S, int NH, size_t esz) {
  trt::Tiling t = trt::make_tiling(nx, ny, mq, W, S, NH);
  return (size_t)4 * ng * NH * trt::block_elems(t) * esz;
}

// Default tiling.  The grid has 4*ng*NH CTAs (NH = direction splits per quadrant) of W warps; every
// CTA of one tiling does the same work, so the busiest SM sets the sweep time.  Candidates keep
// 16 warps per SM resident at <= 128 registers: NH = 1, 2, 4 with W = 8, 4, 2.  The one whose
// busiest SM carries the least work (ceil(CTAs / SMs) / NH) wins, ties to fewer splits.  C1
// (50 groups): 200 CTAs put 2 on some SMs (1.48x the mean), 400 half-size CTAs put 3 halves
// (1.11x the mean): NH = 2, measured 12% faster in FP64 and 11% in FP32.  Fewer warps when a
// round would exceed the grid height by far.
int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) ==
                                                  cudaSuccess && v > 0)
      n = v;
    else {
      cudaGetLastError();
      n = 148;
    }
  }
  return n;
}

int default_W(int R, int ny, int W = 8) {
  while (W > 1 && (W / 2) * R >= ny) W /= 2;
  return W;
}

// part_bytes_per_split: the moment partial records one split count adds (4 quadrants x cells x groups x record);
// more splits only balance the SMs, so a split count whose records would take more than 16 GB (an instance
// large enough to fill the SMs without it, e.g. 1024^2 x 64 groups) is not chosen.
void default_split(int ng, int mq, int* NH, int* W, size_t part_bytes_per_split = 0) {
  const int sms = sm_count();
  *NH = 1;
  *W = 8;
  double best = 0.0;
  for (int nh = 1; nh <= 4; nh *= 2) {
    if (nh > 1 && mq < 4 * nh) break;   // at least 4 directions per split
    if (nh > 1 && part_bytes_per_split * nh > ((size_t)16 << 30)) break;
    const long long ctas = 4LL * ng * nh;
    const double busiest = (double)((ctas + sms - 1) / sms) / nh;   // work of the busiest SM
    const double load = (double)ctas / sms / nh / busiest;           // mean / busiest
    if (load > best + 0.02) {
      best = load;
      *NH = nh;
      *W = 8 / nh;
    }
  }
}

size_t part_bytes(const trt_ctx* c) {
  const size_t rec = c->prec == TRT_PREC_FP64 ? trt::part_rec<double>() * sizeof(double)
                                                : trt::part_rec<float>() * sizeof(float);
  return (size_t)4 * c->t.NH * c->ng * c->nx * c->ny * rec;
}
size_t wrap_bytes(const trt_ctx* c) { return (size_t)4 * c->ng * c->t.NH * c->nx * c->t.mqc * 2 * c->esz(); }

// (Re)compute the tiling and (re)allocate the layout-dependent buffers (state, source, round wrap
// buffer, moment partials).
int setup_layout(trt_ctx* c) {
  int NH = 1, Wdef = 8;
  const size_t rec_bytes = c->prec == TRT_PREC_FP64 ? trt::part_rec<double>() * sizeof(double)
                                                     : trt::part_rec<float>() * sizeof(float);
  default_split(c->ng, c->mq, &NH, &Wdef, (size_t)4 * c->ng * c->nx * c->ny * rec_bytes);
  if (c->NHreq) NH = c->NHreq;
  if (NH < 1 || NH > c->mq) return TRT_ERR_ARG;
  const int mqc = (c->mq + NH - 1) / NH;
  if (!pick_cfg(mqc, c->prec, c->Sreq, &c->kc)) return c->Sreq ? TRT_ERR_ARG : TRT_ERR_UNSUPPORTED;
  const int R = 32 / c->kc.S;
  const int W = c->Wreq ? c->Wreq : default_W(R, c->ny, c->NHreq ? std::max(1, 8 / NH) : Wdef);
  const size_t esz = c->esz();
  // sizes of the current buffers (t still describes them)
  const size_t sbytes_old = c->blk ? (size_t)c->state_elems() * esz : 0;
  const size_t src_old = sbytes_old;
  const size_t wrap_old = c->blk ? wrap_bytes(c) : 0, part_old = c->blk ? part_bytes(c) : 0;
  // band CTAs per sweep: requested (trt_set_bands, trt_autotune), else one
  int NB = c->NBreq > 0 ? c->NBreq : 1;
  if (NB > 8) return TRT_ERR_ARG;
  const trt::Tiling t = trt::make_tiling(c->nx, c->ny, c->mq, W, c->kc.S, NH, NB);
  // pipeline depth limited by shared memory
  const long long chunk = trt::chunk_elems(t);
  auto smem_at = [&](int st) {
    return c->prec == TRT_PREC_FP64 ? trt::sweep_smem_bytes<double>(W, chunk, st, t.mqc, t.D, t.S)
                                    : trt::sweep_smem_bytes<float>(W, chunk, st, t.mqc, t.D, t.S);
  };
  int stages = c->stages;
  while (stages > 1 && smem_at(stages) > (size_t)200 * 1024) stages--;
  if (smem_at(stages) > (size_t)220 * 1024) return TRT_ERR_ARG;   // tiling does not fit an SM
  if (c->ext_state) {   // a bound external state is dropped with the layout it was sized for
    c->d_state[0] = c->d_state[1] = nullptr;
    c->ext_state = nullptr;
  }
  if (c->d_state[1] == c->d_state[0]) c->d_state[1] = nullptr;   // in place: one buffer
  for (int k = 0; k < 2; ++k) {
    c->dfree(c->d_state[k], sbytes_old);
    c->d_state[k] = nullptr;
  }
  c->dfree(c->d_srcfull, src_old);
  c->d_srcfull = nullptr;
  c->dfree(c->d_wrap, wrap_old);
  c->d_wrap = nullptr;
  c->dfree(c->d_part, part_old);
  c->d_part = nullptr;
  c->use_srcfull = false;
  c->have_state = false;
  c->swept = false;
  c->have_moments = false;
  c->stages = stages;
  c->t = t;
  c->chunk = chunk;
  c->blk = trt::block_elems(t);
  // the highest register level whose variant keeps the whole grid resident (CTAs of at most 4 warps)
  c->regs = 0;
  const int cap = c->regs_req < 0 ? 2 : c->regs_req;
  for (int level = cap; level >= 1 && 32 * W <= 128; --level) {
    const size_t smem = smem_at(stages);
    const int per = c->prec == TRT_PREC_FP64 ? sweep_ctas_per_sm<double>(c->kc, 32 * W, smem, level)
                                             : sweep_ctas_per_sm<float>(c->kc, 32 * W, smem, level);
    if (per > 0 && 4LL * c->ng * NH * t.NB <= (long long)per * sm_count()) {
      c->regs = level;
      break;
    }
  }
  const size_t sbytes = (size_t)c->state_elems() * esz;
  for (int k = 0; k < (c->inplace ? 1 : 2); ++k) {
    int rc = c->dalloc(&c->d_state[k], sbytes);
    if (rc) return rc;
    TRT_CUDA(cudaMemsetAsync(c->d_state[k], 0, sbytes, c->stream));
  }
  if (c->inplace) c->d_state[1] = c->d_state[0];
  int rc = c->dalloc(&c->d_wrap, wrap_bytes(c));
  if (rc) return rc;
  if ((rc = c->dalloc(&c->d_part, part_bytes(c)))) return rc;
  TRT_CUDA(cudaMemsetAsync(c->d_part, 0, part_bytes(c), c->stream));
  return TRT_OK;
}

template <class Real>
void fill_dirtab(const trt_ctx* c, std::vector<Real>& tab, std::vector<double>& full, trt::WeightSums& ws) {
  const int nm = c->nm, mq = c->mq;
  tab.assign((size_t)4 * trt::kNDirRow * mq, Real(0));
  full.assign((size_t)trt::kNDirRow * nm, 0.0);
  std::memset(&ws, 0, sizeof(ws));
  for (int m = 0; m < nm; ++m) {
    const double ox = c->omx[m], oy = c->omy[m], ww = c->w[m];
    double v[trt::kNDirRow];
    v[trt::kAx] = std::fabs(ox);
    v[trt::kAy] = std::fabs(oy);
    v[trt::kW] = ww;
    v[trt::kWxx] = (ox * ox) * ww;
    v[trt::kWyy] = (oy * oy) * ww;
    v[trt::kWxy] = ox * oy * ww;
    v[trt::kWx] = ox * ww;
    v[trt::kWy] = oy * ww;
    const int q = m / mq, ml = m % mq;
    for (int r = 0; r < trt::kNDirRow; ++r) {
      tab[((size_t)q * trt::kNDirRow + r) * mq + ml] = (Real)v[r];
      full[(size_t)r * nm + m] = v[r];
      if (r >= trt::kW) ws.s[q][r] += v[r];
    }
  }
}

// The step's material handed to the handle in one pass over SMs (a device-to-device cudaMemcpyAsync runs on a
// copy engine, about 1 ms for C1's four planes): the FP64 copies (kap64, q64; skipped when null, i.e. the
// sources are those arrays already) and the sweep's Real copies.
template <class Real>
__global__ void material_copy_kernel(long long n, const double* __restrict__ kin, const double* __restrict__ qin,
                                     double* __restrict__ kap64, double* __restrict__ q64, Real* __restrict__ kapR,
                                     Real* __restrict__ qR) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double a = kin[k], b = qin[k];
    if (kap64) {
      kap64[k] = a;
      q64[k] = b;
    }
    kapR[k] = (Real)a;
    qR[k] = (Real)b;
  }
}

int ensure_stage(trt_ctx* c) {
  if (c->d_stage) return TRT_OK;
  return alloc_t(c, &c->d_stage, (size_t)4 * c->nx * c->ny * c->nm);
}

// Upload a Fortran corner array (2nx,2ny,nm,ng) into a skewed buffer, one group slab at a time.
template <class Real>
int pack_corner_array(trt_ctx* c, const double* host, void* dst) {
  int rc = ensure_stage(c);
  if (rc) return rc;
  const long long slab = 4LL * c->nx * c->ny * c->nm;
  trt::Geo G = c->geo();
  for (int g = 0; g < c->ng; ++g) {
    TRT_CUDA(cudaMemcpyAsync(c->d_stage, host + slab * g, slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    trt::Geo Gg = G;
    Gg.ng = 1;
    // pack one group: shift the skewed base to group g (block index (g*4 + q)*NH + h)
    Real* base = static_cast<Real*>(dst) + (long long)g * 4 * c->t.NH * c->blk;
    trt::pack_state_kernel<Real><<<grid_for(slab), 256, 0, c->stream>>>(Gg, c->d_stage, base);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
  }
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

template <class Real>
int unpack_corner_array(trt_ctx* c, const void* src, double* host) {
  int rc = ensure_stage(c);
  if (rc) return rc;
  const long long slab = 4LL * c->nx * c->ny * c->nm;
  trt::Geo G = c->geo();
  for (int g = 0; g < c->ng; ++g) {
    trt::Geo Gg = G;
    Gg.ng = 1;
    const Real* base = static_cast<const Real*>(src) + (long long)g * 4 * c->t.NH * c->blk;
    trt::unpack_state_kernel<Real><<<grid_for(slab), 256, 0, c->stream>>>(Gg, base, c->d_stage);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    TRT_CUDA(cudaMemcpyAsync(host + slab * g, c->d_stage, slab * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(cudaStreamSynchronize(c->stream));
  }
  return TRT_OK;
}

int check_err(trt_ctx* c) {
  int h = 0;
  TRT_CUDA(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  if (h) {
    TRT_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    return TRT_ERR_TIMEOUT;
  }
  return TRT_OK;
}

template <class Real>
trt::SweepArgs<Real> make_sweep_args(const trt_ctx* c) {
  trt::SweepArgs<Real> a{};
  a.nx = c->nx; a.ny = c->ny; a.nm = c->nm; a.ng = c->ng; a.mq = c->mq;
  a.t = c->t;
  a.stages = c->stages;
  a.chunk = c->chunk;
  a.blk = c->blk;
  a.rcdt = (Real)(1.0 / (c->c * c->dt));
  a.dx = (const Real*)c->d_dxr;
  a.dy = (const Real*)c->d_dyr;
  a.area = (const Real*)c->d_arear;
  a.kap = (const Real*)c->d_kap;
  a.qiso = c->use_srcfull ? nullptr : (const Real*)c->d_q;
  a.srcfull = c->use_srcfull ? (const Real*)c->d_srcfull : nullptr;
  a.dirtab = (const Real*)c->d_dirtab;
  a.dir64 = c->d_dir;
  a.Iold = (const Real*)c->d_state[c->cur];
  a.Inew = (Real*)c->d_state[1 - c->cur];
  a.bndV = (Real*)c->d_bndV;
  a.bndH = (Real*)c->d_bndH;
  a.wrap = (Real*)c->d_wrap;
  a.part = (Real*)c->d_part;
  a.err = c->d_err;
  a.max_polls = c->wait_polls;
  a.drain_polls = 1u << 24;
  return a;
}

template <class Real>
size_t sweep_smem(const trt_ctx* c) {
  return trt::sweep_smem_bytes<Real>(c->t.W, c->chunk, c->stages, c->t.mqc, c->t.D, c->t.S);
}

template <class Real>
int sweep_epilogue(trt_ctx* c, unsigned flags);

template <class Real>
int sweep_impl(trt_ctx* c, unsigned flags) {
  // in place, a sweep overwrites I_crn_old: the next one must start a new step (roll) and the residuals,
  // which read I_crn_old after the sweep, are not available
  if (c->inplace && ((c->swept && !(flags & TRT_ROLL_STATE)) || (flags & TRT_RES_CALC))) return TRT_ERR_STATE;
  if (flags & TRT_ROLL_STATE) c->cur = 1 - c->cur;   // I_crn_old <- I_crn (ALGORITHMS.f08:397)
  const trt::SweepArgs<Real> a = make_sweep_args<Real>(c);
  cudaError_t e = launch_sweep<Real>(c->kc, c->use_srcfull, c->use_srcfull ? 0 : c->regs,
                                     4 * c->ng * c->t.NH * c->t.NB, 32 * c->t.W, sweep_smem<Real>(c), c->stream, a);
  TRT_LAUNCHED();
  if (e != cudaSuccess) return TRT_ERR_CUDA;
  c->swept = true;
  return sweep_epilogue<Real>(c, flags);
}

// Moments / QD factors and residual norms after a sweep (on the handle's stream).
template <class Real>
int sweep_epilogue(trt_ctx* c, unsigned flags) {
  if ((flags & TRT_MOMENTS) && c->out_pending) {
    // the outputs of the previous step are still being copied out (trt_moments_async)
    TRT_CUDA(cudaStreamWaitEvent(c->stream, c->ev_out, 0));
    c->out_pending = false;
  }
  if (flags & TRT_MOMENTS) {
    trt::CombineArgs A{};
    A.nx = c->nx; A.ny = c->ny; A.nm = c->nm; A.ng = c->ng; A.mq = c->mq; A.nh = c->t.NH;
    A.eps = 1e-25 / c->comp_unit;
    A.c = c->c;
    for (int k = 0; k < 4; ++k) A.bc[k] = c->bc[k];
    A.ws = c->ws;
    A.part = c->d_part;
    A.dir = c->d_dir;
    // interior: one CTA per kCombTX x kCombTY tile of cells of one group
    const dim3 cgrid((c->nx + trt::kCombTX - 1) / trt::kCombTX, (c->ny + trt::kCombTY - 1) / trt::kCombTY, c->ng);
    cudaFuncSetAttribute(trt::combine_cells_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)trt::comb_smem<Real>());
    trt::combine_cells_kernel<Real><<<cgrid, trt::kCombTX * trt::kCombTY, trt::comb_smem<Real>(), c->stream>>>(A,
                                                                                                           c->dout);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    const long long nb = 2LL * (c->nx + c->ny) * c->ng;
    trt::combine_boundary_kernel<Real><<<grid_for(nb), 256, 0, c->stream>>>(A, (const Real*)c->d_bndV,
                                                                            (const Real*)c->d_bndH, c->dout);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    trt::group_sum_kernel<<<grid_for(trt::group_sum_items(c->nx, c->ny)), 256, 0, c->stream>>>(c->nx, c->ny,
                                                                                               c->ng, c->dout);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    c->have_moments = true;
  }
  if (flags & TRT_RES_CALC) {
    if (!c->d_res_m) {
      int rc = alloc_t(c, &c->d_res_m, (size_t)5 * c->nm * c->ng);
      if (!rc) rc = alloc_t(c, &c->d_res_loc, (size_t)2 * c->nm * c->ng);
      if (!rc) rc = alloc_t(c, &c->d_res, (size_t)20 * c->ng);
      if (!rc) rc = alloc_t(c, &c->d_resx, (size_t)20 * c->ng);
      if (!rc) rc = alloc_t(c, &c->d_resy, (size_t)20 * c->ng);
      if (rc) return rc;
    }
    trt::ResidualArgs<Real> ra{};
    ra.G = c->geo();
    // Omega_x and Omega_y follow the kNDirRow rows of the direction table
    ra.omx = c->d_dir + (size_t)trt::kNDirRow * c->nm;
    ra.omy = ra.omx + c->nm;
    ra.dx = c->d_dx; ra.dy = c->d_dy; ra.area = c->d_area;
    ra.kap = c->d_kap64;
    ra.rcdt = 1.0 / (c->c * c->dt);
    ra.Inew = (const Real*)c->d_state[1 - c->cur];
    ra.Iold = (const Real*)c->d_state[c->cur];
    ra.qiso = c->use_srcfull ? nullptr : (const Real*)c->d_q;
    ra.srcfull = c->use_srcfull ? (const Real*)c->d_srcfull : nullptr;
    ra.bndV = (const Real*)c->d_bndV;
    ra.bndH = (const Real*)c->d_bndH;
    ra.per_m = c->d_res_m;
    ra.per_m_loc = c->d_res_loc;
    trt::residual_kernel<Real><<<(c->nm * c->ng + 63) / 64, 64, 0, c->stream>>>(ra);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    trt::residual_reduce_kernel<<<(4 * c->ng + 63) / 64, 64, 0, c->stream>>>(c->nx, c->ny, c->nm, c->ng, c->d_res_m,
                                                                            c->d_res_loc, c->d_res, c->d_resx,
                                                                            c->d_resy);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    c->have_res = true;
  }
  return TRT_OK;
}

template <class Real>
int set_material_impl(trt_ctx* c, const double* kap, const double* q, bool device) {
  const size_t n = (size_t)c->nx * c->ny * c->ng;
  if (device) {
    material_copy_kernel<Real><<<grid_for(n), 256, 0, c->stream>>>(n, kap, q, c->d_kap64, c->d_q64, (Real*)c->d_kap,
                                                                   (Real*)c->d_q);
  } else {
    TRT_CUDA(cudaMemcpyAsync(c->d_kap64, kap, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TRT_CUDA(cudaMemcpyAsync(c->d_q64, q, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    material_copy_kernel<Real><<<grid_for(n), 256, 0, c->stream>>>(n, c->d_kap64, c->d_q64, nullptr, nullptr,
                                                                   (Real*)c->d_kap, (Real*)c->d_q);
  }
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  if (!device) TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

// Boundary corner-edge values on the inflow faces from full reference arrays.
template <class Real>
int set_boundary_impl(trt_ctx* c, const double* IcV, const double* IcH) {
  const int nx = c->nx, ny = c->ny, nm = c->nm, ng = c->ng;
  const size_t nV = (size_t)2 * ng * nm * 2 * ny, nH = (size_t)2 * ng * nm * 2 * nx;
  std::vector<Real> bV(nV, Real(0)), bH(nH, Real(0));
  if (IcV) {
    for (int side = 0; side < 2; ++side)
      for (int g = 0; g < ng; ++g)
        for (int m = 0; m < nm; ++m)
          for (int iy = 0; iy < 2 * ny; ++iy) {
            const int f = side ? nx : 0;
            bV[((size_t)(side * ng + g) * nm + m) * 2 * ny + iy] =
                (Real)IcV[f + (size_t)(nx + 1) * (iy + (size_t)2 * ny * (m + (size_t)nm * g))];
          }
  }
  if (IcH) {
    for (int side = 0; side < 2; ++side)
      for (int g = 0; g < ng; ++g)
        for (int m = 0; m < nm; ++m)
          for (int ix = 0; ix < 2 * nx; ++ix) {
            const int f = side ? ny : 0;
            bH[((size_t)(side * ng + g) * nm + m) * 2 * nx + ix] =
                (Real)IcH[ix + (size_t)2 * nx * (f + (size_t)(ny + 1) * (m + (size_t)nm * g))];
          }
  }
  TRT_CUDA(cudaMemcpyAsync(c->d_bndV, bV.data(), nV * sizeof(Real), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaMemcpyAsync(c->d_bndH, bH.data(), nH * sizeof(Real), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

template <class Real>
int bc_update_impl(trt_ctx* c, const int* bc, const double* Tb, double cu, const double* nu) {
  std::vector<double> bval((size_t)4 * c->ng, 0.0);
  for (int s = 0; s < 4; ++s)
    for (int g = 0; g < c->ng; ++g) bval[(size_t)s * c->ng + g] = bg_planck_h(Tb[s], nu[g], nu[g + 1], cu);
  TRT_CUDA(cudaMemcpyAsync(c->d_bval, bval.data(), bval.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  const long long n = 2LL * c->ng * c->nm * 2 * std::max(c->nx, c->ny);
  trt::bc_update_kernel<Real><<<grid_for(n), 256, 0, c->stream>>>(c->nx, c->ny, c->nm, c->ng,
                                                                   make_int4(bc[0], bc[1], bc[2], bc[3]), c->d_bval,
                                                                   (Real*)c->d_bndV, (Real*)c->d_bndH);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

template <class Real>
int init_state_impl(trt_ctx* c, double Tini, const double* Tb, double cu, const double* nu) {
  std::vector<double> per_g(c->ng);
  for (int g = 0; g < c->ng; ++g) per_g[g] = bg_planck_h(Tini, nu[g], nu[g + 1], cu);
  // per-group values staged in the boundary-value buffer (bc_update_impl below overwrites it later in
  // stream order), then streaming fills of both states and of every boundary value: RT_INIT sets all of
  // Ic_edgV/H to Bg(Tini) before the Planck inflow faces
  double* d_pg = c->d_bval;
  TRT_CUDA(cudaMemcpyAsync(d_pg, per_g.data(), c->ng * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  const long long per_group = 4LL * c->t.NH * c->blk;
  for (int k = 0; k < 2; ++k) {
    trt::fill_groups_kernel<Real><<<grid_for(per_group * c->ng), 256, 0, c->stream>>>(per_group, c->ng, d_pg,
                                                                                       (Real*)c->d_state[k]);
    TRT_LAUNCHED();
  }
  const long long pv = (long long)c->nm * 2 * c->ny, ph = (long long)c->nm * 2 * c->nx;
  for (int side = 0; side < 2; ++side) {
    trt::fill_groups_kernel<Real><<<grid_for(pv * c->ng), 256, 0, c->stream>>>(
        pv, c->ng, d_pg, (Real*)c->d_bndV + (size_t)side * c->ng * pv);
    TRT_LAUNCHED();
    trt::fill_groups_kernel<Real><<<grid_for(ph * c->ng), 256, 0, c->stream>>>(
        ph, c->ng, d_pg, (Real*)c->d_bndH + (size_t)side * c->ng * ph);
    TRT_LAUNCHED();
  }
  TRT_CUDA(cudaGetLastError());
  int rc;
  const int zero[4] = {0, 0, 0, 0};
  rc = bc_update_impl<Real>(c, zero, Tb, cu, nu);
  if (rc) return rc;
  c->have_state = true;
  c->swept = false;
  return TRT_OK;
}

template <class Real>
int get_angular_impl(trt_ctx* c, double* I_avg, double* I_edgV, double* I_edgH, double* Ic_edgV, double* Ic_edgH) {
  const int nx = c->nx, ny = c->ny, nm = c->nm, ng = c->ng;
  double* outs[5] = {I_avg, I_edgV, I_edgH, Ic_edgV, Ic_edgH};
  const long long sz[5] = {(long long)nx * ny * nm * ng, (long long)(nx + 1) * ny * nm * ng,
                           (long long)nx * (ny + 1) * nm * ng, (long long)(nx + 1) * 2 * ny * nm * ng,
                           (long long)2 * nx * (ny + 1) * nm * ng};
  const void* st = c->d_state[c->swept ? 1 - c->cur : c->cur];
  for (int k = 0; k < 5; ++k) {
    if (!outs[k]) continue;
    double* d = nullptr;
    int rc = alloc_t(c, &d, (size_t)sz[k]);
    if (rc) return rc;
    double* p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    p[k] = d;
    trt::export_angular_kernel<Real><<<grid_for(sz[k]), 256, 0, c->stream>>>(
        c->geo(), (const Real*)st, (const Real*)c->d_bndV, (const Real*)c->d_bndH, p[0], p[1], p[2], p[3], p[4]);
    TRT_LAUNCHED();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(outs[k], d, sz[k] * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    c->dfree(d, sz[k] * sizeof(double));
    if (e != cudaSuccess) return TRT_ERR_CUDA;
  }
  return TRT_OK;
}

int create_buffers(trt_ctx* c) {
  int rc;
  const size_t esz = c->esz();
  const int nx = c->nx, ny = c->ny, nm = c->nm, ng = c->ng;
  // direction table: kNDirRow rows, then Omega_x and Omega_y rows
  std::vector<double> full;
  if (c->prec == TRT_PREC_FP64) {
    std::vector<double> tab;
    fill_dirtab<double>(c, tab, full, c->ws);
    if ((rc = c->dalloc(&c->d_dirtab, tab.size() * sizeof(double)))) return rc;
    TRT_CUDA(cudaMemcpy(c->d_dirtab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
  } else {
    std::vector<float> tab;
    fill_dirtab<float>(c, tab, full, c->ws);
    if ((rc = c->dalloc(&c->d_dirtab, tab.size() * sizeof(float)))) return rc;
    TRT_CUDA(cudaMemcpy(c->d_dirtab, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  full.insert(full.end(), c->omx.begin(), c->omx.end());
  full.insert(full.end(), c->omy.begin(), c->omy.end());
  if ((rc = alloc_t(c, &c->d_dir, full.size()))) return rc;
  TRT_CUDA(cudaMemcpy(c->d_dir, full.data(), full.size() * sizeof(double), cudaMemcpyHostToDevice));

  std::vector<double> area((size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) area[i + (size_t)nx * j] = c->dx[i] * c->dy[j];   // OUTER_PROD, INITIALIZERS.f08:152
  if ((rc = alloc_t(c, &c->d_dx, nx)) || (rc = alloc_t(c, &c->d_dy, ny)) || (rc = alloc_t(c, &c->d_area, (size_t)nx * ny)))
    return rc;
  TRT_CUDA(cudaMemcpy(c->d_dx, c->dx.data(), nx * sizeof(double), cudaMemcpyHostToDevice));
  TRT_CUDA(cudaMemcpy(c->d_dy, c->dy.data(), ny * sizeof(double), cudaMemcpyHostToDevice));
  TRT_CUDA(cudaMemcpy(c->d_area, area.data(), area.size() * sizeof(double), cudaMemcpyHostToDevice));
  if ((rc = c->dalloc(&c->d_dxr, nx * esz)) || (rc = c->dalloc(&c->d_dyr, ny * esz)) ||
      (rc = c->dalloc(&c->d_arear, (size_t)nx * ny * esz)))
    return rc;
  if (c->prec == TRT_PREC_FP64) {
    TRT_CUDA(cudaMemcpy(c->d_dxr, c->d_dx, nx * esz, cudaMemcpyDeviceToDevice));
    TRT_CUDA(cudaMemcpy(c->d_dyr, c->d_dy, ny * esz, cudaMemcpyDeviceToDevice));
    TRT_CUDA(cudaMemcpy(c->d_arear, c->d_area, (size_t)nx * ny * esz, cudaMemcpyDeviceToDevice));
  } else {
    std::vector<float> f(c->dx.begin(), c->dx.end());
    TRT_CUDA(cudaMemcpy(c->d_dxr, f.data(), nx * esz, cudaMemcpyHostToDevice));
    f.assign(c->dy.begin(), c->dy.end());
    TRT_CUDA(cudaMemcpy(c->d_dyr, f.data(), ny * esz, cudaMemcpyHostToDevice));
    f.assign(area.begin(), area.end());
    TRT_CUDA(cudaMemcpy(c->d_arear, f.data(), (size_t)nx * ny * esz, cudaMemcpyHostToDevice));
  }
  const size_t ncell = (size_t)nx * ny * ng;
  if ((rc = alloc_t(c, &c->d_kap64, ncell)) || (rc = alloc_t(c, &c->d_q64, ncell)) ||
      (rc = c->dalloc(&c->d_kap, ncell * esz)) || (rc = c->dalloc(&c->d_q, ncell * esz)))
    return rc;
  if ((rc = c->dalloc(&c->d_bndV, (size_t)2 * ng * nm * 2 * ny * esz)) ||
      (rc = c->dalloc(&c->d_bndH, (size_t)2 * ng * nm * 2 * nx * esz)))
    return rc;
  TRT_CUDA(cudaMemset(c->d_bndV, 0, (size_t)2 * ng * nm * 2 * ny * esz));
  TRT_CUDA(cudaMemset(c->d_bndH, 0, (size_t)2 * ng * nm * 2 * nx * esz));
  if ((rc = alloc_t(c, &c->d_err, 1))) return rc;
  TRT_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
  if ((rc = alloc_t(c, &c->d_bval, (size_t)4 * ng))) return rc;
  long long sz[kNOut];
  output_sizes(nx, ny, ng, sz);
  long long tot = 0;
  for (int k = 0; k < kNOut; ++k) tot += sz[k];
  if ((rc = alloc_t(c, &c->d_outs, (size_t)tot))) return rc;
  TRT_CUDA(cudaMemset(c->d_outs, 0, (size_t)tot * sizeof(double)));
  double** f = reinterpret_cast<double**>(&c->dout);
  long long off = 0;
  for (int k = 0; k < kNOut; ++k) {
    f[k] = c->d_outs + off;
    off += sz[k];
  }
  return setup_layout(c);
}

int transport_scb_impl(trt_ctx* c, int nx, int ny, int nm, int ng, double* I_avg, double* I_edgV, double* I_edgH,
                       double* I_crn, double* Ic_edgV, double* Ic_edgH, const double* A, const double* KapE_in,
                       const double* Src_in, const double* I_crn_old, double cl, double Delt, double* RT_Residual,
                       int* RT_ResLoc_x, int* RT_ResLoc_y, int Res_Calc) {
  int rc;
  // The reference builds gamma from Delx*Dely (SCB_BGEN :342) and the source term from A(i,j);
  // this library uses A(i,j) for the source term as well.
  std::vector<double> area(A, A + (size_t)nx * ny);
  TRT_CUDA(cudaMemcpyAsync(c->d_area, area.data(), area.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaMemcpyAsync(c->d_arear, c->d_area, area.size() * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  const size_t ncell = (size_t)nx * ny * ng;
  TRT_CUDA(cudaMemcpyAsync(c->d_kap64, KapE_in, ncell * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaMemcpyAsync(c->d_kap, c->d_kap64, ncell * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  c->c = cl;
  c->dt = Delt;
  c->have_material = true;
  if ((rc = pack_corner_array<double>(c, I_crn_old, c->d_state[c->cur]))) return rc;
  if (!c->d_srcfull && (rc = c->dalloc(&c->d_srcfull, (size_t)c->state_elems() * c->esz()))) return rc;
  if ((rc = pack_corner_array<double>(c, Src_in, c->d_srcfull))) return rc;
  c->use_srcfull = true;
  if ((rc = set_boundary_impl<double>(c, Ic_edgV, Ic_edgH))) return rc;
  // the caller's I_edgV/I_edgH on inflow faces are not written by TRANSPORT_SCB: keep them
  const int q = nm / 4;
  std::vector<double> keepV((size_t)2 * ny * nm * ng), keepH((size_t)2 * nx * nm * ng);
  for (int g = 0; g < ng; ++g)
    for (int m = 0; m < nm; ++m) {
      const bool xpos = (m < q || m >= 3 * q), ypos = (m < 2 * q);
      for (int j = 0; j < ny; ++j)
        keepV[(size_t)(g * nm + m) * ny + j] =
            I_edgV[(xpos ? 0 : nx) + (size_t)(nx + 1) * (j + (size_t)ny * (m + (size_t)nm * g))];
      for (int i = 0; i < nx; ++i)
        keepH[(size_t)(g * nm + m) * nx + i] =
            I_edgH[i + (size_t)nx * ((ypos ? 0 : ny) + (size_t)(ny + 1) * (m + (size_t)nm * g))];
    }
  unsigned flags = Res_Calc ? TRT_RES_CALC : 0u;
  if ((rc = sweep_impl<double>(c, flags))) return rc;
  if ((rc = check_err(c))) return rc;
  if ((rc = unpack_corner_array<double>(c, c->d_state[1 - c->cur], I_crn))) return rc;
  if ((rc = get_angular_impl<double>(c, I_avg, I_edgV, I_edgH, Ic_edgV, Ic_edgH))) return rc;
  for (int g = 0; g < ng; ++g)
    for (int m = 0; m < nm; ++m) {
      const bool xpos = (m < q || m >= 3 * q), ypos = (m < 2 * q);
      for (int j = 0; j < ny; ++j)
        I_edgV[(xpos ? 0 : nx) + (size_t)(nx + 1) * (j + (size_t)ny * (m + (size_t)nm * g))] =
            keepV[(size_t)(g * nm + m) * ny + j];
      for (int i = 0; i < nx; ++i)
        I_edgH[i + (size_t)nx * ((ypos ? 0 : ny) + (size_t)(ny + 1) * (m + (size_t)nm * g))] =
            keepH[(size_t)(g * nm + m) * nx + i];
    }
  if (Res_Calc) {
    // cells not updated by the reference keep the caller's RT_ResLoc values: read them first
    std::vector<int> lx(RT_ResLoc_x, RT_ResLoc_x + 20 * ng), ly(RT_ResLoc_y, RT_ResLoc_y + 20 * ng);
    TRT_CUDA(cudaMemcpyAsync(c->d_resx, lx.data(), lx.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    TRT_CUDA(cudaMemcpyAsync(c->d_resy, ly.data(), ly.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    trt::residual_reduce_kernel<<<(4 * ng + 63) / 64, 64, 0, c->stream>>>(nx, ny, nm, ng, c->d_res_m, c->d_res_loc,
                                                                         c->d_res, c->d_resx, c->d_resy);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    TRT_CUDA(cudaMemcpyAsync(RT_Residual, c->d_res, 20 * ng * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(cudaMemcpyAsync(RT_ResLoc_x, c->d_resx, 20 * ng * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(cudaMemcpyAsync(RT_ResLoc_y, c->d_resy, 20 * ng * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    TRT_CUDA(cudaStreamSynchronize(c->stream));
  }
  return TRT_OK;
}

// Cached handle for the reference-signature entry points, keyed by shape and directions.
struct DropinCache {
  std::mutex mu;
  trt_ctx* ctx = nullptr;
  std::vector<double> key;
} g_cache;

trt_ctx* cached_ctx(int nx, int ny, int nm, int ng, const double* ox, const double* oy, const double* dx,
                    const double* dy, int* rc) {
  std::vector<double> key = {(double)nx, (double)ny, (double)nm, (double)ng};
  key.insert(key.end(), ox, ox + nm);
  key.insert(key.end(), oy, oy + nm);
  key.insert(key.end(), dx, dx + nx);
  key.insert(key.end(), dy, dy + ny);
  if (g_cache.ctx && g_cache.key == key) {
    *rc = TRT_OK;
    return g_cache.ctx;
  }
  if (g_cache.ctx) trt_destroy(g_cache.ctx);
  g_cache.ctx = nullptr;
  std::vector<double> w(nm, 1.0);
  trt_ctx* c = trt_create(nx, ny, nm, ng, ox, oy, w.data(), dx, dy, TRT_PREC_FP64, 0, rc);
  if (!c) return nullptr;
  g_cache.ctx = c;
  g_cache.key = key;
  return c;
}

// Scoped device buffer for the stateless entry points.
struct DBuf {
  double* p = nullptr;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t n) {
    if (cudaMalloc(&p, (n ? n : 1) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return TRT_ERR_NOMEM;
    }
    return TRT_OK;
  }
  int put(const double* h, size_t n) {
    int rc = alloc(n);
    if (rc) return rc;
    return cudaMemcpy(p, h, n * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess ? TRT_OK : TRT_ERR_CUDA;
  }
  int get(double* h, size_t n) const {
    return cudaMemcpy(h, p, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess ? TRT_OK : TRT_ERR_CUDA;
  }
};

// ---------------------------------------------------------------------------------------------
// Transport-only time step (run_type 'tr_no_qd', ALGORITHMS.f08:389-421, 524-572, 662-668, 816-836).
// ---------------------------------------------------------------------------------------------

// MATERIAL_UPDATE (UPDATES.f08:110-152) from the device temperature into the sweep's material.
template <class Real>
int material_update_impl(trt_ctx* c, double* mgsrc = nullptr) {
  const long long n = (long long)c->nx * c->ny * c->ng;
  trt::material_update_kernel<Real><<<grid_for(n), 256, 0, c->stream>>>(
      c->nx, c->ny, c->ng, c->d_T, c->d_nu, c->d_kmult, c->comp_unit, c->d_kap64, c->d_q64, (Real*)c->d_kap,
      (Real*)c->d_q, mgsrc, c->ts_law);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  c->use_srcfull = false;
  c->have_material = true;
  return TRT_OK;
}

// CONVERGENCE (CONVERGENCE_CHECKS.f08:7-44) from the reduced data {max|x-xo|, max|xo-xo2|, max|x|,
// min|x|, max|1-xo/x|}.
bool convergence(int conv_type, double eps, const double* r, int its, double* norm) {
  const double rho = its > 1 ? r[0] / r[1] : 2.0;
  double nrm = 0.0;
  if (conv_type == 1) nrm = r[0] / r[2];
  else if (conv_type == 2) nrm = r[4];
  else nrm = r[0] / r[3];
  *norm = nrm;
  const double new_eps = std::fabs(1.0 / rho - 1.0) * eps;
  return !(nrm > new_eps);
}

// Phases of one time step of the transport-only loop, shared by the single-handle and batched drivers.
// Start of a step: Temp_old <- Temp (ALGORITHMS.f08:395-396) and the outer-iteration history reset
// (:518-521).
int tstep_begin(trt_ctx* c) {
  const size_t bytes = (size_t)c->nx * c->ny * sizeof(double);
  TRT_CUDA(cudaMemcpyAsync(c->d_Told, c->d_T, bytes, cudaMemcpyDeviceToDevice, c->stream));
  for (double* p : {c->d_Trt1, c->d_Trt2, c->d_Ert1, c->d_Ert2}) TRT_CUDA(cudaMemsetAsync(p, 0, bytes, c->stream));
  return TRT_OK;
}

// After an outer iteration's sweep and moments: RT_BC_UPDATE on reflective sides, MEB_SOLVE with the
// transport group energies (:666), MATERIAL_UPDATE (:668) and the convergence reductions of T and the
// transport E (:816-818), whose 10 values are copied to `host` (read after the stream synchronises).
template <class Real>
int tstep_after_sweep(trt_ctx* c, unsigned long long* host) {
  const size_t nxy = (size_t)c->nx * c->ny;
  const bool reflective = c->ts_bc[0] > 0 || c->ts_bc[1] > 0 || c->ts_bc[2] > 0 || c->ts_bc[3] > 0;
  int rc;
  if (reflective && (rc = bc_update_impl<Real>(c, c->ts_bc, c->ts_Tb, c->comp_unit, c->ts_nu.data()))) return rc;
  if (c->ts_law == trt::kLawConfig)
    trt::meb_law_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>(c->nx, c->ny, c->ng, c->dout.Eg_avg,
                                                                          c->d_kap64, c->d_Told, c->d_cv, c->d_nu,
                                                                          c->dt, c->comp_unit, c->c, c->d_T);
  else
    trt::meb_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>(c->nx, c->ny, c->ng, c->dout.Eg_avg, c->d_kap64,
                                                                      c->d_Told, c->d_cv, c->dt, c->ts_Kap0,
                                                                      c->comp_unit, c->d_T);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  if ((rc = material_update_impl<Real>(c))) return rc;
  static const unsigned long long init[10] = {0, 0, 0, 0x7ff0000000000000ULL, 0, 0, 0, 0, 0x7ff0000000000000ULL, 0};
  TRT_CUDA(cudaMemcpyAsync(c->d_conv, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  trt::conv_reduce_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>((long long)nxy, c->d_T, c->d_Trt1,
                                                                            c->d_Trt2, c->d_conv);
  TRT_LAUNCHED();
  trt::conv_reduce_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>((long long)nxy, c->dout.E_avg, c->d_Ert1,
                                                                            c->d_Ert2, c->d_conv + 5);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  TRT_CUDA(cudaMemcpyAsync(host, c->d_conv, 10 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  return TRT_OK;
}

// With the reductions on the host: CONVERGENCE of T and E, then current iterate -> last iterate (:834-837).
bool tstep_decide(trt_ctx* c, const unsigned long long* host, int its, double* tn, double* en) {
  double r[10];
  std::memcpy(r, host, sizeof(r));
  const bool tconv = convergence(c->ts_conv_type, c->ts_conv_ho, r, its, tn);
  const bool econv = convergence(c->ts_conv_type, c->ts_conv_ho, r + 5, its, en);
  const size_t bytes = (size_t)c->nx * c->ny * sizeof(double);
  cudaMemcpyAsync(c->d_Ert2, c->d_Ert1, bytes, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_Ert1, c->dout.E_avg, bytes, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_Trt2, c->d_Trt1, bytes, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_Trt1, c->d_T, bytes, cudaMemcpyDeviceToDevice, c->stream);
  return tconv && econv;
}

// Group-partial time step (trt_tstep_partials / trt_tstep_finish): the energy balance from group sums that
// the caller has added over every handle that holds a share of the groups.
int tstep_partials_impl(trt_ctx* c, double* part) {
  const size_t nxy = (size_t)c->nx * c->ny;
  trt::meb_partial_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>(c->nx, c->ny, c->ng, c->ts_law,
                                                                            c->dout.Eg_avg, c->d_kap64, c->d_T,
                                                                            c->d_nu, c->comp_unit, c->c, part);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  return TRT_OK;
}

template <class Real>
int tstep_finish_impl(trt_ctx* c, const double* sum, int its, int* conv_out, double* tn, double* en) {
  const size_t nxy = (size_t)c->nx * c->ny;
  trt::meb_finish_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>(c->nx, c->ny, c->ts_law, sum, c->d_Told,
                                                                           c->d_cv, c->dt, c->ts_Kap0, c->comp_unit,
                                                                           c->d_T, c->dout.E_avg);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  int rc = material_update_impl<Real>(c);
  if (rc) return rc;
  static const unsigned long long init[10] = {0, 0, 0, 0x7ff0000000000000ULL, 0, 0, 0, 0, 0x7ff0000000000000ULL, 0};
  TRT_CUDA(cudaMemcpyAsync(c->d_conv, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  trt::conv_reduce_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>((long long)nxy, c->d_T, c->d_Trt1,
                                                                            c->d_Trt2, c->d_conv);
  TRT_LAUNCHED();
  trt::conv_reduce_kernel<<<grid_for((long long)nxy), 256, 0, c->stream>>>((long long)nxy, c->dout.E_avg, c->d_Ert1,
                                                                            c->d_Ert2, c->d_conv + 5);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  unsigned long long h[10];
  TRT_CUDA(cudaMemcpyAsync(h, c->d_conv, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  if ((rc = check_err(c))) return rc;
  const bool conv = tstep_decide(c, h, its, tn, en);
  if (conv_out) *conv_out = conv ? 1 : 0;
  return TRT_OK;
}

template <class Real>
int tstep_impl(trt_ctx* c, int* its_out, double* tnorm_out, double* enorm_out) {
  int rc = tstep_begin(c);
  if (rc) return rc;
  int its = 0;
  bool conv = false;
  double tn = 0.0, en = 0.0;
  unsigned long long h[10];
  while (!conv && its < c->ts_maxit) {
    ++its;
    // RTE solve with the collapse, fg and Cg (:547-569); I_crn_old <- I_crn only on the first
    if ((rc = sweep_impl<Real>(c, (its == 1 ? TRT_ROLL_STATE : 0u) | TRT_MOMENTS))) return rc;
    if ((rc = tstep_after_sweep<Real>(c, h))) return rc;
    TRT_CUDA(cudaStreamSynchronize(c->stream));
    if ((rc = check_err(c))) return rc;
    conv = tstep_decide(c, h, its, &tn, &en);
  }
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  if (its_out) *its_out = its;
  if (tnorm_out) *tnorm_out = tn;
  if (enorm_out) *enorm_out = en;
  return TRT_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Batched instances: one sweep launch per tiling class over the CTAs of many handles.
// ---------------------------------------------------------------------------------------------
struct trt_batch {
  std::vector<trt_ctx*> h;
  cudaStream_t stream = nullptr;             // epilogues and the time-loop kernels of every handle
  std::vector<cudaStream_t> gstreams;        // one per launch group (their sweeps overlap)
  std::vector<cudaEvent_t> gevents;
  cudaEvent_t start = nullptr;
  void* d_args = nullptr;                    // SweepArgs of every handle, grouped
  size_t d_args_cap = 0;
  int* d_first = nullptr;                    // first CTA of each handle in its group's launch
  size_t d_first_cap = 0;
  bool persistent = true;                    // classes without band CTAs: one wave of CTAs drains a task queue
  int* d_queue = nullptr;                    // task counter of each launch group
  size_t d_queue_cap = 0;
  unsigned char* h_args = nullptr;           // pinned staging of d_args / d_first
  size_t h_args_cap = 0;
  unsigned long long* h_norms = nullptr;     // pinned, 10 convergence values per handle
  int* h_err = nullptr;                      // pinned, error word of each handle
  std::vector<cudaStream_t> estreams;        // the per-handle work after a batched sweep, spread over these
  std::vector<cudaEvent_t> eevents;
};

namespace {

// Run a handle's own calls on another stream for the lifetime of this object.
struct StreamSwap {
  trt_ctx* c;
  cudaStream_t old;
  StreamSwap(trt_ctx* ctx, cudaStream_t s) : c(ctx), old(ctx->stream) { c->stream = s; }
  ~StreamSwap() { c->stream = old; }
};

template <class Real>
int batch_group_launch(trt_batch* b, std::vector<trt_ctx*>& grp, size_t args_off, size_t first_off, size_t done,
                       cudaStream_t gs, size_t qslot) {
  // largest CTAs first: the block scheduler then starts the long sweeps before the short ones
  std::stable_sort(grp.begin(), grp.end(), [](const trt_ctx* x, const trt_ctx* y) {
    return (long long)x->t.Tb * x->t.D > (long long)y->t.Tb * y->t.D;
  });
  auto* ha = reinterpret_cast<trt::SweepArgs<Real>*>(b->h_args + args_off);
  auto* hf = reinterpret_cast<int*>(b->h_args + first_off);
  long long total = 0;
  size_t smem = 0;
  for (size_t k = 0; k < grp.size(); ++k) {
    ha[k] = make_sweep_args<Real>(grp[k]);
    hf[k] = (int)total;
    total += 4LL * grp[k]->ng * grp[k]->t.NH * grp[k]->t.NB;
    smem = std::max(smem, sweep_smem<Real>(grp[k]));
    grp[k]->swept = true;
  }
  if (total > (1LL << 30)) return TRT_ERR_ARG;
  auto* da = reinterpret_cast<trt::SweepArgs<Real>*>(static_cast<unsigned char*>(b->d_args) + args_off);
  int* df = b->d_first + done;   // the device copy holds only the first-CTA table
  TRT_CUDA(cudaMemcpyAsync(da, ha, grp.size() * sizeof(trt::SweepArgs<Real>), cudaMemcpyHostToDevice, gs));
  TRT_CUDA(cudaMemcpyAsync(df, hf, grp.size() * sizeof(int), cudaMemcpyHostToDevice, gs));
  // the up-to-170-register variant when every CTA of the launch is resident at once with it
  int level = 0;
  if (32 * grp[0]->t.W <= 128 && !grp[0]->use_srcfull) {
    SweepBatchKernel<Real> k1 = sweep_batch_kernel_for<Real>(grp[0]->kc, false, 1);
    int per = 0;
    if (k1 && cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k1, 32 * grp[0]->t.W, smem) == cudaSuccess &&
        total <= (long long)per * sm_count())
      level = 1;
    cudaGetLastError();
  }
  if (b->persistent && grp[0]->t.NB == 1) {
    // one wave of resident CTAs that drains the (instance, group, quadrant, split) queue in the table's order
    SweepQueueKernel<Real> kq = sweep_queue_kernel_for<Real>(grp[0]->kc, grp[0]->use_srcfull, level);
    if (!kq) return TRT_ERR_UNSUPPORTED;
    cudaFuncSetAttribute(kq, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kq, 32 * grp[0]->t.W, smem) != cudaSuccess || per < 1) {
      cudaGetLastError();
      per = 1;
    }
    const long long grid = std::min<long long>(total, (long long)per * sm_count());
    int* q = b->d_queue + qslot;
    TRT_CUDA(cudaMemsetAsync(q, 0, sizeof(int), gs));
    kq<<<(unsigned)grid, 32 * grp[0]->t.W, smem, gs>>>(da, df, (int)grp.size(), (int)total, q);
    TRT_LAUNCHED();
    TRT_CUDA(cudaGetLastError());
    return TRT_OK;
  }
  SweepBatchKernel<Real> k = sweep_batch_kernel_for<Real>(grp[0]->kc, grp[0]->use_srcfull, level);
  if (!k) return TRT_ERR_UNSUPPORTED;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  TRT_CUDA(launch_banded(k, grp[0]->t.NB, (int)total, 32 * grp[0]->t.W, smem, gs, (const trt::SweepArgs<Real>*)da,
                         (const int*)df, (int)grp.size()));
  TRT_LAUNCHED();
  return TRT_OK;
}

// Sweep the handles act (rolling the state of those with roll[k]) in one launch per tiling class;
// on return b->stream is ordered after every sweep.
int batch_sweep_launch(trt_batch* b, const std::vector<int>& act, const std::vector<char>& roll) {
  TRT_CUDA(cudaStreamSynchronize(b->stream));   // the staging buffers of the previous launch are free
  struct Key {
    int prec, S, D, W, stages, srcfull, NB;
    bool operator==(const Key& o) const {
      return prec == o.prec && S == o.S && D == o.D && W == o.W && stages == o.stages && srcfull == o.srcfull &&
             NB == o.NB;
    }
  };
  std::vector<Key> keys;
  std::vector<std::vector<trt_ctx*>> groups;
  for (size_t i = 0; i < act.size(); ++i) {
    trt_ctx* c = b->h[act[i]];
    if (roll[i]) c->cur = 1 - c->cur;   // I_crn_old <- I_crn (ALGORITHMS.f08:397)
    const Key key{c->prec, c->kc.S, c->kc.D, c->t.W, c->stages, c->use_srcfull ? 1 : 0, c->t.NB};
    size_t g = 0;
    while (g < keys.size() && !(keys[g] == key)) ++g;
    if (g == keys.size()) {
      keys.push_back(key);
      groups.emplace_back();
    }
    groups[g].push_back(c);
  }
  // staging: args (max of both precisions' struct sizes) then first indices, per group
  const size_t asz = std::max(sizeof(trt::SweepArgs<double>), sizeof(trt::SweepArgs<float>));
  const size_t args_bytes = (act.size() * asz + 255) & ~size_t(255);
  const size_t need = args_bytes + act.size() * sizeof(int) + 256;
  if (need > b->h_args_cap) {
    if (b->h_args) cudaFreeHost(b->h_args);
    b->h_args = nullptr;
    if (cudaMallocHost((void**)&b->h_args, need) != cudaSuccess) {
      cudaGetLastError();
      b->h_args_cap = 0;
      return TRT_ERR_NOMEM;
    }
    b->h_args_cap = need;
  }
  if (args_bytes > b->d_args_cap) {
    if (b->d_args) cudaFree(b->d_args);
    if (cudaMalloc(&b->d_args, args_bytes) != cudaSuccess) {
      cudaGetLastError();
      b->d_args = nullptr;
      b->d_args_cap = 0;
      return TRT_ERR_NOMEM;
    }
    b->d_args_cap = args_bytes;
  }
  if (act.size() * sizeof(int) > b->d_first_cap) {
    if (b->d_first) cudaFree(b->d_first);
    if (cudaMalloc((void**)&b->d_first, act.size() * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      b->d_first = nullptr;
      b->d_first_cap = 0;
      return TRT_ERR_NOMEM;
    }
    b->d_first_cap = act.size() * sizeof(int);
  }
  if (groups.size() > b->d_queue_cap) {
    if (b->d_queue) cudaFree(b->d_queue);
    if (cudaMalloc((void**)&b->d_queue, groups.size() * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      b->d_queue = nullptr;
      b->d_queue_cap = 0;
      return TRT_ERR_NOMEM;
    }
    b->d_queue_cap = groups.size();
  }
  while (b->gstreams.size() < groups.size()) {
    cudaStream_t st;
    cudaEvent_t ev;
    TRT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    TRT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->gstreams.push_back(st);
    b->gevents.push_back(ev);
  }
  TRT_CUDA(cudaEventRecord(b->start, b->stream));
  size_t done = 0;
  for (size_t g = 0; g < groups.size(); ++g) {
    cudaStream_t gs = b->gstreams[g];
    TRT_CUDA(cudaStreamWaitEvent(gs, b->start, 0));
    const size_t args_off = done * asz, first_off = args_bytes + done * sizeof(int);
    int rc = keys[g].prec == TRT_PREC_FP64 ? batch_group_launch<double>(b, groups[g], args_off, first_off, done, gs, g)
                                           : batch_group_launch<float>(b, groups[g], args_off, first_off, done, gs, g);
    if (rc) return rc;
    done += groups[g].size();
    TRT_CUDA(cudaEventRecord(b->gevents[g], gs));
    TRT_CUDA(cudaStreamWaitEvent(b->stream, b->gevents[g], 0));
  }
  return TRT_OK;
}

int batch_prepare(trt_batch* b, bool tstep) {
  for (trt_ctx* c : b->h) {
    if (tstep ? !c->ts_ready : !c->have_material) return TRT_ERR_STATE;
    if (!c->have_state && !c->swept) return TRT_ERR_STATE;
    TRT_CUDA(cudaStreamSynchronize(c->stream));   // order after the handle's own earlier calls
  }
  return TRT_OK;
}

// Later calls on each handle's own stream wait for the batch's work.
int batch_release(trt_batch* b) {
  TRT_CUDA(cudaEventRecord(b->start, b->stream));
  for (trt_ctx* c : b->h) TRT_CUDA(cudaStreamWaitEvent(c->stream, b->start, 0));
  return TRT_OK;
}

int batch_sweep_impl(trt_batch* b, unsigned flags) {
  int rc = batch_prepare(b, false);
  if (rc) return rc;
  std::vector<int> act(b->h.size());
  for (size_t k = 0; k < act.size(); ++k) act[k] = (int)k;
  std::vector<char> roll(act.size(), (flags & TRT_ROLL_STATE) ? 1 : 0);
  if ((rc = batch_sweep_launch(b, act, roll))) return rc;
  for (trt_ctx* c : b->h) {
    StreamSwap sw(c, b->stream);
    rc = c->prec == TRT_PREC_FP64 ? sweep_epilogue<double>(c, flags & ~TRT_ROLL_STATE)
                                  : sweep_epilogue<float>(c, flags & ~TRT_ROLL_STATE);
    if (rc) return rc;
  }
  return batch_release(b);
}

int batch_tstep_impl(trt_batch* b, int* its_out, double* tn_out, double* en_out) {
  int rc = batch_prepare(b, true);
  if (rc) return rc;
  const size_t n = b->h.size();
  std::vector<StreamSwap> swaps;
  swaps.reserve(n);
  for (trt_ctx* c : b->h) swaps.emplace_back(c, b->stream);
  for (trt_ctx* c : b->h)
    if ((rc = tstep_begin(c))) return rc;
  std::vector<int> its(n, 0), act(n);
  std::vector<double> tn(n, 0.0), en(n, 0.0);
  for (size_t k = 0; k < n; ++k) act[k] = (int)k;
  while (!act.empty()) {
    std::vector<char> roll(act.size());
    for (size_t i = 0; i < act.size(); ++i) roll[i] = (++its[act[i]] == 1) ? 1 : 0;
    if ((rc = batch_sweep_launch(b, act, roll))) return rc;
    // each handle's epilogue, MEB, material update and reductions on one of the epilogue streams, so the
    // small kernels of different handles overlap; one synchronisation for all
    TRT_CUDA(cudaEventRecord(b->start, b->stream));
    for (cudaStream_t es : b->estreams) TRT_CUDA(cudaStreamWaitEvent(es, b->start, 0));
    for (size_t i = 0; i < act.size(); ++i) {
      const int k = act[i];
      trt_ctx* c = b->h[k];
      StreamSwap sw(c, b->estreams[i % b->estreams.size()]);
      rc = c->prec == TRT_PREC_FP64 ? sweep_epilogue<double>(c, TRT_MOMENTS) : sweep_epilogue<float>(c, TRT_MOMENTS);
      if (!rc) rc = c->prec == TRT_PREC_FP64 ? tstep_after_sweep<double>(c, b->h_norms + 10 * k)
                                             : tstep_after_sweep<float>(c, b->h_norms + 10 * k);
      if (rc) return rc;
      TRT_CUDA(cudaMemcpyAsync(b->h_err + k, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    }
    for (size_t e = 0; e < b->estreams.size(); ++e) {
      TRT_CUDA(cudaEventRecord(b->eevents[e], b->estreams[e]));
      TRT_CUDA(cudaStreamWaitEvent(b->stream, b->eevents[e], 0));
    }
    TRT_CUDA(cudaStreamSynchronize(b->stream));
    std::vector<int> next;
    for (int k : act) {
      trt_ctx* c = b->h[k];
      if (b->h_err[k]) {   // a bounded wait of this handle's sweep gave up (see check_err)
        TRT_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
        TRT_CUDA(cudaStreamSynchronize(c->stream));
        return TRT_ERR_TIMEOUT;
      }
      const bool conv = tstep_decide(c, b->h_norms + 10 * k, its[k], &tn[k], &en[k]);
      if (!conv && its[k] < c->ts_maxit) next.push_back(k);
    }
    act.swap(next);
  }
  TRT_CUDA(cudaStreamSynchronize(b->stream));
  for (size_t k = 0; k < n; ++k) {
    if (its_out) its_out[k] = its[k];
    if (tn_out) tn_out[k] = tn[k];
    if (en_out) en_out[k] = en[k];
  }
  swaps.clear();
  return batch_release(b);
}

}  // namespace

extern "C" {

trt_batch* trt_batch_create(trt_ctx* const* handles, int n, int* status) {
  int dummy;
  if (!status) status = &dummy;
  if (!handles || n < 1) {
    *status = TRT_ERR_ARG;
    return nullptr;
  }
  for (int k = 0; k < n; ++k)
    for (int j = 0; j <= k; ++j)
      if (!handles[k] || (j < k && handles[j] == handles[k])) {
        *status = TRT_ERR_ARG;
        return nullptr;
      }
  trt_batch* b = new (std::nothrow) trt_batch();
  if (!b) {
    *status = TRT_ERR_NOMEM;
    return nullptr;
  }
  b->h.assign(handles, handles + n);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost((void**)&b->h_norms, (size_t)10 * n * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost((void**)&b->h_err, (size_t)n * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    trt_batch_destroy(b);
    *status = TRT_ERR_CUDA;
    return nullptr;
  }
  for (int k = 0; k < 8 && k < n; ++k) {
    cudaStream_t st;
    cudaEvent_t ev;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      trt_batch_destroy(b);
      *status = TRT_ERR_CUDA;
      return nullptr;
    }
    b->estreams.push_back(st);
    b->eevents.push_back(ev);
  }
  *status = TRT_OK;
  return b;
}

void trt_batch_destroy(trt_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (cudaStream_t s : b->gstreams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : b->gevents) cudaEventDestroy(e);
  for (cudaStream_t s : b->estreams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : b->eevents) cudaEventDestroy(e);
  if (b->h_err) cudaFreeHost(b->h_err);
  if (b->start) cudaEventDestroy(b->start);
  if (b->d_args) cudaFree(b->d_args);
  if (b->d_queue) cudaFree(b->d_queue);
  if (b->d_first) cudaFree(b->d_first);
  if (b->h_args) cudaFreeHost(b->h_args);
  if (b->h_norms) cudaFreeHost(b->h_norms);
  if (b->stream) cudaStreamDestroy(b->stream);
  cudaGetLastError();
  delete b;
}

int trt_batch_sweep(trt_batch* b, unsigned flags) {
  if (!b) return TRT_ERR_ARG;
  return batch_sweep_impl(b, flags);
}

int trt_batch_set_persistent(trt_batch* b, int on) {
  if (!b || (on != 0 && on != 1)) return TRT_ERR_ARG;
  b->persistent = on == 1;
  return TRT_OK;
}

int trt_batch_sync(trt_batch* b) {
  if (!b) return TRT_ERR_ARG;
  TRT_CUDA(cudaStreamSynchronize(b->stream));
  for (trt_ctx* c : b->h) {
    int rc = check_err(c);
    if (rc) return rc;
  }
  return TRT_OK;
}

int trt_batch_tstep(trt_batch* b, int* rt_its, double* T_norms, double* E_norms) {
  if (!b) return TRT_ERR_ARG;
  return batch_tstep_impl(b, rt_its, T_norms, E_norms);
}

const char* trt_strerror(int code) {
  switch (code) {
    case TRT_OK: return "ok";
    case TRT_ERR_ARG: return "invalid argument or array extent";
    case TRT_ERR_CUDA: return "CUDA runtime error";
    case TRT_ERR_NOMEM: return "device memory allocation failed";
    case TRT_ERR_BUDGET: return "request exceeds the device-memory budget of the handle";
    case TRT_ERR_TIMEOUT: return "a bounded device-side wait gave up (the handle stays usable)";
    case TRT_ERR_STATE: return "call order: a required input has not been set";
    case TRT_ERR_NODEV: return "no CUDA device available";
    case TRT_ERR_UNSUPPORTED: return "shape outside the compiled kernel set";
    case TRT_ERR_SCRATCH: return "problem exceeds the fixed scratch of the no-allocation entry point (n_m*n_g > 65536)";
    case TRT_ERR_NOCONV: return "the low-order linear solve of a group stopped without converging";
    default: return "unknown error";
  }
}

unsigned long long trt_kernel_launches(void) { return g_launches.load(); }

double trt_bg_planck(double T, double nu_low, double nu_high, double Comp_Unit) {
  return bg_planck_h(T, nu_low, nu_high, Comp_Unit);
}

size_t trt_required_bytes(int n_x, int n_y, int n_m, int n_g, int precision) {
  if (!valid_shape(n_x, n_y, n_m, n_g)) return 0;
  const int mq = n_m / 4;
  KernelCfg kc;
  if (!pick_cfg(mq, precision, 0, &kc)) return 0;
  const size_t esz = precision == TRT_PREC_FP64 ? 8 : 4;
  int NH = 1, W = 8;
  default_split(n_g, mq, &NH, &W, (size_t)4 * n_g * n_x * n_y * (precision == TRT_PREC_FP64 ? 112 : 64));
  if (!pick_cfg((mq + NH - 1) / NH, precision, 0, &kc)) return 0;
  W = default_W(32 / kc.S, n_y, W);
  const int mqc = (mq + NH - 1) / NH;
  size_t b = 2 * layout_state_bytes(n_x, n_y, mq, n_g, W, kc.S, NH, esz);   // I_crn_old, I_crn
  const size_t ncell = (size_t)n_x * n_y * n_g;
  b += ncell * (16 + 2 * esz);
  b += (size_t)2 * n_g * n_m * 2 * (n_x + n_y) * esz;
  b += (size_t)4 * n_g * NH * n_x * mqc * 2 * esz;
  b += (size_t)4 * NH * n_g * n_x * n_y * (precision == TRT_PREC_FP64 ? 112 : 64);   // partial records
  long long sz[kNOut];
  output_sizes(n_x, n_y, n_g, sz);
  for (int k = 0; k < kNOut; ++k) b += sz[k] * 8;
  b += (size_t)4 * n_x * n_y * n_m * 8;   // staging slab
  return b + (1 << 20);
}

trt_ctx* trt_create(int n_x, int n_y, int n_m, int n_g, const double* Omega_x, const double* Omega_y,
                    const double* quad_weight, const double* Delx, const double* Dely, int precision,
                    size_t hbm_budget, int* status) {
  int dummy;
  if (!status) status = &dummy;
  const bool inplace = (precision & TRT_CREATE_INPLACE) != 0;
  precision &= ~TRT_CREATE_INPLACE;
  if (!valid_shape(n_x, n_y, n_m, n_g) || !Omega_x || !Omega_y || !quad_weight || !Delx || !Dely ||
      (precision != TRT_PREC_FP64 && precision != TRT_PREC_FP32)) {
    *status = TRT_ERR_ARG;
    return nullptr;
  }
  if ((*status = device_check())) return nullptr;
  trt_ctx* c = new (std::nothrow) trt_ctx();
  if (!c) {
    *status = TRT_ERR_NOMEM;
    return nullptr;
  }
  c->nx = n_x; c->ny = n_y; c->nm = n_m; c->ng = n_g; c->mq = n_m / 4;
  c->prec = precision;
  c->inplace = inplace;   // one state buffer from the start (an instance whose two buffers would not fit)
  c->budget = hbm_budget;
  c->omx.assign(Omega_x, Omega_x + n_m);
  c->omy.assign(Omega_y, Omega_y + n_m);
  c->w.assign(quad_weight, quad_weight + n_m);
  c->dx.assign(Delx, Delx + n_x);
  c->dy.assign(Dely, Dely + n_y);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    *status = TRT_ERR_CUDA;
    return nullptr;
  }
  int rc = create_buffers(c);
  if (rc == TRT_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = TRT_ERR_CUDA;
  if (rc) {
    trt_destroy(c);
    *status = rc;
    return nullptr;
  }
  *status = TRT_OK;
  return c;
}

void trt_destroy(trt_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (cudaStream_t q : {c->s_in, c->s_out})
    if (q) {
      cudaStreamSynchronize(q);
      cudaStreamDestroy(q);
    }
  for (cudaEvent_t e : {c->ev_staged, c->ev_stage_free, c->ev_epi, c->ev_out})
    if (e) cudaEventDestroy(e);
  if (c->lo && c->lo_free) c->lo_free(c->lo);
  for (void* p : c->allocs) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int trt_autotune(trt_ctx* c, int* warps_out, int* slices_out, int* splits_out, float* ms_out) {
  if (!c) return TRT_ERR_ARG;
  const bool had_material = c->have_material;
  const size_t ncell = (size_t)c->nx * c->ny * c->ng;
  if (!had_material) {   // trial sweeps on a zero material
    TRT_CUDA(cudaMemsetAsync(c->d_kap, 0, ncell * c->esz(), c->stream));
    TRT_CUDA(cudaMemsetAsync(c->d_q, 0, ncell * c->esz(), c->stream));
  }
  cudaEvent_t e0, e1;
  TRT_CUDA(cudaEventCreate(&e0));
  TRT_CUDA(cudaEventCreate(&e1));
  const int sms = sm_count();
  int bestNH = 0, bestW = 0, bestNB = 1;
  float best = 0.0f;
  const int nhs[] = {1, 2, 3, 4}, ws[] = {2, 3, 4, 5, 6, 8}, nbs[] = {1, 2, 4};
  for (int NH : nhs) {
    if (NH > c->mq) continue;
    for (int W : ws)
    for (int NB : nbs) {
      c->NHreq = NH;
      c->Wreq = W;
      c->NBreq = NB;
      c->Sreq = 0;
      c->stages = 2;
      if (setup_layout(c) != TRT_OK || c->t.NB != NB) continue;
      // only tilings whose CTAs are all resident at once
      const size_t smem = c->prec == TRT_PREC_FP64
                              ? trt::sweep_smem_bytes<double>(c->t.W, c->chunk, c->stages, c->t.mqc, c->t.D, c->t.S)
                              : trt::sweep_smem_bytes<float>(c->t.W, c->chunk, c->stages, c->t.mqc, c->t.D, c->t.S);
      const int per = c->prec == TRT_PREC_FP64 ? sweep_ctas_per_sm<double>(c->kc, 32 * c->t.W, smem, c->regs)
                                               : sweep_ctas_per_sm<float>(c->kc, 32 * c->t.W, smem, c->regs);
      if (per <= 0 || 4LL * c->ng * NH * c->t.NB > (long long)per * sms) continue;
      c->have_state = true;
      c->have_material = true;
      const unsigned tf = TRT_ROLL_STATE;   // trial data: rolling changes nothing measured, and in place it must
      int rc = c->prec == TRT_PREC_FP64 ? sweep_impl<double>(c, tf) : sweep_impl<float>(c, tf);
      if (rc) continue;
      TRT_CUDA(cudaEventRecord(e0, c->stream));
      for (int k = 0; k < 2 && !rc; ++k)
        rc = c->prec == TRT_PREC_FP64 ? sweep_impl<double>(c, tf) : sweep_impl<float>(c, tf);
      TRT_CUDA(cudaEventRecord(e1, c->stream));
      TRT_CUDA(cudaStreamSynchronize(c->stream));
      if (rc || check_err(c)) continue;
      float ms = 0.0f;
      TRT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      ms *= 0.5f;
      if (bestNH == 0 || ms < best) {
        best = ms;
        bestNH = NH;
        bestW = W;
        bestNB = NB;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->NHreq = bestNH;
  c->Wreq = bestW;
  c->NBreq = bestNB;
  c->Sreq = 0;
  c->stages = 2;
  int rc = setup_layout(c);
  c->have_state = false;
  c->swept = false;
  c->have_moments = false;
  c->have_material = had_material;
  if (rc) return rc;
  if (!bestNH) return TRT_ERR_UNSUPPORTED;
  if (warps_out) *warps_out = c->t.W;
  if (slices_out) *slices_out = c->t.S;
  if (splits_out) *splits_out = c->t.NH;
  if (ms_out) *ms_out = best;
  return TRT_OK;
}

int trt_set_tiling(trt_ctx* c, int warps_per_cta, int slices, int stages, int splits) {
  if (!c || warps_per_cta < 0 || warps_per_cta > 16 || stages < 0 || stages > 4) return TRT_ERR_ARG;
  if (slices && (slices & (slices - 1))) return TRT_ERR_ARG;
  if (slices > 32 || splits < 0 || splits > c->mq) return TRT_ERR_ARG;
  c->Wreq = warps_per_cta;
  c->Sreq = slices;
  c->NHreq = splits;
  c->stages = stages ? stages : 2;
  return setup_layout(c);
}

int trt_set_inplace(trt_ctx* c, int on) {
  if (!c || (on != 0 && on != 1)) return TRT_ERR_ARG;
  if (c->inplace == (on == 1)) return TRT_OK;
  // release the current buffers under the current mode, then lay out again under the new one
  const size_t sbytes = c->blk ? (size_t)c->state_elems() * c->esz() : 0;
  if (c->ext_state) {
    c->d_state[0] = c->d_state[1] = nullptr;
    c->ext_state = nullptr;
  }
  if (c->d_state[1] == c->d_state[0]) c->d_state[1] = nullptr;
  for (int k = 0; k < 2; ++k) {
    c->dfree(c->d_state[k], sbytes);
    c->d_state[k] = nullptr;
  }
  c->inplace = on == 1;
  return setup_layout(c);
}

size_t trt_state_bytes(const trt_ctx* c) { return c ? (size_t)c->state_elems() * c->esz() : 0; }

int trt_bind_state(trt_ctx* c, void* device_state, size_t bytes) {
  if (!c || !device_state || !c->inplace || bytes < trt_state_bytes(c) ||
      (reinterpret_cast<uintptr_t>(device_state) & 127))
    return TRT_ERR_ARG;
  if (!c->ext_state) c->dfree(c->d_state[0], trt_state_bytes(c));
  c->d_state[0] = c->d_state[1] = device_state;
  c->ext_state = device_state;
  c->have_state = false;
  c->swept = false;
  return TRT_OK;
}

int trt_state_written(trt_ctx* c) {
  if (!c) return TRT_ERR_ARG;
  c->have_state = true;
  c->swept = false;
  return TRT_OK;
}

int trt_snapshot_angular_groups(trt_ctx* c, int g0, int n_groups, float* I_avg_device) {
  if (!c || !I_avg_device || g0 < 0 || n_groups < 1 || g0 + n_groups > c->ng) return TRT_ERR_ARG;
  if (!c->have_state && !c->swept) return TRT_ERR_STATE;
  const void* st = c->d_state[c->swept ? 1 - c->cur : c->cur];
  const long long n = (long long)c->nx * c->ny * c->nm * n_groups;
  if (c->prec == TRT_PREC_FP64)
    trt::snapshot_avg_kernel<double><<<grid_for(n), 256, 0, c->stream>>>(c->geo(), (const double*)st, I_avg_device, g0,
                                                                         n_groups);
  else
    trt::snapshot_avg_kernel<float><<<grid_for(n), 256, 0, c->stream>>>(c->geo(), (const float*)st, I_avg_device, g0,
                                                                        n_groups);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  return TRT_OK;
}

int trt_set_bands(trt_ctx* c, int bands) {
  if (!c || bands < 0 || bands > 8) return TRT_ERR_ARG;
  c->NBreq = bands;
  return setup_layout(c);
}

int trt_get_bands(const trt_ctx* c) { return c ? c->t.NB : TRT_ERR_ARG; }

int trt_set_register_mode(trt_ctx* c, int mode) {
  if (!c || mode < -1 || mode > 2) return TRT_ERR_ARG;
  c->regs_req = mode;
  return setup_layout(c);
}

int trt_get_register_mode(const trt_ctx* c) { return c ? c->regs : TRT_ERR_ARG; }

int trt_get_tiling(const trt_ctx* c, int* W, int* S, int* D, int* stages, int* splits) {
  if (!c) return TRT_ERR_ARG;
  if (W) *W = c->t.W;
  if (S) *S = c->t.S;
  if (D) *D = c->t.D;
  if (stages) *stages = c->stages;
  if (splits) *splits = c->t.NH;
  return TRT_OK;
}

int trt_set_material(trt_ctx* c, const double* KapE_in, const double* src_iso, double cl, double Delt,
                     double Comp_Unit) {
  if (!c || !KapE_in || !src_iso || !(cl > 0) || !(Delt > 0) || !(Comp_Unit > 0)) return TRT_ERR_ARG;
  c->c = cl; c->dt = Delt; c->comp_unit = Comp_Unit;
  int rc = c->prec == TRT_PREC_FP64 ? set_material_impl<double>(c, KapE_in, src_iso, false)
                                    : set_material_impl<float>(c, KapE_in, src_iso, false);
  if (!rc) c->have_material = true;
  return rc;
}

int trt_set_material_device(trt_ctx* c, const double* KapE_in, const double* src_iso, double cl, double Delt,
                            double Comp_Unit) {
  if (!c || !KapE_in || !src_iso || !(cl > 0) || !(Delt > 0) || !(Comp_Unit > 0)) return TRT_ERR_ARG;
  c->c = cl; c->dt = Delt; c->comp_unit = Comp_Unit;
  int rc = c->prec == TRT_PREC_FP64 ? set_material_impl<double>(c, KapE_in, src_iso, true)
                                    : set_material_impl<float>(c, KapE_in, src_iso, true);
  if (!rc) c->have_material = true;
  return rc;
}

int trt_set_source_full(trt_ctx* c, const double* Src_in) {
  if (!c) return TRT_ERR_ARG;
  if (!Src_in) {
    c->use_srcfull = false;
    return TRT_OK;
  }
  const size_t bytes = (size_t)c->state_elems() * c->esz();
  if (!c->d_srcfull) {
    int rc = c->dalloc(&c->d_srcfull, bytes);
    if (rc) return rc;
  }
  int rc = c->prec == TRT_PREC_FP64 ? pack_corner_array<double>(c, Src_in, c->d_srcfull)
                                    : pack_corner_array<float>(c, Src_in, c->d_srcfull);
  if (!rc) c->use_srcfull = true;
  return rc;
}

int trt_set_boundary(trt_ctx* c, const double* Ic_edgV, const double* Ic_edgH, const int* BC_Type) {
  if (!c) return TRT_ERR_ARG;
  if (BC_Type)
    for (int k = 0; k < 4; ++k) c->bc[k] = BC_Type[k];
  return c->prec == TRT_PREC_FP64 ? set_boundary_impl<double>(c, Ic_edgV, Ic_edgH)
                                  : set_boundary_impl<float>(c, Ic_edgV, Ic_edgH);
}

int trt_bc_update(trt_ctx* c, const int* BC_Type, double bcT_left, double bcT_lower, double bcT_right,
                  double bcT_upper, double Comp_Unit, const double* Nu_g) {
  if (!c || !BC_Type || !Nu_g) return TRT_ERR_ARG;
  for (int k = 0; k < 4; ++k) c->bc[k] = BC_Type[k];
  const double Tb[4] = {bcT_left, bcT_lower, bcT_right, bcT_upper};
  return c->prec == TRT_PREC_FP64 ? bc_update_impl<double>(c, BC_Type, Tb, Comp_Unit, Nu_g)
                                  : bc_update_impl<float>(c, BC_Type, Tb, Comp_Unit, Nu_g);
}

int trt_init_state(trt_ctx* c, double Tini, double bcT_left, double bcT_lower, double bcT_right, double bcT_upper,
                   double Comp_Unit, const double* Nu_g) {
  if (!c || !Nu_g || !(Comp_Unit > 0)) return TRT_ERR_ARG;
  c->comp_unit = Comp_Unit;
  const double Tb[4] = {bcT_left, bcT_lower, bcT_right, bcT_upper};
  c->swept = false;
  return c->prec == TRT_PREC_FP64 ? init_state_impl<double>(c, Tini, Tb, Comp_Unit, Nu_g)
                                  : init_state_impl<float>(c, Tini, Tb, Comp_Unit, Nu_g);
}

int trt_put_state(trt_ctx* c, const double* I_crn) {
  if (!c || !I_crn) return TRT_ERR_ARG;
  int rc = c->prec == TRT_PREC_FP64 ? pack_corner_array<double>(c, I_crn, c->d_state[c->cur])
                                    : pack_corner_array<float>(c, I_crn, c->d_state[c->cur]);
  if (!rc) {
    c->have_state = true;
    c->swept = false;
  }
  return rc;
}

int trt_get_state(trt_ctx* c, double* I_crn) {
  if (!c || !I_crn) return TRT_ERR_ARG;
  const void* st = c->d_state[c->swept ? 1 - c->cur : c->cur];
  return c->prec == TRT_PREC_FP64 ? unpack_corner_array<double>(c, st, I_crn)
                                  : unpack_corner_array<float>(c, st, I_crn);
}

int trt_sweep(trt_ctx* c, unsigned flags) {
  if (!c) return TRT_ERR_ARG;
  if (!c->have_material || (!c->have_state && !c->swept)) return TRT_ERR_STATE;
  return c->prec == TRT_PREC_FP64 ? sweep_impl<double>(c, flags) : sweep_impl<float>(c, flags);
}

int trt_sync(trt_ctx* c) {
  if (!c) return TRT_ERR_ARG;
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  for (cudaStream_t q : {c->s_in, c->s_out})
    if (q) TRT_CUDA(cudaStreamSynchronize(q));
  return check_err(c);
}

// Copy streams, events and the staging pair of the pipelined calls (first use).
static int pipe_init(trt_ctx* c) {
  if (c->s_in) return TRT_OK;
  const size_t n = (size_t)c->nx * c->ny * c->ng;
  int rc;
  if ((rc = alloc_t(c, &c->d_kap_in, n)) || (rc = alloc_t(c, &c->d_q_in, n))) return rc;
  for (cudaEvent_t* e : {&c->ev_staged, &c->ev_stage_free, &c->ev_epi, &c->ev_out})
    TRT_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  TRT_CUDA(cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking));
  TRT_CUDA(cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking));
  TRT_CUDA(cudaEventRecord(c->ev_stage_free, c->stream));
  return TRT_OK;
}

int trt_set_material_async(trt_ctx* c, const double* KapE_in, const double* src_iso, double cl, double Delt,
                           double Comp_Unit) {
  if (!c || !KapE_in || !src_iso || !(cl > 0) || !(Delt > 0) || !(Comp_Unit > 0)) return TRT_ERR_ARG;
  int rc = pipe_init(c);
  if (rc) return rc;
  const size_t n = (size_t)c->nx * c->ny * c->ng;
  // host -> staging on the input stream, once the previous material has left the staging pair
  TRT_CUDA(cudaStreamWaitEvent(c->s_in, c->ev_stage_free, 0));
  TRT_CUDA(cudaMemcpyAsync(c->d_kap_in, KapE_in, n * sizeof(double), cudaMemcpyHostToDevice, c->s_in));
  TRT_CUDA(cudaMemcpyAsync(c->d_q_in, src_iso, n * sizeof(double), cudaMemcpyHostToDevice, c->s_in));
  TRT_CUDA(cudaEventRecord(c->ev_staged, c->s_in));
  // staging -> the handle's material, in order on the handle's stream (after every earlier reader)
  TRT_CUDA(cudaStreamWaitEvent(c->stream, c->ev_staged, 0));
  c->c = cl; c->dt = Delt; c->comp_unit = Comp_Unit;
  rc = c->prec == TRT_PREC_FP64 ? set_material_impl<double>(c, c->d_kap_in, c->d_q_in, true)
                                : set_material_impl<float>(c, c->d_kap_in, c->d_q_in, true);
  if (rc) return rc;
  TRT_CUDA(cudaEventRecord(c->ev_stage_free, c->stream));
  c->have_material = true;
  return TRT_OK;
}

int trt_moments_async(trt_ctx* c, const trt_moments_host* out) {
  if (!c || !out) return TRT_ERR_ARG;
  if (!c->have_moments) return TRT_ERR_STATE;
  int rc = pipe_init(c);
  if (rc) return rc;
  long long sz[kNOut];
  output_sizes(c->nx, c->ny, c->ng, sz);
  TRT_CUDA(cudaEventRecord(c->ev_epi, c->stream));
  TRT_CUDA(cudaStreamWaitEvent(c->s_out, c->ev_epi, 0));
  const double* const* h = reinterpret_cast<const double* const*>(out);
  double* const* d = reinterpret_cast<double* const*>(&c->dout);
  for (int k = 0; k < kNOut; ++k)
    if (h[k]) TRT_CUDA(cudaMemcpyAsync((void*)h[k], d[k], sz[k] * sizeof(double), cudaMemcpyDeviceToHost, c->s_out));
  TRT_CUDA(cudaEventRecord(c->ev_out, c->s_out));
  c->out_pending = true;
  return TRT_OK;
}

int trt_moments(trt_ctx* c, const trt_moments_host* out) {
  if (!c || !out) return TRT_ERR_ARG;
  if (!c->have_moments) return TRT_ERR_STATE;
  int rc = trt_sync(c);
  if (rc) return rc;
  long long sz[kNOut];
  output_sizes(c->nx, c->ny, c->ng, sz);
  const double* const* h = reinterpret_cast<const double* const*>(out);
  double* const* d = reinterpret_cast<double* const*>(&c->dout);
  for (int k = 0; k < kNOut; ++k)
    if (h[k]) TRT_CUDA(cudaMemcpyAsync((void*)h[k], d[k], sz[k] * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

int trt_get_angular(trt_ctx* c, double* I_avg, double* I_edgV, double* I_edgH, double* Ic_edgV, double* Ic_edgH) {
  if (!c) return TRT_ERR_ARG;
  int rc = trt_sync(c);
  if (rc) return rc;
  return c->prec == TRT_PREC_FP64 ? get_angular_impl<double>(c, I_avg, I_edgV, I_edgH, Ic_edgV, Ic_edgH)
                                  : get_angular_impl<float>(c, I_avg, I_edgV, I_edgH, Ic_edgV, Ic_edgH);
}

int trt_snapshot_angular(trt_ctx* c, float* I_avg_device) {
  if (!c || !I_avg_device) return TRT_ERR_ARG;
  if (!c->have_state && !c->swept) return TRT_ERR_STATE;
  const void* st = c->d_state[c->swept ? 1 - c->cur : c->cur];
  const long long n = (long long)c->nx * c->ny * c->nm * c->ng;
  if (c->prec == TRT_PREC_FP64)
    trt::snapshot_avg_kernel<double><<<grid_for(n), 256, 0, c->stream>>>(c->geo(), (const double*)st, I_avg_device, 0,
                                                                         c->ng);
  else
    trt::snapshot_avg_kernel<float><<<grid_for(n), 256, 0, c->stream>>>(c->geo(), (const float*)st, I_avg_device, 0,
                                                                        c->ng);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  return TRT_OK;
}

int trt_snapshot_output(trt_ctx* c, const char* name, double* dst_device) {
  if (!c || !name || !dst_device) return TRT_ERR_ARG;
  if (!c->have_moments) return TRT_ERR_STATE;
  long long sz[kNOut];
  output_sizes(c->nx, c->ny, c->ng, sz);
  double* const* d = reinterpret_cast<double* const*>(&c->dout);
  for (int k = 0; k < kNOut; ++k)
    if (std::strcmp(kOutNames[k], name) == 0) {
      TRT_CUDA(cudaMemcpyAsync(dst_device, d[k], sz[k] * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      return TRT_OK;
    }
  return TRT_ERR_ARG;
}

int trt_get_residual(trt_ctx* c, double* RT_Residual, int* RT_ResLoc_x, int* RT_ResLoc_y) {
  if (!c || !RT_Residual || !RT_ResLoc_x || !RT_ResLoc_y) return TRT_ERR_ARG;
  if (!c->have_res) return TRT_ERR_STATE;
  int rc = trt_sync(c);
  if (rc) return rc;
  TRT_CUDA(cudaMemcpy(RT_Residual, c->d_res, 20 * c->ng * sizeof(double), cudaMemcpyDeviceToHost));
  TRT_CUDA(cudaMemcpy(RT_ResLoc_x, c->d_resx, 20 * c->ng * sizeof(int), cudaMemcpyDeviceToHost));
  TRT_CUDA(cudaMemcpy(RT_ResLoc_y, c->d_resy, 20 * c->ng * sizeof(int), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

void* trt_stream(trt_ctx* c) { return c ? (void*)c->stream : nullptr; }

int trt_set_wait_limit(trt_ctx* c, unsigned polls) {
  if (!c) return TRT_ERR_ARG;
  c->wait_polls = polls ? polls : kDefaultWaitPolls;
  return TRT_OK;
}

int trt_set_wait_limit_zero(trt_ctx* c) {
  if (!c) return TRT_ERR_ARG;
  c->wait_polls = 0;
  return TRT_OK;
}

int trt_tstep_setup(trt_ctx* c, const double* Nu_g, const double* kappa_mult, const double* cV, const double* Temp,
                    double Kap0, double Comp_Unit, double cl, double Delt, const int* BC_Type, const double* bcT,
                    int conv_type, double conv_ho, int maxit_rte) {
  if (!c || !Nu_g || !kappa_mult || !cV || !Temp || !BC_Type || !bcT || !(Comp_Unit > 0) || !(cl > 0) ||
      !(Delt > 0) || conv_type < 1 || conv_type > 3 || maxit_rte < 1 || !(conv_ho >= 0))
    return TRT_ERR_ARG;
  const size_t nxy = (size_t)c->nx * c->ny;
  int rc = TRT_OK;
  if (!c->d_T) {
    for (double** p : {&c->d_T, &c->d_Told, &c->d_Trt1, &c->d_Trt2, &c->d_Ert1, &c->d_Ert2, &c->d_kmult, &c->d_cv})
      if ((rc = alloc_t(c, p, nxy))) return rc;
    if ((rc = alloc_t(c, &c->d_nu, (size_t)c->ng + 1))) return rc;
    if ((rc = alloc_t(c, &c->d_conv, 10))) return rc;
  }
  TRT_CUDA(cudaMemcpyAsync(c->d_T, Temp, nxy * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaMemcpyAsync(c->d_kmult, kappa_mult, nxy * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaMemcpyAsync(c->d_cv, cV, nxy * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  TRT_CUDA(cudaMemcpyAsync(c->d_nu, Nu_g, (c->ng + 1) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  c->ts_nu.assign(Nu_g, Nu_g + c->ng + 1);
  for (int k = 0; k < 4; ++k) {
    c->ts_bc[k] = BC_Type[k];
    c->bc[k] = BC_Type[k];
    c->ts_Tb[k] = bcT[k];
  }
  c->ts_Kap0 = Kap0;
  c->ts_conv_type = conv_type;
  c->ts_conv_ho = conv_ho;
  c->ts_maxit = maxit_rte;
  c->c = cl;
  c->dt = Delt;
  c->comp_unit = Comp_Unit;
  // initial material from the initial temperature (INITIALIZERS.f08:137)
  rc = c->prec == TRT_PREC_FP64 ? material_update_impl<double>(c) : material_update_impl<float>(c);
  if (rc) return rc;
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  c->ts_ready = true;
  return TRT_OK;
}

static_assert(TRT_LAW_FLECK_CUMMINGS == trt::kLawFleckCummings && TRT_LAW_CONFIG == trt::kLawConfig,
              "material law numbering");

int trt_tstep_begin(trt_ctx* c) {
  if (!c) return TRT_ERR_ARG;
  if (!c->ts_ready || (!c->have_state && !c->swept)) return TRT_ERR_STATE;
  return tstep_begin(c);
}

int trt_tstep_sweep(trt_ctx* c, int its) {
  if (!c || its < 1) return TRT_ERR_ARG;
  if (!c->ts_ready || (!c->have_state && !c->swept)) return TRT_ERR_STATE;
  const unsigned flags = (its == 1 ? TRT_ROLL_STATE : 0u) | TRT_MOMENTS;
  const bool reflective = c->ts_bc[0] > 0 || c->ts_bc[1] > 0 || c->ts_bc[2] > 0 || c->ts_bc[3] > 0;
  int rc = c->prec == TRT_PREC_FP64 ? sweep_impl<double>(c, flags) : sweep_impl<float>(c, flags);
  if (rc) return rc;
  if (reflective)
    rc = c->prec == TRT_PREC_FP64 ? bc_update_impl<double>(c, c->ts_bc, c->ts_Tb, c->comp_unit, c->ts_nu.data())
                                  : bc_update_impl<float>(c, c->ts_bc, c->ts_Tb, c->comp_unit, c->ts_nu.data());
  c->have_moments = true;
  return rc;
}

int trt_tstep_partials(trt_ctx* c, double* part_device) {
  if (!c || !part_device) return TRT_ERR_ARG;
  if (!c->ts_ready || !c->have_moments) return TRT_ERR_STATE;
  return tstep_partials_impl(c, part_device);
}

int trt_tstep_finish(trt_ctx* c, const double* sum_device, int its, int* converged, double* T_norm, double* E_norm) {
  if (!c || !sum_device || its < 1) return TRT_ERR_ARG;
  if (!c->ts_ready || !c->have_moments) return TRT_ERR_STATE;
  return c->prec == TRT_PREC_FP64 ? tstep_finish_impl<double>(c, sum_device, its, converged, T_norm, E_norm)
                                  : tstep_finish_impl<float>(c, sum_device, its, converged, T_norm, E_norm);
}

int trt_tstep_set_law(trt_ctx* c, int law) {
  if (!c || (law != trt::kLawFleckCummings && law != trt::kLawConfig)) return TRT_ERR_ARG;
  c->ts_law = law;
  if (c->ts_ready) {   // the material follows the law at once
    int rc = c->prec == TRT_PREC_FP64 ? material_update_impl<double>(c) : material_update_impl<float>(c);
    if (rc) return rc;
    TRT_CUDA(cudaStreamSynchronize(c->stream));
  }
  return TRT_OK;
}

int trt_tstep(trt_ctx* c, int* rt_its, double* T_norm, double* E_norm) {
  if (!c) return TRT_ERR_ARG;
  if (!c->ts_ready || (!c->have_state && !c->swept)) return TRT_ERR_STATE;
  if (c->inplace && c->ts_maxit > 1) return TRT_ERR_STATE;   // later outer iterations re-read I_crn_old
  return c->prec == TRT_PREC_FP64 ? tstep_impl<double>(c, rt_its, T_norm, E_norm)
                                  : tstep_impl<float>(c, rt_its, T_norm, E_norm);
}

int trt_get_temperature(trt_ctx* c, double* Temp) {
  if (!c || !Temp) return TRT_ERR_ARG;
  if (!c->ts_ready) return TRT_ERR_STATE;
  TRT_CUDA(cudaMemcpyAsync(Temp, c->d_T, (size_t)c->nx * c->ny * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

int trt_put_temperature(trt_ctx* c, const double* Temp) {
  if (!c || !Temp) return TRT_ERR_ARG;
  if (!c->ts_ready) return TRT_ERR_STATE;
  TRT_CUDA(cudaMemcpyAsync(c->d_T, Temp, (size_t)c->nx * c->ny * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = c->prec == TRT_PREC_FP64 ? material_update_impl<double>(c) : material_update_impl<float>(c);
  if (rc) return rc;
  TRT_CUDA(cudaStreamSynchronize(c->stream));
  return TRT_OK;
}

const double* trt_device_output(trt_ctx* c, const char* name) {
  if (!c || !name) return nullptr;
  double* const* d = reinterpret_cast<double* const*>(&c->dout);
  for (int k = 0; k < kNOut; ++k)
    if (std::strcmp(kOutNames[k], name) == 0) return d[k];
  return nullptr;
}

int trt_transport_scb(int n_x, int n_y, int n_m, int n_g, double* I_avg, double* I_edgV, double* I_edgH,
                      double* I_crn, double* Ic_edgV, double* Ic_edgH, const double* Omega_x,
                      const double* Omega_y, const double* Delx, const double* Dely, const double* A,
                      const double* KapE_in, const double* Src_in, const double* I_crn_old, double c,
                      double Delt, int Open_Threads, double* RT_Residual, int* RT_ResLoc_x, int* RT_ResLoc_y,
                      int Res_Calc) {
  (void)Open_Threads;
  if (!valid_shape(n_x, n_y, n_m, n_g) || !I_avg || !I_edgV || !I_edgH || !I_crn || !Ic_edgV || !Ic_edgH ||
      !Omega_x || !Omega_y || !Delx || !Dely || !A || !KapE_in || !Src_in || !I_crn_old ||
      (Res_Calc && (!RT_Residual || !RT_ResLoc_x || !RT_ResLoc_y)))
    return TRT_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_cache.mu);
  int rc = TRT_OK;
  trt_ctx* ctx = cached_ctx(n_x, n_y, n_m, n_g, Omega_x, Omega_y, Delx, Dely, &rc);
  if (!ctx) return rc;
  return transport_scb_impl(ctx, n_x, n_y, n_m, n_g, I_avg, I_edgV, I_edgH, I_crn, Ic_edgV, Ic_edgH, A, KapE_in,
                            Src_in, I_crn_old, c, Delt, RT_Residual, RT_ResLoc_x, RT_ResLoc_y, Res_Calc);
}

int trt_collapse_intensities(int n_x, int n_y, int n_m, int n_g, int Open_Threads, const double* I_avg,
                             const double* I_edgV, const double* I_edgH, const double* Omega_x,
                             const double* Omega_y, const double* quad_weight, double Comp_Unit,
                             double* Hg_avg_xx, double* Hg_avg_yy, double* Hg_avg_xy, double* Hg_edgV_xx,
                             double* Hg_edgV_xy, double* Hg_edgH_yy, double* Hg_edgH_xy, double* Eg_edgV,
                             double* Eg_edgH, double* Eg_avg, double* Fxg_edgV, double* Fyg_edgH,
                             double* E_edgV, double* E_edgH, double* E_avg, double* Fx_edgV, double* Fy_edgH) {
  (void)Open_Threads;
  if (!valid_shape(n_x, n_y, n_m, n_g) || !(Comp_Unit != 0)) return TRT_ERR_ARG;
  int rc = device_check();
  if (rc) return rc;
  const size_t nA = (size_t)n_x * n_y, nV = (size_t)(n_x + 1) * n_y, nH = (size_t)n_x * (n_y + 1);
  DBuf dIa, dIv, dIh, dox, doy, dw;
  if ((rc = dIa.put(I_avg, nA * n_m * n_g)) || (rc = dIv.put(I_edgV, nV * n_m * n_g)) ||
      (rc = dIh.put(I_edgH, nH * n_m * n_g)) || (rc = dox.put(Omega_x, n_m)) || (rc = doy.put(Omega_y, n_m)) ||
      (rc = dw.put(quad_weight, n_m)))
    return rc;
  DBuf o[17];
  const size_t szs[17] = {nA * n_g, nA * n_g, nA * n_g, nV * n_g, nV * n_g, nH * n_g, nH * n_g, nV * n_g, nH * n_g,
                          nA * n_g, nV * n_g, nH * n_g, nV,       nH,       nA,       nV,       nH};
  for (int k = 0; k < 17; ++k)
    if ((rc = o[k].alloc(szs[k]))) return rc;
  double eps = 1e-25;
  eps = eps / Comp_Unit;
  trt::collapse_dropin_kernel<<<grid_for((long long)nV * n_g + nH * n_g), 256>>>(
      n_x, n_y, n_m, n_g, dIa.p, dIv.p, dIh.p, dox.p, doy.p, dw.p, eps, o[0].p, o[1].p, o[2].p, o[3].p, o[4].p,
      o[5].p, o[6].p, o[7].p, o[8].p, o[9].p, o[10].p, o[11].p);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  trt::MomentOut M{};
  M.Eg_avg = o[9].p; M.Eg_edgV = o[7].p; M.Eg_edgH = o[8].p; M.Fxg_edgV = o[10].p; M.Fyg_edgH = o[11].p;
  M.E_edgV = o[12].p; M.E_edgH = o[13].p; M.E_avg = o[14].p; M.Fx_edgV = o[15].p; M.Fy_edgH = o[16].p;
  trt::group_sum_kernel<<<grid_for(trt::group_sum_items(n_x, n_y)), 256>>>(n_x, n_y, n_g, M);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  double* hs[17] = {Hg_avg_xx, Hg_avg_yy, Hg_avg_xy, Hg_edgV_xx, Hg_edgV_xy, Hg_edgH_yy, Hg_edgH_xy, Eg_edgV, Eg_edgH,
                    Eg_avg,    Fxg_edgV,  Fyg_edgH,  E_edgV,     E_edgH,     E_avg,      Fx_edgV,    Fy_edgH};
  for (int k = 0; k < 17; ++k)
    if (hs[k] && (rc = o[k].get(hs[k], szs[k]))) return rc;
  return TRT_OK;
}

int trt_fg_calc(int n_x, int n_y, int n_g, double* fg_avg_xx, double* fg_avg_yy, double* fg_avg_xy,
                double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy, double* fg_edgH_xy,
                const double* Hg_avg_xx, const double* Hg_avg_yy, const double* Hg_avg_xy,
                const double* Hg_edgV_xx, const double* Hg_edgV_xy, const double* Hg_edgH_yy,
                const double* Hg_edgH_xy, const double* HO_Eg_avg, const double* HO_Eg_edgV,
                const double* HO_Eg_edgH, double c, int Open_Threads) {
  (void)Open_Threads;
  if (n_x < 1 || n_y < 1 || n_g < 1) return TRT_ERR_ARG;
  int rc = device_check();
  if (rc) return rc;
  const size_t nA = (size_t)n_x * n_y * n_g, nV = (size_t)(n_x + 1) * n_y * n_g, nH = (size_t)n_x * (n_y + 1) * n_g;
  DBuf in[10], out[7];
  const double* hin[10] = {Hg_avg_xx, Hg_avg_yy, Hg_avg_xy, Hg_edgV_xx, Hg_edgV_xy, Hg_edgH_yy, Hg_edgH_xy,
                           HO_Eg_avg, HO_Eg_edgV, HO_Eg_edgH};
  const size_t nin[10] = {nA, nA, nA, nV, nV, nH, nH, nA, nV, nH};
  for (int k = 0; k < 10; ++k)
    if ((rc = in[k].put(hin[k], nin[k]))) return rc;
  double* hout[7] = {fg_avg_xx, fg_avg_yy, fg_avg_xy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy};
  const size_t nout[7] = {nA, nA, nA, nV, nV, nH, nH};
  for (int k = 0; k < 7; ++k)
    if ((rc = out[k].alloc(nout[k]))) return rc;
  trt::fg_dropin_kernel<<<grid_for((long long)nV + nH), 256>>>(
      (long long)nA, (long long)nV, (long long)nH, c, in[0].p, in[1].p, in[2].p, in[3].p, in[4].p, in[5].p, in[6].p,
      in[7].p, in[8].p, in[9].p, out[0].p, out[1].p, out[2].p, out[3].p, out[4].p, out[5].p, out[6].p);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  for (int k = 0; k < 7; ++k)
    if ((rc = out[k].get(hout[k], nout[k]))) return rc;
  return TRT_OK;
}

static int boundary_common(int n_x, int n_y, int n_m, int n_g, int mode, const int* BC_Type, const double* I_edgV,
                           const double* I_edgH, const double* Ox, const double* Oy, const double* w, double eps,
                           double c, double* L, double* B, double* R, double* T, double* FL, double* FB, double* FR,
                           double* FT) {
  if (!valid_shape(n_x, n_y, n_m, n_g) || !BC_Type) return TRT_ERR_ARG;
  int rc = device_check();
  if (rc) return rc;
  const size_t nV = (size_t)(n_x + 1) * n_y * n_m * n_g, nH = (size_t)n_x * (n_y + 1) * n_m * n_g;
  DBuf dV, dH, dox, doy, dw, o[8];
  if ((rc = dV.put(I_edgV, nV)) || (rc = dH.put(I_edgH, nH)) || (rc = dox.put(Ox, n_m)) || (rc = doy.put(Oy, n_m)) ||
      (rc = dw.put(w, n_m)))
    return rc;
  const size_t ny_g = (size_t)n_y * n_g, nx_g = (size_t)n_x * n_g;
  const size_t sz[8] = {ny_g, nx_g, ny_g, nx_g, ny_g, nx_g, ny_g, nx_g};
  for (int k = 0; k < 8; ++k)
    if ((rc = o[k].alloc(sz[k]))) return rc;
  trt::boundary_dropin_kernel<<<grid_for(2LL * (n_x + n_y) * n_g), 256>>>(
      n_x, n_y, n_m, n_g, mode, make_int4(BC_Type[0], BC_Type[1], BC_Type[2], BC_Type[3]), dV.p, dH.p, dox.p, doy.p,
      dw.p, eps, c, o[0].p, o[1].p, o[2].p, o[3].p, o[4].p, o[5].p, o[6].p, o[7].p);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  double* h[8] = {L, B, R, T, FL, FB, FR, FT};
  for (int k = 0; k < (mode == 0 ? 4 : 8); ++k)
    if (h[k] && (rc = o[k].get(h[k], sz[k]))) return rc;
  return TRT_OK;
}

int trt_cg_calc(int n_x, int n_y, int n_m, int n_g, double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T,
                const double* I_edgV, const double* I_edgH, const double* Omega_x, const double* Omega_y,
                const double* quad_weight, double Comp_Unit, const int* BC_Type, int Open_Threads) {
  (void)Open_Threads;
  if (!(Comp_Unit != 0)) return TRT_ERR_ARG;
  double eps = 1e-25;
  eps = eps / Comp_Unit;
  return boundary_common(n_x, n_y, n_m, n_g, 0, BC_Type, I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, eps, 1.0, Cg_L,
                         Cg_B, Cg_R, Cg_T, nullptr, nullptr, nullptr, nullptr);
}

int trt_mgqd_in_calc(int n_x, int n_y, int n_m, int n_g, double* Eg_in_L, double* Eg_in_B, double* Eg_in_R,
                     double* Eg_in_T, double* Fg_in_L, double* Fg_in_B, double* Fg_in_R, double* Fg_in_T,
                     const double* I_edgV, const double* I_edgH, const double* Omega_x, const double* Omega_y,
                     const double* quad_weight, double c, double Comp_Unit, const int* BC_Type,
                     int Open_Threads) {
  (void)Open_Threads;
  (void)Comp_Unit;
  return boundary_common(n_x, n_y, n_m, n_g, 1, BC_Type, I_edgV, I_edgH, Omega_x, Omega_y, quad_weight, 0.0, c,
                         Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T);
}

int trt_gqd_in_calc(int n_x, int n_y, int n_g, double* E_in_L, double* E_in_B, double* E_in_R, double* E_in_T,
                    double* F_in_L, double* F_in_B, double* F_in_R, double* F_in_T, const double* Eg_in_L,
                    const double* Eg_in_B, const double* Eg_in_R, const double* Eg_in_T, const double* Fg_in_L,
                    const double* Fg_in_B, const double* Fg_in_R, const double* Fg_in_T) {
  if (n_x < 1 || n_y < 1 || n_g < 1) return TRT_ERR_ARG;
  int rc = device_check();
  if (rc) return rc;
  const size_t ny_g = (size_t)n_y * n_g, nx_g = (size_t)n_x * n_g;
  DBuf in[8], out[8];
  const double* hin[8] = {Eg_in_L, Eg_in_B, Eg_in_R, Eg_in_T, Fg_in_L, Fg_in_B, Fg_in_R, Fg_in_T};
  const size_t nin[8] = {ny_g, nx_g, ny_g, nx_g, ny_g, nx_g, ny_g, nx_g};
  for (int k = 0; k < 8; ++k)
    if ((rc = in[k].put(hin[k], nin[k]))) return rc;
  double* hout[8] = {E_in_L, E_in_B, E_in_R, E_in_T, F_in_L, F_in_B, F_in_R, F_in_T};
  const size_t nout[8] = {(size_t)n_y, (size_t)n_x, (size_t)n_y, (size_t)n_x,
                          (size_t)n_y, (size_t)n_x, (size_t)n_y, (size_t)n_x};
  for (int k = 0; k < 8; ++k)
    if ((rc = out[k].alloc(nout[k]))) return rc;
  trt::MomentOut M{};
  M.Eg_in_L = in[0].p; M.Eg_in_B = in[1].p; M.Eg_in_R = in[2].p; M.Eg_in_T = in[3].p;
  M.Fg_in_L = in[4].p; M.Fg_in_B = in[5].p; M.Fg_in_R = in[6].p; M.Fg_in_T = in[7].p;
  M.E_in_L = out[0].p; M.E_in_B = out[1].p; M.E_in_R = out[2].p; M.E_in_T = out[3].p;
  M.F_in_L = out[4].p; M.F_in_B = out[5].p; M.F_in_R = out[6].p; M.F_in_T = out[7].p;
  trt::group_sum_kernel<<<grid_for(trt::group_sum_items(n_x, n_y)), 256>>>(n_x, n_y, n_g, M);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  for (int k = 0; k < 8; ++k)
    if ((rc = out[k].get(hout[k], nout[k]))) return rc;
  return TRT_OK;
}

int trt_rt_bc_update(int n_x, int n_y, int n_m, int n_g, const int* BC_Type, double bcT_left, double bcT_lower,
                     double bcT_right, double bcT_upper, double Comp_Unit, const double* Nu_g, double* I_edgV,
                     double* I_edgH, double* Ic_edgV, double* Ic_edgH) {
  if (!valid_shape(n_x, n_y, n_m, n_g) || !BC_Type || !Nu_g || !I_edgV || !I_edgH || !Ic_edgV || !Ic_edgH)
    return TRT_ERR_ARG;
  int rc = device_check();
  if (rc) return rc;
  // Boundary faces are gathered into face-major device arrays, updated on the device by the same
  // kernel the resident handle uses, and scattered back.  I_edgV/I_edgH faces travel as pairs of
  // equal values so that one kernel serves both the corner-edge and the cell-edge arrays.
  const int nx = n_x, ny = n_y, nm = n_m, ng = n_g;
  const size_t nbV = (size_t)2 * ng * nm * 2 * ny, nbH = (size_t)2 * ng * nm * 2 * nx;
  std::vector<double> cV(nbV), cH(nbH), eV(nbV), eH(nbH);
  for (int side = 0; side < 2; ++side)
    for (int g = 0; g < ng; ++g)
      for (int m = 0; m < nm; ++m) {
        const size_t bv = ((size_t)(side * ng + g) * nm + m) * 2 * ny, bh = ((size_t)(side * ng + g) * nm + m) * 2 * nx;
        const int fv = side ? nx : 0, fh = side ? ny : 0;
        for (int iy = 0; iy < 2 * ny; ++iy) cV[bv + iy] = Ic_edgV[fv + (size_t)(nx + 1) * (iy + (size_t)2 * ny * (m + (size_t)nm * g))];
        for (int ix = 0; ix < 2 * nx; ++ix) cH[bh + ix] = Ic_edgH[ix + (size_t)2 * nx * (fh + (size_t)(ny + 1) * (m + (size_t)nm * g))];
        for (int j = 0; j < ny; ++j) eV[bv + 2 * j] = eV[bv + 2 * j + 1] = I_edgV[fv + (size_t)(nx + 1) * (j + (size_t)ny * (m + (size_t)nm * g))];
        for (int i = 0; i < nx; ++i) eH[bh + 2 * i] = eH[bh + 2 * i + 1] = I_edgH[i + (size_t)nx * (fh + (size_t)(ny + 1) * (m + (size_t)nm * g))];
      }
  std::vector<double> bval((size_t)4 * ng);
  const double Tb[4] = {bcT_left, bcT_lower, bcT_right, bcT_upper};
  for (int s = 0; s < 4; ++s)
    for (int g = 0; g < ng; ++g) bval[(size_t)s * ng + g] = bg_planck_h(Tb[s], Nu_g[g], Nu_g[g + 1], Comp_Unit);
  DBuf dcV, dcH, deV, deH, dbv;
  if ((rc = dcV.put(cV.data(), nbV)) || (rc = dcH.put(cH.data(), nbH)) || (rc = deV.put(eV.data(), nbV)) ||
      (rc = deH.put(eH.data(), nbH)) || (rc = dbv.put(bval.data(), bval.size())))
    return rc;
  const int4 bc = make_int4(BC_Type[0], BC_Type[1], BC_Type[2], BC_Type[3]);
  const long long n = 2LL * ng * nm * 2 * std::max(nx, ny);
  trt::bc_update_kernel<double><<<grid_for(n), 256>>>(nx, ny, nm, ng, bc, dbv.p, dcV.p, dcH.p);
  TRT_LAUNCHED();
  trt::bc_update_kernel<double><<<grid_for(n), 256>>>(nx, ny, nm, ng, bc, dbv.p, deV.p, deH.p);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  if ((rc = dcV.get(cV.data(), nbV)) || (rc = dcH.get(cH.data(), nbH)) || (rc = deV.get(eV.data(), nbV)) ||
      (rc = deH.get(eH.data(), nbH)))
    return rc;
  for (int side = 0; side < 2; ++side)
    for (int g = 0; g < ng; ++g)
      for (int m = 0; m < nm; ++m) {
        const size_t bv = ((size_t)(side * ng + g) * nm + m) * 2 * ny, bh = ((size_t)(side * ng + g) * nm + m) * 2 * nx;
        const int fv = side ? nx : 0, fh = side ? ny : 0;
        for (int iy = 0; iy < 2 * ny; ++iy) Ic_edgV[fv + (size_t)(nx + 1) * (iy + (size_t)2 * ny * (m + (size_t)nm * g))] = cV[bv + iy];
        for (int ix = 0; ix < 2 * nx; ++ix) Ic_edgH[ix + (size_t)2 * nx * (fh + (size_t)(ny + 1) * (m + (size_t)nm * g))] = cH[bh + ix];
        for (int j = 0; j < ny; ++j) I_edgV[fv + (size_t)(nx + 1) * (j + (size_t)ny * (m + (size_t)nm * g))] = eV[bv + 2 * j];
        for (int i = 0; i < nx; ++i) I_edgH[i + (size_t)nx * (fh + (size_t)(ny + 1) * (m + (size_t)nm * g))] = eH[bh + 2 * i];
      }
  return TRT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// trt_transport_residual_noalloc: the corner-balance residual norms of TRANSPORT_SCB computed
// without allocating device memory.
//
// Some callers cannot call cudaMalloc: a host code that hands the library a fixed, pre-sized device
// arena and owns all allocation itself, or a solver loop that must not pay cudaMalloc/cudaFree's
// implicit device synchronisation in the middle of an iteration.  For them the residual kernel's
// per-(direction, group) scratch lives in the file-scope array below instead of in memory the
// resident handle allocates; the caller passes every input and output as device pointers.
//
// Limit: n_m * n_g <= kNoAllocMaxDirGroups (65536 direction-group pairs, 3 MiB of scratch that every
// GPU which loads the library holds until the process exits).  Larger problems are rejected with
// TRT_ERR_SCRATCH before anything is launched.
// ---------------------------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxDirGroups = 1 << 16;
constexpr size_t kNoAllocNormBytes = (size_t)kNoAllocMaxDirGroups * 5 * sizeof(double);
constexpr size_t kNoAllocScratchBytes = kNoAllocNormBytes + (size_t)kNoAllocMaxDirGroups * 2 * sizeof(int);
// In host code this name is only a host-side stand-in: its device address comes from
// cudaGetSymbolAddress (noalloc_scratch below) and is what the kernels receive.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per device (with that device
// current) on the first call made on it.
int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return TRT_ERR_NODEV;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) return TRT_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return TRT_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return TRT_OK;
}

// Residual norms of one (m, g) over the reference layouts I_crn(2nx,2ny,nm,ng),
// Ic_edgV(nx+1,2ny,nm,ng), Ic_edgH(2nx,ny+1,nm,ng); the expressions and loop order of
// TRANSPORT_SOLVES.f08:256-309, the source formed as the sweep forms it (fma(I_crn_old, 1/(c dt),
// Src_in)).
__global__ void residual_fortran_kernel(int nx, int ny, int nm, int ng, const double* __restrict__ I_crn,
                                        const double* __restrict__ Ic_edgV, const double* __restrict__ Ic_edgH,
                                        const double* __restrict__ omx, const double* __restrict__ omy,
                                        const double* __restrict__ Delx, const double* __restrict__ Dely,
                                        const double* __restrict__ A, const double* __restrict__ KapE_in,
                                        const double* __restrict__ Src_in, const double* __restrict__ I_crn_old,
                                        double rcdt, double* per_m, int* per_m_loc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nm * ng) return;
  const int m = k % nm, g = k / nm;
  const double Ox = omx[m], Oy = omy[m];
  const long long n2x = 2LL * nx, n2y = 2LL * ny;
  const long long cbase = n2x * n2y * (m + (long long)nm * g);
  const long long vbase = (long long)(nx + 1) * n2y * (m + (long long)nm * g);
  const long long hbase = n2x * (ny + 1) * (m + (long long)nm * g);
  double vmax = 0.0, sums[4] = {0.0, 0.0, 0.0, 0.0};
  int li = 0, lj = 0;
  for (int j = 0; j < ny; ++j) {
    for (int i = 0; i < nx; ++i) {
      const double Aij = A[i + (long long)nx * j];
      const double kp = KapE_in[i + (long long)nx * (j + (long long)ny * g)] + rcdt;
      const double dxx = Delx[i], dyy = Dely[j];
      double I[2][2], Sr[2][2];
      for (int cx = 0; cx < 2; ++cx)
        for (int cy = 0; cy < 2; ++cy) {
          const long long ci = cbase + (2 * i + cx) + n2x * (2 * j + cy);
          I[cx][cy] = I_crn[ci];
          Sr[cx][cy] = fma(I_crn_old[ci], rcdt, Src_in[ci]);
        }
      auto V = [&](int f, int iy) { return Ic_edgV[vbase + f + (long long)(nx + 1) * iy]; };
      auto H = [&](int ix, int f) { return Ic_edgH[hbase + ix + n2x * f]; };
      double res[4];
      res[0] = fabs((Ox * dyy + Oy * dxx + kp * Aij) * I[0][0] / 4.0 + Ox * dyy * I[1][0] / 4.0 +
                    Oy * dxx * I[0][1] / 4.0 - Ox * dyy * V(i, 2 * j) / 2.0 - Oy * dxx * H(2 * i, j) / 2.0 -
                    Aij * Sr[0][0] / 4.0);
      res[1] = fabs((-Ox * dyy + Oy * dxx + kp * Aij) * I[1][0] / 4.0 - Ox * dyy * I[0][0] / 4.0 +
                    Oy * dxx * I[1][1] / 4.0 + Ox * dyy * V(i + 1, 2 * j) / 2.0 - Oy * dxx * H(2 * i + 1, j) / 2.0 -
                    Aij * Sr[1][0] / 4.0);
      res[2] = fabs((-Ox * dyy - Oy * dxx + kp * Aij) * I[1][1] / 4.0 - Ox * dyy * I[0][1] / 4.0 -
                    Oy * dxx * I[1][0] / 4.0 + Ox * dyy * V(i + 1, 2 * j + 1) / 2.0 +
                    Oy * dxx * H(2 * i + 1, j + 1) / 2.0 - Aij * Sr[1][1] / 4.0);
      res[3] = fabs((Ox * dyy - Oy * dxx + kp * Aij) * I[0][1] / 4.0 + Ox * dyy * I[1][1] / 4.0 -
                    Oy * dxx * I[0][0] / 4.0 - Ox * dyy * V(i, 2 * j + 1) / 2.0 + Oy * dxx * H(2 * i, j + 1) / 2.0 -
                    Aij * Sr[0][1] / 4.0);
      for (int kk = 0; kk < 4; ++kk) {
        if (res[kk] > vmax) {
          vmax = res[kk];
          li = i + 1;
          lj = j + 1;
        }
        sums[0] = sums[0] + res[kk];
        sums[1] = sums[1] + res[kk] * res[kk];
        sums[2] = sums[2] + Aij * res[kk] / 4.0;
        sums[3] = sums[3] + Aij * (res[kk] * res[kk]) / 4.0;
      }
    }
  }
  double* o = per_m + ((size_t)g * nm + m) * 5;
  o[0] = vmax; o[1] = sums[0]; o[2] = sums[1]; o[3] = sums[2]; o[4] = sums[3];
  int* l = per_m_loc + ((size_t)g * nm + m) * 2;
  l[0] = li;
  l[1] = lj;
}

}  // namespace

extern "C" int trt_transport_residual_noalloc(int n_x, int n_y, int n_m, int n_g, const double* I_crn,
                                              const double* Ic_edgV, const double* Ic_edgH, const double* Omega_x,
                                              const double* Omega_y, const double* Delx, const double* Dely,
                                              const double* A, const double* KapE_in, const double* Src_in,
                                              const double* I_crn_old, double c, double Delt, double* RT_Residual,
                                              int* RT_ResLoc_x, int* RT_ResLoc_y, void* stream) {
  if (!valid_shape(n_x, n_y, n_m, n_g) || !I_crn || !Ic_edgV || !Ic_edgH || !Omega_x || !Omega_y || !Delx ||
      !Dely || !A || !KapE_in || !Src_in || !I_crn_old || !RT_Residual || !RT_ResLoc_x || !RT_ResLoc_y ||
      !(c > 0) || !(Delt > 0))
    return TRT_ERR_ARG;
  if ((long long)n_m * n_g > kNoAllocMaxDirGroups) return TRT_ERR_SCRATCH;
  void* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  double* per_m = static_cast<double*>(scratch);
  int* per_m_loc = reinterpret_cast<int*>(static_cast<unsigned char*>(scratch) + kNoAllocNormBytes);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // every scratch slot the reduction reads is written by the first kernel of the same call, so no
  // clearing is needed; RT_ResLoc_x/y keep the caller's values where no norm exceeds zero, as in
  // the reference
  const int mg = n_m * n_g;
  residual_fortran_kernel<<<(mg + 63) / 64, 64, 0, st>>>(n_x, n_y, n_m, n_g, I_crn, Ic_edgV, Ic_edgH, Omega_x,
                                                         Omega_y, Delx, Dely, A, KapE_in, Src_in, I_crn_old,
                                                         1.0 / (c * Delt), per_m, per_m_loc);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  trt::residual_reduce_kernel<<<(4 * n_g + 63) / 64, 64, 0, st>>>(n_x, n_y, n_m, n_g, per_m, per_m_loc, RT_Residual,
                                                                  RT_ResLoc_x, RT_ResLoc_y);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  return TRT_OK;
}

namespace trt_host {
// launch counter shared with the other translation units of the library
void add_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace trt_host

// ---------------------------------------------------------------------------------------------
// Hooks for the low-order time loop of mgqd.cu (handle_hooks.h).
// ---------------------------------------------------------------------------------------------
namespace trt_host {

int handle_view(trt_ctx* c, HandleView* v) {
  if (!c || !v) return TRT_ERR_ARG;
  if (!c->ts_ready) return TRT_ERR_STATE;
  v->nx = c->nx;
  v->ny = c->ny;
  v->nm = c->nm;
  v->ng = c->ng;
  v->prec = c->prec;
  for (int k = 0; k < 4; ++k) {
    v->bc[k] = c->ts_bc[k];
    v->Tb[k] = c->ts_Tb[k];
  }
  v->c = c->c;
  v->dt = c->dt;
  v->comp_unit = c->comp_unit;
  v->Kap0 = c->ts_Kap0;
  v->conv_type = c->ts_conv_type;
  v->maxit_rte = c->ts_maxit;
  v->conv_ho = c->ts_conv_ho;
  v->stream = c->stream;
  v->dx = c->d_dx;
  v->dy = c->d_dy;
  v->area = c->d_area;
  v->T = c->d_T;
  v->kap64 = c->d_kap64;
  v->omx = c->omx.data();
  v->omy = c->omy.data();
  v->w = c->w.data();
  v->nu = c->ts_nu.data();
  v->cv = c->d_cv;
  v->law = c->ts_law;
  v->kmult = c->d_kmult;
  v->nu_dev = c->d_nu;
  return TRT_OK;
}

int handle_outer_sweep(trt_ctx* c, bool roll) {
  const unsigned flags = (roll ? TRT_ROLL_STATE : 0u) | TRT_MOMENTS;
  const bool reflective = c->ts_bc[0] > 0 || c->ts_bc[1] > 0 || c->ts_bc[2] > 0 || c->ts_bc[3] > 0;
  int rc;
  if (c->prec == TRT_PREC_FP64) {
    if ((rc = sweep_impl<double>(c, flags))) return rc;
    if (reflective && (rc = bc_update_impl<double>(c, c->ts_bc, c->ts_Tb, c->comp_unit, c->ts_nu.data()))) return rc;
  } else {
    if ((rc = sweep_impl<float>(c, flags))) return rc;
    if (reflective && (rc = bc_update_impl<float>(c, c->ts_bc, c->ts_Tb, c->comp_unit, c->ts_nu.data()))) return rc;
  }
  c->have_moments = true;
  return TRT_OK;
}

int handle_material(trt_ctx* c, double* mgsrc) {
  return c->prec == TRT_PREC_FP64 ? material_update_impl<double>(c, mgsrc) : material_update_impl<float>(c, mgsrc);
}

int handle_conv_reduce(trt_ctx* c, long long n, const double* x, const double* xo, const double* xo2,
                       unsigned long long* dev_out) {
  static const unsigned long long init[5] = {0, 0, 0, 0x7ff0000000000000ULL, 0};
  TRT_CUDA(cudaMemcpyAsync(dev_out, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  trt::conv_reduce_kernel<<<grid_for(n), 256, 0, c->stream>>>(n, x, xo, xo2, dev_out);
  TRT_LAUNCHED();
  TRT_CUDA(cudaGetLastError());
  return TRT_OK;
}

bool handle_convergence(int conv_type, double eps, const double* r, int its, double* norm) {
  return convergence(conv_type, eps, r, its, norm);
}

int handle_check(trt_ctx* c) { return check_err(c); }

void handle_attach(trt_ctx* c, void* obj, void (*release)(void*)) {
  if (c->lo && c->lo_free) {
    cudaStreamSynchronize(c->stream);
    c->lo_free(c->lo);
  }
  c->lo = obj;
  c->lo_free = release;
}

void* handle_attached(trt_ctx* c) { return c->lo; }

}  // namespace trt_host
