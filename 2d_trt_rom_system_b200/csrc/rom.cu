// Reduced-order model path on the device: the POD of QD-factor snapshots that the reference's offline
// decomposer computes (POD_Calc with SVD_Calc_Cntr, Decomposer/DecompSrc/POD_ROUTINES.c:75-120 and
// LA_ROUTINES.c:50-170) and the online reconstruction of a snapshot from it (POD_RECONSTRUCT,
// MainSrc/POD_ROUTINES.f08:372-432).  Declarations and contracts: include/trt_sweep.h.
#include <cublas_v2.h>
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <vector>

#include "trt_sweep.h"
#include "handle_hooks.h"

namespace {

#define ROM_CUDA(expr)                                  \
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

int grid_of(long long n) { return (int)std::min<long long>((n + 255) / 256, 148LL * 32); }

// SVD_Calc_Cntr's centring: center(i) = sum_t X(i, t) / n_t, the sum taken in t order, and the centred
// copy Xc(i, t) = X(i, t) - center(i).  Column t of X starts at X + t * col_stride.
__global__ void center_kernel(long long clen, int n_t, long long col_stride, const double* __restrict__ X,
                              double* __restrict__ center, double* __restrict__ Xc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < clen; i += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int t = 0; t < n_t; ++t) s = s + X[i + col_stride * t];
    const double c = s / (double)n_t;
    center[i] = c;
    for (int t = 0; t < n_t; ++t) Xc[i + clen * t] = X[i + col_stride * t] - c;
  }
}

// out(j, i) = in(i, j) for an (rows x cols) column-major matrix.
__global__ void transpose_kernel(long long rows, long long cols, const double* __restrict__ in, double* __restrict__ out) {
  const long long n = rows * cols;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % rows, j = k / rows;
    out[j + cols * i] = in[k];
  }
}

// POD_RECONSTRUCT: dat(i) = sum_r S(r) U(i, r) V(r, t) (modes in order, each product as (S U) V), then
// + C(i).  Groupwise (gsum = 0): the data vector is n_g blocks of glen values; group g has rank(g) modes,
// packed after those of the earlier groups (offsets off[g] = sum of the earlier ranks): S(off + r),
// U(glen * off + i + glen * r), V(n_t * off + r + rank(g) * t).  Whole space (gsum = 1): one block of len
// values with rank(0) modes.
__global__ void pod_reconstruct_kernel(long long glen, int n_blocks, int n_t, int t, const int* __restrict__ rank,
                                       const long long* __restrict__ off, const double* __restrict__ C,
                                       const double* __restrict__ S, const double* __restrict__ U,
                                       const double* __restrict__ V, double* __restrict__ dat) {
  const long long n = glen * n_blocks;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(k / glen);
    const long long i = k % glen;
    const int rg = rank[g];
    const long long o = off[g];
    const double* Ug = U + glen * o;
    const double* Vg = V + (long long)n_t * o + (long long)rg * t;
    double acc = 0.0;
    for (int r = 0; r < rg; ++r) acc = acc + (S[o + r] * Ug[i + glen * r]) * Vg[r];
    dat[k] = acc + C[k];
  }
}

// DMD_RECONSTRUCT: dat(i) = Re( sum_r B(r) W(i, r) exp(L(r) Time) ) + C(i), modes in order, each term formed as
// (B W) e with the complex products written out as the reference's COMPLEX*16 arithmetic does (re = ac - bd,
// im = ad + bc).  e(r) = exp(L(r) Time) is computed once per mode by the host and passed in.  Groupwise
// (n_blocks > 1): block g has rank(g) modes packed after the earlier blocks' (offsets off[g]).
__global__ void dmd_reconstruct_kernel(long long glen, int n_blocks, const int* __restrict__ rank,
                                       const long long* __restrict__ off, const double* __restrict__ C,
                                       const double2* __restrict__ B, const double2* __restrict__ W,
                                       const double2* __restrict__ E, double* __restrict__ dat) {
  const long long n = glen * n_blocks;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(k / glen);
    const long long i = k % glen;
    const long long o = off[g];
    const double2* Wg = W + glen * o;
    double re = 0.0, im = 0.0;
    for (int r = 0; r < rank[g]; ++r) {
      const double2 b = B[o + r], w = Wg[i + glen * r], e = E[o + r];
      const double pr = b.x * w.x - b.y * w.y, pi = b.x * w.y + b.y * w.x;   // B W
      const double tr = pr * e.x - pi * e.y, ti = pr * e.y + pi * e.x;       // (B W) e
      re = re + tr;
      im = im + ti;
    }
    dat[k] = re + C[k];
  }
}

// Device scratch of the ROM routines: one arena per host thread, grown by whole blocks, from which every call
// takes its temporaries in stack order (a Dev gives back what it took when it goes out of scope).  Repeated
// calls (a POD per group, a reconstruction per time step) then allocate nothing: cudaMalloc and cudaFree cost
// up to milliseconds each, and cudaFree synchronises the device.  Blocks of at most kKeep bytes are kept for
// the next call; larger ones are freed when the outermost Dev goes out of scope.
struct Arena {
  static constexpr size_t kBlock = size_t(64) << 20, kKeep = size_t(256) << 20;
  int device = -1;
  std::vector<std::pair<char*, size_t>> blocks;   // base, capacity
  size_t blk = 0, off = 0;                          // first free byte: block index, offset in it
  int depth = 0;                                    // Devs alive
  void release_large() {   // only with no Dev alive (nothing handed out)
    for (size_t k = blocks.size(); k-- > 0;) {
      if (blocks[k].second > kKeep) {
        cudaFree(blocks[k].first);
        blocks.erase(blocks.begin() + (long)k);
      }
    }
    blk = off = 0;
  }
  void release_all() {
    for (auto& b : blocks) cudaFree(b.first);
    blocks.clear();
    blk = off = 0;
  }
};
Arena& arena() {
  thread_local Arena a;
  return a;
}

struct Dev {
  size_t blk0 = 0, off0 = 0;
  Dev() {
    Arena& a = arena();
    int dev = 0;
    if (a.depth == 0 && cudaGetDevice(&dev) == cudaSuccess && dev != a.device) {
      a.release_all();   // blocks of the device this thread used before
      a.device = dev;
    }
    blk0 = a.blk;
    off0 = a.off;
    ++a.depth;
  }
  ~Dev() {
    Arena& a = arena();
    // what this call took may still be read or written by its launches: wait for them, as the cudaFree of a
    // per-call allocation would
    if (a.blk != blk0 || a.off != off0) cudaDeviceSynchronize();
    a.blk = blk0;
    a.off = off0;
    if (--a.depth == 0) a.release_large();
  }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  template <class T>
  int get(T** out, size_t n) {
    Arena& a = arena();
    const size_t bytes = ((std::max<size_t>(n, 1) * sizeof(T)) + 255) & ~size_t(255);
    for (; a.blk < a.blocks.size(); ++a.blk, a.off = 0) {
      if (a.off + bytes <= a.blocks[a.blk].second) {
        *out = reinterpret_cast<T*>(a.blocks[a.blk].first + a.off);
        a.off += bytes;
        return TRT_OK;
      }
    }
    // a new block after the last; a larger one than kKeep is freed again at the end of the outermost call
    const size_t cap = std::max(bytes, Arena::kBlock);
    void* q = nullptr;
    if (cudaMalloc(&q, cap) != cudaSuccess) {
      cudaGetLastError();
      return TRT_ERR_NOMEM;
    }
    a.blocks.emplace_back(static_cast<char*>(q), cap);
    a.blk = a.blocks.size() - 1;
    a.off = bytes;
    *out = static_cast<T*>(q);
    return TRT_OK;
  }
};

int device_present() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
    cudaGetLastError();
    return TRT_ERR_NODEV;
  }
  return TRT_OK;
}

// cuSOLVER / cuBLAS handles, created once per host thread and device (creating them costs milliseconds) and
// kept until the process exits: destroying them from a thread-exit hook could run after the CUDA runtime has
// been torn down.
struct Handles {
  int device = -1;
  cusolverDnHandle_t s = nullptr;
  cublasHandle_t b = nullptr;
};
int handles(cusolverDnHandle_t* s, cublasHandle_t* b) {
  thread_local Handles h;
  int dev = 0;
  ROM_CUDA(cudaGetDevice(&dev));
  if (h.device != dev) {
    if (h.b) cublasDestroy(h.b);
    if (h.s) cusolverDnDestroy(h.s);
    h.s = nullptr;
    h.b = nullptr;
    h.device = -1;
    if (cusolverDnCreate(&h.s) != CUSOLVER_STATUS_SUCCESS) {
      h.s = nullptr;
      return TRT_ERR_CUDA;
    }
    if (cublasCreate(&h.b) != CUBLAS_STATUS_SUCCESS) {
      h.b = nullptr;
      return TRT_ERR_CUDA;
    }
    h.device = dev;
  }
  *s = h.s;
  if (b) *b = h.b;
  return TRT_OK;
}

// R(n x n) = the upper triangle of the first n rows of A (column-major, leading dimension lda), zero below.
__global__ void upper_kernel(int n, long long lda, const double* __restrict__ A, double* __restrict__ R) {
  const long long nn = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn; k += (long long)gridDim.x * blockDim.x) {
    const long long i = k % n, j = k / n;
    R[k] = i <= j ? A[i + lda * j] : 0.0;
  }
}

// Thin SVD of a tall (m >= n) column-major matrix A, which is overwritten: A = Q R (geqrf), R = U_R S V^T
// (gesvd of the n x n triangle), U = Q [U_R; 0] (ormqr).  Both routes are backward stable; for m >> n this one
// runs the SVD on an n x n matrix instead of the m x n one.  Outputs U (m x n), S (n), VT (n x n).
int thin_svd_tall(cusolverDnHandle_t h, cudaStream_t st, Dev& dv, double* A, int m, int n, double* U, double* S,
                  double* VT) {
  int rc;
  double *tau, *R, *UR, *work;
  int* info;
  if ((rc = dv.get(&tau, (size_t)n)) || (rc = dv.get(&R, (size_t)n * n)) || (rc = dv.get(&UR, (size_t)n * n)) ||
      (rc = dv.get(&info, 3)))
    return rc;
  int l1 = 0, l2 = 0, l3 = 0;
  if (cusolverDnDgeqrf_bufferSize(h, m, n, A, m, &l1) != CUSOLVER_STATUS_SUCCESS ||
      cusolverDnDgesvd_bufferSize(h, n, n, &l2) != CUSOLVER_STATUS_SUCCESS ||
      cusolverDnDormqr_bufferSize(h, CUBLAS_SIDE_LEFT, CUBLAS_OP_N, m, n, n, A, m, tau, U, m, &l3) !=
          CUSOLVER_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  const int lw = std::max(l1, std::max(l2, l3));
  if ((rc = dv.get(&work, (size_t)lw))) return rc;
  if (cusolverDnDgeqrf(h, m, n, A, m, tau, work, lw, info) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
  upper_kernel<<<grid_of((long long)n * n), 256, 0, st>>>(n, m, A, R);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  if (cusolverDnDgesvd(h, 'S', 'S', n, n, R, n, S, UR, n, VT, n, work, lw, nullptr, info + 1) !=
      CUSOLVER_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  ROM_CUDA(cudaMemsetAsync(U, 0, sizeof(double) * (size_t)m * n, st));
  ROM_CUDA(cudaMemcpy2DAsync(U, sizeof(double) * (size_t)m, UR, sizeof(double) * (size_t)n, sizeof(double) * (size_t)n,
                             n, cudaMemcpyDeviceToDevice, st));
  if (cusolverDnDormqr(h, CUBLAS_SIDE_LEFT, CUBLAS_OP_N, m, n, n, A, m, tau, U, m, work, lw, info + 2) !=
      CUSOLVER_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  int hinfo[3] = {0, 0, 0};
  ROM_CUDA(cudaMemcpyAsync(hinfo, info, sizeof(hinfo), cudaMemcpyDeviceToHost, st));
  ROM_CUDA(cudaStreamSynchronize(st));
  if (hinfo[1] > 0) return TRT_ERR_NOCONV;
  if (hinfo[0] || hinfo[1] || hinfo[2]) return TRT_ERR_ARG;
  return TRT_OK;
}

// Centring + thin SVD of the (clen x n_t) matrix whose column t starts at X + t * col_stride (device).
// Outputs on the device: center(clen), umat(clen, k), sig(k), vtmat(k, n_t), k = min(clen, n_t).
int pod_device(const double* X, long long col_stride, long long clen, int n_t, double* center, double* umat,
               double* sig, double* vtmat, cudaStream_t st) {
  const long long k = std::min<long long>(clen, n_t);
  Dev dv;
  double* Xc = nullptr;
  int rc;
  if ((rc = dv.get(&Xc, (size_t)clen * n_t))) return rc;
  center_kernel<<<grid_of(clen), 256, 0, st>>>(clen, n_t, col_stride, X, center, Xc);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  cusolverDnHandle_t h = nullptr;
  if ((rc = handles(&h, nullptr))) return rc;
  if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
  if (clen >= 2LL * n_t) {   // tall-skinny (the usual snapshot block): QR first
    if ((rc = thin_svd_tall(h, st, dv, Xc, (int)clen, n_t, umat, sig, vtmat))) return rc;
    ROM_CUDA(cudaStreamSynchronize(st));
    return TRT_OK;
  }
  // cuSOLVER's gesvd wants rows >= columns: a wide matrix is decomposed through its transpose
  const bool tall = clen >= n_t;
  const int m = (int)(tall ? clen : n_t), n = (int)(tall ? n_t : clen);
  double* A = Xc;
  if (!tall) {
    if ((rc = dv.get(&A, (size_t)clen * n_t))) return rc;
    transpose_kernel<<<grid_of(clen * n_t), 256, 0, st>>>(clen, n_t, Xc, A);
    trt_host::add_launches(1);
    ROM_CUDA(cudaGetLastError());
  }
  double *Um = nullptr, *VT = nullptr, *work = nullptr;
  int* info = nullptr;
  int lwork = 0;
  if ((rc = dv.get(&Um, (size_t)m * n)) || (rc = dv.get(&VT, (size_t)n * n)) || (rc = dv.get(&info, 1))) return rc;
  if (cusolverDnDgesvd_bufferSize(h, m, n, &lwork) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
  if ((rc = dv.get(&work, (size_t)lwork))) return rc;
  if (cusolverDnDgesvd(h, 'S', 'S', m, n, A, m, sig, Um, m, VT, n, work, lwork, nullptr, info) !=
      CUSOLVER_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  int hinfo = 0;
  ROM_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  ROM_CUDA(cudaStreamSynchronize(st));
  if (hinfo != 0) return hinfo > 0 ? TRT_ERR_NOCONV : TRT_ERR_ARG;
  if (tall) {   // X = U S V^T: U is (clen x n_t), V^T is (n_t x n_t)
    ROM_CUDA(cudaMemcpyAsync(umat, Um, sizeof(double) * (size_t)clen * k, cudaMemcpyDeviceToDevice, st));
    ROM_CUDA(cudaMemcpyAsync(vtmat, VT, sizeof(double) * (size_t)k * n_t, cudaMemcpyDeviceToDevice, st));
  } else {      // X^T = U' S V'^T: U = V' = (V'^T)^T is (clen x clen), V^T = U'^T is (clen x n_t)
    transpose_kernel<<<grid_of((long long)n * n), 256, 0, st>>>(n, n, VT, umat);
    trt_host::add_launches(1);
    transpose_kernel<<<grid_of((long long)m * n), 256, 0, st>>>(m, n, Um, vtmat);
    trt_host::add_launches(1);
    ROM_CUDA(cudaGetLastError());
  }
  ROM_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

// LINEAR_INTERPOLATION: v1 = v1 + (xm - x1) (v2 - v1) / (x2 - x1), value by value.
__global__ void linear_interpolation_kernel(double* __restrict__ v1, const double* __restrict__ v2, double xm, double x1,
                                            double x2, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    v1[k] = v1[k] + (xm - x1) * (v2[k] - v1[k]) / (x2 - x1);
}

// Offsets of each block's modes (the sum of the earlier ranks), every rank checked against [0, max_rank].
int mode_offsets(const int* rank, int nb, long long max_rank, std::vector<long long>& off, long long& tot) {
  off.assign((size_t)nb, 0);
  tot = 0;
  for (int g = 0; g < nb; ++g) {
    if (rank[g] < 0 || rank[g] > max_rank) return TRT_ERR_ARG;
    off[g] = tot;
    tot += rank[g];
  }
  return TRT_OK;
}

// POD_RECONSTRUCT of one field (len values; N_g blocks with PODgsum = 0, one with PODgsum = 1) into device memory
// dst at data time level a (1-based); when level b differs, also at b, followed by LINEAR_INTERPOLATION(dst,
// level b, xm, x1, x2), as the reconstruction drivers do.  C, S, U, V are host arrays (uploaded here), or device
// arrays when resident; rank is a host array; the launches go to stream st.
int pod_field(Dev& dv, double* dst, const double* C, const double* S, const double* U, const double* V,
              const int* rank, long long len, int N_g, int N_t, int PODgsum, int a, int b, double xm, double x1,
              double x2, bool resident = false, cudaStream_t st = nullptr) {
  if (!C || !S || !U || !V || !rank || len < 1 || N_t < 1 || a < 1 || a > N_t || b < 1 || b > N_t ||
      (PODgsum != 0 && PODgsum != 1) || (PODgsum == 0 && (N_g < 1 || len % N_g != 0)) || (a != b && !(x2 != x1)))
    return TRT_ERR_ARG;
  const int nb = PODgsum == 0 ? N_g : 1;
  const long long glen = len / nb;
  std::vector<long long> off;
  long long tot = 0;
  int rc = mode_offsets(rank, nb, std::min<long long>(glen, N_t), off, tot);
  if (rc) return rc;
  const double *dC = C, *dS = S, *dU = U, *dV = V;
  int* dr;
  long long* doff;
  if ((rc = dv.get(&dr, (size_t)nb)) || (rc = dv.get(&doff, (size_t)nb))) return rc;
  if (!resident) {
    double *hC, *hS, *hU, *hV;
    if ((rc = dv.get(&hC, (size_t)len)) || (rc = dv.get(&hS, (size_t)tot)) ||
        (rc = dv.get(&hU, (size_t)(glen * tot))) || (rc = dv.get(&hV, (size_t)(N_t * tot))))
      return rc;
    ROM_CUDA(cudaMemcpy(hC, C, (size_t)len * sizeof(double), cudaMemcpyHostToDevice));
    ROM_CUDA(cudaMemcpy(hS, S, (size_t)tot * sizeof(double), cudaMemcpyHostToDevice));
    ROM_CUDA(cudaMemcpy(hU, U, (size_t)(glen * tot) * sizeof(double), cudaMemcpyHostToDevice));
    ROM_CUDA(cudaMemcpy(hV, V, (size_t)(N_t * tot) * sizeof(double), cudaMemcpyHostToDevice));
    dC = hC;
    dS = hS;
    dU = hU;
    dV = hV;
  }
  ROM_CUDA(cudaMemcpyAsync(dr, rank, (size_t)nb * sizeof(int), cudaMemcpyHostToDevice, st));
  ROM_CUDA(cudaMemcpyAsync(doff, off.data(), (size_t)nb * sizeof(long long), cudaMemcpyHostToDevice, st));
  pod_reconstruct_kernel<<<grid_of(len), 256, 0, st>>>(glen, nb, N_t, a - 1, dr, doff, dC, dS, dU, dV, dst);
  trt_host::add_launches(1);
  if (b != a) {
    double* f3;
    if ((rc = dv.get(&f3, (size_t)len))) return rc;
    pod_reconstruct_kernel<<<grid_of(len), 256, 0, st>>>(glen, nb, N_t, b - 1, dr, doff, dC, dS, dU, dV, f3);
    linear_interpolation_kernel<<<grid_of(len), 256, 0, st>>>(dst, f3, xm, x1, x2, len);
    trt_host::add_launches(2);
  }
  ROM_CUDA(cudaGetLastError());
  return TRT_OK;
}

// DMD_RECONSTRUCT of one field (len values; N_g blocks with DMDgsum = 0) at time Time from host arrays (L, B, W
// as interleaved complex doubles) into device memory dst.
int dmd_field(Dev& dv, double* dst, const double* L, const double* B, const double* W, const double* C,
              const int* rank, long long len, int N_g, int DMDgsum, double Time) {
  if (!L || !B || !W || !C || !rank || len < 1 || (DMDgsum != 0 && DMDgsum != 1) ||
      (DMDgsum == 0 && (N_g < 1 || len % N_g != 0)))
    return TRT_ERR_ARG;
  const int nb = DMDgsum == 0 ? N_g : 1;
  const long long glen = len / nb;
  std::vector<long long> off;
  long long tot = 0;
  int rc = mode_offsets(rank, nb, std::numeric_limits<int>::max(), off, tot);
  if (rc) return rc;
  // exp(L(r) Time) once per mode (the reference evaluates it once per mode too, before the value loop)
  std::vector<double> E(2 * (size_t)tot);
  for (long long r = 0; r < tot; ++r) {
    const double zr = L[2 * r] * Time, zi = L[2 * r + 1] * Time;
    const double m = std::exp(zr);
    E[2 * r] = m * std::cos(zi);
    E[2 * r + 1] = m * std::sin(zi);
  }
  double *dC, *dB, *dW, *dE;
  int* dr;
  long long* doff;
  if ((rc = dv.get(&dC, (size_t)len)) || (rc = dv.get(&dB, 2 * (size_t)tot)) ||
      (rc = dv.get(&dW, 2 * (size_t)(glen * tot))) || (rc = dv.get(&dE, 2 * (size_t)tot)) ||
      (rc = dv.get(&dr, (size_t)nb)) || (rc = dv.get(&doff, (size_t)nb)))
    return rc;
  ROM_CUDA(cudaMemcpy(dC, C, (size_t)len * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dB, B, 2 * (size_t)tot * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dW, W, 2 * (size_t)(glen * tot) * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dE, E.data(), E.size() * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dr, rank, (size_t)nb * sizeof(int), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(doff, off.data(), (size_t)nb * sizeof(long long), cudaMemcpyHostToDevice));
  dmd_reconstruct_kernel<<<grid_of(len), 256>>>(glen, nb, dr, doff, dC, reinterpret_cast<const double2*>(dB),
                                               reinterpret_cast<const double2*>(dW),
                                               reinterpret_cast<const double2*>(dE), dst);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  return TRT_OK;
}

}  // namespace

extern "C" {

int trt_pod_calc(const double* data, long long n_t, long long n_g, long long clen, long long g, double* center,
                 double* umat, double* sig, double* vtmat) {
  if (!data || !center || !umat || !sig || !vtmat || n_t < 1 || clen < 1 || n_g < 0 || g < 0 ||
      (n_g > 0 && g >= n_g) || n_t > 65535 || clen > 0x7fffffffLL)   // cuSOLVER takes 32-bit extents
    return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  const long long ng = n_g > 0 ? n_g : 1, k = std::min(clen, n_t);
  // the columns of the chosen group, gathered on the host as gdat_reform does (LA_ROUTINES.c:279-294)
  std::vector<double> cols((size_t)clen * n_t);
  for (long long t = 0; t < n_t; ++t)
    std::copy(data + (size_t)(g * clen + t * ng * clen), data + (size_t)(g * clen + t * ng * clen + clen),
              cols.begin() + (size_t)(t * clen));
  Dev dv;
  double *X, *dc, *du, *ds, *dvt;
  if ((rc = dv.get(&X, cols.size())) || (rc = dv.get(&dc, (size_t)clen)) || (rc = dv.get(&du, (size_t)(clen * k))) ||
      (rc = dv.get(&ds, (size_t)k)) || (rc = dv.get(&dvt, (size_t)(k * n_t))))
    return rc;
  ROM_CUDA(cudaMemcpy(X, cols.data(), cols.size() * sizeof(double), cudaMemcpyHostToDevice));
  if ((rc = pod_device(X, clen, clen, (int)n_t, dc, du, ds, dvt, nullptr))) return rc;
  ROM_CUDA(cudaMemcpy(center, dc, (size_t)clen * sizeof(double), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(umat, du, (size_t)(clen * k) * sizeof(double), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(sig, ds, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(vtmat, dvt, (size_t)(k * n_t) * sizeof(double), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

int trt_pod_calc_device(const double* data, long long n_t, long long n_g, long long clen, long long g, double* center,
                        double* umat, double* sig, double* vtmat, void* stream) {
  if (!data || !center || !umat || !sig || !vtmat || n_t < 1 || clen < 1 || n_g < 0 || g < 0 ||
      (n_g > 0 && g >= n_g) || n_t > 65535 || clen > 0x7fffffffLL)
    return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  const long long ng = n_g > 0 ? n_g : 1;
  return pod_device(data + g * clen, ng * clen, clen, (int)n_t, center, umat, sig, vtmat,
                    static_cast<cudaStream_t>(stream));
}

int trt_pod_reconstruct(double* dat, const double* C, const double* S, const double* U, const double* V,
                        const int* rank, int len, int N_g, int N_t, int t, int PODgsum) {
  if (!dat || !C || !S || !U || !V || !rank || len < 1 || N_t < 1 || t < 1 || t > N_t ||
      (PODgsum != 0 && PODgsum != 1) || (PODgsum == 0 && (N_g < 1 || len % N_g != 0)))
    return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  Dev dv;
  double* dd;
  if ((rc = dv.get(&dd, (size_t)std::max(len, 1))) ||
      (rc = pod_field(dv, dd, C, S, U, V, rank, len, N_g, N_t, PODgsum, t, t, 0.0, 0.0, 0.0)))
    return rc;
  ROM_CUDA(cudaMemcpy(dat, dd, (size_t)len * sizeof(double), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

int trt_pod_reconstruct_device(double* dat, const double* C, const double* S, const double* U, const double* V,
                               const int* rank, const long long* offsets, int len, int n_blocks, int N_t, int t,
                               void* stream) {
  if (!dat || !C || !S || !U || !V || !rank || !offsets || len < 1 || n_blocks < 1 || len % n_blocks != 0 || N_t < 1 ||
      t < 1 || t > N_t)
    return TRT_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  pod_reconstruct_kernel<<<grid_of(len), 256, 0, st>>>(len / n_blocks, n_blocks, N_t, t - 1, rank, offsets, C, S, U, V,
                                                       dat);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  ROM_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

int trt_dmd_reconstruct(double* dat, const double* L, const double* B, const double* W, const double* C,
                        const int* rank, int len, int N_g, int DMDgsum, double Time) {
  if (!dat || !L || !B || !W || !C || !rank || len < 1 || (DMDgsum != 0 && DMDgsum != 1) ||
      (DMDgsum == 0 && (N_g < 1 || len % N_g != 0)))
    return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  Dev dv;
  double* dd;
  if ((rc = dv.get(&dd, (size_t)std::max(len, 1))) ||
      (rc = dmd_field(dv, dd, L, B, W, C, rank, len, N_g, DMDgsum, Time)))
    return rc;
  ROM_CUDA(cudaMemcpy(dat, dd, (size_t)len * sizeof(double), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// DMD of snapshots: DMD_Calc, Coef_Calc and Omega_Calc (Decomposer/DecompSrc/DMD_ROUTINES.c:100-470).
// ------------------------------------------------------------------------------------------------

namespace {

using cplx = std::complex<double>;

// dst = (double2) src for n values.
__global__ void to_complex_kernel(long long n, const double* __restrict__ src, double2* __restrict__ dst) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    dst[k] = make_double2(src[k], 0.0);
}

// Column j of the (rows x cols) complex matrix M divided by lam(j) (complex division as C's operator/).
__global__ void divide_columns_kernel(long long rows, int cols, double2* __restrict__ M, const double2* __restrict__ lam) {
  const long long n = rows * cols;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double2 l = lam[k / rows];
    M[k] = cuCdiv(M[k], l);
  }
}

// SVD_Rank_Calc (LA_ROUTINES.c:178-208) with opt = 1: the first i whose tail energy sqrt(sum_{j>=i} s_j^2),
// relative to the total, is at most svd_eps.
long long svd_rank(long long frank, double svd_eps, const double* s) {
  double fsum = 0.0;
  for (long long i = 0; i < frank; ++i) fsum = fsum + std::pow(s[i], 2);
  fsum = std::sqrt(fsum);
  for (long long i = 0; i < frank; ++i) {
    double sum = 0.0;
    for (long long j = i; j < frank; ++j) sum = sum + std::pow(s[j], 2);
    sum = std::sqrt(sum) / fsum;
    if (sum <= svd_eps) return i;
  }
  return frank;
}

// Omega_Calc (DMD_ROUTINES.c:100-152): the continuous-time exponent log(lambda)/delt with the reference's
// branch choices for the argument.
cplx omega_of(cplx lam, double delt) {
  const double pi = 4.0 * std::atan(1.0);
  const double clam = lam.imag(), rlam = lam.real();
  if (clam == 0.0) {
    if (rlam > 0.0) return cplx(std::log(std::fabs(rlam)) / delt, 0.0);
    if (rlam < 0.0) return cplx(std::log(std::fabs(rlam)), pi) / delt;
    return cplx(0.0, 0.0);   // the reference leaves this entry unset
  }
  if (rlam == 0.0) {
    if (clam > 0.0) return cplx(std::log(std::fabs(clam)), pi / 2.0) / delt;
    return cplx(std::log(std::fabs(clam)), 3.0 * pi / 2.0) / delt;
  }
  double theta = std::atan(std::fabs(clam) / std::fabs(rlam));
  const double radius = std::sqrt(std::pow(rlam, 2) + std::pow(clam, 2));
  if (rlam < 0.0 && clam > 0.0) theta = pi - theta;
  else if (rlam < 0.0 && clam < 0.0) theta += pi;
  else if (rlam > 0.0 && clam < 0.0) theta = 2.0 * pi - theta;
  return cplx(std::log(radius), theta) / delt;
}

// A x = b by LU with partial pivoting (the zgesv of cGaussElim, DMD_ROUTINES.c); A column-major n x n.
int lu_solve(int n, std::vector<cplx> A, std::vector<cplx>& b) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::abs(A[i + (size_t)n * k]) > std::abs(A[p + (size_t)n * k])) p = i;
    if (A[p + (size_t)n * k] == cplx(0.0, 0.0)) return TRT_ERR_NOCONV;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(A[k + (size_t)n * j], A[p + (size_t)n * j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      const cplx f = A[i + (size_t)n * k] / A[k + (size_t)n * k];
      for (int j = k; j < n; ++j) A[i + (size_t)n * j] -= f * A[k + (size_t)n * j];
      b[i] -= f * b[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    cplx s = b[k];
    for (int j = k + 1; j < n; ++j) s -= A[k + (size_t)n * j] * b[j];
    b[k] = s / A[k + (size_t)n * k];
  }
  return TRT_OK;
}

}  // namespace

extern "C" {

int trt_dmd_calc(const double* data, long long N_t, long long N_g, long long clen, long long g, int base_subtract,
                 double svd_eps, double delt, long long* N_modes, double* lambda, double* omega, double* b,
                 double* wmat, double* wmat_proj, double* umat, double* wmat_tild, double* cvec) {
  const long long shift = base_subtract ? 2 : 1;
  if (!data || !N_modes || !lambda || !omega || !b || !wmat || !wmat_proj || !umat || !wmat_tild || !cvec ||
      clen < 1 || N_g < 0 || g < 0 || (N_g > 0 && g >= N_g) || N_t - shift < 1 || N_t > 65535 || !(delt > 0.0) ||
      clen > 0x7fffffffLL)
    return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  const long long ng = N_g > 0 ? N_g : 1, n = N_t - shift, k = std::min(clen, n);
  // block g (gdat_reform), the base vector, X = columns 0..n-1 and Y = columns 1..n, less the base
  auto col = [&](long long t) { return data + (size_t)(g * clen + t * ng * clen); };
  for (long long i = 0; i < clen; ++i) cvec[i] = base_subtract ? col(N_t - 1)[i] : 0.0;
  std::vector<double> X((size_t)clen * n), Y((size_t)clen * n);
  for (long long t = 0; t < n; ++t)
    for (long long i = 0; i < clen; ++i) {
      X[(size_t)(i + clen * t)] = col(t)[i] - cvec[i];
      Y[(size_t)(i + clen * t)] = col(t + 1)[i] - cvec[i];
    }
  Dev dv;
  double *dX, *dY, *dc, *dU, *dS, *dVT;
  if ((rc = dv.get(&dX, X.size())) || (rc = dv.get(&dY, Y.size())) || (rc = dv.get(&dc, (size_t)clen)) ||
      (rc = dv.get(&dU, (size_t)(clen * k))) || (rc = dv.get(&dS, (size_t)k)) || (rc = dv.get(&dVT, (size_t)(k * n))))
    return rc;
  ROM_CUDA(cudaMemcpy(dX, X.data(), X.size() * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dY, Y.data(), Y.size() * sizeof(double), cudaMemcpyHostToDevice));
  // thin SVD of X itself (DMD does not centre; SVD_Calc, LA_ROUTINES.c:95-130)
  cusolverDnHandle_t sh = nullptr;
  cublasHandle_t bh = nullptr;
  if ((rc = handles(&sh, &bh))) return rc;
  if (cusolverDnSetStream(sh, nullptr) != CUSOLVER_STATUS_SUCCESS || cublasSetStream(bh, nullptr) != CUBLAS_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  {
    const bool tall = clen >= n;
    const int m = (int)(tall ? clen : n), nn = (int)(tall ? n : clen);
    double* A = dX;
    if (!tall) {
      if ((rc = dv.get(&A, X.size()))) return rc;
      transpose_kernel<<<grid_of(clen * n), 256>>>(clen, n, dX, A);
      trt_host::add_launches(1);
    }
    double *Um, *VT, *work;
    int* info;
    int lwork = 0;
    if ((rc = dv.get(&Um, (size_t)m * nn)) || (rc = dv.get(&VT, (size_t)nn * nn)) || (rc = dv.get(&info, 1))) return rc;
    if (cusolverDnDgesvd_bufferSize(sh, m, nn, &lwork) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
    if ((rc = dv.get(&work, (size_t)lwork))) return rc;
    if (cusolverDnDgesvd(sh, 'S', 'S', m, nn, A, m, dS, Um, m, VT, nn, work, lwork, nullptr, info) !=
        CUSOLVER_STATUS_SUCCESS)
      return TRT_ERR_CUDA;
    int hinfo = 0;
    ROM_CUDA(cudaMemcpy(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost));
    if (hinfo != 0) return hinfo > 0 ? TRT_ERR_NOCONV : TRT_ERR_ARG;
    if (tall) {
      ROM_CUDA(cudaMemcpy(dU, Um, sizeof(double) * (size_t)(clen * k), cudaMemcpyDeviceToDevice));
      ROM_CUDA(cudaMemcpy(dVT, VT, sizeof(double) * (size_t)(k * n), cudaMemcpyDeviceToDevice));
    } else {
      transpose_kernel<<<grid_of((long long)nn * nn), 256>>>(nn, nn, VT, dU);
      transpose_kernel<<<grid_of((long long)m * nn), 256>>>(m, nn, Um, dVT);
      trt_host::add_launches(2);
    }
    ROM_CUDA(cudaDeviceSynchronize());
  }
  std::vector<double> S((size_t)k), VTh((size_t)(k * n));
  ROM_CUDA(cudaMemcpy(S.data(), dS, S.size() * sizeof(double), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(VTh.data(), dVT, VTh.size() * sizeof(double), cudaMemcpyDeviceToHost));
  const long long xr = svd_eps < 0.0 ? k : svd_rank(k, svd_eps, S.data());
  if (xr < 1) return TRT_ERR_ARG;
  // XV = V(:, 1:xr) S^-1 (n x xr), as the reference scales the transposed V^T
  std::vector<double> XV((size_t)(n * xr));
  for (long long i = 0; i < xr; ++i)
    for (long long j = 0; j < n; ++j) XV[(size_t)(j + n * i)] = VTh[(size_t)(i + k * j)] / S[(size_t)i];
  double *dXV, *dXm, *dAt;
  if ((rc = dv.get(&dXV, XV.size())) || (rc = dv.get(&dXm, (size_t)(clen * xr))) ||
      (rc = dv.get(&dAt, (size_t)(xr * xr))))
    return rc;
  ROM_CUDA(cudaMemcpy(dXV, XV.data(), XV.size() * sizeof(double), cudaMemcpyHostToDevice));
  const double one = 1.0, zero = 0.0;
  // Xm = Y XV (clen x xr); A~ = U(:, 1:xr)^T Xm (xr x xr)
  if (cublasDgemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, (int)clen, (int)xr, (int)n, &one, dY, (int)clen, dXV, (int)n, &zero, dXm,
                  (int)clen) != CUBLAS_STATUS_SUCCESS ||
      cublasDgemm(bh, CUBLAS_OP_T, CUBLAS_OP_N, (int)xr, (int)xr, (int)clen, &one, dU, (int)clen, dXm, (int)clen, &zero,
                  dAt, (int)xr) != CUBLAS_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  // eigenpairs of A~ (EIG_Calc; complex arithmetic throughout, right eigenvectors of unit norm)
  double2 *dAc, *dW, *dVR;
  if ((rc = dv.get(&dAc, (size_t)(xr * xr))) || (rc = dv.get(&dW, (size_t)xr)) || (rc = dv.get(&dVR, (size_t)(xr * xr))))
    return rc;
  to_complex_kernel<<<grid_of(xr * xr), 256>>>(xr * xr, dAt, dAc);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  cusolverDnParams_t prm = nullptr;
  if (cusolverDnCreateParams(&prm) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
  size_t wd = 0, wh = 0;
  cusolverStatus_t es = cusolverDnXgeev_bufferSize(sh, prm, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, xr,
                                                   CUDA_C_64F, dAc, xr, CUDA_C_64F, dW, CUDA_C_64F, nullptr, 1,
                                                   CUDA_C_64F, dVR, xr, CUDA_C_64F, &wd, &wh);
  if (es != CUSOLVER_STATUS_SUCCESS) {
    cusolverDnDestroyParams(prm);
    return TRT_ERR_UNSUPPORTED;
  }
  char* dwork = nullptr;
  int* dinfo = nullptr;
  if ((rc = dv.get(&dwork, wd)) || (rc = dv.get(&dinfo, 1))) {
    cusolverDnDestroyParams(prm);
    return rc;
  }
  std::vector<char> hwork(std::max<size_t>(wh, 1));
  es = cusolverDnXgeev(sh, prm, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, xr, CUDA_C_64F, dAc, xr,
                       CUDA_C_64F, dW, CUDA_C_64F, nullptr, 1, CUDA_C_64F, dVR, xr, CUDA_C_64F, dwork, wd, hwork.data(),
                       wh, dinfo);
  cusolverDnDestroyParams(prm);
  if (es != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_UNSUPPORTED;
  int hinfo = 0;
  ROM_CUDA(cudaMemcpy(&hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost));
  if (hinfo != 0) return hinfo > 0 ? TRT_ERR_NOCONV : TRT_ERR_ARG;
  // modes: wmat = Xm W~ / lambda, wmat_proj = U W~
  double2 *dXmc, *dUc, *dWm, *dWp;
  if ((rc = dv.get(&dXmc, (size_t)(clen * xr))) || (rc = dv.get(&dUc, (size_t)(clen * xr))) ||
      (rc = dv.get(&dWm, (size_t)(clen * xr))) || (rc = dv.get(&dWp, (size_t)(clen * xr))))
    return rc;
  to_complex_kernel<<<grid_of(clen * xr), 256>>>(clen * xr, dXm, dXmc);
  to_complex_kernel<<<grid_of(clen * xr), 256>>>(clen * xr, dU, dUc);
  trt_host::add_launches(2);
  const cuDoubleComplex c1 = make_cuDoubleComplex(1.0, 0.0), c0 = make_cuDoubleComplex(0.0, 0.0);
  if (cublasZgemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, (int)clen, (int)xr, (int)xr, &c1, dXmc, (int)clen, dVR, (int)xr, &c0, dWm,
                  (int)clen) != CUBLAS_STATUS_SUCCESS ||
      cublasZgemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, (int)clen, (int)xr, (int)xr, &c1, dUc, (int)clen, dVR, (int)xr, &c0, dWp,
                  (int)clen) != CUBLAS_STATUS_SUCCESS)
    return TRT_ERR_CUDA;
  divide_columns_kernel<<<grid_of(clen * xr), 256>>>(clen, (int)xr, dWm, dW);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  ROM_CUDA(cudaDeviceSynchronize());
  std::vector<cplx> lam((size_t)xr), Wt((size_t)(xr * xr));
  ROM_CUDA(cudaMemcpy(lam.data(), dW, lam.size() * sizeof(cplx), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(Wt.data(), dVR, Wt.size() * sizeof(cplx), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(wmat, dWm, (size_t)(clen * xr) * sizeof(cplx), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(wmat_proj, dWp, (size_t)(clen * xr) * sizeof(cplx), cudaMemcpyDeviceToHost));
  ROM_CUDA(cudaMemcpy(umat, dU, (size_t)(clen * xr) * sizeof(double), cudaMemcpyDeviceToHost));
  std::memcpy(wmat_tild, Wt.data(), Wt.size() * sizeof(cplx));
  // Coef_Calc: b solves W~ b = U^T a0, a0 the first snapshot (less the base only for an undivided data set,
  // as the reference does)
  std::vector<double> Uh((size_t)(clen * xr));
  std::memcpy(Uh.data(), umat, Uh.size() * sizeof(double));
  std::vector<cplx> rhs((size_t)xr, cplx(0.0, 0.0));
  for (long long r = 0; r < xr; ++r) {
    cplx sacc(0.0, 0.0);
    for (long long i = 0; i < clen; ++i) {
      const double a0 = N_g > 0 ? col(0)[i] : col(0)[i] - cvec[i];
      sacc += cplx(Uh[(size_t)(i + clen * r)], 0.0) * cplx(a0, 0.0);
    }
    rhs[(size_t)r] = sacc;
  }
  if ((rc = lu_solve((int)xr, Wt, rhs))) return rc;
  // A~ is real: dgeev returns its real eigenvalues with a zero imaginary part, the complex solver with one at
  // round-off level, which would move Omega_Calc onto the 2 pi branch.  Such parts are set to zero.
  double lam_max = 0.0;
  for (const cplx& l : lam) lam_max = std::max(lam_max, std::abs(l));
  for (cplx& l : lam)
    if (std::fabs(l.imag()) <= 1e-13 * lam_max) l = cplx(l.real(), 0.0);
  for (long long r = 0; r < xr; ++r) {
    b[2 * r] = rhs[(size_t)r].real();
    b[2 * r + 1] = rhs[(size_t)r].imag();
    lambda[2 * r] = lam[(size_t)r].real();
    lambda[2 * r + 1] = lam[(size_t)r].imag();
    const cplx om = omega_of(lam[(size_t)r], delt);
    omega[2 * r] = om.real();
    omega[2 * r + 1] = om.imag();
  }
  *N_modes = xr;
  return TRT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Grid and time mapping of reconstructed data: FMAP with BILINEAR_INTERPOLATE and LINEAR_INTERPOLATION
// (MainSrc/GRID_FUNCTIONS.f08:14-44, 366-401, 819-836).
// ------------------------------------------------------------------------------------------------

namespace {

// BILINEAR_INTERPOLATE, its branches and operation order.
__device__ __forceinline__ double bilinear(double f11, double f12, double f21, double f22, double x, double x1, double x2,
                                           double y, double y1, double y2) {
  if ((x2 - x1) == 0.0) {
    if ((y2 - y1) == 0.0) return f11;
    const double yy1 = y - y1, yy2 = y2 - y;
    return (f11 * yy2 + f12 * yy1) / (y2 - y1);
  }
  if ((y2 - y1) == 0.0) {
    const double xx1 = x - x1, xx2 = x2 - x;
    return (f11 * xx2 + f21 * xx1) / (x2 - x1);
  }
  const double xx1 = x - x1, xx2 = x2 - x, yy1 = y - y1, yy2 = y2 - y;
  return (f11 * xx2 * yy2 + f21 * xx1 * yy2 + f12 * xx2 * yy1 + f22 * xx1 * yy1) / ((x2 - x1) * (y2 - y1));
}

// FMAP: for each of the flen2 / Glen2 blocks (groups), every point j of grid 2 from the four grid-1 values that
// VMap names (1-based, within the block) and the corner coordinates GMap names (1-based index of an x, its y
// following).  One thread per output value.
__global__ void fmap_kernel(const double* __restrict__ f1, double* __restrict__ f2, const double* __restrict__ G1,
                            const double* __restrict__ G2, const int* __restrict__ GMap, const int* __restrict__ VMap,
                            int Glen1, int Glen2, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long blk = k / Glen2;
    const int j = (int)(k % Glen2);
    const double* f = f1 + blk * (long long)Glen1 - 1;   // 1-based within the block
    const int* vm = VMap + 4 * j;
    const int* gm = GMap + 4 * j;
    f2[k] = bilinear(f[vm[0]], f[vm[2]], f[vm[1]], f[vm[3]], G2[2 * j], G1[gm[0] - 1], G1[gm[3] - 1], G2[2 * j + 1],
                     G1[gm[0]], G1[gm[3]]);
  }
}

}  // namespace

extern "C" {

int trt_fmap(const double* f1, double* f2, const double* Grid1, const double* Grid2, const int* GMap, const int* VMap,
             int Glen1, int Glen2, int flen1, int flen2) {
  if (!f1 || !f2 || !Grid1 || !Grid2 || !GMap || !VMap || Glen1 < 1 || Glen2 < 1 || flen2 % Glen2 != 0 ||
      (long long)(flen2 / Glen2) * Glen1 > flen1)
    return TRT_ERR_ARG;
  // every map entry must name a value of the block and a coordinate pair of grid 1 (checked before any launch)
  for (long long j = 0; j < 4LL * Glen2; ++j)
    if (VMap[j] < 1 || VMap[j] > Glen1 || GMap[j] < 1 || GMap[j] > 2 * Glen1 - 1) return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  Dev dv;
  double *d1, *d2, *g1, *g2;
  int *gm, *vm;
  if ((rc = dv.get(&d1, (size_t)flen1)) || (rc = dv.get(&d2, (size_t)flen2)) || (rc = dv.get(&g1, 2 * (size_t)Glen1)) ||
      (rc = dv.get(&g2, 2 * (size_t)Glen2)) || (rc = dv.get(&gm, 4 * (size_t)Glen2)) || (rc = dv.get(&vm, 4 * (size_t)Glen2)))
    return rc;
  ROM_CUDA(cudaMemcpy(d1, f1, (size_t)flen1 * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(g1, Grid1, 2 * (size_t)Glen1 * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(g2, Grid2, 2 * (size_t)Glen2 * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(gm, GMap, 4 * (size_t)Glen2 * sizeof(int), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(vm, VMap, 4 * (size_t)Glen2 * sizeof(int), cudaMemcpyHostToDevice));
  fmap_kernel<<<grid_of(flen2), 256>>>(d1, d2, g1, g2, gm, vm, Glen1, Glen2, (long long)flen2);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  ROM_CUDA(cudaMemcpy(f2, d2, (size_t)flen2 * sizeof(double), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

int trt_linear_interpolation(double* v1, const double* v2, double xm, double x1, double x2, int len) {
  if (!v1 || !v2 || len < 0 || !(x2 != x1)) return TRT_ERR_ARG;
  if (len == 0) return TRT_OK;
  int rc = device_present();
  if (rc) return rc;
  Dev dv;
  double *a, *b;
  if ((rc = dv.get(&a, (size_t)len)) || (rc = dv.get(&b, (size_t)len))) return rc;
  ROM_CUDA(cudaMemcpy(a, v1, (size_t)len * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(b, v2, (size_t)len * sizeof(double), cudaMemcpyHostToDevice));
  linear_interpolation_kernel<<<grid_of(len), 256>>>(a, b, xm, x1, x2, len);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  ROM_CUDA(cudaMemcpy(v1, a, (size_t)len * sizeof(double), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Grid coordinates and the maps FMAP reads: GRIDMAP_GEN_AVG / _EDGV / _EDGH and MAP_GRIDS
// (MainSrc/GRID_FUNCTIONS.f08:49-133, 222-351).  Host set-up code (no device work), as in the reference.
// ------------------------------------------------------------------------------------------------

extern "C" {

int trt_gridmap_gen(int kind, const double* Delx, const double* Dely, int N_x, int N_y, double* GridMap) {
  if (!Delx || !Dely || !GridMap || N_x < 1 || N_y < 1 || kind < 0 || kind > 2) return TRT_ERR_ARG;
  std::vector<double> xloc((size_t)N_x);
  if (kind == 1) {   // vertical edges: x at the cell faces
    xloc[0] = 0.0;
    for (int i = 1; i < N_x; ++i) xloc[i] = xloc[i - 1] + Delx[i - 1];
  } else {           // cell centres (and horizontal edges): x at the cell centres
    xloc[0] = Delx[0] / 2.0;
    for (int i = 1; i < N_x; ++i) xloc[i] = xloc[i - 1] + (Delx[i - 1] + Delx[i]) / 2.0;
  }
  long long p = 0;
  double yloc = 0.0;
  for (int j = 0; j < N_y; ++j) {
    if (kind != 2) yloc = yloc + Dely[j] / 2.0;
    for (int i = 0; i < N_x; ++i) {
      GridMap[p++] = xloc[i];
      GridMap[p++] = yloc;
    }
    if (kind != 2) yloc = yloc + Dely[j] / 2.0;
    else if (j + 1 < N_y) yloc = yloc + Dely[j];   // horizontal edges: N_y rows of points, N_y - 1 widths used
  }
  return TRT_OK;
}

}  // extern "C"

namespace {

// MAP_GRIDS searching the first len1 values of Grid1, whose array holds len1_array >= len1 values: the boundary
// maps of GENERATE_GRIDS_XY search all but the last point of a side, which a bracket may still reach.
int map_grids_impl(int* Map, const double* Grid1, const double* Grid2, int len1, long long len1_array, int len2,
                   int xlen1, int* Vec_Locs) {
  if (!Map || !Grid1 || !Grid2 || len1 < 2 || len2 < 2 || len1 % 2 || len2 % 2 || xlen1 < 0 || xlen1 % 2 ||
      len1_array < len1)
    return TRT_ERR_ARG;
  auto G1 = [&](long long i) { return Grid1[i - 1]; };   // 1-based, as the reference indexes
  auto G2 = [&](long long j) { return Grid2[j - 1]; };
  long long mp = 0;
  for (long long j = 1; j <= len2; j += 2) {
    double d = std::numeric_limits<double>::max();   // HUGE(0d0)
    long long l[4] = {0, 0, 0, 0};
    for (long long i = 1; i <= len1; i += 2) {   // closest point of grid 1 (DIST), first one on ties
      // DIST's integer powers (xp1 - xp2)**2 are products
      const double ddx = G1(i) - G2(j), ddy = G1(i + 1) - G2(j + 1);
      const double r = std::fabs(std::sqrt(ddx * ddx + ddy * ddy));
      if (r < d) {
        d = r;
        l[0] = i;
      }
    }
    const double dx = G1(l[0]) - G2(j), dy = G1(l[0] + 1) - G2(j + 1);
    if (dx < -1e-10) {
      if (dy < -1e-10) {                 // bottom left
        l[1] = l[0] + 2; l[2] = l[0] + xlen1; l[3] = l[2] + 2;
      } else if (dy > 1e-10) {           // top left
        l[2] = l[0]; l[0] = l[2] - xlen1; l[1] = l[0] + 2; l[3] = l[2] + 2;
      } else {                           // exact left
        l[1] = l[0] + 2; l[2] = l[0]; l[3] = l[1];
      }
    } else if (dx > 1e-10) {
      if (dy < -1e-10) {                 // bottom right
        l[1] = l[0]; l[0] = l[1] - 2; l[2] = l[0] + xlen1; l[3] = l[2] + 2;
      } else if (dy > 1e-10) {           // top right
        l[3] = l[0]; l[1] = l[3] - xlen1; l[0] = l[1] - 2; l[2] = l[3] - 2;
      } else {                           // exact right
        l[1] = l[0]; l[0] = l[1] - 2; l[2] = l[0]; l[3] = l[1];
      }
    } else {
      if (dy < -1e-10) {                 // exact bottom
        l[1] = l[0]; l[2] = l[0] + xlen1; l[3] = l[2];
      } else if (dy > 1e-10) {           // exact top
        l[2] = l[0]; l[0] = l[2] - xlen1; l[1] = l[0]; l[3] = l[2];
      } else {                           // exact point
        l[1] = l[0]; l[2] = l[0]; l[3] = l[0];
      }
    }
    for (int k = 0; k < 4; ++k) {
      // a grid 2 point outside grid 1's extent has no bracketing cell (the reference reads past its arrays)
      if (l[k] < 1 || l[k] > len1_array - 1) return TRT_ERR_ARG;
      Map[mp + k] = (int)l[k];
    }
    mp += 4;
  }
  if (Vec_Locs)
    for (long long j = 0; j < 2LL * len2; ++j) Vec_Locs[j] = (Map[j] + 1) / 2;
  return TRT_OK;
}

}  // namespace

extern "C" {

int trt_map_grids(int* Map, const double* Grid1, const double* Grid2, int len1, int len2, int xlen1, int* Vec_Locs) {
  return map_grids_impl(Map, Grid1, Grid2, len1, len1, len2, xlen1, Vec_Locs);
}

int trt_gridmap_gen_bnd(int side, const double* Del, double pos, int N, double* GridMap) {
  if (!Del || !GridMap || N < 1 || (side != 0 && side != 1)) return TRT_ERR_ARG;
  double loc = 0.0;
  for (int i = 0; i < N; ++i) {   // GRIDMAP_GEN_LR_BND (side 0: x = pos) / GRIDMAP_GEN_BT_BND (side 1: y = pos)
    loc = loc + Del[i] / 2.0;
    GridMap[2 * i] = side == 0 ? pos : loc;
    GridMap[2 * i + 1] = side == 0 ? loc : pos;
    loc = loc + Del[i] / 2.0;
  }
  return TRT_OK;
}

int trt_generate_grids_xy(const double* Delx_d, const double* Dely_d, const double* Delx, const double* Dely,
                          double xlen_d, double ylen_d, double xlen, double ylen, int dN_x, int dN_y, int N_x, int N_y,
                          double* Sim_Grid_Avg, double* Sim_Grid_EdgV, double* Sim_Grid_EdgH, double* Sim_Grid_Bnds,
                          double* Dat_Grid_Avg, double* Dat_Grid_EdgV, double* Dat_Grid_EdgH, double* Dat_Grid_Bnds,
                          int* GMap_xyAvg, int* GMap_xyEdgV, int* GMap_xyEdgH, int* GMap_xyBnds, int* VMap_xyAvg,
                          int* VMap_xyEdgV, int* VMap_xyEdgH, int* VMap_xyBnds) {
  const void* ptrs[] = {Delx_d, Dely_d, Delx, Dely, Sim_Grid_Avg, Sim_Grid_EdgV, Sim_Grid_EdgH, Sim_Grid_Bnds,
                        Dat_Grid_Avg, Dat_Grid_EdgV, Dat_Grid_EdgH, Dat_Grid_Bnds, GMap_xyAvg, GMap_xyEdgV,
                        GMap_xyEdgH, GMap_xyBnds, VMap_xyAvg, VMap_xyEdgV, VMap_xyEdgH, VMap_xyBnds};
  for (const void* q : ptrs)
    if (!q) return TRT_ERR_ARG;
  if (dN_x < 1 || dN_y < 1 || N_x < 1 || N_y < 1) return TRT_ERR_ARG;
  // the data grid padded with a zero-width cell on each side
  std::vector<double> Dx2((size_t)dN_x + 2, 0.0), Dy2((size_t)dN_y + 2, 0.0);
  std::copy(Delx_d, Delx_d + dN_x, Dx2.begin() + 1);
  std::copy(Dely_d, Dely_d + dN_y, Dy2.begin() + 1);
  int rc;
  if ((rc = trt_gridmap_gen(0, Delx, Dely, N_x, N_y, Sim_Grid_Avg)) ||
      (rc = trt_gridmap_gen(1, Delx, Dely, N_x + 1, N_y, Sim_Grid_EdgV)) ||
      (rc = trt_gridmap_gen(2, Delx, Dely, N_x, N_y + 1, Sim_Grid_EdgH)) ||
      (rc = trt_gridmap_gen_bnd(0, Dely, 0.0, N_y, Sim_Grid_Bnds)) ||
      (rc = trt_gridmap_gen_bnd(1, Delx, 0.0, N_x, Sim_Grid_Bnds + 2 * N_y)) ||
      // the reference places the right side at ylen and the top at xlen (equal on its square domains)
      (rc = trt_gridmap_gen_bnd(0, Dely, ylen, N_y, Sim_Grid_Bnds + 2 * (N_y + N_x))) ||
      (rc = trt_gridmap_gen_bnd(1, Delx, xlen, N_x, Sim_Grid_Bnds + 4 * N_y + 2 * N_x)))
    return rc;
  if ((rc = trt_gridmap_gen(0, Dx2.data(), Dy2.data(), dN_x + 2, dN_y + 2, Dat_Grid_Avg)) ||
      (rc = trt_gridmap_gen(1, Delx_d, Dy2.data(), dN_x + 1, dN_y + 2, Dat_Grid_EdgV)) ||
      (rc = trt_gridmap_gen(2, Dx2.data(), Dely_d, dN_x + 2, dN_y + 1, Dat_Grid_EdgH)) ||
      (rc = trt_gridmap_gen_bnd(0, Dy2.data(), 0.0, dN_y + 2, Dat_Grid_Bnds)) ||
      (rc = trt_gridmap_gen_bnd(1, Dx2.data(), 0.0, dN_x + 2, Dat_Grid_Bnds + 2 * dN_y + 4)) ||
      (rc = trt_gridmap_gen_bnd(0, Dy2.data(), ylen_d, dN_y + 2, Dat_Grid_Bnds + 2 * (dN_y + dN_x) + 8)) ||
      (rc = trt_gridmap_gen_bnd(1, Dx2.data(), xlen_d, dN_x + 2, Dat_Grid_Bnds + 4 * dN_y + 2 * dN_x + 12)))
    return rc;
  const int la = 2 * (dN_x + 2) * (dN_y + 2), lv = 2 * (dN_x + 1) * (dN_y + 2), lh = 2 * (dN_x + 2) * (dN_y + 1);
  if ((rc = map_grids_impl(GMap_xyAvg, Dat_Grid_Avg, Sim_Grid_Avg, la, la, 2 * N_x * N_y, 2 * (dN_x + 2), VMap_xyAvg)) ||
      (rc = map_grids_impl(GMap_xyEdgV, Dat_Grid_EdgV, Sim_Grid_EdgV, lv, lv, 2 * (N_x + 1) * N_y, 2 * (dN_x + 1),
                           VMap_xyEdgV)) ||
      (rc = map_grids_impl(GMap_xyEdgH, Dat_Grid_EdgH, Sim_Grid_EdgH, lh, lh, 2 * N_x * (N_y + 1), 2 * (dN_x + 2),
                           VMap_xyEdgH)))
    return rc;
  // boundary maps: each side's search covers all but its last point set entry (whose array holds one more the
  // brackets may reach); the reference passes the left side's counts for all four sides, which is the same on
  // its square grids and reads past its arrays on others
  const int lby = 2 * dN_y + 2, lbx = 2 * dN_x + 2;
  if ((rc = map_grids_impl(GMap_xyBnds, Dat_Grid_Bnds, Sim_Grid_Bnds, lby, lby + 2, 2 * N_y, 2, VMap_xyBnds)) ||
      (rc = map_grids_impl(GMap_xyBnds + 4 * N_y, Dat_Grid_Bnds + 2 * dN_y + 4, Sim_Grid_Bnds + 2 * N_y, lbx,
                           lbx + 2, 2 * N_x, 0, VMap_xyBnds + 4 * N_y)) ||
      (rc = map_grids_impl(GMap_xyBnds + 4 * (N_y + N_x), Dat_Grid_Bnds + 2 * (dN_y + dN_x) + 8,
                           Sim_Grid_Bnds + 2 * (N_y + N_x), lby, lby + 2, 2 * N_y, 2, VMap_xyBnds + 4 * (N_y + N_x))) ||
      (rc = map_grids_impl(GMap_xyBnds + 8 * N_y + 4 * N_x, Dat_Grid_Bnds + 4 * dN_y + 2 * dN_x + 12,
                           Sim_Grid_Bnds + 4 * N_y + 2 * N_x, lbx, lbx + 2, 2 * N_x, 0,
                           VMap_xyBnds + 8 * N_y + 4 * N_x)))
    return rc;
  return TRT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Time map and boundary helpers of the ROM reconstruction: GENERATE_GRIDS_T, COLLECT_LR_BND, COLLECT_BT_BND,
// COLLECT_CRN_BND, EXTND_BT_BND, EXTND_LR_BND, AVG_APND_BND (MainSrc/GRID_FUNCTIONS.f08:406-656, 754-814).
// Host code; each loop keeps the reference's traversal (pointers advanced in its order, 0-based here).
// ------------------------------------------------------------------------------------------------

extern "C" {

int trt_generate_grids_t(double Delt_d, double Delt, double Start_Time_d, double Start_Time, int dN_t, int N_t,
                         double* Sim_TGrid, double* Dat_TGrid, int* TMap) {
  if (!Sim_TGrid || !Dat_TGrid || !TMap || dN_t < 1 || N_t < 1) return TRT_ERR_ARG;
  Dat_TGrid[0] = Start_Time_d + Delt_d;
  for (int j = 1; j < dN_t; ++j) Dat_TGrid[j] = Dat_TGrid[j - 1] + Delt_d;
  Sim_TGrid[0] = Start_Time + Delt;
  for (int j = 1; j < N_t; ++j) Sim_TGrid[j] = Sim_TGrid[j - 1] + Delt;
  int k = 0;
  for (int i = 0; i < N_t; ++i) {
    const double ts = Sim_TGrid[i];
    if (Dat_TGrid[0] >= ts) {
      TMap[k] = 1;
      TMap[++k] = 1;
    } else if (Dat_TGrid[dN_t - 1] <= ts) {
      TMap[k] = dN_t;
      TMap[++k] = dN_t;
    } else {
      for (int j = 1; j < dN_t; ++j) {   // data levels 2..dN_t (1-based)
        if (std::fabs(Dat_TGrid[j] - ts) / Dat_TGrid[j] <= 1e-14) {
          TMap[k] = j + 1;
          TMap[++k] = j + 1;
          break;
        } else if (Dat_TGrid[j] > ts) {
          TMap[k] = j + 1;
          TMap[++k] = j;
          break;
        }
      }
    }
    ++k;
  }
  return TRT_OK;
}

int trt_collect_lr_bnd(double* bnd, const double* f, int N_g, int N_y, int N_x) {
  if (!bnd || !f || N_g < 1 || N_y < 1 || N_x < 1) return TRT_ERR_ARG;
  long long p1 = 0, p2 = 0;   // 1-based positions as the reference advances them
  for (int g = 0; g < N_g; ++g)
    for (int j = 0; j < N_y; ++j) {
      p1 += 1;
      bnd[p2++] = f[p1 - 1];
      p1 += N_x - 1;
      bnd[p2++] = f[p1 - 1];
    }
  return TRT_OK;
}

int trt_collect_bt_bnd(double* bnd, const double* f, int N_g, int N_y, int N_x) {
  if (!bnd || !f || N_g < 1 || N_y < 2 || N_x < 1) return TRT_ERR_ARG;
  long long p1 = 0, p2 = 0;
  for (int g = 0; g < N_g; ++g) {
    for (int i = 0; i < N_x; ++i) bnd[p2++] = f[p1++];
    p1 += (long long)(N_y - 2) * N_x;
    for (int i = 0; i < N_x; ++i) bnd[p2++] = f[p1++];
  }
  return TRT_OK;
}

int trt_collect_crn_bnd(double* bnd, const double* f, int N_g, int N_y, int N_x) {
  if (!bnd || !f || N_g < 1 || N_y < 2 || N_x < 1) return TRT_ERR_ARG;
  long long p1 = 0, p2 = 0;
  for (int g = 0; g < N_g; ++g) {
    p1 += 1;
    bnd[p2++] = f[p1 - 1];
    p1 += N_x - 1;
    bnd[p2++] = f[p1 - 1];
    p1 += (long long)(N_y - 2) * N_x + 1;
    bnd[p2++] = f[p1 - 1];
    p1 += N_x - 1;
    bnd[p2++] = f[p1 - 1];
  }
  return TRT_OK;
}

int trt_extnd_bt_bnd(double* f_out, const double* f_in, int N_g, int N_y, int N_x) {
  if (!f_out || !f_in || N_g < 1 || N_y < 1 || N_x < 1) return TRT_ERR_ARG;
  long long p1 = 0, p2 = 0;
  for (int g = 0; g < N_g; ++g) {
    for (int i = 0; i < N_x; ++i) f_out[p2++] = f_in[p1++];   // bottom row repeated below
    p1 -= N_x;
    for (int j = 0; j < N_y; ++j)
      for (int i = 0; i < N_x; ++i) f_out[p2++] = f_in[p1++];
    p1 -= N_x;
    for (int i = 0; i < N_x; ++i) f_out[p2++] = f_in[p1++];   // top row repeated above
  }
  return TRT_OK;
}

int trt_extnd_lr_bnd(double* f_out, const double* f_in, int N_g, int N_y, int N_x) {
  if (!f_out || !f_in || N_g < 1 || N_y < 1 || N_x < 1) return TRT_ERR_ARG;
  long long p1 = 0, p2 = 0;
  for (int g = 0; g < N_g; ++g)
    for (int j = 0; j < N_y; ++j) {
      f_out[p2++] = f_in[p1];                                 // first value of the row repeated on the left
      for (int i = 0; i < N_x; ++i) f_out[p2++] = f_in[p1++];
      f_out[p2++] = f_in[p1 - 1];                             // last value repeated on the right
    }
  return TRT_OK;
}

int trt_avg_apnd_bnd(double* f_out, const double* f_in, const double* LR_Bnd, const double* BT_Bnd,
                     const double* Crn_Bnd, int N_g, int N_y, int N_x) {
  if (!f_out || !f_in || !LR_Bnd || !BT_Bnd || !Crn_Bnd || N_g < 1 || N_y < 1 || N_x < 1) return TRT_ERR_ARG;
  long long po = 0, pi = 0, plr = 0, pbt = 0, pc = 0;
  for (int g = 0; g < N_g; ++g) {
    f_out[po++] = Crn_Bnd[pc++];
    for (int i = 0; i < N_x; ++i) f_out[po++] = BT_Bnd[pbt++];
    f_out[po++] = Crn_Bnd[pc++];
    for (int j = 0; j < N_y; ++j) {
      f_out[po++] = LR_Bnd[plr++];
      for (int i = 0; i < N_x; ++i) f_out[po++] = f_in[pi++];
      f_out[po++] = LR_Bnd[plr++];
    }
    f_out[po++] = Crn_Bnd[pc++];
    for (int i = 0; i < N_x; ++i) f_out[po++] = BT_Bnd[pbt++];
    f_out[po++] = Crn_Bnd[pc++];
  }
  return TRT_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Online reconstruction drivers: POD_RECONSTRUCT_fg / _BCg (MainSrc/POD_ROUTINES.f08:28-353) and
// DMD_RECONSTRUCT_fg / _BCg (MainSrc/DMD_ROUTINES.f08:131-424).  Every field is reconstructed on the data grid
// (POD: at one data time level, or at the two that bracket the step with the linear time interpolation between
// them; DMD: at the step's time), padded with the values the reference appends for the mapping (EXTND_BT_BND,
// EXTND_LR_BND, AVG_APND_BND of COLLECT_*_BND values; the boundary factors' end values repeated) and mapped to
// the simulation grid by FMAP, all on the device.  The padding only moves values, so every output equals the
// reference's sequence of calls.
// ------------------------------------------------------------------------------------------------

namespace {

enum PadKind { PAD_BT = 0, PAD_LR = 1, PAD_AVG_XX = 2, PAD_AVG_YY = 3 };

__device__ __forceinline__ int clamp_to(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// One padded field per group from an ny x nx field f.  PAD_BT: EXTND_BT_BND (first and last rows repeated below
// and above; ny + 2 rows).  PAD_LR: EXTND_LR_BND (first and last columns repeated; nx + 2 columns).  PAD_AVG_XX
// / PAD_AVG_YY: AVG_APND_BND (ny + 2 by nx + 2) of a cell field framed by its own first/last rows, columns and
// corners, except the left/right columns, which XX takes from the first and last columns of the vertical-edge
// field side (ny by nx + 1), and the bottom/top rows, which YY takes from the first and last rows of the
// horizontal-edge field side (ny + 1 by nx).
__global__ void pad_kernel(int kind, const double* __restrict__ f, const double* __restrict__ side, int n_g, int ny,
                           int nx, double* __restrict__ out) {
  const long long R = kind == PAD_LR ? ny : ny + 2, Cc = kind == PAD_BT ? nx : nx + 2;
  const long long n = (long long)n_g * R * Cc;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const long long g = k / (R * Cc), rem = k % (R * Cc);
    const int r = (int)(rem / Cc), c = (int)(rem % Cc);
    const double* fg = f + g * ny * nx;
    double v;
    if (kind == PAD_BT)
      v = fg[(long long)clamp_to(r - 1, ny - 1) * nx + c];
    else if (kind == PAD_LR)
      v = fg[(long long)r * nx + clamp_to(c - 1, nx - 1)];
    else if (kind == PAD_AVG_XX && r >= 1 && r <= ny && (c == 0 || c == nx + 1))
      v = side[g * ny * (nx + 1) + (long long)(r - 1) * (nx + 1) + (c == 0 ? 0 : nx)];
    else if (kind == PAD_AVG_YY && c >= 1 && c <= nx && (r == 0 || r == ny + 1))
      v = side[g * (ny + 1) * nx + (long long)(r == 0 ? 0 : ny) * nx + (c - 1)];
    else
      v = fg[(long long)clamp_to(r - 1, ny - 1) * nx + clamp_to(c - 1, nx - 1)];
    out[k] = v;
  }
}

// One boundary factor side per group (the CL2 / CB2 / CR2 / CT2 of the BCg drivers): the side's n values at
// offset off of each group's block of blk values, with the first repeated before and the last after.
__global__ void side_pad_kernel(const double* __restrict__ BC, int n_g, long long blk, long long off, int n,
                                double* __restrict__ out) {
  const long long m = (long long)n_g * (n + 2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x) {
    const long long g = k / (n + 2);
    const int j = (int)(k % (n + 2));
    out[k] = BC[g * blk + off + clamp_to(j - 1, n - 1)];
  }
}

// A point-set pair with its maps (host arrays): the data grid (glen1 points), the simulation grid (glen2) and
// GMap / VMap (4 glen2 entries each).
struct MapSet {
  const double* dat;
  const double* sim;
  const int* gmap;
  const int* vmap;
  long long glen1, glen2;
};

struct DevSet {
  const double *dat, *sim;
  const int *gmap, *vmap;
  int glen1, glen2;
};

// Flags a map entry outside grid 1 (VMap outside [1, glen1], GMap outside [1, 2 glen1 - 1]).
__global__ void check_maps_kernel(const int* __restrict__ gmap, const int* __restrict__ vmap, long long n, int glen1,
                                  int* __restrict__ bad) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    if (vmap[k] < 1 || vmap[k] > glen1 || gmap[k] < 1 || gmap[k] > 2 * glen1 - 1) atomicOr(bad, 1);
}

// Sets whose grids and maps already live on the device: their maps are checked on the device (one pass per set,
// one verdict for all of them read back with a single synchronisation) before any FMAP reads through them.
int device_sets(Dev& dv, const MapSet* s, DevSet* d, int n, cudaStream_t st) {
  for (int k = 0; k < n; ++k)
    if (!s[k].dat || !s[k].sim || !s[k].gmap || !s[k].vmap || s[k].glen1 < 1 || s[k].glen2 < 1 ||
        2 * s[k].glen1 > INT_MAX || 4 * s[k].glen2 > INT_MAX)
      return TRT_ERR_ARG;
  int* bad;
  int rc = dv.get(&bad, 1);
  if (rc) return rc;
  ROM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
  for (int k = 0; k < n; ++k) {
    check_maps_kernel<<<grid_of(4 * s[k].glen2), 256, 0, st>>>(s[k].gmap, s[k].vmap, 4 * s[k].glen2, (int)s[k].glen1,
                                                               bad);
    trt_host::add_launches(1);
    ROM_CUDA(cudaGetLastError());
  }
  int hbad = 0;
  ROM_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  ROM_CUDA(cudaStreamSynchronize(st));
  if (hbad) return TRT_ERR_ARG;
  for (int k = 0; k < n; ++k) d[k] = {s[k].dat, s[k].sim, s[k].gmap, s[k].vmap, (int)s[k].glen1, (int)s[k].glen2};
  return TRT_OK;
}

// Checks a set's maps on the host (every VMap entry a value of the block, every GMap entry an x of grid 1), then
// uploads the grids and maps.
int upload_set(Dev& dv, const MapSet& s, DevSet& d) {
  if (!s.dat || !s.sim || !s.gmap || !s.vmap || s.glen1 < 1 || s.glen2 < 1 || 2 * s.glen1 > INT_MAX ||
      4 * s.glen2 > INT_MAX)
    return TRT_ERR_ARG;
  for (long long j = 0; j < 4 * s.glen2; ++j)
    if (s.vmap[j] < 1 || s.vmap[j] > s.glen1 || s.gmap[j] < 1 || s.gmap[j] > 2 * s.glen1 - 1) return TRT_ERR_ARG;
  int rc;
  double *dat, *sim;
  int *gmap, *vmap;
  if ((rc = dv.get(&dat, 2 * (size_t)s.glen1)) || (rc = dv.get(&sim, 2 * (size_t)s.glen2)) ||
      (rc = dv.get(&gmap, 4 * (size_t)s.glen2)) || (rc = dv.get(&vmap, 4 * (size_t)s.glen2)))
    return rc;
  ROM_CUDA(cudaMemcpy(dat, s.dat, 2 * (size_t)s.glen1 * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(sim, s.sim, 2 * (size_t)s.glen2 * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(gmap, s.gmap, 4 * (size_t)s.glen2 * sizeof(int), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(vmap, s.vmap, 4 * (size_t)s.glen2 * sizeof(int), cudaMemcpyHostToDevice));
  d = {dat, sim, gmap, vmap, (int)s.glen1, (int)s.glen2};
  return TRT_OK;
}

// Host sets are checked and uploaded; resident ones are checked on the device, all n with one synchronisation.
int make_sets(Dev& dv, const MapSet* s, DevSet* d, int n, bool resident, cudaStream_t st) {
  if (resident) return device_sets(dv, s, d, n, st);
  for (int k = 0; k < n; ++k) {
    const int rc = upload_set(dv, s[k], d[k]);
    if (rc) return rc;
  }
  return TRT_OK;
}

// FMAP of n_g blocks of the padded device field f2 (glen1 values each) into out (n_g glen2 values): a device
// array when resident, else a host array (through a device buffer).
int map_out(Dev& dv, const DevSet& d, const double* f2, int n_g, double* out, bool resident = false,
            cudaStream_t st = nullptr) {
  if (!out) return TRT_ERR_ARG;
  const long long n = (long long)n_g * d.glen2;
  double* o = out;
  int rc;
  if (!resident && (rc = dv.get(&o, (size_t)n))) return rc;
  fmap_kernel<<<grid_of(n), 256, 0, st>>>(f2, o, d.dat, d.sim, d.gmap, d.vmap, d.glen1, d.glen2, n);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  if (!resident) ROM_CUDA(cudaMemcpy(out, o, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
  return TRT_OK;
}

int pad(Dev& dv, int kind, const double* f, const double* side, int n_g, int ny, int nx, double** out,
        cudaStream_t st) {
  const long long n = (long long)n_g * (kind == PAD_LR ? ny : ny + 2) * (kind == PAD_BT ? nx : nx + 2);
  int rc = dv.get(out, (size_t)n);
  if (rc) return rc;
  pad_kernel<<<grid_of(n), 256, 0, st>>>(kind, f, side, n_g, ny, nx, *out);
  trt_host::add_launches(1);
  ROM_CUDA(cudaGetLastError());
  return TRT_OK;
}

bool grid_dims_ok(int dN_x, int dN_y, int dN_g, int N_x, int N_y, int N_g) {
  // the drivers map group g of the data to group g of the simulation
  return dN_x >= 1 && dN_y >= 1 && dN_g >= 1 && N_x >= 1 && N_y >= 1 && N_g == dN_g &&
         (long long)(dN_x + 2) * (dN_y + 2) * dN_g <= INT_MAX && (long long)(N_x + 1) * (N_y + 1) * N_g <= INT_MAX;
}

// The data levels bracketing simulation level t (TMap(2t-1), TMap(2t)) and the times of the interpolation.
int time_levels(const int* TMap, const double* Sim_TGrid, const double* Dat_TGrid, int dN_t, int N_t, int t, int& a,
                int& b, double& xm, double& x1, double& x2) {
  if (!TMap || !Sim_TGrid || !Dat_TGrid || dN_t < 1 || t < 1 || t > N_t) return TRT_ERR_ARG;
  a = TMap[2 * t - 2];
  b = TMap[2 * t - 1];
  if (a < 1 || a > dN_t || b < 1 || b > dN_t) return TRT_ERR_ARG;
  xm = Sim_TGrid[t - 1];
  x1 = Dat_TGrid[a - 1];
  x2 = Dat_TGrid[b - 1];
  if (a != b && !(x2 != x1)) return TRT_ERR_ARG;
  if (a == b) x1 = x2 = xm = 0.0;
  return TRT_OK;
}

// Reconstructs field k on the data grid (len values) into device memory; fields in the order of the
// decompositions' arguments: 0 avg_xx, 1 edgV_xx, 2 avg_yy, 3 edgH_yy, 4 edgV_xy, 5 edgH_xy.  Outputs: 0 avg_xx,
// 1 avg_yy, 2 edgV_xx, 3 edgV_xy, 4 edgH_yy, 5 edgH_xy; host arrays, or device arrays (grids and maps too) when
// resident, with the launches on stream st.
template <class Rec>
int fg_driver(Dev& dv, const Rec& rec, double* const out[6], int dN_x, int dN_y, int dN_g, int N_x, int N_y, int N_g,
              const double* const sim[3], const double* const dat[3], const int* const gmap[3],
              const int* const vmap[3], bool resident = false, cudaStream_t st = nullptr) {
  const long long la = (long long)dN_x * dN_y * dN_g, lv = (long long)(dN_x + 1) * dN_y * dN_g,
                  lh = (long long)dN_x * (dN_y + 1) * dN_g;
  const long long lens[6] = {la, lv, la, lh, lv, lh};
  // sets 0 cell averages, 1 vertical edges, 2 horizontal edges, checked before any reconstruction
  const MapSet ms[3] = {{dat[0], sim[0], gmap[0], vmap[0], (long long)(dN_x + 2) * (dN_y + 2), (long long)N_x * N_y},
                        {dat[1], sim[1], gmap[1], vmap[1], (long long)(dN_x + 1) * (dN_y + 2), (long long)(N_x + 1) * N_y},
                        {dat[2], sim[2], gmap[2], vmap[2], (long long)(dN_x + 2) * (dN_y + 1), (long long)N_x * (N_y + 1)}};
  DevSet ds[3];
  int rc;
  if ((rc = make_sets(dv, ms, ds, 3, resident, st))) return rc;
  double* f[6];
  for (int k = 0; k < 6; ++k)
    if ((rc = dv.get(&f[k], (size_t)lens[k])) || (rc = rec(k, lens[k], f[k]))) return rc;
  double* p;
  if ((rc = pad(dv, PAD_BT, f[1], nullptr, dN_g, dN_y, dN_x + 1, &p, st)) ||
      (rc = map_out(dv, ds[1], p, N_g, out[2], resident, st)) ||
      (rc = pad(dv, PAD_BT, f[4], nullptr, dN_g, dN_y, dN_x + 1, &p, st)) ||
      (rc = map_out(dv, ds[1], p, N_g, out[3], resident, st)) ||
      (rc = pad(dv, PAD_LR, f[3], nullptr, dN_g, dN_y + 1, dN_x, &p, st)) ||
      (rc = map_out(dv, ds[2], p, N_g, out[4], resident, st)) ||
      (rc = pad(dv, PAD_LR, f[5], nullptr, dN_g, dN_y + 1, dN_x, &p, st)) ||
      (rc = map_out(dv, ds[2], p, N_g, out[5], resident, st)) ||
      (rc = pad(dv, PAD_AVG_XX, f[0], f[1], dN_g, dN_y, dN_x, &p, st)) ||
      (rc = map_out(dv, ds[0], p, N_g, out[0], resident, st)) ||
      (rc = pad(dv, PAD_AVG_YY, f[2], f[3], dN_g, dN_y, dN_x, &p, st)) ||
      (rc = map_out(dv, ds[0], p, N_g, out[1], resident, st)))
    return rc;
  return TRT_OK;
}

// The four boundary factors from the device vector BC (per group: left dN_y, bottom dN_x, right dN_y, top dN_x
// values), each padded and mapped with its side's slice of the boundary point sets and maps (host arrays, or
// device arrays when resident, like the outputs).
int bcg_sets(Dev& dv, DevSet ds[4], int dN_x, int dN_y, int N_x, int N_y, const double* Sim_Grid_Bnds,
             const double* Dat_Grid_Bnds, const int* GMap, const int* VMap, bool resident, cudaStream_t st) {
  if (!Sim_Grid_Bnds || !Dat_Grid_Bnds || !GMap || !VMap) return TRT_ERR_ARG;
  const int n[4] = {dN_y, dN_x, dN_y, dN_x}, m[4] = {N_y, N_x, N_y, N_x};
  const long long dat_off[4] = {0, 2LL * dN_y + 4, 2LL * (dN_y + dN_x) + 8, 4LL * dN_y + 2LL * dN_x + 12};
  const long long sim_off[4] = {0, 2LL * N_y, 2LL * (N_y + N_x), 4LL * N_y + 2LL * N_x};
  const long long map_off[4] = {0, 4LL * N_y, 4LL * (N_y + N_x), 8LL * N_y + 4LL * N_x};
  MapSet ms[4];
  for (int s = 0; s < 4; ++s)
    ms[s] = {Dat_Grid_Bnds + dat_off[s], Sim_Grid_Bnds + sim_off[s], GMap + map_off[s], VMap + map_off[s], n[s] + 2,
             m[s]};
  return make_sets(dv, ms, ds, 4, resident, st);
}

int bcg_driver(Dev& dv, const double* BC, double* const out[4], int dN_x, int dN_y, int dN_g, int N_g,
               const DevSet ds[4], bool resident = false, cudaStream_t st = nullptr) {
  const long long blk = 2LL * (dN_x + dN_y);
  const int n[4] = {dN_y, dN_x, dN_y, dN_x};
  const long long off[4] = {0, dN_y, (long long)dN_y + dN_x, 2LL * dN_y + dN_x};
  int rc;
  for (int s = 0; s < 4; ++s) {
    double* p;
    if ((rc = dv.get(&p, (size_t)dN_g * (n[s] + 2)))) return rc;
    side_pad_kernel<<<grid_of((long long)dN_g * (n[s] + 2)), 256, 0, st>>>(BC, dN_g, blk, off[s], n[s], p);
    trt_host::add_launches(1);
    ROM_CUDA(cudaGetLastError());
    if ((rc = map_out(dv, ds[s], p, N_g, out[s], resident, st))) return rc;
  }
  return TRT_OK;
}

}  // namespace

extern "C" {

int trt_pod_reconstruct_fg(
    double* fg_avg_xx, double* fg_avg_yy, double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy,
    double* fg_edgH_xy, const double* C_fg_avg_xx, const double* S_fg_avg_xx, const double* U_fg_avg_xx,
    const double* V_fg_avg_xx, const double* C_fg_edgV_xx, const double* S_fg_edgV_xx, const double* U_fg_edgV_xx,
    const double* V_fg_edgV_xx, const double* C_fg_avg_yy, const double* S_fg_avg_yy, const double* U_fg_avg_yy,
    const double* V_fg_avg_yy, const double* C_fg_edgH_yy, const double* S_fg_edgH_yy, const double* U_fg_edgH_yy,
    const double* V_fg_edgH_yy, const double* C_fg_edgV_xy, const double* S_fg_edgV_xy, const double* U_fg_edgV_xy,
    const double* V_fg_edgV_xy, const double* C_fg_edgH_xy, const double* S_fg_edgH_xy, const double* U_fg_edgH_xy,
    const double* V_fg_edgH_xy, const int* rrank_fg_avg_xx, const int* rrank_fg_edgV_xx, const int* rrank_fg_avg_yy,
    const int* rrank_fg_edgH_yy, const int* rrank_fg_edgV_xy, const int* rrank_fg_edgH_xy, int dN_x, int dN_y,
    int dN_g, int dN_t, int N_x, int N_y, int N_g, int N_t, int t, int PODgsum, const double* Sim_Grid_Avg,
    const double* Sim_Grid_EdgV, const double* Sim_Grid_EdgH, const double* Dat_Grid_Avg, const double* Dat_Grid_EdgV,
    const double* Dat_Grid_EdgH, const double* Sim_TGrid, const double* Dat_TGrid, const int* GMap_xyAvg,
    const int* GMap_xyEdgV, const int* GMap_xyEdgH, const int* VMap_xyAvg, const int* VMap_xyEdgV,
    const int* VMap_xyEdgH, const int* TMap) {
  double* const out[6] = {fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy};
  const double* const C[6] = {C_fg_avg_xx, C_fg_edgV_xx, C_fg_avg_yy, C_fg_edgH_yy, C_fg_edgV_xy, C_fg_edgH_xy};
  const double* const S[6] = {S_fg_avg_xx, S_fg_edgV_xx, S_fg_avg_yy, S_fg_edgH_yy, S_fg_edgV_xy, S_fg_edgH_xy};
  const double* const U[6] = {U_fg_avg_xx, U_fg_edgV_xx, U_fg_avg_yy, U_fg_edgH_yy, U_fg_edgV_xy, U_fg_edgH_xy};
  const double* const V[6] = {V_fg_avg_xx, V_fg_edgV_xx, V_fg_avg_yy, V_fg_edgH_yy, V_fg_edgV_xy, V_fg_edgH_xy};
  const int* const rr[6] = {rrank_fg_avg_xx, rrank_fg_edgV_xx, rrank_fg_avg_yy,
                            rrank_fg_edgH_yy, rrank_fg_edgV_xy, rrank_fg_edgH_xy};
  for (int k = 0; k < 6; ++k)
    if (!out[k] || !C[k] || !S[k] || !U[k] || !V[k] || !rr[k]) return TRT_ERR_ARG;
  if (!grid_dims_ok(dN_x, dN_y, dN_g, N_x, N_y, N_g) || dN_t < 1 || (PODgsum != 0 && PODgsum != 1)) return TRT_ERR_ARG;
  int a, b;
  double xm, x1, x2;
  int rc = time_levels(TMap, Sim_TGrid, Dat_TGrid, dN_t, N_t, t, a, b, xm, x1, x2);
  if (rc) return rc;
  if ((rc = device_present())) return rc;
  const double* const sim[3] = {Sim_Grid_Avg, Sim_Grid_EdgV, Sim_Grid_EdgH};
  const double* const dat[3] = {Dat_Grid_Avg, Dat_Grid_EdgV, Dat_Grid_EdgH};
  const int* const gm[3] = {GMap_xyAvg, GMap_xyEdgV, GMap_xyEdgH};
  const int* const vm[3] = {VMap_xyAvg, VMap_xyEdgV, VMap_xyEdgH};
  Dev dv;
  auto rec = [&](int k, long long len, double* dst) {
    return pod_field(dv, dst, C[k], S[k], U[k], V[k], rr[k], len, dN_g, dN_t, PODgsum, a, b, xm, x1, x2);
  };
  return fg_driver(dv, rec, out, dN_x, dN_y, dN_g, N_x, N_y, N_g, sim, dat, gm, vm);
}

int trt_pod_reconstruct_bcg(double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T, const double* C_BCg,
                            const double* S_BCg, const double* U_BCg, const double* V_BCg, const int* rrank_BCg,
                            int dN_x, int dN_y, int dN_g, int dN_t, int N_x, int N_y, int N_g, int N_t, int t,
                            int PODgsum, const double* Sim_Grid_Bnds, const double* Dat_Grid_Bnds,
                            const double* Sim_TGrid, const double* Dat_TGrid, const int* GMap_xyBnds,
                            const int* VMap_xyBnds, const int* TMap) {
  double* const out[4] = {Cg_L, Cg_B, Cg_R, Cg_T};
  for (double* o : out)
    if (!o) return TRT_ERR_ARG;
  if (!C_BCg || !S_BCg || !U_BCg || !V_BCg || !rrank_BCg || !grid_dims_ok(dN_x, dN_y, dN_g, N_x, N_y, N_g) ||
      dN_t < 1 || (PODgsum != 0 && PODgsum != 1))
    return TRT_ERR_ARG;
  int a, b;
  double xm, x1, x2;
  int rc = time_levels(TMap, Sim_TGrid, Dat_TGrid, dN_t, N_t, t, a, b, xm, x1, x2);
  if (rc) return rc;
  if ((rc = device_present())) return rc;
  Dev dv;
  const long long len = 2LL * dN_g * (dN_x + dN_y);
  double* BC;
  DevSet ds[4];
  if ((rc = bcg_sets(dv, ds, dN_x, dN_y, N_x, N_y, Sim_Grid_Bnds, Dat_Grid_Bnds, GMap_xyBnds, VMap_xyBnds, false,
                     nullptr)) ||
      (rc = dv.get(&BC, (size_t)len)) ||
      (rc = pod_field(dv, BC, C_BCg, S_BCg, U_BCg, V_BCg, rrank_BCg, len, dN_g, dN_t, PODgsum, a, b, xm, x1, x2)))
    return rc;
  return bcg_driver(dv, BC, out, dN_x, dN_y, dN_g, N_g, ds);
}

int trt_pod_reconstruct_fg_device(
    double* fg_avg_xx, double* fg_avg_yy, double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy,
    double* fg_edgH_xy, const double* C_fg_avg_xx, const double* S_fg_avg_xx, const double* U_fg_avg_xx,
    const double* V_fg_avg_xx, const double* C_fg_edgV_xx, const double* S_fg_edgV_xx, const double* U_fg_edgV_xx,
    const double* V_fg_edgV_xx, const double* C_fg_avg_yy, const double* S_fg_avg_yy, const double* U_fg_avg_yy,
    const double* V_fg_avg_yy, const double* C_fg_edgH_yy, const double* S_fg_edgH_yy, const double* U_fg_edgH_yy,
    const double* V_fg_edgH_yy, const double* C_fg_edgV_xy, const double* S_fg_edgV_xy, const double* U_fg_edgV_xy,
    const double* V_fg_edgV_xy, const double* C_fg_edgH_xy, const double* S_fg_edgH_xy, const double* U_fg_edgH_xy,
    const double* V_fg_edgH_xy, const int* rrank_fg_avg_xx, const int* rrank_fg_edgV_xx, const int* rrank_fg_avg_yy,
    const int* rrank_fg_edgH_yy, const int* rrank_fg_edgV_xy, const int* rrank_fg_edgH_xy, int dN_x, int dN_y,
    int dN_g, int dN_t, int N_x, int N_y, int N_g, int N_t, int t, int PODgsum, const double* Sim_Grid_Avg,
    const double* Sim_Grid_EdgV, const double* Sim_Grid_EdgH, const double* Dat_Grid_Avg, const double* Dat_Grid_EdgV,
    const double* Dat_Grid_EdgH, const double* Sim_TGrid, const double* Dat_TGrid, const int* GMap_xyAvg,
    const int* GMap_xyEdgV, const int* GMap_xyEdgH, const int* VMap_xyAvg, const int* VMap_xyEdgV,
    const int* VMap_xyEdgH, const int* TMap, void* stream) {
  double* const out[6] = {fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy};
  const double* const C[6] = {C_fg_avg_xx, C_fg_edgV_xx, C_fg_avg_yy, C_fg_edgH_yy, C_fg_edgV_xy, C_fg_edgH_xy};
  const double* const S[6] = {S_fg_avg_xx, S_fg_edgV_xx, S_fg_avg_yy, S_fg_edgH_yy, S_fg_edgV_xy, S_fg_edgH_xy};
  const double* const U[6] = {U_fg_avg_xx, U_fg_edgV_xx, U_fg_avg_yy, U_fg_edgH_yy, U_fg_edgV_xy, U_fg_edgH_xy};
  const double* const V[6] = {V_fg_avg_xx, V_fg_edgV_xx, V_fg_avg_yy, V_fg_edgH_yy, V_fg_edgV_xy, V_fg_edgH_xy};
  const int* const rr[6] = {rrank_fg_avg_xx, rrank_fg_edgV_xx, rrank_fg_avg_yy,
                            rrank_fg_edgH_yy, rrank_fg_edgV_xy, rrank_fg_edgH_xy};
  for (int k = 0; k < 6; ++k)
    if (!out[k] || !C[k] || !S[k] || !U[k] || !V[k] || !rr[k]) return TRT_ERR_ARG;
  if (!grid_dims_ok(dN_x, dN_y, dN_g, N_x, N_y, N_g) || dN_t < 1 || (PODgsum != 0 && PODgsum != 1)) return TRT_ERR_ARG;
  int a, b;
  double xm, x1, x2;
  int rc = time_levels(TMap, Sim_TGrid, Dat_TGrid, dN_t, N_t, t, a, b, xm, x1, x2);
  if (rc) return rc;
  if ((rc = device_present())) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double* const sim[3] = {Sim_Grid_Avg, Sim_Grid_EdgV, Sim_Grid_EdgH};
  const double* const dat[3] = {Dat_Grid_Avg, Dat_Grid_EdgV, Dat_Grid_EdgH};
  const int* const gm[3] = {GMap_xyAvg, GMap_xyEdgV, GMap_xyEdgH};
  const int* const vm[3] = {VMap_xyAvg, VMap_xyEdgV, VMap_xyEdgH};
  Dev dv;
  auto rec = [&](int k, long long len, double* dst) {
    return pod_field(dv, dst, C[k], S[k], U[k], V[k], rr[k], len, dN_g, dN_t, PODgsum, a, b, xm, x1, x2, true, st);
  };
  if ((rc = fg_driver(dv, rec, out, dN_x, dN_y, dN_g, N_x, N_y, N_g, sim, dat, gm, vm, true, st))) return rc;
  ROM_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

int trt_pod_reconstruct_bcg_device(double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T, const double* C_BCg,
                                   const double* S_BCg, const double* U_BCg, const double* V_BCg,
                                   const int* rrank_BCg, int dN_x, int dN_y, int dN_g, int dN_t, int N_x, int N_y,
                                   int N_g, int N_t, int t, int PODgsum, const double* Sim_Grid_Bnds,
                                   const double* Dat_Grid_Bnds, const double* Sim_TGrid, const double* Dat_TGrid,
                                   const int* GMap_xyBnds, const int* VMap_xyBnds, const int* TMap, void* stream) {
  double* const out[4] = {Cg_L, Cg_B, Cg_R, Cg_T};
  for (double* o : out)
    if (!o) return TRT_ERR_ARG;
  if (!C_BCg || !S_BCg || !U_BCg || !V_BCg || !rrank_BCg || !grid_dims_ok(dN_x, dN_y, dN_g, N_x, N_y, N_g) ||
      dN_t < 1 || (PODgsum != 0 && PODgsum != 1))
    return TRT_ERR_ARG;
  int a, b;
  double xm, x1, x2;
  int rc = time_levels(TMap, Sim_TGrid, Dat_TGrid, dN_t, N_t, t, a, b, xm, x1, x2);
  if (rc) return rc;
  if ((rc = device_present())) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Dev dv;
  const long long len = 2LL * dN_g * (dN_x + dN_y);
  double* BC;
  DevSet ds[4];
  if ((rc = bcg_sets(dv, ds, dN_x, dN_y, N_x, N_y, Sim_Grid_Bnds, Dat_Grid_Bnds, GMap_xyBnds, VMap_xyBnds, true,
                     st)) ||
      (rc = dv.get(&BC, (size_t)len)) ||
      (rc = pod_field(dv, BC, C_BCg, S_BCg, U_BCg, V_BCg, rrank_BCg, len, dN_g, dN_t, PODgsum, a, b, xm, x1, x2, true,
                      st)) ||
      (rc = bcg_driver(dv, BC, out, dN_x, dN_y, dN_g, N_g, ds, true, st)))
    return rc;
  ROM_CUDA(cudaStreamSynchronize(st));
  return TRT_OK;
}

int trt_dmd_reconstruct_fg(
    double* fg_avg_xx, double* fg_avg_yy, double* fg_edgV_xx, double* fg_edgV_xy, double* fg_edgH_yy,
    double* fg_edgH_xy, const double* L_fg_avg_xx, const double* B_fg_avg_xx, const double* W_fg_avg_xx,
    const double* C_fg_avg_xx, const double* L_fg_edgV_xx, const double* B_fg_edgV_xx, const double* W_fg_edgV_xx,
    const double* C_fg_edgV_xx, const double* L_fg_avg_yy, const double* B_fg_avg_yy, const double* W_fg_avg_yy,
    const double* C_fg_avg_yy, const double* L_fg_edgH_yy, const double* B_fg_edgH_yy, const double* W_fg_edgH_yy,
    const double* C_fg_edgH_yy, const double* L_fg_edgV_xy, const double* B_fg_edgV_xy, const double* W_fg_edgV_xy,
    const double* C_fg_edgV_xy, const double* L_fg_edgH_xy, const double* B_fg_edgH_xy, const double* W_fg_edgH_xy,
    const double* C_fg_edgH_xy, const int* rrank_fg_avg_xx, const int* rrank_fg_edgV_xx, const int* rrank_fg_avg_yy,
    const int* rrank_fg_edgH_yy, const int* rrank_fg_edgV_xy, const int* rrank_fg_edgH_xy, int dN_x, int dN_y,
    int dN_g, int N_x, int N_y, int N_g, double Time, int DMDgsum, const double* Sim_Grid_Avg,
    const double* Sim_Grid_EdgV, const double* Sim_Grid_EdgH, const double* Dat_Grid_Avg, const double* Dat_Grid_EdgV,
    const double* Dat_Grid_EdgH, const int* GMap_xyAvg, const int* GMap_xyEdgV, const int* GMap_xyEdgH,
    const int* VMap_xyAvg, const int* VMap_xyEdgV, const int* VMap_xyEdgH) {
  double* const out[6] = {fg_avg_xx, fg_avg_yy, fg_edgV_xx, fg_edgV_xy, fg_edgH_yy, fg_edgH_xy};
  const double* const L[6] = {L_fg_avg_xx, L_fg_edgV_xx, L_fg_avg_yy, L_fg_edgH_yy, L_fg_edgV_xy, L_fg_edgH_xy};
  const double* const B[6] = {B_fg_avg_xx, B_fg_edgV_xx, B_fg_avg_yy, B_fg_edgH_yy, B_fg_edgV_xy, B_fg_edgH_xy};
  const double* const W[6] = {W_fg_avg_xx, W_fg_edgV_xx, W_fg_avg_yy, W_fg_edgH_yy, W_fg_edgV_xy, W_fg_edgH_xy};
  const double* const C[6] = {C_fg_avg_xx, C_fg_edgV_xx, C_fg_avg_yy, C_fg_edgH_yy, C_fg_edgV_xy, C_fg_edgH_xy};
  const int* const rr[6] = {rrank_fg_avg_xx, rrank_fg_edgV_xx, rrank_fg_avg_yy,
                            rrank_fg_edgH_yy, rrank_fg_edgV_xy, rrank_fg_edgH_xy};
  for (int k = 0; k < 6; ++k)
    if (!out[k] || !L[k] || !B[k] || !W[k] || !C[k] || !rr[k]) return TRT_ERR_ARG;
  if (!grid_dims_ok(dN_x, dN_y, dN_g, N_x, N_y, N_g) || (DMDgsum != 0 && DMDgsum != 1)) return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  const double* const sim[3] = {Sim_Grid_Avg, Sim_Grid_EdgV, Sim_Grid_EdgH};
  const double* const dat[3] = {Dat_Grid_Avg, Dat_Grid_EdgV, Dat_Grid_EdgH};
  const int* const gm[3] = {GMap_xyAvg, GMap_xyEdgV, GMap_xyEdgH};
  const int* const vm[3] = {VMap_xyAvg, VMap_xyEdgV, VMap_xyEdgH};
  Dev dv;
  auto rec = [&](int k, long long len, double* dst) {
    return dmd_field(dv, dst, L[k], B[k], W[k], C[k], rr[k], len, N_g, DMDgsum, Time);
  };
  return fg_driver(dv, rec, out, dN_x, dN_y, dN_g, N_x, N_y, N_g, sim, dat, gm, vm);
}

int trt_dmd_reconstruct_bcg(double* Cg_L, double* Cg_B, double* Cg_R, double* Cg_T, const double* L_BCg,
                            const double* B_BCg, const double* W_BCg, const double* C_BCg, const int* rrank_BCg,
                            int dN_x, int dN_y, int dN_g, int N_x, int N_y, int N_g, double Time, int DMDgsum,
                            const double* Sim_Grid_Bnds, const double* Dat_Grid_Bnds, const int* GMap_xyBnds,
                            const int* VMap_xyBnds) {
  double* const out[4] = {Cg_L, Cg_B, Cg_R, Cg_T};
  for (double* o : out)
    if (!o) return TRT_ERR_ARG;
  if (!L_BCg || !B_BCg || !W_BCg || !C_BCg || !rrank_BCg || !grid_dims_ok(dN_x, dN_y, dN_g, N_x, N_y, N_g) ||
      (DMDgsum != 0 && DMDgsum != 1))
    return TRT_ERR_ARG;
  int rc = device_present();
  if (rc) return rc;
  Dev dv;
  const long long len = 2LL * dN_g * (dN_x + dN_y);
  double* BC;
  DevSet ds[4];
  if ((rc = bcg_sets(dv, ds, dN_x, dN_y, N_x, N_y, Sim_Grid_Bnds, Dat_Grid_Bnds, GMap_xyBnds, VMap_xyBnds, false,
                     nullptr)) ||
      (rc = dv.get(&BC, (size_t)len)) ||
      (rc = dmd_field(dv, BC, L_BCg, B_BCg, W_BCg, C_BCg, rrank_BCg, len, N_g, DMDgsum, Time)))
    return rc;
  return bcg_driver(dv, BC, out, dN_x, dN_y, dN_g, N_g, ds);
}

}  // extern "C"

extern "C" {

int trt_rrank_calc(const double* sig, double eps, int len, int* rank) {
  if (!sig || !rank || len < 1) return TRT_ERR_ARG;
  double sum1 = 0.0;
  for (int i = 0; i < len; ++i) sum1 = sum1 + sig[i] * sig[i];
  const double eps2 = eps * std::sqrt(sum1);
  *rank = len;
  for (int i = 1; i <= len; ++i) {   // the first i whose discarded tail sig(i+1:len) has norm <= eps2
    double sum2 = 0.0;
    for (int j = i + 1; j <= len; ++j) sum2 = sum2 + sig[j - 1] * sig[j - 1];
    if (std::sqrt(sum2) <= eps2) {
      *rank = i;
      break;
    }
  }
  return TRT_OK;
}

}  // extern "C"
