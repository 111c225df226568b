// Reduced-order model path on the device: the POD of QD-factor snapshots that the reference's offline
// decomposer computes (POD_Calc with SVD_Calc_Cntr, Decomposer/DecompSrc/POD_ROUTINES.c:75-120 and
// LA_ROUTINES.c:50-170) and the online reconstruction of a snapshot from it (POD_RECONSTRUCT,
// MainSrc/POD_ROUTINES.f08:372-432).  Declarations and contracts: include/trt_sweep.h.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
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

struct Dev {
  std::vector<void*> p;
  ~Dev() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  int get(T** out, size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      return TRT_ERR_NOMEM;
    }
    p.push_back(q);
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
  if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
  struct Guard {
    cusolverDnHandle_t h;
    ~Guard() { cusolverDnDestroy(h); }
  } guard{h};
  if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return TRT_ERR_CUDA;
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

}  // namespace

extern "C" {

int trt_pod_calc(const double* data, long long n_t, long long n_g, long long clen, long long g, double* center,
                 double* umat, double* sig, double* vtmat) {
  if (!data || !center || !umat || !sig || !vtmat || n_t < 1 || clen < 1 || n_g < 0 || g < 0 ||
      (n_g > 0 && g >= n_g) || n_t > 65535)
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
      (n_g > 0 && g >= n_g) || n_t > 65535)
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
  const int nb = PODgsum == 0 ? N_g : 1;
  const long long glen = len / nb;
  std::vector<long long> off(nb);
  long long tot = 0;
  for (int g = 0; g < nb; ++g) {
    if (rank[g] < 0 || rank[g] > std::min<long long>(glen, N_t)) return TRT_ERR_ARG;
    off[g] = tot;
    tot += rank[g];
  }
  Dev dv;
  double *dC, *dS, *dU, *dV, *dd;
  int* dr;
  long long* doff;
  if ((rc = dv.get(&dC, (size_t)len)) || (rc = dv.get(&dS, (size_t)tot)) || (rc = dv.get(&dU, (size_t)(glen * tot))) ||
      (rc = dv.get(&dV, (size_t)(N_t * tot))) || (rc = dv.get(&dd, (size_t)len)) || (rc = dv.get(&dr, (size_t)nb)) ||
      (rc = dv.get(&doff, (size_t)nb)))
    return rc;
  ROM_CUDA(cudaMemcpy(dC, C, (size_t)len * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dS, S, (size_t)tot * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dU, U, (size_t)(glen * tot) * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dV, V, (size_t)(N_t * tot) * sizeof(double), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(dr, rank, (size_t)nb * sizeof(int), cudaMemcpyHostToDevice));
  ROM_CUDA(cudaMemcpy(doff, off.data(), (size_t)nb * sizeof(long long), cudaMemcpyHostToDevice));
  if ((rc = trt_pod_reconstruct_device(dd, dC, dS, dU, dV, dr, doff, len, nb, N_t, t, nullptr))) return rc;
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

}  // extern "C"
