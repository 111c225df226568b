// Internal interface between the two translation units of libtrt_sweep.so: the resident handle
// (trt_api.cu) lends its stream, device fields and sweep to the low-order time loop (mgqd.cu).
// Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "trt_sweep.h"

namespace trt_host {

void add_launches(unsigned long long n);   // library-wide launch counter

// What the low-order side reads of a handle.  Device pointers stay valid for the handle's lifetime.
struct HandleView {
  int nx, ny, nm, ng, prec;
  int bc[4];                        // BC_Type (L, B, R, T) of the time loop
  double Tb[4];                     // boundary temperatures (L, B, R, T)
  double c, dt, comp_unit, Kap0;
  int conv_type, maxit_rte;         // CONVERGENCE type and outer-iteration limit of trt_tstep_setup
  double conv_ho;                   // outer-iteration tolerance
  cudaStream_t stream;
  const double *dx, *dy, *area;     // Delx, Dely, A = Delx (x) Dely (FP64, device)
  double* T;                        // temperature (device)
  const double* kap64;              // KapE = KapB = KapR of the latest material update (device)
  const double *omx, *omy, *w;      // direction set (host)
  const double* nu;                 // group edges Nu_g (host, n_g + 1)
  const double* cv;                 // heat capacity per cell (device)
  int law;                          // material law (TRT_LAW_*)
  const double* kmult;              // Kappa_Mult(Mat(i,j)), or kappa0(i,j) of the configurations' law (device)
  const double* nu_dev;             // group edges Nu_g (device, n_g + 1)
};

// Requires trt_tstep_setup to have run on the handle.
int handle_view(trt_ctx* c, HandleView* v);
// One outer-iteration sweep in the handle's precision with the fused moment epilogue (I_crn_old <- I_crn
// first when roll), then RT_BC_UPDATE on reflective sides; enqueued on the handle's stream.
int handle_outer_sweep(trt_ctx* c, bool roll);
// MATERIAL_UPDATE from the device temperature; also writes MGQD_Src = 4 pi KapB Bg into mgsrc.
int handle_material(trt_ctx* c, double* mgsrc);
// Convergence data {max|x-xo|, max|xo-xo2|, max|x|, min|x|, max|1-xo/x|} of n values into dev_out[5]
// (reset first), on the handle's stream.
int handle_conv_reduce(trt_ctx* c, long long n, const double* x, const double* xo, const double* xo2,
                       unsigned long long* dev_out);
// CONVERGENCE (CONVERGENCE_CHECKS.f08:7-44) from that data.
bool handle_convergence(int conv_type, double eps, const double* r, int its, double* norm);
// Synchronise the handle's stream and report a device-side timeout of the sweep.
int handle_check(trt_ctx* c);
// Attach an object to the handle, released by trt_destroy (or by the next attach).
void handle_attach(trt_ctx* c, void* obj, void (*release)(void*));
void* handle_attached(trt_ctx* c);

}  // namespace trt_host
