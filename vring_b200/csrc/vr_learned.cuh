// vr_learned.cuh -- internal interface between the Krylov solvers
// (vr_krylov.cu) and the learned preconditioner (vr_unet.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/vring_b200.h"

namespace vr {

// z = s D N(D r / s), D = dscale (per cell, may be NULL for 1) and
// s = sqrt(*ss / n) with ss = sum (D r)^2 read on the device; r and z device
// arrays of nr*nz doubles; does nothing once flags[0] is set
int unet_precondition(const vr_unet *u, const double *r, double *z, const double *dscale, const double *ss,
                      const int *flags, cudaStream_t s);

// grid of a network (nr, nz)
void unet_dims(const vr_unet *u, int *nr, int *nz);

// D^-1/2 of the symmetric operator's diagonal, per cell (device)
const double *k2d_dhalf(const vr_k2d *k);

// Training pair of one sample: r = S e, ss = sum (D r)^2, er = e . r
// (device scalars); r a device array of nr*nz
cudaError_t k2d_train_in(vr_k2d *k, const double *e, double *r, double *ss, double *er, cudaStream_t s);
// Energy-norm loss of the network output yhat (float) for the pair (e, r):
//   y = s D yhat, res = S y - r, loss_acc += (y - e) . res / er,
//   gyhat = 2 s D res / er  (the gradient of the loss with respect to yhat)
cudaError_t k2d_train_grad(vr_k2d *k, const float *yhat, const double *e, const double *r, const double *ss,
                           const double *er, float *gyhat, double *loss_acc, cudaStream_t s);

}  // namespace vr
