// vr_learned.cuh -- internal interface between the Krylov solvers
// (vr_krylov.cu) and the learned preconditioner (vr_unet.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/vring_b200.h"

namespace vr {

// z = s N(r / s) with s = sqrt(*rr / n) read on the device (rr = r . r),
// r and z device arrays of nr*nz doubles; does nothing once flags[0] is set
int unet_precondition(const vr_unet *u, const double *r, double *z, const double *rr, const int *flags,
                      cudaStream_t s);

// grid of a network (nr, nz)
void unet_dims(const vr_unet *u, int *nr, int *nz);

// The training loss of one sample through the operator of k:
//   e = S y - x, loss = ||e||^2 / ||x||^2, gy = 2 S e / ||x||^2
// y (float, the network output) and x (double) device arrays of nr*nz;
// ||x||^2 is given (xx); adds loss to *loss_acc (device double).
cudaError_t k2d_loss_grad(vr_k2d *k, const float *y, const double *x, double xx, float *gy, double *loss_acc,
                          cudaStream_t s);
// rr[0] = x . x for a device array of nr*nz doubles (deterministic)
cudaError_t k2d_dot_self(vr_k2d *k, const double *x, double *rr, cudaStream_t s);

}  // namespace vr
