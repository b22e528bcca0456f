/* Tensor-core kernels of the learned warm start: 3x3x3 convolutions (stride 1, zero padding 1) of channels-last BF16
 * volumes as implicit GEMMs on the 5th-generation tensor cores (tcgen05.mma, BF16 operands staged in shared memory,
 * FP32 accumulators in tensor memory): the forward pass and the weight gradient of the U-Net that predicts the
 * steady flow of an obstacle channel from its solid mask.  The input gradient is the forward pass of the output
 * gradient with the flipped, transposed weights wt[cin][26 - tap][cout].  No counterpart in the reference.
 *
 * Layouts: x [batch][depth][height][width][cin] BF16; w [cout][27][cin] BF16 with tap = 9 (dz + 1) + 3 (dy + 1) +
 * (dx + 1); y [batch][depth][height][width][cout] BF16; bias [cout] FP32 or NULL.  cin a multiple of 8, cout a
 * multiple of 16 and at most 256.  Pointers are device memory; the calls are asynchronous on `stream` (a
 * cudaStream_t, NULL for the default stream).
 */
#ifndef LBM_B200_WARMSTART_H
#define LBM_B200_WARMSTART_H

#include "lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* y = conv(x, w) + bias, then max(y, 0) when relu != 0. */
LbmStatus lbm_conv3d_forward(const void* x, const void* w, const float* bias, void* y, int batch, int depth, int height,
                             int width, int cin, int cout, int relu, void* stream);

/* dw[cout][27][cin] += sum over the voxels of dy[voxel][cout] x[voxel + tap offset][cin] (zero outside), FP32. */
LbmStatus lbm_conv3d_weight_grad(const void* x, const void* dy, float* dw, int batch, int depth, int height, int width,
                                 int cin, int cout, void* stream);

/* Synchronizes `stream` and returns the status of the convolutions launched since the last call: LBM_OK, or
 * LBM_ERR_DEVICE_TIMEOUT if a wait for the tensor cores gave up (its results are not valid). */
LbmStatus lbm_conv3d_status(void* stream);

/* Polls of the bounded waits for the tensor cores on the current device, for tests of the timeout path: a wait that
 * runs out of polls makes its convolution leave (after the tensor cores finish the stage in flight) and the next
 * lbm_conv3d_status return LBM_ERR_DEVICE_TIMEOUT.  0 makes every wait give up at once; a negative value restores the
 * default (2^24 polls).  No counterpart in the reference. */
LbmStatus lbm_conv3d_set_wait_limit(long long polls);

#ifdef __cplusplus
}
#endif

#endif
