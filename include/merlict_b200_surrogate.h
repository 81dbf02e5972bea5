/*
 * merlict_b200_surrogate.h -- the learned surrogate of the photon
 * propagation, on the tensor cores of sm_100a.
 *
 * No counterpart in the reference: merlict traces every photon.  The
 * surrogate is an additional form beside the tracers of merlict_b200.h.  A
 * small MLP maps a photon's entrance state -- support x, y on the entrance
 * plane, direction x, y and wavelength, normalised -- to the probability of
 * reaching a sensor and to a Gaussian mixture over the photon's final hit
 * point on the sensor plane and its direction there; samples of the mixture
 * are given to the sensors by an exact lookup of the hexagonal sensor grid
 * (the HexagonalPrismZ test of merlict/scenery/geometry/HexagonalPrismZ.cpp:
 * 18-29).  The network is trained on photons traced by the exact tracer.
 *
 * Network: 5 inputs, encoded into 128 features (the inputs, sin(pi 2^l x)
 * and cos(pi 2^l x) for 12 octaves l, zeros), then 128 -> 256 -> 256 ->
 * 256 -> 256 -> 73 with SiLU on the four hidden layers.  All five layers
 * are BF16 GEMMs on the tensor cores (tcgen05.mma, FP32 accumulators in
 * tensor memory), operands staged in shared memory by bulk copies; the
 * encoding lets a small network resolve the fine structure of the optics
 * (the lens grid).  Outputs: one reach logit, then
 * for each of 8 mixture components one weight logit, 4 means and 4 log
 * standard deviations (of the normalised targets).
 *
 * Matrices the tensor cores read are kept in "tile images": an R x K BF16
 * matrix (R a multiple of 128, K a multiple of 64) stored as K/64 column
 * blocks of R/8 atoms of 8 rows x 128 bytes, each atom in the 128-byte
 * swizzled layout the tensor cores read, so that any 128-row x 64-column
 * tile is one contiguous 16 KB copy (mlgpu_sg_image_offset).
 *
 * All pointers are device pointers; calls are asynchronous on `cuda_stream`.
 * Device errors (a wait on the tensor cores that timed out) are reported by
 * mlgpu_sg_sync_errors.
 */
#ifndef MERLICT_B200_SURROGATE_H_
#define MERLICT_B200_SURROGATE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLGPU_SG_INPUTS 5
#define MLGPU_SG_OCTAVES 12          /* sin/cos octaves of the input encoding */
#define MLGPU_SG_ENCODED 128         /* encoded input width (5 + 5 * 2 * 12, zero-padded) */
#define MLGPU_SG_HIDDEN 256
#define MLGPU_SG_LAYERS 5            /* weight matrices, all on the tensor cores */
#define MLGPU_SG_COMPONENTS 8
#define MLGPU_SG_DIMS 4
#define MLGPU_SG_OUTPUTS 73          /* 1 + 8 * (1 + 4 + 4) */
#define MLGPU_SG_OUTPUTS_PADDED 80   /* the output layer's N on the tensor cores */

/* Byte offset of element (r, k) in a tile image with `rows` rows. */
size_t mlgpu_sg_image_offset(uint32_t rows, uint32_t r, uint32_t k);

/* C = A B^T on the tensor cores: A is an M x K tile image (rows = a_rows),
 * B an N x K tile image (rows = b_rows), K = 64 * k_chunks; M a multiple of
 * 128, N one of 80, 128 or 256 (per CTA; the grid covers N in steps of N),
 * written as FP32 row-major C[m][n] (ld = N) with bias[n] added if bias is
 * not NULL.  The building block of the surrogate's layers, exposed for
 * testing against a reference GEMM.                                      */
int mlgpu_sg_gemm_f32(const void* a_img, uint32_t a_rows, const void* b_img, uint32_t b_rows,
                      uint32_t m, uint32_t n, uint32_t k_chunks, const float* bias, float* c,
                      void* cuda_stream);

/* Network state: FP32 master weights and biases of the 5 layers, in one
 * buffer of mlgpu_sg_param_count() floats (layer l: W[out][in] then b[out];
 * layer 0 has in = 128 encoded features), plus the BF16 tile images of the
 * weights (forward, and transposed for layers 1..4) in a buffer of
 * mlgpu_sg_image_bytes() bytes.                                           */
uint64_t mlgpu_sg_param_count(void);
uint64_t mlgpu_sg_image_bytes(void);

/* Rebuilds the BF16 weight images from the FP32 master weights. */
int mlgpu_sg_pack_weights(const float* params, void* images, void* cuda_stream);

/* Scratch of a training step or a forward pass over `batch` photons
 * (a multiple of 128); `training` selects the training-step layout.       */
uint64_t mlgpu_sg_workspace_bytes(uint32_t batch, int training);

/* Forward pass: inputs [batch][8] FP32 (the 5 normalised inputs, 3 unused)
 * -> outputs [batch][80] FP32 (the 73 outputs, 7 unused).  One launch:
 * all five layers of each 128-row tile run with the activations in shared
 * and tensor memory.  `workspace` is not used (may be NULL).             */
int mlgpu_sg_forward(const float* params, const void* images, const float* inputs,
                     uint32_t batch, float* outputs, void* workspace, void* cuda_stream);

/* The same forward pass one tensor-core launch per layer, the activations
 * in `workspace` (mlgpu_sg_workspace_bytes(batch, 0) bytes): the form the
 * training step runs.  Its outputs equal mlgpu_sg_forward's bit for bit.  */
int mlgpu_sg_forward_layered(const float* params, const void* images, const float* inputs,
                             uint32_t batch, float* outputs, void* workspace,
                             void* cuda_stream);

/* One training step: forward, the loss (binary cross-entropy of the reach
 * logit plus, for photons that reached a sensor, the negative log-
 * likelihood of the targets [batch][4] under the mixture), backward, and
 * Adam on `params` with moments m, v (each mlgpu_sg_param_count() floats),
 * step number `step` (1-based), then the images are rebuilt.  `reached`
 * is [batch] uint8.  `loss` (may be NULL) receives the batch-mean loss
 * (device FP32, written at the end of the step).  `grads` (may be NULL)
 * receives the gradient of the batch-mean loss (mlgpu_sg_param_count()
 * floats) before the update; with lr = 0 the parameters do not change.  */
int mlgpu_sg_train_step(float* params, void* images, float* adam_m, float* adam_v,
                        const float* inputs, const float* targets, const uint8_t* reached,
                        uint32_t batch, uint32_t step, float lr, float* loss, float* grads,
                        void* workspace, void* cuda_stream);

/* Exact lookup of hexagonal sensors on one plane: cells of a uniform grid
 * list the sensors whose circumscribed circle meets the cell.            */
typedef struct mlgpu_sg_sensor_grid {
    uint32_t num_sensors;
    const float* center;      /* [num_sensors][2] world x, y of each sensor */
    const float* rotation;    /* [num_sensors][2] cos, sin of its rotation about z */
    const float* inner;       /* [num_sensors] inner hex radius */
    const int32_t* sensor_id; /* [num_sensors] */
    double x0, y0, cell;      /* grid origin and cell size */
    uint32_t nx, ny;
    const uint32_t* cell_start;   /* [nx * ny + 1] into cell_items */
    const uint32_t* cell_items;   /* sensor indices */
    double hex_u[2], hex_v[2], hex_w[2];   /* HexagonalPrismZ unit vectors (x, y) */
} mlgpu_sg_sensor_grid;

/* Sampling: per photon i, with Philox stream (photon_offset + i) of `seed`:
 * reach if u < sigmoid(logit); a component by the mixture weights; a point
 * t = mean + sigma * normal (Box-Muller); target = base + scale * t, where
 * base = A x + b (the linear part, `linear` = [4][6]: A row then b) and
 * scale[4]; the sensor by the grid lookup of target x, y.  A photon whose
 * inputs lie outside [-in_limit, in_limit] or whose chosen component has a
 * position sigma (metres) above `sigma_limit` is flagged for exact tracing
 * (fallback[i] = 1, sensor -1).  Outputs: sensor, x, y (target plane),
 * direction x, y, fallback.  With grid = NULL there is no lookup: a photon
 * that reaches gets sensor -2 and its sampled plane point and direction are
 * for the caller to trace on (the exact tracer as the sensor lookup).    */
int mlgpu_sg_sample(const float* outputs, const float* inputs, uint32_t n,
                    const float* linear, const float* scale, float in_limit, float sigma_limit,
                    uint64_t seed, uint64_t photon_offset, const mlgpu_sg_sensor_grid* grid,
                    int32_t* sensor, float* x, float* y, float* cx, float* cy,
                    uint8_t* fallback, void* cuda_stream);

/* First device error since the last call (waits for the stream). */
int mlgpu_sg_sync_errors(void* cuda_stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* MERLICT_B200_SURROGATE_H_ */
