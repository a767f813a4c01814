/*
 * turbch_les.h -- the learned LES closure of turbchannel_b200: training data produced
 * by the solver itself (box-filtered snapshots, sub-filter stresses), the closure's
 * training and inference kernels (BF16 tensor cores, FP32 accumulation) and its use in
 * a run through tc_set_turb_model(h, TC_TURB_MLP, params).  None of this has a
 * counterpart in the reference, whose only subgrid model is the Smagorinsky fallback
 * (staggered/func_global.h:815-890); it is the closure the task asks for beside it.
 *
 * The closure: nu_t / nu = softplus(MLP(f)), MLP 6 -> 64 -> 64 -> 1 with SiLU, BF16
 * weights and activations.  f: asinh of the five invariants tr(S^2), tr(O^2), tr(S^3),
 * tr(O^2 S), tr(O^2 S^2) of the resolved velocity gradient in wall units (S, O its
 * symmetric and antisymmetric parts times nu/u_tau^2, u_tau = inv_length_scale * visc)
 * and log(1 + y+)/4.  Parameters are a packed float vector of TC_MLP_NPAR values:
 * W1[6][64], b1[64], W2[64][64], b2[64], w3[64], b3 (W[in][out]).
 * Samples (tc_les_filter, tc_les_samples): staggered schemes.  A run with TC_TURB_MLP:
 * staggered (nu_t per cell) and collocated (nu_t per element between 8 nodes, from the
 * element gradient; the inputs are the same physical invariants, so one network serves
 * both at the filter width it was trained for).  Every call returns TC_OK or a TC_E_*
 * code (tc_last_error).
 */
#ifndef TURBCH_LES_H
#define TURBCH_LES_H
#include "turbch.h"

#ifdef __cplusplus
extern "C" {
#endif

#define TC_MLP_NPAR 4673

/* Box filter of width `width` cells in x and y (must divide NX and NY) and `width_z`
 * cells in z (must divide NZ; volume-weighted by the cell heights, so the coarse cells are
 * those of the grid with every width_z-th z-face) of ring level `level`: 10 fields of
 * M = (NX/width)(NY/width)(NZ/width_z) floats, field-major, cells [Z][Y][X]: the means of
 * the cell-centred u, v, w, p, then of uu, vv, ww, uv, uw, vw. */
int tc_les_filter(tc_handle* h, int level, int width, int width_z, float* fields);

/* Training samples of the closure from the same filter: features[M][6] (above) and
 * targets[M] = nu* / nu, nu* = -tau^d_ij S_ij / (2 S_kl S_kl) the least-squares eddy
 * viscosity of the sub-filter stress tau_ij = <u_i u_j> - <u_i><u_j> (negative where the
 * sub-filter scales return energy; 0 where S = 0). */
int tc_les_samples(tc_handle* h, int level, int width, int width_z, float* features, float* targets);

typedef struct tc_mlp tc_mlp;
/* A network on `device` with seeded initial parameters (weights uniform in
 * +-1/sqrt(fan_in) from MT19937-64(seed), biases 0, b3 = -2) and Adam state. */
int tc_mlp_create(int device, unsigned long long seed, tc_mlp** out);
int tc_mlp_destroy(tc_mlp* m);
int tc_mlp_get_params(tc_mlp* m, float* params);       /* TC_MLP_NPAR floats */
int tc_mlp_set_params(tc_mlp* m, const float* params); /* also resets the Adam state */
/* Training data (copied to the device): features[n][6], targets[n]. */
int tc_mlp_set_data(tc_mlp* m, const float* features, const float* targets, long long n);
/* `epochs` passes over the data in consecutive mini-batches of `batch` samples, Adam
 * (beta 0.9, 0.999, eps 1e-8, learning rate lr) on the mean-square error; epoch_loss[e]
 * (optional) is the mean loss of epoch e over its batches. */
int tc_mlp_train(tc_mlp* m, int epochs, long long batch, float lr, float* epoch_loss);
/* Gradient of the mean-square error over n host samples (no update): grad[TC_MLP_NPAR];
 * loss (optional) the error itself. */
int tc_mlp_grad(tc_mlp* m, const float* features, const float* targets, long long n, float* grad, float* loss);
/* out[n] = nu_t / nu for n feature rows. */
int tc_mlp_forward(tc_mlp* m, const float* features, long long n, float* out);

/* Where a run with TC_TURB_MLP on a staggered grid evaluates the closure (no counterpart
 * in the reference, whose Smagorinsky nu_t is a separate pass, staggered/func_global.h:
 * 875-890).  mode 0 (default): a separate pass writes nu_t, the flux kernel reads it;
 * 1: the flux kernel evaluates the network itself for the planes it stages (tile plus a
 * one-cell halo) and also writes nu_t.  Both give the same nu_t and step. */
int tc_set_mlp_fusion(tc_handle* h, int mode);

#ifdef __cplusplus
}
#endif
#endif
