// VQE drivers (internal interface).
#pragma once
#include "ops.h"

namespace bsim {

// v <- prod_i exp(thetas[param_idx[i]] G_{op_idx[i]}) |ref>, components applied
// in order i = 0..n_ops-1; |ref> = sum_j ref_val[j] e_{ref_idx[j]}.
template <typename Ti>
int prepare_state(const DevBasis<Ti> *B, const DevNet<Ti> *P, i64 n_ops, const i64 *op_idx, const i64 *param_idx,
                  const double *thetas, const i64 *ref_idx, const double *ref_val, i64 n_ref, double *v,
                  cudaStream_t s);

// Energy, variance and adjoint gradient (host outputs); lv, rv are device work
// vectors of length dim (on return lv holds the uncomputed reference state).
template <typename Ti>
int vqe_energy_grad(const DevBasis<Ti> *B, const DevNet<Ti> *H, const DevNet<Ti> *P, i64 n_ops, const i64 *op_idx,
                    const i64 *param_idx, i64 n_params, const double *thetas, const i64 *ref_idx,
                    const double *ref_val, i64 n_ref, i64 ckpt_every, double *lv, double *rv, double *energy,
                    double *variance, double *grad, cudaStream_t s);

}  // namespace bsim
