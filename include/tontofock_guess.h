/*
 * tontofock_guess.h — kernels of the learned initial-density network.
 *
 * No counterpart in the reference: Tonto starts an SCF from the core Hamiltonian
 * or a promolecule density (molecule.scf.foo:4650-4930).  These entry points train
 * and evaluate the small MLP that proposes a starting density for water clusters;
 * the SCF itself (and hence the converged answer) is unchanged by it.
 *
 * All arrays are FP32 device arrays, row-major; every call is asynchronous on
 * `stream` (a cudaStream_t or NULL).  Return 0 on success, negative on error.
 */
#ifndef TONTOFOCK_GUESS_H
#define TONTOFOCK_GUESS_H

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] (= beta*C +) sum_k A(i,k) B(k,j) (+ bias[j]), then SiLU if act != 0.
 * A(i,k) = A[i*sai + k*sak], B(k,j) = B[k*sbk + j*sbj] (transposes via strides).
 * Zout (optional): the pre-activation values. */
int tf_mlp_gemm(int M, int N, int K, const float* A, long sai, long sak, const float* B, long sbk, long sbj,
                const float* bias, int act, float* Zout, float* C, float beta, void* stream);

/* dZ = dA * silu'(Z), n elements. */
int tf_mlp_silu_bwd(long n, const float* dA, const float* Z, float* dZ, void* stream);

/* db[j] = sum_i dZ[i*N + j]. */
int tf_mlp_colsum(int M, int N, const float* dZ, float* db, void* stream);

/* Weighted squared error: loss_part[b] partial sums (n_blocks of them) of
 * w_i (Y - T)^2 * inv_norm, and dY = 2 w_i (Y - T) inv_norm.  w may be NULL. */
int tf_mlp_mse(int M, int N, const float* Y, const float* T, const float* w, float inv_norm, float* dY,
               float* loss_part, int n_blocks, void* stream);

/* Adam step (bias-corrected at `step` >= 1) with decoupled-from-nothing L2 term
 * weight_decay * p added to the gradient. */
int tf_mlp_adam(long n, float* p, const float* g, float* m, float* v, float lr, float beta1, float beta2, float eps,
                int step, float weight_decay, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TONTOFOCK_GUESS_H */
