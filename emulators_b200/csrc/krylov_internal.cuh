// Shared state of the Lanczos iteration (krylov.cu) and the adjoint (adjoint.cu).
#pragma once

#include "hpsi_kernel.cuh"

namespace emusv {

constexpr int KMAX = 128;  // largest max_krylov_dim supported

// KS_TIMEOUT equals EMUSV_TIMEOUT: the streaming kernels write it on a bounded-wait timeout.
enum KStatus { KS_RUNNING = 0, KS_CONVERGED = 1, KS_HAPPY = 2, KS_MAXDIM = 3, KS_NONFINITE = 4,
               KS_TIMEOUT = EMUSV_TIMEOUT };

struct KState {
    int status;
    int iters;
    int nvec;
    int kerr;  // error word of the streaming kernels (EMUSV_TIMEOUT), read by k_small
    double s0, err, outnorm2;
    double shift;  // sigma: the run works on H - sigma (the previous step's energy), see k_init
    double a_re[KMAX], a_im[KMAX];   // T_H[k][k]   = <v_k, H v_k> - b_k <v_k, v_{k-1}>
    double b_re[KMAX], b_im[KMAX];   // T_H[k-1][k] = ||w_{k-1}|| (= <v_{k-1}, H v_k> exactly)
    double vv_re[KMAX + 2], vv_im[KMAX + 2];  // <v_k, v_{k-1}>: residual non-orthogonality
    double r[KMAX];                  // T_H[k+1][k] = ||w_k||
    double hn[KMAX];                 // ||H v_k||
    double scale[KMAX + 2];          // v_k = scale[k] * stored_k
    double c_re[KMAX + 2], c_im[KMAX + 2];  // result coefficients
    double ocoef[4];  // recurrence coefficients on the stored vectors (fused pass L)
    // H-first iteration: <v_k, (H - sigma) v_k> (real part), and its part from the diagonal
    // and the pass-L tile flips, which the pass producing v_k computes
    double e_re[KMAX];
    double el_re[KMAX + 2], el_im[KMAX + 2];
    unsigned hh_cnt[1040];  // fused pass H: group-1 tiles per super-tile, the item counter
    int lz_flag[KMAX];      // H-first iteration: outcome flag of iteration k (krylov_norms)
};


// One Lanczos run on the device: v0 (with scale 1/||v0||) is basis vector 0, basis
// vectors 1.. are stored unnormalised at basis + k*vec_bytes (k >= 1; slot 0 of `basis`
// holds the partial sums of the two-pass H*psi).  Stops like krylov_exp.py:49-106 (and
// double_krylov.py:79-110, which has the same tests).  Returns an emusv status; the
// run's own outcome is in ks->status.
int lanczos_run(const HamParams &P, int dtype, double dt, const void *v0, KState *ks,
                double *part_h, double *part_o, unsigned char *basis, int capacity,
                double exp_tol, double norm_tol, int maxdim, int hint, bool energy_shift,
                cudaStream_t s, int *status_out);
int read_status(KState *ks, cudaStream_t s, int *out);
// Input norm and KState reset (k_norm2 + k_init); with energy_shift, sigma = the previous
// finished run's sigma + a_re[0] (the workspace must be zeroed before its first run).
int krylov_begin(int dtype, const void *psi_in, i64 D, KState *ks, double *partials, bool energy_shift,
                 cudaStream_t s);
// out = s0 sum_k c_k scale_k stored_k (ks->nvec vectors; stored_0 = psi_in, stored_k at
// basis + k*D), and ks->outnorm2.
int krylov_combine(int dtype, KState *ks, const void *psi_in, const unsigned char *basis, i64 D,
                   void *out, double *partials, cudaStream_t s);
int krylov_stream_grid(i64 D);   // grid of the streaming vector kernels for length D
size_t krylov_header_bytes();    // KState + partial buffers at the head of a workspace

}  // namespace emusv
