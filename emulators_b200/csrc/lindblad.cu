// Lindblad density-matrix path (C ABI emusv_lindblad_*, emusv_dm_*): the reference's
// RydbergLindbladian (emu_sv/lindblad_operator.py:11-218) applied to a density matrix and
// its Krylov exponential (EvolveDensityMatrix, emu_sv/time_evolution/implementations.py:
// 63-120), for registers up to 15 qubits.
//
// The 2^N x 2^N density matrix is the vector of 2N bits it is in memory (row index in the
// high N bits).  For Hermitian rho the reference's operator
//     L(rho) = Heff rho - (Heff rho)^dag + i sum_k sum_q L_kq rho L_kq^dag
// (Heff = H - 0.5i sum L^dag L on every qubit; lindblad_operator.py:184-211) is, on that
// vector, the 2N-bit operator
//     Heff (x) I  -  I (x) conj(Heff)  +  i sum_q K_q,    K = sum_k L_k (x) conj(L_k):
// the first two terms are a Rydberg-type operator on 2N bits (flips with per-bit
// coefficients, fields, pair couplings U on the row bits and -U on the column bits, the
// noise diagonal), applied by the same streaming H*psi kernels; the jump term couples the
// row bit and the column bit of each qubit (k_lindblad_jumps).  The Krylov vectors of a
// Hermitian rho stay Hermitian, so (Heff rho)^dag = rho Heff^dag holds on every vector the
// exponential touches.
#include <string.h>

#include "hpsi_kernel.cuh"
#include "krylov_internal.cuh"
#include "profile.cuh"

namespace emusv {

int launch_hpsi(int dtype, int mode, const HamParams &P, HpsiArgs A, int max_grid,
                cudaStream_t s, int *grid_out);
int hpsi_tile_bits(int n);
int arnoldi_run(const HamParams &P, const LindbladJumps *J, int dtype, double dt, const void *psi_in,
                void *psi_out, double exp_tolerance, double norm_tolerance, int max_krylov_dim,
                int krylov_dim_hint, void *workspace, size_t workspace_bytes,
                emusv_krylov_info *info, void *stream);

constexpr int DM_MAXQ = EMUSV_MAX_QUBITS / 2;

// The 2N-bit operator Heff (x) I - I (x) conj(Heff) (or, with row_only, Heff (x) I without
// noise: the h_eff of the energy observables, lindblad_operator.py:138-155).  noise: the
// 2x2 matrix -0.5i sum L^dag L (8 doubles) or null.
static bool make_lindblad_params(int n, const double *omegas, const double *deltas, const double *phis,
                                 const double *interaction, const double *noise, bool row_only,
                                 HamParams *P) {
    if (n < 1 || n > DM_MAXQ) return false;
    HamParams H;
    if (!make_params(n, omegas, deltas, phis, interaction, &H)) return false;
    if (noise && !add_noise(noise, &H)) return false;  // Heff's per-qubit terms
    memset(P, 0, sizeof(*P));
    P->n = 2 * n;
    P->real_coef = 0;
    for (int p = 0; p < n; ++p) {
        const int pr = n + p, pc = p;  // row bit and column bit of the qubit at bit p
        P->up_re[pr] = H.up_re[p];
        P->up_im[pr] = H.up_im[p];
        P->dn_re[pr] = H.dn_re[p];
        P->dn_im[pr] = H.dn_im[p];
        P->field[pr] = H.field[p];
        if (!row_only) {  // -conj(Heff) on the column index
            P->up_re[pc] = -H.up_re[p];
            P->up_im[pc] = H.up_im[p];
            P->dn_re[pc] = -H.dn_re[p];
            P->dn_im[pc] = H.dn_im[p];
            P->field[pc] = -H.field[p];
        }
        for (int q = 0; q < n; ++q) {
            P->U[pr * MAXQ + (n + q)] = H.U[p * MAXQ + q];
            if (!row_only) P->U[pc * MAXQ + q] = -H.U[p * MAXQ + q];
        }
    }
    if (H.noisy && !row_only) {
        // row: n00 on every |g>, n11 on every |r>; column: -conj of the same.  Real parts
        // cancel in the constant and sit in the fields; imaginary parts add up to
        // 2 N Im(n00) + Im(n11 - n00) per excitation of either index.
        P->noisy = 1;
        P->dc_re = 0.0;
        P->dc_im = 2.0 * H.dc_im;
        P->dg_im = H.dg_im;
    }
    return true;
}

// noise = -0.5i sum_k L_k^dag L_k (emu_base/jump_lindblad_operators.py:79-93), 8 doubles
static void noise_term(int nops, const double *ops, double *noise) {
    for (int e = 0; e < 8; ++e) noise[e] = 0.0;
    for (int k = 0; k < nops; ++k) {
        const double *L = ops + 8 * k;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                double re = 0.0, im = 0.0;  // (L^dag L)[a][b] = sum_c conj(L[c][a]) L[c][b]
                for (int c = 0; c < 2; ++c) {
                    const double xr = L[(2 * c + a) * 2], xi = -L[(2 * c + a) * 2 + 1];
                    const double yr = L[(2 * c + b) * 2], yi = L[(2 * c + b) * 2 + 1];
                    re += xr * yr - xi * yi;
                    im += xr * yi + xi * yr;
                }
                noise[(2 * a + b) * 2] += 0.5 * im;  // -0.5i (re + i im)
                noise[(2 * a + b) * 2 + 1] += -0.5 * re;
            }
    }
}

static bool make_jumps(int n, int nops, const double *ops, LindbladJumps *J) {
    memset(J, 0, sizeof(*J));
    J->nq = n;
    if (nops < 0 || (nops > 0 && !ops)) return false;
    for (int k = 0; k < nops; ++k) {
        const double *L = ops + 8 * k;  // [a][b] at (2a + b) * 2
        for (int e = 0; e < 8; ++e)
            if (!isfinite(L[e])) return false;
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int i2 = 0; i2 < 2; ++i2)
                    for (int j2 = 0; j2 < 2; ++j2) {
                        // L[i][i2] * conj(L[j][j2])
                        const double ar = L[(2 * i + i2) * 2], ai = L[(2 * i + i2) * 2 + 1];
                        const double br = L[(2 * j + j2) * 2], bi = -L[(2 * j + j2) * 2 + 1];
                        const int e = (i * 2 + j) * 4 + (i2 * 2 + j2);
                        J->K[2 * e] += ar * br - ai * bi;
                        J->K[2 * e + 1] += ar * bi + ai * br;
                    }
    }
    for (int e = 0; e < 16; ++e)
        if (J->K[2 * e] != 0.0 || J->K[2 * e + 1] != 0.0) J->mask |= 1u << e;
    return true;
}

// out[x] += i su sum_q sum_{i',j'} K[(i,j),(i',j')] u[x with the row/column bits of q set to
// (i', j')], (i, j) = the row and column bits of q in x.
template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_lindblad_jumps(const LindbladJumps J, const void *u_, const double *su_p, void *out_, i64 D,
                 const int *gate) {
    typedef typename cvec<R>::T C;
    if (gate && *gate != 0) return;
    const C *u = reinterpret_cast<const C *>(u_);
    C *out = reinterpret_cast<C *>(out_);
    const double su = su_p ? *su_p : 1.0;
    const int n = J.nq;
    for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < D; x += (i64)gridDim.x * blockDim.x) {
        double ar = 0.0, ai = 0.0;
        for (int pc = 0; pc < n; ++pc) {
            const int pr = pc + n;
            const int i = (int)((x >> pr) & 1), j = (int)((x >> pc) & 1);
            const i64 xb = x & ~((i64(1) << pr) | (i64(1) << pc));
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int e = (i * 2 + j) * 4 + t;
                if (!((J.mask >> e) & 1)) continue;
                const i64 y = xb | ((i64)(t >> 1) << pr) | ((i64)(t & 1) << pc);
                const C v = u[y];
                const double kr = J.K[2 * e], ki = J.K[2 * e + 1];
                ar += kr * double(v.x) - ki * double(v.y);
                ai += kr * double(v.y) + ki * double(v.x);
            }
        }
        const C o = out[x];
        // + i su (ar + i ai) = su (-ai + i ar)
        out[x] = cmake<C>(double(o.x) - su * ai, double(o.y) + su * ar);
    }
}

int launch_lindblad_jumps(int dtype, const LindbladJumps &J, const void *u, const double *su,
                          void *out, const int *gate, cudaStream_t s) {
    if (!J.mask) return EMUSV_OK;
    const i64 D = i64(1) << (2 * J.nq);
    i64 g = (D + BLOCK - 1) / BLOCK;
    if (g > (i64)sm_count() * 8) g = (i64)sm_count() * 8;
    {
        ProfScope ps_(PROF_HPSI, s);
        if (dtype == EMUSV_C128)
            k_lindblad_jumps<double><<<(int)g, BLOCK, 0, s>>>(J, u, su, out, D, gate);
        else
            k_lindblad_jumps<float><<<(int)g, BLOCK, 0, s>>>(J, u, su, out, D, gate);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

// dst[r] = sqrt(max(Re rho[r][r], 0)): amplitudes whose |.|^2 are the diagonal of rho, so
// the state-vector occupation and correlation reductions give Tr(rho n_i), Tr(rho n_i n_j).
template <typename R>
__global__ void __launch_bounds__(BLOCK) k_dm_diag_amp(const void *rho_, int n, void *dst_) {
    typedef typename cvec<R>::T C;
    const C *rho = reinterpret_cast<const C *>(rho_);
    C *dst = reinterpret_cast<C *>(dst_);
    const i64 Dn = i64(1) << n;
    for (i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x; r < Dn; r += (i64)gridDim.x * blockDim.x) {
        const double d = double(rho[r * Dn + r].x);
        dst[r] = cmake<C>(d > 0.0 ? sqrt(d) : 0.0, 0.0);
    }
}

// partials[block][0..1] = sum_r X[r][r] (complex trace)
template <typename R>
__global__ void __launch_bounds__(BLOCK) k_dm_trace(const void *X_, int n, double *partials) {
    typedef typename cvec<R>::T C;
    const C *X = reinterpret_cast<const C *>(X_);
    __shared__ double red[(BLOCK / 32) * NRED];
    const i64 Dn = i64(1) << n;
    double acc[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) acc[k] = 0.0;
    for (i64 r = (i64)blockIdx.x * blockDim.x + threadIdx.x; r < Dn; r += (i64)gridDim.x * blockDim.x) {
        const C v = X[r * Dn + r];
        acc[0] += double(v.x);
        acc[1] += double(v.y);
    }
    block_sum<NRED>(acc, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < NRED; ++k) partials[(i64)blockIdx.x * NRED + k] = acc[k];
}

__global__ void k_dm_finish(const double *partials, int nb, double *out) {
    if (threadIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int k = 0; k < nb; ++k) {
        a += partials[(i64)k * NRED];
        b += partials[(i64)k * NRED + 1];
    }
    out[0] = a;
    out[1] = b;
}

static int dm_grid(i64 n) {
    i64 g = ((i64(1) << n) + BLOCK - 1) / BLOCK;
    return (int)(g < sm_count() * 4 ? g : sm_count() * 4);
}

}  // namespace emusv

using namespace emusv;

extern "C" {

int emusv_lindblad_apply(int nqubits, int dtype, const double *omegas, const double *deltas,
                         const double *phis, const double *interaction, int nops, const double *ops,
                         const void *rho, void *out, void *stream) {
    HamParams P;
    LindbladJumps J;
    double noise[8];
    if (!rho || !out || rho == out || nops < 0 || (nops > 0 && !ops)) return EMUSV_BAD_ARGUMENT;
    noise_term(nops, ops, noise);
    if (!make_lindblad_params(nqubits, omegas, deltas, phis, interaction, nops ? noise : nullptr, false, &P) ||
        !make_jumps(nqubits, nops, ops, &J))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    HpsiArgs A = {};
    A.u = rho;
    A.su = 1.0;
    A.out = out;
    A.part_buf = out;
    A.err = device_error_word();
    A.tile_bits = hpsi_tile_bits(P.n);
    int st = launch_hpsi(dtype, HP_STORE, P, A, 0, s, nullptr);
    if (st) return st;
    return launch_lindblad_jumps(dtype, J, rho, nullptr, out, nullptr, s);
}

size_t emusv_lindblad_workspace_bytes(int nqubits, int dtype, int basis_capacity) {
    if (nqubits < 1 || nqubits > DM_MAXQ) return 0;
    return emusv_arnoldi_workspace_bytes(2 * nqubits, dtype, basis_capacity);
}

int emusv_lindblad_arnoldi_step(int nqubits, int dtype, double dt, const double *omegas,
                                const double *deltas, const double *phis, const double *interaction,
                                int nops, const double *ops, const void *rho_in, void *rho_out,
                                double exp_tolerance, double norm_tolerance, int max_krylov_dim,
                                int krylov_dim_hint, void *workspace, size_t workspace_bytes,
                                emusv_krylov_info *info, void *stream) {
    HamParams P;
    LindbladJumps J;
    double noise[8];
    if (nops < 0 || (nops > 0 && !ops)) return EMUSV_BAD_ARGUMENT;
    noise_term(nops, ops, noise);
    if (!make_lindblad_params(nqubits, omegas, deltas, phis, interaction, nops ? noise : nullptr, false, &P) ||
        !make_jumps(nqubits, nops, ops, &J))
        return EMUSV_BAD_ARGUMENT;
    return arnoldi_run(P, J.mask ? &J : nullptr, dtype, dt, rho_in, rho_out, exp_tolerance,
                       norm_tolerance, max_krylov_dim, krylov_dim_hint, workspace, workspace_bytes,
                       info, stream);
}

size_t emusv_dm_scratch_bytes(int nqubits, int dtype) {
    if (nqubits < 1 || nqubits > DM_MAXQ) return 0;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    return 2 * (size_t(1) << (2 * nqubits)) * es + sizeof(double) * (size_t)sm_count() * 4 * NRED + 512;
}

// result_dev[0..1] = Tr(H rho), [2..3] = Tr(H^2 rho) (H without noise: the h_eff of the
// energy observables, lindblad_operator.py:138-155, 213-218; custom_callback_
// implementations.py:150-200).
int emusv_dm_energy(int nqubits, int dtype, const double *omegas, const double *deltas,
                    const double *phis, const double *interaction, const void *rho, double *result_dev,
                    void *scratch, size_t scratch_bytes, void *stream) {
    HamParams P;
    if (!rho || !result_dev || !scratch || scratch_bytes < emusv_dm_scratch_bytes(nqubits, dtype) ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64) ||
        !make_lindblad_params(nqubits, omegas, deltas, phis, interaction, nullptr, true, &P))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    const size_t vb = (size_t(1) << (2 * nqubits)) * es;
    unsigned char *p = reinterpret_cast<unsigned char *>(scratch);
    void *X = p, *Y = p + vb;
    double *partials = reinterpret_cast<double *>(p + 2 * vb);
    const int g = dm_grid(nqubits);
    for (int pass = 0; pass < 2; ++pass) {
        HpsiArgs A = {};
        A.u = pass == 0 ? rho : X;
        A.su = 1.0;
        A.out = pass == 0 ? X : Y;
        A.part_buf = A.out;
        A.err = device_error_word();
        A.tile_bits = hpsi_tile_bits(P.n);
        int st = launch_hpsi(dtype, HP_STORE, P, A, 0, s, nullptr);
        if (st) return st;
        {
            ProfScope ps_(PROF_OBS, s);
            if (dtype == EMUSV_C128) k_dm_trace<double><<<g, BLOCK, 0, s>>>(A.out, nqubits, partials);
            else k_dm_trace<float><<<g, BLOCK, 0, s>>>(A.out, nqubits, partials);
            k_dm_finish<<<1, 32, 0, s>>>(partials, g, result_dev + 2 * pass);
        }
        EMUSV_CHECK_LAUNCH();
    }
    return EMUSV_OK;
}

int emusv_dm_diagonal_amplitudes(int nqubits, int dtype, const void *rho, void *amps, void *stream) {
    if (nqubits < 1 || nqubits > DM_MAXQ || !rho || !amps || (dtype != EMUSV_C128 && dtype != EMUSV_C64))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    {
        ProfScope ps_(PROF_OBS, s);
        if (dtype == EMUSV_C128) k_dm_diag_amp<double><<<dm_grid(nqubits), BLOCK, 0, s>>>(rho, nqubits, amps);
        else k_dm_diag_amp<float><<<dm_grid(nqubits), BLOCK, 0, s>>>(rho, nqubits, amps);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

}  // extern "C"
