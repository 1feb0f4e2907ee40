// Arnoldi exponential step for the non-Hermitian Hamiltonian with the noise term (C ABI
// emusv_arnoldi_step): exp(-i dt H) psi with H = H_Rydberg - 0.5i sum_j L_j^dag L_j, the
// Krylov path of the Monte Carlo stepper (emu_sv/time_evolution/implementations.py:148-166,
// krylov_exp.py:23-106 with is_hermitian=False).
//
// Per iteration j (basis vectors stored unnormalised with FP64 scales, as in krylov.cu):
//   1. w = (H - sigma) v_j by the streaming H*psi kernels (noise diagonal fused into pass
//      L; sigma = the previous step's energy, as in the Lanczos step: same basis, T minus
//      sigma on its diagonal, added back in every exponential);
//   2. k_arn_ortho<DOTS>:    h_k = <v_k, w> for all k <= j and ||w|| in one pass;
//   3. k_arn_ortho<UPDATE_DOTS>: w' = w - sum h_k v_k (and, for a second round, the dots
//      g_k = <v_k, w'>) in one pass;
//   4. k_arn_ortho<UPDATE>:  w'' = w' - sum g_k v_k and ||w''|| (second round only).
//   Classical Gram-Schmidt, repeated when the first round removed more than half of
//   ||w||^2 (the DGKS test): the same Hessenberg column T[k][j] = h_k (+ g_k) and vector as
//   the reference's modified Gram-Schmidt (krylov_exp.py:54-58) in exact arithmetic, in two
//   or three streaming passes instead of 2(j+1) dependent dot/axpy pairs.  The shift keeps
//   ||(H - sigma) v_j|| near the spread of the spectrum, so the second round is rare.
//   5. k_arn_decide (one CTA, FP64): ||w''||, the happy-breakdown test (krylov_exp.py:
//   63-71) at every iteration, and from the host's hint on the exponential of the extended
//   Hessenberg matrix and the Expokit error estimate (krylov_exp.py:76-86); when the first
//   tested iteration already converges, the untested earlier ones are tested in order.
// The small exponentials: exp(A) e_0 of the dense extended Hessenberg matrix by s
// substeps of a 34-term Taylor series with ||A/s||_1 <= 4 (truncation below 1e-19 per
// substep), matrix-vector products split over 2-8 threads per row.
#include <string.h>

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

constexpr int ARN_KMAX = 100;                  // largest Arnoldi max_krylov_dim
constexpr int ARN_M = ARN_KMAX + 2;            // largest extended matrix
constexpr int ARN_PS = 2 * (ARN_KMAX + 1) + 2;  // partial-row stride: dots re/im, norm
constexpr int ARN_NORM = 2 * (ARN_KMAX + 1);   // norm slot of a partial row
constexpr int ORTHO_THREADS = 256;
constexpr int DECIDE_THREADS = 256;

struct ArnState {
    double2 T[ARN_M * ARN_M];  // Hessenberg matrix of H - sigma (row-major [r][c]), basis v_k
    double2 coef[ARN_M];       // coefficients of the next Gram-Schmidt update
    int reorth;                // this iteration takes the second Gram-Schmidt round
    int rounds2;               // second rounds taken in this run
};

// Pass A: dots.  Pass B: update with h; with reorth also the dots of the result.  Pass C:
// update with the second round's coefficients (returns at once without reorth).
enum ArnMode { ARN_DOTS = 0, ARN_UPDATE_DOTS = 1, ARN_UPDATE = 2 };

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// One streaming pass over w and v_0..v_j (see the header).  Partials per block:
// [2k], [2k+1] = <v_k, w_out> (DOTS, UPDATE_DOTS), [ARN_NORM] = ||w_out||^2.
// E amplitudes per thread per chunk.  UPDATE_DOTS reads every v_k twice per chunk (the
// update needs all of them before the dots of the result).
template <typename R, int MODE, int E, int KB = 4>
__global__ void __launch_bounds__(ORTHO_THREADS)
k_arn_ortho(const KState *ks, const ArnState *as, int j, const void *v0_, const unsigned char *basis,
            i64 D, void *w_, double *part) {
    typedef typename cvec<R>::T C;
    if (ks->status != KS_RUNNING) return;
    const bool reorth = as->reorth != 0;
    if (MODE == ARN_UPDATE && !reorth) return;
    const bool dots = MODE == ARN_DOTS || (MODE == ARN_UPDATE_DOTS && reorth);
    constexpr int NW = ORTHO_THREADS / 32;
    __shared__ double2 cf[ARN_M];
    __shared__ double sc[ARN_M];
    __shared__ double2 sacc[NW][ARN_KMAX + 1];
    __shared__ double snorm[NW];
    const int nk = j + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < nk; k += ORTHO_THREADS) {
        sc[k] = ks->scale[k];
        const double2 c = as->coef[k];
        cf[k] = make_double2(c.x * ks->scale[k], c.y * ks->scale[k]);
    }
    for (int k = tid; k < NW * (ARN_KMAX + 1); k += ORTHO_THREADS)
        (&sacc[0][0])[k] = make_double2(0.0, 0.0);
    __syncthreads();
    const C *v0 = reinterpret_cast<const C *>(v0_);
    const C *bs = reinterpret_cast<const C *>(basis);
    C *w = reinterpret_cast<C *>(w_);
    auto vk = [&](int k) -> const C * { return k == 0 ? v0 : bs + (i64)k * D; };
    double nacc = 0.0;
    const i64 CH = (i64)ORTHO_THREADS * E;
    for (i64 c0 = (i64)blockIdx.x * CH; c0 < D; c0 += (i64)gridDim.x * CH) {
        double wr[E], wi[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
            wr[e] = wi[e] = 0.0;
            if (x < D) {
                const C a = w[x];
                wr[e] = double(a.x);
                wi[e] = double(a.y);
            }
        }
        if (MODE != ARN_DOTS) {
            // KB vectors per step: KB * E independent loads in flight per thread
            int k = 0;
            for (; k + KB <= nk; k += KB) {
                C a[KB][E];
#pragma unroll
                for (int kb = 0; kb < KB; ++kb)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                        a[kb][e] = x < D ? vk(k + kb)[x] : cmake<C>(0.0, 0.0);
                    }
#pragma unroll
                for (int kb = 0; kb < KB; ++kb) {
                    const double2 c = cf[k + kb];
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        wr[e] -= c.x * double(a[kb][e].x) - c.y * double(a[kb][e].y);
                        wi[e] -= c.x * double(a[kb][e].y) + c.y * double(a[kb][e].x);
                    }
                }
            }
            for (; k < nk; ++k) {
                const C *v = vk(k);
                const double2 c = cf[k];
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                    if (x < D) {
                        const C a = v[x];
                        wr[e] -= c.x * double(a.x) - c.y * double(a.y);
                        wi[e] -= c.x * double(a.y) + c.y * double(a.x);
                    }
                }
            }
#pragma unroll
            for (int e = 0; e < E; ++e) {  // store, and continue with the stored (rounded) values
                const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                if (x < D) {
                    const C o = cmake<C>(wr[e], wi[e]);
                    w[x] = o;
                    wr[e] = double(o.x);
                    wi[e] = double(o.y);
                }
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) nacc += wr[e] * wr[e] + wi[e] * wi[e];
        if (dots) {
            int k = 0;
            for (; k + KB <= nk; k += KB) {
                C a[KB][E];
#pragma unroll
                for (int kb = 0; kb < KB; ++kb)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                        a[kb][e] = x < D ? vk(k + kb)[x] : cmake<C>(0.0, 0.0);
                    }
                double dr[KB], di[KB];
#pragma unroll
                for (int kb = 0; kb < KB; ++kb) {
                    dr[kb] = di[kb] = 0.0;
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        dr[kb] += double(a[kb][e].x) * wr[e] + double(a[kb][e].y) * wi[e];
                        di[kb] += double(a[kb][e].x) * wi[e] - double(a[kb][e].y) * wr[e];
                    }
                }
#pragma unroll
                for (int kb = 0; kb < KB; ++kb) {
                    dr[kb] = warp_sum(dr[kb]);
                    di[kb] = warp_sum(di[kb]);
                }
                if (lane == 0) {
#pragma unroll
                    for (int kb = 0; kb < KB; ++kb) {
                        sacc[warp][k + kb].x += dr[kb];
                        sacc[warp][k + kb].y += di[kb];
                    }
                }
            }
            for (; k < nk; ++k) {
                const C *v = vk(k);
                double dr = 0.0, di = 0.0;  // sum conj(v) w
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                    if (x < D) {
                        const C a = v[x];
                        dr += double(a.x) * wr[e] + double(a.y) * wi[e];
                        di += double(a.x) * wi[e] - double(a.y) * wr[e];
                    }
                }
                dr = warp_sum(dr);
                di = warp_sum(di);
                if (lane == 0) {
                    sacc[warp][k].x += dr;
                    sacc[warp][k].y += di;
                }
            }
        }
    }
    nacc = warp_sum(nacc);
    if (lane == 0) snorm[warp] = nacc;
    __syncthreads();
    double *row = part + (i64)blockIdx.x * ARN_PS;
    if (dots) {
        for (int k = tid; k < nk; k += ORTHO_THREADS) {
            double2 t = make_double2(0.0, 0.0);
            for (int q = 0; q < NW; ++q) {
                t.x += sacc[q][k].x;
                t.y += sacc[q][k].y;
            }
            row[2 * k] = sc[k] * t.x;
            row[2 * k + 1] = sc[k] * t.y;
        }
    }
    if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < NW; ++q) t += snorm[q];
        row[ARN_NORM] = t;
    }
}

// Sum of value i of the ortho partial rows over nb blocks by one warp (lanes stride over
// the blocks, then a fixed shuffle tree: deterministic).  Result in every lane.
__device__ __forceinline__ double arn_sum_warp(const double *part, int nb, int i) {
    double t = 0.0;
    for (int b = threadIdx.x & 31; b < nb; b += 32) t += part[(i64)b * ARN_PS + i];
    return warp_sum(t);
}

// After the DOTS (stage 0) or UPDATE_DOTS (stage 1) pass: column j of T and the next
// update's coefficients; stage 0 also records ||H v_j|| (krylov_exp.py:52).
__global__ void __launch_bounds__(DECIDE_THREADS)
k_arn_stage(KState *ks, ArnState *as, int j, const double *part, int nb, int stage) {
    if (ks->status != KS_RUNNING) return;
    if (stage == 1 && !as->reorth) return;
    __shared__ int bad;
    __shared__ double hsq[DECIDE_THREADS / 32];
    if (threadIdx.x == 0) bad = 0;
    if (threadIdx.x < DECIDE_THREADS / 32) hsq[threadIdx.x] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NWD = DECIDE_THREADS / 32;
    for (int k = warp; k <= j; k += NWD) {  // one warp per column entry
        const double2 h = make_double2(arn_sum_warp(part, nb, 2 * k), arn_sum_warp(part, nb, 2 * k + 1));
        if (lane == 0) {
            if (!isfinite(h.x) || !isfinite(h.y)) bad = 1;
            double2 &t = as->T[k * ARN_M + j];
            t = stage == 0 ? h : make_double2(t.x + h.x, t.y + h.y);
            as->coef[k] = h;
            hsq[warp] += h.x * h.x + h.y * h.y;
            if (stage == 0 && k == j) ks->a_re[j] = h.x;  // Re <v_j, (H - sigma) v_j>
        }
    }
    __syncthreads();
    if (stage == 0 && warp == 0) {
        const double n2 = arn_sum_warp(part, nb, ARN_NORM);  // ||(H - sigma) v_j||^2
        if (lane == 0) {
            double hs = 0.0;
            for (int q = 0; q < DECIDE_THREADS / 32; ++q) hs += hsq[q];
            // ||H v_j|| (krylov_exp.py:52) from the shifted product
            const double sg = ks->shift;
            ks->hn[j] = sqrt(fmax(0.0, n2 + 2.0 * sg * ks->a_re[j] + sg * sg));
            // second round unless the projection kept more than half of ||w||^2 (Daniel,
            // Gragg, Kaufman and Stewart's test with eta = 1/sqrt(2)); ||w'||^2 is taken as
            // ||w||^2 - sum |h_k|^2, the exact value for an orthonormal basis
            as->reorth = !(n2 - hs > 0.5 * n2);
            as->rounds2 = (j == 0 ? 0 : as->rounds2) + as->reorth;
            if (!isfinite(n2)) bad = 1;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && bad) {
        ks->status = KS_NONFINITE;
        ks->iters = j + 1;
    }
}

// y = exp(A) e_0 for the M x M matrix A in shared memory (column-major A[c*M + r]).
// s substeps of sum_{k<=34} (A/s)^k / k! with ||A/s||_1 <= 4: truncation below
// 4^35/35! ~ 1e-19 relative per substep, terms at most 4^4/4! ~ 11 times the result (about
// one digit of cancellation).  Returns false when the norm is not finite or would need
// more than 2^20 substeps.  All threads of the block.
__device__ bool arn_expm_col0(const double2 *A, int M, double2 *y, double2 *t, double2 *tn,
                              double *red) {
    const int tid = threadIdx.x;
    // ||A||_1: column sums
    double cs = 0.0;
    if (tid < M)
        for (int r = 0; r < M; ++r) cs += hypot(A[tid * M + r].x, A[tid * M + r].y);
    red[tid] = cs;
    __syncthreads();
    for (int o = DECIDE_THREADS / 2; o > 0; o >>= 1) {
        if (tid < o) red[tid] = fmax(red[tid], red[tid + o]);
        __syncthreads();
    }
    const double nrm = red[0];
    __syncthreads();
    if (!isfinite(nrm) || nrm > 4.0 * 1048576.0) return false;
    const int s = nrm > 4.0 ? (int)ceil(nrm / 4.0) : 1;
    const int TPR = M <= 32 ? 8 : (M <= 64 ? 4 : 2);
    const int r = tid / TPR, q = tid % TPR;
    if (tid < M) y[tid] = make_double2(tid == 0 ? 1.0 : 0.0, 0.0);
    __syncthreads();
    for (int step = 0; step < s; ++step) {
        if (tid < M) t[tid] = y[tid];
        __syncthreads();
        for (int k = 1; k <= 34; ++k) {
            double2 acc = make_double2(0.0, 0.0);
            if (r < M) {
                for (int c = q; c < M; c += TPR) {
                    const double2 a = A[c * M + r], v = t[c];
                    acc.x += a.x * v.x - a.y * v.y;
                    acc.y += a.x * v.y + a.y * v.x;
                }
            }
            for (int o = TPR >> 1; o > 0; o >>= 1) {  // TPR lanes of one warp
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
            }
            const double f = 1.0 / ((double)s * (double)k);
            if (q == 0 && r < M) tn[r] = make_double2(acc.x * f, acc.y * f);
            __syncthreads();
            if (tid < M) {
                t[tid] = tn[tid];
                y[tid].x += tn[tid].x;
                y[tid].y += tn[tid].y;
            }
            __syncthreads();
        }
    }
    return true;
}

// Extended matrix of iteration jj (krylov_exp.py:77-78) in my basis: A = -i dt T[:jj+2,
// :jj+1] plus A[jj+2][jj+1] = 1 (M = jj + 3); happy: A = -i dt T[:jj+1, :jj+1] (M = jj + 1).
__device__ void arn_build(const ArnState *as, int jj, double dt, double sigma, bool happy, double2 *A,
                          int *Mo) {
    const int M = happy ? jj + 1 : jj + 3;
    for (int i = threadIdx.x; i < M * M; i += DECIDE_THREADS) {
        const int c = i / M, r = i % M;
        double2 v = make_double2(0.0, 0.0);
        if (c <= jj && r <= c + 1 && r <= (happy ? jj : jj + 1)) {  // Hessenberg entries
            double2 h = as->T[r * ARN_M + c];
            if (r == c) h.x += sigma;  // T of H itself
            v = make_double2(dt * h.y, -dt * h.x);  // -i dt h
        }
        if (!happy && c == jj + 1 && r == jj + 2) v = make_double2(1.0, 0.0);
        A[i] = v;
    }
    *Mo = M;
    __syncthreads();
}

// Error estimate of iteration jj (krylov_exp.py:81-84); writes c[0..jj+1].  The estimate
// is NaN when both terms are zero (0 * 0 / 0, as in the reference, where NaN fails the
// convergence test); *fail is set when the exponential itself failed.
__device__ double arn_eval(KState *ks, const ArnState *as, int jj, double dt, double2 *A, double2 *y,
                           double2 *t, double2 *tn, double *red, bool *fail) {
    int M;
    arn_build(as, jj, dt, ks->shift, false, A, &M);
    if (!arn_expm_col0(A, M, y, t, tn, red)) {
        *fail = true;
        return nan("");
    }
    for (int k = threadIdx.x; k <= jj + 1; k += DECIDE_THREADS) {
        ks->c_re[k] = y[k].x;
        ks->c_im[k] = y[k].y;
    }
    const double err1 = hypot(y[jj + 1].x, y[jj + 1].y);
    const double err2 = hypot(y[jj + 2].x, y[jj + 2].y) * (fabs(dt) * ks->hn[jj]);
    __syncthreads();
    return err1 < err2 ? err1 : (err1 * err2 / (err1 - err2));
}

__global__ void __launch_bounds__(DECIDE_THREADS)
k_arn_decide(KState *ks, ArnState *as, int j, const double *part, int nb, double dt, double exp_tol,
             double norm_tol, int poll, int first_poll, int maxdim) {
    if (ks->status != KS_RUNNING) return;
    extern __shared__ __align__(16) unsigned char arn_smem[];
    const int Mmax = maxdim + 2;
    double2 *A = reinterpret_cast<double2 *>(arn_smem);
    double2 *y = A + Mmax * Mmax;
    double2 *t = y + Mmax;
    double2 *tn = t + Mmax;
    double *red = reinterpret_cast<double *>(tn + Mmax);  // [DECIDE_THREADS]
    const int tid = threadIdx.x;
    if (ks->kerr) {  // a streaming kernel gave up on a bounded wait
        if (tid == 0) {
            ks->status = KS_TIMEOUT;
            ks->iters = j + 1;
        }
        return;
    }
    __shared__ double n2s;
    if (tid < 32) {
        const double v = arn_sum_warp(part, nb, ARN_NORM);
        if (tid == 0) n2s = v;
    }
    __syncthreads();
    const double r = sqrt(n2s);
    if (!isfinite(r)) {
        if (tid == 0) {
            ks->status = KS_NONFINITE;
            ks->iters = j + 1;
        }
        return;
    }
    if (tid == 0) {
        as->T[(j + 1) * ARN_M + j] = make_double2(r, 0.0);  // krylov_exp.py:61
        ks->r[j] = r;
        ks->scale[j + 1] = 1.0 / r;
    }
    __syncthreads();
    if (fabs(dt) * r < norm_tol) {  // happy breakdown (krylov_exp.py:63-71)
        int M;
        arn_build(as, j, dt, ks->shift, true, A, &M);
        const bool ok = arn_expm_col0(A, M, y, t, tn, red);
        for (int k = tid; k < M; k += DECIDE_THREADS) {
            ks->c_re[k] = y[k].x;
            ks->c_im[k] = y[k].y;
        }
        if (tid == 0) {
            ks->nvec = j + 1;
            ks->iters = j + 1;
            ks->status = ok ? KS_HAPPY : KS_NONFINITE;
        }
        return;
    }
    if (!poll) return;
    bool fail = false;
    double err = arn_eval(ks, as, j, dt, A, y, t, tn, red, &fail);
    int jc = j;
    // the first test also looks at the untested iterations, in order, when this one
    // converges or its estimate is NaN (both error terms underflowed: an earlier
    // iteration may have converged already)
    if ((err < exp_tol || err != err) && first_poll && j > 0 && !fail) {
        for (int jj = 0; jj < j; ++jj) {
            const double e = arn_eval(ks, as, jj, dt, A, y, t, tn, red, &fail);
            if (e < exp_tol) {
                err = e;
                jc = jj;
                break;
            }
        }
        if (jc == j) err = arn_eval(ks, as, j, dt, A, y, t, tn, red, &fail);
    }
    if (tid == 0) {
        ks->err = err;
        ks->nvec = jc + 2;
        ks->iters = jc + 1;
        if (fail)
            ks->status = KS_NONFINITE;
        else if (err < exp_tol)
            ks->status = KS_CONVERGED;
        else if (j + 1 >= maxdim)
            ks->status = KS_MAXDIM;
    }
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static size_t arn_header_bytes() {
    return align_up(sizeof(KState), 256) + align_up(sizeof(ArnState), 256) +
           align_up(sizeof(double) * (size_t)sm_count() * 8 * ARN_PS, 256) +
           align_up(sizeof(double) * (size_t)sm_count() * 8 * NRED, 256);
}

static size_t decide_smem(int maxdim) {
    const size_t M = (size_t)maxdim + 2;
    return sizeof(double2) * (M * M + 3 * M) + sizeof(double) * DECIDE_THREADS;
}

// Grid of the ortho passes: the streaming grid of the vector kernels (up to four blocks per
// SM), never more blocks than chunks; *grid_out receives it (the number of partial rows).
// Measured on B200 (N=22, complex128, j ~ 35): one block per SM with chunks small enough
// for the update-and-dots pass to find its second reads in L2 was 1.5x slower than the
// wide grid that re-reads them from HBM.
template <typename R>
static int launch_ortho(int mode, const KState *ks, const ArnState *as, int j, const void *v0,
                        const unsigned char *basis, i64 D, void *w, double *part, cudaStream_t s,
                        int *grid_out) {
    constexpr int E = 4;
    i64 grid = krylov_stream_grid(D);
    const i64 chunks = (D + (i64)ORTHO_THREADS * E - 1) / ((i64)ORTHO_THREADS * E);
    if (grid > chunks) grid = chunks;
    *grid_out = (int)grid;
    ProfScope ps_(PROF_ORTH, s);
#define ARN_LAUNCH(M) k_arn_ortho<R, M, E><<<(int)grid, ORTHO_THREADS, 0, s>>>(ks, as, j, v0, basis, D, w, part)
    if (mode == ARN_DOTS)
        ARN_LAUNCH(ARN_DOTS);
    else if (mode == ARN_UPDATE)
        ARN_LAUNCH(ARN_UPDATE);
    else
        ARN_LAUNCH(ARN_UPDATE_DOTS);
#undef ARN_LAUNCH
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

}  // namespace emusv

using namespace emusv;

extern "C" {

size_t emusv_arnoldi_workspace_bytes(int nqubits, int dtype, int basis_capacity) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS || basis_capacity < 0 ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64))
        return 0;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    return arn_header_bytes() + (size_t)(basis_capacity + 1) * (size_t(1) << nqubits) * es;
}

int emusv_arnoldi_step(int nqubits, int dtype, double dt, const double *omegas, const double *deltas,
                       const double *phis, const double *interaction, const double *noise,
                       const void *psi_in, void *psi_out, double exp_tolerance, double norm_tolerance,
                       int max_krylov_dim, int krylov_dim_hint, void *workspace,
                       size_t workspace_bytes, emusv_krylov_info *info, void *stream) {
    HamParams P;
    if (!make_params(nqubits, omegas, deltas, phis, interaction, &P) || !add_noise(noise, &P))
        return EMUSV_BAD_ARGUMENT;
    return arnoldi_run(P, nullptr, dtype, dt, psi_in, psi_out, exp_tolerance, norm_tolerance,
                       max_krylov_dim, krylov_dim_hint, workspace, workspace_bytes, info, stream);
}

}  // extern "C"

namespace emusv {

// The Arnoldi step for the operator of P (nqubits = P.n bits), plus, when J is given, the
// Lindblad jump term i sum_q K_q added to every product (lindblad.cu).
int arnoldi_run(const HamParams &P, const LindbladJumps *J, int dtype, double dt, const void *psi_in,
                void *psi_out, double exp_tolerance, double norm_tolerance, int max_krylov_dim,
                int krylov_dim_hint, void *workspace, size_t workspace_bytes,
                emusv_krylov_info *info, void *stream) {
    const int nqubits = P.n;
    if (!psi_in || !psi_out || !workspace || (dtype != EMUSV_C128 && dtype != EMUSV_C64) ||
        max_krylov_dim < 1 || max_krylov_dim > ARN_KMAX || !isfinite(dt))
        return EMUSV_BAD_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) || (reinterpret_cast<uintptr_t>(psi_in) & 15) ||
        (reinterpret_cast<uintptr_t>(psi_out) & 15))
        return EMUSV_BAD_ARGUMENT;
    if (workspace_bytes < arn_header_bytes()) return EMUSV_WORKSPACE_TOO_SMALL;
    cudaStream_t s = as_stream(stream);
    const i64 D = i64(1) << nqubits;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    unsigned char *p = reinterpret_cast<unsigned char *>(workspace);
    KState *ks = reinterpret_cast<KState *>(p);
    p += align_up(sizeof(KState), 256);
    ArnState *as = reinterpret_cast<ArnState *>(p);
    p += align_up(sizeof(ArnState), 256);
    double *part = reinterpret_cast<double *>(p);
    p += align_up(sizeof(double) * (size_t)sm_count() * 8 * ARN_PS, 256);
    double *part_n = reinterpret_cast<double *>(p);
    p += align_up(sizeof(double) * (size_t)sm_count() * 8 * NRED, 256);
    unsigned char *basis = p;  // slot 0: partial sums of the multi-pass H*psi; slots 1..
    const int capacity = (int)((workspace_bytes - arn_header_bytes()) / (D * es)) - 1;
    if (capacity < 1) return EMUSV_WORKSPACE_TOO_SMALL;
    auto stored = [&](int k) -> const void * {
        return k == 0 ? psi_in : (const void *)(basis + (size_t)k * D * es);
    };
    const size_t dsmem = decide_smem(max_krylov_dim);
    EMUSV_CHECK(cudaFuncSetAttribute(k_arn_decide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsmem));
    int st = krylov_begin(dtype, psi_in, D, ks, part_n, true, s);
    if (st) return st;

    int status = KS_RUNNING;
    bool polled = false;
    for (int j = 0; j < max_krylov_dim; ++j) {
        if (j + 1 > capacity) {
            if ((st = read_status(ks, s, &status))) return st;
            if (status == KS_RUNNING) return EMUSV_WORKSPACE_TOO_SMALL;
            break;
        }
        void *w = const_cast<void *>(stored(j + 1));
        HpsiArgs A = {};
        A.u = stored(j);
        A.su_dev = &ks->scale[j];
        A.out = w;
        A.tile_bits = hpsi_tile_bits(nqubits);
        A.gate = &ks->status;
        A.err = &ks->kerr;
        A.part_buf = basis;
        A.eshift = &ks->shift;
        if ((st = launch_hpsi(dtype, HP_STORE, P, A, 0, s, nullptr))) return st;
        if (J && (st = launch_lindblad_jumps(dtype, *J, stored(j), &ks->scale[j], w, &ks->status, s)))
            return st;
        int og = 0;
        for (int mode = ARN_DOTS; mode <= ARN_UPDATE; ++mode) {
            st = dtype == EMUSV_C128
                     ? launch_ortho<double>(mode, ks, as, j, psi_in, basis, D, w, part, s, &og)
                     : launch_ortho<float>(mode, ks, as, j, psi_in, basis, D, w, part, s, &og);
            if (st) return st;
            if (mode != ARN_UPDATE) {
                ProfScope ps_(PROF_SMALL, s);
                k_arn_stage<<<1, DECIDE_THREADS, 0, s>>>(ks, as, j, part, og, mode);
                EMUSV_CHECK_LAUNCH();
            }
        }
        const bool poll = (j + 1 >= krylov_dim_hint) || (j + 1 >= max_krylov_dim);
        {
            ProfScope ps_(PROF_SMALL, s);
            k_arn_decide<<<1, DECIDE_THREADS, dsmem, s>>>(ks, as, j, part, og, dt, exp_tolerance,
                                                          norm_tolerance, poll ? 1 : 0,
                                                          (poll && !polled) ? 1 : 0, max_krylov_dim);
            EMUSV_CHECK_LAUNCH();
        }
        if (poll) {
            polled = true;
            if ((st = read_status(ks, s, &status))) return st;
            if (status != KS_RUNNING) break;
        }
    }
    if (status == KS_RUNNING)
        if ((st = read_status(ks, s, &status))) return st;
    if (status == KS_TIMEOUT) {
        if (info) memset(info, 0, sizeof(*info));
        return EMUSV_TIMEOUT;
    }
    if (status == KS_NONFINITE || status == KS_RUNNING) {
        if (info) memset(info, 0, sizeof(*info));
        return EMUSV_NONFINITE;
    }
    if ((st = krylov_combine(dtype, ks, psi_in, basis, D, psi_out, part_n, s))) return st;
    if (info) {
        KState h;
        int r2 = 0;
        EMUSV_CHECK(cudaMemcpyAsync(&h, ks, offsetof(KState, a_re), cudaMemcpyDeviceToHost, s));
        EMUSV_CHECK(cudaMemcpyAsync(&r2, &as->rounds2, sizeof(int), cudaMemcpyDeviceToHost, s));
        EMUSV_CHECK(cudaStreamSynchronize(s));
        info->iterations = h.iters;
        info->happy_breakdown = h.status == KS_HAPPY;
        info->converged = h.status == KS_HAPPY || h.status == KS_CONVERGED;
        info->basis_vectors = h.nvec;
        info->error_estimate = h.err;
        info->input_norm = h.s0;
        info->output_norm = sqrt(h.outnorm2);
        info->second_rounds = r2;
    }
    return status == KS_MAXDIM ? EMUSV_NOT_CONVERGED : EMUSV_OK;
}

}  // namespace emusv
