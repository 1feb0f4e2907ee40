// Arnoldi exponential step for the non-Hermitian Hamiltonian with the noise term (C ABI
// emusv_arnoldi_step): exp(-i dt H) psi with H = H_Rydberg - 0.5i sum_j L_j^dag L_j, the
// Krylov path of the Monte Carlo stepper (emu_sv/time_evolution/implementations.py:148-166,
// krylov_exp.py:23-106 with is_hermitian=False).
//
// Per iteration j (basis vectors stored unnormalised with FP64 scales, as in krylov.cu):
//   1. w = (H - sigma) v~_j by the streaming H*psi kernels (noise diagonal fused into pass
//      L; sigma = the previous step's energy, as in the Lanczos step: same basis, T minus
//      sigma on its diagonal, added back in every exponential);
//   2. two Gram-Schmidt passes with the second round of v~_j lagged into them (see
//      k_arn_lagdots below): the same Hessenberg matrix and basis as the reference's
//      modified Gram-Schmidt (krylov_exp.py:54-58) in exact arithmetic, every vector
//      orthogonalised twice, in two streaming passes instead of 2(j+1) dependent dot/axpy
//      pairs;
//   3. k_arn_decide (one CTA, FP64): ||w'||, the happy-breakdown test (krylov_exp.py:
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
constexpr int ARN_KA = ARN_KMAX + 1;           // finalised basis vectors at most
// partial row of a pass: z_k = <v_k, w> (re, im), s_k = <v_k, vt>, a = <vt, w>, ||w||^2,
// ||vt||^2 (pass A); pass B writes its norm at ARN_NORM
constexpr int ARN_S0 = 2 * ARN_KA, ARN_A0 = 4 * ARN_KA, ARN_NORM = ARN_A0 + 2;
constexpr int ARN_PS = ARN_A0 + 4;
constexpr int ORTHO_THREADS = 256;
constexpr int DECIDE_THREADS = 256;

struct ArnState {
    double2 T[ARN_M * ARN_M];  // Hessenberg matrix of H - sigma (row-major [r][c]), basis v_k
    double2 cw1[ARN_M];        // pass B: w' = cw w - ct vt - sum cw1_l v_l
    double2 cvj[ARN_M];        //         v_j = cv vt - sum cvj_l v_l
    double2 ct;
    double cw, cv;
};

// The orthogonalisation is classical Gram-Schmidt with its second round lagged by one
// iteration (the low-synchronisation "DCGS2" form): iteration j receives w = (H - sigma) vt
// for the not yet reorthogonalised vt = v~_j, and
//   pass A (k_arn_lagdots): one pass over w, vt and the final v_0..v_{j-1}: z = V^H w,
//     s = V^H vt, <vt, w>, ||w||^2, ||vt||^2;
//   k_arn_lagstage: v_j = (vt - V s) / alpha (alpha^2 = ||vt||^2 - |s|^2) corrects the
//     previous Hessenberg column (T[:, j-1] += beta s, T[j][j-1] = beta alpha), H v_j =
//     (w - V_j T s) / alpha by the Arnoldi relation, h = V_j^H H v_j from z, s and T;
//   pass B (k_arn_lagupdate): w' = H v_j - V_j h and the corrected v_j in one pass (both
//     combinations of w, vt and V), ||w'||^2.
// Two streaming passes per iteration; every basis vector but the newest is orthogonalised
// twice, as in classical Gram-Schmidt with reorthogonalisation.
template <typename R, int E = 4, int KB = 4>
__global__ void __launch_bounds__(ORTHO_THREADS)
k_arn_lagdots(const KState *ks, int j, const void *v0_, const unsigned char *basis, i64 D,
              const void *w_, double *part) {
    typedef typename cvec<R>::T C;
    if (ks->status != KS_RUNNING) return;
    constexpr int NW = ORTHO_THREADS / 32;
    __shared__ double sc[ARN_M];
    __shared__ double2 accz[NW][ARN_KA], accs[NW][ARN_KA];
    __shared__ double sa[NW][4];
    const bool has_vt = j >= 1;
    const int nk = has_vt ? j : 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < nk; k += ORTHO_THREADS) sc[k] = ks->scale[k];
    for (int k = tid; k < NW * ARN_KA; k += ORTHO_THREADS) {
        (&accz[0][0])[k] = make_double2(0.0, 0.0);
        (&accs[0][0])[k] = make_double2(0.0, 0.0);
    }
    const double st = has_vt ? ks->scale[j] : 0.0;
    __syncthreads();
    const C *v0 = reinterpret_cast<const C *>(v0_);
    const C *bs = reinterpret_cast<const C *>(basis);
    const C *w = reinterpret_cast<const C *>(w_);
    const C *vt = has_vt ? bs + (i64)j * D : nullptr;
    auto vk = [&](int k) -> const C * { return k == 0 ? v0 : bs + (i64)k * D; };
    double nw = 0.0, nv = 0.0, ar = 0.0, ai = 0.0;
    const i64 CH = (i64)ORTHO_THREADS * E;
    for (i64 c0 = (i64)blockIdx.x * CH; c0 < D; c0 += (i64)gridDim.x * CH) {
        double wr[E], wi[E], tr[E], ti[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
            wr[e] = wi[e] = tr[e] = ti[e] = 0.0;
            if (x < D) {
                const C a = w[x];
                wr[e] = double(a.x);
                wi[e] = double(a.y);
                if (has_vt) {
                    const C b = vt[x];
                    tr[e] = st * double(b.x);
                    ti[e] = st * double(b.y);
                }
            }
            nw += wr[e] * wr[e] + wi[e] * wi[e];
            nv += tr[e] * tr[e] + ti[e] * ti[e];
            ar += tr[e] * wr[e] + ti[e] * wi[e];
            ai += tr[e] * wi[e] - ti[e] * wr[e];
        }
        int k = 0;
        for (; k < nk; k += KB) {
            C a[KB][E];
#pragma unroll
            for (int kb = 0; kb < KB; ++kb)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                    a[kb][e] = (k + kb < nk && x < D) ? vk(k + kb)[x] : cmake<C>(0.0, 0.0);
                }
            double zr[KB], zi[KB], sr[KB], si[KB];
#pragma unroll
            for (int kb = 0; kb < KB; ++kb) {
                zr[kb] = zi[kb] = sr[kb] = si[kb] = 0.0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const double px = double(a[kb][e].x), py = double(a[kb][e].y);
                    zr[kb] += px * wr[e] + py * wi[e];
                    zi[kb] += px * wi[e] - py * wr[e];
                    sr[kb] += px * tr[e] + py * ti[e];
                    si[kb] += px * ti[e] - py * tr[e];
                }
            }
#pragma unroll
            for (int kb = 0; kb < KB; ++kb) {
                zr[kb] = warp_sum(zr[kb]);
                zi[kb] = warp_sum(zi[kb]);
                if (has_vt) {
                    sr[kb] = warp_sum(sr[kb]);
                    si[kb] = warp_sum(si[kb]);
                }
            }
            if (lane == 0) {
#pragma unroll
                for (int kb = 0; kb < KB; ++kb) {
                    if (k + kb >= nk) break;
                    accz[warp][k + kb].x += zr[kb];
                    accz[warp][k + kb].y += zi[kb];
                    accs[warp][k + kb].x += sr[kb];
                    accs[warp][k + kb].y += si[kb];
                }
            }
        }
    }
    nw = warp_sum(nw);
    nv = warp_sum(nv);
    ar = warp_sum(ar);
    ai = warp_sum(ai);
    if (lane == 0) {
        sa[warp][0] = ar;
        sa[warp][1] = ai;
        sa[warp][2] = nw;
        sa[warp][3] = nv;
    }
    __syncthreads();
    double *row = part + (i64)blockIdx.x * ARN_PS;
    for (int k = tid; k < nk; k += ORTHO_THREADS) {
        double2 z = make_double2(0.0, 0.0), q = make_double2(0.0, 0.0);
        for (int u = 0; u < NW; ++u) {
            z.x += accz[u][k].x;
            z.y += accz[u][k].y;
            q.x += accs[u][k].x;
            q.y += accs[u][k].y;
        }
        row[2 * k] = sc[k] * z.x;
        row[2 * k + 1] = sc[k] * z.y;
        row[ARN_S0 + 2 * k] = sc[k] * q.x;
        row[ARN_S0 + 2 * k + 1] = sc[k] * q.y;
    }
    if (tid < 4) {
        double t = 0.0;
        for (int u = 0; u < NW; ++u) t += sa[u][tid];
        row[ARN_A0 + tid] = t;
    }
}

// Pass B: w' = cw w - ct vt - sum cw1_l v_l (in place over w) and, for j >= 1, the
// corrected v_j = cv vt - sum cvj_l v_l (in place over vt, stored with scale 1); ||w'||^2.
template <typename R, int E = 4, int KB = 4>
__global__ void __launch_bounds__(ORTHO_THREADS)
k_arn_lagupdate(const KState *ks, const ArnState *as, int j, const void *v0_, unsigned char *basis,
                i64 D, void *w_, double *part) {
    typedef typename cvec<R>::T C;
    if (ks->status != KS_RUNNING) return;
    constexpr int NW = ORTHO_THREADS / 32;
    __shared__ double2 c1[ARN_M], c2[ARN_M];
    __shared__ double snorm[NW];
    const bool has_vt = j >= 1;
    const int nk = has_vt ? j : 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < nk; k += ORTHO_THREADS) {
        const double sk = ks->scale[k];
        c1[k] = make_double2(as->cw1[k].x * sk, as->cw1[k].y * sk);
        c2[k] = make_double2(as->cvj[k].x * sk, as->cvj[k].y * sk);
    }
    const double st = has_vt ? ks->scale[j] : 0.0;
    const double cw = as->cw, cv = as->cv * st;
    const double2 ct = make_double2(as->ct.x * st, as->ct.y * st);
    __syncthreads();
    const C *v0 = reinterpret_cast<const C *>(v0_);
    C *bs = reinterpret_cast<C *>(basis);
    C *w = reinterpret_cast<C *>(w_);
    C *vt = has_vt ? bs + (i64)j * D : nullptr;
    auto vk = [&](int k) -> const C * { return k == 0 ? v0 : bs + (i64)k * D; };
    double nacc = 0.0;
    const i64 CH = (i64)ORTHO_THREADS * E;
    for (i64 c0 = (i64)blockIdx.x * CH; c0 < D; c0 += (i64)gridDim.x * CH) {
        double ur[E], ui[E], qr[E], qi[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
            ur[e] = ui[e] = qr[e] = qi[e] = 0.0;
            if (x < D) {
                const C a = w[x];
                ur[e] = cw * double(a.x);
                ui[e] = cw * double(a.y);
                if (has_vt) {
                    const C b = vt[x];
                    const double bx = double(b.x), by = double(b.y);
                    ur[e] -= ct.x * bx - ct.y * by;
                    ui[e] -= ct.x * by + ct.y * bx;
                    qr[e] = cv * bx;
                    qi[e] = cv * by;
                }
            }
        }
        int k = 0;
        for (; k < nk; k += KB) {
            C a[KB][E];
#pragma unroll
            for (int kb = 0; kb < KB; ++kb)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
                    a[kb][e] = (k + kb < nk && x < D) ? vk(k + kb)[x] : cmake<C>(0.0, 0.0);
                }
#pragma unroll
            for (int kb = 0; kb < KB; ++kb) {
                if (k + kb >= nk) break;
                const double2 p1 = c1[k + kb], p2 = c2[k + kb];
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const double px = double(a[kb][e].x), py = double(a[kb][e].y);
                    ur[e] -= p1.x * px - p1.y * py;
                    ui[e] -= p1.x * py + p1.y * px;
                    qr[e] -= p2.x * px - p2.y * py;
                    qi[e] -= p2.x * py + p2.y * px;
                }
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const i64 x = c0 + tid + (i64)e * ORTHO_THREADS;
            if (x < D) {
                const C o = cmake<C>(ur[e], ui[e]);
                w[x] = o;
                nacc += double(o.x) * double(o.x) + double(o.y) * double(o.y);
                if (has_vt) vt[x] = cmake<C>(qr[e], qi[e]);
            }
        }
    }
    nacc = warp_sum(nacc);
    if (lane == 0) snorm[warp] = nacc;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int u = 0; u < NW; ++u) t += snorm[u];
        part[(i64)blockIdx.x * ARN_PS + ARN_NORM] = t;
    }
}

// Sum of value i of the pass partial rows over nb blocks by one warp (lanes stride over
// the blocks, then a fixed shuffle tree: deterministic).  Result in every lane.
__device__ __forceinline__ double arn_sum_warp(const double *part, int nb, int i) {
    double t = 0.0;
    for (int b = threadIdx.x & 31; b < nb; b += 32) t += part[(i64)b * ARN_PS + i];
    return warp_sum(t);
}

__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a) b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// After pass A of iteration j: the lagged correction of v_j and of column j-1, column j of
// T, ||H v_j|| (krylov_exp.py:52), and pass B's coefficients (see the pass comments).
__global__ void __launch_bounds__(DECIDE_THREADS)
k_arn_lagstage(KState *ks, ArnState *as, int j, const double *part, int nb) {
    if (ks->status != KS_RUNNING) return;
    __shared__ double2 zs[ARN_M], ss[ARN_M], hs[ARN_M], cc[ARN_M];
    __shared__ double sa[4];
    __shared__ double salpha;
    __shared__ int bad;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NWD = DECIDE_THREADS / 32;
    const bool has_vt = j >= 1;
    const int nk = has_vt ? j : 1;
    if (tid == 0) bad = 0;
    for (int k = warp; k < nk; k += NWD) {  // one warp per value
        const double2 z = make_double2(arn_sum_warp(part, nb, 2 * k), arn_sum_warp(part, nb, 2 * k + 1));
        const double2 q = make_double2(arn_sum_warp(part, nb, ARN_S0 + 2 * k),
                                       arn_sum_warp(part, nb, ARN_S0 + 2 * k + 1));
        if (lane == 0) {
            zs[k] = z;
            ss[k] = has_vt ? q : make_double2(0.0, 0.0);
        }
    }
    if (warp == NWD - 1) {
        for (int i = 0; i < 4; ++i) {
            const double v = arn_sum_warp(part, nb, ARN_A0 + i);
            if (lane == 0) sa[i] = v;
        }
    }
    __syncthreads();
    if (tid == 0) {
        double alpha = 1.0;
        if (has_vt) {
            double s2 = 0.0;
            for (int k = 0; k < nk; ++k) s2 += ss[k].x * ss[k].x + ss[k].y * ss[k].y;
            const double a2 = sa[3] - s2;  // ||vt||^2 - |V^H vt|^2
            alpha = a2 > 0.0 ? sqrt(a2) : 0.0;
            if (!(alpha > 0.0) || !isfinite(alpha)) bad = 1;
            const double beta = ks->r[j - 1];
            for (int l = 0; l < j; ++l) {  // column j-1: w'_{j-1} = beta (alpha v_j + V s)
                double2 &t = as->T[l * ARN_M + (j - 1)];
                t.x += beta * ss[l].x;
                t.y += beta * ss[l].y;
            }
            as->T[j * ARN_M + (j - 1)] = make_double2(beta * alpha, 0.0);
            ks->r[j - 1] = beta * alpha;
        }
        salpha = alpha;
    }
    __syncthreads();
    const double alpha = salpha;
    // (T s)_l for l <= j over the columns k < j (Hessenberg rows: k >= l - 1)
    for (int l = tid; l <= j; l += DECIDE_THREADS) {
        double2 acc = make_double2(0.0, 0.0);
        if (has_vt)
            for (int k = l > 0 ? l - 1 : 0; k < j; ++k) {
                const double2 t = as->T[l * ARN_M + k], q = ss[k];
                acc.x += t.x * q.x - t.y * q.y;
                acc.y += t.x * q.y + t.y * q.x;
            }
        hs[l] = acc;
    }
    __syncthreads();
    if (tid == 0) {  // <v_j, w> = (<vt, w> - s^H z) / alpha
        if (has_vt) {
            double2 t = make_double2(sa[0], sa[1]);
            for (int k = 0; k < nk; ++k) {
                const double2 p = cmulc(ss[k], zs[k]);
                t.x -= p.x;
                t.y -= p.y;
            }
            zs[j] = make_double2(t.x / alpha, t.y / alpha);
        }
    }
    __syncthreads();
    for (int l = tid; l <= j; l += DECIDE_THREADS) {  // h_l = (z_l - (T s)_l) / alpha
        const double2 h = make_double2((zs[l].x - hs[l].x) / alpha, (zs[l].y - hs[l].y) / alpha);
        if (!isfinite(h.x) || !isfinite(h.y)) bad = 1;
        as->T[l * ARN_M + j] = h;
        cc[l] = make_double2(hs[l].x + alpha * h.x, hs[l].y + alpha * h.y);
        if (l == j) ks->a_re[j] = h.x;  // Re <v_j, (H - sigma) v_j>
    }
    __syncthreads();
    // pass B: w' = (w - V_j c) / alpha with v_j = (vt - V s) / alpha substituted
    for (int l = tid; l < nk; l += DECIDE_THREADS) {
        const double2 sl = ss[l], cj = has_vt ? cc[j] : make_double2(0.0, 0.0);
        const double2 p = make_double2((cj.x * sl.x - cj.y * sl.y) / alpha, (cj.x * sl.y + cj.y * sl.x) / alpha);
        as->cw1[l] = has_vt ? make_double2((cc[l].x - p.x) / alpha, (cc[l].y - p.y) / alpha) : cc[l];
        as->cvj[l] = make_double2(sl.x / alpha, sl.y / alpha);
    }
    if (tid == 0) {
        as->cw = 1.0 / alpha;
        as->cv = 1.0 / alpha;
        as->ct = has_vt ? make_double2(cc[j].x / (alpha * alpha), cc[j].y / (alpha * alpha))
                        : make_double2(0.0, 0.0);
        // ||(H - sigma) v_j||^2 = ||w - V_j (T s)||^2 / alpha^2, then ||H v_j||
        double n2 = sa[2];
        for (int l = 0; l <= j; ++l) {
            if (!has_vt && l > 0) break;
            const double2 p = cmulc(hs[l], zs[l]);
            n2 += -2.0 * p.x + hs[l].x * hs[l].x + hs[l].y * hs[l].y;
        }
        n2 /= alpha * alpha;
        const double sg = ks->shift;
        ks->hn[j] = sqrt(fmax(0.0, n2 + 2.0 * sg * ks->a_re[j] + sg * sg));
        if (!isfinite(n2)) bad = 1;
        if (bad) {
            ks->status = KS_NONFINITE;
            ks->iters = j + 1;
        }
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

// y = exp(A) e_0 for a caller's dense complex M x M matrix (row-major, complex128, in
// global memory): one block, the Arnoldi decision's Taylor routine; *status = 0, or
// EMUSV_NONFINITE when the matrix norm is not finite or too large for the substeps.
__global__ void __launch_bounds__(DECIDE_THREADS)
k_dense_expm_col(int M, const double2 *a_rowmajor, double2 *x, int *status) {
    extern __shared__ __align__(16) unsigned char arn_smem[];
    double2 *A = reinterpret_cast<double2 *>(arn_smem);
    double2 *y = A + M * M;
    double2 *t = y + M;
    double2 *tn = t + M;
    double *red = reinterpret_cast<double *>(tn + M);  // [DECIDE_THREADS]
    for (int i = threadIdx.x; i < M * M; i += DECIDE_THREADS) {
        const int r = i / M, c = i % M;
        A[c * M + r] = a_rowmajor[i];
    }
    __syncthreads();
    const bool ok = arn_expm_col0(A, M, y, t, tn, red);
    for (int k = threadIdx.x; k < M; k += DECIDE_THREADS)
        x[k] = ok ? y[k] : make_double2(nan(""), nan(""));
    if (threadIdx.x == 0) *status = ok ? EMUSV_OK : EMUSV_NONFINITE;
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
        as->T[(j + 1) * ARN_M + j] = make_double2(r, 0.0);  // krylov_exp.py:61 (until corrected)
        ks->r[j] = r;
        ks->scale[j + 1] = 1.0 / r;
        if (j >= 1) ks->scale[j] = 1.0;  // pass B stored the corrected v_j normalised
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

// Grid of the Gram-Schmidt passes: the streaming grid of the vector kernels (up to four
// blocks per SM), never more blocks than chunks; *grid_out receives it (the number of
// partial rows).
template <typename R>
static int launch_lagged(int pass, const KState *ks, const ArnState *as, int j, const void *v0,
                         unsigned char *basis, i64 D, void *w, double *part, cudaStream_t s,
                         int *grid_out) {
    constexpr int E = 4;
    i64 grid = krylov_stream_grid(D);
    const i64 chunks = (D + (i64)ORTHO_THREADS * E - 1) / ((i64)ORTHO_THREADS * E);
    if (grid > chunks) grid = chunks;
    *grid_out = (int)grid;
    ProfScope ps_(PROF_ORTH, s);
    if (pass == 0)
        k_arn_lagdots<R, E><<<(int)grid, ORTHO_THREADS, 0, s>>>(ks, j, v0, basis, D, w, part);
    else
        k_arn_lagupdate<R, E><<<(int)grid, ORTHO_THREADS, 0, s>>>(ks, as, j, v0, basis, D, w, part);
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

}  // namespace emusv

using namespace emusv;

extern "C" {

static size_t dense_expm_smem(int m) {
    return sizeof(double2) * ((size_t)m * m + 3 * (size_t)m) + sizeof(double) * DECIDE_THREADS;
}

size_t emusv_dense_expm_scratch_bytes(int m) {
    if (m < 1 || m > ARN_M) return 0;
    return align_up(sizeof(double2) * (size_t)m * m, 256) + align_up(sizeof(double2) * m, 256) + 256;
}

int emusv_dense_expm_col(int m, const double *a, double *x_dev, void *scratch, size_t scratch_bytes,
                         void *stream) {
    if (m < 1 || m > ARN_M || !a || !x_dev || !scratch || scratch_bytes < emusv_dense_expm_scratch_bytes(m))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    unsigned char *p = reinterpret_cast<unsigned char *>(scratch);
    double2 *A = reinterpret_cast<double2 *>(p);
    int *status = reinterpret_cast<int *>(p + align_up(sizeof(double2) * (size_t)m * m, 256) +
                                          align_up(sizeof(double2) * m, 256));
    EMUSV_CHECK(cudaMemcpyAsync(A, a, sizeof(double2) * (size_t)m * m, cudaMemcpyHostToDevice, s));
    const size_t smem = dense_expm_smem(m);
    EMUSV_CHECK(cudaFuncSetAttribute(k_dense_expm_col, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
        ProfScope ps_(PROF_SMALL, s);
        k_dense_expm_col<<<1, DECIDE_THREADS, smem, s>>>(m, A, reinterpret_cast<double2 *>(x_dev), status);
    }
    EMUSV_CHECK_LAUNCH();
    int h = 0;
    EMUSV_CHECK(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));  // the host matrix may be reused once this returns
    return h;
}

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
        for (int pass = 0; pass < 2; ++pass) {
            st = dtype == EMUSV_C128
                     ? launch_lagged<double>(pass, ks, as, j, psi_in, basis, D, w, part, s, &og)
                     : launch_lagged<float>(pass, ks, as, j, psi_in, basis, D, w, part, s, &og);
            if (st) return st;
            if (pass == 0) {
                ProfScope ps_(PROF_SMALL, s);
                k_arn_lagstage<<<1, DECIDE_THREADS, 0, s>>>(ks, as, j, part, og);
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
        EMUSV_CHECK(cudaMemcpyAsync(&h, ks, offsetof(KState, a_re), cudaMemcpyDeviceToHost, s));
        EMUSV_CHECK(cudaStreamSynchronize(s));
        info->iterations = h.iters;
        info->happy_breakdown = h.status == KS_HAPPY;
        info->converged = h.status == KS_HAPPY || h.status == KS_CONVERGED;
        info->basis_vectors = h.nvec;
        info->error_estimate = h.err;
        info->input_norm = h.s0;
        info->output_norm = sqrt(h.outnorm2);
        info->second_rounds = h.iters > 0 ? h.iters - 1 : 0;  // every vector but the first
    }
    return status == KS_MAXDIM ? EMUSV_NOT_CONVERGED : EMUSV_OK;
}

}  // namespace emusv
