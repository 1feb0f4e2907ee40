// Adjoint of one Krylov time step on the GPU (C ABI emusv_adjoint_step).
//
// Follows the reference backward pass (emu_sv/time_evolution/torch.py:223-378 with
// emu_base/math/double_krylov.py:5-113):
//   1. Lanczos bases V_s of the step's input state and V_g of the incoming gradient, with
//      double_krylov's stopping rule (lanczos_run, shared with the forward step);
//   2. dS = top-right block of exp([[T_s, c e0 e0^T], [0, T_g]]), c = |state| |grad|
//      (double_krylov.py:54-57), computed on the device: dS is linear in c, so the
//      exponential is taken with c = 1 (one warp per column, FP64 Taylor series with
//      scaling) and scaled afterwards;
//   3. E = dS^T V_s (torch.py:322), a register-blocked combination kernel;
//   4. one pass over the amplitudes: rho(x) = sum_k conj(Vg_k(x)) E_k(x), and for every
//      bit p the flip sums tau_p = sum_x sum_k conj(Vg_k(x)) E_k(x ^ bit_p), split by the
//      bit value of x -- all derivative operators of torch.py:36-119 reduce to these;
//   5. a pair-sum pass over rho for the detuning and interaction derivatives.
// The host turns the sums into dL/dOmega, dL/ddelta, dL/dphi, dL/dU exactly as
// torch.py:324-353 does with the sparse derivative operators.
#include <math.h>
#include <string.h>

#include <initializer_list>

#include "krylov_device.cuh"
#include "profile.cuh"

namespace emusv {

constexpr int ADJ_MAXQ = 20;  // largest register the adjoint handles (register accumulators)
constexpr int ADJ_KC = 8;     // outputs per thread of the combination kernel

struct AdjScal {
    double sums[4 * ADJ_MAXQ + 8];  // [T_re, T_im, U_re, U_im] x bits, then rho sums
    double pairs[2 * ADJ_MAXQ * ADJ_MAXQ];
};

static size_t al(size_t v) { return (v + 255) / 256 * 256; }

struct AdjWorkspace {
    KState *ks_s, *ks_g;
    double *part_h, *part_o, *part_c;
    double2 *dS;  // [KMAX][KMAX] (row i of the state basis, column k of the grad basis)
    AdjScal *scal;
    unsigned char *basis_s, *basis_g, *E, *rho;
    int capacity;
};

int max_grid_blocks();
static size_t part_bytes() { return al(sizeof(double) * max_grid_blocks() * (4 * ADJ_MAXQ + 8)); }
static size_t adj_header() {
    return 2 * al(sizeof(KState)) + 3 * part_bytes() + al(sizeof(double2) * KMAX * KMAX) +
           al(sizeof(AdjScal));
}

static bool carve_adj(void *ws, size_t bytes, int64_t D, size_t es, AdjWorkspace *W) {
    unsigned char *p = reinterpret_cast<unsigned char *>(ws);
    size_t off = 0;
    auto take = [&](size_t b) {
        unsigned char *q = p + off;
        off += al(b);
        return q;
    };
    W->ks_s = reinterpret_cast<KState *>(take(sizeof(KState)));
    W->ks_g = reinterpret_cast<KState *>(take(sizeof(KState)));
    W->part_h = reinterpret_cast<double *>(take(part_bytes()));
    W->part_o = reinterpret_cast<double *>(take(part_bytes()));
    W->part_c = reinterpret_cast<double *>(take(part_bytes()));
    W->dS = reinterpret_cast<double2 *>(take(sizeof(double2) * KMAX * KMAX));
    W->scal = reinterpret_cast<AdjScal *>(take(sizeof(AdjScal)));
    if (bytes < off) return false;
    const size_t vb = (size_t)D * es;
    // remaining: rho (16 bytes per amplitude), then basis_s, basis_g and E (cap+1 each)
    const size_t rb = al((size_t)D * 16);
    if (bytes < off + rb) return false;
    const int64_t nvec = (int64_t)((bytes - off - rb) / vb);
    const int cap = (int)(nvec / 3) - 1;
    if (cap < 1) return false;
    W->rho = p + off;
    off += rb;
    W->capacity = cap;
    W->basis_s = p + off;
    W->basis_g = W->basis_s + (size_t)(cap + 1) * vb;
    W->E = W->basis_g + (size_t)(cap + 1) * vb;
    return true;
}

// ------------------------------------------------------------------ dS = exp(B) block
// Column col of dS: y = exp(B) e_{ms+col} for B = [[A_s, e0 e0^T], [0, A_g]] (A = -i dt T
// of each basis, coupling 1; double_krylov.py:54-57), rows 0..ms-1.  T (double_krylov.py:
// 100-113) has size m = j+2 after convergence (last row: T[j+1][j] = ||w_j||, T[j+1][j+1]
// = 0) or j+1 after a happy breakdown.  One warp per column, Chebyshev form
// (cheb_expm: the spectrum of B is that of its two blocks).
__device__ __forceinline__ void adj_block_row(const KState *ks, int kk, int m, double dt,
                                              double2 &d, double2 &l, double2 &u, double &td,
                                              double &tr) {
    const int jj = ks->iters - 1;
    d = l = u = make_double2(0.0, 0.0);
    td = tr = 0.0;
    if (kk <= jj) {
        d = make_double2(dt * ks->a_im[kk], -dt * (ks->a_re[kk] + ks->shift));
        td = ks->a_re[kk] + ks->shift;
        tr = fabs(ks->a_im[kk]);
    }
    if (kk >= 1) {
        l = make_double2(0.0, -dt * ks->r[kk - 1]);
        tr += fabs(ks->r[kk - 1]);
    }
    if (kk + 1 <= jj && kk + 1 < m) {
        u = make_double2(dt * ks->b_im[kk + 1], -dt * ks->b_re[kk + 1]);
        tr += hypot(ks->b_re[kk + 1], ks->b_im[kk + 1]);
    }
}

constexpr int DS_WARPS = 4;
constexpr int ADS_NE = (2 * KMAX + 31) / 32;

__global__ void __launch_bounds__(32 * DS_WARPS)
k_dS(const KState *ks_s, const KState *ks_g, double dt, double2 *dS) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ms = ks_s->status == 2 ? ks_s->iters : ks_s->iters + 1;
    const int mg = ks_g->status == 2 ? ks_g->iters : ks_g->iters + 1;
    const int M = ms + mg;
    const int col = blockIdx.x * DS_WARPS + warp;
    if (col >= mg || M > 32 * ADS_NE) return;
    double2 d[ADS_NE], l[ADS_NE], u[ADS_NE], y[ADS_NE];
    double td[ADS_NE], tr[ADS_NE];
#pragma unroll
    for (int e = 0; e < ADS_NE; ++e) {
        const int k = lane * ADS_NE + e;
        d[e] = l[e] = u[e] = make_double2(0.0, 0.0);
        td[e] = tr[e] = 0.0;
        if (k < ms) adj_block_row(ks_s, k, ms, dt, d[e], l[e], u[e], td[e], tr[e]);
        else if (k < M) adj_block_row(ks_g, k - ms, mg, dt, d[e], l[e], u[e], td[e], tr[e]);
        if (k == 0) tr[e] += 1.0 / fabs(dt);  // the coupling entry 1 in T units
    }
    cheb_expm<ADS_NE>(d, l, u, ms, make_double2(1.0, 0.0), ms + col, dt, td, tr, M, y);
#pragma unroll
    for (int e = 0; e < ADS_NE; ++e) {
        const int r = lane * ADS_NE + e;
        if (r < ms) dS[r * KMAX + col] = y[e];
    }
}

// ------------------------------------------------------------------ E = dS^T V_s
// E_k = sum_i dS[i][k] * scale_s[i] * stored_s_i, k < mg.  Each thread: one amplitude,
// ADJ_KC outputs.
template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_ecomb(const KState *ks_s, const KState *ks_g, const double2 *dS, const void *v0_,
        const unsigned char *basis_s, unsigned char *E_, int64_t D) {
    typedef typename cvec<R>::T C;
    __shared__ double2 cf[KMAX][ADJ_KC];
    const int ms = ks_s->status == 2 ? ks_s->iters : ks_s->iters + 1;
    const int mg = ks_g->status == 2 ? ks_g->iters : ks_g->iters + 1;
    const int k0 = blockIdx.y * ADJ_KC;
    if (k0 >= mg) return;
    for (int e = threadIdx.x; e < ms * ADJ_KC; e += blockDim.x) {
        const int i = e / ADJ_KC, kk = e % ADJ_KC;
        const double sc = ks_s->scale[i];
        const double2 v = (k0 + kk < mg) ? dS[i * KMAX + k0 + kk] : make_double2(0.0, 0.0);
        cf[i][kk] = make_double2(sc * v.x, sc * v.y);
    }
    __syncthreads();
    const C *v0 = reinterpret_cast<const C *>(v0_);
    const C *bs = reinterpret_cast<const C *>(basis_s);
    C *E = reinterpret_cast<C *>(E_);
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < D;
         x += (int64_t)gridDim.x * blockDim.x) {
        double ar[ADJ_KC], ai[ADJ_KC];
#pragma unroll
        for (int kk = 0; kk < ADJ_KC; ++kk) ar[kk] = ai[kk] = 0.0;
        for (int i = 0; i < ms; ++i) {
            const C a = i == 0 ? v0[x] : bs[(int64_t)i * D + x];
            const double xr = double(a.x), xi = double(a.y);
#pragma unroll
            for (int kk = 0; kk < ADJ_KC; ++kk) {
                const double2 c = cf[i][kk];
                ar[kk] += c.x * xr - c.y * xi;
                ai[kk] += c.x * xi + c.y * xr;
            }
        }
#pragma unroll
        for (int kk = 0; kk < ADJ_KC; ++kk)
            if (k0 + kk < mg) E[(int64_t)(k0 + kk) * D + x] = cmake<C>(ar[kk], ai[kk]);
    }
}

// ------------------------------------------------------------------ contractions
// Per block partials: [T_re, T_im, U_re, U_im] for each bit p < n (T = sum tau_p,
// U = the part of that sum over amplitudes x with bit p set), then sum rho.  rho(x) is
// also written out for the pair sums.  NB >= n bounds the register accumulators.
template <typename R, int NB>
__global__ void __launch_bounds__(BLOCK)
k_contract(const KState *ks_g, int n, const void *g0_, const unsigned char *basis_g,
           const unsigned char *E_, int64_t D, double *rho_out, double *partials) {
    typedef typename cvec<R>::T C;
    __shared__ double red[(BLOCK / 32) * 4];
    __shared__ double gsc[KMAX + 2];
    const int mg = ks_g->status == 2 ? ks_g->iters : ks_g->iters + 1;
    for (int k = threadIdx.x; k < mg; k += blockDim.x) gsc[k] = ks_g->scale[k];
    __syncthreads();
    const C *g0 = reinterpret_cast<const C *>(g0_);
    const C *bg = reinterpret_cast<const C *>(basis_g);
    const C *E = reinterpret_cast<const C *>(E_);
    double Tr[NB], Ti[NB], Ur[NB], Ui[NB];
#pragma unroll
    for (int p = 0; p < NB; ++p) Tr[p] = Ti[p] = Ur[p] = Ui[p] = 0.0;
    double sr = 0.0, si = 0.0;
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < D;
         x += (int64_t)gridDim.x * blockDim.x) {
        double rr = 0.0, ri = 0.0;
        for (int k = 0; k < mg; ++k) {
            const C gv = k == 0 ? g0[x] : bg[(int64_t)k * D + x];
            const double gr = gsc[k] * double(gv.x), gi = -gsc[k] * double(gv.y);  // conj
            const C *Ek = E + (int64_t)k * D;
            const C e = Ek[x];
            rr += gr * double(e.x) - gi * double(e.y);
            ri += gr * double(e.y) + gi * double(e.x);
#pragma unroll
            for (int p = 0; p < NB; ++p) {
                if (p < n) {
                    const C w = Ek[x ^ (int64_t(1) << p)];
                    const double tr = gr * double(w.x) - gi * double(w.y);
                    const double ti = gr * double(w.y) + gi * double(w.x);
                    const double bit = double((x >> p) & 1);
                    Tr[p] += tr;
                    Ti[p] += ti;
                    Ur[p] += bit * tr;
                    Ui[p] += bit * ti;
                }
            }
        }
        rho_out[2 * x] = rr;
        rho_out[2 * x + 1] = ri;
        sr += rr;
        si += ri;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int PSTRIDE = 4 * ADJ_MAXQ + 8;
#pragma unroll
    for (int p = 0; p <= NB; ++p) {
        if (p > n) break;
        double v4[4];
        if (p < n) {
            v4[0] = Tr[p < NB ? p : 0];
            v4[1] = Ti[p < NB ? p : 0];
            v4[2] = Ur[p < NB ? p : 0];
            v4[3] = Ui[p < NB ? p : 0];
        } else {  // after the bits: the rho sums
            v4[0] = sr;
            v4[1] = si;
            v4[2] = v4[3] = 0.0;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) v4[c] = warp_sum(v4[c]);
        if (lane == 0)
#pragma unroll
            for (int c = 0; c < 4; ++c) red[warp * 4 + c] = v4[c];
        __syncthreads();
        if (threadIdx.x < 4) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w * 4 + threadIdx.x];
            const int v = 4 * p + threadIdx.x;
            if (p < n || threadIdx.x < 2) partials[(int64_t)blockIdx.x * PSTRIDE + v] = t;
        }
        __syncthreads();
    }
}

__global__ void k_sum_adj(const double *partials, int nblocks, int nv, double *out) {
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partials[(int64_t)b * (4 * ADJ_MAXQ + 8) + v];
        out[v] = s;
    }
}

constexpr int PAIR_HB = 6;  // high bits enumerated per thread by k_pairs

// Pair sums S_PQ = sum_x x_P x_Q rho(x) for bit positions P <= Q (complex).  Thread t owns
// the amplitudes x = t + (k << s), s = n - h, k < 2^h (h = min(n, PAIR_HB)): its low s
// bits are fixed, so only the h high bits need per-amplitude accumulators (the total, one
// per high bit, one per high pair); the low bits enter when the pairs are reduced.
__global__ void __launch_bounds__(BLOCK)
k_pairs(const double *rho, int n, double *partials) {
    __shared__ double acc[2 * ADJ_MAXQ * ADJ_MAXQ];
    constexpr int NHH = PAIR_HB * (PAIR_HB + 1) / 2;
    const int h = n < PAIR_HB ? n : PAIR_HB, s = n - h;
    for (int k = threadIdx.x; k < 2 * n * n; k += blockDim.x) acc[k] = 0.0;
    __syncthreads();
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double Rr = 0.0, Ri = 0.0, Hr[PAIR_HB], Hi[PAIR_HB], HHr[NHH], HHi[NHH];
#pragma unroll
    for (int q = 0; q < PAIR_HB; ++q) Hr[q] = Hi[q] = 0.0;
#pragma unroll
    for (int q = 0; q < NHH; ++q) HHr[q] = HHi[q] = 0.0;
    if (t < (int64_t(1) << s)) {
        for (int k = 0; k < (1 << h); ++k) {
            const int64_t x = t + ((int64_t)k << s);
            const double rr = rho[2 * x], ri = rho[2 * x + 1];
            Rr += rr;
            Ri += ri;
            int idx = 0;
#pragma unroll
            for (int q = 0; q < PAIR_HB; ++q) {
                const double fq = double((k >> q) & 1);
                Hr[q] += fq * rr;
                Hi[q] += fq * ri;
#pragma unroll
                for (int p = 0; p <= q; ++p, ++idx) {
                    const double f = fq * double((k >> p) & 1);
                    HHr[idx] += f * rr;
                    HHi[idx] += f * ri;
                }
            }
        }
    }
    const int lane = threadIdx.x & 31;
    auto add = [&](int P, int Q, double vr, double vi) {
        vr = warp_sum(vr);
        vi = warp_sum(vi);
        if (lane == 0) {
            atomicAdd(&acc[2 * (P * n + Q)], vr);
            atomicAdd(&acc[2 * (P * n + Q) + 1], vi);
        }
    };
    for (int P = 0; P < s; ++P) {
        const double fP = double((t >> P) & 1);
        for (int Q = P; Q < s; ++Q) {  // both bits low: fixed for this thread
            const double f = fP * double((t >> Q) & 1);
            add(P, Q, f * Rr, f * Ri);
        }
#pragma unroll
        for (int q = 0; q < PAIR_HB; ++q)  // P low, Q = s + q high
            if (q < h) add(P, s + q, fP * Hr[q], fP * Hi[q]);
    }
    int idx = 0;
#pragma unroll
    for (int q = 0; q < PAIR_HB; ++q)
#pragma unroll
        for (int p = 0; p <= q; ++p, ++idx)
            if (q < h) add(s + p, s + q, HHr[idx], HHi[idx]);
    __syncthreads();
    for (int k = threadIdx.x; k < 2 * n * n; k += blockDim.x)
        partials[(int64_t)blockIdx.x * 2 * ADJ_MAXQ * ADJ_MAXQ + k] = acc[k];
}

__global__ void k_sum_pairs(const double *partials, int nblocks, int n, double *out) {
    for (int k = threadIdx.x; k < 2 * n * n; k += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partials[(int64_t)b * 2 * ADJ_MAXQ * ADJ_MAXQ + k];
        out[k] = s;
    }
}

}  // namespace emusv

using namespace emusv;

extern "C" {

size_t emusv_adjoint_workspace_bytes(int nqubits, int dtype, int basis_capacity) {
    if (nqubits < 1 || nqubits > ADJ_MAXQ || basis_capacity < 1 ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64))
        return 0;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    const size_t vb = (size_t(1) << nqubits) * es;
    return adj_header() + al((size_t(1) << nqubits) * 16) +
           (size_t)(3 * (basis_capacity + 1)) * vb + 4096;
}

int emusv_adjoint_step(int nqubits, int dtype, double dt, const double *omegas,
                       const double *deltas, const double *phis, const double *interaction,
                       const void *state, const void *grad_out, double tolerance,
                       int max_krylov_dim, double *g_omegas, double *g_deltas, double *g_phis,
                       double *g_interaction, void *workspace, size_t workspace_bytes,
                       void *stream) {
    HamParams P;
    if (nqubits < 1 || nqubits > ADJ_MAXQ || !state || !grad_out || !workspace ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64) || max_krylov_dim < 1 ||
        max_krylov_dim > KMAX - 2 || !isfinite(dt) ||
        !make_params(nqubits, omegas, deltas, phis, interaction, &P))
        return EMUSV_BAD_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return EMUSV_BAD_ARGUMENT;
    const int64_t D = int64_t(1) << nqubits;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    AdjWorkspace W;
    if (!carve_adj(workspace, workspace_bytes, D, es, &W)) return EMUSV_WORKSPACE_TOO_SMALL;
    cudaStream_t s = as_stream(stream);
    const int n = nqubits;

    // 1. the two Lanczos bases (double_krylov.py:51-52), both tolerances = tolerance
    int st_s = 0, st_g = 0;
    int st = lanczos_run(P, dtype, dt, state, W.ks_s, W.part_h, W.part_o, W.basis_s, W.capacity,
                         tolerance, tolerance, max_krylov_dim, 0, false, s, &st_s);
    if (st) return st;
    if (st_s == 0) return EMUSV_WORKSPACE_TOO_SMALL;
    st = lanczos_run(P, dtype, dt, grad_out, W.ks_g, W.part_h, W.part_o, W.basis_g, W.capacity,
                     tolerance, tolerance, max_krylov_dim, 0, false, s, &st_g);
    if (st) return st;
    if (st_g == 0) return EMUSV_WORKSPACE_TOO_SMALL;
    int hg[2];
    double s0[2];
    EMUSV_CHECK(cudaMemcpyAsync(hg, &W.ks_g->status, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaMemcpyAsync(&s0[0], &W.ks_s->s0, sizeof(double), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaMemcpyAsync(&s0[1], &W.ks_g->s0, sizeof(double), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));
    if (s0[0] == 0.0 || s0[1] == 0.0) {  // a zero state or gradient: dU|s><g| = 0
        for (int i = 0; i < n; ++i) {
            if (g_omegas) g_omegas[i] = 0.0;
            if (g_deltas) g_deltas[i] = 0.0;
            if (g_phis) g_phis[i] = 0.0;
        }
        if (g_interaction) memset(g_interaction, 0, sizeof(double) * n * n);
        return EMUSV_OK;
    }
    for (int r : {st_s, st_g}) {
        if (r == KS_MAXDIM) return EMUSV_NOT_CONVERGED;  // double_krylov.py:107-110
        if (r == EMUSV_TIMEOUT) return EMUSV_TIMEOUT;
        if (r != KS_CONVERGED && r != KS_HAPPY) return EMUSV_NONFINITE;
    }
    // size of the gradient basis (the dS columns)
    const int mg = hg[0] == KS_HAPPY ? hg[1] : hg[1] + 1;

    // 2. dS (c = 1; scaled by c = |state||grad| below)
    {
        ProfScope ps_(PROF_ADJOINT, s);
        k_dS<<<(mg + DS_WARPS - 1) / DS_WARPS, 32 * DS_WARPS, 0, s>>>(W.ks_s, W.ks_g, dt, W.dS);
    }
    EMUSV_CHECK_LAUNCH();
    // 3. E = dS^T V_s
    int gx = (int)((D + BLOCK - 1) / BLOCK);
    if (gx > sm_count() * 4) gx = sm_count() * 4;
    {
        dim3 grid(gx, (mg + ADJ_KC - 1) / ADJ_KC);
        ProfScope ps_(PROF_ADJOINT, s);
        if (dtype == EMUSV_C128)
            k_ecomb<double><<<grid, BLOCK, 0, s>>>(W.ks_s, W.ks_g, W.dS, state, W.basis_s, W.E, D);
        else
            k_ecomb<float><<<grid, BLOCK, 0, s>>>(W.ks_s, W.ks_g, W.dS, state, W.basis_s, W.E, D);
    }
    EMUSV_CHECK_LAUNCH();
    // 4. flip sums and rho
    double *rho = reinterpret_cast<double *>(W.rho);
    {
        ProfScope ps_(PROF_ADJOINT, s);
#define EMUSV_CONTRACT(R, NB) \
    k_contract<R, NB><<<gx, BLOCK, 0, s>>>(W.ks_g, n, grad_out, W.basis_g, W.E, D, rho, W.part_c)
        if (dtype == EMUSV_C128) {
            if (n <= 12) EMUSV_CONTRACT(double, 12);
            else if (n <= 16) EMUSV_CONTRACT(double, 16);
            else EMUSV_CONTRACT(double, 20);
        } else {
            if (n <= 12) EMUSV_CONTRACT(float, 12);
            else if (n <= 16) EMUSV_CONTRACT(float, 16);
            else EMUSV_CONTRACT(float, 20);
        }
#undef EMUSV_CONTRACT
    }
    EMUSV_CHECK_LAUNCH();
    {
        ProfScope ps_(PROF_ADJOINT, s);
        k_sum_adj<<<1, BLOCK, 0, s>>>(W.part_c, gx, 4 * n + 2, W.scal->sums);
    }
    EMUSV_CHECK_LAUNCH();
    const bool want_pairs = g_deltas || g_interaction;
    if (want_pairs) {
        // the pair partials reuse part_h/part_o (both Lanczos runs are finished)
        const int hb = n < PAIR_HB ? n : PAIR_HB;
        const int gp = (int)(((int64_t(1) << (n - hb)) + BLOCK - 1) / BLOCK);
        const size_t per = 2 * ADJ_MAXQ * ADJ_MAXQ;
        if ((size_t)gp * per > 2 * part_bytes() / sizeof(double)) return EMUSV_BAD_ARGUMENT;
        {
            ProfScope ps_(PROF_ADJOINT, s);
            k_pairs<<<gp, BLOCK, 0, s>>>(rho, n, W.part_h);
            k_sum_pairs<<<1, BLOCK, 0, s>>>(W.part_h, gp, n, W.scal->pairs);
        }
        EMUSV_CHECK_LAUNCH();
    }
    AdjScal H;
    EMUSV_CHECK(cudaMemcpyAsync(&H, W.scal, sizeof(AdjScal), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));

    // 5. gradients (torch.py:324-353): g = Re(-i dt * c * <contraction>)
    const double c = s0[0] * s0[1];
    auto pre = [&](double re, double im, double *out) {  // Re(-i dt c (re + i im))
        *out = dt * c * im;
    };
    for (int i = 0; i < n; ++i) {
        const int p = n - 1 - i;  // qubit i is bit n-1-i
        const double Tre = H.sums[4 * p], Tim = H.sums[4 * p + 1];
        const double Ure = H.sums[4 * p + 2], Uim = H.sums[4 * p + 3];
        const double Dre = Tre - Ure, Dim = Tim - Uim;  // sum over x with bit p clear
        // derivative coefficient a on |r><g| (x_p = 1 side) and conj(a) on |g><r|
        auto flip = [&](double ar, double ai, double *out) {
            const double re = ar * Ure - ai * Uim + ar * Dre + ai * Dim;
            const double im = ar * Uim + ai * Ure + ar * Dim - ai * Dre;
            pre(re, im, out);
        };
        if (g_omegas) {  // DHDOmegaSparse: a = 0.5 e^{i phi}
            flip(0.5 * cos(phis[i]), 0.5 * sin(phis[i]), &g_omegas[i]);
        }
        if (g_phis) {  // DHDPhiSparse: a = 0.5 Omega e^{i (phi + pi/2)}
            flip(-0.5 * omegas[i] * sin(phis[i]), 0.5 * omegas[i] * cos(phis[i]), &g_phis[i]);
        }
        if (g_deltas) {  // DHDDeltaSparse: -n_i
            const double re = -H.pairs[2 * (p * n + p)], im = -H.pairs[2 * (p * n + p) + 1];
            pre(re, im, &g_deltas[i]);
        }
    }
    if (g_interaction) {  // DHDUSparse: n_i n_j, upper triangle (torch.py:347-353)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double g = 0.0;
                if (j > i) {
                    const int p = n - 1 - j, q = n - 1 - i;  // p < q
                    pre(H.pairs[2 * (p * n + q)], H.pairs[2 * (p * n + q) + 1], &g);
                }
                g_interaction[i * n + j] = g;
            }
    }
    return EMUSV_OK;
}

}  // extern "C"
