// Batched time evolution in ONE persistent launch (C ABI emusv_batch_*).
//
// Many registers of uneven size (up to BMAXQ qubits each), each with its own pulse, are
// evolved through all their Krylov steps (krylov_exp.py:23-131 per step, as
// emusv_krylov_step does for one register) by a single cooperative kernel that keeps
// every SM busy with every register's work:
//
//  * vectors: one "slot" holds one vector of every instance back to back (instance i at
//    amplitude offset off_i); slot 0 is the caller's packed states (evolved in place),
//    slots 1..capacity the stored Lanczos vectors.  A tile is 2^T consecutive amplitudes of
//    one instance; tiles of all instances form one list that warps take in order from a
//    global counter (dynamic balance; neighbouring tiles run together, so partner tiles of
//    the bits above T are read from L2).
//  * a warp owns a tile: lane bits (tile bits 0-4) flip by shuffles, register bits (5..T-1)
//    inside the thread, bits >= T from the partner tiles, staged through the warp's
//    shared-memory stages by cp.async (three in flight); the diagonal is rebuilt from an
//    FP64 per-instance table of the low-bit pair energies plus per-tile fields of the high
//    bits.
//  * per Lanczos iteration j, two grid-wide phases: A_j (H v_j for every running
//    instance, FP64 partials of ||Hv||^2 and <v_j,Hv>) and B_j (three-term recurrence and
//    partials of ||w||^2, <v_j,w>).  The per-instance decision for iteration j (norm,
//    happy breakdown, extended tridiagonal exponential, error estimate: krylov_decide)
//    runs in warp 0 of one CTA per instance during phase A_{j+1}, overlapping the next
//    H v, whose result is discarded if the instance converged.  After the iterations of
//    a step, a combination phase writes psi' = s0 sum_k c_k v_k in place and its norm.
//  * grid barriers are an arrival counter plus a generation word; every wait is bounded
//    (about a second of SM clock): on a timeout the kernel records EMUSV_TIMEOUT and
//    every CTA returns.  The launch is cooperative, so all CTAs are co-resident.
//  * convergence is tested from a per-instance hint (the previous step's count - 3); a
//    first test that already converges tests the skipped iterations in order
//    (krylov_decide), so each instance stops where the reference would.
//  * a second scheduler, the phase engine (run_jobs, below), lets every register run its
//    own sequence of phases -- norm, A_0, B_0, ..., B_e, combination -- with no grid
//    barrier: warps visit registers in proportion to their size and take tiles of the
//    visited register's current phase from its take counter.  It builds the adjoint's
//    two bases per step (k_batch_adj_rounds) and is a forward choice
//    (emusv_batch_set_engine; BatchEvolution's autotuner times both).  The lock-step
//    rounds win on batches of uneven registers (256 registers of 12-18 qubits, 150
//    steps: 0.79 s against 0.92 s), the phases on uniform ones (64 registers of 16 qubits,
//    the gradient batch's forward).
#include <math.h>
#include <string.h>

#include <initializer_list>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "krylov_device.cuh"
#include "profile.cuh"

namespace emusv {

constexpr int BMAXQ = 20;   // largest register of a batch
constexpr int BWARPS = 8;   // warps per CTA
constexpr int BS_IDLE = 16;      // instance has no step left
constexpr int BS_CAPACITY = 17;  // Krylov basis larger than the workspace's capacity
constexpr long long BAR_LIMIT = 2000000000LL;  // clock cycles a barrier waits at most

// One Lanczos "job": an instance's state (the forward evolution, or the state half of an
// adjoint step) or an adjoint step's incoming gradient.
struct BInst {
    int n, nsteps, tile0, ntiles;
    long long off;   // amplitude offset of this job in every stored-vector slot
    long long off0;  // offset of its vector 0 in the buffer v0[src]
    double dt;
    int coef0;       // index of the instance's step-0 record in the coefficient array
    int pidx;        // instance index (interaction tables)
    int src;         // vector 0 lives in v0[src]
    int pad;
};

// Per (instance, step) coefficients by bit position p (qubit n-1-p).
struct BCoef {
    double up_re[BMAXQ], up_im[BMAXQ];  // coefficient of |1><0| on bit p (Omega/2 e^{i phi})
    double field[BMAXQ];                // -delta
    double om[BMAXQ], ph[BMAXQ];        // Omega and phi (the adjoint's derivative operators)
    float fup_re[BMAXQ], fup_im[BMAXQ];
};

struct BCtl {
    unsigned bar_count, bar_gen;
    unsigned tile_ctr[2];
    int err;
    unsigned idle;                // phase engine: jobs with no phase left in this launch
    unsigned long long item;      // phase engine: the visit cursor
};

struct BArgs {
    int ninst, T, total_tiles, maxdim, capacity, max_steps;
    double exp_tol, norm_tol;
    const BInst *inst;
    const BCoef *coef;
    const double *Ubits;  // [ninst][BMAXQ*BMAXQ], U of bit positions p < q at [p*BMAXQ+q]
    const double *Elow;   // [ninst][2^T]: sum over bit pairs p<q<T of U_pq x_p x_q
    KState *ks;           // [ninst]
    int *hint, *polled, *fail, *status_out;  // [ninst]
    int *iters_out;       // [ninst][max_steps]
    double *partA, *partB, *partN;  // [total_tiles][4] per-tile FP64 partial sums
    double *sumA, *sumB, *sumN;     // [ninst][4] their per-instance totals
    unsigned *cnt;                  // [3][ninst] tiles done per phase kind (A, B, N)
    int *ranB;                      // [ninst] 1 + last round whose phase B ran the instance
    unsigned long long *jst;        // [ninst] phase engine: (phases completed << 32) | the
                                    // code of the job's next phase (see run_jobs)
    unsigned long long *take;       // [ninst] phase engine: (current phase << 32) | tiles taken
    void *v0[2];          // buffers holding every job's vector 0 (forward: the packed states,
                          // evolved in place; adjoint: states and incoming gradients)
    unsigned char *slots;  // slots 1..capacity
    long long slot_amps;
    BCtl *ctl;
    // set per launch
    int first_step;       // absolute index of the launch's first step
    int run_steps;        // steps this launch takes
    int combine;          // phase engine: 1 ends each step with the combination, 0 (the
                          // adjoint's bases) leaves the step's Krylov basis
    void *hist;           // optional: states after every hist_every-th step
    int hist_every;
    long long hist_stride;  // amplitudes per history slot
    // grid barrier: clock cycles a wait lasts at most (BAR_LIMIT unless a test shortens
    // it) and the failure-path test switch (emusv_batch_set_barrier_test): the last CTA
    // does not arrive at a launch's first barrier, so every other CTA's wait runs out
    long long bar_limit;
    int test_skip_arrival;
};

// Adjoint step (k_batch_adj): jobs 2i (state psi_i) and 2i+1 (gradient g_i) of instance i.
struct BAdj {
    int ninst, step, mmax;  // instances, absolute step, largest basis (scratch sizing)
    double2 *dS;            // [ninst][mmax*mmax]: dS[r][k] at r*mmax + k
    unsigned char *E;       // E_k of every instance: [mmax][inst_amps]
    long long inst_amps;
    double *partC;          // [total job tiles][NCP] contraction partials
    double *grads;          // [ninst][3][BMAXQ] dL/dOmega, dL/ddelta, dL/dphi by qubit
    void *gout;             // packed state gradient exp(+i dt H) g
    unsigned *cntC;         // [ninst]
    int *astatus;           // [ninst] emusv status of the instance's adjoint
};
constexpr int NCP = 6 * BMAXQ;  // per bit: T_re, T_im, U_re, U_im, S_re, S_im

// ---------------------------------------------------------------- grid barrier
// Arrival counter + generation; the last arriver also clears the tile counter of the
// phase after next.  Returns false (and every CTA then returns) on a timeout: a wait
// gives up after A.bar_limit clock cycles or as soon as another CTA recorded an error.
__device__ bool grid_sync(const BArgs &A, unsigned &ph) {
    __shared__ int s_ok;  // the CTA's outcome, read by every thread (all return together)
    BCtl *ctl = A.ctl;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *genp = &ctl->bar_gen;
        const unsigned g = *genp;
        __threadfence();
        const bool skip = A.test_skip_arrival && ph == 0 && blockIdx.x == gridDim.x - 1;
        const unsigned arrived = skip ? 0u : atomicAdd(&ctl->bar_count, 1u);
        if (!skip && arrived == gridDim.x - 1) {
            ctl->bar_count = 0;
            ctl->tile_ctr[(ph + 1) & 1] = 0;
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            const long long t0 = clock64();
            int polls = 0;
            while (*genp == g) {
                if (++polls == 64) {
                    polls = 0;
                    if (clock64() - t0 > A.bar_limit || *(volatile int *)&ctl->err) {
                        atomicExch(&ctl->err, EMUSV_TIMEOUT);
                        break;
                    }
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        s_ok = *(volatile int *)&ctl->err == 0;
    }
    __syncthreads();
    ++ph;
    return s_ok != 0;
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ int next_tile(BCtl *ctl, unsigned ph) {
    int t = 0;
    if ((threadIdx.x & 31) == 0) t = (int)atomicAdd(&ctl->tile_ctr[ph & 1], 1u);
    return __shfl_sync(0xffffffffu, t, 0);
}

__device__ __forceinline__ int inst_of_tile(const BArgs &A, int t) {
    int lo = 0, hi = A.ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&A.inst[mid].tile0) <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Deterministic FP64 sums of an instance's per-tile partials (same order everywhere).
__device__ __forceinline__ double3 inst_sum(const double *part, int tile0, int ntiles) {
    const int lane = threadIdx.x & 31;
    double a = 0.0, b = 0.0, c = 0.0;
    for (int k = lane; k < ntiles; k += 32) {
        const double2 v01 = __ldcg(reinterpret_cast<const double2 *>(part + 4 * (size_t)(tile0 + k)));
        a += v01.x;
        b += v01.y;
        c += __ldcg(part + 4 * (size_t)(tile0 + k) + 2);
    }
    return make_double3(warp_sum(a), warp_sum(b), warp_sum(c));
}

// After a warp wrote its tile's partials: count the tile; the warp that completes the
// instance adds the instance's partials (inst_sum: the same order whichever warp it is)
// into sum[4 i..], clears the counter for the next phase of this kind and returns true.
__device__ __forceinline__ bool tile_done(unsigned *cnt, const double *part, double *sum, int i,
                                          int tile0, int ntiles) {
    const int lane = threadIdx.x & 31;
    unsigned old = 0;
    if (lane == 0) {
        __threadfence();
        old = atomicAdd(&cnt[i], 1u);
    }
    old = __shfl_sync(0xffffffffu, old, 0);
    const bool last = old == (unsigned)ntiles - 1;
    if (last) {
        __threadfence();
        const double3 s = inst_sum(part, tile0, ntiles);
        if (lane == 0) {
            sum[4 * (size_t)i] = s.x;
            sum[4 * (size_t)i + 1] = s.y;
            sum[4 * (size_t)i + 2] = s.z;
            cnt[i] = 0;
            __threadfence();
        }
    }
    __syncwarp();
    return last;
}

__device__ __forceinline__ double3 ld_sum(const double *sum, int i) {
    return make_double3(__ldcg(sum + 4 * (size_t)i), __ldcg(sum + 4 * (size_t)i + 1),
                        __ldcg(sum + 4 * (size_t)i + 2));
}

// |o|^2 added to an FP64 sum with explicit fused operations, so the norm of a vector
// written by a combination and the norm of the same vector read back agree to the bit.
template <typename C>
__device__ __forceinline__ void add_sq(double &acc, C o) {
    acc = fma(double(o.x), double(o.x), fma(double(o.y), double(o.y), acc));
}

template <typename C>
__device__ __forceinline__ C *vec_ptr(const BArgs &A, int k, const BInst &I) {
    if (k == 0) return reinterpret_cast<C *>(A.v0[I.src]) + I.off0;
    return reinterpret_cast<C *>(A.slots + (size_t)(k - 1) * (size_t)A.slot_amps * sizeof(C)) + I.off;
}

__device__ __forceinline__ float2 ldcg(const float2 *p) { return __ldcg(p); }
__device__ __forceinline__ double2 ldcg(const double2 *p) { return __ldcg(p); }

__device__ __forceinline__ double2 shfl_c(double2 v, int m) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ float2 shfl_c(float2 v, int m) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// acc += (cr + i ci) * w
template <typename R, typename C>
__device__ __forceinline__ void cfma(R cr, R ci, C w, R &ar, R &ai) {
    ar = fma(cr, (R)w.x, fma(-ci, (R)w.y, ar));
    ai = fma(cr, (R)w.y, fma(ci, (R)w.x, ai));
}

// ---------------------------------------------------------------- partner-tile stages
// Each warp of the H v phase owns PSTAGES shared-memory stages of one tile (2^T amplitudes)
// in the kernel's dynamic shared memory.
constexpr int PSTAGES = 3;
template <typename C, int T>
__host__ __device__ constexpr size_t hpsi_stage_bytes() {
    return (size_t)BWARPS * PSTAGES * (sizeof(C) << T);
}
template <typename C, int T>
__device__ __forceinline__ C *hpsi_stages() {
    extern __shared__ __align__(16) unsigned char bsm[];
    return reinterpret_cast<C *>(bsm + (size_t)(threadIdx.x >> 5) * PSTAGES * (sizeof(C) << T));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------- phase A: H v_j on a tile
template <typename R, int T>
__device__ bool tile_hpsi(const BArgs &A, const BInst &I, int i, int t, int step, int j,
                          double sj) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    const int lane = threadIdx.x & 31;
    const int n = I.n;
    const long long base = (long long)(t - I.tile0) << T;
    const BCoef &cf = A.coef[I.coef0 + step];  // step: absolute
    const double *Ub = A.Ubits + (size_t)I.pidx * BMAXQ * BMAXQ;
    const C *u = vec_ptr<C>(A, j, I);
    C *out = vec_ptr<C>(A, j + 1, I);
    // per-tile diagonal terms: fields of the low bits including the high bits' pairs
    double fl = 0.0;  // lane p < T: effective field of low bit p
    if (lane < T) {
        fl = __ldg(&cf.field[lane]);
        for (int q = T; q < n; ++q)
            if ((base >> q) & 1) fl += __ldg(&Ub[lane * BMAXQ + q]);
    }
    double eh = 0.0;  // energy of the high bits (lane = high bit q - T)
    {
        const int q = T + lane;
        if (q < n && ((base >> q) & 1)) {
            eh = __ldg(&cf.field[q]);
            for (int r = q + 1; r < n; ++r)
                if ((base >> r) & 1) eh += __ldg(&Ub[q * BMAXQ + r]);
        }
        eh = warp_sum(eh);
    }
    double dlane = eh;  // + lane-bit fields
#pragma unroll
    for (int p = 0; p < 5; ++p) {
        const double f = __shfl_sync(0xffffffffu, fl, p);
        if ((lane >> p) & 1) dlane += f;
    }
    double freg[T - 5];
#pragma unroll
    for (int k = 0; k < T - 5; ++k) freg[k] = __shfl_sync(0xffffffffu, fl, 5 + k);
    const double *El = A.Elow + ((size_t)I.pidx << T);

    C v[AMP];
    R ar[AMP], ai[AMP];
#pragma unroll
    for (int a = 0; a < AMP; ++a) v[a] = ldcg(u + base + lane + 32 * a);
#pragma unroll
    for (int a = 0; a < AMP; ++a) {
        double d = dlane + __ldg(&El[lane + 32 * a]);
#pragma unroll
        for (int k = 0; k < T - 5; ++k)
            if ((a >> k) & 1) d += freg[k];
        const R dr = (R)d;
        ar[a] = dr * (R)v[a].x;
        ai[a] = dr * (R)v[a].y;
    }
    // coefficient of a flip of bit p for an amplitude whose bit p is `bit`
    auto coef = [&](int p, int bit, R &cr, R &ci) {
        if constexpr (sizeof(R) == 4) {
            cr = __ldg(&cf.fup_re[p]);
            ci = __ldg(&cf.fup_im[p]);
        } else {
            cr = __ldg(&cf.up_re[p]);
            ci = __ldg(&cf.up_im[p]);
        }
        if (!bit) ci = -ci;
    };
#pragma unroll
    for (int p = 0; p < 5; ++p) {  // lane bits
        R cr, ci;
        coef(p, (lane >> p) & 1, cr, ci);
#pragma unroll
        for (int a = 0; a < AMP; ++a) cfma(cr, ci, shfl_c(v[a], 1 << p), ar[a], ai[a]);
    }
#pragma unroll
    for (int k = 0; k < T - 5; ++k) {  // register bits
        R ucr, uci, dcr, dci;
        coef(5 + k, 1, ucr, uci);
        coef(5 + k, 0, dcr, dci);
#pragma unroll
        for (int a = 0; a < AMP; ++a) {
            const bool bit = (a >> k) & 1;
            cfma(bit ? ucr : dcr, bit ? uci : dci, v[a ^ (1 << k)], ar[a], ai[a]);
        }
    }
    // bits above the tile: the partner tiles, staged through the warp's shared-memory
    // stages by cp.async (PSTAGES partner tiles in flight and no registers held by the
    // copies), then read back in the lanes' amplitude layout
    C *stage0 = hpsi_stages<C, T>();
    auto issue = [&](int p, int st) {
        const char *src = reinterpret_cast<const char *>(u + (base ^ (1LL << p)));
        char *dst = reinterpret_cast<char *>(stage0 + ((size_t)st << T));
        constexpr int CP = (int)(sizeof(C) << T) / (16 * 32);  // 16-byte copies per lane
#pragma unroll
        for (int m = 0; m < CP; ++m) cp_async16(dst + 16 * (lane + 32 * m), src + 16 * (lane + 32 * m));
        cp_async_commit();
    };
    const int np = n - T;
    for (int q = 0; q < PSTAGES - 1; ++q) {
        if (q < np) issue(T + q, q);
        else cp_async_commit();  // empty groups keep the group count uniform
    }
    for (int q = 0; q < np; ++q) {
        const int qn = q + PSTAGES - 1;  // into the stage read in iteration q - 1
        if (qn < np) issue(T + qn, qn % PSTAGES);
        else cp_async_commit();
        cp_async_wait<PSTAGES - 1>();  // this lane's copies of partner tile q landed
        __syncwarp();                  // and every lane's
        const int p = T + q;
        R cr, ci;
        coef(p, (int)((base >> p) & 1), cr, ci);
        const C *w = stage0 + ((size_t)(q % PSTAGES) << T) + lane;
#pragma unroll
        for (int a = 0; a < AMP; ++a) cfma(cr, ci, w[32 * a], ar[a], ai[a]);
        __syncwarp();  // the stage is read before it is refilled
    }
    cp_async_wait<0>();
    // H v = sj * H stored_j; partials ||Hv||^2 and <v_j, Hv> = sj^2 <stored, H stored>
    R h2 = 0, dr = 0, di = 0;
#pragma unroll
    for (int a = 0; a < AMP; ++a) {
        const R hr = (R)sj * ar[a], hi = (R)sj * ai[a];
        out[base + lane + 32 * a] = cmake<C>(hr, hi);
        h2 = fma(hr, hr, fma(hi, hi, h2));
        dr = fma((R)v[a].x, hr, fma((R)v[a].y, hi, dr));
        di = fma((R)v[a].x, hi, fma(-(R)v[a].y, hr, di));
    }
    const double s2 = warp_sum((double)h2), s_r = warp_sum(sj * (double)dr),
                 s_i = warp_sum(sj * (double)di);
    if (lane == 0) {
        double *pa = A.partA + 4 * (size_t)t;
        pa[0] = s2;
        pa[1] = s_r;
        pa[2] = s_i;
    }
    return tile_done(A.cnt, A.partA, A.sumA, i, I.tile0, I.ntiles);
}

// ---------------------------------------------------------------- phase B: recurrence
template <typename R, int T>
__device__ bool tile_orth(const BArgs &A, const BInst &I, int i, int t, int j, double car,
                          double cai, double cb, double sj) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    const int lane = threadIdx.x & 31;
    const long long base = (long long)(t - I.tile0) << T;
    C *w = vec_ptr<C>(A, j + 1, I);
    const C *vj = vec_ptr<C>(A, j, I);
    const C *vp = j > 0 ? vec_ptr<C>(A, j - 1, I) : nullptr;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    constexpr int CH = AMP < 8 ? AMP : 8;  // amplitudes per lane with loads in flight
    for (int a0 = 0; a0 < AMP; a0 += CH) {
        C h[CH], q[CH], pv[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const long long x = base + lane + 32 * (a0 + c);
            h[c] = ldcg(w + x);
            q[c] = ldcg(vj + x);
            pv[c] = j > 0 ? ldcg(vp + x) : cmake<C>(0.0, 0.0);
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const long long x = base + lane + 32 * (a0 + c);
            double wr = double(h[c].x) - (car * double(q[c].x) - cai * double(q[c].y));
            double wi = double(h[c].y) - (car * double(q[c].y) + cai * double(q[c].x));
            wr -= cb * double(pv[c].x);
            wi -= cb * double(pv[c].y);
            const C o = cmake<C>(wr, wi);
            w[x] = o;
            const double orr = double(o.x), oi = double(o.y);
            const double vr = sj * double(q[c].x), vi = sj * double(q[c].y);
            acc0 += orr * orr + oi * oi;
            acc1 += vr * orr + vi * oi;
            acc2 += vr * oi - vi * orr;
        }
    }
    acc0 = warp_sum(acc0);
    acc1 = warp_sum(acc1);
    acc2 = warp_sum(acc2);
    if (lane == 0) {
        double *pb = A.partB + 4 * (size_t)t;
        pb[0] = acc0;
        pb[1] = acc1;
        pb[2] = acc2;
    }
    return tile_done(A.cnt + A.ninst, A.partB, A.sumB, i, I.tile0, I.ntiles);
}

template <typename R, int T>
__device__ bool tile_norm(const BArgs &A, const BInst &I, int i, int t) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    const int lane = threadIdx.x & 31;
    const long long base = (long long)(t - I.tile0) << T;
    const C *u = vec_ptr<C>(A, 0, I);
    double nrm = 0.0;
#pragma unroll 8
    for (int a = 0; a < AMP; ++a) add_sq(nrm, ldcg(u + base + lane + 32 * a));
    nrm = warp_sum(nrm);
    if (lane == 0) A.partN[4 * (size_t)t] = nrm;
    return tile_done(A.cnt + 2 * A.ninst, A.partN, A.sumN, i, I.tile0, I.ntiles);
}

__device__ __forceinline__ int ld_status(const KState *ks) {
    return *(volatile const int *)&ks->status;
}
__device__ __forceinline__ int ld_vol(const int *p) { return *(volatile const int *)p; }

// ---------------------------------------------------------------- phases
// Decision for iteration j of job i (krylov_exp.py:60-96) by warp 0 of the job's CTA
// (not inlined: its registers would otherwise crowd the tile loops, which then spill):
// convergence is tested from the job's hint (the previous step's count - 3); a first test
// that already converges tests the skipped iterations in order (krylov_decide), so each
// job stops where the reference would.
__device__ __noinline__ bool job_decide(const BArgs &A, int i, int j, int rstep) {
    const int lane = threadIdx.x & 31;
    KState *ks = A.ks + i;
    const double3 sb = ld_sum(A.sumB, i);
    const int hint = A.hint[i];
    const bool poll = (j + 1 >= hint) || (j + 1 >= A.maxdim);
    const bool first = poll && !A.polled[i];
    __syncwarp();
    if (lane == 0 && poll) A.polled[i] = 1;
    krylov_decide(ks, j, sb.x, sb.y, sb.z, A.inst[i].dt, A.exp_tol, A.norm_tol, poll, first,
                  A.maxdim);
    int st = KS_RUNNING;
    if (lane == 0) {
        st = ks->status;
        if (st == KS_RUNNING && j + 2 > A.capacity) {
            st = BS_CAPACITY;
            ks->status = st;
        }
        if (st == KS_NONFINITE || st == BS_CAPACITY) A.fail[i] = st;
        if (st != KS_RUNNING) {
            A.iters_out[(size_t)i * A.max_steps + rstep] = ks->iters;
            A.hint[i] = ks->iters > 3 ? ks->iters - 3 : 0;  // poll a little early
        }
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, st, 0) == KS_RUNNING;
}

// Phase bookkeeping keeps every job's tiles either all processed or all skipped in a
// phase (so the per-job tile counters complete): phase A_j runs a job if its step starts
// (j = 0) or if phase B of the previous round ran it (ranB), never from a status that the
// decisions of the same phase may be changing.

// Norms of every job's vector 0 (into sumN).
template <typename R, int T>
__device__ void norm_phase(const BArgs &A, unsigned ph) {
    for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
        const int i = inst_of_tile(A, t);
        tile_norm<R, T>(A, A.inst[i], i, t);
    }
}

// All Lanczos iterations of one step of every job (krylov_exp.py:49-106 per job).
// gstep: absolute step (coefficients, whether the job still has this step); rstep: the
// launch-relative step (iteration record).  Returns false if a barrier gave up.
template <typename R, int T>
__device__ bool krylov_rounds(const BArgs &A, int gstep, int rstep, unsigned &ph, int &round,
                              int &s_flag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = 0;; ++j) {
        // ---------------- phase A_j: decisions for j-1 (init at j = 0), tiles H v_j
        if (warp == 0) {
            for (int i = blockIdx.x; i < A.ninst; i += gridDim.x) {
                const BInst I = A.inst[i];
                KState *ks = A.ks + i;
                if (j == 0) {
                    if (lane == 0) {
                        const double s0 = sqrt(__ldcg(A.sumN + 4 * (size_t)i));
                        int st = KS_RUNNING;
                        const int f = ld_vol(&A.fail[i]);
                        if (f) st = f;
                        else if (gstep >= I.nsteps) st = BS_IDLE;
                        else if (!(isfinite(s0) && s0 > 0.0)) st = KS_NONFINITE;
                        ks->s0 = s0;
                        ks->shift = 0.0;
                        ks->scale[0] = 1.0 / s0;
                        ks->iters = 0;
                        ks->nvec = 0;
                        ks->kerr = 0;
                        ks->err = 0.0;
                        A.polled[i] = 0;
                        ks->status = st;
                        if (st == KS_NONFINITE) A.fail[i] = st;
                    }
                    __syncwarp();
                    continue;
                }
                if (ld_status(ks) != KS_RUNNING) continue;
                job_decide(A, i, j - 1, rstep);
            }
        }
        if (j < A.maxdim && j + 1 <= A.capacity) {
            for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
                const int i = inst_of_tile(A, t);
                const BInst I = A.inst[i];
                double sj;
                if (j == 0) {
                    if (gstep >= I.nsteps || ld_vol(&A.fail[i])) continue;
                    sj = 1.0 / sqrt(__ldcg(A.sumN + 4 * (size_t)i));
                } else {
                    if (ld_vol(&A.ranB[i]) != round) continue;  // B ran it last round
                    sj = 1.0 / sqrt(__ldcg(A.sumB + 4 * (size_t)i));
                }
                if (!isfinite(sj) || sj <= 0.0) continue;  // the same for all its tiles
                tile_hpsi<R, T>(A, I, i, t, gstep, j, sj);
            }
        }
        if (!grid_sync(A, ph)) return false;
        // does any job still iterate?
        if (warp == 0) {
            int any = 0;
            for (int i = lane; i < A.ninst; i += 32) any |= ld_status(A.ks + i) == KS_RUNNING;
            any = __any_sync(0xffffffffu, any);
            if (lane == 0) s_flag = any;
        }
        __syncthreads();
        if (!s_flag) return true;
        // ---------------- phase B_j: w = H v_j - a v_j - b v_{j-1}
        {
            int ci = -1;
            double car = 0, cai = 0, cb = 0, sj = 0;
            for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
                const int i = inst_of_tile(A, t);
                KState *ks = A.ks + i;
                if (ld_status(ks) != KS_RUNNING) continue;
                const BInst I = A.inst[i];
                if (i != ci) {
                    const double3 sa = ld_sum(A.sumA, i);
                    const double b = j > 0 ? __ldcg(&ks->r[j - 1]) : 0.0;
                    const double vr = j > 0 ? __ldcg(&ks->vv_re[j]) : 0.0;
                    const double vi = j > 0 ? __ldcg(&ks->vv_im[j]) : 0.0;
                    const double ar = sa.y - b * vr, ai = sa.z - b * vi;
                    sj = __ldcg(&ks->scale[j]);
                    const double sp = j > 0 ? __ldcg(&ks->scale[j - 1]) : 0.0;
                    car = ar * sj;
                    cai = ai * sj;
                    cb = b * sp;
                    ci = i;
                    // the warp of the job's first tile records T_H's column j (a warp meets a
                    // given job's first tile before any other of its tiles)
                    if (t == I.tile0 && lane == 0) {
                        ks->a_re[j] = ar;
                        ks->a_im[j] = ai;
                        ks->b_re[j] = b;
                        ks->b_im[j] = 0.0;
                        ks->hn[j] = sqrt(sa.x);
                        A.ranB[i] = round + 1;  // 0 (cleared at launch) = never
                    }
                }
                tile_orth<R, T>(A, I, i, t, j, car, cai, cb, sj);
            }
        }
        if (!grid_sync(A, ph)) return false;
        ++round;
    }
}

// Lane k % 32 holds coefficient block k / 32 (k < 128): f * c_k with f = s0 scale_k, or
// the conjugate of c_k (exp(+i dt H) from the same basis).
__device__ __forceinline__ void load_coefs(const KState *ks, int nvec, bool conj_c, double (&cr)[4],
                                           double (&cim)[4]) {
    const int lane = threadIdx.x & 31;
    const double s0 = __ldcg(&ks->s0);
#pragma unroll
    for (int blk = 0; blk < 4; ++blk) {
        const int k = lane + 32 * blk;
        double a = 0.0, b = 0.0;
        if (k < nvec) {
            const double f = s0 * __ldcg(&ks->scale[k]);
            a = f * __ldcg(&ks->c_re[k]);
            b = f * __ldcg(&ks->c_im[k]);
            if (conj_c) b = -b;
        }
        cr[blk] = a;
        cim[blk] = b;
    }
}

// out(tile) = sum_k coef_k stored_k(tile) over k < nvec; returns the tile's ||out||^2.
template <typename R, int T>
__device__ double tile_lincomb(const BArgs &A, const BInst &I, int t, int nvec, const double (&cr)[4],
                               const double (&cim)[4], typename cvec<R>::T *out) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    constexpr int CH = AMP < 4 ? AMP : 4;
    const int lane = threadIdx.x & 31;
    const long long base = (long long)(t - I.tile0) << T;
    double nrm = 0.0;
    for (int a0 = 0; a0 < AMP; a0 += CH) {
        double re[CH], im[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) re[c] = im[c] = 0.0;
        for (int k = 0; k < nvec; ++k) {
            const int src = k & 31, blk = k >> 5;
            const double vr = blk == 0 ? cr[0] : blk == 1 ? cr[1] : blk == 2 ? cr[2] : cr[3];
            const double vi = blk == 0 ? cim[0] : blk == 1 ? cim[1] : blk == 2 ? cim[2] : cim[3];
            const double c_r = __shfl_sync(0xffffffffu, vr, src);
            const double c_i = __shfl_sync(0xffffffffu, vi, src);
            const C *vk = vec_ptr<C>(A, k, I) + base + lane;
            C b[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) b[c] = ldcg(vk + 32 * (a0 + c));
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                re[c] += c_r * double(b[c].x) - c_i * double(b[c].y);
                im[c] += c_r * double(b[c].y) + c_i * double(b[c].x);
            }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const C o = cmake<C>(re[c], im[c]);
            out[base + lane + 32 * (a0 + c)] = o;
            add_sq(nrm, o);
        }
    }
    return warp_sum(nrm);
}

// psi' = s0 sum_k c_k v_k for every job that took the step (norm partials for the next
// step), optionally also into the history buffer.
template <typename R, int T>
__device__ void combine_phase(const BArgs &A, int rstep, unsigned ph) {
    typedef typename cvec<R>::T C;
    const int lane = threadIdx.x & 31;
    int ci = -1, nvec = 0;
    double cr[4], cim[4];
    const bool hist = A.hist && ((rstep + 1) % A.hist_every) == 0;
    for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
        const int i = inst_of_tile(A, t);
        const KState *ks = A.ks + i;
        const int st = ld_status(ks);
        const BInst I = A.inst[i];
        if (st != KS_CONVERGED && st != KS_HAPPY && st != KS_MAXDIM) {
            tile_norm<R, T>(A, I, i, t);  // idle or failed: keep the state, refresh its norm
            continue;
        }
        if (i != ci) {
            nvec = __ldcg(&ks->nvec);
            load_coefs(ks, nvec, false, cr, cim);
            ci = i;
        }
        C *out = vec_ptr<C>(A, 0, I);
        const double nrm = tile_lincomb<R, T>(A, I, t, nvec, cr, cim, out);
        if (hist) {  // copy the new tile into the history slot
            constexpr int AMP = 1 << (T - 5);
            const long long base = (long long)(t - I.tile0) << T;
            C *h = reinterpret_cast<C *>(A.hist) +
                   (size_t)((rstep + 1) / A.hist_every - 1) * (size_t)A.hist_stride + I.off0;
            __syncwarp();
            for (int a = 0; a < AMP; ++a) h[base + lane + 32 * a] = out[base + lane + 32 * a];
        }
        if (lane == 0) A.partN[4 * (size_t)t] = nrm;
        tile_done(A.cnt + 2 * A.ninst, A.partN, A.sumN, i, I.tile0, I.ntiles);
    }
}

// ---------------------------------------------------------------- forward kernel
template <typename R, int T, int MINB>
__global__ void __launch_bounds__(BWARPS * 32, MINB) k_batch(const BArgs A) {
    __shared__ int s_flag;
    const int lane = threadIdx.x & 31;
    unsigned ph = 0;
    int round = 0;  // phase-B rounds so far (the same in every CTA)
    norm_phase<R, T>(A, ph);
    if (!grid_sync(A, ph)) return;
    for (int step = 0; step < A.run_steps; ++step) {
        if (!krylov_rounds<R, T>(A, A.first_step + step, step, ph, round, s_flag)) return;
        combine_phase<R, T>(A, step, ph);
        if (!grid_sync(A, ph)) return;
    }
    if (threadIdx.x < 32) {  // final statuses
        for (int i = blockIdx.x * 32 + lane; i < A.ninst; i += gridDim.x * 32) {
            const int st = ld_status(A.ks + i);
            const int f = A.fail[i];
            A.status_out[i] = f ? f : (st == BS_IDLE ? KS_CONVERGED : st);
        }
    }
}

// ---------------------------------------------------------------- the phase engine
// Every job runs its own sequence of phases: the norm of its vector 0, then per step
// A_0, B_0, A_1, B_1, ..., B_e (e: the decision that ends the step) and the combination
// C; then the next step's A_0, and so on, until the job is idle.  A job's state word holds
// the number of phases it completed and the code of its next phase; the warp that
// completes a phase (the last of its tiles) takes the phase's decision and publishes the
// next code.
enum { PK_NORM = 0, PK_A = 1, PK_B = 2, PK_C = 3, PK_IDLE = 4 };
constexpr int BCHUNK = 4;  // tiles a warp takes per visit

__device__ __forceinline__ unsigned pcode(int kind, int rstep, int j) {
    return (unsigned)kind << 24 | ((unsigned)rstep & 0xffffu) << 8 | (unsigned)j;
}
__device__ __forceinline__ int pkind(unsigned c) { return (int)(c >> 24); }
__device__ __forceinline__ int prstep(unsigned c) { return (int)((c >> 8) & 0xffffu); }
__device__ __forceinline__ int pj(unsigned c) { return (int)(c & 0xffu); }

__device__ __forceinline__ unsigned long long ld_acq64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_rel64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_vol_u(const unsigned *p) { return *(volatile const unsigned *)p; }

// Warp-collective bounded wait until job i completed `phi` phases or is idle; the state
// word in w.  False once the wait ran out (it records EMUSV_TIMEOUT) or another warp
// recorded an error.
__device__ bool wait_phase(const BArgs &A, int i, unsigned phi, unsigned long long &w) {
    unsigned long long v = 0;
    int ok = 1;
    if ((threadIdx.x & 31) == 0) {
        v = ld_acq64(&A.jst[i]);
        if ((unsigned)(v >> 32) < phi && pkind((unsigned)v) != PK_IDLE) {
            const long long t0 = clock64();
            for (int polls = 1;; ++polls) {
                __nanosleep(64);
                v = ld_acq64(&A.jst[i]);
                if ((unsigned)(v >> 32) >= phi || pkind((unsigned)v) == PK_IDLE) break;
                if ((polls & 15) == 0 && (clock64() - t0 > A.bar_limit || ld_vol(&A.ctl->err))) {
                    atomicCAS(&A.ctl->err, 0, EMUSV_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
    }
    __syncwarp();
    w = __shfl_sync(0xffffffffu, v, 0);
    return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// Phase phi of job i is complete: publish phase phi + 1 with code c, then open its tiles
// (lane 0 of the completing warp; its tiles' writes and the phase's sums precede both
// releases, and a warp whose take lands on the new phase finds its code published).  The
// failure-path test switch withholds job 0's first publication: no warp then finds work
// for job 0 again, and every warp's starvation limit runs out.
__device__ void publish(const BArgs &A, int i, unsigned phi, unsigned c) {
    if ((threadIdx.x & 31) == 0 && !(A.test_skip_arrival && i == 0 && phi == 0)) {
        __threadfence();
        st_rel64(&A.jst[i], (unsigned long long)(phi + 1) << 32 | c);
        st_rel64(&A.take[i], (unsigned long long)(phi + 1) << 32);  // the new phase's tiles
    }
    __syncwarp();
}

// The job has no phase left in this launch: its final status, then the idle count.
__device__ void job_idle(const BArgs &A, int i, unsigned phi) {
    if ((threadIdx.x & 31) == 0) {
        const int st = ld_status(A.ks + i);
        const int f = ld_vol(&A.fail[i]);
        A.status_out[i] = f ? f : (st == BS_IDLE ? KS_CONVERGED : st);
    }
    publish(A, i, phi, pcode(PK_IDLE, 0, 0));
    if ((threadIdx.x & 31) == 0) {
        __threadfence();
        atomicAdd(&A.ctl->idle, 1u);
    }
    __syncwarp();
}

// Start of step gstep for job i, from the norm of its vector 0 in sumN: the step's
// Krylov state; true if the job iterates (false: idle, failed or a non-finite norm).
__device__ bool job_init(const BArgs &A, int i, int gstep) {
    int st = KS_RUNNING;
    if ((threadIdx.x & 31) == 0) {
        KState *ks = A.ks + i;
        const double s0 = sqrt(__ldcg(A.sumN + 4 * (size_t)i));
        const int f = ld_vol(&A.fail[i]);
        if (f) st = f;
        else if (gstep >= A.inst[i].nsteps) st = BS_IDLE;
        else if (!(isfinite(s0) && s0 > 0.0)) st = KS_NONFINITE;
        ks->s0 = s0;
        ks->shift = 0.0;
        ks->scale[0] = 1.0 / s0;
        ks->iters = 0;
        ks->nvec = 0;
        ks->kerr = 0;
        ks->err = 0.0;
        A.polled[i] = 0;
        ks->status = st;
        if (st == KS_NONFINITE) A.fail[i] = st;
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, st, 0) == KS_RUNNING;
}

// Combination tile of step rstep: psi' = s0 sum_k c_k v_k in place for a job whose step
// ended with a result (optionally also into the history buffer), else (failed) the norm
// of the kept state; the tile's norm partial.  True for the warp that completes the job.
template <typename R, int T>
__device__ bool tile_combine(const BArgs &A, const BInst &I, int i, int t, int rstep) {
    typedef typename cvec<R>::T C;
    const int lane = threadIdx.x & 31;
    const KState *ks = A.ks + i;
    const int st = ld_status(ks);
    if (st != KS_CONVERGED && st != KS_HAPPY && st != KS_MAXDIM) return tile_norm<R, T>(A, I, i, t);
    const int nvec = __ldcg(&ks->nvec);
    double cr[4], cim[4];
    load_coefs(ks, nvec, false, cr, cim);
    C *out = vec_ptr<C>(A, 0, I);
    const double nrm = tile_lincomb<R, T>(A, I, t, nvec, cr, cim, out);
    if (A.hist && ((rstep + 1) % A.hist_every) == 0) {  // the new tile into the history slot
        constexpr int AMP = 1 << (T - 5);
        const long long base = (long long)(t - I.tile0) << T;
        C *h = reinterpret_cast<C *>(A.hist) +
               (size_t)((rstep + 1) / A.hist_every - 1) * (size_t)A.hist_stride + I.off0;
        __syncwarp();
        for (int a = 0; a < AMP; ++a) h[base + lane + 32 * a] = out[base + lane + 32 * a];
    }
    if (lane == 0) A.partN[4 * (size_t)t] = nrm;
    return tile_done(A.cnt + 2 * A.ninst, A.partN, A.sumN, i, I.tile0, I.ntiles);
}

// The phase engine (krylov_exp.py:23-131 per job and step, every job of the batch in one
// persistent launch).  Warps never wait for a particular phase: a cursor over the tiles
// of all jobs picks the jobs to visit (so a job is visited in proportion to its size),
// and the warp takes up to BCHUNK tiles of each visited job's current phase from the
// job's take counter, (phase << 32) | tiles taken.  A job whose current phase has no tile
// left (its last tiles are still running, or it is idle) is passed over; an idle job's
// tiles are jumped over (atomicMax on the cursor).  The warp that completes a phase (the
// last of its tiles) takes the phase's decision, publishes the next phase's code, then
// resets the take counter.  The launch ends when every job is idle.
enum { V_WORK = 0, V_BUSY = 1, V_IDLE = 2, V_STOP = 3 };

// One visit of job i (cursor sweep `sweep`): take up to BCHUNK tiles of its current
// phase and run them.  cphi / c cache the phase's scalars (A: sj; B: car, cai, cb, sjb)
// for the warp's current job.
template <typename R, int T>
__device__ int visit_job(const BArgs &A, int i, const BInst &I, unsigned long long sweep,
                         unsigned &cphi, double (&c)[4]) {
    const int lane = threadIdx.x & 31;
    unsigned long long w = 0, tk = 0;
    if (lane == 0) {  // the state and the take in one round trip (a take of an idle job is
                      // never used)
        tk = atomicAdd(&A.take[i], (unsigned long long)BCHUNK);
        w = ld_acq64(&A.jst[i]);
    }
    w = __shfl_sync(0xffffffffu, w, 0);
    tk = __shfl_sync(0xffffffffu, tk, 0);
    unsigned code = (unsigned)w, phi = (unsigned)(w >> 32);
    if (pkind(code) == PK_IDLE) {
        if (lane == 0)
            atomicMax(&A.ctl->item, sweep * (unsigned long long)A.total_tiles +
                                        (unsigned long long)(I.tile0 + I.ntiles));
        return V_IDLE;
    }
    const unsigned phit = (unsigned)(tk >> 32), n0 = (unsigned)tk;
    if (phit != phi || n0 >= (unsigned)I.ntiles) {
        if (!(phit > phi && n0 < (unsigned)I.ntiles)) return V_BUSY;  // nothing free now
        // the take counter was already reset for a later phase: these tiles are that
        // phase's, whose code was published just before the reset
        if (!wait_phase(A, i, phit, w)) return V_STOP;
        code = (unsigned)w;
        phi = phit;
        if (pkind(code) == PK_IDLE) return V_IDLE;  // the job went idle: no tiles
        if ((unsigned)(w >> 32) != phit) {  // cannot happen
            if (lane == 0) atomicCAS(&A.ctl->err, 0, EMUSV_BAD_ARGUMENT);
            return V_STOP;
        }
    }
    const int kind = pkind(code), j = pj(code), rstep = prstep(code);
    KState *ks = A.ks + i;
    if (phi != cphi) {  // the phase's scalars
        cphi = phi;
        if (kind == PK_A) {
            const double sn = __ldcg((j == 0 ? A.sumN : A.sumB) + 4 * (size_t)i);
            c[0] = 1.0 / sqrt(sn);
            // ||w_{j-1}|| zero or not finite: the decision of j - 1 ended the step unless
            // a tolerance of zero let it go on; the tiles run on zeros
            if (!isfinite(c[0]) || c[0] <= 0.0) c[0] = 0.0;
        } else if (kind == PK_B) {
            const double3 sa = ld_sum(A.sumA, i);
            const double b = j > 0 ? __ldcg(&ks->r[j - 1]) : 0.0;
            const double vr = j > 0 ? __ldcg(&ks->vv_re[j]) : 0.0;
            const double vi = j > 0 ? __ldcg(&ks->vv_im[j]) : 0.0;
            const double ar = sa.y - b * vr, ai = sa.z - b * vi;
            c[3] = __ldcg(&ks->scale[j]);
            const double sp = j > 0 ? __ldcg(&ks->scale[j - 1]) : 0.0;
            c[0] = ar * c[3];
            c[1] = ai * c[3];
            c[2] = b * sp;
            // the warp that took the job's first tile records T_H's column j (read by the
            // decision, which follows every tile of the phase)
            if (n0 == 0 && lane == 0) {
                ks->a_re[j] = ar;
                ks->a_im[j] = ai;
                ks->b_re[j] = b;
                ks->b_im[j] = 0.0;
                ks->hn[j] = sqrt(sa.x);
            }
            __syncwarp();
        }
    }
    const int n1 = min((int)n0 + BCHUNK, I.ntiles);
    for (int t = I.tile0 + (int)n0; t < I.tile0 + n1; ++t) {
        if (kind == PK_NORM) {
            if (tile_norm<R, T>(A, I, i, t)) {
                if (job_init(A, i, A.first_step + rstep)) publish(A, i, phi, pcode(PK_A, rstep, 0));
                else job_idle(A, i, phi);
            }
        } else if (kind == PK_A) {  // H v_j
            if (tile_hpsi<R, T>(A, I, i, t, A.first_step + rstep, j, c[0]))
                publish(A, i, phi, pcode(PK_B, rstep, j));
        } else if (kind == PK_B) {  // w = H v_j - a v_j - b v_{j-1}, then the decision
            if (tile_orth<R, T>(A, I, i, t, j, c[0], c[1], c[2], c[3])) {
                if (job_decide(A, i, j, rstep)) publish(A, i, phi, pcode(PK_A, rstep, j + 1));
                else if (A.combine) publish(A, i, phi, pcode(PK_C, rstep, 0));
                else job_idle(A, i, phi);
            }
        } else {  // PK_C: the combination, then the next step
            if (tile_combine<R, T>(A, I, i, t, rstep)) {
                if (rstep + 1 < A.run_steps && job_init(A, i, A.first_step + rstep + 1))
                    publish(A, i, phi, pcode(PK_A, rstep + 1, 0));
                else job_idle(A, i, phi);
            }
        }
    }
    return V_WORK;
}

template <typename R, int T>
__device__ void run_jobs(const BArgs &A) {
    const int lane = threadIdx.x & 31;
    BCtl *ctl = A.ctl;
    const unsigned long long total = (unsigned long long)A.total_tiles;
    int ci = -1;                  // the warp's current job, its BInst and phase scalars
    BInst I = {};
    unsigned cphi = 0xffffffffu;
    double c[4] = {0.0, 0.0, 0.0, 0.0};
    unsigned long long qn = 0;    // the next visit, taken while this one runs
    if (lane == 0) qn = atomicAdd(&ctl->item, (unsigned long long)BCHUNK);
    // a warp that finds no tile to run for A.bar_limit clock cycles gives up (a phase
    // completion that never comes): EMUSV_TIMEOUT, and every warp returns
    long long idle_since = -1;
    for (;;) {
        const unsigned long long q0 = __shfl_sync(0xffffffffu, qn, 0);
        if (lane == 0) qn = atomicAdd(&ctl->item, (unsigned long long)BCHUNK);
        const unsigned long long sweep = q0 / total;
        const int t0 = (int)(q0 - sweep * total);
        // every job whose tiles meet [t0, t0 + BCHUNK) (a job smaller than a visit is
        // never passed over)
        for (int tj = t0;; tj = I.tile0 + I.ntiles) {
            if (ci < 0 || tj < I.tile0 || tj >= I.tile0 + I.ntiles) {
                const int ni = inst_of_tile(A, tj);
                if (ni != ci) cphi = 0xffffffffu;
                ci = ni;
                I = A.inst[ci];
            }
            const int v = visit_job<R, T>(A, ci, I, sweep, cphi, c);
            if (v == V_STOP) return;
            if (v == V_WORK) {
                idle_since = -1;
            } else {
                if (v == V_IDLE && ld_vol_u(&ctl->idle) >= (unsigned)A.ninst) return;
                const long long now = clock64();
                if (idle_since < 0) idle_since = now;
                if (now - idle_since > A.bar_limit) {
                    if (lane == 0) atomicCAS(&ctl->err, 0, EMUSV_TIMEOUT);
                    return;
                }
                if (ld_vol(&ctl->err)) return;
                if (v == V_BUSY) __nanosleep(128);
            }
            if (I.tile0 + I.ntiles >= t0 + BCHUNK || ci + 1 >= A.ninst) break;
        }
    }
}

// The forward steps by the phase engine (each job at its own pace, emusv_batch_set_engine
// 1): the choice for batches whose registers need similar iteration counts, where the
// lock-step rounds above spend little on waiting but the phases' finer-grained overlap wins.
template <typename R, int T, int MINB>
__global__ void __launch_bounds__(BWARPS * 32, MINB) k_batch_phase(const BArgs A) {
    run_jobs<R, T>(A);
}

// ---------------------------------------------------------------- adjoint kernel
// Basis size of a finished Lanczos job (double_krylov.py:100-113).
__device__ __forceinline__ int basis_size(const KState *ks) {
    const int st = ld_status(ks);
    const int it = __ldcg(&ks->iters);
    return st == KS_HAPPY ? it : it + 1;
}

__device__ __forceinline__ bool job_ok(const KState *ks) {
    const int st = ld_status(ks);
    return st == KS_CONVERGED || st == KS_HAPPY;
}

// dS column `col` of instance i: y = exp(B) e_{ms+col} for the block matrix
// B = [[A_s, e0 e0^T], [0, A_g]] (A = -i dt T of each basis, the coupling taken as 1:
// double_krylov.py:54-57 scales it by |state||grad| afterwards), rows 0..ms-1 of y.
// One warp per column, Chebyshev form (the spectrum of B is that of the two blocks).
__device__ __forceinline__ void block_row(const KState *ks, int kk, int m, double dt, double2 &d,
                                          double2 &l, double2 &u, double &td, double &tr) {
    const int jj = __ldcg(&ks->iters) - 1;  // last Lanczos column; row jj+1 is the appended one
    d = l = u = make_double2(0.0, 0.0);
    td = tr = 0.0;
    if (kk <= jj) {
        const double ar = __ldcg(&ks->a_re[kk]) + __ldcg(&ks->shift), ai = __ldcg(&ks->a_im[kk]);
        d = make_double2(dt * ai, -dt * ar);
        td = ar;
        tr = fabs(ai);
    }
    if (kk >= 1) {
        const double r = __ldcg(&ks->r[kk - 1]);
        l = make_double2(0.0, -dt * r);
        tr += fabs(r);
    }
    if (kk + 1 <= jj && kk + 1 < m) {
        const double br = __ldcg(&ks->b_re[kk + 1]), bi = __ldcg(&ks->b_im[kk + 1]);
        u = make_double2(dt * bi, -dt * br);
        tr += hypot(br, bi);
    }
}

constexpr int DS_NE = 8;  // block matrices up to 256 rows

__global__ void __launch_bounds__(BWARPS * 32) k_batch_dS(const BArgs A, const BAdj D) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.y, col = blockIdx.x * BWARPS + warp;
    const KState *kss = A.ks + 2 * i, *ksg = A.ks + 2 * i + 1;
    if (!job_ok(kss) || !job_ok(ksg)) return;
    const int ms = basis_size(kss), mg = basis_size(ksg), M = ms + mg;
    if (col >= mg || M > 32 * DS_NE || ms > D.mmax || mg > D.mmax) return;
    const double dt = A.inst[2 * i].dt;
    double2 d[DS_NE], l[DS_NE], u[DS_NE], y[DS_NE];
    double td[DS_NE], tr[DS_NE];
#pragma unroll
    for (int e = 0; e < DS_NE; ++e) {
        const int k = lane * DS_NE + e;
        d[e] = l[e] = u[e] = make_double2(0.0, 0.0);
        td[e] = tr[e] = 0.0;
        if (k < ms) block_row(kss, k, ms, dt, d[e], l[e], u[e], td[e], tr[e]);
        else if (k < M) block_row(ksg, k - ms, mg, dt, d[e], l[e], u[e], td[e], tr[e]);
        if (k == 0) tr[e] += 1.0 / fabs(dt);  // the coupling entry 1 in T units
    }
    cheb_expm<DS_NE>(d, l, u, ms, make_double2(1.0, 0.0), ms + col, dt, td, tr, M, y);
    double2 *out = D.dS + (size_t)i * D.mmax * D.mmax;
#pragma unroll
    for (int e = 0; e < DS_NE; ++e) {
        const int r = lane * DS_NE + e;
        if (r < ms) out[r * D.mmax + col] = y[e];
    }
}

// The adjoint's Krylov bases of one step (the state's and the incoming gradient's per
// instance): the phase engine without the combination (the launch sets first_step = the
// step, run_steps = 1, combine = 0).  Each job runs norm, A_0, B_0, ... to its ending
// decision at its own pace, with no round in which a finished job is passed over.
template <typename R, int T, int MINB>
__global__ void __launch_bounds__(BWARPS * 32, MINB) k_batch_adj_rounds(const BArgs A, const BAdj D) {
    run_jobs<R, T>(A);
}

template <typename R, int T, int MINB>
__global__ void __launch_bounds__(BWARPS * 32, MINB) k_batch_adj_post(const BArgs A, const BAdj D) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    const int lane = threadIdx.x & 31;
    unsigned ph = 0;

    // ---------------- E_k = sum_r dS[r][k] v^s_r (state tiles); g_out (gradient tiles)
    for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
        const int J = inst_of_tile(A, t), i = J >> 1;
        const KState *kss = A.ks + 2 * i, *ksg = A.ks + 2 * i + 1;
        const BInst I = A.inst[J];
        const long long base = (long long)(t - I.tile0) << T;
        if (!job_ok(kss) || !job_ok(ksg)) {
            if ((J & 1) && __ldcg(&ksg->s0) == 0.0) {  // exp(+i dt H) 0 = 0
                C *o = reinterpret_cast<C *>(D.gout) + I.off0 + base + lane;
                for (int a = 0; a < AMP; ++a) o[32 * a] = cmake<C>(0.0, 0.0);
            }
            continue;
        }
        const int ms = basis_size(kss), mg = basis_size(ksg);
        if (J & 1) {  // state gradient from the gradient basis
            double cr[4], cim[4];
            const int nvec = __ldcg(&ksg->nvec);
            load_coefs(ksg, nvec, true, cr, cim);
            tile_lincomb<R, T>(A, I, t, nvec, cr, cim, reinterpret_cast<C *>(D.gout) + I.off0);
            continue;
        }
        const double2 *dS = D.dS + (size_t)i * D.mmax * D.mmax;
        // KC outputs per pass over the state basis: every loaded amplitude feeds KC MACs
        constexpr int KC = 16;
        for (int k0 = 0; k0 < mg; k0 += KC) {
            const int kn = mg - k0 < KC ? mg - k0 : KC;
            for (int a = 0; a < AMP; ++a) {
                double er[KC], ei[KC];
#pragma unroll
                for (int kk = 0; kk < KC; ++kk) er[kk] = ei[kk] = 0.0;
                const long long x = base + lane + 32 * a;
#pragma unroll 4
                for (int r = 0; r < ms; ++r) {
                    const double sc = __ldcg(&kss->scale[r]);
                    const C v = ldcg(vec_ptr<C>(A, r, I) + x);
                    const double vx = sc * double(v.x), vy = sc * double(v.y);
                    const double2 *drow = dS + (size_t)r * D.mmax + k0;
#pragma unroll
                    for (int kk = 0; kk < KC; ++kk) {
                        if (kk < kn) {
                            const double2 d = drow[kk];
                            er[kk] += d.x * vx - d.y * vy;
                            ei[kk] += d.x * vy + d.y * vx;
                        }
                    }
                }
#pragma unroll
                for (int kk = 0; kk < KC; ++kk) {
                    if (kk < kn) {
                        C *Ek = reinterpret_cast<C *>(D.E + (size_t)(k0 + kk) * D.inst_amps * sizeof(C)) + I.off0;
                        Ek[x] = cmake<C>(er[kk], ei[kk]);
                    }
                }
            }
        }
    }
    if (!grid_sync(A, ph)) return;

    // ---------------- contractions over state tiles; the last tile of an instance turns
    // its sums into the step's gradients (torch.py:324-353)
    for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
        const int J = inst_of_tile(A, t), i = J >> 1;
        if (J & 1) continue;
        const KState *kss = A.ks + 2 * i, *ksg = A.ks + 2 * i + 1;
        const BInst I = A.inst[J], IG = A.inst[J + 1];
        const int n = I.n;
        const long long base = (long long)(t - I.tile0) << T;
        double acc[6] = {0, 0, 0, 0, 0, 0};  // lane p: T, U, S sums of bit p
        const bool ok = job_ok(kss) && job_ok(ksg);
        if (ok) {
            const int mg = basis_size(ksg);
            double rr[AMP], ri[AMP];
#pragma unroll
            for (int a = 0; a < AMP; ++a) rr[a] = ri[a] = 0.0;
            for (int k = 0; k < mg; ++k) {
                const double gs = __ldcg(&ksg->scale[k]);
                const C *gk = vec_ptr<C>(A, k, IG) + base + lane;
                const C *Ek = reinterpret_cast<const C *>(D.E + (size_t)k * D.inst_amps * sizeof(C)) + I.off0;
                double gr[AMP], gi[AMP];
                C e[AMP];
#pragma unroll
                for (int a = 0; a < AMP; ++a) {
                    const C g = ldcg(gk + 32 * a);
                    gr[a] = gs * double(g.x);
                    gi[a] = -gs * double(g.y);  // conj
                    e[a] = ldcg(Ek + base + lane + 32 * a);
                    rr[a] += gr[a] * double(e[a].x) - gi[a] * double(e[a].y);
                    ri[a] += gr[a] * double(e[a].y) + gi[a] * double(e[a].x);
                }
                // per bit p: sum conj(G) E(x^p) and its part with x_p = 1; the partner is
                // in another lane (p < 5), another register (p < T, compile-time index so
                // e[] stays in registers) or another tile (p >= T)
                auto bit_sums = [&](int p, double tr, double ti, double ur, double ui) {
                    tr = warp_sum(tr);
                    ti = warp_sum(ti);
                    ur = warp_sum(ur);
                    ui = warp_sum(ui);
                    if (lane == p) {
                        acc[0] += tr;
                        acc[1] += ti;
                        acc[2] += ur;
                        acc[3] += ui;
                    }
                };
                auto term = [&](int a, const C &w, bool bit, double &tr, double &ti, double &ur,
                                double &ui) {
                    const double pr = gr[a] * double(w.x) - gi[a] * double(w.y);
                    const double pi = gr[a] * double(w.y) + gi[a] * double(w.x);
                    tr += pr;
                    ti += pi;
                    if (bit) {
                        ur += pr;
                        ui += pi;
                    }
                };
                if constexpr (AMP <= 16 && MINB == 1) {  // unrolled: e[] stays in registers
#pragma unroll
                    for (int p = 0; p < 5; ++p) {
                        double tr = 0, ti = 0, ur = 0, ui = 0;
#pragma unroll
                        for (int a = 0; a < AMP; ++a)
                            term(a, shfl_c(e[a], 1 << p), (lane >> p) & 1, tr, ti, ur, ui);
                        bit_sums(p, tr, ti, ur, ui);
                    }
#pragma unroll
                    for (int p = 5; p < T; ++p) {
                        double tr = 0, ti = 0, ur = 0, ui = 0;
#pragma unroll
                        for (int a = 0; a < AMP; ++a)
                            term(a, e[a ^ (1 << (p - 5))], (a >> (p - 5)) & 1, tr, ti, ur, ui);
                        bit_sums(p, tr, ti, ur, ui);
                    }
                } else {  // the unrolled form would not fit the register budget
                    for (int p = 0; p < T; ++p) {
                        double tr = 0, ti = 0, ur = 0, ui = 0;
#pragma unroll
                        for (int a = 0; a < AMP; ++a) {
                            if (p < 5) term(a, shfl_c(e[a], 1 << p), (lane >> p) & 1, tr, ti, ur, ui);
                            else term(a, e[a ^ (1 << (p - 5))], (a >> (p - 5)) & 1, tr, ti, ur, ui);
                        }
                        bit_sums(p, tr, ti, ur, ui);
                    }
                }
                for (int p = T; p < n; ++p) {
                    double tr = 0, ti = 0, ur = 0, ui = 0;
                    const bool bit = (base >> p) & 1;
#pragma unroll
                    for (int a = 0; a < AMP; ++a)
                        term(a, ldcg(Ek + (base ^ (1LL << p)) + lane + 32 * a), bit, tr, ti, ur, ui);
                    bit_sums(p, tr, ti, ur, ui);
                }
            }
            for (int p = 0; p < n; ++p) {  // S_pp = sum over x with bit p of rho(x)
                double sr = 0, si = 0;
#pragma unroll
                for (int a = 0; a < AMP; ++a) {
                    const long long x = base + lane + 32 * a;
                    if ((x >> p) & 1) {
                        sr += rr[a];
                        si += ri[a];
                    }
                }
                sr = warp_sum(sr);
                si = warp_sum(si);
                if (lane == p) {
                    acc[4] += sr;
                    acc[5] += si;
                }
            }
        }
        double *pc = D.partC + (size_t)t * NCP;
        if (lane < n)
#pragma unroll
            for (int c = 0; c < 6; ++c) pc[6 * lane + c] = acc[c];
        // count the tile; the instance's last tile finalises
        unsigned old = 0;
        if (lane == 0) {
            __threadfence();
            old = atomicAdd(&D.cntC[i], 1u);
        }
        old = __shfl_sync(0xffffffffu, old, 0);
        if (old != (unsigned)I.ntiles - 1) continue;
        __threadfence();
        if (lane == 0) D.cntC[i] = 0;
        double *g = D.grads + (size_t)i * 3 * BMAXQ;
        if (!ok) {  // a zero gradient (or a failed basis): no parameter gradient
            const bool zero = __ldcg(&ksg->s0) == 0.0;
            if (lane < n) g[lane] = g[BMAXQ + lane] = g[2 * BMAXQ + lane] = 0.0;
            if (lane == 0) {
                int e = EMUSV_OK;
                if (!zero) {
                    e = EMUSV_NONFINITE;
                    for (const KState *k2 : {kss, ksg}) {
                        const int st = ld_status(k2);
                        if (st == KS_MAXDIM) e = EMUSV_NOT_CONVERGED;  // double_krylov.py:107-110
                        if (st == BS_CAPACITY) e = EMUSV_WORKSPACE_TOO_SMALL;
                    }
                }
                D.astatus[i] = e;
            }
            continue;
        }
        double sum[6] = {0, 0, 0, 0, 0, 0};  // lane p: instance sums of bit p
        if (lane < n)
            for (int tt = 0; tt < I.ntiles; ++tt)
#pragma unroll
                for (int c = 0; c < 6; ++c) sum[c] += __ldcg(D.partC + (size_t)(I.tile0 + tt) * NCP + 6 * lane + c);
        if (lane < n) {
            const int p = lane, q = n - 1 - p;  // bit p is qubit q
            const BCoef &cf = A.coef[I.coef0 + D.step];
            const double dt = I.dt, c = __ldcg(&kss->s0) * __ldcg(&ksg->s0);
            const double Ure = sum[2], Uim = sum[3], Dre = sum[0] - sum[2], Dim = sum[1] - sum[3];
            // Re(-i dt c <.>) for a flip with coefficient a on |1><0| and conj(a) on |0><1|
            auto flip = [&](double ar, double ai) {
                const double im = ar * Uim + ai * Ure + ar * Dim - ai * Dre;
                return dt * c * im;
            };
            const double om = cf.om[p], phv = cf.ph[p];
            g[q] = flip(0.5 * cos(phv), 0.5 * sin(phv));                     // DHDOmegaSparse
            g[BMAXQ + q] = dt * c * (-sum[5]);                              // DHDDeltaSparse: -n
            g[2 * BMAXQ + q] = flip(-0.5 * om * sin(phv), 0.5 * om * cos(phv));  // DHDPhiSparse
        }
        if (lane == 0) D.astatus[i] = EMUSV_OK;
    }
}

// ---------------------------------------------------------------- host side
static size_t al256(size_t v) { return (v + 255) / 256 * 256; }

// Workspace layout.  Forward: one job per instance.  Adjoint: jobs 2i (state) and 2i+1
// (gradient) per instance, plus the adjoint's own arrays.
struct BLayout {
    size_t args, ctl, ints, inst, coef, ubits, elow, ks, sums, iters, partA, partB, partN, slots;
    size_t dS, escr, E, partC, total;
    int njobs, total_tiles, coef_count, max_steps, mmax, escr_warps;
    long long inst_amps, slot_amps;
};


static bool layout(int ninst, const int *nq, const int *nsteps, int es, int T, int capacity,
                   bool adjoint, BLayout *L) {
    long long amps = 0;
    int tiles = 0, coefs = 0, max_steps = 0;
    for (int i = 0; i < ninst; ++i) {
        if (nq[i] < T || nq[i] > BMAXQ || nsteps[i] < 0) return false;
        amps += 1LL << nq[i];
        tiles += 1 << (nq[i] - T);
        coefs += nsteps[i];
        max_steps = nsteps[i] > max_steps ? nsteps[i] : max_steps;
    }
    const int nj = adjoint ? 2 * ninst : ninst;
    L->njobs = nj;
    L->inst_amps = amps;
    L->slot_amps = adjoint ? 2 * amps : amps;
    L->total_tiles = adjoint ? 2 * tiles : tiles;
    L->coef_count = coefs;
    L->max_steps = adjoint ? 1 : max_steps;
    L->mmax = capacity + 1;
    size_t off = 0;
    auto take = [&](size_t b) { const size_t o = off; off += al256(b); return o; };
    L->args = take(sizeof(BArgs));
    // control block and integer flags, contiguous so that a launch clears them in one go:
    // per job the phase engine's state and take words (two ints each, 8-byte aligned after
    // the 32-byte control block), hint, polled, fail, status, ranB, cnt[3], then the
    // adjoint's counters
    L->ctl = off;
    off += sizeof(BCtl);
    L->ints = off;
    off += sizeof(int) * (12 * (size_t)nj + ninst);
    off = al256(off);
    L->inst = take(sizeof(BInst) * nj);
    L->coef = take(sizeof(BCoef) * (coefs > 0 ? coefs : 1));
    L->ubits = take(sizeof(double) * BMAXQ * BMAXQ * ninst);
    L->elow = take(sizeof(double) * ((size_t)ninst << T));
    L->ks = take(sizeof(KState) * nj);
    L->sums = take(sizeof(double) * 12 * nj);
    L->iters = take(sizeof(int) * (size_t)nj * (L->max_steps > 0 ? L->max_steps : 1));
    L->partA = take(sizeof(double) * 4 * L->total_tiles);
    L->partB = take(sizeof(double) * 4 * L->total_tiles);
    L->partN = take(sizeof(double) * 4 * L->total_tiles);
    L->slots = take((size_t)capacity * (size_t)L->slot_amps * es);
    L->dS = L->escr = L->E = L->partC = off;
    L->escr_warps = 0;
    if (adjoint) {
        L->dS = take(sizeof(double2) * ninst * (size_t)L->mmax * L->mmax);
        L->E = take((size_t)L->mmax * (size_t)amps * es);
        L->partC = take(sizeof(double) * NCP * (size_t)L->total_tiles);
    }
    L->total = off;
    return true;
}

template <typename R, int T>
struct Shape {
    // register-heavy shapes (32 complex64 or 16 complex128 amplitudes per lane) keep one
    // CTA per SM; the smaller ones are compiled for two
    static constexpr int MINB = (sizeof(R) == 4 ? T >= 10 : T >= 9) ? 1 : 2;
};

// kind 0: forward (lock-step rounds); 1: adjoint rounds; 2: adjoint post-processing;
// 3: forward (phase engine)
static void *pick_kernel(int dtype, int T, int kind) {
#define EMUSV_K(R, TT)                                                                   \
    (kind == 1   ? reinterpret_cast<void *>(k_batch_adj_rounds<R, TT, Shape<R, TT>::MINB>) \
     : kind == 2 ? reinterpret_cast<void *>(k_batch_adj_post<R, TT, Shape<R, TT>::MINB>)   \
     : kind == 3 ? reinterpret_cast<void *>(k_batch_phase<R, TT, Shape<R, TT>::MINB>)      \
                 : reinterpret_cast<void *>(k_batch<R, TT, Shape<R, TT>::MINB>))
    if (dtype == EMUSV_C64) {
        if (T == 8) return EMUSV_K(float, 8);
        if (T == 9) return EMUSV_K(float, 9);
        if (T == 10) return EMUSV_K(float, 10);
    } else if (dtype == EMUSV_C128) {
        if (T == 8) return EMUSV_K(double, 8);
        if (T == 9) return EMUSV_K(double, 9);
    }
#undef EMUSV_K
    return nullptr;
}

// Dynamic shared memory of a kernel kind: the H v phase's partner-tile stages (kinds 0
// and 1; the post-processing kernel has none).  Set as the kernel's limit before its
// occupancy is queried or it is launched.
static size_t kernel_smem(int dtype, int T, int kind) {
    if (kind == 2) return 0;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    return (size_t)BWARPS * PSTAGES * (es << T);
}
static int configure_smem(void *kern, size_t smem) {
    if (!smem) return EMUSV_OK;
    EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return EMUSV_OK;
}

// Host copies of the argument blocks prepared per workspace (launches pass them by value,
// so the kernel reads them from the parameter bank).
struct Prepared {
    BArgs A;
    BAdj D;
    BLayout L;
    bool adjoint;
    int engine;  // forward launches: 0 lock-step rounds, 1 phase engine
};
static std::mutex g_args_mu;
static std::unordered_map<const void *, Prepared> g_args;

static int prepare_common(int ninst, const int *nqubits, const int *nsteps, const double *dt,
                          int dtype, const double *omegas, const double *deltas, const double *phis,
                          const double *interactions, void *states, double exp_tolerance,
                          double norm_tolerance, int max_krylov_dim, int T, int capacity,
                          bool adjoint, void *workspace, size_t workspace_bytes, cudaStream_t s) {
    if (ninst < 1 || !nqubits || !nsteps || !dt || !omegas || !deltas || !phis || !interactions ||
        !workspace || max_krylov_dim < 1 || max_krylov_dim > KMAX - 2 || capacity < 1 ||
        capacity > KMAX - 2 || !pick_kernel(dtype, T, adjoint ? 1 : 0) ||
        (reinterpret_cast<uintptr_t>(workspace) & 255) || (reinterpret_cast<uintptr_t>(states) & 15))
        return EMUSV_BAD_ARGUMENT;
    for (int i = 0; i < ninst; ++i)
        if (!isfinite(dt[i])) return EMUSV_BAD_ARGUMENT;
    // the shared-memory limits of the kernels the launches may use (host calls, so that a
    // launch recorded into a CUDA graph issues none)
    for (int kind : {0, 1, 3}) {
        const int st = configure_smem(pick_kernel(dtype, T, kind), kernel_smem(dtype, T, kind));
        if (st) return st;
    }
    const int es = dtype == EMUSV_C128 ? 16 : 8;
    BLayout L;
    if (!layout(ninst, nqubits, nsteps, es, T, capacity, adjoint, &L)) return EMUSV_BAD_ARGUMENT;
    if (workspace_bytes < L.total) return EMUSV_WORKSPACE_TOO_SMALL;
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    const int nj = L.njobs;

    std::vector<BInst> inst(nj);
    std::vector<BCoef> coef(L.coef_count > 0 ? L.coef_count : 1);
    std::vector<double> ub((size_t)BMAXQ * BMAXQ * ninst, 0.0);
    std::vector<double> elow((size_t)ninst << T, 0.0);
    long long off = 0;
    int c0 = 0;
    size_t pofs = 0, uofs = 0;  // offsets into the packed parameter arrays
    for (int i = 0; i < ninst; ++i) {
        const int n = nqubits[i];
        for (int k = 0; k < nsteps[i]; ++k) {
            BCoef &C = coef[c0 + k];
            memset(&C, 0, sizeof(C));
            for (int q = 0; q < n; ++q) {
                const int p = n - 1 - q;  // qubit q is bit n-1-q
                const double om = omegas[pofs + (size_t)k * n + q];
                const double de = deltas[pofs + (size_t)k * n + q];
                const double ph = phis[pofs + (size_t)k * n + q];
                if (!isfinite(om) || !isfinite(de) || !isfinite(ph)) return EMUSV_BAD_ARGUMENT;
                C.up_re[p] = 0.5 * om * cos(ph);  // hamiltonian.py:52,62-64
                C.up_im[p] = ph == 0.0 ? 0.0 : 0.5 * om * sin(ph);
                C.field[p] = -de;
                C.om[p] = om;
                C.ph[p] = ph;
                C.fup_re[p] = (float)C.up_re[p];
                C.fup_im[p] = (float)C.up_im[p];
            }
        }
        double *U = ub.data() + (size_t)i * BMAXQ * BMAXQ;
        for (int a = 0; a < n; ++a)
            for (int b = a + 1; b < n; ++b) {  // upper triangle of qubit pairs
                const double u = interactions[uofs + (size_t)a * n + b];
                if (!isfinite(u)) return EMUSV_BAD_ARGUMENT;
                const int p = n - 1 - b, q = n - 1 - a;  // p < q
                U[p * BMAXQ + q] = u;
                U[q * BMAXQ + p] = u;
            }
        double *E = elow.data() + ((size_t)i << T);
        for (int l = 0; l < (1 << T); ++l) {
            double e = 0.0;
            for (int p = 0; p < T; ++p)
                if ((l >> p) & 1)
                    for (int q = p + 1; q < T; ++q)
                        if ((l >> q) & 1) e += U[p * BMAXQ + q];
            E[l] = e;
        }
        const int per = adjoint ? 2 : 1;
        for (int r = 0; r < per; ++r) {
            BInst &I = inst[per * i + r];
            I.n = n;
            I.nsteps = adjoint ? (1 << 30) : nsteps[i];
            I.ntiles = 1 << (n - T);
            I.off0 = off;
            I.dt = dt[i];
            I.coef0 = c0;
            I.pidx = i;
            I.src = r;
            I.pad = 0;
        }
        off += 1LL << n;
        c0 += nsteps[i];
        pofs += (size_t)nsteps[i] * n;
        uofs += (size_t)n * n;
    }
    long long joff = 0;
    int tile = 0;
    for (int J = 0; J < nj; ++J) {  // stored-vector offsets and tiles, jobs back to back
        inst[J].off = joff;
        inst[J].tile0 = tile;
        joff += 1LL << inst[J].n;
        tile += inst[J].ntiles;
    }
    Prepared P;
    memset(&P, 0, sizeof(P));
    P.L = L;
    P.adjoint = adjoint;
    BArgs &A = P.A;
    A.ninst = nj;
    A.T = T;
    A.total_tiles = L.total_tiles;
    A.maxdim = max_krylov_dim;
    A.capacity = capacity;
    A.max_steps = L.max_steps;
    A.exp_tol = exp_tolerance;
    A.norm_tol = norm_tolerance;
    A.inst = reinterpret_cast<BInst *>(ws + L.inst);
    A.coef = reinterpret_cast<BCoef *>(ws + L.coef);
    A.Ubits = reinterpret_cast<double *>(ws + L.ubits);
    A.Elow = reinterpret_cast<double *>(ws + L.elow);
    A.ks = reinterpret_cast<KState *>(ws + L.ks);
    int *ints = reinterpret_cast<int *>(ws + L.ints);
    A.jst = reinterpret_cast<unsigned long long *>(ints);
    A.take = reinterpret_cast<unsigned long long *>(ints + 2 * nj);
    A.hint = ints + 4 * nj;
    A.polled = ints + 5 * nj;
    A.fail = ints + 6 * nj;
    A.status_out = ints + 7 * nj;
    A.ranB = ints + 8 * nj;
    A.cnt = reinterpret_cast<unsigned *>(ints + 9 * nj);
    double *sums = reinterpret_cast<double *>(ws + L.sums);
    A.sumA = sums;
    A.sumB = sums + 4 * nj;
    A.sumN = sums + 8 * nj;
    A.iters_out = reinterpret_cast<int *>(ws + L.iters);
    A.partA = reinterpret_cast<double *>(ws + L.partA);
    A.partB = reinterpret_cast<double *>(ws + L.partB);
    A.partN = reinterpret_cast<double *>(ws + L.partN);
    A.v0[0] = states;
    A.v0[1] = nullptr;
    A.slots = ws + L.slots;
    A.slot_amps = L.slot_amps;
    A.ctl = reinterpret_cast<BCtl *>(ws + L.ctl);
    A.first_step = 0;
    A.run_steps = L.max_steps;
    A.hist = nullptr;
    A.hist_every = 1;
    A.hist_stride = L.inst_amps;
    A.bar_limit = BAR_LIMIT;
    A.test_skip_arrival = 0;
    A.combine = adjoint ? 0 : 1;
    if (adjoint) {
        BAdj &D = P.D;
        D.ninst = ninst;
        D.mmax = L.mmax;
        D.dS = reinterpret_cast<double2 *>(ws + L.dS);
        D.E = ws + L.E;
        D.inst_amps = L.inst_amps;
        D.partC = reinterpret_cast<double *>(ws + L.partC);
        D.cntC = reinterpret_cast<unsigned *>(ints + 12 * nj);
    }
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.args, &A, sizeof(A), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.inst, inst.data(), sizeof(BInst) * nj, cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.coef, coef.data(), sizeof(BCoef) * coef.size(), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.ubits, ub.data(), sizeof(double) * ub.size(), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.elow, elow.data(), sizeof(double) * elow.size(), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemsetAsync(ws + L.ctl, 0, sizeof(BCtl) + sizeof(int) * (12 * (size_t)nj + ninst), s));
    EMUSV_CHECK(cudaStreamSynchronize(s));  // the host tables go out of scope
    {
        std::lock_guard<std::mutex> g(g_args_mu);
        g_args[workspace] = P;
    }
    return EMUSV_OK;
}

static int lookup(const void *workspace, bool adjoint, Prepared *out) {
    std::lock_guard<std::mutex> g(g_args_mu);
    auto it = g_args.find(workspace);
    if (it == g_args.end() || it->second.adjoint != adjoint) return EMUSV_BAD_ARGUMENT;
    *out = it->second;
    return EMUSV_OK;
}

static int cooperative_launch(void *kern, int blocks_per_sm, void **args, cudaStream_t s,
                              int *grid_out, int prof_kind = PROF_BATCH, size_t smem = 0) {
    int per_sm = 0;
    EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BWARPS * 32, smem));
    if (per_sm < 1) return EMUSV_CUDA_ERROR;
    const int bps = blocks_per_sm < per_sm ? blocks_per_sm : per_sm;
    const int grid = bps * sm_count();
    if (grid_out) *grid_out = grid;
    ProfScope ps_(prof_kind, s);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(BWARPS * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    EMUSV_CHECK(cudaLaunchKernelExC(&cfg, kern, args));
    return EMUSV_OK;
}

}  // namespace emusv

using namespace emusv;

extern "C" {

int emusv_batch_max_qubits(void) { return BMAXQ; }

size_t emusv_batch_workspace_bytes(int ninst, const int *nqubits, const int *nsteps, int dtype,
                                   int tile_bits, int basis_capacity) {
    if (ninst < 1 || !nqubits || !nsteps || basis_capacity < 1 || basis_capacity > KMAX - 2 ||
        !pick_kernel(dtype, tile_bits, 0))
        return 0;
    BLayout L;
    if (!layout(ninst, nqubits, nsteps, dtype == EMUSV_C128 ? 16 : 8, tile_bits, basis_capacity,
                false, &L))
        return 0;
    return L.total;
}

int emusv_batch_prepare(int ninst, const int *nqubits, const int *nsteps, const double *dt,
                        int dtype, const double *omegas, const double *deltas, const double *phis,
                        const double *interactions, void *states, double exp_tolerance,
                        double norm_tolerance, int max_krylov_dim, int tile_bits,
                        int basis_capacity, void *workspace, size_t workspace_bytes,
                        void *stream) {
    if (!states) return EMUSV_BAD_ARGUMENT;
    return prepare_common(ninst, nqubits, nsteps, dt, dtype, omegas, deltas, phis, interactions,
                          states, exp_tolerance, norm_tolerance, max_krylov_dim, tile_bits,
                          basis_capacity, false, workspace, workspace_bytes, as_stream(stream));
}

int emusv_batch_launch_steps(int dtype, int tile_bits, int blocks_per_sm, int first_step,
                             int steps, void *states, void *history, int history_every,
                             void *workspace, void *stream) {
    Prepared P;
    if (!workspace || blocks_per_sm < 1 || lookup(workspace, false, &P)) return EMUSV_BAD_ARGUMENT;
    const int kind = P.engine ? 3 : 0;
    void *kern = pick_kernel(dtype, tile_bits, kind);
    if (!kern) return EMUSV_BAD_ARGUMENT;
    BArgs A = P.A;
    if (first_step < 0 || steps < 0 || (P.engine && (steps < 1 || steps > 65535)) ||
        first_step + steps > P.L.max_steps || history_every < 1 ||
        (states && (reinterpret_cast<uintptr_t>(states) & 15)))
        return EMUSV_BAD_ARGUMENT;
    if (A.T != tile_bits) return EMUSV_BAD_ARGUMENT;
    if (states) A.v0[0] = states;
    A.first_step = first_step;
    A.run_steps = steps;
    A.hist = history;
    A.hist_every = history_every;
    cudaStream_t s = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    // control block, flags, hints and tile counters start at zero
    EMUSV_CHECK(cudaMemsetAsync(ws + P.L.ctl, 0, sizeof(BCtl) + sizeof(int) * 12 * (size_t)A.ninst, s));
    void *args[] = {(void *)&A};
    return cooperative_launch(kern, blocks_per_sm, args, s, nullptr, PROF_BATCH,
                              kernel_smem(dtype, tile_bits, kind));
}

// Scheduling of a prepared forward workspace's launches: 0 (default) lock-step rounds,
// 1 the phase engine.  Host-side only (takes effect at the next launch).
int emusv_batch_set_engine(void *workspace, int engine) {
    if (!workspace || engine < 0 || engine > 1) return EMUSV_BAD_ARGUMENT;
    std::lock_guard<std::mutex> g(g_args_mu);
    auto it = g_args.find(workspace);
    if (it == g_args.end() || it->second.adjoint) return EMUSV_BAD_ARGUMENT;
    it->second.engine = engine;
    return EMUSV_OK;
}

// Clears the control block and launches the persistent kernel over every step on the
// states given to emusv_batch_prepare.  Issues only stream-ordered device work (one memset
// and one cooperative launch), so the call can be recorded into a CUDA graph and replayed.
int emusv_batch_launch(int dtype, int tile_bits, int blocks_per_sm, void *workspace, void *stream) {
    Prepared P;
    if (!workspace || lookup(workspace, false, &P)) return EMUSV_BAD_ARGUMENT;
    return emusv_batch_launch_steps(dtype, tile_bits, blocks_per_sm, 0, P.L.max_steps, nullptr,
                                    nullptr, 1, workspace, stream);
}

int emusv_batch_max_blocks_per_sm(int dtype, int tile_bits) {
    void *kern = pick_kernel(dtype, tile_bits, 0);
    if (!kern) return 0;
    const size_t smem = kernel_smem(dtype, tile_bits, 0);
    if (configure_smem(kern, smem)) return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BWARPS * 32, smem) != cudaSuccess)
        return 0;
    return per_sm;
}

int emusv_batch_results(int ninst, int max_steps, void *workspace, int *status_out,
                        int *iterations_out, void *stream) {
    Prepared P;
    if (!workspace || ninst < 1 || lookup(workspace, false, &P)) return EMUSV_BAD_ARGUMENT;
    if (P.A.ninst != ninst || P.A.max_steps != max_steps) return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    BCtl C;
    std::vector<int> st(ninst);
    EMUSV_CHECK(cudaMemcpyAsync(&C, ws + P.L.ctl, sizeof(C), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaMemcpyAsync(st.data(), P.A.status_out, sizeof(int) * ninst, cudaMemcpyDeviceToHost, s));
    if (iterations_out && max_steps > 0)
        EMUSV_CHECK(cudaMemcpyAsync(iterations_out, P.A.iters_out, sizeof(int) * (size_t)ninst * max_steps,
                                    cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));
    if (C.err) return C.err;
    int worst = EMUSV_OK;
    for (int i = 0; i < ninst; ++i) {
        int e = EMUSV_OK;
        switch (st[i]) {
            case KS_CONVERGED: case KS_HAPPY: e = EMUSV_OK; break;
            case KS_MAXDIM: e = EMUSV_NOT_CONVERGED; break;
            case BS_CAPACITY: e = EMUSV_WORKSPACE_TOO_SMALL; break;
            default: e = EMUSV_NONFINITE; break;
        }
        if (status_out) status_out[i] = e;
        if (e != EMUSV_OK && (worst == EMUSV_OK || e == EMUSV_WORKSPACE_TOO_SMALL)) worst = e;
    }
    return worst;
}

// ---- batched adjoint steps
size_t emusv_batch_adjoint_workspace_bytes(int ninst, const int *nqubits, const int *nsteps,
                                           int dtype, int tile_bits, int basis_capacity) {
    if (ninst < 1 || !nqubits || !nsteps || basis_capacity < 1 || basis_capacity > KMAX - 2 ||
        !pick_kernel(dtype, tile_bits, 1))
        return 0;
    BLayout L;
    if (!layout(ninst, nqubits, nsteps, dtype == EMUSV_C128 ? 16 : 8, tile_bits, basis_capacity,
                true, &L))
        return 0;
    return L.total;
}

int emusv_batch_adjoint_prepare(int ninst, const int *nqubits, const int *nsteps, const double *dt,
                                int dtype, const double *omegas, const double *deltas,
                                const double *phis, const double *interactions, double tolerance,
                                int max_krylov_dim, int tile_bits, int basis_capacity,
                                void *workspace, size_t workspace_bytes, void *stream) {
    return prepare_common(ninst, nqubits, nsteps, dt, dtype, omegas, deltas, phis, interactions,
                          nullptr, tolerance, tolerance, max_krylov_dim, tile_bits, basis_capacity,
                          true, workspace, workspace_bytes, as_stream(stream));
}

int emusv_batch_adjoint_launch(int dtype, int tile_bits, int blocks_per_sm, int step,
                               const void *states, const void *grad_in, void *grad_out,
                               double *grads_dev, int *status_dev, void *workspace, void *stream) {
    void *k1 = pick_kernel(dtype, tile_bits, 1), *k3 = pick_kernel(dtype, tile_bits, 2);
    Prepared P;
    if (!k1 || !workspace || !states || !grad_in || !grad_out || !grads_dev || !status_dev ||
        blocks_per_sm < 1 || lookup(workspace, true, &P))
        return EMUSV_BAD_ARGUMENT;
    if (P.A.T != tile_bits || step < 0) return EMUSV_BAD_ARGUMENT;
    for (const void *q : {states, grad_in, (const void *)grad_out})
        if (reinterpret_cast<uintptr_t>(q) & 15) return EMUSV_BAD_ARGUMENT;
    BArgs A = P.A;
    BAdj D = P.D;
    A.v0[0] = const_cast<void *>(states);
    A.v0[1] = const_cast<void *>(grad_in);
    D.step = step;
    A.first_step = step;  // the phase engine's one "step": the bases of this adjoint step
    A.run_steps = 1;
    D.grads = grads_dev;
    D.gout = grad_out;
    D.astatus = status_dev;
    cudaStream_t s = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    // clear the control block and everything after the hints and polled flags (the
    // hints carry from one step to the next)
    const int nj = A.ninst;
    EMUSV_CHECK(cudaMemsetAsync(ws + P.L.ctl, 0, sizeof(BCtl) + sizeof(int) * 4 * (size_t)nj, s));
    EMUSV_CHECK(cudaMemsetAsync(A.fail, 0, sizeof(int) * (6 * (size_t)nj + D.ninst), s));
    void *args[] = {(void *)&A, (void *)&D};
    int st = cooperative_launch(k1, blocks_per_sm, args, s, nullptr, PROF_BATCH,
                                kernel_smem(dtype, tile_bits, 1));
    if (st) return st;
    {
        ProfScope ps_(PROF_ADJOINT, s);
        dim3 grid((D.mmax + BWARPS - 1) / BWARPS, D.ninst);
        k_batch_dS<<<grid, BWARPS * 32, 0, s>>>(A, D);
    }
    EMUSV_CHECK_LAUNCH();
    EMUSV_CHECK(cudaMemsetAsync(ws + P.L.ctl, 0, sizeof(BCtl), s));
    return cooperative_launch(k3, blocks_per_sm, args, s, nullptr, PROF_ADJOINT);
}

// Failure-path test switch of a prepared workspace (forward or adjoint): later launches
// wait at most wait_cycles clock cycles at a grid barrier or for work (<= 0: the default,
// about 1 s) and, when skip_first_arrival != 0, the last CTA does not arrive at each
// launch's first barrier (lock-step rounds) or register 0's first phase is never
// published (phase engine), so the bounded waits run out and the launch reports
// EMUSV_TIMEOUT.
int emusv_batch_set_barrier_test(void *workspace, long long wait_cycles, int skip_first_arrival) {
    if (!workspace) return EMUSV_BAD_ARGUMENT;
    std::lock_guard<std::mutex> g(g_args_mu);
    auto it = g_args.find(workspace);
    if (it == g_args.end()) return EMUSV_BAD_ARGUMENT;
    it->second.A.bar_limit = wait_cycles > 0 ? wait_cycles : BAR_LIMIT;
    it->second.A.test_skip_arrival = skip_first_arrival ? 1 : 0;
    return EMUSV_OK;
}

// Krylov iteration counts of the last adjoint launch: [ninst][2] (state, gradient basis).
int emusv_batch_adjoint_iterations(int ninst, void *workspace, int *iterations_out, void *stream) {
    Prepared P;
    if (!workspace || !iterations_out || lookup(workspace, true, &P) || P.D.ninst != ninst)
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    EMUSV_CHECK(cudaMemcpyAsync(iterations_out, P.A.iters_out, sizeof(int) * 2 * (size_t)ninst,
                                cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));
    return EMUSV_OK;
}

}  // extern "C"
