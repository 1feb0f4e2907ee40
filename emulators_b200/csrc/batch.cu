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
//    inside the thread, bits >= T by coalesced loads of the partner tile; the diagonal is
//    rebuilt from an FP64 per-instance table of the low-bit pair energies plus per-tile
//    fields of the high bits.
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
//  * convergence is tested from a per-instance hint (the previous step's count - 1), and
//    the first test of a step looks back over the untested iterations (krylov_decide), so
//    each instance stops where the reference would.
#include <math.h>
#include <string.h>

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

struct BInst {
    int n, nsteps, tile0, ntiles;
    long long off;  // amplitude offset of this instance in every slot
    double dt;
    int coef0;      // index of this instance's step-0 record in the coefficient array
    int pad;
};

// Per (instance, step) coefficients by bit position p (qubit n-1-p).
struct BCoef {
    double up_re[BMAXQ], up_im[BMAXQ];  // coefficient of |1><0| on bit p (Omega/2 e^{i phi})
    double field[BMAXQ];                // -delta
    float fup_re[BMAXQ], fup_im[BMAXQ];
};

struct BCtl {
    unsigned bar_count, bar_gen;
    unsigned tile_ctr[2];
    int err;
    int pad[3];
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
    void *states;         // slot 0 (the caller's packed states, in place)
    unsigned char *slots;  // slots 1..capacity
    long long slot_amps;
    BCtl *ctl;
};

// ---------------------------------------------------------------- grid barrier
// Arrival counter + generation; the last arriver also clears the tile counter of the
// phase after next.  Returns false (and every CTA then returns) on a timeout.
__device__ bool grid_sync(BCtl *ctl, unsigned &ph) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *genp = &ctl->bar_gen;
        const unsigned g = *genp;
        __threadfence();
        const unsigned arrived = atomicAdd(&ctl->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
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
                    if (clock64() - t0 > BAR_LIMIT || *(volatile int *)&ctl->err) {
                        atomicExch(&ctl->err, EMUSV_TIMEOUT);
                        break;
                    }
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
    ++ph;
    return *(volatile int *)&ctl->err == 0;
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
// into sum[4 i..] and clears the counter for the next phase of this kind.
__device__ __forceinline__ void tile_done(unsigned *cnt, const double *part, double *sum, int i,
                                          int tile0, int ntiles) {
    const int lane = threadIdx.x & 31;
    unsigned old = 0;
    if (lane == 0) {
        __threadfence();
        old = atomicAdd(&cnt[i], 1u);
    }
    old = __shfl_sync(0xffffffffu, old, 0);
    if (old == (unsigned)ntiles - 1) {
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
}

__device__ __forceinline__ double3 ld_sum(const double *sum, int i) {
    return make_double3(__ldcg(sum + 4 * (size_t)i), __ldcg(sum + 4 * (size_t)i + 1),
                        __ldcg(sum + 4 * (size_t)i + 2));
}

template <typename C>
__device__ __forceinline__ C *vec_ptr(const BArgs &A, int k, const BInst &I) {
    if (k == 0) return reinterpret_cast<C *>(A.states) + I.off;
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

// ---------------------------------------------------------------- phase A: H v_j on a tile
template <typename R, int T>
__device__ void tile_hpsi(const BArgs &A, const BInst &I, int i, int t, int step, int j,
                          double sj) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    const int lane = threadIdx.x & 31;
    const int n = I.n;
    const long long base = (long long)(t - I.tile0) << T;
    const BCoef &cf = A.coef[I.coef0 + step];
    const double *Ub = A.Ubits + (size_t)i * BMAXQ * BMAXQ;
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
    const double *El = A.Elow + ((size_t)i << T);

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
    for (int p = T; p < n; ++p) {  // bits above the tile: the partner tile, from L2
        R cr, ci;
        coef(p, (int)((base >> p) & 1), cr, ci);
        const C *w = u + (base ^ (1LL << p)) + lane;
#pragma unroll
        for (int a = 0; a < AMP; ++a) cfma(cr, ci, ldcg(w + 32 * a), ar[a], ai[a]);
    }
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
    tile_done(A.cnt, A.partA, A.sumA, i, I.tile0, I.ntiles);
}

// ---------------------------------------------------------------- phase B: recurrence
template <typename R, int T>
__device__ void tile_orth(const BArgs &A, const BInst &I, int i, int t, int j, double car,
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
    tile_done(A.cnt + A.ninst, A.partB, A.sumB, i, I.tile0, I.ntiles);
}

template <typename R, int T>
__device__ void tile_norm(const BArgs &A, const BInst &I, int i, int t) {
    typedef typename cvec<R>::T C;
    constexpr int AMP = 1 << (T - 5);
    const int lane = threadIdx.x & 31;
    const long long base = (long long)(t - I.tile0) << T;
    const C *u = vec_ptr<C>(A, 0, I);
    double nrm = 0.0;
#pragma unroll 8
    for (int a = 0; a < AMP; ++a) {
        const C o = ldcg(u + base + lane + 32 * a);
        nrm += double(o.x) * double(o.x) + double(o.y) * double(o.y);
    }
    nrm = warp_sum(nrm);
    if (lane == 0) A.partN[4 * (size_t)t] = nrm;
    tile_done(A.cnt + 2 * A.ninst, A.partN, A.sumN, i, I.tile0, I.ntiles);
}

__device__ __forceinline__ int ld_status(const KState *ks) {
    return *(volatile const int *)&ks->status;
}
__device__ __forceinline__ int ld_vol(const int *p) { return *(volatile const int *)p; }

// ---------------------------------------------------------------- the persistent kernel
// Phase bookkeeping keeps every instance's tiles either all processed or all skipped in a
// phase (so the per-instance tile counters complete): phase A_j runs an instance if its
// step starts (j = 0) or if phase B of the previous round ran it (ranB), never from a
// status that the decisions of the same phase may be changing.
template <typename R, int T, int MINB>
__global__ void __launch_bounds__(BWARPS * 32, MINB) k_batch(const BArgs A) {
    typedef typename cvec<R>::T C;
    __shared__ KSmem S;
    __shared__ int s_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned ph = 0;
    int round = 0;  // phase-B rounds so far (the same in every CTA)

    // initial norms
    for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
        const int i = inst_of_tile(A, t);
        tile_norm<R, T>(A, A.inst[i], i, t);
    }
    if (!grid_sync(A.ctl, ph)) return;

    for (int step = 0; step < A.max_steps; ++step) {
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
                            else if (step >= I.nsteps) st = BS_IDLE;
                            else if (!(isfinite(s0) && s0 > 0.0)) st = KS_NONFINITE;
                            ks->s0 = s0;
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
                    const int jj = j - 1;
                    const double3 sb = ld_sum(A.sumB, i);
                    const int hint = A.hint[i];
                    const bool poll = (jj + 1 >= hint) || (jj + 1 >= A.maxdim);
                    const bool first = poll && !A.polled[i];
                    __syncwarp();
                    if (lane == 0 && poll) A.polled[i] = 1;
                    krylov_decide(ks, jj, sb.x, sb.y, sb.z, I.dt, A.exp_tol, A.norm_tol, poll,
                                  first, A.maxdim, S);
                    if (lane == 0) {
                        int st = ks->status;
                        if (st == KS_RUNNING && jj + 2 > A.capacity) {
                            st = BS_CAPACITY;
                            ks->status = st;
                        }
                        if (st == KS_NONFINITE || st == BS_CAPACITY) A.fail[i] = st;
                        if (st != KS_RUNNING) {
                            A.iters_out[(size_t)i * A.max_steps + step] = ks->iters;
                            A.hint[i] = ks->iters > 1 ? ks->iters - 1 : 0;
                        }
                    }
                    __syncwarp();
                }
            }
            if (j < A.maxdim && j + 1 <= A.capacity) {
                for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
                    const int i = inst_of_tile(A, t);
                    const BInst I = A.inst[i];
                    double sj;
                    if (j == 0) {
                        if (step >= I.nsteps || ld_vol(&A.fail[i])) continue;
                        sj = 1.0 / sqrt(__ldcg(A.sumN + 4 * (size_t)i));
                    } else {
                        if (ld_vol(&A.ranB[i]) != round) continue;  // B ran it last round
                        sj = 1.0 / sqrt(__ldcg(A.sumB + 4 * (size_t)i));
                    }
                    if (!isfinite(sj) || sj <= 0.0) continue;  // the same for all its tiles
                    tile_hpsi<R, T>(A, I, i, t, step, j, sj);
                }
            }
            if (!grid_sync(A.ctl, ph)) return;
            // does any instance still iterate?
            if (warp == 0) {
                int any = 0;
                for (int i = lane; i < A.ninst; i += 32) any |= ld_status(A.ks + i) == KS_RUNNING;
                any = __any_sync(0xffffffffu, any);
                if (lane == 0) s_flag = any;
            }
            __syncthreads();
            if (!s_flag) break;
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
                        const double3 s = ld_sum(A.sumA, i);
                        const double b = j > 0 ? __ldcg(&ks->r[j - 1]) : 0.0;
                        const double vr = j > 0 ? __ldcg(&ks->vv_re[j]) : 0.0;
                        const double vi = j > 0 ? __ldcg(&ks->vv_im[j]) : 0.0;
                        const double ar = s.y - b * vr, ai = s.z - b * vi;
                        sj = __ldcg(&ks->scale[j]);
                        const double sp = j > 0 ? __ldcg(&ks->scale[j - 1]) : 0.0;
                        car = ar * sj;
                        cai = ai * sj;
                        cb = b * sp;
                        ci = i;
                        // the warp of the instance's first tile records T_H's column j (a warp
                        // meets a given instance's first tile before any other of its tiles)
                        if (t == I.tile0 && lane == 0) {
                            ks->a_re[j] = ar;
                            ks->a_im[j] = ai;
                            ks->b_re[j] = b;
                            ks->b_im[j] = 0.0;
                            ks->hn[j] = sqrt(s.x);
                            A.ranB[i] = round + 1;  // 0 (cleared at launch) = never
                        }
                    }
                    tile_orth<R, T>(A, I, i, t, j, car, cai, cb, sj);
                }
            }
            if (!grid_sync(A.ctl, ph)) return;
            ++round;
        }
        // ---------------- combination of every instance that took this step
        {
            int ci = -1, nvec = 0;
            double cr0 = 0, ci0 = 0, cr1 = 0, ci1 = 0, cr2 = 0, ci2 = 0, cr3 = 0, ci3 = 0;
            for (int t = next_tile(A.ctl, ph); t < A.total_tiles; t = next_tile(A.ctl, ph)) {
                const int i = inst_of_tile(A, t);
                const KState *ks = A.ks + i;
                const int st = ld_status(ks);
                const BInst I = A.inst[i];
                if (st != KS_CONVERGED && st != KS_HAPPY && st != KS_MAXDIM) {
                    // idle or failed: keep the state, refresh its norm for the next step
                    tile_norm<R, T>(A, I, i, t);
                    continue;
                }
                if (i != ci) {
                    // coefficients s0 scale_k c_k (k < nvec <= 128): lane k % 32 holds block
                    // k / 32 in registers; the combination reads them by shuffles
                    nvec = __ldcg(&ks->nvec);
                    const double s0 = __ldcg(&ks->s0);
                    double *cr[4] = {&cr0, &cr1, &cr2, &cr3}, *cim[4] = {&ci0, &ci1, &ci2, &ci3};
#pragma unroll
                    for (int blk = 0; blk < 4; ++blk) {
                        const int k = lane + 32 * blk;
                        double a = 0.0, b = 0.0;
                        if (k < nvec) {
                            const double f = s0 * __ldcg(&ks->scale[k]);
                            a = f * __ldcg(&ks->c_re[k]);
                            b = f * __ldcg(&ks->c_im[k]);
                        }
                        *cr[blk] = a;
                        *cim[blk] = b;
                    }
                    ci = i;
                }
                constexpr int AMP = 1 << (T - 5);
                constexpr int CH = AMP < 4 ? AMP : 4;
                const long long base = (long long)(t - I.tile0) << T;
                C *out = vec_ptr<C>(A, 0, I);
                double nrm = 0.0;
                for (int a0 = 0; a0 < AMP; a0 += CH) {
                    double re[CH], im[CH];
#pragma unroll
                    for (int c = 0; c < CH; ++c) re[c] = im[c] = 0.0;
                    for (int k = 0; k < nvec; ++k) {
                        const int src = k & 31, blk = k >> 5;
                        const double vr = blk == 0 ? cr0 : blk == 1 ? cr1 : blk == 2 ? cr2 : cr3;
                        const double vi = blk == 0 ? ci0 : blk == 1 ? ci1 : blk == 2 ? ci2 : ci3;
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
                        nrm += double(o.x) * double(o.x) + double(o.y) * double(o.y);
                    }
                }
                nrm = warp_sum(nrm);
                if (lane == 0) A.partN[4 * (size_t)t] = nrm;
                tile_done(A.cnt + 2 * A.ninst, A.partN, A.sumN, i, I.tile0, I.ntiles);
            }
        }
        if (!grid_sync(A.ctl, ph)) return;
    }
    // final statuses
    if (threadIdx.x < 32) {
        for (int i = blockIdx.x * 32 + lane; i < A.ninst; i += gridDim.x * 32) {
            const int st = ld_status(A.ks + i);
            A.status_out[i] = A.fail[i] ? A.fail[i] : (st == BS_IDLE ? KS_CONVERGED : st);
        }
    }
}

// ---------------------------------------------------------------- host side
static size_t al256(size_t v) { return (v + 255) / 256 * 256; }

struct BLayout {
    size_t args, ctl, ints, inst, coef, ubits, elow, ks, sums, iters, partA, partB, partN, slots,
        total;
    int total_tiles;
    long long slot_amps;
    int coef_count;
};

static bool layout(int ninst, const int *nq, const int *nsteps, int es, int T, int capacity,
                   int max_steps, BLayout *L) {
    long long amps = 0;
    int tiles = 0, coefs = 0;
    for (int i = 0; i < ninst; ++i) {
        if (nq[i] < T || nq[i] > BMAXQ || nsteps[i] < 0) return false;
        amps += 1LL << nq[i];
        tiles += 1 << (nq[i] - T);
        coefs += nsteps[i] > 0 ? nsteps[i] : 0;
    }
    size_t off = 0;
    auto take = [&](size_t b) { const size_t o = off; off += al256(b); return o; };
    L->args = take(sizeof(BArgs));
    // control block and per-instance integer flags, contiguous: cleared by every launch
    L->ctl = off;
    off += sizeof(BCtl);
    L->ints = off;
    off += sizeof(int) * 8 * ninst;  // hint, polled, fail, status, ranB, cnt[3]
    off = al256(off);
    L->inst = take(sizeof(BInst) * ninst);
    L->coef = take(sizeof(BCoef) * (coefs > 0 ? coefs : 1));
    L->ubits = take(sizeof(double) * BMAXQ * BMAXQ * ninst);
    L->elow = take(sizeof(double) * ((size_t)ninst << T));
    L->ks = take(sizeof(KState) * ninst);
    L->sums = take(sizeof(double) * 12 * ninst);
    L->iters = take(sizeof(int) * (size_t)ninst * (max_steps > 0 ? max_steps : 1));
    L->partA = take(sizeof(double) * 4 * tiles);
    L->partB = take(sizeof(double) * 4 * tiles);
    L->partN = take(sizeof(double) * 4 * tiles);
    L->slots = take((size_t)capacity * (size_t)amps * es);
    L->total = off;
    L->total_tiles = tiles;
    L->slot_amps = amps;
    L->coef_count = coefs;
    return true;
}

// Register-heavy shapes (32 complex64 or 16 complex128 amplitudes per lane) keep one CTA
// per SM; the smaller ones are compiled for two.
template <typename R, int T>
static void *kernel_ptr() {
    constexpr int MINB = (sizeof(R) == 4 ? T >= 10 : T >= 9) ? 1 : 2;
    return reinterpret_cast<void *>(k_batch<R, T, MINB>);
}

// Host copies of the argument blocks prepared per workspace (the launch passes the block
// by value, so the kernel reads it from the parameter bank).
static std::mutex g_args_mu;
static std::unordered_map<const void *, BArgs> g_args;

static void *pick_kernel(int dtype, int T) {
    if (dtype == EMUSV_C64) {
        if (T == 8) return kernel_ptr<float, 8>();
        if (T == 9) return kernel_ptr<float, 9>();
        if (T == 10) return kernel_ptr<float, 10>();
    } else if (dtype == EMUSV_C128) {
        if (T == 8) return kernel_ptr<double, 8>();
        if (T == 9) return kernel_ptr<double, 9>();
    }
    return nullptr;
}

}  // namespace emusv

using namespace emusv;

extern "C" {

int emusv_batch_max_qubits(void) { return BMAXQ; }

size_t emusv_batch_workspace_bytes(int ninst, const int *nqubits, const int *nsteps, int dtype,
                                   int tile_bits, int basis_capacity) {
    if (ninst < 1 || !nqubits || !nsteps || basis_capacity < 1 || !pick_kernel(dtype, tile_bits))
        return 0;
    int max_steps = 0;
    for (int i = 0; i < ninst; ++i) max_steps = nsteps[i] > max_steps ? nsteps[i] : max_steps;
    BLayout L;
    if (!layout(ninst, nqubits, nsteps, dtype == EMUSV_C128 ? 16 : 8, tile_bits, basis_capacity,
                max_steps, &L))
        return 0;
    return L.total;
}

int emusv_batch_prepare(int ninst, const int *nqubits, const int *nsteps, const double *dt,
                        int dtype, const double *omegas, const double *deltas, const double *phis,
                        const double *interactions, void *states, double exp_tolerance,
                        double norm_tolerance, int max_krylov_dim, int tile_bits,
                        int basis_capacity, void *workspace, size_t workspace_bytes,
                        void *stream) {
    if (ninst < 1 || !nqubits || !nsteps || !dt || !omegas || !deltas || !phis || !interactions ||
        !states || (reinterpret_cast<uintptr_t>(states) & 15) ||
        !workspace || max_krylov_dim < 1 || max_krylov_dim > KMAX - 2 || basis_capacity < 1 ||
        !pick_kernel(dtype, tile_bits) || (reinterpret_cast<uintptr_t>(workspace) & 255))
        return EMUSV_BAD_ARGUMENT;
    const int T = tile_bits;
    int max_steps = 0;
    for (int i = 0; i < ninst; ++i) {
        if (!isfinite(dt[i])) return EMUSV_BAD_ARGUMENT;
        max_steps = nsteps[i] > max_steps ? nsteps[i] : max_steps;
    }
    const int es = dtype == EMUSV_C128 ? 16 : 8;
    BLayout L;
    if (!layout(ninst, nqubits, nsteps, es, T, basis_capacity, max_steps, &L))
        return EMUSV_BAD_ARGUMENT;
    if (workspace_bytes < L.total) return EMUSV_WORKSPACE_TOO_SMALL;
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    cudaStream_t s = as_stream(stream);

    // host tables
    std::vector<BInst> inst(ninst);
    std::vector<BCoef> coef(L.coef_count > 0 ? L.coef_count : 1);
    std::vector<double> ub((size_t)BMAXQ * BMAXQ * ninst, 0.0);
    std::vector<double> elow((size_t)ninst << T, 0.0);
    long long off = 0;
    int tile = 0, c0 = 0;
    size_t pofs = 0, uofs = 0;  // offsets into the packed parameter arrays
    for (int i = 0; i < ninst; ++i) {
        const int n = nqubits[i];
        BInst &I = inst[i];
        I.n = n;
        I.nsteps = nsteps[i];
        I.tile0 = tile;
        I.ntiles = 1 << (n - T);
        I.off = off;
        I.dt = dt[i];
        I.coef0 = c0;
        I.pad = 0;
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
                C.up_im[p] = 0.5 * om * sin(ph);
                if (ph == 0.0) C.up_im[p] = 0.0;
                C.field[p] = -de;
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
        off += 1LL << n;
        tile += 1 << (n - T);
        c0 += nsteps[i] > 0 ? nsteps[i] : 0;
        pofs += (size_t)(nsteps[i] > 0 ? nsteps[i] : 0) * n;
        uofs += (size_t)n * n;
    }
    BArgs A;
    memset(&A, 0, sizeof(A));
    A.ninst = ninst;
    A.T = T;
    A.total_tiles = L.total_tiles;
    A.maxdim = max_krylov_dim;
    A.capacity = basis_capacity;
    A.max_steps = max_steps;
    A.exp_tol = exp_tolerance;
    A.norm_tol = norm_tolerance;
    A.inst = reinterpret_cast<BInst *>(ws + L.inst);
    A.coef = reinterpret_cast<BCoef *>(ws + L.coef);
    A.Ubits = reinterpret_cast<double *>(ws + L.ubits);
    A.Elow = reinterpret_cast<double *>(ws + L.elow);
    A.ks = reinterpret_cast<KState *>(ws + L.ks);
    int *ints = reinterpret_cast<int *>(ws + L.ints);
    A.hint = ints;
    A.polled = ints + ninst;
    A.fail = ints + 2 * ninst;
    A.status_out = ints + 3 * ninst;
    A.ranB = ints + 4 * ninst;
    A.cnt = reinterpret_cast<unsigned *>(ints + 5 * ninst);
    double *sums = reinterpret_cast<double *>(ws + L.sums);
    A.sumA = sums;
    A.sumB = sums + 4 * ninst;
    A.sumN = sums + 8 * ninst;
    A.iters_out = reinterpret_cast<int *>(ws + L.iters);
    A.partA = reinterpret_cast<double *>(ws + L.partA);
    A.partB = reinterpret_cast<double *>(ws + L.partB);
    A.partN = reinterpret_cast<double *>(ws + L.partN);
    A.states = states;
    A.slots = ws + L.slots;
    A.slot_amps = L.slot_amps;
    A.ctl = reinterpret_cast<BCtl *>(ws + L.ctl);
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.args, &A, sizeof(A), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.inst, inst.data(), sizeof(BInst) * ninst, cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.coef, coef.data(), sizeof(BCoef) * coef.size(), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.ubits, ub.data(), sizeof(double) * ub.size(), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(ws + L.elow, elow.data(), sizeof(double) * elow.size(), cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));  // the host tables go out of scope
    {
        std::lock_guard<std::mutex> g(g_args_mu);
        g_args[workspace] = A;
    }
    return EMUSV_OK;
}

// Clears the control block and launches the persistent kernel on the states given to
// emusv_batch_prepare.  Issues only stream-ordered device work (one memset and one
// cooperative launch), so the call can be recorded into a CUDA graph and replayed.
int emusv_batch_launch(int dtype, int tile_bits, int blocks_per_sm, void *workspace, void *stream) {
    void *kern = pick_kernel(dtype, tile_bits);
    if (!kern || !workspace || blocks_per_sm < 1) return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    int per_sm = 0;
    EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BWARPS * 32, 0));
    if (per_sm < 1) return EMUSV_CUDA_ERROR;
    const int bps = blocks_per_sm < per_sm ? blocks_per_sm : per_sm;
    const int grid = bps * sm_count();
    BArgs A;
    {
        std::lock_guard<std::mutex> g(g_args_mu);
        auto it = g_args.find(workspace);
        if (it == g_args.end()) return EMUSV_BAD_ARGUMENT;  // not prepared
        A = it->second;
    }
    // control block, flags, hints and tile counters start at zero
    const size_t clr = sizeof(BCtl) + sizeof(int) * 8 * (size_t)A.ninst;
    EMUSV_CHECK(cudaMemsetAsync(ws + al256(sizeof(BArgs)), 0, clr, s));
    void *args[] = {(void *)&A};
    {
        ProfScope ps_(PROF_BATCH, s);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(BWARPS * 32);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        EMUSV_CHECK(cudaLaunchKernelExC(&cfg, kern, args));
    }
    return EMUSV_OK;
}

// Largest CTAs per SM the persistent kernel can keep resident (the cooperative limit).
int emusv_batch_max_blocks_per_sm(int dtype, int tile_bits) {
    void *kern = pick_kernel(dtype, tile_bits);
    if (!kern) return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BWARPS * 32, 0) != cudaSuccess)
        return 0;
    return per_sm;
}

// Statuses (emusv_status per instance) and Krylov iteration counts [ninst][max_steps]
// to host arrays; returns EMUSV_TIMEOUT if a grid barrier gave up.  Synchronises.
int emusv_batch_results(int ninst, int max_steps, void *workspace, int *status_out,
                        int *iterations_out, void *stream) {
    if (!workspace || ninst < 1) return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    unsigned char *ws = reinterpret_cast<unsigned char *>(workspace);
    BArgs A;
    BCtl C;
    EMUSV_CHECK(cudaMemcpyAsync(&A, ws, sizeof(A), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaMemcpyAsync(&C, ws + al256(sizeof(BArgs)), sizeof(C), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));
    if (A.ninst != ninst || A.max_steps != max_steps) return EMUSV_BAD_ARGUMENT;
    std::vector<int> st(ninst);
    EMUSV_CHECK(cudaMemcpyAsync(st.data(), A.status_out, sizeof(int) * ninst, cudaMemcpyDeviceToHost, s));
    if (iterations_out && max_steps > 0)
        EMUSV_CHECK(cudaMemcpyAsync(iterations_out, A.iters_out, sizeof(int) * (size_t)ninst * max_steps,
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

}  // extern "C"
