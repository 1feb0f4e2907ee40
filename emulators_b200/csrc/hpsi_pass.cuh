// Two-pass fused H*psi for large registers (sm_100a).
//
// H = D + sum_p X_p-terms.  The flip terms of every bit are applied on chip, split over
// two streaming passes so that no amplitude is fetched more than once per pass:
//
//  pass L  tile = 2^TB consecutive amplitudes (bits 0..TB-1) staged in shared memory;
//          a cluster of 2^pb CTAs holds 2^pb neighbouring tiles, so the flips of bits
//          TB..TB+pb-1 read the partner amplitude from a sibling CTA's shared memory
//          (DSMEM).  The diagonal (detunings + C6/r^6 interactions) is rebuilt here from
//          per-thread / per-tile FP64 partial energies.  Output: the partial sum (or the
//          final H v when no bit is left).
//  pass H  tile = 2^c contiguous amplitudes (the c low bits, already done by pass L) x
//          2^g combinations of the g top bits, so the flips of the top bits are again
//          shared-memory reads; adds them to the partial sum and runs the epilogue.
//
// Register blocking: each of the NT = 2^(TB-RB) threads owns NA = 2^RB amplitudes that
// differ in the RB highest tile bits, so those flips are register-register; the other
// tile bits are one shared-memory load per flip at an offset known at compile time.
// Coefficients of compile-time bit positions are kernel-parameter (constant bank)
// operands.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace emusv {

namespace cg = cooperative_groups;

#ifndef PASS_MIN_BLOCKS
#define PASS_MIN_BLOCKS 1
#endif

enum PassEpi {
    EPI_PARTIAL = 0,  // store the partial sum (another pass follows)
    EPI_STORE = 1,    // store H v
    EPI_LANCZOS = 2,  // store H v; ||Hv||^2, <v,Hv>, <vp,Hv>, <v,vp> partials
};

struct PassParams {
    int n;
    int real_coef;
    // coefficients by bit position: "up" = target bit 1, "dn" = target bit 0
    float fup_re[MAXQ], fup_im[MAXQ], fdn_re[MAXQ], fdn_im[MAXQ];
    double dup_re[MAXQ], dup_im[MAXQ], ddn_re[MAXQ], ddn_im[MAXQ];
    double field[MAXQ];
    double U[MAXQ * MAXQ];
    double ER[32];  // energies of the register-bit patterns of pass L (fields + pairs)
    // layout
    int tb, rb;     // tile bits / register bits of the instantiation these tables are for
    int pb;         // pass L: cluster bits (cluster size 2^pb)
    int hc, hg;     // pass H: chunk bits c and group bits g (group = bits n-hg .. n-1 minus extra)
    int hpos;       // pass H: global position of the first group bit
    int xb_lo, xb_hi;  // pass H: bits [xb_lo, xb_hi) applied from global memory (fallback)
};

struct PassArgs {
    const void *u;          // stored input vector (raw); v = su * u
    const double *su_dev;   // device scale (or null: su)
    double su;
    const void *up;         // previous Lanczos vector (EPI_LANCZOS, may be null)
    const double *sp_dev;
    double sp;
    void *out;              // partial / final output
    double *partials;       // [gridDim.x * NRED]
    const int *gate;        // kernel returns at once when *gate != 0
};

template <typename R> struct Coef;
template <> struct Coef<float> {
    __device__ static float ure(const PassParams &P, int p) { return P.fup_re[p]; }
    __device__ static float uim(const PassParams &P, int p) { return P.fup_im[p]; }
    __device__ static float dre(const PassParams &P, int p) { return P.fdn_re[p]; }
    __device__ static float dim(const PassParams &P, int p) { return P.fdn_im[p]; }
};
template <> struct Coef<double> {
    __device__ static double ure(const PassParams &P, int p) { return P.dup_re[p]; }
    __device__ static double uim(const PassParams &P, int p) { return P.dup_im[p]; }
    __device__ static double dre(const PassParams &P, int p) { return P.ddn_re[p]; }
    __device__ static double dim(const PassParams &P, int p) { return P.ddn_im[p]; }
};

// acc += c * w  with c = up (bit==1) or dn (bit==0) of bit position p
template <typename R, bool REALC, typename C>
__device__ __forceinline__ void flip_acc(const PassParams &P, int p, bool bit, const C &w, R &ar,
                                         R &ai) {
    if (REALC) {
        const R c = Coef<R>::ure(P, p);
        ar = fmar(c, w.x, ar);
        ai = fmar(c, w.y, ai);
    } else {
        const R cr = bit ? Coef<R>::ure(P, p) : Coef<R>::dre(P, p);
        const R ci = bit ? Coef<R>::uim(P, p) : Coef<R>::dim(P, p);
        ar = fmar(cr, w.x, fmar(-ci, w.y, ar));
        ai = fmar(cr, w.y, fmar(ci, w.x, ai));
    }
}

// Epilogue shared by both passes: h = su * acc_total (+ su * d * u for pass L).
template <typename C, int EPI>
__device__ __forceinline__ void epilogue(const PassArgs &A, int64_t x, double hr, double hi,
                                         double vr, double vi, double sp, double (&red)[NRED]) {
    C *out = reinterpret_cast<C *>(A.out);
    out[x] = cmake<C>(hr, hi);
    if (EPI == EPI_LANCZOS) {
        red[0] += hr * hr + hi * hi;
        red[1] += vr * hr + vi * hi;
        red[2] += vr * hi - vi * hr;
        if (A.up) {
            const C q = reinterpret_cast<const C *>(A.up)[x];
            const double pr = sp * double(q.x), pi = sp * double(q.y);
            red[3] += pr * hr + pi * hi;
            red[4] += pr * hi - pi * hr;
            red[5] += vr * pr + vi * pi;
            red[6] += vr * pi - vi * pr;
        }
    }
}

template <int EPI>
__device__ __forceinline__ void write_partials(const PassArgs &A, double (&red)[NRED], double *scratch) {
    if (EPI != EPI_LANCZOS) return;
    block_sum<NRED>(red, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NRED; ++k) A.partials[(int64_t)blockIdx.x * NRED + k] = red[k];
    }
}

// ------------------------------------------------------------------------- pass L
template <typename R, bool REALC, int TB, int RB, int EPI>
__global__ void __launch_bounds__(1 << (TB - RB), PASS_MIN_BLOCKS)
k_pass_low(const PassParams P, PassArgs A) {
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    C *tile = reinterpret_cast<C *>(smem);
    double *sh = reinterpret_cast<double *>(smem + (sizeof(C) << TB));  // per-tile scalars
    double *crossT = sh;            // [SB]  sum_{p high set} U[q][p], q < SB
    double *crossR = sh + SB;       // [RB]
    double *eh = sh + SB + RB;      // [1]   energy of the high bits
    double *red_scr = sh + 32;      // block reduction scratch

    cg::cluster_group cl = cg::this_cluster();
    const int pb = P.pb;
    const unsigned rank = pb ? cl.block_rank() : 0;
    const int n = P.n;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;

    // per-thread constants: energy of the thread bits and thread x register crosses
    double ET = 0.0;
#pragma unroll
    for (int q = 0; q < SB; ++q) {
        if ((tid >> q) & 1) {
            ET += P.field[q];
#pragma unroll
            for (int q2 = q + 1; q2 < SB; ++q2)
                if ((tid >> q2) & 1) ET += P.U[q * MAXQ + q2];
        }
    }
    double fR[RB];
#pragma unroll
    for (int k = 0; k < RB; ++k) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < SB; ++q)
            if ((tid >> q) & 1) s += P.U[(SB + k) * MAXQ + q];
        fR[k] = s;
    }

    const double su = A.su_dev ? *A.su_dev : A.su;
    const double sp = (EPI == EPI_LANCZOS && A.up) ? (A.sp_dev ? *A.sp_dev : A.sp) : 0.0;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;

    const int CS = 1 << pb;
    const int64_t nsuper = int64_t(1) << (n - TB - pb);
    const int nclusters = gridDim.x >> pb;
    const int cid = blockIdx.x >> pb;
    for (int64_t s = cid; s < nsuper; s += nclusters) {
        const int64_t t = (s << pb) | rank;
        const int64_t base = t << TB;
        // stage own amplitudes (coalesced) into registers and shared memory
        C v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) v[a] = u[base + tid + a * NT];
        if (warp == 0) {
            // per-tile high-bit energy and crosses (bits >= TB are fixed by `base`)
            double e = 0.0;
            for (int p = TB + lane; p < n; p += 32) {
                if (!((base >> p) & 1)) continue;
                e += P.field[p];
                for (int p2 = p + 1; p2 < n; ++p2)
                    if ((base >> p2) & 1) e += P.U[p * MAXQ + p2];
            }
            e = warp_sum(e);
            if (lane == 0) eh[0] = e;
            if (lane < TB) {
                double c = 0.0;
                for (int p = TB; p < n; ++p)
                    if ((base >> p) & 1) c += P.U[lane * MAXQ + p];
                if (lane < SB) crossT[lane] = c;
                else crossR[lane - SB] = c;
            }
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) tile[tid + a * NT] = v[a];
        if (pb) cl.sync(); else __syncthreads();

        double St = ET + eh[0];
#pragma unroll
        for (int q = 0; q < SB; ++q)
            if ((tid >> q) & 1) St += crossT[q];
        double hR[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) hR[k] = fR[k] + crossR[k];

#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int l = tid + a * NT;
            R ar = R(0), ai = R(0);
            // thread bits: partner in shared memory
#pragma unroll
            for (int q = 0; q < SB; ++q) {
                const C w = tile[l ^ (1 << q)];
                flip_acc<R, REALC>(P, q, (tid >> q) & 1, w, ar, ai);
            }
            // register bits: partner in registers
#pragma unroll
            for (int k = 0; k < RB; ++k)
                flip_acc<R, REALC>(P, SB + k, (a >> k) & 1, v[a ^ (1 << k)], ar, ai);
            // cluster bits: partner tile in a sibling CTA
            for (int r = 0; r < pb; ++r) {
                const C *rt = cl.map_shared_rank(tile, rank ^ (1u << r));
                flip_acc<R, REALC>(P, TB + r, (rank >> r) & 1, rt[l], ar, ai);
            }
            // diagonal: St + E_R[a] + sum_{k in a} hR[k]
            double d = St + P.ER[a];
#pragma unroll
            for (int k = 0; k < RB; ++k)
                if ((a >> k) & 1) d += hR[k];
            const int64_t x = base + l;
            const double ur = double(v[a].x), ui = double(v[a].y);
            const double hr = su * (double(ar) + d * ur), hi = su * (double(ai) + d * ui);
            if (EPI == EPI_PARTIAL) {
                // partial sum without the scale (pass H applies su once)
                reinterpret_cast<C *>(A.out)[x] = cmake<C>(double(ar) + d * ur, double(ai) + d * ui);
            } else {
                epilogue<C, EPI>(A, x, hr, hi, su * ur, su * ui, sp, red);
            }
        }
        if (pb) cl.sync(); else __syncthreads();  // siblings done reading this tile
    }
    write_partials<EPI>(A, red, red_scr);
}

// ------------------------------------------------------------------------- pass H
// Tile local index l = (j << c) | i, i < 2^c (contiguous low bits), j < 2^g (group bits
// hpos..hpos+g-1, g = TB - c).  The thread owns l = tid + a*NT;
// x = base + (l & cmask) + ((l >> c) << hpos), where base enumerates bits c..hpos-1 and
// bits >= hpos+g.  Flips of local bits k >= c (global bit hpos + k - c) are applied;
// the chunk bits were applied by pass L.
template <typename R, bool REALC, int TB, int RB, int EPI>
__global__ void __launch_bounds__(1 << (TB - RB), PASS_MIN_BLOCKS)
k_pass_high(const PassParams P, PassArgs A) {
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    C *tile = reinterpret_cast<C *>(smem);
    double *red_scr = reinterpret_cast<double *>(smem + (sizeof(C) << TB));
    const int n = P.n, c = P.hc, g = P.hg, hpos = P.hpos;
    const int tid = threadIdx.x;
    const int64_t cmask = (int64_t(1) << c) - 1;
    const int lowbits = hpos - c;  // base bits between the chunk and the group
    const int64_t ntiles = int64_t(1) << (n - c - g);

    // coefficients of the shared-memory bits (direction fixed by the thread's own bits)
    R cr_s[SB], ci_s[SB];
#pragma unroll
    for (int k = 0; k < SB; ++k) {
        const int p = hpos + k - c;
        const bool ok = k >= c;
        const bool bit = (tid >> k) & 1;
        cr_s[k] = ok ? (bit ? Coef<R>::ure(P, p) : Coef<R>::dre(P, p)) : R(0);
        ci_s[k] = ok ? (bit ? Coef<R>::uim(P, p) : Coef<R>::dim(P, p)) : R(0);
    }
    // coefficients of the register bits (direction depends on the amplitude)
    R ur_r[RB], ui_r[RB], dr_r[RB], di_r[RB];
#pragma unroll
    for (int k = 0; k < RB; ++k) {
        const int p = hpos + SB + k - c;
        const bool ok = SB + k >= c;
        ur_r[k] = ok ? Coef<R>::ure(P, p) : R(0);
        ui_r[k] = ok ? Coef<R>::uim(P, p) : R(0);
        dr_r[k] = ok ? Coef<R>::dre(P, p) : R(0);
        di_r[k] = ok ? Coef<R>::dim(P, p) : R(0);
    }
    const double su = A.su_dev ? *A.su_dev : A.su;
    const double sp = (EPI == EPI_LANCZOS && A.up) ? (A.sp_dev ? *A.sp_dev : A.sp) : 0.0;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    C *outp = reinterpret_cast<C *>(A.out);
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;

    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t base = ((t & ((int64_t(1) << lowbits) - 1)) << c) |
                             ((t >> lowbits) << (hpos + g));
        C v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int64_t l = tid + a * NT;
            v[a] = u[base + (l & cmask) + ((l >> c) << hpos)];
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) tile[tid + a * NT] = v[a];
        __syncthreads();
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int l = tid + a * NT;
            const int64_t x = base + (l & cmask) + ((int64_t)(l >> c) << hpos);
            R ar = R(0), ai = R(0);
#pragma unroll
            for (int k = 0; k < SB; ++k) {
                if (k < c) continue;  // uniform: chunk bits were applied by pass L
                const C w = tile[l ^ (1 << k)];
                if (REALC) {
                    ar = fmar(cr_s[k], w.x, ar);
                    ai = fmar(cr_s[k], w.y, ai);
                } else {
                    ar = fmar(cr_s[k], w.x, fmar(-ci_s[k], w.y, ar));
                    ai = fmar(cr_s[k], w.y, fmar(ci_s[k], w.x, ai));
                }
            }
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                if (SB + k < c) continue;
                const C w = v[a ^ (1 << k)];
                const bool bit = (a >> k) & 1;
                const R cr = bit ? ur_r[k] : dr_r[k];
                if (REALC) {
                    ar = fmar(cr, w.x, ar);
                    ai = fmar(cr, w.y, ai);
                } else {
                    const R ci = bit ? ui_r[k] : di_r[k];
                    ar = fmar(cr, w.x, fmar(-ci, w.y, ar));
                    ai = fmar(cr, w.y, fmar(ci, w.x, ai));
                }
            }
            // bits beyond both tiles (very large registers): partner from global memory
            for (int p = P.xb_lo; p < P.xb_hi; ++p) {
                const C w = u[x ^ (int64_t(1) << p)];
                flip_acc<R, REALC>(P, p, (x >> p) & 1, w, ar, ai);
            }
            const C part = outp[x];
            const double hr = su * (double(part.x) + double(ar));
            const double hi = su * (double(part.y) + double(ai));
            epilogue<C, EPI>(A, x, hr, hi, su * double(v[a].x), su * double(v[a].y), sp, red);
        }
        __syncthreads();
    }
    write_partials<EPI>(A, red, red_scr);
}

}  // namespace emusv
