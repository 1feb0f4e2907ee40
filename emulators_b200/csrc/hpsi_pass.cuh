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
    int hc, hg;     // pass H: chunk bits c and group bits g
    int hpos;       // pass H: global position of the first group bit
    int pbh;        // pass H: cluster bits (positions hpos+hg .. hpos+hg+pbh-1)
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
    const void *part;       // pass H: partial sum written by pass L (null: in place in out)
    double *partials;       // [gridDim.x * NRED]
    const int *gate;        // kernel returns at once when *gate != 0
};

// Map a local shared-memory address to the same offset in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_addr(const void *smem_ptr, uint32_t rank) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem_ptr);
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ float2 ld_cluster(uint32_t addr, const float2 *) {
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ double2 ld_cluster(uint32_t addr, const double2 *) {
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr));
    return v;
}

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

// Epilogue shared by both passes: store h; Lanczos reductions with v and vp = sp * up[x].
template <typename C, int EPI>
__device__ __forceinline__ void epilogue(C *__restrict__ out, const C *__restrict__ upv, int64_t x,
                                         double hr, double hi, double vr, double vi, double sp,
                                         double (&red)[NRED]) {
    out[x] = cmake<C>(hr, hi);
    if (EPI == EPI_LANCZOS) {
        red[0] += hr * hr + hi * hi;
        red[1] += vr * hr + vi * hi;
        red[2] += vr * hi - vi * hr;
        if (upv) {
            const C q = upv[x];
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

constexpr int PBMAX_ALL = 3;  // largest cluster (2^3 CTAs) either pass uses

// ------------------------------------------------------------------------- pass L
// Shared memory: tile [2^TB] | U [MAXQ*MAXQ] | field [MAXQ] | per-tile scalars | scratch
template <typename C, int TB>
__host__ __device__ constexpr size_t pass_low_smem() {
    return (sizeof(C) << TB) + sizeof(double) * (MAXQ * MAXQ + MAXQ + 64 + 8 * NRED);
}

template <typename R, bool REALC, int TB, int RB, int EPI>
__global__ void __launch_bounds__(1 << (TB - RB), 2)
k_pass_low(const PassParams P, PassArgs A) {
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    C *tile = reinterpret_cast<C *>(smem);
    double *Ush = reinterpret_cast<double *>(smem + (sizeof(C) << TB));
    double *fld = Ush + MAXQ * MAXQ;
    double *crossT = fld + MAXQ;     // [SB] then crossR [RB] (lanes < TB)
    double *crossR = crossT + SB;
    double *eh = crossT + TB;
    double *red_scr = crossT + 64;

    const int n = P.n, pb = P.pb;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < MAXQ * MAXQ; k += NT) Ush[k] = P.U[k];
    for (int k = tid; k < MAXQ; k += NT) fld[k] = P.field[k];
    uint32_t rank = 0;
    if (pb) asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    // sibling tiles and the coefficients of the cluster bits (fixed per CTA)
    uint32_t raddr[PBMAX_ALL];
    R ccr[PBMAX_ALL], cci[PBMAX_ALL];
#pragma unroll
    for (int r = 0; r < PBMAX_ALL; ++r) {
        raddr[r] = 0;
        ccr[r] = cci[r] = R(0);
        if (r < pb) {
            raddr[r] = cluster_addr(tile, rank ^ (1u << r));
            const bool bit = (rank >> r) & 1;
            ccr[r] = bit ? Coef<R>::ure(P, TB + r) : Coef<R>::dre(P, TB + r);
            cci[r] = bit ? Coef<R>::uim(P, TB + r) : Coef<R>::dim(P, TB + r);
        }
    }
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
        double sacc = 0.0;
#pragma unroll
        for (int q = 0; q < SB; ++q)
            if ((tid >> q) & 1) sacc += P.U[(SB + k) * MAXQ + q];
        fR[k] = sacc;
    }
    __syncthreads();

    const double su = A.su_dev ? *A.su_dev : A.su;
    const bool has_up = EPI == EPI_LANCZOS && A.up != nullptr;
    const double sp = has_up ? (A.sp_dev ? *A.sp_dev : A.sp) : 0.0;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    const C *__restrict__ upv = reinterpret_cast<const C *>(A.up);
    C *__restrict__ out = reinterpret_cast<C *>(A.out);
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;

    const int64_t nsuper = int64_t(1) << (n - TB - pb);
    const int nclusters = gridDim.x >> pb;
    const int cid = blockIdx.x >> pb;
    for (int64_t s = cid; s < nsuper; s += nclusters) {
        const int64_t base = ((s << pb) | rank) << TB;
        C v[NA];
#pragma unroll
        for (int a = 0; a < NA; ++a) v[a] = u[base + tid + a * NT];
        if (warp == 0) {
            // energy of the tile's high bits and their crosses with the tile bits
            double e = 0.0;
            for (int p = TB + lane; p < n; p += 32) {
                if (!((base >> p) & 1)) continue;
                e += fld[p];
                for (int p2 = p + 1; p2 < n; ++p2)
                    if ((base >> p2) & 1) e += Ush[p * MAXQ + p2];
            }
            e = warp_sum(e);
            if (lane == 0) eh[0] = e;
            if (lane < TB) {
                double cx = 0.0;
                for (int p = TB; p < n; ++p)
                    if ((base >> p) & 1) cx += Ush[lane * MAXQ + p];
                crossT[lane] = cx;  // lanes >= SB land in crossR
            }
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) tile[tid + a * NT] = v[a];
        if (pb) {
            asm volatile("barrier.cluster.arrive.release.aligned;\n"
                         "barrier.cluster.wait.acquire.aligned;" ::: "memory");
        } else {
            __syncthreads();
        }
        double St = ET + eh[0];
#pragma unroll
        for (int k = 0; k < SB; ++k)
            if ((tid >> k) & 1) St += crossT[k];
        double hR[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k) hR[k] = fR[k] + crossR[k];

#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int l = tid + a * NT;
            R ar = R(0), ai = R(0);
#pragma unroll
            for (int k = 0; k < SB; ++k)  // thread bits: partner in shared memory
                flip_acc<R, REALC>(P, k, (tid >> k) & 1, tile[l ^ (1 << k)], ar, ai);
#pragma unroll
            for (int k = 0; k < RB; ++k)  // register bits
                flip_acc<R, REALC>(P, SB + k, (a >> k) & 1, v[a ^ (1 << k)], ar, ai);
#pragma unroll
            for (int r = 0; r < PBMAX_ALL; ++r) {  // cluster bits: sibling CTA's tile
                if (r < pb) {
                    const C w = ld_cluster(raddr[r] + (uint32_t)(l * sizeof(C)), (const C *)nullptr);
                    if (REALC) {
                        ar = fmar(ccr[r], w.x, ar);
                        ai = fmar(ccr[r], w.y, ai);
                    } else {
                        ar = fmar(ccr[r], w.x, fmar(-cci[r], w.y, ar));
                        ai = fmar(ccr[r], w.y, fmar(cci[r], w.x, ai));
                    }
                }
            }
            double d = St + P.ER[a];
#pragma unroll
            for (int k = 0; k < RB; ++k)
                if ((a >> k) & 1) d += hR[k];
            const int64_t x = base + l;
            const double ur = double(v[a].x), ui = double(v[a].y);
            const double tr = double(ar) + d * ur, ti = double(ai) + d * ui;
            if (EPI == EPI_PARTIAL)
                out[x] = cmake<C>(tr, ti);  // unscaled partial; pass H applies su
            else
                epilogue<C, EPI>(out, has_up ? upv : nullptr, x, su * tr, su * ti, su * ur, su * ui,
                                 sp, red);
        }
        if (pb) {
            asm volatile("barrier.cluster.arrive.release.aligned;\n"
                         "barrier.cluster.wait.acquire.aligned;" ::: "memory");
        } else {
            __syncthreads();
        }
    }
    write_partials<EPI>(A, red, red_scr);
}

// ------------------------------------------------------------------------- pass H
// Tile local index l = (j << c) | i, i < 2^c (contiguous low bits, applied by pass L),
// j < 2^g (group bits hpos..hpos+g-1).  A cluster of 2^pbh CTAs holds the tiles that
// differ in bits hpos+g..hpos+g+pbh-1.  The thread owns l = tid + a*NT;
// x = base + (l & cmask) + ((l >> c) << hpos).
template <typename C, int TB>
__host__ __device__ constexpr size_t pass_high_smem() {
    return (sizeof(C) << TB) + sizeof(double) * 8 * NRED;
}

template <typename R, bool REALC, int TB, int RB, int EPI, bool INPL>
__global__ void __launch_bounds__(1 << (TB - RB), 2)
k_pass_high(const PassParams P, PassArgs A) {
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    C *tile = reinterpret_cast<C *>(smem);
    double *red_scr = reinterpret_cast<double *>(smem + (sizeof(C) << TB));
    const int n = P.n, c = P.hc, g = P.hg, hpos = P.hpos, pbh = P.pbh;
    const int tid = threadIdx.x;
    const int64_t cmask = (int64_t(1) << c) - 1;
    const int lowbits = hpos - c;
    const int64_t lowmask = (int64_t(1) << lowbits) - 1;
    const int cpos = hpos + g;  // first cluster bit

    uint32_t rank = 0;
    if (pbh) asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    uint32_t raddr[PBMAX_ALL];
    R ccr[PBMAX_ALL], cci[PBMAX_ALL];
#pragma unroll
    for (int r = 0; r < PBMAX_ALL; ++r) {
        raddr[r] = 0;
        ccr[r] = cci[r] = R(0);
        if (r < pbh) {
            raddr[r] = cluster_addr(tile, rank ^ (1u << r));
            const bool bit = (rank >> r) & 1;
            ccr[r] = bit ? Coef<R>::ure(P, cpos + r) : Coef<R>::dre(P, cpos + r);
            cci[r] = bit ? Coef<R>::uim(P, cpos + r) : Coef<R>::dim(P, cpos + r);
        }
    }
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
    const bool has_up = EPI == EPI_LANCZOS && A.up != nullptr;
    const double sp = has_up ? (A.sp_dev ? *A.sp_dev : A.sp) : 0.0;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    const C *__restrict__ upv = reinterpret_cast<const C *>(A.up);
    C *__restrict__ outp = reinterpret_cast<C *>(A.out);
    // INPL: the partial sum is read from `out` itself (all loads of a tile are issued
    // before its stores); otherwise from a separate buffer.
    const C *__restrict__ partp = reinterpret_cast<const C *>(INPL ? A.out : A.part);
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;

    const int64_t nsuper = int64_t(1) << (n - c - g - pbh);
    const int nclusters = gridDim.x >> pbh;
    const int cid = blockIdx.x >> pbh;
    for (int64_t s = cid; s < nsuper; s += nclusters) {
        const int64_t base = ((s & lowmask) << c) | ((int64_t)rank << cpos) |
                             ((s >> lowbits) << (cpos + pbh));
        C v[NA], part[INPL ? NA : 1];
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int64_t l = tid + a * NT;
            const int64_t x = base + (l & cmask) + ((l >> c) << hpos);
            v[a] = u[x];
            if (INPL) part[a] = partp[x];
        }
#pragma unroll
        for (int a = 0; a < NA; ++a) tile[tid + a * NT] = v[a];
        if (pbh) {
            asm volatile("barrier.cluster.arrive.release.aligned;\n"
                         "barrier.cluster.wait.acquire.aligned;" ::: "memory");
        } else {
            __syncthreads();
        }
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
#pragma unroll
            for (int r = 0; r < PBMAX_ALL; ++r) {  // cluster bits: sibling CTA's tile
                if (r < pbh) {
                    const C w = ld_cluster(raddr[r] + (uint32_t)(l * sizeof(C)), (const C *)nullptr);
                    if (REALC) {
                        ar = fmar(ccr[r], w.x, ar);
                        ai = fmar(ccr[r], w.y, ai);
                    } else {
                        ar = fmar(ccr[r], w.x, fmar(-cci[r], w.y, ar));
                        ai = fmar(ccr[r], w.y, fmar(cci[r], w.x, ai));
                    }
                }
            }
            // bits beyond the tiles and the cluster (very large registers): global partner
            for (int p = P.xb_lo; p < P.xb_hi; ++p) {
                const C w = u[x ^ (int64_t(1) << p)];
                flip_acc<R, REALC>(P, p, (x >> p) & 1, w, ar, ai);
            }
            const C pt = INPL ? part[INPL ? a : 0] : partp[x];
            const double hr = su * (double(pt.x) + double(ar));
            const double hi = su * (double(pt.y) + double(ai));
            epilogue<C, EPI>(outp, has_up ? upv : nullptr, x, hr, hi, su * double(v[a].x),
                             su * double(v[a].y), sp, red);
        }
        if (pbh) {
            asm volatile("barrier.cluster.arrive.release.aligned;\n"
                         "barrier.cluster.wait.acquire.aligned;" ::: "memory");
        } else {
            __syncthreads();
        }
    }
    write_partials<EPI>(A, red, red_scr);
}

}  // namespace emusv
