// Multi-pass fused H*psi for large registers (sm_100a), TMA-staged, three tiles in flight.
//
// H = D + sum_p (coefficient x flip of bit p).  Every flip is applied on chip, split over
// streaming passes so that each amplitude is read from HBM once per pass:
//
//  pass L  tile = 2^TB consecutive amplitudes (bits 0..TB-1), brought into shared memory
//          by one cp.async.bulk per tile.  The diagonal (detunings + C6/r^6 interactions)
//          is rebuilt from per-thread / per-tile FP64 partial energies.  Output: the
//          partial sum (or H v when no bit is left).
//  pass H  tile = 2^c contiguous amplitudes (the c low bits, done by pass L) x 2^g
//          combinations of g higher bits, gathered by a 5-D TMA tensor-map load (rows of
//          32 B or more).  Adds the flips of those bits to the partial sum (also
//          TMA-staged) and runs the epilogue (partial, store, Lanczos FP64 reductions).
//          Registers with more than TB + (TB - c) qubits take two H passes.
//
// Both kernels are templated on a thread-block-cluster size (PB, PBH bits) whose sibling
// CTAs would serve the next bits from distributed shared memory; the library instantiates
// PB = PBH = 0 only, because on B200 the per-element DSMEM loads made both passes about
// twice as slow as one more streaming pass.
//
// Each pass keeps SL (SH) = 3 tile buffers in flight: the load of tile i+2 is issued when
// tile i starts computing.  mbarrier waits are bounded (about 2 s of clock): on a timeout
// the kernel records status EMUSV_TIMEOUT in *A.err, skips the arithmetic and keeps taking
// part in the block barriers so that no thread is left waiting.
//
// Register blocking: each of the NT = 2^(TB-RB) threads owns NA = 2^RB amplitudes that
// differ in the RB highest tile bits, so those flips are register-register; the other
// tile bits are one shared-memory load per flip at a compile-time offset.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "common.cuh"

namespace emusv {

enum PassEpi {
    EPI_PARTIAL = 0,  // store the partial sum (another pass follows)
    EPI_STORE = 1,    // store H v
    EPI_LANCZOS = 2,  // store H v; FP64 partials ||Hv||^2, <v,Hv>
    // flips of the pass's group bits only, unscaled (the Lanczos iteration's pass H, which
    // runs before its pass L): out = X u (first pass, no partial-sum input) or
    // out = part + X u; FP64 partials of <u, X u> (0 re, 1 im)
    EPI_X_FIRST = 3,
    EPI_X_ADD = 4,
};
template <int EPI> __host__ __device__ constexpr bool epi_has_part() { return EPI != EPI_X_FIRST; }
template <int EPI> __host__ __device__ constexpr bool epi_reduces() {
    return EPI == EPI_LANCZOS || EPI == EPI_X_FIRST || EPI == EPI_X_ADD;
}

constexpr int PBMAX_ALL = 3;  // largest cluster (2^3 CTAs) either pass uses

struct PassParams {
    int n;
    int real_coef;
    // coefficients by bit position: "up" = target bit 1, "dn" = target bit 0
    float fup_re[MAXQ], fup_im[MAXQ], fdn_re[MAXQ], fdn_im[MAXQ];
    double dup_re[MAXQ], dup_im[MAXQ], ddn_re[MAXQ], ddn_im[MAXQ];
    double field[MAXQ];
    double U[MAXQ * MAXQ];
    double ER[32];  // energies of the register-bit patterns of pass L (fields + pairs)
    float ERf[32];  // the same, rounded to FP32 (complex64 path)
    int pb;         // pass L: cluster bits (cluster size 2^pb)
    int hc, hg;     // pass H: chunk bits c and group bits g
    int hpos;       // pass H: global position of the first group bit
    int pbh;        // pass H: cluster bits (positions hpos+hg .. hpos+hg+pbh-1)
    int hbox_rows;  // pass H: group rows per TMA box (<= 256)
    int hskip;      // pass H: group bits below this position were applied by pass L
    double dc_re, dc_im, dg_im;  // noise term of the diagonal (HamParams)
};

struct PassArgs {
    const void *u;          // stored input vector (raw); v = su * u
    const double *su_dev;   // device scale (or null: su)
    double su;
    void *out;              // partial / final output
    double *partials;       // [gridDim.x * NRED]
    const int *gate;        // kernel returns at once when *gate != 0
    int *err;               // receives EMUSV_TIMEOUT when a bounded wait gives up
    const double *eshift;   // pass L: if non-null, the diagonal is taken minus *eshift
};

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t cluster_addr(const void *smem_ptr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(smem_ptr)), "r"(rank));
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
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait (a few seconds of SM clock); false on timeout.  The clock is read once
// per 1024 polls so that waiting warps do not crowd the issue slots.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023u) == 0 && clock64() - t0 > 4000000000LL) return false;
    }
}
// 1-D bulk copy global -> own shared memory, completion on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Bulk prefetch of global memory into the L2 (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// 5-D tiled tensor-map load (no multicast), completion on `bar`.
__device__ __forceinline__ void tmap_load5(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                           int c3, int c4, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
          "r"(smem_u32(bar))
        : "memory");
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

// Complex accumulator of the flip terms.  complex64 uses Blackwell's packed FP32x2 FMA
// (one instruction per real coefficient and amplitude); complex128 uses two DFMA.
__device__ __forceinline__ unsigned long long pk2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

template <typename R> struct Acc;
template <> struct Acc<float> {
    unsigned long long a = 0ull;
    __device__ __forceinline__ void real(float c, const float2 &w) { a = fma2(pk2(c, c), pk2(w.x, w.y), a); }
    __device__ __forceinline__ void cplx(float cr, float ci, const float2 &w) {
        a = fma2(pk2(cr, cr), pk2(w.x, w.y), a);
        a = fma2(pk2(-ci, ci), pk2(w.y, w.x), a);
    }
    __device__ __forceinline__ double re() const { return double(upk2(a).x); }
    __device__ __forceinline__ double im() const { return double(upk2(a).y); }
    // a += d * w (real d)
    __device__ __forceinline__ void diag(float d, const float2 &w) { a = fma2(pk2(d, d), pk2(w.x, w.y), a); }
};
template <> struct Acc<double> {
    double r = 0.0, i = 0.0;
    __device__ __forceinline__ void real(double c, const double2 &w) {
        r = fma(c, w.x, r);
        i = fma(c, w.y, i);
    }
    __device__ __forceinline__ void cplx(double cr, double ci, const double2 &w) {
        r = fma(cr, w.x, fma(-ci, w.y, r));
        i = fma(cr, w.y, fma(ci, w.x, i));
    }
    __device__ __forceinline__ double re() const { return r; }
    __device__ __forceinline__ double im() const { return i; }
};

// acc += c * w  with c = up (bit==1) or dn (bit==0) of bit position p (compile-time p:
// the coefficient comes from the constant bank).
template <typename R, bool REALC, typename C>
__device__ __forceinline__ void flip_acc(const PassParams &P, int p, bool bit, const C &w, Acc<R> &acc) {
    if (REALC) {
        acc.real(Coef<R>::ure(P, p), w);
    } else {
        acc.cplx(bit ? Coef<R>::ure(P, p) : Coef<R>::dre(P, p), bit ? Coef<R>::uim(P, p) : Coef<R>::dim(P, p), w);
    }
}
template <typename R, bool REALC, typename C>
__device__ __forceinline__ void flip_reg(R cr, R ci, const C &w, Acc<R> &acc) {
    if (REALC) acc.real(cr, w);
    else acc.cplx(cr, ci, w);
}

template <int EPI>
__device__ __forceinline__ void write_partials(const PassArgs &A, double (&red)[NRED], double *scratch) {
    if (!epi_reduces<EPI>()) return;
    block_sum<NRED>(red, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NRED; ++k) A.partials[(int64_t)blockIdx.x * NRED + k] = red[k];
    }
}

__device__ __forceinline__ void report_timeout(const PassArgs &A) {
    if (A.err) atomicExch(A.err, (int)EMUSV_TIMEOUT);
}

// ------------------------------------------------------------------------- pass L
// Shared memory: 2 tiles | mbarriers | U (padded rows) | field | per-tile scalars x2 | scratch
constexpr int UPAD = MAXQ + 1;  // row stride of the shared U table (no bank conflicts)
constexpr int SL = 3;           // pass L pipeline stages (tiles in flight per CTA)
constexpr int SH = 3;           // pass H pipeline stages

template <typename C, int TB>
__host__ __device__ constexpr size_t pass_low_smem() {
    return SL * (sizeof(C) << TB) + 8 * SL + sizeof(double) * (MAXQ * UPAD + MAXQ + SL * 64 + 8 * NRED);
}

// NOISY: the diagonal has the imaginary part dc_im + dg_im * popcount(x) (noise term).
template <typename R, bool REALC, int TB, int RB, int EPI, int PB, bool NOISY = false>
__global__ void __launch_bounds__(1 << (TB - RB), 2)
k_pass_low(const PassParams P, PassArgs A) {
    const double eshift = A.eshift ? *A.eshift : 0.0;
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    constexpr uint32_t TILE_BYTES = sizeof(C) << TB;
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(128) unsigned char smem_pass[];
    C *tiles = reinterpret_cast<C *>(smem_pass);                      // [SL][2^TB]
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_pass + SL * TILE_BYTES);  // [SL]
    double *Ush = reinterpret_cast<double *>(smem_pass + SL * TILE_BYTES + 8 * SL);
    double *fld = Ush + MAXQ * UPAD;
    double *scal = fld + MAXQ;       // [SL][64]: crossT[SB] crossR[RB] eh
    double *red_scr = scal + SL * 64;

    const int n = P.n;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t rank = PB ? cluster_rank() : 0;
    const int64_t nsuper = int64_t(1) << (n - TB - PB);
    const int nclusters = gridDim.x >> PB;
    const int cid = blockIdx.x >> PB;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    C *__restrict__ out = reinterpret_cast<C *>(A.out);

    for (int k = tid; k < MAXQ * MAXQ; k += NT) Ush[(k / MAXQ) * UPAD + (k % MAXQ)] = P.U[k];
    for (int k = tid; k < MAXQ; k += NT) fld[k] = P.field[k];
    if (tid == 0) {
        for (int b = 0; b < SL; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // prologue: the first SL-1 tiles of this CTA
    if (tid == 0) {
        for (int b = 0; b < SL - 1; ++b) {
            const int64_t s0 = cid + (int64_t)b * nclusters;
            if (s0 >= nsuper) break;
            mbar_expect_tx(&bars[b], TILE_BYTES);
            bulk_load(tiles + ((int64_t)b << TB), u + (((s0 << PB) | rank) << TB), TILE_BYTES, &bars[b]);
        }
    }

    bool ok = true;

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
    // sibling CTAs and the coefficients of the cluster bits (fixed per CTA)
    uint32_t raddr[PB > 0 ? PB : 1];
    R ccr[PB > 0 ? PB : 1], cci[PB > 0 ? PB : 1];
#pragma unroll
    for (int r = 0; r < PB; ++r) {
        raddr[r] = cluster_addr(tiles, rank ^ (1u << r)) + (uint32_t)(tid * sizeof(C));
        const bool bit = (rank >> r) & 1;
        ccr[r] = bit ? Coef<R>::ure(P, TB + r) : Coef<R>::dre(P, TB + r);
        cci[r] = bit ? Coef<R>::uim(P, TB + r) : Coef<R>::dim(P, TB + r);
    }
    const double su = A.su_dev ? *A.su_dev : A.su;
    const float suf = float(su);
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;

    int it = 0, buf = 0;
    uint32_t phase = 0;
    for (int64_t s = cid; s < nsuper; s += nclusters, ++it) {
        const int64_t base = ((s << PB) | rank) << TB;
        C *tile = tiles + ((int64_t)buf << TB);
        double *sc = scal + buf * 64;
        if (warp == 0) {
            // energy of the tile's high bits and their crosses with the tile bits
            double e = 0.0;
            for (int p = TB + lane; p < n; p += 32) {
                if (!((base >> p) & 1)) continue;
                e += fld[p];
                for (int p2 = p + 1; p2 < n; ++p2)
                    if ((base >> p2) & 1) e += Ush[p * UPAD + p2];
            }
            e = warp_sum(e);
            if (lane == 0) sc[TB] = e - eshift + P.dc_re;
            if (lane < TB) {
                double cx = 0.0;
                for (int p = TB; p < n; ++p)
                    if ((base >> p) & 1) cx += Ush[lane * UPAD + p];
                sc[lane] = cx;  // crossT[0..SB) then crossR[0..RB)
            }
        }
        if (ok && !mbar_wait(&bars[buf], phase)) {
            ok = false;
            report_timeout(A);
        }
        // every CTA of the cluster has its tile; everyone is done with the previous buffer
        if (PB) cluster_sync_all(); else __syncthreads();
        {
            const int64_t sn = s + (int64_t)(SL - 1) * nclusters;  // refill the freed buffer
            const int nbuf = buf == 0 ? SL - 1 : buf - 1;
            if (tid == 0 && sn < nsuper && ok) {
                mbar_expect_tx(&bars[nbuf], TILE_BYTES);
                bulk_load(tiles + ((int64_t)nbuf << TB), u + (((sn << PB) | rank) << TB), TILE_BYTES,
                          &bars[nbuf]);
            }
        }
        if (ok) {
            double St = ET + sc[TB];
#pragma unroll
            for (int k = 0; k < SB; ++k)
                if ((tid >> k) & 1) St += sc[k];
            double hR[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) hR[k] = fR[k] + sc[SB + k];
            // FP32 copies (complex64 path): one rounding per tile and thread
            const float Stf = float(St);
            float hRf[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) hRf[k] = float(hR[k]);
            float rf[3] = {0.f, 0.f, 0.f};
            const uint32_t boff = (uint32_t)buf * TILE_BYTES;
            C v[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] = tile[tid + a * NT];
            C *out_t = out + base + tid;
            // noise: imaginary diagonal of x = base + tid + a*NT (disjoint bit fields)
            const double dI0 = NOISY ? P.dc_im + P.dg_im * double(__popcll((unsigned long long)base) +
                                                                  __popc((unsigned)tid))
                                     : 0.0;
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int l = tid + a * NT;
                Acc<R> acc;
#pragma unroll
                for (int k = 0; k < SB; ++k)  // thread bits: partner in shared memory
                    flip_acc<R, REALC>(P, k, (tid >> k) & 1, tile[l ^ (1 << k)], acc);
#pragma unroll
                for (int k = 0; k < RB; ++k)  // register bits
                    flip_acc<R, REALC>(P, SB + k, (a >> k) & 1, v[a ^ (1 << k)], acc);
#pragma unroll
                for (int r = 0; r < PB; ++r)  // cluster bits: sibling CTA's tile
                    flip_reg<R, REALC>(ccr[r], cci[r],
                                       ld_cluster(raddr[r] + boff + (uint32_t)(a * NT * sizeof(C)),
                                                  (const C *)nullptr), acc);
                if constexpr (std::is_same<R, float>::value) {
                    // complex64: all per-amplitude arithmetic in FP32 / packed FP32x2 (the
                    // FP64 <-> FP32 conversions would bound the kernel on the XU pipe)
                    float d = Stf + P.ERf[a];
#pragma unroll
                    for (int k = 0; k < RB; ++k)
                        if ((a >> k) & 1) d += hRf[k];
                    acc.diag(d, v[a]);
                    if (NOISY) {  // + i dI v
                        const float dI = float(dI0 + P.dg_im * double(__popc((unsigned)a)));
                        acc.a = fma2(pk2(-dI, dI), pk2(v[a].y, v[a].x), acc.a);
                    }
                    const float2 t = upk2(acc.a);
                    if (EPI == EPI_PARTIAL) {
                        out_t[a * NT] = t;  // unscaled partial; pass H applies su
                    } else {
                        const float2 h = make_float2(suf * t.x, suf * t.y);
                        out_t[a * NT] = h;
                        if (EPI == EPI_LANCZOS) {
                            rf[0] = fmaf(h.x, h.x, fmaf(h.y, h.y, rf[0]));
                            rf[1] = fmaf(v[a].x, h.x, fmaf(v[a].y, h.y, rf[1]));
                            rf[2] = fmaf(v[a].x, h.y, fmaf(-v[a].y, h.x, rf[2]));
                        }
                    }
                } else {
                    double d = St + P.ER[a];
#pragma unroll
                    for (int k = 0; k < RB; ++k)
                        if ((a >> k) & 1) d += hR[k];
                    const double ur = double(v[a].x), ui = double(v[a].y);
                    double tr = acc.re() + d * ur, ti = acc.im() + d * ui;
                    if (NOISY) {
                        const double dI = dI0 + P.dg_im * double(__popc((unsigned)a));
                        tr -= dI * ui;
                        ti += dI * ur;
                    }
                    if (EPI == EPI_PARTIAL) {
                        out_t[a * NT] = cmake<C>(tr, ti);  // unscaled partial; pass H applies su
                    } else {
                        const double hr = su * tr, hi = su * ti;
                        out_t[a * NT] = cmake<C>(hr, hi);
                        if (EPI == EPI_LANCZOS) {
                            const double vr = su * ur, vi = su * ui;
                            red[0] += hr * hr + hi * hi;
                            red[1] += vr * hr + vi * hi;
                            red[2] += vr * hi - vi * hr;
                        }
                    }
                }
            }
            if constexpr (std::is_same<R, float>::value) {
                if (EPI == EPI_LANCZOS) {  // per-tile FP32 partial sums -> FP64 accumulators
                    red[0] += double(rf[0]);
                    red[1] += su * double(rf[1]);
                    red[2] += su * double(rf[2]);
                }
            }
        }
        if (++buf == SL) {
            buf = 0;
            phase ^= 1u;
        }
    }
    // no CTA may leave while a sibling can still read its shared memory
    if (PB) cluster_sync_all();
    write_partials<EPI>(A, red, red_scr);
}

// ------------------------------------------------------------------------- pass H
// Tile local index l = (j << c) | i, i < 2^c (contiguous low bits, applied by pass L),
// j < 2^g (group bits hpos..hpos+g-1).  A cluster of 2^pbh CTAs holds the tiles that
// differ in bits hpos+g..hpos+g+pbh-1.  The thread owns l = tid + a*NT;
// x = base + (l & cmask) + ((l >> c) << hpos).  Group bits below P.hskip (already applied
// by pass L when the group overlaps the pass-L tile) are skipped.
// Tensor map (8-byte elements, dims innermost first): [2^c*K, 2^(hpos-c), 2^g, 2^pbh, rest]
// with K = sizeof(C)/8.
template <typename C, int TB, bool HASPART = true>
__host__ __device__ constexpr size_t pass_high_smem() {
    return (HASPART ? 2 : 1) * SH * (sizeof(C) << TB) + 8 * SH + sizeof(double) * 8 * NRED;
}

struct PassHighMaps {
    CUtensorMap u;     // input vector
    CUtensorMap part;  // partial sums of pass L
};

// CT: chunk bits c (compile time); PBH: cluster bits.  CHUNKF (EPI_X_FIRST / EPI_X_ADD of
// the Lanczos iteration): the pass also applies the flips of the chunk bits 0..c-1 (the
// partners lie in the tile's rows) and counts them in <u, X u>; the recurrence pass L
// then leaves those bits out.
template <typename R, bool REALC, int TB, int RB, int EPI, int CT, int PBH, bool CHUNKF = false>
__global__ void __launch_bounds__(1 << (TB - RB), 1)
k_pass_high(const PassParams P, PassArgs A, const __grid_constant__ PassHighMaps M) {
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    constexpr uint32_t TILE_BYTES = sizeof(C) << TB;
    constexpr bool HASPART = epi_has_part<EPI>();
    constexpr int NBUF = HASPART ? 2 : 1;
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(128) unsigned char smem_pass[];
    C *tiles = reinterpret_cast<C *>(smem_pass);  // [SH][2^TB] values, then [SH][2^TB] partials
    C *parts = tiles + ((int64_t)SH << TB);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_pass + NBUF * SH * TILE_BYTES);
    double *red_scr = reinterpret_cast<double *>(smem_pass + NBUF * SH * TILE_BYTES + 8 * SH);
    static_assert(CT >= 1 && CT <= TB - RB, "chunk bits must lie below the register bits");
    const int n = P.n, hpos = P.hpos;
    constexpr int c = CT, g = TB - CT;
    const int tid = threadIdx.x;
    const int64_t cmask = (int64_t(1) << c) - 1;
    const int lowbits = hpos - c;
    const int64_t lowmask = (int64_t(1) << lowbits) - 1;
    const int cpos = hpos + g;  // first cluster bit
    const uint32_t rank = PBH ? cluster_rank() : 0;
    const int64_t nsuper = int64_t(1) << (n - c - g - PBH);
    const int nclusters = gridDim.x >> PBH;
    const int cid = blockIdx.x >> PBH;
    const int rows = P.hbox_rows, nbox = (1 << g) / rows;
    const uint32_t box_bytes = TILE_BYTES / nbox;

    if (tid == 0) {
        for (int b = 0; b < SH; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // TMA loads of super-tile s into buffer buf (coordinates per the layouts above)
    auto issue = [&](int64_t s, int buf) {
        const int slo = (int)(s & lowmask);
        const int shi = (int)(s >> lowbits);
        mbar_expect_tx(&bars[buf], NBUF * TILE_BYTES);
        for (int b = 0; b < nbox; ++b) {
            unsigned char *dv = reinterpret_cast<unsigned char *>(tiles + ((int64_t)buf << TB)) + b * box_bytes;
            tmap_load5(dv, &M.u, 0, slo, b * rows, (int)rank, shi, &bars[buf]);
            if (HASPART) {
                unsigned char *dp =
                    reinterpret_cast<unsigned char *>(parts + ((int64_t)buf << TB)) + b * box_bytes;
                tmap_load5(dp, &M.part, 0, slo, b * rows, (int)rank, shi, &bars[buf]);
            }
        }
    };
    if (tid == 0) {
        for (int b = 0; b < SH - 1; ++b) {
            const int64_t s0 = cid + (int64_t)b * nclusters;
            if (s0 >= nsuper) break;
            issue(s0, b);
        }
    }

    uint32_t raddr[PBH > 0 ? PBH : 1];
    R ccr[PBH > 0 ? PBH : 1], cci[PBH > 0 ? PBH : 1];
#pragma unroll
    for (int r = 0; r < PBH; ++r) {
        raddr[r] = cluster_addr(tiles, rank ^ (1u << r)) + (uint32_t)(tid * sizeof(C));
        const bool bit = (rank >> r) & 1;
        ccr[r] = bit ? Coef<R>::ure(P, cpos + r) : Coef<R>::dre(P, cpos + r);
        cci[r] = bit ? Coef<R>::uim(P, cpos + r) : Coef<R>::dim(P, cpos + r);
    }
    // tile bits whose flips this pass applies: group bits at or above P.hskip
    uint32_t apply = CHUNKF ? (1u << c) - 1u : 0u;
    for (int k = c; k < TB; ++k)
        if (hpos + k - c >= P.hskip) apply |= 1u << k;
    // coefficients of the shared-memory bits (direction fixed by the thread's own bits);
    // tile bit k < c is bit k of x, tile bit k >= c is bit hpos + k - c
    R cr_s[SB], ci_s[SB];
#pragma unroll
    for (int k = 0; k < SB; ++k) {
        const int p = k < c ? k : hpos + k - c;
        const bool okk = k >= c || CHUNKF;
        const bool bit = (tid >> k) & 1;
        cr_s[k] = okk ? (bit ? Coef<R>::ure(P, p) : Coef<R>::dre(P, p)) : R(0);
        ci_s[k] = okk ? (bit ? Coef<R>::uim(P, p) : Coef<R>::dim(P, p)) : R(0);
    }
    // coefficients of the register bits (direction depends on the amplitude)
    R ur_r[RB], ui_r[RB], dr_r[RB], di_r[RB];
#pragma unroll
    for (int k = 0; k < RB; ++k) {
        const int p = hpos + SB + k - c;
        const bool okk = SB + k >= c;
        ur_r[k] = okk ? Coef<R>::ure(P, p) : R(0);
        ui_r[k] = okk ? Coef<R>::uim(P, p) : R(0);
        dr_r[k] = okk ? Coef<R>::dre(P, p) : R(0);
        di_r[k] = okk ? Coef<R>::dim(P, p) : R(0);
    }
    const double su = A.su_dev ? *A.su_dev : A.su;
    const float suf = float(su);
    C *__restrict__ outp = reinterpret_cast<C *>(A.out);
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;
    bool ok = true;
    // x offset of amplitude a of this thread: (tid & cmask) + ((tid + a*NT) >> c) << hpos
    const int64_t xt = (tid & cmask) + ((int64_t)(tid >> c) << hpos);
    const int ash = hpos + SB - c;  // c <= SB: the x offset of amplitude a is a << ash

    int it = 0, buf = 0;
    uint32_t phase = 0;
    for (int64_t s = cid; s < nsuper; s += nclusters, ++it) {
        const int64_t base = ((s & lowmask) << c) | ((int64_t)rank << cpos) |
                             ((s >> lowbits) << (cpos + PBH));
        const C *tile = tiles + ((int64_t)buf << TB);
        const C *ptile = parts + ((int64_t)buf << TB);
        if (ok && !mbar_wait(&bars[buf], phase)) {
            ok = false;
            report_timeout(A);
        }
        if (PBH) cluster_sync_all(); else __syncthreads();
        {
            const int64_t sn = s + (int64_t)(SH - 1) * nclusters;  // refill the freed buffer
            if (tid == 0 && sn < nsuper && ok) issue(sn, buf == 0 ? SH - 1 : buf - 1);
        }
        if (ok) {
            const uint32_t boff = (uint32_t)buf * TILE_BYTES;
            float rf[3] = {0.f, 0.f, 0.f};
            C v[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] = tile[tid + a * NT];
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int l = tid + a * NT;
                const int64_t x = base + xt + ((int64_t)a << ash);
                Acc<R> acc;
#pragma unroll
                for (int k = 0; k < SB; ++k) {
                    if (k < c && !CHUNKF) continue;  // chunk bits were applied by pass L
                    if (!((apply >> k) & 1)) continue;
                    flip_reg<R, REALC>(cr_s[k], ci_s[k], tile[l ^ (1 << k)], acc);
                }
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    if (!((apply >> (SB + k)) & 1)) continue;
                    const bool bit = (a >> k) & 1;
                    flip_reg<R, REALC>(bit ? ur_r[k] : dr_r[k], bit ? ui_r[k] : di_r[k],
                                       v[a ^ (1 << k)], acc);
                }
#pragma unroll
                for (int r = 0; r < PBH; ++r)  // cluster bits: sibling CTA's tile
                    flip_reg<R, REALC>(ccr[r], cci[r],
                                       ld_cluster(raddr[r] + boff + (uint32_t)(a * NT * sizeof(C)),
                                                  (const C *)nullptr), acc);
                const C pt = HASPART ? ptile[l] : cmake<C>(0.0, 0.0);
                if (EPI == EPI_X_FIRST || EPI == EPI_X_ADD) {  // unscaled X u; <u, X u>
                    if constexpr (std::is_same<R, float>::value) {
                        const float2 t = upk2(acc.a);
                        outp[x] = HASPART ? make_float2(pt.x + t.x, pt.y + t.y) : t;
                        rf[0] = fmaf(v[a].x, t.x, fmaf(v[a].y, t.y, rf[0]));
                        rf[1] = fmaf(v[a].x, t.y, fmaf(-v[a].y, t.x, rf[1]));
                    } else {
                        const double tr = acc.re(), ti = acc.im();
                        outp[x] = HASPART ? cmake<C>(double(pt.x) + tr, double(pt.y) + ti) : cmake<C>(tr, ti);
                        const double vr = double(v[a].x), vi = double(v[a].y);
                        red[0] += vr * tr + vi * ti;
                        red[1] += vr * ti - vi * tr;
                    }
                } else if (EPI == EPI_PARTIAL) {  // another pass follows: unscaled running sum
                    if constexpr (std::is_same<R, float>::value) {
                        const float2 t = upk2(acc.a);
                        outp[x] = make_float2(pt.x + t.x, pt.y + t.y);
                    } else {
                        outp[x] = cmake<C>(double(pt.x) + acc.re(), double(pt.y) + acc.im());
                    }
                } else if constexpr (std::is_same<R, float>::value) {
                    const float2 t = upk2(acc.a);
                    const float2 h = make_float2(suf * (pt.x + t.x), suf * (pt.y + t.y));
                    outp[x] = h;
                    if (EPI == EPI_LANCZOS) {
                        rf[0] = fmaf(h.x, h.x, fmaf(h.y, h.y, rf[0]));
                        rf[1] = fmaf(v[a].x, h.x, fmaf(v[a].y, h.y, rf[1]));
                        rf[2] = fmaf(v[a].x, h.y, fmaf(-v[a].y, h.x, rf[2]));
                    }
                } else {
                    const double hr = su * (double(pt.x) + acc.re());
                    const double hi = su * (double(pt.y) + acc.im());
                    outp[x] = cmake<C>(hr, hi);
                    if (EPI == EPI_LANCZOS) {
                        const double vr = su * double(v[a].x), vi = su * double(v[a].y);
                        red[0] += hr * hr + hi * hi;
                        red[1] += vr * hr + vi * hi;
                        red[2] += vr * hi - vi * hr;
                    }
                }
            }
            if constexpr (std::is_same<R, float>::value) {
                if (EPI == EPI_LANCZOS) {  // per-tile FP32 partial sums -> FP64 accumulators
                    red[0] += double(rf[0]);
                    red[1] += su * double(rf[1]);
                    red[2] += su * double(rf[2]);
                }
                if (EPI == EPI_X_FIRST || EPI == EPI_X_ADD) {
                    red[0] += double(rf[0]);
                    red[1] += double(rf[1]);
                }
            }
        }
        if (++buf == SH) {
            buf = 0;
            phase ^= 1u;
        }
    }
    if (PBH) cluster_sync_all();
    write_partials<EPI>(A, red, red_scr);
}


// ------------------------------------------------ fused two-group pass H (persistent)
// The two strided passes over the bits above the pass-L tile of a large register, in ONE
// persistent launch, so that the second group reads its inputs from the L2:
//  * group 1: tiles of the chunk bits [0, c) x the g bits [hs, hs + g) (hs = the pass-L
//    tile width), applying the flips of the bits [hs, hpos2): part = X_1 u;
//  * group 2: tiles of the chunk bits x the top g bits [hpos2, n) (hpos2 = n - g), applying
//    those flips and the chunk bits': part = part + X_2 u.
// A "super-tile" is a value of the bits [c, hs): it is both a union of 2^(n-hs-g) group-1
// tiles (tile index: the bits [hs + g, n)) and of as many group-2 tiles (bits [hs, hpos2)),
// so a group-2 tile needs exactly the group-1 tiles of its super-tile (2^(c + n - hs)
// amplitudes: 2 MB of complex64 at N = 26).  Items run in one order: the
// group-1 stream first by LAG items, then the two streams alternate, then the rest of the
// group-2 stream; CTAs take the next item from a global counter when they prefetch it.
// Ordering: the CTA adds a group-1 tile to its super-tile's counter after the next tile's
// block barrier, thread 0 fencing first (cumulative over the block's stores that the
// barrier ordered before it).  A group-2 tile's intermediate sums are loaded by tensor map
// after an acquire of that counter and a proxy fence: at prefetch time if the counter is
// already complete, else when the tile is computed (a bounded wait, about 2 s of clock,
// then EMUSV_TIMEOUT in *A.err).  Waits happen only when computing, only on tiles taken
// earlier, so they end.
constexpr int HH_MAX_NS_BITS = 10;  // super-tiles of the fused pass H: at most 2^10
constexpr int HH_LAG = 512;         // group-1 items ahead of the first group-2 item
constexpr int HH_CNT_WORDS = (1 << HH_MAX_NS_BITS) + 1;
struct HHArgs {
    const void *u;        // stored v (unscaled)
    void *part;           // the sums (written by group 1, completed by group 2)
    double *partials;     // [gridDim.x * NRED]: <u, X u> of the applied bits (0 re, 1 im)
    const int *gate;
    int *err;
    unsigned *cnt;        // [2^ns_bits + 1]: group-1 tiles done per super-tile, then the
                          // item counter; zero at launch (HH_CNT_WORDS words at most)
    int hs, hpos2, ns_bits, tps_bits;
};
struct PassHHMaps {
    CUtensorMap u1;  // input, group-1 layout (hpos = hs)
    CUtensorMap u2;  // input, group-2 layout (hpos = hpos2)
    CUtensorMap p2;  // intermediate sums, group-2 layout
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

template <typename C, int TB>
__host__ __device__ constexpr size_t pass_hh_smem() {
    return 2 * SH * (sizeof(C) << TB) + 16 * SH + 16 * SH + sizeof(double) * 8 * NRED;
}

template <typename R, bool REALC, int TB, int RB, int CT>
__global__ void __launch_bounds__(1 << (TB - RB), 1)
k_pass_hh(const PassParams P, HHArgs A, const __grid_constant__ PassHHMaps M) {
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB;
    constexpr uint32_t TILE_BYTES = sizeof(C) << TB;
    constexpr int c = CT, g = TB - CT;
    static_assert(CT >= 1 && CT <= TB - RB, "chunk bits must lie below the register bits");
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(128) unsigned char smem_pass[];
    C *tiles = reinterpret_cast<C *>(smem_pass);  // [SH][2^TB] u
    C *parts = tiles + ((int64_t)SH << TB);       // [SH][2^TB] intermediate sums (group 2)
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_pass + 2 * SH * TILE_BYTES);  // [SH] u
    uint64_t *pbars = bars + SH;                                                       // [SH] sums
    int64_t *ring = reinterpret_cast<int64_t *>(pbars + SH);  // [SH] item in each buffer
    int *defer = reinterpret_cast<int *>(ring + SH);           // [SH] sums not loaded yet
    double *red_scr = reinterpret_cast<double *>(smem_pass + 2 * SH * TILE_BYTES + 32 * SH);
    const int tid = threadIdx.x;
    const int nsb = A.ns_bits, tb = A.tps_bits;
    const int64_t TPS = int64_t(1) << tb, NT1 = int64_t(1) << (nsb + tb);
    const int64_t nitems = 2 * NT1;
    const int64_t LAG = NT1 < HH_LAG ? NT1 : HH_LAG;
    const int rows = P.hbox_rows, nbox = (1 << g) / rows;
    const uint32_t box_bytes = TILE_BYTES / nbox;
    const int64_t cmask = (int64_t(1) << c) - 1;
    unsigned *next_item = A.cnt + (int64_t(1) << nsb);

    // item q -> (group 1 or 2, super-tile s, tile t within it)
    auto decode = [&](int64_t q, int &grp, int64_t &s, int64_t &t) {
        int64_t i;
        if (q < LAG) {
            grp = 1;
            i = q;
        } else {
            const int64_t r = q - LAG;
            if (r < 2 * (NT1 - LAG)) {
                grp = (r & 1) ? 1 : 2;
                i = (r & 1) ? LAG + (r >> 1) : (r >> 1);
            } else {
                grp = 2;
                i = (NT1 - LAG) + (r - 2 * (NT1 - LAG));
            }
        }
        s = i >> tb;
        t = i & (TPS - 1);
    };
    auto load_sums = [&](int64_t s, int64_t t, int buf) {
        fence_proxy_async_global();
        mbar_expect_tx(&pbars[buf], TILE_BYTES);
        const int slo = (int)(s | (t << nsb));
        for (int b = 0; b < nbox; ++b) {
            unsigned char *dp = reinterpret_cast<unsigned char *>(parts + ((int64_t)buf << TB)) + b * box_bytes;
            tmap_load5(dp, &M.p2, 0, slo, b * rows, 0, 0, &pbars[buf]);
        }
    };
    // take item q into buffer buf and start its loads (thread 0, never blocks); the item
    // numbers come from the global counter one tile ahead of their use
    auto take = [&](int buf, int64_t q) {
        ring[buf] = q;
        defer[buf] = 0;
        if (q >= nitems) return;
        int grp;
        int64_t s, t;
        decode(q, grp, s, t);
        mbar_expect_tx(&bars[buf], TILE_BYTES);
        for (int b = 0; b < nbox; ++b) {
            unsigned char *dv = reinterpret_cast<unsigned char *>(tiles + ((int64_t)buf << TB)) + b * box_bytes;
            if (grp == 1) tmap_load5(dv, &M.u1, 0, (int)s, b * rows, 0, (int)t, &bars[buf]);
            else tmap_load5(dv, &M.u2, 0, (int)(s | (t << nsb)), b * rows, 0, 0, &bars[buf]);
        }
        if (grp == 2) {
            if (ld_acquire_u32(A.cnt + s) >= (unsigned)TPS) load_sums(s, t, buf);
            else defer[buf] = 1;
        }
    };

    if (tid == 0) {
        for (int b = 0; b < SH; ++b) {
            mbar_init(&bars[b], 1);
            mbar_init(&pbars[b], 1);
        }
        fence_mbar_init();
        for (int b = 0; b < SH - 1; ++b) take(b, (int64_t)atomicAdd(next_item, 1u));
    }
    // thread 0: the item number for the next take, requested a tile ahead
    unsigned next_q = tid == 0 ? atomicAdd(next_item, 1u) : 0u;
    __syncthreads();
    bool ok = true;
    C *__restrict__ outp = reinterpret_cast<C *>(A.part);
    double red[2] = {0.0, 0.0};
    int64_t pend = -1;  // super-tile of the last group-1 tile, counted after the next barrier
    int buf = 0;
    uint32_t vph = 0, pph = 0;  // mbarrier phase bits per buffer
    for (;;) {
        const int64_t q = ring[buf];
        if (q >= nitems) break;
        int grp;
        int64_t s, t;
        decode(q, grp, s, t);
        const int hpos = grp == 1 ? A.hs : A.hpos2;
        const C *tile = tiles + ((int64_t)buf << TB);
        const C *ptile = parts + ((int64_t)buf << TB);
        if (ok && !mbar_wait(&bars[buf], (vph >> buf) & 1u)) {
            ok = false;
            if (A.err) atomicExch(A.err, (int)EMUSV_TIMEOUT);
        }
        vph ^= 1u << buf;
        // the tile is here; everyone is done with the previous buffer and has issued the
        // previous tile's stores
        __syncthreads();
        // warp 1 counts the previous group-1 tile (its fence waits for the block's stores)
        // while thread 0 takes the next item, so the two serial chains overlap
        if (tid == 32 && pend >= 0) {
            __threadfence();
            atomicAdd(A.cnt + pend, 1u);
        }
        pend = -1;
        if (tid == 0) {
            const int64_t qt = (int64_t)next_q;
            if (ok && qt < nitems) next_q = atomicAdd(next_item, 1u);
            if (ok) take(buf == 0 ? SH - 1 : buf - 1, qt);
            else ring[buf == 0 ? SH - 1 : buf - 1] = nitems;
            if (grp == 2 && defer[buf]) {  // group 1 of this super-tile was not done at take
                bool got = ok;
                const long long t0 = clock64();
                while (got && ld_acquire_u32(A.cnt + s) < (unsigned)TPS) {
                    __nanosleep(64);
                    if (clock64() - t0 > 4000000000LL || (A.err && *(volatile int *)A.err)) {
                        got = false;
                        if (A.err) atomicExch(A.err, (int)EMUSV_TIMEOUT);
                    }
                }
                if (got) {
                    load_sums(s, t, buf);
                } else {
                    ok = false;
                    mbar_expect_tx(&pbars[buf], 0);  // release the waiters: nothing will arrive
                }
            }
        }
        if (grp == 2) {
            if (!mbar_wait(&pbars[buf], (pph >> buf) & 1u)) {
                ok = false;
                if (A.err) atomicExch(A.err, (int)EMUSV_TIMEOUT);
            }
            pph ^= 1u << buf;
        }
        if (A.err && *(volatile int *)A.err) ok = false;
        // the tile's work, compiled once per group (GRP 1 or 2) so that the group tests
        // leave the amplitude loop
        auto work = [&](auto grp_c) {
            constexpr int GRP = decltype(grp_c)::value;
            // this group's geometry: tile bit k < c is bit k of x, k >= c bit hpos + k - c;
            // applied: group 1 the bits [hs, hpos2), group 2 all its bits and the chunk bits
            uint32_t apply = GRP == 2 ? (1u << c) - 1u : 0u;
            for (int k = c; k < TB; ++k)
                if (GRP == 2 || hpos + k - c < A.hpos2) apply |= 1u << k;
            R cr_s[SB], ci_s[SB];
#pragma unroll
            for (int k = 0; k < SB; ++k) {
                const int p = k < c ? k : hpos + k - c;
                const bool bit = (tid >> k) & 1;
                const bool on = (apply >> k) & 1;
                cr_s[k] = on ? (bit ? Coef<R>::ure(P, p) : Coef<R>::dre(P, p)) : R(0);
                ci_s[k] = on ? (bit ? Coef<R>::uim(P, p) : Coef<R>::dim(P, p)) : R(0);
            }
            R ur_r[RB], ui_r[RB], dr_r[RB], di_r[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                const int p = hpos + SB + k - c;
                const bool on = (apply >> (SB + k)) & 1;
                ur_r[k] = on ? Coef<R>::ure(P, p) : R(0);
                ui_r[k] = on ? Coef<R>::uim(P, p) : R(0);
                dr_r[k] = on ? Coef<R>::dre(P, p) : R(0);
                di_r[k] = on ? Coef<R>::dim(P, p) : R(0);
            }
            const int64_t base = GRP == 1 ? ((s << c) | (t << (hpos + g))) : ((s | (t << nsb)) << c);
            const int64_t xt = (tid & cmask) + ((int64_t)(tid >> c) << hpos);
            const int ash = hpos + SB - c;
            float rf[2] = {0.f, 0.f};  // complex64: per-tile FP32 sums
            (void)rf;
            C v[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] = tile[tid + a * NT];
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int l = tid + a * NT;
                const int64_t x = base + xt + ((int64_t)a << ash);
                Acc<R> acc;
#pragma unroll
                for (int k = 0; k < SB; ++k) {
                    if (!((apply >> k) & 1)) continue;
                    flip_reg<R, REALC>(cr_s[k], ci_s[k], tile[l ^ (1 << k)], acc);
                }
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    if (!((apply >> (SB + k)) & 1)) continue;
                    const bool bit = (a >> k) & 1;
                    flip_reg<R, REALC>(bit ? ur_r[k] : dr_r[k], bit ? ui_r[k] : di_r[k], v[a ^ (1 << k)], acc);
                }
                if constexpr (std::is_same<R, float>::value) {
                    const float2 tt = upk2(acc.a);
                    if constexpr (GRP == 2) {
                        const C pt = ptile[l];
                        outp[x] = make_float2(pt.x + tt.x, pt.y + tt.y);
                    } else {
                        outp[x] = tt;
                    }
                    rf[0] = fmaf(v[a].x, tt.x, fmaf(v[a].y, tt.y, rf[0]));
                    rf[1] = fmaf(v[a].x, tt.y, fmaf(-v[a].y, tt.x, rf[1]));
                } else {
                    const double tr = acc.re(), ti = acc.im();
                    if constexpr (GRP == 2) {
                        const C pt = ptile[l];
                        outp[x] = cmake<C>(double(pt.x) + tr, double(pt.y) + ti);
                    } else {
                        outp[x] = cmake<C>(tr, ti);
                    }
                    const double vr = double(v[a].x), vi = double(v[a].y);
                    red[0] += vr * tr + vi * ti;
                    red[1] += vr * ti - vi * tr;
                }
            }
            if constexpr (std::is_same<R, float>::value) {
                red[0] += double(rf[0]);
                red[1] += double(rf[1]);
            }
        };
        if (ok) {
            if (grp == 1) work(std::integral_constant<int, 1>{});
            else work(std::integral_constant<int, 2>{});
            if (grp == 1) pend = s;  // counted after the next block barrier
        }
        if (++buf == SH) buf = 0;
    }
    __syncthreads();
    if (tid == 0 && pend >= 0) {
        __threadfence();
        atomicAdd(A.cnt + pend, 1u);
    }
    double rr[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) rr[k] = k < 2 ? red[k] : 0.0;
    block_sum<NRED>(rr, red_scr);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NRED; ++k) A.partials[(int64_t)blockIdx.x * NRED + k] = rr[k];
    }
}

// ------------------------------------------------------------- Lanczos pass L
// The last pass of the Lanczos iteration (after the pass H kernels in EPI_X_FIRST /
// EPI_X_ADD mode wrote part = X_high u_j, the flips of every bit above the tile, unscaled):
// per tile of 2^TB consecutive amplitudes (bits 0..TB-1)
//    H v_j = su_j ((D - sigma) u_j + X_low u_j + part)            (formed on chip only)
//    w     = H v_j - (a_j su_j) u_j - (b_j su_{j-1}) u_{j-1}        (stored: u_{j+1})
// with FP64 partials 0 ||w||^2, 1-2 <v_j, w>, 3 ||(H - sigma) v_j||^2 and 4 the part of the
// NEXT iteration's <w, (H - sigma) w> that this tile can see, Re <w, (D - sigma + X_low) w>
// (w is written into a shared-memory buffer whose flips are applied one tile later, after
// the next tile's block barrier, so the pass keeps one barrier per tile).  The flips of
// the higher bits of <w, H w> come from the next iteration's pass H, which reads w anyway.
// X_low is the flips of tile bits C0..TB-1: the pass H kernels apply the flips of bits
// 0..C0-1 (their rows' chunk bits) and count them in <v, H v>.
// E0: the start of a run: no recurrence, partials 4-5 = <u, (D - sigma + X_low) u>.
// u_j arrives by cp.async.bulk into SL stages; part and u_{j-1} are read with streaming
// loads one tile ahead into registers, after a bulk L2 prefetch two tiles ahead.  The
// per-tile scalars of the diagonal (energy of the bits above the tile and their crosses
// with the tile bits) are computed one tile ahead by all warps, one value per warp.
// block_sum scratch: (threads / 32) * NRED doubles, up to 512 threads
constexpr int LZ_MAX_THREADS = 512;
template <typename C, int TB>
__host__ __device__ constexpr size_t pass_lz_smem() {
    return (SL + 2) * (sizeof(C) << TB) + 8 * SL +
           sizeof(double) * (MAXQ * UPAD + MAXQ + SL * 64 + (LZ_MAX_THREADS / 32) * NRED);
}

template <typename C> __device__ __forceinline__ C ldcs_c(const C *p) { return __ldcs(p); }

// (hr, hi) = acc + d v, in the accumulator's own precision (packed FP32x2 for complex64)
template <typename R, typename C>
__device__ __forceinline__ void acc_diag_parts(Acc<R> &acc, R d, const C &v, R &hr, R &hi) {
    if constexpr (std::is_same<R, float>::value) {
        acc.diag(d, v);
        const float2 t = upk2(acc.a);
        hr = t.x;
        hi = t.y;
    } else {
        hr = fma(d, v.x, acc.r);
        hi = fma(d, v.y, acc.i);
    }
}

// Scalars of the tile at `base` (TB + 1 values into sc: crosses sum_{p >= TB, x_p = 1}
// U[q][p] for q < TB, then the energy of the bits above the tile minus sigma), value i by
// warp i mod NW, the high bits over the lanes.
template <int TB>
__device__ __forceinline__ void lz_tile_scalars(int64_t base, int n, const double *fld, const double *Ush,
                                                double sigma, double *sc, int warp, int lane, int nw) {
    const int p = TB + lane;
    const bool on = p < n && ((base >> p) & 1);
    for (int i = warp; i <= TB; i += nw) {
        double v = 0.0;
        if (on) {
            if (i < TB) {
                v = Ush[i * UPAD + p];
            } else {
                v = fld[p];
                for (int p2 = p + 1; p2 < n; ++p2)
                    if ((base >> p2) & 1) v += Ush[p * UPAD + p2];
            }
        }
        v = warp_sum(v);
        if (lane == 0) sc[i] = i == TB ? v - sigma : v;
    }
}

// Modes of k_pass_lz: the recurrence pass of a Lanczos iteration; the start-of-run energy
// pass; and the moments of H (emusv_expect): H u = (D + X_low) u + part formed per tile
// (no store), partials 0 ||H u||^2, 1-2 <u, H u>.
enum LzMode { LZ_ITER = 0, LZ_E0 = 1, LZ_M2 = 2 };

// C0: bits 0..C0-1 are flipped (and counted in <v, H v>) by the pass H kernels.
template <typename R, bool REALC, int TB, int RB, int MODE, int C0>
__global__ void __launch_bounds__(1 << (TB - RB), (sizeof(R) == 4) ? 2 : 1)
k_pass_lz(const PassParams P, LzArgs A) {
    constexpr bool E0 = MODE == LZ_E0, M2 = MODE == LZ_M2;
    typedef typename cvec<R>::T C;
    constexpr int SB = TB - RB, NT = 1 << SB, NA = 1 << RB, NW = NT / 32;
    constexpr uint32_t TILE_BYTES = sizeof(C) << TB;
    constexpr bool F32 = std::is_same<R, float>::value;
    static_assert(NT <= LZ_MAX_THREADS, "block_sum scratch is sized for LZ_MAX_THREADS");
    if (A.gate && *A.gate != 0) return;
    extern __shared__ __align__(128) unsigned char smem_pass[];
    C *tiles = reinterpret_cast<C *>(smem_pass);               // [SL][2^TB]: u_j
    C *wsm = tiles + ((int64_t)SL << TB);                      // [2][2^TB]: w
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_pass + (SL + 2) * TILE_BYTES);
    double *Ush = reinterpret_cast<double *>(smem_pass + (SL + 2) * TILE_BYTES + 8 * SL);
    double *fld = Ush + MAXQ * UPAD;
    double *scal = fld + MAXQ;  // [SL][64]: crossT[SB] crossR[RB] eh
    double *red_scr = scal + SL * 64;

    const int n = P.n;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int64_t ntiles = int64_t(1) << (n - TB);
    const int64_t grid = gridDim.x;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    const C *__restrict__ part = reinterpret_cast<const C *>(A.part);
    const C *__restrict__ up = reinterpret_cast<const C *>(A.up);
    C *__restrict__ out = reinterpret_cast<C *>(A.out);

    for (int k = tid; k < MAXQ * MAXQ; k += NT) Ush[(k / MAXQ) * UPAD + (k % MAXQ)] = P.U[k];
    for (int k = tid; k < MAXQ; k += NT) fld[k] = P.field[k];
    if (tid == 0) {
        for (int b = 0; b < SL; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    const double sigma = A.eshift ? *A.eshift : 0.0;
    __syncthreads();
    if (tid == 0) {
        for (int b = 0; b < SL - 1; ++b) {
            const int64_t s0 = blockIdx.x + (int64_t)b * grid;
            if (s0 >= ntiles) break;
            mbar_expect_tx(&bars[b], TILE_BYTES);
            bulk_load(tiles + ((int64_t)b << TB), u + (s0 << TB), TILE_BYTES, &bars[b]);
            if (!E0 && b == 0) {  // the loop's L2 prefetch runs two tiles ahead: tile 1 here
                const int64_t s2 = s0 + grid;
                if (s2 < ntiles) {
                    bulk_prefetch_l2(part + (s2 << TB), TILE_BYTES);
                    if (up) bulk_prefetch_l2(up + (s2 << TB), TILE_BYTES);
                }
            }
        }
    }
    // scalars of the first tile (visible after the loop's first barrier)
    if ((int64_t)blockIdx.x < ntiles)
        lz_tile_scalars<TB>((int64_t)blockIdx.x << TB, n, fld, Ush, sigma, scal, warp, lane, NW);
    double su = 1.0, car = 0.0, cai = 0.0, cb = 0.0;
    if (MODE == LZ_ITER) {
        su = *A.su;
        car = A.ocoef[0];
        cai = A.ocoef[1];
        cb = up ? A.ocoef[2] : 0.0;
    }
    const R suR = R(su), carR = R(car), caiR = R(cai), cbR = R(cb);

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
    double red[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) red[k] = 0.0;

    // part and u_{j-1} of the next tile, in flight while the current one is computed
    C pn[NA], qn[NA];
    auto prefetch = [&](int64_t s) {
        const int64_t b0 = (s << TB) + tid;
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            pn[a] = ldcs_c(part + b0 + a * NT);
            qn[a] = up ? ldcs_c(up + b0 + a * NT) : cmake<C>(0.0, 0.0);
        }
    };
    // w of the previous tile (own amplitudes) and its shifted diagonal, for the energy
    C wp[NA];
    R dp[NA];
    // Re <w, (D - sigma + X_low) w> of the tile held in wsm[wbuf]
    // (lane bits and register bits: the flip sums; warp bits: the pair form
    // <w, X_p w> = 2 Re sum_{x: bit p = 0} conj(w[x]) dn_p w[x ^ 2^p] of a Hermitian flip,
    // read by the warps whose bit p is 0; bits below c0 are the pass H kernels')
    constexpr int LB = SB < 5 ? SB : 5;  // lane bits
    auto tile_energy = [&](int wbuf) {
        const C *wt = wsm + ((int64_t)wbuf << TB);
        R e = R(0);
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            const int l = tid + a * NT;
            Acc<R> acc;
#pragma unroll
            for (int k = C0; k < LB; ++k)
                flip_acc<R, REALC>(P, k, (tid >> k) & 1, wt[l ^ (1 << k)], acc);
#pragma unroll
            for (int k = 0; k < RB; ++k)
                flip_acc<R, REALC>(P, SB + k, (a >> k) & 1, wp[a ^ (1 << k)], acc);
            R fr, fi;
            acc_diag_parts<R>(acc, dp[a], wp[a], fr, fi);
            e += R(wp[a].x) * fr + R(wp[a].y) * fi;
        }
        R pr = R(0);
#pragma unroll
        for (int k = (C0 > 5 ? C0 : 5); k < SB; ++k) {
            if ((tid >> k) & 1) continue;  // uniform in the warp
            const R cr = Coef<R>::dre(P, k), ci = REALC ? R(0) : Coef<R>::dim(P, k);
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const C q = wt[(tid ^ (1 << k)) + a * NT];
                const R wr = wp[a].x, wi = wp[a].y;
                // Re(conj(w) (cr + i ci) q) = cr (wr qr + wi qi) - ci (wr qi - wi qr)
                pr += cr * (wr * R(q.x) + wi * R(q.y));
                if (!REALC) pr -= ci * (wr * R(q.y) - wi * R(q.x));
            }
        }
        e += R(2) * pr;
        red[4] += double(e);
    };

    bool ok = true, have_prev = false;
    int buf = 0, wb = 0;
    uint32_t phase = 0;
    if (!E0 && (int64_t)blockIdx.x < ntiles) prefetch(blockIdx.x);
    for (int64_t s = blockIdx.x; s < ntiles; s += grid) {
        const int64_t base = s << TB;
        C *tile = tiles + ((int64_t)buf << TB);
        const double *sc = scal + buf * 64;
        if (ok && !mbar_wait(&bars[buf], phase)) {
            ok = false;
            if (A.err) atomicExch(A.err, (int)EMUSV_TIMEOUT);
        }
        // the tile and its scalars are visible; everyone is done with the previous tile's
        // u buffer and with the w buffer written two tiles ago
        __syncthreads();
        const int nbuf = buf == 0 ? SL - 1 : buf - 1;
        if (tid == 0 && ok) {
            const int64_t sn = s + (int64_t)(SL - 1) * grid;  // refill the freed buffer
            if (sn < ntiles) {
                mbar_expect_tx(&bars[nbuf], TILE_BYTES);
                bulk_load(tiles + ((int64_t)nbuf << TB), u + (sn << TB), TILE_BYTES, &bars[nbuf]);
            }
            const int64_t s2 = s + 2 * grid;
            if (!E0 && s2 < ntiles) {
                bulk_prefetch_l2(part + (s2 << TB), TILE_BYTES);
                if (up) bulk_prefetch_l2(up + (s2 << TB), TILE_BYTES);
            }
        }
        {  // scalars of the next tile into the slot after this one
            const int64_t s1 = s + grid;
            const int b1 = buf + 1 == SL ? 0 : buf + 1;
            if (s1 < ntiles) lz_tile_scalars<TB>(s1 << TB, n, fld, Ush, sigma, scal + b1 * 64, warp, lane, NW);
        }
        if (MODE == LZ_ITER && have_prev && ok) tile_energy(wb ^ 1);
        if (ok) {
            double St = ET + sc[TB];
#pragma unroll
            for (int k = 0; k < SB; ++k)
                if ((tid >> k) & 1) St += sc[k];
            double hR[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) hR[k] = fR[k] + sc[SB + k];
            const R StR = R(St);
            R hRR[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) hRR[k] = R(hR[k]);
            C pc[NA], qc[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                pc[a] = pn[a];
                qc[a] = qn[a];
            }
            C v[NA];
#pragma unroll
            for (int a = 0; a < NA; ++a) v[a] = tile[tid + a * NT];
            R rq[4] = {R(0), R(0), R(0), R(0)};  // ||w||^2, <u_j, w> re/im, ||Hv||^2 (tile sums)
            C *wt = wsm + ((int64_t)wb << TB);
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                const int l = tid + a * NT;
                Acc<R> acc;
#pragma unroll
                for (int k = C0; k < SB; ++k)  // thread bits: partner in shared memory
                    flip_acc<R, REALC>(P, k, (tid >> k) & 1, tile[l ^ (1 << k)], acc);
#pragma unroll
                for (int k = 0; k < RB; ++k)  // register bits
                    flip_acc<R, REALC>(P, SB + k, (a >> k) & 1, v[a ^ (1 << k)], acc);
                R d = StR + (F32 ? R(P.ERf[a]) : R(P.ER[a]));
#pragma unroll
                for (int k = 0; k < RB; ++k)
                    if ((a >> k) & 1) d += hRR[k];
                const R vr = v[a].x, vi = v[a].y;
                R hur, hui;
                acc_diag_parts<R>(acc, d, v[a], hur, hui);
                if (E0) {  // <u, (D - sigma + X_low) u>
                    rq[0] += vr * hur + vi * hui;
                    rq[1] += vr * hui - vi * hur;
                    continue;
                }
                if (M2) {  // H u = (D + X_low) u + part: ||H u||^2, <u, H u>
                    const R hr = hur + R(pc[a].x), hi = hui + R(pc[a].y);
                    rq[0] += hr * hr + hi * hi;
                    rq[1] += vr * hr + vi * hi;
                    rq[2] += vr * hi - vi * hr;
                    continue;
                }
                const R hr = suR * (hur + R(pc[a].x)), hi = suR * (hui + R(pc[a].y));
                const R wr = hr - (carR * vr - caiR * vi) - cbR * R(qc[a].x);
                const R wi = hi - (carR * vi + caiR * vr) - cbR * R(qc[a].y);
                const C o = cmake<C>(wr, wi);
                out[base + l] = o;
                wt[l] = o;
                wp[a] = o;
                dp[a] = d;
                const R orr = o.x, oi = o.y;
                rq[0] += orr * orr + oi * oi;
                rq[1] += vr * orr + vi * oi;  // <u_j, w>
                rq[2] += vr * oi - vi * orr;
                rq[3] += hr * hr + hi * hi;
            }
            if (E0) {
                red[4] += double(rq[0]);
                red[5] += double(rq[1]);
            } else if (M2) {
                red[0] += double(rq[0]);
                red[1] += double(rq[1]);
                red[2] += double(rq[2]);
                const int64_t s1 = s + grid;
                if (s1 < ntiles) prefetch(s1);
            } else {
                red[0] += double(rq[0]);
                red[1] += su * double(rq[1]);
                red[2] += su * double(rq[2]);
                red[3] += double(rq[3]);
                const int64_t s1 = s + grid;
                if (s1 < ntiles) prefetch(s1);
            }
        }
        have_prev = true;
        wb ^= 1;
        if (++buf == SL) {
            buf = 0;
            phase ^= 1u;
        }
    }
    if (MODE == LZ_ITER) {
        __syncthreads();  // the last tile's w buffer is complete
        if (have_prev && ok) tile_energy(wb ^ 1);
    }
    block_sum<NRED>(red, red_scr);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NRED; ++k) A.partials[(int64_t)blockIdx.x * NRED + k] = red[k];
    }
}

}  // namespace emusv
