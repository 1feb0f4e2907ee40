// Fused H*psi for the Rydberg Hamiltonian (sm_100a).
//
// One pass over the state: every output amplitude gets the diagonal term (detunings and
// C6/r^6 interactions, rebuilt on chip) plus the N single-qubit flip terms.
//
// Layout: the state is processed in tiles of 2^b consecutive amplitudes (the b low bits,
// i.e. the last b qubits).  A tile is staged in shared memory with coalesced loads, so
// flips of the b low bits read shared memory; flips of bits >= b read the partner
// amplitude from global memory (coalesced across a warp; the L2 serves the recently
// touched partners).  The diagonal of an amplitude x = (base | l) is
//   E_high(base) + E_low[l] + G1[l & 63] + G2[l >> 6]
// where E_low is a per-CTA table over the low bits, E_high the energy of the tile's
// high bits and G1/G2 the low-bit x high-bit cross terms of that tile, so the
// O(N^2) interaction sum costs four shared-memory reads per amplitude.
#pragma once

#include "common.cuh"

namespace emusv {

enum HpsiMode {
    HP_STORE = 0,    // out = H v
    HP_ENERGY = 1,   // no store; <v,Hv>, ||Hv||^2
    HP_LANCZOS = 2,  // out = H v; ||Hv||^2, <v,Hv>, <vp,Hv>, <v,vp>
    HP_DIAG = 3      // out (float64) = diag
};

struct HpsiArgs {
    const void *u;     // input (stored) vector; v = su * u
    double su;
    const double *su_dev;     // if non-null, su is read from here (device scalar)
    const void *up;    // previous Lanczos vector (HP_LANCZOS, may be null); vp = sp * up
    double sp;
    const double *sp_dev;
    void *out;
    double *partials;  // [gridDim.x * NRED]
    int tile_bits;
    const int *gate;   // if non-null and *gate != 0 the kernel returns at once
    void *part_buf;    // two-pass H*psi: buffer for the partial sums of pass L
    int *err;          // device word receiving EMUSV_TIMEOUT if a bounded wait gives up
    const double *eshift;  // HP_LANCZOS, HP_STORE: if non-null, the diagonal is taken minus *eshift
};

// Arguments of the Lanczos iteration's pass L (k_pass_lz in hpsi_pass.cuh).
struct LzArgs {
    const void *u;         // stored v_j (v_j = su u_j)
    const void *part;      // X_high u_j (unscaled); null with E0
    const void *up;        // stored v_{j-1}, or null
    void *out;             // w (stored form of v_{j+1})
    const double *su;      // device scale of v_j
    const double *ocoef;   // device [3]: a_re su_j, a_im su_j, b su_{j-1}
    const double *eshift;  // device sigma, or null
    double *partials;      // [gridDim.x * NRED]
    const int *gate;
    int *err;
};

struct SmemLayout {
    size_t tile, elow, g1, g2, coef, ush, gv, red, total;
};

template <typename C>
__host__ __device__ inline SmemLayout hpsi_smem(int b) {
    SmemLayout L;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += (bytes + 15) & ~size_t(15);
        return o;
    };
    L.tile = take(sizeof(C) << b);
    L.elow = take(sizeof(double) << b);
    L.g1 = take(sizeof(double) * 64);
    L.g2 = take(sizeof(double) * (b > 6 ? (size_t(1) << (b - 6)) : 1));
    L.coef = take(sizeof(double) * 5 * MAXQ);
    L.ush = take(sizeof(double) * MAXQ * MAXQ);
    L.gv = take(sizeof(double) * (MAXQ + 2));
    L.red = take(sizeof(double) * (BLOCK / 32) * NRED);
    L.total = off;
    return L;
}

template <typename R, bool REALC, int MODE>
__global__ void __launch_bounds__(BLOCK)
k_hpsi(const HamParams P, HpsiArgs A) {
    typedef typename cvec<R>::T C;
    extern __shared__ __align__(16) unsigned char smem[];
    if (A.gate && *A.gate != 0) return;  // uniform across the grid
    const int n = P.n, b = A.tile_bits;
    const int TILE = 1 << b;
    const SmemLayout L = hpsi_smem<C>(b);
    C *tile = reinterpret_cast<C *>(smem + L.tile);
    double *elow = reinterpret_cast<double *>(smem + L.elow);
    double *G1 = reinterpret_cast<double *>(smem + L.g1);
    double *G2 = reinterpret_cast<double *>(smem + L.g2);
    double *coef = reinterpret_cast<double *>(smem + L.coef);  // up_re, up_im, dn_re, dn_im, field
    double *Ush = reinterpret_cast<double *>(smem + L.ush);
    double *gv = reinterpret_cast<double *>(smem + L.gv);       // gv[0..b) cross, gv[MAXQ] Ehigh
    double *red = reinterpret_cast<double *>(smem + L.red);

    const int tid = threadIdx.x;
    for (int k = tid; k < MAXQ; k += BLOCK) {
        coef[k] = P.up_re[k];
        coef[MAXQ + k] = P.up_im[k];
        coef[2 * MAXQ + k] = P.dn_re[k];
        coef[3 * MAXQ + k] = P.dn_im[k];
        coef[4 * MAXQ + k] = P.field[k];
    }
    for (int k = tid; k < MAXQ * MAXQ; k += BLOCK) Ush[k] = P.U[k];
    __syncthreads();
    const double *field = coef + 4 * MAXQ;
    // E_low over the b low bits (fields and low-low interactions), once per CTA.
    for (int l = tid; l < TILE; l += BLOCK) {
        double e = 0.0;
        for (int p = 0; p < b; ++p) {
            if (!((l >> p) & 1)) continue;
            e += field[p];
            for (int q = p + 1; q < b; ++q)
                if ((l >> q) & 1) e += Ush[p * MAXQ + q];
        }
        elow[l] = e;
    }

    const double su = A.su_dev ? *A.su_dev : A.su;
    const double sp = (MODE == HP_LANCZOS && A.up) ? (A.sp_dev ? *A.sp_dev : A.sp) : 0.0;
    const C *__restrict__ u = reinterpret_cast<const C *>(A.u);
    const C *__restrict__ upv = reinterpret_cast<const C *>(A.up);

    double acc_r[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) acc_r[k] = 0.0;

    const i64 ntiles = i64(1) << (n - b);
    const int ng2 = b > 6 ? (1 << (b - 6)) : 1;
    const int lane = tid & 31, warp = tid >> 5;

    for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const i64 base = t << b;
        __syncthreads();  // previous tile finished with shared memory
        if (MODE != HP_DIAG) {
            for (int k = tid; k < TILE; k += BLOCK) tile[k] = u[base + k];
        }
        if (warp == 0) {
            // E_high and the cross terms of this tile's high bits.
            double e = 0.0;
            for (int p = b + lane; p < n; p += 32) {
                if (!((base >> p) & 1)) continue;
                e += field[p];
                for (int q = p + 1; q < n; ++q)
                    if ((base >> q) & 1) e += Ush[p * MAXQ + q];
            }
            e = warp_sum(e);
            if (lane == 0) gv[MAXQ] = e;
            for (int p = lane; p < b; p += 32) {
                double g = 0.0;
                for (int q = b; q < n; ++q)
                    if ((base >> q) & 1) g += Ush[p * MAXQ + q];
                gv[p] = g;
            }
        }
        __syncthreads();
        for (int a = tid; a < 64 + ng2; a += BLOCK) {
            double s = 0.0;
            if (a < 64) {
                for (int p = 0; p < (b < 6 ? b : 6); ++p)
                    if ((a >> p) & 1) s += gv[p];
                G1[a] = s;
            } else {
                const int c = a - 64;
                for (int p = 6; p < b; ++p)
                    if ((c >> (p - 6)) & 1) s += gv[p];
                G2[c] = s;
            }
        }
        __syncthreads();
        const double ehigh = gv[MAXQ] - ((MODE == HP_LANCZOS || MODE == HP_STORE) && A.eshift ? *A.eshift : 0.0) +
                             (MODE == HP_DIAG ? 0.0 : P.dc_re);

        for (int k = tid; k < TILE; k += BLOCK) {
            const i64 x = base + k;
            const double d = ehigh + elow[k] + G1[k & 63] + G2[k >> 6];
            if (MODE == HP_DIAG) {
                reinterpret_cast<double *>(A.out)[x] = d;
                continue;
            }
            const C v = tile[k];
            R ar = R(0), ai = R(0);
            // low bits: partners in shared memory
            for (int p = 0; p < b; ++p) {
                const C w = tile[k ^ (1 << p)];
                const int s = ((k >> p) & 1) ? 0 : 2;
                const R cr = R(coef[s * MAXQ + p]);
                if (REALC) {
                    ar = fmar(cr, w.x, ar);
                    ai = fmar(cr, w.y, ai);
                } else {
                    const R ci = R(coef[(s + 1) * MAXQ + p]);
                    ar = fmar(cr, w.x, fmar(-ci, w.y, ar));
                    ai = fmar(cr, w.y, fmar(ci, w.x, ai));
                }
            }
            // high bits: partners in global memory
#pragma unroll 4
            for (int p = b; p < n; ++p) {
                const C w = __ldg(u + (x ^ (i64(1) << p)));
                const int s = ((x >> p) & 1) ? 0 : 2;
                const R cr = R(coef[s * MAXQ + p]);
                if (REALC) {
                    ar = fmar(cr, w.x, ar);
                    ai = fmar(cr, w.y, ai);
                } else {
                    const R ci = R(coef[(s + 1) * MAXQ + p]);
                    ar = fmar(cr, w.x, fmar(-ci, w.y, ar));
                    ai = fmar(cr, w.y, fmar(ci, w.x, ai));
                }
            }
            // H v = su * (flip sum + diag * u), diagonal product in FP64; with the noise
            // term the diagonal has the imaginary part dc_im + dg_im * popcount(x)
            double hr, hi;
            if (P.noisy) {
                const double dI = P.dc_im + P.dg_im * __popcll((unsigned long long)x);
                hr = su * (double(ar) + d * double(v.x) - dI * double(v.y));
                hi = su * (double(ai) + d * double(v.y) + dI * double(v.x));
            } else {
                hr = su * (double(ar) + d * double(v.x));
                hi = su * (double(ai) + d * double(v.y));
            }
            const double vr = su * double(v.x), vi = su * double(v.y);
            if (MODE == HP_STORE || MODE == HP_LANCZOS)
                reinterpret_cast<C *>(A.out)[x] = cmake<C>(hr, hi);
            if (MODE == HP_ENERGY || MODE == HP_LANCZOS) {
                acc_r[0] += hr * hr + hi * hi;
                acc_r[1] += vr * hr + vi * hi;  // <v, Hv>
                acc_r[2] += vr * hi - vi * hr;
            }
            if (MODE == HP_LANCZOS && upv) {
                const C q = upv[x];
                const double pr = sp * double(q.x), pi = sp * double(q.y);
                acc_r[3] += pr * hr + pi * hi;  // <vp, Hv>
                acc_r[4] += pr * hi - pi * hr;
                acc_r[5] += vr * pr + vi * pi;  // <v, vp>
                acc_r[6] += vr * pi - vi * pr;
            }
        }
    }
    if (MODE == HP_ENERGY || MODE == HP_LANCZOS) {
        block_sum<NRED>(acc_r, red);
        if (tid == 0) {
#pragma unroll
            for (int k = 0; k < NRED; ++k) A.partials[(i64)blockIdx.x * NRED + k] = acc_r[k];
        }
    }
}

}  // namespace emusv
