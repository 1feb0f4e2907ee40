// Device code shared by the single-instance Krylov step (krylov.cu) and the batched
// persistent engine (batch.cu): the one-warp tridiagonal exponential with the Expokit
// extension rows, and the per-iteration Lanczos decision (krylov_exp.py:60-96).
#pragma once

#include "krylov_internal.cuh"

namespace emusv {

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// One warp: y = exp(A) e_0 for a complex tridiagonal m x m matrix A
//   (d[k] = A[k][k], up[k] = A[k-1][k], lo[k] = A[k+1][k]),
// plus Z1 = int_0^1 y_{m-1}(s) ds and Z2 = int_0^1 (1-s) y_{m-1}(s) ds, which give the
// two Expokit extension rows exactly: for the extended matrix
// [[A,0,0],[l e_{m-1}^T,0,0],[0,1,0]],  exp(.) e_0 = (y, l Z1, l Z2).
// Method: Taylor series of exp(hA) applied to the vector, h = 1/s with ||hA||_1 <= 2,
// repeated s times; the integrals come from the same series term by term
// (int_0^h (tau/h)^q dtau = h/(q+1), int_0^h (h-tau)(tau/h)^q dtau = h^2/((q+1)(q+2))).
// smem arrays hold m+2 entries with a zero pad on each side (index k+1 for entry k).
static __device__ __noinline__ void warp_expm_col(int m, const double2 *d, const double2 *up, const double2 *lo,
                              double2 *y, double2 *t, double2 *tn, double2 *acc,
                              double2 *Z1, double2 *Z2) {
    const int lane = threadIdx.x & 31;
    double nrm = 0.0;
    for (int k = lane; k < m; k += 32) {
        double c = hypot(d[k].x, d[k].y);
        if (k > 0) c += hypot(up[k].x, up[k].y);
        if (k < m - 1) c += hypot(lo[k].x, lo[k].y);
        nrm = fmax(nrm, c);
    }
    nrm = warp_max(nrm);
    const double THETA = 2.0;
    // ||hA||_1 <= THETA; the sub-step count is capped (callers check finiteness first)
    int s = 1;
    if (nrm > THETA) s = nrm < THETA * (1 << 20) ? (int)ceil(nrm / THETA) : (1 << 20);
    const double h = 1.0 / s;
    // reciprocals 1/q (q < 84) by the warp in parallel: no FP64 division in the series
    __shared__ double inv[84];
    for (int q = lane; q < 84; q += 32) inv[q] = q ? 1.0 / q : 0.0;
    // padded vectors: index k+1 holds entry k; pads stay zero
    for (int k = lane; k < m + 2; k += 32) {
        y[k] = make_double2(k == 1 ? 1.0 : 0.0, 0.0);
        t[k] = make_double2(0.0, 0.0);
        tn[k] = make_double2(0.0, 0.0);
        acc[k] = make_double2(0.0, 0.0);
    }
    __syncwarp();
    double2 z1 = make_double2(0.0, 0.0), z2 = make_double2(0.0, 0.0);
    for (int step = 0; step < s; ++step) {
        for (int k = lane; k < m; k += 32) {
            t[k + 1] = y[k + 1];
            acc[k + 1] = y[k + 1];
        }
        __syncwarp();
        double2 tl = t[m];  // last entry of t_0
        double2 S1 = tl, S2 = make_double2(0.5 * tl.x, 0.5 * tl.y);
        double2 *cur = t, *nxt = tn;
        for (int q = 1; q < 80; ++q) {
            const double f = h * inv[q];
            double tmax = 0.0, amax = 0.0;
            for (int k = lane; k < m; k += 32) {
                const double2 a0 = cur[k + 1], am = cur[k], ap = cur[k + 2];
                double re = d[k].x * a0.x - d[k].y * a0.y;
                double im = d[k].x * a0.y + d[k].y * a0.x;
                if (k > 0) {  // A[k][k-1] = lo[k-1]
                    re += lo[k - 1].x * am.x - lo[k - 1].y * am.y;
                    im += lo[k - 1].x * am.y + lo[k - 1].y * am.x;
                }
                if (k < m - 1) {  // A[k][k+1] = up[k+1]
                    re += up[k + 1].x * ap.x - up[k + 1].y * ap.y;
                    im += up[k + 1].x * ap.y + up[k + 1].y * ap.x;
                }
                const double2 o = make_double2(f * re, f * im);
                nxt[k + 1] = o;
                double2 ac = acc[k + 1];
                ac.x += o.x;
                ac.y += o.y;
                acc[k + 1] = ac;
                tmax = fmax(tmax, fmax(fabs(o.x), fabs(o.y)));
                amax = fmax(amax, fmax(fabs(ac.x), fabs(ac.y)));
            }
            __syncwarp();
            const double2 last = nxt[m];
            const double w1 = inv[q + 1], w2 = inv[q + 1] * inv[q + 2];
            S1.x += w1 * last.x;
            S1.y += w1 * last.y;
            S2.x += w2 * last.x;
            S2.y += w2 * last.y;
            double2 *tmp = cur;
            cur = nxt;
            nxt = tmp;
            if ((q & 3) == 0) {  // test the term size every fourth term (warp shuffles)
                tmax = warp_max(tmax);
                amax = warp_max(amax);
                if (tmax <= 1e-18 * fmax(amax, 1e-300)) break;
            }
        }
        z2.x += h * z1.x + h * h * S2.x;
        z2.y += h * z1.y + h * h * S2.y;
        z1.x += h * S1.x;
        z1.y += h * S1.y;
        for (int k = lane; k < m; k += 32) y[k + 1] = acc[k + 1];
        __syncwarp();
    }
    *Z1 = z1;
    *Z2 = z2;
}

// Extended exponential of iteration jj (the matrix A = -i dt T_H of size jj+1 with the
// extension entry lo[jj] = -i dt r_jj): writes the coefficients c[0..jj+1] and returns the
// Expokit error estimate (krylov_exp.py:77-84).  One warp.
// ---------------------------------------------------------------- register form
// One warp, exp(A) e_col for a complex tridiagonal M x M matrix A (plus, optionally, one
// coupling entry A[0][cpl] = 1), with the vectors in registers: lane L owns the entries
// k = L * NE + e (e < NE), so the tridiagonal products need two lane shuffles per term.
// Row form: A[k][k] = d[e], A[k][k-1] = l[e], A[k][k+1] = u[e] (zero outside the matrix).
// Method: Taylor series of exp(hA) on the vector, h = 1/s with ||hA||_inf <= 2, s times;
// when zlast >= 0 the Expokit integrals Z1 = int_0^1 y_zlast, Z2 = int_0^1 (1-s) y_zlast
// come from the same series term by term (as warp_expm_col).
template <int NE>
__device__ __forceinline__ double2 reg_pick(const double2 (&v)[NE], int k) {
    const int owner = k / NE, e = k - owner * NE;
    double2 r = v[0];
#pragma unroll
    for (int q = 1; q < NE; ++q)
        if (q == e) r = v[q];
    r.x = __shfl_sync(0xffffffffu, r.x, owner);
    r.y = __shfl_sync(0xffffffffu, r.y, owner);
    return r;
}

template <int NE>
static __device__ void reg_expm(int M, const double2 (&d)[NE], const double2 (&l)[NE],
                                const double2 (&u)[NE], int cpl, int col, double2 (&y)[NE],
                                int zlast, double2 *Z1, double2 *Z2) {
    const int lane = threadIdx.x & 31;
    double nrm = 0.0;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        double c = hypot(d[e].x, d[e].y) + hypot(l[e].x, l[e].y) + hypot(u[e].x, u[e].y);
        if (cpl >= 0 && lane * NE + e == 0) c += 1.0;
        nrm = fmax(nrm, c);
    }
    nrm = warp_max(nrm);
    int s = 1;
    if (nrm > 2.0) s = nrm < 2.0 * (1 << 20) ? (int)ceil(nrm / 2.0) : (1 << 20);
    const double h = 1.0 / s;
#pragma unroll
    for (int e = 0; e < NE; ++e) y[e] = make_double2(lane * NE + e == col ? 1.0 : 0.0, 0.0);
    double2 z1 = make_double2(0.0, 0.0), z2 = make_double2(0.0, 0.0);
    for (int st = 0; st < s; ++st) {
        double2 t[NE], acc[NE];
#pragma unroll
        for (int e = 0; e < NE; ++e) t[e] = acc[e] = y[e];
        double2 S1 = make_double2(0.0, 0.0), S2 = S1;
        if (zlast >= 0) {
            S1 = reg_pick(t, zlast);
            S2 = make_double2(0.5 * S1.x, 0.5 * S1.y);
        }
        for (int q = 1; q < 90; ++q) {
            const double f = h / q;
            // neighbours across the lane boundary
            double2 prev, next;
            prev.x = __shfl_up_sync(0xffffffffu, t[NE - 1].x, 1);
            prev.y = __shfl_up_sync(0xffffffffu, t[NE - 1].y, 1);
            next.x = __shfl_down_sync(0xffffffffu, t[0].x, 1);
            next.y = __shfl_down_sync(0xffffffffu, t[0].y, 1);
            if (lane == 0) prev = make_double2(0.0, 0.0);
            if (lane == 31) next = make_double2(0.0, 0.0);
            double2 cp = make_double2(0.0, 0.0);
            if (cpl >= 0) cp = reg_pick(t, cpl);
            double2 nt[NE];
            double tmax = 0.0;
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                const double2 a0 = t[e];
                const double2 am = e > 0 ? t[e - 1] : prev;
                const double2 ap = e < NE - 1 ? t[e + 1] : next;
                double re = d[e].x * a0.x - d[e].y * a0.y + l[e].x * am.x - l[e].y * am.y +
                            u[e].x * ap.x - u[e].y * ap.y;
                double im = d[e].x * a0.y + d[e].y * a0.x + l[e].x * am.y + l[e].y * am.x +
                            u[e].x * ap.y + u[e].y * ap.x;
                if (cpl >= 0 && lane == 0 && e == 0) {
                    re += cp.x;
                    im += cp.y;
                }
                nt[e] = make_double2(f * re, f * im);
                acc[e].x += nt[e].x;
                acc[e].y += nt[e].y;
                tmax = fmax(tmax, fmax(fabs(nt[e].x), fabs(nt[e].y)));
            }
#pragma unroll
            for (int e = 0; e < NE; ++e) t[e] = nt[e];
            if (zlast >= 0) {
                const double2 last = reg_pick(t, zlast);
                const double w1 = 1.0 / (q + 1), w2 = w1 / (q + 2);
                S1.x += w1 * last.x;
                S1.y += w1 * last.y;
                S2.x += w2 * last.x;
                S2.y += w2 * last.y;
            }
            if ((q & 3) == 0) {
                double amax = 0.0;
#pragma unroll
                for (int e = 0; e < NE; ++e) amax = fmax(amax, fmax(fabs(acc[e].x), fabs(acc[e].y)));
                tmax = warp_max(tmax);
                amax = warp_max(amax);
                if (tmax <= 1e-18 * fmax(amax, 1e-300)) break;
            }
        }
        z2.x += h * z1.x + h * h * S2.x;
        z2.y += h * z1.y + h * h * S2.y;
        z1.x += h * S1.x;
        z1.y += h * S1.y;
#pragma unroll
        for (int e = 0; e < NE; ++e) y[e] = acc[e];
    }
    if (Z1) *Z1 = z1;
    if (Z2) *Z2 = z2;
}

// ---------------------------------------------------------------- Chebyshev form
// One warp, y = exp(A) e_col for A = -i dt T with T tridiagonal (plus optionally one
// coupling entry A[0][cpl] = cplv, plus any non-symmetric rows whose eigenvalues are
// inside T's Gershgorin interval), held in rows by the lanes as in reg_expm.  With
// T's spectrum in [c - R, c + R] (Gershgorin), A = -i dt (c + R X) and
//   exp(-i z x) = J_0(z) + 2 sum_{k>=1} (-i)^k J_k(z) T_k(x),   z = dt R,
// so exp(A) e_col = e^{-i dt c} sum_k coef_k T_k(X) e_col, summed by Clenshaw's
// recurrence from the top term down while Miller's backward recurrence produces the
// Bessel values J_k(|z|) in the same order (normalised at the end by
// J_0 + 2 sum J_2k = 1).  About |z| + 40 tridiagonal products instead of the Taylor
// form's ~12 |z|.  `Tdiag[e]` is T's (real) diagonal centre of row e and `Trad[e]` its
// Gershgorin radius (|row| off-diagonal sum of T).
template <int NE>
static __device__ void cheb_expm(const double2 (&d)[NE], const double2 (&l)[NE], const double2 (&u)[NE],
                                 int cpl, double2 cplv, int col, double dt, const double (&Tdiag)[NE],
                                 const double (&Trad)[NE], int M, double2 (&y)[NE]) {
    const int lane = threadIdx.x & 31;
    double lo = 1e300, hi = -1e300;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        if (lane * NE + e < M) {
            lo = fmin(lo, Tdiag[e] - Trad[e]);
            hi = fmax(hi, Tdiag[e] + Trad[e]);
        }
    }
    lo = -warp_max(-lo);
    hi = warp_max(hi);
    const double c = 0.5 * (lo + hi);
    // radius at least 1/|dt| (z >= 1): keeps X = (T - c)/R bounded when T's own spread is
    // tiny, and Miller's recurrence (factors 2k/z) far from overflow
    const double R = fmax(0.5 * (hi - lo), 1.0 / fabs(dt));
    const double z = fabs(dt) * R;
    const double sgn = dt >= 0.0 ? 1.0 : -1.0;
    // X = (A - alpha) / beta,  alpha = -i dt c,  beta = -i dt R;  1/beta = i / (dt R)
    const double2 ib = make_double2(0.0, 1.0 / (dt * R));
    const double2 alpha = make_double2(0.0, -dt * c);
    auto cm = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    double2 xd[NE], xl[NE], xu[NE];
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        xd[e] = cm(make_double2(d[e].x - alpha.x, d[e].y - alpha.y), ib);
        xl[e] = cm(l[e], ib);
        xu[e] = cm(u[e], ib);
        if (lane * NE + e >= M) xd[e] = make_double2(0.0, 0.0);
    }
    const double2 xc = cm(cplv, ib);
    // X v for a vector held in the row layout
    auto xmul = [&](const double2 (&v)[NE], double2 (&out)[NE]) {
        double2 prev, next;
        prev.x = __shfl_up_sync(0xffffffffu, v[NE - 1].x, 1);
        prev.y = __shfl_up_sync(0xffffffffu, v[NE - 1].y, 1);
        next.x = __shfl_down_sync(0xffffffffu, v[0].x, 1);
        next.y = __shfl_down_sync(0xffffffffu, v[0].y, 1);
        if (lane == 0) prev = make_double2(0.0, 0.0);
        if (lane == 31) next = make_double2(0.0, 0.0);
        double2 cp = make_double2(0.0, 0.0);
        if (cpl >= 0) cp = reg_pick(v, cpl);
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const double2 am = e > 0 ? v[e - 1] : prev;
            const double2 ap = e < NE - 1 ? v[e + 1] : next;
            double2 o = cm(xd[e], v[e]);
            const double2 t1 = cm(xl[e], am), t2 = cm(xu[e], ap);
            o.x += t1.x + t2.x;
            o.y += t1.y + t2.y;
            if (cpl >= 0 && lane == 0 && e == 0) {
                const double2 t3 = cm(xc, cp);
                o.x += t3.x;
                o.y += t3.y;
            }
            out[e] = o;
        }
    };
    const int N = (int)ceil(1.1 * z) + 40;  // terms kept
    const int K = N + 30;                   // Miller's start
    const double twoz = z > 0.0 ? 2.0 / z : 0.0;  // no division inside the recurrence
    double2 b1[NE], b2[NE];  // b_{k+1}, b_{k+2}
#pragma unroll
    for (int e = 0; e < NE; ++e) b1[e] = b2[e] = make_double2(0.0, 0.0);
    double jk1 = 0.0, jk = 1e-280, S = 0.0;  // J~_{k+1}, J~_k, normalisation sum
    // (-i sgn)^k at k = K, stepped down by multiplying with (i sgn)
    double2 ph;
    {
        const int r = K & 3;
        const double2 base = make_double2(0.0, -sgn);
        ph = make_double2(1.0, 0.0);
        for (int q = 0; q < r; ++q) ph = cm(ph, base);
    }
    const double2 up_step = make_double2(0.0, sgn);
    for (int k = K; k >= 1; --k) {
        if ((k & 1) == 0) S += 2.0 * jk;
        if (k <= N) {  // b_k = coef_k e_col + 2 X b_{k+1} - b_{k+2}
            double2 xb[NE];
            xmul(b1, xb);
            const double2 ck = make_double2(2.0 * jk * ph.x, 2.0 * jk * ph.y);
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                double2 nb = make_double2(2.0 * xb[e].x - b2[e].x, 2.0 * xb[e].y - b2[e].y);
                if (lane * NE + e == col) {
                    nb.x += ck.x;
                    nb.y += ck.y;
                }
                b2[e] = b1[e];
                b1[e] = nb;
            }
        }
        // J~_{k-1} = (2k / z) J~_k - J~_{k+1}
        const double jm = (twoz * k) * jk - jk1;
        jk1 = jk;
        jk = jm;
        ph = cm(ph, up_step);
        if (fabs(jk) > 1e250) {  // rescale everything linear in the J~
            const double f = 1e-250;
            jk *= f;
            jk1 *= f;
            S *= f;
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                b1[e].x *= f;
                b1[e].y *= f;
                b2[e].x *= f;
                b2[e].y *= f;
            }
        }
    }
    // now jk = J~_0, b1 = b_1, b2 = b_2:  sum = J~_0 e_col + X b_1 - b_2
    S += jk;
    double2 xb[NE];
    xmul(b1, xb);
    const double2 ea = make_double2(cos(alpha.y), sin(alpha.y));  // e^{alpha}, alpha imaginary
    const double inv = z > 0.0 ? 1.0 / S : 1.0;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        double2 v = make_double2(xb[e].x - b2[e].x, xb[e].y - b2[e].y);
        if (lane * NE + e == col) v.x += jk;
        if (z == 0.0) v = make_double2(lane * NE + e == col ? 1.0 : 0.0, 0.0);
        v.x *= inv;
        v.y *= inv;
        y[e] = cm(ea, v);
    }
}

// Rows of A = -i dt T_H (the first m rows of a Lanczos run) in the register layout.
template <int NE>
__device__ __forceinline__ void load_rows(const KState *ks, int m, double dt, double2 (&d)[NE],
                                          double2 (&l)[NE], double2 (&u)[NE], double (&td)[NE],
                                          double (&tr)[NE]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const int k = lane * NE + e;
        d[e] = l[e] = u[e] = make_double2(0.0, 0.0);
        td[e] = tr[e] = 0.0;
        if (k < m) {
            const double ar = ks->a_re[k] + ks->shift;  // a_k of H (the run may use H - sigma)
            d[e] = make_double2(dt * ks->a_im[k], -dt * ar);
            td[e] = ar;
            if (k > 0) {
                l[e] = make_double2(0.0, -dt * ks->r[k - 1]);  // A[k][k-1]
                tr[e] += fabs(ks->r[k - 1]);
            }
            if (k + 1 < m) {
                u[e] = make_double2(dt * ks->b_im[k + 1], -dt * ks->b_re[k + 1]);  // A[k][k+1]
                tr[e] += hypot(ks->b_re[k + 1], ks->b_im[k + 1]);
            }
            tr[e] += fabs(ks->a_im[k]);
        }
    }
}

// Extended exponential of iteration jj: exp of the (jj+3) x (jj+3) matrix
// [[A, 0, 0], [l e_jj^T, 0, 0], [0, 1, 0]] (A = -i dt T_H of size jj+1, l = -i dt r_jj)
// applied to e_0 = (y, x1, x2) (krylov_exp.py:77-78); writes the coefficients
// c[0..jj+1] = (y, x1) and returns the Expokit error estimate (krylov_exp.py:81-84).
// One warp, Chebyshev form.
// NE entries per lane: the smallest layout that holds the jj + 3 rows (the work of every
// Chebyshev term scales with NE; each entry's arithmetic is the same in every layout).
template <int NE>
static __device__ __noinline__ double krylov_eval_ne(KState *ks, int jj, double dt) {
    const int lane = threadIdx.x & 31;
    const int m = jj + 1, M = m + 2;
    double2 d[NE], l[NE], u[NE], y[NE];
    double td[NE], tr[NE];
    load_rows<NE>(ks, m, dt, d, l, u, td, tr);
#pragma unroll
    for (int e = 0; e < NE; ++e) {  // the two extension rows (eigenvalue 0 of T)
        const int k = lane * NE + e;
        if (k == m) {  // T units: centre 0, the entry r_jj
            l[e] = make_double2(0.0, -dt * ks->r[jj]);
            td[e] = 0.0;
            tr[e] = fabs(ks->r[jj]);
        }
        if (k == m + 1) {  // the entry 1 of A is 1/|dt| in T units
            l[e] = make_double2(1.0, 0.0);
            td[e] = 0.0;
            tr[e] = 1.0 / fabs(dt);
        }
    }
    cheb_expm<NE>(d, l, u, -1, make_double2(0.0, 0.0), 0, dt, td, tr, M, y);
    const double2 x1 = reg_pick(y, m), x2 = reg_pick(y, m + 1);
    const double err1 = hypot(x1.x, x1.y);                             // krylov_exp.py:81
    const double err2 = hypot(x2.x, x2.y) * (fabs(dt) * ks->hn[jj]);  // krylov_exp.py:82
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const int k = lane * NE + e;
        if (k <= m) {  // c[m] = x1 multiplies v_{jj+1} (krylov_exp.py:88-90)
            ks->c_re[k] = y[e].x;
            ks->c_im[k] = y[e].y;
        }
    }
    __syncwarp();
    return err1 < err2 ? err1 : (err1 * err2 / (err1 - err2));  // krylov_exp.py:84
}
static __device__ double krylov_eval(KState *ks, int jj, double dt) {
    constexpr int NEMAX = (KMAX + 2 + 31) / 32;
    const int M = jj + 3;
    if (M <= 32) return krylov_eval_ne<1>(ks, jj, dt);
    if (M <= 64) return krylov_eval_ne<2>(ks, jj, dt);
    if (M <= 96) return krylov_eval_ne<3>(ks, jj, dt);
    return krylov_eval_ne<NEMAX>(ks, jj, dt);
}

// Decide iteration j of a Lanczos run from the FP64 sums v = ||w_j||^2 and
// (vr, vi) = <v_j, w_j>, in two parts.
// krylov_norms: ||w_j||, <v_{j+1}, v_j> and scale_{j+1} (what iteration j+1 needs), and
// the outcome flag: KD_NONFINITE (a non-finite value), KD_HAPPY (the happy breakdown of
// krylov_exp.py:63-71, tested every iteration) or 0.  Writes no status.
// krylov_conclude: every status change of iteration j -- NONFINITE, HAPPY (with the
// exponential of T[:j+1,:j+1]) or, when `poll`, the extended exponential, the error
// estimate and CONVERGED / MAXDIM.  Iterations that were not polled are not tested, so
// when the first poll (`first_poll`) already converges the warp tests the earlier
// iterations in order and stops at the first that converges -- where the reference, which
// tests every iteration, stops.  One warp each; ks->status must be KS_RUNNING.
// Happy breakdown after m vectors: c = exp(T[:m,:m]) e_0 (krylov_exp.py:63-71), in the
// smallest register layout that holds the m rows (a separate, non-inlined function per
// layout, so the large layouts do not raise the register demand of the kernels that call
// the decision).
template <int NE>
static __device__ __noinline__ void krylov_happy_ne(KState *ks, int m, double dt) {
    const int lane = threadIdx.x & 31;
    double2 d[NE], l[NE], u[NE], y[NE];
    double td[NE], tr[NE];
    load_rows<NE>(ks, m, dt, d, l, u, td, tr);
    cheb_expm<NE>(d, l, u, -1, make_double2(0.0, 0.0), 0, dt, td, tr, m, y);
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const int k = lane * NE + e;
        if (k < m) {
            ks->c_re[k] = y[e].x;
            ks->c_im[k] = y[e].y;
        }
    }
    __syncwarp();
}
static __device__ void krylov_happy(KState *ks, int m, double dt) {
    constexpr int NEMAX = (KMAX + 2 + 31) / 32;
    if (m <= 32) krylov_happy_ne<1>(ks, m, dt);
    else if (m <= 64) krylov_happy_ne<2>(ks, m, dt);
    else if (m <= 96) krylov_happy_ne<3>(ks, m, dt);
    else krylov_happy_ne<NEMAX>(ks, m, dt);
}

enum { KD_OK = 0, KD_NONFINITE = 1, KD_HAPPY = 2 };

static __device__ int krylov_norms(KState *ks, int j, double v, double vr, double vi, double dt,
                                   double norm_tol) {
    const int lane = threadIdx.x & 31;
    const double r = sqrt(v);
    const double n2 = fabs(dt) * r;  // ||w|| of the operator -i dt H (krylov_exp.py:60)
    if (!isfinite(r) || !isfinite(ks->hn[j]) || !isfinite(ks->a_re[j]) || !isfinite(ks->a_im[j]) ||
        !isfinite(ks->b_re[j]) || !isfinite(ks->b_im[j]))
        return KD_NONFINITE;
    if (lane == 0) {
        ks->r[j] = r;
        ks->vv_re[j + 1] = vr / r;  // <v_{j+1}, v_j> = conj(<v_j, w>) / ||w||
        ks->vv_im[j + 1] = -vi / r;
        ks->scale[j + 1] = 1.0 / r;
    }
    __syncwarp();
    return n2 < norm_tol ? KD_HAPPY : KD_OK;
}

static __device__ void krylov_conclude(KState *ks, int j, int flag, double dt, double exp_tol, bool poll,
                                       bool first_poll, int maxdim) {
    const int lane = threadIdx.x & 31;
    if (flag == KD_NONFINITE) {
        if (lane == 0) {
            ks->status = KS_NONFINITE;
            ks->iters = j + 1;
        }
        __syncwarp();
        return;
    }
    const int m = j + 1;
    if (flag == KD_HAPPY) {  // krylov_exp.py:63-71: exp(T[:j+1,:j+1]) e_0 over j+1 vectors
        krylov_happy(ks, m, dt);
        if (lane == 0) {
            ks->nvec = m;
            ks->iters = j + 1;
            ks->status = KS_HAPPY;
        }
        __syncwarp();
        return;
    }
    if (!poll) return;
    double err = krylov_eval(ks, j, dt);
    int jc = j;  // the stopping iteration
    // NaN (both error terms zero: 0 * 0 / 0 fails the test, as in the reference) also
    // sends the first test back over the untested iterations
    if ((err < exp_tol || err != err) && first_poll && j > 0) {
        // the untested iterations, in order: the first that converges is where the
        // reference (testing every iteration) stops
        for (int jj = 0; jj < j; ++jj) {
            const double e = krylov_eval(ks, jj, dt);
            if (e < exp_tol) {
                err = e;
                jc = jj;
                break;
            }
        }
        if (jc == j) krylov_eval(ks, j, dt);  // its coefficients again
    }
    if (lane == 0) {
        ks->err = err;
        ks->nvec = jc + 2;
        ks->iters = jc + 1;
        if (err < exp_tol)
            ks->status = KS_CONVERGED;
        else if (j + 1 >= maxdim)
            ks->status = KS_MAXDIM;
    }
    __syncwarp();
}

// Both parts in one warp (the single-kernel decision of the batched engine and of the
// small registers' iteration).
static __device__ void krylov_decide(KState *ks, int j, double v, double vr, double vi, double dt,
                              double exp_tol, double norm_tol, bool poll, bool first_poll,
                              int maxdim) {
    const int flag = krylov_norms(ks, j, v, vr, vi, dt, norm_tol);
    krylov_conclude(ks, j, flag, dt, exp_tol, poll, first_poll, maxdim);
}

}  // namespace emusv
