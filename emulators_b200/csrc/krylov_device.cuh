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
static __device__ __noinline__ double krylov_eval(KState *ks, int jj, double dt, double2 *d, double2 *up,
                              double2 *lo, double2 *y, double2 *t, double2 *tn, double2 *acc) {
    const int lane = threadIdx.x & 31;
    const int m = jj + 1;
    for (int k = lane; k < m; k += 32) {
        d[k] = make_double2(dt * ks->a_im[k], -dt * ks->a_re[k]);
        up[k] = k > 0 ? make_double2(dt * ks->b_im[k], -dt * ks->b_re[k]) : make_double2(0.0, 0.0);
        lo[k] = make_double2(0.0, -dt * ks->r[k]);
    }
    __syncwarp();
    double2 Z1, Z2;
    warp_expm_col(m, d, up, lo, y, t, tn, acc, &Z1, &Z2);
    // extension: x_{jj+1} = l Z1, x_{jj+2} = l Z2 with l = A[jj+1][jj] = -i dt r_jj
    const double2 l = lo[jj];
    const double2 x1 = make_double2(l.x * Z1.x - l.y * Z1.y, l.x * Z1.y + l.y * Z1.x);
    const double2 x2 = make_double2(l.x * Z2.x - l.y * Z2.y, l.x * Z2.y + l.y * Z2.x);
    const double err1 = hypot(x1.x, x1.y);                             // krylov_exp.py:81
    const double err2 = hypot(x2.x, x2.y) * (fabs(dt) * ks->hn[jj]);  // krylov_exp.py:82
    for (int k = lane; k < m; k += 32) {
        ks->c_re[k] = y[k + 1].x;
        ks->c_im[k] = y[k + 1].y;
    }
    if (lane == 0) {
        ks->c_re[m] = x1.x;  // expd[j+1, 0] multiplies v_{j+1} (krylov_exp.py:88-90)
        ks->c_im[m] = x1.y;
    }
    __syncwarp();
    return err1 < err2 ? err1 : (err1 * err2 / (err1 - err2));  // krylov_exp.py:84
}

// Scratch of the one-warp tridiagonal exponential (shared memory).
struct KSmem {
    double2 d[KMAX + 2], up[KMAX + 2], lo[KMAX + 2];
    double2 y[KMAX + 4], t[KMAX + 4], tn[KMAX + 4], acc[KMAX + 4];
};

// Decide iteration j of a Lanczos run from the FP64 sums v = ||w_j||^2 and
// (vr, vi) = <v_j, w_j>: ||w_j||, happy breakdown (every iteration), and, when `poll`, the
// extended exponential and the error estimate.  Iterations that were not polled are not
// tested, so on the first poll (`first_poll`) that finds convergence the warp walks back
// over the earlier iterations while they also converge, and stops at the earliest of that
// run -- the iteration where the reference, which tests every iteration, would have
// stopped (the estimate decreases with j).  One warp; ks->status must be KS_RUNNING.
static __device__ void krylov_decide(KState *ks, int j, double v, double vr, double vi, double dt,
                              double exp_tol, double norm_tol, bool poll, bool first_poll,
                              int maxdim, KSmem &S) {
    const int lane = threadIdx.x & 31;
    const double r = sqrt(v);
    const double adt = fabs(dt);
    const double n2 = adt * r;  // ||w|| of the operator -i dt H (krylov_exp.py:60)
    if (!isfinite(r) || !isfinite(ks->hn[j]) || !isfinite(ks->a_re[j]) || !isfinite(ks->a_im[j]) ||
        !isfinite(ks->b_re[j]) || !isfinite(ks->b_im[j])) {
        if (lane == 0) {
            ks->status = KS_NONFINITE;
            ks->iters = j + 1;
        }
        __syncwarp();
        return;
    }
    if (lane == 0) {
        ks->r[j] = r;
        ks->vv_re[j + 1] = vr / r;  // <v_{j+1}, v_j> = conj(<v_j, w>) / ||w||
        ks->vv_im[j + 1] = -vi / r;
        ks->scale[j + 1] = 1.0 / r;
    }
    __syncwarp();
    const int m = j + 1;
    if (n2 < norm_tol) {  // krylov_exp.py:63-71: exp(T[:j+1,:j+1]) e_0 over j+1 vectors
        for (int k = lane; k < m; k += 32) {
            S.d[k] = make_double2(dt * ks->a_im[k], -dt * ks->a_re[k]);
            S.up[k] = k > 0 ? make_double2(dt * ks->b_im[k], -dt * ks->b_re[k]) : make_double2(0.0, 0.0);
            S.lo[k] = make_double2(0.0, -dt * ks->r[k]);
        }
        __syncwarp();
        double2 Z1, Z2;
        warp_expm_col(m, S.d, S.up, S.lo, S.y, S.t, S.tn, S.acc, &Z1, &Z2);
        for (int k = lane; k < m; k += 32) {
            ks->c_re[k] = S.y[k + 1].x;
            ks->c_im[k] = S.y[k + 1].y;
        }
        if (lane == 0) {
            ks->nvec = m;
            ks->iters = j + 1;
            ks->status = KS_HAPPY;
        }
        __syncwarp();
        return;
    }
    if (!poll) return;
    double err = krylov_eval(ks, j, dt, S.d, S.up, S.lo, S.y, S.t, S.tn, S.acc);
    int jc = j;  // the stopping iteration
    if (err < exp_tol && first_poll) {
        int last = j;  // iteration whose coefficients are in ks->c
        for (int jj = j - 1; jj >= 0; --jj) {
            const double e = krylov_eval(ks, jj, dt, S.d, S.up, S.lo, S.y, S.t, S.tn, S.acc);
            last = jj;
            if (!(e < exp_tol)) break;
            err = e;
            jc = jj;
        }
        if (last != jc) krylov_eval(ks, jc, dt, S.d, S.up, S.lo, S.y, S.t, S.tn, S.acc);
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

}  // namespace emusv
