/*
 * ORACLE -- test infrastructure only.  CPU restatement of the reference emu-sv hot-path
 * arithmetic on 2^N-sized vectors, used by tests/, the smoke check and the CPU baseline
 * leg of bench.py as the checker.  The product path never links or calls this file.
 *
 * Conventions (reference emu_sv/hamiltonian.py, emu_sv/state_vector.py):
 *   - amplitude index x in [0, 2^n); qubit i is bit (n-1-i) of x (qubit 0 = MSB);
 *   - bit value 1 = Rydberg |r>, n_i = |r><r|;
 *   - complex vectors are interleaved (re, im) float64 pairs (torch.complex128 layout).
 *
 * Parity is pinned against fixtures produced by running the reference itself
 * (tests/golden/make_golden.py); see tests/test_oracle_golden.py.
 *
 * Build: gcc -O3 -fopenmp -shared -fPIC, by build() in oracle/oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <omp.h>

typedef int64_t i64;

/* Parallel regions only pay off on vectors of a few hundred KB and more. */
#define PAR(D) ((D) >= (1 << 15))

static inline int bit_of(i64 x, int n, int q) { return (int)((x >> (n - 1 - q)) & 1); }

int or_num_threads(void) { return omp_get_max_threads(); }
void or_set_threads(int t) { if (t > 0) omp_set_num_threads(t); }

/* diag[x] = -sum_i delta_i x_i + sum_{i<j} U_ij x_i x_j   (hamiltonian.py:139-162;
 * only the upper triangle of U is read, hamiltonian.py:153-161). U is n x n row-major. */
void or_diag(int n, const double *delta, const double *U, double *diag)
{
    i64 D = (i64)1 << n;
#pragma omp parallel for schedule(static) if (PAR(D))
    for (i64 x = 0; x < D; ++x) {
        double e = 0.0;
        for (int i = 0; i < n; ++i) {
            if (!bit_of(x, n, i)) continue;
            e -= delta[i];
            for (int j = i + 1; j < n; ++j)
                if (bit_of(x, n, j)) e += U[i * n + j];
        }
        diag[x] = e;
    }
}

/* out = H psi  (hamiltonian.py:69-137).
 * coef: [n][4] doubles = (up_re, up_im, down_re, down_im), where "up" multiplies the
 * transfer |g> -> |r> (the coefficient of |r><g|, Omega/2 e^{i phi}, hamiltonian.py:62-64)
 * and "down" the transfer |r> -> |g> (its conjugate).  In the real case
 * (hamiltonian.py:93-110) both are Omega/2.
 * out[x] = diag[x] psi[x] + sum_i c_i(x) psi[x ^ bit_i], c_i(x) = up if x_i = 1 else down. */
void or_hpsi(int n, const double *coef, const double *diag, const double *psi, double *out)
{
    i64 D = (i64)1 << n;
#pragma omp parallel for schedule(static) if (PAR(D))
    for (i64 x = 0; x < D; ++x) {
        double re = diag[x] * psi[2 * x], im = diag[x] * psi[2 * x + 1];
        for (int i = 0; i < n; ++i) {
            i64 y = x ^ ((i64)1 << (n - 1 - i));
            const double *c = coef + 4 * i + (bit_of(x, n, i) ? 0 : 2);
            double pr = psi[2 * y], pi = psi[2 * y + 1];
            re += c[0] * pr - c[1] * pi;
            im += c[0] * pi + c[1] * pr;
        }
        out[2 * x] = re;
        out[2 * x + 1] = im;
    }
}

/* <a, b> = sum conj(a) b  (torch.vdot / tensordot(a.conj(), b)). */
void or_vdot(i64 D, const double *a, const double *b, double *res)
{
    double sr = 0.0, si = 0.0;
#pragma omp parallel for reduction(+ : sr, si) schedule(static) if (PAR(D))
    for (i64 k = 0; k < D; ++k) {
        double ar = a[2 * k], ai = a[2 * k + 1], br = b[2 * k], bi = b[2 * k + 1];
        sr += ar * br + ai * bi;
        si += ar * bi - ai * br;
    }
    res[0] = sr;
    res[1] = si;
}

double or_norm2(i64 D, const double *a)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static) if (PAR(D))
    for (i64 k = 0; k < 2 * D; ++k) s += a[k] * a[k];
    return s;
}

/* y += alpha x */
void or_axpy(i64 D, double ar, double ai, const double *x, double *y)
{
#pragma omp parallel for schedule(static) if (PAR(D))
    for (i64 k = 0; k < D; ++k) {
        double xr = x[2 * k], xi = x[2 * k + 1];
        y[2 * k] += ar * xr - ai * xi;
        y[2 * k + 1] += ar * xi + ai * xr;
    }
}

/* x *= alpha (complex) */
void or_scale(i64 D, double ar, double ai, double *x)
{
#pragma omp parallel for schedule(static) if (PAR(D))
    for (i64 k = 0; k < D; ++k) {
        double xr = x[2 * k], xi = x[2 * k + 1];
        x[2 * k] = ar * xr - ai * xi;
        x[2 * k + 1] = ar * xi + ai * xr;
    }
}

/* out = sum_k c_k V_k ; V is m x D contiguous (krylov_exp.py:88-90). */
void or_combine(i64 D, int m, const double *c, const double *V, double *out)
{
#pragma omp parallel for schedule(static) if (PAR(D))
    for (i64 x = 0; x < D; ++x) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k < m; ++k) {
            const double *v = V + 2 * ((i64)k * D + x);
            re += c[2 * k] * v[0] - c[2 * k + 1] * v[1];
            im += c[2 * k] * v[1] + c[2 * k + 1] * v[0];
        }
        out[2 * x] = re;
        out[2 * x + 1] = im;
    }
}

/* occ[i] = sum_x |psi[x]|^2 x_i   (custom_callback_implementations.py:30-47). */
void or_occupation(int n, const double *psi, double *occ)
{
    i64 D = (i64)1 << n;
    for (int i = 0; i < n; ++i) occ[i] = 0.0;
#pragma omp parallel if (PAR(D))
    {
        double loc[64] = {0};
#pragma omp for schedule(static)
        for (i64 x = 0; x < D; ++x) {
            double p = psi[2 * x] * psi[2 * x] + psi[2 * x + 1] * psi[2 * x + 1];
            for (int i = 0; i < n; ++i)
                if (bit_of(x, n, i)) loc[i] += p;
        }
#pragma omp critical
        for (int i = 0; i < n; ++i) occ[i] += loc[i];
    }
}

/* corr[i][j] = sum_x |psi[x]|^2 x_i x_j   (custom_callback_implementations.py:77-102). */
void or_correlation(int n, const double *psi, double *corr)
{
    i64 D = (i64)1 << n;
    memset(corr, 0, sizeof(double) * n * n);
#pragma omp parallel if (PAR(D))
    {
        double loc[32 * 32];
        memset(loc, 0, sizeof(loc));
#pragma omp for schedule(static)
        for (i64 x = 0; x < D; ++x) {
            double p = psi[2 * x] * psi[2 * x] + psi[2 * x + 1] * psi[2 * x + 1];
            for (int i = 0; i < n; ++i) {
                if (!bit_of(x, n, i)) continue;
                for (int j = i; j < n; ++j)
                    if (bit_of(x, n, j)) loc[i * 32 + j] += p;
            }
        }
#pragma omp critical
        for (int i = 0; i < n; ++i)
            for (int j = i; j < n; ++j) corr[i * n + j] += loc[i * 32 + j];
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) corr[i * n + j] = corr[j * n + i];
}

/* Gradient contractions of the adjoint (emu_sv/time_evolution/torch.py:322-353):
 *   rho(x)      = sum_k conj(G[k,x]) E[k,x]
 *   tau_i(x)    = sum_k conj(G[k,x]) E[k, x ^ bit_i]
 * out_diag[i*n+j] (i<=j) = sum_x x_i x_j rho(x)        (complex; i==j gives sum x_i rho)
 * out_flip[i] = (sum_{x: x_i=1} tau_i(x), sum_{x: x_i=0} tau_i(x))   (2 complex per i)
 * G and E are m x D. */
void or_grad_contract(int n, int m, const double *G, const double *E, double *out_diag,
                      double *out_flip)
{
    i64 D = (i64)1 << n;
    memset(out_diag, 0, sizeof(double) * 2 * n * n);
    memset(out_flip, 0, sizeof(double) * 4 * n);
#pragma omp parallel if (PAR(D))
    {
        double ld[2 * 32 * 32];
        double lf[4 * 32];
        memset(ld, 0, sizeof(ld));
        memset(lf, 0, sizeof(lf));
#pragma omp for schedule(static)
        for (i64 x = 0; x < D; ++x) {
            double rr = 0.0, ri = 0.0;
            for (int k = 0; k < m; ++k) {
                const double *g = G + 2 * ((i64)k * D + x), *e = E + 2 * ((i64)k * D + x);
                rr += g[0] * e[0] + g[1] * e[1];
                ri += g[0] * e[1] - g[1] * e[0];
            }
            for (int i = 0; i < n; ++i) {
                if (!bit_of(x, n, i)) continue;
                for (int j = i; j < n; ++j)
                    if (bit_of(x, n, j)) {
                        ld[2 * (i * 32 + j)] += rr;
                        ld[2 * (i * 32 + j) + 1] += ri;
                    }
            }
            for (int i = 0; i < n; ++i) {
                i64 y = x ^ ((i64)1 << (n - 1 - i));
                double tr = 0.0, ti = 0.0;
                for (int k = 0; k < m; ++k) {
                    const double *g = G + 2 * ((i64)k * D + x), *e = E + 2 * ((i64)k * D + y);
                    tr += g[0] * e[0] + g[1] * e[1];
                    ti += g[0] * e[1] - g[1] * e[0];
                }
                int s = bit_of(x, n, i) ? 0 : 1;
                lf[4 * i + 2 * s] += tr;
                lf[4 * i + 2 * s + 1] += ti;
            }
        }
#pragma omp critical
        {
            for (int i = 0; i < n; ++i)
                for (int j = i; j < n; ++j) {
                    out_diag[2 * (i * n + j)] += ld[2 * (i * 32 + j)];
                    out_diag[2 * (i * n + j) + 1] += ld[2 * (i * 32 + j) + 1];
                }
            for (int k = 0; k < 4 * n; ++k) out_flip[k] += lf[k];
        }
    }
}
