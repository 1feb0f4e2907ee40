// Drive preparation on the GPU (C ABI emusv_pchip_eval): shape-preserving piecewise-cubic
// Hermite interpolation (PCHIP) of many sampled signals at many query times, the
// interpolation the reference's adapter runs per qubit and per laser parameter to get the
// midpoint drive samples (emu_base/math/pchip_torch.py:218-269 PCHIP1D;
// emu_base/pulser_adapter.py:155-231).
//
// One thread per (signal, query): the interval is found by binary search over the shared
// knots (searchsorted right=True, clamped to [0, n-2]); the two knot derivatives of that
// interval are rebuilt from at most four neighbouring secants (weighted harmonic mean of
// same-sign neighbours, else 0; one-sided three-point estimate with the sign and 3x limiter
// at the ends; the secant itself for two knots) and the cubic is evaluated in Horner form.
// Every operation is rounded separately in the reference's order (no contraction into
// FMAs), so the values equal the reference's float64 ones.
#include "common.cuh"
#include "profile.cuh"

namespace emusv {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// secant slope of interval k: (y[k+1] - y[k]) / (x[k+1] - x[k])
__device__ __forceinline__ double secant(const double *x, const double *y, int k) {
    return ddiv(dsub(y[k + 1], y[k]), dsub(x[k + 1], x[k]));
}

// _weighted_harmonic_mean (pchip_torch.py:97-106)
__device__ __forceinline__ double harmonic(double dl, double dr, double hl, double hr) {
    const double wl = dadd(hl, dmul(2.0, hr));
    const double wr = dadd(dmul(2.0, hl), hr);
    return ddiv(dadd(wl, wr), dadd(ddiv(wl, dl), ddiv(wr, dr)));
}

// _endpoint_slope + _limit_endpoint (pchip_torch.py:109-143)
__device__ __forceinline__ double endpoint(double dl, double dr, double hl, double hr) {
    const double w1 = dadd(dmul(2.0, hl), hr);
    double d = ddiv(dsub(dmul(w1, dl), dmul(hl, dr)), dadd(hl, hr));
    if (dmul(d, dl) < 0.0) d = 0.0;
    if (dmul(dl, dr) < 0.0 && fabs(d) > dmul(3.0, fabs(dl))) d = dmul(3.0, dl);
    return d;
}

// knot derivative d[k] (pchip_torch.py:146-184)
__device__ double knot_slope(const double *x, const double *y, int n, int k) {
    if (n == 2) return secant(x, y, 0);
    if (k == 0)
        return endpoint(secant(x, y, 0), secant(x, y, 1), dsub(x[1], x[0]), dsub(x[2], x[1]));
    if (k == n - 1)
        return endpoint(secant(x, y, n - 2), secant(x, y, n - 3), dsub(x[n - 1], x[n - 2]),
                        dsub(x[n - 2], x[n - 3]));
    const double dl = secant(x, y, k - 1), dr = secant(x, y, k);
    if (!(dmul(dl, dr) > 0.0)) return 0.0;
    return harmonic(dl, dr, dsub(x[k], x[k - 1]), dsub(x[k + 1], x[k]));
}

__global__ void __launch_bounds__(BLOCK)
k_pchip(int n, const double *__restrict__ x, int nsig, const double *__restrict__ y, i64 ystride,
        int nq, const double *__restrict__ xq, double *__restrict__ out, i64 ostride) {
    const i64 total = (i64)nsig * nq;
    for (i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (i64)gridDim.x * blockDim.x) {
        const int s = (int)(g / nq), q = (int)(g % nq);
        const double t = xq[q];
        // searchsorted(x, t, right=True) - 1, clamped to [0, n-2]
        int lo = 0, hi = n;  // first index with x > t lies in [lo, hi]
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (x[mid] <= t) lo = mid + 1; else hi = mid;
        }
        int i = lo - 1;
        i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
        const double *ys = y + (i64)s * ystride;
        const double h = dsub(x[i + 1], x[i]);
        const double delta = secant(x, ys, i);
        const double di = knot_slope(x, ys, n, i), dj = knot_slope(x, ys, n, i + 1);
        // _polynomial_coeffs (pchip_torch.py:187-215)
        const double p0 = ys[i], p1 = di;
        const double p2 = ddiv(dsub(dsub(dmul(3.0, delta), dmul(2.0, di)), dj), h);
        const double p3 = ddiv(dsub(dadd(di, dj), dmul(2.0, delta)), dmul(h, h));
        const double u = dsub(t, x[i]);
        // p0 + t * (p1 + t * (p2 + t * p3))  (pchip_torch.py:262-269)
        out[(i64)s * ostride + q] = dadd(p0, dmul(u, dadd(p1, dmul(u, dadd(p2, dmul(u, p3))))));
    }
}

}  // namespace emusv

using namespace emusv;

extern "C" {

int emusv_pchip_eval(int nknots, const double *x, int nsignals, const double *y, int64_t y_stride,
                     int nqueries, const double *xq, double *out, int64_t out_stride, void *stream) {
    if (nknots < 2 || nsignals < 0 || nqueries < 0 || !x || !xq || !y || !out || y_stride < nknots ||
        out_stride < nqueries)
        return EMUSV_BAD_ARGUMENT;
    const i64 total = (i64)nsignals * nqueries;
    if (total == 0) return EMUSV_OK;
    cudaStream_t s = as_stream(stream);
    i64 g = (total + BLOCK - 1) / BLOCK;
    if (g > (i64)sm_count() * 16) g = (i64)sm_count() * 16;
    {
        ProfScope ps_(PROF_OBS, s);
        k_pchip<<<(int)g, BLOCK, 0, s>>>(nknots, x, nsignals, y, y_stride, nqueries, xq, out, out_stride);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

}  // extern "C"
