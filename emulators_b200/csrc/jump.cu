// Quantum-jump helpers of the Monte Carlo stepper (C ABI emusv_qubit_densities,
// emusv_apply_1q): the single-qubit reduced density matrices of a state, whose traces with
// L^dag L give the jump weights of every (qubit, operator) pair (emu_sv/algebra.py:4-25,
// expect_batch), and a 2x2 operator applied to one qubit in place (algebra.py:28-37).
#include "hpsi_kernel.cuh"
#include "profile.cuh"

namespace emusv {

constexpr int RHO_THREADS = 256;

// partials[block][p][4]: sum over pairs (x0, x1 = x0 | 2^p) of |psi_x0|^2, |psi_x1|^2 and
// psi_x1 conj(psi_x0) (re, im), for every bit p.
template <typename R>
__global__ void __launch_bounds__(RHO_THREADS) k_qubit_rho(const void *psi_, int n, double *partials) {
    typedef typename cvec<R>::T C;
    const C *psi = reinterpret_cast<const C *>(psi_);
    __shared__ double red[(RHO_THREADS / 32) * 4];
    const i64 half = i64(1) << (n - 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int p = 0; p < n; ++p) {
        const i64 lowmask = (i64(1) << p) - 1;
        double a00 = 0.0, a11 = 0.0, cr = 0.0, ci = 0.0;
        for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += (i64)gridDim.x * blockDim.x) {
            const i64 x0 = ((i >> p) << (p + 1)) | (i & lowmask);
            const C a = psi[x0], b = psi[x0 | (i64(1) << p)];
            const double ar = double(a.x), ai = double(a.y), br = double(b.x), bi = double(b.y);
            a00 += ar * ar + ai * ai;
            a11 += br * br + bi * bi;
            cr += br * ar + bi * ai;  // b conj(a)
            ci += bi * ar - br * ai;
        }
        a00 = warp_sum(a00);
        a11 = warp_sum(a11);
        cr = warp_sum(cr);
        ci = warp_sum(ci);
        if (lane == 0) {
            red[warp * 4 + 0] = a00;
            red[warp * 4 + 1] = a11;
            red[warp * 4 + 2] = cr;
            red[warp * 4 + 3] = ci;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w * 4 + threadIdx.x];
            partials[((i64)blockIdx.x * MAXQ + p) * 4 + threadIdx.x] = t;
        }
        __syncthreads();
    }
}

// rho[i] (qubit i = bit n-1-i): 2x2 complex row-major, 8 doubles: [00, 01, 10, 11].
__global__ void k_finish_rho(const double *partials, int nb, int n, double *rho) {
    const int i = threadIdx.x;
    if (i >= n) return;
    const int p = n - 1 - i;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < 4; ++k) v[k] += partials[((i64)b * MAXQ + p) * 4 + k];
    double *o = rho + 8 * i;
    o[0] = v[0];  // rho_00
    o[1] = 0.0;
    o[2] = v[2];  // rho_01 = sum psi_0 conj(psi_1) = conj(rho_10)
    o[3] = -v[3];
    o[4] = v[2];  // rho_10 = sum psi_1 conj(psi_0)
    o[5] = v[3];
    o[6] = v[1];  // rho_11
    o[7] = 0.0;
}

template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_apply_1q(void *psi_, int n, int p, double o00r, double o00i, double o01r, double o01i, double o10r,
           double o10i, double o11r, double o11i) {
    typedef typename cvec<R>::T C;
    C *psi = reinterpret_cast<C *>(psi_);
    const i64 half = i64(1) << (n - 1);
    const i64 lowmask = (i64(1) << p) - 1;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += (i64)gridDim.x * blockDim.x) {
        const i64 x0 = ((i >> p) << (p + 1)) | (i & lowmask), x1 = x0 | (i64(1) << p);
        const C a = psi[x0], b = psi[x1];
        const double ar = double(a.x), ai = double(a.y), br = double(b.x), bi = double(b.y);
        psi[x0] = cmake<C>(o00r * ar - o00i * ai + o01r * br - o01i * bi,
                           o00r * ai + o00i * ar + o01r * bi + o01i * br);
        psi[x1] = cmake<C>(o10r * ar - o10i * ai + o11r * br - o11i * bi,
                           o10r * ai + o10i * ar + o11r * bi + o11i * br);
    }
}

static int rho_grid(int n) {
    const i64 half = i64(1) << (n - 1);
    i64 g = (half + RHO_THREADS - 1) / RHO_THREADS;
    const i64 cap = (i64)sm_count() * 4;
    return (int)(g < cap ? g : cap);
}

}  // namespace emusv

using namespace emusv;

extern "C" {

size_t emusv_qubit_densities_scratch_bytes(int nqubits) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS) return 0;
    return sizeof(double) * (size_t)sm_count() * 4 * MAXQ * 4 + 256;
}

int emusv_qubit_densities(int nqubits, int dtype, const void *psi, double *rho_dev, void *scratch,
                          size_t scratch_bytes, void *stream) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS || !psi || !rho_dev || !scratch ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64) ||
        scratch_bytes < emusv_qubit_densities_scratch_bytes(nqubits))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    double *partials = reinterpret_cast<double *>(scratch);
    const int g = rho_grid(nqubits);
    {
        ProfScope ps_(PROF_OBS, s);
        if (dtype == EMUSV_C128) k_qubit_rho<double><<<g, RHO_THREADS, 0, s>>>(psi, nqubits, partials);
        else k_qubit_rho<float><<<g, RHO_THREADS, 0, s>>>(psi, nqubits, partials);
        k_finish_rho<<<1, 32, 0, s>>>(partials, g, nqubits, rho_dev);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

int emusv_apply_1q(int nqubits, int dtype, void *psi, int qubit, const double *op, void *stream) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS || !psi || !op || qubit < 0 || qubit >= nqubits ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64))
        return EMUSV_BAD_ARGUMENT;
    for (int k = 0; k < 8; ++k)
        if (!isfinite(op[k])) return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const int p = nqubits - 1 - qubit;
    const i64 half = i64(1) << (nqubits - 1);
    i64 g = (half + BLOCK - 1) / BLOCK;
    if (g > (i64)sm_count() * 8) g = (i64)sm_count() * 8;
    {
        ProfScope ps_(PROF_OBS, s);
        if (dtype == EMUSV_C128)
            k_apply_1q<double><<<(int)g, BLOCK, 0, s>>>(psi, nqubits, p, op[0], op[1], op[2], op[3],
                                                         op[4], op[5], op[6], op[7]);
        else
            k_apply_1q<float><<<(int)g, BLOCK, 0, s>>>(psi, nqubits, p, op[0], op[1], op[2], op[3],
                                                        op[4], op[5], op[6], op[7]);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

}  // extern "C"
