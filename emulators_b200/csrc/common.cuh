// Shared device/host helpers for the emusv_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "emusv_b200.h"

namespace emusv {

constexpr int MAXQ = 32;        // parameter tables are sized for up to 32 qubits
constexpr int BLOCK = 256;      // threads per block of the streaming kernels
constexpr int NRED = 8;         // FP64 partial sums a streaming kernel can emit

typedef int64_t i64;

// ---------------------------------------------------------------- complex storage
template <typename R> struct cvec;
template <> struct cvec<double> { typedef double2 T; };
template <> struct cvec<float> { typedef float2 T; };

template <typename C> __device__ __forceinline__ C cmake(double re, double im);
template <> __device__ __forceinline__ double2 cmake<double2>(double re, double im) {
    return make_double2(re, im);
}
template <> __device__ __forceinline__ float2 cmake<float2>(double re, double im) {
    return make_float2((float)re, (float)im);
}

__device__ __forceinline__ float fmar(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmar(double a, double b, double c) { return fma(a, b, c); }

// ---------------------------------------------------------------- Hamiltonian block
// Parameters by BIT POSITION p = n-1-i of qubit i (bit 0 = least significant).
struct HamParams {
    int n;
    int real_coef;             // 1 when every phase is zero: up == dn == Omega/2 (real)
    double up_re[MAXQ];        // coefficient of |r><g| on bit p (target bit 1)
    double up_im[MAXQ];
    double dn_re[MAXQ];        // coefficient of |g><r| (target bit 0)
    double dn_im[MAXQ];
    double field[MAXQ];        // -delta (plus the real part of the noise per excitation)
    double U[MAXQ * MAXQ];     // symmetric U by bit positions, zero diagonal
    // non-Hermitian noise term -0.5i sum_j L_j^dag L_j (the same 2x2 matrix on every
    // qubit, hamiltonian.py:61-67,147-151): its off-diagonal entries are added to up/dn,
    // the real part of its diagonal to field[] and dc_re; the imaginary part of the
    // diagonal of x is dc_im + dg_im * popcount(x)
    int noisy;
    double dc_re, dc_im, dg_im;
};

// Build a HamParams from host arrays in reference (qubit) order.
// Returns false on a bad argument.
bool make_params(int n, const double *omegas, const double *deltas, const double *phis,
                 const double *interaction, HamParams *P);
// Add the noise matrix `noise` (2x2 complex, row-major, re/im interleaved: 8 doubles) to
// P.  Returns false on a non-finite entry.
bool add_noise(const double *noise, HamParams *P);

// The jump term of a Lindbladian on a density matrix stored as a vector of 2N bits (row
// index in the high N bits): i sum_q K_q, K = sum_k L_k (x) conj(L_k) acting on the row
// bit and the column bit of qubit q; K[(i*2 + j)*4 + (i'*2 + j')] (re, im interleaved).
struct LindbladJumps {
    int nq;          // N
    unsigned mask;   // nonzero entries of K
    double K[32];
};
// out += i * (*su) * sum_q K_q u  (device vectors of 4^N amplitudes); returns at once when
// *gate != 0.
int launch_lindblad_jumps(int dtype, const LindbladJumps &J, const void *u, const double *su,
                          void *out, const int *gate, cudaStream_t s);

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread; result valid in thread 0. `scratch` holds
// (blockDim/32) * NV doubles.  Must be called by all threads of the block.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) scratch[warp * NV + k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nw; ++w) {
#pragma unroll
            for (int k = 0; k < NV; ++k) v[k] += scratch[w * NV + k];
        }
    }
    __syncthreads();
}

// Deterministic sum of per-block partials: partials[b * stride + k], b < nblocks.
// Every thread of the calling block gets the same result (fixed order).
template <int NV>
__device__ __forceinline__ void sum_partials(const double *partials, int nblocks, int stride,
                                             double (&out)[NV], double *scratch) {
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += partials[(i64)b * stride + k];
    }
    block_sum<NV>(v, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) scratch[k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = scratch[k];
    __syncthreads();
}

// ---------------------------------------------------------------- host helpers
int sm_count();                       // SMs of the current device (cached per device)
int stream_status(cudaError_t e);     // map a CUDA error to emusv_status
int *device_error_word();             // library-wide device error word (current device)
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace emusv

#define EMUSV_CHECK(call)                                   \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return emusv::stream_status(e_); \
    } while (0)

#define EMUSV_CHECK_LAUNCH() EMUSV_CHECK(cudaGetLastError())
