// Bitstring sampling by inverting the cumulative distribution of |psi|^2 (C ABI
// emusv_sample), the large-register path of emu_sv/utils.py:17-49 (sample_indices:
// cdf = cumsum(p) in FP64, index = searchsorted(cdf / cdf[-1], u, right=True), clamped)
// without materialising the CDF:
//   1. per-block FP64 sums of |psi|^2 over blocks of SB amplitudes (one pass over psi);
//   2. one CTA: exclusive prefix of the block sums (FP64);
//   3. one warp per draw: binary search of the block whose prefix range holds u * total,
//      then a warp-wide running prefix over that block's amplitudes to the first index
//      whose cumulative sum exceeds u * total (right-continuous, as searchsorted right=True).
#include "hpsi_kernel.cuh"
#include "profile.cuh"

namespace emusv {

constexpr int SB_BITS = 12;  // amplitudes per block sum
constexpr int SCAN_THREADS = 1024;

template <typename R>
__global__ void __launch_bounds__(BLOCK) k_block_sums(const void *psi_, i64 D, double *bsum) {
    typedef typename cvec<R>::T C;
    const C *psi = reinterpret_cast<const C *>(psi_);
    __shared__ double red[BLOCK / 32];
    const i64 SB = i64(1) << SB_BITS;
    const i64 nb = (D + SB - 1) / SB;
    for (i64 b = blockIdx.x; b < nb; b += gridDim.x) {
        double acc = 0.0;
        const i64 lo = b * SB, hi = lo + SB < D ? lo + SB : D;
        for (i64 x = lo + threadIdx.x; x < hi; x += blockDim.x) {
            const C v = psi[x];
            acc = fma(double(v.x), double(v.x), fma(double(v.y), double(v.y), acc));
        }
        acc = warp_sum(acc);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x < 32) {
            double t = threadIdx.x < BLOCK / 32 ? red[threadIdx.x] : 0.0;
            t = warp_sum(t);
            if (threadIdx.x == 0) bsum[b] = t;
        }
        __syncthreads();
    }
}

// prefix[b] = sum of bsum[0..b), prefix[nb] = total (one CTA, FP64, sequential chunks).
__global__ void __launch_bounds__(SCAN_THREADS) k_block_prefix(const double *bsum, i64 nb, double *prefix) {
    __shared__ double part[SCAN_THREADS];
    const i64 per = (nb + SCAN_THREADS - 1) / SCAN_THREADS;
    const i64 lo = threadIdx.x * per, hi = lo + per < nb ? lo + per : nb;
    double s = 0.0;
    for (i64 b = lo; b < hi; ++b) s += bsum[b];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive scan of the chunk totals
        double run = 0.0;
        for (int t = 0; t < SCAN_THREADS; ++t) {
            const double v = part[t];
            part[t] = run;
            run += v;
        }
        prefix[nb] = run;
    }
    __syncthreads();
    double run = part[threadIdx.x];
    for (i64 b = lo; b < hi; ++b) {
        prefix[b] = run;
        run += bsum[b];
    }
}

template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_draw(const void *psi_, i64 D, const double *prefix, i64 nb, const double *u, int shots,
       long long *out, int *bad) {
    typedef typename cvec<R>::T C;
    const C *psi = reinterpret_cast<const C *>(psi_);
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= shots) return;
    const double total = prefix[nb];
    if (!(total > 0.0)) {
        if (lane == 0) *bad = 1;
        return;
    }
    const double t = u[w] * total;
    // last block whose start prefix is <= t (prefix is non-decreasing, prefix[0] = 0)
    i64 lo = 0, hi = nb - 1;
    while (lo < hi) {
        const i64 mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const i64 SB = i64(1) << SB_BITS;
    double run = prefix[lo];
    long long found = -1;
    for (i64 x0 = lo * SB; x0 < D && found < 0; x0 += 32) {
        const i64 x = x0 + lane;
        double p = 0.0;
        if (x < D) {
            const C v = psi[x];
            p = fma(double(v.x), double(v.x), double(v.y) * double(v.y));
        }
        // inclusive warp scan of p
        double sc = p;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double n = __shfl_up_sync(0xffffffffu, sc, o);
            if (lane >= o) sc += n;
        }
        const unsigned hit = __ballot_sync(0xffffffffu, x < D && run + sc > t);
        if (hit) found = x0 + __ffs(hit) - 1;
        run += __shfl_sync(0xffffffffu, sc, 31);
    }
    if (lane == 0) out[w] = found < 0 ? (long long)(D - 1) : found;  // searchsorted clamp
}

}  // namespace emusv

using namespace emusv;

extern "C" {

size_t emusv_sample_scratch_bytes(int nqubits) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS) return 0;
    const i64 nb = ((i64(1) << nqubits) + (i64(1) << SB_BITS) - 1) >> SB_BITS;
    return sizeof(double) * (size_t)(2 * nb + 1) + 256;
}

int emusv_sample(int nqubits, int dtype, const void *psi, int num_shots, const double *uniforms,
                 long long *indices, void *scratch, size_t scratch_bytes, void *stream) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS || !psi || num_shots < 0 || !uniforms ||
        !indices || !scratch || (dtype != EMUSV_C128 && dtype != EMUSV_C64) ||
        scratch_bytes < emusv_sample_scratch_bytes(nqubits))
        return EMUSV_BAD_ARGUMENT;
    if (num_shots == 0) return EMUSV_OK;
    cudaStream_t s = as_stream(stream);
    const i64 D = i64(1) << nqubits;
    const i64 nb = (D + (i64(1) << SB_BITS) - 1) >> SB_BITS;
    double *bsum = reinterpret_cast<double *>(scratch);
    double *prefix = bsum + nb;
    int *bad = reinterpret_cast<int *>(prefix + nb + 1);
    EMUSV_CHECK(cudaMemsetAsync(bad, 0, sizeof(int), s));
    {
        ProfScope ps_(PROF_OBS, s);
        const int g = (int)(nb < 4 * sm_count() ? nb : 4 * sm_count());
        if (dtype == EMUSV_C128) k_block_sums<double><<<g, BLOCK, 0, s>>>(psi, D, bsum);
        else k_block_sums<float><<<g, BLOCK, 0, s>>>(psi, D, bsum);
        k_block_prefix<<<1, SCAN_THREADS, 0, s>>>(bsum, nb, prefix);
        const int gd = (int)(((i64)num_shots * 32 + BLOCK - 1) / BLOCK);
        if (dtype == EMUSV_C128)
            k_draw<double><<<gd, BLOCK, 0, s>>>(psi, D, prefix, nb, uniforms, num_shots, indices, bad);
        else
            k_draw<float><<<gd, BLOCK, 0, s>>>(psi, D, prefix, nb, uniforms, num_shots, indices, bad);
    }
    EMUSV_CHECK_LAUNCH();
    int hbad = 0;
    EMUSV_CHECK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));
    return hbad ? EMUSV_NONFINITE : EMUSV_OK;
}

}  // extern "C"
