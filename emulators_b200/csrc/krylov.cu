// Lanczos time step exp(-i dt H) psi on the GPU (C ABI emusv_krylov_step) and the
// building blocks of the generic krylov_exp.
//
// Per Lanczos iteration j (reference emu_base/math/krylov_exp.py:49-96), registers wider
// than one pass-L tile (the H-first order, lanczos_run):
//   1. pass H kernels (k_pass_high, EPI_X_FIRST / EPI_X_ADD): part = the flips of the bits
//      above the pass-L tile applied to v_j, and their share of <v_j, H v_j>;
//   2. k_lz_coef: a_j = <v_j, H v_j> - b_j <v_j, v_{j-1}> with b_j = ||w_{j-1}|| (the
//      modified Gram-Schmidt values of krylov_exp.py:55-58 in exact arithmetic);
//   3. pass L (k_pass_lz): H v_j formed tile by tile on chip, w = H v_j - a_j v_j -
//      b_j v_{j-1} stored into basis slot j+1, FP64 partials of ||w||^2, <v_j, w>,
//      ||H v_j||^2 and the pass-L share of the next <v, H v>;
//   4. k_lz_norms (one warp): ||w||, ||H v_j||, the next scale and the happy-breakdown
//      test (krylov_exp.py:63-71) -- all the next iteration needs;
//   5. k_lz_decide (one warp, on a second stream, overlapping iteration j+1): the
//      exponential of the extended Krylov matrix and the Expokit error estimate
//      (krylov_exp.py:77-86), all FP64 on the device.
// Smaller registers: k_hpsi<HP_LANCZOS> (H v with its reductions), k_orth (the recurrence),
// k_small.
// Basis vectors are stored unnormalised with a device scale factor (v_k = scale_k u_k),
// so no separate normalisation pass exists; the input vector is basis vector 0 in place.
// Every kernel after the first reads a device status word and exits at once when the
// iteration has already finished, so the host only synchronises where it tests
// convergence.
#include <string.h>

#include <mutex>

#include "krylov_device.cuh"
#include "profile.cuh"

namespace emusv {

int hpsi_tile_bits(int n);
int launch_hpsi(int dtype, int mode, const HamParams &P, HpsiArgs A, int max_grid,
                cudaStream_t s, int *grid_out);
bool lanczos_h_first(int dtype, int n);
int lz_energy0(int dtype, const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out);
int lz_low(int dtype, const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out);
int lz_high(int dtype, const HamParams &H, const void *u, void *part, double *partials, const int *gate,
            int *err, unsigned *cnt, cudaStream_t s, int *nblocks_out);
int max_grid_blocks();

struct Workspace {
    KState *ks;
    double *part_h, *part_o, *part_c;
    unsigned char *basis;
    size_t basis_bytes;
};

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static size_t header_bytes() {
    return align_up(sizeof(KState), 256) + 3 * align_up(sizeof(double) * max_grid_blocks() * NRED, 256);
}

static Workspace carve(void *ws, size_t bytes) {
    Workspace W;
    unsigned char *p = reinterpret_cast<unsigned char *>(ws);
    size_t off = 0;
    W.ks = reinterpret_cast<KState *>(p);
    off += align_up(sizeof(KState), 256);
    const size_t pb = align_up(sizeof(double) * max_grid_blocks() * NRED, 256);
    W.part_h = reinterpret_cast<double *>(p + off);
    off += pb;
    W.part_o = reinterpret_cast<double *>(p + off);
    off += pb;
    W.part_c = reinterpret_cast<double *>(p + off);
    off += pb;
    W.basis = p + off;
    W.basis_bytes = bytes > off ? bytes - off : 0;
    return W;
}

static int stream_grid(i64 D) {
    i64 g = (D + BLOCK - 1) / BLOCK;
    const i64 cap = (i64)sm_count() * 4;
    return (int)(g < cap ? g : cap);
}

// ---------------------------------------------------------------- small kernels
template <typename R>
__global__ void __launch_bounds__(BLOCK) k_norm2(const void *v_, i64 D, double *partials) {
    typedef typename cvec<R>::T C;
    const C *v = reinterpret_cast<const C *>(v_);
    __shared__ double red[(BLOCK / 32) * NRED];
    double acc[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) acc[k] = 0.0;
    for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < D; x += (i64)gridDim.x * blockDim.x) {
        const C a = v[x];
        acc[0] += double(a.x) * double(a.x) + double(a.y) * double(a.y);
    }
    block_sum<NRED>(acc, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < NRED; ++k) partials[(i64)blockIdx.x * NRED + k] = acc[k];
}

// Start of a run: the input norm, and sigma, the energy the run subtracts from H.  With
// energy_shift, sigma = the previous run's <v_0, H v_0> (sigma_prev + a_0) when that run
// finished, else 0.  The Lanczos recurrence of H - sigma has the same basis and the
// tridiagonal matrix minus sigma (a_k is stored shifted); the exponentials add sigma back
// (load_rows), so coefficients and error estimates are those of H itself -- only the
// complex64 rounding of the diagonal inside H*psi shrinks.
__global__ void k_init(KState *ks, const double *partials, int nblocks, int energy_shift) {
    __shared__ double red[(BLOCK / 32) * NRED];
    double v[NRED];
    sum_partials<NRED>(partials, nblocks, NRED, v, red);
    if (threadIdx.x == 0) {
        double sh = 0.0;
        if (energy_shift && (ks->status == KS_CONVERGED || ks->status == KS_HAPPY) && ks->iters > 0) {
            sh = ks->shift + ks->a_re[0];
            if (!isfinite(sh) || fabs(sh) > 1e12) sh = 0.0;
        }
        ks->shift = sh;
        const double s0 = sqrt(v[0]);  // krylov_exp.py:43
        ks->s0 = s0;
        ks->scale[0] = 1.0 / s0;       // krylov_exp.py:44 (applied on load)
        ks->status = (isfinite(s0) && s0 > 0.0) ? KS_RUNNING : KS_NONFINITE;
        ks->iters = 0;
        ks->nvec = 0;
        ks->kerr = 0;
        ks->err = 0.0;
        ks->outnorm2 = 0.0;
    }
}

// Three-term recurrence w <- H v_j - b v_{j-1} - a v_j with b = ||w_{j-1}|| (which equals
// <v_{j-1}, H v_j> in exact arithmetic) and a = <v_j, H v_j> - b <v_j, v_{j-1}>, the
// modified Gram-Schmidt value of krylov_exp.py:55-58 with the measured non-orthogonality
// <v_j, v_{j-1}> carried over from the previous iteration.  FP64 partials: ||w||^2 and
// <v_j, w> (the next iteration's <v_{j+1}, v_j>).
template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_orth(KState *ks, int j, const double *part_h, int nb_h, const void *vj_, const void *vp_,
       void *w_, i64 D, double *part_o) {
    typedef typename cvec<R>::T C;
    if (ks->status != KS_RUNNING) return;
    __shared__ double red[(BLOCK / 32) * NRED];
    double s[NRED];
    sum_partials<NRED>(part_h, nb_h, NRED, s, red);
    // s: 0 ||Hv||^2, 1-2 <v,Hv>
    const double b = j > 0 ? ks->r[j - 1] : 0.0;
    const double cr = j > 0 ? ks->vv_re[j] : 0.0, ci = j > 0 ? ks->vv_im[j] : 0.0;
    const double ar = s[1] - b * cr;
    const double ai = s[2] - b * ci;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ks->a_re[j] = ar;
        ks->a_im[j] = ai;
        ks->b_re[j] = b;
        ks->b_im[j] = 0.0;
        // ||H v||^2 = ||(H - sigma) v||^2 + 2 sigma Re<v,(H - sigma) v> + sigma^2
        const double sg = ks->shift;
        ks->hn[j] = sqrt(fmax(0.0, s[0] + 2.0 * sg * s[1] + sg * sg));
    }
    const double sj = ks->scale[j];
    const double sp = j > 0 ? ks->scale[j - 1] : 0.0;
    // coefficients on the stored (unscaled) vectors
    const double car = ar * sj, cai = ai * sj, cb = b * sp;
    const C *vj = reinterpret_cast<const C *>(vj_);
    const C *vp = reinterpret_cast<const C *>(vp_);
    C *w = reinterpret_cast<C *>(w_);
    double acc[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) acc[k] = 0.0;
    for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < D; x += (i64)gridDim.x * blockDim.x) {
        const C h = w[x];
        const C a = vj[x];
        double wr = double(h.x) - (car * double(a.x) - cai * double(a.y));
        double wi = double(h.y) - (car * double(a.y) + cai * double(a.x));
        if (j > 0) {
            const C p = vp[x];
            wr -= cb * double(p.x);
            wi -= cb * double(p.y);
        }
        const C o = cmake<C>(wr, wi);
        w[x] = o;
        const double orr = double(o.x), oi = double(o.y);
        const double vr = sj * double(a.x), vi = sj * double(a.y);
        acc[0] += orr * orr + oi * oi;
        acc[1] += vr * orr + vi * oi;  // <v_j, w>
        acc[2] += vr * oi - vi * orr;
    }
    block_sum<NRED>(acc, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < NRED; ++k) part_o[(i64)blockIdx.x * NRED + k] = acc[k];
}

// H-first iteration j: <v_j, (H - sigma) v_j> is the pass-L part el (computed by the pass
// that produced v_j -- the previous iteration's pass L, or for j = 0 the start-of-run
// energy pass, partials 4-5 of part_e0) plus the pass-H part (partials 0-1 of part_h, on
// the stored vector: times scale_j^2); a, b and the recurrence coefficients on the stored
// vectors follow.
__global__ void k_lz_coef(KState *ks, int j, const double *part_h, int nb_h, const double *part_e0,
                          int nb_e0) {
    if (ks->status != KS_RUNNING) return;
    __shared__ double red[(BLOCK / 32) * NRED];
    double s[NRED], e0[NRED];
    sum_partials<NRED>(part_h, nb_h, NRED, s, red);
    if (j == 0) sum_partials<NRED>(part_e0, nb_e0, NRED, e0, red);
    if (threadIdx.x == 0) {
        const double sj = ks->scale[j], s2 = sj * sj;
        double elr, eli;
        if (j == 0) {
            elr = e0[4] * s2;
            eli = e0[5] * s2;
            ks->el_re[0] = elr;
            ks->el_im[0] = eli;
        } else {
            elr = ks->el_re[j];
            eli = ks->el_im[j];
        }
        const double er = elr + s[0] * s2, ei = eli + s[1] * s2;
        const double b = j > 0 ? ks->r[j - 1] : 0.0;
        const double cr = j > 0 ? ks->vv_re[j] : 0.0, ci = j > 0 ? ks->vv_im[j] : 0.0;
        const double ar = er - b * cr, ai = ei - b * ci;
        ks->a_re[j] = ar;
        ks->a_im[j] = ai;
        ks->b_re[j] = b;
        ks->b_im[j] = 0.0;
        ks->e_re[j] = er;
        const double sp = j > 0 ? ks->scale[j - 1] : 0.0;
        ks->ocoef[0] = ar * sj;
        ks->ocoef[1] = ai * sj;
        ks->ocoef[2] = b * sp;
    }
}

// Decide iteration j (krylov_decide) from the orthogonalisation's partial sums.  Later
// kernels of the step return at once once the status leaves KS_RUNNING.
__global__ void __launch_bounds__(32)
k_small(KState *ks, int j, const double *part_o, int nb_o, double dt, double exp_tol,
        double norm_tol, int poll, int first_poll, int maxdim) {
    if (ks->status != KS_RUNNING) return;
    if (ks->kerr) {  // a streaming kernel gave up on a bounded wait
        if (threadIdx.x == 0) {
            ks->status = KS_TIMEOUT;
            ks->iters = j + 1;
        }
        return;
    }
    const int lane = threadIdx.x;
    // deterministic sums of the ||w||^2 and <v_j, w> partials by one warp
    double v = 0.0, vr = 0.0, vi = 0.0;
    for (int b = lane; b < nb_o; b += 32) {
        v += part_o[(i64)b * NRED];
        vr += part_o[(i64)b * NRED + 1];
        vi += part_o[(i64)b * NRED + 2];
    }
    v = warp_sum(v);
    vr = warp_sum(vr);
    vi = warp_sum(vi);
    krylov_decide(ks, j, v, vr, vi, dt, exp_tol, norm_tol, poll != 0, first_poll != 0, maxdim);
}

// H-first iteration j, first part (on the step's stream): from the pass-L partials
// (0 ||w||^2, 1-2 <v_j, w>, 3 ||(H - sigma) v_j||^2, 4 the pass-L part of <w, (H - sigma) w>)
// ||H v_j||, ||w||, <v_{j+1}, v_j>, scale_{j+1} and the next el -- everything iteration
// j+1 needs -- and the outcome flag; no status change.
__global__ void __launch_bounds__(BLOCK)
k_lz_norms(KState *ks, int j, const double *part_o, int nb_o, double dt, double norm_tol) {
    if (ks->status != KS_RUNNING) return;
    // the whole block sums the partial rows (one row or two per thread, all loads in
    // flight at once), then warp 0 decides
    __shared__ double red[(BLOCK / 32) * NRED];
    double sums[NRED];
    sum_partials<NRED>(part_o, nb_o, NRED, sums, red);
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const double v = sums[0], vr = sums[1], vi = sums[2], hh = sums[3], el = sums[4];
    if (lane == 0) {
        // ||H v||^2 = ||(H - sigma) v||^2 + 2 sigma Re<v,(H - sigma) v> + sigma^2
        const double sg = ks->shift;
        ks->hn[j] = sqrt(fmax(0.0, hh + 2.0 * sg * ks->e_re[j] + sg * sg));
    }
    __syncwarp();
    const int flag = krylov_norms(ks, j, v, vr, vi, dt, norm_tol);
    if (lane == 0) {
        ks->lz_flag[j] = flag;
        ks->el_re[j + 1] = v > 0.0 ? el / v : 0.0;  // v_{j+1} = w / ||w||
        ks->el_im[j + 1] = 0.0;
    }
}

// Second part (on the decision stream, in iteration order, overlapping the next
// iteration's passes): every status change of iteration j (krylov_conclude), and a timeout
// a streaming kernel recorded.
__global__ void __launch_bounds__(32)
k_lz_decide(KState *ks, int j, double dt, double exp_tol, int poll, int first_poll, int maxdim) {
    if (ks->status != KS_RUNNING) return;
    if (ks->kerr) {  // a streaming kernel gave up on a bounded wait
        if (threadIdx.x == 0) {
            ks->status = KS_TIMEOUT;
            ks->iters = j + 1;
        }
        return;
    }
    krylov_conclude(ks, j, ks->lz_flag[j], dt, exp_tol, poll != 0, first_poll != 0, maxdim);
}

// The decision stream of the H-first iteration, one per device (created on first use).
// Used for vectors of at most 32 MB, where the decision (about 20 us) is a large share of
// an iteration (N=20 complex128: 1.99 -> 1.79 ms per 23-iteration step).  On larger
// registers every SM's register file is full of a streaming kernel's CTAs, so the
// decision warp only delays one of them and lengthens that kernel by about as much as it
// saves (N=26 complex64: 0.891 -> 0.914 ms per iteration): there it stays on the step's
// stream.
static bool decision_overlaps(int dtype, int n) {
    const double bytes = (double)(1ll << n) * (dtype == EMUSV_C128 ? 16.0 : 8.0);
    return bytes <= 32.0 * 1024 * 1024;
}
static cudaStream_t decision_stream() {
    static std::mutex mu;
    static cudaStream_t streams[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess)
        streams[dev] = nullptr;
    return streams[dev];
}

// out = s0 * sum_k c_k scale_k stored_k ;  ||out||^2 partials.
template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_combine(const KState *ks, const void *v0_, const unsigned char *basis, i64 D, void *out_,
          double *partials) {
    typedef typename cvec<R>::T C;
    __shared__ double cr[KMAX + 2], ci[KMAX + 2];
    __shared__ double red[(BLOCK / 32) * NRED];
    const int nv = ks->nvec;
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
        const double f = ks->s0 * ks->scale[k];
        cr[k] = f * ks->c_re[k];
        ci[k] = f * ks->c_im[k];
    }
    __syncthreads();
    const C *v0 = reinterpret_cast<const C *>(v0_);  // may equal out (in place, per element)
    const C *__restrict__ bs = reinterpret_cast<const C *>(basis);
    C *out = reinterpret_cast<C *>(out_);
    double acc[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) acc[k] = 0.0;
    // XA amplitudes per thread (grid-strided, so every load instruction is coalesced) and
    // KU basis vectors per step: XA * KU independent loads in flight per thread
    constexpr int XA = 4, KU = 4;
    const i64 G = (i64)gridDim.x * blockDim.x;
    for (i64 x0 = (i64)blockIdx.x * blockDim.x + threadIdx.x; x0 < D; x0 += XA * G) {
        double re[XA], im[XA];
#pragma unroll
        for (int a = 0; a < XA; ++a) {
            const i64 x = x0 + a * G;
            re[a] = im[a] = 0.0;
            if (x < D) {
                const C v = __ldcs(v0 + x);
                re[a] = cr[0] * double(v.x) - ci[0] * double(v.y);
                im[a] = cr[0] * double(v.y) + ci[0] * double(v.x);
            }
        }
        int k = 1;
        for (; k + KU <= nv; k += KU) {
            C b[KU][XA];
#pragma unroll
            for (int u = 0; u < KU; ++u)
#pragma unroll
                for (int a = 0; a < XA; ++a) {
                    const i64 x = x0 + a * G;
                    b[u][a] = x < D ? __ldcs(bs + (i64)(k + u) * D + x) : cmake<C>(0.0, 0.0);
                }
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                const double r_ = cr[k + u], i_ = ci[k + u];
#pragma unroll
                for (int a = 0; a < XA; ++a) {
                    re[a] += r_ * double(b[u][a].x) - i_ * double(b[u][a].y);
                    im[a] += r_ * double(b[u][a].y) + i_ * double(b[u][a].x);
                }
            }
        }
        for (; k < nv; ++k) {
            const double r_ = cr[k], i_ = ci[k];
#pragma unroll
            for (int a = 0; a < XA; ++a) {
                const i64 x = x0 + a * G;
                if (x < D) {
                    const C b = __ldcs(bs + (i64)k * D + x);
                    re[a] += r_ * double(b.x) - i_ * double(b.y);
                    im[a] += r_ * double(b.y) + i_ * double(b.x);
                }
            }
        }
#pragma unroll
        for (int a = 0; a < XA; ++a) {
            const i64 x = x0 + a * G;
            if (x < D) {
                const C o = cmake<C>(re[a], im[a]);
                out[x] = o;
                acc[0] += double(o.x) * double(o.x) + double(o.y) * double(o.y);
            }
        }
    }
    block_sum<NRED>(acc, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < NRED; ++k) partials[(i64)blockIdx.x * NRED + k] = acc[k];
}

__global__ void k_finish_combine(KState *ks, const double *partials, int nblocks) {
    __shared__ double red[(BLOCK / 32) * NRED];
    double v[NRED];
    sum_partials<NRED>(partials, nblocks, NRED, v, red);
    if (threadIdx.x == 0) ks->outnorm2 = v[0];
}

// ---------------------------------------------------------------- generic helpers
template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_dot(const void *a_, const void *b_, i64 len, double *partials) {
    typedef typename cvec<R>::T C;
    const C *a = reinterpret_cast<const C *>(a_);
    const C *b = reinterpret_cast<const C *>(b_);
    __shared__ double red[(BLOCK / 32) * NRED];
    double acc[NRED];
#pragma unroll
    for (int k = 0; k < NRED; ++k) acc[k] = 0.0;
    for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < len; x += (i64)gridDim.x * blockDim.x) {
        const C p = a[x], q = b[x];
        acc[0] += double(p.x) * double(q.x) + double(p.y) * double(q.y);
        acc[1] += double(p.x) * double(q.y) - double(p.y) * double(q.x);
    }
    block_sum<NRED>(acc, red);
    if (threadIdx.x == 0)
        for (int k = 0; k < NRED; ++k) partials[(i64)blockIdx.x * NRED + k] = acc[k];
}

__global__ void k_sum2(const double *partials, int nblocks, double *out) {
    __shared__ double red[(BLOCK / 32) * NRED];
    double v[NRED];
    sum_partials<NRED>(partials, nblocks, NRED, v, red);
    if (threadIdx.x == 0) {
        out[0] = v[0];
        out[1] = v[1];
    }
}

template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_axpy(double ar, double ai, const void *x_, void *y_, i64 len) {
    typedef typename cvec<R>::T C;
    const C *x = reinterpret_cast<const C *>(x_);
    C *y = reinterpret_cast<C *>(y_);
    for (i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x; k < len; k += (i64)gridDim.x * blockDim.x) {
        const C a = x[k];
        C b = y[k];
        const double re = double(b.x) + ar * double(a.x) - ai * double(a.y);
        const double im = double(b.y) + ar * double(a.y) + ai * double(a.x);
        y[k] = cmake<C>(re, im);
    }
}

template <typename R>
__global__ void __launch_bounds__(BLOCK)
k_vcombine(int nk, const double2 *coef, const void *V_, i64 len, void *out_) {
    typedef typename cvec<R>::T C;
    const C *V = reinterpret_cast<const C *>(V_);
    C *out = reinterpret_cast<C *>(out_);
    for (i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x; x < len; x += (i64)gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int k = 0; k < nk; ++k) {
            const C b = V[(i64)k * len + x];
            const double2 c = coef[k];
            re += c.x * double(b.x) - c.y * double(b.y);
            im += c.x * double(b.y) + c.y * double(b.x);
        }
        out[x] = cmake<C>(re, im);
    }
}

struct TriArgs {
    double2 d[KMAX + 2], up[KMAX + 2], lo[KMAX + 2];
};

__global__ void __launch_bounds__(32) k_tridiag_expm(int m, const TriArgs *A, double2 *xout) {
    __shared__ double2 y[KMAX + 4], t[KMAX + 4], tn[KMAX + 4], acc[KMAX + 4];
    double2 Z1, Z2;
    warp_expm_col(m, A->d, A->up, A->lo, y, t, tn, acc, &Z1, &Z2);
    for (int k = threadIdx.x; k < m; k += 32) xout[k] = y[k + 1];
}

}  // namespace emusv

using namespace emusv;

namespace emusv {
namespace {
thread_local int *pinned_status = nullptr;
}  // namespace

// Input norm and KState reset, as the start of lanczos_run (k_init).
int krylov_begin(int dtype, const void *psi_in, i64 D, KState *ks, double *partials, bool energy_shift,
                 cudaStream_t s) {
    const int sg = stream_grid(D);
    {
        ProfScope ps_(PROF_ORTH, s);
        if (dtype == EMUSV_C128) k_norm2<double><<<sg, BLOCK, 0, s>>>(psi_in, D, partials);
        else k_norm2<float><<<sg, BLOCK, 0, s>>>(psi_in, D, partials);
    }
    EMUSV_CHECK_LAUNCH();
    {
        ProfScope ps_(PROF_SMALL, s);
        k_init<<<1, BLOCK, 0, s>>>(ks, partials, sg, energy_shift ? 1 : 0);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

// out = s0 * sum_k c_k scale_k stored_k over ks->nvec vectors, and ks->outnorm2.
int krylov_combine(int dtype, KState *ks, const void *psi_in, const unsigned char *basis, i64 D,
                   void *out, double *partials, cudaStream_t s) {
    const int sg = stream_grid(D);
    {
        ProfScope ps_(PROF_COMBINE, s);
        if (dtype == EMUSV_C128) k_combine<double><<<sg, BLOCK, 0, s>>>(ks, psi_in, basis, D, out, partials);
        else k_combine<float><<<sg, BLOCK, 0, s>>>(ks, psi_in, basis, D, out, partials);
    }
    EMUSV_CHECK_LAUNCH();
    {
        ProfScope ps_(PROF_SMALL, s);
        k_finish_combine<<<1, BLOCK, 0, s>>>(ks, partials, sg);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

int krylov_stream_grid(i64 D) { return stream_grid(D); }
size_t krylov_header_bytes() { return header_bytes(); }

int read_status(KState *ks, cudaStream_t s, int *out) {
    if (!pinned_status) {
        if (cudaHostAlloc((void **)&pinned_status, 4 * sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
            pinned_status = nullptr;
            return EMUSV_CUDA_ERROR;
        }
    }
    EMUSV_CHECK(cudaMemcpyAsync(pinned_status, &ks->status, sizeof(int), cudaMemcpyDeviceToHost, s));
    EMUSV_CHECK(cudaStreamSynchronize(s));
    *out = pinned_status[0];
    return EMUSV_OK;
}
}  // namespace emusv

namespace emusv {

int lanczos_run(const HamParams &P, int dtype, double dt, const void *v0, KState *ks,
                double *part_h, double *part_o, unsigned char *basis, int capacity,
                double exp_tol, double norm_tol, int maxdim, int hint, bool energy_shift,
                cudaStream_t s, int *status_out) {
    const int nqubits = P.n;
    const i64 D = i64(1) << nqubits;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    void *part_vec = basis;
    auto stored = [&](int k) -> const void * {
        return k == 0 ? v0 : (const void *)(basis + (size_t)k * D * es);
    };
    const int sg = stream_grid(D);
    const double exp_tolerance = exp_tol, norm_tolerance = norm_tol;
    const int max_krylov_dim = maxdim, krylov_dim_hint = hint;
    const void *psi_in = v0;
    struct { KState *ks; double *part_h, *part_o; } W = {ks, part_h, part_o};

    if (dtype == EMUSV_C128)
        {
            ProfScope ps_(PROF_ORTH, s);
            k_norm2<double><<<sg, BLOCK, 0, s>>>(psi_in, D, W.part_h);
        }
    else
        {
            ProfScope ps_(PROF_ORTH, s);
            k_norm2<float><<<sg, BLOCK, 0, s>>>(psi_in, D, W.part_h);
        }
    EMUSV_CHECK_LAUNCH();
    {
        ProfScope ps_(PROF_SMALL, s);
        k_init<<<1, BLOCK, 0, s>>>(W.ks, W.part_h, sg, energy_shift ? 1 : 0);
    }
    EMUSV_CHECK_LAUNCH();

    int status = KS_RUNNING;
    // Registers wider than one pass-L tile run the H-first iteration: the pass H kernels
    // write part = X_high v_j (the flips of the bits above the pass-L tile) and their share
    // of <v_j, H v_j>; k_lz_coef forms a_j; the pass L kernel forms H v_j tile by tile and
    // writes w = H v_j - a_j v_j - b_j v_{j-1} and the pass-L share of <w, H w> for the
    // next a; k_lz_norms and k_lz_decide conclude the iteration.  Streamed vector units per iteration: pass L 4 (read v_j,
    // part, v_{j-1}; write w), one H pass 2 (read v_j, write part) or two H passes 2 + 3.
    const bool hfirst = lanczos_h_first(dtype, nqubits);
    if (hfirst) {
        // with `overlap`, the decision of iteration j (k_lz_decide) runs on a second stream
        // while the main stream goes on with iteration j+1, which needs only k_lz_norms'
        // outputs (k_lz_decide reads a, r, b up to index j and hn[j]; iteration j+1 writes
        // index j+1 and above); kernels launched after the device decided return at once,
        // and the host reads the status only after the decision stream's event
        const bool overlap = decision_overlaps(dtype, nqubits);
        cudaStream_t sd = overlap ? decision_stream() : s;
        cudaEvent_t ev_n = nullptr, ev_d = nullptr;
        if ((overlap && !sd) || cudaEventCreateWithFlags(&ev_n, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_d, cudaEventDisableTiming) != cudaSuccess) {
            if (ev_n) cudaEventDestroy(ev_n);
            return EMUSV_CUDA_ERROR;
        }
        struct Events {
            cudaEvent_t a, b;
            ~Events() {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } evs{ev_n, ev_d};
        // status after every decision taken so far (main stream joins the decision stream)
        auto status_now = [&](int *out) -> int {
            if (overlap) {
                EMUSV_CHECK(cudaEventRecord(ev_d, sd));
                EMUSV_CHECK(cudaStreamWaitEvent(s, ev_d, 0));
            }
            return read_status(W.ks, s, out);
        };
        LzArgs E = {};
        E.u = stored(0);
        E.eshift = &W.ks->shift;
        E.partials = W.part_o;
        E.gate = &W.ks->status;
        E.err = &W.ks->kerr;
        int ge0 = 0;
        int st = lz_energy0(dtype, P, E, s, &ge0);
        if (st) return st;
        bool joined = false;
        for (int j = 0; j < max_krylov_dim; ++j) {
            if (j + 1 > capacity) {
                st = status_now(&status);
                joined = true;
                if (st) return st;
                if (status == KS_RUNNING) return EMUSV_WORKSPACE_TOO_SMALL;
                break;
            }
            int gh = 0, go = 0;
            if ((st = lz_high(dtype, P, stored(j), part_vec, W.part_h, &W.ks->status, &W.ks->kerr,
                              W.ks->hh_cnt, s, &gh)))
                return st;
            {
                ProfScope ps_(PROF_SMALL, s);
                k_lz_coef<<<1, BLOCK, 0, s>>>(W.ks, j, W.part_h, gh, W.part_o, ge0);
            }
            EMUSV_CHECK_LAUNCH();
            LzArgs B = {};
            B.u = stored(j);
            B.part = part_vec;
            B.up = j > 0 ? stored(j - 1) : nullptr;
            B.out = const_cast<void *>(stored(j + 1));
            B.su = &W.ks->scale[j];
            B.ocoef = W.ks->ocoef;
            B.eshift = &W.ks->shift;
            B.partials = W.part_o;
            B.gate = &W.ks->status;
            B.err = &W.ks->kerr;
            if ((st = lz_low(dtype, P, B, s, &go))) return st;
            {
                ProfScope ps_(PROF_SMALL, s);
                k_lz_norms<<<1, BLOCK, 0, s>>>(W.ks, j, W.part_o, go, dt, norm_tolerance);
            }
            EMUSV_CHECK_LAUNCH();
            if (overlap) {
                EMUSV_CHECK(cudaEventRecord(ev_n, s));
                EMUSV_CHECK(cudaStreamWaitEvent(sd, ev_n, 0));
            }
            {
                ProfScope ps_(PROF_SMALL, sd);
                k_lz_decide<<<1, 32, 0, sd>>>(W.ks, j, dt, exp_tolerance, 1, j == 0, max_krylov_dim);
            }
            EMUSV_CHECK_LAUNCH();
            const int poll = (j + 1 >= krylov_dim_hint) || (j + 1 >= max_krylov_dim);
            if (poll) {
                st = status_now(&status);
                joined = true;
                if (st) return st;
                if (status != KS_RUNNING) break;
            } else {
                joined = false;
            }
        }
        if (overlap && !joined) {  // the step's later work (the combination) follows every decision
            EMUSV_CHECK(cudaEventRecord(ev_d, sd));
            EMUSV_CHECK(cudaStreamWaitEvent(s, ev_d, 0));
        }
    }
    for (int j = 0; !hfirst && j < max_krylov_dim; ++j) {
        if (j + 1 > capacity) {
            int st = read_status(W.ks, s, &status);
            if (st) return st;
            if (status == KS_RUNNING) return EMUSV_WORKSPACE_TOO_SMALL;
            break;
        }
        HpsiArgs A = {};
        A.u = stored(j);
        A.su_dev = &W.ks->scale[j];
        A.up = nullptr;  // b comes from the previous norm (see k_orth)
        A.out = const_cast<void *>(stored(j + 1));
        A.partials = W.part_h;
        A.tile_bits = hpsi_tile_bits(nqubits);
        A.gate = &W.ks->status;
        A.err = &W.ks->kerr;
        A.part_buf = part_vec;
        A.eshift = &W.ks->shift;
        int gh = 0;
        int st = launch_hpsi(dtype, HP_LANCZOS, P, A, max_grid_blocks(), s, &gh);
        if (st) return st;
        if (dtype == EMUSV_C128)
            {
                ProfScope ps_(PROF_ORTH, s);
                k_orth<double><<<sg, BLOCK, 0, s>>>(W.ks, j, W.part_h, gh, stored(j),
                                                    j > 0 ? stored(j - 1) : nullptr,
                                                    const_cast<void *>(stored(j + 1)), D, W.part_o);
            }
        else
            {
                ProfScope ps_(PROF_ORTH, s);
                k_orth<float><<<sg, BLOCK, 0, s>>>(W.ks, j, W.part_h, gh, stored(j),
                                                   j > 0 ? stored(j - 1) : nullptr,
                                                   const_cast<void *>(stored(j + 1)), D, W.part_o);
            }
        EMUSV_CHECK_LAUNCH();
        // the device tests convergence at every iteration, as the reference does; the host
        // reads the status (one synchronisation) from the hint on, and kernels launched
        // after the device converged return at once
        const int poll = (j + 1 >= krylov_dim_hint) || (j + 1 >= max_krylov_dim);
        {
            ProfScope ps_(PROF_SMALL, s);
            k_small<<<1, 32, 0, s>>>(W.ks, j, W.part_o, sg, dt, exp_tolerance, norm_tolerance, 1,
                                     j == 0, max_krylov_dim);
        }
        EMUSV_CHECK_LAUNCH();
        if (poll) {
            st = read_status(W.ks, s, &status);
            if (st) return st;
            if (status != KS_RUNNING) break;
        }
    }
    if (status == KS_RUNNING) {
        int st = read_status(W.ks, s, &status);
        if (st) return st;
    }
    *status_out = status;
    return EMUSV_OK;
}

}  // namespace emusv

extern "C" {

size_t emusv_krylov_workspace_bytes(int nqubits, int dtype, int basis_capacity) {
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS || basis_capacity < 0) return 0;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    return header_bytes() + (size_t)(basis_capacity + 1) * (size_t(1) << nqubits) * es;
}

int emusv_krylov_step(int nqubits, int dtype, double dt, const double *omegas,
                      const double *deltas, const double *phis, const double *interaction,
                      const void *psi_in, void *psi_out, double exp_tolerance,
                      double norm_tolerance, int max_krylov_dim, int krylov_dim_hint,
                      void *workspace, size_t workspace_bytes, emusv_krylov_info *info,
                      void *stream) {
    HamParams P;
    if (!psi_in || !psi_out || !workspace || (dtype != EMUSV_C128 && dtype != EMUSV_C64) ||
        max_krylov_dim < 1 || max_krylov_dim > KMAX - 2 || !isfinite(dt) ||
        !make_params(nqubits, omegas, deltas, phis, interaction, &P))
        return EMUSV_BAD_ARGUMENT;
    if (workspace_bytes < header_bytes()) return EMUSV_WORKSPACE_TOO_SMALL;
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) || (reinterpret_cast<uintptr_t>(psi_in) & 15) ||
        (reinterpret_cast<uintptr_t>(psi_out) & 15))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const i64 D = i64(1) << nqubits;
    const size_t es = dtype == EMUSV_C128 ? 16 : 8;
    Workspace W = carve(workspace, workspace_bytes);
    // basis region: [partial-sum vector of the two-pass H*psi][stored_1][stored_2]...
    const int capacity = (int)(W.basis_bytes / (D * es)) - 1;
    if (capacity < 1) return EMUSV_WORKSPACE_TOO_SMALL;
    const int sg = stream_grid(D);

    int status = KS_RUNNING;
    {
        const int st = lanczos_run(P, dtype, dt, psi_in, W.ks, W.part_h, W.part_o, W.basis, capacity,
                                   exp_tolerance, norm_tolerance, max_krylov_dim, krylov_dim_hint,
                                   true, s, &status);
        if (st) return st;
    }
    if (status == KS_TIMEOUT) {
        if (info) memset(info, 0, sizeof(*info));
        return EMUSV_TIMEOUT;
    }
    if (status == KS_NONFINITE || status == KS_RUNNING) {
        if (info) memset(info, 0, sizeof(*info));
        return EMUSV_NONFINITE;
    }
    if (dtype == EMUSV_C128)
        {
            ProfScope ps_(PROF_COMBINE, s);
            k_combine<double><<<sg, BLOCK, 0, s>>>(W.ks, psi_in, W.basis, D, psi_out, W.part_c);
        }
    else
        {
            ProfScope ps_(PROF_COMBINE, s);
            k_combine<float><<<sg, BLOCK, 0, s>>>(W.ks, psi_in, W.basis, D, psi_out, W.part_c);
        }
    EMUSV_CHECK_LAUNCH();
    {
        ProfScope ps_(PROF_SMALL, s);
        k_finish_combine<<<1, BLOCK, 0, s>>>(W.ks, W.part_c, sg);
    }
    EMUSV_CHECK_LAUNCH();
    if (info) {
        KState h;
        EMUSV_CHECK(cudaMemcpyAsync(&h, W.ks, offsetof(KState, a_re), cudaMemcpyDeviceToHost, s));
        EMUSV_CHECK(cudaStreamSynchronize(s));
        info->iterations = h.iters;
        info->happy_breakdown = h.status == KS_HAPPY;
        info->converged = h.status == KS_HAPPY || h.status == KS_CONVERGED;
        info->basis_vectors = h.nvec;
        info->error_estimate = h.err;
        info->input_norm = h.s0;
        info->output_norm = sqrt(h.outnorm2);
        info->second_rounds = 0;
    }
    return status == KS_MAXDIM ? EMUSV_NOT_CONVERGED : EMUSV_OK;
}

int emusv_vec_dot(int64_t len, int dtype, const void *a, const void *b, double *res_dev,
                  void *scratch, size_t scratch_bytes, void *stream) {
    if (len < 1 || !a || !b || !res_dev || !scratch ||
        scratch_bytes < sizeof(double) * (size_t)max_grid_blocks() * NRED)
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    double *partials = reinterpret_cast<double *>(scratch);
    const int g = stream_grid(len);
    if (dtype == EMUSV_C128)
        {
            ProfScope ps_(PROF_ORTH, s);
            k_dot<double><<<g, BLOCK, 0, s>>>(a, b, len, partials);
        }
    else if (dtype == EMUSV_C64)
        {
            ProfScope ps_(PROF_ORTH, s);
            k_dot<float><<<g, BLOCK, 0, s>>>(a, b, len, partials);
        }
    else
        return EMUSV_BAD_ARGUMENT;
    EMUSV_CHECK_LAUNCH();
    {
        ProfScope ps_(PROF_SMALL, s);
        k_sum2<<<1, BLOCK, 0, s>>>(partials, g, res_dev);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

int emusv_vec_axpy(int64_t len, int dtype, const double *alpha, const void *x, void *y,
                   void *stream) {
    if (len < 1 || !alpha || !x || !y) return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const int g = stream_grid(len);
    if (dtype == EMUSV_C128)
        {
            ProfScope ps_(PROF_ORTH, s);
            k_axpy<double><<<g, BLOCK, 0, s>>>(alpha[0], alpha[1], x, y, len);
        }
    else if (dtype == EMUSV_C64)
        {
            ProfScope ps_(PROF_ORTH, s);
            k_axpy<float><<<g, BLOCK, 0, s>>>(alpha[0], alpha[1], x, y, len);
        }
    else
        return EMUSV_BAD_ARGUMENT;
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

int emusv_vec_combine(int64_t len, int dtype, int k, const double *coef_dev, const void *V,
                      void *out, void *stream) {
    if (len < 1 || k < 1 || !coef_dev || !V || !out) return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    const int g = stream_grid(len);
    const double2 *c = reinterpret_cast<const double2 *>(coef_dev);
    if (dtype == EMUSV_C128)
        {
            ProfScope ps_(PROF_COMBINE, s);
            k_vcombine<double><<<g, BLOCK, 0, s>>>(k, c, V, len, out);
        }
    else if (dtype == EMUSV_C64)
        {
            ProfScope ps_(PROF_COMBINE, s);
            k_vcombine<float><<<g, BLOCK, 0, s>>>(k, c, V, len, out);
        }
    else
        return EMUSV_BAD_ARGUMENT;
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}

size_t emusv_tridiag_scratch_bytes(void) { return align_up(sizeof(TriArgs), 256); }

int emusv_tridiag_expm_col(int m, const double *diag, const double *upper, const double *lower,
                           double *x_dev, void *scratch, size_t scratch_bytes, void *stream) {
    if (m < 1 || m > KMAX || !diag || !upper || !lower || !x_dev || !scratch ||
        scratch_bytes < sizeof(TriArgs))
        return EMUSV_BAD_ARGUMENT;
    cudaStream_t s = as_stream(stream);
    TriArgs *A = reinterpret_cast<TriArgs *>(scratch);
    EMUSV_CHECK(cudaMemcpyAsync(A->d, diag, sizeof(double2) * m, cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(A->up, upper, sizeof(double2) * m, cudaMemcpyHostToDevice, s));
    EMUSV_CHECK(cudaMemcpyAsync(A->lo, lower, sizeof(double2) * m, cudaMemcpyHostToDevice, s));
    {
        ProfScope ps_(PROF_SMALL, s);
        k_tridiag_expm<<<1, 32, 0, s>>>(m, A, reinterpret_cast<double2 *>(x_dev));
    }
    EMUSV_CHECK_LAUNCH();
    // host arrays may be reused by the caller once this returns
    EMUSV_CHECK(cudaStreamSynchronize(s));
    return EMUSV_OK;
}

}  // extern "C"
