// Host side of the two-pass H*psi: layout choice, parameter tables, cluster launches.
#include <cudaTypedefs.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>

#include "hpsi_kernel.cuh"
#include "hpsi_pass.cuh"
#include "profile.cuh"

namespace emusv {

// Tile shapes: 2^TB amplitudes per CTA (64 KiB of shared memory either way), 2^RB of them
// in each thread's registers, 256 threads.
template <typename R> struct PassShape;
// c64: 4096-amplitude tiles (32 KiB), 16 amplitudes per thread; c128: 2048-amplitude
// tiles (32 KiB), 8 per thread; 256 threads.  CMIN: chunk bits of the pass H rows, 64
// bytes (measured on B200, 32-byte rows made the N=26 complex64 Krylov step 9 % slower);
// complex128 registers whose high bits do not fit two 64-byte-row passes (n > 29) use
// 32-byte rows (CMIN - 1).
// No thread-block clusters: measured on B200, reading partner amplitudes from a sibling
// CTA's shared memory amplitude by amplitude (and the per-tile cluster barrier) cost more
// than a further streaming pass, so every pass keeps its flips inside one CTA's tile.
template <> struct PassShape<float> {
    static constexpr int TB = 12, RB = 4, CMIN = 3;
};
template <> struct PassShape<double> {
    static constexpr int TB = 11, RB = 3, CMIN = 2;
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map of a 2^n vector of `es`-byte amplitudes for pass H (see hpsi_pass.cuh).
static bool encode_pass_high(CUtensorMap *map, const void *base, int n, int es, const PassParams &P) {
    auto fn = encode_fn();
    if (!fn) return false;
    const int K = es / 8;
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
    const int c = P.hc, g = P.hg, hpos = P.hpos, pbh = P.pbh;
    dims[0] = (cuuint64_t(1) << c) * K;
    dims[1] = cuuint64_t(1) << (hpos - c);
    dims[2] = cuuint64_t(1) << g;
    dims[3] = cuuint64_t(1) << pbh;
    dims[4] = cuuint64_t(1) << (n - hpos - g - pbh);
    strides[0] = (cuuint64_t(es) << c);
    strides[1] = (cuuint64_t(es) << hpos);
    strides[2] = (cuuint64_t(es) << (hpos + g));
    strides[3] = (cuuint64_t(es) << (hpos + g + pbh));
    box[0] = (cuuint32_t)dims[0];
    box[1] = 1;
    box[2] = (cuuint32_t)P.hbox_rows;
    box[3] = 1;
    box[4] = 1;
    const cuuint64_t chunk_bytes = (cuuint64_t(es) << c);
    const CUtensorMapL2promotion promo =
        chunk_bytes >= 256 ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
                           : (chunk_bytes >= 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B
                                                 : CU_TENSOR_MAP_L2_PROMOTION_NONE);
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void *>(base), dims,
                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

int pass_min_qubits(int dtype) {
    return dtype == EMUSV_C64 ? PassShape<float>::TB : PassShape<double>::TB;
}

static void fill_params(const HamParams &H, int TB, int RB, PassParams *P) {
    memset(P, 0, sizeof(*P));
    P->n = H.n;
    P->real_coef = H.real_coef;
    for (int p = 0; p < MAXQ; ++p) {
        P->dup_re[p] = H.up_re[p];
        P->dup_im[p] = H.up_im[p];
        P->ddn_re[p] = H.dn_re[p];
        P->ddn_im[p] = H.dn_im[p];
        P->fup_re[p] = (float)H.up_re[p];
        P->fup_im[p] = (float)H.up_im[p];
        P->fdn_re[p] = (float)H.dn_re[p];
        P->fdn_im[p] = (float)H.dn_im[p];
        P->field[p] = H.field[p];
    }
    memcpy(P->U, H.U, sizeof(P->U));
    P->dc_re = H.dc_re;
    P->dc_im = H.dc_im;
    P->dg_im = H.dg_im;
    const int SB = TB - RB;
    for (int a = 0; a < (1 << RB); ++a) {  // fields and pairs of the register bits
        double e = 0.0;
        for (int k = 0; k < RB; ++k) {
            if (!((a >> k) & 1)) continue;
            e += H.field[SB + k];
            for (int k2 = k + 1; k2 < RB; ++k2)
                if ((a >> k2) & 1) e += H.U[(SB + k) * MAXQ + SB + k2];
        }
        P->ER[a] = e;
        P->ERf[a] = (float)e;
    }
}

template <typename R, bool REALC, int EPI, bool NOISY>
static int launch_low(const PassParams &P, const PassArgs &A, cudaStream_t s, int *grid_out) {
    typedef typename cvec<R>::T C;
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, NT = 1 << (TB - RB);
    auto kern = k_pass_low<R, REALC, TB, RB, EPI, 0, NOISY>;
    const size_t smem = pass_low_smem<C, TB>();
    EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    const int64_t ntiles = int64_t(1) << (P.n - TB);
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > ntiles) grid = ntiles;
    {
        ProfScope ps_(PROF_HPSI, s);
        kern<<<(unsigned)grid, NT, smem, s>>>(P, A);
    }
    EMUSV_CHECK_LAUNCH();
    if (grid_out) *grid_out = (int)grid;
    return EMUSV_OK;
}

// One strided pass over the group bits [hpos, hpos + TB - CMIN) with CMIN chunk bits;
// group bits below hskip (the pass-L tile width) were applied by pass L and are skipped.
template <typename R, bool REALC, int EPI, int CMIN, bool CHUNKF = false>
static int launch_high(PassParams P, int hpos, const PassArgs &A, const void *part,
                       cudaStream_t s, int *grid_out, int hskip = PassShape<R>::TB) {
    typedef typename cvec<R>::T C;
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, NT = 1 << (TB - RB);
    constexpr bool HASPART = epi_has_part<EPI>();
    const int n = P.n, g = TB - CMIN;
    if (hpos < CMIN || hpos + g > n) return EMUSV_BAD_ARGUMENT;
    P.hg = g;
    P.hc = CMIN;
    P.hpos = hpos;
    P.pbh = 0;
    P.hskip = hskip;
    P.hbox_rows = g > 8 ? 256 : (1 << g);
    PassHighMaps M;
    memset(&M, 0, sizeof(M));
    if (!encode_pass_high(&M.u, A.u, n, (int)sizeof(C), P) ||
        (HASPART && !encode_pass_high(&M.part, part, n, (int)sizeof(C), P)))
        return EMUSV_CUDA_ERROR;
    auto kern = k_pass_high<R, REALC, TB, RB, EPI, CMIN, 0, CHUNKF>;
    const size_t smem = pass_high_smem<C, TB, HASPART>();
    EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    const int64_t ntiles = int64_t(1) << (n - TB);
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > ntiles) grid = ntiles;
    {
        ProfScope ps_(PROF_HPSI_HIGH, s);
        kern<<<(unsigned)grid, NT, smem, s>>>(P, A, M);
    }
    EMUSV_CHECK_LAUNCH();
    if (grid_out) *grid_out = (int)grid;
    return EMUSV_OK;
}

// H v in two or three streaming passes: L (bits 0..TB-1, diagonal), then strided passes
// over groups of G = TB - CMIN bits: the final one over the top G bits [n - G, n), and,
// when n - TB > G, one before it over [n - 2G, n - G).  Group bits below TB (covered by
// pass L) are skipped, so every H pass keeps the compile-time chunk of CMIN bits.  The
// partial sums live in HA.part_buf (which may be HA.out: every pass reads a tile before
// writing it).
template <typename R, bool REALC, int EPI_F, int CMIN, bool NOISY>
static int run_passes(const HamParams &H, const HpsiArgs &HA, cudaStream_t s, int *grid_out) {
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB;
    const int n = H.n;
    PassParams P;
    fill_params(H, TB, RB, &P);
    P.pb = 0;
    const int rem = n - TB, G = TB - CMIN;
    if (rem > 2 * G) return EMUSV_BAD_ARGUMENT;  // more than three passes: n too large
    if (rem > 0 && !HA.part_buf) return EMUSV_BAD_ARGUMENT;

    PassArgs A = {};
    A.u = HA.u;
    A.su_dev = HA.su_dev;
    A.su = HA.su;
    A.partials = HA.partials;
    A.gate = HA.gate;
    A.err = HA.err;
    A.eshift = HA.eshift;  // null unless the caller shifts the diagonal
    int st;
    if (rem == 0) {
        A.out = HA.out;
        return launch_low<R, REALC, EPI_F, NOISY>(P, A, s, grid_out);
    }
    A.out = HA.part_buf;
    if ((st = launch_low<R, REALC, EPI_PARTIAL, NOISY>(P, A, s, nullptr))) return st;
    if (rem > G) {
        if ((st = launch_high<R, REALC, EPI_PARTIAL, CMIN>(P, n - 2 * G, A, HA.part_buf, s, nullptr)))
            return st;
    }
    A.out = HA.out;
    return launch_high<R, REALC, EPI_F, CMIN>(P, n - G, A, HA.part_buf, s, grid_out);
}

// 64-byte rows (PassShape CMIN) where two H passes cover the bits above pass L, else
// 32-byte rows
template <typename R, bool REALC, int EPI_F, bool NOISY = false>
static int run_passes(const HamParams &H, const HpsiArgs &HA, cudaStream_t s, int *grid_out) {
    constexpr int TB = PassShape<R>::TB, CMIN = PassShape<R>::CMIN;
    if (H.n - TB <= 2 * (TB - CMIN)) return run_passes<R, REALC, EPI_F, CMIN, NOISY>(H, HA, s, grid_out);
    return run_passes<R, REALC, EPI_F, CMIN - 1, NOISY>(H, HA, s, grid_out);
}

// mode: HP_STORE or HP_LANCZOS (values of HpsiMode)
int launch_hpsi_passes(int dtype, int mode, const HamParams &H, const HpsiArgs &A,
                       cudaStream_t s, int *grid_out) {
    const bool lz = mode == HP_LANCZOS;
    if (H.noisy) {  // the non-Hermitian noise term: store mode only (Arnoldi, H*psi)
        if (lz) return EMUSV_BAD_ARGUMENT;
        return dtype == EMUSV_C64 ? run_passes<float, false, EPI_STORE, true>(H, A, s, grid_out)
                                  : run_passes<double, false, EPI_STORE, true>(H, A, s, grid_out);
    }
    if (dtype == EMUSV_C64) {
        if (H.real_coef)
            return lz ? run_passes<float, true, EPI_LANCZOS>(H, A, s, grid_out)
                      : run_passes<float, true, EPI_STORE>(H, A, s, grid_out);
        return lz ? run_passes<float, false, EPI_LANCZOS>(H, A, s, grid_out)
                  : run_passes<float, false, EPI_STORE>(H, A, s, grid_out);
    }
    if (dtype == EMUSV_C128) {
        if (H.real_coef)
            return lz ? run_passes<double, true, EPI_LANCZOS>(H, A, s, grid_out)
                      : run_passes<double, true, EPI_STORE>(H, A, s, grid_out);
        return lz ? run_passes<double, false, EPI_LANCZOS>(H, A, s, grid_out)
                  : run_passes<double, false, EPI_STORE>(H, A, s, grid_out);
    }
    return EMUSV_BAD_ARGUMENT;
}


// ------------------------------------------------------ Lanczos iteration, H-first order
// Pass L of the Lanczos iteration (k_pass_lz): 2^11-amplitude tiles; complex64 8
// amplitudes per thread (256 threads, two CTAs per SM), complex128 4 per thread (512
// threads, one CTA per SM).
template <typename R> struct LzShape;
template <> struct LzShape<float> {
    static constexpr int TB = 11, RB = 3;
};
template <> struct LzShape<double> {
    static constexpr int TB = 11, RB = 2;
};

// The chunk bits of the pass H rows of this register (the bits the recurrence pass L
// leaves out): 64-byte rows where two H passes cover the bits above pass L, else 32-byte.
template <typename R> static int lz_chunk_bits(int n) {
    constexpr int TB = PassShape<R>::TB, CMIN = PassShape<R>::CMIN, TBL = LzShape<R>::TB;
    return n - TBL <= 2 * (TB - CMIN) ? CMIN : CMIN - 1;
}
// The two pass H groups of the Lanczos iteration run as two launches unless
// EMUSV_FUSED_PASS_H=1 selects the fused persistent kernel (k_pass_hh).  Measured on B200 at
// N=26 complex64: the fused kernel moves about 2 vector units of DRAM traffic instead of 5
// and leaves the sums in the L2 for the recurrence pass L (0.383 against 0.409 ms), but
// takes 0.556 ms against 0.509 ms for the two launches (its tile work compiled per group;
// 0.90 ms when the group was a run-time branch of the amplitude loop): it executes the same
// instructions at a lower issue rate, waiting at each tile's block barrier for the
// completion counting and the next take.  Iteration 0.955 against 0.935 ms.
static bool hh_forced_off() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("EMUSV_FUSED_PASS_H");
        v = (e && e[0] == '1') ? 0 : 1;
    }
    return v == 1;
}

// The Lanczos iteration of this register runs in the H-first order (pass H kernels, then
// the recurrence pass L): registers wider than one pass-L tile.
bool lz_applies(int dtype, int n) {
    if (dtype == EMUSV_C64) return n > LzShape<float>::TB;
    if (dtype == EMUSV_C128) return n > LzShape<double>::TB;
    return false;
}

template <typename R, bool REALC, int MODE, int C0>
static int launch_lz_c(const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out) {
    typedef typename cvec<R>::T C;
    constexpr int TB = LzShape<R>::TB, RB = LzShape<R>::RB, NT = 1 << (TB - RB);
    PassParams P;
    fill_params(H, TB, RB, &P);
    auto kern = k_pass_lz<R, REALC, TB, RB, MODE, C0>;
    const size_t smem = pass_lz_smem<C, TB>();
    EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    const int64_t ntiles = int64_t(1) << (H.n - TB);
    int64_t grid = (int64_t)sm_count() * per_sm;
    if (grid > ntiles) grid = ntiles;
    {
        ProfScope ps_(MODE == LZ_ITER ? PROF_HPSI : PROF_HPSI_AUX, s);
        kern<<<(unsigned)grid, NT, smem, s>>>(P, A);
    }
    EMUSV_CHECK_LAUNCH();
    if (grid_out) *grid_out = (int)grid;
    return EMUSV_OK;
}

// The pass L leaves out the chunk bits of the register's pass H rows.
template <typename R, bool REALC, int MODE>
static int launch_lz(const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out) {
    constexpr int CMIN = PassShape<R>::CMIN;
    if (lz_chunk_bits<R>(H.n) == CMIN) return launch_lz_c<R, REALC, MODE, CMIN>(H, A, s, grid_out);
    return launch_lz_c<R, REALC, MODE, CMIN - 1>(H, A, s, grid_out);
}
template <int MODE>
static int launch_lz_mode(int dtype, const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out) {
    if (H.noisy || !lz_applies(dtype, H.n)) return EMUSV_BAD_ARGUMENT;
    if (dtype == EMUSV_C64)
        return H.real_coef ? launch_lz<float, true, MODE>(H, A, s, grid_out)
                           : launch_lz<float, false, MODE>(H, A, s, grid_out);
    return H.real_coef ? launch_lz<double, true, MODE>(H, A, s, grid_out)
                       : launch_lz<double, false, MODE>(H, A, s, grid_out);
}

// Start of a run: partials 4-5 of <u, (D - sigma + X_low) u> (A.u, A.eshift, A.partials,
// A.gate, A.err).
int lz_energy0(int dtype, const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out) {
    return launch_lz_mode<LZ_E0>(dtype, H, A, s, grid_out);
}

// The recurrence pass: w = H v_j - a v_j - b v_{j-1} (see k_pass_lz).
int lz_low(int dtype, const HamParams &H, const LzArgs &A, cudaStream_t s, int *grid_out) {
    return launch_lz_mode<LZ_ITER>(dtype, H, A, s, grid_out);
}

// Both groups of a two-group pass H in one persistent launch (k_pass_hh): group 1 on the
// g bits from hskip (the pass-L tile width), applying [hskip, n - g); group 2 on the top g
// bits.  cnt: HH_CNT_WORDS zero-initialised words of device memory.
template <typename R, bool REALC, int CMIN>
static int launch_hh(PassParams P, const PassArgs &A, unsigned *cnt, int hskip, cudaStream_t s,
                     int *grid_out) {
    typedef typename cvec<R>::T C;
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, NT = 1 << (TB - RB);
    const int n = P.n, g = TB - CMIN, hs = hskip, hpos2 = n - g, nsb = hs - CMIN, tb = n - hs - g;
    if (!cnt || nsb < 1 || nsb > HH_MAX_NS_BITS || tb < 1 || hpos2 > hs + g) return EMUSV_BAD_ARGUMENT;
    static_assert(HH_CNT_WORDS <= 1040, "KState::hh_cnt holds the fused pass H counters");
    auto kern = k_pass_hh<R, REALC, TB, RB, CMIN>;
    const size_t smem = pass_hh_smem<C, TB>();
    EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) per_sm = 1;
    const int64_t grid = (int64_t)sm_count() * per_sm;
    P.hg = g;
    P.hc = CMIN;
    P.pbh = 0;
    P.hskip = hskip;
    P.hbox_rows = g > 8 ? 256 : (1 << g);
    PassHHMaps M;
    memset(&M, 0, sizeof(M));
    P.hpos = hs;
    if (!encode_pass_high(&M.u1, A.u, n, (int)sizeof(C), P)) return EMUSV_CUDA_ERROR;
    P.hpos = hpos2;
    if (!encode_pass_high(&M.u2, A.u, n, (int)sizeof(C), P) ||
        !encode_pass_high(&M.p2, A.out, n, (int)sizeof(C), P))
        return EMUSV_CUDA_ERROR;
    HHArgs H = {};
    H.u = A.u;
    H.part = A.out;
    H.partials = A.partials;
    H.gate = A.gate;
    H.err = A.err;
    H.cnt = cnt;
    H.hs = hs;
    H.hpos2 = hpos2;
    H.ns_bits = nsb;
    H.tps_bits = tb;
    EMUSV_CHECK(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * ((size_t(1) << nsb) + 1), s));
    {
        ProfScope ps_(PROF_HPSI_HIGH, s);
        kern<<<(unsigned)grid, NT, smem, s>>>(P, H, M);
    }
    EMUSV_CHECK_LAUNCH();
    if (grid_out) *grid_out = (int)grid;
    return EMUSV_OK;
}

// part = X_high u (unscaled flips of every bit above the pass-L tile, and of the CMIN
// chunk bits of the pass H rows, applied by the last pass) in one or two strided passes;
// their <u, X u> partials go to partials[0 .. *nblocks_out) (rows of NRED); *c0_out = CMIN
// (the bits the recurrence pass L leaves out).
template <typename R, bool REALC, int CMIN>
static int lz_high_t(const HamParams &H, const void *u, void *part, double *partials, const int *gate,
                     int *err, unsigned *cnt, cudaStream_t s, int *nblocks_out, int *c0_out) {
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, TBL = LzShape<R>::TB;
    const int n = H.n, rem = n - TBL, G = TB - CMIN;
    if (rem < 1 || rem > 2 * G) return EMUSV_BAD_ARGUMENT;
    PassParams P;
    fill_params(H, TB, RB, &P);
    PassArgs A = {};
    A.u = u;
    A.su = 1.0;
    A.out = part;
    A.partials = partials;
    A.gate = gate;
    A.err = err;
    int g1 = 0, g2 = 0, st;
    *c0_out = CMIN;
    if (rem > G && !hh_forced_off() &&
        launch_hh<R, REALC, CMIN>(P, A, cnt, TBL, s, &g2) == EMUSV_OK) {  // one fused launch
        *nblocks_out = g2;
        return EMUSV_OK;
    }
    if (rem > G) {
        if ((st = launch_high<R, REALC, EPI_X_FIRST, CMIN>(P, n - 2 * G, A, nullptr, s, &g1, TBL))) return st;
        A.partials = partials + (size_t)g1 * NRED;
        if ((st = launch_high<R, REALC, EPI_X_ADD, CMIN, true>(P, n - G, A, part, s, &g2, TBL))) return st;
    } else {
        if ((st = launch_high<R, REALC, EPI_X_FIRST, CMIN, true>(P, n - G, A, nullptr, s, &g2, TBL)))
            return st;
    }
    *nblocks_out = g1 + g2;
    return EMUSV_OK;
}

template <typename R, bool REALC>
static int lz_high_rows(const HamParams &H, const void *u, void *part, double *partials, const int *gate,
                        int *err, unsigned *cnt, cudaStream_t s, int *nb) {
    constexpr int CMIN = PassShape<R>::CMIN;
    int c0 = 0;
    if (lz_chunk_bits<R>(H.n) == CMIN) return lz_high_t<R, REALC, CMIN>(H, u, part, partials, gate, err, cnt, s, nb, &c0);
    return lz_high_t<R, REALC, CMIN - 1>(H, u, part, partials, gate, err, cnt, s, nb, &c0);
}

int lz_high(int dtype, const HamParams &H, const void *u, void *part, double *partials, const int *gate,
            int *err, unsigned *cnt, cudaStream_t s, int *nblocks_out);

// Moments of H on psi through the passes (registers wider than one pass-L tile): the pass
// H kernels write part = X_high psi into `part` (a vector of the register's size), then the
// moments pass forms H psi tile by tile: partials 0 ||H psi||^2, 1-2 <psi, H psi> into
// `partials` (*grid_out rows); the pass H kernels' own partials go to `part_h`.
int lz_moments(int dtype, const HamParams &H, const void *psi, void *part, double *partials,
               double *part_h, unsigned *cnt, int *err, cudaStream_t s, int *grid_out) {
    int nh = 0;
    int st = lz_high(dtype, H, psi, part, part_h, nullptr, err, cnt, s, &nh);
    if (st) return st;
    LzArgs A = {};
    A.u = psi;
    A.part = part;
    A.partials = partials;
    A.err = err;
    return launch_lz_mode<LZ_M2>(dtype, H, A, s, grid_out);
}

int lz_high(int dtype, const HamParams &H, const void *u, void *part, double *partials, const int *gate,
            int *err, unsigned *cnt, cudaStream_t s, int *nblocks_out) {
    if (H.noisy || !lz_applies(dtype, H.n)) return EMUSV_BAD_ARGUMENT;
    if (dtype == EMUSV_C64)
        return H.real_coef ? lz_high_rows<float, true>(H, u, part, partials, gate, err, cnt, s, nblocks_out)
                           : lz_high_rows<float, false>(H, u, part, partials, gate, err, cnt, s, nblocks_out);
    return H.real_coef ? lz_high_rows<double, true>(H, u, part, partials, gate, err, cnt, s, nblocks_out)
                       : lz_high_rows<double, false>(H, u, part, partials, gate, err, cnt, s, nblocks_out);
}

}  // namespace emusv
