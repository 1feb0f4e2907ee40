// Host side of the two-pass H*psi: layout choice, parameter tables, cluster launches.
#include <cudaTypedefs.h>
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

template <typename R, bool REALC, int EPI, bool NOISY, bool ORTH = false>
static int launch_low(const PassParams &P, const PassArgs &A, cudaStream_t s, int *grid_out) {
    typedef typename cvec<R>::T C;
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, NT = 1 << (TB - RB);
    auto kern = k_pass_low<R, REALC, TB, RB, EPI, 0, NOISY, ORTH>;
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
// group bits below TB were applied by pass L and are skipped.
template <typename R, bool REALC, int EPI, int CMIN>
static int launch_high(PassParams P, int hpos, const PassArgs &A, const void *part,
                       cudaStream_t s, int *grid_out) {
    typedef typename cvec<R>::T C;
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, NT = 1 << (TB - RB);
    const int n = P.n, g = TB - CMIN;
    if (hpos < CMIN || hpos + g > n) return EMUSV_BAD_ARGUMENT;
    P.hg = g;
    P.hc = CMIN;
    P.hpos = hpos;
    P.pbh = 0;
    P.hskip = TB;
    P.hbox_rows = g > 8 ? 256 : (1 << g);
    PassHighMaps M;
    if (!encode_pass_high(&M.u, A.u, n, (int)sizeof(C), P) ||
        !encode_pass_high(&M.part, part, n, (int)sizeof(C), P))
        return EMUSV_CUDA_ERROR;
    auto kern = k_pass_high<R, REALC, TB, RB, EPI, CMIN, 0>;
    const size_t smem = pass_high_smem<C, TB>();
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
// stages: bit 0 = pass L, bit 1 = the H passes, bit 2 = pass L with the Lanczos recurrence
// fused in front (ORTH; the H passes of the same H*psi follow in a later call)
template <typename R, bool REALC, int EPI_F, int CMIN, bool NOISY>
static int run_passes(const HamParams &H, const HpsiArgs &HA, cudaStream_t s, int *grid_out,
                      int stages = 3) {
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
        if (stages != 3) return EMUSV_BAD_ARGUMENT;
        A.out = HA.out;
        return launch_low<R, REALC, EPI_F, NOISY>(P, A, s, grid_out);
    }
    A.out = HA.part_buf;
    if (stages & 4) {
        if constexpr (!NOISY) {
            A.vj = HA.vj;
            A.vp = HA.vp;
            A.ocoef = HA.ocoef;
            A.oscale = HA.oscale;
            A.part_o = HA.part_o;
            return launch_low<R, REALC, EPI_PARTIAL, false, true>(P, A, s, grid_out);
        }
        return EMUSV_BAD_ARGUMENT;
    }
    if (stages & 1)
        if ((st = launch_low<R, REALC, EPI_PARTIAL, NOISY>(P, A, s, nullptr))) return st;
    if (!(stages & 2)) return EMUSV_OK;
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
static int run_passes(const HamParams &H, const HpsiArgs &HA, cudaStream_t s, int *grid_out,
                      int stages = 3) {
    constexpr int TB = PassShape<R>::TB, CMIN = PassShape<R>::CMIN;
    if (H.n - TB <= 2 * (TB - CMIN))
        return run_passes<R, REALC, EPI_F, CMIN, NOISY>(H, HA, s, grid_out, stages);
    return run_passes<R, REALC, EPI_F, CMIN - 1, NOISY>(H, HA, s, grid_out, stages);
}

// The stages of a multi-pass Lanczos H*psi launched separately (stages as run_passes):
// 1 = pass L of v_0, 2 = the H passes (their partial sums from a previous pass L),
// 4 = the recurrence of the previous iteration fused into this iteration's pass L.
int launch_hpsi_stage(int dtype, int stages, const HamParams &H, const HpsiArgs &A, cudaStream_t s,
                      int *grid_out) {
    if (H.noisy) return EMUSV_BAD_ARGUMENT;
    if (dtype == EMUSV_C64)
        return H.real_coef ? run_passes<float, true, EPI_LANCZOS>(H, A, s, grid_out, stages)
                           : run_passes<float, false, EPI_LANCZOS>(H, A, s, grid_out, stages);
    if (dtype == EMUSV_C128)
        return H.real_coef ? run_passes<double, true, EPI_LANCZOS>(H, A, s, grid_out, stages)
                           : run_passes<double, false, EPI_LANCZOS>(H, A, s, grid_out, stages);
    return EMUSV_BAD_ARGUMENT;
}

// Registers whose H*psi takes more than one pass (the fused recurrence needs pass L to
// produce partial sums for later passes).
bool hpsi_multipass(int dtype, int n) {
    return n > (dtype == EMUSV_C64 ? PassShape<float>::TB : PassShape<double>::TB);
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

}  // namespace emusv
