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
// tiles (32 KiB), 8 per thread; 256 threads and two CTAs per SM either way.  Clusters of
// up to 8 CTAs in pass L and pass H; pass H reads 32-byte chunks.
template <> struct PassShape<float> {
    static constexpr int TB = 12, RB = 4, PBMAX = 2, PBHMAX = 3, CMIN = 2;
};
template <> struct PassShape<double> {
    static constexpr int TB = 11, RB = 3, PBMAX = 3, PBHMAX = 3, CMIN = 1;
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
static bool encode_pass_high(CUtensorMap *map, const void *base, int n, int es, const PassParams &P,
                             int cm) {
    auto fn = encode_fn();
    if (!fn) return false;
    const int K = es / 8;
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
    const int c = P.hc, g = P.hg, hpos = P.hpos, pbh = P.pbh;
    if (P.hsplit == 0) {
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
    } else {
        dims[0] = (cuuint64_t(1) << cm) * K;
        dims[1] = cuuint64_t(1) << (c - cm);
        dims[2] = cuuint64_t(1) << (hpos - c);
        dims[3] = cuuint64_t(1) << g;
        dims[4] = cuuint64_t(1) << (n - hpos - g);
        strides[0] = (cuuint64_t(es) << cm);
        strides[1] = (cuuint64_t(es) << c);
        strides[2] = (cuuint64_t(es) << hpos);
        strides[3] = (cuuint64_t(es) << (hpos + g));
        box[0] = (cuuint32_t)dims[0];
        box[1] = (cuuint32_t)dims[1];
        box[2] = 1;
        box[3] = (cuuint32_t)P.hbox_rows;
        box[4] = 1;
    }
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

// Kernel pointers by run-time layout (template arguments are compile-time).
template <typename R, bool REALC, int TB, int RB, int EPI>
static auto low_kernel(int pb) -> decltype(&k_pass_low<R, REALC, TB, RB, EPI, 0>) {
    switch (pb) {
    case 0: return k_pass_low<R, REALC, TB, RB, EPI, 0>;
    case 1: return k_pass_low<R, REALC, TB, RB, EPI, 1>;
    case 2: return k_pass_low<R, REALC, TB, RB, EPI, 2>;
    default: return k_pass_low<R, REALC, TB, RB, EPI, 3>;
    }
}
template <typename R, bool REALC, int TB, int RB, int EPI, int CMIN>
static auto high_kernel(bool hot, int pbh) -> decltype(&k_pass_high<R, REALC, TB, RB, EPI, 0, 0>) {
    if (hot) {
        switch (pbh) {
        case 0: return k_pass_high<R, REALC, TB, RB, EPI, CMIN, 0>;
        case 1: return k_pass_high<R, REALC, TB, RB, EPI, CMIN, 1>;
        case 2: return k_pass_high<R, REALC, TB, RB, EPI, CMIN, 2>;
        default: return k_pass_high<R, REALC, TB, RB, EPI, CMIN, 3>;
        }
    }
    return pbh == 0 ? k_pass_high<R, REALC, TB, RB, EPI, 0, 0> : k_pass_high<R, REALC, TB, RB, EPI, 0, 3>;
}

template <typename R, bool REALC, int EPI_H>
static int run_passes(const HamParams &H, const HpsiArgs &HA, cudaStream_t s, int *grid_out) {
    typedef typename cvec<R>::T C;
    constexpr int TB = PassShape<R>::TB, RB = PassShape<R>::RB, NT = 1 << (TB - RB);
    constexpr int CMIN = PassShape<R>::CMIN;
    const int n = H.n;
    PassParams P;
    fill_params(H, TB, RB, &P);
    int pb = n - TB;
    if (pb > PassShape<R>::PBMAX) pb = PassShape<R>::PBMAX;
    P.pb = pb;
    const int rem = n - TB - pb;
    int g = rem;
    if (g > TB - CMIN) g = TB - CMIN;
    int pbh = rem - g;
    if (pbh > PassShape<R>::PBHMAX) pbh = PassShape<R>::PBHMAX;
    P.hg = g;
    P.hc = TB - g;
    P.hpos = TB + pb;
    P.pbh = pbh;
    P.xb_lo = TB + pb + g + pbh;
    P.xb_hi = n;
    constexpr int K = sizeof(C) / 8;
    // chunk rows wider than one 256-element TMA box dimension are split in two dims
    int cm = 0;
    while (((1 << (cm + 1)) * K) <= 256 && cm + 1 <= P.hc) ++cm;
    P.hsplit = ((1 << P.hc) * K > 256) ? 1 : 0;
    P.hbox_rows = g > 8 ? 256 : (1 << g);
    if (P.hsplit && pbh) return EMUSV_BAD_ARGUMENT;  // not a layout the sizes above produce
    const bool hot = P.hc == CMIN && P.xb_lo == n;
    if (!hot && pbh != 0 && pbh != 3) return EMUSV_BAD_ARGUMENT;

    PassArgs A = {};
    A.u = HA.u;
    A.su_dev = HA.su_dev;
    A.su = HA.su;
    A.out = rem > 0 ? HA.part_buf : HA.out;  // pass L output
    A.partials = HA.partials;
    A.gate = HA.gate;
    A.err = HA.err;
    if (rem > 0 && !HA.part_buf) return EMUSV_BAD_ARGUMENT;  // pass H needs the partial buffer

    const size_t smem_l = pass_low_smem<C, TB>(), smem_h = pass_high_smem<C, TB>();
    const int nsm = sm_count();
    // ---- pass L
    {
        auto kern = (rem > 0) ? low_kernel<R, REALC, TB, RB, EPI_PARTIAL>(pb)
                              : low_kernel<R, REALC, TB, RB, EPI_H>(pb);
        EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_l));
        int per_sm = 0;
        EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem_l));
        if (per_sm < 1) per_sm = 1;
        const int CS = 1 << pb;
        const int64_t ncta = int64_t(1) << (n - TB);
        int64_t grid = (int64_t)nsm * per_sm;
        if (grid > ncta) grid = ncta;
        grid = grid / CS * CS;
        if (grid < CS) grid = CS;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid, 1, 1);
        cfg.blockDim = dim3(NT, 1, 1);
        cfg.dynamicSmemBytes = smem_l;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CS;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        {
            ProfScope ps_(PROF_HPSI, s);
            EMUSV_CHECK(cudaLaunchKernelEx(&cfg, kern, P, A));
        }
        if (rem == 0 && grid_out) *grid_out = (int)grid;
    }
    if (rem == 0) return EMUSV_OK;
    // ---- pass H: partial sums (pass L output) and values staged by TMA, final into HA.out
    {
        PassHighMaps M;
        if (!encode_pass_high(&M.u, HA.u, n, (int)sizeof(C), P, cm) ||
            !encode_pass_high(&M.part, HA.part_buf, n, (int)sizeof(C), P, cm))
            return EMUSV_CUDA_ERROR;
        PassArgs AH = A;
        AH.out = HA.out;
        auto kern = high_kernel<R, REALC, TB, RB, EPI_H, CMIN>(hot, pbh);
        EMUSV_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_h));
        int per_sm = 0;
        EMUSV_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem_h));
        if (per_sm < 1) per_sm = 1;
        const int CS = 1 << pbh;
        const int64_t ntiles = int64_t(1) << (n - P.hc - P.hg);
        int64_t grid = (int64_t)nsm * per_sm;
        if (grid > ntiles) grid = ntiles;
        grid = grid / CS * CS;
        if (grid < CS) grid = CS;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid, 1, 1);
        cfg.blockDim = dim3(NT, 1, 1);
        cfg.dynamicSmemBytes = smem_h;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CS;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        {
            ProfScope ps_(PROF_HPSI_HIGH, s);
            EMUSV_CHECK(cudaLaunchKernelEx(&cfg, kern, P, AH, M));
        }
        if (grid_out) *grid_out = (int)grid;
    }
    return EMUSV_OK;
}

// mode: HP_STORE or HP_LANCZOS (values of HpsiMode)
int launch_hpsi_passes(int dtype, int mode, const HamParams &H, const HpsiArgs &A,
                       cudaStream_t s, int *grid_out) {
    const bool lz = mode == HP_LANCZOS;
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
