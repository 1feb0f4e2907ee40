// Energy moments without any allocation: the partial-sum scratch of the reduction is a
// file-scope static device array owned by this library.
//
// Who needs it: code that must not allocate device memory at the point of the call --
// for example a caller running under an external memory manager that forbids
// cudaMalloc/cudaFree, or a host runtime (a C or Fortran simulator, an FFI binding) that
// has no device allocator of its own to hand over a scratch buffer.  emusv_expect needs a
// caller-provided scratch buffer; this entry point needs none.
//
// Limits and sharing:
//  * the scratch holds FP64 partial sums of at most NOALLOC_BLOCKS thread blocks plus the
//    final sums (about 66 KB per GPU); it lives on every GPU that loads the library until
//    the process exits;
//  * registers of up to EMUSV_MAX_QUBITS qubits are accepted (the launch never uses more
//    blocks than the scratch holds: larger registers are walked grid-stride); larger
//    requests are rejected with EMUSV_BAD_ARGUMENT;
//  * every call shares the one array: calls whose work overlaps on the GPU (different
//    streams without ordering) race on it and must be serialised by the caller;
//  * nothing in the array has to start at zero: every block overwrites its own partial
//    sums before they are added up;
//  * the array's device address is resolved by the first call on each device and kept for
//    the process; a cudaDeviceReset of that device invalidates it, so a process that
//    resets a device must not call this entry point on it afterwards.
#include <mutex>

#include "hpsi_kernel.cuh"
#include "profile.cuh"

namespace emusv {

int hpsi_tile_bits(int n);
int launch_hpsi(int dtype, int mode, const HamParams &P, HpsiArgs A, int max_grid,
                cudaStream_t s, int *grid_out);

namespace {

constexpr int NOALLOC_BLOCKS = 1024;
constexpr int NOALLOC_DOUBLES = NOALLOC_BLOCKS * NRED + 64;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double *g_scratch_ptr[MAX_DEVICES] = {};

// Device address of the static scratch on the current device: the first call on a device
// resolves it with cudaGetSymbolAddress (with that device current) and keeps it.
int scratch_address(double **out) {
    int dev = 0;
    EMUSV_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return EMUSV_BAD_ARGUMENT;
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        EMUSV_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_ptr[dev] = reinterpret_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return EMUSV_OK;
}

// One block: result[0..1] = <v,Hv>, result[2] = ||Hv||^2 from the per-block partials.
__global__ void k_noalloc_finish(const double *partials, int nblocks, double *result) {
    __shared__ double red[(BLOCK / 32) * NRED];
    double v[NRED];
    sum_partials<NRED>(partials, nblocks, NRED, v, red);
    if (threadIdx.x == 0) {
        result[0] = v[1];
        result[1] = v[2];
        result[2] = v[0];
    }
}

}  // namespace
}  // namespace emusv

using namespace emusv;

extern "C" int emusv_expect_noalloc(int nqubits, int dtype, const double *omegas,
                                    const double *deltas, const double *phis,
                                    const double *interaction, const void *psi,
                                    double *result_dev, void *stream) {
    HamParams P;
    if (nqubits < 1 || nqubits > EMUSV_MAX_QUBITS || !psi || !result_dev ||
        (dtype != EMUSV_C128 && dtype != EMUSV_C64) ||
        !make_params(nqubits, omegas, deltas, phis, interaction, &P))
        return EMUSV_BAD_ARGUMENT;
    double *scratch = nullptr;
    int st = scratch_address(&scratch);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    HpsiArgs A = {};
    A.u = psi;
    A.su = 1.0;
    A.partials = scratch;
    A.tile_bits = hpsi_tile_bits(nqubits);
    int grid = 0;
    // max_grid = NOALLOC_BLOCKS: the energy reduction (single-pass kernel) never launches
    // more blocks than that, walking larger registers grid-stride, so the partial sums
    // fit the static array
    st = launch_hpsi(dtype, HP_ENERGY, P, A, NOALLOC_BLOCKS, s, &grid);
    if (st) return st;
    {
        ProfScope ps_(PROF_SMALL, s);
        k_noalloc_finish<<<1, BLOCK, 0, s>>>(scratch, grid, result_dev);
    }
    EMUSV_CHECK_LAUNCH();
    return EMUSV_OK;
}
