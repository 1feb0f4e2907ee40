// Launch accounting hooks (see profile.cu).
#pragma once

#include "common.cuh"

namespace emusv {

enum ProfKind {
    PROF_HPSI = 0,     // fused H*psi (all modes)
    PROF_ORTH = 1,     // Gram-Schmidt / axpy / norm passes
    PROF_SMALL = 2,    // small FP64 kernels (Krylov exponential, reductions' tails)
    PROF_COMBINE = 3,  // Krylov-basis combination
    PROF_OBS = 4,      // observables
    PROF_ADJOINT = 5,  // adjoint contractions
    PROF_BATCH = 6,    // batched persistent evolution
    PROF_HPSI_HIGH = 7,  // pass H of the two-pass H*psi
    PROF_HPSI_AUX = 8,   // the Lanczos pass L's other modes: start-of-step energy, moments
    PROF_KINDS = 9
};

void prof_begin_launch(int kind, cudaStream_t s, void **token);
void prof_end_launch(void *token, cudaStream_t s);

// RAII bracket around one kernel launch.
struct ProfScope {
    void *tok;
    cudaStream_t s;
    ProfScope(int kind, cudaStream_t st) : tok(nullptr), s(st) { prof_begin_launch(kind, st, &tok); }
    ~ProfScope() { prof_end_launch(tok, s); }
};

}  // namespace emusv
