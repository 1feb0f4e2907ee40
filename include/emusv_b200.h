/*
 * emusv_b200 -- C ABI of the B200-native emu-sv time-evolution hot path.
 *
 * Every entry point takes plain pointers and sizes, runs on the CUDA stream passed as
 * `stream` (a cudaStream_t; NULL = legacy default stream), and returns an emusv_status.
 * Vectors are device pointers to interleaved complex amplitudes of length 2^nqubits:
 * complex128 (double re, im) for EMUSV_C128 and complex64 (float re, im) for EMUSV_C64.
 * Qubit 0 is the most significant bit of the amplitude index; bit value 1 is the Rydberg
 * state |r> (reference emu_sv/state_vector.py, emu_sv/hamiltonian.py).
 *
 * Hamiltonian parameters are HOST pointers:
 *   omegas[n]      Rabi frequencies Omega_i (rad/us; halved inside, hamiltonian.py:52)
 *   deltas[n]      detunings delta_i (rad/us)
 *   phis[n]        laser phases phi_i (rad)
 *   interaction[n*n] row-major U_ij (rad/us); only the upper triangle i<j is read
 *                  (hamiltonian.py:153-161).
 *   H = sum_i Omega_i/2 (cos phi_i X_i + sin phi_i Y_i) - sum_i delta_i n_i
 *       + sum_{i<j} U_ij n_i n_j
 *
 * Workspace-taking calls use only the memory they are given; none of them allocates.
 */
#ifndef EMUSV_B200_H
#define EMUSV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMUSV_MAX_QUBITS 30

typedef enum {
    EMUSV_OK = 0,
    EMUSV_NOT_CONVERGED = 1,      /* Krylov iteration reached max_krylov_dim (RecursionError) */
    EMUSV_NONFINITE = 2,          /* NaN/Inf met in a reduction */
    EMUSV_BAD_ARGUMENT = 3,       /* size, pointer or alignment check failed */
    EMUSV_WORKSPACE_TOO_SMALL = 4, /* the Krylov basis needs more vectors than given */
    EMUSV_CUDA_ERROR = 5,         /* a CUDA runtime call failed */
    EMUSV_TIMEOUT = 6             /* a bounded device-side wait gave up */
} emusv_status;

typedef enum { EMUSV_C128 = 0, EMUSV_C64 = 1 } emusv_dtype;

/* Per-call Krylov statistics (host struct, filled on return). */
typedef struct {
    int iterations;       /* Lanczos iterations j+1 at exit (krylov_exp.py:92-96) */
    int happy_breakdown;  /* 1 if ||w|| < norm_tolerance ended the iteration */
    int converged;        /* 1 if the error estimate fell below exp_tolerance */
    int basis_vectors;    /* Krylov vectors combined into the result */
    double error_estimate; /* last Expokit estimate (krylov_exp.py:81-84) */
    double input_norm;    /* ||psi_in|| */
    double output_norm;   /* ||psi_out|| (FP64 reduction fused into the combination) */
    int second_rounds;    /* emusv_arnoldi_step: basis vectors orthogonalised a second time
                             (lagged into the next iteration; 0 for the Lanczos steps) */
} emusv_krylov_info;

/* Library identification: returns the sm architecture compiled in (e.g. 100). */
int emusv_build_arch(void);
const char *emusv_status_string(int status);
/* Reads and clears the device error word of calls that have no status output of their
 * own (emusv_hpsi): EMUSV_OK, or EMUSV_TIMEOUT if a bounded device-side wait gave up.
 * Synchronises the stream. */
int emusv_device_error(void *stream);

/* Diagonal of H, float64 [2^n] on the device.
 * Replaces RydbergHamiltonian._create_diagonal (emu_sv/hamiltonian.py:139-162). */
int emusv_hamiltonian_diag(int nqubits, const double *deltas, const double *interaction,
                           double *diag_out, void *stream);

/* out = H psi, fused in one pass (diagonal rebuilt on chip, all flip terms).
 * Replaces RydbergHamiltonian.__mul__ (emu_sv/hamiltonian.py:69-137). out != psi. */
int emusv_hpsi(int nqubits, int dtype, const double *omegas, const double *deltas,
               const double *phis, const double *interaction, const void *psi, void *out,
               void *stream);

/* Bytes of device scratch the reduction entry points below need: FP64 partial sums, and
 * for emusv_expect on registers wider than one streaming tile (complex64 and complex128
 * from 12 qubits) one vector of the register's size, which holds the flips of the high
 * bits between the streaming passes.  The scratch must be 256-byte aligned. */
size_t emusv_scratch_bytes(int nqubits, int dtype);

/* result_dev[0..1] = <psi|H|psi> (re, im), result_dev[2] = <H psi|H psi>; device
 * float64 [3], no synchronisation.  Registers wider than one streaming tile run the
 * pass H kernels (the flips of the high bits into the scratch vector) and one pass that
 * forms H psi tile by tile without storing it; smaller ones one fused pass.  Replaces RydbergHamiltonian.expect
 * (hamiltonian.py:164-172) and the vdot(h, h) of energy_second_moment_sv_impl /
 * energy_variance_sv_impl (emu_sv/custom_callback_implementations.py:131-185). */
int emusv_expect(int nqubits, int dtype, const double *omegas, const double *deltas,
                 const double *phis, const double *interaction, const void *psi,
                 double *result_dev, void *scratch, size_t scratch_bytes, void *stream);

/* The same energy moments as emusv_expect with no scratch argument and no allocation:
 * the partial sums go to a static device array inside the library (about 66 KB per GPU,
 * kept until the process exits).  For callers that cannot allocate device memory at the
 * call site (code under an external memory manager that forbids cudaMalloc/cudaFree, host
 * runtimes without a device allocator).  Registers up to EMUSV_MAX_QUBITS; larger ones give
 * EMUSV_BAD_ARGUMENT.  The first call on a device resolves the array's address
 * (cudaGetSymbolAddress, with that device current) and should come before any stream
 * capture; the address is kept for the process, so the entry point must not be used on a
 * device after a cudaDeviceReset of it.  All calls share the array, so calls that overlap
 * on the GPU race.  No counterpart in the reference: it has no C interface. */
int emusv_expect_noalloc(int nqubits, int dtype, const double *omegas, const double *deltas,
                         const double *phis, const double *interaction, const void *psi,
                         double *result_dev, void *stream);

/* occ_dev[i] = sum_x |psi_x|^2 x_i (device float64 [n]), one pass over psi.
 * Replaces qubit_occupation_sv_impl (emu_sv/custom_callback_implementations.py:30-47). */
int emusv_occupation(int nqubits, int dtype, const void *psi, double *occ_dev, void *scratch,
                     size_t scratch_bytes, void *stream);

/* corr_dev[i*n+j] = sum_x |psi_x|^2 x_i x_j (device float64 [n*n]), one pass over psi.
 * Replaces correlation_matrix_sv_impl (custom_callback_implementations.py:77-102). */
int emusv_correlation(int nqubits, int dtype, const void *psi, double *corr_dev, void *scratch,
                      size_t scratch_bytes, void *stream);

/* Bytes of device workspace emusv_krylov_step needs for a basis of `basis_capacity`
 * stored Krylov vectors (the input vector is used in place and is not counted; one more
 * vector holds the partial sums of the two-pass H*psi). */
size_t emusv_krylov_workspace_bytes(int nqubits, int dtype, int basis_capacity);

/* One time step psi_out = exp(-i dt H) psi_in by Lanczos with the Expokit error
 * estimate, all arithmetic on the GPU (FP64 scalars and tridiagonal exponential).
 * Replaces DifferentiableStateVectorEvolution.forward/evolve
 * (emu_sv/time_evolution/torch.py:143-219) with krylov_exp
 * (emu_base/math/krylov_exp.py:23-131) and RydbergHamiltonian.__mul__ as the operator.
 * Convergence is tested on the device at every iteration, as the reference does; the
 * host reads the device's decision from iteration `krylov_dim_hint` on (0: every
 * iteration), so the hint only saves host synchronisations and never moves the stopping
 * iteration.
 * The workspace carries one value from call to call: the previous step's energy, which
 * the next step subtracts from H inside H*psi (same basis and coefficients; less
 * complex64 rounding of the diagonal).  Zero the workspace once before its first call.
 * psi_out may equal psi_in.  Returns EMUSV_NOT_CONVERGED (result still written, as
 * krylov_exp_impl does) or EMUSV_WORKSPACE_TOO_SMALL (nothing written; retry with a
 * larger basis).  `info` (host) may be NULL.  Synchronises the stream at every
 * convergence test. */
int emusv_krylov_step(int nqubits, int dtype, double dt, const double *omegas,
                      const double *deltas, const double *phis, const double *interaction,
                      const void *psi_in, void *psi_out, double exp_tolerance,
                      double norm_tolerance, int max_krylov_dim, int krylov_dim_hint,
                      void *workspace, size_t workspace_bytes, emusv_krylov_info *info,
                      void *stream);

/* Bytes of device workspace emusv_adjoint_step needs when each of its two Lanczos bases
 * may hold `basis_capacity` vectors (3 * (capacity + 1) + 1 vectors of 2^n amplitudes
 * plus small tables); 0 for registers above 20 qubits. */
size_t emusv_adjoint_workspace_bytes(int nqubits, int dtype, int basis_capacity);

/* Adjoint of one time step psi_out = exp(-i dt H) state: given grad_out = dL/dpsi_out
 * (torch's convention for complex tensors), writes dL/dOmega_i, dL/ddelta_i, dL/dphi_i
 * and dL/dU_ij (i < j; host float64 arrays, any of them may be NULL to skip it).
 * Replaces DifferentiableStateVectorEvolution.backward (emu_sv/time_evolution/torch.py:
 * 223-353) with double_krylov (emu_base/math/double_krylov.py:5-113); the state gradient
 * exp(+i dt H) grad_out (torch.py:355-366) is a separate emusv_krylov_step with -dt.
 * Returns EMUSV_NOT_CONVERGED (RecursionError, double_krylov.py:107-110) or
 * EMUSV_WORKSPACE_TOO_SMALL (retry with a larger capacity).  Registers up to 20 qubits.
 * Synchronises the stream. */
int emusv_adjoint_step(int nqubits, int dtype, double dt, const double *omegas,
                       const double *deltas, const double *phis, const double *interaction,
                       const void *state, const void *grad_out, double tolerance,
                       int max_krylov_dim, double *g_omegas, double *g_deltas, double *g_phis,
                       double *g_interaction, void *workspace, size_t workspace_bytes,
                       void *stream);

/* Bitstring sampling (emu_sv/utils.py:17-49 sample_indices, its inverse-CDF path for
 * every size): indices[k] = the first index whose FP64 cumulative |psi|^2 exceeds
 * uniforms[k] * sum|psi|^2 (searchsorted right=True), clamped to 2^n - 1.  uniforms
 * (device, [num_shots], in [0,1)) and indices (device int64) are caller-owned; the CDF is
 * never formed (block sums, their prefix, one warp per draw).  EMUSV_NONFINITE when the
 * total probability is not positive (the reference raises RuntimeError).  Synchronises. */
size_t emusv_sample_scratch_bytes(int nqubits);
int emusv_sample(int nqubits, int dtype, const void *psi, int num_shots, const double *uniforms,
                 long long *indices, void *scratch, size_t scratch_bytes, void *stream);

/* ---- noisy (non-Hermitian) path of the Monte Carlo stepper ----
 * `noise` (host, 8 doubles) is the 2x2 complex matrix -0.5i sum_j L_j^dag L_j of
 * compute_noise_from_lindbladians (emu_base/jump_lindblad_operators.py:79-93), row-major
 * with re/im interleaved: [00, 01, 10, 11]; it acts on every qubit. */

/* out = H psi with the noise term.  Replaces RydbergHamiltonian.__mul__ with noise
 * (emu_sv/hamiltonian.py:61-67 coefficients, 147-151 diagonal). out != psi. */
int emusv_hpsi_noisy(int nqubits, int dtype, const double *omegas, const double *deltas,
                     const double *phis, const double *interaction, const double *noise,
                     const void *psi, void *out, void *stream);

/* Bytes of device workspace emusv_arnoldi_step needs for `basis_capacity` stored vectors
 * (plus one vector of H*psi partial sums, the Hessenberg matrix and partial sums). */
size_t emusv_arnoldi_workspace_bytes(int nqubits, int dtype, int basis_capacity);

/* One step psi_out = exp(-i dt H) psi_in with H non-Hermitian (noise may be NULL: the
 * Hermitian H through the same Arnoldi path) by Arnoldi with the Expokit error estimate.
 * Like emusv_krylov_step, the workspace carries the previous step's energy, subtracted
 * from H inside H*psi (same basis and coefficients): zero it once before its first call. 
 * Replaces EvolveMonteCarlo.evolve (emu_sv/time_evolution/implementations.py:148-166),
 * i.e. krylov_exp with is_hermitian=False (emu_base/math/krylov_exp.py:23-131): full
 * orthogonalisation (classical Gram-Schmidt with the second round lagged by one iteration:
 * two streaming passes per iteration),
 * happy-breakdown test every iteration, convergence tested on the device from iteration
 * `krylov_dim_hint` on (0: every iteration); when the first test already converges the
 * earlier iterations are tested in order, so the stopping iteration is the reference's.
 * max_krylov_dim <= 100.  Same return codes as emusv_krylov_step.  Synchronises. */
int emusv_arnoldi_step(int nqubits, int dtype, double dt, const double *omegas, const double *deltas,
                       const double *phis, const double *interaction, const double *noise,
                       const void *psi_in, void *psi_out, double exp_tolerance, double norm_tolerance,
                       int max_krylov_dim, int krylov_dim_hint, void *workspace,
                       size_t workspace_bytes, emusv_krylov_info *info, void *stream);

/* Single-qubit reduced density matrices rho_i (i = qubit, device float64 [n][8]: 2x2
 * complex row-major) of an unnormalised state: Tr(O rho_i) is expect_batch's entry for
 * qubit i and operator O (emu_sv/algebra.py:4-25), the jump weights of
 * EvolveMonteCarlo.do_quantum_jump (implementations.py:168-190). */
size_t emusv_qubit_densities_scratch_bytes(int nqubits);
int emusv_qubit_densities(int nqubits, int dtype, const void *psi, double *rho_dev, void *scratch,
                          size_t scratch_bytes, void *stream);

/* psi <- op (x) on qubit `qubit`, in place; op host 2x2 complex (8 doubles).  Replaces
 * emu_sv/algebra.py:28-37 (apply). */
int emusv_apply_1q(int nqubits, int dtype, void *psi, int qubit, const double *op, void *stream);

/* ---- Lindblad density-matrix path (registers up to EMUSV_MAX_QUBITS / 2 qubits) ----
 * A density matrix is a device array of 2^N x 2^N complex amplitudes, row-major (the
 * reference's tensor layout).  `ops` (host, nops x 8 doubles) are the 2x2 jump operators
 * L_k, row-major with re/im interleaved; every L_k acts on every qubit. */

/* out = L(rho) = Heff rho - rho Heff^dag + i sum_kq L_kq rho L_kq^dag (Heff = H -
 * 0.5i sum L^dag L), the reference's RydbergLindbladian.__matmul__
 * (emu_sv/lindblad_operator.py:184-211) for Hermitian rho.  out != rho. */
int emusv_lindblad_apply(int nqubits, int dtype, const double *omegas, const double *deltas,
                         const double *phis, const double *interaction, int nops, const double *ops,
                         const void *rho, void *out, void *stream);

/* Workspace of emusv_lindblad_arnoldi_step for `basis_capacity` stored 4^N vectors. */
size_t emusv_lindblad_workspace_bytes(int nqubits, int dtype, int basis_capacity);

/* rho_out = exp(-i dt L) rho_in by the Arnoldi step of emusv_arnoldi_step on the 4^N
 * vector: EvolveDensityMatrix.apply (emu_sv/time_evolution/implementations.py:87-120,
 * krylov_exp with is_hermitian=False).  Same contract and return codes as
 * emusv_arnoldi_step (zero the workspace once; max_krylov_dim <= 100). */
int emusv_lindblad_arnoldi_step(int nqubits, int dtype, double dt, const double *omegas,
                                const double *deltas, const double *phis, const double *interaction,
                                int nops, const double *ops, const void *rho_in, void *rho_out,
                                double exp_tolerance, double norm_tolerance, int max_krylov_dim,
                                int krylov_dim_hint, void *workspace, size_t workspace_bytes,
                                emusv_krylov_info *info, void *stream);

/* Scratch of emusv_dm_energy (two 4^N vectors and partial sums). */
size_t emusv_dm_scratch_bytes(int nqubits, int dtype);

/* result_dev[0..1] = Tr(H rho), [2..3] = Tr(H^2 rho) (device float64 [4]; H without the
 * noise term): RydbergLindbladian.expect and the density-matrix energy moments
 * (lindblad_operator.py:213-218, custom_callback_implementations.py:150-200). */
int emusv_dm_energy(int nqubits, int dtype, const double *omegas, const double *deltas,
                    const double *phis, const double *interaction, const void *rho, double *result_dev,
                    void *scratch, size_t scratch_bytes, void *stream);

/* amps[r] = sqrt(max(Re rho[r][r], 0)) (device, 2^N amplitudes of rho's dtype): the
 * state-vector occupation / correlation reductions applied to it give Tr(rho n_i) and
 * Tr(rho n_i n_j) (custom_callback_implementations.py:50-135, the density-matrix forms). */
int emusv_dm_diagonal_amplitudes(int nqubits, int dtype, const void *rho, void *amps, void *stream);

/* Drive preparation: out[s * out_stride + q] = PCHIP interpolant of the knots
 * (x[k], y[s * y_stride + k]), k < nknots, at xq[q], for every signal s < nsignals and
 * query q < nqueries (device float64 arrays; x strictly increasing -- the caller checks,
 * as PCHIP1D._validate_xy does).  Replaces PCHIP1D (emu_base/math/pchip_torch.py:218-269)
 * as used per qubit and laser parameter by _extract_omega_delta_phi
 * (emu_base/pulser_adapter.py:155-231): monotone cubic Hermite interpolation, boundary
 * cubics extended outside [x[0], x[n-1]], every operation rounded as the reference
 * rounds it.  No synchronisation. */
int emusv_pchip_eval(int nknots, const double *x, int nsignals, const double *y, int64_t y_stride,
                     int nqueries, const double *xq, double *out, int64_t out_stride, void *stream);

/* ---- batched evolution: many registers in one persistent launch ----
 * Replaces running the reference's time loop (emu_sv/sv_backend_impl.py:197-209, one
 * krylov_exp per step, krylov_exp.py:23-131) once per register: every register of the
 * batch (its own size up to emusv_batch_max_qubits(), pulse and step count) takes all its
 * steps inside ONE cooperative persistent kernel.  States are packed back to back in
 * instance order (2^n_i amplitudes each) in one device buffer and evolved in place.
 * Host arrays, packed in instance order: omegas/deltas/phis [sum_i nsteps_i * n_i]
 * (step-major per instance, qubit order), interactions [sum_i n_i * n_i] (row-major,
 * upper triangle read), dt [ninst] (us).  tile_bits T (8-10 for complex64, 8-9 for
 * complex128, T <= every n_i) and blocks_per_sm are launch shapes (autotuned by the
 * Python layer); basis_capacity bounds the Krylov basis of every instance. */
int emusv_batch_max_qubits(void);
size_t emusv_batch_workspace_bytes(int ninst, const int *nqubits, const int *nsteps, int dtype,
                                   int tile_bits, int basis_capacity);
/* Uploads the tables (coefficients, interaction tables, per-instance layout) into the
 * workspace and records `states`; synchronises the stream. */
int emusv_batch_prepare(int ninst, const int *nqubits, const int *nsteps, const double *dt,
                        int dtype, const double *omegas, const double *deltas, const double *phis,
                        const double *interactions, void *states, double exp_tolerance,
                        double norm_tolerance, int max_krylov_dim, int tile_bits,
                        int basis_capacity, void *workspace, size_t workspace_bytes,
                        void *stream);
/* One memset and one cooperative launch (stream-ordered only, so it can be captured in a
 * CUDA graph and replayed): evolves every instance through all its steps. */
int emusv_batch_launch(int dtype, int tile_bits, int blocks_per_sm, void *workspace, void *stream);
/* Steps [first_step, first_step + steps) of the prepared batch on `states` (NULL: the
 * prepared states), in place; when `history` is given, the packed states after every
 * `history_every`-th step of the launch are also written to history slot
 * (k + 1) / history_every - 1 (slots of sum_i 2^n_i amplitudes): the checkpoints of a
 * checkpointed adjoint and the states it recomputes between them.  Capturable. */
int emusv_batch_launch_steps(int dtype, int tile_bits, int blocks_per_sm, int first_step,
                             int steps, void *states, void *history, int history_every,
                             void *workspace, void *stream);
/* CTAs per SM the persistent kernel can keep resident for this shape (0: no such shape). */
int emusv_batch_max_blocks_per_sm(int dtype, int tile_bits);
/* Per-instance emusv_status (EMUSV_NOT_CONVERGED = RecursionError of that instance,
 * EMUSV_WORKSPACE_TOO_SMALL = basis_capacity too small) and the Krylov iteration count of
 * every step [ninst][max_steps] into host arrays; returns the worst status, or
 * EMUSV_TIMEOUT if a grid barrier gave up.  Synchronises the stream. */
int emusv_batch_results(int ninst, int max_steps, void *workspace, int *status_out,
                        int *iterations_out, void *stream);

/* ---- batched adjoint steps: DifferentiableStateVectorEvolution.backward
 * (emu_sv/time_evolution/torch.py:223-378, double_krylov.py:5-113) for every instance of a
 * batch in one persistent launch.  Prepared like a batch (all steps' pulses); each launch
 * takes step `step` of every instance: states (psi_step, packed) and grad_in (dL/dpsi
 * after the step, packed) in, grad_out (dL/dpsi before the step = exp(+i dt H) grad_in)
 * and grads_dev [ninst][3][20] (dL/dOmega_q, dL/ddelta_q, dL/dphi_q by qubit q; FP64,
 * device) out, plus an emusv status per instance in status_dev [ninst] (device).  The
 * interaction-matrix gradient is not formed here (emusv_adjoint_step has it).
 * Capturable: a launch issues two memsets and one cooperative kernel. */
size_t emusv_batch_adjoint_workspace_bytes(int ninst, const int *nqubits, const int *nsteps,
                                           int dtype, int tile_bits, int basis_capacity);
int emusv_batch_adjoint_prepare(int ninst, const int *nqubits, const int *nsteps, const double *dt,
                                int dtype, const double *omegas, const double *deltas,
                                const double *phis, const double *interactions, double tolerance,
                                int max_krylov_dim, int tile_bits, int basis_capacity,
                                void *workspace, size_t workspace_bytes, void *stream);
int emusv_batch_adjoint_launch(int dtype, int tile_bits, int blocks_per_sm, int step,
                               const void *states, const void *grad_in, void *grad_out,
                               double *grads_dev, int *status_dev, void *workspace, void *stream);
/* Krylov iteration counts of the last adjoint launch, [ninst][2] (state basis, gradient
 * basis), to a host array.  Synchronises the stream. */
int emusv_batch_adjoint_iterations(int ninst, void *workspace, int *iterations_out, void *stream);
/* Scheduling of a prepared forward batch workspace (no counterpart in the reference):
 * engine 0 (the default) runs every register's Lanczos iterations in lock-step rounds of
 * the whole batch, engine 1 lets each register run its own sequence of phases (norm,
 * H v, recurrence, ..., combination) with no grid barrier.  Results are the same; the
 * faster one depends on the batch (BatchEvolution's autotuner times both).  Host-side
 * only (takes effect at the next launch); EMUSV_BAD_ARGUMENT for an adjoint workspace. */
int emusv_batch_set_engine(void *workspace, int engine);
/* Failure-path test switch of a prepared batch workspace (forward or adjoint; no
 * counterpart in the reference, whose loop has no device-side waits): later launches wait
 * at most wait_cycles SM clock cycles at a grid barrier (<= 0 restores the default, about
 * 1 s), and with skip_first_arrival != 0 the last CTA does not arrive at each launch's
 * first barrier (lock-step rounds; with the phase engine, register 0's first phase is never
 * published), so every other CTA's bounded wait runs out, all CTAs return and
 * emusv_batch_results reports EMUSV_TIMEOUT; the device stays usable.  Off by default;
 * for tests.  Host-side only (takes effect at the next launch). */
int emusv_batch_set_barrier_test(void *workspace, long long wait_cycles, int skip_first_arrival);

/* ---- building blocks of the generic krylov_exp(op, v, ...) (krylov_exp.py:23-106) ----
 * For an arbitrary operator applied by the caller, these give the FP64-accumulated
 * Lanczos arithmetic and the on-device exponential of the extended Krylov matrix. */

/* res_dev[0..1] (device float64) = <a, b> = sum conj(a) b.  scratch: emusv_scratch_bytes. */
int emusv_vec_dot(int64_t len, int dtype, const void *a, const void *b, double *res_dev,
                  void *scratch, size_t scratch_bytes, void *stream);
/* y = y + alpha x  (alpha: host complex [2]) */
int emusv_vec_axpy(int64_t len, int dtype, const double *alpha, const void *x, void *y,
                   void *stream);
/* out = sum_k coef[k] V[k]; V = k vectors of `len` amplitudes back to back; coef_dev is a
 * device complex128 [k] array. */
int emusv_vec_combine(int64_t len, int dtype, int k, const double *coef_dev, const void *V,
                      void *out, void *stream);

/* x_dev = exp(A) e_0 (device complex128 [m]) for a complex tridiagonal m x m matrix given
 * by host complex arrays diag[m], upper[m] (upper[k] = A[k-1][k]) and lower[m]
 * (lower[k] = A[k+1][k]); FP64 Taylor series with scaling, on the device.  Replaces the
 * torch.linalg.matrix_exp of krylov_exp.py:66,78.  Synchronises the stream. */
/* x_dev (device complex128 [m]) = exp(A) e_0 for a dense complex m x m matrix A (host,
 * row-major, complex128 interleaved: a[2*(r*m + c)] real, +1 imaginary), m <= 102: the
 * matrix_exp(T)[:, 0] of the non-Hermitian (Arnoldi) krylov_exp_impl (krylov_exp.py:65,
 * 78), whose T is upper Hessenberg plus the extension entry.  EMUSV_NONFINITE when the
 * norm of A is not finite.  Synchronises the stream (the host matrix may be reused). */
size_t emusv_dense_expm_scratch_bytes(int m);
int emusv_dense_expm_col(int m, const double *a, double *x_dev, void *scratch, size_t scratch_bytes,
                         void *stream);
size_t emusv_tridiag_scratch_bytes(void);
int emusv_tridiag_expm_col(int m, const double *diag, const double *upper, const double *lower,
                           double *x_dev, void *scratch, size_t scratch_bytes, void *stream);

/* ---- launch accounting (no reference counterpart: measurement support) ----
 * emusv_profile_begin resets the per-kind launch counters; with event_timing != 0 every
 * later launch is bracketed by CUDA events on its stream.  emusv_profile_end waits for
 * those events and returns, per kind, the summed device milliseconds and the launch
 * count.  Kinds: 0 H*psi, 1 orthogonalisation/axpy/norm passes, 2 small FP64 kernels,
 * 3 basis combination, 4 observables, 5 adjoint contractions, 6 batched evolution. */
#define EMUSV_PROFILE_KINDS 8
void emusv_profile_begin(int event_timing);
int emusv_profile_end(double *ms_by_kind, long long *launches_by_kind, int nkinds);

#ifdef __cplusplus
}
#endif

#endif /* EMUSV_B200_H */
