/*
 * mpc_tdse.h -- C ABI of the B200 implementation of MP-CITDSE's `tdse`
 * propagation (libmpc_tdse.so).
 *
 * Everything is plain C: ints, doubles, host or device pointers and sizes.
 * Every function returns MPC_OK (0) or a negative MPC_ERR_* code; the text of
 * the last error on the calling thread is available from mpc_last_error().
 *
 * Array conventions are the reference's (citations are paths inside the
 * MP-CITDSE source tree):
 *   - state_sz[L], L = 0..L_max: states kept per angular-momentum block, as
 *     Propagator_Settings.states_in_l (src/tdse/td_read.cpp:17-26);
 *   - eig: the per-block eigenenergies concatenated (tdrd::readEnergies,
 *     src/tdse/td_read.cpp:50-86);
 *   - dip: the dipole blocks back to back, block L row-major
 *     [state_sz[L] x state_sz[L+1]] (tdrd::readDipoles,
 *     src/tdse/td_read.cpp:88-120);
 *   - a state (ct) is interleaved complex128: 2*sum(state_sz) doubles
 *     (state_type, src/tdse/tdse.cpp:3).
 *
 * A context owns its device copies, its CUDA stream and its work buffers.
 * Contexts are not thread-safe: use one per host thread.
 */
#ifndef MPC_TDSE_H_
#define MPC_TDSE_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPC_OK 0
#define MPC_ERR_ARG (-1)      /* invalid argument                          */
#define MPC_ERR_CUDA (-2)     /* a CUDA runtime call failed                */
#define MPC_ERR_DEVICE (-3)   /* a kernel reported a failure (status word) */
#define MPC_ERR_NOMEM (-4)    /* device allocation failed                  */
#define MPC_ERR_UNSTABLE (-5) /* dt outside the RKF78 stability interval   */

/* Field shapes: pulse::sineEE, sineAA, sineAE, sineEA and gauss
 * (src/tdse/pulse.cpp:34-97). */
#define MPC_FIELD_SINE_EE 0
#define MPC_FIELD_SINE_AA 1
#define MPC_FIELD_SINE_AE 2
#define MPC_FIELD_SINE_EA 3
#define MPC_FIELD_GAUSS 4

/* pulse::params (src/tdse/include/pulse.hpp:20-26) plus the field function
 * the reference's main binds to it (src/tdse/tdse_main.cpp:166-192). */
typedef struct mpc_pulse {
  int kind; /* MPC_FIELD_* */
  double Eo, w, cepd, a, b;
} mpc_pulse;

typedef struct mpc_ctx mpc_ctx;

/* Version of this ABI (major*10000 + minor*100 + patch). */
int mpc_version(void);

/* Copies the last error message of the calling thread into buf. */
int mpc_last_error(char *buf, size_t len);

/* Pulse set-up in atomic units, as pulse::sineESetup / sineASetup /
 * gaussESetup / gaussASetup (src/tdse/pulse.cpp:10-32,41-47,69-75):
 * shape 0 = sin^2 envelope, 1 = Gaussian; gauge 'l' gives an E-defined pulse
 * (sineEE / gauss), 'v' an A-defined one (sineAA / gauss). */
int mpc_pulse_setup(int shape, char gauge, double Io_au, double w_au, double cepd, int cycles,
                    double tau, mpc_pulse *out);

/* pulse::toAU (src/tdse/pulse.cpp:3-6), pulse::period (:8). */
int mpc_to_au(double Io_Wcm2, double w_eV, double *Io_au, double *w_au);
double mpc_period(double w_au, int cycles);

/* The field function bound to `p` at time t (src/tdse/pulse.cpp:34-97). */
double mpc_field(const mpc_pulse *p, double t);

/* Creates a context on CUDA device `device` holding H0 and the dipole
 * blocks.  Replaces the MatVecV / MatVecL set-up in tdse::propV / propL
 * (src/tdse/tdse.cpp:159-169): the blocks are copied to HBM once and stay
 * resident.  gauge: 'l' (MatVecL) or 'v' (MatVecV). */
int mpc_ctx_create(int L_max, const int *state_sz, const double *eig, const double *dip,
                   char gauge, int device, mpc_ctx **out);
int mpc_ctx_destroy(mpc_ctx *ctx);

/* Which kernels run mpc_propagate / mpc_advance:
 *   MPC_PATH_AUTO (0)      resident when the coupling fits in shared memory,
 *                          streaming otherwise (default);
 *   MPC_PATH_STREAMING (1) per-stage kernels streaming the dipole blocks
 *                          from HBM (any size);
 *   MPC_PATH_RESIDENT (2)  one persistent cooperative kernel per call, each
 *                          CTA holding its rows' coupling in shared memory
 *                          (MPC_ERR_ARG if the system does not fit).
 * Both give the same results within rounding (tested). */
#define MPC_PATH_AUTO 0
#define MPC_PATH_STREAMING 1
#define MPC_PATH_RESIDENT 2
int mpc_ctx_set_path(mpc_ctx *ctx, int path);
int mpc_ctx_get_path(mpc_ctx *ctx);   /* the path mpc_advance will take */

/* Failure detection (new: the reference has no device code to watch).  The
 * persistent cooperative kernels (the resident single-pulse propagation, its
 * adjoint sweep and the resident batched tail) meet at grid barriers whose
 * waits are bounded: a CTA that waits longer than this limit (default 2 s)
 * stops, every other CTA stops at its own bounded wait, the call returns
 * MPC_ERR_DEVICE ("wait timeout") and the context stays usable.  seconds in
 * [1e-6, 60].  The streaming kernel's TMA ring waits keep a fixed 2 s bound. */
int mpc_ctx_set_wait_limit(mpc_ctx *ctx, double seconds);

/* Fault injection for tests of the failure detection above: the next
 * persistent launch on this context gets grid-barrier targets one arrival
 * beyond what its CTAs can make, so its first barrier wait runs out after the
 * wait limit and the call reports the timeout.  Later launches are normal. */
int mpc_ctx_inject_barrier_timeout(mpc_ctx *ctx);

/* Total number of states sum(state_sz). */
int mpc_ctx_size(const mpc_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that record
 * events or order their own work after the library's. */
int mpc_ctx_stream(const mpc_ctx *ctx, void **stream);

/* One right-hand-side evaluation dxdt = f(x) at field value F:
 * MatVecV::operator() / MatVecL::operator() (src/tdse/tdse.cpp:14-73,
 * :85-143).  Host buffers of 2*size doubles. */
int mpc_rhs(mpc_ctx *ctx, double F, const double *x, double *dxdt);

/* One rkf.do_step(sys, x, t, dt) with the field frozen at F
 * (src/tdse/tdse.cpp:190): 13 stages, 8th-order solution, no
 * renormalisation.  x: host, in/out. */
int mpc_rk78_step(mpc_ctx *ctx, double F, double dt, double *x);

/* The propagation loop of tdse::propV / tdse::propL
 * (src/tdse/tdse.cpp:186-215): for each of `steps` steps, F = field(t+dt)
 * frozen for the step, one RKF78 step, t += dt, ct /= ||ct||_2.
 * ct: host, in/out.  Optional host outputs (NULL to skip):
 *   pop_out[steps+1]   |ct[pop_index]|^2 at t0 and after every step
 *                      (the reference's _pop<n><l>.dat column);
 *   field_out[steps]   the field used by each step (_field.dat column);
 *   norm_out[steps]    ||ct|| before each renormalisation (norm drift).
 * Returns MPC_ERR_UNSTABLE if dt*max|E| lies outside the RKF78
 * imaginary-axis stability interval (the field coupling widens the spectrum
 * further; keeping dt inside the interval for H0 + F*D is the caller's job,
 * as it is in the reference, whose states_in_l truncation serves it). */
int mpc_propagate(mpc_ctx *ctx, const mpc_pulse *pulse, double t0, double dt, int steps,
                  int pop_index, double *ct, double *pop_out, double *field_out,
                  double *norm_out);

/* Device-resident form of mpc_propagate: the state stays in the context.
 * mpc_state_set / mpc_state_get copy it in / out (host buffers);
 * mpc_advance runs the loop on the resident state without host copies
 * (history outputs stay on the device and can be fetched with
 * mpc_history_get). */
int mpc_state_set(mpc_ctx *ctx, const double *ct);
int mpc_state_get(mpc_ctx *ctx, double *ct);
int mpc_advance(mpc_ctx *ctx, const mpc_pulse *pulse, double t0, double dt, int steps,
                int pop_index);
int mpc_history_get(mpc_ctx *ctx, int steps, double *pop_out, double *field_out,
                    double *norm_out);

/* Batched right-hand side (new: the reference evaluates one state at a
 * time): B states x [B][2*size] (host, each state contiguous) at fields
 * F[B]; dxdt [B][2*size].  The coupling is applied as one FP64 tensor-core
 * GEMM over all B states. */
int mpc_batch_rhs(mpc_ctx *ctx, int B, const double *F, const double *x, double *dxdt);

/* Batched adaptive RKF78 (new: the reference propagates one pulse per run,
 * with a fixed step).  B pulses, each with its own field (pulses[b]), start
 * time t0[b] and end time t_end[b], advance together on the GPU; each has
 * its own step size and accept/reject history:
 *   stage fields F_b(t + c_s h) (continuous field), 8th-order solution,
 *   embedded 7th-order error e, err = max_i |e_i| / (atol + rtol *
 *   max(|x_i|, |x_new_i|)), accept if err <= 1, then x = x_new / ||x_new||;
 *   next h = h * clamp(0.9 * err^(-1/8), 0.2, 5) (at most 1 after a
 *   rejection), capped at dt_max and at t_end - t.
 * ct: host [B][2*size] in/out.  accepted / rejected / t_final (host arrays of
 * B, optional) receive each pulse's accepted and rejected step counts and
 * end time.  max_attempts (<= 0: unlimited) bounds the attempts per pulse;
 * a pulse that hits it stops and the call returns MPC_ERR_DEVICE. */
int mpc_batch_propagate(mpc_ctx *ctx, int B, const mpc_pulse *pulses, const double *t0,
                        const double *t_end, double h0, double dt_max, double rtol, double atol,
                        int max_attempts, double *ct, int *accepted, int *rejected,
                        double *t_final);

/* Batched fixed-step propagation with the reference's semantics (new: the
 * reference runs one pulse per process).  B pulses advance together, each
 * exactly as mpc_propagate -- the loop of tdse::propV / propL,
 * src/tdse/tdse.cpp:186-215 -- would advance it alone: per step the field
 * F_b(t_b + dt) is frozen for the 13 stages, one RKF78 step (8th-order
 * solution), t_b += dt, c_b /= ||c_b||.  Pulse b runs steps[b] steps from
 * t0[b]; a pulse that has finished retires and the batch narrows (each stage
 * is one FP64 tensor-core GEMM over the active pulses; the last few pulses
 * finish in the persistent resident kernel when the coupling fits on chip).
 * ct: host [B][2*size] in/out.  Optional host outputs (NULL to skip), with
 * M = max(steps):
 *   pop_out [B][M+1]   |c_b[pop_index]|^2 at t0[b] and after every step
 *                      (the _pop column; entries past steps[b] are unset);
 *   norm_out [B][M]    ||c_b|| before each renormalisation.
 * Returns MPC_ERR_DEVICE (non-finite norm) if a pulse's norm stops being
 * finite, MPC_ERR_UNSTABLE as mpc_propagate does. */
int mpc_batch_advance(mpc_ctx *ctx, int B, const mpc_pulse *pulses, const double *t0, double dt,
                      const int *steps, int pop_index, double *ct, double *pop_out,
                      double *norm_out);

/* Single-pulse adaptive RKF78 (new: the reference steps with a fixed dt):
 * mpc_batch_propagate with B = 1 and the pulse's own t0, t_end; ct: host
 * [2*size] in/out; accepted / rejected / t_final (optional) are scalars. */
int mpc_propagate_adaptive(mpc_ctx *ctx, const mpc_pulse *pulse, double t0, double t_end,
                           double h0, double dt_max, double rtol, double atol, int max_attempts,
                           double *ct, int *accepted, int *rejected, double *t_final);

/* The batched adaptive propagation under the name of the propagate family;
 * arguments and results exactly as mpc_batch_propagate. */
int mpc_propagate_batch(mpc_ctx *ctx, int B, const mpc_pulse *pulses, const double *t0,
                        const double *t_end, double h0, double dt_max, double rtol, double atol,
                        int max_attempts, double *ct, int *accepted, int *rejected,
                        double *t_final);

/* Tile autotuner of the batched path (new).  Times each tile variant of the
 * batched right-hand side GEMM (pulse-column tile width x cp.async pipeline
 * depth x k split) on this context's system at widths 1, 2, 4, ... up to B pulses and
 * keeps the fastest per width for the context's later batched calls
 * (mpc_batch_propagate runs it on first use; every variant sums in the same
 * order, so the choice never changes results).  If table is non-null it
 * receives up to cap rows of 5 doubles: pulses, tile width (real columns),
 * pipeline depth, k split (1: the two coupled blocks of a tile run in two
 * CTAs), microseconds per right-hand side of the chosen variant.
 * Returns the number of rows (>= 0) or an error code. */
int mpc_batch_autotune(mpc_ctx *ctx, int B, double *table, int cap);

/* How the batched fixed step (mpc_batch_advance) ran at each width: on its
 * first use the library times, at widths 1, 2, 4, ... pulses, a whole step
 * as one launch per Horner product on each cp.async-fed tile variant, as one
 * persistent launch on each unsplit tile shape, and as one TMA-fed launch per
 * product on each TMA tile shape, and keeps the fastest (every choice gives
 * the same bits).  Rows of 5 doubles, up to cap: pulses, kind (0 one
 * cp.async-fed launch per product, 1 persistent, 2 one TMA-fed launch per
 * product, 3 one cp.async-fed launch per product with each tile's two
 * coupled blocks in two CTAs), tile width (real columns), ring depth,
 * microseconds per step.  Returns the number of rows (0 before any
 * fixed-step call). */
int mpc_batch_fixed_plan(mpc_ctx *ctx, double *table, int cap);

/* Objective and gradient (new: the reference has no gradients).
 *
 * The field of the fixed-step propagation (mpc_propagate semantics: F frozen
 * at t+dt per step, renormalisation after every step) is the pulse plus a
 * piecewise-cubic perturbation dE(t) = sum_k u[k] phi((t - t_k)/g),
 * t_k = k*T/(K-1), phi the Catmull-Rom (Keys a = -1/2) cubic kernel, zero
 * outside [0, T].  J = 1 - sum_{eig < thr} |c_i(t_N)|^2 (the yield above the
 * threshold thr, 0 unless mpc_objective_threshold set it: ionisation for 1e;
 * for 2e CI energies measured from the doubly-charged ion, double
 * ionisation, and thr = -Z^2/2 gives single ionisation) for target < 0, else
 * |c_target(t_N)|^2.  The final state has unit norm, so the yield is
 * evaluated as sum_{eig >= thr} |c_i|^2 (no cancellation for small yields).
 *
 * mpc_objective runs the forward pass from ct0 (host) and keeps a state every
 * ckpt_every steps (<= 0: 64); mpc_objective_backward then returns dJ/du
 * (grad_u[K]) and dJ/dF_n per step (dJdF[steps]), either may be NULL, by the
 * discrete adjoint: each checkpoint segment is recomputed and walked back
 * through the transposed RKF78 stages (about 3 forward passes in all).
 * mpc_objective_gradient does both. */
int mpc_objective_threshold(mpc_ctx *ctx, double thr);
int mpc_objective(mpc_ctx *ctx, const mpc_pulse *pulse, int K, const double *u, double T,
                  double t0, double dt, int steps, int target, int ckpt_every, const double *ct0,
                  double *J);
int mpc_objective_backward(mpc_ctx *ctx, double *grad_u, double *dJdF);
int mpc_objective_gradient(mpc_ctx *ctx, const mpc_pulse *pulse, int K, const double *u,
                           double T, double t0, double dt, int steps, int target, int ckpt_every,
                           const double *ct0, double *J, double *grad_u, double *dJdF);

/* One call from controls to gradient: exactly mpc_objective_gradient
 * (objective J, dJ/du and dJ/dF_n of one pulse by the checkpointed discrete
 * adjoint). */
int mpc_adjoint(mpc_ctx *ctx, const mpc_pulse *pulse, int K, const double *u, double T,
                double t0, double dt, int steps, int target, int ckpt_every, const double *ct0,
                double *J, double *grad_u, double *dJdF);

/* Batched objective and gradient (new).  B pulses at once with the semantics
 * of mpc_objective / mpc_objective_backward per pulse: pulse b has its own
 * field pulses[b], K controls u[b*K .. b*K+K) on its own window [0, T[b]]
 * (u and T may be NULL when K == 0), and all share t0, dt, steps, target,
 * the yield threshold and ckpt_every.  ct0: host [B][2*size]; J: host [B].
 * The forward and the adjoint stages run as FP64 tensor-core GEMMs over all
 * pulses (the couplings are read once per stage for the whole batch).
 * mpc_batch_objective_backward returns grad_u [B][K] and dJdF [B][steps]
 * (either may be NULL) for the last mpc_batch_objective call.  Device memory:
 * about (steps/ckpt_every + 13*ckpt_every + 20) x size x 16 x ceil32(B) bytes;
 * ckpt_every <= 0 picks the longest interval that fits in 85 % of the free
 * device memory (every step kept, no recomputation, when that fits).  The
 * forward keeps its last segment, which the backward pass then does not
 * recompute. */
int mpc_batch_objective(mpc_ctx *ctx, int B, const mpc_pulse *pulses, int K, const double *u,
                        const double *T, double t0, double dt, int steps, int target,
                        int ckpt_every, const double *ct0, double *J);
int mpc_batch_objective_backward(mpc_ctx *ctx, double *grad_u, double *dJdF);
/* The checkpoint interval and segment count the last mpc_batch_objective
 * used (chosen there when its ckpt_every was <= 0) and the device bytes of its
 * buffers; any output may be NULL. */
int mpc_batch_objective_info(mpc_ctx *ctx, int *ckpt_every, int *segments, double *device_bytes);
int mpc_batch_objective_gradient(mpc_ctx *ctx, int B, const mpc_pulse *pulses, int K,
                                 const double *u, const double *T, double t0, double dt,
                                 int steps, int target, int ckpt_every, const double *ct0,
                                 double *J, double *grad_u, double *dJdF);

/* Photoelectron spectrum and populations of the context's current state
 * (after mpc_propagate / mpc_advance), or of ct (host, 2*size doubles) when
 * non-NULL: pes::genPES1e / genPES2e (src/pes/pes.cpp:48-262) without their
 * text round trip.  electrons 1: spectrum of each block l binned onto the
 * l = 1 energies (grid slot k holds bin k, 1 <= k <= state_sz[0]-2);
 * electrons 2: per-state densities at E_i - threshold (threshold = the
 * lowest 1e energy of l = 0, as the reference reads it), slot i of block L.
 * pes: host [(L_max+1) x ngrid], ngrid >= the largest block; stats: host
 * [4] = ground-state population, norm, yield, excited population (2e). */
int mpc_pes(mpc_ctx *ctx, int electrons, double threshold, const double *ct, double *pes,
            int ngrid, double *stats);

/* The summed spectrum of `pes -s` for the same state (src/pes/pes.cpp
 * :127-137, :215-245): 1e, the blocks' binned spectra added per bin; 2e,
 * every state i >= 1 of every block binned onto the L = 1 energies (first
 * matching bin 1 <= k <= n_1 - 1, the bin's upper neighbour for k = n_1 - 1
 * being the first L = 2 energy, as the reference indexes it; bins stop at
 * n_1 - 2 when L_max = 1), density |c_i|^2 * 2 / (dn + dp).  grid[k]
 * receives E1[k] (1e) or E1[k] - threshold (2e) and pes[k] the density,
 * k < n_1 = state_sz[1]; ngrid >= n_1 (entries past n_1 are zeroed).  The
 * reference writes the rows k <= n_1 - 2 (1e: n_0 - 2) with grid[k] > 0.
 * The reference sizes its accumulator by state_sz[L_max] and reads one
 * energy past block 1; here the bins have their own array of n_1. */
int mpc_pes_summed(mpc_ctx *ctx, int electrons, double threshold, const double *ct, double *grid,
                   double *pes, int ngrid);

/* Measures the FP64 tensor-core (mma.sync .f64) and FP64 FMA throughput of
 * CUDA device `device` in TFLOP/s: the roofline denominators of the batched
 * GEMM.  Takes ~50 ms. */
int mpc_probe_fp64_peak(int device, double *dmma_tflops, double *dfma_tflops);

/* Kernel timing (profiling aid).  While enabled, CUDA events on the
 * context's stream bracket every launch of each kernel kind:
 *   MPC_KERNEL_RHS_STREAM (0)  the dipole-block streaming pass,
 *   MPC_KERNEL_COMBINE (1)     the per-stage epilogue,
 *   MPC_KERNEL_RENORM (2)      the per-step renormalisation.
 * mpc_profile_read returns the summed device milliseconds and the number of
 * launches of one kind since the last read (and resets that kind). */
#define MPC_KERNEL_RHS_STREAM 0
#define MPC_KERNEL_COMBINE 1
#define MPC_KERNEL_RENORM 2
#define MPC_KERNEL_BATCH_STAGE 3   /* the batched GEMM + RK epilogue */
#define MPC_KERNEL_BATCH_OTHER 4   /* batched control, apply, compaction */
#define MPC_KERNEL_RESIDENT 5      /* the resident single-pulse propagation */
int mpc_profile_enable(mpc_ctx *ctx, int on);
int mpc_profile_read(mpc_ctx *ctx, int kind, double *total_ms, long long *launches);

/* Number of kernel launches the library issued on this context since it was
 * created (all kinds). */
long long mpc_launch_count(const mpc_ctx *ctx);

/* Right-hand side without any allocation.  No counterpart in the reference
 * (it has no GPU path).
 *
 * For callers that cannot allocate device memory: a host framework whose
 * caching allocator owns the device (a raw cudaMalloc can fail or fragment
 * its pool), a plugin inside a simulation code that forbids allocation after
 * start-up, a time-critical loop that cannot afford cudaMalloc/cudaFree and
 * their implicit synchronisation.  Computes dxdt = f(x) at field F -- the
 * same result as mpc_rhs -- on caller-owned DEVICE buffers of the current
 * CUDA device: d_eig [sum(state_sz)], d_dip (blocks back to back, block L
 * row-major [state_sz[L] x state_sz[L+1]]), d_x and d_dxdt [2*sum(state_sz)]
 * doubles.  state_sz is a host array.  Runs asynchronously on `stream`
 * (a cudaStream_t; NULL = the legacy default stream).  d_x and d_dxdt must be
 * 16-byte aligned (they are read and written as complex pairs) and d_eig and
 * d_dip 8-byte aligned; a misaligned view (say, a slice starting one double
 * in) is refused with MPC_ERR_ARG before anything is launched.
 *
 * Its scratch is a static device array of MPC_NOALLOC_SCRATCH_BYTES (16 MiB)
 * that every GPU loading the library holds until the process exits.  Systems
 * needing more -- 16 B x (sum over dipole blocks of ceil(n_{L+1}/256) x n_L
 * + 256 per column-partial slot) -- or more than 256 column strips are
 * rejected with MPC_ERR_ARG.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture begins.  The address is cached per CUDA context: after
 * cudaDeviceReset, or with another context current, the next call looks it up
 * again (so that call, too, should come before any capture).  All calls share the array and it keeps the
 * last call's contents: calls whose kernels overlap on the GPU race, so
 * serialise them.  No cudaMalloc, cudaFree or host heap allocation. */
#define MPC_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int mpc_rhs_noalloc(int L_max, const int *state_sz, const double *d_eig, const double *d_dip,
                    char gauge, double F, const double *d_x, double *d_dxdt, void *stream);

/* Waits for the context's stream and returns any kernel-reported failure
 * (MPC_ERR_DEVICE) or CUDA error. */
int mpc_sync(mpc_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
