/*
 * stratiflow_b200 — C-ABI of the B200 IMEX-RK time-step engine.
 *
 * The reference (jeremypparker/Stratiflow) has no FFI: its hot path is the
 * C++ class IMEXRK (IMEXRK.h:31-670), held as the static StateVector::solver
 * (StateVector.h:546) and driven by StateVector::FullEvolve / FixedEvolve /
 * LinearEvolve (StateVector.cpp:3-156). Each entry point below replaces one
 * member of that surface; the comment on each names the member it replaces.
 *
 * Conventions
 *   - Every function returns 0 on success and a negative SF_E* code on
 *     failure; sf_last_error() then returns a message (thread-local). No C++
 *     exception crosses this boundary.
 *   - A solver owns one CUDA stream on one device and all its device memory.
 *     Calls on one solver must come from one host thread at a time.
 *   - Grid sizes are runtime values (the reference fixes them at compile time,
 *     Parameters.h:42-43). N1 and N2 are powers of two, 16 <= N1 <= 512,
 *     N2 == 1 (2D) or 16 <= N2 <= 256 (3D); N3 % 4 == 0, 16 <= N3 <= 1024.
 *   - A solver advances `nrun` independent runs of the same grid together
 *     (ensemble members, Krylov directions); each run has its own Ri,
 *     background profile and state.
 *   - Field data in the reference layout is std::complex<float> interleaved,
 *     z fastest: index (M1*n2 + n1)*N3 + n3 with M1 = N1/2+1 (Field.h:399,410),
 *     i.e. exactly ModalField::Raw(). Only the kept (2/3-dealiased) modes are
 *     stored on the device; set_field ignores the others and get_field writes
 *     them as zero (the state the reference's FilterAll leaves them in).
 *   - The compact device layout ("kept layout") is complex<float>
 *     [N3][plane], plane = roundup(K1*K2, 16), mode index m = q*K1 + j1,
 *     K1 = N1/3 x-modes, K2 = 1 (2D) or 2*(N2/3)-1 y-modes in the order
 *     ky = 0..N2/3-1, -(N2/3-1)..-1.
 */
#ifndef STRATIFLOW_B200_H
#define STRATIFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SF_OK 0
#define SF_EINVAL (-1)   /* bad argument or grid */
#define SF_ECUDA (-2)    /* CUDA runtime error */
#define SF_ENOMEM (-3)   /* device allocation failed */
#define SF_ESTATE (-4)   /* call out of order (e.g. linear step without base) */

/* field selectors: IMEXRK public members u1,u2,u3,b,p (IMEXRK.h:605-606) */
#define SF_U1 0
#define SF_U2 1
#define SF_U3 2
#define SF_B 3
#define SF_P 4

typedef struct sf_solver sf_solver;

/* gridParams (Parameters.h:6-18, 42-43) plus the batch size */
typedef struct {
  int N1, N2, N3;
  int nrun;
} sf_grid;

/* flowParams (Parameters.h:20-30, Parameters.cpp:5-6); Ri is set per run */
typedef struct {
  double L1, L2, L3, Re, Pr;
} sf_flow;

/* IMEXRK::IMEXRK (IMEXRK.h:37-81): builds the Laplacian factors and, via
 * UpdateForTimestep, the Crank-Nicolson factors for deltaT = dt. All runs
 * start with Ri = 0, a zero background and a zero state. */
int sf_create(const sf_grid* grid, const sf_flow* flow, double dt, int device, sf_solver** out);

/* releases the device memory, graphs and stream */
int sf_destroy(sf_solver* s);

/* message of the last failing call on this host thread */
const char* sf_last_error(void);

/* IMEXRK::deltaT + UpdateForTimestep (IMEXRK.h:502-545): re-factorises the
 * tridiagonal systems in FP64 on the device */
int sf_set_dt(sf_solver* s, double dt);

/* flowParams.Ri for one run (enters BuildRHS only, IMEXRK.cpp:143) */
int sf_set_ri(sf_solver* s, int run, double Ri);

/* IMEXRK::SetBackground(Neumann1D) (IMEXRK.h:321-332): U_[N3] at the
 * Neumann levels, plus the background stratification dB/dz[N3] at the same
 * levels, which generalises the dB/dz = 1 hard-wired in BuildRHS
 * (IMEXRK.cpp:145-147; pass all ones for the reference's behaviour). */
int sf_set_background(sf_solver* s, int run, const double* U, const double* dBdz);

/* assignment to solver.u1/u2/u3/b/p (StateVector::CopyToSolver,
 * StateVector.h:511-525) from host memory in the reference layout */
int sf_set_field(sf_solver* s, int run, int field, const float* ref_layout);

/* StateVector::CopyFromSolver (StateVector.h:532-543) into host memory in
 * the reference layout */
int sf_get_field(sf_solver* s, int run, int field, float* ref_layout);

/* whole state (u1,u2,u3,b,p) of every run, host <-> device, in the kept
 * layout, one contiguous buffer [nrun][5][N3][plane] of complex<float> */
int sf_set_state_kept(sf_solver* s, const float* host);
int sf_get_state_kept(sf_solver* s, float* host);

/* CopyToSolver, nsteps x TimeStep, CopyFromSolver (StateVector.h:511-543 around
 * IMEXRK::TimeStep, IMEXRK.cpp:5-24) for a stream of independent states held in
 * host memory: enqueues the copy of host_in (all runs, kept layout) to the
 * device, the steps, and the copy of the result to host_out, and returns.
 * Consecutive calls overlap: the input copy of call k+1 and the output copy of
 * call k-1 run on their own streams while call k steps (two device staging
 * buffers per direction). host_in must stay unchanged and host_out unread until
 * sf_synchronize; pinned host memory makes the copies asynchronous. */
int sf_step_host_async(sf_solver* s, const float* host_in, float* host_out, int nsteps);

/* device pointer of the current state in the kept layout (valid until the
 * next step call), and its size in bytes */
int sf_state_device(sf_solver* s, void** dptr, size_t* bytes);
/* copy a device buffer in the kept layout into the current state */
int sf_set_state_device(sf_solver* s, const void* dptr);

/* StateVector::FixedEvolve's set-up (StateVector.cpp:94-97): FilterAll,
 * PopulateNodalVariables, RemoveDivergence(0) for every run */
int sf_prepare(sf_solver* s);

/* IMEXRK::RemoveDivergence(pressureMultiplier) (IMEXRK.cpp:43-73) */
int sf_remove_divergence(sf_solver* s, double pressure_multiplier);

/* nsteps x IMEXRK::TimeStep (IMEXRK.cpp:8-24) for every run; replays a
 * captured CUDA graph of one step; asynchronous on the solver's stream */
int sf_step(sf_solver* s, int nsteps);

/* IMEXRK::SetBackground(u1,u2,u3,b) (IMEXRK.h:334-352): the frozen base state
 * of TimeStepLinear for one run, modal, reference layout */
int sf_set_base(sf_solver* s, int run, const float* u1, const float* u2, const float* u3,
                const float* b);
/* SetBackground(u1,u2,u3,b) from a state already on the device in the kept
 * layout [5][N3][plane] (e.g. an sf_vecs vector); synchronises */
int sf_set_base_device(sf_solver* s, int run, const void* kept_state);

/* nsteps x IMEXRK::TimeStepLinear (IMEXRK.cpp:26-41) */
int sf_step_linear(sf_solver* s, int nsteps);

/* IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126, BuildRHSAdjoint IMEXRK.cpp:260-379,
 * the mixing objective of UpdateAdjointVariables IMEXRK.h:461-500): one step of
 * every run's adjoint state backwards, given the direct state at the step's
 * two ends as device arrays of nrun states in the kept layout [5][N3][plane]
 * (below = the earlier time, above = the later; u1, u2, u3, b are read). */
int sf_step_adjoint(sf_solver* s, const void* below, const void* above);

/* Tangent-linear batch (no counterpart in the reference, whose
 * TimeStepLinear keeps its base frozen, IMEXRK.h:334-352): with nbase > 0,
 * sf_step advances runs 0..nbase-1 by TimeStep and every run r >= nbase by
 * TimeStepLinear about the live state of run (r - nbase) % nbase at the same
 * RK stage, i.e. the exact derivative of the discrete step map applied to the
 * perturbation in run r. nbase must divide nrun; 0 switches it off. */
int sf_set_tangent(sf_solver* s, int nbase);

/* Nodal fields of one run's state in the reference's nodal layout
 * (N1*n2 + n1)*N3 + n3, float (Field.h:399-410), field SF_U1..SF_B:
 * sf_get_nodal is PopulateNodalVariables of that field (IMEXRK.h:141-162);
 * sf_set_nodal is ToModal with its 1/(N1 N2) and Filter (Field.h:734-769)
 * into the state. Both synchronise. They read and write .fields files
 * (IMEXRK::SaveFlow / LoadFlow, IMEXRK.h:415-443). */
int sf_get_nodal(sf_solver* s, int run, int field, float* host);
int sf_set_nodal(sf_solver* s, int run, int field, const float* host);

/* The maxima over the nodal grid of |U1 + U_|, |U2|, |U3| of one run's state:
 * the inputs of IMEXRK::CFL (IMEXRK.h:355-373); synchronises */
int sf_velocity_maxima(sf_solver* s, int run, double* out3);

/* IMEXRK::CFL's number (IMEXRK.h:355-366) for one run at the current dt
 * (without the reference's update of dt, which FullEvolve does); and the dt */
int sf_cfl(sf_solver* s, int run, double* cfl);
int sf_get_dt(sf_solver* s, double* dt);
/* the number of runs of the solver's batch */
int sf_get_runs(sf_solver* s, int* nrun);

/* Launch tuning of the x pass (no counterpart in the reference): the number
 * of consecutive z-slabs one block walks through (0: chosen from the grid
 * size). The results do not depend on it. */
int sf_set_xpass_slabs(sf_solver* s, int slabs);

/* Launch tuning of the 3D x-y pass (no counterpart in the reference): the
 * number of level bands (1..8) whose y transforms run on side streams beside
 * the x passes of the neighbouring bands; 1 runs the three kernels one after
 * the other over all levels. The results do not depend on it. */
int sf_set_xy_bands(sf_solver* s, int bands);

/* Launch tuning of the z solves (no counterpart in the reference): the
 * warps per block of the z solves, 8 or 16 (0: 16 when one block per group
 * of 16 modes leaves SMs idle, else 8). Each warp takes one z-chunk of every
 * Thomas system in z kernels 0 and 1 (sf_set_z_kernel) and two in the
 * default kernel 2, which needs N3 >= 64 for 16 warps (else it takes 8). The
 * results depend on it only through rounding (the chunked solve
 * reassociates the recurrence). */
int sf_set_z_chunks(sf_solver* s, int chunks);

/* Launch tuning of the z pass (no counterpart in the reference): kind 2 (the
 * default) runs it as k_z_step_c, one lane per complex mode in paired FP32
 * instructions and two z-chunks per warp (16 chunks per block; grids with
 * N3 >= 32, else kind 0 runs); kind 0 as k_z_step, one lane per real
 * component and one chunk per warp; kind 1 as k_z_step_tma, k_z_step with
 * each warp's first-sweep inputs brought into shared memory by
 * tensor-memory-accelerator copies and the Thomas intermediates in tensor
 * memory (with 8 z chunks; a wait for its tiles that runs out is reported by
 * sf_synchronize). The three solve the same systems with the same terms; the
 * results differ by rounding (the chunk count reassociates the recurrences). */
int sf_set_z_kernel(sf_solver* s, int kind);

/* Launch tuning of the x pass (no counterpart in the reference): lane groups
 * (one transform at a time each) per block, 1..32 (0: enough for one slab's
 * inverse transforms in one round). More groups keep more warps resident;
 * groups without a task in a round idle through it. Results do not depend
 * on it. */
int sf_set_xpass_groups(sf_solver* s, int groups);

/* Launch tuning of the 3D nonlinear x pass (no counterpart in the reference):
 * kind 1 (the default) runs it as lane groups that each own a y row and
 * march up a range of levels, transforming two fields or products per packed
 * FP32 instruction; kind 0 as blocks over slabs of levels (the kernel that
 * every other x pass uses). The results agree to rounding (the z stencils'
 * terms are summed in another order). Grids with N1 other than 64, 128 or 256
 * always take kind 0. */
int sf_set_xpass_kernel(sf_solver* s, int kind);

/* IMEXRK::KE / PE (IMEXRK.h:395-411) of one run, accumulated in FP64 */
int sf_energy(sf_solver* s, int run, double* ke, double* pe);

/* Dissipation rates of one run in the normalisation of IMEXRK::KE / PE
 * (IMEXRK.h:395-411), FP64 accumulation. The reference has no such
 * diagnostic; these are the sinks of KE and PE due to the viscous and
 * diffusive terms of its CrankNicolson (IMEXRK.cpp:75-105):
 *   eps = (1/Re) sum_i InnerProd(grad u_i, grad u_i)
 *   chi = Ri/(Re Pr) InnerProd(grad b, grad b)
 * with the Fourier multipliers for ddx, ddy and the staggered ddz of
 * Differentiation.cpp:35-61, each component integrated (Integration.h:5-35)
 * on the levels where it lives. */
int sf_dissipation(sf_solver* s, int run, double* eps, double* chi);

/* StateVector::Dot (StateVector.h:122-134) between run a of solver sa and
 * run b of solver sb (same grid), FP64 accumulation; Ri of run a weights b */
int sf_dot(sf_solver* sa, int run_a, sf_solver* sb, int run_b, double* out);

/* Per-kernel timing of one step (no counterpart in the reference, which has
 * no timers): runs nsteps steps eagerly (not from the graph) with CUDA events
 * between kernel launches and writes the average milliseconds of each kernel
 * slot of one step into ms[0..*nslots); the state advances as by sf_step /
 * sf_step_linear (linear != 0). Slot order is that of sf_profile_names. */
int sf_profile_step(sf_solver* s, int nsteps, int linear, int cap, double* ms, int* nslots);

/* comma-separated kernel names of the profile slots */
int sf_profile_names(sf_solver* s, char* buf, size_t len);

/* RemoveDivergence(pressure_multiplier) for callers that cannot allocate
 * device memory (no counterpart in the reference). It projects one run's
 * fields that the caller owns on the device, in the kept layout
 * [N3][plane]: u1, u2 (3D only; may be NULL in 2D) and u3 are updated in
 * place, p_out = p_in + pressure_multiplier * q (p_out may equal p_in).
 * It calls no allocator: its working memory is a fixed 2 MiB device array
 * inside this library, which limits it to N3 * plane <= 131072 and
 * N3 <= 1024, plane = roundup(K1*K2, 16) (256 x 1 x 1024, 512 x 1 x 744 and
 * 64 x 32 x 320 fit; larger grids return SF_EINVAL). The first call on a device
 * looks that array up (cudaGetSymbolAddress), so make it before any stream
 * capture. Work is queued on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and the call returns without waiting. All calls share the array:
 * calls whose GPU work overlaps race and must be serialised by the caller. */
int sf_remove_divergence_noalloc(const sf_grid* grid, const sf_flow* flow, double pressure_multiplier,
                                 void* u1, void* u2, void* u3, const void* p_in, void* p_out,
                                 void* stream);

/* ---- ensembles of 2D runs on different grids (no counterpart in the
 * reference, whose grid is a compile-time constant, Parameters.h:42-43, held
 * by one static solver, StateVector.h:546) ----
 * nrun independent 2D runs, run r on grids[r] (N2 = 1; the nrun field is
 * ignored) with flows[r] and time step dt[r]. Each run is a member solver
 * (sf_ensemble_member) that takes every single-solver call: sf_set_ri,
 * sf_set_background, sf_set_field / sf_get_field, sf_prepare, sf_energy, ...
 * sf_ensemble_step advances every member by nsteps IMEXRK::TimeStep
 * (IMEXRK.cpp:8-24) with one launch per RK stage over all members' x-pass
 * and z-solve work items (one CUDA graph per step); it waits for the
 * members' own queued work first and returns without waiting for the steps:
 * call sf_ensemble_synchronize before using a member again. Members must not
 * be stepped on their own in between (sf_ensemble_step then reports
 * SF_ESTATE if their state parities differ). The member handles belong to
 * the ensemble: sf_ensemble_destroy frees them. */
typedef struct sf_ensemble sf_ensemble;
int sf_ensemble_create(int nrun, const sf_grid* grids, const sf_flow* flows, const double* dt, int device,
                       sf_ensemble** out);
int sf_ensemble_destroy(sf_ensemble* e);
int sf_ensemble_member(sf_ensemble* e, int run, sf_solver** s);
int sf_ensemble_step(sf_ensemble* e, int nsteps);
int sf_ensemble_synchronize(sf_ensemble* e);
int sf_ensemble_launch_count(sf_ensemble* e, long long* count);
int sf_ensemble_stream(sf_ensemble* e, void** stream);
/* nsteps steps run eagerly with CUDA events around every launch: the average
 * milliseconds of one x-pass launch and of one z-solve launch (all members) */
int sf_ensemble_profile(sf_ensemble* e, int nsteps, double* ms_x, double* ms_z);

/* ---- device state vectors (StateVector algebra, StateVector.h:40-149) ----
 * A store holds nvec states of one grid on the device, each in the kept
 * layout [5][N3][plane] (u1,u2,u3,b,p), and shares the stream of the solver
 * it was created from. Reductions accumulate in FP64. These are the Krylov
 * bases and iterates of the Newton-Krylov, Arnoldi and continuation drivers,
 * which in the reference are host std::vector<StateVector> (NewtonKrylov.h:239).
 * Once the solver is destroyed, sf_vecs_destroy is the only valid call on
 * its stores. */
typedef struct sf_vecs sf_vecs;
int sf_vecs_create(sf_solver* like, int nvec, sf_vecs** out);
int sf_vecs_destroy(sf_vecs* v);
int sf_vecs_count(sf_vecs* v, int* n);
/* device address of vector i */
int sf_vecs_device(sf_vecs* v, int i, void** ptr);
/* CopyFromSolver / CopyToSolver (StateVector.h:511-543): runs
 * run..run+count-1 <-> vectors i..i+count-1 */
int sf_vecs_from_run(sf_vecs* v, int i, sf_solver* s, int run, int count);
int sf_vecs_to_run(sf_vecs* v, int i, sf_solver* s, int run, int count);
int sf_vecs_copy(sf_vecs* v, int dst, sf_vecs* w, int src);
int sf_vecs_set_host(sf_vecs* v, int i, const float* host);
int sf_vecs_get_host(sf_vecs* v, int i, float* host);
/* Range operations act on `count` consecutive vectors in one launch.
 * StateVector::MulAdd (StateVector.h:67-78): v[y+k] += alpha * w[x+k], u1..b */
int sf_vecs_axpy(sf_vecs* v, int y, double alpha, sf_vecs* w, int x, int count);
/* v[y+k] = a v[y+k] + b w[x+k] on all five fields */
int sf_vecs_lincomb(sf_vecs* v, int y, double a, double b, sf_vecs* w, int x, int count);
/* StateVector::operator*= (StateVector.h:80-91) on all five fields */
int sf_vecs_scale(sf_vecs* v, int i, double alpha, int count);
/* out[k] = StateVector::Dot(v[first+k], w[x]) (StateVector.h:122-134), FP64 */
int sf_vecs_dots(sf_vecs* v, int first, int count, sf_vecs* w, int x, double Ri, double* out);
/* *out = sum_k StateVector::Dot(v[a+k], w[b+k]), FP64 */
int sf_vecs_dot_sum(sf_vecs* v, int a, sf_vecs* w, int b, int count, double Ri, double* out);
/* StateVector::EnforceBCs (StateVector.h:415-421) */
int sf_vecs_enforce_bcs(sf_vecs* v, int i, int count);
/* StateVector::RemovePhaseShift (StateVector.h:103-120); computes the shift
 * from u1(1,0,N3/2) unless use_given, and returns it in *shift */
int sf_vecs_phase_shift(sf_vecs* v, int i, int use_given, double* shift);
/* RemoveAverage (Integration.h:236-240) of field 0 (u1) or 3 (b) */
int sf_vecs_remove_average(sf_vecs* v, int i, int field, double L3);
/* Block operations of the block Krylov solvers (nb <= 32), FP64 sums:
 * out[i*nb + k] = Dot(v[a+i], w[b+k]) for i < na, k < nb */
int sf_vecs_gram(sf_vecs* v, int a, int na, sf_vecs* w, int b, int nb, double Ri, double* out);
/* w[b+k] += alpha * sum_i coef[i*nb + k] v[a+i] on u1..b (coef host, na x nb;
 * the two ranges must not overlap) */
int sf_vecs_update(sf_vecs* w, int b, int nb, double alpha, sf_vecs* v, int a, int na, const double* coef);
/* keep only the fields of field_mask (bit 0 u1, 1 u2, 2 u3, 3 b) and the
 * modes with j1_lo <= j1 < j1_hi in vector i; p is zeroed */
int sf_vecs_band(sf_vecs* v, int i, int field_mask, int j1_lo, int j1_hi);
/* the z column (N3 complex values) of kept mode `mode` of `field` of vector
 * i, to the host (write = 0) or from it (write = 1); synchronises */
int sf_vecs_column(sf_vecs* v, int i, int field, int mode, float* host, int write);
/* zero the p field of vectors i..i+count-1 */
int sf_vecs_zero_pressure(sf_vecs* v, int i, int count);
int sf_vecs_synchronize(sf_vecs* v);

/* ---- learned continuation predictor (no counterpart in the reference; it
 * stands beside the secant predictor of PseudoArclength.cpp:33-61) ----
 * nlayers 1D convolutions along z (5 taps, zero padding 2) with ReLU between
 * them; channels[0] inputs, channels[nlayers] outputs, each a multiple of 8.
 * Tensors are FP32 on the host, channel-last [batch][Z][C]; on the device
 * the operands are BF16 and the tensor-core contractions accumulate in FP32.
 * Parameters, FP32: for each layer W[Cout][5][Cin] then bias[Cout]. The
 * weights start He-normal from `seed`, the output layer at zero. stream is
 * a cudaStream_t (NULL: legacy default stream). */
typedef struct sf_net sf_net;
int sf_net_create(int nlayers, const int* channels, int Z, int max_batch, unsigned long long seed, void* stream,
                  sf_net** out);
int sf_net_destroy(sf_net* n);
int sf_net_num_params(sf_net* n, long long* count);
int sf_net_get_params(sf_net* n, float* host);
/* also resets the Adam moments */
int sf_net_set_params(sf_net* n, const float* host);
/* y[batch][Z][Cout] = net(x[batch][Z][Cin]); discards the training data */
int sf_net_forward(sf_net* n, const float* x, int batch, float* y);
/* uploads a training set: inputs x[batch][Z][Cin], targets [batch][Z][Cout] */
int sf_net_set_data(sf_net* n, const float* x, const float* target, int batch);
/* mean-square loss over the training set and its gradient (parameter layout) */
int sf_net_gradient(sf_net* n, float* grad, double* loss);
/* `steps` full-batch Adam steps (lr; beta 0.9, 0.999; eps 1e-8); losses[s]
 * (may be NULL) is the loss before step s */
int sf_net_train(sf_net* n, int steps, double lr, double* losses);

/* waits for all work queued on the solver's stream */
int sf_synchronize(sf_solver* s);

/* the solver's stream (cudaStream_t) for callers that order their own work */
int sf_stream(sf_solver* s, void** stream);

/* number of this library's kernel launches issued so far by the solver */
int sf_launch_count(sf_solver* s, long long* count);

#ifdef __cplusplus
}
#endif

#endif /* STRATIFLOW_B200_H */
