/*
 * bph.h -- C ABI of the B200 self-gravity Poisson solver (bipoly_hydro's
 * potsetup + potential_solver path).
 *
 * Plain pointers and sizes only.  Host arrays are Fortran column-major
 * real(8) rho(numr,numz,numphi) / pot(numr,numz,numphi) including the guard
 * zones, exactly the COMMON /poisson/ pot, rho layout of the reference
 * (potential_solver.F90:18-19).  Device arrays use the same layout.
 *
 * Every call returns an int status (BPH_OK = 0, negative on error) and
 * bph_last_error() gives the text of the last failure on the calling
 * thread.  A context is not thread-safe: use one per host thread or
 * serialise calls on it.
 */
#ifndef BPH_H
#define BPH_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BPH_OK 0
#define BPH_ERR_INVALID (-1)   /* bad grid, argument or layout */
#define BPH_ERR_NOMEM (-2)     /* device memory exhausted / admission refused */
#define BPH_ERR_NONFINITE (-3) /* NaN or Inf in the density */
#define BPH_ERR_CUDA (-4)      /* CUDA runtime failure (text in bph_last_error) */
#define BPH_ERR_TIMEOUT (-5)   /* a bounded wait expired */
#define BPH_ERR_STATE (-6)     /* call made in the wrong state */
#define BPH_PENDING 1          /* request not finished yet (bph_server_poll) */

/* Grid and solver constants.  potsetup reads these from runhydro.h
 * (numr, numz, numphi), setup_frac.F90:374-376 (dr; dz = dr), the fort.7
 * deck (isym) and pot.h:3 (mmax).  One rank: numr_dd = numr, numz_dd = numz. */
typedef struct bph_grid {
    int numr;    /* radial zones incl. guard J=1 and boundary J=numr, >= 5 */
    int numz;    /* vertical zones incl. guard K=1 and boundary K=numz, >= 5 */
    int numphi;  /* azimuthal zones: power of two, >= 2*mmax (4*mmax for isym 3) */
    double dr;   /* zone size in r and z */
    int isym;    /* 1: no symmetry, 2: equatorial, 3: pi + equatorial */
    int mmax;    /* boundary modes, 30 in the reference; 2..64 */
} bph_grid_t;

typedef struct bph_ctx bph_ctx_t;

/* Replaces potsetup.F90:6 (called once at setup_frac.F90:689).  Builds the
 * Green-function tables (tm.F90, sm.F90, bm.F90 with elle/ellf/rf/rd/
 * gammln), the azimuthal trig data and the ADI coefficients, all on the
 * current CUDA device, and returns a context that owns them. */
int bph_setup(const bph_grid_t *grid, bph_ctx_t **ctx);

/* Replaces potential_solver.F90:6 (called at setup_frac.F90:690 and
 * main.F90:396).  rho and pot are HOST arrays.  tstep > 1 runs 5 ADI steps
 * from the previous solution kept on the device; otherwise 20 steps from
 * zero (potential_solver.F90:80-94).  Synchronous: returns after pot is
 * written. */
int bph_potential_solver(bph_ctx_t *ctx, const double *rho, double *pot, int tstep);

/* Same solve on DEVICE arrays, enqueued on the context's stream; returns
 * without waiting.  A non-finite density is reported by bph_synchronize. */
int bph_potential_solver_device(bph_ctx_t *ctx, const double *d_rho, double *d_pot, int tstep);

/* One SCF-like iteration on DEVICE arrays in one call (no counterpart in
 * the reference, whose SCF code produced the models scfin_frac.F90:105-125
 * reads from disk): the density is mixed with a seeded perturbation of
 * itself, rho <- 0.9 rho + 0.1 rho (1 + eps xi), xi ~ N(0,1) per zone
 * from a counter-based generator keyed by (seed, iteration, zone), so a
 * sequence is reproducible; renormalised so that its interior mass
 * sum_{J=2..numr-1, K=2..numz-1, L} rho rhf(J) dr dz dphi equals `mass`
 * (mass <= 0 keeps the mass it had before the update); then solved as
 * potential_solver (tstep > 1 warm from the kept potential, else cold).
 * d_rho is updated in place, d_pot receives the potential.  Enqueued on
 * the context's stream; a non-finite density is reported by
 * bph_synchronize. */
int bph_scf_step(bph_ctx_t *ctx, double *d_rho, double *d_pot, double eps, double mass, unsigned long long seed,
                 int iteration, int tstep);
/* Target mass and renormalisation factor of the last bph_scf_step
 * (synchronises the context's stream); either pointer may be NULL. */
int bph_scf_mass(bph_ctx_t *ctx, double *mass_out, double *scale_out);

/* Explicit step count (helmadi(nsteps)); cold != 0 starts from zero.
 * on_device != 0 means rho/pot are device arrays (asynchronous). */
int bph_solve_nsteps(bph_ctx_t *ctx, const double *rho, double *pot, int nsteps, int cold,
                     int on_device);

/* Converged FP64 solve: the nsteps schedule is repeated until the relative
 * change of the Fourier-space potential over one cycle is <= tol, or
 * max_cycles ran.  Synchronous; cycles_out and resid_out (weighted
 * relative residual ||-4 pi rho_hat - A phi_hat|| / ||4 pi rho_hat||) may
 * be NULL.  The reference has no such mode (it always runs 5 or 20 steps);
 * this is the fully converged discrete solution the mixed-precision solver
 * is measured against. */
int bph_solve_converged(bph_ctx_t *ctx, const double *rho, double *pot, int nsteps, int cold,
                        double tol, int max_cycles, int on_device, int *cycles_out,
                        double *resid_out);

/* potential_solver plus the effective potential the hydro source step
 * builds from pot next (source.F90:156, make_source_temp.F90:121):
 * phieff(J,K,L) = pot(J,K,L) - 0.5*omega_frame^2*rhf(J)^2, written by the
 * same kernel that writes pot.  on_device selects device or host arrays. */
int bph_potential_solver_phieff(bph_ctx_t *ctx, const double *rho, double *pot, double *phieff,
                                double omega_frame, int tstep, int on_device);

/* Warm state from a potential, e.g. one read back from a continuation file
 * (ritecont_frac_new.F90:151-160 writes pot): the next tstep > 1 solve
 * starts its 5 ADI steps from this potential, as potential_solver does from
 * its kept potp (potential_solver.F90:80-87).  The reference instead starts
 * cold after a restart (setup_frac.F90:690). */
int bph_set_potential(bph_ctx_t *ctx, const double *pot, int on_device);

/* Reads the reference's continuation record: the fort.12.<tstep>.<rank>
 * file that ritecont_frac_new.F90:151-160 writes with
 *     write(12) s, t, a, rho, tau, pot, tempa, frac1, frac2
 * (one Fortran unformatted sequential record of nine real(8) arrays of
 * the grid's shape, 4-byte record markers; subrecords with negative
 * leading markers and big-endian files are recognised) and that
 * setup_frac.F90:647-648 reads for a continued run.  rho_out / pot_out
 * (host arrays of numr*numz*numphi doubles, either may be NULL) receive
 * the density and the potential.  BPH_ERR_INVALID when the file is
 * missing or its record does not hold nine arrays of the grid's shape. */
int bph_read_continuation(const char *path, const bph_grid_t *grid, double *rho_out, double *pot_out);

/* bph_read_continuation on the context's grid, then bph_set_potential
 * with the stored potential: the next tstep > 1 solve continues warm from
 * the potential of the run that wrote the file.  rho_out may be NULL. */
int bph_restore_continuation(bph_ctx_t *ctx, const char *path, double *rho_out);

/* Mixed-precision converged solve (no counterpart in the reference, which
 * always runs a fixed 5 or 20 FP64 steps): iterative refinement in which
 * every cycle forms the FP64 residual -4 pi rho_hat - A phi, runs the nsteps
 * ADI schedule on the defect equation A delta = r in FP32 on chip, and adds
 * delta to phi in FP64, until |delta|/|phi| <= tol or max_cycles.  The
 * boundary potential, the FFTs and every residual/update stay FP64, so the
 * result converges to the FP64 discrete solution (bph_solve_converged).
 * It also stops once a cycle no longer halves the update (the FP32 inner
 * solves have reached their accuracy).  Arguments as bph_solve_converged. */
int bph_solve_converged_mixed(bph_ctx_t *ctx, const double *rho, double *pot, int nsteps, int cold,
                              double tol, int max_cycles, int on_device, int *cycles_out,
                              double *resid_out);

/* ---- batches: many independent solves on one grid ----------------- */

/* A batch holds the warm states of up to `capacity` independent solves on
 * the context's grid (SCF sweeps over mass ratio and separation, ensembles,
 * many clients).  No counterpart in the reference, which solves one density
 * per call.  The instances share the context's Green tables: one pass over
 * the tables serves every instance's boundary potential. */
typedef struct bph_batch bph_batch_t;
int bph_batch_create(bph_ctx_t *ctx, int capacity, bph_batch_t **batch);

/* potential_solver for instances 0..n-1 (n <= capacity), all at the same
 * tstep (warm 5 steps if tstep > 1, else cold 20); instance i keeps its own
 * warm state between calls.  rho[i]/pot[i] are device arrays when
 * on_device != 0 (asynchronous on the context's stream), else host arrays
 * (synchronous).  Results equal n separate bph_potential_solver calls to
 * rounding. */
int bph_batch_solve(bph_batch_t *batch, int n, const double *const *rho, double *const *pot, int tstep,
                    int on_device);

/* As bph_batch_solve for the n distinct instances instances[0..n-1]
 * (each in 0..capacity-1): position i of rho/pot belongs to instance
 * instances[i]; the other instances keep their state untouched. */
int bph_batch_solve_instances(bph_batch_t *batch, int n, const int *instances, const double *const *rho,
                              double *const *pot, int tstep, int on_device);
/* Converged solves of instances 0..n-1 (the bph_solve_converged /
 * bph_solve_converged_mixed forms for a batch): the transforms and the
 * boundary once per call, then cycles of nsteps ADI steps from each
 * instance's warm state (cold != 0: from zero) until every instance's
 * relative update is at most tol (mixed != 0: FP32 refinement cycles on the
 * FP64 defect, which also stop once a cycle no longer halves the update) or
 * max_cycles.  cycles_out: cycles run; resid_out: the largest relative FP64
 * residual over the instances (NULL skips it).  One host synchronisation
 * per cycle.  Mixed runs the context's refinement kernel (on-chip, or the
 * grid-wide one for slots beyond shared memory). */
int bph_batch_solve_converged(bph_batch_t *batch, int n, const double *const *rho, double *const *pot, int nsteps,
                              int cold, double tol, int max_cycles, int mixed, int on_device, int *cycles_out,
                              double *resid_out);
int bph_batch_destroy(bph_batch_t *batch);
size_t bph_batch_device_bytes(const bph_batch_t *batch);
/* Boundary moments of batch positions 0..n-1 from the last batched call
 * (inspection): out[pos][m][b][cos|sin], the bph_copy_moments layout per
 * position; count >= n*mmax*nb*2. */
int bph_batch_copy_moments(bph_batch_t *batch, int n, double *out, size_t count);

/* ---- plans: batches on several grids as one graph launch -------------
 *
 * No counterpart in the reference.  A plan records the device work of
 * several batches (typically one per grid shape, each batch on its own
 * context) into one CUDA graph whose branches run concurrently, so that a
 * mixed set of small and large grids fills the GPU and costs one launch.
 * Part p solves instances 0..counts[p]-1 of batches[p], reading
 * rho[p][i] and writing pot[p][i]: DEVICE arrays fixed at creation (refill
 * them between launches).  The contexts must live on one device and must
 * not be used by other calls while a launch of the plan runs. */
typedef struct bph_plan bph_plan_t;
int bph_plan_create(int nparts, bph_batch_t *const *batches, const int *counts, const double *const *const *rho,
                    double *const *const *pot, bph_plan_t **plan);
/* Asynchronous replay on `stream` (a cudaStream_t, NULL = default stream):
 * every instance of every part at this tstep (warm 5 steps if tstep > 1,
 * else cold 20; one graph per kind, recorded on first use). */
int bph_plan_launch(bph_plan_t *plan, int tstep, void *stream);
/* Waits for the launches on `stream` and reports non-finite densities. */
int bph_plan_synchronize(bph_plan_t *plan, void *stream);
/* Kernel launches one replay makes (both kinds record the same count). */
int bph_plan_launches(const bph_plan_t *plan);
int bph_plan_destroy(bph_plan_t *plan);

/* ---- serving: continuous batching (no counterpart in the reference) ----
 *
 * A server drives one context from a worker thread (make no other call on
 * that context until bph_server_destroy).  A client is a resident instance:
 * its -4 pi rho_hat and its last potential stay on the device, its first
 * request is a cold 20-step solve and every later one a warm 5-step solve
 * from its previous potential (potential_solver.F90:80-94), as a sequence
 * of potential_solver calls would be.  Requests queue in arrival order;
 * whenever the GPU is free the worker takes the oldest pending request of
 * every client that has one (at most max_batch; 0 = no limit) and solves
 * them together (bph_batch_solve_instances: one pass over the tables),
 * so requests that arrive while a batch runs join the next one.  Results
 * equal the client's own sequence of single solves to rounding.
 *
 * Admission: the number of resident clients is fixed at creation by
 * mem_cap_bytes (0 = no cap) and the free device memory, each client
 * counting its slot arrays, moments and host staging; opening a client
 * beyond that returns BPH_ERR_NOMEM.  rho/pot are arrays of the grid's
 * layout that the caller keeps valid until the request completes (pot is
 * written then).  A request whose density holds NaN or Inf completes with
 * BPH_ERR_NONFINITE and its client's next request runs cold; the other
 * requests of its batch are unaffected. */
typedef struct bph_server bph_server_t;
/* flags: BPH_SERVER_DEVICE_ARRAYS makes rho/pot device arrays of the
 * context's GPU (their writes must be complete when submitted; pot is
 * complete when the request is reported done); else host arrays. */
#define BPH_SERVER_DEVICE_ARRAYS 1
int bph_server_create(bph_ctx_t *ctx, int max_clients, size_t mem_cap_bytes, int max_batch, int flags,
                      bph_server_t **server);
/* Converged mode: from the next batch on, every request is a converged
 * solve (bph_batch_solve_converged with nsteps, tol, max_cycles; mixed != 0:
 * FP32 refinement on the FP64 defect; first requests of a client cold, later
 * ones from its last potential).  nsteps = 0 returns to the drop-in solve.
 * Best called before submitting; FP64 mode reserves one more slot array per
 * resident client. */
int bph_server_set_converged(bph_server_t *server, int nsteps, double tol, int max_cycles, int mixed);
/* Resident clients this server admits. */
int bph_server_capacity(const bph_server_t *server);
int bph_server_open_client(bph_server_t *server, int *client);
/* Queued requests of the client still complete; its slot is reused after. */
int bph_server_close_client(bph_server_t *server, int client);
int bph_server_submit(bph_server_t *server, int client, const double *rho, double *pot, long long *request);
/* BPH_PENDING, or the request's final status (then forgotten); latency_s
 * (may be NULL) receives submit-to-completion seconds. */
int bph_server_poll(bph_server_t *server, long long request, double *latency_s);
/* Blocks until the request completes (timeout_s <= 0: no limit; else
 * BPH_ERR_TIMEOUT when it expires), then reports as bph_server_poll. */
int bph_server_wait(bph_server_t *server, long long request, double timeout_s, double *latency_s);
int bph_server_stats(const bph_server_t *server, long long *batches, long long *solves);
/* Finishes the queued requests, stops the worker, frees the clients. */
int bph_server_destroy(bph_server_t *server);

/* Pins a host array for the life of the run (cudaHostRegister, portable to
 * every device) so that bph_potential_solver and the other host-array calls
 * copy it at pinned-memory speed instead of through the driver's pageable
 * staging.  Meant for arrays at fixed addresses such as the reference's
 * COMMON /poisson/ rho and pot (potential_solver.F90:18-19): the Fortran
 * shim registers both once in potsetup.  No counterpart in the reference.
 * Registering an already registered range is not an error.  Unregister
 * (bph_unregister_host, same pointer) before freeing the memory. */
int bph_register_host(void *ptr, size_t bytes);
int bph_unregister_host(void *ptr);

/* Stream used for all later work of this context (a cudaStream_t; NULL is
 * CUDA's default stream).  Until the first call the context uses a
 * non-blocking stream of its own. */
int bph_set_stream(bph_ctx_t *ctx, void *cuda_stream);

/* Wait for the context's stream; returns the first deferred error
 * (e.g. BPH_ERR_NONFINITE) of the calls since the last synchronize. */
int bph_synchronize(bph_ctx_t *ctx);

/* Releases the caller's handle: no call may use `ctx` afterwards.  The
 * device state is freed at once, or, while batches created on the context
 * still exist, when the last of them is destroyed (so the two may be
 * destroyed in either order, as a garbage-collected host does). */
int bph_destroy(bph_ctx_t *ctx);

/* Text of the last error on this thread ("" if none). */
const char *bph_last_error(void);

/* Library version string. */
const char *bph_version(void);

/* ---- inspection (tests and diagnostics) --------------------------- */

/* Number of boundary rows nb: (numr-2)+(numz-2), plus (numr-2) for isym 1. */
int bph_num_boundary_rows(const bph_ctx_t *ctx);

/* Copies the Green tables to host memory, layout G[m][b][p] with
 * p = (jl-2) + (numr-2)*(kl-2) and b = top jg-2 | side (numr-2)+kg-2 |
 * bottom (isym 1).  n = mmax*nb*(numr-2)*(numz-2) doubles. */
int bph_copy_green(bph_ctx_t *ctx, double *host_out, size_t n);

/* Copies the boundary moments S[m][b][2] (cos, sin) of the last solve. */
int bph_copy_moments(bph_ctx_t *ctx, double *host_out, size_t n);

/* Phases of one solve, for timing a single kernel (bph_run_phase). */
#define BPH_PHASE_FFT_RHO 0   /* k_fft_fwd: rho -> -4 pi rho_hat + moments */
#define BPH_PHASE_CONTRACT 1  /* k_green_contract: tables x moments -> S and the Dirichlet slots */
#define BPH_PHASE_SLOTS 2     /* k_boundary_slots: S -> Dirichlet slots (standalone form; solves write them in the contraction) */
#define BPH_PHASE_ADI 3       /* k_adi: nsteps warm ADI steps */
#define BPH_PHASE_FFT_INV 4   /* k_fft_inv: slots -> pot */

/* Enqueues exactly one phase of a solve on the context's stream (device
 * arrays; nsteps only for BPH_PHASE_ADI).  Diagnostic: phases run in order
 * reproduce bph_solve_nsteps with on_device=1 and cold=0. */
int bph_run_phase(bph_ctx_t *ctx, int phase, const double *d_rho, double *d_pot, int nsteps);

/* Boundary contraction without any device allocation.  No counterpart in
 * the reference (its bessel.F90:186-296 sums run on host memory).
 *
 * For callers that may not call cudaMalloc where they need the boundary
 * moments (an application memory pool that must not grow, a real-time loop
 * that cannot afford cudaMalloc's device synchronisation, code that only
 * holds pointers its caller gave it).  Inputs: ctx (its Green tables, built
 * earlier by bph_setup) and d_mom, the interior density moments on the
 * device, layout mom[m][cos|sin][p], p = (J-2) + (numr-2)*(K-2), with
 * mom = sum_l rho(J,K,l) (cos|sin)(f m (l-1/2) dphi), f = 2 for isym 3
 * else 1.  Output: d_S on the device, S[m][b][cos|sin] (bph_copy_moments'
 * layout).  Enqueued on the context's stream; allocates nothing.
 *
 * Scratch: an 8 MiB file-scope device array per GPU, held until the
 * process exits.  Grids whose 64 KiB of arrival counters (mmax * ceil(nb/8)
 * tiles) or whose mmax*nb*2 partial sums per split exceed it are rejected
 * with BPH_ERR_INVALID before any device work.  bph_setup looks up the
 * array's device address for its context (cudaGetSymbolAddress), so this
 * call makes no runtime lookup.  All calls on a device share the array and
 * it keeps the last call's contents; calls that overlap on the GPU race
 * and must be serialised by the caller. */
int bph_green_contract_noalloc(bph_ctx_t *ctx, const double *d_mom, double *d_S);

/* Launch-configuration facts of a context (diagnostics; -1 if unknown). */
#define BPH_INFO_ADI_THREADS 0        /* threads of the FP64 on-chip ADI kernel (0: other variant) */
#define BPH_INFO_ADI_SMEM 1           /* its dynamic shared bytes */
#define BPH_INFO_MIXED_THREADS 2      /* threads of the FP32 refinement ADI kernel */
#define BPH_INFO_MIXED_SMEM 3         /* its dynamic shared bytes */
#define BPH_INFO_MIXED_CTAS_PER_SM 4  /* its resident CTAs per SM */
#define BPH_INFO_CONTRACT_SPLIT 5     /* slices of the split-K Green contraction */
#define BPH_INFO_MIXED_KIND 6         /* refinement ADI kernel in use (BPH_MIXED_ADI_*) */
#define BPH_INFO_MIXED_FORWARD_NS 7   /* setup-time duration of a 10-step forwarding-form launch, ns (0: not timed) */
#define BPH_INFO_MIXED_INCREMENT_NS 8 /* the same for the increment form */
#define BPH_INFO_ADI_PREFETCH 9       /* bulk-copy factor prefetch: bit 0 FP64 ADI, bit 1 FP32 refinement ADI */
#define BPH_INFO_ADI_KERNEL 10        /* FP64 drop-in ADI kernel in use (BPH_ADI_KERNEL_*) */
#define BPH_INFO_ADI_WARP_SMEM 11     /* dynamic shared bytes of the warp-cooperative kernel (0: not used) */
#define BPH_INFO_MIXED_WARP_NS 12     /* setup-time duration of a 10-step warp-cooperative refinement launch, ns */
#define BPH_INFO_GREEN_SMS 13         /* SMs of the contraction's partition in the overlapped solve (0: not requested,
                                         negative: the set-up step that failed) */
#define BPH_INFO_CONTRACT_KIND 14     /* boundary contraction of the single solve (BPH_CONTRACT_*) */
#define BPH_INFO_FFT_DENSE 15         /* 1: FFT tiles compiled for eight CTAs per SM (autotuned, or BPH_FFT_DENSE) */
#define BPH_INFO_CONTRACT_FULL_NS 16  /* set-up autotune: one full-table contraction, ns (0: not timed) */
#define BPH_INFO_CONTRACT_COMPACT_NS 17 /* the same for the compact contraction */
#define BPH_INFO_FFT_NS 18            /* set-up autotune: forward + inverse FFT with regular tiles, ns */
#define BPH_INFO_FFT_DENSE_NS 19      /* the same with dense tiles */
#define BPH_INFO_ADI_SEG_NS 20        /* set-up autotune: 5 ADI steps of every slot, segmented kernel, ns */
#define BPH_INFO_ADI_WARP_NS 21       /* the same with the warp-cooperative kernel */
#define BPH_INFO_MIXED_DIRECT_NS 22   /* setup-time duration of one direct FP32 defect solve, ns (0: not timed) */
#define BPH_CONTRACT_FULL 1           /* streams the full tables G[m][b][p] */
#define BPH_CONTRACT_COMPACT 2        /* streams the symmetric tiles and side vectors (2/3 fewer bytes) */
#define BPH_ADI_KERNEL_WARP 1         /* warp-cooperative line solves, shuffle carries (128x96, 64x64 interiors) */
#define BPH_ADI_KERNEL_SEGMENTED 2    /* CTA-wide segmented line solves (other grids whose slot fits on chip) */
#define BPH_ADI_KERNEL_ONCHIP 3       /* one thread per line, slot on chip */
#define BPH_ADI_KERNEL_GRID_WIDE 4    /* slots beyond shared memory: grid-wide panel kernels */
long long bph_info(const bph_ctx_t *ctx, int what);

/* Tuning knobs (no counterpart in the reference).
 *
 * BPH_CFG_MIXED_ADI selects the FP32 ADI kernel of the mixed-precision
 * refinement (bph_solve_converged_mixed):
 *   BPH_MIXED_ADI_AUTO       time the on-chip kernels that fit this grid and keep the fastest
 *                            (what bph_setup does unless the environment sets
 *                            BPH_AUTOTUNE=0, which keeps the forwarding form);
 *   BPH_MIXED_ADI_FORWARD    helmadi's right-hand-side form in FP32, the next
 *                            half-step's right-hand side written by the
 *                            current one (fewer instructions per step);
 *   BPH_MIXED_ADI_INCREMENT  every half-step solves for an increment of the
 *                            residual r - A delta (more instructions, smaller
 *                            shared-memory footprint).
 *   BPH_MIXED_ADI_GLOBAL     the same cycle with the slot's arrays in global
 *                            memory, for grids whose slots exceed shared memory.
 * All converge to the same discrete solution.  Returns BPH_ERR_INVALID for
 * an on-chip kind that does not fit this grid. */
#define BPH_CFG_MIXED_ADI 0
#define BPH_MIXED_ADI_AUTO 0
#define BPH_MIXED_ADI_FORWARD 1
#define BPH_MIXED_ADI_INCREMENT 2
/* the forwarding form with its slot in global memory: any grid size, the
 * choice when neither on-chip kernel fits (e.g. 258x194x512) */
#define BPH_MIXED_ADI_GLOBAL 3
/* the forwarding form with warp-cooperative line solves (shuffle carries,
 * two CTAs per SM), for 128 x 96 interiors (130x98 grids) */
#define BPH_MIXED_ADI_WARP 4
/* not an ADI: the defect equation solved directly in FP32 (eigen-transform of
 * the vertical operator, one radial tridiagonal per vertical mode, inverse
 * transform), one kernel per cycle, for slots whose FP32 residual and vertical
 * transform fit in one CTA's shared memory (128 x 96 interiors: 100 KB, two
 * CTAs per SM); each refinement cycle then gains about the FP32 accuracy of
 * the solve instead of one ADI cycle's reduction.  The cycle's nsteps is not
 * used. */
#define BPH_MIXED_DIRECT 5
int bph_configure(bph_ctx_t *ctx, int key, int value);

/* Number of kernels this context has launched so far. */
long long bph_launch_count(const bph_ctx_t *ctx);

/* Device bytes held by the context. */
size_t bph_device_bytes(const bph_ctx_t *ctx);

#ifdef __cplusplus
}
#endif
#endif
