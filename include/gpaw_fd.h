/*
 * gpaw_fd.h -- C ABI of libgpawfd.so, the B200 (sm_100a) implementation of
 * GPAW's real-space finite-difference path.
 *
 * Every entry point takes plain pointers and sizes.  Array arguments named
 * in/out/func/source/phi/rho are DEVICE pointers to C-contiguous arrays of
 * shape (nin, n0, n1, n2) (complex values interleaved re, im), exactly the
 * layout of the numpy arrays the reference passes to its C extension.
 * `stream` is a cudaStream_t (NULL = legacy default stream).  Work is
 * enqueued on that stream and the call returns without waiting, except where
 * a result must reach the host (gfd_poisson_solve, gfd_grid_sum).
 *
 * Every call returns a status code; gfd_last_error() gives the message of the
 * last failing call on the calling thread.  Nothing aborts or traps.
 *
 * Reference interfaces replaced (paths relative to the GPAW source tree):
 *   _gpaw.Operator      c/operators.c:465-498 (constructor), :316-405 (apply),
 *                       :49-91 (relax), :408-421 (get_diagonal_element)
 *   _gpaw.Transformer   c/transformers.c:222-265 (constructor), :127-185 (apply)
 *   PoissonSolver       gpaw/poisson.py:21-276 (set_grid_descriptor,
 *                       initialize, solve, solve_neutral, iterate2)
 *   GridDescriptor.integrate  gpaw/grid_descriptor.py:197-215
 */
#ifndef GPAW_FD_H
#define GPAW_FD_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GFD_API __attribute__((visibility("default")))
#else
#define GFD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define GFD_OK 0
#define GFD_EINVAL 1      /* bad shape, size, pointer, dtype or argument */
#define GFD_ENOMEM 2      /* device allocation failed */
#define GFD_ENOCONV 3     /* Poisson solve reached maxiter (PoissonConvergenceError) */
#define GFD_ETIMEOUT 4    /* a bounded device-side wait ran out */
#define GFD_ECUDA 5       /* a CUDA runtime call failed */
#define GFD_EUNSUPPORTED 6 /* valid in the reference but not provided here */
#define GFD_ENEEDGAUSS 7  /* charged non-periodic solve before gfd_poisson_load_gauss */

/* Element types (the `dtype` argument).  The FP32 types are the reduced-
 * precision variants; the reference computes in float64 / complex128 only. */
#define GFD_FLOAT64 0
#define GFD_COMPLEX128 1
#define GFD_FLOAT32 2
#define GFD_COMPLEX64 3

/* Relaxation methods, numbered as in gpaw/poisson.py:28-36. */
#define GFD_RELAX_GS 1      /* Gauss-Seidel; here multicolour, see relax below */
#define GFD_RELAX_JACOBI 2  /* weighted Jacobi */

typedef struct gfd_operator gfd_operator;
typedef struct gfd_transformer gfd_transformer;
typedef struct gfd_poisson gfd_poisson;

/* Message of the last failing call on this thread ("" if none).  Returns the
 * full message length; writes at most len-1 characters plus a NUL. */
GFD_API size_t gfd_last_error(char* buf, size_t len);

/* Library version string, e.g. "gpaw-fd-b200 0.1 sm_100a". */
GFD_API const char* gfd_version(void);

/* ------------------------------------------------------------------------
 * Finite-difference operator.
 * Replaces _gpaw.Operator(coefs, offsets, size, range, neighbors, real,
 * comm, cfd) -- c/operators.c:465-498 -- whose Python caller is
 * FDOperator.__init__ / allocate (gpaw/fd_operators.py:21-70).
 *
 *   ncoefs, coefs[ncoefs]  stencil weights (coefs[0] must be the diagonal
 *                          for relax, as the reference assumes)
 *   offsets[ncoefs*3]      integer (d0, d1, d2) offset of each weight.  The
 *                          reference passes flat offsets on its padded grid;
 *                          the padded grid does not exist here.
 *   size[3]                points per axis (n_c)
 *   range                  halo width (mp, the largest offset)
 *   neighbors[6]           neighbor_cd as (axis, side): 0 = this domain
 *                          (periodic wrap), -1 = none (zero boundary)
 *   real                   1 for float arrays, 0 for complex (the reference
 *                          builds one object per dtype)
 *   cfd                    1 when no offset has two nonzero components
 * ---------------------------------------------------------------------- */
GFD_API int gfd_operator_create(int ncoefs, const double* coefs, const int64_t* offsets,
                        const int64_t size[3], int range, const int64_t neighbors[6],
                        int real, int cfd, gfd_operator** op);
GFD_API int gfd_operator_destroy(gfd_operator* op);

/* out[x] = sum_p coefs[p] * in[x + offsets[p]] for x in 0..nin-1, halos zero
 * or periodic times phase_cd (Operator_apply, c/operators.c:316-405).
 * phase_cd: 12 host doubles, phase_cd[c][d] as (re, im) at 4*c + 2*d, used
 * for complex dtypes only (may be NULL: all phases 1).  The low halo on axis
 * c takes phase_cd[c][1], the high halo phase_cd[c][0] (c/bc.c:234-249).
 * in and out must not overlap. */
GFD_API int gfd_operator_apply(gfd_operator* op, int dtype, const void* in, void* out, int64_t nin,
                       const double* phase_cd, void* stream);

/* nrelax sweeps of relaxation for "operator func = source", in place on
 * func (Operator_relax, c/operators.c:49-91; bmgs_relax, c/bmgs/relax.c).
 * Real dtypes only.  GFD_RELAX_JACOBI: weighted Jacobi with weight w, as
 * the reference.  GFD_RELAX_GS: the reference's lexicographic Gauss-Seidel
 * is a sequential sweep; it is replaced by multicolour Gauss-Seidel
 * ((i0+i1+i2) mod (range+1) colours, a valid colouring for axis-aligned
 * stencils), compared by the converged result, not by iterates.
 * Uses a device scratch array of one grid owned by the operator. */
GFD_API int gfd_operator_relax(gfd_operator* op, int dtype, int relax_method, void* func,
                       const void* source, int nrelax, double w, void* stream);

/* The same sweeps as gfd_operator_relax, allocating no device memory.  This
 * entry point has no counterpart in the reference.
 * gfd_operator_relax takes one grid of scratch from cudaMalloc on first use;
 * callers that cannot allocate -- code running while a CUDA graph is being
 * captured, hosts whose own pool allocator owns all device memory, loops that
 * cannot afford an allocation's implicit synchronisation -- use this call.
 * Its scratch is a 16 MiB array compiled into the library, held on every GPU
 * that loads the library until the process exits, so the grid may have at
 * most 2,097,152 float64 or 4,194,304 float32 points; larger grids return
 * GFD_EINVAL with a message.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before starting any stream capture.  After a device
 * reset (cudaDeviceReset) the next call sees a new context and looks the
 * address up again, so it too must come before any capture.  All calls share
 * the one array: calls that overlap on the GPU (on different streams, or
 * from different threads) race on it and must be serialised by the caller. */
GFD_API int gfd_operator_relax_noalloc(gfd_operator* op, int dtype, int relax_method, void* func,
                                       const void* source, int nrelax, double w, void* stream);

/* Weight of the zero offset (Operator_get_diagonal_element,
 * c/operators.c:408-421). */
GFD_API int gfd_operator_get_diagonal_element(const gfd_operator* op, double* d);

/* out = L in + v * in for nin bands: the kinetic operator and the local
 * potential in one pass.  Replaces FDWaveFunctions.apply_pseudo_hamiltonian
 * (gpaw/wavefunctions/fd.py:50-52): kin.apply(psit, Htpsit, phase_cd)
 * followed by Hamiltonian.apply_local_potential (gpaw/hamiltonian.py:
 * 371-398, Htpsit += psit * vt).  v: device grid of n0*n1*n2 real values,
 * float64 for float64/complex128 bands and float32 for float32/complex64.
 * Axis-aligned operators fuse the potential into the stencil's centre
 * weight (one read and one write per band); other offset sets add it in a
 * second pass. */
GFD_API int gfd_operator_apply_potential(gfd_operator* op, int dtype, const void* in, void* out,
                                         int64_t nin, const double* phase_cd, const void* v,
                                         void* stream);

/* ------------------------------------------------------------------------
 * Band preconditioner.  Replaces gpaw.preconditioner.Preconditioner
 * (gpaw/preconditioner.py:13-70): two coarser levels with nn = 1 kinetic
 * operators (Laplace(gd, -0.5, 1)) and nn = 1 transformers, step =
 * 0.66666666 / kin0.get_diagonal_element().  The handles are borrowed and
 * must outlive the preconditioner; block is the most bands per pass (the
 * scratch holds that many bands on the coarse levels and on the fine grid).
 * ---------------------------------------------------------------------- */
typedef struct gfd_preconditioner gfd_preconditioner;

GFD_API int gfd_preconditioner_create(gfd_operator* kin0, gfd_operator* kin1, gfd_operator* kin2,
                                      gfd_transformer* restrict0, gfd_transformer* restrict1,
                                      gfd_transformer* interpolate2,
                                      gfd_transformer* interpolate1, int dtype, int64_t block,
                                      gfd_preconditioner** out);
GFD_API int gfd_preconditioner_destroy(gfd_preconditioner* pc);
/* out = the preconditioned residuals (Preconditioner.__call__,
 * gpaw/preconditioner.py:45-70) for nb bands; phase_cd: the k-point's Bloch
 * phases (12 doubles, host) for complex bands, else NULL. */
GFD_API int gfd_preconditioner_apply(gfd_preconditioner* pc, int dtype, const void* residuals,
                                     void* out, int64_t nb, const double* phase_cd, void* stream);

/* Pseudo density to the fine grid: Density.interpolate
 * (gpaw/density.py:217-235).  nt_sg = interpolate(nt_sG) for nspins real
 * grids; then, when renormalize != 0 (the caller's "not all periodic") and
 * |pseudo_charge| > 1e-14, nt_sg *= pseudo_charge / (dv_fine * sum(nt_sg)),
 * the reference's x = pseudo_charge / finegd.integrate(nt_sg).sum().  The
 * sum stays on the device; the host does not wait. */
GFD_API int gfd_density_interpolate(gfd_transformer* tr, const double* nt_sG, double* nt_sg,
                                    int64_t nspins, double pseudo_charge, double dv_fine,
                                    int renormalize, void* stream);

/* Device-side error flags of the current device, then cleared: *flags != 0
 * when a stencil kernel gave up on a bounded wait since the last call (its
 * output is then incomplete).  No counterpart in the reference, whose CPU
 * kernels have no such waits. */
GFD_API int gfd_device_errors(int* flags);

/* Fault injection for tests of the out-of-memory paths (no counterpart in
 * the reference, whose GPAW_MALLOC aborts): n > 0 makes the n-th device
 * allocation the library makes from now on fail with GFD_ENOMEM, without
 * touching the device; 0 cancels a planned failure.  Host-side only. */
GFD_API int gfd_test_fail_alloc(long long n);

/* Self-test of the bounded waits behind gfd_device_errors (no counterpart in
 * the reference): one small kernel waits, with the stencil kernels' bounded
 * mbarrier wait limited to max_cycles SM cycles (1 .. about 4e9), on a
 * barrier that nothing completes, sets the device error flag when the wait
 * runs out and returns; nothing is copied, so the early exit leaves no work
 * in flight.  Waits for the device.  gfd_device_errors then reports 1. */
GFD_API int gfd_wait_selftest(long long max_cycles);

/* ------------------------------------------------------------------------
 * Grid transformer (restriction / interpolation).
 * Replaces _gpaw.Transformer(size_in, size_out, k, paddings, npaddings,
 * skip, neighbors, real, comm, interpolate) -- c/transformers.c:222-265 --
 * built by _Transformer (gpaw/transformers.py:19-79).  k = 2*nn in
 * {2, 4, 6, 8}; pad/npad/skip/neighbors are [3][2] as (axis, side).
 * ---------------------------------------------------------------------- */
GFD_API int gfd_transformer_create(const int64_t size_in[3], const int64_t size_out[3], int k,
                           const int64_t pad[6], const int64_t npad[6], const int64_t skip[6],
                           const int64_t neighbors[6], int real, int interpolate,
                           gfd_transformer** tr);
GFD_API int gfd_transformer_destroy(gfd_transformer* tr);

/* Transformer_apply (c/transformers.c:127-185): in has shape
 * (nin, size_in), out (nin, size_out); phases as for gfd_operator_apply. */
GFD_API int gfd_transformer_apply(gfd_transformer* tr, int dtype, const void* in, void* out,
                          int64_t nin, const double* phases, void* stream);

/* ------------------------------------------------------------------------
 * Multigrid Poisson solver (gpaw/poisson.py:21-276).
 * Built from the level operators and transformers exactly as
 * PoissonSolver.set_grid_descriptor builds them: ops[0..levels] with
 * ops[0] the fine-grid Laplace (scale -1/(4 pi), nn) and ops[l>=1] nn=1;
 * restrictors[l] / interpolators[l] between level l and l+1 (nn=1).
 * presmooths/postsmooths/weights have levels+1 entries; the coarsest entry
 * of presmooths/postsmooths is used as given (the reference sets it to 8).
 * dv is the fine-grid volume element.  pbc_all is 1 when every axis is
 * periodic (mean of phi removed after the solve).
 * precision: GFD_POISSON_FP64 runs the V-cycle in float64 as the reference;
 * GFD_POISSON_MIXED runs FP32 V-cycles inside an FP64 defect-correction
 * loop (residual, update and norm in FP64).
 * The solver allocates its level arrays on the device.
 * ---------------------------------------------------------------------- */
#define GFD_POISSON_FP64 0
#define GFD_POISSON_MIXED 1

GFD_API int gfd_poisson_create(int levels, gfd_operator* const* ops, gfd_transformer* const* restrictors,
                       gfd_transformer* const* interpolators, const int* presmooths,
                       const int* postsmooths, const double* weights, int relax_method,
                       double dv, int pbc_all, int precision, gfd_poisson** ps);
GFD_API int gfd_poisson_destroy(gfd_poisson* ps);

/* Right-hand-side operator of the Mehrstellen solver (nn = 'M',
 * gpaw/poisson.py:53-59): the level-0 source becomes B (rho - background),
 * as solve_neutral applies self.B (gpaw/poisson.py:196-199); the level-0
 * operator given to gfd_poisson_create is then LaplaceA.  B is borrowed, on
 * the level-0 grid, real.  NULL removes it.  Batches built earlier keep the
 * previous form. */
GFD_API int gfd_poisson_set_rhs_operator(gfd_poisson* ps, gfd_operator* B);

/* PoissonSolver.solve(phi, rho, charge=None, eps, maxcharge)
 * (gpaw/poisson.py:124-218).  phi (in: initial guess, out: solution) and rho
 * are device float64 arrays of the fine grid.  charge: pass NaN for None
 * (the integral of rho is used).  maxiter = 1000 in the reference.
 *   |charge| <= maxcharge: the neutral solve of rho - background.
 *   charged, every axis periodic: the neutral solve shifted by
 *     charge * madelung (gfd_poisson_set_madelung; GFD_EUNSUPPORTED if unset).
 *   charged, no axis periodic: the monopole (the integral of rho) is carried
 *     by the L = 0 Gaussian of gfd_poisson_load_gauss, whose potential is
 *     added back; GFD_ENEEDGAUSS, with phi unchanged, if it is not loaded.
 *   charged, mixed boundary conditions: GFD_EUNSUPPORTED (the reference
 *     raises NotImplementedError).
 * On return (the call waits for the stream) *niter holds the V-cycle count
 * and *error the last residual norm sum(r^2) dv; GFD_ENOCONV when
 * niter reached maxiter, as PoissonConvergenceError. */
GFD_API int gfd_poisson_solve(gfd_poisson* ps, double* phi, const double* rho, double charge,
                      double eps, double maxcharge, int maxiter, int* niter, double* error,
                      void* stream);
/* The same with flags: GFD_SOLVE_ZERO_INITIAL_PHI is the reference's
 * zero_initial_phi=True -- the charged branches start from phi = 0 instead
 * of the shifted guess; the neutral branch keeps phi as given, as in the
 * reference (gpaw/poisson.py:124-138). */
#define GFD_SOLVE_ZERO_INITIAL_PHI 1
GFD_API int gfd_poisson_solve_ex(gfd_poisson* ps, double* phi, const double* rho, double charge,
                                 double eps, double maxcharge, int maxiter, int flags,
                                 int* niter, double* error, void* stream);

/* The compensating Gaussian of the charged non-periodic branch: Poisson-
 * Solver.load_gauss (gpaw/poisson.py:118-123) with Gaussian(gd).get_gauss(0)
 * and get_gauss_pot(0) (gpaw/utilities/gauss.py:47-82):
 *   g(r) = sqrt(4 a^3) / pi exp(-a r^2),  v(r) = 2 sqrt(pi) erf(sqrt(a) r) / r,
 * r the distance of grid point i (coordinates (i + beg_c) h_cv) from
 * center_v, r^2 clamped to at least 1e-12 (gpaw/utilities/tools.py:92-118).
 * The reference's a = 4 * 19 * max_c sum_v icell_cv^2 and center_v = half
 * the cell's diagonal.  Computed on the device into two level-0 arrays the
 * solver owns; the call waits for the stream. */
GFD_API int gfd_poisson_load_gauss(gfd_poisson* ps, const double h_cv[9], const int64_t beg_c[3],
                                   const double center_v[3], double a, void* stream);
/* Potential shift per unit charge of the charged periodic branch
 * (charged_periodic_correction = madelung(cell_cv), gpaw/poisson.py:143-151). */
GFD_API int gfd_poisson_set_madelung(gfd_poisson* ps, double madelung);
/* madelung(cell_cv) of gpaw/utilities/ewald.py:148: the Ewald potential at a
 * probe charge -1 from its periodic images in a neutralising background
 * (G = 5 / longest lattice vector, 9^3 reciprocal and 3^3 real-space shells
 * either side), computed on the host. */
GFD_API int gfd_madelung(const double cell_cv[9], double* out);

/* Asynchronous form of gfd_poisson_solve for callers that keep several solves
 * in flight (serving).  Enqueues the whole solve on `stream` -- copies of
 * phi/rho into the solver, one graph launch, copy of the result back into
 * phi -- and returns at once.  Once the stream has passed that point (an
 * event or a synchronisation), gfd_poisson_result gives the V-cycle count,
 * the last residual norm and the status gfd_poisson_solve would have
 * returned.  A solver runs one solve at a time: do not enqueue a second solve
 * on the same solver before the first has completed.  (The reference's solve
 * is synchronous; this split has no counterpart there.) */
GFD_API int gfd_poisson_solve_async(gfd_poisson* ps, double* phi, const double* rho, double charge,
                                    double eps, double maxcharge, int maxiter, void* stream);
GFD_API int gfd_poisson_result(const gfd_poisson* ps, int* niter, double* error);

/* Batch of independent solvers (any grid sizes, one solver at most once),
 * captured as parallel branches of a single CUDA graph: one launch runs every
 * solve's V-cycle loop concurrently on the device, each stopping on its own
 * criterion.  phis[i] / rhos[i] belong to solvers[i]; results per solver via
 * gfd_poisson_result.  Each solver keeps its own buffers, so a solver must not
 * run in two batches, or in a batch and a single solve, at the same time.
 * (No counterpart in the reference, which solves one grid per call.) */
typedef struct gfd_poisson_batch gfd_poisson_batch;
GFD_API int gfd_poisson_batch_create(int nsolvers, gfd_poisson* const* solvers,
                                     gfd_poisson_batch** batch);
/* The same with flags: GFD_BATCH_NO_GROUPS runs every solver as its own
 * graph branch (no grouped launches).  Grouping pays for one large batch of
 * small grids; when many batches are in flight at once, as in a serving
 * loop, plain branches overlap better. */
#define GFD_BATCH_NO_GROUPS 1
GFD_API int gfd_poisson_batch_create_ex(int nsolvers, gfd_poisson* const* solvers, int flags,
                                        gfd_poisson_batch** batch);
GFD_API int gfd_poisson_batch_destroy(gfd_poisson_batch* batch);
/* phis[i] = rhos[i] = NULL leaves slot i unused in this launch: its solver
 * runs no V-cycle and its result reads as refused (GFD_EUNSUPPORTED), so a
 * batch captured once can serve fewer requests than it has slots. */
GFD_API int gfd_poisson_batch_solve_async(gfd_poisson_batch* batch, double* const* phis,
                                          const double* const* rhos, double eps, double maxcharge,
                                          int maxiter, void* stream);
/* *grouped = how many of the batch's solvers run grouped.  Solvers of one
 * structure (levels, smoothing, weights, stencil radius or colouring and
 * boundary conditions per level, transfer orders; float64, no Mehrstellen
 * right-hand side) form a group: every V-cycle step is ONE launch over all
 * the group's grids, a persistent kernel whose CTAs pull work tiles from a
 * queue, and the stopping rule runs per solve on the device.  Groups and the
 * remaining solvers run as parallel graph branches (all solvers alone with
 * GFD_BATCH_GROUPED=0). */
GFD_API int gfd_poisson_batch_grouped(const gfd_poisson_batch* batch, int* grouped);

/* ------------------------------------------------------------------------
 * Launch-plan autotuning.  No counterpart in the reference, whose CPU code
 * has one path per operation; it serves the same call sites (Operator.apply
 * and relax, c/operators.c:316-405 and :49-91; Transformer.apply,
 * c/transformers.c:127-185) by choosing how they run on the GPU.
 *
 * A plan fixes the kernel form (one thread per point, or the marching
 * kernel that streams planes along axis 0), the marching tile and the
 * axis-0 split (target CTAs per SM, i.e. the planes each CTA marches
 * through).  gfd_autotune_operator / _transformer time every candidate with
 * CUDA events on the caller's buffers and stream (reps timed launches each,
 * after one untimed launch; the output buffer is overwritten) and cache the
 * fastest under (operation, dtype, mode, grid, radius or order, boundary
 * conditions, floor(log2(bands))).  Later launches with that key use it;
 * others keep the built-in rules.  Marching candidates give bit-identical
 * results; the one-thread-per-point form sums a stencil's terms in another
 * order (rounding-level differences).  Residual sweeps keep the built-in
 * rules.  Not allowed on a stream that is being captured.
 * Plans take effect at the next launch: a Poisson solver's or batch's
 * captured graph keeps the plans it was captured with
 * (gfd_poisson_autotune recaptures).  GFD_TUNE_CACHE=<path> loads a saved
 * cache on first use.
 * ---------------------------------------------------------------------- */
#define GFD_TUNE_APPLY 0      /* gfd_operator_apply */
#define GFD_TUNE_JACOBI 1     /* one weighted-Jacobi sweep (src = rho, weight w) */
#define GFD_TUNE_POTENTIAL 3  /* gfd_operator_apply_potential (src = v) */

typedef struct gfd_tune_plan {
  int form;         /* 0: one thread per point; 1: marching kernel */
  int tile;         /* marching tile: 0 32 columns, 1 16, 2 8, 3 32 columns x 8 rows,
                       4 complex bands with re / im on lane pairs (radius <= 3),
                       5 the same for complex128 on full rows staged by TMA,
                       6 complex128, 48 columns x 8 rows (axis-2 lengths that are
                       multiples of 48) */
  int ctas_per_sm;  /* axis-0 split target */
  double us;        /* measured time per launch, microseconds */
} gfd_tune_plan;

GFD_API int gfd_autotune_operator(gfd_operator* op, int dtype, int mode, const void* in, void* out,
                                  const void* src, int64_t nin, const double* phase_cd, double w,
                                  int reps, void* stream, gfd_tune_plan* best);
GFD_API int gfd_autotune_transformer(gfd_transformer* tr, int dtype, const void* in, void* out,
                                     int64_t nin, int reps, void* stream, gfd_tune_plan* best);
/* The cached plan for a launch: *found = 1 and *plan filled, or *found = 0. */
GFD_API int gfd_autotune_operator_plan(const gfd_operator* op, int dtype, int mode, int64_t nin,
                                       gfd_tune_plan* plan, int* found);
GFD_API int gfd_autotune_transformer_plan(const gfd_transformer* tr, int dtype, int64_t nin,
                                          gfd_tune_plan* plan, int* found);
GFD_API int gfd_autotune_count(int* n);
GFD_API int gfd_autotune_clear(void);
/* Text file, one plan per line; load merges into the cache. */
GFD_API int gfd_autotune_save(const char* path);
GFD_API int gfd_autotune_load(const char* path);
/* Tune every level's Jacobi sweep and every restriction and interpolation of
 * a solver on its own level buffers, then drop its captured graph so the next
 * solve uses the plans.  Batches capture at creation: tune first. */
GFD_API int gfd_poisson_autotune(gfd_poisson* ps, int reps, void* stream);

/* ------------------------------------------------------------------------
 * Reductions.
 * sum over all points of a float64 array of n elements, times scale (the
 * integral of GridDescriptor.integrate, gpaw/grid_descriptor.py:197-215).
 * Deterministic: a fixed reduction tree independent of timing.  Waits for
 * the stream and writes the result to *result (host).
 * ---------------------------------------------------------------------- */
GFD_API int gfd_grid_sum(const double* a, int64_t n, double scale, double* result, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GPAW_FD_H */
