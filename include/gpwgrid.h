/*
 * gpwgrid.h -- C ABI of the B200 (sm_100a) implementation of GPAW's
 * real-space grid hot path: finite-difference stencils with halo fill,
 * restriction / interpolation transformers, weighted-Jacobi relaxation and
 * the multigrid Poisson V-cycle.
 *
 * The entry points replace the reference's extension types for this path,
 *   _gpaw.Operator     c/operators.c:462-495   (registered at c/_gpaw.c:154)
 *   _gpaw.Transformer  c/transformers.c:219-262 (registered at c/_gpaw.c:157)
 * and the kernels beneath them (c/bmgs/fd.c, relax.c, restrict.c,
 * interpolate.c, cut.c, paste.c, translate.c, zero.c and the serial halo fill
 * of c/bc.c).  Constructor arguments keep the reference's meaning and
 * layout; arrays are device pointers owned by the caller (as in the
 * reference, where the caller owns every NumPy array and C keeps raw pointers
 * only for the duration of a call).
 *
 * Conventions
 *   - Grids are C-contiguous (..., n0, n1, n2); `nin` leading grids are
 *     processed by one call (c/operators.c:325-327).
 *   - `phases` is the (3, 2) complex Bloch phase table phase_cd as 12 doubles
 *     (re, im interleaved), host memory, required for complex data on periodic
 *     axes; NULL means all phases 1.
 *   - `stream` is a cudaStream_t (NULL: legacy default stream).  Calls are
 *     asynchronous on that stream unless stated otherwise.
 *   - Every function returns GPW_OK or an error code; gpw_last_error() gives
 *     a message.  Handles are not thread-safe.
 *   - No handle or function here uses MPI; the reference's `comm` argument is
 *     dropped (single GPU, no domain decomposition).
 */
#ifndef GPWGRID_H
#define GPWGRID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define GPW_OK 0
#define GPW_ENOMEM 12     /* device allocation failed */
#define GPW_EINVAL 22     /* bad shape / dtype / argument */
#define GPW_ENOTSUP 95    /* valid request the library does not implement */
#define GPW_ETIMEDOUT 110 /* a bounded device-side wait gave up */
#define GPW_ECONV 1001    /* Poisson V-cycles reached maxiter (PoissonConvergenceError) */
#define GPW_ECUDA 1002    /* a CUDA runtime call failed */

/* ------------------------------------------------------------ element types */
#define GPW_F64 0  /* float64     (reference NPY_DOUBLE) */
#define GPW_C128 1 /* complex128  (reference NPY_CDOUBLE) */
#define GPW_F32 2  /* float32     (new form, no reference counterpart) */
#define GPW_C64 3  /* complex64   (new form, no reference counterpart) */

typedef struct gpw_operator gpw_operator;
typedef struct gpw_transformer gpw_transformer;
typedef struct gpw_woperator gpw_woperator;
typedef struct gpw_poisson gpw_poisson;
typedef void *gpw_stream; /* cudaStream_t */

/* Message of the last failing call on this host thread ("" if none). */
const char *gpw_last_error(void);
/* Library version string. */
const char *gpw_version(void);

/* ------------------------------------------------------------ FD operator */

/* Replaces _gpaw.Operator(coefs, offsets, size, range, neighbors, real, comm,
 * cfd), c/operators.c:462-495 (built by gpaw/fd_operators.py:75-77).
 *   coefs[ncoefs]     stencil coefficients (float64)
 *   offsets[ncoefs]   linear offsets into the grid padded by `range` on all
 *                     six faces (gpaw/fd_operators.py:50-52)
 *   size[3]           interior extent n_c
 *   range             padding mp (largest offset)
 *   neighbors[3][2]   neighbor_cd: 0 = this domain (periodic wrap), -1 = zero
 *                     boundary (gpaw/domain.py:111-139, serial)
 *   real              1 for float data, 0 for complex (sets the halo type)
 *   cfd               1 if every offset lies on one axis (star stencil)     */
int gpw_operator_new(const double *coefs, const int64_t *offsets, int ncoefs,
                     const int64_t size[3], int range,
                     const int64_t neighbors[6], int real, int cfd,
                     gpw_operator **out);

/* Operator.apply(input, output, phases), c/operators.c:316-405:
 * out[x] = sum_p coef_p * in_padded[x + offset_p] for `nin` grids.  `in` may
 * equal `out` (in-place, as the reference allows).                          */
int gpw_operator_apply(gpw_operator *op, int dtype, const void *in, void *out,
                       int64_t nin, const double *phases, gpw_stream stream);

/* The kinetic operator and the local potential in one pass over the bands:
 * out[x] = (A in)[x] + pot * in[x].  Replaces kin.apply(psit_xG, Htpsit_xG,
 * phase_cd) followed by ham.apply_local_potential(psit_xG, Htpsit_xG, s),
 * i.e. Htpsit_G += psit_G * vt_G (gpaw/wavefunctions/fd.py:77-80,
 * gpaw/hamiltonian.py:397-424).  `pot` is one real grid of the operator's
 * shape in the element's scalar type (float64 for float64 / complex128,
 * float32 for float32 / complex64), shared by all `nin` grids.             */
int gpw_operator_apply_potential(gpw_operator *op, int dtype, const void *in,
                                 void *out, int64_t nin, const double *phases,
                                 const void *pot, gpw_stream stream);

/* The apply with the NumPy glue that follows it folded into its output
 * stage: out = A in + pot in + aux_scale aux (pot and aux may be NULL; aux
 * is `nin` grids of the element type, as `out`, and may be `out` itself:
 * such a call is never timed by the tile autotuner).  Together with an operator
 * whose coefficients were scaled on the host it replaces sequences such as
 * the preconditioner's `kin0.apply(d0, q0); q0 -= residuals; axpy(-step,
 * q0, d0); d0 *= -1` (gpaw/preconditioner.py:56-60) by one pass.          */
int gpw_operator_apply_fused(gpw_operator *op, int dtype, const void *in,
                             void *out, int64_t nin, const double *phases,
                             const void *pot, const void *aux,
                             double aux_scale, gpw_stream stream);

/* Operator.relax(relax_method, func, source, nrelax, w), c/operators.c:49-91
 * and c/bmgs/relax.c:7-73.  relax_method 2 = weighted Jacobi (each sweep
 * func = (1-w) func + w (source - sum_{p!=0} c_p func[x+o_p]) / c_0);
 * relax_method 1 = lexicographic Gauss-Seidel (w ignored), computed as a
 * hyperplane wavefront that reproduces the lexicographic update order.
 * dtype GPW_F64 (reference) or GPW_F32.  func is updated in place.
 * `nin` independent grids (func, source of shape (nin, n0, n1, n2)) are
 * relaxed by one call (nin = 1 is the reference's call).                    */
int gpw_operator_relax(gpw_operator *op, int dtype, int relax_method,
                       void *func, const void *source, int64_t nin,
                       int nrelax, double w, gpw_stream stream);

/* Operator.get_diagonal_element(), c/operators.c:408-421.                   */
int gpw_operator_get_diagonal_element(const gpw_operator *op, double *out);

/* Fused residual r = A func - source and sum |r|^2 (new; replaces the
 * apply + `residual -= rho` + np.dot sequence of gpaw/poisson.py:357-361).
 * r may be NULL (norm only).  sumsq_dev points to `nin` device doubles;
 * each receives its grid's sum |r|^2, reduced in a fixed order.            */
int gpw_operator_residual(gpw_operator *op, int dtype, const void *func,
                          const void *source, void *r, int64_t nin,
                          double *sumsq_dev, gpw_stream stream);

/* Allocation-free gpw_operator_residual (no counterpart in the reference).
 * For callers that must not allocate device memory during a call -- code
 * running inside another framework's memory pool or allocator hook, or a
 * process that reserves all device memory up front: the partial sums of the
 * norm reduction live in a fixed 540,672-byte (~528 KB) array compiled into
 * the library
 * (resident on every GPU that loads it until exit) instead of a workspace
 * grown with cudaMalloc.  Same arguments and results as
 * gpw_operator_residual.  Limits: nin <= 4096 grids and at most 65536
 * reduction blocks per call (blocks x nin), else GPW_EINVAL.  The first call
 * on a device looks the array's address up (keep that call outside stream
 * capture).  Calls share the array: calls that overlap on the GPU race.     */
int gpw_operator_residual_noalloc(gpw_operator *op, int dtype, const void *func,
                                  const void *source, void *r, int64_t nin,
                                  double *sumsq_dev, gpw_stream stream);

void gpw_operator_free(gpw_operator *op);

/* ------------------------------------------------------- weighted operator */

/* Replaces _gpaw.WOperator(nweights, weights, coefs, offsets, size, range,
 * neighbors, real, comm, cfd), c/woperators.c:497-588, built by
 * gpaw/wfd_operators.py:8-76: A = sum_i w_i(r) S_i with nweights <= 4
 * stencils S_i (coefs[i], linear offsets[i] into the range-padded array,
 * ncoefs[i] <= 40 taps, offsets[i][0] == 0).  The weight grids are not held
 * by the operator: every call passes the nweights device pointers (one
 * float64 grid each), so a caller that updates them in place (as the
 * dielectric solver restricts them to the coarse levels) is always seen.  */
int gpw_woperator_new(int nweights, const double *const *coefs,
                      const int64_t *const *offsets, const int *ncoefs,
                      const int64_t size[3], int range,
                      const int64_t neighbors[6], int real, int cfd,
                      gpw_woperator **out);
/* WOperator.apply(input, output, phases), c/woperators.c:362-465 with
 * c/bmgs/wfd.c: float64 or complex128 grids, `in` may equal `out`.  The
 * reference's nin > 1 reads each grid's weights past the end of the weight
 * arrays; here every grid of the call uses the same weights.              */
int gpw_woperator_apply(gpw_woperator *op, int dtype,
                        const double *const *weights, const void *in,
                        void *out, int64_t nin, const double *phases,
                        gpw_stream stream);
/* WOperator.relax(relax_method, func, source, nrelax, w),
 * c/woperators.c:61-108 with c/bmgs/wrelax.c: weighted Gauss-Seidel (1) or
 * Jacobi (2) on one float64 grid, in place.                               */
int gpw_woperator_relax(gpw_woperator *op, int relax_method,
                        const double *const *weights, double *func,
                        const double *source, int nrelax, double w,
                        gpw_stream stream);
/* WOperator.get_diagonal_element(), c/woperators.c:466-496: the largest
 * |sum_i w_i(r) c_i0| over the grid (blocks until it is known).           */
int gpw_woperator_get_diagonal_element(gpw_woperator *op,
                                       const double *const *weights,
                                       double *out, gpw_stream stream);
void gpw_woperator_free(gpw_woperator *op);

/* ------------------------------------------------------------ transformer */

/* Replaces _gpaw.Transformer(size_in, size_out, k, paddings, npaddings, skip,
 * neighbors, real, comm, interpolate), c/transformers.c:219-262 (built by
 * gpaw/transformers.py:71-76).  k = 2 nn in {2, 4, 6, 8}; paddings,
 * npaddings, skip and neighbors are (3, 2) tables as the reference computes
 * them (gpaw/transformers.py:31-54).                                        */
int gpw_transformer_new(const int64_t size_in[3], const int64_t size_out[3],
                        int k, const int64_t paddings[6],
                        const int64_t npaddings[6], const int64_t skip[6],
                        const int64_t neighbors[6], int real, int interpolate,
                        gpw_transformer **out);

/* Transformer.apply(input, output, phases), c/transformers.c:127-185:
 * halo fill then restriction (c/bmgs/restrict.c:137-154) or interpolation
 * (c/bmgs/interpolate.c:141-168) of `nin` grids.                            */
int gpw_transformer_apply(gpw_transformer *tr, int dtype, const void *in,
                          void *out, int64_t nin, const double *phases,
                          gpw_stream stream);

/* out = base - I(in) for an interpolating transformer: the interpolation
 * and the subtraction that follows it (gpaw/poisson.py:351-352 `phis -=
 * residual`, gpaw/preconditioner.py:49-50 `d1 -= q1`) in one pass; `base`
 * has the output's shape and must not alias `out`.                         */
int gpw_transformer_apply_subtract(gpw_transformer *tr, int dtype,
                                   const void *in, const void *base,
                                   void *out, int64_t nin,
                                   const double *phases, gpw_stream stream);

void gpw_transformer_free(gpw_transformer *tr);

/* ------------------------------------------------------------ grid BLAS */
/* The NumPy / BLAS glue around the hot path (gpaw/utilities/blas.py axpy,
 * scal; gpaw/grid_descriptor.py:263-292 integrate) as device kernels.
 * n counts elements of `dtype`.                                             */

/* y = alpha * x + y   (complex alpha as (re, im); imaginary part ignored for
 * real dtypes)                                                              */
int gpw_axpy(int dtype, int64_t n, double alpha_re, double alpha_im,
             const void *x, void *y, gpw_stream stream);
/* x = alpha * x                                                             */
int gpw_scal(int dtype, int64_t n, double alpha_re, double alpha_im, void *x,
             gpw_stream stream);
/* out[m] = sum_i x[m, i] for m < nvec vectors of length n (real dtypes; for
 * complex dtypes out holds (re, im) pairs).  Deterministic order.          */
int gpw_sum(int dtype, int64_t nvec, int64_t n, const void *x, double *out_dev,
            gpw_stream stream);
/* out[m] = sum_i conj(x[m, i]) y[m, i] (real part only for complex).        */
int gpw_dot(int dtype, int64_t nvec, int64_t n, const void *x, const void *y,
            double *out_dev, gpw_stream stream);
/* gd.integrate(a_xg, b_yg), gpaw/grid_descriptor.py:294-319 (the gemm with
 * transa 'c' it calls): out[ix * ny + iy] = sum_i conj(x[ix, i]) y[iy, i] for
 * every pair of nx x-vectors and ny y-vectors of length n.  Real dtypes give
 * one double per pair, complex dtypes a (re, im) pair.  nx * ny <= 65535.
 * Deterministic order.                                                      */
int gpw_dotc_pairs(int dtype, int64_t nx, int64_t ny, int64_t n, const void *x,
                   const void *y, double *out_dev, gpw_stream stream);
/* dst[dst_off + i] = src[src_off + i] over a box of contiguous (n0, n1, n2)
 * grids: the array copies of extend_array / deextend_array
 * (gpaw/utilities/extend_grid.py:46-56, grid2grid with an offset) for the
 * extended Poisson solver.                                                */
int gpw_copy_box(int dtype, const void *src, const int64_t src_n[3],
                 const int64_t src_off[3], void *dst, const int64_t dst_n[3],
                 const int64_t dst_off[3], const int64_t box[3],
                 gpw_stream stream);
/* out = x * y elementwise, float64 (the NumPy products rho * mask_g of
 * gpaw/poisson_extended.py:214).                                          */
int gpw_mul(int64_t n, const double *x, const double *y, double *out,
            gpw_stream stream);
/* y = x + c (real dtypes, c added to every element)                         */
int gpw_add_scalar(int dtype, int64_t n, double c, const void *x, void *y,
                   gpw_stream stream);

/* ------------------------------------------------------------ autotuner */

/* The launch choices the autotuners made so far in this process (tile
 * variants and chunkings of the zero-boundary TMA stencil kernel, layouts of
 * the periodic / Bloch row kernel, per element type, radius, epilogue, grid
 * and batch) as text: a header naming the device and its SM count, then
 * one record a line.  No counterpart in the reference (which has no
 * autotuner).  Writes at most cap bytes (NUL included) and sets *needed;
 * buf NULL only queries the size.                                          */
int gpw_tune_export(char *buf, int64_t cap, int64_t *needed);
/* Merge records written by gpw_tune_export into the tuners, so that a new
 * process skips timing the shapes already tuned.  Records from another
 * device or SM count are refused (GPW_EINVAL); records whose layout is not
 * available for their shape are skipped.  *imported (may be NULL) receives
 * the number of records taken.                                             */
int gpw_tune_import(const char *text, int *imported);

/* ------------------------------------------------------------ Poisson */

/* The charge branches of PoissonSolver.solve, gpaw/poisson.py:209-299, for
 * nb float64 (rho, phi) pairs of n points each, on the device with no host
 * round trip: charge = sum(rho) dv; neutral (|charge| <= maxcharge) or all
 * axes periodic: rho_out = rho - charge / dv / npts_global (charged periodic
 * with zero_initial_phi: phi = 0); charged with no periodic axis and the
 * Gaussian arrays given: q = charge / sqrt(4 pi), rho_out = rho - q rho_gauss,
 * phi -= q phi_gauss (or phi = 0).  q_dev[b] receives q (0 outside the
 * Gaussian branch; NaN for a charged member with mixed boundaries, which
 * the caller reports as the reference's NotImplementedError).  pbc_mask bit
 * c set = axis c periodic.  After the neutral solve on rho_out,
 * gpw_poisson_charge_finish adds q phi_gauss back (poisson.py:298-299).     */
int gpw_poisson_charge_prepare(int64_t nb, int64_t n, const double *rho,
                               double *rho_out, double *phi,
                               const double *rho_gauss,
                               const double *phi_gauss, double dv,
                               double npts_global, double maxcharge,
                               int pbc_mask, int zero_initial_phi,
                               double *q_dev, gpw_stream stream);
int gpw_poisson_charge_finish(int64_t nb, int64_t n, double *phi,
                              const double *phi_gauss, const double *q_dev,
                              gpw_stream stream);

/* Multigrid engine behind FDPoissonSolver (gpaw/poisson.py:61-366).  The
 * level hierarchy is the one gpaw/poisson.py:91-132 builds: operators[0..L]
 * (level 0 the caller's Laplacian, coarse levels nn=1), restrictors[0..L-1]
 * (level l -> l+1) and interpolators[0..L-1] (level l+1 -> l), smoothing
 * counts presmooths/postsmooths[0..L] and Jacobi weights[0..L] (schedule of
 * gpaw/poisson.py:111-128, 191-192).  The handles must outlive the engine.
 * nbatch_max: largest number of independent same-grid solves per call.      */
int gpw_poisson_new(int nlevels, gpw_operator *const *operators,
                    gpw_transformer *const *restrictors,
                    gpw_transformer *const *interpolators,
                    const int *presmooths, const int *postsmooths,
                    const double *weights, int relax_method, double dv,
                    int64_t nbatch_max, gpw_poisson **out);

/* solve_neutral + iterate2 (gpaw/poisson.py:306-366) for `nbatch`
 * independent grids phi[b], rho[b] (device, float64, contiguous n_c):
 * V-cycles until error = sum r^2 dv <= eps[b] or niter == maxiter.
 * precision 0: plain float64 V-cycles (the reference's method).
 * precision 1: float32 V-cycles inside a float64 defect-correction loop
 *              (float64 residual, update and norms).
 * Writes niter[b] and the final error[b] (host arrays).  Synchronises the
 * stream.  Returns GPW_ECONV if any solve reached maxiter.                  */
int gpw_poisson_solve(gpw_poisson *ps, double *phi, const double *rho,
                      int64_t nbatch, const double *eps, int maxiter,
                      int precision, int *niter, double *error,
                      gpw_stream stream);

/* The same solve enqueued on `stream` without waiting for it (no
 * counterpart in the reference): for callers that overlap host transfers
 * or other work with solves.  The per-solve results land in mailbox `slot`
 * (0 or 1) and are read by gpw_poisson_collect after the caller has seen
 * the stream's work finish (an event or a stream synchronisation); a slot
 * is not reused before its solve has been collected.  Needs the device-side
 * loop (GPW_ENOTSUP where conditional graph nodes are unavailable).        */
int gpw_poisson_solve_async(gpw_poisson *ps, double *phi, const double *rho,
                            int64_t nbatch, const double *eps, int maxiter,
                            int precision, int slot, gpw_stream stream);

/* Reads the per-solve results of a finished asynchronous solve from mailbox
 * `slot`: niter[b], error[b]; GPW_ECONV if any solve reached maxiter.       */
int gpw_poisson_collect(gpw_poisson *ps, int64_t nbatch, int maxiter,
                        int precision, int slot, int *niter, double *error);

/* Several engines (e.g. one per grid size) solved by ONE graph launch (no
 * counterpart in the reference, which solves one grid per call): each
 * engine's convergence loop runs on the device as a conditional while node
 * of one parent graph, the loops being independent branches that run
 * concurrently.  Arguments per engine i as in gpw_poisson_solve (phis[i],
 * rhos[i]: nbatch[i] grids of that engine's shape).  The graph is built on
 * the first call for a set of (engines, batch sizes, precision) and reused.
 * Synchronises the stream; GPW_ECONV if any solve reached maxiter.          */
int gpw_poisson_solve_many(int nengines, gpw_poisson *const *engines,
                           double *const *phis, const double *const *rhos,
                           const int64_t *nbatch, const double *const *eps,
                           int maxiter, int precision, int *const *niters,
                           double *const *errors, gpw_stream stream);

/* Per-solve latency of the engine's last solve (milliseconds of device time
 * from the start of the iterations to the end of the iteration in which
 * each of the `nbatch` solves converged; for gpw_poisson_solve_many, from
 * the start of the one launch).  No counterpart in the reference.          */
int gpw_poisson_last_latency(gpw_poisson *ps, int64_t nbatch, double *ms,
                             gpw_stream stream);

/* Counters of the last gpw_poisson_solve call: device kernels launched
 * (graph kernel nodes x replays + direct launches) and graph replays.       */
int gpw_poisson_last_stats(const gpw_poisson *ps, int64_t *kernel_launches,
                           int64_t *graph_launches);

/* Times one level-0 kernel of the engine on its own buffers (contents are
 * overwritten; call between solves): `which` 0 = float64 Jacobi sweep,
 * 1 = float64 residual + norm, 2 = float32 Jacobi sweep, 3 = float32 sweep
 * adding into float64 phi (defect-correction update), 4 = float64 defect
 * (float32 rhs + norm, and the first sweep unless the next sweep forms it),
 * 5 = float32 residual (no norm), 6 = float32 residual restricted into
 * level 1 (rho and first sweep; the float32 form's level-0 residual
 * launch), 7 = float32 sweep reading the defect alone and forming the first
 * sweep's iterate itself (GPW_ENOTSUP where the plan does not use it).
 * `reps` launches between CUDA events
 * on `stream`; writes the mean milliseconds per launch and the algorithmic
 * bytes per launch (each compulsory read and write counted once).          */
int gpw_poisson_time_level0(gpw_poisson *ps, int64_t nbatch, int which,
                            int reps, double *ms_per_launch,
                            double *bytes_per_launch, gpw_stream stream);

/* Convergence loop driver of a Poisson engine (no counterpart in the
 * reference): on = 1 (default) runs the whole loop on the device as a
 * conditional graph node; on = 0 replays the iteration graph from the host,
 * one graph launch per outer iteration (the same kernels and results;
 * profilers that cannot look inside conditional graph nodes need it).     */
int gpw_poisson_set_device_loop(gpw_poisson *ps, int on);

/* Launch plan of the float32 form's inner V-cycles (no counterpart in the
 * reference): on = 1 (default) runs the level above the one-CTA coarse
 * levels (31^3 at N_c = 128) together with them as one launch of a
 * thread-block cluster per solve; on = 0 runs that level as separate
 * stencil and transfer launches.  The two plans sum the stencil terms in a
 * different order (results within float32 rounding of each other).       */
int gpw_poisson_set_cluster(gpw_poisson *ps, int on);

/* Launch plan of the float32 form (no counterpart in the reference):
 * on = 1 (default) computes the level-0 residual and restricts it into
 * level 1 (its rho and first Jacobi sweep) in one launch, without storing
 * the residual, lets (with two or more level-0 pre-sweeps) the second
 * pre-sweep read the float32 defect alone and form the first sweep's
 * iterate itself, so the float64 defect stores no iterate, and fuses the
 * residual and restriction of the coarser levels the same way where the
 * next level is a cluster or stencil level (not the one-CTA kernel's);
 * on = 2 keeps the level-0 plan and launches the coarser levels' residuals
 * and restrictions separately (identical values); on = 0 launches every
 * residual and restriction separately and stores the first iterate (the
 * level-0 inner corrections then differ from on = 1 by float32 rounding:
 * the fused second pre-sweep scales the stencil of the defect instead of
 * taking the stencil of the stored iterate).                              */
int gpw_poisson_set_fusion(gpw_poisson *ps, int on);

/* Programmatic dependent launch of the V-cycle's kernels (no counterpart in
 * the reference): on = 1 (default) lets each stencil / transfer / coarse
 * kernel be dispatched while its predecessor drains (the kernel waits for
 * the predecessor's results before touching memory); on = 0 launches them
 * strictly one after another.  Results are identical either way.
 * Process-wide; takes effect for graphs captured afterwards.              */
int gpw_set_pdl(int on);

/* Pins the tile variant of the TMA star-stencil kernels (no counterpart in
 * the reference): with variant >= 0 every later TMA stencil launch whose
 * element type and radius have that variant uses it, with `nchunk` axis-0
 * chunks (0 = the wave model, -1 = a balanced split of the tile columns'
 * planes over one CTA per resident slot -- the wave model for launches
 * that sum a norm --, < -1 = the model's count times -nchunk); variant -1
 * returns to the autotuned choice.  Variants 0-4 and 10 (48-wide
 * tiles) exist for both element types, 5-9 (4 points per thread) for float32
 * only.  Process-wide; meant for tests and tuning studies.  GPW_EINVAL
 * outside [-1, 10].                                                        */
int gpw_set_tma_variant(int variant, int nchunk);

/* Pins the tile layout of the star-stencil kernel that serves applies on
 * grids with a periodic axis (no counterpart in the reference): each shape
 * has up to 4 candidate layouts (a warp per row with 4 or 8 warps per CTA;
 * for complex rows wider than a warp, one point a lane with several warps
 * per row); k >= 1 pins the k-th (shapes with fewer keep the tuned one),
 * 0 returns to the tuned choice.  Process-wide; for tests and tuning
 * studies.  GPW_EINVAL outside [0, 16].                                   */
int gpw_set_bloch_layout(int k);

/* Launches of that kernel so far in this process (tests use it to see that
 * a shape took the kernel rather than the general one).                   */
int64_t gpw_bloch_launch_count(void);

/* Pins the kernel that serves restrictions (no counterpart in the
 * reference): 1 = the tile kernel (2D tiles with halos on both in-plane
 * axes), 2 / 3 = the row kernel (whole fine rows per plane, 384 / 192
 * threads a CTA; 8- or 16-byte elements with 16-byte rows and strides, else
 * the tile kernel), 0 = the launcher's choice.  Results are identical
 * either way.  Process-wide; for tests and tuning studies.  GPW_EINVAL
 * outside [0, 3].                                                          */
int gpw_set_restrict_layout(int k);

/* Launches of the row restriction kernel so far in this process.         */
int64_t gpw_restrict_rows_launch_count(void);

/* Inner V-cycle schedule of the float32 defect-correction form
 * (precision 1; no counterpart in the reference, whose only schedule is the
 * float64 one of gpaw/poisson.py:111-128, 191-192, which precision 0 keeps).
 * Level l runs npre[l] pre- and npost[l] post-smoothing weighted-Jacobi
 * sweeps, each with its own weight: `weights` lists, level by level,
 * npre[l] pre-sweep weights then npost[l] post-sweep weights (nweights =
 * the total).  The coarsest level runs only its post-sweeps.  Level 0 needs
 * at least one sweep of each kind; at most 16 sweeps per level.  Default
 * (never called): the reference schedule.                                   */
int gpw_poisson_set_inner_schedule(gpw_poisson *ps, const int *npre,
                                   const int *npost, const double *weights,
                                   int nweights);

/* Live per-launch breakdown of one iteration of the engine (a profiling aid
 * with no counterpart in the reference beyond its Timer): the iteration's
 * launches run eagerly on the engine's buffers (contents overwritten; call
 * between solves, after a solve of this batch size and precision), each
 * followed by a CUDA event; averaged over `reps` repetitions after one
 * warm-up.  Writes up to `cap` entries: NUL-separated labels into `labels`
 * (`labels_len` bytes), milliseconds into ms[], the entry count into
 * *count.  Synchronises the stream.                                        */
int gpw_poisson_profile_iteration(gpw_poisson *ps, int64_t nbatch,
                                  int precision, int reps, char *labels,
                                  int labels_len, double *ms, int cap,
                                  int *count, gpw_stream stream);

void gpw_poisson_free(gpw_poisson *ps);

/* ------------------------------------------------------------ learned warm start */
/* Kernels of the 3D convolutional U-Net that supplies the float32 solve's
 * initial potential (no counterpart in the reference).  Activations are
 * bf16 NDHWC ([B][D][H][W][C]), C in {16, 32, 64}; conv weights bf16
 * [27 taps][cout][cin] with tap = (kd * 3 + kh) * 3 + kw; accumulation and
 * every gradient reduction in fp32.  All calls are asynchronous on `stream`.*/

/* 3x3x3 convolution, stride 1, zero padding 1 (cross-correlation), on the
 * tensor cores: out = epilogue(conv(x, w) + bias + add); epilogue 0 linear,
 * 1 GELU (erf form; z, if non-null, receives the pre-activation).  bias
 * (fp32 [cout]) and add ([..][cout]) may be NULL.  The data gradient of a
 * convolution is this call on the output gradient with the weights of
 * gpw_nn_flip_weights (cin and cout swapped).                              */
int gpw_nn_conv3(int cin, int cout, int epilogue, const void *x,
                 const void *w, const float *bias, const void *add, void *z,
                 void *out, int B, int D, int H, int W, gpw_stream stream);
/* dw[27][cout][cin] (fp32) = sum over points of dz[p][co] x[p + tap][ci];
 * scratch: gpw_nn_wgrad_scratch(cin, cout) floats of partial sums.        */
int64_t gpw_nn_wgrad_scratch(int cin, int cout);
int gpw_nn_conv3_wgrad(int cin, int cout, const void *x, const void *dz,
                       float *dw, float *scratch, int64_t scratch_floats,
                       int B, int D, int H, int W, gpw_stream stream);
/* wt[tap][ci][co] = w[26 - tap][co][ci]                                     */
int gpw_nn_flip_weights(int cin, int cout, const void *w, void *wt,
                        gpw_stream stream);
/* dz = da * GELU'(z), n elements                                            */
int gpw_nn_gelu_backward(int64_t n, const void *z, const void *da, void *dz,
                         gpw_stream stream);
/* 2x2x2 average pooling of x (dims D, H, W, even) and its gradient
 * (dx (+)= dy / 8 on the children)                                         */
int gpw_nn_pool2(int c, const void *x, void *y, int B, int D, int H, int W,
                 gpw_stream stream);
int gpw_nn_pool2_backward(int c, const void *dy, void *dx, int B, int D,
                          int H, int W, int accumulate, gpw_stream stream);
/* y = nearest 2x upsampling of x (+ skip), y of dims D, H, W; gradient
 * dx (+)= sum of the 2x2x2 children of dy                                   */
int gpw_nn_upsample2_add(int c, const void *x, const void *skip, void *y,
                         int B, int D, int H, int W, gpw_stream stream);
int gpw_nn_upsample2_backward(int c, const void *dy, void *dx, int B, int D,
                              int H, int W, int accumulate, gpw_stream stream);
/* 1x1x1 head to one fp32 channel, c in {16, 64}: out[p] = w . x[p] + bias;
 * backward: dx (+)= w dout, dwb[0..c-1] = dw, dwb[c] = dbias (scratch:
 * gpw_nn_partials() * (c + 1) floats)                                       */
int gpw_nn_head(int c, int64_t npts, const void *x, const float *w,
                const float *bias, float *out, gpw_stream stream);
int gpw_nn_head_backward(int c, int64_t npts, const void *x, const float *w,
                         const float *dout, void *dx, int accumulate,
                         float *dwb, float *scratch, int64_t scratch_floats,
                         gpw_stream stream);
/* number of CTA partials of gpw_nn_mse / gpw_nn_head_backward              */
int gpw_nn_partials(void);
/* out[c] = sum over the npts points of x[p][c] (a bias gradient); scratch:
 * gpw_nn_partials() * c floats                                             */
int gpw_nn_channel_sum(int c, int64_t npts, const void *x, float *out,
                       float *scratch, int64_t scratch_floats,
                       gpw_stream stream);
/* x[B][N^3][16] bf16: channel 0 = rho[b] * scale[b] on the n^3 interior     */
int gpw_nn_pack_input(const double *rho, const double *scale, int B, int n,
                      int N, void *x, gpw_stream stream);
/* fine (+)= nearest f-fold upsampling of coarse (fp32, N^3 / (N/f)^3) and
 * its gradient (coarse = sum of the f^3 children)                           */
int gpw_nn_upsample_add_f32(int f, const float *coarse, float *fine, int B,
                            int N, gpw_stream stream);
int gpw_nn_downsum_f32(int f, const float *fine, float *coarse, int B, int N,
                       gpw_stream stream);
/* mean squared error on the n^3 interior: diff = pred - target * tscale[b];
 * dpred = d loss / d pred; partial[0..gpw_nn_partials()) sum to the loss    */
int gpw_nn_mse(const float *pred, const double *target, const double *tscale,
               int B, int n, int N, float *dpred, double *partial,
               int64_t partial_len, gpw_stream stream);
/* phi[b] (float64 n^3) = pred[b] * scale[b]                                 */
int gpw_nn_unpack_output(const float *pred, const double *scale, int B, int n,
                         int N, double *phi, gpw_stream stream);
/* Adam step `step` (1-based) on fp32 params; param_bf16 (may be NULL)
 * receives the updated values rounded to bf16                               */
int gpw_nn_adam(int64_t n, float *param, const float *grad, float *m,
                float *v, double lr, double b1, double b2, double eps,
                int step, void *param_bf16, gpw_stream stream);
/* Gaussian-sum densities on the device: rho[b][i0][i1][i2] = sum over k <
 * counts[b] of q (2 pi s^2)^(-3/2) exp(-|r - c|^2 / 2 s^2) at r = (index +
 * beg) h; params[b][k] = (cx, cy, cz, s, q), maxg entries per b.            */
int gpw_nn_gaussians(int B, int n, double h, double beg, int maxg,
                     const int *counts, const double *params, double *rho,
                     gpw_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* GPWGRID_H */
