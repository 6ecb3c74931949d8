/*
 * agb.h -- C ABI of the B200 evaluator for Agama-style galactic potentials.
 *
 * Plain C: device pointers, host pointers to small descriptor structs, sizes
 * and a CUDA stream passed as void*.  No torch or CuPy types.  Every function
 * returns 0 on success or a negative AGB_ERR_* code; agb_last_error() gives
 * a thread-local message for the last failure on the calling thread.
 *
 * Two families of entry points:
 *
 *  1. Kernel-signature entries (agb_multipole_*, agb_cylspl_*): one per
 *     reference kernel, same arguments in the same order and with the same
 *     meaning, plus a trailing stream.  They replace the CuPy RawKernel
 *     launches of the reference's wrapper one for one.  Outputs keep the
 *     reference's convention (gradient and Hessian of Phi, not force).
 *
 *  2. The fused entry agb_eval(): any composite of Multipole, CylSpline and
 *     analytic components, each seen through a Shifted/Scaled/Evolving
 *     transform ("leaf"), summed per point in one kernel launch.  This is what
 *     the Python PotentialGPU classes call.  It replaces the per-component
 *     launches plus CuPy elementwise glue of CompositePotentialGPU
 *     (gpu_potential.py:1439-1529), EvolvingPotentialGPU (:1536-1644),
 *     ShiftedPotentialGPU (:1651-1764) and ScaledPotentialGPU (:1767-1918).
 *
 * All positions, tables and outputs are FP64 and live in device memory unless
 * stated otherwise; the caller owns every buffer.
 */
#ifndef AGB_H
#define AGB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AGB_OK               0
#define AGB_ERR_ARG         -1   /* bad argument (null pointer, size, kind)  */
#define AGB_ERR_DEVICE      -2   /* CUDA error reported by the runtime       */
#define AGB_ERR_UNSUPPORTED -3   /* valid request this build cannot serve    */
#define AGB_ERR_TIMEOUT     -4   /* a bounded device wait gave up            */

/* evaluation modes */
#define AGB_MODE_POT   0   /* Phi                                     */
#define AGB_MODE_GRAD  1   /* Phi and grad Phi                        */
#define AGB_MODE_HESS  2   /* Phi, grad Phi and the Hessian           */
#define AGB_MODE_DENS  3   /* density = Laplacian(Phi) / (4 pi G)     */
#define AGB_MODE_VJP   4   /* dL/dx from dL/dPhi and dL/dF (agb_eval_vjp) */

/* arithmetic of the Multipole harmonic sums */
#define AGB_PREC_FP64  0   /* everything FP64                                      */
#define AGB_PREC_MIXED 1   /* FP32 Legendre/m-phi recurrences and spline polynomials,
                              FP64 for log r, interval index/offset, monopole,
                              extrapolation, per-|m| partial sums and the
                              composite sum                                       */

/* output flags for agb_eval */
#define AGB_OUT_NEGATE     1   /* write -grad (force) and -Hessian (forceDeriv layout) */
#define AGB_OUT_NO_BINNING 2   /* evaluate the points in input order (no scratch memory) */
#define AGB_OUT_BIN_ALWAYS 4   /* sort by interval even below AGB_BIN_MIN_POINTS points */
#define AGB_OUT_STAGE      32  /* batches (mixed precision, pre-sorted points): each
                                  tile's interval rows of the unit's keyed Multipole are
                                  bulk-copied (TMA, cp.async.bulk) into shared memory and
                                  read there */
/* batches with AGB_OUT_STAGE, for tests of the failure path of the bounded
   waits: every block gives up its first wait for a bulk copy at once, records the
   error (agb_batch_stage_errors then returns 1), waits for that copy to land
   (bounded) and reads global memory from then on: the results are those of the
   unstaged kernel */
#define AGB_OUT_STAGE_GIVE_UP (1 << 24)
/* Launch-shape knobs of the evaluation kernel.  Results do not depend on them;
   the autotuner (agama_gpu_b200/autotune.py) times them.  No counterpart in the
   reference, whose launch shape is fixed.
   bits 8-11:  blocks per resident slot of the grid, 1-15 (0: the default, one
               slot's worth above 2^21 points, two below).
   bits 12-13: threads per block: 0 = the default, 1 = 128, 2 = 512 (512 in the
               potential, force and density modes; the Hessian modes keep 256).
               The default is 256, except for calls of more than 2^21 points of a
               tree with a Multipole and no other shape bit set: force and density
               calls take 512 threads, one block per SM; Hessian calls 128 threads
               (and 16 points per thread in FP64).  Host-leaf calls of agb_eval / agb_eval_ws /
               agb_eval_static only.
   bits 16-19: points per thread p, 1-15: each block takes a contiguous range of
               threads x 2^(p-1) points and the grid grows with n (overrides
               bits 8-11; 0: off). */
#define AGB_OUT_GRID_SHIFT  8
#define AGB_OUT_GRID(w)     (((w) & 15) << AGB_OUT_GRID_SHIFT)
#define AGB_OUT_BLOCK_SHIFT 12
#define AGB_OUT_BLOCK(b)    (((b) & 3) << AGB_OUT_BLOCK_SHIFT)
#define AGB_OUT_PPT_SHIFT   16
#define AGB_OUT_PPT(p)      (((p) & 15) << AGB_OUT_PPT_SHIFT)

/* agb_eval sorts the points by the radial interval of its heaviest Multipole
   leaf (a counting sort in device scratch) when there are at least this many */
#define AGB_BIN_MIN_POINTS 16384

/* component kinds */
#define AGB_KIND_MULTIPOLE      1
#define AGB_KIND_CYLSPLINE      2
#define AGB_KIND_NFW           10
#define AGB_KIND_PLUMMER       11
#define AGB_KIND_HERNQUIST     12
#define AGB_KIND_DEHNEN        13
#define AGB_KIND_ISOCHRONE     14
#define AGB_KIND_MIYAMOTONAGAI 15
#define AGB_KIND_LOGHALO       16
#define AGB_KIND_DISKANSATZ    17
#define AGB_KIND_UNIFORMACC    18

/* Multipole table layouts (agb_component.layout) */
#define AGB_LAYOUT_HARMONIC_MAJOR 0  /* poly[(c*n_int + k)*6 + j]: the reference's layout */
#define AGB_LAYOUT_INTERVAL_MAJOR 1  /* poly[(k*n_lm + c)*6 + j]: one contiguous slab per
                                        radial interval                                  */

/* Multipole column structure (agb_component.structure) */
#define AGB_STRUCT_LIST 0
#define AGB_STRUCT_ALL  1
#define AGB_STRUCT_EVEN 2

#define AGB_MAX_LEAVES 32
#define AGB_MAX_COMPONENTS 24
#define AGB_MAX_LMAX 32

/*
 * One potential component.  Static for the life of its tables.
 *
 * MULTIPOLE  (tables from the quintic-spline builder, gpu_potential.py:408-631)
 *   table      FP64 poly, layout per `layout`
 *   table32    FP32 copy of the same polynomials (needed for AGB_PREC_MIXED),
 *              interval-major with 8-float records (a0..a5, 2 pads); with a
 *              regular structure each m>0 (cos, sin) column pair is one 16-float
 *              record, cos and sin interleaved: c0 s0 c1 s1 ... c5 s5, 4 pads
 *   lm         packed harmonic list, lm[c] = (l << 16) | (m & 0xffff), sorted by
 *              (|m|, l, cos before sin), lm[0] = (0,0)
 *   n_lm, n_int, lmax, log_scaling, layout
 *   structure  AGB_STRUCT_LIST: the columns are exactly the harmonics in lm;
 *              AGB_STRUCT_ALL / AGB_STRUCT_EVEN: the columns are every (l, m)
 *              with l <= lmax (every l, or even l only), ordered by (|m|, l,
 *              cos before sin), pruned harmonics present as zero columns; the
 *              kernel then walks the harmonics without reading lm; in these
 *              structures column (l, m) holds its coefficients multiplied by
 *              C_l^|m| = prod_{j=|m|+1..l} sqrt((4j^2 - 1) / (j^2 - m^2)) (both
 *              tables), the normalisation the kernels' rescaled Legendre
 *              recurrence leaves out
 *   p[0..9]    logr_min, dlogr, inv_dlogr, invPhi0, inner_s, inner_U, inner_W,
 *              outer_s, outer_U, outer_W
 * CYLSPLINE  (tables from gpu_potential.py:1143-1253, relaid per cell)
 *   table      cell-major nodes: ((iR*(nz-1) + iz)*n_lm + h)*16 doubles:
 *              {fval, fx, fy, fxy} at the (lo,lo), (lo,hi), (hi,lo), (hi,hi) corners
 *   lm         m of each harmonic h
 *   grid_a     lR grid [n_int], grid_b lz grid [nz], extra W_outer [(8+1)^2]
 *   n_lm = n_harm, n_int = nR, nz, log_scaling, lmax = lmax_outer
 *   p[0] Rscale, p[1] r0_outer, p[2] mmax_outer
 * Analytic kinds: p[] holds the profile parameters (see the Python layer).
 */
typedef struct agb_component {
    int32_t kind;
    int32_t n_lm;
    int32_t n_int;
    int32_t nz;
    int32_t lmax;
    int32_t log_scaling;
    int32_t layout;
    int32_t structure;
    const double*  table;
    const float*   table32;
    const int32_t* lm;
    const double*  grid_a;
    const double*  grid_b;
    const double*  extra;
    double p[16];
} agb_component;

/*
 * A component seen through the modifier chain at the evaluation time:
 *   Phi(x) += ampl * Phi_comp(sigma * x - gamma)
 *   grad   += ampl * sigma   * grad_comp
 *   Hessian/density += ampl * sigma^2 * (...)_comp
 * Shifted(c): sigma 1, gamma c.  Scaled(s=1/scale, a): sigma s, ampl a*s.
 * Evolving: the two bracketing snapshots with ampl (1-alpha) and alpha.
 */
typedef struct agb_leaf {
    int32_t comp;       /* index into the component array */
    int32_t reserved;
    double  sigma;
    double  gamma[3];
    double  ampl;
} agb_leaf;

/* ---- library ---- */
/* Live FMA throughput of the current GPU in TFLOP/s (precision AGB_PREC_FP64 ->
   FP64, AGB_PREC_MIXED -> FP32).  A measurement utility for roofline reports;
   no counterpart in the reference. */
int agb_measure_fma_peak(int precision, double* tflops, void* stream);

const char* agb_last_error(void);
const char* agb_version(void);
/* number of kernel launches issued by this library on the calling thread since
   the last reset (for launch accounting in benchmarks) */
int64_t agb_launch_count(void);
void    agb_launch_count_reset(void);

/*
 * Fused evaluation of a composite at N points.
 *   xyz   device, N x 3 row-major (x, y, z per point)
 *   phi   device [N]     (may be NULL in GRAD/HESS modes)
 *   grad  device [N*3]   (GRAD/HESS; may be NULL in HESS mode)
 *   hess  device [N*6]   [Hxx, Hyy, Hzz, Hxy, Hyz, Hxz] (HESS)
 *   rho   device [N]     (DENS)
 *   out_flags AGB_OUT_NEGATE: grad -> force, hess -> forceDeriv
 * Replaces the per-component launch chains listed in the file comment.
 */
int agb_eval(const agb_component* comps, int n_comps,
             const agb_leaf* leaves, int n_leaves,
             const double* xyz, int64_t n, int mode, int precision,
             double* phi, double* grad, double* hess, double* rho,
             int out_flags, void* stream);

/*
 * agb_eval with caller-provided device scratch for the interval sort (no
 * allocation inside).  workspace: 256-byte aligned, at least
 * agb_eval_workspace_bytes(...) bytes (0 when the call does not sort; then
 * workspace may be NULL).  The scratch is about 32 bytes per point.
 */
size_t agb_eval_workspace_bytes(const agb_component* comps, int n_comps,
                                const agb_leaf* leaves, int n_leaves, int64_t n,
                                int out_flags);
int agb_eval_ws(const agb_component* comps, int n_comps,
                const agb_leaf* leaves, int n_leaves,
                const double* xyz, int64_t n, int mode, int precision,
                double* phi, double* grad, double* hess, double* rho,
                int out_flags, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Points that one wave of the evaluator's resident threads holds on the current
 * device (SMs x resident blocks x 256) for the kernel this tree, mode and
 * precision select; 0 for bad arguments.  A call of n points with
 * AGB_OUT_GRID(1) takes ceil(n / wave) passes of its threads over the points, so
 * callers that split work into several calls (the pipelined host path) size the
 * calls in multiples of it.  No reference counterpart: the reference evaluates
 * one host array per call.
 */
int64_t agb_eval_wave_points(const agb_component* comps, int n_comps,
                             const agb_leaf* leaves, int n_leaves, int mode, int precision);

/*
 * Vector-Jacobian product of the composite w.r.t. positions (the backward of
 * a potential/force evaluation):  g_xyz = g_phi * grad(Phi) - H g_force,
 * H the Hessian of Phi (F = -grad Phi, dF/dx = -H).  One fused launch: every
 * component is evaluated with its Hessian and the contraction happens per
 * point, H is never written.  g_phi [N] and g_force [N,3] may be NULL (zero).
 * workspace as for agb_eval_ws (NULL: allocated stream-ordered inside).
 * No counterpart in the reference (it has no derivatives w.r.t. inputs).
 */
int agb_eval_vjp(const agb_component* comps, int n_comps,
                 const agb_leaf* leaves, int n_leaves,
                 const double* xyz, int64_t n, int precision,
                 const double* g_phi, const double* g_force, double* g_xyz,
                 void* workspace, size_t workspace_bytes, void* stream);

/*
 * agb_eval_vjp that also writes the force of the same leaves, F = -grad Phi,
 * into force [N,3] (assigned), from the per-point sums the VJP forms anyway.
 * A reverse-time adjoint uses it to step the trajectory backwards from a
 * checkpoint without a separate force evaluation.  No counterpart in the
 * reference.
 */
int agb_eval_vjp_force(const agb_component* comps, int n_comps,
                       const agb_leaf* leaves, int n_leaves,
                       const double* xyz, int64_t n, int precision,
                       const double* g_phi, const double* g_force, double* g_xyz,
                       double* force, void* workspace, size_t workspace_bytes,
                       void* stream);

/*
 * Gradient of a loss with respect to one Multipole leaf's quintic coefficients
 * (the table half of the backward): accumulates into g_table, laid out like the
 * component's interval-major FP64 table [n_int][n_lm][6], the sum over points
 * of dL/da_{c,k,j} for cotangents g_phi [N] (dL/dPhi) and g_force [N,3]
 * (dL/dF) of the composite's outputs; leaf gives the component's transform.
 * g_const (NULL, or AGB_MP_NCONST = 8 doubles, accumulated): the gradient with
 * respect to the scalars the table builder derives from the nodes -- invPhi0
 * (p[3]; from the points inside the grid), the inner s, U, W (p[4..6]; points
 * inside the first node) and, for the points beyond the last node, the outer
 * fit in the well-conditioned variables eps = s + 1, T = U eps, S = U + W of
 * (s, U, W) = p[7..9] (the fit is usually degenerate: s = -1 to rounding,
 * U ~ -W ~ 1e16) -- and 0.  FP64; points are sorted by interval in scratch
 * (workspace as for agb_eval_ws, NULL: allocated stream-ordered inside) and
 * each warp reduces its lanes before one atomic add per coefficient.
 * No counterpart in the reference.
 */
#define AGB_MP_NCONST 8
size_t agb_multipole_table_vjp_workspace_bytes(const agb_component* comp,
                                               const agb_leaf* leaf, int64_t n);
int agb_multipole_table_vjp(const agb_component* comp, const agb_leaf* leaf,
                            const double* xyz, int64_t n, const double* g_phi,
                            const double* g_force, double* g_table, double* g_const,
                            void* workspace, size_t workspace_bytes, void* stream);

/*
 * Fused adjoint of one Multipole leaf: one walk over the harmonics per point
 * ADDS this leaf's position VJP, A sigma (g_phi grad Phi - sigma H g_force),
 * into g_xyz [N,3] and accumulates the coefficient gradient into g_table as
 * agb_multipole_table_vjp does.  Needs a regular column structure
 * (AGB_STRUCT_ALL/EVEN).  precision: AGB_PREC_FP64 or AGB_PREC_MIXED (FP32
 * walk and warp reductions, FP64 accumulation).  Same workspace rules as
 * agb_multipole_table_vjp; with agb_multipole_adjoint_workspace_bytes() bytes
 * (with_force 1 for agb_multipole_adjoint_force) the per-point results are
 * written in sorted order and added back in input order by a second launch
 * instead of scattered read-modify-writes.  No counterpart in the reference.
 */
size_t agb_multipole_adjoint_workspace_bytes(const agb_component* comp, const agb_leaf* leaf,
                                             int64_t n, int with_force);
int agb_multipole_adjoint(const agb_component* comp, const agb_leaf* leaf,
                          const double* xyz, int64_t n, int precision,
                          const double* g_phi, const double* g_force, double* g_xyz,
                          double* g_table, double* g_const, void* workspace,
                          size_t workspace_bytes, void* stream);

/*
 * agb_multipole_adjoint that also ADDS this leaf's force, -A sigma grad Phi,
 * into force [N,3] (for the reverse-time adjoint, as agb_eval_vjp_force).
 * No counterpart in the reference.
 */
int agb_multipole_adjoint_force(const agb_component* comp, const agb_leaf* leaf,
                                const double* xyz, int64_t n, int precision,
                                const double* g_phi, const double* g_force,
                                double* g_xyz, double* force, double* g_table,
                                double* g_const, void* workspace, size_t workspace_bytes,
                                void* stream);

/*
 * One backward step of the leapfrog adjoint for a tree of one Multipole leaf
 * (mp_leaf, regular column structure) and analytic leaves, in two launches:
 * the fused Multipole adjoint (coefficient gradient added into g_table, its
 * per-point VJP and force kept in the workspace in sorted order), then per
 * particle the analytic leaves' VJP and force at x, the Multipole part added,
 *     lx += gx;  lv = fma(dt, lx, lv);  gF = c lv                    (the kick)
 * and with flags & AGB_ADJ_DRIFT the time-reversed drift with the total force
 *     vh = fma(-k, F, vh);  x = fma(-dt_drift, vh, x).
 * gF is read as the cotangent of the force at x and overwritten with c lv;
 * with flags & AGB_ADJ_LV_COT the cotangent is c_in lv (lv as it is on entry:
 * the c lv of the previous step) and gF is neither read nor written (it may
 * be null), which saves one [N,3] array's read and write per step.
 * The same arithmetic, in the same order, as agb_eval_vjp_force (analytic
 * leaves) + agb_multipole_adjoint_force + agb_adjoint_kick + agb_reverse_drift,
 * with two launches fewer and no intermediate gx / F arrays.  The workspace
 * (agb_adjoint_step_workspace_bytes, 256-byte aligned) is required.  No
 * counterpart in the reference.
 */
#define AGB_ADJ_DRIFT 1
#define AGB_ADJ_LV_COT 2
size_t agb_adjoint_step_workspace_bytes(const agb_component* comps, int n_comps,
                                        const agb_leaf* leaves, int n_leaves, int mp_leaf,
                                        int64_t n, int flags);
int agb_adjoint_step(const agb_component* comps, int n_comps, const agb_leaf* leaves,
                     int n_leaves, int mp_leaf, int precision, double* x, double* vh,
                     double* lx, double* lv, double* gF, double* g_table, double* g_const,
                     int64_t n, double dt, double c, double c_in, double k, double dt_drift,
                     int flags, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Leapfrog adjoint, per-step vector updates on [N,3] device arrays (one launch each):
 *   agb_adjoint_kick:  lx += gx;  lv += dt lx;  gF = c lv
 *   agb_reverse_drift: vh -= k F; x -= dt vh     (the time-reversed drift)
 * No counterpart in the reference (it has no integrator).
 */
int agb_adjoint_kick(double* lx, double* lv, const double* gx, double* gF, int64_t n,
                     double dt, double c, void* stream);
int agb_reverse_drift(double* x, double* vh, const double* F, int64_t n, double k,
                      double dt, void* stream);

/*
 * Gradient of a loss with respect to one CylSpline leaf's node table: adds into
 * g_cells, laid out like the component's cell-major FP64 table
 * [(nR-1)(nz-1)][n_harm][16] (each cell record holds its four corners' f, f_R,
 * f_z, f_Rz, so a node's gradient is the sum over the up to four records that
 * hold it), the sum over points of dL/dv for cotangents g_phi [N] and g_force
 * [N,3] of the composite's outputs; leaf gives the component's transform.
 * Points outside the grid contribute nothing (the outer asymptote and Rscale
 * are held fixed).  FP64, no scratch.  No counterpart in the reference.
 */
int agb_cylspline_table_vjp(const agb_component* comp, const agb_leaf* leaf,
                            const double* xyz, int64_t n, const double* g_phi,
                            const double* g_force, double* g_cells, void* stream);

/*
 * agb_eval_static -- agb_eval that allocates nothing.  No counterpart in the
 * reference: it exists for callers that may not allocate device memory (a
 * code that reserved the GPU for its own pools, a loop that must not pay
 * cudaMalloc's device synchronisation, a C/Fortran caller that only passes
 * arrays it owns).  The point-sorting scratch is a fixed 32 MiB device array
 * inside this library (held on every GPU that loads it), so one call takes at
 * most AGB_STATIC_MAX_POINTS points; larger calls fail with
 * AGB_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * address (make it before any stream capture); after a device reset the next
 * call looks it up again.  All calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller.
 */
#define AGB_STATIC_SCRATCH_BYTES (32 * 1024 * 1024)
#define AGB_STATIC_MAX_POINTS 1000000
int agb_eval_static(const agb_component* comps, int n_comps,
                    const agb_leaf* leaves, int n_leaves,
                    const double* xyz, int64_t n, int mode, int precision,
                    double* phi, double* grad, double* hess, double* rho,
                    int out_flags, void* stream);

/*
 * Batched evaluation of many independent work units in ONE launch: unit u is a
 * potential (its leaves [unit_leaf_offsets[u], unit_leaf_offsets[u+1]) of
 * `leaves`, which index `comps`) evaluated at its own points, rows
 * [point_offsets[u], point_offsets[u+1]) of one shared xyz array.  The plan
 * uploads the descriptors once (it owns that device memory until
 * agb_batch_destroy) and cuts the units into tiles of at most tile_points
 * points (0: 4096), ordered by estimated cost, largest first.  agb_batch_eval
 * then launches one persistent kernel whose blocks take tiles from a device
 * work queue (an atomic counter reset by a memset node before the launch), so
 * a call makes no host-side copies or allocations.  One plan serves one stream
 * at a time (the queue counter is per plan).  Modes POT/GRAD/HESS/DENS; the
 * precision is fixed per plan.  Results equal per-unit agb_eval calls point by
 * point.  Replaces the per-potential launch loop a caller of the reference
 * writes around gpu_potential.py:826-935 (one call per potential and point
 * set); the reference has no batched entry point.
 */
typedef struct agb_batch agb_batch;
int agb_batch_create(const agb_component* comps, int n_comps,
                     const agb_leaf* leaves, const int32_t* unit_leaf_offsets, int n_units,
                     const int64_t* point_offsets, int precision, int tile_points,
                     agb_batch** out);
int agb_batch_eval(const agb_batch* plan, const double* xyz, int mode,
                   double* phi, double* grad, double* hess, double* rho,
                   int out_flags, void* stream);
int64_t agb_batch_points(const agb_batch* plan);
int     agb_batch_tiles(const agb_batch* plan);
void    agb_batch_destroy(agb_batch* plan);

/*
 * agb_batch_eval with a caller-owned device workspace (256-byte aligned) that
 * turns on a device-wide pre-sort: every unit's points are counting-sorted by
 * the radial interval of the unit's heaviest Multipole, each unit within its own
 * rows, so that a tile is a run of sorted points spanning a few intervals and
 * the kernel's table reads hit L1 (the in-tile sort is then skipped).  Three
 * small launches before the kernel.  agb_batch_workspace_bytes(plan, mode) is
 * the size that also holds sorted-order output records (gathered back by one
 * more launch, every output array written contiguously); a workspace of at
 * least the pre-sort's own part (32 bytes per point plus the bin counters) but
 * smaller makes the kernel write each point's outputs in place.  Returns 0 when
 * the plan cannot be pre-sorted (a unit with more than 8190 intervals); a null
 * workspace is agb_batch_eval.  Results equal agb_batch_eval's bit for bit.
 */
size_t  agb_batch_workspace_bytes(const agb_batch* plan, int mode);
/*
 * The pre-sort's permutation alone: perm[pos] = the row at sorted position pos
 * (each unit's rows ordered by the radial interval of its sort key, inside the
 * unit's own rows).  A caller that keeps its particle arrays in this order (an
 * integrator between re-sorts) evaluates them with AGB_OUT_NO_BINNING in out_flags:
 * the rows are then visited in order, with no pre-sort, no in-tile sort and no
 * workspace.  Workspace: agb_batch_sort_workspace_bytes(plan) bytes, 256-byte
 * aligned.  Results do not depend on the order.
 */
size_t  agb_batch_sort_workspace_bytes(const agb_batch* plan);
/* 1 when a staged launch (AGB_OUT_STAGE) of this plan gave up waiting for one of its
   bulk copies and read global memory instead (results are unaffected); 0 otherwise;
   -1 on error.  Synchronous. */
int     agb_batch_stage_errors(const agb_batch* plan);
int     agb_batch_sort(const agb_batch* plan, const double* xyz, int32_t* perm,
                       void* workspace, size_t workspace_bytes, void* stream);
int     agb_batch_eval_ws(const agb_batch* plan, const double* xyz, int mode,
                          double* phi, double* grad, double* hess, double* rho,
                          int out_flags, void* workspace, size_t workspace_bytes,
                          void* stream);

/*
 * Time-dependent leaves evaluated on the device.  The reference evaluates the
 * Shifted centre, the Scaled factors and the Evolving bracket on the host at
 * every call (gpu_potential.py:1716-1734, :1845-1871, :1559-1612), so the
 * time is a host value baked into every launch.  A time plan instead holds, per
 * leaf slot, a program of modifier operations and their tables (splines as
 * breakpoints and cubic coefficients, snapshot times) in device memory; a small
 * kernel turns a device-resident step counter into the leaves at
 *     t = (t0 + step * dt) + off
 * right before the evaluation kernel, so a sequence of launches can be captured
 * once in a CUDA graph and replayed at every step.  The device arithmetic is
 * that of the host path operation by operation (no contraction into FMA, the
 * spline evaluated as sum c_k s^k with s^k by repeated multiplication, the
 * bracket by the same bisection), so the leaves equal the host's bit for bit.
 * No counterpart in the reference.
 *
 * A program starts from (comp, sigma 1, gamma 0, ampl 1) and applies its ops,
 * innermost modifier first:
 *   AGB_OP_SHIFT   gamma += sigma * c(t)
 *   AGB_OP_SCALE   (s, a) = (1/scale(t), ampl(t)); sigma *= s; ampl = (a*s)*ampl
 *   AGB_OP_EVOLVE  bracket t in the snapshot times: comp += chosen snapshot,
 *                  ampl *= its weight; slot 0 takes the lower snapshot with
 *                  weight 1-alpha (1 at alpha 0, 0 at alpha 1), slot 1 the
 *                  upper with alpha; with interpolation off (or one snapshot)
 *                  slot 0 takes the nearest with weight 1
 * Table data at arg[k] (doubles):
 *   SHIFT   [0, cx, cy, cz] (static) or
 *           [1, T, t0, tN, p0[3], pN[3], v0[3], vN[3], x[T], c[4][T-1][3]]
 *   SCALE   [0, scale, ampl] (static) or
 *           [1, T, t0, tN, scale0, scaleN, dscale0, dscaleN, has_ampl, ampl,
 *            ampl0, amplN, dampl0, damplN, x[T], cs[4][T-1] (, ca[4][T-1])]
 *   EVOLVE  [n, interpolate, times[n]]
 * (c: cubic coefficients, highest power first, of the centre, scale and
 * amplitude splines; outside [t0, tN] a spline is extended linearly from its
 * end value and slope.)  pair = 1 lets this slot and the next share one
 * harmonic walk (both Multipoles of one grid and column structure, the same
 * transform), as agb_eval does for the two snapshots of an Evolving.
 */
#define AGB_OP_SHIFT  1
#define AGB_OP_SCALE  2
#define AGB_OP_EVOLVE 3
#define AGB_MAX_LEAF_OPS 6

typedef struct agb_leaf_prog {
    int32_t comp;                     /* component index (EVOLVE: of snapshot 0) */
    int32_t n_ops;
    int32_t op[AGB_MAX_LEAF_OPS];     /* AGB_OP_*, innermost first */
    int32_t arg[AGB_MAX_LEAF_OPS];    /* offset of the op's data in the table */
    int32_t slot;                     /* EVOLVE: 0 lower / nearest, 1 upper */
    int32_t pair;
} agb_leaf_prog;

typedef struct agb_time_plan agb_time_plan;
/* validates the programs against the table (host arrays) and copies both to
   the current device (one allocation, owned by the plan) */
int agb_time_plan_create(const agb_leaf_prog* progs, int n_progs, const double* table,
                         int64_t n_table, agb_time_plan** out);
void agb_time_plan_destroy(agb_time_plan* plan);
/* the same programs evaluated on the host at time t (the device kernel's
   arithmetic, for checking): leaves[n_progs] */
int agb_time_plan_leaves_host(const agb_time_plan* plan, double t, agb_leaf* leaves);
/* the device leaves at t = (t0 + (*step) * dt) + off, written to leaves_dev
   [n_progs] (device); step is a device int64 (NULL: step 0) */
int agb_time_plan_leaves(const agb_time_plan* plan, const int64_t* step, double t0, double dt,
                         double off, agb_leaf* leaves_dev, void* stream);
/*
 * agb_eval_ws with the plan's leaves at t = (t0 + (*step) * dt) + off computed on
 * the device in the same stream: no host value of t enters a launch.  The
 * workspace (agb_eval_timed_workspace_bytes) holds the device leaves and the
 * interval-sort scratch.
 */
size_t agb_eval_timed_workspace_bytes(const agb_component* comps, int n_comps,
                                      const agb_time_plan* plan, int64_t n, int out_flags);
int agb_eval_timed(const agb_component* comps, int n_comps, const agb_time_plan* plan,
                   const int64_t* step, double t0, double dt, double off,
                   const double* xyz, int64_t n, int mode, int precision,
                   double* phi, double* grad, double* hess, double* rho, int out_flags,
                   void* workspace, size_t workspace_bytes, void* stream);

/*
 * Leapfrog vector updates of one (sub)step boundary, one launch, in place:
 *   v = fma(h1, F, v)   if flags & 1   (closing half-kick of the last substep)
 *   v = fma(h2, F, v)   if flags & 2   (opening half-kick of the next one)
 *   x = fma(dt, v, x)   if flags & 4   (drift)
 *   (*step)++           if flags & 8   (step counter of agb_eval_timed; thread 0)
 * x, v, F are [n, 3] device arrays.  No counterpart in the reference (it has no
 * integrator).
 */
int agb_leapfrog_kick_drift(double* x, double* v, const double* F, int64_t n, double h1,
                            double h2, double dt, int flags, int64_t* step, void* stream);

/*
 * Kernel-signature entries.  Arguments are those of the reference kernels, in
 * order, with SoA x, y, z device arrays, the reference's harmonic-major poly
 * layout and lm_l/lm_m arrays sorted as gpu_potential.py:516 sorts them.
 *   agb_multipole_potential  replaces multipole_potential_kernel
 *                            (_multipole_potential_kernel.cu:415-434)
 *   agb_multipole_force      replaces multipole_force_kernel (:436-455)
 *   agb_multipole_hess       replaces multipole_hess_kernel (:466-800)
 *   agb_multipole_density    replaces multipole_density_kernel (:809-958)
 */
int agb_multipole_potential(const double* x, const double* y, const double* z,
        const double* poly, double logr_min, double dlogr, double inv_dlogr,
        int n_intervals, int n_lm, int lmax, const int* lm_l, const int* lm_m,
        int log_scaling, double invPhi0, double inner_s, double inner_U, double inner_W,
        double outer_s, double outer_U, double outer_W,
        double* phi_out, double* grad_out, int N, void* stream);
int agb_multipole_force(const double* x, const double* y, const double* z,
        const double* poly, double logr_min, double dlogr, double inv_dlogr,
        int n_intervals, int n_lm, int lmax, const int* lm_l, const int* lm_m,
        int log_scaling, double invPhi0, double inner_s, double inner_U, double inner_W,
        double outer_s, double outer_U, double outer_W,
        double* phi_out, double* grad_out, int N, void* stream);
int agb_multipole_hess(const double* x, const double* y, const double* z,
        const double* poly, double logr_min, double dlogr, double inv_dlogr,
        int n_intervals, int n_lm, int lmax, const int* lm_l, const int* lm_m,
        int log_scaling, double invPhi0, double inner_s, double inner_U, double inner_W,
        double outer_s, double outer_U, double outer_W,
        double* phi_out, double* grad_out, double* hess_out, int N, void* stream);
int agb_multipole_density(const double* x, const double* y, const double* z,
        const double* poly, double logr_min, double dlogr, double inv_dlogr,
        int n_intervals, int n_lm, int lmax, const int* lm_l, const int* lm_m,
        int log_scaling, double invPhi0, double inner_s, double inner_U, double inner_W,
        double outer_s, double outer_U, double outer_W, double inv_4piG,
        double* rho_out, int N, void* stream);

/*
 *   agb_cylspl_potential  replaces cylspl_potential_kernel (_cylspl_potential_kernel.cu:871-899)
 *   agb_cylspl_force      replaces cylspl_force_kernel (:902-935)
 *   agb_cylspl_hess       replaces cylspl_hess_kernel (:938-972)
 * node_arr is the reference's layout [(mm*nR + iR)*nz + iz][4].
 */
int agb_cylspl_potential(const double* x, const double* y, const double* z,
        double Rscale, const double* lR_grid, int nR, const double* lz_grid, int nz,
        const double* node_arr, int n_harm, const int* m_arr, int mmax, int log_scaling,
        const double* W_outer, double r0_outer, int lmax_outer, int mmax_outer,
        double* phi_out, int N, void* stream);
int agb_cylspl_force(const double* x, const double* y, const double* z,
        double Rscale, const double* lR_grid, int nR, const double* lz_grid, int nz,
        const double* node_arr, int n_harm, const int* m_arr, int mmax, int log_scaling,
        const double* W_outer, double r0_outer, int lmax_outer, int mmax_outer,
        double* phi_out, double* grad_out, int N, void* stream);
int agb_cylspl_hess(const double* x, const double* y, const double* z,
        double Rscale, const double* lR_grid, int nR, const double* lz_grid, int nz,
        const double* node_arr, int n_harm, const int* m_arr, int mmax, int log_scaling,
        const double* W_outer, double r0_outer, int lmax_outer, int mmax_outer,
        double* phi_out, double* grad_out, double* hess_out, int N, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AGB_H */
