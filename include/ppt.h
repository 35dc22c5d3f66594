/*
 * ppt.h -- C ABI of libppt.so, the B200 (sm_100a) particle pusher with fused
 * trilinear E/B field-map interpolation.
 *
 * Every entry point returns an int status (PPT_OK = 0, negative PPT_ERR_*),
 * never throws, and leaves a thread-local message for ppt_last_error().
 * Device work is ordered on the caller's stream (a cudaStream_t passed as
 * void*; NULL = the legacy default stream).  All particle arrays, snapshot
 * buffers and outputs are caller-owned DEVICE memory; the library never frees
 * them.  Field maps are library-owned device copies behind an opaque handle.
 *
 * Reference interfaces each group replaces (DanielWinklehner/PyPATools,
 * paths inside that project):
 *   ppt_fieldmap_*  Field.from_arrays / get_interpolator / NumbaInterpolator
 *                   construction (src/PyPATools/field.py:345-387,
 *                   src/PyPATools/field_src/interpolators.py:299-347, :533-610)
 *   ppt_field_eval  Field.__call__ -> _get_field_3d -> NumbaInterpolator.__call__
 *                   -> _interp3d_batch (field.py:213-244, :491-504,
 *                   interpolators.py:349-402, :259-267, :88-135)
 *   ppt_track       Pusher.track_batch's step loop with push_batch and the
 *                   per-algorithm batch kernels (src/PyPATools/pusher.py:894-1012,
 *                   :699-801, :369-404, :803-892)
 *   ppt_state_*     the (M,3) float64 r/v arrays track_batch takes and returns
 *                   (pusher.py:934-962, :1012)
 *   ppt_moments     ParticleDistribution statistics (src/PyPATools/particles.py:
 *                   693-719, :761-788, :507-525, :393-457)
 *   ppt_deposit_cic PyAMGPoissonSolver's CIC charge deposition
 *                   (src/PyPATools/poisson_amg.py:849-911)
 *   ppt_poisson_*, ppt_field_from_potential  PyAMGPoissonSolver.solve's
 *                   linear solve and E = -grad phi (poisson_amg.py:616-797)
 *   ppt_surface_*   PyElectrodeAssembly.segment_intersects_surface, the collision
 *                   test track_batch makes each step (pusher.py:982-990; the
 *                   assembly comes from the external py_electrodes package)
 *   ppt_polar_to_cartesian  the RegularGridInterpolator resampling of the
 *                   cylindrical-map loaders (field_loaders.py:612-640, :836-899)
 *   ppt_cell_sort   no reference counterpart: particle reordering for gather
 *                   locality (the reference has no particle ordering step)
 *   ppt_restore_order  no reference counterpart: back to row order
 */
#ifndef PPT_H
#define PPT_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPT_ABI_VERSION 4

/* status codes */
#define PPT_OK               0
#define PPT_ERR_ARG         -1   /* bad argument (null pointer, size, enum) */
#define PPT_ERR_OOM         -2   /* device allocation failed */
#define PPT_ERR_CUDA        -3   /* a CUDA runtime call failed */
#define PPT_ERR_UNSUPPORTED -4   /* valid request this build does not handle */
#define PPT_ERR_TIMEOUT     -5   /* a bounded device wait expired */
#define PPT_ERR_DEVICE      -6   /* the device status word reported a fault */

/* Algorithms: the reference's Pusher.ALGORITHMS order (pusher.py:465-466),
 * then two additions that conserve |u| in a pure magnetic field. */
#define PPT_ALG_LEAPFROG     0
#define PPT_ALG_BORIS        1   /* non-relativistic Boris, pusher.py:124-165 */
#define PPT_ALG_RK4          2
#define PPT_ALG_YOSHIDA      3
#define PPT_ALG_VAY_REL      4   /* the reference's 'vay_rel' as written, pusher.py:216-279 */
#define PPT_ALG_RK4_REL      5
#define PPT_ALG_YOSHIDA_REL  6
#define PPT_ALG_BORIS_REL    7   /* relativistic Boris in u = gamma v (addition) */
#define PPT_ALG_VAY          8   /* Vay (2008) as published (addition) */
#define PPT_ALG_COUNT        9

/* Precision forms */
#define PPT_PREC_F64    0   /* the reference method in float64 (the drop-in) */
#define PPT_PREC_MIXED  1   /* int cell + float32 offset, float32 gathers and
                               rotation, float-float velocity accumulation */

/* Element types */
#define PPT_DTYPE_F64 0
#define PPT_DTYPE_F32 1

/* Track flags */
#define PPT_TRACK_INIT   1   /* this call starts the track: Boris-family
                                half step back and record 0 */
#define PPT_TRACK_FINAL  2   /* this call ends the track: Boris-family final
                                half step, v of the last record overwritten */

/* Device status bits (OR-ed into *status) */
#define PPT_STATUS_NONFINITE  1  /* a particle's state became NaN/Inf */
#define PPT_STATUS_BOUNDS     2  /* a debug-build bounds check failed */
#define PPT_STATUS_RANGE      4  /* mixed form: a particle went 2^24 cells or more from the map
                                    (beyond the exact range of its float cell index) */

#define PPT_MAX_MAPS 4

typedef struct ppt_fieldmap ppt_fieldmap;   /* opaque */

/* Node grid of one map: n[d] >= 2 sorted node coordinates per axis, given
 * as HOST arrays (copied).  Node values are indexed [i][j][k] with k
 * fastest, the 'ij' meshgrid order NumbaInterpolator uses.
 * n[d] == 1 (axis[d] is then ignored and may be NULL): the map does not vary
 * along axis d and has no bounds on it -- the reference's 1D fields
 * (n = {1, 1, nz}, values along z) and 2D fields (n = {nx, ny, 1}), which
 * Field._get_field_1d / _get_field_2d evaluate at z and at (x, y)
 * (src/PyPATools/field.py:457-489).  At least one axis needs 2 nodes. */
typedef struct {
    int64_t n[3];
    const double* axis[3];
} ppt_grid_desc;

/* Create a zero-valued map on the current device.  has_e / has_b say which
 * fields it stores; store_dtype is PPT_DTYPE_F64 (plain form) or
 * PPT_DTYPE_F32 (mixed form, needs uniform axes).  The same as
 * ppt_fieldmap_create_masked with the mask 0x07, 0x38 or 0x3F. */
int ppt_fieldmap_create(const ppt_grid_desc* grid, int has_e, int has_b, int store_dtype,
                        ppt_fieldmap** out);

/* Field components, bit c of a component mask (c = Ex, Ey, Ez, Bx, By, Bz). */
#define PPT_COMP_EX 0x01
#define PPT_COMP_EY 0x02
#define PPT_COMP_EZ 0x04
#define PPT_COMP_BX 0x08
#define PPT_COMP_BY 0x10
#define PPT_COMP_BZ 0x20

/* Record layout a map storing the components of comp_mask uses: the
 * smallest of the layouts {Bz}, {Ez Bz}, {Ex Ey Ez}, {Bx By Bz}, {Ex Ey Bz},
 * {all six} that contains comp_mask, as a component mask.  Layouts of 1, 2
 * or 3 components store them packed in Ex..Bz order in records of 1, 2 or
 * 4 elements; the six-component layout is [Ex Ey Ez 0 | Bx By Bz 0].
 * Returns PPT_ERR_ARG for a mask that is 0 or above 0x3F. */
int ppt_fieldmap_layout(uint32_t comp_mask);

/* Create a zero-valued map storing only the components of comp_mask (laid
 * out as ppt_fieldmap_layout(comp_mask)): components that are identically
 * zero in every term of a field need neither storage nor gathers, and the
 * mixed-form kernels, compiled per layout, drop them from the arithmetic.
 * The mixed form needs the six-component layout when the fields have
 * constant parts (ppt_fields.e_const / b_const not zero). */
int ppt_fieldmap_create_masked(const ppt_grid_desc* grid, uint32_t comp_mask, int store_dtype,
                               ppt_fieldmap** out);

/* map += scale[c] * comp[c] for c in (Ex,Ey,Ez,Bx,By,Bz).  comp[c] is a
 * DEVICE pointer to an n[0]*n[1]*n[2] C-contiguous array of src_dtype, or
 * NULL (adds nothing); a component the map's layout does not store must be
 * NULL.  Used once per term of a composite / scaled field. */
int ppt_fieldmap_add(ppt_fieldmap* map, const void* const comp[6], const double scale[6],
                     int src_dtype, void* stream);

int ppt_fieldmap_destroy(ppt_fieldmap* map);

/* bytes of device memory held, and flags: bit0 has_e, bit1 has_b,
 * bit2 all axes uniform, bit3 float32 storage, bits 8-13 the layout's
 * component mask */
int ppt_fieldmap_info(const ppt_fieldmap* map, int64_t* bytes, int* flags);

/* The fields a pusher sees: E = e_const + sum over maps of the map's E,
 * B likewise; maps outside their grid contribute 0 (fill_value = 0,
 * field.py:337-338). */
typedef struct {
    const ppt_fieldmap* maps[PPT_MAX_MAPS];
    int32_t n_maps;
    double e_const[3];
    double b_const[3];
} ppt_fields;

/* E and B at n points.  pts: device (n,3) float64; e_out, b_out: device
 * (n,3) float64 (either may be NULL). */
int ppt_field_eval(const ppt_fields* fields, int64_t n, const double* pts,
                   double* e_out, double* b_out, void* stream);

/* Particle state on the device, structure of arrays:
 *   PPT_PREC_F64:   f64[6*n]  = x | y | z | w_x | w_y | w_z
 *   PPT_PREC_MIXED: i32[3*n]  = cell i | j | k  (on map 0's grid)
 *                   f32[12*n] = offset_hi x|y|z | w_hi x|y|z | w_lo x|y|z | offset_lo x|y|z
 *                   (position = lo + (cell + offset_hi + offset_lo) d; the high
 *                   offset is in [0, 1] after steps that may see a field and
 *                   may pass 1 between the whole-cell carries of field-free
 *                   steps)
 * w is the velocity v [m/s], or u = gamma v for BORIS_REL / VAY. */
typedef struct {
    int32_t precision;
    int32_t algorithm;
    int64_t n;
    double* f64;
    int32_t* i32;
    float* f32;
} ppt_state;

/* Fill the state from (n,3) float64 r [m] and v [m/s] (device, row-major).
 * The mixed form locates cells on fields->maps[0]'s grid. */
int ppt_state_load(ppt_state* st, const ppt_fields* fields, const double* r, const double* v,
                   void* stream);

/* Write the state back as (n,3) float64 r and v (v = u/gamma for u-state
 * algorithms).  order (device int64[n], or NULL) maps slot -> row. */
int ppt_state_store(const ppt_state* st, const ppt_fields* fields, const int64_t* order,
                    double* r, double* v, void* stream);

typedef struct {
    int64_t step0;        /* global index of this call's first step */
    int64_t nsteps;       /* steps in this call */
    int64_t nsteps_total; /* steps of the whole track (record count, final half step) */
    int64_t rec_every;    /* record every N steps (>= 1) */
    int32_t flags;        /* PPT_TRACK_INIT | PPT_TRACK_FINAL */
    int32_t reserved;
    double dt;
    double q_over_m;
    double t0;            /* field time of step 0 */
    double rf_omega;      /* E multiplied by cos(rf_omega t + rf_phase[i]) ... */
    const double* rf_phase; /* ... when non-NULL: device float64 [n], in state (slot) order */
    double* r_hist;       /* device (nsteps_total/rec_every + 1, n, 3) or NULL */
    double* v_hist;
    const int64_t* order; /* slot -> row (after ppt_cell_sort), NULL = identity */
    int32_t* status;      /* device int32, OR-ed with PPT_STATUS_* bits, or NULL */
    unsigned long long* counters; /* device u64[2]: +in-map gathers, +particle steps; or NULL */
    const struct ppt_surface* surface; /* electrode surface (float64 form), or NULL: see below */
    uint8_t* active;      /* with a surface: device uint8[n] in ROW order, 1 = still tracked */
    const double* dt_rows; /* device float64[n] in ROW order: one time step per particle for the
                            * float64 form's RK4 and rk4_rel (the reference's batch RK4 step
                            * broadcasts an array dt over the particles, pusher.py:815-816);
                            * NULL = dt for every particle.  Other algorithms and the mixed form:
                            * PPT_ERR_UNSUPPORTED. */
} ppt_track_args;

/* Advance every particle nsteps steps in ONE kernel launch, state kept in
 * registers, fields gathered on the fly, snapshots written into r_hist /
 * v_hist at the reference's record indices.
 * With args->surface (float64 form only; PPT_ERR_UNSUPPORTED otherwise) each
 * step's segment (position before -> after the step) of every active particle
 * is tested against the surface after the step's snapshot, and a particle
 * that hits is stopped: active[row] = 0, its state stays at the step's end,
 * later snapshots and the final half step leave its rows untouched
 * (pusher.py:966-1007).  Set active to 1 before the first call. */
int ppt_track(ppt_state* st, const ppt_fields* fields, const ppt_track_args* args, void* stream);

/* ---- cylindrical maps onto a Cartesian grid -------------------------------
 * The resampling step of the reference's cylindrical-map loaders
 * (load_opal_midplane, load_aima_agora: field_loaders.py:612-640, :836-899).
 * r: device nr node radii; theta: device nt node angles [deg]; both increasing. */
typedef struct {
    int64_t nr, nt;
    const double* r;
    const double* theta;
} ppt_polar_grid;

/* For every Cartesian node (x[i], y[j]) (device arrays): r = |(x, y)| * r_scale,
 * theta = atan2(y, x) in degrees, wrapped to [0, 360); (B_r, B_theta, B_z) =
 * bilinear interpolation of comp[0..2] (device (nr, nt) float64, NULL = zero)
 * on the polar grid, 0 outside it; out[0] = B_r cos - B_theta sin, out[1] =
 * B_r sin + B_theta cos, out[2] = B_z: device (nx, ny) float64, NULL = skip. */
int ppt_polar_to_cartesian(const ppt_polar_grid* grid, const double* const comp[3], int64_t nx,
                           const double* x, int64_t ny, const double* y, double r_scale,
                           double* const out[3], void* stream);

/* ---- electrode surfaces -------------------------------------------------
 * Replaces the external PyElectrodeAssembly the reference calls each step
 * (segment_intersects_surface, pusher.py:984): a triangle mesh, copied to the
 * device with a cell grid over it.  vertices: HOST (n_vertices, 3) float64;
 * triangles: HOST (n_triangles, 3) int64 vertex indices. */
typedef struct ppt_surface ppt_surface;   /* opaque */

int ppt_surface_create(int64_t n_vertices, const double* vertices, int64_t n_triangles,
                       const int64_t* triangles, ppt_surface** out);
int ppt_surface_destroy(ppt_surface* surface);

/* device bytes held, and the cell grid's dimensions */
int ppt_surface_info(const ppt_surface* surface, int64_t* bytes, int32_t dims[3]);

/* hit[i] = 1 when the segment p0[i] -> p1[i] meets a triangle (Moller-Trumbore
 * test, segment parameter 0 <= t <= 1, triangle edges included), else 0.
 * p0, p1: device (n,3) float64; hit: device uint8[n]. */
int ppt_surface_segments_hit(const ppt_surface* surface, int64_t n, const double* p0, const double* p1,
                             uint8_t* hit, void* stream);

/* For each point and each direction d = +x, -x, +y, -y, +z, -z (in that
 * order): hits[6 i + d] = the number of triangles the ray from the point
 * along d crosses (Moller-Trumbore, t >= 0), min_dist[6 i + d] = the distance
 * to the nearest of them (INFINITY without any).  The axis-aligned ray casting
 * the reference's solver asks of its electrode assembly to classify mesh
 * cells (compute_axis_aligned_surface_intersections, poisson_amg.py:249-251).
 * points: device (n,3) float64; min_dist: device (n,6) float64; hits: device
 * (n,6) int32. */
int ppt_surface_axis_rays(const ppt_surface* surface, int64_t n, const double* points, double* min_dist,
                          int32_t* hits, void* stream);

/* ---- serving: many jobs per launch -------------------------------------
 * No reference counterpart (the reference runs one track_batch at a time,
 * pusher.py:894-1012).  A job is one track_batch call's device state. */
typedef struct {
    ppt_state state;          /* the job's particle state (loaded with ppt_state_load) */
    ppt_fields fields;
    int64_t nsteps_total;
    int64_t rec_every;
    double dt;
    double q_over_m;
    double t0;
    double rf_omega;
    const double* rf_phase;   /* device float64 [n] or NULL */
    double* r_hist;           /* device (nsteps_total/rec_every + 1, n, 3) or NULL */
    double* v_hist;
    int32_t* status;          /* device int32 or NULL */
    int64_t steps_done;       /* steps already taken (a table rebuilt mid-track resumes here) */
    int64_t tick_steps;       /* steps this job advances per tick; 0 = the tick's chunk */
} ppt_job_desc;

typedef struct ppt_jobs ppt_jobs;   /* opaque host handle */

/* Device bytes ppt_jobs_create needs for n_jobs jobs. */
int64_t ppt_jobs_scratch_bytes(int n_jobs);

/* Write the job table into scratch (device, ppt_jobs_scratch_bytes bytes;
 * caller-owned, must outlive the handle) with every job at step 0.  The
 * descriptors' device buffers must outlive the handle too. */
int ppt_jobs_create(const ppt_job_desc* jobs, int n_jobs, void* scratch, ppt_jobs** out, void* stream);

/* Advance every unfinished job by up to chunk steps (its tick_steps when
 * that is set; Boris-family half steps and snapshots exactly as ppt_track).  Reads no host data and does not
 * synchronise: a captured CUDA graph of this call can be replayed. */
int ppt_jobs_tick(ppt_jobs* jobs, int64_t chunk, void* stream);

/* Device pointers to the per-job steps done (int64[n_jobs]) and done flags
 * (int32[n_jobs], 1 once a job's last step ran). */
int ppt_jobs_progress(const ppt_jobs* jobs, int64_t** steps, int32_t** done);

int ppt_jobs_destroy(ppt_jobs* jobs);

/* Reorder particles by the cell of map 0 (locality of the corner gathers).
 * Permutes the state, rf_phase and order arrays in place.  Decided on the
 * device: the permutation runs when at least n/16 particles are inside the
 * map, or when the warps holding in-map particles exceed the ones they need
 * by n/512; otherwise the call is a no-op that never waits on the host.
 * scratch: device buffer of ppt_cell_sort_scratch_bytes(n) bytes. */
int64_t ppt_cell_sort_scratch_bytes(int64_t n);
int ppt_cell_sort(ppt_state* st, const ppt_fields* fields, int64_t* order, double* rf_phase,
                  void* scratch, void* stream);

/* Put particles back in row order (slot s moves to position order[s]) and
 * set order to the identity: once a bunch has left its maps the cell order
 * buys nothing, and in row order the snapshot rows are written coalesced.
 * order must be a permutation of 0 .. n-1 (as ppt_cell_sort keeps it);
 * scratch as for ppt_cell_sort.  Always permutes (the caller decides when). */
int ppt_restore_order(ppt_state* st, int64_t* order, double* rf_phase, void* scratch, void* stream);

/* Poisson mesh of the reference's space-charge solver: cells[d] nodes per
 * axis spaced extent[d] / cells[d], the first at -extent[d] / 2 (the
 * reference's domain_extent and mesh_cells). */
typedef struct {
    double extent[3];
    int64_t cells[3];
} ppt_mesh_desc;

/* Cloud-in-cell charge deposition (PyAMGPoissonSolver._bin_particles_cic_cpu
 * and _cic_deposit_numba, src/PyPATools/poisson_amg.py:849-911): rho (device
 * float64, cells[0]*cells[1]*cells[2], [i][j][k] with k fastest) is
 * overwritten with the charge per cell volume of the n particles at r
 * (device (n,3) float64) with charges q (device float64 [n]).  Positions are
 * clamped onto the mesh as the reference does (a particle on or beyond the
 * last node lands on the node before it); a NaN position deposits nothing.
 * Float64 atomics: results agree with the sequential sum to rounding. */
int ppt_deposit_cic(int64_t n, const double* r, const double* q, const ppt_mesh_desc* mesh, double* rho,
                    void* stream);

/* ---- space charge: the potential and field on the solver's mesh ----------
 * PyAMGPoissonSolver's linear solve and field step for a domain without
 * conductor cells (src/PyPATools/poisson_amg.py:616-797; operator :293-443,
 * rhs = rho / eps0 :913-921, E = -grad phi :98-130).  The mesh has cells[a]
 * cells of size extent[a] / cells[a] centred at -extent/2 + (i + 1/2) h;
 * rhs, phi, ex, ey, ez are device (nx, ny, nz) float64 arrays.
 * ppt_poisson_solve: conjugate gradients, matrix-free, from the initial guess
 * in phi until |r| <= rel_tol |rhs| or max_iter iterations; synchronises the
 * stream a few times; reports the iterations and the final |r| / |rhs|.
 * ppt_field_from_potential: central differences at cells whose three indices
 * are interior, 0 on the outer layer (any of ex, ey, ez may be NULL). */
int64_t ppt_poisson_scratch_bytes(const ppt_mesh_desc* mesh);
int ppt_poisson_solve(const ppt_mesh_desc* mesh, const double* rhs, double* phi, void* scratch, double rel_tol,
                      int64_t max_iter, int64_t* iterations, double* rel_residual, void* stream);
int ppt_field_from_potential(const ppt_mesh_desc* mesh, const double* phi, double* ex, double* ey, double* ez,
                             void* stream);

/* The same solve with per-cell coefficients, for a domain with conductor
 * cells (the reference's Shortley-Weller rows, poisson_amg.py:293-443):
 * coef: device (nx*ny*nz, 7) float64 = diagonal and the +x, -x, +y, -y, +z,
 * -z couplings of each cell's row (0 for a neighbour outside the box or in a
 * conductor; a conductor cell's row is the identity, its rhs 0).  The
 * operator is not symmetric: BiCGSTAB.  Scratch: ppt_poisson_coef_scratch_bytes. */
int64_t ppt_poisson_coef_scratch_bytes(const ppt_mesh_desc* mesh);
int ppt_poisson_solve_coef(const ppt_mesh_desc* mesh, const double* coef, const double* rhs, double* phi,
                           void* scratch, double rel_tol, int64_t max_iter, int64_t* iterations,
                           double* rel_residual, void* stream);

/* Bunch moments of n particles from (n,3) float64 positions and velocities
 * (device), in float64:
 *   out[0..2]   centroid            out[3..5]   x_std
 *   out[6..8]   xp_std              out[9..11]  xp_mean
 *   out[12..15] xxp yyp xyp yxp     out[16]     mean |p| (beta gamma)
 *   out[17..19] mean p              out[20]     mean Ekin [MeV]
 *   out[21]     std Ekin [MeV]
 * Velocities go through the reference's per-component v -> p -> v
 * conversion first.  scratch: device buffer of ppt_moments_scratch_bytes(n). */
#define PPT_MOMENTS_LEN 22
int64_t ppt_moments_scratch_bytes(int64_t n);
int ppt_moments(int64_t n, const double* r, const double* v, double mass_mev,
                double* out, void* scratch, void* stream);

/* ppt_moments without any device allocation, for callers that may not
 * allocate device memory while they run (an application whose GPU memory is
 * all owned by another allocator's pool, or an analysis hook inside a
 * latency-bound loop where cudaMalloc/cudaFree, which can synchronise the
 * device, are not allowed).  No counterpart in the reference.
 * Scratch: a static 52 KB device array, held by every GPU that loads the
 * library until the process exits.  The first call on a device looks up its
 * address (cudaGetSymbolAddress), and so does the first call in a new context
 * of that device (after cudaDeviceReset, or in a context the caller made
 * current); make that first call before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race.
 * n must be in [1, 2^53]; anything else returns PPT_ERR_ARG. */
int ppt_moments_noalloc(int64_t n, const double* r, const double* v, double mass_mev,
                        double* out, void* stream);

const char* ppt_last_error(void);
int ppt_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PPT_H */
