/*
 * ecsg_b200.h -- C ABI of the B200 implementation of ECSG's composite-
 * staggered-grid time loop (libecsg_b200.so).
 *
 * Plain C: POD structs, raw pointers and sizes, integer status codes.  Every
 * entry point returns ECSG_OK (0) or a negative ECSG_ERR_* code; the message of
 * the last failure on a simulation is ecsg_last_error(sim).  Calls on one
 * simulation must come from one host thread at a time.  Host buffers are read
 * or written before the call returns unless the name says _async.
 *
 * Array layouts
 *   "Field layout": the reference's Field storage (field.cpp:85-149): x fastest,
 *   len[d] = n[d] + 1 + 2R on node dims and n[d] + 2R on staggered dims, the
 *   first element is (-R,-R,-R).  Staggered positions per component are those
 *   of init_del_sim.cpp:14-24 (vx 000, vy 110, vz 101, sxx/syy/szz 100,
 *   syz 111, sxz 001, sxy 010).
 *   "Node layout": (nz+1) x (ny+1) x (nx+1) values, x fastest (the RSF inputs
 *   buoy_N, s11_N, s13_N of init_del_par_field.cpp:23-118).
 *
 * Component order: 0 vx, 1 vy, 2 vz, 3 sxx, 4 syy, 5 szz, 6 syz, 7 sxz, 8 sxy.
 * Grid 0 is the top (finest) grid; interface i couples grid i-1 (fine) and
 * grid i (coarse), as main.cpp:206-209 and 240-251 index them.
 */
#ifndef ECSG_B200_H
#define ECSG_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ECSG_ABI_VERSION 1

enum {
    ECSG_OK = 0,
    ECSG_ERR_INVALID = -1,      /* bad argument or unsupported configuration */
    ECSG_ERR_CUDA = -2,         /* a CUDA call failed; see ecsg_last_error */
    ECSG_ERR_NO_DEVICE = -3,    /* no usable sm_100 device */
    ECSG_ERR_STATE = -4,        /* call out of order (e.g. run before medium set) */
    ECSG_ERR_NOT_CONVERGED = -5 /* a Jacobi solve hit its iteration cap (status) */
};

enum { ECSG_F32 = 0, ECSG_F64 = 1 };                     /* field precision */
enum { ECSG_MEDIUM_ISO = 0, ECSG_MEDIUM_ORTHO9 = 1, ECSG_MEDIUM_GEN21 = 2 };   /* stiffness form */
enum { ECSG_MODE_II = 0, ECSG_MODE_ECI = 1 };            /* interface mode (main.cpp:54) */

/* Device status bits (ecsg_get_status). */
enum { ECSG_ST_JACOBI_CAP = 1, ECSG_ST_BARRIER_TIMEOUT = 2, ECSG_ST_NONFINITE = 4, ECSG_ST_PIPE_TIMEOUT = 8 };

/* One uniform sub-grid: Grid (grid.hpp:6-11) without the name.  size[] are
 * cell counts (points - 1), step[] the spacings.  z origins are stacked as
 * init_del_par_field.cpp:55-57 does. */
typedef struct ecsg_grid_desc {
    int size[3];
    double step[3];
} ecsg_grid_desc;

/* Run parameters: the key=value parameters of main.cpp:36-67. */
typedef struct ecsg_config {
    int num_grids;        /* num_grids */
    int radius;           /* stencil radius 1..6 (init_del_fdcoeff.cpp:38-85); composites
                           * and 21-Cij media need 1 (the interface conditions are
                           * derived for radius 1) */
    double dt;            /* time step */
    int imode;            /* ECSG_MODE_ECI (1), or ECSG_MODE_II (0: ratio-2 interfaces only) */
    int top_bc;           /* 0 rigid, 1 free surface */
    int precision;        /* ECSG_F32 or ECSG_F64 */
    int medium;           /* ECSG_MEDIUM_ISO, ECSG_MEDIUM_ORTHO9 or ECSG_MEDIUM_GEN21 */
    int energy;           /* allocate velocity copies for the energy (check_energy) */
    int jacobi_max_iter;  /* cap on sxz Jacobi sweeps per solve; <= 0 selects 10000 */
    int device;           /* CUDA device ordinal */
    int mirror_fix;       /* 0: the reference's halo mirrors exactly; 1: the vy wall
                           * mirrors also cover the top-most updated plane of vy
                           * (update_vel.cpp:211-246 stop one plane short), which
                           * makes the composite energy exactly conserved */
    int ii_skip_end_column; /* imode 0 only.  0: update_ghost_vz.cpp as it stands.
                           * 1: leave the fine vz ghosts of the last x column
                           * untouched, as the revision that produced the
                           * reference's II golden traces did (its line 98
                           * declared a new `int i1` instead of setting i0) */
} ecsg_config;

typedef struct ecsg_sim ecsg_sim;

/* Creates the device state of a composite run: 9 fields per grid (InitSim,
 * init_del_sim.cpp:3-40), ghost-solve work space (InitGhostContainer,
 * init_del_ghost_container.cpp:4-42) and FD coefficients dt/h (InitFDcoeff,
 * init_del_fdcoeff.cpp:7-22).  Fields start at zero.  Refinement ratio between
 * consecutive grids is step[i]/step[i-1] (2 or 3, equal in x and y, and size
 * must satisfy size_fine = ratio * size_coarse in x and y). */
int ecsg_create(const ecsg_grid_desc *grids, const ecsg_config *cfg, ecsg_sim **out);
int ecsg_destroy(ecsg_sim *sim);
const char *ecsg_last_error(const ecsg_sim *sim);
int ecsg_device_count(void);

/* Isotropic medium of grid g from node-layout float32 arrays: buoyancy, s11,
 * s13 (InitParField, init_del_par_field.cpp:23-149: s44 = s11 - s13 and the
 * staggered averages are formed on the device). */
int ecsg_set_medium_iso(ecsg_sim *sim, int g, const float *buoy, const float *s11, const float *s13);
/* Orthorhombic medium: node-layout buoyancy and the 9 stiffness arrays in the
 * order c11 c22 c33 c23 c13 c12 c44 c55 c66 (update_stress.cpp:17-25), each
 * in Field layout with R = 0 at its staggered position (c11..c12 at 100, c44
 * at 111, c55 at 001, c66 at 010).  As in the reference, the shear entries are
 * the stored 2*mu-type moduli that the update multiplies by 0.5. */
int ecsg_set_medium_ortho9(ecsg_sim *sim, int g, const double *buoy, const double *const c[9]);
/* General anisotropic medium (21 Cij, Voigt, engineering shear strains; no
 * counterpart in the reference, which reads isotropic media only).  c[k] in
 * Field layout with R = 0 at the slot's position: slots 0..14 = C11 C12 C13
 * C22 C23 C33 C14 C15 C16 C24 C25 C26 C34 C35 C36 at the normal-stress
 * position (1,0,0); 15..17 = C44 C45 C46 at the syz position (1,1,1); 18..19
 * = C55 C56 at the sxz position (0,0,1); 20 = C66 at the sxy position (0,1,0).
 * With the 12 off-block slots zero this is the orthorhombic update with
 * C44 = c44/2 etc. of ecsg_set_medium_ortho9.  With cfg.energy the stress
 * update also sums the velocities it reads (three displacement sums U, the
 * strains being linear in the velocities) so that ecsg_energy can return
 * 1/2 (rho v, v') + 1/2 (eps, sigma) with eps the strain differences of U. */
int ecsg_set_medium_cij21(ecsg_sim *sim, int g, const double *buoy, const double *const c[21]);
/* Tilted transversely isotropic medium built on the device into the 21-Cij
 * slots (no counterpart in the reference).  Node-layout float arrays (R = 0,
 * like ecsg_set_medium_iso): vp, vs (vs < vp), rho, the tilt of the symmetry
 * axis from vertical (dip) and its azimuth from x, both in radians; Thomsen's
 * epsilon, delta, gamma for the whole grid.  Buoyancy = 1/rho at the nodes;
 * each Cij is rotated with the Bond matrix at the nodes and averaged to its
 * slot position with the 2/4/8-point means of ReshapeField
 * (field.cpp:428-476). */
int ecsg_set_medium_tti(ecsg_sim *sim, int g, const float *vp, const float *vs, const float *rho, const float *dip,
                        const float *azimuth, double epsilon, double delta, double gamma);

/* Field component k of grid g in Field layout (radius R of ecsg_config), in
 * double (Field::GetPtr1 of the reference, field.hpp:84-85). */
int ecsg_set_field(ecsg_sim *sim, int g, int k, const double *src);
int ecsg_get_field(ecsg_sim *sim, int g, int k, double *dst);
/* Number of elements of component k of grid g in Field layout. */
long long ecsg_field_elems(const ecsg_sim *sim, int g, int k);

/* One operator on the device state, in place (sim_utils.hpp:127-148). */
int ecsg_update_vel(ecsg_sim *sim, int g);       /* UpdateVel    update_vel.cpp:4-249 */
int ecsg_update_stress(ecsg_sim *sim, int g);
/* UpdateVel / UpdateStress with the boundary roles passed explicitly, as the
 * reference's own signatures take them (update_vel.cpp:4 and
 * update_stress.cpp:4: top, bottom); the plain forms derive them from the
 * grid's place in the composite. */
int ecsg_update_vel_ex(ecsg_sim *sim, int g, int top, int bottom);
int ecsg_update_stress_ex(ecsg_sim *sim, int g, int top, int bottom);
/* FD coefficients of grid g as the caller computed them (InitFDcoeff,
 * init_del_fdcoeff.cpp:7-22: coeff[g][d][0] = dt / h_d for radius 1); by
 * default they are formed from cfg.dt and the grid steps. */
int ecsg_set_coefficients(ecsg_sim *sim, int g, const double k[3]);    /* UpdateStress update_stress.cpp:4-311 */
int ecsg_ghost_vz(ecsg_sim *sim, int i);         /* UpdateGhostVZ  update_ghost_vz.cpp:8-251 */
int ecsg_ghost_sxz(ecsg_sim *sim, int i);        /* UpdateGhostSXZ update_ghost_sxz.cpp:16-298 + Jacobi2D/Norm2D */
int ecsg_ghost_syz(ecsg_sim *sim, int i);        /* UpdateGhostSYZ update_ghost_syz.cpp:6-241 */
/* Jacobi warm-start vector X of interface i ((nx2+1)*(ny2+1) doubles, the
 * reference's g_sxz array) and the sweep count / tolerance of the last solve. */
int ecsg_get_sxz_state(ecsg_sim *sim, int i, double *X, int *last_iters, double *last_tol, long long *total_iters);
int ecsg_set_sxz_state(ecsg_sim *sim, int i, const double *X);

/* Energy (ComputeEnergy, compute_energy.cpp:34-54, summed over grids as
 * main.cpp:217-225).  ecsg_copy_vel stores v^{n-1/2} (main.cpp:173-176);
 * requires cfg.energy. */
int ecsg_copy_vel(ecsg_sim *sim);
int ecsg_energy(ecsg_sim *sim, double *energy);
/* Interface residues of interface i (compute_res.cpp:4-95) in the res_trace
 * order [res vx-sxz, avg|vx2|, avg|sxz2|, res vy-syz, avg|vy2|, avg|syz2|,
 * res vz-szz, avg|vz2|, avg|szz2|]; which: bit 0/1/2 selects the groups. */
int ecsg_residues(ecsg_sim *sim, int i, int which, double out[9]);

/* Source (InitSrc init_src.cpp:7-49 + main.cpp:193-195): component comp of
 * grid g at index (ix,iy,iz) gets += scale*trace[n] (float product) at step n
 * for n < nt.  The reference uses comp 0 (vx) and scale 1000. */
int ecsg_set_source(ecsg_sim *sim, int g, int ix, int iy, int iz, int comp, const float *trace, int nt, float scale);
/* Receivers (InitRecTrace init_del_rec_trace.cpp:8-56 + main.cpp:182-184):
 * loc4[4*i] = {grid, ix, iy, iz}; component comp is sampled after the velocity
 * update and before the source injection. */
int ecsg_set_receivers(ecsg_sim *sim, const int *loc4, int n, int comp);
/* Maps a point to (grid, ix, iy, iz) like init_src.cpp:33-45. */
int ecsg_locate(const ecsg_sim *sim, const double xyz[3], int loc4[4]);

/* Runs steps n0 .. n0+nsteps-1 of the time loop of main.cpp:165-261 on the
 * device (movie output excluded).  traces (may be NULL): nsteps x nrec
 * float32, time-major, copied to the host.  energy (may be NULL, needs
 * cfg.energy): one double per step where (n % energy_every == 0), others NaN.
 * residues (may be NULL): nsteps x (num_grids-1) x 9 doubles.  use_graph != 0
 * captures one step in a CUDA graph and replays it. */
int ecsg_run(ecsg_sim *sim, int n0, int nsteps, float *traces, double *energy, int energy_every, double *residues,
             int use_graph);

/* Run state for checkpoint / resume (no reference counterpart): the fields of
 * every grid in the library's own layout and precision, the sxz warm starts
 * and, when the simulation keeps them, the displacement sums of 21-Cij
 * media, as one opaque buffer of ecsg_state_bytes(sim) bytes (host or device
 * memory).  Loading it into a simulation created with the same grids,
 * configuration and medium continues the run bit for bit: pass the next step
 * index as n0 of ecsg_run. */
long long ecsg_state_bytes(const ecsg_sim *sim);
int ecsg_save_state(ecsg_sim *sim, void *dst);
int ecsg_load_state(ecsg_sim *sim, const void *src);

/* Movie frames (InitMovie/PrintMovie, init_del_movie.cpp:5-95, print.cpp:89-104):
 * the computational domain of field k of grid g (no halo), dims[0] x dims[1]
 * x dims[2] with x fastest, as float32, packed on the device and copied to
 * dst (pinned memory from ecsg_host_alloc makes the copy asynchronous-rate);
 * returns once dst holds the frame. */
int ecsg_domain_shape(const ecsg_sim *sim, int g, int k, int dims[3]);
int ecsg_get_domain(ecsg_sim *sim, int g, int k, float *dst);
/* Page-locked host memory for frame and trace buffers. */
int ecsg_host_alloc(size_t bytes, void **out);
int ecsg_host_free(void *p);

/* Device time (CUDA events around the step loop) of the last ecsg_run and the
 * number of kernels it launched. */
int ecsg_last_run(ecsg_sim *sim, double *device_ms, long long *launches);
/* CUDA events on the simulation's stream around any sequence of calls. */
int ecsg_timer_start(ecsg_sim *sim);
int ecsg_timer_stop(ecsg_sim *sim, double *ms);
/* Runs nsteps steps one kernel at a time with events around each and writes
 * the mean milliseconds per step into ms[7*8]: ms[0*8+g] velocity kernel of
 * grid g, ms[1*8+g] its halo mirrors, ms[2*8+g] stress kernel of grid g,
 * ms[3*8+i] vz solve of interface i, ms[4*8+i] sxz solve, ms[5*8+i] syz
 * solve, ms[6*8] receiver/source kernel.  The state advances by nsteps. */
int ecsg_time_kernels(ecsg_sim *sim, int nsteps, double *ms);

/* ---------------------------------------------------------------------------
 * Allocation-free sxz interface solve.  No counterpart in the reference: it
 * exists for callers that cannot allocate device memory (their device memory
 * belongs to another framework's allocator, or a fixed budget was reserved up
 * front), who hold the two grids' fields themselves and pass them in.
 *
 * It runs the same energy-conserving sxz solve as ecsg_ghost_sxz (matrix,
 * right-hand side, warm-started Jacobi with the reference stopping rule, coarse
 * and fine ghost values written into the sxz fields) and calls no cudaMalloc,
 * cudaFree or allocating library routine.  Its work space is one static device
 * array of about 11.6 MB that every GPU loading the library keeps until exit;
 * interfaces with more than ECSG_NOALLOC_MAX_UNKNOWNS interior coarse nodes
 * ((nx2-1)*(ny2-1)) or ECSG_NOALLOC_MAX_NODES nodes ((nx2+1)*(ny2+1)) are
 * rejected with ECSG_ERR_INVALID and a message (362 x 362 coarse cells fit).
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  All calls share the array and it keeps
 * the last call's contents (each call clears what must start at zero), so calls
 * that overlap on the GPU race: serialise them on one stream.
 *
 * Fields are passed in the device layout of ecsg_grid_view (the layout an
 * ecsg_sim uses internally).  X is the caller's device array of
 * (nx2+1)*(ny2+1) doubles with a zero border: the warm start on entry, the new
 * coarse ghost values on return (the reference's g_sxz array).  stream is a
 * cudaStream_t (NULL: the legacy default stream); the call is asynchronous
 * unless iters is non-null, in which case it waits for the solve and returns
 * ECSG_ERR_NOT_CONVERGED when the sweep cap was hit.  errbuf (may be NULL)
 * receives the message of a failure.  The views are checked before anything
 * runs: the x and y step ratios must be the same integer >= 2 (as in
 * ecsg_create), fine sizes ratio * coarse sizes in x and y, pitches at least
 * size + 1 + 2 * radius, and the halo of every component inside the box the
 * pitches span with 32-bit indices; a view that fails is ECSG_ERR_INVALID.
 *
 * An asynchronous call (iters == NULL) cannot return the solve's outcome, so
 * every call ORs its device status bits (ECSG_ST_JACOBI_CAP: the sweep cap
 * was hit and X holds the last iterate; ECSG_ST_BARRIER_TIMEOUT: a grid
 * barrier gave up) into a sticky word of the static array that no solve
 * clears.  ecsg_ghost_sxz_noalloc_status waits for stream, returns that word
 * of the current device in *status and, when clear is non-zero, resets it.
 * It allocates nothing either.
 * ------------------------------------------------------------------------- */
#define ECSG_NOALLOC_MAX_UNKNOWNS 131072
#define ECSG_NOALLOC_MAX_NODES 132496

/* One grid in device memory: element (x,y,z) of every component, x,y,z from
 * -radius, is at index origin + (z*pitch[1] + y)*pitch[0] + x. */
typedef struct ecsg_grid_view {
    int size[3];          /* cells */
    double step[3];
    int radius;           /* halo radius (1) */
    int pitch[3];         /* elements per row, rows per plane, planes */
    long long origin;     /* index of element (0,0,0) */
    void *field[9];       /* component order of this header; float or double */
    const void *buoy;     /* buoyancy at nodes, same layout and type */
} ecsg_grid_view;

int ecsg_ghost_sxz_noalloc(const ecsg_grid_view *fine, const ecsg_grid_view *coarse, double dt, int precision,
                           double *X, int max_iter, void *stream, int *iters, char *errbuf, size_t errlen);
int ecsg_ghost_sxz_noalloc_status(void *stream, int *status, int clear);

int ecsg_synchronize(ecsg_sim *sim);
/* Device status bits accumulated since the last clear (ECSG_ST_*). */
int ecsg_get_status(ecsg_sim *sim, int *status, int clear);
/* Bytes of device memory held by the simulation. */
long long ecsg_device_bytes(const ecsg_sim *sim);

/* ---------------------------------------------------------------------------
 * Adjoint and misfit gradients (no counterpart in the reference).  21-Cij
 * media (ECSG_MEDIUM_GEN21) only.  Every operator of the time loop is an
 * affine map of the full field state (halos and ghosts included); its
 * adjoint applies the transposed map to an adjoint state held beside the
 * fields and accumulates the gradient of <adjoint, operator output> with
 * respect to the node buoyancy and the 21 stiffness slots.
 * ------------------------------------------------------------------------- */
enum { ECSG_ADJ_VEL = 0, ECSG_ADJ_STRESS = 1, ECSG_ADJ_GHOST_VZ = 2, ECSG_ADJ_GHOST_SXZ = 3, ECSG_ADJ_GHOST_SYZ = 4 };
/* Zero the adjoint fields and gradients (allocates them on first use). */
int ecsg_adjoint_reset(ecsg_sim *sim);
/* Adjoint field k of grid g, Field layout as ecsg_set_field. */
int ecsg_set_adjoint_field(ecsg_sim *sim, int g, int k, const double *src);
int ecsg_get_adjoint_field(ecsg_sim *sim, int g, int k, double *dst);
/* Apply the transpose of one operator in place on the adjoint fields and add
 * its medium gradient.  op = ECSG_ADJ_VEL / ECSG_ADJ_STRESS (index = grid;
 * the velocity operator includes its halo mirrors) or ECSG_ADJ_GHOST_VZ / SXZ
 * / SYZ (index = interface, 1 .. num_grids-1).  The simulation's fields must
 * hold the operator's output state (what the forward call left). */
int ecsg_adjoint_op(ecsg_sim *sim, int op, int index);
/* Gradient of grid g: which = 0 buoyancy at the nodes ((nz+1)(ny+1)(nx+1),
 * x fastest), which = 1 + k the stiffness slot k of ecsg_set_medium_cij21 in
 * that slot's R = 0 layout. */
int ecsg_get_gradient(ecsg_sim *sim, int g, int which, double *dst);
/* The 22 gradient volumes of grid g in one FP64 DEVICE buffer of
 * ecsg_gradient_elems(sim, g) doubles (the layouts of ecsg_get_gradient, which
 * = 0 .. 21 back to back), for a sum over processes (e.g. an NCCL all-reduce
 * of the shots' gradients; no reference counterpart).  Both are enqueued on
 * the simulation's stream (ecsg_stream) and return before they complete;
 * unpack overwrites the gradient with the buffer, converted to the
 * simulation's precision. */
long long ecsg_gradient_elems(const ecsg_sim *sim, int g);
int ecsg_pack_gradient(ecsg_sim *sim, int g, double *dst_device);
int ecsg_unpack_gradient(ecsg_sim *sim, int g, const double *src_device);
/* The CUDA stream (cudaStream_t) the simulation's work runs on. */
void *ecsg_stream(const ecsg_sim *sim);
/* Misfit L = 1/2 sum_n sum_r (v_r(n) - observed[n * n_rec + r])^2 over nsteps
 * steps from rest (receivers as set by ecsg_set_receivers, sampled as the
 * traces), and its gradient with respect to the medium: the forward run keeps
 * the state every ckpt_every steps; the reverse run recomputes each segment
 * from its checkpoint and applies the operator adjoints in reverse order.
 * The gradients are then read with ecsg_get_gradient; the fields are left at
 * the final forward state. */
int ecsg_misfit_gradient(ecsg_sim *sim, int nsteps, const float *observed, int ckpt_every, double *loss);

/* ---------------------------------------------------------------------------
 * Batches (no counterpart in the reference).
 * ------------------------------------------------------------------------- */
/* A new instance with the grids and configuration of model whose medium IS
 * the model's (one copy on the device; set the model's medium first, keep the
 * model alive while shots exist; ecsg_set_medium_* on a shot fails).  Own
 * fields, source, receivers, adjoint state. */
int ecsg_create_shot(const ecsg_sim *model, ecsg_sim **out);
/* Advance n instances (any sizes and media, one precision, one device) by
 * nsteps steps starting at step n0 (source index and trace row 0): one CUDA
 * graph holds one step of every instance, each on its own stream, and is
 * launched once per step.  traces[b] (may be null) receives instance b's
 * receiver traces (nsteps x n_rec); ms the device time of the steps. */
int ecsg_batch_run(ecsg_sim *const *sims, int n, int n0, int nsteps, float *const *traces, double *ms);
/* ecsg_misfit_gradient of n instances at once (one host thread and stream
 * each, so their kernels overlap); observed[b] as for a single instance. */
int ecsg_batch_misfit_gradient(ecsg_sim *const *sims, int n, int nsteps, const float *const *observed, int ckpt_every,
                               double *losses);
/* dst's gradients = the sum of the instances' gradients, accumulated in FP64
 * (dst may be one of them; same geometry and precision). */
int ecsg_sum_gradients(ecsg_sim *dst, ecsg_sim *const *srcs, int n);
/* The misfit gradients of n shots (n <= 16) that share one medium (the
 * instances of one model made by ecsg_create_shot, with the same receiver
 * count and component), advanced in lockstep on sims[0]'s stream: each phase
 * of a forward or adjoint step runs for all shots before the next, so the
 * phases that read the medium or solve the interface systems do so once for
 * all of them.  No reference counterpart: it batches the time loop of
 * main.cpp:165-261 (a shot = one pass of it) and the adjoint of
 * ecsg_misfit_gradient.  Checkpoints every ckpt_every steps; inside a
 * segment the states are recomputed from its checkpoint.  With
 * 0 < sub_every < ckpt_every, through sub-checkpoints every sub_every steps.
 * With sub_every <= 0, when the checkpoints and a segment's states of all n
 * shots do not fit in device memory: a shorter checkpoint interval that fits;
 * else groups of fewer shots that fit, run one after the other (their
 * gradients summed); else sub-checkpoints every ~sqrt(ckpt_every) steps (one
 * more forward pass of each segment).  Leaves in sims[0]'s
 * gradient arrays the gradient of the sum of the n misfits (the medium
 * adjoints accumulate every shot's terms in the field precision; the
 * interface adjoints' shares are summed in FP64 at the end); losses[b] (may
 * be NULL) receives shot b's misfit; every instance is left at its final
 * forward state. */
int ecsg_shots_misfit_gradient(ecsg_sim *const *sims, int n, int nsteps, const float *const *observed, int ckpt_every,
                               int sub_every, double *losses);
/* Autotuner: for each grid, time the FP32 velocity and stress sweeps over
 * candidate z-march depths (chunks per column) on the simulation's own state
 * (restored afterwards) and keep the fastest; reps timed repetitions each.
 * ecsg_get_tuning returns the chosen chunk counts (0 = the built-in choice). */
int ecsg_autotune(ecsg_sim *sim, int reps);
int ecsg_get_tuning(const ecsg_sim *sim, int g, int chunks[2]);

#ifdef __cplusplus
}
#endif
#endif
