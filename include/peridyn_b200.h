/*
 * peridyn_b200.h -- C ABI of libperidyn_b200.so, the B200 (sm_100a)
 * implementation of PeriDyn's per-step force path.
 *
 * The library is the body behind the reference's CUDA dispatch points:
 *   force_density_T!(f, y, limits, mat, ::Type{Val{:cuda}})
 *       reference: src/materials/general_material.jl:388-390 (throws today)
 *   dilatation!(theta, ..., ::Type{Val{:cuda}})     src/peri.jl:283-315
 *   short_range_contact!(..., ::Type{Val{:cuda}})   src/contacts/contacts.jl:189-336
 *   update_contact_neighs!(..., ::Type{Val{:cuda}}) src/contacts/contacts.jl:434-639
 *   apply_solver!(env, ::DSVelocityVerlet)           src/solvers/velocity_verlet.jl:27
 *   apply_solver!(env, ::QSDrag)                     src/solvers/minimize.jl:74
 *   update_acc!(env)                                 src/solvers/solvers.jl:320-336
 *   cal_damage(env)                                  src/peri.jl:587-594
 *
 * Conventions
 *  - Host arrays use the reference's layouts: positions/velocities/
 *    accelerations are 3xN column-major Float64 (x[3*i + d]); family is
 *    M'xN column-major Int64, 1-based block-local indices in descending order
 *    with 0 padding; intact is M'xN Bool (uint8).
 *  - Every function returns a pd_status; 0 is success.  No C++ exception
 *    and no abort crosses the ABI.  pd_last_error() returns a message for
 *    the most recent failure on the calling thread.
 *  - The library copies host inputs into device-owned memory; no host
 *    pointer is kept after a call returns.
 *  - An environment is not thread-safe: one host thread per pd_env.  Each
 *    environment owns one CUDA stream on its device.
 *  - There is no CPU fallback: without a usable CUDA device every compute
 *    call fails with PD_ERR_NO_DEVICE.
 */
#ifndef PERIDYN_B200_H
#define PERIDYN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PD_ABI_VERSION 2

#if defined(__GNUC__)
#define PD_API __attribute__((visibility("default")))
#else
#define PD_API
#endif

typedef int32_t pd_status;
enum {
    PD_OK = 0,
    PD_ERR_ARG = 1,             /* invalid argument / inconsistent sizes        */
    PD_ERR_OOM = 2,             /* device or host allocation failed             */
    PD_ERR_FAMILY_OVERFLOW = 3, /* a family does not fit max_neigh (reference:
                                   BoundsError in cal_family!/GeneralMaterial) */
    PD_ERR_NAN = 4,             /* NaN/Inf detected by pd_env_check_finite      */
    PD_ERR_CUDA = 5,            /* CUDA runtime error                           */
    PD_ERR_TIMEOUT = 6,         /* a bounded device wait gave up                */
    PD_ERR_STATE = 7,           /* call not valid in the environment's state    */
    PD_ERR_NO_DEVICE = 8,       /* no usable CUDA device                        */
    PD_ERR_UNSUPPORTED = 9      /* valid input the chosen mode does not support */
};

/* Material kinds: src/materials/bond_based.jl, ordinary_state_based.jl,
 * skip_specific.jl, elasto_plastic.jl (ElastoPlasticSolidSpecific, Von
 * Mises; all three precisions; the device-pointer entry points take the
 * other kinds only). */
enum { PD_MAT_BOND_BASED = 0, PD_MAT_ORDINARY_STATE_BASED = 1, PD_MAT_SKIP = 2, PD_MAT_ELASTO_PLASTIC = 3 };

/* Arithmetic modes.
 * PD_PREC_FP64_SERIAL: FP64, no fused multiply-add, every particle's
 *   force summed in the exact order of the reference's serial loop
 *   (general_material.jl:330-368) -> bit-identical forces, trajectories and
 *   broken-bond sets.
 * PD_PREC_FP64: FP64, one gather pass per bond pair side, FMA allowed.
 * PD_PREC_FP32C: FP32 bond arithmetic on FP32 displacements with the
 *   cancellation-free stretch, FP64 position accumulator. */
enum { PD_PREC_FP64_SERIAL = 0, PD_PREC_FP64 = 1, PD_PREC_FP32C = 2 };

/* Boundary conditions: FixBC.jl, ToFroBC.jl (MoveBC = ToFroBC, freq=Inf),
 * DeltaScaleBC.jl, ScaleFixWaitBC.jl, ContainerBC.jl. */
enum {
    PD_BC_FIX = 0,
    PD_BC_TOFRO = 1,
    PD_BC_DELTA_SCALE = 2,
    PD_BC_SCALE_FIX_WAIT = 3,
    PD_BC_CONTAINER = 4
};

/* Contact models: contacts.jl ContactModel12 (two blocks) / ContactModel11
 * (self contact of one block); force law nonlinearspring.jl:124-145.
 * PD_CONTACT_11 reproduces the reference's neighbour search, whose merge
 * walk (contacts.jl:554-557) assumes ascending families and so finds at most
 * the first family member; PD_CONTACT_11_ORDERED (extension) takes every
 * family member whose bond is broken, in an adjacent search cell and within
 * equi_dist, in family order, up to max_neighs. */
enum { PD_CONTACT_12 = 0, PD_CONTACT_11 = 1, PD_CONTACT_11_ORDERED = 2 };

typedef struct pd_env pd_env;

/* Specific-material parameters of one block (reference: BondBasedSpecific /
 * OrdinaryStateBasedSpecific / SkipSpecific).  Matrices are ntypes x ntypes
 * column-major and must be symmetric; density has ntypes entries.  Types are
 * the reference's global type ids; the block's types are
 * type_start .. type_start+ntypes-1 (mat.type = minimum:maximum). */
typedef struct pd_material_desc {
    int32_t kind;                   /* PD_MAT_*                                  */
    int32_t ntypes;                 /* >= 1, <= 255                              */
    int64_t type_start;             /* first global type id of the block         */
    const double *bond_stiffness;   /* PMB: 18K/(pi*horizon^4) (bond_based.jl:58) */
    const double *bulk_modulus;     /* LPS: K                                     */
    const double *shear_modulus;    /* LPS: G                                     */
    const double *critical_stretch; /* all kinds (SKIP: ignored)                  */
    const double *density;          /* ntypes                                     */
    double horizon;
    double particle_size;           /* GeneralMaterial particle_size              */
    int64_t max_neigh;              /* GeneralMaterial max_neigh                  */
    const double *plastic_psi;      /* ELASTO_PLASTIC: psi = 75/(8 pi) sigma_e^2 /
                                       horizon^5 per type pair (elasto_plastic.jl:60-68) */
} pd_material_desc;

/* ---------------------------------------------------------------------- */
/* Library                                                                 */
/* ---------------------------------------------------------------------- */
PD_API int pd_abi_version(void);
PD_API const char *pd_status_string(pd_status s);
PD_API const char *pd_last_error(void);
/* Number of CUDA devices visible (0 when none). */
PD_API pd_status pd_device_count(int32_t *count);

/* ---------------------------------------------------------------------- */
/* Environment assembly: Env(id, materials, contacts, bcs, dt)             */
/* (src/environment.jl:166-235)                                           */
/* ---------------------------------------------------------------------- */
PD_API pd_status pd_env_create(pd_env **out, int32_t device, int32_t precision, double dt);
PD_API pd_status pd_env_destroy(pd_env *env);

/* Append one material block (GeneralMaterial(y0, v0, x, volume, type,
 * horizon; max_neigh), general_material.jl:81-98).  Blocks occupy
 * consecutive particle ranges in call order.  x, y, v: 3xn; volume: n;
 * type: n global type ids. */
PD_API pd_status pd_env_add_block(pd_env *env, int64_t n, const double *x, const double *y,
                           const double *v, const double *volume, const int64_t *type,
                           const pd_material_desc *mat, int64_t *out_block);

/* Replace the family of a block with one computed by the host (the
 * reference layout: rows x n, 1-based block-local, descending, 0 pad).
 * intact may be NULL (all entries > 0 intact).  Must precede finalize. */
PD_API pd_status pd_env_set_family(pd_env *env, int64_t block, int64_t rows, const int64_t *family,
                            const uint8_t *intact);

/* Contact model between blocks (kind PD_CONTACT_12, block1 -> pair[1],
 * block2 -> pair[2]) or within block1 (PD_CONTACT_11, block2 ignored).
 * equi_dist, distance, max_neighs as computed by ContactModel12_gcal /
 * ContactModel11_gcal (contacts.jl:76-124). */
PD_API pd_status pd_env_add_contact(pd_env *env, int32_t kind, int64_t block1, int64_t block2,
                             double exponent, double stiffness, double equi_dist,
                             double distance, int64_t max_neighs, int64_t *out_contact);

/* Boundary condition over all N particles of the environment (mask: N
 * bytes).  dims: 3 flags; rate: 3 values (TOFRO); freq: direction flip
 * period (INFINITY for MoveBC); applyafter: steps before flipping starts. */
PD_API pd_status pd_env_add_bc(pd_env *env, int32_t kind, const uint8_t *mask, const uint8_t *dims,
                        const double *rate, double freq, int64_t applyafter,
                        int32_t onlyatstart, int64_t *out_bc);

/* DeltaScaleBC(bool, scale, fixpoint; dims, onlyatstart) (DeltaScaleBC.jl:
 * 47-60): y = (last - fixpoint) * (1 + scale*dt*time_step) + fixpoint,
 * v = 0, last = y at apply_bc_at0.  kind PD_BC_DELTA_SCALE; wait and
 * scalemask are ignored.
 * ScaleFixWaitBC(bool, scale, fixpoint, wait, scalebool; dims, applyafter,
 * onlyatstart) (ScaleFixWaitBC.jl:46-71): y = last, v = 0, and at every
 * step with time_step % wait == 0 the particles of scalemask are scaled
 * about fixpoint by sqrt(1 + 2*scale*dt) and last is re-read.  kind
 * PD_BC_SCALE_FIX_WAIT.  scale, fixpoint: 3 values; masks: N bytes. */
PD_API pd_status pd_env_add_scaled_bc(pd_env *env, int32_t kind, const uint8_t *mask, const uint8_t *dims,
                                      const double *scale, const double *fixpoint, int64_t wait,
                                      const uint8_t *scalemask, int32_t onlyatstart, int64_t *out_bc);
/* ContainerBC(bool; limits, dims, onlyatstart) (ContainerBC.jl:48-74): the
 * velocity of a particle of the mask whose position leaves
 * [limits[d], limits[3 + d]] in a constrained dimension d is set to 0 in
 * those dimensions; positions are untouched.  limits: 3x2 column-major
 * (lower bounds, then upper bounds), or NULL for the reference's
 * limits=nothing form, which does nothing.  (The reference's constructor
 * tests an undefined name `limit`; this is the documented behaviour.) */
PD_API pd_status pd_env_add_container_bc(pd_env *env, const uint8_t *mask, const uint8_t *dims,
                                         const double *limits, int32_t onlyatstart, int64_t *out_bc);

/* Build everything on the device: families (GPU cell binning + sort,
 * peri.jl:459-576 and general_material.jl:85-90, unless set by
 * pd_env_set_family), weighted volumes (peri.jl:342-354), intact0
 * (environment.jl:169), masses/densities (environment.jl:173-214). */
PD_API pd_status pd_env_finalize(pd_env *env);

/* Sizes after finalize. */
PD_API pd_status pd_env_num_particles(const pd_env *env, int64_t *n);
PD_API pd_status pd_env_num_bonds(pd_env *env, int64_t *intact_bonds);
PD_API pd_status pd_env_family_rows(const pd_env *env, int64_t block, int64_t *rows);
/* Family / intact of a block in the reference layout (rows x n). */
PD_API pd_status pd_env_get_family(pd_env *env, int64_t block, int64_t *family, uint8_t *intact);
/* Weighted volume m of a block (n). */
PD_API pd_status pd_env_get_weighted_volume(pd_env *env, int64_t block, double *m);
/* Dilatation theta of an LPS block as of the last force evaluation (n). */
PD_API pd_status pd_env_get_theta(pd_env *env, int64_t block, double *theta);
/* Plastic deviatoric strain edp of an elasto-plastic block in the reference
 * layout (rows x n, column-major, aligned with pd_env_get_family). */
PD_API pd_status pd_env_get_plastic_strain(pd_env *env, int64_t block, double *edp);

/* ---------------------------------------------------------------------- */
/* State                                                                   */
/* ---------------------------------------------------------------------- */
/* Any pointer may be NULL.  3xN column-major. */
PD_API pd_status pd_env_get_state(pd_env *env, double *y, double *v, double *f, double *p);
PD_API pd_status pd_env_set_state(pd_env *env, const double *y, const double *v, const double *f);
/* Per-particle mass, volume and density (N each; NULL skips). */
PD_API pd_status pd_env_get_mass(pd_env *env, double *mass, double *volume, double *density);
PD_API pd_status pd_env_get_time_step(const pd_env *env, int64_t *time_step);
PD_API pd_status pd_env_set_time_step(pd_env *env, int64_t time_step);
/* Reset every intact flag to the state right after finalize. */
PD_API pd_status pd_env_reset_bonds(pd_env *env);
/* Reset the per-block "deformed" flags (general_material.jl:54, set when a
 * block first leaves rigid motion) to their state right after finalize. */
PD_API pd_status pd_env_reset_deformed(pd_env *env);

/* ---------------------------------------------------------------------- */
/* Solver entry points                                                     */
/* ---------------------------------------------------------------------- */
/* apply_bc_at0 (solvers.jl:200-206): snapshot BC.last = y[dims, bool]. */
PD_API pd_status pd_env_apply_bc_at0(pd_env *env);
/* update_acc! (solvers.jl:320-336): f = material + contact accelerations,
 * p = m v; breaks bonds with s >= critical stretch. */
PD_API pd_status pd_env_update_acc(pd_env *env);
/* nsteps x velocity_verlet_step! (velocity_verlet.jl:57-89). */
PD_API pd_status pd_env_vv_steps(pd_env *env, int64_t nsteps);
/* pd_env_vv_steps without waiting for the steps to finish (extension, no
 * reference counterpart): enqueues them on the environment's stream and
 * returns.  An environment whose blocks have all deformed, or whose gate
 * is held (pd_env_set_deformed), needs no read-back of the gate flags;
 * otherwise the call waits as pd_env_vv_steps does.  Errors of the
 * enqueued work surface at the next waiting call.  The slab decomposition
 * uses it to run slabs on several GPUs at once and to order its halo
 * exchange with events. */
PD_API pd_status pd_env_vv_steps_async(pd_env *env, int64_t nsteps);
/* minimize! (minimize.jl:105-231): one QSDrag solver step.  *iters
 * receives the iteration count (NULL allowed). */
PD_API pd_status pd_env_qsdrag(pd_env *env, double step_size, double drag, int64_t max_iter,
                        double x_tol, double f_tol, int64_t *iters);
/* update_neighs! (solvers.jl:351-361): contact neighbour lists. */
PD_API pd_status pd_env_update_neighs(pd_env *env, int64_t max_part);
/* Contact neighbour list in the reference layout (rows x n1 Int64, 1-based
 * into the pair[2] subset for 12, block-local for 11).  *rows receives
 * the row count; neighs may be NULL to query it. */
PD_API pd_status pd_env_get_contact_neighs(pd_env *env, int64_t contact, int64_t *rows,
                                    int64_t *neighs);

/* ---------------------------------------------------------------------- */
/* Diagnostics                                                             */
/* ---------------------------------------------------------------------- */
/* environment.jl:169 intact0: bonds per particle at finalize (environment
 * order; N_env values). */
PD_API pd_status pd_env_intact0(pd_env *env, int64_t *intact0);
/* cal_damage (peri.jl:587-594): N values. */
PD_API pd_status pd_env_damage(pd_env *env, double *damage);
/* printdata (environment.jl:308-320): out[0..2] = sum p, out[3..5] =
 * sum f, out[6] = mean damage, out[7] = intact bond count. */
PD_API pd_status pd_env_diagnostics(pd_env *env, double *out8);
/* 1 when every block has left the undeformed state (general_material.jl:
 * 243-255 gate), per block in flags (NULL allowed). */
PD_API pd_status pd_env_deformed(pd_env *env, uint8_t *flags);
/* PD_ERR_NAN when y, v or f holds a NaN or Inf (const_macros.jl:60-74). */
PD_API pd_status pd_env_check_finite(pd_env *env);
/* Bond storage of a finalized environment (extension, no reference
 * counterpart): out4[0] = 32-particle slices, out4[1] = slices stored as a
 * shared neighbour-offset stencil, out4[2] = bond slots, out4[3] = entries
 * of the neighbour-index array.  PD_FAMILY_LAYOUT=explicit in the process
 * environment at finalize disables the stencil form. */
PD_API pd_status pd_env_layout(const pd_env *env, int64_t *out4);
/* The same and more (extension): out[0..3] as pd_env_layout, out[4] =
 * slices with a record staging plan, out[5] = slots the step kernels walk
 * (per slice, 32 lanes x the slots up to the last family member of any of
 * its particles; bond slots also count the padding of each slice's slot
 * list to a multiple of 32, which no kernel walks).  Writes min(n, 6)
 * values. */
PD_API pd_status pd_env_layout_stats(const pd_env *env, int64_t *out, int64_t n);

/* Halo exchange of a slab decomposition of one specimen (extension: the
 * multi-GPU plan of a single large body; the reference runs one body on
 * one device).  idx: n environment-order particle indices, buf: 9 n
 * doubles, both in device memory of the environment's GPU.  Pack writes,
 * per particle, q (y in PD_PREC_FP64_SERIAL, the FP64 displacement u in
 * the throughput modes), v and f; unpack writes them into the listed
 * particles of another environment of the same precision, between steps.
 * Both enqueue on the environment's stream and return without waiting. */
PD_API pd_status pd_env_pack_halo(pd_env *env, const int64_t *idx, int64_t n, double *buf);
PD_API pd_status pd_env_unpack_halo(pd_env *env, const int64_t *idx, int64_t n, const double *buf);
/* Sets the per-block deformed flags of the general_material.jl:240-256
 * gate (extension).  hold != 0: the library no longer evaluates the gate
 * itself; the flags stay as set (slabs of one body: a gate decided on one
 * slab's particles would differ from the whole body's). */
PD_API pd_status pd_env_set_deformed(pd_env *env, const uint8_t *flags, int32_t hold);

/* ---------------------------------------------------------------------- */
/* Device-pointer entry point for a single block                           */
/* ---------------------------------------------------------------------- */
/* force_density_T!(f, y, limits, mat, Val{:cuda}) for block `block`, on
 * caller-owned DEVICE arrays of the whole environment (3xN column-major,
 * e.g. a CuArray's pointer): adds the block's accelerations into f over
 * its particle range and updates the block's intact flags, exactly as the
 * reference CPU loop does.  Runs the dilatation pass first for LPS.
 * stream: cudaStream_t (NULL = the environment's stream). */
PD_API pd_status pd_force_density_device(pd_env *env, int64_t block, double *f_dev,
                                  const double *y_dev, void *stream);

/* Same computation as pd_force_density_device, for callers that cannot
 * allocate device memory during the call (a host whose GPU memory belongs
 * to another allocator's pool, or a time-step loop that must not take the
 * implicit synchronisation of cudaMalloc/cudaFree).  It has no counterpart
 * in the reference.  Its scratch is a fixed device array compiled into the
 * library (4 MiB per GPU, held until exit): the block may hold at most 65536
 * particles (padded to a multiple of 32), larger blocks get
 * PD_ERR_UNSUPPORTED.  All calls on one GPU share that array, so calls that
 * overlap on the GPU race; the first call on each device looks the array
 * up and should precede any stream capture on that device.  The address is
 * kept until exit: do not reset the device while the library is loaded. */
PD_API pd_status pd_force_density_device_static(pd_env *env, int64_t block, double *f_dev,
                                                const double *y_dev, void *stream);

/* ---------------------------------------------------------------------- */
/* Instrumentation                                                         */
/* ---------------------------------------------------------------------- */
/* The environment's CUDA stream (cudaStream_t) -- for timing with events. */
PD_API pd_status pd_env_stream(pd_env *env, void **stream);
/* Total kernel launches issued by the library since it was loaded. */
PD_API pd_status pd_kernel_launches(int64_t *count);
/* enable != 0: bracket the bond kernels of every step (dilatation,
 * td_norm2 and force; in the throughput modes each replay of a captured
 * multi-step graph as a whole) with CUDA events on the environment's
 * stream, without changing how steps are launched; resets the accumulated
 * time.  pd_env_profile_read returns the summed device time (ms) and the
 * number of steps it covers since enabling. */
PD_API pd_status pd_env_profile(pd_env *env, int32_t enable);
PD_API pd_status pd_env_profile_read(pd_env *env, double *total_ms, int64_t *launches);
/* Kernel shape of the throughput modes (extension): warps per 32-particle
 * slice (1, 2, 4, 8) and bonds in flight per thread (FP32C: 2 or 4, FP64:
 * 1 or 2).  (0, 0) returns to the autotuner, which times every shape on
 * the first step and caches the fastest per problem size. */
PD_API pd_status pd_env_set_kernel_shape(pd_env *env, int32_t warps_per_slice, int32_t unroll);
/* The shape the throughput path runs with (after autotuning); (0, 0)
 * before the first throughput-mode step or in the serial mode. */
PD_API pd_status pd_env_kernel_shape(pd_env *env, int32_t *warps_per_slice, int32_t *unroll);
/* Record staging of the FP32C kernels (extension): a stencil slice's
 * neighbour records -- a few ranges of consecutive records -- are copied
 * into shared memory by bulk asynchronous copies before its bonds are
 * walked, with 4 or 8 warps per slice.  mode 0 (default): never; 1: staged
 * shapes only (with a fixed kernel shape: its staged form); 2: the
 * autotuner times staged and unstaged shapes.  Results are identical
 * either way. */
PD_API pd_status pd_env_set_record_staging(pd_env *env, int32_t mode);
/* staged = 1 when the running FP32C shape stages; slices with a staging
 * plan and the largest plan in records (any pointer may be NULL). */
PD_API pd_status pd_env_record_staging(pd_env *env, int32_t *staged, int64_t *slices, int64_t *max_records);
/* Measured pipe rates of GPU `device` (extension; the compute-side
 * denominators of the bond walk's roofline), each the best of three ~10 ms
 * launches over every SM: out[0] FP32 FMA and out[1] packed f32x2 FMA lane
 * operations per second, out[2] MUFU sqrt.approx and out[3] MUFU
 * rcp.approx lane operations per second, out[4] warp instructions issued
 * per second by a mix of FP32 FMA and integer logic (both pipes busy). */
PD_API pd_status pd_pipe_peaks(int32_t device, double *out5);

/* ---------------------------------------------------------------------- */
/* Serving (extension): a request loop that admits simulation jobs by HBM  */
/* footprint, keeps their state resident and advances every admitted job   */
/* on its own stream in chunks, so the work of jobs that arrive while      */
/* others run overlaps on the device (continuous batching).  Thread-safe.  */
/* ---------------------------------------------------------------------- */
typedef struct pd_server pd_server;
enum { PD_JOB_QUEUED = 0, PD_JOB_RUNNING = 1, PD_JOB_DONE = 2, PD_JOB_FAILED = 3, PD_JOB_CANCELLED = 4 };
typedef struct pd_job_info {
    int32_t state;            /* PD_JOB_* */
    int32_t status;           /* pd_status of a failed job, else PD_OK */
    int64_t steps_done;       /* velocity-Verlet steps completed */
    int64_t particles;        /* environment particles */
    int64_t footprint_bytes;  /* HBM reserved at admission */
    int64_t bond_updates;     /* intact directed bonds x steps (mean of start and end) */
    double queue_ms;          /* submit -> admission */
    double latency_ms;        /* submit -> completion (0 until done) */
} pd_job_info;
/* hbm_budget_bytes <= 0: 90% of the device's free memory at creation.
 * max_active: jobs resident at once.  chunk_steps: steps a job advances
 * per scheduling round (rounded to the graph replay length when larger). */
PD_API pd_status pd_server_create(pd_server **out, int32_t device, int64_t hbm_budget_bytes, int32_t max_active,
                                  int64_t chunk_steps);
/* Takes ownership of an assembled, NOT finalized environment (blocks, BCs
 * and contacts added) on the server's device; the server finalizes it at
 * admission, applies the BC snapshot and the initial force evaluation
 * (run!'s save_state! at t0, solvers.jl:97-187), then advances nsteps
 * velocity-Verlet steps.  The kernel shape of throughput-mode jobs is fixed
 * from the problem size (not timed), so a job's result does not depend on
 * what else runs beside it. */
PD_API pd_status pd_server_submit(pd_server *srv, pd_env *env, int64_t nsteps, int64_t *job);
PD_API pd_status pd_server_poll(pd_server *srv, int64_t job, pd_job_info *info);
/* Blocks until the job is done, failed or cancelled, or timeout_s passes
 * (PD_ERR_TIMEOUT). */
PD_API pd_status pd_server_wait(pd_server *srv, int64_t job, double timeout_s, pd_job_info *info);
/* Final state of a done job in environment order (y, v: 3 x N column-major;
 * damage: N; any may be NULL); releases the job's record. */
PD_API pd_status pd_server_result(pd_server *srv, int64_t job, double *y, double *v, double *damage);
PD_API pd_status pd_server_cancel(pd_server *srv, int64_t job);
/* ---------------------------------------------------------------------- */
/* Output staging (extension): the save_state! snapshot (io.jl:44-54)       */
/* without stalling the time loop.                                        */
/* ---------------------------------------------------------------------- */
/* Enqueue a snapshot of y, v, f (and damage) into staging slot 0 or 1: the
 * state is packed on the environment's stream and copied to pinned host
 * memory on a separate copy stream, so later steps run while the copy is in
 * flight.  A slot holds one snapshot; staging into a slot whose previous
 * snapshot was not read first waits for that copy. */
PD_API pd_status pd_env_stage_state(pd_env *env, int32_t slot);
/* Wait for the slot's copy and return it in environment order (y, v, f:
 * 3 x N column-major; damage: N; any may be NULL) with the time_step it was
 * taken at.  PD_ERR_STATE when nothing is staged in the slot. */
PD_API pd_status pd_env_stage_read(pd_env *env, int32_t slot, double *y, double *v, double *f, double *damage,
                                   int64_t *time_step);

/* Cancels queued and running jobs and joins the worker. */
PD_API pd_status pd_server_destroy(pd_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* PERIDYN_B200_H */
