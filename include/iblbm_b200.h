/*
 * iblbm_b200.h — C ABI of the B200-native IB-LBM hot path (libiblbm_b200.so).
 *
 * Plain C: device pointers are `void*`/typed pointers into CUDA global memory
 * (any allocator; the Python host uses PyTorch tensors), sizes are ints, the
 * stream is a `cudaStream_t` passed as `void*`.  Every entry point returns 0 on
 * success and a negative IBLBM_E_* code on a rejected argument or a CUDA launch
 * error; kernels that can fail at run time (bounded iteration, capacity) report
 * through a device-side status word that the caller reads.
 *
 * The reference (mulgae-life/iblbm-mechanism-resolved) binds its GPU path from
 * Python through CuPy RawModule kernels wrapped in iblbm/gpu_kernels.py; the
 * "Replaces" line of each entry point names the wrapper and its caller it
 * stands in for.  Population arrays of the reference-shaped entry points use
 * the reference's AoS layout f[n*9 + q], n = j*nx + i; the fused step engine
 * uses the pitched structure-of-arrays layout described by iblbm_geom.
 */
#ifndef IBLBM_B200_H
#define IBLBM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define IBLBM_OK 0
#define IBLBM_E_ARG -1      /* bad argument (null pointer, size, unknown id) */
#define IBLBM_E_LAUNCH -2   /* CUDA launch / configuration error */
#define IBLBM_E_CAPACITY -3 /* a size exceeds the scratch capacity the caller provided */

/* collision ids */
#define IBLBM_COLL_BGK 0
#define IBLBM_COLL_TRT 1
#define IBLBM_COLL_CMMRT 2
/* boundary closure ids (iblbm/boundary/*.py) */
#define IBLBM_BC_DIRICHLET_NEUMANN 0
#define IBLBM_BC_OPEN 1
#define IBLBM_BC_SETTLING 2
#define IBLBM_BC_VELOCITY_INLET 3
#define IBLBM_BC_TG 4 /* Taylor-Green analytic faces (iblbm/boundary/tg_analytical.py) */
/* immersed-boundary method ids (iblbm/ibm/strategies/*.py) */
#define IBLBM_IBM_NONE 0
#define IBLBM_IBM_DF 1
#define IBLBM_IBM_MDF 2
#define IBLBM_IBM_DFC 3
/* delta kernel ids (iblbm/ibm/common.py:52-119) */
#define IBLBM_DELTA_PESKIN4 0
#define IBLBM_DELTA_HAT 1

/* Lattice geometry of the fused engine: population q of node (i, j) is element
 * q*qstride + j*pitch + i of a population buffer; pitch >= nx is a multiple of 32. */
typedef struct {
    int nx, ny, pitch;
    long long qstride;
} iblbm_geom;

/* Physical/numerical parameters of one lattice case (host-computed with the
 * reference's formulas, iblbm/init.py:116-265 and lbm/collision/*.py). */
typedef struct {
    int collision;       /* IBLBM_COLL_* */
    int bc;              /* IBLBM_BC_* */
    int incompressible;  /* SimConfig.incompressible_lbgk */
    double tau, dt;
    double s_minus;      /* TRT: 1/tau_minus */
    double S[9];         /* CM-MRT relaxation rates */
    double inflow_u, dens;
    /* IBLBM_BC_TG only (else NULL): the analytic velocity of every boundary node
     * without its decay factor, (ux, uy) pairs for the left face j = 0..ny-1, the
     * right face j = 0..ny-1, the bottom face i = 1..nx-2, the top face
     * i = 1..nx-2 and the corners (0,0), (nx-1,0), (0,ny-1), (nx-1,ny-1); and a
     * device scalar holding the decay factor of the current step.  The closure
     * imposes tg_face * (*tg_decay). */
    const double *tg_face;
    const double *tg_decay;
} iblbm_case;

/* Band: the lattice nodes under the marker stencils.  `box` holds x0, y0, w, h
 * of the box enclosing the band; `map` is a full-lattice int array (nx*ny) that
 * holds the band index of band nodes and -1 elsewhere inside the box. */
typedef struct {
    const int *box;
    const int *map;
    const double *fib;  /* band x 2: IB force density (DF/MDF) */
    const double *df;   /* band x 9: distribution correction (DFC) */
} iblbm_band_view;

/* One fused timestep over the whole lattice (FP64, the reference's arithmetic):
 * pull-streaming from fpost_prev, boundary closure, band correction, macroscopic
 * moments, velocity correction, equilibrium and collision into fpost_next.
 * Optional outputs (may be NULL): ro/U (nx*ny, nx*ny*2, AoS) after the velocity
 * correction, fstar (SoA like fpost) after streaming/closure/DFC. */
typedef struct {
    iblbm_geom g;
    iblbm_case c;
    int ibm;                    /* IBLBM_IBM_* applied on the band */
    const double *fpost_prev;   /* SoA, 9 * qstride */
    double *fpost_next;
    const double *uring_prev;   /* nx*ny*2, previous step's U on rows/cols 1,2,n-3,n-2 */
    double *uring_next;
    iblbm_band_view band;
    double *ro_out, *U_out, *fstar_out;
    const int *skip_box;        /* device x0, y0, w, h: nodes left to the box pass (NULL: none) */
    const int *only_box;        /* device x0, y0, w, h: update only these nodes (box pass; NULL: all) */
    int box_blocks;             /* grid of the box pass (blocks of 128 threads, grid-stride) */
} iblbm_dense_args;

/* Replaces (fused): collision_gpu/collision_trt_gpu/collision_cm_mrt_gpu
 * (iblbm/gpu_kernels.py:760-843), streaming_gpu (:846-875), the boundary
 * closures (iblbm/boundary/*.py apply_bc_*), macroscopic_gpu (:878-903),
 * velocity_correction_gpu (:930-948) and feq_gpu (:906-927), in the order of
 * iblbm/runtime/loop.py:63-138. */
int iblbm_dense_step_f64(const iblbm_dense_args *a, void *stream);

/* Immersed-boundary band step (one CTA): rebuilds the band from the current
 * markers (when `rebuild` or the markers move), computes the post-streaming
 * populations and moments on the band, and runs DF / MDF / coupled MDF / DFC.
 * Marker positions are in domain units (x / dx is the lattice coordinate). */
typedef struct {
    iblbm_geom g;
    iblbm_case c;
    int method;        /* IBLBM_IBM_DF / MDF / DFC */
    int delta_type;    /* IBLBM_DELTA_* */
    int rebuild;       /* 1: rebuild stencils, band and lists this step */
    int n_particles;   /* >= 1; markers of particle p are [moff[p], moff[p+1]) */
    int lb_total;      /* moff[n_particles] (sizes the shared-memory marker arrays) */
    const int *moff;   /* device, n_particles + 1 */
    const double *Lx, *Ly;   /* device, marker positions (Lb_total) */
    const double *dvel;      /* device, desired velocity (Lb_total x 2) */
    const double *larea;     /* device, arc length per particle */
    double dx, dy;
    /* motion from a table: when xt_table != NULL the markers this step are
     * Lx = Lx_c - xt_table[*step_counter], desired velocity (xt, 0)
     * (iblbm/physics/motion.py:15-52); step_counter is incremented. */
    const double *Lx_c, *Ly_c, *xt_table;
    int *step_counter;
    int xt_len;        /* entries in xt_table; a counter past the end sets status 4 */
    /* MDF */
    int mdf_iterations, mdf_min_iterations, mdf_coupled;
    double mdf_omega, mdf_tol, mdf_omega_max;
    /* DFC */
    double *lambda;    /* Lb_total: lambda(k) */
    int *lambda_valid; /* device flag: lambda holds a cached value */
    int dfc_cache_lambda; /* 1 for fixed bodies: compute lambda once, then reuse (strategies/dfc.py:32,48-49) */
    double correction_scale;
    /* inputs */
    const double *fpost_prev, *uring_prev;
    /* band state (written) */
    int *box, *map, *band_nodes, *band_count; /* map: nx*ny ints, -1 outside the band */
    int *list_cache;   /* iblbm_ibm_list_cache_ints(...) ints: contribution lists kept between steps */
    const int *excl_cur;  /* optional: this step's exclusion box; the band must lie inside (status 5) */
    int *excl_next;       /* optional: written with the band box dilated by one node */
    int band_capacity, box_capacity;
    double *band_fib, *band_df;        /* band x 2, band x 9 */
    double *band_fib_part;             /* particles x band_capacity x 2 (per-particle totals) */
    double *scratch;                   /* >= iblbm_ibm_scratch_doubles(...) doubles */
    int *iscratch;                     /* >= iblbm_ibm_scratch_ints(...) ints */
    /* per-marker outputs (Lb_total): interpolated velocity, force, DFC force */
    double *Lux, *Luy, *Lfx, *Lfy, *dfc_force;
    /* stats: [iter_count, diverged, converged, guard_trips, status]
     * (guard_trips: coupled MDF; -1 when the FP32 band step ran a single
     * body's MDF iterations in marker space, -2 when the FP64 step ran them in
     * the restructured node-space loop), dstats: [last_residual, omega_used] */
    int *stats;
    double *dstats;
    /* reference-shaped calls (iblbm/gpu_kernels.py:956-1223): the band takes
     * its moments from the given fields instead of the lattice (fpost_prev and
     * uring_prev unused).  DF / MDF read density field_ro[n] and velocity
     * (field_ux[n * s], field_uy[n * s]), s = field_ustride, n = j*nx + i;
     * DFC reads the post-streaming populations field_fstar[9n + q].  NULL: off. */
    const double *field_ro, *field_ux, *field_uy, *field_fstar;
    int field_ustride;
    /* NULL, or a device scalar scaling every desired velocity this step
     * (dvel * (*dvel_scale); the Taylor-Green markers' analytic decay) */
    const double *dvel_scale;
    /* DFC: fluid density rho_f of lambda(k) = 1 / (2 rho_f ds W_sum(k))
     * (iblbm/ibm/dfc.py:126-186); 0 means 1.0, the solver's value */
    double dfc_rho_f;
    /* polls of each bounded wait on a bulk copy before the step gives up with
     * status 6 (0: the default, 2^22) */
    long long wait_limit;
    /* failure-path testing only (0 in normal use): 1 skips issuing a fixed
     * body's restore copy while its wait still expects it, so the wait runs
     * out and the step reports status 6 with no copy in flight */
    int test_skip_copy;
    /* MDF of one fixed body on a thread-block cluster of cluster_size CTAs
     * (2, 4 or 8) instead of one CTA: NULL / 0 keep the single-CTA step.  The
     * plan (iblbm_ibm_cluster_plan_ints(lb_total, delta_type, cluster_size)
     * ints, 8-byte aligned) is built by every rebuild step and read by the
     * steps after it, so pass the same buffer on every step of the body.
     * Results are bit for bit those of the single-CTA step; stats[3] is -3
     * when the cluster ran the iterations. */
    int *cluster_plan;
    int cluster_size;
    /* DF only: 1 spreads the marker forces given in Lfx / Lfy (inputs) instead
     * of computing them from the velocity (the spreading half of the
     * reference's raw DF kernels); Lux / Luy are then left 0 */
    int df_given_force;
} iblbm_ibm_args;

/* Replaces: ibm_direct_forcing_gpu (iblbm/gpu_kernels.py:956-1042) called from
 * ibm/strategies/df.py:27-49, the MDF loop of iblbm/ibm/mdf.py:61-229 (and the
 * coupled multi-particle loop of iblbm/ibm/multi_particle.py:62-316), and
 * compute_lambda_gpu + dfc_correction_gpu (gpu_kernels.py:1091-1223) called
 * from ibm/strategies/dfc.py:31-54.
 * Sizes: the band layout (iblbm_ibm_smem_bytes) lives in shared memory while it
 * fits (220 KB); beyond that the step keeps its contribution lists and stencil
 * weights in list_cache (global memory, L2-resident) and only the per-step
 * arrays on chip, so a single body of any marker count within the other limits
 * runs (band_capacity <= 2048; an MDF body <= 512 markers). */
int iblbm_ibm_step_f64(const iblbm_ibm_args *a, void *stream);
/* Ints of the cluster plan of one body (iblbm_ibm_args.cluster_plan), or 0
 * when a body of lb_total markers cannot run on a cluster of that size (a
 * CTA holds its markers' warps and one thread per band node under their
 * stencils; a band whose ranks cover more nodes than a CTA has threads left
 * steps through the single-CTA fallback).  No reference counterpart. */
int iblbm_ibm_cluster_plan_ints(int lb_total, int delta_type, int cluster_size);
/* Same band step for callers that cannot allocate device memory at call time
 * (a host framework that owns all device allocations, or a service that
 * forbids cudaMalloc after start-up).  No counterpart in the reference.  The
 * scratch and iscratch fields of *a are ignored: the per-launch scratch comes
 * from a fixed array in the library (about 230 KB per GPU, held until exit).
 * Limits: band_capacity <= 2048, lb_total <= 1024, else IBLBM_E_CAPACITY.
 * Calls share that array, so calls that overlap on the GPU race; the first
 * call on a device resolves the array's address and should precede any stream
 * capture.  The address is kept for the life of the process (it assumes the
 * device's primary context lives as long: no call after cudaDeviceReset).
 * Allocates nothing. */
int iblbm_ibm_step_f64_noalloc(const iblbm_ibm_args *a, void *stream);
/* The plain form of the batched sweep: band steps of n independent cases in
 * one launch (one CTA per case), as iblbm_ibm_step_f32_batch on the FP64
 * lattice; each case's results are bit for bit those of iblbm_ibm_step_f64.
 * No reference counterpart (the reference steps one case at a time). */
int iblbm_ibm_step_f64_batch(const iblbm_ibm_args *host_args, const iblbm_ibm_args *dev_args, int n,
                             void *stream);
/* The FP64 collide-stream pass of n <= 72 cases of one kind (collision,
 * closure, compressibility, band method; all bulk/whole-lattice or all box
 * passes) in one launch, lattices of any size; no ro/U/fstar outputs, no
 * Taylor-Green closure.  Same per-node arithmetic as iblbm_dense_step_f64, so
 * bit-identical per case.  No reference counterpart. */
int iblbm_dense_step_f64_batch(const iblbm_dense_args *a, int n, void *stream);
int iblbm_ibm_scratch_doubles(int lb_total, int band_capacity, int n_particles);
int iblbm_ibm_scratch_ints(int lb_total, int band_capacity, int delta_type);
int iblbm_ibm_list_cache_ints(int lb_total, int band_capacity, int delta_type);
/* Shared memory of the band layout of one band step (lists, weights, band
 * moments); the step itself adds what its options need and checks the total. */
int iblbm_ibm_smem_bytes(int lb_total, int band_capacity, int delta_type);

/* ---- FP32 shifted-population form ----------------------------------------
 * Populations are held as deviations g = f - w from the lattice weights, in
 * FP32 (72 bytes per lattice update instead of 144).  Equilibria, closures and
 * collisions are rewritten on g (rho = 1 + sum g); marker positions, desired
 * velocities, per-marker forces, the MDF residual norm and everything downstream
 * of the marker forces (force sums, Newton-Euler) stay FP64.  Same layout and
 * schedule as the FP64 entries; no reference counterpart (the reference is
 * FP64 throughout), the FP64 entries are its drop-in. */
typedef struct {
    const int *box;
    const int *map;
    const float *fib;   /* band x 2 */
    const float *df;    /* band x 9 */
} iblbm_band_view32;

typedef struct {
    iblbm_geom g;
    iblbm_case c;               /* FP64 parameters, rounded to FP32 at launch */
    int ibm;
    const float *fpost_prev;    /* SoA deviations g = f - w */
    float *fpost_next;
    const float *uring_prev;
    float *uring_next;
    iblbm_band_view32 band;
    float *ro_out, *U_out, *fstar_out;  /* ro is rho (not rho - 1); fstar is shifted */
    const int *skip_box;
    const int *only_box;
    int box_blocks;
    int tile;      /* IBLBM_TILE_*: shape of the whole-lattice / bulk pass */
    int *status;   /* optional device int: set to 1 if a pipeline wait ran out */
    /* PIPE tiles: polls of each bounded pipeline wait (0: the default, 2^24);
     * test_skip_copy = 1 (failure-path testing only) makes the producer issue
     * no copy, so the consumers' waits run out (status 1, nothing in flight) */
    long long wait_limit;
    int test_skip_copy;
} iblbm_dense32_args;

/* Tile shapes of the FP32 pass.  PIPE_RxS: persistent CTAs of R consumer warps
 * (R lattice rows x 128 columns per tile) and one producer warp staging S tiles
 * ahead in shared memory with bulk copies; NODE: one thread per node; ROWSn:
 * one thread per n nodes stacked in y, all their loads issued first.  Population
 * buffers must be 16-byte aligned (pitch a multiple of 32 as everywhere).
 * Output steps (ro/U/fstar requested) use NODE. */
#define IBLBM_TILE_PIPE_4x2 0
#define IBLBM_TILE_NODE 1
#define IBLBM_TILE_PIPE_8x2 2
#define IBLBM_TILE_ROWS2 3
#define IBLBM_TILE_ROWS4 4

/* Fused timestep on the shifted FP32 form (see iblbm_dense_step_f64). */
int iblbm_dense_step_f32(const iblbm_dense32_args *a, void *stream);
/* The pass of n <= 72 independent cases of one kind (same collision, closure,
 * compressibility, band method, and all bulk/whole-lattice or all box passes)
 * in one launch; lattices may differ in size.  Bulk passes without a band
 * (ibm = IBLBM_IBM_NONE, no only_box) may mix kinds: each CTA then dispatches
 * on its case's collision, closure and compressibility.  The Taylor-Green
 * closure (IBLBM_BC_TG) is not batched.  Tile NODE, ROWS2 or ROWS4 (taken
 * from a[0]); no ro/U/fstar outputs.  Host threads may call it concurrently
 * (the parameter block is built per call). */
int iblbm_dense_step_f32_batch(const iblbm_dense32_args *a, int n, void *stream);
/* f (FP64 AoS, the reference's f[N, 9]) -> g = f - w (FP32 SoA), and back. */
int iblbm_to_shifted_f32(const double *aos, iblbm_geom g, float *soa, void *stream);
int iblbm_from_shifted_f32(const float *soa, iblbm_geom g, double *aos, void *stream);

/* Band step on the shifted FP32 lattice.  Fields as iblbm_ibm_args; the
 * lattice inputs, band forces/corrections and scratch are FP32, the marker
 * arrays and per-marker outputs FP64. */
typedef struct {
    iblbm_geom g;
    iblbm_case c;
    int method, delta_type, rebuild, n_particles, lb_total;
    const int *moff;
    const double *Lx, *Ly;
    const double *dvel;
    const double *larea;
    double dx, dy;
    const double *Lx_c, *Ly_c, *xt_table;
    int *step_counter;
    int xt_len;
    int mdf_iterations, mdf_min_iterations, mdf_coupled;
    double mdf_omega, mdf_tol, mdf_omega_max;
    double *lambda;
    int *lambda_valid;
    int dfc_cache_lambda;
    double correction_scale;
    const float *fpost_prev, *uring_prev;
    int *box, *map, *band_nodes, *band_count;
    int *list_cache;   /* iblbm_ibm32_list_cache_ints(...) ints */
    const int *excl_cur;
    int *excl_next;
    int band_capacity, box_capacity;
    float *band_fib, *band_df;
    float *band_fib_part;
    float *scratch;    /* >= iblbm_ibm_scratch_doubles(...) floats */
    int *iscratch;
    double *Lux, *Luy, *Lfx, *Lfy, *dfc_force;
    int *stats;
    double *dstats;
    const float *field_ro, *field_ux, *field_uy, *field_fstar;
    int field_ustride;
    const double *dvel_scale;
    double dfc_rho_f;
    long long wait_limit;
    int test_skip_copy;
    int *cluster_plan;  /* not used by the FP32 step yet: NULL / 0 */
    int cluster_size;
    int df_given_force;
    /* learned MDF warm start (single-body MDF only): mlp_mode bit 1 writes each
     * marker's 64 features before the MDF loop (mlp_features, lb_total x 64) and
     * the force it accumulates, sum over iterations of omega * Lf (mlp_targets,
     * lb_total x 2); bit 2 predicts that force with the network in mlp_params
     * (iblbm_mlp_param_count() floats) and starts the loop from it.  mlp_uref
     * scales velocities (the inflow speed), mlp_re is the Reynolds number. */
    int mlp_mode;
    float mlp_uref, mlp_re;
    const float *mlp_params;
    float *mlp_features, *mlp_targets;
} iblbm_ibm32_args;

/* Sizes as iblbm_ibm_step_f64. */
int iblbm_ibm_step_f32(const iblbm_ibm32_args *a, void *stream);
/* Band steps of n independent cases in one launch (one CTA per case; stencil,
 * method and coupling may differ between cases).  host_args and dev_args hold
 * the same n argument blocks, on the host (checked here, sizes the shared
 * memory) and in device memory (read by the kernel).  Every case's band layout
 * must fit in shared memory (else IBLBM_E_CAPACITY): a larger body is stepped
 * on its own. */
int iblbm_ibm_step_f32_batch(const iblbm_ibm32_args *host_args, const iblbm_ibm32_args *dev_args, int n,
                             void *stream);
int iblbm_ibm32_list_cache_ints(int lb_total, int band_capacity, int delta_type);
/* As iblbm_ibm_smem_bytes; a single body's MDF step adds the marker coupling
 * matrix when it fits, and the learned warm start its buffers. */
int iblbm_ibm32_smem_bytes(int lb_total, int band_capacity, int delta_type);

/* ---- learned MDF warm start: the network's training and inference ---------
 * A 64 -> 64 -> 64 -> 64 -> 2 ReLU MLP in FP32 whose parameter block holds the
 * feature normalisation (mean, inverse scale), the target scales and the
 * weights (layout in csrc/mlp.cuh: hidden weight rows padded to 72 floats).
 * The hidden layers run on the tensor cores (TF32 operands, FP32
 * accumulation).  No reference counterpart: the reference has no learned
 * component. */
int iblbm_mlp_param_count(void);
/* Floats of the gradient buffer of a training step on n samples: the summed
 * gradient (param_count floats, padded), then one slot per 64 samples. */
int iblbm_mlp_grad_floats(int n);
/* y[n x 2] = network(x[n x 64]) in the targets' units. */
int iblbm_mlp_infer(const float *params, const float *x, int n, float *y, void *stream);
/* One training step on n samples (x[n x 64], t[n x 2]), mean squared error on
 * the scaled targets; deterministic (every block of 64 samples writes its own
 * gradient slot, a second launch sums the slots in order).  grad holds
 * iblbm_mlp_grad_floats(n) floats (no initial contents needed).  apply = 1:
 * Adam (step >= 1, learning rate lr; adam_m / adam_v: param_count floats
 * each); apply = 0: the summed gradient is left in grad[0 .. param_count).
 * loss (optional) has the batch loss added to it. */
int iblbm_mlp_train_step(float *params, float *adam_m, float *adam_v, float *grad, const float *x, const float *t,
                         int n, float lr, int step, float *loss, int apply, void *stream);

/* ---- rigid particles of sedimentation runs on the device -------------------
 * Replaces the host particle steps of runtime/scenarios/sedimentation_multi.py:
 * the Velocity-Verlet step (:36-111, with the angular half and full kicks of
 * physics/rigid_body.py:65-82 when rotation is on) and the explicit Euler step
 * (:126-190, physics/rigid_body.py:84-121), inertia models none /
 * explicit_history / feng_b2.  Per particle, state holds
 * IBLBM_PARTICLE_STATE doubles: pos(2), vel(2), vel_prev(2), vel_half(2),
 * force(2), pos_next(2), omega, omega_half, angle, torque, and the half step's
 * look-ahead vel_half(2), omega_half, angle of the next step (pos_next,
 * vel_half, omega_half and angle become current in its full step, so between
 * launches the state is that of the last completed step), then the omega of
 * the last step's rigid-body marker velocity, and the fluid's angular
 * momentum inside the disc at the last Euler step; consts holds
 * IBLBM_PARTICLE_CONSTS doubles: mass, 1/rho_ratio, pi r^2/mass, net gravity
 * (2), initial centre (2), moment of inertia, disc radius (domain units),
 * marker arc length.  phase FULL finishes the
 * current Verlet step from the band kernel's per-particle forces
 * (band_fib_part, particles x band_capacity x 2, FP32 when fib_f32); phase HALF
 * starts the next one: new marker positions Lx, Ly and desired velocities
 * dvel; phase EULER (alone) does a whole explicit Euler step after the band
 * kernel (with rotation: after the whole lattice pass) and leaves the next
 * step's markers and desired velocities. */
#define IBLBM_PARTICLE_STATE 22
#define IBLBM_PARTICLE_CONSTS 10
#define IBLBM_PARTICLES_FULL 1
#define IBLBM_PARTICLES_HALF 2
#define IBLBM_PARTICLES_EULER 4
#define IBLBM_INERTIA_NONE 0
#define IBLBM_INERTIA_EXPLICIT_HISTORY 1
#define IBLBM_INERTIA_FENG_B2 2
#define IBLBM_LAGRANGIAN_DF 1
#define IBLBM_LAGRANGIAN_DFC 2
typedef struct {
    int n_particles, phase, model, fib_f32;
    const int *moff;
    const double *Lx_c, *Ly_c;
    double *Lx, *Ly, *dvel;
    double *state;
    const double *consts;
    double dt, dx;
    const void *band_fib_part;
    const int *band_count;
    int band_capacity;
    double *forces_out;   /* optional: particles x 2, the forces of the full step */
    /* Optional (pw_leaf NULL: a fixed tree order instead): each force as numpy
     * sums the reference's dense n_nodes x 2 force field (np.sum, pairwise
     * summation), bit for bit.  The summation tree depends only on n_nodes and
     * comes from the host (iblbm_b200.physics.pairwise_tree): pw_leaf holds the
     * (offset, length) of its pw_leaves leaf blocks left to right, pw_node the
     * two child ids of each of its pw_internal inner nodes (ids below
     * pw_leaves are leaves, inner node k has id pw_leaves + k), ordered by
     * depth from the deepest, pw_level[d] .. pw_level[d + 1] the nodes of the
     * d-th group; pw_lut[i] the leaf holding element 64 i and pw_span the
     * first and last leaf under each inner node (pairwise_tree_index).
     * band_nodes: the band's lattice indices, ascending.  pw_scratch:
     * (pw_leaves + pw_internal) x 2 x n_particles doubles. */
    int n_nodes;
    const int *band_nodes;
    int pw_leaves, pw_internal, pw_levels;
    const int *pw_leaf;
    const int *pw_node;
    const int *pw_level;
    const int *pw_lut;
    const int *pw_span;
    double *pw_scratch;
    /* Rotation (Verlet only): the torque T = -sum over the lattice of
     * (i - x/dx) fy - (j - y/dy) fx (node (i, j) = band_nodes entry e as
     * (e % nx, e / nx), x, y the centre), summed like the forces; markers
     * X = R(angle) (X_c - X_0) + x; semi_implicit adds omega x r to the desired
     * velocity (physics/markers.py:41-60).  Needs band_nodes and nx.
     * euler_trapezoidal: the position update of the Euler step with the mean of
     * the old and new velocities (else the new one). */
    int rotation, semi_implicit, euler_trapezoidal, nx;
    double dy;
    /* Rotating Euler steps (physics/rigid_body.py:101-121): the change of the
     * fluid's angular momentum inside each disc, sum over the lattice nodes
     * within the disc radius of (i - x/dx) rho uy - (j - y/dx) rho ux, taken
     * from this step's rho and U (n_nodes and n_nodes x 2, FP32 when
     * moments_f32) over the box of diagnostics/internal_flow.py:220-262 and
     * summed like numpy sums the masked values.  The launch follows the whole
     * lattice pass.  lint_scratch: lint_capacity doubles, at least the
     * largest box, (2 (int(r/dx) + 2) + 1)^2. */
    const void *rho, *U;
    int moments_f32, ny;
    double *lint_scratch;
    int lint_capacity;
    /* lagrangian: IBLBM_LAGRANGIAN_DF / _DFC take each particle's force and
     * torque from its markers' forces instead of the band field (multi-particle
     * DF: Lfx, Lfy times the particle's arc length, consts[9]; DFC: dfc_force,
     * markers x 2), summed over its markers like numpy; lint_scratch then holds
     * at least the most markers of a particle. */
    int lagrangian;
    const double *Lfx, *Lfy, *dfc_force;
    /* half_kick_omega: the semi-implicit marker velocity takes the step's
     * half-kicked omega, as the single-particle runtime does
     * (runtime/scenarios/sedimentation_single.py:148-158), not the last step's. */
    int half_kick_omega;
    /* prescribed: the disc moves at prescribed_velocity (lattice units per step,
     * runtime/scenarios/sedimentation_single.py:91-97,174-180): the half step
     * moves it and its markers, whose desired velocity is that velocity, and the
     * full step records the force and keeps the velocity; no rotation. */
    int prescribed;
    double prescribed_velocity[2];
} iblbm_particles_args;

int iblbm_particles_step_f64(const iblbm_particles_args *a, void *stream);

/* ---- diagnostics reduced on the device -----------------------------------
 * Replaces the host reductions of iblbm/runtime/loop.py:97-126: Cd / Cl
 * (iblbm/diagnostics/core.py:53-113, compute_drag_lift_coefficient) and the
 * velocity-convergence error (core.py:116-135).  Deterministic FP64 sums in a
 * fixed order (equal to numpy's pairwise sums up to rounding); each call is
 * one launch that reads the output step's fields in place and leaves its
 * result in device memory, so calls can be queued (and graph-captured)
 * without a host synchronisation.  `partials` holds iblbm_diag_partials(n)
 * doubles and `ticket` one unsigned zero before the first call (each call
 * leaves it zero); calls sharing them must be ordered (one stream). */
typedef struct {
    const void *ro;          /* n_nodes densities of the output step (FP32 when f32, else FP64) */
    int n_nodes;
    int f32;
    int method;              /* IBLBM_IBM_*: DF/MDF sum band_fib, DFC sums dfc_force, NONE no force */
    const void *band_fib;    /* band x 2 (FP32 when f32) */
    const int *band_count;   /* device: band nodes */
    const double *dfc_force; /* lb_total x 2 */
    int lb_total;
    double u_ref, lattice_r; /* Cd = |sum Fx| / (mean(rho) u_ref^2 R), Cl = sum Fy / (...) */
    double *partials;
    unsigned *ticket;
    double *ring;            /* ring_len x 5: Cd, Cl, mean rho, sum Fx, sum Fy */
    int ring_len;
    int *ring_pos;           /* device counter: the call writes entry (*ring_pos % ring_len), then increments */
} iblbm_force_coeff_args;

int iblbm_force_coeffs(const iblbm_force_coeff_args *a, void *stream);

typedef struct {
    const void *U;           /* n_nodes x 2 velocities of the output step (FP32 when f32) */
    double *U_prev;          /* n_nodes x 2 FP64: the last check's field; replaced by U */
    int n_nodes;
    int f32;
    double *partials;
    unsigned *ticket;
    double *out;             /* 3 doubles: sum (U - U_prev)^2, sum U_prev^2, the error sqrt(ratio) (1 if 0) */
} iblbm_velocity_change_args;

int iblbm_velocity_change(const iblbm_velocity_change_args *a, void *stream);
int iblbm_diag_partials(int n_nodes);

/* ---- reference-shaped kernels (AoS, one op per call, FP64) ------------- */
/* Replaces feq_gpu (iblbm/gpu_kernels.py:906-927) <- lbm/equilibrium.py:45-50 */
int iblbm_feq(const double *ro, const double *U, int N, int incompressible, double *feq, void *stream);
/* Replaces macroscopic_gpu (gpu_kernels.py:878-903) <- lbm/macroscopic.py:52-59 */
int iblbm_macroscopic(const double *fstar, int N, int incompressible, double *ro, double *U, void *stream);
/* Replaces collision_gpu (gpu_kernels.py:760-784) <- lbm/collision/bgk.py:55-57 */
int iblbm_collision_bgk(const double *fstar, const double *feq, const double *U, const double *fib, int N,
                        double tau, double dt, double *f, void *stream);
/* Replaces collision_trt_gpu (gpu_kernels.py:787-812) <- lbm/collision/trt.py:88-90 */
int iblbm_collision_trt(const double *fstar, const double *feq, const double *U, const double *fib, int N,
                        double tau, double tau_minus, double dt, double *f, void *stream);
/* Replaces collision_cm_mrt_gpu (gpu_kernels.py:815-843) <- lbm/collision/cm_mrt.py:198-200 */
int iblbm_collision_cm_mrt(const double *fstar, const double *U, const double *fib, int N,
                           const double *S_diag_host, double dt, double *f, void *stream);
/* Replaces streaming_gpu (gpu_kernels.py:846-875) <- lbm/streaming.py:80-84 */
int iblbm_streaming(const double *fstar_old, const double *f, int nx, int ny, double *fstar_new, void *stream);
/* Replaces velocity_correction_gpu (gpu_kernels.py:930-948) <- ibm/dispatch.py:18-33 */
int iblbm_velocity_correction(double *U, const double *fib, const double *ro, int N, double dt,
                              int incompressible, void *stream);

/* ---- layout conversion between the reference AoS and the engine SoA ----- */
int iblbm_aos_to_soa(const double *aos, iblbm_geom g, double *soa, void *stream);
int iblbm_soa_to_aos(const double *soa, iblbm_geom g, double *aos, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* IBLBM_B200_H */
