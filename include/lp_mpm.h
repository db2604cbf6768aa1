/*
 * lp_mpm.h - C ABI of the B200-native MLS-MPM substep (litter-physics research core).
 *
 * This is the drop-in boundary under the reference core's step/fixture API.  A Rust host
 * binds it with `extern "C"` declarations, Python binds it with ctypes (see
 * litter_physics_b200/_lib.py).  Every entry point takes plain pointers and sizes; all
 * device memory is owned by the library behind the opaque handles.  Calls on one handle
 * are not thread-safe (the reference takes `&mut self`).  Errors are returned as
 * `lp_status`; `lp_last_error()` gives a thread-local message for the last failure.
 *
 * Reference interface each entry point replaces (paths inside nredd/litter-physics):
 *   lp_material_*                 core/src/mpm/constitutive.rs:146-243  Material::{paste,
 *                                 paste_from_shear_rheology, liquid, wave_speed, diffusivity}
 *   lp_sim_create                 core/src/mpm/fixtures.rs:238-268      FixtureSpec::build
 *   lp_sim_advance                core/src/mpm/solver.rs:402-472        advance_to/advance_while
 *   lp_sim_try_step               core/src/mpm/solver.rs:535-611        try_step (one trial)
 *   lp_sim_stability_limit        core/src/mpm/solver.rs:477-498        stability_limit
 *   lp_sim_get_ledger             core/src/mpm/solver.rs:65-124         Ledger (pub field)
 *   lp_sim_get_counters           core/src/mpm/solver.rs:332-352        time/step_count/... fields
 *   lp_sim_export/import_particles core/src/mpm/particles.rs:11-32     ParticleSet (pub field),
 *                                 used by checkpoints in core/src/research.rs:308-368
 *   lp_sim_get/set_pellet         core/src/mpm/rigid.rs:30-49           Pellet (pub field)
 *   lp_sim_observables            core/src/mpm/fixtures.rs:369-461      FixtureSpec::observables
 *   lp_sim_energies               core/src/mpm/solver.rs:1000-1099      residual/energy accessors
 *   lp_hb_return_batch            core/src/mpm/constitutive.rs:280-362  solve_herschel_bulkley_return
 *   lp_update_paste_batch         core/src/mpm/constitutive.rs:456-531  update_paste
 *   lp_update_liquid_batch        core/src/mpm/constitutive.rs:557-589  update_liquid
 *   lp_batch_*                    no single reference call: python/litter_physics/sweep.py:206
 *                                 runs the same jobs one after another; the batch runs them
 *                                 as one ensemble on the device.
 *   lp_mlp_*                      no reference counterpart (learned Newton warm start).
 */
#ifndef LP_MPM_H
#define LP_MPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LP_ABI_VERSION 1

/* Status codes (0 ok).  LP_MIN_STEP mirrors SolverError::MinimumStepReached
 * (core/src/mpm/solver.rs:128-142); LP_BUDGET is the resumable budget stop of
 * advance_while returning Ok(false) (solver.rs:421-423). */
typedef enum lp_status {
  LP_OK = 0,
  LP_INVALID = 1,
  LP_MIN_STEP = 2,
  LP_BUDGET = 3,
  LP_DEVICE = 4,
  LP_UNSUPPORTED = 5
} lp_status;

typedef enum lp_fixture { LP_SLUMP = 0, LP_HYDROSTATIC = 1, LP_DAM_BREAK = 2, LP_COUPLED_PATCH = 3 } lp_fixture;
typedef enum lp_material_kind { LP_PASTE = 0, LP_LIQUID = 1 } lp_material_kind;

/* Mirror of Material (constitutive.rs:111-131). */
typedef struct lp_material {
  int32_t kind;          /* lp_material_kind */
  int32_t _pad;
  double density;        /* kg/m^3 */
  double shear_modulus;  /* mu, Pa */
  double lame_lambda;    /* lambda, Pa */
  double bulk_modulus;   /* Pa */
  double yield_stress;   /* von Mises sigma_y, Pa */
  double consistency;    /* von Mises K (paste) or dynamic viscosity (liquid) */
  double flow_index;     /* n */
  double tait_gamma;     /* extension: liquid EOS exponent; 1 = reference linear EOS p = K (1/J - 1) */
} lp_material;

/* Mirror of FixtureSpec + SolverConfig + ContactParams (fixtures.rs:94-115, solver.rs:48-62,
 * rigid.rs:68-75), plus labelled extensions that default to reference behaviour. */
typedef struct lp_fixture_spec {
  int32_t fixture;            /* lp_fixture */
  int32_t has_pellet;         /* 1: pellet geometry given (coupled_patch only) */
  lp_material material;
  double grid_spacing;        /* m */
  double domain[3];           /* m */
  double initial_size[3];     /* m */
  double initial_velocity[3]; /* m/s */
  uint64_t seed;
  double pellet_radius, pellet_length, pellet_density;
  double gravity[3];
  double wall_friction;       /* one Coulomb mu for all six walls (reference) */
  double cfl, max_dt, min_dt;
  double contact_stiffness, contact_restitution, contact_friction;
  uint64_t max_particles, max_nodes;
  /* ---- extensions (zero-initialised spec == reference behaviour) ---- */
  int32_t face_mode_enabled;  /* 1: use face_friction/face_sticky below instead of wall_friction */
  int32_t face_sticky[6];     /* faces: 2*axis + (0 low, 1 high); sticky = tangential stops on contact */
  double face_friction[6];
  double newton_tolerance;    /* relative HB return tolerance; 0 -> reference 1e-12 */
  int32_t yield_random;       /* 1: per-particle sigma_y ~ U(yield_min, yield_max) (von Mises) */
  int32_t _pad2;
  double yield_min, yield_max;
  /* pellet bed (config 4): bed_count >= 2 pellets of the geometry above (has_pellet = 1, fixture
   * slump), centres and orientations drawn from bed_seed inside [bed_lo, bed_hi] without overlap,
   * Hertz-Mindlin sphere contact between pellets; bed_count < 2 keeps the reference */
  int32_t bed_count;
  int32_t _pad3;
  uint64_t bed_seed;
  double bed_lo[3], bed_hi[3];
  double hm_young, hm_poisson, hm_friction, hm_restitution;
  /* contact law between bed pellets: LP_BED_HERTZ_MINDLIN (hm_* above) or LP_BED_LINEAR, the
   * household DEM's linear spring-dashpot with a tangential spring and rolling resistance
   * (replaces World::contact_force, core/src/dem.rs:789-834): normal stiffness dem_stiffness
   * N/m, rolling friction dem_rolling, friction hm_friction, restitution hm_restitution */
  int32_t bed_law;
  int32_t _pad4;
  double dem_stiffness, dem_rolling;
} lp_fixture_spec;

enum { LP_BED_HERTZ_MINDLIN = 0, LP_BED_LINEAR = 1 };

/* Mirror of Ledger (solver.rs:65-124), FP64. */
typedef struct lp_ledger {
  double initial_mass;
  double outflow_mass;
  double initial_momentum[3];
  double initial_mechanical_energy;
  double gravity_impulse[3];
  double wall_impulse[3];
  double pellet_wall_impulse[3];
  double coupling_impulse[3];
  double coupling_angular_impulse[3];
  double wall_normal_projection_energy;
  double wall_friction_dissipation;
  double wall_normal_traction_energy;
  double pellet_wall_work;
  double coupling_grid_energy;
  double coupling_pellet_energy;
  double plastic_dissipation;
  double outflow_momentum[3];
} lp_ledger;

/* Simulation counters (solver.rs:332-352). */
typedef struct lp_counters {
  double time;
  uint64_t step_count, limited_steps, rejected_steps;
  double dt_scale, min_dt_used, max_dt_used; /* min_dt_used = +inf before the first step */
  uint64_t particle_count;
  uint64_t newton_iterations; /* total HB return iterations of accepted steps (diagnostic) */
  uint64_t yielded_particles; /* particles that went through the return in the last accepted step */
} lp_counters;

/* Host view of ParticleSet (particles.rs:11-32).  Matrices are row-major 3x3. */
typedef struct lp_particles {
  uint64_t count;
  uint32_t* id;
  double* position;       /* 3*count */
  double* velocity;       /* 3*count */
  double* affine;         /* 9*count */
  double* deformation;    /* 9*count */
  double* volume_ratio;   /* count */
  double* kirchhoff;      /* 9*count */
  double* plastic_strain; /* count */
  double* mass;           /* count */
  double* volume0;        /* count */
  double* yield_stress;   /* count, optional (NULL = material value) */
} lp_particles;

/* Mirror of Pellet (rigid.rs:30-49). orientation = (i, j, k, w). */
typedef struct lp_pellet {
  double radius, length, mass;
  double inertia_body[3];
  double position[3];
  double orientation[4];
  double velocity[3];
  double angular_momentum[3];
  int32_t sphere_count;
  int32_t _pad;
  double sphere_offsets[64];
} lp_pellet;

/* Energy audit of one trial step (audit.rs:254-271), all energies in J.  before / after:
 * EnergyState (translation, APIC affine norm h^2/8 sum m |C|^2, elastic, potential, pellet).
 * stages: grid_transport, grid_after_stress, grid_after_traction, grid_after_gravity,
 * grid_after_walls, grid_after_coupling, pellet_after_coupling, plastic_dissipation.
 * increments: ledger differences of plastic dissipation, wall friction, wall normal projection,
 * wall normal traction, coupling grid, coupling pellet, pellet wall work.
 * terms: p2g transfer loss, g2p transfer loss, stress/storage/plastic mismatch, uncoupled
 * gravity/potential mismatch (NaN when coupled), coupled grid-gravity plus potential change
 * (NaN when uncoupled), pellet integrator change, traction change, walls change, coupling
 * change, augmented energy change, telescoping sum, telescoping error. */
typedef struct lp_energy_audit {
  double time, dt;
  double before[5], after[5];
  double stages[8];
  double increments[7];
  double terms[12];
  int32_t coupled;
  int32_t _pad;
} lp_energy_audit;

typedef struct lp_sim lp_sim;
typedef struct lp_batch lp_batch;

/* Budget callback of advance_while (solver.rs:413-417); return nonzero to continue. */
typedef int (*lp_keep_going_fn)(void* ctx);

/* ---------------- library ---------------- */
int32_t lp_abi_version(void);
const char* lp_last_error(void);
/* Number of CUDA kernels this library launched since load (for launch accounting). */
uint64_t lp_kernel_launches(void);
/* sizeof of lp_material, lp_fixture_spec, lp_ledger, lp_counters, lp_particles, lp_pellet
 * (lets bindings check their struct mirrors without a GPU). */
void lp_abi_struct_sizes(uint64_t out[6]);

/* ---------------- materials (constitutive.rs:146-243) ---------------- */
lp_material lp_material_paste(double density, double young_modulus, double poisson_ratio,
                              double yield_stress, double consistency, double flow_index);
lp_material lp_material_paste_from_shear_rheology(double density, double young_modulus,
                                                  double poisson_ratio, double shear_yield_stress,
                                                  double shear_consistency, double flow_index);
lp_material lp_material_liquid(double density, double young_modulus, double poisson_ratio,
                               double viscosity);
double lp_material_wave_speed(const lp_material* m);
double lp_material_diffusivity(const lp_material* m);

/* ---------------- one simulation ---------------- */
lp_status lp_sim_create(const lp_fixture_spec* spec, lp_sim** out);
void lp_sim_destroy(lp_sim* sim);
/* cudaStream_t as void*; NULL restores the library's own stream. */
lp_status lp_sim_set_stream(lp_sim* sim, void* stream);
lp_status lp_sim_advance(lp_sim* sim, double target_time, lp_keep_going_fn keep_going, void* ctx,
                         int32_t* reached);
/* One trial step of exactly dt (no dt control); accepted = 1 if committed. */
lp_status lp_sim_try_step(lp_sim* sim, double dt, int32_t* accepted, char* reason, size_t reason_len);
/* Run `steps` fixed-size attempts of dt (capped by the stability limit like advance does)
 * asynchronously on the stream without host synchronisation (benchmark/graph path). */
lp_status lp_sim_run_substeps(lp_sim* sim, int32_t steps);
lp_status lp_sim_sync(lp_sim* sim);
lp_status lp_sim_stability_limit(lp_sim* sim, double* out);
/* Energy audit of one trial step of exactly dt (replaces Simulation::audit_step,
 * core/src/mpm/audit.rs:284-353).  dt must lie in [min_dt, min(dt_scale * stability limit,
 * max_dt)]; a refused or rejected trial returns LP_INVALID with the reason in lp_last_error().
 * The simulation's committed state is unchanged. */
lp_status lp_sim_audit_step(lp_sim* sim, double dt, lp_energy_audit* out);
lp_status lp_sim_get_ledger(lp_sim* sim, lp_ledger* out);
lp_status lp_sim_set_ledger(lp_sim* sim, const lp_ledger* in);
lp_status lp_sim_get_counters(lp_sim* sim, lp_counters* out);
lp_status lp_sim_set_counters(lp_sim* sim, const lp_counters* in);
lp_status lp_sim_particle_count(lp_sim* sim, uint64_t* out);
/* Export copies the device state into caller buffers sized for `count` particles (set
 * out->count to the buffer capacity on entry). */
lp_status lp_sim_export_particles(lp_sim* sim, lp_particles* out);
lp_status lp_sim_import_particles(lp_sim* sim, const lp_particles* in);
/* Extension, no reference counterpart: page-lock (cudaHostRegister) a caller's host buffer, or
 * release it.  Export and import move arrays that are page-locked from the first to the last
 * byte by DMA straight between them and the device, without the library's pinned staging copy;
 * arrays in pageable memory go through the staging copy as before.  A caller that keeps its
 * particle set resident in host memory pins it once and reuses it for every checkpoint. */
lp_status lp_host_pin(void* ptr, uint64_t bytes);
lp_status lp_host_unpin(void* ptr);
lp_status lp_sim_get_pellet(lp_sim* sim, lp_pellet* out, int32_t* has_pellet);
lp_status lp_sim_set_pellet(lp_sim* sim, const lp_pellet* in);
/* Pellet bed (extension, no reference counterpart): the committed state of every pellet, in
 * pellet index order; *count = number of pellets (0 without a bed), at most cap written. */
lp_status lp_sim_get_pellets(lp_sim* sim, lp_pellet* out, int32_t cap, int32_t* count);
/* Pellet bed: replace the pose, velocity and angular momentum of every pellet (geometry must
 * match); the sphere-contact histories restart empty. */
lp_status lp_sim_set_pellets(lp_sim* sim, const lp_pellet* in, int32_t count);
/* Observables as sorted name/value pairs (fixtures.rs:369-461).  names is a buffer of
 * `capacity` entries of 64 chars each; *count receives the number written. */
lp_status lp_sim_observables(lp_sim* sim, char* names, double* values, int32_t capacity,
                             int32_t* count);
/* kinetic, potential, elastic, mechanical energy; mass residual; momentum residual xyz;
 * energy residual (solver.rs:1000-1099). */
lp_status lp_sim_energies(lp_sim* sim, double out[9]);
/* Enable the learned Newton warm start (weights from lp_mlp_*); 0 disables. */
lp_status lp_sim_set_warm_start(lp_sim* sim, const float* weights, int32_t nweights, int32_t enable);
/* Logit table of the warm start.  Within one instance and one dt the network's six features
 * depend on la8 = log((trial - yield) / K) / 8 alone, so the solver evaluates the network
 * (the lp_mlp_forward_mma pass) once per instance and dt at the nodes
 * la8_j = LP_MLP_TAB_LO + j * LP_MLP_TAB_H, j < LP_MLP_TAB_N, which cover every finite FP32
 * la8, and interpolates linearly between them.  Copies the table of instance `instance`
 * (0 for a simulation) to out[LP_MLP_TAB_N]; *dt = the dt it was built for, or NaN (out
 * untouched) while none is built.  No counterpart in the reference. */
#define LP_MLP_TAB_N 2049
#define LP_MLP_TAB_LO (-10.75f)
#define LP_MLP_TAB_H (11.0f / 1024.0f)
lp_status lp_sim_warm_table(lp_sim* sim, float* out, int32_t capacity, double* dt);
/* Conservation probe: scatter the committed state to the grid with step dt (P2G only) and
 * return out[0] = grid mass, out[1..3] = grid momentum (exact fixed-point sums over nodes),
 * out[4] = particle mass, out[5..7] = particle momentum (FP64 sums); the grid is then cleared. */
lp_status lp_sim_grid_totals(lp_sim* sim, double dt, double out[8]);
/* Grid probe: P2G + wall traction of the committed state with step dt; copies node mass
 * (node_count), momentum (3*node_count, without reactions) and signed wall reactions
 * (3*node_count) to the caller (node order of the dense padded grid), then clears the grid. */
lp_status lp_sim_grid_dump(lp_sim* sim, double dt, double* mass, double* momentum, double* reaction,
                           int64_t node_count);
/* Time `steps` attempts kernel by kernel with CUDA events on the simulation's stream:
 * ms[k] = mean duration of kernel k, names = 32-char slots; *count = kernels per attempt. */
lp_status lp_sim_kernel_times(lp_sim* sim, int32_t steps, double* ms, char* names, int32_t capacity,
                              int32_t* count);
/* Measurement: run `steps` attempts (real steps, time advances) with G2P's clock-instrumented
 * instantiation and return in *share the fraction of G2P warp time spent in the FP64
 * Herschel-Bulkley return (per round, the longest lane's time in the return, over each warp's
 * time in its tiles).  It bounds what any Newton start, the learned warm start included, can
 * save in G2P.  No counterpart in the reference. */
lp_status lp_sim_g2p_return_share(lp_sim* sim, int32_t steps, double* share);
/* Capture run_substeps into a CUDA graph of `steps` attempts (0 disables graphs). */
lp_status lp_sim_use_graph(lp_sim* sim, int32_t steps);
/* Build that graph now (capture and instantiate, no launch) if the launch shape asks for one and
 * it is not built, so that the next run_substeps pays no capture.  Changing the launch shape,
 * the stream, the warm start or the Newton log drops the graph again.  No counterpart in the
 * reference. */
lp_status lp_sim_prepare(lp_sim* sim);

/* ---------------- batched ensembles (extension) ---------------- */
lp_status lp_batch_create(const lp_fixture_spec* specs, int32_t count, lp_batch** out);
void lp_batch_destroy(lp_batch* b);
lp_status lp_batch_set_stream(lp_batch* b, void* stream);
lp_status lp_batch_advance(lp_batch* b, double target_time, lp_keep_going_fn keep_going, void* ctx,
                           int32_t* all_reached);
lp_status lp_batch_run_substeps(lp_batch* b, int32_t steps);
lp_status lp_batch_sync(lp_batch* b);
lp_status lp_batch_get_counters(lp_batch* b, int32_t index, lp_counters* out);
lp_status lp_batch_get_ledger(lp_batch* b, int32_t index, lp_ledger* out);
lp_status lp_batch_export_particles(lp_batch* b, int32_t index, lp_particles* out);
lp_status lp_batch_total_particles(lp_batch* b, uint64_t* out);
lp_status lp_batch_set_warm_start(lp_batch* b, const float* weights, int32_t nweights, int32_t enable);
/* lp_sim_warm_table for member `instance` of a batch. */
lp_status lp_batch_warm_table(lp_batch* b, int32_t instance, float* out, int32_t capacity, double* dt);
lp_status lp_batch_use_graph(lp_batch* b, int32_t steps);
/* lp_sim_prepare for a whole batch. */
lp_status lp_batch_prepare(lp_batch* b);
/* lp_sim_kernel_times for a whole batch: each kernel's mean duration over `steps` attempts of
 * every instance at once.  No counterpart in the reference. */
lp_status lp_batch_kernel_times(lp_batch* b, int32_t steps, double* ms, char* names, int32_t capacity,
                                int32_t* count);
/* Per-instance views, so that each instance of a batched sweep reports what the reference's
 * sweep (python/litter_physics/sweep.py:206-262) gets from running that job alone. */
lp_status lp_batch_get_pellet(lp_batch* b, int32_t index, lp_pellet* out, int32_t* has_pellet);
lp_status lp_batch_observables(lp_batch* b, int32_t index, char* names, double* values, int32_t capacity,
                               int32_t* count);
lp_status lp_batch_energies(lp_batch* b, int32_t index, double out[9]);
/* *state: 0 running, 1 reached its target, 2 aborted below the minimum step, 3 leaked particles
 * beyond the padded grid; a stopped instance's reason goes to `message`.  Stopped instances
 * stay stopped while the others advance. */
lp_status lp_batch_instance_state(lp_batch* b, int32_t index, int32_t* state, char* message, size_t message_len);
/* Launch shape of the persistent tile kernels (bin sort, P2G, G2P) and of the attempt loop.  No
 * counterpart in the reference (its loops run on rayon's pool).  Every shape gives the same
 * results; only the speed differs.
 *   g2p_variant    G2P CTAs of 0: 256 threads (2 per SM), 1-3: 128 threads with registers sized
 *                  for 4, 5 or 6 CTAs per SM (more resident warps against some spilled registers)
 *   g2p_per_sm     persistent G2P CTAs per SM (0, or more than fit: as many as fit)
 *   p2g_variant    P2G chunks of 0: 1024 particles, 1: 512 particles, 2: 512 particles whose state
 *                  is copied into shared memory (cp.async) one chunk ahead, across tiles
 *   p2g_per_sm     persistent P2G CTAs per SM (0, or more than fit: as many as fit)
 *   dynamic_tiles  1: CTAs take occupied tiles from an atomic cursor, 0: round robin
 *   graph_attempts attempts captured per CUDA graph replay of run_substeps (0 or 1: no graph)
 * The getter reports the CTAs per SM the launches use. */
typedef struct lp_launch_shape {
  int32_t g2p_variant, g2p_per_sm, p2g_variant, p2g_per_sm, dynamic_tiles, graph_attempts;
} lp_launch_shape;
lp_status lp_sim_set_launch_shape(lp_sim* sim, const lp_launch_shape* shape);
lp_status lp_sim_get_launch_shape(lp_sim* sim, lp_launch_shape* out);
lp_status lp_batch_set_launch_shape(lp_batch* b, const lp_launch_shape* shape);
lp_status lp_batch_get_launch_shape(lp_batch* b, lp_launch_shape* out);
/* Autotuner: a coordinate search over the launch shape on the live ensemble (tile scheduling,
 * G2P block shape and CTAs per SM, P2G chunk and CTAs per SM, attempts per graph), each candidate
 * timed over trial_steps real attempts (time advances); keeps the fastest shape and writes one
 * line per candidate and the choice to report. */
lp_status lp_batch_autotune(lp_batch* b, int32_t trial_steps, char* report, size_t report_len);
lp_status lp_sim_autotune(lp_sim* sim, int32_t trial_steps, char* report, size_t report_len);

/* ---------------- constitutive kernels on host arrays (unit parity) ---------------- */
/* out[3*i] = equivalent stress, out[3*i+1] = plastic increment, out[3*i+2] = iterations;
 * status[i] = 0 ok, 1 not converged, 2 non-finite.  tol_rel 0 -> 1e-12. */
lp_status lp_hb_return_batch(int64_t n, const double* trial, const double* yield, const double* consistency,
                             const double* flow_index, const double* shear_modulus, const double* dt,
                             double tol_rel, const float* mlp_weights, int32_t nweights, double* out,
                             int32_t* status);
/* F_trial row-major 9 per item (FP64 in, FP32 device arithmetic); outputs F_new, tau (9 each),
 * plastic increment, dissipation density, equivalent stress; status 0 ok, >0 failure code. */
lp_status lp_update_paste_batch(int64_t n, const double* f_trial, const lp_material* m, double dt,
                                double* f_new, double* tau, double* dep, double* diss, double* eq,
                                int32_t* status);
lp_status lp_update_liquid_batch(int64_t n, const double* volume_ratio, const double* velocity_gradient,
                                 const lp_material* m, double dt, double* j_new, double* tau,
                                 double* pressure, int32_t* status);

/* ---------------- learned warm start (extension, no reference counterpart) ---------------- */
/* MLP 6 -> 64 -> 64 -> 1 (SiLU), FP32 weights; forward/backward/Adam on the device. */
int32_t lp_mlp_weight_count(void);
lp_status lp_mlp_init(float* weights, int32_t nweights, uint64_t seed);
/* Features x[6*n] (see lp_hb_features), targets y[n]; runs `epochs` passes of minibatch Adam. */
lp_status lp_mlp_train(float* weights, int32_t nweights, const float* x, const float* y, int64_t n,
                       int32_t epochs, int32_t batch, float lr, float* final_loss);
/* FP32 forward pass (the training kernels' arithmetic). */
lp_status lp_mlp_forward(const float* weights, int32_t nweights, const float* x, int64_t n, float* y);
/* Forward pass the solver uses for the warm start: one warp per 32 rows on the tensor cores
 * (mma.sync m16n8k16, BF16 weights and activations, inputs as BF16 hi + lo pairs, FP32
 * accumulation, hardware tanh in SiLU). */
lp_status lp_mlp_forward_mma(const float* weights, int32_t nweights, const float* x, int64_t n, float* y);
/* Loss and gradient of mean squared error over n samples (FP32), for gradient checks. */
lp_status lp_mlp_loss_grad(const float* weights, int32_t nweights, const float* x, const float* y,
                           int64_t n, float* loss, float* grad);
/* Loss and gradient of the warm-start network without allocating any device memory.
 * No counterpart in the reference.  Meant for callers that cannot call cudaMalloc, such as a
 * host framework that owns all device memory through its own pool, or code running while
 * allocation is forbidden.  Inputs and outputs are caller-owned DEVICE pointers:
 * weights[lp_mlp_weight_count()], x[6*n], y[n] in; loss[1], grad[lp_mlp_weight_count()] out.
 * Work space is a fixed static device array of the library sized for at most
 * LP_MLP_NOALLOC_MAX_SAMPLES samples (about 4.5 MB per GPU that loads the library, held until
 * exit); larger n returns LP_INVALID.  With CUDA's lazy module loading the driver reserves
 * that array when the library's device code is first used on a device, by this call or by any
 * earlier library call: a caller whose memory pool takes all free device memory makes one
 * library call first.  The first call on each device looks up that array's device address,
 * so make that first call before any stream capture; the address stays valid until the
 * device's primary context is reset (cudaDeviceReset), after which the library must be
 * reloaded.  All calls share the array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.  stream is a cudaStream_t
 * (NULL = default stream); the call returns after queueing the work. */
#define LP_MLP_NOALLOC_MAX_SAMPLES 4096
lp_status lp_mlp_loss_grad_noalloc(const float* weights, const float* x, const float* y, int64_t n, float* loss,
                                   float* grad, void* stream);
/* Feature map of one return problem: trial stress, yield, consistency, flow index, mu, dt. */
void lp_hb_features(double trial, double yield, double consistency, double flow_index, double mu,
                    double dt, float out[6]);
/* Collect (features, target) pairs logged by the plain Newton during lp_sim runs. */
lp_status lp_sim_enable_newton_log(lp_sim* sim, int64_t capacity);
lp_status lp_sim_read_newton_log(lp_sim* sim, float* x, float* y, int64_t capacity, int64_t* count);

#ifdef __cplusplus
}
#endif
#endif /* LP_MPM_H */
