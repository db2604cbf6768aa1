/*
 * lp_oracle.h - C ABI of the FP64 CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a restatement, in C++, of the reference's
 * CPU MLS-MPM step (nredd/litter-physics core/src/mpm/{rng,grid,particles,constitutive,
 * solver,rigid,fixtures}.rs).  It exists to check the CUDA product path and to time the
 * reference algorithm on the host cores.  Only tests/, __graft_entry__.smoke() and
 * bench.py (cpu_baseline leg and --impl reference arm) may load it.  The product library
 * never links or calls it.
 *
 * It shares the POD structs of include/lp_mpm.h so both sides speak the same layouts.
 */
#ifndef LP_ORACLE_H
#define LP_ORACLE_H

#include "../include/lp_mpm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_sim ora_sim;

int32_t ora_sim_create(const lp_fixture_spec* spec, ora_sim** out, char* err, int32_t errlen);
void ora_sim_destroy(ora_sim* s);
/* Advance toward target; stops early (status LP_BUDGET) after max_accepted accepted steps
 * when max_accepted > 0.  *reached = 1 when target reached. */
int32_t ora_sim_advance(ora_sim* s, double target, int64_t max_accepted, int32_t* reached, char* err,
                        int32_t errlen);
int32_t ora_sim_try_step(ora_sim* s, double dt, int32_t* accepted, char* reason, int32_t len);
double ora_sim_stability_limit(ora_sim* s);
/* Energy audit of one trial step on a copy (audit.rs:284-353); the simulation is unchanged. */
int32_t ora_sim_audit_step(ora_sim* s, double dt, lp_energy_audit* out, char* err, int32_t errlen);
void ora_sim_counters(ora_sim* s, lp_counters* out);
/* counters as lp_sim_set_counters takes them (time, step counts, dt_scale in (0, 1]) */
int32_t ora_sim_set_counters(ora_sim* s, const lp_counters* in);
void ora_sim_ledger(ora_sim* s, lp_ledger* out);
void ora_sim_set_ledger(ora_sim* s, const lp_ledger* in);
uint64_t ora_sim_particle_count(ora_sim* s);
void ora_sim_export_particles(ora_sim* s, lp_particles* out);
int32_t ora_sim_import_particles(ora_sim* s, const lp_particles* in);
int32_t ora_sim_get_pellet(ora_sim* s, lp_pellet* out);
void ora_sim_set_pellet(ora_sim* s, const lp_pellet* in);
/* pellet bed (extension): committed pellets in index order (returns the count); replace poses */
int32_t ora_sim_get_pellets(ora_sim* s, lp_pellet* out, int32_t cap);
int32_t ora_sim_set_pellets(ora_sim* s, const lp_pellet* in, int32_t count);
int32_t ora_sim_observables(ora_sim* s, char* names, double* values, int32_t capacity);
void ora_sim_energies(ora_sim* s, double out[9]);
/* Threads used by the node/particle-parallel loops (0 = OpenMP default). */
void ora_set_threads(int32_t threads);

/* One P2G + wall traction on the current state (no grid update); returns active node
 * count and copies mass/momentum of the dense grid into the caller arrays when non-NULL. */
int64_t ora_sim_probe_p2g(ora_sim* s, double dt, double* mass, double* momentum, double* traction_energy,
                          double traction_impulse[3]);

/* Grid probe of one step's scatter (solver.rs:632-661 then 725-819) on a copy: node mass,
 * node momentum before the wall reactions, and the signed reaction impulse of each node
 * (3 per node), in dense padded node order; returns the active node count. */
int64_t ora_sim_probe_grid(ora_sim* s, double dt, double* mass, double* momentum, double* reaction);

/* constitutive.rs functions on scalars */
int32_t ora_hb_return(double trial, double yield, double consistency, double flow_index, double mu,
                      double dt, double tol_rel, double out[3]);
int32_t ora_update_paste(const double f_trial[9], const lp_material* m, double yield_override, double dt,
                         double tol_rel, double f_new[9], double tau[9], double out[3]);
int32_t ora_update_liquid(double volume_ratio, const double grad[9], const lp_material* m, double dt,
                          double* j_new, double tau[9], double* pressure);
int32_t ora_eigen3(const double m[9], double values[3], double vectors[9]);
int32_t ora_stencil(double spacing, const int32_t nodes[3], const double x[3], int32_t base[3],
                    double weights[9], double offsets[9]);
double ora_splitmix_next_unit(uint64_t* state);
uint64_t ora_splitmix_next_u64(uint64_t* state);
lp_material ora_material_paste(double density, double e, double nu, double ys, double k, double n);
lp_material ora_material_paste_shear(double density, double e, double nu, double tys, double ks, double n);
lp_material ora_material_liquid(double density, double e, double nu, double visc);
/* Grid update of one node holding `mass` and `momentum` at padded coords (probe of
 * solver.rs:822-892): out = velocity[3], wall_impulse[3], projection energy, friction. */
int32_t ora_grid_update_node(const lp_fixture_spec* spec, const int32_t coords[3], double mass,
                             const double momentum[3], const double traction[3], double dt, double out[8]);

#ifdef __cplusplus
}
#endif
#endif
