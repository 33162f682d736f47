/*
 * oracle.h -- CPU FP64 restatement of the GENESIS per-tick particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it to
 * compute the reference answer on the host.  Nothing in the product path
 * (genesis_b200/, include/) links, loads or calls it.
 *
 * Parity status: pinned by the known-answer tests of the reference's own
 * test modules (tests/golden/reference_known_answers.json, transcribed from
 * src/physics/forces.rs, src/physics/grid.rs, src/analysis/mod.rs and
 * src/analysis/pairs.rs) and by property tests that re-run the reference's
 * seeded invariant tests with this project's generator.  The reference
 * itself (pure Rust, unvendored crates) cannot be compiled here, so no
 * output of the reference binary pins it directly.
 *
 * Every function restates a reference function operation by operation so
 * that FP64 results round identically (compile with -ffp-contract=off, as
 * Rust never contracts a*b+c into an FMA).  Each definition cites the
 * reference file:line it follows.
 */
#ifndef GENESIS_ORACLE_H
#define GENESIS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NELEM 10

/* Force-pass / integrator parameters: the subset of the reference Config
 * that src/systems/{forces,integrate,boundary,thermostat}.rs read. */
typedef struct {
    double box[3];                 /* universe.size */
    double dt;                     /* universe.dt */
    double thermal_constant;       /* physics.thermal_constant (k) */
    double sigma[ORC_NELEM];       /* affinity table after overrides */
    double epsilon_k[ORC_NELEM];
    double charge[ORC_NELEM];
    double lj_cutoff_factor;       /* LJ_CUTOFF_FACTOR = 2.5 */
    double coulomb_constant;
    double coulomb_cutoff;
    double gravity_constant;
    double gravity_cutoff;
    double bond_k_bind;
    double thermostat_temperature;
    double thermostat_tau;
    int32_t enable_electrostatics;
    int32_t enable_gravity;
    int32_t enable_bond_interaction;
    int32_t enable_thermostat;
    int32_t enable_boundaries;
    int32_t enable_collisions;
    int32_t reserved[2];
    double particle_radius;
} orc_params;

/* One CollisionSystem pass (src/systems/collisions.rs:40-88) on vel; returns
 * the collisions counted. */
size_t orc_collisions(const orc_params* p, size_t n, const double* pos, double* vel, const double* mass);

/* export::write_frame's text (src/export/mod.rs:152-172) for n atoms (pos
 * n x 3, elem 0..9); returns its size and copies it to out when cap allows. */
size_t orc_xyz_frame(size_t n, uint64_t tick, const double* pos, const uint8_t* elem, char* out, size_t cap);

/* ---- pair laws: src/physics/forces.rs ---- */
void orc_lj_table(const orc_params* p, double* pair_sigma /*100*/,
                  double* pair_eps /*100*/, double* rc, double* r_on);
void orc_lj_raw(double sigma, double eps, double r, double* m, double* v);
void orc_smooth_cutoff(double r, double r_on, double rc, double* sw, double* dsw);
void orc_switched(double f, double v, double sw, double dsw, double* fo, double* vo);
void orc_force_switched_scalar(double sigma, double eps, double r, double r_on,
                               double rc, double* m, double* v);
void orc_coulomb_raw(double k_e, double qa, double qb, double r, double* f, double* v);
void orc_gravity_raw(double g, double ma, double mb, double r, double* f, double* v);
void orc_bond_harmonic_raw(double k, double r_eq, double r, double* f, double* v);
double orc_well_curvature(double eps, double sigma);
double orc_vib_period(double eps, double sigma, double mu);
double orc_equilibrium_distance(double sigma);

/* ---- uniform grid: src/physics/grid.rs ---- */
void orc_grid_dims(const double box[3], double min_cell, uint32_t dims[3]);
void orc_cell_of(size_t n, const double* pos, const double box[3], double min_cell,
                 uint32_t* cell);
/* Pairs reported by SpatialGrid::build + neighbors, in the reference's
 * emission order.  Writes up to cap pairs (a,b) and their unit normals;
 * returns the total number of pairs (may exceed cap). */
size_t orc_neighbors(size_t n, const double* pos, const double box[3],
                     double min_cell, double cutoff, uint32_t* pairs,
                     double* normals, size_t cap);
void orc_min_image(const double d[3], const double box[3], double out[3]);

/* ---- force pass: src/systems/forces.rs:100-353 ---- */
/* pos: AoS xyz per slot; elem: element index 0..9 per slot; charge/mass per
 * slot; bonds: nbonds slot pairs (already reduced to one entry per bond).
 * nthreads <= 1 is the sequential fold; nthreads > 1 splits the pair list
 * into contiguous chunks (rayon-like) and merges in split order.
 * Returns the number of pairs in the list. */
size_t orc_forces(const orc_params* p, size_t n, const double* pos,
                  const uint8_t* elem, const double* charge, const double* mass,
                  size_t nbonds, const uint32_t* bonds, double* acc,
                  double* potential, double* bond_potential, int nthreads);

/* ---- integrator / boundary / thermostat / stats ---- */
void orc_half_kick(size_t n, double* vel, const double* acc, double dt);
void orc_drift(size_t n, double* pos, const double* vel, double dt);
void orc_wrap(size_t n, double* pos, const double box[3]);
/* Returns 1 when the scale was applied; kinetic and lambda are outputs. */
int orc_thermostat(size_t n, double* vel, const double* mass, double k,
                   double target, double tau, double* kinetic, double* lambda);
void orc_stats(size_t n, const double* vel, const double* mass, double* kinetic,
               double* speed_sum);

/* One or more ticks of the force schedule (src/universe/mod.rs:355-369):
 * kick, drift, [wrap], forces, kick, [thermostat].  out_stats, if non-null,
 * receives per tick {K, V, Vbond, lambda, npairs}. */
int orc_ticks(const orc_params* p, size_t n, double* pos, double* vel, double* acc,
              const uint8_t* elem, const double* charge, const double* mass,
              size_t nbonds, const uint32_t* bonds, int nticks, int nthreads,
              double* out_stats);

/* ---- adjoint reference (oracle_dual.cpp) ----
 * The NVE tick templated on the scalar type.  Returns per tick V_t and the
 * time-averaged Gaussian-kernel g_k; when dpotential / dgr are non-null the
 * run uses dual numbers and also returns dV_t/dtheta [nsteps][20] and
 * dg_k/dtheta [gr_bins][20], theta = (sigma[0..9], epsilon_k[0..9]).
 * Returns -1 with bonds or thermostat on, -2 when gr_rmax + gr_support *
 * gr_width exceeds the force cutoff, -3 on bad arguments. */
int orc_adjoint_forward(const orc_params* p, size_t n, const double* pos, const double* vel,
                        const double* acc, const uint8_t* elem, const double* charge,
                        const double* mass, int nsteps, int gr_bins, int gr_every, double gr_rmax,
                        double gr_width, double gr_support, int nthreads, double* potential,
                        double* gr, double* dpotential, double* dgr);
/* The template's T = double trajectory (in place), for the bit-for-bit
 * comparison with orc_ticks. */
int orc_adjoint_trajectory(const orc_params* p, size_t n, double* pos, double* vel, double* acc,
                           const uint8_t* elem, const double* charge, const double* mass,
                           int nsteps, int nthreads, double* potential);

/* ---- bond observation (oracle_bonds.cpp) ----
 * A stateful restatement of PairTracker + BondObservationSystem::run
 * (src/analysis/pairs.rs:38-94, src/systems/bonds.rs:73-185), pairs keyed by
 * slot.  orc_bond_observe feeds one tick's bound pairs (slot pairs, any
 * orientation) and returns stats[8] = {bonded_pairs, bonded_entities,
 * mean_coordination, bonds_formed, lifetime_sum_ticks, open episodes,
 * completed episodes, completed ticks}, the 10x10 species matrix and the
 * persistent pairs (a < b, ascending) -- the Bonds adjacency. */
typedef struct orc_tracker orc_tracker;
orc_tracker* orc_tracker_new(int debounce);
void orc_tracker_free(orc_tracker* t);
void orc_tracker_close_all(orc_tracker* t);
uint64_t orc_bond_threshold(const orc_params* p, double min_periods, int ea, int eb);
int orc_bond_observe(orc_tracker* t, const orc_params* p, double min_periods, size_t nbound,
                     const uint32_t* bound, const uint8_t* elem_of_slot, uint64_t tick,
                     double* stats, uint64_t* matrix, uint32_t* persistent, size_t cap,
                     size_t* npersistent);

/* ---- lenses: src/analysis/mod.rs, src/analysis/pairs.rs ---- */
int orc_radial_distribution(size_t n, const double* pos, const double box[3],
                            double r_max, size_t nbins, uint64_t* counts,
                            double* bins, double* r_max_out, double* dr_out);
int orc_radial_distribution_between(size_t n, const double* pos, const uint8_t* elem,
                                    uint8_t ta, uint8_t tb, const double box[3],
                                    double r_max, size_t nbins, uint64_t* counts,
                                    double* bins, double* r_max_out, double* dr_out);
/* FoF: labels[i] = smallest slot index in i's component.  stats =
 * {monomers, aggregates, largest, bound_pairs}; mean_size separately. */
int orc_clusters(size_t n, const double* pos, const uint8_t* elem,
                 const double box[3], double bond_factor, const double sigma[10],
                 uint32_t* labels, uint64_t stats[4], double* mean_size);
/* Bound pairs (entity index pairs, a<b) in emission order; returns total. */
size_t orc_bound_pairs(size_t n, const double* pos, const uint8_t* elem,
                       const uint32_t* entity, const double box[3], double k_bind,
                       const double sigma[10], uint32_t* out, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
