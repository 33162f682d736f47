/*
 * genesis_gpu.h -- C ABI of the B200 (sm_100a) per-tick particle hot path.
 *
 * One gx_handle is one universe held resident on one GPU (or, for the
 * gx_batch_* calls, many small universes advanced together).  The caller
 * owns every host array; the library owns all device memory.  A handle is
 * not re-entrant: one host thread drives it at a time (the reference's
 * Scheduler::run calls systems sequentially on one thread,
 * src/scheduler/mod.rs:83-89).  Every call returns a gx_status; on error
 * gx_last_error() gives the text.
 *
 * Slot order.  Per-atom host arrays are in the order the reference's
 * World::for_each3::<Position, Mass, AtomType> visits entities
 * (src/ecs/world.rs:345-383) -- the "slot" order of ForceSystem
 * (src/systems/forces.rs:179-203).  `entity` carries EntityId::index per
 * slot (src/ecs/entity.rs:28-30).  Internally atoms are kept sorted by cell;
 * the library converts on the way in and out.
 *
 * Each entry point below names the reference interface it replaces.
 */
#ifndef GENESIS_GPU_H
#define GENESIS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GX_NELEM 10 /* AtomType::COUNT, src/components/atom_type.rs:34 */

typedef enum {
    GX_OK = 0,
    GX_ERR_ARG = -1,          /* invalid argument (null pointer, bad size) */
    GX_ERR_OOM = -2,          /* device allocation failed */
    GX_ERR_CUDA = -3,         /* a CUDA runtime call failed */
    GX_ERR_CAPACITY = -4,     /* an output buffer or a per-cell capacity was too small */
    GX_ERR_SATURATION = -5,   /* a fixed-point force/energy left the int64 range */
    GX_ERR_NONFINITE = -6,    /* non-finite position or velocity seen on device */
    GX_ERR_TIMEOUT = -7,      /* a bounded device wait gave up */
    GX_ERR_UNSUPPORTED = -8,  /* configuration not supported by this path */
    GX_ERR_STATE = -9         /* call out of order (e.g. no state uploaded) */
} gx_status;

typedef enum {
    GX_FP64 = 0,  /* plain path: FP64 throughout, per-pair arithmetic bit-exact to the reference */
    GX_MIXED = 1  /* FP32 pair arithmetic, 64-bit fixed-point force/energy accumulation */
} gx_precision;

/* Parameters: the Config fields the force, integrator, boundary and
 * thermostat systems read (src/config/mod.rs:15-229), with the affinity
 * table already resolved (ElementTable::apply_overrides,
 * src/physics/forces.rs:90-109).  Element order: H He C N O Na Si P S Fe
 * (element_index, src/physics/forces.rs:176-189). */
typedef struct {
    double box[3];                 /* universe.size */
    double dt;                     /* universe.dt */
    double thermal_constant;       /* physics.thermal_constant */
    double sigma[GX_NELEM];        /* LjElement::sigma */
    double epsilon_k[GX_NELEM];    /* LjElement::epsilon_k (kelvin) */
    double charge[GX_NELEM];       /* LjElement::charge */
    double lj_cutoff_factor;       /* LJ_CUTOFF_FACTOR = 2.5 */
    double coulomb_constant;       /* physics.coulomb_constant */
    double coulomb_cutoff;         /* physics.coulomb_cutoff (x max sigma) */
    double gravity_constant;       /* physics.gravity_constant */
    double gravity_cutoff;         /* physics.gravity_cutoff (x max sigma) */
    double bond_k_bind;            /* stats.bond_k_bind */
    double thermostat_temperature; /* physics.thermostat_temperature */
    double thermostat_tau;         /* physics.thermostat_tau (ticks) */
    int32_t enable_electrostatics; /* systems.enable_electrostatics */
    int32_t enable_gravity;        /* systems.enable_gravity */
    int32_t enable_bond_interaction; /* systems.enable_bond_interaction */
    int32_t enable_thermostat;     /* systems.enable_thermostat */
    int32_t enable_boundaries;     /* systems.enable_boundaries */
    int32_t precision;             /* gx_precision */
    int32_t device;                /* CUDA device ordinal */
    int32_t enable_collisions;     /* systems.enable_collisions */
    int32_t reserved[2];           /* must be zero */
    double particle_radius;        /* physics.particle_radius (collision contact at 2 r) */
} gx_params;

/* Per-tick observables, what StatsSystem reads after the force schedule
 * (src/systems/aggregate.rs:86-143) plus the force-pass counters. */
typedef struct {
    double kinetic;         /* sum 0.5*m*|v|^2 after the thermostat */
    double speed_sum;       /* sum |v| */
    double potential;       /* PotentialEnergy (LJ + Coulomb + gravity) */
    double bond_energy;     /* BondEnergy */
    double lambda;          /* Berendsen scale applied this tick (1 when off) */
    uint64_t pairs;         /* pair-list entries within the cutoff this tick */
} gx_tick_stats;

typedef struct gx_handle gx_handle;

/* ---- lifecycle ------------------------------------------------------- */

/* ForceSystem::new (src/systems/forces.rs:100-142) + ThermostatSystem::new
 * (src/systems/thermostat.rs:26-32): builds the LJ table
 * (LjTable::new, src/physics/forces.rs:223-237), the cutoffs and the grid
 * geometry, and creates the CUDA stream the handle uses. */
int gx_create(const gx_params* params, gx_handle** out);
void gx_destroy(gx_handle* h);
const char* gx_last_error(const gx_handle* h);
const char* gx_status_string(int status);
int gx_set_precision(gx_handle* h, int precision);
/* Tuning knob of the mixed pair pass: 0 = automatic (6 where it applies,
 * else 4), 1 = one thread per atom over the canonical half shell,
 * 2 = warp-tiled cell pairs with ballot compaction, 3 = thread per atom with
 * staged rows, 4 = thread per atom with per-thread candidate lists (all
 * four re-sort the atoms by the force grid every tick, as the reference
 * rebuilds its grid, src/systems/forces.rs:228-232), 5 = persistent
 * neighbour list: pairs within r_c + skin on a grid of cells >= r_c + skin,
 * rebuilt (re-sort included) only when an atom has moved more than skin/2,
 * one thread per atom over its full list, no atomics; 6 = the same with a
 * half list (each pair once, the far end's force through integer atomics);
 * 7 = the half list of 6 with each thread's in-cutoff entries first
 * collected in shared memory, so that the warp evaluates the pair law on
 * them together (fewer idle lanes; same forces as 6, bit for bit);
 * 8 = the half list of 6 evaluated brick by brick (4 or 8 list-grid cells of
 * one x-row), the brick's neighbour rows staged in shared memory once and
 * read from there (same forces as 6, bit for bit); 8 also builds its lists
 * brick by brick from shared memory (the same lists).
 * 5-8 need >= 3 list-grid cells per axis, else they fall back to 4.  Variants 2 and 3 need >= 3 force-grid
 * cells per axis and fall back to 1 otherwise.  Variants 1-4 give
 * bit-identical forces, and so do 5-8 (fixed-point sums); 5-8
 * evaluate the same pair set in a cell-local frame whose origin is the
 * atom's cell at the last rebuild, so their FP32 forces can differ from 1-4
 * in the last bits (same error bound). */
int gx_set_kernel_variant(gx_handle* h, int variant);
/* Autotuner: times `reps` mixed pair passes of variants 1-4 on the resident
 * state (left bit-identical: they give the same fixed-point sums) and, where
 * variants 5-8 apply, full ticks of the best of them against full ticks
 * of 5-8, each list variant with its own work shape (lanes per atom and
 * far-end block, stash size, brick length) tuned first on a list built for
 * it, each from a snapshot of (x, v, a) restored afterwards.
 * Selects the fastest and returns it in *best.  ms[1..4], when given,
 * receive the per-pass milliseconds, ms[0], ms[5..8] the per-tick
 * milliseconds of the best pass variant and of 5-8 (-1 = not run); ms has
 * 9 entries.  Where a list variant wins, the list skin is
 * then chosen the same way over whole ticks among 0.05, 0.1, 0.15 and
 * 0.2 r_c (the list-grid cell is r_c + skin; gx_get_list_config reports
 * the choice), and the lanes per atom (the stash size of 7, the brick
 * length of 8) over passes
 * on a list of that skin.  The state is left as it was. */
int gx_autotune(gx_handle* h, int reps, int* best, double* ms);
/* No counterpart in the reference.  Skin of the variant-5/6 neighbour list
 * (default 0.1 r_c); 0 rebuilds every tick. */
int gx_set_list_skin(gx_handle* h, double skin);
/* Threads per atom of the variant-5/6 list pass: 1, 2, 4 or 8 lanes share
 * one atom's list (default 1; the autotuner picks the fastest).  Every
 * choice gives the same bits (integer sums).  No counterpart in the
 * reference. */
int gx_set_list_threads(gx_handle* h, int threads_per_atom);
/* Stash size of the variant-7 list pass: 8 or 16 in-cutoff entries per
 * thread are collected in shared memory before the warp evaluates them
 * (default 16; the autotuner picks the faster).  Both give the same bits.
 * No counterpart in the reference. */
int gx_set_list_stash(gx_handle* h, int slots);
/* The half-list pass with one lane per atom (variant 6): 128 or 256 atoms
 * per block with the far end of every pair inside the block summed in
 * shared memory (two 32-bit words with the carry), so that only the other
 * pairs send their far end's force to global memory; 0 = every far end to
 * global memory.  Default 0; the autotuner picks among 256, 128, 0 and the
 * wider lanes per atom.  All give the same bits.  No counterpart in the
 * reference. */
int gx_set_list_block(gx_handle* h, int threads);
/* The list pass's work shape as set or tuned: threads per atom, far-end
 * block (0, 128, 256), variant-7 stash slots (8, 16) and variant-8 brick
 * length (4, 8 cells). */
int gx_get_list_shape(gx_handle* h, int* threads_per_atom, int* block, int* stash_slots, int* brick_cells);
/* Brick length of the variant-8 list pass: 4 or 8 list-grid cells per brick
 * (at most 1024 or 2048 staged atoms; a brick with more reads global
 * memory).  Default 8; the autotuner picks the faster.  Both give the same
 * bits.  No counterpart in the reference. */
int gx_set_list_brick(gx_handle* h, int cells);
/* Skin and threads per atom of the variant-5/6 list pass. */
int gx_get_list_config(gx_handle* h, double* skin, int* threads_per_atom);
/* Occupancy of the current neighbour list: the entries it holds (pairs
 * within r_c + skin, each once on a half list) and the atoms whose list
 * overflowed its per-atom capacity (they scan their cells directly).  Zeros
 * when no list is built.  Synchronises the stream.  No counterpart in the
 * reference. */
int gx_list_stats(gx_handle* h, uint64_t* entries, uint64_t* overflowed_atoms);
/* Number of variant-5/6 list rebuilds so far (synchronises the stream). */
int gx_list_rebuilds(gx_handle* h, uint64_t* rebuilds);
/* Pair-pass timing: with `on`, every tick records two CUDA events around
 * its pair pass, also inside the captured tick (external event nodes of
 * the graph), so that gx_pass_ms gives the device time of the last tick's
 * pass as the replayed graph runs it.  Re-captures the ticks.  No
 * counterpart in the reference. */
int gx_set_pass_timing(gx_handle* h, int on);
int gx_pass_ms(gx_handle* h, double* ms);

/* ---- state ----------------------------------------------------------- */

/* Upload the ECS columns the hot path reads: Position, Velocity,
 * Acceleration (Vec3 AoS f64), AtomType as element index 0..9, Charge,
 * Mass, and EntityId::index per slot (src/systems/forces.rs:185-200;
 * src/components/*.rs).  acc may be NULL (zero, as spawn_atom writes,
 * src/universe/mod.rs:272); entity may be NULL (slot number). */
int gx_set_state(gx_handle* h, size_t n, const double* pos, const double* vel,
                 const double* acc, const uint8_t* elem, const double* charge,
                 const double* mass, const uint32_t* entity);
/* Download Position, Velocity, Acceleration in slot order (the write-backs
 * of src/systems/integrate.rs:40-43,63-66, boundary.rs:28-34,
 * forces.rs:343-345, thermostat.rs:68-70).  Any NULL pointer is skipped. */
int gx_get_state(gx_handle* h, double* pos, double* vel, double* acc);
size_t gx_num_atoms(const gx_handle* h);
/* Observed bonds as slot pairs, one entry per bond: the adjacency that
 * ForceSystem builds from the Bonds component (src/systems/forces.rs:208-226). */
int gx_set_bonds(gx_handle* h, size_t nbonds, const uint32_t* slot_pairs);

/* ---- systems of the force schedule (src/universe/mod.rs:356-369) ------ */

int gx_half_kick(gx_handle* h);  /* VelocityHalfKick::run, src/systems/integrate.rs:38-45 */
int gx_drift(gx_handle* h);      /* PositionDrift::run, src/systems/integrate.rs:61-67 */
int gx_wrap(gx_handle* h);       /* BoundarySystem::run, src/systems/boundary.rs:22-35 */
/* ForceSystem::run, src/systems/forces.rs:163-353: rebuilds the cell list
 * (counting sort by cell) and runs the pair pass; outputs PotentialEnergy,
 * BondEnergy and the number of pairs within the cutoff.  Any output may be NULL. */
int gx_forces(gx_handle* h, double* potential, double* bond_energy, uint64_t* pairs);
/* ThermostatSystem::run, src/systems/thermostat.rs:47-71. */
int gx_thermostat(gx_handle* h, double* kinetic, double* lambda);
/* StatsSystem reductions, src/systems/aggregate.rs:86-93. */
int gx_stats(gx_handle* h, double* kinetic, double* speed_sum);
/* nsteps ticks of the whole chain: kick, drift, [wrap], forces, kick,
 * [thermostat] -- Universe::tick with the force schedule
 * (src/universe/mod.rs:141-159, 356-369).  stats may be NULL, else it
 * receives nsteps entries.  Runs as one captured CUDA graph per tick
 * shape when use_graph != 0. */
int gx_step(gx_handle* h, int nsteps, gx_tick_stats* stats, int use_graph);

/* ---- parity probes and lenses ---------------------------------------- */

/* SpatialGrid::new + cell_of + encode (src/physics/grid.rs:67-86,228-246):
 * cell index of every atom, slot order, for a grid of cells >= min_cell. */
int gx_cell_assign(gx_handle* h, double min_cell, uint32_t* cells);
/* SpatialGrid::build + neighbors (src/physics/grid.rs:99-153): every pair
 * (slot a, slot b) with distance < cutoff on a grid of cells >= min_cell,
 * with the reference's multiplicity (a pair is repeated when an axis has
 * exactly two cells).  Order is unspecified.  Writes min(total, cap) pairs;
 * *npairs receives the total. */
int gx_neighbors(gx_handle* h, double min_cell, double cutoff, uint32_t* pairs,
                 size_t cap, size_t* npairs);
/* radial_distribution (src/analysis/mod.rs:87-133).  sample_cap is
 * G_SAMPLE_CAP (8192) for the reference's evenly spaced subsample, 0 for
 * every atom.  counts: nbins u64; bins: nbins f64 (may be NULL). */
int gx_radial_distribution(gx_handle* h, double r_max, size_t nbins, size_t sample_cap,
                           uint64_t* counts, double* bins, double* r_max_out,
                           double* dr_out);
/* radial_distribution_between (src/analysis/mod.rs:143-201). */
int gx_radial_distribution_between(gx_handle* h, uint8_t ta, uint8_t tb, double r_max,
                                   size_t nbins, size_t sample_cap, uint64_t* counts,
                                   double* bins, double* r_max_out, double* dr_out);
/* No counterpart in the reference.  g(r) for callers that cannot allocate
 * device memory: code held to a fixed device-memory budget, or code that must
 * not call cudaMalloc/cudaFree because those can synchronise the whole
 * device.  Same result as gx_radial_distribution with sample_cap = 8192, but
 * computed from host positions (pos: n x 3 f64, slot order) on the current
 * CUDA device, with every intermediate in one fixed file-scope device array
 * (about 1.9 MB per GPU that loads the library, held until exit); the call
 * allocates nothing.  Limits: the g(r) grid, floor(L/r_max) cells per axis,
 * may hold at most 65536 cells (GX_ERR_CAPACITY otherwise); nbins is clamped
 * to [1, 65536] like the reference; the sample never exceeds 8192 atoms.
 * The first call on a device looks up the array's address and should come
 * before any stream capture; the address is kept for the life of the
 * process, so a device reset (cudaDeviceReset) after that first call is not
 * supported.  Every call runs on the legacy default stream and waits for it,
 * so it must not run while another thread captures a graph in global mode.
 * Calls share the array: calls that overlap on the GPU race. */
int gx_radial_distribution_noalloc(size_t n, const double* pos, const double box[3], double r_max,
                                   size_t nbins, uint64_t* counts, double* bins, double* r_max_out,
                                   double* dr_out);
/* clusters (src/analysis/mod.rs:221-284): friends-of-friends with
 * r < bond_factor * sigma_ij.  labels[slot] = smallest slot of its
 * component; stats = {monomers, aggregates, largest, bound_pairs}. */
int gx_clusters(gx_handle* h, double bond_factor, uint32_t* labels, uint64_t stats[4],
                double* mean_size);
/* bound_pairs_with_grid (src/analysis/pairs.rs:132-174): entity-index pairs
 * (a < b) with r < k_bind * sigma_ij, reference multiplicity, unspecified
 * order. */
int gx_bound_pairs(gx_handle* h, double k_bind, uint32_t* pairs, size_t cap, size_t* npairs);

/* ---- snapshot ------------------------------------------------------- */

/* The world section of Universe::save (src/serialization/mod.rs:38-56,
 * 85-104): the bincode 1 encoding of Vec<EntitySnapshot> for the resident
 * atoms in ECS slot order, every record with all seven components (position,
 * velocity, mass, charge, atom type, bonds, acceleration), encoded on the
 * device.  Entity indices are the ones given to gx_set_state (else the slot);
 * generation[slot] (may be null: 0) gives each id's generation.  Bonds are
 * the handle's bond list, each slot's partners in ascending slot order.
 * *len receives the byte count (8 + 115 n + 16 bonds); GX_ERR_CAPACITY when
 * cap is smaller (out may be null to ask for the size).  The format number,
 * configuration, clock, RNG and statistics that precede the world in a
 * snapshot file come from the caller's own encoder. */
int gx_snapshot_world(gx_handle* h, const uint32_t* generation, uint8_t* out, size_t cap, size_t* len);

/* ---- bond observation ----------------------------------------------- */

/* One tick of BondObservationSystem::run (src/systems/bonds.rs:73-185) with
 * its PairTracker (src/analysis/pairs.rs:38-94), on the device: the bound
 * pairs (d < k_bind * sigma_ij, pairs.rs:132-174), episodes closed after
 * `debounce` consecutive absent ticks (DEBOUNCE = 2, bonds.rs:27), a pair
 * persistent once its episode lasts ceil(max(min_periods, 0.1) *
 * vib_period(eps_ij, sigma_ij, mu_ij) / dt) ticks (element masses,
 * bonds.rs:94-99), lifetimes from the tick a pair became persistent to the
 * tick its episode closed.  The open episodes stay on the device between
 * calls (pairs keyed by slot; gx_set_state starts afresh).  With
 * apply_bonds the persistent pairs replace the handle's bond list (the Bonds
 * component the next force pass reads, bonds.rs:116-121). */
typedef struct {
    uint64_t tick;               /* Time::tick passed in */
    uint64_t bound_pairs;        /* bound pairs this tick */
    uint64_t bonded_pairs;       /* BondObservation::bonded_pairs */
    uint64_t bonded_entities;    /* BondObservation::bonded_entities */
    double mean_coordination;    /* BondObservation::mean_coordination */
    uint64_t bonds_formed;       /* cumulative, BondObservation::bonds_formed */
    double lifetime_sum_ticks;   /* cumulative, BondObservation::lifetime_sum_ticks */
    uint64_t open_episodes;      /* PairTracker::open_count */
    uint64_t completed_episodes; /* PairTracker::completed().len() */
    uint64_t completed_ticks;    /* sum of the completed episodes' ticks */
    uint64_t species_matrix[GX_NELEM * GX_NELEM]; /* BondObservation::species_matrix */
} gx_bond_observation;

int gx_bond_observe(gx_handle* h, double k_bind, double min_periods, int debounce, uint64_t tick,
                    int apply_bonds, gx_bond_observation* out);
/* Drops the open episodes and the cumulative counts. */
int gx_bond_tracker_reset(gx_handle* h);
/* The connected components of the handle's bond list, for the bond-graph
 * chemistry lens (bond_components, src/analysis/mod.rs:331-411, used by
 * BondStructureSystem, src/systems/bond_structure.rs:66-117).  labels (may
 * be NULL; n entries, slot order): the smallest slot of the atom's
 * component, 0xFFFFFFFF for an atom in no bond.  edge_energy (may be NULL;
 * energy_cap >= *nbonds entries, gx_get_bonds order): the raw unswitched
 * pair energy of each bond at the current positions (pair_potential_raw,
 * src/physics/forces.rs:355-384), whose sums over a component's bonds are
 * its binding energy.  *nbonds (may be NULL) receives the bond count. */
int gx_bond_components(gx_handle* h, uint32_t* labels, double* edge_energy, size_t energy_cap, size_t* nbonds);
/* The handle's bond list as slot pairs (a < b for observed bonds). */
int gx_get_bonds(gx_handle* h, uint32_t* pairs, size_t cap, size_t* nbonds);

/* CollisionSystem::run (src/systems/collisions.rs:40-88) once on the
 * resident state: the pairs within 2 * particle_radius on a grid of that
 * cell (reference multiplicity on axes of 2 cells), the elastic impulse of
 * each approaching pair (elastic_pair, src/physics/collision.rs:16-32) from
 * the velocities before the pass, applied to every velocity once any pair
 * collided.  *collisions (may be NULL) receives the pairs that collided.
 * With gx_params.enable_collisions, gx_step runs the same pass after the
 * force pass of every tick (src/universe/mod.rs:362-365). */
int gx_collisions(gx_handle* h, uint64_t* collisions);
/* Collisions counted by every pass so far (CollisionCounter). */
int gx_collision_count(gx_handle* h, uint64_t* total);

/* ---- export ------------------------------------------------------------ */

/* One XYZ position frame of the current state, replaces export::write_frame
 * (src/export/mod.rs:152-172) minus the file write: "{n}\nframe {tick}\n",
 * then "{symbol} {x:.6} {y:.6} {z:.6}\n" per atom in slot order (the order
 * the caller gathered the world in).  Each coordinate is the exact value of
 * the double rounded to 6 decimals, ties to even, with '-' whenever the sign
 * bit is set, "NaN", "inf", "-inf": the bytes Rust's `{:.6}` prints.  The
 * text is formatted on the device and copied into out (cap bytes, no
 * terminating NUL); *len receives its size.  GX_ERR_CAPACITY when cap is
 * short (out may be NULL: a size query), GX_ERR_UNSUPPORTED for a
 * coordinate of magnitude >= 2^100. */
int gx_xyz_frame(gx_handle* h, uint64_t tick, char* out, size_t cap, size_t* len);

/* Per-tick column sync of a drop-in system whose ECS lives on the host:
 * overwrite Position, Velocity and Acceleration (slot order, AoS f64) of the
 * resident atoms without touching the static columns (AtomType, Mass,
 * Charge, EntityId).  Any pointer may be NULL (column unchanged). */
int gx_set_dynamic(gx_handle* h, const double* pos, const double* vel, const double* acc);
/* One Universe::tick (src/universe/mod.rs:141-159) of the force schedule
 * against host ECS columns: reads Position, Velocity and Acceleration (slot
 * order, AoS f64, all three required), runs the tick and writes the three
 * columns back in place -- the same results as gx_set_dynamic +
 * gx_step(h, 1, stats, 1) + gx_get_state, in one call.  The copies run on a
 * stream of their own and overlap the tick: each column is scattered to the
 * device order as it lands, and on the neighbour-list path the positions go
 * back while the pair pass runs.  Page-locked (pinned) columns give the
 * overlap; pageable ones are correct but copy synchronously.  stats may be
 * NULL, else it receives the tick's record.  Waits for the tick and
 * reports its pair-pass errors like gx_step. */
int gx_tick_host(gx_handle* h, double* pos, double* vel, double* acc, gx_tick_stats* stats);

/* ---- batched replicas (temperature sweep) ------------------------------ */

/* The reference sweeps temperatures with one fresh Universe per T, run one
 * after another (examples/temperature_sweep.rs:70-113).  A gx_batch holds
 * nrep independent universes of uneven sizes that share the laws in `base`
 * (mixed precision) and advances all of them together: as one captured
 * graph of all-replica kernels, in one persistent launch with one CTA per
 * replica, in one persistent cooperative launch that runs the
 * all-replica phases for every tick, or as the captured all-replica graph
 * over persistent neighbour lists (gx_batch_set_mode).  box: 3 doubles per replica; target_T: Berendsen target
 * per replica (<= 0 or base->enable_thermostat == 0: NVE); NULL uses
 * base->thermostat_temperature.  Each replica's force grid must have >= 1
 * and <= 4096 cells. */
typedef struct gx_batch gx_batch;
int gx_batch_create(const gx_params* base, int nrep, const double* box, const double* target_T,
                    gx_batch** out);
void gx_batch_destroy(gx_batch* b);
const char* gx_batch_last_error(const gx_batch* b);
/* Replica r owns atoms [sum(natoms[0..r)), +natoms[r]) of the concatenated
 * AoS/per-atom arrays (same column meaning as gx_set_state).  acc, charge,
 * mass may be NULL. */
int gx_batch_set_state(gx_batch* b, const uint32_t* natoms, const double* pos, const double* vel,
                       const double* acc, const uint8_t* elem, const double* charge,
                       const double* mass);
/* nsteps ticks of every replica in one launch.  stats (may be NULL): 4
 * doubles per replica after the last tick -- kinetic energy after the
 * thermostat, potential energy, lambda, pairs.  device_ms (may be NULL):
 * CUDA-event time of the launch. */
int gx_batch_step(gx_batch* b, int nsteps, double* stats, double* device_ms);
int gx_batch_get_state(gx_batch* b, double* pos, double* vel, double* acc);
/* Execution mode: 1 = one persistent launch, one CTA per replica (every
 * replica grid <= 4096 force cells, else GX_ERR_CAPACITY at the step);
 * 2 = every phase of the tick as one kernel over the atoms of all
 * replicas (a global cell index, per-replica geometry), captured once as a
 * CUDA graph; 3 = the phases of mode 2 inside one persistent cooperative
 * launch for all the ticks of a step call, separated by grid barriers
 * whose waits are bounded (GX_ERR_TIMEOUT if one gives up); 4 = the
 * all-replica graph of mode 2 over persistent half neighbour lists (a list
 * grid of cells >= r_c + skin per replica, a rebuild only after some atom
 * moved more than skin/2, as the single-universe variant 6; every replica
 * must hold >= 128 atoms and >= 3 list-grid cells per axis, else the step
 * returns GX_ERR_UNSUPPORTED); 0 = the default (2).  Modes 1-3 give each
 * NVE replica the same bits as a gx_handle on pair-pass variants 1-4, and
 * modes 2 and 3 give each other the same bits with the thermostat on; mode
 * 4 evaluates the same pairs in the list grid's cell-local frame, so its
 * forces differ from mode 2's in the last FP32 bits (same error bound). */
int gx_batch_set_mode(gx_batch* b, int mode);
int gx_batch_get_mode(gx_batch* b, int* mode);
/* Times `ticks` ticks in each mode from a snapshot of the state (restored
 * afterwards), keeps the fastest; ms[0..3] (may be NULL) receive the
 * per-tick device milliseconds of modes 1-4 (-1: mode skipped, 1 because a
 * replica grid exceeds its limit, 4 because a replica is too small). */
int gx_batch_autotune(gx_batch* b, int ticks, int* mode, double* ms);
/* Mode 4's list skin (default 0.15 r_c; the list grid's cells are >= r_c +
 * skin; gx_batch_autotune picks among 0.1, 0.15 and 0.2 r_c when it times
 * mode 4).  No counterpart in the reference. */
int gx_batch_set_list_skin(gx_batch* b, double skin);
/* Mode 4's list rebuilds so far (synchronises the batch's stream). */
int gx_batch_list_rebuilds(gx_batch* b, uint64_t* rebuilds);
/* Mode 4's current lists: entries held (an overflowed slot counts those it
 * found) and slots whose list overflowed (they scan their 27 home-grid
 * cells directly, the same pairs).  Synchronises. */
int gx_batch_list_stats(gx_batch* b, uint64_t* entries, uint64_t* overflowed_slots);

/* ---- adjoint: derivatives of short NVE horizons ----------------------- */

/* No counterpart in the reference, which has no derivatives.  Reverse-mode
 * gradients with respect to the per-element sigma[10] and epsilon_k[10] of
 * gx_params, of any loss of two smoothed observables of the trajectory that
 * starts from the handle's current state (the state is left unchanged):
 *   V_t  the potential energy (LJ + Coulomb + gravity) after tick t = 1..T;
 *   g_k  a Gaussian-kernel pair distribution averaged over the ticks
 *        t = gr_every, 2 gr_every, ... <= T:
 *          g_k = c_k * sum over pair-list entries with |d - r_k| < gr_support * w
 *                of exp(-(d - r_k)^2 / (2 w^2)),
 *          r_k = (k + 1/2) gr_rmax / gr_bins,  w = gr_width,
 *          c_k = L_x L_y L_z / (N (N - 1) / 2 * 4 pi r_k^2 * sqrt(2 pi) w).
 * The ticks are the reference's (src/universe/mod.rs:356-369: kick, drift,
 * wrap, forces, kick): on a GX_FP64 handle in FP64 with its per-pair
 * arithmetic; on a GX_MIXED handle in the mixed method (the FP32 pair law on
 * the FP64 displacement rounded to FP32, forces summed in 2^-32 fixed point,
 * FP64 positions, velocities and observables), at most 16 kinds.  The
 * adjoint is FP64 in both, linearised on the forward's trajectory.
 * gx_adjoint_forward keeps a checkpoint of (x, v, a)
 * every checkpoint_every ticks; gx_adjoint_backward recomputes each segment
 * from its checkpoint and runs the adjoint of the velocity-Verlet step and
 * of the force pass backwards through it.  The cutoffs (LJ, Coulomb,
 * gravity) are multiples of max sigma: their derivative goes to the
 * lowest-index element with the largest sigma.  Supported: LJ, Coulomb,
 * gravity, periodic wrap, every epsilon_k > 0; the thermostat and the bond
 * spring give GX_ERR_UNSUPPORTED.  gr_rmax + gr_support * gr_width must not
 * exceed the force cutoff; gr_bins <= 512. */
typedef struct {
    int32_t nsteps;           /* horizon T >= 1 */
    int32_t checkpoint_every; /* K >= 1 */
    int32_t gr_bins;          /* number of g bin centres; 0 = no g observable */
    int32_t gr_every;         /* sample g every this many ticks (>= 1) */
    double gr_rmax;
    double gr_width;          /* kernel width w */
    double gr_support;        /* kernel truncated at gr_support * w */
} gx_adjoint_spec;

/* potential: [nsteps] V_t.  gr: [gr_bins] the time-averaged g_k, or NULL. */
int gx_adjoint_forward(gx_handle* h, const gx_adjoint_spec* spec, double* potential, double* gr);
/* dl_dpotential [nsteps] and dl_dgr [gr_bins] are the cotangents dL/dV_t and
 * dL/dg_k of the caller's loss L (NULL = zero).  Writes dL/dsigma[10] and
 * dL/depsilon_k[10]; grad_pos0 / grad_vel0 / grad_acc0 (slot-ordered [3n] or
 * NULL) receive dL/d(initial position, velocity, acceleration).  Uses the
 * checkpoints of the last gx_adjoint_forward on this handle. */
int gx_adjoint_backward(gx_handle* h, const double* dl_dpotential, const double* dl_dgr, double* grad_sigma,
                        double* grad_epsilon_k, double* grad_pos0, double* grad_vel0, double* grad_acc0);

/* ---- timing ---------------------------------------------------------- */

/* Waits for the handle's stream; reports an error an asynchronous gx_step
 * left (see gx_set_step_async). */
int gx_synchronize(gx_handle* h);
/* on = 1: gx_step without per-tick records returns once its work is queued,
 * without waiting for the GPU; an error its pair pass raised (saturation,
 * non-finite force, timeout) is returned by the next call that waits:
 * gx_synchronize, gx_get_state, gx_bond_observe, or gx_set_step_async(h, 0).
 * Lets a host scheduler queue the force systems and the observation of one
 * tick behind a single wait.  Default 0: gx_step waits and reports. */
int gx_set_step_async(gx_handle* h, int on);
/* Records CUDA event `slot` (0..15) on the handle's stream. */
int gx_timer_mark(gx_handle* h, int slot);
/* Milliseconds between two recorded events (waits for the second). */
int gx_timer_elapsed(gx_handle* h, int from_slot, int to_slot, double* ms);
/* Number of kernels this handle has launched since creation. */
uint64_t gx_launch_count(const gx_handle* h);
/* Diagnostic: measured FP32 FMA throughput of this GPU in TFLOP/s (a
 * dependent-FMA loop on every SM; roofline denominator for the pair pass). */
int gx_measure_fp32_peak(int device, double* tflops);
/* The same measurement for the FP64 pipe (independent FP64 FMA chains on every
 * SM): the denominator of the plain FP64 pair pass's roofline.  No
 * counterpart in the reference. */
int gx_measure_fp64_peak(int device, double* tflops);
/* Per-kernel CUDA-event timing of gx_step/gx_forces launches (on the
 * handle's stream).  When enabled, each launch is bracketed by events. */
int gx_profile_enable(gx_handle* h, int on);
/* Names, launch counts and summed milliseconds since the last reset;
 * returns the number of kernels (up to cap entries written). */
int gx_profile_read(gx_handle* h, const char** names, uint64_t* launches, double* ms,
                    int cap, int reset);

#ifdef __cplusplus
}
#endif
#endif /* GENESIS_GPU_H */
