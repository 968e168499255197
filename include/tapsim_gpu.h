/* tapsim_gpu.h — C ABI of the B200 implementation of TAPSim's per-event hot
 * path (relax -> field ratio / argmax -> atom removal -> ion flight).
 *
 * The reference has no plugin or FFI layer: the path sits behind the C++
 * class API that Process::evaporation (tapsim/process.cpp:441-1124) calls.
 * Every device entry point below replaces one of those calls and names it.
 * Plain pointers and sizes only; all device memory is owned by the handle;
 * inputs are copied at the call, outputs go to caller-allocated host arrays.
 * Errors are int status codes (TG_OK == 0); nothing throws across the ABI.
 * A handle is used from one host thread; its work is ordered on one CUDA
 * stream.
 */
#ifndef TAPSIM_GPU_H
#define TAPSIM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    TG_OK = 0,
    TG_ERR_ARGUMENT = 1,        /* invalid argument / size */
    TG_ERR_CUDA = 2,            /* CUDA runtime error (message via tg_last_error) */
    TG_ERR_NAN = 3,             /* NaN in a potential, field or trajectory */
    TG_ERR_SINGULAR = 4,        /* singular 3x3 system in field_o1 */
    TG_ERR_NOT_SURFACE = 5,     /* removal of a node that is not a surface cell */
    TG_ERR_RELAX_FAULT = 6,     /* stagnation (Grid_3d::Table::RelaxationFault) */
    TG_ERR_ITERATION_CAP = 7,   /* iteration cap reached before the tolerance */
    TG_ERR_OUTSIDE = 8,         /* trajectory start point outside the mesh */
    TG_ERR_WALK_LIMIT = 9,      /* tetrahedron walk exceeded its step bound */
    TG_ERR_NO_SURFACE = 10,     /* surface set is empty */
    TG_ERR_HOST = 11,           /* host-side failure (file, mesh build) */
    TG_ERR_UNKNOWN_TYPE = 12,   /* cell type id not in the type table */
    TG_ERR_TIMEOUT = 13         /* a bounded wait inside a kernel ran out */
};

/* Trajectory status, values of Trajectory_3d's enum (trajectory_3d.h:89). */
enum {
    TG_TRAJ_INVALID = -1,
    TG_TRAJ_NO_INTEGRATION = 0,
    TG_TRAJ_NO_FIELD = 1,
    TG_TRAJ_STEPPER_LIMIT_PASSED = 2,
    TG_TRAJ_ITERATION_LIMIT_PASSED = 3,
    TG_TRAJ_GEOMETRY_LIMIT_PASSED = 4,
    TG_TRAJ_SYSTEM_LIMIT_PASSED = 5
};

/* ---- cell types: Configuration::NodeData (configuration.h:70-160) -------- */
typedef struct {
    int32_t id;               /* NodeId value 0..127 */
    float charge_density;     /* [C/m^3] */
    float epsilon;            /* relative permittivity */
    int32_t removable;
    int32_t neumann;
    int32_t dirichlet;
    float phi;                /* preset potential [V] */
    float mass;               /* [amu] */
    int32_t evap_charge;      /* charge state */
    float evap_field;         /* [V/m] */
    float evap_energy;        /* [eV] */
} tg_type;

/* ---- mesh description (replaces System_3d, system_3d.h:29-42) ------------
 * Node order is the node-file order; all indices are node-file indices.   */
typedef struct {
    int32_t num_nodes;
    const float* xyz;              /* [3N] Geometry_3d::NodeData::coords [m] */
    const int8_t* type_id;         /* [N]  Grid_3d::Node::id */
    const uint8_t* hull;           /* [N]  Geometry_3d::NodeData::boundary */
    const float* phi;              /* [N]  initial potential [V] */
    const int32_t* row_ptr;        /* [N+1] Delaunay neighbours, ascending */
    const int32_t* col;            /* [nnz] */
    const double* coupling;        /* [nnz] c_ij as Grid_3d::Table::fastSync leaves it */
    const double* geom;            /* [nnz] face area(0.5 d)/d; NULL: derived from coupling */
    const uint8_t* area_pos;       /* [nnz] face area(1.0) > 0; NULL: coupling-derived */
    const double* volume;          /* [N]  capped Voronoi volume; NULL: zero charge */
    int32_t num_tets;
    const int32_t* tet_v;          /* [4T] vertices, positively oriented */
    const int32_t* tet_n;          /* [4T] neighbour k opposite vertex k, -1 on the hull */
    const int32_t* node_tet;       /* [N]  associated tetrahedron */
    int32_t num_types;
    const tg_type* types;
} tg_mesh_desc;

typedef struct tg_handle tg_handle;

/* Creates the device state from a mesh description.  Copies every array. */
int tg_create(const tg_mesh_desc* desc, tg_handle** out);
void tg_destroy(tg_handle* h);
/* Last error message of the handle (or of the process when h == NULL). */
const char* tg_last_error(const tg_handle* h);
int tg_num_nodes(const tg_handle* h);

/* ---- potentials: Grid_3d::Table ---------------------------------------- */
/* Grid_3d::Table::relax(n) (grid_3d.cpp:591-609): n coloured Gauss-Seidel
 * sweeps over all free cells (computePotential, grid_3d.cpp:1317-1371);
 * *deviation = max |phi_new - phi_old| of the last sweep. */
int tg_relax_cycles(tg_handle* h, int32_t n, double* deviation);
/* Grid_3d::Table::relax(thr, cycle, queue) (grid_3d.cpp:611-671): repeats
 * relax(cycle) until the deviation is <= thr; TG_ERR_RELAX_FAULT on the
 * stagnation rule (zero regression slope over `queue` deviations),
 * TG_ERR_ITERATION_CAP after max_sweeps. */
int tg_relax_threshold(tg_handle* h, double threshold, int32_t cycle, int32_t queue, int64_t max_sweeps,
                       int64_t* iterations, double* deviation);
/* Grid_3d::Table::localRelax(idx, order, thr, cycle, queue)
 * (grid_3d.cpp:707-795, find_localNodes :1284-1315). */
int tg_local_relax(tg_handle* h, int32_t node, int32_t shell, double threshold, int32_t cycle, int32_t queue,
                   int64_t* iterations, double* deviation);

/* Solves the finite-volume system to a relative residual ||r||_2/||b||_2 <=
 * rel_tol (r_i = sum_j c_ij (phi_j - phi_i) - q_i over free cells, b = the
 * Dirichlet part).  FP64 residual and update, FP32 inner iterations.  No
 * counterpart in the reference, which stops on max |delta phi| instead. */
typedef struct {
    double rel_tol;           /* e.g. 1e-8 */
    int32_t max_outer;        /* FP64 defect-correction steps */
    int32_t max_inner;        /* inner iterations per step */
    double inner_rtol;        /* inner relative reduction per step */
    /* Start of a solve that follows removals from a converged state:
     *   0  the current potentials (the previous event's solution; plain),
     *   1  plus the previous event's correction on the non-Neumann free
     *      cells (the smooth far field of one removal changes little
     *      from one site to the next),
     *   2  as 1, plus the prediction of an attached learner on the free
     *      cells around the removed atom (tg_learner_attach, mode bit 1),
     *      which also joins the recorded correction; the first residual is
     *      updated in FP64 on those cells' rows and their neighbours'
     *      instead of a pass over every row.
     * The solve always ends at rel_tol, whatever the start. */
    int32_t warm_start;
    /* Preconditioner of the inner iterations on the non-Neumann free cells:
     *   0  Jacobi (the diagonal),
     *   1  a smoothed-aggregation multigrid V(1,1)-cycle, its hierarchy
     *      built on the host at the first solve that asks for it and again
     *      once removals have added 2% more cells to the system. */
    int32_t preconditioner;
    /* Arithmetic of the inner iterations on the non-Neumann free cells:
     *   0  FP32 (couplings, vectors and recurrences; the default),
     *   1  FP64 couplings, vectors and recurrences, the multigrid V-cycle
     *      still FP32 (needs preconditioner 1 and warm_start 0).  Its FP64
     *      copy of the couplings is built at the first such solve.
     * The residual test, its norm and the potential update are FP64 in both;
     * the Neumann rows' inner iterations are FP32 in both. */
    int32_t inner_precision;
} tg_solve_opts;
typedef struct {
    int32_t outer;            /* defect-correction steps taken */
    int32_t inner;            /* FP32 iterations taken in total */
    double rel_residual;      /* final ||r||/||b|| */
    double initial_rel_residual;
    int32_t inner_neumann;    /* of `inner`, the iterations on the Neumann rows */
    int32_t residual_cells;   /* cells flipped since the last converged solve whose rows, and their
                                 neighbours', the first residual recomputed from the kept residuals;
                                 0 when the first residual was a pass over every row */
    double setup_seconds;     /* multigrid hierarchy built during this solve [s], 0 if none */
} tg_solve_info;
int tg_solve(tg_handle* h, const tg_solve_opts* opts, tg_solve_info* info);
/* The schedule of one level of the multigrid hierarchy (no counterpart in
 * the reference): its rows, and the lanes per CSR row of its operator
 * (levels smoothed with CSR rows) and of its restriction (every level but
 * the coarsest), 0 where the level has none; for level 0, a_lanes is the
 * number of coupling loads each lane of the SELL-32 smoothing pass issues
 * ahead of their gathers (4, 8 or 16; 1004 or 1008 for the software-
 * pipelined pass, which loads the next 4 or 8 while it gathers the current
 * ones).  The hierarchy build chooses them
 * one at a time, from a row-length rule, by timing whole V-cycles with
 * each candidate, and keeps a change that takes 3% off the cycle; a_ms /
 * r_ms are the kept kernels' own launch times [ms]. */
int tg_amg_schedule(tg_handle* h, int32_t level, int32_t* rows, int32_t* a_lanes, int32_t* r_lanes, float* a_ms,
                    float* r_ms);
/* ||r||_2 / ||b||_2 of the current potentials (FP64). */
int tg_residual(tg_handle* h, double* rel_residual);

int tg_get_phi(tg_handle* h, double* phi_out);       /* [N] */
int tg_set_phi(tg_handle* h, const double* phi_in);  /* [N] */
/* Grid_3d::Table::field_o1 (grid_3d.cpp:909-991) for a list of nodes. */
int tg_field_o1(tg_handle* h, int32_t count, const int32_t* nodes, double* field_out /* [3*count] */);
/* tg_field_o1 that makes no device allocation; no counterpart in the
 * reference.  For callers that cannot allocate device memory when they ask
 * for fields: all device memory already committed to the mesh and to another
 * allocator's pool, or a real-time loop that must stay off the allocator.
 * tg_field_o1 grows per-handle staging buffers with cudaMalloc; this call
 * stages the node list and the results in a fixed scratch array that is part
 * of the library's device image instead.
 *   - At most TG_FIELD_O1_NOALLOC_MAX nodes per call; a longer list fails
 *     with TG_ERR_ARGUMENT before anything runs.  Node indices are checked
 *     against the mesh (TG_ERR_ARGUMENT when out of range).
 *   - The first call on a device looks up the scratch's device address
 *     (which can load the library's device image onto that device); make
 *     that first call before any stream capture.
 *   - There is one scratch per device, shared by all handles and threads of
 *     the process: calls that overlap on the same device (from two threads,
 *     or two handles) race on it and return each other's results.  Calls
 *     made one after another are safe.
 * Results equal tg_field_o1's for the same nodes. */
#define TG_FIELD_O1_NOALLOC_MAX 65536
int tg_field_o1_noalloc(tg_handle* h, int32_t count, const int32_t* nodes, double* field_out /* [3*count] */);
/* Current coupling, type and effective diagonal (for checks). */
int tg_get_couplings(tg_handle* h, double* coupling_out /* [nnz] */);
int tg_get_types(tg_handle* h, int8_t* type_out /* [N] */);

/* ---- surface: Surface_3d --------------------------------------------- */
/* Surface_3d::Table::init (surface_3d.cpp:50-81). */
int tg_surface_init(tg_handle* h, int32_t vacuum_id, int32_t* num_surface);
/* evap_compute_specificFields + evap_compute_probabilities(PROB_LINEAR_FIELD)
 * + evapMaximum (surface_3d.cpp:194-219, 267-297, 423-431) in one pass:
 * ratio_i = |E_i| / E_evap(type_i); the candidate is the first maximum in
 * ascending node order; second is the runner-up (near-tie margin). */
typedef struct {
    int32_t num_surface;
    int32_t candidate;          /* node index, -1 when the surface is empty */
    float best_ratio;           /* = scaling reference */
    float second_ratio;
    double ratio_sum;
    float probability;          /* the candidate's normalised probability */
    int32_t apex;               /* Surface_3d::Table::apex (surface_3d.cpp:171-190) */
    int32_t prob_mode;          /* probability mode of this selection */
    float best_probability;     /* the two largest normalised probabilities */
    float second_probability;   /* (near-tie margin = (best - second) / best) */
    double score_sum;           /* sum of the scores before normalisation */
} tg_select_info;
int tg_surface_select(tg_handle* h, tg_select_info* info);
/* The same with Surface_3d::evap_compute_probabilities' mode
 * (surface_3d.cpp:220-399): 0 linear field, 1 Boltzmann at `temperature`
 * [K] (> 0), 2 linear force (field_o2, grid_3d.cpp:993-1199), 3 Voronoi
 * flux force.  The candidate is evapMaximum's: the first maximum of the
 * normalised probabilities in ascending node order. */
int tg_surface_select_mode(tg_handle* h, int32_t prob_mode, float temperature, tg_select_info* info);
/* evapMonteCarlo (surface_3d.cpp:433-449) on the last selection: the first
 * surface cell, in ascending node order, whose cumulative probability
 * reaches u in [0, 1] (the last cell when none does). */
int tg_surface_pick(tg_handle* h, double u, int32_t* node, float* probability);
int tg_get_surface(tg_handle* h, int32_t capacity, int32_t* nodes, float* ratios, int32_t* count);
/* Surface_3d::Table::normal (surface_3d.cpp:123-169). */
int tg_surface_normal(tg_handle* h, int32_t node, float normal_out[3]);
/* evap_takeAway (surface_3d.cpp:507-564): flip to vacuum, fastResync
 * (grid_3d.cpp:555-589), surface update (surface_3d.cpp:83-119) and removal
 * of detached neighbours.  detached_out receives up to `capacity` indices. */
int tg_take_away(tg_handle* h, int32_t node, int32_t capacity, int32_t* detached_out, int32_t* num_detached);
/* update_coordination (surface_3d.cpp:568-593). */
int tg_update_coordination(tg_handle* h);

/* Potential, field_o1 and Grid_3d::Table::force (grid_3d.cpp:1201-1236) of
 * cells nodes[0..count), as float (the values LogGrid::push and
 * LogSurface::prepare collect, logGrid.cpp:119-143, logSurface.cpp:159-201);
 * nodes NULL: every cell (count = N).  Any output may be NULL. */
int tg_cell_values(tg_handle* h, int32_t count, const int32_t* nodes, float* phi_out, float* field_out /* [3*count] */,
                   float* force_out /* [3*count] */);
/* Surface_3d::Table::normal of each listed cell, one block per cell. */
int tg_surface_normals(tg_handle* h, int32_t count, const int32_t* nodes, float* normals_out /* [3*count] */);
/* The surface set in ascending index order with the probabilities of
 * METHOD_EVAPORATION_PROBABILITY prob_mode, normalised as
 * evap_compute_probabilities leaves them (surface_3d.cpp:220-420).  *count
 * is the set's size; at most capacity cells are written. */
int tg_surface_cells(tg_handle* h, int32_t prob_mode, float temperature, int32_t capacity, int32_t* count,
                     int32_t* cells, float* probability);
/* LogGrid::push + its writer thread (logGrid.cpp:119-245) for the handle's
 * current state: writes path.%08u (index) in ASCII or binary.  numbers:
 * the cells' unique numbers (tg_mesh_numbers), NULL for index + 1. */
int tg_log_grid(tg_handle* h, const char* path, int32_t index, int32_t binary, const uint32_t* numbers);
/* LogSurface::push + writer (logSurface.cpp:130-293) for the handle's
 * current state and probability mode: writes path.%08u (index). */
int tg_log_surface(tg_handle* h, const char* path, int32_t index, int32_t binary, int32_t with_neighbours,
                   int32_t prob_mode, float temperature, const uint32_t* numbers);

/* ---- ion flights: Trajectory_3d ---------------------------------------- */
typedef struct {
    double time_step;           /* TRAJECTORY_INITIAL_TIME_STEP [s] */
    double min_time_step;       /* TRAJECTORY_MINIMUM_TIME_STEP [s] */
    double error_threshold;     /* TRAJECTORY_ERROR_THRESHOLD */
    int32_t max_steps;          /* iteration bound per ion */
    int32_t stepper_limit;      /* trial steps per accepted step */
    int32_t walk_limit;         /* tetrahedra per point location */
    int32_t integrator;         /* TRAJECTORY_INTEGRATOR_TYPE: 0 Euler, 1 Cash-Karp (the reference's default) */
    int32_t stepper;            /* TRAJECTORY_STEPPER_TYPE: 0 none, 1 error-restricted (default),
                                   2 geometry-restricted, 3 adaptive (trajectory_3d.cpp:358-532) */
    /* Arithmetic of the Cash-Karp steps and of the error-restricted step
     * control: 0 FP64 (default), 1 FP32 (as the reference integrates,
     * trajectory_3d.cpp:583-676), 2 FP64 while the ion is within fp64_radius
     * [m] of its start, where the field is steep, and FP32 beyond.  Point
     * location and field interpolation are FP64 (exact orientation) in all
     * three; the Euler integrator is FP64. */
    int32_t precision;
    double fp64_radius;
} tg_trace_opts;
typedef struct {
    float stop[3];              /* impact after extrapolation to the top plane [m] */
    float stop_time;            /* [s] */
    float last_pos[3];          /* last point inside the mesh [m] */
    int32_t last_tet;
    float last_phi;             /* Grid_3d::potential at last_pos [V] */
    int32_t steps;              /* accepted steps */
    int32_t status;             /* TG_TRAJ_* */
    int32_t trials;             /* integrator trial steps, accepted and rejected */
} tg_impact;
/* Trajectory_3d::init/integrate/extrapolate (trajectory_3d.cpp:99-209,
 * 303-332) with o5_integrator (Cash-Karp, :583-676) and
 * errorRestricted_stepper (:358-425), batched: one ion per thread. */
int tg_trace(tg_handle* h, int32_t n_ions, const float* start_xyz, const float* start_vel,
             const float* charge_over_mass, const int32_t* tet_guess, const tg_trace_opts* opts, tg_impact* out);
/* One phase-space point of a flight, Trajectory_3d::phaseVector
 * (trajectory_3d.h:40-80): time [s] from the start, position [m], velocity
 * [m/s], tetrahedron (-1 outside the mesh). */
typedef struct {
    float time;
    float position[3];
    float velocity[3];
    int32_t tet;
} tg_path_point;
/* tg_trace that also keeps each flight's path as Trajectory_3d::data()
 * holds it: the start, one point per accepted step (the one that leaves the
 * mesh with tet -1) and the point extrapolated to the top plane
 * (trajectory_3d.cpp:99-209, 303-332), plus error_estimate(): the
 * component-wise root sum of squares of the accepted steps' error vectors
 * (cumulative_error, :683-700), the position part grown by the extrapolation
 * time times the velocity part (:329).  Ion k's path fills
 * points[k*cap .. k*cap + cap-1]; it has impact.steps + 2 points (0 when the
 * start is outside the mesh), and a path longer than cap keeps its first cap
 * points.  errors[6k .. 6k+5] = position x, y, z, velocity x, y, z. */
int tg_trace_path(tg_handle* h, int32_t n_ions, const float* start_xyz, const float* start_vel,
                  const float* charge_over_mass, const int32_t* tet_guess, const tg_trace_opts* opts, int32_t cap,
                  tg_impact* out, tg_path_point* points, float* errors);
/* Grid_3d::potential(geom, grid, pos, tet) (grid_3d.cpp:1585-1602). */
int tg_potential_at(tg_handle* h, int32_t n, const float* xyz, const int32_t* tet_guess, float* phi_out);

/* ---- one evaporation event: Process::evaporation steps I-VI ------------ */
typedef struct {
    int32_t vacuum_id;
    int32_t relax_mode;         /* 0: reference (local + global sweeps, refresh), 1: solve to rel_tol */
    /* relax_mode 0: LOCAL_RELAXATION_*, GLOBAL_RELAXATION_STEPS, REFRESH_RELAXATION_* */
    double local_threshold;
    int32_t local_shell, local_cycle, local_queue;
    int32_t global_steps;
    int32_t refresh_interval;
    double refresh_threshold;
    int32_t refresh_cycle, refresh_queue;
    int64_t refresh_max_sweeps;
    /* relax_mode 1 */
    tg_solve_opts solve;
    tg_trace_opts trace;
    int32_t trace_enabled;
    int32_t normal_enabled;
    /* METHOD_EVAPORATION_PROBABILITY (0 linear field, 1 Boltzmann, 2 linear
     * force, 3 Voronoi flux force) and METHOD_EVAPORATION_CHOICE (0
     * maximum, 1 Monte-Carlo); the configuration's TEMPERATURE [K] for
     * Boltzmann; the seed of the handle's Monte-Carlo stream, which draws
     * like rand() after srand(seed) (the reference seeds 99, tapsim.cpp:235),
     * seeded at the first Monte-Carlo choice of the handle */
    int32_t prob_mode;
    int32_t choice_mode;
    float temperature;
    uint32_t rng_seed;
    /* !TRAJECTORY_NO_INITIAL_VELOCITY: draw the ion's initial velocity as
     * evap_initialVelocity does (surface_3d.cpp:472-503) from the same
     * stream; 0 starts it at rest (the reference's default) */
    int32_t initial_velocity;
    /* path_cap > 0 keeps each event's flight path for the trajectory log
     * (LogTrajectory, logTrajectory.cpp:137-300) as tg_trace_path does: the
     * k-th event of a call writes path_points[k*path_cap ..] (host memory,
     * count*path_cap points) and path_errors[6k .. 6k+5] */
    int32_t path_cap;
    tg_path_point* path_points;
    float* path_errors;
    /* Forced removals (the reference harness's --force, for comparing a run
     * with another one event by event past a near-tie): when force_nodes is
     * not NULL, the k-th event of a call (k < force_count) removes
     * force_nodes[k] instead of the chosen cell; later events choose as
     * usual.  The cell must be on the surface (TG_ERR_ARGUMENT otherwise).
     * The record's probability is then the forced cell's, while
     * best_probability stays the chosen cell's: probability <
     * best_probability marks an event where the forced cell was not this
     * run's choice.  No counterpart in Process::evaporation. */
    const int32_t* force_nodes;
    int32_t force_count;
} tg_event_opts;
typedef struct {
    int32_t node;
    int32_t type_id;
    float probability;
    float best_ratio, second_ratio;  /* near-tie margin = (best - second)/best */
    float scaling_reference;         /* of the selection step */
    float phi_before, field_before[3];
    float phi_after, field_after[3];
    float apex[3];
    float normal[3];
    tg_impact impact;
    int32_t detached;
    int32_t relax_iterations;
    double rel_residual;
    int32_t relax_status;
    float best_probability, second_probability;  /* of the selection that chose node */
} tg_event_record;
int tg_run_event(tg_handle* h, const tg_event_opts* opts, int32_t event_index, tg_event_record* rec);
/* `count` events in one call (indices first_index, first_index+1, ...):
 * the same steps and records as tg_run_event, with each event's ion flight
 * on a second stream overlapping the next event's removal and relaxation
 * (the flight reads snapshots of the vertex fields and potentials taken
 * after its own event's relaxation).  *done = events completed; on an error
 * the records before it are complete. */
int tg_run_events(tg_handle* h, const tg_event_opts* opts, int32_t first_index, int32_t count,
                  tg_event_record* recs, int32_t* done);
/* One event on each of `count` independent tips (many-tip serving; no
 * counterpart in the reference, which evaporates one specimen per process):
 * tg_run_events(handles[k], &opts[k], first_index, 1, &recs[k]) for every k,
 * the handles driven concurrently from a pool of host threads (threads <= 0:
 * one per handle up to the host's cores; each handle by one thread, so the
 * one-thread-per-handle rule holds), their device work overlapping on the
 * handles' own streams.  latency_ms[k]: the host wall time of tip k's event;
 * status[k]: its return code.  Returns TG_OK when every tip's event ran, else
 * the first failing code (TG_ERR_NO_SURFACE for a tip that has run out). */
int tg_run_tips(tg_handle* const* handles, int32_t count, const tg_event_opts* opts, int32_t first_index,
                tg_event_record* recs, float* latency_ms, int32_t* status, int32_t threads);

/* ---- learned near-field warm start (no counterpart in the reference) -----
 * A message-passing network (an input layer and four message layers of
 * width 64, BF16 tensor-core GEMMs with FP32 accumulation) on the free cells
 * within `hops` steps of a removed atom predicts the part of the event's
 * correction on those cells that the start leaves (the recycled far field
 * of warm_start 1, or the plain start).  Samples are (features of the state
 * the solve starts from, converged correction) pairs that tg_solve collects
 * while a learner is attached in collect mode; the network is trained on
 * them on the device; tg_solve with warm_start 2 adds its prediction on top
 * of the recycled far field before the inner iterations.  The solve still
 * ends at rel_tol. */
typedef struct tg_learner tg_learner;
int tg_learner_create(int32_t hops, int32_t max_cells, int32_t ell_width, uint64_t seed, tg_learner** out);
void tg_learner_destroy(tg_learner* L);
const char* tg_learner_last_error(const tg_learner* L);
int32_t tg_learner_num_params(void);
/* multiplier of the prediction that warm_start 2 adds (default 1; 0: no
 * prediction, the sweeps below alone) */
int tg_learner_set_gain(tg_learner* L, float gain);
/* damped Jacobi sweeps (weight 0.8) over the graph's cells after the
 * prediction, every other cell held (computePotential's update); they
 * remove the prediction's high-frequency error.  Default 0; graphs of at
 * most 4096 cells. */
int tg_learner_set_refine(tg_learner* L, int32_t sweeps);
/* mode: 0 detach, bit 0 collect samples, bit 1 predict (for warm_start 2).
 * The learner's graph width must hold the mesh's longest row. */
int tg_learner_attach(tg_handle* h, tg_learner* L, int32_t mode);
int tg_learner_samples(const tg_learner* L, int32_t* count, int64_t* cells);
int tg_learner_get_params(tg_learner* L, float* params /* [num_params] */);
int tg_learner_set_params(tg_learner* L, const float* params);
/* sample idx to host: *n cells, features [n*16], ELL columns / weights
 * [n*ell_width] (graph-local indices, -1 padding), target [n]; any output
 * may be NULL */
int tg_learner_get_sample(tg_learner* L, int32_t idx, int32_t* n, float* features, int32_t* ell_col, float* ell_w,
                          float* target);
/* loss, gradient [num_params] and outputs [cells] over samples
 * first..first+count-1 taken as one batch (no update) */
int tg_learner_gradients(tg_learner* L, int32_t first, int32_t count, float* loss, float* grads, float* outputs);
/* `steps` Adam steps on random batches of `batch` samples drawn from
 * first..first+count-1 (count <= 0: to the end); *mean_loss over the last
 * tenth of the steps */
int tg_learner_train(tg_learner* L, int32_t steps, int32_t batch, float lr, uint64_t seed, int32_t first,
                     int32_t count, float* mean_loss);

/* ---- measurement (no counterpart in the reference) ---------------------- */
/* CUDA events on the handle's stream around a region of calls. */
int tg_timer_start(tg_handle* h);
int tg_timer_stop(tg_handle* h, float* elapsed_ms);
/* Kernels launched in this process so far (every handle; the kernels of a
 * replayed CUDA graph count at each replay). */
int64_t tg_launch_count(const tg_handle* h);
/* How the multigrid solve's FP32 CG iterations reach the device: 1
 * replays one iteration (update, V-cycle, SpMV) captured as a CUDA
 * graph, whose kernels read the iteration index and target from device
 * memory (captured again when the hierarchy or the slots in use change),
 * the host reading rho back between batches of replays; 2 (the default)
 * replays it inside a device-side loop (a while-conditional graph node whose last
 * kernel stops it at the target or the iteration cap), one launch per
 * inner solve, its iteration count read with the solve's next residual;
 * 0 launches each kernel from the host.  All run the same kernels on the
 * same data; the node-space CG of the Neumann rows replays its iteration
 * in modes 1 and 2. */
int tg_set_launch_mode(tg_handle* h, int32_t mode);
/* Times `iters` back-to-back launches of one hot kernel on the handle's
 * stream with CUDA events: 0 = FP32 CG SpMV over the non-Neumann free rows,
 * 1 = FP64 residual over all free rows, 2 = the multigrid's level-0
 * smoothing pass t = b - A y (after a multigrid solve has built the
 * hierarchy).  Reports the mean duration of one
 * launch and the algorithmic bytes one launch moves (CSR rows, coupling and
 * neighbour-index streams, one compulsory read of every gathered vector
 * entry, the row outputs). */
int tg_bench_kernel(tg_handle* h, int32_t which, int32_t iters, float* avg_ms, double* algorithmic_bytes);
/* The tensor-core GEMM of the learned warm start on host arrays (a check
 * hook; no counterpart in the reference): C[M x N] (FP32) = A[M x K] *
 * B[N x K]^T with A, B BF16 bit patterns, row-major; M % 128 == 0,
 * N in {64, 128}, K % 64 == 0. */
int tg_gemm_bf16(const uint16_t* A, const uint16_t* B, float* C, int32_t M, int32_t N, int32_t K);
/* The multigrid hierarchy that tg_solve builds for preconditioner 1, built on
 * the host from a matrix the caller gives (a check hook; no counterpart in
 * the reference, no device work): row_ptr / col / val hold a symmetric
 * n x n M-matrix in CSR with its diagonal. */
typedef struct tg_amg_host tg_amg_host;
int tg_amg_host_build(int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val, tg_amg_host** out);
/* Levels, the finest (the matrix given) and the coarsest included. */
int32_t tg_amg_host_levels(const tg_amg_host* a);
/* One matrix of a level in CSR: which 0 = the level's operator A, 1 = its
 * prolongator P (rows x the next level's rows), 2 = its restriction R = P^T
 * (the coarsest level has only A).  Null arrays are skipped, so a first call
 * with rows / cols / nnz alone sizes the second. */
int tg_amg_host_matrix(const tg_amg_host* a, int32_t level, int32_t which, int32_t* rows, int32_t* cols, int64_t* nnz,
                       int32_t* ptr, int32_t* col, double* val);
void tg_amg_host_destroy(tg_amg_host* a);
/* Test hook, no counterpart in the reference: while on is non-zero, one
 * worker thread of every threaded pass of tg_amg_host_build (and of the
 * hierarchy tg_solve builds) throws std::bad_alloc, as an allocation failure
 * in that thread would.  The build must report TG_ERR_HOST, not terminate. */
void tg_amg_host_inject_worker_failure(int32_t on);

/* ---- host-side mesh building (setup, not device work) ------------------ */
typedef struct tg_mesh tg_mesh;
typedef struct {
    double lattice_a, cap_radius, shank_length, half_angle_deg;
    double box_half_width, box_height, fine_shell;
    int32_t layers_per_level;
    double coarsen, max_spacing;
    double solute_fraction, precip_density, precip_rmin, precip_rmax, precip_mu, precip_sigma;
    uint64_t seed;
} tg_tip_params;
void tg_tip_params_default(tg_tip_params* p);
/* bcc [110] tip + coarsened vacuum -> Delaunay -> FP64 Voronoi tables. */
int tg_mesh_from_tip(const tg_tip_params* p, int32_t threads, tg_mesh** out);
/* Node file + config (meshgen output / File_Io::readGeomGrid input). */
int tg_mesh_from_files(const char* node_file, const char* config_file, int32_t threads, tg_mesh** out);
/* MeshGen's role for an arbitrary sample (meshgen/meshgen.cpp:2506-3986,
 * replacing `meshgen sample out`): reads the sample node file (meshgen's
 * readSample input, :197-360: the node-file layout with ids), places graded
 * vacuum around it by the distance to its nearest atom (level 0 at the
 * sample's median nearest-neighbour spacing h0 out to fine_shell, no nearer
 * than exclusion * h0 to an atom; coarser levels by `coarsen` every
 * layers_per_level layers), the box faces z = 0 (bottom marker), z =
 * box_height (top) and |x|, |y| = box_half_width (sides, with every edge and
 * corner node, :3855-3892), appends the sample last (:3908) and builds the
 * Delaunay mesh and Voronoi couplings.  The sample must lie above z = 0 and
 * fit into the box with its fine shell.  config_file NULL takes meshgen's
 * configuration template (writeConfig, :491-595: top and sides Dirichlet
 * 0 V, bottom Neumann, sample ids removable Dirichlet 1000 V with mass and
 * evaporation field 0, which an evaporation run needs filled in);
 * tg_mesh_write_config writes it out.  threads <= 0: all host cores.
 * Deterministic in seed, whatever the thread count. */
typedef struct {
    double box_half_width, box_height, fine_shell, exclusion;
    int32_t layers_per_level;
    double coarsen, max_spacing;
    int32_t vacuum_id, top_id, bottom_id, sides_id;
    uint64_t seed;
} tg_sample_params;
void tg_sample_params_default(tg_sample_params* p);
int tg_mesh_from_sample(const char* sample_file, const char* config_file, const tg_sample_params* p, int32_t threads,
                        tg_mesh** out);
/* TAPSIM dump (File_Io::readSystem); keeps the dump's float couplings.
 * config_file may be NULL to use the dump's own table. */
int tg_mesh_from_dump(const char* dump_file, const char* config_file, tg_mesh** out);
void tg_mesh_destroy(tg_mesh* m);
/* Configuration::Table::temperature of the mesh's configuration [K] */
float tg_mesh_temperature(const tg_mesh* m);
/* Configuration::Table::operator[](name).id() (configuration.h): the id of
 * the cell type with that name in the mesh's configuration, -1 if none
 * (VACUUM_CELL_IDENTIFIER -> the vacuum id the event loop takes). */
int32_t tg_mesh_type_id(const tg_mesh* m, const char* name);
/* Fills a description whose pointers stay valid while the mesh lives. */
int tg_mesh_describe(const tg_mesh* m, tg_mesh_desc* desc, int32_t* nnz);
int tg_mesh_write_node_file(const tg_mesh* m, const char* path, int32_t binary);
/* File_Io::writeGeomGrid (file_io.cpp:765-820) with numbers and potentials:
 * the node file a relaxation leaves (tapsim.cpp:129-139), the potentials
 * given (NULL: the mesh's own) as floats. */
int tg_mesh_write_grid_nodes(const tg_mesh* m, const char* path, int32_t binary, const float* phi);
int tg_mesh_write_config(const tg_mesh* m, const char* path);
/* Writes a TAPSIM dump (File_Io::writeSystem layout) of the mesh with the
 * given potentials (NULL: the mesh's own). */
int tg_mesh_write_dump(const tg_mesh* m, const char* path, const float* phi);
/* The event index a dump holds (LAST_INDEX, File_Io::readSystem's index,
 * file_io.cpp:1027-1062) for a mesh read from one, else 0; a resumption
 * numbers its events on from it (tapsim.cpp:206-225), and
 * tg_mesh_write_dump writes it back. */
uint32_t tg_mesh_dump_index(const tg_mesh* m);
/* Grid_3d::Node::number of every node: the unique numbers of the node file
 * or dump (File_Io::readGeomGrid numbering, file_io.cpp:975-1000), index + 1
 * for a generated tip.  numbers_out: [N]. */
int tg_mesh_numbers(const tg_mesh* m, uint32_t* numbers_out);

/* ---- results and trajectory files: File_Io::LogResults / LogTrajectory -- */
/* One results row, LogResults::Dataset (logResults.h:41-66). */
typedef struct {
    uint32_t index;
    int32_t id;                 /* written as short */
    uint32_t number;
    float voltage;
    float start[3], stop[3];
    float tof;
    float probability;
    float potential_before, field_before[3];
    float potential_after, field_after[3];
    float normal[3], apex[3];
} tg_result_row;
/* Writes results files in LogResults' layout (logResults.cpp:135-381), ASCII
 * or binary.  With chunk_size > 0 the rows go to files path.%08u named after
 * the index of the row opening each chunk (a new chunk when index %
 * chunk_size == 0), the header text only in the first, as the reference's
 * writer thread does; otherwise to path.  header: extra header lines (may
 * be NULL). */
int tg_results_write(const char* path, int32_t binary, const char* header, int32_t count, const tg_result_row* rows,
                     int32_t chunk_size);
/* One trajectory, as LogTrajectory::push receives it
 * (logTrajectory.cpp:104-135): the points' times are written as given
 * (the caller multiplies by the time scale, as the writer thread does). */
typedef struct {
    uint32_t index;
    uint32_t number;
    float time_scale;
    int32_t status;             /* TG_TRAJ_* */
    float charge, mass;         /* [C], [kg] */
    int32_t num_points;
    const tg_path_point* points;
    float error[6];             /* error estimate: position x, y, z, velocity x, y, z */
} tg_trajectory_item;
/* Writes trajectory files in LogTrajectory's layout
 * (logTrajectory.cpp:137-300), chunked as tg_results_write with the header
 * in every file. */
int tg_trajectory_write(const char* path, int32_t binary, int32_t count, const tg_trajectory_item* items,
                        int32_t chunk_size);

/* ---- grid and surface snapshots: File_Io::LogGrid / LogSurface ---------- */
/* Writes one grid snapshot file in LogGrid's layout (logGrid.cpp:197-245):
 * for each of n cells the type id, unique number, potential, field [3] and
 * force [3]. */
int tg_grid_log_write(const char* path, int32_t binary, int32_t n, const int32_t* id, const uint32_t* number,
                      const float* phi, const float* field, const float* force);
/* Writes one surface snapshot file in LogSurface's layout
 * (logSurface.cpp:203-293): n_cells surface cells (ascending) with type,
 * unique number, probability and, when neighbour_ptr is not NULL, their
 * neighbour lists neighbours[neighbour_ptr[c] .. neighbour_ptr[c+1]); then
 * n_nodes cells (ascending) with potential, field [3] and normal [3]. */
int tg_surface_log_write(const char* path, int32_t binary, int32_t n_cells, const int32_t* cells, const int32_t* type,
                         const uint32_t* number, const float* probability, const int32_t* neighbour_ptr,
                         const int32_t* neighbours, int32_t n_nodes, const int32_t* nodes, const float* phi,
                         const float* field, const float* normal);

#ifdef __cplusplus
}
#endif

#endif /* TAPSIM_GPU_H */
