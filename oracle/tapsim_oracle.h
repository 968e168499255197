/* CPU restatement of TAPSim's per-event hot path in FP64 (test oracle).
 *
 * This is test infrastructure: only tests/, __graft_entry__.smoke() and the
 * CPU leg of bench.py load it, and only as the checker.  Each function cites
 * the reference routine it restates (paths inside the reference tree).
 * Arrays follow the layout of tg_mesh_desc (include/tapsim_gpu.h).
 */
#ifndef TAPSIM_ORACLE_H
#define TAPSIM_ORACLE_H

#include <stdint.h>

typedef struct {
    int32_t present, removable, neumann, dirichlet;
    double epsilon, evap_field, charge_density, phi, mass;
    int32_t evap_charge;
    double evap_energy;        /* [eV] */
} orc_type;

typedef struct {
    int32_t n;
    const float* xyz;          /* [3n] */
    int8_t* type;              /* [n], mutable */
    const uint8_t* hull;       /* [n] */
    const int32_t* row_ptr;    /* [n+1] */
    const int32_t* col;        /* [nnz] */
    double* c;                 /* [nnz] coupling, mutable */
    const double* geom;        /* [nnz] area(0.5d)/d */
    const uint8_t* area_pos;   /* [nnz] */
    double* phi;               /* [n] mutable */
    double* q;                 /* [n] mutable (charge term) */
    const double* volume;      /* [n] or NULL */
    int32_t ntets;
    const int32_t* tet_v;      /* [4T] */
    const int32_t* tet_n;      /* [4T] */
    const orc_type* types;     /* [128] by id */
    uint8_t* surface;          /* [n] surface flag, mutable */
} orc_mesh;

/* relative residual ||r||/||b|| (r over free rows, computePotential rule) */
double orc_residual(const orc_mesh* m);
/* SOR sweeps in ascending node order until the relative residual is <= tol;
 * returns sweeps done, -1 on the cap.  omega = 1 is Gauss-Seidel. */
int64_t orc_solve(orc_mesh* m, double tol, int64_t max_sweeps, double omega, double* rel_out);
/* n reference-style sweeps (Gauss-Seidel, ascending order); returns max |delta| of the last */
double orc_relax_cycles(orc_mesh* m, int32_t n);
/* find_localNodes (grid_3d.cpp:1284-1315) minus the Dirichlet cells, as
 * localRelax forms its set (:707-721), ascending; returns the count */
int32_t orc_local_set(const orc_mesh* m, int32_t node, int32_t shell, int32_t* out, int32_t cap);
/* the fixed point of localRelax on a cell list (every other cell held):
 * Gauss-Seidel until a sweep moves no potential by more than tol; returns
 * the sweeps, -1 on the cap */
int64_t orc_local_solve(orc_mesh* m, const int32_t* cells, int32_t count, double tol, int64_t max_sweeps);
/* the stagnation rule of relax(thr, cycle, queue) (grid_3d.cpp:625-654) on
 * the last `queue` of `count` deviations: 1 for a zero slope */
int32_t orc_stagnated(const double* dev, int32_t count, int32_t queue, int32_t cycle);
/* Grid_3d::Table::field_o1; returns 0 when the 3x3 system is singular */
int orc_field_o1(const orc_mesh* m, int32_t i, double E[3]);
/* Grid_3d::Table::force (grid_3d.cpp:1201-1236) */
void orc_force(const orc_mesh* m, int32_t i, double F[3]);
/* Surface_3d::Table::init; returns the number of surface cells */
int32_t orc_surface_init(orc_mesh* m, int32_t vacuum_id);
/* specific fields + probabilities + evapMaximum + apex over the surface set */
typedef struct {
    int32_t candidate, apex, num_surface;
    float best, second;
    double sum;
} orc_select_info;
void orc_select(const orc_mesh* m, float* ratio_out /* [n] or NULL */, orc_select_info* info);
/* Grid_3d::Table::field_o2 (grid_3d.cpp:993-1199): second-order fit over all
 * neighbours; field and charge (0 on hull cells); returns 0 when singular */
int orc_field_o2(const orc_mesh* m, int32_t i, double E[3], double* charge);
/* score of one surface cell before normalisation (surface_3d.cpp:222-399):
 * mode 0 |E|/E_evap, 1 Boltzmann, 2 linear force (field_o2), 3 Voronoi flux
 * force; temperature [K] for mode 1 */
double orc_score(const orc_mesh* m, int32_t i, int32_t mode, double temperature);
/* evap_compute_probabilities + evapMaximum over the surface set in
 * ascending order: score_out[i] = score (float), info->candidate = first
 * maximum of score / sum, best / second = the two largest normalised
 * probabilities, sum = the score sum */
void orc_select_mode(const orc_mesh* m, int32_t mode, double temperature, float* score_out, orc_select_info* info);
/* evapMonteCarlo (surface_3d.cpp:433-449): the first surface cell (ascending)
 * whose cumulative probability score/sum reaches u; the last one if none */
int32_t orc_pick(const orc_mesh* m, const float* score, double sum, double u);
/* evap_takeAway; returns the number of detached cells (written to detached) */
int32_t orc_take_away(orc_mesh* m, int32_t node, int32_t vacuum_id, int32_t* detached, int32_t cap);
/* update_coordination */
void orc_update_coordination(orc_mesh* m);
/* one ion: Trajectory_3d init/integrate/extrapolate in FP64 */
typedef struct {
    double stop[3];
    double stop_time;
    double last_pos[3];
    int32_t last_tet;
    double last_phi;
    int32_t steps;
    int32_t status;
} orc_impact;
void orc_trace(const orc_mesh* m, const double start[3], double qm, int32_t tet_guess, double dt0, double dt_min,
               double tol, int32_t max_steps, int32_t stepper_limit, double top_z, orc_impact* out);
/* the same with an initial velocity, TRAJECTORY_INTEGRATOR_TYPE (0 Euler,
 * 1 Cash-Karp) and TRAJECTORY_STEPPER_TYPE (0 none, 1 error-restricted,
 * 2 geometry-restricted, 3 adaptive) */
void orc_trace_ext(const orc_mesh* m, const double start[3], const double vel[3], double qm, int32_t tet_guess,
                   double dt0, double dt_min, double tol, int32_t max_steps, int32_t stepper_limit, double top_z,
                   int32_t integrator, int32_t stepper, orc_impact* out);
/* orc_trace_ext keeping the path as Trajectory_3d::data() holds it (start,
 * each accepted step, the extrapolated point; at most cap points of 8
 * doubles: time, position, velocity, tetrahedron) and the cumulative error
 * estimate err[6] (position, velocity) */
void orc_trace_path(const orc_mesh* m, const double start[3], const double vel[3], double qm, int32_t tet_guess,
                    double dt0, double dt_min, double tol, int32_t max_steps, int32_t stepper_limit, double top_z,
                    int32_t integrator, int32_t stepper, orc_impact* out, int32_t cap, double* path, double* err);
/* Grid_3d::potential(pos, tet) */
double orc_potential_at(const orc_mesh* m, const double p[3], int32_t tet_guess);

#endif
