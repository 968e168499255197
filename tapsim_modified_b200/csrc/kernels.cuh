// Device data layout and host-side launchers of the hot-path kernels.
//
// HBM layout (one copy per handle, node-file order, CSR rows ascending):
//   per node   xyz float[3], type int8, flags uint8, phi64 double, diag64
//              double, diag32 float, q64 double, colour int32
//   per entry  col int32, rev int32, c64 double (the Grid_3d coupling),
//              ceff64 double / ceff32 float (coupling as the row's update
//              sees it: 0 for a Neumann neighbour of a non-Neumann row),
//              geom double (Voronoi area / distance), area_pos uint8
//   free rows  int32 lists grouped by colour, non-Neumann and Neumann apart
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"

namespace tgd {

// process-wide count of kernels launched by this library (handle.cu)
void count_launch();
long long launches_so_far();

struct DevMesh {
    int n, nnz, ntets;
    const float* xyz;
    int8_t* type;
    uint8_t* flags;
    const int32_t* row_ptr;
    const int32_t* col;
    const int32_t* rev;
    const double* geom;
    const uint8_t* area_pos;
    const double* volume;
    double* c64;
    const uint8_t* cnz;           // [nnz] 1 where c64 != 0 (a flip never changes it)
    double* ceff64;
    float* ceff32;
    double* diag64;
    float* diag32;
    double* q64;
    double* phi64;
    const int32_t* colour;
    const int32_t* tet_v;
    const int32_t* tet_n;
    const int32_t* node_tet;
    const DType* types;
    int* status;
    double snap;   // power-of-two scale to the integer grid of the exact predicates
    double* vfield;    // [3n] vertex fields of the current flight call
    double* phiTrace;  // [n] potentials of the current flight call
    const float* tetpack;  // [32 ntets] packed tetrahedra (flight.cu)
};

// Free-row bookkeeping kept on the device so that removals can append rows
// without a host round trip.
struct RowLists {
    int32_t* rowsV;        // non-Neumann free rows, colour segments
    int32_t* rowsN;        // Neumann free rows, colour segments
    const int32_t* segStart;  // [ncolours] segment start (same for V and N)
    int32_t* countV;       // [ncolours] rows in use
    int32_t* countN;
    int32_t* allV;         // the same rows as one compact list each
    int32_t* allN;
    int32_t* countAll;     // [2]: rows in allV, allN
    int ncolours;
};

struct Surface {
    int32_t* list;         // surface node per slot, -1 for a removed entry
    int32_t* slot;         // [n] list slot of a surface node
    int32_t* count;        // slots in use (device counter)
    float* ratio;          // per slot |E|/E_evap of the last selection
    float* score;          // per slot score of the probability mode (before normalisation)
    int capacity;
};

// Non-Neumann free rows in their own slot order, couplings in SELL-32
// (cg.cu).  Vectors hold capacity+1 entries; entry `capacity` is the zero
// slot that entries of non-free neighbours point at.
// damped-Jacobi weight of the multigrid's smoothing steps (amg.cu)
constexpr float kAmgSmooth = 0.9f;

struct VSys {
    int32_t* slot_of;             // [n] node -> slot, -1
    int32_t* node_of;             // [capacity] slot -> node, -1 for padding
    const int32_t* slice_start;   // [slices] first storage index of a slice
    const int32_t* slice_width;   // [slices] entries per row in the slice
    int32_t* col;                 // slot of the neighbour (or the zero slot)
    float* val;                   // coupling as the row sees it
    __nv_bfloat16* val16;         // the same rounded to bf16, for the multigrid's smoothing pass
    float* g;                     // [capacity + 1] row sum: d minus the row's stored val
    int32_t* vpos;                // [nnz] global CSR entry -> storage index, -1
    float *d, *x, *r, *u, *w, *p, *sv;
    float* hist;                  // correction of the last event's solve (warm start)
    double* scal;                 // gamma, delta, alpha per iteration
    int32_t* count;               // next free slot (device counter)
    int capacity;
    // FP64 inner iterations (tg_solve_opts.inner_precision 1), allocated at
    // the first solve that asks for them, null before: the couplings and the
    // diagonal in FP64 at the same positions as val and d (kept in step by
    // every write of those once allocated), and the CG vectors in FP64
    double* val64;
    double *d64, *x64, *r64, *p64, *s64, *w64;
    // CG iterations replayed from a CUDA graph: the iteration index counts
    // from the device counter *iter and the relative target is *rel2 (both
    // null when the host launches each iteration with its own values)
    const int32_t* iter;
    const double* rel2;
};
// Early exit of the kernels of CG iteration `it` (cg.cu, amg.cu): they do
// nothing once rho_it <= rel2 * rho_0 (rel2 < 0: never), so that
// iterations queue before the host has seen rho_0.  With itBase the index
// is it + *itBase, and with rel2Dev the target is *rel2Dev (an iteration
// replayed from a CUDA graph).
struct Gate {
    const double* scal;
    int it;
    double rel2;
    const int32_t* itBase;
    const double* rel2Dev;
    __device__ __forceinline__ int iter() const { return itBase ? it + *itBase : it; }
    __device__ __forceinline__ bool done() const {
        const double t = rel2Dev ? *rel2Dev : rel2;
        return t >= 0.0 && scal[4 * iter() + 3] <= t * scal[3];
    }
};
inline Gate make_gate(const VSys& v, int it, double rel2) { return Gate{v.scal, it, rel2, v.iter, v.rel2}; }
// a gate that never closes (timing and setup launches)
inline Gate open_gate() { return Gate{nullptr, 0, -1.0, nullptr, nullptr}; }
// jacobi: the Jacobi preconditioner (u = r / d inside init / update);
// otherwise u comes from launch_amg_vcycle and the SpMV adds gamma = r.u.
// `target` of the iteration kernels (and of the V-cycle) is relative: they
// do nothing once rho_it <= target * rho_0; a negative target never skips
void launch_vcg_init(const VSys& v, int slots, bool jacobi, cudaStream_t s);
void launch_vcg_spmv(const VSys& v, int slots, int it, double target, bool withGamma, cudaStream_t s);
// smoothY (multigrid preconditioner): also the V-cycle's first step,
// smoothY = kAmgSmooth r / d, so that the cycle that follows skips it
void launch_vcg_update(const VSys& v, int slots, int it, double target, bool jacobi, cudaStream_t s,
                       float* smoothY = nullptr);
// the counter, target and cap of iterations replayed from a CUDA graph:
// set to 0, rel2 and maxIter before the first replay, stepped by 1 at the
// end of each
void launch_vcg_replay_begin(int32_t* iter, double* rel2Dev, double rel2, int maxIter, cudaStream_t s);
// the condition kernel of the device-side loop around the replayed
// iteration (the last node of the loop's body): steps *iter, then sets the
// loop's condition; *done: the iterations run
void launch_vcg_loop_cond(cudaGraphConditionalHandle loop, int32_t* iter, const double* scal,
                          const double* rel2Dev, int32_t* done, cudaStream_t s);
void launch_vcg_replay_step(int32_t* iter, cudaStream_t s);
// FP64 inner iterations with the multigrid preconditioner: the V-cycle runs
// in FP32 on r rounded to float and its u enters the FP64 recurrences
// exactly.  init64 takes the right-hand side from the FP64 residual by node
// (the kept residuals of the first pass); apply64 adds x64 to the potentials.
void launch_vcg64_derive(const DevMesh& m, const VSys& v, int nnz, cudaStream_t s);
void launch_vcg64_init(const VSys& v, int slots, const double* rnode, cudaStream_t s);
void launch_vcg64_spmv(const VSys& v, int slots, int it, double target, cudaStream_t s);
void launch_vcg64_update(const VSys& v, int slots, int it, double target, cudaStream_t s);
void launch_vcg64_apply(const DevMesh& m, const VSys& v, int slots, bool record, cudaStream_t s);

// ---- multigrid preconditioner (amg.cu) ----
constexpr int kAmgMaxLevels = 12;
struct AmgDevLevel {
    int n;                                  // rows (level 0: slots covered by its prolongator)
    const int32_t *a_ptr, *a_col;           // operator, levels >= 1 (CSR with diagonal)
    const float *a_val, *diag;
    const int32_t *p_ptr, *p_col;           // prolongator: n rows
    const float* p_val;
    const int32_t *r_ptr, *r_col;           // restriction: the next level's rows
    const float* r_val;
    float *b, *y, *x, *t;                   // right-hand side, work, result, residual (levels >= 1)
    int a_lanes, r_lanes;                   // lanes per row of the operator and of the restriction (2..32)
};
constexpr int kFinePipe = 1000;             // AmgDev::fine_unroll offset of the pipelined level-0 pass
struct AmgDev {
    int levels;                             // including level 0 (the V system) and the coarsest
    AmgDevLevel lev[kAmgMaxLevels];
    float *y0, *t0;                         // level-0 work vectors (capacity + 1)
    const float* coarse_inv;                // dense inverse of the coarsest operator, row-major
    int fine_unroll;                        // level-0 pass: loads per lane ahead of their gathers (4, 8, 16),
                                            // plus kFinePipe for the software-pipelined kernel (4, 8)
};
// Autotuner of the hierarchy's schedules: the level-0 pass's loads per
// lane (4, 8, 16, or the pipelined kernel with 4 or 8; fine_unroll), and
// for the restriction of every level and
// the operator of every level smoothed by CSR rows the lane-group size
// (2..32 lanes per row; r_lanes / a_lanes), chosen one at a time from the
// row-length rule's schedule by timing whole V-cycles (the least of three
// batches of three, CUDA events on s), a change kept when it takes 3% off.
// aMs / rMs (kAmgMaxLevels entries) and fineMs (may be null) receive the
// kept kernels' own times [ms].  Returns 0, or -1 on a CUDA error.
int amg_tune_lanes(AmgDev& g, const VSys& v, int slots, cudaStream_t s, float* aMs, float* rMs, float* fineMs);
// the level-0 smoothing pass t = b - A y alone (timing hook)
void launch_amg_fine_residual(const VSys& v, int slots, const AmgDev& g, cudaStream_t s);
// u = M^-1 r, one V(1,1)-cycle, for CG iteration `it`
// y0Ready: g.y0 already holds kAmgSmooth r / d (written by the CG update)
void launch_amg_vcycle(const VSys& v, int slots, const AmgDev& g, int it, double target, cudaStream_t s,
                       bool y0Ready = false);
// phi64 += x on the V rows; with record, hist += x as well
void launch_vcg_apply(const DevMesh& m, const VSys& v, int slots, bool record, cudaStream_t s);
// warm start: hist *= alpha, phi64 += hist on the V rows
void launch_vcg_warm(const DevMesh& m, const VSys& v, int slots, float alpha, cudaStream_t s);
// r -= A hist on the V system (FP32), sum r^2 into *acc
// sum of r^2 over the V slots into *acc (the FP32 right-hand side as it is)
void launch_vcg_rnorm(const VSys& v, int slots, double* acc, cudaStream_t s);
void launch_vcg_warm_residual(const VSys& v, int slots, double* acc, cudaStream_t s);
void launch_vcg_couple_neumann(const DevMesh& m, const VSys& v, const int32_t* rows, int count, float* rN,
                               cudaStream_t s, bool fromX64 = false);
// FP64 residual of the V rows (rows: their compact list, in node order)
// into the V system's r; with bacc, also ||b||^2 of those rows.  With r64
// (by node) each row's FP64 residual is kept, and with bacc and b64 its
// Dirichlet part
void launch_vcg_residual(const DevMesh& m, const VSys& v, const int32_t* rows, int count, double* acc, double* bacc,
                         cudaStream_t s, double* r64 = nullptr, double* b64 = nullptr);
// the residuals of the flipped cells and their neighbours after removals,
// from the values the last full passes kept in r64 / b64: rsum[0..2] (the V
// rows' r^2, the Neumann rows' r^2, ||b||^2) take the differences, the V
// system's r and rN the new values.  stamp (by node) holds a value other
// than epoch for every row
void launch_residual_rows(const DevMesh& m, const VSys& v, float* rN, const int32_t* flips, int count, int32_t* stamp,
                          int epoch, double* r64, double* b64, double* rsum, cudaStream_t s,
                          const int32_t* countDev = nullptr);
void launch_vsys_add_rows(const DevMesh& m, const VSys& v, const int32_t* nodes, int count, cudaStream_t s);
// re-copies the couplings and diagonals that flips of the listed cells
// changed into the V system (rows that existed before the flips)
void launch_vsys_refresh(const DevMesh& m, const VSys& v, const int32_t* nodes, int count, cudaStream_t s);
// val16 and g of every slot from val and d (after the upload)
void launch_vsys_derive(const VSys& v, size_t stored, cudaStream_t s);

// ---- relaxation (relax.cu) ----
// coloured Gauss-Seidel sweep of one row list, FP64, max |delta| to *maxdev
void launch_sweep64(const DevMesh& m, const int32_t* rows, int count, double* maxdev, cudaStream_t s);
// r_i (FP64) for a row list; accumulates sum r^2 into *acc; optionally
// stores r as float into r32
// with bacc, also the squared norm of the rows' Dirichlet part (as
// launch_bnorm) into *bacc
// slotOf (may be null): r32 is indexed by slotOf[i] instead of i
void launch_residual(const DevMesh& m, const int32_t* rows, int count, float* r32, double* acc, cudaStream_t s,
                     double* bacc = nullptr, double* r64 = nullptr, double* b64 = nullptr,
                     const int32_t* slotOf = nullptr);
// b_i = sum over Dirichlet neighbours c_ij phi_j - q_i; sum b^2 into *acc
void launch_bnorm(const DevMesh& m, const int32_t* rows, int count, double* acc, cudaStream_t s);
// FP32 conjugate gradients on the rows of one list (Jacobi preconditioner)
struct CGVectors {
    float *x, *r, *z, *p, *ap;
    double* scal;  // [3*(max_iter+2)] accumulators: rz, pAp per iteration
    // iterations replayed from a CUDA graph: the index counts from the
    // device counter *iter and the targets (rel2, abs2) are tgt[0], tgt[1]
    // (both null when the host launches each iteration with its own values)
    const int32_t* iter;
    const double* tgt;
};
void launch_cg_init(const DevMesh& m, const int32_t* rows, int count, CGVectors v, cudaStream_t s);
// the counter and targets of node-space CG iterations replayed from a CUDA
// graph: set to 0, rel2 and abs2 before the first replay; the step adds 1
void launch_cg_replay_begin(int32_t* iter, double* tgt, double rel2, double abs2, cudaStream_t s);
void launch_cg_replay_step(int32_t* iter, cudaStream_t s);
// one CG iteration; all of it is skipped once r.r (scal[3it+2]) <=
// max(rel2 * r.r at the start (scal[2]), abs2)
void launch_cg_iter(const DevMesh& m, const int32_t* rows, int count, CGVectors v, int it, double rel2, double abs2,
                    cudaStream_t s);
// the SpMV kernel of one CG iteration on its own (timing hook)
void launch_cg_spmv_only(const DevMesh& m, const int32_t* rows, int count, CGVectors v, cudaStream_t s);
// rhs_N += sum over non-Neumann free neighbours c_ij x_j (coupling of the
// Neumann rows to the correction found for the non-Neumann rows)
void launch_add_coupled(const DevMesh& m, const int32_t* rows, int count, const float* xV, float* r, cudaStream_t s);
// phi64[i] += x[i] for a row list, and clears the CG vectors on those rows
void launch_apply_correction(const DevMesh& m, const int32_t* rows, int count, CGVectors v, cudaStream_t s);
// coupling rows: diag64/diag32/ceff from c64 and the flags of all nodes
void launch_rebuild_rows(const DevMesh& m, cudaStream_t s);
// k-hop node set (find_localNodes) restricted to non-Dirichlet cells; writes
// rows grouped by colour into out (capacity cap) and per-colour counts
void launch_local_set(const DevMesh& m, int node, int hops, int32_t* out, int32_t* outCount, int cap,
                      int32_t* scratch, int scratchCap, int ncolours, cudaStream_t s);

// ---- surface (surface.cu) ----
void launch_surface_init(const DevMesh& m, Surface sf, int vacuumId, cudaStream_t s);
// fields, ratios and scores of probability mode `mode` (0 linear field,
// 1 Boltzmann at `temperature`, 2 linear force, 3 Voronoi flux force);
// keys[0] max ratio, keys[1] apex, keys[2] min / keys[3] max surface node;
// acc[0] sum of ratios, acc[1] sum of scores
void launch_surface_select(const DevMesh& m, Surface sf, int slots, int mode, float temperature,
                           unsigned long long* keys, double* acc, cudaStream_t s);
// keys[4] candidate (first maximum of score / sum, sum = acc[1]), then
// keys[5] runner-up probability (excluding the candidate) and keys[6]
// runner-up ratio (excluding the best-ratio node of keys[0]); both read what
// they need from device memory, so the selection needs one read at its end
void launch_surface_best(Surface sf, int slots, const double* acc, unsigned long long* keys, cudaStream_t s);
void launch_surface_second(Surface sf, int slots, const double* acc, unsigned long long* keys, cudaStream_t s);
void launch_surface_prefix(Surface sf, int slots, float sum, int upTo, double* acc, cudaStream_t s);
void launch_field_o1(const DevMesh& m, const int32_t* nodes, int count, double* out, cudaStream_t s);
// evap_takeAway in one small kernel; result[0] = number of detached nodes,
// result[1..] their indices
void launch_take_away(const DevMesh& m, RowLists rl, Surface sf, int node, int vacuumId, int32_t* result,
                      int resultCap, cudaStream_t s);
void launch_update_coordination(const DevMesh& m, int8_t* scratchType, cudaStream_t s);
void launch_surface_normal(const DevMesh& m, Surface sf, int node, int vacuumId, float* out, cudaStream_t s);
// the normals of a list of cells, one block each
void launch_surface_normals(const DevMesh& m, const int32_t* nodes, int count, int vacuumId, float* out,
                            cudaStream_t s);
// potential, field_o1 and Grid_3d force (float) of a list of cells, or of
// every cell when nodes is null; outputs may be null
void launch_cell_values(const DevMesh& m, const int32_t* nodes, int count, float* phi, float* field, float* force,
                        cudaStream_t s);

// ---- flights (flight.cu) ----
struct TraceParams {
    double dt0, dt_min, tol;
    int max_steps, stepper_limit, walk_limit;
    float top_z;
    int integrator;  // 0 Euler, 1 Cash-Karp (TRAJECTORY_INTEGRATOR_TYPE)
    int stepper;     // 0 none, 1 error-restricted, 2 geometry-restricted, 3 adaptive
    // optional path recording (null path: none): ion k keeps up to path_cap
    // points of 8 words (time, position, velocity, tetrahedron bits) at
    // path + k * path_cap * 8, and 12 words at path_err + 12k: its
    // cumulative error estimate (position, velocity), then the latest trial
    // step's error
    float* path;
    float* path_err;
    int path_cap;
    // arithmetic of the Cash-Karp steps: 0 FP64, 1 FP32 (as the reference),
    // 2 FP64 within sqrt(fp64_radius2) of the start and FP32 beyond
    int precision;
    double fp64_radius2;
};
struct ImpactOut {
    float stop[3];
    float stop_time;
    float last_pos[3];
    int32_t last_tet;
    float last_phi;
    int32_t steps;
    int32_t status;
    int32_t trials;  // integrator trial steps, accepted and rejected
};
// packed tetrahedron records (32 words each) from tet_v, tet_n and xyz
void launch_pack_tets(const DevMesh& m, float* pack, cudaStream_t s);
// field_o1 of every node from the current potentials into m.vfield
// vertex fields (field_o1 of every cell) into m.vfield; with cells, only the
// listed cells (the others keep their values)
void launch_vertex_fields(const DevMesh& m, cudaStream_t s, const int32_t* cells = nullptr, int count = 0);
void launch_trace(const DevMesh& m, int nIons, const float* start, const float* vel, const float* qm,
                  const int32_t* guess, TraceParams tp, ImpactOut* out, cudaStream_t s);
// one ion from rest at start (values passed to the kernel)
void launch_trace_one(const DevMesh& m, const float start[3], const float vel[3], float qm, int guess, TraceParams tp,
                      ImpactOut* out, cudaStream_t s);
void launch_potential_at(const DevMesh& m, int n, const float* xyz, const int32_t* guess, int walkLimit,
                         float* out, cudaStream_t s);

// ---- learned warm start (mpnn.cu) ----
// C[M x N] (FP32) = A[M x K] * B[N x K]^T, A and B BF16 row-major, on the
// tensor cores; M % 128 == 0, N in {64, 128}, K % 64 == 0
bool gemm_shape_ok(int M, int N, int K);
cudaError_t launch_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int* status,
                             cudaStream_t s);
void launch_ball_bfs(const DevMesh& m, int site, int hops, int cap, int32_t* nodes, int8_t* level, int32_t* count,
                     int32_t* localOf, cudaStream_t s);
void launch_ball_reset(const int32_t* nodes, const int32_t* count, int32_t* localOf, int cap, cudaStream_t s);
void launch_ball_features(const DevMesh& m, int site, int hops, int D, const int32_t* nodes, const int8_t* level,
                          const int32_t* count, const int32_t* localOf, float* scale, float* X, int32_t* ellCol,
                          float* ellW, double* phiStart, int cap, cudaStream_t s);
// nDev (may be null): a device-side row count that caps n
void launch_input_bf16(const float* X, int n, int npad, void* Z, void* ZT, cudaStream_t s,
                       const int32_t* nDev = nullptr);
void launch_bias_act(const float* C, const float* b, const float* hPrev, float* u, float* h, int npad, cudaStream_t s);
void launch_message_concat(const float* h, const int32_t* ellCol, const float* ellW, int D, int n, int npad, void* Z,
                           void* ZT, cudaStream_t s, const int32_t* nDev = nullptr);
void launch_readout(const float* h, const float* w, const float* b, int n, float* y, cudaStream_t s,
                    const int32_t* nDev = nullptr);
void launch_loss(const float* y, const float* tgt, int n, float invCount, float* dy, float* loss, cudaStream_t s);
void launch_readout_back(const float* h, const float* dy, const float* w, int n, int npad, float* gw, float* gb,
                         float* dh, cudaStream_t s);
void launch_act_back(const float* dh, const float* u, int npad, void* DU, void* DUT, float* gb, cudaStream_t s);
void launch_message_back(const float* dh, const float* dz, const int32_t* ellCol, const float* ellW, int D, int n,
                         int npad, float* dhPrev, cudaStream_t s);
void launch_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2, float eps,
                 float c1, float c2, cudaStream_t s);
void launch_weights_bf16(const float* W, void* Wb, void* WTb, cudaStream_t s);
// damped Jacobi sweeps on the graph's cells (at most 4096), the rest held;
// the change joins hist (V slots) when given
void launch_local_refine(const DevMesh& m, const int32_t* nodes, const int32_t* count, int cap, int sweeps,
                         float omega, const int32_t* slotOf, float* hist, cudaStream_t s);
void launch_apply_prediction(const DevMesh& m, const int32_t* nodes, const int32_t* count, const float* y,
                             const float* scale, float gain, const int32_t* slotOf, float* hist, int cap,
                             cudaStream_t s);
void launch_collect_target(const DevMesh& m, const int32_t* nodes, const int32_t* count, const double* phiStart,
                           const float* scale, float* tgt, int cap, cudaStream_t s);
void launch_shift_cols(int32_t* col, int count, int shift, cudaStream_t s);

}  // namespace tgd
