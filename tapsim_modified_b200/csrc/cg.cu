// FP32 conjugate gradients on the non-Neumann free rows ("V system"), the
// inner solver of the FP64 defect-correction solve.
//
// Layout.  The V rows get their own dense slot numbering.  Couplings are
// stored SELL-32: slices of 32 consecutive slots, column-major inside a
// slice, each slice as wide as its longest row, rows sorted by length
// within windows of 1024 slots so that slices are nearly full.  One warp
// handles one slice and every coupling load is a coalesced 128-byte line.
// A row keeps an entry for every neighbour that is free or may become free
// (removable Dirichlet atoms); entries of non-free neighbours point at the
// zero slot, whose vector entries stay 0.  A removal therefore never changes
// the structure: it appends the new row in a reserve of fixed-width slices
// and repoints the neighbours' entries (vpos maps a global CSR entry to its
// SELL position).
//
// Iteration.  Chronopoulos-Gear single-reduction PCG with the Jacobi
// preconditioner: one pointwise kernel (p, s, x, r, u updates and r.u) and
// one SpMV kernel (w = A u and w.u) per iteration; alpha and beta are
// computed by every thread from the per-iteration scalars.
#include "kernels.cuh"

namespace tgd {
namespace {

constexpr int kBlock = 256;

// per iteration i: gamma_i = r.u, delta_i = w.u, alpha_i and rho_i = r.r at
// scal[4i .. 4i+3].  A kernel of iteration it does nothing once rho_it <=
// rel2 * rho_0 (rel2 < 0: never), so that iterations can be queued before
// the host has seen rho_0.
__device__ __forceinline__ bool cg_done(const double* scal, int it, double rel2) {
    return rel2 >= 0.0 && scal[4 * it + 3] <= rel2 * scal[3];
}

__device__ __forceinline__ void cg_coeffs(const double* scal, int it, double* alpha, double* beta) {
    const double g = scal[4 * it], d = scal[4 * it + 1];
    if (it == 0) {
        *beta = 0.0;
        *alpha = d > 0.0 ? g / d : 0.0;
    } else {
        const double gp = scal[4 * (it - 1)], ap = scal[4 * (it - 1) + 2];
        *beta = gp > 0.0 ? g / gp : 0.0;
        const double den = d - *beta * g / ap;
        *alpha = den > 0.0 ? g / den : 0.0;
    }
}

// x = 0, rho_0 = r.r; with the Jacobi preconditioner also u = r / d and
// gamma_0 = r.u (with the multigrid one the V-cycle makes u and the SpMV
// gamma)
__global__ void k_vcg_init(VSys v, int slots, int jacobi) {
    double g = 0.0, rr = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        const float r = v.r[s];
        if (jacobi) {
            const float u = r / v.d[s];
            v.u[s] = u;
            g += (double)r * (double)u;
        }
        v.x[s] = 0.0f;
        v.p[s] = 0.0f;
        v.sv[s] = 0.0f;
        rr += (double)r * (double)r;
    }
    block_sum2_atomic<kBlock>(g, rr, &v.scal[0], &v.scal[3]);
}

// w = A u over SELL-32 slices; delta -> scal[4*it+1] (it = iteration whose
// u this is), and with withGamma gamma = r.u -> scal[4*it]; skipped once
// iteration it has converged (cg_done)
__global__ void k_vcg_spmv(VSys v, int slices, Gate gate, int withGamma) {
    if (gate.done()) return;
    const int it = gate.iter();
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    double dl = 0.0, gl = 0.0;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < slices; warp += warps) {
        const int base = v.slice_start[warp];
        const int width = v.slice_width[warp];
        const int s = warp * 32 + lane;
        const int* __restrict__ col = v.col + base + lane;
        const float* __restrict__ val = v.val + base + lane;
        const float* __restrict__ uu = v.u;
        float acc = 0.0f;
        // eight independent column/value loads ahead of their gathers keep
        // enough bytes in flight per warp; the matrix is streamed once per
        // iteration (evict-first), the gathered vector stays cached
        int k = 0;
        for (; k + 8 <= width; k += 8) {
            int c[8];
            float a[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                c[j] = __ldcs(col + 32 * (k + j));
                a[j] = __ldcs(val + 32 * (k + j));
            }
#pragma unroll
            for (int j = 0; j < 8; j++) acc += a[j] * __ldg(uu + c[j]);
        }
        for (; k < width; k++) acc += __ldcs(val + 32 * k) * __ldg(uu + __ldcs(col + 32 * k));
        const float u = v.u[s];
        const float w = v.d[s] * u - acc;
        v.w[s] = w;
        dl += (double)w * (double)u;
        if (withGamma) gl += (double)v.r[s] * (double)u;
    }
    const int at = 4 * it;
    if (withGamma) block_sum2_atomic<kBlock>(dl, gl, &v.scal[at + 1], &v.scal[at]);
    else block_sum_atomic<kBlock>(dl, &v.scal[at + 1]);
}

// p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s,
// rho_{it+1} = r.r; with the Jacobi preconditioner also u = r / d and
// gamma_{it+1} = r.u; with smoothY (the multigrid one) the V-cycle's first
// step smoothY = w r / d, one launch fewer per iteration
__global__ void k_vcg_update(VSys v, int slots, Gate gate, int jacobi, float* smoothY) {
    if (gate.done()) return;
    const int it = gate.iter();
    double alpha, beta;
    cg_coeffs(v.scal, it, &alpha, &beta);
    if (blockIdx.x == 0 && threadIdx.x == 0) v.scal[4 * it + 2] = alpha;
    const float a = (float)alpha, b = (float)beta;
    double g = 0.0, rr = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        const float p = v.u[s] + b * v.p[s];
        const float sv = v.w[s] + b * v.sv[s];
        v.p[s] = p;
        v.sv[s] = sv;
        v.x[s] += a * p;
        const float r = v.r[s] - a * sv;
        v.r[s] = r;
        if (jacobi) {
            const float u = r / v.d[s];
            v.u[s] = u;
            g += (double)r * (double)u;
        } else if (smoothY) {
            smoothY[s] = kAmgSmooth * r / v.d[s];  // as k_amg_jacobi computes it
        }
        rr += (double)r * (double)r;
    }
    block_sum2_atomic<kBlock>(g, rr, &v.scal[4 * (it + 1)], &v.scal[4 * (it + 1) + 3]);
}

// the replayed CG iterations' counter and target
__global__ void k_vcg_replay_begin(int32_t* iter, double* rel2Dev, double rel2, int maxIter) {
    *iter = 0;
    rel2Dev[0] = rel2;
    rel2Dev[1] = (double)maxIter;
}
__global__ void k_vcg_replay_step(int32_t* iter) { *iter += 1; }

// The end of a pass of the device-side loop around the replayed iteration:
// the counter steps (the loop's counterpart of k_vcg_replay_step), then the
// loop goes on while fewer than the cap (rel2Dev[1]) have run and rho_k >
// rel2 rho_0; a NaN stops it.  *done gets the iterations the solve took (0
// when rho_0 is 0, as the host loop counts them).  The counter steps once per
// pass, so the loop ends after the cap at the latest.
__global__ void k_vcg_loop_cond(cudaGraphConditionalHandle loop, int32_t* iter, const double* scal,
                                const double* rel2Dev, int32_t* done) {
    const int k = *iter + 1;
    *iter = k;
    const double rho0 = scal[3];
    const bool more = k < (int)rel2Dev[1] && rho0 > 0.0 && scal[4 * k + 3] > rel2Dev[0] * rho0;
    *done = rho0 > 0.0 ? k : 0;
    cudaGraphSetConditional(loop, more ? 1u : 0u);
}

// phi64[node] += x[slot] (and hist[slot] += x[slot] when recording);
// clears the slot's vectors
__global__ void k_vcg_apply(DevMesh m, VSys v, int slots, int record) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots) return;
    const int i = v.node_of[s];
    if (i >= 0) {
        m.phi64[i] += (double)v.x[s];
        if (record) v.hist[s] += v.x[s];
    }
    v.x[s] = v.r[s] = v.u[s] = v.w[s] = v.p[s] = v.sv[s] = 0.0f;
}

// hist *= alpha; phi64[node] += hist[slot]
__global__ void k_vcg_warm(DevMesh m, VSys v, int slots, float alpha) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots) return;
    const int i = v.node_of[s];
    if (i < 0) return;
    const float h = alpha * v.hist[s];
    v.hist[s] = h;
    m.phi64[i] += (double)h;
}

// The first residual of a warm solve: after the warm start has added hist to
// the V rows' potentials, r -= A hist on the V system (FP32 operator, as the
// inner solve applies it) and sum r^2 into *acc.  The residual it starts
// from is the one of the potentials before the start, kept from the last
// full pass and updated on the rows that removals touched.
__global__ void k_vcg_warm_residual(VSys v, int slices, double* acc) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    double r2 = 0.0;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < slices; warp += warps) {
        const int base = v.slice_start[warp];
        const int width = v.slice_width[warp];
        const int s = warp * 32 + lane;
        const int* __restrict__ col = v.col + base + lane;
        const float* __restrict__ val = v.val + base + lane;
        const float* __restrict__ hh = v.hist;
        float acc_ = 0.0f;
        int k = 0;
        for (; k + 8 <= width; k += 8) {
            int c[8];
            float a[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                c[j] = __ldcs(col + 32 * (k + j));
                a[j] = __ldcs(val + 32 * (k + j));
            }
#pragma unroll
            for (int j = 0; j < 8; j++) acc_ += a[j] * __ldg(hh + c[j]);
        }
        for (; k < width; k++) acc_ += __ldcs(val + 32 * k) * __ldg(hh + __ldcs(col + 32 * k));
        const float r = v.r[s] - (v.d[s] * hh[s] - acc_);
        v.r[s] = r;
        r2 += (double)r * (double)r;
    }
    block_sum_atomic<kBlock>(r2, acc);
}

// sum of r^2 over the V slots into *acc
__global__ void k_vcg_rnorm(VSys v, int slots, double* acc) {
    double r2 = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        const double r = v.r[s];
        r2 += r * r;
    }
    block_sum_atomic<kBlock>(r2, acc);
}

// r of the Neumann rows += sum over V neighbours ceff_ij x_j
// (x from the FP64 vector when x64 is given)
__global__ void k_vcg_couple_neumann(DevMesh m, VSys v, const int32_t* rows, int count, float* rN,
                                     const double* x64) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int i = rows[t];
    float s = 0.0f;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        const int sl = v.slot_of[m.col[q]];
        if (sl >= 0) s += m.ceff32[q] * (x64 ? (float)x64[sl] : v.x[sl]);
    }
    rN[i] += s;
}

// ---- FP64 inner iterations (tg_solve_opts.inner_precision 1) ----
// The same single-reduction PCG with its operator (FP64 couplings and
// diagonal at the SELL positions of the FP32 ones), vectors and recurrences
// in FP64.  The multigrid V-cycle stays FP32: it reads r rounded to float
// (written beside r64 by init and update) and returns u in FP32, which the
// FP64 recurrences take exactly.

// val64 and d64 from the FP64 couplings the rows see (ceff64) and the FP64
// diagonals, through the global-entry -> SELL-position map; the padding
// entries keep the zeros they were cleared to
__global__ void k_vcg64_derive(DevMesh m, VSys v, int nnz) {
    const int stride = gridDim.x * blockDim.x;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += stride) {
        const int p = v.vpos[q];
        if (p >= 0) v.val64[p] = m.ceff64[q];
    }
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= v.capacity; s += stride) {
        const int i = s < v.capacity ? v.node_of[s] : -1;
        v.d64[s] = i >= 0 ? m.diag64[i] : 1.0;
    }
}

// r64 = the kept FP64 residual of the slot's node (0 for padding), r = its
// float copy for the V-cycle, x64 = p64 = s64 = 0, rho_0 = r.r
__global__ void k_vcg64_init(VSys v, int slots, const double* __restrict__ rnode) {
    double rr = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        const int i = v.node_of[s];
        const double r = i >= 0 ? rnode[i] : 0.0;
        v.r64[s] = r;
        v.r[s] = (float)r;
        v.x64[s] = 0.0;
        v.p64[s] = 0.0;
        v.s64[s] = 0.0;
        rr += r * r;
    }
    block_sum_atomic<kBlock>(rr, &v.scal[3]);
}

// w64 = A64 u over SELL-32 slices; delta = w.u -> scal[4*it+1], gamma = r.u
// -> scal[4*it]
__global__ void k_vcg64_spmv(VSys v, int slices, int it, double target) {
    if (cg_done(v.scal, it, target)) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    double dl = 0.0, gl = 0.0;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < slices; warp += warps) {
        const int base = v.slice_start[warp];
        const int width = v.slice_width[warp];
        const int s = warp * 32 + lane;
        const int* __restrict__ col = v.col + base + lane;
        const double* __restrict__ val = v.val64 + base + lane;
        const float* __restrict__ uu = v.u;
        double acc = 0.0;
        int k = 0;
        for (; k + 8 <= width; k += 8) {
            int c[8];
            double a[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                c[j] = __ldcs(col + 32 * (k + j));
                a[j] = __ldcs(val + 32 * (k + j));
            }
#pragma unroll
            for (int j = 0; j < 8; j++) acc += a[j] * (double)__ldg(uu + c[j]);
        }
        for (; k < width; k++) acc += __ldcs(val + 32 * k) * (double)__ldg(uu + __ldcs(col + 32 * k));
        const double u = (double)v.u[s];
        const double w = v.d64[s] * u - acc;
        v.w64[s] = w;
        dl += w * u;
        gl += v.r64[s] * u;
    }
    block_sum2_atomic<kBlock>(dl, gl, &v.scal[4 * it + 1], &v.scal[4 * it]);
}

// p64 = u + beta p64, s64 = w64 + beta s64, x64 += alpha p64,
// r64 -= alpha s64 (and its float copy), rho_{it+1} = r.r
__global__ void k_vcg64_update(VSys v, int slots, int it, double target) {
    if (cg_done(v.scal, it, target)) return;
    double alpha, beta;
    cg_coeffs(v.scal, it, &alpha, &beta);
    if (blockIdx.x == 0 && threadIdx.x == 0) v.scal[4 * it + 2] = alpha;
    double rr = 0.0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += gridDim.x * blockDim.x) {
        const double p = (double)v.u[s] + beta * v.p64[s];
        const double sv = v.w64[s] + beta * v.s64[s];
        v.p64[s] = p;
        v.s64[s] = sv;
        v.x64[s] += alpha * p;
        const double r = v.r64[s] - alpha * sv;
        v.r64[s] = r;
        v.r[s] = (float)r;
        rr += r * r;
    }
    block_sum_atomic<kBlock>(rr, &v.scal[4 * (it + 1) + 3]);
}

// phi64[node] += x64[slot] (hist[slot] += x64[slot] when recording); clears
// the slot's vectors
__global__ void k_vcg64_apply(DevMesh m, VSys v, int slots, int record) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots) return;
    const int i = v.node_of[s];
    if (i >= 0) {
        m.phi64[i] += v.x64[s];
        if (record) v.hist[s] += (float)v.x64[s];
    }
    v.x64[s] = v.r64[s] = v.p64[s] = v.s64[s] = v.w64[s] = 0.0;
    v.x[s] = v.r[s] = v.u[s] = v.w[s] = v.p[s] = v.sv[s] = 0.0f;
}

// One row's FP64 residual r and Dirichlet part b, summed as the full pass
// (k_residual, relax.cu) sums them: in CSR order, products and sums
// unfused, so that a value kept from a full pass and one recomputed here
// agree to the bit when the row is unchanged.
__device__ void resid_row(const DevMesh& m, int i, double& r, double& b) {
    double s = 0.0, sb = 0.0;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        const int j = m.col[q];
        const double c = __dmul_rn(m.ceff64[q], m.phi64[j]);
        s = __dadd_rn(s, c);
        if (m.flags[j] & F_DIRICHLET) sb = __dadd_rn(sb, c);
    }
    const double qi = m.q64[i];
    r = __dsub_rn(__dsub_rn(s, __dmul_rn(m.diag64[i], m.phi64[i])), qi);
    b = __dsub_rn(sb, qi);
}

// Residuals of the rows that removals have changed since the last full
// pass: the flipped cells and their neighbours, the only rows whose
// couplings, class or neighbour potentials a flip touches.  One warp per
// flipped cell; a row shared by several is taken by the first warp to stamp
// it.  Each row's residual and Dirichlet part are recomputed as the full
// passes compute them; the differences of their squares to the stored
// values go into rsum (V rows, Neumann rows, b), and the FP32 right-hand
// sides of the inner solves get the new values.
// countDev (may be null): a device-side count that caps `count`, for a list
// whose length only the device knows (the learned start's cells).
__global__ void k_residual_rows(DevMesh m, VSys v, float* rN, const int32_t* __restrict__ flips, int count,
                                const int32_t* countDev, int32_t* stamp, int epoch, double* r64, double* b64,
                                double* rsum) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (countDev && *countDev < count) count = *countDev;
    if (warp >= count) return;
    const int f = flips[warp];
    const int q0 = m.row_ptr[f], q1 = m.row_ptr[f + 1];
    for (int k = lane - 1; k < q1 - q0; k += 32) {
        const int i = k < 0 ? f : m.col[q0 + k];
        if (m.flags[i] & F_DIRICHLET) continue;
        if (atomicExch(stamp + i, epoch) == epoch) continue;
        double r, b;
        resid_row(m, i, r, b);
        const double r0 = r64[i], b0 = b64[i];
        r64[i] = r;
        b64[i] = b;
        const bool neumann = (m.flags[i] & F_NEUMANN) != 0;
        if (neumann) rN[i] = (float)r;
        else v.r[v.slot_of[i]] = (float)r;
        atomicAdd(rsum + (neumann ? 1 : 0), r * r - r0 * r0);
        atomicAdd(rsum + 2, b * b - b0 * b0);
    }
}

// Row sum of a V row: d minus its stored couplings, summed in FP64 and
// rounded once.  With it the multigrid's smoothing pass applies the
// operator from bf16 couplings as (g + sum a16) y_s - sum a16 y_col, which
// keeps every row sum of the FP32 operator (constants stay in its near
// null space) and its symmetry.
__device__ __forceinline__ void vsys_set_row_sum(VSys v, int s) {
    const int base = v.slice_start[s >> 5] + (s & 31);
    const int width = v.slice_width[s >> 5];
    double sum = 0.0;
    for (int k = 0; k < width; k++) sum += v.val[base + 32 * k];
    v.g[s] = (float)((double)v.d[s] - sum);
}

__device__ __forceinline__ void vsys_set_val(VSys v, int p, float a, double a64) {
    v.val[p] = a;
    v.val16[p] = __float2bfloat16_rn(a);
    if (v.val64) v.val64[p] = a64;
}

__device__ __forceinline__ void vsys_set_diag(const DevMesh& m, VSys v, int s, int i) {
    v.d[s] = m.diag32[i];
    if (v.d64) v.d64[s] = m.diag64[i];
}

// Appends the row of a node that has just become a non-Neumann free cell
// and repoints its free neighbours' entries at it.  One warp.
__device__ void vsys_add_row(const DevMesh& m, VSys v, int i) {
    const int lane = threadIdx.x & 31;
    int s = -1;
    if (lane == 0) {
        s = atomicAdd(v.count, 1);
        if (s >= v.capacity) {
            atomicOr(m.status, S_CAPACITY);
            s = -1;
        } else {
            v.slot_of[i] = s;
            v.node_of[s] = i;
            vsys_set_diag(m, v, s, i);
        }
    }
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s < 0) return;
    __syncwarp();
    const int slice = s >> 5, r = s & 31;
    const int base = v.slice_start[slice] + r;
    const int width = v.slice_width[slice];
    const int q0 = m.row_ptr[i], q1 = m.row_ptr[i + 1];
    // entries of the new row (sequential positions among kept neighbours)
    if (lane == 0) {
        int k = 0;
        for (int q = q0; q < q1; q++) {
            const int j = m.col[q];
            const uint8_t fj = m.flags[j];
            const bool keep = !(fj & F_NEUMANN) && (!(fj & F_DIRICHLET) || m.types[m.type[j]].removable);
            if (!keep || k >= width) {
                v.vpos[q] = -1;
                continue;
            }
            const int sj = v.slot_of[j];
            v.col[base + 32 * k] = sj >= 0 ? sj : v.capacity;
            vsys_set_val(v, base + 32 * k, m.ceff32[q], m.ceff64[q]);
            v.vpos[q] = base + 32 * k;
            k++;
        }
        for (; k < width; k++) {
            v.col[base + 32 * k] = v.capacity;
            vsys_set_val(v, base + 32 * k, 0.0f, 0.0);
        }
        vsys_set_row_sum(v, s);
    }
    __syncwarp();
    // neighbours that are V rows: their entry for i now points at slot s
    for (int q = q0 + lane; q < q1; q += 32) {
        const int j = m.col[q];
        const int sj = v.slot_of[j];
        if (sj < 0) continue;
        const int p = v.vpos[m.rev[q]];
        if (p >= 0) {
            v.col[p] = s;
            vsys_set_val(v, p, m.ceff32[m.rev[q]], m.ceff64[m.rev[q]]);
        }
        vsys_set_diag(m, v, sj, j);
        vsys_set_row_sum(v, sj);
    }
    __syncwarp();
}

__global__ void k_vsys_add_rows(DevMesh m, VSys v, const int32_t* nodes, int count) {
    for (int k = 0; k < count; k++) vsys_add_row(m, v, nodes[k]);
}

// After a flip has resynced the couplings of cell i (flip_and_resync), the
// V system's copies of them: i's own row when it has one, the entries of
// its V neighbours that point at it, and those rows' diagonals.  One warp
// per cell.
__global__ void k_vsys_refresh(DevMesh m, VSys v, const int32_t* nodes, int count) {
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < count; k++) {
        const int i = nodes[k];
        const int si = v.slot_of[i];
        if (si >= 0 && lane == 0) vsys_set_diag(m, v, si, i);
        for (int q = m.row_ptr[i] + lane; q < m.row_ptr[i + 1]; q += 32) {
            if (si >= 0 && v.vpos[q] >= 0) vsys_set_val(v, v.vpos[q], m.ceff32[q], m.ceff64[q]);
            const int j = m.col[q];
            const int sj = v.slot_of[j];
            if (sj < 0) continue;
            const int p = v.vpos[m.rev[q]];
            if (p >= 0) vsys_set_val(v, p, m.ceff32[m.rev[q]], m.ceff64[m.rev[q]]);
            vsys_set_diag(m, v, sj, j);
            vsys_set_row_sum(v, sj);
        }
        __syncwarp();
        if (si >= 0 && lane == 0) vsys_set_row_sum(v, si);
        __syncwarp();
    }
}

__global__ void k_vsys_derive(VSys v, size_t stored) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < stored; e += stride)
        v.val16[e] = __float2bfloat16_rn(v.val[e]);
    for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < (size_t)v.capacity; s += stride)
        vsys_set_row_sum(v, (int)s);
    if (blockIdx.x == 0 && threadIdx.x == 0) v.g[v.capacity] = 0.0f;
}

inline int blocks(int n) { return (n + kBlock - 1) / kBlock; }

// Pointwise kernels that end in a global reduction loop over their rows
// with a grid of at most eight blocks per SM (full occupancy at 256
// threads), so that the reduction costs ~1.2K same-address atomics instead
// of one per 256 rows.  The SpMV keeps one warp per slice over the full
// grid: slices differ in width, and many small blocks balance them.
inline int reduce_blocks(int n) {
    static const int cap = [] {  // initialised once, also under concurrent host threads
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return 8 * (sms > 0 ? sms : 148);
    }();
    const int b = blocks(n);
    return b < cap ? b : cap;
}

}  // namespace

void launch_vcg_init(const VSys& v, int slots, bool jacobi, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg_init<<<reduce_blocks(slots), kBlock, 0, s>>>(v, slots, jacobi ? 1 : 0); }
}
void launch_vcg_spmv(const VSys& v, int slots, int it, double target, bool withGamma, cudaStream_t s) {
    const int slices = (slots + 31) / 32;
    if (slices > 0) {
        count_launch();
        k_vcg_spmv<<<blocks(slices * 32), kBlock, 0, s>>>(v, slices, make_gate(v, it, target), withGamma ? 1 : 0);
    }
}
void launch_vcg_update(const VSys& v, int slots, int it, double target, bool jacobi, cudaStream_t s,
                       float* smoothY) {
    if (slots > 0) {
        count_launch();
        k_vcg_update<<<reduce_blocks(slots), kBlock, 0, s>>>(v, slots, make_gate(v, it, target), jacobi ? 1 : 0,
                                                             jacobi ? nullptr : smoothY);
    }
}
void launch_vcg_replay_begin(int32_t* iter, double* rel2Dev, double rel2, int maxIter, cudaStream_t s) {
    count_launch();
    k_vcg_replay_begin<<<1, 1, 0, s>>>(iter, rel2Dev, rel2, maxIter);
}
void launch_vcg_loop_cond(cudaGraphConditionalHandle loop, int32_t* iter, const double* scal,
                          const double* rel2Dev, int32_t* done, cudaStream_t s) {
    count_launch();
    k_vcg_loop_cond<<<1, 1, 0, s>>>(loop, iter, scal, rel2Dev, done);
}
void launch_vcg_replay_step(int32_t* iter, cudaStream_t s) {
    count_launch();
    k_vcg_replay_step<<<1, 1, 0, s>>>(iter);
}
void launch_vcg_apply(const DevMesh& m, const VSys& v, int slots, bool record, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg_apply<<<blocks(slots), kBlock, 0, s>>>(m, v, slots, record ? 1 : 0); }
}
void launch_vcg_warm(const DevMesh& m, const VSys& v, int slots, float alpha, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg_warm<<<blocks(slots), kBlock, 0, s>>>(m, v, slots, alpha); }
}
void launch_vcg_rnorm(const VSys& v, int slots, double* acc, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg_rnorm<<<reduce_blocks(slots), kBlock, 0, s>>>(v, slots, acc); }
}
void launch_vcg_warm_residual(const VSys& v, int slots, double* acc, cudaStream_t s) {
    const int slices = (slots + 31) / 32;
    if (slices > 0) {
        count_launch();
        k_vcg_warm_residual<<<blocks(slices * 32), kBlock, 0, s>>>(v, slices, acc);
    }
}
void launch_vcg_couple_neumann(const DevMesh& m, const VSys& v, const int32_t* rows, int count, float* rN,
                               cudaStream_t s, bool fromX64) {
    if (count > 0) {
        count_launch();
        k_vcg_couple_neumann<<<blocks(count), kBlock, 0, s>>>(m, v, rows, count, rN, fromX64 ? v.x64 : nullptr);
    }
}
void launch_vcg64_derive(const DevMesh& m, const VSys& v, int nnz, cudaStream_t s) {
    count_launch();
    k_vcg64_derive<<<4096, kBlock, 0, s>>>(m, v, nnz);
}
void launch_vcg64_init(const VSys& v, int slots, const double* rnode, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg64_init<<<reduce_blocks(slots), kBlock, 0, s>>>(v, slots, rnode); }
}
void launch_vcg64_spmv(const VSys& v, int slots, int it, double target, cudaStream_t s) {
    const int slices = (slots + 31) / 32;
    if (slices > 0) { count_launch(); k_vcg64_spmv<<<blocks(slices * 32), kBlock, 0, s>>>(v, slices, it, target); }
}
void launch_vcg64_update(const VSys& v, int slots, int it, double target, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg64_update<<<reduce_blocks(slots), kBlock, 0, s>>>(v, slots, it, target); }
}
void launch_vcg64_apply(const DevMesh& m, const VSys& v, int slots, bool record, cudaStream_t s) {
    if (slots > 0) { count_launch(); k_vcg64_apply<<<blocks(slots), kBlock, 0, s>>>(m, v, slots, record ? 1 : 0); }
}
void launch_vcg_residual(const DevMesh& m, const VSys& v, const int32_t* rows, int count, double* acc, double* bacc,
                         cudaStream_t s, double* r64, double* b64) {
    // the residual pass of relax.cu, writing each row's float residual to
    // its slot of the V system
    launch_residual(m, rows, count, v.r, acc, s, bacc, r64, b64, v.slot_of);
}
void launch_residual_rows(const DevMesh& m, const VSys& v, float* rN, const int32_t* flips, int count, int32_t* stamp,
                          int epoch, double* r64, double* b64, double* rsum, cudaStream_t s, const int32_t* countDev) {
    if (count > 0) {
        count_launch();
        k_residual_rows<<<(count + kBlock / 32 - 1) / (kBlock / 32), kBlock, 0, s>>>(m, v, rN, flips, count, countDev,
                                                                                     stamp, epoch, r64, b64, rsum);
    }
}
void launch_vsys_add_rows(const DevMesh& m, const VSys& v, const int32_t* nodes, int count, cudaStream_t s) {
    if (count > 0) { count_launch(); k_vsys_add_rows<<<1, 32, 0, s>>>(m, v, nodes, count); }
}
void launch_vsys_derive(const VSys& v, size_t stored, cudaStream_t s) {
    count_launch();
    k_vsys_derive<<<4096, kBlock, 0, s>>>(v, stored);
}
void launch_vsys_refresh(const DevMesh& m, const VSys& v, const int32_t* nodes, int count, cudaStream_t s) {
    if (count > 0) { count_launch(); k_vsys_refresh<<<1, 32, 0, s>>>(m, v, nodes, count); }
}

}  // namespace tgd
