// Finite-volume relaxation kernels: coloured Gauss-Seidel sweeps (the
// reference's computePotential update), FP64 residual and norm reductions,
// and the FP32 conjugate-gradient iterations used inside the FP64
// defect-correction solve.
//
// Update rule restated from Grid_3d::Table::computePotential
// (tapsim/grid_3d.cpp:1317-1371):
//   Dirichlet row: unchanged
//   Neumann row:   phi_i = (sum_j c_ij phi_j - q_i) / sum_j c_ij      (all j)
//   other rows:    the same sums skipping Neumann neighbours
// The skip is folded into ceff (0 for a Neumann neighbour of a non-Neumann
// row), so every free row is phi_i = (sum_j ceff_ij phi_j - q_i) / diag_i.
#include "kernels.cuh"

namespace tgd {
namespace {

constexpr int kBlock = 256;

__global__ void k_sweep64(DevMesh m, const int32_t* __restrict__ rows, int count, double* maxdev) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double dev = 0.0;
    if (t < count) {
        const int i = rows[t];
        const int q0 = m.row_ptr[i], q1 = m.row_ptr[i + 1];
        double s = 0.0;
        for (int q = q0; q < q1; q++) s += m.ceff64[q] * m.phi64[m.col[q]];
        const double d = m.diag64[i];
        const double v = (s - m.q64[i]) / d;
        if (!(v == v)) {
            atomicOr(m.status, S_NAN);
        } else {
            dev = fabs(v - m.phi64[i]);
            m.phi64[i] = v;
        }
    }
    if (maxdev) {
        __shared__ double red[kBlock / 32];
        dev = warp_max_d(dev);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dev;
        __syncthreads();
        if (threadIdx.x < 32) {
            double v = threadIdx.x < kBlock / 32 ? red[threadIdx.x] : 0.0;
            v = warp_max_d(v);
            if (threadIdx.x == 0 && v > 0.0) atomic_max_double_nonneg(maxdev, v);
        }
    }
}

// FP64 residual r_i = sum_j ceff_ij phi_j - diag_i phi_i - q_i of a row
// list, sum r^2 into *acc; one thread per row, the row's entries in CSR
// order with unfused products and sums (resid_row in cg.cu repeats them for
// the incremental residuals, bit for bit).  One thread per row keeps a
// row's whole chain of loads in flight per thread; groups of lanes per row,
// or a warp staging its rows' span in shared memory first, measured slower
// on the 7.3M-cell tip (2.4 and 3.0 TB/s against 4.1).
// r32 (may be null) gets r as float, at slotOf[i] when slotOf is given (the
// V system's slot) and at i otherwise; r64 and b64 (may be null) keep r and
// the Dirichlet part by node.  With bacc, also the squared norm of the rows'
// Dirichlet part b_i = sum over Dirichlet neighbours ceff_ij phi_j - q_i
// (k_bnorm's value) from the same pass.
__global__ void k_residual(DevMesh m, const int32_t* __restrict__ rows, int count, float* r32,
                           const int32_t* __restrict__ slotOf, double* acc, double* bacc, double* r64, double* b64) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool withB = bacc != nullptr;  // uniform over the grid
    double r2 = 0.0, b2 = 0.0;
    if (t < count) {
        const int i = rows[t];
        const int q0 = m.row_ptr[i], q1 = m.row_ptr[i + 1];
        double s = 0.0, sb = 0.0;
        for (int q = q0; q < q1; q++) {
            const int j = m.col[q];
            const double c = __dmul_rn(m.ceff64[q], m.phi64[j]);
            s = __dadd_rn(s, c);
            if (withB && (m.flags[j] & F_DIRICHLET)) sb = __dadd_rn(sb, c);
        }
        const double qi = m.q64[i];
        const double r = __dsub_rn(__dsub_rn(s, __dmul_rn(m.diag64[i], m.phi64[i])), qi);
        const double b = __dsub_rn(sb, qi);
        if (r32) r32[slotOf ? slotOf[i] : i] = (float)r;
        if (r64) r64[i] = r;
        if (b64) b64[i] = b;
        r2 = r * r;
        b2 = b * b;
    }
    if (withB) block_sum2_atomic<kBlock>(r2, b2, acc, bacc);
    else block_sum_atomic<kBlock>(r2, acc);
}

__global__ void k_bnorm(DevMesh m, const int32_t* __restrict__ rows, int count, double* acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double b = 0.0;
    if (t < count) {
        const int i = rows[t];
        const int q0 = m.row_ptr[i], q1 = m.row_ptr[i + 1];
        double s = 0.0;
        for (int q = q0; q < q1; q++) {
            const int j = m.col[q];
            if (m.flags[j] & F_DIRICHLET) s += m.ceff64[q] * m.phi64[j];
        }
        b = s - m.q64[i];
    }
    block_sum_atomic<kBlock>(b * b, acc);
}

// z = r / diag, p = z, rz -> scal[0]
__global__ void k_cg_init(DevMesh m, const int32_t* __restrict__ rows, int count, CGVectors v) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double rz = 0.0, rr = 0.0;
    if (t < count) {
        const int i = rows[t];
        const float r = v.r[i];
        const float z = r / m.diag32[i];
        v.z[i] = z;
        v.p[i] = z;
        v.x[i] = 0.0f;
        rz = (double)r * (double)z;
        rr = (double)r * (double)r;
    }
    block_sum_atomic<kBlock>(rz, &v.scal[0]);
    block_sum_atomic<kBlock>(rr, &v.scal[2]);
}

// The target of r.r: rel2 times its start value (scal[2]), and at least
// abs2; an iteration whose r.r (scal[3it+2]) meets it is done (rel2 < 0:
// never).  Formed on
// the device, so that iterations queue before the host has read r.r.
__device__ __forceinline__ bool cg_met(const double* scal, int it, double rel2, double abs2) {
    if (rel2 < 0.0) return false;  // never (launch_cg_spmv_only)
    return scal[3 * it + 2] <= fmax(rel2 * scal[2], abs2);
}

// an iteration replayed from a CUDA graph takes its index and targets from
// device memory (CGVectors::iter, tgt)
__device__ __forceinline__ void cg_replayed(const CGVectors& v, int& it, double& rel2, double& abs2) {
    if (v.iter) {
        it += *v.iter;
        rel2 = v.tgt[0];
        abs2 = v.tgt[1];
    }
}

// ap = A p on the rows (A = diag - offdiag), pAp -> scal[3it+1]; all three
// kernels of an iteration are skipped once it is done (cg_met)
__global__ void k_cg_spmv(DevMesh m, const int32_t* __restrict__ rows, int count, CGVectors v, int it, double rel2,
                          double abs2) {
    cg_replayed(v, it, rel2, abs2);
    if (cg_met(v.scal, it, rel2, abs2)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double pap = 0.0;
    if (t < count) {
        const int i = rows[t];
        const int q0 = m.row_ptr[i], q1 = m.row_ptr[i + 1];
        float s = 0.0f;
        for (int q = q0; q < q1; q++) s += m.ceff32[q] * v.p[m.col[q]];
        const float pi = v.p[i];
        const float ap = m.diag32[i] * pi - s;
        v.ap[i] = ap;
        pap = (double)pi * (double)ap;
    }
    block_sum_atomic<kBlock>(pap, &v.scal[3 * it + 1]);
}

// x += a p, r -= a ap, z = r/diag, rz_next -> scal[3(it+1)], r.r -> scal[3(it+1)+2]
__global__ void k_cg_update(DevMesh m, const int32_t* __restrict__ rows, int count, CGVectors v, int it, double rel2,
                            double abs2) {
    cg_replayed(v, it, rel2, abs2);
    const double rz = v.scal[3 * it];
    if (cg_met(v.scal, it, rel2, abs2)) return;
    const double pap = v.scal[3 * it + 1];
    const float alpha = pap > 0.0 ? (float)(rz / pap) : 0.0f;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double rzn = 0.0, rrn = 0.0;
    if (t < count) {
        const int i = rows[t];
        v.x[i] += alpha * v.p[i];
        const float r = v.r[i] - alpha * v.ap[i];
        v.r[i] = r;
        const float z = r / m.diag32[i];
        v.z[i] = z;
        rzn = (double)r * (double)z;
        rrn = (double)r * (double)r;
    }
    block_sum_atomic<kBlock>(rzn, &v.scal[3 * (it + 1)]);
    block_sum_atomic<kBlock>(rrn, &v.scal[3 * (it + 1) + 2]);
}

// p = z + beta p
__global__ void k_cg_pupdate(const int32_t* __restrict__ rows, int count, CGVectors v, int it, double rel2,
                             double abs2) {
    cg_replayed(v, it, rel2, abs2);
    const double rz = v.scal[3 * it];
    if (cg_met(v.scal, it, rel2, abs2)) return;
    const double rzn = v.scal[3 * (it + 1)];
    const float beta = (float)(rzn / rz);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) {
        const int i = rows[t];
        v.p[i] = v.z[i] + beta * v.p[i];
    }
}

__global__ void k_cg_replay_begin(int32_t* iter, double* tgt, double rel2, double abs2) {
    *iter = 0;
    tgt[0] = rel2;
    tgt[1] = abs2;
}
__global__ void k_cg_replay_step(int32_t* iter) { *iter += 1; }

__global__ void k_add_coupled(DevMesh m, const int32_t* __restrict__ rows, int count, const float* xV, float* r) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int i = rows[t];
    float s = 0.0f;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) s += m.ceff32[q] * xV[m.col[q]];
    r[i] += s;
}

__global__ void k_apply_correction(DevMesh m, const int32_t* __restrict__ rows, int count, CGVectors v) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int i = rows[t];
    m.phi64[i] += (double)v.x[i];
    v.x[i] = 0.0f;
    v.r[i] = 0.0f;
    v.z[i] = 0.0f;
    v.p[i] = 0.0f;
    v.ap[i] = 0.0f;
}

__global__ void k_rebuild_rows(DevMesh m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.n) return;
    const bool neuI = (m.flags[i] & F_NEUMANN) != 0;
    double d = 0.0;
    for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) {
        const bool neuJ = (m.flags[m.col[q]] & F_NEUMANN) != 0;
        const double c = (!neuI && neuJ) ? 0.0 : m.c64[q];
        m.ceff64[q] = c;
        m.ceff32[q] = (float)c;
        d += c;
    }
    m.diag64[i] = d;
    m.diag32[i] = (float)d;
}

// Breadth-first k-hop neighbourhood of one node, one block.  The visited set
// is an open-addressing hash in shared memory; frontiers live in global
// scratch.  Non-Dirichlet members are written grouped by colour.
constexpr int kHashSize = 8192;

__global__ void k_local_set(DevMesh m, int node, int hops, int32_t* out, int32_t* outCount, int cap, int32_t* scratch,
                            int scratchCap, int ncolours) {
    __shared__ int32_t hashKeys[kHashSize];
    __shared__ int frontierStart, frontierEnd, tail, overflow;
    __shared__ int colourCount[64], colourOffset[64];
    for (int k = threadIdx.x; k < kHashSize; k += blockDim.x) hashKeys[k] = -1;
    if (threadIdx.x < 64) colourCount[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        scratch[0] = node;
        frontierStart = 0;
        frontierEnd = 1;
        tail = 1;
        overflow = 0;
    }
    __syncthreads();
    // the start node is only recorded when reached again (find_localNodes)
    for (int h = 0; h < hops; h++) {
        const int fs = frontierStart, fe = frontierEnd;
        for (int f = fs + threadIdx.x; f < fe; f += blockDim.x) {
            const int u = scratch[f];
            for (int q = m.row_ptr[u]; q < m.row_ptr[u + 1]; q++) {
                const int v = m.col[q];
                uint32_t hsh = ((uint32_t)v * 2654435761u) & (kHashSize - 1);
                bool inserted = false;
                for (int probe = 0; probe < kHashSize; probe++) {
                    const int prev = atomicCAS(&hashKeys[hsh], -1, v);
                    if (prev == -1) { inserted = true; break; }
                    if (prev == v) break;
                    hsh = (hsh + 1) & (kHashSize - 1);
                }
                if (inserted) {
                    const int pos = atomicAdd(&tail, 1);
                    if (pos < scratchCap) scratch[pos] = v;
                    else overflow = 1;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            frontierStart = fe;
            frontierEnd = min(tail, scratchCap);
        }
        __syncthreads();
    }
    // members: scratch[1 .. tail) plus the start node if it was reached again
    const int members = min(tail, scratchCap);
    for (int f = 1 + threadIdx.x; f < members; f += blockDim.x) {
        const int v = scratch[f];
        if (!(m.flags[v] & F_DIRICHLET)) atomicAdd(&colourCount[m.colour[v]], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int c = 0; c < ncolours; c++) {
            colourOffset[c] = s;
            outCount[c] = colourCount[c];
            s += colourCount[c];
            colourCount[c] = 0;
        }
        outCount[ncolours] = s;
        outCount[ncolours + 1] = overflow;
    }
    __syncthreads();
    for (int f = 1 + threadIdx.x; f < members; f += blockDim.x) {
        const int v = scratch[f];
        if (!(m.flags[v] & F_DIRICHLET)) {
            const int c = m.colour[v];
            const int pos = colourOffset[c] + atomicAdd(&colourCount[c], 1);
            if (pos < cap) out[pos] = v;
        }
    }
}

inline int blocks(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

void launch_sweep64(const DevMesh& m, const int32_t* rows, int count, double* maxdev, cudaStream_t s) {
    if (count > 0) { count_launch(); k_sweep64<<<blocks(count), kBlock, 0, s>>>(m, rows, count, maxdev); }
}
void launch_residual(const DevMesh& m, const int32_t* rows, int count, float* r32, double* acc, cudaStream_t s,
                     double* bacc, double* r64, double* b64, const int32_t* slotOf) {
    if (count <= 0) return;
    count_launch();
    b64 = bacc ? b64 : nullptr;
    k_residual<<<blocks(count), kBlock, 0, s>>>(m, rows, count, r32, slotOf, acc, bacc, r64, b64);
}
void launch_bnorm(const DevMesh& m, const int32_t* rows, int count, double* acc, cudaStream_t s) {
    if (count > 0) { count_launch(); k_bnorm<<<blocks(count), kBlock, 0, s>>>(m, rows, count, acc); }
}
void launch_cg_init(const DevMesh& m, const int32_t* rows, int count, CGVectors v, cudaStream_t s) {
    if (count > 0) { count_launch(); k_cg_init<<<blocks(count), kBlock, 0, s>>>(m, rows, count, v); }
}
void launch_cg_iter(const DevMesh& m, const int32_t* rows, int count, CGVectors v, int it, double rel2, double abs2,
                    cudaStream_t s) {
    if (count <= 0) return;
    { count_launch(); k_cg_spmv<<<blocks(count), kBlock, 0, s>>>(m, rows, count, v, it, rel2, abs2); }
    { count_launch(); k_cg_update<<<blocks(count), kBlock, 0, s>>>(m, rows, count, v, it, rel2, abs2); }
    { count_launch(); k_cg_pupdate<<<blocks(count), kBlock, 0, s>>>(rows, count, v, it, rel2, abs2); }
}
void launch_cg_replay_begin(int32_t* iter, double* tgt, double rel2, double abs2, cudaStream_t s) {
    count_launch();
    k_cg_replay_begin<<<1, 1, 0, s>>>(iter, tgt, rel2, abs2);
}
void launch_cg_replay_step(int32_t* iter, cudaStream_t s) {
    count_launch();
    k_cg_replay_step<<<1, 1, 0, s>>>(iter);
}
void launch_cg_spmv_only(const DevMesh& m, const int32_t* rows, int count, CGVectors v, cudaStream_t s) {
    if (count > 0) { count_launch(); k_cg_spmv<<<blocks(count), kBlock, 0, s>>>(m, rows, count, v, 0, -1.0, -1.0); }
}
void launch_add_coupled(const DevMesh& m, const int32_t* rows, int count, const float* xV, float* r, cudaStream_t s) {
    if (count > 0) { count_launch(); k_add_coupled<<<blocks(count), kBlock, 0, s>>>(m, rows, count, xV, r); }
}
void launch_apply_correction(const DevMesh& m, const int32_t* rows, int count, CGVectors v, cudaStream_t s) {
    if (count > 0) { count_launch(); k_apply_correction<<<blocks(count), kBlock, 0, s>>>(m, rows, count, v); }
}
void launch_rebuild_rows(const DevMesh& m, cudaStream_t s) {
    if (m.n > 0) { count_launch(); k_rebuild_rows<<<blocks(m.n), kBlock, 0, s>>>(m); }
}
void launch_local_set(const DevMesh& m, int node, int hops, int32_t* out, int32_t* outCount, int cap, int32_t* scratch,
                      int scratchCap, int ncolours, cudaStream_t s) {
    { count_launch(); k_local_set<<<1, 512, 0, s>>>(m, node, hops, out, outCount, cap, scratch, scratchCap, ncolours); }
}

}  // namespace tgd
