// Smoothed-aggregation multigrid V-cycle as the preconditioner of the V
// system's conjugate gradients: u = M^-1 r.
//
// Level 0 is the live V system (SELL-32, cg.cu), so the fine operator is
// always the current one; the prolongator P_0 covers the slots that existed
// when the hierarchy was built, and slots appended later by removals are
// only smoothed.  Levels 1.. hold their Galerkin operators R A P in CSR
// (FP32), and the coarsest level is solved with a dense inverse.  The cycle
// is V(1,1) with damped Jacobi (weight 0.9) before and after the coarse
// correction, which keeps the preconditioner symmetric:
//     y = w D^-1 b;  t = b - A y;  b' = R t;  x' = cycle(b');  y += P x';
//     x = y + w D^-1 (b - A y)
// Every kernel returns at once when the CG iteration it belongs to has
// already met its target, as the CG kernels do.
#include "kernels.cuh"

namespace tgd {
namespace {

constexpr int kBlock = 256;
// damped-Jacobi weight of the smoothing steps: below 1, so that the
// smoother converges in the energy norm (rho(D^-1 A) <= 2 for these
// diagonally dominant matrices) and the cycle stays symmetric positive
// definite; 0.9 took 21 CG iterations to 1e-8 on the 3.2M-row system of the
// 7.3M-cell tip where 2/3 took 27
constexpr float kSmooth = kAmgSmooth;

// y = w b / d
__global__ void k_amg_jacobi(int n, const float* b, const float* d, float* y, Gate gate) {
    if (gate.done()) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = kSmooth * b[i] / d[i];
}

// Level 0 over SELL-32 slices: mode 0: t = b - A y; mode 1: x = y + w (b - A y) / d.
// A is applied from the bf16 couplings and the FP32 row sums g:
// (A y)_s = (g_s + sum a16) y_s - sum a16 y_col.  Its entries differ from
// the CG's FP32 operator by at most 2^-9 relative and its row sums not at
// all, so it is spectrally within a fraction of a percent of it; the
// smoothing steps divide by the FP32 diagonal d on both sides of the cycle,
// which keeps the preconditioner symmetric.
// The entries k..width-1 (fewer than U) of a lane's row as one round: every
// column and value load is issued before the first gather, so that a slice's
// remainder costs one round trip, not one per entry.  The sums take the
// entries in the same order as a loop over them would.
template <int U>
__device__ __forceinline__ void fine_last_round(const int* __restrict__ col, const __nv_bfloat16* __restrict__ val,
                                                const float* __restrict__ y, int k, int width, float& acc,
                                                float& sum) {
    if (k >= width) return;
    int c[U];
    float a[U];
#pragma unroll
    for (int j = 0; j < U; j++) {
        const bool in = k + j < width;
        c[j] = in ? __ldcs(col + 32 * (k + j)) : 0;
        a[j] = in ? __bfloat162float(__ldcs(val + 32 * (k + j))) : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < U; j++)
        if (k + j < width) {
            acc += a[j] * __ldg(y + c[j]);
            sum += a[j];
        }
}

// U: the column/value loads a lane issues ahead of their gathers (the bytes
// a warp keeps in flight), chosen per hierarchy by timed trials.
template <int U>
__global__ void k_amg_fine(VSys v, int slices, const float* b, const float* y, float* out, int mode, Gate gate) {
    if (gate.done()) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < slices; warp += warps) {
        const int base = v.slice_start[warp];
        const int width = v.slice_width[warp];
        const int s = warp * 32 + lane;
        const int* __restrict__ col = v.col + base + lane;
        const __nv_bfloat16* __restrict__ val = v.val16 + base + lane;
        float acc = 0.0f, sum = 0.0f;
        int k = 0;
        for (; k + U <= width; k += U) {
            int c[U];
            float a[U];
#pragma unroll
            for (int j = 0; j < U; j++) {
                c[j] = __ldcs(col + 32 * (k + j));
                a[j] = __bfloat162float(__ldcs(val + 32 * (k + j)));
            }
#pragma unroll
            for (int j = 0; j < U; j++) {
                acc += a[j] * __ldg(y + c[j]);
                sum += a[j];
            }
        }
        fine_last_round<U>(col, val, y, k, width, acc, sum);
        const float ys = y[s];
        const float t = b[s] - ((v.g[s] + sum) * ys - acc);
        out[s] = mode == 0 ? t : ys + kSmooth * t / v.d[s];
    }
}

// The level-0 pass software-pipelined: a lane loads the columns and values
// of its next U entries before it gathers the y of the current U, so that
// the next round's loads from DRAM wait out the current round's gathers
// (chosen per hierarchy against k_amg_fine by timed trials).
template <int U>
__global__ void k_amg_fine_pipe(VSys v, int slices, const float* b, const float* y, float* out, int mode,
                                Gate gate) {
    if (gate.done()) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; warp < slices; warp += warps) {
        const int base = v.slice_start[warp];
        const int width = v.slice_width[warp];
        const int s = warp * 32 + lane;
        const int* __restrict__ col = v.col + base + lane;
        const __nv_bfloat16* __restrict__ val = v.val16 + base + lane;
        float acc = 0.0f, sum = 0.0f;
        const int rounds = width / U;
        int c[U];
        float a[U];
        if (rounds > 0) {
#pragma unroll
            for (int j = 0; j < U; j++) {
                c[j] = __ldcs(col + 32 * j);
                a[j] = __bfloat162float(__ldcs(val + 32 * j));
            }
        }
        for (int r = 0; r < rounds; r++) {
            int cn[U];
            float an[U];
            const bool more = r + 1 < rounds;
            if (more) {
#pragma unroll
                for (int j = 0; j < U; j++) {
                    cn[j] = __ldcs(col + 32 * ((r + 1) * U + j));
                    an[j] = __bfloat162float(__ldcs(val + 32 * ((r + 1) * U + j)));
                }
            }
#pragma unroll
            for (int j = 0; j < U; j++) {
                acc += a[j] * __ldg(y + c[j]);
                sum += a[j];
            }
            if (more) {
#pragma unroll
                for (int j = 0; j < U; j++) {
                    c[j] = cn[j];
                    a[j] = an[j];
                }
            }
        }
        fine_last_round<U>(col, val, y, rounds * U, width, acc, sum);
        const float ys = y[s];
        const float t = b[s] - ((v.g[s] + sum) * ys - acc);
        out[s] = mode == 0 ? t : ys + kSmooth * t / v.d[s];
    }
}

// Rows of the coarse operators and of the restrictions hold tens to a few
// hundred entries: a group of L lanes per row (L from the matrix's mean row
// length, AmgDevLevel::a_lanes / r_lanes), one row per group, a grid with a
// group for every row (no grid-stride loop, so that every row's loads are in
// flight at once).  Each lane loads four of its entries before it gathers
// their y, so that a row of up to 4 L entries costs one round trip.
template <int L>
__device__ __forceinline__ float row_dot(const int32_t* ptr, const int32_t* col, const float* val, const float* y,
                                         int row, int lane) {
    float acc = 0.0f;
    const int q1 = ptr[row + 1];
    for (int q = ptr[row] + lane; q < q1; q += 4 * L) {
        int c[4];
        float a[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool in = q + j * L < q1;
            c[j] = in ? __ldcs(col + q + j * L) : -1;
            a[j] = in ? __ldcs(val + q + j * L) : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (c[j] >= 0) acc += a[j] * __ldg(y + c[j]);
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// Rows of a CSR operator A (with its diagonal):
// mode 0: t = b - A y; mode 1: x = y + w (b - A y) / diag
template <int L>
__global__ void k_amg_csr(int n, const int32_t* ptr, const int32_t* col, const float* val, const float* diag,
                          const float* b, const float* y, float* out, int mode, Gate gate) {
    if (gate.done()) return;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = gid % L;
    const int row = min(gid / L, n - 1);  // whole groups stay active for the shuffles
    const float acc = row_dot<L>(ptr, col, val, y, row, lane);
    if (lane == 0 && gid / L < n) {
        const float t = b[row] - acc;
        out[row] = mode == 0 ? t : y[row] + kSmooth * t / diag[row];
    }
}

// out = M y for a CSR matrix (restriction R t); with diag, also the coarse
// level's pre-smoothing step ysm = w out / diag (the Jacobi step of the level
// it restricts to, in the same arithmetic as k_amg_jacobi)
template <int L>
__global__ void k_amg_mv(int n, const int32_t* ptr, const int32_t* col, const float* val, const float* y, float* out,
                         const float* diag, float* ysm, Gate gate) {
    if (gate.done()) return;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = gid % L;
    const int row = min(gid / L, n - 1);
    const float acc = row_dot<L>(ptr, col, val, y, row, lane);
    if (lane == 0 && gid / L < n) {
        out[row] = acc;
        if (diag) ysm[row] = kSmooth * acc / diag[row];
    }
}

// y += P x' (prolongation, a few entries per row), one thread per row
__global__ void k_amg_prolong(int n, const int32_t* ptr, const int32_t* col, const float* val, const float* xc,
                              float* y, Gate gate) {
    if (gate.done()) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (int q = ptr[i]; q < ptr[i + 1]; q++) acc += val[q] * __ldg(xc + col[q]);
        y[i] += acc;
    }
}

// x = C^-1 b with the coarsest level's dense inverse (row-major), one warp per row
__global__ void k_amg_dense(int n, const float* inv, const float* b, float* x, Gate gate) {
    if (gate.done()) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += warps) {
        float acc = 0.0f;
        for (int k = lane; k < n; k += 32) acc += inv[(size_t)row * n + k] * b[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) x[row] = acc;
    }
}

// a thread for every lane of every slice (the SELL kernels' grid-stride
// loop then makes one pass)
inline unsigned grid_full(long long threads) { return (unsigned)((threads + kBlock - 1) / kBlock); }

// the level-0 pass with the hierarchy's load depth (AmgDev::fine_unroll;
// plus kFinePipe: the software-pipelined kernel)
void launch_fine(int U, const VSys& v, int slices, const float* b, const float* y, float* out, int mode, Gate gate,
                 cudaStream_t s) {
    count_launch();
    const unsigned grid = grid_full((long long)slices * 32);
    if (U == kFinePipe + 4) k_amg_fine_pipe<4><<<grid, kBlock, 0, s>>>(v, slices, b, y, out, mode, gate);
    else if (U == kFinePipe + 8) k_amg_fine_pipe<8><<<grid, kBlock, 0, s>>>(v, slices, b, y, out, mode, gate);
    else if (U == 4) k_amg_fine<4><<<grid, kBlock, 0, s>>>(v, slices, b, y, out, mode, gate);
    else if (U == 16) k_amg_fine<16><<<grid, kBlock, 0, s>>>(v, slices, b, y, out, mode, gate);
    else k_amg_fine<8><<<grid, kBlock, 0, s>>>(v, slices, b, y, out, mode, gate);
}

// a group of L threads for every row
inline unsigned grid_rows(int n, int L) { return (unsigned)(((long long)n * L + kBlock - 1) / kBlock); }

// the lane-group kernels for L = 2 .. 32
void launch_csr(int L, int n, const int32_t* ptr, const int32_t* col, const float* val, const float* diag,
                const float* b, const float* y, float* out, int mode, Gate gate, cudaStream_t s) {
    count_launch();
    switch (L) {
        case 2: k_amg_csr<2><<<grid_rows(n, 2), kBlock, 0, s>>>(n, ptr, col, val, diag, b, y, out, mode, gate); break;
        case 4: k_amg_csr<4><<<grid_rows(n, 4), kBlock, 0, s>>>(n, ptr, col, val, diag, b, y, out, mode, gate); break;
        case 8: k_amg_csr<8><<<grid_rows(n, 8), kBlock, 0, s>>>(n, ptr, col, val, diag, b, y, out, mode, gate); break;
        case 16: k_amg_csr<16><<<grid_rows(n, 16), kBlock, 0, s>>>(n, ptr, col, val, diag, b, y, out, mode, gate); break;
        default: k_amg_csr<32><<<grid_rows(n, 32), kBlock, 0, s>>>(n, ptr, col, val, diag, b, y, out, mode, gate); break;
    }
}
void launch_mv(int L, int n, const int32_t* ptr, const int32_t* col, const float* val, const float* y, float* out,
               Gate gate, cudaStream_t s, const float* diag = nullptr, float* ysm = nullptr) {
    count_launch();
    switch (L) {
        case 2: k_amg_mv<2><<<grid_rows(n, 2), kBlock, 0, s>>>(n, ptr, col, val, y, out, diag, ysm, gate); break;
        case 4: k_amg_mv<4><<<grid_rows(n, 4), kBlock, 0, s>>>(n, ptr, col, val, y, out, diag, ysm, gate); break;
        case 8: k_amg_mv<8><<<grid_rows(n, 8), kBlock, 0, s>>>(n, ptr, col, val, y, out, diag, ysm, gate); break;
        case 16: k_amg_mv<16><<<grid_rows(n, 16), kBlock, 0, s>>>(n, ptr, col, val, y, out, diag, ysm, gate); break;
        default: k_amg_mv<32><<<grid_rows(n, 32), kBlock, 0, s>>>(n, ptr, col, val, y, out, diag, ysm, gate); break;
    }
}

inline int grid_for(long long threads) {
    static const int cap = [] {  // initialised once, also under concurrent host threads
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return 16 * (sms > 0 ? sms : 148);
    }();
    const long long b = (threads + kBlock - 1) / kBlock;
    return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// Time of one launch of f() on s: after a warm-up launch, the least mean of
// three batches of `trials` launches (the least, so that a batch slowed by
// anything else on the device does not decide).
template <class F>
float time_launches(F f, int trials, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    f();
    float best = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(e0, s);
        for (int k = 0; k < trials; k++) f();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = fminf(best, ms / trials);
    }
    return best;
}

}  // namespace

int amg_tune_lanes(AmgDev& g, const VSys& v, int slots, cudaStream_t s, float* aMs, float* rMs, float* fineMs) {
    static const int kCand[5] = {2, 4, 8, 16, 32};
    constexpr int kTrials = 3;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return -1;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return -1;
    }
    // The objective is the whole V-cycle as the solve runs it (its output u
    // and the levels' work vectors are scratch until the solve writes them):
    // timed alone, a coarse level's matrix stays in L2 and more lanes look
    // faster, while inside the cycle the fine level's stream has evicted it.
    // One choice at a time, from the row-length rule's schedule, each kept
    // only when it takes at least 3% off the cycle.
    auto cycle = [&] { return time_launches([&] { launch_amg_vcycle(v, slots, g, 0, -1.0, s); }, kTrials, s, e0, e1); };
    constexpr float kMargin = 0.97f;
    float best = cycle();
    auto tryChoice = [&](int* knob, const int* cands, int nc) {
        const int keep = *knob;
        int chosen = keep;
        for (int k = 0; k < nc; k++) {
            if (cands[k] == keep) continue;
            *knob = cands[k];
            const float ms = cycle();
            if (ms < kMargin * best) {
                best = ms;
                chosen = cands[k];
            }
        }
        *knob = chosen;
    };
    static const int kUnroll[5] = {4, 8, 16, kFinePipe + 4, kFinePipe + 8};
    tryChoice(&g.fine_unroll, kUnroll, 5);
    for (int l = 0; l + 1 < g.levels; l++) {
        tryChoice(&g.lev[l].r_lanes, kCand, 5);
        if (l + 2 < g.levels) tryChoice(&g.lev[l + 1].a_lanes, kCand, 5);
    }
    // the kept kernels' own times, for the record
    if (fineMs) {
        const int slices = (slots + 31) / 32;
        *fineMs = time_launches([&] { launch_fine(g.fine_unroll, v, slices, v.r, g.y0, g.t0, 0, open_gate(), s); },
                                kTrials, s, e0, e1);
    }
    for (int l = 0; l + 1 < g.levels; l++) {
        AmgDevLevel& L = g.lev[l];
        AmgDevLevel& C = g.lev[l + 1];
        if (rMs)
            rMs[l] = time_launches(
                [&] {
                    const bool last = l + 2 == g.levels;  // C is the coarsest level (dense solve)
                    launch_mv(L.r_lanes, C.n, L.r_ptr, L.r_col, L.r_val, l == 0 ? g.t0 : L.t, C.b, open_gate(), s,
                              last ? nullptr : C.diag, last ? nullptr : C.y);
                },
                kTrials, s, e0, e1);
        if (aMs && l + 2 < g.levels)
            aMs[l + 1] = time_launches(
                [&] { launch_csr(C.a_lanes, C.n, C.a_ptr, C.a_col, C.a_val, C.diag, C.b, C.y, C.t, 0, open_gate(), s); },
                kTrials, s, e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

void launch_amg_fine_residual(const VSys& v, int slots, const AmgDev& g, cudaStream_t s) {
    const int slices = (slots + 31) / 32;
    launch_fine(g.fine_unroll, v, slices, v.r, g.y0, g.t0, 0, open_gate(), s);
}

void launch_amg_vcycle(const VSys& v, int slots, const AmgDev& g, int it, double target, cudaStream_t s,
                       bool y0Ready) {
    const Gate gate = make_gate(v, it, target);
    // level 0: b = r, output u
    const int slices = (slots + 31) / 32;
    if (!y0Ready) {
        count_launch();
        k_amg_jacobi<<<grid_for(slots), kBlock, 0, s>>>(slots, v.r, v.d, g.y0, gate);
    }
    if (g.levels > 1) {
        launch_fine(g.fine_unroll, v, slices, v.r, g.y0, g.t0, 0, gate, s);
        // down: restrict, smooth, residual
        for (int l = 0; l + 1 < g.levels; l++) {
            const AmgDevLevel& L = g.lev[l];
            const AmgDevLevel& C = g.lev[l + 1];
            const float* t = l == 0 ? g.t0 : L.t;
            if (l + 1 == g.levels - 1) {
                launch_mv(L.r_lanes, C.n, L.r_ptr, L.r_col, L.r_val, t, C.b, gate, s);
                count_launch();
                k_amg_dense<<<grid_for((long long)C.n * 32), kBlock, 0, s>>>(C.n, g.coarse_inv, C.b, C.x, gate);
            } else {
                // the restriction also takes the coarse level's pre-smoothing step
                launch_mv(L.r_lanes, C.n, L.r_ptr, L.r_col, L.r_val, t, C.b, gate, s, C.diag, C.y);
                launch_csr(C.a_lanes, C.n, C.a_ptr, C.a_col, C.a_val, C.diag, C.b, C.y, C.t, 0, gate, s);
            }
        }
        // up: prolong, post-smooth
        for (int l = g.levels - 2; l >= 0; l--) {
            const AmgDevLevel& L = g.lev[l];
            const AmgDevLevel& C = g.lev[l + 1];
            float* y = l == 0 ? g.y0 : L.y;
            count_launch();
            k_amg_prolong<<<grid_for(L.n), kBlock, 0, s>>>(L.n, L.p_ptr, L.p_col, L.p_val, C.x, y, gate);
            if (l == 0) {
                launch_fine(g.fine_unroll, v, slices, v.r, g.y0, v.u, 1, gate, s);
            } else {
                launch_csr(L.a_lanes, L.n, L.a_ptr, L.a_col, L.a_val, L.diag, L.b, L.y, L.x, 1, gate, s);
            }
        }
    } else {
        // a single level: Jacobi twice (y, then the post-smoothing step)
        launch_fine(g.fine_unroll, v, slices, v.r, g.y0, v.u, 1, gate, s);
    }
}

}  // namespace tgd
