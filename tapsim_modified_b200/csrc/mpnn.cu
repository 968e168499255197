// Kernels of the learned warm start (sm_100a).
//
// Tensor-core GEMM (tcgen05):
// C[M x N] (FP32) = A[M x K] (BF16, row-major) * B[N x K]^T (BF16, row-major),
// M a multiple of 128, N 64 or 128, K a multiple of 64.  One CTA of four
// warps computes a 128 x N tile: K is staged in chunks of 64 into shared
// memory in the canonical K-major layout without swizzle (core matrices of
// 8 rows x 16 bytes; the two core matrices of one K = 16 step 128 bytes
// apart, 8-row groups 1024 bytes apart), one thread issues four
// tcgen05.mma.kind::f16 per chunk into a TMEM accumulator of N columns and
// commits them to an mbarrier, and after the last chunk each warp reads its
// 32 TMEM lanes (rows) with tcgen05.ld.  Every wait on the mbarrier is
// bounded: on timeout the kernel sets S_TIMEOUT, waits once more (bounded)
// for the MMAs in flight, frees its TMEM and returns.
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace tgd {
namespace {

constexpr int kGemmThreads = 128;
// dynamic shared memory per CTA: tiles (16 KB + 16 KB) plus slack, sized so
// that at most four CTAs share an SM and their TMEM (4 x 128 columns) fits
constexpr int kGemmSmem = 56 * 1024;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start, leading (K) and stride (8-row
// group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// instruction descriptor: D FP32, A and B BF16, both K-major, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(128 >> 4) << 24);
}

// bounded wait for the mbarrier phase of the given parity
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// byte offset of the 16-byte piece (row r, K group k8) of a staged chunk
__device__ __forceinline__ int tile_off(int r, int k8) { return (r >> 3) * 1024 + k8 * 128 + (r & 7) * 16; }

template <int N>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16(const __nv_bfloat16* __restrict__ A,
                                                            const __nv_bfloat16* __restrict__ B, float* __restrict__ C,
                                                            int M, int K, int* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem;
    unsigned char* sB = smem + 16384;
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmemSlot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row0 = blockIdx.x * 128;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemSlot)),
                     "r"(N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmemSlot;
    const uint32_t mb = smem_u32(&mbar);

    bool ok = true;
    int issued = 0;  // chunks committed to the mbarrier
    const int nk = K / 64;
    for (int kc = 0; kc < nk; kc++) {
        for (int i = tid; i < 128 * 8; i += kGemmThreads) {
            const int r = i >> 3, c = i & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)(row0 + r) * K + kc * 64 + c * 8);
            *reinterpret_cast<uint4*>(sA + tile_off(r, c)) = v;
        }
        for (int i = tid; i < N * 8; i += kGemmThreads) {
            const int r = i >> 3, c = i & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)r * K + kc * 64 + c * 8);
            *reinterpret_cast<uint4*>(sB + tile_off(r, c)) = v;
        }
        // the tensor core reads shared memory through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int ks = 0; ks < 4; ks++) {
                const uint64_t ad = umma_desc(smem_u32(sA) + ks * 256, 128, 1024);
                const uint64_t bd = umma_desc(smem_u32(sB) + ks * 256, 128, 1024);
                const uint32_t accumulate = (kc > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc_bf16(N)), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        issued++;
        ok = mbar_wait(mb, kc & 1);
        ok = __syncthreads_and(ok);
        if (!ok) break;
    }
    if (!ok) {
        // let the MMAs in flight finish (bounded) before the TMEM is freed
        if (tid == 0) atomicOr(status, S_TIMEOUT);
        mbar_wait(mb, (issued - 1) & 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
        const int r = row0 + warp * 32 + (tid & 31);
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (r < M) {
                float4* out = reinterpret_cast<float4*>(C + (size_t)r * N + c0);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    out[j] = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                         __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(N));
}

// ---------------------------------------------------------------------------
// Message-passing network on the free cells around a removed atom.
//
// Graph: the free cells within `hops` steps of the removed cell (a BFS over
// the coupling graph that does not enter Dirichlet cells), edges weighted
// a_ij = c_ij / d_i (the Jacobi weights of the relaxation), stored ELL
// (width D, -1 padding).  Per node 16 input features (below); an input
// layer and four message layers of width 64:
//   h0 = relu(x W0 + b0);  h_l = h_{l-1} + relu([h_{l-1}, A h_{l-1}] W_l + b_l)
//   y  = h4 . w_out + b_out,   predicted correction = sigma * y
// with sigma = |r_site| / d_site, the Jacobi step of the removed cell.  The
// GEMMs run on the tensor cores (BF16 operands, FP32 accumulate); the rest
// is FP32 on the CUDA cores.  Inputs are padded to 128 columns so that every
// GEMM has M % 128 == 0 and K % 64 == 0.
// ---------------------------------------------------------------------------
constexpr int kFeat = 16, kHid = 64, kCat = 128;

// Breadth-first search from `site` over the free cells, `hops` levels, one
// CTA: each warp takes a frontier cell and its lanes its neighbours, which
// claim their cell with an atomic on localOf (-1 -> -2), so a level costs
// one round of loads instead of one per neighbour.  The list order follows
// the claims (it varies from run to run; nothing downstream depends on it).
__global__ void k_ball_bfs(DevMesh m, int site, int hops, int cap, int32_t* nodes, int8_t* level, int32_t* count,
                           int32_t* localOf) {
    __shared__ int lvlStart, lvlEnd, total;
    if (threadIdx.x == 0) {
        nodes[0] = site;
        level[0] = 0;
        localOf[site] = 0;
        lvlStart = 0;
        lvlEnd = 1;
        total = 1;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int L = 0; L < hops; L++) {
        const int s0 = lvlStart, s1 = lvlEnd;
        for (int t = s0 + warp; t < s1; t += nwarps) {
            const int u = nodes[t];
            const int q1 = m.row_ptr[u + 1];
            for (int q = m.row_ptr[u] + lane; q < q1; q += 32) {
                const int j = m.col[q];
                if (m.flags[j] & F_DIRICHLET) continue;
                if (atomicCAS(&localOf[j], -1, -2) != -1) continue;
                const int idx = atomicAdd(&total, 1);
                if (idx < cap) {
                    nodes[idx] = j;
                    level[idx] = (int8_t)(L + 1);
                    localOf[j] = idx;
                } else {
                    localOf[j] = -1;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            lvlStart = s1;
            lvlEnd = min(total, cap);
        }
        __syncthreads();
    }
    // a neighbourhood larger than `cap` is cut at cap cells (a smaller
    // prediction region, not an error: the solve still converges)
    if (threadIdx.x == 0) *count = min(total, cap);
}

__global__ void k_ball_reset(const int32_t* nodes, const int32_t* count, int32_t* localOf) {
    const int n = *count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) localOf[nodes[t]] = -1;
}

// scale[0] = sigma = |r_site| / d_site, scale[1] = mean distance from the
// site to its neighbours
__global__ void k_site_scale(DevMesh m, int site, float* scale) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sum = 0.0, dist = 0.0;
    int nbs = 0;
    const double xs = m.xyz[3 * site], ys = m.xyz[3 * site + 1], zs = m.xyz[3 * site + 2];
    for (int q = m.row_ptr[site]; q < m.row_ptr[site + 1]; q++) {
        const int j = m.col[q];
        sum += m.ceff64[q] * m.phi64[j];
        const double dx = m.xyz[3 * j] - xs, dy = m.xyz[3 * j + 1] - ys, dz = m.xyz[3 * j + 2] - zs;
        dist += sqrt(dx * dx + dy * dy + dz * dz);
        nbs++;
    }
    const double r = sum - m.diag64[site] * m.phi64[site] - m.q64[site];
    const double d = m.diag64[site];
    double sigma = d > 0.0 ? fabs(r) / d : 0.0;
    if (!(sigma > 1e-30)) sigma = 1e-30;
    scale[0] = (float)sigma;
    scale[1] = nbs > 0 ? (float)(dist / nbs) : 1.0f;
}

// features, ELL rows and (for sample collection) the start potentials; one
// warp per cell, its lanes over the cell's neighbours (warp sums, and the
// ELL row compacted in CSR order by ballots)
__global__ void k_ball_features(DevMesh m, int site, int hops, int D, const int32_t* nodes, const int8_t* level,
                                const int32_t* count, const int32_t* localOf, const float* scale, float* X,
                                int32_t* ellCol, float* ellW, double* phiStart) {
    const int n = *count;
    const int lane = threadIdx.x & 31;
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= n) return;
    const int g = nodes[t];
    const double sigma = scale[0], ell = scale[1];
    const double xs = m.xyz[3 * site], ys = m.xyz[3 * site + 1], zs = m.xyz[3 * site + 2];
    const double dx = m.xyz[3 * g] - xs, dy = m.xyz[3 * g + 1] - ys, dz = m.xyz[3 * g + 2] - zs;
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    double sum = 0.0, fixedC = 0.0, allC = 0.0;
    int k = 0;  // ELL entries written so far (the same in every lane)
    const double dg = m.diag64[g];
    const int q0 = m.row_ptr[g], q1 = m.row_ptr[g + 1];
    for (int base = q0; base < q1; base += 32) {
        const int q = base + lane;
        int lj = -1;
        double c = 0.0;
        if (q < q1) {
            const int j = m.col[q];
            c = m.ceff64[q];
            sum += c * m.phi64[j];
            const double c64 = m.c64[q];
            allC += c64;
            if (m.flags[j] & F_DIRICHLET) fixedC += c64;
            lj = localOf[j];
        }
        const bool take = q < q1 && lj >= 0 && lj < n && c != 0.0;
        const unsigned mask = __ballot_sync(0xffffffffu, take);
        const int at = k + __popc(mask & ((1u << lane) - 1u));
        if (take && at < D) {
            ellCol[(size_t)t * D + at] = lj;
            ellW[(size_t)t * D + at] = dg > 0.0 ? (float)(c / dg) : 0.0f;
        }
        k = min(D, k + __popc(mask));
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        allC += __shfl_xor_sync(0xffffffffu, allC, o);
        fixedC += __shfl_xor_sync(0xffffffffu, fixedC, o);
    }
    for (int e = k + lane; e < D; e += 32) {
        ellCol[(size_t)t * D + e] = -1;
        ellW[(size_t)t * D + e] = 0.0f;
    }
    if (lane != 0) return;
    const double r = sum - dg * m.phi64[g] - m.q64[g];
    float* x = X + (size_t)t * kFeat;
    x[0] = (float)(dx / ell);
    x[1] = (float)(dy / ell);
    x[2] = (float)(dz / ell);
    x[3] = (float)(dist / ell);
    x[4] = (float)level[t] / (float)hops;
    x[5] = g == site ? 1.0f : 0.0f;
    x[6] = (m.flags[g] & F_NEUMANN) ? 1.0f : 0.0f;
    x[7] = allC > 0.0 ? (float)(fixedC / allC) : 0.0f;
    x[8] = dg > 0.0 ? (float)(r / (dg * sigma)) : 0.0f;
    x[9] = (float)(m.phi64[g] - m.phi64[site]);
    x[10] = (dg > 0.0 && m.diag64[site] > 0.0) ? (float)log(dg / m.diag64[site]) : 0.0f;
    x[11] = (float)(log10(sigma) / 10.0);
    x[12] = x[13] = x[14] = x[15] = 0.0f;
    if (phiStart) phiStart[t] = m.phi64[g];
}

// BF16 input block: features in columns 0..15, zeros to 128; also the
// transposed copy (column-major) for the weight gradient
// nDev (may be null): the graph's row count on the device, which caps n
__global__ void k_input_bf16(const float* X, int n, const int32_t* nDev, int npad, __nv_bfloat16* Z,
                             __nv_bfloat16* ZT) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kCat) return;
    if (nDev && *nDev < n) n = *nDev;
    const int i = t / kCat, f = t % kCat;
    const float v = (i < n && f < kFeat) ? X[(size_t)i * kFeat + f] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    Z[t] = b;
    ZT[(size_t)f * npad + i] = b;
}

// u = C + b; h = hPrev + relu(u) (hPrev may be null)
__global__ void k_bias_act(const float* C, const float* b, const float* hPrev, float* u, float* h, int npad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kHid) return;
    const float v = C[t] + b[t % kHid];
    u[t] = v;
    h[t] = (hPrev ? hPrev[t] : 0.0f) + fmaxf(v, 0.0f);
}

// z = [h, A h] in BF16 (row-major and transposed)
__global__ void k_message_concat(const float* h, const int32_t* ellCol, const float* ellW, int D, int n,
                                 const int32_t* nDev, int npad, __nv_bfloat16* Z, __nv_bfloat16* ZT) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kHid) return;
    if (nDev && *nDev < n) n = *nDev;
    const int i = t / kHid, f = t % kHid;
    float hv = 0.0f, mv = 0.0f;
    if (i < n) {
        hv = h[t];
        for (int k = 0; k < D; k++) {
            const int j = ellCol[(size_t)i * D + k];
            if (j < 0) break;
            mv += ellW[(size_t)i * D + k] * h[(size_t)j * kHid + f];
        }
    }
    const __nv_bfloat16 hb = __float2bfloat16_rn(hv), mbv = __float2bfloat16_rn(mv);
    Z[(size_t)i * kCat + f] = hb;
    Z[(size_t)i * kCat + kHid + f] = mbv;
    ZT[(size_t)f * npad + i] = hb;
    ZT[(size_t)(kHid + f) * npad + i] = mbv;
}

__global__ void k_readout(const float* h, const float* w, const float* b, int n, const int32_t* nDev, float* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (nDev && *nDev < n) n = *nDev;
    if (i >= n) return;
    float s = b[0];
    for (int f = 0; f < kHid; f++) s += h[(size_t)i * kHid + f] * w[f];
    y[i] = s;
}

// loss = sum (y - t)^2 / count over the nodes; dy = 2 (y - t) / count
__global__ void k_loss(const float* y, const float* tgt, int n, float invCount, float* dy, float* loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < n) {
        const float e = y[i] - tgt[i];
        dy[i] = 2.0f * e * invCount;
        l = e * e * invCount;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// gradients of the readout; dh = dy w (zero on padding rows)
__global__ void k_readout_back(const float* h, const float* dy, const float* w, int n, int npad, float* gw, float* gb,
                               float* dh) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kHid) return;
    const int i = t / kHid, f = t % kHid;
    const float d = i < n ? dy[i] : 0.0f;
    dh[t] = d * w[f];
    if (d != 0.0f) {
        atomicAdd(&gw[f], d * h[t]);
        if (f == 0) atomicAdd(gb, d);
    }
}

// du = dh * [u > 0] (BF16, row-major and transposed); gb += sum du
__global__ void k_act_back(const float* dh, const float* u, int npad, __nv_bfloat16* DU, __nv_bfloat16* DUT,
                           float* gb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kHid) return;
    const int i = t / kHid, f = t % kHid;
    const float d = u[t] > 0.0f ? dh[t] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(d);
    DU[t] = b;
    DUT[(size_t)f * npad + i] = b;
    if (d != 0.0f) atomicAdd(&gb[f], d);
}

// dhPrev = dh + dz[:, :64]; the message half flows back along the edges:
// dhPrev[j] += a_ij dz[i, 64 + f]
__global__ void k_message_back(const float* dh, const float* dz, const int32_t* ellCol, const float* ellW, int D, int n,
                               int npad, float* dhPrev) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npad * kHid) return;
    const int i = t / kHid, f = t % kHid;
    atomicAdd(&dhPrev[t], dh[t] + dz[(size_t)i * kCat + f]);
    if (i >= n) return;
    const float dm = dz[(size_t)i * kCat + kHid + f];
    if (dm == 0.0f) return;
    for (int k = 0; k < D; k++) {
        const int j = ellCol[(size_t)i * D + k];
        if (j < 0) break;
        atomicAdd(&dhPrev[(size_t)j * kHid + f], ellW[(size_t)i * D + k] * dm);
    }
}

// Adam on the FP32 parameters
__global__ void k_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const float gt = g[t];
    const float a = b1 * m1[t] + (1.0f - b1) * gt;
    const float v = b2 * m2[t] + (1.0f - b2) * gt * gt;
    m1[t] = a;
    m2[t] = v;
    p[t] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// BF16 copies of one layer's weights: W (in x out) and W^T (out x in)
__global__ void k_weights_bf16(const float* W, __nv_bfloat16* Wb, __nv_bfloat16* WTb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kCat * kHid) return;
    const int i = t / kHid, o = t % kHid;
    const __nv_bfloat16 b = __float2bfloat16_rn(W[t]);
    Wb[t] = b;
    WTb[(size_t)o * kCat + i] = b;
}

// phi += sigma y on the graph's cells (and on the recorded correction of the
// V rows, so that the next event recycles the whole correction)
__global__ void k_apply_prediction(DevMesh m, const int32_t* nodes, const int32_t* count, const float* y,
                                   const float* scale, float gain, const int32_t* slotOf, float* hist) {
    const int n = *count;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int g = nodes[t];
    const float d = gain * scale[0] * y[t];
    m.phi64[g] += (double)d;
    if (hist) {
        const int s = slotOf[g];
        if (s >= 0) hist[s] += d;
    }
}

// Damped Jacobi sweeps over the graph's cells after the prediction, every
// other cell held: phi_i += omega ((sum_j ceff_ij phi_j - q_i) / diag_i -
// phi_i) (computePotential's update, grid_3d.cpp:1317-1371).  One CTA: each
// sweep computes every cell's new value from the old ones, then writes them
// (the same result for any thread count).  The change joins the recorded
// correction of the cells' V slots when hist is given.  The graph has at
// most cap <= kRefineMax cells.
constexpr int kRefineMax = 4096;
__global__ void __launch_bounds__(1024) k_local_refine(DevMesh m, const int32_t* nodes, const int32_t* count,
                                                       int cap, int sweeps, float omega, const int32_t* slotOf,
                                                       float* hist) {
    extern __shared__ double refineShared[];  // start[cap], next[cap]
    double* start = refineShared;
    double* next = refineShared + cap;
    const int n = min(*count, cap);
    for (int t = threadIdx.x; t < n; t += blockDim.x) start[t] = m.phi64[nodes[t]];
    __syncthreads();
    for (int sw = 0; sw < sweeps; sw++) {
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
            const int i = nodes[t];
            const double d = m.diag64[i];
            double sum = 0.0;
            for (int q = m.row_ptr[i]; q < m.row_ptr[i + 1]; q++) sum += m.ceff64[q] * m.phi64[m.col[q]];
            const double pi = m.phi64[i];
            next[t] = d > 0.0 ? pi + (double)omega * ((sum - m.q64[i]) / d - pi) : pi;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < n; t += blockDim.x) m.phi64[nodes[t]] = next[t];
        __syncthreads();
    }
    if (hist)
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
            const int sl = slotOf[nodes[t]];
            if (sl >= 0) hist[sl] += (float)(m.phi64[nodes[t]] - start[t]);
        }
}

// training target: (phi_final - phi_start) / sigma
__global__ void k_collect_target(DevMesh m, const int32_t* nodes, const int32_t* count, const double* phiStart,
                                 const float* scale, float* tgt) {
    const int n = *count;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    tgt[t] = (float)((m.phi64[nodes[t]] - phiStart[t]) / (double)scale[0]);
}

// ELL columns of a sample shifted to its place in a batch
__global__ void k_shift_cols(int32_t* col, int count, int shift) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count && col[t] >= 0) col[t] += shift;
}

inline unsigned nblk(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

}  // namespace

bool gemm_shape_ok(int M, int N, int K) { return M > 0 && M % 128 == 0 && (N == 64 || N == 128) && K > 0 && K % 64 == 0; }

cudaError_t launch_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K, int* status,
                             cudaStream_t s) {
    static std::atomic<uint64_t> attrSet{0};
    cudaError_t e = once_per_device(attrSet, [] {
        cudaError_t r = cudaFuncSetAttribute(k_gemm_bf16<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
        if (r == cudaSuccess)
            r = cudaFuncSetAttribute(k_gemm_bf16<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
        return r;
    });
    if (e != cudaSuccess) return e;
    const auto* a = static_cast<const __nv_bfloat16*>(A);
    const auto* b = static_cast<const __nv_bfloat16*>(B);
    count_launch();
    if (N == 64)
        k_gemm_bf16<64><<<M / 128, kGemmThreads, kGemmSmem, s>>>(a, b, C, M, K, status);
    else
        k_gemm_bf16<128><<<M / 128, kGemmThreads, kGemmSmem, s>>>(a, b, C, M, K, status);
    return cudaGetLastError();
}

void launch_ball_bfs(const DevMesh& m, int site, int hops, int cap, int32_t* nodes, int8_t* level, int32_t* count,
                     int32_t* localOf, cudaStream_t s) {
    count_launch();
    k_ball_bfs<<<1, 512, 0, s>>>(m, site, hops, cap, nodes, level, count, localOf);
}
void launch_ball_reset(const int32_t* nodes, const int32_t* count, int32_t* localOf, int cap, cudaStream_t s) {
    count_launch();
    k_ball_reset<<<nblk(cap), 256, 0, s>>>(nodes, count, localOf);
}
void launch_ball_features(const DevMesh& m, int site, int hops, int D, const int32_t* nodes, const int8_t* level,
                          const int32_t* count, const int32_t* localOf, float* scale, float* X, int32_t* ellCol,
                          float* ellW, double* phiStart, int cap, cudaStream_t s) {
    count_launch();
    k_site_scale<<<1, 32, 0, s>>>(m, site, scale);
    count_launch();
    k_ball_features<<<nblk((long long)cap * 32), 256, 0, s>>>(m, site, hops, D, nodes, level, count, localOf, scale, X,
                                                               ellCol, ellW,
                                               phiStart);
}
void launch_input_bf16(const float* X, int n, int npad, void* Z, void* ZT, cudaStream_t s, const int32_t* nDev) {
    count_launch();
    k_input_bf16<<<nblk((long long)npad * kCat), 256, 0, s>>>(X, n, nDev, npad, static_cast<__nv_bfloat16*>(Z),
                                                                static_cast<__nv_bfloat16*>(ZT));
}
void launch_bias_act(const float* C, const float* b, const float* hPrev, float* u, float* h, int npad,
                     cudaStream_t s) {
    count_launch();
    k_bias_act<<<nblk((long long)npad * kHid), 256, 0, s>>>(C, b, hPrev, u, h, npad);
}
void launch_message_concat(const float* h, const int32_t* ellCol, const float* ellW, int D, int n, int npad, void* Z,
                           void* ZT, cudaStream_t s, const int32_t* nDev) {
    count_launch();
    k_message_concat<<<nblk((long long)npad * kHid), 256, 0, s>>>(h, ellCol, ellW, D, n, nDev, npad,
                                                                    static_cast<__nv_bfloat16*>(Z),
                                                                    static_cast<__nv_bfloat16*>(ZT));
}
void launch_readout(const float* h, const float* w, const float* b, int n, float* y, cudaStream_t s,
                    const int32_t* nDev) {
    count_launch();
    k_readout<<<nblk(n), 256, 0, s>>>(h, w, b, n, nDev, y);
}
void launch_loss(const float* y, const float* tgt, int n, float invCount, float* dy, float* loss, cudaStream_t s) {
    count_launch();
    k_loss<<<nblk(n), 256, 0, s>>>(y, tgt, n, invCount, dy, loss);
}
void launch_readout_back(const float* h, const float* dy, const float* w, int n, int npad, float* gw, float* gb,
                         float* dh, cudaStream_t s) {
    count_launch();
    k_readout_back<<<nblk((long long)npad * kHid), 256, 0, s>>>(h, dy, w, n, npad, gw, gb, dh);
}
void launch_act_back(const float* dh, const float* u, int npad, void* DU, void* DUT, float* gb, cudaStream_t s) {
    count_launch();
    k_act_back<<<nblk((long long)npad * kHid), 256, 0, s>>>(dh, u, npad, static_cast<__nv_bfloat16*>(DU),
                                                              static_cast<__nv_bfloat16*>(DUT), gb);
}
void launch_message_back(const float* dh, const float* dz, const int32_t* ellCol, const float* ellW, int D, int n,
                         int npad, float* dhPrev, cudaStream_t s) {
    count_launch();
    k_message_back<<<nblk((long long)npad * kHid), 256, 0, s>>>(dh, dz, ellCol, ellW, D, n, npad, dhPrev);
}
void launch_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2, float eps,
                 float c1, float c2, cudaStream_t s) {
    count_launch();
    k_adam<<<nblk(count), 256, 0, s>>>(p, g, m1, m2, count, lr, b1, b2, eps, c1, c2);
}
void launch_weights_bf16(const float* W, void* Wb, void* WTb, cudaStream_t s) {
    count_launch();
    k_weights_bf16<<<nblk(kCat * kHid), 256, 0, s>>>(W, static_cast<__nv_bfloat16*>(Wb),
                                                     static_cast<__nv_bfloat16*>(WTb));
}
void launch_apply_prediction(const DevMesh& m, const int32_t* nodes, const int32_t* count, const float* y,
                             const float* scale, float gain, const int32_t* slotOf, float* hist, int cap,
                             cudaStream_t s) {
    count_launch();
    k_apply_prediction<<<nblk(cap), 256, 0, s>>>(m, nodes, count, y, scale, gain, slotOf, hist);
}
void launch_local_refine(const DevMesh& m, const int32_t* nodes, const int32_t* count, int cap, int sweeps,
                         float omega, const int32_t* slotOf, float* hist, cudaStream_t s) {
    if (sweeps <= 0 || cap <= 0 || cap > kRefineMax) return;
    static std::atomic<uint64_t> opted{0};
    once_per_device(opted, [] {
        return cudaFuncSetAttribute(k_local_refine, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(2 * sizeof(double) * kRefineMax));
    });
    count_launch();
    k_local_refine<<<1, 1024, 2 * sizeof(double) * (size_t)cap, s>>>(m, nodes, count, cap, sweeps, omega, slotOf,
                                                                     hist);
}
void launch_collect_target(const DevMesh& m, const int32_t* nodes, const int32_t* count, const double* phiStart,
                           const float* scale, float* tgt, int cap, cudaStream_t s) {
    count_launch();
    k_collect_target<<<nblk(cap), 256, 0, s>>>(m, nodes, count, phiStart, scale, tgt);
}
void launch_shift_cols(int32_t* col, int count, int shift, cudaStream_t s) {
    if (count <= 0 || shift == 0) return;
    count_launch();
    k_shift_cols<<<nblk(count), 256, 0, s>>>(col, count, shift);
}

}  // namespace tgd
