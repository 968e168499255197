// Learned near-field warm start: the network's parameters, its training on
// samples the solver collects, and its inference inside tg_solve.
//
// A sample is one removal: the graph of free cells within `hops` steps of
// the removed cell, 16 features per cell taken from the state the solve
// starts from (after the removal and, with a recycled start, the previous
// event's correction), and the target (phi_final - phi_start) / sigma on the
// same cells, where phi_final is the potential the solve converged to.  Training minimises the mean squared error over the cells of a batch
// of samples with Adam; forward and backward GEMMs run on the tensor cores
// (mpnn.cu).  Inference adds sigma * y to the potentials (and to the
// recorded correction) before the CG starts; the solve still ends at its
// tolerance, so a poor prediction costs iterations, never accuracy.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/tapsim_gpu.h"
#include "kernels.cuh"
#include "learn.h"

namespace tgapi {
void set_process_error(const std::string& msg);
}

using namespace tgd;

namespace {

constexpr int kFeat = 16, kHid = 64, kCat = 128, kLayers = 5;  // input layer + four message layers
constexpr int kLayerParams = kCat * kHid + kHid;
constexpr int kParams = kLayers * kLayerParams + kHid + 1;

template <typename T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        release();
        n = count;
        return count ? cudaMalloc(&p, count * sizeof(T)) : cudaSuccess;
    }
    // grows to at least `count`, keeping the contents (callers make sure no
    // work on the buffer is in flight)
    cudaError_t grow(size_t count) {
        if (count <= n) return cudaSuccess;
        const size_t cap = std::max(count, 2 * n + 1024);
        T* q = nullptr;
        cudaError_t e = cudaMalloc(&q, cap * sizeof(T));
        if (e != cudaSuccess) return e;
        if (p && n) e = cudaMemcpy(q, p, n * sizeof(T), cudaMemcpyDeviceToDevice);
        if (p) cudaFree(p);
        p = q;
        n = cap;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

inline int roundup128(int n) { return (n + 127) / 128 * 128; }

}  // namespace

struct tg_learner {
    int hops = 6, cap = 4096, D = 32;
    int device = -1;    // current at tg_learner_create; made current by every entry point
    float gain = 1.0f;  // multiplier of the prediction added in tg_solve
    int refine = 0;     // damped Jacobi sweeps over the graph's cells after the prediction
    std::string err;
    cudaStream_t stream = nullptr;
    // parameters, gradients, Adam moments (FP32), BF16 weight copies
    Buf<float> P, G, M1, M2;
    Buf<__nv_bfloat16> Wb, WTb;  // per layer: W (in x out) and W^T (out x in)
    int64_t adamStep = 0;
    Buf<int> status;
    // one graph (inference and collection)
    Buf<int32_t> nodes, count, localOf;
    Buf<int8_t> level;
    Buf<float> scale, X, ellW;
    Buf<int32_t> ellCol;
    Buf<double> phiStart;
    size_t meshNodes = 0;
    bool collecting = false;
    // activations for up to `npadMax` rows
    int npadMax = 0;
    Buf<__nv_bfloat16> Z, ZT, DU, DUT;  // Z, ZT: one block per layer
    Buf<float> U, H, C, y, dy, dH, dHp, loss;
    // batch staging
    Buf<float> bX, bW, bT;
    Buf<int32_t> bCol;
    // samples: concatenated per-cell data, host index
    Buf<float> sX, sW, sT;
    Buf<int32_t> sCol;
    std::vector<int64_t> sOff;  // cell offset of each sample
    std::vector<int32_t> sLen;
    int64_t sNodes = 0;

    float* Wl(int l) { return P.p + (size_t)l * kLayerParams; }
    float* bl(int l) { return P.p + (size_t)l * kLayerParams + kCat * kHid; }
    float* gWl(int l) { return G.p + (size_t)l * kLayerParams; }
    float* gbl(int l) { return G.p + (size_t)l * kLayerParams + kCat * kHid; }
    float* wout() { return P.p + (size_t)kLayers * kLayerParams; }
    float* bout() { return wout() + kHid; }
    __nv_bfloat16* Wbl(int l) { return Wb.p + (size_t)l * kCat * kHid; }
    __nv_bfloat16* WTbl(int l) { return WTb.p + (size_t)l * kCat * kHid; }
    __nv_bfloat16* Zl(int l) { return Z.p + (size_t)l * npadMax * kCat; }
    __nv_bfloat16* ZTl(int l) { return ZT.p + (size_t)l * npadMax * kCat; }
    float* Ul(int l) { return U.p + (size_t)l * npadMax * kHid; }
    float* Hl(int l) { return H.p + (size_t)l * npadMax * kHid; }
};

namespace {

int lfail(tg_learner* L, int code, const std::string& msg) {
    if (L) L->err = msg;
    tgapi::set_process_error(msg);
    return code;
}

#define LCK(expr)                                                                                          \
    do {                                                                                                   \
        const cudaError_t _e = (expr);                                                                     \
        if (_e != cudaSuccess)                                                                             \
            return lfail(L, TG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));             \
    } while (0)

int ensure_rows(tg_learner* L, int npad) {
    if (npad <= L->npadMax) return TG_OK;
    const int m = roundup128(std::max(npad, 2 * L->npadMax));
    L->npadMax = m;
    LCK(L->Z.alloc((size_t)kLayers * m * kCat));
    LCK(L->ZT.alloc((size_t)kLayers * m * kCat));
    LCK(L->DU.alloc((size_t)m * kHid));
    LCK(L->DUT.alloc((size_t)m * kHid));
    LCK(L->U.alloc((size_t)kLayers * m * kHid));
    LCK(L->H.alloc((size_t)kLayers * m * kHid));
    LCK(L->C.alloc((size_t)m * kCat));
    LCK(L->y.alloc(m));
    LCK(L->dy.alloc(m));
    LCK(L->dH.alloc((size_t)m * kHid));
    LCK(L->dHp.alloc((size_t)m * kHid));
    LCK(L->bX.alloc((size_t)m * kFeat));
    LCK(L->bW.alloc((size_t)m * L->D));
    LCK(L->bCol.alloc((size_t)m * L->D));
    LCK(L->bT.alloc(m));
    return TG_OK;
}

int refresh_bf16(tg_learner* L) {
    for (int l = 0; l < kLayers; l++) launch_weights_bf16(L->Wl(l), L->Wbl(l), L->WTbl(l), L->stream);
    LCK(cudaGetLastError());
    return TG_OK;
}

int check_status(tg_learner* L, const char* where) {
    LCK(cudaStreamSynchronize(L->stream));
    int st = 0;
    LCK(cudaMemcpy(&st, L->status.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (st == 0) return TG_OK;
    LCK(cudaMemset(L->status.p, 0, sizeof(int)));
    return lfail(L, (st & S_TIMEOUT) ? TG_ERR_TIMEOUT : TG_ERR_CUDA, std::string(where) + ": device status");
}

int gemm(tg_learner* L, const void* A, const void* B, float* C, int M, int N, int K) {
    if (!gemm_shape_ok(M, N, K)) return lfail(L, TG_ERR_ARGUMENT, "learner: GEMM shape");
    LCK(launch_gemm_bf16(A, B, C, M, N, K, L->status.p, L->stream));
    return TG_OK;
}

// Forward pass over n rows (features X, ELL col/w); the readout lands in L->y.
// nDev (may be null): the row count on the device, at most n; the rows
// beyond it enter the GEMMs as zeros, so that n (the graph's capacity) sizes
// the launches without the host reading the count.
int forward(tg_learner* L, const float* X, const int32_t* col, const float* w, int n, const int32_t* nDev = nullptr) {
    const int npad = roundup128(std::max(n, 1));
    int rc = ensure_rows(L, npad);
    if (rc != TG_OK) return rc;
    cudaStream_t s = L->stream;
    launch_input_bf16(X, n, npad, L->Zl(0), L->ZTl(0), s, nDev);
    if ((rc = gemm(L, L->Zl(0), L->WTbl(0), L->C.p, npad, kHid, kCat)) != TG_OK) return rc;
    launch_bias_act(L->C.p, L->bl(0), nullptr, L->Ul(0), L->Hl(0), npad, s);
    for (int l = 1; l < kLayers; l++) {
        launch_message_concat(L->Hl(l - 1), col, w, L->D, n, npad, L->Zl(l), L->ZTl(l), s, nDev);
        if ((rc = gemm(L, L->Zl(l), L->WTbl(l), L->C.p, npad, kHid, kCat)) != TG_OK) return rc;
        launch_bias_act(L->C.p, L->bl(l), L->Hl(l - 1), L->Ul(l), L->Hl(l), npad, s);
    }
    launch_readout(L->Hl(kLayers - 1), L->wout(), L->bout(), n, L->y.p, s, nDev);
    LCK(cudaGetLastError());
    return TG_OK;
}

// Loss and gradients (into L->G) of the rows forwarded last, against tgt
int backward(tg_learner* L, const int32_t* col, const float* w, const float* tgt, int n, float* lossOut) {
    const int npad = roundup128(std::max(n, 1));
    cudaStream_t s = L->stream;
    LCK(cudaMemsetAsync(L->G.p, 0, sizeof(float) * kParams, s));
    LCK(cudaMemsetAsync(L->loss.p, 0, sizeof(float), s));
    launch_loss(L->y.p, tgt, n, 1.0f / (float)std::max(n, 1), L->dy.p, L->loss.p, s);
    launch_readout_back(L->Hl(kLayers - 1), L->dy.p, L->wout(), n, npad, L->gWl(kLayers) /* w_out */,
                        L->gWl(kLayers) + kHid /* b_out */, L->dH.p, s);
    int rc;
    for (int l = kLayers - 1; l >= 0; l--) {
        launch_act_back(L->dH.p, L->Ul(l), npad, L->DU.p, L->DUT.p, L->gbl(l), s);
        // dW_l = z_l^T du   (128 x 64, K = rows)
        if ((rc = gemm(L, L->ZTl(l), L->DUT.p, L->gWl(l), kCat, kHid, npad)) != TG_OK) return rc;
        if (l == 0) break;
        // dz = du W_l^T     (rows x 128, K = 64)
        if ((rc = gemm(L, L->DU.p, L->Wbl(l), L->C.p, npad, kCat, kHid)) != TG_OK) return rc;
        LCK(cudaMemsetAsync(L->dHp.p, 0, sizeof(float) * (size_t)npad * kHid, s));
        launch_message_back(L->dH.p, L->C.p, col, w, L->D, n, npad, L->dHp.p, s);
        std::swap(L->dH.p, L->dHp.p);
    }
    LCK(cudaGetLastError());
    if (lossOut) LCK(cudaMemcpyAsync(lossOut, L->loss.p, sizeof(float), cudaMemcpyDeviceToHost, s));
    return TG_OK;
}

// Copies samples `idx` into the batch staging buffers; returns the rows
int stage_batch(tg_learner* L, const std::vector<int>& idx, int* rowsOut) {
    int64_t rows = 0;
    for (int k : idx) rows += L->sLen[k];
    if (rows > (1 << 22)) return lfail(L, TG_ERR_ARGUMENT, "learner: batch too large");
    int rc = ensure_rows(L, roundup128((int)std::max<int64_t>(rows, 1)));
    if (rc != TG_OK) return rc;
    cudaStream_t s = L->stream;
    int64_t at = 0;
    for (int k : idx) {
        const int64_t o = L->sOff[k];
        const int len = L->sLen[k];
        LCK(cudaMemcpyAsync(L->bX.p + at * kFeat, L->sX.p + o * kFeat, sizeof(float) * len * kFeat,
                            cudaMemcpyDeviceToDevice, s));
        LCK(cudaMemcpyAsync(L->bW.p + at * L->D, L->sW.p + o * L->D, sizeof(float) * len * L->D,
                            cudaMemcpyDeviceToDevice, s));
        LCK(cudaMemcpyAsync(L->bCol.p + at * L->D, L->sCol.p + o * L->D, sizeof(int32_t) * len * L->D,
                            cudaMemcpyDeviceToDevice, s));
        LCK(cudaMemcpyAsync(L->bT.p + at, L->sT.p + o, sizeof(float) * len, cudaMemcpyDeviceToDevice, s));
        launch_shift_cols(L->bCol.p + at * L->D, len * L->D, (int)at, s);
        at += len;
    }
    *rowsOut = (int)rows;
    return TG_OK;
}

// Builds the graph of `site` from the current state on stream s; with nOut
// its size is read back (a synchronisation), otherwise it stays on the
// device (L->count)
int build_graph(tg_learner* L, const DevMesh& m, int site, cudaStream_t s, int* nOut) {
    if ((size_t)m.n != L->meshNodes) return lfail(L, TG_ERR_ARGUMENT, "learner: attached to another mesh");
    launch_ball_bfs(m, site, L->hops, L->cap, L->nodes.p, L->level.p, L->count.p, L->localOf.p, s);
    launch_ball_features(m, site, L->hops, L->D, L->nodes.p, L->level.p, L->count.p, L->localOf.p, L->scale.p, L->X.p,
                         L->ellCol.p, L->ellW.p, L->collecting ? L->phiStart.p : nullptr, L->cap, s);
    launch_ball_reset(L->nodes.p, L->count.p, L->localOf.p, L->cap, s);
    if (!nOut) return TG_OK;
    int n = 0;
    LCK(cudaMemcpyAsync(&n, L->count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    LCK(cudaStreamSynchronize(s));
    *nOut = n;
    return TG_OK;
}

}  // namespace

// ---- hooks called by tg_solve (handle.cu) ----

int learner_device(const tg_learner* L) { return L->device; }

int learner_attach_mesh(tg_learner* L, size_t meshNodes, int maxRow) {
    if (maxRow > L->D)
        return lfail(L, TG_ERR_ARGUMENT, "learner: graph width " + std::to_string(L->D) +
                                             " below the mesh's row length " + std::to_string(maxRow));
    if (L->meshNodes == meshNodes) return TG_OK;
    LCK(L->localOf.alloc(meshNodes));
    LCK(cudaMemset(L->localOf.p, 0xFF, sizeof(int32_t) * meshNodes));
    L->meshNodes = meshNodes;
    return TG_OK;
}

void learner_graph_cells(const tg_learner* L, const int32_t** nodes, const int32_t** count, int* capacity) {
    *nodes = L->nodes.p;
    *count = L->count.p;
    *capacity = L->cap;
}

int learner_predict(tg_learner* L, const DevMesh& m, int site, cudaStream_t s, bool collect, bool predict,
                    const int32_t* slotOf, float* hist) {
    const cudaStream_t own = L->stream;
    L->stream = s;
    L->collecting = collect;
    // the graph's size is read back only to store a sample; a prediction
    // alone runs over the graph's capacity with the size on the device
    int n = 0;
    int rc = build_graph(L, m, site, s, collect ? &n : nullptr);
    if (rc == TG_OK && collect) {
        // the sample's features are the state before any prediction; the
        // stream is idle here (build_graph synchronised it)
        const int64_t o = L->sNodes;
        if (L->sX.grow((size_t)(o + n) * kFeat) != cudaSuccess || L->sW.grow((size_t)(o + n) * L->D) != cudaSuccess ||
            L->sCol.grow((size_t)(o + n) * L->D) != cudaSuccess || L->sT.grow((size_t)(o + n)) != cudaSuccess)
            rc = lfail(L, TG_ERR_CUDA, "learner: sample storage");
        if (rc == TG_OK) {
            cudaMemcpyAsync(L->sX.p + o * kFeat, L->X.p, sizeof(float) * n * kFeat, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(L->sW.p + o * L->D, L->ellW.p, sizeof(float) * n * L->D, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(L->sCol.p + o * L->D, L->ellCol.p, sizeof(int32_t) * n * L->D, cudaMemcpyDeviceToDevice, s);
        }
    }
    if (rc == TG_OK && predict) {
        // gain 0: no prediction, the sweeps alone (to isolate the network)
        if (L->gain > 0.0f) {
            rc = collect ? forward(L, L->X.p, L->ellCol.p, L->ellW.p, n)
                         : forward(L, L->X.p, L->ellCol.p, L->ellW.p, L->cap, L->count.p);
            if (rc == TG_OK)
                launch_apply_prediction(m, L->nodes.p, L->count.p, L->y.p, L->scale.p, L->gain, slotOf, hist, L->cap,
                                        s);
        }
        if (rc == TG_OK) launch_local_refine(m, L->nodes.p, L->count.p, L->cap, L->refine, 0.8f, slotOf, hist, s);
    }
    L->stream = own;
    if (rc == TG_OK && cudaGetLastError() != cudaSuccess) rc = lfail(L, TG_ERR_CUDA, "learner: launch");
    if (rc != TG_OK) L->collecting = false;
    return rc;
}

void learner_collect_cancel(tg_learner* L) {
    if (L) L->collecting = false;
}

int learner_collect_end(tg_learner* L, const DevMesh& m, cudaStream_t s) {
    if (!L->collecting) return TG_OK;
    L->collecting = false;
    int n = 0;
    LCK(cudaMemcpyAsync(&n, L->count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    LCK(cudaStreamSynchronize(s));
    const int64_t o = L->sNodes;
    launch_collect_target(m, L->nodes.p, L->count.p, L->phiStart.p, L->scale.p, L->sT.p + o, L->cap, s);
    LCK(cudaGetLastError());
    LCK(cudaStreamSynchronize(s));
    L->sOff.push_back(o);
    L->sLen.push_back(n);
    L->sNodes += n;
    return TG_OK;
}

extern "C" {

int tg_learner_create(int32_t hops, int32_t max_nodes, int32_t ell_width, uint64_t seed, tg_learner** out) {
    if (!out || hops < 1 || hops > 32 || max_nodes < 128 || max_nodes > (1 << 20) || ell_width < 4 ||
        ell_width > 256)
        return lfail(nullptr, TG_ERR_ARGUMENT, "tg_learner_create: bad argument");
    tg_learner* L = new tg_learner();
    if (cudaGetDevice(&L->device) != cudaSuccess) {
        delete L;
        return lfail(nullptr, TG_ERR_CUDA, "tg_learner_create: no current CUDA device");
    }
    L->hops = hops;
    L->cap = max_nodes;
    L->D = ell_width;
    auto fin = [&](int rc) -> int {
        if (rc != TG_OK) {
            tg_learner_destroy(L);
            return rc;
        }
        *out = L;
        return (int)TG_OK;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking);
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(L->P.alloc(kParams));
    chk(L->G.alloc(kParams));
    chk(L->M1.alloc(kParams));
    chk(L->M2.alloc(kParams));
    chk(L->Wb.alloc((size_t)kLayers * kCat * kHid));
    chk(L->WTb.alloc((size_t)kLayers * kCat * kHid));
    chk(L->status.alloc(1));
    chk(L->nodes.alloc(max_nodes));
    chk(L->level.alloc(max_nodes));
    chk(L->count.alloc(1));
    chk(L->scale.alloc(2));
    chk(L->X.alloc((size_t)max_nodes * kFeat));
    chk(L->ellW.alloc((size_t)max_nodes * ell_width));
    chk(L->ellCol.alloc((size_t)max_nodes * ell_width));
    chk(L->phiStart.alloc(max_nodes));
    chk(L->loss.alloc(1));
    if (e != cudaSuccess) return fin(lfail(L, TG_ERR_CUDA, std::string("tg_learner_create: ") + cudaGetErrorString(e)));
    // He-scaled normal weights (rows of the input layer beyond the 16
    // features stay zero), zero biases, a small readout
    std::vector<float> p(kParams, 0.0f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int l = 0; l < kLayers; l++) {
        const int fanIn = l == 0 ? kFeat : kCat;
        const float sd = std::sqrt(2.0f / fanIn);
        for (int i = 0; i < fanIn; i++)
            for (int o = 0; o < kHid; o++) p[(size_t)l * kLayerParams + i * kHid + o] = sd * nd(rng);
    }
    for (int o = 0; o < kHid; o++) p[(size_t)kLayers * kLayerParams + o] = 0.01f * nd(rng);
    chk(cudaMemcpy(L->P.p, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice));
    chk(cudaMemset(L->M1.p, 0, sizeof(float) * kParams));
    chk(cudaMemset(L->M2.p, 0, sizeof(float) * kParams));
    chk(cudaMemset(L->status.p, 0, sizeof(int)));
    if (e != cudaSuccess) return fin(lfail(L, TG_ERR_CUDA, std::string("tg_learner_create: ") + cudaGetErrorString(e)));
    int rc = refresh_bf16(L);
    if (rc == TG_OK) rc = check_status(L, "tg_learner_create");
    return fin(rc);
}

void tg_learner_destroy(tg_learner* L) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L) return;
    if (L->stream) cudaStreamSynchronize(L->stream);
    L->P.release(); L->G.release(); L->M1.release(); L->M2.release(); L->Wb.release(); L->WTb.release();
    L->status.release(); L->nodes.release(); L->count.release(); L->localOf.release(); L->level.release();
    L->scale.release(); L->X.release(); L->ellW.release(); L->ellCol.release(); L->phiStart.release();
    L->Z.release(); L->ZT.release(); L->DU.release(); L->DUT.release(); L->U.release(); L->H.release();
    L->C.release(); L->y.release(); L->dy.release(); L->dH.release(); L->dHp.release();
    L->loss.release(); L->bX.release(); L->bW.release(); L->bT.release(); L->bCol.release();
    L->sX.release(); L->sW.release(); L->sT.release(); L->sCol.release();
    if (L->stream) cudaStreamDestroy(L->stream);
    delete L;
}

const char* tg_learner_last_error(const tg_learner* L) { return L ? L->err.c_str() : ""; }

int32_t tg_learner_num_params(void) { return kParams; }

int tg_learner_set_refine(tg_learner* L, int32_t sweeps) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || sweeps < 0 || sweeps > 256) return lfail(L, TG_ERR_ARGUMENT, "tg_learner_set_refine: sweeps in [0, 256]");
    if (sweeps > 0 && L->cap > 4096)
        return lfail(L, TG_ERR_ARGUMENT, "tg_learner_set_refine: the sweeps take graphs of at most 4096 cells");
    L->refine = sweeps;
    return TG_OK;
}

int tg_learner_set_gain(tg_learner* L, float gain) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || !(gain >= 0.0f) || gain > 4.0f) return lfail(L, TG_ERR_ARGUMENT, "tg_learner_set_gain: gain in [0, 4]");
    L->gain = gain;
    return TG_OK;
}

int tg_learner_samples(const tg_learner* L, int32_t* count, int64_t* cells) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L) return lfail(nullptr, TG_ERR_ARGUMENT, "tg_learner_samples: null learner");
    if (count) *count = (int32_t)L->sLen.size();
    if (cells) *cells = L->sNodes;
    return TG_OK;
}

int tg_learner_get_params(tg_learner* L, float* out) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || !out) return lfail(L, TG_ERR_ARGUMENT, "tg_learner_get_params: null argument");
    LCK(cudaStreamSynchronize(L->stream));
    LCK(cudaMemcpy(out, L->P.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    return TG_OK;
}

int tg_learner_set_params(tg_learner* L, const float* in) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || !in) return lfail(L, TG_ERR_ARGUMENT, "tg_learner_set_params: null argument");
    LCK(cudaStreamSynchronize(L->stream));
    LCK(cudaMemcpy(L->P.p, in, sizeof(float) * kParams, cudaMemcpyHostToDevice));
    const int rc = refresh_bf16(L);
    return rc == TG_OK ? check_status(L, "tg_learner_set_params") : rc;
}

int tg_learner_get_sample(tg_learner* L, int32_t idx, int32_t* n, float* features, int32_t* ell_col, float* ell_w,
                          float* target) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || idx < 0 || idx >= (int32_t)L->sLen.size() || !n)
        return lfail(L, TG_ERR_ARGUMENT, "tg_learner_get_sample: bad index");
    const int len = L->sLen[idx];
    const int64_t o = L->sOff[idx];
    *n = len;
    if (features) LCK(cudaMemcpy(features, L->sX.p + o * kFeat, sizeof(float) * len * kFeat, cudaMemcpyDeviceToHost));
    if (ell_col) LCK(cudaMemcpy(ell_col, L->sCol.p + o * L->D, sizeof(int32_t) * len * L->D, cudaMemcpyDeviceToHost));
    if (ell_w) LCK(cudaMemcpy(ell_w, L->sW.p + o * L->D, sizeof(float) * len * L->D, cudaMemcpyDeviceToHost));
    if (target) LCK(cudaMemcpy(target, L->sT.p + o, sizeof(float) * len, cudaMemcpyDeviceToHost));
    return TG_OK;
}

int tg_learner_gradients(tg_learner* L, int32_t first, int32_t count, float* loss, float* grads, float* outputs) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || first < 0 || count < 1 || first + count > (int32_t)L->sLen.size())
        return lfail(L, TG_ERR_ARGUMENT, "tg_learner_gradients: bad sample range");
    std::vector<int> idx;
    for (int k = first; k < first + count; k++) idx.push_back(k);
    int rows = 0;
    int rc = stage_batch(L, idx, &rows);
    if (rc == TG_OK) rc = forward(L, L->bX.p, L->bCol.p, L->bW.p, rows);
    float l = 0.0f;
    if (rc == TG_OK) rc = backward(L, L->bCol.p, L->bW.p, L->bT.p, rows, &l);
    if (rc == TG_OK) rc = check_status(L, "tg_learner_gradients");
    if (rc != TG_OK) return rc;
    if (loss) *loss = l;
    if (grads) LCK(cudaMemcpy(grads, L->G.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    if (outputs) LCK(cudaMemcpy(outputs, L->y.p, sizeof(float) * rows, cudaMemcpyDeviceToHost));
    return TG_OK;
}

int tg_learner_train(tg_learner* L, int32_t steps, int32_t batch, float lr, uint64_t seed, int32_t first,
                     int32_t count, float* mean_loss) {
    ScopedDevice dev_scope(L ? L->device : -1);
    if (!L || steps < 0 || batch < 1 || !(lr > 0.0f)) return lfail(L, TG_ERR_ARGUMENT, "tg_learner_train: bad argument");
    const int total = (int)L->sLen.size();
    if (count <= 0) count = total - first;
    if (first < 0 || count < 1 || first + count > total) return lfail(L, TG_ERR_ARGUMENT, "tg_learner_train: no samples");
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> pick(first, first + count - 1);
    std::vector<float> losses(steps, 0.0f);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int s = 0; s < steps; s++) {
        std::vector<int> idx(batch);
        for (int& k : idx) k = pick(rng);
        int rows = 0;
        int rc = stage_batch(L, idx, &rows);
        if (rc == TG_OK) rc = forward(L, L->bX.p, L->bCol.p, L->bW.p, rows);
        if (rc == TG_OK) rc = backward(L, L->bCol.p, L->bW.p, L->bT.p, rows, &losses[s]);
        if (rc != TG_OK) return rc;
        L->adamStep++;
        const float c1 = 1.0f - std::pow(b1, (float)L->adamStep), c2 = 1.0f - std::pow(b2, (float)L->adamStep);
        launch_adam(L->P.p, L->G.p, L->M1.p, L->M2.p, kParams, lr, b1, b2, eps, c1, c2, L->stream);
        if ((rc = refresh_bf16(L)) != TG_OK) return rc;
    }
    const int rc = check_status(L, "tg_learner_train");
    if (rc != TG_OK) return rc;
    if (mean_loss) {
        const int tail = std::max(1, steps / 10);
        double acc = 0.0;
        for (int s = std::max(0, steps - tail); s < steps; s++) acc += losses[s];
        *mean_loss = steps ? (float)(acc / tail) : 0.0f;
    }
    return TG_OK;
}

}  // extern "C"
