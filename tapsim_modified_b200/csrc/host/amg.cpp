#include "amg.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <mutex>
#include <new>
#include <thread>

namespace tg_host {

// Test hook (amg_inject_worker_failure): while set, one worker of every
// threaded pass throws std::bad_alloc, as a failed allocation there would.
static std::atomic<bool> g_fail_workers(false);

void amg_inject_worker_failure(bool on) { g_fail_workers.store(on); }

namespace {

// Runs body(t) for t < T on T threads and joins every thread it started.  An
// exception leaving a worker (std::bad_alloc from one of the per-thread
// buffers, say) would call std::terminate; it is caught in the worker
// instead and the first one is rethrown on the calling thread after the
// joins.  If starting a thread throws, the threads already running are
// joined before that error propagates.
template <class F>
void run_threads(int T, F body) {
    std::mutex m;
    std::exception_ptr first;
    auto guarded = [&](int t) {
        try {
            if (g_fail_workers.load() && t == T - 1) throw std::bad_alloc();
            body(t);
        } catch (...) {
            std::lock_guard<std::mutex> lock(m);
            if (!first) first = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    try {
        pool.reserve(T);
        for (int t = 0; t < T; t++) pool.emplace_back(guarded, t);
    } catch (...) {
        for (auto& th : pool) th.join();
        throw;
    }
    for (auto& th : pool) th.join();
    if (first) std::rethrow_exception(first);
}

template <class F>
void parallel_rows(int n, int threads, F f) {
    if (threads <= 1 || n < 256) {
        f(0, n, 0);
        return;
    }
    const int chunk = (n + threads - 1) / threads;
    const int T = (n + chunk - 1) / chunk;
    run_threads(T, [&](int t) { f(t * chunk, std::min(n, (t + 1) * chunk), t); });
}

// R = P^T.  Each thread takes a contiguous block of P's rows and writes its
// entries after those of the blocks before it, so that every row of R lists
// P's rows in ascending order, as a serial pass would.
AmgCsr transpose(const AmgCsr& P, int threads) {
    AmgCsr R;
    R.rows = P.cols;
    R.cols = P.rows;
    const int T = std::max(1, threads);
    std::vector<std::vector<int32_t>> count(T);
    parallel_rows(P.rows, T, [&](int b, int e, int t) {
        count[t].assign(R.rows, 0);
        for (int q = P.ptr[b]; q < P.ptr[e]; q++) count[t][P.col[q]]++;
    });
    R.ptr.assign(R.rows + 1, 0);
    for (int c = 0; c < R.rows; c++) {
        int32_t at = R.ptr[c];
        for (int t = 0; t < T; t++) {
            if (count[t].empty()) continue;
            const int32_t k = count[t][c];
            count[t][c] = at;  // becomes the block's next position in row c
            at += k;
        }
        R.ptr[c + 1] = at;
    }
    R.col.resize(P.col.size());
    R.val.resize(P.val.size());
    parallel_rows(P.rows, T, [&](int b, int e, int t) {
        std::vector<int32_t>& next = count[t];
        for (int i = b; i < e; i++)
            for (int q = P.ptr[i]; q < P.ptr[i + 1]; q++) {
                const int k = next[P.col[q]]++;
                R.col[k] = i;
                R.val[k] = P.val[q];
            }
    });
    return R;
}

// Strong off-diagonal entries: |a_ij| >= theta sqrt(a_ii a_jj).
std::vector<char> strength(const AmgCsr& A, const std::vector<double>& diag, double theta, int threads) {
    std::vector<char> s(A.col.size(), 0);
    parallel_rows(A.rows, threads, [&](int b, int e, int) {
        for (int i = b; i < e; i++)
            for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++) {
                const int j = A.col[q];
                if (j == i) continue;
                s[q] = std::fabs(A.val[q]) >= theta * std::sqrt(std::fabs(diag[i] * diag[j]));
            }
    });
    return s;
}

// Greedy aggregation (Vanek et al. 1996, section 5): whole strong
// neighbourhoods first, then the left-over rows join the aggregate they are
// most strongly connected to, then what remains forms aggregates of its own.
// Rows without any off-diagonal entry stay out (-2).
std::vector<int32_t> aggregate(const AmgCsr& A, const std::vector<char>& strong, int* count) {
    const int n = A.rows;
    std::vector<int32_t> agg(n, -1);
    for (int i = 0; i < n; i++) {
        bool any = false;
        for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++) any |= A.col[q] != i;
        if (!any) agg[i] = -2;
    }
    int nc = 0;
    for (int i = 0; i < n; i++) {
        if (agg[i] != -1) continue;
        bool free = true, hasStrong = false;
        for (int q = A.ptr[i]; q < A.ptr[i + 1] && free; q++)
            if (strong[q]) {
                hasStrong = true;
                free = agg[A.col[q]] == -1;
            }
        if (!free || !hasStrong) continue;
        agg[i] = nc;
        for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++)
            if (strong[q]) agg[A.col[q]] = nc;
        nc++;
    }
    const std::vector<int32_t> first = agg;
    for (int i = 0; i < n; i++) {
        if (agg[i] != -1) continue;
        double best = 0.0;
        for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++) {
            const int j = A.col[q];
            if (strong[q] && first[j] >= 0 && std::fabs(A.val[q]) > best) {
                best = std::fabs(A.val[q]);
                agg[i] = first[j];
            }
        }
    }
    for (int i = 0; i < n; i++) {
        if (agg[i] != -1) continue;
        agg[i] = nc;
        for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++)
            if (strong[q] && agg[A.col[q]] == -1) agg[A.col[q]] = nc;
        nc++;
    }
    *count = nc;
    return agg;
}

// P = (I - omega D_F^-1 A_F) P0 with the filtered matrix A_F (weak entries
// lumped into the diagonal) and the tentative P0 (one per row, its aggregate).
AmgCsr smoothed_prolongator(const AmgCsr& A, const std::vector<char>& strong, const std::vector<int32_t>& agg,
                            int nc, double omega, int threads) {
    const int n = A.rows;
    // each row's entries (merged by aggregate) go to its slot of an
    // upper-bound layout (1 + its strong entries), then are compacted
    std::vector<int64_t> bound(n + 1, 0);
    parallel_rows(n, threads, [&](int b, int e, int) {
        for (int i = b; i < e; i++) {
            int k = agg[i] < 0 ? 0 : 1;
            if (agg[i] >= 0)
                for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++) k += strong[q] && A.col[q] != i;
            bound[i + 1] = k;
        }
    });
    for (int i = 0; i < n; i++) bound[i + 1] += bound[i];
    std::vector<int32_t> tcol(bound[n]), cnt(n, 0);
    std::vector<double> tval(bound[n]);
    parallel_rows(n, threads, [&](int b, int e, int) {
        std::vector<std::pair<int32_t, double>> tmp;
        for (int i = b; i < e; i++) {
            if (agg[i] < 0) continue;
            double dF = 0.0;
            for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++)
                if (A.col[q] == i || !strong[q]) dF += A.val[q];
            tmp.clear();
            tmp.emplace_back(agg[i], 1.0 - omega);
            for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++) {
                const int j = A.col[q];
                if (j == i || !strong[q] || agg[j] < 0) continue;
                tmp.emplace_back(agg[j], -omega * A.val[q] / dF);
            }
            std::sort(tmp.begin(), tmp.end());
            int k = 0;
            const int64_t base = bound[i];
            for (const auto& e2 : tmp) {
                if (k > 0 && tcol[base + k - 1] == e2.first) {
                    tval[base + k - 1] += e2.second;
                } else {
                    tcol[base + k] = e2.first;
                    tval[base + k] = e2.second;
                    k++;
                }
            }
            cnt[i] = k;
        }
    });
    AmgCsr P;
    P.rows = n;
    P.cols = nc;
    P.ptr.assign(n + 1, 0);
    for (int i = 0; i < n; i++) P.ptr[i + 1] = P.ptr[i] + cnt[i];
    P.col.resize(P.ptr[n]);
    P.val.resize(P.ptr[n]);
    parallel_rows(n, threads, [&](int b, int e, int) {
        for (int i = b; i < e; i++)
            for (int k = 0; k < cnt[i]; k++) {
                P.col[P.ptr[i] + k] = tcol[bound[i] + k];
                P.val[P.ptr[i] + k] = tval[bound[i] + k];
            }
    });
    return P;
}

// A_c = R A P, one coarse row per step, dense accumulator per thread.  The
// rows go to the threads in blocks of 64 as they free up (row costs vary
// with the aggregates' sizes), each thread appends its rows to a buffer of
// its own, and the rows are then copied into place; every row is summed in
// the same order whichever thread takes it.
AmgCsr galerkin(const AmgCsr& R, const AmgCsr& A, const AmgCsr& P, int threads) {
    const int nc = R.rows;
    const int T = nc < 256 ? 1 : std::max(1, threads);
    std::vector<int32_t> cnt(nc), owner(nc);
    std::vector<int64_t> off(nc);
    std::vector<std::vector<int32_t>> bufc(T);
    std::vector<std::vector<double>> bufv(T);
    std::atomic<int> next(0);
    constexpr int kRowsPerTake = 64;
    auto work = [&](int t) {
        std::vector<double> acc(nc, 0.0);
        std::vector<char> used(nc, 0);
        std::vector<int32_t> touched;
        std::vector<int32_t>& bc = bufc[t];
        std::vector<double>& bv = bufv[t];
        for (;;) {
            const int b = next.fetch_add(kRowsPerTake);
            if (b >= nc) break;
            const int e = std::min(nc, b + kRowsPerTake);
            for (int c = b; c < e; c++) {
                touched.clear();
                for (int qr = R.ptr[c]; qr < R.ptr[c + 1]; qr++) {
                    const int i = R.col[qr];
                    const double rci = R.val[qr];
                    for (int qa = A.ptr[i]; qa < A.ptr[i + 1]; qa++) {
                        const int k = A.col[qa];
                        const double w = rci * A.val[qa];
                        for (int qp = P.ptr[k]; qp < P.ptr[k + 1]; qp++) {
                            const int cc = P.col[qp];
                            if (!used[cc]) {
                                used[cc] = 1;
                                touched.push_back(cc);
                            }
                            acc[cc] += w * P.val[qp];
                        }
                    }
                }
                std::sort(touched.begin(), touched.end());
                owner[c] = t;
                off[c] = (int64_t)bc.size();
                cnt[c] = (int32_t)touched.size();
                for (int32_t cc : touched) {
                    bc.push_back(cc);
                    bv.push_back(acc[cc]);
                    acc[cc] = 0.0;
                    used[cc] = 0;
                }
            }
        }
    };
    if (T == 1) {
        work(0);
    } else {
        run_threads(T, work);
    }
    AmgCsr Ac;
    Ac.rows = Ac.cols = nc;
    Ac.ptr.assign(nc + 1, 0);
    for (int c = 0; c < nc; c++) Ac.ptr[c + 1] = Ac.ptr[c] + cnt[c];
    Ac.col.resize(Ac.ptr[nc]);
    Ac.val.resize(Ac.ptr[nc]);
    parallel_rows(nc, threads, [&](int b, int e, int) {
        for (int c = b; c < e; c++) {
            const int32_t* sc = bufc[owner[c]].data() + off[c];
            const double* sv = bufv[owner[c]].data() + off[c];
            std::copy(sc, sc + cnt[c], Ac.col.begin() + Ac.ptr[c]);
            std::copy(sv, sv + cnt[c], Ac.val.begin() + Ac.ptr[c]);
        }
    });
    return Ac;
}

// Drops the entries |a_ij| < drop sqrt(a_ii a_jj) of a coarse operator and
// adds them to a_ii, which keeps every row sum (and so the constants in the
// near null space) as it was.  Rows without a positive diagonal are kept whole.
// Two passes over the rows in parallel: count the kept entries, then write
// them (the dropped ones summed in row order, as one pass would).
void drop_weak(AmgCsr* A, double drop, int threads) {
    const int n = A->rows;
    std::vector<double> diag(n, 0.0);
    parallel_rows(n, threads, [&](int b, int e, int) {
        for (int i = b; i < e; i++)
            for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++)
                if (A->col[q] == i) diag[i] = A->val[q];
    });
    auto keep = [&](int i, int q) {
        const int j = A->col[q];
        return j == i || !(diag[i] > 0.0) || !(diag[j] > 0.0) ||
               std::fabs(A->val[q]) >= drop * std::sqrt(diag[i] * diag[j]);
    };
    std::vector<int32_t> ptr(n + 1, 0);
    parallel_rows(n, threads, [&](int b, int e, int) {
        for (int i = b; i < e; i++) {
            int32_t k = 0;
            for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) k += keep(i, q);
            ptr[i + 1] = k;
        }
    });
    for (int i = 0; i < n; i++) ptr[i + 1] += ptr[i];
    std::vector<int32_t> col(ptr[n]);
    std::vector<double> val(ptr[n]);
    parallel_rows(n, threads, [&](int b, int e, int) {
        for (int i = b; i < e; i++) {
            int32_t k = ptr[i], dpos = -1;
            double lump = 0.0;
            for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) {
                if (!keep(i, q)) {
                    lump += A->val[q];
                    continue;
                }
                if (A->col[q] == i) dpos = k;
                col[k] = A->col[q];
                val[k] = A->val[q];
                k++;
            }
            if (dpos >= 0) val[dpos] += lump;
        }
    });
    A->ptr.swap(ptr);
    A->col.swap(col);
    A->val.swap(val);
}

// Gauss-Jordan inverse with partial pivoting (row-major, in place).
bool dense_inverse(int n, std::vector<double>& a, std::vector<double>* inv) {
    inv->assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) (*inv)[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++)
            if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)p * n + c])) p = r;
        const double piv = a[(size_t)p * n + c];
        if (piv == 0.0 || !std::isfinite(piv)) return false;
        if (p != c)
            for (int k = 0; k < n; k++) {
                std::swap(a[(size_t)p * n + k], a[(size_t)c * n + k]);
                std::swap((*inv)[(size_t)p * n + k], (*inv)[(size_t)c * n + k]);
            }
        const double s = 1.0 / piv;
        for (int k = 0; k < n; k++) {
            a[(size_t)c * n + k] *= s;
            (*inv)[(size_t)c * n + k] *= s;
        }
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            const double f = a[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; k++) {
                a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
                (*inv)[(size_t)r * n + k] -= f * (*inv)[(size_t)c * n + k];
            }
        }
    }
    return true;
}

}  // namespace

std::string amg_build(AmgCsr&& A0, const AmgOptions& opt, AmgHierarchy* out) {
    const int threads = opt.threads > 0 ? opt.threads : std::max(1u, std::thread::hardware_concurrency());
    out->levels.clear();
    out->coarse_inv.clear();
    AmgCsr A = std::move(A0);
    for (int lev = 0;; lev++) {
        std::vector<double> diag(A.rows, 0.0);
        for (int i = 0; i < A.rows; i++)
            for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++)
                if (A.col[q] == i) diag[i] = A.val[q];
        for (int i = 0; i < A.rows; i++)
            if (!(diag[i] > 0.0)) {
                // rows without an entry (padding) keep a unit diagonal
                bool any = false;
                for (int q = A.ptr[i]; q < A.ptr[i + 1]; q++) any |= A.col[q] != i;
                if (any) return "amg: non-positive diagonal";
                diag[i] = 1.0;
            }
        AmgLevel L;
        const bool last = A.rows <= opt.max_coarse || lev + 1 >= opt.max_levels;
        if (!last) {
            const std::vector<char> strong = strength(A, diag, lev == 0 ? opt.theta : opt.theta_coarse, threads);
            int nc = 0;
            const std::vector<int32_t> agg = aggregate(A, strong, &nc);
            if (nc == 0 || nc > (int)(0.8 * A.rows)) {
                L.A = std::move(A);
                out->levels.push_back(std::move(L));
                break;
            }
            L.P = smoothed_prolongator(A, strong, agg, nc, opt.omega, threads);
            L.R = transpose(L.P, threads);
            AmgCsr Ac = galerkin(L.R, A, L.P, threads);
            if (opt.coarse_drop > 0.0) drop_weak(&Ac, opt.coarse_drop, threads);
            L.A = std::move(A);
            out->levels.push_back(std::move(L));
            A = std::move(Ac);
            continue;
        }
        L.A = std::move(A);
        out->levels.push_back(std::move(L));
        break;
    }
    // coarsest level: dense inverse
    const AmgCsr& C = out->levels.back().A;
    if (C.rows > 4096) return "amg: coarsest level too large for a dense inverse";
    std::vector<double> dense((size_t)C.rows * C.rows, 0.0);
    for (int i = 0; i < C.rows; i++) {
        bool any = false;
        for (int q = C.ptr[i]; q < C.ptr[i + 1]; q++) {
            dense[(size_t)i * C.rows + C.col[q]] = C.val[q];
            any = true;
        }
        if (!any) dense[(size_t)i * C.rows + i] = 1.0;
    }
    if (!dense_inverse(C.rows, dense, &out->coarse_inv)) return "amg: singular coarsest operator";
    return std::string();
}

}  // namespace tg_host
