// Host-only access to the multigrid hierarchy (amg.cpp) behind the C ABI:
// the hierarchy tg_solve builds for preconditioner 1, built from any matrix
// the caller gives, so that its construction can be checked without a
// device.  No counterpart in the reference.
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/tapsim_gpu.h"
#include "amg.h"

namespace tgapi {
void set_process_error(const std::string& msg);  // handle.cu: read by tg_last_error(NULL)
}

struct tg_amg_host {
    tg_host::AmgHierarchy h;
};

namespace {

int amg_fail(const std::string& m, int code) {
    tgapi::set_process_error(m);
    return code;
}

}  // namespace

extern "C" {

int tg_amg_host_build(int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val, tg_amg_host** out) {
    if (!out || n < 1 || !row_ptr || !col || !val) return amg_fail("tg_amg_host_build: bad argument", TG_ERR_ARGUMENT);
    *out = nullptr;
    if (row_ptr[0] != 0) return amg_fail("tg_amg_host_build: row_ptr[0] must be 0", TG_ERR_ARGUMENT);
    for (int32_t i = 0; i < n; i++)
        if (row_ptr[i + 1] < row_ptr[i]) return amg_fail("tg_amg_host_build: row_ptr not ascending", TG_ERR_ARGUMENT);
    const int32_t nnz = row_ptr[n];
    for (int32_t q = 0; q < nnz; q++)
        if (col[q] < 0 || col[q] >= n) return amg_fail("tg_amg_host_build: column out of range", TG_ERR_ARGUMENT);
    // no exception crosses the C ABI: an allocation failure is a host error
    try {
        tg_host::AmgCsr A;
        A.rows = A.cols = n;
        A.ptr.assign(row_ptr, row_ptr + n + 1);
        A.col.assign(col, col + nnz);
        A.val.assign(val, val + nnz);
        std::unique_ptr<tg_amg_host> a(new tg_amg_host);
        const std::string err = tg_host::amg_build(std::move(A), tg_host::AmgOptions(), &a->h);
        if (!err.empty()) return amg_fail("tg_amg_host_build: " + err, TG_ERR_HOST);
        *out = a.release();
    } catch (const std::exception& e) {
        return amg_fail(std::string("tg_amg_host_build: ") + e.what(), TG_ERR_HOST);
    }
    return TG_OK;
}

int32_t tg_amg_host_levels(const tg_amg_host* a) { return a ? (int32_t)a->h.levels.size() : 0; }

int tg_amg_host_matrix(const tg_amg_host* a, int32_t level, int32_t which, int32_t* rows, int32_t* cols, int64_t* nnz,
                       int32_t* ptr, int32_t* col, double* val) {
    if (!a || level < 0 || level >= (int32_t)a->h.levels.size() || which < 0 || which > 2)
        return amg_fail("tg_amg_host_matrix: bad level or matrix", TG_ERR_ARGUMENT);
    const tg_host::AmgLevel& L = a->h.levels[level];
    if (which > 0 && level + 1 == (int32_t)a->h.levels.size())
        return amg_fail("tg_amg_host_matrix: the coarsest level has no transfer operators", TG_ERR_ARGUMENT);
    const tg_host::AmgCsr& M = which == 0 ? L.A : (which == 1 ? L.P : L.R);
    if (rows) *rows = M.rows;
    if (cols) *cols = M.cols;
    if (nnz) *nnz = (int64_t)M.val.size();
    if (ptr) std::memcpy(ptr, M.ptr.data(), sizeof(int32_t) * M.ptr.size());
    if (col && !M.col.empty()) std::memcpy(col, M.col.data(), sizeof(int32_t) * M.col.size());
    if (val && !M.val.empty()) std::memcpy(val, M.val.data(), sizeof(double) * M.val.size());
    return TG_OK;
}

void tg_amg_host_destroy(tg_amg_host* a) { delete a; }

void tg_amg_host_inject_worker_failure(int32_t on) { tg_host::amg_inject_worker_failure(on != 0); }

}  // extern "C"
