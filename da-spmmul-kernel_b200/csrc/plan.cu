// plan.cu -- planned SpMM: one sparse matrix, many products.
//
// daspmm_spmm is stateless: every call recomputes the chunk boundaries of the
// balanced split (k_partition over rowPtr) before the gather, so a caller may
// change the matrix between calls.  A caller that multiplies the same matrix
// by many dense operands (an iterative solver, a GNN layer over one graph, a
// serving loop over a resident matrix) can instead create a plan: the
// boundaries, and the list of chunks with an empty row (which the walk kernel
// sums), are computed once into a workspace the plan owns, and each product is
// the worker-group window kernel plus the walk over that fixed list -- no
// partition pass.  Between products nothing is reset: the split-row counters
// return to zero by themselves (the last piece of a row clears its counter),
// and each call counts its queue claims on from where the previous call's
// ended (a call makes exactly one claim per chunk group).  Results are
// bit-identical to daspmm_spmm with the same configuration (same chunks, same
// order of summation).  Calls the window kernel does not take (beta != 0, B
// or C not 32-byte aligned, tiles other than 128 or 64 columns) run the
// stateless path on the plan's workspace, and the next planned call first
// writes the boundaries and the list again.
#include "internal.h"

#include <cuda_runtime.h>

#include <new>
#include <vector>

struct daspmm_plan_s {
    daspmm::Resolved r;
    int nr, nc, nnz, nv;
    const int *rowPtr, *colIdx;
    const float *values;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    std::vector<int> list;   // [count, chunk ids...]: chunks with an empty row
    bool fresh = false;      // boundaries and list in the workspace are the plan's
    unsigned long long calls = 0;  // planned products since they were written
    int dev = 0;
};

namespace {

// Boundaries (k_partition, which also zeroes the queue heads and split-row
// counters) and the fixed walk list into the plan's workspace.
daspmm_status refresh(daspmm_plan p, cudaStream_t st)
{
    daspmm::carve_and_partition(p->r, p->nr, p->nnz, p->rowPtr, p->ws, st);
    const int2 *meta = nullptr;
    int *list = nullptr;
    daspmm::workspace_tables(p->r, p->ws, &meta, &list);
    cudaError_t e = cudaMemcpyAsync(list, p->list.data(), sizeof(int) * p->list.size(),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return daspmm::cuda_fail(e);
    p->fresh = true;
    p->calls = 0;
    return DASPMM_OK;
}

// The chunks whose rows [s_c, s_{c+1}) hold an empty row: the window kernel
// cannot sum them (a bitmask of row ends cannot express two rows ending at
// one position), the walk kernel does.  Same rule as the window kernel's.
daspmm_status build_list(daspmm_plan p, cudaStream_t st)
{
    const int nch = p->r.nchunks;
    std::vector<int2> meta((size_t)nch + 1);
    std::vector<int> rp((size_t)p->nr + 1);
    const int2 *d_meta = nullptr;
    int *d_list = nullptr;
    daspmm::workspace_tables(p->r, p->ws, &d_meta, &d_list);
    daspmm::carve_and_partition(p->r, p->nr, p->nnz, p->rowPtr, p->ws, st);
    cudaError_t e = cudaMemcpyAsync(meta.data(), d_meta, sizeof(int2) * meta.size(),
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(rp.data(), p->rowPtr, sizeof(int) * rp.size(),
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return daspmm::cuda_fail(e);
    p->list.assign(1, 0);
    for (int c = 0; c < nch; ++c) {
        for (int r = meta[c].y; r < meta[c + 1].y; ++r) {
            if (rp[r] == rp[r + 1]) {
                p->list.push_back(c);
                break;
            }
        }
    }
    p->list[0] = (int)p->list.size() - 1;
    return DASPMM_OK;
}

}  // namespace

extern "C" {

daspmm_status daspmm_plan_create(const daspmm_config *cfg, int nr, int nc, int nnz, int nv,
                                 const int *rowPtr, const int *colIdx, const float *values,
                                 void *stream, daspmm_plan *out)
{
    if (!out) return DASPMM_ERR_INVALID;
    *out = nullptr;
    daspmm_config c = cfg ? *cfg : daspmm_config{};
    if (!cfg) c.alg = DASPMM_ALG_CSR_BALANCED;
    if (c.alg != DASPMM_ALG_CSR_BALANCED) return DASPMM_ERR_UNSUPPORTED;
    if (nr < 0 || nc < 0 || nnz < 0 || nv < 1 || !rowPtr || (nnz > 0 && (!colIdx || !values)))
        return DASPMM_ERR_INVALID;
    daspmm::Resolved r;
    daspmm_status s = daspmm::resolve(&c, DASPMM_ROW_MAJOR, nr, nc, nnz, nv, nullptr, nullptr, &r);
    if (s != DASPMM_OK) return s;
    auto *p = new (std::nothrow) daspmm_plan_s();
    if (!p) return DASPMM_ERR_INVALID;
    p->r = r;
    p->nr = nr; p->nc = nc; p->nnz = nnz; p->nv = nv;
    p->rowPtr = rowPtr; p->colIdx = colIdx; p->values = values;
    cudaGetDevice(&p->dev);
    p->ws_bytes = daspmm::workspace_bytes(r, nv);
    cudaStream_t st = (cudaStream_t)stream;
    if (p->ws_bytes) {
        cudaError_t e = cudaMalloc(&p->ws, p->ws_bytes);
        if (e != cudaSuccess) {
            delete p;
            return daspmm::cuda_fail(e);
        }
    }
    if (r.pipe == 4 && nr > 0) {
        s = build_list(p, st);
        if (s == DASPMM_OK) s = refresh(p, st);
        if (s == DASPMM_OK) {
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) s = daspmm::cuda_fail(e);
        }
        if (s != DASPMM_OK) {
            cudaFree(p->ws);
            delete p;
            return s;
        }
    }
    *out = p;
    return DASPMM_OK;
}

daspmm_status daspmm_plan_spmm(daspmm_plan p, const float *B, float *C, float beta, void *stream)
{
    if (!p) return DASPMM_ERR_INVALID;
    if (p->nr == 0) return DASPMM_OK;
    if (!B || !C) return DASPMM_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (beta == 0.0f && p->r.pipe == 4) {
        if (!p->fresh) {
            daspmm_status s = refresh(p, st);
            if (s != DASPMM_OK) return s;
        }
        if (daspmm::run_planned(p->r, p->nr, p->nc, p->nnz, p->nv, p->rowPtr, p->colIdx,
                                p->values, B, C, p->ws, p->calls, st)) {
            ++p->calls;
            cudaError_t e = cudaGetLastError();
            return e == cudaSuccess ? DASPMM_OK : daspmm::cuda_fail(e);
        }
    }
    // the stateless path on the plan's workspace: it rewrites the boundaries,
    // the queue heads and the list, so the next planned call refreshes them
    p->fresh = false;
    return daspmm::run_resolved(p->r, DASPMM_ROW_MAJOR, p->nr, p->nc, p->nnz, p->nv, p->rowPtr,
                                nullptr, p->colIdx, p->values, B, C, beta, p->ws, p->ws_bytes,
                                st);
}

daspmm_status daspmm_plan_config(daspmm_plan p, daspmm_config *out)
{
    if (!p || !out) return DASPMM_ERR_INVALID;
    *out = daspmm::to_config(p->r);
    return DASPMM_OK;
}

daspmm_status daspmm_plan_destroy(daspmm_plan p)
{
    if (!p) return DASPMM_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->dev) cudaSetDevice(p->dev);
    cudaError_t e = p->ws ? cudaFree(p->ws) : cudaSuccess;
    if (cur != p->dev) cudaSetDevice(cur);
    delete p;
    return e == cudaSuccess ? DASPMM_OK : daspmm::cuda_fail(e);
}

}  // extern "C"
