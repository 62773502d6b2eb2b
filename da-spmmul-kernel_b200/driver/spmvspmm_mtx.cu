// spmvspmm_mtx.cu -- the benchmark driver for Matrix Market files, with the
// reference's command line and CSV rows (spmvspmm_benchmark.cu:336-420 and
// run.sh), built on libdaspmm.
//
//   spmvspmm_mtx <file.mtx> [profile <maxNv>] [--with-balanced]
//   spmvspmm_mtx --header [--with-balanced]       # run.sh's log.csv header
//
// For nv = 1, 2, 4, ... up to calcMaxNv (spmvspmm_benchmark.cu:78-90) it first
// checks every variant against a host loop (|out - ref| <= 1e-3, as
// checkAlgorithms, :118-232) and then prints one row per nv:
//
//   filename,nv,<8 variants: SR/PR x RB/EB x RM/CM>,<cuSPARSE columns>
//
// in GFLOP/s (2*nnz*nv / time), the variants timed by SpmvSpmmProblem::benchmark
// (the drop-in header) and cuSPARSE by its generic SpMV / SpMM API with the
// algorithms the reference times (:303-326): 4 columns for nv = 1, 10 for
// nv > 1.  --with-balanced appends this library's balanced-CSR kernel
// (DASPMM_ALG_CSR_BALANCED, row-major) as a last column.  "profile" runs each
// variant a few times without printing, as the reference's profile mode.
#include "daspmm.h"
#include "helper.h"
#include "spmvspmm.h"

#include <cuda_runtime.h>
#include <cusparse.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

const int kMaxNv = 128;
const int kMinNv = 1;

const char *kHeader =
    "filename,KDense,SR_RB_RM,PR_RB_RM,SR_EB_RM,PR_EB_RM,SR_RB_CM,PR_RB_CM,SR_EB_CM,PR_EB_CM,"
    "cusparse_default,cusparse_1,cusparse_2,cusparse_3,cusparse_4,cusparse_5,cusparse_6,"
    "cusparse_7,cusparse_8,cusparse_9";

int calc_max_nv(int nr, int nc, int nnz)
{
    cudaDeviceProp prop;
    CUDA_CHECK(cudaGetDeviceProperties(&prop, 0));
    const size_t mem = prop.totalGlobalMem;
    const size_t sp = ((size_t)nr + 1 + 2 * (size_t)nnz) * sizeof(int) + (size_t)nnz * sizeof(float);
    const long long max_nv = (long long)((mem - sp) / sizeof(float) / ((size_t)nr + nc));
    int nv = kMaxNv;
    while (nv > max_nv && nv > 0) nv /= 2;
    return nv;
}

// Host product in `layout` (the driver's own check, as cpuSpmvReference).
void host_spmm(bool cm, int nr, int nc, int nv, const std::vector<int> &rp,
               const std::vector<int> &ci, const std::vector<float> &va,
               const std::vector<float> &B, std::vector<float> &C)
{
    C.assign((size_t)nr * nv, 0.0f);
    for (int r = 0; r < nr; ++r)
        for (int k = 0; k < nv; ++k) {
            float acc = 0.0f;
            for (int p = rp[r]; p < rp[r + 1]; ++p)
                acc += va[p] * (cm ? B[(size_t)k * nc + ci[p]] : B[(size_t)ci[p] * nv + k]);
            C[cm ? (size_t)k * nr + r : (size_t)r * nv + k] = acc;
        }
}

bool close_enough(const std::vector<float> &ref, const float *out, size_t n, const char *what)
{
    for (size_t i = 0; i < n; ++i)
        if (std::fabs(out[i] - ref[i]) > 1e-3f) {
            std::fprintf(stderr, "Check Failed %s at %zu: %f != %f\n", what, i, out[i], ref[i]);
            return false;
        }
    return true;
}

struct Cusparse {
    cusparseHandle_t h = nullptr;
    cusparseSpMatDescr_t csr = nullptr, coo = nullptr;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    int nr, nc;

    Cusparse(int nr_, int nc_, int nnz, int *rp, int *ri, int *ci, float *va) : nr(nr_), nc(nc_)
    {
        cusparseCreate(&h);
        cusparseCreateCsr(&csr, nr, nc, nnz, rp, ci, va, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F);
        cusparseCreateCoo(&coo, nr, nc, nnz, ri, ci, va, CUSPARSE_INDEX_32I,
                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_32F);
    }
    ~Cusparse()
    {
        cudaFree(ws);
        cusparseDestroySpMat(csr);
        cusparseDestroySpMat(coo);
        cusparseDestroy(h);
    }
    bool grow(size_t need)
    {
        if (need <= ws_bytes) return true;
        cudaFree(ws);
        ws = nullptr;
        ws_bytes = 0;
        if (cudaMalloc(&ws, need) != cudaSuccess) return false;
        ws_bytes = need;
        return true;
    }
    // Runs (reps > 0: times) one SpMM / SpMV; returns ms per call or -1.
    float go(bool use_coo, bool cm, int nv, int alg, float *B, float *C, int warm, int reps)
    {
        const float one = 1.0f, zero = 0.0f;
        cusparseSpMatDescr_t A = use_coo ? coo : csr;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float ms = -1.0f;
        if (nv == 1) {
            cusparseDnVecDescr_t x, y;
            cusparseCreateDnVec(&x, nc, B, CUDA_R_32F);
            cusparseCreateDnVec(&y, nr, C, CUDA_R_32F);
            size_t need = 0;
            const cusparseSpMVAlg_t a = (cusparseSpMVAlg_t)alg;
            if (cusparseSpMV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, x, &zero,
                                        y, CUDA_R_32F, a, &need) == CUSPARSE_STATUS_SUCCESS &&
                grow(need)) {
                bool ok = true;
                for (int i = 0; i < warm + 1 && ok; ++i)
                    ok = cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, x, &zero, y,
                                      CUDA_R_32F, a, ws) == CUSPARSE_STATUS_SUCCESS;
                cudaEventRecord(e0);
                for (int i = 0; i < reps && ok; ++i)
                    ok = cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, x, &zero, y,
                                      CUDA_R_32F, a, ws) == CUSPARSE_STATUS_SUCCESS;
                cudaEventRecord(e1);
                cudaEventSynchronize(e1);
                if (ok) {
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms = reps ? ms / reps : 0.0f;
                }
            }
            cusparseDestroyDnVec(x);
            cusparseDestroyDnVec(y);
        } else {
            cusparseDnMatDescr_t Bd, Cd;
            const cusparseOrder_t ord = cm ? CUSPARSE_ORDER_COL : CUSPARSE_ORDER_ROW;
            cusparseCreateDnMat(&Bd, nc, nv, cm ? nc : nv, B, CUDA_R_32F, ord);
            cusparseCreateDnMat(&Cd, nr, nv, cm ? nr : nv, C, CUDA_R_32F, ord);
            size_t need = 0;
            const cusparseSpMMAlg_t a = (cusparseSpMMAlg_t)alg;
            if (cusparseSpMM_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE,
                                        CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, Bd, &zero, Cd,
                                        CUDA_R_32F, a, &need) == CUSPARSE_STATUS_SUCCESS &&
                grow(need)) {
                bool ok = true;
                for (int i = 0; i < warm + 1 && ok; ++i)
                    ok = cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE,
                                      CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, Bd, &zero, Cd,
                                      CUDA_R_32F, a, ws) == CUSPARSE_STATUS_SUCCESS;
                cudaEventRecord(e0);
                for (int i = 0; i < reps && ok; ++i)
                    ok = cusparseSpMM(h, CUSPARSE_OPERATION_NON_TRANSPOSE,
                                      CUSPARSE_OPERATION_NON_TRANSPOSE, &one, A, Bd, &zero, Cd,
                                      CUDA_R_32F, a, ws) == CUSPARSE_STATUS_SUCCESS;
                cudaEventRecord(e1);
                cudaEventSynchronize(e1);
                if (ok) {
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms = reps ? ms / reps : 0.0f;
                }
            }
            cusparseDestroyDnMat(Bd);
            cusparseDestroyDnMat(Cd);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return ms;
    }
};

struct CusparseCase {
    bool coo, cm;
    int alg;
};

// The cuSPARSE columns of one row, in the reference's order (:303-326).
std::vector<CusparseCase> cusparse_cases(int nv)
{
    if (nv == 1)
        return {{false, false, (int)CUSPARSE_SPMV_ALG_DEFAULT},
                {false, false, (int)CUSPARSE_SPMV_CSR_ALG1},
                {true, false, (int)CUSPARSE_SPMV_ALG_DEFAULT},
                {true, false, (int)CUSPARSE_SPMV_COO_ALG1}};
    return {{false, false, (int)CUSPARSE_SPMM_ALG_DEFAULT}, {false, false, (int)CUSPARSE_SPMM_CSR_ALG2},
            {true, false, (int)CUSPARSE_SPMM_ALG_DEFAULT},  {true, false, (int)CUSPARSE_SPMM_COO_ALG4},
            {false, true, (int)CUSPARSE_SPMM_ALG_DEFAULT},  {false, true, (int)CUSPARSE_SPMM_CSR_ALG1},
            {true, true, (int)CUSPARSE_SPMM_ALG_DEFAULT},   {true, true, (int)CUSPARSE_SPMM_COO_ALG1},
            {true, true, (int)CUSPARSE_SPMM_COO_ALG2},      {true, true, (int)CUSPARSE_SPMM_COO_ALG3}};
}

const SPMV_SPMM_ALG kAlgs[4] = {ALG_CSR_SCALAR, ALG_CSR_VECTOR, ALG_COO_SCALAR, ALG_COO_VECTOR};

}  // namespace

int main(int argc, char **argv)
{
    bool with_balanced = false, header = false, profile = false;
    int profile_nv = 0;
    std::vector<std::string> pos;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--with-balanced") with_balanced = true;
        else if (a == "--header") header = true;
        else pos.push_back(a);
    }
    if (header) {
        std::printf("%s%s\n", kHeader, with_balanced ? ",BAL_RM" : "");
        return 0;
    }
    if (pos.empty()) {
        std::fprintf(stderr, "usage: %s <filename> [profile <maxNv>] [--with-balanced]\n", argv[0]);
        return EXIT_SUCCESS;
    }
    if (pos.size() > 1 && pos[1] == "profile") {
        profile = true;
        profile_nv = pos.size() > 2 ? std::atoi(pos[2].c_str()) : 0;
    }
    const char *path = pos[0].c_str();
    daspmm_mtx_header mh;
    daspmm_status st = daspmm_mtx_info(path, &mh);
    if (st != DASPMM_OK) {
        std::fprintf(stderr, "cannot read %s: %s\n", path, daspmm_status_string(st));
        return EXIT_FAILURE;
    }
    const int nr = mh.nr, nc = mh.nc;
    std::vector<int> rp(nr + 1), ri(std::max<long long>(1, mh.nnz_max)),
        ci(std::max<long long>(1, mh.nnz_max));
    std::vector<float> va(std::max<long long>(1, mh.nnz_max));
    int nnz = 0;
    st = daspmm_mtx_read(path, 0, mh.nnz_max, rp.data(), ri.data(), ci.data(), va.data(), &nnz);
    if (st != DASPMM_OK) {
        std::fprintf(stderr, "cannot read %s: %s\n", path, daspmm_status_string(st));
        return EXIT_FAILURE;
    }
    int max_nv = calc_max_nv(nr, nc, nnz);
    if (profile) max_nv = profile_nv;
    std::fprintf(stderr, "Read file finished. nrows = %d, ncols = %d, nnz = %d, maxNv = %d\n", nr,
                 nc, nnz, max_nv);
    if (max_nv == 0) {
        std::fprintf(stderr, "Error: get maxNv=0.\n");
        return EXIT_FAILURE;
    }
    ri.resize(std::max(1, nnz));
    ci.resize(std::max(1, nnz));
    va.resize(std::max(1, nnz));

    hgpu::CUArray<int> d_rp(rp), d_ri(ri), d_ci(ci);
    hgpu::CUArray<float> d_va(va);
    d_rp.sync_device();
    d_ri.sync_device();
    d_ci.sync_device();
    d_va.sync_device();
    hgpu::CUArray<float> in, out;
    in.init_random(nc * max_nv);
    out.init_zeros(nr * max_nv);
    in.sync_device();
    out.sync_device();
    SpmvSpmmProblem prob(nr, nc, nnz, max_nv, d_rp.get_device_data(), d_ri.get_device_data(),
                         d_ci.get_device_data(), d_va.get_device_data(), in.get_device_data(),
                         out.get_device_data());
    Cusparse cs(nr, nc, nnz, d_rp.get_device_data(), d_ri.get_device_data(), d_ci.get_device_data(),
                d_va.get_device_data());
    float *B = in.get_device_data(), *C = out.get_device_data();
    const size_t cbytes = (size_t)nr * max_nv * sizeof(float);

    if (profile) {
        for (int nv = kMinNv; nv <= max_nv; nv *= 2)
            for (int l = 0; l < 2; ++l)
                for (SPMV_SPMM_ALG a : kAlgs) prob.dry_run(l ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR, nv, a, 5);
        return 0;
    }

    // checks first (checkAlgorithms): the variants, the balanced kernel, cuSPARSE
    bool passed = true;
    std::vector<float> ref, host_out((size_t)nr * max_nv);
    for (int nv = kMinNv; nv <= max_nv && passed; nv *= 2) {
        const std::vector<float> &Bh = in.get_host_array();
        for (int l = 0; l < 2 && passed; ++l) {
            const bool cm = l == 1;
            host_spmm(cm, nr, nc, nv, rp, ci, va, Bh, ref);
            for (SPMV_SPMM_ALG a : kAlgs) {
                CUDA_CHECK(cudaMemset(C, 0, cbytes));
                prob.run(cm ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR, nv, a);
                CUDA_CHECK(cudaMemcpy(host_out.data(), C, (size_t)nr * nv * 4, cudaMemcpyDeviceToHost));
                passed = passed && close_enough(ref, host_out.data(), (size_t)nr * nv, "variant");
            }
            if (!cm && with_balanced) {
                st = daspmm_spmm(DASPMM_ALG_CSR_BALANCED, DASPMM_ROW_MAJOR, nr, nc, nnz, nv,
                                 d_rp.get_device_data(), nullptr, d_ci.get_device_data(),
                                 d_va.get_device_data(), B, C, 0.0f, nullptr);
                CUDA_CHECK(cudaMemcpy(host_out.data(), C, (size_t)nr * nv * 4, cudaMemcpyDeviceToHost));
                passed = passed && st == DASPMM_OK &&
                         close_enough(ref, host_out.data(), (size_t)nr * nv, "balanced");
            }
            for (const CusparseCase &k : cusparse_cases(nv)) {
                if (k.cm != cm) continue;
                CUDA_CHECK(cudaMemset(C, 0, cbytes));
                if (cs.go(k.coo, k.cm, nv, k.alg, B, C, 0, 0) < 0) continue;  // not offered
                CUDA_CHECK(cudaMemcpy(host_out.data(), C, (size_t)nr * nv * 4, cudaMemcpyDeviceToHost));
                passed = passed && close_enough(ref, host_out.data(), (size_t)nr * nv, "cusparse");
            }
        }
    }
    if (!passed) return -1;

    for (int nv = kMinNv; nv <= max_nv; nv *= 2) {
        const double mflop = (double)nnz / 1e6 * 2 * nv;
        std::printf("%s,%d", path, nv);
        for (int l = 0; l < 2; ++l)
            for (SPMV_SPMM_ALG a : kAlgs) {
                const float ms = prob.benchmark(l ? DENSE_COL_MAJOR : DENSE_ROW_MAJOR, nv, a);
                std::printf(",%g", mflop / ms);
            }
        for (const CusparseCase &k : cusparse_cases(nv)) {
            const float ms = cs.go(k.coo, k.cm, nv, k.alg, B, C, 20, 200);
            if (ms > 0) std::printf(",%g", mflop / ms);
            else std::printf(",nan");
        }
        if (with_balanced) {
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            for (int i = 0; i < 5; ++i)
                daspmm_spmm(DASPMM_ALG_CSR_BALANCED, DASPMM_ROW_MAJOR, nr, nc, nnz, nv,
                            d_rp.get_device_data(), nullptr, d_ci.get_device_data(),
                            d_va.get_device_data(), B, C, 0.0f, nullptr);
            cudaEventRecord(e0);
            for (int i = 0; i < 50; ++i)
                daspmm_spmm(DASPMM_ALG_CSR_BALANCED, DASPMM_ROW_MAJOR, nr, nc, nnz, nv,
                            d_rp.get_device_data(), nullptr, d_ci.get_device_data(),
                            d_va.get_device_data(), B, C, 0.0f, nullptr);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            std::printf(",%g", mflop / (ms / 50));
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        std::printf("\n");
        std::fflush(stdout);
    }
    return 0;
}
