// helper.h -- drop-in for the reference's helper.h (ASPLOS-2022/DA-SpMMul-kernel
// helper.h:1-323): the names its benchmark driver and kernels use, with the
// same values and signatures, implemented for this library.
//
//   CUDA_CHECK                     helper.h:25-34 (prints and exits; caller-side macro)
//   hgpu::InitGen / CUArray /      helper.h:41-154 (host+device array mirror)
//   hgpu::GpuTimer                 helper.h:158-191 (events on stream 0)
//   ldg_float<T> / st_float<T>     helper.h:214-223 (4/8/16-byte vector access)
//   SparseFormat, DenseLayout      helper.h:256-264 (same enumerator values)
//   FULLMASK, DIV_UP,              helper.h:266-281 (warp sum, segmented
//   SHFL_DOWN_REDUCE, SEG_SHFL_SCAN                    suffix sum keyed by row)
//
// Differences, deliberate: InitGen draws from a seeded splitmix64 stream
// (seed 0 unless the DASPMM_SEED environment variable says otherwise) instead
// of a time(0)-seeded rand(), so runs are reproducible.
#ifndef SPMV_SPMM_HELPER
#define SPMV_SPMM_HELPER

#include <stddef.h>
#include <stdint.h>

#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <iostream>
#include <math.h>
#include <stdexcept>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_profiler_api.h>

#define CUDA_CHECK(status)                                                         \
    {                                                                              \
        cudaError_t daspmm_chk_err_ = (status);                                    \
        if (daspmm_chk_err_ != cudaSuccess) {                                      \
            std::cerr << "Got bad cuda status: " << cudaGetErrorString(daspmm_chk_err_) \
                      << " at line: " << __LINE__ << " of file " << __FILE__       \
                      << std::endl;                                                \
            exit(EXIT_FAILURE);                                                    \
        }                                                                          \
    }

namespace hgpu {

namespace detail {
inline uint64_t next_u64(uint64_t &s)
{
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
inline unsigned default_seed()
{
    const char *e = std::getenv("DASPMM_SEED");
    return e ? (unsigned)std::strtoul(e, nullptr, 10) : 0u;
}
}  // namespace detail

template <typename DType>
struct InitGen {
    uint64_t state;
    unsigned seed;
    InitGen() : state(detail::default_seed()), seed(detail::default_seed()) {}
    explicit InitGen(unsigned s) : state(s), seed(s) {}
    DType gen_next() { return (DType)0; }
};

template <>
struct InitGen<int> {
    uint64_t state;
    unsigned seed;
    InitGen() : state(detail::default_seed()), seed(detail::default_seed()) {}
    explicit InitGen(unsigned s) : state(s), seed(s) {}
    int gen_next() { return (int)(detail::next_u64(state) % 100) - 50; }  // [-50, 50)
};

template <>
struct InitGen<float> {
    uint64_t state;
    unsigned seed;
    InitGen() : state(detail::default_seed()), seed(detail::default_seed()) {}
    explicit InitGen(unsigned s) : state(s), seed(s) {}
    // same grid as the reference: multiples of 1/1000 in [-0.5, 0.5)
    float gen_next() { return (float)((int)(detail::next_u64(state) % 1000) - 500) / 1000; }
};

// Host vector with a device mirror (one cudaMalloc per sync_device).
template <typename DType>
class CUArray {
    std::vector<DType> host_;
    DType *dev_ = nullptr;
    int size_ = 0;

public:
    CUArray() {}
    explicit CUArray(std::vector<DType> &data) : host_(data), size_((int)data.size()) {}
    ~CUArray() { free_(); }
    CUArray(const CUArray &) = delete;
    CUArray &operator=(const CUArray &) = delete;

    void free_()
    {
        if (dev_) {
            CUDA_CHECK(cudaFree(dev_));
            dev_ = nullptr;
        }
    }
    void init_random(int size)
    {
        host_.assign(size, DType());
        InitGen<DType> g;
        for (int i = 0; i < size; ++i) host_[i] = g.gen_next();
        size_ = size;
    }
    void init_zeros(int size)
    {
        host_.assign(size, (DType)0);
        size_ = size;
    }
    void assign(std::vector<DType> &data)
    {
        host_ = data;
        size_ = (int)data.size();
        free_();
    }
    void sync_device()
    {
        free_();
        CUDA_CHECK(cudaMalloc((void **)&dev_, (size_t)size_ * sizeof(DType)));
        CUDA_CHECK(cudaMemcpy(dev_, host_.data(), (size_t)size_ * sizeof(DType),
                              cudaMemcpyHostToDevice));
    }
    std::vector<DType> sync_host()
    {
        assert(size_ == (int)host_.size());
        CUDA_CHECK(cudaMemcpy(host_.data(), dev_, (size_t)size_ * sizeof(DType),
                              cudaMemcpyDeviceToHost));
        return host_;
    }
    DType *get_device_data() { return dev_; }
    int get_size() { return size_; }
    DType *get_host_data() { return host_.data(); }
    std::vector<DType> &get_host_array() { return host_; }
};

// Event timer on the legacy default stream (helper.h:158-191).
struct GpuTimer {
    cudaEvent_t startEvent, stopEvent;
    GpuTimer()
    {
        cudaEventCreate(&startEvent);
        cudaEventCreate(&stopEvent);
    }
    ~GpuTimer()
    {
        cudaEventDestroy(startEvent);
        cudaEventDestroy(stopEvent);
    }
    void start() { cudaEventRecord(startEvent, 0); }
    void stop()
    {
        cudaEventRecord(stopEvent, 0);
        cudaEventSynchronize(stopEvent);
    }
    float elapsed_msecs()
    {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, startEvent, stopEvent);
        return ms;
    }
};

}  // namespace hgpu

// ---------------------------------------------------------------- vector access
#ifdef __CUDACC__
template <typename T>
__device__ __forceinline__ void ldg_float(float *r, const float *a)
{
    *reinterpret_cast<T *>(r) = __ldg(reinterpret_cast<const T *>(a));
}
template <typename T>
__device__ __forceinline__ void st_float(float *a, float *v)
{
    *reinterpret_cast<T *>(a) = *reinterpret_cast<const T *>(v);
}
#endif

// ---------------------------------------------------------------- enums
enum SparseFormat { SPARSE_FORMAT_CSR = 0, SPARSE_FORMAT_COO = 1 };
enum DenseLayout { DENSE_ROW_MAJOR = 0, DENSE_COL_MAJOR = 1 };

#define FULLMASK 0xffffffff
#define DIV_UP(x, y) (((x) + (y)-1) / (y))

#ifdef __CUDACC__
// Full-warp tree sum; lane 0 ends with the total (helper.h:269-274).
__device__ __forceinline__ float daspmm_warp_sum_down(float v)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(FULLMASK, v, d);
    return v;
}
// Segmented inclusive suffix sum over a warp whose keys (rows) are sorted:
// each lane ends with the sum of its own value and those of the following
// lanes that carry the same key (helper.h:276-281).
__device__ __forceinline__ float daspmm_warp_seg_suffix(float v, int key, int lane)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const float o = __shfl_down_sync(FULLMASK, v, d);
        const int ok = __shfl_down_sync(FULLMASK, key, d);
        if (lane + d < 32 && ok == key) v += o;
    }
    return v;
}
#define SHFL_DOWN_REDUCE(v) v = daspmm_warp_sum_down(v);
// The reference's macro reads a variable named lane_id from the caller's scope.
#define SEG_SHFL_SCAN(v, tmpv, segid, tmps) \
    v = daspmm_warp_seg_suffix(v, segid, lane_id); (void)tmpv; (void)tmps;
#endif

#endif  // SPMV_SPMM_HELPER
