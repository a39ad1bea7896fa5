// Process-wide plumbing of libhsb200: error strings, the device error word,
// launch counting, tensor-map encoding.
#include <cudaTypedefs.h>

#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "hs_common.cuh"

namespace {
thread_local std::string g_last_error;
thread_local int32_t g_singular_col = 0;
std::atomic<int64_t> g_launches{0};
std::mutex g_mu;
int32_t* g_err_word[64] = {nullptr};   // per device
int g_sm_count[64] = {0};

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
}  // namespace

namespace hs {

int set_error(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return status;
}

int cuda_error(cudaError_t e, const char* what) {
    int st = (e == cudaErrorMemoryAllocation) ? HS_ERR_OOM : HS_ERR_CUDA;
    cudaGetLastError();  // clear sticky-free errors
    return set_error(st, "%s: %s", what, cudaGetErrorString(e));
}

void count_launch(int64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

int32_t* device_error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_err_word[dev]) {
        int32_t* p = nullptr;
        if (cudaMalloc(&p, sizeof(int32_t)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, sizeof(int32_t));
        cudaDeviceSynchronize();
        g_err_word[dev] = p;
    }
    return g_err_word[dev];
}

int num_sms() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!g_sm_count[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        g_sm_count[dev] = v > 0 ? v : 148;
    }
    return g_sm_count[dev];
}

int ensure_dynamic_smem(const void* kern, int bytes) {
    // The attribute is a property of the kernel on one device: remember the
    // largest value set per (kernel, device), so a host thread that drives
    // several GPUs raises it on each of them.
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    int& have = done[std::make_pair(kern, dev)];
    if (bytes > have) {
        HS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        have = bytes;
    }
    return HS_OK;
}

int set_singular_col(int32_t col1) {
    g_singular_col = col1;
    return HS_ERR_SINGULAR;
}

int encode_tensor_map_2d(CUtensorMap* map, const void* base, int dtype, uint64_t inner, uint64_t outer,
                         uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer) {
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000,
                                                         cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return set_error(HS_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMapDataType dt = dtype == HS_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = g_encode(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(HS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return HS_OK;
}

}  // namespace hs

extern "C" {

const char* hs_last_error(void) { return g_last_error.c_str(); }

int32_t hs_last_singular_col(void) { return g_singular_col; }

int hs_device_error(void* stream, int32_t* code) {
    if (!code) return hs::set_error(HS_ERR_ARG, "hs_device_error: code is NULL");
    int32_t* w = hs::device_error_word();
    if (!w) return hs::set_error(HS_ERR_CUDA, "device error word unavailable");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int32_t v = 0;
    HS_CUDA(cudaMemcpyAsync(&v, w, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    HS_CUDA(cudaMemsetAsync(w, 0, sizeof(int32_t), s));
    HS_CUDA(cudaStreamSynchronize(s));
    *code = v;
    return HS_OK;
}

int64_t hs_kernel_launches(void) { return g_launches.load(); }

const char* hs_version(void) { return "hsb200 0.1.0 (sm_100a)"; }

}  // extern "C"
