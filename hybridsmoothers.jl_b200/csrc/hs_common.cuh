// Common device/host helpers for libhsb200 (sm_100a).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "hsb200.h"

// ---------------------------------------------------------------------------
// Host-side error plumbing
// ---------------------------------------------------------------------------
namespace hs {

int set_error(int status, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);
void count_launch(int64_t k = 1);
int32_t* device_error_word();   // device pointer to the bounded-wait error word
int num_sms();
int set_singular_col(int32_t col1);
// Raises the dynamic shared-memory limit of `kern` on the current device to
// at least `bytes` (cached per kernel and device).
int ensure_dynamic_smem(const void* kern, int bytes);

}  // namespace hs

#define HS_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) return hs::cuda_error(e_, #call);        \
    } while (0)

#define HS_LAUNCH_CHECK(what)                                           \
    do {                                                                \
        hs::count_launch();                                             \
        cudaError_t e_ = cudaGetLastError();                            \
        if (e_ != cudaSuccess) return hs::cuda_error(e_, what);         \
    } while (0)

// ---------------------------------------------------------------------------
// Arithmetic with explicit rounding.  Julia evaluates `acc += a*b` as two
// rounded operations and never contracts them into an FMA; these wrappers
// keep nvcc from contracting either, which is what makes the sweeps
// bit-identical to the reference's order of operations.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <typename T> __device__ __forceinline__ T sub_rn(T a, T b);
template <typename T> __device__ __forceinline__ T div_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ double sub_rn<double>(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ double div_rn<double>(double a, double b) { return __ddiv_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ float sub_rn<float>(float a, float b) { return __fsub_rn(a, b); }
template <> __device__ __forceinline__ float div_rn<float>(float a, float b) { return __fdiv_rn(a, b); }

template <typename T> __device__ __forceinline__ T abs_t(T a) { return a < T(0) ? -a : a; }
template <> __device__ __forceinline__ double abs_t<double>(double a) { return fabs(a); }
template <> __device__ __forceinline__ float abs_t<float>(float a) { return fabsf(a); }

template <typename T> struct dtype_of;
template <> struct dtype_of<double> { static constexpr int value = HS_F64; };
template <> struct dtype_of<float> { static constexpr int value = HS_F32; };

// ---------------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk.tensor) helpers.  No cluster multicast is used
// anywhere in this library.
// ---------------------------------------------------------------------------
namespace hsdev {

// Spin limit for every device-side wait (~seconds with try_wait's own
// suspend); a wait that runs out sets the error word and the kernel returns.
constexpr uint32_t kWaitLimit = 1u << 24;
constexpr int32_t kErrWaitTimeout = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One bounded probe loop; returns true when the phase with `parity` completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Non-blocking probe: true when the phase with `parity` has completed.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Plain arrive (count 1), release semantics at CTA scope.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// 2D tiled TMA load, global -> shared, completion on an mbarrier (no multicast).
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int32_t x, int32_t y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 1D bulk copy, global -> shared, completion on an mbarrier (no multicast).
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(gsrc)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Per-thread asynchronous copy of B (4, 8 or 16) bytes, global -> shared;
// both addresses B-byte aligned.  Completes at cp_async_wait_all.
template <int B>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(smem_dst)),
                 "l"(reinterpret_cast<uint64_t>(gsrc)), "n"(B)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
// 16 bytes, L2 only (no L1 allocation).
__device__ __forceinline__ void cp_async_cg16(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)),
                 "l"(reinterpret_cast<uint64_t>(gsrc))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most N of this thread's committed groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void report_error(int32_t* word, int32_t code) {
    if (word) atomicOr(word, code);
}

}  // namespace hsdev

// Host: encode a 2D tiled tensor map through the driver entry point (no -lcuda).
namespace hs {
int encode_tensor_map_2d(CUtensorMap* map, const void* base, int dtype, uint64_t inner, uint64_t outer,
                         uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer);
}
