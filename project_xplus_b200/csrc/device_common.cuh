// device_common.cuh -- element loads, warp/block reductions and the bounded grid barrier
// shared by the sm_100a kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace xplus {
namespace dev {

// ---------------------------------------------------------------------------------------
// Read-only loads of the matrix stream: through L1 (__ldg), or with NA set past it
// (ld.global.nc.L1::no_allocate), so a kernel that streams the matrix once per iteration
// keeps its L1 for the neighbour records it gathers again and again.
__device__ __forceinline__ float ld_na(const float* p) {
    float v; asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p)); return v; }
__device__ __forceinline__ float2 ld_na(const float2* p) {
    float2 v; asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p)); return v; }
__device__ __forceinline__ float4 ld_na(const float4* p) {
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_na(const double* p) {
    double v; asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p)); return v; }
__device__ __forceinline__ double2 ld_na(const double2* p) {
    double2 v; asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p)); return v; }
__device__ __forceinline__ int ld_na(const int* p) {
    int v; asm volatile("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p)); return v; }
__device__ __forceinline__ int2 ld_na(const int2* p) {
    int2 v; asm volatile("ld.global.nc.L1::no_allocate.v2.s32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p)); return v; }
__device__ __forceinline__ int4 ld_na(const int4* p) {
    int4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ unsigned int ld_na(const unsigned int* p) {
    unsigned int v; asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p)); return v; }
__device__ __forceinline__ uint2 ld_na(const uint2* p) {
    uint2 v; asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p)); return v; }
__device__ __forceinline__ unsigned short ld_na(const unsigned short* p) {
    unsigned short v; asm volatile("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(v) : "l"(p)); return v; }
__device__ __forceinline__ short ld_na(const short* p) {
    short v; asm volatile("ld.global.nc.L1::no_allocate.s16 %0, [%1];" : "=h"(v) : "l"(p)); return v; }
// Load flavours of the matrix streams: through the read-only path (kLdg), read-only without L1
// allocation (kLdNoAlloc), or a plain load (kLdPlain: for arrays staged in shared memory, where
// the read-only global forms would be wrong).
constexpr int kLdg = 0, kLdNoAlloc = 1, kLdPlain = 2;
template <int NA, typename T>
__device__ __forceinline__ T ldro(const T* p) {
    if constexpr (NA == kLdNoAlloc) return ld_na(p);
    else if constexpr (NA == kLdPlain) return *p;
    else return __ldg(p);
}

// Matrix chunk loads: CHUNK consecutive slots of one row, as one vector load in the flavour NA
// (the matrix never changes inside a kernel).
// ---------------------------------------------------------------------------------------
template <typename VT, int CHUNK, int NA = kLdg>
struct ChunkLoad;

template <int NA>
struct ChunkLoad<float, 1, NA> {
    static __device__ __forceinline__ void run(const float* p, float* o) { o[0] = ldro<NA>(p); }
};
template <int NA>
struct ChunkLoad<float, 2, NA> {
    static __device__ __forceinline__ void run(const float* p, float* o) {
        const float2 v = ldro<NA>(reinterpret_cast<const float2*>(p));
        o[0] = v.x; o[1] = v.y;
    }
};
template <int NA>
struct ChunkLoad<float, 4, NA> {
    static __device__ __forceinline__ void run(const float* p, float* o) {
        const float4 v = ldro<NA>(reinterpret_cast<const float4*>(p));
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
};
template <int NA>
struct ChunkLoad<double, 1, NA> {
    static __device__ __forceinline__ void run(const double* p, double* o) { o[0] = ldro<NA>(p); }
};
template <int NA>
struct ChunkLoad<double, 2, NA> {
    static __device__ __forceinline__ void run(const double* p, double* o) {
        const double2 v = ldro<NA>(reinterpret_cast<const double2*>(p));
        o[0] = v.x; o[1] = v.y;
    }
};
template <int NA>
struct ChunkLoad<double, 4, NA> {
    static __device__ __forceinline__ void run(const double* p, double* o) {
        const double2 a = ldro<NA>(reinterpret_cast<const double2*>(p));
        const double2 b = ldro<NA>(reinterpret_cast<const double2*>(p + 2));
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
};
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }
template <int NA>
struct ChunkLoad<__nv_bfloat16, 1, NA> {
    static __device__ __forceinline__ void run(const __nv_bfloat16* p, float* o) {
        const unsigned short v = ldro<NA>(reinterpret_cast<const unsigned short*>(p));
        o[0] = __uint_as_float(static_cast<uint32_t>(v) << 16);
    }
};
template <int NA>
struct ChunkLoad<__nv_bfloat16, 2, NA> {
    static __device__ __forceinline__ void run(const __nv_bfloat16* p, float* o) {
        const uint32_t v = ldro<NA>(reinterpret_cast<const unsigned int*>(p));
        o[0] = bf16_lo(v); o[1] = bf16_hi(v);
    }
};
template <int NA>
struct ChunkLoad<__nv_bfloat16, 4, NA> {
    static __device__ __forceinline__ void run(const __nv_bfloat16* p, float* o) {
        const uint2 v = ldro<NA>(reinterpret_cast<const uint2*>(p));
        o[0] = bf16_lo(v.x); o[1] = bf16_hi(v.x); o[2] = bf16_lo(v.y); o[3] = bf16_hi(v.y);
    }
};

__device__ __forceinline__ float f16_lo(uint32_t w) {
    return __half2float(__ushort_as_half(static_cast<unsigned short>(w & 0xFFFFu)));
}
__device__ __forceinline__ float f16_hi(uint32_t w) {
    return __half2float(__ushort_as_half(static_cast<unsigned short>(w >> 16)));
}
template <int NA>
struct ChunkLoad<__half, 1, NA> {
    static __device__ __forceinline__ void run(const __half* p, float* o) {
        o[0] = __half2float(__ushort_as_half(ldro<NA>(reinterpret_cast<const unsigned short*>(p))));
    }
};
template <int NA>
struct ChunkLoad<__half, 2, NA> {
    static __device__ __forceinline__ void run(const __half* p, float* o) {
        const uint32_t v = ldro<NA>(reinterpret_cast<const unsigned int*>(p));
        o[0] = f16_lo(v); o[1] = f16_hi(v);
    }
};
template <int NA>
struct ChunkLoad<__half, 4, NA> {
    static __device__ __forceinline__ void run(const __half* p, float* o) {
        const uint2 v = ldro<NA>(reinterpret_cast<const uint2*>(p));
        o[0] = f16_lo(v.x); o[1] = f16_hi(v.x); o[2] = f16_lo(v.y); o[3] = f16_hi(v.y);
    }
};

// Column loads: absolute int32 columns, or int16 offsets from the row (lossless when the
// bandwidth of the ordered matrix is below 32768) returned as absolute columns.
template <int CHUNK, typename IT, int NA = kLdg>
struct ColLoad;
template <int NA>
struct ColLoad<1, int, NA> {
    static __device__ __forceinline__ void run(const int* p, int, int* o) { o[0] = ldro<NA>(p); }
};
template <int NA>
struct ColLoad<2, int, NA> {
    static __device__ __forceinline__ void run(const int* p, int, int* o) {
        const int2 v = ldro<NA>(reinterpret_cast<const int2*>(p));
        o[0] = v.x; o[1] = v.y;
    }
};
template <int NA>
struct ColLoad<4, int, NA> {
    static __device__ __forceinline__ void run(const int* p, int, int* o) {
        const int4 v = ldro<NA>(reinterpret_cast<const int4*>(p));
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
};
__device__ __forceinline__ int lo16(uint32_t w) { return static_cast<int>(static_cast<short>(w & 0xFFFFu)); }
__device__ __forceinline__ int hi16(uint32_t w) { return static_cast<int>(static_cast<short>(w >> 16)); }
template <int NA>
struct ColLoad<1, short, NA> {
    static __device__ __forceinline__ void run(const short* p, int row, int* o) { o[0] = row + ldro<NA>(p); }
};
template <int NA>
struct ColLoad<2, short, NA> {
    static __device__ __forceinline__ void run(const short* p, int row, int* o) {
        const uint32_t v = ldro<NA>(reinterpret_cast<const unsigned int*>(p));
        o[0] = row + lo16(v); o[1] = row + hi16(v);
    }
};
template <int NA>
struct ColLoad<4, short, NA> {
    static __device__ __forceinline__ void run(const short* p, int row, int* o) {
        const uint2 v = ldro<NA>(reinterpret_cast<const uint2*>(p));
        o[0] = row + lo16(v.x); o[1] = row + hi16(v.x); o[2] = row + lo16(v.y); o[3] = row + hi16(v.y);
    }
};

// The arithmetic type of a matrix value: bf16 values are widened to float.
template <typename VT> struct ValArith { using type = VT; };
template <> struct ValArith<__nv_bfloat16> { using type = float; };
template <> struct ValArith<__half> { using type = float; };

// ---------------------------------------------------------------------------------------
// Reductions in FP64 with a fixed combination order (results identical in every block).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums NV values per thread over the block; result valid in every thread.
// scratch: at least 32 * NV doubles of shared memory.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) scratch[q * 32 + warp] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double t = lane < nwarps ? scratch[q * 32 + lane] : 0.0;
        v[q] = warp_sum(t);
    }
}

__device__ __forceinline__ long long globaltimer_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Arrival at a grid barrier: the add is a release (this thread's earlier writes, and those of
// the CTA that a preceding __syncthreads ordered before it, are visible before it) and an
// acquire (the block that arrives last, and sees the full count in the value returned, then
// sees every other block's writes); the old value is returned.
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ int ld_volatile_int(const int* p) {
    return *reinterpret_cast<const volatile int*>(p);
}

// ---------------------------------------------------------------------------------------
// Grid barrier for a cooperative (co-resident) launch.  The counter only grows: barrier k
// completes when it reaches k * gridDim.x.  Every wait is bounded: after timeout_ns the
// waiting block raises *err (1) and returns false; blocks that see *err set leave too, so
// no block spins forever.  The fences on both sides give the acquire/release ordering that
// makes plain global stores before the barrier visible to plain loads after it.
// ---------------------------------------------------------------------------------------
struct GridBarrier {
    unsigned* counter;
    int* err;
    long long timeout_ns;
    unsigned epoch;
    int skip_block;  // test-only: this block withholds its arrival at the first barrier (-1: none)

    __device__ __forceinline__ bool sync(int* s_flag) {
        if (gridDim.x == 1 && skip_block < 0) {
            // one CTA: the CTA barrier orders its global-memory accesses as well
            __syncthreads();
            return true;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            ++epoch;
            const unsigned target = epoch * gridDim.x;
            // ordering through the counter alone (no separate fences): the arrival is an
            // acquire-release add and the polling loads are acquires; the counter's adds form
            // one release sequence, so the load that sees the full count synchronizes with
            // every block's arrival
            unsigned seen = target;  // a withheld arrival never completes the barrier
            if (!(static_cast<int>(blockIdx.x) == skip_block && epoch == 1u)) seen = atom_add_acq_rel_gpu(counter, 1u) + 1u;
            else seen = 0u;
            int ok = 1;
            // the last block to arrive sees the full count in its own atomic: no polling
            if (seen < target && ld_acquire_gpu(counter) < target) {
                const long long t0 = globaltimer_ns();
                unsigned spins = 0;
                while (ld_acquire_gpu(counter) < target) {
                    if ((++spins & 63u) == 0) {
                        if (ld_volatile_int(err) != 0) { ok = 0; break; }
                        if (globaltimer_ns() - t0 > timeout_ns) {
                            atomicExch(err, 1);
                            ok = 0;
                            break;
                        }
                    }
                }
            }
            *s_flag = ok;
        }
        __syncthreads();
        return *s_flag != 0;
    }
};

}  // namespace dev
}  // namespace xplus
