// fm_device.cuh -- small device helpers shared by the single-system kernels
// (fm_kernels.cu) and the multi-job slot engine (fm_engine.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fm {

// |v|^2 in the reference's dot_product order, no contraction.
__device__ __forceinline__ double norm2_rn(double x, double y, double z)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

// Programmatic dependent launch (kernels started with pdl_launch): wait for
// the predecessor grid to complete and its memory to be visible before
// touching anything, then let the successor grid begin launching.  Both are
// no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Set while a CUDA graph is being captured on this thread: its kernels are
// ordered by the graph's edges, launched without the attribute below.
extern thread_local bool pdl_capture;

// Launches k with programmatic stream serialization: the next kernel of the
// step may be launched while k's last blocks run, and waits in pdl_enter for
// k to complete before it reads anything (so the chain of small, often gated
// kernels of a step does not pay a full launch gap each).
template <typename... P, typename... A>
void pdl_launch(void (*k)(P...), dim3 grid, dim3 block, cudaStream_t st, A... args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = 0;
    c.stream = st;
    c.attrs = at;
    c.numAttrs = pdl_capture ? 0 : 1;
    cudaLaunchKernelEx(&c, k, args...);
}

// pdl_launch with dynamic shared memory.
template <typename... P, typename... A>
void pdl_launch_smem(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = smem;
    c.stream = st;
    c.attrs = at;
    c.numAttrs = pdl_capture ? 0 : 1;
    cudaLaunchKernelEx(&c, k, args...);
}

// Neighbour-list entries are read once per step and never again before the
// next step: keep them out of L1, so that the partner positions they point at
// stay cached there.
__device__ __forceinline__ int4 ld_stream_int4(const int4 *p)
{
    int4 r;
    asm("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p));
    return r;
}

// FP32 reciprocal of the precision form's pair magnitudes (s = 1/r^2): the
// hardware's approximate reciprocal (rcp.approx.ftz.f32, about 1 ulp; r^2 is
// never subnormal here), one instruction where a correctly rounded
// reciprocal takes a short sequence with a slow path.
__device__ __forceinline__ float rcp_f32(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Read-only gather of one double4 (32-byte aligned) as a single 256-bit load:
// one L1 request per partner instead of two.
__device__ __forceinline__ double4 ldg_pos(const double4 *p)
{
    double4 r;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
    return r;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Float min/max over the warp with one integer reduction each: the bit
// pattern with the magnitude bits flipped for negatives orders like the
// float (finite values).
__device__ __forceinline__ int float_order_key(float v)
{
    const int b = __float_as_int(v);
    return b ^ ((b >> 31) & 0x7fffffff);
}
__device__ __forceinline__ float float_from_order_key(int k) { return __int_as_float(k ^ ((k >> 31) & 0x7fffffff)); }
__device__ __forceinline__ float warp_min(float v)
{
    return float_from_order_key(__reduce_min_sync(0xffffffffu, float_order_key(v)));
}
__device__ __forceinline__ float warp_max(float v)
{
    return float_from_order_key(__reduce_max_sync(0xffffffffu, float_order_key(v)));
}

// icell = ceiling((r + halfdomain)/cellsidelength) + 1 (1-based, halo = 1 and
// ncells+2); the 0-based extended index is the ceiling itself.  Out-of-grid
// values are clamped and flagged.
__device__ __forceinline__ int bin_axis(double x, double hd, double cs, int ne, bool &bad)
{
    double q = __ddiv_rn(__dadd_rn(x, hd), cs);
    if (!(q == q)) { bad = true; return 0; }
    int c = __double2int_ru(q);  // round toward +inf == ceiling for in-range values
    if (c < 0 || c > ne - 1) { bad = true; c = c < 0 ? 0 : ne - 1; }
    return c;
}

__device__ __forceinline__ bool is_halo(int x, int ne) { return x == 0 || x == ne - 1; }

// Periodic image of a coordinate: one FP64 add of +/-L, as the reference's
// halo copy r(k,np+m) = r(k,np+m) +/- domain(k).
__device__ __forceinline__ double image(double x, int s, double L)
{
    return s ? __dadd_rn(x, s > 0 ? L : -L) : x;
}

// Neumaier-compensated accumulation.
__device__ __forceinline__ void neumaier(double &sum, double &cmp, double x)
{
    double t = sum + x;
    cmp += fabs(sum) >= fabs(x) ? (sum - t) + x : (x - t) + sum;
    sum = t;
}

}  // namespace fm
