// Sliced ELL layout of the stencil index and weight arrays.
//
// Rows are grouped in slices of 32; a row's n4 slots (n_pad rounded up to 4)
// are split in chunks of four consecutive slots.  Element (row i, slot s) sits at
//   (((i / 32) * nc + s / 4) * 32 + i % 32) * 4 + s % 4,     nc = n4 / 4,
// so the four slots of one chunk of one row are contiguous (one 16-byte index
// load, one or two 16-byte weight loads), and the same chunk of the 32 rows of
// a slice is one contiguous 512-byte (FP32/int32) run: a warp with one row per
// lane reads whole 128-byte lines while each lane still walks its own row in
// stencil order.  Padding rows (N rounded up to 32) hold index 0 and weight 0.
#pragma once

#include <cuda_runtime.h>

// element offset of slot 4*c of row i
__host__ __device__ __forceinline__ size_t sell_off(int i, int c, int nc)
{
    return ((((size_t)(i >> 5) * nc + c) << 5) + (size_t)(i & 31)) << 2;
}

__host__ __device__ __forceinline__ size_t sell_elem(int i, int s, int nc) { return sell_off(i, s >> 2, nc) + (s & 3); }

__device__ __forceinline__ int4 ld_idx4(const int* p) { return __ldg(reinterpret_cast<const int4*>(p)); }

// Ask the memory system to bring the line holding p into L2 (no register,
// no wait): issued a few chunks ahead of the loads that will use it.
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ __forceinline__ void ld_w4(const float* p, float (&w)[4])
{
    float4 t = __ldg(reinterpret_cast<const float4*>(p));
    w[0] = t.x;
    w[1] = t.y;
    w[2] = t.z;
    w[3] = t.w;
}

__device__ __forceinline__ void ld_w4(const double* p, double (&w)[4])
{
    double2 a = __ldg(reinterpret_cast<const double2*>(p));
    double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    w[0] = a.x;
    w[1] = a.y;
    w[2] = b.x;
    w[3] = b.y;
}

// four consecutive weights from shared memory (16-byte aligned)
__device__ __forceinline__ void ld_w4_shared(const float* p, float (&w)[4])
{
    const float4 t = *reinterpret_cast<const float4*>(p);
    w[0] = t.x;
    w[1] = t.y;
    w[2] = t.z;
    w[3] = t.w;
}

__device__ __forceinline__ void ld_w4_shared(const double* p, double (&w)[4])
{
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    w[0] = a.x;
    w[1] = a.y;
    w[2] = b.x;
    w[3] = b.y;
}

template <typename T>
__device__ __forceinline__ T fma_rn(T a, T b, T c);
template <>
__device__ __forceinline__ double fma_rn<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <>
__device__ __forceinline__ float fma_rn<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Arithmetic with a fixed rounding sequence (no contraction or reassociation
// by the compiler): every kernel that must reproduce another's result bit for
// bit spells its operations through these.
template <typename T>
struct Ar;
template <>
struct Ar<double> {
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
template <>
struct Ar<float> {
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};

// a*b + c with one rounding (PLAIN = false: the fused multiply-add), or with
// two, product then sum (PLAIN = true: the arithmetic of a CPU build without
// FMA instructions, such as the reference's own x86-64 build).
template <typename T, bool PLAIN>
__device__ __forceinline__ T madd(T a, T b, T c)
{
    if (PLAIN) return Ar<T>::add(Ar<T>::mul(a, b), c);
    return Ar<T>::fma(a, b, c);
}

// Sum of G lanes' partial values (lanes of a group are consecutive in the warp).
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v)
{
#pragma unroll
    for (int m = G / 2; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m, G);
    return v;
}
