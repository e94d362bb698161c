// TEST INFRASTRUCTURE -- not part of the product.
//
// Minimal CUDA execution-model stand-in that lets the reference's __global__
// kernels compile as ordinary host C++ (g++) and run on the CPU: one call of
// the kernel body per (block, thread) index, with the built-in index
// variables held per OpenMP thread.  Used only to pin the oracle against the
// reference's own kernel code.
#pragma once
struct uint3 { unsigned x, y, z; };
struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
