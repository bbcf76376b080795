/*
 * cuda_emu.h — a minimal CUDA execution model for compiling the reference's kernel
 * sources (support_funcs.cu, UVZSolver_multithread.cu, Sediment_Transport.cu) as
 * plain C++ and running them on the CPU, one thread at a time in launch order.
 *
 * TEST INFRASTRUCTURE ONLY: it lets the reference's own code be executed in a
 * container without a GPU, so that the oracle restatement can be checked against
 * it bit for bit.
 *
 * Execution order: blocks in (z, y, x) order with x fastest, threads likewise.
 * __syncthreads() is a no-op.  The only live kernel that calls it is
 * _calculate_abcd (UVZSolver_multithread.cu:436), whose overrides after the
 * barrier are re-applied by every later thread of the segment, so sequential
 * thread order gives the barrier's result.  Kernels that the reference launches
 * with 32 identical threads per line are launched with one thread here.
 */
#ifndef HYDIST_CUDA_EMU_H
#define HYDIST_CUDA_EMU_H

#include <cmath>
#include <cstdio>
#include <cstdlib>

struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct emu_uint3 {
    unsigned x, y, z;
};

extern emu_uint3 threadIdx, blockIdx;
extern dim3 blockDim, gridDim;

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ static
#define __forceinline__ inline

inline void __syncthreads() {}
/* round to nearest, ties to even, like the device intrinsic */
inline int __double2int_rn(double x) { return (int)std::nearbyint(x); }

/* device-side overloads of the math the kernels use */
using std::abs;
inline double min(double a, double b) { return std::fmin(a, b); }
inline double max(double a, double b) { return std::fmax(a, b); }
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }

template <class F>
inline void emu_launch(dim3 g, dim3 b, F&& body) {
    gridDim = g;
    blockDim = b;
    for (unsigned bz = 0; bz < g.z; bz++)
        for (unsigned by = 0; by < g.y; by++)
            for (unsigned bx = 0; bx < g.x; bx++) {
                blockIdx = {bx, by, bz};
                for (unsigned tz = 0; tz < b.z; tz++)
                    for (unsigned ty = 0; ty < b.y; ty++)
                        for (unsigned tx = 0; tx < b.x; tx++) {
                            threadIdx = {tx, ty, tz};
                            body();
                        }
            }
}

#endif
