// Host stand-in for the few CUDA names the device headers tested on the CPU
// use (the shared-memory FFT engine, the ghost-entry writers), so that they
// run with one thread doing all the work: a FFT stage's butterflies touch
// disjoint elements, so sequential order is valid and the barrier is a no-op.
#pragma once
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
struct double2 { double x, y; };
struct float2 { float x, y; };
struct HostDim3 { unsigned x, y, z; };
static HostDim3 threadIdx{0, 0, 0}, blockDim{1, 1, 1};
inline void __syncthreads() {}
