// shim.h — TEST INFRASTRUCTURE ONLY.
//
// Gives CUDA kernel source a host meaning so that the reference's own kernels
// (Multiphase/Multiphase/spray_k.cu) compile with g++ and run on the CPU, one
// emulated thread after another (oracle/make_refhost.py, refhost/stages.inc).
//
//   * __global__/__device__/__constant__ are plain C++; threadIdx, blockIdx,
//     blockDim and gridDim are thread-local globals that host_launch() sets
//     per emulated thread (host_launch_sync() runs a block's threads as
//     cooperative fibers, for the kernels that call __syncthreads);
//   * helper_math.h's float3 arithmetic (a CUDA samples header the reference
//     includes, not present here) is restated with the same operation order
//     (componentwise, one rounding per operation);
//   * rsqrtf is 1/sqrtf (CUDA's is an approximation; the oracle and the
//     library use the same exact form in normalize());
//   * atomics are plain read-modify-writes: with threads run in ascending
//     order, every float atomic adds its contributions in ascending thread
//     order, the order the oracle defines for the reference's unordered
//     atomics; a launch whose threads also read what the atomics write can
//     defer them to the end of the launch (rh_defer_atomics);
//   * tex1Dfetch reads a host array bound to the texture reference.
#pragma once
#define __host__
#define __device__
#define __global__
#define __constant__
#define __shared__
#define __forceinline__ inline
#include <vector_types.h>
#include <vector_functions.h>
#include <cmath>
#include <math.h>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <algorithm>
#include <vector>
#include <functional>
#include <ucontext.h>

static thread_local uint3 threadIdx, blockIdx;
static thread_local dim3 blockDim, gridDim;

// Runs f once per thread of a <<<grid, block>>> launch, blocks and threads in
// ascending order.
template <class F>
static void host_launch(dim3 grid, dim3 block, F&& f) {
    gridDim = grid;
    blockDim = block;
    for (unsigned bz = 0; bz < grid.z; bz++)
        for (unsigned by = 0; by < grid.y; by++)
            for (unsigned bx = 0; bx < grid.x; bx++)
                for (unsigned tz = 0; tz < block.z; tz++)
                    for (unsigned ty = 0; ty < block.y; ty++)
                        for (unsigned tx = 0; tx < block.x; tx++) {
                            blockIdx = make_uint3(bx, by, bz);
                            threadIdx = make_uint3(tx, ty, tz);
                            f();
                        }
}

// A launch of a kernel that synchronises its block (__syncthreads over
// shared memory): each CUDA thread of the one-dimensional block is a
// cooperative fiber (ucontext) on this host thread; the fibers run in thread
// order up to their next __syncthreads, one round after another, so every
// thread reaches a barrier before any passes it.  The blocks run one after
// another.  Shared arrays declared `extern __shared__` are host globals
// (globals.inc); a `__shared__` array inside a kernel becomes a local array of
// each thread, which is what kernels that only use their own slots need.
static bool rh_in_fiber = false;
static ucontext_t rh_sched;
static std::vector<ucontext_t> rh_fiber;
static std::vector<char> rh_fiber_done;
static unsigned rh_cur = 0;
static std::function<void()> rh_fiber_fn;
static void rh_fiber_entry() {
    unsigned t = rh_cur;
    rh_fiber_fn();
    rh_fiber_done[t] = 1;          // returns to rh_sched through uc_link
}
static inline void __syncthreads() {
    if (rh_in_fiber) swapcontext(&rh_fiber[rh_cur], &rh_sched);
}
template <class F>
static void host_launch_sync(unsigned grid, unsigned block, F&& f) {
    static std::vector<std::vector<char>> stacks;
    const size_t stack_bytes = 64 * 1024;
    if (stacks.size() < block) stacks.resize(block);
    for (auto& st : stacks) if (st.size() < stack_bytes) st.assign(stack_bytes, 0);
    rh_fiber.assign(block, ucontext_t());
    rh_fiber_fn = f;
    gridDim = dim3(grid);
    blockDim = dim3(block);
    for (unsigned b = 0; b < grid; b++) {
        blockIdx = make_uint3(b, 0, 0);
        rh_fiber_done.assign(block, 0);
        for (unsigned t = 0; t < block; t++) {
            getcontext(&rh_fiber[t]);
            rh_fiber[t].uc_stack.ss_sp = stacks[t].data();
            rh_fiber[t].uc_stack.ss_size = stack_bytes;
            rh_fiber[t].uc_link = &rh_sched;
            makecontext(&rh_fiber[t], rh_fiber_entry, 0);
        }
        rh_in_fiber = true;
        for (bool all_done = false; !all_done;) {
            all_done = true;
            for (unsigned t = 0; t < block; t++) {
                if (rh_fiber_done[t]) continue;
                rh_cur = t;
                threadIdx = make_uint3(t, 0, 0);
                swapcontext(&rh_sched, &rh_fiber[t]);
                all_done = all_done && rh_fiber_done[t];
            }
        }
        rh_in_fiber = false;
    }
}

static inline int __mul24(int a, int b) { return a * b; }
static inline unsigned __umul24(unsigned a, unsigned b) { return a * b; }
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }

// CUDA's min/max overloads for the mixed argument types the kernels use
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }
static inline unsigned min(unsigned a, unsigned b) { return a < b ? a : b; }
static inline float max(float a, float b) { return fmaxf(a, b); }
static inline float min(float a, float b) { return fminf(a, b); }
static inline float max(int a, float b) { return fmaxf((float)a, b); }
static inline float max(float a, int b) { return fmaxf(a, (float)b); }
static inline float min(int a, float b) { return fminf((float)a, b); }
static inline float min(float a, int b) { return fminf(a, (float)b); }
static inline double max(float a, double b) { return fmax((double)a, b); }
static inline double max(double a, float b) { return fmax(a, (double)b); }
static inline double min(float a, double b) { return fmin((double)a, b); }
static inline double min(double a, float b) { return fmin(a, (double)b); }

// atomics: sequential read-modify-write, returning the old value.  With
// rh_defer_atomics set, float adds are logged instead and applied, in launch
// order, by rh_apply_atomics() after the launch: every thread then reads the
// arrays as they were before the launch.
struct RHAtomic { float* a; float v; };
static bool rh_defer_atomics = false;
static std::vector<RHAtomic> rh_atomic_log;
static inline float atomicAdd(float* a, float v) {
    float o = *a;
    if (rh_defer_atomics) rh_atomic_log.push_back({a, v});
    else *a = o + v;
    return o;
}
static inline void rh_apply_atomics() {
    for (auto& r : rh_atomic_log) *r.a = *r.a + r.v;
    rh_atomic_log.clear();
}
static inline int atomicAdd(int* a, int v) { int o = *a; *a = o + v; return o; }
static inline unsigned atomicAdd(unsigned* a, unsigned v) { unsigned o = *a; *a = o + v; return o; }
static inline int atomicCAS(int* a, int cmp, int v) { int o = *a; if (o == cmp) *a = v; return o; }
static inline unsigned atomicCAS(unsigned* a, unsigned cmp, unsigned v) { unsigned o = *a; if (o == cmp) *a = v; return o; }
static inline int atomicExch(int* a, int v) { int o = *a; *a = v; return o; }
static inline float atomicExch(float* a, float v) { float o = *a; *a = v; return o; }
static inline int atomicMax(int* a, int v) { int o = *a; if (v > o) *a = v; return o; }
static inline int atomicMin(int* a, int v) { int o = *a; if (v < o) *a = v; return o; }
static inline int __float_as_int(float f) { int i; memcpy(&i, &f, 4); return i; }
static inline float __int_as_float(int i) { float f; memcpy(&f, &i, 4); return f; }

struct HostTex { const unsigned* p = nullptr; };
template <class T> static inline T tex1Dfetch(const HostTex& t, int i) { return (T)t.p[i]; }
static inline unsigned tex1Dfetch(const HostTex& t, int i) { return t.p[i]; }

// ---- helper_math.h float3 arithmetic, restated ------------------------------
static inline float3 make_float3(float s) { return make_float3(s, s, s); }
static inline float3 make_float3(int3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
static inline float3 make_float3(uint3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
static inline float3 make_float3(float4 a) { return make_float3(a.x, a.y, a.z); }
static inline float4 make_float4(float3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
static inline int3 make_int3(float3 a) { return make_int3((int)a.x, (int)a.y, (int)a.z); }
static inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
static inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float3 operator+(float3 a, float b) { return make_float3(a.x + b, a.y + b, a.z + b); }
static inline float3 operator+(float b, float3 a) { return make_float3(a.x + b, a.y + b, a.z + b); }
static inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float3 operator-(float3 a, float b) { return make_float3(a.x - b, a.y - b, a.z - b); }
static inline float3 operator-(float b, float3 a) { return make_float3(b - a.x, b - a.y, b - a.z); }
static inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float3 operator*(float3 a, float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
static inline float3 operator*(float b, float3 a) { return make_float3(b * a.x, b * a.y, b * a.z); }
static inline float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline float3 operator/(float3 a, float b) { return make_float3(a.x / b, a.y / b, a.z / b); }
static inline float3 operator/(float b, float3 a) { return make_float3(b / a.x, b / a.y, b / a.z); }
static inline void operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
static inline void operator+=(float3& a, float b) { a.x += b; a.y += b; a.z += b; }
static inline void operator-=(float3& a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
static inline void operator-=(float3& a, float b) { a.x -= b; a.y -= b; a.z -= b; }
static inline void operator*=(float3& a, float3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; }
static inline void operator*=(float3& a, float b) { a.x *= b; a.y *= b; a.z *= b; }
static inline void operator/=(float3& a, float3 b) { a.x /= b.x; a.y /= b.y; a.z /= b.z; }
static inline void operator/=(float3& a, float b) { a.x /= b; a.y /= b; a.z /= b; }
static inline int3 operator+(int3 a, int3 b) { return make_int3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline int3 operator-(int3 a, int3 b) { return make_int3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(float3 v) { return sqrtf(dot(v, v)); }
static inline float3 normalize(float3 v) { float inv = rsqrtf(dot(v, v)); return v * inv; }
static inline float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float lerp(float a, float b, float t) { return a + t * (b - a); }
static inline float3 lerp(float3 a, float3 b, float t) { return a + t * (b - a); }
static inline float3 fminf(float3 a, float3 b) { return make_float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
static inline float3 fmaxf(float3 a, float3 b) { return make_float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
static inline float clamp(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }
static inline float3 clamp(float3 v, float a, float b) { return make_float3(clamp(v.x, a, b), clamp(v.y, a, b), clamp(v.z, a, b)); }
static inline float3 floorf(float3 v) { return make_float3(floorf(v.x), floorf(v.y), floorf(v.z)); }
static inline float3 fabs(float3 v) { return make_float3(fabsf(v.x), fabsf(v.y), fabsf(v.z)); }

// make_float3(a, b, c) as a braced initializer, so that its arguments are
// evaluated left to right.  C++ leaves the order of a call's argument
// evaluation unspecified and g++ evaluates them right to left; the reference
// reads three consecutive random numbers inside one make_float3 call
// (GenerateGasParticle_k's randpos), which the oracle defines as x, y, z in
// table order.
static inline float3 rh_make_float3_1(float s) { return make_float3(s, s, s); }
static inline float3 rh_make_float3_1(int3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
static inline float3 rh_make_float3_1(uint3 a) { return make_float3((float)a.x, (float)a.y, (float)a.z); }
static inline float3 rh_make_float3_1(float4 a) { return make_float3(a.x, a.y, a.z); }
#define RH_F3_3(a, b, c) (float3{(float)(a), (float)(b), (float)(c)})
#define RH_F3_1(a) rh_make_float3_1(a)
#define RH_F3_PICK(_1, _2, _3, NAME, ...) NAME
#define make_float3(...) RH_F3_PICK(__VA_ARGS__, RH_F3_3, RH_F3_2_UNUSED, RH_F3_1)(__VA_ARGS__)
