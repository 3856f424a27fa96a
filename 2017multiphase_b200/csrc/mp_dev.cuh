// mp_dev.cuh — device-side helpers shared by the kernels of the B200 step.
//
// The float3 arithmetic restates helper_math.h from the CUDA samples, which
// the reference kernels use (Multiphase/Multiphase/spray_k.cu:4): same
// operations, same left-to-right evaluation. The library is compiled with
// -fmad=false so that a*b+c is two rounded operations, as in the reference
// source text; normalize() divides by sqrtf instead of multiplying by the
// approximate rsqrtf so that the result is reproducible.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mp.h"

#define MPD __device__ __forceinline__

namespace mpk {

// ---- float3 ------------------------------------------------------------------
MPD float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
MPD float3 mk3(float s) { return make_float3(s, s, s); }
MPD float3 operator+(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
MPD float3 operator-(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
MPD float3 operator-(float3 a) { return mk3(-a.x, -a.y, -a.z); }
MPD float3 operator*(float3 a, float3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
MPD float3 operator/(float3 a, float3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
MPD float3 operator*(float3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
MPD float3 operator*(float s, float3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
MPD float3 operator/(float3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
MPD void operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
MPD void operator-=(float3& a, float3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
MPD void operator*=(float3& a, float s) { a.x *= s; a.y *= s; a.z *= s; }
MPD void operator/=(float3& a, float s) { a.x /= s; a.y /= s; a.z /= s; }
MPD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MPD float length(float3 v) { return sqrtf(dot(v, v)); }
MPD float3 normalize(float3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return v * inv; }
MPD float3 cross(float3 a, float3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
MPD float3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }

// particle packing: pos4 = (x, y, z, flag bits), vel4 = (vx, vy, vz, mass),
// heat4 = (temperature, latent heat, solubility, gas content)
MPD int pflag(float4 p) { return __float_as_int(p.w); }
MPD float flagbits(int f) { return __int_as_float(f); }

// ---- grid geometry, passed by value to every kernel --------------------------
struct Grid {
    int NX, NY, NZ, n, nfx, nfy, nfz;
    float h;
    float gx0, gy0, gz0;       // domain origin
};

MPD int cid(const Grid& g, int i, int j, int k) { return i * g.NY * g.NZ + j * g.NZ + k; }
MPD bool vc(const Grid& g, int i, int j, int k) {
    return !(i < 0 || i > g.NX - 1 || j < 0 || j > g.NY - 1 || k < 0 || k > g.NZ - 1);
}
MPD void getijk(const Grid& g, int idx, int& i, int& j, int& k) {
    i = idx / (g.NZ * g.NY); j = idx / g.NZ % g.NY; k = idx % g.NZ;
}
// getijk(i,j,k,idx,w,h,d) of utility.h:90-95
MPD void getijk3(int idx, int hh, int d, int& i, int& j, int& k) {
    i = idx / d / hh; j = idx / d % hh; k = idx % d;
}
// getijkfrompos (spray_k.cu:51-57): an axis outside the grid maps to 0
MPD void ijkpos(const Grid& g, float3 p, int& i, int& j, int& k) {
    p = (p - mk3(g.gx0, g.gy0, g.gz0)) / mk3(g.h, g.h, g.h);
    i = (p.x >= 0 && p.x < g.NX) ? (int)p.x : 0;
    j = (p.y >= 0 && p.y < g.NY) ? (int)p.y : 0;
    k = (p.z >= 0 && p.z < g.NZ) ? (int)p.z : 0;
}
// not on the outer cell shell; the shell is always BOUNDARY in a valid state,
// so kernels that read +-1 neighbours use this only as a memory-safety guard
MPD bool interior(const Grid& g, int idx) {
    int i, j, k; getijk(g, idx, i, j, k);
    return i > 0 && i < g.NX - 1 && j > 0 && j < g.NY - 1 && k > 0 && k < g.NZ - 1;
}
MPD int fxi(const Grid& g, int i, int j, int k) { return i * g.NY * g.NZ + j * g.NZ + k; }
MPD int fyi(const Grid& g, int i, int j, int k) { return i * (g.NY + 1) * g.NZ + j * g.NZ + k; }
MPD int fzi(const Grid& g, int i, int j, int k) { return i * g.NY * (g.NZ + 1) + j * (g.NZ + 1) + k; }

// trilinear (spray_k.cu:111-122) on an array of dims (w, hh, d)
MPD float trilinear(const float* __restrict__ u, float x, float y, float z, int w, int hh, int d) {
    x = fmaxf(0.0f, fminf(x, (float)w));
    y = fmaxf(0.0f, fminf(y, (float)hh));
    z = fmaxf(0.0f, fminf(z, (float)d));
    int i = (int)fminf(x, (float)(w - 2));
    int j = (int)fminf(y, (float)(hh - 2));
    int k = (int)fminf(z, (float)(d - 2));
    int b = i * hh * d + j * d + k;
    int sj = d, si = hh * d;
    float u000 = __ldg(u + b), u100 = __ldg(u + b + si), u010 = __ldg(u + b + sj), u110 = __ldg(u + b + si + sj);
    float u001 = __ldg(u + b + 1), u101 = __ldg(u + b + si + 1), u011 = __ldg(u + b + sj + 1), u111 = __ldg(u + b + si + sj + 1);
    float fi1 = (float)(i + 1) - x, fi0 = x - (float)i;
    float fj1 = (float)(j + 1) - y, fj0 = y - (float)j;
    return ((float)(k + 1) - z) * (fj1 * (fi1 * u000 + fi0 * u100) + fj0 * (fi1 * u010 + fi0 * u110))
         + (z - (float)k) * (fj1 * (fi1 * u001 + fi0 * u101) + fj0 * (fi1 * u011 + fi0 * u111));
}
// getParticleVelFromGrid (spray_k.cu:227-240)
MPD float3 velFromGrid(const Grid& g, float3 p, const float* ux, const float* uy, const float* uz) {
    float x = p.x / g.h, y = p.y / g.h, z = p.z / g.h;
    return mk3(trilinear(ux, x, y - 0.5f, z - 0.5f, g.NX + 1, g.NY, g.NZ),
               trilinear(uy, x - 0.5f, y, z - 0.5f, g.NX, g.NY + 1, g.NZ),
               trilinear(uz, x - 0.5f, y - 0.5f, z, g.NX, g.NY, g.NZ + 1));
}
// getScaleFromFrid (spray_k.cu:140-153)
MPD float scaleFromGrid(const Grid& g, float3 p, const float* f) {
    float x = p.x / g.h, y = p.y / g.h, z = p.z / g.h;
    return trilinear(f, x - 0.5f, y - 0.5f, z - 0.5f, g.NX, g.NY, g.NZ);
}
// getVectorFromGrid (spray_k.cu:124-138)
MPD float3 vecFromGrid(const Grid& g, float3 p, const float* a, const float* b, const float* c) {
    float x = p.x / g.h, y = p.y / g.h, z = p.z / g.h;
    return mk3(trilinear(a, x - 0.5f, y - 0.5f, z - 0.5f, g.NX, g.NY, g.NZ),
               trilinear(b, x - 0.5f, y - 0.5f, z - 0.5f, g.NX, g.NY, g.NZ),
               trilinear(c, x - 0.5f, y - 0.5f, z - 0.5f, g.NX, g.NY, g.NZ));
}
MPD float sharp_kernel(float r2, float hh) {   // spray_k.cu:255-258
    return fmaxf(hh * hh / fmaxf(r2, 0.0001f) - 1.0f, 0.0f);
}
MPD float smooth_kernel(float r2, float hh) {  // spray_k.cu:1330-1332
    return fmaxf(1.0f - r2 / (hh * hh), 0.0f);
}

// cell ranges of the sorted particle array: CSR offsets off[c]..off[c+1]
struct Cells {
    const uint32_t* __restrict__ off;
    const uint8_t* __restrict__ tmask;   // bit t set if the cell holds a particle of type t
};

// 3-D tiles of 2 x 4 x 32 (i, j, k) points per 256-thread block, k fastest, so a
// warp covers 32 consecutive k and a block's gather window (the union of its
// points' neighbour cells) is compact, which lets L1 serve most re-reads.
constexpr int TILE_I = 2, TILE_J = 4, TILE_K = 32;
struct Tiles {
    int W, H, D;        // points along i, j, k
    int ti, tj, tk;     // tiles along i, j, k
    __host__ __device__ long long threads() const { return (long long)ti * tj * tk * 256; }
};
__host__ __device__ inline Tiles make_tiles(int W, int H, int D) {
    return Tiles{W, H, D, (W + TILE_I - 1) / TILE_I, (H + TILE_J - 1) / TILE_J, (D + TILE_K - 1) / TILE_K};
}
MPD bool tile_ijk(const Tiles& T, int t, int& i, int& j, int& k) {
    int tile = t >> 8, o = t & 255;
    int a = tile % T.tk, r = tile / T.tk;
    int b = r % T.tj, c = r / T.tj;
    k = a * TILE_K + (o & 31);
    j = b * TILE_J + ((o >> 5) & 3);
    i = c * TILE_I + (o >> 7);
    return i < T.W && j < T.H && k < T.D;
}

// grid-stride loop with a 32-bit index (every element count here is below 2^31
// minus one grid stride; mp_create rejects grids that could exceed it)
#define MP_GRID_LOOP(idx, N) for (int idx = (int)(blockIdx.x * blockDim.x + threadIdx.x); idx < (int)(N); idx += (int)(gridDim.x * blockDim.x))

// Sorts the DISTINCT values a[s0 .. s0+cnt) ascending and calls each(v) once
// per value. Up to RUN_REG values are loaded together into registers and each
// is stored at its rank (the count of smaller values), so a short run costs
// one round trip to memory instead of a chain of dependent ones; longer runs
// use an insertion sort in place.
constexpr int RUN_REG = 16;
template <class F>
__device__ __forceinline__ void sort_distinct_run(uint32_t* a, uint32_t s0, uint32_t cnt, F each) {
    if (cnt <= (uint32_t)RUN_REG) {
        uint32_t v[RUN_REG];
        #pragma unroll
        for (int q = 0; q < RUN_REG; q++) v[q] = (q < (int)cnt) ? a[s0 + q] : 0xffffffffu;
        #pragma unroll
        for (int q = 0; q < RUN_REG; q++) {
            if (q < (int)cnt) {
                uint32_t rk = 0;
                #pragma unroll
                for (int t = 0; t < RUN_REG; t++) rk += (v[t] < v[q]) ? 1u : 0u;
                a[s0 + rk] = v[q];
                each(v[q]);
            }
        }
        return;
    }
    const uint32_t s1 = s0 + cnt;
    for (uint32_t s = s0 + 1; s < s1; s++) {
        uint32_t x = a[s], t = s;
        while (t > s0 && a[t - 1] > x) { a[t] = a[t - 1]; t--; }
        a[t] = x;
    }
    for (uint32_t s = s0; s < s1; s++) each(a[s]);
}

}  // namespace mpk
