// k_p2g.cu — particle <-> grid transfers as gathers over the sorted particles.
//
// P2G: mapvelp2g_k_fluidSolid / mapvelp2g_k_air (Multiphase/Multiphase/
// spray_k.cu:2809-2937): a face takes the mass- and sharp-kernel-weighted mean
// velocity of the particles in a window of cells; no atomics. One thread owns
// the x-, y- and z-face with the same (i,j,k) and walks the union of their
// three windows once, in the reference's (di,dj,dk,particle) order; each face
// accumulates only the cells of its own window, so every face sees exactly
// the reference's summation order while every particle is read once.
// Drag: calDragForce (spray_k.cu:5127-5165) adds six face contributions per
// solo-air particle with float atomics; here a per-particle kernel computes
// the contributions and a per-face gather adds them in ascending particle
// order. G2P: computeDeltaU (spray_k.cu:997-1006) + mapvelg2p_flip_bubble
// (spray_k.cu:3525-3540). Heat: mapHeatp2g_hash (spray_k.cu:4619-4653),
// mapHeatg2p[_MeltAndBoil] (spray_k.cu:4655-4679).
#include "ctx.cuh"

using namespace mpk;

namespace {

// The air P2G (mapvelp2g_k_air, spray_k.cu:2894-2937): AIR particles, window
// -2..1 along the face normal and -2..2 across (100 cells). One thread owns the
// x-, y- and z-face with the same (i,j,k) and walks the union of their windows
// once; each face accumulates only the cells of its own window, in the
// reference's (di,dj,dk,particle) order. Bubbles are sparse, so each cell's type
// mask is tested first and only cells with an AIR particle are walked.
// sharp_kernel(r2, 1.4) is exactly zero once r2 exceeds 1.4^2, and a zero
// weight adds +-0 to both sums, so such pairs are skipped, and the velocity is
// read only when some face takes the particle.
// A face triple whose 5x5x5-cell window touches no 4x4x4-cell brick holding an
// air particle (the bit map of the last sort) has no pair: its faces take 0,
// as the walk would give them.
__global__ void __launch_bounds__(256, 4) k_p2g_air(Grid g, Cells cl, const float4* __restrict__ pos,
                                                    const float4* __restrict__ vel, float* __restrict__ ux,
                                                    float* __restrict__ uy, float* __restrict__ uz,
                                                    const uint32_t* __restrict__ air_brick) {
    constexpr int R = 2;       // union window -R..R
    constexpr int HI = 1;      // upper bound along the face normal
    const Tiles T = make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1);
    const float scale = 1.0f / g.h;
    const float cut = (1.4f * 1.4f) * 1.0001f;
    MP_GRID_LOOP(t, T.threads()) {
        int i, j, k; if (!tile_ijk(T, t, i, j, k)) continue;
        bool hx = (j < g.NY && k < g.NZ), hy = (i < g.NX && k < g.NZ), hz = (i < g.NX && j < g.NY);
        float wx = 0, sx = 0, wy = 0, sy = 0, wz = 0, sz = 0;
        bool air_near = false;
        {
            const int bw = (g.NZ + 3) / 4, bh = (g.NY + 3) / 4;
            const int bi0 = max(i - R, 0) >> 2, bi1 = min(i + R, g.NX - 1) >> 2;
            const int bj0 = max(j - R, 0) >> 2, bj1 = min(j + R, g.NY - 1) >> 2;
            const int bk0 = max(k - R, 0) >> 2, bk1 = min(k + R, g.NZ - 1) >> 2;
            for (int bi = bi0; bi <= bi1 && !air_near; bi++)
                for (int bj = bj0; bj <= bj1 && !air_near; bj++)
                    for (int bk = bk0; bk <= bk1; bk++) {
                        const int br = (bi * bh + bj) * bw + bk;
                        if ((__ldg(air_brick + (br >> 5)) >> (br & 31)) & 1u) { air_near = true; break; }
                    }
        }
        if (!air_near) {
            if (hx) ux[fxi(g, i, j, k)] = 0.0f;
            if (hy) uy[fyi(g, i, j, k)] = 0.0f;
            if (hz) uz[fzi(g, i, j, k)] = 0.0f;
            continue;
        }
        const float3 gpx = mk3((float)i, (float)j + 0.5f, (float)k + 0.5f);
        const float3 gpy = mk3((float)i + 0.5f, (float)j, (float)k + 0.5f);
        const float3 gpz = mk3((float)i + 0.5f, (float)j + 0.5f, (float)k);
        const int klo = max(k - R, 0), khi = min(k + R, g.NZ - 1);
        for (int di = -R; di <= R; di++) {
            int a = i + di; if (a < 0 || a > g.NX - 1) continue;
            const bool ax = hx && di <= HI;
            for (int dj = -R; dj <= R; dj++) {
                int b = j + dj; if (b < 0 || b > g.NY - 1) continue;
                const bool ay = hy && dj <= HI;
                if (!(ax || ay || hz)) continue;
                const int cb = cid(g, a, b, 0);
                for (int cc = klo; cc <= khi; cc++) {
                    const bool az = hz && cc - k <= HI;
                    if (!(ax || ay || az)) continue;
                    // the type mask is built at sort time; AIR <-> AIRSOLO flips since then
                    // (markSoloAirParticle) keep the union bit valid
                    if (!(__ldg(cl.tmask + cb + cc) & ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO)))) continue;
                    const uint32_t s1 = __ldg(cl.off + cb + cc + 1);
                    for (uint32_t p = __ldg(cl.off + cb + cc); p < s1; ++p) {
                        const float4 q = __ldg(pos + p);
                        if (pflag(q) != MP_TYPEAIR) continue;
                        const float3 ps = mk3(q.x, q.y, q.z) * scale;
                        const float3 dx = ps - gpx, dy = ps - gpy, dz = ps - gpz;
                        const float r2x = dot(dx, dx), r2y = dot(dy, dy), r2z = dot(dz, dz);
                        const bool tx = ax && r2x <= cut, ty = ay && r2y <= cut, tz = az && r2z <= cut;
                        if (!(tx || ty || tz)) continue;
                        const float4 v = __ldg(vel + p);
                        if (tx) { float w = v.w * sharp_kernel(r2x, 1.4f); wx += w; sx += w * v.x; }
                        if (ty) { float w = v.w * sharp_kernel(r2y, 1.4f); wy += w; sy += w * v.y; }
                        if (tz) { float w = v.w * sharp_kernel(r2z, 1.4f); wz += w; sz += w * v.z; }
                    }
                }
            }
        }
        if (hx) ux[fxi(g, i, j, k)] = (wx > 0) ? (sx / wx) : 0.0f;
        if (hy) uy[fyi(g, i, j, k)] = (wy > 0) ? (sy / wy) : 0.0f;
        if (hz) uz[fzi(g, i, j, k)] = (wz > 0) ? (sz / wz) : 0.0f;
    }
}

#ifndef P2G_CAP
#define P2G_CAP 320
#endif
#ifndef P2G_SMINB
#define P2G_SMINB 2
#endif
// padded slot of the t-th staged particle: one spare float4 per 8, so lanes
// whose ranges start about a cell (8 particles) apart hit different banks
__device__ __forceinline__ uint32_t p2g_slot(uint32_t t) { return t + (t >> 3); }
__host__ __device__ constexpr int p2g_slots(int cap) { return cap + cap / 8; }

// The water P2G (mapvelp2g_k_fluidSolid, spray_k.cu:2829-2892): FLUID and
// SOLID particles, window -1..0 along the face normal and -1..1 across (18
// cells), with each warp's particle loads coalesced.
// A warp holds the nodes (i, j, k0 .. k0+31); for one (di, dj) its lanes'
// windows are overlapping ranges of the cells (a, b, k0-1 .. k0+32), which are
// consecutive in the sorted order. The warp copies that particle range, CAP at
// a time, into shared memory with coalesced loads (scaled position, water test,
// velocity and mass), then each lane walks its own part of the chunk in
// ascending order. Per-lane loads from global memory hit ~32 separate lines per
// warp instruction and saturate L1; the staged reads do not. Every face adds
// the same particles in the same order with the same arithmetic as
// the one-thread-per-face-triple gather, so the fields are bit-identical.
template <int CAP>
__global__ void __launch_bounds__(256, P2G_SMINB) k_p2g_water(Grid g, Cells cl, const float4* __restrict__ pos,
                                                              const float4* __restrict__ vel, float* __restrict__ ux,
                                                              float* __restrict__ uy, float* __restrict__ uz) {
    extern __shared__ float4 p2g_sm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float4* sp = p2g_sm + (size_t)warp * 2 * p2g_slots(CAP);   // (x, y, z) / h and the water test
    float4* sv = sp + p2g_slots(CAP);                           // velocity and mass
    const Tiles T = make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1);
    const float scale = 1.0f / g.h;
    const float cut = (1.4f * 1.4f) * 1.0001f;
    // T.threads() is a multiple of 256 and so is the stride: a warp's lanes run
    // the same iterations, and every lane takes part in the staging
    MP_GRID_LOOP(t, T.threads()) {
        int i, j, k;
        const bool act = tile_ijk(T, t, i, j, k);
        // i and j are the same across the warp, and lane 0 holds the lowest k
        if (!__any_sync(0xffffffffu, act)) continue;
        bool hx = act && (j < g.NY && k < g.NZ), hy = act && (i < g.NX && k < g.NZ), hz = act && (i < g.NX && j < g.NY);
        float wx = 0, sx = 0, wy = 0, sy = 0, wz = 0, sz = 0;
        const float3 gpx = mk3((float)i, (float)j + 0.5f, (float)k + 0.5f);
        const float3 gpy = mk3((float)i + 0.5f, (float)j, (float)k + 0.5f);
        const float3 gpz = mk3((float)i + 0.5f, (float)j + 0.5f, (float)k);
        const int klo = max(k - 1, 0), khi = min(k + 1, g.NZ - 1);
        for (int di = -1; di <= 1; di++) {
            int a = i + di; if (a < 0 || a > g.NX - 1) continue;
            const bool ax = hx && di <= 0;
            for (int dj = -1; dj <= 1; dj++) {
                int b = j + dj; if (b < 0 || b > g.NY - 1) continue;
                const bool ay = hy && dj <= 0;
                const bool need = ax || ay || hz;
                if (!__any_sync(0xffffffffu, need)) continue;
                const int cb = cid(g, a, b, 0);
                uint32_t s0 = 0, s1 = 0, sz0 = 0;
                if (need) {
                    s0 = __ldg(cl.off + cb + klo); s1 = __ldg(cl.off + cb + khi + 1);
                    sz0 = hz ? __ldg(cl.off + cb + min(k, khi) + 1) : s0;
                }
                // the warp's range: from lane 0's first particle to the largest end
                const uint32_t A = __shfl_sync(0xffffffffu, s0, 0);
                const uint32_t B = __reduce_max_sync(0xffffffffu, need ? s1 : A);
                for (uint32_t c0 = A; c0 < B; c0 += CAP) {
                    const uint32_t n = min(B - c0, (uint32_t)CAP);
                    __syncwarp();
                    for (uint32_t u = lane; u < n; u += 32) {
                        const float4 q = __ldg(pos + c0 + u);
                        const int f = pflag(q);
                        const float3 ps = mk3(q.x, q.y, q.z) * scale;
                        sp[p2g_slot(u)] = make_float4(ps.x, ps.y, ps.z, (f == MP_TYPEFLUID || f == MP_TYPESOLID) ? 1.0f : 0.0f);
                        sv[p2g_slot(u)] = __ldg(vel + c0 + u);
                    }
                    __syncwarp();
                    if (!need) continue;
                    const uint32_t lo = max(s0, c0), hi = min(s1, c0 + n);
                    for (uint32_t p = lo; p < hi; ++p) {
                        const float4 q = sp[p2g_slot(p - c0)];
                        if (q.w == 0.0f) continue;
                        const float3 ps = mk3(q.x, q.y, q.z);
                        float3 dx = ps - gpx, dy = ps - gpy, dz = ps - gpz;
                        float r2x = dot(dx, dx), r2y = dot(dy, dy), r2z = dot(dz, dz);
                        bool tx = ax && r2x <= cut, ty = ay && r2y <= cut, tz = p < sz0 && r2z <= cut;
                        if (!(tx || ty || tz)) continue;
                        const float4 v = sv[p2g_slot(p - c0)];
                        if (tx) { float w = v.w * sharp_kernel(r2x, 1.4f); wx += w; sx += w * v.x; }
                        if (ty) { float w = v.w * sharp_kernel(r2y, 1.4f); wy += w; sy += w * v.y; }
                        if (tz) { float w = v.w * sharp_kernel(r2z, 1.4f); wz += w; sz += w * v.z; }
                    }
                }
            }
        }
        if (hx) ux[fxi(g, i, j, k)] = (wx > 0) ? (sx / wx) : 0.0f;
        if (hy) uy[fyi(g, i, j, k)] = (wy > 0) ? (sy / wy) : 0.0f;
        if (hz) uz[fzi(g, i, j, k)] = (wz > 0) ? (sz / wz) : 0.0f;
    }
}

// per-face copies into the *_old fields (the D2D copies of spray.cu:1578-1587)
__global__ void k_copy3(long long n0, long long n1, long long n2, const float* a0, const float* a1, const float* a2,
                        float* b0, float* b1, float* b2) {
    long long tot = n0 + n1 + n2;
    MP_GRID_LOOP(t, tot) {
        if (t < n0) b0[t] = a0[t];
        else if (t < n0 + n1) b1[t - n0] = a1[t - n0];
        else b2[t - n0 - n1] = a2[t - n0 - n1];
    }
}

// calDragForce, part 1: the velocity change each solo-air particle gives the
// water faces, from the field as it is before the stage
__global__ void k_drag_particle(Grid g, int np, const float4* __restrict__ pos, float4* __restrict__ vel,
                                const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
                                float4* __restrict__ dv, float4* __restrict__ wt, float dps, float dpg, float dt,
                                int selfkick) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        if (pflag(q) != MP_TYPEAIRSOLO) continue;
        float3 ip = xyz(q);
        float4 v4 = vel[p];
        float3 iv = xyz(v4);
        int i, j, k; ijkpos(g, ip, i, j, k);
        float3 gv = velFromGrid(g, ip, ux, uy, uz);
        float3 diff = gv - iv;
        float3 dfb = (dps * length(diff)) * diff;
        float3 vcg = (-dfb) * dpg * dt;
        float3 w = ip / g.h - mk3((float)i, (float)j, (float)k);
        dv[p] = make_float4(vcg.x, vcg.y, vcg.z, 0.f);
        wt[p] = make_float4(w.x, w.y, w.z, 0.f);
        if (selfkick) { iv += dfb * dt; vel[p] = make_float4(iv.x, iv.y, iv.z, v4.w); }
    }
}
// part 2: each face adds the contributions of the particles in the two cells
// that touch it, lower cell first (ascending particle order)
__global__ void k_drag_faces(Grid g, Cells cl, const float4* __restrict__ pos, const float4* __restrict__ dv,
                             const float4* __restrict__ wt, float* __restrict__ ux, float* __restrict__ uy,
                             float* __restrict__ uz) {
    const int W = g.NX + 1, Hh = g.NY + 1, D = g.NZ + 1;
    long long tot = (long long)W * Hh * D;
    // union with AIR: the mask predates markSoloAirParticle's AIR -> AIRSOLO flips
    const uint32_t bit = (1u << MP_TYPEAIRSOLO) | (1u << MP_TYPEAIR);
    MP_GRID_LOOP(t, tot) {
        int i, j, k; getijk3((int)t, Hh, D, i, j, k);
        #pragma unroll
        for (int axis = 0; axis < 3; axis++) {
            bool has = axis == 0 ? (j < g.NY && k < g.NZ) : (axis == 1 ? (i < g.NX && k < g.NZ) : (i < g.NX && j < g.NY));
            if (!has) continue;
            int li = i - (axis == 0), lj = j - (axis == 1), lk = k - (axis == 2);   // lower cell
            bool lo_ok = li >= 0 && lj >= 0 && lk >= 0;
            bool hi_ok = i < g.NX && j < g.NY && k < g.NZ;
            int clo = lo_ok ? cid(g, li, lj, lk) : -1, chi = hi_ok ? cid(g, i, j, k) : -1;
            bool any = (clo >= 0 && (__ldg(cl.tmask + clo) & bit)) || (chi >= 0 && (__ldg(cl.tmask + chi) & bit));
            if (!any) continue;
            float* u = axis == 0 ? ux : (axis == 1 ? uy : uz);
            int fidx = axis == 0 ? fxi(g, i, j, k) : (axis == 1 ? fyi(g, i, j, k) : fzi(g, i, j, k));
            float acc = u[fidx];
            if (clo >= 0)
                for (uint32_t p = cl.off[clo]; p < cl.off[clo + 1]; p++) {
                    if (pflag(pos[p]) != MP_TYPEAIRSOLO) continue;
                    float4 d = dv[p], w = wt[p];
                    float dd = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
                    float ww = axis == 0 ? w.x : (axis == 1 ? w.y : w.z);
                    acc += dd * ww;
                }
            if (chi >= 0)
                for (uint32_t p = cl.off[chi]; p < cl.off[chi + 1]; p++) {
                    if (pflag(pos[p]) != MP_TYPEAIRSOLO) continue;
                    float4 d = dv[p], w = wt[p];
                    float dd = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
                    float ww = axis == 0 ? w.x : (axis == 1 ? w.y : w.z);
                    acc += dd * (1 - ww);
                }
            u[fidx] = acc;
        }
    }
}

// computeDeltaU for water and air: old <- new - old
__global__ void k_delta_u(long long n0, long long n1, long long n2, const float* w0, const float* w1, const float* w2,
                          float* o0, float* o1, float* o2, const float* a0, const float* a1, const float* a2,
                          float* q0, float* q1, float* q2) {
    long long tot = n0 + n1 + n2;
    MP_GRID_LOOP(t, tot) {
        if (t < n0) { o0[t] = w0[t] - o0[t]; q0[t] = a0[t] - q0[t]; }
        else if (t < n0 + n1) { long long s = t - n0; o1[s] = w1[s] - o1[s]; q1[s] = a1[s] - q1[s]; }
        else { long long s = t - n0 - n1; o2[s] = w2[s] - o2[s]; q2[s] = a2[s] - q2[s]; }
    }
}

struct FaceSet { const float* x; const float* y; const float* z; };

// mapvelg2p_flip_bubble; alpha < 1 blends with the new grid velocity as
// advectparticle_RK2_bubble does (spray_k.cu:3487-3490)
__global__ void __launch_bounds__(256) k_g2p(Grid g, int np, const float4* __restrict__ pos, float4* __restrict__ vel,
                                             FaceSet dw, FaceSet da, FaceSet uw, FaceSet ua, float alpha) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        float3 ip = xyz(q);
        float4 v = vel[p];
        float3 iv = xyz(v);
        bool water = (f == MP_TYPEFLUID || f == MP_TYPESOLID), air = (f == MP_TYPEAIR);
        float3 gv = mk3(0.0f);
        if (water) gv = velFromGrid(g, ip, dw.x, dw.y, dw.z);
        else if (air) gv = velFromGrid(g, ip, da.x, da.y, da.z);
        if (alpha == 1.0f || !(water || air)) iv += gv;
        else {
            float3 ug = water ? velFromGrid(g, ip, uw.x, uw.y, uw.z) : velFromGrid(g, ip, ua.x, ua.y, ua.z);
            iv = (1 - alpha) * ug + alpha * (iv + gv);
        }
        vel[p] = make_float4(iv.x, iv.y, iv.z, v.w);
    }
}

// mapHeatp2g_hash: cell-centred, 27 cells, all particles, unweighted by mass
__global__ void __launch_bounds__(256) k_heat_p2g(Grid g, Cells cl, const float4* __restrict__ pos,
                                                  const float4* __restrict__ heat, float* __restrict__ Tp, float dflt) {
    const float scale = 1.0f / g.h;
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float3 gp = mk3((float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f);
        float ws = 0, hs = 0;
        for (int di = -1; di <= 1; di++) {
            int a = i + di; if (a < 0 || a > g.NX - 1) continue;
            for (int dj = -1; dj <= 1; dj++) {
                int b = j + dj; if (b < 0 || b > g.NY - 1) continue;
                int k0 = max(k - 1, 0), k1 = min(k + 1, g.NZ - 1);
                uint32_t s0 = __ldg(cl.off + cid(g, a, b, k0)), s1 = __ldg(cl.off + cid(g, a, b, k1) + 1);
                for (uint32_t p = s0; p < s1; ++p) {
                    float4 q = __ldg(pos + p);
                    float3 d = mk3(q.x, q.y, q.z) * scale - gp;
                    float w = sharp_kernel(dot(d, d), 1.4f);
                    ws += w;
                    hs += w * __ldg(&heat[p].x);
                }
            }
        }
        Tp[idx] = (ws > 0) ? (hs / ws) : dflt;
    }
}

__global__ void k_heat_g2p(Grid g, int np, const float4* __restrict__ pos, float4* __restrict__ heat,
                           const float* __restrict__ dT, const float* __restrict__ T, float a, int meltboil) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        float3 ip = xyz(q);
        float4 hh = heat[p];
        float nt = a * (hh.x + scaleFromGrid(g, ip, dT)) + (1 - a) * scaleFromGrid(g, ip, T);
        if (meltboil && pflag(q) == MP_TYPESOLID) hh.x = 0.95f * (hh.x) + 0.05f * nt;
        else hh.x = nt;
        heat[p] = hh;
    }
}

// computeDeltaU on the water faces only (the water mode, spray.cu:362-376)
__global__ void k_delta_u_water(long long n0, long long n1, long long n2, const float* w0, const float* w1,
                                const float* w2, float* o0, float* o1, float* o2) {
    long long tot = n0 + n1 + n2;
    MP_GRID_LOOP(t, tot) {
        if (t < n0) o0[t] = w0[t] - o0[t];
        else if (t < n0 + n1) { long long s = t - n0; o1[s] = w1[s] - o1[s]; }
        else { long long s = t - n0 - n1; o2[s] = w2[s] - o2[s]; }
    }
}
// mapvelg2p_flip (spray_k.cu:242-253): every particle takes the interpolated
// water velocity change, whatever its type
__global__ void k_g2p_flip_all(Grid g, int np, const float4* __restrict__ pos, float4* __restrict__ vel, FaceSet d) {
    MP_GRID_LOOP(p, np) {
        float3 ip = xyz(pos[p]);
        float4 v = vel[p];
        float3 iv = xyz(v) + velFromGrid(g, ip, d.x, d.y, d.z);
        vel[p] = make_float4(iv.x, iv.y, iv.z, v.w);
    }
}

}  // namespace

static Cells cells_of(MpCtx* c) { return Cells{c->cell_off, c->tmask}; }

int k_p2g_faces(MpCtx* c, float** out, int which) {
    const Grid& g = c->G;
    long long tot = make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1).threads();
    if (which == 0) {
        const int smem = 8 * 2 * p2g_slots(P2G_CAP) * (int)sizeof(float4);
        MP_CUDA(c, cudaFuncSetAttribute(k_p2g_water<P2G_CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        k_p2g_water<P2G_CAP><<<mp_blocks(tot, 256), 256, smem, c->stream>>>(g, cells_of(c), c->pos, c->vel, out[0], out[1], out[2]);
    }
    else
        k_p2g_air<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g, cells_of(c), c->pos, c->vel, out[0], out[1], out[2],
                                                              c->air_brick);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// mapvelp2g_bubble (spray.cu:1562-1588)
int k_p2g(MpCtx* c) {
    {
        KtScope kt(c, MP_KT_P2G);
        MP_TRY(k_p2g_faces(c, c->wu, 0));
        MP_TRY(k_p2g_faces(c, c->au, 1));
    }
    const Grid& g = c->G;
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    k_copy3<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g.nfx, g.nfy, g.nfz, c->wu[0], c->wu[1], c->wu[2], c->wuo[0], c->wuo[1], c->wuo[2]);
    k_copy3<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g.nfx, g.nfy, g.nfz, c->au[0], c->au[1], c->au[2], c->auo[0], c->auo[1], c->auo[2]);
    c->launches += 2;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// mapvelp2g of the water mode (spray.cu:340-353): the water faces, then
// their copy for the FLIP update (velmode FLIP)
int k_water_p2g(MpCtx* c) {
    {
        KtScope kt(c, MP_KT_P2G);
        MP_TRY(k_p2g_faces(c, c->wu, 0));
    }
    const Grid& g = c->G;
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    k_copy3<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g.nfx, g.nfy, g.nfz, c->wu[0], c->wu[1], c->wu[2], c->wuo[0],
                                                        c->wuo[1], c->wuo[2]);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// mapvelg2p of the water mode (spray.cu:362-376): computeDeltaU on the water
// faces, then mapvelg2p_flip
int k_water_g2p(MpCtx* c) {
    const Grid& g = c->G;
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    k_delta_u_water<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g.nfx, g.nfy, g.nfz, c->wu[0], c->wu[1], c->wu[2],
                                                                c->wuo[0], c->wuo[1], c->wuo[2]);
    c->launches++;
    int np = c->np();
    if (np > 0) {
        KtScope kt(c, MP_KT_G2P);
        k_g2p_flip_all<<<mp_blocks(np, 256), 256, 0, c->stream>>>(g, np, c->pos, c->vel,
                                                                  FaceSet{c->wuo[0], c->wuo[1], c->wuo[2]});
        c->launches++;
    }
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// enforceDragForce (spray.cu:2953-2957)
int k_drag(MpCtx* c) {
    int np = c->np();
    if (np == 0) return MP_OK;
    const Grid& g = c->G;
    int sk = (c->P.scene == MP_SCENE_INTERACTION || c->P.scene == MP_SCENE_INTERACTION_HIGHRES) ? 1 : 0;
    k_drag_particle<<<mp_blocks(np, 256), 256, 0, c->stream>>>(g, np, c->pos, c->vel, c->wu[0], c->wu[1], c->wu[2],
                                                               c->pscr, c->pscr2, c->P.drag_param_solo,
                                                               c->P.drag_param_grid, c->P.dt, sk);
    long long tot = (long long)(g.NX + 1) * (g.NY + 1) * (g.NZ + 1);
    k_drag_faces<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g, cells_of(c), c->pos, c->pscr, c->pscr2,
                                                             c->wu[0], c->wu[1], c->wu[2]);
    c->launches += 2;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_delta_u(MpCtx* c) {
    const Grid& g = c->G;
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    k_delta_u<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(g.nfx, g.nfy, g.nfz, c->wu[0], c->wu[1], c->wu[2],
                                                          c->wuo[0], c->wuo[1], c->wuo[2], c->au[0], c->au[1], c->au[2],
                                                          c->auo[0], c->auo[1], c->auo[2]);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// mapvelg2p_bubble (spray.cu:1689-1705)
int k_g2p(MpCtx* c) {
    MP_TRY(k_delta_u(c));
    int np = c->np();
    if (np == 0) return MP_OK;
    KtScope kt(c, MP_KT_G2P);
    FaceSet dw{c->wuo[0], c->wuo[1], c->wuo[2]}, da{c->auo[0], c->auo[1], c->auo[2]};
    FaceSet uw{c->wu[0], c->wu[1], c->wu[2]}, ua{c->au[0], c->au[1], c->au[2]};
    k_g2p<<<mp_blocks(np, 256), 256, 0, c->stream>>>(c->G, np, c->pos, c->vel, dw, da, uw, ua, c->P.flip_alpha);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_heat_p2g_launch(MpCtx* c) {
    k_heat_p2g<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, cells_of(c), c->pos, c->heat, c->Tp,
                                                              c->P.default_temperature);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_heat_g2p_launch(MpCtx* c) {
    int np = c->np();
    if (np == 0) return MP_OK;
    int sc = c->P.scene;
    int mab = (sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL) ? 1 : 0;
    k_heat_g2p<<<mp_blocks(np, 256), 256, 0, c->stream>>>(c->G, np, c->pos, c->heat, c->Tp_save, c->Tp,
                                                          c->P.alpha_temp_trans, mab);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}
