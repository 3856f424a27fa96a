// k_part.cu — per-particle stages of the step.
//
// Reference kernels (Multiphase/Multiphase/spray_k.cu): addgravityforce_k 330,
// addbuoyancyforce_vel 356, verifySoloAirParticle 4223, enforcesurfacetension_p
// 3639, calcDensPress_Air 4284, enforceForceSoloAirP 4335, CollisionWithSolid_k
// 5276, CollisionWithSolid_Freezing 5348, correctparticlepos 1357,
// correctbubblepos 3884, correctbubblepos_air 3941, setVelZeroSolid_k 5213,
// solidCollisionWithBound 5478, compute_cI_k 5188, computeVelSolid_k 5220,
// computePosSolid_k 5243, updateLatentHeat_k 5546, initHeatParticle 4681,
// initsolubility_k 4700, updatesolubility 4719, GenerateGasParticle_k 4730,
// sweepVacuum 4117, markDeleteAirParticle 4134, deleteparticles 4172,
// MeltingSolidByHeat 5059, FreezingSolidByHeat 5074.
// Kernels that read neighbours while the reference writes them in place
// (enforceForceSoloAirP, CollisionWithSolid_Freezing, FreezingSolidByHeat,
// sweepVacuum) read a snapshot here; the gas append is ordered by cell.
#include "ctx.cuh"
#include <cmath>

using namespace mpk;

namespace {

__device__ __forceinline__ float4 with_xyz(float4 v, float3 a) { return make_float4(a.x, a.y, a.z, v.w); }

__global__ void k_forces(int np, const float4* __restrict__ pos, float4* __restrict__ vel, float dt, float gx, float gy,
                         float gz, float velMax, float bra, float brs) {
    MP_GRID_LOOP(p, np) {
        int f = pflag(pos[p]);
        float4 v = vel[p];
        float3 iv = xyz(v);
        if (f == MP_TYPEFLUID || f == MP_TYPESOLID) iv += dt * mk3(gx, gy, gz);
        float rate = fmaxf(velMax - iv.z, 0.0f) / velMax;
        if (f == MP_TYPEAIR) iv.z -= dt * gz * rate * bra;
        else if (f == MP_TYPEAIRSOLO) iv.z -= dt * gz * rate * brs;
        else if (f == MP_TYPESOLID) iv.z += dt * gz * 0.1f;
        vel[p] = with_xyz(v, iv);
    }
}

__device__ __forceinline__ bool in_boundary_cell(const Grid& g, int x, int y) {
    const int lv = 2;
    return x <= lv || x >= g.NX - 1 - lv || y <= lv || y >= g.NY - 1 - lv;
}

// AIR <-> AIRSOLO transitions. Neighbour flags may flip between the two air
// types while this runs; both are counted alike, so the result is unaffected.
__global__ void k_solo_air(Grid g, Cells cl, int np, float4* __restrict__ pos, float4* __restrict__ vel,
                           const float* __restrict__ lsm, const float* __restrict__ ax, const float* __restrict__ ay,
                           const float* __restrict__ az, float tol1, float tol2) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f == MP_TYPEFLUID || f == MP_TYPESOLID) continue;
        float3 ip = xyz(q);
        float ls = scaleFromGrid(g, ip, lsm);
        float h = g.h;
        int i, j, k; ijkpos(g, ip, i, j, k);
        int cnt = 0;
        for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
            if (!vc(g, i + di, j + dj, k + dk)) continue;
            int c = cid(g, i + di, j + dj, k + dk);
            if (!(cl.tmask[c] & ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO)))) continue;
            for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                float4 o = pos[s];
                int fo = pflag(o);
                float d = length(xyz(o) - ip);
                if (d < h && (fo == MP_TYPEAIR || fo == MP_TYPEAIRSOLO)) ++cnt;
            }
        }
        bool ib = in_boundary_cell(g, i, j);
        if ((cnt >= 10 || ls > tol1 * h) && f == MP_TYPEAIRSOLO && !ib) {
            if (cnt >= 3) pos[p] = make_float4(q.x, q.y, q.z, flagbits(MP_TYPEAIR));
        } else if (f == MP_TYPEAIR && (ib || ls < tol2 * h || cnt <= 1)) {
            float3 nv = velFromGrid(g, ip, ax, ay, az);
            vel[p] = with_xyz(vel[p], nv);
            pos[p] = make_float4(q.x, q.y, q.z, flagbits(MP_TYPEAIRSOLO));
        }
    }
}

__global__ void k_st_particles(Grid g, int np, const float4* __restrict__ pos, float4* __restrict__ vel,
                               const float* __restrict__ lsm, const float* __restrict__ sf, const float* __restrict__ gx,
                               const float* __restrict__ gy, const float* __restrict__ gz, const int8_t* __restrict__ mark,
                               int scene, float dt) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f == MP_TYPESOLID || f == MP_TYPEFLUID) continue;
        if ((scene != MP_SCENE_MELTANDBOIL && scene != MP_SCENE_MELTANDBOIL_HIGHRES && f == MP_TYPEAIRSOLO) ||
            (scene != MP_SCENE_ALL && f == MP_TYPEAIRSOLO)) continue;
        float3 ip = xyz(q);
        float il = scaleFromGrid(g, ip, lsm);
        float isf = scaleFromGrid(g, ip, sf);
        float3 dir = vecFromGrid(g, ip, gx, gy, gz);
        float ld = length(dir);
        if (ld == 0) continue;
        dir /= ld; il /= ld;
        int i, j, k; ijkpos(g, ip, i, j, k);
        int cnt = (mark[cid(g, i, j, k)] == MP_TYPEAIR) ? 1 : 0;
        for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2)
            if (vc(g, i + di, j + dj, k + dk) && mark[cid(g, i + di, j + dj, k + dk)] == MP_TYPEAIR) cnt++;
        if (cnt == 0) continue;
        if (fabsf(il) < g.h) {
            float3 fo = (-isf) * dir;
            float4 v = vel[p];
            float3 iv = xyz(v);
            iv += fo * dt;
            vel[p] = with_xyz(v, iv);
        }
    }
}

// calcDensPress_Air; also snapshots the velocity of air particles for the force pass
__global__ void k_air_dens(Grid g, Cells cl, int np, const float4* __restrict__ pos, const float4* __restrict__ vel,
                           float* __restrict__ dens, float* __restrict__ prs, float4* __restrict__ vsnap, float m0p6,
                           float rho) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f != MP_TYPEAIR && f != MP_TYPEAIRSOLO) continue;
        float3 ip = xyz(q);
        float h = g.h, h2 = h * h;
        int i, j, k; ijkpos(g, ip, i, j, k);
        float d = 0;
        for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
            if (!vc(g, i + di, j + dj, k + dk)) continue;
            int c = cid(g, i + di, j + dj, k + dk);
            float res = 0;
            if (cl.tmask[c] & ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO)))
                for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                    float4 o = pos[s];
                    int fo = pflag(o);
                    if (fo != MP_TYPEAIR && fo != MP_TYPEAIRSOLO) continue;
                    float3 dd = xyz(o) - ip;
                    float d2 = dot(dd, dd);
                    if (d2 < h2) res += powf(h2 - d2, 3.0f);
                }
            d += res;
        }
        d *= m0p6;
        if (d == 0) d = 1.0f;
        dens[p] = 1.0f / d;
        prs[p] = 1.5f * (d - rho * 0.5f);
        vsnap[p] = vel[p];
    }
}
__global__ void k_air_force(Grid g, Cells cl, int np, const float4* __restrict__ pos, float4* __restrict__ vel,
                            const float4* __restrict__ vsnap, const float* __restrict__ dens, const float* __restrict__ prs,
                            float spiky, float vterm, float airm0, float dt) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f != MP_TYPEAIRSOLO && f != MP_TYPEAIR) continue;
        float3 ip = xyz(q);
        float4 v4 = vsnap[p];
        float3 iv = xyz(v4);
        float ipr = prs[p], idn = dens[p], hh = g.h;
        int i, j, k; ijkpos(g, ip, i, j, k);
        float3 force = mk3(0.0f);
        for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
            if (!vc(g, i + di, j + dj, k + dk)) continue;
            int c = cid(g, i + di, j + dj, k + dk);
            float3 res = mk3(0.0f);
            if (cl.tmask[c] & ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO)))
                for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                    float4 o = pos[s];
                    float3 dir = ip - xyz(o);
                    float dis = length(dir);
                    int fo = pflag(o);
                    if (dis > 0 && dis < hh && (fo == MP_TYPEAIRSOLO || fo == MP_TYPEAIR)) {
                        float cc = hh - dis;
                        float pterm = -0.5f * cc * spiky * (ipr + prs[s]) / dis;
                        float dterm = cc * idn * dens[s];
                        res += (pterm * dir + vterm * (xyz(vsnap[s]) - iv)) * dterm;
                    }
                }
            force += res;
        }
        force *= airm0;
        iv += force * dt;
        vel[p] = with_xyz(vel[p], iv);
    }
}

__global__ void k_collide(Grid g, int np, float4* __restrict__ pos, float4* __restrict__ vel, const float* __restrict__ phis,
                          const float* __restrict__ sx, const float* __restrict__ sy, const float* __restrict__ sz,
                          int scene, float bvp, float bpp, float dt) {
    const float h = g.h;
    const float3 g0 = mk3(g.gx0, g.gy0, g.gz0);
    const float3 g1 = g0 + mk3((float)g.NX, (float)g.NY, (float)g.NZ) * h;
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f == MP_TYPESOLID) continue;
        float3 ip = xyz(q);
        float4 v4 = vel[p];
        float3 iv = xyz(v4);
        float iphi = scaleFromGrid(g, ip, phis);
        if (iphi <= 0.5f) {
            float3 sv = velFromGrid(g, ip, sx, sy, sz);
            float3 rv = iv - sv;
            float d = h * 0.5f;
            float3 pg;
            pg.x = scaleFromGrid(g, ip + mk3(d, 0, 0), phis) - scaleFromGrid(g, ip - mk3(d, 0, 0), phis);
            pg.y = scaleFromGrid(g, ip + mk3(0, d, 0), phis) - scaleFromGrid(g, ip - mk3(0, d, 0), phis);
            pg.z = scaleFromGrid(g, ip + mk3(0, 0, d), phis) - scaleFromGrid(g, ip - mk3(0, 0, d), phis);
            if (length(pg) > 0) {
                pg = normalize(pg);
                if (dot(rv, pg) < 0 || scene == MP_SCENE_FREEZING) {
                    iv -= bvp * dot(rv, pg) * pg;
                    if (scene == MP_SCENE_FREEZING) iv -= 0.1f * (rv - dot(rv, pg) * pg);
                }
                ip += bpp * pg * (0.5f - iphi) * h;
            }
        }
        ip += iv * dt;
        float rate = (f == MP_TYPEAIRSOLO) ? 0.8f : 0.5f;
        float3 tmin = g0 + (mk3(h, h, h) + mk3(rate * h));
        float3 tmax = g1 - (mk3(h, h, h) + mk3(rate * h));
        if (ip.x <= tmin.x) { ip.x = tmin.x; iv.x = 0.0f; }
        if (ip.y <= tmin.y) { ip.y = tmin.y; iv.y = 0.0f; }
        if (ip.z <= tmin.z) { ip.z = tmin.z; iv.z = 0.0f; }
        if (ip.x >= tmax.x) { ip.x = tmax.x; iv.x = 0.0f; }
        if (ip.y >= tmax.y) { ip.y = tmax.y; iv.y = 0.0f; }
        if (ip.z >= tmax.z) { ip.z = tmax.z; iv.z = 0.0f; }
        vel[p] = with_xyz(v4, iv);
        pos[p] = with_xyz(q, ip);
    }
}

__global__ void k_collide_freezing(Grid g, Cells cl, int np, const float4* __restrict__ opos, float4* __restrict__ pos,
                                   float4* __restrict__ vel, const float* __restrict__ phis, float samplespace, float dt) {
    const float h = g.h;
    const float3 g0 = mk3(g.gx0, g.gy0, g.gz0);
    const float3 g1 = g0 + mk3((float)g.NX, (float)g.NY, (float)g.NZ) * h;
    MP_GRID_LOOP(p, np) {
        float4 q = opos[p];
        if (pflag(q) == MP_TYPESOLID) continue;
        float3 ip = xyz(q);
        float4 v4 = vel[p];
        float3 iv = xyz(v4);
        int i, j, k; ijkpos(g, ip, i, j, k);
        float iphi = scaleFromGrid(g, ip, phis);
        if (iphi <= 1.0f) {
            float r = 0.25f * h;
            float3 cpos = mk3(0.0f);
            float depth = 0, adh = 0;
            int ccol = 0, cadh = 0;
            float hh = 4 * r;
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(g, i + di, j + dj, k + dk)) continue;
                int c = cid(g, i + di, j + dj, k + dk);
                for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                    float3 o = xyz(opos[s]);
                    float3 dir = ip - o;
                    float dis = length(dir);
                    if (dis > 0 && dis < 2 * r) { cpos += o; depth = fmaxf(depth, 2 * r - dis); ccol++; }
                    else if (dis < hh) { adh += dis; cadh++; }
                }
            }
            float3 nn;
            float d = h * 0.5f;
            nn.x = scaleFromGrid(g, ip + mk3(d, 0, 0), phis) - scaleFromGrid(g, ip - mk3(d, 0, 0), phis);
            nn.y = scaleFromGrid(g, ip + mk3(0, d, 0), phis) - scaleFromGrid(g, ip - mk3(0, d, 0), phis);
            nn.z = scaleFromGrid(g, ip + mk3(0, 0, d), phis) - scaleFromGrid(g, ip - mk3(0, 0, d), phis);
            float3 ov = iv;
            if (length(nn) > 0) {
                nn = normalize(nn);
                if (ccol > 0) {
                    cpos /= (float)ccol;
                    if (length(nn) > 0) { iv -= dot(ov, nn) * nn; ip += depth * nn; }
                } else if (cadh > 0) {
                    float alpha = 0.1f;
                    iv -= nn * alpha * length(iv);
                }
            }
        }
        float3 tmin = g0 + (mk3(h, h, h) + mk3(0.3f * samplespace));
        float3 tmax = g1 - (mk3(h, h, h) + mk3(0.3f * samplespace));
        if (ip.x > tmax.x) { iv.x *= -0.5f; ip.x = tmax.x; }
        if (ip.x < tmin.x) { iv.x *= -0.5f; ip.x = tmin.x; }
        if (ip.y > tmax.y) { iv.y *= -0.5f; ip.y = tmax.y; }
        if (ip.y < tmin.y) { iv.y *= -0.5f; ip.y = tmin.y; }
        if (ip.z > tmax.z) { iv.z *= -0.5f; ip.z = tmax.z; }
        if (ip.z < tmin.z) { iv.z *= -0.5f; ip.z = tmin.z; }
        ip += iv * dt;
        vel[p] = with_xyz(v4, iv);
        pos[p] = with_xyz(q, ip);
    }
}

// correctparticlepos: reads pos, writes out (out of place)
__global__ void __launch_bounds__(256, 6) k_correct_pos(Grid g, Cells cl, int np, const float4* __restrict__ pos, const float4* __restrict__ vel,
                              float4* __restrict__ out, float re, float spring_k, float samplespace, float dt) {
    const float h = g.h;
    const float3 g0 = mk3(g.gx0, g.gy0, g.gz0);
    const float3 g1 = g0 + mk3((float)g.NX, (float)g.NY, (float)g.NZ) * h;
    const float3 tmin = g0 + (mk3(h, h, h) + mk3(0.5f * samplespace));
    const float3 tmax = g1 - (mk3(h, h, h) + mk3(0.5f * samplespace));
    const float re2_skip = re * re * 1.001f;
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f == MP_TYPESOLID || f == MP_TYPEAIRSOLO) { out[p] = q; continue; }
        float3 ip = xyz(q);
        int i, j, k; ijkpos(g, ip, i, j, k);
        float3 spring = mk3(0.0f);
        // With re below half a cell, a neighbour cell on the far side of the
        // particle's own half-cell holds only particles whose d2 exceeds
        // re2_skip (its whole extent is more than 1.002 re away along that
        // axis, with a margin for the rounding of the cell coordinates), so
        // every pair in it would be skipped: the cell is not visited.
        const float3 rel = (ip - g0) / mk3(h, h, h);
        const float cut_lo = 1.002f * (re / h) + 2e-4f;
        auto span = [&](float r, int n, int c, int& lo, int& hi) {
            lo = -1; hi = 1;
            if (r >= 0 && r < (float)n) {
                float fr = r - (float)c;
                if (fr > cut_lo) lo = 0;
                if (1.0f - fr > cut_lo) hi = 0;
            }
        };
        int ilo, ihi, jlo, jhi, klo, khi;
        span(rel.x, g.NX, i, ilo, ihi); span(rel.y, g.NY, j, jlo, jhi); span(rel.z, g.NZ, k, klo, khi);
        // the cells of a (di,dj) column are contiguous: their range bounds are
        // read together, then each cell is summed on its own
        // Two phases keep the warp's lanes together: the scan collects the
        // pairs within re (a few of the ~64 candidates) in visiting order,
        // with the ordinal of their cell; the spring terms of the collected
        // pairs are then formed in that order, each cell's sum added to the
        // total when the next cell starts (a cell without pairs adds +0, a
        // no-op). A full buffer is drained in the middle of the scan.
        constexpr int CP_BUF = 16;
        uint32_t ent[CP_BUF];
        uint8_t eo[CP_BUF];
        int ne = 0, cur = -1;
        float3 s = mk3(0.0f);
        auto drain = [&]() {
            for (int e = 0; e < ne; e++) {
                if ((int)eo[e] != cur) { spring += s; s = mk3(0.0f); cur = eo[e]; }
                const uint32_t t = ent[e];
                float3 o = xyz(__ldg(pos + t));
                float3 dd = o - ip;
                float m = __ldg(&vel[t].w);
                float dist = length(dd);
                float w = m * smooth_kernel(dist * dist, re);
                if (dist > 0.1f * re) s += w * (ip - o) / dist;
            }
            ne = 0;
        };
        const int k0 = max(k + klo, 0), k1 = min(k + khi, g.NZ - 1);
        int ord = 0;
        for (int di = ilo; di <= ihi; di++) for (int dj = jlo; dj <= jhi; dj++) {
            if (!vc(g, i + di, j + dj, k)) continue;
            const int cb = cid(g, i + di, j + dj, k0);
            uint32_t bnd[4];
            #pragma unroll
            for (int q = 0; q < 4; q++) bnd[q] = (q <= k1 - k0 + 1) ? __ldg(cl.off + cb + q) : 0u;
            for (int cc = 0; cc <= k1 - k0; cc++, ord++) {
                for (uint32_t t = bnd[cc]; t < bnd[cc + 1]; ++t) {
                    float3 o = xyz(__ldg(pos + t));
                    float3 dd = o - ip;
                    // beyond re the kernel weight is exactly zero and the pair adds a
                    // signed zero, which leaves the sum unchanged: skip it (exact test
                    // with margin: dist*dist >= re*re whenever d2 > 1.001 re*re)
                    if (dot(dd, dd) > re2_skip) continue;
                    if (ne == CP_BUF) drain();
                    ent[ne] = t; eo[ne] = (uint8_t)ord; ne++;
                }
            }
        }
        drain();
        spring += s;
        spring *= spring_k * re;
        if (length(dt * spring) > 0.3f * h) ip += h * 0.3f * spring / length(spring);
        else ip += dt * spring;
        ip.x = fmaxf(tmin.x, fminf(tmax.x, ip.x));
        ip.y = fmaxf(tmin.y, fminf(tmax.y, ip.y));
        ip.z = fmaxf(tmin.z, fminf(tmax.z, ip.z));
        out[p] = with_xyz(q, ip);
    }
}

__global__ void k_correct_bubble(Grid g, int np, float4* __restrict__ pos, const float* __restrict__ lsm,
                                 const float* __restrict__ gx, const float* __restrict__ gy, const float* __restrict__ gz,
                                 const float* __restrict__ lsa, const float* __restrict__ gxa, const float* __restrict__ gya,
                                 const float* __restrict__ gza, int airver) {
    const float h = g.h, rs = 0.5f * h;
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f == MP_TYPEAIRSOLO || f == MP_TYPESOLID) continue;
        float3 ip = xyz(q);
        float s = (f == MP_TYPEFLUID) ? -1.0f : 1.0f;
        float3 dir = vecFromGrid(g, ip, gx, gy, gz);
        float dl = length(dir);
        if (dl == 0) continue;
        dir = normalize(dir);
        float d = scaleFromGrid(g, ip, lsm) / dl;
        if (!airver) {
            if (s * d < 0 && fabsf(d) < 0.5f * h) {
                if (f == MP_TYPEAIR && fabsf(d) > 0.3f * h) ip = ip - d * dir;
                else if (f == MP_TYPEFLUID) {
                    ip = ip - d * dir;
                    dir = vecFromGrid(g, ip, gx, gy, gz);
                    dl = length(dir);
                    if (dl == 0) continue;
                    dir = normalize(dir);
                    d = scaleFromGrid(g, ip, lsm) / dl;
                    ip = ip + s * (rs - s * d) * dir;
                }
            } else if (f == MP_TYPEFLUID && s * d < rs * 0.5f && s * d >= 0) {
                ip = ip + s * (rs - s * d) * dir;
            }
        } else {
            if (s * d < 0 && fabsf(d) < 0.5f * h) {
                if (f == MP_TYPEAIR && fabsf(d) > 0.3f * h) ip = ip - d * dir;
            }
            if (f == MP_TYPEFLUID) {
                dir = vecFromGrid(g, ip, gxa, gya, gza);
                dl = length(dir);
                if (dl == 0) continue;
                dir = normalize(dir);
                d = scaleFromGrid(g, ip, lsa) / dl;
                if (d < -1.3f * rs) ip = ip - (d - rs) * dir;
            }
        }
        pos[p] = with_xyz(q, ip);
    }
}

// ---- solid motion --------------------------------------------------------------
__global__ void k_vel_zero_solid(int np, const float4* __restrict__ pos, float4* __restrict__ vel) {
    MP_GRID_LOOP(p, np) if (pflag(pos[p]) == MP_TYPESOLID) { float4 v = vel[p]; vel[p] = make_float4(0.f, 0.f, 0.f, v.w); }
}
__global__ void k_solid_bound(Grid g, int np, const float4* __restrict__ pos, float4* __restrict__ vel, float sb, int ns,
                              float samplespace) {
    const float h = g.h;
    const float3 g0 = mk3(g.gx0, g.gy0, g.gz0);
    const float3 g1 = g0 + mk3((float)g.NX, (float)g.NY, (float)g.NZ) * h;
    const float3 tmin = g0 + (mk3(h, h, h) + mk3(0.3f * samplespace));
    const float3 tmax = g1 - (mk3(h, h, h) + mk3(0.3f * samplespace));
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        if (pflag(q) != MP_TYPESOLID) continue;
        float4 v = vel[p];
        float3 iv = xyz(v);
        if (q.x < tmin.x) iv.x += (tmin.x - q.x) * sb * ns;
        if (q.x > tmax.x) iv.x -= (q.x - tmax.x) * sb * ns;
        if (q.y < tmin.y) iv.y += (tmin.y - q.y) * sb * ns;
        if (q.y > tmax.y) iv.y -= (q.y - tmax.y) * sb * ns;
        if (q.z < tmin.z) iv.z += (tmin.z - q.z) * sb * ns;
        if (q.z > tmax.z) iv.z -= (q.z - tmax.z) * sb * ns;
        vel[p] = with_xyz(v, iv);
    }
}
// FP64 block sums of solid (pos, vel) or (c, I) -> 6 doubles per block
__global__ void k_solid_sums(int np, const float4* __restrict__ pos, const float4* __restrict__ vel, float3 rg0, int mode,
                             double* __restrict__ part) {
    __shared__ double sm[6][8];
    double a[6] = {0, 0, 0, 0, 0, 0};
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        if (pflag(q) != MP_TYPESOLID) continue;
        float3 ip = xyz(q), iv = xyz(vel[p]);
        if (mode == 0) { a[0] += ip.x; a[1] += ip.y; a[2] += ip.z; a[3] += iv.x; a[4] += iv.y; a[5] += iv.z; }
        else {
            float dis = length(ip - rg0);
            if (dis > 1e-6) {
                float3 c = cross(ip - rg0, iv);
                a[0] += c.x; a[1] += c.y; a[2] += c.z; a[3] += dis;
            }
        }
    }
    for (int q = 0; q < 6; q++) {
        double v = a[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sm[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sm[threadIdx.x][w];
        part[blockIdx.x * 6 + threadIdx.x] = s;
    }
}
struct Mat3 { float m[9]; };
__global__ void k_solid_move(int np, float4* __restrict__ pos, float4* __restrict__ vel, float3 rg0, float3 rg, float3 R,
                             float3 T, Mat3 rm) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        if (pflag(q) != MP_TYPESOLID) continue;
        float3 ip = xyz(q);
        float4 v = vel[p];
        float3 vh = cross(R, ip - rg0);
        vh += T;
        vh = 0.5f * (xyz(v) + vh);
        vel[p] = with_xyz(v, vh);
        float3 t = ip - rg0;
        const float* m = rm.m;
        float3 r2 = mk3(t.x * m[0] + t.y * m[3] + t.z * m[6], t.x * m[1] + t.y * m[4] + t.z * m[7],
                        t.x * m[2] + t.y * m[5] + t.z * m[8]);
        pos[p] = with_xyz(q, r2 + rg);
    }
}

// computeSolidVertex_k (spray_k.cu:5254-5263): the stored solid surface moves
// with the rigid motion of the solid particles (transposeParticle as above)
__global__ void k_solid_vertex(int nv, float3* __restrict__ vtx, float3 rg0, float3 rg, Mat3 rm) {
    MP_GRID_LOOP(v, nv) {
        float3 t = vtx[v] - rg0;
        const float* m = rm.m;
        float3 r2 = mk3(t.x * m[0] + t.y * m[3] + t.z * m[6], t.x * m[1] + t.y * m[4] + t.z * m[7],
                        t.x * m[2] + t.y * m[5] + t.z * m[8]);
        vtx[v] = r2 + rg;
    }
}

// pouringwater (spray_k.cu:5575-5596): emitter point idx appends particle
// np + idx with jitter from the random table. The callers pass frame 0, so
// the table offset is idx % (nrand - 6). The reference leaves the slot's
// solubility as it was; here it is 0 (updatesolubility sets it before use).
__global__ void k_pour_particles(int n, int np, const float* __restrict__ ppos, const float* __restrict__ pvel,
                                 const float* __restrict__ rf, int nrand, float4* __restrict__ pos,
                                 float4* __restrict__ vel, float4* __restrict__ heat, int flag, float posrand,
                                 float velrand, float samplespace, float m0, float T, float L) {
    MP_GRID_LOOP(idx, n) {
        int rb = (0 + idx) % (nrand - 6);
        float3 rv = mk3(rf[rb] * 2.0f - 1.0f, rf[rb + 1] * 2.0f - 1.0f, rf[rb + 2] * 2.0f - 1.0f);
        rb += 3;
        float3 rp = mk3(rf[rb] * 2.0f - 1.0f, rf[rb + 1] * 2.0f - 1.0f, rf[rb + 2] * 2.0f - 1.0f);
        float3 p = mk3(ppos[3 * idx], ppos[3 * idx + 1], ppos[3 * idx + 2]) + rp * posrand * samplespace;
        float3 v = mk3(pvel[3 * idx], pvel[3 * idx + 1], pvel[3 * idx + 2]) + rv * velrand;
        pos[np + idx] = make_float4(p.x, p.y, p.z, flagbits(flag));
        vel[np + idx] = make_float4(v.x, v.y, v.z, m0);
        heat[np + idx] = make_float4(T, L, 0.0f, 0.0f);
    }
}

// advectparticle_RK2 (spray_k.cu:409-458) with velmode FLIP: the particle
// velocity blends the grid velocity with FLIP_ALPHA = 0.95 (utility.h:9), the
// position takes a midpoint step through the grid velocity, and both are
// clamped one cell and half a sample spacing inside the walls. SOLID
// particles keep their position.
__global__ void k_advect_rk2(Grid g, int np, float4* __restrict__ pos, float4* __restrict__ vel,
                             const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
                             float dt, float samplespace) {
    const float h = g.h;
    const float3 g0 = mk3(g.gx0, g.gy0, g.gz0);
    const float3 g1 = g0 + mk3((float)g.NX, (float)g.NY, (float)g.NZ) * h;
    const float flip = 0.95f;
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p], v4 = vel[p];
        float3 ip = xyz(q), iv = xyz(v4);
        float3 tmin = g0 + (mk3(h, h, h) + mk3(0.5f * samplespace));
        float3 tmax = g1 - (mk3(h, h, h) + mk3(0.5f * samplespace));
        float3 gv = velFromGrid(g, ip, ux, uy, uz);
        iv = (1 - flip) * gv + flip * iv;
        float3 mid = ip + gv * dt * 0.5f;
        float3 gvm = velFromGrid(g, mid, ux, uy, uz);
        ip += gvm * dt;
        if (ip.x <= tmin.x) { ip.x = tmin.x; iv.x = 0.0f; }
        if (ip.y <= tmin.y) { ip.y = tmin.y; iv.y = 0.0f; }
        if (ip.z <= tmin.z) { ip.z = tmin.z; iv.z = 0.0f; }
        if (ip.x >= tmax.x) { ip.x = tmax.x; iv.x = 0.0f; }
        if (ip.y >= tmax.y) { ip.y = tmax.y; iv.y = 0.0f; }
        if (ip.z >= tmax.z) { ip.z = tmax.z; iv.z = 0.0f; }
        if (pflag(q) != MP_TYPESOLID) {
            vel[p] = with_xyz(v4, iv);
            pos[p] = with_xyz(q, ip);
        } else vel[p] = with_xyz(v4, iv);
    }
}

// ---- heat / phase change -----------------------------------------------------
__global__ void k_latent(int np, const float4* __restrict__ pos, float4* __restrict__ heat, float mp, float bp, float lth) {
    MP_GRID_LOOP(p, np) {
        int f = pflag(pos[p]);
        float4 hh = heat[p];
        float T = hh.x, L = hh.y;
        if (f == MP_TYPESOLID && T > mp) { L += T - mp; T = mp; }
        if (f == MP_TYPEFLUID) {
            if (T < mp) { L -= mp - T; T = mp; }
            else if (T > bp) { L += T - bp; T = bp; }
            else L = lth;
        }
        heat[p] = make_float4(T, L, hh.z, hh.w);
    }
}
__global__ void k_init_heat(int np, const float4* __restrict__ pos, float4* __restrict__ heat, float sT, float lT,
                            float lth, float dgr, float igr, float airm0, float coef, float T0,
                            unsigned int* __restrict__ nsolid) {
    MP_GRID_LOOP(p, np) {
        int f = pflag(pos[p]);
        float T, L, so, ga;
        if (f == MP_TYPESOLID) { T = sT; L = 0; atomicAdd(nsolid, 1u); }
        else { T = lT; L = lth; }
        if (f == MP_TYPEFLUID || f == MP_TYPESOLID) {
            so = dgr * airm0 * expf(coef * (1.0f / T - 1.0f / T0));
            ga = igr * so;
        } else { so = 0; ga = 0; }
        heat[p] = make_float4(T, L, so, ga);
    }
}
__global__ void k_solubility(int np, const float4* __restrict__ pos, float4* __restrict__ heat, float dgr, float airm0,
                             float coef, float T0) {
    MP_GRID_LOOP(p, np) {
        if (pflag(pos[p]) != MP_TYPEFLUID) continue;
        float4 hh = heat[p];
        hh.z = dgr * airm0 * expf(coef * (1.0f / hh.x - 1.0f / T0));
        heat[p] = hh;
    }
}
struct GasParams {
    float m0a, lth, vgr, h;
    int frame, nrand, nseed;
};
// GenerateGasParticle_k, pass 1: decide per cell, clamp the donors
__global__ void k_gas_decide(Grid g, Cells cl, const float4* __restrict__ pos, const float4* __restrict__ vel,
                             float4* __restrict__ heat, const int32_t* __restrict__ seeds, GasParams gp,
                             uint32_t* __restrict__ add) {
    MP_GRID_LOOP(idx, g.n) {
        add[idx] = 0;
        int i, j, k; getijk(g, (int)idx, i, j, k);
        if (k <= 1 || in_boundary_cell(g, i, j)) continue;
        uint32_t s0 = cl.off[idx], s1 = cl.off[idx + 1];
        if (s0 == s1) continue;
        float gc = 0, gs = 0, vsum = 0;
        int gcnt = 0;
        for (uint32_t p = s0; p < s1; p++) {
            int f = pflag(pos[p]);
            if (f == MP_TYPEFLUID) {
                float4 hh = heat[p];
                gc += hh.w; gs += hh.z;
                vsum += fmaxf(0.0f, hh.y - gp.lth) * gp.vgr * gp.m0a;
            } else if (f == MP_TYPEAIRSOLO || f == MP_TYPEAIR) gcnt++;
        }
        bool hasseed = false;
        for (int s = 0; s < gp.nseed; s++) if (seeds[s] == (int)idx) hasseed = true;
        if (gc - gs + vsum > gp.m0a && (hasseed || gcnt > 0)) {
            add[idx] = 1;
            for (uint32_t p = s0; p < s1; p++) {
                if (pflag(pos[p]) != MP_TYPEFLUID) continue;
                float4 hh = heat[p];
                hh.w = fminf(hh.w, hh.z);
                hh.y = fminf(hh.y, gp.lth);
                heat[p] = hh;
            }
        }
    }
}
// pass 2: write the new solo-air particle of each deciding cell at np + rank
__global__ void k_gas_append(Grid g, Cells cl, float4* __restrict__ pos, float4* __restrict__ vel, float4* __restrict__ heat,
                             const float* __restrict__ randf, const float* __restrict__ Tp, GasParams gp,
                             const uint32_t* __restrict__ add, const uint32_t* __restrict__ rank, int np, int cap) {
    MP_GRID_LOOP(idx, g.n) {
        if (!add[idx]) continue;
        int slot = np + (int)rank[idx];
        if (slot >= cap) continue;
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float3 gaspos = mk3(0.0f);
        int gcnt = 0;
        for (uint32_t p = cl.off[idx]; p < cl.off[idx + 1]; p++) {
            float4 q = pos[p];
            int f = pflag(q);
            if (f == MP_TYPEAIRSOLO || f == MP_TYPEAIR) { gaspos += xyz(q); gcnt++; }
        }
        int rc = gp.nrand;
        int base = (int)(((long long)idx * (long long)gp.frame) % (long long)(rc - 200));
        float3 rp = mk3(randf[(base + 0) % rc], randf[(base + 1) % rc], randf[(base + 2) % rc]);
        float rn = randf[(base + 3) % rc];
        float r = gp.h * 0.25f;
        float3 np3;
        if (gcnt > 0) np3 = gaspos / (float)gcnt + (fmaxf(0.5f, rn) * r) * (rp - mk3(0.5f)) * 2;
        else np3 = mk3((float)i, (float)j, (float)k) * gp.h + gp.h * rp;
        pos[slot] = make_float4(np3.x, np3.y, np3.z, flagbits(MP_TYPEAIRSOLO));
        vel[slot] = make_float4(0.f, 0.f, 0.f, gp.m0a);
        heat[slot] = make_float4(Tp[idx], 0.f, 0.f, 0.f);
    }
}

// sweepVacuum, one Jacobi pass
__global__ void k_sweep_vacuum(Grid g, const int8_t* __restrict__ in, int8_t* __restrict__ out) {
    MP_GRID_LOOP(idx, g.n) {
        int8_t m = in[idx];
        if (m == MP_TYPEAIR && interior(g, (int)idx)) {
            int i, j, k; getijk(g, (int)idx, i, j, k);
            for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2)
                if (in[cid(g, i + di, j + dj, k + dk)] == MP_TYPEVACUUM) m = MP_TYPEVACUUM;
        }
        out[idx] = m;
    }
}
__global__ void k_mark_delete(Grid g, int np, const float4* __restrict__ pos, const float4* __restrict__ vel,
                              const int8_t* __restrict__ mark, const float* __restrict__ lsa, uint32_t* __restrict__ keep) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        int f = pflag(q);
        if (f == MP_TYPESOLID) { keep[p] = 1; continue; }
        float3 ip = xyz(q);
        if (f == MP_TYPEFLUID) {
            float l = scaleFromGrid(g, ip, lsa);
            keep[p] = (l < -g.h) ? 0u : 1u;
            continue;
        }
        int i, j, k; ijkpos(g, ip, i, j, k);
        int c = 0;
        for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++)
            if (vc(g, i + di, j + dj, k + dk) && mark[cid(g, i + di, j + dj, k + dk)] == MP_TYPEVACUUM) c++;
        keep[p] = (c == 0 && vel[p].w > 0.000001f) ? 1u : 0u;
    }
}
__global__ void k_compact(int np, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ scan,
                          const float4* __restrict__ p0, const float4* __restrict__ v0, const float4* __restrict__ h0,
                          float4* __restrict__ p1, float4* __restrict__ v1, float4* __restrict__ h1) {
    MP_GRID_LOOP(p, np) {
        if (!keep[p]) continue;
        uint32_t o = scan[p];
        p1[o] = p0[p]; v1[o] = v0[p]; h1[o] = h0[p];
    }
}
__global__ void k_melt(int np, float4* __restrict__ pos, float4* __restrict__ heat, float lth, unsigned int* __restrict__ cnt) {
    MP_GRID_LOOP(p, np) {
        float4 q = pos[p];
        if (pflag(q) != MP_TYPESOLID) continue;
        float4 hh = heat[p];
        if (hh.y > lth) {
            pos[p] = make_float4(q.x, q.y, q.z, flagbits(MP_TYPEFLUID));
            hh.y = lth;
            heat[p] = hh;
            atomicAdd(cnt, 1u);
        }
    }
}
__global__ void k_freeze(Grid g, Cells cl, int np, const float4* __restrict__ opos, float4* __restrict__ pos,
                         float4* __restrict__ heat, float samplespace, unsigned int* __restrict__ cnt) {
    const float h = g.h;
    MP_GRID_LOOP(p, np) {
        float4 q = opos[p];
        if (pflag(q) != MP_TYPEFLUID) continue;
        float4 hh = heat[p];
        if (!(hh.y < 0)) continue;
        float3 ip = xyz(q);
        int i, j, k; ijkpos(g, ip, i, j, k);
        float mind = 1000; int mi = -1, cs = 0;
        for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
            if (!vc(g, i + di, j + dj, k + dk)) continue;
            int c = cid(g, i + di, j + dj, k + dk);
            if (!(cl.tmask[c] & (1u << MP_TYPESOLID))) continue;
            for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                float4 o = opos[s];
                if (pflag(o) != MP_TYPESOLID) continue;
                float d = length(xyz(o) - ip);
                if (d < h) cs++;
                if (d < mind) { mind = d; mi = (int)s; }
            }
        }
        if (mi != -1 && mind < h && cs > 2) {
            float3 np3 = ip;
            if (mind > samplespace) {
                float3 o = xyz(opos[mi]);
                np3 = normalize(ip - o) * samplespace + o;
            }
            pos[p] = make_float4(np3.x, np3.y, np3.z, flagbits(MP_TYPESOLID));
            hh.y = 0;
            heat[p] = hh;
            atomicAdd(cnt, 1u);
        }
    }
}

}  // namespace

static Cells cells_of(MpCtx* c) { return Cells{c->cell_off, c->tmask}; }
#define PB(np) mp_blocks((np), 256), 256, 0, c->stream

int k_external_force(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    const mp_params& P = c->P;
    k_forces<<<PB(np)>>>(np, c->pos, c->vel, P.dt, P.gravity_x, P.gravity_y, P.gravity_z, P.bubble_max_vel,
                         P.buoyance_rate_air, P.buoyance_rate_solo);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_mark_solo_air(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    float tol1 = -1.45f, tol2 = -0.5f;
    int sc = c->P.scene;
    if (sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL) { tol1 = 0.05f; tol2 = -0.8f; }
    else if (sc == MP_SCENE_INTERACTION) { tol1 = 0.2f; tol2 = -0.5f; }
    k_solo_air<<<PB(np)>>>(c->G, cells_of(c), np, c->pos, c->vel, c->lsmerge, c->au[0], c->au[1], c->au[2], tol1, tol2);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_surface_tension(MpCtx* c) {
    MP_TRY(k_surface_tension_grid(c));
    int np = c->np();
    if (!np) return MP_OK;
    k_st_particles<<<PB(np)>>>(c->G, np, c->pos, c->vel, c->lsmerge, c->sf, c->gx, c->gy, c->gz, c->mark, c->P.scene,
                               c->P.dt);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_solo_air_update(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    const mp_params& P = c->P;
    k_air_dens<<<PB(np)>>>(c->G, cells_of(c), np, c->pos, c->vel, c->pdens, c->pprs, c->pscr, P.airm0 * P.poly6kern,
                           P.waterrho);
    // `dens *= dparam.airm0 * dparam.poly6kern` multiplies by the product (spray_k.cu:4305)
    k_air_force<<<PB(np)>>>(c->G, cells_of(c), np, c->pos, c->vel, c->pscr, c->pdens, c->pprs, P.spikykern,
                            P.lapkern * P.viscosity_sph, P.airm0, P.dt);
    c->launches += 2;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// CollisionSolid (spray.cu:2959-2983)
// skip_empty_solid: leave the solid velocity faces as they are when no cell
// holds a SOLID particle. The collision reads them only where the solid level
// set is at most half a cell, and without solid cells it is 3 NX everywhere.
int k_collide_advect(MpCtx* c, bool skip_empty_solid) {
    MP_TRY(k_solid_phi(c));   // raises u32_scratch[2] when a cell holds a SOLID particle
    bool need_su = true;
    if (skip_empty_solid) {
        uint32_t any = 1;
        MP_CUDA(c, cudaMemcpyAsync(&any, c->u32_scratch + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
        MP_CUDA(c, cudaStreamSynchronize(c->stream));
        need_su = any != 0;
    }
    if (need_su) MP_TRY(k_p2g_faces(c, c->su, 0));
    int np = c->np();
    if (!np) return MP_OK;
    const mp_params& P = c->P;
    if (P.scene == MP_SCENE_FREEZING || P.scene == MP_SCENE_MELTINGPOUR) {
        MP_CUDA(c, cudaMemcpyAsync(c->pos2, c->pos, sizeof(float4) * np, cudaMemcpyDeviceToDevice, c->stream));
        k_collide_freezing<<<PB(np)>>>(c->G, cells_of(c), np, c->pos2, c->pos, c->vel, c->phisolid, P.samplespace, P.dt);
    } else {
        k_collide<<<PB(np)>>>(c->G, np, c->pos, c->vel, c->phisolid, c->su[0], c->su[1], c->su[2], P.scene,
                              P.bounce_vel_param, P.bounce_pos_param, P.dt);
    }
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_correct_pos(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    const mp_params& P = c->P;
    KtScope kt(c, MP_KT_CORRECT);
    k_correct_pos<<<PB(np)>>>(c->G, cells_of(c), np, c->pos, c->vel, c->pos2, P.correction_radius * c->G.h,
                              P.correction_spring, P.samplespace, P.dt);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    std::swap(c->pos, c->pos2);
    return MP_OK;
}

int k_correct_pos_bubble(MpCtx* c) {
    int sc = c->P.scene;
    int airver = (sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_INTERACTION ||
                  sc == MP_SCENE_ALL) ? 1 : 0;
    if (airver) MP_TRY(k_phigra(c, c->gxa, c->gya, c->gza, c->lsair));
    int np = c->np();
    if (!np) return MP_OK;
    k_correct_bubble<<<PB(np)>>>(c->G, np, c->pos, c->lsmerge, c->gx, c->gy, c->gz, c->lsair, c->gxa, c->gya, c->gza,
                                 airver);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

static int solid_sums(MpCtx* c, int mode, float3 rg0, double out[6]) {
    int np = c->np();
    int nb = mp_blocks(np, 256);
    k_solid_sums<<<nb, 256, 0, c->stream>>>(np, c->pos, c->vel, rg0, mode, c->red);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    std::vector<double> h((size_t)nb * 6);
    MP_CUDA(c, cudaMemcpyAsync(h.data(), c->red, sizeof(double) * 6 * nb, cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 6; q++) out[q] = 0;
    for (int b = 0; b < nb; b++) for (int q = 0; q < 6; q++) out[q] += h[(size_t)b * 6 + q];
    return MP_OK;
}

// solidmotion_fixed / solidmotion (spray.cu:2685-2775)
int k_solid_motion(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    const mp_params& P = c->P;
    if (P.b_fix_solid) {
        k_vel_zero_solid<<<PB(np)>>>(np, c->pos, c->vel);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        return MP_OK;
    }
    int ns = c->S.n_real_solpoint;
    if (ns <= 0) return MP_OK;
    k_solid_bound<<<PB(np)>>>(c->G, np, c->pos, c->vel, P.solid_bounce_param, ns, P.samplespace);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    double s[6];
    MP_TRY(solid_sums(c, 0, make_float3(0, 0, 0), s));
    float fs = (float)ns;
    float3 T = make_float3((float)s[3] / fs, (float)s[4] / fs, (float)s[5] / fs);
    if (P.scene == MP_SCENE_INTERACTION) T.y = 0.0f;
    float3 rg0 = make_float3((float)s[0] / fs, (float)s[1] / fs, (float)s[2] / fs);
    float3 rg = make_float3(rg0.x + P.dt * T.x, rg0.y + P.dt * T.y, rg0.z + P.dt * T.z);
    MP_TRY(solid_sums(c, 1, rg0, s));
    float tIx = (float)s[3];
    float3 R = make_float3((float)s[0], (float)s[1], (float)s[2]);
    if (tIx <= 0) tIx = 1;
    tIx /= fs;
    R = make_float3(R.x / tIx / tIx, R.y / tIx / tIx, R.z / tIx / tIx);
    R = make_float3(R.x / fs, R.y / fs, R.z / fs);
    float3 axis = R;
    float theta = -sqrtf(R.x * R.x + R.y * R.y + R.z * R.z) * P.dt;
    if (fabsf(theta) > 1e-6) {
        float inv = 1.0f / sqrtf(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
        axis = make_float3(axis.x * inv, axis.y * inv, axis.z * inv);
    } else { axis = make_float3(1, 0, 0); theta = 0; }
    float x = axis.x, y = axis.y, z = axis.z;
    float cc = cosf(theta), sn = sinf(theta);
    Mat3 rm;
    rm.m[0] = cc + (1 - cc) * x * x;     rm.m[1] = (1 - cc) * x * y - sn * z; rm.m[2] = (1 - cc) * x * z + sn * y;
    rm.m[3] = (1 - cc) * y * x + sn * z; rm.m[4] = cc + (1 - cc) * y * y;     rm.m[5] = (1 - cc) * y * z - sn * x;
    rm.m[6] = (1 - cc) * z * x - sn * y; rm.m[7] = (1 - cc) * z * y + sn * x; rm.m[8] = cc + (1 - cc) * z * z;
    k_solid_move<<<PB(np)>>>(np, c->pos, c->vel, rg0, rg, R, T, rm);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    // the solid surface extracted once (bRunMCSolid off) follows the same motion
    const int sc = P.scene;
    const McSurface& sm = c->mc[MP_MC_SOLID];
    if ((sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES || sc == MP_SCENE_MELTANDBOIL ||
         sc == MP_SCENE_MELTANDBOIL_HIGHRES) && c->S.frame > 0 && !P.b_run_mc_solid && P.b_run_mc && sm.nverts > 0) {
        k_solid_vertex<<<mp_blocks(sm.nverts, 256), 256, 0, c->stream>>>(sm.nverts, sm.verts, rg0, rg, rm);
        c->launches++;
        MP_CHECK_LAUNCH(c);
    }
    return MP_OK;
}

// wateradvect (spray.cu:293-305)
int k_water_advect(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    k_advect_rk2<<<PB(np)>>>(c->G, np, c->pos, c->vel, c->wu[0], c->wu[1], c->wu[2], c->P.dt, c->P.samplespace);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    c->mc_sorted = 0;
    return MP_OK;
}

// pouring / pouringgas (spray.cu:3012-3043): water every 4th frame; in the
// interaction scenes from begin_frame on, AIRSOLO gas every 6th frame; only
// when the emitter's points fit under par_num_max
int k_pour(MpCtx* c) {
    const mp_params& P = c->P;
    const int sc = P.scene, frame = c->S.frame;
    const bool gas = (sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES) && frame >= P.begin_frame;
    const int every = gas ? 6 : 4;
    const int n = c->pour_n, np = c->np();
    if (frame % every != 0 || n == 0 || (long long)n + np > P.par_num_max) return MP_OK;
    if (c->nrand <= 6) { c->err = "pour: random table not set"; return MP_ERR_STATE; }
    k_pour_particles<<<mp_blocks(n, 256), 256, 0, c->stream>>>(
        n, np, c->pour_pos, c->pour_vel, c->randf, c->nrand, c->pos, c->vel, c->heat,
        gas ? MP_TYPEAIRSOLO : MP_TYPEFLUID, P.pos_rand_param, P.vel_rand_param, P.samplespace, P.m0,
        P.default_liquid_T, P.liquid_heat_th);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    c->S.par_num_now = np + n;
    c->mc_sorted = 0;
    return MP_OK;
}

int k_latent_heat(MpCtx* c) {
    int np = c->np();
    if (!np) return MP_OK;
    k_latent<<<PB(np)>>>(np, c->pos, c->heat, c->P.melting_point, c->P.boiling_point, c->P.liquid_heat_th);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_init_particle_heat(MpCtx* c) {
    int np = c->np();
    const mp_params& P = c->P;
    MP_CUDA(c, cudaMemsetAsync(c->u32_scratch, 0, sizeof(uint32_t), c->stream));
    if (np) {
        k_init_heat<<<PB(np)>>>(np, c->pos, c->heat, P.default_solid_T, P.default_liquid_T, P.liquid_heat_th,
                                P.init_dissolve_gas_rate, P.init_gas_rate, P.airm0, P.solubility_coef, P.temperature0,
                                c->u32_scratch);
        c->launches++;
        MP_CHECK_LAUNCH(c);
    }
    uint32_t ns = 0;
    MP_CUDA(c, cudaMemcpyAsync(&ns, c->u32_scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->S.n_real_solpoint = (int)ns;
    return MP_OK;
}

// GenerateGasParticle (spray.cu:2653-2683)
int k_gen_gas(MpCtx* c) {
    int np = c->np();
    const mp_params& P = c->P;
    if (c->nrand <= 200) { c->err = "gen_gas: random table not set"; return MP_ERR_STATE; }
    if (np) {
        k_solubility<<<PB(np)>>>(np, c->pos, c->heat, P.init_dissolve_gas_rate, P.airm0, P.solubility_coef, P.temperature0);
        c->launches++;
    }
    GasParams gp{P.airm0, P.liquid_heat_th, P.vapor_gen_rate, c->G.h, c->S.frame, c->nrand, c->nseed};
    uint32_t* add = c->cell_cnt;          // zero between sorts; restored below
    uint32_t* rank = c->keys;             // n+1 entries (keys hold par_num_max >= n+1? checked at create)
    int n = c->G.n;
    k_gas_decide<<<mp_blocks(n, 256), 256, 0, c->stream>>>(c->G, cells_of(c), c->pos, c->vel, c->heat, c->seeds, gp, add);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_TRY(mp_scan_u32(c, add, rank, (size_t)n));
    uint32_t total = 0;
    MP_CUDA(c, cudaMemcpyAsync(&total, rank + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    k_gas_append<<<mp_blocks(n, 256), 256, 0, c->stream>>>(c->G, cells_of(c), c->pos, c->vel, c->heat, c->randf, c->Tp,
                                                          gp, add, rank, np, P.par_num_max);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_CUDA(c, cudaMemsetAsync(add, 0, sizeof(uint32_t) * n, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    if ((long long)np + total > P.par_num_max) {
        c->S.par_num_now = P.par_num_max;
        c->err = "gen_gas: par_num_max exceeded";
        return MP_ERR_CAPACITY;
    }
    c->S.par_num_now = np + (int)total;
    return MP_OK;
}

// deleteAirFluidParticle (spray.cu:2194-2248)
int k_delete(MpCtx* c) {
    const mp_params& P = c->P;
    int passes = 20;
    if (P.scene == MP_SCENE_INTERACTION) passes = (c->S.frame % 2 == 0) ? 1 : 0;
    for (int t = 0; t < passes; t++) {
        k_sweep_vacuum<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, c->mark, c->mark_tmp);
        c->launches++;
        std::swap(c->mark, c->mark_tmp);
    }
    MP_CHECK_LAUNCH(c);
    int np = c->np();
    if (!np) return MP_OK;
    uint32_t* keep = c->keys;
    uint32_t* scan = c->perm;
    k_mark_delete<<<PB(np)>>>(c->G, np, c->pos, c->vel, c->mark, c->lsair, keep);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_TRY(mp_scan_u32(c, keep, scan, (size_t)np));
    uint32_t total = 0;
    MP_CUDA(c, cudaMemcpyAsync(&total, scan + np, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    k_compact<<<PB(np)>>>(np, keep, scan, c->pos, c->vel, c->heat, c->pos2, c->vel2, c->heat2);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    std::swap(c->pos, c->pos2); std::swap(c->vel, c->vel2); std::swap(c->heat, c->heat2);
    c->S.par_num_now = (int)total;
    return MP_OK;
}

int k_melt(MpCtx* c) {
    int np = c->np();
    MP_CUDA(c, cudaMemsetAsync(c->u32_scratch, 0, sizeof(uint32_t), c->stream));
    if (np) {
        k_melt<<<PB(np)>>>(np, c->pos, c->heat, c->P.liquid_heat_th, c->u32_scratch);
        c->launches++;
        MP_CHECK_LAUNCH(c);
    }
    uint32_t cnt = 0;
    MP_CUDA(c, cudaMemcpyAsync(&cnt, c->u32_scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->S.n_real_solpoint -= (int)cnt;
    return MP_OK;
}

int k_freeze(MpCtx* c) {
    int np = c->np();
    MP_CUDA(c, cudaMemsetAsync(c->u32_scratch, 0, sizeof(uint32_t), c->stream));
    if (np) {
        MP_CUDA(c, cudaMemcpyAsync(c->pos2, c->pos, sizeof(float4) * np, cudaMemcpyDeviceToDevice, c->stream));
        k_freeze<<<PB(np)>>>(c->G, cells_of(c), np, c->pos2, c->pos, c->heat, c->P.samplespace, c->u32_scratch);
        c->launches++;
        MP_CHECK_LAUNCH(c);
    }
    uint32_t cnt = 0;
    MP_CUDA(c, cudaMemcpyAsync(&cnt, c->u32_scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->S.n_real_solpoint += (int)cnt;
    return MP_OK;
}
