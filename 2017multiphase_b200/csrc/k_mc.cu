// k_mc.cu — marching-cubes surface extraction on the 2x grid.
//
// Reference: runMC_smooth (Multiphase/Multiphase/spray.cu:804-979) with the
// density kernels genWaterDensfield_GY / _liquidAndGas / _Gas
// (spray_k.cu:1528-1772), classifyVoxel (1853), compactVoxels (1891),
// markActiveEdge_MC (2172), generateTriangles_indices (2074), the Taubin
// smoothing kernels (2408-2440) and calnormal_k / normalizeTriangleNor_k
// (2223-2260). Differences that make the output deterministic:
//   * each shared vertex is interpolated once, from its edge's lower node
//     (the reference lets every voxel touching the edge write it);
//   * smoothing displacements and normals are per-vertex gathers over the
//     incident triangles in ascending triangle order (the reference uses
//     float atomics);
//   * output buffers are device memory owned by the context (the reference
//     wrote into OpenGL vertex buffers).
// The reference's smoothMesh applies lambda = 0.5 and then mu = -0.53 with the
// weights already cleared, so only the lambda half-step has an effect; that is
// what is computed here.
#include "ctx.cuh"

using namespace mpk;

namespace {

struct McGrid {
    int NXMC, NYMC, NZMC;   // voxels
    int W, H, D;            // nodes
    float hm;               // node spacing
};

// One thread computes NJ x NK nodes, (i, j0 + nj, k0 + nk). Neighbouring
// nodes share most of their 4 x 4 x 4 cell windows, so the thread walks the
// union window once, (a, b, c) ascending, and each node takes only the cells
// of its own window: every node sees its cells, and the particles in them, in
// the reference's (di, dj, dk, particle) order, and keeps its own per-cell
// partial sum (res) and running sums, so each field value is bit-identical to
// the one-node-per-thread gather. A cell's header (type mask, range) and its
// particles are loaded once for all the nodes that need them.
// GAS2 (with SURF == MP_MC_FLUID): the gas field is accumulated in the same
// pass into dens2. Both surfaces use the same radius and weight, the gas
// particles are a subset of the fluid ones, and each sum keeps its own
// accumulators in the same visiting order, so both fields equal the separate
// passes bit for bit.
template <int SURF, bool GAS2, int NJ, int NK, int MINB>
__global__ void __launch_bounds__(256, MINB) k_mc_density(McGrid m, Tiles T, Cells cl, const float4* __restrict__ pos,
                                                          float* __restrict__ dens, int scene, float* __restrict__ dens2) {
    const float hm = m.hm;
    const uint32_t need = SURF == MP_MC_SOLID ? (1u << MP_TYPESOLID)
                        : SURF == MP_MC_FLUID ? ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO) | (1u << MP_TYPEFLUID))
                                              : ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO));
    const float R = SURF == MP_MC_SOLID ? hm : hm * 2;
    const float cut = SURF == MP_MC_SOLID ? hm * hm * 1.001f : R * R * 1.001f;
    MP_GRID_LOOP(t, T.threads()) {
        int i, jt, kt; if (!tile_ijk(T, t, i, jt, kt)) continue;
        const int j0 = jt * NJ, k0 = kt * NK;
        const float px = (float)i * hm;
        float py[NJ], pz[NK];
        #pragma unroll
        for (int n = 0; n < NJ; n++) py[n] = (float)(j0 + n) * hm;
        #pragma unroll
        for (int n = 0; n < NK; n++) pz[n] = (float)(k0 + n) * hm;
        float cx[NJ][NK], cy[NJ][NK], cz[NJ][NK], ws[NJ][NK];
        float gx[NJ][NK], gy[NJ][NK], gz[NJ][NK], gw[NJ][NK];
        #pragma unroll
        for (int u = 0; u < NJ; u++)
            #pragma unroll
            for (int v = 0; v < NK; v++) {
                cx[u][v] = cy[u][v] = cz[u][v] = ws[u][v] = 0.0f;
                gx[u][v] = gy[u][v] = gz[u][v] = gw[u][v] = 0.0f;
            }
        // the cell loops stay rolled: unrolled, they multiply the particle loop's
        // code until the instruction cache misses dominate
        #pragma unroll 1
        for (int di = -2; di <= 1; ++di) {
            int a = i + di; if (a < 0 || a > m.NXMC - 1) continue;
            #pragma unroll 1
            for (int b = j0 - 2; b <= j0 + NJ; ++b) {
                if (b < 0 || b > m.NYMC - 1) continue;
                const int cb = a * m.NYMC * m.NZMC + b * m.NZMC;
                const int cc0 = max(k0 - 2, 0), cc1 = min(k0 + NK, m.NZMC - 1);
                // the column's cells are consecutive ranges: each cell's end is
                // the next one's start. An empty cell adds +0 to every node's
                // sums, which leaves them unchanged, so it is skipped.
                uint32_t qlo = __ldg(cl.off + cb + cc0);
                #pragma unroll 1
                for (int cc = cc0; cc <= cc1; ++cc) {
                    int c = cb + cc;
                    const uint32_t q1 = __ldg(cl.off + c + 1);
                    const uint32_t q0 = qlo;
                    qlo = q1;
                    if (q0 == q1 || !(__ldg(cl.tmask + c) & need)) continue;
                    float rx[NJ][NK], ry[NJ][NK], rz[NJ][NK];
                    float sx[NJ][NK], sy[NJ][NK], sz[NJ][NK];
                    #pragma unroll
                    for (int u = 0; u < NJ; u++)
                        #pragma unroll
                        for (int v = 0; v < NK; v++) rx[u][v] = ry[u][v] = rz[u][v] = sx[u][v] = sy[u][v] = sz[u][v] = 0.0f;
                    #pragma unroll 1
                    for (uint32_t q = q0; q < q1; ++q) {
                        float4 o = __ldg(pos + q);
                        int f = pflag(o);
                        bool ok = SURF == MP_MC_SOLID ? (f == MP_TYPESOLID)
                                : SURF == MP_MC_FLUID ? (f == MP_TYPEAIR || f == MP_TYPEAIRSOLO || f == MP_TYPEFLUID)
                                                      : (f == MP_TYPEAIR || (f == MP_TYPEAIRSOLO && scene != MP_SCENE_INTERACTION));
                        if (!ok) continue;
                        const bool gas = GAS2 && (f == MP_TYPEAIR || (f == MP_TYPEAIRSOLO && scene != MP_SCENE_INTERACTION));
                        const float dx = o.x - px;
                        #pragma unroll
                        for (int u = 0; u < NJ; u++) {
                            // node j0 + u takes cells j0 + u - 2 .. j0 + u + 1
                            if (b - j0 - u < -2 || b - j0 - u > 1) continue;
                            const float dy = o.y - py[u];
                            const float dxy = dx * dx + dy * dy;
                            #pragma unroll
                            for (int v = 0; v < NK; v++) {
                                if (cc - k0 - v < -2 || cc - k0 - v > 1) continue;
                                const float dz = o.z - pz[v];
                                // dot(d, d) evaluates (x*x + y*y) + z*z; beyond the kernel
                                // radius the weight is exactly zero and the pair adds nothing:
                                // skip it before the sqrt (exact test with margin)
                                const float d2 = dxy + dz * dz;
                                if (d2 > cut) continue;
                                const float dis = sqrtf(d2);
                                if (!(dis < R)) continue;
                                float w;
                                if (SURF == MP_MC_SOLID) {
                                    w = dis / (4 * hm);
                                    w = 1 - w * w;
                                    w = (float)fmax((double)(w * w * w), 0.0);
                                } else {
                                    w = R * R - dis * dis;
                                    w = w * w * w;
                                }
                                rx[u][v] += o.x * w; ry[u][v] += o.y * w; rz[u][v] += o.z * w; ws[u][v] += w;
                                if (gas) { sx[u][v] += o.x * w; sy[u][v] += o.y * w; sz[u][v] += o.z * w; gw[u][v] += w; }
                            }
                        }
                    }
                    // a node outside this cell's window kept res = +0, and center + (+0)
                    // is center (center is never -0: it starts at +0 and sums of finite
                    // values round to +0)
                    #pragma unroll
                    for (int u = 0; u < NJ; u++)
                        #pragma unroll
                        for (int v = 0; v < NK; v++) {
                            cx[u][v] += rx[u][v]; cy[u][v] += ry[u][v]; cz[u][v] += rz[u][v];
                            if (GAS2) { gx[u][v] += sx[u][v]; gy[u][v] += sy[u][v]; gz[u][v] += sz[u][v]; }
                        }
                }
            }
        }
        #pragma unroll
        for (int u = 0; u < NJ; u++)
            #pragma unroll
            for (int v = 0; v < NK; v++) {
                const int j = j0 + u, k = k0 + v;
                if (j >= m.H || k >= m.D) continue;
                const float3 p = mk3(px, py[u], pz[v]);
                float3 center = mk3(cx[u][v], cy[u][v], cz[u][v]);
                const float wsum = ws[u][v];
                bool border = (i * j * k == 0 || i == m.NXMC || j == m.NYMC || k == m.NZMC);
                float phi;
                if (SURF == MP_MC_SOLID) {
                    float r = 0.75f * hm, thigh = 0.51f, tlow = 0.49f;
                    if (wsum > 0) {
                        center /= wsum;
                        float Ev = fmaxf(center.x, fmaxf(center.y, center.z)) / (4 * hm);
                        float gamma = (thigh - Ev) / (thigh - tlow);
                        float f = (Ev < tlow) ? 1 : gamma * gamma * gamma - 3 * gamma * gamma + 3 * gamma;
                        phi = (length(p - center) - r * f);
                    } else phi = -r;
                    if (border) phi = fminf(phi, -10.0f);
                } else {
                    float r = SURF == MP_MC_FLUID ? 0.5f * hm : 0.8f * hm;
                    if (wsum > 0) { center /= wsum; phi = r - length(p - center); }
                    else phi = -r;
                    if (border) phi = -1000.0f;
                    if (GAS2) {
                        const float r2 = 0.8f * hm;
                        float3 center2 = mk3(gx[u][v], gy[u][v], gz[u][v]);
                        const float wsum2 = gw[u][v];
                        float phi2;
                        if (wsum2 > 0) { center2 /= wsum2; phi2 = r2 - length(p - center2); }
                        else phi2 = -r2;
                        if (border) phi2 = -1000.0f;
                        dens2[(i * m.H + j) * m.D + k] = phi2;
                    }
                }
                dens[(i * m.H + j) * m.D + k] = phi;
            }
    }
}

// raises *flag when some cell's type mask has `bits`
__global__ void k_mc_any_type(long long n, const uint8_t* __restrict__ tmask, uint32_t bits, uint32_t* flag) {
    MP_GRID_LOOP(c, n) {
        bool hit = (tmask[c] & bits) != 0;
        if (__any_sync(__activemask(), hit) && (threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1))
            atomicOr(flag, 1u);
    }
}
// the solid field when no cell holds a SOLID particle: every node has wsum = 0,
// so the density pass writes -r, and -10 on the border (its min with -r)
__global__ void k_mc_solid_empty(McGrid m, float* __restrict__ dens) {
    const long long tot = (long long)m.W * m.H * m.D;
    const float r = 0.75f * m.hm;
    MP_GRID_LOOP(t, tot) {
        int i, j, k; getijk3((int)t, m.H, m.D, i, j, k);
        bool border = (i * j * k == 0 || i == m.NXMC || j == m.NYMC || k == m.NZMC);
        dens[t] = border ? fminf(-r, -10.0f) : -r;
    }
}

__device__ __forceinline__ float node(const McGrid& m, const float* d, int i, int j, int k) {
    return d[(size_t)i * m.H * m.D + (size_t)j * m.D + k];
}
__device__ __forceinline__ uint32_t cube_index(const McGrid& m, const float* d, int i, int j, int k) {
    float f[8] = {node(m, d, i, j, k), node(m, d, i + 1, j, k), node(m, d, i + 1, j + 1, k), node(m, d, i, j + 1, k),
                  node(m, d, i, j, k + 1), node(m, d, i + 1, j, k + 1), node(m, d, i + 1, j + 1, k + 1), node(m, d, i, j + 1, k + 1)};
    uint32_t ci = 0;
    #pragma unroll
    for (int v = 0; v < 8; v++) ci += (uint32_t)(f[v] < 0.0f) << v;
    return ci;
}
__global__ void k_mc_classify(McGrid m, const float* __restrict__ dens, const int32_t* __restrict__ nvt,
                              uint8_t* __restrict__ cube, uint32_t* __restrict__ nverts, uint32_t* __restrict__ occ) {
    long long tot = (long long)m.NXMC * m.NYMC * m.NZMC;
    MP_GRID_LOOP(t, tot) {
        int i, j, k; getijk3((int)t, m.NYMC, m.NZMC, i, j, k);
        uint32_t ci = cube_index(m, dens, i, j, k);
        uint32_t nv = (uint32_t)__ldg(nvt + ci);
        cube[t] = (uint8_t)ci;
        nverts[t] = nv;
        occ[t] = nv > 0 ? 1u : 0u;
    }
}
__global__ void k_mc_compact(long long nvox, const uint32_t* __restrict__ occ, const uint32_t* __restrict__ scan,
                             uint32_t* __restrict__ out) {
    MP_GRID_LOOP(t, nvox) if (occ[t]) out[scan[t]] = (uint32_t)t;
}
// edge id = 3 * node + (x: 1, y: 0, z: 2) at the edge's lower node (GetEdgeID, spray_k.cu:1926-1959)
__device__ __forceinline__ uint32_t edge_gid(const McGrid& m, int i, int j, int k, int e) {
    // corner offsets of the lower node and the axis of each of the 12 cube edges
    const int lo[12][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,0},{0,0,1},{1,0,1},{0,1,1},{0,0,1},{0,0,0},{1,0,0},{1,1,0},{0,1,0}};
    const int ax[12] = {0, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2};
    uint32_t nd = (uint32_t)((i + lo[e][0]) * m.H * m.D + (j + lo[e][1]) * m.D + (k + lo[e][2]));
    int off = ax[e] == 0 ? 1 : (ax[e] == 1 ? 0 : 2);
    return 3u * nd + (uint32_t)off;
}
__global__ void k_mc_mark_edges(McGrid m, uint32_t nact, const uint32_t* __restrict__ act, const uint8_t* __restrict__ cube,
                                const int32_t* __restrict__ nvt, const int32_t* __restrict__ tri, uint32_t* __restrict__ em) {
    MP_GRID_LOOP(a, nact) {
        uint32_t v = act[a];
        int i, j, k; getijk3((int)v, m.NYMC, m.NZMC, i, j, k);
        int ci = cube[v];
        int nv = __ldg(nvt + ci);
        for (int t = 0; t < nv; t++) em[edge_gid(m, i, j, k, __ldg(tri + ci * 16 + t))] = 1u;
    }
}
__global__ void k_mc_vertices(McGrid m, long long nedge, const uint32_t* __restrict__ em, const uint32_t* __restrict__ es,
                              const float* __restrict__ dens, float3* __restrict__ verts) {
    MP_GRID_LOOP(e, nedge) {
        if (!em[e]) continue;
        uint32_t nd = (uint32_t)(e / 3);
        int off = (int)(e % 3);
        int axis = off == 1 ? 0 : (off == 0 ? 1 : 2);
        int i = (int)(nd / ((uint32_t)m.H * m.D)), j = (int)((nd / m.D) % m.H), k = (int)(nd % m.D);
        float vs = m.hm;
        float3 p0 = mk3((float)i * vs, (float)j * vs, (float)k * vs);
        float3 p1 = p0 + (axis == 0 ? mk3(vs, 0, 0) : (axis == 1 ? mk3(0, vs, 0) : mk3(0, 0, vs)));
        float f0 = node(m, dens, i, j, k);
        float f1 = axis == 0 ? node(m, dens, i + 1, j, k) : (axis == 1 ? node(m, dens, i, j + 1, k) : node(m, dens, i, j, k + 1));
        float t = (0.0f - f0) / (f1 - f0);
        verts[es[e]] = p0 + t * (p1 - p0);
    }
}
__global__ void k_mc_indices(McGrid m, uint32_t nact, const uint32_t* __restrict__ act, const uint8_t* __restrict__ cube,
                             const uint32_t* __restrict__ vscan, const int32_t* __restrict__ nvt,
                             const int32_t* __restrict__ tri, const uint32_t* __restrict__ es, uint32_t* __restrict__ idx) {
    MP_GRID_LOOP(a, nact) {
        uint32_t v = act[a];
        int i, j, k; getijk3((int)v, m.NYMC, m.NZMC, i, j, k);
        int ci = cube[v];
        int nv = __ldg(nvt + ci);
        uint32_t base = vscan[v];
        for (int t = 0; t < nv; t++) idx[base + t] = es[edge_gid(m, i, j, k, __ldg(tri + ci * 16 + t))];
    }
}
// vertex -> incident (triangle corner) slots, ascending
__global__ void k_mc_inc_count(uint32_t nidx, const uint32_t* __restrict__ idx, uint32_t* __restrict__ cnt) {
    MP_GRID_LOOP(s, nidx) atomicAdd(cnt + idx[s], 1u);
}
__global__ void k_mc_inc_fill(uint32_t nidx, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ start,
                              uint32_t* __restrict__ cnt, uint32_t* __restrict__ inc) {
    MP_GRID_LOOP(s, nidx) {
        uint32_t v = idx[s];
        uint32_t r = atomicSub(cnt + v, 1u) - 1u;
        inc[start[v] + r] = (uint32_t)s;
    }
}
__global__ void k_mc_inc_sort(uint32_t nv, const uint32_t* __restrict__ start, uint32_t* __restrict__ inc) {
    MP_GRID_LOOP(v, nv) {
        uint32_t s0 = start[v];
        sort_distinct_run(inc, s0, start[v + 1] - s0, [](uint32_t) {});
    }
}
__global__ void k_mc_smooth(uint32_t nv, const uint32_t* __restrict__ start, const uint32_t* __restrict__ inc,
                            const uint32_t* __restrict__ idx, const float3* __restrict__ vin, float3* __restrict__ vout) {
    MP_GRID_LOOP(v, nv) {
        float3 pq = vin[v];
        float3 disp = mk3(0.0f);
        int w = 0;
        for (uint32_t s = start[v]; s < start[v + 1]; s++) {
            uint32_t slot = inc[s];
            uint32_t t = slot / 3, c = slot % 3;
            uint32_t o1 = idx[3 * t + (c == 0 ? 1 : 0)];
            uint32_t o2 = idx[3 * t + (c == 2 ? 1 : 2)];
            disp += vin[o1] - pq;
            disp += vin[o2] - pq;
            w += 2;
        }
        vout[v] = (w > 0) ? pq + 0.5f * disp / (float)w : pq;
    }
}
__global__ void k_mc_normals(uint32_t nv, const uint32_t* __restrict__ start, const uint32_t* __restrict__ inc,
                             const uint32_t* __restrict__ idx, const float3* __restrict__ verts, float3* __restrict__ nrm) {
    MP_GRID_LOOP(v, nv) {
        float3 n = mk3(0.0f);
        for (uint32_t s = start[v]; s < start[v + 1]; s++) {
            uint32_t t = inc[s] / 3;
            float3 p1 = verts[idx[3 * t]], p2 = verts[idx[3 * t + 1]], p3 = verts[idx[3 * t + 2]];
            n += cross(p2 - p1, p3 - p1);
        }
        if (length(n) > 0) n = normalize(n);
        nrm[v] = n;
    }
}

}  // namespace

static int readback(MpCtx* c, const uint32_t* dptr, uint32_t* h) {
    MP_CUDA(c, cudaMemcpyAsync(h, dptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

static McGrid mc_grid(const MpCtx* c) {
    McGrid m;
    m.NXMC = 2 * c->G.NX; m.NYMC = 2 * c->G.NY; m.NZMC = 2 * c->G.NZ;
    m.W = m.NXMC + 1; m.H = m.NYMC + 1; m.D = m.NZMC + 1;
    m.hm = c->G.h / (float)(m.NXMC / c->G.NX);
    return m;
}

// nodes per thread of the density gather (along j, along k) and its
// resident-blocks hint, for the single-field and the fused fluid + gas passes
#ifndef MC_DENS_NJ
#define MC_DENS_NJ 1
#endif
#ifndef MC_DENS_NK
#define MC_DENS_NK 1
#endif
#ifndef MC_DENS_MINB
#define MC_DENS_MINB 6
#endif
#ifndef MC_GAS2_NJ
#define MC_GAS2_NJ 2
#endif
#ifndef MC_GAS2_NK
#define MC_GAS2_NK 1
#endif
#ifndef MC_GAS2_MINB
#define MC_GAS2_MINB 4
#endif
template <int SURF, bool GAS2>
static void launch_density(const McGrid& m, Cells cl, const float4* pos, float* dens, int scene, float* dens2,
                           cudaStream_t s) {
    constexpr int NJ = GAS2 ? MC_GAS2_NJ : MC_DENS_NJ, NK = GAS2 ? MC_GAS2_NK : MC_DENS_NK;
    constexpr int MINB = GAS2 ? MC_GAS2_MINB : MC_DENS_MINB;
    const Tiles T = make_tiles(m.W, (m.H + NJ - 1) / NJ, (m.D + NK - 1) / NK);
    k_mc_density<SURF, GAS2, NJ, NK, MINB><<<mp_blocks(T.threads(), 256), 256, 0, s>>>(m, T, cl, pos, dens, scene, dens2);
}
static int mc_extract(MpCtx* c, const McGrid& m, int surface, const float* dens);

// one runMC_smooth surface (spray.cu:804-979)
int k_mc(MpCtx* c, int surface) {
    if (!c->mc_sorted) { c->err = "mc: particles are not sorted on the 2x grid (call mp_mc_presort)"; return MP_ERR_STATE; }
    const McGrid m = mc_grid(c);
    Cells cl{c->cell_off, c->tmask};
    cudaStream_t s = c->stream;
    bool solid_empty = false;
    if (surface == MP_MC_SOLID) {
        const long long nvox = (long long)m.NXMC * m.NYMC * m.NZMC;
        MP_CUDA(c, cudaMemsetAsync(c->u32_scratch + 4, 0, sizeof(uint32_t), s));
        k_mc_any_type<<<mp_blocks(nvox, 256), 256, 0, s>>>(nvox, c->tmask, 1u << MP_TYPESOLID, c->u32_scratch + 4);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        uint32_t any = 1;
        MP_TRY(readback(c, c->u32_scratch + 4, &any));
        solid_empty = any == 0;
    }
    if (solid_empty) {
        k_mc_solid_empty<<<mp_blocks((long long)m.W * m.H * m.D, 256), 256, 0, s>>>(m, c->mc_dens);
    } else {
        KtScope kt(c, MP_KT_MC_DENS);
        if (surface == MP_MC_SOLID) launch_density<MP_MC_SOLID, false>(m, cl, c->pos, c->mc_dens, c->P.scene, nullptr, s);
        else if (surface == MP_MC_FLUID) launch_density<MP_MC_FLUID, false>(m, cl, c->pos, c->mc_dens, c->P.scene, nullptr, s);
        else launch_density<MP_MC_GAS, false>(m, cl, c->pos, c->mc_dens, c->P.scene, nullptr, s);
    }
    c->launches++;
    return mc_extract(c, m, surface, c->mc_dens);
}

// the fluid and gas surfaces of one step from a single density pass (the
// same fields and meshes as k_mc(FLUID) followed by k_mc(GAS))
int k_mc_fluid_gas(MpCtx* c) {
    if (!c->mc_sorted) { c->err = "mc: particles are not sorted on the 2x grid (call mp_mc_presort)"; return MP_ERR_STATE; }
    const McGrid m = mc_grid(c);
    Cells cl{c->cell_off, c->tmask};
    {
        KtScope kt(c, MP_KT_MC_DENS);
        launch_density<MP_MC_FLUID, true>(m, cl, c->pos, c->mc_dens, c->P.scene, c->mc_dens2, c->stream);
    }
    c->launches++;
    MP_TRY(mc_extract(c, m, MP_MC_FLUID, c->mc_dens));
    return mc_extract(c, m, MP_MC_GAS, c->mc_dens2);
}

// incidence lists of a surface's vertices (vstart: nv+1, inc: nidx), each
// list ascending
static int mc_incidence(MpCtx* c, const McSurface& out, uint32_t nv, uint32_t nidx) {
    cudaStream_t s = c->stream;
    MP_CUDA(c, cudaMemsetAsync(c->mc_fill, 0, sizeof(uint32_t) * (nv + 1), s));
    k_mc_inc_count<<<mp_blocks(nidx, 256), 256, 0, s>>>(nidx, out.indices, c->mc_fill);
    c->launches++;
    MP_TRY(mp_scan_u32(c, c->mc_fill, c->mc_vstart, nv));
    k_mc_inc_fill<<<mp_blocks(nidx, 256), 256, 0, s>>>(nidx, out.indices, c->mc_vstart, c->mc_fill, c->mc_inc);
    k_mc_inc_sort<<<mp_blocks(nv, 256), 256, 0, s>>>(nv, c->mc_vstart, c->mc_inc);
    c->launches += 2;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// runMC_interaction's stored-surface branch (spray.cu:788-794): calNormals
// on the surface as it stands (moved by the solid motion), no re-extraction
int k_mc_renormal(MpCtx* c, int surface) {
    McSurface& out = c->mc[surface];
    const uint32_t nv = (uint32_t)out.nverts, nidx = (uint32_t)out.nindices;
    if (nv == 0) return MP_OK;
    MP_TRY(mc_incidence(c, out, nv, nidx));
    k_mc_normals<<<mp_blocks(nv, 256), 256, 0, c->stream>>>(nv, c->mc_vstart, c->mc_inc, out.indices, out.verts,
                                                              out.normals);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// classification, compaction, vertices, indices, smoothing and normals of one
// surface from its nodal field
static int mc_extract(MpCtx* c, const McGrid& m, int surface, const float* dens) {
    long long nnode = (long long)m.W * m.H * m.D;
    long long nvox = (long long)m.NXMC * m.NYMC * m.NZMC;
    cudaStream_t s = c->stream;
    McSurface& out = c->mc[surface];
    out.nverts = out.nindices = out.active = 0;
    c->mc_last_dens = dens;
    k_mc_classify<<<mp_blocks(nvox, 256), 256, 0, s>>>(m, dens, c->mc_numverts, c->mc_cube, c->mc_vverts, c->mc_vflag);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_TRY(mp_scan_u32(c, c->mc_vflag, c->mc_vscan, (size_t)nvox));
    uint32_t nact = 0;
    MP_TRY(readback(c, c->mc_vscan + nvox, &nact));
    out.active = (int)nact;
    c->S.mc_active_voxels[surface] = (int)nact;
    c->S.mc_verts[surface] = 0; c->S.mc_indices[surface] = 0;
    if (nact == 0) return MP_OK;
    k_mc_compact<<<mp_blocks(nvox, 256), 256, 0, s>>>(nvox, c->mc_vflag, c->mc_vscan, c->mc_compact);
    c->launches++;
    MP_TRY(mp_scan_u32(c, c->mc_vverts, c->mc_vvscan, (size_t)nvox));
    uint32_t nidx = 0;
    MP_TRY(readback(c, c->mc_vvscan + nvox, &nidx));
    if ((long long)nidx > 3LL * c->P.mc_max_tris) { c->err = "mc: triangle cap exceeded"; return MP_ERR_CAPACITY; }
    long long nedge = 3 * nnode;
    MP_CUDA(c, cudaMemsetAsync(c->mc_emark, 0, sizeof(uint32_t) * nedge, s));
    k_mc_mark_edges<<<mp_blocks(nact, 256), 256, 0, s>>>(m, nact, c->mc_compact, c->mc_cube, c->mc_numverts, c->mc_tri, c->mc_emark);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_TRY(mp_scan_u32(c, c->mc_emark, c->mc_escan, (size_t)nedge));
    uint32_t nv = 0;
    MP_TRY(readback(c, c->mc_escan + nedge, &nv));
    if ((long long)nv > c->P.mc_max_verts) { c->err = "mc: vertex cap exceeded"; return MP_ERR_CAPACITY; }
    k_mc_vertices<<<mp_blocks(nedge, 256), 256, 0, s>>>(m, nedge, c->mc_emark, c->mc_escan, dens, out.verts);
    k_mc_indices<<<mp_blocks(nact, 256), 256, 0, s>>>(m, nact, c->mc_compact, c->mc_cube, c->mc_vvscan, c->mc_numverts,
                                                      c->mc_tri, c->mc_escan, out.indices);
    c->launches += 2;
    MP_CHECK_LAUNCH(c);
    MP_TRY(mc_incidence(c, out, nv, nidx));
    if (c->P.b_smooth_mc) {
        for (int it = 0; it < c->P.smooth_iters; it++) {
            k_mc_smooth<<<mp_blocks(nv, 256), 256, 0, s>>>(nv, c->mc_vstart, c->mc_inc, out.indices, out.verts, c->mc_tmpv);
            c->launches++;
            MP_CUDA(c, cudaMemcpyAsync(out.verts, c->mc_tmpv, sizeof(float3) * nv, cudaMemcpyDeviceToDevice, s));
        }
    }
    k_mc_normals<<<mp_blocks(nv, 256), 256, 0, s>>>(nv, c->mc_vstart, c->mc_inc, out.indices, out.verts, out.normals);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    out.nverts = (int)nv; out.nindices = (int)nidx;
    c->S.mc_verts[surface] = (int)nv;
    c->S.mc_indices[surface] = (int)nidx;
    return MP_OK;
}
