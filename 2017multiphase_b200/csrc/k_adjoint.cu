// k_adjoint.cu — reverse-mode derivative of the FLUID (and AIR) step.
//
// The reference has no differentiation. This module differentiates the
// program the bubblesim step (spray.cpp:979-1233) runs for a scene of FLUID
// particles, or of FLUID and AIR particles, with the position corrections and
// the solo-air stages off:
//   external forces (addexternalforce: gravity on FLUID, the buoyancy of AIR)
//   -> velocity splats to faces (mapvelp2g_k_fluidSolid, spray_k.cu:2809-2866,
//      and mapvelp2g_k_air, spray_k.cu:2894-2937)
//   -> extrapolation, two Jacobi passes (sweepu_k_bubble, spray_k.cu:3779-3880)
//   -> wall rules (setWaterBoundaryU_k, spray_k.cu:956-995)
//   -> projection (cptdivergence_bubble2 with the level-set blend at
//      liquid-air faces, solver_cg_bubble, subGradPress on both fields)
//   -> extrapolation + wall rules again
//   -> FLIP/PIC gather of each phase's field (mapvelg2p_flip_bubble,
//      spray_k.cu:3525-3540, blended with the new grid velocity by flip_alpha
//      as spray_k.cu:3487-3490)
//   -> advection with the wall clamp (CollisionWithSolid_k, spray_k.cu:5276)
// and, after the last step, the loss sum_s phi(y_s)^2 of the fluid distance
// field (genlevelset, spray_k.cu:2753-2806) at target points y_s.
//
// Discrete state is recorded by running the engine's own stages once
// (mp_adj_record) and then held fixed: the particle order and cell ranges of
// each step's splat, the cell marks, the extrapolation distance field and the
// nearest particle of each cell at the end. The derivative is that of the
// program with this state frozen (the program is piecewise smooth; the frozen
// state is the piece the recorded run lies on). The replay of the continuous
// part and its transpose are templated on the arithmetic type: FP32 (the
// engine's) and FP64 (the reference gradient and finite differences).
//
// Every transpose is a gather (faces over the particles of nearby cells,
// particles over nearby faces, cells over nearby samples), so gradients are
// deterministic. The projection's transpose is a second CG solve on the
// symmetric pressure matrix. States are checkpointed every `every` steps and
// recomputed segment by segment during the reverse sweep; each step's
// intermediates are recomputed from its state just before its transpose, so
// only one step's are held (the splats and the pressure and heat solves of
// the first replay are kept per step, so the recomputations neither splat
// nor solve).
#include "ctx.cuh"
#include <algorithm>
#include <cstring>
#include <vector>

using namespace mpk;

int k_hash_sort(MpCtx* c);

struct AdjTape {
    int np = 0, nsteps = 0, every = 0;
    std::vector<uint32_t*> order, off;   // per step: sorted slot -> particle id; cell ranges
    std::vector<int8_t*> mark;           // per step: cell marks
    std::vector<float*> phi;             // per step: fluid extrapolation distance
    float* x0 = nullptr;                 // initial positions (id order, xyz)
    float* v0 = nullptr;                 // initial velocities (id order, xyz)
    float* mass = nullptr;               // id order
    uint32_t* ids = nullptr;             // engine slot -> particle id while recording
    uint32_t* ids2 = nullptr;
    uint32_t* nearest = nullptr;         // per cell: nearest FLUID particle id at the end, or ~0u
    float* samples = nullptr;            // target points sorted by their base cell
    int nsamples = 0;
    uint32_t* s_off = nullptr;           // per base cell: range of its samples (n + 1)
    // the heat stage (b_heat_trans): per step, the sort and the cell marks it ran on
    bool heat = false;
    std::vector<uint32_t*> order_h, off_h;
    std::vector<int8_t*> mark_h;
    float* T0 = nullptr;                 // initial temperatures (id order)
    float* fixedheat = nullptr;          // the fixed-heat field (b_fixed_heat), or null
    // the air phase (AIR particles present): each particle's phase (0 FLUID,
    // 1 AIR; fixed, the program has no AIR <-> AIRSOLO transitions), the splat
    // masses of each phase (0 for the other phase's particles), and per step
    // the merged level set (the divergence's blend) and the air extrapolation
    // distance
    bool air = false;
    uint8_t* phase = nullptr;
    char* arena = nullptr;               // every step's recorded state, one allocation
    float* mass_w = nullptr;
    float* mass_a = nullptr;
    std::vector<float*> lsm, phia;
    // the engine's projection of each step (its right-hand side and pressure),
    // kept when the engine's solve is the one the FP32 replay runs (mixed
    // precision, the reference's coefficients, no refinement or periodic true
    // residual): a replay step whose right-hand side equals the engine's bit
    // for bit takes the engine's pressure instead of solving again (the solve
    // is deterministic, so it would give the same)
    bool eng = false;
    std::vector<float*> eng_b, eng_p;
    // the engine's state (positions, velocities in recording order) at the
    // start of every segment after the first and at the end: at the recorded
    // inputs the FP32 replay reproduces it bit for bit, so a gradient there
    // needs no first replay over all steps (each segment's replay checks that
    // it ends on the engine's state)
    float* eng_xs = nullptr;
    float* eng_vs = nullptr;
    // replay / adjoint work, sized for `wesz`-byte elements
    size_t wesz = 0;
    int wk_ns = 0;                       // samples the work was sized for
    std::vector<void*> wk;
};

namespace {

constexpr uint32_t NONE = 0xffffffffu;

template <class T> struct Fc { T* x; T* y; T* z; };
template <class T> Fc<T> faces_of(void* base, const Grid& g) {
    T* b = static_cast<T*>(base);
    return Fc<T>{b, b + g.nfx, b + g.nfx + g.nfy};
}
// flat face index t -> axis and (i,j,k) in that axis' face grid
__device__ __forceinline__ int face_decode(const Grid& g, long long t, int& i, int& j, int& k, int& idx) {
    if (t < g.nfx) { idx = (int)t; getijk3(idx, g.NY, g.NZ, i, j, k); return 0; }
    if (t < (long long)g.nfx + g.nfy) { idx = (int)(t - g.nfx); getijk3(idx, g.NY + 1, g.NZ, i, j, k); return 1; }
    idx = (int)(t - g.nfx - g.nfy); getijk3(idx, g.NY, g.NZ + 1, i, j, k); return 2;
}
__device__ __forceinline__ int face_index(const Grid& g, int ax, int i, int j, int k) {
    return ax == 0 ? fxi(g, i, j, k) : (ax == 1 ? fyi(g, i, j, k) : fzi(g, i, j, k));
}
template <class T> __device__ __forceinline__ T* fsel(const Fc<T>& f, int ax) { return ax == 0 ? f.x : (ax == 1 ? f.y : f.z); }

// ---- recording helpers --------------------------------------------------------
__global__ void k_ad_iota(int n, uint32_t* a) { MP_GRID_LOOP(i, n) a[i] = (uint32_t)i; }
__global__ void k_ad_permute_ids(int n, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ in,
                                 uint32_t* __restrict__ out) {
    MP_GRID_LOOP(s, n) out[s] = in[perm[s]];
}
__global__ void k_ad_snapshot(int n, const uint32_t* __restrict__ ids, const float4* __restrict__ pos,
                              const float4* __restrict__ vel, float* __restrict__ x, float* __restrict__ v,
                              float* __restrict__ m) {
    MP_GRID_LOOP(s, n) {
        uint32_t id = ids[s];
        float4 p = pos[s], q = vel[s];
        x[3 * id] = p.x; x[3 * id + 1] = p.y; x[3 * id + 2] = p.z;
        v[3 * id] = q.x; v[3 * id + 1] = q.y; v[3 * id + 2] = q.z;
        m[id] = q.w;
    }
}
__global__ void k_ad_snapshot_T(int n, const uint32_t* __restrict__ ids, const float4* __restrict__ heat,
                                float* __restrict__ T) {
    MP_GRID_LOOP(s, n) T[ids[s]] = heat[s].x;
}
// counts the particles that are neither FLUID nor AIR (cnt[0]) and the AIR ones (cnt[2])
__global__ void k_ad_count_types(int n, const float4* __restrict__ pos, uint32_t* cnt) {
    MP_GRID_LOOP(s, n) {
        const int f = pflag(pos[s]);
        if (f != MP_TYPEFLUID && f != MP_TYPEAIR) atomicAdd(cnt, 1u);
        else if (f == MP_TYPEAIR) atomicAdd(cnt + 2, 1u);
    }
}
// each particle's phase and per-phase splat mass
__global__ void k_ad_snapshot_phase(int n, const uint32_t* __restrict__ ids, const float4* __restrict__ pos,
                                    const float4* __restrict__ vel, uint8_t* __restrict__ phase,
                                    float* __restrict__ mw, float* __restrict__ ma) {
    MP_GRID_LOOP(s, n) {
        const uint32_t id = ids[s];
        const bool air = pflag(pos[s]) == MP_TYPEAIR;
        const float m = vel[s].w;
        phase[id] = air ? 1 : 0;
        mw[id] = air ? 0.0f : m;
        ma[id] = air ? m : 0.0f;
    }
}
// nearest FLUID particle of each cell centre within the genlevelset window
// (2.5 cells; the +-2 cell box in a fixed order, first minimum kept)
__global__ void k_ad_nearest(Grid g, Cells cl, const float4* __restrict__ pos, const uint32_t* __restrict__ ids,
                             uint32_t* __restrict__ nearest) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        float h = g.h;
        float3 gp = (mk3((float)i, (float)j, (float)k) + mk3(0.5f, 0.5f, 0.5f)) * h;
        const float cap = 6.25f * h * h;
        // a bound from the 27 nearest cells first: a window cell (di,dj,dk)
        // holds no particle closer than ((|d|-0.5)h)^2 summed over the axes
        // (shrunk by 1e-4 relative against the rounding of d2), so the ones
        // whose bound exceeds it cannot hold the minimum or a tie with it
        float bound = cap;
        for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
            int a = i + di, b = j + dj, cc = k + dk;
            if (a < 0 || a >= g.NX || b < 0 || b >= g.NY || cc < 0 || cc >= g.NZ) continue;
            int c = cid(g, a, b, cc);
            for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                float4 q = pos[s];
                if (pflag(q) != MP_TYPEFLUID) continue;
                float3 d = xyz(q) - gp;
                bound = fminf(bound, dot(d, d));
            }
        }
        // the fixed order of the +-2 box, first minimum kept
        float best = cap;
        uint32_t who = NONE;
        for (int di = -2; di <= 2; di++) for (int dj = -2; dj <= 2; dj++) for (int dk = -2; dk <= 2; dk++) {
            int a = i + di, b = j + dj, cc = k + dk;
            if (a < 0 || a >= g.NX || b < 0 || b >= g.NY || cc < 0 || cc >= g.NZ) continue;
            const float bx = di == 0 ? 0.f : ((float)abs(di) - 0.5f), by = dj == 0 ? 0.f : ((float)abs(dj) - 0.5f);
            const float bz = dk == 0 ? 0.f : ((float)abs(dk) - 0.5f);
            if ((bx * bx + by * by + bz * bz) * h * h * 0.9999f > bound) continue;
            int c = cid(g, a, b, cc);
            for (uint32_t s = cl.off[c]; s < cl.off[c + 1]; s++) {
                float4 q = pos[s];
                if (pflag(q) != MP_TYPEFLUID) continue;
                float3 d = xyz(q) - gp;
                float d2 = dot(d, d);
                if (d2 < best) { best = d2; who = ids[s]; }
            }
        }
        nearest[idx] = who;
    }
}

// raises *flag when a and b differ in some bit
__global__ void k_ad_differ(int n, const float* __restrict__ a, const float* __restrict__ b, uint32_t* flag) {
    MP_GRID_LOOP(i, n) {
        const bool d = __float_as_uint(a[i]) != __float_as_uint(b[i]);
        if (__any_sync(__activemask(), d) && (threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1))
            atomicOr(flag, 1u);
    }
}
// ---- replay of the continuous part ----------------------------------------------
template <class T>
__global__ void k_ad_gravity(int np, const T* __restrict__ v, T* __restrict__ va, T dtg) {
    MP_GRID_LOOP(p, np) {
        va[3 * p] = v[3 * p]; va[3 * p + 1] = v[3 * p + 1];
        va[3 * p + 2] = v[3 * p + 2] + dtg;
    }
}
// addexternalforce for FLUID and AIR particles (k_forces): FLUID v += dt g; AIR
// v_z -= dt g_z rate bra with rate = max(vmax - v_z, 0) / vmax
template <class T>
__global__ void k_ad_forces(int np, const uint8_t* __restrict__ phase, const T* __restrict__ v, T* __restrict__ va,
                            T dtg, T bra, T vmax) {
    MP_GRID_LOOP(p, np) {
        va[3 * p] = v[3 * p]; va[3 * p + 1] = v[3 * p + 1];
        T vz = v[3 * p + 2];
        if (phase[p] == 0) vz = vz + dtg;
        else {
            T r = vmax - vz;
            r = r > (T)0 ? r : (T)0;
            vz = vz - dtg * (r / vmax) * bra;
        }
        va[3 * p + 2] = vz;
    }
}
// its transpose, in place on the velocity cotangent (v the step's input)
template <class T>
__global__ void k_ad_forces_adj(int np, const uint8_t* __restrict__ phase, const T* __restrict__ v,
                                const T* __restrict__ vab, T* __restrict__ vb, T dtg, T bra, T vmax) {
    MP_GRID_LOOP(p, np) {
        vb[3 * p] = vab[3 * p]; vb[3 * p + 1] = vab[3 * p + 1];
        T d = (T)1;
        if (phase[p] != 0 && vmax - v[3 * p + 2] > (T)0) d = (T)1 + dtg * bra / vmax;
        vb[3 * p + 2] = d * vab[3 * p + 2];
    }
}
template <class T> __device__ __forceinline__ T sharpk(T r2) {
    const T c = (T)1.4f * (T)1.4f;
    T rr = r2 > (T)0.0001f ? r2 : (T)0.0001f;
    T w = c / rr - (T)1;
    return w > (T)0 ? w : (T)0;
}
// d sharpk / d r2 (zero where the weight is clamped)
template <class T> __device__ __forceinline__ T sharpk_d(T r2) {
    const T c = (T)1.4f * (T)1.4f;
    if (!(r2 > (T)0.0001f)) return (T)0;
    if (!(c / r2 - (T)1 > (T)0)) return (T)0;
    return -c / (r2 * r2);
}
// face position in cell units
__device__ __forceinline__ void face_pos(int ax, int i, int j, int k, float& gx, float& gy, float& gz) {
    gx = (float)i + (ax == 0 ? 0.0f : 0.5f);
    gy = (float)j + (ax == 1 ? 0.0f : 0.5f);
    gz = (float)k + (ax == 2 ? 0.0f : 0.5f);
}
// cells holding an AIR particle in a step's recorded order (the air splat and
// the air faces' gather skip the others, as the engine's air splat skips cells
// by their type mask)
__global__ void k_ad_air_cells(int n, const uint32_t* __restrict__ off, const uint32_t* __restrict__ order,
                               const uint8_t* __restrict__ phase, uint8_t* __restrict__ airc) {
    MP_GRID_LOOP(c, n) {
        uint8_t a = 0;
        for (uint32_t q = off[c]; q < off[c + 1]; q++)
            if (phase[order[q]]) { a = 1; break; }
        airc[c] = a;
    }
}
// the splat windows: a face e along its normal takes the cells [e-LO, e+HI],
// across [-AC, AC]: the water splat (mapvelp2g_k_fluidSolid) [-1, 0] and
// [-1, 1], the air splat (mapvelp2g_k_air) [-2, 1] and [-2, 2]
template <int PH> struct SplatWin {
    static constexpr int LO = PH ? 2 : 1, HI = PH ? 1 : 0, AC = PH ? 2 : 1;
};
// splat: per face, the mass-weighted sharp-kernel average of the particles of
// its window's cells, in the order of the reference's loops (cells a, b, c
// ascending, then the particles of a cell); the records hold each particle's
// phase mass (0 for the other phase, which then adds nothing), and a pair
// beyond the kernel radius (weight 0) is skipped. A warp handles 32 nodes
// along k (i, j fixed), a thread a node's three faces: for each column (a, b)
// of the window the particles of the warp's cells along k are one contiguous
// range of the recorded order; the warp stages it in shared memory CAP
// records at a time with coalesced loads, and each lane walks its own part.
template <class T, int PH>
__global__ void __launch_bounds__(256) k_ad_p2g_w(Grid g, const uint32_t* __restrict__ off,
                                                  const T* __restrict__ xs4, const T* __restrict__ vs4, Fc<T> u,
                                                  Fc<T> W, const uint8_t* __restrict__ cellmask) {
    using Wn = SplatWin<PH>;
    constexpr int CAP = sizeof(T) == 4 ? 128 : 64;
    constexpr int R = Wn::AC;   // the union window: [-AC, AC] on every axis (LO == AC, HI <= AC)
    __shared__ T sm_x[8][CAP][4];
    __shared__ T sm_v[8][CAP][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Tiles Tl = make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1);
    const T scale = (T)1 / (T)g.h;
    const T cker = (T)1.4f * (T)1.4f;
    MP_GRID_LOOP(t, Tl.threads()) {
        int i, j, k;
        const bool act = tile_ijk(Tl, t, i, j, k);
        if (!__any_sync(0xffffffffu, act)) continue;
        const bool hx = act && j < g.NY && k < g.NZ, hy = act && i < g.NX && k < g.NZ, hz = act && i < g.NX && j < g.NY;
        T wx = 0, sx = 0, wy = 0, sy = 0, wz = 0, sz = 0;
        const T ti = (T)(float)i, tj = (T)(float)j, tk = (T)(float)k;
        const T half = (T)0.5f;
        const int klo = max(k - R, 0), khi = min(k + R, g.NZ - 1), kzhi = min(k + Wn::HI, g.NZ - 1);
        for (int di = -R; di <= R; di++) {
            const int a = i + di;
            if (a < 0 || a > g.NX - 1) continue;   // the same for the whole warp
            const bool ax = hx && di >= -Wn::LO && di <= Wn::HI;
            for (int dj = -R; dj <= R; dj++) {
                const int b = j + dj;
                if (b < 0 || b > g.NY - 1) continue;
                const bool ay = hy && dj >= -Wn::LO && dj <= Wn::HI;
                bool need = (ax || ay || hz) && klo <= khi;
                const int cb = cid(g, a, b, 0);
                if (need && cellmask) {
                    bool any = false;
                    for (int cc = klo; cc <= khi; cc++) any = any || cellmask[cb + cc];
                    need = any;
                }
                if (!__any_sync(0xffffffffu, need)) continue;
                uint32_t s0 = 0, s1 = 0, sz1 = 0;
                if (need) {
                    s0 = off[cb + klo]; s1 = off[cb + khi + 1];
                    sz1 = hz ? off[cb + kzhi + 1] : s0;
                }
                // the warp's range: the lanes' windows along k overlap, so their
                // ranges join into one
                const uint32_t A = __reduce_min_sync(0xffffffffu, need ? s0 : 0xffffffffu);
                const uint32_t B = __reduce_max_sync(0xffffffffu, need ? s1 : 0u);
                for (uint32_t c0 = A; c0 < B; c0 += CAP) {
                    const uint32_t n = min(B - c0, (uint32_t)CAP);
                    __syncwarp();
                    for (uint32_t q = lane; q < n; q += 32) {
                        const T* r = xs4 + 4 * (size_t)(c0 + q);
                        const T* v = vs4 + 4 * (size_t)(c0 + q);
                        sm_x[warp][q][0] = r[0]; sm_x[warp][q][1] = r[1]; sm_x[warp][q][2] = r[2];
                        sm_x[warp][q][3] = r[3];
                        sm_v[warp][q][0] = v[0]; sm_v[warp][q][1] = v[1]; sm_v[warp][q][2] = v[2];
                    }
                    __syncwarp();
                    if (!need) continue;
                    const uint32_t lo = max(s0, c0), hi = min(s1, c0 + n);
                    for (uint32_t p = lo; p < hi; ++p) {
                        const T m = sm_x[warp][p - c0][3];
                        if (m == (T)0) continue;   // the other phase: adds +0
                        const T X = sm_x[warp][p - c0][0] * scale, Y = sm_x[warp][p - c0][1] * scale;
                        const T Z = sm_x[warp][p - c0][2] * scale;
                        if (ax) {
                            const T dx = X - ti, dy = Y - (tj + half), dz = Z - (tk + half);
                            const T r2 = dx * dx + dy * dy + dz * dz;
                            if (r2 < cker) { const T wp = m * sharpk(r2); wx += wp; sx += wp * sm_v[warp][p - c0][0]; }
                        }
                        if (ay) {
                            const T dx = X - (ti + half), dy = Y - tj, dz = Z - (tk + half);
                            const T r2 = dx * dx + dy * dy + dz * dz;
                            if (r2 < cker) { const T wp = m * sharpk(r2); wy += wp; sy += wp * sm_v[warp][p - c0][1]; }
                        }
                        if (hz && p < sz1) {
                            const T dx = X - (ti + half), dy = Y - (tj + half), dz = Z - tk;
                            const T r2 = dx * dx + dy * dy + dz * dz;
                            if (r2 < cker) { const T wp = m * sharpk(r2); wz += wp; sz += wp * sm_v[warp][p - c0][2]; }
                        }
                    }
                }
            }
        }
        if (hx) { const int f = fxi(g, i, j, k); W.x[f] = wx; u.x[f] = wx > (T)0 ? sx / wx : (T)0; }
        if (hy) { const int f = fyi(g, i, j, k); W.y[f] = wy; u.y[f] = wy > (T)0 ? sy / wy : (T)0; }
        if (hz) { const int f = fzi(g, i, j, k); W.z[f] = wz; u.z[f] = wz > (T)0 ? sz / wz : (T)0; }
    }
}
// particle records in a step's recorded sorted order: (a xyz, mass or 0) and
// (b xyz, 0), so the face gathers read contiguous records within a cell
template <class T>
__global__ void k_ad_slot_gather(int np, const uint32_t* __restrict__ order, const T* __restrict__ a,
                                 const T* __restrict__ b, const float* __restrict__ mass, T* __restrict__ oa,
                                 T* __restrict__ ob) {
    MP_GRID_LOOP(s, np) {
        const uint32_t p = order[s];
        oa[4 * (size_t)s] = a[3 * p]; oa[4 * (size_t)s + 1] = a[3 * p + 1]; oa[4 * (size_t)s + 2] = a[3 * p + 2];
        oa[4 * (size_t)s + 3] = mass ? (T)mass[p] : (T)0;
        ob[4 * (size_t)s] = b[3 * p]; ob[4 * (size_t)s + 1] = b[3 * p + 1]; ob[4 * (size_t)s + 2] = b[3 * p + 2];
        ob[4 * (size_t)s + 3] = (T)0;
    }
}
// per-slot records (b xyz, 0) of one phase's particles, zero for the other's
template <class T>
__global__ void k_ad_slot_gather_ph(int np, const uint32_t* __restrict__ order, const T* __restrict__ b,
                                    const uint8_t* __restrict__ phase, int want, T* __restrict__ ob) {
    MP_GRID_LOOP(s, np) {
        const uint32_t p = order[s];
        const bool on = phase[p] == want;
        ob[4 * (size_t)s] = on ? b[3 * p] : (T)0; ob[4 * (size_t)s + 1] = on ? b[3 * p + 1] : (T)0;
        ob[4 * (size_t)s + 2] = on ? b[3 * p + 2] : (T)0; ob[4 * (size_t)s + 3] = (T)0;
    }
}
template <class T> __global__ void k_ad_copy(long long n, const T* __restrict__ a, T* __restrict__ b) {
    MP_GRID_LOOP(t, n) b[t] = a[t];
}
template <class T> __global__ void k_ad_sub(long long n, const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ o) {
    MP_GRID_LOOP(t, n) o[t] = a[t] - b[t];
}
template <class T> __global__ void k_ad_axpy(long long n, T s, const T* __restrict__ a, T* __restrict__ o) {
    MP_GRID_LOOP(t, n) o[t] += s * a[t];
}

// The octant an extrapolation pass picks for a face and its three weights
// (sweepu_k_bubble: the last octant of the loop whose weights are all
// non-negative). Returns false when the face keeps its value.
__device__ bool sweep_sel(const Grid& g, int ax, int i, int j, int k, const float* __restrict__ ls,
                          const int8_t* __restrict__ mark, int fl, int& sdi, int& sdj, int& sdk, float& swx,
                          float& swy, float& swz) {
    int n_ax = ax == 0 ? g.NX : (ax == 1 ? g.NY : g.NZ);
    int e = ax == 0 ? i : (ax == 1 ? j : k);
    if (!(e > 1 && e < n_ax - 1)) return false;
    int i1 = i - (ax == 0), j1 = j - (ax == 1), k1 = k - (ax == 2);
    if (mark[cid(g, i, j, k)] == fl || mark[cid(g, i1, j1, k1)] == fl) return false;
    float l0 = ls[cid(g, i, j, k)], l1 = ls[cid(g, i1, j1, k1)];
    bool found = false;
    for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2) {
        float wx, wy, wz;
        if (ax == 0) {
            if (j + dj < 0 || j + dj > g.NY - 1 || k + dk < 0 || k + dk > g.NZ - 1) continue;
            wx = (float)(-di) * (l0 - l1);
            if (wx < 0) continue;
            wy = (l0 + l1 - ls[cid(g, i, j + dj, k)] - ls[cid(g, i - 1, j + dj, k)]) * 0.5f;
            if (wy < 0) continue;
            wz = (l0 + l1 - ls[cid(g, i, j, k + dk)] - ls[cid(g, i - 1, j, k + dk)]) * 0.5f;
            if (wz < 0) continue;
        } else if (ax == 1) {
            if (i + di < 0 || i + di > g.NX - 1 || k + dk < 0 || k + dk > g.NZ - 1) continue;
            wy = (float)(-dj) * (l0 - l1);
            if (wy < 0) continue;
            wx = (l0 + l1 - ls[cid(g, i + di, j, k)] - ls[cid(g, i + di, j - 1, k)]) * 0.5f;
            if (wx < 0) continue;
            wz = (l0 + l1 - ls[cid(g, i, j, k + dk)] - ls[cid(g, i, j - 1, k + dk)]) * 0.5f;
            if (wz < 0) continue;
        } else {
            if (i + di < 0 || i + di > g.NX - 1 || j + dj < 0 || j + dj > g.NY - 1) continue;
            wz = (float)(-dk) * (l0 - l1);
            if (wz < 0) continue;
            wy = (l0 + l1 - ls[cid(g, i, j + dj, k)] - ls[cid(g, i, j + dj, k - 1)]) * 0.5f;
            if (wy < 0) continue;
            wx = (l0 + l1 - ls[cid(g, i + di, j, k)] - ls[cid(g, i + di, j, k - 1)]) * 0.5f;
            if (wx < 0) continue;
        }
        float ws = wx + wy + wz;
        if (ws == 0) wx = wy = wz = 1.0f / 3;
        else { wx /= ws; wy /= ws; wz /= ws; }
        sdi = di; sdj = dj; sdk = dk; swx = wx; swy = wy; swz = wz;
        found = true;
    }
    return found;
}
// each face's extrapolation choice for one step, computed once and shared by
// the forward passes and their transposes: bit 7 set when the pass overwrites
// the face, bits 0-2 the chosen octant's signs (di, dj, dk > 0), and the three
// normalised weights
__global__ void k_ad_sweep_sel(Grid g, const float* __restrict__ ls, const int8_t* __restrict__ mark, int fl,
                               uint8_t* __restrict__ sel, float* __restrict__ sw) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        int di, dj, dk; float wx = 0, wy = 0, wz = 0;
        uint8_t code = 0;
        if (sweep_sel(g, ax, i, j, k, ls, mark, fl, di, dj, dk, wx, wy, wz))
            code = (uint8_t)(0x80 | (di > 0 ? 1 : 0) | (dj > 0 ? 2 : 0) | (dk > 0 ? 4 : 0));
        sel[t] = code;
        sw[3 * t] = wx; sw[3 * t + 1] = wy; sw[3 * t + 2] = wz;
    }
}
__device__ __forceinline__ long long face_flat(const Grid& g, int ax, int i, int j, int k) {
    return ax == 0 ? (long long)fxi(g, i, j, k)
                   : (ax == 1 ? (long long)g.nfx + fyi(g, i, j, k) : (long long)g.nfx + g.nfy + fzi(g, i, j, k));
}
// one extrapolation pass (sweepu_k_bubble's arithmetic) from the stored choices
template <class T>
__global__ void k_ad_sweepu_s(Grid g, Fc<T> in, Fc<T> out, const uint8_t* __restrict__ sel, const float* __restrict__ sw) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        const T* f = fsel(in, ax);
        T res = f[idx];
        const uint8_t code = sel[t];
        if (code & 0x80) {
            const int di = code & 1 ? 1 : -1, dj = code & 2 ? 1 : -1, dk = code & 4 ? 1 : -1;
            res = (T)sw[3 * t] * f[face_index(g, ax, i + di, j, k)] + (T)sw[3 * t + 1] * f[face_index(g, ax, i, j + dj, k)] +
                  (T)sw[3 * t + 2] * f[face_index(g, ax, i, j, k + dk)];
        }
        fsel(out, ax)[idx] = res;
    }
}
// its transpose: an input face keeps its own adjoint unless the pass
// overwrote it, and receives from the (up to six) faces whose chosen octant
// reads it
template <class T>
__global__ void k_ad_sweepu_adj_s(Grid g, Fc<T> ob, Fc<T> ib, const uint8_t* __restrict__ sel,
                                  const float* __restrict__ sw) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        const T* o = fsel(ob, ax);
        T acc = (sel[t] & 0x80) ? (T)0 : o[idx];
        const int W = ax == 0 ? g.NX + 1 : g.NX, H = ax == 1 ? g.NY + 1 : g.NY, D = ax == 2 ? g.NZ + 1 : g.NZ;
        for (int dir = 0; dir < 3; dir++) for (int d = -1; d <= 1; d += 2) {
            int fi = i - (dir == 0 ? d : 0), fj = j - (dir == 1 ? d : 0), fk = k - (dir == 2 ? d : 0);
            if (fi < 0 || fi >= W || fj < 0 || fj >= H || fk < 0 || fk >= D) continue;
            const long long ft = face_flat(g, ax, fi, fj, fk);
            const uint8_t code = sel[ft];
            if (!(code & 0x80)) continue;
            const int chosen = (code >> dir) & 1 ? 1 : -1;
            if (chosen != d) continue;
            acc += (T)sw[3 * ft + dir] * o[face_index(g, ax, fi, fj, fk)];
        }
        fsel(ib, ax)[idx] = acc;
    }
}
// raises *flag when some particle's cell from its replay position differs from
// its recorded cell (the G2P transposes then search a wider window), and with
// `cellbad` marks the recorded cell of each such particle
template <class T>
__global__ void k_ad_cell_mismatch(Grid g, int np, const T* __restrict__ x, const uint32_t* __restrict__ cellof,
                                   uint32_t* flag, uint8_t* __restrict__ cellbad) {
    MP_GRID_LOOP(p, np) {
        int a, b, c; getijk3((int)cellof[p], g.NY, g.NZ, a, b, c);
        const T X = x[3 * p] / (T)g.h, Y = x[3 * p + 1] / (T)g.h, Z = x[3 * p + 2] / (T)g.h;
        bool bad = !(X >= (T)0 && Y >= (T)0 && Z >= (T)0) || (int)X != a || (int)Y != b || (int)Z != c;
        if (bad && cellbad) cellbad[cellof[p]] = 1;   // every writer stores 1
        if (__any_sync(__activemask(), bad) && (threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1))
            atomicOr(flag, 1u);
    }
}
// near[c]: some cell of c's 3x3x3 neighbourhood holds a particle whose replay
// cell is not its recorded one
__global__ void k_ad_dilate(Grid g, const uint8_t* __restrict__ bad, uint8_t* __restrict__ near) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        uint8_t v = 0;
        for (int a = max(i - 1, 0); a <= min(i + 1, g.NX - 1); a++)
            for (int b = max(j - 1, 0); b <= min(j + 1, g.NY - 1); b++)
                for (int cc = max(k - 1, 0); cc <= min(k + 1, g.NZ - 1); cc++) v |= bad[cid(g, a, b, cc)];
        near[idx] = v;
    }
}
// wall rules (setWaterBoundaryU_k), in place; `zceil` marks the top z faces
// that took the face below
__device__ __forceinline__ bool bmis(const Grid& g, const int8_t* mark, int i, int j, int k, int i1, int j1, int k1) {
    return (mark[cid(g, i, j, k)] == MP_TYPEBOUNDARY) != (mark[cid(g, i1, j1, k1)] == MP_TYPEBOUNDARY);
}
// 0: keep, 1: zero, 2: z ceiling rule (takes min(below, 0) of the face below)
__device__ __forceinline__ int bound_rule(const Grid& g, const int8_t* mark, int ax, int i, int j, int k) {
    if (ax == 0) {
        if (i <= 1 || i >= g.NX + 1 - 2) return 1;
        if (i > 1 && i < g.NX - 1 && bmis(g, mark, i, j, k, i - 1, j, k)) return 1;
    } else if (ax == 1) {
        if (j <= 1 || j >= g.NY + 1 - 2) return 1;
        if (j > 0 && j < g.NY && bmis(g, mark, i, j, k, i, j - 1, k)) return 1;
    } else {
        if (k <= 1 || k >= g.NZ + 1 - 1) return 1;
        if (k == g.NZ + 1 - 2) return 2;
        if (k > 0 && k < g.NZ && bmis(g, mark, i, j, k, i, j, k - 1)) return 1;
    }
    return 0;
}
// whether the face below a ceiling face passes its value to the rule
__device__ __forceinline__ bool zrule_pass(const Grid& g, const int8_t* mark, int i, int j, int kb) {
    if (kb <= 1) return false;
    if (kb > 0 && kb < g.NZ && bmis(g, mark, i, j, kb, i, j, kb - 1)) return false;
    return true;
}
template <class T>
__global__ void k_ad_bound(Grid g, Fc<T> u, Fc<T> uo, const int8_t* __restrict__ mark) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        const int r = bound_rule(g, mark, ax, i, j, k);
        T v = fsel(u, ax)[idx];
        if (r == 1) v = (T)0;
        else if (r == 2) {
            T below = zrule_pass(g, mark, i, j, k - 1) ? u.z[fzi(g, i, j, k - 1)] : (T)0;
            v = below < (T)0 ? below : (T)0;
        }
        fsel(uo, ax)[idx] = v;
    }
}
// transpose; `u` is the rule's input field (its value decides the ceiling rule)
template <class T>
__global__ void k_ad_bound_adj(Grid g, Fc<T> ob, Fc<T> ib, Fc<T> u, const int8_t* __restrict__ mark) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        const int r = bound_rule(g, mark, ax, i, j, k);
        T acc = r == 0 ? fsel(ob, ax)[idx] : (T)0;
        if (ax == 2 && k + 1 == g.NZ + 1 - 2 && bound_rule(g, mark, 2, i, j, k + 1) == 2 &&
            zrule_pass(g, mark, i, j, k) && u.z[idx] < (T)0)
            acc += ob.z[fzi(g, i, j, k + 1)];
        fsel(ib, ax)[idx] = acc;
    }
}
__device__ __forceinline__ bool unknown(const Grid& g, const int8_t* mark, int idx, int i, int j, int k) {
    int m = mark[idx];
    return (m == MP_TYPEFLUID || m == MP_TYPEAIR) && i > 0 && i < g.NX - 1 && j > 0 && j < g.NY - 1 && k > 0 &&
           k < g.NZ - 1;
}
template <class T>
__global__ void k_ad_div(Grid g, const int8_t* __restrict__ mark, Fc<T> u, T* __restrict__ b) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        T out = 0;
        if (unknown(g, mark, idx, i, j, k))
            out = (u.x[fxi(g, i + 1, j, k)] - u.x[fxi(g, i, j, k)] + u.y[fyi(g, i, j + 1, k)] - u.y[fyi(g, i, j, k)] +
                   u.z[fzi(g, i, j, k + 1)] - u.z[fzi(g, i, j, k)]) / (T)g.h;
        b[idx] = out;
    }
}
template <class T>
__global__ void k_ad_subgrad(Grid g, const T* __restrict__ p, Fc<T> u, Fc<T> uo) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    const T hh = (T)g.h;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        T v = fsel(u, ax)[idx];
        int e = ax == 0 ? i : (ax == 1 ? j : k), n = ax == 0 ? g.NX : (ax == 1 ? g.NY : g.NZ);
        if (e > 0 && e < n) {
            T d = (p[cid(g, i, j, k)] - p[cid(g, i - (ax == 0), j - (ax == 1), k - (ax == 2))]) / hh;
            v = v - d;
        }
        fsel(uo, ax)[idx] = v;
    }
}
// pbar = -G^T ubar on the unknown cells
template <class T>
__global__ void k_ad_pbar(Grid g, const int8_t* __restrict__ mark, Fc<T> ub, T* __restrict__ pb) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        T out = 0;
        if (unknown(g, mark, idx, i, j, k))
            out = (ub.x[fxi(g, i + 1, j, k)] - ub.x[fxi(g, i, j, k)] + ub.y[fyi(g, i, j + 1, k)] - ub.y[fyi(g, i, j, k)] +
                   ub.z[fzi(g, i, j, k + 1)] - ub.z[fzi(g, i, j, k)]) / (T)g.h;
        pb[idx] = out;
    }
}
// ub_out = ub_in + D^T q (q is zero off the unknowns)
template <class T>
__global__ void k_ad_divT(Grid g, const T* __restrict__ q, Fc<T> ubi, Fc<T> ubo) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        int e = ax == 0 ? i : (ax == 1 ? j : k), n = ax == 0 ? g.NX : (ax == 1 ? g.NY : g.NZ);
        T acc = fsel(ubi, ax)[idx];
        T lo = e > 0 ? q[cid(g, i - (ax == 0), j - (ax == 1), k - (ax == 2))] : (T)0;
        T hi = e < n ? q[cid(g, i, j, k)] : (T)0;
        acc += (lo - hi) / (T)g.h;
        fsel(ubo, ax)[idx] = acc;
    }
}
// The two-phase divergence (cptdivergence_bubble2, spray_k.cu:3138-3263): an
// unknown cell of type m reads across each face the value of its own phase,
// or, where the neighbour is of the other phase, the blend with theta =
// -l_c / (l_n - l_c) of the merged level set: theta of its own phase's face
// velocity and 1 - theta of the other's. blend_coef gives the weights (cw, ca)
// of the water and air velocities of the face.
template <class T>
__device__ __forceinline__ void blend_coef(int m, int mn, T lc, T ln, T& cw, T& ca) {
    if (m == MP_TYPEFLUID && mn != MP_TYPEAIR) { cw = (T)1; ca = (T)0; return; }
    if (m == MP_TYPEAIR && mn != MP_TYPEFLUID) { cw = (T)0; ca = (T)1; return; }
    const T th = ((T)0 - lc) / (ln - lc);
    if (m == MP_TYPEFLUID) { cw = th; ca = (T)1 - th; }
    else { cw = (T)1 - th; ca = th; }
}
template <class T>
__device__ __forceinline__ T blend_face(const Grid& g, const int8_t* mark, const float* ls, int m, T lc, int q, T wv,
                                        T av) {
    const int mn = mark[q];
    if (m == MP_TYPEFLUID && mn != MP_TYPEAIR) return wv;
    if (m == MP_TYPEAIR && mn != MP_TYPEFLUID) return av;
    const T th = ((T)0 - lc) / ((T)ls[q] - lc);
    if (m == MP_TYPEFLUID) return th * wv + ((T)1 - th) * av;
    return th * av + ((T)1 - th) * wv;
}
template <class T>
__global__ void k_ad_div2(Grid g, const int8_t* __restrict__ mark, const float* __restrict__ ls, Fc<T> uw, Fc<T> ua,
                          T* __restrict__ b) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        T out = 0;
        if (unknown(g, mark, idx, i, j, k)) {
            const int m = mark[idx];
            const T lc = (T)ls[idx];
            int f;
            f = fxi(g, i + 1, j, k); T x1 = blend_face<T>(g, mark, ls, m, lc, cid(g, i + 1, j, k), uw.x[f], ua.x[f]);
            f = fxi(g, i, j, k);     T x0 = blend_face<T>(g, mark, ls, m, lc, cid(g, i - 1, j, k), uw.x[f], ua.x[f]);
            f = fyi(g, i, j + 1, k); T y1 = blend_face<T>(g, mark, ls, m, lc, cid(g, i, j + 1, k), uw.y[f], ua.y[f]);
            f = fyi(g, i, j, k);     T y0 = blend_face<T>(g, mark, ls, m, lc, cid(g, i, j - 1, k), uw.y[f], ua.y[f]);
            f = fzi(g, i, j, k + 1); T z1 = blend_face<T>(g, mark, ls, m, lc, cid(g, i, j, k + 1), uw.z[f], ua.z[f]);
            f = fzi(g, i, j, k);     T z0 = blend_face<T>(g, mark, ls, m, lc, cid(g, i, j, k - 1), uw.z[f], ua.z[f]);
            out = (x1 - x0 + y1 - y0 + z1 - z0) / (T)g.h;
        }
        b[idx] = out;
    }
}
// pbar = -G^T (ub_w + ub_a) on the unknown cells: both face fields take the
// same pressure gradient
template <class T>
__global__ void k_ad_pbar2(Grid g, const int8_t* __restrict__ mark, Fc<T> uw, Fc<T> ua, T* __restrict__ pb) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        T out = 0;
        if (unknown(g, mark, idx, i, j, k)) {
            const int x1 = fxi(g, i + 1, j, k), x0 = fxi(g, i, j, k), y1 = fyi(g, i, j + 1, k), y0 = fyi(g, i, j, k);
            const int z1 = fzi(g, i, j, k + 1), z0 = fzi(g, i, j, k);
            out = ((uw.x[x1] + ua.x[x1]) - (uw.x[x0] + ua.x[x0]) + (uw.y[y1] + ua.y[y1]) - (uw.y[y0] + ua.y[y0]) +
                   (uw.z[z1] + ua.z[z1]) - (uw.z[z0] + ua.z[z0])) / (T)g.h;
        }
        pb[idx] = out;
    }
}
// the two-phase divergence's transpose: (ubw, uba)_out = (ubw, uba)_in + D^T q.
// A face is the upper face of the cell below it (+1/h there) and the lower
// face of the cell above it (-1/h), each weighted by that cell's blend
// weights toward the other
template <class T>
__global__ void k_ad_divT2(Grid g, const int8_t* __restrict__ mark, const float* __restrict__ ls,
                           const T* __restrict__ q, Fc<T> wi, Fc<T> ai, Fc<T> wo, Fc<T> ao) {
    const long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx; const int ax = face_decode(g, t, i, j, k, idx);
        int e = ax == 0 ? i : (ax == 1 ? j : k), n = ax == 0 ? g.NX : (ax == 1 ? g.NY : g.NZ);
        T aw = fsel(wi, ax)[idx], aa = fsel(ai, ax)[idx];
        const int lo_i = i - (ax == 0), lo_j = j - (ax == 1), lo_k = k - (ax == 2);
        T sw = 0, sa = 0;
        if (e > 0) {
            const int c = cid(g, lo_i, lo_j, lo_k);
            if (unknown(g, mark, c, lo_i, lo_j, lo_k) && e < n) {
                T cw, ca; blend_coef<T>(mark[c], mark[cid(g, i, j, k)], (T)ls[c], (T)ls[cid(g, i, j, k)], cw, ca);
                sw += cw * q[c]; sa += ca * q[c];
            }
        }
        if (e < n) {
            const int c = cid(g, i, j, k);
            if (unknown(g, mark, c, i, j, k) && e > 0) {
                T cw, ca; blend_coef<T>(mark[c], mark[cid(g, lo_i, lo_j, lo_k)], (T)ls[c], (T)ls[cid(g, lo_i, lo_j, lo_k)],
                                        cw, ca);
                sw -= cw * q[c]; sa -= ca * q[c];
            }
        }
        fsel(wo, ax)[idx] = aw + sw / (T)g.h;
        fsel(ao, ax)[idx] = aa + sa / (T)g.h;
    }
}
// trilinear of the face/cell grids (the engine's trilinear) with its gradient
// in grid units
template <class T>
__device__ __forceinline__ T tri(const T* u, T x, T y, T z, int w, int hh, int d, T* gx, T* gy, T* gz) {
    x = x < (T)0 ? (T)0 : (x > (T)w ? (T)w : x);
    y = y < (T)0 ? (T)0 : (y > (T)hh ? (T)hh : y);
    z = z < (T)0 ? (T)0 : (z > (T)d ? (T)d : z);
    int i = (int)(x < (T)(w - 2) ? x : (T)(w - 2));
    int j = (int)(y < (T)(hh - 2) ? y : (T)(hh - 2));
    int k = (int)(z < (T)(d - 2) ? z : (T)(d - 2));
    int b = i * hh * d + j * d + k, sj = d, si = hh * d;
    T u000 = u[b], u100 = u[b + si], u010 = u[b + sj], u110 = u[b + si + sj];
    T u001 = u[b + 1], u101 = u[b + si + 1], u011 = u[b + sj + 1], u111 = u[b + si + sj + 1];
    T fi1 = (T)(i + 1) - x, fi0 = x - (T)i, fj1 = (T)(j + 1) - y, fj0 = y - (T)j, fk1 = (T)(k + 1) - z, fk0 = z - (T)k;
    T a0 = fj1 * (fi1 * u000 + fi0 * u100) + fj0 * (fi1 * u010 + fi0 * u110);
    T a1 = fj1 * (fi1 * u001 + fi0 * u101) + fj0 * (fi1 * u011 + fi0 * u111);
    if (gx) {
        *gx = fk1 * (fj1 * (u100 - u000) + fj0 * (u110 - u010)) + fk0 * (fj1 * (u101 - u001) + fj0 * (u111 - u011));
        *gy = fk1 * ((fi1 * u010 + fi0 * u110) - (fi1 * u000 + fi0 * u100)) +
              fk0 * ((fi1 * u011 + fi0 * u111) - (fi1 * u001 + fi0 * u101));
        *gz = a1 - a0;
    }
    return fk1 * a0 + fk0 * a1;
}
// the interpolation point of a particle for face axis `ax` (grid units)
template <class T> __device__ __forceinline__ void ipos(int ax, T X, T Y, T Z, T& x, T& y, T& z) {
    x = ax == 0 ? X : X - (T)0.5f; y = ax == 1 ? Y : Y - (T)0.5f; z = ax == 2 ? Z : Z - (T)0.5f;
}
// mapvelg2p_flip_bubble: each particle reads its own phase's fields (with
// `phase` null every particle is FLUID)
template <class T>
__global__ void k_ad_g2p(Grid g, int np, const T* __restrict__ x, const T* __restrict__ va, Fc<T> ufw, Fc<T> duw,
                         T alpha, T* __restrict__ vg, const uint8_t* __restrict__ phase, Fc<T> ufa, Fc<T> dua) {
    MP_GRID_LOOP(p, np) {
        T X = x[3 * p] / (T)g.h, Y = x[3 * p + 1] / (T)g.h, Z = x[3 * p + 2] / (T)g.h;
        const bool air = phase && phase[p];
        const Fc<T> uf = air ? ufa : ufw, du = air ? dua : duw;
        for (int ax = 0; ax < 3; ax++) {
            const int w = ax == 0 ? g.NX + 1 : g.NX, hh = ax == 1 ? g.NY + 1 : g.NY, d = ax == 2 ? g.NZ + 1 : g.NZ;
            T a, b, c; ipos(ax, X, Y, Z, a, b, c);
            T gv = tri<T>(fsel(du, ax), a, b, c, w, hh, d, nullptr, nullptr, nullptr);
            T iv = va[3 * p + ax];
            if (alpha == (T)1) iv = iv + gv;
            else {
                T ug = tri<T>(fsel(uf, ax), a, b, c, w, hh, d, nullptr, nullptr, nullptr);
                iv = ((T)1 - alpha) * ug + alpha * (iv + gv);
            }
            vg[3 * p + ax] = iv;
        }
    }
}
template <class T>
__global__ void k_ad_advect(Grid g, int np, const T* __restrict__ x, const T* __restrict__ vg, T* __restrict__ xo,
                            T* __restrict__ vo, T dt) {
    const T h = (T)g.h;
    MP_GRID_LOOP(p, np) {
        for (int a = 0; a < 3; a++) {
            const int n = a == 0 ? g.NX : (a == 1 ? g.NY : g.NZ);
            const T lo = (T)0 + (h + (T)0.5f * h), hi = (T)n * h - (h + (T)0.5f * h);
            T ip = x[3 * p + a] + vg[3 * p + a] * dt, iv = vg[3 * p + a];
            if (ip <= lo) { ip = lo; iv = (T)0; }
            if (ip >= hi) { ip = hi; iv = (T)0; }
            xo[3 * p + a] = ip; vo[3 * p + a] = iv;
        }
    }
}

// ---- loss ------------------------------------------------------------------------
template <class T>
__global__ void k_ad_phi(Grid g, const T* __restrict__ x, const uint32_t* __restrict__ nearest, T* __restrict__ phi) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        const T h = (T)g.h, cap = (T)2.5f * h;
        T d = cap;
        uint32_t p = nearest[idx];
        if (p != NONE) {
            T dx = x[3 * p] - ((T)i + (T)0.5f) * h, dy = x[3 * p + 1] - ((T)j + (T)0.5f) * h, dz = x[3 * p + 2] - ((T)k + (T)0.5f) * h;
            T dd = sqrt(dx * dx + dy * dy + dz * dz);
            d = dd < cap ? dd : cap;
        }
        phi[idx] = d - (T)0.5f * h;
    }
}
// loss = sum_s phi(y_s)^2 in FP64, one block in a fixed order; also keeps phi(y_s)
template <class T>
__global__ void k_ad_loss(Grid g, int ns, const float* __restrict__ sp, const T* __restrict__ phi, double* __restrict__ sv,
                          double* __restrict__ loss) {
    __shared__ double part[256];
    double acc = 0;
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        T X = (T)sp[3 * s] / (T)g.h - (T)0.5f, Y = (T)sp[3 * s + 1] / (T)g.h - (T)0.5f, Z = (T)sp[3 * s + 2] / (T)g.h - (T)0.5f;
        T v = tri<T>(phi, X, Y, Z, g.NX, g.NY, g.NZ, nullptr, nullptr, nullptr);
        sv[s] = (double)v;
        acc += (double)v * (double)v;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int q = 0; q < (int)blockDim.x; q++) t += part[q];
        *loss = t;
    }
}
// the sample's base cell of the cell-centred trilinear
__host__ __device__ inline void sample_base(float h, int NX, int NY, int NZ, float px, float py, float pz, int& i,
                                            int& j, int& k) {
    float x = px / h - 0.5f, y = py / h - 0.5f, z = pz / h - 0.5f;
    x = x < 0 ? 0 : (x > NX ? NX : x); y = y < 0 ? 0 : (y > NY ? NY : y); z = z < 0 ? 0 : (z > NZ ? NZ : z);
    i = (int)(x < NX - 2 ? x : NX - 2); j = (int)(y < NY - 2 ? y : NY - 2); k = (int)(z < NZ - 2 ? z : NZ - 2);
}
// phibar_c = sum over samples whose stencil holds c of 2 phi(y_s) w_sc
template <class T>
__global__ void k_ad_phibar(Grid g, const float* __restrict__ sp, const uint32_t* __restrict__ soff,
                            const double* __restrict__ sv, T* __restrict__ pb) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        T acc = 0;
        for (int a = 0; a <= 1; a++) for (int b = 0; b <= 1; b++) for (int c = 0; c <= 1; c++) {
            int bi = i - a, bj = j - b, bk = k - c;
            if (bi < 0 || bj < 0 || bk < 0) continue;
            int base = cid(g, bi, bj, bk);
            for (uint32_t s = soff[base]; s < soff[base + 1]; s++) {
                T X = (T)sp[3 * s] / (T)g.h - (T)0.5f, Y = (T)sp[3 * s + 1] / (T)g.h - (T)0.5f, Z = (T)sp[3 * s + 2] / (T)g.h - (T)0.5f;
                X = X < (T)0 ? (T)0 : (X > (T)g.NX ? (T)g.NX : X);
                Y = Y < (T)0 ? (T)0 : (Y > (T)g.NY ? (T)g.NY : Y);
                Z = Z < (T)0 ? (T)0 : (Z > (T)g.NZ ? (T)g.NZ : Z);
                T fx = a ? X - (T)bi : (T)(bi + 1) - X, fy = b ? Y - (T)bj : (T)(bj + 1) - Y, fz = c ? Z - (T)bk : (T)(bk + 1) - Z;
                acc += (T)2 * (T)sv[s] * fx * fy * fz;
            }
        }
        pb[idx] = acc;
    }
}
// xbar of each particle from the cells it is nearest to (+-3 cell box)
template <class T>
__global__ void k_ad_phi_x(Grid g, int np, const T* __restrict__ x, const uint32_t* __restrict__ nearest,
                           const T* __restrict__ pb, T* __restrict__ xb) {
    MP_GRID_LOOP(p, np) {
        const T h = (T)g.h, cap = (T)2.5f * h;
        int ci = (int)(x[3 * p] / h), cj = (int)(x[3 * p + 1] / h), ck = (int)(x[3 * p + 2] / h);
        T gx = 0, gy = 0, gz = 0;
        for (int di = -3; di <= 3; di++) for (int dj = -3; dj <= 3; dj++) for (int dk = -3; dk <= 3; dk++) {
            int a = ci + di, b = cj + dj, c = ck + dk;
            if (a < 0 || a >= g.NX || b < 0 || b >= g.NY || c < 0 || c >= g.NZ) continue;
            int idx = cid(g, a, b, c);
            if (nearest[idx] != (uint32_t)p) continue;
            T dx = x[3 * p] - ((T)a + (T)0.5f) * h, dy = x[3 * p + 1] - ((T)b + (T)0.5f) * h, dz = x[3 * p + 2] - ((T)c + (T)0.5f) * h;
            T dd = sqrt(dx * dx + dy * dy + dz * dz);
            if (!(dd < cap) || dd == (T)0) continue;
            T s = pb[idx] / dd;
            gx += s * dx; gy += s * dy; gz += s * dz;
        }
        xb[3 * p] = gx; xb[3 * p + 1] = gy; xb[3 * p + 2] = gz;
    }
}

// ---- transposes of the particle stages -------------------------------------------
// advection with the clamp: a clamped component passes nothing back
template <class T>
__global__ void k_ad_advect_adj(Grid g, int np, const T* __restrict__ x, const T* __restrict__ vg, T dt,
                                T* __restrict__ xb, const T* __restrict__ vb, T* __restrict__ vgb) {
    const T h = (T)g.h;
    MP_GRID_LOOP(p, np) {
        for (int a = 0; a < 3; a++) {
            const int n = a == 0 ? g.NX : (a == 1 ? g.NY : g.NZ);
            const T lo = (T)0 + (h + (T)0.5f * h), hi = (T)n * h - (h + (T)0.5f * h);
            T ip = x[3 * p + a] + vg[3 * p + a] * dt;
            bool clamped = false;
            if (ip <= lo) { ip = lo; clamped = true; }
            if (ip >= hi) { ip = hi; clamped = true; }
            T xin = xb[3 * p + a];
            if (clamped) { xb[3 * p + a] = (T)0; vgb[3 * p + a] = (T)0; }
            else { vgb[3 * p + a] = vb[3 * p + a] + dt * xin; }
        }
    }
}
// gather part of the particle side of the G2P transpose: vabar and the
// position derivative of the interpolation
template <class T>
__global__ void k_ad_g2p_adj_p(Grid g, int np, const uint32_t* __restrict__ order, const T* __restrict__ x, Fc<T> ufw,
                               Fc<T> duw, T alpha, const T* __restrict__ vgb, T* __restrict__ vab, T* __restrict__ xb,
                               const uint8_t* __restrict__ phase, Fc<T> ufa, Fc<T> dua) {
    // particles in sorted order, so neighbouring threads read neighbouring faces
    MP_GRID_LOOP(sl, np) {
        const uint32_t p = order[sl];
        const bool air = phase && phase[p];
        const Fc<T> uf = air ? ufa : ufw, du = air ? dua : duw;
        const T ih = (T)1 / (T)g.h;
        T X = x[3 * p] / (T)g.h, Y = x[3 * p + 1] / (T)g.h, Z = x[3 * p + 2] / (T)g.h;
        const T cdu = alpha == (T)1 ? (T)1 : alpha, cu = alpha == (T)1 ? (T)0 : (T)1 - alpha;
        T gxs = 0, gys = 0, gzs = 0;
        for (int ax = 0; ax < 3; ax++) {
            const int w = ax == 0 ? g.NX + 1 : g.NX, hh = ax == 1 ? g.NY + 1 : g.NY, d = ax == 2 ? g.NZ + 1 : g.NZ;
            T a, b, c; ipos(ax, X, Y, Z, a, b, c);
            T vb = vgb[3 * p + ax];
            T gx1, gy1, gz1, gx2 = 0, gy2 = 0, gz2 = 0;
            tri<T>(fsel(du, ax), a, b, c, w, hh, d, &gx1, &gy1, &gz1);
            if (cu != (T)0) tri<T>(fsel(uf, ax), a, b, c, w, hh, d, &gx2, &gy2, &gz2);
            gxs += vb * (cdu * gx1 + cu * gx2); gys += vb * (cdu * gy1 + cu * gy2); gzs += vb * (cdu * gz1 + cu * gz2);
            vab[3 * p + ax] = cdu * vb;
        }
        xb[3 * p] += gxs * ih; xb[3 * p + 1] += gys * ih; xb[3 * p + 2] += gzs * ih;
    }
}
// face side of the G2P transpose: q_f = sum of w_pf vgbar_p over the particles
// whose interpolation stencil holds f. Those lie in cells [i-1,i] along the
// face normal and [-1,1] across of their replay positions (the water splat's
// window); the candidates come from the recorded cell lists, so a face takes
// them one cell wider (the air splat's window) when near[] is set in the
// 3x3x3 cells around its node, i.e. near a particle whose replay cell is not
// its recorded one. Membership is decided from the replay's own positions, and
// a face adds its members in (a, b, c, particle) order in either window.
// A warp handles 32 nodes along k (i, j fixed), a thread a node's three
// faces, with the candidates of each column (a, b) staged in shared memory
// as in k_ad_p2g_w.
template <class T>
__global__ void __launch_bounds__(256) k_ad_g2p_adj_w(Grid g, const uint32_t* __restrict__ off,
                                                      const T* __restrict__ xs4, const T* __restrict__ vgs4, Fc<T> q,
                                                      const uint8_t* __restrict__ cellmask,
                                                      const uint8_t* __restrict__ near) {
    constexpr int CAP = sizeof(T) == 4 ? 128 : 64;
    __shared__ T sm_x[8][CAP][4];
    __shared__ T sm_v[8][CAP][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Tiles Tl = make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1);
    MP_GRID_LOOP(t, Tl.threads()) {
        int i, j, k;
        const bool act = tile_ijk(Tl, t, i, j, k);
        if (!__any_sync(0xffffffffu, act)) continue;
        const bool hx = act && j < g.NY && k < g.NZ, hy = act && i < g.NX && k < g.NZ, hz = act && i < g.NX && j < g.NY;
        bool wide = near == nullptr;   // no map: every face takes the wider window
        if (act && near)
            for (int a = max(i - 1, 0); a <= min(i + 1, g.NX - 1); a++)
                for (int b = max(j - 1, 0); b <= min(j + 1, g.NY - 1); b++)
                    for (int cc = max(k - 1, 0); cc <= min(k + 1, g.NZ - 1); cc++) wide = wide || near[cid(g, a, b, cc)];
        // this lane's windows: along the normal [-LO, HI], across [-AC, AC]
        const int LO = wide ? 2 : 1, HI = wide ? 1 : 0, AC = wide ? 2 : 1;
        const int R = __reduce_max_sync(0xffffffffu, act ? AC : 1);
        T qx = 0, qy = 0, qz = 0;
        const int klo = max(k - AC, 0), khi = min(k + AC, g.NZ - 1), kzhi = min(k + HI, g.NZ - 1);
        const int W0 = g.NX + 1, H1 = g.NY + 1, D2 = g.NZ + 1;
        for (int di = -R; di <= R; di++) {
            const int a = i + di;
            if (a < 0 || a > g.NX - 1) continue;   // the same for the whole warp
            const bool ax = hx && di >= -LO && di <= HI, inx = di >= -AC && di <= AC;
            for (int dj = -R; dj <= R; dj++) {
                const int b = j + dj;
                if (b < 0 || b > g.NY - 1) continue;
                const bool ay = hy && inx && dj >= -LO && dj <= HI;
                const bool axc = ax && dj >= -AC && dj <= AC;
                const bool azc = hz && inx && dj >= -AC && dj <= AC;
                bool need = (axc || ay || azc) && klo <= khi;
                const int cb = cid(g, a, b, 0);
                if (need && cellmask) {
                    bool any = false;
                    for (int cc = klo; cc <= khi; cc++) any = any || cellmask[cb + cc];
                    need = any;
                }
                if (!__any_sync(0xffffffffu, need)) continue;
                uint32_t s0 = 0, s1 = 0, sz1 = 0;
                if (need) {
                    s0 = off[cb + klo]; s1 = off[cb + khi + 1];
                    sz1 = azc ? off[cb + kzhi + 1] : s0;
                }
                const uint32_t A = __reduce_min_sync(0xffffffffu, need ? s0 : 0xffffffffu);
                const uint32_t B = __reduce_max_sync(0xffffffffu, need ? s1 : 0u);
                for (uint32_t c0 = A; c0 < B; c0 += CAP) {
                    const uint32_t n = min(B - c0, (uint32_t)CAP);
                    __syncwarp();
                    for (uint32_t e = lane; e < n; e += 32) {
                        const T* r = xs4 + 4 * (size_t)(c0 + e);
                        const T* v = vgs4 + 4 * (size_t)(c0 + e);
                        sm_x[warp][e][0] = r[0]; sm_x[warp][e][1] = r[1]; sm_x[warp][e][2] = r[2];
                        sm_v[warp][e][0] = v[0]; sm_v[warp][e][1] = v[1]; sm_v[warp][e][2] = v[2];
                    }
                    __syncwarp();
                    if (!need) continue;
                    const uint32_t lo = max(s0, c0), hi = min(s1, c0 + n);
                    for (uint32_t p = lo; p < hi; ++p) {
                        const T X = sm_x[warp][p - c0][0] / (T)g.h, Y = sm_x[warp][p - c0][1] / (T)g.h;
                        const T Z = sm_x[warp][p - c0][2] / (T)g.h;
                        #pragma unroll
                        for (int f = 0; f < 3; f++) {
                            const bool on = f == 0 ? axc : (f == 1 ? ay : (azc && p < sz1));
                            if (!on) continue;
                            const int w = f == 0 ? W0 : g.NX, hh = f == 1 ? H1 : g.NY, d = f == 2 ? D2 : g.NZ;
                            T px, py, pz; ipos(f, X, Y, Z, px, py, pz);
                            px = px < (T)0 ? (T)0 : (px > (T)w ? (T)w : px);
                            py = py < (T)0 ? (T)0 : (py > (T)hh ? (T)hh : py);
                            pz = pz < (T)0 ? (T)0 : (pz > (T)d ? (T)d : pz);
                            const int bi = (int)(px < (T)(w - 2) ? px : (T)(w - 2));
                            const int bj = (int)(py < (T)(hh - 2) ? py : (T)(hh - 2));
                            const int bk = (int)(pz < (T)(d - 2) ? pz : (T)(d - 2));
                            const int ei = i - bi, ej = j - bj, ek = k - bk;
                            if (ei < 0 || ei > 1 || ej < 0 || ej > 1 || ek < 0 || ek > 1) continue;
                            const T fx = ei ? px - (T)bi : (T)(bi + 1) - px, fy = ej ? py - (T)bj : (T)(bj + 1) - py;
                            const T fz = ek ? pz - (T)bk : (T)(bk + 1) - pz;
                            const T term = fx * fy * fz * sm_v[warp][p - c0][f];
                            if (f == 0) qx += term; else if (f == 1) qy += term; else qz += term;
                        }
                    }
                }
            }
        }
        if (hx) q.x[fxi(g, i, j, k)] = qx;
        if (hy) q.y[fyi(g, i, j, k)] = qy;
        if (hz) q.z[fzi(g, i, j, k)] = qz;
    }
}
// per face ub/W of a splat (0 where the face took no weight): the factor every
// particle of the face's window takes
template <class T>
__global__ void k_ad_ub_over_w(long long nf, const T* __restrict__ ub, const T* __restrict__ W, T* __restrict__ o) {
    MP_GRID_LOOP(t, nf) o[t] = W[t] > (T)0 ? ub[t] / W[t] : (T)0;
}
// splat transpose per particle over the faces whose window holds its cell
// (the particle's cell is the recorded one: window membership is frozen)
template <class T, int PH>
__global__ void k_ad_p2g_adj(Grid g, int np, const uint32_t* __restrict__ order, const T* __restrict__ x,
                             const T* __restrict__ va, const float* __restrict__ mass,
                             const uint32_t* __restrict__ cellof, Fc<T> u, Fc<T> ubw, T* __restrict__ vab,
                             T* __restrict__ xb) {
    const T cker = (T)1.4f * (T)1.4f;
    const T scale = (T)1 / (T)g.h;
    // particles in sorted order, so neighbouring threads read neighbouring faces
    MP_GRID_LOOP(sl, np) {
        const uint32_t p = order[sl];
        T X = x[3 * p] * scale, Y = x[3 * p + 1] * scale, Z = x[3 * p + 2] * scale;
        int ca, cb, cc;
        getijk3((int)cellof[p], g.NY, g.NZ, ca, cb, cc);
        const T m = (T)mass[p];
        if (m == (T)0) continue;   // the other phase's particle: not in this splat
        using Wn = SplatWin<PH>;
        T vb[3] = {0, 0, 0}, gxs = 0, gys = 0, gzs = 0;
        for (int ax = 0; ax < 3; ax++) {
            const int W_ = ax == 0 ? g.NX + 1 : g.NX, H_ = ax == 1 ? g.NY + 1 : g.NY, D_ = ax == 2 ? g.NZ + 1 : g.NZ;
            // a face e whose window along the normal holds cell c, e-LO <= c <= e+HI,
            // lies in [c-HI, c+LO]; across, in [c-AC, c+AC]
            const int fi0 = ca - (ax == 0 ? Wn::HI : Wn::AC), fi1 = ca + (ax == 0 ? Wn::LO : Wn::AC);
            const int j0 = cb - (ax == 1 ? Wn::HI : Wn::AC), j1 = cb + (ax == 1 ? Wn::LO : Wn::AC);
            const int k0 = cc - (ax == 2 ? Wn::HI : Wn::AC), k1 = cc + (ax == 2 ? Wn::LO : Wn::AC);
            const T pv = va[3 * p + ax];
            for (int fi = fi0; fi <= fi1; fi++) {
                if (fi < 0 || fi >= W_) continue;
                for (int fj = j0; fj <= j1; fj++) {
                    if (fj < 0 || fj >= H_) continue;
                    for (int fk = k0; fk <= k1; fk++) {
                        if (fk < 0 || fk >= D_) continue;
                        float gx, gy, gz; face_pos(ax, fi, fj, fk, gx, gy, gz);
                        T dx = X - (T)gx, dy = Y - (T)gy, dz = Z - (T)gz;
                        T r2 = dx * dx + dy * dy + dz * dz;
                        // beyond the kernel radius the weight and its slope are zero
                        if (!(r2 < cker)) continue;
                        const int f = face_index(g, ax, fi, fj, fk);
                        // ub/W of the face (0 where the face took no weight)
                        const T a = fsel(ubw, ax)[f];
                        if (a == (T)0) continue;
                        // the kernel c/r2 - 1 and its slope -c/r2^2 (zero below
                        // the clamp at r2 = 1e-4) from one division
                        T k_, kd;
                        if (r2 > (T)0.0001f) {
                            const T qv = cker / r2;
                            k_ = qv - (T)1; kd = -qv / r2;
                            if (!(k_ > (T)0)) continue;
                        } else {
                            k_ = cker / (T)0.0001f - (T)1; kd = (T)0;
                        }
                        vb[ax] += a * m * k_;
                        const T sv = (pv - fsel(u, ax)[f]) * a * m * kd * (T)2 * scale;
                        gxs += sv * dx; gys += sv * dy; gzs += sv * dz;
                    }
                }
            }
        }
        vab[3 * p] += vb[0]; vab[3 * p + 1] += vb[1]; vab[3 * p + 2] += vb[2];
        xb[3 * p] += gxs; xb[3 * p + 1] += gys; xb[3 * p + 2] += gzs;
    }
}
// ---- heat (updateTemperature for FLUID particles, spray.cu:1889-1947) --------------
// The heat stage after advection: mapHeatp2g_hash (cell temperature = sharp-
// kernel mean of the particle temperatures over the 27 cells, spray_k.cu:
// 4619-4653), the implicit diffusion solve (compb_heat, solver_cg_heat,
// setBoundaryHeat), the change per cell (compTpChange) and mapHeatg2p
// (T_p <- a (T_p + I dT) + (1 - a) I T_new, spray_k.cu:4655-4679), then
// updateLatentHeat_k's clamp of FLUID temperatures to [melting, boiling].
struct HeatCoef {
    float alpha[MP_TYPECNT];
    float dt;
    __device__ __forceinline__ float al(int m) const {
        float a = alpha[0];
        #pragma unroll
        for (int t = 1; t < MP_TYPECNT; t++) a = (m == t) ? alpha[t] : a;
        return a;
    }
};
// sorted-slot records (x, y, z, s) of the positions and one scalar per particle
template <class T>
__global__ void k_ad_slot_gather1(int np, const uint32_t* __restrict__ order, const T* __restrict__ x,
                                  const T* __restrict__ sc, T* __restrict__ o4) {
    MP_GRID_LOOP(s, np) {
        const uint32_t p = order[s];
        o4[4 * (size_t)s] = x[3 * p]; o4[4 * (size_t)s + 1] = x[3 * p + 1]; o4[4 * (size_t)s + 2] = x[3 * p + 2];
        o4[4 * (size_t)s + 3] = sc[p];
    }
}
template <class T>
__global__ void k_ad_heat_p2g(Grid g, const uint32_t* __restrict__ off, const T* __restrict__ xs4, T dflt,
                              T* __restrict__ Tc, T* __restrict__ Wc) {
    const T scale = (T)1 / (T)g.h;
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        const T gx = (T)i + (T)0.5f, gy = (T)j + (T)0.5f, gz = (T)k + (T)0.5f;
        T ws = 0, hs = 0;
        for (int a = i - 1; a <= i + 1; a++) {
            if (a < 0 || a > g.NX - 1) continue;
            for (int b = j - 1; b <= j + 1; b++) {
                if (b < 0 || b > g.NY - 1) continue;
                const int k0 = max(k - 1, 0), k1 = min(k + 1, g.NZ - 1);
                for (uint32_t q = off[cid(g, a, b, k0)]; q < off[cid(g, a, b, k1) + 1]; q++) {
                    const T* r = xs4 + 4 * (size_t)q;
                    const T dx = r[0] * scale - gx, dy = r[1] * scale - gy, dz = r[2] * scale - gz;
                    const T w = sharpk(dx * dx + dy * dy + dz * dz);
                    ws += w; hs += w * r[3];
                }
            }
        }
        Tc[idx] = ws > (T)0 ? hs / ws : dflt;
        Wc[idx] = ws;
    }
}
// right-hand side of the implicit solve: T h^2 / (alpha dt), with the fixed
// temperature where one is set
template <class T>
__global__ void k_ad_heat_rhs(Grid g, const T* __restrict__ Tc, const int8_t* __restrict__ mark,
                              const float* __restrict__ fixedheat, HeatCoef hc, T* __restrict__ b) {
    MP_GRID_LOOP(idx, g.n) {
        T t = Tc[idx];
        if (fixedheat && fixedheat[idx] != MP_UNDEF_TEMPERATURE) t = (T)fixedheat[idx];
        b[idx] = t * (T)g.h * (T)g.h / (T)hc.al(mark[idx]) / (T)hc.dt;
    }
}
// setBoundaryHeat: a shell cell takes its inner neighbour's value (x, then y,
// then z walls first)
__device__ __forceinline__ int heat_src(const Grid& g, int i, int j, int k) {
    if (i == g.NX - 1) return cid(g, i - 1, j, k);
    if (i == 0) return cid(g, i + 1, j, k);
    if (j == g.NY - 1) return cid(g, i, j - 1, k);
    if (j == 0) return cid(g, i, j + 1, k);
    if (k == g.NZ - 1) return cid(g, i, j, k - 1);
    if (k == 0) return cid(g, i, j, k + 1);
    return cid(g, i, j, k);
}
template <class T>
__global__ void k_ad_heat_ext(Grid g, const T* __restrict__ in, T* __restrict__ out) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        out[idx] = in[heat_src(g, i, j, k)];
    }
}
// its transpose as a gather: a cell collects its own cotangent (if it is not
// a shell cell) and those of the shell neighbours that copy from it
template <class T>
__global__ void k_ad_heat_ext_adj(Grid g, const T* __restrict__ ob, T* __restrict__ ib) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        T acc = heat_src(g, i, j, k) == idx ? ob[idx] : (T)0;
        const int nb[6][3] = {{i + 1, j, k}, {i - 1, j, k}, {i, j + 1, k}, {i, j - 1, k}, {i, j, k + 1}, {i, j, k - 1}};
        for (int q = 0; q < 6; q++) {
            const int a = nb[q][0], b = nb[q][1], c = nb[q][2];
            if (a < 0 || a > g.NX - 1 || b < 0 || b > g.NY - 1 || c < 0 || c > g.NZ - 1) continue;
            const int s = cid(g, a, b, c);
            if (s != idx && heat_src(g, a, b, c) == idx) acc += ob[s];
        }
        ib[idx] = acc;
    }
}
template <class T>
__global__ void k_ad_heat_dT(int n, const T* __restrict__ Te, const T* __restrict__ Tc, const int8_t* __restrict__ mark,
                             T* __restrict__ dT) {
    MP_GRID_LOOP(idx, n) dT[idx] = mark[idx] != MP_TYPEBOUNDARY ? Te[idx] - Tc[idx] : (T)0;
}
// mapHeatg2p, then the latent-heat clamp of FLUID temperatures
template <class T>
__global__ void k_ad_heat_g2p(Grid g, int np, const T* __restrict__ x, const T* __restrict__ Tp,
                              const T* __restrict__ dT, const T* __restrict__ Te, T a, T mp, T bp,
                              T* __restrict__ T1, T* __restrict__ T2) {
    MP_GRID_LOOP(p, np) {
        const T X = x[3 * p] / (T)g.h - (T)0.5f, Y = x[3 * p + 1] / (T)g.h - (T)0.5f, Z = x[3 * p + 2] / (T)g.h - (T)0.5f;
        const T id = tri<T>(dT, X, Y, Z, g.NX, g.NY, g.NZ, nullptr, nullptr, nullptr);
        const T it = tri<T>(Te, X, Y, Z, g.NX, g.NY, g.NZ, nullptr, nullptr, nullptr);
        const T t1 = a * (Tp[p] + id) + ((T)1 - a) * it;
        T1[p] = t1;
        T2[p] = t1 < mp ? mp : (t1 > bp ? bp : t1);
    }
}
// particle side of the G2P transpose: the clamp passes nothing back where it
// clamped; Tpb = a T1bar; xbar += T1bar (a grad I dT + (1 - a) grad I Te) / h.
// T1bar is kept in q1 for the cell side.
template <class T>
__global__ void k_ad_heat_g2p_adj_p(Grid g, int np, const T* __restrict__ x, const T* __restrict__ T1,
                                    const T* __restrict__ dT, const T* __restrict__ Te, T a, T mp, T bp,
                                    T* __restrict__ Tb, T* __restrict__ q1, T* __restrict__ xb) {
    MP_GRID_LOOP(p, np) {
        const T t1 = T1[p];
        const T b1 = (t1 < mp || t1 > bp) ? (T)0 : Tb[p];
        q1[p] = b1;
        Tb[p] = a * b1;
        const T X = x[3 * p] / (T)g.h - (T)0.5f, Y = x[3 * p + 1] / (T)g.h - (T)0.5f, Z = x[3 * p + 2] / (T)g.h - (T)0.5f;
        T gx1, gy1, gz1, gx2, gy2, gz2;
        tri<T>(dT, X, Y, Z, g.NX, g.NY, g.NZ, &gx1, &gy1, &gz1);
        tri<T>(Te, X, Y, Z, g.NX, g.NY, g.NZ, &gx2, &gy2, &gz2);
        const T ih = (T)1 / (T)g.h;
        xb[3 * p] += b1 * (a * gx1 + ((T)1 - a) * gx2) * ih;
        xb[3 * p + 1] += b1 * (a * gy1 + ((T)1 - a) * gy2) * ih;
        xb[3 * p + 2] += b1 * (a * gz1 + ((T)1 - a) * gz2) * ih;
    }
}
// cell side: q_c = sum over the particles whose trilinear stencil holds c of
// w_pc T1bar_p (candidates from the recorded cells, one cell wider when some
// replay position left its recorded cell)
template <class T, bool WIDE>
__global__ void k_ad_heat_g2p_adj_c(Grid g, const uint32_t* __restrict__ off, const T* __restrict__ xs4,
                                    T* __restrict__ q) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk3(idx, g.NY, g.NZ, i, j, k);
        const int wd = WIDE ? 2 : 1;
        T acc = 0;
        for (int a = i - wd; a <= i + wd; a++) {
            if (a < 0 || a > g.NX - 1) continue;
            for (int b = j - wd; b <= j + wd; b++) {
                if (b < 0 || b > g.NY - 1) continue;
                const int k0 = max(k - wd, 0), k1 = min(k + wd, g.NZ - 1);
                for (uint32_t s = off[cid(g, a, b, k0)]; s < off[cid(g, a, b, k1) + 1]; s++) {
                    const T* r = xs4 + 4 * (size_t)s;
                    T px = r[0] / (T)g.h - (T)0.5f, py = r[1] / (T)g.h - (T)0.5f, pz = r[2] / (T)g.h - (T)0.5f;
                    px = px < (T)0 ? (T)0 : (px > (T)g.NX ? (T)g.NX : px);
                    py = py < (T)0 ? (T)0 : (py > (T)g.NY ? (T)g.NY : py);
                    pz = pz < (T)0 ? (T)0 : (pz > (T)g.NZ ? (T)g.NZ : pz);
                    const int bi = (int)(px < (T)(g.NX - 2) ? px : (T)(g.NX - 2));
                    const int bj = (int)(py < (T)(g.NY - 2) ? py : (T)(g.NY - 2));
                    const int bk = (int)(pz < (T)(g.NZ - 2) ? pz : (T)(g.NZ - 2));
                    const int ei = i - bi, ej = j - bj, ek = k - bk;
                    if (ei < 0 || ei > 1 || ej < 0 || ej > 1 || ek < 0 || ek > 1) continue;
                    const T fx = ei ? px - (T)bi : (T)(bi + 1) - px, fy = ej ? py - (T)bj : (T)(bj + 1) - py;
                    const T fz = ek ? pz - (T)bk : (T)(bk + 1) - pz;
                    acc += fx * fy * fz * r[3];
                }
            }
        }
        q[idx] = acc;
    }
}
// dT = Te - Tc off the walls: Tebar = (1 - a) q + dTbar, Tcbar = -dTbar
template <class T>
__global__ void k_ad_heat_mix(int n, const int8_t* __restrict__ mark, const T* __restrict__ q, T a, T* __restrict__ Teb,
                              T* __restrict__ Tcb) {
    MP_GRID_LOOP(idx, n) {
        const T dtb = mark[idx] != MP_TYPEBOUNDARY ? a * q[idx] : (T)0;
        Teb[idx] = ((T)1 - a) * q[idx] + dtb;
        Tcb[idx] = -dtb;
    }
}
// Tcbar += bbar h^2 / (alpha dt) where the right-hand side took the cell's
// own temperature (bbar is zero off the solve's unknowns)
template <class T>
__global__ void k_ad_heat_rhs_adj(Grid g, const T* __restrict__ bb, const int8_t* __restrict__ mark,
                                  const float* __restrict__ fixedheat, HeatCoef hc, T* __restrict__ Tcb) {
    MP_GRID_LOOP(idx, g.n) {
        // walls (alpha 0, outside the solve) and held cells pass nothing back
        if (mark[idx] == MP_TYPEBOUNDARY || (fixedheat && fixedheat[idx] != MP_UNDEF_TEMPERATURE)) continue;
        Tcb[idx] += bb[idx] * (T)g.h * (T)g.h / (T)hc.al(mark[idx]) / (T)hc.dt;
    }
}
// mapHeatp2g transpose per particle over the cells whose window holds its
// recorded cell: Tpbar += Tcbar w / W, xbar += Tcbar (T_p - Tc) / W dw/dx
template <class T>
__global__ void k_ad_heat_p2g_adj(Grid g, int np, const T* __restrict__ x, const T* __restrict__ Tp,
                                  const uint32_t* __restrict__ cellof, const T* __restrict__ Tc,
                                  const T* __restrict__ Wc, const T* __restrict__ Tcb, T* __restrict__ Tb,
                                  T* __restrict__ xb) {
    const T scale = (T)1 / (T)g.h;
    MP_GRID_LOOP(p, np) {
        int ca, cb, cc; getijk3((int)cellof[p], g.NY, g.NZ, ca, cb, cc);
        const T X = x[3 * p] * scale, Y = x[3 * p + 1] * scale, Z = x[3 * p + 2] * scale;
        const T tp = Tp[p];
        T tb = 0, gxs = 0, gys = 0, gzs = 0;
        for (int a = ca - 1; a <= ca + 1; a++) {
            if (a < 0 || a > g.NX - 1) continue;
            for (int b = cb - 1; b <= cb + 1; b++) {
                if (b < 0 || b > g.NY - 1) continue;
                for (int c = cc - 1; c <= cc + 1; c++) {
                    if (c < 0 || c > g.NZ - 1) continue;
                    const int idx = cid(g, a, b, c);
                    const T W = Wc[idx];
                    if (!(W > (T)0)) continue;
                    const T dx = X - ((T)a + (T)0.5f), dy = Y - ((T)b + (T)0.5f), dz = Z - ((T)c + (T)0.5f);
                    const T r2 = dx * dx + dy * dy + dz * dz;
                    const T w = sharpk(r2), kd = sharpk_d(r2);
                    const T cb_ = Tcb[idx];
                    tb += cb_ * w / W;
                    const T sgr = cb_ * (tp - Tc[idx]) / W * kd * (T)2 * scale;
                    gxs += sgr * dx; gys += sgr * dy; gzs += sgr * dz;
                }
            }
        }
        Tb[p] += tb;
        xb[3 * p] += gxs; xb[3 * p + 1] += gys; xb[3 * p + 2] += gzs;
    }
}

// the cell each particle had in a step's recorded sort
__global__ void k_ad_cellof(int ncell, const uint32_t* __restrict__ order, const uint32_t* __restrict__ off,
                            uint32_t* __restrict__ cellof) {
    MP_GRID_LOOP(c, ncell) for (uint32_t s = off[c]; s < off[c + 1]; s++) cellof[order[s]] = (uint32_t)c;
}
template <class T> __global__ void k_ad_to_double(long long n, const T* __restrict__ a, double* __restrict__ o) {
    MP_GRID_LOOP(t, n) o[t] = (double)a[t];
}
template <class T> __global__ void k_ad_from_float(long long n, const float* __restrict__ a, T* __restrict__ o) {
    MP_GRID_LOOP(t, n) o[t] = (T)a[t];
}
template <class T> __global__ void k_ad_from_double(long long n, const double* __restrict__ a, T* __restrict__ o) {
    MP_GRID_LOOP(t, n) o[t] = (T)a[t];
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void k_adj_free(MpCtx* c) {
    AdjTape* t = c->adj;
    if (!t) return;
    // the per-step arrays point into the arena
    for (void* p : {(void*)t->x0, (void*)t->v0, (void*)t->mass, (void*)t->ids, (void*)t->ids2, (void*)t->nearest,
                    (void*)t->samples, (void*)t->s_off, (void*)t->T0, (void*)t->fixedheat, (void*)t->phase,
                    (void*)t->mass_w, (void*)t->mass_a, (void*)t->arena, (void*)t->eng_xs, (void*)t->eng_vs})
        if (p) cudaFree(p);
    for (void* p : t->wk) if (p) cudaFree(p);
    delete t;
    c->adj = nullptr;
}

template <class T> static int amalloc(MpCtx* c, T** p, size_t count) {
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
    if (e != cudaSuccess) { c->err = std::string("adjoint: cudaMalloc: ") + cudaGetErrorString(e); return MP_ERR_CUDA; }
    return MP_OK;
}
#define ADJ_LAUNCH(c) MP_CHECK_LAUNCH(c)

static int sorted_ids(MpCtx* c, AdjTape* t) {
    // after k_hash_sort: when the particles moved, slot s now holds the
    // particle of old slot perm[s]
    MP_TRY(k_hash_sort(c));
    uint32_t moved = 0;
    MP_CUDA(c, cudaMemcpyAsync(&moved, c->u32_scratch + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    if (moved) {
        k_ad_permute_ids<<<mp_blocks(t->np, 256), 256, 0, c->stream>>>(t->np, c->perm, t->ids, t->ids2);
        ADJ_LAUNCH(c);
        std::swap(t->ids, t->ids2);
    }
    return MP_OK;
}

static int record_tape(MpCtx* c, AdjTape* t, bool air);

int k_adj_record(MpCtx* c, int nsteps, int every) {
    const mp_params& P = c->P;
    if (nsteps < 1 || every < 1) { c->err = "adj_record: nsteps and checkpoint interval must be positive"; return MP_ERR_ARG; }
    if (P.b_correct_position || P.b_gen_gas || P.b_melt || P.b_freeze || P.b_solid) {
        c->err = "adj_record: the adjoint covers the FLUID and AIR step without position correction, gas, "
                 "melting, freezing or solids";
        return MP_ERR_STATE;
    }
    const int sc = P.scene;
    const bool boil = sc == MP_SCENE_BOILING || sc == MP_SCENE_BOILING_HIGHRES || sc == MP_SCENE_MELTANDBOIL ||
                      sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL;
    if (P.b_heat_trans && (P.b_add_heat_bottom || boil)) {
        c->err = "adj_record: the heat stage is differentiated without the bottom heat increment and outside "
                 "the boiling scenes (whose heat matrix is not symmetric)";
        return MP_ERR_STATE;
    }
    const int np = c->np();
    if (np == 0) { c->err = "adj_record: no particles"; return MP_ERR_STATE; }
    MP_CUDA(c, cudaMemsetAsync(c->u32_scratch + 3, 0, 3 * sizeof(uint32_t), c->stream));
    k_ad_count_types<<<mp_blocks(np, 256), 256, 0, c->stream>>>(np, c->pos, c->u32_scratch + 3);
    uint32_t cnt[3] = {0, 0, 0};
    MP_CUDA(c, cudaMemcpyAsync(cnt, c->u32_scratch + 3, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    if (cnt[0]) { c->err = "adj_record: every particle must be FLUID or AIR"; return MP_ERR_STATE; }
    if (cnt[2] && P.b_heat_trans) {
        c->err = "adj_record: the heat stage is differentiated for FLUID particles only (no AIR)";
        return MP_ERR_STATE;
    }
    k_adj_free(c);
    AdjTape* t = new AdjTape();
    c->adj = t;
    t->np = np; t->nsteps = nsteps; t->every = every;
    const int rc = record_tape(c, t, cnt[2] != 0);
    // a recording that stopped part-way keeps no tape: its missing steps
    // hold no state, and a replay would read past the recorded ones
    if (rc != MP_OK) k_adj_free(c);
    return rc;
}

// the snapshots and every step's recorded state, stepping the engine
static int record_tape(MpCtx* c, AdjTape* t, bool air) {
    const mp_params& P = c->P;
    const int np = t->np, nsteps = t->nsteps, every = t->every;
    const Grid& g = c->G;
    MP_TRY(amalloc(c, &t->ids, np)); MP_TRY(amalloc(c, &t->ids2, np));
    MP_TRY(amalloc(c, &t->x0, 3 * (size_t)np)); MP_TRY(amalloc(c, &t->v0, 3 * (size_t)np));
    MP_TRY(amalloc(c, &t->mass, np)); MP_TRY(amalloc(c, &t->nearest, g.n));
    k_ad_iota<<<mp_blocks(np, 256), 256, 0, c->stream>>>(np, t->ids);
    k_ad_snapshot<<<mp_blocks(np, 256), 256, 0, c->stream>>>(np, t->ids, c->pos, c->vel, t->x0, t->v0, t->mass);
    ADJ_LAUNCH(c);
    t->air = air;
    if (t->air) {
        MP_TRY(amalloc(c, &t->phase, np)); MP_TRY(amalloc(c, &t->mass_w, np)); MP_TRY(amalloc(c, &t->mass_a, np));
        k_ad_snapshot_phase<<<mp_blocks(np, 256), 256, 0, c->stream>>>(np, t->ids, c->pos, c->vel, t->phase,
                                                                       t->mass_w, t->mass_a);
        ADJ_LAUNCH(c);
    }
    t->heat = P.b_heat_trans != 0;
    if (t->heat) {
        MP_TRY(amalloc(c, &t->T0, np));
        k_ad_snapshot_T<<<mp_blocks(np, 256), 256, 0, c->stream>>>(np, t->ids, c->heat, t->T0);
        ADJ_LAUNCH(c);
        if (P.b_fixed_heat) {
            MP_TRY(amalloc(c, &t->fixedheat, g.n));
            MP_CUDA(c, cudaMemcpyAsync(t->fixedheat, c->fixedheat, sizeof(float) * g.n, cudaMemcpyDeviceToDevice,
                                       c->stream));
        }
    }
    // every step's recorded state in one allocation (allocating per step in
    // the loop costs more than the copies)
    const auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t n = (size_t)g.n, snp = (size_t)np;
    t->eng = P.precision == MP_PREC_MIXED && P.coef_mode == MP_COEF_REF && P.cg_refine_tol == 0.0f &&
             P.cg_true_residual_every == 0;
    const size_t per = up(4 * snp) + up(4 * (n + 1)) + up(n) + up(4 * n) + (t->air ? 2 * up(4 * n) : 0) +
                       (t->heat ? up(4 * snp) + up(4 * (n + 1)) + up(n) : 0) + (t->eng ? 2 * up(4 * n) : 0);
    MP_TRY(amalloc(c, &t->arena, per * (size_t)nsteps));
    const int nseg = (nsteps + every - 1) / every;
    if (t->eng && !t->heat) {
        MP_TRY(amalloc(c, &t->eng_xs, 3 * snp * (size_t)nseg));
        MP_TRY(amalloc(c, &t->eng_vs, 3 * snp * (size_t)nseg));
    }
    auto eng_state = [&](int e) -> int {
        k_ad_snapshot<<<mp_blocks(np, 256), 256, 0, c->stream>>>(np, t->ids, c->pos, c->vel, t->eng_xs + 3 * snp * e,
                                                                 t->eng_vs + 3 * snp * e, t->mass);
        ADJ_LAUNCH(c);
        return MP_OK;
    };
    for (int k = 0; k < nsteps; k++) {
        if (t->eng_xs && k > 0 && k % every == 0) MP_TRY(eng_state(k / every - 1));
        char* slab = t->arena + per * (size_t)k;
        auto carve = [&](size_t bytes) { char* q = slab; slab += up(bytes); return q; };
        MP_TRY(sorted_ids(c, t));
        MP_TRY(k_external_force(c));
        MP_TRY(k_levelset(c)); MP_TRY(k_sweep_ls_mark(c));
        uint32_t* ord = reinterpret_cast<uint32_t*>(carve(4 * snp)); t->order.push_back(ord);
        uint32_t* off = reinterpret_cast<uint32_t*>(carve(4 * (n + 1))); t->off.push_back(off);
        int8_t* mk = reinterpret_cast<int8_t*>(carve(n)); t->mark.push_back(mk);
        float* ph = reinterpret_cast<float*>(carve(4 * n)); t->phi.push_back(ph);
        MP_CUDA(c, cudaMemcpyAsync(ord, t->ids, sizeof(uint32_t) * np, cudaMemcpyDeviceToDevice, c->stream));
        MP_CUDA(c, cudaMemcpyAsync(off, c->cell_off, sizeof(uint32_t) * ((size_t)g.n + 1), cudaMemcpyDeviceToDevice, c->stream));
        MP_CUDA(c, cudaMemcpyAsync(mk, c->mark, g.n, cudaMemcpyDeviceToDevice, c->stream));
        MP_TRY(k_p2g(c));
        if (t->air) {
            // bubblesim's order: the air phase's extrapolation first
            float* lm = reinterpret_cast<float*>(carve(4 * n)); t->lsm.push_back(lm);
            float* pa = reinterpret_cast<float*>(carve(4 * n)); t->phia.push_back(pa);
            MP_CUDA(c, cudaMemcpyAsync(lm, c->lsmerge, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, c->stream));
            MP_TRY(k_sweep_phi(c, MP_TYPEAIR));
            MP_CUDA(c, cudaMemcpyAsync(pa, c->phiair, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, c->stream));
            MP_TRY(k_sweep_u(c, MP_TYPEAIR));
        }
        MP_TRY(k_sweep_phi(c, MP_TYPEFLUID));
        MP_CUDA(c, cudaMemcpyAsync(ph, c->phifluid, sizeof(float) * g.n, cudaMemcpyDeviceToDevice, c->stream));
        MP_TRY(k_sweep_u(c, MP_TYPEFLUID));
        if (t->air) MP_TRY(k_set_boundary_u(c, MP_TYPEAIR));
        MP_TRY(k_set_boundary_u(c, MP_TYPEFLUID));
        int st = k_project(c, nullptr, nullptr);
        if (st != MP_OK && st != MP_ERR_NOCONVERGE) return st;
        if (t->eng) {
            float* eb = reinterpret_cast<float*>(carve(4 * n)); t->eng_b.push_back(eb);
            float* ep = reinterpret_cast<float*>(carve(4 * n)); t->eng_p.push_back(ep);
            MP_CUDA(c, cudaMemcpyAsync(eb, c->divg, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
            MP_CUDA(c, cudaMemcpyAsync(ep, c->press, sizeof(float) * n, cudaMemcpyDeviceToDevice, c->stream));
        }
        if (t->air) MP_TRY(k_sweep_u(c, MP_TYPEAIR));
        MP_TRY(k_sweep_u(c, MP_TYPEFLUID));
        if (t->air) MP_TRY(k_set_boundary_u(c, MP_TYPEAIR));
        MP_TRY(k_set_boundary_u(c, MP_TYPEFLUID));
        MP_TRY(k_g2p(c));
        MP_TRY(sorted_ids(c, t));
        MP_TRY(k_collide_advect(c, true));
        MP_TRY(sorted_ids(c, t));
        if (t->heat) {
            // bubblesim without position correction: level set and marks of
            // the advected particles, a sort, then updateTemperature
            MP_TRY(k_levelset(c)); MP_TRY(k_sweep_ls_mark(c));
            MP_TRY(sorted_ids(c, t));
            uint32_t* oh = reinterpret_cast<uint32_t*>(carve(4 * snp)); t->order_h.push_back(oh);
            uint32_t* fh = reinterpret_cast<uint32_t*>(carve(4 * (n + 1))); t->off_h.push_back(fh);
            int8_t* mh = reinterpret_cast<int8_t*>(carve(n)); t->mark_h.push_back(mh);
            MP_CUDA(c, cudaMemcpyAsync(oh, t->ids, sizeof(uint32_t) * np, cudaMemcpyDeviceToDevice, c->stream));
            MP_CUDA(c, cudaMemcpyAsync(fh, c->cell_off, sizeof(uint32_t) * ((size_t)g.n + 1), cudaMemcpyDeviceToDevice,
                                       c->stream));
            MP_CUDA(c, cudaMemcpyAsync(mh, c->mark, g.n, cudaMemcpyDeviceToDevice, c->stream));
            int st = k_heat(c);
            if (st != MP_OK && st != MP_ERR_NOCONVERGE) return st;
        }
        c->S.frame++;
    }
    if (t->eng_xs) MP_TRY(eng_state(nseg - 1));
    // nearest particle of each cell at the end (cells from the last sort)
    k_ad_nearest<<<mp_blocks(g.n, 256), 256, 0, c->stream>>>(g, Cells{c->cell_off, c->tmask}, c->pos, t->ids, t->nearest);
    ADJ_LAUNCH(c);
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

int k_adj_set_targets(MpCtx* c, const float* sp, int ns) {
    AdjTape* t = c->adj;
    if (!t) { c->err = "adj_set_targets: record first"; return MP_ERR_STATE; }
    if (ns < 1 || !sp) { c->err = "adj_set_targets: no samples"; return MP_ERR_ARG; }
    const Grid& g = c->G;
    std::vector<std::pair<int, int>> key(ns);
    for (int s = 0; s < ns; s++) {
        int i, j, k; sample_base(g.h, g.NX, g.NY, g.NZ, sp[3 * s], sp[3 * s + 1], sp[3 * s + 2], i, j, k);
        key[s] = {(i * g.NY + j) * g.NZ + k, s};
    }
    std::stable_sort(key.begin(), key.end());
    std::vector<float> sorted(3 * (size_t)ns);
    std::vector<uint32_t> off((size_t)g.n + 1, 0);
    for (int s = 0; s < ns; s++) {
        for (int a = 0; a < 3; a++) sorted[3 * s + a] = sp[3 * key[s].second + a];
        off[key[s].first + 1]++;
    }
    for (int q = 0; q < g.n; q++) off[q + 1] += off[q];
    if (t->samples) cudaFree(t->samples);
    if (t->s_off) cudaFree(t->s_off);
    // no samples until the new ones are on the device (a failure below
    // leaves the tape without targets, not with freed ones)
    t->samples = nullptr; t->s_off = nullptr; t->nsamples = 0;
    MP_TRY(amalloc(c, &t->samples, 3 * (size_t)ns)); MP_TRY(amalloc(c, &t->s_off, (size_t)g.n + 1));
    MP_CUDA(c, cudaMemcpy(t->samples, sorted.data(), sizeof(float) * 3 * ns, cudaMemcpyHostToDevice));
    MP_CUDA(c, cudaMemcpy(t->s_off, off.data(), sizeof(uint32_t) * (g.n + 1), cudaMemcpyHostToDevice));
    t->nsamples = ns;
    return MP_OK;
}

namespace {
// work layout: element counts per buffer; W_I* hold one step's intermediates
// (each step is replayed again just before its transpose)
enum {
    W_XS, W_VS, W_XB, W_VB, W_VAB, W_VGB, W_X, W_V, W_XN, W_VN,
    W_T0, W_UPROJ, W_B0, W_B1, W_B2,
    W_IVA, W_IVG, W_CUP, W_CWT, W_IUE, W_IUF, W_IDU, W_ISEL, W_ISW,
    W_CB, W_CP, W_CQ, W_PHI, W_SV, W_LOSS, W_CELLOF, W_FLAG, W_S4A, W_S4B, W_PST,
    // heat: temperatures (current, next, segment states, cotangent), per-slot
    // intermediates (cell temperature and weight, extended solution, change;
    // particle temperature before the clamp), scratch, cached solves
    W_T, W_TN, W_TS, W_TB, W_HT1, W_HTC, W_HWC, W_HTE, W_HDT, W_HB, W_HBB, W_HQ, W_HQ1, W_HTEB, W_HTCB, W_HST,
    W_HS4, W_HCELLOF,
    // the air phase: its splat's old field, projected field and scratch, its
    // splat records, and its per-slot intermediates (splat, weights,
    // extrapolated, final, change; extrapolation choices)
    W_UPROJA, W_A0, W_A1, W_A2, W_S4C, W_CUPA, W_CWTA, W_IUEA, W_IUFA, W_IDUA, W_ISELA, W_ISWA, W_AIRC,
    W_CBAD, W_CNEAR,   // per cell: holds a particle whose replay cell moved; near one
    W_COUNT
};
}

// one step's intermediates (what its transpose reads)
template <class T> struct Inter {
    T* va; T* vg; Fc<T> up, wt, ue, uf, du; uint8_t* sel; float* sw;
    T* Tc; T* Wc; T* Te; T* dT; T* T1;   // heat stage (when recorded)
    Fc<T> upa, wta, uea, ufa, dua; uint8_t* sela; float* swa;   // air phase (when recorded)
};

template <class T> struct Replay {
    MpCtx* c; AdjTape* t; Grid g; long long nf; int np;
    T* a(int w) const { return static_cast<T*>(t->wk[w]); }
    Fc<T> f(int w) const { return faces_of<T>(t->wk[w], g); }
    T* seg_x(int s) const { return a(W_XS) + (size_t)s * 3 * np; }
    T* seg_v(int s) const { return a(W_VS) + (size_t)s * 3 * np; }
    Inter<T> inter(int j) const {
        const size_t np3 = 3 * (size_t)np, nfs = (size_t)nf;
        Inter<T> I;
        I.va = a(W_IVA) + j * np3; I.vg = a(W_IVG) + j * np3;
        I.ue = faces_of<T>(a(W_IUE) + j * nfs, g); I.uf = faces_of<T>(a(W_IUF) + j * nfs, g);
        I.du = faces_of<T>(a(W_IDU) + j * nfs, g);
        I.sel = static_cast<uint8_t*>(t->wk[W_ISEL]) + j * nfs;
        I.sw = static_cast<float*>(t->wk[W_ISW]) + 3 * j * nfs;
        const size_t n = t->heat ? (size_t)g.n : 0, npp = t->heat ? (size_t)np : 0;
        I.Tc = a(W_HTC) + j * n; I.Wc = a(W_HWC) + j * n; I.Te = a(W_HTE) + j * n; I.dT = a(W_HDT) + j * n;
        I.T1 = a(W_HT1) + j * npp;
        const size_t nfa = t->air ? nfs : 0;
        I.uea = faces_of<T>(a(W_IUEA) + j * nfa, g); I.ufa = faces_of<T>(a(W_IUFA) + j * nfa, g);
        I.dua = faces_of<T>(a(W_IDUA) + j * nfa, g);
        I.sela = static_cast<uint8_t*>(t->wk[W_ISELA]) + j * nfa;
        I.swa = static_cast<float*>(t->wk[W_ISWA]) + 3 * j * nfa;
        return I;
    }
    T* seg_T(int s) const { return a(W_TS) + (size_t)s * np; }
    // step k's splats (field and weights of each phase): the first replay
    // computes them, the later replays of the reverse sweep (same inputs)
    // read them back
    Inter<T> with_splat(const Inter<T>& I0, int k) const {
        Inter<T> I = I0;
        const size_t ks = (size_t)k * (size_t)nf, ka = t->air ? ks : 0;
        I.up = faces_of<T>(a(W_CUP) + ks, g); I.wt = faces_of<T>(a(W_CWT) + ks, g);
        I.upa = faces_of<T>(a(W_CUPA) + ka, g); I.wta = faces_of<T>(a(W_CWTA) + ka, g);
        return I;
    }
};

template <class T> static int adj_work(MpCtx* c, AdjTape* t) {
    if (t->wesz == sizeof(T) && (int)t->wk.size() == W_COUNT && t->wk_ns >= t->nsamples) return MP_OK;
    for (void* p : t->wk) if (p) cudaFree(p);
    t->wk.assign(W_COUNT, nullptr);
    // marked unusable until every array below is allocated: a failed
    // allocation leaves null arrays that no later call may take as ready
    t->wesz = 0; t->wk_ns = 0;
    const Grid& g = c->G;
    const size_t np3 = 3 * (size_t)t->np, nf = (size_t)g.nfx + g.nfy + g.nfz, n = g.n;
    const int nseg = (t->nsteps + t->every - 1) / t->every;
    const size_t E = 1;   // intermediates of one step at a time (adj_run)
    size_t cnt[W_COUNT], es[W_COUNT];
    for (int w = 0; w < W_COUNT; w++) es[w] = sizeof(T);
    cnt[W_XS] = cnt[W_VS] = np3 * (size_t)(nseg + t->every);   // segment starts, then one segment's steps
    for (int w : {W_XB, W_VB, W_VAB, W_VGB, W_X, W_V, W_XN, W_VN}) cnt[w] = np3;
    for (int w : {W_T0, W_UPROJ, W_B0, W_B1, W_B2}) cnt[w] = nf;
    cnt[W_IVA] = cnt[W_IVG] = np3 * E;
    for (int w : {W_IUE, W_IUF, W_IDU}) cnt[w] = nf * E;
    for (int w : {W_CUP, W_CWT}) cnt[w] = nf * (size_t)t->nsteps;
    cnt[W_ISEL] = nf * E; es[W_ISEL] = 1;
    cnt[W_ISW] = 3 * nf * E; es[W_ISW] = sizeof(float);
    for (int w : {W_CB, W_CP, W_CQ, W_PHI}) cnt[w] = n;
    cnt[W_SV] = (size_t)std::max(t->nsamples, 1) * 2; es[W_SV] = sizeof(double);
    cnt[W_LOSS] = 2; es[W_LOSS] = sizeof(double);
    cnt[W_CELLOF] = (size_t)t->np; es[W_CELLOF] = sizeof(uint32_t);
    cnt[W_FLAG] = 4; es[W_FLAG] = sizeof(uint32_t);
    cnt[W_S4A] = cnt[W_S4B] = 4 * (size_t)t->np;
    cnt[W_PST] = n * (size_t)t->nsteps;   // each step's pressure from the first replay
    const size_t hn = t->heat ? n : 0, hp = t->heat ? (size_t)t->np : 0;
    for (int w : {W_T, W_TN, W_TB, W_HQ1}) cnt[w] = hp;
    cnt[W_TS] = hp * (size_t)(nseg + t->every);
    cnt[W_HT1] = hp * E;
    for (int w : {W_HTC, W_HWC, W_HTE, W_HDT}) cnt[w] = hn * E;
    for (int w : {W_HB, W_HBB, W_HQ, W_HTEB, W_HTCB}) cnt[w] = hn;
    cnt[W_HST] = hn * (size_t)t->nsteps;
    cnt[W_HS4] = 4 * hp;
    cnt[W_HCELLOF] = hp; es[W_HCELLOF] = sizeof(uint32_t);
    const size_t af = t->air ? nf : 0;
    for (int w : {W_UPROJA, W_A0, W_A1, W_A2}) cnt[w] = af;
    cnt[W_S4C] = t->air ? 4 * (size_t)t->np : 0;
    for (int w : {W_IUEA, W_IUFA, W_IDUA}) cnt[w] = af * E;
    for (int w : {W_CUPA, W_CWTA}) cnt[w] = af * (size_t)t->nsteps;
    cnt[W_ISELA] = af * E; es[W_ISELA] = 1;
    cnt[W_ISWA] = 3 * af * E; es[W_ISWA] = sizeof(float);
    cnt[W_AIRC] = t->air ? n : 0; es[W_AIRC] = 1;
    cnt[W_CBAD] = cnt[W_CNEAR] = n; es[W_CBAD] = es[W_CNEAR] = 1;
    for (int w = 0; w < W_COUNT; w++) {
        size_t bytes = es[w] * std::max<size_t>(cnt[w], 1);
        cudaError_t e = cudaMalloc(&t->wk[w], bytes);
        if (e != cudaSuccess) { c->err = std::string("adjoint work: ") + cudaGetErrorString(e); return MP_ERR_CUDA; }
    }
    t->wesz = sizeof(T);
    t->wk_ns = t->nsamples;
    return MP_OK;
}

template <class T> static int cg_tol_of(const MpCtx* c, int& mode, float& tol, int& maxit) {
    if (sizeof(T) == sizeof(double)) { mode = MP_TOL_REL; tol = 1e-13f; maxit = std::max(c->P.cg_max_iter, 6000); }
    else { mode = c->P.cg_tol_mode; tol = c->P.cg_tol; maxit = c->P.cg_max_iter; }
    return MP_OK;
}

static HeatCoef heat_coef(const mp_params& P) {
    HeatCoef hc;
    hc.alpha[MP_TYPEFLUID] = P.heatalpha_fluid; hc.alpha[MP_TYPEAIR] = P.heatalpha_air;
    hc.alpha[MP_TYPEVACUUM] = P.heatalpha_vacuum; hc.alpha[MP_TYPESOLID] = P.heatalpha_solid;
    hc.alpha[MP_TYPEAIRSOLO] = P.heatalpha_air; hc.alpha[MP_TYPEBOUNDARY] = 0;
    hc.dt = P.dt;
    return hc;
}

// the heat stage of step k on the advected positions x1: temperatures Tin ->
// Tout, keeping its intermediates in I (its solve cached per step in W_HST)
template <class T> static int heat_fwd(const Replay<T>& R, int k, const T* x1, const T* Tin, T* Tout,
                                       const Inter<T>& I, bool solve) {
    MpCtx* c = R.c; AdjTape* t = R.t; const Grid& g = R.g;
    cudaStream_t s = c->stream;
    const mp_params& P = c->P;
    const int nbp = mp_blocks(R.np, 256), nbc = mp_blocks(g.n, 256);
    k_ad_slot_gather1<T><<<nbp, 256, 0, s>>>(R.np, t->order_h[k], x1, Tin, R.a(W_HS4));
    k_ad_heat_p2g<T><<<nbc, 256, 0, s>>>(g, t->off_h[k], R.a(W_HS4), (T)P.default_temperature, I.Tc, I.Wc);
    k_ad_heat_rhs<T><<<nbc, 256, 0, s>>>(g, I.Tc, t->mark_h[k], t->fixedheat, heat_coef(P), R.a(W_HB));
    MP_CHECK_LAUNCH(c);
    T* tn = R.a(W_HST) + (size_t)k * g.n;
    if (solve) {
        // the engine's stop rule in FP32 (absolute, as updateTemperature); FP64: relative 1e-13
        const bool f64 = sizeof(T) == sizeof(double);
        int it = 0; double res = 0;
        int st = k_heat_cg_solve(c, t->mark_h[k], tn, R.a(W_HB), f64 ? std::max(P.heat_cg_max_iter, 6000) : P.heat_cg_max_iter,
                                 f64 ? MP_TOL_REL : MP_TOL_REF_ABS, f64 ? 1e-13f : 0.01f, &it, &res);
        if (st != MP_OK && st != MP_ERR_NOCONVERGE) return st;
    }
    if (P.b_extend_heat_to_boundary) k_ad_heat_ext<T><<<nbc, 256, 0, s>>>(g, tn, I.Te);
    else k_ad_copy<T><<<nbc, 256, 0, s>>>(g.n, tn, I.Te);
    k_ad_heat_dT<T><<<nbc, 256, 0, s>>>(g.n, I.Te, I.Tc, t->mark_h[k], I.dT);
    k_ad_heat_g2p<T><<<nbp, 256, 0, s>>>(g, R.np, x1, Tin, I.dT, I.Te, (T)P.alpha_temp_trans, (T)P.melting_point,
                                         (T)P.boiling_point, I.T1, Tout);
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// transpose of the heat stage: Tb holds the cotangent of Tout on entry and of
// Tin on exit; the cotangent of x1 is added to xb
template <class T> static int heat_adj(const Replay<T>& R, int k, const T* x1, const T* Tin, const Inter<T>& I, T* Tb,
                                       T* xb) {
    MpCtx* c = R.c; AdjTape* t = R.t; const Grid& g = R.g;
    cudaStream_t s = c->stream;
    const mp_params& P = c->P;
    const int nbp = mp_blocks(R.np, 256), nbc = mp_blocks(g.n, 256);
    const T a = (T)P.alpha_temp_trans;
    uint32_t* cellof = static_cast<uint32_t*>(t->wk[W_HCELLOF]);
    uint32_t* flag = static_cast<uint32_t*>(t->wk[W_FLAG]);
    k_ad_cellof<<<nbc, 256, 0, s>>>(g.n, t->order_h[k], t->off_h[k], cellof);
    MP_CUDA(c, cudaMemsetAsync(flag, 0, sizeof(uint32_t), s));
    k_ad_cell_mismatch<T><<<nbp, 256, 0, s>>>(g, R.np, x1, cellof, flag, nullptr);
    k_ad_heat_g2p_adj_p<T><<<nbp, 256, 0, s>>>(g, R.np, x1, I.T1, I.dT, I.Te, a, (T)P.melting_point,
                                               (T)P.boiling_point, Tb, R.a(W_HQ1), xb);
    k_ad_slot_gather1<T><<<nbp, 256, 0, s>>>(R.np, t->order_h[k], x1, R.a(W_HQ1), R.a(W_HS4));
    MP_CHECK_LAUNCH(c);
    uint32_t wide = 1;
    MP_CUDA(c, cudaMemcpyAsync(&wide, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    if (wide) k_ad_heat_g2p_adj_c<T, true><<<nbc, 256, 0, s>>>(g, t->off_h[k], R.a(W_HS4), R.a(W_HQ));
    else k_ad_heat_g2p_adj_c<T, false><<<nbc, 256, 0, s>>>(g, t->off_h[k], R.a(W_HS4), R.a(W_HQ));
    k_ad_heat_mix<T><<<nbc, 256, 0, s>>>(g.n, t->mark_h[k], R.a(W_HQ), a, R.a(W_HTEB), R.a(W_HTCB));
    if (P.b_extend_heat_to_boundary) k_ad_heat_ext_adj<T><<<nbc, 256, 0, s>>>(g, R.a(W_HTEB), R.a(W_HBB));
    else k_ad_copy<T><<<nbc, 256, 0, s>>>(g.n, R.a(W_HTEB), R.a(W_HBB));
    MP_CHECK_LAUNCH(c);
    // the transposed solve (the heat matrix is symmetric): relative stop, the
    // cotangent's scale being arbitrary
    {
        const bool f64 = sizeof(T) == sizeof(double);
        int it = 0; double res = 0;
        int st = k_heat_cg_solve(c, t->mark_h[k], R.a(W_HB), R.a(W_HBB),
                                 f64 ? std::max(P.heat_cg_max_iter, 6000) : P.heat_cg_max_iter, MP_TOL_REL,
                                 f64 ? 1e-13f : 1e-6f, &it, &res);
        if (st != MP_OK && st != MP_ERR_NOCONVERGE) return st;
    }
    k_ad_heat_rhs_adj<T><<<nbc, 256, 0, s>>>(g, R.a(W_HB), t->mark_h[k], t->fixedheat, heat_coef(P), R.a(W_HTCB));
    k_ad_heat_p2g_adj<T><<<nbp, 256, 0, s>>>(g, R.np, x1, Tin, cellof, I.Tc, I.Wc, R.a(W_HTCB), Tb, xb);
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// one step of the replay from (x, v) to (xo, vo), keeping what its transpose
// needs in I
// The pressure solve's result is stored in pst (first replay) or copied from
// it (segment replays): the inputs are the same bit for bit, so is the result.
template <class T> static int fwd_step(const Replay<T>& R, int k, const T* x, const T* v, T* xo, T* vo,
                                       const T* Tin, T* Tout, const Inter<T>& I0, bool solve, bool splat) {
    MpCtx* c = R.c; AdjTape* t = R.t; const Grid& g = R.g;
    const Inter<T> I = R.with_splat(I0, k);
    cudaStream_t s = c->stream;
    const int nbp = mp_blocks(R.np, 256), nbf = mp_blocks(R.nf, 256), nbc = mp_blocks(g.n, 256);
    const mp_params& P = c->P;
    const bool air = t->air;
    k_ad_sweep_sel<<<nbf, 256, 0, s>>>(g, t->phi[k], t->mark[k], MP_TYPEFLUID, I.sel, I.sw);
    if (air) {
        k_ad_sweep_sel<<<nbf, 256, 0, s>>>(g, t->phia[k], t->mark[k], MP_TYPEAIR, I.sela, I.swa);
        k_ad_forces<T><<<nbp, 256, 0, s>>>(R.np, t->phase, v, I.va, (T)P.dt * (T)P.gravity_z,
                                           (T)P.buoyance_rate_air, (T)P.bubble_max_vel);
    } else {
        k_ad_gravity<T><<<nbp, 256, 0, s>>>(R.np, v, I.va, (T)P.dt * (T)P.gravity_z);
    }
    // the splats (kept per step: the replays after the first read them back);
    // each splat stays as it is through the step and is its FLIP old field
    const int nbw = mp_blocks(make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1).threads(), 256);
    if (splat) {
        k_ad_slot_gather<T><<<nbp, 256, 0, s>>>(R.np, t->order[k], x, I.va, air ? t->mass_w : t->mass, R.a(W_S4A),
                                                R.a(W_S4B));
        k_ad_p2g_w<T, 0><<<nbw, 256, 0, s>>>(g, t->off[k], R.a(W_S4A), R.a(W_S4B), I.up, I.wt, nullptr);
    }
    if (air) {
        uint8_t* airc = static_cast<uint8_t*>(t->wk[W_AIRC]);
        k_ad_air_cells<<<nbc, 256, 0, s>>>(g.n, t->off[k], t->order[k], t->phase, airc);
        if (splat) {
            k_ad_slot_gather<T><<<nbp, 256, 0, s>>>(R.np, t->order[k], x, I.va, t->mass_a, R.a(W_S4C), R.a(W_S4B));
            k_ad_p2g_w<T, 1><<<nbw, 256, 0, s>>>(g, t->off[k], R.a(W_S4C), R.a(W_S4B), I.upa, I.wta, airc);
        }
        k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, I.upa, R.f(W_T0), I.sela, I.swa);
        k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_T0), R.f(W_A0), I.sela, I.swa);
    }
    k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, I.up, R.f(W_T0), I.sel, I.sw);
    k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_T0), R.f(W_B0), I.sel, I.sw);
    if (air) k_ad_bound<T><<<nbf, 256, 0, s>>>(g, R.f(W_A0), I.uea, t->mark[k]);
    k_ad_bound<T><<<nbf, 256, 0, s>>>(g, R.f(W_B0), I.ue, t->mark[k]);
    if (air) k_ad_div2<T><<<nbc, 256, 0, s>>>(g, t->mark[k], t->lsm[k], I.ue, I.uea, R.a(W_CB));
    else k_ad_div<T><<<nbc, 256, 0, s>>>(g, t->mark[k], I.ue, R.a(W_CB));
    MP_CHECK_LAUNCH(c);
    T* pk = R.a(W_PST) + (size_t)k * g.n;
    if (solve) {
        bool same = false;
        if constexpr (sizeof(T) == sizeof(float)) {
            if (t->eng) {
                uint32_t* flag = static_cast<uint32_t*>(t->wk[W_FLAG]) + 1;
                MP_CUDA(c, cudaMemsetAsync(flag, 0, sizeof(uint32_t), s));
                k_ad_differ<<<nbc, 256, 0, s>>>(g.n, reinterpret_cast<const float*>(R.a(W_CB)), t->eng_b[k], flag);
                uint32_t differ = 1;
                MP_CUDA(c, cudaMemcpyAsync(&differ, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                MP_CUDA(c, cudaStreamSynchronize(s));
                same = differ == 0;
                if (same)
                    MP_CUDA(c, cudaMemcpyAsync(pk, t->eng_p[k], sizeof(float) * g.n, cudaMemcpyDeviceToDevice, s));
            }
        }
        if (!same) {
            int mode, maxit; float tol; cg_tol_of<T>(c, mode, tol, maxit);
            int it = 0; double res = 0;
            int st = k_cg_solve(c, t->mark[k], pk, R.a(W_CB), maxit, mode, tol, &it, &res);
            if (st != MP_OK && st != MP_ERR_NOCONVERGE) return st;
        }
    }
    k_ad_subgrad<T><<<nbf, 256, 0, s>>>(g, pk, I.ue, R.f(W_UPROJ));
    if (air) {
        k_ad_subgrad<T><<<nbf, 256, 0, s>>>(g, pk, I.uea, R.f(W_UPROJA));
        k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_UPROJA), R.f(W_A1), I.sela, I.swa);
        k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_A1), R.f(W_A2), I.sela, I.swa);
    }
    k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_UPROJ), R.f(W_B1), I.sel, I.sw);
    k_ad_sweepu_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_B1), R.f(W_B2), I.sel, I.sw);
    if (air) {
        k_ad_bound<T><<<nbf, 256, 0, s>>>(g, R.f(W_A2), I.ufa, t->mark[k]);
        k_ad_sub<T><<<nbf, 256, 0, s>>>(R.nf, I.ufa.x, I.upa.x, I.dua.x);
    }
    k_ad_bound<T><<<nbf, 256, 0, s>>>(g, R.f(W_B2), I.uf, t->mark[k]);
    k_ad_sub<T><<<nbf, 256, 0, s>>>(R.nf, I.uf.x, I.up.x, I.du.x);
    k_ad_g2p<T><<<nbp, 256, 0, s>>>(g, R.np, x, I.va, I.uf, I.du, (T)P.flip_alpha, I.vg, air ? t->phase : nullptr,
                                    I.ufa, I.dua);
    k_ad_advect<T><<<nbp, 256, 0, s>>>(g, R.np, x, I.vg, xo, vo, (T)P.dt);
    MP_CHECK_LAUNCH(c);
    if (t->heat) MP_TRY(heat_fwd<T>(R, k, xo, Tin, Tout, I, solve));
    return MP_OK;
}

// transpose of a step from its intermediates: (xb, vb) hold the adjoint of the
// step's outputs on entry and of its inputs on exit; v is the step's input
// velocity (the air force's slope depends on it)
template <class T> static int adj_step(const Replay<T>& R, int k, const T* x, const T* v, const T* x1, const T* Tin,
                                       const Inter<T>& I0, T* xb, T* vb, T* Tb) {
    MpCtx* c = R.c; AdjTape* t = R.t; const Grid& g = R.g;
    const Inter<T> I = R.with_splat(I0, k);
    // the heat stage ran last, on the advected positions x1
    if (t->heat) MP_TRY(heat_adj<T>(R, k, x1, Tin, I, Tb, xb));
    cudaStream_t s = c->stream;
    const int nbp = mp_blocks(R.np, 256), nbf = mp_blocks(R.nf, 256), nbc = mp_blocks(g.n, 256);
    const mp_params& P = c->P;
    const T alpha = (T)P.flip_alpha;
    const bool air = t->air;
    uint32_t* cellof = static_cast<uint32_t*>(t->wk[W_CELLOF]);
    uint32_t* flag = static_cast<uint32_t*>(t->wk[W_FLAG]);
    k_ad_cellof<<<nbc, 256, 0, s>>>(g.n, t->order[k], t->off[k], cellof);
    MP_CUDA(c, cudaMemsetAsync(flag, 0, sizeof(uint32_t), s));
    uint8_t* cellbad = static_cast<uint8_t*>(t->wk[W_CBAD]);
    uint8_t* near = static_cast<uint8_t*>(t->wk[W_CNEAR]);
    MP_CUDA(c, cudaMemsetAsync(cellbad, 0, (size_t)g.n, s));
    k_ad_cell_mismatch<T><<<nbp, 256, 0, s>>>(g, R.np, x, cellof, flag, cellbad);
    k_ad_advect_adj<T><<<nbp, 256, 0, s>>>(g, R.np, x, I.vg, (T)P.dt, xb, vb, R.a(W_VGB));
    k_ad_g2p_adj_p<T><<<nbp, 256, 0, s>>>(g, R.np, t->order[k], x, I.uf, I.du, alpha, R.a(W_VGB), R.a(W_VAB), xb,
                                          air ? t->phase : nullptr, I.ufa, I.dua);
    if (air) {
        // the face side per phase: each field gathers only its own particles
        k_ad_slot_gather<T><<<nbp, 256, 0, s>>>(R.np, t->order[k], x, R.a(W_VGB), nullptr, R.a(W_S4A), R.a(W_S4B));
        k_ad_slot_gather_ph<T><<<nbp, 256, 0, s>>>(R.np, t->order[k], R.a(W_VGB), t->phase, 0, R.a(W_S4B));
        k_ad_slot_gather_ph<T><<<nbp, 256, 0, s>>>(R.np, t->order[k], R.a(W_VGB), t->phase, 1, R.a(W_S4C));
    } else {
        k_ad_slot_gather<T><<<nbp, 256, 0, s>>>(R.np, t->order[k], x, R.a(W_VGB), nullptr, R.a(W_S4A), R.a(W_S4B));
    }
    MP_CHECK_LAUNCH(c);
    uint32_t anybad = 1;
    MP_CUDA(c, cudaMemcpyAsync(&anybad, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    // the faces near a particle whose replay cell is not its recorded one take
    // the wider window (none when no particle changed cell: cellbad is zero)
    const uint8_t* nearp = cellbad;
    if (anybad) {
        k_ad_dilate<<<nbc, 256, 0, s>>>(g, cellbad, near);
        nearp = near;
    }
    // q = I^T vgbar on B0 (A0 for the air faces); ufbar = q, uoldbar = -cdu q
    const int nbw = mp_blocks(make_tiles(g.NX + 1, g.NY + 1, g.NZ + 1).threads(), 256);
    k_ad_g2p_adj_w<T><<<nbw, 256, 0, s>>>(g, t->off[k], R.a(W_S4A), R.a(W_S4B), R.f(W_B0), nullptr, nearp);
    if (air) {
        // the air cell mask of this step, from its forward replay
        const uint8_t* airc = static_cast<const uint8_t*>(t->wk[W_AIRC]);
        k_ad_g2p_adj_w<T><<<nbw, 256, 0, s>>>(g, t->off[k], R.a(W_S4A), R.a(W_S4C), R.f(W_A0), airc, nearp);
    }
    const T cdu = alpha == (T)1 ? (T)1 : alpha;
    // wall rules then the two passes, transposed (B0 -> B1 -> T0 -> B1); the
    // ceiling rule's decision reads the rule's output, equal to its input
    // wherever the decision matters
    k_ad_bound_adj<T><<<nbf, 256, 0, s>>>(g, R.f(W_B0), R.f(W_B1), I.uf, t->mark[k]);
    k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_B1), R.f(W_T0), I.sel, I.sw);
    k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_T0), R.f(W_B1), I.sel, I.sw);
    if (air) {
        k_ad_bound_adj<T><<<nbf, 256, 0, s>>>(g, R.f(W_A0), R.f(W_A1), I.ufa, t->mark[k]);
        k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_A1), R.f(W_T0), I.sela, I.swa);
        k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_T0), R.f(W_A1), I.sela, I.swa);
    }
    // projection: ubar_e = ubar_proj + D^T L^-1 (-G^T ubar_proj), with both
    // phases' fields taking the one pressure gradient
    if (air) k_ad_pbar2<T><<<nbc, 256, 0, s>>>(g, t->mark[k], R.f(W_B1), R.f(W_A1), R.a(W_CB));
    else k_ad_pbar<T><<<nbc, 256, 0, s>>>(g, t->mark[k], R.f(W_B1), R.a(W_CB));
    MP_CHECK_LAUNCH(c);
    int mode, maxit; float tol; cg_tol_of<T>(c, mode, tol, maxit);
    int it = 0; double res = 0;
    int st = k_cg_solve(c, t->mark[k], R.a(W_CQ), R.a(W_CB), maxit, mode, tol, &it, &res);
    if (st != MP_OK && st != MP_ERR_NOCONVERGE) return st;
    if (air) {
        k_ad_divT2<T><<<nbf, 256, 0, s>>>(g, t->mark[k], t->lsm[k], R.a(W_CQ), R.f(W_B1), R.f(W_A1), R.f(W_B2),
                                          R.f(W_A2));
        k_ad_bound_adj<T><<<nbf, 256, 0, s>>>(g, R.f(W_A2), R.f(W_A1), I.uea, t->mark[k]);
        k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_A1), R.f(W_A2), I.sela, I.swa);
        k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_A2), R.f(W_A1), I.sela, I.swa);
        k_ad_axpy<T><<<nbf, 256, 0, s>>>(R.nf, -cdu, R.a(W_A0), R.a(W_A1));
    } else {
        k_ad_divT<T><<<nbf, 256, 0, s>>>(g, R.a(W_CQ), R.f(W_B1), R.f(W_B2));
    }
    k_ad_bound_adj<T><<<nbf, 256, 0, s>>>(g, R.f(W_B2), R.f(W_B1), I.ue, t->mark[k]);
    k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_B1), R.f(W_B2), I.sel, I.sw);
    k_ad_sweepu_adj_s<T><<<nbf, 256, 0, s>>>(g, R.f(W_B2), R.f(W_B1), I.sel, I.sw);
    // upbar = that + uoldbar
    k_ad_axpy<T><<<nbf, 256, 0, s>>>(R.nf, -cdu, R.a(W_B0), R.a(W_B1));
    // splat transposes (vabar += ..., xbar += ...), with ub/W per face on T0
    // (A2 for the air faces)
    k_ad_ub_over_w<T><<<nbf, 256, 0, s>>>(R.nf, R.a(W_B1), I.wt.x, R.a(W_T0));
    k_ad_p2g_adj<T, 0><<<nbp, 256, 0, s>>>(g, R.np, t->order[k], x, I.va, air ? t->mass_w : t->mass, cellof, I.up,
                                           R.f(W_T0), R.a(W_VAB), xb);
    if (air) {
        k_ad_ub_over_w<T><<<nbf, 256, 0, s>>>(R.nf, R.a(W_A1), I.wta.x, R.a(W_A2));
        k_ad_p2g_adj<T, 1><<<nbp, 256, 0, s>>>(g, R.np, t->order[k], x, I.va, t->mass_a, cellof, I.upa, R.f(W_A2),
                                               R.a(W_VAB), xb);
    }
    // external forces: vbar = dva/dv^T vabar
    if (air)
        k_ad_forces_adj<T><<<nbp, 256, 0, s>>>(R.np, t->phase, v, R.a(W_VAB), vb, (T)P.dt * (T)P.gravity_z,
                                               (T)P.buoyance_rate_air, (T)P.bubble_max_vel);
    else k_ad_copy<T><<<nbp, 256, 0, s>>>(3LL * R.np, R.a(W_VAB), vb);
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

template <class T> static int adj_loss_fwd(const Replay<T>& R, const T* x, double* loss_host) {
    MpCtx* c = R.c; AdjTape* t = R.t;
    k_ad_phi<T><<<mp_blocks(R.g.n, 256), 256, 0, c->stream>>>(R.g, x, t->nearest, R.a(W_PHI));
    double* sv = static_cast<double*>(t->wk[W_SV]);
    double* dl = static_cast<double*>(t->wk[W_LOSS]);
    k_ad_loss<T><<<1, 256, 0, c->stream>>>(R.g, t->nsamples, t->samples, R.a(W_PHI), sv, dl);
    MP_CHECK_LAUNCH(c);
    MP_CUDA(c, cudaMemcpyAsync(loss_host, dl, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

// What one replay computes. Primal inputs and outputs and all cotangents are
// device arrays of doubles, xyz per particle in recording order.
struct AdjIO {
    const double* x0 = nullptr;   // initial positions (NULL: the recorded ones)
    const double* v0 = nullptr;   // initial velocities (NULL: the recorded ones)
    const double* T0 = nullptr;   // initial temperatures, one per particle (heat recorded; NULL: the recorded ones)
    double* xT = nullptr;         // final positions (NULL: not wanted)
    double* vT = nullptr;         // final velocities
    double* TT = nullptr;         // final temperatures
    bool loss = false;            // evaluate the level-set loss; with `reverse`, seed the sweep with its cotangent
    double* loss_out = nullptr;
    const double* xTb = nullptr;  // otherwise the seed: cotangents of the final positions / velocities /
    const double* vTb = nullptr;  // temperatures (NULL: 0)
    const double* TTb = nullptr;
    bool reverse = false;         // run the reverse sweep
    double* x0b = nullptr;        // cotangents of the initial positions / velocities / temperatures
    double* v0b = nullptr;        // (NULL: not wanted)
    double* T0b = nullptr;
};

// bit patterns of a and b differ somewhere (*flag raised); T float
template <class T>
__global__ void k_ad_differ_t(long long n, const T* __restrict__ a, const float* __restrict__ b, uint32_t* flag) {
    MP_GRID_LOOP(i, n) {
        const bool d = __float_as_uint((float)a[i]) != __float_as_uint(b[i]);
        if (__any_sync(__activemask(), d) && (threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1))
            atomicOr(flag, 1u);
    }
}

template <class T> static int adj_run(MpCtx* c, const AdjIO& io, bool allow_engine = true);
template <class T> static int adj_run(MpCtx* c, const AdjIO& io, bool allow_engine) {
    AdjTape* t = c->adj;
    if (!t) { c->err = "adjoint: record first (mp_adj_record)"; return MP_ERR_STATE; }
    if (io.loss && !t->nsamples) { c->err = "adjoint: no target samples (mp_adj_set_targets)"; return MP_ERR_STATE; }
    MP_TRY(adj_work<T>(c, t));
    Replay<T> R{c, t, c->G, (long long)c->G.nfx + c->G.nfy + c->G.nfz, t->np};
    cudaStream_t s = c->stream;
    const long long np3 = 3LL * t->np;
    const int nb3 = mp_blocks(np3, 256);
    // forward over all steps, keeping the segment starts (slot 0 holds each
    // step's intermediates in passing)
    T* x = R.a(W_X); T* v = R.a(W_V); T* xn = R.a(W_XN); T* vn = R.a(W_VN);
    if (io.x0) k_ad_from_double<T><<<nb3, 256, 0, s>>>(np3, io.x0, x);
    else k_ad_from_float<T><<<nb3, 256, 0, s>>>(np3, t->x0, x);
    if (io.v0) k_ad_from_double<T><<<nb3, 256, 0, s>>>(np3, io.v0, v);
    else k_ad_from_float<T><<<nb3, 256, 0, s>>>(np3, t->v0, v);
    const int nb1 = mp_blocks(t->np, 256);
    T* Tc = t->heat ? R.a(W_T) : nullptr; T* Tn = t->heat ? R.a(W_TN) : nullptr;
    if (t->heat) {
        if (io.T0) k_ad_from_double<T><<<nb1, 256, 0, s>>>(t->np, io.T0, Tc);
        else k_ad_from_float<T><<<nb1, 256, 0, s>>>(t->np, t->T0, Tc);
    }
    MP_CHECK_LAUNCH(c);
    const int E = t->every, nseg = (t->nsteps + E - 1) / E;
    std::vector<T*> ckx(nseg), ckv(nseg), ckT(nseg, nullptr);
    const Inter<T> scratch = R.inter(0);
    // for a gradient at the recorded inputs, the engine's states stand in for
    // the first replay: the segment starts and the final state come from the
    // recording, each step's pressure is the engine's, and the splats are
    // formed when a segment is replayed, which is checked against the
    // engine's state at its end
    const bool engine = allow_engine && io.reverse && sizeof(T) == sizeof(float) && t->eng_xs && !io.x0 && !io.v0 &&
                        !t->heat;
    const size_t sn = (size_t)c->G.n;
    if (engine) {
        for (int sgi = 0; sgi < nseg; sgi++) {
            ckx[sgi] = R.seg_x(sgi); ckv[sgi] = R.seg_v(sgi);
            if (sgi == 0) {
                MP_CUDA(c, cudaMemcpyAsync(ckx[0], x, sizeof(T) * np3, cudaMemcpyDeviceToDevice, s));
                MP_CUDA(c, cudaMemcpyAsync(ckv[0], v, sizeof(T) * np3, cudaMemcpyDeviceToDevice, s));
            } else {
                k_ad_from_float<T><<<nb3, 256, 0, s>>>(np3, t->eng_xs + (size_t)np3 * (sgi - 1), ckx[sgi]);
                k_ad_from_float<T><<<nb3, 256, 0, s>>>(np3, t->eng_vs + (size_t)np3 * (sgi - 1), ckv[sgi]);
            }
        }
        k_ad_from_float<T><<<nb3, 256, 0, s>>>(np3, t->eng_xs + (size_t)np3 * (nseg - 1), x);
        k_ad_from_float<T><<<nb3, 256, 0, s>>>(np3, t->eng_vs + (size_t)np3 * (nseg - 1), v);
        for (int k = 0; k < t->nsteps; k++)
            MP_CUDA(c, cudaMemcpyAsync(R.a(W_PST) + (size_t)k * sn, t->eng_p[k], sizeof(float) * sn,
                                       cudaMemcpyDeviceToDevice, s));
        MP_CHECK_LAUNCH(c);
    }
    for (int k = 0; k < t->nsteps && !engine; k++) {
        if (k % E == 0) {
            int sgi = k / E;
            ckx[sgi] = R.seg_x(sgi); ckv[sgi] = R.seg_v(sgi);
            MP_CUDA(c, cudaMemcpyAsync(ckx[sgi], x, sizeof(T) * np3, cudaMemcpyDeviceToDevice, s));
            MP_CUDA(c, cudaMemcpyAsync(ckv[sgi], v, sizeof(T) * np3, cudaMemcpyDeviceToDevice, s));
            if (t->heat) {
                ckT[sgi] = R.seg_T(sgi);
                MP_CUDA(c, cudaMemcpyAsync(ckT[sgi], Tc, sizeof(T) * t->np, cudaMemcpyDeviceToDevice, s));
            }
        }
        MP_TRY(fwd_step<T>(R, k, x, v, xn, vn, Tc, Tn, scratch, true, true));
        std::swap(x, xn); std::swap(v, vn); std::swap(Tc, Tn);
    }
    if (io.xT) k_ad_to_double<T><<<nb3, 256, 0, s>>>(np3, x, io.xT);
    if (io.vT) k_ad_to_double<T><<<nb3, 256, 0, s>>>(np3, v, io.vT);
    if (io.TT && t->heat) k_ad_to_double<T><<<nb1, 256, 0, s>>>(t->np, Tc, io.TT);
    MP_CHECK_LAUNCH(c);
    if (io.loss) {
        double L = 0;
        MP_TRY(adj_loss_fwd<T>(R, x, &L));
        if (io.loss_out) *io.loss_out = L;
    }
    if (!io.reverse) {
        MP_CUDA(c, cudaStreamSynchronize(s));
        return MP_OK;
    }
    // the seed of the reverse sweep
    T* xb = R.a(W_XB); T* vb = R.a(W_VB);
    if (io.loss) {
        k_ad_phibar<T><<<mp_blocks(c->G.n, 256), 256, 0, s>>>(c->G, t->samples, t->s_off,
                                                              static_cast<double*>(t->wk[W_SV]), R.a(W_CQ));
        k_ad_phi_x<T><<<mp_blocks(t->np, 256), 256, 0, s>>>(c->G, t->np, x, t->nearest, R.a(W_CQ), xb);
        MP_CUDA(c, cudaMemsetAsync(vb, 0, sizeof(T) * np3, s));
    } else {
        if (io.xTb) k_ad_from_double<T><<<nb3, 256, 0, s>>>(np3, io.xTb, xb);
        else MP_CUDA(c, cudaMemsetAsync(xb, 0, sizeof(T) * np3, s));
        if (io.vTb) k_ad_from_double<T><<<nb3, 256, 0, s>>>(np3, io.vTb, vb);
        else MP_CUDA(c, cudaMemsetAsync(vb, 0, sizeof(T) * np3, s));
    }
    T* Tb = t->heat ? R.a(W_TB) : nullptr;
    if (t->heat) {
        if (!io.loss && io.TTb) k_ad_from_double<T><<<nb1, 256, 0, s>>>(t->np, io.TTb, Tb);
        else MP_CUDA(c, cudaMemsetAsync(Tb, 0, sizeof(T) * t->np, s));
    }
    MP_CHECK_LAUNCH(c);
    // reverse sweep, segment by segment: the segment is replayed from its
    // start, each step's state kept in its slot, then the steps are reversed
    for (int sg = nseg - 1; sg >= 0; sg--) {
        const int k0 = sg * E, len = std::min(t->nsteps, k0 + E) - k0;
        MP_CUDA(c, cudaMemcpyAsync(R.seg_x(nseg), ckx[sg], sizeof(T) * np3, cudaMemcpyDeviceToDevice, s));
        MP_CUDA(c, cudaMemcpyAsync(R.seg_v(nseg), ckv[sg], sizeof(T) * np3, cudaMemcpyDeviceToDevice, s));
        if (t->heat)
            MP_CUDA(c, cudaMemcpyAsync(R.seg_T(nseg), ckT[sg], sizeof(T) * t->np, cudaMemcpyDeviceToDevice, s));
        auto xs = [&](int j) { return j < len ? R.seg_x(nseg + j) : R.a(W_XN); };
        auto vs = [&](int j) { return j < len ? R.seg_v(nseg + j) : R.a(W_VN); };
        auto Ts = [&](int j) -> T* { return !t->heat ? nullptr : (j < len ? R.seg_T(nseg + j) : R.a(W_TN)); };
        // one step's intermediates are kept at a time: the states of the
        // segment first, then each step is replayed again (its pressure from
        // the first replay, so no solve) just before its transpose. The replay
        // is deterministic, so it rewrites the same next state.
        const Inter<T> I = R.inter(0);
        for (int j = 0; j < len; j++)
            MP_TRY(fwd_step<T>(R, k0 + j, xs(j), vs(j), xs(j + 1), vs(j + 1), Ts(j), Ts(j + 1), I, false, engine));
        if (engine) {
            // the segment's replay must end on the engine's state; if it does
            // not, the gradient is taken again with the first replay
            uint32_t* flag = static_cast<uint32_t*>(t->wk[W_FLAG]) + 2;
            MP_CUDA(c, cudaMemsetAsync(flag, 0, sizeof(uint32_t), s));
            k_ad_differ_t<T><<<nb3, 256, 0, s>>>(np3, xs(len), t->eng_xs + (size_t)np3 * sg, flag);
            k_ad_differ_t<T><<<nb3, 256, 0, s>>>(np3, vs(len), t->eng_vs + (size_t)np3 * sg, flag);
            uint32_t differ = 1;
            MP_CUDA(c, cudaMemcpyAsync(&differ, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            MP_CUDA(c, cudaStreamSynchronize(s));
            if (differ) return adj_run<T>(c, io, false);
        }
        for (int j = len - 1; j >= 0; j--) {
            if (j < len - 1)
                MP_TRY(fwd_step<T>(R, k0 + j, xs(j), vs(j), xs(j + 1), vs(j + 1), Ts(j), Ts(j + 1), I, false, false));
            MP_TRY(adj_step<T>(R, k0 + j, xs(j), vs(j), xs(j + 1), Ts(j), I, xb, vb, Tb));
        }
    }
    c->work[engine ? MP_WC_ADJ_ENGINE : MP_WC_ADJ_REPLAY]++;
    if (io.v0b) k_ad_to_double<T><<<nb3, 256, 0, s>>>(np3, vb, io.v0b);
    if (io.x0b) k_ad_to_double<T><<<nb3, 256, 0, s>>>(np3, xb, io.x0b);
    if (io.T0b && t->heat) k_ad_to_double<T><<<nb1, 256, 0, s>>>(t->np, Tb, io.T0b);
    MP_CHECK_LAUNCH(c);
    MP_CUDA(c, cudaStreamSynchronize(s));
    return MP_OK;
}

// the level-set loss of given final positions and its cotangent
template <class T> static int adj_ls_loss(MpCtx* c, const double* xT, double* loss, double* xTb) {
    AdjTape* t = c->adj;
    if (!t) { c->err = "adjoint: record first (mp_adj_record)"; return MP_ERR_STATE; }
    if (!t->nsamples) { c->err = "adjoint: no target samples (mp_adj_set_targets)"; return MP_ERR_STATE; }
    MP_TRY(adj_work<T>(c, t));
    Replay<T> R{c, t, c->G, (long long)c->G.nfx + c->G.nfy + c->G.nfz, t->np};
    cudaStream_t s = c->stream;
    const long long np3 = 3LL * t->np;
    const int nb3 = mp_blocks(np3, 256);
    T* x = R.a(W_X);
    k_ad_from_double<T><<<nb3, 256, 0, s>>>(np3, xT, x);
    MP_CHECK_LAUNCH(c);
    double L = 0;
    MP_TRY(adj_loss_fwd<T>(R, x, &L));
    if (loss) *loss = L;
    if (xTb) {
        T* xb = R.a(W_XB);
        k_ad_phibar<T><<<mp_blocks(c->G.n, 256), 256, 0, s>>>(c->G, t->samples, t->s_off,
                                                              static_cast<double*>(t->wk[W_SV]), R.a(W_CQ));
        k_ad_phi_x<T><<<mp_blocks(t->np, 256), 256, 0, s>>>(c->G, t->np, x, t->nearest, R.a(W_CQ), xb);
        k_ad_to_double<T><<<nb3, 256, 0, s>>>(np3, xb, xTb);
        MP_CHECK_LAUNCH(c);
        MP_CUDA(c, cudaStreamSynchronize(s));
    }
    return MP_OK;
}

int k_adj_run(MpCtx* c, int precision, const double* v0, double* grad, double* loss) {
    AdjIO io;
    io.v0 = v0; io.loss = true; io.loss_out = loss; io.reverse = grad != nullptr; io.v0b = grad;
    if (precision == MP_PREC_FP64) return adj_run<double>(c, io);
    return adj_run<float>(c, io);
}
int k_adj_forward(MpCtx* c, int precision, const mp_grad* in, mp_grad* out) {
    AdjIO io;
    if (in) { io.x0 = in->pos; io.v0 = in->vel; io.T0 = in->temp; }
    io.xT = out->pos; io.vT = out->vel; io.TT = out->temp;
    if (precision == MP_PREC_FP64) return adj_run<double>(c, io);
    return adj_run<float>(c, io);
}
int k_adj_vjp(MpCtx* c, int precision, const mp_grad* in, const mp_grad* dout, mp_grad* din) {
    AdjIO io;
    if (in) { io.x0 = in->pos; io.v0 = in->vel; io.T0 = in->temp; }
    io.xTb = dout->pos; io.vTb = dout->vel; io.TTb = dout->temp;
    io.reverse = true;
    io.x0b = din->pos; io.v0b = din->vel; io.T0b = din->temp;
    if (precision == MP_PREC_FP64) return adj_run<double>(c, io);
    return adj_run<float>(c, io);
}
int k_adj_ls_loss(MpCtx* c, int precision, const double* xT, double* loss, double* xTb) {
    if (precision == MP_PREC_FP64) return adj_ls_loss<double>(c, xT, loss, xTb);
    return adj_ls_loss<float>(c, xT, loss, xTb);
}
int k_adj_order(MpCtx* c, uint32_t* ids) {
    if (!c->adj) { c->err = "adjoint: record first"; return MP_ERR_STATE; }
    if (c->np() != c->adj->np) { c->err = "adjoint: the particles changed since the recording"; return MP_ERR_STATE; }
    MP_CUDA(c, cudaMemcpyAsync(ids, c->adj->ids, sizeof(uint32_t) * (size_t)c->adj->np, cudaMemcpyDeviceToDevice,
                               c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}
int k_adj_np(MpCtx* c, int* np, int* nsteps) {
    if (!c->adj) { c->err = "adjoint: record first"; return MP_ERR_STATE; }
    if (np) *np = c->adj->np;
    if (nsteps) *nsteps = c->adj->nsteps;
    return MP_OK;
}
