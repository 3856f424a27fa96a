// scene.cpp — scene and parameter set-up for the five benchmark
// configurations; the drop-in for the per-scene branches of
// cspray::initparam (Multiphase/Multiphase/spray.cpp:83-547),
// initparticle_solidCoupling (spray.cu:395-484), initTemperature /
// initSolubility (spray.cu:1989-1999) and initSeedCell (spray.cu:2907-2933).
//
// The reference seeds a regular lattice at half-cell spacing; the
// configurations ask for 8 particles per cell jittered inside the cell, so
// each cell is split into 2x2x2 sub-cells and each sub-cell gets one particle
// at a uniform position inside it. Random numbers come from SplitMix64
// (Steele, Lea, Flood 2014) keyed by (seed, stream, counter), so every
// implementation given the same seed sees the same inputs. The reference's
// cuRAND table (spray.cu:180-190) becomes an input table drawn the same way.
// Temperatures are normalised so that the boiling point is 1.0; the
// reference's Kelvin constants are rescaled by 373.15 K where they enter
// (solubility exponent, T0), which leaves its formulas unchanged.
#include "../../../include/mp.h"
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// uniform in [0,1) from (seed, stream, counter)
inline float u01(uint64_t seed, uint64_t stream, uint64_t ctr) {
    uint64_t k = splitmix64(seed ^ splitmix64(stream * 0xD1B54A32D192ED03ull + ctr));
    return (float)(k >> 40) * (1.0f / 16777216.0f);
}
inline float gauss(uint64_t seed, uint64_t stream, uint64_t ctr) {   // Box-Muller
    float a = u01(seed, stream, 2 * ctr), b = u01(seed, stream, 2 * ctr + 1);
    float r = sqrtf(-2.0f * logf(1.0f - a));
    return r * cosf(6.28318530718f * b);
}
enum { ST_JITTER = 1, ST_TEMP = 2, ST_VEL = 3, ST_TABLE = 4, ST_SEEDS = 5, ST_BUBBLE = 6 };

const float kKelvinScale = 373.15f;   // boiling point of the reference scenes

struct Bubble { float x, y, z, r; };

// 200 non-overlapping bubbles, radius U[0.01, 0.04], inside the liquid (rejection sampling)
std::vector<Bubble> column_bubbles(uint64_t seed, float level, float h) {
    std::vector<Bubble> b;
    uint64_t ctr = 0;
    while (b.size() < 200 && ctr < 4000000) {
        float r = 0.01f + 0.03f * u01(seed, ST_BUBBLE, ctr++);
        float lo = 2 * h + r, hi = 1.0f - 2 * h - r;
        float x = lo + (hi - lo) * u01(seed, ST_BUBBLE, ctr++);
        float y = lo + (hi - lo) * u01(seed, ST_BUBBLE, ctr++);
        float z = lo + (level - 2 * h - r - lo) * u01(seed, ST_BUBBLE, ctr++);
        bool ok = true;
        for (const Bubble& o : b) {
            float dx = x - o.x, dy = y - o.y, dz = z - o.z;
            if (sqrtf(dx * dx + dy * dy + dz * dz) < r + o.r + h) { ok = false; break; }
        }
        if (ok) b.push_back({x, y, z, r});
    }
    return b;
}

float liquid_level(int config) {
    switch (config) {
    case 1: return 0.6f;
    case 2: return 0.4f;
    case 3: return 0.5f;
    case 4: return 0.6f;
    default: return 0.8f;
    }
}
int default_n(int config) {
    switch (config) {
    case 1: return 32;
    case 2: return 64;
    case 3: return 128;
    case 4: return 64;
    default: return 256;
    }
}

}  // namespace

extern "C" int mp_scene_params(int config, int n, mp_params* p) {
    if (!p || config < 1 || config > 5) return MP_ERR_ARG;
    if (n == 0) n = default_n(config);
    if (n < 8) return MP_ERR_ARG;
    float level = liquid_level(config);
    // capacity: 8 per cell of the liquid region, plus room for generated gas
    long long cells = (long long)(n - 2) * (n - 2) * (long long)std::min(n - 2, (int)ceilf(level * n) + 1);
    long long cap = 8 * cells + cells / 4 + 4096;
    int rc = mp_params_default(p, n, n, n, (int)std::min(cap, 0x7ffffff0LL));
    if (rc) return rc;
    p->cellsize = 1.0f / (float)n;
    p->samplespace = 0.5f * p->cellsize;
    p->dt = 1.0f / 240.0f;
    p->flip_alpha = 0.95f;
    p->cg_tol_mode = MP_TOL_REL;
    p->cg_tol = 1e-6f;
    p->cg_max_iter = 2000;
    p->cg_true_residual_every = 0;
    p->density_ratio = 1000.0f;
    p->surfacetension_sigma = 0.0f;
    switch (config) {
    case 1:   // rising air bubble (MULTIBUBBLE switches, spray.cpp:191-214)
        p->scene = MP_SCENE_MULTIBUBBLE;
        p->mc_every = 2;
        break;
    case 2:   // pool boiling (BOILING, spray.cpp:114-151)
        p->scene = MP_SCENE_BOILING;
        p->b_gen_gas = 1; p->b_heat_trans = 1; p->b_add_heat_bottom = 0; p->b_extend_heat_to_boundary = 1;
        p->b_fixed_heat = 1;
        p->boiling_point = 1.0f;
        p->melting_point = 273.15f / kKelvinScale;
        p->temperature0 = 273.15f / kKelvinScale;
        p->solubility_coef = 1018.9f / kKelvinScale;
        p->default_temperature = 0.95f; p->default_liquid_T = 0.95f; p->default_solid_T = 0.7f;
        p->liquid_heat_th = 0.5f;
        p->heatalpha_fluid = 0.18f; p->heatalpha_air = 0.08f;
        p->vapor_gen_rate = 0.01f;
        p->init_dissolve_gas_rate = 0.95f; p->init_gas_rate = 0.88f;
        p->drag_param_solo = 5; p->drag_param_grid = 0.12f;
        p->mc_every = 2;
        break;
    case 3:   // melting / freezing (MELTING, spray.cpp:215-240, with FREEZING's phase switch)
        p->scene = MP_SCENE_MELTING;
        p->b_solid = 1; p->b_melt = 1; p->b_freeze = 1; p->b_fix_solid = 1;
        p->b_heat_trans = 1; p->b_add_heat_bottom = 0; p->b_extend_heat_to_boundary = 1; p->b_fixed_heat = 1;
        p->melting_point = 1.0f; p->boiling_point = 10.0f;
        p->temperature0 = 273.15f / kKelvinScale;
        p->solubility_coef = 1018.9f / kKelvinScale;
        p->default_temperature = 1.15f; p->default_liquid_T = 1.15f; p->default_solid_T = 0.7f;
        p->liquid_heat_th = 0.05f;
        p->heatalpha_fluid = 0.01f; p->heatalpha_solid = 0.01f; p->heatalpha_air = 0.01f; p->heatalpha_vacuum = 0.0001f;
        p->mc_every = 2;
        break;
    case 4:   // differentiable dam break: the FLUID-only program the adjoint covers
        p->scene = MP_SCENE_DAMBREAK;
        p->b_run_mc = 0;
        p->b_correct_position = 0;
        break;
    case 5:   // bubble column at scale, marching cubes every step
        p->scene = MP_SCENE_MULTIBUBBLE;
        p->mc_every = 1;
        p->cg_max_iter = 3000;
        // The solo-air SPH force (enforceForceSoloAirP) is explicit and its
        // viscous part grows as 1/h^2, so a fixed step that is stable on 64^3
        // is not on finer grids: at 256^3 and 1/240 the bubbles' particles
        // reach hundreds of units/s within ten steps. The step shrinks with
        // h^2 from 1/240 at 64^3 (1/3840 at 256^3).
        if (n > 64) p->dt = (1.0f / 240.0f) * (64.0f / (float)n) * (64.0f / (float)n);
        // hundreds of bubbles: the three meshes are far larger than a few
        // surface layers of the 2x grid
        p->mc_max_verts = 64000000; p->mc_max_tris = 128000000;
        break;
    }
    return mp_params_derive(p);
}

extern "C" int mp_scene_particles(const mp_params* p, int config, uint64_t seed, int cap, int* nout, float* pos3,
                                  float* vel3, int8_t* flag, float* mass, float* temp, float* lheat, float* sol,
                                  float* gas) {
    if (!p || !nout || config < 1 || config > 5) return MP_ERR_ARG;
    const int N = p->nx;
    const float h = p->cellsize;
    const float level = liquid_level(config);
    std::vector<Bubble> bubbles;
    if (config == 1) bubbles.push_back({0.5f, 0.5f, 0.25f, 0.15f});
    if (config == 5) bubbles = column_bubbles(seed, level, h);
    const float sx = 0.5f, sy = 0.5f, sz = 0.3f, sr = 0.2f;   // solid sphere of configuration 3
    long long cnt = 0;
    for (int i = 1; i <= p->nx - 2; i++)
        for (int j = 1; j <= p->ny - 2; j++)
            for (int k = 1; k <= p->nz - 2; k++) {
                if ((float)k * h >= level && !(config == 3 && (float)k * h < sz + sr)) continue;
                for (int q = 0; q < 8; q++) {
                    long long ctr = (((long long)i * N + j) * N + k) * 8 + q;
                    // jitter kept 0.1% away from the sub-cell faces so that rounding
                    // never moves a particle into the neighbouring cell
                    float ux = 0.001f + 0.998f * u01(seed, ST_JITTER, 3 * ctr),
                          uy = 0.001f + 0.998f * u01(seed, ST_JITTER, 3 * ctr + 1),
                          uz = 0.001f + 0.998f * u01(seed, ST_JITTER, 3 * ctr + 2);
                    float x = ((float)i + 0.5f * ((float)(q & 1) + ux)) * h;
                    float y = ((float)j + 0.5f * ((float)((q >> 1) & 1) + uy)) * h;
                    float z = ((float)k + 0.5f * ((float)((q >> 2) & 1) + uz)) * h;
                    bool in_liquid = z < level && (config != 4 || x < 0.4f);
                    bool in_solid = false;
                    if (config == 3) {
                        float dx = x - sx, dy = y - sy, dz = z - sz;
                        in_solid = sqrtf(dx * dx + dy * dy + dz * dz) < sr;
                    }
                    if (!in_liquid && !in_solid) continue;
                    int8_t f = MP_TYPEFLUID;
                    for (const Bubble& b : bubbles) {
                        float dx = x - b.x, dy = y - b.y, dz = z - b.z;
                        if (sqrtf(dx * dx + dy * dy + dz * dz) < b.r) { f = MP_TYPEAIR; break; }
                    }
                    if (in_solid) f = MP_TYPESOLID;
                    if (pos3) {
                        if (cnt >= cap) return MP_ERR_CAPACITY;
                        pos3[3 * cnt] = x; pos3[3 * cnt + 1] = y; pos3[3 * cnt + 2] = z;
                        float vx = 0, vy = 0, vz = 0;
                        if (config == 4) {
                            vx = 0.1f * gauss(seed, ST_VEL, 3 * ctr);
                            vy = 0.1f * gauss(seed, ST_VEL, 3 * ctr + 1);
                            vz = 0.1f * gauss(seed, ST_VEL, 3 * ctr + 2);
                        }
                        if (vel3) { vel3[3 * cnt] = vx; vel3[3 * cnt + 1] = vy; vel3[3 * cnt + 2] = vz; }
                        flag[cnt] = f;
                        mass[cnt] = (f == MP_TYPESOLID) ? p->m0 * 0.8f : p->m0;
                        // initHeatParticle / initsolubility_k (spray_k.cu:4681-4717)
                        float T = (f == MP_TYPESOLID) ? p->default_solid_T : p->default_liquid_T;
                        if (config == 2 && f == MP_TYPEFLUID) T = 0.95f + 0.01f * gauss(seed, ST_TEMP, ctr);
                        float L = (f == MP_TYPESOLID) ? 0.0f : p->liquid_heat_th;
                        float so = 0, ga = 0;
                        if (f == MP_TYPEFLUID || f == MP_TYPESOLID) {
                            so = p->init_dissolve_gas_rate * p->airm0 * expf(p->solubility_coef * (1.0f / T - 1.0f / p->temperature0));
                            ga = p->init_gas_rate * so;
                        }
                        if (temp) temp[cnt] = T;
                        if (lheat) lheat[cnt] = L;
                        if (sol) sol[cnt] = so;
                        if (gas) gas[cnt] = ga;
                    }
                    cnt++;
                }
            }
    if (cnt > 0x7fffffffLL) return MP_ERR_CAPACITY;
    *nout = (int)cnt;
    return MP_OK;
}

extern "C" int mp_scene_tables(const mp_params* p, int config, uint64_t seed, float* randfloat, int nrand,
                               int32_t* seeds, int maxseed, int* nseed) {
    if (!p || !randfloat || nrand <= 200 || !nseed) return MP_ERR_ARG;
    for (int q = 0; q < nrand; q++) randfloat[q] = u01(seed, ST_TABLE, q);
    *nseed = 0;
    if (config == 2) {   // 16 nucleation cells on the bottom (initSeedCell: z = 2, x,y in [2, N-3])
        int want = std::min(16, maxseed);
        uint64_t ctr = 0;
        int got = 0;
        while (got < want && ctr < 100000) {
            int x = 2 + (int)(u01(seed, ST_SEEDS, ctr++) * (float)(p->nx - 4));
            int y = 2 + (int)(u01(seed, ST_SEEDS, ctr++) * (float)(p->ny - 4));
            int id = x * p->ny * p->nz + y * p->nz + 2;
            bool dup = false;
            for (int s = 0; s < got; s++) if (seeds[s] == id) dup = true;
            if (!dup) seeds[got++] = id;
        }
        *nseed = got;
    }
    return MP_OK;
}

extern "C" int mp_scene_fixed_heat(const mp_params* p, int config, float* fh) {
    if (!p || !fh) return MP_ERR_ARG;
    int NX = p->nx, NY = p->ny, NZ = p->nz;
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ; k++) {
                float v = MP_UNDEF_TEMPERATURE;
                bool inner = i >= 1 && i < NX - 1 && j >= 1 && j < NY - 1;
                if (config == 2 && inner && k <= 3) v = 1.25f;          // heated bottom wall
                if (config == 3 && inner && k >= NZ - 4) v = 0.6f;      // cold top plate
                fh[(size_t)i * NY * NZ + (size_t)j * NZ + k] = v;
            }
    return MP_OK;
}

// CompPouringParam_Freezing / _Ineraction / _Ineraction2 (spray.cpp:1416-1545):
// the emitter disc(s) as a square lattice in the xy plane, points farther
// than `radius` from the centre dropped; float arithmetic as the reference's
// host code (ipos = centre + (x*ss, y*ss, 0), length(ipos - centre))
extern "C" int mp_scene_pour(int variant, float samplespace, float radius, const float* center, const float* center2,
                             const float* vel, int cap, float* pos3, float* vel3, int* n) {
    if (!center || !vel || !n || cap < 0 || samplespace <= 0 || radius < 0) return MP_ERR_ARG;
    if (variant == MP_POUR_INTERACTION2 && !center2) return MP_ERR_ARG;
    if (variant < MP_POUR_FREEZING || variant > MP_POUR_INTERACTION2) return MP_ERR_ARG;
    const float ss = variant == MP_POUR_FREEZING ? samplespace : samplespace * 2.0f;
    const int num = variant == MP_POUR_FREEZING ? (int)(radius / samplespace) * 3 : (int)(radius / ss);
    int cnt = 0;
    auto disc = [&](const float* c) {
        for (int x = -num; x <= num; x++)
            for (int y = -num; y <= num; y++) {
                float px = c[0] + (float)x * ss, py = c[1] + (float)y * ss, pz = c[2] + 0.0f;
                float dx = px - c[0], dy = py - c[1], dz = pz - c[2];
                if (sqrtf(dx * dx + dy * dy + dz * dz) > radius) continue;
                if (cnt < cap) {
                    if (pos3) { pos3[3 * cnt] = px; pos3[3 * cnt + 1] = py; pos3[3 * cnt + 2] = pz; }
                    if (vel3) { vel3[3 * cnt] = vel[0]; vel3[3 * cnt + 1] = vel[1]; vel3[3 * cnt + 2] = vel[2]; }
                }
                cnt++;
            }
    };
    disc(center);
    if (variant == MP_POUR_INTERACTION2) disc(center2);
    *n = cnt;
    return MP_OK;
}

// ---------------------------------------------------------------------------
// cspray::initparam (spray.cpp:23-626) for the reference's named scenes
// ---------------------------------------------------------------------------
#define MP_TRY_HOST(x)                        \
    do {                                      \
        int rc_ = (x);                        \
        if (rc_ != MP_OK) return rc_;         \
    } while (0)

namespace {
void set3(float* d, float x, float y, float z) { d[0] = x; d[1] = y; d[2] = z; }
// the grid each branch insists on (initparam exits on any other)
bool scene_grid(int scene, int& nx, int& ny, int& nz) {
    switch (scene) {
    case MP_SCENE_DAMBREAK: nx = 32; ny = 32; nz = 32; return true;
    case MP_SCENE_FLUIDSPHERE: nx = 24; ny = 24; nz = 96; return true;
    case MP_SCENE_BOILING: nx = 64; ny = 64; nz = 64; return true;
    case MP_SCENE_BOILING_HIGHRES: nx = 128; ny = 128; nz = 96; return true;
    case MP_SCENE_MULTIBUBBLE: nx = 32; ny = 32; nz = 64; return true;
    case MP_SCENE_MELTING: case MP_SCENE_MELTINGPOUR: case MP_SCENE_FREEZING: nx = 64; ny = 64; nz = 64; return true;
    case MP_SCENE_INTERACTION: case MP_SCENE_MELTANDBOIL: nx = 64; ny = 48; nz = 64; return true;
    case MP_SCENE_INTERACTION_HIGHRES: nx = 96; ny = 64; nz = 96; return true;
    case MP_SCENE_MELTANDBOIL_HIGHRES: nx = 96; ny = 96; nz = 96; return true;
    case MP_SCENE_ALL: nx = 96; ny = 128; nz = 128; return true;
    case MP_SCENE_HEATTRANSFER: nx = 256; ny = 256; nz = 256; return true;
    default: return false;   // SMOKE has no initparam branch
    }
}
}  // namespace

extern "C" int mp_reference_scene(int scene, mp_params* p, mp_scene_info* info) {
    int nx, ny, nz;
    if (!p || !scene_grid(scene, nx, ny, nz)) return MP_ERR_ARG;
    mp_scene_info I;
    memset(&I, 0, sizeof(I));
    I.nx = nx; I.ny = ny; I.nz = nz;
    I.pour_variant = -1;
    MP_TRY_HOST(mp_params_default(p, nx, ny, nz, 0));
    p->scene = scene;
    // common defaults (spray.cpp:29-78)
    p->mc_every = 2;                                     // outputframeDelta
    p->surfacetension_sigma = 1.0f;
    p->heatalpha_fluid = 0.02f; p->heatalpha_air = 0.008f;
    p->heatalpha_solid = 0.2f; p->heatalpha_vacuum = 0.0001f;
    p->default_temperature = 293.15f; p->temperature0 = 273.15f;
    p->melting_point = 273.15f; p->boiling_point = 373.15f;
    p->drag_param_solo = 10; p->drag_param_grid = 0.05f;
    p->viscosity_sph = 1.8f;
    p->b_solid = 0; p->b_melt = 0; p->b_freeze = 0; p->b_fix_solid = 0;
    p->b_gen_gas = 1; p->b_heat_trans = 1; p->b_add_heat_bottom = 1;
    p->b_extend_heat_to_boundary = 0; p->b_correct_position = 1;
    p->solid_bounce_param = 0.5f;
    p->default_solid_T = 263.15f; p->default_liquid_T = 293.15f; p->liquid_heat_th = 10;
    p->pos_rand_param = 0.1f; p->vel_rand_param = 0.0f;
    p->alpha_temp_trans = 0.0f;
    p->bounce_vel_param = 1.0f; p->bounce_pos_param = 0;
    I.seed_num = 4;
    p->init_dissolve_gas_rate = 1.0f; p->init_gas_rate = 0.7f;
    p->vapor_gen_rate = 0.01f;
    I.t_render_max = 373; I.t_render_min = 273.0f;
    p->b_smooth_mc = 1;
    p->b_run_mc_solid = 1;
    I.frame_max = 1500;
    p->bubble_max_vel = 6.5f;
    p->update_seed_frame_delta = 15;
    p->buoyance_rate_air = 1.25f; p->buoyance_rate_solo = 1.05f;
    p->begin_frame = 0;
    I.output_colored_particles = 1;
    p->gravity_x = 0; p->gravity_y = 0; p->gravity_z = -9.8f;
    p->cellsize = 1.0f / 64;
    p->samplespace = 0.5f * p->cellsize;
    // heatIncreaseBottom is set only by the scenes below; elsewhere 0 here
    p->heat_increase_bottom = 0.0f;
    I.split_num = 1;
    I.sim_mode = MP_SIM_BUBBLE;
    // the scene's branch (spray.cpp:83-547)
    switch (scene) {
    case MP_SCENE_DAMBREAK:
        I.split_num = 1; I.init_fluid_particles = 81920; I.par_num_extra = 0;
        I.sim_mode = MP_SIM_SOLIDCOUPLING;
        set3(I.solid_init_pos, 0.25f, 0.25f, 0.2f);
        p->b_solid = 1;
        break;
    case MP_SCENE_FLUIDSPHERE:
        I.split_num = 2; I.init_fluid_particles = 200000;
        I.sim_mode = MP_SIM_WATER;
        break;
    case MP_SCENE_BOILING:
    case MP_SCENE_BOILING_HIGHRES: {
        const bool hi = scene == MP_SCENE_BOILING_HIGHRES;
        p->b_solid = 0; p->b_melt = 0; p->b_freeze = 0; p->b_gen_gas = 1; p->b_heat_trans = 1;
        p->b_add_heat_bottom = 1; p->b_extend_heat_to_boundary = 1;
        if (hi) { I.split_num = 1; I.init_fluid_particles = 3000000; I.par_num_extra = 1000000; }
        else { I.split_num = 2; I.init_fluid_particles = 800000; }
        set3(I.solid_init_pos, 0.20f, 0.20f, 0.7f);
        p->default_temperature = 293.0f;
        p->vapor_gen_rate = 0.01f;
        p->default_liquid_T = 293.0f;
        p->init_dissolve_gas_rate = 0.95f; p->init_gas_rate = 0.88f;
        p->heat_increase_bottom = hi ? 3.0f : 1.5f;
        p->heatalpha_fluid = 0.18f; p->heatalpha_air = 0.08f;
        I.seed_num = hi ? 3 : 2;
        p->drag_param_solo = 5; p->drag_param_grid = hi ? 0.15f : 0.12f;
        I.t_render_max = 373; I.t_render_min = 273.0f;
        I.frame_max = hi ? 2000 : 1000;
        break;
    }
    case MP_SCENE_MULTIBUBBLE:
        p->b_solid = 0; p->b_melt = 0; p->b_freeze = 0; p->b_fix_solid = 0; p->b_gen_gas = 0; p->b_heat_trans = 0;
        p->b_add_heat_bottom = 0; p->b_extend_heat_to_boundary = 0; p->b_correct_position = 1;
        I.split_num = 2; I.init_fluid_particles = 250000;
        set3(I.solid_init_pos, 0.5f, 0.5f, 0.2f);
        p->surfacetension_sigma = 0;
        break;
    case MP_SCENE_MELTING:
        p->b_melt = 1; p->b_solid = 1; p->b_add_heat_bottom = 0;
        I.split_num = 1; I.init_fluid_particles = 350000;
        set3(I.solid_init_pos, 0.5f, 0.5f, 0.15f);
        p->default_temperature = 293.15f;
        p->heatalpha_fluid = 0.020000f;
        p->heatalpha_air = 0.00008f;
        break;
    case MP_SCENE_MELTINGPOUR:
        p->b_melt = 1; p->b_solid = 1; p->b_fix_solid = 1; p->b_freeze = 0; p->b_gen_gas = 0;
        p->b_add_heat_bottom = 0; p->b_extend_heat_to_boundary = 1;
        I.output_colored_particles = 1;
        I.split_num = 1; I.init_fluid_particles = 0; I.par_num_extra = 100000;
        I.pour_variant = MP_POUR_FREEZING; I.pour_radius = 0.035f;
        set3(I.pour_pos, 0.6f, 0.45f, 0.75f); set3(I.pour_vel, 0.0f, 0.0f, -0.50f);
        set3(I.solid_init_pos, 0.55f, 0.45f, -0.33f);
        p->default_temperature = 273.15f;
        p->melting_point = 265.15f;
        p->default_solid_T = 263.15f; p->default_liquid_T = 293.15f;
        p->heatalpha_fluid = 0.01f; p->heatalpha_air = 05.15f;
        p->bounce_vel_param = 1.3f; p->bounce_pos_param = 1.0f;
        I.t_render_max = 283; I.t_render_min = 263;
        p->alpha_temp_trans = 0.95f;
        break;
    case MP_SCENE_FREEZING:
        p->b_melt = 0; p->b_solid = 1; p->b_fix_solid = 1; p->b_freeze = 1; p->b_correct_position = 1;
        p->b_add_heat_bottom = 1;
        I.output_colored_particles = 1;
        I.split_num = 2; I.init_fluid_particles = 0; I.par_num_extra = 100000;
        I.pour_variant = MP_POUR_FREEZING; I.pour_radius = 0.035f;
        set3(I.pour_pos, 0.60f, 0.48f, 0.75f); set3(I.pour_vel, 0.0f, 0.0f, -0.5f);
        set3(I.solid_init_pos, 0.55f, 0.45f, -0.330f);
        p->default_temperature = 265.15f;
        p->heatalpha_fluid = 0.00001f; p->heatalpha_air = 0.00008f;
        p->default_solid_T = 263.15f; p->default_liquid_T = 280.15f; p->liquid_heat_th = 10;
        p->bounce_vel_param = 1.0f; p->bounce_pos_param = 0.5f;
        p->alpha_temp_trans = 0.98f;
        p->viscosity_sph = 1.2f;
        I.t_render_max = 276; I.t_render_min = 264;
        break;
    case MP_SCENE_INTERACTION:
    case MP_SCENE_INTERACTION_HIGHRES: {
        const bool hi = scene == MP_SCENE_INTERACTION_HIGHRES;
        p->b_melt = 0; p->b_freeze = 0; p->b_fix_solid = hi ? 0 : 1; p->b_solid = 1; p->b_gen_gas = 0;
        p->b_heat_trans = 0; p->b_add_heat_bottom = 0;
        p->b_run_mc_solid = 0;
        I.split_num = 1;
        I.init_fluid_particles = hi ? 1500000 : 280000; I.par_num_extra = hi ? 200000 : 100000;
        if (hi) {
            I.pour_variant = MP_POUR_INTERACTION; I.pour_radius = 0.060f;
            set3(I.pour_pos, 0.25f, 0.25f, 0.05f); set3(I.pour_vel, 0.0f, 0.0f, 1.5f);
            set3(I.solid_init_pos, 0.750f, 0.58f, 0.8f);
        } else {
            I.pour_variant = MP_POUR_INTERACTION2; I.pour_radius = 0.05f;
            set3(I.pour_pos, 0.27f, 0.25f, 0.05f); set3(I.pour_pos2, 0.45f, 0.25f, 0.05f);
            set3(I.pour_vel, 0.0f, 0.0f, 1.1f);
            set3(I.solid_init_pos, 0.41f, 0.28f, 0.2f);
        }
        p->default_temperature = 293.15f;
        p->heatalpha_fluid = 0.0008f; p->heatalpha_air = 0.0008f;
        p->bounce_vel_param = 1.3f; p->bounce_pos_param = 1.0f;
        p->drag_param_solo = 5;
        if (!hi) {
            p->drag_param_grid = 0.08f;
            p->surfacetension_sigma = 0.6f;
            p->begin_frame = 20;
        }
        break;
    }
    case MP_SCENE_MELTANDBOIL:
    case MP_SCENE_MELTANDBOIL_HIGHRES:
    case MP_SCENE_ALL: {
        const bool hi = scene == MP_SCENE_MELTANDBOIL_HIGHRES, all = scene == MP_SCENE_ALL;
        p->b_melt = 1; p->b_freeze = 0; p->b_fix_solid = 1; p->b_solid = 1; p->b_gen_gas = 1; p->b_heat_trans = 1;
        p->b_add_heat_bottom = 1; p->b_extend_heat_to_boundary = 1;
        p->b_run_mc_solid = 1;
        I.split_num = 1;
        I.init_fluid_particles = all ? 3100000 : (hi ? 2400000 : 400000);
        I.par_num_extra = all ? 500000 : (hi ? 600000 : 100000);
        if (all) set3(I.solid_init_pos, 0.8f, 01.30f, 0.2f);
        else if (hi) set3(I.solid_init_pos, 0.850f, 0.68f, 0.65f);
        else set3(I.solid_init_pos, 0.50f, 0.38f, 0.2f);
        p->default_temperature = 293.0f;
        p->boiling_point = 373.15f;
        if (all) { p->heatalpha_fluid = 0.0001f; p->heatalpha_air = 00.0008f; }
        else if (hi) { p->heatalpha_fluid = 0.12f; p->heatalpha_air = 0.08f; }
        else { p->heatalpha_fluid = 0.1f; p->heatalpha_air = 0.08f; }
        p->init_dissolve_gas_rate = 0.95f; p->init_gas_rate = 0.95f;
        if (all) { p->default_solid_T = 223.15f; p->default_liquid_T = 280.15f; p->liquid_heat_th = 10; }
        else if (hi) { p->default_solid_T = 243.15f; p->default_liquid_T = 350.15f; p->liquid_heat_th = 20; }
        else { p->default_solid_T = 233.15f; p->default_liquid_T = 350.15f; p->liquid_heat_th = 20; }
        p->vapor_gen_rate = hi ? 0.017f : 0.015f;
        p->heat_increase_bottom = all ? 50.0f : 1.5f;
        I.seed_num = hi ? 8 : 2;
        I.t_render_max = 373; I.t_render_min = 353;
        p->drag_param_solo = 5; p->drag_param_grid = hi ? 0.08f : 0.03f;
        p->bubble_max_vel = 9.5f;
        p->update_seed_frame_delta = 12;
        p->buoyance_rate_air = 1.45f; p->buoyance_rate_solo = 1.05f;
        I.frame_max = 2000;
        break;
    }
    case MP_SCENE_HEATTRANSFER:
        I.sim_mode = MP_SIM_HEATONLY;
        p->b_extend_heat_to_boundary = 1;
        I.split_num = 0; I.init_fluid_particles = 0; I.par_num_extra = 1;
        I.t_render_max = 100.5f; I.t_render_min = -0.5f;
        p->heatalpha_fluid = 0.0001f; p->heatalpha_air = 0.005f;
        p->heatalpha_solid = 0.015f; p->heatalpha_vacuum = 0.05f;
        break;
    default: return MP_ERR_ARG;
    }
    // after the branches (spray.cpp:570-626)
    p->dt = 0.003f;
    p->gmin_x = p->gmin_y = p->gmin_z = 0.0f;
    p->waterrho = 1000.0f; p->solidrho = 800.0f;
    p->mc_density = 0.5f;
    p->smooth_iters = 5;
    p->correction_spring = 500000.0f;
    p->correction_radius = 0.5f;
    p->par_num_max = I.par_num_extra + I.init_fluid_particles * I.split_num;
    MP_TRY_HOST(mp_params_derive(p));
    if (info) *info = I;
    return MP_OK;
}
