/*
 * mp.h — C ABI of the B200 multiphase FLIP step.
 *
 * One entry point per stage method of the reference's `cspray` class
 * (Multiphase/Multiphase/spray.h:18-389), plus the full time step
 * (`cspray::bubblesim`, spray.cpp:979-1233). Plain C types only: host
 * pointers and sizes, an opaque context, `int` status codes.
 *
 * Layouts follow the reference:
 *   cells  idx = i*NY*NZ + j*NZ + k                    (utility.h:55-58)
 *   x-faces (NX+1)*NY*NZ, y-faces NX*(NY+1)*NZ, z-faces NX*NY*(NZ+1)
 *   particles as structure-of-arrays: pos float3, vel float3, flag int8,
 *   mass, temperature, latent heat, solubility, gas content (float each)
 *                                                      (spray.h:165-170,278)
 * Particle and cell type codes are the reference's TYPE* values
 * (utility.h:13-19).
 *
 * Error convention (replaces getLastCudaError/exit and `mpause`):
 * every function returns MP_OK or one MP_ERR_* code; mp_last_error()
 * gives the message. Nothing calls exit().
 *
 * Threading: one context per host thread; all device work of a context is
 * ordered on its stream (mp_set_stream). Entry points return after the
 * work is enqueued unless stated; functions that hand data to the host
 * synchronise the stream.
 */
#ifndef MP_H
#define MP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define MP_OK              0
#define MP_ERR_CUDA        1   /* a CUDA runtime call failed                 */
#define MP_ERR_CAPACITY    2   /* par_num_max or a marching-cubes cap hit    */
#define MP_ERR_NOCONVERGE  3   /* CG stopped at its iteration limit          */
#define MP_ERR_TIMEOUT     4   /* a bounded device-side wait gave up         */
#define MP_ERR_ARG         5   /* bad argument (null, size, id)              */
#define MP_ERR_STATE       6   /* call not valid in the current state        */
#define MP_ERR_IO          7   /* an output file could not be opened/written */

/* ---- particle / cell types (utility.h:13-19) ------------------------- */
#define MP_TYPEFLUID    0
#define MP_TYPEAIR      1
#define MP_TYPEBOUNDARY 2
#define MP_TYPEVACUUM   3
#define MP_TYPEAIRSOLO  4
#define MP_TYPESOLID    5
#define MP_TYPECNT      6
#define MP_CELL_UNDEF   0xffffffffu   /* empty cell marker (utility.h:22) */

/* ---- scenes (utility.h:114-131); only the branches the step takes ---- */
#define MP_SCENE_FLUIDSPHERE            0
#define MP_SCENE_SMOKE                  1
#define MP_SCENE_BOILING                2
#define MP_SCENE_BOILING_HIGHRES        3
#define MP_SCENE_MULTIBUBBLE            4
#define MP_SCENE_DAMBREAK               5
#define MP_SCENE_MELTING                6
#define MP_SCENE_MELTINGPOUR            7
#define MP_SCENE_FREEZING               8
#define MP_SCENE_INTERACTION            9
#define MP_SCENE_INTERACTION_HIGHRES   10
#define MP_SCENE_MELTANDBOIL           11
#define MP_SCENE_MELTANDBOIL_HIGHRES   12
#define MP_SCENE_HEATTRANSFER          13
#define MP_SCENE_ALL                   15

/* ---- solver modes ----------------------------------------------------- */
#define MP_TOL_REF_ABS   0   /* stop when r.r < cg_tol*n  (spray.cu:1619,1666) */
#define MP_TOL_REL       1   /* stop when |r| <= cg_tol*|b|                    */
#define MP_PREC_MIXED    0   /* FP32 vectors, FP64 dots/alpha/beta            */
#define MP_PREC_FP64     1   /* divergence, pressure CG, gradient and the heat CG in FP64 */
#define MP_COEF_REF      0   /* constant-coefficient Laplacian (reference)    */
#define MP_COEF_GFM      1   /* variable density, ghost-fluid face weights (extension)                 */

#define MP_PARAMS_VERSION 4

/*
 * Runtime parameters: the reference's FlipConstant (utility.h:26-46), the
 * per-scene members set by cspray::initparam (spray.cpp:23-626) and the
 * solver switches this implementation adds. All fields are 4 bytes.
 * Fill with mp_params_default(), then edit.
 */
typedef struct mp_params {
    int32_t version;
    int32_t nx, ny, nz;              /* grid (spray.h:14, now runtime)        */
    int32_t par_num_max;             /* particle capacity (spray.h:170)       */
    int32_t scene;                   /* MP_SCENE_* (spray.h:191)              */
    float   cellsize;                /* hparam.cellsize.x                     */
    float   dt;                      /* hparam.dt                             */
    float   gravity_x, gravity_y, gravity_z;
    float   gmin_x, gmin_y, gmin_z;  /* domain origin (hparam.gmin)           */
    float   samplespace;             /* hparam.samplespace                    */
    float   m0, airm0, waterrho, solidrho, pradius;   /* solidrho (buoyancyForSolid,
                                        launch commented out) and pradius (triangle
                                        hashing for rendering) are kept for
                                        FlipConstant parity; the step reads neither */
    float   poly6kern, spikykern, lapkern;
    /* scene switches (spray.h:344-358) */
    int32_t b_solid, b_melt, b_freeze, b_fix_solid, b_gen_gas, b_heat_trans;
    int32_t b_add_heat_bottom, b_extend_heat_to_boundary, b_correct_position;
    int32_t b_smooth_mc, b_run_mc;
    int32_t mc_every;                /* outputframeDelta                      */
    int32_t smooth_iters;            /* smoothIterTimes                       */
    /* scene constants (spray.h:275-293, spray.cpp:31-78) */
    float   surfacetension_sigma;
    float   heatalpha_fluid, heatalpha_air, heatalpha_solid, heatalpha_vacuum;
    float   default_temperature, temperature0, melting_point, boiling_point;
    float   drag_param_solo, drag_param_grid, viscosity_sph;
    float   default_solid_T, default_liquid_T, liquid_heat_th, alpha_temp_trans;
    float   bounce_vel_param, bounce_pos_param, heat_increase_bottom;
    float   bubble_max_vel, max_vel_for_bubble;   /* the second clamps nothing: its
                                        use in enforceForceSoloAirP is commented out
                                        (spray_k.cu:4366-4367) */
    float   buoyance_rate_air, buoyance_rate_solo;
    float   vapor_gen_rate, init_dissolve_gas_rate, init_gas_rate;
    float   correction_spring, correction_radius;
    float   mc_density;              /* fMCDensity: passed to the step's density
                                        kernels, which do not read it          */
    float   heat_clamp;              /* 378.0 in addHeatAtBottom (spray_k.cu:4502) */
    float   solubility_coef;         /* 1018.9 in updatesolubility (spray_k.cu:4725) */
    float   solid_bounce_param;      /* SolidbounceParam                      */
    /* solver switches (new) */
    float   flip_alpha;              /* 1.0 = pure FLIP as bubblesim ships    */
    int32_t cg_tol_mode;             /* MP_TOL_*                              */
    float   cg_tol;                  /* 0.01 (ref_abs) or 1e-6 (rel)          */
    int32_t cg_max_iter;             /* 800 (spray.cu:1642)                   */
    int32_t heat_cg_max_iter;        /* 3800 (spray.cu:1804)                  */
    int32_t cg_true_residual_every;  /* recompute r = b - A x every k its     */
    int32_t precision;               /* MP_PREC_*                             */
    int32_t coef_mode;               /* MP_COEF_*                             */
    float   density_ratio;           /* rho_liquid / rho_air for MP_COEF_GFM  */
    int32_t mc_max_verts, mc_max_tris;
    int32_t seed_redraw;             /* must be 0: updateSeedCell's re-draw with
                                        the host rand() is not supported; the
                                        nucleation cells are mp_set_tables'   */
    int32_t update_seed_frame_delta;
    /* 1: cells whose MP_F_FIXEDHEAT value is not MP_UNDEF_TEMPERATURE are held
     * at it, the reference's dormant Dirichlet path (compb_heat,
     * spray_k.cu:4515-4519, updateFixedHeat spray_k.cu:4478) */
    int32_t b_fixed_heat;
    /* pouring emitters and the interaction scenes (spray.h:94, 138, 357) */
    float   pos_rand_param;          /* posrandparam: emitter position jitter, samplespace units */
    float   vel_rand_param;          /* velrandparam: emitter velocity jitter                   */
    int32_t begin_frame;             /* m_beginFrame: first gas-pouring / solid-release frame   */
    int32_t b_run_mc_solid;          /* bRunMCSolid: 0 = extract the solid surface once, then
                                        move it with the rigid solid motion                     */
    /* > 0: the MP_PREC_MIXED pressure solve runs as mixed-precision iterative
     * refinement: x and the true residual r = b - A x are kept and recomputed
     * in FP64 (right-hand side from the FP64 divergence), each correction is
     * an FP32-vector CG on r to this relative tolerance, and the stop rule
     * (cg_tol_mode, cg_tol) is tested on the FP64 true residual. 0: one CG
     * pass (the reference's recurrence). */
    float   cg_refine_tol;
    int32_t reserved[2];
} mp_params;

#define MP_UNDEF_TEMPERATURE (-10000.0f)   /* utility.h:24 */

/* Field identifiers for mp_get_field / mp_set_field. */
enum mp_field {
    /* cell fields, float[n] */
    MP_F_PRESS = 0, MP_F_DIV, MP_F_LSFLUID, MP_F_LSAIR, MP_F_LSMERGE,
    MP_F_PHIFLUID, MP_F_PHIAIR, MP_F_PHISOLID,
    MP_F_PHIGRAX, MP_F_PHIGRAY, MP_F_PHIGRAZ,
    MP_F_PHIGRAX_AIR, MP_F_PHIGRAY_AIR, MP_F_PHIGRAZ_AIR,
    MP_F_SURFTENSION, MP_F_TP, MP_F_TP_SAVE, MP_F_TP_OLD, MP_F_FIXEDHEAT,
    /* cell marks, int8[n] */
    MP_F_MARK,
    /* face fields, float[(nx+1)ny nz] / [nx(ny+1)nz] / [nx ny(nz+1)] */
    MP_F_WATERUX, MP_F_WATERUY, MP_F_WATERUZ,
    MP_F_WATERUX_OLD, MP_F_WATERUY_OLD, MP_F_WATERUZ_OLD,
    MP_F_AIRUX, MP_F_AIRUY, MP_F_AIRUZ,
    MP_F_AIRUX_OLD, MP_F_AIRUY_OLD, MP_F_AIRUZ_OLD,
    MP_F_SOLIDUX, MP_F_SOLIDUY, MP_F_SOLIDUZ,
    /* cell ranges of the last particle sort, uint32[n] (read only) */
    MP_F_CELLSTART, MP_F_CELLEND,
    /* particle attributes, [par_num_now] */
    MP_P_POS,        /* float[3*np] */
    MP_P_VEL,        /* float[3*np] */
    MP_P_FLAG,       /* int8[np]    */
    MP_P_MASS, MP_P_TEMP, MP_P_LHEAT, MP_P_SOLUBILITY, MP_P_GASCONTAIN,
    MP_FIELD_COUNT
};

/* Step-level scalars carried between stages. */
typedef struct mp_state {
    int32_t frame;            /* mframe                                        */
    int32_t par_num_now;      /* parNumNow                                     */
    int32_t n_real_solpoint;  /* nRealSolpoint                                 */
    int32_t last_cg_iters;    /* pressure CG iterations of the last projection */
    double  last_cg_residual; /* its final r.r                                 */
    int32_t last_heat_cg_iters;
    double  last_heat_cg_residual;
    int32_t mc_verts[3];      /* last marching-cubes vertex counts per surface */
    int32_t mc_indices[3];    /* last index counts (3 per triangle)            */
    int32_t mc_active_voxels[3];
    int32_t reserved[6];
} mp_state;

/* Marching-cubes surfaces, in the order bubblesim extracts them
 * (spray.cpp:1192-1201). */
#define MP_MC_SOLID 0
#define MP_MC_FLUID 1
#define MP_MC_GAS   2

/* Kernel classes whose launches can be timed with CUDA events. */
#define MP_KT_CG_STENCIL   0   /* pressure CG: A p and p.Ap                */
#define MP_KT_CG_UPDATE    1   /* pressure CG: x, r update and r.r          */
#define MP_KT_P2G          2   /* water + air particle-to-grid gather       */
#define MP_KT_G2P          3   /* FLIP grid-to-particle                     */
#define MP_KT_SORT         4   /* hash + counting sort + reorder            */
#define MP_KT_LEVELSET     5   /* genlevelset                               */
#define MP_KT_MC_DENS      6   /* marching-cubes density field              */
#define MP_KT_CORRECT      7   /* particle spacing correction (correctpos)  */
#define MP_KT_COUNT        8

/* ---- parameters ------------------------------------------------------- */

/* Defaults of the reference (spray.cpp:29-78, 573-626) for a grid of
 * nx,ny,nz cells with cellsize 1/64, scene MULTIBUBBLE. */
int mp_params_default(mp_params* p, int nx, int ny, int nz, int par_num_max);
/* Recompute the derived constants m0, airm0, pradius, *kern from
 * cellsize/samplespace/waterrho exactly as initparam does (spray.cpp:573-588). */
int mp_params_derive(mp_params* p);
/* Field table of mp_params for bindings: name, byte offset, kind (0 int32, 1 float). */
int mp_params_describe(int index, const char** name, int* offset, int* kind);
int mp_params_size(void);

/* ---- context ---------------------------------------------------------- */

/* Allocates every device buffer (replaces cspray::initmem_bubble,
 * spray.cu:25-218, and initMC, spray.cu:709-757). */
int mp_create(const mp_params* p, void** ctx);
int mp_destroy(void* ctx);
int mp_set_params(void* ctx, const mp_params* p);
int mp_get_params(void* ctx, mp_params* p);
int mp_get_state(void* ctx, mp_state* s);
int mp_set_state(void* ctx, const mp_state* s);
int mp_last_error(void* ctx, char* buf, size_t len);
/* Stream the context enqueues on (a cudaStream_t passed as a pointer). */
int mp_set_stream(void* ctx, void* stream);
int mp_get_stream(void* ctx, void** stream);
int mp_synchronize(void* ctx);
/* Device id the context was created on. */
int mp_get_device(void* ctx, int* device);

/* ---- data in / out ---------------------------------------------------- */

/* Copies n particles from HOST arrays (structure of arrays as in the
 * reference; any of T/L/sol/gas may be NULL = zero). Sets par_num_now.
 * Every flag must be an MP_TYPE* value (else MP_ERR_ARG, nothing copied).
 * Replaces the H2D copies of initparticle_solidCoupling (spray.cu:465-470). */
int mp_upload_particles(void* ctx, int n, const float* pos3, const float* vel3,
                        const int8_t* flag, const float* mass, const float* temp,
                        const float* lheat, const float* solubility,
                        const float* gascontain);
int mp_download_particles(void* ctx, int* n, float* pos3, float* vel3,
                          int8_t* flag, float* mass, float* temp, float* lheat,
                          float* solubility, float* gascontain);
/* Element count and element size of a field (particle fields: per current np). */
int mp_field_info(void* ctx, int field, size_t* count, size_t* elem_bytes);
int mp_get_field(void* ctx, int field, void* host_dst, size_t bytes);
int mp_set_field(void* ctx, int field, const void* host_src, size_t bytes);
/* The random table (spray.cu:180-190) and nucleation seed cells
 * (spray.cu:2907-2933) are inputs, so every implementation sees the same. */
int mp_set_tables(void* ctx, const float* randfloat, int nrand,
                  const int32_t* seedcells, int nseed);
/* Marching-cubes case tables this build uses (numVerts[256], tri[256*16],
 * edge[256]); generated, not copied (see mc_tables.cpp). */
int mp_mc_tables(int32_t* num_verts, int32_t* tri, int32_t* edge);
/* Replaces the context's marching-cubes case tables (numVerts[256],
 * tri[256*16]) for its later extractions, e.g. with the reference's own
 * tables.h (spray_k.cu reads them through edgeTex/triTex/numVertsTex,
 * spray_k.cu:2262-2277) to reproduce its triangulation.  Every count must be
 * 0..15 in steps of 3 and every listed edge one that the case crosses
 * (MP_ERR_ARG otherwise). */
int mp_set_mc_tables(void* ctx, const int32_t* num_verts, const int32_t* tri);

/* ---- scene set-up (cspray::init, spray.cpp:628-670) -------------------- */

/* Parameters of benchmark configuration `config` (1..5: rising bubble 32^3,
 * pool boiling 64^3, melting/freezing 128^3, dam break 64^3, bubble column
 * 256^3) on an n^3 grid (n = 0: the configuration's own size). Replaces the
 * per-scene branches of cspray::initparam (spray.cpp:83-547). */
int mp_scene_params(int config, int n, mp_params* p);
/* Seeds the configuration's particles (cspray::initparticle_solidCoupling,
 * spray.cu:395-484, with jittered 2x2x2 sub-cell sampling): writes up to cap
 * particles into the host arrays and their count into *n; with pos3 == NULL
 * only counts. Temperatures, latent heat, solubility and gas content follow
 * initTemperature/initSolubility (spray.cu:1989-1999) with the
 * configuration's per-particle noise. */
int mp_scene_particles(const mp_params* p, int config, uint64_t seed, int cap, int* n,
                       float* pos3, float* vel3, int8_t* flag, float* mass, float* temp,
                       float* lheat, float* solubility, float* gascontain);
/* Random table (nrand uniforms in [0,1)) and nucleation seed cells of the
 * configuration; *nseed is set to the number written (at most maxseed). */
int mp_scene_tables(const mp_params* p, int config, uint64_t seed, float* randfloat, int nrand,
                    int32_t* seeds, int maxseed, int* nseed);
/* Fixed-temperature plate of the configuration (MP_F_FIXEDHEAT, n floats). */
int mp_scene_fixed_heat(const mp_params* p, int config, float* fixedheat);

/* initTemperature + initSolubility (spray.cu:1989-1999) on the uploaded
 * particles; sets n_real_solpoint to the number of SOLID particles. */
int mp_init_particle_heat(void* ctx);

/* ---- stages, one per cspray method (spray.h:21-337) -------------------- */

int mp_hash_sort(void* ctx);                 /* hashAndSortParticles  spray.cu:614  */
int mp_external_force(void* ctx);            /* addexternalforce      spray.cu:376  */
int mp_levelset(void* ctx, float offset);    /* computeLevelset       spray.cu:1465 */
int mp_sweep_ls_mark(void* ctx);             /* sweepLSAndMardGrid    spray.cu:2011 */
int mp_mark_solo_air(void* ctx);             /* markSoloAirParticle   spray.cu:2614 */
int mp_surface_tension(void* ctx);           /* computesurfacetension spray.cu:2001 */
int mp_markgrid_bubble(void* ctx);           /* markgrid_bubble       spray.cu:511  */
int mp_p2g(void* ctx);                       /* mapvelp2g_bubble      spray.cu:1562 */
int mp_drag(void* ctx);                      /* enforceDragForce      spray.cu:2953 */
int mp_sweep_phi(void* ctx, int phase);      /* sweepPhi  (phase = MP_TYPEFLUID|MP_TYPEAIR) spray.cu:570 */
int mp_sweep_u(void* ctx, int phase);        /* sweepU                spray.cu:585  */
int mp_set_boundary_u(void* ctx, int phase); /* setWaterBoundaryU     spray.cu:605  */
int mp_project(void* ctx, int* iters, double* residual); /* project_CG_bubble spray.cu:1590 */
/* The pressure CG of mp_project as a standalone call that allocates nothing
 * (no cudaMalloc, cudaFree or allocating library routine). No counterpart in
 * the reference. It is for callers that cannot allocate device memory while
 * they run: code embedded in a host application that owns a fixed device
 * budget (its own memory pool, or the rest of the GPU already taken), and
 * code inside a frame or stream loop where cudaFree, which synchronises the
 * whole device, would stall everything else on the GPU.
 * The caller passes device arrays of nx*ny*nz cells: mark (int8, MP_TYPE*),
 * divergence (float, the right-hand side mp_project builds, field MP_F_DIV)
 * and pressure (float, written). It solves mp_project's system with
 * mp_project's stop rule (tol_mode, tol, max_iter) and returns the same
 * pressure, iteration count and residual as mp_project does for
 * MP_PREC_MIXED, MP_COEF_REF, the bubble mode (FLUID and AIR cells are
 * unknowns) and cg_true_residual_every = 0; it has no FP64, ghost-fluid,
 * single-phase or true-residual variant. Runs on `stream` (NULL: the default
 * stream), synchronises it (the stop flag is read back between iteration
 * batches) and returns after it has finished, so it must not be called on a
 * stream that is being captured.
 * All working storage (residual, two direction vectors, neighbour bytes,
 * reduction partials) lives in one fixed array of about 3.3 MB that the
 * library holds on every GPU it is loaded on, until the process exits; grids
 * above 262,144 cells (64^3) are rejected with MP_ERR_CAPACITY before any GPU
 * work. Each call looks up that array's address in the current context
 * (cudaGetSymbolAddress, which allocates nothing), so it stays valid across
 * cudaDeviceReset and in a caller's own context. Every call reuses the same
 * array (the parts that must start at zero are cleared at each call), so
 * calls whose GPU work overlaps, from other streams or host threads on the
 * same device, race and give wrong results. Errors are read with
 * mp_last_error(NULL, ...). */
int mp_pressure_cg_static(int nx, int ny, int nz, float cellsize, const int8_t* mark,
                          const float* divergence, float* pressure, int max_iter, int tol_mode,
                          float tol, void* stream, int* iters, double* residual);
int mp_g2p(void* ctx);                       /* mapvelg2p_bubble      spray.cu:1689 */
int mp_solid_motion(void* ctx);              /* solidmotion[_fixed]   spray.cu:2685 */
int mp_solo_air_update(void* ctx);           /* updateSoloAirParticle spray.cu:2620 */
int mp_collide_advect(void* ctx);            /* CollisionSolid        spray.cu:2959 */
int mp_correct_pos(void* ctx);               /* correctpos            spray.cu:328  */
int mp_correct_pos_bubble(void* ctx);        /* correctpos_bubble     spray.cu:2067 */
int mp_heat(void* ctx);                      /* updateTemperature     spray.cu:1889 */
int mp_gen_gas(void* ctx);                   /* GenerateGasParticle   spray.cu:2653 */
int mp_delete(void* ctx);                    /* deleteAirFluidParticle spray.cu:2194 */
int mp_melt(void* ctx);                      /* MeltSolid             spray.cu:2816 */
int mp_freeze(void* ctx);                    /* Freezing              spray.cu:2860 */
/* preMC + one runMC_smooth surface (spray.cu:759-979); the 2x re-sort is
 * done by mp_mc_presort (hashAndSortParticles_MC, spray.cu:639). */
int mp_mc_presort(void* ctx);
int mp_mc(void* ctx, int surface);
/* Vertex positions (float3), normals (float3) and uint32 indices of the
 * last extraction of `surface`; counts from mp_state. */
int mp_mc_download(void* ctx, int surface, float* verts, float* normals,
                   uint32_t* indices, int max_verts, int max_indices);
/* MC density field (float[(2nx+1)(2ny+1)(2nz+1)]) and per-voxel case index
 * (uint8[8n]) of the last extraction. */
int mp_mc_download_field(void* ctx, float* dens, uint8_t* cubeindex);

/* ---- the reference's scenes (cspray::initparam, spray.cpp:23-626) -------
 * mp_reference_scene fills `p` with the parameters initparam gives scene
 * `scene` (MP_SCENE_*): its common defaults (spray.cpp:29-78), the scene's
 * branch (83-547) and the derived constants (573-626), in the reference's
 * units (Kelvin temperatures); fields this library adds keep
 * mp_params_default's values. `info` (may be NULL) gets the rest of the
 * branch. Host code only. */
#define MP_SIM_WATER          0   /* SIMULATIONMODE (utility.h:105-111)     */
#define MP_SIM_SOLIDCOUPLING  1   /* SPH solid coupling: not in this library */
#define MP_SIM_SMOKE          2   /* not in this library                    */
#define MP_SIM_BUBBLE         3   /* mp_step                                */
#define MP_SIM_HEATONLY       4   /* mp_heatsim                             */
typedef struct mp_scene_info {
    int32_t nx, ny, nz;             /* the grid initparam requires (it exits otherwise) */
    int32_t sim_mode;               /* MP_SIM_*                                */
    int32_t init_fluid_particles;   /* initfluidparticle                       */
    int32_t split_num;              /* par_num_max = par_num_extra +           */
    int32_t par_num_extra;          /*   (fluid + solid points) * split_num    */
    int32_t seed_num;               /* seednum: nucleation cells               */
    int32_t pour_variant;           /* MP_POUR_* of CompPouringParam_*, or -1  */
    float   pour_radius, pour_pos[3], pour_pos2[3], pour_vel[3];
    float   solid_init_pos[3];      /* solidInitPos                            */
    float   t_render_min, t_render_max;
    int32_t frame_max;
    int32_t output_colored_particles;   /* bOutputColoredParticle          */
    int32_t reserved[8];
} mp_scene_info;
int mp_reference_scene(int scene, mp_params* p, mp_scene_info* info);

/* ---- pouring emitters (spray.cpp:1416-1545, spray.cu:3012-3043) ---------
 * The emitter is a set of points with a velocity each (dpourpos /
 * dpourvel). mp_scene_pour lays one out as the scene set-up does:
 * MP_POUR_FREEZING = CompPouringParam_Freezing (disc of radius `radius` at
 * `center`, samplespace spacing); MP_POUR_INTERACTION = CompPouringParam_
 * Ineraction (2 x samplespace spacing); MP_POUR_INTERACTION2 = _Ineraction2
 * (two such discs, at `center` and `center2`). All points get `vel`. It writes
 * at most `cap` points (pos3/vel3 may be NULL to count) and sets *n to the
 * number of points of the emitter; host code only. */
#define MP_POUR_FREEZING      0
#define MP_POUR_INTERACTION   1
#define MP_POUR_INTERACTION2  2
int mp_scene_pour(int variant, float samplespace, float radius, const float* center, const float* center2,
                  const float* vel, int cap, float* pos3, float* vel3, int* n);
/* Sets the context's emitter (copied); n = 0 removes it. */
int mp_set_pour(void* ctx, const float* pos3, const float* vel3, int n);
/* pouring / pouringgas: appends the emitter's n particles (pouringwater,
 * spray_k.cu:5575-5596: position jitter pos_rand_param * samplespace, velocity
 * jitter vel_rand_param, both from the random table) as FLUID every 4th frame
 * or, in MP_SCENE_INTERACTION(_HIGHRES) from begin_frame on, as AIRSOLO every
 * 6th frame; nothing when they would exceed par_num_max. mp_step calls it
 * first. */
int mp_pour(void* ctx);

/* ---- heat-only mode (SIMULATION_HEATONLY, MP_SCENE_HEATTRANSFER) --------
 * mp_init_heat_grid: initheat_grid (spray.cu:1949-1955): in every xz-section
 * a SOLID disc at 100 and a FLUID disc at 0 (radius 0.15 nx, centres at
 * (nx/4, nz/4) and (3nx/4, 3nz/4)), VACUUM at 20 below nz/2, AIR at 80
 * above, and the outer shell BOUNDARY; it sets MP_F_TP and MP_F_MARK.
 * mp_heatsim: heatsim (spray.cu:1959-1987): one implicit diffusion step of
 * the cell temperatures (compb_heat, the heat CG, setBoundaryHeat when
 * b_extend_heat_to_boundary), with the cell marks as they are and no
 * particles; advances the frame. The reference's scene uses heatalpha
 * fluid 0.0001, air 0.005, solid 0.015, vacuum 0.05 (spray.cpp:531-546). */
int mp_init_heat_grid(void* ctx);
int mp_heatsim(void* ctx);

/* ---- water-only mode (SIMULATION_WATER, cspray::watersim) ----------------
 * Stages of the single-phase FLIP step, under the reference's names:
 * flipMark_sphere (spray.cu:515: VACUUM cells become AIR), mapvelp2g
 * (spray.cu:340: water faces from FLUID and SOLID particles, copied for the
 * FLIP update), project_CG (spray.cu:241: cptdivergence over FLUID cells, CG
 * with FLUID unknowns and AIR at zero pressure, subGradPress on the water
 * faces; MP_PREC_MIXED and MP_COEF_REF only), mapvelg2p (spray.cu:362:
 * computeDeltaU on the water faces, every particle takes the change) and
 * wateradvect (spray.cu:293: advectparticle_RK2, velocity blended with the
 * grid as FLIP_ALPHA = 0.95, midpoint position step, wall clamp). mp_watersim
 * runs the step of spray.cpp:741-797 and extracts the FLUID surface when
 * b_run_mc is set; it re-sorts on the 2x grid before the extraction, which
 * the reference omits. With mp_set_output it writes the FLUID surface's files
 * as mp_step does. */
int mp_flip_mark(void* ctx);
int mp_water_p2g(void* ctx);
int mp_project_water(void* ctx, int* iters, double* res);
int mp_water_g2p(void* ctx);
int mp_water_advect(void* ctx);
int mp_watersim(void* ctx);

/* The whole bubblesim step in the reference's order and cadence
 * (spray.cpp:979-1233): pouring, the frame-scripted parameter switches of
 * MP_SCENE_ALL / MELTANDBOIL(_HIGHRES) / INTERACTION(_HIGHRES)
 * (spray.cpp:1007-1047; they change the context's parameters, as
 * mp_get_params shows), then the stages. In those scenes with
 * b_run_mc_solid = 0 the solid surface is extracted at frame 0 only, moved
 * with the rigid solid motion (computeSolidVertex_k) and re-normalled
 * (runMC_interaction). Synchronous at exit. Its solid-velocity faces
 * (MP_F_SOLIDU*) are left as they were when no cell holds a SOLID particle:
 * the collision reads them only within half a cell of a solid. */
int mp_step(void* ctx);

/* ---- per-frame files (cspray::output*, spray.cu:2250-2526) --------------
 * The reference's writers, byte for byte with its printf formats: an empty
 * mesh gives an empty file, a vertex or normal with a NaN component is
 * written as (0,0,0) (verifyfloat3, spray.cu:999), OBJ indices are 1-based,
 * and the BOBJ face block is preceded by the number of indices (not of
 * triangles). BOBJ is gzip at level 1 ("wb1"). A file that cannot be opened
 * or written gives MP_ERR_IO (the reference printed and paused). */
#define MP_OUT_POV_MESH  0   /* outputPovRaywater: POV-Ray mesh2   (spray.cu:2250) */
#define MP_OUT_OBJ_MESH  1   /* outputOBJwater: Wavefront OBJ      (spray.cu:2308) */
#define MP_OUT_BOBJ_GZ   2   /* outputBOBJwater: Blender .bobj.gz  (spray.cu:2373) */
#define MP_OUT_PARTICLES_COLORED 0  /* outputColoredParticle: all particles,
                                       coloured by temperature  (spray.cu:2440) */
#define MP_OUT_PARTICLES_SOLO    1  /* outputSoloBubblePovRay: AIRSOLO (spray.cu:2468) */
#define MP_OUT_PARTICLES_AIR     2  /* outputAirParticlePovRay: AIR    (spray.cu:2498) */

/* One mesh from host arrays: float3 vertices and normals, uint32 indices
 * (3 per triangle, each below nverts). object_name names the POV-Ray
 * material (`<name>_material`). */
int mp_write_mesh(int format, const char* path, const char* object_name, const float* verts,
                  const float* normals, int nverts, const uint32_t* indices, int nindices);
/* POV-Ray spheres from host arrays: float3 positions, int8 flags (SOLO/AIR
 * kinds), temperatures (COLORED: colour of (T - t_min)/(t_max - t_min)*6
 * on mapColorBlue2Red_h, spray.cpp:1299). */
int mp_write_particles(int kind, const char* path, const float* pos, const int8_t* flag,
                       const float* temperature, int n, float t_min, float t_max);
/* The same writers on the context's data: the last extraction of `surface`
 * (MP_MC_*), named "solid" / "water" / "gas" as runMC_solid / runMC_fluid /
 * runMC_gas name it (spray.cu:767-784), and the current particles. */
int mp_export_mesh(void* ctx, int surface, int format, const char* path);
int mp_export_particles(void* ctx, int kind, const char* path, float t_min, float t_max);

/* Per-frame output of bubblesim. With it set, every mp_step that extracts
 * the meshes (frame % mc_every == 0, mc_every = outputframeDelta) writes, as
 * runMC_smooth (spray.cu:954-958, 858-863) and bubblesim (spray.cpp:1208-1216) do,
 * with F = frame / mc_every:
 *   pov: <dir>waterdata/<name>%05d.pov per surface; the particle files
 *        <dir>waterdata/allparticles%05d.pov (colored_particles),
 *        <dir>waterdata/solobubble%05d.pov (AIRSOLO spheres in
 *        MP_SCENE_INTERACTION, AIR spheres in MP_SCENE_BOILING);
 *   obj: <dir><name>BOBJdata/fluidsurface_final_%04d.bobj.gz with F - 1,
 *        or, for an empty surface, an empty <dir>waterOBJdata/<name>%05d.obj;
 *        a solid surface kept from frame 0 (b_run_mc_solid = 0 in the
 *        interaction scenes) goes to <dir>waterOBJdata/solid%05d.obj.
 * `dir` is a prefix used as written (end it with '/'); the directories must
 * exist, as in the reference. NULL turns the output off (the default). */
typedef struct mp_output {
    const char* dir;           /* outputdir                                */
    int32_t pov;               /* boutputpovray                            */
    int32_t obj;               /* boutputobj                               */
    int32_t colored_particles; /* bOutputColoredParticle                   */
    float   t_render_min;      /* temperatureMin_render                    */
    float   t_render_max;      /* temperatureMax_render                    */
} mp_output;
int mp_set_output(void* ctx, const mp_output* out);

/* ---- adjoint (no counterpart in the reference) -------------------------------
 * Reverse-mode derivative of the step for a scene of FLUID particles, or of
 * FLUID and AIR particles (bubbles), with position correction, gas, melting,
 * freezing and solids off (configuration 4, the dam break; configurations 1
 * and 5 with position correction off). The program is bubblesim's: external
 * forces (gravity on FLUID, the buoyancy of AIR), the water and air splats,
 * extrapolation of both fields, wall rules, the two-phase projection (the
 * level-set blend of cptdivergence_bubble2 at liquid-air faces), the FLIP/PIC
 * gather of each phase's field and advection; the solo-air stages
 * (markSoloAirParticle, the drag and SPH forces) are not part of it, so AIR
 * particles stay AIR. The heat stage (b_heat_trans) is differentiated for
 * FLUID-only scenes. mp_adj_record runs `nsteps` steps of this program with
 * the engine's own stages from the current particles (advancing the context)
 * and records the discrete state of each step (splat order and cell ranges,
 * cell marks, the merged level set and the extrapolation distance fields,
 * and at the end each cell's nearest FLUID particle); the derivative is that
 * of the program with this state held fixed. A recording that fails (an
 * MP_ERR_* code from a step or an allocation) keeps no tape, and the context
 * has advanced by the steps it ran; mp_adj_* calls then return
 * MP_ERR_STATE until the next mp_adj_record.
 * mp_adj_set_targets takes the target points y_s (host float xyz) of the
 * loss L = sum_s phi(y_s)^2, phi the fluid distance field of genlevelset
 * after the last step. mp_adj_loss replays the program from the recorded
 * initial particles with initial velocities v0 (device, double xyz per
 * particle in the order the particles had at mp_adj_record; NULL: the
 * recorded ones) and returns L; mp_adj_gradient also writes dL/dv0 (device,
 * double xyz). precision: MP_PREC_MIXED replays in FP32 (CG dots in FP64),
 * MP_PREC_FP64 in FP64 with a 1e-13 relative CG stop. States are kept every
 * `checkpoint_every` steps and recomputed segment by segment backwards.
 * Device memory: the recording holds, per step, the sort order (4 B per
 * particle) and cell fields (9 B per cell, 17 B with AIR, another 8 B for the
 * engine's projection in the mixed form; the heat stage adds its own sort:
 * 4 B per particle and 5 B per cell) and, per segment,
 * the engine's state (24 B per particle); a gradient in FP32 holds the
 * checkpoints and one segment's states (24 B per particle each) and one
 * step's intermediates. */
int mp_adj_record(void* ctx, int nsteps, int checkpoint_every);
/* The recorded program as a differentiable map of the particles' initial
 * state to their final state, (x0, v0) -> (xT, vT), with the general
 * vector-Jacobian product of it (no counterpart in the reference).
 * Every array is a device array of doubles, xyz per particle in the order the
 * particles had at mp_adj_record; a NULL member of `in` means the recorded
 * values, a NULL member of `dout` a zero cotangent, a NULL member of `out` or
 * `din` that the result is not wanted.
 * mp_adj_forward replays the program from `in` and writes `out`.
 * mp_step_adjoint replays it from `in` and writes the cotangents of the
 * initial state, din = J^T dout, by the reverse sweep (the transposed splat,
 * extrapolation, wall rules, projection as a second CG solve on the pressure
 * matrix, FLIP/PIC gather and advection), recomputing each segment of
 * `checkpoint_every` steps from its checkpoint.
 * mp_adj_level_set_loss evaluates the loss of mp_adj_set_targets at final
 * positions `pos` and writes dloss/dpos (NULL: not wanted), so the loss can
 * be composed with the map. */
typedef struct mp_grad {
    double* pos;   /* xyz per particle */
    double* vel;   /* xyz per particle */
    double* temp;  /* one per particle; used when the recording ran the heat stage */
} mp_grad;
int mp_adj_forward(void* ctx, int precision, const mp_grad* in, mp_grad* out);
int mp_step_adjoint(void* ctx, int precision, const mp_grad* in, const mp_grad* dout, mp_grad* din);
int mp_adj_level_set_loss(void* ctx, int precision, const double* pos, double* loss, double* dloss_dpos);
int mp_adj_set_targets(void* ctx, const float* samples3, int nsamples);
int mp_adj_info(void* ctx, int* np, int* nsteps);
/* The recording order of the context's current particles: ids[s] (device,
 * one uint32 per particle) is the index, in the order the particles had at
 * mp_adj_record, of the particle now in slot s (mp_download_particles'
 * order), so the engine's state after the recording can be set beside the
 * replay's final state. */
int mp_adj_order(void* ctx, uint32_t* ids);
int mp_adj_loss(void* ctx, int precision, const double* v0, double* loss);
int mp_adj_gradient(void* ctx, int precision, const double* v0, double* grad_v0, double* loss);
int mp_adj_release(void* ctx);

/* Checkpoint / resume of the state a step starts from: particles, the random
 * table, nucleation cells, the fixed-heat field, the heat grid and mp_state.
 * A context created with identical parameters that loads a checkpoint and
 * steps reproduces the saving context's steps bit for bit. The reference
 * keeps this state only in its process (no counterpart). Host buffers;
 * mp_checkpoint_size gives the bytes needed; load rejects a checkpoint taken
 * with other parameters (MP_ERR_STATE) or of another format (MP_ERR_ARG). */
int mp_checkpoint_size(void* ctx, size_t* bytes);
int mp_checkpoint_save(void* ctx, void* host_dst, size_t bytes);
int mp_checkpoint_load(void* ctx, const void* host_src, size_t bytes);

/* ---- measurement -------------------------------------------------------- */

/* Record CUDA events around every launch of a kernel class on the context
 * stream; read back the summed device time (ms) and the launch count. */
int mp_kernel_timing(void* ctx, int kernel_class, int enable);
int mp_kernel_timing_read(void* ctx, int kernel_class, double* ms, int64_t* launches);
int mp_kernel_timing_reset(void* ctx);
/* Number of this library's kernel launches since the last reset. */
int64_t mp_launch_count(void* ctx);
/* Work counters since the last mp_kernel_timing_reset, for the byte models
 * of the measurement: particle sorts that reordered the particles, sorts
 * that found them already in cell order (keys and ranges only), and CG
 * iterations performed (pressure and heat solves; the launches of an
 * iteration batch after the stop test are not iterations); and the adjoint's
 * reverse sweeps that took the engine's recorded states in place of a first
 * replay (a gradient at the recorded inputs) and those that replayed every
 * step first. `n` may be smaller than MP_WC_COUNT. */
#define MP_WC_SORT_FULL  0
#define MP_WC_SORT_FAST  1
#define MP_WC_CG_ITERS   2
#define MP_WC_ADJ_ENGINE 3
#define MP_WC_ADJ_REPLAY 4
#define MP_WC_COUNT      5
int mp_work_counts(void* ctx, int64_t* counts, int n);

#ifdef __cplusplus
}
#endif
#endif /* MP_H */
