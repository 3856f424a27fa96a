// ctx.cuh — the device context behind the C ABI (replaces the state members of
// the reference's cspray class, Multiphase/Multiphase/spray.h:153-389).
//
// HBM layout (all row-major, x slowest, as the reference):
//   cell fields float[n], marks int8[n], face fields float[nf axis],
//   particles as three float4 streams sorted by cell:
//     pos4  = (x, y, z, flag bits)   vel4 = (vx, vy, vz, mass)
//     heat4 = (temperature, latent heat, solubility, gas content)
//   each stream double-buffered for the sort gather and the deletion compaction.
//   cell ranges as CSR offsets off[n+1] (off[c]..off[c+1] is cell c).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <string>
#include <vector>
#include "mp_dev.cuh"

struct McSurface {
    float3* verts = nullptr;
    float3* normals = nullptr;
    uint32_t* indices = nullptr;
    int nverts = 0, nindices = 0, active = 0;
};

struct MpCtx {
    mp_params P{};
    mp_state S{};
    int device = 0;
    cudaStream_t stream = 0;
    bool own_stream = false;
    mpk::Grid G{};
    std::string err;

    // per-frame files written by mp_step (mp_set_output)
    bool out_on = false;
    std::string out_dir;
    int out_pov = 0, out_obj = 0, out_colored = 0;
    float out_tmin = 0.0f, out_tmax = 1.0f;

    // cell fields
    float *press = 0, *divg = 0, *lsfluid = 0, *lsair = 0, *lsmerge = 0;
    float *phifluid = 0, *phiair = 0, *phisolid = 0;
    float *gx = 0, *gy = 0, *gz = 0, *gxa = 0, *gya = 0, *gza = 0, *sf = 0;
    float *Tp = 0, *Tp_save = 0, *Tp_old = 0, *fixedheat = 0;
    float *cell_tmp = 0;        // Jacobi double buffer for cell sweeps
    int8_t *mark = 0, *mark_tmp = 0;
    // face fields
    float *wu[3] = {0, 0, 0}, *wuo[3] = {0, 0, 0}, *au[3] = {0, 0, 0}, *auo[3] = {0, 0, 0};
    float *su[3] = {0, 0, 0}, *tmpu[3] = {0, 0, 0};
    // CG work vectors
    float *cg_r = 0, *cg_p = 0, *cg_z = 0;
    double *cg64 = 0;            // x, b, r, p, z in FP64 (precision = MP_PREC_FP64)
    double *red = 0;             // reduction partials
    double *scal = 0;            // device scalars (see k_cg.cu)
    unsigned int *red_count = 0; // last-block counters
    int red_blocks = 0;
    // CG kernels (tuning knobs read from the environment at mp_create):
    // MP_CG_KERNEL=v4 keeps the float4-group passes where the TMA plane
    // marching applies; MP_CG_TMA_CHUNK sets its planes per CTA (0: derived)
    int cg_use_tma = 1;
    int cg_tma_chunk = 0;
    float *gfm_beta = 0;         // ghost-fluid face weights (x, y, z faces), allocated on first use
    float *gfm_s = 0;            // its Jacobi scaling per cell
    // particles
    float4 *pos = 0, *vel = 0, *heat = 0;
    float4 *pos2 = 0, *vel2 = 0, *heat2 = 0;
    float *pdens = 0, *pprs = 0;
    float4 *pscr = 0;            // per-particle scratch (drag delta, snapshots)
    float4 *pscr2 = 0;
    int8_t *flag_snap = 0;
    uint8_t *pflag8 = 0, *pflag8s = 0;   // particle types as bytes: from the sort's count pass, and sorted
    // sort
    uint32_t *keys = 0, *perm = 0;
    uint32_t *cell_cnt = 0, *cell_off = 0;   // sized for the 2x marching-cubes grid
    uint8_t *tmask = 0;
    uint32_t *air_brick = 0;     // bit per 4x4x4-cell brick holding an AIR/AIRSOLO particle (last sort)
    size_t air_brick_words = 0;
    uint32_t *scan_tmp = 0;
    size_t scan_tmp_elems = 0;
    uint32_t *u32_scratch = 0;   // small device counters
    // tables
    float *randf = 0; int nrand = 0;
    float *pour_pos = 0, *pour_vel = 0; int pour_n = 0;   // emitter (dpourpos / dpourvel), float3 each
    int32_t *seeds = 0; int nseed = 0;
    int32_t *mc_numverts = 0, *mc_tri = 0;
    // marching cubes
    float *mc_dens = 0;
    float *mc_dens2 = 0;              // gas field of the fused fluid+gas density pass
    const float* mc_last_dens = 0;    // field of the last extraction
    uint8_t *mc_cube = 0;
    uint32_t *mc_vflag = 0, *mc_vscan = 0, *mc_compact = 0, *mc_vverts = 0, *mc_vvscan = 0;
    uint32_t *mc_emark = 0, *mc_escan = 0;
    uint32_t *mc_vstart = 0, *mc_inc = 0, *mc_fill = 0;
    float3 *mc_tmpv = 0;
    size_t mc_edges = 0;
    int mc_sorted = 0;           // particles currently sorted on the 2x grid
    McSurface mc[3];
    int mc_cap_verts = 0, mc_cap_idx = 0;

    // kernel timing
    bool kt_on[MP_KT_COUNT] = {};
    double kt_ms[MP_KT_COUNT] = {};
    int64_t kt_launch[MP_KT_COUNT] = {};
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kt_pending[MP_KT_COUNT];
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kt_pool;
    int64_t launches = 0;
    int64_t work[MP_WC_COUNT] = {};   // mp_work_counts

    struct AdjTape* adj = nullptr;   // the adjoint module's tape (k_adjoint.cu)

    int np() const { return S.par_num_now; }
};

// error helpers -------------------------------------------------------------
#define MP_CUDA(ctx, call)                                                        \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
            return MP_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)
#define MP_CHECK_LAUNCH(ctx)                                                      \
    do {                                                                          \
        cudaError_t e_ = cudaGetLastError();                                      \
        if (e_ != cudaSuccess) {                                                  \
            (ctx)->err = std::string("kernel launch: ") + cudaGetErrorString(e_); \
            return MP_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)
#define MP_TRY(x)                 \
    do {                          \
        int rc_ = (x);            \
        if (rc_ != MP_OK) return rc_; \
    } while (0)

// launch geometry: grid-stride loops sized to a multiple of the SM count
inline int mp_blocks(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    const long long cap = 148LL * 32;   // 148 SMs x 32 resident 256-thread blocks at most
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// a named range on the host timeline for nsys / ncu --nvtx; without a tool
// attached the calls do nothing
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
// one stage of a step, under the reference method's name
#define MP_STAGE(name, call)   \
    do {                       \
        NvtxRange r_(name);    \
        MP_TRY(call);          \
    } while (0)

// kernel-class timing (events around launches on the context stream)
void kt_begin(MpCtx* c, int cls, cudaEvent_t* ev_end);
void kt_end(MpCtx* c, int cls, cudaEvent_t ev_end);
struct KtScope {
    MpCtx* c; int cls; cudaEvent_t e1 = 0;
    KtScope(MpCtx* c_, int cls_) : c(c_), cls(cls_) { kt_begin(c, cls, &e1); }
    ~KtScope() { kt_end(c, cls, e1); }
};

// stage entry points implemented across the kernel files
int mp_scan_u32(MpCtx* c, const uint32_t* in, uint32_t* out, size_t n);   // exclusive scan, out[n] = total
int k_hash_sort(MpCtx* c);
int k_mc_presort(MpCtx* c);
int k_external_force(MpCtx* c);
int k_levelset(MpCtx* c);
int k_sweep_ls_mark(MpCtx* c);
int k_mark_solo_air(MpCtx* c);
int k_surface_tension(MpCtx* c);
int k_markgrid_bubble(MpCtx* c);
int k_p2g(MpCtx* c);
int k_drag(MpCtx* c);
int k_sweep_phi(MpCtx* c, int phase);
int k_sweep_u(MpCtx* c, int phase);
int k_set_boundary_u(MpCtx* c, int phase);
int k_project(MpCtx* c, int* iters, double* res);
int k_g2p(MpCtx* c);
int k_solid_motion(MpCtx* c);
int k_pour(MpCtx* c);
int k_heatsim(MpCtx* c);
int k_flip_mark(MpCtx* c);
int k_water_p2g(MpCtx* c);
int k_project_water(MpCtx* c, int* iters, double* res);
int k_water_g2p(MpCtx* c);
int k_water_advect(MpCtx* c);
int k_init_heat_grid_launch(MpCtx* c);
int k_mc_renormal(MpCtx* c, int surface);
int k_solo_air_update(MpCtx* c);
int k_collide_advect(MpCtx* c, bool skip_empty_solid = false);
int k_correct_pos(MpCtx* c);
int k_correct_pos_bubble(MpCtx* c);
int k_heat(MpCtx* c);
int k_gen_gas(MpCtx* c);
int k_delete(MpCtx* c);
int k_melt(MpCtx* c);
int k_freeze(MpCtx* c);
int k_mc(MpCtx* c, int surface);
int k_mc_fluid_gas(MpCtx* c);
int k_cg_solve(MpCtx* c, const int8_t* mark, float* x, const float* b, int maxiter, int tolmode, float tol, int* iters,
               double* res);
int k_cg_solve(MpCtx* c, const int8_t* mark, double* x, const double* b, int maxiter, int tolmode, float tol,
               int* iters, double* res);
void k_adj_free(MpCtx* c);
int k_adj_record(MpCtx* c, int nsteps, int every);
int k_adj_set_targets(MpCtx* c, const float* samples3, int nsamples);
int k_adj_run(MpCtx* c, int precision, const double* v0, double* grad, double* loss);
int k_adj_np(MpCtx* c, int* np, int* nsteps);
int k_adj_order(MpCtx* c, uint32_t* ids);
int k_heat_cg_solve(MpCtx* c, const int8_t* mark, float* x, const float* b, int maxiter, int tolmode, float tol,
                    int* iters, double* res);
int k_heat_cg_solve(MpCtx* c, const int8_t* mark, double* x, const double* b, int maxiter, int tolmode, float tol,
                    int* iters, double* res);
int k_adj_forward(MpCtx* c, int precision, const mp_grad* in, mp_grad* out);
int k_adj_vjp(MpCtx* c, int precision, const mp_grad* in, const mp_grad* dout, mp_grad* din);
int k_adj_ls_loss(MpCtx* c, int precision, const double* xT, double* loss, double* xTb);
int k_init_particle_heat(MpCtx* c);
int k_pack_particles(MpCtx* c, int n, const float* pos3, const float* vel3, const int8_t* flag,
                     const float* mass, const float* T, const float* L, const float* sol, const float* gas);
int k_unpack_particles(MpCtx* c, int n, float* pos3, float* vel3, int8_t* flag, float* mass,
                       float* T, float* L, float* sol, float* gas);
int k_cells_to_startend(MpCtx* c, uint32_t* start, uint32_t* end);
int k_phigra(MpCtx* c, float* ax, float* ay, float* az, const float* ls);
int k_sweep_pass_swap(MpCtx* c, float** phi, int typeflag);
int k_surface_tension_grid(MpCtx* c);
int k_solid_phi(MpCtx* c);
int k_delta_u(MpCtx* c);
int k_p2g_faces(MpCtx* c, float** out, int which);
