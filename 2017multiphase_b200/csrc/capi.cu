// capi.cu — the C ABI (include/mp.h): context life cycle, data movement,
// stage entry points and the full bubblesim step.
//
// The context replaces the state of the reference's cspray class
// (Multiphase/Multiphase/spray.h:153-389); mp_create is its initmem_bubble
// (spray.cu:25-218) plus initMC (spray.cu:709-757); mp_step is bubblesim
// (spray.cpp:979-1233).
#include "ctx.cuh"
#include <cmath>
#include <cstring>
#include <cstddef>
#include <algorithm>
#include <new>

extern "C" void mp_internal_mc_tables(int32_t* nv, int32_t* tri, int32_t* edge);

// parameters: mp_params_size/describe/default/derive live in host/params.cpp

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
static int dalloc(MpCtx* c, void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        c->err = std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e);
        return MP_ERR_CUDA;
    }
    return MP_OK;
}
template <class T>
static int dalloc_t(MpCtx* c, T** p, size_t count) { return dalloc(c, (void**)p, sizeof(T) * count); }

static void free_all(MpCtx* c) {
    void* ptrs[] = {c->press, c->divg, c->lsfluid, c->lsair, c->lsmerge, c->phifluid, c->phiair, c->phisolid,
                    c->gx, c->gy, c->gz, c->gxa, c->gya, c->gza, c->sf, c->Tp, c->Tp_save, c->Tp_old, c->fixedheat,
                    c->cell_tmp, c->mark, c->mark_tmp, c->cg_r, c->cg_p, c->cg_z, c->cg64, c->red, c->scal, c->red_count,
                    c->pos, c->vel, c->heat, c->pos2, c->vel2, c->heat2, c->pdens, c->pprs, c->pscr, c->pscr2,
                    c->flag_snap, c->pflag8, c->pflag8s, c->keys, c->perm, c->cell_cnt, c->cell_off, c->tmask, c->air_brick, c->scan_tmp, c->u32_scratch,
                    c->randf, c->seeds, c->mc_numverts, c->mc_tri, c->mc_dens, c->mc_dens2, c->gfm_beta, c->gfm_s, c->mc_cube, c->mc_vflag, c->mc_vscan,
                    c->mc_compact, c->mc_vverts, c->mc_vvscan, c->mc_emark, c->mc_escan, c->mc_vstart, c->mc_inc,
                    c->mc_fill, c->mc_tmpv, c->pour_pos, c->pour_vel};
    k_adj_free(c);
    for (void* p : ptrs) if (p) cudaFree(p);
    for (int a = 0; a < 3; a++) {
        for (float* p : {c->wu[a], c->wuo[a], c->au[a], c->auo[a], c->su[a], c->tmpu[a]}) if (p) cudaFree(p);
        if (c->mc[a].verts) cudaFree(c->mc[a].verts);
        if (c->mc[a].normals) cudaFree(c->mc[a].normals);
        if (c->mc[a].indices) cudaFree(c->mc[a].indices);
    }
    for (auto& e : c->kt_pool) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    for (int k = 0; k < MP_KT_COUNT; k++)
        for (auto& e : c->kt_pending[k]) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
}

static size_t scan_scratch(size_t n) {
    size_t tot = 64;
    while (n > 4096) { size_t nb = (n + 4095) / 4096; tot += 2 * nb + 2; n = nb; }
    return tot;
}

static int create_impl(MpCtx* c, const mp_params* p) {
    c->P = *p;
    memset(&c->S, 0, sizeof(c->S));
    MP_CUDA(c, cudaGetDevice(&c->device));
    MP_CUDA(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
    mpk::Grid& g = c->G;
    g.NX = p->nx; g.NY = p->ny; g.NZ = p->nz;
    g.n = g.NX * g.NY * g.NZ;
    g.nfx = (g.NX + 1) * g.NY * g.NZ; g.nfy = g.NX * (g.NY + 1) * g.NZ; g.nfz = g.NX * g.NY * (g.NZ + 1);
    g.h = p->cellsize; g.gx0 = p->gmin_x; g.gy0 = p->gmin_y; g.gz0 = p->gmin_z;
    size_t n = g.n;
    float** cellf[] = {&c->press, &c->divg, &c->lsfluid, &c->lsair, &c->lsmerge, &c->phifluid, &c->phiair, &c->phisolid,
                       &c->gx, &c->gy, &c->gz, &c->gxa, &c->gya, &c->gza, &c->sf, &c->Tp, &c->Tp_save, &c->Tp_old,
                       &c->fixedheat, &c->cell_tmp, &c->cg_r, &c->cg_p, &c->cg_z};
    for (float** f : cellf) { MP_TRY(dalloc_t(c, f, n)); MP_CUDA(c, cudaMemset(*f, 0, sizeof(float) * n)); }
    MP_TRY(dalloc_t(c, &c->mark, n)); MP_TRY(dalloc_t(c, &c->mark_tmp, n));
    MP_CUDA(c, cudaMemset(c->mark, 0, n));
    {   // fixed heat defaults to "not fixed"
        std::vector<float> u(n, MP_UNDEF_TEMPERATURE);
        MP_CUDA(c, cudaMemcpy(c->fixedheat, u.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    }
    size_t nf[3] = {(size_t)g.nfx, (size_t)g.nfy, (size_t)g.nfz};
    for (int a = 0; a < 3; a++) {
        for (float** f : {&c->wu[a], &c->wuo[a], &c->au[a], &c->auo[a], &c->su[a], &c->tmpu[a]}) {
            MP_TRY(dalloc_t(c, f, nf[a]));
            MP_CUDA(c, cudaMemset(*f, 0, sizeof(float) * nf[a]));
        }
    }
    MP_TRY(dalloc_t(c, &c->cg64, 5 * n));
    c->red_blocks = mp_blocks((long long)n, 256);
    if (const char* e = getenv("MP_CG_KERNEL")) c->cg_use_tma = strcmp(e, "v4") != 0;
    if (const char* e = getenv("MP_CG_TMA_CHUNK")) c->cg_tma_chunk = atoi(e);
    MP_TRY(dalloc_t(c, &c->red, (size_t)148 * 32 * 6));
    MP_TRY(dalloc_t(c, &c->scal, 16));
    MP_TRY(dalloc_t(c, &c->red_count, 16));
    MP_CUDA(c, cudaMemset(c->red_count, 0, 16 * sizeof(unsigned int)));
    MP_CUDA(c, cudaMemset(c->scal, 0, 16 * sizeof(double)));
    size_t cap = (size_t)std::max(p->par_num_max, 1);
    for (float4** f : {&c->pos, &c->vel, &c->heat, &c->pos2, &c->vel2, &c->heat2, &c->pscr, &c->pscr2})
        MP_TRY(dalloc_t(c, f, cap));
    MP_TRY(dalloc_t(c, &c->pdens, cap)); MP_TRY(dalloc_t(c, &c->pprs, cap));
    size_t n8 = c->P.b_run_mc ? 8 * n : n;
    size_t kcap = std::max(cap, n) + 1;
    MP_TRY(dalloc_t(c, &c->keys, kcap)); MP_TRY(dalloc_t(c, &c->perm, kcap));
    MP_TRY(dalloc_t(c, &c->pflag8, cap)); MP_TRY(dalloc_t(c, &c->pflag8s, cap));
    MP_TRY(dalloc_t(c, &c->cell_cnt, n8 + 1)); MP_TRY(dalloc_t(c, &c->cell_off, n8 + 1));
    MP_CUDA(c, cudaMemset(c->cell_cnt, 0, sizeof(uint32_t) * (n8 + 1)));
    MP_CUDA(c, cudaMemset(c->cell_off, 0, sizeof(uint32_t) * (n8 + 1)));
    {
        const size_t bricks = (size_t)((p->nx + 3) / 4) * ((p->ny + 3) / 4) * ((p->nz + 3) / 4);
        c->air_brick_words = (bricks + 31) / 32;
        MP_TRY(dalloc_t(c, &c->air_brick, c->air_brick_words));
        MP_CUDA(c, cudaMemset(c->air_brick, 0, sizeof(uint32_t) * c->air_brick_words));
    }
    // type masks are OR-ed in by 32-bit words: whole words
    const size_t n8w = (n8 + 3) / 4 * 4;
    MP_TRY(dalloc_t(c, &c->tmask, n8w));
    MP_CUDA(c, cudaMemset(c->tmask, 0, n8w));
    MP_TRY(dalloc_t(c, &c->u32_scratch, 16));
    // marching cubes tables and buffers
    MP_TRY(dalloc_t(c, &c->mc_numverts, 256)); MP_TRY(dalloc_t(c, &c->mc_tri, 256 * 16));
    {
        int32_t nv[256], tri[256 * 16];
        mp_internal_mc_tables(nv, tri, nullptr);
        MP_CUDA(c, cudaMemcpy(c->mc_numverts, nv, sizeof(nv), cudaMemcpyHostToDevice));
        MP_CUDA(c, cudaMemcpy(c->mc_tri, tri, sizeof(tri), cudaMemcpyHostToDevice));
    }
    size_t scan_max = std::max(kcap, n8 + 1);
    if (c->P.b_run_mc) {
        size_t nnode = (size_t)(2 * g.NX + 1) * (2 * g.NY + 1) * (2 * g.NZ + 1);
        size_t nvox = 8 * n;
        c->mc_edges = 3 * nnode;
        MP_TRY(dalloc_t(c, &c->mc_dens, nnode)); MP_TRY(dalloc_t(c, &c->mc_dens2, nnode));
        MP_TRY(dalloc_t(c, &c->mc_cube, nvox));
        MP_TRY(dalloc_t(c, &c->mc_vflag, nvox)); MP_TRY(dalloc_t(c, &c->mc_vscan, nvox + 1));
        MP_TRY(dalloc_t(c, &c->mc_compact, nvox));
        MP_TRY(dalloc_t(c, &c->mc_vverts, nvox)); MP_TRY(dalloc_t(c, &c->mc_vvscan, nvox + 1));
        MP_TRY(dalloc_t(c, &c->mc_emark, c->mc_edges)); MP_TRY(dalloc_t(c, &c->mc_escan, c->mc_edges + 1));
        size_t mv = (size_t)c->P.mc_max_verts, mi = 3 * (size_t)c->P.mc_max_tris;
        MP_TRY(dalloc_t(c, &c->mc_vstart, mv + 1)); MP_TRY(dalloc_t(c, &c->mc_fill, mv + 1));
        MP_TRY(dalloc_t(c, &c->mc_inc, mi)); MP_TRY(dalloc_t(c, &c->mc_tmpv, mv));
        for (int a = 0; a < 3; a++) {
            MP_TRY(dalloc_t(c, &c->mc[a].verts, mv)); MP_TRY(dalloc_t(c, &c->mc[a].normals, mv));
            MP_TRY(dalloc_t(c, &c->mc[a].indices, mi));
        }
        scan_max = std::max(scan_max, std::max(c->mc_edges + 1, mv + 1));
    }
    c->scan_tmp_elems = scan_scratch(scan_max);
    MP_TRY(dalloc_t(c, &c->scan_tmp, c->scan_tmp_elems));
    MP_CUDA(c, cudaDeviceSynchronize());
    return MP_OK;
}

static MpCtx* C(void* ctx) { return reinterpret_cast<MpCtx*>(ctx); }
#define CTX_OR_ARG(c) do { if (!(c)) return MP_ERR_ARG; } while (0)

static int check_params(const mp_params* p, std::string& err) {
    if (!p) { err = "null params"; return MP_ERR_ARG; }
    if (p->version != MP_PARAMS_VERSION) { err = "params version mismatch"; return MP_ERR_ARG; }
    if (p->nx < 4 || p->ny < 4 || p->nz < 4) { err = "grid must be at least 4^3"; return MP_ERR_ARG; }
    // row-per-block launches put i and j in the grid's z and y extents
    if (p->nx > 65534 || p->ny > 65534) { err = "grid x and y extents must be below 65535"; return MP_ERR_ARG; }
    long long n = (long long)p->nx * p->ny * p->nz;
    if (8 * n + 1 > 0x7fffffffLL || 3LL * (2 * p->nx + 1) * (2 * p->ny + 1) * (2 * p->nz + 1) > 0x7fffffffLL) {
        err = "grid too large for 32-bit indexing"; return MP_ERR_ARG;
    }
    if (p->par_num_max < 0) { err = "par_num_max < 0"; return MP_ERR_ARG; }
    if (!(p->cellsize > 0) || !(p->dt > 0)) { err = "cellsize and dt must be positive"; return MP_ERR_ARG; }
    if (p->mc_every < 0 || p->smooth_iters < 0 || p->cg_max_iter < 0 || p->heat_cg_max_iter < 0) { err = "negative count"; return MP_ERR_ARG; }
    if (p->scene < 0 || p->scene > MP_SCENE_ALL) { err = "bad scene"; return MP_ERR_ARG; }
    if (p->precision != MP_PREC_MIXED && p->precision != MP_PREC_FP64) { err = "bad precision"; return MP_ERR_ARG; }
    if (p->cg_tol_mode != MP_TOL_REF_ABS && p->cg_tol_mode != MP_TOL_REL) { err = "bad cg_tol_mode"; return MP_ERR_ARG; }
    if (p->coef_mode != MP_COEF_REF && p->coef_mode != MP_COEF_GFM) { err = "unknown coef_mode"; return MP_ERR_ARG; }
    if (!(p->cg_refine_tol >= 0.0f && p->cg_refine_tol < 1.0f)) { err = "cg_refine_tol must be in [0, 1)"; return MP_ERR_ARG; }
    if (p->coef_mode == MP_COEF_GFM && !(p->density_ratio > 0)) { err = "density_ratio must be positive"; return MP_ERR_ARG; }
    if (p->mc_max_verts < 1 || p->mc_max_tris < 1) { err = "marching-cubes caps must be positive"; return MP_ERR_ARG; }
    if (p->seed_redraw != 0) {
        // updateSeedCell draws with the host's rand(): not part of this step;
        // the nucleation cells stay those of mp_set_tables
        err = "seed_redraw is not supported: set the nucleation cells with mp_set_tables"; return MP_ERR_ARG;
    }
    return MP_OK;
}

static thread_local std::string g_create_err;
// context-free calls report through the same slot (mp_last_error(NULL, ...))
void mp_internal_set_global_error(const char* msg) { g_create_err = msg; }

extern "C" int mp_create(const mp_params* p, void** ctx) {
    if (!ctx) return MP_ERR_ARG;
    *ctx = nullptr;
    int rc = check_params(p, g_create_err);
    if (rc) return rc;
    MpCtx* c = new (std::nothrow) MpCtx();
    if (!c) return MP_ERR_CAPACITY;
    rc = create_impl(c, p);
    if (rc != MP_OK) { g_create_err = c->err; free_all(c); delete c; return rc; }
    *ctx = c;
    return MP_OK;
}

extern "C" int mp_destroy(void* ctx) {
    MpCtx* c = C(ctx);
    CTX_OR_ARG(c);
    cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
    return MP_OK;
}

extern "C" int mp_set_params(void* ctx, const mp_params* p) {
    MpCtx* c = C(ctx);
    CTX_OR_ARG(c);
    int rc = check_params(p, c->err);
    if (rc) return rc;
    if (p->nx != c->P.nx || p->ny != c->P.ny || p->nz != c->P.nz || p->par_num_max != c->P.par_num_max ||
        p->b_run_mc != c->P.b_run_mc || p->mc_max_verts != c->P.mc_max_verts || p->mc_max_tris != c->P.mc_max_tris) {
        c->err = "grid size, capacity and marching-cubes buffers are fixed at mp_create";
        return MP_ERR_ARG;
    }
    c->P = *p;
    c->G.h = p->cellsize; c->G.gx0 = p->gmin_x; c->G.gy0 = p->gmin_y; c->G.gz0 = p->gmin_z;
    return MP_OK;
}
extern "C" int mp_get_params(void* ctx, mp_params* p) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); if (!p) return MP_ERR_ARG;
    *p = c->P; return MP_OK;
}
extern "C" int mp_get_state(void* ctx, mp_state* s) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); if (!s) return MP_ERR_ARG;
    *s = c->S; return MP_OK;
}
extern "C" int mp_set_state(void* ctx, const mp_state* s) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); if (!s) return MP_ERR_ARG;
    if (s->par_num_now < 0 || s->par_num_now > c->P.par_num_max) { c->err = "par_num_now out of range"; return MP_ERR_ARG; }
    c->S.frame = s->frame; c->S.par_num_now = s->par_num_now; c->S.n_real_solpoint = s->n_real_solpoint;
    return MP_OK;
}
extern "C" int mp_last_error(void* ctx, char* buf, size_t len) {
    if (!buf || len == 0) return MP_ERR_ARG;
    const std::string& e = ctx ? C(ctx)->err : g_create_err;
    size_t k = std::min(len - 1, e.size());
    memcpy(buf, e.data(), k);
    buf[k] = 0;
    return MP_OK;
}
extern "C" int mp_set_stream(void* ctx, void* stream) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->own_stream) { cudaStreamDestroy(c->stream); c->own_stream = false; }
    c->stream = (cudaStream_t)stream;
    return MP_OK;
}
extern "C" int mp_get_stream(void* ctx, void** stream) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); if (!stream) return MP_ERR_ARG;
    *stream = (void*)c->stream; return MP_OK;
}
extern "C" int mp_synchronize(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}
extern "C" int mp_get_device(void* ctx, int* device) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); if (!device) return MP_ERR_ARG;
    *device = c->device; return MP_OK;
}

// ---------------------------------------------------------------------------
// data in / out
// ---------------------------------------------------------------------------
// every flag one of the particle types (the stages select on them, and the
// sort keeps the low three bits as the type)
static bool flags_valid(const int8_t* flag, int n) {
    for (int p = 0; p < n; p++)
        if (flag[p] < 0 || flag[p] >= MP_TYPECNT) return false;
    return true;
}
extern "C" int mp_upload_particles(void* ctx, int n, const float* pos3, const float* vel3, const int8_t* flag,
                                   const float* mass, const float* temp, const float* lheat, const float* sol,
                                   const float* gas) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (n < 0 || (n > 0 && (!pos3 || !flag || !mass))) { c->err = "upload: bad arguments"; return MP_ERR_ARG; }
    if (n > c->P.par_num_max) { c->err = "upload: more particles than par_num_max"; return MP_ERR_CAPACITY; }
    if (!flags_valid(flag, n)) { c->err = "upload: a particle flag is not an MP_TYPE* value"; return MP_ERR_ARG; }
    MP_TRY(k_pack_particles(c, n, pos3, vel3, flag, mass, temp, lheat, sol, gas));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->S.par_num_now = n;
    c->mc_sorted = 0;
    return MP_OK;
}
extern "C" int mp_download_particles(void* ctx, int* n, float* pos3, float* vel3, int8_t* flag, float* mass,
                                     float* temp, float* lheat, float* sol, float* gas) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (n) *n = c->np();
    return k_unpack_particles(c, c->np(), pos3, vel3, flag, mass, temp, lheat, sol, gas);
}

static void* field_dev(MpCtx* c, int f, size_t& count, size_t& eb) {
    const mpk::Grid& g = c->G;
    eb = 4;
    switch (f) {
    case MP_F_PRESS: count = g.n; return c->press;
    case MP_F_DIV: count = g.n; return c->divg;
    case MP_F_LSFLUID: count = g.n; return c->lsfluid;
    case MP_F_LSAIR: count = g.n; return c->lsair;
    case MP_F_LSMERGE: count = g.n; return c->lsmerge;
    case MP_F_PHIFLUID: count = g.n; return c->phifluid;
    case MP_F_PHIAIR: count = g.n; return c->phiair;
    case MP_F_PHISOLID: count = g.n; return c->phisolid;
    case MP_F_PHIGRAX: count = g.n; return c->gx;
    case MP_F_PHIGRAY: count = g.n; return c->gy;
    case MP_F_PHIGRAZ: count = g.n; return c->gz;
    case MP_F_PHIGRAX_AIR: count = g.n; return c->gxa;
    case MP_F_PHIGRAY_AIR: count = g.n; return c->gya;
    case MP_F_PHIGRAZ_AIR: count = g.n; return c->gza;
    case MP_F_SURFTENSION: count = g.n; return c->sf;
    case MP_F_TP: count = g.n; return c->Tp;
    case MP_F_TP_SAVE: count = g.n; return c->Tp_save;
    case MP_F_TP_OLD: count = g.n; return c->Tp_old;
    case MP_F_FIXEDHEAT: count = g.n; return c->fixedheat;
    case MP_F_MARK: count = g.n; eb = 1; return c->mark;
    case MP_F_WATERUX: count = g.nfx; return c->wu[0];
    case MP_F_WATERUY: count = g.nfy; return c->wu[1];
    case MP_F_WATERUZ: count = g.nfz; return c->wu[2];
    case MP_F_WATERUX_OLD: count = g.nfx; return c->wuo[0];
    case MP_F_WATERUY_OLD: count = g.nfy; return c->wuo[1];
    case MP_F_WATERUZ_OLD: count = g.nfz; return c->wuo[2];
    case MP_F_AIRUX: count = g.nfx; return c->au[0];
    case MP_F_AIRUY: count = g.nfy; return c->au[1];
    case MP_F_AIRUZ: count = g.nfz; return c->au[2];
    case MP_F_AIRUX_OLD: count = g.nfx; return c->auo[0];
    case MP_F_AIRUY_OLD: count = g.nfy; return c->auo[1];
    case MP_F_AIRUZ_OLD: count = g.nfz; return c->auo[2];
    case MP_F_SOLIDUX: count = g.nfx; return c->su[0];
    case MP_F_SOLIDUY: count = g.nfy; return c->su[1];
    case MP_F_SOLIDUZ: count = g.nfz; return c->su[2];
    default: count = 0; return nullptr;
    }
}

extern "C" int mp_field_info(void* ctx, int f, size_t* count, size_t* eb) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    size_t cnt = 0, e = 4;
    if (f == MP_F_CELLSTART || f == MP_F_CELLEND) { cnt = c->G.n; e = 4; }
    else if (f == MP_P_POS || f == MP_P_VEL) { cnt = 3 * (size_t)c->np(); e = 4; }
    else if (f == MP_P_FLAG) { cnt = c->np(); e = 1; }
    else if (f >= MP_P_MASS && f <= MP_P_GASCONTAIN) { cnt = c->np(); e = 4; }
    else if (!field_dev(c, f, cnt, e)) { c->err = "unknown field"; return MP_ERR_ARG; }
    if (count) *count = cnt;
    if (eb) *eb = e;
    return MP_OK;
}

// particle attribute <-> (float4 stream, component)
static bool pattr(int f, int& stream, int& comp) {
    switch (f) {
    case MP_P_MASS: stream = 1; comp = 3; return true;
    case MP_P_TEMP: stream = 2; comp = 0; return true;
    case MP_P_LHEAT: stream = 2; comp = 1; return true;
    case MP_P_SOLUBILITY: stream = 2; comp = 2; return true;
    case MP_P_GASCONTAIN: stream = 2; comp = 3; return true;
    default: return false;
    }
}

extern "C" int mp_get_field(void* ctx, int f, void* dst, size_t bytes) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    size_t cnt, e;
    MP_TRY(mp_field_info(ctx, f, &cnt, &e));
    if (bytes != cnt * e || (bytes && !dst)) { c->err = "get_field: size mismatch"; return MP_ERR_ARG; }
    if (!bytes) return MP_OK;
    if (c->mc_sorted && (f == MP_F_CELLSTART || f == MP_F_CELLEND)) { c->err = "cell ranges are on the 2x grid"; return MP_ERR_STATE; }
    int np = c->np();
    if (f == MP_F_CELLSTART || f == MP_F_CELLEND) {
        uint32_t* st = c->keys; uint32_t* en = c->perm;   // scratch, n entries each
        MP_TRY(k_cells_to_startend(c, st, en));
        MP_CUDA(c, cudaMemcpyAsync(dst, f == MP_F_CELLSTART ? st : en, bytes, cudaMemcpyDeviceToHost, c->stream));
    } else if (f >= MP_P_POS && f <= MP_P_GASCONTAIN) {
        std::vector<float> p3, v3, m, T, L, so, ga;
        std::vector<int8_t> fl;
        p3.resize(3 * (size_t)np); v3.resize(3 * (size_t)np); fl.resize(np); m.resize(np); T.resize(np);
        L.resize(np); so.resize(np); ga.resize(np);
        MP_TRY(k_unpack_particles(c, np, p3.data(), v3.data(), fl.data(), m.data(), T.data(), L.data(), so.data(), ga.data()));
        const void* src = nullptr;
        switch (f) {
        case MP_P_POS: src = p3.data(); break;
        case MP_P_VEL: src = v3.data(); break;
        case MP_P_FLAG: src = fl.data(); break;
        case MP_P_MASS: src = m.data(); break;
        case MP_P_TEMP: src = T.data(); break;
        case MP_P_LHEAT: src = L.data(); break;
        case MP_P_SOLUBILITY: src = so.data(); break;
        default: src = ga.data(); break;
        }
        memcpy(dst, src, bytes);
        return MP_OK;
    } else {
        void* d = field_dev(c, f, cnt, e);
        MP_CUDA(c, cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    }
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

extern "C" int mp_set_field(void* ctx, int f, const void* src, size_t bytes) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    size_t cnt, e;
    MP_TRY(mp_field_info(ctx, f, &cnt, &e));
    if (bytes != cnt * e || (bytes && !src)) { c->err = "set_field: size mismatch"; return MP_ERR_ARG; }
    if (f == MP_F_CELLSTART || f == MP_F_CELLEND) { c->err = "cell ranges are derived by mp_hash_sort"; return MP_ERR_ARG; }
    if (!bytes) return MP_OK;
    if (f >= MP_P_POS && f <= MP_P_GASCONTAIN) {
        int np = c->np();
        std::vector<float> p3(3 * (size_t)np), v3(3 * (size_t)np), m(np), T(np), L(np), so(np), ga(np);
        std::vector<int8_t> fl(np);
        MP_TRY(k_unpack_particles(c, np, p3.data(), v3.data(), fl.data(), m.data(), T.data(), L.data(), so.data(), ga.data()));
        void* dstp = nullptr;
        switch (f) {
        case MP_P_POS: dstp = p3.data(); break;
        case MP_P_VEL: dstp = v3.data(); break;
        case MP_P_FLAG: dstp = fl.data(); break;
        case MP_P_MASS: dstp = m.data(); break;
        case MP_P_TEMP: dstp = T.data(); break;
        case MP_P_LHEAT: dstp = L.data(); break;
        case MP_P_SOLUBILITY: dstp = so.data(); break;
        default: dstp = ga.data(); break;
        }
        if (f == MP_P_FLAG && !flags_valid(static_cast<const int8_t*>(src), np)) {
            c->err = "set_field: a particle flag is not an MP_TYPE* value"; return MP_ERR_ARG;
        }
        memcpy(dstp, src, bytes);
        MP_TRY(k_pack_particles(c, np, p3.data(), v3.data(), fl.data(), m.data(), T.data(), L.data(), so.data(), ga.data()));
    } else {
        void* d = field_dev(c, f, cnt, e);
        MP_CUDA(c, cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, c->stream));
    }
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

extern "C" int mp_set_tables(void* ctx, const float* randfloat, int nrand, const int32_t* seeds, int nseed) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (nrand <= 200 || !randfloat || nseed < 0 || (nseed > 0 && !seeds)) { c->err = "set_tables: need > 200 random values"; return MP_ERR_ARG; }
    // a table being replaced counts as absent until its new array exists, so
    // a failed allocation leaves "not set" (which the stages check), not a
    // size over a freed array
    if (nrand != c->nrand) {
        if (c->randf) cudaFree(c->randf);
        c->randf = nullptr; c->nrand = 0;
        MP_TRY(dalloc_t(c, &c->randf, nrand));
        c->nrand = nrand;
    }
    if (nseed != c->nseed || !c->seeds) {
        if (c->seeds) cudaFree(c->seeds);
        c->seeds = nullptr; c->nseed = 0;
        MP_TRY(dalloc_t(c, &c->seeds, std::max(nseed, 1)));
        c->nseed = nseed;
    }
    MP_CUDA(c, cudaMemcpyAsync(c->randf, randfloat, sizeof(float) * nrand, cudaMemcpyHostToDevice, c->stream));
    if (nseed) MP_CUDA(c, cudaMemcpyAsync(c->seeds, seeds, sizeof(int32_t) * nseed, cudaMemcpyHostToDevice, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

// ---------------------------------------------------------------------------
// adjoint of the FLUID and AIR step (k_adjoint.cu)
// ---------------------------------------------------------------------------
extern "C" int mp_adj_record(void* ctx, int nsteps, int checkpoint_every) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_adj_record(c, nsteps, checkpoint_every);
}
extern "C" int mp_adj_set_targets(void* ctx, const float* samples3, int nsamples) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_adj_set_targets(c, samples3, nsamples);
}
extern "C" int mp_adj_info(void* ctx, int* np, int* nsteps) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_adj_np(c, np, nsteps);
}
extern "C" int mp_adj_order(void* ctx, uint32_t* ids) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!ids) return MP_ERR_ARG;
    return k_adj_order(c, ids);
}
extern "C" int mp_adj_loss(void* ctx, int precision, const double* v0, double* loss) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!loss || (precision != MP_PREC_MIXED && precision != MP_PREC_FP64)) return MP_ERR_ARG;
    return k_adj_run(c, precision, v0, nullptr, loss);
}
extern "C" int mp_adj_gradient(void* ctx, int precision, const double* v0, double* grad_v0, double* loss) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!grad_v0 || (precision != MP_PREC_MIXED && precision != MP_PREC_FP64)) return MP_ERR_ARG;
    return k_adj_run(c, precision, v0, grad_v0, loss);
}
extern "C" int mp_adj_forward(void* ctx, int precision, const mp_grad* in, mp_grad* out) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!out || (precision != MP_PREC_MIXED && precision != MP_PREC_FP64)) return MP_ERR_ARG;
    return k_adj_forward(c, precision, in, out);
}
extern "C" int mp_step_adjoint(void* ctx, int precision, const mp_grad* in, const mp_grad* dout, mp_grad* din) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!dout || !din || (precision != MP_PREC_MIXED && precision != MP_PREC_FP64)) return MP_ERR_ARG;
    return k_adj_vjp(c, precision, in, dout, din);
}
extern "C" int mp_adj_level_set_loss(void* ctx, int precision, const double* pos, double* loss, double* dloss_dpos) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!pos || !loss || (precision != MP_PREC_MIXED && precision != MP_PREC_FP64)) return MP_ERR_ARG;
    return k_adj_ls_loss(c, precision, pos, loss, dloss_dpos);
}
extern "C" int mp_adj_release(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c); k_adj_free(c); return MP_OK;
}

// ---------------------------------------------------------------------------
// checkpoint / resume: everything a step starts from. The grid fields are all
// rebuilt from the particles inside a step, except the heat grid (kept, as the
// heat stage reads it before its particle splat overwrites the cells it
// reaches) and the fixed-heat input.
// ---------------------------------------------------------------------------
namespace {
struct CkptHeader {
    char magic[8];
    uint32_t version, params_bytes, state_bytes, pad;
    int64_t np, nrand, nseed, ncell;
    mp_params params;
    mp_state state;
};
constexpr char kCkptMagic[8] = {'M', 'P', 'C', 'K', 'P', 'T', '0', '1'};
size_t ckpt_bytes(const MpCtx* c) {
    return sizeof(CkptHeader) + 3 * sizeof(float4) * (size_t)c->np() + sizeof(float) * (size_t)c->nrand +
           sizeof(int32_t) * (size_t)c->nseed + 2 * sizeof(float) * (size_t)c->G.n;
}
}  // namespace

extern "C" int mp_checkpoint_size(void* ctx, size_t* bytes) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!bytes) return MP_ERR_ARG;
    *bytes = ckpt_bytes(c);
    return MP_OK;
}

extern "C" int mp_checkpoint_save(void* ctx, void* host_dst, size_t bytes) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!host_dst) return MP_ERR_ARG;
    if (bytes < ckpt_bytes(c)) { c->err = "checkpoint_save: buffer smaller than mp_checkpoint_size"; return MP_ERR_CAPACITY; }
    CkptHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, kCkptMagic, 8);
    h.version = 1; h.params_bytes = sizeof(mp_params); h.state_bytes = sizeof(mp_state);
    h.np = c->np(); h.nrand = c->nrand; h.nseed = c->nseed; h.ncell = c->G.n;
    h.params = c->P; h.state = c->S;
    char* o = static_cast<char*>(host_dst);
    memcpy(o, &h, sizeof(h)); o += sizeof(h);
    cudaStream_t s = c->stream;
    const size_t pb = sizeof(float4) * (size_t)h.np;
    if (pb) {
        MP_CUDA(c, cudaMemcpyAsync(o, c->pos, pb, cudaMemcpyDeviceToHost, s)); o += pb;
        MP_CUDA(c, cudaMemcpyAsync(o, c->vel, pb, cudaMemcpyDeviceToHost, s)); o += pb;
        MP_CUDA(c, cudaMemcpyAsync(o, c->heat, pb, cudaMemcpyDeviceToHost, s)); o += pb;
    }
    if (h.nrand) { MP_CUDA(c, cudaMemcpyAsync(o, c->randf, sizeof(float) * h.nrand, cudaMemcpyDeviceToHost, s)); o += sizeof(float) * h.nrand; }
    if (h.nseed) { MP_CUDA(c, cudaMemcpyAsync(o, c->seeds, sizeof(int32_t) * h.nseed, cudaMemcpyDeviceToHost, s)); o += sizeof(int32_t) * h.nseed; }
    MP_CUDA(c, cudaMemcpyAsync(o, c->fixedheat, sizeof(float) * h.ncell, cudaMemcpyDeviceToHost, s)); o += sizeof(float) * h.ncell;
    MP_CUDA(c, cudaMemcpyAsync(o, c->Tp, sizeof(float) * h.ncell, cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    return MP_OK;
}

extern "C" int mp_checkpoint_load(void* ctx, const void* host_src, size_t bytes) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!host_src || bytes < sizeof(CkptHeader)) { c->err = "checkpoint_load: no or short buffer"; return MP_ERR_ARG; }
    CkptHeader h;
    memcpy(&h, host_src, sizeof(h));
    if (memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1 || h.params_bytes != sizeof(mp_params) ||
        h.state_bytes != sizeof(mp_state)) { c->err = "checkpoint_load: not a checkpoint of this format"; return MP_ERR_ARG; }
    if (memcmp(&h.params, &c->P, sizeof(mp_params)) != 0) {
        c->err = "checkpoint_load: the checkpoint was taken with other parameters";
        return MP_ERR_STATE;
    }
    if (h.np < 0 || h.np > c->P.par_num_max || h.ncell != c->G.n || h.nrand <= 200 || h.nseed < 0) {
        c->err = "checkpoint_load: sizes do not fit this context"; return MP_ERR_ARG;
    }
    // the state's particle count is the one every later kernel runs over
    if (h.state.par_num_now != h.np) {
        c->err = "checkpoint_load: the state's particle count differs from the stored particles"; return MP_ERR_ARG;
    }
    const size_t need = sizeof(CkptHeader) + 3 * sizeof(float4) * (size_t)h.np + sizeof(float) * (size_t)h.nrand +
                        sizeof(int32_t) * (size_t)h.nseed + 2 * sizeof(float) * (size_t)h.ncell;
    if (bytes < need) { c->err = "checkpoint_load: buffer shorter than its header says"; return MP_ERR_ARG; }
    const char* o = static_cast<const char*>(host_src) + sizeof(CkptHeader);
    const float* rf = reinterpret_cast<const float*>(o + 3 * sizeof(float4) * (size_t)h.np);
    const int32_t* sd = reinterpret_cast<const int32_t*>(rf + h.nrand);
    MP_TRY(mp_set_tables(ctx, rf, (int)h.nrand, h.nseed ? sd : nullptr, (int)h.nseed));
    cudaStream_t s = c->stream;
    const size_t pb = sizeof(float4) * (size_t)h.np;
    if (pb) {
        MP_CUDA(c, cudaMemcpyAsync(c->pos, o, pb, cudaMemcpyHostToDevice, s)); o += pb;
        MP_CUDA(c, cudaMemcpyAsync(c->vel, o, pb, cudaMemcpyHostToDevice, s)); o += pb;
        MP_CUDA(c, cudaMemcpyAsync(c->heat, o, pb, cudaMemcpyHostToDevice, s)); o += pb;
    }
    o = reinterpret_cast<const char*>(sd + h.nseed);
    MP_CUDA(c, cudaMemcpyAsync(c->fixedheat, o, sizeof(float) * h.ncell, cudaMemcpyHostToDevice, s)); o += sizeof(float) * h.ncell;
    MP_CUDA(c, cudaMemcpyAsync(c->Tp, o, sizeof(float) * h.ncell, cudaMemcpyHostToDevice, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    c->S = h.state;
    c->mc_sorted = 0;
    return MP_OK;
}

extern "C" int mp_mc_tables(int32_t* num_verts, int32_t* tri, int32_t* edge) {
    mp_internal_mc_tables(num_verts, tri, edge);
    return MP_OK;
}

extern "C" int mp_set_mc_tables(void* ctx, const int32_t* num_verts, const int32_t* tri) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!num_verts || !tri) { c->err = "set_mc_tables: null table"; return MP_ERR_ARG; }
    // the cube's edges as corner pairs, corner v being bit v of the case index
    static const int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                     {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    for (int cs = 0; cs < 256; cs++) {
        int nv = num_verts[cs];
        if (nv < 0 || nv > 15 || nv % 3) { c->err = "set_mc_tables: a vertex count is not 0..15 in steps of 3"; return MP_ERR_ARG; }
        for (int t = 0; t < nv; t++) {
            int e = tri[cs * 16 + t];
            if (e < 0 || e > 11 || ((cs >> kEdge[e][0]) & 1) == ((cs >> kEdge[e][1]) & 1)) {
                c->err = "set_mc_tables: a triangle uses an edge its case does not cross";
                return MP_ERR_ARG;
            }
        }
    }
    MP_CUDA(c, cudaMemcpyAsync(c->mc_numverts, num_verts, sizeof(int32_t) * 256, cudaMemcpyHostToDevice, c->stream));
    MP_CUDA(c, cudaMemcpyAsync(c->mc_tri, tri, sizeof(int32_t) * 256 * 16, cudaMemcpyHostToDevice, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

// ---------------------------------------------------------------------------
// kernel timing
// ---------------------------------------------------------------------------
static void kt_harvest(MpCtx* c, int cls) {
    auto& pend = c->kt_pending[cls];
    size_t keep = 0;
    for (size_t q = 0; q < pend.size(); q++) {
        if (cudaEventQuery(pend[q].second) == cudaSuccess) {
            float ms = 0;
            cudaEventElapsedTime(&ms, pend[q].first, pend[q].second);
            c->kt_ms[cls] += ms;
            c->kt_launch[cls]++;
            c->kt_pool.push_back(pend[q]);
        } else pend[keep++] = pend[q];
    }
    pend.resize(keep);
}
void kt_begin(MpCtx* c, int cls, cudaEvent_t* ev_end) {
    *ev_end = 0;
    if (cls < 0 || cls >= MP_KT_COUNT || !c->kt_on[cls]) return;
    std::pair<cudaEvent_t, cudaEvent_t> e;
    if (!c->kt_pool.empty()) { e = c->kt_pool.back(); c->kt_pool.pop_back(); }
    else { cudaEventCreate(&e.first); cudaEventCreate(&e.second); }
    cudaEventRecord(e.first, c->stream);
    c->kt_pending[cls].push_back(e);
    *ev_end = e.second;
}
void kt_end(MpCtx* c, int cls, cudaEvent_t ev_end) {
    if (!ev_end) return;
    cudaEventRecord(ev_end, c->stream);
    if (c->kt_pending[cls].size() > 4096) { cudaStreamSynchronize(c->stream); kt_harvest(c, cls); }
}
extern "C" int mp_kernel_timing(void* ctx, int cls, int enable) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (cls < 0 || cls >= MP_KT_COUNT) return MP_ERR_ARG;
    c->kt_on[cls] = enable != 0;
    return MP_OK;
}
extern "C" int mp_kernel_timing_read(void* ctx, int cls, double* ms, int64_t* launches) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (cls < 0 || cls >= MP_KT_COUNT) return MP_ERR_ARG;
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    kt_harvest(c, cls);
    if (ms) *ms = c->kt_ms[cls];
    if (launches) *launches = c->kt_launch[cls];
    return MP_OK;
}
extern "C" int mp_kernel_timing_reset(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < MP_KT_COUNT; k++) { kt_harvest(c, k); c->kt_ms[k] = 0; c->kt_launch[k] = 0; }
    c->launches = 0;
    for (int k = 0; k < MP_WC_COUNT; k++) c->work[k] = 0;
    return MP_OK;
}
extern "C" int mp_work_counts(void* ctx, int64_t* counts, int n) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!counts || n < 0) return MP_ERR_ARG;
    for (int k = 0; k < n && k < MP_WC_COUNT; k++) counts[k] = c->work[k];
    return MP_OK;
}
extern "C" int64_t mp_launch_count(void* ctx) {
    MpCtx* c = C(ctx);
    return c ? c->launches : -1;
}

// ---------------------------------------------------------------------------
// stages
// ---------------------------------------------------------------------------
static int need_cells(MpCtx* c) {
    if (c->mc_sorted) { c->err = "particles are sorted on the marching-cubes grid; call mp_hash_sort first"; return MP_ERR_STATE; }
    return MP_OK;
}
#define STAGE(name, body)                                  \
    extern "C" int name(void* ctx) {                       \
        MpCtx* c = C(ctx); CTX_OR_ARG(c);                  \
        body;                                              \
    }

extern "C" int mp_init_particle_heat(void* ctx) { MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_init_particle_heat(c); }
STAGE(mp_hash_sort, return k_hash_sort(c))
STAGE(mp_external_force, return k_external_force(c))
extern "C" int mp_levelset(void* ctx, float offset) {
    (void)offset;   // ignored by genlevelset (spray_k.cu:2803-2804)
    MpCtx* c = C(ctx); CTX_OR_ARG(c); MP_TRY(need_cells(c)); return k_levelset(c);
}
STAGE(mp_sweep_ls_mark, return k_sweep_ls_mark(c))
STAGE(mp_mark_solo_air, MP_TRY(need_cells(c)); return k_mark_solo_air(c))
STAGE(mp_surface_tension, return k_surface_tension(c))
STAGE(mp_markgrid_bubble, MP_TRY(need_cells(c)); return k_markgrid_bubble(c))
STAGE(mp_p2g, MP_TRY(need_cells(c)); return k_p2g(c))
STAGE(mp_drag, MP_TRY(need_cells(c)); return k_drag(c))
extern "C" int mp_sweep_phi(void* ctx, int ph) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (ph != MP_TYPEFLUID && ph != MP_TYPEAIR) return MP_ERR_ARG;
    return k_sweep_phi(c, ph);
}
extern "C" int mp_sweep_u(void* ctx, int ph) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (ph != MP_TYPEFLUID && ph != MP_TYPEAIR) return MP_ERR_ARG;
    return k_sweep_u(c, ph);
}
extern "C" int mp_set_boundary_u(void* ctx, int ph) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (ph != MP_TYPEFLUID && ph != MP_TYPEAIR) return MP_ERR_ARG;
    return k_set_boundary_u(c, ph);
}
extern "C" int mp_project(void* ctx, int* iters, double* residual) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    return k_project(c, iters, residual);
}
STAGE(mp_g2p, return k_g2p(c))
STAGE(mp_solid_motion, return k_solid_motion(c))
STAGE(mp_solo_air_update, MP_TRY(need_cells(c)); return k_solo_air_update(c))
STAGE(mp_collide_advect, MP_TRY(need_cells(c)); return k_collide_advect(c))
STAGE(mp_correct_pos, MP_TRY(need_cells(c)); return k_correct_pos(c))
STAGE(mp_correct_pos_bubble, return k_correct_pos_bubble(c))
STAGE(mp_heat, MP_TRY(need_cells(c)); return k_heat(c))
STAGE(mp_gen_gas, MP_TRY(need_cells(c)); return k_gen_gas(c))
STAGE(mp_delete, return k_delete(c))
STAGE(mp_melt, return k_melt(c))
STAGE(mp_freeze, MP_TRY(need_cells(c)); return k_freeze(c))
STAGE(mp_mc_presort, if (!c->P.b_run_mc) { c->err = "marching cubes disabled at mp_create"; return MP_ERR_STATE; } return k_mc_presort(c))
extern "C" int mp_mc(void* ctx, int surface) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (surface < 0 || surface > 2) return MP_ERR_ARG;
    if (!c->P.b_run_mc) { c->err = "marching cubes disabled at mp_create"; return MP_ERR_STATE; }
    return k_mc(c, surface);
}
extern "C" int mp_mc_download(void* ctx, int surface, float* verts, float* normals, uint32_t* indices, int max_verts,
                              int max_indices) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (surface < 0 || surface > 2 || !c->P.b_run_mc) return MP_ERR_ARG;
    McSurface& m = c->mc[surface];
    if (m.nverts > max_verts || m.nindices > max_indices) { c->err = "mc_download: buffers too small"; return MP_ERR_CAPACITY; }
    if (verts && m.nverts) MP_CUDA(c, cudaMemcpyAsync(verts, m.verts, 12 * (size_t)m.nverts, cudaMemcpyDeviceToHost, c->stream));
    if (normals && m.nverts) MP_CUDA(c, cudaMemcpyAsync(normals, m.normals, 12 * (size_t)m.nverts, cudaMemcpyDeviceToHost, c->stream));
    if (indices && m.nindices) MP_CUDA(c, cudaMemcpyAsync(indices, m.indices, 4 * (size_t)m.nindices, cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}
extern "C" int mp_mc_download_field(void* ctx, float* dens, uint8_t* cube) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!c->P.b_run_mc) return MP_ERR_STATE;
    size_t nnode = (size_t)(2 * c->G.NX + 1) * (2 * c->G.NY + 1) * (2 * c->G.NZ + 1), nvox = 8 * (size_t)c->G.n;
    const float* src = c->mc_last_dens ? c->mc_last_dens : c->mc_dens;
    if (dens) MP_CUDA(c, cudaMemcpyAsync(dens, src, 4 * nnode, cudaMemcpyDeviceToHost, c->stream));
    if (cube) MP_CUDA(c, cudaMemcpyAsync(cube, c->mc_cube, nvox, cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

// ---------------------------------------------------------------------------
// pouring emitters (dpourpos / dpourvel, spray.cpp:1416-1545; spray.cu:3012-3043)
// ---------------------------------------------------------------------------
extern "C" int mp_set_pour(void* ctx, const float* pos3, const float* vel3, int n) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (n < 0 || (n > 0 && (!pos3 || !vel3))) { c->err = "set_pour: bad arguments"; return MP_ERR_ARG; }
    if (n > c->pour_n) {
        if (c->pour_pos) cudaFree(c->pour_pos);
        if (c->pour_vel) cudaFree(c->pour_vel);
        c->pour_pos = c->pour_vel = nullptr; c->pour_n = 0;
        MP_TRY(dalloc_t(c, &c->pour_pos, 3 * (size_t)n));
        MP_TRY(dalloc_t(c, &c->pour_vel, 3 * (size_t)n));
    }
    if (n > 0) {
        MP_CUDA(c, cudaMemcpyAsync(c->pour_pos, pos3, 12 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
        MP_CUDA(c, cudaMemcpyAsync(c->pour_vel, vel3, 12 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
        MP_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    c->pour_n = n;
    return MP_OK;
}
extern "C" int mp_heatsim(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    return k_heatsim(c);
}
extern "C" int mp_init_heat_grid(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    return k_init_heat_grid_launch(c);
}
// ---- the water mode (SIMULATION_WATER) ------------------------------------
extern "C" int mp_flip_mark(void* ctx) { MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_flip_mark(c); }
extern "C" int mp_water_p2g(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    MP_TRY(need_cells(c));
    return k_water_p2g(c);
}
extern "C" int mp_project_water(void* ctx, int* iters, double* res) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    return k_project_water(c, iters, res);
}
extern "C" int mp_water_g2p(void* ctx) { MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_water_g2p(c); }
extern "C" int mp_water_advect(void* ctx) { MpCtx* c = C(ctx); CTX_OR_ARG(c); return k_water_advect(c); }

static int step_output_meshes(MpCtx* c, int F, bool kept_solid, bool fluid_only);

// watersim (spray.cpp:741-797). Where the reference extracts the fluid surface
// from the cell ranges of the last (simulation-grid) sort, this step re-sorts
// on the 2x grid first, as the density pass requires (preMC).
extern "C" int mp_watersim(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    NvtxRange step_range("watersim");
    const mp_params& P = c->P;
    int warn = MP_OK, st;
    MP_STAGE("hashAndSortParticles", k_hash_sort(c));
    MP_STAGE("sweepPhi", k_sweep_phi(c, MP_TYPEFLUID));
    MP_STAGE("computeLevelset", k_levelset(c)); MP_STAGE("sweepLSAndMardGrid", k_sweep_ls_mark(c));
    MP_STAGE("flipMark_sphere", k_flip_mark(c));
    MP_STAGE("computesurfacetension", k_surface_tension(c));
    MP_STAGE("mapvelp2g", k_water_p2g(c));
    MP_STAGE("sweepU", k_sweep_u(c, MP_TYPEFLUID)); MP_STAGE("setWaterBoundaryU", k_set_boundary_u(c, MP_TYPEFLUID));
    {
        NvtxRange r_("project_CG");
        st = k_project_water(c, nullptr, nullptr);
    }
    if (st == MP_ERR_NOCONVERGE) warn = st; else MP_TRY(st);
    MP_STAGE("sweepU", k_sweep_u(c, MP_TYPEFLUID)); MP_STAGE("setWaterBoundaryU", k_set_boundary_u(c, MP_TYPEFLUID));
    MP_STAGE("mapvelg2p", k_water_g2p(c));
    MP_STAGE("wateradvect", k_water_advect(c));
    MP_STAGE("hashAndSortParticles", k_hash_sort(c));
    MP_STAGE("correctpos", k_correct_pos(c));
    int out_rc = MP_OK;
    if (P.b_run_mc) {
        MP_STAGE("preMC", k_mc_presort(c));
        MP_STAGE("runMC_smooth", k_mc(c, MP_MC_FLUID));
        // runMC_fluid's files (spray.cu:954-958, 858-863) on output frames
        if (c->out_on && P.mc_every > 0 && c->S.frame % P.mc_every == 0)
            out_rc = step_output_meshes(c, c->S.frame / P.mc_every, false, true);
    }
    c->S.frame++;
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    MP_CHECK_LAUNCH(c);
    return out_rc != MP_OK ? out_rc : warn;
}

extern "C" int mp_pour(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    return k_pour(c);
}

// the frame-scripted switches of bubblesim (spray.cpp:1007-1047), applied to
// the context's parameters at the start of the step
static void scene_toggles(MpCtx* c) {
    mp_params& P = c->P;
    const int sc = P.scene, f = c->S.frame;
    if (sc == MP_SCENE_ALL && f == 0) {
        P.b_fix_solid = 0; P.b_add_heat_bottom = 0; P.b_gen_gas = 0; P.b_melt = 0;
        P.b_freeze = 1;
    }
    if (sc == MP_SCENE_ALL && f == 500) P.b_freeze = 0;
    if (sc == MP_SCENE_ALL && f == 520) { P.b_add_heat_bottom = 1; P.b_melt = 1; }
    if (sc == MP_SCENE_ALL && f == 1250) P.b_gen_gas = 1;
    if ((sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES) && f == 300) P.b_fix_solid = 0;
    if (sc == MP_SCENE_MELTANDBOIL_HIGHRES && f == 400) P.b_add_heat_bottom = 0;
    if (sc == MP_SCENE_MELTANDBOIL_HIGHRES && f == 700) P.b_add_heat_bottom = 1;
    if (sc == MP_SCENE_MELTANDBOIL && f == 400) P.b_gen_gas = !P.b_gen_gas;
    if (sc == MP_SCENE_MELTANDBOIL && f == 700) {
        P.b_gen_gas = !P.b_gen_gas; P.drag_param_grid = 0.03f; P.vapor_gen_rate = 0.005f;
    }
    if ((sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES) && f == P.begin_frame) P.b_fix_solid = 0;
}

// ---------------------------------------------------------------------------
// per-frame files: the writers of host/export.cpp on the context's data
// ---------------------------------------------------------------------------
// runMC_solid / runMC_fluid / runMC_gas pass these object names (spray.cu:767-784)
static const char* mc_object_name(int surface) {
    return surface == MP_MC_SOLID ? "solid" : (surface == MP_MC_FLUID ? "water" : "gas");
}
static int io_error(MpCtx* c, int rc, const std::string& path) {
    if (rc == MP_ERR_IO) c->err = "cannot open or write " + path;
    else if (rc != MP_OK) c->err = "export: bad arguments for " + path;
    return rc;
}
static int export_mesh(MpCtx* c, int surface, int format, const std::string& path) {
    const McSurface& m = c->mc[surface];
    std::vector<float> v(3 * (size_t)m.nverts), nrm(3 * (size_t)m.nverts);
    std::vector<uint32_t> idx((size_t)m.nindices);
    if (m.nverts) {
        MP_CUDA(c, cudaMemcpyAsync(v.data(), m.verts, 12 * (size_t)m.nverts, cudaMemcpyDeviceToHost, c->stream));
        MP_CUDA(c, cudaMemcpyAsync(nrm.data(), m.normals, 12 * (size_t)m.nverts, cudaMemcpyDeviceToHost, c->stream));
    }
    if (m.nindices)
        MP_CUDA(c, cudaMemcpyAsync(idx.data(), m.indices, 4 * (size_t)m.nindices, cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return io_error(c, mp_write_mesh(format, path.c_str(), mc_object_name(surface), v.data(), nrm.data(), m.nverts,
                                     idx.data(), m.nindices), path);
}
static int export_particles(MpCtx* c, int kind, const std::string& path, float tmin, float tmax) {
    const int np = c->np();
    std::vector<float> pos(3 * (size_t)np), T((size_t)np);
    std::vector<int8_t> flag((size_t)np);
    MP_TRY(k_unpack_particles(c, np, pos.data(), nullptr, flag.data(), nullptr, T.data(), nullptr, nullptr, nullptr));
    return io_error(c, mp_write_particles(kind, path.c_str(), pos.data(), flag.data(), T.data(), np, tmin, tmax), path);
}
static std::string fmt_path(const char* f, const std::string& dir, const char* name, int frame) {
    char buf[64];
    if (name) std::snprintf(buf, sizeof(buf), f, name, frame);
    else std::snprintf(buf, sizeof(buf), f, frame);
    return dir + buf;
}

extern "C" int mp_export_mesh(void* ctx, int surface, int format, const char* path) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!path || surface < 0 || surface > 2 || format < MP_OUT_POV_MESH || format > MP_OUT_BOBJ_GZ) {
        c->err = "export_mesh: bad arguments"; return MP_ERR_ARG;
    }
    if (!c->P.b_run_mc) { c->err = "export_mesh: marching cubes is off (b_run_mc)"; return MP_ERR_STATE; }
    return export_mesh(c, surface, format, path);
}
extern "C" int mp_export_particles(void* ctx, int kind, const char* path, float t_min, float t_max) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!path || kind < MP_OUT_PARTICLES_COLORED || kind > MP_OUT_PARTICLES_AIR) {
        c->err = "export_particles: bad arguments"; return MP_ERR_ARG;
    }
    return export_particles(c, kind, path, t_min, t_max);
}
extern "C" int mp_set_output(void* ctx, const mp_output* o) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    if (!o) { c->out_on = false; return MP_OK; }
    if (!o->dir) { c->err = "set_output: dir is null"; return MP_ERR_ARG; }
    c->out_on = true;
    c->out_dir = o->dir;
    c->out_pov = o->pov; c->out_obj = o->obj; c->out_colored = o->colored_particles;
    c->out_tmin = o->t_render_min; c->out_tmax = o->t_render_max;
    return MP_OK;
}

// the meshes just extracted, as runMC_smooth writes them (spray.cu:858-863,
// 954-958): POV-Ray mesh2 when pov; BOBJ when obj, or an empty OBJ for an
// empty surface; in extraction order solid, water, gas. A solid surface kept
// from frame 0 (runMC_interaction, spray.cu:790-799) goes to a text OBJ.
static int step_output_meshes(MpCtx* c, int F, bool kept_solid, bool fluid_only) {
    for (int s : {MP_MC_SOLID, MP_MC_FLUID, MP_MC_GAS}) {
        if (fluid_only && s != MP_MC_FLUID) continue;
        const char* nm = mc_object_name(s);
        const bool empty = c->mc[s].nverts == 0;
        const bool text_obj = empty || (kept_solid && s == MP_MC_SOLID);
        if (c->out_pov) MP_TRY(export_mesh(c, s, MP_OUT_POV_MESH, fmt_path("waterdata/%s%05d.pov", c->out_dir, nm, F)));
        if (c->out_obj) {
            if (text_obj) MP_TRY(export_mesh(c, s, MP_OUT_OBJ_MESH, fmt_path("waterOBJdata/%s%05d.obj", c->out_dir, nm, F)));
            else MP_TRY(export_mesh(c, s, MP_OUT_BOBJ_GZ,
                                    c->out_dir + nm + fmt_path("BOBJdata/fluidsurface_final_%04d.bobj.gz", "", nullptr, F - 1)));
        }
    }
    return MP_OK;
}
// the particle files at the end of bubblesim (spray.cpp:1208-1216)
static int step_output_particles(MpCtx* c, int F) {
    if (!c->out_pov) return MP_OK;
    const int sc = c->P.scene;
    if (sc == MP_SCENE_INTERACTION)
        MP_TRY(export_particles(c, MP_OUT_PARTICLES_SOLO, fmt_path("waterdata/solobubble%05d.pov", c->out_dir, nullptr, F),
                                c->out_tmin, c->out_tmax));
    if (c->out_colored)
        MP_TRY(export_particles(c, MP_OUT_PARTICLES_COLORED,
                                fmt_path("waterdata/allparticles%05d.pov", c->out_dir, nullptr, F), c->out_tmin, c->out_tmax));
    if (sc == MP_SCENE_BOILING)
        MP_TRY(export_particles(c, MP_OUT_PARTICLES_AIR, fmt_path("waterdata/solobubble%05d.pov", c->out_dir, nullptr, F),
                                c->out_tmin, c->out_tmax));
    return MP_OK;
}

// bubblesim (spray.cpp:979-1233): the stage order and cadence of the reference,
// starting with pouring (spray.cpp:998-1001) and the frame-scripted switches
// (spray.cpp:1007-1047). Seed re-draws with the host rand() are not part of
// this step.
extern "C" int mp_step(void* ctx) {
    MpCtx* c = C(ctx); CTX_OR_ARG(c);
    NvtxRange step_range("bubblesim");
    const mp_params& P = c->P;
    int sc = P.scene;
    int warn = MP_OK, st;
    MP_STAGE("pouring", k_pour(c));
    scene_toggles(c);
    MP_STAGE("hashAndSortParticles", k_hash_sort(c));
    MP_STAGE("addexternalforce", k_external_force(c));
    MP_STAGE("computeLevelset", k_levelset(c)); MP_STAGE("sweepLSAndMardGrid", k_sweep_ls_mark(c));
    MP_STAGE("markSoloAirParticle", k_mark_solo_air(c));
    MP_STAGE("computesurfacetension", k_surface_tension(c));
    if (sc == MP_SCENE_MELTING || sc == MP_SCENE_FREEZING) MP_STAGE("markgrid_bubble", k_markgrid_bubble(c));
    MP_STAGE("mapvelp2g_bubble", k_p2g(c));
    MP_STAGE("enforceDragForce", k_drag(c));
    MP_STAGE("sweepPhi", k_sweep_phi(c, MP_TYPEAIR)); MP_STAGE("sweepU", k_sweep_u(c, MP_TYPEAIR));
    MP_STAGE("sweepPhi", k_sweep_phi(c, MP_TYPEFLUID)); MP_STAGE("sweepU", k_sweep_u(c, MP_TYPEFLUID));
    MP_STAGE("setWaterBoundaryU", k_set_boundary_u(c, MP_TYPEAIR)); MP_STAGE("setWaterBoundaryU", k_set_boundary_u(c, MP_TYPEFLUID));
    {
        NvtxRange r_("project_CG_bubble");
        st = k_project(c, nullptr, nullptr);
    }
    if (st == MP_ERR_NOCONVERGE) warn = st; else MP_TRY(st);
    MP_STAGE("sweepU", k_sweep_u(c, MP_TYPEAIR)); MP_STAGE("sweepU", k_sweep_u(c, MP_TYPEFLUID));
    MP_STAGE("setWaterBoundaryU", k_set_boundary_u(c, MP_TYPEAIR)); MP_STAGE("setWaterBoundaryU", k_set_boundary_u(c, MP_TYPEFLUID));
    MP_STAGE("mapvelg2p_bubble", k_g2p(c));
    MP_STAGE("solidmotion", k_solid_motion(c));
    MP_STAGE("updateSoloAirParticle", k_solo_air_update(c));
    MP_STAGE("hashAndSortParticles", k_hash_sort(c)); MP_STAGE("CollisionSolid", k_collide_advect(c, true));
    if (P.b_correct_position) {
        MP_STAGE("hashAndSortParticles", k_hash_sort(c)); MP_STAGE("correctpos", k_correct_pos(c));
        MP_STAGE("hashAndSortParticles", k_hash_sort(c)); MP_STAGE("computeLevelset", k_levelset(c)); MP_STAGE("sweepLSAndMardGrid", k_sweep_ls_mark(c)); MP_STAGE("correctpos_bubble", k_correct_pos_bubble(c));
    } else {
        MP_STAGE("hashAndSortParticles", k_hash_sort(c)); MP_STAGE("computeLevelset", k_levelset(c)); MP_STAGE("sweepLSAndMardGrid", k_sweep_ls_mark(c));
    }
    MP_STAGE("hashAndSortParticles", k_hash_sort(c));
    if (P.b_heat_trans) {
        {
            NvtxRange r_("updateTemperature");
            st = k_heat(c);
        }
        if (st == MP_ERR_NOCONVERGE) warn = st; else MP_TRY(st);
    }
    if (P.b_gen_gas && c->S.frame % 2 == 0) MP_STAGE("GenerateGasParticle", k_gen_gas(c));
    MP_STAGE("hashAndSortParticles", k_hash_sort(c)); MP_STAGE("deleteAirFluidParticle", k_delete(c));
    MP_STAGE("hashAndSortParticles", k_hash_sort(c));
    if (P.b_melt) MP_STAGE("MeltSolid", k_melt(c));
    if (P.b_freeze) MP_STAGE("Freezing", k_freeze(c));
    const bool out_frame = c->out_on && P.mc_every > 0 && c->S.frame % P.mc_every == 0;
    // runMC_interaction (spray.cu:788-802): with bRunMCSolid off the solid
    // surface of frame 0 is kept, moved by the solid motion, and only its
    // normals are recomputed
    const bool inter = sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES ||
                       sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL;
    const bool kept_solid = inter && c->S.frame > 0 && !P.b_run_mc_solid;
    if (P.b_run_mc && P.mc_every > 0 && c->S.frame % P.mc_every == 0) {
        MP_STAGE("preMC", k_mc_presort(c));
        if (kept_solid) MP_STAGE("runMC_interaction", k_mc_renormal(c, MP_MC_SOLID));
        else MP_STAGE("runMC_smooth", k_mc(c, MP_MC_SOLID));
        MP_STAGE("runMC_fluid_gas", k_mc_fluid_gas(c));
    }
    // a file that cannot be written ends the step's output, not the step
    // (the reference printed and paused); the frame still advances
    int out_rc = MP_OK;
    if (out_frame) {
        const int F = c->S.frame / P.mc_every;
        if (P.b_run_mc) out_rc = step_output_meshes(c, F, kept_solid, false);
        if (out_rc == MP_OK) out_rc = step_output_particles(c, F);
    }
    c->S.frame++;
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    MP_CHECK_LAUNCH(c);
    return out_rc != MP_OK ? out_rc : warn;
}
