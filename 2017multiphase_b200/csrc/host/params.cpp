// params.cpp — the parameter block's table, defaults and derived constants
// (cspray::initparam, Multiphase/Multiphase/spray.cpp:29-78, 573-626). Host
// code only: libmp.so links it, and so does the CPU oracle's library, whose
// scene inputs then come from the same definitions without loading libmp.so.
#include "../../../include/mp.h"
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

struct ParamField { const char* name; int offset; int kind; };
#define PF_I(f) {#f, (int)offsetof(mp_params, f), 0}
#define PF_F(f) {#f, (int)offsetof(mp_params, f), 1}
static const ParamField kParamFields[] = {
    PF_I(version), PF_I(nx), PF_I(ny), PF_I(nz), PF_I(par_num_max), PF_I(scene),
    PF_F(cellsize), PF_F(dt), PF_F(gravity_x), PF_F(gravity_y), PF_F(gravity_z),
    PF_F(gmin_x), PF_F(gmin_y), PF_F(gmin_z), PF_F(samplespace),
    PF_F(m0), PF_F(airm0), PF_F(waterrho), PF_F(solidrho), PF_F(pradius),
    PF_F(poly6kern), PF_F(spikykern), PF_F(lapkern),
    PF_I(b_solid), PF_I(b_melt), PF_I(b_freeze), PF_I(b_fix_solid), PF_I(b_gen_gas), PF_I(b_heat_trans),
    PF_I(b_add_heat_bottom), PF_I(b_extend_heat_to_boundary), PF_I(b_correct_position),
    PF_I(b_smooth_mc), PF_I(b_run_mc), PF_I(mc_every), PF_I(smooth_iters),
    PF_F(surfacetension_sigma), PF_F(heatalpha_fluid), PF_F(heatalpha_air), PF_F(heatalpha_solid),
    PF_F(heatalpha_vacuum), PF_F(default_temperature), PF_F(temperature0), PF_F(melting_point),
    PF_F(boiling_point), PF_F(drag_param_solo), PF_F(drag_param_grid), PF_F(viscosity_sph),
    PF_F(default_solid_T), PF_F(default_liquid_T), PF_F(liquid_heat_th), PF_F(alpha_temp_trans),
    PF_F(bounce_vel_param), PF_F(bounce_pos_param), PF_F(heat_increase_bottom),
    PF_F(bubble_max_vel), PF_F(max_vel_for_bubble), PF_F(buoyance_rate_air), PF_F(buoyance_rate_solo),
    PF_F(vapor_gen_rate), PF_F(init_dissolve_gas_rate), PF_F(init_gas_rate),
    PF_F(correction_spring), PF_F(correction_radius), PF_F(mc_density), PF_F(heat_clamp),
    PF_F(solubility_coef), PF_F(solid_bounce_param), PF_F(flip_alpha), PF_I(cg_tol_mode), PF_F(cg_tol),
    PF_I(cg_max_iter), PF_I(heat_cg_max_iter), PF_I(cg_true_residual_every), PF_I(precision),
    PF_I(coef_mode), PF_F(density_ratio), PF_I(mc_max_verts), PF_I(mc_max_tris), PF_I(seed_redraw),
    PF_I(update_seed_frame_delta), PF_I(b_fixed_heat), PF_F(pos_rand_param), PF_F(vel_rand_param),
    PF_I(begin_frame), PF_I(b_run_mc_solid), PF_F(cg_refine_tol),
};

extern "C" int mp_params_size(void) { return (int)sizeof(mp_params); }

extern "C" int mp_params_describe(int index, const char** name, int* offset, int* kind) {
    int cnt = (int)(sizeof(kParamFields) / sizeof(kParamFields[0]));
    if (index < 0 || index >= cnt) return MP_ERR_ARG;
    if (name) *name = kParamFields[index].name;
    if (offset) *offset = kParamFields[index].offset;
    if (kind) *kind = kParamFields[index].kind;
    return MP_OK;
}

// spray.cpp:573-588: m0 from the sample spacing, SPH kernel constants from the cell size
extern "C" int mp_params_derive(mp_params* p) {
    if (!p) return MP_ERR_ARG;
    p->m0 = (1.0f * p->waterrho) / powf(1.0f / p->samplespace, 3.0f);
    p->airm0 = p->m0;
    p->pradius = (float)pow((double)(p->m0 / p->waterrho * 3.0f / 4.0f) / M_PI, 1.0 / 3.0f);
    p->poly6kern = 315.0f / (64.0f * 3.141592f * powf(p->cellsize, 9.0f));
    p->spikykern = -45.0f / (3.141592f * powf(p->cellsize, 6.0f));
    p->lapkern = 45.0f / (3.141592f * powf(p->cellsize, 6.0f));
    p->max_vel_for_bubble = p->cellsize / p->dt;
    return MP_OK;
}

// cspray::initparam defaults (spray.cpp:29-78, 573-626) with the MULTIBUBBLE
// scene switches (spray.cpp:191-214)
extern "C" int mp_params_default(mp_params* p, int nx, int ny, int nz, int par_num_max) {
    if (!p || nx < 4 || ny < 4 || nz < 4 || par_num_max < 0) return MP_ERR_ARG;
    memset(p, 0, sizeof(*p));
    p->version = MP_PARAMS_VERSION;
    p->nx = nx; p->ny = ny; p->nz = nz; p->par_num_max = par_num_max;
    p->scene = MP_SCENE_MULTIBUBBLE;
    p->cellsize = 1.0f / 64;
    p->dt = 0.003f;
    p->gravity_x = 0; p->gravity_y = 0; p->gravity_z = -9.8f;
    p->samplespace = 0.5f * p->cellsize;
    p->waterrho = 1000.0f; p->solidrho = 800.0f;
    p->b_solid = 0; p->b_melt = 0; p->b_freeze = 0; p->b_fix_solid = 0; p->b_gen_gas = 0; p->b_heat_trans = 0;
    p->b_add_heat_bottom = 0; p->b_extend_heat_to_boundary = 0; p->b_correct_position = 1;
    p->b_smooth_mc = 1; p->b_run_mc = 1; p->mc_every = 2; p->smooth_iters = 5;
    p->surfacetension_sigma = 0.0f;
    p->heatalpha_fluid = 0.02f; p->heatalpha_air = 0.008f; p->heatalpha_solid = 0.2f; p->heatalpha_vacuum = 0.0001f;
    p->default_temperature = 293.15f; p->temperature0 = 273.15f;
    p->melting_point = 273.15f; p->boiling_point = 373.15f;
    p->drag_param_solo = 10; p->drag_param_grid = 0.05f; p->viscosity_sph = 1.8f;
    p->default_solid_T = 263.15f; p->default_liquid_T = 293.15f; p->liquid_heat_th = 10; p->alpha_temp_trans = 0.0f;
    p->bounce_vel_param = 1.0f; p->bounce_pos_param = 0;
    p->heat_increase_bottom = 0.0f;
    p->bubble_max_vel = 6.5f;
    p->buoyance_rate_air = 1.25f; p->buoyance_rate_solo = 1.05f;
    p->vapor_gen_rate = 0.01f; p->init_dissolve_gas_rate = 1.0f; p->init_gas_rate = 0.7f;
    p->correction_spring = 500000.0f; p->correction_radius = 0.5f;
    p->mc_density = 0.5f;
    p->heat_clamp = 378.0f;
    p->solubility_coef = 1018.9f;
    p->solid_bounce_param = 0.5f;
    p->flip_alpha = 1.0f;
    p->cg_tol_mode = MP_TOL_REF_ABS; p->cg_tol = 0.01f;
    p->cg_max_iter = 800; p->heat_cg_max_iter = 3800; p->cg_true_residual_every = 0;
    p->precision = MP_PREC_MIXED; p->coef_mode = MP_COEF_REF; p->density_ratio = 1000.0f;
    // the reference fixes 6e6 vertices / 12e6 triangles (spray.cu:721-722); here the
    // caps scale with the 2x grid's cross-section (a few surface layers)
    long long mv = std::max(100000LL, 64LL * (2 * nx) * (2 * ny));
    mv = std::min(mv, 64000000LL);
    p->mc_max_verts = (int)mv; p->mc_max_tris = (int)std::min(2 * mv, 128000000LL);
    p->seed_redraw = 0; p->update_seed_frame_delta = 15;
    p->b_fixed_heat = 0;
    p->pos_rand_param = 0.1f; p->vel_rand_param = 0.0f;   // spray.cpp:55
    p->begin_frame = 0;                                   // spray.cpp:73
    p->b_run_mc_solid = 1;                                // spray.cpp:63
    return mp_params_derive(p);
}

