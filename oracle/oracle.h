/*
 * oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's multiphase FLIP step
 * (gaoyangVR/2017Multiphase, Multiphase/Multiphase/spray.cpp:979-1233 and
 * the kernels of spray_k.cu it launches). It is the checker for the CUDA
 * path: only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * may load it. Nothing in the product links or calls it.
 *
 * Parity status: pinned to the reference's own kernels.  The reference
 * does not build here as a program (Windows, GL, CUDA texture references
 * removed in CUDA 12, missing CUDA-samples headers) and ships no tests or
 * golden vectors, but its kernels compile for the host: oracle/
 * make_refhost.py takes their text from spray_k.cu unchanged, and
 * oracle/refhost/stages.inc launches them as spray.cu does.  The tests
 * tests/test_refhost_*.py run every stage of this file against them on the
 * same inputs and require bit-equal results.  Where the reference's
 * outcome depends on thread scheduling (in-place sweeps, float atomics,
 * atomic appends, float reductions) this file states the definition it
 * uses, and the kernel launches there follow the same definition.  The
 * marching-cubes triangle lists follow the generated case table
 * (csrc/mc_tables.cpp), which triangulates some cases differently from
 * tables.h.
 *
 * Build: g++ -O2 -fopenmp -ffp-contract=off (see oracle/Makefile).
 */
#ifndef MP_ORACLE_H
#define MP_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#include "../include/mp.h"

#ifdef __cplusplus
extern "C" {
#endif

int  or_create(const mp_params* p, void** out);
void or_destroy(void* o);
int  or_set_params(void* o, const mp_params* p);
int  or_get_state(void* o, mp_state* s);
int  or_set_state(void* o, const mp_state* s);
int  or_upload_particles(void* o, int n, const float* pos3, const float* vel3,
                         const int8_t* flag, const float* mass, const float* temp,
                         const float* lheat, const float* sol, const float* gas);
int  or_field_info(void* o, int field, size_t* count, size_t* elem_bytes);
int  or_get_field(void* o, int field, void* dst, size_t bytes);
int  or_set_field(void* o, int field, const void* src, size_t bytes);
int  or_set_tables(void* o, const float* randfloat, int nrand, const int32_t* seeds, int nseed);
int  or_set_mc_tables(void* o, const int32_t* num_verts, const int32_t* tri);
int  or_init_particle_heat(void* o);

int or_hash_sort(void* o);
int or_external_force(void* o);
int or_levelset(void* o, float offset);
int or_sweep_ls_mark(void* o);
int or_mark_solo_air(void* o);
int or_surface_tension(void* o);
int or_markgrid_bubble(void* o);
int or_p2g(void* o);
int or_drag(void* o);
int or_sweep_phi(void* o, int phase);
int or_sweep_u(void* o, int phase);
int or_set_boundary_u(void* o, int phase);
int or_project(void* o, int* iters, double* residual);
int or_g2p(void* o);
int or_solid_motion(void* o);
int or_solo_air_update(void* o);
int or_collide_advect(void* o);
int or_correct_pos(void* o);
int or_correct_pos_bubble(void* o);
int or_heat(void* o);
int or_heatsim(void* o);          /* heatsim (spray.cu:1959-1987)            */
int or_set_pour(void* o, const float* pos3, const float* vel3, int n);   /* dpourpos / dpourvel */
int or_get_params(void* o, mp_params* p);   /* the parameters as the scene switches left them */
int or_pour(void* o);             /* pouring / pouringgas (spray.cu:3012-3043) */
/* the extraction of `surface` from genSphereDensfield's sphere (spray_k.cu:1827) */
int or_mc_sphere(void* o, int surface, float cx, float cy, float cz, float radius);
/* the water mode (watersim, spray.cpp:741-797) and its stages */
int or_flip_mark(void* o);
int or_water_p2g(void* o);
int or_project_water(void* o, int* iters, double* res);
int or_water_g2p(void* o);
int or_water_advect(void* o);
int or_watersim(void* o);
int or_init_heat_grid(void* o);   /* initheat_grid (spray.cu:1949-1955)      */
int or_gen_gas(void* o);
int or_delete(void* o);
int or_melt(void* o);
int or_freeze(void* o);
int or_mc_presort(void* o);
int or_mc(void* o, int surface);
int or_mc_get(void* o, int surface, float* verts, float* normals, uint32_t* indices,
              int max_verts, int max_indices);
int or_mc_get_field(void* o, float* dens, uint8_t* cubeindex);
int or_step(void* o);
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
