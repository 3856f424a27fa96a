// oracle.cpp — TEST INFRASTRUCTURE ONLY (see oracle.h for scope and status).
//
// CPU restatement of the reference step. Every function cites the reference
// file:line it restates; paths are relative to Multiphase/Multiphase/.
// Semantics that differ from the reference's GPU code on purpose (all of
// them places where the reference races or is unordered):
//   * in-place sweeps (sweepphibytype, sweepphi, sweepVacuum, setBoundaryHeat)
//     are Jacobi: every cell reads the values from before the pass;
//   * particle kernels that read neighbours while writing themselves
//     (enforceForceSoloAirP, FreezingSolidByHeat) read a snapshot;
//   * float atomics (calDragForce, smooth_computedisplacement, calnormal_k)
//     are gathers that add contributions in ascending particle / triangle
//     order; the atomic append of GenerateGasParticle_k is ordered by cell;
//   * reductions (product(), accumulate_GPU_f3) are FP64 sums;
//   * normalize(v) is v * (1/sqrtf(dot(v,v))) (the reference used rsqrtf).
#include "oracle.h"
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include <numeric>
#include <string>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- float3 arithmetic of helper_math.h, restated ---------------------------
struct F3 { float x, y, z; };
static inline F3 mk(float x, float y, float z) { return F3{x, y, z}; }
static inline F3 mk(float s) { return F3{s, s, s}; }
static inline F3 operator+(F3 a, F3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline F3 operator-(F3 a, F3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline F3 operator-(F3 a) { return mk(-a.x, -a.y, -a.z); }
static inline F3 operator*(F3 a, F3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline F3 operator/(F3 a, F3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline F3 operator*(F3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline F3 operator*(float s, F3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline F3 operator/(F3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline void operator+=(F3& a, F3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
static inline void operator-=(F3& a, F3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
static inline void operator*=(F3& a, float s) { a.x *= s; a.y *= s; a.z *= s; }
static inline void operator/=(F3& a, float s) { a.x /= s; a.y /= s; a.z /= s; }
static inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(F3 v) { return sqrtf(dot(v, v)); }
static inline F3 normalize(F3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return v * inv; }
static inline F3 cross(F3 a, F3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

enum { TF = MP_TYPEFLUID, TA = MP_TYPEAIR, TB = MP_TYPEBOUNDARY, TV = MP_TYPEVACUUM,
       TS = MP_TYPEAIRSOLO, TSOL = MP_TYPESOLID };
static const uint32_t UNDEF = 0xffffffffu;

struct MCOut {
    std::vector<F3> verts, normals;
    std::vector<uint32_t> indices;
    int active = 0;
};

struct Oracle {
    mp_params P{};
    int NX = 0, NY = 0, NZ = 0, n = 0, nfx = 0, nfy = 0, nfz = 0;
    float h = 0;
    // grids
    std::vector<float> press, divg, lsfluid, lsair, lsmerge, phifluid, phiair, phisolid;
    std::vector<float> gx, gy, gz, gxa, gya, gza, sf, Tp, Tp_save, Tp_old, fixedheat;
    std::vector<int8_t> mark;
    std::vector<float> wu[3], wuo[3], au[3], auo[3], su[3];
    std::vector<uint32_t> cstart, cend;
    // particles (reference structure of arrays)
    int np = 0;
    std::vector<F3> pos, vel;
    std::vector<int8_t> flag;
    std::vector<float> mass, T, L, sol, gas, dens, prs;
    // scalars
    int frame = 0, nreal_solid = 0;
    int last_iters = 0, last_heat_iters = 0;
    double last_res = 0, last_heat_res = 0;
    std::vector<float> randf;
    std::vector<int32_t> seeds;
    // marching cubes
    std::vector<int32_t> mc_numverts, mc_tri;
    int NXMC = 0, NYMC = 0, NZMC = 0;
    std::vector<uint32_t> mc_cstart, mc_cend;
    std::vector<float> mc_dens;
    std::vector<uint8_t> mc_cube;
    MCOut mc_out[3];
    std::string err;

    // ---- index helpers (utility.h:55-95, spray_k.cu:44-74) -----------------
    inline int cid(int i, int j, int k) const { return i * NY * NZ + j * NZ + k; }
    inline bool vc(int i, int j, int k) const {
        return !(i < 0 || i > NX - 1 || j < 0 || j > NY - 1 || k < 0 || k > NZ - 1);
    }
    inline void getijk(int idx, int& i, int& j, int& k) const {
        i = idx / (NZ * NY); j = idx / NZ % NY; k = idx % NZ;
    }
    // getijk(i,j,k,idx,w,h,d) of utility.h:90-95
    static inline void getijk3(int idx, int w, int hh, int d, int& i, int& j, int& k) {
        (void)w; i = idx / d / hh; j = idx / d % hh; k = idx % d;
    }
    // getijkfrompos (spray_k.cu:51-57): an axis outside the grid maps to 0
    inline void ijkpos(F3 p, int& i, int& j, int& k) const {
        F3 g = mk(P.gmin_x, P.gmin_y, P.gmin_z);
        p = (p - g) / mk(h, h, h);
        i = (p.x >= 0 && p.x < NX) ? (int)p.x : 0;
        j = (p.y >= 0 && p.y < NY) ? (int)p.y : 0;
        k = (p.z >= 0 && p.z < NZ) ? (int)p.z : 0;
    }
    // face field accessors; dims (NX+1,NY,NZ), (NX,NY+1,NZ), (NX,NY,NZ+1)
    inline int fx(int i, int j, int k) const { return i * NY * NZ + j * NZ + k; }
    inline int fy(int i, int j, int k) const { return i * (NY + 1) * NZ + j * NZ + k; }
    inline int fz(int i, int j, int k) const { return i * NY * (NZ + 1) + j * (NZ + 1) + k; }

    // trilinear (spray_k.cu:111-122) on an array of dims (w,hh,d)
    static float trilinear(const float* u, float x, float y, float z, int w, int hh, int d) {
        x = fmaxf(0.0f, fminf(x, (float)w));
        y = fmaxf(0.0f, fminf(y, (float)hh));
        z = fmaxf(0.0f, fminf(z, (float)d));
        int i = (int)fminf(x, (float)(w - 2));
        int j = (int)fminf(y, (float)(hh - 2));
        int k = (int)fminf(z, (float)(d - 2));
        auto U = [&](int a, int b, int c) { return u[a * hh * d + b * d + c]; };
        return ((float)(k + 1) - z) * (((float)(j + 1) - y) * (((float)(i + 1) - x) * U(i, j, k) + (x - (float)i) * U(i + 1, j, k))
                                     + (y - (float)j) * (((float)(i + 1) - x) * U(i, j + 1, k) + (x - (float)i) * U(i + 1, j + 1, k)))
             + (z - (float)k) * (((float)(j + 1) - y) * (((float)(i + 1) - x) * U(i, j, k + 1) + (x - (float)i) * U(i + 1, j, k + 1))
                                 + (y - (float)j) * (((float)(i + 1) - x) * U(i, j + 1, k + 1) + (x - (float)i) * U(i + 1, j + 1, k + 1)));
    }
    // getParticleVelFromGrid (spray_k.cu:227-240)
    F3 velFromGrid(F3 p, const std::vector<float>* u) const {
        float x = p.x / h, y = p.y / h, z = p.z / h;
        return mk(trilinear(u[0].data(), x, y - 0.5f, z - 0.5f, NX + 1, NY, NZ),
                  trilinear(u[1].data(), x - 0.5f, y, z - 0.5f, NX, NY + 1, NZ),
                  trilinear(u[2].data(), x - 0.5f, y - 0.5f, z, NX, NY, NZ + 1));
    }
    // getScaleFromFrid (spray_k.cu:140-153)
    float scaleFromGrid(F3 p, const std::vector<float>& f) const {
        float x = p.x / h, y = p.y / h, z = p.z / h;
        return trilinear(f.data(), x - 0.5f, y - 0.5f, z - 0.5f, NX, NY, NZ);
    }
    // getVectorFromGrid (spray_k.cu:124-138)
    F3 vecFromGrid(F3 p, const std::vector<float>& a, const std::vector<float>& b,
                   const std::vector<float>& c) const {
        float x = p.x / h, y = p.y / h, z = p.z / h;
        return mk(trilinear(a.data(), x - 0.5f, y - 0.5f, z - 0.5f, NX, NY, NZ),
                  trilinear(b.data(), x - 0.5f, y - 0.5f, z - 0.5f, NX, NY, NZ),
                  trilinear(c.data(), x - 0.5f, y - 0.5f, z - 0.5f, NX, NY, NZ));
    }
    static inline float sharp_kernel(float r2, float hh) {   // spray_k.cu:255-258
        return fmaxf(hh * hh / fmaxf(r2, 0.0001f) - 1.0f, 0.0f);
    }
    static inline float smooth_kernel(float r2, float hh) {  // spray_k.cu:1330-1332
        return fmaxf(1.0f - r2 / (hh * hh), 0.0f);
    }
    inline bool cell_empty(int c) const { return cstart[c] == UNDEF; }

    void resize_grids() {
        NX = P.nx; NY = P.ny; NZ = P.nz; n = NX * NY * NZ; h = P.cellsize;
        nfx = (NX + 1) * NY * NZ; nfy = NX * (NY + 1) * NZ; nfz = NX * NY * (NZ + 1);
        for (auto* v : {&press, &divg, &lsfluid, &lsair, &lsmerge, &phifluid, &phiair, &phisolid,
                        &gx, &gy, &gz, &gxa, &gya, &gza, &sf, &Tp, &Tp_save, &Tp_old, &fixedheat})
            v->assign(n, 0.0f);
        mark.assign(n, 0);
        int nf[3] = {nfx, nfy, nfz};
        for (int a = 0; a < 3; a++) {
            wu[a].assign(nf[a], 0.f); wuo[a].assign(nf[a], 0.f); au[a].assign(nf[a], 0.f);
            auo[a].assign(nf[a], 0.f); su[a].assign(nf[a], 0.f);
        }
        cstart.assign(n, UNDEF); cend.assign(n, 0);
    }
    void resize_particles(int cap) {
        pos.resize(cap); vel.resize(cap); flag.resize(cap); mass.resize(cap); T.resize(cap);
        L.resize(cap); sol.resize(cap); gas.resize(cap); dens.resize(cap); prs.resize(cap);
    }

    // ======================================================================
    // hashAndSortParticles (spray.cu:614-637): calcHashD (spray_k.cu:1010),
    // thrust::sort_by_key (stable, spray_thrust.cu:12-17),
    // reorderDataAndFindCellStartD (spray_k.cu:1052-1129).
    // ======================================================================
    void sort_by_keys(const std::vector<uint32_t>& key, int ncells,
                      std::vector<uint32_t>& cs, std::vector<uint32_t>& ce) {
        std::vector<uint32_t> idx(np);
        std::iota(idx.begin(), idx.end(), 0u);
        std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
        auto perm = [&](auto& v) {
            auto old = v;
            for (int p = 0; p < np; p++) v[p] = old[idx[p]];
        };
        perm(pos); perm(vel); perm(flag); perm(mass); perm(T); perm(L); perm(sol); perm(gas);
        cs.assign(ncells, UNDEF); ce.assign(ncells, 0);
        for (int p = 0; p < np; p++) {
            uint32_t kk = key[idx[p]];
            if (p == 0 || kk != key[idx[p - 1]]) {
                cs[kk] = p;
                if (p > 0) ce[key[idx[p - 1]]] = p;
            }
            if (p == np - 1) ce[kk] = p + 1;
        }
    }
    void hash_sort() {
        std::vector<uint32_t> key(np);
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            int i, j, k; ijkpos(pos[p], i, j, k);
            key[p] = (uint32_t)cid(i, j, k);
        }
        sort_by_keys(key, n, cstart, cend);
    }

    // addexternalforce (spray.cu:376-393)
    void external_force() {
        float dt = P.dt;
        F3 g = mk(P.gravity_x, P.gravity_y, P.gravity_z);
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // addgravityforce_k (spray_k.cu:330-338)
            if (flag[p] == TF || flag[p] == TSOL) vel[p] += dt * g;
        }
        float velMax = P.bubble_max_vel;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // addbuoyancyforce_vel (spray_k.cu:356-371)
            float rate = fmaxf(velMax - vel[p].z, 0.0f) / velMax;
            if (flag[p] == TA) vel[p].z -= dt * g.z * rate * P.buoyance_rate_air;
            else if (flag[p] == TS) vel[p].z -= dt * g.z * rate * P.buoyance_rate_solo;
            else if (flag[p] == TSOL) vel[p].z += dt * g.z * 0.1f;
        }
    }

    // computeLevelset -> genlevelset (spray.cu:1465-1471, spray_k.cu:2753-2806)
    void levelset(float offset) {
        (void)offset;  // ignored by the reference (spray_k.cu:2803-2804)
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            mark[idx] = TV;
            float r = 0.5f * h;
            int i, j, k; getijk3(idx, NX, NY, NZ, i, j, k);
            F3 gp = (mk((float)i, (float)j, (float)k) + mk(0.5f, 0.5f, 0.5f)) * h;
            float mair = 2.5f * h, mfl = 2.5f * h;
            for (int di = -2; di <= 2; ++di) for (int dj = -2; dj <= 2; ++dj) for (int dk = -2; dk <= 2; ++dk) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                if (cell_empty(c)) continue;
                for (uint32_t p = cstart[c]; p < cend[c]; ++p) {
                    float d = length(pos[p] - gp);
                    if (flag[p] == TA || flag[p] == TS) mair = (d < mair) ? d : mair;
                    else if (flag[p] == TF || flag[p] == TSOL) mfl = (d < mfl) ? d : mfl;
                }
            }
            mair -= r; mfl -= r;
            lsfluid[idx] = mfl;
            lsair[idx] = mair;
        }
    }

    // solvedistance (spray_k.cu:746-754)
    static inline void solvedistance(float a, float b, float c, float& x) {
        float d = fminf(a, fminf(b, c)) + 1;
        if (d > fmaxf(a, fmaxf(b, c)))
            d = (a + b + c + sqrtf(3 - (a - b) * (a - b) - (a - c) * (a - c) - (b - c) * (b - c))) / 3;
        if (d < x) x = d;
    }
    // sweepphibytype (spray_k.cu:771-788), Jacobi. typeflag < 0: sweepphi (:755)
    void sweep_pass(std::vector<float>& phi, int typeflag) {
        std::vector<float> in = phi;
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            if (typeflag >= 0 && mark[idx] == typeflag) continue;
            int i, j, k; getijk(idx, i, j, k);
            float res = in[idx];
            for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2) {
                if (vc(i + di, j, k) && vc(i, j + dj, k) && vc(i, j, k + dk))
                    solvedistance(in[cid(i + di, j, k)], in[cid(i, j + dj, k)], in[cid(i, j, k + dk)], res);
            }
            phi[idx] = res;
        }
    }

    // sweepLSAndMardGrid (spray.cu:2011-2065)
    void sweep_ls_one(std::vector<float>& ls) {
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // markLS_bigpositive (spray_k.cu:3683-3697)
            ls[idx] = ls[idx] / h;
            if (ls[idx] > 1.99f) { ls[idx] = 5.0f; mark[idx] = TA; }
            else mark[idx] = TF;
        }
        for (int it = 0; it < 5; it++) sweep_pass(ls, TF);
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) ls[idx] = ls[idx] * h;            // setLSback_bigpositive (:3699)
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // preparels (:3708-3722)
            ls[idx] = -ls[idx] / h;
            if (ls[idx] > 0) { ls[idx] = 5.0f; mark[idx] = TA; }
            else mark[idx] = TF;
        }
        for (int it = 0; it < 5; it++) sweep_pass(ls, TF);
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) ls[idx] = -ls[idx] * h;           // setLSback (:3724)
    }
    void compute_phigra(std::vector<float>& ax, std::vector<float>& ay, std::vector<float>& az,
                        const std::vector<float>& ls) {   // computePhigra (spray_k.cu:3994-4019)
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            int i, j, k; getijk(idx, i, j, k);
            float c = ls[idx];
            float x1 = vc(i + 1, j, k) ? ls[cid(i + 1, j, k)] : c;
            float x0 = vc(i - 1, j, k) ? ls[cid(i - 1, j, k)] : c;
            float y1 = vc(i, j + 1, k) ? ls[cid(i, j + 1, k)] : c;
            float y0 = vc(i, j - 1, k) ? ls[cid(i, j - 1, k)] : c;
            float z1 = vc(i, j, k + 1) ? ls[cid(i, j, k + 1)] : c;
            float z0 = vc(i, j, k - 1) ? ls[cid(i, j, k - 1)] : c;
            ax[idx] = ((x1 - x0) * 0.5f) / h;
            ay[idx] = ((y1 - y0) * 0.5f) / h;
            az[idx] = ((z1 - z0) * 0.5f) / h;
        }
    }
    void sweep_ls_mark() {
        sweep_ls_one(lsfluid);
        sweep_ls_one(lsair);
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // mergeLSAndMarkGrid (spray_k.cu:3733-3777)
            float lf = lsfluid[idx], la = lsair[idx];
            if (la > 4.99f * h) { lsmerge[idx] = lf; mark[idx] = (lf > 0) ? TV : TF; }
            else if (lf > 4.99f * h) { lsmerge[idx] = la; mark[idx] = (la > 0) ? TV : TA; }
            else if (la > 0.8f * h && lf > 0.8f * h) { mark[idx] = TV; lsmerge[idx] = std::min(lf, la); }
            else {
                lsmerge[idx] = (lf - la) * 0.5f;
                mark[idx] = (lsmerge[idx] > 0) ? TA : TF;
            }
            int i, j, k; getijk(idx, i, j, k);
            if (i == 0 || i == NX - 1 || j == 0 || j == NY - 1 || k == 0 || k == NZ - 1) {
                mark[idx] = TB; lsmerge[idx] = -0.5f * h;
            }
        }
        compute_phigra(gx, gy, gz, lsmerge);
    }

    // isInBoundaryCell (spray_k.cu:4214-4221)
    bool inBoundaryCell(int x, int y, int z) const {
        (void)z; int lv = 2;
        return x <= lv || x >= NX - 1 - lv || y <= lv || y >= NY - 1 - lv;
    }

    // markSoloAirParticle -> verifySoloAirParticle (spray.cu:2614-2618, spray_k.cu:4196-4262)
    void mark_solo_air() {
        std::vector<int8_t> oflag(flag.begin(), flag.begin() + np);
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            int8_t f = oflag[p];
            if (f == TF || f == TSOL) continue;
            F3 ip = pos[p];
            float ls = scaleFromGrid(ip, lsmerge);
            int i, j, k; ijkpos(ip, i, j, k);
            int cnt = 0;
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                if (cell_empty(c)) continue;
                for (uint32_t q = cstart[c]; q < cend[c]; q++) {
                    float d = length(pos[q] - ip);
                    if (d < h && (oflag[q] == TA || oflag[q] == TS)) ++cnt;
                }
            }
            float tol1 = -1.45f, tol2 = -0.5f;
            int sc = P.scene;
            if (sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL) { tol1 = 0.05f; tol2 = -0.8f; }
            else if (sc == MP_SCENE_INTERACTION) { tol1 = 0.2f; tol2 = -0.5f; }
            if ((cnt >= 10 || ls > tol1 * h) && f == TS && !inBoundaryCell(i, j, k)) {
                if (cnt >= 3) flag[p] = TA;
            } else if (f == TA && (inBoundaryCell(i, j, k) || ls < tol2 * h || cnt <= 1)) {
                vel[p] = velFromGrid(ip, au);
                flag[p] = TS;
            }
        }
    }

    // computesurfacetension (spray.cu:2001-2009)
    void surface_tension() {
        float sigma = P.surfacetension_sigma;
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // compsurfacetension_k (spray_k.cu:3543-3637)
            if (mark[idx] == TB) { sf[idx] = 0; continue; }
            int i, j, k; getijk(idx, i, j, k);
            float res;
            F3 c = mk(gx[idx], gy[idx], gz[idx]);
            float len = length(c);
            if (len == 0) res = 0;
            else {
                c /= len;
                auto comp = [&](int ii, int jj, int kk, int axis, float dflt) {
                    if (!vc(ii, jj, kk)) return dflt;
                    int q = cid(ii, jj, kk);
                    float l = length(mk(gx[q], gy[q], gz[q]));
                    if (l == 0) return dflt;
                    float v = axis == 0 ? gx[q] : (axis == 1 ? gy[q] : gz[q]);
                    return v / l;
                };
                float x1 = comp(i + 1, j, k, 0, c.x), x0 = comp(i - 1, j, k, 0, c.x);
                float y1 = comp(i, j + 1, k, 1, c.y), y0 = comp(i, j - 1, k, 1, c.y);
                float z1 = comp(i, j, k + 1, 2, c.z), z0 = comp(i, j, k - 1, 2, c.z);
                res = (x1 - x0 + y1 - y0 + z1 - z0) / h * 0.5f;
            }
            sf[idx] = res * sigma;
        }
        int sc = P.scene;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {        // enforcesurfacetension_p (spray_k.cu:3639-3680)
            int8_t f = flag[p];
            if (f == TSOL || f == TF) continue;
            if ((sc != MP_SCENE_MELTANDBOIL && sc != MP_SCENE_MELTANDBOIL_HIGHRES && f == TS) ||
                (sc != MP_SCENE_ALL && f == TS)) continue;
            F3 ip = pos[p];
            float ilsm = scaleFromGrid(ip, lsmerge);
            float isf = scaleFromGrid(ip, sf);
            F3 dir = vecFromGrid(ip, gx, gy, gz);
            float ld = length(dir);
            if (ld == 0) continue;
            dir /= ld; ilsm /= ld;
            int i, j, k; ijkpos(ip, i, j, k);
            int cnt = (mark[cid(i, j, k)] == TA) ? 1 : 0;
            for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2)
                if (vc(i + di, j + dj, k + dk) && mark[cid(i + di, j + dj, k + dk)] == TA) cnt++;
            if (cnt == 0) continue;
            if (fabsf(ilsm) < h) {
                F3 fo = (-isf) * dir;
                vel[p] += fo * P.dt;
            }
        }
    }

    // markgrid_bubble (spray.cu:511-518): markfluid_dense launched with the
    // particle grid (pblocknum x 512 threads) but indexing cells, so only
    // cells below that thread count are marked (spray_k.cu:506-533).
    void markgrid_bubble() {
        int pblocks = std::max(1, (np + 511) / 512);
        int lim = std::min(n, pblocks * 512);
        #pragma omp parallel for
        for (int idx = 0; idx < lim; idx++) {
            int cfs = 0, ca = 0;
            if (!cell_empty(idx))
                for (uint32_t p = cstart[idx]; p < cend[idx]; ++p) {
                    if (flag[p] == TF || flag[p] == TSOL) cfs++;
                    else if (flag[p] == TA) ca++;
                }
            if (cfs == 0 && ca == 0) mark[idx] = TV;
            else if (cfs > ca) mark[idx] = TF;
            else mark[idx] = TA;
        }
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // markBoundaryCell (spray_k.cu:535-545)
            int i, j, k; getijk(idx, i, j, k);
            if (i == 0 || i == NX - 1 || j == 0 || j == NY - 1 || k == 0 || k == NZ - 1) mark[idx] = TB;
        }
    }

    // face gather of mapvelp2g_k_fluidSolid / _air (spray_k.cu:2809-2937)
    // axis 0/1/2; lo/hi: window along the face normal, lo2/hi2: the other two axes
    float face_gather(int axis, int i, int j, int k, int lo, int hi, int lo2, int hi2, int which) const {
        float scale = 1.0f / h;   // `1 / dparam.cellsize.x`
        F3 gp;
        if (axis == 0) gp = mk((float)i, (float)j + 0.5f, (float)k + 0.5f);
        else if (axis == 1) gp = mk((float)i + 0.5f, (float)j, (float)k + 0.5f);
        else gp = mk((float)i + 0.5f, (float)j + 0.5f, (float)k);
        int r0[3], r1[3];
        for (int a = 0; a < 3; a++) { r0[a] = lo2; r1[a] = hi2; }
        r0[axis] = lo; r1[axis] = hi;
        float weight = 0, us = 0;
        for (int di = r0[0]; di <= r1[0]; di++) for (int dj = r0[1]; dj <= r1[1]; dj++) for (int dk = r0[2]; dk <= r1[2]; dk++) {
            if (!vc(i + di, j + dj, k + dk)) continue;
            int c = cid(i + di, j + dj, k + dk);
            if (cell_empty(c)) continue;
            for (uint32_t p = cstart[c]; p < cend[c]; ++p) {
                int8_t f = flag[p];
                bool ok = which == 0 ? (f == TF || f == TSOL) : (f == TA);
                if (!ok) continue;
                F3 d = pos[p] * scale - gp;
                float dis2 = dot(d, d);
                float w = mass[p] * sharp_kernel(dis2, 1.4f);
                weight += w;
                float v = axis == 0 ? vel[p].x : (axis == 1 ? vel[p].y : vel[p].z);
                us += w * v;
            }
        }
        return (weight > 0) ? (us / weight) : 0.0f;
    }
    void p2g_into(std::vector<float>* u, int which) {
        int lo = which == 0 ? -1 : -2, hi = which == 0 ? 0 : 1, lo2 = which == 0 ? -1 : -2, hi2 = which == 0 ? 1 : 2;
        #pragma omp parallel for
        for (int idx = 0; idx < nfx; idx++) { int i, j, k; getijk3(idx, NX + 1, NY, NZ, i, j, k); u[0][idx] = face_gather(0, i, j, k, lo, hi, lo2, hi2, which); }
        #pragma omp parallel for
        for (int idx = 0; idx < nfy; idx++) { int i, j, k; getijk3(idx, NX, NY + 1, NZ, i, j, k); u[1][idx] = face_gather(1, i, j, k, lo, hi, lo2, hi2, which); }
        #pragma omp parallel for
        for (int idx = 0; idx < nfz; idx++) { int i, j, k; getijk3(idx, NX, NY, NZ + 1, i, j, k); u[2][idx] = face_gather(2, i, j, k, lo, hi, lo2, hi2, which); }
    }
    // mapvelp2g_bubble (spray.cu:1562-1588)
    void p2g() {
        p2g_into(wu, 0);
        p2g_into(au, 1);
        for (int a = 0; a < 3; a++) { wuo[a] = wu[a]; auo[a] = au[a]; }
    }

    // enforceDragForce -> calDragForce (spray.cu:2953-2957, spray_k.cu:5127-5165).
    // The per-particle velocity change is computed from the water field as it
    // was before the stage; the six face contributions are added to each face
    // in ascending particle order.
    void drag() {
        std::vector<F3> vcg(np);
        std::vector<char> is_solo(np, 0);
        bool any = false;
        for (int p = 0; p < np; p++) if (flag[p] == TS) { is_solo[p] = 1; any = true; }
        if (!any) return;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            if (!is_solo[p]) continue;
            F3 ip = pos[p], iv = vel[p];
            F3 gv = velFromGrid(ip, wu);
            F3 diff = gv - iv;
            F3 dfb = (P.drag_param_solo * length(diff)) * diff;
            vcg[p] = (-dfb) * P.drag_param_grid * P.dt;
            if (P.scene == MP_SCENE_INTERACTION || P.scene == MP_SCENE_INTERACTION_HIGHRES)
                vel[p] += dfb * P.dt;
        }
        for (int p = 0; p < np; p++) {
            if (!is_solo[p]) continue;
            F3 ip = pos[p];
            int i, j, k; ijkpos(ip, i, j, k);
            F3 w = ip / h - mk((float)i, (float)j, (float)k);
            F3 g = vcg[p];
            wu[0][fx(i, j, k)] += g.x * (1 - w.x);
            wu[0][fx(i + 1, j, k)] += g.x * w.x;
            wu[1][fy(i, j, k)] += g.y * (1 - w.y);
            wu[1][fy(i, j + 1, k)] += g.y * w.y;
            wu[2][fz(i, j, k)] += g.z * (1 - w.z);
            wu[2][fz(i, j, k + 1)] += g.z * w.z;
        }
    }

    // sweepPhi (spray.cu:570-583): initphi (spray_k.cu:712-722) + 3 sweeps
    void sweep_phi(int phase) {
        std::vector<float>& phi = phase == TA ? phiair : phifluid;
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) phi[idx] = (mark[idx] == phase) ? -0.5f : (float)(NX * 3);
        for (int it = 0; it < 3; it++) sweep_pass(phi, phase);
    }

    // sweepu_k_bubble (spray_k.cu:3779-3880), one pass in -> out
    void sweepu_pass(std::vector<float>* out, const std::vector<float>* in, const std::vector<float>& ls, int fl) {
        auto LS = [&](int i, int j, int k) { return ls[cid(i, j, k)]; };
        auto M = [&](int i, int j, int k) { return mark[cid(i, j, k)]; };
        #pragma omp parallel for
        for (int idx = 0; idx < nfx; idx++) {
            out[0][idx] = in[0][idx];
            int i, j, k; getijk3(idx, NX + 1, NY, NZ, i, j, k);
            if (!(i > 1 && i < NX - 1)) continue;
            if (!(M(i, j, k) != fl && M(i - 1, j, k) != fl)) continue;
            for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2) {
                if (j + dj < 0 || j + dj > NY - 1 || k + dk < 0 || k + dk > NZ - 1) continue;
                float wx = (float)(-di) * (LS(i, j, k) - LS(i - 1, j, k));
                if (wx < 0) continue;
                float wy = (LS(i, j, k) + LS(i - 1, j, k) - LS(i, j + dj, k) - LS(i - 1, j + dj, k)) * 0.5f;
                if (wy < 0) continue;
                float wz = (LS(i, j, k) + LS(i - 1, j, k) - LS(i, j, k + dk) - LS(i - 1, j, k + dk)) * 0.5f;
                if (wz < 0) continue;
                float ws = wx + wy + wz;
                if (ws == 0) wx = wy = wz = 1.0f / 3;
                else { wx /= ws; wy /= ws; wz /= ws; }
                out[0][idx] = wx * in[0][fx(i + di, j, k)] + wy * in[0][fx(i, j + dj, k)] + wz * in[0][fx(i, j, k + dk)];
            }
        }
        #pragma omp parallel for
        for (int idx = 0; idx < nfy; idx++) {
            out[1][idx] = in[1][idx];
            int i, j, k; getijk3(idx, NX, NY + 1, NZ, i, j, k);
            if (!(j > 1 && j < NY - 1)) continue;
            if (!(M(i, j, k) != fl && M(i, j - 1, k) != fl)) continue;
            for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2) {
                if (i + di < 0 || i + di > NX - 1 || k + dk < 0 || k + dk > NZ - 1) continue;
                float wy = (float)(-dj) * (LS(i, j, k) - LS(i, j - 1, k));
                if (wy < 0) continue;
                float wx = (LS(i, j, k) + LS(i, j - 1, k) - LS(i + di, j, k) - LS(i + di, j - 1, k)) * 0.5f;
                if (wx < 0) continue;
                float wz = (LS(i, j, k) + LS(i, j - 1, k) - LS(i, j, k + dk) - LS(i, j - 1, k + dk)) * 0.5f;
                if (wz < 0) continue;
                float ws = wx + wy + wz;
                if (ws == 0) wx = wy = wz = 1.0f / 3;
                else { wx /= ws; wy /= ws; wz /= ws; }
                out[1][idx] = wx * in[1][fy(i + di, j, k)] + wy * in[1][fy(i, j + dj, k)] + wz * in[1][fy(i, j, k + dk)];
            }
        }
        #pragma omp parallel for
        for (int idx = 0; idx < nfz; idx++) {
            out[2][idx] = in[2][idx];
            int i, j, k; getijk3(idx, NX, NY, NZ + 1, i, j, k);
            if (!(k > 1 && k < NZ - 1)) continue;
            if (!(M(i, j, k) != fl && M(i, j, k - 1) != fl)) continue;
            for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2) {
                if (i + di < 0 || i + di > NX - 1 || j + dj < 0 || j + dj > NY - 1) continue;
                float wz = (float)(-dk) * (LS(i, j, k) - LS(i, j, k - 1));
                if (wz < 0) continue;
                float wy = (LS(i, j, k) + LS(i, j, k - 1) - LS(i, j + dj, k) - LS(i, j + dj, k - 1)) * 0.5f;
                if (wy < 0) continue;
                float wx = (LS(i, j, k) + LS(i, j, k - 1) - LS(i + di, j, k) - LS(i + di, j, k - 1)) * 0.5f;
                if (wx < 0) continue;
                float ws = wx + wy + wz;
                if (ws == 0) wx = wy = wz = 1.0f / 3;
                else { wx /= ws; wy /= ws; wz /= ws; }
                out[2][idx] = wx * in[2][fz(i + di, j, k)] + wy * in[2][fz(i, j + dj, k)] + wz * in[2][fz(i, j, k + dk)];
            }
        }
    }
    // sweepU (spray.cu:585-598): two double-buffered passes
    void sweep_u(int phase) {
        std::vector<float>* u = phase == TA ? au : wu;
        const std::vector<float>& phi = phase == TA ? phiair : phifluid;
        std::vector<float> tmp[3];
        for (int a = 0; a < 3; a++) tmp[a].resize(u[a].size());
        for (int it = 0; it < 2; it++) {
            sweepu_pass(tmp, u, phi, phase);
            for (int a = 0; a < 3; a++) u[a].swap(tmp[a]);
        }
    }

    // setWaterBoundaryU_k (spray_k.cu:956-995). The ceiling rule reads the
    // face below after that face's own rule has been applied.
    void set_boundary_u(int phase) {
        std::vector<float>* u = phase == TA ? au : wu;
        auto M = [&](int i, int j, int k) { return mark[cid(i, j, k)]; };
        #pragma omp parallel for
        for (int idx = 0; idx < nfx; idx++) {
            int i, j, k; getijk3(idx, NX + 1, NY, NZ, i, j, k);
            if (i <= 1 || i >= NX + 1 - 2) u[0][idx] = 0.0f;
            else if (i > 1 && i < NX - 1 && ((M(i, j, k) == TB) != (M(i - 1, j, k) == TB))) u[0][idx] = 0.0f;
        }
        #pragma omp parallel for
        for (int idx = 0; idx < nfy; idx++) {
            int i, j, k; getijk3(idx, NX, NY + 1, NZ, i, j, k);
            if (j <= 1 || j >= NY + 1 - 2) u[1][idx] = 0.0f;
            else if (j > 0 && j < NY && ((M(i, j, k) == TB) != (M(i, j - 1, k) == TB))) u[1][idx] = 0.0f;
        }
        std::vector<float> in = u[2];
        auto zrule = [&](int i, int j, int k, float v) -> float {   // rule for faces k <= NZ-2
            if (k <= 1) return 0.0f;
            if (k > 0 && k < NZ && ((M(i, j, k) == TB) != (M(i, j, k - 1) == TB))) return 0.0f;
            return v;
        };
        #pragma omp parallel for
        for (int idx = 0; idx < nfz; idx++) {
            int i, j, k; getijk3(idx, NX, NY, NZ + 1, i, j, k);
            if (k <= 1 || k >= NZ + 1 - 1) u[2][idx] = 0.0f;
            else if (k == NZ + 1 - 2) {
                float below = zrule(i, j, k - 1, in[fz(i, j, k - 1)]);
                u[2][idx] = (below < 0) ? below : 0;
            } else u[2][idx] = zrule(i, j, k, in[idx]);
        }
    }

    // ---- projection ------------------------------------------------------
    // cptdivergence_bubble2 (spray_k.cu:3138-3263)
    template <class R>
    void divergence(std::vector<R>& out) {
        out.assign(n, (R)0);
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            int m = mark[idx];
            if (!(m == TF || m == TA)) { out[idx] = 0; continue; }
            int i, j, k; getijk(idx, i, j, k);
            auto LS = [&](int a, int b, int c) { return (R)lsmerge[cid(a, b, c)]; };
            // one face value: cell (i,j,k), neighbour (a,b,c), face index f on axis
            auto face = [&](int a, int b, int c, int axis, int f) -> R {
                int mn = mark[cid(a, b, c)];
                R wv = (R)wu[axis][f], av = (R)au[axis][f];
                if (m == TF && mn != TA) return wv;
                if (m == TA && mn != TF) return av;
                R th = ((R)0 - LS(i, j, k)) / (LS(a, b, c) - LS(i, j, k));
                if (m == TF) return th * wv + (1 - th) * av;
                return th * av + (1 - th) * wv;
            };
            R ux1 = face(i + 1, j, k, 0, fx(i + 1, j, k));
            R ux0 = face(i - 1, j, k, 0, fx(i, j, k));
            R uy1 = face(i, j + 1, k, 1, fy(i, j + 1, k));
            R uy0 = face(i, j - 1, k, 1, fy(i, j, k));
            R uz1 = face(i, j, k + 1, 2, fz(i, j, k + 1));
            R uz0 = face(i, j, k - 1, 2, fz(i, j, k));
            out[idx] = (ux1 - ux0 + uy1 - uy0 + uz1 - uz0) / (R)h;
        }
    }

    // FP64 dot product with a fixed summation tree (blocks of 4096, then serial)
    template <class A, class B>
    static double ddot(const std::vector<A>& a, const std::vector<B>& b, int nn) {
        const int BS = 4096;
        int nb = (nn + BS - 1) / BS;
        std::vector<double> part(nb, 0.0);
        #pragma omp parallel for
        for (int q = 0; q < nb; q++) {
            double s = 0;
            int e = std::min(nn, (q + 1) * BS);
            for (int i = q * BS; i < e; i++) s += (double)a[i] * (double)b[i];
            part[q] = s;
        }
        double s = 0;
        for (int q = 0; q < nb; q++) s += part[q];
        return s;
    }

    // computeAx_bubble (spray_k.cu:3423-3447)
    template <class R>
    void ax_bubble(std::vector<R>& out, const std::vector<R>& x) {
        R h2 = (R)h * (R)h;
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            int m = mark[idx];
            if (!(m == TF || m == TA)) { out[idx] = 0; continue; }
            int i, j, k; getijk(idx, i, j, k);
            R c = x[idx];
            R s = (R)(-6.0f) * c;
            auto nb = [&](int a, int b, int cc) { int q = cid(a, b, cc); return (mark[q] == TB) ? c : x[q]; };
            s += nb(i + 1, j, k); s += nb(i, j + 1, k); s += nb(i, j, k + 1);
            s += nb(i - 1, j, k); s += nb(i, j - 1, k); s += nb(i, j, k - 1);
            out[idx] = s / h2;
        }
    }
    // computeAx_heat (spray_k.cu:4526-4568); BOUNDARY rows are written 0
    void ax_heat(std::vector<float>& out, const std::vector<float>& x, const float* alpha_of_type) {
        bool boil = P.scene == MP_SCENE_BOILING || P.scene == MP_SCENE_BOILING_HIGHRES ||
                    P.scene == MP_SCENE_MELTANDBOIL || P.scene == MP_SCENE_MELTANDBOIL_HIGHRES || P.scene == MP_SCENE_ALL;
        float dt = P.dt;
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            int m = mark[idx];
            if (m == TB) { out[idx] = 0; continue; }
            float alpha = alpha_of_type[m];
            int i, j, k; getijk(idx, i, j, k);
            float c = x[idx];
            float s = (h * h / alpha / dt + 6.0f) * c;
            auto nb = [&](int a, int b, int cc) {
                int q = cid(a, b, cc);
                bool fixedc = boil ? (mark[q] == TB || mark[q] == TV) : (mark[q] == TB);
                return fixedc ? c : x[q];
            };
            s -= nb(i + 1, j, k); s -= nb(i, j + 1, k); s -= nb(i, j, k + 1);
            s -= nb(i - 1, j, k); s -= nb(i, j - 1, k); s -= nb(i, j, k - 1);
            out[idx] = s;
        }
    }

    // solver_cg_bubble / solver_cg_heat (spray.cu:1613-1687, 1780-1852) with
    // FP64 scalars. mask(idx) selects the unknowns; A(out, x) applies the matrix.
    template <class R, class Mask, class Apply>
    int cg(std::vector<R>& x, const std::vector<R>& b, Mask mask, Apply A, int maxiter,
           int tolmode, float tol, int true_every, double& res_out, bool& capped) {
        std::vector<R> z(n), r(n), p(n);
        capped = false;
        A(z, x);
        #pragma omp parallel for
        for (int i = 0; i < n; i++) r[i] = mask(i) ? (R)(b[i] + (R)(-1.0f) * z[i]) : (R)0;
        double rr = ddot(r, r, n);
        double eps;
        if (tolmode == MP_TOL_REF_ABS) eps = (double)((float)tol * (float)n);
        else { double bb = ddot(b, b, n); eps = (double)tol * (double)tol * bb; }
        res_out = rr;
        if (rr < eps || (tolmode == MP_TOL_REL && eps == 0.0)) return 0;
        z = r; p = z;
        double a = rr;
        int k = 0;
        for (;; k++) {
            if (k >= maxiter) { capped = true; break; }
            A(z, p);
            double zp = ddot(z, p, n);
            if (zp == 0) { res_out = rr; return k; }
            double alpha = a / zp;
            R af = (R)alpha;
            #pragma omp parallel for
            for (int i = 0; i < n; i++) {
                if (mask(i)) { x[i] = x[i] + af * p[i]; r[i] = r[i] + (-af) * z[i]; }
                else { x[i] = 0; r[i] = 0; }
            }
            if (true_every > 0 && (k + 1) % true_every == 0) {
                A(z, x);
                #pragma omp parallel for
                for (int i = 0; i < n; i++) r[i] = mask(i) ? (R)(b[i] + (R)(-1.0f) * z[i]) : (R)0;
            }
            rr = ddot(r, r, n);
            res_out = rr;
            if (rr < eps) { k++; break; }
            double beta = rr / a;
            R bf = (R)beta;
            #pragma omp parallel for
            for (int i = 0; i < n; i++) p[i] = mask(i) ? (R)(r[i] + bf * p[i]) : (R)0;
            a = rr;
        }
        return k;
    }

    // subGradPress (spray_k.cu:198-224) on one face field set
    template <class R>
    void subgrad(std::vector<float>* u, const std::vector<R>& p) {
        R hh = (R)h;
        #pragma omp parallel for
        for (int idx = 0; idx < nfx; idx++) {
            int i, j, k; getijk3(idx, NX + 1, NY, NZ, i, j, k);
            if (i > 0 && i < NX) u[0][idx] = (float)((R)u[0][idx] - (p[cid(i, j, k)] - p[cid(i - 1, j, k)]) / hh);
        }
        #pragma omp parallel for
        for (int idx = 0; idx < nfy; idx++) {
            int i, j, k; getijk3(idx, NX, NY + 1, NZ, i, j, k);
            if (j > 0 && j < NY) u[1][idx] = (float)((R)u[1][idx] - (p[cid(i, j, k)] - p[cid(i, j - 1, k)]) / hh);
        }
        #pragma omp parallel for
        for (int idx = 0; idx < nfz; idx++) {
            int i, j, k; getijk3(idx, NX, NY, NZ + 1, i, j, k);
            if (k > 0 && k < NZ) u[2][idx] = (float)((R)u[2][idx] - (p[cid(i, j, k)] - p[cid(i, j, k - 1)]) / hh);
        }
    }

    // project_CG_bubble (spray.cu:1590-1611)
    template <class R>
    int project_t(int* iters, double* residual) {
        std::vector<R> b, x(n, (R)0);
        divergence<R>(b);
        for (int i = 0; i < n; i++) divg[i] = (float)b[i];
        auto mask = [&](int i) { return mark[i] == TF || mark[i] == TA; };
        auto A = [&](std::vector<R>& o, const std::vector<R>& v) { ax_bubble<R>(o, v); };
        bool capped = false;
        double res = 0;
        int it = cg<R>(x, b, mask, A, P.cg_max_iter, P.cg_tol_mode, P.cg_tol, P.cg_true_residual_every, res, capped);
        for (int i = 0; i < n; i++) press[i] = (float)x[i];
        subgrad<R>(wu, x);
        subgrad<R>(au, x);
        last_iters = it; last_res = res;
        if (iters) *iters = it;
        if (residual) *residual = res;
        return capped ? MP_ERR_NOCONVERGE : MP_OK;
    }
    // Ghost-fluid variable density (MP_COEF_GFM, an extension; the reference's
    // projection is constant-coefficient): face weights beta = 1/rho_face with
    // rho_liquid = 1, rho_air = 1/ratio, theta-blended across liquid-air faces
    // (theta = -ls_L / (ls_G - ls_L), clamped to [0, 1]); the system
    //   sum over non-wall neighbours of beta_f (p_nb - p_c) / h^2 = div
    // solved in FP64 to a 1e-12 relative residual (Jacobi-scaled CG), then
    // u -= beta grad p on both velocity fields. The reference solution the GPU
    // form is checked against.
    int project_gfm(int* iters, double* residual) {
        std::vector<double> b;
        divergence<double>(b);
        for (int i = 0; i < n; i++) divg[i] = (float)b[i];
        const float rho_air = 1.0f / P.density_ratio;
        std::vector<float> beta[3] = {std::vector<float>(nfx, 0.f), std::vector<float>(nfy, 0.f),
                                      std::vector<float>(nfz, 0.f)};
        auto unknown = [&](int m) { return m == TF || m == TA; };
        auto rho = [&](int m) { return m == TA ? rho_air : 1.0f; };
        for (int ax = 0; ax < 3; ax++) {
            int nf = ax == 0 ? nfx : (ax == 1 ? nfy : nfz);
            #pragma omp parallel for
            for (int idx = 0; idx < nf; idx++) {
                int i, j, k;
                if (ax == 0) getijk3(idx, NX + 1, NY, NZ, i, j, k);
                else if (ax == 1) getijk3(idx, NX, NY + 1, NZ, i, j, k);
                else getijk3(idx, NX, NY, NZ + 1, i, j, k);
                int e = ax == 0 ? i : (ax == 1 ? j : k), nn = ax == 0 ? NX : (ax == 1 ? NY : NZ);
                float bt = 0.f;
                if (e > 0 && e < nn) {
                    int cb = cid(i, j, k), ca = cid(i - (ax == 0), j - (ax == 1), k - (ax == 2));
                    int ma = mark[ca], mb = mark[cb];
                    if (unknown(ma) && unknown(mb)) {
                        if (ma == mb) bt = 1.0f / rho(ma);
                        else {
                            int cl = ma == TF ? ca : cb, cg = ma == TF ? cb : ca;
                            float ll = lsmerge[cl], lg = lsmerge[cg];
                            float th = (lg == ll) ? 0.5f : (0.0f - ll) / (lg - ll);
                            th = std::min(1.0f, std::max(0.0f, th));
                            bt = 1.0f / (th * 1.0f + (1.0f - th) * rho_air);
                        }
                    } else if (unknown(ma)) bt = 1.0f / rho(ma);
                    else if (unknown(mb)) bt = 1.0f / rho(mb);
                }
                beta[ax][idx] = bt;
            }
        }
        auto inner = [&](int i, int j, int k) { return i > 0 && i < NX - 1 && j > 0 && j < NY - 1 && k > 0 && k < NZ - 1; };
        auto mask = [&](int c) { int i, j, k; getijk(c, i, j, k); return unknown(mark[c]) && inner(i, j, k); };
        // the six (neighbour, face weight) pairs of a cell
        auto nbrs = [&](int c, int* q, double* w) {
            int i, j, k; getijk(c, i, j, k);
            q[0] = cid(i + 1, j, k); w[0] = beta[0][fx(i + 1, j, k)];
            q[1] = cid(i, j + 1, k); w[1] = beta[1][fy(i, j + 1, k)];
            q[2] = cid(i, j, k + 1); w[2] = beta[2][fz(i, j, k + 1)];
            q[3] = cid(i - 1, j, k); w[3] = beta[0][fx(i, j, k)];
            q[4] = cid(i, j - 1, k); w[4] = beta[1][fy(i, j, k)];
            q[5] = cid(i, j, k - 1); w[5] = beta[2][fz(i, j, k)];
        };
        const double h2 = (double)h * (double)h;
        std::vector<double> S(n, 0.0), bs(n, 0.0), y(n, 0.0);
        #pragma omp parallel for
        for (int c = 0; c < n; c++) {
            if (!mask(c)) continue;
            int q[6]; double w[6]; nbrs(c, q, w);
            double d = 0;
            for (int t = 0; t < 6; t++) if (mark[q[t]] != TB) d += w[t];
            d /= h2;
            S[c] = d > 0 ? 1.0 / std::sqrt(d) : 0.0;
            bs[c] = S[c] * b[c];
        }
        auto A = [&](std::vector<double>& o, const std::vector<double>& v) {
            #pragma omp parallel for
            for (int c = 0; c < n; c++) {
                if (!mask(c)) { o[c] = 0; continue; }
                int q[6]; double w[6]; nbrs(c, q, w);
                double s = 0;
                for (int t = 0; t < 6; t++)
                    if (mark[q[t]] != TB) s += w[t] * (S[q[t]] * v[q[t]] - S[c] * v[c]);
                o[c] = S[c] * s / h2;
            }
        };
        bool capped = false;
        double res = 0;
        int it = cg<double>(y, bs, mask, A, std::max(P.cg_max_iter, 20000), MP_TOL_REL, 1e-12f, 0, res, capped);
        std::vector<double> p(n);
        for (int c = 0; c < n; c++) { p[c] = S[c] * y[c]; press[c] = (float)p[c]; }
        for (int ax = 0; ax < 3; ax++) {
            int nf = ax == 0 ? nfx : (ax == 1 ? nfy : nfz);
            #pragma omp parallel for
            for (int idx = 0; idx < nf; idx++) {
                int i, j, k;
                if (ax == 0) getijk3(idx, NX + 1, NY, NZ, i, j, k);
                else if (ax == 1) getijk3(idx, NX, NY + 1, NZ, i, j, k);
                else getijk3(idx, NX, NY, NZ + 1, i, j, k);
                int e = ax == 0 ? i : (ax == 1 ? j : k), nn = ax == 0 ? NX : (ax == 1 ? NY : NZ);
                if (!(e > 0 && e < nn)) continue;
                double d = (double)beta[ax][idx] *
                           (p[cid(i, j, k)] - p[cid(i - (ax == 0), j - (ax == 1), k - (ax == 2))]) / (double)h;
                wu[ax][idx] = (float)((double)wu[ax][idx] - d);
                au[ax][idx] = (float)((double)au[ax][idx] - d);
            }
        }
        last_iters = it; last_res = res;
        if (iters) *iters = it;
        if (residual) *residual = res;
        return capped ? MP_ERR_NOCONVERGE : MP_OK;
    }
    int project(int* iters, double* residual) {
        if (P.coef_mode == MP_COEF_GFM) return project_gfm(iters, residual);
        if (P.precision == MP_PREC_FP64) return project_t<double>(iters, residual);
        return project_t<float>(iters, residual);
    }

    // mapvelg2p_bubble (spray.cu:1689-1705): computeDeltaU (spray_k.cu:997-1006)
    // and mapvelg2p_flip_bubble (spray_k.cu:3525-3540); flip_alpha < 1 blends
    // as advectparticle_RK2_bubble does (spray_k.cu:3487-3490).
    void g2p() {
        for (int a = 0; a < 3; a++) {
            #pragma omp parallel for
            for (size_t i = 0; i < wu[a].size(); i++) wuo[a][i] = wu[a][i] - wuo[a][i];
            #pragma omp parallel for
            for (size_t i = 0; i < au[a].size(); i++) auo[a][i] = au[a][i] - auo[a][i];
        }
        float al = P.flip_alpha;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            F3 ip = pos[p];
            int8_t f = flag[p];
            F3 gv = mk(0.0f);
            const std::vector<float>* du = nullptr; const std::vector<float>* uu = nullptr;
            if (f == TF || f == TSOL) { du = wuo; uu = wu; }
            else if (f == TA) { du = auo; uu = au; }
            if (du) gv = velFromGrid(ip, du);
            if (al == 1.0f || !du) vel[p] += gv;
            else {
                F3 ug = velFromGrid(ip, uu);
                vel[p] = (1 - al) * ug + al * (vel[p] + gv);
            }
        }
    }

    // ---- the water mode (watersim, spray.cpp:741-797) -------------------------
    void flip_mark() {   // flipAirVacuum (spray_k.cu:461-469)
        for (int idx = 0; idx < n; idx++) if (mark[idx] == TV) mark[idx] = TA;
    }
    void water_p2g() {   // mapvelp2g (spray.cu:340-353)
        p2g_into(wu, 0);
        for (int a = 0; a < 3; a++) wuo[a] = wu[a];
    }
    // project_CG (spray.cu:241-271): cptdivergence (spray_k.cu:86-100) over
    // FLUID cells, CG with FLUID unknowns (computeAx, spray_k.cu:2300-2322),
    // subGradPress on the water faces
    int project_water(int* iters, double* residual) {
        std::vector<float> b(n, 0.0f), x(n, 0.0f);
        for (int idx = 0; idx < n; idx++) {
            int i, j, k; getijk(idx, i, j, k);
            if (mark[idx] == TF)
                b[idx] = (wu[0][fx(i + 1, j, k)] - wu[0][fx(i, j, k)] + wu[1][fy(i, j + 1, k)] - wu[1][fy(i, j, k)] +
                          wu[2][fz(i, j, k + 1)] - wu[2][fz(i, j, k)]) / h;
        }
        divg = b;
        auto mask = [&](int i) { return mark[i] == TF; };
        auto A = [&](std::vector<float>& o, const std::vector<float>& v) {
            float h2 = h * h;
            #pragma omp parallel for
            for (int idx = 0; idx < n; idx++) {
                if (mark[idx] != TF) { o[idx] = 0; continue; }
                int i, j, k; getijk(idx, i, j, k);
                float c = v[idx];
                float s = -6.0f * c;
                auto nb = [&](int a, int bb, int cc) { int q = cid(a, bb, cc); return (mark[q] == TB) ? c : v[q]; };
                s += nb(i + 1, j, k); s += nb(i, j + 1, k); s += nb(i, j, k + 1);
                s += nb(i - 1, j, k); s += nb(i, j - 1, k); s += nb(i, j, k - 1);
                o[idx] = s / h2;
            }
        };
        bool capped = false;
        double res = 0;
        int it = cg<float>(x, b, mask, A, P.cg_max_iter, P.cg_tol_mode, P.cg_tol, P.cg_true_residual_every, res, capped);
        press = x;
        subgrad<float>(wu, x);
        last_iters = it; last_res = res;
        if (iters) *iters = it;
        if (residual) *residual = res;
        return capped ? MP_ERR_NOCONVERGE : MP_OK;
    }
    void water_g2p() {   // mapvelg2p (spray.cu:362-376): computeDeltaU, mapvelg2p_flip
        for (int a = 0; a < 3; a++)
            for (size_t i = 0; i < wu[a].size(); i++) wuo[a][i] = wu[a][i] - wuo[a][i];
        #pragma omp parallel for
        for (int p = 0; p < np; p++) vel[p] += velFromGrid(pos[p], wuo);
    }
    void water_advect() {   // advectparticle_RK2 (spray_k.cu:409-458), velmode FLIP
        F3 g0 = mk(P.gmin_x, P.gmin_y, P.gmin_z);
        F3 g1 = g0 + mk((float)NX, (float)NY, (float)NZ) * h;
        const float flip = 0.95f;   // FLIP_ALPHA (utility.h:9)
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            F3 ip = pos[p], iv = vel[p];
            F3 tmin = g0 + (mk(h, h, h) + mk(0.5f * P.samplespace));
            F3 tmax = g1 - (mk(h, h, h) + mk(0.5f * P.samplespace));
            F3 gv = velFromGrid(ip, wu);
            iv = (1 - flip) * gv + flip * iv;
            F3 mid = ip + gv * P.dt * 0.5f;
            F3 gvm = velFromGrid(mid, wu);
            ip += gvm * P.dt;
            if (ip.x <= tmin.x) { ip.x = tmin.x; iv.x = 0.0f; }
            if (ip.y <= tmin.y) { ip.y = tmin.y; iv.y = 0.0f; }
            if (ip.z <= tmin.z) { ip.z = tmin.z; iv.z = 0.0f; }
            if (ip.x >= tmax.x) { ip.x = tmax.x; iv.x = 0.0f; }
            if (ip.y >= tmax.y) { ip.y = tmax.y; iv.y = 0.0f; }
            if (ip.z >= tmax.z) { ip.z = tmax.z; iv.z = 0.0f; }
            vel[p] = iv;
            if (flag[p] != TSOL) pos[p] = ip;
        }
    }
    int watersim() {
        int rc = MP_OK, st;
        hash_sort();
        sweep_phi(TF);
        levelset(0); sweep_ls_mark();
        flip_mark();
        surface_tension();
        water_p2g();
        sweep_u(TF); set_boundary_u(TF);
        st = project_water(nullptr, nullptr); if (st) rc = st;
        sweep_u(TF); set_boundary_u(TF);
        water_g2p();
        water_advect();
        hash_sort();
        correct_pos();
        if (P.b_run_mc) { mc_presort(); st = mc(MP_MC_FLUID); if (st) return st; }
        frame++;
        return rc;
    }

    // FP64 sum of a float3 array over SOLID-masked entries (accumulate_GPU_f3)
    static void dsum3(const std::vector<F3>& a, int nn, double out[3]) {
        out[0] = out[1] = out[2] = 0;
        for (int i = 0; i < nn; i++) { out[0] += a[i].x; out[1] += a[i].y; out[2] += a[i].z; }
    }
    // solidmotion_fixed / solidmotion (spray.cu:2685-2798)
    void solid_motion() {
        if (P.b_fix_solid) {   // setVelZeroSolid_k (spray_k.cu:5213)
            for (int p = 0; p < np; p++) if (flag[p] == TSOL) vel[p] = mk(0.0f);
            return;
        }
        if (nreal_solid <= 0) return;
        {   // solidCollisionWithBound (spray_k.cu:5478-5508)
            F3 g0 = mk(P.gmin_x, P.gmin_y, P.gmin_z);
            F3 g1 = g0 + mk((float)NX, (float)NY, (float)NZ) * h;
            F3 tmin = g0 + (mk(h, h, h) + mk(0.3f * P.samplespace));
            F3 tmax = g1 - (mk(h, h, h) + mk(0.3f * P.samplespace));
            float sb = P.solid_bounce_param;
            int ns = nreal_solid;
            for (int p = 0; p < np; p++) {
                if (flag[p] != TSOL) continue;
                F3 ip = pos[p], iv = vel[p];
                if (ip.x < tmin.x) iv.x += (tmin.x - ip.x) * sb * ns;
                if (ip.x > tmax.x) iv.x -= (ip.x - tmax.x) * sb * ns;
                if (ip.y < tmin.y) iv.y += (tmin.y - ip.y) * sb * ns;
                if (ip.y > tmax.y) iv.y -= (ip.y - tmax.y) * sb * ns;
                if (ip.z < tmin.z) iv.z += (tmin.z - ip.z) * sb * ns;
                if (ip.z > tmax.z) iv.z -= (ip.z - tmax.z) * sb * ns;
                vel[p] = iv;
            }
        }
        std::vector<F3> sp(np), sv(np), c(np), I(np);
        for (int p = 0; p < np; p++) {
            bool s = flag[p] == TSOL;
            sp[p] = s ? pos[p] : mk(0.0f);
            sv[p] = s ? vel[p] : mk(0.0f);
        }
        float fs = (float)nreal_solid;
        double d[3];
        dsum3(sv, np, d);
        F3 Tt = mk((float)d[0], (float)d[1], (float)d[2]) / fs;
        if (P.scene == MP_SCENE_INTERACTION) Tt.y = 0.0f;
        dsum3(sp, np, d);
        F3 rg0 = mk((float)d[0], (float)d[1], (float)d[2]) / fs;
        F3 rg = rg0 + P.dt * Tt;
        for (int p = 0; p < np; p++) {   // compute_cI_k (spray_k.cu:5188-5211)
            if (flag[p] == TSOL) {
                float dis = length(pos[p] - rg0);
                if (dis > 1e-6) { c[p] = cross(pos[p] - rg0, vel[p]); I[p] = mk(dis, 0, 0); }
                else c[p] = I[p] = mk(0.0f);
            } else c[p] = I[p] = mk(0.0f);
        }
        dsum3(I, np, d);
        F3 tI = mk((float)d[0], (float)d[1], (float)d[2]);
        dsum3(c, np, d);
        F3 R = mk((float)d[0], (float)d[1], (float)d[2]);
        if (tI.x <= 0) tI.x = 1;
        tI.x /= fs;
        R = R / tI.x / tI.x;
        R /= fs;
        for (int p = 0; p < np; p++) {   // computeVelSolid_k (spray_k.cu:5220-5232), called with rg0
            if (flag[p] != TSOL) continue;
            F3 vh = cross(R, pos[p] - rg0);
            vh += Tt;
            vh = 0.5f * (vel[p] + vh);
            vel[p] = vh;
        }
        F3 axis = R;
        float theta = -length(R) * P.dt;
        if (fabsf(theta) > 1e-6) axis = normalize(axis);
        else { axis = mk(1, 0, 0); theta = 0; }
        float x = axis.x, y = axis.y, z = axis.z;
        float cc = cosf(theta), s = sinf(theta);
        float m00 = cc + (1 - cc) * x * x, m01 = (1 - cc) * x * y - s * z, m02 = (1 - cc) * x * z + s * y;
        float m10 = (1 - cc) * y * x + s * z, m11 = cc + (1 - cc) * y * y, m12 = (1 - cc) * y * z - s * x;
        float m20 = (1 - cc) * z * x - s * y, m21 = (1 - cc) * z * y + s * x, m22 = cc + (1 - cc) * z * z;
        for (int p = 0; p < np; p++) {   // computePosSolid_k (spray_k.cu:5243-5252)
            if (flag[p] != TSOL) continue;
            F3 t = pos[p] - rg0;
            F3 r2 = mk(t.x * m00 + t.y * m10 + t.z * m20, t.x * m01 + t.y * m11 + t.z * m21,
                       t.x * m02 + t.y * m12 + t.z * m22);
            pos[p] = r2 + rg;
        }
        // computeSolidVertex_k (spray_k.cu:5254-5263) on the solid surface kept
        // from frame 0 when bRunMCSolid is off (spray.cu:2771-2772)
        const int sc = P.scene;
        if ((sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES || sc == MP_SCENE_MELTANDBOIL ||
             sc == MP_SCENE_MELTANDBOIL_HIGHRES) && frame > 0 && !P.b_run_mc_solid && P.b_run_mc) {
            for (F3& v : mc_out[MP_MC_SOLID].verts) {
                F3 t = v - rg0;
                F3 r2 = mk(t.x * m00 + t.y * m10 + t.z * m20, t.x * m01 + t.y * m11 + t.z * m21,
                           t.x * m02 + t.y * m12 + t.z * m22);
                v = r2 + rg;
            }
        }
    }

    // updateSoloAirParticle (spray.cu:2620-2651)
    void solo_air_update() {
        float hh = h, h2 = hh * hh;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // calcDensPress_Air (spray_k.cu:4284-4309)
            if (flag[p] != TA && flag[p] != TS) continue;
            F3 ip = pos[p];
            int i, j, k; ijkpos(ip, i, j, k);
            float d = 0;
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                float res = 0;   // sumdensity (spray_k.cu:4265-4282)
                if (!cell_empty(c))
                    for (uint32_t q = cstart[c]; q < cend[c]; q++) {
                        if (flag[q] != TA && flag[q] != TS) continue;
                        F3 dd = pos[q] - ip;
                        float d2 = dot(dd, dd);
                        if (d2 < h2) res += powf(h2 - d2, 3.0f);
                    }
                d += res;
            }
            d *= P.airm0 * P.poly6kern;
            if (d == 0) d = 1.0f;
            dens[p] = 1.0f / d;
            prs[p] = 1.5f * (d - P.waterrho * 0.5f);
        }
        std::vector<F3> ovel(vel.begin(), vel.begin() + np);
        float vterm = P.lapkern * P.viscosity_sph;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // enforceForceSoloAirP (spray_k.cu:4335-4373)
            if (flag[p] != TS && flag[p] != TA) continue;
            F3 ip = pos[p], iv = ovel[p];
            float ipr = prs[p], idn = dens[p];
            int i, j, k; ijkpos(ip, i, j, k);
            F3 force = mk(0.0f);
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                F3 res = mk(0.0f);   // sumforce (spray_k.cu:4311-4333)
                if (!cell_empty(c))
                    for (uint32_t q = cstart[c]; q < cend[c]; q++) {
                        F3 dir = ip - pos[q];
                        float dis = length(dir);
                        if (dis > 0 && dis < hh && (flag[q] == TS || flag[q] == TA)) {
                            float cc = hh - dis;
                            float pterm = -0.5f * cc * P.spikykern * (ipr + prs[q]) / dis;
                            float dterm = cc * idn * dens[q];
                            res += (pterm * dir + vterm * (ovel[q] - iv)) * dterm;
                        }
                    }
                force += res;
            }
            force *= P.airm0;
            iv += force * P.dt;
            vel[p] = iv;
        }
    }

    // CollisionSolid (spray.cu:2959-2983)
    void collide_advect() {
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // initSolidPhi (spray_k.cu:724-744)
            bool fl = false;
            if (!cell_empty(idx))
                for (uint32_t s = cstart[idx]; s < cend[idx]; s++) if (flag[s] == TSOL) fl = true;
            phisolid[idx] = fl ? -0.5f : (float)(3 * NX);
        }
        for (int it = 0; it < 3; it++) sweep_pass(phisolid, -1);
        p2g_into(su, 0);   // mapvelp2g_k_fluidSolid into solidu*
        bool freezing = P.scene == MP_SCENE_FREEZING || P.scene == MP_SCENE_MELTINGPOUR;
        F3 g0 = mk(P.gmin_x, P.gmin_y, P.gmin_z);
        F3 g1 = g0 + mk((float)NX, (float)NY, (float)NZ) * h;
        if (!freezing) {
            #pragma omp parallel for
            for (int p = 0; p < np; p++) {   // CollisionWithSolid_k (spray_k.cu:5276-5346)
                if (flag[p] == TSOL) continue;
                F3 ip = pos[p], iv = vel[p];
                float iphi = scaleFromGrid(ip, phisolid);
                if (iphi <= 0.5f) {
                    F3 sv = velFromGrid(ip, su);
                    F3 rv = iv - sv;
                    float d = h * 0.5f;
                    F3 pg;
                    pg.x = scaleFromGrid(ip + mk(d, 0, 0), phisolid) - scaleFromGrid(ip - mk(d, 0, 0), phisolid);
                    pg.y = scaleFromGrid(ip + mk(0, d, 0), phisolid) - scaleFromGrid(ip - mk(0, d, 0), phisolid);
                    pg.z = scaleFromGrid(ip + mk(0, 0, d), phisolid) - scaleFromGrid(ip - mk(0, 0, d), phisolid);
                    if (length(pg) > 0) {
                        pg = normalize(pg);
                        if (dot(rv, pg) < 0 || P.scene == MP_SCENE_FREEZING) {
                            iv -= P.bounce_vel_param * dot(rv, pg) * pg;
                            if (P.scene == MP_SCENE_FREEZING) iv -= 0.1f * (rv - dot(rv, pg) * pg);
                        }
                        ip += P.bounce_pos_param * pg * (0.5f - iphi) * h;
                    }
                }
                ip += iv * P.dt;
                float rate = 0.5f;
                if (flag[p] == TS) rate = 0.8f;
                F3 tmin = g0 + (mk(h, h, h) + mk(rate * h));
                F3 tmax = g1 - (mk(h, h, h) + mk(rate * h));
                if (ip.x <= tmin.x) { ip.x = tmin.x; iv.x = 0.0f; }
                if (ip.y <= tmin.y) { ip.y = tmin.y; iv.y = 0.0f; }
                if (ip.z <= tmin.z) { ip.z = tmin.z; iv.z = 0.0f; }
                if (ip.x >= tmax.x) { ip.x = tmax.x; iv.x = 0.0f; }
                if (ip.y >= tmax.y) { ip.y = tmax.y; iv.y = 0.0f; }
                if (ip.z >= tmax.z) { ip.z = tmax.z; iv.z = 0.0f; }
                vel[p] = iv; pos[p] = ip;
            }
        } else {
            std::vector<F3> opos(pos.begin(), pos.begin() + np);
            #pragma omp parallel for
            for (int p = 0; p < np; p++) {   // CollisionWithSolid_Freezing (spray_k.cu:5348-5447)
                if (flag[p] == TSOL) continue;
                F3 ip = opos[p], iv = vel[p];
                int i, j, k; ijkpos(ip, i, j, k);
                float iphi = scaleFromGrid(ip, phisolid);
                if (iphi <= 1.0f) {
                    float r = 0.25f * h;
                    F3 cpos = mk(0.0f);
                    float depth = 0, adh = 0;
                    int ccol = 0, cadh = 0;
                    float hh = 4 * r;
                    for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                        if (!vc(i + di, j + dj, k + dk)) continue;
                        int c = cid(i + di, j + dj, k + dk);
                        if (cell_empty(c)) continue;
                        for (uint32_t q = cstart[c]; q < cend[c]; q++) {
                            F3 dir = ip - opos[q];
                            float dis = length(dir);
                            if (dis > 0 && dis < 2 * r) { cpos += opos[q]; depth = fmaxf(depth, 2 * r - dis); ccol++; }
                            else if (dis < hh) { adh += dis; cadh++; }
                        }
                    }
                    F3 nn;
                    float d = h * 0.5f;
                    nn.x = scaleFromGrid(ip + mk(d, 0, 0), phisolid) - scaleFromGrid(ip - mk(d, 0, 0), phisolid);
                    nn.y = scaleFromGrid(ip + mk(0, d, 0), phisolid) - scaleFromGrid(ip - mk(0, d, 0), phisolid);
                    nn.z = scaleFromGrid(ip + mk(0, 0, d), phisolid) - scaleFromGrid(ip - mk(0, 0, d), phisolid);
                    F3 ov = iv;
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
                F3 tmin = g0 + (mk(h, h, h) + mk(0.3f * P.samplespace));
                F3 tmax = g1 - (mk(h, h, h) + mk(0.3f * P.samplespace));
                if (ip.x > tmax.x) { iv.x *= -0.5f; ip.x = tmax.x; }
                if (ip.x < tmin.x) { iv.x *= -0.5f; ip.x = tmin.x; }
                if (ip.y > tmax.y) { iv.y *= -0.5f; ip.y = tmax.y; }
                if (ip.y < tmin.y) { iv.y *= -0.5f; ip.y = tmin.y; }
                if (ip.z > tmax.z) { iv.z *= -0.5f; ip.z = tmax.z; }
                if (ip.z < tmin.z) { iv.z *= -0.5f; ip.z = tmin.z; }
                ip += iv * P.dt;
                vel[p] = iv; pos[p] = ip;
            }
        }
    }

    // correctpos -> correctparticlepos (spray.cu:328-338, spray_k.cu:1334-1411)
    void correct_pos() {
        std::vector<F3> out(np);
        F3 g0 = mk(P.gmin_x, P.gmin_y, P.gmin_z);
        F3 g1 = g0 + mk((float)NX, (float)NY, (float)NZ) * h;
        F3 tmin = g0 + (mk(h, h, h) + mk(0.5f * P.samplespace));
        F3 tmax = g1 - (mk(h, h, h) + mk(0.5f * P.samplespace));
        float re = P.correction_radius * h;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            if (flag[p] == TSOL || flag[p] == TS) { out[p] = pos[p]; continue; }
            F3 ip = pos[p];
            int i, j, k; ijkpos(ip, i, j, k);
            F3 spring = mk(0.0f);
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                F3 s = mk(0.0f);
                if (!cell_empty(c))
                    for (uint32_t q = cstart[c]; q < cend[c]; ++q) {
                        float dist = length(pos[q] - ip);
                        float w = mass[q] * smooth_kernel(dist * dist, re);
                        if (dist > 0.1f * re) s += w * (ip - pos[q]) / dist;
                    }
                spring += s;
            }
            spring *= P.correction_spring * re;
            if (length(P.dt * spring) > 0.3f * h) ip += h * 0.3f * spring / length(spring);
            else ip += P.dt * spring;
            ip.x = fmaxf(tmin.x, fminf(tmax.x, ip.x));
            ip.y = fmaxf(tmin.y, fminf(tmax.y, ip.y));
            ip.z = fmaxf(tmin.z, fminf(tmax.z, ip.z));
            out[p] = ip;
        }
        for (int p = 0; p < np; p++) pos[p] = out[p];
    }

    // correctpos_bubble (spray.cu:2067-2107)
    void correct_pos_bubble() {
        int sc = P.scene;
        bool airver = sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES ||
                      sc == MP_SCENE_INTERACTION || sc == MP_SCENE_ALL;
        if (airver) compute_phigra(gxa, gya, gza, lsair);
        float rs = 0.5f * h;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            int8_t f = flag[p];
            if (f == TS || f == TSOL) continue;
            F3 ip = pos[p];
            int s = (f == TF) ? -1 : 1;
            F3 dir = vecFromGrid(ip, gx, gy, gz);
            float dl = length(dir);
            if (dl == 0) continue;
            dir = normalize(dir);
            float d = scaleFromGrid(ip, lsmerge) / dl;
            if (!airver) {   // correctbubblepos (spray_k.cu:3884-3939)
                if ((float)s * d < 0 && fabsf(d) < 0.5f * h) {
                    if (f == TA && fabsf(d) > 0.3f * h) ip = ip - d * dir;
                    else if (f == TF) {
                        ip = ip - d * dir;
                        dir = vecFromGrid(ip, gx, gy, gz);
                        dl = length(dir);
                        if (dl == 0) continue;
                        dir = normalize(dir);
                        d = scaleFromGrid(ip, lsmerge) / dl;
                        ip = ip + (float)s * (rs - (float)s * d) * dir;
                    }
                } else if (f == TF && (float)s * d < rs * 0.5f && (float)s * d >= 0) {
                    ip = ip + (float)s * (rs - (float)s * d) * dir;
                }
                pos[p] = ip;
            } else {         // correctbubblepos_air (spray_k.cu:3941-3991)
                if ((float)s * d < 0 && fabsf(d) < 0.5f * h) {
                    if (f == TA && fabsf(d) > 0.3f * h) ip = ip - d * dir;
                }
                if (f == TF) {
                    dir = vecFromGrid(ip, gxa, gya, gza);
                    dl = length(dir);
                    if (dl == 0) continue;
                    dir = normalize(dir);
                    d = scaleFromGrid(ip, lsair) / dl;
                    if (d < -1.3f * rs) ip = ip - (d - rs) * dir;
                }
                pos[p] = ip;
            }
        }
    }

    // ---- heat ------------------------------------------------------------
    void alpha_table(float a[MP_TYPECNT]) const {   // initHeatAlphaArray (spray.cu:3076-3090)
        a[TF] = P.heatalpha_fluid; a[TA] = P.heatalpha_air; a[TV] = P.heatalpha_vacuum;
        a[TSOL] = P.heatalpha_solid; a[TS] = P.heatalpha_air; a[TB] = 0;
    }
    // updateTemperature (spray.cu:1889-1947)
    int heat() {
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // mapHeatp2g_hash (spray_k.cu:4619-4653)
            int i, j, k; getijk(idx, i, j, k);
            F3 gp = mk((float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f);
            float scale = 1.0f / h, wsum = 0, hs = 0;
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                if (cell_empty(c)) continue;
                for (uint32_t p = cstart[c]; p < cend[c]; ++p) {
                    F3 d = pos[p] * scale - gp;
                    float w = sharp_kernel(dot(d, d), 1.4f);
                    wsum += w;
                    hs += w * T[p];
                }
            }
            Tp[idx] = (wsum > 0) ? (hs / wsum) : P.default_temperature;
        }
        if (P.b_add_heat_bottom) {
            #pragma omp parallel for
            for (int idx = 0; idx < n; idx++) {   // addHeatAtBottom (spray_k.cu:4492-4504)
                int i, j, k; getijk(idx, i, j, k);
                if (i >= 1 && i < NX - 1 && j >= 1 && j < NY - 1 && k <= 3) Tp[idx] += P.heat_increase_bottom;
                Tp[idx] = fminf(P.heat_clamp, Tp[idx]);
            }
        }
        bool capped = heat_solve();
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++)     // compTpChange (spray_k.cu:4607-4617)
            Tp_save[idx] = (mark[idx] != TB) ? Tp[idx] - Tp_save[idx] : 0;
        bool mab = P.scene == MP_SCENE_MELTANDBOIL || P.scene == MP_SCENE_MELTANDBOIL_HIGHRES || P.scene == MP_SCENE_ALL;
        float a = P.alpha_temp_trans;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // mapHeatg2p[_MeltAndBoil] (spray_k.cu:4655-4679)
            F3 ip = pos[p];
            float nt = a * (T[p] + scaleFromGrid(ip, Tp_save)) + (1 - a) * scaleFromGrid(ip, Tp);
            if (mab && flag[p] == TSOL) T[p] = 0.95f * (T[p]) + 0.05f * nt;
            else T[p] = nt;
        }
        float mp_ = P.melting_point, bp = P.boiling_point, lth = P.liquid_heat_th;
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // updateLatentHeat_k (spray_k.cu:5546-5573)
            if (flag[p] == TSOL && T[p] > mp_) { L[p] += T[p] - mp_; T[p] = mp_; }
            if (flag[p] == TF) {
                if (T[p] < mp_) { L[p] -= mp_ - T[p]; T[p] = mp_; }
                else if (T[p] > bp) { L[p] += T[p] - bp; T[p] = bp; }
                else L[p] = lth;
            }
        }
        return capped ? MP_ERR_NOCONVERGE : MP_OK;
    }
    // compb_heat, solver_cg_heat, setBoundaryHeat (spray.cu:1780-1852); true
    // when the CG stopped at its cap
    bool heat_solve() {
        Tp_save = Tp;
        float at[MP_TYPECNT]; alpha_table(at);
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {   // compb_heat (spray_k.cu:4507-4523)
            float alpha = at[(int)mark[idx]];
            if (P.b_fixed_heat && fixedheat[idx] != MP_UNDEF_TEMPERATURE)   // dormant branch :4515-4519
                Tp_old[idx] = fixedheat[idx] * h * h / alpha / P.dt;
            else
                Tp_old[idx] = Tp[idx] * h * h / alpha / P.dt;
        }
        std::fill(Tp.begin(), Tp.end(), 0.0f);
        auto mask = [&](int i) { return mark[i] != TB; };
        auto A = [&](std::vector<float>& o, const std::vector<float>& v) { ax_heat(o, v, at); };
        bool capped = false;
        double res = 0;
        int it = cg<float>(Tp, Tp_old, mask, A, P.heat_cg_max_iter, MP_TOL_REF_ABS, 0.01f, 0, res, capped);
        last_heat_iters = it; last_heat_res = res;
        if (P.b_extend_heat_to_boundary) {   // setBoundaryHeat (spray_k.cu:4585-4605), Jacobi
            std::vector<float> in = Tp;
            #pragma omp parallel for
            for (int idx = 0; idx < n; idx++) {
                int i, j, k; getijk(idx, i, j, k);
                if (i == NX - 1) Tp[idx] = in[cid(i - 1, j, k)];
                else if (i == 0) Tp[idx] = in[cid(i + 1, j, k)];
                else if (j == NY - 1) Tp[idx] = in[cid(i, j - 1, k)];
                else if (j == 0) Tp[idx] = in[cid(i, j + 1, k)];
                else if (k == NZ - 1) Tp[idx] = in[cid(i, j, k - 1)];
                else if (k == 0) Tp[idx] = in[cid(i, j, k + 1)];
            }
        }
        return capped;
    }
    // heatsim (spray.cu:1959-1987)
    int heatsim() {
        bool capped = heat_solve();
        frame++;
        return capped ? MP_ERR_NOCONVERGE : MP_OK;
    }
    // initheat_grid_k + markBoundaryCell (spray_k.cu:5603-5621, 535-545)
    void init_heat_grid() {
        for (int idx = 0; idx < n; idx++) {
            int i, j, k; getijk(idx, i, j, k);
            float x = (float)i, z = (float)k;
            float r = (float)(NX * 0.15);
            float a = x - (float)(NX / 4), b = z - (float)(NZ / 4);
            float a2 = x - (float)(NX / 4 * 3), b2 = z - (float)(NZ / 4 * 3);
            if (sqrtf(a * a + b * b) <= r) { Tp[idx] = 100; mark[idx] = TSOL; }
            else if (sqrtf(a2 * a2 + b2 * b2) <= r) { Tp[idx] = 0; mark[idx] = TF; }
            else if (z < (float)(NZ / 2)) { Tp[idx] = 20; mark[idx] = MP_TYPEVACUUM; }
            else { Tp[idx] = 80; mark[idx] = MP_TYPEAIR; }
            if (i == 0 || i == NX - 1 || j == 0 || j == NY - 1 || k == 0 || k == NZ - 1) mark[idx] = TB;
        }
    }

    // GenerateGasParticle (spray.cu:2653-2683): updatesolubility (spray_k.cu:4719-4727),
    // GenerateGasParticle_k (spray_k.cu:4730-4817) with slots ordered by cell.
    int gen_gas() {
        float dgr = P.init_dissolve_gas_rate;
        #pragma omp parallel for
        for (int p = 0; p < np; p++)
            if (flag[p] == TF) sol[p] = dgr * P.airm0 * expf(P.solubility_coef * (1.0f / T[p] - 1.0f / P.temperature0));
        std::vector<uint8_t> add(n, 0);
        struct NewP { F3 pos; float T; };
        std::vector<NewP> np_(n);
        float m0a = P.airm0;
        int rc = (int)randf.size();
        #pragma omp parallel for
        for (int idx = 0; idx < n; idx++) {
            int i, j, k; getijk(idx, i, j, k);
            if (k <= 1 || inBoundaryCell(i, j, k)) continue;
            if (cell_empty(idx)) continue;
            float gc = 0, gs = 0, gair = 0, vsum = 0;
            int lcnt = 0, gcnt = 0;
            F3 gpos = mk((float)i, (float)j, (float)k) * h;
            F3 gaspos = mk(0.0f), gasvel = mk(0.0f);
            for (uint32_t p = cstart[idx]; p < cend[idx]; p++) {
                if (flag[p] == TF) {
                    gc += gas[p]; gs += sol[p];
                    vsum += fmaxf(0.0f, L[p] - P.liquid_heat_th) * P.vapor_gen_rate * m0a;
                    lcnt++;
                } else if (flag[p] == TS || flag[p] == TA) {
                    gair += mass[p]; gaspos += pos[p]; gasvel += vel[p]; gcnt++;
                }
            }
            bool hasseed = false;
            for (size_t s = 0; s < seeds.size(); s++) if (seeds[s] == idx) hasseed = true;
            long long rb = ((long long)idx * (long long)frame) % (long long)(rc - 200);
            int base = (int)rb;
            F3 rp = mk(randf[(base + 0) % rc], randf[(base + 1) % rc], randf[(base + 2) % rc]);
            float rn = randf[(base + 3) % rc];
            float r = h * 0.25f;
            if (gc - gs + vsum > m0a && (hasseed || gcnt > 0)) {
                add[idx] = 1;
                if (gcnt > 0) np_[idx].pos = gaspos / (float)gcnt + (fmaxf(0.5f, rn) * r) * (rp - mk(0.5f)) * 2;
                else np_[idx].pos = gpos + h * rp;
                np_[idx].T = Tp[idx];
                for (uint32_t p = cstart[idx]; p < cend[idx]; p++)
                    if (flag[p] == TF) { gas[p] = fminf(gas[p], sol[p]); L[p] = fminf(L[p], P.liquid_heat_th); }
            }
        }
        int cnt = 0;
        for (int idx = 0; idx < n; idx++) cnt += add[idx];
        if (np + cnt > P.par_num_max) { err = "gen_gas: par_num_max exceeded"; return MP_ERR_CAPACITY; }
        int slot = np;
        for (int idx = 0; idx < n; idx++) {
            if (!add[idx]) continue;
            mass[slot] = m0a; pos[slot] = np_[idx].pos; vel[slot] = mk(0.0f);
            flag[slot] = TS; T[slot] = np_[idx].T; L[slot] = 0; gas[slot] = 0.0f; sol[slot] = 0.0f;
            slot++;
        }
        np += cnt;
        return MP_OK;
    }

    // deleteAirFluidParticle (spray.cu:2194-2248)
    void del() {
        int passes = 20;
        if (P.scene == MP_SCENE_INTERACTION) passes = (frame % 2 == 0) ? 1 : 0;
        for (int t = 0; t < passes; t++) {   // sweepVacuum (spray_k.cu:4117-4132), Jacobi
            std::vector<int8_t> in = mark;
            #pragma omp parallel for
            for (int idx = 0; idx < n; idx++) {
                if (in[idx] != TA) continue;
                int i, j, k; getijk(idx, i, j, k);
                for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2)
                    if (in[cid(i + di, j + dj, k + dk)] == TV) mark[idx] = TV;
            }
        }
        std::vector<uint8_t> keep(np);
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {   // markDeleteAirParticle (spray_k.cu:4134-4170)
            if (flag[p] == TSOL) { keep[p] = 1; continue; }
            int i, j, k; ijkpos(pos[p], i, j, k);
            if (flag[p] == TF) {
                float lsa = scaleFromGrid(pos[p], lsair);
                keep[p] = (lsa < -h) ? 0 : 1;
                continue;
            }
            int c = 0;
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++)
                if (vc(i + di, j + dj, k + dk) && mark[cid(i + di, j + dj, k + dk)] == TV) c++;
            keep[p] = (c == 0 && mass[p] > 0.000001f) ? 1 : 0;
        }
        int o = 0;   // deleteparticles (spray_k.cu:4172-4194)
        for (int p = 0; p < np; p++) {
            if (!keep[p]) continue;
            pos[o] = pos[p]; vel[o] = vel[p]; mass[o] = mass[p]; flag[o] = flag[p];
            T[o] = T[p]; L[o] = L[p]; sol[o] = sol[p]; gas[o] = gas[p];
            o++;
        }
        np = o;
    }

    // MeltSolid -> MeltingSolidByHeat (spray.cu:2816-2831, spray_k.cu:5059-5072)
    void melt() {
        int c = 0;
        for (int p = 0; p < np; p++)
            if (flag[p] == TSOL && L[p] > P.liquid_heat_th) { flag[p] = TF; L[p] = P.liquid_heat_th; c++; }
        nreal_solid -= c;
    }
    // Freezing -> FreezingSolidByHeat (spray.cu:2860-2875, spray_k.cu:5074-5124), snapshot reads
    void freeze() {
        std::vector<int8_t> of(flag.begin(), flag.begin() + np);
        std::vector<F3> op(pos.begin(), pos.begin() + np);
        int total = 0;
        #pragma omp parallel for reduction(+:total)
        for (int p = 0; p < np; p++) {
            if (of[p] != TF || !(L[p] < 0)) continue;
            F3 ip = op[p];
            int i, j, k; ijkpos(ip, i, j, k);
            float mind = 1000; int mi = -1, cs = 0;
            for (int di = -1; di <= 1; di++) for (int dj = -1; dj <= 1; dj++) for (int dk = -1; dk <= 1; dk++) {
                if (!vc(i + di, j + dj, k + dk)) continue;
                int c = cid(i + di, j + dj, k + dk);
                if (cell_empty(c)) continue;
                for (uint32_t q = cstart[c]; q < cend[c]; q++) {
                    if (of[q] != TSOL) continue;
                    float d = length(op[q] - ip);
                    if (d < h) cs++;
                    if (d < mind) { mind = d; mi = (int)q; }
                }
            }
            if (mi != -1 && mind < h && cs > 2) {
                flag[p] = TSOL; L[p] = 0; total++;
                if (mind > P.samplespace) pos[p] = normalize(ip - op[mi]) * P.samplespace + op[mi];
            }
        }
        nreal_solid += total;
    }

    // ---- marching cubes ----------------------------------------------------
    // preMC + hashAndSortParticles_MC (spray.cu:759-765, 639-662; calcHashD_MC spray_k.cu:1030)
    void mc_presort() {
        NXMC = 2 * NX; NYMC = 2 * NY; NZMC = 2 * NZ;
        float dx = h / (float)NXMC * (float)NX;
        std::vector<uint32_t> key(np);
        F3 g0 = mk(P.gmin_x, P.gmin_y, P.gmin_z);
        #pragma omp parallel for
        for (int p = 0; p < np; p++) {
            F3 q = (pos[p] - g0) / mk(dx, dx, dx);
            int i = (q.x >= 0 && q.x < NXMC) ? (int)q.x : 0;
            int j = (q.y >= 0 && q.y < NYMC) ? (int)q.y : 0;
            int k = (q.z >= 0 && q.z < NZMC) ? (int)q.z : 0;
            key[p] = (uint32_t)(i * NYMC * NZMC + j * NZMC + k);
        }
        sort_by_keys(key, NXMC * NYMC * NZMC, mc_cstart, mc_cend);
    }
    // density fields: genWaterDensfield_GY (solid), _liquidAndGas (fluid),
    // _Gas (gas) (spray_k.cu:1528-1772)
    void mc_density(int surface) {
        int W = NXMC + 1, H = NYMC + 1, D = NZMC + 1;
        size_t nn = (size_t)W * H * D;
        mc_dens.assign(nn, 0.0f);
        float hm = h / (float)(NXMC / NX);
        int sc = P.scene;
        #pragma omp parallel for
        for (long long idx = 0; idx < (long long)nn; idx++) {
            int i, j, k; getijk3((int)idx, W, H, D, i, j, k);
            F3 p = mk((float)i, (float)j, (float)k) * hm;
            F3 center = mk(0.0f);
            float wsum = 0.0f;
            float phi;
            for (int di = -2; di <= 1; ++di) for (int dj = -2; dj <= 1; ++dj) for (int dk = -2; dk <= 1; ++dk) {
                int a = i + di, b = j + dj, c = k + dk;
                if (a < 0 || a > NXMC - 1 || b < 0 || b > NYMC - 1 || c < 0 || c > NZMC - 1) continue;
                int g = a * NYMC * NZMC + b * NZMC + c;
                F3 res = mk(0.0f);
                if (mc_cstart[g] != UNDEF) {
                    for (uint32_t q = mc_cstart[g]; q < mc_cend[g]; ++q) {
                        int f = flag[q];
                        if (surface == MP_MC_SOLID) {
                            if (f != TSOL) continue;
                            float dis = length(pos[q] - p);
                            if (dis < hm) {
                                float w = dis / (4 * hm);
                                w = 1 - w * w;
                                w = (float)std::max((double)(w * w * w), 0.0);
                                res += pos[q] * w; wsum += w;
                            }
                        } else {
                            bool ok = surface == MP_MC_FLUID ? (f == TA || f == TS || f == TF)
                                                             : (f == TA || (f == TS && sc != MP_SCENE_INTERACTION));
                            if (!ok) continue;
                            float R = hm * 2;
                            float dis = length(pos[q] - p);
                            if (dis < R) {
                                float w = R * R - dis * dis;
                                w = w * w * w;
                                res += pos[q] * w; wsum += w;
                            }
                        }
                    }
                }
                center += res;
            }
            bool border = (i * j * k == 0 || i == NXMC || j == NYMC || k == NZMC);
            if (surface == MP_MC_SOLID) {
                float r = 0.75f * hm, thigh = 0.51f, tlow = 0.49f;
                if (wsum > 0) {
                    center /= wsum;
                    F3 delta = center;   // centertmp is the zero vector the host passes
                    float Ev = fmaxf(delta.x, fmaxf(delta.y, delta.z)) / (4 * hm);
                    float gamma = (thigh - Ev) / (thigh - tlow);
                    float f = (Ev < tlow) ? 1 : gamma * gamma * gamma - 3 * gamma * gamma + 3 * gamma;
                    phi = (length(p - center) - r * f);
                } else phi = -r;
                if (border) phi = fminf(phi, -10.0f);
            } else {
                float r = surface == MP_MC_FLUID ? 0.5f * hm : 0.8f * hm;
                if (wsum > 0) { center /= wsum; phi = r - length(p - center); }
                else phi = -r;
                if (border) phi = -1000.0f;
            }
            mc_dens[idx] = phi;
        }
    }
    int mc(int surface) {
        mc_density(surface);
        return mc_extract(surface);
    }
    // genSphereDensfield (spray_k.cu:1827-1846): the analytic sphere field the
    // reference used to test its extraction, then the extraction itself
    int mc_sphere(int surface, F3 center, float radius) {
        NXMC = 2 * NX; NYMC = 2 * NY; NZMC = 2 * NZ;
        const int W = NXMC + 1, H = NYMC + 1, D = NZMC + 1;
        mc_dens.assign((size_t)W * H * D, 0.0f);
        for (int i = 0; i < W; i++) for (int j = 0; j < H; j++) for (int k = 0; k < D; k++) {
            float phi;
            if (i * j * k == 0 || i == NXMC || j == NYMC || k == NZMC) phi = -0.1f;
            else {
                F3 pp = mk((float)i, (float)j, (float)k) * h / (float)(NXMC / NX);
                phi = radius - length(pp - center);
            }
            mc_dens[((size_t)i * H + j) * D + k] = phi;
        }
        return mc_extract(surface);
    }
    int mc_extract(int surface) {
        int W = NXMC + 1, H = NYMC + 1, D = NZMC + 1;
        int nvox = NXMC * NYMC * NZMC;
        mc_cube.assign(nvox, 0);
        auto V = [&](int i, int j, int k) { return mc_dens[(size_t)i * H * D + (size_t)j * D + k]; };
        std::vector<uint32_t> nverts(nvox);
        #pragma omp parallel for
        for (int idx = 0; idx < nvox; idx++) {   // classifyVoxel (spray_k.cu:1853-1889)
            int i, j, k; getijk3(idx, NXMC, NYMC, NZMC, i, j, k);
            float f[8] = {V(i, j, k), V(i + 1, j, k), V(i + 1, j + 1, k), V(i, j + 1, k),
                          V(i, j, k + 1), V(i + 1, j, k + 1), V(i + 1, j + 1, k + 1), V(i, j + 1, k + 1)};
            uint32_t ci = 0;
            for (int v = 0; v < 8; v++) ci += (uint32_t)(f[v] < 0.0f) << v;
            mc_cube[idx] = (uint8_t)ci;
            nverts[idx] = (uint32_t)mc_numverts[ci];
        }
        MCOut& out = mc_out[surface];
        out.verts.clear(); out.normals.clear(); out.indices.clear(); out.active = 0;
        std::vector<int> act;
        for (int v = 0; v < nvox; v++) if (nverts[v] > 0) act.push_back(v);   // compactVoxels
        out.active = (int)act.size();
        if (act.empty()) return MP_OK;
        // edge ids: 3*node + axis (GetVertexID/GetEdgeID, spray_k.cu:1921-1959)
        static const int ecorner[12][2] = {{0,1},{1,2},{3,2},{0,3},{4,5},{5,6},{7,6},{4,7},{0,4},{1,5},{2,6},{3,7}};
        static const int cofs[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
        auto edge_gid = [&](int i, int j, int k, int e) -> size_t {
            const int* a = cofs[ecorner[e][0]];
            const int* b = cofs[ecorner[e][1]];
            int axis = (a[0] != b[0]) ? 0 : (a[1] != b[1] ? 1 : 2);
            size_t node = (size_t)(i + a[0]) * H * D + (size_t)(j + a[1]) * D + (k + a[2]);
            int ax = axis == 0 ? 0 : (axis == 1 ? 1 : 2);
            // reference: x-edges +1? GetEdgeID maps edge 0 (x) -> +1, edge 3 (y) -> +0, edge 8 (z) -> +2
            int off = ax == 0 ? 1 : (ax == 1 ? 0 : 2);
            return 3 * node + off;
        };
        size_t nedges = 3 * (size_t)W * H * D;
        std::vector<uint32_t> emark(nedges, 0);
        for (int v : act) {   // markActiveEdge_MC (spray_k.cu:2172-2220)
            int i, j, k; getijk3(v, NXMC, NYMC, NZMC, i, j, k);
            int ci = mc_cube[v];
            for (int t = 0; t < mc_numverts[ci]; t++) emark[edge_gid(i, j, k, mc_tri[ci * 16 + t])] = 1;
        }
        std::vector<uint32_t> escan(nedges);
        uint32_t tv = 0;
        for (size_t e = 0; e < nedges; e++) { escan[e] = tv; tv += emark[e]; }
        uint32_t ti = 0;
        std::vector<uint32_t> vscan(act.size());
        for (size_t a = 0; a < act.size(); a++) { vscan[a] = ti; ti += nverts[act[a]]; }
        if ((int)tv > P.mc_max_verts || (int)ti > 3 * P.mc_max_tris) { err = "mc: cap exceeded"; return MP_ERR_CAPACITY; }
        out.verts.assign(tv, mk(0.0f));
        out.indices.assign(ti, 0);
        float vs = h / (float)(NXMC / NX);
        // vertex positions, one per active edge from its lower node (vertexInterp, spray_k.cu:1904-1910)
        for (size_t e = 0; e < nedges; e++) {
            if (!emark[e]) continue;
            size_t node = e / 3; int off = (int)(e % 3);
            int axis = off == 1 ? 0 : (off == 0 ? 1 : 2);
            int i = (int)(node / ((size_t)H * D)), j = (int)((node / D) % H), k = (int)(node % D);
            F3 p0 = mk((float)i * vs, (float)j * vs, (float)k * vs);
            F3 p1 = p0 + (axis == 0 ? mk(vs, 0, 0) : (axis == 1 ? mk(0, vs, 0) : mk(0, 0, vs)));
            float f0 = V(i, j, k);
            float f1 = axis == 0 ? V(i + 1, j, k) : (axis == 1 ? V(i, j + 1, k) : V(i, j, k + 1));
            float t = (0.0f - f0) / (f1 - f0);
            out.verts[escan[e]] = p0 + t * (p1 - p0);
        }
        for (size_t a = 0; a < act.size(); a++) {   // generateTriangles_indices (spray_k.cu:2074-2170)
            int v = act[a];
            int i, j, k; getijk3(v, NXMC, NYMC, NZMC, i, j, k);
            int ci = mc_cube[v];
            for (int t = 0; t < mc_numverts[ci]; t++)
                out.indices[vscan[a] + t] = escan[edge_gid(i, j, k, mc_tri[ci * 16 + t])];
        }
        int ntri = (int)ti / 3;
        int nv = (int)tv;
        // vertex -> incident triangles in ascending triangle order
        std::vector<uint32_t> vstart(nv + 1, 0);
        for (uint32_t x : out.indices) vstart[x + 1]++;
        for (int q = 0; q < nv; q++) vstart[q + 1] += vstart[q];
        std::vector<uint32_t> inc(ti), fillp(vstart.begin(), vstart.end() - 1);
        for (int t = 0; t < ntri; t++)
            for (int c = 0; c < 3; c++) inc[fillp[out.indices[3 * t + c]]++] = 3 * t + c;
        if (P.b_smooth_mc) {   // smoothMesh (spray.cu:1271-1288), smooth_* (spray_k.cu:2408-2440)
            for (int it = 0; it < P.smooth_iters; it++) {
                std::vector<F3> np2 = out.verts;
                for (int q = 0; q < nv; q++) {
                    F3 disp = mk(0.0f); int w = 0;
                    F3 pq = out.verts[q];
                    for (uint32_t s = vstart[q]; s < vstart[q + 1]; s++) {
                        uint32_t slot = inc[s]; int t = slot / 3, c = slot % 3;
                        uint32_t o1 = out.indices[3 * t + (c == 0 ? 1 : 0)];
                        uint32_t o2 = out.indices[3 * t + (c == 2 ? 1 : 2)];
                        disp += out.verts[o1] - pq;
                        disp += out.verts[o2] - pq;
                        w += 2;
                    }
                    if (w > 0) np2[q] = pq + 0.5f * disp / (float)w;
                }
                out.verts.swap(np2);
                // the mu = -0.53 pass sees zeroed weights in the reference and changes nothing
            }
        }
        normals_of(out, vstart, inc);
        return MP_OK;
    }
    // calNormals (spray.cu:924-940; spray_k.cu:2223-2260)
    static void normals_of(MCOut& out, const std::vector<uint32_t>& vstart, const std::vector<uint32_t>& inc) {
        const int nv = (int)out.verts.size();
        out.normals.assign(nv, mk(0.0f));
        for (int q = 0; q < nv; q++) {
            F3 nrm = mk(0.0f);
            for (uint32_t s = vstart[q]; s < vstart[q + 1]; s++) {
                int t = inc[s] / 3;
                F3 p1 = out.verts[out.indices[3 * t]], p2 = out.verts[out.indices[3 * t + 1]], p3 = out.verts[out.indices[3 * t + 2]];
                nrm += cross(p2 - p1, p3 - p1);
            }
            if (length(nrm) > 0) nrm = normalize(nrm);
            out.normals[q] = nrm;
        }
    }
    // runMC_interaction's stored-surface branch (spray.cu:788-794)
    void renormal(int surface) {
        MCOut& out = mc_out[surface];
        const int nv = (int)out.verts.size(), ntri = (int)out.indices.size() / 3;
        std::vector<uint32_t> vstart(nv + 1, 0);
        for (uint32_t x : out.indices) vstart[x + 1]++;
        for (int q = 0; q < nv; q++) vstart[q + 1] += vstart[q];
        std::vector<uint32_t> inc(out.indices.size()), fillp(vstart.begin(), vstart.end() - 1);
        for (int t = 0; t < ntri; t++)
            for (int c = 0; c < 3; c++) inc[fillp[out.indices[3 * t + c]]++] = 3 * t + c;
        normals_of(out, vstart, inc);
    }

    // ---- initTemperature / initSolubility (spray.cu:1989-1999) -------------
    void init_particle_heat() {
        int ns = 0;
        for (int p = 0; p < np; p++) {   // initHeatParticle (spray_k.cu:4681-4698)
            if (flag[p] == TSOL) { T[p] = P.default_solid_T; L[p] = 0; ns++; }
            else { T[p] = P.default_liquid_T; L[p] = P.liquid_heat_th; }
        }
        for (int p = 0; p < np; p++) {   // initsolubility_k (spray_k.cu:4700-4717)
            if (flag[p] == TF || flag[p] == TSOL) {
                sol[p] = P.init_dissolve_gas_rate * P.airm0 * expf(P.solubility_coef * (1.0f / T[p] - 1.0f / P.temperature0));
                gas[p] = P.init_gas_rate * sol[p];
            } else { sol[p] = 0; gas[p] = 0; }
        }
        nreal_solid = ns;
    }

    // ---- bubblesim (spray.cpp:979-1233) ----------------------------------
    // ---- pouring and the frame-scripted switches (spray.cpp:998-1047) ----------
    std::vector<F3> pour_pos, pour_vel;
    void pour() {   // pouring / pouringgas (spray.cu:3012-3043), pouringwater (spray_k.cu:5575-5596)
        const int sc = P.scene;
        const bool is_gas = (sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES) && frame >= P.begin_frame;
        const int every = is_gas ? 6 : 4, npour = (int)pour_pos.size();
        if (frame % every != 0 || npour == 0 || (long long)npour + np > P.par_num_max) return;
        const int nr = (int)randf.size();
        if ((int)pos.size() < np + npour) return;
        for (int idx = 0; idx < npour; idx++) {
            int rb = (0 + idx) % (nr - 6);
            F3 rv = mk(randf[rb] * 2.0f - 1.0f, randf[rb + 1] * 2.0f - 1.0f, randf[rb + 2] * 2.0f - 1.0f);
            rb += 3;
            F3 rp = mk(randf[rb] * 2.0f - 1.0f, randf[rb + 1] * 2.0f - 1.0f, randf[rb + 2] * 2.0f - 1.0f);
            const int q = np + idx;
            pos[q] = pour_pos[idx] + rp * P.pos_rand_param * P.samplespace;
            vel[q] = pour_vel[idx] + rv * P.vel_rand_param;
            mass[q] = P.m0;
            flag[q] = (int8_t)(is_gas ? TS : TF);
            T[q] = P.default_liquid_T; L[q] = P.liquid_heat_th;
            sol[q] = 0.0f; gas[q] = 0.0f;
        }
        np += npour;
    }
    void scene_toggles() {
        const int sc = P.scene, f = frame;
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
        if (sc == MP_SCENE_MELTANDBOIL && f == 700) { P.b_gen_gas = !P.b_gen_gas; P.drag_param_grid = 0.03f; P.vapor_gen_rate = 0.005f; }
        if ((sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES) && f == P.begin_frame) P.b_fix_solid = 0;
    }

    int step() {
        int rc = MP_OK, st;
        pour();
        scene_toggles();
        int sc = P.scene;
        hash_sort();
        external_force();
        levelset(0); sweep_ls_mark();
        mark_solo_air();
        surface_tension();
        if (sc == MP_SCENE_MELTING || sc == MP_SCENE_FREEZING) markgrid_bubble();
        p2g();
        drag();
        sweep_phi(TA); sweep_u(TA); sweep_phi(TF); sweep_u(TF);
        set_boundary_u(TA); set_boundary_u(TF);
        st = project(nullptr, nullptr); if (st) rc = st;
        sweep_u(TA); sweep_u(TF);
        set_boundary_u(TA); set_boundary_u(TF);
        g2p();
        solid_motion();
        solo_air_update();
        hash_sort(); collide_advect();
        if (P.b_correct_position) {
            hash_sort(); correct_pos();
            hash_sort(); levelset(0.15f); sweep_ls_mark(); correct_pos_bubble();
        } else {
            hash_sort(); levelset(0.15f); sweep_ls_mark();
        }
        hash_sort();
        if (P.b_heat_trans) { st = heat(); if (st && !rc) rc = st; }
        if (P.b_gen_gas && frame % 2 == 0) { st = gen_gas(); if (st) return st; }
        hash_sort(); del();
        hash_sort();
        if (P.b_melt) melt();
        if (P.b_freeze) freeze();
        if (P.b_run_mc && P.mc_every > 0 && frame % P.mc_every == 0) {
            mc_presort();
            const bool inter = sc == MP_SCENE_INTERACTION || sc == MP_SCENE_INTERACTION_HIGHRES ||
                               sc == MP_SCENE_MELTANDBOIL || sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL;
            for (int s = 0; s < 3; s++) {
                if (s == MP_MC_SOLID && inter && frame > 0 && !P.b_run_mc_solid) { renormal(s); continue; }
                st = mc(s); if (st) return st;
            }
        }
        frame++;
        return rc;
    }

    // ---- field table --------------------------------------------------------
    void* field_ptr(int f, size_t& count, size_t& eb) {
        eb = 4;
        switch (f) {
        case MP_F_PRESS: count = n; return press.data();
        case MP_F_DIV: count = n; return divg.data();
        case MP_F_LSFLUID: count = n; return lsfluid.data();
        case MP_F_LSAIR: count = n; return lsair.data();
        case MP_F_LSMERGE: count = n; return lsmerge.data();
        case MP_F_PHIFLUID: count = n; return phifluid.data();
        case MP_F_PHIAIR: count = n; return phiair.data();
        case MP_F_PHISOLID: count = n; return phisolid.data();
        case MP_F_PHIGRAX: count = n; return gx.data();
        case MP_F_PHIGRAY: count = n; return gy.data();
        case MP_F_PHIGRAZ: count = n; return gz.data();
        case MP_F_PHIGRAX_AIR: count = n; return gxa.data();
        case MP_F_PHIGRAY_AIR: count = n; return gya.data();
        case MP_F_PHIGRAZ_AIR: count = n; return gza.data();
        case MP_F_SURFTENSION: count = n; return sf.data();
        case MP_F_TP: count = n; return Tp.data();
        case MP_F_TP_SAVE: count = n; return Tp_save.data();
        case MP_F_TP_OLD: count = n; return Tp_old.data();
        case MP_F_FIXEDHEAT: count = n; return fixedheat.data();
        case MP_F_MARK: count = n; eb = 1; return mark.data();
        case MP_F_WATERUX: case MP_F_WATERUY: case MP_F_WATERUZ: {
            int a = f - MP_F_WATERUX; count = wu[a].size(); return wu[a].data(); }
        case MP_F_WATERUX_OLD: case MP_F_WATERUY_OLD: case MP_F_WATERUZ_OLD: {
            int a = f - MP_F_WATERUX_OLD; count = wuo[a].size(); return wuo[a].data(); }
        case MP_F_AIRUX: case MP_F_AIRUY: case MP_F_AIRUZ: {
            int a = f - MP_F_AIRUX; count = au[a].size(); return au[a].data(); }
        case MP_F_AIRUX_OLD: case MP_F_AIRUY_OLD: case MP_F_AIRUZ_OLD: {
            int a = f - MP_F_AIRUX_OLD; count = auo[a].size(); return auo[a].data(); }
        case MP_F_SOLIDUX: case MP_F_SOLIDUY: case MP_F_SOLIDUZ: {
            int a = f - MP_F_SOLIDUX; count = su[a].size(); return su[a].data(); }
        case MP_F_CELLSTART: count = n; return cstart.data();
        case MP_F_CELLEND: count = n; return cend.data();
        case MP_P_POS: count = (size_t)np * 3; return pos.data();
        case MP_P_VEL: count = (size_t)np * 3; return vel.data();
        case MP_P_FLAG: count = np; eb = 1; return flag.data();
        case MP_P_MASS: count = np; return mass.data();
        case MP_P_TEMP: count = np; return T.data();
        case MP_P_LHEAT: count = np; return L.data();
        case MP_P_SOLUBILITY: count = np; return sol.data();
        case MP_P_GASCONTAIN: count = np; return gas.data();
        default: count = 0; return nullptr;
        }
    }
};

}  // namespace

extern "C" {

void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int or_create(const mp_params* p, void** out) {
    if (!p || !out) return MP_ERR_ARG;
    Oracle* o = new Oracle();
    o->P = *p;
    o->resize_grids();
    o->resize_particles(p->par_num_max);
    *out = o;
    return MP_OK;
}
void or_destroy(void* o) { delete (Oracle*)o; }
int or_set_params(void* v, const mp_params* p) {
    Oracle* o = (Oracle*)v;
    if (p->nx != o->P.nx || p->ny != o->P.ny || p->nz != o->P.nz || p->par_num_max != o->P.par_num_max) return MP_ERR_ARG;
    o->P = *p; o->h = p->cellsize; return MP_OK;
}
int or_get_state(void* v, mp_state* s) {
    Oracle* o = (Oracle*)v;
    memset(s, 0, sizeof(*s));
    s->frame = o->frame; s->par_num_now = o->np; s->n_real_solpoint = o->nreal_solid;
    s->last_cg_iters = o->last_iters; s->last_cg_residual = o->last_res;
    s->last_heat_cg_iters = o->last_heat_iters; s->last_heat_cg_residual = o->last_heat_res;
    for (int q = 0; q < 3; q++) {
        s->mc_verts[q] = (int)o->mc_out[q].verts.size();
        s->mc_indices[q] = (int)o->mc_out[q].indices.size();
        s->mc_active_voxels[q] = o->mc_out[q].active;
    }
    return MP_OK;
}
int or_set_state(void* v, const mp_state* s) {
    Oracle* o = (Oracle*)v;
    if (s->par_num_now < 0 || s->par_num_now > o->P.par_num_max) return MP_ERR_ARG;
    o->frame = s->frame; o->np = s->par_num_now; o->nreal_solid = s->n_real_solpoint;
    return MP_OK;
}
int or_upload_particles(void* v, int n, const float* pos3, const float* vel3, const int8_t* flag,
                        const float* mass, const float* temp, const float* lheat, const float* sol, const float* gas) {
    Oracle* o = (Oracle*)v;
    if (n < 0 || n > o->P.par_num_max) return MP_ERR_CAPACITY;
    o->np = n;
    for (int p = 0; p < n; p++) {
        o->pos[p] = mk(pos3[3 * p], pos3[3 * p + 1], pos3[3 * p + 2]);
        o->vel[p] = vel3 ? mk(vel3[3 * p], vel3[3 * p + 1], vel3[3 * p + 2]) : mk(0.0f);
        o->flag[p] = flag[p];
        o->mass[p] = mass[p];
        o->T[p] = temp ? temp[p] : 0.f; o->L[p] = lheat ? lheat[p] : 0.f;
        o->sol[p] = sol ? sol[p] : 0.f; o->gas[p] = gas ? gas[p] : 0.f;
    }
    return MP_OK;
}
int or_field_info(void* v, int f, size_t* count, size_t* eb) {
    Oracle* o = (Oracle*)v;
    size_t c, e; void* ptr = o->field_ptr(f, c, e);
    if (!ptr && c == 0 && !(f >= MP_P_POS && f <= MP_P_GASCONTAIN)) return MP_ERR_ARG;
    *count = c; *eb = e; return MP_OK;
}
int or_get_field(void* v, int f, void* dst, size_t bytes) {
    Oracle* o = (Oracle*)v;
    size_t c, e; void* ptr = o->field_ptr(f, c, e);
    if (bytes != c * e) return MP_ERR_ARG;
    if (bytes) memcpy(dst, ptr, bytes);
    return MP_OK;
}
int or_set_field(void* v, int f, const void* src, size_t bytes) {
    Oracle* o = (Oracle*)v;
    size_t c, e; void* ptr = o->field_ptr(f, c, e);
    if (bytes != c * e) return MP_ERR_ARG;
    if (f == MP_F_CELLSTART || f == MP_F_CELLEND) {   // cell ranges must stay inside the particle array
        const uint32_t* s = (const uint32_t*)src;
        for (size_t q = 0; q < c; q++)
            if (s[q] != UNDEF && s[q] > (uint32_t)o->np) return MP_ERR_ARG;
    }
    if (bytes) memcpy(ptr, src, bytes);
    return MP_OK;
}
int or_set_tables(void* v, const float* rf, int nrand, const int32_t* seeds, int nseed) {
    Oracle* o = (Oracle*)v;
    if (nrand <= 200) return MP_ERR_ARG;
    o->randf.assign(rf, rf + nrand);
    o->seeds.assign(seeds, seeds + nseed);
    return MP_OK;
}
int or_set_mc_tables(void* v, const int32_t* nv, const int32_t* tri) {
    Oracle* o = (Oracle*)v;
    o->mc_numverts.assign(nv, nv + 256);
    o->mc_tri.assign(tri, tri + 256 * 16);
    return MP_OK;
}
int or_init_particle_heat(void* v) { ((Oracle*)v)->init_particle_heat(); return MP_OK; }
int or_hash_sort(void* v) { ((Oracle*)v)->hash_sort(); return MP_OK; }
int or_external_force(void* v) { ((Oracle*)v)->external_force(); return MP_OK; }
int or_levelset(void* v, float off) { ((Oracle*)v)->levelset(off); return MP_OK; }
int or_sweep_ls_mark(void* v) { ((Oracle*)v)->sweep_ls_mark(); return MP_OK; }
int or_mark_solo_air(void* v) { ((Oracle*)v)->mark_solo_air(); return MP_OK; }
int or_surface_tension(void* v) { ((Oracle*)v)->surface_tension(); return MP_OK; }
int or_markgrid_bubble(void* v) { ((Oracle*)v)->markgrid_bubble(); return MP_OK; }
int or_p2g(void* v) { ((Oracle*)v)->p2g(); return MP_OK; }
int or_drag(void* v) { ((Oracle*)v)->drag(); return MP_OK; }
int or_sweep_phi(void* v, int ph) { ((Oracle*)v)->sweep_phi(ph); return MP_OK; }
int or_sweep_u(void* v, int ph) { ((Oracle*)v)->sweep_u(ph); return MP_OK; }
int or_set_boundary_u(void* v, int ph) { ((Oracle*)v)->set_boundary_u(ph); return MP_OK; }
int or_project(void* v, int* it, double* res) { return ((Oracle*)v)->project(it, res); }
int or_g2p(void* v) { ((Oracle*)v)->g2p(); return MP_OK; }
int or_solid_motion(void* v) { ((Oracle*)v)->solid_motion(); return MP_OK; }
int or_solo_air_update(void* v) { ((Oracle*)v)->solo_air_update(); return MP_OK; }
int or_collide_advect(void* v) { ((Oracle*)v)->collide_advect(); return MP_OK; }
int or_correct_pos(void* v) { ((Oracle*)v)->correct_pos(); return MP_OK; }
int or_correct_pos_bubble(void* v) { ((Oracle*)v)->correct_pos_bubble(); return MP_OK; }
int or_heat(void* v) { return ((Oracle*)v)->heat(); }
int or_heatsim(void* v) { return ((Oracle*)v)->heatsim(); }
int or_set_pour(void* v, const float* pos3, const float* vel3, int n) {
    Oracle* o = (Oracle*)v;
    o->pour_pos.resize(n); o->pour_vel.resize(n);
    for (int i = 0; i < n; i++) {
        o->pour_pos[i] = mk(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]);
        o->pour_vel[i] = mk(vel3[3 * i], vel3[3 * i + 1], vel3[3 * i + 2]);
    }
    return MP_OK;
}
int or_get_params(void* v, mp_params* p) { *p = ((Oracle*)v)->P; return MP_OK; }
int or_pour(void* v) { ((Oracle*)v)->pour(); return MP_OK; }
int or_mc_sphere(void* v, int s, float cx, float cy, float cz, float r) {
    Oracle* o = (Oracle*)v;
    if (s < 0 || s > 2 || o->mc_numverts.empty()) return MP_ERR_STATE;
    return o->mc_sphere(s, mk(cx, cy, cz), r);
}
int or_flip_mark(void* v) { ((Oracle*)v)->flip_mark(); return MP_OK; }
int or_water_p2g(void* v) { ((Oracle*)v)->water_p2g(); return MP_OK; }
int or_project_water(void* v, int* it, double* res) { return ((Oracle*)v)->project_water(it, res); }
int or_water_g2p(void* v) { ((Oracle*)v)->water_g2p(); return MP_OK; }
int or_water_advect(void* v) { ((Oracle*)v)->water_advect(); return MP_OK; }
int or_watersim(void* v) { return ((Oracle*)v)->watersim(); }
int or_init_heat_grid(void* v) { ((Oracle*)v)->init_heat_grid(); return MP_OK; }
int or_gen_gas(void* v) { return ((Oracle*)v)->gen_gas(); }
int or_delete(void* v) { ((Oracle*)v)->del(); return MP_OK; }
int or_melt(void* v) { ((Oracle*)v)->melt(); return MP_OK; }
int or_freeze(void* v) { ((Oracle*)v)->freeze(); return MP_OK; }
int or_mc_presort(void* v) { ((Oracle*)v)->mc_presort(); return MP_OK; }
int or_mc(void* v, int s) {
    Oracle* o = (Oracle*)v;
    if (s < 0 || s > 2 || o->mc_numverts.empty() || o->NXMC == 0) return MP_ERR_STATE;
    return o->mc(s);
}
int or_mc_get(void* v, int s, float* verts, float* normals, uint32_t* indices, int maxv, int maxi) {
    Oracle* o = (Oracle*)v;
    if (s < 0 || s > 2) return MP_ERR_ARG;
    MCOut& m = o->mc_out[s];
    if ((int)m.verts.size() > maxv || (int)m.indices.size() > maxi) return MP_ERR_CAPACITY;
    if (verts) memcpy(verts, m.verts.data(), m.verts.size() * 12);
    if (normals) memcpy(normals, m.normals.data(), m.normals.size() * 12);
    if (indices) memcpy(indices, m.indices.data(), m.indices.size() * 4);
    return MP_OK;
}
int or_mc_get_field(void* v, float* dens, uint8_t* cube) {
    Oracle* o = (Oracle*)v;
    if (dens) memcpy(dens, o->mc_dens.data(), o->mc_dens.size() * 4);
    if (cube) memcpy(cube, o->mc_cube.data(), o->mc_cube.size());
    return MP_OK;
}
int or_step(void* v) { return ((Oracle*)v)->step(); }

}  // extern "C"
