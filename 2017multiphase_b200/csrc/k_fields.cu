// k_fields.cu — level set, Eikonal sweeps, cell marks, velocity extrapolation
// and boundary conditions on the staggered grid.
//
// Reference kernels (Multiphase/Multiphase/spray_k.cu): genlevelset 2753-2806,
// sweepphibytype/sweepphi/solvedistance 746-788, markLS_bigpositive 3683,
// setLSback_bigpositive 3699, preparels 3708, setLSback 3724,
// mergeLSAndMarkGrid 3733, computePhigra 3994, sweepu_k_bubble 3779,
// setWaterBoundaryU_k 956, initphi 712, initSolidPhi 724, markfluid_dense 506,
// markBoundaryCell 535, compsurfacetension_k 3543.
// The reference updates the sweeps in place while neighbours read them (a
// data race); here every pass reads the previous pass (Jacobi) through a
// second buffer, so results do not depend on thread scheduling.
#include "ctx.cuh"

using namespace mpk;

namespace {

// genlevelset: unsigned distance to the nearest air / liquid particle in a
// 5x5x5 cell window, minus half a cell. min over sqrt(d2) == sqrt(min d2)
// because sqrtf is correctly rounded and monotone, so one sqrt per cell and
// phase gives the reference's value bit for bit.
// The window is visited nearest cells first and a cell is skipped when no
// particle in it can lower either minimum: a particle keyed to window cell
// (di,dj,dk) is at least (|d|-0.5)h away from the centre along each axis
// (particles keyed to cell 0 from outside the domain are further still), and
// distances of 2.5h or more are clamped anyway. The bound is shrunk by 1e-4
// relative so that float rounding of d2 can never make a skipped particle the
// minimum; the result is therefore identical to visiting every particle.
__constant__ signed char kWin[125][3] = {
    {0,0,0}, {-1,0,0}, {0,-1,0}, {0,0,-1}, {0,0,1}, {0,1,0}, {1,0,0}, {-1,-1,0}, {-1,0,-1}, {-1,0,1}, {-1,1,0}, {0,-1,-1}, {0,-1,1}, {0,1,-1}, {0,1,1}, {1,-1,0}, {1,0,-1}, {1,0,1}, {1,1,0}, {-1,-1,-1}, {-1,-1,1}, {-1,1,-1}, {-1,1,1}, {1,-1,-1}, {1,-1,1}, {1,1,-1}, {1,1,1}, {-2,0,0}, {0,-2,0}, {0,0,-2}, {0,0,2}, {0,2,0}, {2,0,0}, {-2,-1,0}, {-2,0,-1}, {-2,0,1}, {-2,1,0}, {-1,-2,0}, {-1,0,-2}, {-1,0,2}, {-1,2,0}, {0,-2,-1}, {0,-2,1}, {0,-1,-2}, {0,-1,2}, {0,1,-2}, {0,1,2}, {0,2,-1}, {0,2,1}, {1,-2,0}, {1,0,-2}, {1,0,2}, {1,2,0}, {2,-1,0}, {2,0,-1}, {2,0,1}, {2,1,0}, {-2,-1,-1}, {-2,-1,1}, {-2,1,-1}, {-2,1,1}, {-1,-2,-1}, {-1,-2,1}, {-1,-1,-2}, {-1,-1,2}, {-1,1,-2}, {-1,1,2}, {-1,2,-1}, {-1,2,1}, {1,-2,-1}, {1,-2,1}, {1,-1,-2}, {1,-1,2}, {1,1,-2}, {1,1,2}, {1,2,-1}, {1,2,1}, {2,-1,-1}, {2,-1,1}, {2,1,-1}, {2,1,1}, {-2,-2,0}, {-2,0,-2}, {-2,0,2}, {-2,2,0}, {0,-2,-2}, {0,-2,2}, {0,2,-2}, {0,2,2}, {2,-2,0}, {2,0,-2}, {2,0,2}, {2,2,0}, {-2,-2,-1}, {-2,-2,1}, {-2,-1,-2}, {-2,-1,2}, {-2,1,-2}, {-2,1,2}, {-2,2,-1}, {-2,2,1}, {-1,-2,-2}, {-1,-2,2}, {-1,2,-2}, {-1,2,2}, {1,-2,-2}, {1,-2,2}, {1,2,-2}, {1,2,2}, {2,-2,-1}, {2,-2,1}, {2,-1,-2}, {2,-1,2}, {2,1,-2}, {2,1,2}, {2,2,-1}, {2,2,1}, {-2,-2,-2}, {-2,-2,2}, {-2,2,-2}, {-2,2,2}, {2,-2,-2}, {2,-2,2}, {2,2,-2}, {2,2,2}};

__global__ void __launch_bounds__(256) k_genlevelset(Grid g, Cells cl, const float4* __restrict__ pos,
                                                     float* __restrict__ lsf, float* __restrict__ lsa,
                                                     int8_t* __restrict__ mark, const uint32_t* __restrict__ air_brick) {
    const uint32_t AIRB = (1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO);
    const uint32_t FLB = (1u << MP_TYPEFLUID) | (1u << MP_TYPESOLID);
    MP_GRID_LOOP(idx, g.n) {
        mark[idx] = MP_TYPEVACUUM;
        float h = g.h;
        float r = 0.5f * h;
        int i, j, k; getijk3((int)idx, g.NY, g.NZ, i, j, k);
        float3 gp = (mk3((float)i, (float)j, (float)k) + mk3(0.5f, 0.5f, 0.5f)) * h;
        const float cap2 = 6.25f * h * h * 1.001f;       // beyond 2.5h nothing changes
        float ma2 = __int_as_float(0x7f800000), mf2 = __int_as_float(0x7f800000);
        // no brick that the window (i-2..i+2, ...) touches holds an air
        // particle: the air distance stays at its cap, and the search for it
        // would visit every cell only to find no air
        bool air_near = false;
        {
            const int bw = (g.NZ + 3) / 4, bh = (g.NY + 3) / 4;
            const int bi0 = max(i - 2, 0) >> 2, bi1 = min(i + 2, g.NX - 1) >> 2;
            const int bj0 = max(j - 2, 0) >> 2, bj1 = min(j + 2, g.NY - 1) >> 2;
            const int bk0 = max(k - 2, 0) >> 2, bk1 = min(k + 2, g.NZ - 1) >> 2;
            for (int bi = bi0; bi <= bi1; bi++)
                for (int bj = bj0; bj <= bj1; bj++)
                    for (int bk = bk0; bk <= bk1; bk++) {
                        const int br = (bi * bh + bj) * bw + bk;
                        air_near |= (__ldg(air_brick + (br >> 5)) >> (br & 31)) & 1u;
                    }
        }
        if (!air_near) ma2 = 0.0f;   // searched no further; the value is replaced below
        for (int w = 0; w < 125; ++w) {
            int di = kWin[w][0], dj = kWin[w][1], dk = kWin[w][2];
            int a = i + di, b = j + dj, cc = k + dk;
            if (a < 0 || a > g.NX - 1 || b < 0 || b > g.NY - 1 || cc < 0 || cc > g.NZ - 1) continue;
            float bx = di == 0 ? 0.f : ((float)abs(di) - 0.5f), by = dj == 0 ? 0.f : ((float)abs(dj) - 0.5f);
            float bz = dk == 0 ? 0.f : ((float)abs(dk) - 0.5f);
            float lb2 = (bx * bx + by * by + bz * bz) * h * h * 0.9999f;
            bool wantA = lb2 < fminf(ma2, cap2), wantF = lb2 < fminf(mf2, cap2);
            // the window is ordered by this bound and the minima only fall:
            // no later cell is wanted either
            if (!wantA && !wantF) break;
            int c = cid(g, a, b, cc);
            uint32_t tm = __ldg(cl.tmask + c);
            if (!((wantA && (tm & AIRB)) || (wantF && (tm & FLB)))) continue;
            uint32_t s0 = __ldg(cl.off + c), s1 = __ldg(cl.off + c + 1);
            for (uint32_t p = s0; p < s1; ++p) {
                float4 q = __ldg(pos + p);
                float3 d = mk3(q.x, q.y, q.z) - gp;
                float d2 = dot(d, d);
                int f = pflag(q);
                if (f == MP_TYPEAIR || f == MP_TYPEAIRSOLO) ma2 = fminf(ma2, d2);
                else if (f == MP_TYPEFLUID || f == MP_TYPESOLID) mf2 = fminf(mf2, d2);
            }
        }
        if (!air_near) ma2 = __int_as_float(0x7f800000);
        float mair = 2.5f * h, mfl = 2.5f * h;
        float da = sqrtf(ma2), df = sqrtf(mf2);
        mair = (da < mair) ? da : mair;
        mfl = (df < mfl) ? df : mfl;
        mair -= r; mfl -= r;
        lsf[idx] = mfl;
        lsa[idx] = mair;
    }
}

__device__ __forceinline__ void solvedistance(float a, float b, float c, float& x) {
    float d = fminf(a, fminf(b, c)) + 1;
    if (d > fmaxf(a, fmaxf(b, c)))
        d = (a + b + c + sqrtf(3 - (a - b) * (a - b) - (a - c) * (a - c) - (b - c) * (b - c))) / 3;
    if (d < x) x = d;
}
// An octant with m = min(a,b,c) >= res cannot lower res, and skips the sqrt
// and the division, when its result is provably not below res: the result is
// m + 1 rounded (>= m) when that is not above the maximum; otherwise
// ((a+b)+c + sqrt(...)) / 3 rounded, which by monotone rounding is at least
// fl(fl(3m) / 3) (or NaN): that is m itself when 3m is exact
// (fl(3m) - 2m == m, the subtraction being exact), and at least m - ulp(m)
// otherwise, so then m two ulps down must still be >= res. sweep_settled(m)
// is the last two conditions, which depend on m alone.
__device__ __forceinline__ bool sweep_settled(float m, float res) {
    const float t = 3.0f * m;
    if (t - 2.0f * m == m) return true;
    return m > 1e-30f && __int_as_float(__float_as_int(m) - 2) >= res;
}
// one cell of a Jacobi pass of sweepphibytype (typeflag >= 0) or sweepphi
// (typeflag < 0)
__device__ __forceinline__ float sweep_cell(const Grid& g, const float* __restrict__ in,
                                            const int8_t* __restrict__ mark, int typeflag, int i, int j, int k,
                                            int idx) {
    const int sI = g.NY * g.NZ, sJ = g.NZ;
    float res = __ldg(in + idx);
    if (typeflag >= 0 && __ldg(mark + idx) == typeflag) return res;
    // the six neighbours, each loaded once; octants in the reference's order
    const bool vx[2] = {i > 0, i < g.NX - 1}, vy[2] = {j > 0, j < g.NY - 1}, vz[2] = {k > 0, k < g.NZ - 1};
    const float nx[2] = {vx[0] ? __ldg(in + idx - sI) : 0.f, vx[1] ? __ldg(in + idx + sI) : 0.f};
    const float ny[2] = {vy[0] ? __ldg(in + idx - sJ) : 0.f, vy[1] ? __ldg(in + idx + sJ) : 0.f};
    const float nz[2] = {vz[0] ? __ldg(in + idx - 1) : 0.f, vz[1] ? __ldg(in + idx + 1) : 0.f};
    // Every octant's minimum is one of the six values and at least their
    // minimum m6. When m6 >= res and each of the six values is settled, every
    // octant is skipped below, so the pass leaves the cell as it is: an exact
    // test, not a tolerance (a NaN among the six is never settled and takes
    // the octant loop). Most cells away from the interface take this exit.
    if (vx[0] && vx[1] && vy[0] && vy[1] && vz[0] && vz[1]) {
        const float m6 = fminf(fminf(fminf(nx[0], nx[1]), fminf(ny[0], ny[1])), fminf(nz[0], nz[1]));
        if (m6 >= res && sweep_settled(nx[0], res) && sweep_settled(nx[1], res) && sweep_settled(ny[0], res) &&
            sweep_settled(ny[1], res) && sweep_settled(nz[0], res) && sweep_settled(nz[1], res))
            return res;
    }
    #pragma unroll
    for (int a = 0; a < 2; a++)
    #pragma unroll
    for (int b = 0; b < 2; b++)
    #pragma unroll
    for (int e = 0; e < 2; e++) {
        if (!(vx[a] && vy[b] && vz[e])) continue;
        const float m = fminf(nx[a], fminf(ny[b], nz[e]));
        if (m >= res) {
            const float mx = fmaxf(nx[a], fmaxf(ny[b], nz[e]));
            if (!(m + 1 > mx)) continue;
            if (sweep_settled(m, res)) continue;
        }
        solvedistance(nx[a], ny[b], nz[e], res);
    }
    return res;
}
// A block covers one k-row of cells (blockIdx.z = i, blockIdx.y = j), a thread
// one cell, or two where the row is longer than the blocks along it, so no
// thread divides to find its cell.
constexpr int SWEEP_K = 128;
inline dim3 sweep_grid(int ni, int nj, int nk) { return dim3(std::max(1, nk / SWEEP_K), nj, ni); }
__global__ void __launch_bounds__(SWEEP_K) k_sweep(Grid g, const float* __restrict__ in, float* __restrict__ out,
                                                   const int8_t* __restrict__ mark, int typeflag) {
    const int j = blockIdx.y, i = blockIdx.z;
    const int row = (i * g.NY + j) * g.NZ;
    for (int k = blockIdx.x * SWEEP_K + threadIdx.x; k < g.NZ; k += gridDim.x * SWEEP_K)
        out[row + k] = sweep_cell(g, in, mark, typeflag, i, j, k, row + k);
}
// markLS_bigpositive (mode 0), setLSback_bigpositive (1), preparels (2), setLSback (3)
__global__ void k_ls_prep(int n, float h, float* __restrict__ ls, int8_t* __restrict__ mark, int mode) {
    MP_GRID_LOOP(idx, n) {
        float v = ls[idx];
        if (mode == 0) {
            v = v / h;
            if (v > 1.99f) { v = 5.0f; mark[idx] = MP_TYPEAIR; } else mark[idx] = MP_TYPEFLUID;
        } else if (mode == 1) {
            v = v * h;
        } else if (mode == 2) {
            v = -v / h;
            if (v > 0) { v = 5.0f; mark[idx] = MP_TYPEAIR; } else mark[idx] = MP_TYPEFLUID;
        } else {
            v = -v * h;
        }
        ls[idx] = v;
    }
}
__global__ void k_merge_ls(Grid g, float* __restrict__ lsm, int8_t* __restrict__ mark,
                           const float* __restrict__ lsf, const float* __restrict__ lsa) {
    MP_GRID_LOOP(idx, g.n) {
        float h = g.h;
        float lf = lsf[idx], la = lsa[idx], out;
        int8_t m;
        if (la > 4.99f * h) { out = lf; m = (lf > 0) ? MP_TYPEVACUUM : MP_TYPEFLUID; }
        else if (lf > 4.99f * h) { out = la; m = (la > 0) ? MP_TYPEVACUUM : MP_TYPEAIR; }
        else if (la > 0.8f * h && lf > 0.8f * h) { m = MP_TYPEVACUUM; out = fminf(lf, la); }
        else { out = (lf - la) * 0.5f; m = (out > 0) ? MP_TYPEAIR : MP_TYPEFLUID; }
        int i, j, k; getijk(g, (int)idx, i, j, k);
        if (i == 0 || i == g.NX - 1 || j == 0 || j == g.NY - 1 || k == 0 || k == g.NZ - 1) {
            m = MP_TYPEBOUNDARY; out = -0.5f * h;
        }
        mark[idx] = m;
        lsm[idx] = out;
    }
}
__global__ void k_phigra(Grid g, const float* __restrict__ ls, float* __restrict__ ax, float* __restrict__ ay,
                         float* __restrict__ az) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float c = ls[idx], h = g.h;
        float x1 = vc(g, i + 1, j, k) ? ls[cid(g, i + 1, j, k)] : c;
        float x0 = vc(g, i - 1, j, k) ? ls[cid(g, i - 1, j, k)] : c;
        float y1 = vc(g, i, j + 1, k) ? ls[cid(g, i, j + 1, k)] : c;
        float y0 = vc(g, i, j - 1, k) ? ls[cid(g, i, j - 1, k)] : c;
        float z1 = vc(g, i, j, k + 1) ? ls[cid(g, i, j, k + 1)] : c;
        float z0 = vc(g, i, j, k - 1) ? ls[cid(g, i, j, k - 1)] : c;
        ax[idx] = ((x1 - x0) * 0.5f) / h;
        ay[idx] = ((y1 - y0) * 0.5f) / h;
        az[idx] = ((z1 - z0) * 0.5f) / h;
    }
}
// initphi (spray_k.cu:712-722)
__global__ void k_initphi(int n, int NX, float* __restrict__ phi, const int8_t* __restrict__ mark, int type) {
    MP_GRID_LOOP(idx, n) phi[idx] = (mark[idx] == type) ? -0.5f : (float)(NX * 3);
}

// sweepu_k_bubble (spray_k.cu:3779-3880): one pass over all three face sets
// One extrapolation pass for a face of axis AX (sweepu_k_bubble): a face
// between two cells that are not of type fl takes the weighted average of
// its three upwind neighbour faces of the last octant (in the reference's
// loop order) whose three weights are all non-negative, else keeps its value.
// The eight level-set values the octants read are loaded once, and only the
// chosen octant's average is formed (the reference overwrites the result
// for every valid octant, so the last one is what remains).
template <int AX>
__device__ __forceinline__ float sweepu_face(const Grid& g, const float* __restrict__ in, const float* __restrict__ ls,
                                             const int8_t* __restrict__ mark, int fl, int i, int j, int k, int idx) {
    const int sI = g.NY * g.NZ, sJ = g.NZ;
    const int c0 = cid(g, i, j, k), c1 = c0 - (AX == 0 ? sI : (AX == 1 ? sJ : 1));
    float res = in[idx];
    const int e = AX == 0 ? i : (AX == 1 ? j : k), n = AX == 0 ? g.NX : (AX == 1 ? g.NY : g.NZ);
    if (!(e > 1 && e < n - 1 && mark[c0] != fl && mark[c1] != fl)) return res;
    // A face that is +0, with every neighbour face an octant can read (along
    // the normal, and across within the grid) +0 as well, stays +0 whatever
    // octant wins: the weights are non-negative, so the average is +0 too.
    // Most faces far from the phase (the air field inside the liquid) are so.
    if (__float_as_uint(res) == 0u) {
        auto fz = [&](int a, int b, int c) {
            const float v = AX == 0 ? in[fxi(g, a, b, c)] : (AX == 1 ? in[fyi(g, a, b, c)] : in[fzi(g, a, b, c)]);
            return __float_as_uint(v) == 0u;
        };
        bool zero = true;
        #pragma unroll
        for (int d = -1; d <= 1; d += 2) {
            if (AX == 0 || (i + d >= 0 && i + d <= g.NX - 1)) zero = zero && fz(i + d, j, k);
            if (AX == 1 || (j + d >= 0 && j + d <= g.NY - 1)) zero = zero && fz(i, j + d, k);
            if (AX == 2 || (k + d >= 0 && k + d <= g.NZ - 1)) zero = zero && fz(i, j, k + d);
        }
        if (zero) return res;
    }
    const float l0 = ls[c0], l1 = ls[c1];
    // the two cross axes (p, q) of this face axis, in the order the weights are named
    const int sP = AX == 0 ? sJ : sI, sQ = AX == 2 ? sJ : 1;
    const int ep = AX == 0 ? j : i, np_ = AX == 0 ? g.NY : g.NX;
    const int eq = AX == 2 ? j : k, nq = AX == 2 ? g.NY : g.NZ;
    // the cross neighbours' values, kept apart so the sums keep the reference's
    // order ((l0 + l1 - l(c0 + s)) - l(c1 + s))
    float p0[2] = {0, 0}, p1[2] = {0, 0}, q0[2] = {0, 0}, q1[2] = {0, 0};
    bool okp[2], okq[2];
    for (int t = 0; t < 2; t++) {
        int d = t == 0 ? -1 : 1;
        okp[t] = ep + d >= 0 && ep + d <= np_ - 1;
        okq[t] = eq + d >= 0 && eq + d <= nq - 1;
        if (okp[t]) { p0[t] = ls[c0 + d * sP]; p1[t] = ls[c1 + d * sP]; }
        if (okq[t]) { q0[t] = ls[c0 + d * sQ]; q1[t] = ls[c1 + d * sQ]; }
    }
    int sd = 0, sp = 0, sq = 0; float w0 = 0, wp = 0, wq = 0; bool found = false;
    // loop order of the reference: di, dj, dk each -1 then +1
    for (int di = -1; di <= 1; di += 2) for (int dj = -1; dj <= 1; dj += 2) for (int dk = -1; dk <= 1; dk += 2) {
        const int dn = AX == 0 ? di : (AX == 1 ? dj : dk);          // along the face normal
        const int dpp = AX == 0 ? dj : di, dqq = AX == 2 ? dj : dk;  // across
        const int tp = dpp > 0, tq = dqq > 0;
        if (!okp[tp] || !okq[tq]) continue;
        float wn = (float)(-dn) * (l0 - l1);
        if (wn < 0) continue;
        float a = (l0 + l1 - p0[tp] - p1[tp]) * 0.5f;
        if (a < 0) continue;
        float b = (l0 + l1 - q0[tq] - q1[tq]) * 0.5f;
        if (b < 0) continue;
        sd = dn; sp = dpp; sq = dqq; w0 = wn; wp = a; wq = b; found = true;
    }
    if (!found) return res;
    // name the weights by axis as the reference does (wx, wy, wz)
    float wx, wy, wz;
    if (AX == 0) { wx = w0; wy = wp; wz = wq; }
    else if (AX == 1) { wy = w0; wx = wp; wz = wq; }
    else { wz = w0; wx = wp; wy = wq; }
    float ws = wx + wy + wz;
    if (ws == 0) wx = wy = wz = 1.0f / 3;
    else { wx /= ws; wy /= ws; wz /= ws; }
    int di, dj, dk;
    if (AX == 0) { di = sd; dj = sp; dk = sq; }
    else if (AX == 1) { dj = sd; di = sp; dk = sq; }
    else { dk = sd; di = sp; dj = sq; }
    if (AX == 0) return wx * in[fxi(g, i + di, j, k)] + wy * in[fxi(g, i, j + dj, k)] + wz * in[fxi(g, i, j, k + dk)];
    if (AX == 1) return wx * in[fyi(g, i + di, j, k)] + wy * in[fyi(g, i, j + dj, k)] + wz * in[fyi(g, i, j, k + dk)];
    return wx * in[fzi(g, i + di, j, k)] + wy * in[fzi(g, i, j + dj, k)] + wz * in[fzi(g, i, j, k + dk)];
}
// one pass over the faces of axis AX, laid out as the cells of k_sweep: a block
// covers one (i, j) row of faces along k
template <int AX>
__global__ void __launch_bounds__(SWEEP_K) k_sweepu(Grid g, const float* __restrict__ in, float* __restrict__ out,
                                                    const float* __restrict__ ls, const int8_t* __restrict__ mark,
                                                    int fl) {
    const int j = blockIdx.y, i = blockIdx.z;
    const int kn = AX == 2 ? g.NZ + 1 : g.NZ;
    const int row = AX == 0 ? fxi(g, i, j, 0) : (AX == 1 ? fyi(g, i, j, 0) : fzi(g, i, j, 0));
    for (int k = blockIdx.x * SWEEP_K + threadIdx.x; k < kn; k += gridDim.x * SWEEP_K)
        out[row + k] = sweepu_face<AX>(g, in, ls, mark, fl, i, j, k, row + k);
}
__device__ __forceinline__ float zrule(const Grid& g, const int8_t* mark, int i, int j, int k, float v) {
    if (k <= 1) return 0.0f;
    if (k > 0 && k < g.NZ && ((mark[cid(g, i, j, k)] == MP_TYPEBOUNDARY) != (mark[cid(g, i, j, k - 1)] == MP_TYPEBOUNDARY)))
        return 0.0f;
    return v;
}
__global__ void k_bound_u(Grid g, float* __restrict__ ux, float* __restrict__ uy, float* __restrict__ uz,
                          const int8_t* __restrict__ mark) {
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k;
        if (t < g.nfx) {
            int idx = (int)t;
            getijk3(idx, g.NY, g.NZ, i, j, k);
            if (i <= 1 || i >= g.NX + 1 - 2) ux[idx] = 0.0f;
            else if (i > 1 && i < g.NX - 1 &&
                     ((mark[cid(g, i, j, k)] == MP_TYPEBOUNDARY) != (mark[cid(g, i - 1, j, k)] == MP_TYPEBOUNDARY)))
                ux[idx] = 0.0f;
        } else if (t < (long long)g.nfx + g.nfy) {
            int idx = (int)(t - g.nfx);
            getijk3(idx, g.NY + 1, g.NZ, i, j, k);
            if (j <= 1 || j >= g.NY + 1 - 2) uy[idx] = 0.0f;
            else if (j > 0 && j < g.NY &&
                     ((mark[cid(g, i, j, k)] == MP_TYPEBOUNDARY) != (mark[cid(g, i, j - 1, k)] == MP_TYPEBOUNDARY)))
                uy[idx] = 0.0f;
        } else {
            int idx = (int)(t - g.nfx - g.nfy);
            getijk3(idx, g.NY, g.NZ + 1, i, j, k);
            if (k <= 1 || k >= g.NZ + 1 - 1) uz[idx] = 0.0f;
            else if (k == g.NZ + 1 - 2) {
                float below = zrule(g, mark, i, j, k - 1, uz[fzi(g, i, j, k - 1)]);
                uz[idx] = (below < 0) ? below : 0;
            } else if (k > 0 && k < g.NZ &&
                       ((mark[cid(g, i, j, k)] == MP_TYPEBOUNDARY) != (mark[cid(g, i, j, k - 1)] == MP_TYPEBOUNDARY))) {
                uz[idx] = 0.0f;
            }
        }
    }
}

// markfluid_dense over the first `lim` cells (spray_k.cu:506-533) then
// markBoundaryCell (spray_k.cu:535-545)
__global__ void k_markfluid_dense(Grid g, Cells cl, const float4* __restrict__ pos, int8_t* __restrict__ mark, int lim) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        if (idx < lim) {
            int cfs = 0, ca = 0;
            for (uint32_t p = cl.off[idx]; p < cl.off[idx + 1]; ++p) {
                int f = pflag(pos[p]);
                if (f == MP_TYPEFLUID || f == MP_TYPESOLID) cfs++;
                else if (f == MP_TYPEAIR) ca++;
            }
            mark[idx] = (cfs == 0 && ca == 0) ? MP_TYPEVACUUM : (cfs > ca ? MP_TYPEFLUID : MP_TYPEAIR);
        }
        if (i == 0 || i == g.NX - 1 || j == 0 || j == g.NY - 1 || k == 0 || k == g.NZ - 1) mark[idx] = MP_TYPEBOUNDARY;
    }
}

// compsurfacetension_k (spray_k.cu:3543-3637)
__device__ __forceinline__ float st_comp(const Grid& g, const float* gx, const float* gy, const float* gz,
                                         int i, int j, int k, int axis, float dflt) {
    if (!vc(g, i, j, k)) return dflt;
    int q = cid(g, i, j, k);
    float a = gx[q], b = gy[q], c = gz[q];
    float l = length(mk3(a, b, c));
    if (l == 0) return dflt;
    float v = axis == 0 ? a : (axis == 1 ? b : c);
    return v / l;
}
__global__ void k_surftension(Grid g, float* __restrict__ sf, const int8_t* __restrict__ mark, const float* __restrict__ gx,
                              const float* __restrict__ gy, const float* __restrict__ gz, float sigma) {
    MP_GRID_LOOP(idx, g.n) {
        if (mark[idx] == MP_TYPEBOUNDARY) { sf[idx] = 0; continue; }
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float3 c = mk3(gx[idx], gy[idx], gz[idx]);
        float len = length(c), res;
        if (len == 0) res = 0;
        else {
            c /= len;
            float x1 = st_comp(g, gx, gy, gz, i + 1, j, k, 0, c.x), x0 = st_comp(g, gx, gy, gz, i - 1, j, k, 0, c.x);
            float y1 = st_comp(g, gx, gy, gz, i, j + 1, k, 1, c.y), y0 = st_comp(g, gx, gy, gz, i, j - 1, k, 1, c.y);
            float z1 = st_comp(g, gx, gy, gz, i, j, k + 1, 2, c.z), z0 = st_comp(g, gx, gy, gz, i, j, k - 1, 2, c.z);
            res = (x1 - x0 + y1 - y0 + z1 - z0) / g.h * 0.5f;
        }
        sf[idx] = res * sigma;
    }
}

// initSolidPhi (spray_k.cu:724-744)
// also raises *any when some cell holds a SOLID particle (one atomic per warp)
__global__ void k_init_solid_phi(Grid g, Cells cl, float* __restrict__ phi, uint32_t* __restrict__ any) {
    MP_GRID_LOOP(idx, g.n) {
        bool f = (cl.tmask[idx] >> MP_TYPESOLID) & 1;
        phi[idx] = f ? -0.5f : (float)(3 * g.NX);
        unsigned b = __ballot_sync(__activemask(), f);
        if (b && (threadIdx.x & 31) == (unsigned)(__ffs(__activemask()) - 1)) atomicOr(any, 1u);
    }
}

// flipAirVacuum (spray_k.cu:461-469): VACUUM cells become AIR (the water
// mode's free surface, a zero-pressure region for the single-phase solve)
__global__ void k_flip_air_vacuum(int n, int8_t* __restrict__ mark) {
    MP_GRID_LOOP(idx, n) if (mark[idx] == MP_TYPEVACUUM) mark[idx] = MP_TYPEAIR;
}

}  // namespace

static Cells cells_of(MpCtx* c) { return Cells{c->cell_off, c->tmask}; }

int k_sweep_pass_swap(MpCtx* c, float** phi, int typeflag) {
    const Grid& g = c->G;
    k_sweep<<<sweep_grid(g.NX, g.NY, g.NZ), SWEEP_K, 0, c->stream>>>(g, *phi, c->cell_tmp, c->mark, typeflag);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    std::swap(*phi, c->cell_tmp);
    return MP_OK;
}

int k_levelset(MpCtx* c) {
    KtScope kt(c, MP_KT_LEVELSET);
    k_genlevelset<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, cells_of(c), c->pos, c->lsfluid, c->lsair, c->mark,
                                                                 c->air_brick);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_phigra(MpCtx* c, float* ax, float* ay, float* az, const float* ls) {
    k_phigra<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, ls, ax, ay, az);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// sweepLSAndMardGrid (spray.cu:2011-2065)
static int sweep_ls_one(MpCtx* c, float** ls) {
    int n = c->G.n, nb = mp_blocks(n, 256);
    k_ls_prep<<<nb, 256, 0, c->stream>>>(n, c->G.h, *ls, c->mark, 0); c->launches++;
    MP_CHECK_LAUNCH(c);
    for (int it = 0; it < 5; it++) MP_TRY(k_sweep_pass_swap(c, ls, MP_TYPEFLUID));
    k_ls_prep<<<nb, 256, 0, c->stream>>>(n, c->G.h, *ls, c->mark, 1); c->launches++;
    k_ls_prep<<<nb, 256, 0, c->stream>>>(n, c->G.h, *ls, c->mark, 2); c->launches++;
    MP_CHECK_LAUNCH(c);
    for (int it = 0; it < 5; it++) MP_TRY(k_sweep_pass_swap(c, ls, MP_TYPEFLUID));
    k_ls_prep<<<nb, 256, 0, c->stream>>>(n, c->G.h, *ls, c->mark, 3); c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}
// flipMark_sphere (spray.cu:515-520)
int k_flip_mark(MpCtx* c) {
    k_flip_air_vacuum<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G.n, c->mark);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_sweep_ls_mark(MpCtx* c) {
    MP_TRY(sweep_ls_one(c, &c->lsfluid));
    MP_TRY(sweep_ls_one(c, &c->lsair));
    k_merge_ls<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, c->lsmerge, c->mark, c->lsfluid, c->lsair);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return k_phigra(c, c->gx, c->gy, c->gz, c->lsmerge);
}

// sweepPhi (spray.cu:570-583)
int k_sweep_phi(MpCtx* c, int phase) {
    float** phi = (phase == MP_TYPEAIR) ? &c->phiair : &c->phifluid;
    k_initphi<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G.n, c->G.NX, *phi, c->mark, phase);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    for (int it = 0; it < 3; it++) MP_TRY(k_sweep_pass_swap(c, phi, phase));
    return MP_OK;
}

// sweepU (spray.cu:585-598): two double-buffered passes
int k_sweep_u(MpCtx* c, int phase) {
    float** u = (phase == MP_TYPEAIR) ? c->au : c->wu;
    const float* phi = (phase == MP_TYPEAIR) ? c->phiair : c->phifluid;
    const Grid& g = c->G;
    for (int it = 0; it < 2; it++) {
        // the three face sets are independent: each reads only its own input
        k_sweepu<0><<<sweep_grid(g.NX + 1, g.NY, g.NZ), SWEEP_K, 0, c->stream>>>(g, u[0], c->tmpu[0], phi, c->mark, phase);
        k_sweepu<1><<<sweep_grid(g.NX, g.NY + 1, g.NZ), SWEEP_K, 0, c->stream>>>(g, u[1], c->tmpu[1], phi, c->mark, phase);
        k_sweepu<2><<<sweep_grid(g.NX, g.NY, g.NZ + 1), SWEEP_K, 0, c->stream>>>(g, u[2], c->tmpu[2], phi, c->mark, phase);
        c->launches += 3;
        MP_CHECK_LAUNCH(c);
        for (int a = 0; a < 3; a++) std::swap(u[a], c->tmpu[a]);
    }
    return MP_OK;
}

// setWaterBoundaryU (spray.cu:605-610)
int k_set_boundary_u(MpCtx* c, int phase) {
    float** u = (phase == MP_TYPEAIR) ? c->au : c->wu;
    long long tot = (long long)c->G.nfx + c->G.nfy + c->G.nfz;
    k_bound_u<<<mp_blocks(tot, 256), 256, 0, c->stream>>>(c->G, u[0], u[1], u[2], c->mark);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

// markgrid_bubble (spray.cu:511-518): the reference launches markfluid_dense
// with the particle grid, so only cells below ceil(np/512)*512 are marked
int k_markgrid_bubble(MpCtx* c) {
    int np = c->np();
    long long lim = (long long)std::max(1, (np + 511) / 512) * 512;
    if (lim > c->G.n) lim = c->G.n;
    k_markfluid_dense<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, cells_of(c), c->pos, c->mark, (int)lim);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_surface_tension_grid(MpCtx* c) {
    k_surftension<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, c->sf, c->mark, c->gx, c->gy, c->gz,
                                                                 c->P.surfacetension_sigma);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_solid_phi(MpCtx* c) {
    MP_CUDA(c, cudaMemsetAsync(c->u32_scratch + 2, 0, sizeof(uint32_t), c->stream));
    k_init_solid_phi<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, cells_of(c), c->phisolid, c->u32_scratch + 2);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    for (int it = 0; it < 3; it++) MP_TRY(k_sweep_pass_swap(c, &c->phisolid, -1));
    return MP_OK;
}
