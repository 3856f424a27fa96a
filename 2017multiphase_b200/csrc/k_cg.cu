// k_cg.cu — two-phase divergence, conjugate-gradient pressure and heat solves,
// pressure gradient, heat-grid bookkeeping.
//
// Reference: cptdivergence_bubble2 (Multiphase/Multiphase/spray_k.cu:3138-3263),
// solver_cg_bubble (spray.cu:1613-1687) with computeAx_bubble / pcg_op_bubble
// (spray_k.cu:3423-3460) and product()/arrayproduct_k (spray.cu:1101-1116,
// spray_k.cu:2279-2297), subGradPress (spray_k.cu:198-224); solver_cg_heat
// (spray.cu:1780-1852) with computeAx_heat / pcg_op_heat (spray_k.cu:4526-4583),
// addHeatAtBottom, compb_heat, setBoundaryHeat, compTpChange (spray_k.cu:4492-4617).
//
// The reference's "preconditioner" is the identity (z = r copies, spray.cu:1632,1671).
// It runs 3 host round trips per iteration (dot products summed on the host in
// FP32). Here alpha, beta and the residual live on the device in FP64; each
// iteration is two kernels, both recomputing A p from p instead of storing it:
//   k_cg_dir : p <- r + beta p (masked, double-buffered), z = A p, p.z
//   k_cg_upd : z = A p, x <- x + alpha p, r <- r - alpha z, r.r, stop test
// Dot products are FP64 block sums finished by the last block in block order,
// so they are deterministic. Vectors are FP32 (MP_PREC_MIXED) or FP64.
#include "ctx.cuh"
#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>

using namespace mpk;

namespace {

constexpr int CG_T = 256;

// device scalar slots
enum { S_A = 0, S_RR = 1, S_ALPHA = 2, S_BETA = 3, S_EPS = 4, S_ZP = 5, S_TRUE = 6 };
// flag slots (unsigned int): done state and iteration count
enum { F_DONE = 0, F_ITERS = 1, F_COUNT = 2 };
enum { DONE_RUN = 0, DONE_CONV = 1, DONE_CAP = 2, DONE_ZP0 = 3, DONE_TIMEOUT = 4 };

struct Red {
    double* part;           // gridDim.x partials
    unsigned int* count;    // last-block counter
    double* scal;
    unsigned int* flag;
};

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[CG_T / 32];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < CG_T / 32; w++) s += ws[w];
    return s;   // valid in thread 0
}
// returns true in thread 0 of the last block, with the total in *tot
__device__ __forceinline__ bool finish_sum(const Red& R, double mine, double* tot) {
    __shared__ bool last;
    double s = block_sum(mine);
    if (threadIdx.x == 0) {
        R.part[blockIdx.x] = s;
        __threadfence();
        unsigned int t = atomicAdd(R.count, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a = 0;   // fixed strided subsets, then a fixed tree (deterministic)
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += CG_T) a += __ldcg(R.part + b);
    double t2 = block_sum(a);
    if (threadIdx.x == 0) { *tot = t2; *R.count = 0; }
    return threadIdx.x == 0;
}

// ---- matrices --------------------------------------------------------------
// Both operators are applied to vectors that are exactly zero outside their
// unknowns (the reference's pcg_op writes 0 there), so a non-BOUNDARY
// neighbour that is not an unknown contributes its stored zero, as in the
// reference, without a test. (i,j,k) is decoded once per cell; neighbours are
// flat offsets. Unknowns are interior cells (the shell is BOUNDARY in a valid
// state; the interior test only keeps memory accesses in bounds otherwise).
__device__ __forceinline__ bool inner(const Grid& g, int i, int j, int k) {
    return i > 0 && i < g.NX - 1 && j > 0 && j < g.NY - 1 && k > 0 && k < g.NZ - 1;
}
// computeAx_bubble (spray_k.cu:3423-3447): rows over FLUID and AIR cells;
// with air = false, computeAx (spray_k.cu:2300-2322) of the single-phase
// solve: rows over FLUID cells only, AIR cells a zero-pressure region
struct PressOp {
    Grid g;
    const int8_t* __restrict__ mark;
    bool air = true;
    // 1/h^2 when h^2 is a power of two (then s * inv_h2 equals s / h^2 bit for
    // bit and saves the division), else 0
    float inv_h2 = 0.0f;
    __device__ __forceinline__ bool mask(int idx, int i, int j, int k) const {
        int m = mark[idx];
        return (m == MP_TYPEFLUID || (air && m == MP_TYPEAIR)) && inner(g, i, j, k);
    }
    template <class R, class F>
    __device__ __forceinline__ R apply(int idx, F val) const {
        const int sI = g.NY * g.NZ, sJ = g.NZ;
        R c = val(idx);
        R s = (R)(-6.0f) * c;
        R h2 = (R)g.h * (R)g.h;
        int q;
        q = idx + sI; s += (mark[q] == MP_TYPEBOUNDARY) ? c : val(q);
        q = idx + sJ; s += (mark[q] == MP_TYPEBOUNDARY) ? c : val(q);
        q = idx + 1;  s += (mark[q] == MP_TYPEBOUNDARY) ? c : val(q);
        q = idx - sI; s += (mark[q] == MP_TYPEBOUNDARY) ? c : val(q);
        q = idx - sJ; s += (mark[q] == MP_TYPEBOUNDARY) ? c : val(q);
        q = idx - 1;  s += (mark[q] == MP_TYPEBOUNDARY) ? c : val(q);
        return s / h2;
    }
    // the same row, piecewise, for the plane-marching kernels
    __device__ __forceinline__ bool fixed(int q) const { return mark[q] == MP_TYPEBOUNDARY; }
    template <class R> __device__ __forceinline__ R start(int, R c) const { return (R)(-6.0f) * c; }
    template <class R> __device__ __forceinline__ R comb(R s, R v) const { return s + v; }
    template <class R> __device__ __forceinline__ R finish(R s) const {
        if (inv_h2 != 0.0f) return s * (R)inv_h2;
        return s / ((R)g.h * (R)g.h);
    }
};
// PressOp with inv_h2 set when h^2 (rounded to float, as the stencil forms it)
// is an exact power of two
inline PressOp press_op(const Grid& g, const int8_t* mark, bool air = true) {
    PressOp op{g, mark, air};
    const float h2 = g.h * g.h;
    int e = 0;
    if (h2 > 0.0f && std::frexp(h2, &e) == 0.5f) op.inv_h2 = 1.0f / h2;
    return op;
}
// computeAx_heat (spray_k.cu:4526-4568): rows over non-BOUNDARY cells
struct HeatOp {
    Grid g;
    const int8_t* __restrict__ mark;
    float alpha[MP_TYPECNT];
    float dt;
    int boil;    // VACUUM neighbours also take the centre value in boiling scenes
    // alpha of a cell type by selects (a dynamic index into the parameter
    // array would copy it to local memory)
    __device__ __forceinline__ float al_of(int m) const {
        float a = alpha[0];
        #pragma unroll
        for (int t = 1; t < MP_TYPECNT; t++) a = (m == t) ? alpha[t] : a;
        return a;
    }
    __device__ __forceinline__ bool mask(int idx, int i, int j, int k) const {
        return mark[idx] != MP_TYPEBOUNDARY && inner(g, i, j, k);
    }
    __device__ __forceinline__ bool fix(int q) const {
        int m = mark[q];
        return boil ? (m == MP_TYPEBOUNDARY || m == MP_TYPEVACUUM) : (m == MP_TYPEBOUNDARY);
    }
    template <class R, class F>
    __device__ __forceinline__ R apply(int idx, F val) const {
        const int sI = g.NY * g.NZ, sJ = g.NZ;
        float al = al_of(mark[idx]);
        float h = g.h;
        R c = val(idx);
        R s = ((R)h * (R)h / (R)al / (R)dt + (R)6.0f) * c;
        int q;
        q = idx + sI; s -= fix(q) ? c : val(q);
        q = idx + sJ; s -= fix(q) ? c : val(q);
        q = idx + 1;  s -= fix(q) ? c : val(q);
        q = idx - sI; s -= fix(q) ? c : val(q);
        q = idx - sJ; s -= fix(q) ? c : val(q);
        q = idx - 1;  s -= fix(q) ? c : val(q);
        return s;
    }
    __device__ __forceinline__ bool fixed(int q) const { return fix(q); }
    template <class R> __device__ __forceinline__ R start(int idx, R c) const {
        float al = al_of(mark[idx]);
        float h = g.h;
        return ((R)h * (R)h / (R)al / (R)dt + (R)6.0f) * c;
    }
    template <class R> __device__ __forceinline__ R comb(R s, R v) const { return s - v; }
    template <class R> __device__ __forceinline__ R finish(R s) const { return s; }
};

// Ghost-fluid variable-density operator (the density-ratio extension; the
// reference's projection is constant-coefficient). Face weights beta = 1/rho
// of the face (kernel k_gfm_beta); rows over FLUID and AIR interior cells:
//   (A p)_c = sum over neighbours that are not walls of beta_f (p_nb - p_c) / h^2
// with p = 0 off the unknowns (beta = 1 everywhere gives computeAx_bubble).
// It is applied Jacobi-scaled, S A S with S = diag^-1/2 (zero off the
// unknowns), so plain CG on it is Jacobi-preconditioned CG on A.
struct GfmOp {
    Grid g;
    const int8_t* __restrict__ mark;
    const float* __restrict__ bx;
    const float* __restrict__ by;
    const float* __restrict__ bz;
    const float* __restrict__ S;
    __device__ __forceinline__ bool mask(int idx, int i, int j, int k) const {
        int m = mark[idx];
        return (m == MP_TYPEFLUID || m == MP_TYPEAIR) && inner(g, i, j, k);
    }
    __device__ __forceinline__ bool fixed(int q) const { return mark[q] == MP_TYPEBOUNDARY; }
    template <class R, class F>
    __device__ __forceinline__ R apply(int idx, F val) const {
        const int sI = g.NY * g.NZ, sJ = g.NZ;
        int i, j, k; getijk(g, idx, i, j, k);
        const R sc = (R)S[idx], c = val(idx);
        R s = 0;
        auto term = [&](int q, float beta) {
            if (mark[q] != MP_TYPEBOUNDARY) s += (R)beta * ((R)S[q] * val(q) - sc * c);
        };
        term(idx + sI, bx[fxi(g, i + 1, j, k)]);
        term(idx + sJ, by[fyi(g, i, j + 1, k)]);
        term(idx + 1, bz[fzi(g, i, j, k + 1)]);
        term(idx - sI, bx[fxi(g, i, j, k)]);
        term(idx - sJ, by[fyi(g, i, j, k)]);
        term(idx - 1, bz[fzi(g, i, j, k)]);
        return sc * s / ((R)g.h * (R)g.h);
    }
};
// operators whose rows are not the unit 7-point stencil take the general
// (one cell per thread) CG passes
template <class Op> struct op_general : std::false_type {};
template <> struct op_general<GfmOp> : std::true_type {};

#define CG_CELL_LOOP(idx, n, i, j, k)                                                  \
    MP_GRID_LOOP(idx, n)                                                               \
        for (int row_ = idx / op.g.NZ, k = idx - row_ * op.g.NZ,                        \
                 i = row_ / op.g.NY, j = row_ - i * op.g.NY, once_ = 1; once_; once_ = 0)

// r = mask ? b : 0 (x = 0, so b - A x = b); rr; a = rr; eps; stop if converged
template <class R, class Op>
__global__ void __launch_bounds__(CG_T) k_cg_init(Op op, int n, const R* __restrict__ b, R* __restrict__ r, Red Rd,
                                                  int tolmode, float tol) {
    double acc = 0;
    CG_CELL_LOOP(idx, n, i, j, k) {
        R v = op.mask((int)idx, i, j, k) ? (R)(b[idx] + (R)(-1.0f) * (R)0) : (R)0;
        r[idx] = v;
        acc += (double)v * (double)v;
    }
    double tot;
    if (finish_sum(Rd, acc, &tot)) {
        double eps = tolmode == MP_TOL_REF_ABS ? (double)(tol * (float)n) : (double)tol * (double)tol * tot;
        Rd.scal[S_RR] = tot; Rd.scal[S_A] = tot; Rd.scal[S_EPS] = eps;
        Rd.flag[F_ITERS] = 0;
        Rd.flag[F_DONE] = (tot < eps || (tolmode == MP_TOL_REL && eps == 0.0)) ? DONE_CONV : DONE_RUN;
    }
}

// p_new = r + beta p_old (first iteration: p = r), zero off the unknowns since
// r and p_old are; z = A p_new; p_new . z
template <class R, class Op>
__global__ void __launch_bounds__(CG_T) k_cg_dir(Op op, int n, const R* __restrict__ r, const R* __restrict__ pold,
                                                 R* __restrict__ pnew, Red Rd, int first) {
    if (Rd.flag[F_DONE] != DONE_RUN) return;
    const R bf = first ? (R)0 : (R)Rd.scal[S_BETA];
    auto pv = [&](int q) -> R { return first ? __ldg(r + q) : (R)(__ldg(r + q) + bf * __ldg(pold + q)); };
    double acc = 0;
    CG_CELL_LOOP(idx, n, i, j, k) {
        int id = (int)idx;
        bool m = op.mask(id, i, j, k);
        R pc = m ? pv(id) : (R)0;
        pnew[idx] = pc;
        if (m) {
            R z = op.template apply<R>(id, pv);
            acc += (double)z * (double)pc;
        }
    }
    double tot;
    if (finish_sum(Rd, acc, &tot)) {
        Rd.scal[S_ZP] = tot;
        if (tot == 0) Rd.flag[F_DONE] = DONE_ZP0;
        else Rd.scal[S_ALPHA] = Rd.scal[S_A] / tot;
    }
}

// z = A p, x += alpha p, r -= alpha z (masked), r.r, stop test, beta
template <class R, class Op>
__global__ void __launch_bounds__(CG_T) k_cg_upd(Op op, int n, const R* __restrict__ p, R* __restrict__ x,
                                                 R* __restrict__ r, Red Rd, int it, int maxiter, int skip_dot) {
    if (Rd.flag[F_DONE] != DONE_RUN) return;
    const R af = (R)Rd.scal[S_ALPHA];
    auto pv = [&](int q) -> R { return __ldg(p + q); };
    double acc = 0;
    CG_CELL_LOOP(idx, n, i, j, k) {
        int id = (int)idx;
        if (op.mask(id, i, j, k)) {
            R z = op.template apply<R>(id, pv);
            R xv = x[idx] + af * p[idx];
            R rv = r[idx] + (-af) * z;
            x[idx] = xv; r[idx] = rv;
            acc += (double)rv * (double)rv;
        } else {
            x[idx] = (R)0; r[idx] = (R)0;
        }
    }
    if (skip_dot) return;   // a true-residual pass follows
    double tot;
    if (finish_sum(Rd, acc, &tot)) {
        Rd.scal[S_RR] = tot;
        Rd.flag[F_ITERS] = it + 1;
        if (tot < Rd.scal[S_EPS]) Rd.flag[F_DONE] = DONE_CONV;
        else if (it + 1 >= maxiter) Rd.flag[F_DONE] = DONE_CAP;
        else { Rd.scal[S_BETA] = tot / Rd.scal[S_A]; Rd.scal[S_A] = tot; }
    }
}

// periodic true residual: r = mask ? b - A x : 0, then the same stop test
template <class R, class Op>
__global__ void __launch_bounds__(CG_T) k_cg_true(Op op, int n, const R* __restrict__ b, const R* __restrict__ x,
                                                  R* __restrict__ r, Red Rd, int it, int maxiter) {
    if (Rd.flag[F_DONE] != DONE_RUN) return;
    auto xv = [&](int q) -> R { return __ldg(x + q); };
    double acc = 0;
    CG_CELL_LOOP(idx, n, i, j, k) {
        int id = (int)idx;
        R v = (R)0;
        if (op.mask(id, i, j, k)) v = (R)(b[idx] + (R)(-1.0f) * op.template apply<R>(id, xv));
        r[idx] = v;
        acc += (double)v * (double)v;
    }
    double tot;
    if (finish_sum(Rd, acc, &tot)) {
        Rd.scal[S_RR] = tot;
        Rd.flag[F_ITERS] = it + 1;
        if (tot < Rd.scal[S_EPS]) Rd.flag[F_DONE] = DONE_CONV;
        else if (it + 1 >= maxiter) Rd.flag[F_DONE] = DONE_CAP;
        else { Rd.scal[S_BETA] = tot / Rd.scal[S_A]; Rd.scal[S_A] = tot; }
    }
}

// mixed-precision refinement: the true residual in FP64, r = mask ? b - A x :
// 0 with the row applied in FP64, its FP32 copy (the next correction's
// right-hand side) and |r|^2 into scal[slot]
template <class Op>
__global__ void __launch_bounds__(CG_T) k_cg_resid64(Op op, int n, const double* __restrict__ b,
                                                     const double* __restrict__ x, double* __restrict__ r,
                                                     float* __restrict__ r32, Red Rd, int slot) {
    auto xv = [&](int q) -> double { return __ldg(x + q); };
    double acc = 0;
    CG_CELL_LOOP(idx, n, i, j, k) {
        int id = (int)idx;
        double v = 0;
        if (op.mask(id, i, j, k)) v = b[idx] - op.template apply<double>(id, xv);
        r[idx] = v;
        r32[idx] = (float)v;
        acc += v * v;
    }
    double tot;
    if (finish_sum(Rd, acc, &tot)) Rd.scal[slot] = tot;
}
__global__ void k_add_f2d(int n, const float* __restrict__ e, double* __restrict__ x) {
    MP_GRID_LOOP(idx, n) x[idx] += (double)e[idx];
}

// ---- plane-marching stencil kernels -------------------------------------------
// A 32x8 thread tile covers (k, j) and marches along i over a chunk of planes.
// The value at (i+1) and (i-1) of a thread's own column lives in registers,
// the +-j / +-k neighbours of plane i come from a shared-memory tile with a
// one-cell halo, and a per-cell byte (built once per solve, k_nb8) says whether
// the cell is an unknown (bit 7) and which of its six neighbours take the
// centre value (bits 0-5, in the reference's order +x +y +z -x -y -z). Each
// value is read from HBM about once; the arithmetic and its order are those
// of PressOp/HeatOp::apply.
constexpr int PM_X = 32, PM_Y = 8;
struct PmGeom { int chunk; };

template <class Op>
__global__ void k_nb8(Op op, int n, uint8_t* __restrict__ nb8) {
    const int sI = op.g.NY * op.g.NZ, sJ = op.g.NZ;
    CG_CELL_LOOP(idx, n, i, j, k) {
        uint8_t m = 0;
        if (op.mask(idx, i, j, k)) {
            m = 0x80;
            if (op.fixed(idx + sI)) m |= 1;
            if (op.fixed(idx + sJ)) m |= 2;
            if (op.fixed(idx + 1)) m |= 4;
            if (op.fixed(idx - sI)) m |= 8;
            if (op.fixed(idx - sJ)) m |= 16;
            if (op.fixed(idx - 1)) m |= 32;
        }
        nb8[idx] = m;
    }
}

__device__ __forceinline__ bool pm_finish(const Red& R, double mine, double* tot) {
    __shared__ double ws[PM_X * PM_Y / 32];
    __shared__ bool last;
    const int tid = threadIdx.x + PM_X * threadIdx.y;
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    double v = mine;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) ws[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int w = 0; w < PM_X * PM_Y / 32; w++) s += ws[w];
        R.part[bid] = s;
        __threadfence();
        unsigned int t = atomicAdd(R.count, 1u);
        last = (t == nblk - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // the last block adds the partials: every thread a fixed strided subset
    // (independent L2 loads), then a fixed tree, so the sum is deterministic
    double a = 0;
    for (unsigned int b = tid; b < nblk; b += PM_X * PM_Y) a += __ldcg(R.part + b);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    __syncthreads();
    if ((tid & 31) == 0) ws[tid >> 5] = a;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int w = 0; w < PM_X * PM_Y / 32; w++) s += ws[w];
        *tot = s; *R.count = 0;
    }
    return tid == 0;
}

// MODE 0 (direction): value = r + beta p_old (first: r); writes p_new; sums p.Ap
// MODE 1 (update):    value = p; x += alpha p, r -= alpha Ap; sums r.r
template <class R, class Op, int MODE>
__global__ void __launch_bounds__(PM_X * PM_Y) k_cg_pm(Op op, PmGeom pg, const uint8_t* __restrict__ nb8,
                                                      const R* __restrict__ va, const R* __restrict__ vb,
                                                      R* __restrict__ pout, R* __restrict__ x, R* __restrict__ r,
                                                      Red Rd, int first, int it, int maxiter, int skip_dot) {
    if (Rd.flag[F_DONE] != DONE_RUN) return;
    __shared__ R tile[PM_Y + 2][PM_X + 2];
    const Grid& g = op.g;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int k = blockIdx.x * PM_X + tx, j = blockIdx.y * PM_Y + ty;
    const int i0 = blockIdx.z * pg.chunk, i1 = min(i0 + pg.chunk, g.NX);
    const bool inb = k < g.NZ && j < g.NY;
    const R bf = (MODE == 0 && !first) ? (R)Rd.scal[S_BETA] : (R)0;
    const R af = MODE == 1 ? (R)Rd.scal[S_ALPHA] : (R)0;
    auto ld = [&](int i, int jj, int kk) -> R {
        if (i < 0 || i >= g.NX || jj < 0 || jj >= g.NY || kk < 0 || kk >= g.NZ) return (R)0;
        int q = (i * g.NY + jj) * g.NZ + kk;
        if (MODE == 1 || first) return __ldg(va + q);
        return (R)(__ldg(va + q) + bf * __ldg(vb + q));
    };
    // halo slots of this thread (an edge thread of the tile owns one or two)
    const int hyj = ty == 0 ? j - 1 : (ty == PM_Y - 1 ? j + 1 : -1);
    const int hxk = tx == 0 ? k - 1 : (tx == PM_X - 1 ? k + 1 : -1);
    auto ldh = [&](int i, R& hy, R& hx) {
        if (hyj != -1) hy = ld(i, hyj, k);
        if (hxk != -1) hx = ld(i, j, hxk);
    };
    auto cell = [&](int i) { return (i * g.NY + j) * g.NZ + k; };
    // software pipeline: everything plane i needs is loaded during plane i-1,
    // the own column's value two planes ahead
    R behind = ld(i0 - 1, j, k), cur = ld(i0, j, k), front = ld(i0 + 1, j, k);
    R hy = 0, hx = 0;
    ldh(i0, hy, hx);
    uint32_t m = (inb && i0 < i1) ? nb8[cell(i0)] : 0u;
    R xc = 0, rc = 0;
    if (MODE == 1 && inb && i0 < i1) { xc = x[cell(i0)]; rc = r[cell(i0)]; }
    double acc = 0;
    for (int i = i0; i < i1; i++) {
        const bool more = i + 1 < i1;
        R front2 = ld(i + 2, j, k);
        R hyn = 0, hxn = 0;
        if (more) ldh(i + 1, hyn, hxn);
        uint32_t mn = 0; R xn = 0, rn = 0;
        if (inb && more) {
            mn = nb8[cell(i + 1)];
            if (MODE == 1) { xn = x[cell(i + 1)]; rn = r[cell(i + 1)]; }
        }
        __syncthreads();
        tile[ty + 1][tx + 1] = cur;
        if (hyj != -1) tile[ty == 0 ? 0 : PM_Y + 1][tx + 1] = hy;
        if (hxk != -1) tile[ty + 1][tx == 0 ? 0 : PM_X + 1] = hx;
        __syncthreads();
        if (inb) {
            const int c = cell(i);
            if (MODE == 0) pout[c] = (m & 0x80) ? cur : (R)0;
            if (m & 0x80) {
                R s = op.template start<R>(c, cur);
                s = op.template comb<R>(s, (m & 1) ? cur : front);
                s = op.template comb<R>(s, (m & 2) ? cur : tile[ty + 2][tx + 1]);
                s = op.template comb<R>(s, (m & 4) ? cur : tile[ty + 1][tx + 2]);
                s = op.template comb<R>(s, (m & 8) ? cur : behind);
                s = op.template comb<R>(s, (m & 16) ? cur : tile[ty][tx + 1]);
                s = op.template comb<R>(s, (m & 32) ? cur : tile[ty + 1][tx]);
                R z = op.template finish<R>(s);
                if (MODE == 0) {
                    acc += (double)z * (double)cur;
                } else {
                    R xv = xc + af * cur;
                    R rv = rc + (-af) * z;
                    x[c] = xv; r[c] = rv;
                    acc += (double)rv * (double)rv;
                }
            } else if (MODE == 1) {
                x[c] = (R)0; r[c] = (R)0;
            }
        }
        behind = cur; cur = front; front = front2;
        hy = hyn; hx = hxn; m = mn; xc = xn; rc = rn;
    }
    if (MODE == 1 && skip_dot) return;
    double tot;
    if (pm_finish(Rd, acc, &tot)) {
        if (MODE == 0) {
            Rd.scal[S_ZP] = tot;
            if (tot == 0) Rd.flag[F_DONE] = DONE_ZP0;
            else Rd.scal[S_ALPHA] = Rd.scal[S_A] / tot;
        } else {
            Rd.scal[S_RR] = tot;
            Rd.flag[F_ITERS] = it + 1;
            if (tot < Rd.scal[S_EPS]) Rd.flag[F_DONE] = DONE_CONV;
            else if (it + 1 >= maxiter) Rd.flag[F_DONE] = DONE_CAP;
            else { Rd.scal[S_BETA] = tot / Rd.scal[S_A]; Rd.scal[S_A] = tot; }
        }
    }
}

// ---- four cells along k per thread (FP32 vectors, NZ a multiple of 4) ---------
// The same two passes as k_cg_pm without shared memory or barriers: a thread
// owns one aligned float4 group of a k-row, loads the centre group, the four
// +-i / +-j groups and the two k-edge scalars, and applies the row of each of
// its four cells in the order of PressOp/HeatOp::apply. Groups without an
// unknown are skipped entirely: x, r and both direction vectors are zero
// there for the whole solve (x and the direction vectors are cleared at the
// start, r by k_cg_init), and nothing writes them.
template <class Op, int MODE>
__global__ void __launch_bounds__(CG_T, 6) k_cg_v4(Op op, const uint8_t* __restrict__ nb8,
                                                const float* __restrict__ va, const float* __restrict__ vb,
                                                float* __restrict__ pout, float* __restrict__ x, float* __restrict__ r,
                                                Red Rd, int first, int it, int maxiter, int skip_dot) {
    if (Rd.flag[F_DONE] != DONE_RUN) return;
    const Grid& g = op.g;
    const int NZ4 = g.NZ >> 2, sJ4 = NZ4, sI4 = g.NY * NZ4, ng = g.n >> 2;
    const float bf = (MODE == 0 && !first) ? (float)Rd.scal[S_BETA] : 0.0f;
    const float af = MODE == 1 ? (float)Rd.scal[S_ALPHA] : 0.0f;
    const float4* __restrict__ a4 = reinterpret_cast<const float4*>(va);
    const float4* __restrict__ b4 = reinterpret_cast<const float4*>(vb);
    auto val4 = [&](int q) -> float4 {
        float4 a = __ldg(a4 + q);
        if (MODE == 1 || first) return a;
        float4 b = __ldg(b4 + q);
        return make_float4(a.x + bf * b.x, a.y + bf * b.y, a.z + bf * b.z, a.w + bf * b.w);
    };
    auto val1 = [&](int q) -> float {
        if (MODE == 1 || first) return __ldg(va + q);
        return __ldg(va + q) + bf * __ldg(vb + q);
    };
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    double acc = 0;
    MP_GRID_LOOP(q, ng) {
        const uint32_t m4 = __ldg(reinterpret_cast<const uint32_t*>(nb8) + q);
        if (!(m4 & 0x80808080u)) continue;
        const int row = q / NZ4, kq = q - row * NZ4;
        const int i = row / g.NY, j = row - i * g.NY;
        const float4 c = val4(q);
        const float4 xp = i + 1 < g.NX ? val4(q + sI4) : zero4;
        const float4 xm = i > 0 ? val4(q - sI4) : zero4;
        const float4 yp = j + 1 < g.NY ? val4(q + sJ4) : zero4;
        const float4 ym = j > 0 ? val4(q - sJ4) : zero4;
        const float zm = kq > 0 ? val1(4 * q - 1) : 0.0f;
        const float zp = kq + 1 < NZ4 ? val1(4 * q + 4) : 0.0f;
        float4 xo = zero4, ro = zero4;
        if (MODE == 1) { xo = reinterpret_cast<const float4*>(x)[q]; ro = reinterpret_cast<const float4*>(r)[q]; }
        const float cv[6] = {zm, c.x, c.y, c.z, c.w, zp};
        const float xpv[4] = {xp.x, xp.y, xp.z, xp.w}, xmv[4] = {xm.x, xm.y, xm.z, xm.w};
        const float ypv[4] = {yp.x, yp.y, yp.z, yp.w}, ymv[4] = {ym.x, ym.y, ym.z, ym.w};
        float xov[4] = {xo.x, xo.y, xo.z, xo.w}, rov[4] = {ro.x, ro.y, ro.z, ro.w};
        float po[4];
        #pragma unroll
        for (int e = 0; e < 4; e++) {
            const uint32_t m = (m4 >> (8 * e)) & 0xffu;
            const float cur = cv[e + 1];
            po[e] = (m & 0x80) ? cur : 0.0f;
            if (m & 0x80) {
                float s = op.template start<float>(4 * q + e, cur);
                s = op.template comb<float>(s, (m & 1) ? cur : xpv[e]);
                s = op.template comb<float>(s, (m & 2) ? cur : ypv[e]);
                s = op.template comb<float>(s, (m & 4) ? cur : cv[e + 2]);
                s = op.template comb<float>(s, (m & 8) ? cur : xmv[e]);
                s = op.template comb<float>(s, (m & 16) ? cur : ymv[e]);
                s = op.template comb<float>(s, (m & 32) ? cur : cv[e]);
                const float z = op.template finish<float>(s);
                if (MODE == 0) {
                    acc += (double)z * (double)cur;
                } else {
                    xov[e] = xov[e] + af * cur;
                    rov[e] = rov[e] + (-af) * z;
                    acc += (double)rov[e] * (double)rov[e];
                }
            }
        }
        if (MODE == 0) {
            reinterpret_cast<float4*>(pout)[q] = make_float4(po[0], po[1], po[2], po[3]);
        } else {
            reinterpret_cast<float4*>(x)[q] = make_float4(xov[0], xov[1], xov[2], xov[3]);
            reinterpret_cast<float4*>(r)[q] = make_float4(rov[0], rov[1], rov[2], rov[3]);
        }
    }
    if (MODE == 1 && skip_dot) return;
    double tot;
    if (finish_sum(Rd, acc, &tot)) {
        if (MODE == 0) {
            Rd.scal[S_ZP] = tot;
            if (tot == 0) Rd.flag[F_DONE] = DONE_ZP0;
            else Rd.scal[S_ALPHA] = Rd.scal[S_A] / tot;
        } else {
            Rd.scal[S_RR] = tot;
            Rd.flag[F_ITERS] = it + 1;
            if (tot < Rd.scal[S_EPS]) Rd.flag[F_DONE] = DONE_CONV;
            else if (it + 1 >= maxiter) Rd.flag[F_DONE] = DONE_CAP;
            else { Rd.scal[S_BETA] = tot / Rd.scal[S_A]; Rd.scal[S_A] = tot; }
        }
    }
}

}  // namespace
#include "cg_tma.cuh"
namespace {

// cptdivergence_bubble2 (spray_k.cu:3138-3263)
template <class R>
__global__ void k_divergence(Grid g, const int8_t* __restrict__ mark, const float* __restrict__ ls,
                             const float* __restrict__ wx, const float* __restrict__ wy, const float* __restrict__ wz,
                             const float* __restrict__ ax, const float* __restrict__ ay, const float* __restrict__ az,
                             R* __restrict__ b, float* __restrict__ divf) {
    MP_GRID_LOOP(idx, g.n) {
        int m = mark[idx];
        R out = 0;
        if ((m == MP_TYPEFLUID || m == MP_TYPEAIR) && interior(g, (int)idx)) {
            int i, j, k; getijk(g, (int)idx, i, j, k);
            R lc = (R)ls[idx];
            auto face = [&](int a, int bb, int cc, R wv, R av) -> R {
                int q = cid(g, a, bb, cc);
                int mn = mark[q];
                if (m == MP_TYPEFLUID && mn != MP_TYPEAIR) return wv;
                if (m == MP_TYPEAIR && mn != MP_TYPEFLUID) return av;
                R th = ((R)0 - lc) / ((R)ls[q] - lc);
                if (m == MP_TYPEFLUID) return th * wv + (1 - th) * av;
                return th * av + (1 - th) * wv;
            };
            int f;
            f = fxi(g, i + 1, j, k); R ux1 = face(i + 1, j, k, (R)wx[f], (R)ax[f]);
            f = fxi(g, i, j, k);     R ux0 = face(i - 1, j, k, (R)wx[f], (R)ax[f]);
            f = fyi(g, i, j + 1, k); R uy1 = face(i, j + 1, k, (R)wy[f], (R)ay[f]);
            f = fyi(g, i, j, k);     R uy0 = face(i, j - 1, k, (R)wy[f], (R)ay[f]);
            f = fzi(g, i, j, k + 1); R uz1 = face(i, j, k + 1, (R)wz[f], (R)az[f]);
            f = fzi(g, i, j, k);     R uz0 = face(i, j, k - 1, (R)wz[f], (R)az[f]);
            out = (ux1 - ux0 + uy1 - uy0 + uz1 - uz0) / (R)g.h;
        }
        b[idx] = out;
        if (divf) divf[idx] = (float)out;
    }
}

// cptdivergence (spray_k.cu:86-100): the single-phase divergence of the water
// faces over FLUID cells, zero elsewhere, in the reference's summation order
__global__ void k_divergence_water(Grid g, const int8_t* __restrict__ mark, const float* __restrict__ ux,
                                   const float* __restrict__ uy, const float* __restrict__ uz, float* __restrict__ div) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float d = 0.0f;
        if (mark[idx] == MP_TYPEFLUID)
            d = (ux[fxi(g, i + 1, j, k)] - ux[fxi(g, i, j, k)] + uy[fyi(g, i, j + 1, k)] - uy[fyi(g, i, j, k)] +
                 uz[fzi(g, i, j, k + 1)] - uz[fzi(g, i, j, k)]) / g.h;
        div[idx] = d;
    }
}

// subGradPress on the water and the air face fields (air skipped when null)
template <class R>
__global__ void k_subgrad(Grid g, const R* __restrict__ p, float* wx, float* wy, float* wz, float* ax, float* ay, float* az,
                          float* __restrict__ pf) {
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    R hh = (R)g.h;
    MP_GRID_LOOP(t, tot) {
        int i, j, k;
        if (t < g.nfx) {
            int idx = (int)t; getijk3(idx, g.NY, g.NZ, i, j, k);
            if (i > 0 && i < g.NX) {
                R d = (p[cid(g, i, j, k)] - p[cid(g, i - 1, j, k)]) / hh;
                wx[idx] = (float)((R)wx[idx] - d); if (ax) ax[idx] = (float)((R)ax[idx] - d);
            }
        } else if (t < (long long)g.nfx + g.nfy) {
            int idx = (int)(t - g.nfx); getijk3(idx, g.NY + 1, g.NZ, i, j, k);
            if (j > 0 && j < g.NY) {
                R d = (p[cid(g, i, j, k)] - p[cid(g, i, j - 1, k)]) / hh;
                wy[idx] = (float)((R)wy[idx] - d); if (ay) ay[idx] = (float)((R)ay[idx] - d);
            }
        } else if (t < (long long)g.nfx + g.nfy + g.nfz) {
            int idx = (int)(t - g.nfx - g.nfy); getijk3(idx, g.NY, g.NZ + 1, i, j, k);
            if (k > 0 && k < g.NZ) {
                R d = (p[cid(g, i, j, k)] - p[cid(g, i, j, k - 1)]) / hh;
                wz[idx] = (float)((R)wz[idx] - d); if (az) az[idx] = (float)((R)az[idx] - d);
            }
        }
        if (pf && t < g.n) pf[t] = (float)p[t];
    }
}

// ---- ghost-fluid coefficients ---------------------------------------------------
// Face weights beta = 1/rho_face, densities rho_liquid = 1 and rho_air =
// 1/ratio. A face between two unknowns of one type takes that type's density;
// between a FLUID and an AIR cell, rho_face = theta rho_liquid + (1 - theta)
// rho_air with theta the liquid fraction of the segment between the centres
// (theta = -ls_L / (ls_G - ls_L) from the merged level set, the fraction the
// two-phase divergence uses, clamped to [0, 1]); a face with one unknown side
// takes that side's density; others 0.
__device__ __forceinline__ bool gfm_unknown(int m) { return m == MP_TYPEFLUID || m == MP_TYPEAIR; }
__global__ void k_gfm_beta(Grid g, const int8_t* __restrict__ mark, const float* __restrict__ ls, float rho_air,
                           float* __restrict__ bx, float* __restrict__ by, float* __restrict__ bz) {
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k, idx, ax;
        if (t < g.nfx) { idx = (int)t; getijk3(idx, g.NY, g.NZ, i, j, k); ax = 0; }
        else if (t < (long long)g.nfx + g.nfy) { idx = (int)(t - g.nfx); getijk3(idx, g.NY + 1, g.NZ, i, j, k); ax = 1; }
        else { idx = (int)(t - g.nfx - g.nfy); getijk3(idx, g.NY, g.NZ + 1, i, j, k); ax = 2; }
        const int e = ax == 0 ? i : (ax == 1 ? j : k), n = ax == 0 ? g.NX : (ax == 1 ? g.NY : g.NZ);
        float beta = 0.0f;
        if (e > 0 && e < n) {
            const int cb = cid(g, i, j, k), ca = cid(g, i - (ax == 0), j - (ax == 1), k - (ax == 2));
            const int ma = mark[ca], mb = mark[cb];
            const bool ua = gfm_unknown(ma), ub = gfm_unknown(mb);
            auto rho = [&](int m) { return m == MP_TYPEAIR ? rho_air : 1.0f; };
            if (ua && ub) {
                if (ma == mb) beta = 1.0f / rho(ma);
                else {
                    const int cl = ma == MP_TYPEFLUID ? ca : cb, cg = ma == MP_TYPEFLUID ? cb : ca;
                    const float ll = ls[cl], lg = ls[cg];
                    float th = (lg == ll) ? 0.5f : (0.0f - ll) / (lg - ll);
                    th = fminf(1.0f, fmaxf(0.0f, th));
                    beta = 1.0f / (th * 1.0f + (1.0f - th) * rho_air);
                }
            } else if (ua) beta = 1.0f / rho(ma);
            else if (ub) beta = 1.0f / rho(mb);
        }
        (ax == 0 ? bx : (ax == 1 ? by : bz))[idx] = beta;
    }
}
// S = diag^-1/2 on the unknowns (0 elsewhere) and bs = S b
template <class R>
__global__ void k_gfm_scale(Grid g, const int8_t* __restrict__ mark, const float* __restrict__ bx,
                            const float* __restrict__ by, const float* __restrict__ bz, const R* __restrict__ b,
                            float* __restrict__ S, R* __restrict__ bs) {
    const int sI = g.NY * g.NZ, sJ = g.NZ;
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, idx, i, j, k);
        float sc = 0.0f;
        if (gfm_unknown(mark[idx]) && inner(g, i, j, k)) {
            float d = 0.0f;
            if (mark[idx + sI] != MP_TYPEBOUNDARY) d += bx[fxi(g, i + 1, j, k)];
            if (mark[idx + sJ] != MP_TYPEBOUNDARY) d += by[fyi(g, i, j + 1, k)];
            if (mark[idx + 1] != MP_TYPEBOUNDARY) d += bz[fzi(g, i, j, k + 1)];
            if (mark[idx - sI] != MP_TYPEBOUNDARY) d += bx[fxi(g, i, j, k)];
            if (mark[idx - sJ] != MP_TYPEBOUNDARY) d += by[fyi(g, i, j, k)];
            if (mark[idx - 1] != MP_TYPEBOUNDARY) d += bz[fzi(g, i, j, k)];
            d /= g.h * g.h;
            sc = d > 0.0f ? 1.0f / sqrtf(d) : 0.0f;
        }
        S[idx] = sc;
        bs[idx] = (R)sc * b[idx];
    }
}
template <class R>
__global__ void k_gfm_unscale(int n, const float* __restrict__ S, R* __restrict__ x) {
    MP_GRID_LOOP(idx, n) x[idx] = (R)S[idx] * x[idx];
}
// u -= beta grad p on the interior faces of both velocity fields
template <class R>
__global__ void k_subgrad_gfm(Grid g, const R* __restrict__ p, const float* __restrict__ bx,
                              const float* __restrict__ by, const float* __restrict__ bz, float* wx, float* wy,
                              float* wz, float* ax, float* ay, float* az) {
    long long tot = (long long)g.nfx + g.nfy + g.nfz;
    MP_GRID_LOOP(t, tot) {
        int i, j, k;
        if (t < g.nfx) {
            int idx = (int)t; getijk3(idx, g.NY, g.NZ, i, j, k);
            if (i > 0 && i < g.NX) {
                const R d = (R)bx[idx] * (p[cid(g, i, j, k)] - p[cid(g, i - 1, j, k)]) / (R)g.h;
                wx[idx] = (float)((R)wx[idx] - d); ax[idx] = (float)((R)ax[idx] - d);
            }
        } else if (t < (long long)g.nfx + g.nfy) {
            int idx = (int)(t - g.nfx); getijk3(idx, g.NY + 1, g.NZ, i, j, k);
            if (j > 0 && j < g.NY) {
                const R d = (R)by[idx] * (p[cid(g, i, j, k)] - p[cid(g, i, j - 1, k)]) / (R)g.h;
                wy[idx] = (float)((R)wy[idx] - d); ay[idx] = (float)((R)ay[idx] - d);
            }
        } else {
            int idx = (int)(t - g.nfx - g.nfy); getijk3(idx, g.NY, g.NZ + 1, i, j, k);
            if (k > 0 && k < g.NZ) {
                const R d = (R)bz[idx] * (p[cid(g, i, j, k)] - p[cid(g, i, j, k - 1)]) / (R)g.h;
                wz[idx] = (float)((R)wz[idx] - d); az[idx] = (float)((R)az[idx] - d);
            }
        }
    }
}

// ---- heat grid ----------------------------------------------------------------
__global__ void k_heat_bottom(Grid g, float* __restrict__ Tp, float inc, float clampv) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float v = Tp[idx];
        if (i >= 1 && i < g.NX - 1 && j >= 1 && j < g.NY - 1 && k <= 3) v += inc;
        Tp[idx] = fminf(clampv, v);
    }
}
// Tp_save copy + compb_heat; with fixed heat the held value feeds the
// right-hand side (the dormant branch of compb_heat, spray_k.cu:4515-4519)
__global__ void k_heat_rhs(Grid g, const float* __restrict__ Tp, float* __restrict__ save, float* __restrict__ bo,
                           const int8_t* __restrict__ mark, const float* __restrict__ fixedheat, HeatOp op) {
    MP_GRID_LOOP(idx, g.n) {
        float t = Tp[idx];
        save[idx] = t;
        float al = op.al_of(mark[idx]);
        if (fixedheat && fixedheat[idx] != MP_UNDEF_TEMPERATURE) t = fixedheat[idx];
        bo[idx] = t * g.h * g.h / al / op.dt;
    }
}
// the same right-hand side in FP64 (the all-FP64 form)
__global__ void k_heat_rhs64(Grid g, const float* __restrict__ Tp, float* __restrict__ save, double* __restrict__ bo,
                             float* __restrict__ bof, const int8_t* __restrict__ mark,
                             const float* __restrict__ fixedheat, HeatOp op) {
    MP_GRID_LOOP(idx, g.n) {
        float t = Tp[idx];
        save[idx] = t;
        double al = op.al_of(mark[idx]);
        if (fixedheat && fixedheat[idx] != MP_UNDEF_TEMPERATURE) t = fixedheat[idx];
        const double b = (double)t * (double)g.h * (double)g.h / al / (double)op.dt;
        bo[idx] = b;
        bof[idx] = (float)b;
    }
}
__global__ void k_d2f(int n, const double* __restrict__ a, float* __restrict__ b) {
    MP_GRID_LOOP(idx, n) b[idx] = (float)a[idx];
}
__global__ void k_heat_bound(Grid g, const float* __restrict__ in, float* __restrict__ out) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float v = in[idx];
        if (i == g.NX - 1) v = in[cid(g, i - 1, j, k)];
        else if (i == 0) v = in[cid(g, i + 1, j, k)];
        else if (j == g.NY - 1) v = in[cid(g, i, j - 1, k)];
        else if (j == 0) v = in[cid(g, i, j + 1, k)];
        else if (k == g.NZ - 1) v = in[cid(g, i, j, k - 1)];
        else if (k == 0) v = in[cid(g, i, j, k + 1)];
        out[idx] = v;
    }
}
__global__ void k_tp_change(int n, const float* __restrict__ Tp, float* __restrict__ save, const int8_t* __restrict__ mark) {
    MP_GRID_LOOP(idx, n) save[idx] = (mark[idx] != MP_TYPEBOUNDARY) ? Tp[idx] - save[idx] : 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
static Red red_of(MpCtx* c) {
    return Red{c->red, c->red_count, c->scal, reinterpret_cast<unsigned int*>(c->red_count + 1)};
}

// Runs CG on x (zeroed here) for A x = b. Batches iterations between host
// checks of the device stop flag; launches after the stop exit at once.
template <class R, class Op>
static int run_cg(MpCtx* c, const Op& op, R* x, const R* b, R* r, R* p0, R* p1, int maxiter, int tolmode, float tol,
                  int true_every, int* iters_out, double* res_out, int kt_stencil) {
    int n = c->G.n;
    int nb = c->red_blocks;
    Red Rd = red_of(c);
    cudaStream_t s = c->stream;
    MP_CUDA(c, cudaMemsetAsync(x, 0, sizeof(R) * n, s));
    k_cg_init<R, Op><<<nb, CG_T, 0, s>>>(op, n, b, r, Rd, tolmode, tol);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    constexpr bool kGeneral = op_general<Op>::value;
    // neighbour bytes for the plane-marching kernels (mark_tmp is free scratch here)
    uint8_t* nb8 = reinterpret_cast<uint8_t*>(c->mark_tmp);
    if constexpr (!kGeneral) {
        k_nb8<Op><<<mp_blocks(n, 256), 256, 0, s>>>(op, n, nb8);
        c->launches++;
    }
    const Grid& gg = c->G;
    dim3 pmb(PM_X, PM_Y);
    int tiles = ((gg.NZ + PM_X - 1) / PM_X) * ((gg.NY + PM_Y - 1) / PM_Y);
    int chunk = std::max(4, (int)((gg.NX * (long long)tiles + 4095) / 4096));   // <= 4096 blocks (partials buffer)
    PmGeom pg{chunk};
    dim3 pmg((gg.NZ + PM_X - 1) / PM_X, (gg.NY + PM_Y - 1) / PM_Y, (gg.NX + chunk - 1) / chunk);
    if ((long long)pmg.x * pmg.y * pmg.z > 148LL * 32) { c->err = "cg: tiling exceeds partials buffer"; return MP_ERR_CAPACITY; }
    // FP32 vectors on a grid whose k-rows split into float4 groups take the
    // four-cells-per-thread kernels; they never write the direction vectors
    // outside the unknowns, so both start cleared
    constexpr bool kF32 = std::is_same<R, float>::value;
    auto al16 = [](const void* q) { return reinterpret_cast<uintptr_t>(q) % 16 == 0; };
    // TMA plane marching: FP32 vectors, NZ a multiple of 16 (the neighbour
    // bytes' row stride), 16-byte aligned vectors
    bool tma = kF32 && !kGeneral && c->cg_use_tma && gg.NZ % 16 == 0 && al16(x) && al16(r) && al16(p0) &&
               al16(p1) && tt_encoder() != nullptr;
    TtMaps tmaps[4];   // direction with p_old = p0 / p1, update with p = p1 / p0
    dim3 tgrid, tgrid0;          // update pass, direction pass
    int tchunk = 0, tchunk0 = 0;
    if constexpr (kF32 && !kGeneral) {
        if (tma) {
            tma = tt_encode(&tmaps[0].a, r, gg, 4, TT_HK, TT_HJ) && tt_encode(&tmaps[0].b, p0, gg, 4, TT_HK, TT_HJ) &&
                  tt_encode(&tmaps[0].nb, nb8, gg, 1, TT_K, TT_J);
            tmaps[1] = tmaps[0];
            tma = tma && tt_encode(&tmaps[1].b, p1, gg, 4, TT_HK, TT_HJ);
            tma = tma && tt_encode(&tmaps[2].a, p1, gg, 4, TT_HK, TT_HJ) && tt_encode(&tmaps[2].b, x, gg, 4, TT_K, TT_J) &&
                  tt_encode(&tmaps[2].c, r, gg, 4, TT_K, TT_J) && tt_encode(&tmaps[2].nb, nb8, gg, 1, TT_K, TT_J);
            tmaps[3] = tmaps[2];
            tma = tma && tt_encode(&tmaps[3].a, p0, gg, 4, TT_HK, TT_HJ);
        }
        if (tma) {
            // the (k, j) tiles of one chunk of planes run together (their halo
            // rows meet in L2); chunks sized for one wave of each pass's
            // resident CTAs per SM
            const int tk = (gg.NZ + TT_K - 1) / TT_K, tj = (gg.NY + TT_J - 1) / TT_J;
            auto chunk_for = [&](int ctas) {
                const int nch = std::max(1, (148 * ctas) / (tk * tj));
                return c->cg_tma_chunk > 0 ? c->cg_tma_chunk : std::max(4, (gg.NX + nch - 1) / nch);
            };
            tchunk0 = chunk_for(tt_ctas<0>());
            tchunk = chunk_for(tt_ctas<1>());
            tgrid0 = dim3(tk, tj, (gg.NX + tchunk0 - 1) / tchunk0);
            tgrid = dim3(tk, tj, (gg.NX + tchunk - 1) / tchunk);
            if ((long long)tgrid0.x * tgrid0.y * tgrid0.z > 148LL * 32 || (long long)tgrid.x * tgrid.y * tgrid.z > 148LL * 32)
                tma = false;   // the partial-sum slots
        }
        if (tma) {
            MP_CUDA(c, cudaFuncSetAttribute(k_cg_tma<Op, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)tt_smem_bytes<0>()));
            MP_CUDA(c, cudaFuncSetAttribute(k_cg_tma<Op, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)tt_smem_bytes<1>()));
        }
    }
    const bool v4 = kF32 && gg.NZ % 4 == 0;
    const int nbv = (int)std::min<long long>(c->red_blocks, ((long long)(n / 4) + CG_T - 1) / CG_T);
    if (v4) {
        MP_CUDA(c, cudaMemsetAsync(p0, 0, sizeof(R) * n, s));
        MP_CUDA(c, cudaMemsetAsync(p1, 0, sizeof(R) * n, s));
    }
    unsigned int hflag[F_COUNT] = {0, 0};
    MP_CUDA(c, cudaMemcpyAsync(hflag, Rd.flag, sizeof(hflag), cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    int it = 0, batch = 8;
    R* pa = p0; R* pb = p1;
    while (hflag[F_DONE] == DONE_RUN && it < maxiter) {
        int end = std::min(maxiter, it + batch);
        for (; it < end; it++) {
            bool tr = true_every > 0 && (it + 1) % true_every == 0;
            if constexpr (kGeneral) {
                {
                    KtScope kt(c, kt_stencil);
                    k_cg_dir<R, Op><<<nb, CG_T, 0, s>>>(op, n, r, pa, pb, Rd, it == 0 ? 1 : 0);
                }
                {
                    KtScope kt(c, MP_KT_CG_UPDATE);
                    k_cg_upd<R, Op><<<nb, CG_T, 0, s>>>(op, n, pb, x, r, Rd, it, maxiter, tr ? 1 : 0);
                }
            } else {
            if constexpr (kF32) {
                if (tma) {
                    const int d = (pa == p0) ? 0 : 1;   // p_old
                    {
                        KtScope kt(c, kt_stencil);
                        MP_CUDA(c, tt_launch(k_cg_tma<Op, 0>, tgrid0, TT_THREADS, tt_smem_bytes<0>(), s, op, tmaps[d],
                                             pb, (float*)nullptr, (float*)nullptr, Rd, tchunk0, it == 0 ? 1 : 0, it,
                                             maxiter, 0));
                    }
                    {
                        KtScope kt(c, MP_KT_CG_UPDATE);
                        MP_CUDA(c, tt_launch(k_cg_tma<Op, 1>, tgrid, TT_THREADS, tt_smem_bytes<1>(), s, op,
                                             tmaps[2 + d], (float*)nullptr, x, r, Rd, tchunk, 0, it, maxiter,
                                             tr ? 1 : 0));
                    }
                } else if (v4) {
                    {
                        KtScope kt(c, kt_stencil);
                        k_cg_v4<Op, 0><<<nbv, CG_T, 0, s>>>(op, nb8, r, pa, pb, nullptr, nullptr, Rd,
                                                            it == 0 ? 1 : 0, it, maxiter, 0);
                    }
                    {
                        KtScope kt(c, MP_KT_CG_UPDATE);
                        k_cg_v4<Op, 1><<<nbv, CG_T, 0, s>>>(op, nb8, pb, nullptr, nullptr, x, r, Rd, 0, it, maxiter,
                                                            tr ? 1 : 0);
                    }
                }
            }
            if (!v4 && !tma) {
                {
                    KtScope kt(c, kt_stencil);
                    k_cg_pm<R, Op, 0><<<pmg, pmb, 0, s>>>(op, pg, nb8, r, pa, pb, nullptr, nullptr, Rd,
                                                          it == 0 ? 1 : 0, it, maxiter, 0);
                }
                {
                    KtScope kt(c, MP_KT_CG_UPDATE);
                    k_cg_pm<R, Op, 1><<<pmg, pmb, 0, s>>>(op, pg, nb8, pb, nullptr, nullptr, x, r, Rd, 0, it, maxiter,
                                                          tr ? 1 : 0);
                }
            }
            }
            if (tr) k_cg_true<R, Op><<<nb, CG_T, 0, s>>>(op, n, b, x, r, Rd, it, maxiter);
            c->launches += tr ? 3 : 2;
            std::swap(pa, pb);
        }
        MP_CHECK_LAUNCH(c);
        MP_CUDA(c, cudaMemcpyAsync(hflag, Rd.flag, sizeof(hflag), cudaMemcpyDeviceToHost, s));
        MP_CUDA(c, cudaStreamSynchronize(s));
        if (batch < 64) batch *= 2;
    }
    double rr = 0;
    MP_CUDA(c, cudaMemcpyAsync(&rr, Rd.scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaMemcpyAsync(hflag, Rd.flag, sizeof(hflag), cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    *iters_out = (int)hflag[F_ITERS];
    *res_out = rr;
    c->work[MP_WC_CG_ITERS] += hflag[F_ITERS];
    if (hflag[F_DONE] == DONE_TIMEOUT) {
        MP_CUDA(c, cudaMemsetAsync(Rd.count, 0, sizeof(unsigned int), s));
        c->err = "cg: a TMA tile wait ran out of time";
        return MP_ERR_TIMEOUT;
    }
    return hflag[F_DONE] == DONE_CAP ? MP_ERR_NOCONVERGE : MP_OK;
}

// Mixed-precision iterative refinement of A x = b: x and the true residual
// r = b - A x live in FP64 (x64, r64) and the residual is recomputed in FP64
// after every correction; each correction e solves A e = r with FP32 vectors
// (run_cg, relative tolerance inner_tol) and is added to x in FP64. The stop
// rule (tolmode, tol) is tested on the FP64 true residual, so the solution's
// accuracy is not bounded by FP32 storage of x. r32 and e32 are FP32 scratch.
template <class Op>
static int run_cg_refined(MpCtx* c, const Op& op, double* x64, const double* b64, double* r64, float* r32,
                          float* e32, int maxiter, int tolmode, float tol, float inner_tol, int* iters_out,
                          double* res_out) {
    const int n = c->G.n;
    cudaStream_t s = c->stream;
    Red Rd = red_of(c);
    MP_CUDA(c, cudaMemsetAsync(x64, 0, sizeof(double) * n, s));
    auto resid = [&](double* rr) -> int {
        k_cg_resid64<Op><<<c->red_blocks, CG_T, 0, s>>>(op, n, b64, x64, r64, r32, Rd, S_TRUE);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        MP_CUDA(c, cudaMemcpyAsync(rr, Rd.scal + S_TRUE, sizeof(double), cudaMemcpyDeviceToHost, s));
        MP_CUDA(c, cudaStreamSynchronize(s));
        return MP_OK;
    };
    double rr0 = 0, rr = 0;
    MP_TRY(resid(&rr0));
    rr = rr0;
    const double eps = tolmode == MP_TOL_REF_ABS ? (double)(tol * (float)n) : (double)tol * (double)tol * rr0;
    int total = 0;
    while (!(rr < eps) && total < maxiter && rr0 > 0) {
        int it = 0; double ri = 0;
        int rc = run_cg<float>(c, op, e32, r32, c->cg_r, c->cg_p, c->cg_z, maxiter - total, MP_TOL_REL, inner_tol, 0,
                               &it, &ri, MP_KT_CG_STENCIL);
        if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
        total += it;
        if (it == 0) break;
        k_add_f2d<<<mp_blocks(n, 256), 256, 0, s>>>(n, e32, x64);
        c->launches++;
        MP_TRY(resid(&rr));
    }
    *iters_out = total;
    *res_out = rr;
    return (rr < eps || rr0 == 0) ? MP_OK : MP_ERR_NOCONVERGE;
}

// The pressure matrix of project_CG_bubble for a given mark field, solved on
// the context's CG scratch (FP32 vectors: cg_r/cg_p/cg_z; FP64: the last
// three fifths of cg64). x is cleared first. Used by the adjoint module.
int k_cg_solve(MpCtx* c, const int8_t* mark, float* x, const float* b, int maxiter, int tolmode, float tol, int* iters,
               double* res) {
    PressOp op = press_op(c->G, mark);
    return run_cg<float>(c, op, x, b, c->cg_r, c->cg_p, c->cg_z, maxiter, tolmode, tol, 0, iters, res,
                         MP_KT_CG_STENCIL);
}
int k_cg_solve(MpCtx* c, const int8_t* mark, double* x, const double* b, int maxiter, int tolmode, float tol,
               int* iters, double* res) {
    PressOp op = press_op(c->G, mark);
    const size_t n = (size_t)c->G.n;
    return run_cg<double>(c, op, x, b, c->cg64 + 2 * n, c->cg64 + 3 * n, c->cg64 + 4 * n, maxiter, tolmode, tol, 0,
                          iters, res, MP_KT_CG_STENCIL);
}

// The heat matrix of updateTemperature for a given mark field (the adjoint's
// replay and transposed solve; boiling scenes, whose VACUUM cells make the
// matrix unsymmetric, are not differentiated), on the context's CG scratch.
static HeatOp heat_op(MpCtx* c, const int8_t* mark) {
    const mp_params& P = c->P;
    HeatOp op;
    op.g = c->G; op.mark = mark; op.dt = P.dt;
    op.alpha[MP_TYPEFLUID] = P.heatalpha_fluid; op.alpha[MP_TYPEAIR] = P.heatalpha_air;
    op.alpha[MP_TYPEVACUUM] = P.heatalpha_vacuum; op.alpha[MP_TYPESOLID] = P.heatalpha_solid;
    op.alpha[MP_TYPEAIRSOLO] = P.heatalpha_air; op.alpha[MP_TYPEBOUNDARY] = 0;
    op.boil = 0;
    return op;
}
int k_heat_cg_solve(MpCtx* c, const int8_t* mark, float* x, const float* b, int maxiter, int tolmode, float tol,
                    int* iters, double* res) {
    return run_cg<float>(c, heat_op(c, mark), x, b, c->cg_r, c->cg_p, c->cg_z, maxiter, tolmode, tol, 0, iters, res,
                         MP_KT_CG_STENCIL);
}
int k_heat_cg_solve(MpCtx* c, const int8_t* mark, double* x, const double* b, int maxiter, int tolmode, float tol,
                    int* iters, double* res) {
    const size_t n = (size_t)c->G.n;
    return run_cg<double>(c, heat_op(c, mark), x, b, c->cg64 + 2 * n, c->cg64 + 3 * n, c->cg64 + 4 * n, maxiter,
                          tolmode, tol, 0, iters, res, MP_KT_CG_STENCIL);
}

// project_CG_bubble (spray.cu:1590-1611)
int k_project(MpCtx* c, int* iters, double* res) {
    const Grid& g = c->G;
    PressOp op = press_op(g, c->mark);
    int nbk = mp_blocks(g.n, 256);
    long long ftot = (long long)g.nfx + g.nfy + g.nfz;
    long long gtot = std::max(ftot, (long long)g.n);
    int it = 0; double rr = 0; int rc;
    if (c->P.coef_mode == MP_COEF_GFM) {
        // ghost-fluid variable density (FP32 vectors, FP64 dots); the scaled
        // right-hand side lives in cell_tmp, free during the projection
        if (!c->gfm_beta) {
            MP_CUDA(c, cudaMalloc((void**)&c->gfm_beta, sizeof(float) * (size_t)ftot));
            MP_CUDA(c, cudaMalloc((void**)&c->gfm_s, sizeof(float) * (size_t)g.n));
        }
        float* bx = c->gfm_beta; float* by = bx + g.nfx; float* bz = by + g.nfy;
        float* x = c->press;
        if (c->P.precision != MP_PREC_FP64 && !(c->P.cg_refine_tol > 0))
            k_divergence<float><<<nbk, 256, 0, c->stream>>>(g, c->mark, c->lsmerge, c->wu[0], c->wu[1], c->wu[2],
                                                            c->au[0], c->au[1], c->au[2], c->divg, nullptr);
        k_gfm_beta<<<mp_blocks(ftot, 256), 256, 0, c->stream>>>(g, c->mark, c->lsmerge, 1.0f / c->P.density_ratio,
                                                                bx, by, bz);
        GfmOp gop{g, c->mark, bx, by, bz, c->gfm_s};
        if (c->P.precision == MP_PREC_MIXED && c->P.cg_refine_tol > 0) {
            // mixed-precision refinement of the scaled system
            double* x64 = c->cg64; double* b64 = x64 + g.n; double* r64 = b64 + g.n;
            k_divergence<double><<<nbk, 256, 0, c->stream>>>(g, c->mark, c->lsmerge, c->wu[0], c->wu[1], c->wu[2],
                                                             c->au[0], c->au[1], c->au[2], b64, c->divg);
            k_gfm_scale<double><<<nbk, 256, 0, c->stream>>>(g, c->mark, bx, by, bz, b64, c->gfm_s, b64);
            c->launches += 3;
            MP_CHECK_LAUNCH(c);
            rc = run_cg_refined(c, gop, x64, b64, r64, c->cell_tmp, x, c->P.cg_max_iter, c->P.cg_tol_mode,
                                c->P.cg_tol, c->P.cg_refine_tol, &it, &rr);
            if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
            k_gfm_unscale<double><<<nbk, 256, 0, c->stream>>>(g.n, c->gfm_s, x64);
            k_d2f<<<nbk, 256, 0, c->stream>>>(g.n, x64, x);
            k_subgrad_gfm<double><<<mp_blocks(ftot, 256), 256, 0, c->stream>>>(g, x64, bx, by, bz, c->wu[0], c->wu[1],
                                                                               c->wu[2], c->au[0], c->au[1], c->au[2]);
            c->launches += 3;
        } else if (c->P.precision == MP_PREC_FP64) {
            // the all-FP64 form: right-hand side, vectors and scalars in FP64
            double* xd = c->cg64; double* bd = xd + g.n; double* rd = bd + g.n;
            double* p0 = rd + g.n; double* p1 = p0 + g.n;
            k_divergence<double><<<nbk, 256, 0, c->stream>>>(g, c->mark, c->lsmerge, c->wu[0], c->wu[1], c->wu[2],
                                                             c->au[0], c->au[1], c->au[2], bd, c->divg);
            k_gfm_scale<double><<<nbk, 256, 0, c->stream>>>(g, c->mark, bx, by, bz, bd, c->gfm_s, bd);
            c->launches += 3;
            MP_CHECK_LAUNCH(c);
            rc = run_cg<double>(c, gop, xd, bd, rd, p0, p1, c->P.cg_max_iter, c->P.cg_tol_mode, c->P.cg_tol, 0, &it,
                                &rr, MP_KT_CG_STENCIL);
            if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
            k_gfm_unscale<double><<<nbk, 256, 0, c->stream>>>(g.n, c->gfm_s, xd);
            k_d2f<<<nbk, 256, 0, c->stream>>>(g.n, xd, x);
            k_subgrad_gfm<double><<<mp_blocks(ftot, 256), 256, 0, c->stream>>>(g, xd, bx, by, bz, c->wu[0], c->wu[1],
                                                                               c->wu[2], c->au[0], c->au[1], c->au[2]);
            c->launches += 3;
        } else {
            k_gfm_scale<float><<<nbk, 256, 0, c->stream>>>(g, c->mark, bx, by, bz, c->divg, c->gfm_s, c->cell_tmp);
            c->launches += 3;
            MP_CHECK_LAUNCH(c);
            rc = run_cg<float>(c, gop, x, c->cell_tmp, c->cg_r, c->cg_p, c->cg_z, c->P.cg_max_iter, c->P.cg_tol_mode,
                               c->P.cg_tol, 0, &it, &rr, MP_KT_CG_STENCIL);
            if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
            k_gfm_unscale<float><<<nbk, 256, 0, c->stream>>>(g.n, c->gfm_s, x);
            k_subgrad_gfm<float><<<mp_blocks(ftot, 256), 256, 0, c->stream>>>(g, x, bx, by, bz, c->wu[0], c->wu[1],
                                                                              c->wu[2], c->au[0], c->au[1], c->au[2]);
            c->launches += 2;
        }
    } else if (c->P.precision == MP_PREC_FP64) {
        double* x = c->cg64;
        double* b = x + g.n; double* r = b + g.n; double* p0 = r + g.n; double* p1 = p0 + g.n;
        k_divergence<double><<<nbk, 256, 0, c->stream>>>(g, c->mark, c->lsmerge, c->wu[0], c->wu[1], c->wu[2],
                                                         c->au[0], c->au[1], c->au[2], b, c->divg);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        rc = run_cg<double>(c, op, x, b, r, p0, p1, c->P.cg_max_iter, c->P.cg_tol_mode, c->P.cg_tol,
                            c->P.cg_true_residual_every, &it, &rr, MP_KT_CG_STENCIL);
        if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
        k_subgrad<double><<<mp_blocks(gtot, 256), 256, 0, c->stream>>>(g, x, c->wu[0], c->wu[1], c->wu[2], c->au[0],
                                                                       c->au[1], c->au[2], c->press);
    } else if (c->P.cg_refine_tol > 0) {
        // mixed-precision refinement: FP64 right-hand side, solution and true
        // residual; FP32-vector corrections
        double* x64 = c->cg64; double* b64 = x64 + g.n; double* r64 = b64 + g.n;
        k_divergence<double><<<nbk, 256, 0, c->stream>>>(g, c->mark, c->lsmerge, c->wu[0], c->wu[1], c->wu[2],
                                                         c->au[0], c->au[1], c->au[2], b64, c->divg);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        rc = run_cg_refined(c, op, x64, b64, r64, c->cell_tmp, c->press, c->P.cg_max_iter, c->P.cg_tol_mode,
                            c->P.cg_tol, c->P.cg_refine_tol, &it, &rr);
        if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
        k_subgrad<double><<<mp_blocks(gtot, 256), 256, 0, c->stream>>>(g, x64, c->wu[0], c->wu[1], c->wu[2], c->au[0],
                                                                       c->au[1], c->au[2], c->press);
    } else {
        float* x = c->press;
        k_divergence<float><<<nbk, 256, 0, c->stream>>>(g, c->mark, c->lsmerge, c->wu[0], c->wu[1], c->wu[2],
                                                        c->au[0], c->au[1], c->au[2], c->divg, nullptr);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        rc = run_cg<float>(c, op, x, c->divg, c->cg_r, c->cg_p, c->cg_z, c->P.cg_max_iter, c->P.cg_tol_mode,
                           c->P.cg_tol, c->P.cg_true_residual_every, &it, &rr, MP_KT_CG_STENCIL);
        if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
        k_subgrad<float><<<mp_blocks(ftot, 256), 256, 0, c->stream>>>(g, x, c->wu[0], c->wu[1], c->wu[2], c->au[0],
                                                                      c->au[1], c->au[2], nullptr);
    }
    c->launches++;
    MP_CHECK_LAUNCH(c);
    c->S.last_cg_iters = it;
    c->S.last_cg_residual = rr;
    if (iters) *iters = it;
    if (res) *res = rr;
    return rc;
}

// project_CG (spray.cu:241-271): the single-phase projection of the water
// mode (FP32 vectors, FP64 dots, as the reference projection's mixed form)
int k_project_water(MpCtx* c, int* iters, double* res) {
    const Grid& g = c->G;
    if (c->P.precision != MP_PREC_MIXED || c->P.coef_mode != MP_COEF_REF) {
        c->err = "project_water: the single-phase solve is MP_PREC_MIXED, MP_COEF_REF only";
        return MP_ERR_STATE;
    }
    PressOp op = press_op(g, c->mark, false);
    long long ftot = (long long)g.nfx + g.nfy + g.nfz;
    k_divergence_water<<<mp_blocks(g.n, 256), 256, 0, c->stream>>>(g, c->mark, c->wu[0], c->wu[1], c->wu[2], c->divg);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    int it = 0; double rr = 0;
    int rc = run_cg<float>(c, op, c->press, c->divg, c->cg_r, c->cg_p, c->cg_z, c->P.cg_max_iter, c->P.cg_tol_mode,
                           c->P.cg_tol, c->P.cg_true_residual_every, &it, &rr, MP_KT_CG_STENCIL);
    if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
    k_subgrad<float><<<mp_blocks(ftot, 256), 256, 0, c->stream>>>(g, c->press, c->wu[0], c->wu[1], c->wu[2], nullptr,
                                                                  nullptr, nullptr, nullptr);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    c->S.last_cg_iters = it;
    c->S.last_cg_residual = rr;
    if (iters) *iters = it;
    if (res) *res = rr;
    return rc;
}

int k_heat_p2g_launch(MpCtx* c);
int k_heat_g2p_launch(MpCtx* c);
int k_latent_heat(MpCtx* c);

// updateTemperature (spray.cu:1889-1947)
// compb_heat, solver_cg_heat and setBoundaryHeat (spray.cu:1780-1852): the
// implicit diffusion of Tp, Tp_save keeping the field before it
static int heat_solve(MpCtx* c) {
    const Grid& g = c->G;
    const mp_params& P = c->P;
    int nb = mp_blocks(g.n, 256);
    HeatOp op;
    op.g = g; op.mark = c->mark; op.dt = P.dt;
    op.alpha[MP_TYPEFLUID] = P.heatalpha_fluid; op.alpha[MP_TYPEAIR] = P.heatalpha_air;
    op.alpha[MP_TYPEVACUUM] = P.heatalpha_vacuum; op.alpha[MP_TYPESOLID] = P.heatalpha_solid;
    op.alpha[MP_TYPEAIRSOLO] = P.heatalpha_air; op.alpha[MP_TYPEBOUNDARY] = 0;
    int sc = P.scene;
    op.boil = (sc == MP_SCENE_BOILING || sc == MP_SCENE_BOILING_HIGHRES || sc == MP_SCENE_MELTANDBOIL ||
               sc == MP_SCENE_MELTANDBOIL_HIGHRES || sc == MP_SCENE_ALL) ? 1 : 0;
    int it = 0; double rr = 0;
    int rc;
    if (P.precision == MP_PREC_FP64) {
        // the all-FP64 form: right-hand side, vectors and scalars in FP64
        double* xd = c->cg64; double* bd = xd + g.n;
        double* rd = bd + g.n; double* p0 = rd + g.n; double* p1 = p0 + g.n;
        k_heat_rhs64<<<nb, 256, 0, c->stream>>>(g, c->Tp, c->Tp_save, bd, c->Tp_old, c->mark,
                                                P.b_fixed_heat ? c->fixedheat : nullptr, op);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        rc = run_cg<double>(c, op, xd, bd, rd, p0, p1, P.heat_cg_max_iter, MP_TOL_REF_ABS, 0.01f, 0, &it, &rr,
                            MP_KT_CG_STENCIL);
        if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
        k_d2f<<<nb, 256, 0, c->stream>>>(g.n, xd, c->Tp);
        c->launches++;
    } else {
        k_heat_rhs<<<nb, 256, 0, c->stream>>>(g, c->Tp, c->Tp_save, c->Tp_old, c->mark,
                                              P.b_fixed_heat ? c->fixedheat : nullptr, op);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        rc = run_cg<float>(c, op, c->Tp, c->Tp_old, c->cg_r, c->cg_p, c->cg_z, P.heat_cg_max_iter, MP_TOL_REF_ABS,
                           0.01f, 0, &it, &rr, MP_KT_CG_STENCIL);
        if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
    }
    c->S.last_heat_cg_iters = it;
    c->S.last_heat_cg_residual = rr;
    if (P.b_extend_heat_to_boundary) {
        k_heat_bound<<<nb, 256, 0, c->stream>>>(g, c->Tp, c->cell_tmp);
        c->launches++;
        std::swap(c->Tp, c->cell_tmp);
    }
    MP_CHECK_LAUNCH(c);
    return rc;
}

int k_heat(MpCtx* c) {
    const Grid& g = c->G;
    const mp_params& P = c->P;
    int nb = mp_blocks(g.n, 256);
    MP_TRY(k_heat_p2g_launch(c));
    if (P.b_add_heat_bottom) {
        k_heat_bottom<<<nb, 256, 0, c->stream>>>(g, c->Tp, P.heat_increase_bottom, P.heat_clamp);
        c->launches++;
    }
    const int rc = heat_solve(c);
    if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
    k_tp_change<<<nb, 256, 0, c->stream>>>(g.n, c->Tp, c->Tp_save, c->mark);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_TRY(k_heat_g2p_launch(c));
    MP_TRY(k_latent_heat(c));
    return rc;
}

// heatsim (spray.cu:1959-1987): the grid-only heat step of SIMULATION_HEATONLY
int k_heatsim(MpCtx* c) {
    const int rc = heat_solve(c);
    if (rc != MP_OK && rc != MP_ERR_NOCONVERGE) return rc;
    c->S.frame++;
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return rc;
}

namespace {
// initheat_grid_k (spray_k.cu:5603-5621) then markBoundaryCell: in each
// xz-section, a hot SOLID disc (100) and a cold FLUID disc (0) of radius
// 0.15 NX, VACUUM (20) below NZ/2 and AIR (80) above
__global__ void k_init_heat_grid(Grid g, float* __restrict__ tp, int8_t* __restrict__ mark) {
    MP_GRID_LOOP(idx, g.n) {
        int i, j, k; getijk(g, (int)idx, i, j, k);
        float x = (float)i, z = (float)k;
        const float r = (float)(g.NX * 0.15);
        float a = x - (float)(g.NX / 4), b = z - (float)(g.NZ / 4);
        float a2 = x - (float)(g.NX / 4 * 3), b2 = z - (float)(g.NZ / 4 * 3);
        if (sqrtf(a * a + b * b) <= r) { tp[idx] = 100; mark[idx] = MP_TYPESOLID; }
        else if (sqrtf(a2 * a2 + b2 * b2) <= r) { tp[idx] = 0; mark[idx] = MP_TYPEFLUID; }
        else if (z < (float)(g.NZ / 2)) { tp[idx] = 20; mark[idx] = MP_TYPEVACUUM; }
        else { tp[idx] = 80; mark[idx] = MP_TYPEAIR; }
        if (i == 0 || i == g.NX - 1 || j == 0 || j == g.NY - 1 || k == 0 || k == g.NZ - 1) mark[idx] = MP_TYPEBOUNDARY;
    }
}
}  // namespace

int k_init_heat_grid_launch(MpCtx* c) {
    k_init_heat_grid<<<mp_blocks(c->G.n, 256), 256, 0, c->stream>>>(c->G, c->Tp, c->mark);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    return MP_OK;
}

// ---------------------------------------------------------------------------
// Pressure CG without allocation (mp_pressure_cg_static)
// ---------------------------------------------------------------------------
// For callers that may not allocate device memory: the solve of mp_project on
// caller-owned arrays, with every working vector in one fixed array that this
// library holds on each GPU it is loaded on, for the life of the process.
// Layout of the array (byte offsets, each part 256-byte aligned).
namespace {
constexpr int NA_MAX_CELLS = 64 * 64 * 64;                 // 262,144 cells
constexpr int NA_MAX_BLOCKS = 148 * 32;                    // = the partial sums of mp_blocks()
constexpr size_t na_up(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t NA_PART = 0;                                            // double[NA_MAX_BLOCKS]
constexpr size_t NA_SCAL = na_up(NA_PART + sizeof(double) * NA_MAX_BLOCKS);   // double[8]
constexpr size_t NA_COUNT = na_up(NA_SCAL + sizeof(double) * 8);         // uint32: counter, flags
constexpr size_t NA_COUNT_BYTES = 64;
constexpr size_t NA_NB8 = na_up(NA_COUNT + NA_COUNT_BYTES);             // uint8[cells]
constexpr size_t NA_R = na_up(NA_NB8 + NA_MAX_CELLS);                   // float[cells] x 3
constexpr size_t NA_P0 = na_up(NA_R + sizeof(float) * NA_MAX_CELLS);
constexpr size_t NA_P1 = na_up(NA_P0 + sizeof(float) * NA_MAX_CELLS);
constexpr size_t NA_BYTES = na_up(NA_P1 + sizeof(float) * NA_MAX_CELLS);   // about 3.3 MB
}  // namespace

// The scratch itself. In host code this name is only a stand-in for the
// device symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char mp_cg_static_scratch[NA_BYTES];

void mp_internal_set_global_error(const char* msg);

namespace {
// Device address of the scratch in the current device's context. It is looked
// up on every call: cudaGetSymbolAddress allocates nothing, and an address
// kept from an earlier call would belong to a context that cudaDeviceReset or
// a caller's own driver-API context may have replaced since.
cudaError_t na_scratch(unsigned char** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, mp_cg_static_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}
}  // namespace

extern "C" int mp_pressure_cg_static(int nx, int ny, int nz, float cellsize, const int8_t* mark,
                                     const float* divergence, float* pressure, int max_iter, int tol_mode, float tol,
                                     void* stream, int* iters, double* residual) {
    auto fail = [](int rc, const std::string& msg) { mp_internal_set_global_error(msg.c_str()); return rc; };
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        return fail(MP_ERR_CUDA, std::string("mp_pressure_cg_static: ") + what + ": " + cudaGetErrorString(e));
    };
    if (nx < 3 || ny < 3 || nz < 3 || !(cellsize > 0) || !mark || !divergence || !pressure || max_iter < 0 ||
        (tol_mode != MP_TOL_REF_ABS && tol_mode != MP_TOL_REL))
        return fail(MP_ERR_ARG, "mp_pressure_cg_static: bad grid, pointer, iteration cap or tolerance mode");
    const long long nll = (long long)nx * ny * nz;
    if (nll > NA_MAX_CELLS)
        return fail(MP_ERR_CAPACITY, "mp_pressure_cg_static: " + std::to_string(nll) + " cells exceed the " +
                                         std::to_string(NA_MAX_CELLS) + "-cell limit of its fixed scratch");
    const int n = (int)nll;
    const int nb = mp_blocks(n, 256);
    const bool v4 = nz % 4 == 0 && reinterpret_cast<uintptr_t>(divergence) % 16 == 0 &&
                    reinterpret_cast<uintptr_t>(pressure) % 16 == 0;
    const int nbv = (int)std::min<long long>(nb, ((long long)(n / 4) + CG_T - 1) / CG_T);
    dim3 pmb(PM_X, PM_Y);
    int tiles = ((nz + PM_X - 1) / PM_X) * ((ny + PM_Y - 1) / PM_Y);
    int chunk = std::max(4, (int)((nx * (long long)tiles + 4095) / 4096));
    PmGeom pg{chunk};
    dim3 pmg((nz + PM_X - 1) / PM_X, (ny + PM_Y - 1) / PM_Y, (nx + chunk - 1) / chunk);
    if ((long long)pmg.x * pmg.y * pmg.z > NA_MAX_BLOCKS || nb > NA_MAX_BLOCKS)
        return fail(MP_ERR_CAPACITY, "mp_pressure_cg_static: launch tiling exceeds the fixed partial-sum slots");

    unsigned char* base = nullptr;
    cudaError_t e = na_scratch(&base);
    if (e != cudaSuccess) return cuda_fail(e, "scratch address");
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Grid g{};
    g.NX = nx; g.NY = ny; g.NZ = nz; g.n = n;
    g.nfx = (nx + 1) * ny * nz; g.nfy = nx * (ny + 1) * nz; g.nfz = nx * ny * (nz + 1);
    g.h = cellsize;
    PressOp op = press_op(g, mark);
    Red Rd{reinterpret_cast<double*>(base + NA_PART), reinterpret_cast<unsigned int*>(base + NA_COUNT),
           reinterpret_cast<double*>(base + NA_SCAL), reinterpret_cast<unsigned int*>(base + NA_COUNT) + 1};
    uint8_t* nb8 = base + NA_NB8;
    float* r = reinterpret_cast<float*>(base + NA_R);
    float* pa = reinterpret_cast<float*>(base + NA_P0);
    float* pb = reinterpret_cast<float*>(base + NA_P1);

    // the scratch keeps the previous call's contents: clear the block counter,
    // the stop flags, the direction vectors and the solution
    if ((e = cudaMemsetAsync(base + NA_COUNT, 0, NA_COUNT_BYTES, s)) != cudaSuccess) return cuda_fail(e, "clear");
    if ((e = cudaMemsetAsync(pa, 0, sizeof(float) * n, s)) != cudaSuccess) return cuda_fail(e, "clear");
    if ((e = cudaMemsetAsync(pb, 0, sizeof(float) * n, s)) != cudaSuccess) return cuda_fail(e, "clear");
    if ((e = cudaMemsetAsync(pressure, 0, sizeof(float) * n, s)) != cudaSuccess) return cuda_fail(e, "clear");

    k_cg_init<float, PressOp><<<nb, CG_T, 0, s>>>(op, n, divergence, r, Rd, tol_mode, tol);
    k_nb8<PressOp><<<mp_blocks(n, 256), 256, 0, s>>>(op, n, nb8);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "launch");
    unsigned int hflag[F_COUNT] = {0, 0};
    if ((e = cudaMemcpyAsync(hflag, Rd.flag, sizeof(hflag), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(e, "stop flag");
    int it = 0, batch = 8;
    while (hflag[F_DONE] == DONE_RUN && it < max_iter) {
        int end = std::min(max_iter, it + batch);
        for (; it < end; it++) {
            if (v4) {
                k_cg_v4<PressOp, 0><<<nbv, CG_T, 0, s>>>(op, nb8, r, pa, pb, nullptr, nullptr, Rd, it == 0 ? 1 : 0,
                                                         it, max_iter, 0);
                k_cg_v4<PressOp, 1><<<nbv, CG_T, 0, s>>>(op, nb8, pb, nullptr, nullptr, pressure, r, Rd, 0, it,
                                                         max_iter, 0);
            } else {
                k_cg_pm<float, PressOp, 0><<<pmg, pmb, 0, s>>>(op, pg, nb8, r, pa, pb, nullptr, nullptr, Rd,
                                                               it == 0 ? 1 : 0, it, max_iter, 0);
                k_cg_pm<float, PressOp, 1><<<pmg, pmb, 0, s>>>(op, pg, nb8, pb, nullptr, nullptr, pressure, r, Rd, 0,
                                                               it, max_iter, 0);
            }
            std::swap(pa, pb);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "launch");
        if ((e = cudaMemcpyAsync(hflag, Rd.flag, sizeof(hflag), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail(e, "stop flag");
        if (batch < 64) batch *= 2;
    }
    double rr = 0;
    if ((e = cudaMemcpyAsync(&rr, Rd.scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hflag, Rd.flag, sizeof(hflag), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(e, "result");
    if (iters) *iters = (int)hflag[F_ITERS];
    if (residual) *residual = rr;
    return hflag[F_DONE] == DONE_CAP ? MP_ERR_NOCONVERGE : MP_OK;
}
