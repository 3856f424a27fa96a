// k_sort.cu — particle spatial hashing as a stable per-cell counting sort,
// device-wide exclusive scan, particle packing.
//
// Replaces cspray::hashAndSortParticles (Multiphase/Multiphase/spray.cu:614-637):
// calcHashD (spray_k.cu:1010-1028), thrust::sort_by_key (spray_thrust.cu:12-17)
// and reorderDataAndFindCellStartD (spray_k.cu:1052-1129). Thrust's sort is
// stable, so within a cell particles keep ascending pre-sort index; this file
// reproduces that order exactly:
//   1. key = cell id, count per cell (atomics)         k_hash_count
//   2. exclusive scan of counts -> CSR offsets         mp_scan_u32
//   3. scatter particle indices into their cell slot    k_scatter (unordered)
//   4. sort each cell's slot range by particle index    k_segsort (+ type mask)
//   5. gather the three float4 particle streams         k_reorder
// The scan is also used for the deletion compaction and marching cubes
// (the reference's ThrustScanWrapper, spray_thrust.cu:19-24).
#include "ctx.cuh"

using namespace mpk;

// ---------------------------------------------------------------------------
// exclusive scan of uint32, out[n] = total. Tiles of 4096 = 256 threads x 16.
// ---------------------------------------------------------------------------
namespace {
constexpr int SCAN_T = 256, SCAN_I = 16, SCAN_TILE = SCAN_T * SCAN_I;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ void load16(const uint32_t* in, size_t n, size_t base, uint32_t v[SCAN_I]) {
    if (base + SCAN_I <= n && ((reinterpret_cast<uintptr_t>(in + base) & 15) == 0)) {
        const uint4* q = reinterpret_cast<const uint4*>(in + base);
        #pragma unroll
        for (int r = 0; r < 4; r++) {
            uint4 w = __ldg(q + r);
            v[4 * r] = w.x; v[4 * r + 1] = w.y; v[4 * r + 2] = w.z; v[4 * r + 3] = w.w;
        }
    } else {
        #pragma unroll
        for (int r = 0; r < SCAN_I; r++) v[r] = (base + r < n) ? in[base + r] : 0u;
    }
}

__global__ void __launch_bounds__(SCAN_T) k_scan_reduce(const uint32_t* __restrict__ in, size_t n, uint32_t* __restrict__ part) {
    __shared__ uint32_t ws[SCAN_T / 32];
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_I;
    uint32_t v[SCAN_I];
    load16(in, n, base, v);
    uint32_t s = 0;
    #pragma unroll
    for (int r = 0; r < SCAN_I; r++) s += v[r];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < SCAN_T / 32; w++) t += ws[w];
        part[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(SCAN_T) k_scan_down(const uint32_t* __restrict__ in, size_t n, const uint32_t* __restrict__ toff,
                                                      uint32_t* __restrict__ out) {
    __shared__ uint32_t ws[SCAN_T / 32];
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_I;
    uint32_t v[SCAN_I];
    load16(in, n, base, v);
    uint32_t s = 0;
    #pragma unroll
    for (int r = 0; r < SCAN_I; r++) s += v[r];
    uint32_t inc = warp_incl_scan(s);
    if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = inc;
    __syncthreads();
    uint32_t wofs = 0;
    for (int w = 0; w < (int)(threadIdx.x >> 5); w++) wofs += ws[w];
    uint32_t run = toff[blockIdx.x] + wofs + inc - s;
    uint32_t o[SCAN_I];
    #pragma unroll
    for (int r = 0; r < SCAN_I; r++) { o[r] = run; run += v[r]; }
    if (base + SCAN_I <= n && ((reinterpret_cast<uintptr_t>(out + base) & 15) == 0)) {
        uint4* q = reinterpret_cast<uint4*>(out + base);
        #pragma unroll
        for (int r = 0; r < 4; r++) q[r] = make_uint4(o[4 * r], o[4 * r + 1], o[4 * r + 2], o[4 * r + 3]);
    } else {
        #pragma unroll
        for (int r = 0; r < SCAN_I; r++) if (base + r < n) out[base + r] = o[r];
    }
}

__global__ void k_scan_single(const uint32_t* __restrict__ in, size_t n, uint32_t* __restrict__ out) {
    // one block, n <= SCAN_TILE
    __shared__ uint32_t ws[SCAN_T / 32];
    size_t base = (size_t)threadIdx.x * SCAN_I;
    uint32_t v[SCAN_I];
    #pragma unroll
    for (int r = 0; r < SCAN_I; r++) v[r] = (base + r < n) ? in[base + r] : 0u;
    uint32_t s = 0;
    #pragma unroll
    for (int r = 0; r < SCAN_I; r++) s += v[r];
    uint32_t inc = warp_incl_scan(s);
    if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = inc;
    __syncthreads();
    uint32_t wofs = 0;
    for (int w = 0; w < (int)(threadIdx.x >> 5); w++) wofs += ws[w];
    uint32_t run = wofs + inc - s;
    #pragma unroll
    for (int r = 0; r < SCAN_I; r++) { if (base + r < n) out[base + r] = run; run += v[r]; }
    if (threadIdx.x == SCAN_T - 1) out[n] = run;
}
}  // namespace

// scan_tmp holds the per-tile partials of every recursion level
static int scan_rec(MpCtx* c, const uint32_t* in, uint32_t* out, size_t n, uint32_t* tmp, size_t tmp_left) {
    if (n <= (size_t)SCAN_TILE) {
        k_scan_single<<<1, SCAN_T, 0, c->stream>>>(in, n, out);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        return MP_OK;
    }
    size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (2 * nb + 2 > tmp_left) { c->err = "scan: scratch too small"; return MP_ERR_CAPACITY; }
    uint32_t* part = tmp;
    uint32_t* poff = tmp + nb;          // nb + 1 entries
    k_scan_reduce<<<(unsigned)nb, SCAN_T, 0, c->stream>>>(in, n, part);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    MP_TRY(scan_rec(c, part, poff, nb, tmp + 2 * nb + 1, tmp_left - (2 * nb + 1)));
    k_scan_down<<<(unsigned)nb, SCAN_T, 0, c->stream>>>(in, n, poff, out);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    // total
    MP_CUDA(c, cudaMemcpyAsync(out + n, poff + nb, sizeof(uint32_t), cudaMemcpyDeviceToDevice, c->stream));
    return MP_OK;
}

int mp_scan_u32(MpCtx* c, const uint32_t* in, uint32_t* out, size_t n) {
    return scan_rec(c, in, out, n, c->scan_tmp, c->scan_tmp_elems);
}

// ---------------------------------------------------------------------------
// hashing and the counting sort
// ---------------------------------------------------------------------------
namespace {
// calcHashD (spray_k.cu:1010-1028) / calcHashD_MC (:1030-1048): cell id on a
// grid of (w,hh,d) cells of size dx; an axis outside maps to 0.
__device__ __forceinline__ uint32_t hash_key(float4 q, float gx0, float gy0, float gz0, float dx, int w, int hh, int d) {
    float3 r = (mk3(q.x, q.y, q.z) - mk3(gx0, gy0, gz0)) / mk3(dx, dx, dx);
    int i = (r.x >= 0 && r.x < w) ? (int)r.x : 0;
    int j = (r.y >= 0 && r.y < hh) ? (int)r.y : 0;
    int k = (r.z >= 0 && r.z < d) ? (int)r.z : 0;
    return (uint32_t)(i * hh * d + j * d + k);
}
// keys, per-cell counts, each particle's type as a byte, and a flag raised
// when the keys are not already in order (then the stable sort is the
// identity and the gather can be skipped)
__global__ void k_hash_count(const float4* __restrict__ pos, int np, float gx0, float gy0, float gz0, float dx,
                             int w, int hh, int d, uint32_t* __restrict__ keys, uint32_t* __restrict__ cnt,
                             uint32_t* __restrict__ unsorted, uint8_t* __restrict__ types) {
    __shared__ uint32_t blk_unsorted;
    if (threadIdx.x == 0) blk_unsorted = 0;
    __syncthreads();
    // a warp-uniform grid-stride loop (blockDim is a multiple of 32): all 32
    // lanes run every iteration, lane l holding particle p0 + l when it is
    // below np, so the shuffle that passes each key to the next lane names
    // the whole warp and lane l - 1 always holds particle p - 1
    const int lane = threadIdx.x & 31;
    const int stride = (int)(gridDim.x * blockDim.x);
    for (int p0 = (int)(blockIdx.x * blockDim.x + (threadIdx.x & ~31u)); p0 < np; p0 += stride) {
        const int p = p0 + lane;
        const bool live = p < np;
        uint32_t key = 0;
        if (live) {
            const float4 q = pos[p];
            key = hash_key(q, gx0, gy0, gz0, dx, w, hh, d);
            types[p] = (uint8_t)(pflag(q) & 7);
            keys[p] = key;
        }
        const uint32_t up = __shfl_up_sync(0xffffffffu, key, 1);
        const unsigned lm = __ballot_sync(0xffffffffu, live);
        if (live) {
            // the previous particle's key: from the lane before, lane 0 computes it
            if (p > 0) {
                const uint32_t prev = lane > 0 ? up : hash_key(pos[p - 1], gx0, gy0, gz0, dx, w, hh, d);
                if (prev > key) blk_unsorted = 1u;
            }
            // one atomic per run of equal keys in the warp (particles arrive nearly sorted)
            const unsigned peers = __match_any_sync(lm, key);
            if (lane == __ffs(peers) - 1) atomicAdd(cnt + key, (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && blk_unsorted) *unsorted = 1u;   // one store per block
}
// place each particle index in its cell's range (order inside a cell fixed later);
// counts run back to zero, ready for the next sort
__global__ void k_scatter(const uint32_t* __restrict__ keys, int np, const uint32_t* __restrict__ off,
                          uint32_t* __restrict__ cnt, uint32_t* __restrict__ perm) {
    MP_GRID_LOOP(p, np) {
        uint32_t key = keys[p];
        // a warp's run of equal keys takes consecutive slots in lane (= index) order
        unsigned peers = __match_any_sync(__activemask(), key);
        int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
        uint32_t cntp = (uint32_t)__popc(peers), base = 0;
        if (lane == leader) base = atomicSub(cnt + key, cntp) - cntp;
        base = __shfl_sync(peers, base, leader);
        uint32_t r = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
        perm[off[key] + r] = (uint32_t)p;
    }
}
// sort each cell's indices ascending (stability of thrust::sort_by_key)
__global__ void k_segsort(const uint32_t* __restrict__ off, int ncell, uint32_t* __restrict__ perm) {
    MP_GRID_LOOP(cc, ncell) {
        const uint32_t s0 = off[cc];
        sort_distinct_run(perm, s0, off[cc + 1] - s0, [&](uint32_t) {});
    }
}
// each cell's type mask (which particle types it holds) from the particles'
// type bytes in cell order (coalesced reads), and with `air_words` (the
// simulation grid's sort) the bit of each 4x4x4-cell brick that holds an AIR
// or AIRSOLO particle
__global__ void k_tmask_sorted(const uint32_t* __restrict__ off, int ncell, int w, int hh, int d,
                               const uint8_t* __restrict__ types, uint8_t* __restrict__ tmask,
                               uint32_t* __restrict__ air_words) {
    MP_GRID_LOOP(cc, ncell) {
        uint32_t m = 0;
        for (uint32_t s = off[cc]; s < off[cc + 1]; s++) m |= 1u << __ldg(types + s);
        tmask[cc] = (uint8_t)m;
        if (air_words && (m & ((1u << MP_TYPEAIR) | (1u << MP_TYPEAIRSOLO)))) {
            const uint32_t kk = (uint32_t)cc % (uint32_t)d, jj = ((uint32_t)cc / (uint32_t)d) % (uint32_t)hh,
                           ii = (uint32_t)cc / ((uint32_t)d * (uint32_t)hh);
            const uint32_t bw = ((uint32_t)d + 3) / 4, bh = ((uint32_t)hh + 3) / 4;
            const uint32_t br = ((ii >> 2) * bh + (jj >> 2)) * bw + (kk >> 2);
            atomicOr(air_words + (br >> 5), 1u << (br & 31));
        }
    }
}
__global__ void k_reorder(const uint32_t* __restrict__ perm, int np,
                          const float4* __restrict__ p0, const float4* __restrict__ v0, const float4* __restrict__ h0,
                          float4* __restrict__ p1, float4* __restrict__ v1, float4* __restrict__ h1,
                          const uint8_t* __restrict__ t0, uint8_t* __restrict__ t1) {
    MP_GRID_LOOP(s, np) {
        uint32_t src = perm[s];
        p1[s] = __ldg(p0 + src);
        v1[s] = __ldg(v0 + src);
        h1[s] = __ldg(h0 + src);
        t1[s] = __ldg(t0 + src);
    }
}
}  // namespace

static int sort_on_grid(MpCtx* c, float dx, int w, int hh, int d) {
    int np = c->np();
    int ncell = w * hh * d;
    uint32_t* unsorted = c->u32_scratch + 1;
    MP_CUDA(c, cudaMemsetAsync(unsorted, 0, sizeof(uint32_t), c->stream));
    const bool sim_grid = w == c->G.NX && hh == c->G.NY && d == c->G.NZ;
    if (sim_grid) MP_CUDA(c, cudaMemsetAsync(c->air_brick, 0, sizeof(uint32_t) * c->air_brick_words, c->stream));
    auto tmask_pass = [&](const uint8_t* types) -> int {
        k_tmask_sorted<<<mp_blocks(ncell, 256), 256, 0, c->stream>>>(c->cell_off, ncell, w, hh, d, types, c->tmask,
                                                                     sim_grid ? c->air_brick : nullptr);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        return MP_OK;
    };
    if (np > 0) {
        k_hash_count<<<mp_blocks(np, 256), 256, 0, c->stream>>>(c->pos, np, c->G.gx0, c->G.gy0, c->G.gz0, dx, w, hh, d,
                                                                c->keys, c->cell_cnt, unsorted, c->pflag8);
        c->launches++;
        MP_CHECK_LAUNCH(c);
    }
    MP_TRY(mp_scan_u32(c, c->cell_cnt, c->cell_off, (size_t)ncell));
    uint32_t h_unsorted = 1;
    MP_CUDA(c, cudaMemcpyAsync(&h_unsorted, unsorted, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
    MP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->work[h_unsorted ? MP_WC_SORT_FULL : MP_WC_SORT_FAST]++;
    if (!h_unsorted) {
        // already in cell order: the stable sort is the identity permutation;
        // the counts still have to run back to zero for the next sort
        MP_CUDA(c, cudaMemsetAsync(c->cell_cnt, 0, sizeof(uint32_t) * ncell, c->stream));
        return tmask_pass(c->pflag8);
    }
    if (np > 0) {
        k_scatter<<<mp_blocks(np, 256), 256, 0, c->stream>>>(c->keys, np, c->cell_off, c->cell_cnt, c->perm);
        c->launches++;
        MP_CHECK_LAUNCH(c);
    }
    k_segsort<<<mp_blocks(ncell, 256), 256, 0, c->stream>>>(c->cell_off, ncell, c->perm);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    if (np > 0) {
        k_reorder<<<mp_blocks(np, 256), 256, 0, c->stream>>>(c->perm, np, c->pos, c->vel, c->heat, c->pos2, c->vel2, c->heat2,
                                                             c->pflag8, c->pflag8s);
        c->launches++;
        MP_CHECK_LAUNCH(c);
        std::swap(c->pos, c->pos2); std::swap(c->vel, c->vel2); std::swap(c->heat, c->heat2);
    }
    return tmask_pass(np > 0 ? c->pflag8s : c->pflag8);
}

int k_hash_sort(MpCtx* c) {
    KtScope kt(c, MP_KT_SORT);
    c->mc_sorted = 0;
    return sort_on_grid(c, c->G.h, c->G.NX, c->G.NY, c->G.NZ);
}

// preMC + hashAndSortParticles_MC (spray.cu:759-765, 639-662): cell size
// cellsize/NXMC*NX on the 2x grid (calcHashD_MC, spray_k.cu:1030-1048)
int k_mc_presort(MpCtx* c) {
    KtScope kt(c, MP_KT_SORT);
    int NXMC = 2 * c->G.NX, NYMC = 2 * c->G.NY, NZMC = 2 * c->G.NZ;
    float dx = c->G.h / (float)NXMC * (float)c->G.NX;
    MP_TRY(sort_on_grid(c, dx, NXMC, NYMC, NZMC));
    c->mc_sorted = 1;
    return MP_OK;
}

// ---------------------------------------------------------------------------
// packing between the reference's structure of arrays and the float4 streams
// ---------------------------------------------------------------------------
namespace {
__global__ void k_pack(int n, const float* __restrict__ p3, const float* __restrict__ v3, const int8_t* __restrict__ fl,
                       const float* __restrict__ m, const float* __restrict__ T, const float* __restrict__ L,
                       const float* __restrict__ so, const float* __restrict__ ga,
                       float4* __restrict__ pos, float4* __restrict__ vel, float4* __restrict__ heat) {
    MP_GRID_LOOP(p, n) {
        pos[p] = make_float4(p3[3 * p], p3[3 * p + 1], p3[3 * p + 2], flagbits((int)fl[p]));
        vel[p] = make_float4(v3[3 * p], v3[3 * p + 1], v3[3 * p + 2], m[p]);
        heat[p] = make_float4(T[p], L[p], so[p], ga[p]);
    }
}
__global__ void k_unpack(int n, const float4* __restrict__ pos, const float4* __restrict__ vel, const float4* __restrict__ heat,
                         float* __restrict__ p3, float* __restrict__ v3, int8_t* __restrict__ fl, float* __restrict__ m,
                         float* __restrict__ T, float* __restrict__ L, float* __restrict__ so, float* __restrict__ ga) {
    MP_GRID_LOOP(p, n) {
        float4 a = pos[p], b = vel[p], hh = heat[p];
        p3[3 * p] = a.x; p3[3 * p + 1] = a.y; p3[3 * p + 2] = a.z; fl[p] = (int8_t)pflag(a);
        v3[3 * p] = b.x; v3[3 * p + 1] = b.y; v3[3 * p + 2] = b.z; m[p] = b.w;
        T[p] = hh.x; L[p] = hh.y; so[p] = hh.z; ga[p] = hh.w;
    }
}
__global__ void k_startend(const uint32_t* __restrict__ off, int n, uint32_t* __restrict__ st, uint32_t* __restrict__ en) {
    MP_GRID_LOOP(cc, n) {
        uint32_t a = off[cc], b = off[cc + 1];
        st[cc] = (a < b) ? a : MP_CELL_UNDEF;
        en[cc] = (a < b) ? b : 0u;
    }
}
}  // namespace

// staging: host SoA lands in the second particle buffers, then one kernel packs
int k_pack_particles(MpCtx* c, int n, const float* pos3, const float* vel3, const int8_t* flag, const float* mass,
                     const float* T, const float* L, const float* sol, const float* gas) {
    if (n == 0) return MP_OK;
    float* sp = reinterpret_cast<float*>(c->pos2);
    float* sv = reinterpret_cast<float*>(c->vel2);
    float* sm = reinterpret_cast<float*>(c->heat2);
    float* sT = sm + n; float* sL = sT + n; float* ss = sL + n;
    float* sg = reinterpret_cast<float*>(c->pscr);
    int8_t* sf = reinterpret_cast<int8_t*>(sg + n);
    cudaStream_t s = c->stream;
    MP_CUDA(c, cudaMemcpyAsync(sp, pos3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
    if (vel3) MP_CUDA(c, cudaMemcpyAsync(sv, vel3, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
    else MP_CUDA(c, cudaMemsetAsync(sv, 0, sizeof(float) * 3 * n, s));
    MP_CUDA(c, cudaMemcpyAsync(sf, flag, n, cudaMemcpyHostToDevice, s));
    MP_CUDA(c, cudaMemcpyAsync(sm, mass, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    const float* srcs[4] = {T, L, sol, gas};
    float* dsts[4] = {sT, sL, ss, sg};
    for (int q = 0; q < 4; q++) {
        if (srcs[q]) MP_CUDA(c, cudaMemcpyAsync(dsts[q], srcs[q], sizeof(float) * n, cudaMemcpyHostToDevice, s));
        else MP_CUDA(c, cudaMemsetAsync(dsts[q], 0, sizeof(float) * n, s));
    }
    k_pack<<<mp_blocks(n, 256), 256, 0, s>>>(n, sp, sv, sf, sm, sT, sL, ss, sg, c->pos, c->vel, c->heat);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}

int k_unpack_particles(MpCtx* c, int n, float* pos3, float* vel3, int8_t* flag, float* mass, float* T, float* L,
                       float* sol, float* gas) {
    if (n == 0) return MP_OK;
    float* sp = reinterpret_cast<float*>(c->pos2);
    float* sv = reinterpret_cast<float*>(c->vel2);
    float* sm = reinterpret_cast<float*>(c->heat2);
    float* sT = sm + n; float* sL = sT + n; float* ss = sL + n;
    float* sg = reinterpret_cast<float*>(c->pscr);
    int8_t* sf = reinterpret_cast<int8_t*>(sg + n);
    cudaStream_t s = c->stream;
    k_unpack<<<mp_blocks(n, 256), 256, 0, s>>>(n, c->pos, c->vel, c->heat, sp, sv, sf, sm, sT, sL, ss, sg);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    void* dst[8] = {pos3, vel3, flag, mass, T, L, sol, gas};
    const void* src[8] = {sp, sv, sf, sm, sT, sL, ss, sg};
    size_t sz[8] = {12, 12, 1, 4, 4, 4, 4, 4};
    for (int q = 0; q < 8; q++)
        if (dst[q]) MP_CUDA(c, cudaMemcpyAsync(dst[q], src[q], sz[q] * n, cudaMemcpyDeviceToHost, s));
    MP_CUDA(c, cudaStreamSynchronize(s));
    return MP_OK;
}

int k_cells_to_startend(MpCtx* c, uint32_t* st, uint32_t* en) {
    int n = c->G.n;
    k_startend<<<mp_blocks(n, 256), 256, 0, c->stream>>>(c->cell_off, n, st, en);
    c->launches++;
    MP_CHECK_LAUNCH(c);
    return MP_OK;
}
