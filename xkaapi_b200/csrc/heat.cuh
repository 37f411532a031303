// Heat-diffusion-2d 5-point Jacobi tile body for sm_100a (device code shared by the
// per-task kernels, the whole-step kernel and the persistent scheduler).
//
// Layout: column-major grid, cell (i, j) at G[j*ld + i]; i (rows) is the contiguous dim.
// Work unit = a warp STRIP: 32*VEC consecutive rows (each lane owns VEC consecutive rows,
// loaded as one 16-byte vector) x a range of columns swept left to right. The sweep keeps
// the west/centre/east columns in registers, so every input cell is read from HBM once per
// strip; north/south neighbours come from the adjacent lanes by shuffle. Strips overlap by
// two rows (a strip writes its 32*VEC-2 inner rows), so no lane needs a halo load. Each batch
// of PF east columns is loaded before any is used, and one bulk L2 prefetch per column runs
// `pfd` columns ahead, keeping enough HBM bytes in flight without spending registers.
//
// Arithmetic matches the reference formula (examples/heat-diffusion-2d/src/main.cc:408-421,
// src/kernels/diffusion.cu:117-121) with DX = DY = 1, in its evaluation order and without
// contraction: A = (S[i+1] - 2S) + S[i-1]; B = (S[j+1] - 2S) + S[j-1]; D = S + c*(A + B).
#pragma once
#include "common.cuh"

#include <type_traits>

namespace xkb {

template <typename T> struct HeatVec;
template <> struct HeatVec<double> { typedef double2 V; static constexpr int N = 2; };
template <> struct HeatVec<float>  { typedef float4  V; static constexpr int N = 4; };

template <typename T, int VEC> struct Cells { T v[VEC]; };

template <bool CG, typename T>
__device__ __forceinline__ T ld_scalar(const T * p) { if constexpr (CG) return __ldcg(p); else return __ldg(p); }

// Load VEC rows [r, r+VEC) of column j. Rows outside [0, nx) read as 0 and are never used.
template <typename T, int VEC, bool CG>
__device__ __forceinline__ Cells<T, VEC> ld_cells(const T * __restrict__ g, int64_t ld, int64_t nx, int64_t r, int64_t j, bool vec_ok)
{
    Cells<T, VEC> c;
    const T * p = g + j * ld + r;
    if (vec_ok && r >= 0 && r + VEC <= nx)
    {
        if constexpr (VEC == 2 && sizeof(T) == 8) {
            double2 v = CG ? __ldcg((const double2 *) p) : __ldg((const double2 *) p);
            c.v[0] = v.x; c.v[1] = v.y;
        } else if constexpr (VEC == 4 && sizeof(T) == 4) {
            float4 v = CG ? __ldcg((const float4 *) p) : __ldg((const float4 *) p);
            c.v[0] = v.x; c.v[1] = v.y; c.v[2] = v.z; c.v[3] = v.w;
        } else if constexpr (VEC == 4 && sizeof(T) == 8) {
            double2 a = CG ? __ldcg((const double2 *) p) : __ldg((const double2 *) p);
            double2 b = CG ? __ldcg((const double2 *) p + 1) : __ldg((const double2 *) p + 1);
            c.v[0] = a.x; c.v[1] = a.y; c.v[2] = b.x; c.v[3] = b.y;
        } else {
#pragma unroll
            for (int e = 0; e < VEC; ++e) c.v[e] = ld_scalar<CG>(p + e);
        }
    }
    else
    {
#pragma unroll
        for (int e = 0; e < VEC; ++e)
            c.v[e] = (r + e >= 0 && r + e < nx) ? ld_scalar<CG>(p + e) : T(0);
    }
    return c;
}

__device__ __forceinline__ double heat_update(double s, double up, double down, double w, double e, double c)
{
    const double s2 = __dmul_rn(2.0, s);
    const double a = __dadd_rn(__dsub_rn(down, s2), up);
    const double b = __dadd_rn(__dsub_rn(e, s2), w);
    return __dadd_rn(s, __dmul_rn(c, __dadd_rn(a, b)));
}

// Bulk L2 prefetch of `bytes` (multiple of 16, 16-byte aligned source) with one instruction.
__device__ __forceinline__ void l2_prefetch_bulk(const void * p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(p), "r"(bytes) : "memory");
}

// Rows a warp strip loads (32 lanes x VEC) and writes: a strip based at row rbase writes rows
// [rbase+1, rbase+1+OUT), so the north/south neighbours of every written row are in the
// strip's own registers; consecutive strips step by OUT rows.
template <int VEC> struct StripGeom {
    static constexpr int LOAD = 32 * VEC;
    static constexpr int OUT = LOAD - VEC;    // row step between strips (keeps VEC alignment)
};

// One warp strip: loads rows [rbase, rbase + 32*VEC) of columns [cy0-1, cy1], writes rows
// [rbase+1, rbase+1+OUT) intersected with [rx0, rx1) of columns [cy0, cy1).
// Preconditions: 1 <= rx0 < rx1 <= nx-1, 1 <= cy0 < cy1 <= ny-1, rbase a multiple of VEC,
// rbase >= 0. `vec_ok` = ld and both base pointers allow VEC-wide aligned accesses.
// FAST = every loaded row is inside [0, nx) and vec_ok (no per-load checks).
template <typename T, int VEC, int PF, bool CG, bool FAST>
__device__ __forceinline__ void heat_strip_impl(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                                int64_t nx, int64_t ny, int64_t rbase, int64_t rx0, int64_t rx1,
                                                int64_t cy0, int64_t cy1, double c, bool vec_ok, int pfd)
{
    const int lane = threadIdx.x & 31;
    const int64_t r = rbase + (int64_t) lane * VEC;
    // rows of this lane that are written
    const int64_t w0 = (r > rbase ? r : rbase + 1) > rx0 ? (r > rbase ? r : rbase + 1) : rx0;
    int64_t w1 = r + VEC; if (w1 > rbase + 1 + StripGeom<VEC>::OUT) w1 = rbase + 1 + StripGeom<VEC>::OUT;
    if (w1 > rx1) w1 = rx1;
    const bool full_store = vec_ok && w0 == r && w1 == r + VEC;
    int64_t pf_rows = nx - rbase; if (pf_rows > StripGeom<VEC>::LOAD) pf_rows = StripGeom<VEC>::LOAD;
    const uint32_t pf_bytes = (uint32_t) ((pf_rows * (int64_t) sizeof(T)) & ~(int64_t) 15);
    const bool pf_on = pfd > 0 && vec_ok && pf_bytes > 0;

    const T * __restrict__ sp = src + r;
    T * __restrict__ dp = dst + r;
    auto load = [&](int64_t j) -> Cells<T, VEC> {
        if constexpr (FAST) {
            Cells<T, VEC> q;
            const T * p = sp + j * ld;
            if constexpr (VEC == 2 && sizeof(T) == 8) {
                double2 v = CG ? __ldcg((const double2 *) p) : __ldg((const double2 *) p);
                q.v[0] = v.x; q.v[1] = v.y;
            } else if constexpr (VEC == 4 && sizeof(T) == 8) {
                double2 a = CG ? __ldcg((const double2 *) p) : __ldg((const double2 *) p);
                double2 b = CG ? __ldcg((const double2 *) p + 1) : __ldg((const double2 *) p + 1);
                q.v[0] = a.x; q.v[1] = a.y; q.v[2] = b.x; q.v[3] = b.y;
            } else {
                float4 v = CG ? __ldcg((const float4 *) p) : __ldg((const float4 *) p);
                q.v[0] = v.x; q.v[1] = v.y; q.v[2] = v.z; q.v[3] = v.w;
            }
            return q;
        } else {
            return ld_cells<T, VEC, CG>(src, ld, nx, r, j, vec_ok);
        }
    };

    Cells<T, VEC> west = load(cy0 - 1);
    Cells<T, VEC> cur  = load(cy0);
    // one block of PF columns from j0; FULL: all PF columns lie before cy1 (no per-column checks)
    auto block = [&](const int64_t j0, auto full_tag) {
        constexpr bool FULL = decltype(full_tag)::value;
        if (pf_on && lane < PF)
        {
            // lane k prefetches column j0 + pfd + k of the strip into L2 with one bulk request
            const int64_t jp = j0 + pfd + lane;
            if (jp <= cy1) l2_prefetch_bulk(src + jp * ld + rbase, pf_bytes);
        }
        Cells<T, VEC> nxt[PF];
#pragma unroll
        for (int k = 0; k < PF; ++k)
            if (FULL || j0 + k + 1 <= cy1) nxt[k] = load(j0 + k + 1);
#pragma unroll
        for (int k = 0; k < PF; ++k)
        {
            const int64_t jc = j0 + k;
            if (!FULL && jc >= cy1) break;               // warp-uniform
            const T north = __shfl_up_sync(0xffffffffu, cur.v[VEC - 1], 1);
            const T south = __shfl_down_sync(0xffffffffu, cur.v[0], 1);
            Cells<T, VEC> out;
#pragma unroll
            for (int e = 0; e < VEC; ++e)
            {
                const double sv = (double) cur.v[e];
                const double up = (double) (e == 0 ? north : cur.v[e - 1]);
                const double dn = (double) (e == VEC - 1 ? south : cur.v[e + 1]);
                out.v[e] = (T) heat_update(sv, up, dn, (double) west.v[e], (double) nxt[k].v[e], c);
            }
            T * q = dp + jc * ld;
            if (full_store)
            {
                if constexpr (VEC == 2 && sizeof(T) == 8) *(double2 *) q = make_double2(out.v[0], out.v[1]);
                else if constexpr (VEC == 4 && sizeof(T) == 8)
                {
                    ((double2 *) q)[0] = make_double2(out.v[0], out.v[1]);
                    ((double2 *) q)[1] = make_double2(out.v[2], out.v[3]);
                }
                else *(float4 *) q = make_float4(out.v[0], out.v[1], out.v[2], out.v[3]);
            }
            else
            {
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                    if (r + e >= w0 && r + e < w1) q[e] = out.v[e];
            }
            west = cur;
            cur = nxt[k];
        }
    };
    int64_t j0 = cy0;
    for (; j0 + PF <= cy1; j0 += PF) block(j0, std::true_type{});
    if (j0 < cy1) block(j0, std::false_type{});
}

// Edge strips (grid bottom rows, unaligned grids) take a checked path kept out of line so the
// fast path's register allocation stays small.
template <typename T, int VEC, int PF, bool CG>
__device__ __noinline__ void heat_strip_edge(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                             int64_t nx, int64_t ny, int64_t rbase, int64_t rx0, int64_t rx1,
                                             int64_t cy0, int64_t cy1, double c, bool vec_ok, int pfd)
{
    heat_strip_impl<T, VEC, 2, CG, false>(src, dst, ld, nx, ny, rbase, rx0, rx1, cy0, cy1, c, vec_ok, pfd);
}

template <typename T, int VEC, int PF, bool CG>
__device__ __forceinline__ void heat_strip(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                           int64_t nx, int64_t ny, int64_t rbase, int64_t rx0, int64_t rx1,
                                           int64_t cy0, int64_t cy1, double c, bool vec_ok, int pfd)
{
    if (vec_ok && rbase + StripGeom<VEC>::LOAD <= nx)
        heat_strip_impl<T, VEC, PF, CG, true>(src, dst, ld, nx, ny, rbase, rx0, rx1, cy0, cy1, c, vec_ok, pfd);
    else
        heat_strip_edge<T, VEC, PF, CG>(src, dst, ld, nx, ny, rbase, rx0, rx1, cy0, cy1, c, vec_ok, pfd);
}

// Cells a tile task writes: its rows/cols clipped to the interior [1, n-1).
struct TileBox { int64_t rx0, rx1, cy0, cy1; };

__host__ __device__ __forceinline__ TileBox heat_tile_box(int64_t nx, int64_t ny, int64_t x0, int64_t x1, int64_t y0, int64_t y1)
{
    TileBox b;
    b.rx0 = x0 > 1 ? x0 : 1;  b.rx1 = x1 < nx - 1 ? x1 : nx - 1;
    b.cy0 = y0 > 1 ? y0 : 1;  b.cy1 = y1 < ny - 1 ? y1 : ny - 1;
    return b;
}

// Tile tasks use HALO strips: a strip based at rbase (multiple of VEC) writes the rows
// [rbase, rbase + 32*VEC) it loads; lanes 0 and 31 fetch the north/south halo cell of each
// column. A 128-row FP64 tile is then exactly two strips (overlapping strips would need three).
template <typename T, int VEC, int PF, bool CG, bool FAST>
__device__ __forceinline__ void heat_strip_halo_impl(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                                     int64_t nx, int64_t rbase, int64_t rx0, int64_t rx1,
                                                     int64_t cy0, int64_t cy1, double c, bool vec_ok, int pfd)
{
    const int lane = threadIdx.x & 31;
    const int64_t r = rbase + (int64_t) lane * VEC;
    const int64_t rn = rbase - 1, rs = rbase + 32 * VEC;
    // halo cells of a block of PF columns. FP32 strips (many columns per block) gather them in
    // lanes: lane k (k < PF) holds the north cell of column j0 + k, lane 16 + k its south cell --
    // one load instruction per block instead of one per column and side, two registers per lane
    // instead of 2 x PF -- and lanes 0 and 31 take them by shuffle (3-4 % faster on the FP32
    // graph); FP64 strips keep one register per column and side in lanes 0 and 31 (1 % faster
    // there than the shuffles).
    constexpr bool HALO_LANES = sizeof(T) == 4;
    static_assert(!HALO_LANES || PF <= 16, "halo lanes");
    const bool has_n = lane == 0 && rn >= 0, has_s = lane == 31 && rs < nx;
    const int hk = lane & 15;
    const bool h_south = lane >= 16;
    const bool h_row_ok = h_south ? rs < nx : rn >= 0;
    const int64_t h_row = h_south ? rs : rn;
    const bool lane_rows = (r + VEC > rx0) && (r < rx1);
    const bool full_store = vec_ok && r >= rx0 && r + VEC <= rx1;
    // the L2 prefetch of a column covers the strip AND its halo rows (VEC rows on each side keep
    // the 16-byte alignment), so the lanes' halo loads hit L2 like the strip's own loads
    const int64_t pf_lo = rbase >= VEC ? rbase - VEC : 0;
    int64_t pf_hi = rbase + 33 * VEC; if (pf_hi > nx) pf_hi = nx;
    const uint32_t pf_bytes = (uint32_t) (((pf_hi - pf_lo) * (int64_t) sizeof(T)) & ~(int64_t) 15);
    const bool pf_on = pfd > 0 && vec_ok && pf_hi > pf_lo && pf_bytes > 0;
    const T * __restrict__ sp = src + r;
    T * __restrict__ dp = dst + r;
    auto load = [&](int64_t j) -> Cells<T, VEC> {
        if constexpr (FAST) {
            Cells<T, VEC> q;
            const T * p = sp + j * ld;
            if constexpr (VEC == 2 && sizeof(T) == 8) {
                double2 v = CG ? __ldcg((const double2 *) p) : __ldg((const double2 *) p);
                q.v[0] = v.x; q.v[1] = v.y;
            } else if constexpr (VEC == 4 && sizeof(T) == 8) {
                double2 a = CG ? __ldcg((const double2 *) p) : __ldg((const double2 *) p);
                double2 b = CG ? __ldcg((const double2 *) p + 1) : __ldg((const double2 *) p + 1);
                q.v[0] = a.x; q.v[1] = a.y; q.v[2] = b.x; q.v[3] = b.y;
            } else {
                float4 v = CG ? __ldcg((const float4 *) p) : __ldg((const float4 *) p);
                q.v[0] = v.x; q.v[1] = v.y; q.v[2] = v.z; q.v[3] = v.w;
            }
            return q;
        } else {
            return ld_cells<T, VEC, CG>(src, ld, nx, r, j, vec_ok);
        }
    };
    Cells<T, VEC> west = load(cy0 - 1);
    Cells<T, VEC> cur  = load(cy0);
    // one block of PF columns from j0; FULL: all PF columns lie before cy1 (no per-column checks)
    auto block = [&](const int64_t j0, auto full_tag) {
        constexpr bool FULL = decltype(full_tag)::value;
        if (pf_on && lane < PF)
        {
            const int64_t jp = j0 + pfd + lane;
            if (jp <= cy1) l2_prefetch_bulk(src + jp * ld + pf_lo, pf_bytes);
        }
        Cells<T, VEC> nxt[PF];
        [[maybe_unused]] T hv = T(0);
        [[maybe_unused]] T hn[HALO_LANES ? 1 : PF], hs[HALO_LANES ? 1 : PF];
        if constexpr (HALO_LANES)
            if (hk < PF && h_row_ok && j0 + hk < cy1) hv = ld_scalar<CG>(src + (j0 + hk) * ld + h_row);
#pragma unroll
        for (int k = 0; k < PF; ++k)
        {
            if (FULL || j0 + k + 1 <= cy1) nxt[k] = load(j0 + k + 1);
            if constexpr (!HALO_LANES)
            {
                const int64_t jc = j0 + k;
                hn[k] = (has_n && jc < cy1) ? ld_scalar<CG>(src + jc * ld + rn) : T(0);
                hs[k] = (has_s && jc < cy1) ? ld_scalar<CG>(src + jc * ld + rs) : T(0);
            }
        }
#pragma unroll
        for (int k = 0; k < PF; ++k)
        {
            const int64_t jc = j0 + k;
            if (!FULL && jc >= cy1) break;               // warp-uniform
            T north = __shfl_up_sync(0xffffffffu, cur.v[VEC - 1], 1);
            T south = __shfl_down_sync(0xffffffffu, cur.v[0], 1);
            T hnk, hsk;
            if constexpr (HALO_LANES) { hnk = __shfl_sync(0xffffffffu, hv, k); hsk = __shfl_sync(0xffffffffu, hv, 16 + k); }
            else { hnk = hn[k]; hsk = hs[k]; }
            if (lane == 0)  north = hnk;
            if (lane == 31) south = hsk;
            if (lane_rows)
            {
                Cells<T, VEC> out;
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                {
                    const double sv = (double) cur.v[e];
                    const double up = (double) (e == 0 ? north : cur.v[e - 1]);
                    const double dn = (double) (e == VEC - 1 ? south : cur.v[e + 1]);
                    out.v[e] = (T) heat_update(sv, up, dn, (double) west.v[e], (double) nxt[k].v[e], c);
                }
                T * q = dp + jc * ld;
                if (full_store)
                {
                    if constexpr (VEC == 2 && sizeof(T) == 8) *(double2 *) q = make_double2(out.v[0], out.v[1]);
                    else if constexpr (VEC == 4 && sizeof(T) == 8)
                    {
                        ((double2 *) q)[0] = make_double2(out.v[0], out.v[1]);
                        ((double2 *) q)[1] = make_double2(out.v[2], out.v[3]);
                    }
                    else *(float4 *) q = make_float4(out.v[0], out.v[1], out.v[2], out.v[3]);
                }
                else
                {
#pragma unroll
                    for (int e = 0; e < VEC; ++e)
                        if (r + e >= rx0 && r + e < rx1) q[e] = out.v[e];
                }
            }
            west = cur;
            cur = nxt[k];
        }
    };
    int64_t j0 = cy0;
    for (; j0 + PF <= cy1; j0 += PF) block(j0, std::true_type{});
    if (j0 < cy1) block(j0, std::false_type{});
}

template <typename T, int VEC, int PF, bool CG>
__device__ __noinline__ void heat_strip_halo_edge(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                                  int64_t nx, int64_t rbase, int64_t rx0, int64_t rx1,
                                                  int64_t cy0, int64_t cy1, double c, bool vec_ok, int pfd)
{
    heat_strip_halo_impl<T, VEC, 2, CG, false>(src, dst, ld, nx, rbase, rx0, rx1, cy0, cy1, c, vec_ok, pfd);
}

template <typename T, int VEC, int PF, bool CG>
__device__ __forceinline__ void heat_strip_halo(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                                int64_t nx, int64_t rbase, int64_t rx0, int64_t rx1,
                                                int64_t cy0, int64_t cy1, double c, bool vec_ok, int pfd)
{
    if (vec_ok && rbase >= 0 && rbase + 32 * VEC <= nx)
        heat_strip_halo_impl<T, VEC, PF, CG, true>(src, dst, ld, nx, rbase, rx0, rx1, cy0, cy1, c, vec_ok, pfd);
    else
        heat_strip_halo_edge<T, VEC, PF, CG>(src, dst, ld, nx, rbase, rx0, rx1, cy0, cy1, c, vec_ok, pfd);
}

// Strips a tile box splits into when `nwarps` warps share it: row groups of 32*VEC rows
// (first base = rx0 rounded down to a multiple of VEC) times column groups.
template <int VEC>
__host__ __device__ __forceinline__ void heat_tile_split(const TileBox & b, int nwarps, int64_t & rbase0,
                                                         int & nrg, int & ncg, int64_t & cols_per)
{
    rbase0 = b.rx0 - (b.rx0 % VEC);
    const int64_t rows = b.rx1 - rbase0;
    nrg = (int) ((rows + 32 * VEC - 1) / (32 * VEC));
    ncg = nwarps / (nrg > 0 ? nrg : 1);
    if (ncg < 1) ncg = 1;
    const int64_t cols = b.cy1 - b.cy0;
    if (ncg > cols) ncg = (int) (cols > 0 ? cols : 1);
    cols_per = (cols + ncg - 1) / ncg;
}

// A team of `nwarps` warps (warp index `warp` within the team) executes one tile task: the
// warps take the tile's strips round-robin.
template <typename T, int VEC, int PF, bool CG>
__device__ __forceinline__ void heat_tile_team(const T * src, T * dst, int64_t ld, int64_t nx, int64_t ny,
                                               int64_t x0, int64_t x1, int64_t y0, int64_t y1, double c, bool vec_ok,
                                               int pfd, int warp, int nwarps)
{
    const TileBox b = heat_tile_box(nx, ny, x0, x1, y0, y1);
    if (b.rx0 >= b.rx1 || b.cy0 >= b.cy1) return;
    int64_t rbase0, cols_per; int nrg, ncg;
    heat_tile_split<VEC>(b, nwarps, rbase0, nrg, ncg, cols_per);
    for (int s = warp; s < nrg * ncg; s += nwarps)
    {
        const int rg = s % nrg, cg = s / nrg;
        const int64_t cy0 = b.cy0 + cg * cols_per;
        int64_t cy1 = cy0 + cols_per; if (cy1 > b.cy1) cy1 = b.cy1;
        if (cy0 >= cy1) continue;
        heat_strip_halo<T, VEC, PF, CG>(src, dst, ld, nx, rbase0 + (int64_t) rg * 32 * VEC, b.rx0, b.rx1, cy0, cy1, c, vec_ok, pfd);
    }
}

// A whole CTA executes one tile task.
template <typename T, int VEC, int PF, bool CG>
__device__ __forceinline__ void heat_tile_cta(const T * src, T * dst, int64_t ld, int64_t nx, int64_t ny,
                                              int64_t x0, int64_t x1, int64_t y0, int64_t y1, double c, bool vec_ok,
                                              int pfd = 0)
{
    heat_tile_team<T, VEC, PF, CG>(src, dst, ld, nx, ny, x0, x1, y0, y1, c, vec_ok, pfd, threadIdx.x >> 5, blockDim.x >> 5);
}

} // namespace xkb
