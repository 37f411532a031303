// Heat-diffusion-2d 5-point Jacobi tile body for sm_100a (device code shared by the
// per-task kernels, the whole-step kernel and the persistent scheduler).
//
// Layout: column-major grid, cell (i, j) at G[j*ld + i]; i (rows) is the contiguous dim.
// Work unit = a warp STRIP: 32*VEC consecutive rows (each lane owns VEC consecutive rows,
// loaded as one 16-byte vector) x a range of columns swept left to right. The sweep keeps
// the west/centre/east columns in registers, so every input cell is read from HBM once per
// strip; north/south neighbours come from the adjacent lanes by shuffle, and only lanes 0
// and 31 fetch one halo cell per column. Each batch of PF east columns is loaded before any
// of them is used, giving PF x 16 B per lane in flight.
//
// Arithmetic matches the reference formula (examples/heat-diffusion-2d/src/main.cc:408-421,
// src/kernels/diffusion.cu:117-121) with DX = DY = 1, in its evaluation order and without
// contraction: A = (S[i+1] - 2S) + S[i-1]; B = (S[j+1] - 2S) + S[j-1]; D = S + c*(A + B).
#pragma once
#include "common.cuh"

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
    const double a = __dadd_rn(__dsub_rn(down, __dmul_rn(2.0, s)), up);
    const double b = __dadd_rn(__dsub_rn(e, __dmul_rn(2.0, s)), w);
    return __dadd_rn(s, __dmul_rn(c, __dadd_rn(a, b)));
}

// One warp strip: rows [rbase, rbase + 32*VEC) intersected with [rx0, rx1), columns
// [cy0, cy1). Preconditions: 1 <= rx0 < rx1 <= nx-1, 1 <= cy0 < cy1 <= ny-1, and rbase a
// multiple of VEC. `vec_ok` = ld and both base pointers allow VEC-wide aligned accesses.
template <typename T, int VEC, int PF, bool CG>
__device__ __forceinline__ void heat_strip(const T * __restrict__ src, T * __restrict__ dst, int64_t ld,
                                           int64_t nx, int64_t rbase, int64_t rx0, int64_t rx1,
                                           int64_t cy0, int64_t cy1, double c, bool vec_ok)
{
    const int lane = threadIdx.x & 31;
    const int64_t r = rbase + (int64_t) lane * VEC;
    const int64_t rn = rbase - 1;                   // north halo row of the strip
    const int64_t rs = rbase + 32 * VEC;            // south halo row of the strip
    const bool lane_rows = (r + VEC > rx0) && (r < rx1);

    Cells<T, VEC> west = ld_cells<T, VEC, CG>(src, ld, nx, r, cy0 - 1, vec_ok);
    Cells<T, VEC> cur  = ld_cells<T, VEC, CG>(src, ld, nx, r, cy0, vec_ok);

    for (int64_t j0 = cy0; j0 < cy1; j0 += PF)
    {
        Cells<T, VEC> nxt[PF];
        T hn[PF], hs[PF];
#pragma unroll
        for (int k = 0; k < PF; ++k)
        {
            const int64_t je = j0 + k + 1;
            if (je <= cy1) nxt[k] = ld_cells<T, VEC, CG>(src, ld, nx, r, je, vec_ok);
            const int64_t jc = j0 + k;
            hn[k] = T(0); hs[k] = T(0);
            if (jc < cy1)
            {
                if (lane == 0 && rn >= 0)   hn[k] = ld_scalar<CG>(src + jc * ld + rn);
                if (lane == 31 && rs < nx)  hs[k] = ld_scalar<CG>(src + jc * ld + rs);
            }
        }
#pragma unroll
        for (int k = 0; k < PF; ++k)
        {
            const int64_t jc = j0 + k;
            if (jc >= cy1) break;
            // neighbours across lanes (warp-uniform control flow up to here)
            T north = __shfl_up_sync(0xffffffffu, cur.v[VEC - 1], 1);
            T south = __shfl_down_sync(0xffffffffu, cur.v[0], 1);
            if (lane == 0)  north = hn[k];
            if (lane == 31) south = hs[k];
            if (lane_rows)
            {
                Cells<T, VEC> out;
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                {
                    const double s  = (double) cur.v[e];
                    const double up = (double) (e == 0 ? north : cur.v[e - 1]);
                    const double dn = (double) (e == VEC - 1 ? south : cur.v[e + 1]);
                    out.v[e] = (T) heat_update(s, up, dn, (double) west.v[e], (double) nxt[k].v[e], c);
                }
                T * q = dst + jc * ld + r;
                if (vec_ok && r >= rx0 && r + VEC <= rx1)
                {
                    if constexpr (VEC == 2 && sizeof(T) == 8)      *(double2 *) q = make_double2(out.v[0], out.v[1]);
                    else if constexpr (VEC == 4 && sizeof(T) == 4) *(float4 *) q = make_float4(out.v[0], out.v[1], out.v[2], out.v[3]);
                    else {
#pragma unroll
                        for (int e = 0; e < VEC; ++e) q[e] = out.v[e];
                    }
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
    }
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

// Number of warp strips a tile box splits into when `nwarps` warps share it: row groups of
// 32*VEC rows (aligned to VEC) times column groups, at least one column per strip.
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

// A whole CTA executes one tile task: the warps take the tile's strips round-robin.
template <typename T, int VEC, int PF, bool CG>
__device__ __forceinline__ void heat_tile_cta(const T * src, T * dst, int64_t ld, int64_t nx, int64_t ny,
                                              int64_t x0, int64_t x1, int64_t y0, int64_t y1, double c, bool vec_ok)
{
    const TileBox b = heat_tile_box(nx, ny, x0, x1, y0, y1);
    if (b.rx0 >= b.rx1 || b.cy0 >= b.cy1) return;
    const int nwarps = blockDim.x >> 5, warp = threadIdx.x >> 5;
    int64_t rbase0, cols_per; int nrg, ncg;
    heat_tile_split<VEC>(b, nwarps, rbase0, nrg, ncg, cols_per);
    for (int s = warp; s < nrg * ncg; s += nwarps)
    {
        const int rg = s % nrg, cg = s / nrg;
        const int64_t cy0 = b.cy0 + cg * cols_per;
        int64_t cy1 = cy0 + cols_per; if (cy1 > b.cy1) cy1 = b.cy1;
        if (cy0 >= cy1) continue;
        heat_strip<T, VEC, PF, CG>(src, dst, ld, nx, rbase0 + (int64_t) rg * 32 * VEC, b.rx0, b.rx1, cy0, cy1, c, vec_ok);
    }
}

} // namespace xkb
