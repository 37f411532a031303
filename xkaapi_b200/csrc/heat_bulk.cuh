// Bulk-staged heat tile body for the persistent scheduler (sm_100a).
//
// Each warp owns a ring of NBUF shared-memory column slots with one mbarrier per slot. To run a
// strip (32*VEC rows x a range of columns, as the register body splits a tile), lane 0 issues
// one bulk asynchronous copy (cp.async.bulk, global -> shared, completion counted in bytes on
// the slot's mbarrier) per source column -- the strip's rows plus the north/south halo row,
// widened to 16-byte boundaries -- keeping up to NBUF columns in flight ahead of the sweep. The
// lanes then sweep the columns west to east as the register body does: each lane reads its VEC
// cells of the next column from the slot, north/south neighbours come from the adjacent lanes by
// shuffle and, at the strip's ends, from the slot's halo rows; a slot is refilled with the column
// NBUF ahead as soon as every lane has read it.
//
// Compared with the register body the halo rows arrive in the same copy as the strip (no
// scalar halo loads), the bytes in flight cost shared memory instead of registers, and one
// instruction moves a whole column. The arithmetic is the register body's (heat_update), so
// results are identical. Measured on the 16384^2 FP64 graph (128^2 tiles) it moves 3.2 TB/s
// against the register body's 4.8 TB/s, with 8 or 16 slots per warp alike: one 544-byte copy
// per column is too small a unit; the scheduler keeps it as an opt-in body.
//
// Ordering: bulk copies read global memory through the async proxy. Tile data written by other
// tasks is published by their release / this task's acquire in the generic proxy, so lane 0
// issues fence.proxy.async before a strip's first copy; a slot read by the lanes (generic) is
// refilled by a copy (async) only after __syncwarp and fence.proxy.async.shared::cta.
//
// Every wait on an mbarrier is bounded (globaltimer); a wait that runs out reports failure,
// the strip drains its remaining copies (again bounded) and the caller records the error.
#pragma once
#include "heat.cuh"

namespace xkb {

// Slot size: the 32*VEC rows of a strip plus VEC rows on each side (16-byte widening of the
// one-row halos): 34*VEC elements = 544 bytes for both FP64 (VEC 2) and FP32 (VEC 4).
constexpr int BULK_SLOT_BYTES = 544;
constexpr int BULK_REFILL = 4;          // slots refilled together

__device__ __forceinline__ uint32_t smem_addr(const void * p) { return (uint32_t) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t * b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t * b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t * b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(smem_addr(b)), "r"(parity) : "memory");
    return ok != 0;
}

// Wait for the phase of `parity` to complete, until globaltimer passes `deadline`.
__device__ __forceinline__ bool mbar_wait(uint64_t * b, uint32_t parity, uint64_t deadline)
{
    for (uint32_t it = 0;; ++it)
    {
        if (mbar_try_wait(b, parity)) return true;
        if ((it & 63) == 63 && xkb_globaltimer() > deadline) return false;
    }
}

__device__ __forceinline__ void bulk_copy_g2s(void * dst, const void * src, uint32_t bytes, uint64_t * bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// A warp's staging ring: NBUF slots, their mbarriers, and the number of columns the warp has
// issued so far (slot = seq % NBUF, phase parity = (seq / NBUF) & 1).
template <int NBUF>
struct BulkRing {
    unsigned char * slots;       // NBUF * BULK_SLOT_BYTES, 128-byte aligned
    uint64_t * bars;             // NBUF
    uint32_t seq;
};

template <int NBUF>
__device__ __forceinline__ void bulk_ring_init(BulkRing<NBUF> & r)
{
    if ((threadIdx.x & 31) == 0)
    {
        for (int k = 0; k < NBUF; ++k) mbar_init(r.bars + k, 1);
        fence_mbar_init();
        fence_proxy_async_smem();
    }
    r.seq = 0;
    __syncwarp();
}

// Can the bulk body run this tile? Rows of every column must start on 16-byte boundaries and the
// 16-byte-widened halo rows must stay inside the grid rows.
template <typename T, int VEC>
__device__ __forceinline__ bool bulk_ok(const T * src, int64_t ld, int64_t nx)
{
    return ((uintptr_t) src % 16) == 0 && (ld * (int64_t) sizeof(T)) % 16 == 0 && nx % VEC == 0;
}

// One strip: rows [rbase, rbase + 32*VEC) intersected with [rx0, rx1), columns [cy0, cy1).
// Same preconditions as the register body; `bulk_ok` holds. Returns false when a wait ran out.
template <typename T, int VEC, int NBUF>
__device__ __noinline__ bool heat_strip_bulk(const T * __restrict__ src, T * __restrict__ dst, int64_t ld, int64_t rbase, int64_t rx0,
                                int64_t rx1, int64_t cy0, int64_t cy1, double c, BulkRing<NBUF> & ring, uint64_t deadline)
{
    static_assert(34 * VEC * sizeof(T) == BULK_SLOT_BYTES, "slot holds a strip and its widened halo rows");
    const int lane = threadIdx.x & 31;
    const int64_t w0 = rbase > rx0 ? rbase : rx0, w1 = rbase + 32 * VEC < rx1 ? rbase + 32 * VEC : rx1;
    if (w0 >= w1 || cy0 >= cy1) return true;
    const int64_t a0 = (w0 - 1) & ~(int64_t) (VEC - 1);                 // first row copied (>= 0: w0 >= 1)
    const int64_t b0 = (w1 + VEC) & ~(int64_t) (VEC - 1);               // one past the last (<= nx)
    const uint32_t bytes = (uint32_t) ((b0 - a0) * (int64_t) sizeof(T));
    const int off = (int) (rbase - a0);                                  // slot index of row rbase: 0 or VEC
    const int nrows = (int) (b0 - a0);
    const int n = (int) (cy1 - cy0) + 2;                                 // source columns cy0-1 .. cy1
    const int64_t r = rbase + (int64_t) lane * VEC;
    const bool lane_rows = r + VEC > w0 && r < w1;
    const bool full_store = r >= w0 && r + VEC <= w1;
    const uint32_t seq0 = ring.seq;
    const T * col0 = src + (cy0 - 1) * ld + a0;

    auto issue = [&](int q) {                                            // lane 0
        const uint32_t s = seq0 + (uint32_t) q, k = s % NBUF;
        mbar_expect_tx(ring.bars + k, bytes);
        bulk_copy_g2s(ring.slots + (size_t) k * BULK_SLOT_BYTES, col0 + (int64_t) q * ld, bytes, ring.bars + k);
    };
    if (lane == 0)
    {
        fence_proxy_async_all();
        for (int q = 0; q < n && q < NBUF; ++q) issue(q);
    }
    int next_issue = n < NBUF ? n : NBUF;                                // columns below it are issued
    int taken = 0;
    bool ok = true;
    // column q into registers: the lane's VEC cells and, for lanes 0 / 31, the halo rows
    auto take = [&](int q, Cells<T, VEC> & v, T & hn, T & hs) {
        const uint32_t s = seq0 + (uint32_t) q, k = s % NBUF;
        if (ok && !mbar_wait(ring.bars + k, (s / NBUF) & 1u, deadline)) ok = false;
        const T * p = (const T *) (ring.slots + (size_t) k * BULK_SLOT_BYTES);
        if (ok)
        {
            if constexpr (VEC == 2 && sizeof(T) == 8) {
                const double2 x = *(const double2 *) (p + off + lane * VEC);
                v.v[0] = x.x; v.v[1] = x.y;
            } else {
                const float4 x = *(const float4 *) (p + off + lane * VEC);
                v.v[0] = x.x; v.v[1] = x.y; v.v[2] = x.z; v.v[3] = x.w;
            }
            hn = (lane == 0 && off > 0) ? p[off - 1] : T(0);
            hs = (lane == 31 && off + 32 * VEC < nrows) ? p[off + 32 * VEC] : T(0);
        }
        __syncwarp();
        taken = q + 1;
        // refill the freed slots BULK_REFILL at a time (one proxy fence per refill)
        if (ok && (taken % BULK_REFILL == 0 || taken == n) && next_issue < n)
        {
            const int upto = taken + NBUF < n ? taken + NBUF : n;
            if (lane == 0)
            {
                fence_proxy_async_smem();
                for (int k = next_issue; k < upto; ++k) issue(k);
            }
            next_issue = upto;
        }
    };

    Cells<T, VEC> west, cur, east;
    T chn, chs, ehn, ehs, unused;
    take(0, west, unused, unused);
    take(1, cur, chn, chs);
    T * dp = dst + r;
    for (int q = 2; q < n && ok; ++q)
    {
        take(q, east, ehn, ehs);
        const int64_t jc = cy0 + q - 2;
        T north = __shfl_up_sync(0xffffffffu, cur.v[VEC - 1], 1);
        T south = __shfl_down_sync(0xffffffffu, cur.v[0], 1);
        if (lane == 0) north = chn;
        if (lane == 31) south = chs;
        if (ok && lane_rows)
        {
            Cells<T, VEC> out;
#pragma unroll
            for (int e = 0; e < VEC; ++e)
            {
                const double sv = (double) cur.v[e];
                const double up = (double) (e == 0 ? north : cur.v[e - 1]);
                const double dn = (double) (e == VEC - 1 ? south : cur.v[e + 1]);
                out.v[e] = (T) heat_update(sv, up, dn, (double) west.v[e], (double) east.v[e], c);
            }
            T * qd = dp + jc * ld;
            if (full_store)
            {
                if constexpr (VEC == 2 && sizeof(T) == 8) *(double2 *) qd = make_double2(out.v[0], out.v[1]);
                else *(float4 *) qd = make_float4(out.v[0], out.v[1], out.v[2], out.v[3]);
            }
            else
            {
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                    if (r + e >= w0 && r + e < w1) qd[e] = out.v[e];
            }
        }
        west = cur; cur = east; chn = ehn; chs = ehs;
    }
    if (!ok)
    {
        // drain the copies still in flight so that none lands after the kernel gives up
        const int issued = next_issue;
        const uint64_t drain = xkb_globaltimer() + 1000000000ull;
        for (int q = taken; q < issued; ++q)
        {
            const uint32_t s = seq0 + (uint32_t) q;
            mbar_wait(ring.bars + s % NBUF, (s / NBUF) & 1u, drain);
        }
    }
    ring.seq = seq0 + (uint32_t) n;
    return ok;
}

// A team of `nwarps` warps runs one tile task with the bulk body: the register body's split
// into strips, each warp taking strips round-robin with its own ring.
template <typename T, int VEC, int NBUF>
__device__ __forceinline__ bool heat_tile_team_bulk(const T * src, T * dst, int64_t ld, int64_t nx, int64_t ny, int64_t x0,
                                                    int64_t x1, int64_t y0, int64_t y1, double c, int warp, int nwarps,
                                                    BulkRing<NBUF> & ring, uint64_t deadline)
{
    const TileBox b = heat_tile_box(nx, ny, x0, x1, y0, y1);
    if (b.rx0 >= b.rx1 || b.cy0 >= b.cy1) return true;
    int64_t rbase0, cols_per; int nrg, ncg;
    heat_tile_split<VEC>(b, nwarps, rbase0, nrg, ncg, cols_per);
    bool ok = true;
    for (int s = warp; s < nrg * ncg && ok; s += nwarps)
    {
        const int rg = s % nrg, cg = s / nrg;
        const int64_t cy0 = b.cy0 + cg * cols_per;
        int64_t cy1 = cy0 + cols_per; if (cy1 > b.cy1) cy1 = b.cy1;
        if (cy0 >= cy1) continue;
        ok = heat_strip_bulk<T, VEC, NBUF>(src, dst, ld, rbase0 + (int64_t) rg * 32 * VEC, b.rx0, b.rx1, cy0, cy1, c, ring, deadline);
    }
    return ok;
}

} // namespace xkb
