// Batched dependency resolver for R/W/RW accesses on LD-strided matrices and segments.
//
// Semantics (what the reference's dependency domains compute; file:line in XKRT):
//  * per task: LINK every access, then PUT every access (src/task/task.cc:285-299);
//  * one interval domain for segments, one BLAS domain per (ld, sizeof) created by the first
//    matrix access naming it, during that task's LINK pass (src/task/task.cc:153-201); a
//    segment also goes to every BLAS domain that exists at that moment (:240-259), and a new
//    BLAS domain first replays the PUT of every earlier segment newest-first
//    (interval/dependency-tree.hpp:355-360 push_front, task.cc:177-198);
//  * frames: matrix tile -> 1-2 rects (byte row mod ld*s, column) (access.hpp:204-287);
//    segment -> [a, b) in the interval domain, 3 rects in a BLAS frame (access.hpp:76-139);
//    a segment's PUT in a BLAS domain only touches rows [a, b) of column 0 of that frame,
//    because BLAS on_insert tests the access's own rects, which a segment keeps in the
//    ld = SIZE_MAX frame (access.hpp:479-514, blas/dependency-tree.hpp:228-256);
//  * per point: LINK(A): W-mode A with readers -> edges from every reader, else edge from
//    the writer; PUT(A): W-mode -> writer = A, readers = {}; mode == R exactly -> readers += A
//    (blas/dependency-tree.hpp:295-355);
//  * handles: one DependencyMap per domain task (src/task/task.cc:226-236), a point per handle
//    with the same LINK/PUT except that any mode with R and without W is recorded as a reader
//    (handle/dependency-map.hpp:157-297; sequential and commutative accesses -- a stream with
//    concurrent ones is expanded first by xkb_handle_map_expand, handles.h).
//
// Method (B200): the host turns the accesses of a batch into each domain's ordered op list
// and keeps a coordinate compression of the domain (elementary cells between all rect
// boundaries seen so far). On the GPU one CTA owns a region of RX x RY cells: it streams the
// batch's ops, keeps those overlapping its region with a ballot + block prefix sum (order
// preserving), and each thread then applies the ops to its own cell's writer/readers state,
// emitting (pred, succ) pairs; lanes emitting the same pred for the same op are merged with
// __match_any_sync. A GPU hash set keeps the unique pairs; finalising counts predecessors,
// scans and scatters the pairs into a successor CSR. Cell state stays in HBM between batches.
#include "common.cuh"
#include "internal.h"
#include "scan.cuh"
#include "workpool.h"

#include <algorithm>
#include <climits>
#include <chrono>
#include <string>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <map>
#include <memory>
#include <new>
#include <thread>
#include <utility>
#include <vector>

namespace xkb {

constexpr uint8_t M_R = 1, M_W = 2;
constexpr int RES_CHUNK_PER_THREAD = 4;
constexpr unsigned long long EDGE_EMPTY = ~0ull;

struct DOp {            // one op in cell coordinates (24 bytes)
    int32_t task;
    uint8_t link;
    uint8_t mode;
    uint16_t pad;
    int32_t cx0, cx1, cy0, cy1;
};

// Cell state: writer, number of readers since that write, head and tail of the reader spill
// chain, and the first RCAP readers. Readers past RCAP go to chains of SPILL-int chunks
// (next chunk, then SPILL - 1 readers) drawn from one pool per resolver, so a cell can collect
// any number of readers (a region that is read every step and never written) while the state
// and the region kernel's shared memory stay small. Chunks of a chain that a write clears are
// not reused.
#ifndef XKB_REGION_RY
#define XKB_REGION_RY 8                 // cell rows of a 2-D region (8 columns each): 8 = two warps per CTA
#endif
constexpr int RCAP = 32;
constexpr int SHDR = 4;
constexpr int STRIDE = SHDR + RCAP;
constexpr int SPILL = 32;
constexpr int SPILL_R = SPILL - 1;

struct ResolveArgs {
    const DOp * ops;
    int nops;
    int ncx, ncy, nrx;
    const int * state_in;     // STRIDE ints per cell
    int * state_out;
    unsigned long long * emit;
    unsigned long long * emit_count;
    unsigned long long emit_cap;
    int * spill;              // chunk pool
    unsigned * spill_ctr;     // [0] chunks handed out, [1] set when the pool ran out
    unsigned spill_cap;       // chunks in the pool
};

// A fresh spill chunk (its next link cleared), or -1 with the out-of-pool flag set.
__device__ __forceinline__ int spill_alloc(int * spill, unsigned * ctr, unsigned cap)
{
    const unsigned c = atomicAdd(ctr, 1u);
    if (c >= cap) { atomicExch(ctr + 1, 1u); return -1; }
    spill[(size_t) c * SPILL] = -1;
    return (int) c;
}

// Pairs are staged per warp in shared memory and appended to a.emit EMIT_BUF - 32 or more at a
// time, with one atomic on the batch's counter per flush instead of one per emitting step.
constexpr int EMIT_BUF = 256;

// Append this warp's n staged pairs to a.emit (coalesced); every lane of the warp calls it.
__device__ __forceinline__ void emit_flush(const ResolveArgs & a, const unsigned long long * buf, int n, int lane)
{
    __syncwarp();
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(a.emit_count, (unsigned long long) n);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (int j = lane; j < n; j += 32)
        if (base + j < a.emit_cap) a.emit[base + j] = buf[j];
    __syncwarp();
}

// BINNED: the CTA's ops come from its region's list (op indices in op order, built by the
// binning kernels below) instead of a scan of every op of the batch.
template <int RX, int RY, bool BINNED>
__global__ void __launch_bounds__(RX * RY)
resolve_region_kernel(ResolveArgs a, const unsigned * __restrict__ roff, const int * __restrict__ rlist)
{
    constexpr int NT = RX * RY;
    constexpr int NW = NT / 32;
    constexpr int CHUNK = NT * RES_CHUNK_PER_THREAD;
    extern __shared__ int rd[];                  // readers: rd[k * NT + tid]
    __shared__ DOp list[CHUNK];
    __shared__ int wcount[NW];
    __shared__ int nlist_s;
    __shared__ unsigned long long ebuf[NW][EMIT_BUF];   // each warp's pairs not yet in a.emit

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rx = blockIdx.x % a.nrx, ry = blockIdx.x / a.nrx;
    const int gx0 = rx * RX, gy0 = ry * RY;
    const int gx1 = min(gx0 + RX, a.ncx), gy1 = min(gy0 + RY, a.ncy);
    const int cx = gx0 + tid % RX, cy = gy0 + tid / RX;
    const bool valid = cx < a.ncx && cy < a.ncy;
    const size_t cell = valid ? (size_t) cy * a.ncx + cx : 0;

    int writer = -1, nr = 0, head = -1, tail = -1;
    int nbuf = 0;                                // pairs in this warp's ebuf (same in every lane)
    if (valid)
    {
        const int * st = a.state_in + cell * STRIDE;
        writer = st[0]; nr = st[1]; head = st[2]; tail = st[3];
        for (int k = 0; k < nr && k < RCAP; ++k) rd[k * NT + tid] = st[SHDR + k];
    }

    const int lo = BINNED ? (int) roff[blockIdx.x] : 0, hi = BINNED ? (int) roff[blockIdx.x + 1] : a.nops;
    for (int base = lo; base < hi; base += CHUNK)
    {
        if constexpr (BINNED)
        {
            // ---- gather the next CHUNK ops of this region's list (already in op order) -----
            for (int j = tid; j < CHUNK && base + j < hi; j += NT) list[j] = a.ops[rlist[base + j]];
            if (tid == 0) nlist_s = min(CHUNK, hi - base);
            __syncthreads();
        }
        else
        {
        // ---- compact the ops of this chunk that overlap the region, in op order ----------
        if (tid == 0) nlist_s = 0;
        __syncthreads();
        for (int j = 0; j < RES_CHUNK_PER_THREAD; ++j)
        {
            const int idx = base + j * NT + tid;
            DOp op;
            bool hit = false;
            if (idx < a.nops)
            {
                op = a.ops[idx];
                hit = op.cx0 < gx1 && gx0 < op.cx1 && op.cy0 < gy1 && gy0 < op.cy1;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) wcount[warp] = __popc(bal);
            __syncthreads();
            int off = nlist_s;
            for (int w = 0; w < warp; ++w) off += wcount[w];
            if (hit) list[off + __popc(bal & ((1u << lane) - 1))] = op;
            __syncthreads();
            if (tid == 0) { int t = 0; for (int w = 0; w < NW; ++w) t += wcount[w]; nlist_s += t; }
            __syncthreads();
        }
        }
        const int nlist = nlist_s;

        // ---- apply them to this thread's cell -----------------------------------------------
        for (int k = 0; k < nlist; ++k)
        {
            const DOp op = list[k];
            const bool in = valid && op.cx0 <= cx && cx < op.cx1 && op.cy0 <= cy && cy < op.cy1;
            if (op.link)
            {
                const bool from_readers = in && (op.mode & M_W) && nr > 0;
                const int cnt = from_readers ? nr : ((in && writer >= 0) ? 1 : 0);
                const int maxcnt = __reduce_max_sync(0xffffffffu, cnt);
                int chunk = head, ci = 0;                // walk of the spill chain past RCAP
                for (int q = 0; q < maxcnt; ++q)
                {
                    int p = -1;
                    if (q < cnt)
                    {
                        if (!from_readers) p = writer;
                        else if (q < RCAP) p = rd[q * NT + tid];
                        else
                        {
                            if (ci == SPILL_R) { chunk = chunk >= 0 ? a.spill[(size_t) chunk * SPILL] : -1; ci = 0; }
                            p = chunk >= 0 ? a.spill[(size_t) chunk * SPILL + 1 + ci] : -1;   // -1: pool ran out, batch redone
                            ++ci;
                        }
                    }
                    const unsigned peers = __match_any_sync(0xffffffffu, p);
                    const bool leader = p >= 0 && lane == __ffs(peers) - 1;
                    const unsigned em = __ballot_sync(0xffffffffu, leader);
                    if (leader)
                        ebuf[warp][nbuf + __popc(em & ((1u << lane) - 1))] = ((unsigned long long) (uint32_t) p << 32) | (uint32_t) op.task;
                    nbuf += __popc(em);
                    if (nbuf > EMIT_BUF - 32) { emit_flush(a, ebuf[warp], nbuf, lane); nbuf = 0; }
                }
            }
            else if (in)
            {
                if (op.mode & M_W) { writer = op.task; nr = 0; head = tail = -1; }
                else if (op.mode == M_R)
                {
                    if (nr < RCAP) rd[nr * NT + tid] = op.task;
                    else
                    {
                        const int slot = (nr - RCAP) % SPILL_R;
                        if (slot == 0)
                        {
                            const int c = spill_alloc(a.spill, a.spill_ctr, a.spill_cap);
                            if (c >= 0) { if (tail >= 0) a.spill[(size_t) tail * SPILL] = c; else head = c; }
                            tail = c;
                        }
                        if (tail >= 0) a.spill[(size_t) tail * SPILL + 1 + slot] = op.task;
                    }
                    ++nr;
                }
            }
        }
        __syncthreads();
    }

    if (nbuf) emit_flush(a, ebuf[warp], nbuf, lane);
    if (valid)
    {
        int * st = a.state_out + cell * STRIDE;
        st[0] = writer; st[1] = nr; st[2] = head; st[3] = tail;
        for (int k = 0; k < nr && k < RCAP; ++k) st[SHDR + k] = rd[k * NT + tid];
    }
}

// ---- time-split resolution of a region ---------------------------------------------------------
// A region's op list is cut into nseg segments (cut s at lo + (hi - lo) * s / nseg). The cell
// state before each cut is all a segment needs to emit its edges, and only PUT ops change the
// state, so:
//  * resolve_puts_kernel (one CTA per region) applies the PUT ops of the whole list -- the
//    cheap half of the work -- writing the state before every cut to `snap` and the final state
//    to state_out; it owns the reader spill chains, exactly as resolve_region_kernel does;
//  * resolve_links_kernel (one CTA per region and segment, nseg times the CTAs) replays its
//    segment from that state: PUT ops update a private copy of the state and LINK ops emit
//    the edges. Readers past RCAP that were in the state at the cut are read from the chain the
//    snapshot names (resolve_puts_kernel only ever appends to a chain past the snapshot's count,
//    and a write drops a chain without reusing it, so the first nr entries stay as they were);
//    readers the segment itself adds past RCAP go to a private chain (chunks from the same pool,
//    never linked into the kept state).
// The edges are those of resolve_region_kernel over the whole list (the same LINK ops see the
// same states); only the order in which pairs reach a.emit differs, which the dedupe ignores.

__device__ __forceinline__ int seg_cut(int lo, int hi, int s, int nseg)
{
    return lo + (int) ((long long) (hi - lo) * s / nseg);
}

template <int RX, int RY>
__global__ void __launch_bounds__(RX * RY)
resolve_puts_kernel(ResolveArgs a, const unsigned * __restrict__ roff, const int * __restrict__ rlist, int nseg,
                    int * __restrict__ snap, size_t ncells)
{
    constexpr int NT = RX * RY;
    constexpr int CHUNK = NT * RES_CHUNK_PER_THREAD;
    extern __shared__ int rd[];                  // readers: rd[k * NT + tid]
    __shared__ DOp list[CHUNK];

    const int tid = threadIdx.x;
    const int rx = blockIdx.x % a.nrx, ry = blockIdx.x / a.nrx;
    const int cx = rx * RX + tid % RX, cy = ry * RY + tid / RX;
    const bool valid = cx < a.ncx && cy < a.ncy;
    const size_t cell = valid ? (size_t) cy * a.ncx + cx : 0;

    int writer = -1, nr = 0, head = -1, tail = -1;
    if (valid)
    {
        const int * st = a.state_in + cell * STRIDE;
        writer = st[0]; nr = st[1]; head = st[2]; tail = st[3];
        for (int k = 0; k < nr && k < RCAP; ++k) rd[k * NT + tid] = st[SHDR + k];
    }
    auto snapshot = [&](int s) {
        if (!valid) return;
        int * st = snap + ((size_t) (s - 1) * ncells + cell) * STRIDE;
        st[0] = writer; st[1] = nr; st[2] = head; st[3] = tail;
        for (int k = 0; k < nr && k < RCAP; ++k) st[SHDR + k] = rd[k * NT + tid];
    };

    const int lo = (int) roff[blockIdx.x], hi = (int) roff[blockIdx.x + 1];
    int seg = 1, cut = nseg > 1 ? seg_cut(lo, hi, 1, nseg) : INT_MAX;
    for (int base = lo; base < hi; base += CHUNK)
    {
        const int n = min(CHUNK, hi - base);
        for (int j = tid; j < n; j += NT) list[j] = a.ops[rlist[base + j]];
        __syncthreads();
        for (int k = 0; k < n; ++k)
        {
            while (base + k == cut) { snapshot(seg); ++seg; cut = seg < nseg ? seg_cut(lo, hi, seg, nseg) : INT_MAX; }
            const DOp op = list[k];
            if (op.link) continue;
            const bool in = valid && op.cx0 <= cx && cx < op.cx1 && op.cy0 <= cy && cy < op.cy1;
            if (!in) continue;
            if (op.mode & M_W) { writer = op.task; nr = 0; head = tail = -1; }
            else if (op.mode == M_R)
            {
                if (nr < RCAP) rd[nr * NT + tid] = op.task;
                else
                {
                    const int slot = (nr - RCAP) % SPILL_R;
                    if (slot == 0)
                    {
                        const int c = spill_alloc(a.spill, a.spill_ctr, a.spill_cap);
                        if (c >= 0) { if (tail >= 0) a.spill[(size_t) tail * SPILL] = c; else head = c; }
                        tail = c;
                    }
                    if (tail >= 0) a.spill[(size_t) tail * SPILL + 1 + slot] = op.task;
                }
                ++nr;
            }
        }
        __syncthreads();
    }
    while (seg < nseg) { snapshot(seg); ++seg; }          // cuts at the end of the list
    if (valid)
    {
        int * st = a.state_out + cell * STRIDE;
        st[0] = writer; st[1] = nr; st[2] = head; st[3] = tail;
        for (int k = 0; k < nr && k < RCAP; ++k) st[SHDR + k] = rd[k * NT + tid];
    }
}

template <int RX, int RY>
__global__ void __launch_bounds__(RX * RY)
resolve_links_kernel(ResolveArgs a, const unsigned * __restrict__ roff, const int * __restrict__ rlist, int nseg,
                     const int * __restrict__ snap, size_t ncells)
{
    constexpr int NT = RX * RY;
    constexpr int NW = NT / 32;
    constexpr int CHUNK = NT * RES_CHUNK_PER_THREAD;
    extern __shared__ int rd[];
    __shared__ DOp list[CHUNK];
    __shared__ unsigned long long ebuf[NW][EMIT_BUF];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int region = blockIdx.x / nseg, s = blockIdx.x % nseg;
    const int rx = region % a.nrx, ry = region / a.nrx;
    const int cx = rx * RX + tid % RX, cy = ry * RY + tid / RX;
    const bool valid = cx < a.ncx && cy < a.ncy;
    const size_t cell = valid ? (size_t) cy * a.ncx + cx : 0;

    int writer = -1, nr = 0, shead = -1;
    if (valid)
    {
        const int * st = s == 0 ? a.state_in + cell * STRIDE : snap + ((size_t) (s - 1) * ncells + cell) * STRIDE;
        writer = st[0]; nr = st[1]; shead = st[2];
        for (int k = 0; k < nr && k < RCAP; ++k) rd[k * NT + tid] = st[SHDR + k];
    }
    int nsnap = nr;                              // readers [RCAP, nsnap) are on the snapshot's chain
    int phead = -1, ptail = -1;                  // readers the segment adds past RCAP
    int nbuf = 0;

    const int lo = (int) roff[region], hi = (int) roff[region + 1];
    const int from = seg_cut(lo, hi, s, nseg), to = seg_cut(lo, hi, s + 1, nseg);
    for (int base = from; base < to; base += CHUNK)
    {
        const int n = min(CHUNK, to - base);
        for (int j = tid; j < n; j += NT) list[j] = a.ops[rlist[base + j]];
        __syncthreads();
        for (int k = 0; k < n; ++k)
        {
            const DOp op = list[k];
            const bool in = valid && op.cx0 <= cx && cx < op.cx1 && op.cy0 <= cy && cy < op.cy1;
            const int pbase = max(RCAP, nsnap);  // first reader position on the private chain
            if (op.link)
            {
                const bool from_readers = in && (op.mode & M_W) && nr > 0;
                const int cnt = from_readers ? nr : ((in && writer >= 0) ? 1 : 0);
                const int maxcnt = __reduce_max_sync(0xffffffffu, cnt);
                int chunk = shead, ci = 0;
                for (int q = 0; q < maxcnt; ++q)
                {
                    int p = -1;
                    if (q < cnt)
                    {
                        if (!from_readers) p = writer;
                        else if (q < RCAP) p = rd[q * NT + tid];
                        else
                        {
                            if (q == pbase) { chunk = phead; ci = 0; }
                            else if (ci == SPILL_R) { chunk = chunk >= 0 ? a.spill[(size_t) chunk * SPILL] : -1; ci = 0; }
                            p = chunk >= 0 ? a.spill[(size_t) chunk * SPILL + 1 + ci] : -1;   // -1: pool ran out, batch redone
                            ++ci;
                        }
                    }
                    const unsigned peers = __match_any_sync(0xffffffffu, p);
                    const bool leader = p >= 0 && lane == __ffs(peers) - 1;
                    const unsigned em = __ballot_sync(0xffffffffu, leader);
                    if (leader)
                        ebuf[warp][nbuf + __popc(em & ((1u << lane) - 1))] = ((unsigned long long) (uint32_t) p << 32) | (uint32_t) op.task;
                    nbuf += __popc(em);
                    if (nbuf > EMIT_BUF - 32) { emit_flush(a, ebuf[warp], nbuf, lane); nbuf = 0; }
                }
            }
            else if (in)
            {
                if (op.mode & M_W) { writer = op.task; nr = 0; nsnap = 0; phead = ptail = -1; }
                else if (op.mode == M_R)
                {
                    if (nr < RCAP) rd[nr * NT + tid] = op.task;
                    else
                    {
                        const int slot = (nr - pbase) % SPILL_R;
                        if (slot == 0)
                        {
                            const int c = spill_alloc(a.spill, a.spill_ctr, a.spill_cap);
                            if (c >= 0) { if (ptail >= 0) a.spill[(size_t) ptail * SPILL] = c; else phead = c; }
                            ptail = c;
                        }
                        if (ptail >= 0) a.spill[(size_t) ptail * SPILL + 1 + slot] = op.task;
                    }
                    ++nr;
                }
            }
        }
        __syncthreads();
    }
    if (nbuf) emit_flush(a, ebuf[warp], nbuf, lane);
}

// ---- binning of ops to regions ----------------------------------------------------------------
// The regions of an op: the RX x RY cell blocks its cell rect overlaps.
__global__ void bin_count_kernel(const DOp * __restrict__ ops, int nops, int RX, int RY, int nrx, unsigned * rcount)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nops) return;
    const DOp o = ops[i];
    if (o.cx0 >= o.cx1 || o.cy0 >= o.cy1) return;
    for (int ry = o.cy0 / RY; ry <= (o.cy1 - 1) / RY; ++ry)
        for (int rx = o.cx0 / RX; rx <= (o.cx1 - 1) / RX; ++rx)
            atomicAdd(rcount + ry * nrx + rx, 1u);
}

__global__ void bin_fill_kernel(const DOp * __restrict__ ops, int nops, int RX, int RY, int nrx, const unsigned * __restrict__ roff,
                                unsigned * cursor, int * list)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nops) return;
    const DOp o = ops[i];
    if (o.cx0 >= o.cx1 || o.cy0 >= o.cy1) return;
    for (int ry = o.cy0 / RY; ry <= (o.cy1 - 1) / RY; ++ry)
        for (int rx = o.cx0 / RX; rx <= (o.cx1 - 1) / RX; ++rx)
        {
            const int r = ry * nrx + rx;
            list[roff[r] + atomicAdd(cursor + r, 1u)] = i;
        }
}

// Block-local binning: with at most BIN_SMEM_REGIONS regions, a block of the count / fill kernels
// counts its ops' regions in shared memory and touches each region's global counter once (the
// kernels above do one global atomic per (op, region) on a few hundred shared counters).
constexpr int BIN_SMEM_REGIONS = 12288;

__global__ void bin_count_smem_kernel(const DOp * __restrict__ ops, int nops, int RX, int RY, int nrx, int nregions,
                                      unsigned * rcount)
{
    extern __shared__ unsigned h[];
    for (int r = threadIdx.x; r < nregions; r += blockDim.x) h[r] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += gridDim.x * blockDim.x)
    {
        const DOp o = ops[i];
        if (o.cx0 >= o.cx1 || o.cy0 >= o.cy1) continue;
        for (int ry = o.cy0 / RY; ry <= (o.cy1 - 1) / RY; ++ry)
            for (int rx = o.cx0 / RX; rx <= (o.cx1 - 1) / RX; ++rx)
                atomicAdd(h + ry * nrx + rx, 1u);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nregions; r += blockDim.x)
        if (h[r]) atomicAdd(rcount + r, h[r]);
}

// Each block counts its own ops' regions, reserves one range per region with one global atomic,
// and places its ops inside its ranges (any op-to-block split works: each region's list is put
// back in op order afterwards).
__global__ void bin_fill_smem_kernel(const DOp * __restrict__ ops, int nops, int RX, int RY, int nrx, int nregions,
                                     const unsigned * __restrict__ roff, unsigned * cursor, int * list)
{
    extern __shared__ unsigned h[];                       // [nregions] counts, then [nregions] bases
    unsigned * base = h + nregions;
    for (int r = threadIdx.x; r < nregions; r += blockDim.x) h[r] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += gridDim.x * blockDim.x)
    {
        const DOp o = ops[i];
        if (o.cx0 >= o.cx1 || o.cy0 >= o.cy1) continue;
        for (int ry = o.cy0 / RY; ry <= (o.cy1 - 1) / RY; ++ry)
            for (int rx = o.cx0 / RX; rx <= (o.cx1 - 1) / RX; ++rx)
                atomicAdd(h + ry * nrx + rx, 1u);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nregions; r += blockDim.x)
    {
        base[r] = h[r] ? roff[r] + atomicAdd(cursor + r, h[r]) : 0u;
        h[r] = 0;
    }
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nops; i += gridDim.x * blockDim.x)
    {
        const DOp o = ops[i];
        if (o.cx0 >= o.cx1 || o.cy0 >= o.cy1) continue;
        for (int ry = o.cy0 / RY; ry <= (o.cy1 - 1) / RY; ++ry)
            for (int rx = o.cx0 / RX; rx <= (o.cx1 - 1) / RX; ++rx)
            {
                const int r = ry * nrx + rx;
                list[base[r] + atomicAdd(h + r, 1u)] = i;
            }
    }
}

constexpr int MAX_SEGMENTS = 8;              // time-split segments per region (resolve_links_kernel)
constexpr int BIN_SORT_THREADS = 1024;
constexpr int BIN_SORT_CAP = 16384;          // ops of one region sortable in one CTA (64 KB of shared memory)

// Put each region's list back in op order (the fill appends in arbitrary order): bitonic sort of
// the region's segment in shared memory. A region holding more than BIN_SORT_CAP ops sets
// *too_long and the batch falls back to the unbinned scan.
__global__ void __launch_bounds__(BIN_SORT_THREADS) bin_sort_kernel(const unsigned * __restrict__ roff, int * list, int * too_long)
{
    extern __shared__ int keys[];
    const unsigned b = roff[blockIdx.x], e = roff[blockIdx.x + 1];
    const int n = (int) (e - b);
    if (n <= 1) return;
    if (n > BIN_SORT_CAP) { if (threadIdx.x == 0) atomicExch(too_long, 1); return; }
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) keys[i] = i < n ? list[b + i] : 0x7fffffff;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1)
        {
            for (int i = threadIdx.x; i < p2; i += blockDim.x)
            {
                const int l = i ^ j;
                if (l > i)
                {
                    const int x = keys[i], y = keys[l];
                    if (((i & k) == 0) == (x > y)) { keys[i] = y; keys[l] = x; }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < n; i += blockDim.x) list[b + i] = keys[i];
}

// New compression refines the old one: every new cell lies inside exactly one old cell (or
// outside the old domain, where the state is empty).
// Every new cell takes the state of the old cell it lies in; a spill chain is copied into fresh
// chunks, since several new cells can come from one old cell and each appends on its own.
__global__ void refine_state_kernel(const int * __restrict__ old_state, int * __restrict__ new_state,
                                    const int * __restrict__ map_x, const int * __restrict__ map_y, int ncx, int ncy, int old_ncx,
                                    int * spill, unsigned * spill_ctr, unsigned spill_cap)
{
    const size_t cell = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= (size_t) ncx * ncy) return;
    const int cx = (int) (cell % ncx), cy = (int) (cell / ncx);
    const int ox = map_x[cx], oy = map_y[cy];
    int * dst = new_state + cell * STRIDE;
    if (ox < 0 || oy < 0) { dst[0] = -1; dst[1] = 0; dst[2] = -1; dst[3] = -1; return; }
    const int * src = old_state + ((size_t) oy * old_ncx + ox) * STRIDE;
    const int n = src[1];
    dst[0] = src[0]; dst[1] = n;
    for (int k = 0; k < n && k < RCAP; ++k) dst[SHDR + k] = src[SHDR + k];
    int head = -1, tail = -1;
    int from = src[2];
    for (int left = n - RCAP; left > 0 && from >= 0; left -= SPILL_R)
    {
        const int c = spill_alloc(spill, spill_ctr, spill_cap);
        if (c < 0) { head = tail = -1; break; }                 // pool ran out: redone after growing
        for (int k = 1; k < SPILL; ++k) spill[(size_t) c * SPILL + k] = spill[(size_t) from * SPILL + k];
        if (tail >= 0) spill[(size_t) tail * SPILL] = c; else head = c;
        tail = c;
        from = spill[(size_t) from * SPILL];
    }
    dst[2] = head; dst[3] = tail;
}

__global__ void init_state_kernel(int * state, size_t ncells)
{
    const size_t cell = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (cell < ncells) { int * st = state + cell * STRIDE; st[0] = -1; st[1] = 0; st[2] = -1; st[3] = -1; }
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long k)
{
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
    return k;
}

__global__ void dedupe_kernel(const unsigned long long * __restrict__ emit, size_t n, unsigned long long * table,
                              unsigned long long mask, unsigned long long * uniq, unsigned long long * nuniq,
                              unsigned long long uniq_cap)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long key = emit[i];
    unsigned long long h = mix64(key) & mask;
    bool fresh = false;
    for (unsigned long long probe = 0; probe <= mask; ++probe)
    {
        const unsigned long long prev = atomicCAS(table + h, EDGE_EMPTY, key);
        if (prev == EDGE_EMPTY) { fresh = true; break; }
        if (prev == key) break;
        h = (h + 1) & mask;
    }
    // one atomic per warp on the shared counter for the warp's new pairs
    const unsigned act = __activemask();
    const unsigned nb = __ballot_sync(act, fresh);
    if (!nb) return;
    const int lane = threadIdx.x & 31, first = __ffs(nb) - 1;
    unsigned long long base = 0;
    if (lane == first) base = atomicAdd(nuniq, (unsigned long long) __popc(nb));
    base = __shfl_sync(act, base, first);
    if (fresh)
    {
        const unsigned long long s = base + __popc(nb & ((1u << lane) - 1));
        if (s < uniq_cap) uniq[s] = key;
    }
}

__global__ void count_edges_kernel(const unsigned long long * __restrict__ e, size_t n, uint32_t * nsucc, uint32_t * npred)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = e[i];
    atomicAdd(nsucc + (uint32_t) (k >> 32), 1u);
    atomicAdd(npred + (uint32_t) k, 1u);
}

__global__ void scatter_edges_kernel(const unsigned long long * __restrict__ e, size_t n, uint32_t * cursor, uint32_t * succ)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = e[i];
    const uint32_t pos = atomicAdd(cursor + (uint32_t) (k >> 32), 1u);
    succ[pos] = (uint32_t) k;
}

// A window of the graph: edges whose ends are both >= first, renumbered from first.
__global__ void count_window_edges_kernel(const unsigned long long * __restrict__ e, size_t n, uint32_t first, uint32_t * nsucc,
                                          uint32_t * npred)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = e[i];
    const uint32_t p = (uint32_t) (k >> 32), q = (uint32_t) k;
    if (p < first || q < first) return;
    atomicAdd(nsucc + (p - first), 1u);
    atomicAdd(npred + (q - first), 1u);
}

__global__ void scatter_window_edges_kernel(const unsigned long long * __restrict__ e, size_t n, uint32_t first, uint32_t * cursor,
                                            uint32_t * succ)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = e[i];
    const uint32_t p = (uint32_t) (k >> 32), q = (uint32_t) k;
    if (p < first || q < first) return;
    succ[atomicAdd(cursor + (p - first), 1u)] = q - first;
}

// Sort each successor list ascending (deterministic CSR). Short lists: one thread, insertion sort.
__global__ void sort_segments_kernel(const uint32_t * __restrict__ ptr, uint32_t * succ, uint32_t ntasks)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntasks) return;
    const uint32_t b = ptr[t], e = ptr[t + 1];
    for (uint32_t i = b + 1; i < e; ++i)
    {
        const uint32_t v = succ[i];
        uint32_t j = i;
        while (j > b && succ[j - 1] > v) { succ[j] = succ[j - 1]; --j; }
        succ[j] = v;
    }
}

// ------------------------------------------------------------------------------------------
// host side

struct HRect { uint64_t x0, x1, y0, y1; };
struct HOp { uint32_t task; uint8_t link; uint8_t mode; HRect r; };

static size_t g_realloc_bytes = 0;               // device bytes allocated by reserve (trace)

// Device memory pool of the resolver's work buffers on the current device (made on first use).
// Buffers only the resolver's own stream touches are allocated from it in stream order, so
// growing one neither waits for the whole device (as cudaFree does) nor asks the driver for
// memory while copies and kernels of other streams run: a runtime streaming windows of tasks
// had its resolution stall for up to 0.3 s in cudaMalloc / cudaFree of a domain's cell states.
// Freed memory stays in the pool for the next resolver of the process, up to 4 GiB
// (XKB_POOL_CACHE=0: none).
static cudaMemPool_t resolver_pool()
{
    static std::mutex mu;
    static cudaMemPool_t pools[256];
    static bool made[256];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) { cudaGetLastError(); return nullptr; }
    std::lock_guard<std::mutex> lk(mu);
    if (!made[dev])
    {
        made[dev] = true;
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (cudaMemPoolCreate(&pools[dev], &props) != cudaSuccess) { cudaGetLastError(); pools[dev] = nullptr; }
        else
        {
            const char * e = getenv("XKB_POOL_CACHE");
            uint64_t keep = (e && atoi(e) == 0) ? 0 : (uint64_t(4) << 30);
            cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    return pools[dev];
}

template <typename T>
struct DevBuf {
    T * p = nullptr;
    size_t cap = 0;
    cudaStream_t st = nullptr;       // pooled: the one stream that uses the buffer
    bool pooled = false;
    ~DevBuf()
    {
        if (!p) return;
        if (!pooled) cudaFree(p);
        else if (cudaFreeAsync(p, st) != cudaSuccess) { cudaGetLastError(); cudaFree(p); }
    }
    // Allocate from the resolver's pool in the order of `s` (before the first allocation only).
    void use_pool(cudaStream_t s)
    {
        if (p) return;
        pooled = resolver_pool() != nullptr;
        st = s;
    }
    int reserve(size_t n)
    {
        if (n <= cap) return XKB_OK;
        size_t c = cap ? cap : 1024;
        while (c < n) c *= 2;
        T * q = nullptr;
        g_realloc_bytes += c * sizeof(T);
        if (pooled)
        {
            cudaError_t e = cudaMallocFromPoolAsync((void **) &q, c * sizeof(T), resolver_pool(), st);
            if (e != cudaSuccess) return xkb_set_cuda_error(e);
            if (p) cudaFreeAsync(p, st);      // after the stream's work queued so far
        }
        else
        {
            cudaError_t e = cudaMalloc(&q, c * sizeof(T));
            if (e != cudaSuccess) return xkb_set_cuda_error(e);
            if (p) cudaFree(p);
        }
        p = q; cap = c;
        return XKB_OK;
    }
};

// ---- coordinate compression on the device ----------------------------------------------------
// Every op's rect boundaries go into two open-addressing hash sets (x and y); each first insert
// appends the key to a compact list, so the host only sorts the distinct boundaries of the batch.
// The tables hold at least twice as many slots as keys can be inserted, so a probe always ends at
// an empty slot. Slots only ever change from empty to a key, so a stale read sees empty at worst
// and the CAS settles it. The key ~0 (the empty marker) is reported through a flag bit instead.
constexpr uint64_t KEY_EMPTY = ~0ull;

__device__ __forceinline__ void hset_insert(uint64_t * tab, uint32_t mask, uint64_t key, uint64_t * out, unsigned * count,
                                            unsigned * flags, unsigned max_bit)
{
    if (key == KEY_EMPTY) { atomicOr(flags, max_bit); return; }
    uint32_t h = (uint32_t) ((key * 0x9e3779b97f4a7c15ull) >> 32) & mask;
    for (;;)
    {
        const uint64_t v = *(volatile uint64_t *) (tab + h);
        if (v == key) return;
        if (v == KEY_EMPTY)
        {
            const uint64_t prev = atomicCAS((unsigned long long *) (tab + h), (unsigned long long) KEY_EMPTY,
                                            (unsigned long long) key);
            if (prev == KEY_EMPTY) { out[atomicAdd(count, 1u)] = key; return; }
            if (prev == key) return;
        }
        h = (h + 1) & mask;
    }
}

// counts[0] / counts[1]: distinct x / y keys appended; counts[2]: bit 1 / 2 when ~0 was an x / y key
__global__ void collect_bounds_kernel(const HOp * __restrict__ ops, int n, uint64_t * tx, uint64_t * ty, uint32_t mask,
                                      uint64_t * ux, uint64_t * uy, unsigned * counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const HRect r = ops[i].r;
    // neighbouring ops mostly share their boundaries (tiles of one grid): one lane per distinct
    // key of the warp probes the table
    const unsigned act = __activemask(), lane = threadIdx.x & 31;
    auto once = [&](uint64_t key, uint64_t * tab, uint64_t * out, unsigned * count, unsigned bit) {
        const unsigned same = __match_any_sync(act, key);
        if ((unsigned) (__ffs(same) - 1) == lane) hset_insert(tab, mask, key, out, count, counts + 2, bit);
    };
    once(r.x0, tx, ux, counts + 0, 1u);
    once(r.x1, tx, ux, counts + 0, 1u);
    once(r.y0, ty, uy, counts + 1, 2u);
    once(r.y1, ty, uy, counts + 1, 2u);
}

__device__ __forceinline__ int32_t lower_index(const uint64_t * __restrict__ v, int n, uint64_t key)
{
    int lo = 0, hi = n;
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (__ldg(v + mid) < key) lo = mid + 1; else hi = mid; }
    return lo;
}

// Ops in cell coordinates: each boundary's index in the domain's sorted boundary lists.
__global__ void map_ops_kernel(const HOp * __restrict__ ops, int n, const uint64_t * __restrict__ xs, int nxs,
                               const uint64_t * __restrict__ ys, int nys, DOp * out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const HOp o = ops[i];
    DOp q;
    q.task = (int32_t) o.task; q.link = o.link; q.mode = o.mode; q.pad = 0;
    q.cx0 = lower_index(xs, nxs, o.r.x0); q.cx1 = lower_index(xs, nxs, o.r.x1);
    q.cy0 = lower_index(ys, nys, o.r.y0); q.cy1 = lower_index(ys, nys, o.r.y1);
    out[i] = q;
}

struct Domain {
    bool interval = false;
    uint64_t ld = 0, s = 0;
    std::vector<uint64_t> xs, ys;       // compression (sorted unique boundaries)
    DevBuf<int> state[2];
    int cur = 0;
    size_t ncells = 0;
    std::vector<HOp> ops;               // ops of the batch being resolved (sequential build)
    size_t nops = 0;                    // ops of the batch (in `ops`, or in the staging buffer)
    size_t stage_off = 0;               // where they start in the staging buffer
};

// Page-locked host memory the parallel build writes the batch's ops into, reused batch after
// batch, so their upload runs at DMA speed.
struct HostStage {
    HOp * p = nullptr;
    size_t cap = 0;
    HostStage() = default;
    HostStage(const HostStage &) = delete;
    HostStage & operator=(const HostStage &) = delete;
    ~HostStage() { if (p) cudaFreeHost(p); }
    int reserve(size_t n)
    {
        if (n <= cap) return XKB_OK;
        size_t c = cap ? cap : size_t(1) << 20;
        while (c < n) c *= 2;
        HOp * q = nullptr;
        cudaError_t e = cudaHostAlloc((void **) &q, c * sizeof(HOp), cudaHostAllocDefault);
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        if (p) cudaFreeHost(p);
        p = q; cap = c;
        return XKB_OK;
    }
};

} // namespace xkb

using namespace xkb;

struct xkb_resolver {
    cudaStream_t stream = nullptr;
    Domain interval;
    Domain handles;                             // handle accesses: one point per handle
    std::vector<std::unique_ptr<Domain>> blas;
    std::map<std::pair<uint64_t, uint64_t>, size_t> blas_index;
    std::vector<xkb_access_rec_t> segments;     // every segment so far, spawn order (replay)
    uint32_t ntasks = 0;
    // device work buffers
    DevBuf<DOp> dops;
    DevBuf<HOp> hops;                           // the batch's ops in byte coordinates
    DevBuf<uint64_t> hset, ukeys, bounds;       // compression: hash sets, distinct keys, sorted boundaries
    DevBuf<unsigned> ucount;
    DevBuf<unsigned long long> emit, table;
    // unique edges, appended batch by batch into segments (a batch's edges all end in the
    // batch's own tasks, so batches never repeat each other's pairs); a new segment starts when
    // the last one cannot take a batch's worst case, so stored edges are never moved
    std::vector<std::unique_ptr<DevBuf<unsigned long long>>> useg;
    std::vector<size_t> useg_n;
    DevBuf<unsigned long long> counters;        // [0] emit count, [1] unique count
    DevBuf<int> spill;                          // reader spill chunks (SPILL ints each)
    DevBuf<unsigned> spill_ctr;                 // [0] chunks handed out, [1] ran-out flag
    size_t spill_chunks = 0;                    // pool capacity in chunks
    unsigned spill_used = 0;                    // chunks in use after the last completed step
    size_t nuniq = 0;
    // graph
    DevBuf<uint32_t> succ_ptr, succ, npred, tmp;
    DevBuf<uint32_t> win_ptr, win_succ, win_npred, win_tmp;   // window graphs (a runtime running the graph in pieces)
    DevBuf<uint32_t> periodic;                  // packed arrays of the periodic form
    DevBuf<unsigned> bin_off, bin_cur;          // ops binned to regions: offsets, fill cursors
    DevBuf<int> bin_list, bin_flag;             // op indices per region; region-too-long flag
    DevBuf<int> snap;                           // cell states at the time-split cuts (resolve_puts_kernel)
    bool graph_valid = false;
    double last_device_ms = 0;
    double last_ops_ms = 0, last_compress_ms = 0;   // host phases of the last batch
    double emit_per_op = 32.0;                  // emitted-pair estimate per op (from the last batch)
    // parallel host passes (validation, op build): the host team and the page-locked staging buffer
    std::unique_ptr<WorkPool> pool;
    HostStage stage;
    bool staged = false;                        // this batch's ops are in `stage`
};

namespace xkb {

static int seg_rects_blas(uint64_t a, uint64_t b, uint64_t ld, uint64_t s, HRect out[3])
{
    const uint64_t LDs = ld * s, size = b - a;
    const uint64_t x0 = a % LDs, x1 = std::min(x0 + size, LDs), dx10 = x1 - x0;
    const uint64_t x3 = (size - dx10) % LDs;
    const uint64_t y0 = a / LDs, y1 = y0 + 1;
    const uint64_t y3 = y0 + (size - dx10 - x3) / LDs + 2, y2 = y3 - 1;
    const HRect r[3] = {{x0, x1, y0, y1}, {0, LDs, y1, y2}, {0, x3, y2, y3}};
    int n = 0;
    for (const HRect & q : r) if (q.x0 < q.x1 && q.y0 < q.y1) out[n++] = q;
    return n;
}

static int mat_rects(const xkb_access_rec_t & r, HRect out[2])
{
    const uint64_t s = r.sizeof_type, ld = r.ld, LDs = ld * s;
    const uint64_t A = r.addr + (r.offset_n * ld + r.offset_m) * s;
    const uint64_t x0 = A % LDs, y0 = A / LDs;
    if (x0 + r.m * s <= LDs) { out[0] = {x0, x0 + r.m * s, y0, y0 + r.n}; return 1; }
    out[0] = {x0, LDs, y0, y0 + r.n};
    out[1] = {0, r.m * s - (LDs - x0), y0 + 1, y0 + r.n + 1};
    return 2;
}

static void push_ops(Domain & d, bool link, const xkb_access_rec_t & r)
{
    HRect rects[3];
    int n;
    if (r.type == XKB_ACCESS_TYPE_HANDLE)
    {
        // a handle is one point of its own domain; the handle map records every access with
        // the R bit and no W bit as a reader (dependency-map.hpp put()), so such modes count as R
        const uint8_t m = ((r.mode & M_R) && !(r.mode & M_W)) ? M_R : r.mode;
        d.ops.push_back({r.task, (uint8_t) link, m, HRect{r.addr, r.addr + 1, 0, 1}});
        return;
    }
    if (d.interval) { rects[0] = {r.addr, r.ld, 0, 1}; n = 1; }
    else if (r.type == XKB_ACCESS_TYPE_SEGMENT) n = seg_rects_blas(r.addr, r.ld, d.ld, d.s, rects);
    else n = mat_rects(r, rects);
    for (int i = 0; i < n; ++i)
    {
        HRect q = rects[i];
        if (!link && !d.interval && r.type == XKB_ACCESS_TYPE_SEGMENT)
        {
            q.x0 = std::max(q.x0, r.addr); q.x1 = std::min(q.x1, r.ld);
            q.y1 = std::min<uint64_t>(q.y1, 1);
            if (q.x0 >= q.x1 || q.y0 >= q.y1) continue;
        }
        d.ops.push_back({r.task, (uint8_t) link, r.mode, q});
    }
}

// First record of [b, e) that is malformed or breaks the dense task numbering (its task must be
// the previous record's or the next one, starting at first_task), with the reason; e if none.
static size_t first_invalid(const xkb_access_rec_t * recs, size_t b, size_t e, uint32_t first_task, const char ** why)
{
    for (size_t i = b; i < e; ++i)
    {
        const xkb_access_rec_t & r = recs[i];
        const uint32_t prev = i == 0 ? first_task : recs[i - 1].task;
        if (r.task < prev || r.task > prev + 1 || (i == 0 && r.task != first_task)) { *why = "task ids must be dense, in spawn order"; return i; }
        if (r.mode == 0 || (r.mode & ~15u)) { *why = "bad mode"; return i; }
        const unsigned conc = r.reserved >> 8;      // sequential (0, 1) or commutative (2)
        if (conc == 4) { *why = "a concurrent access: expand the stream with xkb_handle_map_expand first"; return i; }
        if (conc > 2) { *why = "bad concurrency"; return i; }
        if (r.type == XKB_ACCESS_TYPE_SEGMENT) {
            if (r.ld <= r.addr) { *why = "empty segment"; return i; }
        } else if (r.type == XKB_ACCESS_TYPE_BLAS_MATRIX) {
            if (!r.ld || !r.sizeof_type || !r.m || !r.n || r.m > r.ld) { *why = "bad matrix tile"; return i; }
        } else if (r.type == XKB_ACCESS_TYPE_HANDLE) {
            if (r.addr == ~0ull) { *why = "handle ~0 is reserved"; return i; }
        } else { *why = "unsupported access type"; return i; }
    }
    return e;
}

// Validate a batch (on the host team when it is large).
static int validate(xkb_resolver * R, const xkb_access_rec_t * recs, size_t n, uint32_t first_task)
{
    const char * why = "";
    size_t bad = n;
    if (n >= 65536 && R->pool && R->pool->size() > 1)
    {
        const unsigned nc = R->pool->size();
        std::vector<size_t> at(nc, n);
        std::vector<const char *> w(nc, "");
        R->pool->run([&](unsigned c) {
            const size_t e = n * (c + 1) / nc;
            const size_t x = first_invalid(recs, n * c / nc, e, first_task, &w[c]);
            at[c] = x == e ? n : x;
        });
        for (unsigned c = 0; c < nc; ++c) if (at[c] < bad) { bad = at[c]; why = w[c]; }
    }
    else bad = first_invalid(recs, 0, n, first_task, &why);
    if (bad < n) return xkb_set_error(XKB_EINVAL, "resolver: access %zu: %s (tasks continue at %u)", bad, why, first_task);
    return XKB_OK;
}

// Rects of a matrix record in its frame (mat_rects' count only).
static inline int mat_nrects(const xkb_access_rec_t & r)
{
    const uint64_t LDs = r.ld * r.sizeof_type, A = r.addr + (r.offset_n * r.ld + r.offset_m) * r.sizeof_type;
    return (A % LDs) + r.m * r.sizeof_type <= LDs ? 1 : 2;
}

// Matrix-only batches whose every (ld, sizeof) already has a domain: each record's ops go to its
// own domain only (LINK ops of a task's records, then their PUT ops), so chunks of whole tasks
// are built by the host team: a counting pass, then every chunk writes its ops straight into the
// page-locked staging buffer, domain after domain and chunks in order within a domain -- the
// order of the sequential build. Counters and cursors live on each member's own stack while it
// runs (members sharing cache lines would serialise on them). Returns 1 (built), 0 (the batch
// needs the sequential path: a segment or handle, a matrix key seen for the first time -- a new
// domain replays earlier segments at that point of the stream -- or a small batch), or an error.
static int build_ops_staged(xkb_resolver * R, const xkb_access_rec_t * recs, size_t n)
{
    if (n < 65536 || !R->pool) return 0;
    const unsigned nc = R->pool->size();
    if (nc < 2) return 0;
    if (R->segments.empty())
    {
        // no segment seen yet, so a new matrix domain replays nothing: create the batch's new
        // ones up front, in the order the sequential build would meet them
        std::vector<char> other(nc, 0), fresh(nc, 0);
        R->pool->run([&](unsigned c) {
            uint64_t lk = ~0ull, ls = ~0ull;
            for (size_t i = n * c / nc; i < n * (c + 1) / nc; ++i)
            {
                const xkb_access_rec_t & r = recs[i];
                if (r.type != XKB_ACCESS_TYPE_BLAS_MATRIX) { other[c] = 1; return; }
                if (r.ld == lk && r.sizeof_type == ls) continue;
                lk = r.ld; ls = r.sizeof_type;
                if (!R->blas_index.count(std::make_pair(r.ld, r.sizeof_type))) fresh[c] = 1;
            }
        });
        for (char o : other) if (o) return 0;
        bool any = false;
        for (char f : fresh) any = any || f;
        uint64_t lk = ~0ull, ls = ~0ull;
        if (any)
            for (size_t i = 0; i < n; ++i)
            {
                if (recs[i].ld == lk && recs[i].sizeof_type == ls) continue;
                lk = recs[i].ld; ls = recs[i].sizeof_type;
                const auto key = std::make_pair(lk, ls);
                if (R->blas_index.count(key)) continue;
                std::unique_ptr<Domain> d(new Domain());
                d->ld = key.first; d->s = key.second;
                d->state[0].use_pool(R->stream); d->state[1].use_pool(R->stream);
                R->blas.push_back(std::move(d));
                R->blas_index.emplace(key, R->blas.size() - 1);
            }
    }
    if (R->blas.empty()) return 0;
    const size_t nd = R->blas.size();
    std::vector<uint64_t> keys(2 * nd);
    for (size_t k = 0; k < nd; ++k) { keys[2 * k] = R->blas[k]->ld; keys[2 * k + 1] = R->blas[k]->s; }
    auto dom_of = [&](const xkb_access_rec_t & r, uint64_t & lk, uint64_t & ls, size_t & li) {
        if (r.ld == lk && r.sizeof_type == ls) return true;
        for (size_t k = 0; k < nd; ++k)
            if (keys[2 * k] == r.ld && keys[2 * k + 1] == r.sizeof_type) { lk = r.ld; ls = r.sizeof_type; li = k; return true; }
        return false;
    };
    std::vector<size_t> cut(nc + 1, n);
    cut[0] = 0;
    for (unsigned t = 1; t < nc; ++t)
    {
        size_t c = std::max(cut[t - 1], n * t / nc);
        while (c > cut[t - 1] && c < n && recs[c].task == recs[c - 1].task) ++c;     // whole tasks per chunk
        cut[t] = c;
    }
    std::vector<size_t> cnt(nc * nd, 0);
    std::vector<char> ok(nc, 1);
    R->pool->run([&](unsigned c) {
        uint64_t lk = ~0ull, ls = ~0ull;
        size_t li = 0;
        std::vector<size_t> my(nd, 0);
        for (size_t i = cut[c]; i < cut[c + 1]; ++i)
        {
            const xkb_access_rec_t & r = recs[i];
            if (r.type != XKB_ACCESS_TYPE_BLAS_MATRIX || !dom_of(r, lk, ls, li)) { ok[c] = 0; return; }
            my[li] += 2 * (size_t) mat_nrects(r);
        }
        std::copy(my.begin(), my.end(), cnt.begin() + c * nd);
    });
    for (char o : ok) if (!o) return 0;
    std::vector<size_t> pos(nc * nd);
    size_t total = 0;
    for (size_t k = 0; k < nd; ++k)
    {
        R->blas[k]->stage_off = total;
        for (unsigned c = 0; c < nc; ++c) { pos[c * nd + k] = total; total += cnt[c * nd + k]; }
        R->blas[k]->nops = total - R->blas[k]->stage_off;
    }
    if (int rc = R->stage.reserve(total ? total : 1)) return rc;
    HOp * out = R->stage.p;
    R->pool->run([&](unsigned c) {
        uint64_t lk = ~0ull, ls = ~0ull;
        size_t li = 0;
        std::vector<size_t> p(pos.begin() + c * nd, pos.begin() + (c + 1) * nd);
        for (size_t i = cut[c]; i < cut[c + 1];)
        {
            size_t j = i;
            while (j < cut[c + 1] && recs[j].task == recs[i].task) ++j;
            for (int pass = 0; pass < 2; ++pass)                 // LINK ops, then PUT ops
                for (size_t a = i; a < j; ++a)
                {
                    dom_of(recs[a], lk, ls, li);
                    HRect rr[2];
                    const int nr = mat_rects(recs[a], rr);
                    for (int q = 0; q < nr; ++q) out[p[li]++] = HOp{recs[a].task, (uint8_t) (pass == 0), recs[a].mode, rr[q]};
                }
            i = j;
        }
    });
    R->staged = true;
    return 1;
}

// Build every domain's op list for the batch, in the order the reference performs them.
static void build_ops(xkb_resolver * R, const xkb_access_rec_t * recs, size_t n)
{
    for (size_t i = 0; i < n;)
    {
        size_t j = i;
        while (j < n && recs[j].task == recs[i].task) ++j;
        for (size_t a = i; a < j; ++a)                          // LINK pass
        {
            const xkb_access_rec_t & r = recs[a];
            if (r.type == XKB_ACCESS_TYPE_HANDLE) push_ops(R->handles, true, r);
            else if (r.type == XKB_ACCESS_TYPE_SEGMENT)
            {
                push_ops(R->interval, true, r);
                for (auto & d : R->blas) push_ops(*d, true, r);
            }
            else
            {
                const auto key = std::make_pair(r.ld, r.sizeof_type);
                auto it = R->blas_index.find(key);
                if (it == R->blas_index.end())
                {
                    std::unique_ptr<Domain> d(new Domain());
                    d->ld = r.ld; d->s = r.sizeof_type;
                    d->state[0].use_pool(R->stream); d->state[1].use_pool(R->stream);
                    for (auto k = R->segments.rbegin(); k != R->segments.rend(); ++k) push_ops(*d, false, *k);
                    R->blas.push_back(std::move(d));
                    it = R->blas_index.emplace(key, R->blas.size() - 1).first;
                }
                push_ops(*R->blas[it->second], true, r);
            }
        }
        for (size_t a = i; a < j; ++a)                          // PUT pass
        {
            const xkb_access_rec_t & r = recs[a];
            if (r.type == XKB_ACCESS_TYPE_HANDLE) push_ops(R->handles, false, r);
            else if (r.type == XKB_ACCESS_TYPE_SEGMENT)
            {
                push_ops(R->interval, false, r);
                for (auto & d : R->blas) push_ops(*d, false, r);
                R->segments.push_back(r);
            }
            else
                push_ops(*R->blas[R->blas_index.at({r.ld, r.sizeof_type})], false, r);
        }
        i = j;
    }
}

// Extend the domain's compression with the batch's boundaries; remap the device state when
// the cell grid changes.
// The spill pool: created on first use; grown keeping its chunks (cell states name them by
// index). reset_spill() rewinds the hand-out counter to the last completed step before a kernel
// that may run out of chunks and be redone.
static int spill_reserve(xkb_resolver * R, size_t chunks)
{
    if (!R->spill_ctr.p)
    {
        int rc = R->spill_ctr.reserve(2);
        if (rc) return rc;
        XKB_CUDA_TRY(cudaMemsetAsync(R->spill_ctr.p, 0, 2 * sizeof(unsigned), R->stream));
    }
    if (chunks <= R->spill_chunks) return XKB_OK;
    size_t c = R->spill_chunks ? R->spill_chunks : 65536;
    while (c < chunks) c *= 2;
    if (c > 0xffffffffu / 2) return xkb_set_error(XKB_ERANGE, "resolver: reader spill pool exceeds 2^31 chunks");
    int * q = nullptr;
    cudaError_t e = cudaMalloc(&q, c * SPILL * sizeof(int));
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    if (R->spill.p && R->spill_used)
    {
        e = cudaMemcpyAsync(q, R->spill.p, (size_t) R->spill_used * SPILL * sizeof(int), cudaMemcpyDeviceToDevice, R->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(R->stream);
        if (e != cudaSuccess) { cudaFree(q); return xkb_set_cuda_error(e); }
    }
    if (R->spill.p) cudaFree(R->spill.p);
    R->spill.p = q; R->spill.cap = c * SPILL; R->spill_chunks = c;
    return XKB_OK;
}

static int reset_spill(xkb_resolver * R)
{
    const unsigned v[2] = {R->spill_used, 0u};
    XKB_CUDA_TRY(cudaMemcpyAsync(R->spill_ctr.p, v, sizeof(v), cudaMemcpyHostToDevice, R->stream));
    XKB_CUDA_TRY(cudaStreamSynchronize(R->stream));   // v is on this stack frame
    return XKB_OK;
}

// After a kernel that draws chunks: true (and the pool grown) if it ran out and must be redone;
// else the chunks it drew become part of the kept state.
static int spill_check(xkb_resolver * R, bool & redo)
{
    unsigned v[2];
    XKB_CUDA_TRY(cudaMemcpyAsync(v, R->spill_ctr.p, sizeof(v), cudaMemcpyDeviceToHost, R->stream));
    XKB_CUDA_TRY(cudaStreamSynchronize(R->stream));
    redo = v[1] != 0;
    if (redo) return spill_reserve(R, (size_t) v[0] + 1);
    R->spill_used = v[0];
    return XKB_OK;
}

// XKB_TRACE_RESOLVE=2: the time each step of a batch's compression and region pass takes
// (host clock, so a step that synchronises includes the device work queued before it).
struct PhaseTrace {
    const bool on;
    const char * what;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    std::string line;
    explicit PhaseTrace(const char * w) : on(trace_level() >= 2), what(w) {}
    static int trace_level() { static const int l = getenv("XKB_TRACE_RESOLVE") ? atoi(getenv("XKB_TRACE_RESOLVE")) : 0; return l; }
    void mark(const char * step)
    {
        if (!on) return;
        const auto n = std::chrono::steady_clock::now();
        char b[96];
        snprintf(b, sizeof(b), " %s %.1f", step, std::chrono::duration<double, std::milli>(n - t).count());
        line += b; t = n;
    }
    ~PhaseTrace() { if (on) fprintf(stderr, "  %s (ms):%s\n", what, line.c_str()); }
};

static int refine_domain(xkb_resolver * R, Domain & d, std::vector<uint64_t> & xs, std::vector<uint64_t> & ys)
{
    if (xs.size() < 2 || ys.size() < 2) { d.xs = xs; d.ys = ys; return XKB_OK; }
    const bool same = xs == d.xs && ys == d.ys;
    const size_t ncx = xs.size() - 1, ncy = ys.size() - 1, ncells = ncx * ncy;
    if (same && d.ncells == ncells) return XKB_OK;
    int rc;
    PhaseTrace pt("refine");
    DevBuf<int> & out = d.state[d.cur ^ 1];
    if ((rc = out.reserve(ncells * STRIDE))) return rc;
    pt.mark("state-reserve");
    if (d.ncells == 0)
    {
        init_state_kernel<<<(unsigned) ((ncells + 255) / 256), 256, 0, R->stream>>>(out.p, ncells);
    }
    else
    {
        const size_t old_ncx = d.xs.size() - 1;
        std::vector<int> mx(ncx), my(ncy);
        for (size_t i = 0; i < ncx; ++i) {
            const uint64_t v = xs[i];
            if (v < d.xs.front() || v >= d.xs.back()) mx[i] = -1;
            else mx[i] = (int) (std::upper_bound(d.xs.begin(), d.xs.end(), v) - d.xs.begin()) - 1;
        }
        for (size_t i = 0; i < ncy; ++i) {
            const uint64_t v = ys[i];
            if (v < d.ys.front() || v >= d.ys.back()) my[i] = -1;
            else my[i] = (int) (std::upper_bound(d.ys.begin(), d.ys.end(), v) - d.ys.begin()) - 1;
        }
        DevBuf<int> dm;
        if ((rc = dm.reserve(ncx + ncy))) return rc;
        XKB_CUDA_TRY(cudaMemcpyAsync(dm.p, mx.data(), ncx * sizeof(int), cudaMemcpyHostToDevice, R->stream));
        XKB_CUDA_TRY(cudaMemcpyAsync(dm.p + ncx, my.data(), ncy * sizeof(int), cudaMemcpyHostToDevice, R->stream));
        pt.mark("maps");
        if ((rc = spill_reserve(R, 1))) return rc;
        pt.mark("spill-reserve");
        for (bool redo = true; redo;)
        {
            if ((rc = reset_spill(R))) return rc;
            refine_state_kernel<<<(unsigned) ((ncells + 255) / 256), 256, 0, R->stream>>>(
                d.state[d.cur].p, out.p, dm.p, dm.p + ncx, (int) ncx, (int) ncy, (int) old_ncx, R->spill.p, R->spill_ctr.p,
                (unsigned) R->spill_chunks);
            XKB_CUDA_TRY(cudaGetLastError());
            if ((rc = spill_check(R, redo))) return rc;   // synchronises: dm is freed on return
            pt.mark("refine-kernel+sync");
        }
    }
    XKB_CUDA_TRY(cudaGetLastError());
    d.cur ^= 1;
    d.xs.swap(xs); d.ys.swap(ys); d.ncells = ncells;
    return XKB_OK;
}

// Bin the batch's ops to regions (counts, offsets, fill, per-region sort) and run the region
// kernel over each region's own list; a region too crowded to sort falls back to the kernel that
// scans every op of the batch.
template <int RX, int RY>
static int launch_region(xkb_resolver * R, ResolveArgs & a, int nregions)
{
    const size_t smem = (size_t) RCAP * RX * RY * sizeof(int);
    cudaStream_t st = R->stream;
    const size_t nb = (size_t) nregions + 1;
    int rc;
    PhaseTrace pt("regions");
    if ((rc = R->bin_off.reserve(nb)) || (rc = R->bin_cur.reserve(nb)) ||
        (rc = R->tmp.reserve(nb / SCAN_TILE + 2)) || (rc = R->bin_flag.reserve(1)))
        return rc;
    pt.mark("reserve");
    XKB_CUDA_TRY(cudaMemsetAsync(R->bin_off.p, 0, nb * sizeof(unsigned), st));
    XKB_CUDA_TRY(cudaMemsetAsync(R->bin_cur.p, 0, nb * sizeof(unsigned), st));
    XKB_CUDA_TRY(cudaMemsetAsync(R->bin_flag.p, 0, sizeof(int), st));
    const unsigned g = (unsigned) ((a.nops + 255) / 256);
    // block-local binning: a grid of a few blocks per SM, each walking its share of the ops
    const char * gb = getenv("XKB_RESOLVE_BIN_GLOBAL");             // 1: the global-atomic binning (tests)
    const bool smem_bins = nregions <= BIN_SMEM_REGIONS && !(gb && atoi(gb) == 1);
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned gs = std::min<unsigned>(g, (unsigned) (2 * sms));
    if (smem_bins)
    {
        XKB_CUDA_TRY(cudaFuncSetAttribute(bin_count_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          BIN_SMEM_REGIONS * (int) sizeof(unsigned)));
        bin_count_smem_kernel<<<gs, 256, (size_t) nregions * sizeof(unsigned), st>>>(a.ops, a.nops, RX, RY, a.nrx, nregions,
                                                                                   R->bin_off.p);
    }
    else
        bin_count_kernel<<<g, 256, 0, st>>>(a.ops, a.nops, RX, RY, a.nrx, R->bin_off.p);
    if ((rc = device_exclusive_scan(R->bin_off.p, R->bin_off.p, nb, R->tmp.p, nullptr, st))) return rc;
    unsigned total = 0;
    XKB_CUDA_TRY(cudaMemcpyAsync(&total, R->bin_off.p + nregions, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    pt.mark("count+sync");
    bool binned = total > 0;
    if (binned)
    {
        if ((rc = R->bin_list.reserve(total))) return rc;
        if (smem_bins)
        {
            XKB_CUDA_TRY(cudaFuncSetAttribute(bin_fill_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              2 * BIN_SMEM_REGIONS * (int) sizeof(unsigned)));
            bin_fill_smem_kernel<<<gs, 256, 2 * (size_t) nregions * sizeof(unsigned), st>>>(a.ops, a.nops, RX, RY, a.nrx, nregions,
                                                                                         R->bin_off.p, R->bin_cur.p, R->bin_list.p);
        }
        else
            bin_fill_kernel<<<g, 256, 0, st>>>(a.ops, a.nops, RX, RY, a.nrx, R->bin_off.p, R->bin_cur.p, R->bin_list.p);
        XKB_CUDA_TRY(cudaFuncSetAttribute(bin_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, BIN_SORT_CAP * (int) sizeof(int)));
        bin_sort_kernel<<<(unsigned) nregions, BIN_SORT_THREADS, BIN_SORT_CAP * sizeof(int), st>>>(R->bin_off.p, R->bin_list.p, R->bin_flag.p);
        int too_long = 0;
        XKB_CUDA_TRY(cudaMemcpyAsync(&too_long, R->bin_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        XKB_CUDA_TRY(cudaStreamSynchronize(st));
        pt.mark("fill+sort+sync");
        binned = !too_long;
    }
    // time split: segments per region from the mean list length (a segment of a few hundred ops
    // still amortises its state load); XKB_RESOLVE_SEGMENTS overrides (1 = one pass per region)
    const char * seg_s = getenv("XKB_RESOLVE_SEGMENTS");
    const int seg_env = seg_s ? atoi(seg_s) : 0;
    int nseg = seg_env > 0 ? seg_env : (int) std::min<size_t>(MAX_SEGMENTS, std::max<size_t>(1, (size_t) total / nregions / 512));
    nseg = std::max(1, std::min(nseg, MAX_SEGMENTS));
    if (binned && nseg > 1)
    {
        const size_t ncells = (size_t) a.ncx * a.ncy;
        if ((rc = R->snap.reserve((size_t) (nseg - 1) * ncells * STRIDE))) return rc;
        XKB_CUDA_TRY(cudaFuncSetAttribute(resolve_puts_kernel<RX, RY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        XKB_CUDA_TRY(cudaFuncSetAttribute(resolve_links_kernel<RX, RY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        resolve_puts_kernel<RX, RY><<<(unsigned) nregions, RX * RY, smem, st>>>(a, R->bin_off.p, R->bin_list.p, nseg, R->snap.p, ncells);
        resolve_links_kernel<RX, RY><<<(unsigned) (nregions * nseg), RX * RY, smem, st>>>(a, R->bin_off.p, R->bin_list.p, nseg,
                                                                                      R->snap.p, ncells);
    }
    else if (binned)
    {
        XKB_CUDA_TRY(cudaFuncSetAttribute(resolve_region_kernel<RX, RY, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        resolve_region_kernel<RX, RY, true><<<(unsigned) nregions, RX * RY, smem, st>>>(a, R->bin_off.p, R->bin_list.p);
    }
    else
    {
        XKB_CUDA_TRY(cudaFuncSetAttribute(resolve_region_kernel<RX, RY, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        resolve_region_kernel<RX, RY, false><<<(unsigned) nregions, RX * RY, smem, st>>>(a, nullptr, nullptr);
    }
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

static int launch_domain(xkb_resolver * R, Domain & d, size_t op_offset, size_t nops)
{
    const int ncx = (int) d.xs.size() - 1, ncy = (int) d.ys.size() - 1;
    ResolveArgs a;
    a.ops = R->dops.p + op_offset; a.nops = (int) nops;
    a.ncx = ncx; a.ncy = ncy;
    a.state_in = d.state[d.cur].p; a.state_out = d.state[d.cur ^ 1].p;
    a.emit = R->emit.p; a.emit_count = R->counters.p; a.emit_cap = R->emit.cap;
    a.spill = R->spill.p; a.spill_ctr = R->spill_ctr.p; a.spill_cap = (unsigned) R->spill_chunks;
    if (ncy == 1)
    {
        constexpr int RX = 64, RY = 1;
        a.nrx = (ncx + RX - 1) / RX;
        return launch_region<RX, RY>(R, a, a.nrx);
    }
    constexpr int RX = 8, RY = XKB_REGION_RY;
    a.nrx = (ncx + RX - 1) / RX;
    const int nry = (ncy + RY - 1) / RY;
    return launch_region<RX, RY>(R, a, a.nrx * nry);
}

// Compress the domain's coordinates with the batch's boundaries (found on the device, merged with
// the domain's earlier ones on the host), refine the cell state, and write the batch's ops in cell
// coordinates to dops. hops / dops: this domain's nops ops on the device.
static int compress_domain(xkb_resolver * R, Domain & d, const HOp * hops, DOp * dops, size_t nops)
{
    cudaStream_t st = R->stream;
    size_t cap = 1024;
    while (cap < 4 * nops) cap *= 2;
    int rc;
    PhaseTrace pt("compress");
    if ((rc = R->hset.reserve(2 * cap)) || (rc = R->ukeys.reserve(4 * nops)) || (rc = R->ucount.reserve(3))) return rc;
    pt.mark("reserve");
    XKB_CUDA_TRY(cudaMemsetAsync(R->hset.p, 0xff, 2 * cap * sizeof(uint64_t), st));
    XKB_CUDA_TRY(cudaMemsetAsync(R->ucount.p, 0, 3 * sizeof(unsigned), st));
    const unsigned g = (unsigned) ((nops + 255) / 256);
    collect_bounds_kernel<<<g, 256, 0, st>>>(hops, (int) nops, R->hset.p, R->hset.p + cap, (uint32_t) (cap - 1),
                                             R->ukeys.p, R->ukeys.p + 2 * nops, R->ucount.p);
    XKB_CUDA_TRY(cudaGetLastError());
    unsigned cnt[3];
    XKB_CUDA_TRY(cudaMemcpyAsync(cnt, R->ucount.p, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    pt.mark("collect+sync");
    std::vector<uint64_t> xs(d.xs.size() + cnt[0] + 1), ys(d.ys.size() + cnt[1] + 1);
    std::copy(d.xs.begin(), d.xs.end(), xs.begin());
    std::copy(d.ys.begin(), d.ys.end(), ys.begin());
    if (cnt[0]) XKB_CUDA_TRY(cudaMemcpyAsync(xs.data() + d.xs.size(), R->ukeys.p, cnt[0] * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    if (cnt[1]) XKB_CUDA_TRY(cudaMemcpyAsync(ys.data() + d.ys.size(), R->ukeys.p + 2 * nops, cnt[1] * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    if (cnt[2] & 1u) xs.back() = KEY_EMPTY; else xs.pop_back();
    if (cnt[2] & 2u) ys.back() = KEY_EMPTY; else ys.pop_back();
    for (std::vector<uint64_t> * v : {&xs, &ys})
    {
        std::sort(v->begin(), v->end());
        v->erase(std::unique(v->begin(), v->end()), v->end());
    }
    pt.mark("keys+sort");
    if ((rc = refine_domain(R, d, xs, ys))) return rc;
    pt.mark("refine");
    if ((rc = R->bounds.reserve(d.xs.size() + d.ys.size()))) return rc;
    XKB_CUDA_TRY(cudaMemcpyAsync(R->bounds.p, d.xs.data(), d.xs.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    XKB_CUDA_TRY(cudaMemcpyAsync(R->bounds.p + d.xs.size(), d.ys.data(), d.ys.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    map_ops_kernel<<<g, 256, 0, st>>>(hops, (int) nops, R->bounds.p, (int) d.xs.size(), R->bounds.p + d.xs.size(),
                                      (int) d.ys.size(), dops);
    XKB_CUDA_TRY(cudaGetLastError());
    // the host vectors above die on return: the copies out of them must be done
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    pt.mark("map+sync");
    return XKB_OK;
}

static int resolve_batch(xkb_resolver * R, const xkb_access_rec_t * recs, size_t n)
{
    int rc;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    R->staged = false;
    rc = build_ops_staged(R, recs, n);
    if (rc < 0) return rc;
    if (!R->staged)
    {
        build_ops(R, recs, n);
        R->interval.nops = R->interval.ops.size(); R->handles.nops = R->handles.ops.size();
        for (auto & d : R->blas) d->nops = d->ops.size();
    }
    const auto t1 = clk::now();
    std::vector<Domain *> doms;
    if (R->interval.nops) doms.push_back(&R->interval);
    if (R->handles.nops) doms.push_back(&R->handles);
    for (auto & d : R->blas) if (d->nops) doms.push_back(d.get());

    std::vector<size_t> offs;
    size_t total = 0;
    for (Domain * d : doms) { offs.push_back(total); total += d->nops; }
    if ((rc = R->hops.reserve(total ? total : 1)) || (rc = R->dops.reserve(total ? total : 1))) return rc;
    if (R->staged)          // domain-major in the staging buffer, in the order of `doms`
    {
        if (total) XKB_CUDA_TRY(cudaMemcpyAsync(R->hops.p, R->stage.p, total * sizeof(HOp), cudaMemcpyHostToDevice, R->stream));
    }
    else
        for (size_t k = 0; k < doms.size(); ++k)
            XKB_CUDA_TRY(cudaMemcpyAsync(R->hops.p + offs[k], doms[k]->ops.data(), doms[k]->nops * sizeof(HOp),
                                         cudaMemcpyHostToDevice, R->stream));
    for (size_t k = 0; k < doms.size(); ++k)
        if ((rc = compress_domain(R, *doms[k], R->hops.p + offs[k], R->dops.p + offs[k], doms[k]->nops))) return rc;
    R->last_ops_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    R->last_compress_ms = std::chrono::duration<double, std::milli>(clk::now() - t1).count();

    static const bool trace = getenv("XKB_TRACE_RESOLVE") != nullptr;
    const size_t realloc0 = g_realloc_bytes;
    // an emit buffer too small costs a second pass of the region kernel: size it from the pairs per
    // op the last batch emitted (32 per op before the first), within 2^28 pairs
    size_t emit_guess = std::max<size_t>(1 << 16, std::min<size_t>(size_t(1) << 28, (size_t) (total * R->emit_per_op)));
    for (int attempt = 0; attempt < 16; ++attempt)
    {
        const auto ta = clk::now();
        if ((rc = R->emit.reserve(emit_guess))) return rc;
        if ((rc = R->counters.reserve(2))) return rc;
        if ((rc = spill_reserve(R, 1)) || (rc = reset_spill(R))) return rc;
        XKB_CUDA_TRY(cudaMemsetAsync(R->counters.p, 0, 2 * sizeof(unsigned long long), R->stream));
        for (size_t k = 0; k < doms.size(); ++k)
        {
            const size_t nops = doms[k]->nops;
            // states must exist for every cell (ncells > 0 when the domain has >= 1 op)
            if ((rc = R->emit.reserve(emit_guess))) return rc;
            if (doms[k]->ncells == 0) continue;
            if ((rc = doms[k]->state[doms[k]->cur ^ 1].reserve(doms[k]->ncells * STRIDE))) return rc;
            if ((rc = launch_domain(R, *doms[k], offs[k], nops))) return rc;
        }
        unsigned long long nemit = 0;
        unsigned sp[2] = {0, 0};
        XKB_CUDA_TRY(cudaMemcpyAsync(&nemit, R->counters.p, sizeof(nemit), cudaMemcpyDeviceToHost, R->stream));
        XKB_CUDA_TRY(cudaMemcpyAsync(sp, R->spill_ctr.p, sizeof(sp), cudaMemcpyDeviceToHost, R->stream));
        XKB_CUDA_TRY(cudaStreamSynchronize(R->stream));
        if (sp[1])
        {
            // the reader spill pool ran out: grow it (keeping its chunks) and redo the batch
            if ((rc = spill_reserve(R, (size_t) sp[0] + 1))) return rc;
            continue;
        }
        const auto tb = clk::now();
        if (nemit > R->emit.cap) { emit_guess = (size_t) nemit; continue; }
        R->spill_used = sp[0];
        if (total) R->emit_per_op = std::max(2.0, 1.25 * (double) nemit / (double) total);

        // success: unique the emitted pairs into the accumulated edge list
        if (nemit)
        {
            size_t tcap = 1024;
            while (tcap < 2 * nemit) tcap *= 2;
            if ((rc = R->table.reserve(tcap))) return rc;
            if (R->useg.empty() || R->useg.back()->cap - R->useg_n.back() < nemit)
            {
                std::unique_ptr<DevBuf<unsigned long long>> seg(new (std::nothrow) DevBuf<unsigned long long>());
                if (seg) seg->use_pool(R->stream);
                if (!seg) return xkb_set_error(XKB_ENOMEM, "resolver: out of host memory");
                // segments double in size, so a long stream allocates a few of them, not one per batch
                const size_t last = R->useg.empty() ? 0 : R->useg.back()->cap;
                if ((rc = seg->reserve(std::max<size_t>({(size_t) nemit, size_t(1) << 24, 2 * last})))) return rc;
                R->useg.push_back(std::move(seg));
                R->useg_n.push_back(0);
            }
            DevBuf<unsigned long long> & seg = *R->useg.back();
            XKB_CUDA_TRY(cudaMemsetAsync(R->table.p, 0xff, tcap * sizeof(unsigned long long), R->stream));
            unsigned long long nu0 = R->useg_n.back();
            XKB_CUDA_TRY(cudaMemcpyAsync(R->counters.p + 1, &nu0, sizeof(nu0), cudaMemcpyHostToDevice, R->stream));
            dedupe_kernel<<<(unsigned) ((nemit + 255) / 256), 256, 0, R->stream>>>(R->emit.p, nemit, R->table.p, tcap - 1,
                                                                                 seg.p, R->counters.p + 1, seg.cap);
            XKB_CUDA_TRY(cudaGetLastError());
            unsigned long long nu = 0;
            XKB_CUDA_TRY(cudaMemcpyAsync(&nu, R->counters.p + 1, sizeof(nu), cudaMemcpyDeviceToHost, R->stream));
            XKB_CUDA_TRY(cudaStreamSynchronize(R->stream));
            R->nuniq += nu - nu0;
            R->useg_n.back() = nu;
        }
        for (Domain * d : doms) { d->cur ^= 1; d->ops.clear(); d->nops = 0; }
        if (trace)
            fprintf(stderr, "resolver batch: %zu ops (built in %.1f ms, compressed in %.1f ms), attempt %d, regions %.1f ms, dedupe %.1f ms, "
                    "%llu emitted, %.1f MB allocated\n",
                    total, R->last_ops_ms, R->last_compress_ms, attempt, std::chrono::duration<double, std::milli>(tb - ta).count(),
                    std::chrono::duration<double, std::milli>(clk::now() - tb).count(), nemit, (g_realloc_bytes - realloc0) / 1e6);
        return XKB_OK;
    }
    return xkb_set_error(XKB_ERANGE, "resolver: batch did not fit after resizing");
}

static int build_graph(xkb_resolver * R)
{
    int rc;
    const size_t nt = R->ntasks, ne = R->nuniq;
    if ((rc = R->succ_ptr.reserve(nt + 1))) return rc;
    if ((rc = R->npred.reserve(nt + 1))) return rc;
    if ((rc = R->succ.reserve(ne ? ne : 1))) return rc;
    if ((rc = R->tmp.reserve(nt + 1 + (nt + 1) / SCAN_TILE + 2))) return rc;
    cudaStream_t st = R->stream;
    XKB_CUDA_TRY(cudaMemsetAsync(R->succ_ptr.p, 0, (nt + 1) * sizeof(uint32_t), st));
    XKB_CUDA_TRY(cudaMemsetAsync(R->npred.p, 0, (nt + 1) * sizeof(uint32_t), st));
    for (size_t k = 0; k < R->useg.size(); ++k)
        if (R->useg_n[k])
            count_edges_kernel<<<(unsigned) ((R->useg_n[k] + 255) / 256), 256, 0, st>>>(R->useg[k]->p, R->useg_n[k], R->succ_ptr.p,
                                                                                       R->npred.p);
    if ((rc = device_exclusive_scan(R->succ_ptr.p, R->succ_ptr.p, nt + 1, R->tmp.p + nt + 1, nullptr, st))) return rc;
    XKB_CUDA_TRY(cudaMemcpyAsync(R->tmp.p, R->succ_ptr.p, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    for (size_t k = 0; k < R->useg.size(); ++k)
        if (R->useg_n[k])
            scatter_edges_kernel<<<(unsigned) ((R->useg_n[k] + 255) / 256), 256, 0, st>>>(R->useg[k]->p, R->useg_n[k], R->tmp.p,
                                                                                         R->succ.p);
    if (nt) sort_segments_kernel<<<(unsigned) ((nt + 255) / 256), 256, 0, st>>>(R->succ_ptr.p, R->succ.p, (uint32_t) nt);
    XKB_CUDA_TRY(cudaGetLastError());
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    R->graph_valid = true;
    return XKB_OK;
}

} // namespace xkb

extern "C" int xkb_resolver_create(xkb_resolver_t ** out, void * stream)
{
    if (!out) return xkb_set_error(XKB_EINVAL, "resolver_create: null output");
    int dev;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    xkb_resolver * R = new (std::nothrow) xkb_resolver();
    if (!R) return xkb_set_error(XKB_ENOMEM, "resolver_create: out of host memory");
    R->interval.interval = true;
    R->handles.interval = true;
    R->stream = (cudaStream_t) stream;
    // work buffers only this resolver's stream touches come from the pool in stream order (the
    // window graphs too: the runtime runs them on this stream); the graph it hands out
    // (succ_ptr, succ, npred, periodic form) stays in plain allocations, as a caller may read it
    // on other streams
    for (Domain * d : {&R->interval, &R->handles}) { d->state[0].use_pool(R->stream); d->state[1].use_pool(R->stream); }
    R->dops.use_pool(R->stream); R->hops.use_pool(R->stream);
    R->hset.use_pool(R->stream); R->ukeys.use_pool(R->stream); R->bounds.use_pool(R->stream); R->ucount.use_pool(R->stream);
    R->emit.use_pool(R->stream); R->table.use_pool(R->stream); R->counters.use_pool(R->stream);
    R->tmp.use_pool(R->stream); R->bin_off.use_pool(R->stream); R->bin_cur.use_pool(R->stream);
    R->bin_list.use_pool(R->stream); R->bin_flag.use_pool(R->stream); R->snap.use_pool(R->stream);
    R->win_ptr.use_pool(R->stream); R->win_succ.use_pool(R->stream); R->win_npred.use_pool(R->stream);
    R->win_tmp.use_pool(R->stream);
    *out = R;
    return XKB_OK;
}

extern "C" int xkb_resolver_destroy(xkb_resolver_t * R)
{
    if (R) { cudaStreamSynchronize(R->stream); delete R; }
    return XKB_OK;
}

// Library-internal: forget every task and domain but keep the device work buffers, so the
// next graph resolves without allocating them again.
// Reserve, up front, the working memory one batch of about `nops` ops uses (the buffers grow on
// demand otherwise): op lists, compression hash sets, emitted and unique edges, staging, the host
// team. The cell states of each domain depend on its boundaries and still grow on demand.
int xkb_internal_resolver_prepare(xkb_resolver_t * R, size_t nops)
{
    if (!R) return xkb_set_error(XKB_EINVAL, "resolver_prepare: null resolver");
    if (nops == 0) return XKB_OK;
    if (!R->pool)
    {
        R->pool.reset(new (std::nothrow) WorkPool(xkb_internal_helpers()));
    }
    size_t cap = 1024;
    while (cap < 4 * nops) cap *= 2;
    // edge pairs: about 9 per op on tile stencils (the emit estimate after the first batches)
    const size_t emit = std::max<size_t>(1 << 16, nops * 12);
    size_t tcap = 1024;
    while (tcap < 2 * emit) tcap *= 2;
    int rc;
    if ((rc = R->hops.reserve(nops)) || (rc = R->dops.reserve(nops)) || (rc = R->hset.reserve(2 * cap)) ||
        (rc = R->ukeys.reserve(4 * nops)) || (rc = R->ucount.reserve(3)) || (rc = R->emit.reserve(emit)) ||
        (rc = R->counters.reserve(2)) || (rc = R->table.reserve(tcap)) || (rc = R->stage.reserve(nops)) || (rc = spill_reserve(R, 1)))
        return rc;
    if (R->useg.empty())
    {
        std::unique_ptr<DevBuf<unsigned long long>> seg(new (std::nothrow) DevBuf<unsigned long long>());
        if (seg) seg->use_pool(R->stream);
        if (!seg) return xkb_set_error(XKB_ENOMEM, "resolver: out of host memory");
        if ((rc = seg->reserve(std::max<size_t>(emit, size_t(1) << 24)))) return rc;
        R->useg.push_back(std::move(seg));
        R->useg_n.push_back(0);
    }
    // the buffers still to come (cell states of each domain, region bins, time-split snapshots,
    // window graphs) grow from the pool: give it room now rather than while batches run
    if (cudaMemPool_t pool = resolver_pool())
    {
        void * w = nullptr;
        if (cudaMallocFromPoolAsync(&w, size_t(256) << 20, pool, R->stream) == cudaSuccess) cudaFreeAsync(w, R->stream);
        else cudaGetLastError();
    }
    XKB_CUDA_TRY(cudaStreamSynchronize(R->stream));
    return XKB_OK;
}

int xkb_internal_resolver_reset(xkb_resolver_t * R)
{
    if (!R) return xkb_set_error(XKB_EINVAL, "resolver_reset: null resolver");
    XKB_CUDA_TRY(cudaStreamSynchronize(R->stream));
    R->interval.xs.clear(); R->interval.ys.clear(); R->interval.ncells = 0; R->interval.ops.clear(); R->interval.nops = 0;
    R->handles.xs.clear(); R->handles.ys.clear(); R->handles.ncells = 0; R->handles.ops.clear(); R->handles.nops = 0;
    R->blas.clear(); R->blas_index.clear(); R->segments.clear();
    R->ntasks = 0; R->nuniq = 0; R->graph_valid = false;
    if (R->useg.size() > 1) { R->useg.resize(1); R->useg_n.resize(1); }   // keep the first edge segment
    for (size_t & n : R->useg_n) n = 0;
    R->spill_used = 0;
    return XKB_OK;
}

extern "C" int xkb_resolver_reset(xkb_resolver_t * R)
{
    return xkb_internal_resolver_reset(R);
}

extern "C" int xkb_resolver_add(xkb_resolver_t * R, const xkb_access_rec_t * recs, size_t n)
{
    if (!R || (n && !recs)) return xkb_set_error(XKB_EINVAL, "resolver_add: bad arguments");
    if (n == 0) return XKB_OK;
    if (!R->pool)
    {
        R->pool.reset(new (std::nothrow) WorkPool(xkb_internal_helpers()));
    }
    int rc = validate(R, recs, n, R->ntasks);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0, R->stream);
    rc = resolve_batch(R, recs, n);
    if (rc == XKB_OK) { R->ntasks = recs[n - 1].task + 1; R->graph_valid = false; }
    cudaEventRecord(e1, R->stream);
    cudaEventSynchronize(e1);
    float ms = 0; cudaEventElapsedTime(&ms, e0, e1);
    R->last_device_ms = ms;
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    return rc;
}

size_t xkb_internal_resolver_nedges(const xkb_resolver_t * R) { return R ? R->nuniq : 0; }

int xkb_internal_resolver_edge_mark(xkb_resolver_t * R, xkb_edge_mark_t * m)
{
    if (!R || !m) return xkb_set_error(XKB_EINVAL, "resolver_edge_mark: bad arguments");
    m->seg = R->useg.empty() ? 0 : R->useg.size() - 1;
    m->off = R->useg.empty() ? 0 : R->useg_n.back();
    m->ntasks = R->ntasks;
    return XKB_OK;
}

int xkb_internal_resolver_window_graph(xkb_resolver_t * R, const xkb_edge_mark_t * m, xkb_task_graph_t * g)
{
    if (!R || !m || !g || m->ntasks > R->ntasks) return xkb_set_error(XKB_EINVAL, "resolver_window_graph: bad arguments");
    const uint32_t first = m->ntasks;
    const size_t nt = R->ntasks - first;
    int rc;
    if ((rc = R->win_ptr.reserve(nt + 1)) || (rc = R->win_npred.reserve(nt + 1)) ||
        (rc = R->win_tmp.reserve(nt + 1 + (nt + 1) / SCAN_TILE + 2)))
        return rc;
    cudaStream_t st = R->stream;
    XKB_CUDA_TRY(cudaMemsetAsync(R->win_ptr.p, 0, (nt + 1) * sizeof(uint32_t), st));
    XKB_CUDA_TRY(cudaMemsetAsync(R->win_npred.p, 0, (nt + 1) * sizeof(uint32_t), st));
    // the edges stored since the mark: the rest of its segment, then every later segment
    auto each_range = [&](auto && fn) {
        for (size_t k = m->seg; k < R->useg.size(); ++k)
        {
            const size_t b = k == m->seg ? m->off : 0;
            if (R->useg_n[k] > b) fn(R->useg[k]->p + b, R->useg_n[k] - b);
        }
    };
    each_range([&](const unsigned long long * e, size_t n) {
        count_window_edges_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(e, n, first, R->win_ptr.p, R->win_npred.p);
    });
    if ((rc = device_exclusive_scan(R->win_ptr.p, R->win_ptr.p, nt + 1, R->win_tmp.p + nt + 1, nullptr, st))) return rc;
    uint32_t ne = 0;
    XKB_CUDA_TRY(cudaMemcpyAsync(&ne, R->win_ptr.p + nt, sizeof(ne), cudaMemcpyDeviceToHost, st));
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    if ((rc = R->win_succ.reserve(ne ? ne : 1))) return rc;
    XKB_CUDA_TRY(cudaMemcpyAsync(R->win_tmp.p, R->win_ptr.p, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    each_range([&](const unsigned long long * e, size_t n) {
        scatter_window_edges_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(e, n, first, R->win_tmp.p, R->win_succ.p);
    });
    if (nt) sort_segments_kernel<<<(unsigned) ((nt + 255) / 256), 256, 0, st>>>(R->win_ptr.p, R->win_succ.p, (uint32_t) nt);
    XKB_CUDA_TRY(cudaGetLastError());
    g->ntasks = nt;
    g->nedges = ne;
    g->succ_ptr = R->win_ptr.p;
    g->succ = R->win_succ.p;
    g->npred = R->win_npred.p;
    return XKB_OK;
}

extern "C" int xkb_resolver_graph(xkb_resolver_t * R, xkb_task_graph_t * g)
{
    if (!R || !g) return xkb_set_error(XKB_EINVAL, "resolver_graph: bad arguments");
    if (!R->graph_valid) { int rc = build_graph(R); if (rc) return rc; }
    g->ntasks = R->ntasks;
    g->nedges = R->nuniq;
    g->succ_ptr = R->succ_ptr.p;
    g->succ = R->succ.p;
    g->npred = R->npred.p;
    return XKB_OK;
}

extern "C" int xkb_resolver_edges(xkb_resolver_t * R, uint32_t * pairs, size_t cap_pairs, size_t * nedges)
{
    if (!R || !nedges) return xkb_set_error(XKB_EINVAL, "resolver_edges: bad arguments");
    if (!R->graph_valid) { int rc = build_graph(R); if (rc) return rc; }
    *nedges = R->nuniq;
    if (R->nuniq > cap_pairs) return xkb_set_error(XKB_ERANGE, "resolver_edges: %zu pairs needed", R->nuniq);
    if (!pairs || R->nuniq == 0) return XKB_OK;
    std::vector<uint32_t> ptr(R->ntasks + 1), succ(R->nuniq);
    XKB_CUDA_TRY(cudaMemcpy(ptr.data(), R->succ_ptr.p, ptr.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    XKB_CUDA_TRY(cudaMemcpy(succ.data(), R->succ.p, succ.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    size_t k = 0;
    for (uint32_t t = 0; t < R->ntasks; ++t)
        for (uint32_t i = ptr[t]; i < ptr[t + 1]; ++i) { pairs[2 * k] = t; pairs[2 * k + 1] = succ[i]; ++k; }
    return XKB_OK;
}

extern "C" int xkb_resolver_stats(xkb_resolver_t * R, uint64_t * ntasks, uint64_t * nedges, double * last_batch_ms)
{
    if (!R) return xkb_set_error(XKB_EINVAL, "resolver_stats: null resolver");
    if (ntasks) *ntasks = R->ntasks;
    if (nedges) *nedges = R->nuniq;
    if (last_batch_ms) *last_batch_ms = R->last_device_ms;
    return XKB_OK;
}

extern "C" int xkb_resolver_timing(xkb_resolver_t * R, double * ops_ms, double * compress_ms, double * batch_ms)
{
    if (!R) return xkb_set_error(XKB_EINVAL, "resolver_timing: null resolver");
    if (ops_ms) *ops_ms = R->last_ops_ms;
    if (compress_ms) *compress_ms = R->last_compress_ms;
    if (batch_ms) *batch_ms = R->last_device_ms;
    return XKB_OK;
}

extern "C" int xkb_resolver_periodic(xkb_resolver_t * R, uint64_t period, xkb_periodic_graph_t * out)
{
    if (!R || !out || period == 0) return xkb_set_error(XKB_EINVAL, "resolver_periodic: bad arguments");
    if (R->ntasks != 3 * period)
        return xkb_set_error(XKB_EINVAL, "resolver_periodic: the resolver must hold exactly 3 windows (%llu tasks), it holds %u",
                             (unsigned long long) (3 * period), R->ntasks);
    if (!R->graph_valid) { int rc = build_graph(R); if (rc) return rc; }
    const size_t nt = R->ntasks, P = period;
    std::vector<uint32_t> ptr(nt + 1), succ(R->nuniq ? R->nuniq : 1), npred(nt);
    XKB_CUDA_TRY(cudaMemcpy(ptr.data(), R->succ_ptr.p, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (R->nuniq) XKB_CUDA_TRY(cudaMemcpy(succ.data(), R->succ.p, R->nuniq * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    XKB_CUDA_TRY(cudaMemcpy(npred.data(), R->npred.p, nt * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    // split the successors of window w into its own window and the next one
    auto split = [&](size_t w, std::vector<uint32_t> & ip, std::vector<uint32_t> & is,
                     std::vector<uint32_t> & xp, std::vector<uint32_t> & xs) -> bool {
        ip.assign(1, 0); xp.assign(1, 0); is.clear(); xs.clear();
        for (size_t t = w * P; t < (w + 1) * P; ++t)
        {
            for (uint32_t i = ptr[t]; i < ptr[t + 1]; ++i)
            {
                const uint32_t s = succ[i];
                if (s < (w + 1) * P) is.push_back((uint32_t) (s - w * P));
                else if (s < (w + 2) * P) xs.push_back((uint32_t) (s - (w + 1) * P));
                else return false;                              // an edge skips a window
            }
            ip.push_back((uint32_t) is.size()); xp.push_back((uint32_t) xs.size());
        }
        return true;
    };
    std::vector<uint32_t> ip0, is0, xp0, xs0, ip1, is1, xp1, xs1;
    if (!split(0, ip0, is0, xp0, xs0) || !split(1, ip1, is1, xp1, xs1))
        return xkb_set_error(XKB_EINVAL, "resolver_periodic: an edge skips a window");
    std::vector<uint32_t> ip2, is2, xp2, xs2;
    {   // window 2's own edges (no next window was resolved)
        ip2.assign(1, 0);
        for (size_t t = 2 * P; t < 3 * P; ++t)
        {
            for (uint32_t i = ptr[t]; i < ptr[t + 1]; ++i) is2.push_back((uint32_t) (succ[i] - 2 * P));
            ip2.push_back((uint32_t) is2.size());
        }
    }
    if (ip0 != ip1 || is0 != is1 || xp0 != xp1 || xs0 != xs1 || ip0 != ip2 || is0 != is2 ||
        !std::equal(npred.begin() + P, npred.begin() + 2 * P, npred.begin() + 2 * P))
        return xkb_set_error(XKB_EINVAL, "resolver_periodic: the windows do not repeat");
    // pack: succ_ptr | succ | xsucc_ptr | xsucc | npred_first | npred_next
    const size_t total = (P + 1) + is0.size() + (P + 1) + xs0.size() + P + P;
    int rc = R->periodic.reserve(total ? total : 1);
    if (rc) return rc;
    std::vector<uint32_t> h;
    h.reserve(total);
    h.insert(h.end(), ip0.begin(), ip0.end());
    h.insert(h.end(), is0.begin(), is0.end());
    h.insert(h.end(), xp0.begin(), xp0.end());
    h.insert(h.end(), xs0.begin(), xs0.end());
    h.insert(h.end(), npred.begin(), npred.begin() + P);
    h.insert(h.end(), npred.begin() + P, npred.begin() + 2 * P);
    XKB_CUDA_TRY(cudaMemcpy(R->periodic.p, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    const uint32_t * d = R->periodic.p;
    out->period = P;
    out->succ_ptr = d; d += P + 1;
    out->succ = d; d += is0.size();
    out->xsucc_ptr = d; d += P + 1;
    out->xsucc = d; d += xs0.size();
    out->npred_first = d; d += P;
    out->npred_next = d;
    return XKB_OK;
}
