// Execution of a transfer plan and the replica-layout heat tile body.
//
// xkb_plan_execute runs a list of planned copies in order on one stream: host<->device copies
// with cudaMemcpy2DAsync (the reference issues one cuMemcpy2DAsync per copy command,
// src/driver/driver_cu.cc:671-761), and the device-to-device copies one access issues as ONE
// gather kernel launch -- one CTA per copy, 16-, 8- or 1-byte moves depending on alignment --
// instead of one copy command each. The copies of one access never alias one another: they
// fill distinct blocks of the access, from views that were coherent before the access. Copies
// of different accesses may (a later access can read what an earlier copy wrote), so a batch
// never spans two accesses.
//
// Host copies are coalesced first: within a run of consecutive copies of one direction (all H2D
// or all D2H) no copy reads what another writes, so their order is free, and blocks that are
// side by side in both address spaces merge into one wider copy, then copies stacked at the
// same pitch merge into one taller copy. A canonical block partition cuts a tile's data into
// many small blocks; merged, a whole band of tiles moves as one cudaMemcpy2DAsync.
//
// xkb_diffusion_views is the reference's tile body contract (diffusion_cuda,
// examples/heat-diffusion-2d/src/kernels/diffusion.cu:107-154) on per-access replicas:
// src/dst point at the tile origin after the launcher's re-basing (main.cc:214-219), with their
// own leading dimensions.
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <atomic>
#include <vector>

namespace xkb {

struct D2D { const uint8_t * src; uint8_t * dst; int64_t src_pitch, dst_pitch, row_bytes, rows; };

__global__ void __launch_bounds__(256) d2d_gather_kernel(const D2D * __restrict__ ops)
{
    const D2D o = ops[blockIdx.x];
    const bool a16 = ((((uintptr_t) o.src) | ((uintptr_t) o.dst) | o.src_pitch | o.dst_pitch | o.row_bytes) & 15) == 0;
    const bool a8 = ((((uintptr_t) o.src) | ((uintptr_t) o.dst) | o.src_pitch | o.dst_pitch | o.row_bytes) & 7) == 0;
    if (a16)
    {
        const int64_t w = o.row_bytes / 16, total = w * o.rows;
        for (int64_t k = threadIdx.x; k < total; k += blockDim.x)
        {
            const int64_t r = k / w, c = k % w;
            *(uint4 *) (o.dst + r * o.dst_pitch + c * 16) = *(const uint4 *) (o.src + r * o.src_pitch + c * 16);
        }
    }
    else if (a8)
    {
        const int64_t w = o.row_bytes / 8, total = w * o.rows;
        for (int64_t k = threadIdx.x; k < total; k += blockDim.x)
        {
            const int64_t r = k / w, c = k % w;
            *(uint2 *) (o.dst + r * o.dst_pitch + c * 8) = *(const uint2 *) (o.src + r * o.src_pitch + c * 8);
        }
    }
    else
    {
        const int64_t total = o.row_bytes * o.rows;
        for (int64_t k = threadIdx.x; k < total; k += blockDim.x)
        {
            const int64_t r = k / o.row_bytes, c = k % o.row_bytes;
            o.dst[r * o.dst_pitch + c] = o.src[r * o.src_pitch + c];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) diffusion_views_kernel(const T * __restrict__ src, int64_t ld_src, T * __restrict__ dst,
                                                              int64_t ld_dst, int64_t i0, int64_t j0, int64_t tsx, int64_t tsy,
                                                              int64_t nx, int64_t ny, double c)
{
    const int64_t li = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t lj = blockIdx.y; lj < tsy; lj += gridDim.y)
    {
        const int64_t i = i0 + li, j = j0 + lj;
        if (li >= tsx || !(i > 0 && i < nx - 1 && j > 0 && j < ny - 1)) continue;
        const T * s = src + lj * ld_src + li;
        const double sv = (double) s[0];
        const double s2 = __dmul_rn(2.0, sv);
        const double a = __dadd_rn(__dsub_rn((double) s[1], s2), (double) s[-1]);
        const double b = __dadd_rn(__dsub_rn((double) s[ld_src], s2), (double) s[-ld_src]);
        dst[lj * ld_dst + li] = (T) __dadd_rn(sv, __dmul_rn(c, __dadd_rn(a, b)));
    }
}

} // namespace xkb

using namespace xkb;

// One host copy: rows x width bytes from src (pitch sp) to dst (pitch dp). A byte range of a
// segment has no pitch (sp = dp = 0): such ranges merge whenever they continue each other.
// `alloc`: the device allocation the copy touches, and in its high bits the span of host memory
// between two cuts its host bytes lie in -- copies of different allocations or spans never merge
// (adjacent allocations, host or device, are still separate allocations to the driver, and a
// copy may not run across the end of one; the cuts are the ends of page-locked pieces).
struct HostCopy { uintptr_t src, dst; int64_t sp, dp, width, rows; int64_t alloc; };

static size_t coalesce(std::vector<HostCopy> & v)
{
    if (v.size() < 2) return v.size();
    // side by side: same rows and pitches, each continuing the previous one in both spaces (byte
    // ranges: any widths)
    std::sort(v.begin(), v.end(), [](const HostCopy & a, const HostCopy & b) {
        if (a.alloc != b.alloc) return a.alloc < b.alloc;
        if (a.sp != b.sp) return a.sp < b.sp;
        if (a.dp != b.dp) return a.dp < b.dp;
        if (a.rows != b.rows) return a.rows < b.rows;
        return a.src < b.src;
    });
    size_t k = 0;
    for (size_t i = 1; i < v.size(); ++i)
    {
        HostCopy & a = v[k];
        const HostCopy & b = v[i];
        const bool range = a.sp == 0 && a.dp == 0;
        if (a.alloc == b.alloc && a.sp == b.sp && a.dp == b.dp && a.rows == b.rows && b.src == a.src + (uintptr_t) a.width &&
            b.dst == a.dst + (uintptr_t) a.width && (range || a.rows == 1 || a.width + b.width <= std::min(a.sp, a.dp)))
        {
            a.width += b.width;
            if (a.rows == 1 && !range) { a.sp = std::max(a.sp, a.width); a.dp = std::max(a.dp, a.width); }
        }
        else v[++k] = b;
    }
    v.resize(k + 1);
    // stacked: same width and pitches, each starting one pitch x rows below the previous one
    std::sort(v.begin(), v.end(), [](const HostCopy & a, const HostCopy & b) {
        if (a.alloc != b.alloc) return a.alloc < b.alloc;
        if (a.sp != b.sp) return a.sp < b.sp;
        if (a.dp != b.dp) return a.dp < b.dp;
        if (a.width != b.width) return a.width < b.width;
        return a.src < b.src;
    });
    k = 0;
    for (size_t i = 1; i < v.size(); ++i)
    {
        HostCopy & a = v[k];
        const HostCopy & b = v[i];
        if (a.alloc == b.alloc && a.sp == b.sp && a.dp == b.dp && a.width == b.width && a.width <= std::min(a.sp, a.dp) &&
            b.src == a.src + (uintptr_t) (a.rows * a.sp) && b.dst == a.dst + (uintptr_t) (a.rows * a.dp))
            a.rows += b.rows;
        else v[++k] = b;
    }
    v.resize(k + 1);
    return v.size();
}

static std::atomic<uint64_t> g_issued_host_copies{0};     // after coalescing (traces)

static int issue_host_copies(std::vector<HostCopy> & v, cudaMemcpyKind kind, cudaStream_t st)
{
    coalesce(v);
    g_issued_host_copies.fetch_add(v.size(), std::memory_order_relaxed);
    for (const HostCopy & c : v)
    {
        // a contiguous range (one row, or full-pitch rows) as a plain copy, else pitched
        const bool flat = c.rows == 1 || (c.width == c.sp && c.width == c.dp);
        cudaError_t e = flat ? cudaMemcpyAsync((void *) c.dst, (const void *) c.src, (size_t) (c.width * c.rows), kind, st)
                             : cudaMemcpy2DAsync((void *) c.dst, (size_t) c.dp, (const void *) c.src, (size_t) c.sp,
                                                 (size_t) c.width, (size_t) c.rows, kind, st);
        if (e != cudaSuccess)
            return xkb_set_error(e == cudaErrorMemoryAllocation ? XKB_ENOMEM : XKB_ECUDA,
                                 "CUDA: %s (%s of %lld x %lld bytes, %p pitch %lld -> %p pitch %lld)", cudaGetErrorString(e),
                                 kind == cudaMemcpyHostToDevice ? "H2D" : "D2H", (long long) c.rows, (long long) c.width,
                                 (const void *) c.src, (long long) c.sp, (void *) c.dst, (long long) c.dp);
    }
    v.clear();
    return XKB_OK;
}

static int plan_execute(const xkb_copy_t * copies, size_t n, void * const * alloc_ptrs, size_t nallocs, cudaStream_t st,
                        const uint64_t * cuts, size_t ncuts)
{
    if (n && (!copies || !alloc_ptrs)) return xkb_set_error(XKB_EINVAL, "plan_execute: bad arguments");
    auto tag = [&](int64_t alloc, uint64_t host) -> int64_t {
        const int64_t span = cuts ? (int64_t) (std::upper_bound(cuts, cuts + ncuts, host) - cuts) : 0;
        return (span << 32) | (alloc & 0xffffffff);
    };
    auto dev_ptr = [&](int64_t alloc, int64_t off) -> uint8_t * {
        return (alloc >= 0 && (size_t) alloc < nallocs) ? (uint8_t *) alloc_ptrs[alloc] + off : nullptr;
    };
    std::vector<D2D> batch;
    D2D * dbatch = nullptr;
    size_t dcap = 0;
    auto flush = [&]() -> int {
        if (batch.empty()) return XKB_OK;
        if (batch.size() > dcap)
        {
            if (dbatch) { cudaStreamSynchronize(st); cudaFree(dbatch); }
            dcap = batch.size() * 2;
            cudaError_t e = cudaMalloc(&dbatch, dcap * sizeof(D2D));
            if (e != cudaSuccess) { dbatch = nullptr; return xkb_set_cuda_error(e); }
        }
        else cudaStreamSynchronize(st);   // the previous batch must have been consumed
        cudaError_t e = cudaMemcpyAsync(dbatch, batch.data(), batch.size() * sizeof(D2D), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        d2d_gather_kernel<<<(unsigned) batch.size(), 256, 0, st>>>(dbatch);
        e = cudaGetLastError();
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        cudaStreamSynchronize(st);         // `batch` (pageable) is reused after this
        batch.clear();
        return XKB_OK;
    };
    std::vector<HostCopy> hrun;          // pending run of host copies, all of kind hkind
    int64_t hkind = -1;
    int rc = XKB_OK;
    for (size_t i = 0; i < n && rc == XKB_OK; ++i)
    {
        const xkb_copy_t & c = copies[i];
        const int64_t row_bytes = c.m * c.sizeof_type;
        const int64_t sp = c.src_ld ? c.src_ld * c.sizeof_type : row_bytes, dp = c.dst_ld ? c.dst_ld * c.sizeof_type : row_bytes;
        if (c.kind != hkind && !hrun.empty() &&
            (rc = issue_host_copies(hrun, hkind == XKB_COPY_H2D ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, st)))
            break;
        if (c.kind == XKB_COPY_D2D)
        {
            if (i > 0 && (copies[i - 1].task != c.task || copies[i - 1].access != c.access) && (rc = flush())) break;
            uint8_t * s = dev_ptr(c.src_alloc, c.src_off), * d = dev_ptr(c.dst_alloc, c.dst_off);
            if (!s || !d) { rc = xkb_set_error(XKB_EINVAL, "plan_execute: copy %zu names an unknown allocation", i); break; }
            batch.push_back({s, d, sp, dp, row_bytes, c.n});
            hkind = c.kind;
            continue;
        }
        if ((rc = flush())) break;
        if (row_bytes <= 0 || c.n <= 0) { hkind = c.kind; continue; }   // nothing to move
        if (c.kind == XKB_COPY_H2D)
        {
            uint8_t * d = dev_ptr(c.dst_alloc, c.dst_off);
            if (!d) { rc = xkb_set_error(XKB_EINVAL, "plan_execute: copy %zu names an unknown allocation", i); break; }
            const bool range = c.src_ld == 0 && c.dst_ld == 0 && c.n == 1;
            hrun.push_back({(uintptr_t) c.src_off, (uintptr_t) d, range ? 0 : sp, range ? 0 : dp, row_bytes, c.n,
                            tag(c.dst_alloc, (uint64_t) c.src_off)});
        }
        else if (c.kind == XKB_COPY_D2H)
        {
            const uint8_t * s = dev_ptr(c.src_alloc, c.src_off);
            if (!s) { rc = xkb_set_error(XKB_EINVAL, "plan_execute: copy %zu names an unknown allocation", i); break; }
            const bool range = c.src_ld == 0 && c.dst_ld == 0 && c.n == 1;
            hrun.push_back({(uintptr_t) s, (uintptr_t) c.dst_off, range ? 0 : sp, range ? 0 : dp, row_bytes, c.n,
                            tag(c.src_alloc, (uint64_t) c.dst_off)});
        }
        else { rc = xkb_set_error(XKB_EINVAL, "plan_execute: copy %zu has an unknown kind", i); break; }
        hkind = c.kind;
    }
    if (rc == XKB_OK && !hrun.empty())
        rc = issue_host_copies(hrun, hkind == XKB_COPY_H2D ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, st);
    if (rc == XKB_OK) rc = flush();
    if (dbatch) { cudaStreamSynchronize(st); cudaFree(dbatch); }
    return rc;
}

extern "C" int xkb_plan_execute(const xkb_copy_t * copies, size_t n, void * const * alloc_ptrs, size_t nallocs, void * stream)
{
    return plan_execute(copies, n, alloc_ptrs, nallocs, xkb_stream(stream), nullptr, 0);
}

uint64_t xkb_internal_issued_host_copies() { return g_issued_host_copies.load(std::memory_order_relaxed); }

int xkb_internal_plan_execute_cut(const xkb_copy_t * copies, size_t n, void * const * alloc_ptrs, size_t nallocs,
                                  cudaStream_t stream, const uint64_t * cuts, size_t ncuts)
{
    return plan_execute(copies, n, alloc_ptrs, nallocs, stream, ncuts ? cuts : nullptr, ncuts);
}

// The cells [i0, i0 + w) x [j0, j0 + h) of the grid (interior ones only), src and dst pointing at
// cell (i0, j0) of their replicas.
int xkb_internal_diffusion_box(int dtype, cudaStream_t stream, const void * src, int64_t ld_src, void * dst, int64_t ld_dst,
                               int64_t i0, int64_t j0, int64_t w, int64_t h, int64_t nx, int64_t ny, double c)
{
    if ((dtype != XKB_F64 && dtype != XKB_F32) || !src || !dst || w <= 0 || h <= 0)
        return xkb_set_error(XKB_EINVAL, "diffusion_views: bad arguments");
    const dim3 block(256), grid((unsigned) ((w + 255) / 256), (unsigned) (h < 1024 ? h : 1024));
    if (dtype == XKB_F64)
        diffusion_views_kernel<double><<<grid, block, 0, stream>>>((const double *) src, ld_src, (double *) dst, ld_dst, i0, j0, w, h, nx, ny, c);
    else
        diffusion_views_kernel<float><<<grid, block, 0, stream>>>((const float *) src, ld_src, (float *) dst, ld_dst, i0, j0, w, h, nx, ny, c);
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

extern "C" int xkb_diffusion_views(int dtype, void * stream, const void * src, int64_t ld_src, void * dst, int64_t ld_dst,
                                   int64_t tile_x, int64_t tile_y, int64_t tsx, int64_t tsy, int64_t nx, int64_t ny, double c)
{
    if (tsx <= 0 || tsy <= 0) return xkb_set_error(XKB_EINVAL, "diffusion_views: bad arguments");
    return xkb_internal_diffusion_box(dtype, xkb_stream(stream), src, ld_src, dst, ld_dst, tile_x * tsx, tile_y * tsy, tsx, tsy, nx,
                                      ny, c);
}
