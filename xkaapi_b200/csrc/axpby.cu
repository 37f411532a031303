// axpby tile body: y = a*x + b*y over FP64 vectors, 128-bit vectorised grid-stride loop.
#include "common.cuh"

namespace xkb {

__device__ __forceinline__ double axpby1(double a, double x, double b, double y)
{
    return __dadd_rn(__dmul_rn(a, x), __dmul_rn(b, y));   // (a*x) + (b*y), no FMA
}

// Body over [lo, hi): the CTA's threads stride through it; used by the per-task kernel and
// by the persistent scheduler. Peeled scalar head/tail keep the double2 accesses aligned.
template <bool CG>
__device__ __forceinline__ void axpby_range(int64_t lo, int64_t hi, double a, const double * __restrict__ x,
                                            double b, double * __restrict__ y, int64_t tid, int64_t nthreads)
{
    if (lo >= hi) return;
    const bool same_phase = (((uintptr_t) (x + lo)) & 15) == (((uintptr_t) (y + lo)) & 15);
    int64_t head = lo;
    if (same_phase && (((uintptr_t) (y + lo)) & 15)) head = lo + 1;
    if (!same_phase) head = hi;   // misaligned against each other: scalar loop
    if (head > hi) head = hi;
    for (int64_t i = lo + tid; i < head; i += nthreads)
        y[i] = axpby1(a, CG ? __ldcg(x + i) : __ldg(x + i), b, CG ? __ldcg(y + i) : y[i]);
    const int64_t nv = (hi - head) / 2;
    const double2 * xv = (const double2 *) (x + head);
    double2 * yv = (double2 *) (y + head);
    for (int64_t v = tid; v < nv; v += nthreads)
    {
        const double2 xx = CG ? __ldcg(xv + v) : __ldg(xv + v);
        const double2 yy = CG ? __ldcg(yv + v) : yv[v];
        yv[v] = make_double2(axpby1(a, xx.x, b, yy.x), axpby1(a, xx.y, b, yy.y));
    }
    for (int64_t i = head + 2 * nv + tid; i < hi; i += nthreads)
        y[i] = axpby1(a, CG ? __ldcg(x + i) : __ldg(x + i), b, CG ? __ldcg(y + i) : y[i]);
}

__global__ void __launch_bounds__(256) axpby_kernel(int64_t n, double a, const double * __restrict__ x, double b, double * __restrict__ y)
{
    axpby_range<false>(0, n, a, x, b, y, (int64_t) blockIdx.x * blockDim.x + threadIdx.x, (int64_t) gridDim.x * blockDim.x);
}

} // namespace xkb

extern "C" int xkb_axpby(int64_t n, double a, const double * x, double b, double * y, void * stream)
{
    if (n < 0 || (n > 0 && (!x || !y))) return xkb_set_error(XKB_EINVAL, "axpby: bad arguments");
    if (n == 0) return XKB_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t want = (n / 2 + 255) / 256;
    int64_t grid = sms * 8;
    if (grid > want) grid = want > 0 ? want : 1;
    xkb::axpby_kernel<<<(unsigned) grid, 256, 0, xkb_stream(stream)>>>(n, a, x, b, y);
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}
