// Heat-diffusion-2d kernels: per-task tile launch (the plain form, one launch per tile task)
// and the whole-step launch (all tile tasks of one step fused into one grid).
#include "heat.cuh"

namespace xkb {

constexpr int HEAT_THREADS = 256;   // 8 warps per CTA
constexpr int HEAT_PF = 6;          // east columns in flight per lane
constexpr int STEP_COLS = 64;       // columns per warp strip in the whole-step kernel

template <typename T, int VEC>
__global__ void __launch_bounds__(HEAT_THREADS, 2)
heat_tile_kernel(const T * __restrict__ src, T * __restrict__ dst, int64_t ld, int64_t nx, int64_t ny,
                 int64_t x0, int64_t x1, int64_t y0, int64_t y1, double c, bool vec_ok)
{
    // blockIdx.x selects a column slab of the tile so one task can still use several SMs.
    const int64_t cols = y1 - y0;
    const int64_t per = (cols + gridDim.x - 1) / gridDim.x;
    const int64_t a = y0 + (int64_t) blockIdx.x * per;
    int64_t b = a + per; if (b > y1) b = y1;
    if (a >= b) return;
    heat_tile_cta<T, VEC, HEAT_PF, false>(src, dst, ld, nx, ny, x0, x1, a, b, c, vec_ok, 8);
}

template <typename T, int VEC, int PF, int MINB>
__global__ void __launch_bounds__(HEAT_THREADS, MINB)
heat_step_kernel(const T * __restrict__ src, T * __restrict__ dst, int64_t ld, int64_t nx, int64_t ny,
                 int64_t nrg, int64_t ncc, int64_t cols, double c, bool vec_ok, int pfd)
{
    const int64_t warps = (int64_t) gridDim.x * (HEAT_THREADS / 32);
    const int64_t nstrips = nrg * ncc;
    for (int64_t s = (int64_t) blockIdx.x * (HEAT_THREADS / 32) + (threadIdx.x >> 5); s < nstrips; s += warps)
    {
        // consecutive warps take consecutive row groups of the same column chunk, so a CTA
        // sweeps a contiguous panel of the grid
        const int64_t rg = s % nrg, cc = s / nrg;
        const int64_t cy0 = 1 + cc * cols;
        int64_t cy1 = cy0 + cols; if (cy1 > ny - 1) cy1 = ny - 1;
        heat_strip<T, VEC, PF, false>(src, dst, ld, nx, ny, rg * StripGeom<VEC>::OUT, 1, nx - 1, cy0, cy1, c, vec_ok, pfd);
    }
}

template <typename T>
static bool vec_ok_for(const void * src, const void * dst, int64_t ld)
{
    constexpr int VEC = HeatVec<T>::N;
    return (ld % VEC == 0) && ((uintptr_t) src % 16 == 0) && ((uintptr_t) dst % 16 == 0);
}

template <typename T>
static int launch_tile(const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                       int64_t x0, int64_t x1, int64_t y0, int64_t y1, double c, cudaStream_t st)
{
    constexpr int VEC = HeatVec<T>::N;
    const TileBox b = heat_tile_box(nx, ny, x0, x1, y0, y1);
    if (b.rx0 >= b.rx1 || b.cy0 >= b.cy1) return XKB_OK;
    // one CTA per 32 columns of the tile (a 128x128 tile runs on 4 SMs)
    const int64_t cols = b.cy1 - b.cy0;
    int grid = (int) ((cols + 31) / 32); if (grid < 1) grid = 1;
    heat_tile_kernel<T, VEC><<<grid, HEAT_THREADS, 0, st>>>((const T *) src, (T *) dst, ld, nx, ny,
                                                           b.rx0, b.rx1, b.cy0, b.cy1, c, vec_ok_for<T>(src, dst, ld));
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

static int sm_count()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    return sms;
}

template <typename T, int PF, int MINB>
static void step_launch(dim3 g, cudaStream_t st, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                        int64_t nrg, int64_t ncc, int64_t cols, double c, bool vok, int pfd)
{
    heat_step_kernel<T, HeatVec<T>::N, PF, MINB><<<g, HEAT_THREADS, 0, st>>>((const T *) src, (T *) dst, ld, nx, ny,
                                                                          nrg, ncc, cols, c, vok, pfd);
}

template <typename T>
static int launch_step(const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny, double c,
                       const xkb_heat_cfg_t & cfg, cudaStream_t st)
{
    constexpr int VEC = HeatVec<T>::N;
    if (nx < 3 || ny < 3) return XKB_OK;
    const int64_t cols = cfg.cols_per_strip > 0 ? cfg.cols_per_strip : 64;
    const int64_t nrg = (nx - 2 + StripGeom<VEC>::OUT - 1) / StripGeom<VEC>::OUT;
    const int64_t ncc = (ny - 2 + cols - 1) / cols;
    const int64_t ctas_needed = (nrg * ncc + (HEAT_THREADS / 32) - 1) / (HEAT_THREADS / 32);
    int64_t grid = (int64_t) sm_count() * (cfg.ctas_per_sm > 0 ? cfg.ctas_per_sm : 8);
    if (grid > ctas_needed) grid = ctas_needed;
    const bool vok = vec_ok_for<T>(src, dst, ld);
    const dim3 g((unsigned) grid);
    const int pfd = cfg.l2_prefetch_cols;
    switch (cfg.pf * 10 + cfg.min_blocks)
    {
        case 21: step_launch<T, 2, 1>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        case 22: step_launch<T, 2, 2>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        case 24: step_launch<T, 2, 4>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        case 41: step_launch<T, 4, 1>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        case 42: step_launch<T, 4, 2>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        case 81: step_launch<T, 8, 1>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        case 82: step_launch<T, 8, 2>(g, st, src, dst, ld, nx, ny, nrg, ncc, cols, c, vok, pfd); break;
        default: return xkb_set_error(XKB_EINVAL, "heat_step: unsupported (pf=%d, min_blocks=%d)", cfg.pf, cfg.min_blocks);
    }
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

} // namespace xkb

using namespace xkb;

static int heat_check(int dtype, const void * src, const void * dst, int64_t ld, int64_t nx, int64_t ny)
{
    if (dtype != XKB_F64 && dtype != XKB_F32) return xkb_set_error(XKB_EINVAL, "heat: dtype must be XKB_F64 or XKB_F32");
    if (!src || !dst || src == dst) return xkb_set_error(XKB_EINVAL, "heat: src and dst must be distinct device grids");
    if (nx < 0 || ny < 0 || ld < nx) return xkb_set_error(XKB_EINVAL, "heat: need 0 <= nx <= ld and ny >= 0");
    return XKB_OK;
}

extern "C" int xkb_heat_tile(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                             int64_t tile_x, int64_t tile_y, int64_t tsx, int64_t tsy, double c, void * stream)
{
    int rc = heat_check(dtype, src, dst, ld, nx, ny);
    if (rc) return rc;
    if (tsx <= 0 || tsy <= 0 || tile_x < 0 || tile_y < 0) return xkb_set_error(XKB_EINVAL, "heat_tile: bad tile");
    const int64_t x0 = tile_x * tsx, y0 = tile_y * tsy;
    const int64_t x1 = x0 + tsx, y1 = y0 + tsy;
    return dtype == XKB_F64 ? launch_tile<double>(src, dst, ld, nx, ny, x0, x1, y0, y1, c, xkb_stream(stream))
                            : launch_tile<float>(src, dst, ld, nx, ny, x0, x1, y0, y1, c, xkb_stream(stream));
}

static const xkb_heat_cfg_t kDefaultStepCfg = {4, 2, 8, 8, 64};

extern "C" int xkb_heat_step(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                             double c, void * stream)
{
    return xkb_heat_step_cfg(dtype, src, dst, ld, nx, ny, c, &kDefaultStepCfg, stream);
}

extern "C" int xkb_heat_step_cfg(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                                 double c, const xkb_heat_cfg_t * cfg, void * stream)
{
    int rc = heat_check(dtype, src, dst, ld, nx, ny);
    if (rc) return rc;
    const xkb_heat_cfg_t & k = cfg ? *cfg : kDefaultStepCfg;
    if (k.l2_prefetch_cols < 0 || k.l2_prefetch_cols > 256 || k.cols_per_strip < 0)
        return xkb_set_error(XKB_EINVAL, "heat_step: bad configuration");
    return dtype == XKB_F64 ? launch_step<double>(src, dst, ld, nx, ny, c, k, xkb_stream(stream))
                            : launch_step<float>(src, dst, ld, nx, ny, c, k, xkb_stream(stream));
}

// ---- FP64 checks of a step's result ---------------------------------------------------------
namespace {

// Non-negative doubles order like their bit patterns, so an integer max is a double max.
__device__ __forceinline__ void atomic_max_nonneg(double * p, double v)
{
    atomicMax((unsigned long long *) p, (unsigned long long) __double_as_longlong(v));
}

// out[0] max |dst| on the boundary, out[1] sum of dst^2 over the interior, out[2] max over the
// interior of |dst - (src + c*lap(src))| with src promoted to double, out[3] max |dst| interior.
// One block per column band; threads over rows; all arithmetic in double.
template <typename T>
__global__ void __launch_bounds__(256) heat_norms_kernel(const T * __restrict__ src, const T * __restrict__ dst, int64_t ld,
                                                         int64_t nx, int64_t ny, double c, double * out)
{
    double bmax = 0, sum = 0, rmax = 0, vmax = 0;
    for (int64_t j = blockIdx.x; j < ny; j += gridDim.x)
        for (int64_t i = threadIdx.x; i < nx; i += blockDim.x)
        {
            const double d = (double) dst[j * ld + i];
            if (i == 0 || j == 0 || i == nx - 1 || j == ny - 1) { bmax = fmax(bmax, fabs(d)); continue; }
            const T * s = src + j * ld + i;
            const double v = (double) s[0];
            const double a = __dadd_rn(__dsub_rn((double) s[1], __dmul_rn(2.0, v)), (double) s[-1]);
            const double b = __dadd_rn(__dsub_rn((double) s[ld], __dmul_rn(2.0, v)), (double) s[-ld]);
            const double e = __dadd_rn(v, __dmul_rn(c, __dadd_rn(a, b)));
            rmax = fmax(rmax, fabs(d - e));
            vmax = fmax(vmax, fabs(d));
            sum += d * d;
        }
    for (int o = 16; o > 0; o >>= 1)
    {
        bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
        rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        atomic_max_nonneg(out + 0, bmax);
        atomicAdd(out + 1, sum);
        atomic_max_nonneg(out + 2, rmax);
        atomic_max_nonneg(out + 3, vmax);
    }
}

} // namespace

extern "C" int xkb_heat_norms(int dtype, const void * src, const void * dst, int64_t ld, int64_t nx, int64_t ny, double c,
                              double * out, void * stream)
{
    int rc = heat_check(dtype, src, dst, ld, nx, ny);
    if (rc) return rc;
    if (!out) return xkb_set_error(XKB_EINVAL, "heat_norms: null output");
    cudaStream_t st = xkb_stream(stream);
    XKB_CUDA_TRY(cudaMemsetAsync(out, 0, 4 * sizeof(double), st));
    if (nx == 0 || ny == 0) return XKB_OK;
    int dev = 0, sms = 148;
    XKB_CUDA_TRY(cudaGetDevice(&dev));
    XKB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned grid = (unsigned) std::min<int64_t>(ny, (int64_t) sms * 8);
    if (dtype == XKB_F64) heat_norms_kernel<double><<<grid, 256, 0, st>>>((const double *) src, (const double *) dst, ld, nx, ny, c, out);
    else heat_norms_kernel<float><<<grid, 256, 0, st>>>((const float *) src, (const float *) dst, ld, nx, ny, c, out);
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}
