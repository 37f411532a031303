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
    heat_tile_cta<T, VEC, HEAT_PF, false>(src, dst, ld, nx, ny, x0, x1, a, b, c, vec_ok);
}

template <typename T, int VEC>
__global__ void __launch_bounds__(HEAT_THREADS, 2)
heat_step_kernel(const T * __restrict__ src, T * __restrict__ dst, int64_t ld, int64_t nx, int64_t ny,
                 int64_t nrg, int64_t ncc, double c, bool vec_ok)
{
    const int64_t warps = (int64_t) gridDim.x * (HEAT_THREADS / 32);
    const int64_t nstrips = nrg * ncc;
    for (int64_t s = (int64_t) blockIdx.x * (HEAT_THREADS / 32) + (threadIdx.x >> 5); s < nstrips; s += warps)
    {
        // consecutive warps take consecutive row groups of the same column chunk, so a CTA
        // sweeps a contiguous panel and its halo rows are shared through L2
        const int64_t rg = s % nrg, cc = s / nrg;
        const int64_t cy0 = 1 + cc * STEP_COLS;
        int64_t cy1 = cy0 + STEP_COLS; if (cy1 > ny - 1) cy1 = ny - 1;
        heat_strip<T, VEC, HEAT_PF, false>(src, dst, ld, nx, rg * 32 * VEC, 1, nx - 1, cy0, cy1, c, vec_ok);
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

template <typename T>
static int launch_step(const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny, double c, cudaStream_t st)
{
    constexpr int VEC = HeatVec<T>::N;
    if (nx < 3 || ny < 3) return XKB_OK;
    const int64_t nrg = (nx - 1 + 32 * VEC - 1) / (32 * VEC);
    const int64_t ncc = (ny - 2 + STEP_COLS - 1) / STEP_COLS;
    const int64_t ctas_needed = (nrg * ncc + (HEAT_THREADS / 32) - 1) / (HEAT_THREADS / 32);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t grid = sms * 8;   // grid-stride over strips, several CTAs resident per SM
    if (grid > ctas_needed) grid = ctas_needed;
    heat_step_kernel<T, VEC><<<(unsigned) grid, HEAT_THREADS, 0, st>>>((const T *) src, (T *) dst, ld, nx, ny,
                                                                      nrg, ncc, c, vec_ok_for<T>(src, dst, ld));
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

extern "C" int xkb_heat_step(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                             double c, void * stream)
{
    int rc = heat_check(dtype, src, dst, ld, nx, ny);
    if (rc) return rc;
    return dtype == XKB_F64 ? launch_step<double>(src, dst, ld, nx, ny, c, xkb_stream(stream))
                            : launch_step<float>(src, dst, ld, nx, ny, c, xkb_stream(stream));
}
