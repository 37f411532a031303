// The user tile kernel of examples/heat_cxx.cc: what a program brings along with its own CUDA
// task body (the reference's examples/heat-diffusion-2d/src/kernels/diffusion.cu plays this part
// there), in FP64 with the reference's update written as separate IEEE operations (no fused
// multiply-add) so the grid can be compared bit for bit with the oracle:
//   D(i,j) = S(i,j) + c*(((S(i+1,j) - 2S(i,j)) + S(i-1,j)) + ((S(i,j+1) - 2S(i,j)) + S(i,j-1)))
// (examples/heat-diffusion-2d/src/main.cc:408-421). One thread per cell of the tile.
#include <cuda_runtime.h>

__global__ void heat_cxx_tile_kernel(const double * __restrict__ src, long ld_src, double * __restrict__ dst, long ld_dst,
                                     long nx, long ny, long x, long y, long ts, double c)
{
    const long li = blockIdx.x * (long) blockDim.x + threadIdx.x, lj = blockIdx.y * (long) blockDim.y + threadIdx.y;
    const long i = x + li, j = y + lj;
    if (li >= ts || lj >= ts || i < 1 || j < 1 || i >= nx - 1 || j >= ny - 1) return;
    const double * s = src + lj * ld_src + li;
    const double v = s[0];
    const double a = __dadd_rn(__dsub_rn(s[1], __dmul_rn(2.0, v)), s[-1]);
    const double b = __dadd_rn(__dsub_rn(s[ld_src], __dmul_rn(2.0, v)), s[-ld_src]);
    dst[lj * ld_dst + li] = __dadd_rn(v, __dmul_rn(c, __dadd_rn(a, b)));
}

// src and dst point at cell (x, y) of their data, each with its own leading dimension
extern "C" void heat_cxx_tile(cudaStream_t stream, const double * src, long ld_src, double * dst, long ld_dst, long nx, long ny,
                              long x, long y, long ts, double c)
{
    const dim3 block(32, 8), grid((unsigned) ((ts + 31) / 32), (unsigned) ((ts + 7) / 8));
    heat_cxx_tile_kernel<<<grid, block, 0, stream>>>(src, ld_src, dst, ld_dst, nx, ny, x, y, ts, c);
}
