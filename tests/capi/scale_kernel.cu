// A kernel for the driver-interface test: loaded as a module image (cubin) at run time.
extern "C" __global__ void xkb_test_scale(double * p, double a, unsigned long n)
{
    const unsigned long i = blockIdx.x * (unsigned long) blockDim.x + threadIdx.x;
    if (i < n) p[i] *= a;
}
