/*
 * swehr_probe.cu -- device-peak probes for the benchmark's roofline (not part
 * of the SWEHR C ABI; built into libswehr_probe.so beside libswehr.so).
 *
 * swehr_probe_fp64_peak: the FP64 vector-pipe ceiling of this GPU, measured.
 * Every thread runs eight independent fused multiply-add chains (enough
 * independent work to cover the pipe's latency at full occupancy) on a grid
 * of eight resident blocks per SM; the value reported is the best of a few
 * timed launches, in TFLOP/s (an FMA counts two floating-point operations).
 * The step kernels' arithmetic is FP64 division, square root and exp/pow
 * sequences that all run on this pipe, so this is the compute roof they are
 * held against (tensor cores are not used by the stencil).
 */
#include <cuda_runtime.h>

static const int PROBE_THREADS = 256;
static const int PROBE_CHAINS = 8;

__global__ void __launch_bounds__(PROBE_THREADS) k_fp64_fma(double *out, int iters, double b, double c)
{
    double a[PROBE_CHAINS];
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; k++) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < PROBE_CHAINS; k++) a[k] = fma(a[k], b, c);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < PROBE_CHAINS; k++) s += a[k];
    if (s == 12345.678) out[blockIdx.x] = s;   /* keeps the chains live; never true */
}

extern "C" int swehr_probe_fp64_peak(double *tflops)
{
    if (!tflops) return 1;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 2;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 2;
    double *out = nullptr;
    if (cudaMalloc(&out, (size_t)sms * 8 * sizeof(double)) != cudaSuccess) return 3;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int grid = sms * 8, iters = 4096;
    double best = 0;
    for (int rep = 0; rep < 6; rep++) {
        cudaEventRecord(e0);
        k_fp64_fma<<<grid, PROBE_THREADS>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * grid * PROBE_THREADS * (double)iters * PROBE_CHAINS;
        if (rep > 0 && ms > 0) {
            const double tf = flops / (ms * 1e-3) / 1e12;
            if (tf > best) best = tf;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const cudaError_t err = cudaGetLastError();
    *tflops = best;
    return err == cudaSuccess ? 0 : 4;
}
