// FP64 throughput probe: the denominator of the pricing kernel's roofline.
//
// The pricing path is bound by the FP64 pipe of the CUDA cores (no tensor
// core work, negligible HBM traffic), and no FP64 figure is published for
// this pool, so the library measures it: every thread runs eight independent
// DFMA chains (enough ILP to saturate the pipe) over a grid of 32 resident
// warps per SM, timed with CUDA events.  Counted as 2 flops per DFMA.
#include <cuda_runtime.h>

#include "cf_device.cuh"
#include "internal.h"

namespace ope {
namespace {

__global__ void __launch_bounds__(256) k_dfma_probe(double b, double c, int iters, double* sink) {
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
    double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
    for (int i = 0; i < iters; ++i) {
        a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
        a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
    const double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 1234.5678) sink[0] = s;  // never true; keeps the chains live
}

// rcp_nr / rsqrt_nr against IEEE 1/x and sqrt over 2^20 inputs spanning
// 1e-300 .. 1e300 (log-uniform exponent, pseudo-random mantissa).  Errors in
// units of the last place of the correctly rounded result.
__global__ void k_selftest_math(unsigned long long* ulp_rcp, unsigned long long* ulp_sqrt) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long h = 0x9E3779B97F4A7C15ull * (i + 1);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double mant = 1.0 + (double)(h >> 12) * 0x1.0p-52;
    const double ex = -996.0 + 1992.0 * ((double)(i & 0xffff) / 65535.0);
    const double x = ldexp(mant, (int)ex);
    const double a = rcp_nr(x), b = 1.0 / x;
    const long long da = llabs(__double_as_longlong(a) - __double_as_longlong(b));
    const double s = x * rsqrt_nr(x), t = sqrt(x);
    const long long ds = llabs(__double_as_longlong(s) - __double_as_longlong(t));
    atomicMax(ulp_rcp, (unsigned long long)da);
    atomicMax(ulp_sqrt, (unsigned long long)ds);
}

// atan2_node against CUDA's atan2 over 2^24 argument pairs: random signs,
// magnitudes from 2^-60 to 2^60 and ratios |y/x| from 2^-45 to 2^45.
// Errors in units of the last place of CUDA's result.
__global__ void k_selftest_atan2(unsigned long long* ulp) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long h = 0x9E3779B97F4A7C15ull * (i + 1);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    unsigned long long g = h * 0x94D049BB133111EBull;
    g ^= g >> 32;
    const double m1 = 1.0 + (double)(h >> 12) * 0x1.0p-52, m2 = 1.0 + (double)(g >> 12) * 0x1.0p-52;
    const int e1 = (int)((h >> 3) % 121) - 60, e2 = (int)((g >> 5) % 91) - 45;
    const double y = ((h & 1) ? -1.0 : 1.0) * ldexp(m1, e1);
    const double x = ((h & 2) ? -1.0 : 1.0) * ldexp(m2, e1 + e2);
    const long long d = llabs(__double_as_longlong(atan2_node(y, x)) - __double_as_longlong(atan2(y, x)));
    atomicMax(ulp, (unsigned long long)d);
}

// log_node against CUDA's log over 2^24 arguments: half with exponents from
// 2^-1000 to 2^1000, half in [0.5, 4) around 1.  Errors in units of the last
// place of CUDA's result.
__global__ void k_selftest_log(unsigned long long* ulp) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long h = 0x9E3779B97F4A7C15ull * (i + 1);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double m = 1.0 + (double)(h >> 12) * 0x1.0p-52;
    const int e = (i & 1) ? (int)((h >> 3) % 2001) - 1000 : (int)((h >> 3) % 3) - 1;
    const double v = ldexp(m, e);
    const long long d = llabs(__double_as_longlong(log_node(v)) - __double_as_longlong(log(v)));
    atomicMax(ulp, (unsigned long long)d);
}

// node_u against IEEE division (1 - t)/t over 2^24 node positions t: uniform
// in (0, 1), and log-uniform from 2^-200 (the smallest panel 200 bisections
// can make) to 1/2.  Counts the positions where the two differ.
__global__ void k_selftest_node_u(unsigned long long* mismatches) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long h = 0x9E3779B97F4A7C15ull * (i + 1);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double r = (double)(h >> 11) * 0x1.0p-53;  // [0, 1)
    const double tn = (i & 1) ? exp2(-200.0 * r - 1.0) : fmax(r, 0x1.0p-53);
    const double omt = 1.0 - tn;
    const double u = node_u(omt, tn, rcp_nr(omt * tn));
    if (u != __ddiv_rn(omt, tn)) atomicAdd(mismatches, 1ull);
}

// log_cr (x = ln(S/K) of every integral) and CUDA's log on given arguments.
__global__ void k_eval_log_cr(const double* v, long long n, double* out_cr, double* out_cuda) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out_cr[i] = log_cr(v[i]);
    out_cuda[i] = log(v[i]);
}

}  // namespace

int selftest_log_cr(const double* v, size_t n, double* out_cr, double* out_cuda) {
    ThreadCtx& c = tctx();
    const size_t b = align_up(n * sizeof(double), 256);
    void* ws;
    OPE_TRY(ensure_workspace(3 * b, &ws, c.stream));
    double* d_v = static_cast<double*>(ws);
    double* d_cr = reinterpret_cast<double*>(static_cast<char*>(ws) + b);
    double* d_cu = reinterpret_cast<double*>(static_cast<char*>(ws) + 2 * b);
    OPE_CHECK(cudaMemcpyAsync(d_v, v, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    k_eval_log_cr<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(d_v, (long long)n, d_cr, d_cu);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    OPE_CHECK(cudaMemcpyAsync(out_cr, d_cr, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaMemcpyAsync(out_cuda, d_cu, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    return OPE_OK;
}

int selftest_node_u(uint64_t* mismatches) {
    ThreadCtx& c = tctx();
    void* ws;
    OPE_TRY(ensure_workspace(256, &ws, c.stream));
    unsigned long long* d = static_cast<unsigned long long*>(ws);
    OPE_CHECK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c.stream));
    k_selftest_node_u<<<1 << 16, 256, 0, c.stream>>>(d);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    unsigned long long h = 0;
    OPE_CHECK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    *mismatches = h;
    return OPE_OK;
}

int selftest_log(uint64_t* ulp) {
    ThreadCtx& c = tctx();
    void* ws;
    OPE_TRY(ensure_workspace(256, &ws, c.stream));
    unsigned long long* d = static_cast<unsigned long long*>(ws);
    OPE_CHECK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c.stream));
    k_selftest_log<<<1 << 16, 256, 0, c.stream>>>(d);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    unsigned long long h = 0;
    OPE_CHECK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    *ulp = h;
    return OPE_OK;
}

int selftest_atan2(uint64_t* ulp) {
    ThreadCtx& c = tctx();
    void* ws;
    OPE_TRY(ensure_workspace(256, &ws, c.stream));
    unsigned long long* d = static_cast<unsigned long long*>(ws);
    OPE_CHECK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), c.stream));
    k_selftest_atan2<<<1 << 16, 256, 0, c.stream>>>(d);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    unsigned long long h = 0;
    OPE_CHECK(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    *ulp = h;
    return OPE_OK;
}

int selftest_math(uint64_t* ulp_rcp, uint64_t* ulp_sqrt) {
    ThreadCtx& c = tctx();
    void* ws;
    OPE_TRY(ensure_workspace(256, &ws, c.stream));
    unsigned long long* d = static_cast<unsigned long long*>(ws);
    OPE_CHECK(cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), c.stream));
    k_selftest_math<<<4096, 256, 0, c.stream>>>(d, d + 1);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    unsigned long long h[2];
    OPE_CHECK(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    *ulp_rcp = h[0];
    *ulp_sqrt = h[1];
    return OPE_OK;
}

int measure_fp64_peak(double* flops, double* ms) {
    ThreadCtx& c = tctx();
    void* ws;
    OPE_TRY(ensure_workspace(256, &ws, c.stream));
    const int threads = 256, blocks = c.sm_count * 4;
    cudaEvent_t e0, e1;
    OPE_CHECK(cudaEventCreate(&e0));
    OPE_CHECK(cudaEventCreate(&e1));
    k_dfma_probe<<<blocks, threads, 0, c.stream>>>(0.999999, 1e-7, 20000, static_cast<double*>(ws));
    OPE_CHECK(cudaGetLastError());
    const int iters = 400000;
    OPE_CHECK(cudaEventRecord(e0, c.stream));
    k_dfma_probe<<<blocks, threads, 0, c.stream>>>(0.999999, 1e-7, iters, static_cast<double*>(ws));
    OPE_CHECK(cudaGetLastError());
    OPE_CHECK(cudaEventRecord(e1, c.stream));
    OPE_CHECK(cudaEventSynchronize(e1));
    float t = 0.f;
    OPE_CHECK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c.launches += 2;
    *ms = t;
    *flops = 2.0 * 8.0 * (double)iters * (double)threads * (double)blocks / (t * 1e-3);
    return OPE_OK;
}

}  // namespace ope
