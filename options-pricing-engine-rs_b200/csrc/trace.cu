// Diagnostic: a step-by-step record of the greedy QAG (heston.rs:193-212)
// on one Gil-Pelaez integral of one contract, made by the same warp routine
// (gk_integrate_warp) and the same node evaluation as the pricing kernel.
//
// The reference's panel choices are decided by comparisons of error
// estimates; where two live panels' estimates are nearly equal, last-ulp
// differences between this library's node values and the reference's (CUDA's
// exp/sin/log against the platform libm, the merged integrand exponent, the
// order of the 15-term sums) can make the two implementations bisect
// different panels from that step on.  The trace lets a test find that step
// and measure the margin.  It is not on any pricing path.
#include <cuda_runtime.h>

#include <cmath>

#include "internal.h"
#include "quadrature.cuh"

namespace ope {

namespace {

// Per step j (0 = the first panel [0, 1], j >= 1 = the j-th bisection),
// OPE_TRACE_FIELDS doubles: a, b and the error estimate of the bisected panel
// (0, 1, 0 at j = 0); kl, el, kr, er of the children (j = 0: the first
// panel's K and error, 0, 0); the running error and total after the step; the
// 15 integrand values of the left child (lanes 0-14) and of the right child
// (lanes 16-30; zeros at j = 0).
struct StepRecorder {
    double* out;
    int max_steps;

    __device__ __forceinline__ void put(int j, int lane, double f, double a, double b, double ew, double kl,
                                        double el, double kr, double er, double err, double total) const {
        if (j >= max_steps) return;
        double* r = out + (size_t)j * OPE_TRACE_FIELDS;
        if (lane == 0) {
            r[0] = a;
            r[1] = b;
            r[2] = ew;
            r[3] = kl;
            r[4] = el;
            r[5] = kr;
            r[6] = er;
            r[7] = err;
            r[8] = total;
        }
        const int node = lane & 15;
        if (node < 15) r[9 + 15 * (lane >> 4) + node] = f;
    }
    __device__ __forceinline__ void first(int lane, double f, double k0, double e0) const {
        put(0, lane, f, 0.0, 1.0, 0.0, k0, e0, 0.0, 0.0, e0, k0);
    }
    __device__ __forceinline__ void step(int j, int lane, double f, double a, double b, double ew, double kl,
                                         double el, double kr, double er, double err, double total) const {
        put(j, lane, f, a, b, ew, kl, el, kr, er, err, total);
    }
};

// One warp.  result[0] = the integral, result[1] = steps (1 + bisections).
template <bool BATES>
__global__ void __launch_bounds__(32) k_trace_integral(const ope_contract* con, const double* params, int which,
                                                       double tol, double* out, int max_steps, double* result) {
    __shared__ PanelStore L;
    __shared__ CfConsts Cs;
    const int lane = threadIdx.x;
    const LaneRule R = lane_rule(lane);
    double pl[8];
#pragma unroll
    for (int i = 0; i < (BATES ? 8 : 5); ++i) pl[i] = params[i];
    const CfConsts Cl = make_consts(con->spot, con->strike, con->expiry, con->rate, pl, BATES, which);
    if (lane == 0) Cs = Cl;
    __syncwarp();
    int nb = 0;
    const StepRecorder tr{out, max_steps};
    const double I = gk_integrate_warp<BATES>(Cs, tol, L, lane, R, &nb, tr);
    if (lane == 0) {
        result[0] = I;
        result[1] = (double)(nb + 1);
    }
}

}  // namespace
}  // namespace ope

using namespace ope;

extern "C" int ope_trace_integral(int32_t model, const ope_contract* contract, const void* params, int32_t which,
                                  double tol, double* out_steps, int32_t max_steps, int32_t* out_n_steps,
                                  double* out_integral) {
    OPE_RANGE("ope.trace_integral");
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES)
        return set_error(OPE_ERR_INVALID_ARG, "model must be OPE_MODEL_HESTON or OPE_MODEL_BATES");
    if (!contract || !params || !out_n_steps || !out_integral || (max_steps > 0 && !out_steps))
        return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (which != 0 && which != 1) return set_error(OPE_ERR_INVALID_ARG, "which must be 0 (P1) or 1 (P2)");
    if (max_steps < 0) return set_error(OPE_ERR_INVALID_ARG, "max_steps must be >= 0");
    if (std::isnan(tol)) return set_error(OPE_ERR_INVALID_ARG, "tol is NaN");
    if (!(tol > 0.0)) tol = OPE_REF_TOL;
    if (!std::isfinite(tol)) return set_error(OPE_ERR_INVALID_ARG, "tol must be finite");
    OPE_TRY(ensure_device());
    ThreadCtx& c = tctx();
    const int stride = param_stride(model);
    // a trace has at most OPE_MAX_PANELS steps (the first panel + 199 bisections)
    const int cap = max_steps < OPE_MAX_PANELS ? max_steps : OPE_MAX_PANELS;
    const size_t b_con = 256, b_par = 256, b_res = 256, b_out = align_up((size_t)cap * OPE_TRACE_FIELDS * 8, 256);
    void* ws;
    OPE_TRY(ensure_workspace(b_con + b_par + b_res + b_out, &ws, c.stream));
    char* p = static_cast<char*>(ws);
    ope_contract* d_con = reinterpret_cast<ope_contract*>(p);
    double* d_par = reinterpret_cast<double*>(p + b_con);
    double* d_res = reinterpret_cast<double*>(p + b_con + b_par);
    double* d_out = reinterpret_cast<double*>(p + b_con + b_par + b_res);
    OPE_CHECK(cudaMemcpyAsync(d_con, contract, sizeof(ope_contract), cudaMemcpyHostToDevice, c.stream));
    OPE_CHECK(cudaMemcpyAsync(d_par, params, stride * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (cap > 0) OPE_CHECK(cudaMemsetAsync(d_out, 0, b_out, c.stream));
    if (model == OPE_MODEL_BATES)
        k_trace_integral<true><<<1, 32, 0, c.stream>>>(d_con, d_par, which, tol, d_out, cap, d_res);
    else
        k_trace_integral<false><<<1, 32, 0, c.stream>>>(d_con, d_par, which, tol, d_out, cap, d_res);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    double res[2];
    OPE_CHECK(cudaMemcpyAsync(res, d_res, sizeof(res), cudaMemcpyDeviceToHost, c.stream));
    if (cap > 0)
        OPE_CHECK(cudaMemcpyAsync(out_steps, d_out, (size_t)cap * OPE_TRACE_FIELDS * sizeof(double),
                                  cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    *out_integral = res[0];
    *out_n_steps = (int32_t)res[1];
    return OPE_OK;
}
