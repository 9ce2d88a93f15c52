// Batched Levenberg-Marquardt calibration on the device (IV-space residuals,
// adjoint Jacobian), one LM state machine per surface.
//
// Reference: calibration.rs:433-569 (calibrate_inner), 573-605 (IV residual,
// d iv / d p = d price / d p / vega_BSM(iv)), 655-668 (J'J, J'r), 673-703
// (lm_step: damped normal equations, Gaussian elimination with partial
// pivoting), 717-768 (Jacobi eigen diagnostic), constants 30-36, bounds
// 115-122 / 158-163.  Same iteration, acceptance and termination rules:
//   iters += 1; J at p; g = J'W r; |g| < 1e-8 -> converged;
//   dp = lm_step(J'WJ, g, lam); p_new out of bounds -> lam = min(10 lam, 1e8);
//   else sse_new < sse -> accept, lam = max(lam / 10, 1e-12), |dp| < 1e-10 ->
//   converged; else lam = min(10 lam, 1e8), lam >= 1e8 -> stop; 200 iterations.
// The Jacobian columns are EXACT (adjoint kernel / BSM vega) for all
// parameters, where the reference uses central finite differences for the
// Heston columns (calibration.rs:639-650) and forward-mode AD for the Bates
// jump columns (calibration.rs:186-198, 625-632).  A quote whose IV solve
// fails contributes a zero residual (calibration.rs:577-580) and a zero
// Jacobian row.  J at a given p is deterministic, so it is recomputed only
// after an accepted step (the reference recomputes the same J after a
// rejected or out-of-bounds step).  Every pricing of the loop (the initial
// one at p0, each trial) stores its integrals' final panel lists in one of
// two slots per surface; an accepted trial's slot becomes the current one,
// so the Jacobian at the new p is only the adjoint's backward pass over
// lists that already exist, not a second pricing.
//
// Optional per surface (CalibExtra): a Tikhonov prior, added as dim pseudo
// rows (p_k - prior_k) / scale_k of weight sqrt(reg_weight) to the SSE, J'J
// and J'r exactly as calibration.rs:448-470 appends them (the final rmse,
// max error and J'J diagnostics stay data-only, calibration.rs:541-568); and
// a restart group for multistart pruning: members publish every accepted SSE
// to the group's shared best (atomicMin on the bits of a non-negative
// double) and, at iterations 10, 20, ..., stop (early_stopped) when their SSE
// exceeds 8x that best (calibration.rs:263-264, 482-490).  All surfaces take
// one LM iteration per pass, so every check in pass k sees exactly the
// accepted steps of passes < k: the restarts run in lockstep, one of the
// schedules the reference's thread-timed sharing allows.
//
// One LM iteration for ALL surfaces is one pass of the body below; the body
// is captured once into a CUDA graph whose conditional WHILE node repeats it
// on the device until every surface has stopped: one graph launch per
// calibration batch, no host round trip per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"
#include "iv_device.cuh"

namespace ope {

namespace {

enum { LM_ACTIVE = 0, LM_CONVERGED = 1, LM_BAILED = 2, LM_MAXITER = 3, LM_PRUNED = 4 };
constexpr int kMaxIter = 200;
constexpr int kPruneEvery = 10;          // calibration.rs:264
constexpr double kPruneFactor = 8.0;     // calibration.rs:263
constexpr double kTolGrad = 1e-8, kTolParams = 1e-10, kLamInit = 1e-3, kLamUp = 10.0, kLamDown = 0.1,
                 kLamMax = 1e8;

struct LMSurf {
    double p[8], p_new[8], dp[8];
    double jtj[64], grad[8];
    double lam, sse;
    int iters, status, need_jac, trial;
};

struct LMDev {
    const ope_contract* q;
    const double* iv_mkt;
    const double* w;
    const int64_t* off;
    const int32_t* sidx;
    int nq, ns, dim;
    LMSurf* st;
    double* pcur;    // ns x dim: parameters the adjoint pass differentiates at
    double* ptrial;  // ns x dim: trial parameters
    int32_t* jmask;  // ns: surfaces needing J this iteration
    int32_t* tmask;  // ns: surfaces with a trial step this iteration
    double* price;   // nq: model prices at the current parameters
    double* price_trial;  // nq: model prices at the trial parameters
    int32_t* jslot;  // ns: panel-list slot of the current parameters
    int32_t* pslot;  // ns: panel-list slot the next pricing writes
    double* pgrad;   // nq x dim
    double* res;     // nq
    double* res_new; // nq
    double* jrow;    // nq x dim
    unsigned int* counters;  // [0] active surfaces, [1] body passes
    const double* prior;     // ns x dim Tikhonov prior, or null
    const double* regw;      // ns regularisation weights
    const int32_t* group;    // ns restart groups, or null (no pruning)
    unsigned long long* gbest;  // per group: shared best SSE (bits of a non-negative double)
};

// calibration.rs:130, 174-177 regularization_scale
__device__ __forceinline__ double reg_scale(int k) {
    constexpr double s[8] = {0.04, 2.0, 0.04, 0.3, 0.3, 0.5, 0.1, 0.15};
    return s[k];
}

// The Tikhonov rows' share of the weighted SSE, added after the data rows in
// row order (calibration.rs:460-465, 589-591).
__device__ double add_reg_sse(const LMDev& D, int s, const double* p, double sse) {
    if (!D.prior) return sse;
    const double rw = sqrt(D.regw[s]);
    for (int k = 0; k < D.dim; ++k) {
        const double r = (p[k] - D.prior[s * D.dim + k]) / reg_scale(k);
        const double t = rw * r;
        sse = sse + t * t;
    }
    return sse;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// calibration.rs:115-122, 158-163
__device__ __forceinline__ bool bounds_ok(const double* v, int dim) {
    const bool feller = (2.0 * v[1]) * v[2] > v[3] * v[3];
    const bool h = feller && v[0] > 1e-8 && v[0] < 5.0 && v[1] > 1e-6 && v[1] < 50.0 && v[2] > 1e-8 &&
                   v[2] < 5.0 && v[3] > 1e-6 && v[3] < 10.0 && v[4] > -0.9999 && v[4] < 0.9999;
    if (dim == 5) return h;
    return h && v[5] >= 0.0 && v[5] < 10.0 && fabs(v[6]) < 2.0 && v[7] > 1e-6 && v[7] < 2.0;
}

// calibration.rs:673-703 (n <= 8)
__device__ void lm_solve(const double* jtj, const double* grad, double lam, int n, double* dp) {
    double a[8][8], b[8];
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < n; ++k) a[i][k] = jtj[i * n + k];
        b[i] = grad[i];
    }
    for (int i = 0; i < n; ++i) { a[i][i] *= 1.0 + lam; b[i] = -b[i]; }
    for (int col = 0; col < n; ++col) {
        int pivot = col;
        for (int i = col + 1; i < n; ++i)
            if (fabs(a[i][col]) >= fabs(a[pivot][col])) pivot = i;
        for (int k = 0; k < n; ++k) { const double t = a[col][k]; a[col][k] = a[pivot][k]; a[pivot][k] = t; }
        { const double t = b[col]; b[col] = b[pivot]; b[pivot] = t; }
        if (fabs(a[col][col]) < 1e-15) continue;
        const double inv = 1.0 / a[col][col];
        for (int row = col + 1; row < n; ++row) {
            const double f = a[row][col] * inv;
            for (int k = col; k < n; ++k) a[row][k] -= f * a[col][k];
            b[row] -= f * b[col];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int k = i + 1; k < n; ++k) s -= a[i][k] * dp[k];
        dp[i] = fabs(a[i][i]) > 1e-15 ? s / a[i][i] : 0.0;
    }
}

// calibration.rs:717-768: eigenvalues/vectors of a symmetric n x n (n <= 8).
__device__ void jacobi_eigen_d(const double* a_in, int n, double* evals, double* evecs) {
    double a[8][8], v[8][8];
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) { a[i][k] = a_in[i * n + k]; v[i][k] = (i == k) ? 1.0 : 0.0; }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i) {
            double row = 0.0;
            for (int j = i + 1; j < n; ++j) row += a[i][j] * a[i][j];
            off += row;
        }
        if (sqrt(off) < 1e-14) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                if (fabs(a[p][q]) < 1e-300) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = theta >= 0.0 ? 1.0 / (theta + sqrt(theta * theta + 1.0))
                                               : -1.0 / (-theta + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0);
                const double s = t * c;
                const double apq = a[p][q];
                a[p][p] -= t * apq;
                a[q][q] += t * apq;
                a[p][q] = 0.0;
                a[q][p] = 0.0;
                for (int i = 0; i < n; ++i) {
                    if (i != p && i != q) {
                        const double aip = a[i][p], aiq = a[i][q];
                        a[i][p] = c * aip - s * aiq; a[p][i] = a[i][p];
                        a[i][q] = s * aip + c * aiq; a[q][i] = a[i][q];
                    }
                }
                for (int row = 0; row < n; ++row) {
                    const double vip = v[row][p], viq = v[row][q];
                    v[row][p] = c * vip - s * viq;
                    v[row][q] = s * vip + c * viq;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) evals[i] = a[i][i];
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) evecs[i * n + k] = v[k][i];
}

__global__ void k_lm_init(LMDev D, const double* p0) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= D.ns) return;
    LMSurf& S = D.st[s];
    for (int k = 0; k < D.dim; ++k) { S.p[k] = p0[s * D.dim + k]; D.pcur[s * D.dim + k] = S.p[k]; S.dp[k] = 0.0; }
    S.lam = kLamInit;
    S.sse = 0.0;
    S.iters = 0;
    S.status = LM_ACTIVE;
    S.need_jac = 1;
    S.trial = 0;
    D.jmask[s] = 1;
    D.tmask[s] = 1;  // the initial pricing pass prices every surface at p0
    D.jslot[s] = 0;  // ... into slot 0, the current parameters' slot
    D.pslot[s] = 0;
}

// IV residual of every quote whose surface is selected by `mask`
// (calibration.rs:573-581): iv(model price) - iv_market, 0 if the solver fails.
__global__ void k_lm_residuals(LMDev D, const int32_t* mask, const double* price, double* res) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nq) return;
    const int s = D.sidx[i];
    if (mask && mask[s] == 0) return;
    double iv;
    const IvC c = iv_contract(D.q[i]);
    res[i] = implied_vol_d(c, price[i], &iv) ? iv - D.iv_mkt[i] : 0.0;
}

// Jacobian rows at p for surfaces in jmask: d iv / d p = d price / d p / vega(iv)
// (calibration.rs:598-605, 625-632); a failed IV or |vega| < 1e-10 gives a zero row.
__global__ void k_lm_jrows(LMDev D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nq) return;
    const int s = D.sidx[i];
    if (D.jmask[s] == 0) return;
    const IvC c = iv_contract(D.q[i]);
    double iv;
    double scale = 0.0;
    if (implied_vol_d(c, D.price[i], &iv)) {
        const double vega = bsm_vega_d(c, iv);
        if (fabs(vega) >= 1e-10) scale = 1.0 / vega;
    }
    for (int k = 0; k < D.dim; ++k) D.jrow[(size_t)i * D.dim + k] = D.pgrad[(size_t)i * D.dim + k] * scale;
}

// J'WJ and J'W r of one surface, warp-cooperative (calibration.rs:655-668).
__device__ void surf_normal_eq(const LMDev& D, int s, int lane, double* jtj, double* grad) {
    const int dim = D.dim;
    double aj[36], ag[8];  // upper triangle (dim <= 8)
    int t = 0;
    for (int a = 0; a < dim; ++a) {
        ag[a] = 0.0;
        for (int b = a; b < dim; ++b) aj[t++] = 0.0;
    }
    for (int64_t i = D.off[s] + lane; i < D.off[s + 1]; i += 32) {
        const double w2 = D.w[i] * D.w[i];
        const double r = D.res[i];
        const double* J = D.jrow + (size_t)i * dim;
        t = 0;
        for (int a = 0; a < dim; ++a) {
            const double wa = w2 * J[a];
            ag[a] += wa * r;
            for (int b = a; b < dim; ++b) aj[t++] += wa * J[b];
        }
    }
    t = 0;
    for (int a = 0; a < dim; ++a) {
        grad[a] = warp_sum(ag[a]);
        for (int b = a; b < dim; ++b) {
            const double v = warp_sum(aj[t++]);
            jtj[a * dim + b] = v;
            jtj[b * dim + a] = v;
        }
    }
}

// One warp per surface: J'J, gradient test, damped step, bounds test.
__global__ void k_lm_step(LMDev D) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= D.ns) return;
    LMSurf& S = D.st[s];
    const int dim = D.dim;
    if (S.need_jac) {  // J was just computed at p (for a stopped surface: its final J)
        double jtj[64], grad[8];
        surf_normal_eq(D, s, lane, jtj, grad);
        if (lane == 0) {
            for (int k = 0; k < dim * dim; ++k) S.jtj[k] = jtj[k];
            for (int k = 0; k < dim; ++k) S.grad[k] = grad[k];
        }
    }
    if (S.status != LM_ACTIVE) {
        if (lane == 0) { S.need_jac = 0; D.jmask[s] = 0; D.tmask[s] = 0; }
        return;
    }
    if (lane != 0) return;
    S.need_jac = 0;
    D.jmask[s] = 0;
    S.iters += 1;
    const int iter = S.iters - 1;
    if (D.group && iter > 0 && iter % kPruneEvery == 0) {
        const double best = __longlong_as_double((long long)D.gbest[D.group[s]]);
        if (isfinite(best) && S.sse > best * kPruneFactor) {
            S.status = LM_PRUNED;
            D.tmask[s] = 0;
            return;
        }
    }
    // J'J and J'r of the data rows, plus the Tikhonov rows' diagonal terms
    double A[64], g[8];
    for (int k = 0; k < dim * dim; ++k) A[k] = S.jtj[k];
    for (int k = 0; k < dim; ++k) g[k] = S.grad[k];
    if (D.prior) {
        const double rw = sqrt(D.regw[s]);
        const double w2 = rw * rw;
        for (int k = 0; k < dim; ++k) {
            const double jk = 1.0 / reg_scale(k);
            const double r = (S.p[k] - D.prior[s * dim + k]) / reg_scale(k);
            g[k] += (w2 * jk) * r;
            A[k * dim + k] += (w2 * jk) * jk;
        }
    }
    double gn = 0.0;
    for (int k = 0; k < dim; ++k) gn += g[k] * g[k];
    if (sqrt(gn) < kTolGrad) {
        S.status = LM_CONVERGED;
        D.tmask[s] = 0;
        return;
    }
    lm_solve(A, g, S.lam, dim, S.dp);
    for (int k = 0; k < dim; ++k) S.p_new[k] = S.p[k] + S.dp[k];
    if (!bounds_ok(S.p_new, dim)) {
        S.lam = fmin(S.lam * kLamUp, kLamMax);
        S.trial = 0;
        D.tmask[s] = 0;
        if (S.iters >= kMaxIter) S.status = LM_MAXITER;
        return;
    }
    S.trial = 1;
    D.tmask[s] = 1;
    for (int k = 0; k < dim; ++k) D.ptrial[s * dim + k] = S.p_new[k];
}

// One warp per surface with a trial step: accept or reject (calibration.rs:513-538).
__global__ void k_lm_accept(LMDev D) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= D.ns) return;
    LMSurf& S = D.st[s];
    if (D.tmask[s] == 0) return;
    double part = 0.0;
    for (int64_t i = D.off[s] + lane; i < D.off[s + 1]; i += 32) {
        const double t = D.w[i] * D.res_new[i];
        part += t * t;
    }
    const double sse_new = add_reg_sse(D, s, S.p_new, warp_sum(part));
    const bool accept = sse_new < S.sse;
    if (accept)
        for (int64_t i = D.off[s] + lane; i < D.off[s + 1]; i += 32) {
            D.res[i] = D.res_new[i];
            D.price[i] = D.price_trial[i];
        }
    if (lane != 0) return;
    const int dim = D.dim;
    D.tmask[s] = 0;
    S.trial = 0;
    if (accept) {
        for (int k = 0; k < dim; ++k) { S.p[k] = S.p_new[k]; D.pcur[s * dim + k] = S.p[k]; }
        S.sse = sse_new;
        S.lam = fmax(S.lam * kLamDown, 1e-12);
        if (D.group) atomicMin(D.gbest + D.group[s], (unsigned long long)__double_as_longlong(sse_new));
        S.need_jac = 1;
        D.jmask[s] = 1;
        D.jslot[s] = D.pslot[s];  // the trial's panel lists are now the current ones
        D.pslot[s] = 1 - D.pslot[s];
        double sn = 0.0;
        for (int k = 0; k < dim; ++k) sn += S.dp[k] * S.dp[k];
        if (sqrt(sn) < kTolParams) { S.status = LM_CONVERGED; return; }  // J at the final p still due
    } else {
        S.lam = fmin(S.lam * kLamUp, kLamMax);
        if (S.lam >= kLamMax) { S.status = LM_BAILED; return; }
    }
    if (S.iters >= kMaxIter) S.status = LM_MAXITER;
}

// Initial weighted SSE at p0, one warp per surface.
__global__ void k_lm_sse0(LMDev D) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= D.ns) return;
    double part = 0.0;
    for (int64_t i = D.off[s] + lane; i < D.off[s + 1]; i += 32) {
        const double t = D.w[i] * D.res[i];
        part += t * t;
    }
    const double sse = warp_sum(part);
    if (lane == 0) {
        D.st[s].sse = add_reg_sse(D, s, D.st[s].p, sse);
        D.tmask[s] = 0;
        D.pslot[s] = 1 - D.jslot[s];  // trials write the other slot
    }
}

// Count surfaces still iterating and drive the graph's WHILE condition.
__global__ void k_lm_continue(LMDev D, cudaGraphConditionalHandle handle) {
    __shared__ unsigned int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < D.ns; s += blockDim.x)
        if (D.st[s].status == LM_ACTIVE) atomicAdd(&cnt, 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int passes = D.counters[1] + 1;
        D.counters[1] = passes;
        D.counters[0] = cnt;
        cudaGraphSetConditional(handle, (cnt > 0 && passes < (unsigned)kMaxIter + 1) ? 1u : 0u);
    }
}

// Final diagnostics (calibration.rs:541-568): data-only rmse and max error,
// J'J at the final parameters, its Jacobi eigen-decomposition.
__global__ void k_lm_final(LMDev D, ope_calib_result* out) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= D.ns) return;
    LMSurf& S = D.st[s];
    const int dim = D.dim;
    double jtj[64], grad[8];
    const bool fresh = S.need_jac != 0;  // last step accepted: J at the final p computed just before
    if (fresh) surf_normal_eq(D, s, lane, jtj, grad);
    double sq = 0.0, ww = 0.0, mx = 0.0;
    for (int64_t i = D.off[s] + lane; i < D.off[s + 1]; i += 32) {
        const double t = D.w[i] * D.res[i];
        sq += t * t;
        ww += D.w[i] * D.w[i];
        mx = fmax(mx, fabs(D.res[i]));
    }
    sq = warp_sum(sq);
    ww = warp_sum(ww);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane != 0) return;
    ope_calib_result r;
    memset(&r, 0, sizeof(r));
    for (int k = 0; k < dim; ++k) r.params[k] = S.p[k];
    r.rmse = sqrt(sq / ww);
    r.max_err = mx;
    const double* A = fresh ? jtj : S.jtj;
    double ev[8], evec[64];
    jacobi_eigen_d(A, dim, ev, evec);
    double mxe = -1.7976931348623157e308, mne = 1.7976931348623157e308;
    for (int k = 0; k < dim; ++k) { mxe = fmax(mxe, ev[k]); mne = fmin(mne, ev[k]); }
    r.condition_number = fabs(mne) > 1e-300 ? fabs(mxe / mne) : __longlong_as_double(0x7ff0000000000000ll);
    int weakest = 0;
    for (int k = 1; k < dim; ++k)
        if (fabs(ev[k]) < fabs(ev[weakest])) weakest = k;
    for (int k = 0; k < dim; ++k) r.weakest_direction[k] = evec[weakest * dim + k];
    r.iters = S.iters;
    r.converged = S.status == LM_CONVERGED ? 1 : 0;
    r.early_stopped = S.status == LM_PRUNED ? 1 : 0;
    r.status = S.status;
    out[s] = r;
}

// Per-thread cache of the instantiated LM graph (its kernels' arguments are
// pointers into the workspace, so it is valid while the workspace layout is).
struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    void* ws = nullptr;
    int model = -1, nq = -1, ns = -1;
    double tol = 0.0;
    cudaStream_t stream = nullptr;
    bool prior = false, group = false;
};
}  // namespace

struct CalibGraph {
    GraphCache cache;
};

namespace {

thread_local CalibGraph g_lm_graph;

struct Layout {
    size_t total;
    size_t q, iv, w, off, sidx, st, pcur, ptrial, jmask, tmask, price, price_trial, jslot, pslot, pgrad, res, res_new,
        jrow, counters, out, prior, regw, group, gbest, sink, bscr, scratch;
};

Layout layout(size_t nq, size_t ns, int dim) {
    Layout L;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o += align_up(bytes, 256); return at; };
    L.q = take(nq * sizeof(ope_contract));
    L.iv = take(nq * sizeof(double));
    L.w = take(nq * sizeof(double));
    L.off = take((ns + 1) * sizeof(int64_t));
    L.sidx = take(nq * sizeof(int32_t));
    L.st = take(ns * sizeof(LMSurf));
    L.pcur = take(ns * dim * sizeof(double));
    L.ptrial = take(ns * dim * sizeof(double));
    L.jmask = take(ns * sizeof(int32_t));
    L.tmask = take(ns * sizeof(int32_t));
    L.price = take(nq * sizeof(double));
    L.price_trial = take(nq * sizeof(double));
    L.jslot = take(ns * sizeof(int32_t));
    L.pslot = take(ns * sizeof(int32_t));
    L.pgrad = take(nq * dim * sizeof(double));
    L.res = take(nq * sizeof(double));
    L.res_new = take(nq * sizeof(double));
    L.jrow = take(nq * dim * sizeof(double));
    L.counters = take(4 * sizeof(unsigned int));
    L.out = take(ns * sizeof(ope_calib_result));
    L.prior = take(ns * dim * sizeof(double));
    L.regw = take(ns * sizeof(double));
    L.group = take(ns * sizeof(int32_t));
    L.gbest = take(ns * sizeof(unsigned long long));
    L.sink = take(panel_sink_bytes(nq, 2));
    L.bscr = take(grad_backward_bytes(nq, dim));
    L.scratch = take(price_scratch_bytes(nq));
    L.total = o;
    return L;
}

LMDev make_dev(char* base, const Layout& L, int nq, int ns, int dim) {
    LMDev D;
    D.q = reinterpret_cast<const ope_contract*>(base + L.q);
    D.iv_mkt = reinterpret_cast<const double*>(base + L.iv);
    D.w = reinterpret_cast<const double*>(base + L.w);
    D.off = reinterpret_cast<const int64_t*>(base + L.off);
    D.sidx = reinterpret_cast<const int32_t*>(base + L.sidx);
    D.nq = nq;
    D.ns = ns;
    D.dim = dim;
    D.st = reinterpret_cast<LMSurf*>(base + L.st);
    D.pcur = reinterpret_cast<double*>(base + L.pcur);
    D.ptrial = reinterpret_cast<double*>(base + L.ptrial);
    D.jmask = reinterpret_cast<int32_t*>(base + L.jmask);
    D.tmask = reinterpret_cast<int32_t*>(base + L.tmask);
    D.price = reinterpret_cast<double*>(base + L.price);
    D.price_trial = reinterpret_cast<double*>(base + L.price_trial);
    D.jslot = reinterpret_cast<int32_t*>(base + L.jslot);
    D.pslot = reinterpret_cast<int32_t*>(base + L.pslot);
    D.pgrad = reinterpret_cast<double*>(base + L.pgrad);
    D.res = reinterpret_cast<double*>(base + L.res);
    D.res_new = reinterpret_cast<double*>(base + L.res_new);
    D.jrow = reinterpret_cast<double*>(base + L.jrow);
    D.counters = reinterpret_cast<unsigned int*>(base + L.counters);
    D.prior = nullptr;
    D.regw = nullptr;
    D.group = nullptr;
    D.gbest = nullptr;
    return D;
}

// The pricing launches' panel-list sink, writing each surface's pslot.
PanelSink pricing_sink(const LMDev& D, char* base, const Layout& L) {
    return carve_panel_sink(base + L.sink, D.nq, 2, D.pslot);
}

// d price / d p at the current parameters of the surfaces in jmask: the
// adjoint's backward pass over the panel lists of the current slot.
int launch_jac(int model, const LMDev& D, char* base, const Layout& L, cudaStream_t st) {
    const PanelSink src = carve_panel_sink(base + L.sink, D.nq, 2, D.jslot);
    OPE_TRY(launch_grad_backward(model, D.q, D.nq, D.off, D.ns, nullptr, D.pcur, src, base + L.bscr, D.pgrad, st,
                                 D.jmask));
    k_lm_jrows<<<(D.nq + 127) / 128, 128, 0, st>>>(D);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 1;
    return OPE_OK;
}

// The LM iteration body (stream-ordered; captured into the WHILE node).
int enqueue_body(int model, const LMDev& D, char* base, const Layout& L, double tol, cudaStream_t st,
                 cudaGraphConditionalHandle handle) {
    const int warps_blocks = (D.ns * 32 + 127) / 128;
    OPE_TRY(launch_jac(model, D, base, L, st));
    k_lm_step<<<warps_blocks, 128, 0, st>>>(D);
    OPE_CHECK(cudaGetLastError());
    const PanelSink sink = pricing_sink(D, base, L);
    OPE_TRY(launch_price_persistent(model, D.q, D.nq, D.off, D.ns, nullptr, D.ptrial, tol, D.price_trial,
                                    carve_price_scratch(base + L.scratch, D.nq), st, nullptr, D.tmask, &sink));
    k_lm_residuals<<<(D.nq + 127) / 128, 128, 0, st>>>(D, D.tmask, D.price_trial, D.res_new);
    OPE_CHECK(cudaGetLastError());
    k_lm_accept<<<warps_blocks, 128, 0, st>>>(D);
    OPE_CHECK(cudaGetLastError());
    k_lm_continue<<<1, 256, 0, st>>>(D, handle);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 4;
    return OPE_OK;
}

int build_graph(int model, const LMDev& D, char* base, const Layout& L, double tol, cudaStream_t st,
                GraphCache& G) {
    if (G.exec) {
        cudaGraphExecDestroy(G.exec);
        cudaGraphDestroy(G.graph);
        G.exec = nullptr;
        G.graph = nullptr;
    }
    cudaGraph_t g;
    OPE_CHECK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle handle;
    OPE_CHECK(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    OPE_CHECK(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    OPE_CHECK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_body(model, D, base, L, tol, st, handle);
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st, &captured);
    if (rc != OPE_OK) { cudaGraphDestroy(g); return rc; }
    if (ec != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(ec, "cudaStreamEndCapture"); }
    cudaGraphExec_t exec;
    const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
    if (ei != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(ei, "cudaGraphInstantiate"); }
    G.exec = exec;
    G.graph = g;
    return OPE_OK;
}

}  // namespace

size_t calib_workspace_bytes(size_t nq, size_t ns, int dim) { return layout(nq, ns, dim).total; }

size_t calib_pinned_bytes(size_t nq, size_t ns, int dim) {
    return align_up(nq * sizeof(int32_t), 256) + align_up(nq * sizeof(double), 256) +
           align_up(ns * dim * sizeof(double), 256);
}

// Stage one calibration batch and enqueue all of it on `st`: inputs (kind:
// host or device), the initial residual pass, the conditional-WHILE LM graph,
// the final Jacobian and the diagnostics, and the copy of the results to
// `out` (out_kind).  off_h is a host copy of the surface offsets; `pin` is a
// pinned host buffer of calib_pinned_bytes(); `dev` a device region of
// calib_workspace_bytes().  The graph is cached in *G when G->cache is set,
// else it is left in *G for the caller to release after the stream completes.
int calib_enqueue(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
                  const int64_t* surf_offsets, const int64_t* off_h, size_t ns, const double* p0,
                  ope_calib_result* out, double tol, cudaMemcpyKind kind, cudaMemcpyKind out_kind, char* dev,
                  char* pin, cudaStream_t st, CalibGraph* G, const CalibExtra* ex) {
    ThreadCtx& c = tctx();
    const int dim = param_stride(model);
    const Layout L = layout(nq, ns, dim);
    char* base = dev;
    if (off_h[0] != 0 || off_h[ns] != (int64_t)nq) return set_error(OPE_ERR_INVALID_ARG, "surf_offsets must span [0, n)");
    int32_t* sidx = reinterpret_cast<int32_t*>(pin);
    for (size_t s = 0; s < ns; ++s) {
        if (off_h[s + 1] < off_h[s]) return set_error(OPE_ERR_INVALID_ARG, "surf_offsets not sorted");
        for (int64_t i = off_h[s]; i < off_h[s + 1]; ++i) sidx[i] = (int32_t)s;
    }
    double* wh = reinterpret_cast<double*>(pin + align_up(nq * sizeof(int32_t), 256));
    double* ph = reinterpret_cast<double*>(pin + align_up(nq * sizeof(int32_t), 256) + align_up(nq * sizeof(double), 256));
    OPE_CHECK(cudaMemcpyAsync(base + L.q, quotes, nq * sizeof(ope_contract), kind, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.iv, iv_market, nq * sizeof(double), kind, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.off, surf_offsets, (ns + 1) * sizeof(int64_t), kind, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.sidx, sidx, nq * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    if (weights) {
        OPE_CHECK(cudaMemcpyAsync(base + L.w, weights, nq * sizeof(double), kind, st));
    } else {
        for (size_t i = 0; i < nq; ++i) wh[i] = 1.0;
        OPE_CHECK(cudaMemcpyAsync(base + L.w, wh, nq * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    const double* p0_dev;
    if (kind == cudaMemcpyDeviceToDevice) {
        p0_dev = p0;
    } else {
        std::memcpy(ph, p0, ns * dim * sizeof(double));
        OPE_CHECK(cudaMemcpyAsync(base + L.ptrial, ph, ns * dim * sizeof(double), cudaMemcpyHostToDevice, st));
        p0_dev = reinterpret_cast<const double*>(base + L.ptrial);
    }
    LMDev D = make_dev(base, L, (int)nq, (int)ns, dim);
    if (ex && ex->prior) {
        if (!ex->reg_weight) return set_error(OPE_ERR_INVALID_ARG, "a prior needs its reg_weight");
        OPE_CHECK(cudaMemcpyAsync(base + L.prior, ex->prior, ns * dim * sizeof(double), cudaMemcpyHostToDevice, st));
        OPE_CHECK(cudaMemcpyAsync(base + L.regw, ex->reg_weight, ns * sizeof(double), cudaMemcpyHostToDevice, st));
        D.prior = reinterpret_cast<const double*>(base + L.prior);
        D.regw = reinterpret_cast<const double*>(base + L.regw);
    }
    if (ex && ex->group) {
        if (ex->n_group < 1 || (size_t)ex->n_group > ns) return set_error(OPE_ERR_INVALID_ARG, "bad restart group count");
        for (size_t s = 0; s < ns; ++s)
            if (ex->group[s] < 0 || ex->group[s] >= ex->n_group) return set_error(OPE_ERR_INVALID_ARG, "bad restart group");
        std::vector<unsigned long long> gb(ex->n_group);
        for (int g = 0; g < ex->n_group; ++g) {
            const double v = ex->gbest0 ? ex->gbest0[g] : __builtin_inf();
            if (!(v >= 0.0)) return set_error(OPE_ERR_INVALID_ARG, "shared best SSE must be >= 0");
            std::memcpy(&gb[g], &v, sizeof(double));
        }
        OPE_CHECK(cudaMemcpyAsync(base + L.group, ex->group, ns * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        OPE_CHECK(cudaMemcpyAsync(base + L.gbest, gb.data(), gb.size() * sizeof(unsigned long long),
                                  cudaMemcpyHostToDevice, st));
        D.group = reinterpret_cast<const int32_t*>(base + L.group);
        D.gbest = reinterpret_cast<unsigned long long*>(base + L.gbest);
    }
    // initial state and residuals at p0 (calibration.rs:472-475)
    k_lm_init<<<((int)ns + 127) / 128, 128, 0, st>>>(D, p0_dev);
    OPE_CHECK(cudaGetLastError());
    const PanelSink sink = pricing_sink(D, base, L);
    OPE_TRY(launch_price_persistent(model, D.q, nq, D.off, ns, nullptr, D.pcur, tol, D.price,
                                    carve_price_scratch(base + L.scratch, nq), st, nullptr, D.tmask, &sink));
    k_lm_residuals<<<((int)nq + 127) / 128, 128, 0, st>>>(D, nullptr, D.price, D.res);
    OPE_CHECK(cudaGetLastError());
    k_lm_sse0<<<((int)ns * 32 + 127) / 128, 128, 0, st>>>(D);
    OPE_CHECK(cudaGetLastError());
    OPE_CHECK(cudaMemsetAsync(D.counters, 0, 4 * sizeof(unsigned int), st));
    c.launches += 3;
    // the LM loop: one conditional-WHILE graph launch
    GraphCache& g = G->cache;
    const bool has_prior = D.prior != nullptr, has_group = D.group != nullptr;
    if (!(g.exec && g.ws == dev && g.model == model && g.nq == (int)nq && g.ns == (int)ns && g.tol == tol &&
          g.stream == st && g.prior == has_prior && g.group == has_group)) {
        OPE_TRY(build_graph(model, D, base, L, tol, st, g));
        g.ws = dev;
        g.model = model;
        g.nq = (int)nq;
        g.ns = (int)ns;
        g.tol = tol;
        g.stream = st;
        g.prior = has_prior;
        g.group = has_group;
    }
    OPE_CHECK(cudaGraphLaunch(g.exec, st));
    // final Jacobian at the last accepted parameters, diagnostics
    OPE_TRY(launch_jac(model, D, base, L, st));
    ope_calib_result* d_out = reinterpret_cast<ope_calib_result*>(base + L.out);
    k_lm_final<<<((int)ns * 32 + 127) / 128, 128, 0, st>>>(D, d_out);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    OPE_CHECK(cudaMemcpyAsync(out, d_out, ns * sizeof(ope_calib_result), out_kind, st));
    return OPE_OK;
}

CalibGraph* calib_graph_new() { return new CalibGraph(); }
void calib_graph_delete(CalibGraph* G) {
    if (!G) return;
    calib_graph_release(G);
    delete G;
}

void calib_graph_release(CalibGraph* G) {
    GraphCache& g = G->cache;
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = GraphCache();
}

int run_calibration(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
                    const int64_t* surf_offsets, size_t ns, const double* p0, ope_calib_result* out, double tol,
                    bool device_ptrs, cudaStream_t ust, const CalibExtra* ex) {
    ThreadCtx& c = tctx();
    const int dim = param_stride(model);
    cudaStream_t st = device_ptrs ? ust : c.stream;
    if (device_ptrs && st == nullptr) st = c.stream;  // capture needs a non-legacy stream
    void* ws;
    OPE_TRY(ensure_workspace(calib_workspace_bytes(nq, ns, dim), &ws, st));
    void* pin;
    OPE_TRY(ensure_pinned(calib_pinned_bytes(nq, ns, dim), &pin));
    std::vector<int64_t> off_h(ns + 1);
    if (device_ptrs) {
        OPE_CHECK(cudaMemcpyAsync(off_h.data(), surf_offsets, (ns + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        OPE_CHECK(cudaStreamSynchronize(st));
    } else {
        std::memcpy(off_h.data(), surf_offsets, (ns + 1) * sizeof(int64_t));
    }
    const cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    OPE_TRY(calib_enqueue(model, quotes, iv_market, weights, nq, surf_offsets, off_h.data(), ns, p0, out, tol, kind,
                          device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, static_cast<char*>(ws),
                          static_cast<char*>(pin), st, &g_lm_graph, ex));
    // the pinned staging is reused by the next call: wait for this one's copies
    OPE_CHECK(cudaStreamSynchronize(st));
    return OPE_OK;
}

namespace {
// batch.rs:51-56 batch_implied_vol: one thread per contract.
__global__ void k_batch_iv(const ope_contract* __restrict__ con, const double* __restrict__ price, long long n,
                           double* __restrict__ iv, int32_t* __restrict__ ok) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    const bool good = implied_vol_d(iv_contract(con[i]), price[i], &v);
    iv[i] = good ? v : 0.0;
    ok[i] = good ? 1 : 0;
}
}  // namespace

int launch_batch_iv(const ope_contract* con, const double* price, size_t n, double* iv, int32_t* ok, cudaStream_t st) {
    if (n == 0) return OPE_OK;
    k_batch_iv<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(con, price, (long long)n, iv, ok);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 1;
    return OPE_OK;
}

int run_calib_jacobian(int model, const ope_contract* quotes, const double* iv_market, size_t nq,
                       const int64_t* surf_offsets, size_t ns, const double* params, double* out_jac,
                       double* out_res, double tol) {
    ThreadCtx& c = tctx();
    const int dim = param_stride(model);
    const Layout L = layout(nq, ns, dim);
    cudaStream_t st = c.stream;
    void* ws;
    OPE_TRY(ensure_workspace(L.total, &ws, st));
    char* base = static_cast<char*>(ws);
    std::vector<int32_t> sidx(nq);
    for (size_t s = 0; s < ns; ++s)
        for (int64_t i = surf_offsets[s]; i < surf_offsets[s + 1]; ++i) sidx[i] = (int32_t)s;
    std::vector<double> wv(nq, 1.0);
    std::vector<int32_t> ones(ns, 1);
    OPE_CHECK(cudaMemcpyAsync(base + L.q, quotes, nq * sizeof(ope_contract), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.iv, iv_market, nq * sizeof(double), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.w, wv.data(), nq * sizeof(double), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.off, surf_offsets, (ns + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.sidx, sidx.data(), nq * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.pcur, params, ns * dim * sizeof(double), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(base + L.jmask, ones.data(), ns * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    LMDev D = make_dev(base, L, (int)nq, (int)ns, dim);
    OPE_CHECK(cudaMemsetAsync(D.pslot, 0, ns * sizeof(int32_t), st));
    OPE_CHECK(cudaMemsetAsync(D.jslot, 0, ns * sizeof(int32_t), st));
    const PanelSink sink = pricing_sink(D, base, L);
    OPE_TRY(launch_price_persistent(model, D.q, nq, D.off, ns, nullptr, D.pcur, tol, D.price,
                                    carve_price_scratch(base + L.scratch, nq), st, nullptr, nullptr, &sink));
    OPE_TRY(launch_jac(model, D, base, L, st));
    k_lm_residuals<<<((int)nq + 127) / 128, 128, 0, st>>>(D, nullptr, D.price, D.res);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    OPE_CHECK(cudaMemcpyAsync(out_jac, D.jrow, nq * dim * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (out_res) OPE_CHECK(cudaMemcpyAsync(out_res, D.res, nq * sizeof(double), cudaMemcpyDeviceToHost, st));
    OPE_CHECK(cudaStreamSynchronize(st));
    return OPE_OK;
}

}  // namespace ope
