// Warp-cooperative greedy globally-adaptive Gauss-Kronrod-15 on [0, 1].
//
// Reference: heston.rs:180-212 (gk15_panel, adaptive_gk), heston.rs:29-59
// (nodes/weights), heston.rs:220-229 (gk_integrate).
//
// One warp integrates one integral.  Each step bisects the live panel with
// the largest error estimate: lanes 0-14 evaluate the 15 Kronrod nodes of the
// left child and lanes 16-30 those of the right child (30 of 32 lanes busy);
// a half-warp reduce-scatter forms the K15 and G7 sums.  The live-panel list
// (at most 200 entries of {err, K, a, b}) sits in shared memory, one list per
// warp, and is maintained exactly as the reference maintains its Vec:
//   * argmax by f64::total_cmp with the LAST maximum winning ties (errors are
//     non-negative, so their IEEE bit patterns compare as unsigned integers
//     in total_cmp order; the warp maximum is three redux.sync steps);
//   * swap_remove of the chosen panel, then push(left), push(right);
//   * total += kl + kr - kw; err += el + er - ew, in that association;
//   * stop when err <= tol or 200 panels are live.
// Node positions c + h*x_i and the panel products K*h, |K-G|*h are rounded
// exactly as the reference rounds them (no FMA contraction), so the panel
// geometry is bit-identical; only the integrand values and the order of the
// 15-term sums differ at the last-ulp level.
#pragma once

#include "cf_device.cuh"
#include "checked.cuh"

namespace ope {

constexpr int kMaxPanels = 200;  // heston.rs:194

// GK15 nodes and weights in the reference's order (heston.rs:29-49) with a
// zero pad at index 15, and the G7 weight scattered onto its Kronrod index
// (G7_IDX = {0,3,4,7,8,11,12}, heston.rs:53-59), zero elsewhere.
static __constant__ double c_gk_x[16] = {
    0.0,
    0.2077849550078985, -0.2077849550078985,
    0.4058451513773972, -0.4058451513773972,
    0.5860872354676911, -0.5860872354676911,
    0.7415311855993945, -0.7415311855993945,
    0.8648644233597691, -0.8648644233597691,
    0.9491079123427585, -0.9491079123427585,
    0.9914553711208126, -0.9914553711208126,
    0.0};
static __constant__ double c_gk_wk[16] = {
    0.2094821410847278,
    0.2044329400752989, 0.2044329400752989,
    0.1903505780647854, 0.1903505780647854,
    0.1690047266392679, 0.1690047266392679,
    0.1406532597155259, 0.1406532597155259,
    0.1047900103222502, 0.1047900103222502,
    0.0630920926299786, 0.0630920926299786,
    0.0229353220105292, 0.0229353220105292,
    0.0};
static __constant__ double c_gk_wg[16] = {
    0.4179591836734694,
    0.0, 0.0,
    0.3818300505051189, 0.3818300505051189,
    0.0, 0.0,
    0.2797053914892766, 0.2797053914892766,
    0.0, 0.0,
    0.1294849661688697, 0.1294849661688697,
    0.0, 0.0,
    0.0};

// One warp's live-panel list (structure of arrays, 6400 bytes).
struct PanelStore {
    unsigned long long ekey[kMaxPanels];  // error as IEEE bits (total_cmp order for err >= 0)
    double k[kMaxPanels];
    double a[kMaxPanels];
    double b[kMaxPanels];
};

// Per-lane quadrature constants, loaded once per warp.
struct LaneRule {
    double x, wk, wg;
    bool node;  // lane holds a Kronrod node (lane % 16 < 15)
    int half;   // 0 = left child, 1 = right child
    // reduce-scatter weights: of the K15 and G7 weights of this lane's node,
    // the one whose product the lane keeps (G7 if lane bit 3 is set) and the
    // one whose product it sends to lane ^ 8
    double wkeep, wsend;
};

__device__ __forceinline__ LaneRule lane_rule(int lane) {
    LaneRule R;
    const int j = lane & 15;
    R.x = c_gk_x[j];
    R.wk = c_gk_wk[j];
    R.wg = c_gk_wg[j];
    R.node = j < 15;
    R.half = lane >> 4;
    R.wkeep = (lane & 8) ? R.wg : R.wk;
    R.wsend = (lane & 8) ? R.wk : R.wg;
    return R;
}

// K15 and G7 sums of both children, in every lane.  A reduce-scatter over
// each half-warp: at the first exchange (lanes i and i^8) the lanes with bit
// 3 clear keep a K15 partial sum and those with it set a G7 partial sum (each
// lane sends the product its partner keeps), and three more xor levels
// finish each sum with one shuffle per level.  Every lane adds the same two
// partial sums at each level (commuted in its partner), so all lanes of a
// quarter hold bit-identical totals, summed in the pairing order (8, 4, 2, 1);
// lanes 0, 8, 16 and 24 then broadcast the four totals.
__device__ __forceinline__ void gk_sums(double f, const LaneRule& R, double& Kl, double& Gl, double& Kr,
                                        double& Gr) {
    const unsigned FULL = 0xffffffffu;
    double v = R.wkeep * f;
    v += __shfl_xor_sync(FULL, R.wsend * f, 8);
    v += __shfl_xor_sync(FULL, v, 4);
    v += __shfl_xor_sync(FULL, v, 2);
    v += __shfl_xor_sync(FULL, v, 1);
    Kl = __shfl_sync(FULL, v, 0);
    Gl = __shfl_sync(FULL, v, 8);
    Kr = __shfl_sync(FULL, v, 16);
    Gr = __shfl_sync(FULL, v, 24);
}

// The run cache: node_cf's values at the panels that the contracts of one
// run (consecutive contracts of one surface with the same expiry and rate,
// integrating the same P1 or P2) have bisected, kept by the one warp that
// integrates the run's contracts one after another.  Every panel of the
// quadrature descends from [0, 1] by bisection and a bisection always
// evaluates both children, so the cached panels form a binary tree: entry 0
// is [0, 1], and each entry records the entries of its two children once
// they have been evaluated.  Each live panel of the running integral carries
// its entry (kNoEntry: not cached, nor are its descendants), so a bisection
// finds its children's values with one load, without searching.  A contract
// whose next panel is in the tree skips node_cf (the CF, its square root,
// logarithm and exponentials) and pays only node_finish (its own phase and
// one sin).  The tree lives in global memory (per warp: cap entries of 15
// nodes x {W, A}); when it is full, further panels are evaluated
// uncached.  The cached values are the ones node_cf's result gives (u is
// recomputed from the node, bit for bit), so a contract's price is
// bit-identical with and without the cache.  An entry's w and a are one
// 128-byte line each (15 nodes and a zero pad, written whole so that L2
// never fetches the rest of a partly written line from DRAM).
constexpr uint16_t kNoEntry = 0xffff;
constexpr uint32_t kNoChildren = 0xffffffffu;

struct RunCacheWarp {
    double* w;          // [cap][16]: W = e^{Re Z} / ((1 - t) t), NaN at nodes that are not live
    double* a;          // [cap][16]: Im Z without the phase
    uint32_t* child;    // [cap]: children's entries, left | right << 16 (kNoChildren: none yet)
    uint16_t* slot;     // shared, [kMaxPanels]: entry of each live panel of the running integral
    int cap;            // entries (<= 65535)
    int n_alloc;        // entries in use (warp-uniform; 0 at the start of a run)
    bool on;            // cache this integral's panels (warp-uniform)
};

// node_cf as a real call, for the cached loop: a cache hit needs few
// registers, and the call keeps the node evaluation's register demand (and
// its spills) out of the hit path.
// (Internal linkage, so that ptxas allocates its registers within the
// calling kernel's budget.)
// It returns the cached form: W with the liveness folded in (node_w_live),
// A and u.
namespace {
struct NodeW {
    double w, a, u;
};
template <bool BATES>
__device__ __noinline__ NodeW node_cf_call(const CfConsts& C, double tn) {
    const NodeCf n = node_cf<BATES>(C, tn);
    return NodeW{node_w_live(tn, n), n.a, n.u};
}
}  // namespace

// End of a run: its entries will be rewritten before they are read again, so
// their lines are dropped from L2 without being written back to DRAM
// (discard.global.L2), which keeps the dead data of finished runs from
// costing DRAM bandwidth.  Warp-collective.
__device__ __forceinline__ void run_cache_discard(RunCacheWarp& rc, int lane) {
    __syncwarp();
    for (int j = lane; j < 2 * rc.n_alloc; j += 32) {
        const double* line = j < rc.n_alloc ? rc.w + (size_t)j * 16 : rc.a + (size_t)(j - rc.n_alloc) * 16;
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(line) : "memory");
    }
    __syncwarp();
    rc.n_alloc = 0;
}

// Step hooks of gk_integrate_warp.  The pricing kernels use NoTrace (empty
// and inlined: no code); the QAG trace kernel (trace.cu) records every step.
//   first(lane, f, k0, e0): the first panel [0, 1] (f: this lane's integrand
//     value, lanes 0-14 hold the 15 nodes);
//   step(j, lane, f, a, b, ew, kl, el, kr, er, err, total): bisection j of
//     panel [a, b] (error estimate ew) into children with K and error
//     estimates kl, el, kr, er, and the running error and total after it.
struct NoTrace {
    __device__ __forceinline__ void first(int, double, double, double) const {}
    __device__ __forceinline__ void step(int, int, double, double, double, double, double, double, double, double,
                                         double, double) const {}
};

// Returns the integral (identical in every lane).  `nbis` receives the
// number of bisections (loop iterations of heston.rs:200-210); the final
// live-panel list (nbis + 1 entries) is left in L.  The first panel and every
// bisection go through ONE call site of the integrand, so the (large) inlined
// node evaluation exists once in the instruction stream.
//
// CACHED: with the run cache `rc` (which may be off for this integral): each
// step first looks its panel(s) up in the tree (a hit: both children, or the
// root, already evaluated) and otherwise evaluates node_cf and, while the
// tree has room and the bisected panel is in it, stores the children.
template <bool BATES, bool CACHED = false, class Trace = NoTrace>
__device__ __forceinline__ double gk_integrate_warp(const CfConsts& C, double tol, PanelStore& L, int lane,
                                                    const LaneRule& R, int* nbis, const Trace& tr = Trace(),
                                                    RunCacheWarp* rc = nullptr) {
    const unsigned FULL = 0xffffffffu;
    double total = 0.0, err = 0.0;
    int len = 0;
    // panel under evaluation in this half-warp; first step: [0, 1] on the left half only
    double pa = 0.0, pb = 1.0;
    bool active = (R.half == 0) && R.node;
    double aw = 0.0, bw = 1.0, m = 0.5, kw = 0.0, ew = 0.0;
    int w = 0;
    // cache mode of the step (warp-uniform): hit = read entries el_/er_,
    // put = evaluate and store into them; neither = evaluate uncached.  The
    // first step's panel [0, 1] is entry 0 (read as the left child).
    bool hit = false, put = false;
    int el_ = kNoEntry, er_ = kNoEntry, sw_ = kNoEntry;  // sw_: entry of the bisected panel
    if (CACHED && rc->on) {
        if (rc->n_alloc > 0) {
            hit = true;
            el_ = 0;
        } else if (rc->cap > 0) {
            put = true;
            el_ = 0;
            rc->n_alloc = 1;
        }
    }
    while (true) {
        const double c = 0.5 * (pa + pb), h = 0.5 * (pb - pa);
        const double tn = __dadd_rn(c, __dmul_rn(h, R.x));
        // the node's strike-free part: W, A, u (from the tree on a hit)
        double nw = 0.0, na = 0.0, nu = 0.0;
        if (CACHED && hit) {
            if (active) {
                const size_t i = (size_t)(R.half ? er_ : el_) * 16 + (lane & 15);
                nw = __ldcg(rc->w + i);
                na = __ldcg(rc->a + i);
                nu = node_u_of(tn);
            }
        } else {
            if (active) {
                if (CACHED) {
                    const NodeW nc = node_cf_call<BATES>(C, tn);
                    nw = nc.w;
                    na = nc.a;
                    nu = nc.u;
                } else {
                    const NodeCf nc = node_cf<BATES>(C, tn);
                    nw = node_w(nc);
                    na = nc.a;
                    nu = nc.u;
                }
            }
            // the half-warps that evaluated a child write its entry, the
            // pad lane (15 or 31) the 16th element
            if (CACHED && put && (active || (!R.node && (len > 0 || R.half == 0)))) {
                const size_t i = (size_t)(R.half ? er_ : el_) * 16 + (lane & 15);
                __stcg(rc->w + i, nw);
                __stcg(rc->a + i, na);
            }
        }
        const double f = active ? node_finish_w<CACHED>(C.x, tn, nw, na, nu) : 0.0;
        double Kl, Gl, Kr, Gr;
        gk_sums(f, R, Kl, Gl, Kr, Gr);
        if (len == 0) {
            const double k0 = __dmul_rn(Kl, 0.5), e0 = __dmul_rn(fabs(Kl - Gl), 0.5);
            if (lane == 0) {
                L.ekey[0] = (unsigned long long)__double_as_longlong(e0);
                L.k[0] = k0;
                L.a[0] = 0.0;
                L.b[0] = 1.0;
            }
            total = k0;
            err = e0;
            len = 1;
            tr.first(lane, f, k0, e0);
            if (CACHED && rc->on && lane == 0) {
                rc->slot[0] = (uint16_t)el_;
                if (put) rc->child[0] = kNoChildren;
            }
        } else {
            const double hl = 0.5 * (m - aw), hr = 0.5 * (bw - m);
            const double kl = __dmul_rn(Kl, hl), el = __dmul_rn(fabs(Kl - Gl), hl);
            const double kr = __dmul_rn(Kr, hr), er = __dmul_rn(fabs(Kr - Gr), hr);
            total = __dadd_rn(total, __dsub_rn(__dadd_rn(kl, kr), kw));
            err = __dadd_rn(err, __dsub_rn(__dadd_rn(el, er), ew));
            tr.step(len, lane, f, aw, bw, ew, kl, el, kr, er, err, total);
            if (lane == 0) {
                const int last = len - 1;
                if (w != last) {  // swap_remove
                    L.ekey[w] = L.ekey[last];
                    L.k[w] = L.k[last];
                    L.a[w] = L.a[last];
                    L.b[w] = L.b[last];
                }
                L.ekey[last] = (unsigned long long)__double_as_longlong(el);
                L.k[last] = kl;
                L.a[last] = aw;
                L.b[last] = m;
                L.ekey[len] = (unsigned long long)__double_as_longlong(er);
                L.k[len] = kr;
                L.a[len] = m;
                L.b[len] = bw;
                if (CACHED && rc->on) {
                    if (w != last) rc->slot[w] = rc->slot[last];
                    rc->slot[last] = (uint16_t)el_;
                    rc->slot[len] = (uint16_t)er_;
                    if (put) {
                        rc->child[el_] = kNoChildren;
                        rc->child[er_] = kNoChildren;
                        rc->child[sw_] = (uint32_t)el_ | ((uint32_t)er_ << 16);
                    } else if (hit) {
                        // the children's own child words, read when they are bisected
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(rc->child + el_));
                        asm volatile("prefetch.global.L1 [%0];" ::"l"(rc->child + er_));
                    }
                }
            }
            ++len;
        }
        __syncwarp();
        if (!(err > tol && len < kMaxPanels)) break;
        if (!ope_check(len < kMaxPanels, CHK_PANEL_COUNT)) break;
        // argmax over the live list, last maximum wins (Iterator::max_by);
        // chunks of 32 entries, stopping (warp-uniformly) after the last one in use
        unsigned long long best = 0ull;
        int bi = -1;
#pragma unroll
        for (int j = 0; j < (kMaxPanels + 31) / 32; ++j) {
            if (32 * j >= len) break;
            const int i = lane + 32 * j;
            if (i < len) {
                const unsigned long long kk = L.ekey[i];
                if (kk >= best) { best = kk; bi = i; }
            }
        }
        // warp maximum of the 64-bit keys (high word, then low word among the
        // lanes holding the top high word), then the largest index holding it
        {
            const unsigned hi = (unsigned)(best >> 32), lo = (unsigned)best;
            const unsigned mh = __reduce_max_sync(FULL, hi);
            const unsigned ml = __reduce_max_sync(FULL, hi == mh ? lo : 0u);
            const unsigned mi = __reduce_max_sync(FULL, (hi == mh && lo == ml) ? (unsigned)(bi + 1) : 0u);
            best = ((unsigned long long)mh << 32) | ml;
            bi = (int)mi - 1;
        }
        if (!ope_check(bi >= 0 && bi < len, CHK_PANEL_INDEX)) bi = 0;
        w = bi;
        ew = __longlong_as_double((long long)best);
        kw = L.k[w];
        aw = L.a[w];
        bw = L.b[w];
        m = 0.5 * (aw + bw);
        pa = R.half ? m : aw;
        pb = R.half ? bw : m;
        active = R.node;
        if (CACHED && rc->on) {
            // the children of panel w: in the tree (hit), or new entries (put)
            // while the tree has room for both and w is in it
            sw_ = rc->slot[w];
            hit = put = false;
            el_ = er_ = kNoEntry;
            if (sw_ != kNoEntry && !ope_check(sw_ < rc->n_alloc, CHK_RUN_ENTRY)) sw_ = kNoEntry;
            if (sw_ != kNoEntry) {
                const uint32_t ch = rc->child[sw_];
                if (ch != kNoChildren) {
                    hit = true;
                    el_ = (int)(ch & 0xffffu);
                    er_ = (int)(ch >> 16);
                    if (!ope_check(el_ < rc->n_alloc && er_ < rc->n_alloc, CHK_RUN_ENTRY)) {
                        hit = false;  // evaluate uncached
                        el_ = er_ = kNoEntry;
                        sw_ = kNoEntry;
                    }
                } else if (rc->n_alloc + 2 <= rc->cap) {
                    put = true;
                    el_ = rc->n_alloc;
                    er_ = rc->n_alloc + 1;
                    rc->n_alloc += 2;
                }
            }
        }
        __syncwarp();  // every lane has read entry w before lane 0 rewrites it
    }
    *nbis = len - 1;
    return total;
}

// heston.rs:95-98 + heston.rs:70 (bates.rs:60-62, 37): the Gil-Pelaez
// combination, the max(.,0) clamp on the call, put by parity.  Rounded in the
// reference's association order (no FMA).
__device__ __forceinline__ double finish_price(double s, double k, double t, double r, double q, int opt_type,
                                               double i1, double i2) {
    const double PI = 3.14159265358979323846;
    const double p1 = __dadd_rn(0.5, i1 / PI);
    const double p2 = __dadd_rn(0.5, i2 / PI);
    const double seq = __dmul_rn(s, exp(-q * t));
    const double ker = __dmul_rn(k, exp(-r * t));
    const double call = fmax(__dsub_rn(__dmul_rn(seq, p1), __dmul_rn(ker, p2)), 0.0);
    if (opt_type == 0) return call;
    return __dadd_rn(__dsub_rn(call, seq), ker);
}

}  // namespace ope
