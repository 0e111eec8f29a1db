// x pass of the fused RK3 stage on long lines, with no barrier and no
// cluster: the x filter (filterCFD + tridiagonalSolver, mathlib.c:296-354,
// 8-30) in one kernel (xf_kernel) and the x derivatives (derivCFD1st/2nd,
// mathlib.c:33-86, 163-218) of the filtered state and of Ey, Ez in another
// (xd_kernel).
//
// Each thread solves one chunk of L rows of one column (lanes: 32 adjacent
// columns, so every row access is a coalesced 256-byte load or store).  The
// chunk's non-cyclic Thomas solve needs two numbers from outside the chunk:
// the forward value y(r0-1) and the backward value x(r1) (r1 = r0 + L).  Both
// are linear functionals of the line:
//   y(r0-1) = sum_k P_k r_k,          P_k = prod_{t=k+1..r0-1} (-m_t),
//   x(r1)   = A y(r1-1) + sum_k c_k r_k,
// with r the stencil right-hand side (a 7-point stencil of the line u).  The
// host composes them with the stencil into taps on u (an FIR of K+6 taps),
// so the kernel forms each inflow as one dot product of the line with the
// taps instead of a sequential lead-in.  The factors decay geometrically
// (|m|, |g| = 0.45 for the derivative matrix, 0.82 for the filter), and the
// host truncates the sums where the dropped weight is below 2^-60 of the
// kept one: K = 56 rows for the derivatives, 216 for the filter.  Chunks
// whose inflows and rows lie in the interior (constant factors, interior
// stencils, no periodic wrap) share one set of taps, passed as a kernel
// parameter (constant bank, so the dot products read their taps as FMA
// operands); the chunks near the line ends take exact functionals of their
// own from a table in global memory (no truncation at all where the line
// ends within reach), with the tabulated factors and the closure stencils.
// The line values enter the dot products as differences to a nearby value u_c
// (plus u_c times the sum of the taps), which keeps the rounding of the
// inflow at the size of the line's variation, not of its mean.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "common.cuh"
#include "xcore.cuh"
#include "xfir.cuh"

namespace mhd {

// ---------------------------------------------------------------------------
// host side: the inflow functionals
// ---------------------------------------------------------------------------

// Host copies of a system's per-row Thomas factors (as xsolve.cu forms them).
struct XHostFactors {
    std::vector<double> m, ib, g;
};


// Weights of the right-hand side of operator `op` at row gr on u(gr-3..gr+3)
// (mathlib.c:46-85, 176-217, 309-353; unwrapped indices, the periodic wrap
// is applied when the line is read).
static void rhs_weights(const Ctx *c, int op, long gr, long n, long double w[7])
{
    const XStencil &s = c->xs[op];
    const long double sc = s.scale;
    for (int k = 0; k < 7; k++) w[k] = 0.0L;
    if (gr == 0) {
        w[1] = sc * s.e0; w[2] = sc * s.e1; w[3] = sc * s.e2; w[4] = sc * s.e3; w[5] = sc * s.e4;
    } else if (gr == n - 1) {
        const long double g = s.edge_sign * sc;
        w[5] = g * s.e0; w[4] = g * s.e1; w[3] = g * s.e2; w[2] = g * s.e3; w[1] = g * s.e4;
    } else if (op == XOP_D1) {
        w[0] = -sc * s.c; w[1] = -sc * s.b; w[2] = -sc * s.a;
        w[4] = sc * s.a; w[5] = sc * s.b; w[6] = sc * s.c;
    } else if (op == XOP_D2) {
        w[0] = w[6] = sc * s.c; w[1] = w[5] = sc * s.b; w[2] = w[4] = sc * s.a;
        w[3] = -2.0L * sc * ((long double)s.a + s.b + s.c);
    } else {
        w[0] = w[6] = s.d; w[1] = w[5] = s.c; w[2] = w[4] = s.b; w[3] = s.a;
    }
}

// A functional sum_j h_j u(j0 + j) (j = 0..h.size()-1), plus the constant A
// of the backward one.
struct XNFun {
    long j0 = 0;
    std::vector<long double> h;
    long double A = 0.0L;
};

// add weight `p` times the right-hand side of row k to f
static void add_row(const Ctx *c, int op, long k, long n, long double p,
                    std::map<long, long double> &acc)
{
    long double w[7];
    rhs_weights(c, op, k, n, w);
    for (int s = 0; s < 7; s++)
        if (w[s] != 0.0L) acc[k - 3 + s] += p * w[s];
}

static XNFun to_fun(const std::map<long, long double> &acc)
{
    XNFun f;
    if (acc.empty()) return f;
    f.j0 = acc.begin()->first;
    const long j1 = acc.rbegin()->first;
    f.h.assign((size_t)(j1 - f.j0 + 1), 0.0L);
    for (const auto &kv : acc) f.h[(size_t)(kv.first - f.j0)] = kv.second;
    return f;
}

// y(r0 - 1) as a functional of the line, the sum truncated after K rows
// (exact when the line starts within them)
static XNFun fwd_fun(const Ctx *c, const XHostFactors &F, int op, long r0, int K)
{
    const long n = c->nx;
    std::map<long, long double> acc;
    long double P = 1.0L;
    for (long k = r0 - 1; k >= 0 && k >= r0 - K; k--) {
        add_row(c, op, k, n, P, acc);
        P *= -(long double)F.m[k];
    }
    return to_fun(acc);
}

// x(r1) = A y(r1 - 1) + functional of the line, truncated after K rows
// (exact when the line ends within them)
static XNFun bwd_fun(const Ctx *c, const XHostFactors &F, int op, long r1, int K)
{
    const long n = c->nx;
    const long kmax = std::min(n - 1, r1 + (long)K - 1);
    if (r1 >= n) return XNFun{};
    // q_k = ib_k prod_{t=r1..k-1} (-g_t); c_i = q_i + (-m_{i+1}) c_{i+1};
    // A = sum_k q_k prod_{t=r1..k} (-m_t) = (-m_{r1}) c_{r1}
    std::vector<long double> q((size_t)(kmax - r1 + 1)), cc(q.size());
    long double G = 1.0L;
    for (long k = r1; k <= kmax; k++) {
        q[(size_t)(k - r1)] = (long double)F.ib[k] * G;
        G *= -(long double)F.g[k];
    }
    long double run = 0.0L;
    for (long i = kmax; i >= r1; i--) {
        run = q[(size_t)(i - r1)] + (i + 1 <= kmax ? -(long double)F.m[i + 1] * run : 0.0L);
        cc[(size_t)(i - r1)] = run;
    }
    std::map<long, long double> acc;
    for (long i = r1; i <= kmax; i++) add_row(c, op, i, n, cc[(size_t)(i - r1)], acc);
    XNFun f = to_fun(acc);
    f.A = -(long double)F.m[r1] * cc[0];
    return f;
}

// The functional rounded to doubles, its sum (from the long doubles) and
// its constant.
struct XNRounded {
    long j0 = 0;
    std::vector<double> h;
    double sum = 0.0, A = 0.0;
};

static XNRounded round_fun(const XNFun &f)
{
    XNRounded r;
    r.j0 = f.j0;
    long double s = 0.0L;
    for (long double v : f.h) {
        r.h.push_back((double)v);
        s += v;
    }
    r.sum = (double)s;
    r.A = (double)f.A;
    return r;
}

static bool same_fun(const XNRounded &a, const XNRounded &b, long shift)
{
    if (a.h.size() != b.h.size() || a.j0 != b.j0 + shift) return false;
    if (std::memcmp(&a.A, &b.A, sizeof(double)) != 0) return false;
    if (std::memcmp(&a.sum, &b.sum, sizeof(double)) != 0) return false;
    return a.h.empty() || std::memcmp(a.h.data(), b.h.data(), sizeof(double) * a.h.size()) == 0;
}

static int host_factors(const Ctx *c, int op, XHostFactors &F)
{
    const long n = c->nx;
    F.m.resize(n);
    F.ib.resize(n);
    F.g.resize(n);
    MHD_CUDA_TRY(cudaMemcpy(F.m.data(), c->xt[op].m, sizeof(double) * n, cudaMemcpyDeviceToHost));
    MHD_CUDA_TRY(cudaMemcpy(F.ib.data(), c->xt[op].invB, sizeof(double) * n, cudaMemcpyDeviceToHost));
    MHD_CUDA_TRY(cudaMemcpy(F.g.data(), c->xt[op].g, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return MHDGPU_OK;
}

// Host side of the chunked x pass: the parameter blocks and the device
// tables they point to.
struct XNHost {
    XDParams d;
    XFParams f;
    std::vector<void *> dev;
};

template <typename T>
static int dev_copy(XNHost *h, const std::vector<T> &v, const T **out)
{
    *out = nullptr;
    if (v.empty()) return MHDGPU_OK;
    void *p = nullptr;
    MHD_CUDA_TRY(cudaMalloc(&p, sizeof(T) * v.size()));
    h->dev.push_back(p);
    MHD_CUDA_TRY(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    *out = static_cast<const T *>(p);
    return MHDGPU_OK;
}

// Chunk the line in pieces of L rows and build, for the systems ops[0..ns)
// sharing the factors F, the interior taps (tap count NT = K + 6) and the
// table of the chunks that cannot use them.  Returns MHDGPU_ERR_UNSUPPORTED
// when the line is too short to have interior chunks or the interior factors
// do not decay below 2^-60 within K rows.
template <int NT>
static int build_set(Ctx *c, XNHost *h, const XHostFactors &F, const int *ops, int ns, int L,
                     XNTaps<NT> *inner, XNCommon &k)
{
    constexpr int K = NT - 6;
    const long n = c->nx;
    const long nch = (n + L - 1) / L;
    // the canonical interior chunk: in the middle of the line; on lines too
    // short to have one every chunk takes its own functionals from the table
    const long rc = (n / 2 / L) * L;
    const bool has_interior = rc - K - 3 >= XF_EDGE && rc + L + K + 3 <= n - XF_EDGE;
    const double m = F.m[n / 2], ib = F.ib[n / 2], g = F.g[n / 2];
    // the truncation: the dropped weights are below 2^-60 of the kept ones
    // (the factors of the middle row are the interior limit on long lines
    // and decay no slower than it on short ones)
    if (std::pow(std::fabs(m), K) >= std::ldexp(1.0, -60) ||
        std::pow(std::fabs(g), K) >= std::ldexp(1.0, -60))
        return MHDGPU_ERR_UNSUPPORTED;
    std::vector<XNRounded> cf(ns), cb(ns);
    for (int s = 0; has_interior && s < ns; s++) {
        cf[s] = round_fun(fwd_fun(c, F, ops[s], rc, K));
        cb[s] = round_fun(bwd_fun(c, F, ops[s], rc + L, K));
        if ((int)cf[s].h.size() != NT || (int)cb[s].h.size() != NT || cf[s].j0 != rc - K - 3 ||
            cb[s].j0 != rc + L - 3)
            return MHDGPU_ERR_UNSUPPORTED;
        for (int t = 0; t < NT; t++) {
            inner[s].f[t] = cf[s].h[t];
            inner[s].b[t] = cb[s].h[t];
        }
        inner[s].fsum = cf[s].sum;
        inner[s].bsum = cb[s].sum;
        inner[s].A = cb[s].A;
    }
    std::vector<int> eidx((size_t)nch, -1);
    std::vector<XNEdge> edges;
    std::vector<double> taps;
    for (long ci = 0; ci < nch; ci++) {
        const long r0 = ci * L, r1 = std::min(n, r0 + L);
        std::vector<XNRounded> ff(ns), fb(ns);
        bool interior = has_interior && r1 - r0 == L && r0 >= 3 && r1 + 3 <= n;
        for (long r = r0; interior && r < r1; r++)
            interior = std::memcmp(&F.m[r], &m, sizeof m) == 0 &&
                       std::memcmp(&F.ib[r], &ib, sizeof ib) == 0 &&
                       std::memcmp(&F.g[r], &g, sizeof g) == 0;
        for (int s = 0; s < ns; s++) {
            ff[s] = round_fun(r0 > 0 ? fwd_fun(c, F, ops[s], r0, K) : XNFun{});
            fb[s] = round_fun(r1 < n ? bwd_fun(c, F, ops[s], r1, K) : XNFun{});
            interior = interior && same_fun(ff[s], cf[s], r0 - rc) && same_fun(fb[s], cb[s], r0 - rc);
        }
        if (interior) continue;
        eidx[(size_t)ci] = (int)edges.size();
        for (int s = 0; s < ns; s++) {
            XNEdge e;
            e.fo = (int)taps.size();
            e.fj0 = (int)ff[s].j0;
            e.fn = (int)ff[s].h.size();
            taps.insert(taps.end(), ff[s].h.begin(), ff[s].h.end());
            e.bo = (int)taps.size();
            e.bj0 = (int)fb[s].j0;
            e.bn = (int)fb[s].h.size();
            taps.insert(taps.end(), fb[s].h.begin(), fb[s].h.end());
            e.fsum = ff[s].sum;
            e.bsum = fb[s].sum;
            e.A = fb[s].A;
            edges.push_back(e);
        }
    }
    int rc2;
    if ((rc2 = dev_copy(h, eidx, &k.eidx))) return rc2;
    if ((rc2 = dev_copy(h, edges, &k.edge))) return rc2;
    if ((rc2 = dev_copy(h, taps, &k.taps))) return rc2;
    k.m = m;
    k.ib = ib;
    k.g = g;
    k.nx = n;
    k.ny = c->ny;
    k.nch = (int)nch;
    k.flag = c->dflag;
    return MHDGPU_OK;
}

// ---------------------------------------------------------------------------
// device side
// ---------------------------------------------------------------------------

// interior right-hand side of operator OP on u(i-3..i+3) = w0..w6, in the
// reference's difference form (mathlib.c:46-85, 176-217, 309-353)
template <int OP>
__device__ __forceinline__ double xn_rhs(const XStencil &s, double w0, double w1, double w2,
                                         double w3, double w4, double w5, double w6)
{
    if (OP == XOP_D1) return s.scale * (s.a * (w4 - w2) + s.b * (w5 - w1) + s.c * (w6 - w0));
    if (OP == XOP_D2)
        return s.scale * (s.a * (w4 - 2 * w3 + w2) + s.b * (w5 - 2 * w3 + w1) + s.c * (w6 - 2 * w3 + w0));
    return s.a * w3 + s.b * (w4 + w2) + s.c * (w5 + w1) + s.d * (w6 + w0);
}

__device__ __forceinline__ long xn_wrap(long r, long n) { return r < 0 ? r + n : (r >= n ? r - n : r); }

// The line(s) a job reads: one field column, or Ey and Ez formed from the
// state's u and B columns (E = -u x B, calcRHS.c:24-43).
struct XNField {
    const double *p;  // the column of the field
    long ny;
    static constexpr int NI = 1;
    __device__ __forceinline__ void get(long r, double *v) const { v[0] = p[r * ny]; }
};
struct XNEfield {
    const double *p;  // the column of field 0 of the state
    long ny, plane;
    static constexpr int NI = 2;
    __device__ __forceinline__ void get(long r, double *v) const
    {
        const double *q = p + r * ny;
        const double ux = q[UX * plane], uy = q[UY * plane], uz = q[UZ * plane];
        const double bx = q[BX * plane], by = q[BY * plane], bz = q[BZ * plane];
        v[0] = ux * bz - uz * bx;  // Ey
        v[1] = uy * bx - ux * by;  // Ez
    }
};

// Thomas solve of one chunk, rows r0 .. r0+len-1, for NS systems sharing the
// factors in k: system s applies operator OPS[s] to input INS[s] of `in`, with the interior taps tp0/tp1 or, for an edge chunk (e >= 0), the
// table entries k.edge[e + E1 * s].  The recurrences run in T.  Results x go to
// emit(s, row, x).
template <int L, typename T, int NS, int NT, int OP0, int OP1, int IN1, int E1, int UNR, class In,
          class Emit>
__device__ __forceinline__ void xn_chunk(const XNCommon &k, const XNTaps<NT> &tp0,
                                         const XNTaps<NT> &tp1, const XStencil &st0,
                                         const XStencil &st1, const In &in, long r0, int len,
                                         int e, Emit emit)
{
    constexpr int NI = In::NI;
    constexpr int ops[2] = {OP0, OP1};
    constexpr int ins[2] = {0, IN1};
    constexpr int eo[2] = {0, E1};  // table entry of each system, from e
#define TP(s) ((s) == 0 ? tp0 : tp1)
#define ST(s) ((s) == 0 ? st0 : st1)
    const long n = k.nx;
    T Y[NS][L];
    T y[NS];
    if (e < 0) {
        // ---- interior chunk: parameter taps, constant factors, no wrap ----
        double uc[NI], acc[NS][2];
        in.get(r0 - 1, uc);
#pragma unroll
        for (int s = 0; s < NS; s++) acc[s][0] = acc[s][1] = 0.0;
#pragma unroll (UNR)
        for (int t = 0; t < NT; t++) {
            double v[NI];
            in.get(r0 - (NT - 6) - 3 + t, v);
#pragma unroll
            for (int s = 0; s < NS; s++)
                acc[s][t & 1] = fma(TP(s).f[t], v[ins[s]] - uc[ins[s]], acc[s][t & 1]);
        }
#pragma unroll
        for (int s = 0; s < NS; s++) y[s] = (T)(acc[s][0] + acc[s][1] + uc[ins[s]] * TP(s).fsum);
        double w[NI][7];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            double v[NI];
            in.get(r0 - 3 + q, v);
#pragma unroll
            for (int i = 0; i < NI; i++) w[i][q] = v[i];
        }
        const T m = (T)k.m;
#pragma unroll
        for (int r = 0; r < L; r++) {
            double v[NI];
            in.get(r0 + r + 3, v);
#pragma unroll
            for (int i = 0; i < NI; i++) w[i][6] = v[i];
#pragma unroll
            for (int s = 0; s < NS; s++) {
                const double *x = w[ins[s]];
                double rhs;
                if (ops[s] == XOP_D1) rhs = xn_rhs<XOP_D1>(ST(s), x[0], x[1], x[2], x[3], x[4], x[5], x[6]);
                else if (ops[s] == XOP_D2) rhs = xn_rhs<XOP_D2>(ST(s), x[0], x[1], x[2], x[3], x[4], x[5], x[6]);
                else rhs = xn_rhs<XOP_F>(ST(s), x[0], x[1], x[2], x[3], x[4], x[5], x[6]);
                y[s] = (T)rhs - m * y[s];
                Y[s][r] = y[s];
            }
#pragma unroll
            for (int i = 0; i < NI; i++)
#pragma unroll
                for (int q = 0; q < 6; q++) w[i][q] = w[i][q + 1];
        }
        in.get(r0 + L, uc);
#pragma unroll
        for (int s = 0; s < NS; s++) acc[s][0] = acc[s][1] = 0.0;
#pragma unroll (UNR)
        for (int t = 0; t < NT; t++) {
            double v[NI];
            in.get(r0 + L - 3 + t, v);
#pragma unroll
            for (int s = 0; s < NS; s++)
                acc[s][t & 1] = fma(TP(s).b[t], v[ins[s]] - uc[ins[s]], acc[s][t & 1]);
        }
        const T ib = (T)k.ib, g = (T)k.g;
#pragma unroll
        for (int s = 0; s < NS; s++) {
            T x = (T)(acc[s][0] + acc[s][1] + uc[ins[s]] * TP(s).bsum + TP(s).A * (double)y[s]);
#pragma unroll
            for (int r = L - 1; r >= 0; r--) {
                x = Y[s][r] * ib - g * x;
                emit(s, r0 + r, x);
            }
        }
        return;
    }
    // ---- chunk near a line end: table taps, tabulated factors, closures ----
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const XNEdge &E = k.edge[e + eo[s]];
        double acc = 0.0, uc[NI];
        if (E.fn > 0) {
            in.get(xn_wrap(r0 - 1, n), uc);
            for (int t = 0; t < E.fn; t++) {
                double v[NI];
                in.get(xn_wrap((long)E.fj0 + t, n), v);
                acc = fma(k.taps[E.fo + t], v[ins[s]] - uc[ins[s]], acc);
            }
            acc += uc[ins[s]] * E.fsum;
        }
        y[s] = (T)acc;
    }
    double w[NI][7];
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double v[NI];
        in.get(xn_wrap(r0 - 3 + q, n), v);
#pragma unroll
        for (int i = 0; i < NI; i++) w[i][q] = v[i];
    }
#pragma unroll
    for (int r = 0; r < L; r++) {
        if (r < len) {
            const long gr = r0 + r;
            double v[NI];
            in.get(xn_wrap(gr + 3, n), v);
#pragma unroll
            for (int i = 0; i < NI; i++) w[i][6] = v[i];
            const T m = (T)k.tm[gr];
#pragma unroll
            for (int s = 0; s < NS; s++) {
                const double *x = w[ins[s]];
                double rhs = stencil(ST(s), x[0], x[1], x[2], x[3], x[4], x[5], x[6], gr, n);
                y[s] = (T)rhs - m * y[s];
                Y[s][r] = y[s];
            }
#pragma unroll
            for (int i = 0; i < NI; i++)
#pragma unroll
                for (int q = 0; q < 6; q++) w[i][q] = w[i][q + 1];
        }
    }
#pragma unroll
    for (int s = 0; s < NS; s++) {
        const XNEdge &E = k.edge[e + eo[s]];
        double acc = 0.0, uc[NI];
        if (E.bn > 0) {
            in.get(xn_wrap(r0 + len, n), uc);
            for (int t = 0; t < E.bn; t++) {
                double v[NI];
                in.get(xn_wrap((long)E.bj0 + t, n), v);
                acc = fma(k.taps[E.bo + t], v[ins[s]] - uc[ins[s]], acc);
            }
            acc += uc[ins[s]] * E.bsum + E.A * (double)y[s];
        }
        T x = (T)acc;
#pragma unroll
        for (int r = L - 1; r >= 0; r--) {
            if (r < len) {
                const long gr = r0 + r;
                x = Y[s][r] * (T)k.tib[gr] - (T)k.tg[gr] * x;
                emit(s, gr, x);
            }
        }
    }
#undef TP
#undef ST
}


// CTAs per SM the register budget is set for.  Measured at 4096^2 on one
// B200 (per launch, FP64 / FP32 derivatives / FP64 filter), with 4 chunks
// per CTA: 1 CTA bound (254 registers, no spills) 1.58 / - / 1.60 ms; 3 (168)
// 1.28 / 1.22 / 1.51 ms; 4 (128) 1.40 / 1.18 / 1.60 ms.  With 2 chunks per
// CTA at the same registers (6 and 8 CTAs): 1.23 / 1.16 / 1.46 ms.  The
// spills this costs stay in L1; the extra resident warps hide the latency of
// the inflow loads.
template <typename T>
constexpr int xn_minb() { return sizeof(T) == 8 ? 6 : 8; }

// One warp per chunk, NW chunks (consecutive along the line) per CTA, 32
// columns per CTA; blockIdx.z: the job.
template <int L, typename T, int UNR, int NW>
__global__ void __launch_bounds__(32 * NW, xn_minb<T>()) xd_kernel(const __grid_constant__ XDParams P)
{
    const int lane = threadIdx.x & 31;
    const long j = (long)blockIdx.x * 32 + lane;
    const int ci = (int)blockIdx.y * NW + (int)(threadIdx.x >> 5);
    if (j >= P.k.ny || ci >= P.k.nch) return;
    const long n = P.k.nx, ny = P.k.ny, plane = n * ny;
    const long r0 = (long)ci * L;
    const int len = (int)min((long)L, n - r0);
    const int e = P.k.eidx[ci];
    const int job = (int)blockIdx.z;
    if (job < P.nvar) {
        const int v = job;
        const XNField in{P.in + (size_t)v * plane + j, ny};
        T *d1 = reinterpret_cast<T *>(P.out1) + (size_t)v * plane + j;
        T *d2 = nullptr;
        if (P.out2a && v >= P.d2a_lo && v < P.d2a_lo + 3)
            d2 = reinterpret_cast<T *>(P.out2a) + (size_t)(v - P.d2a_lo) * plane + j;
        else if (P.out2b && v >= P.d2b_lo && v < P.d2b_lo + 3)
            d2 = reinterpret_cast<T *>(P.out2b) + (size_t)(v - P.d2b_lo) * plane + j;
        if (d2)  // d/dx and d2/dx2 share the matrix: one pass over the line
            xn_chunk<L, T, 2, XN_TD, XOP_D1, XOP_D2, 0, 1, UNR>(
                P.k, P.s[0], P.s[1], P.st[0], P.st[1], in, r0, len, e,
                [&](int s, long row, T x) { (s == 0 ? d1 : d2)[row * ny] = x; });
        else
            xn_chunk<L, T, 1, XN_TD, XOP_D1, XOP_D1, 0, 0, UNR>(
                P.k, P.s[0], P.s[0], P.st[0], P.st[0], in, r0, len, e,
                [&](int, long row, T x) { d1[row * ny] = x; });
    } else {  // d/dx of Ey and Ez, formed from the state as the lines are read
        const XNEfield in{P.in + j, ny, plane};
        T *ey = reinterpret_cast<T *>(P.outE) + j, *ez = ey + plane;
        xn_chunk<L, T, 2, XN_TD, XOP_D1, XOP_D1, 1, 0, UNR>(
            P.k, P.s[0], P.s[0], P.st[0], P.st[0], in, r0, len, e,
            [&](int s, long row, T x) { (s == 0 ? ey : ez)[row * ny] = x; });
    }
}

template <int L, typename T, int UNR, int NW>
__global__ void __launch_bounds__(32 * NW, xn_minb<T>()) xf_kernel(const __grid_constant__ XFParams P)
{
    static_assert(sizeof(T) == 8, "the x filter runs in FP64 in both precisions");
    const int lane = threadIdx.x & 31;
    const long j = (long)blockIdx.x * 32 + lane;
    const int ci = (int)blockIdx.y * NW + (int)(threadIdx.x >> 5);
    if (j >= P.k.ny || ci >= P.k.nch) return;
    const long n = P.k.nx, ny = P.k.ny, plane = n * ny;
    const long r0 = (long)ci * L;
    const int len = (int)min((long)L, n - r0);
    const int e = P.k.eidx[ci];
    const int v = (int)blockIdx.z;
    const XNField in{P.in + (size_t)v * plane + j, ny};
    double *out = P.out + (size_t)v * plane + j;
    xn_chunk<L, double, 1, XN_TF, XOP_F, XOP_F, 0, 0, UNR>(
        P.k, P.s, P.s, P.st, P.st, in, r0, len, e,
        [&](int, long row, double x) { out[row * ny] = x; });
}

// ---------------------------------------------------------------------------
// host side: set-up and launches
// ---------------------------------------------------------------------------
// chunks (one warp each) per CTA: at one CTA per SM 4 measured faster than
// 8, and at the register budget of xn_minb 2 faster than 4 (smaller CTAs to
// place; the L1 reuse of the inflow rows is per SM either way)
constexpr int XN_NW = 2;
constexpr int XN_LD = 16;  // rows per chunk of the derivative kernel
constexpr int XN_LF = 32;  // rows per chunk of the filter kernel
// Lines shorter than this keep the cluster x pass (xline.cu), which holds a
// whole short line in one CTA with no redundant work; MHDGPU_XN_MIN_NX sets
// another bound (the chunked pass needs nx >= 2 chunks of XN_LF rows).
// Measured on one B200: a job alone steps faster with the chunked pass from
// 128^2 up (0.61 vs 1.66 ms per step at 128^2, 1.29 vs 1.68 ms at 512^2),
// but the inflow dot products cost more work per cell on short lines, and
// the 64-job ensemble served concurrently (the GPU full) runs 8 % faster
// with the cluster pass below 1024 rows (335 M vs 310 M cell-updates/s).
constexpr long XN_MIN_NX = 1024;

int xn_setup(Ctx *c)
{
    c->xn_on = 0;
    long min_nx = XN_MIN_NX;
    if (const char *e = getenv("MHDGPU_XN_MIN_NX")) min_nx = std::max(2L * XN_LF, atol(e));
    if (c->nx < min_nx || getenv("MHDGPU_NO_XN")) return MHDGPU_OK;
    XNHost *h = new (std::nothrow) XNHost();
    if (!h) return mhd_set_error(MHDGPU_ERR_NOMEM);
    std::memset(&h->d, 0, sizeof h->d);
    std::memset(&h->f, 0, sizeof h->f);
    c->xn = h;
    XHostFactors FD, FD2, FF;
    int rc;
    if ((rc = host_factors(c, XOP_D1, FD)) || (rc = host_factors(c, XOP_D2, FD2)) ||
        (rc = host_factors(c, XOP_F, FF)))
        return rc;
    if (FD.m != FD2.m || FD.ib != FD2.ib || FD.g != FD2.g) return MHDGPU_OK;  // not one matrix
    {
        const int ops[2] = {XOP_D1, XOP_D2};
        rc = build_set<XN_TD>(c, h, FD, ops, 2, XN_LD, h->d.s, h->d.k);
        if (rc == MHDGPU_ERR_UNSUPPORTED) return MHDGPU_OK;
        if (rc) return rc;
        h->d.k.tm = c->xt[XOP_D1].m;
        h->d.k.tib = c->xt[XOP_D1].invB;
        h->d.k.tg = c->xt[XOP_D1].g;
        h->d.st[0] = c->xs[XOP_D1];
        h->d.st[1] = c->xs[XOP_D2];
    }
    {
        XFParams &f = h->f;
        const int ops[1] = {XOP_F};
        rc = build_set<XN_TF>(c, h, FF, ops, 1, XN_LF, &f.s, f.k);
        if (rc == MHDGPU_ERR_UNSUPPORTED) return MHDGPU_OK;
        if (rc) return rc;
        f.k.tm = c->xt[XOP_F].m;
        f.k.tib = c->xt[XOP_F].invB;
        f.k.tg = c->xt[XOP_F].g;
        f.st = c->xs[XOP_F];
    }
    const size_t plane = (size_t)c->nx * c->ny;
    MHD_CUDA_TRY(cudaMalloc(&c->xn_state, sizeof(double) * plane * c->nvar));
    c->xn_on = 1;
    return MHDGPU_OK;
}

void xn_free(Ctx *c)
{
    XNHost *h = static_cast<XNHost *>(c->xn);
    if (h) {
        for (void *p : h->dev) cudaFree(p);
        delete h;
    }
    c->xn = nullptr;
    cudaFree(c->xn_state);
    c->xn_state = nullptr;
    c->xn_on = 0;
}

int launch_xd(Ctx *c, const double *in)
{
    XNHost *h = static_cast<XNHost *>(c->xn);
    if (!c->xn_on || !h) return mhd_set_error(MHDGPU_ERR_INVALID);
    XDParams P = h->d;
    const mhdgpu_params &p = c->p;
    const size_t plane = (size_t)c->nx * c->ny;
    P.in = in;
    P.nvar = c->nvar;
    P.out1 = c->arr[MHDGPU_DUDX];
    P.out2a = p.viscosity > 0 ? c->arr[MHDGPU_D2UDX2] : nullptr;
    P.d2a_lo = UX;
    P.out2b = (p.resistivity > 0 || p.Hall == 1) ? c->arr[MHDGPU_D2BDX2] : nullptr;
    P.d2b_lo = BX;
    // dEdx planes 1 and 2 (Ey, Ez), in the stored element type
    P.outE = c->mixed ? static_cast<void *>(reinterpret_cast<float *>(c->arr[MHDGPU_DEDX]) + plane)
                      : static_cast<void *>(c->arr[MHDGPU_DEDX] + plane);
    const int n2 = (P.out2a ? 3 : 0) + (P.out2b ? 3 : 0);
    const double eb = c->mixed ? 4.0 : 8.0;
    const double bytes = (double)plane * (8.0 * c->nvar + eb * (c->nvar + n2 + 2));
    dim3 grid((unsigned)((c->ny + 31) / 32), (unsigned)((P.k.nch + XN_NW - 1) / XN_NW),
              (unsigned)(c->nvar + 1));
    prof_begin(c, KC_FUSED_X, bytes);
#define XD_LAUNCH(U, W)                                                                          \
    do {                                                                                         \
        if (c->mixed) xd_kernel<XN_LD, float, U, W><<<grid, 32 * W, 0, c->stream>>>(P);          \
        else xd_kernel<XN_LD, double, U, W><<<grid, 32 * W, 0, c->stream>>>(P);                  \
    } while (0)
    // the inflow dot products fully unrolled: every tap's load in flight at
    // once (twice as fast on B200 as unrolling by 8)
    XD_LAUNCH(XN_TD, XN_NW);
#undef XD_LAUNCH
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

int launch_xf(Ctx *c, const double *in, double *out)
{
    XNHost *h = static_cast<XNHost *>(c->xn);
    if (!c->xn_on || !h || in == out) return mhd_set_error(MHDGPU_ERR_INVALID);
    // Mixed precision too takes the FP64 filter: the inflow dot products are
    // FP64 either way, and the FP32 change-system variant (d = A^-1 (B - A) u
    // added to u) measured slower on B200 (2.04 vs 1.58 ms per launch at
    // 4096^2: it spills at the fully unrolled taps); the FP64 filter is also
    // the exact one.
    XFParams P = h->f;
    P.in = in;
    P.out = out;
    const size_t plane = (size_t)c->nx * c->ny;
    const double bytes = (double)plane * 16.0 * c->nvar;
    dim3 grid((unsigned)((c->ny + 31) / 32), (unsigned)((P.k.nch + XN_NW - 1) / XN_NW),
              (unsigned)c->nvar);
    prof_begin(c, KC_FUSED_XF, bytes);
    // the inflow dot products fully unrolled: every tap's load in flight at
    // once (twice as fast on B200 as unrolling by 8)
    xf_kernel<XN_LF, double, XN_TF, XN_NW><<<grid, 32 * XN_NW, 0, c->stream>>>(P);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

}  // namespace mhd
