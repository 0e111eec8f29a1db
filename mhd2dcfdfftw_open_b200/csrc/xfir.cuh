// Shared declarations of the chunked x pass (xfir.cu): the kernel parameter
// blocks with the interior inflow taps, and the table entries of the chunks
// near the line ends.
#pragma once

#include "common.cuh"

namespace mhd {

constexpr int XN_KD = 56;             // rows kept in the derivative inflows
constexpr int XN_KF = 216;            // rows kept in the filter inflows
constexpr int XN_TD = XN_KD + 6;      // taps of a derivative inflow
constexpr int XN_TF = XN_KF + 6;      // taps of a filter inflow

// The interior inflows of one system: y(r0-1) = sum_t f[t] u(r0-K-3+t) and
// x(r1) = A y(r1-1) + sum_t b[t] u(r1-3+t); fsum, bsum are the tap sums.
template <int NT>
struct XNTaps {
    double f[NT], b[NT];
    double fsum, bsum, A;
};

// The inflows of one system for a chunk near a line end: taps
// taps[fo + t] on u(fj0 + t), t < fn (likewise bo, bj0, bn), unwrapped rows.
struct XNEdge {
    int fo, fj0, fn, bo, bj0, bn;
    double fsum, bsum, A;
};

struct XNCommon {
    const double *tm, *tib, *tg;  // per-row Thomas factors of the system's matrix
    const int *eidx;              // per chunk: -1 interior, else its first XNEdge
    const XNEdge *edge;
    const double *taps;           // taps of the edge functionals
    double m, ib, g;              // interior factors
    long nx, ny;
    int nch;                      // chunks per line
    int *flag;
};

// x derivatives of the (filtered) state: per field d/dx (and d2/dx2 of u, B),
// and d/dx of Ey, Ez.  Job z < nvar: field z; job nvar: Ey, Ez.
struct XDParams {
    XNTaps<XN_TD> s[2];           // 0: d/dx, 1: d2/dx2
    XStencil st[2];
    XNCommon k;
    const double *in;             // the state the derivatives are taken of
    void *out1;                   // d/dx of every field (T)
    void *out2a, *out2b;          // d2/dx2 of u (fields d2a_lo..+2), of B (d2b_lo..+2), or null
    void *outE;                   // d/dx of Ey, Ez: planes 0, 1 (T)
    int nvar, d2a_lo, d2b_lo;
};

// x filter of every field: out = F_x(in), in FP64 in both precisions.
struct XFParams {
    XNTaps<XN_TF> s;
    XStencil st;
    XNCommon k;
    const double *in;
    double *out;
};

int xn_setup(Ctx *c);
void xn_free(Ctx *c);
// XF: x filter of every field of `in` into `out` (out != in)
int launch_xf(Ctx *c, const double *in, double *out);
// XD: x derivatives of `in` into the context's derivative arrays
int launch_xd(Ctx *c, const double *in);

}  // namespace mhd
