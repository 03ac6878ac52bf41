// Term tables of the permutationally invariant polynomials, evaluated from
// data instead of straight-line code.
//
// A polynomial of the reference's generated-polynomial convention is linear
// in its fitted coefficients a (poly_2b_v6x::eval(nd, a, x),
// potential/2b/poly-2b-v6x.h:78; poly_3b_v2x::eval(a, x), poly-3b-v2x.h:73;
// the MB-nrg eval(a, x) / eval(x, a) programs).  Expanded, it is
//     P(a, x) = sum_t a[k_t] * c_t * prod_i x[v_t,i]^e_t,i
// over its terms t.  A table holds one int4 per term plus its multiplicity
// c_t (a double):
//     x: k_t (index of the fitted coefficient; the table is sorted by k)
//     y, z, w: six (variable, exponent) byte pairs, low byte the variable
//              (255: unused), high byte the exponent, in the order the
//              variables appear in the term
// Six pairs cover every table of the library (at most six distinct
// variables per term; a single variable may carry an exponent up to 23).
//
// Three uses share the decoding below: the warp-per-n-mer evaluation of the
// evaluators without straight-line code (holder_table_kernel), the adjoint
// with respect to the coefficients (holder_dcoef_table_kernel) and the
// generated-polynomial entry point over caller-supplied variables
// (poly_table_kernel).
#pragma once
#include <cuda_runtime.h>

#define MBX_TERM_PAIRS 6

__device__ __forceinline__ void term_pair(const int4& tm, int i, int& v, int& e) {
    const int word = i < 2 ? tm.y : (i < 4 ? tm.z : tm.w);
    const int p = (word >> (16 * (i & 1))) & 0xffff;
    v = p & 255;
    e = p >> 8;
}

// c * prod_i x[v_i]^e_i, multiplied left to right in the order of the table.
template <int NP, class X>
__device__ __forceinline__ double term_value(const int4& tm, double c, const X& x) {
    double m = c;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        int v, e;
        term_pair(tm, i, v, e);
        if (v != 255) {
            const double xv = x(v);
#pragma unroll 1
            for (int j = 0; j < e; ++j) m *= xv;
        }
    }
    return m;
}

// c * prod x^e, and for every pair i of the term the derivative
// dm/dx[v_i] = c * e_i x[v_i]^(e_i - 1) * prod_{j != i} x[v_j]^e_j handed to
// sink(v_i, value).  Returns the term's value.
template <int NP, class X, class Sink>
__device__ __forceinline__ double term_value_grad(const int4& tm, double c, const X& x, Sink&& sink) {
    int v[NP];
    double p[NP], d[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        int e;
        term_pair(tm, i, v[i], e);
        p[i] = 1.0;
        d[i] = 0.0;
        if (v[i] != 255) {
            const double xv = x(v[i]);
            double pw = 1.0;
#pragma unroll 1
            for (int j = 1; j < e; ++j) pw *= xv;
            d[i] = (double)e * pw;
            p[i] = pw * xv;
        }
    }
    double pre[NP];
    double acc = c;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        pre[i] = acc;
        acc *= p[i];
    }
    double suf = 1.0;
#pragma unroll
    for (int i = NP - 1; i >= 0; --i) {
        if (v[i] != 255) sink(v[i], pre[i] * d[i] * suf);
        suf *= p[i];
    }
    return acc;
}
