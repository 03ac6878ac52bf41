// Device building blocks shared by every 2-body/3-body evaluator kernel.
//
// Each function restates one piece of the reference evaluators:
//   var_exp / dvar_exp    variable::v_exp0 + variable::grads
//                         (potential/2b/x2b-v9x.cpp:54-69, 96-103)
//   var_coul / dvar_coul  variable::v_coul (x2b-v9x.cpp:73-92)
//   lp_sites / lp_grads   monomer::setup / monomer::grads, the MB-pol
//                         lone-pair sites (x2b-v9x.cpp:119-160)
//   f_switch              cosine switching function (x2b-v9x.cpp:1349-1362)
//   close_image           GetCloseDimerImage (bblock/sys_tools.cpp:322-366),
//                         evaluated with explicitly rounded operations so it
//                         matches the reference's non-contracted x86 arithmetic
#pragma once
#include <cuda_runtime.h>
#include <math.h>

// Two FP32 lanes in one 64-bit register (low half: first value), operated on
// by the paired FP32 instructions of sm_100 (one instruction, two results).
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
    f2_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
    f2_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
    f2_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2_t f2_pack(float lo, float hi) {
    return (f2_t)__float_as_uint(lo) | ((f2_t)__float_as_uint(hi) << 32);
}
__device__ __forceinline__ float f2_lo(f2_t a) { return __uint_as_float((unsigned)a); }
__device__ __forceinline__ float f2_hi(f2_t a) { return __uint_as_float((unsigned)(a >> 32)); }

// A 32-bit shared-memory load the compiler may neither remove nor merge with
// another (the coset-form pieces re-read their column offsets at each use
// instead of holding 36 of them in registers).
__device__ __forceinline__ int lds_pinned(const int* p) {
    int v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"((unsigned)__cvta_generic_to_shared(p)));
    return v;
}

#define MBX_LP_GAMMA_IN (-9.721486914088159e-02)
#define MBX_LP_GAMMA_OUT (9.859272078406150e-02)

struct BoxParams {
    double box[9];
    double inv[9];
    int use_pbc;
};

__device__ __forceinline__ double dist3(const double (&p1)[3], const double (&p2)[3], double& d0, double& d1,
                                        double& d2) {
    d0 = p1[0] - p2[0];
    d1 = p1[1] - p2[1];
    d2 = p1[2] - p2[2];
    return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

// v = exp(k (d0 - r))
__device__ __forceinline__ double var_exp(const double (&p1)[3], const double (&p2)[3], double k, double d0) {
    double a, b, c;
    const double r = dist3(p1, p2, a, b, c);
    return exp(k * (d0 - r));
}

// v = exp(k (d0 - r)) / r
__device__ __forceinline__ double var_coul(const double (&p1)[3], const double (&p2)[3], double k, double d0) {
    double a, b, c;
    const double r = dist3(p1, p2, a, b, c);
    return exp(k * (d0 - r)) / r;
}

// Adds gv * dv/dp1 to sg1 and gv * dv/dp2 to sg2 (dv/dp2 = -dv/dp1).
__device__ __forceinline__ void dvar_exp(const double (&p1)[3], const double (&p2)[3], double k, double d0, double gv,
                                         double (&sg1)[3], double (&sg2)[3]) {
    double a, b, c;
    const double r = dist3(p1, p2, a, b, c);
    const double v = exp(k * (d0 - r));
    const double f = gv * (-k * v / r);
    sg1[0] += f * a; sg1[1] += f * b; sg1[2] += f * c;
    sg2[0] -= f * a; sg2[1] -= f * b; sg2[2] -= f * c;
}

__device__ __forceinline__ void dvar_coul(const double (&p1)[3], const double (&p2)[3], double k, double d0,
                                          double gv, double (&sg1)[3], double (&sg2)[3]) {
    double a, b, c;
    const double r = dist3(p1, p2, a, b, c);
    const double rinv = 1.0 / r;
    const double v = exp(k * (d0 - r)) * rinv;
    const double f = gv * (-(k + rinv) * v * rinv);
    sg1[0] += f * a; sg1[1] += f * b; sg1[2] += f * c;
    sg2[0] -= f * a; sg2[1] -= f * b; sg2[2] -= f * c;
}

// The variable together with its radial factor q, dv/d(p1 - p2) = q (p1 - p2),
// for the mixed path (pair_vars_kernel): 1 / r from one reciprocal square
// root instead of a square root and a division (1-2 ulp, far below what the
// FP32 shifted variables and the FP32-accurate gradient keep).
__device__ __forceinline__ double var_exp_q(const double (&p1)[3], const double (&p2)[3], double k, double d0,
                                           double& q) {
    const double a = p1[0] - p2[0], b = p1[1] - p2[1], c = p1[2] - p2[2];
    const double d2 = a * a + b * b + c * c;
    const double rinv = rsqrt(d2), r = d2 * rinv;
    const double v = exp(k * (d0 - r));
    q = -k * v * rinv;
    return v;
}

__device__ __forceinline__ double var_coul_q(const double (&p1)[3], const double (&p2)[3], double k, double d0,
                                            double& q) {
    const double a = p1[0] - p2[0], b = p1[1] - p2[1], c = p1[2] - p2[2];
    const double d2 = a * a + b * b + c * c;
    const double rinv = rsqrt(d2), r = d2 * rinv;
    const double v = exp(k * (d0 - r)) * rinv;
    q = -(k + rinv) * v * rinv;
    return v;
}

// Adds gv q (p1 - p2) to sg1 and subtracts it from sg2 (dvar_exp / dvar_coul
// with the radial factor q already known).
__device__ __forceinline__ void dvar_q(const double (&p1)[3], const double (&p2)[3], double gv, double q,
                                       double (&sg1)[3], double (&sg2)[3]) {
    const double a = p1[0] - p2[0], b = p1[1] - p2[1], c = p1[2] - p2[2];
    const double f = gv * q;
    sg1[0] += f * a; sg1[1] += f * b; sg1[2] += f * c;
    sg2[0] -= f * a; sg2[1] -= f * b; sg2[2] -= f * c;
}

// The two lone-pair sites of a water (O, H1, H2).
__device__ __forceinline__ void lp_sites(const double (&o)[3], const double (&h1)[3], const double (&h2)[3],
                                         double (&xp)[3], double (&xm)[3]) {
    const double a0 = h1[0] - o[0], a1 = h1[1] - o[1], a2 = h1[2] - o[2];
    const double b0 = h2[0] - o[0], b1 = h2[1] - o[1], b2 = h2[2] - o[2];
    const double v0 = a1 * b2 - a2 * b1, v1 = a2 * b0 - a0 * b2, v2 = a0 * b1 - a1 * b0;
    const double i0 = o[0] + 0.5 * MBX_LP_GAMMA_IN * (a0 + b0);
    const double i1 = o[1] + 0.5 * MBX_LP_GAMMA_IN * (a1 + b1);
    const double i2 = o[2] + 0.5 * MBX_LP_GAMMA_IN * (a2 + b2);
    xp[0] = i0 + MBX_LP_GAMMA_OUT * v0; xp[1] = i1 + MBX_LP_GAMMA_OUT * v1; xp[2] = i2 + MBX_LP_GAMMA_OUT * v2;
    xm[0] = i0 - MBX_LP_GAMMA_OUT * v0; xm[1] = i1 - MBX_LP_GAMMA_OUT * v1; xm[2] = i2 - MBX_LP_GAMMA_OUT * v2;
}

// Moves the lone-pair site gradients gp (X+) and gm (X-) onto O, H1, H2.
__device__ __forceinline__ void lp_grads(const double (&o)[3], const double (&h1)[3], const double (&h2)[3],
                                         const double (&gp)[3], const double (&gmn)[3], double (&go)[3],
                                         double (&gh1)[3], double (&gh2)[3]) {
    const double a0 = h1[0] - o[0], a1 = h1[1] - o[1], a2 = h1[2] - o[2];
    const double b0 = h2[0] - o[0], b1 = h2[1] - o[1], b2 = h2[2] - o[2];
    const double m0 = gp[0] - gmn[0], m1 = gp[1] - gmn[1], m2 = gp[2] - gmn[2];
    const double t1[3] = {b1 * m2 - b2 * m1, b2 * m0 - b0 * m2, b0 * m1 - b1 * m0};
    const double t2[3] = {a1 * m2 - a2 * m1, a2 * m0 - a0 * m2, a0 * m1 - a1 * m0};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double gsum = gp[i] + gmn[i];
        const double in_plane = 0.5 * MBX_LP_GAMMA_IN * gsum;
        const double g1 = in_plane + MBX_LP_GAMMA_OUT * t1[i];
        const double g2 = in_plane - MBX_LP_GAMMA_OUT * t2[i];
        go[i] += gsum - (g1 + g2);
        gh1[i] += g1;
        gh2[i] += g2;
    }
}

__device__ __forceinline__ double f_switch(double r, double ri, double rf, double& g) {
    if (r > rf) {
        g = 0.0;
        return 0.0;
    } else if (r > ri) {
        const double t1 = M_PI / (rf - ri);
        const double x = (r - ri) * t1;
        double s, c;
        sincos(x, &s, &c);
        g = -s * t1 / 2.0;
        return (1.0 + c) / 2.0;
    }
    g = 0.0;
    return 1.0;
}

// Fractional / Cartesian conversions with every product and sum rounded on
// its own (no FMA contraction), in the reference's operand order.
__device__ __forceinline__ void to_frac_rn(const double* inv, const double (&p)[3], double (&f)[3]) {
    f[0] = __dadd_rn(__dadd_rn(__dmul_rn(inv[0], p[0]), __dmul_rn(inv[3], p[1])), __dmul_rn(inv[6], p[2]));
    f[1] = __dadd_rn(__dadd_rn(__dmul_rn(inv[1], p[0]), __dmul_rn(inv[4], p[1])), __dmul_rn(inv[7], p[2]));
    f[2] = __dadd_rn(__dadd_rn(__dmul_rn(inv[2], p[0]), __dmul_rn(inv[5], p[1])), __dmul_rn(inv[8], p[2]));
}

__device__ __forceinline__ void to_cart_rn(const double* b, const double (&f)[3], double (&p)[3]) {
    p[0] = __dadd_rn(__dadd_rn(__dmul_rn(b[0], f[0]), __dmul_rn(b[3], f[1])), __dmul_rn(b[6], f[2]));
    p[1] = __dadd_rn(__dadd_rn(__dmul_rn(b[1], f[0]), __dmul_rn(b[4], f[1])), __dmul_rn(b[7], f[2]));
    p[2] = __dadd_rn(__dadd_rn(__dmul_rn(b[2], f[0]), __dmul_rn(b[5], f[1])), __dmul_rn(b[8], f[2]));
}

// Integer lattice shift that brings a monomer whose first atom is at q0 next
// to the monomer whose first atom is at p0 (GetCloseDimerImage).
__device__ __forceinline__ void image_shift(const BoxParams& bp, const double (&p0)[3], const double (&q0)[3],
                                            double (&d)[3]) {
    double f1[3], f2[3];
    to_frac_rn(bp.inv, p0, f1);
    to_frac_rn(bp.inv, q0, f2);
    d[0] = floor(__dadd_rn(__dsub_rn(f2[0], f1[0]), 0.5));
    d[1] = floor(__dadd_rn(__dsub_rn(f2[1], f1[1]), 0.5));
    d[2] = floor(__dadd_rn(__dsub_rn(f2[2], f1[2]), 0.5));
}

// Applies a shift from image_shift to one atom (in place).
__device__ __forceinline__ void apply_shift(const BoxParams& bp, const double (&d)[3], double (&q)[3]) {
    double f[3];
    to_frac_rn(bp.inv, q, f);
    f[0] = __dsub_rn(f[0], d[0]);
    f[1] = __dsub_rn(f[1], d[1]);
    f[2] = __dsub_rn(f[2], d[2]);
    to_cart_rn(bp.box, f, q);
}

// Warp + block reduction of NV doubles into out[] with one atomic per block.
template <int NV>
__device__ __forceinline__ void block_reduce_add(double (&v)[NV], double* out) {
    __shared__ double red[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        double x = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        v[i] = x;
    }
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) red[warp][i] = v[i];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double x = lane < nw ? red[lane][i] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0 && x != 0.0) atomicAdd(out + i, x);
        }
    }
}
