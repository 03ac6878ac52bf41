// The 1-body term of MB-pol water on the GPU: the Partridge-Schwenke surface
// that System::Get1B evaluates for every local water through
// e1b::get_1b_energy -> ps::pot_nasa (bblock/system.cpp:2269-2401,
// potential/1b/energy1b.cpp:39-58, potential/1b/ps.cpp:346-640).
//
// One thread per water: the two O-H vectors and the H-H vector, their
// lengths and the bend cosine; the Morse O-H terms and the exponential H-H
// term; powers up to 15 of the three polynomial variables; the 244-term
// polynomial sums and their derivatives (generated straight-line code,
// gen/ps1b.inc); the energy in cm^-1 converted to kcal/mol; the gradient on
// O, H1, H2 and the virial.  Products and sums are rounded one by one in
// the reference's operand order (no fused multiply-add), so the energy
// differs from the reference's only through exp's last bit.
#include <cuda_runtime.h>

#include "holder_common.cuh"
#include "gen/ps1b.inc"

struct OneBodyArgs {
    const double* xyz;     // site coordinates (3 per site), internal order
    const int* first;      // first site of each water to evaluate (local waters of the topology)
    long n;                // number of waters
    double* grad;          // site gradient (+=), or null for energy only
    double* out;           // [0] energy, [1..6] virial xx xy xz yy yz zz (+=)
};

namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// Energy (kcal/mol) of one water and, with grads, dE/d(O, H1, H2).
__device__ __forceinline__ double ps1b_water(const double (&o)[3], const double (&h1)[3], const double (&h2)[3],
                                             bool grads, double (&go)[3], double (&g1)[3], double (&g2)[3]) {
    double r1[3], r2[3], rhh[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r1[c] = sub(h1[c], o[c]);
        r2[c] = sub(h2[c], o[c]);
        rhh[c] = sub(h1[c], h2[c]);
    }
    const double d1 = sqrt(add(add(mul(r1[0], r1[0]), mul(r1[1], r1[1])), mul(r1[2], r1[2])));
    const double d2 = sqrt(add(add(mul(r2[0], r2[0]), mul(r2[1], r2[1])), mul(r2[2], r2[2])));
    const double dhh = sqrt(add(add(mul(rhh[0], rhh[0]), mul(rhh[1], rhh[1])), mul(rhh[2], rhh[2])));
    const double costh =
        add(add(mul(r1[0], r2[0]), mul(r1[1], r2[1])), mul(r1[2], r2[2])) / mul(d1, d2);

    const double exp1 = exp(mul(-PS1B_ALPHAOH, sub(d1, PS1B_ROH)));
    const double exp2 = exp(mul(-PS1B_ALPHAOH, sub(d2, PS1B_ROH)));
    const double va = mul(PS1B_DEOH, add(mul(exp1, sub(exp1, 2.0)), mul(exp2, sub(exp2, 2.0))));
    const double vb = mul(PS1B_PHH1, exp(mul(-PS1B_PHH2, dhh)));

    const double x1 = sub(d1, PS1B_REOH) / PS1B_REOH;
    const double x2 = sub(d2, PS1B_REOH) / PS1B_REOH;
    const double x3 = sub(costh, PS1B_COSTHE);
    double f0[16], f1[16], f2[16];
    f0[0] = f1[0] = f2[0] = 0.0;
    f0[1] = f1[1] = f2[1] = 1.0;
#pragma unroll
    for (int j = 2; j < 16; ++j) {
        f0[j] = mul(f0[j - 1], x1);
        f1[j] = mul(f1[j - 1], x2);
        f2[j] = mul(f2[j - 1], x3);
    }
    const double e1s = sub(d1, PS1B_REOH), e2s = sub(d2, PS1B_REOH);
    const double efac = exp(mul(-PS1B_B1, add(mul(e1s, e1s), mul(e2s, e2s))));
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    ps1b_sums(f0, f1, f2, s0, s1, s2, s3);
    const double vc = add(mul(2.0, PS1B_C0), mul(efac, s0));
    const double e = mul(add(add(add(va, vb), vc), PS1B_OFFSET), PS1B_CM1_KCALMOL);
    if (!grads) return e;

    const double dva1 = mul(mul(mul(mul(2.0, PS1B_ALPHAOH), PS1B_DEOH), exp1), sub(1.0, exp1)) / d1;
    const double dva2 = mul(mul(mul(mul(2.0, PS1B_ALPHAOH), PS1B_DEOH), exp2), sub(1.0, exp2)) / d2;
    const double dvb = mul(-PS1B_PHH2, vb) / dhh;
    const double dvc1 = add(mul(mul(mul(mul(-2.0, PS1B_B1), efac), e1s), s0), mul(efac, s1) / PS1B_REOH) / d1;
    const double dvc2 = add(mul(mul(mul(mul(-2.0, PS1B_B1), efac), e2s), s0), mul(efac, s2) / PS1B_REOH) / d2;
    const double dvcth = mul(efac, s3);
    const double d12 = mul(d1, d2), d11 = mul(d1, d1), d22 = mul(d2, d2);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double a1 = add(add(add(mul(dva1, r1[c]), mul(dvb, rhh[c])), mul(dvc1, r1[c])),
                              mul(dvcth, sub(r2[c] / d12, mul(costh, r1[c]) / d11)));
        const double a2 = add(add(sub(mul(dva2, r2[c]), mul(dvb, rhh[c])), mul(dvc2, r2[c])),
                              mul(dvcth, sub(r1[c] / d12, mul(costh, r2[c]) / d22)));
        g1[c] = mul(a1, PS1B_CM1_KCALMOL);
        g2[c] = mul(a2, PS1B_CM1_KCALMOL);
        go[c] = -add(g1[c], g2[c]);
    }
    return e;
}

__global__ void __launch_bounds__(128) k_ps1b(const OneBodyArgs A) {
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const bool grads = A.grad != nullptr;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < A.n; i += (long)gridDim.x * blockDim.x) {
        const long s = A.first[i];
        const double* p = A.xyz + 3 * s;
        double o[3], h1[3], h2[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            o[c] = p[c];
            h1[c] = p[3 + c];
            h2[c] = p[6 + c];
        }
        double go[3], g1[3], g2[3];
        acc[0] += ps1b_water(o, h1, h2, grads, go, g1, g2);
        if (!grads) continue;
        // virial -sum r (x) g over the three atoms (ps.cpp:606-620)
        const double* r[3] = {o, h1, h2};
        const double* g[3] = {go, g1, g2};
        const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            double v = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a) v = sub(v, mul(r[a][ia[k]], g[a][ib[k]]));
            acc[1 + k] += v;
        }
        double* q = A.grad + 3 * s;   // one thread per water: no other thread writes these sites
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            q[c] += go[c];
            q[3 + c] += g1[c];
            q[6 + c] += g2[c];
        }
    }
    block_reduce_add<7>(acc, A.out);
}

}  // namespace

int mbx_launch_ps1b(const OneBodyArgs& A, int sms, cudaStream_t s) {
    if (A.n <= 0) return 0;
    const long want = (A.n + 127) / 128;
    const int grid = (int)(want < (long)sms * 4 ? want : (long)sms * 4);
    k_ps1b<<<grid, 128, 0, s>>>(A);
    return (int)cudaGetLastError();
}
