// The generated-polynomial calling convention over a term table: energies and
// gradients of a polynomial at caller-supplied variables.
//
// This is the convention of the reference's generated programs
// (poly_2b_v6x::eval(nd, a, x, t, g), potential/2b/poly-2b-v6x.h:95, with
// x[v * nd + i]; the per-configuration MB-nrg eval(a, x, g) programs are the
// nd = 1 case), served for every evaluator from the term tables the
// table-driven kernels use (term_table.cuh) and the coefficients currently set
// on the device.  A warp per configuration: lane l takes terms l, l+32, ...;
// the configuration's variables and gradient accumulators sit in shared
// memory (gradient by shared-memory atomics), the energy is reduced across
// the warp.
#include <cuda_runtime.h>

#include "term_table.cuh"

#define MBX_POLY_WARPS 4
#define MBX_POLY_MAXV 128

template <int NP>
__global__ void __launch_bounds__(MBX_POLY_WARPS * 32)
    poly_table_kernel(long nd, int nvars, const double* __restrict__ x_soa, double* __restrict__ g_soa,
                      double* __restrict__ e, const int4* __restrict__ terms, const double* __restrict__ tcoef,
                      long nterms, const double* __restrict__ coef) {
    __shared__ double xs[MBX_POLY_WARPS][MBX_POLY_MAXV];
    __shared__ double gs[MBX_POLY_WARPS][MBX_POLY_MAXV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long stride = (long)gridDim.x * MBX_POLY_WARPS;
    for (long i = blockIdx.x * (long)MBX_POLY_WARPS + w; i < nd; i += stride) {
        for (int v = lane; v < nvars; v += 32) {
            xs[w][v] = x_soa[(long)v * nd + i];
            gs[w][v] = 0.0;
        }
        __syncwarp();
        const auto xv = [&](int v) { return xs[w][v]; };
        double en = 0.0;
        for (long q = lane; q < nterms; q += 32) {
            const int4 tm = __ldg(terms + q);
            const double c = __ldg(coef + tm.x) * __ldg(tcoef + q);
            if (g_soa)
                en += term_value_grad<NP>(tm, c, xv, [&](int v, double dv) { atomicAdd(&gs[w][v], dv); });
            else
                en += term_value<NP>(tm, c, xv);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) en += __shfl_xor_sync(0xffffffffu, en, o);
        __syncwarp();
        if (lane == 0) e[i] = en;
        if (g_soa)
            for (int v = lane; v < nvars; v += 32) g_soa[(long)v * nd + i] = gs[w][v];
        __syncwarp();
    }
}

// pairs: (variable, exponent) pairs per term of this table, at most.
int mbx_launch_poly_table(long nd, int nvars, const double* x, double* g, double* e, const int4* terms,
                          const double* tcoef, long nterms, const double* coef, int pairs, int sms, cudaStream_t s) {
    if (nvars < 1 || nvars > MBX_POLY_MAXV || pairs < 1 || pairs > MBX_TERM_PAIRS) return (int)cudaErrorInvalidValue;
    const long want = (nd + MBX_POLY_WARPS - 1) / MBX_POLY_WARPS;
    const int grid = (int)(want < (long)sms * 8 ? (want > 0 ? want : 1) : (long)sms * 8);
    if (pairs <= 4)
        poly_table_kernel<4><<<grid, MBX_POLY_WARPS * 32, 0, s>>>(nd, nvars, x, g, e, terms, tcoef, nterms, coef);
    else
        poly_table_kernel<MBX_TERM_PAIRS><<<grid, MBX_POLY_WARPS * 32, 0, s>>>(nd, nvars, x, g, e, terms, tcoef,
                                                                                nterms, coef);
    return (int)cudaGetLastError();
}
