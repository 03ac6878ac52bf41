// Evaluation kernels for the 2-body/3-body evaluators (one template for all
// types; the per-type pieces come from the generated traits T in gen/*.cuh).
//
// One n-mer per thread for the straight-line polynomials: the n-mer's atoms
// are gathered, moved to the image next to the n-mer's first monomer
// (GetCloseDimerImage / GetCloseTrimerImage), the polynomial variables are
// built in FP64, the polynomial and its gradient run out of registers (the
// generated Horner trie), then the switch, the chain rule to atoms (including
// the lone-pair redistribution), the virial and the gradient scatter follow.
// This is the work of x2b_v9x::eval / x3b_v2x::eval / the MB-nrg evaluators
// (potential/2b/x2b-v9x.cpp:1514-1819, potential/3b/x3b-v2x.cpp:1403-1808,
// x2b_A1B2Z2_C1D4_deg3_exp0_v1x.cpp:954, x2b_A1B4_A1B4_deg4_exp0_v1x.cpp:1600,
// mbnrg_3b_A1B4_C1D2_C1D2_deg3_v1.cpp:1481) fused with the gather, image and
// scatter steps of System::Get2B/Get3B (bblock/system.cpp:2425-2725,
// 2769-3073).
//
// The evaluators without straight-line code (the CH4-CH4 polynomial with its
// 201k terms and the widened MB-nrg types) are evaluated by a warp per n-mer
// that walks the polynomial's term table (holder_table_kernel below).
#pragma once
#include "holder_common.cuh"
#include "term_table.cuh"

// Precision / output modes.
// HM_GRAD_SHIFT32 names the paired FP32 kernels (pair_*_kernel) where a
// template needs to tell the two gradient kernels apart.
enum { HM_ENERGY = 0, HM_GRAD_FP64 = 1, HM_GRAD_SHIFT32 = 4 };

// Scratch of the mixed-precision evaluation (three kernels: variables, the
// paired FP32 trie, chain rule), for up to cap n-mers: the shifted FP32
// variables and the trie's gradient, variable-major ([v * cap + t]), the
// polynomial's value and whether the n-mer is within the evaluator's cutoff.
struct PairScratch {
    float* dx;
    double* q;    // radial factor of each variable (var_exp_q), for the chain rule of pair_finish_kernel
    float* g;
    double* ep;
    unsigned char* live;
    long cap;
    int* err;   // status word: kernels that wait on barriers report a timeout here (bit 8)
};

struct HolderArgs {
    long n;                    // number of n-mers (capacity when n_dev is set)
    const int* n_dev;          // optional device-side count (read by the kernel, clamped to n)
    const int* status;         // optional: a nonzero word means the n-mer build failed; do nothing
    int* counter;              // work counter (zeroed before the launch): warps claim chunks of 32 n-mers
    const int4* nmers;         // system input: (m0, m1, m2, anchor slot), holder order
    const double* xyz;         // system input: site array (3 per site); AoS input: [n][NREAL*3]
    const int* first_index;    // system input: first site of every monomer
    BoxParams bp;
    double* grad;              // system: site-array gradient (+=); AoS: [n][NREAL*3] (+=)
    double* out;               // [0] energy, [1..6] virial xx xy xz yy yz zz (+=)
    double* e_per;             // optional: switched energy of every n-mer
    const double* coef;        // custom linear coefficients (global) or null
    int aos;                   // 1: AoS per-n-mer input (already imaged, no gather)
    // batched configurations (system input): per-configuration boxes and
    // energy + virial sums (8 doubles each), the configuration of every monomer
    const BoxParams* conf_bp;  // null: one configuration in bp
    const int* mon_conf;
    double* conf_out;
    // term table of the polynomial (term_table.cuh), for the table-driven kernels
    const int4* terms;         // (k, six (variable, exponent) byte pairs)
    const double* tcoef;       // term multiplicities
    long nterms;
    // code prefetch launch of a lockstep kernel (prime_passes > 0; see
    // prime_pieces): of the rest only out (null) is read
    int prime_passes, prime_npieces;
    PairScratch ps;            // mixed precision: scratch of the three kernels
};

// Coefficient source: a global pointer, read through the read-only path.
struct GlobalCoef {
    const double* __restrict__ p;
    __device__ __forceinline__ double operator[](int k) const { return __ldg(p + k); }
    __device__ __forceinline__ float f(int k) const { return (float)__ldg(p + k); }
};

__device__ __forceinline__ double ld_volatile(const double* p) {
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

// Real atoms of the evaluator's largest monomer (loop bound over one monomer's atoms).
template <class T>
__host__ __device__ constexpr int max_nat() {
    return T::NAT0 > T::NAT1 ? (T::NAT0 > T::NAT2 ? T::NAT0 : T::NAT2) : (T::NAT1 > T::NAT2 ? T::NAT1 : T::NAT2);
}

// GetCloseDimerImage / GetCloseTrimerImage: every monomer but the anchor slot
// moved to the image next to the anchor's first atom.
template <class T>
__device__ __forceinline__ void image_nmer(const BoxParams& bp, int anchor, double (&r)[T::NREAL][3]) {
    const int nat[3] = {T::NAT0, T::NAT1, T::NAT2};
    const int first[3] = {T::FIRST0, T::FIRST1, T::FIRST2};
    {
        double p0[3];
#pragma unroll
        for (int s = 0; s < T::NBODY; ++s)
            if (s == anchor) { p0[0] = r[first[s]][0]; p0[1] = r[first[s]][1]; p0[2] = r[first[s]][2]; }
#pragma unroll
        for (int s = 0; s < T::NBODY; ++s) {
            if (s == anchor) continue;
            double q0[3] = {r[first[s]][0], r[first[s]][1], r[first[s]][2]};
            double d[3];
            image_shift(bp, p0, q0, d);
#pragma unroll
            for (int a = 0; a < max_nat<T>(); ++a) {
                if (a < nat[s]) {
                    double q[3] = {r[first[s] + a][0], r[first[s] + a][1], r[first[s] + a][2]};
                    apply_shift(bp, d, q);
                    r[first[s] + a][0] = q[0];
                    r[first[s] + a][1] = q[1];
                    r[first[s] + a][2] = q[2];
                }
            }
        }
    }
}

template <class T, bool VOL>
__device__ __forceinline__ void load_nmer(const HolderArgs& A, long t, double (&r)[T::NREAL][3]) {
    constexpr int MAXNAT = max_nat<T>();
    if (A.aos) {
        const double* p = A.xyz + (size_t)t * (T::NREAL * 3);
#pragma unroll
        for (int i = 0; i < T::NREAL; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) r[i][c] = VOL ? ld_volatile(p + 3 * i + c) : __ldg(p + 3 * i + c);
        return;
    }
    const int4 nm = __ldg(A.nmers + t);
    const int mon[3] = {nm.x, nm.y, nm.z};
    const int nat[3] = {T::NAT0, T::NAT1, T::NAT2};
    const int first[3] = {T::FIRST0, T::FIRST1, T::FIRST2};
#pragma unroll
    for (int s = 0; s < T::NBODY; ++s) {
        const double* p = A.xyz + 3 * (size_t)__ldg(A.first_index + mon[s]);
#pragma unroll
        for (int a = 0; a < 3 * MAXNAT; ++a) {
            if (a < 3 * nat[s]) r[first[s] + a / 3][a % 3] = VOL ? ld_volatile(p + a) : __ldg(p + a);
        }
    }
    if (A.conf_bp) {
        const BoxParams& bp = A.conf_bp[__ldg(A.mon_conf + nm.x)];
        if (bp.use_pbc) image_nmer<T>(bp, nm.w, r);
    } else if (A.bp.use_pbc) {
        image_nmer<T>(A.bp, nm.w, r);
    }
}

// First-atom distances (pairs 01, 02, 12) and the skip rule of the type.
template <class T>
__device__ __forceinline__ bool pair_dists(const double (&r)[T::NREAL][3], double (&d)[3][3], double (&rr)[3]) {
    const int first[3] = {T::FIRST0, T::FIRST1, T::FIRST2};
    const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
    constexpr int NP = T::NBODY == 2 ? 1 : 3;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        const int i = first[pa[p]], j = first[pb[p]];
        d[p][0] = r[i][0] - r[j][0];
        d[p][1] = r[i][1] - r[j][1];
        d[p][2] = r[i][2] - r[j][2];
        rr[p] = sqrt(d[p][0] * d[p][0] + d[p][1] * d[p][1] + d[p][2] * d[p][2]);
    }
    const double rf = T::RF;
    if (T::SKIP == 0) return rr[0] > rf;
    if (T::SKIP == 1)
        return (rr[0] > rf && rr[1] > rf) || (rr[0] > rf && rr[2] > rf) || (rr[1] > rf && rr[2] > rf);
    return rr[0] > rf && rr[1] > rf && rr[2] > rf;
}

// Switch value and the gradient of the switch with respect to first atoms,
// scaled by the unswitched energy ep, added into tg.
template <class T>
__device__ __forceinline__ double apply_switch(const double (&d)[3][3], const double (&rr)[3], double ep,
                                               double (&tg)[T::NREAL][3], bool grads) {
    const int first[3] = {T::FIRST0, T::FIRST1, T::FIRST2};
    if (!T::SWITCH_TRIPLE) {
        double gs;
        const double sw = f_switch(rr[0], T::RI, T::RF, gs);
        if (grads) {
            const double f = gs * ep / rr[0];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                tg[first[0]][c] += f * d[0][c];
                tg[first[1]][c] -= f * d[0][c];
            }
        }
        return sw;
    }
    // SWITCH_TRIPLE 1: s0 s1 + s0 s2 + s1 s2; 2: the same minus 2 s0 s1 s2;
    // 3: 1 - cos^2((S - 1) pi / 2) on S = s0 + s1 + s2, 0 below S = 1 and 1
    // above S = 2 (mbnrg_3b_A1B2C4_D1E2_D1E2_deg3_v1.cpp:2464-2471, gradient
    // -(pi / 2) sin(pi S) strictly inside (1, 2), :2563-2570)
    double g0, g1, g2;
    const double s0 = f_switch(rr[0], T::RI, T::RF, g0);
    const double s1 = f_switch(rr[1], T::RI, T::RF, g1);
    const double s2 = f_switch(rr[2], T::RI, T::RF, g2);
    if (T::SWITCH_TRIPLE == 3) {
        const double S = s0 + s1 + s2;
        if (grads && S > 1.0 && S < 2.0) {
            const double dS = -(M_PI / 2.0) * sin(M_PI * S) * ep;
            const double f0 = g0 * dS / rr[0], f1 = g1 * dS / rr[1], f2 = g2 * dS / rr[2];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                tg[first[0]][c] += f0 * d[0][c] + f1 * d[1][c];
                tg[first[1]][c] += f2 * d[2][c] - f0 * d[0][c];
                tg[first[2]][c] -= f1 * d[1][c] + f2 * d[2][c];
            }
        }
        if (S < 1.0) return 0.0;
        if (S > 2.0) return 1.0;
        const double cs = cos((S - 1.0) * M_PI / 2.0);
        return 1.0 - cs * cs;
    }
    const double c = T::SWITCH_TRIPLE == 2 ? 2.0 : 0.0;
    if (grads) {
        const double f0 = g0 * (s1 + s2 - c * s1 * s2) * ep / rr[0];
        const double f1 = g1 * (s0 + s2 - c * s0 * s2) * ep / rr[1];
        const double f2 = g2 * (s0 + s1 - c * s0 * s1) * ep / rr[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            tg[first[0]][c] += f0 * d[0][c] + f1 * d[1][c];
            tg[first[1]][c] += f2 * d[2][c] - f0 * d[0][c];
            tg[first[2]][c] -= f1 * d[1][c] + f2 * d[2][c];
        }
    }
    return s0 * s1 + s0 * s2 + s1 * s2 - c * s0 * s1 * s2;
}

// Adds v[0..7) into dst[0..7) (one configuration's energy and virial), one
// atomic per value for all lanes of the warp that are here with the same dst.
__device__ __forceinline__ void conf_accumulate(double* dst, const double (&v)[7]) {
    const int lane = threadIdx.x & 31;
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, (unsigned long long)dst);
    const int leader = __ffs(peers) - 1;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        double sum = 0.0;
        for (unsigned m = peers; m; m &= m - 1) sum += __shfl_sync(peers, v[i], __ffs(m) - 1);
        if (lane == leader && sum != 0.0) atomicAdd(dst + i, sum);
    }
}

// The chain rule from dP/dv: g is an array of T::NVARS doubles, or a reader
// indexed the same way; PairFactors (below) also brings the variables'
// radial factors, so that nothing is recomputed.
template <class T, class G>
__device__ __forceinline__ void chain_rule(const double (&s)[T::NSITES][3], const G& g, double (&sg)[T::NSITES][3]) {
    T::chain(s, g, sg);
}

// dP/dv (FP32) and the radial factors (FP64) of n-mer t in the mixed path's
// scratch, read where the chain rule uses them
struct PairGrad {
    const float* __restrict__ g;
    long cap, t;
    __device__ __forceinline__ double operator[](int v) const { return (double)__ldg(g + v * cap + t); }
};
struct PairQ {
    const double* __restrict__ q;
    long cap, t;
    __device__ __forceinline__ double operator[](int v) const { return __ldcs(q + v * cap + t); }
};
struct PairFactors {
    PairGrad g;
    PairQ q;
};
template <class T>
__device__ __forceinline__ void chain_rule(const double (&s)[T::NSITES][3], const PairFactors& f,
                                           double (&sg)[T::NSITES][3]) {
    T::chain_q(s, f.g, f.q, sg);
}

// Everything after the polynomial: chain rule, switch, virial, scatter.  g:
// dP/dv as chain_rule takes it.
template <class T, class G>
__device__ __forceinline__ void finish_nmer(const HolderArgs& A, long t, double ep, const G& g, bool grads,
                                            double (&acc)[7]) {
    double r[T::NREAL][3];
    load_nmer<T, true>(A, t, r);
    double d[3][3], rr[3];
    pair_dists<T>(r, d, rr);
    double tg[T::NREAL][3];
    if (grads) {
        double s[T::NSITES][3], sg[T::NSITES][3];
        T::sites(r, s);
        chain_rule<T>(s, g, sg);
#pragma unroll
        for (int i = 0; i < T::NREAL; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) tg[i][c] = sg[i][c];
    }
    const double sw = apply_switch<T>(d, rr, ep, tg, false);
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    auto virial = [&]() {
#pragma unroll
        for (int i = 0; i < T::NREAL; ++i) {
            v[1] -= r[i][0] * tg[i][0];
            v[2] -= r[i][0] * tg[i][1];
            v[3] -= r[i][0] * tg[i][2];
            v[4] -= r[i][1] * tg[i][1];
            v[5] -= r[i][1] * tg[i][2];
            v[6] -= r[i][2] * tg[i][2];
        }
    };
    if (grads) {
        // VIRIAL_RAW: the evaluator's virial is that of the polynomial
        // gradient alone, before the switch (x2b_A1B2C4_D1E2_deg3_v1x.cpp:1353-1391)
        if (T::VIRIAL_RAW) virial();
#pragma unroll
        for (int i = 0; i < T::NREAL; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) tg[i][c] *= sw;
        apply_switch<T>(d, rr, ep, tg, true);
        if (!T::VIRIAL_RAW) virial();
    }
    const double es = sw * ep;
    if (A.e_per) A.e_per[t] = es;
    v[0] = es;
    if (A.conf_out) {
        conf_accumulate(A.conf_out + 8 * __ldg(A.mon_conf + __ldg(A.nmers + t).x), v);
    } else {
#pragma unroll
        for (int i = 0; i < 7; ++i) acc[i] += v[i];
    }
    if (!grads) return;
    if (A.aos) {
        double* p = A.grad + (size_t)t * (T::NREAL * 3);
#pragma unroll
        for (int i = 0; i < T::NREAL; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) p[3 * i + c] += tg[i][c];
        return;
    }
    const int4 nm = __ldg(A.nmers + t);
    const int mon[3] = {nm.x, nm.y, nm.z};
    const int nat[3] = {T::NAT0, T::NAT1, T::NAT2};
    const int first[3] = {T::FIRST0, T::FIRST1, T::FIRST2};
#pragma unroll
    for (int s = 0; s < T::NBODY; ++s) {
        double* p = A.grad + 3 * (size_t)__ldg(A.first_index + mon[s]);
#pragma unroll
        for (int a = 0; a < max_nat<T>(); ++a)
            if (a < nat[s])
#pragma unroll
                for (int c = 0; c < 3; ++c) atomicAdd(p + 3 * a + c, tg[first[s] + a][c]);
    }
}

// Number of n-mers to evaluate (0 when the n-mer build reported a failure).
__device__ __forceinline__ long nmer_count(const HolderArgs& A) {
    if (A.status && *A.status) return 0;
    if (!A.n_dev) return A.n;
    const long c = *A.n_dev;
    return c < A.n ? c : A.n;
}

// The polynomial (and its gradient) in the precision mode of the kernel, with
// a block barrier after every separately compiled piece of the trie; x and
// the gradient accumulators in shared memory, [v][thread], at the thread's
// column (xs, gs).
template <class T, int MODE, class C>
__device__ __forceinline__ double run_pip_lock(const C& coef, const double* xs, double* gs) {
    if constexpr (MODE == HM_ENERGY) {
        return T::template pip_e_lock<T::LOCK_THREADS>(coef, xs);
    } else {
        static_assert(MODE == HM_GRAD_FP64, "unknown mode");
        return T::template pip_lock<T::LOCK_THREADS>(coef, xs, gs);
    }
}

// Dynamic shared memory of the lockstep kernels (their x/g columns).
extern __shared__ __align__(16) unsigned char mbx_dyn_smem[];

// FP64 coefficients copied from constant to shared memory once per block
// (types with T::SMEM_COEF).
template <class CC>
struct SharedCoef {
    const double* p;
    __device__ __forceinline__ double operator[](int k) const { return p[k]; }
};

// Code prefetch mode of the lockstep kernels.  Their trie is ~10^5
// instructions of straight-line code.  Once other work has evicted it from
// L2 (the rest of an MD step between two force calls), the first pass of
// each SM through it waits on DRAM for every instruction fetch: ~0.4 ms of a
// 1.3 ms FP64 evaluation of the 2048-water trimers, ~0.5 ms of the 0.8 ms
// paired FP32 one.  An SM only gains from code that SMs of its own half of
// the chip have fetched (one block through the whole trie beforehand
// recovers half; a block on every SM, all of it).  A prefetch launch of the
// same kernel (ptxas compiles a __noinline__ piece separately for every
// kernel that calls it, so only the kernel's own launch fetches the code the
// evaluation runs) has one warp per block run piece (block + j * grid) mod
// npieces in pass j: every piece fetched by several SMs spread over the chip,
// all pieces at once.  It is launched beside the n-mer search, ahead of the
// evaluation.  The lanes' x and g columns share one [v][L] array (x at
// columns 0-31, g at 32-63) of zeros; the results are discarded.
template <int L, class V, class Piece>
__device__ __forceinline__ void prime_pieces(const HolderArgs& A, int nvars, Piece&& piece) {
    static_assert(L >= 64, "x and g columns of the prefetch overlap");
    V* xs = reinterpret_cast<V*>(mbx_dyn_smem) + threadIdx.x;
    V* gs = xs + 32;
#pragma unroll 1
    for (int v = 0; v < nvars; ++v) {
        xs[v * L] = V(0);
        gs[v * L] = V(0);
    }
    __syncwarp();
    double sum = 0.0;
#pragma unroll 1
    for (int j = 0; j < A.prime_passes; ++j) {
        const int k = (int)(((long)blockIdx.x + (long)j * gridDim.x) % A.prime_npieces);
        sum += piece(k, xs, gs);
        __syncwarp();
    }
    if (A.out) A.out[threadIdx.x] = sum;   // null in a prefetch launch; keeps the calls
}

// One n-mer per thread, all warps of a block in lockstep through the trie:
// the straight-line polynomial is ~10^5 instructions, far more than the
// instruction cache holds, so the block's warps go through it piece by piece
// together (a barrier after each piece) and one fetch of a piece's code serves
// all of them.  Threads without an n-mer (past the end, or beyond the
// evaluator's cutoff) run the pieces on zero variables and discard the result.
// Persistent grid; a block claims chunks of blockDim.x n-mers from
// A.counter (or strides statically without it).
template <class T, class CC, int MODE, bool CUSTOM>
__global__ void __launch_bounds__(T::LOCK_THREADS, 1) holder_lock_kernel(const HolderArgs A) {
    constexpr bool grads = (MODE == HM_GRAD_FP64);
    constexpr int L = T::LOCK_THREADS;   // == blockDim.x
    double* xs = reinterpret_cast<double*>(mbx_dyn_smem) + threadIdx.x;
    double* gs = xs + T::NVARS * L;      // used in gradient mode only
    __shared__ long s_base;
    __shared__ double s_coef[T::SMEM_COEF ? T::NCOEF : 1];
    if constexpr (T::SMEM_COEF && !CUSTOM) {
        for (int k = threadIdx.x; k < T::NCOEF; k += blockDim.x) s_coef[k] = CC{}[k];
        __syncthreads();
    }
    if constexpr (!CUSTOM) {
        if (A.prime_passes > 0) {
            prime_pieces<L, double>(A, T::NVARS, [&](int k, const double* x, double* g) -> double {
                if constexpr (MODE == HM_ENERGY) {
                    if constexpr (T::SMEM_COEF) return T::template pip_e_piece<L>(k, SharedCoef<CC>{s_coef}, x);
                    else return T::template pip_e_piece<L>(k, CC{}, x);
                } else {
                    if constexpr (T::SMEM_COEF) return T::template pip_piece<L>(k, SharedCoef<CC>{s_coef}, x, g);
                    else return T::template pip_piece<L>(k, CC{}, x, g);
                }
            });
            return;
        }
    }
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const long n = nmer_count(A);
    long static_next = blockIdx.x * (long)blockDim.x;
    for (;;) {
        long base;
        if (A.counter) {
            if (threadIdx.x == 0) s_base = atomicAdd(A.counter, (int)blockDim.x);
            __syncthreads();
            base = s_base;
            __syncthreads();
        } else {
            base = static_next;
            static_next += (long)gridDim.x * blockDim.x;
        }
        if (base >= n) break;
        const long t = base + threadIdx.x;
        bool live = t < n;
        {
            double x[T::NVARS];
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) x[v] = 0.0;
            if (live) {
                double r[T::NREAL][3];
                load_nmer<T, false>(A, t, r);
                double d[3][3], rr[3];
                if (pair_dists<T>(r, d, rr)) {
                    if (A.e_per) A.e_per[t] = 0.0;
                    live = false;
                } else {
                    double s[T::NSITES][3];
                    T::sites(r, s);
                    T::vars(s, x);
                }
            }
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) {
                xs[v * L] = x[v];
                if (grads) gs[v * L] = 0.0;
            }
        }
        double ep;
        if constexpr (CUSTOM) ep = run_pip_lock<T, MODE>(GlobalCoef{A.coef}, xs, gs);
        else if constexpr (T::SMEM_COEF) ep = run_pip_lock<T, MODE>(SharedCoef<CC>{s_coef}, xs, gs);
        else ep = run_pip_lock<T, MODE>(CC{}, xs, gs);
        if (live) {
            double g[T::NVARS];
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) g[v] = grads ? gs[v * L] : 0.0;
            finish_nmer<T>(A, t, ep, g, grads, acc);
        }
    }
    block_reduce_add<7>(acc, A.out);
}

// Variables of n-mer t shifted to the type's FP32 basis, dx = x - x0 rounded
// to FP32 (x itself is built in FP64).  Returns false, with x = 0, for t >= n
// or an n-mer beyond the evaluator's cutoff.
template <class T>
__device__ __forceinline__ bool nmer_vars_f32(const HolderArgs& A, long t, long n, float (&xf)[T::NVARS],
                                              double* q = nullptr) {
    double x[T::NVARS];
#pragma unroll
    for (int v = 0; v < T::NVARS; ++v) x[v] = 0.0;
    bool live = t < n;
    if (live) {
        double r[T::NREAL][3];
        load_nmer<T, false>(A, t, r);
        double d[3][3], rr[3];
        if (pair_dists<T>(r, d, rr)) {
            if (A.e_per) A.e_per[t] = 0.0;
            live = false;
        } else {
            double s[T::NSITES][3];
            T::sites(r, s);
            if (q) {
                // with the radial factors, stored for pair_finish_kernel as
                // they are computed (streaming stores: read once, by that
                // kernel, they should not push other data out of L2)
                struct {
                    double* p;
                    long cap, t;
                    __device__ __forceinline__ void put(int v, double f) { __stcs(p + v * cap + t, f); }
                } qw{q, A.ps.cap, t};
                T::vars_q(s, x, qw);
            } else {
                T::vars(s, x);
            }
        }
    }
    T::shift(x, xf);
    return live;
}

// Mixed-precision evaluation in three kernels.  The FP64 work around the
// polynomial (gather, image, variables; later the switch, chain rule,
// virial and scatter) is latency-bound and needs many warps, the paired FP32
// trie needs few warps with all registers in lockstep; in one kernel both
// ran at 8 warps per SM, so the FP64 parts took ~0.2 of the ~0.9 ms the
// 2048-water trimers take.  Here:
//   pair_vars_kernel    one n-mer per thread at full occupancy: the FP64
//                       variables, shifted to the FP32 basis, into A.ps.dx
//   pair_trie_kernel    the paired FP32 trie in lockstep blocks (two n-mers
//                       per thread), dx in, gradient and value out
//   pair_finish_kernel  one n-mer per thread at full occupancy: switch,
//                       chain rule (FP64), virial, scatter, energy sums
// The variables, switch, chain rule and sums stay FP64 as before.
template <class T>
__global__ void __launch_bounds__(256, 2) pair_vars_kernel(const HolderArgs A) {
    const long n = nmer_count(A);
    const long cap = A.ps.cap;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        float xf[T::NVARS];
        const bool live = nmer_vars_f32<T>(A, t, n, xf, A.ps.q);
#pragma unroll
        for (int v = 0; v < T::NVARS; ++v) {
            A.ps.dx[v * cap + t] = xf[v];
            A.ps.g[v * cap + t] = 0.0f;   // the tensor-core kernel adds into g and ep
        }
        A.ps.ep[t] = 0.0;
        A.ps.live[t] = live ? 1 : 0;
    }
}

// Coefficient pairs of the FP32 basis copied from constant to shared memory
// once per block (a shared-memory operand costs fewer instructions per leaf
// than a constant-bank one in the paired form).
template <class CC>
struct SharedPairs {
    const f2_t* p;
    __device__ __forceinline__ f2_t f2(int k) const { return p[k]; }
    __device__ __forceinline__ double b0() const { return CC{}.b0(); }
};

// The paired FP32 trie: two n-mers per thread, one in each half of the
// paired FP32 registers, through the type's FP32-basis trie (T::SHIFTED) in
// lockstep blocks; a block claims chunks of 2 x blockDim.x n-mers.
template <class T, class CC>
__global__ void __launch_bounds__(T::LOCK_THREADS_S, 1) pair_trie_kernel(const HolderArgs A) {
    constexpr int L = T::LOCK_THREADS_S;   // == blockDim.x
    f2_t* xs = reinterpret_cast<f2_t*>(mbx_dyn_smem) + threadIdx.x;
    f2_t* gs = xs + T::NVARS * L;
    __shared__ long s_base;
    __shared__ f2_t s_coef[T::NORB];
    for (int k = threadIdx.x; k < T::NORB; k += blockDim.x) s_coef[k] = CC{}.f2(k);
    __syncthreads();
    const SharedPairs<CC> coef{s_coef};
    if (A.prime_passes > 0) {
        prime_pieces<L, f2_t>(A, T::NVARS, [&](int k, const f2_t* x, f2_t* g) -> double {
            const double2 e = T::template pip_s32_piece<L>(k, coef, x, g);
            return e.x + e.y;
        });
        return;
    }
    const long n = nmer_count(A);
    const long cap = A.ps.cap;
    const long chunk = 2L * blockDim.x;
    for (;;) {
        if (threadIdx.x == 0) s_base = atomicAdd(A.counter, (int)chunk);
        __syncthreads();
        const long base = s_base;
        __syncthreads();
        if (base >= n) break;
        const long t0 = base + threadIdx.x, t1 = t0 + blockDim.x;
#pragma unroll
        for (int v = 0; v < T::NVARS; ++v) {
            const float lo = t0 < n ? A.ps.dx[v * cap + t0] : 0.0f;
            const float hi = t1 < n ? A.ps.dx[v * cap + t1] : 0.0f;
            xs[v * L] = f2_pack(lo, hi);
            gs[v * L] = 0ull;
        }
        const double2 ep = T::template pip_s32_lock<L>(coef, xs, gs);
        if (t0 < n) {
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) A.ps.g[v * cap + t0] = f2_lo(gs[v * L]);
            A.ps.ep[t0] = coef.b0() + ep.x;
        }
        if (t1 < n) {
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) A.ps.g[v * cap + t1] = f2_hi(gs[v * L]);
            A.ps.ep[t1] = coef.b0() + ep.y;
        }
    }
}

template <class T>
__global__ void __launch_bounds__(128, 4) pair_finish_kernel(const HolderArgs A) {
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const long n = nmer_count(A);
    const long cap = A.ps.cap;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
        if (!A.ps.live[t]) continue;
        // the chain rule from the radial factors pair_vars_kernel stored: no
        // square root, exponential or division per variable here
        finish_nmer<T>(A, t, A.ps.ep[t], PairFactors{{A.ps.g, cap, t}, {A.ps.q, cap, t}}, true, acc);
    }
    block_reduce_add<7>(acc, A.out);
}

// Table-driven evaluation (evaluators without straight-line code): a warp
// per n-mer, lane l taking terms l, l+32, ... of the term table
// (term_table.cuh); the n-mer's variables and gradient accumulators live in
// shared memory, the gradient summed with shared-memory atomics.  The rest
// (gather, image, variables, switch, chain rule, scatter) is the same code
// as the straight-line kernels.
template <class T, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) holder_table_kernel(const HolderArgs A, int grads) {
    __shared__ double xs[WARPS][T::NVARS];
    __shared__ double gs[WARPS][T::NVARS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const long stride = (long)gridDim.x * WARPS;
    const long n = nmer_count(A);
    for (long t = blockIdx.x * (long)WARPS + w; t < n; t += stride) {
        double r[T::NREAL][3];
        load_nmer<T, false>(A, t, r);
        double d[3][3], rr[3];
        if (pair_dists<T>(r, d, rr)) {
            if (lane == 0 && A.e_per) A.e_per[t] = 0.0;
            continue;
        }
        if (lane == 0) {
            double s[T::NSITES][3], x[T::NVARS];
            T::sites(r, s);
            T::vars(s, x);
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) { xs[w][v] = x[v]; gs[w][v] = 0.0; }
        }
        __syncwarp();
        const auto xv = [&](int v) { return xs[w][v]; };
        double e = 0.0;
        for (long q = lane; q < A.nterms; q += 32) {
            const int4 tm = __ldg(A.terms + q);
            const double c = __ldg(A.coef + tm.x) * __ldg(A.tcoef + q);
            if (grads)
                e += term_value_grad<T::TPAIRS>(tm, c, xv, [&](int v, double dv) { atomicAdd(&gs[w][v], dv); });
            else
                e += term_value<T::TPAIRS>(tm, c, xv);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
        __syncwarp();
        if (lane == 0) {
            double g[T::NVARS];
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) g[v] = gs[w][v];
            finish_nmer<T>(A, t, e, g, grads != 0, acc);
        }
        __syncwarp();
    }
    block_reduce_add<7>(acc, A.out);
}

// Table-driven evaluation, a lane per n-mer: the warp walks the whole term
// table in step, every lane applying each term to its own n-mer, whose
// variables and gradient accumulators sit in shared-memory columns [v][lane]
// (conflict-free, no atomics).  This is the form for the many-n-mer buckets
// of a liquid (a warp per n-mer would serialise on shared-memory atomics of
// the few variables); the 201k-term CH4-CH4 table, with few dimers per box,
// keeps the warp-per-n-mer form above.  Dynamic shared memory:
// 4 warps x 2 x NVARS x 32 doubles.
template <class T>
__global__ void __launch_bounds__(128) holder_table_lane_kernel(const HolderArgs A, int grads) {
    double* xc = reinterpret_cast<double*>(mbx_dyn_smem) + ((threadIdx.x >> 5) * 2 * T::NVARS) * 32 +
                 (threadIdx.x & 31);
    double* gc = xc + T::NVARS * 32;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const long n = nmer_count(A);
    for (long base = blockIdx.x * (long)blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
        const long t = base + threadIdx.x;
        bool live = t < n;
        {
            double x[T::NVARS];
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) x[v] = 0.0;
            if (live) {
                double r[T::NREAL][3];
                load_nmer<T, false>(A, t, r);
                double d[3][3], rr[3];
                if (pair_dists<T>(r, d, rr)) {
                    if (A.e_per) A.e_per[t] = 0.0;
                    live = false;
                } else {
                    double s[T::NSITES][3];
                    T::sites(r, s);
                    T::vars(s, x);
                }
            }
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) {
                xc[v * 32] = x[v];
                gc[v * 32] = 0.0;
            }
        }
        __syncwarp();
        double e = 0.0;
        if (__any_sync(0xffffffffu, live)) {
            const auto xv = [&](int v) { return xc[v * 32]; };
            for (long q = 0; q < A.nterms; ++q) {
                const int4 tm = __ldg(A.terms + q);
                const double c = __ldg(A.coef + tm.x) * __ldg(A.tcoef + q);
                if (grads)
                    e += term_value_grad<T::TPAIRS>(tm, c, xv, [&](int v, double dv) { gc[v * 32] += dv; });
                else
                    e += term_value<T::TPAIRS>(tm, c, xv);
            }
        }
        __syncwarp();
        if (live) {
            double g[T::NVARS];
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) g[v] = grads ? gc[v * 32] : 0.0;
            finish_nmer<T>(A, t, e, g, grads != 0, acc);
        }
        __syncwarp();
    }
    block_reduce_add<7>(acc, A.out);
}

// 1-body MB-nrg evaluation (x1b_*::eval, e.g. x1b_A1B4_v1x::eval,
// potential/1b/x1b_A1B4_deg5_exp0_v1x.cpp:361-419): no image, no switch, no
// cutoff.  A lane per monomer, the warp walking the term table in step (as
// holder_table_lane_kernel); variables, chain rule and the virial
// -sum r (x) g over the monomer's atoms as the reference's evaluator does.
// A.first_index: first site of each monomer to evaluate (A.n of them); one
// thread per monomer writes its gradient, so no atomics.  Dynamic shared
// memory: 4 warps x 2 x NVARS x 32 doubles.
template <class T>
__global__ void __launch_bounds__(128) onebody_table_kernel(const HolderArgs A) {
    static_assert(T::NBODY == 1, "1-body evaluators only");
    double* xc = reinterpret_cast<double*>(mbx_dyn_smem) + ((threadIdx.x >> 5) * 2 * T::NVARS) * 32 +
                 (threadIdx.x & 31);
    double* gc = xc + T::NVARS * 32;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const bool grads = A.grad != nullptr;
    for (long base = blockIdx.x * (long)blockDim.x; base < A.n; base += (long)gridDim.x * blockDim.x) {
        const long t = base + threadIdx.x;
        const bool live = t < A.n;
        double r[T::NREAL][3];
        double s[T::NSITES][3];
        {
            double x[T::NVARS];
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) x[v] = 0.0;
            if (live) {
                const double* p = A.xyz + 3 * (size_t)__ldg(A.first_index + t);
#pragma unroll
                for (int i = 0; i < T::NREAL; ++i)
#pragma unroll
                    for (int c = 0; c < 3; ++c) r[i][c] = p[3 * i + c];
                T::sites(r, s);
                T::vars(s, x);
            }
#pragma unroll
            for (int v = 0; v < T::NVARS; ++v) {
                xc[v * 32] = x[v];
                gc[v * 32] = 0.0;
            }
        }
        __syncwarp();
        double e = 0.0;
        if (__any_sync(0xffffffffu, live)) {
            const auto xv = [&](int v) { return xc[v * 32]; };
            for (long q = 0; q < A.nterms; ++q) {
                const int4 tm = __ldg(A.terms + q);
                const double c = __ldg(A.coef + tm.x) * __ldg(A.tcoef + q);
                if (grads)
                    e += term_value_grad<T::TPAIRS>(tm, c, xv, [&](int v, double dv) { gc[v * 32] += dv; });
                else
                    e += term_value<T::TPAIRS>(tm, c, xv);
            }
        }
        __syncwarp();
        if (live) {
            acc[0] += e;
            if (grads) {
                double g[T::NVARS];
#pragma unroll
                for (int v = 0; v < T::NVARS; ++v) g[v] = gc[v * 32];
                double sg[T::NSITES][3];
                T::chain(s, g, sg);
                const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    double v = 0.0;
#pragma unroll
                    for (int i = 0; i < T::NREAL; ++i) v -= r[i][ia[k]] * sg[i][ib[k]];
                    acc[1 + k] += v;
                }
                double* q = A.grad + 3 * (size_t)__ldg(A.first_index + t);
#pragma unroll
                for (int i = 0; i < T::NREAL; ++i)
#pragma unroll
                    for (int c = 0; c < 3; ++c) q[3 * i + c] += sg[i][c];
            }
        }
        __syncwarp();
    }
    block_reduce_add<7>(acc, A.out);
}

// Gradient with respect to the linear coefficients: out[k] += sum over n-mers
// of w[n] * sw(n) * dP/da_k(x(n)), the monomials recomputed from the
// coordinates (adjoint of E = sum_n sw(n) P(a, x(n)) for refitting), from the
// term table.  A lane per n-mer, its variables in a shared-memory column; the
// warp walks the table (sorted by coefficient) in step, and at the end of a
// coefficient's terms the lanes' sums are reduced across the warp into a
// per-block shared array, added to out at the end.
// Dynamic shared memory: NCOEF doubles + 4 warps x NVARS x 32 doubles.
template <class T>
__global__ void __launch_bounds__(128) holder_dcoef_table_kernel(const HolderArgs A, const double* __restrict__ w,
                                                                 double* __restrict__ out) {
    double* part = reinterpret_cast<double*>(mbx_dyn_smem);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* xcol = part + T::NCOEF + (warp * T::NVARS) * 32 + lane;
    for (int k = threadIdx.x; k < T::NCOEF; k += blockDim.x) part[k] = 0.0;
    __syncthreads();
    const long nt = nmer_count(A);
    for (long base = blockIdx.x * (long)blockDim.x; base < nt; base += (long)gridDim.x * blockDim.x) {
        const long t = base + threadIdx.x;
        double scale = 0.0;
        double x[T::NVARS];
#pragma unroll
        for (int v = 0; v < T::NVARS; ++v) x[v] = 0.0;
        if (t < nt) {
            double r[T::NREAL][3];
            load_nmer<T, false>(A, t, r);
            double d[3][3], rr[3];
            if (!pair_dists<T>(r, d, rr)) {
                double s[T::NSITES][3];
                T::sites(r, s);
                T::vars(s, x);
                double tg[T::NREAL][3];
                scale = apply_switch<T>(d, rr, 0.0, tg, false) * (w ? w[t] : 1.0);
            }
        }
#pragma unroll
        for (int v = 0; v < T::NVARS; ++v) xcol[v * 32] = x[v];
        __syncwarp();
        if (__any_sync(0xffffffffu, scale != 0.0)) {
            const auto xv = [&](int v) { return xcol[v * 32]; };
            double sum = 0.0;
            int4 tm = __ldg(A.terms);
            for (long q = 0; q < A.nterms; ++q) {
                const int4 nx = q + 1 < A.nterms ? __ldg(A.terms + q + 1) : make_int4(-1, 0, 0, 0);
                sum += term_value<T::TPAIRS>(tm, __ldg(A.tcoef + q), xv);
                if (nx.x != tm.x) {
                    double v = sum * scale;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                    if (lane == 0 && v != 0.0) atomicAdd(&part[tm.x], v);
                    sum = 0.0;
                }
                tm = nx;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int k = threadIdx.x; k < T::NCOEF; k += blockDim.x)
        if (part[k] != 0.0) atomicAdd(out + k, part[k]);
}
