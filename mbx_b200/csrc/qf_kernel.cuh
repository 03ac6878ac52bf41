// Tensor-core evaluation of a degree-4 polynomial written as a quadratic
// form, P(d) = m(d)^T C m(d) over a basis m of monomials of degree <= 2
// (mbx_b200/codegen/qf.py).  It replaces the paired FP32 trie in the mixed
// path: between pair_vars_kernel (the shifted FP32 variables d of every
// n-mer, A.ps.dx) and pair_finish_kernel (chain rule, sums, scatter), it
// writes P and dP/dd of every n-mer (A.ps.ep, A.ps.g) exactly as the trie
// does.
//
// One CTA per SM, persistent over tiles of 128 n-mers.  For a tile, Y = M C
// (128 x NB, NB = 480) is a product of FP16 operands accumulated in FP32 in
// tensor memory by tcgen05.mma (M = 128, K = 16), in Q::NPASS passes over
// the output columns (two of 240 for MB-pol 3b: an MMA of M = 128, K = 16
// takes the same ~130 SM cycles for N = 128 and N = 256, so the widest
// passes take the fewest):
//   A operand  the tile's basis values, split hi + lo, written to shared
//              memory by the row threads, K block by K block (the same blocks
//              in every pass);
//   B operand  C split hi + mid + lo, prepared on the host in the canonical
//              no-swizzle K-major layout (8 x 16-byte core matrices, row
//              groups contiguous, see sdesc), one bulk copy (cp.async.bulk)
//              per K block and pass from the type's image;
//   products   hi.hi into the pass's main accumulator, hi.mid + lo.hi, and
//              hi.lo on the first Q::KT blocks, into its correction
//              accumulator.  The tensor core's FP32 accumulation aligns the
//              addends of an MMA to the largest and truncates; the main
//              partial sums are large next to their final values (the
//              polynomial cancels), so keeping the corrections out of them
//              cuts the truncation steps of the large sums from 98 to 30.
// A pass of 240 columns takes 480 TMEM columns (main + correction), so the
// 512 hold one buffer: the MMAs of pass q + 1 start once pass q is read
// back (passes of at most 128 columns get two buffers, see Layout).
// Warps 0-7 are the row threads, in two sets of 128 (thread i of a set owns
// n-mer i of the tile and reads TMEM lane i): set 0 generates the even
// stages of A and reads back the even chunks of 16 columns of both
// accumulators (tcgen05.ld) for the energy m . y and the gradient
// 2 sum_j y_j dm_j/dd; set 1 the odd ones.  Warp 8 lane 0 issues the bulk
// copies, warp 9 lane 0 the MMAs; warp 9 also owns the TMEM allocation.
// Shared-memory slots of one stage each (Layout::BPS K blocks of A and B)
// cycle through NS slots with mbarriers:
//   afull[s]   128 arrivals of the set that writes the stage (A written, proxy-fenced)
//   bfull[s]   the producer's expect_tx + the copies' bytes
//   empty[s]   tcgen05.commit after the stage's MMAs
//   tfull[b]   tcgen05.commit after a pass's last stage (buffer b complete)
//   tempty[b]  256 row-thread arrivals (buffer b read out)
// Every wait is bounded (QF_WAIT_NS of %globaltimer): on a timeout the CTA
// sets an abort flag that ends every role's loop, drains its MMAs and
// copies, frees its TMEM and reports MBX_STATUS_WAIT_TIMEOUT in *A.ps.err.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include "holder_kernel.cuh"
#include "nmer_build.h"

namespace qf {

constexpr int A_PART = 128 * 16 * 2;  // bytes of one FP16 part of an A block (128 rows x K 16)
constexpr int A_BYTES = 2 * A_PART;
constexpr int PARK_SET = 128 * (36 + 2) * 4; // one row set's gradient (36 floats) and energy of each row
constexpr int PARK = 2 * PARK_SET;
constexpr int SMEM_MAX = 232448;
constexpr int ROW_WARPS = 8;                  // two sets of 4 warps over the 128 rows
constexpr int PRODUCER_WARP = ROW_WARPS, MMA_WARP = ROW_WARPS + 1;
constexpr int THREADS = 32 * (ROW_WARPS + 2);
constexpr unsigned long long QF_WAIT_NS = 4000000000ull;
// Suspend-time hint of every wait: a thread whose phase is not complete
// sleeps until it completes (or this many ns pass) instead of spinning, so
// that waiting warps take no issue slots from the MMA issuer and the row
// threads that share their SM sub-partition.
constexpr uint32_t QF_SUSPEND_NS = 1000000;
// tcgen05 instruction descriptor, kind::f16: F32 accumulator (bits 4-5 = 1),
// F16 A and B (formats 0), both K-major, N (bits 17-22: N >> 3), M = 128
// (bits 24-28: M >> 4)
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}
// Shared memory and tensor memory of a quadratic form Q: a stage is BPS
// consecutive K blocks, and its slot holds their A blocks (A_BYTES each) and
// the widest pass's B chunks (BCHUNK each); passes of at most 128 columns get
// two TMEM buffers of 256 columns (main + correction accumulator of 128 each:
// the MMAs of a pass run while the previous one is read back), wider ones
// (up to 256) one buffer, the correction accumulator at column 256.  Two
// blocks per stage halve the barrier waits of the MMA issuer per MMA: the
// issuer's waits, not the tensor core, bounded the one-block stages.
template <class Q>
struct Layout {
    static constexpr int MAXN = Q::pass_n(0);   // passes are widest first
    static constexpr int BPS = 2;               // K blocks per stage
    static constexpr int NSTAGE = Q::KS / BPS;  // stages per pass
    static constexpr int BCHUNK = 3 * MAXN * 32;
    static constexpr int BOFF = BPS * A_BYTES;  // B chunks after the A blocks
    static constexpr int SLOT = (BPS * (A_BYTES + BCHUNK) + 1023) / 1024 * 1024;
    static constexpr int NS_FIT = (SMEM_MAX - 1024 - PARK) / SLOT;
    static constexpr int NS = NS_FIT < 9 ? NS_FIT : 9;   // shared-memory stages
    static constexpr int SMEM = NS * SLOT + 1024 + PARK;  // + alignment of the first slot
    static constexpr bool DB = MAXN <= 128;              // double-buffered tensor memory
    static constexpr int CORR_COL = DB ? 128 : 256;
    static_assert(MAXN <= 256 && NS >= 3 && SMEM <= SMEM_MAX && Q::KS % BPS == 0, "quadratic form does not fit");
    __host__ __device__ static constexpr int buf(long q) { return DB ? (int)(q & 1) : 0; }
    __host__ __device__ static constexpr long use(long q) { return DB ? q >> 1 : q; }   // uses of buf(q) before pass q
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(QF_SUSPEND_NS)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the completion of the phase of parity `parity`; false (and the
// abort flag set) after QF_WAIT_NS, false at once when another role aborted.
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (global_ns() - t0 > QF_WAIT_NS) {
            *abort_flag = 1;
            return false;
        }
    }
}

// Same, ignoring the abort flag (cleanup of work already in flight).
__device__ __forceinline__ bool wait_drain(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > QF_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor: K-major, no swizzle (core matrices of
// 8 rows x 16 bytes stored as 128 contiguous bytes), successive 8-row groups
// 128 bytes apart (stride byte offset), the second core-matrix column of the
// K block (k 8..15) lbo bytes after the first (leading byte offset); version
// 1 (bit 46).  With the row groups contiguous, the groups that the tensor
// core reads together sit in distinct shared-memory banks (groups 256 bytes
// apart, the K block's two columns interleaved, put them in the same banks:
// the kernel ran at a third of the tensor rate).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
}
constexpr uint32_t A_LBO = 16 * 128;   // A block: 16 row groups (128 rows) per core-matrix column
// a B chunk of n rows: n / 8 row groups per core-matrix column

// D[tmem] (+)= A[smem] B[smem]^T, one thread issues.
__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 consecutive FP32 columns of the warp's 32 TMEM lanes (lane = thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// tcgen05.wait::ld, with the loaded registers as operands so that no use of
// them is scheduled before the wait.
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// hi and lo FP16 parts of two values (lo = the FP16 rounding of the exact
// FP32 remainder)
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 f = __half22float2(h);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = pack_h2(a - f.x, b - f.y);
}

}  // namespace qf

// One pass's epilogue for one row set: main + correction accumulator of
// the set's chunks of 16 columns (chunks SET, SET + 2, ... of the pass),
// Q::epi on each (the chunk index a constant).  The TMEM loads of the next
// chunk are in flight while the current chunk's arithmetic runs.  g must
// enter zeroed: the energy is completed from it.
template <class Q, int PASS, int SET, int NV>
__device__ __forceinline__ double qf_epilogue_pass(uint32_t tbuf, const float (&d)[NV], float (&g)[NV]) {
    constexpr int HC = Q::pass_n(PASS) / 16;   // chunks of 16 columns in the pass
    constexpr int NCH = (HC - SET + 1) / 2;    // this set's chunks
    constexpr int C0 = Q::pass_col(PASS) / 16;
    double P = 0.0;
    uint32_t ym[2][16], yc[2][16];
    qf::tmem_ld16(tbuf + (uint32_t)(SET * 16), ym[0]);
    constexpr uint32_t CC = (uint32_t)qf::Layout<Q>::CORR_COL;
    qf::tmem_ld16(tbuf + CC + (uint32_t)(SET * 16), yc[0]);
    qf::tmem_wait_ld(ym[0]);
    qf::tmem_wait_ld(yc[0]);
#pragma unroll
    for (int k = 0; k < NCH; ++k) {
        const int b = k & 1, cc = SET + 2 * k;
        if (k + 1 < NCH) {
            qf::tmem_ld16(tbuf + (uint32_t)((cc + 2) * 16), ym[b ^ 1]);
            qf::tmem_ld16(tbuf + CC + (uint32_t)((cc + 2) * 16), yc[b ^ 1]);
        }
        // z = (main + correction) x column scale, two columns per paired
        // FP32 instruction (the same roundings as one column at a time)
        float z[16];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const f2_t y2 = f2_add(f2_pack(__uint_as_float(ym[b][2 * i]), __uint_as_float(ym[b][2 * i + 1])),
                                   f2_pack(__uint_as_float(yc[b][2 * i]), __uint_as_float(yc[b][2 * i + 1])));
            const f2_t z2 = f2_mul(y2, Q::colf2((C0 + cc) * 8 + i));
            z[2 * i] = f2_lo(z2);
            z[2 * i + 1] = f2_hi(z2);
        }
        P += (double)Q::epi(C0 + cc, z, d, g);
        if (k + 1 < NCH) {
            qf::tmem_wait_ld(ym[b ^ 1]);
            qf::tmem_wait_ld(yc[b ^ 1]);
        }
    }
    // the degree-2 columns' energy, sum_j m_j z_j = (sum_u d_u g_u) / 2 over
    // them (Q::epi), here with the degree-1 columns' share (also in g)
    double dg = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) dg = fma((double)d[v], (double)g[v], dg);
    return P + 0.5 * dg;
}

template <class Q, int SET, int NV>
__device__ __forceinline__ double qf_epilogue(int pass, uint32_t tbuf, const float (&d)[NV], float (&g)[NV]) {
    switch (pass) {
        case 0: return qf_epilogue_pass<Q, 0, SET>(tbuf, d, g);
        case 1: return qf_epilogue_pass<Q, 1, SET>(tbuf, d, g);
        case 2: return qf_epilogue_pass<Q, 2, SET>(tbuf, d, g);
        default: return qf_epilogue_pass<Q, 3, SET>(tbuf, d, g);
    }
}

// Stage st of pass q (ring index q NSTAGE + st) of A for one row: wait for
// the slot, generate the row's 16 values (hi and lo parts) of each of the
// stage's K blocks from the variables d and row scales sc, store, fence for
// the tensor core, arrive.  false (warp-uniform) when the CTA aborted.  Every
// pass of a tile generates the same blocks (the passes differ in the columns
// of C).
template <class Q, int NV, int ST>
__device__ __forceinline__ bool qf_gen_stage(long q, float (&d)[NV], float (&sc)[Q::NT], uint32_t arow,
                                             uint64_t* bar_empty, uint64_t* bar_afull, volatile int* abort_flag) {
    using namespace qf;
    using L = Layout<Q>;
    constexpr int NS = L::NS, SLOT = L::SLOT;
    const uint32_t it = (uint32_t)q * L::NSTAGE + (uint32_t)ST;   // ring index (32 bits: see the kernel)
    const uint32_t slot = it % NS, use = it / NS;
    const bool free_slot = use == 0 || wait(smem_u32(&bar_empty[slot]), (use - 1) & 1u, abort_flag);
    if (!__all_sync(0xffffffffu, free_slot)) return false;
#pragma unroll
    for (int j = 0; j < L::BPS; ++j) {
        // generate each block here, not earlier: the same blocks recur in
        // every pass, and hoisting them costs registers
#pragma unroll
        for (int v = 0; v < NV; ++v) asm volatile("" : "+f"(d[v]));
#pragma unroll
        for (int k = 0; k < Q::NT; ++k) asm volatile("" : "+f"(sc[k]));
        uint32_t hi[8], lo[8];
        Q::gen(ST * L::BPS + j, d, sc, hi, lo);
        const uint32_t a = arow + slot * SLOT + (uint32_t)(j * A_BYTES);
        st_shared_v4(a, make_uint4(hi[0], hi[1], hi[2], hi[3]));
        st_shared_v4(a + A_LBO, make_uint4(hi[4], hi[5], hi[6], hi[7]));
        st_shared_v4(a + A_PART, make_uint4(lo[0], lo[1], lo[2], lo[3]));
        st_shared_v4(a + A_PART + A_LBO, make_uint4(lo[4], lo[5], lo[6], lo[7]));
    }
    fence_proxy_async();
    mbar_arrive(smem_u32(&bar_afull[slot]));
    return true;
}

// The stages lo <= st < hi of one set's parity for pass q.
template <class Q, int NV, int ST = 0>
__device__ __forceinline__ bool qf_gen_pass(int set, long q, int lo, int hi, float (&d)[NV], float (&sc)[Q::NT],
                                            uint32_t arow, uint64_t* bar_empty, uint64_t* bar_afull,
                                            volatile int* abort_flag) {
    if constexpr (ST < qf::Layout<Q>::NSTAGE) {
        if ((ST & 1) == set && ST >= lo && ST < hi &&
            !qf_gen_stage<Q, NV, ST>(q, d, sc, arow, bar_empty, bar_afull, abort_flag))
            return false;
        return qf_gen_pass<Q, NV, ST + 1>(set, q, lo, hi, d, sc, arow, bar_empty, bar_afull, abort_flag);
    }
    return true;
}

// T: the evaluator traits (NVARS); Q: the generated quadratic form
// (<name>_qf.cuh): KS K blocks of 16, the first KT with the third C part,
// NPASS passes over the columns, the (block, pass) chunks of the image, the
// row-scale classes, gen(s) and epi(c).
template <class T, class Q>
__global__ void __launch_bounds__(qf::THREADS, 1) qf_eval_kernel(const HolderArgs A) {
    using namespace qf;
    using L = Layout<Q>;
    constexpr int NV = T::NVARS;
    constexpr int NP = Q::NPASS;
    constexpr int NS = L::NS, SLOT = L::SLOT;
    __shared__ __align__(8) uint64_t bar_afull[NS], bar_bfull[NS], bar_empty[NS];
    __shared__ __align__(8) uint64_t bar_tfull[2], bar_tempty[2], bar_drain;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ long s_n;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_u32(mbx_dyn_smem) + 1023u) & ~1023u;
    const long cap = A.ps.cap;

    if (tid == 0) {
        // read once: every role must walk the same tiles (another CTA may set
        // the status word meanwhile)
        s_n = nmer_count(A);
        for (int s = 0; s < NS; ++s) {
            mbar_init(smem_u32(&bar_afull[s]), 128);
            mbar_init(smem_u32(&bar_bfull[s]), 1);
            mbar_init(smem_u32(&bar_empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&bar_tfull[b]), 1);
            mbar_init(smem_u32(&bar_tempty[b]), 32 * ROW_WARPS);
        }
        mbar_init(smem_u32(&bar_drain), 1);
        s_abort = 0;
        fence_mbar_init();
    }
    if (warp == MMA_WARP) {
        tmem_alloc(smem_u32(&s_tmem), 512);
        tmem_relinquish();
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = s_tmem;
    const long n = s_n;
    const long ntiles = (n + 127) / 128;
    // passes of this CTA: NP per tile, tiles blockIdx.x, + gridDim.x, ...
    const long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long npasses = my_tiles * NP;
    // the shared-memory ring index (pass x KS + block) is kept in 32 bits:
    // 2^32 / KS passes per CTA, far above any box (2 x 10^9 n-mers are
    // 2 x 10^5 passes per CTA on 148 SMs)

    if (warp < ROW_WARPS) {
        // ---- row threads.  Two sets of 128 threads, thread i of a set on
        // row i: set 0 (warps 0-3) generates the even stages and reads the
        // even 16-column chunks of a pass back, set 1 (warps 4-7) the odd
        // ones.  Software pipeline over the passes: generate the first AHEAD
        // stages of pass q + 1, then read pass q back.  With two TMEM buffers
        // that is all of pass q + 1, whose MMAs fill the other buffer
        // meanwhile; with one, the NS stages that fit the ring, written while
        // the last MMAs of pass q run, so that the MMAs of pass q + 1 start
        // as soon as pass q is read back.  Each set sums its share of a
        // tile's energy and gradient over the passes in shared memory and
        // adds the totals to the outputs (zeroed by pair_vars_kernel; two
        // addends onto zero, so the result does not depend on their order).
        const int set = warp / 4;
        const int row = tid & 127;
        const uint32_t arow = base + (uint32_t)((row >> 3) * 128 + (row & 7) * 16);
        const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);   // the warp's TMEM lane quarter
        float* park_g = reinterpret_cast<float*>(mbx_dyn_smem + (base - smem_u32(mbx_dyn_smem)) + NS * SLOT) +
                        set * (PARK_SET / 4);
        double* park_p = reinterpret_cast<double*>(park_g + 36 * 128);
        static_assert(NV <= 36, "park area holds 36 gradient entries");
        auto load_vars = [&](long tl, float (&dv)[NV], float (&sv)[Q::NT]) -> float {
            const long tt = tl * 128 + row;
#pragma unroll
            for (int v = 0; v < NV; ++v) dv[v] = tt < n ? A.ps.dx[v * cap + tt] : 0.0f;
            return Q::row_scales(dv, sv);
        };
        // stages of pass q + 1 generated before pass q is read back (with one
        // buffer, more would wait for ring slots that only the MMAs of pass
        // q + 1 free, and those wait for the read-back)
        constexpr int AHEAD = L::DB ? L::NSTAGE : (NS < L::NSTAGE ? NS : L::NSTAGE);
        float de[NV], dg[NV], sg[Q::NT];   // variables of the tile read back / being generated
        float rinv_e = 1.0f, rinv_g = 1.0f;
        if (npasses > 0) {
            rinv_g = load_vars(blockIdx.x, dg, sg);
#pragma unroll
            for (int v = 0; v < NV; ++v) de[v] = dg[v];
            rinv_e = rinv_g;
            if (!qf_gen_pass<Q, NV>(set, 0, 0, AHEAD, dg, sg, arow, bar_empty, bar_afull, &s_abort)) goto rows_done;
        }
        for (long q = 0; q < npasses; ++q) {
            const int p = (int)(q % NP);
            const long tile = blockIdx.x + (q / NP) * gridDim.x;
            // the rest of pass q, then the first stages of pass q + 1
            if (!qf_gen_pass<Q, NV>(set, q, AHEAD, L::NSTAGE, dg, sg, arow, bar_empty, bar_afull, &s_abort))
                goto rows_done;
            if (q + 1 < npasses) {
                if (p == NP - 1) rinv_g = load_vars(tile + gridDim.x, dg, sg);
                if (!qf_gen_pass<Q, NV>(set, q + 1, 0, AHEAD, dg, sg, arow, bar_empty, bar_afull, &s_abort))
                    goto rows_done;
            }
            const int bi = L::buf(q);
            // warp-uniform: the TMEM loads below are warp-collective
            if (!__all_sync(0xffffffffu, wait(smem_u32(&bar_tfull[bi]), (uint32_t)(L::use(q) & 1), &s_abort)))
                goto rows_done;
            tc_after();
            {
                float g[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) g[v] = 0.0f;
                const uint32_t tbuf = trow + (uint32_t)(bi * 256);
                const double P = set == 0 ? qf_epilogue<Q, 0>(p, tbuf, de, g) : qf_epilogue<Q, 1>(p, tbuf, de, g);
                tc_before();
                mbar_arrive(smem_u32(&bar_tempty[bi]));
                // the set's running sums of the tile
#pragma unroll
                for (int v = 0; v < NV; ++v) park_g[v * 128 + row] = (p == 0 ? 0.0f : park_g[v * 128 + row]) + g[v];
                park_p[row] = (p == 0 ? 0.0 : park_p[row]) + P;
            }
            if (p == NP - 1) {
                const long t = tile * 128 + row;
                if (t < n) {
                    const float gs = 2.0f * rinv_e;
#pragma unroll
                    for (int v = 0; v < NV; ++v) atomicAdd(A.ps.g + v * cap + t, park_g[v * 128 + row] * gs);
                    atomicAdd(A.ps.ep + t, (set == 0 ? Q::b0() : 0.0) + park_p[row] * (double)rinv_e);
                }
#pragma unroll
                for (int v = 0; v < NV; ++v) de[v] = dg[v];
                rinv_e = rinv_g;
            }
        }
    rows_done:;
    } else if (warp == PRODUCER_WARP) {
        // ---- producer: one bulk copy of C's (K block, pass) chunk per stage ----
        if (lane == 0) {
            uint32_t it = 0, slot = 0, phase = 0;   // ring index, its slot and use parity
            for (long q = 0; q < npasses; ++q) {
                const int p = (int)(q % NP);
                for (int st = 0; st < L::NSTAGE; ++st, ++it) {
                    if (it >= NS && !wait(smem_u32(&bar_empty[slot]), phase ^ 1u, &s_abort)) goto producer_done;
                    uint32_t bytes = 0;
                    for (int j = 0; j < L::BPS; ++j) bytes += (uint32_t)Q::chunk_bytes(st * L::BPS + j, p);
                    const uint32_t bar = smem_u32(&bar_bfull[slot]);
                    mbar_arrive_tx(bar, bytes);
                    for (int j = 0; j < L::BPS; ++j) {
                        const int s = st * L::BPS + j;
                        bulk_g2s(base + slot * SLOT + (uint32_t)(L::BOFF + j * L::BCHUNK),
                                 Q::image() + Q::chunk_offset(s, p), (uint32_t)Q::chunk_bytes(s, p), bar);
                    }
                    if (++slot == NS) slot = 0, phase ^= 1u;
                }
            }
        producer_done:
            // copies in flight complete on their own: wait for them before the
            // shared memory goes away (the last use of every slot)
            for (uint32_t k = 0; k < NS && k < it; ++k) {
                const uint32_t qq = it - 1 - k;   // ring index of the last copy into slot qq % NS
                wait_drain(smem_u32(&bar_bfull[qq % NS]), (qq / NS) & 1u);
            }
        }
    } else {
        // ---- MMA issuer ----
        if (lane == 0) {
            uint32_t slot = 0, phase = 0;   // ring slot and use parity
            bool issued = false;
            for (long q = 0; q < npasses; ++q) {
                const int p = (int)(q % NP);
                const int b = L::buf(q);
                const long u = L::use(q);
                if (u >= 1) {
                    // the buffer's previous pass has been read back
                    if (!wait(smem_u32(&bar_tempty[b]), (uint32_t)((u - 1) & 1), &s_abort)) goto mma_done;
                    tc_after();
                }
                const int nn = Q::pass_n(p);
                const uint32_t id = idesc(nn), blbo = (uint32_t)(nn / 8) * 128, bpart = (uint32_t)nn * 32;
                const uint32_t dmain = tmem + (uint32_t)(b * 256), dcorr = dmain + (uint32_t)L::CORR_COL;
                // descriptors of slot 0; a slot's are these plus its offset
                // (the 14-bit address field holds every shared address >> 4)
                const uint64_t da0 = sdesc(base, A_LBO), db0 = sdesc(base + L::BOFF, blbo);
                for (int st = 0; st < L::NSTAGE; ++st) {
                    if (!wait(smem_u32(&bar_afull[slot]), phase, &s_abort)) goto mma_done;
                    if (!wait(smem_u32(&bar_bfull[slot]), phase, &s_abort)) goto mma_done;
                    tc_after();
                    const uint64_t off = (uint64_t)((slot * SLOT) >> 4);
#pragma unroll
                    for (int j = 0; j < L::BPS; ++j) {
                        const int s = st * L::BPS + j;
                        const uint64_t a_hi = da0 + off + (uint64_t)(j * A_BYTES >> 4), a_lo = a_hi + (A_PART >> 4);
                        const uint64_t b_hi = db0 + off + (uint64_t)(j * L::BCHUNK >> 4), b_mid = b_hi + (bpart >> 4);
                        const uint32_t acc = s > 0 ? 1u : 0u;
                        mma(dmain, a_hi, b_hi, id, acc);          // main: hi.hi
                        mma(dcorr, a_hi, b_mid, id, acc);         // corrections
                        mma(dcorr, a_lo, b_hi, id, 1u);
                        if (s < Q::KT) mma(dcorr, a_hi, b_mid + (bpart >> 4), id, 1u);
                    }
                    commit(smem_u32(&bar_empty[slot]));
                    issued = true;
                    if (++slot == NS) slot = 0, phase ^= 1u;
                }
                commit(smem_u32(&bar_tfull[b]));
            }
        mma_done:
            if (issued) {
                // every MMA issued so far has completed once this arrives
                commit(smem_u32(&bar_drain));
                wait_drain(smem_u32(&bar_drain), 0);
            }
        }
    }
    __syncwarp();
    tc_before();
    __syncthreads();
    if (warp == MMA_WARP) {
        tc_after();
        tmem_dealloc(tmem, 512);
    }
    if (tid == 0 && s_abort && A.ps.err) atomicOr(A.ps.err, MBX_STATUS_WAIT_TIMEOUT);
}
