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
// tensor memory by tcgen05.mma (M = 128, N = 240, K = 16), in two passes
// over the N halves (columns 240 h .. 240 h + 239):
//   A operand  the tile's basis values, split hi + lo, written to shared
//              memory by the 128 row threads, K block by K block (again in
//              the second pass);
//   B operand  C split hi + mid + lo, prepared on the host in the canonical
//              no-swizzle K-major layout (8 x 16-byte core matrices), one
//              bulk copy (cp.async.bulk) per K block and N half from the
//              type's image;
//   products   hi.hi into the main accumulator (TMEM columns 0..239),
//              hi.mid + lo.hi, and hi.lo on the first Q::KT blocks, into the
//              correction accumulator (columns 256..495).  FP32 accumulation
//              rounds after every MMA; the main accumulator's partial sums are
//              large next to its final value (the polynomial cancels), so
//              keeping the corrections out of it cuts the rounding steps of
//              the large sums from 98 to 30 per output (9x less error of the
//              summed energy over a liquid box).
// Warps 0-3 are the row threads (thread i owns n-mer i of the tile and TMEM
// lane i): they generate the A blocks and, once a pass's MMAs have
// completed, read both accumulators back (tcgen05.ld) for the energy m . y
// and the gradient 2 sum_j y_j dm_j/dd of that half.  Warp 4 lane 0 issues
// the bulk copies, warp 5 lane 0 the MMAs; warp 5 also owns the TMEM
// allocation.  Shared-memory slots of one K block each (A and B) cycle
// through NS stages with mbarriers:
//   afull[s]  128 row-thread arrivals (A written, proxy-fenced)
//   bfull[s]  the producer's expect_tx + the copy's bytes
//   empty[s]  tcgen05.commit after the block's MMAs
//   tfull     tcgen05.commit after a pass's last block (its half of Y done)
//   tempty    128 row-thread arrivals (that half read out)
// Every wait is bounded (QF_WAIT_NS of %globaltimer): on a timeout the CTA
// sets an abort flag that ends every role's loop, drains its MMAs and
// copies, frees its TMEM and reports MBX_STATUS_WAIT_TIMEOUT in *A.ps.err.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include "holder_kernel.cuh"
#include "nmer_build.h"

namespace qf {

constexpr int NS = 6;                 // shared-memory stages
constexpr int A_PART = 128 * 16 * 2;  // bytes of one FP16 part of an A block (128 rows x K 16)
constexpr int B_PART = 240 * 16 * 2;  // bytes of one FP16 part of a B chunk (240 rows x K 16)
constexpr int A_BYTES = 2 * A_PART;
constexpr int SLOT = 31 * 1024;              // A (8 KiB) + 3 B parts (22.5 KiB), rounded to 1 KiB
static_assert(A_BYTES + 3 * B_PART <= SLOT, "slot too small");
constexpr int PARK = 128 * (36 + 2) * 4;     // first pass's gradient (36 floats) and energy of each row
constexpr int SMEM = NS * SLOT + 1024 + PARK; // + alignment of the first slot
constexpr int THREADS = 192;
constexpr unsigned long long QF_WAIT_NS = 4000000000ull;
// tcgen05 instruction descriptor, kind::f16: F32 accumulator (bits 4-5 = 1),
// F16 A and B (formats 0), both K-major, N = 240 (bits 17-22: N >> 3),
// M = 128 (bits 24-28: M >> 4)
constexpr uint32_t IDESC = (1u << 4) | ((240u >> 3) << 17) | ((128u >> 4) << 24);
constexpr int CORR_COL = 256;         // TMEM column of the correction accumulator

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
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
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
// 8 rows x 16 bytes stored as 128 contiguous bytes), the two core matrices of
// a K block 128 bytes apart (leading byte offset), successive 8-row groups
// 256 bytes apart (stride byte offset); descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           (1ull << 46);
}

// D[tmem] (+)= A[smem] B[smem]^T, one thread issues.
__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
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

// One pass's half of the epilogue: main + correction accumulator of the 240
// columns, then Q::epi on each chunk of 16 (the chunk index a constant).
template <class Q, int H, int NV>
__device__ __forceinline__ double qf_epilogue_half(uint32_t trow, const float (&d)[NV], float (&g)[NV]) {
    double P = 0.0;
#pragma unroll
    for (int cc = 0; cc < Q::KS / 2; ++cc) {
        uint32_t ym[16], yc[16];
        qf::tmem_ld16(trow + (uint32_t)(cc * 16), ym);
        qf::tmem_ld16(trow + (uint32_t)(qf::CORR_COL + cc * 16), yc);
        qf::tmem_wait_ld(ym);
        qf::tmem_wait_ld(yc);
#pragma unroll
        for (int i = 0; i < 16; ++i) ym[i] = __float_as_uint(__uint_as_float(ym[i]) + __uint_as_float(yc[i]));
        P += (double)Q::epi(H * (Q::KS / 2) + cc, ym, d, g);
    }
    return P;
}

// T: the evaluator traits (NVARS); Q: the generated quadratic form
// (<name>_qf.cuh): KS K blocks of 16, the first KT with the third C part,
// stage image offsets/bytes, the row-scale classes, gen(s) and epi(c).
template <class T, class Q>
__global__ void __launch_bounds__(qf::THREADS, 1) qf_eval_kernel(const HolderArgs A) {
    using namespace qf;
    constexpr int NV = T::NVARS;
    __shared__ __align__(8) uint64_t bar_afull[NS], bar_bfull[NS], bar_empty[NS];
    __shared__ __align__(8) uint64_t bar_tfull, bar_tempty, bar_drain;
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
        mbar_init(smem_u32(&bar_tfull), 1);
        mbar_init(smem_u32(&bar_tempty), 128);
        mbar_init(smem_u32(&bar_drain), 1);
        s_abort = 0;
        fence_mbar_init();
    }
    if (warp == 5) {
        tmem_alloc(smem_u32(&s_tmem), 512);
        tmem_relinquish();
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = s_tmem;
    const long n = s_n;
    const long ntiles = (n + 127) / 128;

    if (warp < 4) {
        // ---- row threads: A blocks of both passes, then each pass's epilogue ----
        const int row = tid;
        const uint32_t arow = base + (uint32_t)((row >> 3) * 256 + (row & 7) * 16);
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        float* park_g = reinterpret_cast<float*>(mbx_dyn_smem + (base - smem_u32(mbx_dyn_smem)) + NS * SLOT);
        double* park_p = reinterpret_cast<double*>(park_g + 36 * 128);
        long it = 0, tp = 0;
        for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const long t = tile * 128 + row;
            const bool valid = t < n;
            float d[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) d[v] = valid ? A.ps.dx[v * cap + t] : 0.0f;
            float sc[Q::NT];
            const float rinv = Q::row_scales(d, sc);
            double P = 0.0;
            float g[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) g[v] = 0.0f;
            static_assert(NV <= 36, "park area holds 36 gradient entries");
            for (int h = 0; h < 2; ++h, ++tp) {
                // (both passes generate the same A blocks: the opaque inputs in
                // the stage loop keep the compiler from hoisting them)
#pragma unroll
                for (int s = 0; s < Q::KS; ++s, ++it) {
                    const int slot = (int)(it % NS);
                    const long use = it / NS;
                    const bool free_slot =
                        use == 0 || wait(smem_u32(&bar_empty[slot]), (uint32_t)((use - 1) & 1), &s_abort);
                    if (!__all_sync(0xffffffffu, free_slot)) goto rows_done;   // warp-uniform exit
                    // generate this block here, not earlier (register pressure)
#pragma unroll
                    for (int v = 0; v < NV; ++v) asm volatile("" : "+f"(d[v]));
#pragma unroll
                    for (int k = 0; k < Q::NT; ++k) asm volatile("" : "+f"(sc[k]));
                    uint32_t hi[8], lo[8];
                    Q::gen(s, d, sc, hi, lo);
                    const uint32_t a = arow + (uint32_t)(slot * SLOT);
                    st_shared_v4(a, make_uint4(hi[0], hi[1], hi[2], hi[3]));
                    st_shared_v4(a + 128, make_uint4(hi[4], hi[5], hi[6], hi[7]));
                    st_shared_v4(a + A_PART, make_uint4(lo[0], lo[1], lo[2], lo[3]));
                    st_shared_v4(a + A_PART + 128, make_uint4(lo[4], lo[5], lo[6], lo[7]));
                    fence_proxy_async();
                    mbar_arrive(smem_u32(&bar_afull[slot]));
                }
                // warp-uniform: the TMEM loads below are warp-collective
                if (!__all_sync(0xffffffffu, wait(smem_u32(&bar_tfull), (uint32_t)(tp & 1), &s_abort)))
                    goto rows_done;
                tc_after();
                P += h == 0 ? qf_epilogue_half<Q, 0>(trow, d, g) : qf_epilogue_half<Q, 1>(trow, d, g);
                tc_before();
                mbar_arrive(smem_u32(&bar_tempty));
                if (h == 0) {
                    // park the first pass's sums in shared memory: registers are
                    // short while the second pass generates its A blocks
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        park_g[v * 128 + row] = g[v];
                        g[v] = 0.0f;
                    }
                    park_p[row] = P;
                    P = 0.0;
                }
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) g[v] += park_g[v * 128 + row];
            P += park_p[row];
            if (valid) {
                const float gs = 2.0f * rinv;
#pragma unroll
                for (int v = 0; v < NV; ++v) A.ps.g[v * cap + t] = g[v] * gs;
                A.ps.ep[t] = Q::b0() + P * (double)rinv;
            }
        }
    rows_done:;
    } else if (warp == 4) {
        // ---- producer: one bulk copy of C's (K block, N half) chunk per stage ----
        if (lane == 0) {
            long it = 0;
            for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
                for (int h = 0; h < 2; ++h) {
                    for (int s = 0; s < Q::KS; ++s, ++it) {
                        const int slot = (int)(it % NS);
                        const long use = it / NS;
                        if (use > 0 && !wait(smem_u32(&bar_empty[slot]), (uint32_t)((use - 1) & 1), &s_abort))
                            goto producer_done;
                        const uint32_t bytes = (uint32_t)Q::chunk_bytes(s);
                        const uint32_t bar = smem_u32(&bar_bfull[slot]);
                        mbar_arrive_tx(bar, bytes);
                        bulk_g2s(base + (uint32_t)(slot * SLOT + A_BYTES), Q::image() + Q::chunk_offset(s, h), bytes,
                                 bar);
                    }
                }
            }
        producer_done:
            // copies in flight complete on their own: wait for them before the
            // shared memory goes away (the last use of every slot)
            for (int k = 0; k < NS && k < it; ++k) {
                const long q = it - 1 - k;   // stage iteration of the last copy into slot q % NS
                wait_drain(smem_u32(&bar_bfull[q % NS]), (uint32_t)((q / NS) & 1));
            }
        }
    } else {
        // ---- MMA issuer ----
        if (lane == 0) {
            long it = 0, tp = 0;
            bool issued = false;
            for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
                for (int h = 0; h < 2; ++h, ++tp) {
                    if (tp > 0) {
                        if (!wait(smem_u32(&bar_tempty), (uint32_t)((tp - 1) & 1), &s_abort)) goto mma_done;
                        tc_after();
                    }
                    for (int s = 0; s < Q::KS; ++s, ++it) {
                        const int slot = (int)(it % NS);
                        const uint32_t par = (uint32_t)((it / NS) & 1);
                        if (!wait(smem_u32(&bar_afull[slot]), par, &s_abort)) goto mma_done;
                        if (!wait(smem_u32(&bar_bfull[slot]), par, &s_abort)) goto mma_done;
                        tc_after();
                        const uint32_t sa = base + (uint32_t)(slot * SLOT);
                        const uint32_t sb = sa + A_BYTES;
                        const uint64_t a_hi = sdesc(sa), a_lo = sdesc(sa + A_PART);
                        const uint64_t b_hi = sdesc(sb), b_mid = sdesc(sb + B_PART);
                        const uint32_t acc = s > 0 ? 1u : 0u;
                        mma(tmem, a_hi, b_hi, acc);                      // main: hi.hi
                        mma(tmem + CORR_COL, a_hi, b_mid, acc);          // corrections
                        mma(tmem + CORR_COL, a_lo, b_hi, 1u);
                        if (s < Q::KT) mma(tmem + CORR_COL, a_hi, sdesc(sb + 2 * B_PART), 1u);
                        commit(smem_u32(&bar_empty[slot]));
                        issued = true;
                    }
                    commit(smem_u32(&bar_tfull));
                }
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
    if (warp == 5) {
        tc_after();
        tmem_dealloc(tmem, 512);
    }
    if (tid == 0 && s_abort && A.ps.err) atomicOr(A.ps.err, MBX_STATUS_WAIT_TIMEOUT);
}
