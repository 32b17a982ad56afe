// CSR-stream SpMV with bulk-copy staging (sm_100a): the column and value streams of each
// row block are moved into shared memory by cp.async.bulk (one elected thread, completion
// tracked by an mbarrier), double-buffered, so the next block's matrix data is in flight
// while the CTA gathers x, rounds the products and sums its rows for the current block.
// The arithmetic is exactly k_spmv_rows's: products v*x rounded, rows summed left to right.
//
// Alignment: a bulk copy needs 16-byte aligned source, destination and size, so each copy
// window is widened to 16-byte boundaries ([e0 & ~3, (e1 + 3) & ~3) for the int32 columns,
// [e0 & ~1, (e1 + 1) & ~1) for the doubles) and the block's entries are read at an offset
// of 0..3 (columns) / 0..1 (values). The widened tail reads at most 12 bytes past a matrix
// array; carve_csr (fiim_solver.cu) leaves 16 bytes after the column and value arrays.
//
// Waits are bounded: an mbarrier that does not complete within the limit sets *fault and
// the CTA stops (after a bounded wait for its own copies); the host turns the flag into
// FIIM_ETIMEOUT. Rows longer than TILE take the unstaged path of k_spmv_rows.
#pragma once

#include "fiim_kernels.cuh"

namespace fiim {

constexpr int kPipeSlack = 16;   // extra entries per staged buffer (alignment widening)

template <int TILE>
struct PipeSmem {
    static constexpr int kCols = ((TILE + kPipeSlack) * 4 + 127) / 128 * 128;   // bytes per column buffer
    static constexpr int kVals = (TILE + kPipeSlack) * 8;                         // bytes per value buffer
    static constexpr int kBuf = kCols + kVals;
    static constexpr int kBytes = 2 * kBuf + 64;                                  // + two mbarriers
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bulk copy global -> shared with an L2 evict-first hint: the matrix streams are read once
// per pass and should not push the gathered vectors out of L2.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}
// Bounded wait for the mbarrier phase with the given parity; false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < (1 << 20); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

template <int TILE, typename Epi>
static __global__ void __launch_bounds__(kThreads)
k_spmv_pipe(CsrView<double> M, const int *__restrict__ rb, int nblk, const double *__restrict__ x, Epi epi,
            DState *st, double *__restrict__ partials, int *fault) {
    pdl_enter();
    if (Epi::GATED && st != nullptr && st->done) return;
    using SM = PipeSmem<TILE>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 2 * SM::kBuf);
    const uint32_t bar0 = smem_addr(&bars[0]), bar1 = smem_addr(&bars[1]);
    auto cols = [&](int b) { return reinterpret_cast<int *>(smem + b * SM::kBuf); };
    auto vals = [&](int b) { return reinterpret_cast<double *>(smem + b * SM::kBuf + SM::kCols); };

    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // Stage block `blk` into buffer `b` (thread 0). Returns whether a copy was issued.
    auto stage = [&](int blk, int b) -> bool {
        const int r0 = __ldg(rb + blk), r1 = __ldg(rb + blk + 1);
        const int e0 = __ldg(M.rp + r0), e1 = __ldg(M.rp + r1);
        if (e1 - e0 > TILE || e1 == e0) return false;
        const int c0 = e0 & ~3, c1 = (e1 + 3) & ~3;
        const int v0 = e0 & ~1, v1 = (e1 + 1) & ~1;
        const uint32_t bar = b ? bar1 : bar0;
        mbar_expect_tx(bar, (uint32_t)((c1 - c0) * 4 + (v1 - v0) * 8));
        bulk_g2s(smem_addr(cols(b)), M.ci + c0, (uint32_t)((c1 - c0) * 4), bar);
        bulk_g2s(smem_addr(vals(b)), M.v + v0, (uint32_t)((v1 - v0) * 8), bar);
        return true;
    };
    auto staged = [&](int blk) -> bool {   // same test as stage(), evaluated by every thread
        const int r0 = __ldg(rb + blk), r1 = __ldg(rb + blk + 1);
        const int e0 = __ldg(M.rp + r0), e1 = __ldg(M.rp + r1);
        return !(e1 - e0 > TILE || e1 == e0);
    };

    double red[Epi::NR];
#pragma unroll
    for (int j = 0; j < Epi::NR; ++j) red[j] = 0.0;
    uint32_t phase0 = 0u, phase1 = 0u;   // parity of each buffer's next completion
    int buf = 0;
    if (threadIdx.x == 0 && (int)blockIdx.x < nblk) stage(blockIdx.x, 0);
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x, buf ^= 1) {
        const int nxt = blk + (int)gridDim.x;
        if (threadIdx.x == 0 && nxt < nblk) stage(nxt, buf ^ 1);
        const int r0 = __ldg(rb + blk), r1 = __ldg(rb + blk + 1);
        const int e0 = __ldg(M.rp + r0), e1 = __ldg(M.rp + r1);
        if (staged(blk)) {
            const uint32_t cur = buf ? phase1 : phase0;
            const bool ok = mbar_wait(buf ? bar1 : bar0, cur);
            if (buf) phase1 ^= 1u;
            else phase0 ^= 1u;
            if (__syncthreads_or(!ok)) {
                // A copy did not complete in time: flag it, give this buffer's copy and the
                // other buffer's copy one more bounded wait each, and stop this CTA, so that
                // no copy is left writing into shared memory it no longer owns.
                if (threadIdx.x == 0) {
                    atomicExch(fault, 1);
                    if (!ok) mbar_wait(buf ? bar1 : bar0, cur);
                    if (nxt < nblk && staged(nxt)) mbar_wait(buf ? bar0 : bar1, buf ? phase0 : phase1);
                }
                return;
            }
            const int *cs = cols(buf) + (e0 & 3);
            double *vs = vals(buf) + (e0 & 1);
            const int len = e1 - e0;
#pragma unroll 4
            for (int q = (int)threadIdx.x; q < len; q += kThreads) vs[q] = __dmul_rn(vs[q], ldx(x + cs[q]));
            __syncthreads();
            const int r = r0 + (int)threadIdx.x;
            if (r < r1) {
                const int b = __ldg(M.rp + r) - e0, e = __ldg(M.rp + r + 1) - e0;
                double s = 0.0;
                for (int k = b; k < e; ++k) s = __dadd_rn(s, vs[k]);
                epi.emit(r, s, red);
            }
            // The generic-proxy writes above must be ordered before the next bulk copy into
            // this buffer (two blocks later).
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        } else if (e1 > e0) {
            // Long row (block of one row with more than TILE entries): unstaged, in order.
            double *prod = vals(buf);
            double s = 0.0;
            for (int c0 = e0; c0 < e1; c0 += TILE) {
                const int c1 = min(c0 + TILE, e1);
                for (int e = c0 + (int)threadIdx.x; e < c1; e += kThreads)
                    prod[e - c0] = __dmul_rn(ldm(M.v + e), ldx(x + ldi(M.ci + e)));
                __syncthreads();
                if (threadIdx.x == 0)
                    for (int k = 0; k < c1 - c0; ++k) s = __dadd_rn(s, prod[k]);
                __syncthreads();
            }
            if (threadIdx.x == 0) epi.emit(r0, s, red);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        } else {
            // Empty rows: every row of the block sums to zero.
            const int r = r0 + (int)threadIdx.x;
            if (r < r1) epi.emit(r, 0.0, red);
        }
    }
    pdl_release();
    if constexpr (Epi::REDUCES) grid_reduce<Epi::NR>(red, partials, st, epi);
}

}  // namespace fiim
