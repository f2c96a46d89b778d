// Forward pass of the hash-grid networks on sm_100a's fifth-generation tensor
// cores (tcgen05): inference for the path tracer (guide lobes, radiance-cache
// prediction) and for the network entry points.
//
// A CTA of 128 threads owns a 128-row tile of encoded samples; thread t owns
// row t, which lives in TMEM lane t (warp w accesses lanes 32w..32w+31).  The
// CTA's 128 TMEM columns hold the layer's FP32 accumulator in [0, 64) and its
// BF16 input rows (the MMA's A operand, two values per 32-bit column, lower
// index in the low half) in [64, 64 + K/2).  Per layer each thread stores its
// input row into TMEM (`tcgen05.st.32x32b`), one thread issues K/16
// `tcgen05.mma.cta_group::1.kind::f16` (M = 128, N = the layer's outputs,
// K = 16; A from tensor memory, B = the weights from shared memory) and
// commits them to an mbarrier, and thread t reads row t of the accumulator
// (`tcgen05.ld.32x32b`), applies ReLU and rounds to BF16: the next layer's
// input row, which goes straight back to TMEM.  Activations never pass
// through shared memory, so a CTA needs only the weights there.  After the
// last layer each thread holds its own row of outputs, so the head (vMF
// lobes, radiance) runs per thread.
//
// The weights use the no-swizzle K-major canonical shared-memory layout:
// 8-row x 16-byte core matrices, rows 16 B apart; the 8-column chunk c of row
// n of layer l (N x K, W[n][k]) at 2 woff(l) + (c N + n) * 16 (LBO = 16 N,
// SBO = 128).  The training kernel (cl_guide.cu) keeps its activation tiles in
// shared memory in the same layout (chunk c of row r at c * 2048 + r * 16),
// because its backward products read them as MN-major operands.
#pragma once

#include "cl_guide.cuh"

namespace clb
{
namespace guide
{
constexpr int      kTcRows    = 128;          // rows per tile (the MMA's M)
constexpr int      kTcThreads = 128;          // one thread per row
constexpr uint32_t kTcChunk   = kTcRows * 16; // bytes of one 8-column chunk of a shared-memory tile (training)
constexpr uint32_t kTcCols    = 128;          // TMEM columns per inference CTA
constexpr uint32_t kTcAcol    = 64;           // first TMEM column of the A operand (accumulator: [0, 64))
constexpr uint32_t kTcTimeout = 0x10u;        // device error flag: a tensor-core wait ran out
static_assert(kTcAcol + kIn / 2 <= kTcCols && kWidth <= int(kTcAcol), "TMEM columns of an inference CTA");

template <class S> struct TcLayout
{
    static constexpr int kWBytes = S::kParams * 2; // canonical-layout BF16 weights
    static constexpr int kBar    = kWBytes;
    static constexpr int kSmem   = kBar + 16;      // + mbarrier and the TMEM address
    static_assert(kWBytes % 16 == 0, "weights: 16-byte chunks");
};

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 in
// bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t tcIdesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(kTcRows >> 4) << 24);
}

// General form: M = 64 or 128, either operand K-major (0) or MN-major (bit
// 15 for A, bit 16 for B).  An MN-major operand in the no-swizzle canonical
// layout stores 8 consecutive M (or N) elements in 16 bytes, 8 such rows of
// consecutive k 16 bytes apart; SBO = the stride of 8-element MN groups and
// LBO = the stride of 8-row k groups.  The K-major tiles of this file,
// viewed this way, are the transposed operands of the training kernel.
__host__ __device__ constexpr uint32_t tcIdescMaj(int m, int n, bool aMN, bool bMN)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(aMN) << 15) | (uint32_t(bMN) << 16) |
           (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

// Shared-memory matrix descriptor: start address, LBO and SBO in 16-byte
// units (bits 0-13, 16-29, 32-45), descriptor version 1 (bits 46-47), base
// offset 0, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t tcDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((addr >> 4) & 0x3fffu) | (uint64_t((lbo >> 4) & 0x3fffu) << 16) |
           (uint64_t((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void tcMma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
                 "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
// The same with A (K-major, 128 rows x 16) in tensor memory at column address a.
__device__ __forceinline__ void tcMmaTs(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d),
                 "r"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tcCommit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes -> visible to the tensor core's reads.
__device__ __forceinline__ void asyncProxyFence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one whole warp; the address lands in shared memory.
__device__ __forceinline__ void tmemAlloc(uint32_t dst, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemFree(uint32_t taddr, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmemLd16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                 "%14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmemWait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 16 consecutive 32-bit columns of this thread's TMEM lane <- v.
__device__ __forceinline__ void tmemSt16(uint32_t taddr, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
                 "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
                 : "memory");
}
__device__ __forceinline__ void tmemWaitSt() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0u;
}
__device__ __forceinline__ uint64_t globalTimerNs()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the mbarrier phase `parity` to complete, for at most about one
// second; false when the wait ran out.
__device__ __forceinline__ bool mbarWait(uint32_t bar, uint32_t parity)
{
    if (mbarTryWait(bar, parity)) return true;
    const uint64_t t0 = globalTimerNs();
    while (!mbarTryWait(bar, parity))
        if (globalTimerNs() - t0 > 1000000000ull) return false;
    return true;
}

// One-dimensional bulk copy (TMA, no multicast) of `bytes` (a multiple of
// 16; both addresses 16-byte aligned) from this GPU's global memory into this
// CTA's shared memory, completing on the mbarrier `bar` (which the issuing
// thread arms with the byte count).
__device__ __forceinline__ void bulkLoad(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Per-CTA setup: weights (canonical layout, global) -> shared memory, the
// mbarrier, and kTcCols TMEM columns (warp 0).  Returns the TMEM address.
template <class S>
__device__ __forceinline__ uint32_t tcSetup(unsigned char* smem, const uint4* __restrict__ wt)
{
    uint4* w = reinterpret_cast<uint4*>(smem);
    for (int i = threadIdx.x; i < TcLayout<S>::kWBytes / 16; i += blockDim.x) w[i] = __ldg(wt + i);
    const uint32_t bar = smemAddr(smem + TcLayout<S>::kBar);
    if (threadIdx.x == 0) mbarInit(bar, 1u);
    if (threadIdx.x < 32) tmemAlloc(bar + 8u, kTcCols);
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    return *reinterpret_cast<volatile uint32_t*>(smem + TcLayout<S>::kBar + 8);
}
__device__ __forceinline__ void tcTeardown(uint32_t tmem)
{
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    if (threadIdx.x < 32) tmemFree(tmem, kTcCols);
}

// Row r of a shared-memory tile (training), 8-column chunk c (16 bytes).
__device__ __forceinline__ uint4* tileChunk(unsigned char* tile, uint32_t row, int c)
{
    return reinterpret_cast<uint4*>(tile + c * kTcChunk + row * 16u);
}

__device__ __forceinline__ uint4 packRelu8(const uint32_t* v)
{
    return make_uint4(packBf16(reluF(__uint_as_float(v[0])), reluF(__uint_as_float(v[1]))),
                      packBf16(reluF(__uint_as_float(v[2])), reluF(__uint_as_float(v[3]))),
                      packBf16(reluF(__uint_as_float(v[4])), reluF(__uint_as_float(v[5]))),
                      packBf16(reluF(__uint_as_float(v[6])), reluF(__uint_as_float(v[7]))));
}

// Forward pass of the tile whose row t is thread t's `in` (the 96 encoded
// inputs as 48 packed BF16 pairs; zero for rows without a sample).  Thread t
// receives row t's outputs.  `phase` is the mbarrier's parity, carried across
// tiles.  Returns false (in every thread) when a tensor-core wait ran out; the
// tile's outputs are then undefined.
template <class S>
__device__ __forceinline__ bool tcForward(unsigned char* smem, uint32_t tmem, const uint32_t (&in)[kIn / 2],
                                          uint32_t& phase, float (&out)[S::kOut])
{
    const uint32_t wS = smemAddr(smem), bar = smemAddr(smem + TcLayout<S>::kBar);
    const uint32_t taddr = tmem + ((threadIdx.x & ~31u) << 16); // this warp's TMEM lanes
    tmemSt16(taddr + kTcAcol, in);
    tmemSt16(taddr + kTcAcol + 16u, in + 16);
    tmemSt16(taddr + kTcAcol + 32u, in + 32);
#pragma unroll 1
    for (int l = 0; l < S::kLayers; ++l)
    {
        tmemWaitSt();
        tcFenceBefore();
        __syncthreads();
        if (threadIdx.x == 0)
        {
            tcFenceAfter();
            const int      K = S::in(l), N = S::out(l);
            const uint32_t idesc = tcIdesc(N), wl = wS + 2u * uint32_t(S::woff(l));
            for (int ks = 0; ks < K / 16; ++ks)
                tcMmaTs(tmem, tmem + kTcAcol + uint32_t(8 * ks),
                        tcDesc(wl + uint32_t(ks * 2 * N * 16), uint32_t(N * 16), 128u), idesc, ks > 0 ? 1u : 0u);
            tcCommit(bar);
        }
        const bool ok = mbarWait(bar, phase);
        phase ^= 1u;
        tcFenceAfter();
        if (!__syncthreads_and(ok)) return false;
        if (l < S::kLayers - 1)
        {
            uint32_t v[kWidth / 16][16];
#pragma unroll
            for (int c = 0; c < kWidth / 16; ++c) tmemLd16(taddr + uint32_t(16 * c), v[c]);
            tmemWait();
            uint32_t a[kWidth / 2];
#pragma unroll
            for (int c = 0; c < kWidth / 16; ++c)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    a[8 * c + j] = packBf16(reluF(__uint_as_float(v[c][2 * j])), reluF(__uint_as_float(v[c][2 * j + 1])));
            tmemSt16(taddr + kTcAcol, a);
            tmemSt16(taddr + kTcAcol + 16u, a + 16);
        }
        else
        {
            uint32_t v[S::kOut / 16][16];
#pragma unroll
            for (int c = 0; c < S::kOut / 16; ++c) tmemLd16(taddr + uint32_t(16 * c), v[c]);
            tmemWait();
#pragma unroll
            for (int c = 0; c < S::kOut / 16; ++c)
#pragma unroll
                for (int j = 0; j < 16; ++j) out[16 * c + j] = __uint_as_float(v[c][j]);
        }
    }
    return true;
}

} // namespace guide
} // namespace clb
