// Kernels of the learned surrogate (include/flysurrogate.h): a BF16 tensor-core GEMM with fused
// epilogues (bias, GELU, GELU gradient, transposed copies for the backward pass), the Poisson
// negative log-likelihood, column sums (bias gradients), Adam, and FP32 -> BF16 conversion.
//
// Every GEMM of the MLP's training step is written as C = A * B^T with both operands stored
// K-contiguous (the forward pass keeps transposed copies of activations and weights for the
// backward pass), so one kernel serves them all. Three forms: k_gemm_tma (the default: tcgen05
// MMAs, accumulator in TMEM, operands by TMA with the 128-byte swizzle), k_gemm_tc (the same with
// cp.async staging, for operands TMA cannot describe) and k_gemm (warp-level BF16 m16n8k16 MMAs
// on 128 x 64 tiles from padded shared memory, kept as the comparison).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include <cstdint>

#include "../../include/flybrain.h"
#include "../../include/flysurrogate.h"

namespace fb {
void set_last_error(const char* msg);
}

namespace {

constexpr int BM = 128, BN = 64, BK = 32, PADK = BK + 8;

__device__ __forceinline__ uint16_t f2bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * expf(-0.5f * z * z) * 0.39894228040143268f;
}

// 8 consecutive bf16 of row `row` from column k (zero outside [0, rows) x [0, K))
__device__ __forceinline__ void load8(const uint16_t* X, int row, int k, int rows, int K, int ld, uint16_t* dst)
{
    if (row < rows && k + 8 <= K) {
        *reinterpret_cast<uint4*>(dst) = __ldg(reinterpret_cast<const uint4*>(X + (int64_t)row * ld + k));
    } else {
#pragma unroll
        for (int u = 0; u < 8; u++) dst[u] = (row < rows && k + u < K) ? X[(int64_t)row * ld + k + u] : (uint16_t)0;
    }
}

__device__ __forceinline__ uint32_t lds32(const uint16_t* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

struct Epi {
    int32_t mode, ldo, ldo_t;
    const float* bias;
    const float* zin;
    float* out_f32;
    uint16_t* out_bf16;
    uint16_t* out_bf16_t;
};

__device__ __forceinline__ void epilogue(const Epi& e, int M, int N, int i, int j, float v)
{
    if (i >= M || j >= N) return;
    const int64_t o = (int64_t)i * e.ldo + j;
    switch (e.mode) {
    case FS_EPI_F32: e.out_f32[o] = v; break;
    case FS_EPI_BIAS_F32: e.out_f32[o] = v + e.bias[j]; break;
    case FS_EPI_BIAS_GELU: {
        const float z = v + e.bias[j];
        e.out_f32[o] = z;
        const uint16_t h = f2bf(gelu(z));
        e.out_bf16[o] = h;
        if (e.out_bf16_t) e.out_bf16_t[(int64_t)j * e.ldo_t + i] = h;
        break;
    }
    default: {   // FS_EPI_GELU_GRAD
        const uint16_t d = f2bf(v * gelu_grad(e.zin[o]));
        e.out_bf16[o] = d;
        if (e.out_bf16_t) e.out_bf16_t[(int64_t)j * e.ldo_t + i] = d;
    }
    }
}

__global__ void __launch_bounds__(256) k_gemm(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B, int M,
                                              int N, int K, int lda, int ldb, Epi e)
{
    __shared__ __align__(16) uint16_t As[BM][PADK];
    __shared__ __align__(16) uint16_t Bs[BN][PADK];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const int wm = warp & 3, wn = warp >> 2;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += BK) {
        for (int c = tid; c < BM * 4; c += 256) load8(A, m0 + (c >> 2), k0 + (c & 3) * 8, M, K, lda, &As[c >> 2][(c & 3) * 8]);
        for (int c = tid; c < BN * 4; c += 256) load8(B, n0 + (c >> 2), k0 + (c & 3) * 8, N, K, ldb, &Bs[c >> 2][(c & 3) * 8]);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int r = wm * 32 + i * 16 + g;
                a[i][0] = lds32(&As[r][kk + 2 * t4]);
                a[i][1] = lds32(&As[r + 8][kk + 2 * t4]);
                a[i][2] = lds32(&As[r][kk + 2 * t4 + 8]);
                a[i][3] = lds32(&As[r + 8][kk + 2 * t4 + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = wn * 32 + j * 8 + g;
                b[j][0] = lds32(&Bs[c][kk + 2 * t4]);
                b[j][1] = lds32(&Bs[c][kk + 2 * t4 + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int r = m0 + wm * 32 + i * 16 + g, c = n0 + wn * 32 + j * 8 + 2 * t4;
            epilogue(e, M, N, r, c, acc[i][j][0]);
            epilogue(e, M, N, r, c + 1, acc[i][j][1]);
            epilogue(e, M, N, r + 8, c, acc[i][j][2]);
            epilogue(e, M, N, r + 8, c + 1, acc[i][j][3]);
        }
}

// ---------------------------------------------------------------------------------------------
// The same GEMM on the 5th-generation tensor cores: tcgen05.mma (kind::f16, BF16 in, FP32
// accumulate) issued by one thread, operands in shared memory in the K-major no-swizzle
// core-matrix layout (8 rows x 16 bytes per core matrix), the 128 x BN accumulator in tensor memory
// (TMEM), read back with tcgen05.ld for the fused epilogue. Four shared-memory stages filled by
// cp.async: later K tiles load while the tensor cores work on the current one (a stage is
// refilled once tcgen05.commit's mbarrier shows its MMAs done).
// ---------------------------------------------------------------------------------------------
constexpr int TC_BM = 128, TC_BK = 64, TC_THREADS = 128, TC_STAGES = 4;
constexpr long long TC_WAIT_CYCLES = 4000000000LL;            // bounded waits (~2 s)

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance between the two 8-column
// halves of a K=16 slice, sbo = byte distance between 8-row groups
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);   // version 1, base offset 0, no swizzle
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity)
{
    const long long t0 = clock64();
    uint32_t done = 0;
    while (!done) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (!done && clock64() - t0 > TC_WAIT_CYCLES) return false;
    }
    return true;
}

// 16-byte global -> shared copy without a register round trip (zero-filled outside the matrix)
__device__ __forceinline__ void cp_async16(void* dst, const uint16_t* X, int row, int k, int rows, int K, int ld)
{
    if (row < rows && k + 8 <= K) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(su32(dst)), "l"(X + (int64_t)row * ld + k)
                     : "memory");
    } else {
        uint16_t tmp[8];
#pragma unroll
        for (int u = 0; u < 8; u++) tmp[u] = (row < rows && k + u < K) ? X[(int64_t)row * ld + k + u] : (uint16_t)0;
        *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(tmp);
    }
}

template <int BN>
__global__ void __launch_bounds__(TC_THREADS) k_gemm_tc(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                         int M, int N, int K, int lda, int ldb, Epi e)
{
    constexpr int A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2, STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ __align__(8) uint64_t mbar[TC_STAGES];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&mbar[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // instruction descriptor: FP32 accumulate (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1),
    // both K-major, N >> 3 at bit 17, M >> 4 at bit 24
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
    const int nk = (K + TC_BK - 1) / TC_BK;
    // one K tile -> stage st: 16-byte chunks (row r, k-chunk kc) in the core-matrix layout
    auto load_tile = [&](int kt) {
        uint8_t* sa = sm + (kt % TC_STAGES) * STAGE;
        uint8_t* sb = sa + A_BYTES;
        const int k0 = kt * TC_BK;
        for (int c = tid; c < TC_BM * 8; c += TC_THREADS) {
            const int r = c >> 3, kc = c & 7;
            cp_async16(sa + (kc * TC_BM + r) * 16, A, m0 + r, k0 + kc * 8, M, K, lda);
        }
        for (int c = tid; c < BN * 8; c += TC_THREADS) {
            const int r = c >> 3, kc = c & 7;
            cp_async16(sb + (kc * BN + r) * 16, B, n0 + r, k0 + kc * 8, N, K, ldb);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    bool ok = true;
    for (int kt = 0; kt < TC_STAGES - 1; kt++) {
        if (kt < nk) load_tile(kt);
        else asm volatile("cp.async.commit_group;" ::: "memory");        // keep the group count uniform
    }
    for (int kt = 0; kt < nk; kt++) {
        const int st = kt % TC_STAGES;
        asm volatile("cp.async.wait_group %0;" ::"n"(TC_STAGES - 2) : "memory");   // tile kt has landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");      // generic writes -> tensor-core reads
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint8_t* sa = sm + st * STAGE;
            uint8_t* sb = sa + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; kk++) {
                const uint64_t ad = smem_desc(su32(sa) + kk * 2 * TC_BM * 16, TC_BM * 16, 128);
                const uint64_t bd = smem_desc(su32(sb) + kk * 2 * BN * 16, BN * 16, 128);
                const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(&mbar[st]))
                         : "memory");
        }
        // refill the stage the previous tile used once its MMAs are done
        const int nxt = kt + TC_STAGES - 1;
        if (nxt < nk) {
            if (kt >= 1) {
                const int ps = (kt - 1) % TC_STAGES;
                ok = tc_wait(su32(&mbar[ps]), (uint32_t)(((kt - 1) / TC_STAGES) & 1)) && ok;
            }
            load_tile(nxt);
        } else {
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // the last commit covers every MMA issued before it
    ok = tc_wait(su32(&mbar[(nk - 1) % TC_STAGES]), (uint32_t)(((nk - 1) / TC_STAGES) & 1)) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w holds rows 32w..32w+31 (TMEM lanes), 16 columns per load
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t v[16];
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (ok) {
#pragma unroll
            for (int j = 0; j < 16; j++) epilogue(e, M, N, row, n0 + c0 + j, __uint_as_float(v[j]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------------------------
// The tcgen05 GEMM fed by the Tensor Memory Accelerator: one thread issues each K tile of A (128 rows)
// and B (BN rows) as two 2-D TMA loads (64 bf16 = 128 bytes of K per row, 128-byte swizzle, zeros
// outside the matrices) into a ring of TMA_STAGES shared-memory stages; one thread issues the
// tensor-core MMAs from swizzled K-major descriptors as each stage lands and releases the stage with
// tcgen05.commit; all four warps then read the accumulator from TMEM for the epilogue. No cluster
// multicast anywhere. Every wait is bounded; after a timeout no result is written.
//
// Split K (gridDim.z = S > 1, launched as clusters of 1 x 1 x S blocks): block z of a cluster
// accumulates K tiles [z * nk / S, (z + 1) * nk / S) of the same output tile, writes its FP32
// partial to its own shared memory (the drained stage ring), and after a cluster barrier each block
// sums its 1/S share of the tile's elements over the S partials in the order z = 0 .. S-1 through
// distributed shared memory (ld.shared::cluster), then applies the epilogue with consecutive
// threads on consecutive columns. The sum order is fixed, so a result depends on S and never on
// scheduling. A second cluster barrier keeps every block's shared memory alive until all reads end.
// ---------------------------------------------------------------------------------------------
constexpr int TMA_STAGES = 4;
constexpr int MAX_SPLIT = 8;                 // portable cluster size

// generic-proxy accesses of shared memory after (or before) the tensor-core / TMA proxy's
__device__ __forceinline__ void fence_async_to_generic() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// the shared-memory address `local` of this block, as seen in block `rank` of the cluster
__device__ __forceinline__ uint32_t map_rank(uint32_t local, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}
__device__ __forceinline__ float ld_cluster_f32(uint32_t addr)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ int ld_cluster_s32(uint32_t addr)
{
    int v;
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

// shared-memory descriptor, K-major with the 128-byte swizzle: 8-row atoms of 1024 bytes (SBO), the
// K offset inside the 128-byte row added to the start address (LBO unused: 16 bytes)
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(mbar)
        : "memory");
}

template <int BN>
__global__ void __launch_bounds__(TC_THREADS) k_gemm_tma(const __grid_constant__ CUtensorMap mapA,
                                                          const __grid_constant__ CUtensorMap mapB, int M, int N, int K,
                                                          Epi e)
{
    constexpr int A_BYTES = TC_BM * 128, B_BYTES = BN * 128, STAGE = A_BYTES + B_BYTES;
    static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "stages must keep 1024-byte alignment");
    constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
    extern __shared__ uint8_t dyn[];
    __shared__ __align__(8) uint64_t full[TMA_STAGES], empty[TMA_STAGES], done;
    __shared__ uint32_t s_tmem;
    __shared__ int s_ok, s_issued, s_used;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;
    const uint32_t base = (su32(dyn) + 1023u) & ~1023u;            // the swizzle needs 1024-byte atoms
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < TMA_STAGES; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&empty[s])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&done)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
        s_issued = 0;
        s_used = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
    // this block's K tiles: all of them, or its share of a split (every share has at least one)
    const int S = (int)gridDim.z, z = S > 1 ? (int)cluster_rank() : 0;
    const int nk_all = (K + 63) / 64, kt0 = (int)((int64_t)z * nk_all / S);
    const int nk = (int)((int64_t)(z + 1) * nk_all / S) - kt0;
    if (tid == 0) {                                   // producer: the TMA loads
        int kt = 0;
        for (; kt < nk; kt++) {
            const int s = kt % TMA_STAGES;
            if (kt >= TMA_STAGES && !tc_wait(su32(&empty[s]), (uint32_t)((kt / TMA_STAGES - 1) & 1))) {
                s_ok = 0;
                break;
            }
            const uint32_t sa = base + s * STAGE;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(&full[s])), "r"(STAGE)
                         : "memory");
            tma_load_2d(sa, &mapA, (kt0 + kt) * 64, m0, su32(&full[s]));
            tma_load_2d(sa + A_BYTES, &mapB, (kt0 + kt) * 64, n0, su32(&full[s]));
        }
        s_issued = kt;
    } else if (tid == 32) {                           // the MMA issuer
        int kt = 0;
        for (; kt < nk; kt++) {
            const int s = kt % TMA_STAGES;
            if (!tc_wait(su32(&full[s]), (uint32_t)((kt / TMA_STAGES) & 1))) {
                s_ok = 0;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = base + s * STAGE, sb = sa + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {              // K = 16 per MMA: 32 bytes along the swizzled row
                const uint64_t ad = smem_desc_sw128(sa + kk * 32), bd = smem_desc_sw128(sb + kk * 32);
                const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             su32(&empty[s]))
                         : "memory");
        }
        s_used = kt;
        // the last commit covers every MMA issued before it
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(&done))
                     : "memory");
    }
    const bool fin = tc_wait(su32(&done), 0u);
    // loads still in flight after a timeout land before the stage ring is reused or the block
    // leaves (bounded)
    if (tid == 0)
        for (int kt = s_used; kt < s_issued; kt++) (void)tc_wait(su32(&full[kt % TMA_STAGES]), (uint32_t)((kt / TMA_STAGES) & 1));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    const bool ok = fin && s_ok != 0;
    const int row = m0 + warp * 32 + lane;
    constexpr int PSTR = BN + 1;                      // partial rows padded: a warp's 32 rows hit 32 banks
    float* part = reinterpret_cast<float*>(dyn + (base - su32(dyn)));
    if (S > 1) fence_async_to_generic();
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t v[16];
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (S > 1) {
#pragma unroll
            for (int j = 0; j < 16; j++) part[(warp * 32 + lane) * PSTR + c0 + j] = __uint_as_float(v[j]);
        } else if (ok) {
#pragma unroll
            for (int j = 0; j < 16; j++) epilogue(e, M, N, row, n0 + c0 + j, __uint_as_float(v[j]));
        }
    }
    if (S > 1) {
        if (tid == 0) s_ok = ok ? 1 : 0;
        cluster_sync_all();                           // every partial is written and visible
        bool all_ok = true;
        for (int r = 0; r < S; r++) all_ok = all_ok && ld_cluster_s32(map_rank(su32(&s_ok), (uint32_t)r)) != 0;
        constexpr int TILE = TC_BM * BN;
        const int chunk = (TILE + S - 1) / S, lo = z * chunk, hi = min(TILE, lo + chunk);
        const uint32_t pbase = su32(part);
        for (int el = lo + tid; el < hi; el += TC_THREADS) {
            const int r = el / BN, c = el - r * BN;
            const uint32_t off = (uint32_t)(r * PSTR + c) * 4u;
            float acc = 0.0f;
            for (int q = 0; q < S; q++) acc += ld_cluster_f32(map_rank(pbase + off, (uint32_t)q));
            if (all_ok) epilogue(e, M, N, m0 + r, n0 + c, acc);
        }
        cluster_sync_all();                           // no block leaves while another reads its partial
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

__global__ void k_poisson(const float* z, const float* y, int M, int D, double* loss, uint16_t* dz, int ldd, uint16_t* dz_t)
{
    __shared__ double part[8];
    double s = 0.0;
    const int64_t total = (int64_t)M * D;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
        const float zz = z[p], yy = y[p];
        const float ez = expf(zz);
        s += (double)ez - (double)yy * (double)zz;
        const uint16_t d = f2bf((ez - yy) / (float)M);
        const int64_t m = p / D, k = p - m * D;
        dz[m * ldd + k] = d;
        if (dz_t) dz_t[k * M + m] = d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        atomicAdd(loss, t);
    }
}

// column sums: a cluster of S blocks per 32 columns, block z of it over rows [z M / S, (z + 1) M / S)
// with its 32 warps on interleaved rows (lanes on consecutive columns); the warps' partials, then
// the blocks' (through distributed shared memory), added in a fixed order
__global__ void __launch_bounds__(1024) k_colsum(const uint16_t* X, int M, int N, int ld, float* grad)
{
    __shared__ float part[32][33];
    __shared__ float tot[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, j = blockIdx.x * 32 + lane;
    const int S = (int)gridDim.y, z = S > 1 ? (int)cluster_rank() : 0;
    const int r0 = (int)((int64_t)z * M / S), r1 = (int)((int64_t)(z + 1) * M / S);
    float s = 0.0f;
    if (j < N) {
#pragma unroll 8
        for (int i = r0 + w; i < r1; i += 32) s += __bfloat162float(__ushort_as_bfloat16(X[(int64_t)i * ld + j]));
    }
    part[w][lane] = s;
    __syncthreads();
    if (w == 0) {
        float t = 0.0f;
        for (int q = 0; q < 32; q++) t += part[q][lane];
        tot[lane] = t;
    }
    if (S > 1) cluster_sync_all();
    else __syncthreads();
    if (z == 0 && w == 0 && j < N) {
        float t = 0.0f;
        for (int q = 0; q < S; q++) t += S > 1 ? ld_cluster_f32(map_rank(su32(&tot[lane]), (uint32_t)q)) : tot[lane];
        grad[j] = t;
    }
    if (S > 1) cluster_sync_all();                    // no block leaves while block 0 reads its sums
}

// Adam on one element; returns the new weight
__device__ __forceinline__ float adam_one(float* w, const float* g, float* m, float* v, int64_t p, float lr, float b1,
                                          float b2, float eps, float c1, float c2)
{
    const float gg = g[p];
    const float mm = b1 * m[p] + (1.0f - b1) * gg;
    const float vv = b2 * v[p] + (1.0f - b2) * gg * gg;
    m[p] = mm;
    v[p] = vv;
    const float ww = w[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    w[p] = ww;
    return ww;
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2, uint16_t* wb)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const uint16_t h = f2bf(adam_one(w, g, m, v, p, lr, b1, b2, eps, c1, c2));
        if (wb) wb[p] = h;
    }
}

// The same on a rows x cols weight in 32 x 32 tiles (block 32 x 8), with its transposed bf16 copy
// written through shared memory so that both copies are stored along rows
__global__ void k_adam_t(float* w, const float* g, float* m, float* v, float lr, float b1, float b2, float eps, float c1,
                         float c2, uint16_t* wb, uint16_t* wbt, int rows, int cols, int ldt)
{
    __shared__ uint16_t tile[32][34];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32, tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        if (r < rows && c < cols) {
            const int64_t p = (int64_t)r * cols + c;
            const uint16_t h = f2bf(adam_one(w, g, m, v, p, lr, b1, b2, eps, c1, c2));
            if (wb) wb[p] = h;
            tile[k][tx] = h;
        }
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;
        if (r < rows && c < cols) wbt[(int64_t)c * ldt + r] = tile[tx][k];
    }
}

__global__ void k_to_bf16(const float* x, int64_t n, uint16_t* out)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x)
        out[p] = f2bf(x[p]);
}

// FP32 -> bf16 of a rows x cols matrix in 32 x 32 tiles (block 32 x 8): the plain copy (when `out`)
// and the transposed one, both stored along rows
__global__ void k_to_bf16_t(const float* x, uint16_t* out, uint16_t* out_t, int rows, int cols, int ldt)
{
    __shared__ uint16_t tile[32][34];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32, tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        if (r < rows && c < cols) {
            const int64_t p = (int64_t)r * cols + c;
            const uint16_t h = f2bf(x[p]);
            if (out) out[p] = h;
            tile[k][tx] = h;
        }
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;
        if (r < rows && c < cols) out_t[(int64_t)c * ldt + r] = tile[tx][k];
    }
}

int g_gemm_kind = FS_GEMM_TCGEN05_TMA;

int fail(const char* msg)
{
    fb::set_last_error(msg);
    return FB_ERR_ARG;
}

int cuda_status()
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return FB_OK;
    fb::set_last_error(cudaGetErrorString(e));
    return FB_ERR_CUDA;
}

template <int BN>
int launch_tc(const uint16_t* A, const uint16_t* B, int M, int N, int K, int lda, int ldb, const Epi& e, cudaStream_t st)
{
    constexpr int smem = TC_STAGES * (TC_BM * TC_BK * 2 + BN * TC_BK * 2);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_gemm_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return cuda_status();
        attr = true;
    }
    dim3 grid((N + BN - 1) / BN, (M + TC_BM - 1) / TC_BM);
    k_gemm_tc<BN><<<grid, TC_THREADS, smem, st>>>(A, B, M, N, K, lda, ldb, e);
    return cuda_status();
}

// A K-contiguous bf16 matrix (rows x K, row stride ld) as a TMA tensor map: boxes of 64 x box_rows
// elements with the 128-byte swizzle. False when the driver entry point is missing or rejects it.
bool tensor_map(CUtensorMap* map, const uint16_t* X, int rows, int K, int ld, int box_rows)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&encode, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            encode = nullptr;
        (void)cudaGetLastError();
    }
    if (!encode || ((uintptr_t)X & 15) || ld % 8) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
    const cuuint32_t elem[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t*>(X), dims, strides, box, elem,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int g_gemm_split = MAX_SPLIT;

// K split of a TMA GEMM: enough blocks to fill the SMs at `per_sm` blocks each (the kernel's
// shared-memory occupancy), at least eight 64-deep K tiles per block (below that the cluster
// reduction costs more than the split saves), at most the set limit
int split_for(int tiles, int K, int per_sm)
{
    if (g_gemm_split <= 1) return 1;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        sms = 148;
    }
    const int nk = (K + 63) / 64;
    return std::max(1, std::min({g_gemm_split, (per_sm * sms) / std::max(tiles, 1), nk / 8}));
}

// 1: launched; 0: not eligible for TMA (the caller falls back); negative: an error code
template <int BN>
int launch_tma(const uint16_t* A, const uint16_t* B, int M, int N, int K, int lda, int ldb, const Epi& e, cudaStream_t st)
{
    CUtensorMap ma, mb;
    if (!tensor_map(&ma, A, M, K, lda, TC_BM) || !tensor_map(&mb, B, N, K, ldb, BN)) return 0;
    constexpr int smem = TMA_STAGES * (TC_BM * 128 + BN * 128) + 1024;
    static_assert(TC_BM * (BN + 1) * 4 <= TMA_STAGES * (TC_BM * 128 + BN * 128), "split-K partials fit the stage ring");
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_gemm_tma<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return -cuda_status();
        attr = true;
    }
    const unsigned gx = (N + BN - 1) / BN, gy = (M + TC_BM - 1) / TC_BM;
    const int S = split_for((int)(gx * gy), K, smem * 2 <= 227 * 1024 ? 2 : 1);
    if (S == 1) {
        k_gemm_tma<BN><<<dim3(gx, gy), TC_THREADS, smem, st>>>(ma, mb, M, N, K, e);
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(gx, gy, (unsigned)S);
        cfg.blockDim = dim3(TC_THREADS);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 1;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = (unsigned)S;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (cudaLaunchKernelEx(&cfg, k_gemm_tma<BN>, ma, mb, M, N, K, e) != cudaSuccess) return -cuda_status();
    }
    const int rc = cuda_status();
    return rc == FB_OK ? 1 : -rc;
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

extern "C" int fs_gemm(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, int32_t lda, int32_t ldb,
                       int32_t epi, const float* bias, const float* zin, float* out_f32, uint16_t* out_bf16,
                       uint16_t* out_bf16_t, int32_t ldo, int32_t ldo_t, void* stream)
{
    if (!A || !B || M <= 0 || N <= 0 || K <= 0) return fail("fs_gemm: bad operands");
    if (lda % 8 || ldb % 8 || lda < K || ldb < K) return fail("fs_gemm: lda, ldb must be multiples of 8 and >= K");
    if (epi < FS_EPI_F32 || epi > FS_EPI_GELU_GRAD) return fail("fs_gemm: unknown epilogue");
    if ((epi == FS_EPI_F32 || epi == FS_EPI_BIAS_F32 || epi == FS_EPI_BIAS_GELU) && !out_f32)
        return fail("fs_gemm: out_f32 needed");
    if ((epi == FS_EPI_BIAS_F32 || epi == FS_EPI_BIAS_GELU) && !bias) return fail("fs_gemm: bias needed");
    if ((epi == FS_EPI_BIAS_GELU || epi == FS_EPI_GELU_GRAD) && !out_bf16) return fail("fs_gemm: out_bf16 needed");
    if (epi == FS_EPI_GELU_GRAD && !zin) return fail("fs_gemm: zin needed");
    Epi e{epi, ldo, ldo_t, bias, zin, out_f32, out_bf16, out_bf16_t};
    cudaStream_t st = (cudaStream_t)stream;
    if (g_gemm_kind == FS_GEMM_TCGEN05_TMA) {
        const int rc = N <= 16 ? launch_tma<16>(A, B, M, N, K, lda, ldb, e, st) : launch_tma<64>(A, B, M, N, K, lda, ldb, e, st);
        if (rc != 0) return rc > 0 ? FB_OK : -rc;
    }
    if (g_gemm_kind == FS_GEMM_TCGEN05 || g_gemm_kind == FS_GEMM_TCGEN05_TMA) {
        if (N <= 16) return launch_tc<16>(A, B, M, N, K, lda, ldb, e, st);
        return launch_tc<64>(A, B, M, N, K, lda, ldb, e, st);
    }
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    k_gemm<<<grid, 256, 0, st>>>(A, B, M, N, K, lda, ldb, e);
    return cuda_status();
}

extern "C" int fs_gemm_kind(int32_t kind)
{
    if (kind != FS_GEMM_MMA_SYNC && kind != FS_GEMM_TCGEN05 && kind != FS_GEMM_TCGEN05_TMA && kind != -1)
        return fail("fs_gemm_kind: unknown kind");
    const int old = g_gemm_kind;
    if (kind >= 0) g_gemm_kind = kind;
    return old;
}

extern "C" int fs_gemm_split(int32_t max_split)
{
    if (max_split == 0 || max_split < -1 || max_split > MAX_SPLIT) return -fail("fs_gemm_split: 1 .. 8, or -1 to keep");
    const int old = g_gemm_split;
    if (max_split > 0) g_gemm_split = max_split;
    return old;
}

extern "C" int fs_poisson_nll(const float* z, const float* y, int32_t M, int32_t D, double* loss_sum, uint16_t* dz,
                              int32_t ldd, uint16_t* dz_t, void* stream)
{
    if (!z || !y || !loss_sum || !dz || M <= 0 || D <= 0 || ldd < D) return fail("fs_poisson_nll: bad arguments");
    k_poisson<<<blocks_for((int64_t)M * D), 256, 0, (cudaStream_t)stream>>>(z, y, M, D, loss_sum, dz, ldd, dz_t);
    return cuda_status();
}

extern "C" int fs_colsum(const uint16_t* X, int32_t M, int32_t N, int32_t ld, float* grad, void* stream)
{
    if (!X || !grad || M <= 0 || N <= 0 || ld < N) return fail("fs_colsum: bad arguments");
    const int S = std::min(MAX_SPLIT, std::max(1, M / 256));    // >= 8 rows per warp
    if (S == 1) {
        k_colsum<<<(N + 31) / 32, 1024, 0, (cudaStream_t)stream>>>(X, M, N, ld, grad);
        return cuda_status();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((N + 31) / 32), (unsigned)S);
    cfg.blockDim = dim3(1024);
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 1;
    at[0].val.clusterDim.y = (unsigned)S;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_colsum, X, M, N, ld, grad) != cudaSuccess) return cuda_status();
    return cuda_status();
}

extern "C" int fs_adam(float* w, const float* grad, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                       float eps, int32_t t, uint16_t* w_bf16, uint16_t* w_bf16_t, int32_t rows, int32_t cols,
                       int32_t ldt, void* stream)
{
    if (!w || !grad || !m || !v || n <= 0 || t < 1) return fail("fs_adam: bad arguments");
    if (w_bf16_t && (rows <= 0 || cols <= 0 || rows > 65535 * 32 || (int64_t)rows * cols != n || ldt < rows))
        return fail("fs_adam: the transposed copy needs 0 < rows <= 2097120, rows * cols == n and ldt >= rows");
    const float c1 = 1.0f - powf(beta1, (float)t), c2 = 1.0f - powf(beta2, (float)t);
    if (w_bf16_t) {
        const dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
        k_adam_t<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(w, grad, m, v, lr, beta1, beta2, eps, c1, c2, w_bf16,
                                                                 w_bf16_t, rows, cols, ldt);
    } else {
        k_adam<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(w, grad, m, v, n, lr, beta1, beta2, eps, c1, c2, w_bf16);
    }
    return cuda_status();
}

extern "C" int fs_to_bf16(const float* x, int64_t n, uint16_t* out, uint16_t* out_t, int32_t rows, int32_t cols,
                          int32_t ldt, void* stream)
{
    if (!x || n <= 0 || (!out && !out_t)) return fail("fs_to_bf16: bad arguments");
    if (out_t && (rows <= 0 || cols <= 0 || rows > 65535 * 32 || (int64_t)rows * cols != n || ldt < rows))
        return fail("fs_to_bf16: the transposed copy needs 0 < rows <= 2097120, rows * cols == n and ldt >= rows");
    if (out_t) {
        const dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
        k_to_bf16_t<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(x, out, out_t, rows, cols, ldt);
    } else {
        k_to_bf16<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(x, n, out);
    }
    return cuda_status();
}
