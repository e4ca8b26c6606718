// Persistent engine: one cooperative launch runs all steps of a run for one group of instances.
//
// Instances are independent, so B is split into groups small enough that a group's neuron state
// (v, g f32 + refractory/flag byte = 9 B per instance-neuron) fits in the shared memory of the
// whole GPU (~148 x 200 KB). Each CTA owns a contiguous slice of the group's (instance, neuron)
// pairs and keeps its state in shared memory for the whole run: per step, HBM/L2 traffic is only
// the synaptic-input accumulator (read + clear, staged into shared memory by TMA 1-D bulk
// copies, 3 stages of 16 KB), the CSR rows of spiking neurons and the atomics they scatter.
//
// Per step, every CTA: (U) advances its pairs, compacts spikes into the group's work list;
// (P) scatters the list of the spikes that arrive next step into the other accumulator;
// then a grid barrier (bounded: after ~4 s it raises the timeout flag and every CTA returns).
// U of step t and P of step t touch different accumulators, so one barrier per step suffices
// (two when n_delay == 1, where P needs this step's spikes).
#pragma once
#include "engine.cuh"

namespace fb {

constexpr int PT = 512;                 // threads per CTA
constexpr int STAGE_BYTES = 16384;      // one TMA stage
constexpr int NSTAGE = 3;
constexpr long long BARRIER_TIMEOUT_CYCLES = 8000000000LL;   // ~4 s at 1.9 GHz

struct PersistPlan {
    int32_t group = 0;        // instances per launch (0: engine unavailable)
    int32_t n_groups = 1;
    int32_t ctas = 0;
    int64_t per = 0;          // pairs per CTA (multiple of 16)
    size_t smem = 0;
    int32_t launches_per_run = 0;
};

struct PersistArgs {
    int64_t t0;
    uint32_t step0;
    int32_t steps;
    const uint32_t* kicks;
    int32_t words;
    int32_t* counts;
    int32_t* step_counts;
    uint64_t* step_digest;
    unsigned int* bar;        // zeroed before the launch
    int32_t* abort_flag;      // zeroed before the launch
};

// ---- PTX helpers: mbarrier, TMA 1-D bulk copy, proxy fences, acquire load --------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// global -> shared bulk copy (addresses 16-byte aligned, size a multiple of 16), completion on bar
__device__ __forceinline__ void tma_load_1d(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_volatile_i32(const int32_t* p) { return *reinterpret_cast<const volatile int32_t*>(p); }

// Grid barrier with a bounded wait. Returns true if the run must stop (timeout here or elsewhere).
__device__ __forceinline__ bool grid_barrier(const PersistArgs& A, unsigned int target, int32_t* err, int tag)
{
    __shared__ int s_stop;
    __syncthreads();
    if (threadIdx.x == 0) {
        int stop = 0;
        __threadfence();
        atomicAdd(A.bar, 1u);
        const long long t0 = clock64();
        while (ld_acquire_u32(A.bar) < target) {
            if (ld_volatile_i32(A.abort_flag)) { stop = 1; break; }
            if (clock64() - t0 > BARRIER_TIMEOUT_CYCLES) {
                stop = 1;
                atomicExch(A.abort_flag, 1);
                atomicCAS(err + 1, 0, tag);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        s_stop = stop;
    }
    __syncthreads();
    return s_stop != 0;
}

// Wait for a TMA stage with a bounded spin; on timeout raise the flag and report failure.
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t parity, const PersistArgs& A, int32_t* err, int tag)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > BARRIER_TIMEOUT_CYCLES) {
            atomicExch(A.abort_flag, 1);
            atomicCAS(err + 1, 0, tag);
            return false;
        }
    }
    return true;
}

template <typename AccT, bool RASTER, bool PLASTIC, bool RECORD, int LANES>
__global__ void __launch_bounds__(PT, 1)
    k_persist(const DevNet N, const DevState S, const PersistArgs A, int32_t b0, int32_t G, int32_t q, int64_t per)
{
    extern __shared__ __align__(128) uint8_t smem[];
    constexpr int SP = STAGE_BYTES / (int)sizeof(AccT);    // pairs per stage (multiple of PT)
    AccT* stage = reinterpret_cast<AccT*>(smem);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + NSTAGE * STAGE_BYTES);
    float* sv = reinterpret_cast<float*>(mbar + NSTAGE);
    float* sg = sv + per;
    uint8_t* sr = reinterpret_cast<uint8_t*>(sg + per);    // bits 0-5 refractory, 6 plastic target, 7 ext
    uint8_t* s_active = sr + per;                          // G flags
    const Lif<float>& L = N.L32;
    const int tid = threadIdx.x;
    const int64_t n = N.n, np = N.n_pad;
    const int64_t lo = (int64_t)blockIdx.x * per;
    const int64_t cnt = max((int64_t)0, min(per, (int64_t)G * np - lo));
    const int64_t acc_base = (int64_t)b0 * np + lo;       // accumulator index of local pair 0
    float* V = reinterpret_cast<float*>(S.v);
    float* Gs = reinterpret_cast<float*>(S.g);

    // ---- load this CTA's state into shared memory ------------------------------------------
    for (int64_t k = tid; k < cnt; k += PT) {
        const int64_t lp = lo + k;
        const int32_t bl = (int32_t)(lp / np), i = (int32_t)(lp - (int64_t)bl * np);
        if (i < n) {
            const int64_t gp = (int64_t)(b0 + bl) * n + i;
            sv[k] = V[gp];
            sg[k] = Gs[gp];
            uint8_t f = (uint8_t)S.ref[gp];
            if (S.ext_idx[i] >= 0) f |= 0x80;
            if (PLASTIC && N.ppost_of[i] >= 0) f |= 0x40;
            sr[k] = f;
        }
    }
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) mbar_init(&mbar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int64_t nchunks = (cnt + SP - 1) / SP;
    uint32_t phase_bits = 0;          // parity of each stage's next completion
    unsigned int barriers = 0;
    int32_t* err = S.err;
    const int32_t nthreads_grid = gridDim.x * PT;
    const int64_t gtid = (int64_t)blockIdx.x * PT + tid;
    const int32_t words = A.words;

    for (int32_t s = 0; s < A.steps; s++) {
        const int64_t t = A.t0 + s;
        const uint32_t step_no = A.step0 + (uint32_t)s;
        if (tid < G) s_active[tid] = t < S.stop_tick[b0 + tid];
        if (blockIdx.x == 0 && tid == 0) *count_of(S, pos_mod(t - N.n_delay, N.R), q) = 0;
        __syncthreads();
        const AccT* acc = reinterpret_cast<const AccT*>((t & 1) ? S.acc1 : S.acc0);
        AccT* accw = const_cast<AccT*>(acc);
        const int64_t slot = pos_mod(t, N.R);

        // ---- U: advance every owned pair -----------------------------------------------------
        if (tid == 0) {
            fence_proxy_async_global();
            for (int64_t c = 0; c < min((int64_t)NSTAGE, nchunks); c++) {
                const uint32_t bytes = (uint32_t)(min((int64_t)SP, cnt - c * SP) * (int64_t)sizeof(AccT));
                mbar_expect_tx(&mbar[c], bytes);
                tma_load_1d(stage + c * SP, acc + acc_base + c * SP, bytes, &mbar[c]);
            }
        }
        int64_t lp = lo + tid;
        int32_t bl = (int32_t)(lp / np), i = (int32_t)(lp - (int64_t)bl * np);
        bool stop = false;
        for (int64_t c = 0; c < nchunks; c++) {
            const int st = (int)(c % NSTAGE);
            if (!stage_wait(&mbar[st], (phase_bits >> st) & 1u, A, err, s + 1)) { stop = true; }
            phase_bits ^= 1u << st;
            const AccT* sa = stage + st * SP;
#pragma unroll 2
            for (int m = 0; m < SP / PT; m++) {
                const int64_t k = c * SP + m * PT + tid;       // local pair
                int nch = 0;
                if (k < cnt && i < n && s_active[bl] && !stop) {
                    const int32_t b = b0 + bl;
                    const AccT x = sa[m * PT + tid];
                    if (x != 0) accw[acc_base + k] = 0;
                    float buf = acc_to_real<float>(x, L.w_syn);
                    const uint8_t f = sr[k];
                    if (PLASTIC && (f & 0x40)) buf = add_rn(buf, take_plastic<float>(N, S, t, b, i));
                    float v = sv[k], g = sg[k];
                    int r = f & 0x3f;
                    float bias = 0.0f;
                    bool kicked = false;
                    const bool ext = (f & 0x80) != 0;
                    const uint32_t tidh = (uint32_t)((int64_t)b * n + i);
                    if (ext) {
                        const int32_t j = S.ext_idx[i];
                        bias = S.bias_ext[(int64_t)b * S.n_ext + j];
                        kicked = kick_of<RASTER>(S, A.kicks, words, N.B, s, b, j, tidh, step_no);
                    }
                    const bool spk = lif_step<float>(v, g, r, buf, ext, bias, kicked, L, N.n_ref, N.contract != 0);
                    sv[k] = v;
                    sg[k] = g;
                    sr[k] = (uint8_t)((f & 0xc0) | r);
                    if (spk) {
                        A.counts[(int64_t)b * n + i] += 1;
                        const int64_t len = N.rowptr[i + 1] - N.rowptr[i];
                        nch = (int)((len + CHUNK - 1) / CHUNK);
                        if (PLASTIC) push_plastic_row(N, S, t, b, i);
                        if (RECORD) {
                            if (A.step_counts) atomicAdd(A.step_counts + (int64_t)s * N.B + b, 1);
                            if (A.step_digest)
                                atomicAdd(reinterpret_cast<unsigned long long*>(A.step_digest + (int64_t)s * N.B + b),
                                          (unsigned long long)spike_tag((uint64_t)i));
                        }
                    }
                }
                warp_append(S, slot, nch, i, b0 + bl);
                i += PT;
                while (i >= np) { i -= (int32_t)np; bl++; }
            }
            stop = __syncthreads_or(stop) != 0;                // stage st consumed by every thread
            if (tid == 0 && c + NSTAGE < nchunks && !stop) {
                fence_proxy_async_shared();
                const int64_t cn = c + NSTAGE;
                const uint32_t bytes = (uint32_t)(min((int64_t)SP, cnt - cn * SP) * (int64_t)sizeof(AccT));
                mbar_expect_tx(&mbar[st], bytes);
                tma_load_1d(stage + st * SP, acc + acc_base + cn * SP, bytes, &mbar[st]);
            }
        }
        if (stop) break;

        // ---- P: scatter the spikes that arrive at t+1 ----------------------------------------
        if (N.n_delay == 1) {
            barriers++;
            if (grid_barrier(A, barriers * gridDim.x, err, s + 1)) break;
        }
        AccT* acc_next = reinterpret_cast<AccT*>(((t + 1) & 1) ? S.acc1 : S.acc0);
        push_list<AccT, LANES>(N, S, t, q, acc_next, gtid, nthreads_grid);
        barriers++;
        if (grid_barrier(A, barriers * gridDim.x, err, s + 1)) break;
    }

    // ---- write the state back ------------------------------------------------------------------
    __syncthreads();
    for (int64_t k = tid; k < cnt; k += PT) {
        const int64_t lp2 = lo + k;
        const int32_t bl2 = (int32_t)(lp2 / np), i2 = (int32_t)(lp2 - (int64_t)bl2 * np);
        if (i2 < n) {
            const int64_t gp = (int64_t)(b0 + bl2) * n + i2;
            V[gp] = sv[k];
            Gs[gp] = sg[k];
            S.ref[gp] = (int8_t)(sr[k] & 0x3f);
        }
    }
}

// Largest group whose state fits in shared memory of `ctas` CTAs; 0 if not even one instance does.
inline PersistPlan plan_persistent(int64_t n, int64_t n_pad, int32_t B, bool f64, int n_ref, int acc_bytes,
                                   int sm_count, int device)
{
    PersistPlan P{};
    if (f64 || n_ref > 63) return P;
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (smem_optin <= 0) smem_optin = 232448;
    const int64_t fixed = NSTAGE * STAGE_BYTES + NSTAGE * 8 + 64 /* group flags */ + 256;
    const int64_t per_max = ((smem_optin - fixed) / 9) / 16 * 16;
    if (per_max <= 0) return P;
    const int ctas = sm_count;
    int64_t gmax = (int64_t)ctas * per_max / n_pad;
    gmax = std::min<int64_t>(gmax, 64);
    if (gmax < 1) return P;
    const int32_t n_groups = (int32_t)((B + gmax - 1) / gmax);
    const int32_t G = (B + n_groups - 1) / n_groups;
    int64_t per = ((int64_t)G * n_pad + ctas - 1) / ctas;
    per = (per + 15) / 16 * 16;
    if (per > per_max) return P;
    P.group = G;
    P.n_groups = n_groups;
    P.ctas = ctas;
    P.per = per;
    P.smem = (size_t)(fixed + per * 9);
    P.launches_per_run = n_groups;
    (void)n; (void)acc_bytes;
    return P;
}

template <typename AccT, bool RASTER, bool PLASTIC, bool RECORD, int LANES>
cudaError_t launch_persist_one(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                               cudaStream_t st)
{
    auto kern = k_persist<AccT, RASTER, PLASTIC, RECORD, LANES>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem);
    if (e != cudaSuccess) return e;
    for (int32_t q = 0; q < P.n_groups; q++) {
        const int32_t b0 = q * P.group;
        const int32_t G = std::min<int32_t>(P.group, N.B - b0);
        e = cudaMemsetAsync(A.bar, 0, sizeof(unsigned int), st);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(P.ctas);
        cfg.blockDim = dim3(PT);
        cfg.dynamicSmemBytes = P.smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, kern, N, S, A, b0, G, q, P.per);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename AccT, bool RASTER, bool PLASTIC, bool RECORD>
cudaError_t launch_persist_lanes(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                                 int lanes, cudaStream_t st)
{
    if (lanes == 8) return launch_persist_one<AccT, RASTER, PLASTIC, RECORD, 8>(P, N, S, A, st);
    if (lanes == 16) return launch_persist_one<AccT, RASTER, PLASTIC, RECORD, 16>(P, N, S, A, st);
    return launch_persist_one<AccT, RASTER, PLASTIC, RECORD, 32>(P, N, S, A, st);
}

template <typename AccT>
cudaError_t launch_persist_acc(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                               bool plastic, bool raster, bool record, int lanes, cudaStream_t st)
{
#define LP_(R_, P_, C_) return launch_persist_lanes<AccT, R_, P_, C_>(P, N, S, A, lanes, st)
    if (raster) {
        if (plastic) { if (record) LP_(true, true, true); LP_(true, true, false); }
        if (record) LP_(true, false, true);
        LP_(true, false, false);
    }
    if (plastic) { if (record) LP_(false, true, true); LP_(false, true, false); }
    if (record) LP_(false, false, true);
    LP_(false, false, false);
#undef LP_
}

inline cudaError_t launch_persistent(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                                     int acc_mode, bool plastic, bool raster, bool record, int lanes, cudaStream_t st)
{
    if (acc_mode == 0) return launch_persist_acc<int32_t>(P, N, S, A, plastic, raster, record, lanes, st);
    return launch_persist_acc<int64_t>(P, N, S, A, plastic, raster, record, lanes, st);
}

}  // namespace fb
